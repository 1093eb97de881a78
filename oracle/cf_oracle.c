/*
 * cf_oracle.c -- CPU restatement of Cosmic-Fields-Lite's lattice time-stepping
 * hot path, in plain C, FP64.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity checker: only tests/, the smoke
 * check and bench.py's CPU-baseline leg load the library built from this file
 * (oracle/liboracle.so).  The product (libcfb200.so) never links or calls it.
 *
 * Each function cites the reference file:line it restates.  Arithmetic follows
 * the reference's operation order where that is cheap to keep, so the restatement
 * agrees with the reference build (oracle/_ref) to rounding; the parity tests
 * check that agreement and pin both against the reference's published outputs
 * (output/Growth_and_FS/*_0.dat).
 *
 * Layout conventions (reference src/fdm3d.hpp:16,24):
 *   state  : 2N^3 doubles [phi | dphi], site (a,b,c) at N*N*a + N*b + c;
 *   HC     : half-complex 2*N*N*(N/2+1) doubles, mode (a,b,c<=N/2) at
 *            2*(N*(N/2+1)*a + (N/2+1)*b + c) (real, imag);
 *   S2 bins: 3*(N/2)^2+1 doubles indexed by s^2 = i^2+j^2+k^2.
 *
 * Equation codes: 0 = KleinGordonEquation (flat), 1 = KleinGordonEquationInFRW,
 * 2 = ComovingCurvatureEquationInFRW, and the GPU-only functors of
 * src/equations_cuda.cu (no CPU twin in the reference; restated from the CUDA
 * kernels and pinned against the reference's own GPU build, tests/golden/):
 * 3 = CudaLambdaEquationInFRW, 4 = CudaSqrtPotentialEquationInFRW,
 * 5 = CudaFixedCurvatureEquationInFRW, 6 = CudaApproximateComovingCurvatureEquationInFRW.
 * Stencil: 7 (reference) or 13 (fourth order; no reference counterpart,
 * restated from the standard 5-point second-derivative formula per axis).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"

#define IDX(N, a, b, c) ((N) * (N) * (a) + (N) * (b) + (c))

static const double CFO_PI = 3.14159265358979323846;

typedef struct {
  int64_t N;
  double L, m;
  double a1, H1, t1, p; /* StaticEOSCosmology, src/physics.hpp:15-56 */
  int eq;
  int stencil;
  double lambda;          /* eq 3: quartic coupling (workspace.lambda) */
  double f_a;             /* eq 4: sqrt-potential scale (workspace.f_a) */
  int64_t M;              /* eq 6: coarse grid (workspace.M) */
  const double *Psi_fixed; /* eq 5: the fixed Psi(x), N^3 (workspace.Psi) */
} cfo_params;

/* ---- cosmology: src/physics.hpp:34-55 ---------------------------------- */
double cfo_a(const cfo_params *P, double t) {
  return P->a1 * pow(1 + (1 + 1 / P->p) * P->H1 * (t - P->t1), P->p / (1 + P->p));
}
double cfo_H(const cfo_params *P, double t) {
  return P->H1 * pow(1 + (1 + 1 / P->p) * P->H1 * (t - P->t1), -1);
}
double cfo_eta(const cfo_params *P, double t) {
  return (P->p / (P->a1 * P->H1)) * pow(1 + (1 + 1 / P->p) * P->H1 * (t - P->t1), 1 / (1 + P->p));
}

/* ---- Psi / dPsi/dt transfer functions: src/equations.cpp:141-183 --------- */
void cfo_psi_dpsidt_fft(int64_t N, const double *R_fft, double *Psi_fft, double *dPsidt_fft,
                        double factor, double H_t) {
  const int64_t nh = N / 2 + 1;
#pragma omp parallel for schedule(static)
  for (int64_t a = 0; a < N; ++a)
    for (int64_t b = 0; b < N; ++b)
      for (int64_t c = 0; c < nh; ++c) {
        int64_t as = (a <= N / 2) ? a : (N - a);
        int64_t bs = (b <= N / 2) ? b : (N - b);
        int64_t s2 = as * as + bs * bs + c * c;
        int64_t o = 2 * (N * nh * a + nh * b + c);
        if (s2 == 0) {
          Psi_fft[o] = Psi_fft[o + 1] = 0;
          if (dPsidt_fft) dPsidt_fft[o] = dPsidt_fft[o + 1] = 0;
          continue;
        }
        double x = sqrt((double)s2) * factor;
        double sv = sin(x), cv = cos(x);
        double common = 2.0 / (x * x * x) / (double)(N * N * N);
        double tp = (sv - x * cv) * common;
        Psi_fft[o] = R_fft[o] * tp;
        Psi_fft[o + 1] = R_fft[o + 1] * tp;
        if (dPsidt_fft) {
          double td = H_t * (3 * x * cv + (x * x - 3.0) * sv) * common;
          dPsidt_fft[o] = R_fft[o] * td;
          dPsidt_fft[o + 1] = R_fft[o + 1] * td;
        }
      }
}

/* Psi(x,t) and (optionally) dPsi/dt(x,t) on the lattice, N^3 each.  The
 * reference computes them with FFTW c2r into dense arrays
 * (src/equations.cpp:215-233 via fftwWrapper::execute_z2d). */
void cfo_psi_fields(const cfo_params *P, const double *R_fft, double t, double *Psi, double *dPsidt) {
  const int64_t N = P->N;
  const size_t hc = (size_t)(2 * N * N * (N / 2 + 1));
  double eta_t = cfo_eta(P, t), H_t = cfo_H(P, t);
  double factor = (2 * CFO_PI / P->L) * eta_t / sqrt(3);
  double *pf = (double *)malloc(sizeof(double) * hc);
  double *df = dPsidt ? (double *)malloc(sizeof(double) * hc) : NULL;
  cfo_psi_dpsidt_fft(N, R_fft, pf, df, factor, H_t);
  fftw_plan pl = fftw_plan_dft_c2r_3d((int)N, (int)N, (int)N, (fftw_complex *)pf, Psi, FFTW_ESTIMATE);
  fftw_execute_dft_c2r(pl, (fftw_complex *)pf, Psi);
  if (dPsidt) fftw_execute_dft_c2r(pl, (fftw_complex *)df, dPsidt);
  fftw_destroy_plan(pl);
  free(pf);
  free(df);
}

/* eq 6: Psi and dPsi/dt on the coarse M^3 grid at t
 * (CudaApproximateComovingCurvatureEquationInFRW::operator(), src/equations_cuda.cu:764-809):
 * the modes of R_fft kept by compute_cutoff_fouriers (src/fdm3d_cuda.cu:118-141,
 * :206-219: M-grid mode a < M/2 from a, a >= M/2 from N-(M-a), same for b, c from c,
 * times 1/(N/M)^3), the comoving transfer functions at lattice size M
 * (src/equations_cuda.cu:209-259) and a 3-D c2r of size M.  Dense M^3 outputs. */
void cfo_approx_fields(const cfo_params *P, const double *R_fft, double t, double *Psi, double *dPsidt) {
  const int64_t N = P->N, M = P->M, nhN = N / 2 + 1, nhM = M / 2 + 1;
  const size_t hcM = (size_t)(2 * M * M * nhM);
  double *cut = (double *)malloc(sizeof(double) * hcM);
  double *pf = (double *)malloc(sizeof(double) * hcM);
  double *df = (double *)malloc(sizeof(double) * hcM);
  const double scale_diff = (double)N / (double)M;
  const double scaling = 1.0 / (scale_diff * scale_diff * scale_diff);
  for (int64_t a = 0; a < M; ++a)
    for (int64_t b = 0; b < M; ++b)
      for (int64_t c = 0; c < nhM; ++c) {
        int64_t aN = (a < M / 2) ? a : (N - (M - a));
        int64_t bN = (b < M / 2) ? b : (N - (M - b));
        int64_t oM = 2 * (M * nhM * a + nhM * b + c), oN = 2 * (N * nhN * aN + nhN * bN + c);
        cut[oM] = R_fft[oN] * scaling;
        cut[oM + 1] = R_fft[oN + 1] * scaling;
      }
  double eta_t = cfo_eta(P, t), H_t = cfo_H(P, t);
  double factor = (2 * CFO_PI / P->L) * eta_t / sqrt(3);
  cfo_psi_dpsidt_fft(M, cut, pf, df, factor, H_t);
  fftw_plan pl = fftw_plan_dft_c2r_3d((int)M, (int)M, (int)M, (fftw_complex *)pf, Psi, FFTW_ESTIMATE);
  fftw_execute_dft_c2r(pl, (fftw_complex *)pf, Psi);
  fftw_execute_dft_c2r(pl, (fftw_complex *)df, dPsidt);
  fftw_destroy_plan(pl);
  free(cut);
  free(pf);
  free(df);
}

/* Lattice Laplacian times h^2 at site (a,b,c): 7-point (reference
 * src/equations.cpp:94-101 summation order) or 13-point fourth order. */
static inline double lap_h2(const double *f, int64_t N, int64_t a, int64_t b, int64_t c, int stencil) {
  int64_t ap = (a + 1) % N, am = (a + N - 1) % N, bp = (b + 1) % N, bm = (b + N - 1) % N;
  int64_t cp = (c + 1) % N, cm = (c + N - 1) % N;
  double f0 = f[IDX(N, a, b, c)];
  if (stencil != 13) {
    double s = -6.0 * f0 + f[IDX(N, ap, b, c)] + f[IDX(N, am, b, c)] + f[IDX(N, a, bp, c)] +
               f[IDX(N, a, bm, c)];
    return s + (f[IDX(N, a, b, cp)] + f[IDX(N, a, b, cm)]);
  }
  int64_t a2p = (a + 2) % N, a2m = (a + 2 * N - 2) % N, b2p = (b + 2) % N, b2m = (b + 2 * N - 2) % N;
  int64_t c2p = (c + 2) % N, c2m = (c + 2 * N - 2) % N;
  double s1 = f[IDX(N, ap, b, c)] + f[IDX(N, am, b, c)] + f[IDX(N, a, bp, c)] + f[IDX(N, a, bm, c)] +
              f[IDX(N, a, b, cp)] + f[IDX(N, a, b, cm)];
  double s2 = f[IDX(N, a2p, b, c)] + f[IDX(N, a2m, b, c)] + f[IDX(N, a, b2p, c)] +
              f[IDX(N, a, b2m, c)] + f[IDX(N, a, b, c2p)] + f[IDX(N, a, b, c2m)];
  return (16.0 * s1 - s2 - 90.0 * f0) / 12.0;
}

/* dxdt = Equation(x, t).
 *   eq 0: src/equations.cpp:8-36   dphi' = -m^2 phi + h^-2 lap phi
 *   eq 1: src/equations.cpp:71-104 dphi' = -3H dphi - m^2 phi + a^-2 h^-2 lap phi
 *   eq 2: src/equations.cpp:186-261
 *         dphi' = (-3H + 4 dPsi/dt) dphi - e^{2Psi} m^2 phi + e^{4Psi} a^-2 h^-2 lap phi
 *   eq 3: src/equations_cuda.cu:38-76   ... - m^2 phi - lambda phi^3 + ...
 *   eq 4: src/equations_cuda.cu:84-104  ... - m^2 phi / sqrt(1 + phi^2 / f_a^2) + ...
 *   eq 5: src/equations_cuda.cu:112-136 eq 2's form with the fixed Psi and dPsi/dt = 0
 *   eq 6: src/equations_cuda.cu:299-329 with the coarse fields of cfo_approx_fields,
 *         sampled at coarse site ((a + s/2) % N) / s per axis, s = N/M, and
 *         e^{2Psi} -> 1 + 2Psi + 2Psi^2, e^{4Psi} -> 1 + 4Psi + 8Psi^2
 * R_fft is used for eq 2 and 6 only. */
void cfo_rhs(const cfo_params *P, const double *x, const double *R_fft, double t, double *dxdt) {
  const int64_t N = P->N, N3 = N * N * N;
  const double m = P->m;
  const double h = P->L / N;
  double inv, H_t = 0;
  if (P->eq == 0) {
    inv = 1.0 / (h * h);
  } else {
    double a_t = cfo_a(P, t);
    H_t = cfo_H(P, t);
    inv = 1.0 / (h * h) / (a_t * a_t);
  }
  double *Psi = NULL, *dPsi = NULL;
  if (P->eq == 2) {
    Psi = (double *)malloc(sizeof(double) * N3);
    dPsi = (double *)malloc(sizeof(double) * N3);
    cfo_psi_fields(P, R_fft, t, Psi, dPsi);
  }
  int64_t M = P->M, sd = 1, hs = 0;
  if (P->eq == 6) {
    Psi = (double *)malloc(sizeof(double) * M * M * M);
    dPsi = (double *)malloc(sizeof(double) * M * M * M);
    cfo_approx_fields(P, R_fft, t, Psi, dPsi);
    sd = N / M;
    hs = sd / 2;
  }
  const double *phi = x, *pi = x + N3;
  /* sites are independent: the a-planes are spread over OpenMP threads (same bits) */
#pragma omp parallel for schedule(static)
  for (int64_t a = 0; a < N; ++a)
    for (int64_t b = 0; b < N; ++b)
      for (int64_t c = 0; c < N; ++c) {
        int64_t i = IDX(N, a, b, c);
        double lap = lap_h2(phi, N, a, b, c, P->stencil);
        double f = phi[i];
        dxdt[i] = pi[i];
        switch (P->eq) {
          case 0:
            dxdt[N3 + i] = (-1.0) * m * m * f + inv * lap;
            break;
          case 1:
            dxdt[N3 + i] = (-3.0) * H_t * pi[i] - m * m * f + inv * lap;
            break;
          case 2:
            dxdt[N3 + i] = (-3.0 * H_t + 4.0 * dPsi[i]) * pi[i] - exp(2 * Psi[i]) * m * m * f +
                           exp(4 * Psi[i]) * inv * lap;
            break;
          case 3:
            dxdt[N3 + i] = (-3.0) * H_t * pi[i] - m * m * f - P->lambda * f * f * f + inv * lap;
            break;
          case 4:
            dxdt[N3 + i] = (-3.0) * H_t * pi[i] - m * m * f / sqrt(1.0 + f * f / (P->f_a * P->f_a)) + inv * lap;
            break;
          case 5: {
            double ps = P->Psi_fixed[i];
            dxdt[N3 + i] = (-3.0) * H_t * pi[i] - exp(2 * ps) * m * m * f + exp(4 * ps) * inv * lap;
            break;
          }
          default: { /* 6 */
            int64_t j = IDX(M, ((a + hs) % N) / sd, ((b + hs) % N) / sd, ((c + hs) % N) / sd);
            double ps = Psi[j];
            dxdt[N3 + i] = (-3.0 * H_t + 4.0 * dPsi[j]) * pi[i] - (1 + 2.0 * ps + 2.0 * ps * ps) * m * m * f +
                           (1 + 4.0 * ps + 8.0 * ps * ps) * inv * lap;
            break;
          }
        }
      }
  free(Psi);
  free(dPsi);
}

/* One classic RK4 step in place, exactly the stage structure of
 * boost/numeric/odeint/stepper/runge_kutta4_classic.hpp:88-138 with the
 * Eigen scale_sum2 / scale_sum5 of src/odeint_eigen/eigen_operations.hpp:33-101:
 *   k1 = f(x,t); y = x + dt/2 k1; k2 = f(y, t+dt/2); y = x + dt/2 k2;
 *   k3 = f(y, t+dt/2); y = x + dt k3; k4 = f(y, t+dt);
 *   x = x + dt/6 k1 + dt/3 k2 + dt/3 k3 + dt/6 k4. */
void cfo_rk4_step(const cfo_params *P, double *x, const double *R_fft, double t, double dt) {
  const size_t n = (size_t)(2 * P->N * P->N * P->N);
  double *k1 = (double *)malloc(sizeof(double) * n * 5);
  double *k2 = k1 + n, *k3 = k2 + n, *k4 = k3 + n, *y = k4 + n;
  const double dh = dt / 2.0, th = t + dh;
  cfo_rhs(P, x, R_fft, t, k1);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; ++i) y[i] = 1.0 * x[i] + dh * k1[i];
  cfo_rhs(P, y, R_fft, th, k2);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; ++i) y[i] = 1.0 * x[i] + dh * k2[i];
  cfo_rhs(P, y, R_fft, th, k3);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; ++i) y[i] = 1.0 * x[i] + dt * k3[i];
  cfo_rhs(P, y, R_fft, t + dt, k4);
  const double dt6 = dt / 6.0, dt3 = dt / 3.0;
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; ++i)
    x[i] = 1.0 * x[i] + dt6 * k1[i] + dt3 * k2[i] + dt3 * k3[i] + dt6 * k4[i];
  free(k1);
}

/* `nsteps` steps of integrate_const's loop body
 * (integrate/detail/integrate_const.hpp:55-64): step j runs at
 * t = t0 + (step0 + j) * dt (direct, not accumulated). */
void cfo_rk4_steps(const cfo_params *P, double *x, const double *R_fft, double t0, double dt,
                   int64_t step0, int64_t nsteps) {
  for (int64_t j = 0; j < nsteps; ++j) {
    double t = t0 + (double)(step0 + j) * dt;
    cfo_rk4_step(P, x, R_fft, t, dt);
  }
}

/* Energy density rho (N^3):
 *   eq 0: src/equations.cpp:38-69, eq 1: :106-138 (inv = h^-2 a^-2),
 *   eq 2 and 6: :265-322 (e^{-2Psi} kinetic, e^{2Psi} gradient weights; the
 *   approximate equation reports the full comoving density, src/equations_cuda.cu:812-815),
 *   rho = 1/2 dphi^2 + 1/2 m^2 phi^2 + 1/8 inv sum_axes (phi_{+1}-phi_{-1})^2;
 *   eq 3: src/equations_cuda.cu:332-369 (+ 1/4 lambda phi^4),
 *   eq 4: :431-449 (potential m^2 f_a^2 (sqrt(1 + phi^2/f_a^2) - 1)),
 *   eq 5: :451-473 with the fixed Psi. */
void cfo_energy_density(const cfo_params *P, const double *x, const double *R_fft, double t, double *rho) {
  const int64_t N = P->N, N3 = N * N * N;
  const double m = P->m, h = P->L / N;
  double inv = 1.0 / (h * h);
  if (P->eq != 0) {
    double a_t = cfo_a(P, t);
    inv = inv / (a_t * a_t);
  }
  double *Psi = NULL;
  if (P->eq == 2 || P->eq == 6) {
    Psi = (double *)malloc(sizeof(double) * N3);
    cfo_psi_fields(P, R_fft, t, Psi, NULL);
  }
  const double *phi = x, *pi = x + N3;
#pragma omp parallel for schedule(static)
  for (int64_t a = 0; a < N; ++a)
    for (int64_t b = 0; b < N; ++b)
      for (int64_t c = 0; c < N; ++c) {
        int64_t i = IDX(N, a, b, c);
        double dx = phi[IDX(N, (a + 1) % N, b, c)] - phi[IDX(N, (a + N - 1) % N, b, c)];
        double dy = phi[IDX(N, a, (b + 1) % N, c)] - phi[IDX(N, a, (b + N - 1) % N, c)];
        double dz = phi[IDX(N, a, b, (c + 1) % N)] - phi[IDX(N, a, b, (c + N - 1) % N)];
        double grad = dx * dx + dy * dy + dz * dz;
        double f = phi[i];
        switch (P->eq) {
          case 2:
          case 6:
            rho[i] = 0.5 * (exp(-2 * Psi[i]) * pi[i] * pi[i] + m * m * f * f + exp(2 * Psi[i]) * 0.25 * inv * grad);
            break;
          case 3:
            rho[i] = 0.5 * pi[i] * pi[i] + (0.5 / 4.0) * inv * grad + 0.5 * m * m * f * f +
                     0.25 * P->lambda * f * f * f * f;
            break;
          case 4:
            rho[i] = 0.5 * pi[i] * pi[i] + (0.5 / 4.0) * inv * grad +
                     m * m * P->f_a * P->f_a * (sqrt(1.0 + f * f / (P->f_a * P->f_a)) - 1.0);
            break;
          case 5: {
            double ps = P->Psi_fixed[i];
            rho[i] = exp(-2 * ps) * 0.5 * pi[i] * pi[i] + exp(2 * ps) * (0.5 / 4.0) * inv * grad + 0.5 * m * m * f * f;
            break;
          }
          default:
            rho[i] = 0.5 * (pi[i] * pi[i] + m * m * f * f + 0.25 * inv * grad);
        }
      }
  free(Psi);
}

/* d rho / dt of KleinGordonEquationInFRW
 * (CudaKleinGordonEquationInFRW::compute_dot_energy_density, src/equations_cuda.cu:372-424,
 * :556-572): dphi lap_inv + 1/4 inv sum_e (dphi_{+e} - dphi_{-e})(phi_{+e} - phi_{-e})
 * - 3H (rho + p), rho = 1/2 dphi^2 + 1/8 inv G + 1/2 m^2 phi^2,
 * p = 1/2 dphi^2 - 1/2 m^2 phi^2 - 1/24 inv G, G = sum_e (phi_{+e} - phi_{-e})^2. */
void cfo_dot_energy_density(const cfo_params *P, const double *x, double t, double *out) {
  const int64_t N = P->N, N3 = N * N * N;
  const double m = P->m, h = P->L / N;
  const double a_t = cfo_a(P, t), H_t = cfo_H(P, t);
  const double inv = 1.0 / (h * h) / (a_t * a_t);
  const double *phi = x, *pi = x + N3;
  for (int64_t a = 0; a < N; ++a)
    for (int64_t b = 0; b < N; ++b)
      for (int64_t c = 0; c < N; ++c) {
        int64_t i = IDX(N, a, b, c);
        int64_t ap = IDX(N, (a + 1) % N, b, c), am = IDX(N, (a + N - 1) % N, b, c);
        int64_t bp = IDX(N, a, (b + 1) % N, c), bm = IDX(N, a, (b + N - 1) % N, c);
        int64_t cp = IDX(N, a, b, (c + 1) % N), cm = IDX(N, a, b, (c + N - 1) % N);
        double f = phi[i];
        double dx = phi[ap] - phi[am], dy = phi[bp] - phi[bm], dz = phi[cp] - phi[cm];
        double ex = pi[ap] - pi[am], ey = pi[bp] - pi[bm], ez = pi[cp] - pi[cm];
        double lap = inv * (-6.0 * f + phi[ap] + phi[am] + phi[bp] + phi[bm] + phi[cp] + phi[cm]);
        double G = dx * dx + dy * dy + dz * dz;
        double rho = 0.5 * pi[i] * pi[i] + (0.5 / 4.0) * inv * G + 0.5 * m * m * f * f;
        double p = 0.5 * pi[i] * pi[i] - 0.5 * m * m * f * f - (1.0 / 4.0 / 6.0) * inv * G;
        double vt = pi[i] * lap + (1.0 / 4.0) * inv * (ex * dx + ey * dy + ez * dz);
        out[i] = vt - 3.0 * H_t * (rho + p);
      }
}

/* r2c of one N^3 field into HC (fftwWrapper::execute_d2z, src/fftw_wrapper.cpp:24-34). */
void cfo_d2z(int64_t N, const double *f, double *hc) {
  fftw_plan pl = fftw_plan_dft_r2c_3d((int)N, (int)N, (int)N, (double *)f, (fftw_complex *)hc, FFTW_ESTIMATE);
  fftw_execute_dft_r2c(pl, (double *)f, (fftw_complex *)hc);
  fftw_destroy_plan(pl);
}

/* out[s^2] = sum over all N^3 modes |f_k|^2 (src/fdm3d.cpp:7-34); length 3(N/2)^2+1. */
void cfo_power_spectrum(int64_t N, const double *f, double *out) {
  const int64_t nh = N / 2 + 1, nb = 3 * (N / 2) * (N / 2) + 1;
  double *hc = (double *)malloc(sizeof(double) * 2 * N * N * nh);
  cfo_d2z(N, f, hc);
  memset(out, 0, sizeof(double) * nb);
  for (int64_t a = 0; a < N; ++a)
    for (int64_t b = 0; b < N; ++b)
      for (int64_t c = 0; c < N; ++c) {
        int64_t as = (a <= N / 2) ? a : (N - a), bs = (b <= N / 2) ? b : (N - b), cs = (c <= N / 2) ? c : (N - c);
        int64_t s2 = as * as + bs * bs + cs * cs;
        int64_t o = 2 * (N * nh * a + nh * b + cs);
        out[s2] += hc[o] * hc[o] + hc[o + 1] * hc[o + 1];
      }
  free(hc);
}

/* out[s^2] = sum |phi_k|^2 + |dphi_k|^2 / (m^2 + (2 pi/L)^2 s^2 / a^2)
 * (src/fdm3d.cpp:36-72). */
void cfo_mode_power_spectrum(int64_t N, double L, double m, double a_t, const double *state, double *out) {
  const int64_t nh = N / 2 + 1, nb = 3 * (N / 2) * (N / 2) + 1, N3 = N * N * N;
  double *h1 = (double *)malloc(sizeof(double) * 4 * N * N * nh);
  double *h2 = h1 + 2 * N * N * nh;
  cfo_d2z(N, state, h1);
  cfo_d2z(N, state + N3, h2);
  memset(out, 0, sizeof(double) * nb);
  for (int64_t a = 0; a < N; ++a)
    for (int64_t b = 0; b < N; ++b)
      for (int64_t c = 0; c < N; ++c) {
        int64_t as = (a <= N / 2) ? a : (N - a), bs = (b <= N / 2) ? b : (N - b), cs = (c <= N / 2) ? c : (N - c);
        int64_t s2 = as * as + bs * bs + cs * cs;
        int64_t o = 2 * (N * nh * a + nh * b + cs);
        out[s2] += h1[o] * h1[o] + h1[o + 1] * h1[o + 1] +
                   (h2[o] * h2[o] + h2[o + 1] * h2[o + 1]) /
                       (m * m + (2 * CFO_PI / L) * (2 * CFO_PI / L) * s2 / (a_t * a_t));
      }
  free(h1);
}

/* Mode multiplicity per s^2 over the lattice momenta -N/2+1..N/2 on each axis
 * (the rule of plot_util.py:53-58), exact integers. */
void cfo_s2_counts(int64_t N, int64_t *counts) {
  const int64_t nb = 3 * (N / 2) * (N / 2) + 1;
  memset(counts, 0, sizeof(int64_t) * nb);
  for (int64_t a = 0; a < N; ++a)
    for (int64_t b = 0; b < N; ++b)
      for (int64_t c = 0; c < N; ++c) {
        int64_t as = (a <= N / 2) ? a : (N - a), bs = (b <= N / 2) ? b : (N - b), cs = (c <= N / 2) ? c : (N - c);
        counts[as * as + bs * bs + cs * cs] += 1;
      }
}

/* Integer square root floor(sqrt(s2)). */
int64_t cfo_isqrt(int64_t s2) {
  int64_t r = (int64_t)sqrt((double)s2);
  while (r * r > s2) --r;
  while ((r + 1) * (r + 1) <= s2) ++r;
  return r;
}

/* Unit-width |k| shells (no reference counterpart): shell i collects the S2
 * bins s^2 in [i^2, (i+1)^2).  nshell = isqrt(3(N/2)^2)+1.  Sums are accumulated
 * in s^2 order in long double, then rounded once. */
void cfo_shells_from_s2(int64_t N, const double *s2bins, const int64_t *s2counts, double *shells,
                        int64_t *shell_counts) {
  const int64_t nb = 3 * (N / 2) * (N / 2) + 1;
  const int64_t ns = cfo_isqrt(nb - 1) + 1;
  long double *acc = (long double *)calloc((size_t)ns, sizeof(long double));
  if (shell_counts) memset(shell_counts, 0, sizeof(int64_t) * ns);
  for (int64_t s = 0; s < nb; ++s) {
    int64_t i = cfo_isqrt(s);
    if (s2bins) acc[i] += s2bins[s];
    if (shell_counts) shell_counts[i] += s2counts[s];
  }
  if (shells)
    for (int64_t i = 0; i < ns; ++i) shells[i] = (double)acc[i];
  free(acc);
}

/* ---- seeded inputs as the reference makes them ---------------------------
 * std::mt19937 (Matsumoto & Nishimura 1998) and libstdc++'s
 * std::normal_distribution (Marsaglia polar method, one cached deviate, uniform
 * deviates from generate_canonical<double,53> = two 32-bit draws / 2^64), as
 * used by RandomNormal (src/random_field.cpp:13-33). */
typedef struct {
  uint32_t mt[624];
  int idx;
  int have_saved;
  double saved;
} cfo_rng;

void cfo_rng_seed(cfo_rng *r, uint32_t seed) {
  r->mt[0] = seed;
  for (int i = 1; i < 624; ++i) r->mt[i] = 1812433253u * (r->mt[i - 1] ^ (r->mt[i - 1] >> 30)) + (uint32_t)i;
  r->idx = 624;
  r->have_saved = 0;
}

static uint32_t mt_next(cfo_rng *r) {
  if (r->idx >= 624) {
    for (int i = 0; i < 624; ++i) {
      uint32_t y = (r->mt[i] & 0x80000000u) | (r->mt[(i + 1) % 624] & 0x7fffffffu);
      uint32_t v = r->mt[(i + 397) % 624] ^ (y >> 1);
      if (y & 1u) v ^= 0x9908b0dfu;
      r->mt[i] = v;
    }
    r->idx = 0;
  }
  uint32_t y = r->mt[r->idx++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

static double canonical53(cfo_rng *r) {
  double lo = (double)mt_next(r);
  double hi = (double)mt_next(r);
  double v = (lo + hi * 4294967296.0) / 18446744073709551616.0;
  if (v >= 1.0) v = nextafter(1.0, 0.0);
  return v;
}

double cfo_rng_normal(cfo_rng *r) {
  if (r->have_saved) {
    r->have_saved = 0;
    return r->saved;
  }
  double x, y, r2;
  do {
    x = 2.0 * canonical53(r) - 1.0;
    y = 2.0 * canonical53(r) - 1.0;
    r2 = x * x + y * y;
  } while (r2 > 1.0 || r2 == 0.0);
  double mult = sqrt(-2 * log(r2) / r2);
  r->saved = x * mult;
  r->have_saved = 1;
  return y * mult;
}

size_t cfo_rng_size(void) { return sizeof(cfo_rng); }

/* Spectrum callback P(k) for the Gaussian random field. */
typedef double (*cfo_spectrum_fn)(double k, const double *args);

/* generate_inhomogeneous_gaussian_random_field (src/random_field.cpp:36-83):
 * white noise / N^3, times exp(Psi) (Psi may be NULL = 0, scaled by psi_scale),
 * r2c, times sqrt(P(|k|)) per half-complex mode, unnormalised c2r. */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as
 * 1, 2, 3", SC'11): the counter-based generator behind the product's device white
 * noise (no reference counterpart).  Ten rounds of two 32x32->64 multiplies by
 * 0xD2511F53 / 0xCD9E8D57 with the Weyl key schedule 0x9E3779B9 / 0xBB67AE85. */
void cfo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n1 = (uint32_t)p1, n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1,
             n3 = (uint32_t)p0;
    c0 = n0, c1 = n1, c2 = n2, c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0, out[1] = c1, out[2] = c2, out[3] = c3;
}

/* The product's device deviates (cf_white_noise): element g of stream `seed` is deviate
 * g % 2 of counter g / 2 -- uniforms u1 = (x0:x1 >> 11 + 1/2) 2^-53, u2 = (x2:x3 >> 11) 2^-53,
 * Box-Muller sqrt(-2 ln u1) (cos 2 pi u2, sin 2 pi u2). */
void cfo_white_noise(uint64_t seed, uint64_t offset, int64_t n, double *out) {
  for (int64_t i = 0; i < n; ++i) {
    uint64_t g = offset + (uint64_t)i, ctr = g >> 1;
    uint32_t c[4] = {(uint32_t)ctr, (uint32_t)(ctr >> 32), 0, 0}, k[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)}, x[4];
    cfo_philox4x32_10(c, k, x);
    uint64_t a = (((uint64_t)x[0] << 32) | x[1]) >> 11, b = (((uint64_t)x[2] << 32) | x[3]) >> 11;
    double u1 = ((double)a + 0.5) * 0x1.0p-53, u2 = (double)b * 0x1.0p-53;
    double rad = sqrt(-2.0 * log(u1));
    out[i] = (g & 1) ? rad * sin(2 * CFO_PI * u2) : rad * cos(2 * CFO_PI * u2);
  }
}

/* n consecutive deviates of the stream (RandomNormal::generate_random_normal, src/random_field.cpp:28-31). */
void cfo_rng_fill(cfo_rng *r, double *out, int64_t n) {
  for (int64_t i = 0; i < n; ++i) out[i] = cfo_rng_normal(r);
}

static void grf_core(int64_t N, double L, const double *Psi, double psi_scale, cfo_spectrum_fn P, const double *args,
                     double *out);

void cfo_grf(cfo_rng *r, int64_t N, double L, const double *Psi, double psi_scale, cfo_spectrum_fn P,
             const double *args, double *out) {
  const int64_t N3 = N * N * N;
  for (int64_t i = 0; i < N3; ++i) out[i] = (1.0 / (double)N3) * cfo_rng_normal(r);
  grf_core(N, L, Psi, psi_scale, P, args, out);
}

/* The same field from given deviates `white` (N^3) instead of the stream. */
void cfo_grf_white(int64_t N, double L, const double *white, const double *Psi, double psi_scale, int kind,
                   const double *args, double *out);

static void grf_core(int64_t N, double L, const double *Psi, double psi_scale, cfo_spectrum_fn P, const double *args,
                     double *out) {
  const int64_t N3 = N * N * N, nh = N / 2 + 1;
  if (Psi)
    for (int64_t i = 0; i < N3; ++i) out[i] = out[i] * exp(psi_scale * Psi[i]);
  double *hc = (double *)malloc(sizeof(double) * 2 * N * N * nh);
  cfo_d2z(N, out, hc);
  for (int64_t a = 0; a < N; ++a)
    for (int64_t b = 0; b < N; ++b)
      for (int64_t c = 0; c < nh; ++c) {
        int64_t as = (a <= N / 2) ? a : (a - N), bs = (b <= N / 2) ? b : (b - N);
        int64_t s2 = as * as + bs * bs + c * c;
        double abs_k = sqrt((double)s2) * 2 * CFO_PI / L;
        double sp = sqrt(P(abs_k, args));
        int64_t o = 2 * (N * nh * a + nh * b + c);
        hc[o] *= sp;
        hc[o + 1] *= sp;
      }
  fftw_plan pl = fftw_plan_dft_c2r_3d((int)N, (int)N, (int)N, (fftw_complex *)hc, out, FFTW_ESTIMATE);
  fftw_execute_dft_c2r(pl, (fftw_complex *)hc, out);
  fftw_destroy_plan(pl);
  free(hc);
}

/* Spectra of src/random_field.cpp:92-121 and :128-134, args as listed. */
/* args = {P_k_ast, k_ast, alpha}: power law with sharp cutoff. */
static double sp_power_law_cutoff(double k, const double *args) {
  return k == 0.0 ? 0.0 : (args[0] * (k <= args[1] ? pow(k / args[1], args[2]) : 0.0));
}
/* args = {P_k_ast, k_ast, alpha, m}: (k^2 + m^2) times the above. */
static double sp_deriv_power_law_cutoff(double k, const double *args) {
  return (k * k + args[3] * args[3]) * sp_power_law_cutoff(k, args);
}
/* args = {P_k0}: scale invariant with k0 = 1. */
static double sp_scale_invariant(double k, const double *args) {
  return k == 0.0 ? 0.0 : (args[0] * pow(k / 1.0, -3));
}

static cfo_spectrum_fn spectrum_of(int kind) {
  return kind == 0 ? sp_power_law_cutoff : kind == 1 ? sp_deriv_power_law_cutoff : sp_scale_invariant;
}

/* kind 0: args = {P_k_ast, k_ast, alpha}; 1: {P_k_ast, k_ast, alpha, m}; 2: {P_k0}. */
void cfo_grf_white(int64_t N, double L, const double *white, const double *Psi, double psi_scale, int kind,
                   const double *args, double *out) {
  const int64_t N3 = N * N * N;
  for (int64_t i = 0; i < N3; ++i) out[i] = (1.0 / (double)N3) * white[i];
  grf_core(N, L, Psi, psi_scale, spectrum_of(kind), args, out);
}

/* sqrt(P(sqrt(s^2) 2 pi / L)) for s^2 = 0 .. 3(N/2)^2: the per-mode factor of the GRF. */
void cfo_sqrtP_table(int64_t N, double L, int kind, const double *args, double *out) {
  const int64_t n = 3 * (N / 2) * (N / 2) + 1;
  cfo_spectrum_fn P = spectrum_of(kind);
  for (int64_t s2 = 0; s2 < n; ++s2) out[s2] = sqrt(P(sqrt((double)s2) * 2 * CFO_PI / L, args));
}

/* P_k_ast of power_law_with_cutoff_given_amplitude_3d (src/random_field.cpp:92-101). */
double cfo_power_law_amplitude(int64_t N, double L, double sigma, double k_ast, double alpha) {
  double P = alpha == -3.0
                 ? 2 * CFO_PI * CFO_PI * sigma * sigma / (k_ast * k_ast * k_ast * log(k_ast * L / (2 * CFO_PI)))
                 : (3 + alpha) * 2 * CFO_PI * CFO_PI * sigma * sigma * (L * L * L * pow(k_ast * L, alpha)) /
                       (pow(k_ast * L, alpha + 3) - pow(2 * CFO_PI, alpha + 3));
  P *= ((double)N / L) * ((double)N / L) * ((double)N / L);
  return P;
}

/* Cosine integral Ci(x), x > 0.  Up to x = 4: the convergent power series
 * gamma + ln x + sum_{k>=1} (-x^2)^k / (2k (2k)!) (Abramowitz & Stegun 5.2.16); beyond,
 * where the series' alternating terms lose digits: Ci(x) = -Re E1(ix) with E1 from its
 * continued fraction E1(z) = e^{-z} / (z + 1 - 1^2 / (z + 3 - 2^2 / (z + 5 - ...)))
 * (A&S 5.1.22), evaluated by the modified Lentz method.  (The reference evaluates a
 * Pade approximant, src/special_function.hpp:4-26; they agree to rounding.) */
double cfo_ci(double x) {
  if (x <= 2.0) {
    double sum = 0.0, term = 1.0;
    for (int k = 1; k < 80; ++k) {
      term *= -x * x / ((2.0 * k - 1) * (2.0 * k));
      double add = term / (2.0 * k);
      sum += add;
      if (fabs(add) < 1e-18 * fabs(sum)) break;
    }
    return 0.57721566490153286061 + log(x) + sum;
  }
  double complex b = 1.0 + x * I, c = 1e300, d = 1.0 / b, h = d;
  for (int i = 1; i < 1000; ++i) {
    double a = -(double)i * i;
    b += 2.0;
    d = 1.0 / (a * d + b);
    c = b + a / c;
    double complex del = c * d;
    h *= del;
    if (cabs(del - 1.0) < 1e-16) break;
  }
  h *= cos(x) - sin(x) * I;
  return -creal(h);
}

/* Rebuilds the initial state and R_fft of the reference driver
 * (src/main.cpp:88-138 with perturbed_grf_and_comoving_curvature_fft,
 * src/initializer.hpp:150-206): params of src/main.cpp:98-122 with N, L given.
 * state: 2N^3, R_fft: HC.  The amplitude A_s follows initializer.hpp:156-166
 * with Ci evaluated by the series above. */
/* Scalars of the reference driver's initializer (src/main.cpp:98-122 parameters,
 * perturbed_grf_and_comoving_curvature_fft, src/initializer.hpp:150-206). */
typedef struct {
  double eta_i, P_k0, alpha_phi, alpha_dphi, args[4];
} driver_consts;

static driver_consts driver_constants(int64_t N, double L) {
  const double m = 1.0, k_ast = 1.0, varphi_std = 1.0, Psi_std = 0.02, a1 = 1.0, H1 = 0.05;
  const double t1 = 1.0 / (2 * H1), t_start = t1;
  cfo_params P = {N, L, m, a1, H1, t1, 1.0, 2, 7};
  const double pi = CFO_PI;
  driver_consts d;
  double eta_i = cfo_eta(&P, t_start);
  double A_s = (-576 * pow(pi, 6) * pow(eta_i, 6) * pow(Psi_std, 2)) /
               (-81 * pow(L, 4) * (pow(L, 2) + 2 * pow(pi, 2) * pow(eta_i, 2)) +
                L * (81 * pow(L, 5) - 54 * pow(L, 3) * pow(pi, 2) * pow(eta_i, 2) + 48 * L * pow(pi, 4) * pow(eta_i, 4)) *
                    cos((4 * pi * eta_i) / (sqrt(3) * L)) +
                256 * pow(pi, 6) * pow(eta_i, 6) * cfo_ci((4 * pi * eta_i) / (sqrt(3) * L)) +
                4 * sqrt(3) * L * pi * eta_i * (27 * pow(L, 4) + 6 * pow(L, 2) * pow(pi, 2) * pow(eta_i, 2) - 16 * pow(pi, 4) * pow(eta_i, 4)) *
                    sin((4 * pi * eta_i) / (sqrt(3) * L)));
  double P_k0 = A_s / ((1.0 * 1.0 * 1.0) / (2 * pi * pi));
  P_k0 *= ((double)N / L) * ((double)N / L) * ((double)N / L);
  double v = k_ast / (a1 * m);
  d.eta_i = eta_i;
  d.P_k0 = P_k0;
  d.alpha_phi = 0.5 * (-3 * pow(4 * pow(v, 2) + 5, 2)) / (12 * pow(v, 4) + 50 * pow(v, 2) + 50);
  d.alpha_dphi = 0.5 * (25 - 20 * pow(v, 2)) / (12 * pow(v, 4) + 50 * pow(v, 2) + 50);
  d.args[0] = cfo_power_law_amplitude(N, L, varphi_std, k_ast, 0);
  d.args[1] = k_ast;
  d.args[2] = 0.0;
  d.args[3] = m;
  return d;
}

/* Psi transfer kernel of the initializer (src/initializer.hpp:184-186) over N^3
 * (the factor compute_field_with_scaled_fourier_modes applies, src/fdm3d.cpp:94). */
static double driver_kernel_scale(int64_t N, double L, double eta_i, int64_t s2) {
  const double pi = CFO_PI;
  double k = sqrt((double)s2) * (2 * pi / L);
  double kern = k == 0.0 ? 0.0
                         : (6 * sqrt(3) * (-((k * eta_i * cos((k * eta_i) / sqrt(3))) / sqrt(3)) + sin((k * eta_i) / sqrt(3)))) /
                               (pow(k, 3) * pow(eta_i, 3));
  return kern / (double)(N * N * N);
}

/* The per-s^2 tables and scalars the driver's initializer uses: sqrt P_R, the Psi
 * kernel / N^3, sqrt P_f, sqrt P_dtf (each 3(N/2)^2+1), alphas = {alpha_phi, alpha_dphi}. */
void cfo_driver_tables(int64_t N, double L, double *sqrtP_R, double *kern, double *sqrtP_f, double *sqrtP_df,
                       double *alphas) {
  driver_consts d = driver_constants(N, L);
  const int64_t n = 3 * (N / 2) * (N / 2) + 1;
  cfo_sqrtP_table(N, L, 2, &d.P_k0, sqrtP_R);
  cfo_sqrtP_table(N, L, 0, d.args, sqrtP_f);
  cfo_sqrtP_table(N, L, 1, d.args, sqrtP_df);
  for (int64_t s2 = 0; s2 < n; ++s2) kern[s2] = driver_kernel_scale(N, L, d.eta_i, s2);
  alphas[0] = d.alpha_phi;
  alphas[1] = d.alpha_dphi;
}

void cfo_driver_initial(int64_t N, double L, uint32_t seed, double *state, double *R_fft) {
  const int64_t N3 = N * N * N;
  cfo_rng *r = (cfo_rng *)malloc(sizeof(cfo_rng));
  cfo_rng_seed(r, seed);
  driver_consts d = driver_constants(N, L);
  double *R = (double *)malloc(sizeof(double) * N3);
  cfo_grf(r, N, L, NULL, 0.0, sp_scale_invariant, &d.P_k0, R);
  /* Psi = compute_field_with_scaled_fourier_modes(R, kernel) (src/fdm3d.cpp:76-102) */
  const int64_t nh = N / 2 + 1;
  double *hc = (double *)malloc(sizeof(double) * 2 * N * N * nh);
  cfo_d2z(N, R, hc);
  for (int64_t a = 0; a < N; ++a)
    for (int64_t b = 0; b < N; ++b)
      for (int64_t c = 0; c < nh; ++c) {
        int64_t as = (a <= N / 2) ? a : (N - a), bs = (b <= N / 2) ? b : (N - b);
        int64_t s2 = as * as + bs * bs + c * c;
        double scale = driver_kernel_scale(N, L, d.eta_i, s2);
        int64_t o = 2 * (N * nh * a + nh * b + c);
        hc[o] *= scale;
        hc[o + 1] *= scale;
      }
  double *Psi = (double *)malloc(sizeof(double) * N3);
  fftw_plan pl = fftw_plan_dft_c2r_3d((int)N, (int)N, (int)N, (fftw_complex *)hc, Psi, FFTW_ESTIMATE);
  fftw_execute_dft_c2r(pl, (fftw_complex *)hc, Psi);
  fftw_destroy_plan(pl);
  cfo_grf(r, N, L, Psi, d.alpha_phi, sp_power_law_cutoff, d.args, state);
  cfo_grf(r, N, L, Psi, d.alpha_dphi, sp_deriv_power_law_cutoff, d.args, state + N3);
  cfo_d2z(N, R, R_fft);
  free(R);
  free(hc);
  free(Psi);
  free(r);
}

/* ---- WKB continuation: WKBSolutionForKleinGordonEquationInFRW, src/wkb.cpp:5-121 ----
 * Radiation domination with t1 = 1/(2 H1) (the reference asserts both).  Modes of
 * a^{3/2} phi at t_i, rotated by the phase integral of the effective frequency from
 * t_i to t_f (the reference's closed form, grouped here by S(t) and U(t)). */
static double wkb_S(double k2, double a1, double H1, double m, double t) {
  return sqrt(H1 * (8 * k2 * t + pow(a1, 2) * H1 * (3 + 16 * pow(m, 2) * pow(t, 2))));
}

double cfo_wkb_phase(double k2, double a1, double H1, double m, double ti, double tf) {
  const double Sf = wkb_S(k2, a1, H1, m, tf), Si = wkb_S(k2, a1, H1, m, ti);
  const double Uf = (3 * pow(a1, 2) * H1 + 4 * k2 * tf) / (sqrt(3) * a1 * Sf);
  const double Ui = (3 * pow(a1, 2) * H1 + 4 * k2 * ti) / (sqrt(3) * a1 * Si);
  return Sf / (4. * a1 * H1) - Si / (4. * a1 * H1) + (sqrt(3) * log((1 - Uf) / (1 - Ui))) / 8. -
         (sqrt(3) * log((1 + Uf) / (1 + Ui))) / 8. +
         (k2 * log((k2 + a1 * m * (4 * a1 * H1 * m * tf + Sf)) / (k2 + a1 * m * (4 * a1 * H1 * m * ti + Si)))) /
             (4. * pow(a1, 2) * H1 * m);
}

void cfo_wkb(const cfo_params *P, const double *x, double t_i, double t_f, double *out) {
  const int64_t N = P->N, N3 = N * N * N, nh = N / 2 + 1, hc = 2 * N * N * nh;
  const double a1 = P->a1, H1 = P->H1, m = P->m, L = P->L;
  double *f = (double *)malloc(sizeof(double) * 4 * hc);
  double *g = f + 2 * hc;
  cfo_d2z(N, x, f);
  cfo_d2z(N, x + N3, f + hc);
  const double ai15 = pow(cfo_a(P, t_i), 1.5), Hi = cfo_H(P, t_i);
  for (int64_t i = 0; i < hc; ++i) f[i] *= ai15;
  for (int64_t i = 0; i < hc; ++i) f[hc + i] = ai15 * f[hc + i] + 1.5 * Hi * f[i];
  for (int64_t a = 0; a < N; ++a)
    for (int64_t b = 0; b < N; ++b)
      for (int64_t c = 0; c < nh; ++c) {
        int64_t as = (a <= N / 2) ? a : (N - a), bs = (b <= N / 2) ? b : (N - b);
        int64_t s2 = as * as + bs * bs + c * c;
        double k2 = s2 * pow(2 * CFO_PI / L, 2);
        int64_t o = 2 * (N * nh * a + nh * b + c);
        double ph = cfo_wkb_phase(k2, a1, H1, m, t_i, t_f);
        double w = sqrt(m * m + k2 / (2 * a1 * a1 * H1 * t_i) + 3 / (16 * t_i * t_i));
        double cv = cos(ph), sv = sin(ph);
        for (int r = 0; r < 2; ++r) {
          g[o + r] = f[o + r] * cv + f[hc + o + r] * sv / sqrt(w);
          g[hc + o + r] = f[hc + o + r] * cv - f[o + r] * sv * sqrt(w);
        }
      }
  fftw_plan pl = fftw_plan_dft_c2r_3d((int)N, (int)N, (int)N, (fftw_complex *)g, out, FFTW_ESTIMATE);
  fftw_execute_dft_c2r(pl, (fftw_complex *)g, out);
  fftw_execute_dft_c2r(pl, (fftw_complex *)(g + hc), out + N3);
  fftw_destroy_plan(pl);
  const double af15 = pow(cfo_a(P, t_f), 1.5), Hf = cfo_H(P, t_f);
  for (int64_t i = 0; i < N3; ++i) {
    double np_ = out[i] / (double)N3, nd = out[N3 + i] / (double)N3;
    out[i] = np_ / af15;
    out[N3 + i] = nd / af15 - 1.5 * Hf * np_ / af15;
  }
  free(f);
}
