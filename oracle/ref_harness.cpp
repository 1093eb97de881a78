/*
 * ref_harness.cpp -- C entry points around the reference's OWN CPU sources.
 *
 * TEST INFRASTRUCTURE ONLY (oracle).  This file is compiled together with the
 * unmodified reference sources src/equations.cpp, src/fdm3d.cpp,
 * src/fftw_wrapper.cpp, src/random_field.cpp, src/io.cpp, src/eigen_wrapper.cpp,
 * src/wkb.cpp (read in place from the reference tree by oracle/Makefile) and the FFTW3
 * restatement oracle/fftw_shim.c, into oracle/_ref/libcfref*.so.  Only tests/,
 * the smoke check and bench.py's CPU-baseline / reference legs load it.
 *
 * Every function drives the reference through its public API, exactly as the
 * reference's driver does (src/main.cpp:82-196):
 *   WorkspaceGeneric<Eigen::VectorXd>(param, initializer)   src/workspace.hpp:81-93
 *   KleinGordonEquation / KleinGordonEquationInFRW /
 *   ComovingCurvatureEquationInFRW                           src/equations.hpp:36-117
 *   runge_kutta4_classic<VectorXd,double,VectorXd,double>    src/main.cpp:153
 *   integrate_const(stepper, eqn, state, t0, t1, dt, obs)    src/main.cpp:183
 *   ConstIntervalObserver<Equation, true, true, false>       src/observer.hpp:64-126
 *   compute_power_spectrum / compute_mode_power_spectrum     src/fdm3d.cpp:7-72
 *
 * Equation codes: 0 = KleinGordonEquation (flat), 1 = KleinGordonEquationInFRW,
 * 2 = ComovingCurvatureEquationInFRW.
 */
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "Eigen/Dense"
#include "equations.hpp"
#include "fdm3d.hpp"
#include "initializer.hpp"
#include "observer.hpp"
#include "param.hpp"
#include "physics.hpp"
#include "random_field.hpp"
#include "wkb.hpp"
#include "workspace.hpp"

namespace {

/* Parameter POD for the flat equation: lattice + mass only, so the workspace
 * keeps its default (Minkowski) cosmology (src/workspace.hpp:86). */
struct FlatParam {
  long long int N;
  double L;
  double m;
  double t_start;
  double t_end;
  double t_interval;
};

/* Parameter POD with FRW background (src/workspace.hpp:35-38). */
struct FRWParam {
  long long int N;
  double L;
  double m;
  double a1;
  double H1;
  double t1;
  double t_start;
  double t_end;
  double t_interval;
};

/* Same field set as the reference driver's MyParam (src/main.cpp:36-64), used to
 * regenerate the published N=384 outputs. */
struct DriverParam {
  long long int N;
  double L;
  double m;
  double lambda;
  double f_a;
  double k_ast;
  double k_Psi;
  double varphi_std_dev;
  double Psi_std_dev;
  double a1;
  double H1;
  double t1;
  double t_start;
  double t_end;
  double t_interval;
  double delta_t;
  long long int M;
  double f;
  double delta_varphi_std_dev;
  double k_delta_varphi;
};

typedef Eigen::VectorXd Vec;

struct HostInit {
  const double *state;
  const double *R_fft;
  long long n_state;
  long long n_hc;
  template <typename P, typename W>
  void operator()(const P &, W &ws) const {
    ws.state.resize(n_state);
    std::memcpy(ws.state.data(), state, sizeof(double) * n_state);
    if (R_fft) {
      ws.R_fft.resize(n_hc);
      std::memcpy(ws.R_fft.data(), R_fft, sizeof(double) * n_hc);
    }
  }
};

/* An observer that does nothing (used for timing the stepping loop alone). */
struct NullObserver {
  template <typename S>
  void operator()(const S &, double) {}
};

template <typename Equation, typename Param>
int integrate_impl(const Param &param, double *state, const double *R_fft, double t_start,
                   double t_end, double dt, const char *dir, double *t_list, int max_saves) {
  const long long N = param.N;
  HostInit init{state, R_fft, 2 * N * N * N, 2 * N * N * (N / 2 + 1)};
  typename Equation::Workspace workspace(param, init);
  Equation eqn(workspace);
  auto stepper = boost::numeric::odeint::runge_kutta4_classic<Vec, double, Vec, double>();
  int nsteps;
  if (dir && dir[0]) {
    ConstIntervalObserver<Equation, true, true, false> observer(std::string(dir), param, eqn);
    nsteps = (int)boost::numeric::odeint::integrate_const(stepper, eqn, workspace.state, t_start,
                                                          t_end, dt, observer);
  } else {
    nsteps = (int)boost::numeric::odeint::integrate_const(stepper, eqn, workspace.state, t_start,
                                                          t_end, dt, NullObserver{});
  }
  std::memcpy(state, workspace.state.data(), sizeof(double) * 2 * N * N * N);
  if (t_list) {
    for (int i = 0; i < (int)workspace.t_list.size() && i < max_saves; ++i) t_list[i] = workspace.t_list[i];
  }
  return dir && dir[0] ? (int)workspace.t_list.size() : nsteps;
}

}  // namespace

extern "C" {

/* Runs integrate_const with the reference's RK4 from t_start to t_end with step dt.
 * state (2N^3, [phi|dphi], IDX_OF layout) is overwritten with the final state.
 * When dir is non-empty the reference observer writes its spectra files there
 * and t_list receives the save times; returns the number of saves, else the
 * number of steps. */
int cfr_integrate(int eq, long long N, double L, double m, double a1, double H1, double t1,
                  double *state, const double *R_fft, double t_start, double t_end, double dt,
                  double t_interval, const char *dir, double *t_list, int max_saves) {
  if (eq == 0) {
    FlatParam p{N, L, m, t_start, t_end, t_interval};
    return integrate_impl<KleinGordonEquation>(p, state, nullptr, t_start, t_end, dt, dir, t_list, max_saves);
  }
  FRWParam p{N, L, m, a1, H1, t1, t_start, t_end, t_interval};
  if (eq == 1)
    return integrate_impl<KleinGordonEquationInFRW>(p, state, nullptr, t_start, t_end, dt, dir, t_list, max_saves);
  return integrate_impl<ComovingCurvatureEquationInFRW>(p, state, R_fft, t_start, t_end, dt, dir, t_list, max_saves);
}

/* One right-hand-side evaluation: dxdt = Equation(x, t). */
void cfr_rhs(int eq, long long N, double L, double m, double a1, double H1, double t1,
             const double *x, const double *R_fft, double t, double *dxdt) {
  HostInit init{x, R_fft, 2 * N * N * N, 2 * N * N * (N / 2 + 1)};
  Vec xv = Eigen::Map<const Vec>(x, 2 * N * N * N);
  Vec out(2 * N * N * N);
  if (eq == 0) {
    FlatParam p{N, L, m, 0, 0, 0};
    KleinGordonEquation::Workspace ws(p, init);
    KleinGordonEquation e(ws);
    e(xv, out, t);
  } else if (eq == 1) {
    FRWParam p{N, L, m, a1, H1, t1, 0, 0, 0};
    KleinGordonEquationInFRW::Workspace ws(p, init);
    KleinGordonEquationInFRW e(ws);
    e(xv, out, t);
  } else {
    FRWParam p{N, L, m, a1, H1, t1, 0, 0, 0};
    ComovingCurvatureEquationInFRW::Workspace ws(p, init);
    ComovingCurvatureEquationInFRW e(ws);
    e(xv, out, t);
  }
  std::memcpy(dxdt, out.data(), sizeof(double) * 2 * N * N * N);
}

/* Equation::compute_energy_density(workspace, t) -> rho (N^3). */
void cfr_energy_density(int eq, long long N, double L, double m, double a1, double H1, double t1,
                        const double *state, const double *R_fft, double t, double *rho) {
  HostInit init{state, R_fft, 2 * N * N * N, 2 * N * N * (N / 2 + 1)};
  Vec r;
  if (eq == 0) {
    FlatParam p{N, L, m, 0, 0, 0};
    KleinGordonEquation::Workspace ws(p, init);
    r = KleinGordonEquation::compute_energy_density(ws, t);
  } else if (eq == 1) {
    FRWParam p{N, L, m, a1, H1, t1, 0, 0, 0};
    KleinGordonEquationInFRW::Workspace ws(p, init);
    r = KleinGordonEquationInFRW::compute_energy_density(ws, t);
  } else {
    FRWParam p{N, L, m, a1, H1, t1, 0, 0, 0};
    ComovingCurvatureEquationInFRW::Workspace ws(p, init);
    r = ComovingCurvatureEquationInFRW::compute_energy_density(ws, t);
  }
  std::memcpy(rho, r.data(), sizeof(double) * N * N * N);
}

/* compute_power_spectrum(N, f, fftw) -> out (3(N/2)^2+1 bins). */
void cfr_power_spectrum(long long N, const double *f, double *out) {
  fftwWrapper fft((int)N);
  Vec fv = Eigen::Map<const Vec>(f, N * N * N);
  Vec s = compute_power_spectrum(N, fv, fft);
  std::memcpy(out, s.data(), sizeof(double) * s.size());
}

/* compute_mode_power_spectrum(N, L, m, a_t, state, fftw) -> out. */
void cfr_mode_power_spectrum(long long N, double L, double m, double a_t, const double *state, double *out) {
  fftwWrapper fft((int)N);
  Vec sv = Eigen::Map<const Vec>(state, 2 * N * N * N);
  Vec s = compute_mode_power_spectrum(N, L, m, a_t, sv, fft);
  std::memcpy(out, s.data(), sizeof(double) * s.size());
}

/* The reference's r2c as used for R_fft (fftwWrapper::execute_d2z). */
void cfr_d2z(long long N, const double *f, double *out_hc) {
  fftwWrapper fft((int)N);
  Vec fv = Eigen::Map<const Vec>(f, N * N * N);
  Vec o = fft.execute_d2z(fv);
  std::memcpy(out_hc, o.data(), sizeof(double) * o.size());
}

/* Reproduces the reference driver's set-up (src/main.cpp:88-177) for a given N, L
 * and seed: seeds RandomNormal, builds the workspace with
 * perturbed_grf_and_comoving_curvature_fft, writes initial_R_spectrum.dat and
 * initial_Psi_spectrum.dat, and runs the observer once at t_start (writing
 * varphi_plus_spectrum_0.dat, rho_spectrum_0.dat, rho_slice_0.dat,
 * rho_axis_average_0.dat) into dir.  If state_out / R_fft_out are non-null the
 * initial state and R_fft are copied there. */
void cfr_driver_initial(long long N, double L, unsigned seed, const char *dir, double *state_out,
                        double *R_fft_out) {
  RandomNormal::set_generator_seed(seed);
  DriverParam param{};
  param.N = N;
  param.L = L;
  param.m = 1.0;
  param.lambda = 0;
  param.k_ast = 1.0;
  param.k_Psi = 1.0;
  param.varphi_std_dev = 1.0;
  param.Psi_std_dev = 0.02;
  param.a1 = 1.0;
  param.H1 = 0.05;
  param.t1 = 1.0 / (2 * param.H1);
  param.t_start = param.t1;
  param.t_end = param.t_start + (pow(3.5 / param.a1, 2) - 1.0) / (2 * param.H1);
  param.t_interval = 49.99;
  param.delta_t = 0.5;
  param.M = 128;
  typedef ComovingCurvatureEquationInFRW Equation;
  Equation::Workspace workspace(param, perturbed_grf_and_comoving_curvature_fft);
  Equation eqn(workspace);
  std::string d(dir);
  {
    double eta_i = workspace.cosmology.eta(param.t_start);
    auto kernel = [eta_i](double k) {
      return k == 0.0 ? 0.0
                      : (6 * sqrt(3) * (-((k * eta_i * cos((k * eta_i) / sqrt(3))) / sqrt(3)) +
                                        sin((k * eta_i) / sqrt(3)))) /
                            (pow(k, 3) * pow(eta_i, 3));
    };
    Eigen::VectorXd R_fft_eigen = workspace.R_fft;
    auto fft_wrapper = fftwWrapper(param.N);
    Eigen::VectorXd R = fft_wrapper.execute_z2d(R_fft_eigen) / pow(param.N, 3);
    Eigen::VectorXd Psi = compute_field_with_scaled_fourier_modes(param.N, param.L, R, kernel, fft_wrapper);
    auto Psi_spectrum = compute_power_spectrum(param.N, Psi, fft_wrapper);
    write_VectorXd_to_file(Psi_spectrum, d + "initial_Psi_spectrum.dat");
    auto R_spectrum = compute_power_spectrum(param.N, R, fft_wrapper);
    write_VectorXd_to_file(R_spectrum, d + "initial_R_spectrum.dat");
  }
  if (state_out) std::memcpy(state_out, workspace.state.data(), sizeof(double) * workspace.state.size());
  if (R_fft_out) std::memcpy(R_fft_out, workspace.R_fft.data(), sizeof(double) * workspace.R_fft.size());
  ConstIntervalObserver<Equation, true, true, true> observer(d, param, eqn);
  observer(workspace.state, param.t_start);
}

/* WKBSolutionForKleinGordonEquationInFRW (src/wkb.hpp:13-27, src/wkb.cpp:5-121): the
 * KG-FRW state x given at t_i, continued to t_f; out = evaluate_at(t_f) (2N^3). */
void cfr_wkb(long long N, double L, double m, double a1, double H1, double t1, const double *x, double t_i,
             double t_f, double *out) {
  HostInit init{x, nullptr, 2 * N * N * N, 2 * N * N * (N / 2 + 1)};
  FRWParam p{N, L, m, a1, H1, t1, 0, 0, 0};
  KleinGordonEquationInFRW::Workspace ws(p, init);
  WKBSolutionForKleinGordonEquationInFRW wkb(ws, t_i);
  Vec r = wkb.evaluate_at(t_f);
  std::memcpy(out, r.data(), sizeof(double) * 2 * N * N * N);
}

}  // extern "C"
