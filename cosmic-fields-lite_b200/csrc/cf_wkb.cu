// cf_wkb.cu -- WKB continuation of a KG-FRW state to a later time
// (WKBSolutionForKleinGordonEquationInFRW, src/wkb.hpp:13-27, src/wkb.cpp:5-121).
//
// At t_i the modes of a^{3/2} phi and of its derivative a^{3/2} (dphi + 3/2 H phi)
// are taken once (one batched D2Z).  Evaluating at t rotates every mode by the phase
// integral of the effective frequency from t_i to t -- a closed form in k^2 only --
// and transforms back (one batched Z2D).  The phase, its cosine and sine and the
// initial frequency depend on a mode only through s^2, so the host evaluates them
// once per s^2 (3(N/2)^2 + 1 values, the reference's expressions) and the device
// applies them per mode: three streaming passes around the FFTs instead of the
// reference's N^3-iteration host loop with two logarithms per mode.
// Radiation domination with t1 = 1/(2 H1) only, as in the reference.

#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "cf_internal.cuh"

struct cf_wkb {
  cf_ctx *ctx = nullptr;
  double t_i = 0;
  double *modes = nullptr;  // 2 HC arrays: a^{3/2} phi, a^{3/2} (dphi + 3/2 H phi) at t_i
  double *work = nullptr;   // 2 HC arrays: the rotated modes
  double *tab = nullptr;    // 3 s2_bins: cos(phase), sin(phase), sqrt(omega_i)
  cufftHandle z2d2 = 0;
  bool have_z2d2 = false;
};

namespace cfb {

// The reference's phase integral (src/wkb.cpp:30-70), grouped by
// S(t) = sqrt(H1 (8 k^2 t + a1^2 H1 (3 + 16 m^2 t^2))) and U(t) = (3 a1^2 H1 + 4 k^2 t) / (sqrt(3) a1 S(t)).
static double wkb_S(double k2, double a1, double H1, double m, double t) {
  return std::sqrt(H1 * (8 * k2 * t + std::pow(a1, 2) * H1 * (3 + 16 * std::pow(m, 2) * std::pow(t, 2))));
}

static double wkb_phase(double k2, double a1, double H1, double m, double ti, double tf) {
  const double Sf = wkb_S(k2, a1, H1, m, tf), Si = wkb_S(k2, a1, H1, m, ti);
  const double Uf = (3 * std::pow(a1, 2) * H1 + 4 * k2 * tf) / (std::sqrt(3) * a1 * Sf);
  const double Ui = (3 * std::pow(a1, 2) * H1 + 4 * k2 * ti) / (std::sqrt(3) * a1 * Si);
  return Sf / (4. * a1 * H1) - Si / (4. * a1 * H1) + (std::sqrt(3) * std::log((1 - Uf) / (1 - Ui))) / 8. -
         (std::sqrt(3) * std::log((1 + Uf) / (1 + Ui))) / 8. +
         (k2 * std::log((k2 + a1 * m * (4 * a1 * H1 * m * tf + Sf)) / (k2 + a1 * m * (4 * a1 * H1 * m * ti + Si)))) /
             (4. * std::pow(a1, 2) * H1 * m);
}

// head *= a^{3/2}; tail = a^{3/2} tail + 3/2 H head   (src/wkb.cpp:17-18)
__global__ void k_wkb_init(double *__restrict__ f, long long hc, double a15, double h15) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < hc; i += stride) {
    const double p = f[i] * a15;
    f[i] = p;
    f[hc + i] = a15 * f[hc + i] + h15 * p;
  }
}

// Rotation of every HC mode by the tables of its s^2 (src/wkb.cpp:79-97).
__global__ void k_wkb_rotate(const double *__restrict__ f, double *__restrict__ g, const double *__restrict__ tab,
                             int N, long long s2_bins) {
  const long long nh = N / 2 + 1;
  const long long modes = (long long)N * N * nh;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const double2 *F = reinterpret_cast<const double2 *>(f);
  double2 *G = reinterpret_cast<double2 *>(g);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < modes; i += stride) {
    const int c = (int)(i % nh);
    const int b = (int)((i / nh) % N);
    const int a = (int)(i / (nh * N));
    const long long as = a <= N / 2 ? a : N - a, bs = b <= N / 2 ? b : N - b;
    const long long s2 = as * as + bs * bs + (long long)c * c;
    const double cv = tab[s2], sv = tab[s2_bins + s2], sw = tab[2 * s2_bins + s2];
    const double2 p = F[i], d = F[modes + i];
    G[i] = make_double2(p.x * cv + d.x * sv / sw, p.y * cv + d.y * sv / sw);
    G[modes + i] = make_double2(d.x * cv - p.x * sv * sw, d.y * cv - p.y * sv * sw);
  }
}

// phi = (z / N^3) / a^{3/2}, dphi = (zd / N^3) / a^{3/2} - 3/2 H (z / N^3) / a^{3/2}   (src/wkb.cpp:103-115)
__global__ void k_wkb_finish(double *__restrict__ x, long long N3, double a15, double h15) {
  const double n3 = (double)N3;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N3; i += stride) {
    const double np = x[i] / n3, nd = x[N3 + i] / n3;
    x[i] = np / a15;
    x[N3 + i] = nd / a15 - h15 * np / a15;
  }
}

static unsigned wkb_blocks(long long n) { return (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16); }

static int wkb_alloc(void **p, size_t bytes, const char *what) {
  if (cudaMalloc(p, bytes) != cudaSuccess) {
    cudaGetLastError();
    set_error("cudaMalloc of %s (%zu bytes) failed", what, bytes);
    return CF_ERR_NOMEM;
  }
  return CF_OK;
}

cf_ctx *wkb_ctx(cf_wkb *w) { return w->ctx; }

void wkb_destroy(cf_wkb *w) {
  if (!w) return;
  if (w->ctx) cudaSetDevice(w->ctx->device);
  cudaFree(w->modes);
  cudaFree(w->work);
  cudaFree(w->tab);
  if (w->have_z2d2) cufftDestroy(w->z2d2);
  delete w;
}

int wkb_create(cf_ctx *ctx, const double *d_state, double t_i, cf_wkb **out, cudaStream_t st) {
  const cf_params &p = ctx->p;
  if (p.equation != CF_EQ_KG_FRW || p.p != 1.0 || p.t1 != 1.0 / (2 * p.H1)) {
    set_error("WKB continuation: CF_EQ_KG_FRW in radiation domination (p = 1) with t1 = 1/(2 H1) only");
    return CF_ERR_UNSUPPORTED;
  }
  if (!(p.m > 0)) {
    set_error("WKB continuation needs m > 0");
    return CF_ERR_INVALID;
  }
  cf_wkb *w = new cf_wkb;
  w->ctx = ctx;
  w->t_i = t_i;
  const size_t hc = (size_t)ctx->hc_count;
  int s = CF_OK;
  if ((s = wkb_alloc((void **)&w->modes, 2 * hc * sizeof(double), "the WKB modes")) != CF_OK ||
      (s = wkb_alloc((void **)&w->work, 2 * hc * sizeof(double), "the WKB work modes")) != CF_OK ||
      (s = wkb_alloc((void **)&w->tab, 3 * (size_t)ctx->s2_bins * sizeof(double), "the WKB tables")) != CF_OK ||
      (s = ensure_spectrum_scratch(ctx, 2)) != CF_OK) {
    wkb_destroy(w);
    return s;
  }
  const int N = (int)ctx->N;
  int n[3] = {N, N, N};
  if (cufftPlanMany(&w->z2d2, 3, n, nullptr, 1, (int)(hc / 2), nullptr, 1, (int)ctx->N3, CUFFT_Z2D, 2) !=
      CUFFT_SUCCESS) {
    set_error("cufftPlanMany (WKB Z2D) failed");
    wkb_destroy(w);
    return CF_ERR_CUFFT;
  }
  w->have_z2d2 = true;
  // phi_ffts = execute_batched_d2z(state)   (src/wkb.cpp:14)
  if (cufftSetStream(ctx->plan_d2z2, st) != CUFFT_SUCCESS ||
      cufftExecD2Z(ctx->plan_d2z2, const_cast<double *>(d_state), (cufftDoubleComplex *)w->modes) != CUFFT_SUCCESS) {
    set_error("cufftExecD2Z (WKB modes) failed");
    wkb_destroy(w);
    return CF_ERR_CUFFT;
  }
  const double a15 = std::pow(cosmo_a(p, t_i), 1.5), h15 = 1.5 * cosmo_H(p, t_i);
  k_wkb_init<<<wkb_blocks((long long)hc), 256, 0, st>>>(w->modes, (long long)hc, a15, h15);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("kernel launch failed: %s", cudaGetErrorString(e));
    wkb_destroy(w);
    return CF_ERR_CUDA;
  }
  ctx->launches++;
  *out = w;
  return CF_OK;
}

int wkb_evaluate(cf_wkb *w, double t, double *d_out, cudaStream_t st) {
  cf_ctx *ctx = w->ctx;
  const cf_params &p = ctx->p;
  const long long bins = ctx->s2_bins;
  const double pi = 3.14159265358979323846;
  const double a1 = p.a1, H1 = p.H1, m = p.m, ti = w->t_i;
  std::vector<double> tab(3 * (size_t)bins);
  for (long long s2 = 0; s2 < bins; ++s2) {
    const double k2 = s2 * std::pow(2 * pi / p.L, 2);  // src/wkb.cpp:82
    const double ph = wkb_phase(k2, a1, H1, m, ti, t);
    const double omega_i = std::sqrt(m * m + k2 / (2 * a1 * a1 * H1 * ti) + 3 / (16 * ti * ti));
    tab[s2] = std::cos(ph);
    tab[bins + s2] = std::sin(ph);
    tab[2 * bins + s2] = std::sqrt(omega_i);
  }
  CF_TRY_CUDA(cudaMemcpyAsync(w->tab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  ProfScope ps(ctx, CF_PROF_OTHER, st);
  k_wkb_rotate<<<wkb_blocks(ctx->hc_count / 2), 256, 0, st>>>(w->modes, w->work, w->tab, (int)ctx->N, bins);
  CF_LAUNCHED(ctx);
  CF_TRY_CUFFT(cufftSetStream(w->z2d2, st));
  CF_TRY_CUFFT(cufftExecZ2D(w->z2d2, (cufftDoubleComplex *)w->work, d_out));
  const double a15 = std::pow(cosmo_a(p, t), 1.5), h15 = 1.5 * cosmo_H(p, t);
  k_wkb_finish<<<wkb_blocks(ctx->N3), 256, 0, st>>>(d_out, ctx->N3, a15, h15);
  CF_LAUNCHED(ctx);
  // the host table must outlive its copy (pageable memory is staged, but be explicit)
  CF_TRY_CUDA(cudaStreamSynchronize(st));
  return CF_OK;
}

}  // namespace cfb
