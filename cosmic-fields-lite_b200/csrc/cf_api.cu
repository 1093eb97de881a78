// cf_api.cu -- the C ABI (include/cfb200.h): context, state transfer, dispatch.

#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <cstdarg>
#include <cstring>
#include <new>

#include "cf_internal.cuh"

namespace cfb {

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

const char *get_error() { return g_err; }

// StaticEOSCosmology::a / H / eta (src/physics.hpp:34-55), same expressions.
double cosmo_a(const cf_params &p, double t) {
  return p.a1 * pow(1 + (1 + 1 / p.p) * p.H1 * (t - p.t1), p.p / (1 + p.p));
}
double cosmo_H(const cf_params &p, double t) { return p.H1 * pow(1 + (1 + 1 / p.p) * p.H1 * (t - p.t1), -1); }
double cosmo_eta(const cf_params &p, double t) {
  return (p.p / (p.a1 * p.H1)) * pow(1 + (1 + 1 / p.p) * p.H1 * (t - p.t1), 1 / (1 + p.p));
}

void stage_coeffs(const cf_params &p, double t, double *inv_ah2, double *H) {
  const double h = p.L / (double)p.N;
  if (p.equation == CF_EQ_KG) {
    *inv_ah2 = 1.0 / (h * h);  // src/equations.cpp:14
    *H = 0.0;
    return;
  }
  const double a_t = cosmo_a(p, t);
  *H = cosmo_H(p, t);
  *inv_ah2 = 1.0 / (h * h) / (a_t * a_t);  // src/equations.cpp:80
}

int ensure_rk4_scratch(cf_ctx *ctx) {
  if (ctx->acc) return CF_OK;
  const size_t bytes = 2 * (size_t)ctx->N3 * ctx->word;
  void *p = nullptr;
  if (cudaMalloc(&p, 3 * bytes) != cudaSuccess) {
    cudaGetLastError();
    set_error("cudaMalloc of the RK4 temporaries (%zu bytes) failed", 3 * bytes);
    return CF_ERR_NOMEM;
  }
  ctx->acc = p;
  ctx->ya = (char *)p + bytes;
  ctx->yb = (char *)p + 2 * bytes;
  return CF_OK;
}

// defined in the other translation units
int rk4_steps(cf_ctx *, void *, double, double, int64_t, int64_t, cudaStream_t);
int rhs(cf_ctx *, const double *, double *, double, cudaStream_t);
int scale_sum(cf_ctx *, double *, int, const double *const *, const double *, int64_t, cudaStream_t);
int set_R_fft(cf_ctx *, const double *, int, cudaStream_t);
int energy_density(cf_ctx *, const void *, double, double *, cudaStream_t);
int dot_energy_density(cf_ctx *, const void *, double, double *, cudaStream_t);
int white_noise(cf_ctx *, uint64_t, uint64_t, double *, int64_t, cudaStream_t);
int density_slices(cf_ctx *, const void *, double, double *, double *, cudaStream_t);
int wkb_create(cf_ctx *, const double *, double, cf_wkb **, cudaStream_t);
int wkb_evaluate(cf_wkb *, double, double *, cudaStream_t);
void wkb_destroy(cf_wkb *);
cf_ctx *wkb_ctx(cf_wkb *);
int grf(cf_ctx *, const double *, const double *, double, const double *, double *, cudaStream_t);
int scale_modes(cf_ctx *, const double *, const double *, double *, cudaStream_t);
int power_spectrum_s2(cf_ctx *, const double *, double *, cudaStream_t);
int mode_power_spectrum_s2(cf_ctx *, const void *, double, double *, cudaStream_t);
int density_spectrum_s2(cf_ctx *, const void *, double, double *, cudaStream_t);
int s2_to_shells(cf_ctx *, double *, int64_t *, cudaStream_t);
int s2_counts(cf_ctx *, int64_t *, cudaStream_t);
int state_export(cf_ctx *, double *, const void *, cudaStream_t);
int state_import(cf_ctx *, void *, const double *, cudaStream_t);
int state_upload_host(cf_ctx *, void *, const double *, cudaStream_t);
int state_download_host(cf_ctx *, double *, const void *, cudaStream_t);
int check_finite(cf_ctx *, const void *, int64_t *, cudaStream_t);
int adjoint_create(cf_ctx *, int64_t, int64_t, cf_adjoint **);
void adjoint_destroy(cf_adjoint *);
int adjoint_forward(cf_adjoint *, void *, double, double, cudaStream_t);
int adjoint_shell_log_loss(cf_adjoint *, const void *, const double *, double, double *, cudaStream_t);
int adjoint_set_lambda(cf_adjoint *, const double *, double, cudaStream_t);
int adjoint_backward(cf_adjoint *, double *, double *, cudaStream_t);
cf_ctx *adjoint_ctx(cf_adjoint *);
int field_from_shell_amplitudes(cf_ctx *, const double *, const double *, const double *, int, int, double *,
                                cudaStream_t);
int shell_amplitude_gradient(cf_ctx *, const double *, const double *, const double *, const double *, int, int,
                             double *, cudaStream_t);

ProfScope::ProfScope(cf_ctx *c, int k, cudaStream_t s) : ctx(c), kind(k), st(s) {
  if (!ctx->prof_on) return;
  if (ctx->prof_pool.empty()) {
    if (cudaEventCreate(&a) != cudaSuccess) {
      a = nullptr;
      return;
    }
  } else {
    a = ctx->prof_pool.back();
    ctx->prof_pool.pop_back();
  }
  cudaEventRecord(a, st);
}

static void prof_drain(cf_ctx *ctx) {
  for (auto &r : ctx->prof_pending) {
    cudaEventSynchronize(r.b);
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      ctx->prof_ms[r.kind] += ms;
      ctx->prof_launches[r.kind] += 1;
    }
    ctx->prof_pool.push_back(r.a);
    ctx->prof_pool.push_back(r.b);
  }
  ctx->prof_pending.clear();
}

ProfScope::~ProfScope() {
  if (!a) return;
  cudaEvent_t b = nullptr;
  if (ctx->prof_pool.empty()) {
    if (cudaEventCreate(&b) != cudaSuccess) return;
  } else {
    b = ctx->prof_pool.back();
    ctx->prof_pool.pop_back();
  }
  cudaEventRecord(b, st);
  ctx->prof_pending.push_back({kind, a, b});
  if (ctx->prof_pending.size() > 8192) prof_drain(ctx);
}

static long long isqrt_host(long long s) {
  long long r = (long long)std::sqrt((double)s);
  while (r * r > s) --r;
  while ((r + 1) * (r + 1) <= s) ++r;
  return r;
}

static int check_ctx(const cf_ctx *ctx) {
  if (!ctx) {
    set_error("NULL context");
    return CF_ERR_INVALID;
  }
  return CF_OK;
}

static int check_ptr(const void *p, const char *what, size_t align = 16) {
  if (!p) {
    set_error("%s is NULL", what);
    return CF_ERR_INVALID;
  }
  if (((uintptr_t)p) % align) {
    set_error("%s is not %zu-byte aligned", what, align);
    return CF_ERR_INVALID;
  }
  return CF_OK;
}

static int use_device(const cf_ctx *ctx) {
  CF_TRY_CUDA(cudaSetDevice(ctx->device));
  return CF_OK;
}

// The curvature input the context's equation needs before it can be evaluated:
// R_fft for the comoving equations, Psi for the fixed-curvature one.
static int check_curvature(const cf_ctx *ctx) {
  const int eq = ctx->p.equation;
  if ((eq == CF_EQ_COMOVING_FRW || eq == CF_EQ_APPROX_COMOVING_FRW) && !ctx->R_fft) {
    set_error("comoving-curvature equation: call cf_set_R_fft first");
    return CF_ERR_INVALID;
  }
  if (eq == CF_EQ_FIXED_CURVATURE_FRW && !ctx->fixed_e2m1) {
    set_error("fixed-curvature equation: call cf_set_psi first");
    return CF_ERR_INVALID;
  }
  return CF_OK;
}

}  // namespace cfb

using namespace cfb;

extern "C" {

const char *cf_last_error(void) { return get_error(); }

int cf_create(const cf_params *params, cf_ctx **out) {
  if (!params || !out) {
    set_error("cf_create: NULL argument");
    return CF_ERR_INVALID;
  }
  *out = nullptr;
  const cf_params &p = *params;
  if (p.N < 8 || p.N > 2048 || p.N % 8 != 0) {
    set_error("N = %lld unsupported: need N %% 8 == 0 and 8 <= N <= 2048", (long long)p.N);
    return CF_ERR_INVALID;
  }
  if (!(p.L > 0) || !std::isfinite(p.L) || !std::isfinite(p.m)) {
    set_error("L must be positive and finite, m finite");
    return CF_ERR_INVALID;
  }
  if (p.equation < CF_EQ_KG || p.equation > CF_EQ_APPROX_COMOVING_FRW) {
    set_error("unknown equation %d", p.equation);
    return CF_ERR_INVALID;
  }
  if (p.precision != CF_FP64 && p.precision != CF_FP32_COMP) {
    set_error("unknown precision %d", p.precision);
    return CF_ERR_INVALID;
  }
  if (p.stencil != 7 && p.stencil != 13) {
    set_error("stencil must be 7 or 13, got %d", p.stencil);
    return CF_ERR_INVALID;
  }
  if (p.flags & ~(CF_FLAG_FULL_PSI_FFT | CF_FLAG_STAGE_KERNELS | CF_FLAG_PAIR_KERNELS | CF_FLAG_PSI_CTA_PASS_C |
                  CF_FLAG_PSI_SERIAL | CF_FLAG_PSI_NO_TMA | CF_FLAG_PSI_NO_REUSE)) {
    set_error("unknown flags 0x%x", (unsigned)p.flags);
    return CF_ERR_INVALID;
  }
  if (p.equation != CF_EQ_KG && (!(p.p > 0) || !std::isfinite(p.a1) || !std::isfinite(p.H1) || !std::isfinite(p.t1))) {
    set_error("FRW parameters must be finite with p > 0");
    return CF_ERR_INVALID;
  }
  if ((p.equation == CF_EQ_COMOVING_FRW || p.equation == CF_EQ_APPROX_COMOVING_FRW) &&
      (p.H1 == 0.0 || p.a1 == 0.0)) {
    set_error("the comoving-curvature equation needs a1 != 0 and H1 != 0 (conformal time)");
    return CF_ERR_INVALID;
  }
  if (p.equation == CF_EQ_LAMBDA_FRW && !std::isfinite(p.lambda)) {
    set_error("lambda must be finite");
    return CF_ERR_INVALID;
  }
  if (p.equation == CF_EQ_SQRT_FRW && !(p.f_a > 0 && std::isfinite(p.f_a))) {
    set_error("the sqrt potential needs a finite f_a > 0");
    return CF_ERR_INVALID;
  }
  if (p.equation == CF_EQ_APPROX_COMOVING_FRW && (p.M < 8 || p.M % 8 != 0 || p.M > p.N || p.N % p.M != 0)) {
    set_error("the approximate comoving equation needs M %% 8 == 0, 8 <= M <= N and N %% M == 0 (M = %lld)",
              (long long)p.M);
    return CF_ERR_INVALID;
  }
  int dev = 0;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    set_error("no usable CUDA device: %s", e != cudaSuccess ? cudaGetErrorString(e) : "device count is 0");
    return CF_ERR_CUDA;
  }
  CF_TRY_CUDA(cudaGetDevice(&dev));
  cf_ctx *ctx = new (std::nothrow) cf_ctx();
  if (!ctx) {
    set_error("host allocation failed");
    return CF_ERR_NOMEM;
  }
  ctx->p = p;
  ctx->N = p.N;
  ctx->N3 = p.N * p.N * p.N;
  ctx->nh = p.N / 2 + 1;
  ctx->hc_count = 2 * p.N * p.N * (p.N / 2 + 1);
  ctx->s2_bins = 3 * (p.N / 2) * (p.N / 2) + 1;
  ctx->shells = isqrt_host(ctx->s2_bins - 1) + 1;
  ctx->device = dev;
  ctx->word = p.precision == CF_FP32_COMP ? 4 : 8;
  *out = ctx;
  return CF_OK;
}

int cf_destroy(cf_ctx *ctx) {
  if (!ctx) return CF_OK;
  cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  prof_drain(ctx);
  for (auto e : ctx->prof_pool) cudaEventDestroy(e);
  cudaFree(ctx->acc);
  cudaFree(ctx->R_fft);
  cudaFree(ctx->psi_hc);
  cudaFree(ctx->psi_table);
  for (auto &s : ctx->slot) {
    cudaFree(s.psi);
    if (s.ready) cudaEventDestroy(s.ready);
  }
  if (ctx->psi_side) {
    cudaStreamSynchronize(ctx->psi_side);
    cudaStreamDestroy(ctx->psi_side);
    cudaEventDestroy(ctx->psi_fork);
    cudaEventDestroy(ctx->psi_join);
    cudaEventDestroy(ctx->psi_stepdone);
  }
  if (ctx->have_plan_psi) cufftDestroy(ctx->plan_psi);
  psi_release(ctx);
  if (ctx->psi_err_h) cudaFreeHost(ctx->psi_err_h);
  if (ctx->pa_diff_h) cudaFreeHost(ctx->pa_diff_h);
  if (ctx->pa_check) cudaEventDestroy(ctx->pa_check);
  approx_release(ctx);
  if (ctx->have_d2z1) cufftDestroy(ctx->plan_d2z1);
  if (ctx->have_z2d1) cufftDestroy(ctx->plan_z2d1);
  cudaFree(ctx->ic_table);
  if (ctx->have_d2z2) cufftDestroy(ctx->plan_d2z2);
  cudaFree(ctx->spec_hc);
  cudaFree(ctx->spec_field);
  cudaFree(ctx->bins);
  cudaFree(ctx->maxbits);
  cudaFree(ctx->s2_counts);
  cudaFree(ctx->stage);
  if (ctx->stage_ev) cudaEventDestroy(ctx->stage_ev);
  delete ctx;
  return CF_OK;
}

int cf_get_info(const cf_ctx *ctx, cf_info *info) {
  CF_TRY(check_ctx(ctx));
  if (!info) {
    set_error("info is NULL");
    return CF_ERR_INVALID;
  }
  info->N = ctx->N;
  info->state_bytes = 16 * ctx->N3;  // 2N^3 doubles, or 4N^3 floats
  info->field_count = ctx->N3;
  info->hc_count = ctx->hc_count;
  info->s2_bins = ctx->s2_bins;
  info->shells = ctx->shells;
  info->psi_route = psi_route(ctx);
  return CF_OK;
}

int64_t cf_launch_count(const cf_ctx *ctx) { return ctx ? ctx->launches : -1; }

int cf_state_upload(cf_ctx *ctx, void *d_state, const double *h_xy, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_state, "d_state"));
  CF_TRY(check_ptr(h_xy, "h_xy", 8));
  CF_TRY(use_device(ctx));
  cudaStream_t st = (cudaStream_t)stream;
  const size_t bytes = 2 * (size_t)ctx->N3 * sizeof(double);
  if (ctx->p.precision == CF_FP64) {
    CF_TRY_CUDA(cudaMemcpyAsync(d_state, h_xy, bytes, cudaMemcpyHostToDevice, st));
    return CF_OK;
  }
  return state_upload_host(ctx, d_state, h_xy, st);
}

int cf_state_download(cf_ctx *ctx, double *h_xy, const void *d_state, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_state, "d_state"));
  CF_TRY(check_ptr(h_xy, "h_xy", 8));
  CF_TRY(use_device(ctx));
  cudaStream_t st = (cudaStream_t)stream;
  const size_t bytes = 2 * (size_t)ctx->N3 * sizeof(double);
  if (ctx->p.precision == CF_FP64) {
    CF_TRY_CUDA(cudaMemcpyAsync(h_xy, d_state, bytes, cudaMemcpyDeviceToHost, st));
    return CF_OK;
  }
  return state_download_host(ctx, h_xy, d_state, st);
}

int cf_state_import(cf_ctx *ctx, void *d_state, const double *d_xy, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_state, "d_state"));
  CF_TRY(check_ptr(d_xy, "d_xy", 8));
  CF_TRY(use_device(ctx));
  return state_import(ctx, d_state, d_xy, (cudaStream_t)stream);
}

int cf_state_export(cf_ctx *ctx, double *d_xy, const void *d_state, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_state, "d_state"));
  CF_TRY(check_ptr(d_xy, "d_xy", 8));
  CF_TRY(use_device(ctx));
  return state_export(ctx, d_xy, d_state, (cudaStream_t)stream);
}

int cf_set_R_fft(cf_ctx *ctx, const double *R_fft, int on_device, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(R_fft, "R_fft", 8));
  CF_TRY(use_device(ctx));
  return set_R_fft(ctx, R_fft, on_device, (cudaStream_t)stream);
}

int cf_set_psi(cf_ctx *ctx, const double *Psi, int on_device, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(Psi, "Psi", 8));
  if (ctx->p.equation != CF_EQ_FIXED_CURVATURE_FRW) {
    set_error("cf_set_psi: the context's equation is not CF_EQ_FIXED_CURVATURE_FRW");
    return CF_ERR_INVALID;
  }
  CF_TRY(use_device(ctx));
  return set_fixed_psi(ctx, Psi, on_device, (cudaStream_t)stream);
}

int cf_psi_fields(cf_ctx *ctx, double t, double *d_out, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_out, "d_out", 8));
  if (ctx->p.equation != CF_EQ_COMOVING_FRW || !ctx->R_fft) {
    set_error("cf_psi_fields: comoving-curvature equation with R_fft set required");
    return CF_ERR_INVALID;
  }
  CF_TRY(use_device(ctx));
  return psi_fields(ctx, t, d_out, (cudaStream_t)stream);
}

int cf_psi_stats(const cf_ctx *ctx, int64_t *refreshes, int64_t *reused) {
  CF_TRY(check_ctx(ctx));
  if (refreshes) *refreshes = ctx->psi_refreshes;
  if (reused) *reused = ctx->psi_reuses;
  return CF_OK;
}

int cf_psi_set_wait_test(cf_ctx *ctx, int extra_bytes, int64_t spin_limit) {
  CF_TRY(check_ctx(ctx));
  if (extra_bytes < 0 || extra_bytes % 16 || spin_limit < 1) {
    set_error("cf_psi_set_wait_test: extra_bytes must be a non-negative multiple of 16, spin_limit >= 1");
    return CF_ERR_INVALID;
  }
  CF_TRY(use_device(ctx));
  CF_TRY_CUDA(cudaDeviceSynchronize());  // no refresh of this context still running
  ctx->pc_tx_extra = extra_bytes;
  ctx->pc_spin_limit = spin_limit;
  if (ctx->psi_err_h) *ctx->psi_err_h = 0;
  return CF_OK;
}

int cf_rk4_steps(cf_ctx *ctx, void *d_state, double t0, double dt, int64_t step0, int64_t nsteps, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_state, "d_state"));
  if (nsteps < 0 || !std::isfinite(t0) || !std::isfinite(dt)) {
    set_error("nsteps must be >= 0 and t0, dt finite");
    return CF_ERR_INVALID;
  }
  CF_TRY(check_curvature(ctx));
  CF_TRY(use_device(ctx));
  return rk4_steps(ctx, d_state, t0, dt, step0, nsteps, (cudaStream_t)stream);
}

int cf_rhs(cf_ctx *ctx, const double *d_x, double *d_dxdt, double t, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_x, "d_x"));
  CF_TRY(check_ptr(d_dxdt, "d_dxdt"));
  const int eq = ctx->p.equation;
  if ((eq == CF_EQ_COMOVING_FRW || eq == CF_EQ_FIXED_CURVATURE_FRW || eq == CF_EQ_APPROX_COMOVING_FRW) &&
      ctx->p.precision != CF_FP64) {
    set_error("cf_rhs of a curvature-coupled equation needs a CF_FP64 context");
    return CF_ERR_UNSUPPORTED;
  }
  CF_TRY(check_curvature(ctx));
  CF_TRY(use_device(ctx));
  return rhs(ctx, d_x, d_dxdt, t, (cudaStream_t)stream);
}

int cf_scale_sum(cf_ctx *ctx, double *d_out, int n, const double *const *d_in, const double *alpha, int64_t len,
                 void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_out, "d_out", 8));
  if (n < 1 || n > 14 || !d_in || !alpha || len < 0) {
    set_error("cf_scale_sum: need 1 <= n <= 14, non-NULL inputs, len >= 0");
    return CF_ERR_INVALID;
  }
  for (int k = 0; k < n; ++k) CF_TRY(check_ptr(d_in[k], "d_in[k]", 8));
  CF_TRY(use_device(ctx));
  return scale_sum(ctx, d_out, n, d_in, alpha, len, (cudaStream_t)stream);
}

int cf_energy_density(cf_ctx *ctx, const void *d_state, double t, double *d_rho, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_state, "d_state"));
  CF_TRY(check_ptr(d_rho, "d_rho", 8));
  CF_TRY(check_curvature(ctx));
  CF_TRY(use_device(ctx));
  return energy_density(ctx, d_state, t, d_rho, (cudaStream_t)stream);
}

int cf_dot_energy_density(cf_ctx *ctx, const void *d_state, double t, double *d_out, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_state, "d_state"));
  CF_TRY(check_ptr(d_out, "d_out", 8));
  if (ctx->p.equation != CF_EQ_KG_FRW) {
    set_error("cf_dot_energy_density: CF_EQ_KG_FRW only (CudaKleinGordonEquationInFRW)");
    return CF_ERR_UNSUPPORTED;
  }
  CF_TRY(use_device(ctx));
  return dot_energy_density(ctx, d_state, t, d_out, (cudaStream_t)stream);
}

int cf_white_noise(cf_ctx *ctx, uint64_t seed, uint64_t offset, double *d_out, int64_t n, void *stream) {
  CF_TRY(check_ctx(ctx));
  if (n < 0) {
    set_error("cf_white_noise: n must be >= 0");
    return CF_ERR_INVALID;
  }
  if (n > 0) CF_TRY(check_ptr(d_out, "d_out", 8));
  CF_TRY(use_device(ctx));
  return white_noise(ctx, seed, offset, d_out, n, (cudaStream_t)stream);
}

static int check_table(const double *h, int64_t n, const char *what) {
  if (!h) {
    set_error("%s is NULL", what);
    return CF_ERR_INVALID;
  }
  for (int64_t i = 0; i < n; ++i)
    if (!std::isfinite(h[i])) {
      set_error("%s[%lld] is not finite", what, (long long)i);
      return CF_ERR_INVALID;
    }
  return CF_OK;
}

int cf_grf(cf_ctx *ctx, const double *d_white, const double *d_psi, double psi_scale, const double *h_sqrtP_s2,
           double *d_out, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_white, "d_white"));
  CF_TRY(check_ptr(d_out, "d_out"));
  if (d_psi) CF_TRY(check_ptr(d_psi, "d_psi", 8));
  if (!std::isfinite(psi_scale)) {
    set_error("psi_scale must be finite");
    return CF_ERR_INVALID;
  }
  CF_TRY(check_table(h_sqrtP_s2, ctx->s2_bins, "h_sqrtP_s2"));
  CF_TRY(use_device(ctx));
  return grf(ctx, d_white, d_psi, psi_scale, h_sqrtP_s2, d_out, (cudaStream_t)stream);
}

int cf_scale_modes(cf_ctx *ctx, const double *d_f, const double *h_scale_s2, double *d_out, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_f, "d_f"));
  CF_TRY(check_ptr(d_out, "d_out"));
  CF_TRY(check_table(h_scale_s2, ctx->s2_bins, "h_scale_s2"));
  CF_TRY(use_device(ctx));
  return scale_modes(ctx, d_f, h_scale_s2, d_out, (cudaStream_t)stream);
}

int cf_power_spectrum_s2(cf_ctx *ctx, const double *d_f, double *d_out, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_f, "d_f"));
  CF_TRY(check_ptr(d_out, "d_out", 8));
  CF_TRY(use_device(ctx));
  return power_spectrum_s2(ctx, d_f, d_out, (cudaStream_t)stream);
}

int cf_mode_power_spectrum_s2(cf_ctx *ctx, const void *d_state, double a_t, double *d_out, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_state, "d_state"));
  CF_TRY(check_ptr(d_out, "d_out", 8));
  if (!std::isfinite(a_t) || a_t == 0.0) {
    set_error("a_t must be finite and non-zero");
    return CF_ERR_INVALID;
  }
  CF_TRY(use_device(ctx));
  return mode_power_spectrum_s2(ctx, d_state, a_t, d_out, (cudaStream_t)stream);
}

int cf_density_spectrum_s2(cf_ctx *ctx, const void *d_state, double t, double *d_out, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_state, "d_state"));
  CF_TRY(check_ptr(d_out, "d_out", 8));
  CF_TRY(check_curvature(ctx));
  CF_TRY(use_device(ctx));
  return density_spectrum_s2(ctx, d_state, t, d_out, (cudaStream_t)stream);
}

int cf_density_slices(cf_ctx *ctx, const void *d_state, double t, double *d_slice, double *d_axis_average,
                      void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_state, "d_state"));
  if (d_slice) CF_TRY(check_ptr(d_slice, "d_slice", 8));
  if (d_axis_average) CF_TRY(check_ptr(d_axis_average, "d_axis_average", 8));
  CF_TRY(check_curvature(ctx));
  CF_TRY(use_device(ctx));
  return density_slices(ctx, d_state, t, d_slice, d_axis_average, (cudaStream_t)stream);
}

int cf_wkb_create(cf_ctx *ctx, const double *d_state, double t_i, cf_wkb **out, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_state, "d_state"));
  if (!out || !std::isfinite(t_i) || !(t_i > 0)) {
    set_error("cf_wkb_create: need out and a finite t_i > 0");
    return CF_ERR_INVALID;
  }
  *out = nullptr;
  CF_TRY(use_device(ctx));
  return wkb_create(ctx, d_state, t_i, out, (cudaStream_t)stream);
}

int cf_wkb_evaluate(cf_wkb *wkb, double t, double *d_out, void *stream) {
  if (!wkb) {
    set_error("NULL WKB handle");
    return CF_ERR_INVALID;
  }
  CF_TRY(check_ptr(d_out, "d_out"));
  if (!std::isfinite(t) || !(t > 0)) {
    set_error("cf_wkb_evaluate: t must be finite and > 0");
    return CF_ERR_INVALID;
  }
  CF_TRY(use_device(wkb_ctx(wkb)));
  return wkb_evaluate(wkb, t, d_out, (cudaStream_t)stream);
}

int cf_wkb_destroy(cf_wkb *wkb) {
  wkb_destroy(wkb);
  return CF_OK;
}

int cf_s2_to_shells(cf_ctx *ctx, double *d_shells, int64_t *d_counts, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_shells, "d_shells", 8));
  CF_TRY(use_device(ctx));
  return s2_to_shells(ctx, d_shells, d_counts, (cudaStream_t)stream);
}

int cf_s2_counts(cf_ctx *ctx, int64_t *d_counts, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_counts, "d_counts", 8));
  CF_TRY(use_device(ctx));
  return s2_counts(ctx, d_counts, (cudaStream_t)stream);
}

int cf_adjoint_create(cf_ctx *ctx, int64_t nsteps, int64_t checkpoint_every, cf_adjoint **out) {
  CF_TRY(check_ctx(ctx));
  if (!out) {
    set_error("out is NULL");
    return CF_ERR_INVALID;
  }
  *out = nullptr;
  CF_TRY(use_device(ctx));
  cf_adjoint *a = nullptr;
  int s = adjoint_create(ctx, nsteps, checkpoint_every, &a);
  if (s != CF_OK) {
    adjoint_destroy(a);
    return s;
  }
  *out = a;
  return CF_OK;
}

int cf_adjoint_destroy(cf_adjoint *adj) {
  adjoint_destroy(adj);
  return CF_OK;
}

int cf_adjoint_forward(cf_adjoint *adj, void *d_state, double t0, double dt, void *stream) {
  if (!adj) {
    set_error("NULL adjoint");
    return CF_ERR_INVALID;
  }
  CF_TRY(check_ptr(d_state, "d_state"));
  CF_TRY(use_device(adjoint_ctx(adj)));
  return adjoint_forward(adj, d_state, t0, dt, (cudaStream_t)stream);
}

int cf_adjoint_shell_log_loss(cf_adjoint *adj, const void *d_state, const double *h_target_shells, double rel_floor,
                              double *h_loss, void *stream) {
  if (!adj || !h_target_shells) {
    set_error("NULL adjoint or target");
    return CF_ERR_INVALID;
  }
  CF_TRY(check_ptr(d_state, "d_state"));
  CF_TRY(use_device(adjoint_ctx(adj)));
  return adjoint_shell_log_loss(adj, d_state, h_target_shells, rel_floor, h_loss, (cudaStream_t)stream);
}

int cf_adjoint_set_lambda(cf_adjoint *adj, const double *d_lambda, double dL_dm_direct, void *stream) {
  if (!adj) {
    set_error("NULL adjoint");
    return CF_ERR_INVALID;
  }
  CF_TRY(check_ptr(d_lambda, "d_lambda"));
  CF_TRY(use_device(adjoint_ctx(adj)));
  return adjoint_set_lambda(adj, d_lambda, dL_dm_direct, (cudaStream_t)stream);
}

int cf_adjoint_backward(cf_adjoint *adj, double *d_lambda0, double *h_dL_dm, void *stream) {
  if (!adj) {
    set_error("NULL adjoint");
    return CF_ERR_INVALID;
  }
  CF_TRY(use_device(adjoint_ctx(adj)));
  return adjoint_backward(adj, d_lambda0, h_dL_dm, (cudaStream_t)stream);
}

int cf_field_from_shell_amplitudes(cf_ctx *ctx, const double *d_xi_hc, const double *d_sqrtP_s2,
                                   const double *h_theta, int ngroups, int shells_per_group, double *d_phi,
                                   void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_xi_hc, "d_xi_hc", 8));
  CF_TRY(check_ptr(d_sqrtP_s2, "d_sqrtP_s2", 8));
  CF_TRY(check_ptr(d_phi, "d_phi", 8));
  if (!h_theta || ngroups < 1 || ngroups > 1024 || shells_per_group < 1) {
    set_error("need theta, 1 <= ngroups <= 1024, shells_per_group >= 1");
    return CF_ERR_INVALID;
  }
  for (int g = 0; g < ngroups; ++g)
    if (!(h_theta[g] >= 0)) {
      set_error("theta must be non-negative");
      return CF_ERR_INVALID;
    }
  CF_TRY(use_device(ctx));
  return field_from_shell_amplitudes(ctx, d_xi_hc, d_sqrtP_s2, h_theta, ngroups, shells_per_group, d_phi,
                                     (cudaStream_t)stream);
}

int cf_shell_amplitude_gradient(cf_ctx *ctx, const double *d_lambda_phi, const double *d_xi_hc,
                                const double *d_sqrtP_s2, const double *h_theta, int ngroups, int shells_per_group,
                                double *h_grad, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_lambda_phi, "d_lambda_phi", 8));
  CF_TRY(check_ptr(d_xi_hc, "d_xi_hc", 8));
  CF_TRY(check_ptr(d_sqrtP_s2, "d_sqrtP_s2", 8));
  if (!h_theta || !h_grad || ngroups < 1 || ngroups > 1024 || shells_per_group < 1) {
    set_error("need theta, grad, 1 <= ngroups <= 1024, shells_per_group >= 1");
    return CF_ERR_INVALID;
  }
  for (int g = 0; g < ngroups; ++g)
    if (!(h_theta[g] > 0)) {
      set_error("theta must be positive for the gradient");
      return CF_ERR_INVALID;
    }
  CF_TRY(use_device(ctx));
  return shell_amplitude_gradient(ctx, d_lambda_phi, d_xi_hc, d_sqrtP_s2, h_theta, ngroups, shells_per_group, h_grad,
                                  (cudaStream_t)stream);
}

int cf_profile_enable(cf_ctx *ctx, int on) {
  CF_TRY(check_ctx(ctx));
  ctx->prof_on = on != 0;
  return CF_OK;
}

int cf_profile_read(cf_ctx *ctx, cf_profile *out) {
  CF_TRY(check_ctx(ctx));
  if (!out) {
    set_error("out is NULL");
    return CF_ERR_INVALID;
  }
  CF_TRY(use_device(ctx));
  prof_drain(ctx);
  for (int k = 0; k < CF_PROF_KINDS; ++k) {
    out->launches[k] = ctx->prof_launches[k];
    out->ms[k] = ctx->prof_ms[k];
  }
  return CF_OK;
}

int cf_profile_reset(cf_ctx *ctx) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(use_device(ctx));
  prof_drain(ctx);
  for (int k = 0; k < CF_PROF_KINDS; ++k) {
    ctx->prof_launches[k] = 0;
    ctx->prof_ms[k] = 0.0;
  }
  return CF_OK;
}

int cf_check_finite(cf_ctx *ctx, const void *d_state, int64_t *h_bad, void *stream) {
  CF_TRY(check_ctx(ctx));
  CF_TRY(check_ptr(d_state, "d_state"));
  CF_TRY(use_device(ctx));
  return check_finite(ctx, d_state, h_bad, (cudaStream_t)stream);
}

}  // extern "C"
