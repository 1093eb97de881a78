// cf_approx.cu -- the curvature inputs of the fixed-curvature and the
// approximate comoving-curvature equations.
//
// Fixed curvature (CudaFixedCurvatureEquationInFRW, src/equations_cuda.cu:107-136,
// :645-675): a time-independent Psi(x) (the workspace's Psi) enters the
// right-hand side as e^{2Psi} and e^{4Psi}; it is kept as one plane of
// e^{2Psi} - 1 in the storage type, the form the stage kernels read.
//
// Approximate comoving curvature (CudaApproximateComovingCurvatureEquationInFRW,
// src/equations_cuda.cu:299-329, :764-809): Psi and dPsi/dt are synthesised on
// a coarse M^3 grid from the modes of R_fft that the M grid holds
// (compute_cutoff_fouriers, src/fdm3d_cuda.cu:118-141, :206-219), with the
// transfer functions of the comoving equation (src/equations_cuda.cu:209-259)
// and a 3-D Z2D of size M, and every lattice site reads the coarse site
// ((a + s/2) % N) / s, s = N / M, in each axis.  The stage kernels take, per
// coarse site, the 4 words (2Psi + 2Psi^2, 4Psi + 8Psi^2, dPsi/dt, 0): the
// reference's quadratic stand-ins for e^{2Psi} - 1 and e^{4Psi} - 1, and dPsi/dt.
// The coarse table is M^3 x 4 words (M = 64: 4 MB in FP32), so the per-site
// gathers hit L2; HBM traffic per site-update is that of the uncoupled equation.

#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "cf_internal.cuh"

namespace cfb {

// ---- fixed curvature ------------------------------------------------------

template <typename S>
__global__ void k_fixed_e2m1(const double *__restrict__ Psi, S *__restrict__ out, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = (S)expm1(2.0 * Psi[i]);
}

int set_fixed_psi(cf_ctx *ctx, const double *Psi, int on_device, cudaStream_t st) {
  const long long n = ctx->N3;
  if (!ctx->fixed_e2m1) {
    if (cudaMalloc(&ctx->fixed_e2m1, (size_t)n * ctx->word) != cudaSuccess) {
      cudaGetLastError();
      set_error("cudaMalloc of the fixed Psi plane failed");
      return CF_ERR_NOMEM;
    }
  }
  const double *src = Psi;
  double *tmp = nullptr;
  if (!on_device) {
    if (cudaMallocAsync((void **)&tmp, (size_t)n * 8, st) != cudaSuccess) {
      cudaGetLastError();
      set_error("cudaMallocAsync Psi staging failed");
      return CF_ERR_NOMEM;
    }
    CF_TRY_CUDA(cudaMemcpyAsync(tmp, Psi, (size_t)n * 8, cudaMemcpyHostToDevice, st));
    src = tmp;
  }
  const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16);
  if (ctx->word == 8)
    k_fixed_e2m1<double><<<blocks, 256, 0, st>>>(src, (double *)ctx->fixed_e2m1, n);
  else
    k_fixed_e2m1<float><<<blocks, 256, 0, st>>>(src, (float *)ctx->fixed_e2m1, n);
  const cudaError_t e = cudaGetLastError();
  if (tmp) cudaFreeAsync(tmp, st);
  if (e != cudaSuccess) {
    set_error("kernel launch failed: %s", cudaGetErrorString(e));
    return CF_ERR_CUDA;
  }
  ctx->launches++;
  return CF_OK;
}

// ---- approximate comoving curvature ---------------------------------------

// M-grid modes of the N-grid HC array `in`, scaled by (M/N)^3: modes a, b < M/2
// are taken from a, b, modes a, b >= M/2 from N - (M - a), N - (M - b); c <= M/2
// from c (the reference's mapping, src/fdm3d_cuda.cu:118-141).
__global__ void k_ap_cutoff(const double *__restrict__ in, double *__restrict__ out, int N, int M, double scaling) {
  const long long nhM = M / 2 + 1, nhN = N / 2 + 1;
  const long long total = (long long)M * M * nhM;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
    const int c = (int)(i % nhM);
    const int b = (int)((i / nhM) % M);
    const int a = (int)(i / (nhM * M));
    const long long aN = a < M / 2 ? a : N - (M - a);
    const long long bN = b < M / 2 ? b : N - (M - b);
    const long long o = (aN * N + bN) * nhN + c;
    out[2 * i] = in[2 * o] * scaling;
    out[2 * i + 1] = in[2 * o + 1] * scaling;
  }
}

// Psi_k and dPsi/dt_k on the M grid (the comoving transfer functions,
// src/equations_cuda.cu:209-259, with the lattice size M): for s^2 > 0 and
// x = sqrt(s^2) factor, T_Psi = 2 (sin x - x cos x) / x^3 / M^3 and
// T_dPsi = H 2 (3 x cos x + (x^2 - 3) sin x) / x^3 / M^3; the s^2 = 0 mode is zero.
__global__ void k_ap_transfer(const double *__restrict__ R, double *__restrict__ Pk, double *__restrict__ Dk, int M,
                              double factor, double H_t) {
  const long long nh = M / 2 + 1;
  const long long total = (long long)M * M * nh;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const int half = M / 2;
  const double M3 = (double)((long long)M * M * M);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
    const int c = (int)(i % nh);
    const int b = (int)((i / nh) % M);
    const int a = (int)(i / (nh * M));
    const int as = a < half ? a : M - a;
    const int bs = b < half ? b : M - b;
    const int s2 = as * as + bs * bs + c * c;
    if (s2 == 0) {
      Pk[2 * i] = Pk[2 * i + 1] = 0.0;
      Dk[2 * i] = Dk[2 * i + 1] = 0.0;
      continue;
    }
    const double x = sqrt((double)s2) * factor;
    double sv, cv;
    sincos(x, &sv, &cv);
    const double common = 2.0 / (x * x * x) / M3;
    const double tp = (sv - x * cv) * common;
    const double td = H_t * (3 * x * cv + (x * x - 3.0) * sv) * common;
    const double rr = R[2 * i], ri = R[2 * i + 1];
    Pk[2 * i] = rr * tp;
    Pk[2 * i + 1] = ri * tp;
    Dk[2 * i] = rr * td;
    Dk[2 * i + 1] = ri * td;
  }
}

// Coarse table: per coarse site (2P + 2P^2, 4P + 8P^2, D, 0) from Psi = P and
// dPsi/dt = D (the factors of src/equations_cuda.cu:319-321, less their 1).
template <typename S>
__global__ void k_ap_table(const double *__restrict__ f, S *__restrict__ tab, long long M3) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < M3; i += stride) {
    const double P = f[i], D = f[M3 + i];
    tab[4 * i] = (S)(2.0 * P + 2.0 * P * P);
    tab[4 * i + 1] = (S)(4.0 * P + 8.0 * P * P);
    tab[4 * i + 2] = (S)D;
    tab[4 * i + 3] = (S)0;
  }
}

static int ap_alloc(void **p, size_t bytes, const char *what) {
  if (cudaMalloc(p, bytes) != cudaSuccess) {
    cudaGetLastError();
    set_error("cudaMalloc of %s (%zu bytes) failed", what, bytes);
    return CF_ERR_NOMEM;
  }
  return CF_OK;
}

static int ensure_approx(cf_ctx *ctx) {
  if (ctx->ap_R) return CF_OK;
  const long long M = ctx->p.M, N = ctx->N;
  const size_t hcM = (size_t)(2 * M * M * (M / 2 + 1));
  const size_t M3 = (size_t)(M * M * M);
  // (each piece once: a call after a failed allocation resumes where it stopped)
  if (!ctx->ap_hc) CF_TRY(ap_alloc((void **)&ctx->ap_hc, 2 * hcM * sizeof(double), "the coarse transfer outputs"));
  if (!ctx->ap_f) CF_TRY(ap_alloc((void **)&ctx->ap_f, 2 * M3 * sizeof(double), "the coarse fields"));
  if (!ctx->ap_cmap) CF_TRY(ap_alloc((void **)&ctx->ap_cmap, (size_t)N * sizeof(int), "the coarse index map"));
  for (auto &s : ctx->ap_slot)
    if (!s.tab) CF_TRY(ap_alloc(&s.tab, 4 * M3 * ctx->word, "a coarse table"));
  if (!ctx->have_plan_ap) {
    int n[3] = {(int)M, (int)M, (int)M};
    CF_TRY_CUFFT(
        cufftPlanMany(&ctx->plan_ap, 3, n, nullptr, 1, (int)(hcM / 2), nullptr, 1, (int)M3, CUFFT_Z2D, 2));
    ctx->have_plan_ap = true;
  }
  // lattice index -> coarse index, the same in every axis
  const long long s = N / M, h = s / 2;
  std::vector<int> cmap((size_t)N);
  for (long long i = 0; i < N; ++i) cmap[(size_t)i] = (int)(((i + h) % N) / s);
  CF_TRY_CUDA(cudaMemcpy(ctx->ap_cmap, cmap.data(), (size_t)N * sizeof(int), cudaMemcpyHostToDevice));
  // ap_R last: it marks the buffers complete
  CF_TRY(ap_alloc((void **)&ctx->ap_R, hcM * sizeof(double), "the coarse R_fft"));
  return CF_OK;
}

void approx_release(cf_ctx *ctx) {
  cudaFree(ctx->ap_R);
  cudaFree(ctx->ap_hc);
  cudaFree(ctx->ap_f);
  cudaFree(ctx->ap_cmap);
  for (auto &s : ctx->ap_slot) cudaFree(s.tab);
  if (ctx->have_plan_ap) cufftDestroy(ctx->plan_ap);
  cudaFree(ctx->fixed_e2m1);
}

int approx_set_R(cf_ctx *ctx, const double *d_R, cudaStream_t st) {
  CF_TRY(ensure_approx(ctx));
  const long long M = ctx->p.M, N = ctx->N;
  const long long modes = M * M * (M / 2 + 1);
  const double sd = (double)N / (double)M;
  const unsigned blocks = (unsigned)std::min<long long>((modes + 255) / 256, 148LL * 8);
  k_ap_cutoff<<<blocks, 256, 0, st>>>(d_R, ctx->ap_R, (int)N, (int)M, 1.0 / (sd * sd * sd));
  CF_LAUNCHED(ctx);
  for (auto &s : ctx->ap_slot) s.valid = false;
  return CF_OK;
}

int approx_at(cf_ctx *ctx, double t, cudaStream_t st, const void **tab) {
  for (auto &s : ctx->ap_slot) {
    if (s.valid && s.t == t) {
      s.stamp = ++ctx->ap_clock;
      *tab = s.tab;
      return CF_OK;
    }
  }
  ApproxSlot *v = &ctx->ap_slot[0];
  for (auto &s : ctx->ap_slot)
    if (!s.valid || s.stamp < v->stamp) v = &s;
  const long long M = ctx->p.M;
  const long long modes = M * M * (M / 2 + 1), M3 = M * M * M;
  const double eta_t = cosmo_eta(ctx->p, t);
  const double H_t = cosmo_H(ctx->p, t);
  const double factor = (2 * 3.14159265358979323846 / ctx->p.L) * eta_t / sqrt(3);
  {
    ProfScope ps(ctx, CF_PROF_PSI_TRANSFER, st);
    const unsigned blocks = (unsigned)std::min<long long>((modes + 255) / 256, 148LL * 8);
    k_ap_transfer<<<blocks, 256, 0, st>>>(ctx->ap_R, ctx->ap_hc, ctx->ap_hc + 2 * modes, (int)M, factor, H_t);
    CF_LAUNCHED(ctx);
  }
  {
    ProfScope ps(ctx, CF_PROF_PSI_FFT, st);
    CF_TRY_CUFFT(cufftSetStream(ctx->plan_ap, st));
    CF_TRY_CUFFT(cufftExecZ2D(ctx->plan_ap, (cufftDoubleComplex *)ctx->ap_hc, ctx->ap_f));
  }
  {
    ProfScope ps(ctx, CF_PROF_PSI_TRANSFER, st);
    const unsigned blocks = (unsigned)std::min<long long>((M3 + 255) / 256, 148LL * 8);
    if (ctx->word == 8)
      k_ap_table<double><<<blocks, 256, 0, st>>>(ctx->ap_f, (double *)v->tab, M3);
    else
      k_ap_table<float><<<blocks, 256, 0, st>>>(ctx->ap_f, (float *)v->tab, M3);
    CF_LAUNCHED(ctx);
  }
  v->t = t;
  v->valid = true;
  v->stamp = ++ctx->ap_clock;
  *tab = v->tab;
  return CF_OK;
}

}  // namespace cfb
