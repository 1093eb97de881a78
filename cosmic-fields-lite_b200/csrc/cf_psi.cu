// cf_psi.cu -- Psi(x,t), dPsi/dt(x,t) for the comoving-curvature equation.
//
// The reference recomputes both fields inside every right-hand-side call: a
// transfer-function kernel over the half-complex grid followed by two in-place
// cuFFT Z2D, with the two HC buffers allocated and freed per call
// (src/equations_cuda.cu:678-731, kernel :210-253).  RK4 evaluates the
// right-hand side at only three distinct times per step (t, t+dt/2 twice, t+dt)
// and t+dt is the next step's t, so here the fields are cached per stage time
// in three persistent slots and refreshed -- transfer kernel + ONE batched
// C2R of both fields -- only when a stage asks for a time no slot holds.
//
// Storage follows the context precision: FP64 (Z2D) or FP32 (C2R); the
// transfer function is always evaluated in FP64.

#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>

#include "cf_internal.cuh"

namespace cfb {

// The transfer functions depend on the mode only through the integer s^2 =
// i^2 + j^2 + k^2, so they are evaluated once per distinct s^2 (3(N/2)^2 + 1
// values, e.g. 196,609 at N = 512 against 33.7M half-complex modes) into a
// table that stays in L2, with exactly the per-mode expression of the
// reference (src/equations_cuda.cu:210-253; src/equations.cpp:141-183):
//   x = sqrt(s^2) * factor, common = 2 / x^3 / N^3,
//   T_Psi  = (sin x - x cos x) * common,
//   T_dPsi = H (3 x cos x + (x^2 - 3) sin x) * common,   T(0) = 0.
__global__ void k_transfer_table(double *__restrict__ table, long long nb, int N, double factor, double H_t) {
  const double inv_n3 = 1.0 / ((double)N * (double)N * (double)N);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long s2 = (long long)blockIdx.x * blockDim.x + threadIdx.x; s2 < nb; s2 += stride) {
    double tp = 0.0, td = 0.0;
    if (s2 != 0) {
      const double x = sqrt((double)s2) * factor;
      double sv, cv;
      sincos(x, &sv, &cv);
      const double common = 2.0 / (x * x * x) * inv_n3;
      tp = (sv - x * cv) * common;
      td = H_t * (3 * x * cv + (x * x - 3.0) * sv) * common;
    }
    table[2 * s2] = tp;
    table[2 * s2 + 1] = td;
  }
}

// Psi_k = R_k T_Psi(s^2), dPsi_k = R_k T_dPsi(s^2); output: two HC arrays of the
// storage complex type, consecutive.  Grid: y/z = the (a, b) row, threads along c
// (no index division; each complex entry is one 8- or 16-byte access).
template <typename S>
struct Cplx;
template <>
struct Cplx<float> {
  using T = float2;
};
template <>
struct Cplx<double> {
  using T = double2;
};

template <typename S>
__global__ void __launch_bounds__(256) k_transfer(const S *__restrict__ R, S *__restrict__ out,
                                                  const double *__restrict__ table, int N, long long hc_pairs) {
  using C = typename Cplx<S>::T;
  const int nh = N / 2 + 1;
  const int a = blockIdx.z, b = blockIdx.y;
  const int as = (a <= N / 2) ? a : N - a;
  const int bs = (b <= N / 2) ? b : N - b;
  const int ab2 = as * as + bs * bs;
  const long long row = ((long long)a * N + b) * nh;
  const C *Rr = reinterpret_cast<const C *>(R) + row;
  C *op = reinterpret_cast<C *>(out) + row;
  C *od = reinterpret_cast<C *>(out) + hc_pairs + row;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nh; c += gridDim.x * blockDim.x) {
    const int s2 = ab2 + c * c;
    const double tp = table[2 * s2], td = table[2 * s2 + 1];
    const C r = Rr[c];
    const double rr = (double)r.x, ri = (double)r.y;
    C p, d;
    p.x = (S)(rr * tp);
    p.y = (S)(ri * tp);
    d.x = (S)(rr * td);
    d.y = (S)(ri * td);
    op[c] = p;
    od[c] = d;
  }
}

template <typename S>
__global__ void k_copy_convert(const double *__restrict__ in, S *__restrict__ out, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = (S)in[i];
}

int ensure_psi(cf_ctx *ctx) {
  if (ctx->have_plan_psi) return CF_OK;
  const int N = (int)ctx->N;
  const size_t w = ctx->word;
  const size_t hc_bytes = (size_t)ctx->hc_count * w;
  if (!ctx->R_fft) {
    if (cudaMalloc(&ctx->R_fft, hc_bytes) != cudaSuccess) {
      set_error("cudaMalloc R_fft (%zu bytes) failed", hc_bytes);
      return CF_ERR_NOMEM;
    }
    CF_TRY_CUDA(cudaMemset(ctx->R_fft, 0, hc_bytes));
  }
  if (cudaMalloc(&ctx->psi_table, 2 * (size_t)ctx->s2_bins * sizeof(double)) != cudaSuccess) {
    set_error("cudaMalloc transfer table failed");
    return CF_ERR_NOMEM;
  }
  if (cudaMalloc(&ctx->psi_hc, 2 * hc_bytes) != cudaSuccess) {
    set_error("cudaMalloc Psi transfer buffers (%zu bytes) failed", 2 * hc_bytes);
    return CF_ERR_NOMEM;
  }
  for (auto &s : ctx->slot) {
    if (cudaMalloc(&s.psi, 2 * (size_t)ctx->N3 * w) != cudaSuccess) {
      set_error("cudaMalloc Psi slot failed");
      return CF_ERR_NOMEM;
    }
    s.dpsi = (char *)s.psi + (size_t)ctx->N3 * w;
    s.valid = false;
  }
  long long n[3] = {N, N, N};
  long long inembed[3] = {N, N, N / 2 + 1};
  long long onembed[3] = {N, N, N};
  const long long idist = ctx->hc_count / 2;  // complex elements per HC array
  const long long odist = ctx->N3;
  CF_TRY_CUFFT(cufftCreate(&ctx->plan_psi));
  size_t work = 0;
  CF_TRY_CUFFT(cufftMakePlanMany64(ctx->plan_psi, 3, n, inembed, 1, idist, onembed, 1, odist,
                                   w == 8 ? CUFFT_Z2D : CUFFT_C2R, 2, &work));
  ctx->have_plan_psi = true;
  return CF_OK;
}

int psi_at(cf_ctx *ctx, double t, cudaStream_t st, const void **psi, const void **dpsi) {
  CF_TRY(ensure_psi(ctx));
  for (auto &s : ctx->slot) {
    if (s.valid && s.t == t) {
      s.stamp = ++ctx->slot_clock;
      *psi = s.psi;
      *dpsi = s.dpsi;
      return CF_OK;
    }
  }
  // refresh the least recently used slot
  PsiSlot *v = &ctx->slot[0];
  for (auto &s : ctx->slot)
    if (!s.valid || s.stamp < v->stamp) v = &s;
  const double eta_t = cosmo_eta(ctx->p, t);
  const double H_t = cosmo_H(ctx->p, t);
  const double factor = (2 * 3.14159265358979323846 / ctx->p.L) * eta_t / sqrt(3);
  const long long pairs = ctx->hc_count / 2;
  CF_TRY_CUFFT(cufftSetStream(ctx->plan_psi, st));
  {
    ProfScope ps(ctx, CF_PROF_PSI_TRANSFER, st);
    unsigned tb = (unsigned)std::min<long long>((ctx->s2_bins + 255) / 256, 148LL * 8);
    k_transfer_table<<<tb, 256, 0, st>>>(ctx->psi_table, ctx->s2_bins, (int)ctx->N, factor, H_t);
    CF_LAUNCHED(ctx);
    const int nh = (int)ctx->N / 2 + 1;
    const dim3 tg((unsigned)((nh + 255) / 256), (unsigned)ctx->N, (unsigned)ctx->N);
    if (ctx->word == 8)
      k_transfer<double><<<tg, 256, 0, st>>>((const double *)ctx->R_fft, (double *)ctx->psi_hc, ctx->psi_table,
                                             (int)ctx->N, pairs);
    else
      k_transfer<float><<<tg, 256, 0, st>>>((const float *)ctx->R_fft, (float *)ctx->psi_hc, ctx->psi_table,
                                            (int)ctx->N, pairs);
    CF_LAUNCHED(ctx);
  }
  {
    ProfScope ps(ctx, CF_PROF_PSI_FFT, st);
    if (ctx->word == 8)
      CF_TRY_CUFFT(cufftExecZ2D(ctx->plan_psi, (cufftDoubleComplex *)ctx->psi_hc, (cufftDoubleReal *)v->psi));
    else
      CF_TRY_CUFFT(cufftExecC2R(ctx->plan_psi, (cufftComplex *)ctx->psi_hc, (cufftReal *)v->psi));
  }
  v->t = t;
  v->valid = true;
  v->stamp = ++ctx->slot_clock;
  *psi = v->psi;
  *dpsi = v->dpsi;
  return CF_OK;
}

int set_R_fft(cf_ctx *ctx, const double *R_fft, int on_device, cudaStream_t st) {
  const size_t hc = (size_t)ctx->hc_count;
  const size_t w = ctx->word;
  if (!ctx->R_fft) {
    if (cudaMalloc(&ctx->R_fft, hc * w) != cudaSuccess) {
      set_error("cudaMalloc R_fft failed");
      return CF_ERR_NOMEM;
    }
  }
  const double *src = R_fft;
  double *tmp = nullptr;
  if (!on_device) {
    if (w == 8) {
      CF_TRY_CUDA(cudaMemcpyAsync(ctx->R_fft, R_fft, hc * 8, cudaMemcpyHostToDevice, st));
      src = nullptr;
    } else {
      if (cudaMallocAsync((void **)&tmp, hc * 8, st) != cudaSuccess) {
        set_error("cudaMallocAsync R_fft staging failed");
        return CF_ERR_NOMEM;
      }
      CF_TRY_CUDA(cudaMemcpyAsync(tmp, R_fft, hc * 8, cudaMemcpyHostToDevice, st));
      src = tmp;
    }
  }
  if (src) {
    unsigned blocks = (unsigned)std::min<size_t>((hc + 255) / 256, 148 * 32);
    if (w == 8) {
      CF_TRY_CUDA(cudaMemcpyAsync(ctx->R_fft, src, hc * 8, cudaMemcpyDeviceToDevice, st));
    } else {
      k_copy_convert<float><<<blocks, 256, 0, st>>>(src, (float *)ctx->R_fft, (long long)hc);
      CF_LAUNCHED(ctx);
    }
  }
  if (tmp) CF_TRY_CUDA(cudaFreeAsync(tmp, st));
  for (auto &s : ctx->slot) s.valid = false;
  return CF_OK;
}

}  // namespace cfb
