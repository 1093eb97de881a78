// cf_init.cu -- initial conditions on the device: white noise, (inhomogeneous)
// Gaussian random fields and Fourier-mode scaling.
//
// The reference builds every initial field on the host, once, before stepping
// (src/initializer.hpp:33-301): N^3 sequential normal draws, a 3-D FFTW r2c, a
// per-mode multiply by sqrt(P(|k|)) and a c2r (generate_inhomogeneous_gaussian_random_field,
// src/random_field.cpp:36-83), and the same transform pair around a per-mode kernel
// (compute_field_with_scaled_fourier_modes, src/fdm3d.cpp:76-102).  Here each is two
// streaming passes around the context's cuFFT D2Z / Z2D.  The spectrum enters as a
// table over s^2 (a mode's |k| depends only on s^2), evaluated by the caller on the
// host with its own spectrum function -- the same value per mode as the reference's
// per-mode call.
//
// White noise: Philox4x32-10 (J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11) -- a counter-based
// generator, so element i is a pure function of (seed, offset + i) and the stream
// can be produced by any number of threads and calls; Box-Muller on two 53-bit
// uniforms per counter.

#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>

#include "cf_internal.cuh"

namespace cfb {

// ---- Philox4x32-10 ----------------------------------------------------------
struct U4 {
  unsigned x, y, z, w;
};

__device__ __forceinline__ U4 philox_round(U4 c, unsigned k0, unsigned k1) {
  const unsigned M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const unsigned hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
  const unsigned hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
  return U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
}

__device__ __forceinline__ U4 philox4x32_10(U4 c, unsigned k0, unsigned k1) {
  const unsigned W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    c = philox_round(c, k0, k1);
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// Thread t makes the pair of deviates of counter ctr0 + t (elements 2 ctr, 2 ctr + 1)
// and stores the ones inside [offset, offset + n).
__global__ void k_white_noise(unsigned long long seed, unsigned long long offset, long long n, double *__restrict__ out) {
  const unsigned long long ctr0 = offset >> 1;
  const unsigned long long pairs = ((offset + (unsigned long long)n + 1) >> 1) - ctr0;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < pairs; t += stride) {
    const unsigned long long ctr = ctr0 + t;
    const U4 r = philox4x32_10(U4{(unsigned)ctr, (unsigned)(ctr >> 32), 0u, 0u}, (unsigned)seed,
                               (unsigned)(seed >> 32));
    const unsigned long long a = ((unsigned long long)r.x << 32 | r.y) >> 11;
    const unsigned long long b = ((unsigned long long)r.z << 32 | r.w) >> 11;
    const double u1 = ((double)a + 0.5) * 0x1.0p-53;  // (0, 1): log(u1) finite
    const double u2 = (double)b * 0x1.0p-53;          // [0, 1)
    const double rad = sqrt(-2.0 * log(u1));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    const unsigned long long g0 = 2 * ctr;  // global element index of the cos deviate
    if (g0 >= offset && g0 < offset + (unsigned long long)n) out[g0 - offset] = rad * c;
    if (g0 + 1 >= offset && g0 + 1 < offset + (unsigned long long)n) out[g0 + 1 - offset] = rad * s;
  }
}

// ---- Gaussian random fields ---------------------------------------------------

// out = w / N^3 * exp(psi_scale * Psi)   (src/random_field.cpp:43-50)
__global__ void k_grf_modulate(const double *w, const double *__restrict__ psi, double psi_scale, double *out,
                               long long N3) {  // out may be w
  const double inv = 1.0 / (double)N3;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N3; i += stride) {
    const double v = inv * w[i];
    out[i] = psi ? v * exp(psi_scale * psi[i]) : v;
  }
}

// Every HC mode times table[s^2] (the per-mode loops of src/random_field.cpp:59-72 and
// src/fdm3d.cpp:86-99; s^2 from the lattice momenta a or a - N, b or b - N, c <= N/2).
__global__ void k_scale_by_s2(double *__restrict__ hc, const double *__restrict__ table, int N) {
  const long long nh = N / 2 + 1;
  const long long total = (long long)N * N * nh;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
    const int c = (int)(i % nh);
    const int b = (int)((i / nh) % N);
    const int a = (int)(i / (nh * N));
    const long long as = a <= N / 2 ? a : N - a, bs = b <= N / 2 ? b : N - b;
    const double f = table[as * as + bs * bs + (long long)c * c];
    double2 v = reinterpret_cast<double2 *>(hc)[i];
    v.x *= f;
    v.y *= f;
    reinterpret_cast<double2 *>(hc)[i] = v;
  }
}

static unsigned blocks_for(long long n) { return (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16); }

// The s^2 table on the device (ctx->ic_table), the HC scratch and both plans.
static int ensure_init(cf_ctx *ctx, const double *h_table, cudaStream_t st) {
  CF_TRY(ensure_spectrum_scratch(ctx, 1));
  if (!ctx->ic_table) {
    if (cudaMalloc(&ctx->ic_table, (size_t)ctx->s2_bins * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      set_error("cudaMalloc of the s^2 table failed");
      return CF_ERR_NOMEM;
    }
  }
  if (!ctx->have_z2d1) {
    const int N = (int)ctx->N;
    CF_TRY_CUFFT(cufftPlan3d(&ctx->plan_z2d1, N, N, N, CUFFT_Z2D));
    ctx->have_z2d1 = true;
  }
  CF_TRY_CUDA(cudaMemcpyAsync(ctx->ic_table, h_table, (size_t)ctx->s2_bins * sizeof(double), cudaMemcpyHostToDevice,
                              st));
  return CF_OK;
}

// out = c2r( table(s^2) r2c(in) ), in may equal out
static int scaled_round_trip(cf_ctx *ctx, const double *in, double *out, cudaStream_t st) {
  double *hc = ctx->spec_hc;
  CF_TRY_CUFFT(cufftSetStream(ctx->plan_d2z1, st));
  CF_TRY_CUFFT(cufftSetStream(ctx->plan_z2d1, st));
  CF_TRY_CUFFT(cufftExecD2Z(ctx->plan_d2z1, const_cast<double *>(in), (cufftDoubleComplex *)hc));
  k_scale_by_s2<<<blocks_for(ctx->hc_count / 2), 256, 0, st>>>(hc, ctx->ic_table, (int)ctx->N);
  CF_LAUNCHED(ctx);
  CF_TRY_CUFFT(cufftExecZ2D(ctx->plan_z2d1, (cufftDoubleComplex *)hc, out));
  return CF_OK;
}

int white_noise(cf_ctx *ctx, uint64_t seed, uint64_t offset, double *d_out, int64_t n, cudaStream_t st) {
  if (n == 0) return CF_OK;
  ProfScope ps(ctx, CF_PROF_OTHER, st);
  k_white_noise<<<blocks_for((n + 1) / 2 + 1), 256, 0, st>>>(seed, offset, n, d_out);
  CF_LAUNCHED(ctx);
  return CF_OK;
}

int grf(cf_ctx *ctx, const double *d_white, const double *d_psi, double psi_scale, const double *h_sqrtP,
        double *d_out, cudaStream_t st) {
  CF_TRY(ensure_init(ctx, h_sqrtP, st));
  ProfScope ps(ctx, CF_PROF_OTHER, st);
  k_grf_modulate<<<blocks_for(ctx->N3), 256, 0, st>>>(d_white, d_psi, psi_scale, d_out, ctx->N3);
  CF_LAUNCHED(ctx);
  return scaled_round_trip(ctx, d_out, d_out, st);
}

int scale_modes(cf_ctx *ctx, const double *d_f, const double *h_scale, double *d_out, cudaStream_t st) {
  CF_TRY(ensure_init(ctx, h_scale, st));
  ProfScope ps(ctx, CF_PROF_OTHER, st);
  return scaled_round_trip(ctx, d_f, d_out, st);
}

}  // namespace cfb
