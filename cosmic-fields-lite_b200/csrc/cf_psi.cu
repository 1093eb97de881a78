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
//
// A slot holds (e^{2 Psi} - 1, dPsi/dt), not Psi: the right-hand side uses Psi
// only through e^{2 Psi} and e^{4 Psi} = (e^{2 Psi})^2, so the exponential is
// taken once per refresh here (at pass C's store, or in place after a cuFFT
// C2R) instead of twice per stage evaluation in the steppers.  expm1 keeps the
// small part of e^{2 Psi} (|Psi| ~ 1e-2) at full relative precision.

#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

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

// ---- pruned synthesis for a band-limited R_fft ------------------------------
// When R_fft is exactly zero outside |i| <= Ka, |j| <= Kb, k <= Kc (a "box" of
// the half-complex grid), the inverse 3-D DFT factorises into three 1-D passes
// that only need the lines crossing the box:
//   A: along a, for the (Kc+1)(2Kb+1) lines (k, j) of the box     (C2C, length N)
//   B: along b, for the (Kc+1) N lines (k, a)                        (C2C, length N)
//   C: along c, for all N^2 rows (a, b), input zero beyond Kc        (C2R, length N)
// (unnormalised inverse transforms, like the full C2R; the transfer factors are
// applied in A's input).  Both fields (Psi, dPsi) go through each pass as one batch.

// Support box of the non-zero entries of an HC array (grid: z = a, y = b, threads c).
template <typename S>
__global__ void k_support(const S *__restrict__ R, int N, int *__restrict__ box) {
  using C = typename Cplx<S>::T;
  const int nh = N / 2 + 1;
  const int a = blockIdx.z, b = blockIdx.y;
  const C *row = reinterpret_cast<const C *>(R) + ((long long)a * N + b) * nh;
  int ma = -1, mb = -1, mc = -1;
  for (int c = threadIdx.x; c < nh; c += blockDim.x) {
    const C v = row[c];
    if (v.x != (S)0 || v.y != (S)0) {
      ma = (a <= N / 2) ? a : N - a;
      mb = (b <= N / 2) ? b : N - b;
      mc = max(mc, c);
    }
  }
  ma = __reduce_max_sync(0xffffffffu, ma);
  mb = __reduce_max_sync(0xffffffffu, mb);
  mc = __reduce_max_sync(0xffffffffu, mc);
  if ((threadIdx.x & 31) == 0 && mc >= 0) {
    atomicMax(box + 0, ma);
    atomicMax(box + 1, mb);
    atomicMax(box + 2, mc);
  }
}

// Pass-A input: pz_a[f][k][jj][a] (f = Psi / dPsi, k <= Kc, jj indexes j in
// -Kb..Kb as 0..Kb, then N-Kb..N-1), zero where |i| > Ka.  Only the band |i| <= Ka is
// written (the zeros stay from the allocation: pass A's C2C runs out of place), one
// thread per a = ii for ii <= Ka and a = ii + N - (2 Ka + 1) above.  With `diff` set,
// each new entry is first compared bit for bit with the one it replaces (the latest
// refresh's) and *diff = 1 marks a difference.  Passes A-C are a fixed sequence of
// deterministic kernels on these entries alone (the zeros and the twiddles do not
// change), so identical entries give a bit-identical synthesis.
__device__ __forceinline__ bool same_bits(float a, float b) { return __float_as_uint(a) == __float_as_uint(b); }
__device__ __forceinline__ bool same_bits(double a, double b) {
  return __double_as_longlong(a) == __double_as_longlong(b);
}
template <typename S>
__global__ void k_prune_a(const S *__restrict__ R, const double *__restrict__ table, S *__restrict__ pz, int N, int Ka,
                          int Kb, int Kc, int *__restrict__ diff) {
  using C = typename Cplx<S>::T;
  const int nh = N / 2 + 1, nj = 2 * Kb + 1, na = 2 * Ka + 1;
  const int jj = blockIdx.y, k = blockIdx.z;
  const int b = (jj <= Kb) ? jj : jj - nj + N;
  const int bs = (b <= N / 2) ? b : N - b;
  const long long fstride = (long long)(Kc + 1) * nj * N;
  C *o0 = reinterpret_cast<C *>(pz) + ((long long)k * nj + jj) * N;
  C *o1 = o0 + fstride;
  for (int ii = blockIdx.x * blockDim.x + threadIdx.x; ii < na; ii += gridDim.x * blockDim.x) {
    const int a = ii <= Ka ? ii : ii + (N - na);
    const int as = ii <= Ka ? ii : na - ii;  // |i| of a
    const int s2 = as * as + bs * bs + k * k;
    const double tp = table[2 * s2], td = table[2 * s2 + 1];
    const C r = reinterpret_cast<const C *>(R)[((long long)a * N + b) * nh + k];
    C p, d;
    p.x = (S)((double)r.x * tp);
    p.y = (S)((double)r.y * tp);
    d.x = (S)((double)r.x * td);
    d.y = (S)((double)r.y * td);
    if (diff) {
      const C q0 = o0[a], q1 = o1[a];
      if (!(same_bits(p.x, q0.x) && same_bits(p.y, q0.y) && same_bits(d.x, q1.x) && same_bits(d.y, q1.y)))
        *reinterpret_cast<volatile int *>(diff) = 1;
    }
    o0[a] = p;
    o1[a] = d;
  }
}

// Pass-B input: pz_b[f][k][a][b] = pz_a2[f][k][jj(b)][a] for b in the box, else 0.
template <typename S>
__global__ void k_prune_b(const S *__restrict__ pa, S *__restrict__ pb, int N, int Kb, int Kc) {
  using C = typename Cplx<S>::T;
  const int nj = 2 * Kb + 1;
  const int a = blockIdx.y, fk = blockIdx.z;  // fk = f * (Kc + 1) + k
  const C *in = reinterpret_cast<const C *>(pa) + (long long)fk * nj * N;
  C *out = reinterpret_cast<C *>(pb) + ((long long)fk * N + a) * N;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < N; b += gridDim.x * blockDim.x) {
    C v;
    v.x = v.y = (S)0;
    const int jj = (b <= Kb) ? b : (b >= N - Kb ? b - N + nj : -1);
    if (jj >= 0) v = in[(long long)jj * N + a];
    out[b] = v;
  }
}

// Pass-C input (the HC rows of the 1-D C2R): pc[f][a][b][k] = pz_b[f][k][a][b] for
// k <= Kc, 0 up to N/2.  Block: one (f, a) and 32 consecutive b; the (Kc+1) x 32
// tile goes through shared memory so both sides are coalesced.
template <typename S>
__global__ void __launch_bounds__(256) k_prune_c(const S *__restrict__ pb, S *__restrict__ pc, int N, int Kc) {
  using C = typename Cplx<S>::T;
  extern __shared__ unsigned char smraw[];
  C *tile = reinterpret_cast<C *>(smraw);  // [Kc+1][33]
  const int nh = N / 2 + 1;
  const int b0 = blockIdx.x * 32, a = blockIdx.y, f = blockIdx.z;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  for (int k = ty; k <= Kc; k += 8)
    tile[k * 33 + tx] = reinterpret_cast<const C *>(pb)[(((long long)f * (Kc + 1) + k) * N + a) * N + b0 + tx];
  __syncthreads();
  C *outbase = reinterpret_cast<C *>(pc) + (((long long)f * N + a) * N + b0) * nh;
  for (int bb = ty; bb < 32; bb += 8) {
    C *row = outbase + (long long)bb * nh;
    for (int k = tx; k < nh; k += 32) {
      C v;
      v.x = v.y = (S)0;
      if (k <= Kc) v = tile[k * 33 + bb];
      row[k] = v;
    }
  }
}

// ---- pass C as one kernel: pruned half-complex rows -> real rows ------------
// For power-of-two N the C2R of pass C runs in one kernel that reads only the
// Kc+1 non-zero entries of each row and writes the real row once (the cuFFT
// route pads every row to N/2+1 entries in HBM and reads it back).
//
// A length-N C2R of a Hermitian row X[0..N/2] is an M = N/2 point complex
// inverse DFT: with z[m] = x[2m] + i x[2m+1] and w = e^{2 pi i / N},
//   Z[k] = (X[k] + conj X[M-k]) + i (X[k] - conj X[M-k]) w^k,
//   z[m] = sum_k Z[k] e^{2 pi i k m / M}          (unnormalised, like cuFFT).
// With X zero beyond Kc < M/2 (the pruned box) this is
//   Z[k]   = X[k] + i X[k] w^k                    for 0 <= k <= Kc,
//   Z[M-j] = conj(X[j] - i X[j] w^j)              for 1 <= j <= Kc,
// and zero in between; X[0] enters by its real part (the Hermitian projection
// every C2R applies).  The M-point DFT is split M = R1 x R2 ("four-step"):
//   pass 1: for each k2 < R2, an R1-point DFT over k1 of Z[k2 + R2 k1], times
//           e^{2 pi i k2 m1 / M};
//   pass 2: for each m1 < R1, an R2-point DFT over k2, giving z[m1 + R1 m2].
// Each R-point DFT (R <= 32) runs in registers (radix-2, unrolled, twiddles
// e^{2 pi i e / 32} from the kernel's parameter bank).  A CTA takes ROWS rows
// (consecutive b of one (f, a)); between the passes the rows sit in shared
// memory as T[m1][k2][r] with the row index fastest, padded to an odd m1
// stride, so pass 1 stores and pass 2 loads are free of bank conflicts, and
// pass 2's global stores run along m1, i.e. along the output row.  The input
// tile holds X[k] and i X[k] w^k (formed once per input at load), and the
// pass-1 twiddles e^{2 pi i k2 m1 / M} are staged in shared memory as TW[m1][k2].

// e^{2 Psi} - 1 in the storage type.  For |2 Psi| <= 1/4 (the fields' range:
// rms 1e-2) the Taylor series of e^x - 1 truncated after x^7 in FP32 (relative
// truncation error < 2^-29) and after x^13 in FP64 (< 2^-62), by Horner's rule;
// outside that range the library expm1.
__device__ __forceinline__ float e2m1_of(float psi) {
  const float x = 2.0f * psi;
  if (fabsf(x) > 0.25f) return expm1f(x);
  float q = 1.0f / 5040.0f;
  q = fmaf(q, x, 1.0f / 720.0f);
  q = fmaf(q, x, 1.0f / 120.0f);
  q = fmaf(q, x, 1.0f / 24.0f);
  q = fmaf(q, x, 1.0f / 6.0f);
  q = fmaf(q, x, 0.5f);
  return fmaf(q, x * x, x);
}
__device__ __forceinline__ double e2m1_of(double psi) {
  const double x = 2.0 * psi;
  if (fabs(x) > 0.25) return expm1(x);
  double q = 1.0 / 6227020800.0;  // 1/13!
  q = fma(q, x, 1.0 / 479001600.0);
  q = fma(q, x, 1.0 / 39916800.0);
  q = fma(q, x, 1.0 / 3628800.0);
  q = fma(q, x, 1.0 / 362880.0);
  q = fma(q, x, 1.0 / 40320.0);
  q = fma(q, x, 1.0 / 5040.0);
  q = fma(q, x, 1.0 / 720.0);
  q = fma(q, x, 1.0 / 120.0);
  q = fma(q, x, 1.0 / 24.0);
  q = fma(q, x, 1.0 / 6.0);
  q = fma(q, x, 0.5);
  return fma(q, x * x, x);
}

// The same for a pair of FP32 values (a complex entry of pass C's output) with the
// sm_100 paired FP32 instructions (FADD2 / FMUL2 / FFMA2): one instruction per Horner
// step for both values, each component rounded exactly as the scalar form above.
// e2m1_poly_pair: the polynomial alone, for values the caller has range-checked.
__device__ __forceinline__ float2 e2m1_poly_pair(float2 psi) {
  const float2 x = __fadd2_rn(psi, psi);  // 2 psi, exact
  float2 q = make_float2(1.0f / 5040.0f, 1.0f / 5040.0f);
  q = __ffma2_rn(q, x, make_float2(1.0f / 720.0f, 1.0f / 720.0f));
  q = __ffma2_rn(q, x, make_float2(1.0f / 120.0f, 1.0f / 120.0f));
  q = __ffma2_rn(q, x, make_float2(1.0f / 24.0f, 1.0f / 24.0f));
  q = __ffma2_rn(q, x, make_float2(1.0f / 6.0f, 1.0f / 6.0f));
  q = __ffma2_rn(q, x, make_float2(0.5f, 0.5f));
  return __ffma2_rn(q, __fmul2_rn(x, x), x);
}
__device__ __forceinline__ float2 e2m1_pair(float2 psi) {
  const float2 x = __fadd2_rn(psi, psi);  // 2 psi, exact
  if (fabsf(x.x) > 0.25f || fabsf(x.y) > 0.25f) return make_float2(e2m1_of(psi.x), e2m1_of(psi.y));
  float2 q = make_float2(1.0f / 5040.0f, 1.0f / 5040.0f);
  q = __ffma2_rn(q, x, make_float2(1.0f / 720.0f, 1.0f / 720.0f));
  q = __ffma2_rn(q, x, make_float2(1.0f / 120.0f, 1.0f / 120.0f));
  q = __ffma2_rn(q, x, make_float2(1.0f / 24.0f, 1.0f / 24.0f));
  q = __ffma2_rn(q, x, make_float2(1.0f / 6.0f, 1.0f / 6.0f));
  q = __ffma2_rn(q, x, make_float2(0.5f, 0.5f));
  return __ffma2_rn(q, __fmul2_rn(x, x), x);
}
__device__ __forceinline__ double2 e2m1_pair(double2 psi) { return make_double2(e2m1_of(psi.x), e2m1_of(psi.y)); }

template <typename S>
__global__ void k_psi_to_e2m1(S *__restrict__ f, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) f[i] = e2m1_of(f[i]);
}

template <typename S>
struct Tw32 {
  typename Cplx<S>::T w[16];  // e^{2 pi i e / 32}, e < 16
};

template <typename C>
__device__ __forceinline__ C c_add(C a, C b) {
  return C{a.x + b.x, a.y + b.y};
}
template <typename C>
__device__ __forceinline__ C c_sub(C a, C b) {
  return C{a.x - b.x, a.y - b.y};
}
template <typename C>
__device__ __forceinline__ C c_mul(C a, C b) {
  return C{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename C>
__device__ __forceinline__ C c_mul_i(C a) {
  return C{-a.y, a.x};
}
// FP32 complex sums as one sm_100 paired instruction (FADD2) each: per component the
// same round-to-nearest sum as the scalar form.
__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
// FP32 complex product as FMUL2 + FFMA2: re = fma(a.x, b.x, rn(-a.y b.y)), im = fma(a.x,
// b.y, rn(a.y b.x)) -- a fixed rounding, whatever contraction the compiler would pick.
__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
  return __ffma2_rn(make_float2(a.x, a.x), b, __fmul2_rn(make_float2(-a.y, a.y), make_float2(b.y, b.x)));
}

__host__ __device__ constexpr int bit_reverse(int i, int R) {
  int r = 0;
  for (int b = 1; b < R; b <<= 1) {
    r = (r << 1) | (i & 1);
    i >>= 1;
  }
  return r;
}

// Bit k set for the rows k < B and k >= R - B of an R-point DFT's input: the band of
// a pruned line, whose other rows are zero.
__host__ __device__ constexpr unsigned band_mask(int R, int B) {
  return 2 * B >= R ? (R == 32 ? 0xffffffffu : (1u << R) - 1u) : ((1u << B) - 1u) | (((1u << B) - 1u) << (R - B));
}

// In-register R-point inverse DFT (e^{+2 pi i k m / R}), natural order in and out.
// NZ: bit k clear where the caller knows v[k] is zero.  Radix-2 butterflies with a
// zero operand reduce to copies and negations (u + 0 = u, 0 + t = t and 0 - t = -t
// exactly), decided at compile time once the loops are unrolled; the non-zero values
// are bit-identical to the full butterfly network's.
template <typename S, int R, unsigned NZ = 0xffffffffu>
__device__ __forceinline__ void dft_inv(typename Cplx<S>::T (&v)[R], const Tw32<S> &tw) {
  static_assert(R >= 2 && R <= 32 && (R & (R - 1)) == 0, "radix");
  using C = typename Cplx<S>::T;
  C a[R];
  bool nz[R];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    a[i] = v[bit_reverse(i, R)];
    nz[i] = (NZ >> bit_reverse(i, R)) & 1u;
  }
#pragma unroll
  for (int len = 2; len <= R; len *= 2) {
#pragma unroll
    for (int i = 0; i < R; i += len) {
#pragma unroll
      for (int j = 0; j < len / 2; ++j) {
        const int p = i + j, q = i + j + len / 2;
        if (!nz[q]) {  // t = 0
          a[q] = a[p];
          nz[q] = nz[p];
          continue;
        }
        const int e = j * (32 / len);  // e^{2 pi i j / len} = e^{2 pi i e / 32}
        C t = a[q];
        if (e == 8)
          t = c_mul_i(t);
        else if (e != 0)
          t = c_mul(t, tw.w[e]);
        if (!nz[p]) {  // u = 0
          a[p] = t;
          a[q] = C{-t.x, -t.y};
          nz[p] = true;
        } else {
          const C u = a[p];
          a[p] = c_add(u, t);
          a[q] = c_sub(u, t);
        }
      }
    }
  }
#pragma unroll
  for (int i = 0; i < R; ++i) v[i] = a[i];
}

// B: Z is zero outside the k1 rows [0, B) and [R1 - B, R1) (the band |k| <= Kc
// with B = ceil((Kc+1)/R2)); as a template argument it gives the pass-1 DFT its
// zero mask (band_mask), so the butterflies on those rows reduce to copies.
// B = R1/2 keeps every row.
template <typename S, int R1, int R2, int ROWS, int B>
__global__ void __launch_bounds__(256) k_prune_c_fft(const S *__restrict__ pb, S *__restrict__ out,
                                                     const typename Cplx<S>::T *__restrict__ wN,
                                                     const typename Cplx<S>::T *__restrict__ twM, int N, int Kc,
                                                     const __grid_constant__ Tw32<S> tw) {
  using C = typename Cplx<S>::T;
  constexpr int M = R1 * R2;  // N == 2 M
  constexpr int TS = R2 * ROWS + 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  C *T = reinterpret_cast<C *>(smraw);  // [R1][TS]
  C *TW = T + R1 * TS;                  // [R1][R2]: e^{2 pi i k2 m1 / M}
  C *Xs = TW + M;                       // [Kc+1][ROWS]: X[k] (X[0] by its real part)
  C *XPs = Xs + (Kc + 1) * ROWS;        // [Kc+1][ROWS]: i X[k] w^k
  const int b0 = blockIdx.x * ROWS, a = blockIdx.y, f = blockIdx.z;
  const C *src = reinterpret_cast<const C *>(pb) + ((long long)f * (Kc + 1) * N + a) * N + b0;
  for (int i = threadIdx.x; i < M; i += blockDim.x) TW[i] = twM[i];
  for (int i = threadIdx.x; i < (Kc + 1) * ROWS; i += blockDim.x) {
    const int k = i / ROWS, r = i - k * ROWS;
    C x = src[(long long)k * N * N + r];
    if (k == 0) x.y = (S)0;
    Xs[i] = x;
    XPs[i] = c_mul_i(c_mul(x, wN[k]));
  }
  __syncthreads();
  for (int task = threadIdx.x; task < R2 * ROWS; task += blockDim.x) {
    const int k2 = task / ROWS, r = task - k2 * ROWS;
    C v[R1];
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      const int k = k2 + R2 * k1;
      C z{(S)0, (S)0};
      if (k1 >= B && k1 < R1 - B) {
        // outside the band's rows: zero
      } else if (k <= Kc) {
        z = c_add(Xs[k * ROWS + r], XPs[k * ROWS + r]);  // X + i X w^k
      } else if (k >= M - Kc) {
        const int j = M - k;
        const C d = c_sub(Xs[j * ROWS + r], XPs[j * ROWS + r]);  // conj(X - i X w^j)
        z = C{d.x, -d.y};
      }
      v[k1] = z;
    }
    dft_inv<S, R1, band_mask(R1, B)>(v, tw);
#pragma unroll
    for (int m1 = 0; m1 < R1; ++m1) {
      C y = v[m1];
      if (m1 > 0) y = c_mul(y, TW[m1 * R2 + k2]);  // e^{2 pi i k2 m1 / M}
      T[m1 * TS + k2 * ROWS + r] = y;
    }
  }
  __syncthreads();
  for (int task = threadIdx.x; task < R1 * ROWS; task += blockDim.x) {
    const int r = task / R1, m1 = task - r * R1;
    C u[R2];
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) u[k2] = T[m1 * TS + k2 * ROWS + r];
    dft_inv<S, R2>(u, tw);
    C *row = reinterpret_cast<C *>(out) + ((long long)(f * N + a) * N + b0 + r) * M;
#pragma unroll
    for (int m2 = 0; m2 < R2; ++m2) {
      C o = u[m2];
      if (f == 0) o = e2m1_pair(o);  // the slot holds e^{2 Psi} - 1
      row[m1 + R1 * m2] = o;
    }
  }
}

// Pass C as a persistent kernel (FP64 storage; pc_persistent).  A CTA walks tiles (f, a, ROWS rows of b) with
// stride gridDim.x; the twiddles e^{2 pi i k2 m1 / M} and w^k are staged once per
// CTA, and the next tile's band rows X[k][b0 .. b0 + ROWS) are copied into shared
// memory by cp.async while the current tile runs its second radix pass, so the
// tile's global loads are not waited on at its start.  The arithmetic is pass 1 /
// pass 2 of k_prune_c_fft; Z[k] = X[k] + i X[k] w^k is formed in pass 1 from the
// staged X.
__device__ __forceinline__ void pc_cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

template <typename S, int R1, int R2, int ROWS, int B>
__global__ void __launch_bounds__(256) k_prune_c_fft_p(const S *__restrict__ pb, S *__restrict__ out,
                                                       const typename Cplx<S>::T *__restrict__ wN,
                                                       const typename Cplx<S>::T *__restrict__ twM, int N, int Kc,
                                                       int ntiles, const __grid_constant__ Tw32<S> tw) {
  using C = typename Cplx<S>::T;
  constexpr int M = R1 * R2;  // N == 2 M
  constexpr int TS = R2 * ROWS + 1;
  constexpr int CPR = ROWS * (int)sizeof(C) / 16;  // 16-byte copies per band row of a tile
  static_assert(ROWS * sizeof(C) % 16 == 0, "tile rows");
  extern __shared__ __align__(16) unsigned char smraw[];
  C *XR = reinterpret_cast<C *>(smraw);  // [Kc+1][ROWS]: X[k] of the tile (16-byte aligned)
  C *T = XR + (Kc + 1) * ROWS;           // [R1][TS]
  C *TW = T + R1 * TS;                   // [R1][R2]: e^{2 pi i k2 m1 / M}
  C *WK = TW + M;                        // [Kc+1]: w^k = e^{2 pi i k / N}
  const int nb = N / ROWS;
  auto issue = [&](int tile) {
    const int bt = tile % nb, a = (tile / nb) % N, f = tile / (nb * N);
    const C *src = reinterpret_cast<const C *>(pb) + ((long long)f * (Kc + 1) * N + a) * N + (long long)bt * ROWS;
    for (int i = threadIdx.x; i < (Kc + 1) * CPR; i += blockDim.x) {
      const int k = i / CPR, j = i - k * CPR;
      pc_cp_async16(reinterpret_cast<unsigned char *>(XR + k * ROWS) + 16 * j,
                    reinterpret_cast<const unsigned char *>(src + (long long)k * N * N) + 16 * j);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  for (int i = threadIdx.x; i < M; i += blockDim.x) TW[i] = twM[i];
  for (int i = threadIdx.x; i <= Kc; i += blockDim.x) WK[i] = wN[i];
  int tile = blockIdx.x;
  if (tile < ntiles) issue(tile);
  for (; tile < ntiles; tile += gridDim.x) {
    const int bt = tile % nb, a = (tile / nb) % N, f = tile / (nb * N);
    const int b0 = bt * ROWS;
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();  // the tile's X (everyone's copies); the last tile's pass 2 is done with T
    for (int task = threadIdx.x; task < R2 * ROWS; task += blockDim.x) {
      const int k2 = task / ROWS, r = task - k2 * ROWS;
      C v[R1];
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) {
        const int k = k2 + R2 * k1;
        C z{(S)0, (S)0};
        if (k1 >= B && k1 < R1 - B) {
          // outside the band's rows: zero
        } else if (k <= Kc) {
          C x = XR[k * ROWS + r];
          if (k == 0) x.y = (S)0;
          const C xp = c_mul_i(c_mul(x, WK[k]));
          z = c_add(x, xp);  // X + i X w^k
        } else if (k >= M - Kc) {
          const int j = M - k;
          const C x = XR[j * ROWS + r];
          const C xp = c_mul_i(c_mul(x, WK[j]));
          const C d = c_sub(x, xp);  // conj(X - i X w^j)
          z = C{d.x, -d.y};
        }
        v[k1] = z;
      }
      dft_inv<S, R1, band_mask(R1, B)>(v, tw);
#pragma unroll
      for (int m1 = 0; m1 < R1; ++m1) {
        C y = v[m1];
        if (m1 > 0) y = c_mul(y, TW[m1 * R2 + k2]);
        T[m1 * TS + k2 * ROWS + r] = y;
      }
    }
    __syncthreads();  // T complete; every read of the tile's X is done
    if (tile + (int)gridDim.x < ntiles) issue(tile + gridDim.x);
    for (int task = threadIdx.x; task < R1 * ROWS; task += blockDim.x) {
      const int r = task / R1, m1 = task - r * R1;
      C u[R2];
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) u[k2] = T[m1 * TS + k2 * ROWS + r];
      dft_inv<S, R2>(u, tw);
      C *row = reinterpret_cast<C *>(out) + ((long long)(f * N + a) * N + b0 + r) * M;
#pragma unroll
      for (int m2 = 0; m2 < R2; ++m2) {
        C o = u[m2];
        if (f == 0) o = e2m1_pair(o);  // the slot holds e^{2 Psi} - 1
        row[m1 + R1 * m2] = o;
      }
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// ---- pass C, one warp per row group (FP32, N = 256, 512, 1024) --------------
// The same four-step arithmetic as k_prune_c_fft without a CTA barrier: a warp owns
// RW = 32 / R2 consecutive rows of one (f, a) plane and does everything for them --
// brings the rows' Kc + 1 band entries into its own shared memory (one tile ahead,
// double-buffered), runs pass 1 with one lane per (row, k2) -- every lane busy --
// forming X + i X w^k from the staged X as it loads, then pass 2 with RW R1 / 32
// (row, m1) tasks per lane through a warp-private transpose, with only __syncwarp
// between them, and stores along the output rows.  Persistent: warps walk the tiles
// (f, a, row group) with stride = warps in the grid, adjacent warps on adjacent rows.
//
// TMA (the default where the tensor map exists): one lane copies a tile's band as one
// 3-D box {RW rows of b, one a, Kc + 1 k} of pass B's lines with cp.async.bulk.tensor,
// completing on the buffer's mbarrier; the gather no longer occupies the LSU pipe
// (each of its 8-byte cp.async took a line of its own).  The box lands as X[k][r].
// Every mbarrier wait is bounded: when one gives up the warp sets the mapped error
// word, waits (bounded again) for its copies still in flight and leaves the loop.
// Otherwise X[r][XPP] by per-lane cp.async (XPP = 8 mod 16 complex, so the two rows a
// half-warp reads sit on disjoint banks).
//
// T[r][RP] with T[r] = [m1][TP], TP = R2 + 1 odd (pass-2 reads free of bank
// conflicts) and RP = R2 mod 16 where R2 < 16.
__host__ __device__ constexpr int pc_xpp(int kn) { return ((kn + 7) & ~15) + 8; }
__host__ __device__ constexpr int pc_rp(int R1, int R2) {
  return R2 >= 16 ? R1 * (R2 + 1) : R1 * (R2 + 1) + ((R2 - (R1 * (R2 + 1)) % 16) + 16) % 16;
}
__host__ __device__ constexpr int pc_up16(int n) { return (n + 15) & ~15; }  // complex: 128 bytes
// X buffers per warp (TMA: boxes two tiles ahead), complex words per X buffer and per warp.
__host__ __device__ constexpr int pc_nbuf(bool tma) { return tma ? 3 : 2; }
__host__ __device__ constexpr int pc_xw(int kn, int RW, bool tma) { return tma ? pc_up16(kn * RW) : RW * pc_xpp(kn); }
__host__ __device__ constexpr int pc_warp_words(int kn, int R1, int R2, bool tma) {
  return tma ? pc_up16(pc_nbuf(true) * pc_xw(kn, 32 / R2, true) + (32 / R2) * pc_rp(R1, R2))
             : pc_nbuf(false) * pc_xw(kn, 32 / R2, false) + (32 / R2) * pc_rp(R1, R2);
}
constexpr int kPcBarBytes = 256;  // 8 warps x 3 mbarriers, rounded to 128 bytes

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ void tma_load_3d(unsigned dst, const void *tmap, int x, int y, int z, unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
          "r"(dst),
      "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}
// The bounded waits of the warp pass C: tests per wait (by default 2^20: try_wait
// suspends the thread for a while between tests, so seconds), and bytes armed on each
// box's barrier beyond what the box delivers (0; cf_psi_set_wait_test sets it so that
// the waits give up, to test that path).
struct PcWait {
  long long spin_limit;
  int tx_extra;
};

template <int R1, int R2, int B, bool TMA>
__global__ void __launch_bounds__(256, 3) k_prune_c_warp(const float *__restrict__ pb, float *__restrict__ out,
                                                     const float2 *__restrict__ wN, const float2 *__restrict__ twM,
                                                     int N, int Kc, int tile0, int ntiles, int log2_groups,
                                                     int log2_n, const __grid_constant__ Tw32<float> tw,
                                                     const __grid_constant__ CUtensorMap tmap, int *err,
                                                     const PcWait wt) {
  constexpr int M = R1 * R2;  // N == 2 M
  constexpr int RW = 32 / R2;
  constexpr int TP = R2 + 1;
  constexpr int RP = pc_rp(R1, R2);
  constexpr int P2 = RW * R1 / 32;  // pass-2 tasks per lane
  static_assert(R2 <= R1 && 32 % R2 == 0 && (RW * R1) % 32 == 0, "shape");
  constexpr int NB = pc_nbuf(TMA);
  extern __shared__ __align__(128) unsigned char pcw_smem[];  // TMA boxes land on 128-byte boundaries
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kn = Kc + 1;
  // [mbarriers: NB per warp] [TW: M] [WK: kn, to 128 bytes] [per warp: NB X buffers, T]
  unsigned long long *bars = reinterpret_cast<unsigned long long *>(pcw_smem);
  float2 *TW = reinterpret_cast<float2 *>(pcw_smem + kPcBarBytes);  // [R1][R2]: e^{2 pi i k2 m1 / M}
  float2 *WK = TW + M;                                              // [Kc+1]: w^k
  const int xw = pc_xw(kn, RW, TMA);
  float2 *W = WK + pc_up16(kn) + (size_t)warp * pc_warp_words(kn, R1, R2, TMA);
  float2 *X0 = W, *T = W + NB * xw;
  for (int i = threadIdx.x; i < M; i += blockDim.x) TW[i] = twM[i];
  for (int i = threadIdx.x; i < kn; i += blockDim.x) WK[i] = wN[i];
  const unsigned bar0 = (unsigned)__cvta_generic_to_shared(bars + NB * warp);
  if constexpr (TMA) {
    if (lane == 0) {
      for (int b = 0; b < NB; ++b) mbar_init(bar0 + 8 * b, 1);
      asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
  }
  __syncthreads();  // the only CTA barrier: the shared twiddles and the initialised mbarriers

  // tile t = (f N + a) groups + g, groups = N / RW row groups per plane (powers of two)
  const int gmask = (1 << log2_groups) - 1, nmask = (1 << log2_n) - 1;
  const long long NN = (long long)N * N;
  const int stride = gridDim.x * (blockDim.x >> 5);
  int tile = tile0 + blockIdx.x * (blockDim.x >> 5) + warp;  // tiles [tile0, ntiles)
  auto issue = [&](int t, int b) {
    const int g = t & gmask, fa = t >> log2_groups;
    const int a = fa & nmask, f = fa >> log2_n;
    float2 *dst = X0 + b * xw;
    if constexpr (TMA) {
      if (lane == 0) {
        // the warp's generic reads of this buffer (ordered by the __syncwarp that ended
        // its last tile) before the async proxy overwrites it
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        const unsigned bar = bar0 + 8 * b;
        mbar_expect_tx(bar, (unsigned)(kn * RW * sizeof(float2)) + (unsigned)wt.tx_extra);
        tma_load_3d((unsigned)__cvta_generic_to_shared(dst), &tmap, 2 * g * RW, a, f * kn, bar);
      }
    } else {
      const int xpp = pc_xpp(kn);
      const float2 *src = reinterpret_cast<const float2 *>(pb) + ((long long)f * kn * N + a) * N + g * RW + lane * NN;
      const unsigned d0 = (unsigned)__cvta_generic_to_shared(dst + lane);
      for (int k = lane; k < kn; k += 32, src += 32 * NN) {
        const unsigned d = d0 + (unsigned)((k - lane) * sizeof(float2));
#pragma unroll
        for (int r = 0; r < RW; ++r)
          asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d + (unsigned)(r * xpp * sizeof(float2))),
                       "l"(src + r)
                       : "memory");
      }
      asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
  };
  // bit b: the parity buffer b's barrier completes next / a copy into buffer b is in
  // flight (bit masks rather than arrays indexed by the buffer, which would live in
  // local memory)
  unsigned phase = 0u, pending = 0u;
  auto wait_buf = [&](int b) -> bool {  // TMA: the buffer's copy has landed (bounded, per lane)
    const unsigned bar = bar0 + 8 * b;
    for (long long i = 0; i < wt.spin_limit; ++i)
      if (mbar_try_wait(bar, (phase >> b) & 1u)) {
        phase ^= 1u << b;
        pending &= ~(1u << b);
        return true;
      }
    return false;
  };
  int buf = 0;
  bool ok = true;
  // prologue: the first NB - 1 tiles' copies; each iteration then issues the tile NB - 1
  // strides ahead into the buffer the previous iteration finished with
  for (int d = 0; d < NB - 1; ++d)
    if (tile + d * stride < ntiles) {
      issue(tile + d * stride, d);
      pending |= 1u << d;
    }
  for (; tile < ntiles; tile += stride) {
    const bool more = tile + stride < ntiles;
    const int ahead = tile + (NB - 1) * stride, abuf = buf == 0 ? NB - 1 : buf - 1;
    if (ahead < ntiles) {
      issue(ahead, abuf);
      pending |= 1u << abuf;
    }
    if constexpr (TMA) {
      // every lane tests the barrier itself; the warp gives up together if any lane did
      if (!__all_sync(0xffffffffu, wait_buf(buf))) {
        ok = false;
        break;
      }
    } else {
      if (more)
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");
      else
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
      pending &= ~(1u << buf);
    }
    __syncwarp();  // the tile's band entries (every lane's copies)
    const float2 *X = X0 + buf * xw;
    // X[k][r] (TMA box) or X[r][XPP] (per-lane copies)
    auto xat = [&](int r, int k) -> float2 { return TMA ? X[k * RW + r] : X[r * pc_xpp(kn) + k]; };
    const int g = tile & gmask, fa = tile >> log2_groups;
    // pass 1: lane (r, k2), an R1-point DFT over the band rows k1, times e^{2 pi i k2 m1 / M}
    {
      const int r = lane / R2, k2 = lane % R2;
      float2 v[R1];
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) {
        // rows k1 < B hold k <= R2 B - 1 <= M/2 - 1 < M - Kc, rows k1 >= R1 - B hold
        // k >= M/2 > Kc (Kc < M/2): each band half tests its own side only
        const int k = k2 + R2 * k1;
        float2 z = make_float2(0.0f, 0.0f);
        if (k1 < B) {
          if (k <= Kc) {
            float2 x = xat(r, k);
            if (k == 0) x.y = 0.0f;  // X[0] by its real part: the Hermitian projection of every C2R
            z = c_add(x, c_mul_i(c_mul(x, WK[k])));  // X + i X w^k
          }
        } else if (k1 >= R1 - B) {
          const int j = M - k;
          if (j <= Kc) {
            const float2 x = xat(r, j);
            const float2 d = c_sub(x, c_mul_i(c_mul(x, WK[j])));  // conj(X - i X w^j)
            z = make_float2(d.x, -d.y);
          }
        }
        v[k1] = z;
      }
      dft_inv<float, R1, band_mask(R1, B)>(v, tw);
      float2 *Tr = T + r * RP + k2;
#pragma unroll
      for (int m1 = 0; m1 < R1; ++m1) {
        float2 y = v[m1];
        if (m1 > 0) y = c_mul(y, TW[m1 * R2 + k2]);
        Tr[m1 * TP] = y;
      }
    }
    __syncwarp();
    // pass 2: task (r, m1), an R2-point DFT over k2, giving z[m1 + R1 m2] of row r
    const bool field0 = fa < N;  // f == 0: the slot holds e^{2 Psi} - 1
#pragma unroll 1
    for (int p = 0; p < P2; ++p) {
      const int task = lane + 32 * p;
      const int r = task / R1, m1 = task % R1;
      float2 u[R2];
      const float2 *Tr = T + r * RP + m1 * TP;
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) u[k2] = Tr[k2];
      dft_inv<float, R2>(u, tw);
      float2 *row = reinterpret_cast<float2 *>(out) + ((long long)fa * N + g * RW + r) * M;
      if (field0) {
        // one range test for the lane's R2 values: all inside |2 Psi| <= 1/4 takes the
        // polynomial directly; otherwise e2m1_pair decides per value as everywhere else
        float mx = 0.0f;
#pragma unroll
        for (int m2 = 0; m2 < R2; ++m2) mx = fmaxf(mx, fmaxf(fabsf(u[m2].x), fabsf(u[m2].y)));
        if (2.0f * mx <= 0.25f) {
#pragma unroll
          for (int m2 = 0; m2 < R2; ++m2) u[m2] = e2m1_poly_pair(u[m2]);
        } else {
#pragma unroll
          for (int m2 = 0; m2 < R2; ++m2) u[m2] = e2m1_pair(u[m2]);
        }
      }
#pragma unroll
      for (int m2 = 0; m2 < R2; ++m2) row[m1 + R1 * m2] = u[m2];
    }
    __syncwarp();  // T and this X buffer are free for the next tiles
    buf = buf + 1 == NB ? 0 : buf + 1;
  }
  if constexpr (TMA) {
    if (!ok) {  // a copy did not land in time: report it, and let the copies in flight finish
      if (lane == 0) {
        *reinterpret_cast<volatile int *>(err) = 1;
        __threadfence_system();
      }
      for (int b = 0; b < NB; ++b)
        if ((pending >> b) & 1u) (void)wait_buf(b);
    }
  }
}

static bool pc_warp_shape(long long N, size_t word, int *R1, int *R2) {
  if (word != 4) return false;
  switch (N) {
    case 256: *R1 = 16, *R2 = 8; return true;
    case 512: *R1 = 16, *R2 = 16; return true;
    case 1024: *R1 = 32, *R2 = 16; return true;
    default: return false;
  }
}
static size_t pc_warp_smem(int Kc, int R1, int R2, bool tma) {
  const int kn = Kc + 1;
  return kPcBarBytes + ((size_t)R1 * R2 + pc_up16(kn) + 8 * (size_t)pc_warp_words(kn, R1, R2, tma)) * sizeof(float2);
}
// Whether the warp pass C takes its band tiles by TMA (a tensor map exists).
static bool pc_warp_tma(const cf_ctx *ctx) { return ctx->have_pc_tmap; }

template <int R1, int R2, int B, bool TMA>
static int launch_pc_warp_b(cf_ctx *ctx, void *out, size_t smem, cudaStream_t st, int f0, int nf) {
  auto kern = k_prune_c_warp<R1, R2, B, TMA>;
  if (smem > 48 * 1024) CF_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  Tw32<float> tw;
  for (int e = 0; e < 16; ++e) {
    const double ang = 2.0 * 3.14159265358979323846 * e / 32.0;
    tw.w[e] = float2{(float)std::cos(ang), (float)std::sin(ang)};
  }
  CUtensorMap tmap;
  static_assert(sizeof(tmap) == sizeof(ctx->pc_tmap), "tensor map size");
  std::memcpy(&tmap, ctx->pc_tmap, sizeof(tmap));
  int sms = 0, per_sm = 0;
  CF_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
  CF_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem));
  const int N = (int)ctx->N, groups = N / (32 / R2);
  const int tile0 = f0 * N * groups, ntiles = (f0 + nf) * N * groups;  // fields [f0, f0 + nf)
  int log2_n = 0, log2_g = 0;
  while ((1 << log2_n) < N) ++log2_n;
  while ((1 << log2_g) < groups) ++log2_g;
  const int grid = std::max(1, std::min((ntiles - tile0 + 7) / 8, sms * std::max(per_sm, 1)));
  kern<<<(unsigned)grid, 256, smem, st>>>((const float *)ctx->pz_b, (float *)out, (const float2 *)ctx->pr_wN,
                                          (const float2 *)ctx->pr_twM, N, ctx->Kc, tile0, ntiles, log2_g, log2_n,
                                          tw, tmap, ctx->psi_err_d, PcWait{ctx->pc_spin_limit, ctx->pc_tx_extra});
  CF_LAUNCHED(ctx);
  return CF_OK;
}

// The smallest compiled band B >= ceil((Kc+1)/R2).
template <int R1, int R2, bool TMA>
static int launch_pc_warp_t(cf_ctx *ctx, void *out, size_t smem, cudaStream_t st, int f0, int nf) {
  const int need = (ctx->Kc + 1 + R2 - 1) / R2;
  if (need <= 2) return launch_pc_warp_b<R1, R2, 2, TMA>(ctx, out, smem, st, f0, nf);
  if (need <= 3) return launch_pc_warp_b<R1, R2, 3, TMA>(ctx, out, smem, st, f0, nf);
  if (need <= 4) return launch_pc_warp_b<R1, R2, 4, TMA>(ctx, out, smem, st, f0, nf);
  if (need <= 6) return launch_pc_warp_b<R1, R2, 6, TMA>(ctx, out, smem, st, f0, nf);
  return launch_pc_warp_b<R1, R2, R1 / 2, TMA>(ctx, out, smem, st, f0, nf);
}

template <bool TMA>
static int launch_pc_warp_m(cf_ctx *ctx, void *out, size_t smem, int R1, int R2, cudaStream_t st, int f0, int nf) {
  if (R1 == 16 && R2 == 8) return launch_pc_warp_t<16, 8, TMA>(ctx, out, smem, st, f0, nf);
  if (R1 == 16 && R2 == 16) return launch_pc_warp_t<16, 16, TMA>(ctx, out, smem, st, f0, nf);
  return launch_pc_warp_t<32, 16, TMA>(ctx, out, smem, st, f0, nf);
}

static int launch_pc_warp(cf_ctx *ctx, void *out, cudaStream_t st, int f0 = 0, int nf = 2) {
  int R1 = 0, R2 = 0;
  if (!pc_warp_shape(ctx->N, ctx->word, &R1, &R2)) return set_error("warp pass C: unsupported N"), CF_ERR_INVALID;
  const bool tma = pc_warp_tma(ctx);
  const size_t smem = pc_warp_smem(ctx->Kc, R1, R2, tma);
  return tma ? launch_pc_warp_m<true>(ctx, out, smem, R1, R2, st, f0, nf)
             : launch_pc_warp_m<false>(ctx, out, smem, R1, R2, st, f0, nf);
}

// The tensor map of the warp pass C's band tiles: pass B's lines pz_b[f][k][a][b]
// (FP32 complex) as a 3-D array of floats {2N (b, re / im), N (a), 2 (Kc + 1) (f, k)}
// with boxes {2 RW, 1, Kc + 1}.  The x coordinate 2 g RW of a box is 8 g RW bytes
// (a multiple of 16 with RW >= 2), the box's inner extent 8 RW bytes.  Without a
// driver entry point, or for Kc + 1 > 256 (a box dimension's limit), the kernel
// copies with cp.async instead, and at N = 1024, where the boxes measured slower: Psi
// synthesis per RK4 step at N = 512 0.851 -> 0.771 ms with boxes one tile ahead, 0.726
// -> 0.702 with boxes two tiles ahead (three buffers); at N = 1024 (82-row boxes,
// 2 CTAs per SM) 7.44 -> 8.56 ms one tile ahead and 6.98 -> 7.17 two tiles ahead
// (with registers up to 128 there, the per-lane copies took 7.06).
static int encode_pc_tmap(cf_ctx *ctx) {
  ctx->have_pc_tmap = false;
  int R1 = 0, R2 = 0;
  if (!ctx->pc_fused || !pc_warp_shape(ctx->N, ctx->word, &R1, &R2) || ctx->N > 512) return CF_OK;
  const int RW = 32 / R2, kn = ctx->Kc + 1;
  if (kn > 256 || RW < 2) return CF_OK;
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
      (void)cudaGetLastError();
      return CF_OK;
    }
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  if (!ctx->psi_err_h) {
    CF_TRY_CUDA(cudaHostAlloc((void **)&ctx->psi_err_h, sizeof(int), cudaHostAllocMapped));
    *ctx->psi_err_h = 0;
    CF_TRY_CUDA(cudaHostGetDevicePointer((void **)&ctx->psi_err_d, ctx->psi_err_h, 0));
  }
  const cuuint64_t N = (cuuint64_t)ctx->N;
  const cuuint64_t dims[3] = {2 * N, N, 2 * (cuuint64_t)kn};
  const cuuint64_t strides[2] = {2 * N * sizeof(float), 2 * N * N * sizeof(float)};
  const cuuint32_t box[3] = {(cuuint32_t)(2 * RW), 1u, (cuuint32_t)kn};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  CUtensorMap m;
  if (encode(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, ctx->pz_b, dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return CF_OK;
  std::memcpy(ctx->pc_tmap, &m, sizeof(m));
  ctx->have_pc_tmap = true;
  return CF_OK;
}

// ---- pass B as one kernel: pruned lines -> full lines -----------------------
// For FP32 storage and power-of-two N (32..1024) the C2C of pass B reads the
// pass-A lines at their 2Kb+1 non-zero b-frequencies only (pz_a2[f][k][jj][a]) and
// writes the full lines pz_b[f][k][a][b] once: no zero-padded copy (k_prune_b)
// and no library pass over the zeros.  The N-point inverse DFT is split
// N = R1 x R2 as in pass C (k = k2 + R2 k1, m = m1 + R1 m2):
//   pass 1: for each k2, an R1-point DFT over k1 -- zero outside the k1 rows
//           [0, B) and [R1 - B, R1), B = ceil((Kb+1)/R2) -- times e^{2 pi i k2 m1 / N};
//   pass 2: for each m1, an R2-point DFT over k2, giving z[m1 + R1 m2].
// A CTA takes LINES consecutive a of one (f, k): the input tile Y[jj][line] is
// read with the lines fastest (coalesced along a), the intermediate sits in
// shared memory as T[m1][k2][line] (odd m1 stride), and pass 2 stores along b.
//
// Persistent: a CTA stages the twiddles once and walks the tiles (f, k, a-range) with
// stride = CTAs in the grid, a fastest (adjacent CTAs read adjacent pieces of the same
// pass-A rows); the next tile's band lines come into the other Ys buffer by cp.async
// while the current tile runs, so no tile waits on its gathered loads.
template <typename S, int R1, int R2, int LINES, int B>
__global__ void __launch_bounds__(R2 *LINES) k_pass_b_fft(const S *__restrict__ pa, S *__restrict__ pb,
                                                         const typename Cplx<S>::T *__restrict__ twN, int N, int Kb,
                                                         int Kc, int f0, int ntiles,
                                                         const __grid_constant__ Tw32<S> tw) {
  using C = typename Cplx<S>::T;
  constexpr int TS = R2 * LINES + 1;
  constexpr int CPC = 16 / (int)sizeof(C);  // complex per 16-byte copy
  constexpr int CH = LINES / CPC;           // 16-byte copies per band line of a tile
  static_assert(LINES % CPC == 0, "lines");
  extern __shared__ __align__(16) unsigned char smraw[];
  C *T = reinterpret_cast<C *>(smraw);  // [R1][TS]
  C *TW = T + R1 * TS;                  // [R1][R2]: e^{2 pi i k2 m1 / N}
  C *Ys = TW + R1 * R2;                 // 2 buffers [2Kb+1][LINES] (R1 R2 is even: 16-byte aligned)
  const int nj = 2 * Kb + 1;
  const int atiles = N / LINES;
  for (int i = threadIdx.x; i < R1 * R2; i += blockDim.x) TW[i] = twN[i];
  auto issue = [&](int t, int b) {
    const long long fk = (long long)f0 * (Kc + 1) + t / atiles;
    const C *src = reinterpret_cast<const C *>(pa) + fk * nj * N + (t % atiles) * LINES;
    C *dst = Ys + b * nj * LINES;
    for (int i = threadIdx.x; i < nj * CH; i += blockDim.x) {
      const int jj = i / CH, c = i - jj * CH;
      const unsigned d = (unsigned)__cvta_generic_to_shared(dst + jj * LINES + c * CPC);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + (long long)jj * N + c * CPC)
                   : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  int b = 0;
  if ((int)blockIdx.x < ntiles) issue(blockIdx.x, 0);
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    if (t + (int)gridDim.x < ntiles) {
      issue(t + gridDim.x, b ^ 1);  // buffer b ^ 1 was last read before the previous tile's second barrier
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    __syncthreads();  // this tile's band lines; the previous tile's pass 2 is done with T
    const C *Y = Ys + b * nj * LINES;
    const long long fk = (long long)f0 * (Kc + 1) + t / atiles;
    const int a0 = (t % atiles) * LINES;
    for (int task = threadIdx.x; task < R2 * LINES; task += blockDim.x) {
      const int k2 = task / LINES, l = task - k2 * LINES;
      C v[R1];
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) {
        const int kk = k2 + R2 * k1;
        C z{(S)0, (S)0};
        if (k1 >= B && k1 < R1 - B) {
          // outside the band's rows: zero
        } else if (kk <= Kb) {
          z = Y[kk * LINES + l];  // b-frequency kk
        } else if (kk >= N - Kb) {
          z = Y[(kk - N + nj) * LINES + l];  // b-frequency kk - N
        }
        v[k1] = z;
      }
      dft_inv<S, R1, band_mask(R1, B)>(v, tw);
#pragma unroll
      for (int m1 = 0; m1 < R1; ++m1) {
        C y = v[m1];
        if (m1 > 0) y = c_mul(y, TW[m1 * R2 + k2]);
        T[m1 * TS + k2 * LINES + l] = y;
      }
    }
    __syncthreads();
    C *dst = reinterpret_cast<C *>(pb) + (fk * N + a0) * N;
    for (int task = threadIdx.x; task < R1 * LINES; task += blockDim.x) {
      const int l = task / R1, m1 = task - l * R1;
      C u[R2];
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) u[k2] = T[m1 * TS + k2 * LINES + l];
      dft_inv<S, R2>(u, tw);
      C *row = dst + (long long)l * N;
#pragma unroll
      for (int m2 = 0; m2 < R2; ++m2) row[m1 + R1 * m2] = u[m2];
    }
    b ^= 1;
  }
}

// Pass-B shapes (N = R1 x R2, LINES lines per CTA, R2 x LINES threads).
struct PbShape {
  int R1, R2, lines;
};
static bool pb_shape(long long N, size_t word, PbShape *sh) {
  if (word != 4 || N < 32 || N > 1024 || (N & (N - 1))) return false;
  switch (N) {
    case 32: *sh = PbShape{8, 4, 16}; break;
    case 64: *sh = PbShape{8, 8, 16}; break;
    case 128: *sh = PbShape{16, 8, 16}; break;
    case 256: *sh = PbShape{16, 16, 16}; break;
    case 512: *sh = PbShape{32, 16, 8}; break;  // 8 lines: 42 KB of shared memory, 5 CTAs per SM
    default: *sh = PbShape{32, 32, 8}; break;
  }
  return true;
}
static size_t pb_fused_smem(const cf_ctx *ctx, const PbShape &sh) {  // T, TW, 2 Ys buffers
  return ((size_t)sh.R1 * (sh.R2 * sh.lines + 1) + (size_t)sh.R1 * sh.R2 + 2 * (size_t)(2 * ctx->Kb + 1) * sh.lines) *
         2 * ctx->word;
}

template <typename S, int R1, int R2, int LINES, int B>
static int launch_pb_fused_b(cf_ctx *ctx, size_t smem, cudaStream_t st, int f0, int nf) {
  using C = typename Cplx<S>::T;
  auto kern = k_pass_b_fft<S, R1, R2, LINES, B>;
  if (smem > 48 * 1024) CF_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  Tw32<S> tw;
  for (int e = 0; e < 16; ++e) {
    const double ang = 2.0 * 3.14159265358979323846 * e / 32.0;
    tw.w[e] = C{(S)std::cos(ang), (S)std::sin(ang)};
  }
  const int N = (int)ctx->N;
  const int ntiles = nf * (ctx->Kc + 1) * (N / LINES);
  int sms = 0, per_sm = 0;
  CF_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
  CF_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, R2 * LINES, smem));
  const int grid = std::max(1, std::min(ntiles, sms * std::max(per_sm, 1)));
  kern<<<(unsigned)grid, R2 * LINES, smem, st>>>((const S *)ctx->pz_a2, (S *)ctx->pz_b, (const C *)ctx->pr_twB, N,
                                                 ctx->Kb, ctx->Kc, f0, ntiles, tw);
  CF_LAUNCHED(ctx);
  return CF_OK;
}

// The smallest compiled band B >= ceil((Kb+1)/R2) (2, 3, 4, 6 or all rows).
template <typename S, int R1, int R2, int LINES>
static int launch_pb_fused_t(cf_ctx *ctx, size_t smem, cudaStream_t st, int f0, int nf) {
  const int need = (ctx->Kb + 1 + R2 - 1) / R2;
  if constexpr (R1 >= 16) {
    if (need <= 2) return launch_pb_fused_b<S, R1, R2, LINES, 2>(ctx, smem, st, f0, nf);
    if (need <= 3) return launch_pb_fused_b<S, R1, R2, LINES, 3>(ctx, smem, st, f0, nf);
    if (need <= 4) return launch_pb_fused_b<S, R1, R2, LINES, 4>(ctx, smem, st, f0, nf);
    if (need <= 6) return launch_pb_fused_b<S, R1, R2, LINES, 6>(ctx, smem, st, f0, nf);
  }
  return launch_pb_fused_b<S, R1, R2, LINES, R1 / 2>(ctx, smem, st, f0, nf);
}

static int launch_pb_fused(cf_ctx *ctx, cudaStream_t st, int f0 = 0, int nf = 2) {
  PbShape sh;
  if (!pb_shape(ctx->N, ctx->word, &sh)) return set_error("fused pass B: unsupported N"), CF_ERR_INVALID;
  const size_t smem = pb_fused_smem(ctx, sh);
#define CF_PB(r1, r2, ln) \
  if (sh.R1 == r1 && sh.R2 == r2 && sh.lines == ln) return launch_pb_fused_t<float, r1, r2, ln>(ctx, smem, st, f0, nf);
  CF_PB(8, 4, 16)
  CF_PB(8, 8, 16)
  CF_PB(16, 8, 16)
  CF_PB(16, 16, 16)
  CF_PB(32, 16, 8)
  CF_PB(32, 32, 8)
#undef CF_PB
  set_error("fused pass B: no kernel for R1=%d R2=%d lines=%d", sh.R1, sh.R2, sh.lines);
  return CF_ERR_INVALID;
}

// Psi -> e^{2 Psi} - 1 in place after a cuFFT C2R (the slot's first field).
static int psi_to_e2m1(cf_ctx *ctx, void *f, cudaStream_t st) {
  ProfScope ps(ctx, CF_PROF_PSI_TRANSFER, st);
  const long long n = ctx->N3;
  const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16);
  if (ctx->word == 8)
    k_psi_to_e2m1<double><<<blocks, 256, 0, st>>>((double *)f, n);
  else
    k_psi_to_e2m1<float><<<blocks, 256, 0, st>>>((float *)f, n);
  CF_LAUNCHED(ctx);
  return CF_OK;
}

// Pass-C shapes (M = N/2 = R1 x R2) and rows per CTA: staging tile <= ~64 KB.
struct PcShape {
  int R1, R2, rows;
};
static bool pc_shape(long long N, size_t word, PcShape *sh) {
  if (N < 32 || N > 2048 || (N & (N - 1))) return false;
  const int M = (int)(N / 2);
  int R1 = 4, R2 = 4;
  switch (M) {
    case 16: R1 = 4, R2 = 4; break;
    case 32: R1 = 8, R2 = 4; break;
    case 64: R1 = 8, R2 = 8; break;
    case 128: R1 = 16, R2 = 8; break;
    case 256: R1 = 16, R2 = 16; break;
    case 512: R1 = 32, R2 = 16; break;
    default: R1 = 32, R2 = 32; break;
  }
  int rows = 16;
  while (rows > 4 && (size_t)M * rows * 2 * word > 64 * 1024) rows /= 2;
  *sh = PcShape{R1, R2, rows};
  return true;
}
// Pass C kernel per storage type, measured at N = 512 (Psi synthesis per RK4 step,
// two refreshes): FP64 k_prune_c_fft_p 1.79 ms against k_prune_c_fft 2.08; FP32
// k_prune_c_fft 0.90 ms against k_prune_c_fft_p 0.91 (0.92 with 5 CTAs/SM forced).
// Both give the same bits.
static bool pc_persistent(const cf_ctx *ctx) { return ctx->word == 8; }
static size_t pc_fused_smem(const cf_ctx *ctx, const PcShape &sh) {
  if (pc_persistent(ctx))  // X, T, TW, w^k
    return ((size_t)(ctx->Kc + 1) * sh.rows + (size_t)sh.R1 * (sh.R2 * sh.rows + 1) + (size_t)sh.R1 * sh.R2 +
            (size_t)(ctx->Kc + 1)) * 2 * ctx->word;
  return ((size_t)sh.R1 * (sh.R2 * sh.rows + 1) + (size_t)sh.R1 * sh.R2 + 2 * (size_t)(ctx->Kc + 1) * sh.rows) * 2 *
         ctx->word;
}

template <typename S, int R1, int R2, int ROWS, int B>
static int launch_pc_fused_b(cf_ctx *ctx, void *out, size_t smem, cudaStream_t st) {
  using C = typename Cplx<S>::T;
  Tw32<S> tw;
  for (int e = 0; e < 16; ++e) {
    const double ang = 2.0 * 3.14159265358979323846 * e / 32.0;
    tw.w[e] = C{(S)std::cos(ang), (S)std::sin(ang)};
  }
  const int N = (int)ctx->N;
  if constexpr (sizeof(S) == 8) {  // pc_persistent: one CTA per resident slot
    auto kern = k_prune_c_fft_p<S, R1, R2, ROWS, B>;
    if (smem > 48 * 1024) CF_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int sms = 0, per_sm = 0;
    CF_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    CF_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem));
    const int ntiles = 2 * N * (N / ROWS);
    const int grid = std::max(1, std::min(ntiles, sms * std::max(per_sm, 1)));
    kern<<<grid, 256, smem, st>>>((const S *)ctx->pz_b, (S *)out, (const C *)ctx->pr_wN, (const C *)ctx->pr_twM, N,
                                  ctx->Kc, ntiles, tw);
  } else {
    auto kern = k_prune_c_fft<S, R1, R2, ROWS, B>;
    if (smem > 48 * 1024) CF_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<dim3(N / ROWS, N, 2), 256, smem, st>>>((const S *)ctx->pz_b, (S *)out, (const C *)ctx->pr_wN,
                                                   (const C *)ctx->pr_twM, N, ctx->Kc, tw);
  }
  CF_LAUNCHED(ctx);
  return CF_OK;
}

// The smallest compiled band B >= ceil((Kc+1)/R2) (2, 3, 4, 6 or all rows).
template <typename S, int R1, int R2, int ROWS>
static int launch_pc_fused_t(cf_ctx *ctx, void *out, size_t smem, cudaStream_t st) {
  const int need = (ctx->Kc + 1 + R2 - 1) / R2;
  if constexpr (R1 >= 16) {
    if (need <= 2) return launch_pc_fused_b<S, R1, R2, ROWS, 2>(ctx, out, smem, st);
    if (need <= 3) return launch_pc_fused_b<S, R1, R2, ROWS, 3>(ctx, out, smem, st);
    if (need <= 4) return launch_pc_fused_b<S, R1, R2, ROWS, 4>(ctx, out, smem, st);
    if (need <= 6) return launch_pc_fused_b<S, R1, R2, ROWS, 6>(ctx, out, smem, st);
  }
  return launch_pc_fused_b<S, R1, R2, ROWS, R1 / 2>(ctx, out, smem, st);
}

template <typename S>
static int launch_pc_fused(cf_ctx *ctx, void *out, cudaStream_t st) {
  PcShape sh;
  if (!pc_shape(ctx->N, sizeof(S), &sh)) return set_error("fused pass C: unsupported N"), CF_ERR_INVALID;
  const size_t smem = pc_fused_smem(ctx, sh);
#define CF_PC(r1, r2, rw) \
  if (sh.R1 == r1 && sh.R2 == r2 && sh.rows == rw) return launch_pc_fused_t<S, r1, r2, rw>(ctx, out, smem, st);
  CF_PC(4, 4, 16)
  CF_PC(8, 4, 16)
  CF_PC(8, 8, 16)
  CF_PC(16, 8, 16)
  CF_PC(16, 16, 16)
  CF_PC(32, 16, 16)
  CF_PC(32, 16, 8)
  CF_PC(32, 32, 8)
  CF_PC(32, 32, 4)
#undef CF_PC
  set_error("fused pass C: no kernel for R1=%d R2=%d rows=%d", sh.R1, sh.R2, sh.rows);
  return CF_ERR_INVALID;
}

// Shared memory of k_prune_c's (Kc+1) x 33 complex tile, and the most it may take.
static size_t prune_c_smem(const cf_ctx *ctx) { return (size_t)(ctx->Kc + 1) * 33 * 2 * ctx->word; }
static constexpr size_t kPruneCSmemMax = 200 * 1024;
static constexpr size_t kPcFusedSmemMax = 200 * 1024;

template <typename S>
__global__ void k_copy_convert(const double *__restrict__ in, S *__restrict__ out, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = (S)in[i];
}

// Slots [slots_alloc, n): 2 N^3 words each and their ready events.
static int alloc_psi_slots(cf_ctx *ctx, int n) {
  const size_t w = ctx->word;
  for (; ctx->slots_alloc < n; ++ctx->slots_alloc) {
    PsiSlot &s = ctx->slot[ctx->slots_alloc];
    if (cudaMalloc(&s.psi, 2 * (size_t)ctx->N3 * w) != cudaSuccess) {
      s.psi = nullptr;
      (void)cudaGetLastError();
      set_error("cudaMalloc Psi slot failed");
      return CF_ERR_NOMEM;
    }
    s.dpsi = (char *)s.psi + (size_t)ctx->N3 * w;
    s.valid = false;
    CF_TRY_CUDA(cudaEventCreateWithFlags(&s.ready, cudaEventDisableTiming));
  }
  return CF_OK;
}

int ensure_psi(cf_ctx *ctx) {
  if (ctx->psi_table) return CF_OK;  // buffers in place
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
  return alloc_psi_slots(ctx, 3);
}

// The two padded HC arrays (Psi_k, dPsi_k) that the cuFFT C2R routes read:
// allocated when a refresh first takes one of them.
static int ensure_psi_hc(cf_ctx *ctx) {
  if (ctx->psi_hc) return CF_OK;
  const size_t bytes = 2 * (size_t)ctx->hc_count * ctx->word;
  if (cudaMalloc(&ctx->psi_hc, bytes) != cudaSuccess) {
    cudaGetLastError();
    set_error("cudaMalloc Psi transfer buffers (%zu bytes) failed", bytes);
    return CF_ERR_NOMEM;
  }
  return CF_OK;
}

// The batched 3-D C2R of the full synthesis (created when a refresh first takes
// the full path, so the pruned path does not hold its work area).
static int ensure_full_plan(cf_ctx *ctx) {
  if (ctx->have_plan_psi) return CF_OK;
  const int N = (int)ctx->N;
  const size_t w = ctx->word;
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

static void free_pruned(cf_ctx *ctx) {
  if (!ctx->have_pruned) return;
  cudaFree(ctx->pz_a);
  cudaFree(ctx->pz_a2);
  cudaFree(ctx->pz_b);
  cudaFree(ctx->pr_wN);
  cudaFree(ctx->pr_twM);
  cudaFree(ctx->pr_twB);
  cufftDestroy(ctx->plan_pa);
  if (!ctx->pb_fused) cufftDestroy(ctx->plan_pb);
  if (!ctx->pc_fused) cufftDestroy(ctx->plan_pc);
  ctx->pz_a = ctx->pz_a2 = ctx->pz_b = ctx->pr_wN = ctx->pr_twM = ctx->pr_twB = nullptr;
  ctx->pa_last_valid = false;
  ctx->have_pc_tmap = false;
  ctx->have_pruned = false;
}

void psi_release(cf_ctx *ctx) { free_pruned(ctx); }

static int ensure_pruned(cf_ctx *ctx, cudaStream_t st) {
  if (ctx->have_pruned && ctx->pr_Ka == ctx->Ka && ctx->pr_Kb == ctx->Kb && ctx->pr_Kc == ctx->Kc) return CF_OK;
  free_pruned(ctx);
  const long long N = ctx->N, nh = N / 2 + 1;
  const long long nj = 2 * ctx->Kb + 1, nk = ctx->Kc + 1;
  const size_t cb = 2 * ctx->word;  // bytes per complex
  if (cudaMalloc(&ctx->pz_a, 2 * nk * nj * N * cb) != cudaSuccess ||
      cudaMalloc(&ctx->pz_a2, 2 * nk * nj * N * cb) != cudaSuccess ||
      cudaMalloc(&ctx->pz_b, 2 * nk * N * N * cb) != cudaSuccess) {
    cudaGetLastError();
    set_error("cudaMalloc of the pruned Psi buffers failed");
    return CF_ERR_NOMEM;
  }
  // the zeros of pass A's input lines outside the band (k_prune_a writes the band only)
  CF_TRY_CUDA(cudaMemsetAsync(ctx->pz_a, 0, 2 * nk * nj * N * cb, st));
  const bool dp = ctx->word == 8;
  long long n1[1] = {N};
  size_t work = 0;
  CF_TRY_CUFFT(cufftCreate(&ctx->plan_pa));
  CF_TRY_CUFFT(cufftMakePlanMany64(ctx->plan_pa, 1, n1, nullptr, 1, N, nullptr, 1, N, dp ? CUFFT_Z2Z : CUFFT_C2C,
                                   2 * nk * nj, &work));
  PbShape bsh;
  ctx->pb_fused = pb_shape(N, ctx->word, &bsh) && pb_fused_smem(ctx, bsh) <= kPcFusedSmemMax;
  if (ctx->pb_fused) {
    // pass-B four-step twiddles e^{2 pi i k2 m1 / N}, laid out [m1][k2] (FP32)
    std::vector<float> t(2 * N);
    for (int m1 = 0; m1 < bsh.R1; ++m1)
      for (int k2 = 0; k2 < bsh.R2; ++k2) {
        const double ang = 2.0 * 3.14159265358979323846 * (double)((long long)k2 * m1 % N) / (double)N;
        t[2 * (m1 * bsh.R2 + k2)] = (float)std::cos(ang);
        t[2 * (m1 * bsh.R2 + k2) + 1] = (float)std::sin(ang);
      }
    if (cudaMalloc(&ctx->pr_twB, (size_t)N * cb) != cudaSuccess) {
      cudaGetLastError();
      set_error("cudaMalloc of the pass-B twiddles failed");
      return CF_ERR_NOMEM;
    }
    CF_TRY_CUDA(cudaMemcpy(ctx->pr_twB, t.data(), (size_t)N * cb, cudaMemcpyHostToDevice));
  } else {
    CF_TRY_CUFFT(cufftCreate(&ctx->plan_pb));
    CF_TRY_CUFFT(cufftMakePlanMany64(ctx->plan_pb, 1, n1, nullptr, 1, N, nullptr, 1, N, dp ? CUFFT_Z2Z : CUFFT_C2C,
                                     2 * nk * N, &work));
  }
  PcShape sh;
  ctx->pc_fused = pc_shape(N, ctx->word, &sh) && pc_fused_smem(ctx, sh) <= kPcFusedSmemMax;
  if (ctx->pc_fused) {
    // e^{2 pi i j / N}, j < N, from the host's double-precision cos / sin
    std::vector<double> w(2 * N);
    for (long long j = 0; j < N; ++j) {
      const double ang = 2.0 * 3.14159265358979323846 * (double)j / (double)N;
      w[2 * j] = std::cos(ang);
      w[2 * j + 1] = std::sin(ang);
    }
    // pass-1 twiddles e^{2 pi i k2 m1 / M} = w^{2 k2 m1}, laid out [m1][k2]
    const long long M = N / 2;
    std::vector<double> t(2 * M);
    for (int m1 = 0; m1 < sh.R1; ++m1)
      for (int k2 = 0; k2 < sh.R2; ++k2) {
        const long long e = (2LL * k2 * m1) % N;
        t[2 * (m1 * sh.R2 + k2)] = w[2 * e];
        t[2 * (m1 * sh.R2 + k2) + 1] = w[2 * e + 1];
      }
    if (cudaMalloc(&ctx->pr_wN, (size_t)N * cb) != cudaSuccess ||
        cudaMalloc(&ctx->pr_twM, (size_t)M * cb) != cudaSuccess) {
      cudaGetLastError();
      set_error("cudaMalloc of the pass-C twiddles failed");
      return CF_ERR_NOMEM;
    }
    if (dp) {
      CF_TRY_CUDA(cudaMemcpy(ctx->pr_wN, w.data(), (size_t)N * cb, cudaMemcpyHostToDevice));
      CF_TRY_CUDA(cudaMemcpy(ctx->pr_twM, t.data(), (size_t)M * cb, cudaMemcpyHostToDevice));
    } else {
      std::vector<float> wf(w.begin(), w.end()), tf(t.begin(), t.end());
      CF_TRY_CUDA(cudaMemcpy(ctx->pr_wN, wf.data(), (size_t)N * cb, cudaMemcpyHostToDevice));
      CF_TRY_CUDA(cudaMemcpy(ctx->pr_twM, tf.data(), (size_t)M * cb, cudaMemcpyHostToDevice));
    }
  } else {
    CF_TRY(ensure_psi_hc(ctx));
    long long ie[1] = {nh}, oe[1] = {N};
    CF_TRY_CUFFT(cufftCreate(&ctx->plan_pc));
    CF_TRY_CUFFT(cufftMakePlanMany64(ctx->plan_pc, 1, n1, ie, 1, nh, oe, 1, N, dp ? CUFFT_Z2D : CUFFT_C2R,
                                     2 * N * N, &work));
  }
  if (!(ctx->p.flags & CF_FLAG_PSI_NO_TMA)) CF_TRY(encode_pc_tmap(ctx));
  if (ctx->word == 4 && !ctx->pa_diff_h) {
    CF_TRY_CUDA(cudaHostAlloc((void **)&ctx->pa_diff_h, sizeof(int), cudaHostAllocMapped));
    *ctx->pa_diff_h = 0;
    CF_TRY_CUDA(cudaHostGetDevicePointer((void **)&ctx->pa_diff_d, ctx->pa_diff_h, 0));
    CF_TRY_CUDA(cudaEventCreateWithFlags(&ctx->pa_check, cudaEventDisableTiming));
  }
  ctx->pa_last_valid = false;
  ctx->have_pruned = true;
  ctx->pr_Ka = ctx->Ka;
  ctx->pr_Kb = ctx->Kb;
  ctx->pr_Kc = ctx->Kc;
  return CF_OK;
}

// check: compare pass A's inputs with those of the latest refresh (in pz_a) and, when
// they are identical, set *same and stop there (the caller takes that refresh's slot).
// The host waits for the comparison, so the caller issues it where the GPU has other
// work queued (the side stream of cf_rk4_steps, behind an enqueued step).
template <typename S>
static int refresh_pruned(cf_ctx *ctx, void *out, cudaStream_t st, bool check = false, bool *same = nullptr) {
  const int N = (int)ctx->N, Ka = ctx->Ka, Kb = ctx->Kb, Kc = ctx->Kc;
  const int nj = 2 * Kb + 1;
  check = check && ctx->pa_last_valid;
  if (check) *reinterpret_cast<volatile int *>(ctx->pa_diff_h) = 0;  // no kernel holds it: the last check was waited for
  {
    ProfScope ps(ctx, CF_PROF_PSI_TRANSFER, st);
    const int na = 2 * Ka + 1;
    k_prune_a<S><<<dim3((na + 127) / 128, nj, Kc + 1), 128, 0, st>>>(
        (const S *)ctx->R_fft, ctx->psi_table, (S *)ctx->pz_a, N, Ka, Kb, Kc, check ? ctx->pa_diff_d : nullptr);
    CF_LAUNCHED(ctx);
  }
  if (check) {
    CF_TRY_CUDA(cudaEventRecord(ctx->pa_check, st));
    CF_TRY_CUDA(cudaEventSynchronize(ctx->pa_check));
    if (*reinterpret_cast<volatile int *>(ctx->pa_diff_h) == 0) {
      *same = true;
      return CF_OK;
    }
  }
  {
    ProfScope ps(ctx, CF_PROF_PSI_FFT, st);
    CF_TRY_CUFFT(cufftSetStream(ctx->plan_pa, st));
    if (ctx->word == 8)
      CF_TRY_CUFFT(cufftExecZ2Z(ctx->plan_pa, (cufftDoubleComplex *)ctx->pz_a, (cufftDoubleComplex *)ctx->pz_a2,
                                CUFFT_INVERSE));
    else
      CF_TRY_CUFFT(cufftExecC2C(ctx->plan_pa, (cufftComplex *)ctx->pz_a, (cufftComplex *)ctx->pz_a2, CUFFT_INVERSE));
  }
  int R1w = 0, R2w = 0;
  const bool warp_c = ctx->pc_fused && !(ctx->p.flags & CF_FLAG_PSI_CTA_PASS_C) &&
                      pc_warp_shape(ctx->N, ctx->word, &R1w, &R2w) && pc_warp_smem(ctx->Kc, R1w, R2w, pc_warp_tma(ctx)) <= kPcFusedSmemMax;
  if (ctx->pb_fused) {
    ProfScope ps(ctx, CF_PROF_PSI_FFT, st);
    CF_TRY(launch_pb_fused(ctx, st));
  } else {
    {
      ProfScope ps(ctx, CF_PROF_PSI_TRANSFER, st);
      k_prune_b<S><<<dim3((N + 255) / 256, N, 2 * (Kc + 1)), 256, 0, st>>>((const S *)ctx->pz_a2, (S *)ctx->pz_b, N,
                                                                           Kb, Kc);
      CF_LAUNCHED(ctx);
    }
    ProfScope ps(ctx, CF_PROF_PSI_FFT, st);
    CF_TRY_CUFFT(cufftSetStream(ctx->plan_pb, st));
    if (ctx->word == 8)
      CF_TRY_CUFFT(cufftExecZ2Z(ctx->plan_pb, (cufftDoubleComplex *)ctx->pz_b, (cufftDoubleComplex *)ctx->pz_b,
                                CUFFT_INVERSE));
    else
      CF_TRY_CUFFT(cufftExecC2C(ctx->plan_pb, (cufftComplex *)ctx->pz_b, (cufftComplex *)ctx->pz_b, CUFFT_INVERSE));
  }
  if (ctx->pc_fused) {
    ProfScope ps(ctx, CF_PROF_PSI_FFT, st);
    if (warp_c) return launch_pc_warp(ctx, out, st);
    return launch_pc_fused<S>(ctx, out, st);
  }
  {
    ProfScope ps(ctx, CF_PROF_PSI_TRANSFER, st);
    const size_t smem = prune_c_smem(ctx);
    if (smem > 48 * 1024)
      CF_TRY_CUDA(cudaFuncSetAttribute(k_prune_c<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_prune_c<S><<<dim3(N / 32, N, 2), 256, smem, st>>>((const S *)ctx->pz_b, (S *)ctx->psi_hc, N, Kc);
    CF_LAUNCHED(ctx);
  }
  {
    ProfScope ps(ctx, CF_PROF_PSI_FFT, st);
    CF_TRY_CUFFT(cufftSetStream(ctx->plan_pc, st));
    if (ctx->word == 8)
      CF_TRY_CUFFT(cufftExecZ2D(ctx->plan_pc, (cufftDoubleComplex *)ctx->psi_hc, (cufftDoubleReal *)out));
    else
      CF_TRY_CUFFT(cufftExecC2R(ctx->plan_pc, (cufftComplex *)ctx->psi_hc, (cufftReal *)out));
  }
  return psi_to_e2m1(ctx, out, st);
}

// Synthesises Psi, dPsi/dt at t into slot v on stream st and records the slot's event.
// cand (may be null): the slot of the latest refresh (pa_last_t), for a time t a few ulp
// from it; when pass A's inputs at t equal that refresh's bit for bit, t becomes cand's
// second time instead of a new synthesis into v.
static int refresh_slot(cf_ctx *ctx, PsiSlot *v, double t, cudaStream_t st, PsiSlot *cand = nullptr) {
  if (ctx->psi_err_h && *reinterpret_cast<volatile int *>(ctx->psi_err_h)) {
    // some earlier refresh left its slot incomplete: none of the cached slots is trusted
    for (int i = 0; i < kPsiSlots; ++i) ctx->slot[i].valid = false;
    ctx->pa_last_valid = false;
    return set_error("Psi synthesis: a band copy of pass C did not land within its wait limit"), CF_ERR_TIMEOUT;
  }
  const double eta_t = cosmo_eta(ctx->p, t);
  const double H_t = cosmo_H(ctx->p, t);
  const double factor = (2 * 3.14159265358979323846 / ctx->p.L) * eta_t / sqrt(3);
  const long long pairs = ctx->hc_count / 2;
  v->valid = false;
  {
    ProfScope ps(ctx, CF_PROF_PSI_TRANSFER, st);
    unsigned tb = (unsigned)std::min<long long>((ctx->s2_bins + 255) / 256, 148LL * 8);
    k_transfer_table<<<tb, 256, 0, st>>>(ctx->psi_table, ctx->s2_bins, (int)ctx->N, factor, H_t);
    CF_LAUNCHED(ctx);
  }
  if (ctx->pruned) {
    CF_TRY(ensure_pruned(ctx, st));
    if (ctx->word == 8) {
      CF_TRY(refresh_pruned<double>(ctx, v->psi, st));
    } else {
      bool same = false;
      const int rc = refresh_pruned<float>(ctx, v->psi, st, cand != nullptr, &same);
      if (rc != CF_OK) {
        ctx->pa_last_valid = false;
        return rc;
      }
      if (same) {
        cand->t_alt = t;
        cand->has_alt = true;
        cand->stamp = ++ctx->slot_clock;
        ctx->pa_last_t = t;
        ctx->psi_reuses++;
        return CF_OK;
      }
      ctx->pa_last_t = t;
      ctx->pa_last_valid = true;
    }
  } else {
    CF_TRY(ensure_psi_hc(ctx));
    CF_TRY(ensure_full_plan(ctx));
    CF_TRY_CUFFT(cufftSetStream(ctx->plan_psi, st));
    {
      ProfScope ps(ctx, CF_PROF_PSI_TRANSFER, st);
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
    CF_TRY(psi_to_e2m1(ctx, v->psi, st));
  }
  CF_TRY_CUDA(cudaEventRecord(v->ready, st));
  v->t = t;
  v->has_alt = false;
  v->valid = true;
  v->stamp = ++ctx->slot_clock;
  ctx->psi_refreshes++;
  return CF_OK;
}

static bool slot_holds(const PsiSlot &s, double t) { return s.valid && (s.t == t || (s.has_alt && s.t_alt == t)); }

static PsiSlot *cached_slot(cf_ctx *ctx, double t) {
  for (int i = 0; i < ctx->slots_alloc; ++i)
    if (slot_holds(ctx->slot[i], t)) return &ctx->slot[i];
  return nullptr;
}

int psi_at(cf_ctx *ctx, double t, cudaStream_t st, const void **psi, const void **dpsi) {
  CF_TRY(ensure_psi(ctx));
  PsiSlot *v = cached_slot(ctx, t);
  if (!v) {  // refresh the least recently used slot
    v = &ctx->slot[0];
    for (int i = 0; i < ctx->slots_alloc; ++i)
      if (!ctx->slot[i].valid || ctx->slot[i].stamp < v->stamp) v = &ctx->slot[i];
    CF_TRY(refresh_slot(ctx, v, t, st));
  }
  v->stamp = ++ctx->slot_clock;
  *psi = v->psi;
  *dpsi = v->dpsi;
  return CF_OK;
}

// ---- refreshes beside the stepping ----------------------------------------
// Psi depends on t only, so the new slots of step j + 1 (two, or three when its start
// time differs from t + dt in the last bit) can be synthesised on a side stream while
// step j's passes run: the refreshes (passes A-C, about a third of a step at N = 512)
// fill the SMs the step's last wave leaves idle.  Six slots: step j reads three, the
// side stream fills the next step's, and a fill overwrites a slot only after the step
// that last read it has finished (psi_stepdone).  The fork and the join are events on
// the caller's stream, so work enqueued after cf_rk4_steps sees every slot complete.
int psi_pipe_begin(cf_ctx *ctx, cudaStream_t st, bool *on) {
  CF_TRY(ensure_psi(ctx));
  *on = false;
  if (alloc_psi_slots(ctx, kPsiSlots) != CF_OK) return CF_OK;  // no room: the caller refreshes in turn
  if (!ctx->psi_side) {
    // default priority: the refreshes take the SMs the step's last wave leaves idle.
    // At the highest priority they displaced the step's CTAs as they retired: N = 256
    // 0.457 -> 0.393 ms per step, but N = 512 2.63 -> 2.68 (the step pass 1.69 ->
    // 2.48 ms) against 2.57 at default priority.
    CF_TRY_CUDA(cudaStreamCreateWithFlags(&ctx->psi_side, cudaStreamNonBlocking));
    CF_TRY_CUDA(cudaEventCreateWithFlags(&ctx->psi_fork, cudaEventDisableTiming));
    CF_TRY_CUDA(cudaEventCreateWithFlags(&ctx->psi_join, cudaEventDisableTiming));
    CF_TRY_CUDA(cudaEventCreateWithFlags(&ctx->psi_stepdone, cudaEventDisableTiming));
  }
  // the side stream starts behind everything enqueued on st (slots read earlier)
  CF_TRY_CUDA(cudaEventRecord(ctx->psi_fork, st));
  CF_TRY_CUDA(cudaStreamWaitEvent(ctx->psi_side, ctx->psi_fork, 0));
  *on = true;
  return CF_OK;
}

// A time a few ulp from the latest FP32 pruned refresh (the next step's t0 + (n + 1) dt
// against this step's t + dt, at about a third of the steps for dt = 0.05 from t = 1)
// is first checked against it on the side stream: the host waits for the comparison
// while the GPU runs the step enqueued before it.
int psi_pipe_fill(cf_ctx *ctx, double t, const double *keep, int nkeep) {
  if (cached_slot(ctx, t)) return CF_OK;
  PsiSlot *v = nullptr;
  for (int i = 0; i < ctx->slots_alloc; ++i) {
    PsiSlot *s = &ctx->slot[i];
    bool kept = false;
    for (int k = 0; k < nkeep; ++k) kept = kept || slot_holds(*s, keep[k]);
    if (kept) continue;
    if (!v || !s->valid || (v->valid && s->stamp < v->stamp)) v = s;
    if (!v->valid) break;
  }
  if (!v) return set_error("Psi slots: no slot outside the kept stage times"), CF_ERR_INVALID;
  PsiSlot *cand = nullptr;
  if (ctx->pruned && ctx->word == 4 && ctx->pa_last_valid && !(ctx->p.flags & CF_FLAG_PSI_NO_REUSE) &&
      std::fabs(t - ctx->pa_last_t) <= 1e-12 * std::fmax(1.0, std::fabs(t))) {
    PsiSlot *c = cached_slot(ctx, ctx->pa_last_t);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CF_TRY_CUDA(cudaStreamIsCapturing(ctx->psi_side, &cs));
    if (c && !c->has_alt && c != v && cs == cudaStreamCaptureStatusNone) cand = c;
  }
  return refresh_slot(ctx, v, t, ctx->psi_side, cand);
}

int psi_pipe_use(cf_ctx *ctx, double t, cudaStream_t st, const void **psi, const void **dpsi) {
  PsiSlot *v = cached_slot(ctx, t);
  if (!v) return set_error("Psi slot for t = %g not filled", t), CF_ERR_INVALID;
  CF_TRY_CUDA(cudaStreamWaitEvent(st, v->ready, 0));
  v->stamp = ++ctx->slot_clock;
  *psi = v->psi;
  *dpsi = v->dpsi;
  return CF_OK;
}

int psi_pipe_step_done(cf_ctx *ctx, cudaStream_t st) {
  CF_TRY_CUDA(cudaEventRecord(ctx->psi_stepdone, st));
  CF_TRY_CUDA(cudaStreamWaitEvent(ctx->psi_side, ctx->psi_stepdone, 0));
  return CF_OK;
}

int psi_pipe_end(cf_ctx *ctx, cudaStream_t st) {
  CF_TRY_CUDA(cudaEventRecord(ctx->psi_join, ctx->psi_side));
  CF_TRY_CUDA(cudaStreamWaitEvent(st, ctx->psi_join, 0));
  return CF_OK;
}

int psi_route(const cf_ctx *ctx) {
  if (ctx->p.equation != CF_EQ_COMOVING_FRW || !ctx->R_fft) return CF_PSI_NONE;
  if (!ctx->pruned) return CF_PSI_FULL;
  PcShape sh;
  return (pc_shape(ctx->N, ctx->word, &sh) && pc_fused_smem(ctx, sh) <= kPcFusedSmemMax) ? CF_PSI_PRUNED_FUSED
                                                                                         : CF_PSI_PRUNED;
}

// Slot -> (Psi, dPsi/dt) in FP64: Psi = log1p(e^{2 Psi} - 1) / 2.
template <typename S>
__global__ void k_slot_to_fields(const S *__restrict__ e2m1, const S *__restrict__ dpsi, double *__restrict__ out,
                                 long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    out[i] = 0.5 * log1p((double)e2m1[i]);
    out[n + i] = (double)dpsi[i];
  }
}

int psi_fields(cf_ctx *ctx, double t, double *d_out, cudaStream_t st) {
  const void *psi = nullptr, *dpsi = nullptr;
  CF_TRY(psi_at(ctx, t, st, &psi, &dpsi));
  const long long n = ctx->N3;
  const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16);
  if (ctx->word == 8)
    k_slot_to_fields<double><<<blocks, 256, 0, st>>>((const double *)psi, (const double *)dpsi, d_out, n);
  else
    k_slot_to_fields<float><<<blocks, 256, 0, st>>>((const float *)psi, (const float *)dpsi, d_out, n);
  CF_LAUNCHED(ctx);
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
  if (ctx->p.equation == CF_EQ_APPROX_COMOVING_FRW) {
    // the coarse grid takes its modes from the FP64 input
    const int s = approx_set_R(ctx, w == 8 ? (const double *)ctx->R_fft : src, st);
    if (s != CF_OK) {
      if (tmp) cudaFreeAsync(tmp, st);
      return s;
    }
  }
  if (tmp) CF_TRY_CUDA(cudaFreeAsync(tmp, st));
  for (int i = 0; i < ctx->slots_alloc; ++i) ctx->slot[i].valid = false;
  ctx->pa_last_valid = false;
  // support of the new R_fft: decides between the pruned and the full synthesis
  int *d_box = nullptr;
  CF_TRY_CUDA(cudaMallocAsync((void **)&d_box, 3 * sizeof(int), st));
  CF_TRY_CUDA(cudaMemsetAsync(d_box, 0xff, 3 * sizeof(int), st));  // -1
  const dim3 sg(1, (unsigned)ctx->N, (unsigned)ctx->N);
  if (w == 8)
    k_support<double><<<sg, 128, 0, st>>>((const double *)ctx->R_fft, (int)ctx->N, d_box);
  else
    k_support<float><<<sg, 128, 0, st>>>((const float *)ctx->R_fft, (int)ctx->N, d_box);
  CF_LAUNCHED(ctx);
  int box[3];
  CF_TRY_CUDA(cudaMemcpyAsync(box, d_box, sizeof(box), cudaMemcpyDeviceToHost, st));
  CF_TRY_CUDA(cudaFreeAsync(d_box, st));
  CF_TRY_CUDA(cudaStreamSynchronize(st));
  ctx->Ka = std::max(box[0], 0);
  ctx->Kb = std::max(box[1], 0);
  ctx->Kc = std::max(box[2], 0);
  const int N = (int)ctx->N;
  // pruned when the box is small against the lattice: passes A and B then touch a
  // small fraction of the lines, and pass C's transpose tile fits shared memory
  PcShape sh;
  const bool pc_ok = (pc_shape(N, ctx->word, &sh) && pc_fused_smem(ctx, sh) <= kPcFusedSmemMax) ||
                     prune_c_smem(ctx) <= kPruneCSmemMax;
  ctx->pruned = !(ctx->p.flags & CF_FLAG_FULL_PSI_FFT) && N % 32 == 0 && 2 * ctx->Ka + 1 <= N / 2 &&
                2 * ctx->Kb + 1 <= N / 2 && ctx->Kc + 1 <= N / 4 && pc_ok;
  return CF_OK;
}

}  // namespace cfb
