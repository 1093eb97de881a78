// cf_spectrum.cu -- energy density, deterministic spectrum binning, spectra.
//
// The reference bins |f_k|^2 into s^2 bins with FP64 atomicAdd, whose result
// depends on the order the atomics land in (src/fdm3d_cuda.cu:3-27, comment at
// :25).  Here every mode value is converted to a 128-bit fixed-point integer
// whose scale is a power of two chosen from an order-independent upper bound on
// any bin -- the largest mode value times the entry count (a max pass over the
// modes), or for the density spectrum N^5 times the largest row sum of rho^2,
// formed by the energy pass itself (Parseval) -- and the bins accumulate those
// integers with 64-bit integer atomics (carry propagated to the high word).
// Integer addition is associative, so the bins are bit-reproducible, and the
// sums are exact up to the fixed-point resolution (2^-126 of the bound).
// Unit-width |k| shells are then exact integer regroupings of the s^2 bins.

#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>

#include "cf_internal.cuh"

namespace cfb {

// ---- energy density -----------------------------------------------------
// Potential term of the energy density by equation (ED_*):
//   ED_QUAD    1/2 m^2 phi^2                                (src/equations_cuda.cu:332-369, lambda = 0)
//   ED_LAMBDA  1/2 m^2 phi^2 + 1/4 lambda phi^4              (:332-369)
//   ED_SQRT    m^2 f_a^2 (sqrt(1 + phi^2/f_a^2) - 1)         (:431-449)
//   ED_CURV    1/2 m^2 phi^2 with e^{-2Psi} kinetic and e^{2Psi} gradient weights (:451-473)
// and rho = 1/2 pi^2 w_k + 1/8 inv w_g sum_axes (phi_{+1} - phi_{-1})^2 + V
// (src/equations.cpp:38-69, :106-138, :265-322 for the CPU twins).  `psi` holds
// e^{2 Psi} - 1.  The sqrt potential is formed as m^2 phi^2 / (sqrt(1 + phi^2/f_a^2) + 1),
// the same value without the cancellation of sqrt(1 + u) - 1 at small u.
enum EdKind : int { ED_QUAD = 0, ED_LAMBDA = 1, ED_SQRT = 2, ED_CURV = 3 };

// With `rowmax` set, the block also forms its row's sum of rho^2 (fixed order: the
// thread's c values in turn, then a shuffle tree, then the warps in turn) and folds it
// into *rowmax with an integer max of the bit pattern; N^2 times the largest row sum
// bounds sum_x rho^2, which Parseval turns into a bound on every spectrum bin.
template <typename S, int ED>
__global__ void __launch_bounds__(128) k_energy(const S *__restrict__ x, const S *__restrict__ xlo,
                                                const S *__restrict__ psi, double *__restrict__ rho, int N, double m2,
                                                double inv, double q, unsigned long long *__restrict__ rowmax) {
  // one lattice row (a, b) per block, threads along c: the row's neighbour rows are
  // found once, only c wraps per site
  double ss = 0.0;
  const long long N3 = (long long)N * N * N;
  const long long NN = (long long)N * N;
  const int a = (int)(blockIdx.x / (unsigned)N), b = (int)(blockIdx.x - (unsigned)a * (unsigned)N);
  const long long row = NN * a + (long long)N * b;
  const long long rap = NN * (a + 1 == N ? 0 : a + 1) + (long long)N * b;
  const long long ram = NN * (a == 0 ? N - 1 : a - 1) + (long long)N * b;
  const long long rbp = NN * a + (long long)N * (b + 1 == N ? 0 : b + 1);
  const long long rbm = NN * a + (long long)N * (b == 0 ? N - 1 : b - 1);
  auto phi = [&](long long i) -> double {
    double v = (double)x[i];
    if (xlo) v += (double)xlo[i];
    return v;
  };
  for (int c = threadIdx.x; c < N; c += blockDim.x) {
    const long long i = row + c;
    const int cp = c + 1 == N ? 0 : c + 1, cm = c == 0 ? N - 1 : c - 1;
    const double dx = phi(rap + c) - phi(ram + c), dy = phi(rbp + c) - phi(rbm + c), dz = phi(row + cp) - phi(row + cm);
    const double grad = dx * dx + dy * dy + dz * dz;
    const double f = phi(i);
    double p = (double)x[N3 + i];
    if (xlo) p += (double)xlo[N3 + i];
    double r;
    if constexpr (ED == ED_CURV) {
      const double e2 = 1.0 + (double)psi[i];
      r = 0.5 * (p * p / e2 + m2 * f * f + e2 * 0.25 * inv * grad);
    } else if constexpr (ED == ED_LAMBDA) {
      r = 0.5 * (p * p + m2 * f * f + 0.25 * inv * grad) + 0.25 * q * f * f * f * f;
    } else if constexpr (ED == ED_SQRT) {  // q = 1 / f_a^2
      r = 0.5 * (p * p + 0.25 * inv * grad) + m2 * f * f / (sqrt(1.0 + f * f * q) + 1.0);
    } else {
      r = 0.5 * (p * p + m2 * f * f + 0.25 * inv * grad);
    }
    rho[i] = r;
    ss += r * r;
  }
  if (!rowmax) return;  // uniform over the block
  __shared__ double part[4];
  for (int o = 16; o > 0; o >>= 1) ss += __shfl_down_sync(0xffffffffu, ss, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = ss;
  __syncthreads();
  if (threadIdx.x == 0) {
    const double t = ((part[0] + part[1]) + part[2]) + part[3];
    // non-negative doubles order like their bit patterns
    atomicMax(rowmax, (unsigned long long)__double_as_longlong(t));
  }
}

// d rho / dt of the FRW Klein-Gordon equation (src/equations_cuda.cu:372-424):
//   pi lap_inv + 1/4 inv sum_axes (dpi_e)(dphi_e) - 3H (rho + p),
//   rho = 1/2 pi^2 + 1/8 inv G + 1/2 m^2 phi^2,  p = 1/2 pi^2 - 1/2 m^2 phi^2 - 1/24 inv G,
// with dphi_e, dpi_e the central differences (phi_{+e} - phi_{-e}) along each axis,
// G = sum_e dphi_e^2 and lap_inv = inv times the 7-point Laplacian sum.
template <typename S>
__global__ void k_dot_energy(const S *__restrict__ x, const S *__restrict__ xlo, double *__restrict__ out, int N,
                             double m2, double inv, double H_t) {
  const long long N3 = (long long)N * N * N;
  const long long NN = (long long)N * N;
  const long long stride = (long long)gridDim.x * blockDim.x;
  auto val = [&](long long i) -> double {
    double v = (double)x[i];
    if (xlo) v += (double)xlo[i];
    return v;
  };
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N3; i += stride) {
    const int c = (int)(i % N);
    const int b = (int)((i / N) % N);
    const int a = (int)(i / NN);
    const long long nb[6] = {NN * ((a + 1) % N) + (long long)N * b + c, NN * ((a + N - 1) % N) + (long long)N * b + c,
                             NN * a + (long long)N * ((b + 1) % N) + c, NN * a + (long long)N * ((b + N - 1) % N) + c,
                             NN * a + (long long)N * b + (c + 1) % N, NN * a + (long long)N * b + (c + N - 1) % N};
    const double f = val(i), p = val(N3 + i);
    double G = 0.0, cross = 0.0, lap = -6.0 * f;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      const double fp = val(nb[2 * e]), fm = val(nb[2 * e + 1]);
      const double df = fp - fm;
      const double dp = val(N3 + nb[2 * e]) - val(N3 + nb[2 * e + 1]);
      G += df * df;
      cross += dp * df;
      lap += fp + fm;
    }
    const double rho = 0.5 * p * p + (0.5 / 4.0) * inv * G + 0.5 * m2 * f * f;
    const double pr = 0.5 * p * p - 0.5 * m2 * f * f - (1.0 / 4.0 / 6.0) * inv * G;
    out[i] = p * (inv * lap) + 0.25 * inv * cross - 3.0 * H_t * (rho + pr);
  }
}

// FP32_COMP state -> FP64 [phi | pi] (hi + lo).
__global__ void k_export_f32(const float *__restrict__ s, double *__restrict__ out, long long n2) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += stride)
    out[i] = (double)s[i] + (double)s[n2 + i];
}

// FP64 [phi | pi] -> FP32_COMP state.
__global__ void k_import_f32(const double *__restrict__ in, float *__restrict__ s, long long n2) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += stride) {
    const double v = in[i];
    const float h = (float)v;
    s[i] = h;
    s[n2 + i] = (float)(v - (double)h);
  }
}

__global__ void k_count_nonfinite(const void *__restrict__ s, long long n, int is_f32,
                                  unsigned long long *__restrict__ bad) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  unsigned long long local = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    double v = is_f32 ? (double)((const float *)s)[i] : ((const double *)s)[i];
    if (!isfinite(v)) ++local;
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(bad, local);
}

// ---- binning --------------------------------------------------------------
struct SpecIn {
  const double *f;  // HC of the field (or phi)
  const double *g;  // HC of dphi (mode spectrum) or nullptr
  int N;
  double k2;   // (2 pi / L)^2
  double m2;   // m^2
  double a2;   // a_t^2
};

// weighted mode value of HC entry (a, b, c): weight 2 for 0 < c < N/2 (the
// entry stands for the conjugate pair c and N - c of the full grid).
__device__ __forceinline__ double mode_value(const SpecIn &A, long long i, int c, long long s2) {
  const double fr = A.f[2 * i], fi = A.f[2 * i + 1];
  double v = fr * fr + fi * fi;
  if (A.g) {
    const double gr = A.g[2 * i], gi = A.g[2 * i + 1];
    v += (gr * gr + gi * gi) / (A.m2 + A.k2 * (double)s2 / A.a2);
  }
  return (c == 0 || 2 * c == A.N) ? v : 2.0 * v;
}

__device__ __forceinline__ void decode_mode(int N, long long i, int &c, long long &s2) {
  const int nh = N / 2 + 1;
  c = (int)(i % nh);
  const long long ab = i / nh;
  const int b = (int)(ab % N);
  const int a = (int)(ab / N);
  const long long as = (a <= N / 2) ? a : N - a;
  const long long bs = (b <= N / 2) ? b : N - b;
  s2 = as * as + bs * bs + (long long)c * c;
}

// ---- orbits of the binning ---------------------------------------------------
// The HC rows (a, b) whose modes share s^2 at every c: a in {as, N - as}, b in
// {bs, N - bs} and, for as != bs, the same with a and b swapped, 0 <= as <= bs <=
// N/2 -- up to 8 rows, and every row lies in exactly one orbit.  A warp takes one
// orbit and its lanes the c values, so the reads are coalesced along c; a lane sums
// the 128-bit fixed-point words of its modes in registers and adds the sum to the
// bin with one pair of 64-bit atomics.  Integer addition is associative, so a bin
// is the same integer as with one atomic pair per mode, at an eighth of the atomics
// (a quarter on the axes).
struct Orbit {
  int as, bs, na, nb, n;  // na, nb: 1 on an axis (0 or N/2), else 2; n rows
  long long ab2;          // as^2 + bs^2
};

__device__ __forceinline__ long long orbit_count(int N) { return (long long)(N / 2 + 1) * (N / 2 + 2) / 2; }

// Orbit o = bs (bs + 1) / 2 + as (0 <= as <= bs <= N/2).
__device__ __forceinline__ bool orbit_of(int N, long long o, Orbit &ob) {
  const int h = N / 2;
  if (o >= orbit_count(N)) return false;
  int bs = (int)((sqrt(8.0 * (double)o + 1.0) - 1.0) * 0.5);
  while ((long long)(bs + 1) * (bs + 2) / 2 <= o) ++bs;
  while ((long long)bs * (bs + 1) / 2 > o) --bs;
  ob.as = (int)(o - (long long)bs * (bs + 1) / 2);
  ob.bs = bs;
  ob.na = (ob.as == 0 || ob.as == h) ? 1 : 2;
  ob.nb = (bs == 0 || bs == h) ? 1 : 2;
  ob.n = ob.na * ob.nb * (ob.as != bs ? 2 : 1);
  ob.ab2 = (long long)ob.as * ob.as + (long long)bs * bs;
  return true;
}

// Row a N + b of the orbit's r-th row (r < n): first a in {as, N - as} with b in {bs,
// N - bs}, then (as != bs) a in {bs, N - bs} with b in {as, N - as}.
__device__ __forceinline__ long long orbit_row(const Orbit &ob, int r, int N) {
  const int m = ob.na * ob.nb;
  int a, b;
  if (r < m) {
    const int i = ob.nb == 2 ? r >> 1 : r, j = ob.nb == 2 ? r & 1 : 0;
    a = i ? N - ob.as : ob.as;
    b = j ? N - ob.bs : ob.bs;
  } else {
    const int q = r - m;
    const int i = ob.na == 2 ? q >> 1 : q, j = ob.na == 2 ? q & 1 : 0;
    a = i ? N - ob.bs : ob.bs;
    b = j ? N - ob.as : ob.as;
  }
  return (long long)a * N + b;
}

// Largest weighted mode value (blockIdx.y: batch entry, HC arrays hc_count apart).
__global__ void __launch_bounds__(256) k_spec_max(SpecIn A, long long hc_count, unsigned long long *maxbits) {
  A.f += (long long)blockIdx.y * hc_count;
  Orbit ob;
  if (!orbit_of(A.N, (long long)blockIdx.x * 8 + (threadIdx.x >> 5), ob)) return;  // whole warps
  const int nh = A.N / 2 + 1;
  long long rows[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) rows[r] = r < ob.n ? orbit_row(ob, r, A.N) * nh : 0;
  double m = 0.0;
  for (int c = threadIdx.x & 31; c < nh; c += 32) {
    const long long s2 = ob.ab2 + (long long)c * c;
#pragma unroll
    for (int r = 0; r < 8; ++r)
      if (r < ob.n) m = fmax(m, mode_value(A, rows[r] + c, c, s2));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  // non-negative doubles order like their bit patterns
  if ((threadIdx.x & 31) == 0) atomicMax(maxbits + blockIdx.y, (unsigned long long)__double_as_longlong(m));
}

// Power-of-two exponent e with (max * entries) * 2^e <= 2^126.
__device__ __forceinline__ int fixed_exponent(unsigned long long maxbits, long long pairs) {
  const double m = __longlong_as_double((long long)maxbits);
  if (!(m > 0.0)) return 0;
  int ex;
  frexp(m * (double)pairs, &ex);  // m*pairs < 2^ex
  return 126 - ex;
}

// One mode value as a 128-bit fixed-point word (lo, hi) at scale 2^e, truncated.
__device__ __forceinline__ void to_fixed(double v, int e, unsigned long long &lo, unsigned long long &hi) {
  const double y = ldexp(v, e);
  hi = __double2ull_rz(ldexp(y, -64));
  lo = __double2ull_rz(y - ldexp((double)hi, 64));
}

// (lo, hi) += (l, h), 128-bit.
__device__ __forceinline__ void add128(unsigned long long &lo, unsigned long long &hi, unsigned long long l,
                                       unsigned long long h) {
  const unsigned long long nl = lo + l;
  hi += h + (nl < lo ? 1ull : 0ull);
  lo = nl;
}

__device__ __forceinline__ void atomic_add128(unsigned long long *bin, unsigned long long lo, unsigned long long hi) {
  unsigned long long carry = 0;
  if (lo) {
    const unsigned long long old = atomicAdd(bin, lo);
    carry = (old + lo < old) ? 1ull : 0ull;
  }
  if (hi + carry) atomicAdd(bin + 1, hi + carry);
}

// Bins of the weighted mode values (blockIdx.y: batch entry; bins 2 nb words apart).
__global__ void __launch_bounds__(256) k_spec_bin(SpecIn A, long long hc_count, long long pairs,
                                                  const unsigned long long *maxbits, unsigned long long *bins,
                                                  long long nb) {
  A.f += (long long)blockIdx.y * hc_count;
  bins += 2 * nb * (long long)blockIdx.y;
  Orbit ob;
  if (!orbit_of(A.N, (long long)blockIdx.x * 8 + (threadIdx.x >> 5), ob)) return;
  const int e = fixed_exponent(maxbits[blockIdx.y], pairs);
  const int nh = A.N / 2 + 1;
  long long rows[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) rows[r] = r < ob.n ? orbit_row(ob, r, A.N) * nh : 0;
  // two c values per iteration: twice the loads in flight (the pass waits on memory;
  // 3.05 -> 2.97 ms per density spectrum at N = 512)
#pragma unroll 2
  for (int c = threadIdx.x & 31; c < nh; c += 32) {
    const long long s2 = ob.ab2 + (long long)c * c;
    unsigned long long lo = 0, hi = 0;
#pragma unroll
    for (int r = 0; r < 8; ++r)
      if (r < ob.n) {
        unsigned long long l, h;
        to_fixed(mode_value(A, rows[r] + c, c, s2), e, l, h);
        add128(lo, hi, l, h);
      }
    atomic_add128(bins + 2 * s2, lo, hi);
  }
}

__device__ __forceinline__ double fixed_to_double(unsigned long long lo, unsigned long long hi, int e) {
  return ldexp(ldexp(__ull2double_rn(hi), 64) + __ull2double_rn(lo), -e);
}

__global__ void k_spec_final(const unsigned long long *bins, const unsigned long long *maxbits, long long pairs,
                             double *out, long long nb) {
  const int e = fixed_exponent(*maxbits, pairs);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < nb; s += stride)
    out[s] = fixed_to_double(bins[2 * s], bins[2 * s + 1], e);
}

__device__ __forceinline__ long long isqrt_ll(long long s) {
  long long r = (long long)sqrt((double)s);
  while (r * r > s) --r;
  while ((r + 1) * (r + 1) <= s) ++r;
  return r;
}

__global__ void k_shells(const unsigned long long *bins, const unsigned long long *maxbits, long long pairs,
                         const long long *s2counts, double *shells, long long *counts, long long nb, long long ns) {
  const int e = fixed_exponent(*maxbits, pairs);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += stride) {
    unsigned long long lo = 0, hi = 0;
    long long cnt = 0;
    const long long s_end = min((i + 1) * (i + 1), nb);
    for (long long s = i * i; s < s_end; ++s) {
      const unsigned long long l = bins[2 * s];
      const unsigned long long nl = lo + l;
      hi += bins[2 * s + 1] + (nl < lo ? 1ull : 0ull);
      lo = nl;
      cnt += s2counts[s];
    }
    if (shells) shells[i] = fixed_to_double(lo, hi, e);
    if (counts) counts[i] = cnt;
  }
}

__global__ void __launch_bounds__(256) k_s2_counts(int N, unsigned long long *counts) {
  Orbit ob;
  if (!orbit_of(N, (long long)blockIdx.x * 8 + (threadIdx.x >> 5), ob)) return;
  for (int c = threadIdx.x & 31; c <= N / 2; c += 32)
    atomicAdd(&counts[ob.ab2 + (long long)c * c], (unsigned long long)ob.n * ((c == 0 || 2 * c == N) ? 1ull : 2ull));
}

// ---- batched binning (blockIdx.y = batch entry; used by ensembles) ----------
__global__ void k_specb_final(const unsigned long long *bins, const unsigned long long *maxbits, long long pairs,
                              double *out, long long nb) {
  const int e = fixed_exponent(maxbits[blockIdx.y], pairs);
  const unsigned long long *bb = bins + 2 * nb * blockIdx.y;
  double *o = out + nb * blockIdx.y;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < nb; s += stride)
    o[s] = fixed_to_double(bb[2 * s], bb[2 * s + 1], e);
}

// Blocks of 8 warps, one orbit per warp.
static unsigned orbit_blocks(int N) {
  const long long norb = (long long)(N / 2 + 1) * (N / 2 + 2) / 2;
  return (unsigned)((norb + 7) / 8);
}

int bin_batched(const double *hc, int N, int batch, unsigned long long *maxbits, unsigned long long *bins, double *out,
                long long nb, cudaStream_t st, cf_ctx *) {
  const long long hc_count = 2LL * N * N * (N / 2 + 1), pairs = hc_count / 2;
  CF_TRY_CUDA(cudaMemsetAsync(maxbits, 0, sizeof(unsigned long long) * batch, st));
  CF_TRY_CUDA(cudaMemsetAsync(bins, 0, sizeof(unsigned long long) * 2 * nb * batch, st));
  SpecIn A{};
  A.f = hc;
  A.N = N;
  const unsigned gx = orbit_blocks(N);
  k_spec_max<<<dim3(gx, batch), 256, 0, st>>>(A, hc_count, maxbits);
  CF_TRY_CUDA(cudaGetLastError());
  k_spec_bin<<<dim3(gx, batch), 256, 0, st>>>(A, hc_count, pairs, maxbits, bins, nb);
  CF_TRY_CUDA(cudaGetLastError());
  const unsigned gf = (unsigned)std::min<long long>((nb + 255) / 256, 148LL * 8);
  k_specb_final<<<dim3(gf, batch), 256, 0, st>>>(bins, maxbits, pairs, out, nb);
  CF_TRY_CUDA(cudaGetLastError());
  return CF_OK;
}

static unsigned grid_for(long long n, int per = 256) {
  long long b = (n + per - 1) / per;
  if (b > 148LL * 32) b = 148LL * 32;
  if (b < 1) b = 1;
  return (unsigned)b;
}

int ensure_spectrum_scratch(cf_ctx *ctx, int nfields) {
  const size_t hc = (size_t)ctx->hc_count;
  if (!ctx->spec_hc) {
    if (cudaMalloc(&ctx->spec_hc, 2 * hc * sizeof(double)) != cudaSuccess) {
      set_error("cudaMalloc spectrum HC scratch failed");
      return CF_ERR_NOMEM;
    }
    if (cudaMalloc(&ctx->spec_field, 2 * (size_t)ctx->N3 * sizeof(double)) != cudaSuccess) {
      set_error("cudaMalloc spectrum field scratch failed");
      return CF_ERR_NOMEM;
    }
    if (cudaMalloc(&ctx->bins, 2 * (size_t)ctx->s2_bins * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&ctx->maxbits, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&ctx->s2_counts, (size_t)ctx->s2_bins * sizeof(int64_t)) != cudaSuccess) {
      set_error("cudaMalloc spectrum bins failed");
      return CF_ERR_NOMEM;
    }
    CF_TRY_CUDA(cudaMemset(ctx->s2_counts, 0, (size_t)ctx->s2_bins * sizeof(int64_t)));
    k_s2_counts<<<orbit_blocks((int)ctx->N), 256>>>((int)ctx->N, (unsigned long long *)ctx->s2_counts);
    CF_LAUNCHED(ctx);
    CF_TRY_CUDA(cudaMemset(ctx->bins, 0, 2 * (size_t)ctx->s2_bins * sizeof(unsigned long long)));
    CF_TRY_CUDA(cudaMemset(ctx->maxbits, 0, sizeof(unsigned long long)));
    CF_TRY_CUDA(cudaDeviceSynchronize());
  }
  const int N = (int)ctx->N;
  if (nfields >= 1 && !ctx->have_d2z1) {
    CF_TRY_CUFFT(cufftPlan3d(&ctx->plan_d2z1, N, N, N, CUFFT_D2Z));
    ctx->have_d2z1 = true;
  }
  if (nfields >= 2 && !ctx->have_d2z2) {
    long long n[3] = {N, N, N};
    long long inembed[3] = {N, N, N};
    long long onembed[3] = {N, N, N / 2 + 1};
    size_t work = 0;
    CF_TRY_CUFFT(cufftCreate(&ctx->plan_d2z2));
    CF_TRY_CUFFT(cufftMakePlanMany64(ctx->plan_d2z2, 3, n, inembed, 1, ctx->N3, onembed, 1, ctx->hc_count / 2,
                                     CUFFT_D2Z, 2, &work));
    ctx->have_d2z2 = true;
  }
  return CF_OK;
}

// Bins the HC data already in ctx->spec_hc (1 field, or phi/dphi for the mode spectrum).
// bound_mult = 0: a max pass finds the largest weighted mode value and the scale bounds
// it times the HC entry count.  bound_mult > 0: ctx->maxbits already holds a value m
// with m * bound_mult >= the sum of all weighted mode values.
static int bin_spectrum(cf_ctx *ctx, bool mode, double a_t, double *d_out, cudaStream_t st,
                        long long bound_mult = 0) {
  const long long pairs = bound_mult > 0 ? bound_mult : ctx->hc_count / 2;
  ctx->spec_mult = pairs;
  SpecIn A{};
  A.f = ctx->spec_hc;
  A.g = mode ? ctx->spec_hc + ctx->hc_count : nullptr;
  A.N = (int)ctx->N;
  const double kir = 2 * 3.14159265358979323846 / ctx->p.L;
  A.k2 = kir * kir;
  A.m2 = ctx->p.m * ctx->p.m;
  A.a2 = a_t * a_t;
  ProfScope ps(ctx, CF_PROF_SPECTRUM, st);
  CF_TRY_CUDA(cudaMemsetAsync(ctx->bins, 0, 2 * (size_t)ctx->s2_bins * sizeof(unsigned long long), st));
  if (bound_mult <= 0) {
    CF_TRY_CUDA(cudaMemsetAsync(ctx->maxbits, 0, sizeof(unsigned long long), st));
    k_spec_max<<<orbit_blocks(A.N), 256, 0, st>>>(A, 0, ctx->maxbits);
    CF_LAUNCHED(ctx);
  }
  k_spec_bin<<<orbit_blocks(A.N), 256, 0, st>>>(A, 0, pairs, ctx->maxbits, ctx->bins, ctx->s2_bins);
  CF_LAUNCHED(ctx);
  if (d_out) {
    k_spec_final<<<grid_for(ctx->s2_bins), 256, 0, st>>>(ctx->bins, ctx->maxbits, pairs, d_out, ctx->s2_bins);
    CF_LAUNCHED(ctx);
  }
  return CF_OK;
}

int power_spectrum_s2(cf_ctx *ctx, const double *d_f, double *d_out, cudaStream_t st) {
  CF_TRY(ensure_spectrum_scratch(ctx, 1));
  CF_TRY_CUFFT(cufftSetStream(ctx->plan_d2z1, st));
  {
    ProfScope ps(ctx, CF_PROF_SPECTRUM, st);
    CF_TRY_CUFFT(cufftExecD2Z(ctx->plan_d2z1, (cufftDoubleReal *)d_f, (cufftDoubleComplex *)ctx->spec_hc));
  }
  return bin_spectrum(ctx, false, 1.0, d_out, st);
}

static const double *state_as_f64(cf_ctx *ctx, const void *d_state, cudaStream_t st, int *err) {
  *err = CF_OK;
  if (ctx->p.precision == CF_FP64) return (const double *)d_state;
  const long long n2 = 2 * ctx->N3;
  k_export_f32<<<grid_for(n2), 256, 0, st>>>((const float *)d_state, ctx->spec_field, n2);
  if (cudaGetLastError() != cudaSuccess) {
    set_error("state export launch failed");
    *err = CF_ERR_CUDA;
  }
  ctx->launches++;
  return ctx->spec_field;
}

int mode_power_spectrum_s2(cf_ctx *ctx, const void *d_state, double a_t, double *d_out, cudaStream_t st) {
  CF_TRY(ensure_spectrum_scratch(ctx, 2));
  int err;
  const double *x = state_as_f64(ctx, d_state, st, &err);
  CF_TRY(err);
  CF_TRY_CUFFT(cufftSetStream(ctx->plan_d2z2, st));
  {
    ProfScope ps(ctx, CF_PROF_SPECTRUM, st);
    CF_TRY_CUFFT(cufftExecD2Z(ctx->plan_d2z2, (cufftDoubleReal *)x, (cufftDoubleComplex *)ctx->spec_hc));
  }
  return bin_spectrum(ctx, true, a_t, d_out, st);
}

template <typename S, int ED>
static void launch_energy(cf_ctx *ctx, const void *d_state, const void *psi, double *d_rho, double m2, double inv,
                          double q, unsigned long long *rowmax, cudaStream_t st) {
  const long long N3 = ctx->N3;
  const S *x = (const S *)d_state;
  k_energy<S, ED><<<(unsigned)(ctx->N * ctx->N), 128, 0, st>>>(x, sizeof(S) == 4 ? x + 2 * N3 : nullptr,
                                                               (const S *)psi, d_rho, (int)ctx->N, m2, inv, q, rowmax);
}

template <int ED>
static void launch_energy_p(cf_ctx *ctx, const void *d_state, const void *psi, double *d_rho, double m2, double inv,
                            double q, unsigned long long *rowmax, cudaStream_t st) {
  if (ctx->p.precision == CF_FP32_COMP)
    launch_energy<float, ED>(ctx, d_state, psi, d_rho, m2, inv, q, rowmax, st);
  else
    launch_energy<double, ED>(ctx, d_state, psi, d_rho, m2, inv, q, rowmax, st);
}

// `rowmax` (optional, zeroed by the caller): receives the largest row sum of rho^2.
static int energy_density_b(cf_ctx *ctx, const void *d_state, double t, double *d_rho, unsigned long long *rowmax,
                            cudaStream_t st) {
  double inv, H;
  stage_coeffs(ctx->p, t, &inv, &H);
  const double m2 = ctx->p.m * ctx->p.m;
  const int eq = ctx->p.equation;
  const void *ps = nullptr, *dps = nullptr;
  // the approximate comoving equation reports the full comoving energy density
  // (src/equations_cuda.cu:812-815)
  if (eq == CF_EQ_COMOVING_FRW || eq == CF_EQ_APPROX_COMOVING_FRW) CF_TRY(psi_at(ctx, t, st, &ps, &dps));
  if (eq == CF_EQ_FIXED_CURVATURE_FRW) ps = ctx->fixed_e2m1;
  ProfScope prof(ctx, CF_PROF_SPECTRUM, st);
  if (ps)
    launch_energy_p<ED_CURV>(ctx, d_state, ps, d_rho, m2, inv, 0.0, rowmax, st);
  else if (eq == CF_EQ_LAMBDA_FRW)
    launch_energy_p<ED_LAMBDA>(ctx, d_state, nullptr, d_rho, m2, inv, ctx->p.lambda, rowmax, st);
  else if (eq == CF_EQ_SQRT_FRW)
    launch_energy_p<ED_SQRT>(ctx, d_state, nullptr, d_rho, m2, inv, 1.0 / (ctx->p.f_a * ctx->p.f_a), rowmax, st);
  else
    launch_energy_p<ED_QUAD>(ctx, d_state, nullptr, d_rho, m2, inv, 0.0, rowmax, st);
  CF_LAUNCHED(ctx);
  return CF_OK;
}

int energy_density(cf_ctx *ctx, const void *d_state, double t, double *d_rho, cudaStream_t st) {
  return energy_density_b(ctx, d_state, t, d_rho, nullptr, st);
}

int dot_energy_density(cf_ctx *ctx, const void *d_state, double t, double *d_out, cudaStream_t st) {
  double inv, H;
  stage_coeffs(ctx->p, t, &inv, &H);
  const double m2 = ctx->p.m * ctx->p.m;
  const long long N3 = ctx->N3;
  ProfScope prof(ctx, CF_PROF_SPECTRUM, st);
  if (ctx->p.precision == CF_FP32_COMP) {
    const float *x = (const float *)d_state;
    k_dot_energy<float><<<grid_for(N3), 256, 0, st>>>(x, x + 2 * N3, d_out, (int)ctx->N, m2, inv, H);
  } else {
    k_dot_energy<double><<<grid_for(N3), 256, 0, st>>>((const double *)d_state, nullptr, d_out, (int)ctx->N, m2,
                                                       inv, H);
  }
  CF_LAUNCHED(ctx);
  return CF_OK;
}

// Mean over a of an N^3 field, per (b, c): out[i] = sum_a f[i + a N^2] / N (coalesced in i).
__global__ void k_axis_mean(const double *__restrict__ f, double *__restrict__ out, long long NN, int N) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < NN; i += stride) {
    double acc = 0.0;
    for (int a = 0; a < N; ++a) acc += f[i + (long long)a * NN];
    out[i] = acc / (double)N;
  }
}

int density_slices(cf_ctx *ctx, const void *d_state, double t, double *d_slice, double *d_avg, cudaStream_t st) {
  CF_TRY(ensure_spectrum_scratch(ctx, 1));
  CF_TRY(energy_density(ctx, d_state, t, ctx->spec_field, st));
  const long long NN = ctx->N * ctx->N;
  if (d_slice)
    CF_TRY_CUDA(cudaMemcpyAsync(d_slice, ctx->spec_field, NN * sizeof(double), cudaMemcpyDeviceToDevice, st));
  if (d_avg) {
    ProfScope ps(ctx, CF_PROF_SPECTRUM, st);
    k_axis_mean<<<grid_for(NN), 256, 0, st>>>(ctx->spec_field, d_avg, NN, (int)ctx->N);
    CF_LAUNCHED(ctx);
  }
  return CF_OK;
}

// The fixed-point scale comes from the energy pass: by Parseval the weighted HC
// values of rho sum to N^3 sum_x rho^2 <= N^5 max_row sum_c rho^2, so no bin can
// exceed that bound, and the binning needs no pass of its own to find a maximum.
int density_spectrum_s2(cf_ctx *ctx, const void *d_state, double t, double *d_out, cudaStream_t st) {
  CF_TRY(ensure_spectrum_scratch(ctx, 1));
  CF_TRY_CUDA(cudaMemsetAsync(ctx->maxbits, 0, sizeof(unsigned long long), st));
  CF_TRY(energy_density_b(ctx, d_state, t, ctx->spec_field, ctx->maxbits, st));
  CF_TRY_CUFFT(cufftSetStream(ctx->plan_d2z1, st));
  {
    ProfScope ps(ctx, CF_PROF_SPECTRUM, st);
    CF_TRY_CUFFT(cufftExecD2Z(ctx->plan_d2z1, (cufftDoubleReal *)ctx->spec_field, (cufftDoubleComplex *)ctx->spec_hc));
  }
  const long long N = ctx->N;
  return bin_spectrum(ctx, false, 1.0, d_out, st, N * N * N * N * N);
}

int s2_to_shells(cf_ctx *ctx, double *d_shells, int64_t *d_counts, cudaStream_t st) {
  CF_TRY(ensure_spectrum_scratch(ctx, 0));
  k_shells<<<grid_for(ctx->shells, 128), 128, 0, st>>>(ctx->bins, ctx->maxbits, ctx->spec_mult,
                                                       (const long long *)ctx->s2_counts, d_shells,
                                                       (long long *)d_counts, ctx->s2_bins, ctx->shells);
  CF_LAUNCHED(ctx);
  return CF_OK;
}

int s2_counts(cf_ctx *ctx, int64_t *d_counts, cudaStream_t st) {
  CF_TRY(ensure_spectrum_scratch(ctx, 0));
  CF_TRY_CUDA(cudaMemcpyAsync(d_counts, ctx->s2_counts, (size_t)ctx->s2_bins * sizeof(int64_t),
                              cudaMemcpyDeviceToDevice, st));
  return CF_OK;
}

int state_export(cf_ctx *ctx, double *d_xy, const void *d_state, cudaStream_t st) {
  const long long n2 = 2 * ctx->N3;
  if (ctx->p.precision == CF_FP64) {
    CF_TRY_CUDA(cudaMemcpyAsync(d_xy, d_state, n2 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    return CF_OK;
  }
  k_export_f32<<<grid_for(n2), 256, 0, st>>>((const float *)d_state, d_xy, n2);
  CF_LAUNCHED(ctx);
  return CF_OK;
}

int state_import(cf_ctx *ctx, void *d_state, const double *d_xy, cudaStream_t st) {
  const long long n2 = 2 * ctx->N3;
  if (ctx->p.precision == CF_FP64) {
    CF_TRY_CUDA(cudaMemcpyAsync(d_state, d_xy, n2 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    return CF_OK;
  }
  k_import_f32<<<grid_for(n2), 256, 0, st>>>(d_xy, (float *)d_state, n2);
  CF_LAUNCHED(ctx);
  return CF_OK;
}

// ---- host <-> device state transfer of the FP32_COMP layout ------------------
// The FP64 [phi | pi] host array goes through two device chunks of the context
// (allocated once, kStageChunk doubles each) in turn: a chunk's copy and its
// conversion are ordered on the caller's stream, and chunk i + 2 reuses chunk i's
// buffer after its conversion.  An event recorded after the last chunk orders the
// next transfer, on whatever stream it runs, behind this one.
__global__ void k_import_f32_part(const double *__restrict__ in, float *__restrict__ s, long long n2, long long off,
                                  long long len) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += stride) {
    const double v = in[i];
    const float h = (float)v;
    s[off + i] = h;
    s[n2 + off + i] = (float)(v - (double)h);
  }
}

__global__ void k_export_f32_part(const float *__restrict__ s, double *__restrict__ out, long long n2, long long off,
                                  long long len) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += stride)
    out[i] = (double)s[off + i] + (double)s[n2 + off + i];
}

static constexpr long long kStageChunk = 16LL << 20;  // doubles per chunk (128 MB)

static int stage_begin(cf_ctx *ctx, cudaStream_t st) {
  if (!ctx->stage) {
    if (cudaMalloc(&ctx->stage, 2 * kStageChunk * sizeof(double)) != cudaSuccess) {
      ctx->stage = nullptr;
      set_error("cudaMalloc state staging chunks failed");
      return CF_ERR_NOMEM;
    }
    CF_TRY_CUDA(cudaEventCreateWithFlags(&ctx->stage_ev, cudaEventDisableTiming));
  }
  if (ctx->stage_used) CF_TRY_CUDA(cudaStreamWaitEvent(st, ctx->stage_ev, 0));
  return CF_OK;
}

static int stage_end(cf_ctx *ctx, cudaStream_t st) {
  CF_TRY_CUDA(cudaEventRecord(ctx->stage_ev, st));
  ctx->stage_used = true;
  return CF_OK;
}

int state_upload_host(cf_ctx *ctx, void *d_state, const double *h_xy, cudaStream_t st) {
  CF_TRY(stage_begin(ctx, st));
  const long long n2 = 2 * ctx->N3;
  for (long long off = 0, i = 0; off < n2; off += kStageChunk, ++i) {
    const long long len = std::min(kStageChunk, n2 - off);
    double *buf = ctx->stage + (i & 1) * kStageChunk;
    CF_TRY_CUDA(cudaMemcpyAsync(buf, h_xy + off, len * sizeof(double), cudaMemcpyHostToDevice, st));
    k_import_f32_part<<<grid_for(len), 256, 0, st>>>(buf, (float *)d_state, n2, off, len);
    CF_LAUNCHED(ctx);
  }
  return stage_end(ctx, st);
}

int state_download_host(cf_ctx *ctx, double *h_xy, const void *d_state, cudaStream_t st) {
  CF_TRY(stage_begin(ctx, st));
  const long long n2 = 2 * ctx->N3;
  for (long long off = 0, i = 0; off < n2; off += kStageChunk, ++i) {
    const long long len = std::min(kStageChunk, n2 - off);
    double *buf = ctx->stage + (i & 1) * kStageChunk;
    k_export_f32_part<<<grid_for(len), 256, 0, st>>>((const float *)d_state, buf, n2, off, len);
    CF_LAUNCHED(ctx);
    CF_TRY_CUDA(cudaMemcpyAsync(h_xy + off, buf, len * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  return stage_end(ctx, st);
}

int check_finite(cf_ctx *ctx, const void *d_state, int64_t *h_bad, cudaStream_t st) {
  unsigned long long *d_bad = nullptr;
  if (cudaMallocAsync((void **)&d_bad, sizeof(unsigned long long), st) != cudaSuccess) {
    set_error("cudaMallocAsync failed");
    return CF_ERR_NOMEM;
  }
  CF_TRY_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(unsigned long long), st));
  const bool f32 = ctx->p.precision == CF_FP32_COMP;
  const long long n = (f32 ? 4 : 2) * ctx->N3;
  k_count_nonfinite<<<grid_for(n), 256, 0, st>>>(d_state, n, f32 ? 1 : 0, d_bad);
  CF_LAUNCHED(ctx);
  unsigned long long h = 0;
  CF_TRY_CUDA(cudaMemcpyAsync(&h, d_bad, sizeof(h), cudaMemcpyDeviceToHost, st));
  CF_TRY_CUDA(cudaFreeAsync(d_bad, st));
  CF_TRY_CUDA(cudaStreamSynchronize(st));
  if (h_bad) *h_bad = (int64_t)h;
  if (h) {
    set_error("state holds %llu non-finite values", h);
    return CF_ERR_NONFINITE;
  }
  return CF_OK;
}

}  // namespace cfb
