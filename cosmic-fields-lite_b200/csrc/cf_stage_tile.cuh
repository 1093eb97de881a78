// cf_stage_tile.cuh -- one fused RK4 stage over one (b, c) tile of one lattice,
// marching along a (shared by the single-lattice stage kernels and the
// ensemble kernels).
//
// Stage semantics (stepper/runge_kutta4_classic.hpp:88-138, with the odeint
// scale_sum combinations of src/odeint_thrust/thrust_operations.cu:238-313 fused in):
//   STAGE 0: dxdt = f(y)                       (plain right-hand side, cf_rhs)
//   STAGE 1: k = f(x)  acc  = k     y' = x + cy k
//   STAGE 2: k = f(y)  acc += 2k    y' = x + cy k
//   STAGE 3: k = f(y)  acc += 2k    y' = x + cy k
//   STAGE 4: k = f(y)  x   += dt/6 (acc + k)   (FP32: hi/lo compensated)
// with f(phi, pi) = (pi, (-3H + 4 dPsi) pi - e^{2Psi} m^2 phi + e^{4Psi} inv lap phi)
// (src/equations_cuda.cu:15-36, :263-287; Psi = dPsi = 0 for EQ_FRW) and the
// other equation shapes of EqShape below.
//
// Tile: TXv x TYv threads; thread (tx, ty) owns V consecutive sites along c
// (16-byte vectors) in row b0 + ty.  phi of planes a-H..a+H of the thread's own
// sites live in a register queue; the current plane plus an H-wide periodic
// halo in b and c is staged in shared memory (sm: (TYv + 2H) x (TXv V + 2H)).
#pragma once

#include <cuda_runtime.h>

#include "cf_f32x2.cuh"

namespace cfb {

// A thread's consecutive sites along c, moved as one vector: V = 4 floats or 2
// doubles (16 bytes) by default; some kernels take V = 2 floats (8 bytes), which
// halves the registers a thread's sites occupy.
template <typename S, int V>
struct VecOf;
template <>
struct VecOf<double, 2> {
  using T = double2;
};
template <>
struct VecOf<float, 4> {
  using T = float4;
};
template <>
struct VecOf<float, 2> {
  using T = float2;
};
template <typename S>
struct VecT {
  static constexpr int n = 16 / sizeof(S);
  using T = typename VecOf<S, n>::T;
};

template <typename S, int V = VecT<S>::n>
struct Pack {
  S v[V];
};

template <typename S, int V>
__device__ __forceinline__ Pack<S, V> unpack(const typename VecOf<S, V>::T &t) {
  Pack<S, V> r;
  if constexpr (V == 2) {
    r.v[0] = t.x;
    r.v[1] = t.y;
  } else {
    r.v[0] = t.x;
    r.v[1] = t.y;
    r.v[2] = t.z;
    r.v[3] = t.w;
  }
  return r;
}

// read-only path (buffers the kernel does not write)
template <typename S, int V = VecT<S>::n>
__device__ __forceinline__ Pack<S, V> ldv(const S *p) {
  return unpack<S, V>(__ldg(reinterpret_cast<const typename VecOf<S, V>::T *>(p)));
}

// plain load for buffers the same kernel also writes (acc, x)
template <typename S, int V = VecT<S>::n>
__device__ __forceinline__ Pack<S, V> ldv_rw(const S *p) {
  return unpack<S, V>(*reinterpret_cast<const typename VecOf<S, V>::T *>(p));
}

template <typename S, int V>
__device__ __forceinline__ void stv(S *p, const Pack<S, V> &r) {
  typename VecOf<S, V>::T t;
  if constexpr (V == 2) {
    t.x = r.v[0];
    t.y = r.v[1];
  } else {
    t.x = r.v[0];
    t.y = r.v[1];
    t.z = r.v[2];
    t.w = r.v[3];
  }
  *reinterpret_cast<typename VecOf<S, V>::T *>(p) = t;
}

template <typename S>
struct StageArgs {
  const S *yin;  // stage input [phi | pi]; for stages 0 and 1 the state x (hi part)
  S *yout;       // stage output [phi | pi] (stages 1-3); dxdt for stage 0
  S *acc;        // k accumulator [phi | pi]
  S *x;          // base state [phi | pi] (hi part in FP32_COMP)
  S *xlo;        // FP32_COMP compensation [phi | pi] (stage 4 only)
  const S *psi;  // EQ_COMOV, EQ_FIXED: e^{2 Psi(t_stage)} - 1, N^3; EQ_APPROX: the coarse table
  const S *dpsi; // EQ_COMOV: dPsi/dt(t_stage), N^3
  const int *cmap;  // EQ_APPROX: coarse index of each lattice index (N entries)
  int M;            // EQ_APPROX: coarse grid size
  int N;
  int a_chunk;
  long long N3;
  double q1, q2;  // EQ_LAMBDA: lambda; EQ_SQRT: f_a^2, 1/f_a^2
  double m2;    // m^2
  double inv;   // h^-2 a^-2
  double hub3;  // 3 H
  double cy;    // y' = x + cy * k
  double dt6;   // dt / 6
};

// Periodic index for i in [-N, 2N): two compares instead of an integer division by
// N.  Every wrapped index of the tile kernels lies within H <= 2 sites of the
// lattice (halo rows and columns of an active tile, planes a - H .. a + H).
__device__ __forceinline__ int wrap_n(int i, int N) { return i < 0 ? i + N : (i >= N ? i - N : i); }

// Arithmetic type of the stage evaluations: FP64 for FP64 storage; FP32 for
// FP32_COMP, whose stage inputs and accumulator are FP32 words anyway.  In FP32
// every rounding must be unbiased, or it acts like a changed time step or mass
// and the error grows with time: coefficients (dt/2, dt/6, h^-2 a^-2, 3H, m^2)
// enter as hi + lo pairs, e^{2 Psi} as 1 + expm1f (never rounded as 1 + eps),
// and the state update x += dt/6 (acc + k4) is formed without rounding error on
// the hi + lo pair (comp_update).
template <typename S>
struct Arith {
  using T = S;
};

// A coefficient in the arithmetic type: FP64 as is, FP32 as hi + lo.
template <typename T>
struct Coef;
template <>
struct Coef<double> {
  double hi;
  __host__ __device__ Coef(double c) : hi(c) {}
  __device__ __forceinline__ double mul(double v) const { return hi * v; }
  __device__ __forceinline__ double fma(double v, double add) const { return add + hi * v; }
};
template <>
struct Coef<float> {
  float hi, lo;
  __host__ __device__ Coef(double c) : hi((float)c), lo((float)(c - (double)(float)c)) {}
  // c v with the product's error random (hi v + lo v); the same operations as c_mul /
  // c_fma of cf_f32x2.cuh
  __device__ __forceinline__ float mul(float v) const { return __fmaf_rn(hi, v, __fmul_rn(lo, v)); }
  // add + c v
  __device__ __forceinline__ float fma(float v, float add) const { return __fadd_rn(add, mul(v)); }
  __device__ __forceinline__ CoefL<float> lane() const { return CoefL<float>{hi, lo}; }
};

// FP32_COMP state update hi + lo + c s as a normalised hi + lo pair (comp_update_f32 of
// cf_f32x2.cuh: error-free product and TwoSum, the small parts added, Fast2Sum).
__device__ __forceinline__ void comp_update(float hi, float lo, float s, const Coef<float> &c, float &oh,
                                            float &ol) {
  comp_update_f32<float>(hi, lo, s, c.lane(), oh, ol);
}

// x += dt/6 s (RK4's last combination): FP64 directly; FP32_COMP on the hi + lo pair.
__device__ __forceinline__ void state_update(double x, double, double s, const Coef<double> &c6, double &ox,
                                             double &) {
  ox = x + c6.hi * s;
}
__device__ __forceinline__ void state_update(float hi, float lo, float s, const Coef<float> &c6, float &oh,
                                             float &ol) {
  comp_update(hi, lo, s, c6, oh, ol);
}

// e^{2 Psi} and e^{4 Psi} from the Psi slot's e^{2 Psi} - 1 (FP64).
__device__ __forceinline__ void psi_factors(double e2m1, double &e2, double &e4) {
  e2 = 1.0 + e2m1;
  e4 = e2 * e2;
}

// Laplacian sum (times h^2) at (row, col) of a staged plane whose a-neighbours
// are q[0..2H] (q[H] the plane itself): 7-point for H = 1, 13-point 4th order for
// H = 2 (src/fdm3d_cuda.cu:20-83; in FP32 the 13-point sum comes times 12, see
// lap13_f32).  The single-stage and the paired-stage tiles both form it here, so
// their sums round identically.
template <typename S, int H, int SP, int V, typename T = typename Arith<S>::T>
__device__ __forceinline__ T lap_at(const Pack<S, V> (&q)[2 * H + 1], const S *sm, int row, int col, int v) {
  const T f0 = (T)q[H].v[v];
  if constexpr (sizeof(T) == 4) {  // FP32: the fixed operation order of cf_f32x2.cuh
    if constexpr (H == 1) {
      return lap7_f32<float>(f0, q[2].v[v], q[0].v[v], sm[(row + 1) * SP + col], sm[(row - 1) * SP + col],
                             sm[row * SP + col + 1], sm[row * SP + col - 1]);
    } else {
      float s1 = p_add(q[3].v[v], q[1].v[v]);
      s1 = p_add(s1, sm[(row + 1) * SP + col]);
      s1 = p_add(s1, sm[(row - 1) * SP + col]);
      s1 = p_add(s1, sm[row * SP + col + 1]);
      s1 = p_add(s1, sm[row * SP + col - 1]);
      float s2 = p_add(q[4].v[v], q[0].v[v]);
      s2 = p_add(s2, sm[(row + 2) * SP + col]);
      s2 = p_add(s2, sm[(row - 2) * SP + col]);
      s2 = p_add(s2, sm[row * SP + col + 2]);
      s2 = p_add(s2, sm[row * SP + col - 2]);
      return lap13_f32<float>(f0, s1, s2);
    }
  } else if constexpr (H == 1) {
    const T s = (T)-6 * f0 + (T)q[2].v[v] + (T)q[0].v[v] + (T)sm[(row + 1) * SP + col] + (T)sm[(row - 1) * SP + col];
    return s + ((T)sm[row * SP + col + 1] + (T)sm[row * SP + col - 1]);
  } else {
    const T s1 = (T)q[3].v[v] + (T)q[1].v[v] + (T)sm[(row + 1) * SP + col] + (T)sm[(row - 1) * SP + col] +
                 (T)sm[row * SP + col + 1] + (T)sm[row * SP + col - 1];
    const T s2 = (T)q[4].v[v] + (T)q[0].v[v] + (T)sm[(row + 2) * SP + col] + (T)sm[(row - 2) * SP + col] +
                 (T)sm[row * SP + col + 2] + (T)sm[row * SP + col - 2];
    return ((T)16 * s1 - s2 - (T)90 * f0) / (T)12;
  }
}

// Equation shapes of the tile kernels: the pointwise terms of the pi component
// of the right-hand side (the phi component is always pi).
enum EqShape : int {
  EQ_FRW = 0,     // -3H pi - m^2 phi + inv lap (flat KG: H = 0, inv = h^-2)
  EQ_COMOV = 1,   // (-3H + 4 dPsi) pi - e^{2Psi} m^2 phi + e^{4Psi} inv lap, Psi(t) planes
  EQ_LAMBDA = 2,  // -3H pi - m^2 phi - lambda phi^3 + inv lap
  EQ_SQRT = 3,    // -3H pi - m^2 phi / sqrt(1 + phi^2 / f_a^2) + inv lap
  EQ_FIXED = 4,   // -3H pi - e^{2Psi} m^2 phi + e^{4Psi} inv lap, one fixed Psi plane
  EQ_APPROX = 5,  // as EQ_COMOV with Psi, dPsi from a coarse table, quadratic exponentials
};

template <int EQ>
struct EqOf {
  static constexpr bool psi_plane = EQ == EQ_COMOV || EQ == EQ_FIXED;  // reads e^{2Psi} - 1 per site
  static constexpr bool dpsi_plane = EQ == EQ_COMOV;                   // reads dPsi/dt per site
  static constexpr bool coarse = EQ == EQ_APPROX;                      // gathers the coarse table
  static constexpr bool coupled = psi_plane || coarse;
};

// Stage coefficients in the arithmetic type (q1, q2: the equation's own
// constants, StageArgs::q1 / q2).
template <typename T>
struct StageCoef {
  Coef<T> m2, inv, hub3, q1, q2;
};

// The per-site curvature values of one stage at a thread's V sites: ps = e^{2Psi}
// - 1 (EQ_APPROX: 2 Psi + 2 Psi^2), dps = dPsi/dt, ps4 = 4 Psi + 8 Psi^2 (EQ_APPROX).
template <typename S, int V>
struct Coupling {
  Pack<S, V> ps, dps, ps4;
};

// The coarse columns of a thread's V sites c..c+V-1 and the coarse row of its b
// (EQ_APPROX; constant along a, so formed once per tile).
template <int V>
struct CoarseCols {
  int col[V];
  int row_b;  // coarse index of b
};

template <int EQ, int V>
__device__ __forceinline__ CoarseCols<V> coarse_cols(const int *cmap, bool act, int b, int c) {
  CoarseCols<V> cc{};
  if constexpr (EqOf<EQ>::coarse) {
    if (act) {  // b < N and c + V <= N only for active threads
      cc.row_b = __ldg(cmap + b);
#pragma unroll
      for (int v = 0; v < V; ++v) cc.col[v] = __ldg(cmap + c + v);
    }
  }
  return cc;
}

// Loads the curvature values of sites (a, b, c..c+V-1): `site` their offset in an
// N^3 plane set; ca the coarse index of a (EQ_APPROX).  The coarse table holds 4
// words per coarse site: (2Psi + 2Psi^2, 4Psi + 8Psi^2, dPsi/dt, 0).
template <int EQ, typename S, int V>
__device__ __forceinline__ void load_coupling(Coupling<S, V> &cp, const S *psi, const S *dpsi, long long site,
                                              int M, int ca, const CoarseCols<V> &cc) {
  if constexpr (EqOf<EQ>::psi_plane) cp.ps = ldv<S, V>(psi + site);
  if constexpr (EqOf<EQ>::dpsi_plane) cp.dps = ldv<S, V>(dpsi + site);
  if constexpr (EqOf<EQ>::coarse) {
    const int row = (ca * M + cc.row_b) * M;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const int idx = row + cc.col[v];
      if constexpr (sizeof(S) == 4) {
        const float4 t = __ldg(reinterpret_cast<const float4 *>(psi) + idx);
        cp.ps.v[v] = t.x;
        cp.ps4.v[v] = t.y;
        cp.dps.v[v] = t.z;
      } else {
        const double2 t0 = __ldg(reinterpret_cast<const double2 *>(psi) + 2 * idx);
        const double2 t1 = __ldg(reinterpret_cast<const double2 *>(psi) + 2 * idx + 1);
        cp.ps.v[v] = t0.x;
        cp.ps4.v[v] = t0.y;
        cp.dps.v[v] = t1.x;
      }
    }
  }
}

// pi component of the right-hand side at site v of a thread's sites
// (src/equations_cuda.cu:15-36 FRW, :38-76 lambda, :84-104 sqrt potential,
// :112-136 fixed Psi, :263-287 comoving, :299-329 approximate comoving).
template <int EQ, typename S, int V, typename T = typename Arith<S>::T>
__device__ __forceinline__ T kpi_of(T p0, T f0, T lap, const Coupling<S, V> &cp, int v, const StageCoef<T> &k) {
  if constexpr (sizeof(T) == 8) {
    if constexpr (EQ == EQ_COMOV || EQ == EQ_FIXED) {
      T e2, e4;
      psi_factors(cp.ps.v[v], e2, e4);
      if constexpr (EQ == EQ_COMOV)
        return (-k.hub3.hi + (T)4 * (T)cp.dps.v[v]) * p0 - e2 * k.m2.hi * f0 + e4 * k.inv.hi * lap;
      else
        return -k.hub3.hi * p0 - e2 * k.m2.hi * f0 + e4 * k.inv.hi * lap;
    } else if constexpr (EQ == EQ_APPROX) {
      const T e2 = (T)1 + (T)cp.ps.v[v], e4 = (T)1 + (T)cp.ps4.v[v];
      return (-k.hub3.hi + (T)4 * (T)cp.dps.v[v]) * p0 - e2 * k.m2.hi * f0 + e4 * k.inv.hi * lap;
    } else if constexpr (EQ == EQ_LAMBDA) {
      return -k.hub3.hi * p0 - k.m2.hi * f0 - k.q1.hi * f0 * f0 * f0 + k.inv.hi * lap;
    } else if constexpr (EQ == EQ_SQRT) {  // q2 = 1 / f_a^2
      return -k.hub3.hi * p0 - k.m2.hi * f0 * rsqrt(1.0 + f0 * f0 * k.q2.hi) + k.inv.hi * lap;
    } else {
      return -k.hub3.hi * p0 - k.m2.hi * f0 + k.inv.hi * lap;
    }
  } else {  // FP32: kpi_f32 of cf_f32x2.cuh, one site
    const StageCoefL<float> kl{k.m2.lane(), k.inv.lane(), k.hub3.lane(), k.q1.lane(), k.q2.lane()};
    float ps = 0.0f, dps = 0.0f, ps4 = 0.0f;
    if constexpr (EqOf<EQ>::coupled) ps = (float)cp.ps.v[v];
    if constexpr (EQ == EQ_COMOV || EQ == EQ_APPROX) dps = (float)cp.dps.v[v];
    if constexpr (EQ == EQ_APPROX) ps4 = (float)cp.ps4.v[v];
    return kpi_f32<EQ, float>(p0, f0, lap, ps, dps, ps4, kl);
  }
}

// Plane staging.  Double-buffered (DB): plane a goes to buffer (a - a_begin) & 1
// and one barrier per plane suffices -- a thread that writes buffer k for plane
// a + 2 has passed the barrier of plane a + 1, which every thread reaches only
// after it has finished reading plane a.  Single-buffered: a second barrier
// before the buffer is overwritten, and fewer live registers (measured faster
// for FP64, where registers limit the resident CTAs; DB is faster for FP32).
template <typename S>
struct DoubleBuffered {
  static constexpr bool value = sizeof(S) == 4;
};

template <typename S, int H, int TXv, int TYv, int VW = VecT<S>::n>
struct TileSmem {
  static constexpr int V = VW;
  static constexpr int TW = TXv * V;
  static constexpr int SP = TW + 2 * H;
  static constexpr int SR = TYv + 2 * H;
  static constexpr int plane = SR * SP;
  static constexpr int count = (DoubleBuffered<S>::value ? 2 : 1) * plane;
};

// FULL: the caller guarantees the tile lies inside the lattice (N % TW == 0 and
// N % TYv == 0), so the active width and height are compile-time constants.
template <typename S, int H, int EQ, int STAGE, int TXv, int TYv, bool FULL = false>
__device__ __forceinline__ void stage_tile(const StageArgs<S> &A, int c0, int b0, int a_begin, int a_end, S *sm2) {
  using TS = TileSmem<S, H, TXv, TYv>;
  constexpr bool DB = DoubleBuffered<S>::value;
  constexpr int V = TS::V;
  constexpr int TW = TS::TW;
  constexpr int SP = TS::SP;
  const int N = A.N;
  const long long N3 = A.N3;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * TXv + tx;
  const int twe = FULL ? TW : min(TW, N - c0);    // active tile width (a multiple of V: N % 8 == 0)
  const int tye = FULL ? TYv : min(TYv, N - b0);  // active tile height
  const int sre = tye + 2 * H;       // shared-memory rows in use
  const int c = c0 + tx * V;
  const int b = b0 + ty;
  const bool act = (tx * V) < twe && ty < tye;
  const long long rowoff = (long long)N * b + c;  // offset within a plane
  const long long NN = (long long)N * N;
  const S *phi_in = A.yin;
  const S *pi_in = A.yin + N3;
  using T = typename Arith<S>::T;
  // FP32: the 13-point sum comes times 12 (lap13_f32), its 1/12 rides on the coefficient
  const double invc = sizeof(T) == 4 ? lap_coef_f32<H>(A.inv) : A.inv;
  const StageCoef<T> kc{Coef<T>(A.m2), Coef<T>(invc), Coef<T>(A.hub3), Coef<T>(A.q1), Coef<T>(A.q2)};
  const Coef<T> cy(A.cy), c6(A.dt6);
  const CoarseCols<V> cc = coarse_cols<EQ, V>(A.cmap, act, b, c);

  Pack<S> q[2 * H + 1];
  if (act) {
#pragma unroll
    for (int j = 0; j < 2 * H; ++j) q[j + 1] = ldv(phi_in + NN * wrap_n(a_begin - H + j, N) + rowoff);
  }

  for (int a = a_begin; a < a_end; ++a) {
    const long long site = NN * a + rowoff;
#pragma unroll
    for (int j = 0; j < 2 * H; ++j) q[j] = q[j + 1];
    Pack<S> pi0, xp, xq, cp, cq, lp{}, lq{};
    Coupling<S, V> cpl;
    if (act) {
      q[2 * H] = ldv(phi_in + NN * wrap_n(a + H, N) + rowoff);
      pi0 = ldv(pi_in + site);
      if constexpr (STAGE == 2 || STAGE == 3 || STAGE == 4) {
        xp = ldv_rw(A.x + site);
        xq = ldv_rw(A.x + N3 + site);
        cp = ldv_rw(A.acc + site);
        cq = ldv_rw(A.acc + N3 + site);
      }
      if constexpr (STAGE == 4 && sizeof(S) == 4) {
        lp = ldv_rw(A.xlo + site);
        lq = ldv_rw(A.xlo + N3 + site);
      }
      if constexpr (EqOf<EQ>::coupled)
        load_coupling<EQ, S, V>(cpl, A.psi, A.dpsi, site, A.M, EqOf<EQ>::coarse ? __ldg(A.cmap + a) : 0, cc);
    }
    S *sm = sm2;
    if constexpr (DB) {
      sm = sm2 + ((a - a_begin) & 1) * TS::plane;
    } else {
      __syncthreads();  // the previous plane's shared-memory reads are complete
    }
    if (act) {
#pragma unroll
      for (int v = 0; v < V; ++v) sm[(ty + H) * SP + H + tx * V + v] = q[H].v[v];
      // halo rows: H above the tile and H below its active height, interior columns
      if (ty < H || ty >= tye - H) {
        const int r = (ty < H) ? ty : ty + 2 * H;
        const int gb = wrap_n(b0 - H + r, N);
        const Pack<S> h = ldv(phi_in + NN * a + (long long)N * gb + c);
#pragma unroll
        for (int v = 0; v < V; ++v) sm[r * SP + H + tx * V + v] = h.v[v];
      }
      // (a thread that is both in the top and the bottom band, tye < 2H, writes its bottom row below)
      if (ty < H && ty >= tye - H) {
        const int r = ty + 2 * H;
        const int gb = wrap_n(b0 - H + r, N);
        const Pack<S> h = ldv(phi_in + NN * a + (long long)N * gb + c);
#pragma unroll
        for (int v = 0; v < V; ++v) sm[r * SP + H + tx * V + v] = h.v[v];
      }
    }
    // halo columns: H left and H right of the active width, all rows in use
    for (int i = tid; i < sre * 2 * H; i += TXv * TYv) {
      const int r = i / (2 * H);
      const int j = i % (2 * H);
      const int gb = wrap_n(b0 - H + r, N);
      int col, gc;
      if (j < H) {
        col = j;
        gc = wrap_n(c0 - H + j, N);
      } else {
        col = twe + H + (j - H);
        gc = wrap_n(c0 + twe + (j - H), N);
      }
      sm[r * SP + col] = phi_in[NN * a + (long long)N * gb + gc];
    }
    __syncthreads();
    if (!act) continue;

    Pack<S> o_phi, o_pi;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const int col = H + tx * V + v;
      const int row = ty + H;
      const T f0 = (T)q[H].v[v];
      const T lap = lap_at<S, H, SP>(q, sm, row, col, v);
      const T p0 = (T)pi0.v[v];
      const T kphi = p0;
      const T kpi = kpi_of<EQ, S, V>(p0, f0, lap, cpl, v, kc);
      if constexpr (STAGE == 0) {
        o_phi.v[v] = (S)kphi;
        o_pi.v[v] = (S)kpi;
      } else if constexpr (STAGE == 1) {
        cp.v[v] = (S)kphi;
        cq.v[v] = (S)kpi;
        o_phi.v[v] = (S)cy.fma(kphi, f0);
        o_pi.v[v] = (S)cy.fma(kpi, p0);
      } else if constexpr (STAGE == 2 || STAGE == 3) {
        cp.v[v] = (S)((T)cp.v[v] + (T)2 * kphi);
        cq.v[v] = (S)((T)cq.v[v] + (T)2 * kpi);
        o_phi.v[v] = (S)cy.fma(kphi, (T)xp.v[v]);
        o_pi.v[v] = (S)cy.fma(kpi, (T)xq.v[v]);
      } else {  // STAGE 4
        state_update(xp.v[v], lp.v[v], (T)cp.v[v] + kphi, c6, xp.v[v], lp.v[v]);
        state_update(xq.v[v], lq.v[v], (T)cq.v[v] + kpi, c6, xq.v[v], lq.v[v]);
      }
    }
    if constexpr (STAGE == 0) {
      stv(A.yout + site, o_phi);
      stv(A.yout + N3 + site, o_pi);
    } else if constexpr (STAGE <= 3) {
      stv(A.acc + site, cp);
      stv(A.acc + N3 + site, cq);
      stv(A.yout + site, o_phi);
      stv(A.yout + N3 + site, o_pi);
    } else {
      stv(A.x + site, xp);
      stv(A.x + N3 + site, xq);
      if constexpr (sizeof(S) == 4) {
        stv(A.xlo + site, lp);
        stv(A.xlo + N3 + site, lq);
      }
    }
  }
  // the caller may stage another tile into the same buffers next (ensemble work lists)
  __syncthreads();
}

}  // namespace cfb
