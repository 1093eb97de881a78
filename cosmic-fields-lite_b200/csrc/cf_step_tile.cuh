// cf_step_tile.cuh -- one whole RK4 step in one pass over a (b, c) tile,
// marching along a (7-point Laplacian).
//
// In f(phi, pi) = (pi, F(phi, pi, lap phi)) only pi has a spatial derivative, so
// every stage input's phi is pointwise in the previous input (cf_pair_tile.cuh).
// Chained over the four stages that makes the whole step depend on x within a
// distance of 2 (stage 3 takes the Laplacian of yb_phi = x_phi + dt/2 ya_pi,
// ya_pi = x_pi + dt/2 k1_pi, k1_pi needs lap x_phi):
//
//   phase 1 (plane q, its tile and a 1-site ring):  from x (planes q-1..q+1, ring 2)
//     k1 = F(x_pi, x_phi, lap x_phi)                    [t]
//     ya_phi = x_phi + dt/2 x_pi,  ya_pi = x_pi + dt/2 k1
//     k2 = F(ya_pi, ya_phi, lap ya_phi)                 [t + dt/2]
//     yb = x + dt/2 (ya_pi, k2),  yc_phi = x_phi + dt yb_pi
//   phase 2 (plane r, its tile):  from yb_phi, yc_phi of planes r-1..r+1 (ring 1)
//     k3 = F(yb_pi, yb_phi, lap yb_phi)                 [t + dt/2]
//     yc_pi = x_pi + dt k3
//     k4 = F(yc_pi, yc_phi, lap yc_phi)                 [t + dt]
//     x += dt/6 (k1 + 2 k2 + 2 k3 + k4)
//
// While plane p = q + 1 streams in, phase 1 runs on plane q = p - 1 and phase 2 on
// plane r = p - 2.  HBM moves the state once (x hi in, x hi out to a second buffer,
// x lo in place) plus the curvature at three times: 8 (+6) words per site-update
// against 18 (+8) for the paired passes.  Every value is formed and rounded where
// the paired-stage kernels form and round it (same lap order, same kpi_of, the same
// storage-type roundings of the stage inputs and the accumulator), so the states are
// bit-identical.
//
// The new phi and pi go to a buffer other than x: ring sites of a plane belong to
// neighbouring tiles, and planes a_begin-2 .. a_end+1 to neighbouring a-chunks, which
// may have moved on already.  The lo words are touched only at a thread's own sites.
//
// Shared memory per CTA: x_phi and x_pi of planes p-3..p+1 with a 2-site ring in a
// ring of four planes, filled by cp.async one plane ahead of use (the copies of
// plane p+1 run under the compute of planes p-1, p-2); yb_phi and yc_phi with a 1-site
// ring in a ring of three planes; and, in a ring of two, what phase 1 hands to phase
// 2 at the tile's own sites one plane later (yb_pi and the accumulator).  Rows have
// the interior at a 16-byte boundary, so a thread reads its own sites and the rows
// and planes next to them as 16-byte vectors (no bank conflicts), and only the two
// c-neighbours beyond its vector as single words.
#pragma once

#include "cf_stage_tile.cuh"

namespace cfb {

template <typename S>
struct StepArgs {
  const S *xphi;  // state phi, pi (hi words in FP32_COMP), read only
  const S *xpi;
  S *ophi;        // the new phi, pi (another buffer)
  S *opi;
  S *xlo;         // FP32_COMP lo words [phi | pi], in place
  const S *psi[3];   // curvature at t, t + dt/2, t + dt (StageArgs::psi / dpsi)
  const S *dpsi[3];
  const int *cmap;
  int M;
  int N;
  int a_chunk;
  long long N3;
  double q1, q2;
  double m2;
  double inv[3], hub3[3];  // h^-2 a^-2 and 3H at t, t + dt/2, t + dt
  double dt2, dt, dt6;
};

template <typename S, int TXv, int TYv>
struct StepSmem {
  static constexpr int V = VecT<S>::n;
  static constexpr int TW = TXv * V;
  static constexpr int O = V;              // column of the first interior site (16-byte aligned)
  static constexpr int SP = TW + 2 * O;    // row pitch of every plane array
  static constexpr int R2 = TYv + 4, P2 = R2 * SP;  // 2-ring planes (x_phi, x_pi)
  static constexpr int R1 = TYv + 2, P1 = R1 * SP;  // 1-ring planes (yb_phi, yc_phi)
  static constexpr int PD = TYv * TW;               // own sites
  static constexpr int count = 4 * 2 * P2 + 3 * 2 * P1 + 2 * 3 * PD;
};

// 7-point Laplacian sum in the order of lap_at: (-6 f0 + a+ + a- + b+ + b-) + (c+ + c-)
template <typename T>
__device__ __forceinline__ T lap7(T f0, T ap, T am, T bp, T bm, T cp, T cm) {
  if constexpr (sizeof(T) == 4) {
    return lap7_f32<float>(f0, ap, am, bp, bm, cp, cm);
  } else {
    const T s = (T)-6 * f0 + ap + am + bp + bm;
    return s + (cp + cm);
  }
}

// Curvature values of one site (a ring site of phase 1).
template <int EQ, typename S>
__device__ __forceinline__ void coupling_at(Coupling<S, 1> &cp, const S *psi, const S *dpsi, long long site,
                                            const int *cmap, int M, int a, int b, int c) {
  if constexpr (EqOf<EQ>::psi_plane) cp.ps.v[0] = __ldg(psi + site);
  if constexpr (EqOf<EQ>::dpsi_plane) cp.dps.v[0] = __ldg(dpsi + site);
  if constexpr (EqOf<EQ>::coarse) {
    const int idx = (__ldg(cmap + a) * M + __ldg(cmap + b)) * M + __ldg(cmap + c);
    cp.ps.v[0] = __ldg(psi + 4 * (long long)idx);
    cp.ps4.v[0] = __ldg(psi + 4 * (long long)idx + 1);
    cp.dps.v[0] = __ldg(psi + 4 * (long long)idx + 2);
  }
}

// Asynchronous global -> shared copies (cp.async; completion per commit group).
__device__ __forceinline__ void cp_async_16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_8(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// A hint that brings `bytes` (a multiple of 16, 16-byte aligned, inside an allocation)
// from global memory into L2 without occupying registers or shared memory.
__device__ __forceinline__ void prefetch_l2(const void *p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// A thread's V sites of a row, 16 bytes from shared memory.
template <typename S, int V>
__device__ __forceinline__ Pack<S, V> lds(const S *p) {
  return unpack<S, V>(*reinterpret_cast<const typename VecOf<S, V>::T *>(p));
}
template <typename S, int V>
__device__ __forceinline__ void sts(S *p, const Pack<S, V> &r) {
  stv<S, V>(p, r);
}

// One site's 7-point stencil values: centre, a+-, b+-, c+-.
template <typename T>
struct Star {
  T f0, ap, am, bp, bm, cp, cm;
};

// The stencil of the V sites of a row at `o` in planes (pm, p0, pp) of pitch SP, as vectors.
template <typename S, int V, int SP>
struct RowStar {
  Pack<S, V> c, n, s, a, b;
  S l, r;
  __device__ __forceinline__ void load(const S *p0, const S *pm, const S *pp, int o) {
    c = lds<S, V>(p0 + o);
    n = lds<S, V>(p0 + o + SP);
    s = lds<S, V>(p0 + o - SP);
    a = lds<S, V>(pp + o);
    b = lds<S, V>(pm + o);
    l = p0[o - 1];
    r = p0[o + V];
  }
  template <typename T>
  __device__ __forceinline__ Star<T> at(int v) const {
    return Star<T>{(T)c.v[v], (T)a.v[v], (T)b.v[v], (T)n.v[v], (T)s.v[v], (T)(v + 1 < V ? c.v[v + 1] : r),
                   (T)(v > 0 ? c.v[v - 1] : l)};
  }
};

template <typename T>
__device__ __forceinline__ T lap_of(const Star<T> &s) {
  return lap7<T>(s.f0, s.ap, s.am, s.bp, s.bm, s.cp, s.cm);
}

// FP32: the stencil of sites (2l, 2l+1) of a row's four as lane pairs (cf_f32x2.cuh).
// The c-neighbours pair across the vector: lane 0 takes (c1, c2) and (l, c0), lane 1
// (c3, r) and (c1, c2).
template <int SP>
__device__ __forceinline__ Star<float2> star2(const RowStar<float, 4, SP> &R, int l) {
  const int v = 2 * l;
  return Star<float2>{make_float2(R.c.v[v], R.c.v[v + 1]), make_float2(R.a.v[v], R.a.v[v + 1]),
                      make_float2(R.b.v[v], R.b.v[v + 1]), make_float2(R.n.v[v], R.n.v[v + 1]),
                      make_float2(R.s.v[v], R.s.v[v + 1]),
                      make_float2(R.c.v[v + 1], l == 0 ? R.c.v[2] : R.r),
                      make_float2(l == 0 ? R.l : R.c.v[1], R.c.v[v])};
}
__device__ __forceinline__ float2 lap_of2(const Star<float2> &s) {
  return lap7_f32<float2>(s.f0, s.ap, s.am, s.bp, s.bm, s.cp, s.cm);
}
template <int V>
__device__ __forceinline__ float2 lane2(const Pack<float, V> &p, int l) {
  return make_float2(p.v[2 * l], p.v[2 * l + 1]);
}
template <int V>
__device__ __forceinline__ void set2(Pack<float, V> &p, int l, float2 x) {
  p.v[2 * l] = x.x;
  p.v[2 * l + 1] = x.y;
}
// The curvature lanes of a stage (ps, dps, ps4 of kpi_f32; zero where the equation has none).
template <int EQ, int V>
__device__ __forceinline__ void coupling2(const Coupling<float, V> &c, int l, float2 &ps, float2 &dps, float2 &ps4) {
  ps = dps = ps4 = make_float2(0.0f, 0.0f);
  if constexpr (EqOf<EQ>::coupled) ps = lane2(c.ps, l);
  if constexpr (EQ == EQ_COMOV || EQ == EQ_APPROX) dps = lane2(c.dps, l);
  if constexpr (EQ == EQ_APPROX) ps4 = lane2(c.ps4, l);
}

// ya_phi = x_phi + dt/2 x_pi at each point of a stencil (the stored stage input of the
// paired kernels, formed here where it is needed).
template <typename S, typename T>
__device__ __forceinline__ Star<T> ya_star(const Star<T> &f, const Star<T> &p, const Coef<T> &ch) {
  return Star<T>{(T)w_of((S)f.f0, (S)p.f0, ch), (T)w_of((S)f.ap, (S)p.ap, ch), (T)w_of((S)f.am, (S)p.am, ch),
                 (T)w_of((S)f.bp, (S)p.bp, ch), (T)w_of((S)f.bm, (S)p.bm, ch), (T)w_of((S)f.cp, (S)p.cp, ch),
                 (T)w_of((S)f.cm, (S)p.cm, ch)};
}

// RINGW: the CTA has two more thread rows (ring warps, ty = TYv and TYv + 1) beside the
// TYv rows of own sites.  They copy the ring rows and columns, form the two ring rows
// of phase 1 while the own rows form theirs, and form the ring columns of plane q
// after the second barrier, while the own rows run phase 2 on plane r: phase 2 reads
// plane q = r + 1 at own sites only (its a-neighbour), and q's ring is first read by
// phase 2 one plane later.  Without RINGW the first two own rows take the ring rows
// and the last threads the ring columns, both before the second barrier.
template <typename S, int EQ, int TXv, int TYv, bool FULL = false, bool RINGW = false>
__device__ __forceinline__ void step_tile(const StepArgs<S> &A, int c0, int b0, int a_begin, int a_end, S *smem) {
  using SM = StepSmem<S, TXv, TYv>;
  using T = typename Arith<S>::T;
  constexpr int V = SM::V, TW = SM::TW, O = SM::O, SP = SM::SP, NT = TXv * (TYv + (RINGW ? 2 : 0)), PD = SM::PD;
  // With ring warps, the threads that form plane q's ring columns (the last 2 (TY + 2))
  // and those that copy the next planes' ring columns (the last 2 (TY + 4)) read and
  // refill the same slot columns ordered by __syncwarp alone: they must share one warp.
  static_assert(!RINGW || (2 * (TYv + 4) <= 32 && NT % 32 == 0), "ring columns outside the last warp");
  S *XF = smem;               // x_phi, 4 planes of P2
  S *XP = XF + 4 * SM::P2;    // x_pi,  4 planes of P2
  S *YB = XP + 4 * SM::P2;    // yb_phi, 3 planes of P1
  S *YC = YB + 3 * SM::P1;    // yc_phi, 3 planes of P1
  S *DL = YC + 3 * SM::P1;    // 2 planes x (yb_pi, acc_phi, acc_pi) of PD
  const int N = A.N;
  const long long N3 = A.N3, NN = (long long)N * N;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TXv + tx;
  const int twe = FULL ? TW : min(TW, N - c0);
  const int tye = FULL ? TYv : min(TYv, N - b0);
  const int c = c0 + tx * V, b = b0 + ty;
  const bool act = (tx * V) < twe && ty < tye;
  const bool colact = (tx * V) < twe;
  const long long rowoff = (long long)N * b + c;
  const StageCoef<T> k1c{Coef<T>(A.m2), Coef<T>(A.inv[0]), Coef<T>(A.hub3[0]), Coef<T>(A.q1), Coef<T>(A.q2)};
  const StageCoef<T> k2c{Coef<T>(A.m2), Coef<T>(A.inv[1]), Coef<T>(A.hub3[1]), Coef<T>(A.q1), Coef<T>(A.q2)};
  const StageCoef<T> k4c{Coef<T>(A.m2), Coef<T>(A.inv[2]), Coef<T>(A.hub3[2]), Coef<T>(A.q1), Coef<T>(A.q2)};
  const Coef<T> ch(A.dt2), cf(A.dt);
  const Coef<T> c6(A.dt6);
  // FP32: the same coefficients as lane pairs for the paired arithmetic
  const C2 M2p = coef_f32x2(A.m2), Q1p = coef_f32x2(A.q1), Q2p = coef_f32x2(A.q2);
  const C2 INVp[3] = {coef_f32x2(A.inv[0]), coef_f32x2(A.inv[1]), coef_f32x2(A.inv[2])};
  const C2 HUBp[3] = {coef_f32x2(A.hub3[0]), coef_f32x2(A.hub3[1]), coef_f32x2(A.hub3[2])};
  const C2 CHp = coef_f32x2(A.dt2), CFp = coef_f32x2(A.dt), C6p = coef_f32x2(A.dt6);
  const CoarseCols<V> cc = coarse_cols<EQ, V>(A.cmap, act, b, c);
  auto s4 = [&](int p) { return (p - a_begin + 4) & 3; };
  auto s3 = [&](int p) { return (p - a_begin + 3) % 3; };
  auto dslot = [&](int p) { return DL + ((p - a_begin + 2) & 1) * 3 * PD; };
  const int own2 = (ty + 2) * SP + O + tx * V;  // own sites in a 2-ring plane
  const int own1 = (ty + 1) * SP + O + tx * V;  // ... in a 1-ring plane
  const int od = ty * TW + tx * V;              // ... in a DL array

  // copies of plane p (x_phi, x_pi; tile and 2-ring) into slot s4(p)
  auto issue = [&](int p) {
    const long long poff = NN * wrap_n(p, N);
    S *xf = XF + s4(p) * SM::P2, *xp = XP + s4(p) * SM::P2;
    if (act) {
      cp_async_16(xf + own2, A.xphi + poff + rowoff);
      cp_async_16(xp + own2, A.xpi + poff + rowoff);
    }
    if constexpr (RINGW) {  // ring rows: ring warp 0 the 2 above the tile, ring warp 1 the 2 below
      if (ty >= TYv && colact) {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const int r2 = ty == TYv ? k : tye + 2 + k;
          const long long off = poff + (long long)N * wrap_n(b0 - 2 + r2, N) + c;
          cp_async_16(xf + r2 * SP + O + tx * V, A.xphi + off);
          cp_async_16(xp + r2 * SP + O + tx * V, A.xpi + off);
        }
      }
    } else if (ty < 4 && colact) {  // ring rows: 2 above the tile, 2 below its active height
      const int r2 = ty < 2 ? ty : tye + ty;
      const long long off = poff + (long long)N * wrap_n(b0 - 2 + r2, N) + c;
      cp_async_16(xf + r2 * SP + O + tx * V, A.xphi + off);
      cp_async_16(xp + r2 * SP + O + tx * V, A.xpi + off);
    }
    for (int i = NT - 1 - tid; i < (tye + 4) * 2; i += NT) {  // ring columns (the last warps): pairs
      const int r2 = i >> 1, side = i & 1;
      const int gc = wrap_n(side ? c0 + twe : c0 - 2, N);
      const int col = side ? O + twe : O - 2;
      const long long off = poff + (long long)N * wrap_n(b0 - 2 + r2, N) + gc;
      if constexpr (sizeof(S) == 8) {
        cp_async_16(xf + r2 * SP + col, A.xphi + off);
        cp_async_16(xp + r2 * SP + col, A.xpi + off);
      } else {
        cp_async_8(xf + r2 * SP + col, A.xphi + off);
        cp_async_8(xp + r2 * SP + col, A.xpi + off);
      }
    }
  };

  // Stages 1-2 at V sites of a row of plane q: returns yb_phi, yc_phi and, for own
  // sites, what phase 2 takes (yb_pi, acc_phi, acc_pi)
  auto phase1_row = [&](int q, int o2, const Coupling<S, V> &ct, const Coupling<S, V> &ch2, Pack<S, V> &yb,
                        Pack<S, V> &yc, Pack<S, V> &ybpi, Pack<S, V> &aphi, Pack<S, V> &api) {
    RowStar<S, V, SP> F, P;
    F.load(XF + s4(q) * SM::P2, XF + s4(q - 1) * SM::P2, XF + s4(q + 1) * SM::P2, o2);
    P.load(XP + s4(q) * SM::P2, XP + s4(q - 1) * SM::P2, XP + s4(q + 1) * SM::P2, o2);
    if constexpr (sizeof(S) == 4) {  // two sites per paired FP32 instruction, same bits
      const StageCoefL<float2> K1{M2p, INVp[0], HUBp[0], Q1p, Q2p}, K2{M2p, INVp[1], HUBp[1], Q1p, Q2p};
#pragma unroll
      for (int l = 0; l < V / 2; ++l) {
        const Star<float2> fs = star2(F, l), ps = star2(P, l);
        const float2 f0 = fs.f0, p0 = ps.f0;
        float2 c_ps, c_dps, c_ps4;
        coupling2<EQ>(ct, l, c_ps, c_dps, c_ps4);
        const float2 k1 = kpi_f32<EQ, float2>(p0, f0, lap_of2(fs), c_ps, c_dps, c_ps4, K1);
        const float2 yapi = c_fma(CHp, k1, p0);
        const Star<float2> ya{c_fma(CHp, ps.f0, fs.f0), c_fma(CHp, ps.ap, fs.ap), c_fma(CHp, ps.am, fs.am),
                              c_fma(CHp, ps.bp, fs.bp), c_fma(CHp, ps.bm, fs.bm), c_fma(CHp, ps.cp, fs.cp),
                              c_fma(CHp, ps.cm, fs.cm)};
        coupling2<EQ>(ch2, l, c_ps, c_dps, c_ps4);
        const float2 k2 = kpi_f32<EQ, float2>(yapi, ya.f0, lap_of2(ya), c_ps, c_dps, c_ps4, K2);
        const float2 bpi = c_fma(CHp, k2, p0);
        set2(yb, l, c_fma(CHp, yapi, f0));
        set2(yc, l, c_fma(CFp, bpi, f0));
        set2(ybpi, l, bpi);
        set2(aphi, l, p_fma(p_splat<float2>(2.0f), yapi, p0));
        set2(api, l, p_fma(p_splat<float2>(2.0f), k2, k1));
      }
    } else {
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const Star<T> fs = F.template at<T>(v), ps = P.template at<T>(v);
        const T f0 = fs.f0, p0 = ps.f0;
        const T k1 = kpi_of<EQ, S, V>(p0, f0, lap_of(fs), ct, v, k1c);
        const S yapi = (S)ch.fma(k1, p0);
        const Star<T> ya = ya_star<S, T>(fs, ps, ch);
        const T k2 = kpi_of<EQ, S, V>((T)yapi, ya.f0, lap_of(ya), ch2, v, k2c);
        const S bpi = (S)ch.fma(k2, p0);
        yb.v[v] = (S)ch.fma((T)yapi, f0);
        yc.v[v] = (S)cf.fma((T)bpi, f0);
        ybpi.v[v] = bpi;
        aphi.v[v] = (S)((T)(S)p0 + (T)2 * (T)yapi);
        api.v[v] = (S)((T)(S)k1 + (T)2 * k2);
      }
    }
  };

  // Stages 1-2 at one ring site (r1, col) of the 1-ring plane q (col in the row's
  // shared-memory coordinates): writes its yb_phi, yc_phi
  auto ring_site = [&](int q, int qm, long long qoff, S *yb, S *yc, int r1, int col) {
    const int o2 = (r1 + 1) * SP + col;
    const int gb = wrap_n(b0 - 1 + r1, N), gc = wrap_n(c0 + col - O, N);
    const long long site = qoff + (long long)N * gb + gc;
    Coupling<S, 1> ct, ch2;
    if constexpr (EqOf<EQ>::coupled) {
      coupling_at<EQ, S>(ct, A.psi[0], A.dpsi[0], site, A.cmap, A.M, qm, gb, gc);
      if constexpr (EQ == EQ_FIXED)
        ch2 = ct;
      else
        coupling_at<EQ, S>(ch2, A.psi[1], A.dpsi[1], site, A.cmap, A.M, qm, gb, gc);
    }
    const S *f0p = XF + s4(q) * SM::P2, *fmp = XF + s4(q - 1) * SM::P2, *fpp = XF + s4(q + 1) * SM::P2;
    const S *x0p = XP + s4(q) * SM::P2, *xmp = XP + s4(q - 1) * SM::P2, *xpp = XP + s4(q + 1) * SM::P2;
    const Star<T> fs{(T)f0p[o2], (T)fpp[o2], (T)fmp[o2], (T)f0p[o2 + SP], (T)f0p[o2 - SP], (T)f0p[o2 + 1],
                     (T)f0p[o2 - 1]};
    const Star<T> ps{(T)x0p[o2], (T)xpp[o2], (T)xmp[o2], (T)x0p[o2 + SP], (T)x0p[o2 - SP], (T)x0p[o2 + 1],
                     (T)x0p[o2 - 1]};
    const T f0 = fs.f0, p0 = ps.f0;
    const T k1 = kpi_of<EQ, S, 1>(p0, f0, lap_of(fs), ct, 0, k1c);
    const S yapi = (S)ch.fma(k1, p0);
    const Star<T> ya = ya_star<S, T>(fs, ps, ch);
    const T k2 = kpi_of<EQ, S, 1>((T)yapi, ya.f0, lap_of(ya), ch2, 0, k2c);
    const S bpi = (S)ch.fma(k2, p0);
    yb[r1 * SP + col] = (S)ch.fma((T)yapi, f0);
    yc[r1 * SP + col] = (S)cf.fma((T)bpi, f0);
  };

  // L2 prefetch, one plane ahead, of what phases 1 and 2 load straight from global
  // memory: the curvature at t and t + dt/2 of plane p for phase 1 (own and ring rows),
  // and the curvature at t + dt and the lo words of plane p for phase 2 (own rows).  One
  // thread per row and array issues it, so those loads wait on L2 rather than HBM; a
  // lead of one plane (a few microseconds) covers the HBM latency without leaving the
  // lines in L2 long enough to be evicted.
  auto prefetch_rows = [&](int p, bool phase1) {
    if (tx != 0 || !colact) return;
    const bool own = ty < TYv;
    if (own ? ty >= tye : (!RINGW || !phase1)) return;
    const int gb = own ? b : wrap_n(ty == TYv ? b0 - 1 : b0 + tye, N);
    const long long off = NN * wrap_n(p, N) + (long long)N * gb + c0;
    const unsigned bytes = (unsigned)(twe * sizeof(S));
    if (phase1) {
      if constexpr (EqOf<EQ>::psi_plane) {
        prefetch_l2(A.psi[0] + off, bytes);
        if constexpr (EQ != EQ_FIXED) prefetch_l2(A.psi[1] + off, bytes);
      }
      if constexpr (EqOf<EQ>::dpsi_plane) {
        prefetch_l2(A.dpsi[0] + off, bytes);
        prefetch_l2(A.dpsi[1] + off, bytes);
      }
    } else {
      if constexpr (EqOf<EQ>::psi_plane && EQ != EQ_FIXED) prefetch_l2(A.psi[2] + off, bytes);
      if constexpr (EqOf<EQ>::dpsi_plane) prefetch_l2(A.dpsi[2] + off, bytes);
      if constexpr (sizeof(S) == 4) {
        prefetch_l2(A.xlo + off, bytes);
        prefetch_l2(A.xlo + N3 + off, bytes);
      }
    }
  };

  issue(a_begin - 2);
  cp_async_commit();
  for (int p = a_begin - 2; p <= a_end + 1; ++p) {
    if (p + 1 <= a_end + 1) issue(p + 1);
    cp_async_commit();
    // phase 1 takes plane p next iteration, phase 2 plane p - 1
    if (p >= a_begin - 1 && p <= a_end) prefetch_rows(p, true);
    if (p - 1 >= a_begin && p - 1 <= a_end - 1) prefetch_rows(p - 1, false);
    cp_async_wait_one();  // this thread's copies of plane p have landed
    __syncthreads();      // everyone's; and phase 2 of the last plane is done with YB / YC

    // ---- phase 1 on plane q = p - 1: the tile and its 1-ring
    const int q = p - 1;
    if (q >= a_begin - 1) {
      const int qm = wrap_n(q, N);
      const long long qoff = NN * qm;
      S *yb = YB + s3(q) * SM::P1, *yc = YC + s3(q) * SM::P1;
      if (act) {  // own sites
        Coupling<S, V> ct, ch2;
        if constexpr (EqOf<EQ>::coupled) {
          const int ca = EqOf<EQ>::coarse ? __ldg(A.cmap + qm) : 0;
          load_coupling<EQ, S, V>(ct, A.psi[0], A.dpsi[0], qoff + rowoff, A.M, ca, cc);
          if constexpr (EQ == EQ_FIXED)
            ch2 = ct;
          else
            load_coupling<EQ, S, V>(ch2, A.psi[1], A.dpsi[1], qoff + rowoff, A.M, ca, cc);
        }
        Pack<S, V> vb, vc, vbp, vap, vpp;
        phase1_row(q, own2, ct, ch2, vb, vc, vbp, vap, vpp);
        sts<S, V>(yb + own1, vb);
        sts<S, V>(yc + own1, vc);
        S *dl = dslot(q);
        sts<S, V>(dl + od, vbp);
        sts<S, V>(dl + PD + od, vap);
        sts<S, V>(dl + 2 * PD + od, vpp);
      }
      // ring rows of the 1-ring plane: b0 - 1 and b0 + tye
      if ((RINGW ? ty >= TYv : ty < 2) && colact) {
        const int r1 = ty == (RINGW ? TYv : 0) ? 0 : tye + 1;
        const int gb = wrap_n(b0 - 1 + r1, N);
        const long long site = qoff + (long long)N * gb + c;
        Coupling<S, V> ct, ch2;
        if constexpr (EqOf<EQ>::coupled) {
          CoarseCols<V> cr = cc;
          if constexpr (EqOf<EQ>::coarse) {
            cr.row_b = __ldg(A.cmap + gb);
#pragma unroll
            for (int v = 0; v < V; ++v) cr.col[v] = __ldg(A.cmap + c + v);
          }
          const int ca = EqOf<EQ>::coarse ? __ldg(A.cmap + qm) : 0;
          load_coupling<EQ, S, V>(ct, A.psi[0], A.dpsi[0], site, A.M, ca, cr);
          if constexpr (EQ == EQ_FIXED)
            ch2 = ct;
          else
            load_coupling<EQ, S, V>(ch2, A.psi[1], A.dpsi[1], site, A.M, ca, cr);
        }
        Pack<S, V> vb, vc, vbp, vap, vpp;
        phase1_row(q, (r1 + 1) * SP + O + tx * V, ct, ch2, vb, vc, vbp, vap, vpp);
        sts<S, V>(yb + r1 * SP + O + tx * V, vb);
        sts<S, V>(yc + r1 * SP + O + tx * V, vc);
      }
      // ring columns of the 1-ring plane (corners included): scalars, on the last warps
      // (the first warp takes the ring rows); with RINGW after the barrier below
      if constexpr (!RINGW)
        for (int i = NT - 1 - tid; i < (tye + 2) * 2; i += NT)
          ring_site(q, qm, qoff, yb, yc, i >> 1, (i & 1) ? O + twe : O - 1);
    }
    // Without ring warps the ring columns of plane q are formed above by the last warps,
    // and the barrier makes them visible before phase 2.  With ring warps nothing after
    // this point needs another thread's phase-1 result of this iteration: phase 2 of
    // plane r reads plane q = r + 1 only at the thread's own sites (its a-neighbour,
    // written by the same thread above) and plane r in full (formed last iteration,
    // visible since the barrier at the top); the ring warps' ring columns of plane q
    // read x only.  The barrier at the top of the next iteration orders all of it.
    if constexpr (!RINGW) __syncthreads();

    // ---- RINGW: the ring columns of plane q, beside phase 2.  They read x of planes
    // q-1..q+1 (slot s4(q-1) is refilled by the next iteration's copies: its ring
    // columns by the same last warp, after the __syncwarp) and write YB / YC of plane
    // q at ring columns, which phase 2 below does not read.
    if constexpr (RINGW) {
      if (q >= a_begin - 1) {
        const int qm = wrap_n(q, N);
        for (int i = NT - 1 - tid; i < (tye + 2) * 2; i += NT)
          ring_site(q, qm, NN * qm, YB + s3(q) * SM::P1, YC + s3(q) * SM::P1, i >> 1, (i & 1) ? O + twe : O - 1);
      }
      __syncwarp();
    }

    // ---- phase 2 on plane r = p - 2 (own sites): stages 3 and 4, the update.  Its x_phi,
    // x_pi are still staged (slot s4(r) is next refilled by the copies of plane r + 4,
    // issued after this); DL entries are written and read by the owning thread only.
    const int r = p - 2;
    if (r >= a_begin && act) {
      const int rm = wrap_n(r, N);
      const long long roff = NN * rm;
      Coupling<S, V> cth, cd;
      if constexpr (EqOf<EQ>::coupled) {
        const int ca = EqOf<EQ>::coarse ? __ldg(A.cmap + rm) : 0;
        load_coupling<EQ, S, V>(cth, A.psi[1], A.dpsi[1], roff + rowoff, A.M, ca, cc);
        if constexpr (EQ == EQ_FIXED)
          cd = cth;
        else
          load_coupling<EQ, S, V>(cd, A.psi[2], A.dpsi[2], roff + rowoff, A.M, ca, cc);
      }
      const S *dl = dslot(r);
      const Pack<S, V> xphi = lds<S, V>(XF + s4(r) * SM::P2 + own2), xpi = lds<S, V>(XP + s4(r) * SM::P2 + own2);
      const Pack<S, V> ybpi = lds<S, V>(dl + od), aphi = lds<S, V>(dl + PD + od), api = lds<S, V>(dl + 2 * PD + od);
      RowStar<S, V, SP> B, C;
      B.load(YB + s3(r) * SM::P1, YB + s3(r - 1) * SM::P1, YB + s3(r + 1) * SM::P1, own1);
      C.load(YC + s3(r) * SM::P1, YC + s3(r - 1) * SM::P1, YC + s3(r + 1) * SM::P1, own1);
      Pack<S, V> o1, o2, o3, o4;
      Pack<S, V> lp{}, lq{};
      if constexpr (sizeof(S) == 4) {
        lp = ldv_rw<S, V>(A.xlo + roff + rowoff);
        lq = ldv_rw<S, V>(A.xlo + N3 + roff + rowoff);
      }
      if constexpr (sizeof(S) == 4) {  // two sites per paired FP32 instruction, same bits
        const StageCoefL<float2> K2{M2p, INVp[1], HUBp[1], Q1p, Q2p}, K4{M2p, INVp[2], HUBp[2], Q1p, Q2p};
#pragma unroll
        for (int l = 0; l < V / 2; ++l) {
          const Star<float2> bs = star2(B, l);
          const float2 p0 = lane2(ybpi, l);
          float2 c_ps, c_dps, c_ps4;
          coupling2<EQ>(cth, l, c_ps, c_dps, c_ps4);
          const float2 k3 = kpi_f32<EQ, float2>(p0, bs.f0, lap_of2(bs), c_ps, c_dps, c_ps4, K2);
          const float2 c1phi = p_fma(p_splat<float2>(2.0f), p0, lane2(aphi, l));
          const float2 c1pi = p_fma(p_splat<float2>(2.0f), k3, lane2(api, l));
          const float2 ycpi = c_fma(CFp, k3, lane2(xpi, l));
          const Star<float2> cs = star2(C, l);
          coupling2<EQ>(cd, l, c_ps, c_dps, c_ps4);
          const float2 k4 = kpi_f32<EQ, float2>(ycpi, cs.f0, lap_of2(cs), c_ps, c_dps, c_ps4, K4);
          float2 h1, l1, h2, l2;
          comp_update_f32<float2>(lane2(xphi, l), lane2(lp, l), p_add(c1phi, ycpi), C6p, h1, l1);
          comp_update_f32<float2>(lane2(xpi, l), lane2(lq, l), p_add(c1pi, k4), C6p, h2, l2);
          set2(o1, l, h1);
          set2(o3, l, l1);
          set2(o2, l, h2);
          set2(o4, l, l2);
        }
      } else
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const Star<T> bs = B.template at<T>(v);
        const T p0 = (T)ybpi.v[v];
        const T k3 = kpi_of<EQ, S, V>(p0, bs.f0, lap_of(bs), cth, v, k2c);
        const S c1phi = (S)((T)aphi.v[v] + (T)2 * p0);
        const S c1pi = (S)((T)api.v[v] + (T)2 * k3);
        const S ycpi = (S)cf.fma(k3, (T)xpi.v[v]);
        const Star<T> cs = C.template at<T>(v);
        const T k4 = kpi_of<EQ, S, V>((T)ycpi, cs.f0, lap_of(cs), cd, v, k4c);
        state_update(xphi.v[v], lp.v[v], (T)c1phi + (T)ycpi, c6, o1.v[v], o3.v[v]);
        state_update(xpi.v[v], lq.v[v], (T)c1pi + k4, c6, o2.v[v], o4.v[v]);
      }
      stv(A.ophi + roff + rowoff, o1);
      stv(A.opi + roff + rowoff, o2);
      if constexpr (sizeof(S) == 4) {
        stv(A.xlo + roff + rowoff, o3);
        stv(A.xlo + N3 + roff + rowoff, o4);
      }
    }
  }
  cp_async_wait_all();
  __syncthreads();
}

}  // namespace cfb
