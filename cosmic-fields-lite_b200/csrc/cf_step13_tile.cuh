// cf_step13_tile.cuh -- one whole RK4 step in one pass over a (b, c) tile,
// marching along a, for the 4th-order 13-point Laplacian (FP32 storage).
//
// The whole-step pass of cf_step_tile.cuh with every distance doubled.  The
// 13-point stencil reaches 2 sites, so a step depends on x within 4 (stage 3 takes
// the Laplacian of yb_phi = x_phi + dt/2 ya_pi, and ya_pi needs lap x_phi):
//
//   phase 1 (plane q, its tile and a 2-site ring), from x of planes q-2..q+2 with a
//   4-site ring:   k1, ya, k2, yb = x + dt/2 (ya_pi, k2), yc_phi = x_phi + dt yb_pi
//   phase 2 (plane r = q - 2, its tile), from yb_phi, yc_phi of planes r-2..r+2 with
//   a 2-site ring: k3, yc_pi = x_pi + dt k3, k4, x += dt/6 (k1 + 2 k2 + 2 k3 + k4)
//
// HBM moves the state once, like the 7-point pass: 8 (+6) words per site-update
// against 18 (+8) for the paired passes.  A thread owns 2 consecutive sites of a row
// -- one FP32 lane pair of cf_f32x2.cuh -- so the tile is 64 x TY sites, and two ring
// warps form the 2-site ring (its rows as lane pairs, its columns one site at a
// time).  Every value is formed and rounded as the paired (cf_pair_tile.cuh) and the
// single-stage (cf_stage_tile.cuh) 13-point passes form it, so all three routes give
// the same bits.
//
// Shared memory: x_phi, x_pi of six planes with a 4-site ring (the one being loaded
// and the five phase 1 reads), yb_phi, yc_phi of five planes with a 2-site ring, and
// what phase 1 hands to phase 2 at a thread's own sites two planes later (yb_pi and
// the accumulator) for three planes: 177 KB at 64 x 16 (one CTA per SM), 108 KB at
// 64 x 8 (two).  The plane
// copies are spread over all threads (16-byte cp.async, the ring columns included),
// so they are issued after the plane's barrier: by then no thread still reads the
// slot they fill.  That barrier is the only one per plane: phase 2 reads the planes
// next to r only at the thread's own sites, which the same thread formed.
#pragma once

#include "cf_step_tile.cuh"

namespace cfb {

template <int TXv, int TYv>
struct Step13Smem {
  static constexpr int V = 2;                  // floats per thread: one lane pair
  static constexpr int TW = TXv * V;
  static constexpr int O = 4;                  // first interior column: 16-byte aligned, 4 ring columns before it
  static constexpr int SP = TW + 2 * O;        // row pitch of every plane array
  static constexpr int R4 = TYv + 8, P4 = R4 * SP;  // 4-ring planes (x_phi, x_pi)
  static constexpr int R2 = TYv + 4, P2 = R2 * SP;  // 2-ring planes (yb_phi, yc_phi)
  static constexpr int PD = TYv * TW;               // own sites
  static constexpr int XS = 6, YS = 5, DS = 3;      // plane slots
  static constexpr int count = XS * 2 * P4 + YS * 2 * P2 + DS * 3 * PD;
};

// One site's 13-point stencil values: centre, the first and the second neighbours.
template <typename T>
struct Star13 {
  T f0, ap1, am1, bp1, bm1, cp1, cm1, ap2, am2, bp2, bm2, cp2, cm2;
};

// The Laplacian sum of lap_at<H = 2> (times 12): first neighbours a+, a-, b+, b-,
// c+, c-, then the second ones in the same order.
template <typename L>
__device__ __forceinline__ L lap13_of(const Star13<L> &s) {
  L s1 = p_add(s.ap1, s.am1);
  s1 = p_add(s1, s.bp1);
  s1 = p_add(s1, s.bm1);
  s1 = p_add(s1, s.cp1);
  s1 = p_add(s1, s.cm1);
  L s2 = p_add(s.ap2, s.am2);
  s2 = p_add(s2, s.bp2);
  s2 = p_add(s2, s.bm2);
  s2 = p_add(s2, s.cp2);
  s2 = p_add(s2, s.cm2);
  return lap13_f32<L>(s.f0, s1, s2);
}

__device__ __forceinline__ float2 ld2s(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ void st2s(float *p, float2 v) { *reinterpret_cast<float2 *>(p) = v; }

// The stencil of a thread's lane pair at offset o of the centre plane c (planes m1,
// p1 = a -/+ 1, m2, p2 = a -/+ 2), pitch SP.  The c-neighbours pair across: the
// first ones are (c1, cp2.x) and (cm2.y, c0).
template <int SP>
__device__ __forceinline__ Star13<float2> star13(const float *c, const float *m1, const float *p1, const float *m2,
                                                 const float *p2, int o) {
  Star13<float2> s;
  s.f0 = ld2s(c + o);
  s.cp2 = ld2s(c + o + 2);
  s.cm2 = ld2s(c + o - 2);
  s.ap1 = ld2s(p1 + o);
  s.am1 = ld2s(m1 + o);
  s.bp1 = ld2s(c + o + SP);
  s.bm1 = ld2s(c + o - SP);
  s.cp1 = make_float2(s.f0.y, s.cp2.x);
  s.cm1 = make_float2(s.cm2.y, s.f0.x);
  s.ap2 = ld2s(p2 + o);
  s.am2 = ld2s(m2 + o);
  s.bp2 = ld2s(c + o + 2 * SP);
  s.bm2 = ld2s(c + o - 2 * SP);
  return s;
}
// One site's stencil (a ring-column site).
template <int SP>
__device__ __forceinline__ Star13<float> star13s(const float *c, const float *m1, const float *p1, const float *m2,
                                                 const float *p2, int o) {
  return Star13<float>{c[o],      p1[o],     m1[o],    c[o + SP],      c[o - SP],      c[o + 1], c[o - 1],
                       p2[o],     m2[o],     c[o + 2 * SP], c[o - 2 * SP], c[o + 2], c[o - 2]};
}

// ya_phi = x_phi + dt/2 x_pi at every point of a stencil (the paired route's w plane).
template <typename L>
__device__ __forceinline__ Star13<L> ya13(const Star13<L> &f, const Star13<L> &p, const CoefL<L> &ch) {
  return Star13<L>{c_fma(ch, p.f0, f.f0),   c_fma(ch, p.ap1, f.ap1), c_fma(ch, p.am1, f.am1),
                   c_fma(ch, p.bp1, f.bp1), c_fma(ch, p.bm1, f.bm1), c_fma(ch, p.cp1, f.cp1),
                   c_fma(ch, p.cm1, f.cm1), c_fma(ch, p.ap2, f.ap2), c_fma(ch, p.am2, f.am2),
                   c_fma(ch, p.bp2, f.bp2), c_fma(ch, p.bm2, f.bm2), c_fma(ch, p.cp2, f.cp2),
                   c_fma(ch, p.cm2, f.cm2)};
}

template <int EQ, int TXv, int TYv, bool FULL = false>
__device__ __forceinline__ void step13_tile(const StepArgs<float> &A, int c0, int b0, int a_begin, int a_end,
                                            float *smem) {
  using SM = Step13Smem<TXv, TYv>;
  constexpr int V = SM::V, TW = SM::TW, O = SM::O, SP = SM::SP, NT = TXv * (TYv + 2), PD = SM::PD;
  float *XF = smem;                     // x_phi, 6 planes of P4
  float *XP = XF + SM::XS * SM::P4;     // x_pi, 6 planes of P4
  float *YB = XP + SM::XS * SM::P4;     // yb_phi, 5 planes of P2
  float *YC = YB + SM::YS * SM::P2;     // yc_phi, 5 planes of P2
  float *DL = YC + SM::YS * SM::P2;     // 3 planes x (yb_pi, acc_phi, acc_pi) of PD
  const int N = A.N;
  const long long N3 = A.N3, NN = (long long)N * N;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TXv + tx;
  const int twe = FULL ? TW : min(TW, N - c0);
  const int tye = FULL ? TYv : min(TYv, N - b0);
  const int c = c0 + tx * V, b = b0 + ty;
  const bool colact = (tx * V) < twe;
  const bool act = colact && ty < tye;
  const long long rowoff = (long long)N * b + c;
  // stage coefficients (the Laplacian's with the 13-point sum's 1/12), per site and per lane pair
  const double inv0 = lap_coef_f32<2>(A.inv[0]), inv1 = lap_coef_f32<2>(A.inv[1]), inv2 = lap_coef_f32<2>(A.inv[2]);
  const StageCoefL<float> K1s{coef_f32(A.m2), coef_f32(inv0), coef_f32(A.hub3[0]), coef_f32(A.q1), coef_f32(A.q2)};
  const StageCoefL<float> K2s{coef_f32(A.m2), coef_f32(inv1), coef_f32(A.hub3[1]), coef_f32(A.q1), coef_f32(A.q2)};
  const StageCoefL<float2> K1{coef_f32x2(A.m2), coef_f32x2(inv0), coef_f32x2(A.hub3[0]), coef_f32x2(A.q1),
                              coef_f32x2(A.q2)};
  const StageCoefL<float2> K2{coef_f32x2(A.m2), coef_f32x2(inv1), coef_f32x2(A.hub3[1]), coef_f32x2(A.q1),
                              coef_f32x2(A.q2)};
  const StageCoefL<float2> K4{coef_f32x2(A.m2), coef_f32x2(inv2), coef_f32x2(A.hub3[2]), coef_f32x2(A.q1),
                              coef_f32x2(A.q2)};
  const CoefL<float> CHs = coef_f32(A.dt2), CFs = coef_f32(A.dt);
  const C2 CH = coef_f32x2(A.dt2), CF = coef_f32x2(A.dt), C6 = coef_f32x2(A.dt6);
  const CoarseCols<V> cc = coarse_cols<EQ, V>(A.cmap, act, b, c);
  auto s6 = [&](int p) { return (p - a_begin + 4) % 6; };  // x planes >= a_begin - 4
  auto s5 = [&](int p) { return (p - a_begin + 2) % 5; };  // yb / yc planes >= a_begin - 2
  auto dslot = [&](int p) { return DL + ((p - a_begin + 2) % 3) * 3 * PD; };
  auto xf = [&](int p) { return XF + s6(p) * SM::P4; };
  auto xp = [&](int p) { return XP + s6(p) * SM::P4; };
  auto yb = [&](int p) { return YB + s5(p) * SM::P2; };
  auto yc = [&](int p) { return YC + s5(p) * SM::P2; };
  const int own4 = (ty + 4) * SP + O + tx * V;  // own sites in a 4-ring plane
  const int own2 = (ty + 2) * SP + O + tx * V;  // ... in a 2-ring plane
  const int od = ty * TW + tx * V;              // ... in a DL array

  // x_phi, x_pi of plane p (tile and 4-ring) into slot s6(p): rows of 16-byte chunks
  // -- the 4 left ring columns, the interior, the 4 right ring columns -- over all threads
  auto issue = [&](int p) {
    const long long poff = NN * wrap_n(p, N);
    float *df = xf(p), *dp = xp(p);
    const int nr = tye + 8, nch = twe / 4 + 2;
    for (int i = tid; i < 2 * nr * nch; i += NT) {
      const int f = i >= nr * nch;
      const int j = f ? i - nr * nch : i;
      const int row = j / nch, ch = j - row * nch;
      const long long grow = poff + (long long)N * wrap_n(b0 - 4 + row, N);
      int scol, gcol;
      if (ch == 0) {
        scol = 0;
        gcol = wrap_n(c0 - 4, N);
      } else if (ch == nch - 1) {
        scol = O + twe;
        gcol = wrap_n(c0 + twe, N);
      } else {
        scol = O + 4 * (ch - 1);
        gcol = c0 + 4 * (ch - 1);
      }
      cp_async_16((f ? dp : df) + row * SP + scol, (f ? A.xpi : A.xphi) + grow + gcol);
    }
    cp_async_commit();
  };

  // Stages 1-2 at the lane pair at offset o4 (4-ring plane) of plane q: yb_phi, yc_phi
  // and what phase 2 takes (yb_pi, acc_phi, acc_pi)
  auto phase1_pair = [&](int q, int o4, const Coupling<float, V> &ct, const Coupling<float, V> &ch2, float2 &vb,
                         float2 &vc, float2 &vbp, float2 &vap, float2 &vpp) {
    const Star13<float2> F = star13<SP>(xf(q), xf(q - 1), xf(q + 1), xf(q - 2), xf(q + 2), o4);
    const Star13<float2> P = star13<SP>(xp(q), xp(q - 1), xp(q + 1), xp(q - 2), xp(q + 2), o4);
    float2 c_ps, c_dps, c_ps4;
    coupling2<EQ>(ct, 0, c_ps, c_dps, c_ps4);
    const float2 k1 = kpi_f32<EQ, float2>(P.f0, F.f0, lap13_of(F), c_ps, c_dps, c_ps4, K1);
    const float2 yapi = c_fma(CH, k1, P.f0);
    const Star13<float2> YA = ya13(F, P, CH);
    coupling2<EQ>(ch2, 0, c_ps, c_dps, c_ps4);
    const float2 k2 = kpi_f32<EQ, float2>(yapi, YA.f0, lap13_of(YA), c_ps, c_dps, c_ps4, K2);
    vbp = c_fma(CH, k2, P.f0);
    vb = c_fma(CH, yapi, F.f0);
    vc = c_fma(CF, vbp, F.f0);
    vap = p_fma(p_splat<float2>(2.0f), yapi, P.f0);
    vpp = p_fma(p_splat<float2>(2.0f), k2, k1);
  };

  // Stages 1-2 at one ring-column site (relative row rr, smem column col) of plane q
  auto ring_site = [&](int q, int qm, long long qoff, int rr, int col) {
    const int o4 = (rr + 4) * SP + col;
    const int gb = wrap_n(b0 + rr, N), gc = wrap_n(c0 + col - O, N);
    const long long site = qoff + (long long)N * gb + gc;
    Coupling<float, 1> ct, ch2;
    if constexpr (EqOf<EQ>::coupled) {
      coupling_at<EQ, float>(ct, A.psi[0], A.dpsi[0], site, A.cmap, A.M, qm, gb, gc);
      if constexpr (EQ == EQ_FIXED)
        ch2 = ct;
      else
        coupling_at<EQ, float>(ch2, A.psi[1], A.dpsi[1], site, A.cmap, A.M, qm, gb, gc);
    }
    const Star13<float> F = star13s<SP>(xf(q), xf(q - 1), xf(q + 1), xf(q - 2), xf(q + 2), o4);
    const Star13<float> P = star13s<SP>(xp(q), xp(q - 1), xp(q + 1), xp(q - 2), xp(q + 2), o4);
    float ps = 0.0f, dps = 0.0f, ps4 = 0.0f;
    if constexpr (EqOf<EQ>::coupled) ps = ct.ps.v[0];
    if constexpr (EQ == EQ_COMOV || EQ == EQ_APPROX) dps = ct.dps.v[0];
    if constexpr (EQ == EQ_APPROX) ps4 = ct.ps4.v[0];
    const float k1 = kpi_f32<EQ, float>(P.f0, F.f0, lap13_of(F), ps, dps, ps4, K1s);
    const float yapi = c_fma(CHs, k1, P.f0);
    const Star13<float> YA = ya13(F, P, CHs);
    if constexpr (EqOf<EQ>::coupled) ps = ch2.ps.v[0];
    if constexpr (EQ == EQ_COMOV || EQ == EQ_APPROX) dps = ch2.dps.v[0];
    if constexpr (EQ == EQ_APPROX) ps4 = ch2.ps4.v[0];
    const float k2 = kpi_f32<EQ, float>(yapi, YA.f0, lap13_of(YA), ps, dps, ps4, K2s);
    const float bpi = c_fma(CHs, k2, P.f0);
    const int o2 = (rr + 2) * SP + col;
    yb(q)[o2] = c_fma(CHs, yapi, F.f0);
    yc(q)[o2] = c_fma(CFs, bpi, F.f0);
  };

  issue(a_begin - 4);
  for (int p = a_begin - 4; p <= a_end + 3; ++p) {
    cp_async_wait_all();  // this thread's copies of plane p have landed
    __syncthreads();      // everyone's; every read of the slots refilled below is done
    if (p + 1 <= a_end + 3) issue(p + 1);

    // ---- phase 1 on plane q = p - 2: the tile and its 2-ring
    const int q = p - 2;
    if (q >= a_begin - 2) {
      const int qm = wrap_n(q, N);
      const long long qoff = NN * qm;
      if (act) {  // own sites
        Coupling<float, V> ct, ch2;
        if constexpr (EqOf<EQ>::coupled) {
          const int ca = EqOf<EQ>::coarse ? __ldg(A.cmap + qm) : 0;
          load_coupling<EQ, float, V>(ct, A.psi[0], A.dpsi[0], qoff + rowoff, A.M, ca, cc);
          if constexpr (EQ == EQ_FIXED)
            ch2 = ct;
          else
            load_coupling<EQ, float, V>(ch2, A.psi[1], A.dpsi[1], qoff + rowoff, A.M, ca, cc);
        }
        float2 vb, vc, vbp, vap, vpp;
        phase1_pair(q, own4, ct, ch2, vb, vc, vbp, vap, vpp);
        st2s(yb(q) + own2, vb);
        st2s(yc(q) + own2, vc);
        float *dl = dslot(q);
        st2s(dl + od, vbp);
        st2s(dl + PD + od, vap);
        st2s(dl + 2 * PD + od, vpp);
      }
      if (ty >= TYv) {  // ring warps: two ring rows each, then the ring columns
        if (colact) {
#pragma unroll
          for (int k = 0; k < 2; ++k) {
            const int rr = ty == TYv ? k - 2 : tye + k;  // rows -2, -1 above, tye, tye + 1 below
            const int gb = wrap_n(b0 + rr, N);
            const long long site = qoff + (long long)N * gb + c;
            Coupling<float, V> ct, ch2;
            if constexpr (EqOf<EQ>::coupled) {
              CoarseCols<V> cr = cc;
              if constexpr (EqOf<EQ>::coarse) {
                cr.row_b = __ldg(A.cmap + gb);
#pragma unroll
                for (int v = 0; v < V; ++v) cr.col[v] = __ldg(A.cmap + c + v);
              }
              const int ca = EqOf<EQ>::coarse ? __ldg(A.cmap + qm) : 0;
              load_coupling<EQ, float, V>(ct, A.psi[0], A.dpsi[0], site, A.M, ca, cr);
              if constexpr (EQ == EQ_FIXED)
                ch2 = ct;
              else
                load_coupling<EQ, float, V>(ch2, A.psi[1], A.dpsi[1], site, A.M, ca, cr);
            }
            float2 vb, vc, vbp, vap, vpp;
            phase1_pair(q, (rr + 4) * SP + O + tx * V, ct, ch2, vb, vc, vbp, vap, vpp);
            st2s(yb(q) + (rr + 2) * SP + O + tx * V, vb);
            st2s(yc(q) + (rr + 2) * SP + O + tx * V, vc);
          }
        }
        // ring columns -2, -1, twe, twe + 1 of rows -2 .. tye + 1
        const int rt = tid - TYv * TXv;  // 0 .. 2 TXv - 1
        for (int i = rt; i < (tye + 4) * 4; i += 2 * TXv) {
          const int rr = i / 4 - 2, k = i & 3;
          const int col = k < 2 ? O - 2 + k : O + twe + (k - 2);
          ring_site(q, qm, qoff, rr, col);
        }
      }
    }

    // ---- phase 2 on plane r = p - 4 (own sites): stages 3 and 4, the update.  Planes
    // r +- 1, r +- 2 are read at own sites only (formed by this thread), plane r in full.
    const int r = p - 4;
    if (r >= a_begin && act) {
      const int rm = wrap_n(r, N);
      const long long roff = NN * rm;
      Coupling<float, V> cth, cd;
      if constexpr (EqOf<EQ>::coupled) {
        const int ca = EqOf<EQ>::coarse ? __ldg(A.cmap + rm) : 0;
        load_coupling<EQ, float, V>(cth, A.psi[1], A.dpsi[1], roff + rowoff, A.M, ca, cc);
        if constexpr (EQ == EQ_FIXED)
          cd = cth;
        else
          load_coupling<EQ, float, V>(cd, A.psi[2], A.dpsi[2], roff + rowoff, A.M, ca, cc);
      }
      const float *dl = dslot(r);
      const float2 xphi = ld2s(xf(r) + own4), xpi = ld2s(xp(r) + own4);
      const float2 ybpi = ld2s(dl + od), aphi = ld2s(dl + PD + od), api = ld2s(dl + 2 * PD + od);
      const float2 lp = *reinterpret_cast<const float2 *>(A.xlo + roff + rowoff);
      const float2 lq = *reinterpret_cast<const float2 *>(A.xlo + N3 + roff + rowoff);
      float2 c_ps, c_dps, c_ps4;
      const Star13<float2> Bs = star13<SP>(yb(r), yb(r - 1), yb(r + 1), yb(r - 2), yb(r + 2), own2);
      coupling2<EQ>(cth, 0, c_ps, c_dps, c_ps4);
      const float2 k3 = kpi_f32<EQ, float2>(ybpi, Bs.f0, lap13_of(Bs), c_ps, c_dps, c_ps4, K2);
      const float2 c1phi = p_fma(p_splat<float2>(2.0f), ybpi, aphi);
      const float2 c1pi = p_fma(p_splat<float2>(2.0f), k3, api);
      const float2 ycpi = c_fma(CF, k3, xpi);
      const Star13<float2> Cs = star13<SP>(yc(r), yc(r - 1), yc(r + 1), yc(r - 2), yc(r + 2), own2);
      coupling2<EQ>(cd, 0, c_ps, c_dps, c_ps4);
      const float2 k4 = kpi_f32<EQ, float2>(ycpi, Cs.f0, lap13_of(Cs), c_ps, c_dps, c_ps4, K4);
      float2 h1, l1, h2, l2;
      comp_update_f32<float2>(xphi, lp, p_add(c1phi, ycpi), C6, h1, l1);
      comp_update_f32<float2>(xpi, lq, p_add(c1pi, k4), C6, h2, l2);
      *reinterpret_cast<float2 *>(A.ophi + roff + rowoff) = h1;
      *reinterpret_cast<float2 *>(A.opi + roff + rowoff) = h2;
      *reinterpret_cast<float2 *>(A.xlo + roff + rowoff) = l1;
      *reinterpret_cast<float2 *>(A.xlo + N3 + roff + rowoff) = l2;
    }
  }
  cp_async_wait_all();
  __syncthreads();
}

}  // namespace cfb
