// cf_pair_tile.cuh -- two consecutive RK4 stages fused into one pass over a
// (b, c) tile, marching along a.
//
// In f(phi, pi) = (pi, F(phi, pi, lap phi)) only the pi component involves a
// spatial derivative, so a stage input y' = x + c k has y'_phi = x_phi + c k_phi
// = x_phi + c y_pi: a pointwise function of the previous stage's input.  The
// second stage's Laplacian can therefore be taken of y'_phi formed on the fly
// from the planes and the halo that the first stage streams anyway -- no wider
// halo, no recomputation, and the intermediate stage input never goes to HBM:
//
//   pass A (stages 1, 2):  u = x,   w = ya_phi = x_phi + dt/2 x_pi
//       reads x, Psi(t), Psi(t+dt/2); writes acc = k1 + 2 k2 and yb = x + dt/2 k2
//   pass B (stages 3, 4):  u = yb,  w = yc_phi = x_phi + dt yb_pi
//       reads yb, x, acc (+ x_lo), Psi(t+dt/2), Psi(t+dt); writes x (+ x_lo)
//
// Words per site-update: FP32_COMP 6 + 12 = 18 (+8 with Psi) against 38 (+8) for
// the four single-stage passes; FP64 6 + 8 = 14 (+8) against 32 (+8).  Every
// value is formed and rounded to the storage type exactly where the single-stage
// kernels (cf_stage_tile.cuh) form and round it, with the same lap_at / kpi_of
// expressions, so both routes produce bit-identical states.
//
// Pass B reads x_phi at the halo (for w) while it writes the new x_phi, so the
// new x_phi goes to a second plane buffer (the caller alternates the two);
// x_pi and x_lo are read and written only at a thread's own sites, in place.
//
// Tile layout as stage_tile: TXv x TYv threads, thread (tx, ty) owns V
// consecutive sites along c in row b0 + ty; u_phi and w of planes a-H..a+H of
// its own sites sit in two register queues, and the current plane of both, with
// an H-wide periodic halo in b and c, in shared memory.
#pragma once

#include "cf_stage_tile.cuh"

namespace cfb {

template <typename S>
struct PairArgs {
  const S *uphi;    // the first stage's input, phi and pi (N^3 each): pass A x, pass B yb
  const S *upi;
  const S *xphi;    // state phi (hi part in FP32_COMP), N^3
  S *xphi_out;      // pass B: the new phi (a buffer other than xphi)
  S *xpi;           // state pi (hi part), N^3; pass B updates it in place
  S *xlo;           // FP32_COMP compensation [phi | pi] (pass B, in place)
  S *acc;           // [phi | pi]: pass A writes k1 + 2 k2; pass B reads it
  S *yb;            // [phi | pi]: pass A output x + dt/2 k2
  const S *psi1;    // curvature (StageArgs::psi / dpsi) at the first stage's time
  const S *dpsi1;
  const S *psi2;    // ... at the second stage's time
  const S *dpsi2;
  const int *cmap;  // EQ_APPROX: coarse index of each lattice index (N entries)
  int M;            // EQ_APPROX: coarse grid size
  int N;
  int a_chunk;
  long long N3;
  double q1, q2;    // EQ_LAMBDA: lambda; EQ_SQRT: f_a^2, 1/f_a^2
  double m2;
  double inv1, hub3_1;  // first stage: h^-2 a^-2, 3H
  double inv2, hub3_2;  // second stage
  double cw;            // w = x_phi + cw u_pi   (pass A dt/2, pass B dt)
  double cy;            // pass A: yb = x + cy k2 (dt/2)
  double dt6;           // pass B: dt / 6
};

template <typename S, int H, int TXv, int TYv, int VW = VecT<S>::n>
struct PairSmem {
  using TS = TileSmem<S, H, TXv, TYv, VW>;
  static constexpr int plane = TS::plane;
  static constexpr int bufs = DoubleBuffered<S>::value ? 2 : 1;
  static constexpr int count = 2 * bufs * plane;  // u and w planes
};

template <typename S, typename T = typename Arith<S>::T>
__device__ __forceinline__ S w_of(S xphi, S upi, const Coef<T> &cw) {
  return (S)cw.fma((T)upi, (T)xphi);
}

template <typename S, int H, int EQ, int PASS, int TXv, int TYv, bool FULL = false, int VW = VecT<S>::n>
__device__ __forceinline__ void pair_tile(const PairArgs<S> &A, int c0, int b0, int a_begin, int a_end, S *smem) {
  using TS = TileSmem<S, H, TXv, TYv, VW>;
  using PS = PairSmem<S, H, TXv, TYv, VW>;
  constexpr bool DB = DoubleBuffered<S>::value;
  constexpr int V = TS::V;
  constexpr int TW = TS::TW;
  constexpr int SP = TS::SP;
  const int N = A.N;
  const long long N3 = A.N3;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * TXv + tx;
  const int twe = FULL ? TW : min(TW, N - c0);
  const int tye = FULL ? TYv : min(TYv, N - b0);
  const int sre = tye + 2 * H;
  const int c = c0 + tx * V;
  const int b = b0 + ty;
  const bool act = (tx * V) < twe && ty < tye;
  const long long rowoff = (long long)N * b + c;
  const long long NN = (long long)N * N;
  const S *uphi = A.uphi;
  const S *upi = A.upi;
  const S *xphi = A.xphi;  // w's base phi (pass A: the same array as uphi)
  using T = typename Arith<S>::T;
  // FP32: the 13-point sum comes times 12 (lap13_f32), its 1/12 rides on the coefficient
  const double inv1 = sizeof(T) == 4 ? lap_coef_f32<H>(A.inv1) : A.inv1;
  const double inv2 = sizeof(T) == 4 ? lap_coef_f32<H>(A.inv2) : A.inv2;
  const StageCoef<T> k1c{Coef<T>(A.m2), Coef<T>(inv1), Coef<T>(A.hub3_1), Coef<T>(A.q1), Coef<T>(A.q2)};
  const StageCoef<T> k2c{Coef<T>(A.m2), Coef<T>(inv2), Coef<T>(A.hub3_2), Coef<T>(A.q1), Coef<T>(A.q2)};
  const Coef<T> cw(A.cw), cy(A.cy), c6(A.dt6);
  const CoarseCols<V> cc = coarse_cols<EQ, V>(A.cmap, act, b, c);

  auto load_w = [&](long long off) -> Pack<S, V> {
    const Pack<S, V> p = ldv<S, V>(upi + off);
    const Pack<S, V> f = (PASS == 1) ? ldv<S, V>(uphi + off) : ldv<S, V>(xphi + off);
    Pack<S, V> w;
#pragma unroll
    for (int v = 0; v < V; ++v) w.v[v] = w_of(f.v[v], p.v[v], cw);
    return w;
  };

  Pack<S, V> qu[2 * H + 1], qw[2 * H + 1];
  if (act) {
#pragma unroll
    for (int j = 0; j < 2 * H; ++j) {
      const long long off = NN * wrap_n(a_begin - H + j, N) + rowoff;
      qu[j + 1] = ldv<S, V>(uphi + off);
      qw[j + 1] = load_w(off);
    }
  }

  for (int a = a_begin; a < a_end; ++a) {
    const long long site = NN * a + rowoff;
#pragma unroll
    for (int j = 0; j < 2 * H; ++j) {
      qu[j] = qu[j + 1];
      qw[j] = qw[j + 1];
    }
    Pack<S, V> p0v, xp, xq, cp, cq, lp{}, lq{};
    Coupling<S, V> cpl1, cpl2;
    if (act) {
      const long long head = NN * wrap_n(a + H, N) + rowoff;
      qu[2 * H] = ldv<S, V>(uphi + head);
      qw[2 * H] = load_w(head);
      p0v = ldv<S, V>(upi + site);
      if constexpr (PASS == 2) {
        xp = ldv<S, V>(xphi + site);
        xq = ldv_rw<S, V>(A.xpi + site);
        cp = ldv<S, V>(A.acc + site);
        cq = ldv<S, V>(A.acc + N3 + site);
        if constexpr (sizeof(S) == 4) {
          lp = ldv_rw<S, V>(A.xlo + site);
          lq = ldv_rw<S, V>(A.xlo + N3 + site);
        }
      }
      if constexpr (EqOf<EQ>::coupled) {
        const int ca = EqOf<EQ>::coarse ? __ldg(A.cmap + a) : 0;
        load_coupling<EQ, S, V>(cpl1, A.psi1, A.dpsi1, site, A.M, ca, cc);
        if constexpr (EQ == EQ_FIXED)
          cpl2 = cpl1;  // a time-independent Psi: both stages read the same plane
        else
          load_coupling<EQ, S, V>(cpl2, A.psi2, A.dpsi2, site, A.M, ca, cc);
      }
    }
    S *smu = smem;
    if constexpr (DB) {
      smu = smem + ((a - a_begin) & 1) * 2 * PS::plane;
    } else {
      __syncthreads();  // the previous plane's shared-memory reads are complete
    }
    S *smw = smu + PS::plane;
    if (act) {
#pragma unroll
      for (int v = 0; v < V; ++v) {
        smu[(ty + H) * SP + H + tx * V + v] = qu[H].v[v];
        smw[(ty + H) * SP + H + tx * V + v] = qw[H].v[v];
      }
      // halo rows: H above the tile and H below its active height, interior columns
#pragma unroll
      for (int pass = 0; pass < 2; ++pass) {
        // pass 0: the top band (ty < H) or the bottom band (ty >= tye - H);
        // pass 1: the bottom row of a thread in both bands (tye < 2H)
        int r = -1;
        if (pass == 0 && (ty < H || ty >= tye - H)) r = (ty < H) ? ty : ty + 2 * H;
        if (pass == 1 && ty < H && ty >= tye - H) r = ty + 2 * H;
        if (r >= 0) {
          const int gb = wrap_n(b0 - H + r, N);
          const long long off = NN * a + (long long)N * gb + c;
          const Pack<S, V> hu = ldv<S, V>(uphi + off);
          const Pack<S, V> hw = load_w(off);
#pragma unroll
          for (int v = 0; v < V; ++v) {
            smu[r * SP + H + tx * V + v] = hu.v[v];
            smw[r * SP + H + tx * V + v] = hw.v[v];
          }
        }
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
      const long long off = NN * a + (long long)N * gb + gc;
      smu[r * SP + col] = uphi[off];
      smw[r * SP + col] = w_of((PASS == 1) ? uphi[off] : xphi[off], upi[off], cw);
    }
    __syncthreads();
    if (!act) continue;

    Pack<S, V> o1, o2, o3, o4;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const int col = H + tx * V + v;
      const int row = ty + H;
      // first stage: input u
      const T f0 = (T)qu[H].v[v];
      const T p0 = (T)p0v.v[v];
      const T lap1 = lap_at<S, H, SP>(qu, smu, row, col, v);
      const T k1pi = kpi_of<EQ, S, V>(p0, f0, lap1, cpl1, v, k1c);
      // the second stage's input: w (phi, already formed) and its pi
      const S wphi = qw[H].v[v];
      S c1phi, c1pi, wpi;
      if constexpr (PASS == 1) {
        c1phi = (S)p0;  // acc = k1 (k1_phi = pi)
        c1pi = (S)k1pi;
        wpi = (S)cw.fma(k1pi, p0);  // ya_pi = x_pi + dt/2 k1_pi
      } else {
        c1phi = (S)((T)cp.v[v] + (T)2 * p0);  // acc += 2 k3
        c1pi = (S)((T)cq.v[v] + (T)2 * k1pi);
        wpi = (S)cw.fma(k1pi, (T)xq.v[v]);  // yc_pi = x_pi + dt k3_pi
      }
      // second stage: input (wphi, wpi)
      const T f1 = (T)wphi;
      const T p1 = (T)wpi;
      const T lap2 = lap_at<S, H, SP>(qw, smw, row, col, v);
      const T k2pi = kpi_of<EQ, S, V>(p1, f1, lap2, cpl2, v, k2c);
      if constexpr (PASS == 1) {
        o1.v[v] = (S)((T)c1phi + (T)2 * p1);  // acc += 2 k2
        o2.v[v] = (S)((T)c1pi + (T)2 * k2pi);
        o3.v[v] = (S)cy.fma(p1, f0);  // yb = x + dt/2 k2  (x = u in pass A)
        o4.v[v] = (S)cy.fma(k2pi, p0);
      } else {
        // x += dt/6 (acc + k4)
        state_update(xp.v[v], lp.v[v], (T)c1phi + p1, c6, o1.v[v], o3.v[v]);
        state_update(xq.v[v], lq.v[v], (T)c1pi + k2pi, c6, o2.v[v], o4.v[v]);
      }
    }
    if constexpr (PASS == 1) {
      stv(A.acc + site, o1);
      stv(A.acc + N3 + site, o2);
      stv(A.yb + site, o3);
      stv(A.yb + N3 + site, o4);
    } else {
      stv(A.xphi_out + site, o1);
      stv(A.xpi + site, o2);
      if constexpr (sizeof(S) == 4) {
        stv(A.xlo + site, o3);
        stv(A.xlo + N3 + site, o4);
      }
    }
  }
  // the caller may stage another tile into the same buffers next (ensemble work lists)
  __syncthreads();
}

}  // namespace cfb
