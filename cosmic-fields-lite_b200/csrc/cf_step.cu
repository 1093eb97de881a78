// cf_step.cu -- fused RK4 stage kernels (the hot path), cf_rhs, cf_scale_sum.
//
// One RK4 step (stepper/runge_kutta4_classic.hpp:88-138) is four stage kernels.
// Each makes ONE pass over HBM: it streams its stage input y through a
// 2.5-D blocked stencil and fuses the odeint linear combinations
// (thrust_operations::scale_sum2 / scale_sum5) into the same pass:
//
//   stage 1 (t)       k1 = f(x)      acc  = k1        y' = x + dt/2 k1
//   stage 2 (t+dt/2)  k2 = f(y)      acc += 2 k2      y' = x + dt/2 k2
//   stage 3 (t+dt/2)  k3 = f(y)      acc += 2 k3      y' = x + dt   k3
//   stage 4 (t+dt)    k4 = f(y)      x   += dt/6 (acc + k4)
//
// with f the Klein-Gordon right-hand side (src/equations_cuda.cu:15-36 for flat
// and FRW, :263-287 for the comoving-curvature coupling):
//   f(phi, pi) = (pi,  (-3H + 4 dPsi) pi - e^{2Psi} m^2 phi + e^{4Psi} a^-2 h^-2 lap phi)
// (Psi = dPsi = 0 for the uncoupled equations).
//
// Blocking: a CTA owns a (b, c) tile of TY rows x TX*V columns and marches along
// the slowest axis a over a chunk of planes.  phi of planes a-H..a+H of the
// thread's own V sites live in a register queue (H = 1 for the 7-point, 2 for
// the 13-point Laplacian); the current plane, with an H-wide periodic halo in b
// and c, is staged in shared memory for the in-plane neighbours.  Every global
// access of the tile interior is a 16-byte vector (double2 / float4) along c.
//
// Storage: S = double (CF_FP64) or float (CF_FP32_COMP).  Arithmetic is FP64 in
// both; in FP32_COMP the state x is an FP32 hi + FP32 lo pair that stage 4 updates
// as a compensated sum, while acc and the stage inputs y are single FP32 words.

#include <cuda_runtime.h>

#include <cmath>

#include "cf_internal.cuh"

namespace cfb {

template <typename S>
struct VecT;
template <>
struct VecT<double> {
  using T = double2;
  static constexpr int n = 2;
};
template <>
struct VecT<float> {
  using T = float4;
  static constexpr int n = 4;
};

template <typename S>
struct Pack {
  S v[VecT<S>::n];
};

template <typename S>
__device__ __forceinline__ Pack<S> ldv(const S *p) {
  Pack<S> r;
  typename VecT<S>::T t = __ldg(reinterpret_cast<const typename VecT<S>::T *>(p));
  if constexpr (VecT<S>::n == 2) {
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

// Plain (non-__ldg) load for buffers the same kernel also writes (acc, x).
template <typename S>
__device__ __forceinline__ Pack<S> ldv_rw(const S *p) {
  Pack<S> r;
  typename VecT<S>::T t = *reinterpret_cast<const typename VecT<S>::T *>(p);
  if constexpr (VecT<S>::n == 2) {
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

template <typename S>
__device__ __forceinline__ void stv(S *p, const Pack<S> &r) {
  typename VecT<S>::T t;
  if constexpr (VecT<S>::n == 2) {
    t.x = r.v[0];
    t.y = r.v[1];
  } else {
    t.x = r.v[0];
    t.y = r.v[1];
    t.z = r.v[2];
    t.w = r.v[3];
  }
  *reinterpret_cast<typename VecT<S>::T *>(p) = t;
}

constexpr int TX = 32;  // threads along c (each owns V consecutive sites)
constexpr int TY = 8;   // threads along b

template <typename S>
struct StageArgs {
  const S *yin;  // stage input [phi | pi]; for stage 1 (and 0) the state x (hi part)
  S *yout;       // stage output [phi | pi] (stages 1-3); dxdt for stage 0
  S *acc;        // k accumulator [phi | pi]
  S *x;          // base state [phi | pi] (hi part in FP32_COMP)
  S *xlo;        // FP32_COMP compensation [phi | pi] (stage 4 only)
  const S *psi;  // comoving: Psi(t_stage), N^3
  const S *dpsi; // comoving: dPsi/dt(t_stage), N^3
  int N;
  int a_chunk;
  long long N3;
  double m2;    // m^2
  double inv;   // h^-2 a^-2
  double hub3;  // 3 H
  double cy;    // y' = x + cy * k
  double dt6;   // dt / 6
};

// exp(2 Psi) and exp(4 Psi).  FP64: the reference's exp of the doubled argument.
// FP32: Psi is an FP32 field of magnitude ~1e-2; 1 + expm1f keeps the absolute
// error of e^{2Psi} near 1e-9 (FP32 relative accuracy on the small part).
__device__ __forceinline__ void psi_factors(double psi, double &e2, double &e4) {
  e2 = exp(2 * psi);
  e4 = exp(4 * psi);
}
__device__ __forceinline__ void psi_factors(float psi, double &e2, double &e4) {
  e2 = 1.0 + (double)expm1f(2.0f * psi);
  e4 = 1.0 + (double)expm1f(4.0f * psi);
}

template <typename S, int H, bool COMOV, int STAGE>
__global__ void __launch_bounds__(TX *TY) k_stage(const StageArgs<S> A) {
  constexpr int V = VecT<S>::n;
  constexpr int TW = TX * V;
  constexpr int SP = TW + 2 * H;  // shared-memory row pitch
  constexpr int SR = TY + 2 * H;  // shared-memory rows
  __shared__ S sm[SR * SP];

  const int N = A.N;
  const long long N3 = A.N3;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * TX + tx;
  const int c0 = blockIdx.x * TW;
  const int b0 = blockIdx.y * TY;
  const int twe = min(TW, N - c0);  // active tile width (N % 8 == 0, so a multiple of V)
  const int a_begin = blockIdx.z * A.a_chunk;
  const int a_end = min(a_begin + A.a_chunk, N);
  const int c = c0 + tx * V;
  const int b = b0 + ty;  // N % TY == 0: always < N
  const bool act = (tx * V) < twe;
  const long long rowoff = (long long)N * b + c;  // offset within a plane
  const long long NN = (long long)N * N;

  const S *phi_in = A.yin;
  const S *pi_in = A.yin + N3;

  // register queue of phi over planes a-H..a+H for this thread's V sites
  Pack<S> q[2 * H + 1];
  if (act) {
#pragma unroll
    for (int j = 0; j < 2 * H; ++j) {
      int ap = (a_begin - H + j + N) % N;
      q[j + 1] = ldv(phi_in + NN * ap + rowoff);
    }
  }

  for (int a = a_begin; a < a_end; ++a) {
    const long long site = NN * a + rowoff;
#pragma unroll
    for (int j = 0; j < 2 * H; ++j) q[j] = q[j + 1];
    Pack<S> pi0, xp, xq, cp, cq, lp, lq, ps, dps;
    if (act) {
      q[2 * H] = ldv(phi_in + NN * ((a + H) % N) + rowoff);
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
      if constexpr (COMOV) {
        ps = ldv(A.psi + site);
        dps = ldv(A.dpsi + site);
      }
    }
    __syncthreads();  // previous plane's shared-memory reads are complete
    if (act) {
#pragma unroll
      for (int v = 0; v < V; ++v) sm[(ty + H) * SP + H + tx * V + v] = q[H].v[v];
    }
    // halo rows (H above, H below the tile), interior columns
    if (ty < H || ty >= TY - H) {
      if (act) {
        int r = (ty < H) ? ty : ty + 2 * H;  // shared-memory row
        int gb = (b0 - H + r + N) % N;
        Pack<S> h = ldv(phi_in + NN * a + (long long)N * gb + c);
#pragma unroll
        for (int v = 0; v < V; ++v) sm[r * SP + H + tx * V + v] = h.v[v];
      }
    }
    // halo columns (H left, H right of the active width), all rows
    for (int i = tid; i < SR * 2 * H; i += TX * TY) {
      int r = i / (2 * H);
      int j = i % (2 * H);
      int gb = (b0 - H + r + N) % N;
      int col, gc;
      if (j < H) {
        col = j;
        gc = (c0 - H + j + N) % N;
      } else {
        col = twe + H + (j - H);
        gc = (c0 + twe + (j - H)) % N;
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
      const double f0 = (double)q[H].v[v];
      double lap;
      if constexpr (H == 1) {
        double s = -6.0 * f0 + (double)q[2].v[v] + (double)q[0].v[v] + (double)sm[(row + 1) * SP + col] +
                   (double)sm[(row - 1) * SP + col];
        lap = s + ((double)sm[row * SP + col + 1] + (double)sm[row * SP + col - 1]);
      } else {
        double s1 = (double)q[3].v[v] + (double)q[1].v[v] + (double)sm[(row + 1) * SP + col] +
                    (double)sm[(row - 1) * SP + col] + (double)sm[row * SP + col + 1] +
                    (double)sm[row * SP + col - 1];
        double s2 = (double)q[4].v[v] + (double)q[0].v[v] + (double)sm[(row + 2) * SP + col] +
                    (double)sm[(row - 2) * SP + col] + (double)sm[row * SP + col + 2] +
                    (double)sm[row * SP + col - 2];
        lap = (16.0 * s1 - s2 - 90.0 * f0) / 12.0;
      }
      const double p0 = (double)pi0.v[v];
      double kphi = p0, kpi;
      if constexpr (COMOV) {
        double e2, e4;
        psi_factors(ps.v[v], e2, e4);
        kpi = (-A.hub3 + 4.0 * (double)dps.v[v]) * p0 - e2 * A.m2 * f0 + e4 * A.inv * lap;
      } else {
        kpi = -A.hub3 * p0 - A.m2 * f0 + A.inv * lap;
      }
      if constexpr (STAGE == 0) {
        o_phi.v[v] = (S)kphi;
        o_pi.v[v] = (S)kpi;
      } else if constexpr (STAGE == 1) {
        cp.v[v] = (S)kphi;
        cq.v[v] = (S)kpi;
        o_phi.v[v] = (S)(f0 + A.cy * kphi);
        o_pi.v[v] = (S)(p0 + A.cy * kpi);
      } else if constexpr (STAGE == 2 || STAGE == 3) {
        cp.v[v] = (S)((double)cp.v[v] + 2.0 * kphi);
        cq.v[v] = (S)((double)cq.v[v] + 2.0 * kpi);
        o_phi.v[v] = (S)((double)xp.v[v] + A.cy * kphi);
        o_pi.v[v] = (S)((double)xq.v[v] + A.cy * kpi);
      } else {  // STAGE 4
        const double ip = A.dt6 * ((double)cp.v[v] + kphi);
        const double iq = A.dt6 * ((double)cq.v[v] + kpi);
        if constexpr (sizeof(S) == 8) {
          xp.v[v] = (S)((double)xp.v[v] + ip);
          xq.v[v] = (S)((double)xq.v[v] + iq);
        } else {
          const double np = ((double)xp.v[v] + (double)lp.v[v]) + ip;
          const double nq = ((double)xq.v[v] + (double)lq.v[v]) + iq;
          const float hp = (float)np, hq = (float)nq;
          xp.v[v] = hp;
          xq.v[v] = hq;
          lp.v[v] = (float)(np - (double)hp);
          lq.v[v] = (float)(nq - (double)hq);
        }
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
}

// Planes per CTA along a: enough CTAs to fill the GPU several times over.
static int pick_a_chunk(int N, int tiles_xy) {
  int chunk = 32;
  while (chunk > 4 && (long long)tiles_xy * ((N + chunk - 1) / chunk) < 148LL * 8) chunk /= 2;
  return chunk;
}

template <typename S, int H, bool COMOV, int STAGE>
static int launch_stage_t(cf_ctx *ctx, const StageArgs<S> &A0, cudaStream_t st) {
  constexpr int TW = TX * VecT<S>::n;
  StageArgs<S> A = A0;
  dim3 block(TX, TY);
  unsigned gx = ceil_div(A.N, TW), gy = (unsigned)(A.N / TY);
  A.a_chunk = pick_a_chunk(A.N, (int)(gx * gy));
  dim3 grid(gx, gy, ceil_div(A.N, A.a_chunk));
  ProfScope ps(ctx, STAGE == 0 ? CF_PROF_OTHER : STAGE - 1, st);
  k_stage<S, H, COMOV, STAGE><<<grid, block, 0, st>>>(A);
  CF_LAUNCHED(ctx);
  return CF_OK;
}

template <typename S, bool COMOV, int STAGE>
static int launch_stage_h(cf_ctx *ctx, int stencil, const StageArgs<S> &A, cudaStream_t st) {
  if (stencil == 13) return launch_stage_t<S, 2, COMOV, STAGE>(ctx, A, st);
  return launch_stage_t<S, 1, COMOV, STAGE>(ctx, A, st);
}

template <typename S, int STAGE>
static int launch_stage(cf_ctx *ctx, const StageArgs<S> &A, cudaStream_t st) {
  if (ctx->p.equation == CF_EQ_COMOVING_FRW) return launch_stage_h<S, true, STAGE>(ctx, ctx->p.stencil, A, st);
  return launch_stage_h<S, false, STAGE>(ctx, ctx->p.stencil, A, st);
}

template <typename S>
static int fill_stage_coeffs(cf_ctx *ctx, StageArgs<S> &A, double t, cudaStream_t st) {
  double inv, H;
  stage_coeffs(ctx->p, t, &inv, &H);
  A.inv = inv;
  A.hub3 = 3.0 * H;
  A.psi = A.dpsi = nullptr;
  if (ctx->p.equation == CF_EQ_COMOVING_FRW) {
    const void *ps, *dps;
    CF_TRY(psi_at(ctx, t, st, &ps, &dps));
    A.psi = (const S *)ps;
    A.dpsi = (const S *)dps;
  }
  return CF_OK;
}

template <typename S>
static int rk4_steps_t(cf_ctx *ctx, void *d_state, double t0, double dt, int64_t step0, int64_t nsteps,
                       cudaStream_t st) {
  CF_TRY(ensure_rk4_scratch(ctx));
  const long long N3 = ctx->N3;
  S *x = (S *)d_state;
  S *xlo = (sizeof(S) == 4) ? x + 2 * N3 : nullptr;
  S *ya = (S *)ctx->ya, *yb = (S *)ctx->yb, *acc = (S *)ctx->acc;
  StageArgs<S> A{};
  A.N = (int)ctx->N;
  A.N3 = N3;
  A.m2 = ctx->p.m * ctx->p.m;
  A.x = x;
  A.xlo = xlo;
  A.acc = acc;
  const double dh = dt / 2.0;
  const double dt6 = dt / 6.0;
  A.dt6 = dt6;
  for (int64_t j = 0; j < nsteps; ++j) {
    const double t = t0 + (double)(step0 + j) * dt;
    const double th = t + dh;
    // stage 1 at t: y_a = x + dt/2 k1
    CF_TRY(fill_stage_coeffs(ctx, A, t, st));
    A.yin = x;
    A.yout = ya;
    A.cy = dh;
    CF_TRY(launch_stage<S, 1>(ctx, A, st));
    // stage 2 at t + dt/2: y_b = x + dt/2 k2
    CF_TRY(fill_stage_coeffs(ctx, A, th, st));
    A.yin = ya;
    A.yout = yb;
    A.cy = dh;
    CF_TRY(launch_stage<S, 2>(ctx, A, st));
    // stage 3 at t + dt/2: y_a = x + dt k3
    A.yin = yb;
    A.yout = ya;
    A.cy = dt;
    CF_TRY(launch_stage<S, 3>(ctx, A, st));
    // stage 4 at t + dt: x += dt/6 (k1 + 2k2 + 2k3 + k4)
    CF_TRY(fill_stage_coeffs(ctx, A, t + dt, st));
    A.yin = ya;
    A.yout = nullptr;
    CF_TRY(launch_stage<S, 4>(ctx, A, st));
  }
  return CF_OK;
}

// One forward stage (1..3) with explicit buffers: the adjoint's recompute of
// the stage inputs y2, y3, y4 of a step (same kernels as rk4_steps, so the
// recomputed values are bit-identical to the forward sweep).
template <typename S>
static int forward_stage_t(cf_ctx *ctx, int stage, const void *yin, void *yout, void *x, void *xlo, double t,
                           double cy, double dt6, cudaStream_t st) {
  CF_TRY(ensure_rk4_scratch(ctx));
  StageArgs<S> A{};
  A.N = (int)ctx->N;
  A.N3 = ctx->N3;
  A.m2 = ctx->p.m * ctx->p.m;
  A.x = (S *)x;
  A.xlo = (S *)xlo;
  A.acc = (S *)ctx->acc;
  A.dt6 = dt6;
  CF_TRY(fill_stage_coeffs(ctx, A, t, st));
  A.yin = (const S *)yin;
  A.yout = (S *)yout;
  A.cy = cy;
  if (stage == 1) return launch_stage<S, 1>(ctx, A, st);
  if (stage == 2) return launch_stage<S, 2>(ctx, A, st);
  if (stage == 3) return launch_stage<S, 3>(ctx, A, st);
  return launch_stage<S, 4>(ctx, A, st);
}

int launch_forward_stage(cf_ctx *ctx, int stage, const void *yin, void *yout, void *x, void *xlo, double t, double cy,
                         double dt6, cudaStream_t st) {
  if (ctx->p.precision == CF_FP32_COMP) return forward_stage_t<float>(ctx, stage, yin, yout, x, xlo, t, cy, dt6, st);
  return forward_stage_t<double>(ctx, stage, yin, yout, x, xlo, t, cy, dt6, st);
}

int rk4_steps(cf_ctx *ctx, void *d_state, double t0, double dt, int64_t step0, int64_t nsteps, cudaStream_t st) {
  if (ctx->p.precision == CF_FP32_COMP) return rk4_steps_t<float>(ctx, d_state, t0, dt, step0, nsteps, st);
  return rk4_steps_t<double>(ctx, d_state, t0, dt, step0, nsteps, st);
}

int rhs(cf_ctx *ctx, const double *d_x, double *d_dxdt, double t, cudaStream_t st) {
  StageArgs<double> A{};
  A.N = (int)ctx->N;
  A.N3 = ctx->N3;
  A.m2 = ctx->p.m * ctx->p.m;
  CF_TRY(fill_stage_coeffs(ctx, A, t, st));
  A.yin = d_x;
  A.yout = d_dxdt;
  return launch_stage<double, 0>(ctx, A, st);
}

// ---- scale_sum: out = sum alpha_i in_i ------------------------------------
struct ScaleSumArgs {
  const double *in[14];
  double alpha[14];
  double *out;
  long long len;
  int n;
};

__global__ void k_scale_sum(const ScaleSumArgs A) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < A.len; i += stride) {
    double s = A.alpha[0] * A.in[0][i];
    for (int k = 1; k < A.n; ++k) s += A.alpha[k] * A.in[k][i];
    A.out[i] = s;
  }
}

int scale_sum(cf_ctx *ctx, double *out, int n, const double *const *in, const double *alpha, int64_t len,
              cudaStream_t st) {
  ScaleSumArgs A{};
  for (int k = 0; k < n; ++k) {
    A.in[k] = in[k];
    A.alpha[k] = alpha[k];
  }
  A.out = out;
  A.len = len;
  A.n = n;
  unsigned blocks = (unsigned)std::min<int64_t>((len + 255) / 256, 148LL * 16);
  if (blocks == 0) blocks = 1;
  ProfScope ps(ctx, CF_PROF_OTHER, st);
  k_scale_sum<<<blocks, 256, 0, st>>>(A);
  CF_LAUNCHED(ctx);
  return CF_OK;
}

}  // namespace cfb
