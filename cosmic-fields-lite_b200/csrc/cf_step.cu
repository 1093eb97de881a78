// cf_step.cu -- fused RK4 stage kernels (the hot path), cf_rhs, cf_scale_sum.
//
// One RK4 step (stepper/runge_kutta4_classic.hpp:88-138) is four stages.  By
// default cf_rk4_steps runs a step as one whole-step pass -- k_step
// (cf_step_tile.cuh) for the 7-point stencil, k_step13 (cf_step13_tile.cuh) for the
// 13-point one in FP32 -- and an FP64 13-point step as two paired-stage passes
// (stages 1+2, 3+4; cf_pair_tile.cuh); all keep the intermediate stage inputs out of
// HBM and give the same bits.  The four single-stage kernels remain for
// CF_FLAG_STAGE_KERNELS, the adjoint's recompute, cf_rk4_steps_noalloc and the
// 13-point persistent ensemble kernel.  A single-stage kernel makes ONE pass over HBM:
// it streams its stage input y through a 2.5-D blocked stencil and fuses the
// odeint linear combinations (thrust_operations::scale_sum2 / scale_sum5) into
// the same pass:
//
//   stage 1 (t)       k1 = f(x)      acc  = k1        y' = x + dt/2 k1
//   stage 2 (t+dt/2)  k2 = f(y)      acc += 2 k2      y' = x + dt/2 k2
//   stage 3 (t+dt/2)  k3 = f(y)      acc += 2 k3      y' = x + dt   k3
//   stage 4 (t+dt)    k4 = f(y)      x   += dt/6 (acc + k4)
//
// with f the Klein-Gordon right-hand side of the context's equation
// (src/equations_cuda.cu:15-36 flat and FRW, :38-76 lambda phi^4, :84-104 sqrt
// potential, :112-136 fixed curvature, :263-287 comoving curvature, :299-329
// approximate comoving curvature; the EqShape of cf_stage_tile.cuh).  The tile code is in
// cf_stage_tile.cuh: a CTA of 32 x 8 threads owns a (b, c) tile of 8 rows x 64
// (FP64) or 128 (FP32) columns and marches along a over a chunk of planes.
//
// Storage: S = double (CF_FP64) or float (CF_FP32_COMP).  FP64 storage steps in
// FP64.  In FP32_COMP the state x is an FP32 hi + FP32 lo pair that stage 4 updates
// error-free, acc and the stage inputs y are single FP32 words, and the stage
// arithmetic is FP32 with hi + lo coefficients (cf_f32x2.cuh).

#include <cuda_runtime.h>

#include <cmath>

#include "cf_internal.cuh"
#include "cf_pair_tile.cuh"
#include "cf_stage_tile.cuh"
#include "cf_step13_tile.cuh"
#include "cf_step_tile.cuh"

namespace cfb {

constexpr int TX = 32;  // threads along c (each owns V consecutive sites)
constexpr int TY = 8;   // threads along b

// Resident CTAs per SM the register allocation must allow (occupancy floor),
// from measurements at N = 512: 4 for FP32 (double-buffered planes) and for the
// uncoupled FP64 stages; the compiler's choice for the FP64 comoving stages,
// whose Psi terms would spill at 64 registers.
template <typename S, int EQ>
struct StageMinBlocks {
  static constexpr int value = (sizeof(S) == 4 || !EqOf<EQ>::coupled) ? 4 : 1;
};

template <typename S, int H, int EQ, int STAGE, bool FULL>
__global__ void __launch_bounds__(TX *TY, (StageMinBlocks<S, EQ>::value)) k_stage(const StageArgs<S> A) {
  using TS = TileSmem<S, H, TX, TY>;
  __shared__ __align__(16) S sm[TS::count];
  const int a_begin = blockIdx.z * A.a_chunk;
  stage_tile<S, H, EQ, STAGE, TX, TY, FULL>(A, blockIdx.x * TS::TW, blockIdx.y * TY, a_begin,
                                            min(a_begin + A.a_chunk, A.N), sm);
}

// Paired-stage kernels: the same tile, two stages per pass.  Occupancy floors
// per storage type (FP32 7-point, FP32 13-point; FP64 uncoupled; FP64 comoving),
// measured at N = 512 (ms per step: FP32 comoving 7-point, floors 2 / 3 / 4 ->
// 4.80 / 4.29 / 4.52; 13-point 5.16 / 5.76 / 6.89; FP64 FRW 7-point 4.60 / 3.64 /
// 3.23, 13-point 5.27 / 4.83 / 5.60; FP64 comoving 7-point, floors 1 / 2 -> 9.49
// / 5.97).
#ifndef CF_PAIR_MB_F32
#define CF_PAIR_MB_F32 3
#endif
// pass A of the uncoupled equations fits 64 registers without spills: 4 CTAs/SM
// (FP32 KG-FRW 7-point pass A: floors 3 / 4 -> 0.93 / 0.80 ms; comoving pass A 1.06 /
// 1.12 ms, pass B 1.71 / 2.05 ms)
#ifndef CF_PAIR_MB_F32_A
#define CF_PAIR_MB_F32_A 4
#endif
#ifndef CF_PAIR_MB_F32_H2
#define CF_PAIR_MB_F32_H2 2
#endif
#ifndef CF_PAIR_MB_F64
#define CF_PAIR_MB_F64 4
#endif
#ifndef CF_PAIR_MB_F64_H2
#define CF_PAIR_MB_F64_H2 3
#endif
#ifndef CF_PAIR_MB_F64_COMOV
#define CF_PAIR_MB_F64_COMOV 2
#endif
// Sites per thread of a paired pass: 16-byte vectors, except the FP32 comoving
// 7-point pass B, the pass with the most live values, which takes 2 floats per
// thread and 4 CTAs/SM without spills (N = 512: 1.71 -> 1.52 ms per step; the
// other FP32 passes measured slower with 2 floats per thread).
// (the FP32 fixed-Psi pass B, with one plane fewer, measured 1.32 ms with 16-byte
// vectors against 1.35 ms with 2 floats; the approximate comoving pass B 1.83 against 1.43)
template <typename S, int H, int EQ, int PASS>
struct PairVec {
  static constexpr int value =
      (sizeof(S) == 4 && EqOf<EQ>::coupled && EQ != EQ_FIXED && H == 1 && PASS == 2) ? 2 : VecT<S>::n;
};
#ifndef CF_PAIR_MB_F32_V2
#define CF_PAIR_MB_F32_V2 4
#endif

// Floors of the other equation shapes (7-point), measured at N = 512 (ms per pass
// A / B): sqrt potential FP64 floors 4/3 -> 1.54 / 1.80, 3/2 -> 1.76 / 2.27; FP32
// 4/3 -> 0.82 / 1.27, 4/4 -> 0.82 / 1.50; FP64 fixed Psi 2 -> 2.31 / 2.31, 3 ->
// 1.78 / 1.89, 4 -> 1.65 / 1.77; FP64 approximate comoving 2 -> 2.37 / 2.26, 3 ->
// 1.95 / 2.21, 4 -> 1.91 / 2.60; FP32 fixed Psi pass A 2 / 3 / 4 -> 1.21 / 0.99 /
// 0.85, FP32 approximate comoving pass A 1.34 / 1.07 / 1.22 (pass B: the FP32
// comoving floors).
#ifndef CF_PAIR_MB_SQRT_A
#define CF_PAIR_MB_SQRT_A 4
#endif
#ifndef CF_PAIR_MB_SQRT_B
#define CF_PAIR_MB_SQRT_B 3
#endif
#ifndef CF_PAIR_MB_F64_FIXED
#define CF_PAIR_MB_F64_FIXED 4
#endif
#ifndef CF_PAIR_MB_F64_APPROX_A
#define CF_PAIR_MB_F64_APPROX_A 4
#endif
#ifndef CF_PAIR_MB_F64_APPROX_B
#define CF_PAIR_MB_F64_APPROX_B 3
#endif
#ifndef CF_PAIR_MB_F32_FIXED_A
#define CF_PAIR_MB_F32_FIXED_A 4
#endif
#ifndef CF_PAIR_MB_F32_APPROX_A
#define CF_PAIR_MB_F32_APPROX_A 3
#endif
template <typename S, int H, int EQ, int PASS>
struct PairMinBlocks {
  static constexpr bool cpl = EqOf<EQ>::coupled;
  static constexpr bool fx = EQ == EQ_FIXED || EQ == EQ_APPROX;
  static constexpr int other =
      EQ == EQ_SQRT    ? (PASS == 1 ? CF_PAIR_MB_SQRT_A : CF_PAIR_MB_SQRT_B)
      : sizeof(S) == 4 ? (EQ == EQ_FIXED ? CF_PAIR_MB_F32_FIXED_A : CF_PAIR_MB_F32_APPROX_A)
      : EQ == EQ_FIXED ? CF_PAIR_MB_F64_FIXED
                       : (PASS == 1 ? CF_PAIR_MB_F64_APPROX_A : CF_PAIR_MB_F64_APPROX_B);
  static constexpr int value =
      (H == 1 && (EQ == EQ_SQRT || (fx && (sizeof(S) == 8 || PASS == 1)))) ? other :
      sizeof(S) == 4
          ? (H == 1 ? (PairVec<S, H, EQ, PASS>::value == 2
                           ? CF_PAIR_MB_F32_V2
                           : ((PASS == 1 && !cpl) ? CF_PAIR_MB_F32_A : CF_PAIR_MB_F32))
                    : CF_PAIR_MB_F32_H2)
          : (cpl ? CF_PAIR_MB_F64_COMOV : (H == 1 ? CF_PAIR_MB_F64 : CF_PAIR_MB_F64_H2));
};

template <typename S, int H, int EQ, int PASS, bool FULL>
__global__ void __launch_bounds__(TX *TY, (PairMinBlocks<S, H, EQ, PASS>::value)) k_pair(const PairArgs<S> A) {
  constexpr int VW = PairVec<S, H, EQ, PASS>::value;
  using PS = PairSmem<S, H, TX, TY, VW>;
  __shared__ __align__(16) S sm[PS::count];
  const int a_begin = blockIdx.z * A.a_chunk;
  pair_tile<S, H, EQ, PASS, TX, TY, FULL, VW>(A, blockIdx.x * PS::TS::TW, blockIdx.y * TY, a_begin,
                                          min(a_begin + A.a_chunk, A.N), sm);
}

// Planes per CTA along a: enough CTAs to fill the GPU several times over.
static int pick_a_chunk(int N, int tiles_xy) {
  int chunk = 32;
  while (chunk > 4 && (long long)tiles_xy * ((N + chunk - 1) / chunk) < 148LL * 8) chunk /= 2;
  return chunk;
}

template <typename S, int H, int EQ, int STAGE>
static int launch_stage_t(cf_ctx *ctx, const StageArgs<S> &A0, cudaStream_t st) {
  constexpr int TW = TX * VecT<S>::n;
  StageArgs<S> A = A0;
  dim3 block(TX, TY);
  unsigned gx = ceil_div(A.N, TW), gy = ceil_div(A.N, TY);
  A.a_chunk = pick_a_chunk(A.N, (int)(gx * gy));
  dim3 grid(gx, gy, ceil_div(A.N, A.a_chunk));
  ProfScope ps(ctx, STAGE == 0 ? CF_PROF_OTHER : STAGE - 1, st);
  if (A.N % TW == 0 && A.N % TY == 0)
    k_stage<S, H, EQ, STAGE, true><<<grid, block, 0, st>>>(A);
  else
    k_stage<S, H, EQ, STAGE, false><<<grid, block, 0, st>>>(A);
  CF_LAUNCHED(ctx);
  return CF_OK;
}

template <typename S, int EQ, int STAGE>
static int launch_stage_h(cf_ctx *ctx, int stencil, const StageArgs<S> &A, cudaStream_t st) {
  if (stencil == 13) return launch_stage_t<S, 2, EQ, STAGE>(ctx, A, st);
  return launch_stage_t<S, 1, EQ, STAGE>(ctx, A, st);
}

// The tile kernels' equation shape of a cf_equation.
static int shape_of(int equation) {
  switch (equation) {
    case CF_EQ_COMOVING_FRW: return EQ_COMOV;
    case CF_EQ_LAMBDA_FRW: return EQ_LAMBDA;
    case CF_EQ_SQRT_FRW: return EQ_SQRT;
    case CF_EQ_FIXED_CURVATURE_FRW: return EQ_FIXED;
    case CF_EQ_APPROX_COMOVING_FRW: return EQ_APPROX;
    default: return EQ_FRW;  // CF_EQ_KG (H = 0), CF_EQ_KG_FRW
  }
}

template <typename S, int STAGE>
static int launch_stage(cf_ctx *ctx, const StageArgs<S> &A, cudaStream_t st) {
  const int sten = ctx->p.stencil;
  switch (shape_of(ctx->p.equation)) {
    case EQ_COMOV: return launch_stage_h<S, EQ_COMOV, STAGE>(ctx, sten, A, st);
    case EQ_LAMBDA: return launch_stage_h<S, EQ_LAMBDA, STAGE>(ctx, sten, A, st);
    case EQ_SQRT: return launch_stage_h<S, EQ_SQRT, STAGE>(ctx, sten, A, st);
    case EQ_FIXED: return launch_stage_h<S, EQ_FIXED, STAGE>(ctx, sten, A, st);
    case EQ_APPROX: return launch_stage_h<S, EQ_APPROX, STAGE>(ctx, sten, A, st);
    default: return launch_stage_h<S, EQ_FRW, STAGE>(ctx, sten, A, st);
  }
}

template <typename S, int H, int EQ, int PASS>
static int launch_pair_t(cf_ctx *ctx, const PairArgs<S> &A0, cudaStream_t st) {
  constexpr int TW = TX * PairVec<S, H, EQ, PASS>::value;
  PairArgs<S> A = A0;
  dim3 block(TX, TY);
  unsigned gx = ceil_div(A.N, TW), gy = ceil_div(A.N, TY);
  A.a_chunk = pick_a_chunk(A.N, (int)(gx * gy));
  dim3 grid(gx, gy, ceil_div(A.N, A.a_chunk));
  ProfScope ps(ctx, PASS == 1 ? CF_PROF_PAIR_A : CF_PROF_PAIR_B, st);
  if (A.N % TW == 0 && A.N % TY == 0)
    k_pair<S, H, EQ, PASS, true><<<grid, block, 0, st>>>(A);
  else
    k_pair<S, H, EQ, PASS, false><<<grid, block, 0, st>>>(A);
  CF_LAUNCHED(ctx);
  return CF_OK;
}

template <typename S, int EQ, int PASS>
static int launch_pair_h(cf_ctx *ctx, const PairArgs<S> &A, cudaStream_t st) {
  if (ctx->p.stencil == 13) return launch_pair_t<S, 2, EQ, PASS>(ctx, A, st);
  return launch_pair_t<S, 1, EQ, PASS>(ctx, A, st);
}

template <typename S, int PASS>
static int launch_pair(cf_ctx *ctx, const PairArgs<S> &A, cudaStream_t st) {
  switch (shape_of(ctx->p.equation)) {
    case EQ_COMOV: return launch_pair_h<S, EQ_COMOV, PASS>(ctx, A, st);
    case EQ_LAMBDA: return launch_pair_h<S, EQ_LAMBDA, PASS>(ctx, A, st);
    case EQ_SQRT: return launch_pair_h<S, EQ_SQRT, PASS>(ctx, A, st);
    case EQ_FIXED: return launch_pair_h<S, EQ_FIXED, PASS>(ctx, A, st);
    case EQ_APPROX: return launch_pair_h<S, EQ_APPROX, PASS>(ctx, A, st);
    default: return launch_pair_h<S, EQ_FRW, PASS>(ctx, A, st);
  }
}

// Time-independent constants of the equation: lambda, or f_a^2 and 1/f_a^2; the
// approximate equation's coarse grid.
static void eq_consts(const cf_ctx *ctx, double *q1, double *q2, const int **cmap, int *M) {
  *q1 = *q2 = 0.0;
  if (ctx->p.equation == CF_EQ_LAMBDA_FRW) *q1 = ctx->p.lambda;
  if (ctx->p.equation == CF_EQ_SQRT_FRW) {
    *q1 = ctx->p.f_a * ctx->p.f_a;
    *q2 = 1.0 / (ctx->p.f_a * ctx->p.f_a);
  }
  *cmap = ctx->ap_cmap;
  *M = (int)ctx->p.M;
}

// The curvature input of a stage at time t: the comoving Psi slot, the fixed Psi
// plane or the approximate equation's coarse table (none for the others).
// pipe: the comoving slot was filled on the side stream (psi_pipe_fill_step); st waits for it.
template <typename S>
static int curvature_at(cf_ctx *ctx, double t, const S **psi, const S **dpsi, cudaStream_t st, bool pipe = false) {
  *psi = *dpsi = nullptr;
  const void *ps = nullptr, *dps = nullptr;
  switch (ctx->p.equation) {
    case CF_EQ_COMOVING_FRW:
      CF_TRY(pipe ? psi_pipe_use(ctx, t, st, &ps, &dps) : psi_at(ctx, t, st, &ps, &dps));
      break;
    case CF_EQ_FIXED_CURVATURE_FRW: ps = ctx->fixed_e2m1; break;
    case CF_EQ_APPROX_COMOVING_FRW: CF_TRY(approx_at(ctx, t, st, &ps)); break;
    default: break;
  }
  *psi = (const S *)ps;
  *dpsi = (const S *)dps;
  return CF_OK;
}

// Stage-time coefficients and curvature input of a paired pass.
template <typename S>
static int pair_coeffs(cf_ctx *ctx, double t, double *inv, double *hub3, const S **psi, const S **dpsi,
                       cudaStream_t st, bool pipe = false) {
  double H;
  stage_coeffs(ctx->p, t, inv, &H);
  *hub3 = 3.0 * H;
  return curvature_at<S>(ctx, t, psi, dpsi, st, pipe);
}

// Comoving curvature: cf_rk4_steps synthesises the next step's new Psi slots on the
// context's side stream while the current step's passes run (psi_pipe_*); the same
// slots and kernels, so the same bits as CF_FLAG_PSI_SERIAL.
static bool psi_pipelined(const cf_ctx *ctx, int64_t nsteps) {
  return ctx->p.equation == CF_EQ_COMOVING_FRW && !(ctx->p.flags & CF_FLAG_PSI_SERIAL) && nsteps >= 2;
}
// Before step j: the slots of step j's stage times (present after step 0) and, but
// for the last step, those of step j + 1, on the side stream.  The times are the
// ones the passes read: t, t + dt/2, t + dt with t = t0 + n dt.
// next = false: step j's own slots (already there but at a call's first step), before
// its passes are enqueued; next = true: step j + 1's, after them, so that the host's
// wait for a pass-A comparison (psi_pipe_fill) finds step j queued on the GPU.
static int psi_pipe_fill_step(cf_ctx *ctx, double t0, double dt, int64_t step0, int64_t j, int64_t nsteps,
                              bool next) {
  const double t = t0 + (double)(step0 + j) * dt, tn = t0 + (double)(step0 + j + 1) * dt;
  const double keep[6] = {t, t + dt / 2.0, t + dt, tn, tn + dt / 2.0, tn + dt};
  if (!next)
    for (int k = 0; k < 3; ++k) CF_TRY(psi_pipe_fill(ctx, keep[k], keep, 3));
  else if (j + 1 < nsteps)
    for (int k = 3; k < 6; ++k) CF_TRY(psi_pipe_fill(ctx, keep[k], keep, 6));
  return CF_OK;
}

// nsteps RK4 steps as paired-stage passes.  The new phi of pass B alternates
// between the state's phi plane and the first half of the ya scratch; after an
// odd number of steps it is copied back.
template <typename S>
static int rk4_steps_pairs_t(cf_ctx *ctx, void *d_state, double t0, double dt, int64_t step0, int64_t nsteps,
                             cudaStream_t st) {
  CF_TRY(ensure_rk4_scratch(ctx));
  const long long N3 = ctx->N3;
  S *x = (S *)d_state;
  S *phi[2] = {x, (S *)ctx->ya};
  int cur = 0;
  PairArgs<S> A{};
  A.N = (int)ctx->N;
  A.N3 = N3;
  A.m2 = ctx->p.m * ctx->p.m;
  eq_consts(ctx, &A.q1, &A.q2, &A.cmap, &A.M);
  A.xpi = x + N3;
  A.xlo = (sizeof(S) == 4) ? x + 2 * N3 : nullptr;
  A.acc = (S *)ctx->acc;
  A.yb = (S *)ctx->yb;
  const double dh = dt / 2.0;
  A.dt6 = dt / 6.0;
  bool pipe = psi_pipelined(ctx, nsteps);
  if (pipe) CF_TRY(psi_pipe_begin(ctx, st, &pipe));
  for (int64_t j = 0; j < nsteps; ++j) {
    const double t = t0 + (double)(step0 + j) * dt;
    const double th = t + dh;
    if (pipe) CF_TRY(psi_pipe_fill_step(ctx, t0, dt, step0, j, nsteps, false));
    // pass A: stages 1 (t) and 2 (t + dt/2)
    CF_TRY(pair_coeffs<S>(ctx, t, &A.inv1, &A.hub3_1, &A.psi1, &A.dpsi1, st, pipe));
    CF_TRY(pair_coeffs<S>(ctx, th, &A.inv2, &A.hub3_2, &A.psi2, &A.dpsi2, st, pipe));
    A.uphi = phi[cur];
    A.upi = x + N3;
    A.xphi = phi[cur];
    A.xphi_out = nullptr;
    A.cw = dh;
    A.cy = dh;
    CF_TRY(launch_pair<S, 1>(ctx, A, st));
    // pass B: stages 3 (t + dt/2) and 4 (t + dt)
    CF_TRY(pair_coeffs<S>(ctx, th, &A.inv1, &A.hub3_1, &A.psi1, &A.dpsi1, st, pipe));
    CF_TRY(pair_coeffs<S>(ctx, t + dt, &A.inv2, &A.hub3_2, &A.psi2, &A.dpsi2, st, pipe));
    A.uphi = A.yb;
    A.upi = A.yb + N3;
    A.xphi = phi[cur];
    A.xphi_out = phi[cur ^ 1];
    A.cw = dt;
    CF_TRY(launch_pair<S, 2>(ctx, A, st));
    if (pipe) CF_TRY(psi_pipe_fill_step(ctx, t0, dt, step0, j, nsteps, true));
    if (pipe) CF_TRY(psi_pipe_step_done(ctx, st));
    cur ^= 1;
  }
  if (pipe) CF_TRY(psi_pipe_end(ctx, st));
  if (cur) CF_TRY_CUDA(cudaMemcpyAsync(x, phi[1], N3 * sizeof(S), cudaMemcpyDeviceToDevice, st));
  return CF_OK;
}

// ---- whole-step passes (7-point) -------------------------------------------
// CTA shape per storage type, measured at N = 512 (ms per step, KG-FRW / comoving
// step kernel): FP32 32 x 8 threads (128 x 8 sites, 2 CTAs/SM) 1.34 / 2.13 against
// 16 x 16 1.41 / 2.22 and 16 x 8 (3 CTAs/SM) 1.59 / 2.41; FP64 16 x 8 threads (32 x 8
// sites, 3 CTAs/SM) 1.71 / 3.14 against 32 x 8 1.85 / 3.19 and 16 x 16 1.81 / 3.32.
template <typename S, int EQ>
struct StepShape;
// RW: two ring warps beside the own rows (step_tile RINGW), measured at N = 512
// (ms per step, step kernel, comoving / KG-FRW): FP32 1.876 / 1.191 against 1.975 /
// 1.195 without; FP64 2.883 / 1.731 against 2.942 / 1.721; bit-identical.
template <int EQ>
struct StepShape<float, EQ> {
  static constexpr int TX = 32, TY = 8, MB = 2;
  static constexpr bool RW = true;
};
// FP64: 32 x 8 sites (57 KB, 3 CTAs per SM), or for the equations with a curvature
// input 64 x 8 (109 KB, 2 CTAs of 10 warps, at most 102 registers, no spills): N = 512
// step kernel, comoving 2.81 -> 2.56 ms, KG-FRW 1.69 -> 1.74 (so it keeps 32 x 8);
// every tile shape forms the same values, so the bits do not change.
template <int EQ>
struct StepShape<double, EQ> {
  static constexpr bool wide = EqOf<EQ>::coupled;
  static constexpr int TX = wide ? 32 : 16, TY = 8, MB = wide ? 2 : 3;
  static constexpr bool RW = true;
};
template <typename S, int EQ>
constexpr int step_threads_y() {
  return StepShape<S, EQ>::TY + (StepShape<S, EQ>::RW ? 2 : 0);
}

template <typename S, int EQ, bool FULL>
__global__ void __launch_bounds__(StepShape<S, EQ>::TX *step_threads_y<S, EQ>(), StepShape<S, EQ>::MB)
    k_step(const StepArgs<S> A) {
  extern __shared__ __align__(16) unsigned char step_smem[];
  constexpr int TXs = StepShape<S, EQ>::TX, TYs = StepShape<S, EQ>::TY;
  using SM = StepSmem<S, TXs, TYs>;
  const int a_begin = blockIdx.z * A.a_chunk;
  step_tile<S, EQ, TXs, TYs, FULL, StepShape<S, EQ>::RW>(A, blockIdx.x * SM::TW, blockIdx.y * TYs, a_begin,
                                                     min(a_begin + A.a_chunk, A.N), reinterpret_cast<S *>(step_smem));
}

// Planes per CTA: each chunk re-reads 4 halo planes, so chunks are long where the
// grid stays several waves deep.
static int step_a_chunk(int N, int tiles_xy) {
  int chunk = 64;
  while (chunk > 4 && (long long)tiles_xy * ((N + chunk - 1) / chunk) < 148LL * 6) chunk /= 2;
  return chunk;
}

template <typename S, int EQ, bool FULL>
static int launch_step_k(cf_ctx *ctx, const StepArgs<S> &A, dim3 grid, cudaStream_t st) {
  using SM = StepSmem<S, StepShape<S, EQ>::TX, StepShape<S, EQ>::TY>;
  constexpr size_t bytes = (size_t)SM::count * sizeof(S);
  static unsigned long long attr_set = 0;  // devices on which this instantiation may use > 48 KB
  const unsigned long long bit = 1ull << (ctx->device & 63);
  if (!(attr_set & bit)) {
    CF_TRY_CUDA(cudaFuncSetAttribute(k_step<S, EQ, FULL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    attr_set |= bit;
  }
  k_step<S, EQ, FULL><<<grid, dim3(StepShape<S, EQ>::TX, step_threads_y<S, EQ>()), bytes, st>>>(A);
  CF_LAUNCHED(ctx);
  return CF_OK;
}

template <typename S, int EQ>
static int launch_step_t(cf_ctx *ctx, const StepArgs<S> &A0, cudaStream_t st) {
  using SM = StepSmem<S, StepShape<S, EQ>::TX, StepShape<S, EQ>::TY>;
  constexpr int TYs = StepShape<S, EQ>::TY;
  StepArgs<S> A = A0;
  unsigned gx = ceil_div(A.N, SM::TW), gy = ceil_div(A.N, TYs);
  A.a_chunk = step_a_chunk(A.N, (int)(gx * gy));
  dim3 grid(gx, gy, ceil_div(A.N, A.a_chunk));
  ProfScope ps(ctx, CF_PROF_STEP, st);
  if (A.N % SM::TW == 0 && A.N % TYs == 0) return launch_step_k<S, EQ, true>(ctx, A, grid, st);
  return launch_step_k<S, EQ, false>(ctx, A, grid, st);
}

// ---- whole-step passes, 13-point stencil (FP32 storage) -------------------
// 64 x 16 sites per CTA, two ring warps, 177 KB of shared memory: 1 CTA per SM.  The
// 2-site ring makes phase 1 form 20 x 68 sites per 1024 own sites (1.33x) against 12 x
// 68 per 512 (1.59x) at 64 x 8 (108 KB, 2 CTAs per SM): KG-FRW at N = 512 2.165 -> 2.076
// ms per step.  For the comoving equation, which the paired passes serve (3.54 ms),
// the whole-step pass measured 3.59 at 64 x 8 and 3.84 at 64 x 16.
constexpr int S13_TX = 32, S13_TY = 16;

template <int EQ, bool FULL>
__global__ void __launch_bounds__(S13_TX *(S13_TY + 2), 1) k_step13(const StepArgs<float> A) {
  extern __shared__ __align__(16) unsigned char step13_smem[];
  using SM = Step13Smem<S13_TX, S13_TY>;
  const int a_begin = blockIdx.z * A.a_chunk;
  step13_tile<EQ, S13_TX, S13_TY, FULL>(A, blockIdx.x * SM::TW, blockIdx.y * S13_TY, a_begin,
                                        min(a_begin + A.a_chunk, A.N), reinterpret_cast<float *>(step13_smem));
}

template <int EQ, bool FULL>
static int launch_step13_k(cf_ctx *ctx, const StepArgs<float> &A, dim3 grid, cudaStream_t st) {
  using SM = Step13Smem<S13_TX, S13_TY>;
  constexpr size_t bytes = (size_t)SM::count * sizeof(float);
  static unsigned long long attr_set = 0;  // devices on which this instantiation may use > 48 KB
  const unsigned long long bit = 1ull << (ctx->device & 63);
  if (!(attr_set & bit)) {
    CF_TRY_CUDA(cudaFuncSetAttribute(k_step13<EQ, FULL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    attr_set |= bit;
  }
  k_step13<EQ, FULL><<<grid, dim3(S13_TX, S13_TY + 2), bytes, st>>>(A);
  CF_LAUNCHED(ctx);
  return CF_OK;
}

template <int EQ>
static int launch_step13_t(cf_ctx *ctx, const StepArgs<float> &A0, cudaStream_t st) {
  using SM = Step13Smem<S13_TX, S13_TY>;
  StepArgs<float> A = A0;
  const unsigned gx = ceil_div(A.N, SM::TW), gy = ceil_div(A.N, S13_TY);
  A.a_chunk = step_a_chunk(A.N, (int)(gx * gy));
  const dim3 grid(gx, gy, ceil_div(A.N, A.a_chunk));
  ProfScope ps(ctx, CF_PROF_STEP, st);
  if (A.N % SM::TW == 0 && A.N % S13_TY == 0) return launch_step13_k<EQ, true>(ctx, A, grid, st);
  return launch_step13_k<EQ, false>(ctx, A, grid, st);
}

template <typename S>
static int launch_step(cf_ctx *ctx, const StepArgs<S> &A, cudaStream_t st) {
  if constexpr (sizeof(S) == 4) {
    if (ctx->p.stencil == 13) {  // the equations without curvature planes (rk4_steps routes the others)
      switch (shape_of(ctx->p.equation)) {
        case EQ_LAMBDA: return launch_step13_t<EQ_LAMBDA>(ctx, A, st);
        case EQ_SQRT: return launch_step13_t<EQ_SQRT>(ctx, A, st);
        case EQ_FRW: return launch_step13_t<EQ_FRW>(ctx, A, st);
        default: return set_error("13-point whole-step pass: curvature-coupled equation"), CF_ERR_INVALID;
      }
    }
  }
  switch (shape_of(ctx->p.equation)) {
    case EQ_COMOV: return launch_step_t<S, EQ_COMOV>(ctx, A, st);
    case EQ_LAMBDA: return launch_step_t<S, EQ_LAMBDA>(ctx, A, st);
    case EQ_SQRT: return launch_step_t<S, EQ_SQRT>(ctx, A, st);
    case EQ_FIXED: return launch_step_t<S, EQ_FIXED>(ctx, A, st);
    case EQ_APPROX: return launch_step_t<S, EQ_APPROX>(ctx, A, st);
    default: return launch_step_t<S, EQ_FRW>(ctx, A, st);
  }
}

// nsteps RK4 steps as whole-step passes.  The new phi and pi alternate between the
// state's planes and the ya scratch; after an odd number of steps they are copied back.
template <typename S>
static int rk4_steps_fused_t(cf_ctx *ctx, void *d_state, double t0, double dt, int64_t step0, int64_t nsteps,
                             cudaStream_t st) {
  CF_TRY(ensure_rk4_scratch(ctx));
  const long long N3 = ctx->N3;
  S *x = (S *)d_state;
  S *buf[2] = {x, (S *)ctx->ya};
  int cur = 0;
  StepArgs<S> A{};
  A.N = (int)ctx->N;
  A.N3 = N3;
  A.m2 = ctx->p.m * ctx->p.m;
  eq_consts(ctx, &A.q1, &A.q2, &A.cmap, &A.M);
  A.xlo = (sizeof(S) == 4) ? x + 2 * N3 : nullptr;
  A.dt2 = dt / 2.0;
  A.dt = dt;
  A.dt6 = dt / 6.0;
  bool pipe = psi_pipelined(ctx, nsteps);
  if (pipe) CF_TRY(psi_pipe_begin(ctx, st, &pipe));
  for (int64_t j = 0; j < nsteps; ++j) {
    const double t = t0 + (double)(step0 + j) * dt;
    const double ts[3] = {t, t + dt / 2.0, t + dt};
    if (pipe) CF_TRY(psi_pipe_fill_step(ctx, t0, dt, step0, j, nsteps, false));
    for (int k = 0; k < 3; ++k) {
      double H;
      stage_coeffs(ctx->p, ts[k], &A.inv[k], &H);
      A.hub3[k] = 3.0 * H;
      CF_TRY(curvature_at<S>(ctx, ts[k], &A.psi[k], &A.dpsi[k], st, pipe));
    }
    A.xphi = buf[cur];
    A.xpi = buf[cur] + N3;
    A.ophi = buf[cur ^ 1];
    A.opi = buf[cur ^ 1] + N3;
    CF_TRY(launch_step<S>(ctx, A, st));
    if (pipe) CF_TRY(psi_pipe_fill_step(ctx, t0, dt, step0, j, nsteps, true));
    if (pipe) CF_TRY(psi_pipe_step_done(ctx, st));
    cur ^= 1;
  }
  if (pipe) CF_TRY(psi_pipe_end(ctx, st));
  if (cur) CF_TRY_CUDA(cudaMemcpyAsync(x, buf[1], 2 * N3 * sizeof(S), cudaMemcpyDeviceToDevice, st));
  return CF_OK;
}

template <typename S>
static int fill_stage_coeffs(cf_ctx *ctx, StageArgs<S> &A, double t, cudaStream_t st) {
  double inv, H;
  stage_coeffs(ctx->p, t, &inv, &H);
  A.inv = inv;
  A.hub3 = 3.0 * H;
  eq_consts(ctx, &A.q1, &A.q2, &A.cmap, &A.M);
  return curvature_at<S>(ctx, t, &A.psi, &A.dpsi, st);
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

// One RK4 step of the uncoupled equations with caller-provided accumulator and
// stage buffers (acc, ya, yb: 2N^3 words each of the storage type); allocates
// nothing.  Same kernels and coefficients as rk4_steps.
template <typename S>
static int rk4_step_buffers_t(cf_ctx *ctx, void *d_state, void *acc, void *ya, void *yb, double t, double dt,
                              cudaStream_t st) {
  const long long N3 = ctx->N3;
  S *x = (S *)d_state;
  StageArgs<S> A{};
  A.N = (int)ctx->N;
  A.N3 = N3;
  A.m2 = ctx->p.m * ctx->p.m;
  A.x = x;
  A.xlo = (sizeof(S) == 4) ? x + 2 * N3 : nullptr;
  A.acc = (S *)acc;
  const double dh = dt / 2.0;
  A.dt6 = dt / 6.0;
  CF_TRY(fill_stage_coeffs(ctx, A, t, st));
  A.yin = x;
  A.yout = (S *)ya;
  A.cy = dh;
  CF_TRY(launch_stage<S, 1>(ctx, A, st));
  CF_TRY(fill_stage_coeffs(ctx, A, t + dh, st));
  A.yin = (const S *)ya;
  A.yout = (S *)yb;
  A.cy = dh;
  CF_TRY(launch_stage<S, 2>(ctx, A, st));
  A.yin = (const S *)yb;
  A.yout = (S *)ya;
  A.cy = dt;
  CF_TRY(launch_stage<S, 3>(ctx, A, st));
  CF_TRY(fill_stage_coeffs(ctx, A, t + dt, st));
  A.yin = (const S *)ya;
  A.yout = nullptr;
  return launch_stage<S, 4>(ctx, A, st);
}

int rk4_step_buffers(cf_ctx *ctx, void *d_state, void *acc, void *ya, void *yb, double t, double dt,
                     cudaStream_t st) {
  if (ctx->p.precision == CF_FP32_COMP) return rk4_step_buffers_t<float>(ctx, d_state, acc, ya, yb, t, dt, st);
  return rk4_step_buffers_t<double>(ctx, d_state, acc, ya, yb, t, dt, st);
}

int rk4_steps(cf_ctx *ctx, void *d_state, double t0, double dt, int64_t step0, int64_t nsteps, cudaStream_t st) {
  const int f = ctx->p.flags;
  const bool f32 = ctx->p.precision == CF_FP32_COMP;
  if (f & CF_FLAG_STAGE_KERNELS)
    return f32 ? rk4_steps_t<float>(ctx, d_state, t0, dt, step0, nsteps, st)
               : rk4_steps_t<double>(ctx, d_state, t0, dt, step0, nsteps, st);
  // 13-point stencil: the whole-step pass for FP32 storage and the equations without
  // curvature planes; the paired passes for FP64 and for the curvature-coupled
  // equations, where they measured faster (N = 512, FP32_COMP, ms per step: KG-FRW
  // whole-step 2.17 / paired 2.55; comoving 3.86 / 3.81, with an L2 prefetch of the
  // curvature rows 4.45 / 3.81)
  const int shape = shape_of(ctx->p.equation);
  const bool coupled = shape == EQ_COMOV || shape == EQ_FIXED || shape == EQ_APPROX;
  if ((f & CF_FLAG_PAIR_KERNELS) || (ctx->p.stencil != 7 && (!f32 || coupled)))
    return f32 ? rk4_steps_pairs_t<float>(ctx, d_state, t0, dt, step0, nsteps, st)
               : rk4_steps_pairs_t<double>(ctx, d_state, t0, dt, step0, nsteps, st);
  return f32 ? rk4_steps_fused_t<float>(ctx, d_state, t0, dt, step0, nsteps, st)
             : rk4_steps_fused_t<double>(ctx, d_state, t0, dt, step0, nsteps, st);
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
