// cf_f32x2.cuh -- the FP32 stage arithmetic, written once for one site (float) and
// for a pair of sites (float2, the sm_100 paired FP32 instructions FADD2 / FMUL2 /
// FFMA2: one issue slot for two lanes, each lane rounded exactly as the scalar
// instruction).
//
// Every FP32 operation of the stepping tiles is spelled out here with explicit
// round-to-nearest intrinsics, so the compiler neither contracts nor reorders it:
// the single-stage and paired-stage tiles evaluate sites one at a time, the
// whole-step tile two at a time, and all of them produce the same bits.
#pragma once

#include <cuda_runtime.h>

namespace cfb {

// ---- primitives, one lane or two ------------------------------------------
__device__ __forceinline__ float p_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float2 p_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float p_sub(float a, float b) { return __fadd_rn(a, -b); }
__device__ __forceinline__ float2 p_sub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float p_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float2 p_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float p_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float2 p_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float p_neg(float a) { return -a; }
__device__ __forceinline__ float2 p_neg(float2 a) { return make_float2(-a.x, -a.y); }

template <typename L>
__device__ __forceinline__ L p_splat(float c);
template <>
__device__ __forceinline__ float p_splat<float>(float c) {
  return c;
}
template <>
__device__ __forceinline__ float2 p_splat<float2>(float c) {
  return make_float2(c, c);
}

// A coefficient c = hi + lo (hi = (float)c, lo = (float)(c - hi)) in the lane type:
// c v is formed as fma(hi, v, lo v), whose error is random rather than the fixed
// relative bias of a rounded coefficient.
template <typename L>
struct CoefL {
  L hi, lo;
};
using C2 = CoefL<float2>;

__host__ __device__ inline CoefL<float> coef_f32(double c) {
  const float hi = (float)c;
  return CoefL<float>{hi, (float)(c - (double)hi)};
}
__host__ __device__ inline C2 coef_f32x2(double c) {
  const float hi = (float)c, lo = (float)(c - (double)hi);
  return C2{make_float2(hi, hi), make_float2(lo, lo)};
}

template <typename L>
__device__ __forceinline__ L c_mul(const CoefL<L> &c, L v) {
  return p_fma(c.hi, v, p_mul(c.lo, v));
}
// add + c v
template <typename L>
__device__ __forceinline__ L c_fma(const CoefL<L> &c, L v, L add) {
  return p_add(add, c_mul(c, v));
}

// The coefficients of one stage evaluation (StageArgs::m2, inv, hub3, q1, q2).
template <typename L>
struct StageCoefL {
  CoefL<L> m2, inv, hub3, q1, q2;
};

// 7-point Laplacian sum (times h^2): ((((-6 f0 + a+) + a-) + b+) + b-) + (c+ + c-).
template <typename L>
__device__ __forceinline__ L lap7_f32(L f0, L ap, L am, L bp, L bm, L cp, L cm) {
  L s = p_fma(p_splat<L>(-6.0f), f0, ap);
  s = p_add(s, am);
  s = p_add(s, bp);
  s = p_add(s, bm);
  return p_add(s, p_add(cp, cm));
}

// 13-point 4th-order Laplacian sum times 12 h^2 from the six first and the six second
// neighbours (each summed a+, a-, b+, b-, c+, c-): 16 s1 - s2 - 90 f0.  The 1/12 goes
// into the stage's h^-2 a^-2 coefficient instead (lap_coef_f32), saving a division and a
// rounding; every FP32 13-point route does the same.
template <typename L>
__device__ __forceinline__ L lap13_f32(L f0, L s1, L s2) {
  const L r = p_fma(p_splat<L>(16.0f), s1, p_neg(s2));
  return p_fma(p_splat<L>(-90.0f), f0, r);
}

// The coefficient of the Laplacian sum in the FP32 stage arithmetic: h^-2 a^-2, and
// h^-2 a^-2 / 12 for the 13-point stencil (whose sum lap13_f32 leaves times 12).
template <int H>
__host__ __device__ inline double lap_coef_f32(double inv) {
  return H == 2 ? inv / 12.0 : inv;
}

// pi component of the right-hand side (src/equations_cuda.cu:15-36 FRW, :38-76
// lambda, :84-104 sqrt potential, :112-136 fixed Psi, :263-287 comoving, :299-329
// approximate comoving) in FP32: ps = e^{2Psi} - 1 (EQ_APPROX: 2Psi + 2Psi^2), dps
// = dPsi/dt, ps4 = 4Psi + 8Psi^2 (EQ_APPROX); e^{2Psi} enters as 1 + ps and is never
// rounded as such.  EQ is an EqShape (cf_stage_tile.cuh).
template <int EQ, typename L>
__device__ __forceinline__ L kpi_f32(L p0, L f0, L lap, L ps, L dps, L ps4, const StageCoefL<L> &k) {
  const L mf = c_mul(k.m2, f0);
  const L g = c_mul(k.inv, lap);
  const L h = c_mul(k.hub3, p0);
  if constexpr (EQ == 1 || EQ == 4 || EQ == 5) {  // EQ_COMOV, EQ_FIXED, EQ_APPROX
    // e^{4Psi} - 1 = (e^{2Psi} - 1)(e^{2Psi} + 1); the approximate equation's own quadratic
    const L e4m1 = (EQ == 5) ? ps4 : p_mul(ps, p_add(ps, p_splat<L>(2.0f)));
    L fr;
    if constexpr (EQ == 4)
      fr = p_neg(h);
    else
      fr = p_fma(p_mul(p_splat<L>(4.0f), dps), p0, p_neg(h));
    return p_add(p_sub(fr, p_fma(ps, mf, mf)), p_fma(e4m1, g, g));
  } else if constexpr (EQ == 2) {  // EQ_LAMBDA: - lambda phi^3
    const L q = c_mul(k.q1, p_mul(p_mul(f0, f0), f0));
    return p_add(p_sub(p_sub(p_neg(h), mf), q), g);
  } else if constexpr (EQ == 3) {  // EQ_SQRT: m^2 phi / sqrt(1 + phi^2 / f_a^2)
    // rsqrtf refined by one Newton step r <- r + r (1 - y r^2) / 2, within a fraction
    // of an ulp of 1/sqrt(y) (rounding errors that average out like the other terms')
    const L y = p_add(p_splat<L>(1.0f), c_mul(k.q2, p_mul(f0, f0)));
    L r0;
    if constexpr (sizeof(L) == 4)
      r0 = rsqrtf(y);
    else
      r0 = make_float2(rsqrtf(y.x), rsqrtf(y.y));
    const L e = p_fma(p_neg(p_mul(y, r0)), r0, p_splat<L>(1.0f));
    const L r = p_fma(p_mul(p_splat<L>(0.5f), r0), e, r0);
    return p_add(p_fma(p_neg(mf), r, p_neg(h)), g);
  } else {  // EQ_FRW
    return p_add(p_sub(p_neg(h), mf), g);
  }
}

// FP32_COMP state update hi + lo + c s as a normalised hi + lo pair, in FP32 alone:
// the product c s exactly as p + pe (FMA), hi + p exactly as t + e (TwoSum, Knuth),
// the small parts added, and the pair renormalised (Fast2Sum, |t| >= |e|).
template <typename L>
__device__ __forceinline__ void comp_update_f32(L hi, L lo, L s, const CoefL<L> &c, L &oh, L &ol) {
  const L p = p_mul(c.hi, s);
  const L pe = p_fma(c.lo, s, p_fma(c.hi, s, p_neg(p)));
  const L t = p_add(hi, p);
  const L z = p_sub(t, hi);
  const L e = p_add(p_add(p_sub(hi, p_sub(t, z)), p_sub(p, z)), p_add(lo, pe));
  oh = p_add(t, e);
  ol = p_sub(e, p_sub(oh, t));
}

}  // namespace cfb
