/*
 * cfb200.h -- C ABI of the B200 lattice time-stepping library (libcfb200.so).
 *
 * Scope: the hot path of Cosmic-Fields-Lite -- RK4 time stepping of the
 * Klein-Gordon family on a periodic N^3 lattice (flat, FRW, lambda phi^4,
 * sqrt potential, fixed and comoving-curvature coupled), the energy density, and the field / density power spectra that the
 * observers save.  Everything runs on one CUDA device; there is no CPU fallback:
 * every call that needs the GPU fails with CF_ERR_CUDA if none is usable.
 *
 * Conventions
 *   - Every function returns int status: CF_OK (0) or a negative cf_status code;
 *     cf_last_error() then returns a message (thread-local).
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *     Calls enqueue work and return; there are no hidden device-wide syncs unless
 *     a function says so.
 *   - Device pointers are plain CUDA device addresses owned by the caller.
 *   - Field layout (reference src/fdm3d.hpp:16): site (a,b,c) of an N^3 field at
 *     N*N*a + N*b + c; a "state" in FP64 is 2N^3 doubles [phi | dphi].
 *   - Half-complex (HC) arrays: 2*N*N*(N/2+1) doubles, mode (a,b,c<=N/2) at
 *     2*(N*(N/2+1)*a + (N/2+1)*b + c) (real, imag) -- the FFTW/cuFFT r2c layout.
 *   - S2 spectra: 3*(N/2)^2+1 doubles indexed by s^2 = i^2+j^2+k^2 with lattice
 *     momenta i,j,k in -N/2+1..N/2 (reference src/fdm3d.hpp:27-40).
 *   - Shell spectra: isqrt(3*(N/2)^2)+1 unit-width |k| shells; shell i holds the
 *     s^2 bins in [i^2, (i+1)^2).
 *   - Requirements: N % 8 == 0 and 8 <= N <= 2048 (the reference's own spectra
 *     assert N % 8 == 0, src/fdm3d_cuda.cu:148,165).
 *   - A context is not thread-safe; separate contexts are independent.
 */
#ifndef CFB200_H
#define CFB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CFB200_ABI_VERSION 2

typedef enum cf_status {
  CF_OK = 0,
  CF_ERR_INVALID = -1,     /* bad argument (size, alignment, enum, NULL) */
  CF_ERR_CUDA = -2,        /* CUDA runtime error (message has the CUDA error string) */
  CF_ERR_CUFFT = -3,       /* cuFFT error */
  CF_ERR_NOMEM = -4,       /* device allocation failed */
  CF_ERR_NONFINITE = -5,   /* a NaN/Inf was found in the state */
  CF_ERR_TIMEOUT = -6,     /* a bounded device wait gave up */
  CF_ERR_UNSUPPORTED = -7  /* combination of options not built */
} cf_status;

typedef enum cf_equation {
  CF_EQ_KG = 0,           /* KleinGordonEquation (src/equations.hpp:36-59) */
  CF_EQ_KG_FRW = 1,       /* KleinGordonEquationInFRW / CudaKleinGordonEquationInFRW */
  CF_EQ_COMOVING_FRW = 2, /* ComovingCurvatureEquationInFRW / CudaComovingCurvatureEquationInFRW */
  /* CudaLambdaEquationInFRW (src/equations_cuda.cuh:36-48, src/equations_cuda.cu:38-76,
   * :575-607): dphi' = -3H dphi - m^2 phi - lambda phi^3 + a^-2 h^-2 lap phi */
  CF_EQ_LAMBDA_FRW = 3,
  /* CudaSqrtPotentialEquationInFRW (src/equations_cuda.cuh:50-62, src/equations_cuda.cu:79-104,
   * :610-642): V = m^2 f_a^2 (sqrt(1 + phi^2/f_a^2) - 1),
   * dphi' = -3H dphi - m^2 phi / sqrt(1 + phi^2/f_a^2) + a^-2 h^-2 lap phi */
  CF_EQ_SQRT_FRW = 4,
  /* CudaFixedCurvatureEquationInFRW (src/equations_cuda.cuh:64-76, src/equations_cuda.cu:107-136,
   * :645-675): a time-independent Psi(x) set with cf_set_psi,
   * dphi' = -3H dphi - e^{2Psi} m^2 phi + e^{4Psi} a^-2 h^-2 lap phi */
  CF_EQ_FIXED_CURVATURE_FRW = 5,
  /* CudaApproximateComovingCurvatureEquationInFRW (src/equations_cuda.cuh:92-104,
   * src/equations_cuda.cu:299-329, :764-815): Psi, dPsi/dt synthesised on a coarse
   * M^3 grid from the modes of R_fft below M/2 and sampled at the nearest coarse
   * site, with e^{2Psi} ~ 1 + 2Psi + 2Psi^2 and e^{4Psi} ~ 1 + 4Psi + 8Psi^2 */
  CF_EQ_APPROX_COMOVING_FRW = 6
} cf_equation;

typedef enum cf_precision {
  CF_FP64 = 0,      /* state stored and stepped in FP64 */
  CF_FP32_COMP = 1  /* state stored as FP32 hi + FP32 lo; stage inputs, accumulator and stage
                       arithmetic in FP32 (coefficients as hi + lo pairs, the state update
                       error-free on the hi + lo pair); a(t), H(t), reductions and spectra FP64 */
} cf_precision;

/* Flat parameter block (replaces the reference's POD Param + WorkspaceGeneric
 * field copy, src/workspace.hpp:81-93).  a1, H1, t1, p describe
 * StaticEOSCosmology (src/physics.hpp:15-56); CF_EQ_KG ignores them.  lambda
 * (CF_EQ_LAMBDA_FRW), f_a (CF_EQ_SQRT_FRW, > 0; the reference's default is 1)
 * and M (CF_EQ_APPROX_COMOVING_FRW: M % 8 == 0, M <= N, N % M == 0) are the
 * workspace fields of the same names (src/workspace.hpp:66-67, :77); other
 * equations ignore them. */
typedef struct cf_params {
  int64_t N;
  double L;
  double m;
  double a1;
  double H1;
  double t1;
  double p;          /* a ~ eta^p; 1 = radiation (the reference's param constructor) */
  int32_t equation;  /* cf_equation */
  int32_t precision; /* cf_precision */
  int32_t stencil;   /* 7 (reference) or 13 (fourth-order Laplacian) */
  int32_t flags;     /* CF_FLAG_* bits, 0 = defaults */
  double lambda;     /* quartic coupling */
  double f_a;        /* scale of the sqrt (monodromy) potential */
  int64_t M;         /* coarse grid of the approximate comoving-curvature equation */
} cf_params;

/* Always synthesise Psi / dPsi/dt with the full 3-D C2R, even when R_fft is
 * band-limited (the pruned synthesis is used by default when R_fft is exactly
 * zero outside a small box of modes; both give the same fields to rounding). */
#define CF_FLAG_FULL_PSI_FFT 1
/* cf_rk4_steps runs each step as four single-stage passes instead of the default
 * route; every route gives bit-identical states. */
#define CF_FLAG_STAGE_KERNELS 2
/* cf_rk4_steps runs each 7-point step as two paired-stage passes (stages 1+2, 3+4)
 * instead of one whole-step pass (the default for the 7-point stencil; the 13-point
 * stencil always takes the paired passes). */
#define CF_FLAG_PAIR_KERNELS 4
/* FP32 storage: the pruned Psi synthesis's last pass (the length-N C2R of every row)
 * runs as the CTA-per-tile kernel instead of the default warp-per-row-group kernel
 * (N = 256, 512, 1024); both compute the same values. */
#define CF_FLAG_PSI_CTA_PASS_C 8
/* Comoving-curvature equation: cf_rk4_steps synthesises each step's Psi slots
 * before the step's passes on the caller's stream, instead of synthesising the next
 * step's slots on a side stream of the context while the current step runs (the
 * default; three more N^3 slot pairs, or the serial order when they do not fit);
 * both give bit-identical states. */
#define CF_FLAG_PSI_SERIAL 16
/* FP32 storage: the warp-per-row-group pass C brings its band tiles into shared
 * memory with per-lane cp.async instead of one TMA box per tile (the default at
 * N = 256 and 512 where the driver provides cuTensorMapEncodeTiled; N = 1024 always
 * uses cp.async); both compute the same values. */
#define CF_FLAG_PSI_NO_TMA 32
/* FP32 storage, pruned synthesis, side-stream refreshes: always synthesise a stage
 * time's slot.  By default a time a few ulp from the latest refresh's (the next step's
 * t0 + (n + 1) dt against this step's t + dt) first has its pass-A inputs compared bit
 * for bit with that refresh's, and takes its slot when they are identical (passes A-C
 * are deterministic in those inputs alone); both give bit-identical states. */
#define CF_FLAG_PSI_NO_REUSE 64

typedef struct cf_ctx cf_ctx;

/* Sizes a caller needs to allocate buffers. */
typedef struct cf_info {
  int64_t N;
  int64_t state_bytes;  /* bytes of one device state in this context's precision */
  int64_t field_count;  /* N^3 */
  int64_t hc_count;     /* doubles in one HC array: 2*N*N*(N/2+1) */
  int64_t s2_bins;      /* 3*(N/2)^2+1 */
  int64_t shells;       /* isqrt(3*(N/2)^2)+1 */
  int64_t psi_route;    /* comoving equation: how Psi is synthesised (CF_PSI_*) */
} cf_info;

/* cf_info.psi_route: 0 = no R_fft set (or not the comoving equation);
 * full 3-D C2R; pruned passes A, B with a padded cuFFT C2R as pass C (N not a
 * power of two); pruned passes A, B with pass C as one kernel. */
#define CF_PSI_NONE 0
#define CF_PSI_FULL 1
#define CF_PSI_PRUNED 2
#define CF_PSI_PRUNED_FUSED 3

/* ---- context --------------------------------------------------------------
 * Replaces WorkspaceGeneric's tools (FFT wrapper, Psi buffers) and the odeint
 * stepper's temporaries: the context owns cuFFT plans and all device scratch
 * (allocated on first use of the function that needs it). */
int cf_create(const cf_params *params, cf_ctx **out);
int cf_destroy(cf_ctx *ctx);
int cf_get_info(const cf_ctx *ctx, cf_info *info);
const char *cf_last_error(void);
/* Number of this library's own kernels the context has launched (cuFFT calls not counted). */
int64_t cf_launch_count(const cf_ctx *ctx);

/* ---- state ----------------------------------------------------------------
 * A device state is cf_info.state_bytes bytes, 16-byte aligned, caller owned.
 * CF_FP64: 2N^3 doubles [phi | dphi] -- identical to the reference State
 *   (thrust::device_vector<double>, src/equations_cuda.cuh:22-23).
 * CF_FP32_COMP: four N^3 float planes [phi_hi | dphi_hi | phi_lo | dphi_lo]
 *   with value = (double)hi + (double)lo. */
int cf_state_upload(cf_ctx *ctx, void *d_state, const double *h_xy, void *stream);
int cf_state_download(cf_ctx *ctx, double *h_xy, const void *d_state, void *stream);
int cf_state_import(cf_ctx *ctx, void *d_state, const double *d_xy, void *stream);
int cf_state_export(cf_ctx *ctx, double *d_xy, const void *d_state, void *stream);

/* R_fft: HC array of the comoving curvature perturbation (the reference's
 * workspace.R_fft, src/initializer.hpp:200-205), host or device pointer. */
int cf_set_R_fft(cf_ctx *ctx, const double *R_fft, int on_device, void *stream);

/* Psi: the fixed curvature perturbation of CF_EQ_FIXED_CURVATURE_FRW (the
 * reference's workspace.Psi, N^3 doubles in site order, set by its initializer),
 * host or device pointer.  Required before stepping that equation. */
int cf_set_psi(cf_ctx *ctx, const double *Psi, int on_device, void *stream);

/* Psi(x, t) and dPsi/dt(x, t) of the comoving-curvature equation into d_out
 * (2 N^3 doubles: Psi, then dPsi), the fields the right-hand side uses at time t
 * (the reference computes them inside Equation::operator(),
 * src/equations_cuda.cu:678-731, and exposes no call of its own). */
int cf_psi_fields(cf_ctx *ctx, double t, double *d_out, void *stream);
/* Failure-detection test hook (no counterpart in the reference): the warp pass C's
 * TMA barriers are armed for `extra_bytes` (a multiple of 16) more than each band box
 * delivers, so every bounded wait gives up after `spin_limit` tests (default 2^20).
 * The kernel then sets the context's error word and leaves; the next refresh returns
 * CF_ERR_TIMEOUT.  A call also clears the error word; (0, 1048576) restores normal
 * operation.  Only for N = 256 and 512 in FP32 storage with the pruned synthesis (the
 * TMA route); elsewhere it changes nothing. */
int cf_psi_set_wait_test(cf_ctx *ctx, int extra_bytes, int64_t spin_limit);
/* Psi slots synthesised, and stage times that took the slot of a refresh with
 * bit-identical pass-A inputs instead (CF_FLAG_PSI_NO_REUSE), since the context was made. */
int cf_psi_stats(const cf_ctx *ctx, int64_t *refreshes, int64_t *reused);

/* ---- the hot path -----------------------------------------------------------
 * nsteps classic RK4 steps in place; step j runs at t = t0 + (step0 + j) * dt
 * (integrate_const's direct time, integrate/detail/integrate_const.hpp:63) with
 * stage times t, t+dt/2, t+dt/2, t+dt (stepper/runge_kutta4_classic.hpp:88-138).
 * Replaces 4 x Equation::operator() + 3 x scale_sum2 + scale_sum5 per step
 * (src/equations_cuda.cu:522-534, :678-731; src/odeint_thrust/thrust_operations.cu:238-313)
 * by one HBM pass per step (7-point stencil; 13-point for the equations without a
 * curvature input) or two (13-point with one); see CF_FLAG_*.  Comoving curvature: the
 * next step's Psi slots are synthesised on a side stream of the context, joined by an
 * event on `stream` before the call returns; the host waits only for a pass-A
 * comparison at a step start a few ulp from the previous step's end (CF_FLAG_PSI_NO_REUSE). */
int cf_rk4_steps(cf_ctx *ctx, void *d_state, double t0, double dt, int64_t step0, int64_t nsteps,
                 void *stream);

/* The same stepping as cf_rk4_steps for callers that must not allocate device
 * memory -- applications that hand all device memory to their own pool and
 * forbid library allocations, or loops that cannot take cudaMalloc's
 * synchronisation or its failure mid-run.  No counterpart in the reference.
 * The three RK4 work buffers come from a fixed 24 MiB array compiled into the
 * library (held by every GPU that loads it until exit) instead of the context:
 * N <= 80 in CF_FP64, N <= 96 in CF_FP32_COMP, CF_EQ_KG / CF_EQ_KG_FRW only;
 * anything else is rejected (CF_ERR_INVALID / CF_ERR_UNSUPPORTED).  All calls on
 * a device share the array, which keeps the last call's contents (nothing needs
 * clearing: each step writes every entry before reading it); calls whose GPU work
 * overlaps race and must be serialised by the caller.  With lazy module loading
 * (the CUDA default) the array is reserved on a device by the first call there:
 * an application that gives its free device memory to its own pool makes one call
 * first (nsteps = 0 only reserves the array and resolves its address) or sets
 * CUDA_MODULE_LOADING=EAGER.  Calls outside stream capture look the array's
 * address up afresh (valid after a cudaDeviceReset); calls during capture reuse
 * the last address, so make one call before capturing.  The caller's current
 * device is restored on return.  Calls no cudaMalloc, cudaFree or allocating
 * library routine. */
int cf_rk4_steps_noalloc(cf_ctx *ctx, void *d_state, double t0, double dt, int64_t step0, int64_t nsteps,
                         void *stream);

/* ---- odeint building blocks (FP64 device arrays of 2N^3) --------------------
 * cf_rhs: dxdt = Equation(x, t)  (Equation::operator(), src/equations_cuda.cu:522-534,
 * :678-731).  cf_scale_sum: out = sum_i alpha_i * in_i over len doubles
 * (thrust_operations::scale_sum1..14, src/odeint_thrust/thrust_operations.cuh:24-353);
 * d_in is a HOST array of n device pointers, 1 <= n <= 14; out may alias in[0]. */
int cf_rhs(cf_ctx *ctx, const double *d_x, double *d_dxdt, double t, void *stream);
int cf_scale_sum(cf_ctx *ctx, double *d_out, int n, const double *const *d_in, const double *alpha,
                 int64_t len, void *stream);

/* ---- observers --------------------------------------------------------------
 * cf_energy_density: Equation::compute_energy_density (src/equations_cuda.cu:537-553,
 *   :733-760; lambda :591-607 with :332-369; sqrt potential :626-642 with :431-449;
 *   fixed curvature :660-675 with :451-473; the approximate comoving equation uses
 *   the full comoving one, :812-815) of a device state at time t into d_rho (N^3 doubles).
 * cf_power_spectrum_s2: compute_power_spectrum (src/fdm3d_cuda.cu:161-176) of an N^3
 *   FP64 field: R2C + deterministic binning into S2 bins.
 * cf_mode_power_spectrum_s2: compute_mode_power_spectrum (src/fdm3d_cuda.cu:144-159)
 *   of a state: |phi_k|^2 + |dphi_k|^2/(m^2 + (2 pi/L)^2 s^2/a_t^2) per S2 bin.
 * cf_density_spectrum_s2: energy density at t followed by cf_power_spectrum_s2 (the
 *   observer's rho spectrum, src/observer.hpp:102-108), without a caller buffer.
 * cf_s2_to_shells: exact regrouping of an S2 spectrum computed by this context
 *   (most recent call) into unit shells, with mode counts; d_counts may be NULL.
 * Sums are exact fixed-point integer sums (order independent, bit-reproducible)
 * converted to FP64 once. */
int cf_energy_density(cf_ctx *ctx, const void *d_state, double t, double *d_rho, void *stream);
/* cf_dot_energy_density: CudaKleinGordonEquationInFRW::compute_dot_energy_density
 *   (src/equations_cuda.cu:372-424, :556-572), d rho / dt of the state at t into
 *   d_out (N^3 doubles); CF_EQ_KG_FRW only. */
int cf_dot_energy_density(cf_ctx *ctx, const void *d_state, double t, double *d_out, void *stream);
int cf_power_spectrum_s2(cf_ctx *ctx, const double *d_f, double *d_out, void *stream);
int cf_mode_power_spectrum_s2(cf_ctx *ctx, const void *d_state, double a_t, double *d_out,
                              void *stream);
int cf_density_spectrum_s2(cf_ctx *ctx, const void *d_state, double t, double *d_out, void *stream);
/* cf_density_slices: the observer's density slices (src/observer.hpp:110-119) of the
 *   energy density at t, formed on the device so that only 2 N^2 values cross to the
 *   host: d_slice (N^2) = rho at a = 0, d_axis_average (N^2) = the mean of rho over a
 *   (summed in increasing a, then divided by N).  Either output may be NULL. */
int cf_density_slices(cf_ctx *ctx, const void *d_state, double t, double *d_slice, double *d_axis_average,
                      void *stream);
int cf_s2_to_shells(cf_ctx *ctx, double *d_shells, int64_t *d_counts, void *stream);

/* Mode multiplicity per S2 bin (exact, the rule of plot_util.py:53-58). */
int cf_s2_counts(cf_ctx *ctx, int64_t *d_counts, void *stream);

/* ---- initial conditions -------------------------------------------------------
 * The reference builds its initial fields on the host once, before stepping
 * (src/initializer.hpp:33-301, src/random_field.cpp:36-89, src/fdm3d.cpp:76-102):
 * single-threaded normal draws, FFTW transforms, per-mode loops.  These run them
 * on the device with the context's cuFFT plans.  All arrays are FP64, device,
 * N^3 fields in site order unless said otherwise.
 *
 * cf_white_noise: n unit-normal deviates into d_out, element i a function of
 *   (seed, offset + i) only: Philox4x32-10 (Salmon et al., SC'11) on the counter
 *   (offset + i) / 2 with key `seed`, two 53-bit uniforms per counter, Box-Muller
 *   (cos for even, sin for odd elements).  Any split of a stream into calls gives
 *   the same deviates.  A stand-in for the reference's std::mt19937 +
 *   std::normal_distribution stream (src/random_field.cpp:13-33), which is
 *   sequential; for bit-identical fields a caller draws that stream on the host
 *   and passes it to cf_grf instead.
 * cf_grf: generate_inhomogeneous_gaussian_random_field (src/random_field.cpp:36-83)
 *   from the deviates d_white (N^3, e.g. from cf_white_noise or uploaded):
 *     out = c2r( sqrtP(s^2) r2c( w / N^3 * exp(psi_scale * Psi) ) ),
 *   d_psi may be NULL (Psi = 0: generate_gaussian_random_field, :85-89);
 *   h_sqrtP_s2 is a HOST array of cf_info.s2_bins values sqrt(P(sqrt(s^2) 2 pi / L)),
 *   the spectrum the reference evaluates per mode.  d_out may equal d_white.
 * cf_scale_modes: compute_field_with_scaled_fourier_modes (src/fdm3d.cpp:76-102):
 *     out = c2r( scale(s^2) r2c(f) ),
 *   h_scale_s2 a HOST array of s2_bins values kernel(sqrt(s^2) 2 pi / L) / N^3
 *   (the factor the reference applies per mode).  d_out may equal d_f.
 * Both use the context's spectrum scratch (two HC arrays) and cuFFT plans. */
int cf_white_noise(cf_ctx *ctx, uint64_t seed, uint64_t offset, double *d_out, int64_t n, void *stream);
int cf_grf(cf_ctx *ctx, const double *d_white, const double *d_psi, double psi_scale, const double *h_sqrtP_s2,
           double *d_out, void *stream);
int cf_scale_modes(cf_ctx *ctx, const double *d_f, const double *h_scale_s2, double *d_out, void *stream);

/* ---- WKB continuation ------------------------------------------------------------
 * WKBSolutionForKleinGordonEquationInFRW (src/wkb.hpp:13-27, src/wkb.cpp:5-121): a
 * KG-FRW state at t_i continued analytically to later times, mode by mode.
 *   cf_wkb_create: takes the modes of d_state (FP64 [phi | dphi], 2 N^3, device) at t_i
 *     (the constructor); the context must be CF_EQ_KG_FRW in radiation domination
 *     (p = 1) with t1 = 1/(2 H1), as the reference asserts, and m > 0.
 *   cf_wkb_evaluate: the continued state at t into d_out (FP64 2 N^3, device)
 *     (evaluate_at); returns once the work is done.
 * The handle keeps the context pointer: destroy it before the context. */
typedef struct cf_wkb cf_wkb;
int cf_wkb_create(cf_ctx *ctx, const double *d_state, double t_i, cf_wkb **out, void *stream);
int cf_wkb_evaluate(cf_wkb *wkb, double t, double *d_out, void *stream);
int cf_wkb_destroy(cf_wkb *wkb);

/* ---- FFT wrapper ---------------------------------------------------------------
 * The reference's cufftWrapperNoBatching (src/cuda_wrapper.cuh:113-130,
 * src/cuda_wrapper.cu:202-255), used through workspace.fft_wrapper by initializers,
 * observers and WKB code: 3-D FP64 transforms of an N^3 lattice (N even, 8..2048),
 * unnormalised, forward sign e^{-2 pi i k.x/N}, HC layout N x N x (N/2+1) complex.
 * The handle belongs to the device current at cf_fft_create; its cuFFT plans are
 * made on first use.
 *   cf_fft_d2z:          N^3 real -> HC                       (execute_d2z)
 *   cf_fft_batched_d2z:  2 N^3 real [phi | dphi] -> 2 HC      (execute_batched_d2z)
 *   cf_fft_z2d:          HC -> N^3 real; overwrites d_in      (execute_z2d)
 *   cf_fft_inplace_z2d:  HC -> real in place, rows padded to 2(N/2+1) doubles
 *                        (PADDED_IDX_OF, src/fdm3d.hpp:24)     (execute_inplace_z2d)
 * Device pointers 16-byte aligned; sizes are the caller's to provide. */
typedef struct cf_fft cf_fft;
int cf_fft_create(int64_t N, cf_fft **out);
int cf_fft_destroy(cf_fft *fft);
int cf_fft_d2z(cf_fft *fft, const double *d_in, double *d_out, void *stream);
int cf_fft_batched_d2z(cf_fft *fft, const double *d_in, double *d_out, void *stream);
int cf_fft_z2d(cf_fft *fft, double *d_in, double *d_out, void *stream);
int cf_fft_inplace_z2d(cf_fft *fft, double *d_inout, void *stream);

/* Scans a state for NaN/Inf; synchronises `stream` and sets *h_bad to the number
 * of non-finite entries found (0 if clean).  Returns CF_ERR_NONFINITE if any. */
int cf_check_finite(cf_ctx *ctx, const void *d_state, int64_t *h_bad, void *stream);

/* ---- adjoint (gradients of a spectrum loss) -------------------------------------
 * Discrete adjoint of cf_rk4_steps for CF_EQ_KG / CF_EQ_KG_FRW (7- or 13-point,
 * either precision; adjoint variables are FP64).  No reference counterpart: the
 * reference has no differentiation.
 *   cf_adjoint_create: checkpoints every `checkpoint_every` of `nsteps` steps.
 *   cf_adjoint_forward: runs the nsteps from d_state (in: x0, out: x_T), t_j = t0 + j dt,
 *     storing checkpoints.
 *   cf_adjoint_shell_log_loss: L = sum_s (log P_s - log T_s)^2 over the unit shells s with
 *     P_s > 0 and T_s > rel_floor * max_s T_s (shells at the rounding floor of the
 *     spectrum carry no smooth information; 0 keeps every shell with T_s > 0), where
 *     P_s is the shell density spectrum of x_T at t_T (as
 *     cf_density_spectrum_s2 + cf_s2_to_shells); sets dL/dx_T as the adjoint seed.
 *   cf_adjoint_set_lambda: sets the seed dL/dx_T (FP64 2N^3, device) directly, with the
 *     part of dL/dm not carried by the state.
 *   cf_adjoint_backward: reverse sweep (recomputing each segment from its checkpoint):
 *     dL/dx_0 -> d_lambda0 (FP64 2N^3, device; may be NULL), dL/dm -> *h_dL_dm.
 * Initial-field parameterisation by shell groups (group g holds unit shells
 * [g*spg, (g+1)*spg), the last group everything beyond):
 *   phi0 = c2r(sqrt(theta_g(k)) sqrtP(s^2) xi_k), xi an HC array, sqrtP indexed by s^2;
 *   cf_shell_amplitude_gradient: dL/dtheta_g from dL/dphi0 (N^3 device, FP64). */
typedef struct cf_adjoint cf_adjoint;
int cf_adjoint_create(cf_ctx *ctx, int64_t nsteps, int64_t checkpoint_every, cf_adjoint **out);
int cf_adjoint_destroy(cf_adjoint *adj);
int cf_adjoint_forward(cf_adjoint *adj, void *d_state, double t0, double dt, void *stream);
int cf_adjoint_shell_log_loss(cf_adjoint *adj, const void *d_state, const double *h_target_shells,
                              double rel_floor, double *h_loss, void *stream);
int cf_adjoint_set_lambda(cf_adjoint *adj, const double *d_lambda, double dL_dm_direct, void *stream);
int cf_adjoint_backward(cf_adjoint *adj, double *d_lambda0, double *h_dL_dm, void *stream);
int cf_field_from_shell_amplitudes(cf_ctx *ctx, const double *d_xi_hc, const double *d_sqrtP_s2,
                                   const double *h_theta, int ngroups, int shells_per_group, double *d_phi,
                                   void *stream);
int cf_shell_amplitude_gradient(cf_ctx *ctx, const double *d_lambda_phi, const double *d_xi_hc,
                                const double *d_sqrtP_s2, const double *h_theta, int ngroups,
                                int shells_per_group, double *h_grad, void *stream);

/* ---- ensembles ------------------------------------------------------------------
 * Independent CF_EQ_KG / CF_EQ_KG_FRW lattices of uneven N (each N % 8 == 0,
 * N <= 1024) sharing equation, precision, stencil, cosmology and time grid,
 * advanced together.  No reference counterpart: the reference runs one lattice
 * per process (src/main.cpp:82-196).
 *   CF_ENS_PERSISTENT: one cooperative kernel for all nsteps (grid barriers between
 *     stages; a barrier that waits too long returns CF_ERR_TIMEOUT, never hangs).
 *   CF_ENS_BATCHED: the passes of cf_rk4_steps over all members: one whole-step
 *     launch per step (7-point), two paired-stage launches per step (13-point:
 *     stages 1+2, 3+4).
 *   CF_ENS_LOOP: the same passes, one launch per member (single-instance path).
 * cf_ensemble_run_graph: nsegments observer intervals of steps_per_segment steps from
 *   t0 (absolute steps 0..): a CUDA graph of one interval -- the persistent kernel
 *   (mode CF_ENS_PERSISTENT) or the batched launches of steps_per_segment steps (mode
 *   CF_ENS_BATCHED), each reading its step from a device counter that the graph
 *   advances -- is captured once and replayed per segment; when d_spectra is non-NULL the members' density
 *   spectra (S2 bins, concatenated member by member, cf_ensemble_info gives the
 *   per-segment length) at each segment end follow each replay.  Needs a
 *   non-default stream.
 * cf_ensemble_autotune: times tile shapes and a-chunk lengths on the members
 *   (of the whole-step work list for the 7-point stencil, of the paired-stage /
 *   persistent one for the 13-point; overwrites their states: tune before
 *   uploading initial data). cf_ensemble_info's work_items counts the items of the
 *   batched schedule. */
typedef enum cf_ens_mode { CF_ENS_PERSISTENT = 0, CF_ENS_BATCHED = 1, CF_ENS_LOOP = 2 } cf_ens_mode;
typedef struct cf_ensemble cf_ensemble;
int cf_ensemble_create(const cf_params *members, int count, cf_ensemble **out);
int cf_ensemble_destroy(cf_ensemble *ens);
int cf_ensemble_info(const cf_ensemble *ens, int64_t *spectra_total, int64_t *work_items);
int64_t cf_ensemble_launch_count(const cf_ensemble *ens);
int cf_ensemble_state_upload(cf_ensemble *ens, int member, const double *h_xy, void *stream);
int cf_ensemble_state_download(cf_ensemble *ens, int member, double *h_xy, void *stream);
int cf_ensemble_rk4_steps(cf_ensemble *ens, double t0, double dt, int64_t step0, int64_t nsteps, int mode,
                          void *stream);
int cf_ensemble_density_spectra_s2(cf_ensemble *ens, double t, double *d_out, void *stream);
int cf_ensemble_run_graph(cf_ensemble *ens, double t0, double dt, int64_t steps_per_segment, int64_t nsegments,
                          int mode, double *d_spectra, void *stream);
int cf_ensemble_autotune(cf_ensemble *ens, double t0, double dt, int64_t steps, void *stream, int *h_shape,
                         int *h_a_chunk);
/* Failure-detection test hook: the persistent kernel's grid barrier waits for
 * `extra_arrivals` CTAs that never come, giving up after `spin_limit` sleep
 * iterations (default 2^24).  The run then returns CF_ERR_TIMEOUT with the
 * state untouched (stage 1 writes only work buffers) and the ensemble stays
 * usable; (0, 2^24) restores normal operation. */
int cf_ensemble_set_barrier_test(cf_ensemble *ens, int extra_arrivals, int64_t spin_limit);

/* ---- profiling ----------------------------------------------------------------
 * When enabled, every kernel (or cuFFT call) the context launches is bracketed by
 * a pair of CUDA events on its stream and its device time is accumulated per
 * kind.  cf_profile_read synchronises on the recorded events. */
typedef enum cf_prof_kind {
  CF_PROF_STAGE1 = 0,  /* RK4 stage kernels 1..4 */
  CF_PROF_STAGE2 = 1,
  CF_PROF_STAGE3 = 2,
  CF_PROF_STAGE4 = 3,
  CF_PROF_PSI_TRANSFER = 4, /* Psi / dPsi transfer-function kernel */
  CF_PROF_PSI_FFT = 5,      /* batched C2R of Psi / dPsi (cuFFT) */
  CF_PROF_SPECTRUM = 6,     /* energy density, R2C, binning */
  CF_PROF_OTHER = 7,
  CF_PROF_PAIR_A = 8,       /* paired-stage passes: stages 1+2, stages 3+4 */
  CF_PROF_PAIR_B = 9,
  CF_PROF_STEP = 10,        /* whole-step pass (all four stages) */
  CF_PROF_KINDS = 11
} cf_prof_kind;

typedef struct cf_profile {
  int64_t launches[CF_PROF_KINDS];
  double ms[CF_PROF_KINDS];
} cf_profile;

int cf_profile_enable(cf_ctx *ctx, int on);
int cf_profile_read(cf_ctx *ctx, cf_profile *out);
int cf_profile_reset(cf_ctx *ctx);

#ifdef __cplusplus
}
#endif

#endif /* CFB200_H */
