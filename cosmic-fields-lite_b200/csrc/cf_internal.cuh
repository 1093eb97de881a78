// cf_internal.cuh -- shared definitions of libcfb200 (context, errors, helpers).
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "cfb200.h"

namespace cfb {

// Thread-local last error message (cf_last_error()).
void set_error(const char *fmt, ...);
const char *get_error();

#define CF_TRY_CUDA(expr)                                                                      \
  do {                                                                                         \
    cudaError_t e_ = (expr);                                                                   \
    if (e_ != cudaSuccess) {                                                                   \
      ::cfb::set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
      return CF_ERR_CUDA;                                                                      \
    }                                                                                          \
  } while (0)

#define CF_TRY_CUFFT(expr)                                                                     \
  do {                                                                                         \
    cufftResult r_ = (expr);                                                                   \
    if (r_ != CUFFT_SUCCESS) {                                                                 \
      ::cfb::set_error("%s failed: cufftResult %d (%s:%d)", #expr, (int)r_, __FILE__, __LINE__); \
      return CF_ERR_CUFFT;                                                                     \
    }                                                                                          \
  } while (0)

#define CF_TRY(...)             \
  do {                          \
    int s_ = (__VA_ARGS__);     \
    if (s_ != CF_OK) return s_; \
  } while (0)

// Checks the launch that was just enqueued.
#define CF_LAUNCHED(ctx)                                                                       \
  do {                                                                                         \
    cudaError_t e_ = cudaGetLastError();                                                       \
    if (e_ != cudaSuccess) {                                                                   \
      ::cfb::set_error("kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_), __FILE__, __LINE__); \
      return CF_ERR_CUDA;                                                                      \
    }                                                                                          \
    (ctx)->launches++;                                                                         \
  } while (0)

// One cached Psi / dPsi/dt pair at a stage time (comoving-curvature equation).
struct PsiSlot {
  double t = 0;
  bool valid = false;
  // A second stage time whose refresh would have given these same bits: its pass-A
  // inputs (FP32) were compared with this slot's on the device and found identical.
  double t_alt = 0;
  bool has_alt = false;
  void *psi = nullptr;   // N^3 of the storage type
  void *dpsi = nullptr;  // N^3 of the storage type
  uint64_t stamp = 0;
  cudaEvent_t ready = nullptr;  // recorded after the slot's last refresh, on the stream that ran it
};
// 3 for a step's stage times t, t + dt/2, t + dt and 3 for the next step's, synthesised
// beside it: the next step starts at t0 + (n + 1) dt, which can differ from t + dt in
// the last bit (odeint's integrate_const forms its times the same way)
constexpr int kPsiSlots = 6;

// One cached coarse curvature table at a stage time (approximate comoving
// equation): M^3 x 4 words of the storage type.
struct ApproxSlot {
  double t = 0;
  bool valid = false;
  void *tab = nullptr;
  uint64_t stamp = 0;
};

}  // namespace cfb

struct cf_ctx {
  cf_params p;
  int64_t N = 0, N3 = 0, nh = 0, hc_count = 0, s2_bins = 0, shells = 0;
  int device = 0;
  int64_t launches = 0;
  size_t word = 8;  // bytes of the storage type (8 FP64, 4 FP32_COMP)

  // RK4 temporaries (storage type): acc and ping-pong stage inputs, 2N^3 words each.
  void *acc = nullptr, *ya = nullptr, *yb = nullptr;

  // Comoving curvature: R_fft in the storage type's complex HC, the transfer
  // outputs (2 HC arrays) and the cached (Psi, dPsi) slots: three allocated with the
  // buffers, three more when cf_rk4_steps first synthesises the next step's slots on
  // the side stream while a step runs (psi_pipe_*).
  void *R_fft = nullptr;
  void *psi_hc = nullptr;  // 2 consecutive HC arrays (Psi_k, dPsi_k), storage type
  double *psi_table = nullptr;  // (T_Psi, T_dPsi) per s^2
  cfb::PsiSlot slot[cfb::kPsiSlots];
  int slots_alloc = 0;
  uint64_t slot_clock = 0;
  cudaStream_t psi_side = nullptr;  // refreshes that overlap the stepping
  cudaEvent_t psi_fork = nullptr, psi_join = nullptr, psi_stepdone = nullptr;
  cufftHandle plan_psi = 0;  // batched (2) C2R/Z2D into dense N^3
  bool have_plan_psi = false;
  // Pruned synthesis when R_fft is exactly zero outside |i|, |j| <= Ka, Kb and
  // k <= Kc (cf_psi.cu): three 1-D passes over the support only.
  bool pruned = false;
  int Ka = -1, Kb = -1, Kc = -1;
  int pr_Ka = -1, pr_Kb = -1, pr_Kc = -1;  // box the pruned plans / buffers were built for
  // pz_a: pass A's input lines, zero outside the band (written once) and the band
  // entries of the latest refresh; pz_a2: their C2C along a (out of place)
  void *pz_a = nullptr, *pz_a2 = nullptr, *pz_b = nullptr;
  cufftHandle plan_pa = 0, plan_pb = 0, plan_pc = 0;
  bool have_pruned = false;
  // Pass C as one kernel (power-of-two N, 32..2048): twiddles e^{2 pi i j / N},
  // j < N, in the storage complex type; no padded HC rows, no C2R plan.
  bool pc_fused = false;
  void *pr_wN = nullptr;
  void *pr_twM = nullptr;  // pass-1 twiddles e^{2 pi i k2 m1 / (N/2)}, [m1][k2]
  // The warp pass C's band tiles by TMA: a tensor map over pass B's lines (a
  // CUtensorMap, 64-byte aligned, encoded when the pruned buffers are made), and a
  // mapped host word its bounded waits set when they give up (read on the host
  // without a synchronisation at the next refresh).
  alignas(64) unsigned char pc_tmap[128] = {};
  bool have_pc_tmap = false;
  int *psi_err_h = nullptr, *psi_err_d = nullptr;
  long long pc_spin_limit = 1LL << 20;  // tests per bounded wait (cf_psi_set_wait_test)
  int pc_tx_extra = 0;                  // bytes armed beyond each box (cf_psi_set_wait_test)
  // Pruned synthesis: pz_a holds the band of pass A's inputs (R_k times the transfer
  // factors) of the latest refresh, at time pa_last_t; an FP32 refresh for a time a few
  // ulp away compares its inputs with them (a mapped host word records a difference)
  // and, when they are identical, takes the slot of pa_last_t instead of synthesising
  // the same bits again.
  bool pa_last_valid = false;
  double pa_last_t = 0;
  int *pa_diff_h = nullptr, *pa_diff_d = nullptr;
  cudaEvent_t pa_check = nullptr;
  int64_t psi_refreshes = 0, psi_reuses = 0;  // cf_psi_stats
  // Pass B as one kernel (FP32, power-of-two N, 32..1024): its four-step twiddles
  // e^{2 pi i k2 m1 / N}, [m1][k2]; no plan_pb then.
  bool pb_fused = false;
  void *pr_twB = nullptr;

  // Fixed curvature: e^{2 Psi(x)} - 1 of cf_set_psi, N^3 of the storage type.
  void *fixed_e2m1 = nullptr;

  // Approximate comoving curvature (cf_approx.cu): the M-grid modes of R_fft,
  // the transfer outputs, the synthesised fields, the lattice-to-coarse index
  // map and three cached coarse tables.
  double *ap_R = nullptr;   // M-grid HC, FP64
  double *ap_hc = nullptr;  // 2 M-grid HC arrays (Psi_k, dPsi_k), FP64
  double *ap_f = nullptr;   // 2 M^3 fields (Psi, dPsi/dt), FP64
  int *ap_cmap = nullptr;   // N ints: ((i + (N/M)/2) % N) / (N/M)
  cfb::ApproxSlot ap_slot[3];
  uint64_t ap_clock = 0;
  cufftHandle plan_ap = 0;  // batched (2) Z2D on M^3
  bool have_plan_ap = false;

  // Spectra: FP64 R2C plans and scratch.
  cufftHandle plan_d2z1 = 0, plan_d2z2 = 0;
  bool have_d2z1 = false, have_d2z2 = false;
  double *spec_hc = nullptr;    // 2 HC arrays (FP64)
  double *spec_field = nullptr; // N^3 FP64 (energy density scratch)
  // Initial conditions (cf_init.cu): a Z2D plan and the per-s^2 table of the last call.
  cufftHandle plan_z2d1 = 0;
  bool have_z2d1 = false;
  double *ic_table = nullptr;
  unsigned long long *bins = nullptr;   // 2 * s2_bins words: (lo, hi) fixed point
  unsigned long long *maxbits = nullptr;
  long long spec_mult = 0;  // scale multiplier of the last binning (bin_spectrum)
  // Host <-> device transfers of an FP32_COMP state (cf_state_upload / download):
  // two FP64 chunks used in turn, and the event that ends the last transfer.
  double *stage = nullptr;
  cudaEvent_t stage_ev = nullptr;
  bool stage_used = false;
  int64_t *s2_counts = nullptr;

  // Profiling (cf_profile_enable): pending event pairs and per-kind totals.
  bool prof_on = false;
  struct ProfRec {
    int kind;
    cudaEvent_t a, b;
  };
  std::vector<ProfRec> prof_pending;
  std::vector<cudaEvent_t> prof_pool;
  int64_t prof_launches[CF_PROF_KINDS] = {};
  double prof_ms[CF_PROF_KINDS] = {};
};

namespace cfb {

// Lazily allocated scratch.
int ensure_rk4_scratch(cf_ctx *ctx);
int ensure_spectrum_scratch(cf_ctx *ctx, int nfields);
int ensure_psi(cf_ctx *ctx);

// Returns the cached Psi / dPsi/dt slot for stage time t, refreshing one slot
// (transfer kernel + batched C2R on `stream`) if t is not cached.
int psi_at(cf_ctx *ctx, double t, cudaStream_t stream, const void **psi, const void **dpsi);
// Refreshes beside the stepping (comoving-curvature equation).  A stepping loop on
// `stream` forks the side stream (begin; *on = false when the extra slots do not fit,
// and the loop then refreshes in turn), has the slots of a step filled there (fill: a
// no-op for a cached time; the victim is a slot whose time is not in keep[0..nkeep)),
// takes them after their refresh (use: `stream` waits on the slot's event), marks
// each step's kernels done (step_done: later fills wait on it before they overwrite a
// slot that step read) and joins the side stream at the end (end).
int psi_pipe_begin(cf_ctx *ctx, cudaStream_t stream, bool *on);
int psi_pipe_fill(cf_ctx *ctx, double t, const double *keep, int nkeep);
int psi_pipe_use(cf_ctx *ctx, double t, cudaStream_t stream, const void **psi, const void **dpsi);
int psi_pipe_step_done(cf_ctx *ctx, cudaStream_t stream);
int psi_pipe_end(cf_ctx *ctx, cudaStream_t stream);
// Psi and dPsi at t, widened to FP64, into d_out (2 N^3 doubles).
int psi_fields(cf_ctx *ctx, double t, double *d_out, cudaStream_t stream);
// CF_PSI_* route the next Psi refresh takes.
int psi_route(const cf_ctx *ctx);
// Approximate comoving equation: takes the M-grid modes of a new R_fft (FP64,
// device), and returns the coarse table for stage time t (refreshing one slot).
int approx_set_R(cf_ctx *ctx, const double *d_R_fft, cudaStream_t stream);
int approx_at(cf_ctx *ctx, double t, cudaStream_t stream, const void **tab);
// Frees the fixed and the approximate curvature buffers (context teardown).
void approx_release(cf_ctx *ctx);
// Fixed curvature: Psi (FP64, N^3, host or device) -> e^{2 Psi} - 1 in the storage type.
int set_fixed_psi(cf_ctx *ctx, const double *Psi, int on_device, cudaStream_t stream);
// Frees the pruned-synthesis buffers and plans (context teardown).
void psi_release(cf_ctx *ctx);

// Host-side StaticEOSCosmology (reference src/physics.hpp:34-55), bit-identical
// to the reference's host code: same expressions, same libm.
double cosmo_a(const cf_params &p, double t);
double cosmo_H(const cf_params &p, double t);
double cosmo_eta(const cf_params &p, double t);

// 1/h^2/a(t)^2 and H(t) exactly as the reference host code forms them
// (src/equations.cpp:199-202, src/equations_cuda.cu:526-529).
void stage_coeffs(const cf_params &p, double t, double *inv_ah2, double *H);

inline unsigned ceil_div(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

// Brackets the launches made between begin and end with profiling events
// (no-op unless profiling is on).
struct ProfScope {
  cf_ctx *ctx;
  int kind;
  cudaStream_t st;
  cudaEvent_t a = nullptr;
  ProfScope(cf_ctx *c, int k, cudaStream_t s);
  ~ProfScope();
};

}  // namespace cfb
