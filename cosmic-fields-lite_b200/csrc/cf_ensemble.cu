// cf_ensemble.cu -- ensembles of FRW Klein-Gordon lattices of uneven N advanced
// together.
//
// Every member is an independent lattice (its own N, L, m; a shared
// cosmology, time grid, precision and stencil).  A step of the whole ensemble is
// the same fused RK4 passes as cf_rk4_steps, applied to a work list of (member,
// b-tile, c-tile, a-chunk) items.  Three schedules:
//
//   CF_ENS_PERSISTENT  one cooperative kernel for all steps: each CTA takes work
//                      items from a shared counter -- whole-step items for the
//                      7-point stencil (cf_step_tile.cuh), single-stage items for
//                      the 13-point one (cf_stage_tile.cuh) -- then a grid barrier
//                      (bounded spin: gives up with CF_ERR_TIMEOUT instead of
//                      hanging) before the next step (stage).  Stage coefficients
//                      come from a per-step table in device memory, so a captured
//                      graph replays it.
//   CF_ENS_BATCHED     the passes of cf_rk4_steps over the whole work list: one
//                      whole-step launch per step for the 7-point stencil
//                      (cf_step_tile.cuh), the two paired passes (stages 1+2, 3+4;
//                      cf_pair_tile.cuh) for the 13-point one.
//   CF_ENS_LOOP        the same passes, one launch per member (the single-instance path).
//
// cf_ensemble_run_graph captures one observer interval -- the batched launches
// (or barrier reset + the persistent kernel) for S steps and the advance of a
// device step counter -- in a CUDA graph and replays it once per interval; the
// members' density spectra at each interval end are enqueued on the same stream
// after the replay.
//
// Tile shapes and a-chunk lengths are chosen per size class by cf_ensemble_autotune
// (timing of the candidates on the members themselves).

#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <vector>

#include "cf_internal.cuh"
#include "cf_pair_tile.cuh"
#include "cf_stage_tile.cuh"
#include "cf_step_tile.cuh"

namespace cfb {

struct EnsMember {
  void *x, *acc, *ya, *yb;  // storage type; x holds [hi | lo] in FP32_COMP
  long long N3;
  int N;
  double m2;
  double inv_scale;  // 1 / h^2 (h = L/N); divided by a^2 per stage
};

struct EnsItem {
  int member, c0, b0, a_begin, a_end, shape;
};

struct EnsCoef {
  double a2;     // a(t)^2 of the stage time (inv = (1/h^2) / a^2, the single-lattice order)
  double hub3;   // 3 H(t)
};

struct EnsArgs {
  const EnsMember *members;
  const EnsItem *items;
  int n_items;
  const EnsCoef *coef;      // 4 per step, indexed by absolute step
  const long long *step_counter;  // absolute index of the first step of this launch (device)
  int nsteps;
  double dt;
  unsigned *bar_count;
  unsigned *bar_gen;
  unsigned *work;  // next work item of the current stage (persistent kernel)
  int *err;
  unsigned bar_extra;    // arrivals the barrier waits for beyond the grid (0; > 0 only in failure tests)
  long long spin_limit;  // bounded wait of the barrier, in sleep iterations
};

// Tile shapes compiled for the ensemble kernels (threads along c x along b).
constexpr int ENS_SHAPES = 2;
template <int SHAPE>
struct EnsShape;
template <>
struct EnsShape<0> {
  static constexpr int TX = 8, TY = 32;
};
template <>
struct EnsShape<1> {
  static constexpr int TX = 16, TY = 16;
};

template <typename S, int H, int SHAPE>
__device__ __forceinline__ void ens_item_stage(const EnsArgs &E, const EnsItem &it, int stage, long long step,
                                               S *sm) {
  constexpr int TXv = EnsShape<SHAPE>::TX, TYv = EnsShape<SHAPE>::TY;
  const EnsMember mb = E.members[it.member];
  StageArgs<S> A;
  A.N = mb.N;
  A.N3 = mb.N3;
  A.m2 = mb.m2;
  A.x = (S *)mb.x;
  A.xlo = (sizeof(S) == 4) ? (S *)mb.x + 2 * mb.N3 : nullptr;
  A.acc = (S *)mb.acc;
  A.psi = A.dpsi = nullptr;
  A.cmap = nullptr;
  A.M = 0;
  A.q1 = A.q2 = 0.0;
  A.a_chunk = 0;
  const EnsCoef cf = E.coef[4 * step + stage - 1];
  A.inv = mb.inv_scale / cf.a2;
  A.hub3 = cf.hub3;
  A.dt6 = E.dt / 6.0;
  switch (stage) {
    case 1:
      A.yin = (const S *)mb.x;
      A.yout = (S *)mb.ya;
      A.cy = E.dt / 2.0;
      stage_tile<S, H, EQ_FRW, 1, TXv, TYv>(A, it.c0, it.b0, it.a_begin, it.a_end, sm);
      break;
    case 2:
      A.yin = (const S *)mb.ya;
      A.yout = (S *)mb.yb;
      A.cy = E.dt / 2.0;
      stage_tile<S, H, EQ_FRW, 2, TXv, TYv>(A, it.c0, it.b0, it.a_begin, it.a_end, sm);
      break;
    case 3:
      A.yin = (const S *)mb.yb;
      A.yout = (S *)mb.ya;
      A.cy = E.dt;
      stage_tile<S, H, EQ_FRW, 3, TXv, TYv>(A, it.c0, it.b0, it.a_begin, it.a_end, sm);
      break;
    default:
      A.yin = (const S *)mb.ya;
      A.yout = nullptr;
      stage_tile<S, H, EQ_FRW, 4, TXv, TYv>(A, it.c0, it.b0, it.a_begin, it.a_end, sm);
      break;
  }
}

// Grid-wide barrier with a bounded spin.  Returns false (and sets *err) if the
// other CTAs did not arrive within the limit; all CTAs are co-resident under a
// cooperative launch, so this only trips if that guarantee is violated.
__device__ __forceinline__ bool grid_barrier(const EnsArgs &E) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    ok = 1;
    volatile unsigned *gen = E.bar_gen;
    const unsigned g = *gen;
    __threadfence();
    const unsigned arrived = atomicAdd(E.bar_count, 1u) + 1u;
    if (arrived == gridDim.x + E.bar_extra) {
      *E.bar_count = 0u;
      *E.work = 0u;  // every CTA has left the stage's fetch loop
      __threadfence();
      atomicAdd((unsigned *)E.bar_gen, 1u);
    } else {
      long long spins = 0;
      while (*gen == g) {
        if (*(volatile int *)E.err) {
          ok = 0;
          break;
        }
        if (++spins > E.spin_limit) {  // default 2^24: seconds with the sleep below
          atomicExch(E.err, 1);
          ok = 0;
          break;
        }
        __nanosleep(128);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

// Resident CTAs per SM that the ensemble kernels' register allocation must
// allow (persistent kernel, paired-stage kernels).  Uncapped, the persistent
// kernel, which inlines all four stages, takes ~180 registers in FP32: one CTA
// per SM.  Measured on B200, 96 FRW lattices 32 x {64,96,128}^3, FP32-comp
// 7-point, single-stage tiles (G site-updates/s, batched / persistent graph):
//   caps 1/1: 17.6 / 17.2;  2/2: 28.9 / 26.3;  3/3: 33.9 / 24.8 (persistent spills).
#ifndef CF_ENS_PERSIST_MIN_BLOCKS
#define CF_ENS_PERSIST_MIN_BLOCKS 2
#endif
#ifndef CF_ENS_PAIR_MIN_BLOCKS
#define CF_ENS_PAIR_MIN_BLOCKS 3
#endif

// One stage of the persistent kernel: CTAs take work items from a shared
// counter (the items differ in cost: edge tiles, a-chunk remainders), then meet
// at the grid barrier, whose last arrival resets the counter.
template <typename S, int H, int SHAPE>
__device__ __forceinline__ bool ens_stage_pass(const EnsArgs &E, int stage, long long step, S *sm) {
  __shared__ int next;
  for (;;) {
    if (threadIdx.x == 0 && threadIdx.y == 0) next = (int)atomicAdd(E.work, 1u);
    __syncthreads();
    const int i = next;
    if (i >= E.n_items) break;
    // stage_tile synchronises the CTA before it returns, so `next` is read by
    // all threads before thread 0 overwrites it
    ens_item_stage<S, H, SHAPE>(E, E.items[i], stage, step, sm);
  }
  return grid_barrier(E);
}

template <typename S, int H, int SHAPE>
__global__ void __launch_bounds__(256, CF_ENS_PERSIST_MIN_BLOCKS) k_ens_persistent(const EnsArgs E) {
  constexpr int TXv = EnsShape<SHAPE>::TX, TYv = EnsShape<SHAPE>::TY;
  __shared__ __align__(16) S sm[TileSmem<S, H, TXv, TYv>::count];
  const long long step0 = *E.step_counter;
  for (int j = 0; j < E.nsteps; ++j) {
    for (int stage = 1; stage <= 4; ++stage)
      if (!ens_stage_pass<S, H, SHAPE>(E, stage, step0 + j, sm)) return;
  }
}

// Paired-stage pass PASS (1: stages 1+2, 2: stages 3+4) of one work item, as
// rk4_steps' paired route with the same coefficients.  Within a run, step j keeps
// phi in x for even j and in the first half of ya for odd j (pass B writes the
// other one); a run of odd length ends with k_ens_phi_back.
template <typename S, int H, int SHAPE, int PASS>
__device__ __forceinline__ void ens_item_pair(const EnsArgs &E, const EnsItem &it, long long step, bool odd, S *sm) {
  constexpr int TXv = EnsShape<SHAPE>::TX, TYv = EnsShape<SHAPE>::TY;
  const EnsMember mb = E.members[it.member];
  S *x = (S *)mb.x, *ya = (S *)mb.ya, *yb = (S *)mb.yb;
  S *phi_cur = odd ? ya : x, *phi_nxt = odd ? x : ya;
  PairArgs<S> A;
  A.N = mb.N;
  A.N3 = mb.N3;
  A.m2 = mb.m2;
  A.a_chunk = 0;
  A.xphi = phi_cur;
  A.xpi = x + mb.N3;
  A.xlo = (sizeof(S) == 4) ? x + 2 * mb.N3 : nullptr;
  A.acc = (S *)mb.acc;
  A.yb = yb;
  A.psi1 = A.dpsi1 = A.psi2 = A.dpsi2 = nullptr;
  A.cmap = nullptr;
  A.M = 0;
  A.q1 = A.q2 = 0.0;
  const EnsCoef c1 = E.coef[4 * step + (PASS == 1 ? 0 : 2)];
  const EnsCoef c2 = E.coef[4 * step + (PASS == 1 ? 1 : 3)];
  A.inv1 = mb.inv_scale / c1.a2;
  A.hub3_1 = c1.hub3;
  A.inv2 = mb.inv_scale / c2.a2;
  A.hub3_2 = c2.hub3;
  A.dt6 = E.dt / 6.0;
  if constexpr (PASS == 1) {
    A.uphi = phi_cur;
    A.upi = x + mb.N3;
    A.xphi_out = nullptr;
    A.cw = E.dt / 2.0;
    A.cy = E.dt / 2.0;
  } else {
    A.uphi = yb;
    A.upi = yb + mb.N3;
    A.xphi_out = phi_nxt;
    A.cw = E.dt;
    A.cy = 0.0;
  }
  pair_tile<S, H, EQ_FRW, PASS, TXv, TYv>(A, it.c0, it.b0, it.a_begin, it.a_end, sm);
}

template <typename S, int H, int SHAPE, int PASS>
__global__ void __launch_bounds__(256, CF_ENS_PAIR_MIN_BLOCKS) k_ens_pair(const EnsArgs E, int step_off) {
  constexpr int TXv = EnsShape<SHAPE>::TX, TYv = EnsShape<SHAPE>::TY;
  __shared__ __align__(16) S sm[PairSmem<S, H, TXv, TYv>::count];
  ens_item_pair<S, H, SHAPE, PASS>(E, E.items[blockIdx.x], *E.step_counter + step_off, (step_off & 1) != 0, sm);
}

// phi back from ya to x over one work item's sites (after a run of odd length).
template <typename S, int SHAPE>
__global__ void __launch_bounds__(256) k_ens_phi_back(const EnsArgs E) {
  constexpr int TXv = EnsShape<SHAPE>::TX;
  constexpr int V = VecT<S>::n, TW = TXv * V;
  const EnsItem it = E.items[blockIdx.x];
  const EnsMember mb = E.members[it.member];
  const int N = mb.N;
  const int c = it.c0 + threadIdx.x * V, b = it.b0 + threadIdx.y;
  if (threadIdx.x * V >= min(TW, N - it.c0) || b >= N) return;
  const long long NN = (long long)N * N;
  for (int a = it.a_begin; a < it.a_end; ++a) {
    const long long site = NN * a + (long long)N * b + c;
    stv((S *)mb.x + site, ldv((const S *)mb.ya + site));
  }
}

__global__ void k_counter_add(long long *c, long long v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *c += v;
}

// Whole-step tiles of the 7-point ensembles (threads along c x along b, CTAs/SM):
// shape 0 is cf_rk4_steps' own (FP32 128 x 8 sites, FP64 32 x 8), shape 1 a
// narrower, taller tile for members whose N is not a multiple of the wide one
// (FP32 64 x 16, FP64 16 x 16).
constexpr int ENS_STEP_SHAPES = 2;
template <typename S, int SS>
struct EnsStepShape;
template <>
struct EnsStepShape<float, 0> {
  static constexpr int TX = 32, TY = 8, MB = 2;
};
template <>
struct EnsStepShape<float, 1> {
  static constexpr int TX = 16, TY = 16, MB = 2;
};
template <>
struct EnsStepShape<double, 0> {
  static constexpr int TX = 16, TY = 8, MB = 3;
};
template <>
struct EnsStepShape<double, 1> {
  static constexpr int TX = 8, TY = 16, MB = 3;
};
template <typename S, int SS>
constexpr size_t ens_step_smem() {
  return (size_t)StepSmem<S, EnsStepShape<S, SS>::TX, EnsStepShape<S, SS>::TY>::count * sizeof(S);
}

// One RK4 step of one work item as cf_rk4_steps' whole-step pass, with the same
// coefficients (1/h^2 / a^2 and 3H at t, t + dt/2, t + dt from the step table).
// Within a run, step j reads phi, pi from x for even j and from ya for odd j and
// writes the other buffer; the lo words stay in x; a run of odd length ends with
// k_ens_xy_back.
template <typename S, int SS>
__device__ __forceinline__ void ens_step_item(const EnsArgs &E, const EnsItem &it, long long step, int step_off,
                                              S *sm) {
  using SH = EnsStepShape<S, SS>;
  const EnsMember mb = E.members[it.member];
  S *x = (S *)mb.x, *ya = (S *)mb.ya;
  S *cur = (step_off & 1) ? ya : x, *nxt = (step_off & 1) ? x : ya;
  StepArgs<S> A{};
  A.xphi = cur;
  A.xpi = cur + mb.N3;
  A.ophi = nxt;
  A.opi = nxt + mb.N3;
  A.xlo = (sizeof(S) == 4) ? x + 2 * mb.N3 : nullptr;
  A.N = mb.N;
  A.N3 = mb.N3;
  A.m2 = mb.m2;
  const int idx[3] = {0, 1, 3};  // stage times t, t + dt/2, t + dt
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const EnsCoef c = E.coef[4 * step + idx[k]];
    A.inv[k] = mb.inv_scale / c.a2;
    A.hub3[k] = c.hub3;
  }
  A.dt2 = E.dt / 2.0;
  A.dt = E.dt;
  A.dt6 = E.dt / 6.0;
  step_tile<S, EQ_FRW, SH::TX, SH::TY, false>(A, it.c0, it.b0, it.a_begin, it.a_end, sm);
}

template <typename S, int SS>
__global__ void __launch_bounds__(EnsStepShape<S, SS>::TX *EnsStepShape<S, SS>::TY, EnsStepShape<S, SS>::MB)
    k_ens_step(const EnsArgs E, int step_off) {
  extern __shared__ __align__(16) unsigned char ens_step_sm[];
  ens_step_item<S, SS>(E, E.items[blockIdx.x], *E.step_counter + step_off, step_off,
                       reinterpret_cast<S *>(ens_step_sm));
}

// phi and pi back from ya to x over one whole-step work item's sites.
template <typename S, int SS>
__device__ __forceinline__ void ens_xy_back_item(const EnsArgs &E, const EnsItem &it) {
  constexpr int V = VecT<S>::n, TW = EnsStepShape<S, SS>::TX * V;
  const EnsMember mb = E.members[it.member];
  const int N = mb.N;
  const int c = it.c0 + threadIdx.x * V, b = it.b0 + threadIdx.y;
  if (threadIdx.x * V >= min(TW, N - it.c0) || b >= N) return;
  const long long NN = (long long)N * N;
  for (int a = it.a_begin; a < it.a_end; ++a) {
    const long long site = NN * a + (long long)N * b + c;
    stv((S *)mb.x + site, ldv((const S *)mb.ya + site));
    stv((S *)mb.x + mb.N3 + site, ldv((const S *)mb.ya + mb.N3 + site));
  }
}

template <typename S, int SS>
__global__ void __launch_bounds__(EnsStepShape<S, SS>::TX *EnsStepShape<S, SS>::TY) k_ens_xy_back(const EnsArgs E) {
  ens_xy_back_item<S, SS>(E, E.items[blockIdx.x]);
}

// The persistent form of the 7-point ensemble step (CF_ENS_PERSISTENT): one
// cooperative launch for all steps, CTAs taking whole-step work items from a shared
// counter (the items differ in cost: edge tiles, a-chunk remainders) and meeting at
// one bounded grid barrier per RK4 step -- every item of step j reads the buffer the
// items of step j - 1 wrote; a run of odd length ends with phi, pi back in x.
template <typename S, int SS>
__global__ void __launch_bounds__(EnsStepShape<S, SS>::TX *EnsStepShape<S, SS>::TY, EnsStepShape<S, SS>::MB)
    k_ens_persistent_step(const EnsArgs E) {
  extern __shared__ __align__(16) unsigned char ens_step_sm[];
  __shared__ int next;
  const long long step0 = *E.step_counter;
  for (int j = 0; j < E.nsteps; ++j) {
    for (;;) {
      if (threadIdx.x == 0 && threadIdx.y == 0) next = (int)atomicAdd(E.work, 1u);
      __syncthreads();
      const int i = next;
      if (i >= E.n_items) break;
      // step_tile synchronises the CTA before it returns, so every thread has read
      // `next` before thread 0 overwrites it
      ens_step_item<S, SS>(E, E.items[i], step0 + j, j, reinterpret_cast<S *>(ens_step_sm));
    }
    if (!grid_barrier(E)) return;
  }
  if (E.nsteps & 1) {
    for (;;) {
      if (threadIdx.x == 0 && threadIdx.y == 0) next = (int)atomicAdd(E.work, 1u);
      __syncthreads();
      const int i = next;
      if (i >= E.n_items) break;
      ens_xy_back_item<S, SS>(E, E.items[i]);
      __syncthreads();
    }
  }
}

// Batched energy density of the members of one size class (blockIdx.y = member in class).
template <typename S>
__global__ void k_ens_energy(const EnsMember *members, const int *class_members, double *rho, int N, double a2) {
  const EnsMember mb = members[class_members[blockIdx.y]];
  const long long N3 = mb.N3, NN = (long long)N * N;
  const S *x = (const S *)mb.x;
  const S *xlo = (sizeof(S) == 4) ? x + 2 * N3 : nullptr;
  double *out = rho + (long long)blockIdx.y * N3;
  const double inv = mb.inv_scale / a2;
  auto phi = [&](long long i) -> double { return (double)x[i] + (xlo ? (double)xlo[i] : 0.0); };
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N3; i += stride) {
    const int c = (int)(i % N), b = (int)((i / N) % N), a = (int)(i / NN);
    const double dx = phi(NN * ((a + 1) % N) + (long long)N * b + c) - phi(NN * ((a + N - 1) % N) + (long long)N * b + c);
    const double dy = phi(NN * a + (long long)N * ((b + 1) % N) + c) - phi(NN * a + (long long)N * ((b + N - 1) % N) + c);
    const double dz = phi(NN * a + (long long)N * b + (c + 1) % N) - phi(NN * a + (long long)N * b + (c + N - 1) % N);
    const double f = phi(i);
    const double p = (double)x[N3 + i] + (xlo ? (double)xlo[N3 + i] : 0.0);
    out[i] = 0.5 * (p * p + mb.m2 * f * f + 0.25 * inv * (dx * dx + dy * dy + dz * dz));
  }
}

// batched binning (blockIdx.y = batch entry), same fixed-point scheme as cf_spectrum.cu
int bin_batched(const double *hc, int N, int batch, unsigned long long *maxbits, unsigned long long *bins,
                double *out, long long nb, cudaStream_t st, cf_ctx *ctx);

}  // namespace cfb

struct cf_ensemble {
  cf_params base{};
  int count = 0;
  int precision = CF_FP64;
  int stencil = 7;
  size_t word = 8;
  std::vector<cf_params> p;
  std::vector<cfb::EnsMember> hm;
  cfb::EnsMember *dm = nullptr;
  std::vector<void *> allocs;
  // work list (per schedule; rebuilt by the autotuner)
  std::vector<cfb::EnsItem> items;
  cfb::EnsItem *d_items = nullptr;
  std::map<int, std::pair<int, int>> tune;  // N -> (shape, a_chunk)
  int shape = 0;                            // shape used by the persistent kernel
  // whole-step work list of the 7-point batched and loop schedules
  std::vector<cfb::EnsItem> sitems;
  cfb::EnsItem *d_sitems = nullptr;
  int sshape = 0, schunk = 32;
  // time table
  cfb::EnsCoef *d_coef = nullptr;
  long long coef_cap = 0;
  double coef_t0 = 0, coef_dt = 0;
  long long *d_step = nullptr;
  unsigned *d_bar = nullptr;  // count, gen, work
  int *d_err = nullptr;
  // spectra per size class
  struct Cls {
    int N;
    std::vector<int> members;
    int *d_members = nullptr;
    double *rho = nullptr, *hc = nullptr;
    cufftHandle plan = 0;
    bool have_plan = false;
  };
  std::vector<Cls> classes;
  unsigned long long *d_max = nullptr, *d_bins = nullptr;
  long long max_bins = 0;
  std::vector<long long> out_offset;  // per member offset into the concatenated spectra
  long long out_total = 0;
  // graph
  cudaGraphExec_t gexec = nullptr;
  long long g_steps = 0;
  double g_t0 = 0, g_dt = 0;
  double *g_out = nullptr;
  int g_mode = -1;
  int64_t g_kernels = 0;  // kernels in one replay of the graph
  bool graph_failed = false;  // capture of the cooperative launch unavailable on this driver
  unsigned bar_extra = 0;
  long long spin_limit = 1LL << 24;
  int64_t launches = 0;
  int coop_blocks = 0;
  int coop_blocks_step = 0;  // resident CTAs of the persistent whole-step kernel
};

namespace cfb {

static int ens_fail(const char *msg) {
  set_error("%s", msg);
  return CF_ERR_INVALID;
}

static void build_items(cf_ensemble *E) {
  E->items.clear();
  for (int i = 0; i < E->count; ++i) {
    const int N = E->hm[i].N;
    auto tn = E->tune.count(N) ? E->tune[N] : std::make_pair(E->shape, 16);
    const int shape = E->shape;  // one kernel instantiation per launch
    const int TX = shape == 0 ? EnsShape<0>::TX : EnsShape<1>::TX;
    const int TY = shape == 0 ? EnsShape<0>::TY : EnsShape<1>::TY;
    const int TW = TX * (E->word == 4 ? VecT<float>::n : VecT<double>::n);
    const int ach = tn.second;
    for (int a = 0; a < N; a += ach)
      for (int b = 0; b < N; b += TY)
        for (int c = 0; c < N; c += TW) E->items.push_back({i, c, b, a, std::min(a + ach, N), shape});
  }
  // largest lattices first: better balance of the round-robin
  std::stable_sort(E->items.begin(), E->items.end(),
                   [&](const EnsItem &x, const EnsItem &y) { return E->hm[x.member].N > E->hm[y.member].N; });
}

static int upload_items(cf_ensemble *E) {
  cudaFree(E->d_items);
  E->d_items = nullptr;
  CF_TRY_CUDA(cudaMalloc(&E->d_items, sizeof(EnsItem) * E->items.size()));
  CF_TRY_CUDA(cudaMemcpy(E->d_items, E->items.data(), sizeof(EnsItem) * E->items.size(), cudaMemcpyHostToDevice));
  return CF_OK;
}

// Whole-step items: tiles of step shape E->sshape, a-chunks of E->schunk planes;
// the CTA shared memory of that shape is allowed above 48 KB here (before any capture).
template <typename S, int SS>
static int step_items_t(cf_ensemble *E) {
  using SH = EnsStepShape<S, SS>;
  constexpr int TW = SH::TX * VecT<S>::n;
  E->sitems.clear();
  for (int i = 0; i < E->count; ++i) {
    const int N = E->hm[i].N;
    for (int a = 0; a < N; a += E->schunk)
      for (int b = 0; b < N; b += SH::TY)
        for (int c = 0; c < N; c += TW) E->sitems.push_back({i, c, b, a, std::min(a + E->schunk, N), SS});
  }
  std::stable_sort(E->sitems.begin(), E->sitems.end(),
                   [&](const EnsItem &x, const EnsItem &y) { return E->hm[x.member].N > E->hm[y.member].N; });
  CF_TRY_CUDA(cudaFuncSetAttribute(k_ens_step<S, SS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)ens_step_smem<S, SS>()));
  CF_TRY_CUDA(cudaFuncSetAttribute(k_ens_persistent_step<S, SS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)ens_step_smem<S, SS>()));
  E->coop_blocks_step = 0;
  cudaFree(E->d_sitems);
  E->d_sitems = nullptr;
  CF_TRY_CUDA(cudaMalloc(&E->d_sitems, sizeof(EnsItem) * E->sitems.size()));
  CF_TRY_CUDA(cudaMemcpy(E->d_sitems, E->sitems.data(), sizeof(EnsItem) * E->sitems.size(), cudaMemcpyHostToDevice));
  return CF_OK;
}

static int build_step_items(cf_ensemble *E) {
  if (E->stencil != 7) return CF_OK;
  if (E->word == 4) return E->sshape ? step_items_t<float, 1>(E) : step_items_t<float, 0>(E);
  return E->sshape ? step_items_t<double, 1>(E) : step_items_t<double, 0>(E);
}

static int ensure_coef(cf_ensemble *E, double t0, double dt, long long nsteps_total, cudaStream_t st) {
  if (E->d_coef && E->coef_cap >= nsteps_total && E->coef_t0 == t0 && E->coef_dt == dt) return CF_OK;
  std::vector<EnsCoef> h((size_t)(4 * nsteps_total));
  cf_params q = E->base;
  for (long long n = 0; n < nsteps_total; ++n) {
    const double t = t0 + (double)n * dt, dh = dt / 2.0;
    const double ts[4] = {t, t + dh, t + dh, t + dt};
    for (int s = 0; s < 4; ++s) {
      if (q.equation == CF_EQ_KG) {
        h[4 * n + s].a2 = 1.0;
        h[4 * n + s].hub3 = 0.0;
      } else {
        const double a = cosmo_a(q, ts[s]);
        h[4 * n + s].a2 = a * a;
        h[4 * n + s].hub3 = 3.0 * cosmo_H(q, ts[s]);
      }
    }
  }
  cudaFree(E->d_coef);
  E->d_coef = nullptr;
  CF_TRY_CUDA(cudaMalloc(&E->d_coef, sizeof(EnsCoef) * h.size()));
  CF_TRY_CUDA(cudaMemcpyAsync(E->d_coef, h.data(), sizeof(EnsCoef) * h.size(), cudaMemcpyHostToDevice, st));
  CF_TRY_CUDA(cudaStreamSynchronize(st));
  E->coef_cap = nsteps_total;
  E->coef_t0 = t0;
  E->coef_dt = dt;
  return CF_OK;
}

template <typename S, int H, int SHAPE>
static int launch_persistent(cf_ensemble *E, int nsteps, double dt, cudaStream_t st) {
  auto kern = k_ens_persistent<S, H, SHAPE>;
  if (!E->coop_blocks) {
    int per_sm = 0, dev = 0, sms = 0;
    CF_TRY_CUDA(cudaGetDevice(&dev));
    CF_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CF_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0));
    if (per_sm < 1) return ens_fail("ensemble: persistent kernel does not fit on an SM");
    E->coop_blocks = per_sm * sms;
  }
  EnsArgs A{};
  A.members = E->dm;
  A.items = E->d_items;
  A.n_items = (int)E->items.size();
  A.coef = E->d_coef;
  A.step_counter = E->d_step;
  A.nsteps = nsteps;
  A.dt = dt;
  A.bar_count = E->d_bar;
  A.bar_gen = E->d_bar + 1;
  A.work = E->d_bar + 2;
  A.err = E->d_err;
  A.bar_extra = E->bar_extra;
  A.spin_limit = E->spin_limit;
  void *args[] = {(void *)&A};
  const int blocks = std::min(E->coop_blocks, A.n_items);
  const dim3 block(EnsShape<SHAPE>::TX, EnsShape<SHAPE>::TY);
  CF_TRY_CUDA(cudaLaunchCooperativeKernel((const void *)kern, dim3(blocks), block, args, 0, st));
  E->launches++;
  return CF_OK;
}

// The persistent whole-step kernel over all step items (7-point), cooperative launch.
template <typename S, int SS>
static int launch_persistent_step_t(cf_ensemble *E, int nsteps, double dt, cudaStream_t st) {
  auto kern = k_ens_persistent_step<S, SS>;
  const dim3 block(EnsStepShape<S, SS>::TX, EnsStepShape<S, SS>::TY);
  const size_t smem = ens_step_smem<S, SS>();
  if (!E->coop_blocks_step) {
    int per_sm = 0, dev = 0, sms = 0;
    CF_TRY_CUDA(cudaGetDevice(&dev));
    CF_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CF_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int)(block.x * block.y), smem));
    if (per_sm < 1) return ens_fail("ensemble: persistent whole-step kernel does not fit on an SM");
    E->coop_blocks_step = per_sm * sms;
  }
  EnsArgs A{};
  A.members = E->dm;
  A.items = E->d_sitems;
  A.n_items = (int)E->sitems.size();
  A.coef = E->d_coef;
  A.step_counter = E->d_step;
  A.nsteps = nsteps;
  A.dt = dt;
  A.bar_count = E->d_bar;
  A.bar_gen = E->d_bar + 1;
  A.work = E->d_bar + 2;
  A.err = E->d_err;
  A.bar_extra = E->bar_extra;
  A.spin_limit = E->spin_limit;
  void *args[] = {(void *)&A};
  const int blocks = std::min(E->coop_blocks_step, A.n_items);
  CF_TRY_CUDA(cudaLaunchCooperativeKernel((const void *)kern, dim3(blocks), block, args, smem, st));
  E->launches++;
  return CF_OK;
}

static int launch_persistent_step(cf_ensemble *E, int nsteps, double dt, cudaStream_t st) {
  if (E->word == 4)
    return E->sshape ? launch_persistent_step_t<float, 1>(E, nsteps, dt, st)
                     : launch_persistent_step_t<float, 0>(E, nsteps, dt, st);
  return E->sshape ? launch_persistent_step_t<double, 1>(E, nsteps, dt, st)
                   : launch_persistent_step_t<double, 0>(E, nsteps, dt, st);
}

// One launch over work items [i0, i1): paired pass PASS (1, 2), or (PASS 0) phi
// back from ya to x.
template <typename S, int H, int SHAPE, int PASS>
static int launch_items_pair(cf_ensemble *E, size_t i0, size_t i1, int step_off, double dt, cudaStream_t st) {
  EnsArgs A{};
  A.members = E->dm;
  A.items = E->d_items + i0;
  A.n_items = (int)(i1 - i0);
  A.coef = E->d_coef;
  A.step_counter = E->d_step;
  A.dt = dt;
  const dim3 block(EnsShape<SHAPE>::TX, EnsShape<SHAPE>::TY);
  if constexpr (PASS == 0)
    k_ens_phi_back<S, SHAPE><<<A.n_items, block, 0, st>>>(A);
  else
    k_ens_pair<S, H, SHAPE, PASS><<<A.n_items, block, 0, st>>>(A, step_off);
  CF_TRY_CUDA(cudaGetLastError());
  E->launches++;
  return CF_OK;
}

// nsteps RK4 steps over work items [i0, i1) as paired passes, steps from the
// device step counter; phi back to x after an odd count.
template <typename S, int H, int SHAPE>
static int pair_steps(cf_ensemble *E, size_t i0, size_t i1, long long nsteps, double dt, cudaStream_t st) {
  for (long long j = 0; j < nsteps; ++j) {
    CF_TRY((launch_items_pair<S, H, SHAPE, 1>(E, i0, i1, (int)j, dt, st)));
    CF_TRY((launch_items_pair<S, H, SHAPE, 2>(E, i0, i1, (int)j, dt, st)));
  }
  if (nsteps & 1) CF_TRY((launch_items_pair<S, H, SHAPE, 0>(E, i0, i1, 0, dt, st)));
  return CF_OK;
}

// One whole-step launch over step items [i0, i1) (BACK: phi, pi back from ya to x).
template <typename S, int SS, bool BACK>
static int launch_items_step(cf_ensemble *E, size_t i0, size_t i1, int step_off, double dt, cudaStream_t st) {
  EnsArgs A{};
  A.members = E->dm;
  A.items = E->d_sitems + i0;
  A.n_items = (int)(i1 - i0);
  A.coef = E->d_coef;
  A.step_counter = E->d_step;
  A.dt = dt;
  const dim3 block(EnsStepShape<S, SS>::TX, EnsStepShape<S, SS>::TY);
  if constexpr (BACK)
    k_ens_xy_back<S, SS><<<A.n_items, block, 0, st>>>(A);
  else
    k_ens_step<S, SS><<<A.n_items, block, ens_step_smem<S, SS>(), st>>>(A, step_off);
  CF_TRY_CUDA(cudaGetLastError());
  E->launches++;
  return CF_OK;
}

// nsteps whole steps over step items [i0, i1) (BATCHED: all of them; LOOP: member by
// member), steps from the device step counter; phi, pi back to x after an odd count.
template <typename S, int SS>
static int step_steps_t(cf_ensemble *E, bool loop, long long nsteps, double dt, cudaStream_t st) {
  std::vector<std::pair<size_t, size_t>> ranges;
  if (!loop) {
    ranges.push_back({0, E->sitems.size()});
  } else {  // each member's items are contiguous
    for (size_t i0 = 0; i0 < E->sitems.size();) {
      size_t i1 = i0;
      while (i1 < E->sitems.size() && E->sitems[i1].member == E->sitems[i0].member) ++i1;
      ranges.push_back({i0, i1});
      i0 = i1;
    }
  }
  for (long long j = 0; j < nsteps; ++j)
    for (auto &r : ranges) CF_TRY((launch_items_step<S, SS, false>(E, r.first, r.second, (int)j, dt, st)));
  if (nsteps & 1)
    for (auto &r : ranges) CF_TRY((launch_items_step<S, SS, true>(E, r.first, r.second, 0, dt, st)));
  return CF_OK;
}

static int step_steps(cf_ensemble *E, bool loop, long long nsteps, double dt, cudaStream_t st) {
  if (E->word == 4)
    return E->sshape ? step_steps_t<float, 1>(E, loop, nsteps, dt, st) : step_steps_t<float, 0>(E, loop, nsteps, dt, st);
  return E->sshape ? step_steps_t<double, 1>(E, loop, nsteps, dt, st) : step_steps_t<double, 0>(E, loop, nsteps, dt, st);
}

template <typename S, int H, int SHAPE>
static int run_t(cf_ensemble *E, int mode, long long step0, long long nsteps, double dt, cudaStream_t st) {
  CF_TRY_CUDA(cudaMemcpyAsync(E->d_step, &step0, sizeof(long long), cudaMemcpyHostToDevice, st));
  if (mode == CF_ENS_PERSISTENT) {
    CF_TRY_CUDA(cudaMemsetAsync(E->d_bar, 0, 3 * sizeof(unsigned), st));
    CF_TRY_CUDA(cudaMemsetAsync(E->d_err, 0, sizeof(int), st));
    if (H == 1)
      CF_TRY(launch_persistent_step(E, (int)nsteps, dt, st));
    else
      CF_TRY((launch_persistent<S, H, SHAPE>(E, (int)nsteps, dt, st)));
    int err = 0;
    CF_TRY_CUDA(cudaMemcpyAsync(&err, E->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CF_TRY_CUDA(cudaStreamSynchronize(st));
    if (err) {
      set_error("ensemble: grid barrier timed out");
      return CF_ERR_TIMEOUT;
    }
    return CF_OK;
  }
  if (H == 1) return step_steps(E, mode == CF_ENS_LOOP, nsteps, dt, st);
  if (mode == CF_ENS_BATCHED) return pair_steps<S, H, SHAPE>(E, 0, E->items.size(), nsteps, dt, st);
  // CF_ENS_LOOP: the single-instance path, member by member (each member's
  // items are contiguous in the work list)
  std::vector<std::pair<size_t, size_t>> ranges;
  for (size_t i0 = 0; i0 < E->items.size();) {
    size_t i1 = i0;
    while (i1 < E->items.size() && E->items[i1].member == E->items[i0].member) ++i1;
    ranges.push_back({i0, i1});
    i0 = i1;
  }
  for (long long j = 0; j < nsteps; ++j) {
    for (auto &r : ranges) CF_TRY((launch_items_pair<S, H, SHAPE, 1>(E, r.first, r.second, (int)j, dt, st)));
    for (auto &r : ranges) CF_TRY((launch_items_pair<S, H, SHAPE, 2>(E, r.first, r.second, (int)j, dt, st)));
  }
  if (nsteps & 1)
    for (auto &r : ranges) CF_TRY((launch_items_pair<S, H, SHAPE, 0>(E, r.first, r.second, 0, dt, st)));
  return CF_OK;
}

template <typename S, int H>
static int run_shape(cf_ensemble *E, int mode, long long step0, long long nsteps, double dt, cudaStream_t st) {
  if (E->shape == 1) return run_t<S, H, 1>(E, mode, step0, nsteps, dt, st);
  return run_t<S, H, 0>(E, mode, step0, nsteps, dt, st);
}

static int run(cf_ensemble *E, int mode, long long step0, long long nsteps, double dt, cudaStream_t st) {
  if (E->word == 4) {
    if (E->stencil == 13) return run_shape<float, 2>(E, mode, step0, nsteps, dt, st);
    return run_shape<float, 1>(E, mode, step0, nsteps, dt, st);
  }
  if (E->stencil == 13) return run_shape<double, 2>(E, mode, step0, nsteps, dt, st);
  return run_shape<double, 1>(E, mode, step0, nsteps, dt, st);
}

template <typename S, int H>
static int batched_launches(cf_ensemble *E, long long steps, double dt, cudaStream_t st) {
  if (E->shape == 1) return pair_steps<S, H, 1>(E, 0, E->items.size(), steps, dt, st);
  return pair_steps<S, H, 0>(E, 0, E->items.size(), steps, dt, st);
}

// One observer segment from the device step counter, then the counter advance
// (graph-capturable: nothing is read from host memory).  CF_ENS_PERSISTENT: barrier
// reset + the persistent kernel; CF_ENS_BATCHED: 2 paired-stage launches per step.
static int segment(cf_ensemble *E, int mode, long long steps, double dt, cudaStream_t st) {
  int s;
  if (mode == CF_ENS_BATCHED) {
    if (E->stencil == 7)
      s = step_steps(E, false, steps, dt, st);
    else if (E->word == 4)
      s = E->stencil == 13 ? batched_launches<float, 2>(E, steps, dt, st) : batched_launches<float, 1>(E, steps, dt, st);
    else
      s = E->stencil == 13 ? batched_launches<double, 2>(E, steps, dt, st)
                           : batched_launches<double, 1>(E, steps, dt, st);
    if (s != CF_OK) return s;
    k_counter_add<<<1, 32, 0, st>>>(E->d_step, steps);
    CF_TRY_CUDA(cudaGetLastError());
    E->launches++;
    return CF_OK;
  }
  CF_TRY_CUDA(cudaMemsetAsync(E->d_bar, 0, 3 * sizeof(unsigned), st));
  if (E->stencil == 7) {
    s = launch_persistent_step(E, (int)steps, dt, st);
  } else if (E->word == 4) {
    if (E->stencil == 13)
      s = E->shape ? launch_persistent<float, 2, 1>(E, (int)steps, dt, st)
                   : launch_persistent<float, 2, 0>(E, (int)steps, dt, st);
    else
      s = E->shape ? launch_persistent<float, 1, 1>(E, (int)steps, dt, st)
                   : launch_persistent<float, 1, 0>(E, (int)steps, dt, st);
  } else {
    if (E->stencil == 13)
      s = E->shape ? launch_persistent<double, 2, 1>(E, (int)steps, dt, st)
                   : launch_persistent<double, 2, 0>(E, (int)steps, dt, st);
    else
      s = E->shape ? launch_persistent<double, 1, 1>(E, (int)steps, dt, st)
                   : launch_persistent<double, 1, 0>(E, (int)steps, dt, st);
  }
  if (s != CF_OK) return s;
  k_counter_add<<<1, 32, 0, st>>>(E->d_step, steps);
  CF_TRY_CUDA(cudaGetLastError());
  E->launches++;
  return CF_OK;
}

static int ensure_spectra(cf_ensemble *E) {
  if (!E->classes.empty()) return CF_OK;
  std::map<int, std::vector<int>> byN;
  for (int i = 0; i < E->count; ++i) byN[E->hm[i].N].push_back(i);
  E->out_offset.assign(E->count, 0);
  long long off = 0;
  for (int i = 0; i < E->count; ++i) {
    E->out_offset[i] = off;
    const long long N = E->hm[i].N;
    off += 3 * (N / 2) * (N / 2) + 1;
  }
  E->out_total = off;
  for (auto &kv : byN) {
    cf_ensemble::Cls c;
    c.N = kv.first;
    c.members = kv.second;
    const long long N = c.N, n = (long long)c.members.size();
    const long long N3 = N * N * N, hc = 2 * N * N * (N / 2 + 1);
    CF_TRY_CUDA(cudaMalloc(&c.d_members, sizeof(int) * n));
    CF_TRY_CUDA(cudaMemcpy(c.d_members, c.members.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    CF_TRY_CUDA(cudaMalloc(&c.rho, sizeof(double) * N3 * n));
    CF_TRY_CUDA(cudaMalloc(&c.hc, sizeof(double) * hc * n));
    long long nn[3] = {N, N, N}, ie[3] = {N, N, N}, oe[3] = {N, N, N / 2 + 1};
    size_t work = 0;
    CF_TRY_CUFFT(cufftCreate(&c.plan));
    CF_TRY_CUFFT(cufftMakePlanMany64(c.plan, 3, nn, ie, 1, N3, oe, 1, hc / 2, CUFFT_D2Z, n, &work));
    c.have_plan = true;
    E->max_bins = std::max<long long>(E->max_bins, (3 * (N / 2) * (N / 2) + 1) * n);
    E->classes.push_back(c);
  }
  CF_TRY_CUDA(cudaMalloc(&E->d_max, sizeof(unsigned long long) * E->count));
  CF_TRY_CUDA(cudaMalloc(&E->d_bins, sizeof(unsigned long long) * 2 * E->max_bins));
  return CF_OK;
}

static int spectra(cf_ensemble *E, double t, double *d_out, cudaStream_t st) {
  CF_TRY(ensure_spectra(E));
  cf_params q = E->base;
  double a2 = 1.0;
  if (q.equation != CF_EQ_KG) {
    const double a = cosmo_a(q, t);
    a2 = a * a;
  }
  for (auto &c : E->classes) {
    const int n = (int)c.members.size();
    const long long N3 = (long long)c.N * c.N * c.N;
    dim3 grid((unsigned)std::min<long long>((N3 + 255) / 256, 148LL * 4), n);
    if (E->word == 4)
      k_ens_energy<float><<<grid, 256, 0, st>>>(E->dm, c.d_members, c.rho, c.N, a2);
    else
      k_ens_energy<double><<<grid, 256, 0, st>>>(E->dm, c.d_members, c.rho, c.N, a2);
    CF_TRY_CUDA(cudaGetLastError());
    E->launches++;
    CF_TRY_CUFFT(cufftSetStream(c.plan, st));
    CF_TRY_CUFFT(cufftExecD2Z(c.plan, c.rho, (cufftDoubleComplex *)c.hc));
    // members of a class are consecutive in the output only if their indices are; bin into
    // a class-contiguous buffer, then copy each member's spectrum to its slot
    const long long nb = 3 * (c.N / 2) * (c.N / 2) + 1;
    double *tmp = c.rho;  // reuse: the density is no longer needed once transformed
    CF_TRY(bin_batched(c.hc, c.N, n, E->d_max, E->d_bins, tmp, nb, st, nullptr));
    E->launches += 3;
    for (int k = 0; k < n; ++k)
      CF_TRY_CUDA(cudaMemcpyAsync(d_out + E->out_offset[c.members[k]], tmp + nb * k, sizeof(double) * nb,
                                  cudaMemcpyDeviceToDevice, st));
  }
  return CF_OK;
}

}  // namespace cfb

using namespace cfb;

extern "C" {

int cf_ensemble_create(const cf_params *members, int count, cf_ensemble **out) {
  if (!members || count < 1 || !out) return ens_fail("cf_ensemble_create: need members, count >= 1, out");
  *out = nullptr;
  const cf_params &b = members[0];
  for (int i = 0; i < count; ++i) {
    const cf_params &p = members[i];
    if (p.N < 8 || p.N > 1024 || p.N % 8) return ens_fail("ensemble member N must be a multiple of 8 in [8, 1024]");
    if (p.equation != b.equation || p.precision != b.precision || p.stencil != b.stencil || p.a1 != b.a1 ||
        p.H1 != b.H1 || p.t1 != b.t1 || p.p != b.p)
      return ens_fail("ensemble members must share equation, precision, stencil and cosmology");
    if (p.equation != CF_EQ_KG && p.equation != CF_EQ_KG_FRW)
      return ens_fail("ensembles cover the flat and FRW Klein-Gordon equations");
    if (!(p.L > 0)) return ens_fail("member L must be positive");
  }
  if (b.stencil != 7 && b.stencil != 13) return ens_fail("stencil must be 7 or 13");
  cf_ensemble *E = new cf_ensemble();
  E->base = b;
  E->count = count;
  E->precision = b.precision;
  E->stencil = b.stencil;
  E->word = b.precision == CF_FP32_COMP ? 4 : 8;
  E->p.assign(members, members + count);
  E->hm.resize(count);
  for (int i = 0; i < count; ++i) {
    const cf_params &p = members[i];
    const long long N3 = p.N * p.N * p.N;
    void *mem = nullptr;
    const size_t sb = 16 * (size_t)N3;  // one state (either precision)
    if (cudaMalloc(&mem, 4 * sb) != cudaSuccess) {
      cudaGetLastError();
      for (void *a : E->allocs) cudaFree(a);
      delete E;
      set_error("ensemble: device allocation failed for member %d", i);
      return CF_ERR_NOMEM;
    }
    E->allocs.push_back(mem);
    EnsMember &m = E->hm[i];
    m.x = mem;
    m.acc = (char *)mem + sb;
    m.ya = (char *)mem + 2 * sb;
    m.yb = (char *)mem + 3 * sb;
    m.N = (int)p.N;
    m.N3 = N3;
    m.m2 = p.m * p.m;
    const double h = p.L / (double)p.N;
    m.inv_scale = 1.0 / (h * h);
  }
  bool ok = cudaMalloc(&E->dm, sizeof(EnsMember) * count) == cudaSuccess &&
            cudaMalloc(&E->d_step, sizeof(long long)) == cudaSuccess &&
            cudaMalloc(&E->d_bar, 3 * sizeof(unsigned)) == cudaSuccess &&
            cudaMalloc(&E->d_err, sizeof(int)) == cudaSuccess;
  if (!ok) {
    set_error("ensemble: device allocation failed");
    *out = E;
    cf_ensemble_destroy(E);
    *out = nullptr;
    return CF_ERR_NOMEM;
  }
  cudaMemcpy(E->dm, E->hm.data(), sizeof(EnsMember) * count, cudaMemcpyHostToDevice);
  cudaMemset(E->d_bar, 0, 3 * sizeof(unsigned));
  cudaMemset(E->d_err, 0, sizeof(int));
  cudaMemset(E->d_step, 0, sizeof(long long));
  build_items(E);
  int s = upload_items(E);
  if (s == CF_OK) s = build_step_items(E);
  if (s != CF_OK) {
    cf_ensemble_destroy(E);
    return s;
  }
  *out = E;
  return CF_OK;
}

int cf_ensemble_destroy(cf_ensemble *E) {
  if (!E) return CF_OK;
  cudaDeviceSynchronize();
  if (E->gexec) cudaGraphExecDestroy(E->gexec);
  for (void *a : E->allocs) cudaFree(a);
  cudaFree(E->dm);
  cudaFree(E->d_items);
  cudaFree(E->d_sitems);
  cudaFree(E->d_coef);
  cudaFree(E->d_step);
  cudaFree(E->d_bar);
  cudaFree(E->d_err);
  for (auto &c : E->classes) {
    cudaFree(c.d_members);
    cudaFree(c.rho);
    cudaFree(c.hc);
    if (c.have_plan) cufftDestroy(c.plan);
  }
  cudaFree(E->d_max);
  cudaFree(E->d_bins);
  delete E;
  return CF_OK;
}

int cf_ensemble_info(const cf_ensemble *E, int64_t *spectra_total, int64_t *work_items) {
  if (!E) return ens_fail("NULL ensemble");
  if (spectra_total) {
    long long off = 0;
    for (int i = 0; i < E->count; ++i) off += 3 * (E->hm[i].N / 2) * (E->hm[i].N / 2) + 1;
    *spectra_total = off;
  }
  if (work_items) *work_items = (int64_t)(E->stencil == 7 ? E->sitems.size() : E->items.size());
  return CF_OK;
}

int64_t cf_ensemble_launch_count(const cf_ensemble *E) { return E ? E->launches : -1; }

int cf_ensemble_state_upload(cf_ensemble *E, int member, const double *h_xy, void *stream) {
  if (!E || member < 0 || member >= E->count || !h_xy) return ens_fail("bad ensemble, member or pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const EnsMember &m = E->hm[member];
  const size_t n2 = 2 * (size_t)m.N3;
  if (E->word == 8) {
    CF_TRY_CUDA(cudaMemcpyAsync(m.x, h_xy, n2 * 8, cudaMemcpyHostToDevice, st));
    return CF_OK;
  }
  std::vector<float> hs(2 * n2);
  for (size_t i = 0; i < n2; ++i) {
    const float h = (float)h_xy[i];
    hs[i] = h;
    hs[n2 + i] = (float)(h_xy[i] - (double)h);
  }
  CF_TRY_CUDA(cudaMemcpyAsync(m.x, hs.data(), hs.size() * 4, cudaMemcpyHostToDevice, st));
  CF_TRY_CUDA(cudaStreamSynchronize(st));
  return CF_OK;
}

int cf_ensemble_state_download(cf_ensemble *E, int member, double *h_xy, void *stream) {
  if (!E || member < 0 || member >= E->count || !h_xy) return ens_fail("bad ensemble, member or pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const EnsMember &m = E->hm[member];
  const size_t n2 = 2 * (size_t)m.N3;
  if (E->word == 8) {
    CF_TRY_CUDA(cudaMemcpyAsync(h_xy, m.x, n2 * 8, cudaMemcpyDeviceToHost, st));
    CF_TRY_CUDA(cudaStreamSynchronize(st));
    return CF_OK;
  }
  std::vector<float> hs(2 * n2);
  CF_TRY_CUDA(cudaMemcpyAsync(hs.data(), m.x, hs.size() * 4, cudaMemcpyDeviceToHost, st));
  CF_TRY_CUDA(cudaStreamSynchronize(st));
  for (size_t i = 0; i < n2; ++i) h_xy[i] = (double)hs[i] + (double)hs[n2 + i];
  return CF_OK;
}

int cf_ensemble_rk4_steps(cf_ensemble *E, double t0, double dt, int64_t step0, int64_t nsteps, int mode,
                          void *stream) {
  if (!E || nsteps < 0 || step0 < 0) return ens_fail("bad ensemble or step range");
  if (mode != CF_ENS_PERSISTENT && mode != CF_ENS_BATCHED && mode != CF_ENS_LOOP) return ens_fail("unknown mode");
  cudaStream_t st = (cudaStream_t)stream;
  CF_TRY(ensure_coef(E, t0, dt, step0 + nsteps, st));
  return run(E, mode, step0, nsteps, dt, st);
}

int cf_ensemble_density_spectra_s2(cf_ensemble *E, double t, double *d_out, void *stream) {
  if (!E || !d_out) return ens_fail("bad ensemble or output");
  return spectra(E, t, d_out, (cudaStream_t)stream);
}

int cf_ensemble_run_graph(cf_ensemble *E, double t0, double dt, int64_t steps_per_segment, int64_t nsegments,
                          int mode, double *d_spectra, void *stream) {
  if (!E || steps_per_segment < 1 || nsegments < 0) return ens_fail("bad ensemble or segment sizes");
  if (mode != CF_ENS_PERSISTENT && mode != CF_ENS_BATCHED) return ens_fail("run_graph: mode must be PERSISTENT or BATCHED");
  if (mode == CF_ENS_BATCHED && steps_per_segment > (1 << 20)) return ens_fail("run_graph: too many steps per segment");
  cudaStream_t st = (cudaStream_t)stream;
  if (!st) return ens_fail("cf_ensemble_run_graph needs a non-default stream (graph capture)");
  CF_TRY(ensure_coef(E, t0, dt, steps_per_segment * std::max<int64_t>(nsegments, 1), st));
  CF_TRY(ensure_spectra(E));
  long long zero = 0;
  CF_TRY_CUDA(cudaMemcpyAsync(E->d_step, &zero, sizeof(zero), cudaMemcpyHostToDevice, st));
  CF_TRY_CUDA(cudaMemsetAsync(E->d_err, 0, sizeof(int), st));
  // The graph holds one segment (its first step read from the device step
  // counter, which the segment advances), so replaying the same graph walks the
  // run forward.  Each segment's spectra are enqueued on the same stream after its
  // replay (their a(t) differs per segment).
  for (int64_t sgi = 0; sgi < nsegments; ++sgi) {
    const bool fallback = mode == CF_ENS_PERSISTENT && E->graph_failed;
    if (!fallback && (!E->gexec || E->g_mode != mode || E->g_steps != steps_per_segment || E->g_t0 != t0 ||
                      E->g_dt != dt || E->g_out != d_spectra)) {
      if (E->gexec) cudaGraphExecDestroy(E->gexec);
      E->gexec = nullptr;
      cudaGraph_t g = nullptr;
      const int64_t l0 = E->launches;
      bool ok = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      int s = ok ? segment(E, mode, steps_per_segment, dt, st) : CF_ERR_CUDA;
      E->g_kernels = E->launches - l0;
      E->launches = l0;
      if (ok) ok = cudaStreamEndCapture(st, &g) == cudaSuccess && s == CF_OK;
      if (ok) ok = cudaGraphInstantiate(&E->gexec, g, 0) == cudaSuccess;
      if (g) cudaGraphDestroy(g);
      if (!ok) {
        // capture of the cooperative launch unavailable: run the same segment
        // launches directly (same kernels, same results)
        cudaGetLastError();
        if (E->gexec) cudaGraphExecDestroy(E->gexec);
        E->gexec = nullptr;
        if (mode == CF_ENS_BATCHED) return ens_fail("run_graph: capture of the batched launches failed");
        E->graph_failed = true;
      } else {
        E->g_mode = mode;
        E->g_steps = steps_per_segment;
        E->g_t0 = t0;
        E->g_dt = dt;
        E->g_out = d_spectra;
      }
    }
    if (E->gexec) {
      CF_TRY_CUDA(cudaGraphLaunch(E->gexec, st));
      E->launches += E->g_kernels;
    } else {
      CF_TRY(segment(E, mode, steps_per_segment, dt, st));
    }
    if (d_spectra) {
      const double t_end = t0 + (double)((sgi + 1) * steps_per_segment) * dt;
      CF_TRY(spectra(E, t_end, d_spectra + sgi * E->out_total, st));
    }
  }
  int err = 0;
  CF_TRY_CUDA(cudaMemcpyAsync(&err, E->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CF_TRY_CUDA(cudaStreamSynchronize(st));
  if (err) {
    set_error("ensemble: grid barrier timed out");
    return CF_ERR_TIMEOUT;
  }
  return CF_OK;
}

int cf_ensemble_set_barrier_test(cf_ensemble *E, int extra_arrivals, int64_t spin_limit) {
  if (!E || extra_arrivals < 0 || spin_limit < 1) return ens_fail("bad ensemble, extra_arrivals or spin_limit");
  E->bar_extra = (unsigned)extra_arrivals;
  E->spin_limit = spin_limit;
  if (E->gexec) {  // a captured graph holds the old kernel arguments
    cudaGraphExecDestroy(E->gexec);
    E->gexec = nullptr;
  }
  return CF_OK;
}

int cf_ensemble_autotune(cf_ensemble *E, double t0, double dt, int64_t steps, void *stream, int *h_shape,
                         int *h_a_chunk) {
  if (!E || steps < 1) return ens_fail("bad ensemble or steps");
  cudaStream_t st = (cudaStream_t)stream;
  CF_TRY(ensure_coef(E, t0, dt, steps, st));
  // the state is not preserved across candidate timings: tune before uploading initial data
  cudaEvent_t a, b;
  CF_TRY_CUDA(cudaEventCreate(&a));
  CF_TRY_CUDA(cudaEventCreate(&b));
  float best = 1e30f;
  int best_shape = 0, best_chunk = 16;
  if (E->stencil == 7) {  // the whole-step work list of the batched schedule
    const int schunks[3] = {16, 32, 64};
    for (int shape = 0; shape < ENS_STEP_SHAPES; ++shape)
      for (int ch : schunks) {
        E->sshape = shape;
        E->schunk = ch;
        CF_TRY(build_step_items(E));
        CF_TRY(step_steps(E, false, 1, dt, st));  // warm
        CF_TRY_CUDA(cudaEventRecord(a, st));
        CF_TRY(step_steps(E, false, steps, dt, st));
        CF_TRY_CUDA(cudaEventRecord(b, st));
        CF_TRY_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        CF_TRY_CUDA(cudaEventElapsedTime(&ms, a, b));
        if (ms < best) {
          best = ms;
          best_shape = shape;
          best_chunk = ch;
        }
      }
    E->sshape = best_shape;
    E->schunk = best_chunk;
    CF_TRY(build_step_items(E));
    if (E->gexec) {
      cudaGraphExecDestroy(E->gexec);
      E->gexec = nullptr;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (h_shape) *h_shape = best_shape;
    if (h_a_chunk) *h_a_chunk = best_chunk;
    return CF_OK;
  }
  const int chunks[3] = {8, 16, 32};
  for (int shape = 0; shape < ENS_SHAPES; ++shape)
    for (int ch : chunks) {
      E->shape = shape;
      E->tune.clear();
      for (int i = 0; i < E->count; ++i) E->tune[E->hm[i].N] = {shape, ch};
      build_items(E);
      CF_TRY(upload_items(E));
      E->coop_blocks = 0;
      CF_TRY(run(E, CF_ENS_BATCHED, 0, 1, dt, st));  // warm
      CF_TRY_CUDA(cudaEventRecord(a, st));
      CF_TRY(run(E, CF_ENS_BATCHED, 0, steps, dt, st));
      CF_TRY_CUDA(cudaEventRecord(b, st));
      CF_TRY_CUDA(cudaEventSynchronize(b));
      float ms = 0;
      CF_TRY_CUDA(cudaEventElapsedTime(&ms, a, b));
      if (ms < best) {
        best = ms;
        best_shape = shape;
        best_chunk = ch;
      }
    }
  E->shape = best_shape;
  E->tune.clear();
  for (int i = 0; i < E->count; ++i) E->tune[E->hm[i].N] = {best_shape, best_chunk};
  build_items(E);
  CF_TRY(upload_items(E));
  E->coop_blocks = 0;
  if (E->gexec) {
    cudaGraphExecDestroy(E->gexec);
    E->gexec = nullptr;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (h_shape) *h_shape = best_shape;
  if (h_a_chunk) *h_a_chunk = best_chunk;
  return CF_OK;
}

}  // extern "C"
