// cf_adjoint.cu -- discrete adjoint of the fused RK4 + stencil stepper and of
// the shell-spectrum log loss, with checkpointing and recompute.
//
// For the Klein-Gordon right-hand side (flat or FRW; src/equations.cpp:8-36,
// :71-104) the stage map is linear, f(t) x = A(t) x with
//   A (phi, pi) = (pi, (-m^2 + inv(t) lap) phi - 3H(t) pi),
//   A^T (u, v)  = ((-m^2 + inv(t) lap) v, u - 3H(t) v)     (lap symmetric, periodic).
// One classic RK4 step (stepper/runge_kutta4_classic.hpp:88-138)
//   y1 = x, y2 = x + h/2 A1 y1, y3 = x + h/2 A2 y2, y4 = x + h A2 y3,
//   x' = x + h/6 A1 y1 + h/3 A2 y2 + h/3 A2 y3 + h/6 A4 y4
// has the exact reverse sweep, for l' = dL/dx':
//   kb4 = h/6 l'              ; yb4 = A4^T kb4
//   kb3 = h/3 l' + h   yb4    ; yb3 = A2^T kb3
//   kb2 = h/3 l' + h/2 yb3    ; yb2 = A2^T kb2
//   kb1 = h/6 l' + h/2 yb2    ; yb1 = A1^T kb1
//   l   = l' + yb4 + yb3 + yb2 + yb1
//   dL/dm += sum_i <kb_i, dA/dm y_i> = sum_i sum_x kb_i.pi(x) (-2 m) y_i.phi(x)
// The four reverse stages are fused one-pass kernels with the same streaming
// stencil as the forward stages, the stencil acting on the pi component of kb.
// The forward stage inputs y_i a reverse step needs (for dL/dm) are recomputed
// from the nearest checkpoint (every `checkpoint_every` steps): a segment is
// re-run forward and its states kept, then walked backwards.
//
// Adjoint variables are FP64 in both precisions; the forward (and its
// recompute) runs in the context precision, bit-identically.

#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <vector>

#include "cf_internal.cuh"

namespace cfb {

constexpr int ATX = 32;
constexpr int ATY = 8;

template <typename S>
struct AdjArgs {
  const double *kin;   // stored reverse-stage input K (2N^3); kb = sin * K
  double sin;
  const double *lamp;  // l' (2N^3)
  double *acc;         // running sum of yb (2N^3)
  double *knext;       // next kb (stages 4, 3, 2)
  double *lam_out;     // stage 1: l = l' + acc + yb1 (may alias lamp)
  const S *yphi;       // phi of the forward stage input y_i (N^3)
  double *dm_partial;  // per-CTA partial sums of dL/dm (accumulated across launches)
  int N;
  int a_chunk;
  long long N3;
  double m2, inv, hub3;
  double cl, cy;       // knext = cl * l' + cy * yb
  double two_m;
};

// STAGE is the forward stage index being reversed: 4, 3, 2 or 1.
template <typename S, int H, int STAGE>
__global__ void __launch_bounds__(ATX *ATY) k_adj_stage(const AdjArgs<S> A) {
  constexpr int TW = ATX * 2;  // two sites per thread (double2)
  constexpr int SP = TW + 2 * H;
  constexpr int SR = ATY + 2 * H;
  __shared__ double sm[SR * SP];
  __shared__ double red[ATX * ATY / 32];
  const int N = A.N;
  const long long N3 = A.N3, NN = (long long)N * N;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * ATX + tx;
  const int c0 = blockIdx.x * TW, b0 = blockIdx.y * ATY;
  const int twe = min(TW, N - c0);
  const int a_begin = blockIdx.z * A.a_chunk, a_end = min(a_begin + A.a_chunk, N);
  const int c = c0 + tx * 2, b = b0 + ty;
  const bool act = (tx * 2) < twe;
  const long long rowoff = (long long)N * b + c;
  const double *vin = A.kin + N3;  // the stencil acts on the pi component
  const double *uin = A.kin;
  double q[2 * H + 1][2];
  if (act) {
#pragma unroll
    for (int j = 0; j < 2 * H; ++j) {
      const double2 t = *reinterpret_cast<const double2 *>(vin + NN * ((a_begin - H + j + N) % N) + rowoff);
      q[j + 1][0] = t.x;
      q[j + 1][1] = t.y;
    }
  }
  double dm = 0.0;
  for (int a = a_begin; a < a_end; ++a) {
    const long long site = NN * a + rowoff;
#pragma unroll
    for (int j = 0; j < 2 * H; ++j) q[j][0] = q[j + 1][0], q[j][1] = q[j + 1][1];
    double2 u2{}, lp{}, lq{}, ap{}, aq{};
    double y0 = 0, y1 = 0;
    if (act) {
      const double2 t = *reinterpret_cast<const double2 *>(vin + NN * ((a + H) % N) + rowoff);
      q[2 * H][0] = t.x;
      q[2 * H][1] = t.y;
      u2 = *reinterpret_cast<const double2 *>(uin + site);
      lp = *reinterpret_cast<const double2 *>(A.lamp + site);
      lq = *reinterpret_cast<const double2 *>(A.lamp + N3 + site);
      if constexpr (STAGE != 4) {
        ap = *reinterpret_cast<const double2 *>(A.acc + site);
        aq = *reinterpret_cast<const double2 *>(A.acc + N3 + site);
      }
      y0 = (double)A.yphi[site];
      y1 = (double)A.yphi[site + 1];
    }
    __syncthreads();
    if (act) {
      sm[(ty + H) * SP + H + tx * 2] = q[H][0];
      sm[(ty + H) * SP + H + tx * 2 + 1] = q[H][1];
    }
    if (ty < H || ty >= ATY - H) {
      if (act) {
        const int r = (ty < H) ? ty : ty + 2 * H;
        const int gb = (b0 - H + r + N) % N;
        const double2 h = *reinterpret_cast<const double2 *>(vin + NN * a + (long long)N * gb + c);
        sm[r * SP + H + tx * 2] = h.x;
        sm[r * SP + H + tx * 2 + 1] = h.y;
      }
    }
    for (int i = tid; i < SR * 2 * H; i += ATX * ATY) {
      const int r = i / (2 * H), j = i % (2 * H);
      const int gb = (b0 - H + r + N) % N;
      int col, gc;
      if (j < H) {
        col = j;
        gc = (c0 - H + j + N) % N;
      } else {
        col = twe + H + (j - H);
        gc = (c0 + twe + (j - H)) % N;
      }
      sm[r * SP + col] = vin[NN * a + (long long)N * gb + gc];
    }
    __syncthreads();
    if (!act) continue;
    double outp[2], outq[2], knp[2], knq[2];
    const double uu[2] = {u2.x, u2.y}, l_p[2] = {lp.x, lp.y}, l_q[2] = {lq.x, lq.y};
    const double a_p[2] = {ap.x, ap.y}, a_q[2] = {aq.x, aq.y}, yy[2] = {y0, y1};
#pragma unroll
    for (int v = 0; v < 2; ++v) {
      const int col = H + tx * 2 + v, row = ty + H;
      const double f0 = q[H][v];
      double lap;
      if constexpr (H == 1) {
        lap = -6.0 * f0 + q[2][v] + q[0][v] + sm[(row + 1) * SP + col] + sm[(row - 1) * SP + col] +
              (sm[row * SP + col + 1] + sm[row * SP + col - 1]);
      } else {
        const double s1 = q[3][v] + q[1][v] + sm[(row + 1) * SP + col] + sm[(row - 1) * SP + col] +
                          sm[row * SP + col + 1] + sm[row * SP + col - 1];
        const double s2 = q[4][v] + q[0][v] + sm[(row + 2) * SP + col] + sm[(row - 2) * SP + col] +
                          sm[row * SP + col + 2] + sm[row * SP + col - 2];
        lap = (16.0 * s1 - s2 - 90.0 * f0) / 12.0;
      }
      const double kv = A.sin * f0, ku = A.sin * uu[v];
      const double ybp = -A.m2 * kv + A.inv * (A.sin * lap);
      const double ybq = ku - A.hub3 * kv;
      dm += kv * yy[v];
      if constexpr (STAGE == 4) {
        outp[v] = ybp;
        outq[v] = ybq;
      } else {
        outp[v] = a_p[v] + ybp;
        outq[v] = a_q[v] + ybq;
      }
      if constexpr (STAGE != 1) {
        knp[v] = A.cl * l_p[v] + A.cy * ybp;
        knq[v] = A.cl * l_q[v] + A.cy * ybq;
      }
    }
    if constexpr (STAGE == 1) {
      *reinterpret_cast<double2 *>(A.lam_out + site) = make_double2(l_p[0] + outp[0], l_p[1] + outp[1]);
      *reinterpret_cast<double2 *>(A.lam_out + N3 + site) = make_double2(l_q[0] + outq[0], l_q[1] + outq[1]);
    } else {
      *reinterpret_cast<double2 *>(A.acc + site) = make_double2(outp[0], outp[1]);
      *reinterpret_cast<double2 *>(A.acc + N3 + site) = make_double2(outq[0], outq[1]);
      *reinterpret_cast<double2 *>(A.knext + site) = make_double2(knp[0], knp[1]);
      *reinterpret_cast<double2 *>(A.knext + N3 + site) = make_double2(knq[0], knq[1]);
    }
  }
  // deterministic CTA reduction of kb.pi * y.phi, then -2m and accumulate into this CTA's slot
  for (int o = 16; o > 0; o >>= 1) dm += __shfl_down_sync(0xffffffffu, dm, o);
  if ((tid & 31) == 0) red[tid >> 5] = dm;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int w = 0; w < ATX * ATY / 32; ++w) s += red[w];
    const long long cta = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    A.dm_partial[cta] += -A.two_m * s;
  }
}

// Adjoint of the energy density rho = 1/2 (pi^2 + m^2 phi^2 + 1/4 inv sum_e (phi_{+e} - phi_{-e})^2):
//   l.pi  = rb pi,
//   l.phi = rb m^2 phi + 1/4 inv sum_e [rb_{-e} (phi - phi_{-2e}) - rb_{+e} (phi_{+2e} - phi)],
//   dL/dm (direct) = sum rb m phi^2  (per-block partials).
__global__ void k_energy_adjoint(const double *__restrict__ x, const double *__restrict__ rb, double *__restrict__ lam,
                                 double *__restrict__ dm_partial, int N, double m, double inv) {
  const long long N3 = (long long)N * N * N, NN = (long long)N * N;
  __shared__ double red[8];
  double dm = 0.0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N3; i += stride) {
    const int c = (int)(i % N), b = (int)((i / N) % N), a = (int)(i / NN);
    auto at = [&](int aa, int bb, int cc) -> long long {
      return NN * ((aa + 2 * N) % N) + (long long)N * ((bb + 2 * N) % N) + ((cc + 2 * N) % N);
    };
    const double f = x[i], r = rb[i];
    double g = 0.0;
    const int da[3] = {1, 0, 0}, db[3] = {0, 1, 0}, dc[3] = {0, 0, 1};
    for (int e = 0; e < 3; ++e) {
      const double rm = rb[at(a - da[e], b - db[e], c - dc[e])];
      const double rp = rb[at(a + da[e], b + db[e], c + dc[e])];
      const double fm2 = x[at(a - 2 * da[e], b - 2 * db[e], c - 2 * dc[e])];
      const double fp2 = x[at(a + 2 * da[e], b + 2 * db[e], c + 2 * dc[e])];
      g += rm * (f - fm2) - rp * (fp2 - f);
    }
    lam[i] = r * m * m * f + 0.25 * inv * g;
    lam[N3 + i] = r * x[N3 + i];
    dm += r * m * f * f;
  }
  for (int o = 16; o > 0; o >>= 1) dm += __shfl_down_sync(0xffffffffu, dm, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dm;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) s += red[w];
    dm_partial[blockIdx.x] = s;
  }
}

__device__ __forceinline__ long long hc_s2(int N, long long i, int &c) {
  const int nh = N / 2 + 1;
  c = (int)(i % nh);
  const long long ab = i / nh;
  const int b = (int)(ab % N), a = (int)(ab / N);
  const long long as = (a <= N / 2) ? a : N - a, bs = (b <= N / 2) ? b : N - b;
  return as * as + bs * bs + (long long)c * c;
}

__device__ __forceinline__ long long isqrt_d(long long s) {
  long long r = (long long)sqrt((double)s);
  while (r * r > s) --r;
  while ((r + 1) * (r + 1) <= s) ++r;
  return r;
}

// Adjoint of the shell power P_s = sum_{k in s} w_k |rho_k|^2 through the r2c:
// with g_s = dL/dP_s, dL/drho = c2r(H), H_k = 2 g_{shell(k)} rho_k (all HC entries).
__global__ void k_shell_loss_adjoint(double *__restrict__ hc, const double *__restrict__ g, int N, long long pairs) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < pairs; i += stride) {
    int c;
    const long long s2 = hc_s2(N, i, c);
    const double w = 2.0 * g[isqrt_d(s2)];
    hc[2 * i] *= w;
    hc[2 * i + 1] *= w;
  }
}

// phi0 = c2r(sqrt(theta_{group(k)}) sqrtP(s^2) xi_k): writes the HC input of the c2r.
__global__ void k_field_from_theta(const double *__restrict__ xi, const double *__restrict__ sqrtP,
                                   const double *__restrict__ sqrt_theta, int shells_per_group, int ngroups,
                                   double *__restrict__ hc, int N, long long pairs) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < pairs; i += stride) {
    int c;
    const long long s2 = hc_s2(N, i, c);
    const int g = (int)min((long long)ngroups - 1, isqrt_d(s2) / shells_per_group);
    const double f = sqrt_theta[g] * sqrtP[s2];
    hc[2 * i] = f * xi[2 * i];
    hc[2 * i + 1] = f * xi[2 * i + 1];
  }
}

// dL/dtheta_g = 1/(2 sqrt(theta_g)) sum_{k in g} w_k Re(sqrtP xi_k conj(lhat_k)), lhat = r2c(dL/dphi0).
// Per-CTA partials per group (deterministic), summed on the host.
__global__ void k_theta_grad(const double *__restrict__ xi, const double *__restrict__ sqrtP,
                             const double *__restrict__ lhat, int shells_per_group, int ngroups,
                             double *__restrict__ partial, int N, long long pairs) {
  extern __shared__ double sg[];  // ngroups per warp
  const int nw = blockDim.x / 32, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int j = threadIdx.x; j < nw * ngroups; j += blockDim.x) sg[j] = 0.0;
  __syncthreads();
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long base = (long long)blockIdx.x * blockDim.x; base < pairs; base += stride) {
    const long long i = base + threadIdx.x;
    double v = 0.0;
    int g = -1;
    if (i < pairs) {
      int c;
      const long long s2 = hc_s2(N, i, c);
      g = (int)min((long long)ngroups - 1, isqrt_d(s2) / shells_per_group);
      const double wk = (c == 0 || 2 * c == N) ? 1.0 : 2.0;
      v = wk * sqrtP[s2] * (xi[2 * i] * lhat[2 * i] + xi[2 * i + 1] * lhat[2 * i + 1]);
    }
    // lanes in fixed order add into their warp's group slots
    for (int l = 0; l < 32; ++l) {
      const int gl = __shfl_sync(0xffffffffu, g, l);
      const double vl = __shfl_sync(0xffffffffu, v, l);
      if (lane == 0 && gl >= 0) sg[w * ngroups + gl] += vl;
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < ngroups; j += blockDim.x) {
    double s = 0.0;
    for (int ww = 0; ww < nw; ++ww) s += sg[ww * ngroups + j];
    partial[(long long)blockIdx.x * ngroups + j] = s;
  }
}

// forward stage launcher and step (cf_step.cu)
int launch_forward_stage(cf_ctx *ctx, int stage, const void *yin, void *yout, void *x, void *xlo, double t,
                         double cy, double dt6, cudaStream_t st);

}  // namespace cfb

struct cf_adjoint {
  cf_ctx *ctx = nullptr;
  int64_t nsteps = 0, every = 0;
  double t0 = 0, dt = 0;
  bool have_forward = false;
  size_t state_bytes = 0;
  std::vector<void *> ckpt;
  void *seg = nullptr;  // `every` states
  void *Y = nullptr;    // forward stage inputs y2, y3, y4 (storage type, 2N^3 each)
  double *lam = nullptr, *ka = nullptr, *kb = nullptr, *accb = nullptr, *rb = nullptr;
  double *dm_partial = nullptr;
  long long dm_slots = 0;
  double dm_direct = 0.0;
  cufftHandle plan_z2d = 0;
  bool have_z2d = false;
};

namespace cfb {

static unsigned gridn(long long n, int per = 256) {
  long long b = (n + per - 1) / per;
  if (b > 148LL * 16) b = 148LL * 16;
  return (unsigned)(b < 1 ? 1 : b);
}

template <typename S, int H, int STAGE>
static int launch_adj(cf_adjoint *adj, AdjArgs<S> A, cudaStream_t st) {
  cf_ctx *ctx = adj->ctx;
  constexpr int TW = ATX * 2;
  dim3 block(ATX, ATY);
  const unsigned gx = ceil_div(A.N, TW), gy = (unsigned)(A.N / ATY);
  A.a_chunk = 16;
  dim3 grid(gx, gy, ceil_div(A.N, A.a_chunk));
  k_adj_stage<S, H, STAGE><<<grid, block, 0, st>>>(A);
  CF_LAUNCHED(ctx);
  return CF_OK;
}

template <typename S, int STAGE>
static int launch_adj_h(cf_adjoint *adj, const AdjArgs<S> &A, cudaStream_t st) {
  if (adj->ctx->p.stencil == 13) return launch_adj<S, 2, STAGE>(adj, A, st);
  return launch_adj<S, 1, STAGE>(adj, A, st);
}

static long long adj_cta_count(const cf_ctx *ctx) {
  const long long N = ctx->N;
  return (long long)ceil_div(N, ATX * 2) * (N / ATY) * ceil_div(N, 16);
}

int adjoint_create(cf_ctx *ctx, int64_t nsteps, int64_t every, cf_adjoint **out) {
  if (ctx->p.equation != CF_EQ_KG && ctx->p.equation != CF_EQ_KG_FRW) {
    set_error("the adjoint covers the flat and FRW Klein-Gordon equations");
    return CF_ERR_UNSUPPORTED;
  }
  if (nsteps < 1 || every < 1) {
    set_error("nsteps and checkpoint_every must be >= 1");
    return CF_ERR_INVALID;
  }
  cf_adjoint *a = new cf_adjoint();
  a->ctx = ctx;
  a->nsteps = nsteps;
  a->every = every;
  a->state_bytes = 16 * (size_t)ctx->N3;
  const size_t sb = a->state_bytes, fb = 8 * (size_t)ctx->N3;
  const long long nck = (nsteps + every - 1) / every;
  auto alloc = [&](void **p, size_t bytes) -> bool { return cudaMalloc(p, bytes) == cudaSuccess; };
  bool ok = true;
  a->ckpt.assign(nck, nullptr);
  for (auto &p : a->ckpt) ok = ok && alloc(&p, sb);
  ok = ok && alloc(&a->seg, sb * (size_t)every) && alloc(&a->Y, 3 * sb);
  ok = ok && alloc((void **)&a->lam, 2 * fb) && alloc((void **)&a->ka, 2 * fb) && alloc((void **)&a->kb, 2 * fb) &&
       alloc((void **)&a->accb, 2 * fb) && alloc((void **)&a->rb, fb);
  a->dm_slots = std::max<long long>(adj_cta_count(ctx), 148 * 16);
  ok = ok && alloc((void **)&a->dm_partial, sizeof(double) * (size_t)a->dm_slots);
  if (!ok) {
    cudaGetLastError();
    set_error("adjoint: device allocation failed (checkpoints + segment need %zu bytes)",
              sb * (size_t)(nck + every + 3) + 9 * fb);
    *out = a;
    return CF_ERR_NOMEM;
  }
  *out = a;
  return CF_OK;
}

void adjoint_destroy(cf_adjoint *a) {
  if (!a) return;
  cudaDeviceSynchronize();
  for (auto p : a->ckpt) cudaFree(p);
  cudaFree(a->seg);
  cudaFree(a->Y);
  cudaFree(a->lam);
  cudaFree(a->ka);
  cudaFree(a->kb);
  cudaFree(a->accb);
  cudaFree(a->rb);
  cudaFree(a->dm_partial);
  if (a->have_z2d) cufftDestroy(a->plan_z2d);
  delete a;
}

int rk4_steps(cf_ctx *, void *, double, double, int64_t, int64_t, cudaStream_t);
int density_spectrum_s2(cf_ctx *, const void *, double, double *, cudaStream_t);
int s2_to_shells(cf_ctx *, double *, int64_t *, cudaStream_t);
int state_export(cf_ctx *, double *, const void *, cudaStream_t);

int adjoint_forward(cf_adjoint *a, void *d_state, double t0, double dt, cudaStream_t st) {
  a->t0 = t0;
  a->dt = dt;
  // one call per checkpoint segment: the steps are those of single-step calls (same
  // kernels, times t0 + n dt), without a state copy-back after every step
  for (int64_t n0 = 0; n0 < a->nsteps; n0 += a->every) {
    CF_TRY_CUDA(cudaMemcpyAsync(a->ckpt[n0 / a->every], d_state, a->state_bytes, cudaMemcpyDeviceToDevice, st));
    CF_TRY(rk4_steps(a->ctx, d_state, t0, dt, n0, std::min<int64_t>(a->every, a->nsteps - n0), st));
  }
  a->have_forward = true;
  return CF_OK;
}

int adjoint_shell_log_loss(cf_adjoint *a, const void *d_state, const double *h_target, double rel_floor,
                           double *h_loss, cudaStream_t st) {
  cf_ctx *ctx = a->ctx;
  const double tT = a->t0 + (double)a->nsteps * a->dt;
  const long long ns = ctx->shells;
  double *d_sh = nullptr;
  CF_TRY_CUDA(cudaMallocAsync((void **)&d_sh, sizeof(double) * ns, st));
  CF_TRY(density_spectrum_s2(ctx, d_state, tT, nullptr, st));
  CF_TRY(s2_to_shells(ctx, d_sh, nullptr, st));
  std::vector<double> P(ns), g(ns, 0.0);
  CF_TRY_CUDA(cudaMemcpyAsync(P.data(), d_sh, sizeof(double) * ns, cudaMemcpyDeviceToHost, st));
  CF_TRY_CUDA(cudaStreamSynchronize(st));
  double loss = 0.0, tmax = 0.0;
  for (long long s = 0; s < ns; ++s) tmax = std::max(tmax, h_target[s]);
  const double floor_v = std::max(0.0, rel_floor) * tmax;
  for (long long s = 0; s < ns; ++s) {
    if (P[s] > 0 && h_target[s] > 0 && h_target[s] > floor_v) {
      const double d = std::log(P[s]) - std::log(h_target[s]);
      loss += d * d;
      g[s] = 2.0 * d / P[s];
    }
  }
  if (h_loss) *h_loss = loss;
  // dL/drho = c2r(H), H_k = 2 g_shell(k) rho_k  (rho_k is still in the spectrum scratch)
  CF_TRY_CUDA(cudaMemcpyAsync(d_sh, g.data(), sizeof(double) * ns, cudaMemcpyHostToDevice, st));
  const long long pairs = ctx->hc_count / 2;
  k_shell_loss_adjoint<<<gridn(pairs), 256, 0, st>>>(ctx->spec_hc, d_sh, (int)ctx->N, pairs);
  CF_LAUNCHED(ctx);
  if (!a->have_z2d) {
    const int N = (int)ctx->N;
    CF_TRY_CUFFT(cufftPlan3d(&a->plan_z2d, N, N, N, CUFFT_Z2D));
    a->have_z2d = true;
  }
  CF_TRY_CUFFT(cufftSetStream(a->plan_z2d, st));
  CF_TRY_CUFFT(cufftExecZ2D(a->plan_z2d, (cufftDoubleComplex *)ctx->spec_hc, a->rb));
  // l_T = adjoint of the energy density at t_T
  const double *x = (const double *)d_state;
  if (ctx->p.precision != CF_FP64) {
    CF_TRY(state_export(ctx, ctx->spec_field, d_state, st));
    x = ctx->spec_field;
  }
  double inv, H;
  stage_coeffs(ctx->p, tT, &inv, &H);
  const unsigned gb = gridn(ctx->N3);
  k_energy_adjoint<<<gb, 256, 0, st>>>(x, a->rb, a->lam, a->dm_partial, (int)ctx->N, ctx->p.m, inv);
  CF_LAUNCHED(ctx);
  std::vector<double> part(gb);
  CF_TRY_CUDA(cudaMemcpyAsync(part.data(), a->dm_partial, sizeof(double) * gb, cudaMemcpyDeviceToHost, st));
  CF_TRY_CUDA(cudaFreeAsync(d_sh, st));
  CF_TRY_CUDA(cudaStreamSynchronize(st));
  double s = 0.0;
  for (double v : part) s += v;
  a->dm_direct = s;
  return CF_OK;
}

template <typename S>
static int backward_t(cf_adjoint *a, double *d_lambda0, double *h_dm, cudaStream_t st) {
  cf_ctx *ctx = a->ctx;
  const long long N3 = ctx->N3;
  const size_t sb = a->state_bytes;
  CF_TRY_CUDA(cudaMemsetAsync(a->dm_partial, 0, sizeof(double) * a->dm_slots, st));
  S *Y2 = (S *)a->Y;
  S *Y3 = (S *)((char *)a->Y + sb);
  S *Y4 = (S *)((char *)a->Y + 2 * sb);
  const double dt = a->dt, dh = dt / 2.0, dt6 = dt / 6.0, dt3 = dt / 3.0;
  AdjArgs<S> A{};
  A.N = (int)ctx->N;
  A.N3 = N3;
  A.m2 = ctx->p.m * ctx->p.m;
  A.two_m = 2.0 * ctx->p.m;
  A.dm_partial = a->dm_partial;
  A.acc = a->accb;
  const long long nseg = (long long)a->ckpt.size();
  for (long long sgi = nseg - 1; sgi >= 0; --sgi) {
    const int64_t n0 = sgi * a->every;
    const int64_t len = std::min<int64_t>(a->every, a->nsteps - n0);
    char *seg = (char *)a->seg;
    CF_TRY_CUDA(cudaMemcpyAsync(seg, a->ckpt[sgi], sb, cudaMemcpyDeviceToDevice, st));
    for (int64_t j = 1; j < len; ++j) {
      CF_TRY_CUDA(cudaMemcpyAsync(seg + j * sb, seg + (j - 1) * sb, sb, cudaMemcpyDeviceToDevice, st));
      CF_TRY(rk4_steps(ctx, seg + j * sb, a->t0, dt, n0 + j - 1, 1, st));
    }
    for (int64_t j = len - 1; j >= 0; --j) {
      const int64_t n = n0 + j;
      const double t = a->t0 + (double)n * dt;
      S *x = (S *)(seg + j * sb);
      S *xlo = (sizeof(S) == 4) ? x + 2 * N3 : nullptr;
      // recompute the forward stage inputs y2, y3, y4 of step n (bit-identical to the forward)
      CF_TRY(launch_forward_stage(ctx, 1, x, Y2, x, xlo, t, dh, dt6, st));
      CF_TRY(launch_forward_stage(ctx, 2, Y2, Y3, x, xlo, t + dh, dh, dt6, st));
      CF_TRY(launch_forward_stage(ctx, 3, Y3, Y4, x, xlo, t + dh, dt, dt6, st));
      double inv, H;
      // reverse stage 4 at t + dt: kb4 = dt/6 l'
      stage_coeffs(ctx->p, t + dt, &inv, &H);
      A.inv = inv;
      A.hub3 = 3.0 * H;
      A.kin = a->lam;
      A.sin = dt6;
      A.lamp = a->lam;
      A.knext = a->ka;
      A.cl = dt3;
      A.cy = dt;
      A.yphi = Y4;
      CF_TRY(launch_adj_h<S, 4>(a, A, st));
      // reverse stage 3 at t + dt/2
      stage_coeffs(ctx->p, t + dh, &inv, &H);
      A.inv = inv;
      A.hub3 = 3.0 * H;
      A.kin = a->ka;
      A.sin = 1.0;
      A.knext = a->kb;
      A.cl = dt3;
      A.cy = dh;
      A.yphi = Y3;
      CF_TRY(launch_adj_h<S, 3>(a, A, st));
      // reverse stage 2 at t + dt/2
      A.kin = a->kb;
      A.knext = a->ka;
      A.cl = dt6;
      A.cy = dh;
      A.yphi = Y2;
      CF_TRY(launch_adj_h<S, 2>(a, A, st));
      // reverse stage 1 at t: l = l' + acc + yb1
      stage_coeffs(ctx->p, t, &inv, &H);
      A.inv = inv;
      A.hub3 = 3.0 * H;
      A.kin = a->ka;
      A.knext = nullptr;
      A.lam_out = a->lam;
      A.yphi = x;
      CF_TRY(launch_adj_h<S, 1>(a, A, st));
    }
  }
  if (d_lambda0)
    CF_TRY_CUDA(cudaMemcpyAsync(d_lambda0, a->lam, 2 * N3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
  std::vector<double> part((size_t)a->dm_slots);
  CF_TRY_CUDA(cudaMemcpyAsync(part.data(), a->dm_partial, sizeof(double) * a->dm_slots, cudaMemcpyDeviceToHost, st));
  CF_TRY_CUDA(cudaStreamSynchronize(st));
  double s = a->dm_direct;
  for (double v : part) s += v;
  if (h_dm) *h_dm = s;
  return CF_OK;
}

int adjoint_backward(cf_adjoint *a, double *d_lambda0, double *h_dm, cudaStream_t st) {
  if (!a->have_forward) {
    set_error("adjoint: run cf_adjoint_forward first");
    return CF_ERR_INVALID;
  }
  if (a->ctx->p.precision == CF_FP32_COMP) return backward_t<float>(a, d_lambda0, h_dm, st);
  return backward_t<double>(a, d_lambda0, h_dm, st);
}

int adjoint_set_lambda(cf_adjoint *a, const double *d_lam, double dm_direct, cudaStream_t st) {
  CF_TRY_CUDA(cudaMemcpyAsync(a->lam, d_lam, 16 * (size_t)a->ctx->N3, cudaMemcpyDeviceToDevice, st));
  a->dm_direct = dm_direct;
  return CF_OK;
}

// ---- shell-amplitude parameterisation of the initial field -------------------
static int ensure_z2d(cf_ctx *ctx, cufftHandle *plan) {
  const int N = (int)ctx->N;
  CF_TRY_CUFFT(cufftPlan3d(plan, N, N, N, CUFFT_Z2D));
  return CF_OK;
}

int field_from_shell_amplitudes(cf_ctx *ctx, const double *d_xi, const double *d_sqrtP, const double *h_theta,
                                int ngroups, int spg, double *d_phi, cudaStream_t st) {
  CF_TRY(ensure_spectrum_scratch(ctx, 1));
  std::vector<double> sq(ngroups);
  for (int g = 0; g < ngroups; ++g) sq[g] = std::sqrt(h_theta[g]);
  double *d_sq = nullptr;
  CF_TRY_CUDA(cudaMallocAsync((void **)&d_sq, sizeof(double) * ngroups, st));
  CF_TRY_CUDA(cudaMemcpyAsync(d_sq, sq.data(), sizeof(double) * ngroups, cudaMemcpyHostToDevice, st));
  const long long pairs = ctx->hc_count / 2;
  k_field_from_theta<<<gridn(pairs), 256, 0, st>>>(d_xi, d_sqrtP, d_sq, spg, ngroups, ctx->spec_hc, (int)ctx->N,
                                                   pairs);
  CF_LAUNCHED(ctx);
  cufftHandle plan;
  CF_TRY(ensure_z2d(ctx, &plan));
  cufftSetStream(plan, st);
  cufftResult r = cufftExecZ2D(plan, (cufftDoubleComplex *)ctx->spec_hc, d_phi);
  CF_TRY_CUDA(cudaFreeAsync(d_sq, st));
  CF_TRY_CUDA(cudaStreamSynchronize(st));
  cufftDestroy(plan);
  if (r != CUFFT_SUCCESS) {
    set_error("cufftExecZ2D failed (%d)", (int)r);
    return CF_ERR_CUFFT;
  }
  return CF_OK;
}

int shell_amplitude_gradient(cf_ctx *ctx, const double *d_lambda_phi, const double *d_xi, const double *d_sqrtP,
                             const double *h_theta, int ngroups, int spg, double *h_grad, cudaStream_t st) {
  CF_TRY(ensure_spectrum_scratch(ctx, 1));
  CF_TRY_CUFFT(cufftSetStream(ctx->plan_d2z1, st));
  CF_TRY_CUFFT(cufftExecD2Z(ctx->plan_d2z1, (cufftDoubleReal *)d_lambda_phi, (cufftDoubleComplex *)ctx->spec_hc));
  const long long pairs = ctx->hc_count / 2;
  const unsigned blocks = 148 * 4;
  double *d_part = nullptr;
  CF_TRY_CUDA(cudaMallocAsync((void **)&d_part, sizeof(double) * blocks * ngroups, st));
  k_theta_grad<<<blocks, 256, sizeof(double) * 8 * ngroups, st>>>(d_xi, d_sqrtP, ctx->spec_hc, spg, ngroups, d_part,
                                                                  (int)ctx->N, pairs);
  CF_LAUNCHED(ctx);
  std::vector<double> part((size_t)blocks * ngroups);
  CF_TRY_CUDA(cudaMemcpyAsync(part.data(), d_part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, st));
  CF_TRY_CUDA(cudaFreeAsync(d_part, st));
  CF_TRY_CUDA(cudaStreamSynchronize(st));
  for (int g = 0; g < ngroups; ++g) {
    double s = 0.0;
    for (unsigned b = 0; b < blocks; ++b) s += part[(size_t)b * ngroups + g];
    h_grad[g] = s / (2.0 * std::sqrt(h_theta[g]));
  }
  return CF_OK;
}

}  // namespace cfb

namespace cfb {
cf_ctx *adjoint_ctx(cf_adjoint *a) { return a->ctx; }
}  // namespace cfb
