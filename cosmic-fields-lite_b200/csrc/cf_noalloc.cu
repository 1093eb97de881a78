// cf_noalloc.cu -- cf_rk4_steps_noalloc: the fused RK4 stepper for callers that
// must not allocate device memory.
//
// Some callers cannot let a library call cudaMalloc: host applications that
// hand every byte of device memory to their own pool or arena and forbid other
// allocations, and time-critical loops that cannot afford cudaMalloc's implicit
// synchronisation or its failure in the middle of a run.  cf_rk4_steps allocates
// its three RK4 work buffers (the stage accumulator and two stage-input buffers,
// 2N^3 words each) on first use; this entry point runs the same four stage
// kernels with those buffers carved out of a fixed array compiled into the
// library instead.  The caller still owns the state.
//
// Limits and sharing rules:
//  - The array is kNoAllocScratchBytes (24 MiB), reserved on every GPU that loads
//    the library until the process exits.  It holds 3 * 2N^3 words: N <= 80 in
//    CF_FP64, N <= 96 in CF_FP32_COMP; larger lattices are rejected.
//  - Every call on a device uses the same array, and the array keeps the last
//    call's contents.  Nothing needs to start at zero: each step writes every
//    buffer entry before reading it.  Calls whose GPU work overlaps (other
//    streams, other host threads) race on the array and must be serialised by
//    the caller.
//  - The array is reserved when the library's device code is first loaded on a
//    device.  With lazy module loading (the default since CUDA 12.2) that is the
//    first call of this entry point there, so an application that hands its free
//    device memory to its own pool makes one call first -- a call with
//    nsteps = 0 does only this -- or runs with CUDA_MODULE_LOADING=EAGER.
//  - A call outside stream capture looks up the array's device address
//    (cudaGetSymbolAddress) with the context's device current, so the address
//    stays right after a cudaDeviceReset; a call during capture uses the address
//    of the last call outside capture, so make one such call before capturing.
//  - Flat and FRW Klein-Gordon only: the comoving-curvature equation needs the
//    Psi buffers and cuFFT plans, which allocate.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>

#include "cf_internal.cuh"

namespace cfb {

int rk4_step_buffers(cf_ctx *ctx, void *d_state, void *acc, void *ya, void *yb, double t, double dt,
                     cudaStream_t st);

constexpr size_t kNoAllocScratchBytes = size_t(24) << 20;

// Host code must not use this name as a device address: it is a host-side
// stand-in.  scratch_address() returns the real device address.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
static void *g_scratch_dev[kMaxDevices];
static std::mutex g_scratch_mu;

// Device address of g_noalloc_scratch on the current device: looked up afresh
// outside stream capture (a cudaDeviceReset may have moved it), the last address
// seen on this device during capture.
static int scratch_address(cudaStream_t st, void **out) {
  int dev = 0;
  CF_TRY_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("cf_rk4_steps_noalloc: device ordinal %d out of range", dev);
    return CF_ERR_INVALID;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CF_TRY_CUDA(cudaStreamIsCapturing(st, &cs));
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (cs == cudaStreamCaptureStatusNone) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_error("cf_rk4_steps_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev, cudaGetErrorString(e));
      return CF_ERR_CUDA;
    }
    g_scratch_dev[dev] = p;
  } else if (!g_scratch_dev[dev]) {
    set_error("cf_rk4_steps_noalloc: first call on device %d made during stream capture; make one call "
              "(nsteps = 0 suffices) before capturing", dev);
    return CF_ERR_INVALID;
  }
  *out = g_scratch_dev[dev];
  return CF_OK;
}

}  // namespace cfb

using namespace cfb;

extern "C" int cf_rk4_steps_noalloc(cf_ctx *ctx, void *d_state, double t0, double dt, int64_t step0, int64_t nsteps,
                                    void *stream) {
  if (!ctx) {
    set_error("NULL context");
    return CF_ERR_INVALID;
  }
  if (!d_state || ((uintptr_t)d_state) % 16) {
    set_error("d_state is NULL or not 16-byte aligned");
    return CF_ERR_INVALID;
  }
  if (nsteps < 0 || !std::isfinite(t0) || !std::isfinite(dt)) {
    set_error("nsteps must be >= 0 and t0, dt finite");
    return CF_ERR_INVALID;
  }
  if (ctx->p.equation != CF_EQ_KG && ctx->p.equation != CF_EQ_KG_FRW) {
    set_error("cf_rk4_steps_noalloc covers the flat and FRW Klein-Gordon equations (the other equations "
              "need their own coefficients, curvature buffers or cuFFT plans)");
    return CF_ERR_UNSUPPORTED;
  }
  const size_t buf = 2 * (size_t)ctx->N3 * ctx->word;  // one RK4 work buffer
  if (3 * buf > kNoAllocScratchBytes) {
    set_error("cf_rk4_steps_noalloc: N = %lld needs %zu bytes of RK4 scratch, the fixed array holds %zu "
              "(N <= 80 in FP64, N <= 96 in FP32_COMP)",
              (long long)ctx->N, 3 * buf, kNoAllocScratchBytes);
    return CF_ERR_INVALID;
  }
  // the context's device for the call; the caller's current device afterwards
  int prev = 0;
  CF_TRY_CUDA(cudaGetDevice(&prev));
  struct Restore {
    int dev;
    ~Restore() { cudaSetDevice(dev); }
  } restore{prev};
  CF_TRY_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  void *base = nullptr;
  CF_TRY(scratch_address(st, &base));
  char *p = static_cast<char *>(base);
  for (int64_t j = 0; j < nsteps; ++j) {
    const double t = t0 + (double)(step0 + j) * dt;
    CF_TRY(rk4_step_buffers(ctx, d_state, p, p + buf, p + 2 * buf, t, dt, st));
  }
  return CF_OK;
}
