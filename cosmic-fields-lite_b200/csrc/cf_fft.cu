// cf_fft.cu -- the FFT wrapper role of the reference (cufftWrapperNoBatching,
// src/cuda_wrapper.cuh:113-130, src/cuda_wrapper.cu:202-255; CPU twin fftwWrapper,
// src/fftw_wrapper.cpp:4-76): 3-D FP64 transforms of an N^3 lattice for code
// that calls workspace.fft_wrapper directly (initializers, observers, WKB).
//
// Same conventions as the reference: unnormalised transforms, forward sign
// e^{-2 pi i k.x / N}; the half-complex (HC) layout N x N x (N/2+1) complex with c
// fastest; Z2D overwrites its input (cuFFT's multi-dimensional C2R does); the
// in-place Z2D returns the real field in the padded layout, rows of 2(N/2+1)
// doubles (PADDED_IDX_OF, src/fdm3d.hpp:24).  Plans are created on first use,
// so a handle that is never executed holds no device memory.

#include <cuda_runtime.h>
#include <cufft.h>

#include "cf_internal.cuh"

struct cf_fft {
  int64_t N = 0;
  int device = 0;
  cufftHandle d2z = 0, z2d = 0;
  bool have_d2z = false, have_z2d = false;
};

namespace cfb {

static int fft_fail(const char *msg) {
  set_error("%s", msg);
  return CF_ERR_INVALID;
}

static int fft_use(cf_fft *f) {
  if (!f) return fft_fail("cf_fft handle is NULL");
  CF_TRY_CUDA(cudaSetDevice(f->device));
  return CF_OK;
}

static int fft_plan(cf_fft *f, bool forward) {
  bool &have = forward ? f->have_d2z : f->have_z2d;
  cufftHandle &h = forward ? f->d2z : f->z2d;
  if (have) return CF_OK;
  const int N = (int)f->N;
  CF_TRY_CUFFT(cufftPlan3d(&h, N, N, N, forward ? CUFFT_D2Z : CUFFT_Z2D));
  have = true;
  return CF_OK;
}

static int fft_args(cf_fft *f, const void *a, const void *b) {
  CF_TRY(fft_use(f));
  if (!a || !b) return fft_fail("NULL device pointer");
  if (((uintptr_t)a | (uintptr_t)b) & 15) return fft_fail("device pointers must be 16-byte aligned");
  return CF_OK;
}

}  // namespace cfb

using namespace cfb;

extern "C" {

int cf_fft_create(int64_t N, cf_fft **out) {
  if (!out) return fft_fail("out is NULL");
  *out = nullptr;
  if (N < 8 || N > 2048 || N % 2) {
    set_error("cf_fft_create: N must be even, 8 <= N <= 2048 (got %lld)", (long long)N);
    return CF_ERR_INVALID;
  }
  cf_fft *f = new cf_fft;
  f->N = N;
  if (cudaGetDevice(&f->device) != cudaSuccess) {
    delete f;
    set_error("cf_fft_create: no CUDA device");
    return CF_ERR_CUDA;
  }
  *out = f;
  return CF_OK;
}

int cf_fft_destroy(cf_fft *f) {
  if (!f) return CF_OK;
  cudaSetDevice(f->device);
  if (f->have_d2z) cufftDestroy(f->d2z);
  if (f->have_z2d) cufftDestroy(f->z2d);
  delete f;
  return CF_OK;
}

int cf_fft_d2z(cf_fft *f, const double *d_in, double *d_out, void *stream) {
  CF_TRY(fft_args(f, d_in, d_out));
  CF_TRY(fft_plan(f, true));
  CF_TRY_CUFFT(cufftSetStream(f->d2z, (cudaStream_t)stream));
  CF_TRY_CUFFT(cufftExecD2Z(f->d2z, const_cast<double *>(d_in), (cufftDoubleComplex *)d_out));
  return CF_OK;
}

int cf_fft_batched_d2z(cf_fft *f, const double *d_in, double *d_out, void *stream) {
  CF_TRY(fft_args(f, d_in, d_out));
  CF_TRY(fft_plan(f, true));
  const long long N = f->N, N3 = N * N * N, hc = N * N * (N / 2 + 1);
  CF_TRY_CUFFT(cufftSetStream(f->d2z, (cudaStream_t)stream));
  CF_TRY_CUFFT(cufftExecD2Z(f->d2z, const_cast<double *>(d_in), (cufftDoubleComplex *)d_out));
  CF_TRY_CUFFT(cufftExecD2Z(f->d2z, const_cast<double *>(d_in) + N3, (cufftDoubleComplex *)d_out + hc));
  return CF_OK;
}

int cf_fft_z2d(cf_fft *f, double *d_in, double *d_out, void *stream) {
  CF_TRY(fft_args(f, d_in, d_out));
  CF_TRY(fft_plan(f, false));
  CF_TRY_CUFFT(cufftSetStream(f->z2d, (cudaStream_t)stream));
  CF_TRY_CUFFT(cufftExecZ2D(f->z2d, (cufftDoubleComplex *)d_in, d_out));
  return CF_OK;
}

int cf_fft_inplace_z2d(cf_fft *f, double *d_inout, void *stream) {
  CF_TRY(fft_args(f, d_inout, d_inout));
  CF_TRY(fft_plan(f, false));
  CF_TRY_CUFFT(cufftSetStream(f->z2d, (cudaStream_t)stream));
  CF_TRY_CUFFT(cufftExecZ2D(f->z2d, (cufftDoubleComplex *)d_inout, d_inout));
  return CF_OK;
}

}  // extern "C"
