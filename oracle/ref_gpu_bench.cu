/*
 * ref_gpu_bench.cu -- times the reference's OWN GPU stepping path, as a reported
 * baseline (not a checker, not part of the product).
 *
 * BASELINE MEASUREMENT ONLY.  Compiled by oracle/Makefile (target ref-gpu)
 * together with the unmodified reference sources src/equations_cuda.cu,
 * src/fdm3d_cuda.cu, src/cuda_wrapper.cu and src/odeint_thrust/thrust_operations.cu,
 * read in place from the reference tree, into oracle/_ref/ref_gpu_bench.
 *
 * It drives the reference exactly as its driver does (src/main.cpp:82-196):
 *   WorkspaceGeneric<thrust::device_vector<double>>(param, initializer)
 *   CudaKleinGordonEquationInFRW / CudaComovingCurvatureEquationInFRW
 *   runge_kutta4_classic<State, double, State, double> with the reference's
 *   thrust algebra and operations (src/odeint_thrust/)
 * and times `steps` do_step calls after `warmup` with CUDA events on the
 * default stream the reference uses.  The initial field is a seeded
 * superposition of plane waves and the comoving curvature a seeded
 * band-limited HC array: timing does not depend on their values.
 *
 * usage: ref_gpu_bench <equation 1|2> <N> <steps> <warmup>
 *   1 = CudaKleinGordonEquationInFRW, 2 = CudaComovingCurvatureEquationInFRW
 * prints one JSON line.
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include <boost/numeric/odeint.hpp>
#include <cuda_runtime.h>
#include <thrust/device_vector.h>

#include "equations_cuda.cuh"
#include "workspace.hpp"

namespace {

struct BenchParam {
  long long int N;
  double L;
  double m;
  double a1;
  double H1;
  double t1;
};

template <typename Equation>
int run(const BenchParam &param, int steps, int warmup) {
  typedef typename Equation::State State;
  const long long N = param.N, N3 = N * N * N;
  auto init = [&](const BenchParam &, auto &ws) {
    std::vector<double> x(2 * N3, 0.0);
    std::mt19937 rng(7);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    for (int w = 0; w < 8; ++w) {  // a few plane waves of random direction and phase
      const int ka = 1 + (int)(u(rng) * 4), kb = (int)(u(rng) * 4), kc = (int)(u(rng) * 4);
      const double ph = 2 * M_PI * u(rng);
      for (long long a = 0; a < N; ++a)
        for (long long b = 0; b < N; ++b)
          for (long long c = 0; c < N; ++c)
            x[(a * N + b) * N + c] += 0.3 * std::cos(2 * M_PI * (ka * a + kb * b + kc * c) / (double)N + ph);
    }
    ws.state = State(x.begin(), x.end());
    const long long nh = N / 2 + 1;
    std::vector<double> R(2 * N * N * nh, 0.0);
    const long long K = std::max(1LL, (long long)(0.5 * param.L / (2 * M_PI)));  // k_max = 0.5
    for (long long a = 0; a < N; ++a)
      for (long long b = 0; b < N; ++b)
        for (long long c = 0; c <= K && c < nh; ++c) {
          const long long as = a <= N / 2 ? a : N - a, bs = b <= N / 2 ? b : N - b;
          if (as * as + bs * bs + c * c > K * K || as + bs + c == 0) continue;
          R[2 * ((a * N + b) * nh + c)] = 1e-3 * (u(rng) - 0.5);
          R[2 * ((a * N + b) * nh + c) + 1] = 1e-3 * (u(rng) - 0.5);
        }
    ws.R_fft = State(R.begin(), R.end());
  };
  typename Equation::Workspace workspace(param, init);
  Equation eqn(workspace);
  boost::numeric::odeint::runge_kutta4_classic<State, double, State, double> stepper;
  double t = param.t1;
  const double dt = 0.05;
  for (int i = 0; i < warmup; ++i, t += dt) stepper.do_step(eqn, workspace.state, t, dt);
  cudaDeviceSynchronize();
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, 0);
  for (int i = 0; i < steps; ++i, t += dt) stepper.do_step(eqn, workspace.state, t, dt);
  cudaEventRecord(e1, 0);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  const cudaError_t err = cudaGetLastError();
  std::printf("{\"impl\": \"reference_gpu\", \"N\": %lld, \"steps\": %d, \"warmup\": %d, \"ms_per_step\": %.6f, "
              "\"site_updates_per_s\": %.6e, \"cuda\": \"%s\"}\n",
              N, steps, warmup, ms / steps, (double)N3 * steps / (ms * 1e-3), cudaGetErrorString(err));
  return err == cudaSuccess ? 0 : 1;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 5) {
    std::fprintf(stderr, "usage: %s <equation 1|2> <N> <steps> <warmup>\n", argv[0]);
    return 2;
  }
  const int eq = std::atoi(argv[1]);
  BenchParam p{std::atoll(argv[2]), 0.0, 1.0, 1.0, 0.5, 1.0};
  p.L = (double)p.N;
  const int steps = std::atoi(argv[3]), warmup = std::atoi(argv[4]);
  if (eq == 2) return run<CudaComovingCurvatureEquationInFRW>(p, steps, warmup);
  return run<CudaKleinGordonEquationInFRW>(p, steps, warmup);
}
