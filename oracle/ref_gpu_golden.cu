/*
 * ref_gpu_golden.cu -- golden vectors from the reference's OWN GPU functors, for
 * the equations that have no CPU twin in the reference (test infrastructure only).
 *
 * Compiled by oracle/Makefile (target ref-golden) together with the unmodified
 * reference sources src/equations_cuda.cu, src/fdm3d_cuda.cu, src/cuda_wrapper.cu
 * and src/odeint_thrust/thrust_operations.cu, read in place from the reference
 * tree, into oracle/_ref/ref_gpu_golden.  Run on a GPU, it writes raw FP64 files
 * <outdir>/<name>.f64 that tests/golden/make_ref_gpu_golden.py packs into
 * tests/golden/ref_gpu_equations.npz.
 *
 * Inputs are a closed-form integer hash of the site / mode index (mix32 below),
 * so numpy rebuilds them bit for bit (tests/golden/ref_gpu_inputs.py):
 *   phi  = 0.5 (2 u(i, 1) - 1),  dphi = 0.3 (2 u(i, 2) - 1),  Psi = 0.02 (2 u(i, 3) - 1),
 *   R_fft (approximate comoving): mode o with |a|, |b| shifted and c all below BAND
 *   gets 1e-3 (2 u(o, 4) - 1) + 1e-3 i (2 u(o, 5) - 1); the c = 0 plane is made
 *   Hermitian by pairing o with the mode of (-a, -b); every other mode is zero.
 * Parameters: m = 1, lambda = 0.8, f_a = 0.7, a1 = 1, H1 = 0.5, t1 = 1, t = 1.3,
 * dt = 0.05; N = 8, L = 5 for the lambda / sqrt / fixed-curvature / dot-rho cases;
 * N = 16, L = 10, M = 8 for the approximate comoving case (BAND = M/2 = 4), and a
 * second one with BAND = N/2 + 1 (every mode of the N grid populated).
 *
 * It drives the functors as the reference driver does (src/main.cpp:82-196):
 * WorkspaceGeneric<thrust::device_vector<double>>(param, initializer), Equation(workspace),
 * operator()(x, dxdt, t), Equation::compute_energy_density(workspace, t),
 * CudaKleinGordonEquationInFRW::compute_dot_energy_density(workspace, t) and one
 * runge_kutta4_classic<State, double, State, double> do_step.
 *
 * usage: ref_gpu_golden <outdir>
 */
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include <boost/numeric/odeint.hpp>
#include <cuda_runtime.h>
#include <thrust/device_vector.h>

#include "equations_cuda.cuh"
#include "workspace.hpp"

namespace {

uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}

double u01(uint64_t i, uint32_t salt) { return (double)mix32((uint32_t)i * 0x9E3779B9U + salt) / 4294967296.0; }

struct GParam {
  long long int N;
  double L;
  double m;
  double lambda;
  double f_a;
  long long int M;
  double a1;
  double H1;
  double t1;
};

std::string g_dir;

void dump(const std::string &name, const thrust::device_vector<double> &v) {
  std::vector<double> h(v.size());
  thrust::copy(v.begin(), v.end(), h.begin());
  const std::string path = g_dir + "/" + name + ".f64";
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) {
    std::fprintf(stderr, "cannot write %s\n", path.c_str());
    std::exit(2);
  }
  std::fwrite(h.data(), sizeof(double), h.size(), f);
  std::fclose(f);
  std::printf("%s %zu\n", name.c_str(), h.size());
}

std::vector<double> state_of(long long N) {
  const long long N3 = N * N * N;
  std::vector<double> x(2 * N3);
  for (long long i = 0; i < N3; ++i) {
    x[i] = 0.5 * (2 * u01(i, 1) - 1);
    x[N3 + i] = 0.3 * (2 * u01(i, 2) - 1);
  }
  return x;
}

std::vector<double> psi_of(long long N) {
  const long long N3 = N * N * N;
  std::vector<double> p(N3);
  for (long long i = 0; i < N3; ++i) p[i] = 0.02 * (2 * u01(i, 3) - 1);
  return p;
}

std::vector<double> R_fft_of(long long N, long long band) {
  const long long nh = N / 2 + 1;
  std::vector<double> R(2 * N * N * nh, 0.0);
  for (long long a = 0; a < N; ++a)
    for (long long b = 0; b < N; ++b)
      for (long long c = 0; c < nh; ++c) {
        const long long as = a <= N / 2 ? a : N - a, bs = b <= N / 2 ? b : N - b;
        if (as >= band || bs >= band || c >= band) continue;
        const long long o = (a * N + b) * nh + c;
        double re = 1e-3 * (2 * u01(o, 4) - 1), im = 1e-3 * (2 * u01(o, 5) - 1);
        if (c == 0 || c == N / 2) {
          const long long oc = (((N - a) % N) * N + (N - b) % N) * nh + c;
          re = 1e-3 * ((2 * u01(o, 4) - 1) + (2 * u01(oc, 4) - 1));
          im = 1e-3 * ((2 * u01(o, 5) - 1) - (2 * u01(oc, 5) - 1));
        }
        R[2 * o] = re;
        R[2 * o + 1] = im;
      }
  return R;
}

template <typename Equation>
void run_case(const std::string &tag, const GParam &param, bool fixed_psi, bool with_R, long long band,
              bool energy, bool step) {
  typedef typename Equation::State State;
  const long long N = param.N;
  const std::vector<double> x = state_of(N);
  auto init = [&](const GParam &, auto &ws) {
    ws.state = State(x.begin(), x.end());
    if (fixed_psi) {
      const std::vector<double> p = psi_of(N);
      ws.Psi = State(p.begin(), p.end());
    }
    if (with_R) {
      const std::vector<double> R = R_fft_of(N, band);
      ws.R_fft = State(R.begin(), R.end());
    }
  };
  typename Equation::Workspace workspace(param, init);
  Equation eqn(workspace);
  const double t = 1.3, dt = 0.05;
  State dxdt(2 * N * N * N);
  eqn(workspace.state, dxdt, t);
  dump(tag + "_rhs", dxdt);
  if (energy) dump(tag + "_rho", Equation::compute_energy_density(workspace, t));
  if (step) {
    boost::numeric::odeint::runge_kutta4_classic<State, double, State, double> stepper;
    stepper.do_step(eqn, workspace.state, t, dt);
    dump(tag + "_step", workspace.state);
  }
}

void run_dot_rho(const GParam &param) {
  typedef CudaKleinGordonEquationInFRW::State State;
  const std::vector<double> x = state_of(param.N);
  auto init = [&](const GParam &, auto &ws) { ws.state = State(x.begin(), x.end()); };
  CudaKleinGordonEquationInFRW::Workspace workspace(param, init);
  dump("kgfrw_dot_rho", CudaKleinGordonEquationInFRW::compute_dot_energy_density(workspace, 1.3));
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <outdir>\n", argv[0]);
    return 2;
  }
  g_dir = argv[1];
  const GParam small{8, 5.0, 1.0, 0.8, 0.7, 8, 1.0, 0.5, 1.0};
  const GParam approx{16, 10.0, 1.0, 0.0, 1.0, 8, 1.0, 0.5, 1.0};
  run_case<CudaLambdaEquationInFRW>("lambda", small, false, false, 0, true, true);
  run_case<CudaSqrtPotentialEquationInFRW>("sqrt", small, false, false, 0, true, true);
  run_case<CudaFixedCurvatureEquationInFRW>("fixed", small, true, false, 0, true, true);
  run_dot_rho(small);
  run_case<CudaApproximateComovingCurvatureEquationInFRW>("approx", approx, false, true, approx.M / 2, false, false);
  run_case<CudaApproximateComovingCurvatureEquationInFRW>("approx_fullband", approx, false, true, approx.N / 2 + 1,
                                                          false, false);
  const cudaError_t e = cudaDeviceSynchronize();
  std::printf("cuda: %s\n", cudaGetErrorString(e));
  return e == cudaSuccess ? 0 : 1;
}
