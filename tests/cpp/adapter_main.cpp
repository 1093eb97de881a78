// adapter_main.cpp -- drives libcfb200.so through include/cfb200_odeint.hpp the
// way the reference driver (src/main.cpp:82-196) drives its own code:
// POD Param + WorkspaceGeneric(param, initializer) + Equation + observer +
// odeint integrate_const.  Used by tests/test_gpu_adapter.py.
//
// usage: adapter_main <mode> <N> <L> <dt> <t_start> <t_end> <t_interval> <in_state.bin> <out_dir/> [R_fft.bin]
//   mode 0: KleinGordonEquationInFRW with the stock odeint runge_kutta4_classic
//           (device State, cfb200 odeint operations: cf_rhs + cf_scale_sum)
//   mode 1: KleinGordonEquationInFRW with cfb200::fused_rk4 (FP64)
//   mode 2: KleinGordonEquationInFRW with cfb200::fused_rk4, FP32-compensated state
//   mode 3: ComovingCurvatureEquationInFRW with cfb200::fused_rk4 (FP64), R_fft from file
//   mode 4: KleinGordonEquation (flat) with the stock runge_kutta4_classic
//   mode 5: CudaLambdaEquationInFRW (lambda = 0.8) with the stock runge_kutta4_classic
//   mode 6: CudaSqrtPotentialEquationInFRW (f_a = 0.7) with cfb200::fused_rk4
//   mode 7: CudaFixedCurvatureEquationInFRW with cfb200::fused_rk4, Psi (N^3) from file
//   mode 8: CudaApproximateComovingCurvatureEquationInFRW (M = N/2) with cfb200::fused_rk4,
//           R_fft from file
//   mode 10: cfb200::WKBSolutionForKleinGordonEquationInFRW of in_state at t_start,
//           evaluated at t_end; writes out_dir/wkb.dat
//   mode 9: no stepping: the reference driver's initializer run on the device
//           (cfb200::perturbed_grf_and_comoving_curvature_fft with the driver's parameters,
//           src/main.cpp:98-122), RandomNormal seeded with <dt> (an integer; noise_seed < 0:
//           the host stream) or, with <t_start> >= 0, device noise of that seed; writes
//           out_dir/state.dat and out_dir/R_fft.dat
// Writes out_dir/state.dat (final FP64 state), the observer's spectra and density
// files, out_dir/t_list.dat and the parameter files param.dat / paramNames.txt /
// paramTypes.txt.  The initializer also uses workspace.fft_wrapper the way
// the reference's initializers do (src/initializer.hpp:204): out_dir/fft_phi0.dat
// is execute_d2z(phi0), out_dir/fft_roundtrip.dat is execute_z2d of it.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "cfb200_odeint.hpp"

struct FRWParam {
  long long int N;
  double L;
  double m;
  double a1;
  double H1;
  double t1;
  double t_start;
  double t_end;
  double t_interval;
  long long int precision;
  long long int stencil;
};

struct FullParam {
  long long int N;
  double L;
  double m;
  double lambda;
  double f_a;
  long long int M;
  double a1;
  double H1;
  double t1;
  double t_start;
  double t_end;
  double t_interval;
  long long int precision;
  long long int stencil;
};

struct FlatParam {
  long long int N;
  double L;
  double m;
  double t_start;
  double t_end;
  double t_interval;
};

struct DriverParam {  // the fields of the reference driver's MyParam that its initializer reads
  long long int N;
  double L;
  double m;
  double k_ast;
  double varphi_std_dev;
  double Psi_std_dev;
  double a1;
  double H1;
  double t1;
  double t_start;
  long long int noise_seed;
};

static int run_init(long long N, double L, unsigned seed, long long noise_seed, const std::string &dir) {
  DriverParam p{N, L, 1.0, 1.0, 1.0, 0.02, 1.0, 0.05, 1.0 / (2 * 0.05), 1.0 / (2 * 0.05), noise_seed};
  cfb200::RandomNormal::set_generator_seed(seed);
  cfb200::WorkspaceGeneric<cfb200::DeviceState> ws(p, cfb200::perturbed_grf_and_comoving_curvature_fft);
  std::vector<double> h;
  cfb200::copy_vector(h, ws.state);
  cfb200::write_vector_to_file(h, dir + "state.dat");
  cfb200::copy_vector(h, ws.R_fft_device);
  cfb200::write_vector_to_file(h, dir + "R_fft.dat");
  return 0;
}

static std::vector<double> read_file(const std::string &name) {
  std::ifstream f(name, std::ios::binary | std::ios::ate);
  if (!f) {
    std::fprintf(stderr, "cannot open %s\n", name.c_str());
    std::exit(2);
  }
  std::streamsize n = f.tellg();
  f.seekg(0);
  std::vector<double> v((size_t)n / 8);
  f.read(reinterpret_cast<char *>(v.data()), n);
  return v;
}

template <typename Equation, typename Stepper, typename Param>
static int run(const Param &param, const std::vector<double> &x0, const std::vector<double> &R_fft, double dt,
               const std::string &dir) {
  auto init = [&](const auto &p, auto &ws) {
    ws.state.copy_from_host(x0.data(), x0.size());
    ws.R_fft = R_fft;  // the optional input file: R_fft (comoving equations) or Psi (fixed curvature)
    ws.Psi = R_fft;
    const size_t N3 = (size_t)p.N * p.N * p.N;
    cfb200::DeviceState phi;
    phi.copy_from_host(x0.data(), N3);
    cfb200::DeviceState fk = ws.fft_wrapper.execute_d2z(phi);
    std::vector<double> h;
    cfb200::copy_vector(h, fk);
    cfb200::write_vector_to_file(h, dir + "fft_phi0.dat");
    cfb200::DeviceState back = ws.fft_wrapper.execute_z2d(fk);
    cfb200::copy_vector(h, back);
    cfb200::write_vector_to_file(h, dir + "fft_roundtrip.dat");
  };
  cfb200::save_param_for_Mathematica(param, dir);  // src/main.cpp:124
  typename Equation::Workspace workspace(param, init);
  Equation eqn(workspace);
  cfb200::ConstIntervalObserver<Equation, true, true, true> observer(dir, param, eqn);
  Stepper stepper;
  size_t steps = boost::numeric::odeint::integrate_const(stepper, eqn, workspace.state, param.t_start, param.t_end,
                                                          dt, observer);
  observer.flush();
  std::vector<double> out;
  cfb200::copy_vector(out, workspace.state);
  cfb200::write_vector_to_file(out, dir + "state.dat");
  cfb200::write_vector_to_file(workspace.t_list, dir + "t_list.dat");
  std::printf("steps=%zu saves=%zu\n", steps, workspace.t_list.size());
  return 0;
}

int main(int argc, char **argv) {
  if (argc < 10) {
    std::fprintf(stderr, "usage: %s mode N L dt t_start t_end t_interval in_state out_dir [R_fft]\n", argv[0]);
    return 2;
  }
  const int mode = std::atoi(argv[1]);
  if (mode == 9) {
    try {
      return run_init(std::atoll(argv[2]), std::atof(argv[3]), (unsigned)std::atoll(argv[4]), std::atoll(argv[5]),
                      argv[9]);
    } catch (const std::exception &e) {
      std::fprintf(stderr, "error: %s\n", e.what());
      return 1;
    }
  }
  const long long N = std::atoll(argv[2]);
  const double L = std::atof(argv[3]), dt = std::atof(argv[4]);
  const double t0 = std::atof(argv[5]), t1 = std::atof(argv[6]), ti = std::atof(argv[7]);
  const std::vector<double> x0 = read_file(argv[8]);
  const std::string dir = argv[9];
  std::vector<double> R_fft;
  if (argc > 10) R_fft = read_file(argv[10]);
  using cfb200::DeviceState;
  typedef boost::numeric::odeint::runge_kutta4_classic<DeviceState, double, DeviceState, double> StockRK4;
  try {
    FRWParam p{N, L, 1.0, 1.0, 0.5, 1.0, t0, t1, ti, CF_FP64, 7};
    switch (mode) {
      case 0:
        return run<cfb200::KleinGordonEquationInFRW, StockRK4>(p, x0, R_fft, dt, dir);
      case 1:
        return run<cfb200::KleinGordonEquationInFRW, cfb200::fused_rk4>(p, x0, R_fft, dt, dir);
      case 2:
        p.precision = CF_FP32_COMP;
        return run<cfb200::KleinGordonEquationInFRW, cfb200::fused_rk4>(p, x0, R_fft, dt, dir);
      case 3:
        return run<cfb200::ComovingCurvatureEquationInFRW, cfb200::fused_rk4>(p, x0, R_fft, dt, dir);
      case 4: {
        FlatParam q{N, L, 1.0, t0, t1, ti};
        return run<cfb200::KleinGordonEquation, StockRK4>(q, x0, R_fft, dt, dir);
      }
      case 10: {
        auto init = [&](const auto &, auto &w) { w.state.copy_from_host(x0.data(), x0.size()); };
        cfb200::WorkspaceGeneric<cfb200::DeviceState> ws(p, init);
        cfb200::CudaKleinGordonEquationInFRW eqn(ws);
        cfb200::WKBSolutionForKleinGordonEquationInFRW wkb(ws, t0);
        std::vector<double> h;
        cfb200::copy_vector(h, wkb.evaluate_at(t1));
        cfb200::write_vector_to_file(h, dir + "wkb.dat");
        return 0;
      }
      case 5: {
        FullParam q{N, L, 1.0, 0.8, 1.0, 0, 1.0, 0.5, 1.0, t0, t1, ti, CF_FP64, 7};
        return run<cfb200::CudaLambdaEquationInFRW, StockRK4>(q, x0, R_fft, dt, dir);
      }
      case 6: {
        FullParam q{N, L, 1.0, 0.0, 0.7, 0, 1.0, 0.5, 1.0, t0, t1, ti, CF_FP64, 7};
        return run<cfb200::CudaSqrtPotentialEquationInFRW, cfb200::fused_rk4>(q, x0, R_fft, dt, dir);
      }
      case 7: {
        FullParam q{N, L, 1.0, 0.0, 1.0, 0, 1.0, 0.5, 1.0, t0, t1, ti, CF_FP64, 7};
        return run<cfb200::CudaFixedCurvatureEquationInFRW, cfb200::fused_rk4>(q, x0, R_fft, dt, dir);
      }
      case 8: {
        FullParam q{N, L, 1.0, 0.0, 1.0, N / 2, 1.0, 0.5, 1.0, t0, t1, ti, CF_FP64, 7};
        return run<cfb200::CudaApproximateComovingCurvatureEquationInFRW, cfb200::fused_rk4>(q, x0, R_fft, dt,
                                                                                             dir);
      }
      default:
        std::fprintf(stderr, "unknown mode %d\n", mode);
        return 2;
    }
  } catch (const std::exception &e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
