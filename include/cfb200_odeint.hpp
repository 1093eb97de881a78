/*
 * cfb200_odeint.hpp -- drop-in C++ adapter: the reference's Equation / Workspace /
 * odeint / observer API over the C ABI of libcfb200.so (include/cfb200.h).
 *
 * A reference driver (src/main.cpp:82-196) switches to the B200 path by changing
 * its typedefs, e.g.
 *
 *   #include "cfb200_odeint.hpp"
 *   typedef cfb200::CudaComovingCurvatureEquationInFRW Equation;   // was ComovingCurvatureEquationInFRW
 *   typedef Equation::Workspace Workspace;                          // cfb200::WorkspaceGeneric<DeviceState>
 *   Workspace workspace(param, initializer);                         // initializer fills state / R_fft on the host
 *   Equation eqn(workspace);
 *   cfb200::ConstIntervalObserver<Equation> observer(dir, param, eqn);
 *   auto stepper = cfb200::fused_rk4();                              // or runge_kutta4_classic<State,double,State,double>()
 *   integrate_const(stepper, eqn, workspace.state, param.t_start, param.t_end, param.delta_t, observer);
 *
 * What maps to what:
 *   - State: cfb200::DeviceState (device memory, RAII, deep copy), the role of
 *     thrust::device_vector<double> (src/equations_cuda.cuh:22-23).  odeint traits
 *     is_resizeable / same_size / resize (src/odeint_thrust/thrust_resize.hpp:37-126) and
 *     algebra_dispatcher -> vector_space_algebra (thrust_algebra_dispatcher.hpp:43-47)
 *     are specialised below; operations_dispatcher -> cfb200::device_operations,
 *     whose scale_sum1..6 call cf_scale_sum (replacing
 *     src/odeint_thrust/thrust_operations.cuh:24-353).
 *   - Equation functors: operator()(x, dxdt, t) -> cf_rhs (the stock odeint steppers
 *     then run on the device); compute_energy_density -> cf_energy_density,
 *     compute_dot_energy_density -> cf_dot_energy_density (src/equations_cuda.cuh:21-103:
 *     the KG, FRW, lambda, sqrt-potential, fixed-, comoving- and approximate
 *     comoving-curvature functors).
 *   - cfb200::fused_rk4: a Stepper (concept as in src/midpoint.hpp:25-101) whose
 *     do_step is ONE cf_rk4_steps call (four fused stage kernels).  It is the path
 *     for the FP32-compensated state (Param field `precision` = CF_FP32_COMP).
 *   - WorkspaceGeneric<DeviceState>(param, initializer): the POD-param + concept
 *     field copy of src/workspace.hpp:20-93 (N, L, m, a1/H1/t1, lambda, f_a, M); the
 *     initializer fills state, and R_fft or Psi where the equation needs them, on the
 *     host.  Optional Param fields `precision` and `stencil` (long long) select
 *     CF_FP32_COMP and the 13-point Laplacian.
 *   - ConstIntervalObserver<Equation, field, density, slices>: the save trigger and
 *     the raw FP64 .dat files of src/observer.hpp:64-126.
 *   - compute_power_spectrum / compute_mode_power_spectrum: src/fdm3d_cuda.cuh:22-31.
 *   - WKBSolutionForKleinGordonEquationInFRW (src/wkb.hpp), the initializers
 *     perturbed_grf_and_comoving_curvature_fft / unperturbed_grf with RandomNormal
 *     (src/initializer.hpp, src/random_field.cpp), save_param_for_Mathematica (src/param.hpp).
 *
 * Requirements: C++20, Boost.odeint headers (the reference vendors Boost 1.84),
 * CUDA runtime headers; link libcfb200.so and cudart.
 */
#ifndef CFB200_ODEINT_HPP
#define CFB200_ODEINT_HPP

#include <cuda_runtime.h>

#include <boost/numeric/odeint.hpp>
#include <boost/pfr.hpp>
#include <cmath>
#include <complex>
#include <concepts>
#include <deque>
#include <functional>
#include <random>
#include <cstdio>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "cfb200.h"

namespace cfb200 {

inline void check(int status) {
  if (status != CF_OK) throw std::runtime_error(std::string("cfb200: ") + cf_last_error());
}

inline void check_cuda(cudaError_t e) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("cfb200: CUDA: ") + cudaGetErrorString(e));
}

/* FRW background of constant equation of state (src/physics.hpp:15-56): same
 * members, constructors and formulas, so host-side stage coefficients agree
 * bit for bit with the reference. */
struct StaticEOSCosmology {
  double a1, H1, t1, p;
  StaticEOSCosmology(double a1_, double H1_, double t1_, double p_) : a1(a1_), H1(H1_), t1(t1_), p(p_) {}
  template <typename T>
  StaticEOSCosmology(const T &param) : a1(param.a1), H1(param.H1), t1(param.t1), p(1.0) {}
  StaticEOSCosmology() : a1(1.0), H1(0), t1(0), p(1.0) {}
  double a(double t) const { return a1 * pow(1 + (1 + 1 / p) * H1 * (t - t1), p / (1 + p)); }
  double H(double t) const { return H1 * pow(1 + (1 + 1 / p) * H1 * (t - t1), -1); }
  double eta(double t) const { return (p / (a1 * H1)) * pow(1 + (1 + 1 / p) * H1 * (t - t1), 1 / (1 + p)); }
};

/* Owns one cf_ctx. */
class Context {
 public:
  explicit Context(const cf_params &p) {
    cf_ctx *c = nullptr;
    check(cf_create(&p, &c));
    ctx_ = c;
    check(cf_get_info(ctx_, &info_));
    params_ = p;
  }
  ~Context() { cf_destroy(ctx_); }
  Context(const Context &) = delete;
  Context &operator=(const Context &) = delete;
  cf_ctx *get() const { return ctx_; }
  const cf_info &info() const { return info_; }
  const cf_params &params() const { return params_; }
  cudaStream_t stream() const { return stream_; }
  void set_stream(cudaStream_t s) { stream_ = s; }

 private:
  cf_ctx *ctx_ = nullptr;
  cf_info info_{};
  cf_params params_{};
  cudaStream_t stream_ = nullptr;
};

/* Device buffer of `size()` doubles' worth of bytes (a state of 2N^3 entries in
 * the context's precision, or any FP64 device vector).  Copies are deep. */
class DeviceState {
 public:
  DeviceState() = default;
  explicit DeviceState(size_t n) { resize(n); }
  DeviceState(const DeviceState &o) : ctx(o.ctx), precision(o.precision) {
    resize(o.n_);
    if (n_) check_cuda(cudaMemcpy(p_, o.p_, n_ * 8, cudaMemcpyDeviceToDevice));
  }
  DeviceState(DeviceState &&o) noexcept { swap(o); }
  DeviceState &operator=(DeviceState o) {
    swap(o);
    return *this;
  }
  ~DeviceState() {
    if (p_) cudaFree(p_);
  }
  void resize(size_t n) {
    if (n == n_) return;
    if (p_) cudaFree(p_);
    p_ = nullptr;
    n_ = 0;
    if (n) check_cuda(cudaMalloc(&p_, n * 8));
    n_ = n;
  }
  size_t size() const { return n_; }
  void *data() { return p_; }
  const void *data() const { return p_; }
  double *f64() { return static_cast<double *>(p_); }
  const double *f64() const { return static_cast<const double *>(p_); }
  void swap(DeviceState &o) noexcept {
    std::swap(p_, o.p_);
    std::swap(n_, o.n_);
    std::swap(ctx, o.ctx);
    std::swap(precision, o.precision);
  }
  /* Host FP64 -> device (FP64 layout; a workspace converts to its precision when bound). */
  void copy_from_host(const double *h, size_t n) {
    resize(n);
    check_cuda(cudaMemcpy(p_, h, n * 8, cudaMemcpyHostToDevice));
  }

  std::shared_ptr<Context> ctx;  // set once the state belongs to a bound workspace
  int precision = CF_FP64;

 private:
  void *p_ = nullptr;
  size_t n_ = 0;
};

/* State -> host FP64 [phi | dphi] (copy_vector, src/cuda_wrapper.cu:45-54). */
inline void copy_vector(std::vector<double> &out, const DeviceState &in) {
  out.resize(in.size());
  if (in.ctx && in.precision != CF_FP64) {
    check(cf_state_download(in.ctx->get(), out.data(), in.data(), in.ctx->stream()));
    check_cuda(cudaStreamSynchronize(in.ctx->stream()));
  } else {
    check_cuda(cudaMemcpy(out.data(), in.data(), in.size() * 8, cudaMemcpyDeviceToHost));
  }
}

/* ---- FFT wrapper (cufftWrapperNoBatching, src/cuda_wrapper.cuh:113-130, and its
 * dispatcher, src/dispatcher.hpp:24-46): what workspace.fft_wrapper gives the
 * reference's initializers, observers and WKB code.  FP64 vectors in the
 * reference's layouts; unnormalised transforms on the default stream, like the
 * reference's.  execute_z2d overwrites its input, as cuFFT's does there. */
class FFTWrapper {
 public:
  int N;
  explicit FFTWrapper(int N_) : N(N_) { check(cf_fft_create(N_, &h_)); }
  ~FFTWrapper() { cf_fft_destroy(h_); }
  FFTWrapper(const FFTWrapper &) = delete;
  FFTWrapper &operator=(const FFTWrapper &) = delete;

  DeviceState execute_d2z(DeviceState &in) {
    DeviceState out(hc());
    check(cf_fft_d2z(h_, in.f64(), out.f64(), nullptr));
    return out;
  }
  DeviceState execute_batched_d2z(DeviceState &in) {
    DeviceState out(2 * hc());
    check(cf_fft_batched_d2z(h_, in.f64(), out.f64(), nullptr));
    return out;
  }
  DeviceState execute_z2d(DeviceState &in) {
    DeviceState out((size_t)N * N * N);
    check(cf_fft_z2d(h_, in.f64(), out.f64(), nullptr));
    return out;
  }
  void execute_inplace_z2d(DeviceState &inout) { check(cf_fft_inplace_z2d(h_, inout.f64(), nullptr)); }

 private:
  size_t hc() const { return 2 * (size_t)N * N * (N / 2 + 1); }
  cf_fft *h_ = nullptr;
};

template <typename Vector>
struct fftWrapperDispatcher;
template <>
struct fftWrapperDispatcher<DeviceState> {
  typedef FFTWrapper Generic;
};

/* odeint operations for DeviceState (replaces thrust_operations::scale_sumN). */
struct device_operations {
  template <size_t K>
  struct scale_sum_k {
    double alpha[K];
    template <typename... S>
    void apply(DeviceState &out, const S &...in) const {
      const double *ptrs[K] = {in.f64()...};
      std::shared_ptr<Context> c = out.ctx;
      ((c = c ? c : in.ctx), ...);
      if (!c) throw std::runtime_error("cfb200: scale_sum on states without a context");
      check(cf_scale_sum(c->get(), out.f64(), (int)K, ptrs, alpha, (int64_t)out.size(), c->stream()));
    }
  };
  template <class F1 = double>
  struct scale_sum1 : scale_sum_k<1> {
    typedef void result_type;
    scale_sum1(F1 a1) { this->alpha[0] = a1; }
    void operator()(DeviceState &o, const DeviceState &s1) const { this->apply(o, s1); }
  };
  template <class F1 = double, class F2 = F1>
  struct scale_sum2 : scale_sum_k<2> {
    typedef void result_type;
    scale_sum2(F1 a1, F2 a2) { this->alpha[0] = a1, this->alpha[1] = a2; }
    void operator()(DeviceState &o, const DeviceState &s1, const DeviceState &s2) const { this->apply(o, s1, s2); }
  };
  template <class F1 = double, class F2 = F1, class F3 = F2>
  struct scale_sum3 : scale_sum_k<3> {
    typedef void result_type;
    scale_sum3(F1 a1, F2 a2, F3 a3) { this->alpha[0] = a1, this->alpha[1] = a2, this->alpha[2] = a3; }
    void operator()(DeviceState &o, const DeviceState &s1, const DeviceState &s2, const DeviceState &s3) const {
      this->apply(o, s1, s2, s3);
    }
  };
  template <class F1 = double, class F2 = F1, class F3 = F2, class F4 = F3>
  struct scale_sum4 : scale_sum_k<4> {
    typedef void result_type;
    scale_sum4(F1 a1, F2 a2, F3 a3, F4 a4) {
      this->alpha[0] = a1, this->alpha[1] = a2, this->alpha[2] = a3, this->alpha[3] = a4;
    }
    void operator()(DeviceState &o, const DeviceState &s1, const DeviceState &s2, const DeviceState &s3,
                    const DeviceState &s4) const {
      this->apply(o, s1, s2, s3, s4);
    }
  };
  template <class F1 = double, class F2 = F1, class F3 = F2, class F4 = F3, class F5 = F4>
  struct scale_sum5 : scale_sum_k<5> {
    typedef void result_type;
    scale_sum5(F1 a1, F2 a2, F3 a3, F4 a4, F5 a5) {
      this->alpha[0] = a1, this->alpha[1] = a2, this->alpha[2] = a3, this->alpha[3] = a4, this->alpha[4] = a5;
    }
    void operator()(DeviceState &o, const DeviceState &s1, const DeviceState &s2, const DeviceState &s3,
                    const DeviceState &s4, const DeviceState &s5) const {
      this->apply(o, s1, s2, s3, s4, s5);
    }
  };
  template <class F1 = double, class F2 = F1, class F3 = F2, class F4 = F3, class F5 = F4, class F6 = F5>
  struct scale_sum6 : scale_sum_k<6> {
    typedef void result_type;
    scale_sum6(F1 a1, F2 a2, F3 a3, F4 a4, F5 a5, F6 a6) {
      this->alpha[0] = a1, this->alpha[1] = a2, this->alpha[2] = a3, this->alpha[3] = a4, this->alpha[4] = a5,
      this->alpha[5] = a6;
    }
    void operator()(DeviceState &o, const DeviceState &s1, const DeviceState &s2, const DeviceState &s3,
                    const DeviceState &s4, const DeviceState &s5, const DeviceState &s6) const {
      this->apply(o, s1, s2, s3, s4, s5, s6);
    }
  };
};

/* ---- workspace (src/workspace.hpp:20-93) ---------------------------------- */
#define CFB200_TYPE_REQUIREMENT(value, type) \
  { std::remove_cvref_t<decltype((value))>() } -> std::same_as<type>;

template <typename Param>
concept HasLatticeParams = requires(Param param) {
  CFB200_TYPE_REQUIREMENT(param.N, long long int)
  CFB200_TYPE_REQUIREMENT(param.L, double)
};
template <typename Param>
concept HasMass = requires(Param param) { CFB200_TYPE_REQUIREMENT(param.m, double) };
template <typename Param>
concept HasFRWParameters = requires(Param param) {
  CFB200_TYPE_REQUIREMENT(param.a1, double)
  CFB200_TYPE_REQUIREMENT(param.H1, double)
  CFB200_TYPE_REQUIREMENT(param.t1, double)
};
template <typename Param>
concept HasLambda = requires(Param param) { CFB200_TYPE_REQUIREMENT(param.lambda, double) };
template <typename Param>
concept HasFa = requires(Param param) { CFB200_TYPE_REQUIREMENT(param.f_a, double) };
template <typename Param>
concept HasPsiApproximationParameters = requires(Param param) { CFB200_TYPE_REQUIREMENT(param.M, long long int) };
template <typename Param>
concept HasPrecision = requires(Param param) { CFB200_TYPE_REQUIREMENT(param.precision, long long int) };
template <typename Param>
concept HasStencil = requires(Param param) { CFB200_TYPE_REQUIREMENT(param.stencil, long long int) };

template <typename Vector = DeviceState>
struct WorkspaceGeneric {
  typedef Vector State;
  long long int N;
  double L;
  double m = 0.0;
  StaticEOSCosmology cosmology{};
  State state;                 /* filled by the initializer with host data (FP64 [phi|dphi]) */
  double lambda{0};
  double f_a{1.0};
  std::vector<double> Psi;     /* host N^3 fixed curvature (fixed-curvature equation) */
  std::vector<double> R_fft;   /* host HC array of the comoving curvature (comoving equations) */
  DeviceState R_fft_device;    /* or the same array on the device (the GPU initializers fill this) */
  long long int M = 0;         /* coarse grid of the approximate comoving equation */
  std::vector<double> t_list;
  int precision = CF_FP64;
  int stencil = 7;
  std::shared_ptr<Context> ctx; /* created when an Equation binds the workspace */
  int equation = -1;
  typename fftWrapperDispatcher<Vector>::Generic fft_wrapper; /* src/workspace.hpp:79 */

  template <HasLatticeParams Param, typename Init>
  WorkspaceGeneric(const Param &param, Init &initializer)
      : N(param.N), L(param.L), fft_wrapper((int)param.N) {
    if constexpr (HasFRWParameters<Param>) cosmology = StaticEOSCosmology(param);
    if constexpr (HasMass<Param>) m = param.m;
    if constexpr (HasLambda<Param>) lambda = param.lambda;
    if constexpr (HasFa<Param>) f_a = param.f_a;
    if constexpr (HasPsiApproximationParameters<Param>) M = param.M;
    if constexpr (HasPrecision<Param>) precision = (int)param.precision;
    if constexpr (HasStencil<Param>) stencil = (int)param.stencil;
    initializer(param, *this);
  }

  /* Creates the context for `eq` and converts the state to its precision. */
  void bind(int eq) {
    if (ctx && equation == eq) return;
    cf_params p{};
    p.N = N;
    p.L = L;
    p.m = m;
    p.a1 = cosmology.a1;
    p.H1 = cosmology.H1;
    p.t1 = cosmology.t1;
    p.p = cosmology.p;
    p.equation = eq;
    p.precision = precision;
    p.stencil = stencil;
    p.lambda = lambda;
    p.f_a = f_a;
    p.M = M;
    ctx = std::make_shared<Context>(p);
    equation = eq;
    if (eq == CF_EQ_COMOVING_FRW || eq == CF_EQ_APPROX_COMOVING_FRW) {
      const size_t hc = (size_t)ctx->info().hc_count;
      if (R_fft_device.size() == hc)
        check(cf_set_R_fft(ctx->get(), R_fft_device.f64(), 1, ctx->stream()));
      else if (R_fft.size() == hc)
        check(cf_set_R_fft(ctx->get(), R_fft.data(), 0, ctx->stream()));
      else
        throw std::runtime_error("cfb200: comoving-curvature equation needs workspace.R_fft (HC array)");
    }
    if (eq == CF_EQ_FIXED_CURVATURE_FRW) {
      if (Psi.size() != (size_t)ctx->info().field_count)
        throw std::runtime_error("cfb200: fixed-curvature equation needs workspace.Psi (N^3 field)");
      check(cf_set_psi(ctx->get(), Psi.data(), 0, ctx->stream()));
    }
    if (precision != CF_FP64 && state.precision == CF_FP64 && state.size()) {
      State conv(state.size());
      check(cf_state_import(ctx->get(), conv.data(), state.f64(), ctx->stream()));
      check_cuda(cudaStreamSynchronize(ctx->stream()));
      state.swap(conv);
    }
    state.ctx = ctx;
    state.precision = precision;
  }
};

typedef WorkspaceGeneric<DeviceState> Workspace;

/* ---- equations (src/equations_cuda.cuh:21-103, src/equations.hpp:36-117) -- */
template <int EQ>
struct DeviceEquation {
  typedef DeviceState Vector;
  typedef Vector State;
  typedef WorkspaceGeneric<Vector> Workspace;
  Workspace &workspace;

  explicit DeviceEquation(Workspace &ws) : workspace(ws) { workspace.bind(EQ); }

  /* dxdt = f(x, t) on the device (FP64 states; the odeint building-block path). */
  void operator()(const State &x, State &dxdt, const double t) {
    if (workspace.precision != CF_FP64)
      throw std::runtime_error("cfb200: the odeint building-block path is FP64; use cfb200::fused_rk4");
    dxdt.ctx = workspace.ctx;
    check(cf_rhs(workspace.ctx->get(), x.f64(), dxdt.f64(), t, workspace.ctx->stream()));
  }

  /* Energy density (N^3 FP64 on the device) of workspace.state at time t. */
  static Vector compute_energy_density(Workspace &ws, const double t) {
    Vector rho((size_t)ws.ctx->info().field_count);
    rho.ctx = ws.ctx;
    check(cf_energy_density(ws.ctx->get(), ws.state.data(), t, rho.f64(), ws.ctx->stream()));
    return rho;
  }

  /* d rho / dt of workspace.state at time t (CudaKleinGordonEquationInFRW only). */
  static Vector compute_dot_energy_density(Workspace &ws, const double t) {
    Vector out((size_t)ws.ctx->info().field_count);
    out.ctx = ws.ctx;
    check(cf_dot_energy_density(ws.ctx->get(), ws.state.data(), t, out.f64(), ws.ctx->stream()));
    return out;
  }
};

typedef DeviceEquation<CF_EQ_KG> KleinGordonEquation;
typedef DeviceEquation<CF_EQ_KG_FRW> KleinGordonEquationInFRW;
typedef DeviceEquation<CF_EQ_KG_FRW> CudaKleinGordonEquationInFRW;
typedef DeviceEquation<CF_EQ_COMOVING_FRW> ComovingCurvatureEquationInFRW;
typedef DeviceEquation<CF_EQ_COMOVING_FRW> CudaComovingCurvatureEquationInFRW;
typedef DeviceEquation<CF_EQ_LAMBDA_FRW> CudaLambdaEquationInFRW;
typedef DeviceEquation<CF_EQ_SQRT_FRW> CudaSqrtPotentialEquationInFRW;
typedef DeviceEquation<CF_EQ_FIXED_CURVATURE_FRW> CudaFixedCurvatureEquationInFRW;
typedef DeviceEquation<CF_EQ_APPROX_COMOVING_FRW> CudaApproximateComovingCurvatureEquationInFRW;

/* ---- fused RK4 stepper (Stepper concept, src/midpoint.hpp:25-101) ---------- */
class fused_rk4 {
 public:
  typedef DeviceState state_type;
  typedef DeviceState deriv_type;
  typedef double value_type;
  typedef double time_type;
  typedef unsigned short order_type;
  typedef boost::numeric::odeint::stepper_tag stepper_category;
  static order_type order() { return 4; }

  template <class System>
  void do_step(System system, state_type &x, time_type t, time_type dt) {
    typename boost::numeric::odeint::unwrap_reference<System>::type &sys = system;
    auto &ws = sys.workspace;
    check(cf_rk4_steps(ws.ctx->get(), x.data(), t, dt, 0, 1, ws.ctx->stream()));
  }
};

/* ---- spectra (src/fdm3d_cuda.cuh:22-31) ----------------------------------- */
inline DeviceState compute_power_spectrum(const long long int N, const DeviceState &f, Context &ctx) {
  (void)N;
  DeviceState out((size_t)ctx.info().s2_bins);
  check(cf_power_spectrum_s2(ctx.get(), f.f64(), out.f64(), ctx.stream()));
  return out;
}

inline DeviceState compute_mode_power_spectrum(const long long int N, const double L, const double m,
                                               const double a_t, const DeviceState &state, Context &ctx) {
  (void)N, (void)L, (void)m;
  DeviceState out((size_t)ctx.info().s2_bins);
  check(cf_mode_power_spectrum_s2(ctx.get(), state.data(), a_t, out.f64(), ctx.stream()));
  return out;
}

/* ---- initial conditions on the device (src/initializer.hpp:33-301,
 * src/random_field.cpp:13-134, src/fdm3d.cpp:76-102) ----------------------------
 * The reference's initializers draw from one std::mt19937 + std::normal_distribution
 * stream and transform on the host.  These draw the SAME stream on the host (so a
 * seed gives the reference's fields) -- or, when the Param has `noise_seed` >= 0,
 * counter-based deviates on the device (cf_white_noise; fast at large N, a different
 * but equally distributed stream) -- and do every transform and per-mode product on
 * the device (cf_grf, cf_scale_modes). */
namespace RandomNormal {
inline std::mt19937 mt{std::random_device{}()};
inline std::normal_distribution<double> dist{0.0, 1.0};
inline void set_generator_seed(std::mt19937::result_type seed) { mt = std::mt19937{seed}; }
inline double generate_random_normal() { return dist(mt); }
}  // namespace RandomNormal

typedef std::function<double(double)> Spectrum;

/* The spectrum factories of src/random_field.cpp:92-134 (same formulas). */
inline Spectrum power_law_with_cutoff_given_amplitude_3d(long long N, double L, double sigma, double k_ast,
                                                         double alpha) {
  const double pi = 3.14159265358979323846;
  if (!(alpha >= -3.0) || !(k_ast * L / (2 * pi) > 1.0))
    throw std::runtime_error("cfb200: power-law spectrum needs alpha >= -3 and k_ast above the box's k_IR");
  double P_k_ast = alpha == -3.0
                       ? 2 * pi * pi * sigma * sigma / (k_ast * k_ast * k_ast * log(k_ast * L / (2 * pi)))
                       : (3 + alpha) * 2 * pi * pi * sigma * sigma * (L * L * L * pow(k_ast * L, alpha)) /
                             (pow(k_ast * L, alpha + 3) - pow(2 * pi, alpha + 3));
  P_k_ast *= (N / L) * (N / L) * (N / L);
  return [=](double k) { return k == 0.0 ? 0.0 : (P_k_ast * (k <= k_ast ? pow(k / k_ast, alpha) : 0.0)); };
}

inline Spectrum scale_invariant_spectrum_3d(long long N, double L, double A_s) {
  const double pi = 3.14159265358979323846;
  const double k0 = 1.0;
  double P_k0 = A_s / ((k0 * k0 * k0) / (2 * pi * pi));
  P_k0 *= (N / L) * (N / L) * (N / L);
  return [=](double k) { return k == 0.0 ? 0.0 : (P_k0 * pow(k / k0, -3)); };
}

inline Spectrum to_deriv_spectrum(double m, const Spectrum &P_f) {
  return [m, P_f](double k) { return (k * k + m * m) * P_f(k); };
}

inline Spectrum to_deriv_spectrum(double m, double a, const Spectrum &P_f) {
  return [m, a, P_f](double k) { return (k * k / (a * a) + m * m) * P_f(k); };
}

/* Cosine integral Ci(x), x > 0: the power series gamma + ln x + sum_k (-x^2)^k / (2k (2k)!)
 * (A&S 5.2.16) up to x = 2; beyond, Ci(x) = -Re E1(ix) with E1 from its continued fraction
 * (A&S 5.1.22), evaluated by the modified Lentz method.  (The reference evaluates a Pade
 * approximant; both agree to rounding on the arguments its initializer uses.) */
inline double cosine_integral(double x) {
  const double euler = 0.57721566490153286061;
  if (x <= 2.0) {
    double sum = 0.0, term = 1.0;
    for (int k = 1; k < 80; ++k) {
      term *= -x * x / ((2.0 * k - 1) * (2.0 * k));
      const double t = term / (2.0 * k);
      sum += t;
      if (std::fabs(t) < 1e-18 * std::fabs(sum)) break;
    }
    return euler + std::log(x) + sum;
  }
  std::complex<double> b(1.0, x), c(1e300, 0.0), d = 1.0 / b, h = d;
  for (int i = 1; i < 1000; ++i) {
    const double a = -(double)i * i;
    b += 2.0;
    d = 1.0 / (a * d + b);
    c = b + a / c;
    const std::complex<double> del = c * d;
    h *= del;
    if (std::abs(del - 1.0) < 1e-16) break;
  }
  h *= std::complex<double>(std::cos(x), -std::sin(x));
  return -h.real();
}

template <typename Param>
concept HasNoiseSeed = requires(Param param) { CFB200_TYPE_REQUIREMENT(param.noise_seed, long long int) };

/* The deviates of successive fields: the host stream (RandomNormal) or the device
 * counter stream of `seed`, N^3 per field in the reference's order. */
class NoiseSource {
 public:
  NoiseSource(Context &ctx, long long seed) : ctx_(ctx), seed_(seed) {}
  void next(DeviceState &out) {
    const size_t n = (size_t)ctx_.info().field_count;
    if (seed_ >= 0) {
      out.resize(n);
      check(cf_white_noise(ctx_.get(), (uint64_t)seed_, pos_, out.f64(), (int64_t)n, ctx_.stream()));
    } else {
      std::vector<double> h(n);
      for (auto &v : h) v = RandomNormal::generate_random_normal();
      out.copy_from_host(h.data(), n);
    }
    pos_ += n;
  }

 private:
  Context &ctx_;
  long long seed_;
  uint64_t pos_ = 0;
};

/* Per-s^2 tables of a spectrum / kernel, with |k| formed as the reference forms it. */
inline std::vector<double> sqrtP_by_s2(const Context &ctx, const Spectrum &P) {
  const double pi = 3.14159265358979323846, L = ctx.params().L;
  std::vector<double> t((size_t)ctx.info().s2_bins);
  for (size_t s2 = 0; s2 < t.size(); ++s2) t[s2] = sqrt(P(sqrt((double)s2) * 2 * pi / L));  // random_field.cpp:67-68
  return t;
}

inline std::vector<double> kernel_by_s2(const Context &ctx, const std::function<double(double)> &kernel) {
  const double pi = 3.14159265358979323846, L = ctx.params().L;
  const long long N = ctx.params().N;
  std::vector<double> t((size_t)ctx.info().s2_bins);
  for (size_t s2 = 0; s2 < t.size(); ++s2) t[s2] = kernel(sqrt((double)s2) * (2 * pi / L)) / (N * N * N);  // fdm3d.cpp:94
  return t;
}

/* generate_inhomogeneous_gaussian_random_field (src/random_field.cpp:36-83): Psi may be
 * null (generate_gaussian_random_field); the field's modulation is exp(psi_scale Psi). */
inline DeviceState generate_inhomogeneous_gaussian_random_field(Context &ctx, NoiseSource &noise, const DeviceState *Psi,
                                                                double psi_scale, const Spectrum &P) {
  DeviceState f;
  noise.next(f);
  const std::vector<double> t = sqrtP_by_s2(ctx, P);
  check(cf_grf(ctx.get(), f.f64(), Psi ? Psi->f64() : nullptr, Psi ? psi_scale : 0.0, t.data(), f.f64(),
               ctx.stream()));
  return f;
}

/* compute_field_with_scaled_fourier_modes (src/fdm3d.cpp:76-102). */
inline DeviceState compute_field_with_scaled_fourier_modes(Context &ctx, const DeviceState &f,
                                                           const std::function<double(double)> &kernel) {
  DeviceState out(f.size());
  const std::vector<double> t = kernel_by_s2(ctx, kernel);
  check(cf_scale_modes(ctx.get(), f.f64(), t.data(), out.f64(), ctx.stream()));
  return out;
}

/* A context for the initializers (cuFFT plans and scratch), freed when they return. */
template <typename Param>
inline std::shared_ptr<Context> init_context(const Param &param) {
  cf_params p{};
  p.N = param.N;
  p.L = param.L;
  p.m = param.m;
  p.a1 = 1.0;
  p.p = 1.0;
  p.equation = CF_EQ_KG;
  p.precision = CF_FP64;
  p.stencil = 7;
  p.f_a = 1.0;
  return std::make_shared<Context>(p);
}

template <typename Param>
inline long long noise_seed_of(const Param &param) {
  if constexpr (HasNoiseSeed<Param>) return param.noise_seed;
  return -1;
}

/* perturbed_grf_and_comoving_curvature_fft (src/initializer.hpp:150-206) on the device:
 * the initializer of the reference driver.  Fills workspace.state ([phi | dphi] FP64)
 * and workspace.R_fft_device. */
inline auto perturbed_grf_and_comoving_curvature_fft = [](const auto &param, auto &workspace) {
  const double pi = 3.14159265358979323846;
  auto ctx = init_context(param);
  NoiseSource noise(*ctx, noise_seed_of(param));
  const double eta_i = workspace.cosmology.eta(param.t_start);
  const double L = param.L;
  const double A_s =
      (-576 * pow(pi, 6) * pow(eta_i, 6) * pow(param.Psi_std_dev, 2)) /
      (-81 * pow(L, 4) * (pow(L, 2) + 2 * pow(pi, 2) * pow(eta_i, 2)) +
       L * (81 * pow(L, 5) - 54 * pow(L, 3) * pow(pi, 2) * pow(eta_i, 2) + 48 * L * pow(pi, 4) * pow(eta_i, 4)) *
           cos((4 * pi * eta_i) / (sqrt(3) * L)) +
       256 * pow(pi, 6) * pow(eta_i, 6) * cosine_integral((4 * pi * eta_i) / (sqrt(3) * L)) +
       4 * sqrt(3) * L * pi * eta_i * (27 * pow(L, 4) + 6 * pow(L, 2) * pow(pi, 2) * pow(eta_i, 2) - 16 * pow(pi, 4) * pow(eta_i, 4)) *
           sin((4 * pi * eta_i) / (sqrt(3) * L)));
  DeviceState R = generate_inhomogeneous_gaussian_random_field(*ctx, noise, nullptr, 0.0,
                                                               scale_invariant_spectrum_3d(param.N, L, A_s));
  auto kernel = [eta_i](double k) {
    return k == 0.0 ? 0.0
                    : (6 * sqrt(3) * (-((k * eta_i * cos((k * eta_i) / sqrt(3))) / sqrt(3)) + sin((k * eta_i) / sqrt(3)))) /
                          (pow(k, 3) * pow(eta_i, 3));
  };
  DeviceState Psi = compute_field_with_scaled_fourier_modes(*ctx, R, kernel);
  const double v = param.k_ast / (param.a1 * param.m);
  const double alpha_varphi_sqr = 0.5 * (-3 * pow(4 * pow(v, 2) + 5, 2)) / (12 * pow(v, 4) + 50 * pow(v, 2) + 50);
  const double alpha_dot_varphi_sqr = 0.5 * (25 - 20 * pow(v, 2)) / (12 * pow(v, 4) + 50 * pow(v, 2) + 50);
  Spectrum P_f = power_law_with_cutoff_given_amplitude_3d(param.N, L, param.varphi_std_dev, param.k_ast, 0);
  Spectrum P_dtf = to_deriv_spectrum(param.m, P_f);
  DeviceState varphi = generate_inhomogeneous_gaussian_random_field(*ctx, noise, &Psi, alpha_varphi_sqr, P_f);
  DeviceState dt_varphi = generate_inhomogeneous_gaussian_random_field(*ctx, noise, &Psi, alpha_dot_varphi_sqr, P_dtf);
  const size_t N3 = varphi.size();
  workspace.state.resize(2 * N3);
  check_cuda(cudaMemcpyAsync(workspace.state.f64(), varphi.f64(), N3 * 8, cudaMemcpyDeviceToDevice, ctx->stream()));
  check_cuda(cudaMemcpyAsync(workspace.state.f64() + N3, dt_varphi.f64(), N3 * 8, cudaMemcpyDeviceToDevice,
                             ctx->stream()));
  workspace.R_fft_device = workspace.fft_wrapper.execute_d2z(R);
  check_cuda(cudaDeviceSynchronize());
};

/* unperturbed_grf (src/initializer.hpp:33-44) on the device. */
inline auto unperturbed_grf = [](const auto &param, auto &workspace) {
  auto ctx = init_context(param);
  NoiseSource noise(*ctx, noise_seed_of(param));
  Spectrum P_f = power_law_with_cutoff_given_amplitude_3d(param.N, param.L, param.varphi_std_dev, param.k_ast, 0);
  Spectrum P_dtf = to_deriv_spectrum(param.m, P_f);
  DeviceState varphi = generate_inhomogeneous_gaussian_random_field(*ctx, noise, nullptr, 0.0, P_f);
  DeviceState dt_varphi = generate_inhomogeneous_gaussian_random_field(*ctx, noise, nullptr, 0.0, P_dtf);
  const size_t N3 = varphi.size();
  workspace.state.resize(2 * N3);
  check_cuda(cudaMemcpyAsync(workspace.state.f64(), varphi.f64(), N3 * 8, cudaMemcpyDeviceToDevice, ctx->stream()));
  check_cuda(cudaMemcpyAsync(workspace.state.f64() + N3, dt_varphi.f64(), N3 * 8, cudaMemcpyDeviceToDevice,
                             ctx->stream()));
  check_cuda(cudaDeviceSynchronize());
};

/* ---- WKB continuation (src/wkb.hpp:13-27, src/wkb.cpp:5-121) ----------------
 * Same members and calls as the reference: construct from a workspace whose state is
 * taken at t_i, then evaluate_at(t) returns the continued FP64 [phi | dphi] on the
 * device.  Radiation domination with t1 = 1/(2 H1) only, as in the reference. */
struct WKBSolutionForKleinGordonEquationInFRW {
  typedef DeviceState Vector;
  typedef Vector State;
  typedef WorkspaceGeneric<Vector> Workspace;

  Workspace &workspace;
  double t_i;

  WKBSolutionForKleinGordonEquationInFRW(Workspace &ws, const double t_i_) : workspace(ws), t_i(t_i_) {
    if (!ws.ctx) ws.bind(CF_EQ_KG_FRW);
    const size_t n = 2 * (size_t)ws.ctx->info().field_count;
    if (ws.state.precision == CF_FP64) {
      check(cf_wkb_create(ws.ctx->get(), ws.state.f64(), t_i, &h_, ws.ctx->stream()));
    } else {  // the modes are taken from the FP64 value of an FP32 hi + lo state
      DeviceState x(n);
      check(cf_state_export(ws.ctx->get(), x.f64(), ws.state.data(), ws.ctx->stream()));
      check(cf_wkb_create(ws.ctx->get(), x.f64(), t_i, &h_, ws.ctx->stream()));
      check_cuda(cudaStreamSynchronize(ws.ctx->stream()));
    }
  }
  ~WKBSolutionForKleinGordonEquationInFRW() { cf_wkb_destroy(h_); }
  WKBSolutionForKleinGordonEquationInFRW(const WKBSolutionForKleinGordonEquationInFRW &) = delete;
  WKBSolutionForKleinGordonEquationInFRW &operator=(const WKBSolutionForKleinGordonEquationInFRW &) = delete;

  Vector evaluate_at(const double t) {
    Vector out(2 * (size_t)workspace.ctx->info().field_count);
    check(cf_wkb_evaluate(h_, t, out.f64(), workspace.ctx->stream()));
    return out;
  }

 private:
  cf_wkb *h_ = nullptr;
};

/* ---- raw FP64 file output (src/io.cpp:53-62) ------------------------------- */
inline void write_vector_to_file(const std::vector<double> &v, const std::string &filename) {
  std::ofstream file(filename, std::ios::binary);
  if (file.is_open()) file.write(reinterpret_cast<const char *>(v.data()), v.size() * sizeof(double));
}

inline void write_vector_to_filename_template(const std::vector<double> &v, const std::string &fmt, int idx) {
  char name[512];
  std::snprintf(name, sizeof(name), fmt.c_str(), idx);
  write_vector_to_file(v, name);
}

/* ---- parameter files (src/param.hpp:40-125) ---------------------------------
 * The reference saves its POD Param three ways for Python / Mathematica readers
 * (plot_util.py:17-34): param.dat (the struct's raw bytes), paramNames.txt (one field
 * name per line) and paramTypes.txt ("Real64" / "Integer64" per line).  Same files
 * here, field names by Boost.PFR reflection as in the reference. */
template <typename T>
inline std::string_view mathematica_format() {
  if constexpr (std::is_same_v<T, double>) return "Real64";
  else if constexpr (std::is_same_v<T, long long int>) return "Integer64";
  else static_assert(sizeof(T) == 0, "Param fields must be double or long long int");
}

template <typename T>
inline void save_param_names(const std::string &filename) {
  std::ofstream out(filename);
  for (auto name : boost::pfr::names_as_array<T>()) out << name << '\n';
}

template <typename T>
inline void save_param_Mathematica_formats(const std::string &filename) {
  std::ofstream out(filename);
  boost::pfr::for_each_field(T(), [&](const auto &field) {
    out << mathematica_format<std::remove_cvref_t<decltype(field)>>() << '\n';
  });
}

template <typename T>
inline void save_param(const T &param, const std::string &filename) {
  std::ofstream out(filename, std::ios::binary);
  if (out.is_open()) out.write(reinterpret_cast<const char *>(&param), sizeof(T));
}

template <typename T>
inline void save_param_for_Mathematica(const T &param, const std::string &dir) {
  save_param_names<T>(dir + "paramNames.txt");
  save_param_Mathematica_formats<T>(dir + "paramTypes.txt");
  save_param<T>(param, dir + "param.dat");
}

template <typename T>
inline void print_param(const T &param) {
  const auto names = boost::pfr::names_as_array<T>();
  std::printf("---- The parameters for the simulation ----\n");
  boost::pfr::for_each_field(param, [&](const auto &field, std::size_t i) {
    std::printf("%.*s: %.17g\n", (int)names[i].size(), names[i].data(), (double)field);
  });
}

inline std::vector<double> load_vector_from_file(const std::string &filename) {
  std::ifstream file(filename, std::ios::binary | std::ios::ate);
  std::vector<double> v;
  if (!file.is_open()) return v;
  const std::streamsize n = file.tellg();
  file.seekg(0);
  v.resize((size_t)n / sizeof(double));
  file.read(reinterpret_cast<char *>(v.data()), (std::streamsize)(v.size() * sizeof(double)));
  return v;
}

/* ---- observer (src/observer.hpp:64-126) ------------------------------------
 * Same trigger (t >= t_last + t_interval, t == t_end or t == t_start), same files.
 * Every output is formed on the device (spectra, the density's a = 0 slice and its
 * mean over a: cf_density_slices), copied into pinned host memory on the workspace's
 * stream and written once the copy has landed, without stopping the stream: a save's
 * files are written at the next save, at t == t_end, by flush(), or when the last copy
 * of the observer goes away (odeint copies observers; the copies share one queue). */
namespace detail {
struct ObserverIO {
  std::shared_ptr<Context> ctx;
  DeviceState d_out;  // field spectrum | density spectrum | slice | axis average
  size_t s2 = 0, nn = 0;
  struct File {
    std::string name;
    size_t offset, count;
  };
  struct Pending {
    cudaEvent_t ev;
    double *host;
    std::vector<File> files;
  };
  std::deque<Pending> pending;
  std::vector<double *> pool;

  void bind(const std::shared_ptr<Context> &c, long long N) {
    if (ctx == c) return;
    drain(true);
    ctx = c;
    s2 = (size_t)c->info().s2_bins;
    nn = (size_t)(N * N);
    d_out.resize(2 * s2 + 2 * nn);
    for (double *h : pool) cudaFreeHost(h);
    pool.clear();
  }
  double *take_host() {
    if (!pool.empty()) {
      double *h = pool.back();
      pool.pop_back();
      return h;
    }
    void *h = nullptr;
    check_cuda(cudaMallocHost(&h, d_out.size() * sizeof(double)));
    return static_cast<double *>(h);
  }
  void write(const Pending &p) {
    for (const File &f : p.files) {
      std::ofstream file(f.name, std::ios::binary);
      if (file.is_open()) file.write(reinterpret_cast<const char *>(p.host + f.offset), f.count * sizeof(double));
    }
  }
  // Writes the saves whose copies have landed, and every save beyond the newest
  // `keep` (all of them when `all`).
  void drain(bool all, size_t keep = 0) {
    while (!pending.empty()) {
      Pending &p = pending.front();
      if (!all && pending.size() <= keep && cudaEventQuery(p.ev) == cudaErrorNotReady) break;
      check_cuda(cudaEventSynchronize(p.ev));
      write(p);
      cudaEventDestroy(p.ev);
      pool.push_back(p.host);
      pending.pop_front();
    }
  }
  ~ObserverIO() {
    try {
      drain(true);
    } catch (...) {
    }
    for (double *h : pool) cudaFreeHost(h);
  }
};
}  // namespace detail

template <typename Equation, bool save_field_spectrum = true, bool save_density_spectrum = true,
          bool save_density = false>
struct ConstIntervalObserver {
  typedef typename Equation::Workspace Workspace;
  typedef typename Workspace::State State;
  Workspace &workspace;
  int idx;
  std::string dir;
  double t_start, t_end, t_interval, t_last;
  std::shared_ptr<detail::ObserverIO> io = std::make_shared<detail::ObserverIO>();

  template <typename Param>
  ConstIntervalObserver(const std::string &dir_, const Param &param, Equation &eqn)
      : workspace(eqn.workspace), idx(0), dir(dir_), t_start(param.t_start), t_end(param.t_end),
        t_interval(param.t_interval), t_last(param.t_start) {}

  /* Writes every pending save's files. */
  void flush() { io->drain(true); }

  void operator()(const State &, double t) {
    if (t >= t_last + t_interval || t == t_end || t == t_start) {
      const long long N = workspace.N;
      Context &ctx = *workspace.ctx;
      io->bind(workspace.ctx, N);
      cudaStream_t st = ctx.stream();
      double *d = io->d_out.f64();
      const size_t s2 = io->s2, nn = io->nn;
      char name[512];
      detail::ObserverIO::Pending p{};
      auto file = [&](const char *fmt, size_t off, size_t count) {
        std::snprintf(name, sizeof(name), (dir + fmt).c_str(), idx);
        p.files.push_back({name, off, count});
      };
      if constexpr (save_field_spectrum) {
        check(cf_mode_power_spectrum_s2(ctx.get(), workspace.state.data(), workspace.cosmology.a(t), d, st));
        file("varphi_plus_spectrum_%d.dat", 0, s2);
      }
      if constexpr (save_density_spectrum) {
        check(cf_density_spectrum_s2(ctx.get(), workspace.state.data(), t, d + s2, st));
        file("rho_spectrum_%d.dat", s2, s2);
      }
      if constexpr (save_density) {
        check(cf_density_slices(ctx.get(), workspace.state.data(), t, d + 2 * s2, d + 2 * s2 + nn, st));
        file("rho_slice_%d.dat", 2 * s2, nn);
        file("rho_axis_average_%d.dat", 2 * s2 + nn, nn);
      }
      p.host = io->take_host();
      check_cuda(cudaMemcpyAsync(p.host, d, io->d_out.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
      check_cuda(cudaEventCreateWithFlags(&p.ev, cudaEventDisableTiming));
      check_cuda(cudaEventRecord(p.ev, st));
      io->pending.push_back(std::move(p));
      io->drain(t == t_end, 2);  // landed saves; at most two in flight
      workspace.t_list.push_back(t);
      t_last = t;
      ++idx;
    }
  }
};

}  // namespace cfb200

/* ---- odeint traits for DeviceState ---------------------------------------- */
namespace boost {
namespace numeric {
namespace odeint {

template <>
struct is_resizeable<cfb200::DeviceState> {
  typedef boost::true_type type;
  static const bool value = type::value;
};

template <>
struct same_size_impl<cfb200::DeviceState, cfb200::DeviceState> {
  static bool same_size(const cfb200::DeviceState &x, const cfb200::DeviceState &y) { return x.size() == y.size(); }
};

template <>
struct resize_impl<cfb200::DeviceState, cfb200::DeviceState> {
  static void resize(cfb200::DeviceState &x, const cfb200::DeviceState &y) {
    x.resize(y.size());
    x.ctx = y.ctx;
    x.precision = CF_FP64;  // odeint temporaries are FP64 device vectors
  }
};

template <>
struct algebra_dispatcher<cfb200::DeviceState> {
  typedef vector_space_algebra algebra_type;
};

template <>
struct operations_dispatcher<cfb200::DeviceState> {
  typedef cfb200::device_operations operations_type;
};

}  // namespace odeint
}  // namespace numeric
}  // namespace boost

#endif /* CFB200_ODEINT_HPP */
