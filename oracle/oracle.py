"""ctypes access to the parity checkers (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline / reference
legs of ``bench.py`` import this module.  It loads

* ``oracle/liboracle.so`` -- the C restatement of the reference's hot path
  (``cf_oracle.c``; each function cites the reference file:line it follows), and
* ``oracle/_ref/libcfref.so`` -- the reference's own CPU sources compiled where
  they lie (``ref_harness.cpp``), present when the reference tree was available
  at build time.

Equation codes: 0 = KleinGordonEquation (flat), 1 = KleinGordonEquationInFRW,
2 = ComovingCurvatureEquationInFRW, 3 = CudaLambdaEquationInFRW,
4 = CudaSqrtPotentialEquationInFRW, 5 = CudaFixedCurvatureEquationInFRW,
6 = CudaApproximateComovingCurvatureEquationInFRW.
"""
from __future__ import annotations

import ctypes
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_vp = ctypes.c_void_p
_d = ctypes.c_double
_i64 = ctypes.c_int64
_i = ctypes.c_int


class Params(ctypes.Structure):
    """Mirror of ``cfo_params`` in cf_oracle.c."""

    _fields_ = [("N", _i64), ("L", _d), ("m", _d), ("a1", _d), ("H1", _d), ("t1", _d),
                ("p", _d), ("eq", _i), ("stencil", _i), ("lam", _d), ("f_a", _d), ("M", _i64),
                ("Psi_fixed", _vp)]


def make_params(N, L, m=1.0, eq=1, a1=1.0, H1=0.0, t1=0.0, p=1.0, stencil=7, lam=0.0, f_a=1.0, M=0,
                psi_fixed=None):
    """Oracle parameters; ``psi_fixed`` (N^3 FP64, eq 5) is kept alive by the result."""
    P = Params(int(N), float(L), float(m), float(a1), float(H1), float(t1), float(p),
               int(eq), int(stencil), float(lam), float(f_a), int(M), None)
    if psi_fixed is not None:
        P._psi = np.ascontiguousarray(psi_fixed, dtype=np.float64)
        P.Psi_fixed = P._psi.ctypes.data
    return P


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


_lib = None
_ref = {}


def lib():
    """The restated oracle (liboracle.so); built by ``make -C oracle``."""
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so is missing: run `make -C oracle`")
        L = ctypes.CDLL(path)
        P = ctypes.POINTER(Params)
        L.cfo_a.restype = _d
        L.cfo_a.argtypes = [P, _d]
        L.cfo_H.restype = _d
        L.cfo_H.argtypes = [P, _d]
        L.cfo_eta.restype = _d
        L.cfo_eta.argtypes = [P, _d]
        L.cfo_rhs.argtypes = [P, _vp, _vp, _d, _vp]
        L.cfo_rk4_step.argtypes = [P, _vp, _vp, _d, _d]
        L.cfo_rk4_steps.argtypes = [P, _vp, _vp, _d, _d, _i64, _i64]
        L.cfo_energy_density.argtypes = [P, _vp, _vp, _d, _vp]
        L.cfo_dot_energy_density.argtypes = [P, _vp, _d, _vp]
        L.cfo_approx_fields.argtypes = [P, _vp, _d, _vp, _vp]
        L.cfo_d2z.argtypes = [_i64, _vp, _vp]
        L.cfo_power_spectrum.argtypes = [_i64, _vp, _vp]
        L.cfo_mode_power_spectrum.argtypes = [_i64, _d, _d, _d, _vp, _vp]
        L.cfo_s2_counts.argtypes = [_i64, _vp]
        L.cfo_shells_from_s2.argtypes = [_i64, _vp, _vp, _vp, _vp]
        L.cfo_isqrt.restype = _i64
        L.cfo_isqrt.argtypes = [_i64]
        L.cfo_psi_fields.argtypes = [P, _vp, _d, _vp, _vp]
        L.cfo_psi_dpsidt_fft.argtypes = [_i64, _vp, _vp, _vp, _d, _d]
        L.cfo_driver_initial.argtypes = [_i64, _d, ctypes.c_uint32, _vp, _vp]
        L.cfo_driver_tables.argtypes = [_i64, _d, _vp, _vp, _vp, _vp, _vp]
        L.cfo_rng_size.restype = ctypes.c_size_t
        L.cfo_rng_seed.argtypes = [_vp, ctypes.c_uint32]
        L.cfo_rng_fill.argtypes = [_vp, _vp, _i64]
        L.cfo_grf_white.argtypes = [_i64, _d, _vp, _vp, _d, _i, _vp, _vp]
        L.cfo_sqrtP_table.argtypes = [_i64, _d, _i, _vp, _vp]
        L.cfo_philox4x32_10.argtypes = [_vp, _vp, _vp]
        L.cfo_white_noise.argtypes = [ctypes.c_uint64, ctypes.c_uint64, _i64, _vp]
        L.cfo_wkb.argtypes = [P, _vp, _d, _d, _vp]
        L.cfo_wkb_phase.restype = _d
        L.cfo_wkb_phase.argtypes = [_d, _d, _d, _d, _d, _d]
        L.cfo_ci.restype = _d
        L.cfo_ci.argtypes = [_d]
        _lib = L
    return _lib


def ref_available(strict=False):
    name = "libcfref_strict.so" if strict else "libcfref.so"
    return os.path.exists(os.path.join(HERE, "_ref", name))


def ref(strict=False):
    """The reference's own CPU code (oracle/_ref/libcfref[_strict].so)."""
    key = bool(strict)
    if key not in _ref:
        name = "libcfref_strict.so" if strict else "libcfref.so"
        path = os.path.join(HERE, "_ref", name)
        if not os.path.exists(path):
            raise RuntimeError(f"oracle/_ref/{name} is missing: run `make -C oracle ref`")
        R = ctypes.CDLL(path)
        R.cfr_integrate.restype = _i
        R.cfr_integrate.argtypes = [_i, ctypes.c_longlong, _d, _d, _d, _d, _d, _vp, _vp, _d, _d, _d,
                                    _d, ctypes.c_char_p, _vp, _i]
        R.cfr_rhs.argtypes = [_i, ctypes.c_longlong, _d, _d, _d, _d, _d, _vp, _vp, _d, _vp]
        R.cfr_energy_density.argtypes = [_i, ctypes.c_longlong, _d, _d, _d, _d, _d, _vp, _vp, _d, _vp]
        R.cfr_power_spectrum.argtypes = [ctypes.c_longlong, _vp, _vp]
        R.cfr_mode_power_spectrum.argtypes = [ctypes.c_longlong, _d, _d, _d, _vp, _vp]
        R.cfr_d2z.argtypes = [ctypes.c_longlong, _vp, _vp]
        R.cfr_driver_initial.argtypes = [ctypes.c_longlong, _d, ctypes.c_uint, ctypes.c_char_p, _vp, _vp]
        _ref[key] = R
    return _ref[key]


# ---------------------------------------------------------------- sizes


def n_s2(N):
    return 3 * (N // 2) ** 2 + 1


def n_hc(N):
    return 2 * N * N * (N // 2 + 1)


def n_shells(N):
    return int(lib().cfo_isqrt(n_s2(N) - 1)) + 1


# ---------------------------------------------------------------- restated oracle


def rhs(P, x, t, R_fft=None):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    lib().cfo_rhs(ctypes.byref(P), _ptr(x), _ptr(R_fft) if R_fft is not None else None, t, _ptr(out))
    return out


def rk4_steps(P, x, t0, dt, nsteps, step0=0, R_fft=None):
    """x advanced by nsteps of integrate_const's loop (t_j = t0 + (step0+j) dt)."""
    y = np.array(x, dtype=np.float64, copy=True)
    lib().cfo_rk4_steps(ctypes.byref(P), _ptr(y), _ptr(R_fft) if R_fft is not None else None,
                        t0, dt, step0, nsteps)
    return y


def energy_density(P, x, t, R_fft=None):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty(P.N ** 3)
    lib().cfo_energy_density(ctypes.byref(P), _ptr(x), _ptr(R_fft) if R_fft is not None else None,
                             t, _ptr(out))
    return out


def dot_energy_density(P, x, t):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty(P.N ** 3)
    lib().cfo_dot_energy_density(ctypes.byref(P), _ptr(x), t, _ptr(out))
    return out


def approx_fields(P, R_fft, t):
    """Coarse (M^3) Psi and dPsi/dt of the approximate comoving equation at t."""
    M3 = P.M ** 3
    psi = np.empty(M3)
    dpsi = np.empty(M3)
    lib().cfo_approx_fields(ctypes.byref(P), _ptr(R_fft), t, _ptr(psi), _ptr(dpsi))
    return psi, dpsi


def d2z(f):
    f = np.ascontiguousarray(f, dtype=np.float64)
    N = round(f.size ** (1 / 3))
    out = np.empty(n_hc(N))
    lib().cfo_d2z(N, _ptr(f), _ptr(out))
    return out


def power_spectrum(f):
    f = np.ascontiguousarray(f, dtype=np.float64)
    N = round(f.size ** (1 / 3))
    out = np.empty(n_s2(N))
    lib().cfo_power_spectrum(N, _ptr(f), _ptr(out))
    return out


def mode_power_spectrum(N, L, m, a_t, state):
    state = np.ascontiguousarray(state, dtype=np.float64)
    out = np.empty(n_s2(N))
    lib().cfo_mode_power_spectrum(N, L, m, a_t, _ptr(state), _ptr(out))
    return out


def s2_counts(N):
    out = np.empty(n_s2(N), dtype=np.int64)
    lib().cfo_s2_counts(N, _ptr(out))
    return out


def shells_from_s2(N, s2bins=None):
    counts = s2_counts(N)
    ns = n_shells(N)
    shells = np.empty(ns)
    sc = np.empty(ns, dtype=np.int64)
    lib().cfo_shells_from_s2(N, _ptr(np.ascontiguousarray(s2bins)) if s2bins is not None else None,
                             _ptr(counts), _ptr(shells), _ptr(sc))
    return (shells if s2bins is not None else None), sc


def psi_fields(P, R_fft, t):
    N3 = P.N ** 3
    psi = np.empty(N3)
    dpsi = np.empty(N3)
    lib().cfo_psi_fields(ctypes.byref(P), _ptr(R_fft), t, _ptr(psi), _ptr(dpsi))
    return psi, dpsi


def a_of_t(P, t):
    return lib().cfo_a(ctypes.byref(P), t)


def H_of_t(P, t):
    return lib().cfo_H(ctypes.byref(P), t)


def eta_of_t(P, t):
    return lib().cfo_eta(ctypes.byref(P), t)


def driver_initial(N, L, seed=0):
    """State and R_fft of the reference driver's set-up, rebuilt by the restatement."""
    state = np.empty(2 * N ** 3)
    R_fft = np.empty(n_hc(N))
    lib().cfo_driver_initial(N, L, seed, _ptr(state), _ptr(R_fft))
    return state, R_fft


def normals(seed, n):
    """The first n deviates of the reference's RandomNormal stream after
    set_generator_seed(seed) (std::mt19937 + libstdc++ normal_distribution, restated)."""
    r = ctypes.create_string_buffer(int(lib().cfo_rng_size()))
    lib().cfo_rng_seed(r, seed)
    out = np.empty(int(n))
    lib().cfo_rng_fill(r, _ptr(out), int(n))
    return out


def philox4x32_10(ctr, key):
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.empty(4, dtype=np.uint32)
    lib().cfo_philox4x32_10(_ptr(c), _ptr(k), _ptr(out))
    return out


def white_noise(seed, offset, n):
    """The deviates cf_white_noise makes (restated)."""
    out = np.empty(int(n))
    lib().cfo_white_noise(int(seed), int(offset), int(n), _ptr(out))
    return out


def wkb(P, x, t_i, t_f):
    """WKBSolutionForKleinGordonEquationInFRW(workspace with state x, t_i).evaluate_at(t_f)."""
    out = np.empty(2 * P.N ** 3)
    lib().cfo_wkb(ctypes.byref(P), _ptr(np.ascontiguousarray(x, dtype=np.float64)), t_i, t_f, _ptr(out))
    return out


def grf_white(N, L, white, kind, args, Psi=None, psi_scale=0.0):
    """generate_inhomogeneous_gaussian_random_field from given deviates; kind 0: power
    law with cutoff {P_k_ast, k_ast, alpha}, 1: its derivative spectrum {.., m}, 2: scale
    invariant {P_k0}."""
    out = np.empty(N ** 3)
    a = np.ascontiguousarray(args, dtype=np.float64)
    lib().cfo_grf_white(N, L, _ptr(np.ascontiguousarray(white)), _ptr(Psi) if Psi is not None else None,
                        psi_scale, kind, _ptr(a), _ptr(out))
    return out


def sqrtP_table(N, L, kind, args):
    out = np.empty(n_s2(N))
    a = np.ascontiguousarray(args, dtype=np.float64)
    lib().cfo_sqrtP_table(N, L, kind, _ptr(a), _ptr(out))
    return out


def driver_tables(N, L):
    """(sqrtP_R, Psi kernel / N^3, sqrtP_f, sqrtP_dtf, (alpha_phi, alpha_dphi)) of the
    reference driver's initializer."""
    t = [np.empty(n_s2(N)) for _ in range(4)]
    al = np.empty(2)
    lib().cfo_driver_tables(N, L, *[_ptr(x) for x in t], _ptr(al))
    return t[0], t[1], t[2], t[3], al


# ---------------------------------------------------------------- the reference itself


def ref_integrate(eq, N, L, m, state, t_start, t_end, dt, a1=1.0, H1=0.0, t1=0.0, R_fft=None,
                  t_interval=None, observe=False, strict=False):
    """integrate_const over the reference's own equation and RK4.  Returns
    (final_state, spectra) where spectra is None or a dict with the observer's
    saved ``t_list``, ``varphi_plus`` and ``rho`` spectra (files it wrote)."""
    R = ref(strict)
    st = np.array(state, dtype=np.float64, copy=True)
    if not observe:
        R.cfr_integrate(eq, N, L, m, a1, H1, t1, _ptr(st), _ptr(R_fft) if R_fft is not None else None,
                        t_start, t_end, dt, t_interval or 1.0, b"", None, 0)
        return st, None
    with tempfile.TemporaryDirectory() as d:
        tl = np.zeros(100000)
        n = R.cfr_integrate(eq, N, L, m, a1, H1, t1, _ptr(st), _ptr(R_fft) if R_fft is not None else None,
                            t_start, t_end, dt, t_interval, (d + "/").encode(), _ptr(tl), tl.size)
        out = {"t_list": tl[:n].copy(), "varphi_plus": [], "rho": []}
        for i in range(n):
            out["varphi_plus"].append(np.fromfile(f"{d}/varphi_plus_spectrum_{i}.dat"))
            out["rho"].append(np.fromfile(f"{d}/rho_spectrum_{i}.dat"))
    return st, out


def ref_rhs(eq, N, L, m, x, t, a1=1.0, H1=0.0, t1=0.0, R_fft=None, strict=False):
    out = np.empty(2 * N ** 3)
    ref(strict).cfr_rhs(eq, N, L, m, a1, H1, t1, _ptr(np.ascontiguousarray(x)),
                        _ptr(R_fft) if R_fft is not None else None, t, _ptr(out))
    return out


def ref_energy_density(eq, N, L, m, x, t, a1=1.0, H1=0.0, t1=0.0, R_fft=None, strict=False):
    out = np.empty(N ** 3)
    ref(strict).cfr_energy_density(eq, N, L, m, a1, H1, t1, _ptr(np.ascontiguousarray(x)),
                                   _ptr(R_fft) if R_fft is not None else None, t, _ptr(out))
    return out


def ref_wkb(N, L, m, x, t_i, t_f, a1=1.0, H1=0.5, strict=False):
    """The reference's own WKB continuation (src/wkb.cpp) of state x from t_i to t_f."""
    R = ref(strict)
    R.cfr_wkb.argtypes = [ctypes.c_longlong, _d, _d, _d, _d, _d, _vp, _d, _d, _vp]
    out = np.empty(2 * N ** 3)
    R.cfr_wkb(N, L, m, a1, H1, 1.0 / (2 * H1), _ptr(np.ascontiguousarray(x)), t_i, t_f, _ptr(out))
    return out


def ref_power_spectrum(f, strict=False):
    f = np.ascontiguousarray(f, dtype=np.float64)
    N = round(f.size ** (1 / 3))
    out = np.empty(n_s2(N))
    ref(strict).cfr_power_spectrum(N, _ptr(f), _ptr(out))
    return out


def ref_mode_power_spectrum(N, L, m, a_t, state, strict=False):
    out = np.empty(n_s2(N))
    ref(strict).cfr_mode_power_spectrum(N, L, m, a_t, _ptr(np.ascontiguousarray(state)), _ptr(out))
    return out


def ref_d2z(f, strict=False):
    f = np.ascontiguousarray(f, dtype=np.float64)
    N = round(f.size ** (1 / 3))
    out = np.empty(n_hc(N))
    ref(strict).cfr_d2z(N, _ptr(f), _ptr(out))
    return out


def ref_driver_initial(N, L, seed, outdir, want_state=False):
    """Runs the reference driver's set-up + first observer call, writing its .dat
    files into outdir; optionally returns (state, R_fft)."""
    st = np.empty(2 * N ** 3) if want_state else None
    rf = np.empty(n_hc(N)) if want_state else None
    ref().cfr_driver_initial(N, L, seed, (outdir.rstrip("/") + "/").encode(),
                             _ptr(st) if st is not None else None, _ptr(rf) if rf is not None else None)
    return (st, rf) if want_state else None
