"""ctypes binding of libcfb200.so (the C ABI in include/cfb200.h).

This is the harness the parity tests and bench.py use to drive the product
through its C ABI; C++ callers use include/cfb200.h (and the odeint adapter
include/cfb200_odeint.hpp) directly.  Device buffers are plain CUDA pointers;
the helpers accept torch CUDA tensors for convenience (torch only provides the
memory and the stream).

There is no CPU fallback: if the library is missing or no GPU is usable, the
calls raise.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "libcfb200.so")
HEADER = os.path.join(ROOT, "include", "cfb200.h")

CF_OK = 0
STATUS = {0: "CF_OK", -1: "CF_ERR_INVALID", -2: "CF_ERR_CUDA", -3: "CF_ERR_CUFFT", -4: "CF_ERR_NOMEM",
          -5: "CF_ERR_NONFINITE", -6: "CF_ERR_TIMEOUT", -7: "CF_ERR_UNSUPPORTED"}
EQ_KG, EQ_KG_FRW, EQ_COMOVING_FRW = 0, 1, 2
EQ_LAMBDA_FRW, EQ_SQRT_FRW, EQ_FIXED_CURVATURE_FRW, EQ_APPROX_COMOVING_FRW = 3, 4, 5, 6
FP64, FP32_COMP = 0, 1
FLAG_FULL_PSI_FFT = 1
FLAG_STAGE_KERNELS = 2
FLAG_PAIR_KERNELS = 4
FLAG_PSI_CTA_PASS_C = 8
FLAG_PSI_SERIAL = 16
FLAG_PSI_NO_TMA = 32
FLAG_PSI_NO_REUSE = 64
PSI_NONE, PSI_FULL, PSI_PRUNED, PSI_PRUNED_FUSED = 0, 1, 2, 3


class CfError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class cf_params(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int64), ("L", ctypes.c_double), ("m", ctypes.c_double),
                ("a1", ctypes.c_double), ("H1", ctypes.c_double), ("t1", ctypes.c_double),
                ("p", ctypes.c_double), ("equation", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("stencil", ctypes.c_int32), ("flags", ctypes.c_int32), ("lam", ctypes.c_double),
                ("f_a", ctypes.c_double), ("M", ctypes.c_int64)]


class cf_info(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int64), ("state_bytes", ctypes.c_int64), ("field_count", ctypes.c_int64),
                ("hc_count", ctypes.c_int64), ("s2_bins", ctypes.c_int64), ("shells", ctypes.c_int64),
                ("psi_route", ctypes.c_int64)]


_vp = ctypes.c_void_p
_d = ctypes.c_double
_i64 = ctypes.c_int64
_i = ctypes.c_int

_SIGS = {
    "cf_create": ([ctypes.POINTER(cf_params), ctypes.POINTER(_vp)], _i),
    "cf_destroy": ([_vp], _i),
    "cf_get_info": ([_vp, ctypes.POINTER(cf_info)], _i),
    "cf_last_error": ([], ctypes.c_char_p),
    "cf_launch_count": ([_vp], _i64),
    "cf_state_upload": ([_vp, _vp, _vp, _vp], _i),
    "cf_state_download": ([_vp, _vp, _vp, _vp], _i),
    "cf_state_import": ([_vp, _vp, _vp, _vp], _i),
    "cf_state_export": ([_vp, _vp, _vp, _vp], _i),
    "cf_set_R_fft": ([_vp, _vp, _i, _vp], _i),
    "cf_set_psi": ([_vp, _vp, _i, _vp], _i),
    "cf_psi_fields": ([_vp, _d, _vp, _vp], _i),
    "cf_psi_set_wait_test": ([_vp, _i, _i64], _i),
    "cf_psi_stats": ([_vp, _vp, _vp], _i),
    "cf_rk4_steps": ([_vp, _vp, _d, _d, _i64, _i64, _vp], _i),
    "cf_rhs": ([_vp, _vp, _vp, _d, _vp], _i),
    "cf_scale_sum": ([_vp, _vp, _i, _vp, _vp, _i64, _vp], _i),
    "cf_energy_density": ([_vp, _vp, _d, _vp, _vp], _i),
    "cf_dot_energy_density": ([_vp, _vp, _d, _vp, _vp], _i),
    "cf_white_noise": ([_vp, ctypes.c_uint64, ctypes.c_uint64, _vp, _i64, _vp], _i),
    "cf_grf": ([_vp, _vp, _vp, _d, _vp, _vp, _vp], _i),
    "cf_scale_modes": ([_vp, _vp, _vp, _vp, _vp], _i),
    "cf_power_spectrum_s2": ([_vp, _vp, _vp, _vp], _i),
    "cf_mode_power_spectrum_s2": ([_vp, _vp, _d, _vp, _vp], _i),
    "cf_density_spectrum_s2": ([_vp, _vp, _d, _vp, _vp], _i),
    "cf_s2_to_shells": ([_vp, _vp, _vp, _vp], _i),
    "cf_density_slices": ([_vp, _vp, _d, _vp, _vp, _vp], _i),
    "cf_wkb_create": ([_vp, _vp, _d, ctypes.POINTER(_vp), _vp], _i),
    "cf_wkb_evaluate": ([_vp, _d, _vp, _vp], _i),
    "cf_wkb_destroy": ([_vp], _i),
    "cf_s2_counts": ([_vp, _vp, _vp], _i),
    "cf_check_finite": ([_vp, _vp, ctypes.POINTER(_i64), _vp], _i),
    "cf_fft_create": ([_i64, _vp], _i),
    "cf_fft_destroy": ([_vp], _i),
    "cf_fft_d2z": ([_vp, _vp, _vp, _vp], _i),
    "cf_fft_batched_d2z": ([_vp, _vp, _vp, _vp], _i),
    "cf_fft_z2d": ([_vp, _vp, _vp, _vp], _i),
    "cf_fft_inplace_z2d": ([_vp, _vp, _vp], _i),
    "cf_adjoint_create": ([_vp, _i64, _i64, ctypes.POINTER(_vp)], _i),
    "cf_adjoint_destroy": ([_vp], _i),
    "cf_adjoint_forward": ([_vp, _vp, _d, _d, _vp], _i),
    "cf_adjoint_shell_log_loss": ([_vp, _vp, _vp, _d, ctypes.POINTER(_d), _vp], _i),
    "cf_adjoint_set_lambda": ([_vp, _vp, _d, _vp], _i),
    "cf_adjoint_backward": ([_vp, _vp, ctypes.POINTER(_d), _vp], _i),
    "cf_field_from_shell_amplitudes": ([_vp, _vp, _vp, _vp, _i, _i, _vp, _vp], _i),
    "cf_shell_amplitude_gradient": ([_vp, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp], _i),
    "cf_ensemble_create": ([_vp, _i, ctypes.POINTER(_vp)], _i),
    "cf_ensemble_destroy": ([_vp], _i),
    "cf_ensemble_info": ([_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64)], _i),
    "cf_ensemble_launch_count": ([_vp], _i64),
    "cf_ensemble_state_upload": ([_vp, _i, _vp, _vp], _i),
    "cf_ensemble_state_download": ([_vp, _i, _vp, _vp], _i),
    "cf_ensemble_rk4_steps": ([_vp, _d, _d, _i64, _i64, _i, _vp], _i),
    "cf_ensemble_density_spectra_s2": ([_vp, _d, _vp, _vp], _i),
    "cf_ensemble_run_graph": ([_vp, _d, _d, _i64, _i64, _i, _vp, _vp], _i),
    "cf_ensemble_autotune": ([_vp, _d, _d, _i64, _vp, ctypes.POINTER(_i), ctypes.POINTER(_i)], _i),
    "cf_ensemble_set_barrier_test": ([_vp, _i, _i64], _i),
    "cf_profile_enable": ([_vp, _i], _i),
    "cf_profile_read": ([_vp, _vp], _i),
    "cf_profile_reset": ([_vp], _i),
}

PROF_KINDS = ["stage1", "stage2", "stage3", "stage4", "psi_transfer", "psi_fft", "spectrum", "other", "pair_a",
              "pair_b", "step"]
STEP_KINDS = ("stage1", "stage2", "stage3", "stage4", "pair_a", "pair_b", "step")


class cf_profile(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_int64 * len(PROF_KINDS)), ("ms", ctypes.c_double * len(PROF_KINDS))]

_lib = None


def header_symbols():
    """Every function name declared in include/cfb200.h."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|const char \*)\s*(cf_\w+)\s*\(", txt, re.M)))


def lib():
    """Loads libcfb200.so (built by `make -C cosmic-fields-lite_b200`)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C cosmic-fields-lite_b200`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def check(code):
    if code != CF_OK:
        msg = lib().cf_last_error()
        raise CfError(code, msg.decode() if msg else "")
    return code


def _ptr(x):
    """Device/host pointer of a torch tensor, numpy array or int."""
    if x is None:
        return None
    if isinstance(x, int):
        return ctypes.c_void_p(x)
    if hasattr(x, "data_ptr"):
        return ctypes.c_void_p(x.data_ptr())
    if hasattr(x, "ctypes"):
        return ctypes.c_void_p(x.ctypes.data)
    raise TypeError(type(x))


def _stream(stream):
    if stream is None:
        try:
            import torch
            return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        except Exception:
            return None
    if isinstance(stream, int):
        return ctypes.c_void_p(stream)
    return ctypes.c_void_p(stream.cuda_stream)


class Context:
    """One cf_ctx: a lattice, an equation, a precision and a stencil."""

    def __init__(self, N, L, m=1.0, equation=EQ_KG_FRW, precision=FP64, stencil=7, a1=1.0, H1=0.0,
                 t1=0.0, p=1.0, flags=0, lam=0.0, f_a=1.0, M=0):
        """lam, f_a, M: the workspace's lambda (EQ_LAMBDA_FRW), f_a (EQ_SQRT_FRW; the
        reference's default 1) and M (EQ_APPROX_COMOVING_FRW)."""
        self.params = cf_params(int(N), float(L), float(m), float(a1), float(H1), float(t1), float(p),
                                int(equation), int(precision), int(stencil), int(flags), float(lam),
                                float(f_a), int(M))
        h = ctypes.c_void_p()
        check(lib().cf_create(ctypes.byref(self.params), ctypes.byref(h)))
        self.h = h
        self.N = int(N)

    @property
    def info(self):
        """cf_get_info, read afresh (psi_route follows cf_set_R_fft)."""
        info = cf_info()
        check(lib().cf_get_info(self.h, ctypes.byref(info)))
        return info

    def close(self):
        if getattr(self, "h", None):
            lib().cf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def launches(self):
        return int(lib().cf_launch_count(self.h))

    # ---- state
    def upload(self, d_state, h_xy, stream=None):
        check(lib().cf_state_upload(self.h, _ptr(d_state), _ptr(h_xy), _stream(stream)))

    def download(self, h_xy, d_state, stream=None):
        check(lib().cf_state_download(self.h, _ptr(h_xy), _ptr(d_state), _stream(stream)))

    def import_f64(self, d_state, d_xy, stream=None):
        check(lib().cf_state_import(self.h, _ptr(d_state), _ptr(d_xy), _stream(stream)))

    def export_f64(self, d_xy, d_state, stream=None):
        check(lib().cf_state_export(self.h, _ptr(d_xy), _ptr(d_state), _stream(stream)))

    def set_R_fft(self, R_fft, on_device, stream=None):
        check(lib().cf_set_R_fft(self.h, _ptr(R_fft), int(on_device), _stream(stream)))

    def set_psi(self, Psi, on_device, stream=None):
        """The fixed Psi(x) of EQ_FIXED_CURVATURE_FRW (N^3 doubles, host or device)."""
        check(lib().cf_set_psi(self.h, _ptr(Psi), int(on_device), _stream(stream)))

    def psi_fields(self, t, d_out, stream=None):
        """Psi and dPsi/dt at time t into d_out (2 N^3 doubles on the device)."""
        check(lib().cf_psi_fields(self.h, float(t), _ptr(d_out), _stream(stream)))

    def psi_stats(self):
        """(slots synthesised, stage times that reused a refresh with identical pass-A inputs)."""
        r, u = ctypes.c_int64(0), ctypes.c_int64(0)
        check(lib().cf_psi_stats(self.h, ctypes.byref(r), ctypes.byref(u)))
        return r.value, u.value

    def psi_set_wait_test(self, extra_bytes, spin_limit=1 << 20):
        """Test hook: pass C's band-copy waits give up (cf_psi_set_wait_test)."""
        check(lib().cf_psi_set_wait_test(self.h, int(extra_bytes), int(spin_limit)))

    # ---- hot path
    def rk4_steps(self, d_state, t0, dt, nsteps, step0=0, stream=None):
        check(lib().cf_rk4_steps(self.h, _ptr(d_state), float(t0), float(dt), int(step0), int(nsteps),
                                 _stream(stream)))

    def rhs(self, d_x, d_dxdt, t, stream=None):
        check(lib().cf_rhs(self.h, _ptr(d_x), _ptr(d_dxdt), float(t), _stream(stream)))

    def scale_sum(self, d_out, d_ins, alphas, length, stream=None):
        n = len(d_ins)
        arr = (ctypes.c_void_p * n)(*[_ptr(x).value for x in d_ins])
        al = (ctypes.c_double * n)(*[float(a) for a in alphas])
        check(lib().cf_scale_sum(self.h, _ptr(d_out), n, ctypes.cast(arr, ctypes.c_void_p),
                                 ctypes.cast(al, ctypes.c_void_p), int(length), _stream(stream)))

    # ---- observers
    def energy_density(self, d_state, t, d_rho, stream=None):
        check(lib().cf_energy_density(self.h, _ptr(d_state), float(t), _ptr(d_rho), _stream(stream)))

    def dot_energy_density(self, d_state, t, d_out, stream=None):
        check(lib().cf_dot_energy_density(self.h, _ptr(d_state), float(t), _ptr(d_out), _stream(stream)))

    def power_spectrum_s2(self, d_f, d_out, stream=None):
        check(lib().cf_power_spectrum_s2(self.h, _ptr(d_f), _ptr(d_out), _stream(stream)))

    def mode_power_spectrum_s2(self, d_state, a_t, d_out, stream=None):
        check(lib().cf_mode_power_spectrum_s2(self.h, _ptr(d_state), float(a_t), _ptr(d_out), _stream(stream)))

    def density_spectrum_s2(self, d_state, t, d_out, stream=None):
        check(lib().cf_density_spectrum_s2(self.h, _ptr(d_state), float(t), _ptr(d_out), _stream(stream)))

    def density_slices(self, d_state, t, d_slice=None, d_axis_average=None, stream=None):
        check(lib().cf_density_slices(self.h, _ptr(d_state), float(t), _ptr(d_slice), _ptr(d_axis_average),
                                      _stream(stream)))

    def s2_to_shells(self, d_shells, d_counts=None, stream=None):
        check(lib().cf_s2_to_shells(self.h, _ptr(d_shells), _ptr(d_counts), _stream(stream)))

    def s2_counts(self, d_counts, stream=None):
        check(lib().cf_s2_counts(self.h, _ptr(d_counts), _stream(stream)))

    # ---- initial conditions
    def white_noise(self, d_out, seed, offset=0, n=None, stream=None):
        """n unit-normal deviates (Philox4x32-10 + Box-Muller) of stream `seed` from `offset`."""
        n = d_out.numel() if n is None else int(n)
        check(lib().cf_white_noise(self.h, int(seed), int(offset), _ptr(d_out), n, _stream(stream)))

    def grf(self, d_white, sqrtP_s2, d_out, d_psi=None, psi_scale=0.0, stream=None):
        """generate_inhomogeneous_gaussian_random_field from the deviates d_white (N^3)."""
        import numpy as np
        tab = np.ascontiguousarray(sqrtP_s2, dtype=np.float64)
        check(lib().cf_grf(self.h, _ptr(d_white), _ptr(d_psi), float(psi_scale), _ptr(tab), _ptr(d_out),
                           _stream(stream)))

    def scale_modes(self, d_f, scale_s2, d_out, stream=None):
        """compute_field_with_scaled_fourier_modes with the per-s^2 factor scale_s2."""
        import numpy as np
        tab = np.ascontiguousarray(scale_s2, dtype=np.float64)
        check(lib().cf_scale_modes(self.h, _ptr(d_f), _ptr(tab), _ptr(d_out), _stream(stream)))

    # ---- profiling
    def profile(self, on=True):
        check(lib().cf_profile_enable(self.h, int(on)))

    def profile_reset(self):
        check(lib().cf_profile_reset(self.h))

    def profile_read(self):
        p = cf_profile()
        check(lib().cf_profile_read(self.h, ctypes.byref(p)))
        return {k: (int(p.launches[i]), float(p.ms[i])) for i, k in enumerate(PROF_KINDS)}

    def check_finite(self, d_state, stream=None):
        bad = _i64(0)
        code = lib().cf_check_finite(self.h, _ptr(d_state), ctypes.byref(bad), _stream(stream))
        return code, int(bad.value)


class Adjoint:
    """cf_adjoint: checkpointed forward run, shell-spectrum log loss, reverse sweep."""

    def __init__(self, ctx, nsteps, checkpoint_every):
        self.ctx = ctx
        h = ctypes.c_void_p()
        check(lib().cf_adjoint_create(ctx.h, int(nsteps), int(checkpoint_every), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().cf_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, d_state, t0, dt, stream=None):
        check(lib().cf_adjoint_forward(self.h, _ptr(d_state), float(t0), float(dt), _stream(stream)))

    def shell_log_loss(self, d_state, target_shells, rel_floor=0.0, stream=None):
        import numpy as np
        tgt = np.ascontiguousarray(target_shells, dtype=np.float64)
        loss = _d(0.0)
        check(lib().cf_adjoint_shell_log_loss(self.h, _ptr(d_state), _ptr(tgt), float(rel_floor), ctypes.byref(loss),
                                              _stream(stream)))
        return float(loss.value)

    def set_lambda(self, d_lambda, dm_direct=0.0, stream=None):
        check(lib().cf_adjoint_set_lambda(self.h, _ptr(d_lambda), float(dm_direct), _stream(stream)))

    def backward(self, d_lambda0=None, stream=None):
        dm = _d(0.0)
        check(lib().cf_adjoint_backward(self.h, _ptr(d_lambda0), ctypes.byref(dm), _stream(stream)))
        return float(dm.value)


class FFT:
    """cf_fft: the reference's fft_wrapper (3-D FP64 D2Z / Z2D of an N^3 lattice)."""

    def __init__(self, N):
        h = ctypes.c_void_p()
        check(lib().cf_fft_create(int(N), ctypes.byref(h)))
        self.h = h
        self.N = int(N)

    def close(self):
        if getattr(self, "h", None):
            lib().cf_fft_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def d2z(self, d_in, d_out, stream=None):
        check(lib().cf_fft_d2z(self.h, _ptr(d_in), _ptr(d_out), _stream(stream)))

    def batched_d2z(self, d_in, d_out, stream=None):
        check(lib().cf_fft_batched_d2z(self.h, _ptr(d_in), _ptr(d_out), _stream(stream)))

    def z2d(self, d_in, d_out, stream=None):
        check(lib().cf_fft_z2d(self.h, _ptr(d_in), _ptr(d_out), _stream(stream)))

    def inplace_z2d(self, d_inout, stream=None):
        check(lib().cf_fft_inplace_z2d(self.h, _ptr(d_inout), _stream(stream)))


class WKB:
    """cf_wkb: WKB continuation of a KG-FRW state (WKBSolutionForKleinGordonEquationInFRW)."""

    def __init__(self, ctx, d_state, t_i, stream=None):
        self.ctx = ctx
        h = ctypes.c_void_p()
        check(lib().cf_wkb_create(ctx.h, _ptr(d_state), float(t_i), ctypes.byref(h), _stream(stream)))
        self.h = h

    def evaluate_at(self, t, d_out, stream=None):
        check(lib().cf_wkb_evaluate(self.h, float(t), _ptr(d_out), _stream(stream)))

    def close(self):
        if getattr(self, "h", None):
            lib().cf_wkb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


ENS_PERSISTENT, ENS_BATCHED, ENS_LOOP = 0, 1, 2


class Ensemble:
    """cf_ensemble: lattices of uneven N stepped together (one work list)."""

    def __init__(self, members):
        """members: list of dicts with N, L, m and the shared equation, precision,
        stencil, a1, H1, t1, p."""
        arr = (cf_params * len(members))()
        for i, d in enumerate(members):
            arr[i] = cf_params(int(d["N"]), float(d["L"]), float(d.get("m", 1.0)), float(d.get("a1", 1.0)),
                               float(d.get("H1", 0.0)), float(d.get("t1", 0.0)), float(d.get("p", 1.0)),
                               int(d.get("equation", EQ_KG_FRW)), int(d.get("precision", FP64)),
                               int(d.get("stencil", 7)), 0, 0.0, 1.0, 0)
        self.members = members
        h = ctypes.c_void_p()
        check(lib().cf_ensemble_create(ctypes.cast(arr, ctypes.c_void_p), len(members), ctypes.byref(h)))
        self.h = h
        tot, items = _i64(0), _i64(0)
        check(lib().cf_ensemble_info(self.h, ctypes.byref(tot), ctypes.byref(items)))
        self.spectra_total = int(tot.value)
        self.work_items = int(items.value)
        self.offsets = []
        off = 0
        for d in members:
            self.offsets.append(off)
            off += 3 * (int(d["N"]) // 2) ** 2 + 1

    def close(self):
        if getattr(self, "h", None):
            lib().cf_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def launches(self):
        return int(lib().cf_ensemble_launch_count(self.h))

    def upload(self, member, h_xy, stream=None):
        check(lib().cf_ensemble_state_upload(self.h, int(member), _ptr(h_xy), _stream(stream)))

    def download(self, member, h_xy, stream=None):
        check(lib().cf_ensemble_state_download(self.h, int(member), _ptr(h_xy), _stream(stream)))

    def rk4_steps(self, t0, dt, nsteps, step0=0, mode=ENS_PERSISTENT, stream=None):
        check(lib().cf_ensemble_rk4_steps(self.h, float(t0), float(dt), int(step0), int(nsteps), int(mode),
                                          _stream(stream)))

    def density_spectra_s2(self, t, d_out, stream=None):
        check(lib().cf_ensemble_density_spectra_s2(self.h, float(t), _ptr(d_out), _stream(stream)))

    def run_graph(self, t0, dt, steps_per_segment, nsegments, d_spectra=None, stream=None, mode=ENS_BATCHED):
        check(lib().cf_ensemble_run_graph(self.h, float(t0), float(dt), int(steps_per_segment), int(nsegments),
                                          int(mode), _ptr(d_spectra), _stream(stream)))

    def set_barrier_test(self, extra_arrivals, spin_limit=1 << 24):
        check(lib().cf_ensemble_set_barrier_test(self.h, int(extra_arrivals), int(spin_limit)))

    def autotune(self, t0, dt, steps=2, stream=None):
        shape, chunk = _i(0), _i(0)
        check(lib().cf_ensemble_autotune(self.h, float(t0), float(dt), int(steps), _stream(stream),
                                         ctypes.byref(shape), ctypes.byref(chunk)))
        return int(shape.value), int(chunk.value)


def field_from_shell_amplitudes(ctx, d_xi, d_sqrtP, theta, shells_per_group, d_phi, stream=None):
    import numpy as np
    th = np.ascontiguousarray(theta, dtype=np.float64)
    check(lib().cf_field_from_shell_amplitudes(ctx.h, _ptr(d_xi), _ptr(d_sqrtP), _ptr(th), th.size,
                                               int(shells_per_group), _ptr(d_phi), _stream(stream)))


def shell_amplitude_gradient(ctx, d_lambda_phi, d_xi, d_sqrtP, theta, shells_per_group, stream=None):
    import numpy as np
    th = np.ascontiguousarray(theta, dtype=np.float64)
    g = np.empty_like(th)
    check(lib().cf_shell_amplitude_gradient(ctx.h, _ptr(d_lambda_phi), _ptr(d_xi), _ptr(d_sqrtP), _ptr(th), th.size,
                                            int(shells_per_group), _ptr(g), _stream(stream)))
    return g


def a_of_t(a1, H1, t1, t, p=1.0):
    """StaticEOSCosmology::a (reference src/physics.hpp:34-36) on the host."""
    return a1 * (1 + (1 + 1 / p) * H1 * (t - t1)) ** (p / (1 + p))
