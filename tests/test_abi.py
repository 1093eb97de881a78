"""CPU checks of the product boundary: libcfb200.so loads and exports every
function include/cfb200.h declares; parameter validation happens on the host
before any device work; the synthetic-input generators keep their contracts."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import cfb200


def test_library_exports_every_header_symbol():
    syms = cfb200.header_symbols()
    assert len(syms) >= 20
    L = cfb200.lib()
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_build_targets_sm100a_only():
    mk = open(os.path.join(cfb200.PKG, "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk
    assert "sm_90" not in mk and "sm_80" not in mk


@pytest.mark.parametrize("kw,msg", [
    (dict(N=12), "N = 12"), (dict(N=4), "N = 4"), (dict(stencil=9), "stencil"),
    (dict(equation=7), "equation"), (dict(precision=5), "precision"), (dict(L=-1.0), "L must"),
    (dict(equation=2, H1=0.0), "conformal"), (dict(equation=6, H1=0.0, M=8), "conformal"),
    (dict(equation=4, f_a=0.0), "f_a"), (dict(equation=4, f_a=float("inf")), "f_a"),
    (dict(equation=3, lam=float("nan")), "lambda"),
    (dict(equation=6, M=0), "M = 0"), (dict(equation=6, M=12), "M = 12"), (dict(equation=6, M=32), "M = 32"),
    (dict(N=24, equation=6, M=16), "M = 16"),
])
def test_create_rejects_bad_parameters_on_host(kw, msg):
    args = dict(N=16, L=16.0, m=1.0, equation=1, precision=0, stencil=7, a1=1.0, H1=0.5, t1=1.0)
    args.update(kw)
    with pytest.raises(cfb200.CfError) as e:
        cfb200.Context(**args)
    assert e.value.code == -1 and msg in str(e.value)


def test_fft_wrapper_rejects_bad_sizes_on_host():
    import ctypes
    h = ctypes.c_void_p()
    for n in (7, 4, 4096):
        assert cfb200.lib().cf_fft_create(n, ctypes.byref(h)) == -1
        assert b"cf_fft_create" in cfb200.lib().cf_last_error()


def test_calls_reject_null_context():
    L = cfb200.lib()
    assert L.cf_rk4_steps(None, None, 0.0, 0.1, 0, 1, None) == -1
    assert b"NULL context" in L.cf_last_error()
    r, u = ctypes.c_int64(7), ctypes.c_int64(7)
    assert L.cf_psi_stats(None, ctypes.byref(r), ctypes.byref(u)) == -1
    assert (r.value, u.value) == (7, 7)
    assert L.cf_psi_set_wait_test(None, 16, 1 << 10) == -1
    assert b"NULL context" in L.cf_last_error()


def test_unknown_flags_are_rejected_on_host():
    args = dict(N=16, L=16.0, m=1.0, equation=2, precision=1, stencil=7, a1=1.0, H1=0.5, t1=1.0)
    assert cfb200.FLAG_PSI_NO_REUSE == 64
    with pytest.raises(cfb200.CfError) as e:
        cfb200.Context(**args, flags=128)
    assert e.value.code == -1 and "unknown flags" in str(e.value)


def test_gaussian_field_contract():
    from cfb200 import fields
    phi = fields.gaussian_field(32, 32.0, 0.5, seed=3)
    assert phi.shape == (32 ** 3,)
    assert abs(phi.mean()) < 1e-12  # P(0) = 0
    assert 0.5 < (phi ** 2).mean() < 1.5
    # same seed, same field
    assert np.array_equal(phi, fields.gaussian_field(32, 32.0, 0.5, seed=3))


def test_curvature_R_fft_contract():
    from cfb200 import fields
    N, L = 32, 32.0
    hc = fields.curvature_R_fft(N, L, eta_start=2.0, psi_rms=1e-2, k_max=0.5, seed=5)
    assert hc.size == 2 * N * N * (N // 2 + 1)
    z = hc.view(complex).reshape(N, N, N // 2 + 1)
    k = fields._kgrid_half(N, L)
    assert np.all(z[k > 0.5] == 0)  # exact: the pruned Psi synthesis relies on the zeros
