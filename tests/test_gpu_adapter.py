"""The C++ drop-in adapter (include/cfb200_odeint.hpp) driven like the
reference driver: WorkspaceGeneric(param, initializer), an Equation functor,
odeint integrate_const with the stock runge_kutta4_classic or the fused
stepper, and ConstIntervalObserver writing the reference's .dat files.

The driver binary (tests/cpp/_build/adapter_main) is compiled by build() where
Boost.odeint headers are available; the outputs are compared with the
reference's own CPU run of the same integrate_const (oracle/_ref) when present,
else with the restated oracle.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from cfb200 import fields  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "cpp", "_build", "adapter_main")
FRW = dict(a1=1.0, H1=0.5, t1=1.0)


def load_params(project_dir):
    """The parameter reader of plot_util.py:17-34 (param.dat unpacked by the types in
    paramTypes.txt, keyed by paramNames.txt)."""
    import struct
    raw = open(project_dir + "param.dat", "rb").read()
    types = open(project_dir + "paramTypes.txt").read().split("\n")[:-1]
    names = open(project_dir + "paramNames.txt").read().split("\n")[:-1]
    fmt = "".join({"Integer64": "q", "Real64": "d"}[t] for t in types)
    vals = struct.unpack_from(fmt, raw)
    return {names[i]: vals[i] for i in range(len(vals))}


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


# adapter_main modes: equation code, and the Param fields the driver sets for it
MODES = {0: (1, {}), 1: (1, {}), 2: (1, {}), 3: (2, {}), 4: (0, {}), 5: (3, dict(lam=0.8)), 6: (4, dict(f_a=0.7)),
         7: (5, {}), 8: (6, dict(M=8))}


@pytest.mark.skipif(not os.path.exists(BIN), reason="adapter driver not built (needs Boost.odeint headers)")
@pytest.mark.parametrize("mode", sorted(MODES))
def test_adapter_integrate_const_matches_reference(mode):
    N, L, dt, nsteps = 16, 16.0, 0.05, 30
    eq, extra = MODES[mode]
    t0 = 0.0 if eq == 0 else 1.0
    t_end = t0 + (nsteps + 0.5) * dt
    ti = 0.499
    x = fields.initial_state(N, L, 0.5, 5 + mode)
    x[N ** 3:] = 0.2 * fields.gaussian_field(N, L, 0.5, 50 + mode)
    # the approximate equation's R_fft is band-limited below the coarse grid's M/2 = 4 modes
    # (k_max 1.5 < 2 pi / L * 4): the coarse c2r then sees Hermitian-consistent input
    Rf = fields.curvature_R_fft(N, L, 2.0, 1e-2, 3.0 if eq == 2 else 1.5, seed=9) if eq in (2, 6) else None
    psi = 0.05 * fields.gaussian_field(N, L, 0.5, 77) if eq == 5 else None
    aux = Rf if Rf is not None else psi
    cos = FRW if eq else {}
    if psi is not None:
        extra = dict(psi_fixed=psi)
    with tempfile.TemporaryDirectory() as d:
        xin = os.path.join(d, "x.bin")
        x.tofile(xin)
        args = [BIN, str(mode), str(N), repr(L), repr(dt), repr(t0), repr(t_end), repr(ti), xin, d + "/"]
        if aux is not None:
            rin = os.path.join(d, "r.bin")
            aux.tofile(rin)
            args.append(rin)
        out = subprocess.run(args, capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        got = np.fromfile(os.path.join(d, "state.dat"))
        t_list = np.fromfile(os.path.join(d, "t_list.dat"))
        spectra = [(np.fromfile(os.path.join(d, f"varphi_plus_spectrum_{i}.dat")),
                    np.fromfile(os.path.join(d, f"rho_spectrum_{i}.dat")),
                    np.fromfile(os.path.join(d, f"rho_slice_{i}.dat"))) for i in range(len(t_list))]
        params = load_params(d + "/")
        axis_avg = np.fromfile(os.path.join(d, f"rho_axis_average_{len(t_list) - 1}.dat"))
        fk = np.fromfile(os.path.join(d, "fft_phi0.dat")).view(complex)
        back = np.fromfile(os.path.join(d, "fft_roundtrip.dat"))
    # workspace.fft_wrapper as the reference's initializers use it (FP64, unnormalised)
    assert rel(fk, np.fft.rfftn(x[: N ** 3].reshape(N, N, N)).ravel()) <= 1e-13
    assert rel(back, x[: N ** 3] * N ** 3) <= 1e-13
    if O.ref_available() and eq <= 2:
        want, obs = O.ref_integrate(eq, N, L, 1.0, x, t0, t_end, dt, R_fft=Rf, t_interval=ti, observe=True, **cos)
        assert np.allclose(t_list, obs["t_list"], rtol=0, atol=1e-12)
    else:  # no CPU twin in the reference for equations 3-6: the restated oracle
        P = O.make_params(N, L, 1.0, eq=eq, **cos, **extra)
        want = O.rk4_steps(P, x, t0, dt, nsteps, R_fft=Rf)
        obs = None
    tol = 2e-6 if mode == 2 else 1e-12
    assert rel(got, want) <= tol
    if obs is not None:
        for i in range(len(t_list)):
            assert rel(spectra[i][0], obs["varphi_plus"][i]) <= max(tol, 1e-12) * 10
            assert rel(spectra[i][1], obs["rho"][i]) <= max(tol, 1e-12) * 10
    P = O.make_params(N, L, 1.0, eq=eq, **cos, **extra)
    rho_last = O.energy_density(P, got, t_list[-1], Rf)
    assert rel(spectra[-1][2], rho_last[: N * N]) <= 1e-12
    assert rel(axis_avg, rho_last.reshape(N, N * N).mean(axis=0)) <= 1e-12
    # param.dat / paramNames.txt / paramTypes.txt read the way plot_util.py reads them
    assert params["N"] == N and params["L"] == L and params["t_interval"] == ti
    assert params["t_start"] == t0 and params["t_end"] == t_end


@pytest.mark.skipif(not os.path.exists(BIN), reason="adapter driver not built (needs Boost.odeint headers)")
@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
def test_adapter_device_initializer_matches_reference_initializer():
    """cfb200::perturbed_grf_and_comoving_curvature_fft (host RandomNormal stream,
    transforms on the device) against the reference's own CPU initializer
    (src/initializer.hpp:150-206 compiled in oracle/_ref) with the same seed, at N = 128
    (the reference's driver parameters carry M = 128 and its workspace asserts N >= M)."""
    N = 128
    L, seed = 0.8 * N, 6
    with tempfile.TemporaryDirectory() as d:
        out = subprocess.run([BIN, "9", str(N), repr(L), str(seed), "-1", "0", "0", "-", d + "/"],
                             capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        state = np.fromfile(os.path.join(d, "state.dat"))
        R_fft = np.fromfile(os.path.join(d, "R_fft.dat"))
    with tempfile.TemporaryDirectory() as d:
        want_state, want_R = O.ref_driver_initial(N, L, seed, d, want_state=True)
    assert np.abs(state - want_state).max() <= 1e-12 * np.abs(want_state).max()
    assert np.abs(R_fft - want_R).max() <= 1e-12 * np.abs(want_R).max()


@pytest.mark.skipif(not os.path.exists(BIN), reason="adapter driver not built (needs Boost.odeint headers)")
def test_adapter_wkb_matches_oracle():
    """cfb200::WKBSolutionForKleinGordonEquationInFRW(workspace, t_i).evaluate_at(t) (mode 10)."""
    N, L, ti, tf = 16, 12.8, 3.0, 11.0
    x = fields.initial_state(N, L, 0.5, 15)
    x[N ** 3:] = 0.2 * fields.gaussian_field(N, L, 0.5, 16)
    with tempfile.TemporaryDirectory() as d:
        xin = os.path.join(d, "x.bin")
        x.tofile(xin)
        out = subprocess.run([BIN, "10", str(N), repr(L), "0.1", repr(ti), repr(tf), "1.0", xin, d + "/"],
                             capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        got = np.fromfile(os.path.join(d, "wkb.dat"))
    want = O.wkb(O.make_params(N, L, 1.0, eq=1, **FRW), x, ti, tf)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
