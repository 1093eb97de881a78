"""The oracles are pinned before anything is checked against them.

* The reference's own CPU sources, compiled here against the FFTW3 restatement
  (oracle/_ref), reproduce the reference's published N=384 outputs
  (output/Growth_and_FS/*_0.dat, initial_*.dat).
* The C restatement (oracle/liboracle.so) reproduces the same published outputs
  from scratch (its own mt19937 + polar normal deviates, GRF, transfer function,
  FFT), and agrees with the reference build on identical inputs at small N for
  every hot-path function.
"""
import os
import tempfile

import numpy as np
import pytest

import oracle as O

N384, L384 = 384, 384 * 0.8


def _cmp_fixture(golden, name, arr, tol):
    idx = golden[name + "_idx"]
    val = golden[name + "_val"]
    assert arr.size == int(golden[name + "_size"][0])
    got = arr[idx]
    big = np.abs(val) >= 1e-10 * np.abs(val).max()
    rel = np.abs(got - val)[big] / np.abs(val)[big]
    assert rel.max() <= tol, (name, rel.max())
    assert abs(arr.sum() - golden[name + "_sum"][0]) <= tol * abs(golden[name + "_sum"][0])


def test_fftw_restatement_matches_numpy():
    for N in (4, 6, 8, 12, 16, 24, 30):
        rng = np.random.default_rng(N)
        x = rng.standard_normal(N ** 3)
        hc = O.d2z(x).view(complex).reshape(N, N, N // 2 + 1)
        ref = np.fft.rfftn(x.reshape(N, N, N))
        assert np.abs(hc - ref).max() <= 1e-14 * np.abs(ref).max()


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
def test_reference_build_reproduces_published_outputs(golden):
    with tempfile.TemporaryDirectory() as d:
        O.ref_driver_initial(N384, L384, 0, d)
        for name in ["initial_R_spectrum", "initial_Psi_spectrum", "rho_spectrum_0",
                     "varphi_plus_spectrum_0", "rho_slice_0", "rho_axis_average_0"]:
            arr = np.fromfile(os.path.join(d, name + ".dat"))
            _cmp_fixture(golden, name, arr, 2e-12)


def test_restatement_reproduces_published_outputs(golden):
    state, R_fft = O.driver_initial(N384, L384, 0)
    P = O.make_params(N384, L384, 1.0, eq=2, a1=1.0, H1=0.05, t1=10.0)
    t0 = 10.0
    # R = z2d(R_fft)/N^3 (src/main.cpp:168) via the restated c2r inside psi machinery:
    z = R_fft.view(complex).reshape(N384, N384, N384 // 2 + 1)
    R = np.fft.irfftn(z, s=(N384,) * 3, axes=(0, 1, 2)).ravel()
    _cmp_fixture(golden, "initial_R_spectrum", O.power_spectrum(R), 2e-12)
    _cmp_fixture(golden, "varphi_plus_spectrum_0",
                 O.mode_power_spectrum(N384, L384, 1.0, O.a_of_t(P, t0), state), 2e-12)
    rho = O.energy_density(P, state, t0, R_fft)
    _cmp_fixture(golden, "rho_spectrum_0", O.power_spectrum(rho), 2e-12)
    _cmp_fixture(golden, "rho_slice_0", rho[: N384 * N384], 2e-12)


def _grf(N, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((2, N, N, N))
    k = np.fft.fftfreq(N) * 2 * np.pi
    kk = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    f = np.fft.ifftn(np.fft.fftn(x, axes=(1, 2, 3)) * np.exp(-kk / (2 * 0.5 ** 2)), axes=(1, 2, 3)).real
    return (f / f.std()).ravel() * np.array([1.0] * N ** 3 + [0.3] * N ** 3)


EQS = [(0, dict()), (1, dict(a1=1.0, H1=0.5, t1=1.0)), (2, dict(a1=1.0, H1=0.5, t1=1.0))]


def _rfft_input(N, seed):
    rng = np.random.default_rng(seed + 99)
    R = 1e-2 * rng.standard_normal(N ** 3)
    return O.d2z(R)


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("eq,cos", EQS)
@pytest.mark.parametrize("N", [8, 12, 16])
def test_restatement_matches_reference_rhs_and_density(eq, cos, N):
    L = float(N) * 0.9
    x = _grf(N, N + eq)
    Rf = _rfft_input(N, N) if eq == 2 else None
    P = O.make_params(N, L, 1.3, eq=eq, **cos)
    t = 1.7
    a = O.rhs(P, x, t, Rf)
    b = O.ref_rhs(eq, N, L, 1.3, x, t, R_fft=Rf, **cos)
    assert np.linalg.norm(a - b) <= 1e-14 * np.linalg.norm(b)
    a = O.energy_density(P, x, t, Rf)
    b = O.ref_energy_density(eq, N, L, 1.3, x, t, R_fft=Rf, **cos)
    assert np.linalg.norm(a - b) <= 1e-14 * np.linalg.norm(b)
    assert np.abs(O.power_spectrum(a) - O.ref_power_spectrum(a)).max() <= 1e-13 * np.abs(O.ref_power_spectrum(a)).max()


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("eq,cos", EQS)
def test_restatement_matches_reference_integrate_const(eq, cos):
    N, L, m = 16, 16.0, 1.0
    x = _grf(N, 7 + eq)
    Rf = _rfft_input(N, 3) if eq == 2 else None
    t0 = 1.0 if eq else 0.0
    dt, nsteps = 0.1, 20
    t_end = t0 + (nsteps + 0.5) * dt  # half a step of margin: see test_reference_noise_floor_is_small
    ref_state, obs = O.ref_integrate(eq, N, L, m, x, t0, t_end, dt, R_fft=Rf, t_interval=0.999,
                                     observe=True, **cos)
    P = O.make_params(N, L, m, eq=eq, **cos)
    mine = O.rk4_steps(P, x, t0, dt, nsteps, R_fft=Rf)
    for part in (slice(0, N ** 3), slice(N ** 3, None)):
        assert np.linalg.norm(mine[part] - ref_state[part]) <= 1e-12 * np.linalg.norm(ref_state[part])
    # the observer saved at t0 and every ~1.0 after it, plus the final time
    assert obs["t_list"][0] == t0 and abs(obs["t_list"][-1] - (t0 + nsteps * dt)) < 1e-12
    last_rho = O.power_spectrum(O.energy_density(P, mine, obs["t_list"][-1], Rf))
    assert np.linalg.norm(last_rho - obs["rho"][-1]) <= 1e-12 * np.linalg.norm(obs["rho"][-1])
    a_t = O.a_of_t(P, obs["t_list"][-1]) if eq else 1.0
    last_fs = O.mode_power_spectrum(N, L, m, a_t, mine)
    assert np.linalg.norm(last_fs - obs["varphi_plus"][-1]) <= 1e-12 * np.linalg.norm(obs["varphi_plus"][-1])


@pytest.mark.skipif(not O.ref_available(strict=True), reason="strict reference build not present")
def test_reference_noise_floor_is_small():
    """-ffast-math (the reference's own flags) vs strict IEEE build of the same
    sources: the noise floor every parity tolerance sits above.

    t_end sits half a step past the last step time: with t_end = t0 + n*dt
    exactly, integrate_const's `t + dt <= t_end + eps` test
    (util/detail/less_with_sign.hpp:47-53) takes n or n-1 steps depending on
    how the compiler rounds t0 + step*dt, and the two builds differ there."""
    N, L, m = 16, 16.0, 1.0
    x = _grf(N, 5)
    a, _ = O.ref_integrate(1, N, L, m, x, 1.0, 3.05, 0.1, a1=1.0, H1=0.5, t1=1.0)
    b, _ = O.ref_integrate(1, N, L, m, x, 1.0, 3.05, 0.1, a1=1.0, H1=0.5, t1=1.0, strict=True)
    assert np.linalg.norm(a - b) <= 1e-13 * np.linalg.norm(b)


def test_mode_counts_match_multiplicity_rule():
    for N in (4, 6, 8, 10):
        r = np.arange(-N // 2 + 1, N // 2 + 1)
        s2 = (r[:, None, None] ** 2 + r[None, :, None] ** 2 + r[None, None, :] ** 2).ravel()
        ref = np.bincount(s2, minlength=3 * (N // 2) ** 2 + 1)
        assert np.array_equal(O.s2_counts(N), ref)
        _, sc = O.shells_from_s2(N)
        assert sc.sum() == N ** 3
        sh = np.floor(np.sqrt(s2)).astype(int)
        assert np.array_equal(sc, np.bincount(sh, minlength=sc.size))


def test_known_answer_homogeneous_field():
    """Flat KG with a homogeneous field: phi(t) = f cos(m t) (RK4 error O(dt^4))."""
    N, L, m, f = 8, 8.0, 1.0, 1.0
    x = np.concatenate([np.full(N ** 3, f), np.zeros(N ** 3)])
    P = O.make_params(N, L, m, eq=0)
    y = O.rk4_steps(P, x, 0.0, 0.1, 100)
    assert np.allclose(y[: N ** 3], f * np.cos(m * 10.0), atol=2e-6)
    assert np.allclose(y[N ** 3:], -f * m * np.sin(m * 10.0), atol=2e-6)


@pytest.mark.parametrize("stencil", [7, 13])
def test_known_answer_plane_wave_dispersion(stencil):
    """plane_wave initial condition (src/initializer.hpp:251-269): cos(2 pi c/N)
    oscillates at the lattice frequency w^2 = m^2 + lambda_h(theta)/h^2."""
    N, L, m = 16, 16.0, 1.0
    c = np.arange(N)
    phi = np.broadcast_to(np.cos(2 * np.pi * c / N), (N, N, N)).ravel()
    x = np.concatenate([phi, np.zeros(N ** 3)])
    P = O.make_params(N, L, m, eq=0, stencil=stencil)
    th = 2 * np.pi / N
    lam = 2 - 2 * np.cos(th) if stencil == 7 else (30 - 32 * np.cos(th) + 2 * np.cos(2 * th)) / 12
    w = np.sqrt(m * m + lam)
    y = O.rk4_steps(P, x, 0.0, 0.02, 250)
    assert np.allclose(y[: N ** 3], phi * np.cos(w * 5.0), atol=1e-7)


@pytest.mark.parametrize("stencil,order", [(7, 2), (13, 4)])
def test_laplacian_convergence_order_on_a_plane_wave(stencil, order):
    """The 7-point Laplacian converges as h^2 and the 13-point one as h^4: on
    cos(2 pi (a + 2 b + 3 c) / N) with L fixed, the right-hand side's pi part
    (flat KG, m = 0: h^-2 Delta_h phi) approaches -(2 pi / L)^2 (1 + 4 + 9) phi,
    and halving h divides the error by 2^order."""
    L = 8.0
    errs = []
    for N in (16, 32, 64):
        i = np.arange(N)
        A, Bb, Cc = np.meshgrid(i, i, i, indexing="ij")
        phi = np.cos(2 * np.pi * (A + 2 * Bb + 3 * Cc) / N).ravel()
        x = np.concatenate([phi, np.zeros(N ** 3)])
        P = O.make_params(N, L, 0.0, eq=0, stencil=stencil)
        lap = O.rhs(P, x, 0.0, None)[N ** 3:]
        exact = -(2 * np.pi / L) ** 2 * 14.0 * phi
        errs.append(float(np.abs(lap - exact).max() / np.abs(exact).max()))
    rates = [np.log2(errs[k] / errs[k + 1]) for k in range(2)]
    assert all(abs(r - order) < 0.15 for r in rates), (errs, rates)


# ---- the GPU-only functors: pinned to the reference's own GPU build ------------
# tests/golden/ref_gpu_equations.npz holds outputs of src/equations_cuda.cu itself
# (oracle/ref_gpu_golden.cu, built from the reference sources and run on a GPU;
# inputs rebuilt bit for bit by tests/golden/ref_gpu_inputs.py).

import sys  # noqa: E402

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import ref_gpu_inputs as G  # noqa: E402

GPU_GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_gpu_equations.npz")


def _relmax(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("case", ["lambda", "sqrt", "fixed", "approx", "approx_fullband"])
def test_restatement_matches_reference_gpu_functors(case):
    """rhs (operator()), energy density and one runge_kutta4_classic step of the
    restated equations 3-6 against the reference's GPU functors on the same inputs
    (1e-12 of the largest value: FP64 rounding of a few operations per site)."""
    g = np.load(GPU_GOLDEN)
    P = G.oracle_params(O, case)
    x, Rf, _ = G.inputs(case)
    assert _relmax(O.rhs(P, x, G.T, Rf), g[case + "_rhs"]) <= 1e-12
    if case + "_rho" in g:
        assert _relmax(O.energy_density(P, x, G.T, Rf), g[case + "_rho"]) <= 1e-12
    if case + "_step" in g:
        assert _relmax(O.rk4_steps(P, x, G.T, G.DT, 1, R_fft=Rf), g[case + "_step"]) <= 1e-12


def test_restatement_matches_reference_gpu_dot_energy_density():
    g = np.load(GPU_GOLDEN)["kgfrw_dot_rho"]
    lat = G.SMALL
    P = O.make_params(lat["N"], lat["L"], lat["m"], eq=1, **G.FRW)
    assert _relmax(O.dot_energy_density(P, G.state(lat["N"]), G.T), g) <= 1e-12


# ---- initial conditions --------------------------------------------------------

def test_philox_known_answers():
    """Philox4x32-10 against the known-answer vectors published with the Random123
    library of Salmon et al. (SC'11): zero, all-ones and pi-digit counters / keys."""
    assert list(O.philox4x32_10([0, 0, 0, 0], [0, 0])) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(O.philox4x32_10([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6,
                                                                         0x6D5451FD]
    assert list(O.philox4x32_10([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0])) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_white_noise_restatement_is_standard_normal():
    w = O.white_noise(7, 0, 1 << 20)
    n = w.size
    assert abs(w.mean()) < 5 / np.sqrt(n)
    assert abs(w.var() - 1) < 5 * np.sqrt(2 / n)
    assert abs((w ** 4).mean() - 3) < 5 * np.sqrt(96 / n)
    assert np.array_equal(O.white_noise(7, 12345, 100), w[12345:12445])


def test_grf_from_the_stream_equals_grf_from_its_deviates():
    """The reference driver's fields rebuilt from the stream's deviates through the
    per-s^2 tables (the form the device path takes) equal the per-mode restatement."""
    N, L = 16, 12.8
    st, Rf = O.driver_initial(N, L, 3)
    w = O.normals(3, 3 * N ** 3)
    tR, kern, tf, tdf, al = O.driver_tables(N, L)
    a = np.arange(N)
    a = np.minimum(a, N - a)
    s2 = a[:, None, None] ** 2 + a[None, :, None] ** 2 + np.arange(N // 2 + 1)[None, None, :] ** 2

    def rt(f, tab):
        return np.fft.irfftn(np.fft.rfftn(f.reshape(N, N, N)) * tab[s2], s=(N,) * 3, axes=(0, 1, 2)).ravel() * N ** 3

    R = rt(w[: N ** 3] / N ** 3, tR)
    Psi = rt(R, kern)
    phi = rt(w[N ** 3: 2 * N ** 3] / N ** 3 * np.exp(al[0] * Psi), tf)
    assert _relmax(phi, st[: N ** 3]) <= 1e-13
    assert _relmax(np.fft.rfftn(R.reshape(N, N, N)).ravel().view(float), Rf) <= 1e-13


def test_cosine_integral_matches_scipy():
    """Ci(x) of the driver's A_s (series to x = 2, continued fraction beyond) against
    scipy.special.sici, absolute error near Ci's zeros."""
    sici = pytest.importorskip("scipy.special").sici
    import ctypes
    L = O.lib()
    L.cfo_ci.restype = ctypes.c_double
    L.cfo_ci.argtypes = [ctypes.c_double]
    for x in np.concatenate([np.linspace(0.05, 2, 40), np.linspace(2.001, 30, 120), [100.0, 1000.0]]):
        want = sici(x)[1]
        assert abs(L.cfo_ci(x) - want) <= 1e-15 * max(1.0, abs(want)) + 2e-16, x


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("N", [8, 16])
def test_restatement_matches_reference_wkb(N):
    """WKBSolutionForKleinGordonEquationInFRW (src/wkb.cpp, compiled in oracle/_ref) against
    the restatement, both FP64 with the FFTW restatement: <= 1e-13 of the largest value."""
    from cfb200 import fields
    L = 0.8 * N
    x = fields.initial_state(N, L, 0.5, 3)
    x[N ** 3:] = 0.3 * fields.gaussian_field(N, L, 0.5, 4)
    P = O.make_params(N, L, 1.0, eq=1, a1=1.0, H1=0.5, t1=1.0)
    for t_f in (6.0, 40.0):
        assert _relmax(O.wkb(P, x, 5.0, t_f), O.ref_wkb(N, L, 1.0, x, 5.0, t_f)) <= 1e-13
