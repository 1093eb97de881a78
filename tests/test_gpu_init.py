"""GPU initial conditions (cf_white_noise, cf_grf, cf_scale_modes and the Python /
C++ initializers built on them) against the oracle and the reference's published
initial outputs.

Tolerances (written per test): deviates from the device generator equal the
restated generator to 1e-14 (CUDA's and glibc's log / sin / cos differ in the last
bits); fields built from the same deviates agree with the oracle to <= 1e-12 of their
largest value (FFT rounding); the published N=384 spectra are matched to 2e-12 per
bin, the tolerance the oracle pins use.
"""
import math

import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cfb200  # noqa: E402
from cfb200 import initializer as I  # noqa: E402


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def relmax(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / np.abs(b).max())


def ctx_of(N, L, eq=cfb200.EQ_KG_FRW, **kw):
    return cfb200.Context(N, L, m=1.0, equation=eq, a1=1.0, H1=kw.pop("H1", 0.5), t1=kw.pop("t1", 1.0), **kw)


def test_white_noise_matches_restatement_and_splits():
    c = ctx_of(16, 16.0)
    n = (1 << 20) + 3
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    c.white_noise(out, 11, offset=5)
    got = out.cpu().numpy()
    want = O.white_noise(11, 5, n)
    assert np.abs(got - want).max() <= 1e-14
    # any split of the stream into calls gives the same deviates (odd offsets included)
    parts = torch.empty(n, dtype=torch.float64, device="cuda")
    c.white_noise(parts[:1001], 11, offset=5, n=1001)
    c.white_noise(parts[1001:], 11, offset=5 + 1001, n=n - 1001)
    assert torch.equal(parts, out)
    assert abs(got.mean()) < 5 / np.sqrt(n) and abs(got.var() - 1) < 5 * np.sqrt(2 / n)
    other = torch.empty(1000, dtype=torch.float64, device="cuda")
    c.white_noise(other, 12)
    assert not np.allclose(other.cpu().numpy(), got[:1000])


@pytest.mark.parametrize("N", [16, 24, 32])
@pytest.mark.parametrize("kind,with_psi", [(0, False), (0, True), (1, True), (2, False)])
def test_grf_matches_oracle(N, kind, with_psi):
    L = 0.8 * N
    c = ctx_of(N, L)
    w = O.normals(5, N ** 3)
    args = {0: [2.3, 1.0, 0.0], 1: [2.3, 1.0, 0.0, 1.0], 2: [1e-5]}[kind]
    psi = 0.05 * O.normals(9, N ** 3) if with_psi else None
    want = O.grf_white(N, L, w, kind, args, psi, -0.4 if with_psi else 0.0)
    out = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
    c.grf(dev(w), O.sqrtP_table(N, L, kind, args), out, d_psi=dev(psi) if with_psi else None,
          psi_scale=-0.4 if with_psi else 0.0)
    assert relmax(out.cpu().numpy(), want) <= 1e-12


def test_scale_modes_and_in_place_calls():
    N, L = 32, 25.6
    c = ctx_of(N, L)
    f = O.normals(2, N ** 3)
    tab = np.cos(0.01 * np.arange(O.n_s2(N))) / N ** 3
    out = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
    c.scale_modes(dev(f), tab, out)
    a = np.arange(N)
    a = np.minimum(a, N - a)
    s2 = a[:, None, None] ** 2 + a[None, :, None] ** 2 + np.arange(N // 2 + 1)[None, None, :] ** 2
    want = np.fft.irfftn(np.fft.rfftn(f.reshape(N, N, N)) * tab[s2], s=(N,) * 3, axes=(0, 1, 2)).ravel() * N ** 3
    assert relmax(out.cpu().numpy(), want) <= 1e-12
    inplace = dev(f)
    c.scale_modes(inplace, tab, inplace)
    assert torch.equal(inplace, out)


@pytest.mark.parametrize("N", [16, 32])
def test_driver_initializer_with_the_reference_stream_matches_oracle(N):
    """The reference driver's initializer on the device (cfb200.initializer) fed the
    reference's own deviates gives the restated initializer's state and R_fft."""
    L = 0.8 * N
    seed = 4
    want_state, want_R = O.driver_initial(N, L, seed)
    c = ctx_of(N, L, eq=cfb200.EQ_COMOVING_FRW, H1=0.05, t1=10.0)
    state, R_fft = I.perturbed_grf_and_comoving_curvature_fft(c, 10.0, 0.02, 1.0, 1.0,
                                                               dev(O.normals(seed, 3 * N ** 3)))
    assert relmax(state.cpu().numpy()[: N ** 3], want_state[: N ** 3]) <= 1e-12
    assert relmax(state.cpu().numpy()[N ** 3:], want_state[N ** 3:]) <= 1e-12
    assert relmax(R_fft.cpu().numpy(), want_R) <= 1e-12


def _cmp_fixture(golden, name, arr, tol):
    idx = golden[name + "_idx"]
    val = golden[name + "_val"]
    assert arr.size == int(golden[name + "_size"][0])
    big = np.abs(val) >= 1e-10 * np.abs(val).max()
    rel = np.abs(arr[idx] - val)[big] / np.abs(val)[big]
    assert rel.max() <= tol, (name, rel.max())


def test_device_initializer_reproduces_published_initial_outputs(golden):
    """N=384, seed 0 (the reference's output/Growth_and_FS run): initial R and Psi
    spectra, rho spectrum, field spectrum and rho slice at t_start, all from fields
    made on the device from the reference's deviate stream."""
    N, L, t0 = 384, 384 * 0.8, 10.0
    c = ctx_of(N, L, eq=cfb200.EQ_COMOVING_FRW, H1=0.05, t1=10.0)
    state, R_fft = I.perturbed_grf_and_comoving_curvature_fft(c, t0, 0.02, 1.0, 1.0, dev(O.normals(0, 3 * N ** 3)))
    spec = torch.empty(O.n_s2(N), dtype=torch.float64, device="cuda")
    # R = z2d(R_fft) / N^3 (src/main.cpp:168), its spectrum and that of Psi
    R = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
    z = R_fft.clone()
    cfb200.FFT(N).z2d(z, R)
    R /= N ** 3
    c.power_spectrum_s2(R, spec)
    _cmp_fixture(golden, "initial_R_spectrum", spec.cpu().numpy(), 2e-12)
    eta_i = 1.0 / 0.05  # conformal time at t1: p / (a1 H1)

    def kernel(k):
        if k == 0.0:
            return 0.0
        r3 = math.sqrt(3)
        return (6 * r3 * (-((k * eta_i * math.cos((k * eta_i) / r3)) / r3) + math.sin((k * eta_i) / r3))) / \
            (k ** 3 * eta_i ** 3)

    Psi = torch.empty_like(R)
    c.scale_modes(R, I.kernel_table(N, L, kernel), Psi)
    c.power_spectrum_s2(Psi, spec)
    _cmp_fixture(golden, "initial_Psi_spectrum", spec.cpu().numpy(), 2e-12)
    a_t = 1.0
    c.mode_power_spectrum_s2(state, a_t, spec)
    _cmp_fixture(golden, "varphi_plus_spectrum_0", spec.cpu().numpy(), 2e-12)
    c.set_R_fft(R_fft, on_device=True)
    rho = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
    c.energy_density(state, t0, rho)
    c.power_spectrum_s2(rho, spec)
    _cmp_fixture(golden, "rho_spectrum_0", spec.cpu().numpy(), 2e-12)
    _cmp_fixture(golden, "rho_slice_0", rho[: N * N].cpu().numpy(), 2e-12)


def test_device_noise_initializer_statistics():
    """With device deviates the fields are a different realisation of the same
    statistics: Psi's rms at t_start is the requested 0.02 (to sampling error)."""
    N, L = 128, 102.4
    c = ctx_of(N, L, eq=cfb200.EQ_COMOVING_FRW, H1=0.05, t1=10.0)
    state, R_fft = I.perturbed_grf_and_comoving_curvature_fft(c, 10.0, 0.02, 1.0, 1.0, noise=123)
    c.set_R_fft(R_fft, on_device=True)
    fields2 = torch.empty(2 * N ** 3, dtype=torch.float64, device="cuda")
    c.psi_fields(10.0, fields2)
    psi = fields2[: N ** 3].cpu().numpy()
    assert 0.01 < psi.std() < 0.04
    phi = state[: N ** 3].cpu().numpy()
    assert 0.5 < phi.std() < 2.0
