"""GPU parity of the GPU-only equation functors of the reference (src/equations_cuda.cu):
lambda phi^4, the sqrt potential, fixed curvature, approximate comoving curvature,
and d rho / dt of the FRW Klein-Gordon equation -- libcfb200.so through its C ABI
against the restated oracle (which tests/test_oracle_pin.py pins to the reference's
own GPU build) and directly against the reference-GPU golden vectors.

Tolerances (written per test): FP64 paths agree to <= 1e-12 relative with the FP64
oracle and the golden vectors (rounding of a few operations per site and stage);
FP32-compensated trajectories to <= 2e-6 relative (the FP32 stage storage budget);
the paired-stage and the single-stage kernels bit for bit.
"""
import os
import sys

import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cfb200  # noqa: E402
from cfb200 import fields  # noqa: E402

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import ref_gpu_inputs as G  # noqa: E402

FRW = dict(a1=1.0, H1=0.5, t1=1.0)
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_gpu_equations.npz")
EQS = {3: dict(lam=0.8), 4: dict(f_a=0.7), 5: {}, 6: {}}


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def relmax(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


def setup(N, L, eq, prec=cfb200.FP64, stencil=7, flags=0, seed=3, M=None):
    """A context for equation eq with its inputs: state, R_fft (eq 6, band-limited
    below the coarse grid's M/2 modes), Psi (eq 5); returns (ctx, x, R_fft, Psi, oracle params)."""
    x = fields.initial_state(N, L, 0.5, seed)
    x[N ** 3:] = 0.3 * fields.gaussian_field(N, L, 0.5, seed + 1)
    kw = dict(EQS[eq])
    Rf = psi = None
    if eq == 6:
        # the coarse grid: M % 8 == 0 and N % M == 0, at most N / 2 unless given
        M = M or max(m for m in range(8, N // 2 + 1, 8) if N % m == 0)
        kw["M"] = M
        k_band = 2 * np.pi / L * (M // 2) * 0.95
        Rf = fields.curvature_R_fft(N, L, eta_start=2.0, psi_rms=2e-2, k_max=k_band, seed=seed + 2)
    if eq == 5:
        psi = 0.05 * fields.gaussian_field(N, L, 0.5, seed + 3)
    c = cfb200.Context(N, L, m=1.0, equation=eq, precision=prec, stencil=stencil, flags=flags, **FRW, **kw)
    if Rf is not None:
        c.set_R_fft(Rf, on_device=False)
    if psi is not None:
        c.set_psi(psi, on_device=False)
    P = O.make_params(N, L, 1.0, eq=eq, stencil=stencil, **FRW, **kw, psi_fixed=psi)
    return c, x, Rf, psi, P


@pytest.mark.parametrize("stencil", [7, 13])
@pytest.mark.parametrize("eq", sorted(EQS))
@pytest.mark.parametrize("N", [16, 40])
def test_rhs_matches_oracle(N, eq, stencil):
    L = 0.8 * N
    c, x, Rf, _, P = setup(N, L, eq, stencil=stencil, seed=10 + N)
    dd = torch.empty(2 * N ** 3, dtype=torch.float64, device="cuda")
    t = 1.37
    c.rhs(dev(x), dd, t)
    got = dd.cpu().numpy()
    want = O.rhs(P, x, t, Rf)
    assert np.array_equal(got[: N ** 3], want[: N ** 3])
    assert relmax(got[N ** 3:], want[N ** 3:]) <= 1e-13


@pytest.mark.parametrize("prec,tol", [(cfb200.FP64, 1e-12), (cfb200.FP32_COMP, 2e-6)])
@pytest.mark.parametrize("stencil", [7, 13])
@pytest.mark.parametrize("eq", sorted(EQS))
def test_rk4_matches_oracle(eq, stencil, prec, tol):
    N, L, nsteps, dt = 32, 28.0, 12, 0.1
    c, x, Rf, _, P = setup(N, L, eq, prec=prec, stencil=stencil, seed=5 + eq)
    st = torch.empty(c.info.state_bytes // 8, dtype=torch.float64, device="cuda")
    c.upload(st, x)
    c.rk4_steps(st, 1.0, dt, nsteps)
    got = np.empty_like(x)
    c.download(got, st)
    torch.cuda.synchronize()
    want = O.rk4_steps(P, x, 1.0, dt, nsteps, R_fft=Rf)
    assert rel(got[: N ** 3], want[: N ** 3]) <= tol
    assert rel(got[N ** 3:], want[N ** 3:]) <= tol


@pytest.mark.parametrize("stencil", [7, 13])
@pytest.mark.parametrize("prec", [cfb200.FP64, cfb200.FP32_COMP])
@pytest.mark.parametrize("N", [64, 40])
@pytest.mark.parametrize("eq", sorted(EQS))
def test_pair_equals_stage_kernels_bitwise(eq, N, prec, stencil):
    """The default route (the whole-step pass; for the 13-point stencil the
    paired passes in FP64 and for the curvature-coupled equations) and the four
    single-stage kernels (CF_FLAG_STAGE_KERNELS) give bit-identical states, odd and
    even step counts, full tiles (N = 64) and ragged ones (N = 40)."""
    L = 0.9 * N
    out = []
    for flags in (0, cfb200.FLAG_STAGE_KERNELS):
        c, x, _, _, _ = setup(N, L, eq, prec=prec, stencil=stencil, flags=flags, seed=21, M=8)
        st = torch.empty(c.info.state_bytes // 8, dtype=torch.float64, device="cuda")
        c.upload(st, x)
        c.rk4_steps(st, 1.0, 0.07, 3)
        got = np.empty_like(x)
        c.download(got, st)
        torch.cuda.synchronize()
        out.append(got)
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("prec,tol", [(cfb200.FP64, 1e-13), (cfb200.FP32_COMP, 1e-6)])
@pytest.mark.parametrize("eq", sorted(EQS))
def test_energy_density_matches_oracle(eq, prec, tol):
    N, L = 24, 20.0
    c, x, Rf, _, P = setup(N, L, eq, prec=prec, seed=31)
    st = torch.empty(c.info.state_bytes // 8, dtype=torch.float64, device="cuda")
    c.upload(st, x)
    rho = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
    c.energy_density(st, 1.3, rho)
    want = O.energy_density(P, x, 1.3, Rf)
    assert relmax(rho.cpu().numpy(), want) <= tol


@pytest.mark.parametrize("prec,tol", [(cfb200.FP64, 1e-13), (cfb200.FP32_COMP, 1e-6)])
def test_dot_energy_density_matches_oracle(prec, tol):
    N, L = 24, 20.0
    x = fields.initial_state(N, L, 0.5, 41)
    x[N ** 3:] = 0.3 * fields.gaussian_field(N, L, 0.5, 42)
    c = cfb200.Context(N, L, m=1.0, equation=cfb200.EQ_KG_FRW, precision=prec, **FRW)
    st = torch.empty(c.info.state_bytes // 8, dtype=torch.float64, device="cuda")
    c.upload(st, x)
    out = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
    c.dot_energy_density(st, 1.3, out)
    want = O.dot_energy_density(O.make_params(N, L, 1.0, eq=1, **FRW), x, 1.3)
    assert relmax(out.cpu().numpy(), want) <= tol


def test_dot_energy_density_is_the_time_derivative():
    """d rho / dt against a centred difference of rho along the trajectory (the
    7-point discretisation's own energy balance; O(dt^2))."""
    N, L, dt = 32, 28.0, 1e-3
    x = fields.initial_state(N, L, 0.5, 43)
    c = cfb200.Context(N, L, m=1.0, equation=cfb200.EQ_KG_FRW, **FRW)
    st = dev(x)
    rho = [torch.empty(N ** 3, dtype=torch.float64, device="cuda") for _ in range(2)]
    t0 = 1.3
    s_m = dev(x)
    c.rk4_steps(s_m, t0, -dt, 1)  # state at t0 - dt
    s_p = dev(x)
    c.rk4_steps(s_p, t0, dt, 1)  # state at t0 + dt
    c.energy_density(s_m, t0 - dt, rho[0])
    c.energy_density(s_p, t0 + dt, rho[1])
    fd = ((rho[1] - rho[0]) / (2 * dt)).cpu().numpy()
    out = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
    c.dot_energy_density(st, t0, out)
    assert rel(out.cpu().numpy(), fd) <= 1e-4


def test_unsupported_combinations_fail_loudly():
    N, L = 16, 12.0
    c = cfb200.Context(N, L, equation=cfb200.EQ_FIXED_CURVATURE_FRW, **FRW)
    st = dev(np.zeros(2 * N ** 3))
    with pytest.raises(cfb200.CfError, match="cf_set_psi"):
        c.rk4_steps(st, 1.0, 0.1, 1)
    c2 = cfb200.Context(N, L, equation=cfb200.EQ_APPROX_COMOVING_FRW, M=8, **FRW)
    with pytest.raises(cfb200.CfError, match="cf_set_R_fft"):
        c2.rk4_steps(st, 1.0, 0.1, 1)
    with pytest.raises(cfb200.CfError, match="not CF_EQ_FIXED"):
        c2.set_psi(np.zeros(N ** 3), on_device=False)
    out = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
    with pytest.raises(cfb200.CfError, match="CF_EQ_KG_FRW only"):
        c2.dot_energy_density(st, 1.0, out)
    c3 = cfb200.Context(N, L, equation=cfb200.EQ_LAMBDA_FRW, precision=cfb200.FP32_COMP, lam=0.5, **FRW)
    with pytest.raises(cfb200.CfError, match="ensembles|adjoint"):
        cfb200.Adjoint(c3, 4, 2)


# ---- the reference's own GPU functors (golden vectors) ------------------------

golden = pytest.mark.skipif(not os.path.exists(GOLDEN), reason="reference-GPU golden vectors not generated")


def golden_ctx(case, prec=cfb200.FP64):
    eq, lat, _, fixed = G.CASES[case]
    x, Rf, psi = G.inputs(case)
    kw = {k: v for k, v in lat.items() if k not in ("N", "L", "m")}
    c = cfb200.Context(lat["N"], lat["L"], m=lat["m"], equation=eq, precision=prec, **G.FRW, **kw)
    if Rf is not None:
        c.set_R_fft(Rf, on_device=False)
    if psi is not None:
        c.set_psi(psi, on_device=False)
    return c, x


@golden
@pytest.mark.parametrize("case", ["lambda", "sqrt", "fixed", "approx", "approx_fullband"])
def test_rhs_matches_reference_gpu(case):
    ref = np.load(GOLDEN)[case + "_rhs"]
    c, x = golden_ctx(case)
    dd = torch.empty(x.size, dtype=torch.float64, device="cuda")
    c.rhs(dev(x), dd, G.T)
    assert relmax(dd.cpu().numpy(), ref) <= 1e-12


@golden
@pytest.mark.parametrize("case", ["lambda", "sqrt", "fixed"])
def test_energy_and_step_match_reference_gpu(case):
    g = np.load(GOLDEN)
    c, x = golden_ctx(case)
    st = dev(x)
    rho = torch.empty(x.size // 2, dtype=torch.float64, device="cuda")
    c.energy_density(st, G.T, rho)
    assert relmax(rho.cpu().numpy(), g[case + "_rho"]) <= 1e-12
    c.rk4_steps(st, G.T, G.DT, 1)
    assert relmax(st.cpu().numpy(), g[case + "_step"]) <= 1e-12


@golden
def test_dot_energy_density_matches_reference_gpu():
    g = np.load(GOLDEN)["kgfrw_dot_rho"]
    lat = G.SMALL
    c = cfb200.Context(lat["N"], lat["L"], m=lat["m"], equation=cfb200.EQ_KG_FRW, **G.FRW)
    out = torch.empty(lat["N"] ** 3, dtype=torch.float64, device="cuda")
    c.dot_energy_density(dev(G.state(lat["N"])), G.T, out)
    assert relmax(out.cpu().numpy(), g) <= 1e-12


@pytest.mark.parametrize("prec", [cfb200.FP64, cfb200.FP32_COMP])
@pytest.mark.parametrize("N,nsteps", [(64, 3), (40, 2), (16, 3), (8, 1)])
@pytest.mark.parametrize("eq", [0, 1, 2, 3, 4, 5, 6])
def test_whole_step_pass_equals_paired_passes_bitwise(eq, N, nsteps, prec):
    """The default 7-point route (one whole-step pass per RK4 step) against the paired
    passes (CF_FLAG_PAIR_KERNELS): bit-identical states for every equation, storage
    type, full (N = 64) and ragged (N = 40) tiles, lattices smaller than a tile and odd
    and even step counts."""
    L = 0.9 * N
    out = []
    for flags in (0, cfb200.FLAG_PAIR_KERNELS):
        if eq in EQS:
            c, x, _, _, _ = setup(N, L, eq, prec=prec, flags=flags, seed=23, M=8)
        else:
            x = fields.initial_state(N, L, 0.5, 23)
            x[N ** 3:] = 0.3 * fields.gaussian_field(N, L, 0.5, 24)
            c = cfb200.Context(N, L, m=1.0, equation=eq, precision=prec, flags=flags, **(FRW if eq else {}))
            if eq == 2:
                c.set_R_fft(fields.curvature_R_fft(N, L, 2.0, 1e-2, 2 * np.pi / L * 3, seed=25), on_device=False)
        st = torch.empty(c.info.state_bytes // 8, dtype=torch.float64, device="cuda")
        c.upload(st, x)
        c.rk4_steps(st, 1.0, 0.07, nsteps)
        got = np.empty_like(x)
        c.download(got, st)
        torch.cuda.synchronize()
        out.append(got)
    assert np.array_equal(out[0], out[1])
