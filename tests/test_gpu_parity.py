"""GPU parity: libcfb200.so (called through its C ABI) against the oracle.

Tolerances (written per test): FP64 paths agree with the FP64 oracle to
<= 1e-12 relative (fields, spectra; the stencil sums are ordered like the
reference, so the difference is rounding of a few operations per step);
FP32-compensated paths are compared against the FP64 oracle with the error
budget of FP32 stage storage; mode counts are exact.
"""
import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cfb200  # noqa: E402
from cfb200 import fields  # noqa: E402

FRW = dict(a1=1.0, H1=0.5, t1=1.0)


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def make_inputs(N, L, eq, seed):
    x = fields.initial_state(N, L, 0.5, seed)
    x[N ** 3:] = 0.3 * fields.gaussian_field(N, L, 0.5, seed + 1)  # non-zero dphi exercises every term
    Rf = fields.curvature_R_fft(N, L, eta_start=2.0, psi_rms=1e-2, k_max=0.5 * 2 * np.pi * 8 / L, seed=seed + 2) \
        if eq == 2 else None
    return x, Rf


def ctx_for(N, L, eq, prec=cfb200.FP64, stencil=7, m=1.0):
    cos = FRW if eq else {}
    return cfb200.Context(N, L, m=m, equation=eq, precision=prec, stencil=stencil, **cos)


@pytest.mark.parametrize("stencil", [7, 13])
@pytest.mark.parametrize("eq", [0, 1, 2])
@pytest.mark.parametrize("N", [16, 24, 40])
def test_rhs_matches_oracle(N, eq, stencil):
    L = 0.8 * N
    x, Rf = make_inputs(N, L, eq, 10 + N)
    c = ctx_for(N, L, eq, stencil=stencil)
    if Rf is not None:
        c.set_R_fft(Rf, on_device=False)
    dx, dd = dev(x), torch.empty(2 * N ** 3, dtype=torch.float64, device="cuda")
    t = 1.37
    c.rhs(dx, dd, t)
    got = dd.cpu().numpy()
    P = O.make_params(N, L, 1.0, eq=eq, stencil=stencil, **(FRW if eq else {}))
    want = O.rhs(P, x, t, Rf)
    assert rel(got[: N ** 3], want[: N ** 3]) <= 1e-15
    assert rel(got[N ** 3:], want[N ** 3:]) <= 1e-13


@pytest.mark.parametrize("stencil", [7, 13])
@pytest.mark.parametrize("eq", [0, 1, 2])
def test_rk4_fp64_matches_oracle(eq, stencil):
    N, L, nsteps, dt = 32, 28.0, 12, 0.1
    x, Rf = make_inputs(N, L, eq, 3 + eq)
    t0 = 1.0 if eq else 0.0
    c = ctx_for(N, L, eq, stencil=stencil)
    if Rf is not None:
        c.set_R_fft(Rf, on_device=False)
    d = dev(x)
    c.rk4_steps(d, t0, dt, nsteps)
    got = d.cpu().numpy()
    P = O.make_params(N, L, 1.0, eq=eq, stencil=stencil, **(FRW if eq else {}))
    want = O.rk4_steps(P, x, t0, dt, nsteps, R_fft=Rf)
    assert rel(got[: N ** 3], want[: N ** 3]) <= 1e-12
    assert rel(got[N ** 3:], want[N ** 3:]) <= 1e-12


@pytest.mark.parametrize("prec,tol", [(cfb200.FP64, 1e-13), (cfb200.FP32_COMP, 1e-6)])
@pytest.mark.parametrize("k_max", [1.0, 2.5])
def test_pruned_psi_synthesis_equals_full(prec, tol, k_max):
    """A band-limited R_fft (exact zeros beyond k_max) takes the pruned three-pass
    synthesis when its support box is small (k_max = 1: |i| <= 10 at N = 64) and
    the full 3-D C2R otherwise (k_max = 2.5); the flag CF_FLAG_FULL_PSI_FFT forces
    the full C2R.  Both give the same fields and the same trajectory."""
    N, L = 64, 64.0
    x, _ = make_inputs(N, L, 1, 5)
    Rf = fields.curvature_R_fft(N, L, 2.0, 1e-2, k_max=k_max, seed=8)
    out = []
    for flags in (0, cfb200.FLAG_FULL_PSI_FFT):
        c = cfb200.Context(N, L, m=1.0, equation=2, precision=prec, flags=flags, **FRW)
        c.set_R_fft(Rf, on_device=False)
        st = torch.empty(c.info.state_bytes // 8, dtype=torch.float64, device="cuda")
        c.upload(st, x)
        c.rk4_steps(st, 1.0, 0.05, 6)
        rho = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
        c.energy_density(st, 1.3, rho)
        got = np.empty_like(x)
        c.download(got, st)
        torch.cuda.synchronize()
        out.append((got, rho.cpu().numpy()))
    assert rel(out[0][0], out[1][0]) <= tol
    assert rel(out[0][1], out[1][1]) <= tol


@pytest.mark.parametrize("prec,tol_pf,tol_or", [(cfb200.FP64, 1e-13, (1e-12, 1e-9)), (cfb200.FP32_COMP, 2e-6, (2e-6, 2e-6))])
@pytest.mark.parametrize("N,k_max,route", [(64, 1.0, cfb200.PSI_PRUNED_FUSED),
                                           (64, 1.5, cfb200.PSI_PRUNED_FUSED),   # Kc = N/4 - 1
                                           (128, 0.6, cfb200.PSI_PRUNED_FUSED),
                                           (256, 0.3, cfb200.PSI_PRUNED_FUSED),  # pass-1 band of 2 rows
                                           (256, 0.6, cfb200.PSI_PRUNED_FUSED),  # 4 rows
                                           (96, 1.0, cfb200.PSI_PRUNED),        # not a power of two
                                           (64, 2.5, cfb200.PSI_FULL)])         # box too wide to prune
def test_psi_fields_each_route_matches_full_c2r_and_oracle(prec, tol_pf, tol_or, N, k_max, route):
    """Psi and dPsi/dt at a stage time, read back through cf_psi_fields: the
    route the box selects (pass C as one kernel for power-of-two N, the padded
    cuFFT pass C otherwise, or the full 3-D C2R) equals the forced full C2R
    (FP64 1e-13) and the oracle's FFTW-based synthesis (FP64: Psi 1e-12, dPsi/dt
    1e-9; FP32 storage 2e-6).  The dPsi/dt bound is the conditioning of the
    reference's transfer function: 3x cos x + (x^2 - 3) sin x ~ -x^5/15 at small
    x = k eta / sqrt(3), so a one-ulp difference between two libraries' sincos
    grows by ~5e-15 / x^4 -- about 5e-9 at the fundamental mode of N = 256
    (x ~ 0.03); both GPU routes, which share one sincos, agree to 1e-13."""
    L = float(N)
    Rf = fields.curvature_R_fft(N, L, 2.0, 1e-2, k_max=k_max, seed=31)
    got = {}
    for flags in (0, cfb200.FLAG_FULL_PSI_FFT):
        c = cfb200.Context(N, L, m=1.0, equation=2, precision=prec, flags=flags, **FRW)
        c.set_R_fft(Rf, on_device=False)
        assert c.info.psi_route == (route if flags == 0 else cfb200.PSI_FULL)
        out = torch.empty(2 * N ** 3, dtype=torch.float64, device="cuda")
        c.psi_fields(1.3, out)
        torch.cuda.synchronize()
        got[flags] = out.cpu().numpy()
    P = O.make_params(N, L, 1.0, eq=2, **FRW)
    psi, dpsi = O.psi_fields(P, Rf, 1.3)
    a, b = got[0], got[cfb200.FLAG_FULL_PSI_FFT]
    for sl, want, tol in ((slice(0, N ** 3), psi, tol_or[0]), (slice(N ** 3, None), dpsi, tol_or[1])):
        assert rel(a[sl], b[sl]) <= tol_pf
        assert rel(a[sl], want) <= tol
        assert rel(b[sl], want) <= tol


@pytest.mark.parametrize("route,stencil", [(0, 7), (cfb200.FLAG_PAIR_KERNELS, 7), (0, 13)])
@pytest.mark.parametrize("prec", [cfb200.FP64, cfb200.FP32_COMP])
@pytest.mark.parametrize("N,k_max", [(64, 1.0),    # pruned, passes B and C as own kernels (FP32)
                                     (96, 1.0),    # pruned, cuFFT pass C
                                     (64, 2.5)])   # full 3-D C2R
def test_psi_side_stream_equals_serial(prec, N, k_max, route, stencil):
    """By default cf_rk4_steps synthesises the next step's Psi slots on a side
    stream while the current step runs (six slots); CF_FLAG_PSI_SERIAL synthesises
    each step's slots before its passes on the caller's stream.  Same slots, same
    kernels: bit-identical states for the whole-step and the paired route, over one
    step, over several (dt = 0.05 from t = 1, where t + dt and the next step's start
    differ in the last bit at some steps), and over calls that continue from cached
    slots, two of them at such a step.  At those steps the FP32 pruned synthesis compares the new time's pass-A
    inputs with the latest refresh's and takes its slot when they are identical
    (CF_FLAG_PSI_NO_REUSE synthesises every time): the same bits again, with fewer
    refreshes."""
    L = float(N)
    x, _ = make_inputs(N, L, 1, 41)
    Rf = fields.curvature_R_fft(N, L, 2.0, 1e-2, k_max=k_max, seed=43)
    got, stats = {}, {}
    for flags in (route, route | cfb200.FLAG_PSI_SERIAL, route | cfb200.FLAG_PSI_NO_REUSE):
        c = cfb200.Context(N, L, m=1.0, equation=2, precision=prec, stencil=stencil, flags=flags, **FRW)
        c.set_R_fft(Rf, on_device=False)
        st = torch.empty(c.info.state_bytes // 8, dtype=torch.float64, device="cuda")
        c.upload(st, x)
        outs = []
        # steps 3 and 8 start a few ulp from the previous step's end: there the check
        # runs at a call's first step, before its pass is enqueued
        for step0, n in ((0, 1), (1, 2), (3, 5), (8, 2)):
            c.rk4_steps(st, 1.0, 0.05, n, step0=step0)
            rho = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
            # the last stage time, t + dt of the call's last step: a cached slot (the end
            # time t0 + (step0 + n) dt itself would be synthesised here at steps 3 and 8)
            c.energy_density(st, 1.0 + 0.05 * (step0 + n - 1) + 0.05, rho)
            outs.append((st.clone(), rho))
        got[flags] = outs
        stats[flags] = c.psi_stats()
        c.close()
    for other in (route | cfb200.FLAG_PSI_SERIAL, route | cfb200.FLAG_PSI_NO_REUSE):
        for (a, ra), (b, rb) in zip(got[route], got[other]):
            assert torch.equal(a, b)
            assert torch.equal(ra, rb)
    (r0, u0), (r1, u1) = stats[route], stats[route | cfb200.FLAG_PSI_NO_REUSE]
    assert u1 == 0 and stats[route | cfb200.FLAG_PSI_SERIAL][1] == 0
    assert r0 + u0 == r1
    if prec == cfb200.FP32_COMP and k_max < 2.0:  # the pruned synthesis
        assert u0 >= 1
    else:
        assert u0 == 0


def test_psi_reuse_at_benchmark_shape_is_bit_identical():
    """N = 256, FP32 storage, whole-step route, 20 steps of dt = 0.05 from t = 1 in
    one call: seven steps start a few ulp from the previous step's t + dt.  With
    the default reuse the states equal those with every slot synthesised, and
    those seven times take the previous refresh's slot (or a few fewer, where a
    pass-A input rounds differently)."""
    N, L = 256, 256.0
    x, _ = make_inputs(N, L, 1, 47)
    Rf = fields.curvature_R_fft(N, L, 2.0, 1e-2, k_max=0.5, seed=49, use_torch=True)
    got, stats = {}, {}
    for flags in (0, cfb200.FLAG_PSI_NO_REUSE):
        c = cfb200.Context(N, L, m=1.0, equation=2, precision=cfb200.FP32_COMP, flags=flags, **FRW)
        c.set_R_fft(Rf, on_device=True)
        st = torch.empty(c.info.state_bytes // 8, dtype=torch.float64, device="cuda")
        c.upload(st, x)
        c.rk4_steps(st, 1.0, 0.05, 20)
        torch.cuda.synchronize()
        got[flags] = st
        stats[flags] = c.psi_stats()
        c.close()
    assert torch.equal(got[0], got[cfb200.FLAG_PSI_NO_REUSE])
    (r0, u0), (r1, u1) = stats[0], stats[cfb200.FLAG_PSI_NO_REUSE]
    assert (r1, u1) == (48, 0)
    assert r0 + u0 == 48 and 5 <= u0 <= 7


@pytest.mark.parametrize("N,k_max", [(256, 0.3), (256, 0.6), (512, 0.5), (1024, 0.5)])
def test_warp_pass_c_equals_cta_pass_c(N, k_max):
    """FP32 storage, N = 256, 512, 1024: the last pass of the pruned synthesis as
    one warp per row group taking its band tiles by TMA (the default up to N = 512),
    the same with per-lane cp.async copies (CF_FLAG_PSI_NO_TMA; the default at
    N = 1024), and one CTA per tile
    (CF_FLAG_PSI_CTA_PASS_C) do the same arithmetic in the same order, so Psi and
    dPsi/dt are bit-identical."""
    L = float(N)
    Rf = fields.curvature_R_fft(N, L, 2.0, 1e-2, k_max=k_max, seed=37, use_torch=True)
    got = {}
    for flags in (0, cfb200.FLAG_PSI_NO_TMA, cfb200.FLAG_PSI_CTA_PASS_C):
        c = cfb200.Context(N, L, m=1.0, equation=2, precision=cfb200.FP32_COMP, flags=flags, **FRW)
        c.set_R_fft(Rf, on_device=True)
        assert c.info.psi_route == cfb200.PSI_PRUNED_FUSED
        out = torch.empty(2 * N ** 3, dtype=torch.float64, device="cuda")
        c.psi_fields(1.3, out)
        torch.cuda.synchronize()
        got[flags] = out
        c.close()
    assert torch.equal(got[0], got[cfb200.FLAG_PSI_CTA_PASS_C])
    assert torch.equal(got[0], got[cfb200.FLAG_PSI_NO_TMA])
    del got
    torch.cuda.empty_cache()


def test_pass_c_copy_wait_timeout_is_reported_and_recoverable():
    """Failure detection without a GPU fault: pass C's band-copy barriers are armed
    for 16 bytes more than each TMA box delivers, so every bounded wait runs out
    (the copies themselves land).  The warps set the context's error word and leave;
    the next refresh returns CF_ERR_TIMEOUT and drops every cached slot; with the
    hook reset the same context gives Psi bit-identical to a fresh context's, at the
    failed refresh's time too."""
    N, L = 256, 256.0
    Rf = fields.curvature_R_fft(N, L, 2.0, 1e-2, k_max=0.5, seed=41, use_torch=True)
    out = torch.empty(2, 2 * N ** 3, dtype=torch.float64, device="cuda")
    want = torch.empty_like(out)
    c = cfb200.Context(N, L, m=1.0, equation=2, precision=cfb200.FP32_COMP, **FRW)
    c.set_R_fft(Rf, on_device=True)
    assert c.info.psi_route == cfb200.PSI_PRUNED_FUSED
    c.psi_fields(1.1, out[0])  # builds the pruned route and its tensor map
    c.psi_set_wait_test(16, spin_limit=1 << 12)
    c.psi_fields(1.2, out[0])
    torch.cuda.synchronize()
    with pytest.raises(cfb200.CfError) as e:
        c.psi_fields(1.3, out[1])
    assert e.value.code == -6
    c.psi_set_wait_test(0)
    c.psi_fields(1.2, out[0])
    c.psi_fields(1.3, out[1])
    torch.cuda.synchronize()
    c.close()
    f = cfb200.Context(N, L, m=1.0, equation=2, precision=cfb200.FP32_COMP, **FRW)
    f.set_R_fft(Rf, on_device=True)
    f.psi_fields(1.2, want[0])
    f.psi_fields(1.3, want[1])
    torch.cuda.synchronize()
    f.close()
    assert torch.equal(out, want)


@pytest.mark.parametrize("N,K,prec,tol", [(512, 41, cfb200.FP32_COMP, 2e-6), (1024, 40, cfb200.FP32_COMP, 2e-6),
                                          (512, 41, cfb200.FP64, 1e-12)])
def test_pruned_psi_at_full_size_equals_full_c2r(N, K, prec, tol):
    """The benchmark's sizes, R_fft band-limited to a box of |i|, |j|, k <= K: the
    pruned route against the forced full 3-D C2R, compared on the device as a
    fraction of the largest value.  FP32 storage: pass B and pass C each as one
    kernel (pass B split 32 x 16 at N = 512 and 32 x 32 at N = 1024), 2e-6 (FP32
    rounding of two FFT orderings).  FP64 storage: pass C as the persistent
    kernel (16 x 16 at N = 512), 1e-12."""
    L = float(N)
    g = torch.Generator(device="cuda")
    g.manual_seed(17)
    hc = torch.fft.rfftn(torch.randn((N, N, N), generator=g, device="cuda", dtype=torch.float64))
    i = torch.arange(N, device="cuda")
    far = torch.minimum(i, N - i) > K
    hc[far] = 0
    hc[:, far] = 0
    hc[:, :, K + 1:] = 0
    Rf = torch.view_as_real(hc * (1e-2 / N ** 1.5)).reshape(-1).contiguous()
    del hc
    got = {}
    for flags in (0, cfb200.FLAG_FULL_PSI_FFT):
        c = cfb200.Context(N, L, m=1.0, equation=2, precision=prec, flags=flags, **FRW)
        c.set_R_fft(Rf, on_device=True)
        assert c.info.psi_route == (cfb200.PSI_PRUNED_FUSED if flags == 0 else cfb200.PSI_FULL)
        out = torch.empty(2 * N ** 3, dtype=torch.float64, device="cuda")
        c.psi_fields(1.3, out)
        torch.cuda.synchronize()
        got[flags] = out
        c.close()
        torch.cuda.empty_cache()
    a, b = got[0], got[cfb200.FLAG_FULL_PSI_FFT]
    for sl in (slice(0, N ** 3), slice(N ** 3, None)):
        err = float((a[sl] - b[sl]).abs().max() / b[sl].abs().max())
        assert err <= tol, err


@pytest.mark.parametrize("prec", [cfb200.FP64, cfb200.FP32_COMP])
@pytest.mark.parametrize("eq", [0, 1, 2])
@pytest.mark.parametrize("stencil", [7, 13])
@pytest.mark.parametrize("N,nsteps", [(32, 5), (40, 4)])
def test_paired_stage_passes_equal_single_stage_passes(prec, eq, stencil, N, nsteps):
    """cf_rk4_steps' default route (stages 1+2 and 3+4 fused, the new phi
    alternating between two planes) equals the four single-stage passes
    (CF_FLAG_STAGE_KERNELS) bit for bit: same roundings, same expressions.  N = 40
    leaves partial tiles; an odd step count ends with phi in the scratch plane."""
    L = float(N)
    x, Rf = make_inputs(N, L, eq, 41)
    t0 = 1.0 if eq else 0.0
    out = []
    for flags in (0, cfb200.FLAG_STAGE_KERNELS):
        cos = FRW if eq else {}
        c = cfb200.Context(N, L, m=1.0, equation=eq, precision=prec, stencil=stencil, flags=flags, **cos)
        if Rf is not None:
            c.set_R_fft(Rf, on_device=False)
        st = torch.empty(c.info.state_bytes // 8, dtype=torch.float64, device="cuda")
        c.upload(st, x)
        c.rk4_steps(st, t0, 0.05, nsteps)
        got = np.empty_like(x)
        c.download(got, st)
        torch.cuda.synchronize()
        out.append(got)
    assert np.array_equal(out[0], out[1]), np.abs(out[0] - out[1]).max()


@pytest.mark.parametrize("eq", [0, 1, 2])
def test_rk4_split_calls_equal_one_call(eq):
    """step0 offsets reproduce integrate_const's direct time t0 + step*dt."""
    N, L, dt = 16, 16.0, 0.05
    x, Rf = make_inputs(N, L, eq, 21)
    t0 = 1.0 if eq else 0.0
    c = ctx_for(N, L, eq)
    if Rf is not None:
        c.set_R_fft(Rf, on_device=False)
    a, b = dev(x), dev(x)
    c.rk4_steps(a, t0, dt, 10)
    c.rk4_steps(b, t0, dt, 4)
    c.rk4_steps(b, t0, dt, 6, step0=4)
    assert torch.equal(a, b)


@pytest.mark.parametrize("eq", [1, 2])
def test_rk4_fp32_comp_error_budget(eq):
    """FP32 hi+lo state, FP32 stage buffers and stage arithmetic, FP64 compensated
    state update: after 40 steps the fields stay within 2e-6 (relative,
    norm-wise) of the FP64 oracle, and the density spectrum within 1e-5."""
    N, L, nsteps, dt = 32, 32.0, 40, 0.05
    x, Rf = make_inputs(N, L, eq, 40 + eq)
    c = ctx_for(N, L, eq, prec=cfb200.FP32_COMP)
    if Rf is not None:
        c.set_R_fft(Rf, on_device=False)
    st = torch.empty(c.info.state_bytes // 8, dtype=torch.float64, device="cuda")
    c.upload(st, x)
    c.rk4_steps(st, 1.0, dt, nsteps)
    got = np.empty(2 * N ** 3)
    c.download(got, st)
    torch.cuda.synchronize()
    P = O.make_params(N, L, 1.0, eq=eq, **FRW)
    want = O.rk4_steps(P, x, 1.0, dt, nsteps, R_fft=Rf)
    assert rel(got[: N ** 3], want[: N ** 3]) <= 2e-6
    assert rel(got[N ** 3:], want[N ** 3:]) <= 2e-6
    t_end = 1.0 + nsteps * dt
    spec = torch.empty(O.n_s2(N), dtype=torch.float64, device="cuda")
    c.density_spectrum_s2(st, t_end, spec)
    want_s = O.power_spectrum(O.energy_density(P, want, t_end, Rf))
    assert rel(spec.cpu().numpy(), want_s) <= 1e-5


def test_fp32_comp_state_roundtrip_is_exact_to_fp48():
    N, L = 16, 16.0
    x, _ = make_inputs(N, L, 1, 77)
    c = ctx_for(N, L, 1, prec=cfb200.FP32_COMP)
    st = torch.empty(c.info.state_bytes // 8, dtype=torch.float64, device="cuda")
    c.upload(st, x)
    back = np.empty_like(x)
    c.download(back, st)
    torch.cuda.synchronize()
    assert np.abs(back - x).max() <= 2.0 ** -46 * np.abs(x).max()


@pytest.mark.parametrize("eq", [0, 1, 2])
@pytest.mark.parametrize("prec", [cfb200.FP64, cfb200.FP32_COMP])
def test_energy_density_matches_oracle(eq, prec):
    N, L = 24, 20.0
    x, Rf = make_inputs(N, L, eq, 55)
    c = ctx_for(N, L, eq, prec=prec)
    if Rf is not None:
        c.set_R_fft(Rf, on_device=False)
    st = torch.empty(c.info.state_bytes // 8, dtype=torch.float64, device="cuda")
    c.upload(st, x)
    rho = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
    t = 2.5
    c.energy_density(st, t, rho)
    P = O.make_params(N, L, 1.0, eq=eq, **(FRW if eq else {}))
    xs = x
    if prec == cfb200.FP32_COMP:  # the oracle sees the same (hi+lo) state
        xs = np.empty_like(x)
        c.download(xs, st)
        torch.cuda.synchronize()
    want = O.energy_density(P, xs, t, Rf)
    tol = 1e-13 if (prec == cfb200.FP64 or eq != 2) else 1e-7  # FP32 Psi in the coupled FP32 mode
    assert rel(rho.cpu().numpy(), want) <= tol


@pytest.mark.parametrize("N", [8, 16, 24, 48])
def test_power_spectrum_s2_matches_oracle_and_reference(N):
    L = float(N)
    f = fields.gaussian_field(N, L, 0.7, 100 + N) ** 2  # a density-like positive field
    c = ctx_for(N, L, 1)
    out = torch.empty(O.n_s2(N), dtype=torch.float64, device="cuda")
    c.power_spectrum_s2(dev(f), out)
    got = out.cpu().numpy()
    want = O.power_spectrum(f)
    big = np.abs(want) >= 1e-10 * np.abs(want).max()
    assert np.max(np.abs(got - want)[big] / np.abs(want)[big]) <= 1e-12
    if O.ref_available():
        assert rel(got, O.ref_power_spectrum(f)) <= 1e-12


@pytest.mark.parametrize("eq,prec", [(1, cfb200.FP64), (1, cfb200.FP32_COMP), (2, cfb200.FP32_COMP)])
def test_density_spectrum_equals_power_spectrum_of_energy_density(eq, prec):
    """The density spectrum takes its fixed-point scale from the energy pass (a Parseval
    bound) instead of a max pass: per bin it is the power spectrum of the energy density
    to the fixed-point resolution, and the shells regroup its own bins."""
    N, L = 48, 38.4
    x, Rf = make_inputs(N, L, eq, 21)
    c = ctx_for(N, L, eq, prec)
    if Rf is not None:
        c.set_R_fft(Rf, on_device=False)
    st = torch.empty(c.info.state_bytes // 8, dtype=torch.float64, device="cuda")
    c.upload(st, x)
    t = 2.5
    rho = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
    c.energy_density(st, t, rho)
    a = torch.empty(O.n_s2(N), dtype=torch.float64, device="cuda")
    b = torch.empty_like(a)
    c.power_spectrum_s2(rho, a)
    c.density_spectrum_s2(st, t, b)
    sh = torch.empty(O.n_shells(N), dtype=torch.float64, device="cuda")
    c.s2_to_shells(sh, None)
    A, B = a.cpu().numpy(), b.cpu().numpy()
    # both are truncations of the same FP64 mode values; a value loses less than one
    # fixed-point unit, 2^-125 of the scale bound: (largest mode value) x (HC entries)
    # for the power spectrum, N^5 x (largest row sum of rho^2) for the density spectrum;
    # the conversion of a bin's 128-bit sum back to FP64 rounds (< 2 ulp)
    counts = torch.empty(O.n_s2(N), dtype=torch.int64, device="cuda")
    c.s2_counts(counts)
    r = rho.cpu().numpy().reshape(N * N, N)
    bound_a = A.max() * N * N * (N // 2 + 1)
    bound_b = float(N) ** 5 * (r * r).sum(axis=1).max()
    tol = counts.cpu().numpy() * 2.0 ** -125 * (bound_a + bound_b) + 4 * np.finfo(float).eps * A
    bad = np.nonzero(np.abs(A - B) > tol)[0]
    assert bad.size == 0, [(int(s), A[s], B[s], tol[s]) for s in bad[:8]]
    big = A >= 1e-6 * A.max()
    assert np.max(np.abs(A - B)[big] / A[big]) <= 1e-15
    want_sh, _ = O.shells_from_s2(N, B)
    assert np.max(np.abs(sh.cpu().numpy() - want_sh) / np.maximum(want_sh, 1e-300)) <= 1e-15


def test_mode_power_spectrum_matches_oracle():
    N, L, m, a_t = 32, 25.6, 1.3, 1.7
    x, _ = make_inputs(N, L, 1, 9)
    c = cfb200.Context(N, L, m=m, equation=1, **FRW)
    out = torch.empty(O.n_s2(N), dtype=torch.float64, device="cuda")
    c.mode_power_spectrum_s2(dev(x), a_t, out)
    want = O.mode_power_spectrum(N, L, m, a_t, x)
    got = out.cpu().numpy()
    # norm-wise 1e-13; per bin 1e-11 over bins >= 1e-10 of the maximum (the
    # smallest bins carry the FFT rounding of the largest modes)
    assert rel(got, want) <= 1e-13
    big = np.abs(want) >= 1e-10 * np.abs(want).max()
    assert np.max(np.abs(got - want)[big] / np.abs(want)[big]) <= 1e-11


def test_spectrum_is_bit_reproducible_and_shells_are_exact():
    N, L = 32, 32.0
    x, _ = make_inputs(N, L, 1, 12)
    c = ctx_for(N, L, 1)
    d = dev(x)
    s1 = torch.empty(O.n_s2(N), dtype=torch.float64, device="cuda")
    s2 = torch.empty_like(s1)
    c.density_spectrum_s2(d, 1.5, s1)
    sh = torch.empty(O.n_shells(N), dtype=torch.float64, device="cuda")
    cnt = torch.empty(O.n_shells(N), dtype=torch.int64, device="cuda")
    c.s2_to_shells(sh, cnt)
    c.density_spectrum_s2(d, 1.5, s2)
    assert torch.equal(s1, s2)  # bit-identical: order-independent integer sums
    want_sh, want_cnt = O.shells_from_s2(N, s1.cpu().numpy())
    assert np.array_equal(cnt.cpu().numpy(), want_cnt)
    assert np.max(np.abs(sh.cpu().numpy() - want_sh) / np.maximum(np.abs(want_sh), 1e-300)) <= 1e-15
    counts = torch.empty(O.n_s2(N), dtype=torch.int64, device="cuda")
    c.s2_counts(counts)
    assert np.array_equal(counts.cpu().numpy(), O.s2_counts(N))


def test_scale_sum_matches_numpy():
    N = 16
    c = ctx_for(N, 16.0, 1)
    rng = np.random.default_rng(0)
    n = 2 * N ** 3
    ins = [rng.standard_normal(n) for _ in range(5)]
    al = [1.0, 0.05 / 6, 0.05 / 3, 0.05 / 3, 0.05 / 6]
    dins = [dev(v) for v in ins]
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    c.scale_sum(out, dins, al, n)
    want = al[0] * ins[0] + al[1] * ins[1] + al[2] * ins[2] + al[3] * ins[3] + al[4] * ins[4]
    assert np.abs(out.cpu().numpy() - want).max() <= 1e-15 * np.abs(want).max()


def test_plain_odeint_path_equals_fused_stepper():
    """cf_rhs + cf_scale_sum composed as runge_kutta4_classic does
    (stepper/runge_kutta4_classic.hpp:88-138) equals the fused cf_rk4_steps."""
    N, L, dt, t = 16, 16.0, 0.1, 1.3
    x, _ = make_inputs(N, L, 1, 31)
    c = ctx_for(N, L, 1)
    n = 2 * N ** 3
    X = dev(x)
    k = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(4)]
    y = torch.empty(n, dtype=torch.float64, device="cuda")
    c.rhs(X, k[0], t)
    c.scale_sum(y, [X, k[0]], [1.0, dt / 2], n)
    c.rhs(y, k[1], t + dt / 2)
    c.scale_sum(y, [X, k[1]], [1.0, dt / 2], n)
    c.rhs(y, k[2], t + dt / 2)
    c.scale_sum(y, [X, k[2]], [1.0, dt], n)
    c.rhs(y, k[3], t + dt)
    c.scale_sum(X, [X] + k, [1.0, dt / 6, dt / 3, dt / 3, dt / 6], n)
    F = dev(x)
    c.rk4_steps(F, t, dt, 1)
    assert rel(X.cpu().numpy(), F.cpu().numpy()) <= 1e-15


def test_check_finite_reports_planted_nan():
    N, L = 16, 16.0
    x, _ = make_inputs(N, L, 1, 2)
    x[1234] = np.nan  # planted on the host
    c = ctx_for(N, L, 1)
    code, bad = c.check_finite(dev(x))
    assert code == -5 and bad == 1
    x[1234] = 0.0
    assert c.check_finite(dev(x)) == (0, 0)


def test_config0_observer_run_matches_reference():
    """Config 0 (flat KG, N=64, L=64, m=1, dt=0.1, 100 steps, spectra every
    unit time): the GPU stepper + observers reproduce the reference's own CPU run
    (oracle/_ref, its ConstIntervalObserver files) within 1e-12."""
    if not O.ref_available():
        pytest.skip("reference build not present")
    N, L, m, dt = 64, 64.0, 1.0, 0.1
    x = fields.initial_state(N, L, 0.5, 0)
    final_ref, obs = O.ref_integrate(0, N, L, m, x, 0.0, 10.05, dt, t_interval=0.999, observe=True)
    c = cfb200.Context(N, L, m=m, equation=0)
    d = dev(x)
    spec = torch.empty(O.n_s2(N), dtype=torch.float64, device="cuda")
    step = 0
    for i, t_save in enumerate(obs["t_list"]):
        target = int(round(t_save / dt))
        c.rk4_steps(d, 0.0, dt, target - step, step0=step)
        step = target
        c.mode_power_spectrum_s2(d, 1.0, spec)
        assert rel(spec.cpu().numpy(), obs["varphi_plus"][i]) <= 1e-12
        c.density_spectrum_s2(d, t_save, spec)
        assert rel(spec.cpu().numpy(), obs["rho"][i]) <= 1e-12
    assert rel(d.cpu().numpy(), final_ref) <= 1e-12


def test_linearity_at_full_size_n256():
    """KG-FRW is linear in the state, so one RK4 step commutes with linear
    combinations up to rounding: step(x + 2y) = step(x) + 2 step(y).  Checked at
    the N=256 configuration size, where the oracle is too slow to run."""
    N, L = 256, 256.0
    c = ctx_for(N, L, 1)
    x = fields.initial_state(N, L, 0.25, 1, use_torch=True)
    y = fields.initial_state(N, L, 0.25, 2, use_torch=True)
    z = x + 2 * y
    for s in (x, y, z):
        c.rk4_steps(s, 1.0, 0.05, 3)
    assert float(torch.linalg.norm(z - (x + 2 * y)) / torch.linalg.norm(z)) <= 1e-14


@pytest.mark.parametrize("eq,prec", [(1, cfb200.FP64), (2, cfb200.FP32_COMP)])
def test_density_slices_match_energy_density(eq, prec):
    """cf_density_slices: the a = 0 slice and the mean over a of the energy density
    (the observer's rho_slice / rho_axis_average, src/observer.hpp:110-119)."""
    N, L = 24, 20.0
    x, Rf = make_inputs(N, L, eq, 71)
    c = ctx_for(N, L, eq, prec=prec)
    if Rf is not None:
        c.set_R_fft(Rf, on_device=False)
    st = torch.empty(c.info.state_bytes // 8, dtype=torch.float64, device="cuda")
    c.upload(st, x)
    rho = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
    c.energy_density(st, 1.3, rho)
    sl = torch.empty(N * N, dtype=torch.float64, device="cuda")
    av = torch.empty(N * N, dtype=torch.float64, device="cuda")
    c.density_slices(st, 1.3, sl, av)
    r = rho.cpu().numpy()
    assert np.array_equal(sl.cpu().numpy(), r[: N * N])
    want = np.zeros(N * N)
    for a in range(N):  # the summation order of the kernel: increasing a
        want += r[a * N * N:(a + 1) * N * N]
    assert np.array_equal(av.cpu().numpy(), want / N)


@pytest.mark.parametrize("stencil,order", [(7, 2), (13, 4)])
def test_gpu_laplacian_convergence_order_on_a_plane_wave(stencil, order):
    """The device stencils' own convergence order (the oracle twin is in
    test_oracle_pin.py): cf_rhs (FP64, flat KG, m = 0) on cos(2 pi (a + 2b + 3c) / N)
    with L fixed approaches -(2 pi / L)^2 14 phi as h^2 (7-point) and h^4 (13-point)."""
    L = 8.0
    errs = []
    for N in (16, 32, 64):
        i = np.arange(N)
        A, Bb, Cc = np.meshgrid(i, i, i, indexing="ij")
        phi = np.cos(2 * np.pi * (A + 2 * Bb + 3 * Cc) / N).ravel()
        x = dev(np.concatenate([phi, np.zeros(N ** 3)]))
        c = ctx_for(N, L, 0, stencil=stencil, m=0.0)
        out = torch.empty_like(x)
        c.rhs(x, out, 0.0)
        torch.cuda.synchronize()
        lap = out[N ** 3:].cpu().numpy()
        exact = -(2 * np.pi / L) ** 2 * 14.0 * phi
        errs.append(float(np.abs(lap - exact).max() / np.abs(exact).max()))
        c.close()
    rates = [np.log2(errs[k] / errs[k + 1]) for k in range(2)]
    assert all(abs(r - order) < 0.15 for r in rates), (errs, rates)
