"""Ensembles of uneven-N FRW Klein-Gordon lattices (config 3 of the benchmark
set, at reduced sizes), through the C ABI.

Every member runs the same fused stage code as the single-lattice stepper with
the same coefficient arithmetic, so each schedule (one persistent cooperative
kernel with grid barriers, the batched passes over the work list -- one
whole-step launch per step for the 7-point stencil, two paired passes for the
13-point one --, the same passes per member, the captured graph) must reproduce
the single-lattice cf_rk4_steps result bit for bit, and the FP64 members match
the oracle.
"""
import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cfb200  # noqa: E402
from cfb200 import fields  # noqa: E402

FRW = dict(a1=1.0, H1=0.5, t1=1.0)


def members_spec(precision, Ns=(16, 24, 32, 16, 40), stencil=7):
    rng = np.random.default_rng(7)
    out = []
    for i, N in enumerate(Ns):
        out.append(dict(N=N, L=float(N), m=float(rng.uniform(0.5, 2.0)), equation=cfb200.EQ_KG_FRW,
                        precision=precision, stencil=stencil, **FRW))
    return out


def initial(d, i):
    x = fields.initial_state(d["N"], d["L"], 0.5, 1000 + i)
    x[d["N"] ** 3:] = 0.1 * fields.gaussian_field(d["N"], d["L"], 0.5, 2000 + i)
    return x


def single_run(d, x, t0, dt, nsteps):
    c = cfb200.Context(d["N"], d["L"], m=d["m"], equation=cfb200.EQ_KG_FRW, precision=d["precision"],
                       stencil=d["stencil"], **FRW)
    st = torch.empty(c.info.state_bytes // 8, dtype=torch.float64, device="cuda")
    c.upload(st, x)
    c.rk4_steps(st, t0, dt, nsteps)
    out = np.empty_like(x)
    c.download(out, st)
    torch.cuda.synchronize()
    return out, c, st


@pytest.mark.parametrize("precision", [cfb200.FP64, cfb200.FP32_COMP])
@pytest.mark.parametrize("mode", [cfb200.ENS_PERSISTENT, cfb200.ENS_BATCHED, cfb200.ENS_LOOP])
def test_ensemble_modes_equal_single_lattice_runs(precision, mode):
    spec = members_spec(precision)
    ens = cfb200.Ensemble(spec)
    xs = [initial(d, i) for i, d in enumerate(spec)]
    for i, x in enumerate(xs):
        ens.upload(i, x)
    t0, dt, n = 1.0, 0.1, 7
    ens.rk4_steps(t0, dt, 3, step0=0, mode=mode)
    ens.rk4_steps(t0, dt, n - 3, step0=3, mode=mode)
    torch.cuda.synchronize()
    for i, d in enumerate(spec):
        got = np.empty_like(xs[i])
        ens.download(i, got)
        want, _, _ = single_run(d, xs[i], t0, dt, n)
        assert np.array_equal(got, want), (i, np.abs(got - want).max())


def test_ensemble_fp64_member_matches_oracle():
    spec = members_spec(cfb200.FP64, Ns=(24, 16))
    ens = cfb200.Ensemble(spec)
    xs = [initial(d, i) for i, d in enumerate(spec)]
    for i, x in enumerate(xs):
        ens.upload(i, x)
    ens.rk4_steps(1.0, 0.1, 10)
    for i, d in enumerate(spec):
        got = np.empty_like(xs[i])
        ens.download(i, got)
        P = O.make_params(d["N"], d["L"], d["m"], eq=1, **FRW)
        want = O.rk4_steps(P, xs[i], 1.0, 0.1, 10)
        assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want)


@pytest.mark.parametrize("mode", [cfb200.ENS_PERSISTENT, cfb200.ENS_BATCHED])
@pytest.mark.parametrize("stencil", [7, 13])
def test_ensemble_graph_run_and_spectra(stencil, mode):
    spec = members_spec(cfb200.FP32_COMP, stencil=stencil)
    ens = cfb200.Ensemble(spec)
    xs = [initial(d, i) for i, d in enumerate(spec)]
    for i, x in enumerate(xs):
        ens.upload(i, x)
    t0, dt, S, nseg = 1.0, 0.1, 5, 3
    out = torch.zeros(nseg * ens.spectra_total, dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        ens.run_graph(t0, dt, S, nseg, out, stream=stream, mode=mode)
    stream.synchronize()
    out = out.cpu().numpy()
    for i, d in enumerate(spec):
        got = np.empty_like(xs[i])
        ens.download(i, got)
        want, c, st = single_run(d, xs[i], t0, dt, S * nseg)
        assert np.array_equal(got, want)
        spec_single = torch.empty(O.n_s2(d["N"]), dtype=torch.float64, device="cuda")
        c.density_spectrum_s2(st, t0 + S * nseg * dt, spec_single)
        seg = out[(nseg - 1) * ens.spectra_total + ens.offsets[i]:][: O.n_s2(d["N"])]
        ref = spec_single.cpu().numpy()
        # batched vs single cuFFT plans may round differently: 1e-12
        assert np.linalg.norm(seg - ref) <= 1e-12 * np.linalg.norm(ref)


def test_ensemble_autotune_keeps_results():
    spec = members_spec(cfb200.FP64, Ns=(32, 24))
    ens = cfb200.Ensemble(spec)
    shape, chunk = ens.autotune(1.0, 0.1, steps=1)
    assert shape in (0, 1) and chunk in (8, 16, 32, 64)
    xs = [initial(d, i) for i, d in enumerate(spec)]
    for i, x in enumerate(xs):
        ens.upload(i, x)
    ens.rk4_steps(1.0, 0.1, 4)
    for i, d in enumerate(spec):
        got = np.empty_like(xs[i])
        ens.download(i, got)
        want, _, _ = single_run(d, xs[i], 1.0, 0.1, 4)
        assert np.array_equal(got, want)


def test_persistent_barrier_timeout_is_reported_and_recoverable():
    """Failure detection without a GPU fault: the grid barrier is made to wait for
    one CTA that never arrives, with a short spin limit.  The bounded wait gives
    up, the call returns CF_ERR_TIMEOUT, the state is untouched, and the same
    ensemble then runs normally."""
    spec = members_spec(cfb200.FP64, Ns=(16, 24))
    ens = cfb200.Ensemble(spec)
    xs = [initial(d, i) for i, d in enumerate(spec)]
    for i, x in enumerate(xs):
        ens.upload(i, x)
    ens.set_barrier_test(1, spin_limit=1 << 16)
    with pytest.raises(cfb200.CfError) as e:
        ens.rk4_steps(1.0, 0.1, 2, mode=cfb200.ENS_PERSISTENT)
    assert e.value.code == -6
    for i, x in enumerate(xs):
        got = np.empty_like(x)
        ens.download(i, got)
        assert np.array_equal(got, x)
    ens.set_barrier_test(0)
    ens.rk4_steps(1.0, 0.1, 3, mode=cfb200.ENS_PERSISTENT)
    for i, d in enumerate(spec):
        got = np.empty_like(xs[i])
        ens.download(i, got)
        want, _, _ = single_run(d, xs[i], 1.0, 0.1, 3)
        assert np.array_equal(got, want)


def test_checkpoint_resume_matches_uninterrupted_run():
    """Checkpoint/resume: stepping 6, downloading the state to the host, loading
    it into a fresh context and stepping 6 more equals 12 uninterrupted steps
    (bit for bit unless a value sits on an FP32 rounding tie when the FP64
    checkpoint is split back into hi + lo; 1e-13 relative covers that)."""
    d = members_spec(cfb200.FP32_COMP, Ns=(32,))[0]
    x = initial(d, 0)
    full, _, _ = single_run(d, x, 1.0, 0.1, 12)
    half, _, _ = single_run(d, x, 1.0, 0.1, 6)
    c = cfb200.Context(d["N"], d["L"], m=d["m"], equation=cfb200.EQ_KG_FRW, precision=d["precision"], **FRW)
    st = torch.empty(c.info.state_bytes // 8, dtype=torch.float64, device="cuda")
    c.upload(st, half)
    c.rk4_steps(st, 1.0, 0.1, 6, step0=6)
    got = np.empty_like(x)
    c.download(got, st)
    torch.cuda.synchronize()
    assert np.linalg.norm(got - full) <= 1e-13 * np.linalg.norm(full)


def test_ensemble_rejects_mixed_settings():
    spec = members_spec(cfb200.FP64, Ns=(16, 24))
    spec[1]["precision"] = cfb200.FP32_COMP
    with pytest.raises(cfb200.CfError):
        cfb200.Ensemble(spec)
