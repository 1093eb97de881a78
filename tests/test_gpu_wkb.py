"""WKB continuation (cf_wkb_*): the device path against the restated oracle and the
reference's own src/wkb.cpp (oracle/_ref), and against real RK4 stepping where the
WKB approximation holds.

Tolerances (written per test): against the oracle and the reference build <= 1e-12
of the largest value (the per-s^2 phase tables are the reference's expressions; the
rest is FFT rounding); against RK4 2e-3 norm-wise (the approximation itself: the
continuation leaves out the slowly varying amplitude factor, and the reference says so).
"""
import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cfb200  # noqa: E402
from cfb200 import fields  # noqa: E402

FRW = dict(a1=1.0, H1=0.5, t1=1.0)


def relmax(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


def state(N, L, seed, k_star=0.5):
    x = fields.initial_state(N, L, k_star, seed)
    x[N ** 3:] = 0.3 * fields.gaussian_field(N, L, k_star, seed + 1)
    return x


def wkb_on_device(N, L, x, t_i, ts, m=1.0):
    c = cfb200.Context(N, L, m=m, equation=cfb200.EQ_KG_FRW, **FRW)
    w = cfb200.WKB(c, torch.from_numpy(x).cuda(), t_i)
    outs = []
    for t in ts:
        out = torch.empty(2 * N ** 3, dtype=torch.float64, device="cuda")
        w.evaluate_at(t, out)
        outs.append(out.cpu().numpy())
    w.close()
    return outs


@pytest.mark.parametrize("N", [16, 24, 32])
def test_wkb_matches_oracle(N):
    L = 0.8 * N
    x = state(N, L, 3)
    ts = [5.0, 12.5, 40.0]
    got = wkb_on_device(N, L, x, 4.0, ts)
    P = O.make_params(N, L, 1.0, eq=1, **FRW)
    for t, g in zip(ts, got):
        assert relmax(g, O.wkb(P, x, 4.0, t)) <= 1e-12


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
def test_wkb_matches_reference_build():
    N, L = 16, 12.8
    x = state(N, L, 5)
    got = wkb_on_device(N, L, x, 3.0, [9.0])[0]
    assert relmax(got, O.ref_wkb(N, L, 1.0, x, 3.0, 9.0)) <= 1e-12


def test_wkb_tracks_rk4_where_it_holds():
    """A long-wavelength field (k << m) from t = 20: WKB at t = 40 against 1000 RK4
    steps of the stepping path itself."""
    N, L = 32, 320.0
    x = fields.initial_state(N, L, 0.05, 3)
    got = wkb_on_device(N, L, x, 20.0, [40.0])[0]
    c = cfb200.Context(N, L, m=1.0, equation=cfb200.EQ_KG_FRW, **FRW)
    st = torch.from_numpy(x.copy()).cuda()
    c.rk4_steps(st, 20.0, 0.02, 1000)
    r = st.cpu().numpy()
    assert np.linalg.norm(got - r) / np.linalg.norm(r) <= 2e-3


def test_wkb_rejects_other_cosmologies():
    N, L = 16, 12.8
    x = torch.zeros(2 * N ** 3, dtype=torch.float64, device="cuda")
    c = cfb200.Context(N, L, m=1.0, equation=cfb200.EQ_KG_FRW, a1=1.0, H1=0.5, t1=2.0)
    with pytest.raises(cfb200.CfError, match="radiation"):
        cfb200.WKB(c, x, 3.0)
    c2 = cfb200.Context(N, L, m=1.0, equation=cfb200.EQ_COMOVING_FRW, **FRW)
    with pytest.raises(cfb200.CfError, match="CF_EQ_KG_FRW"):
        cfb200.WKB(c2, x, 3.0)
