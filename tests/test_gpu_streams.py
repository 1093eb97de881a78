"""Two streams on one context: a state upload on a copy stream into one device
state, while RK4 steps run on another stream over a second state.

cf_state_upload touches only its stream-ordered staging buffer and the target
state, so overlapping it with cf_rk4_steps (as a caller that double-buffers its
inputs does) must leave both results bit-identical to running them one after
the other.  Each case is checked against that serial order on the same inputs.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cfb200  # noqa: E402
from cfb200 import fields  # noqa: E402

FRW = dict(a1=1.0, H1=0.5, t1=1.0)


def _inputs(N, L, seed):
    x = fields.initial_state(N, L, 0.5, seed)
    x[N ** 3:] = 0.3 * fields.gaussian_field(N, L, 0.5, seed + 1)
    Rf = fields.curvature_R_fft(N, L, eta_start=2.0, psi_rms=1e-2, k_max=0.5 * 2 * np.pi * 8 / L, seed=seed + 2)
    return x, Rf


@pytest.mark.parametrize("prec", [cfb200.FP64, cfb200.FP32_COMP])
def test_upload_on_copy_stream_overlapping_steps(prec):
    N, L, steps, dt = 48, 38.4, 12, 0.05
    xa, Rf = _inputs(N, L, 71)
    xb, _ = _inputs(N, L, 91)
    c = cfb200.Context(N, L, m=1.0, equation=2, precision=prec, **FRW)
    c.set_R_fft(Rf, on_device=False)
    words = c.info.state_bytes // 8
    ha = torch.from_numpy(xa).pin_memory()
    hb = torch.from_numpy(xb).pin_memory()

    # serial order: upload A, step A, upload B, step B
    sa = torch.empty(words, dtype=torch.float64, device="cuda")
    sb = torch.empty(words, dtype=torch.float64, device="cuda")
    c.upload(sa, ha.data_ptr())
    c.rk4_steps(sa, 1.0, dt, steps)
    c.upload(sb, hb.data_ptr())
    c.rk4_steps(sb, 1.0, dt, steps, step0=steps)
    want_a, want_b = np.empty_like(xa), np.empty_like(xb)
    c.download(want_a, sa)
    c.download(want_b, sb)
    torch.cuda.synchronize()

    # overlapped: B's upload on a copy stream while A steps on the compute stream
    compute = torch.cuda.current_stream()
    copy = torch.cuda.Stream()
    ta = torch.full_like(sa, float("nan"))
    tb = torch.full_like(sb, float("nan"))
    torch.cuda.synchronize()
    c.upload(ta, ha.data_ptr(), stream=compute)
    c.rk4_steps(ta, 1.0, dt, steps, stream=compute)
    c.upload(tb, hb.data_ptr(), stream=copy)
    done = torch.cuda.Event()
    done.record(copy)
    compute.wait_event(done)
    c.rk4_steps(tb, 1.0, dt, steps, step0=steps, stream=compute)
    got_a, got_b = np.empty_like(xa), np.empty_like(xb)
    c.download(got_a, ta)
    c.download(got_b, tb)
    torch.cuda.synchronize()
    c.close()
    assert np.array_equal(got_a, want_a)
    assert np.array_equal(got_b, want_b)
    assert np.all(np.isfinite(got_b))
