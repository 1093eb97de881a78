"""cf_rk4_steps_noalloc: the RK4 stepper for callers that must not allocate
device memory (applications that hand all device memory to their own pool, or
loops that cannot take cudaMalloc's synchronisation or failure mid-run).  Its
three RK4 work buffers live in a fixed 24 MiB array inside the library instead
of context allocations.

Checked through the C ABI against the allocating entry point cf_rk4_steps on
the same inputs: two calls in a row (the second continuing the first), both
precisions, both stencils, flat and FRW equations.  The routes differ -- the
no-allocation entry point runs the four single-stage kernels, cf_rk4_steps the
whole-step pass (7-point) or the paired passes (13-point) -- but every route forms
and rounds each value identically, so the states must be bit-identical.  A call
with nsteps = 0 is accepted and changes nothing.  Sizes beyond the array and the
comoving-curvature equation are rejected with a clear error.  This file is
collected last.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cfb200  # noqa: E402
from cfb200 import fields  # noqa: E402

FRW = dict(a1=1.0, H1=0.5, t1=1.0)


def _noalloc():
    f = cfb200.lib().cf_rk4_steps_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int64,
                  ctypes.c_int64, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _run_noalloc(ctx, st, t0, dt, nsteps, step0):
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return _noalloc()(ctx.h, ctypes.c_void_p(st.data_ptr()), t0, dt, step0, nsteps, stream)


def _rel(a, b):
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


@pytest.mark.parametrize("stencil", [7, 13])
@pytest.mark.parametrize("eq", [cfb200.EQ_KG, cfb200.EQ_KG_FRW])
@pytest.mark.parametrize("prec,N", [(cfb200.FP64, 64), (cfb200.FP64, 80), (cfb200.FP32_COMP, 96)])
def test_noalloc_matches_allocating_stepper_on_two_calls(eq, prec, N, stencil):
    L = float(N)
    cos = FRW if eq == cfb200.EQ_KG_FRW else {}
    ctx = cfb200.Context(N, L, m=1.0, equation=eq, precision=prec, stencil=stencil, **cos)
    x = fields.initial_state(N, L, 0.5, seed=N + eq)
    a = torch.empty(ctx.info.state_bytes // 8, dtype=torch.float64, device="cuda")
    ctx.upload(a, x)
    b = a.clone()
    t0, dt = (1.0 if cos else 0.0), 0.05
    # a zero-step call reserves the array and resolves its address, nothing else
    assert _run_noalloc(ctx, b, t0, dt, 0, 0) == cfb200.CF_OK, cfb200.lib().cf_last_error()
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    for call, (step0, n) in enumerate([(0, 4), (4, 3)]):
        ctx.rk4_steps(a, t0, dt, n, step0=step0)
        assert _run_noalloc(ctx, b, t0, dt, n, step0) == cfb200.CF_OK, cfb200.lib().cf_last_error()
        torch.cuda.synchronize()
        assert torch.equal(a, b), (call, _rel(b, a))
    ctx.close()


def test_noalloc_rejects_lattices_beyond_the_array():
    ctx = cfb200.Context(128, 128.0, m=1.0, equation=cfb200.EQ_KG_FRW, precision=cfb200.FP64, **FRW)
    st = torch.zeros(ctx.info.state_bytes // 8, dtype=torch.float64, device="cuda")
    assert _run_noalloc(ctx, st, 1.0, 0.05, 1, 0) == -1
    assert b"fixed array" in cfb200.lib().cf_last_error()
    ctx.close()


def test_noalloc_rejects_the_comoving_equation():
    ctx = cfb200.Context(32, 32.0, m=1.0, equation=cfb200.EQ_COMOVING_FRW, precision=cfb200.FP64, **FRW)
    st = torch.zeros(ctx.info.state_bytes // 8, dtype=torch.float64, device="cuda")
    assert _run_noalloc(ctx, st, 1.0, 0.05, 1, 0) == -7
    ctx.close()
