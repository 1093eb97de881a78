"""The FFT wrapper (cf_fft_*: the reference's cufftWrapperNoBatching, used through
workspace.fft_wrapper) against numpy's FFT: unnormalised 3-D D2Z / Z2D in FP64,
half-complex layout N x N x (N/2+1), batched D2Z of [phi | dphi], and the padded
in-place Z2D (rows of 2(N/2+1) doubles).  Tolerance 1e-13 relative (FP64 FFT
rounding), through the C ABI."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cfb200  # noqa: E402


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("N", [16, 24, 32])
def test_fft_wrapper_matches_numpy(N):
    rng = np.random.default_rng(N)
    x = rng.standard_normal(2 * N ** 3)
    f = cfb200.FFT(N)
    hc_n = N * N * (N // 2 + 1)
    d_x = torch.from_numpy(x).cuda()
    # execute_d2z
    out = torch.empty(2 * hc_n, dtype=torch.float64, device="cuda")
    f.d2z(d_x, out)
    want = np.fft.rfftn(x[: N ** 3].reshape(N, N, N))
    got = out.cpu().numpy().view(complex).reshape(N, N, N // 2 + 1)
    assert rel(got, want) <= 1e-13
    # execute_batched_d2z
    out2 = torch.empty(4 * hc_n, dtype=torch.float64, device="cuda")
    f.batched_d2z(d_x, out2)
    g2 = out2.cpu().numpy().view(complex).reshape(2, N, N, N // 2 + 1)
    assert rel(g2[0], want) <= 1e-13
    assert rel(g2[1], np.fft.rfftn(x[N ** 3:].reshape(N, N, N))) <= 1e-13
    # execute_z2d: unnormalised inverse, N^3 x
    back = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
    f.z2d(out.clone(), back)
    assert rel(back.cpu().numpy(), x[: N ** 3] * N ** 3) <= 1e-13
    # execute_inplace_z2d: the real field in rows padded to 2(N/2+1)
    buf = out.clone()
    f.inplace_z2d(buf)
    torch.cuda.synchronize()
    pad = buf.cpu().numpy().reshape(N, N, 2 * (N // 2 + 1))[:, :, :N]
    assert rel(pad.ravel(), x[: N ** 3] * N ** 3) <= 1e-13
    f.close()
