"""Adjoint gradients of the shell-spectrum log loss (config 4 of the benchmark
set: FRW Klein-Gordon, initial field parameterised by shell-group amplitudes
theta, and the mass m), checked against central finite differences and across
precisions.

    phi0 = c2r(sqrt(theta_g(k)) sqrtP(|k|) xi_k),  dphi0 = 0
    x_T  = RK4^n(x0)  (t0 = 1, a = t^1/2)
    L    = sum_s (log P_rho,s(x_T) - log P_target,s)^2

The torch.autograd.Function below is test-harness glue only: forward and
backward both call the C ABI (cf_adjoint_*, cf_field_from_shell_amplitudes,
cf_shell_amplitude_gradient).
"""
import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cfb200  # noqa: E402
from cfb200 import fields  # noqa: E402

FRW = dict(a1=1.0, H1=0.5, t1=1.0)


class Problem:
    def __init__(self, N, L, nsteps, every, ngroups=32, k_star=0.25, seed=11, dt=0.05, t0=1.0):
        self.N, self.L, self.nsteps, self.every, self.dt, self.t0 = N, L, nsteps, every, dt, t0
        self.xi = torch.from_numpy(fields.white_noise_hc(N, seed)).cuda()
        self.sqrtP = torch.from_numpy(fields.gaussian_sqrtP_by_s2(N, L, k_star)).cuda()
        self.nshells = O.n_shells(N)
        self.spg = -(-self.nshells // ngroups)
        self.ngroups = ngroups

    def run(self, theta, m, precision=cfb200.FP64, target=None, stencil=7, grad=False, floor=0.0):
        """Loss (and gradients w.r.t. theta and m) through the C ABI; shells whose
        target power is below floor * max(target) are left out of the loss."""
        N = self.N
        ctx = cfb200.Context(N, self.L, m=m, equation=cfb200.EQ_KG_FRW, precision=precision, stencil=stencil, **FRW)
        phi = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
        cfb200.field_from_shell_amplitudes(ctx, self.xi, self.sqrtP, theta, self.spg, phi)
        x0 = torch.cat([phi, torch.zeros_like(phi)])
        st = torch.empty(ctx.info.state_bytes // 8, dtype=torch.float64, device="cuda")
        ctx.import_f64(st, x0)
        adj = cfb200.Adjoint(ctx, self.nsteps, self.every)
        adj.forward(st, self.t0, self.dt)
        if target is None:
            out = np.empty(self.nshells)
            sh = torch.empty(self.nshells, dtype=torch.float64, device="cuda")
            s2 = torch.empty(ctx.info.s2_bins, dtype=torch.float64, device="cuda")
            ctx.density_spectrum_s2(st, self.t0 + self.nsteps * self.dt, s2)
            ctx.s2_to_shells(sh)
            out[:] = sh.cpu().numpy()
            adj.close()
            return out
        loss = adj.shell_log_loss(st, target, floor)
        if not grad:
            adj.close()
            return loss
        lam0 = torch.empty(2 * N ** 3, dtype=torch.float64, device="cuda")
        dm = adj.backward(lam0)
        gth = cfb200.shell_amplitude_gradient(ctx, lam0[: N ** 3], self.xi, self.sqrtP, theta, self.spg)
        adj.close()
        return loss, gth, dm


class SpectrumLoss(torch.autograd.Function):
    """theta (ngroups), m (scalar) -> L, with the adjoint as backward."""

    @staticmethod
    def forward(ctxf, theta, m, prob, target, precision):
        loss, gth, dm = prob.run(theta.detach().cpu().numpy(), float(m), precision, target, grad=True)
        ctxf.save_for_backward(torch.from_numpy(gth), torch.tensor(dm, dtype=torch.float64))
        return torch.tensor(loss, dtype=torch.float64)

    @staticmethod
    def backward(ctxf, gout):
        gth, dm = ctxf.saved_tensors
        return gout * gth, gout * dm, None, None, None


@pytest.fixture(scope="module")
def small():
    prob = Problem(32, 32.0, nsteps=40, every=10, ngroups=8, k_star=0.5)
    theta0 = np.ones(prob.ngroups)
    target = prob.run(theta0, 1.1)
    return prob, target


def _fd(prob, target, theta, m, which, h=1e-4):
    if which == "m":
        return (prob.run(theta, m + h, target=target) - prob.run(theta, m - h, target=target)) / (2 * h)
    tp, tm = theta.copy(), theta.copy()
    tp[which] += h
    tm[which] -= h
    return (prob.run(tp, m, target=target) - prob.run(tm, m, target=target)) / (2 * h)


def test_adjoint_matches_central_differences_fp64(small):
    prob, target = small
    theta = np.linspace(0.8, 1.3, prob.ngroups)
    m = 1.0
    loss, gth, dm = prob.run(theta, m, target=target, grad=True)
    assert loss > 0
    scale = max(np.abs(gth).max(), abs(dm))
    for j in range(prob.ngroups):
        fd = _fd(prob, target, theta, m, j)
        assert abs(gth[j] - fd) <= 1e-5 * scale + 1e-6 * abs(fd), (j, gth[j], fd)
    fd = _fd(prob, target, theta, m, "m")
    assert abs(dm - fd) <= 1e-5 * abs(fd), (dm, fd)


def test_adjoint_13_point_stencil(small):
    prob, target = small
    theta = np.linspace(1.2, 0.9, prob.ngroups)
    loss, gth, dm = prob.run(theta, 1.05, target=target, grad=True, stencil=13)
    h = 1e-4

    def L(m):
        return prob.run(theta, m, target=target, stencil=13)

    fd = (L(1.05 + h) - L(1.05 - h)) / (2 * h)
    assert abs(dm - fd) <= 1e-5 * abs(fd)


def test_adjoint_fp32_comp_agrees_with_fp64(small):
    """FP32 hi+lo state storage adds rounding noise near 1e-15 of the peak
    density power; over the shells within 6 decades of the peak the loss and
    its gradients agree with the FP64 run to 1e-3."""
    prob, target = small
    theta = np.linspace(0.9, 1.1, prob.ngroups)
    l64, g64, m64 = prob.run(theta, 1.0, cfb200.FP64, target=target, grad=True, floor=1e-6)
    l32, g32, m32 = prob.run(theta, 1.0, cfb200.FP32_COMP, target=target, grad=True, floor=1e-6)
    assert abs(l32 - l64) <= 1e-3 * abs(l64)
    assert np.abs(g32 - g64).max() <= 1e-3 * np.abs(g64).max()
    assert abs(m32 - m64) <= 1e-3 * abs(m64)


def test_autograd_function_roundtrip(small):
    prob, target = small
    theta = torch.full((prob.ngroups,), 1.05, dtype=torch.float64, requires_grad=True)
    m = torch.tensor(0.97, dtype=torch.float64, requires_grad=True)
    L = SpectrumLoss.apply(theta, m, prob, target, cfb200.FP64)
    L.backward()
    loss, gth, dm = prob.run(theta.detach().numpy(), 0.97, target=target, grad=True)
    assert np.allclose(theta.grad.numpy(), gth, rtol=0, atol=0)
    assert float(m.grad) == dm


def test_loss_matches_oracle_small():
    """The forward loss through the C ABI equals the oracle's (restated RK4,
    energy density, spectrum, shells) on the same initial field."""
    prob = Problem(16, 16.0, nsteps=10, every=5, ngroups=4, k_star=0.5)
    theta = np.array([1.0, 0.7, 1.3, 1.1])
    target = prob.run(np.ones(4), 1.2)
    loss = prob.run(theta, 1.0, target=target)
    ctx = cfb200.Context(16, 16.0, m=1.0, equation=1, **FRW)
    phi = torch.empty(16 ** 3, dtype=torch.float64, device="cuda")
    cfb200.field_from_shell_amplitudes(ctx, prob.xi, prob.sqrtP, theta, prob.spg, phi)
    x0 = np.concatenate([phi.cpu().numpy(), np.zeros(16 ** 3)])
    P = O.make_params(16, 16.0, 1.0, eq=1, **FRW)
    xT = O.rk4_steps(P, x0, 1.0, 0.05, 10)
    rho = O.energy_density(P, xT, 1.5)
    sh, _ = O.shells_from_s2(16, O.power_spectrum(rho))
    ok = (sh > 0) & (target > 0)
    want = float(np.sum((np.log(sh[ok]) - np.log(target[ok])) ** 2))
    assert abs(loss - want) <= 1e-10 * abs(want)


def test_config4_full_size_gradient_n256():
    """Config 4 at full size: N = 256, L = 256, 200 RK4 steps (dt = 0.05),
    checkpoints every 20 steps, 32 shell-group amplitudes + m, target from the
    m = 1.1 run.  At k* = 0.25 the highest density shells lie ~50 decades below
    the peak, i.e. at the FP64 rounding floor, where log P is noise; the loss
    keeps the shells within 12 decades of the peak.  Adjoint vs central
    differences (h = 1e-4) on m and on three shell groups in FP64, and the
    FP32-comp adjoint vs the FP64 adjoint over the shells within 6 decades."""
    prob = Problem(256, 256.0, nsteps=200, every=20, ngroups=32, k_star=0.25)
    theta = np.ones(prob.ngroups)
    target = prob.run(theta, 1.1)
    floor = 1e-12

    def fd(which, h=1e-4):
        if which == "m":
            return (prob.run(theta, 1.0 + h, target=target, floor=floor) -
                    prob.run(theta, 1.0 - h, target=target, floor=floor)) / (2 * h)
        tp, tm = theta.copy(), theta.copy()
        tp[which] += h
        tm[which] -= h
        return (prob.run(tp, 1.0, target=target, floor=floor) - prob.run(tm, 1.0, target=target, floor=floor)) / (2 * h)

    loss, gth, dm = prob.run(theta, 1.0, target=target, grad=True, floor=floor)
    scale = np.abs(gth).max()
    for j in (0, 1, 3):
        f = fd(j)
        assert abs(gth[j] - f) <= 1e-5 * scale, (j, gth[j], f)
    f = fd("m")
    assert abs(dm - f) <= 1e-5 * abs(f), (dm, f)
    l64, g64, m64 = prob.run(theta, 1.0, target=target, grad=True, floor=1e-6)
    l32, g32, m32 = prob.run(theta, 1.0, cfb200.FP32_COMP, target=target, grad=True, floor=1e-6)
    assert np.abs(g32 - g64).max() <= 1e-3 * np.abs(g64).max()
    assert abs(m32 - m64) <= 1e-3 * abs(m64)
