"""Initial conditions on the device, mirroring the reference's initializers.

The reference builds its initial fields on the host before stepping
(src/initializer.hpp:33-301, src/random_field.cpp:36-134, src/fdm3d.cpp:76-102).
Here the transforms and per-mode products run on the GPU through the C ABI
(cf_white_noise, cf_grf, cf_scale_modes); the spectra stay host callables, as in
the reference, and are evaluated once per s^2 (a mode's |k| depends only on s^2).

Noise: the reference draws N^3 deviates per field from one std::mt19937 +
std::normal_distribution stream (src/random_field.cpp:13-33).  `noise` below is
either an int seed -- device deviates from cf_white_noise, fields after fields
along one counter stream -- or a CUDA tensor of deviates supplied by the caller
(for example the reference's own stream drawn on the host), consumed N^3 per field
in the reference's order.
"""
from __future__ import annotations

import math

import numpy as np


# ---- spectra (src/random_field.cpp:92-134) -----------------------------------

def power_law_with_cutoff_given_amplitude_3d(N, L, sigma, k_ast, alpha):
    pi = math.pi
    assert alpha >= -3.0 and k_ast * L / (2 * pi) > 1.0
    if alpha == -3.0:
        P_k_ast = 2 * pi * pi * sigma * sigma / (k_ast * k_ast * k_ast * math.log(k_ast * L / (2 * pi)))
    else:
        P_k_ast = (3 + alpha) * 2 * pi * pi * sigma * sigma * (L * L * L * (k_ast * L) ** alpha) / \
            ((k_ast * L) ** (alpha + 3) - (2 * pi) ** (alpha + 3))
    P_k_ast *= (N / L) * (N / L) * (N / L)
    return lambda k: 0.0 if k == 0.0 else (P_k_ast * ((k / k_ast) ** alpha if k <= k_ast else 0.0))


def scale_invariant_spectrum_3d(N, L, A_s):
    pi = math.pi
    k0 = 1.0
    P_k0 = A_s / ((k0 * k0 * k0) / (2 * pi * pi))
    P_k0 *= (N / L) * (N / L) * (N / L)
    return lambda k: 0.0 if k == 0.0 else (P_k0 * (k / k0) ** -3)


def to_deriv_spectrum(m, P_f, a=None):
    if a is None:
        return lambda k: (k * k + m * m) * P_f(k)
    return lambda k: (k * k / (a * a) + m * m) * P_f(k)


def n_s2(N):
    return 3 * (N // 2) ** 2 + 1


def sqrtP_table(N, L, P):
    """sqrt(P(|k|)) per s^2, |k| = sqrt(s^2) * 2 * pi / L as the GRF forms it
    (src/random_field.cpp:67-68)."""
    return np.array([math.sqrt(P(math.sqrt(s2) * 2 * math.pi / L)) for s2 in range(n_s2(N))])


def kernel_table(N, L, kernel):
    """kernel(|k|) / N^3 per s^2, |k| = sqrt(s^2) * (2 pi / L) as
    compute_field_with_scaled_fourier_modes forms it (src/fdm3d.cpp:94)."""
    return np.array([kernel(math.sqrt(s2) * (2 * math.pi / L)) / (N * N * N) for s2 in range(n_s2(N))])


# ---- fields -------------------------------------------------------------------

class _Noise:
    """The deviates of successive fields: a device counter stream or a given tensor."""

    def __init__(self, ctx, noise, N3):
        self.ctx, self.noise, self.N3, self.pos = ctx, noise, N3, 0

    def next(self, buf):
        if isinstance(self.noise, int):
            self.ctx.white_noise(buf, self.noise, offset=self.pos, n=self.N3)
        else:
            buf.copy_(self.noise[self.pos:self.pos + self.N3])
        self.pos += self.N3
        return buf


def gaussian_random_field(ctx, noise_src, P, Psi=None, psi_scale=1.0, out=None):
    """generate_(inhomogeneous_)gaussian_random_field on the device (N^3 CUDA float64)."""
    import torch
    N = ctx.N
    out = torch.empty(N ** 3, dtype=torch.float64, device="cuda") if out is None else out
    noise_src.next(out)
    ctx.grf(out, sqrtP_table(N, ctx.params.L, P), out, d_psi=Psi, psi_scale=psi_scale if Psi is not None else 0.0)
    return out


def perturbed_grf_and_comoving_curvature_fft(ctx, t_start, Psi_std_dev, varphi_std_dev, k_ast, noise):
    """The initializer of the reference driver (src/initializer.hpp:150-206) on the device.

    Returns (state [phi | dphi] as an N^3 x 2 CUDA float64 tensor, R_fft as an HC CUDA
    float64 tensor), for the context's N, L, m, a1, H1, t1 and p.  `noise`: seed (int)
    or a CUDA tensor of at least 3 N^3 deviates.
    """
    import torch
    from scipy.special import sici

    p = ctx.params
    N, L, m = ctx.N, p.L, p.m
    pi = math.pi
    eta_i = (p.p / (p.a1 * p.H1)) * (1 + (1 + 1 / p.p) * p.H1 * (t_start - p.t1)) ** (1 / (1 + p.p))
    x = (4 * pi * eta_i) / (math.sqrt(3) * L)
    A_s = (-576 * pi ** 6 * eta_i ** 6 * Psi_std_dev ** 2) / (
        -81 * L ** 4 * (L ** 2 + 2 * pi ** 2 * eta_i ** 2)
        + L * (81 * L ** 5 - 54 * L ** 3 * pi ** 2 * eta_i ** 2 + 48 * L * pi ** 4 * eta_i ** 4) * math.cos(x)
        + 256 * pi ** 6 * eta_i ** 6 * sici(x)[1]
        + 4 * math.sqrt(3) * L * pi * eta_i * (27 * L ** 4 + 6 * L ** 2 * pi ** 2 * eta_i ** 2 - 16 * pi ** 4 * eta_i ** 4)
        * math.sin(x))
    src = _Noise(ctx, noise, N ** 3)
    R = gaussian_random_field(ctx, src, scale_invariant_spectrum_3d(N, L, A_s))

    def kernel(k):
        if k == 0.0:
            return 0.0
        return (6 * math.sqrt(3) * (-((k * eta_i * math.cos((k * eta_i) / math.sqrt(3))) / math.sqrt(3))
                                    + math.sin((k * eta_i) / math.sqrt(3)))) / (k ** 3 * eta_i ** 3)

    Psi = torch.empty_like(R)
    ctx.scale_modes(R, kernel_table(N, L, kernel), Psi)
    v = k_ast / (p.a1 * m)
    alpha_phi = 0.5 * (-3 * (4 * v ** 2 + 5) ** 2) / (12 * v ** 4 + 50 * v ** 2 + 50)
    alpha_dphi = 0.5 * (25 - 20 * v ** 2) / (12 * v ** 4 + 50 * v ** 2 + 50)
    P_f = power_law_with_cutoff_given_amplitude_3d(N, L, varphi_std_dev, k_ast, 0)
    P_dtf = to_deriv_spectrum(m, P_f)
    state = torch.empty(2 * N ** 3, dtype=torch.float64, device="cuda")
    gaussian_random_field(ctx, src, P_f, Psi, alpha_phi, out=state[: N ** 3])
    gaussian_random_field(ctx, src, P_dtf, Psi, alpha_dphi, out=state[N ** 3:])
    from . import FFT
    R_fft = torch.empty(2 * N * N * (N // 2 + 1), dtype=torch.float64, device="cuda")
    FFT(N).d2z(R, R_fft)  # workspace.R_fft = fft_wrapper.execute_d2z(R)
    return state, R_fft
