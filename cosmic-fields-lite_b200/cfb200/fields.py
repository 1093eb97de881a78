"""Seeded synthetic initial data with the shapes of the benchmark configurations.

The reference builds its initial fields on the host (src/random_field.cpp:36-83,
src/initializer.hpp:33-206): white noise / N^3, r2c, multiply by sqrt(P(|k|)),
unnormalised c2r, so that <phi^2> = sum_k P(k) / N^3.  The same construction is
used here with numpy (or torch on the GPU for large N, where numpy is slow);
initial conditions are not part of the accelerated path.

* gaussian_field: P(k) = A exp(-k^2 / (2 k*^2)), P(0) = 0, A set so <phi^2> = 1
  (the "GRF with k*" of the configurations).
* curvature_R_fft: R with P_R(k) = A_R k^-3 for 0 < k <= k_max, A_R set so that
  Psi(t_start) = T(k eta/sqrt3) R has expected rms psi_rms, returned as the HC
  array R_fft = r2c(R) (the reference's workspace.R_fft).
"""
from __future__ import annotations

import numpy as np


def _kgrid_half(N, L):
    k1 = np.fft.fftfreq(N, d=1.0 / N) * (2 * np.pi / L)
    kz = np.arange(N // 2 + 1) * (2 * np.pi / L)
    return np.sqrt(k1[:, None, None] ** 2 + k1[None, :, None] ** 2 + kz[None, None, :] ** 2)


def _mult_half(N):
    """Number of full-grid modes each half-complex entry stands for."""
    w = np.full(N // 2 + 1, 2.0)
    w[0] = 1.0
    w[N // 2] = 1.0
    return w[None, None, :]


def gaussian_spectrum_amplitude(N, L, k_star):
    k = _kgrid_half(N, L)
    P = np.exp(-k ** 2 / (2 * k_star ** 2))
    P[0, 0, 0] = 0.0
    return N ** 3 / float((P * _mult_half(N)).sum())


def _grf_from_sqrtP(N, sqrtP, rng, use_torch=False):
    if use_torch:
        import torch
        g = torch.Generator(device="cuda")
        g.manual_seed(int(rng.integers(1 << 62)))
        w = torch.randn((N, N, N), generator=g, device="cuda", dtype=torch.float64) / N ** 3
        hk = torch.fft.rfftn(w) * torch.from_numpy(sqrtP).to("cuda")
        return (torch.fft.irfftn(hk, s=(N, N, N)) * N ** 3).reshape(-1)
    w = rng.standard_normal((N, N, N)) / N ** 3
    hk = np.fft.rfftn(w) * sqrtP
    return np.fft.irfftn(hk, s=(N, N, N), axes=(0, 1, 2)).ravel() * N ** 3


def gaussian_field(N, L, k_star, seed, use_torch=False):
    """phi with <phi^2> = 1 and Gaussian spectrum of width k_star; returns numpy
    (or a CUDA float64 tensor with use_torch)."""
    k = _kgrid_half(N, L)
    A = gaussian_spectrum_amplitude(N, L, k_star)
    P = A * np.exp(-k ** 2 / (2 * k_star ** 2))
    P[0, 0, 0] = 0.0
    return _grf_from_sqrtP(N, np.sqrt(P), np.random.default_rng(seed), use_torch)


def initial_state(N, L, k_star, seed, use_torch=False):
    """[phi | dphi] with phi a Gaussian random field (<phi^2> = 1) and dphi = 0."""
    phi = gaussian_field(N, L, k_star, seed, use_torch)
    if use_torch:
        import torch
        return torch.cat([phi, torch.zeros_like(phi)])
    return np.concatenate([phi, np.zeros_like(phi)])


def white_noise_hc(N, seed):
    """xi = r2c(w / N^3) of seeded white noise w (the first two steps of the
    reference GRF, src/random_field.cpp:36-56), as an HC float64 array."""
    w = np.random.default_rng(seed).standard_normal((N, N, N)) / N ** 3
    return np.ascontiguousarray(np.fft.rfftn(w)).view(np.float64).ravel()


def gaussian_sqrtP_by_s2(N, L, k_star):
    """sqrt(P(k)) tabulated by s^2 = i^2+j^2+k^2 for the Gaussian spectrum of
    gaussian_field (P(0) = 0, <phi^2> = 1): c2r(sqrtP * xi) is that field."""
    A = gaussian_spectrum_amplitude(N, L, k_star)
    s2 = np.arange(3 * (N // 2) ** 2 + 1, dtype=np.float64)
    k2 = s2 * (2 * np.pi / L) ** 2
    P = A * np.exp(-k2 / (2 * k_star ** 2))
    P[0] = 0.0
    return np.sqrt(P)


def transfer_psi(x):
    """Psi_k / R_k at x = k eta / sqrt(3): 2 (sin x - x cos x) / x^3
    (src/equations.cpp:141-183 without the 1/N^3 of the unnormalised c2r)."""
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    nz = x != 0
    xx = x[nz]
    out[nz] = 2 * (np.sin(xx) - xx * np.cos(xx)) / xx ** 3
    return out


def curvature_R_fft(N, L, eta_start, psi_rms, k_max, seed, use_torch=False):
    """HC array R_fft (2N^2(N/2+1) doubles) of a scale-invariant R (alpha = -3)
    with a sharp cutoff at k_max, normalised so that Psi at conformal time
    eta_start has expected rms psi_rms."""
    k = _kgrid_half(N, L)
    shape = np.zeros_like(k)
    m = (k > 0) & (k <= k_max)
    shape[m] = k[m] ** -3.0
    T = transfer_psi(k * eta_start / np.sqrt(3.0))
    var1 = float((shape * T ** 2 * _mult_half(N)).sum()) / N ** 3
    A = psi_rms ** 2 / var1 if var1 > 0 else 0.0
    # The reference's R_fft = r2c(c2r(sqrtP r2c(w / N^3))) equals sqrtP r2c(w) up to
    # rounding; building it directly keeps the modes beyond k_max exactly zero.
    sqrtP = np.sqrt(A * shape)
    rng = np.random.default_rng(seed)
    if use_torch:
        import torch
        g = torch.Generator(device="cuda")
        g.manual_seed(int(rng.integers(1 << 62)))
        w = torch.randn((N, N, N), generator=g, device="cuda", dtype=torch.float64)
        hc = torch.fft.rfftn(w) * torch.from_numpy(sqrtP).to("cuda")
        return torch.view_as_real(hc).reshape(-1).contiguous()
    hc = np.fft.rfftn(rng.standard_normal((N, N, N))) * sqrtP
    return np.ascontiguousarray(hc).view(np.float64).ravel()
