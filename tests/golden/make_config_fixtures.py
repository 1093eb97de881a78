#!/usr/bin/env python
"""Golden fixtures of the benchmark configurations at their stated sizes.

Test infrastructure: the fixtures are made by the reference's OWN CPU build
(oracle/_ref/libcfref.so -- src/equations.cpp + Eigen + Boost.odeint
runge_kutta4_classic + integrate_const + ConstIntervalObserver, FFTs through the
FFTW3 restatement of oracle/fftw_shim.c) and cross-checked against the C
restatement (oracle/liboracle.so); both figures are stored in the file.

    python tests/golden/make_config_fixtures.py config1
        -> tests/golden/config1_kgfrw_n256.npz (with the reference's own -ffast-math /
           strict-FP spread as floor_* entries; `config1-floor` adds only those)
    python tests/golden/make_config_fixtures.py config2
        -> tests/golden/config2_comoving_n512.npz

config1: KleinGordonEquationInFRW, radiation era (a1 = 1, H1 = 0.5, t1 = 1, so
  a = t^1/2), N = 256, L = 256, m = 1.  phi(0) = fields.initial_state(256, 256,
  k* = 0.25, seed = 1) (numpy), dphi(0) = 0.  RK4 dt = 0.05 from t = 1 for 1000
  steps (t_end = t0 + 1000.5 dt, so that integrate_const takes exactly 1000
  steps), observer every dt_save = 5 (src/observer.hpp:87-125).  Stored: the
  observer's save times and steps, the unit-shell sums of both saved spectra
  (varphi_plus = mode power spectrum, rho = density power spectrum) at every
  save, both full s^2 spectra and the a = 0 planes of phi and dphi after 1000
  steps, and sum / sum of squares of the initial state (so a test can
  check that it regenerated the same input).
config2: ComovingCurvatureEquationInFRW (src/equations.cpp:186-261), same
  cosmology, N = 512, L = 512, m = 1.  phi(0) = fields.initial_state(512, 512,
  0.25, seed = 2), dphi(0) = 0; R_fft = fields.curvature_R_fft(512, 512, eta(1) =
  2, psi_rms = 1e-2, k_max = 0.5, seed = 3) (the k^-3 spectrum with cutoff).
  RK4 dt = 0.05 from t = 1 for 3 steps.  Stored: the density power spectrum (s^2
  bins and unit shells) and the mode power spectrum (unit shells) at t = 1.15, the
  first 64 rows of the a = 0 planes of phi and dphi, input checksums.

The reference build must exist (make -C oracle ref REF=<reference tree>).
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "cosmic-fields-lite_b200")]

import oracle as O  # noqa: E402
from cfb200 import fields  # noqa: E402

FRW = dict(a1=1.0, H1=0.5, t1=1.0)


def checksum(x):
    return np.array([x.sum(), (x * x).sum()])


def shells(N, s2):
    return O.shells_from_s2(N, s2)[0]


def rel_max(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def config1(out):
    N, L, m, dt, t0, nsteps, every = 256, 256.0, 1.0, 0.05, 1.0, 1000, 100
    x0 = fields.initial_state(N, L, 0.25, seed=1)
    t_end = t0 + (nsteps + 0.5) * dt
    t = time.time()
    xr, sp = O.ref_integrate(1, N, L, m, x0, t0, t_end, dt, t_interval=every * dt, observe=True, **FRW)
    print(f"reference build: {time.time() - t:.0f} s, {len(sp['t_list'])} saves", flush=True)
    tl = sp["t_list"]
    steps = np.rint((tl - t0) / dt).astype(np.int64)
    # the restatement along the same save steps
    P = O.make_params(N, L, m, eq=1, **FRW)
    y = x0.copy()
    done = 0
    rest_rho, rest_phi = [], []
    t = time.time()
    for s, ts in zip(steps, tl):
        y = O.rk4_steps(P, y, t0, dt, int(s - done), step0=done)
        done = int(s)
        rest_rho.append(O.power_spectrum(O.energy_density(P, y, ts)))
        rest_phi.append(O.mode_power_spectrum(N, L, m, O.a_of_t(P, ts), y))
    print(f"restatement: {time.time() - t:.0f} s", flush=True)
    cross = max(max(rel_max(a, b) for a, b in zip(rest_rho, sp["rho"])),
                max(rel_max(a, b) for a, b in zip(rest_phi, sp["varphi_plus"])),
                rel_max(y, xr))
    print(f"restatement vs reference build: {cross:.3e}", flush=True)
    # both spectra of the state after exactly nsteps steps (the last save may come earlier)
    t1 = t0 + nsteps * dt
    rho_final = O.ref_power_spectrum(O.ref_energy_density(1, N, L, m, xr, t1, **FRW))
    mode_final = O.ref_mode_power_spectrum(N, L, m, O.a_of_t(P, t1), xr)
    N2 = N * N
    np.savez(out, N=N, L=L, m=m, dt=dt, t0=t0, nsteps=nsteps, k_star=0.25, seed=1, t_final=t1,
             rho_s2_final=rho_final, varphi_plus_s2_final=mode_final,
             input_checksum=checksum(x0), t_list=tl, steps=steps,
             rho_shells=np.array([shells(N, s) for s in sp["rho"]]),
             varphi_plus_shells=np.array([shells(N, s) for s in sp["varphi_plus"]]),
             phi_plane0=xr[:N2], dphi_plane0=xr[N ** 3:N ** 3 + N2],
             restatement_vs_reference=cross)


def config2(out):
    N, L, m, dt, t0, nsteps = 512, 512.0, 1.0, 0.05, 1.0, 3
    x0 = fields.initial_state(N, L, 0.25, seed=2)
    eta0 = 2.0 * t0 ** 0.5
    Rf = fields.curvature_R_fft(N, L, eta0, 1e-2, 0.5, seed=3)
    t_end = t0 + (nsteps + 0.5) * dt
    t1 = t0 + nsteps * dt
    t = time.time()
    xr, _ = O.ref_integrate(2, N, L, m, x0, t0, t_end, dt, R_fft=Rf, **FRW)
    print(f"reference build: {time.time() - t:.0f} s", flush=True)
    rho = O.ref_power_spectrum(O.ref_energy_density(2, N, L, m, xr, t1, R_fft=Rf, **FRW))
    P = O.make_params(N, L, m, eq=2, **FRW)
    mode = O.ref_mode_power_spectrum(N, L, m, O.a_of_t(P, t1), xr)
    t = time.time()
    y = O.rk4_steps(P, x0, t0, dt, nsteps, R_fft=Rf)
    print(f"restatement: {time.time() - t:.0f} s", flush=True)
    rho_r = O.power_spectrum(O.energy_density(P, y, t1, Rf))
    cross = max(rel_max(y, xr), rel_max(rho_r, rho))
    print(f"restatement vs reference build: {cross:.3e}", flush=True)
    R = 64 * N  # the first 64 rows of the a = 0 plane
    np.savez(out, N=N, L=L, m=m, dt=dt, t0=t0, nsteps=nsteps, k_star=0.25, seed=2, R_seed=3, psi_rms=1e-2,
             k_max=0.5, input_checksum=checksum(x0), R_checksum=checksum(Rf), t_final=t1,
             rho_s2=rho, rho_shells=shells(N, rho), varphi_plus_shells=shells(N, mode),
             phi_rows=xr[:R], dphi_rows=xr[N ** 3:N ** 3 + R], restatement_vs_reference=cross)


def config1_floor(path):
    """The reference's own noise floor at config 1: its -O2 build without -ffast-math
    (oracle/_ref/libcfref_strict.so) against the fixture's -ffast-math build, per
    metric, added to the fixture as floor_*."""
    g = dict(np.load(path))
    N, L, m, dt, t0, nsteps = int(g["N"]), float(g["L"]), float(g["m"]), float(g["dt"]), float(g["t0"]), int(g["nsteps"])
    x0 = fields.initial_state(N, L, float(g["k_star"]), seed=int(g["seed"]))
    t = time.time()
    xs, sp = O.ref_integrate(1, N, L, m, x0, t0, t0 + (nsteps + 0.5) * dt, dt, t_interval=float(g["t_list"][1] - t0),
                             observe=True, strict=True, **FRW)
    print(f"strict reference build: {time.time() - t:.0f} s", flush=True)
    P = O.make_params(N, L, m, eq=1, **FRW)
    t1 = float(g["t_final"])
    rho = O.ref_power_spectrum(O.ref_energy_density(1, N, L, m, xs, t1, strict=True, **FRW), strict=True)
    mode = O.ref_mode_power_spectrum(N, L, m, O.a_of_t(P, t1), xs, strict=True)

    def per_bin(a, b, floor=1e-10):
        big = np.abs(b) >= floor * np.abs(b).max()
        return float(np.max(np.abs(a[big] - b[big]) / np.abs(b[big])))

    def norm_rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    N2 = N * N
    g["floor_rho_s2_final"] = per_bin(rho, g["rho_s2_final"])
    g["floor_varphi_plus_s2_final"] = per_bin(mode, g["varphi_plus_s2_final"])
    g["floor_rho_shells"] = max(per_bin(shells(N, a), b) for a, b in zip(sp["rho"], g["rho_shells"]))
    g["floor_varphi_plus_shells"] = max(per_bin(shells(N, a), b)
                                        for a, b in zip(sp["varphi_plus"], g["varphi_plus_shells"]))
    g["floor_phi_plane0"] = norm_rel(xs[:N2], g["phi_plane0"])
    g["floor_dphi_plane0"] = norm_rel(xs[N ** 3:N ** 3 + N2], g["dphi_plane0"])
    print({k: float(v) for k, v in g.items() if k.startswith("floor_")}, flush=True)
    np.savez(path, **g)


if __name__ == "__main__":
    if not O.ref_available():
        sys.exit("oracle/_ref/libcfref.so is missing: make -C oracle ref REF=<reference tree>")
    which = sys.argv[1] if len(sys.argv) > 1 else "config1"
    if which == "config1":
        config1(os.path.join(HERE, "config1_kgfrw_n256.npz"))
        config1_floor(os.path.join(HERE, "config1_kgfrw_n256.npz"))
    elif which == "config1-floor":
        config1_floor(os.path.join(HERE, "config1_kgfrw_n256.npz"))
    elif which == "config2":
        config2(os.path.join(HERE, "config2_comoving_n512.npz"))
    else:
        sys.exit(f"unknown fixture {which}")
