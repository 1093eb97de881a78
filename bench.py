#!/usr/bin/env python
"""RK4 site-updates/s of the B200 lattice time stepper (libcfb200.so).

Workload (the configuration the headline metric is quoted on): the
comoving-curvature-coupled Klein-Gordon equation in radiation-dominated FRW
(a1 = 1, H1 = 0.5, t1 = 1, so a = t^1/2), N = 512, L = 512, m = 1, FP32 hi+lo
compensated state (stage arithmetic in FP32 with hi + lo coefficients, an
error-free FP32 state update; FP64 background, reductions and spectra),
7-point Laplacian, RK4 dt = 0.05 from t = 1.  phi(0) is a Gaussian random field (k* = 0.25, <phi^2> = 1), dphi(0) = 0;
R is a k^-3 field with cutoff k_max = 0.5 normalised to rms Psi = 1e-2.
Seeded synthetic inputs; no dataset is involved.

One bench step = one RK4 step of the whole lattice (one whole-step pass and the
Psi / dPsi refreshes at the two new stage times).  The state (1 GB) and all
RK4 buffers are far larger than the 126 MB L2, so no L2 flush is needed between
steps.  Times are CUDA events on the stepping stream, max over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cfb200|reference]

With N > 1 (torchrun), every rank runs an independent replica on its own GPU
(the path has no data-parallel exchange); value = total site updates / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cosmic-fields-lite_b200"))

METRIC = "RK4 site-updates/s @N=512: FP32-comp vs FP64 at ≤1e-6 spectrum err; %HBM peak"
UNIT = "site-updates/s"

FRW = dict(a1=1.0, H1=0.5, t1=1.0)
WORKLOAD = dict(workload="comoving-curvature KG, radiation FRW, N=512^3, L=512, m=1, FP32-comp, 7-point, "
                         "RK4 dt=0.05 from t=1", N=512, L=512.0, m=1.0, dt=0.05, t0=1.0, k_star=0.25,
                psi_rms=1e-2, k_max=0.5)

# Algorithmic HBM bytes per site and RK4 step, by route.
def stage_bytes_per_site(precision, comoving, route="step"):
    """Algorithmic HBM bytes per site-update of one RK4 step.
    route "step" (one whole-step pass, the 7-point default): the state in and out --
    FP64 phi, pi (4 words), FP32-comp hi and lo of phi, pi (8 words) -- plus Psi, dPsi
    at three stage times (+6 words, comoving).  route "pair" (stages 1+2, 3+4; the
    13-point route): FP64 6 + 8 words, FP32-comp 6 + 12, Psi at four stage times +8.
    route "stage" (four single-stage passes): FP64 32, FP32-comp 38, +8."""
    w = 8 if precision == "fp64" else 4
    if route == "step":
        words = (4 if precision == "fp64" else 8) + (6 if comoving else 0)
    elif route == "pair":
        words = (14 if precision == "fp64" else 18) + (8 if comoving else 0)
    else:
        words = (32 if precision == "fp64" else 38) + (8 if comoving else 0)
    return words * w


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profiles(name):
    """DRAM bytes per site-update measured by ncu, from the committed summary."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_site_update:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
            # the timed region starts once the sampler is running (its first line is out)
            t_end = time.time() + 3.0
            while time.time() < t_end and os.path.getsize(self.f.name) == 0:
                time.sleep(0.02)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.f:
            return None
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.f.name)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(x, pg):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


# ---------------------------------------------------------------- reference arm


def cpu_reference_rate(N, steps, threads, comoving=True):
    """The reference's own CPU path (oracle/_ref: src/equations.cpp + Eigen +
    Boost.odeint RK4) on the same workload at lattice size N: site-updates/s."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from cfb200 import fields

    os.environ["CF_FFT_THREADS"] = str(threads)
    W = WORKLOAD
    L = float(N)
    x = fields.initial_state(N, L, W["k_star"], seed=2)
    eta0 = 2.0 * W["t0"] ** 0.5
    Rf = fields.curvature_R_fft(N, L, eta0, W["psi_rms"], W["k_max"], seed=3) if comoving else None
    eq = 2 if comoving else 1
    t_end = W["t0"] + (steps + 0.5) * W["dt"]
    t = time.perf_counter()
    O.ref_integrate(eq, N, L, W["m"], x, W["t0"], t_end, W["dt"], R_fft=Rf, **FRW)
    el = time.perf_counter() - t
    return N ** 3 * steps / el, el


def run_reference_arm(args):
    """The reference's own CPU path (oracle/_ref: src/equations.cpp
    ComovingCurvatureEquationInFRW + Eigen + Boost.odeint runge_kutta4_classic,
    FFTs through the FFTW3 restatement spread over all host cores) on the same
    workload, N = 512.  One RK4 step is timed first; when the run's W + K steps
    at that rate exceed the few-minute bound of this arm, it prints an
    `unavailable` line that carries the measured per-step time instead of
    substituting another lattice."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:  # rank 0 alone runs the CPU path; the others exit without work
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference CPU build) missing"}))
        return
    cores = os.cpu_count() or 1
    os.environ["CF_FFT_THREADS"] = str(cores)
    import numpy as np

    from cfb200 import fields
    W = WORKLOAD
    N, L = W["N"], W["L"]
    t = time.perf_counter()
    x = fields.initial_state(N, L, W["k_star"], seed=2)
    eta0 = 2.0 * W["t0"] ** 0.5
    Rf = fields.curvature_R_fft(N, L, eta0, W["psi_rms"], W["k_max"], seed=3)
    setup_s = time.perf_counter() - t

    def one_step(state, step):
        t0 = W["t0"] + step * W["dt"]
        t = time.perf_counter()
        out, _ = O.ref_integrate(2, N, L, W["m"], state, t0, t0 + 1.5 * W["dt"], W["dt"], R_fft=Rf, **FRW)
        return out, time.perf_counter() - t

    x, first = one_step(x, 0)
    budget_s = 240.0
    sample = (f"reference CPU path (src/equations.cpp ComovingCurvatureEquationInFRW + Eigen + Boost.odeint "
              f"runge_kutta4_classic) on the workload itself, N={N}: one RK4 step per bench step; the stepping "
              f"is single-threaded as shipped, its FFTs (FFTW3 restatement) use {cores} threads")
    if (args.warmup + args.steps - 1) * first > budget_s:
        print(json.dumps({"impl": "reference",
                          "unavailable": f"the reference CPU path takes {first:.1f} s per N={N} RK4 step on this "
                                         f"host ({cores} cores; stepping single-threaded as shipped); "
                                         f"{args.warmup + args.steps} steps exceed this arm's {budget_s:.0f} s "
                                         f"bound",
                          "measured_s_per_step": first, "measured_site_updates_per_s": N ** 3 / first,
                          "setup_s": setup_s, "config": dict(WORKLOAD), "sample": sample}))
        return
    for i in range(1, args.warmup):
        x, _ = one_step(x, i)
    times = []
    for i in range(args.steps):
        x, el = one_step(x, args.warmup + i)
        times.append(el)
    el = sum(times)
    value = N ** 3 * len(times) / el
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                      "steps": len(times), "warmup": args.warmup, "ms_per_step": 1e3 * el / len(times),
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                      "data": "synthetic", "config": dict(WORKLOAD),
                      "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                                       "sample": sample},
                      "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


# ---------------------------------------------------------------- product arm


def make_case(N, L, precision, stencil, comoving, use_torch_inputs=True):
    import torch

    import cfb200
    from cfb200 import fields
    W = WORKLOAD
    prec = cfb200.FP32_COMP if precision == "fp32comp" else cfb200.FP64
    eq = cfb200.EQ_COMOVING_FRW if comoving else cfb200.EQ_KG_FRW
    ctx = cfb200.Context(N, L, m=W["m"], equation=eq, precision=prec, stencil=stencil, **FRW)
    x = fields.initial_state(N, L, W["k_star"], seed=2, use_torch=use_torch_inputs)
    st = torch.empty(ctx.info.state_bytes // 8, dtype=torch.float64, device="cuda")
    ctx.import_f64(st, x)
    if comoving:
        eta0 = 2.0 * W["t0"] ** 0.5
        Rf = fields.curvature_R_fft(N, L, eta0, W["psi_rms"], W["k_max"], seed=3, use_torch=use_torch_inputs)
        ctx.set_R_fft(Rf, on_device=True)
        del Rf
    del x
    torch.cuda.synchronize()
    return ctx, st


def accuracy_run(N, L, nsteps, every):
    """Density-spectrum error of the FP32-comp stepper against the FP64 stepper
    (which matches the FP64 oracle to 1e-12 in the parity tests) on the headline
    workload: both start from the same state; the density spectra are compared
    every `every` steps (100 steps = dt_save 5); the worst norm-wise error and the
    worst per-bin error (bins >= 1e-6 of the peak) over all checkpoints."""
    import numpy as np
    import torch
    W = WORKLOAD
    c32, x32 = make_case(N, L, "fp32comp", 7, True)
    c64, x64 = make_case(N, L, "fp64", 7, True)
    a = torch.empty(c32.info.s2_bins, dtype=torch.float64, device="cuda")
    b = torch.empty_like(a)
    worst, worst_bin, final = 0.0, 0.0, None
    for k in range(nsteps // every):
        c32.rk4_steps(x32, W["t0"], W["dt"], every, step0=k * every)
        c64.rk4_steps(x64, W["t0"], W["dt"], every, step0=k * every)
        t = W["t0"] + (k + 1) * every * W["dt"]
        c32.density_spectrum_s2(x32, t, a)
        c64.density_spectrum_s2(x64, t, b)
        torch.cuda.synchronize()
        sa, sb = a.cpu().numpy(), b.cpu().numpy()
        err = float(np.linalg.norm(sa - sb) / np.linalg.norm(sb))
        big = np.abs(sb) >= 1e-6 * np.abs(sb).max()
        worst = max(worst, err)
        worst_bin = max(worst_bin, float(np.max(np.abs(sa - sb)[big] / np.abs(sb)[big])))
        final = err
    del c32, x32, c64, x64
    torch.cuda.empty_cache()
    return {"steps": nsteps, "every": every, "normwise_max": worst, "normwise_final": final,
            "max_bin_rel_ge_1e-6_max": worst_bin}


def adjoint_bench(N=256, nsteps=200, every=20, ngroups=32, floor=1e-12):
    """Config 4: plain FRW KG at N=256, L=256, 200 RK4 steps (dt = 0.05 from t = 1)
    with checkpoints every 20 steps; phi0 = c2r(sqrt(theta_g) sqrtP(k) xi_k) with 32
    shell-group amplitudes theta (GRF baseline k* = 0.25), dphi0 = 0; loss = sum over
    the shells within 12 decades of the peak of (log P_rho - log P_target)^2, the
    target from the m = 1.1 run.  Times one gradient (checkpointed forward, loss,
    reverse sweep, theta gradient) in FP64 and FP32-comp, and checks dL/dm and
    dL/dtheta_0 of the FP64 adjoint against central differences (h = 1e-4)."""
    import numpy as np
    import torch

    import cfb200
    from cfb200 import fields
    L, dt, t0 = float(N), 0.05, 1.0
    xi = torch.from_numpy(fields.white_noise_hc(N, 11)).cuda()
    sqrtP = torch.from_numpy(fields.gaussian_sqrtP_by_s2(N, L, 0.25)).cuda()

    def run(theta, m, precision, target=None, grad=False):
        ctx = cfb200.Context(N, L, m=m, equation=cfb200.EQ_KG_FRW, precision=precision, stencil=7, **FRW)
        nsh = ctx.info.shells
        spg = -(-nsh // ngroups)
        phi = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
        cfb200.field_from_shell_amplitudes(ctx, xi, sqrtP, theta, spg, phi)
        st = torch.empty(ctx.info.state_bytes // 8, dtype=torch.float64, device="cuda")
        ctx.import_f64(st, torch.cat([phi, torch.zeros_like(phi)]))
        adj = cfb200.Adjoint(ctx, nsteps, every)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        adj.forward(st, t0, dt)
        if target is None:
            sh = torch.empty(nsh, dtype=torch.float64, device="cuda")
            s2 = torch.empty(ctx.info.s2_bins, dtype=torch.float64, device="cuda")
            ctx.density_spectrum_s2(st, t0 + nsteps * dt, s2)
            ctx.s2_to_shells(sh)
            out = sh.cpu().numpy()
            adj.close()
            return out
        loss = adj.shell_log_loss(st, target, floor)
        if not grad:
            adj.close()
            return loss
        lam0 = torch.empty(2 * N ** 3, dtype=torch.float64, device="cuda")
        dm = adj.backward(lam0)
        gth = cfb200.shell_amplitude_gradient(ctx, lam0[: N ** 3], xi, sqrtP, theta, spg)
        e1.record()
        torch.cuda.synchronize()
        adj.close()
        return loss, gth, dm, e0.elapsed_time(e1)

    theta = np.ones(ngroups)
    target = run(theta, 1.1, cfb200.FP64)
    res = {"N": N, "steps": nsteps, "checkpoint_every": every, "parameters": ngroups + 1}
    for name, prec in (("fp64", cfb200.FP64), ("fp32comp", cfb200.FP32_COMP)):
        run(theta, 1.0, prec, target, grad=True)  # warm
        loss, gth, dm, ms = run(theta, 1.0, prec, target, grad=True)
        res[name] = {"ms_per_gradient": ms, "loss": loss, "dL_dm": dm}
        if name == "fp64":
            h = 1e-4
            fd_m = (run(theta, 1.0 + h, prec, target) - run(theta, 1.0 - h, prec, target)) / (2 * h)
            tp, tm = theta.copy(), theta.copy()
            tp[0] += h
            tm[0] -= h
            fd_t = (run(tp, 1.0, prec, target) - run(tm, 1.0, prec, target)) / (2 * h)
            res["fd_check_fp64"] = {"dL_dm_rel_err": abs(dm - fd_m) / abs(fd_m),
                                    "dL_dtheta0_err_rel_to_max_grad": abs(gth[0] - fd_t) / np.abs(gth).max()}
    torch.cuda.empty_cache()
    return res


def ensemble_bench(steps=500, per_segment=50):
    """Config 3: 96 FRW Klein-Gordon lattices (32 x 64^3, 32 x 96^3, 32 x 128^3),
    L = N, m ~ U[0.5, 2] (seed 12345), GRF initial fields (k* = 0.5, <phi^2> = 1,
    dphi = 0, seeds 1000 + i), FP32-comp, 7-point, dt = 0.1 from t = 1, density
    spectra every 50 steps.  The same `steps` are timed as CUDA-graph replays of
    one interval (the batched whole-step launches, one per step, or the persistent
    kernel) + the spectra, as direct batched launches, and as one whole-step launch
    per step per member (the single-instance path)."""
    import numpy as np
    import torch

    import cfb200
    from cfb200 import fields
    rng = np.random.default_rng(12345)
    sizes = [64] * 32 + [96] * 32 + [128] * 32
    spec = [dict(N=n, L=float(n), m=float(rng.uniform(0.5, 2.0)), equation=cfb200.EQ_KG_FRW,
                 precision=cfb200.FP32_COMP, stencil=7, **FRW) for n in sizes]
    ens = cfb200.Ensemble(spec)
    tune = ens.autotune(1.0, 0.1, steps=2)
    x0 = [fields.initial_state(d["N"], d["L"], 0.5, 1000 + i, use_torch=True).cpu().numpy()
          for i, d in enumerate(spec)]
    sites = sum(n ** 3 for n in sizes)
    out = torch.empty((steps // per_segment) * ens.spectra_total, dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    res = {"members": len(sizes), "sites": sites, "steps": steps, "autotune": {"shape": tune[0], "a_chunk": tune[1]},
           "work_items": ens.work_items}
    for name in ("graph_batched", "graph_persistent", "loop_single_launches", "batched_launches"):
        for i, x in enumerate(x0):
            ens.upload(i, x)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        l0 = ens.launches
        with torch.cuda.stream(stream):
            if name.startswith("graph_"):
                gmode = cfb200.ENS_BATCHED if name == "graph_batched" else cfb200.ENS_PERSISTENT
                ens.run_graph(1.0, 0.1, per_segment, 1, None, stream=stream, mode=gmode)  # capture + warm
                for i, x in enumerate(x0):
                    ens.upload(i, x, stream=stream)
                l0 = ens.launches
                e0.record(stream)
                ens.run_graph(1.0, 0.1, per_segment, steps // per_segment, out, stream=stream, mode=gmode)
                e1.record(stream)
            else:
                mode = cfb200.ENS_LOOP if name == "loop_single_launches" else cfb200.ENS_BATCHED
                ens.rk4_steps(1.0, 0.1, 2, mode=mode, stream=stream)  # warm
                for i, x in enumerate(x0):
                    ens.upload(i, x, stream=stream)
                e0.record(stream)
                for s in range(steps // per_segment):
                    ens.rk4_steps(1.0, 0.1, per_segment, step0=s * per_segment, mode=mode, stream=stream)
                    ens.density_spectra_s2(1.0 + (s + 1) * per_segment * 0.1,
                                           out[s * ens.spectra_total:], stream=stream)
                e1.record(stream)
        stream.synchronize()
        ms = e0.elapsed_time(e1)
        res[name] = {"site_updates_per_s": sites * steps / (ms * 1e-3), "ms": ms, "launches": ens.launches - l0}
    res["graph_vs_loop"] = res["graph_batched"]["site_updates_per_s"] / res["loop_single_launches"]["site_updates_per_s"]
    ens.close()
    torch.cuda.empty_cache()
    return res


def reference_gpu_bench():
    """The reference's own GPU stepping path on this B200, as a reported baseline
    (not the product): oracle/_ref/ref_gpu_bench drives the reference's unmodified
    src/equations_cuda.cu, fdm3d_cuda.cu, cuda_wrapper.cu and
    odeint_thrust/thrust_operations.cu the way src/main.cpp does (thrust-vector
    workspace, Cuda*Equation, runge_kutta4_classic with the thrust algebra), FP64,
    and times do_step with CUDA events."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_bench")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/ref_gpu_bench (the reference's GPU build) missing"}
    res = {"kind": "the reference's own GPU code (FP64), oracle/_ref/ref_gpu_bench"}
    for name, argv in (("comoving_7pt_n512", ["2", "512", "5", "2"]), ("kgfrw_7pt_n512", ["1", "512", "10", "3"]),
                       ("kgfrw_7pt_n256", ["1", "256", "20", "3"])):
        try:
            out = subprocess.run([exe] + argv, capture_output=True, text=True, timeout=600)
            line = [l for l in out.stdout.splitlines() if l.startswith("{")]
            res[name] = json.loads(line[-1]) if line else {"error": (out.stderr or out.stdout)[-300:]}
        except Exception as e:  # reported, not hidden
            res[name] = {"error": str(e)}
    return res


def spectrum_bench(ctx, st, t, reps=5):
    """The spectrum step on the headline state (N = 512, FP32-comp, comoving), the
    observer's density spectrum: energy density (state hi + lo and the cached Psi
    slot in, rho out; the pass also bounds sum rho^2 for the fixed-point scale), the
    FP64 R2C, the orbit binning and the s^2 bins.  Algorithmic bytes per site: 16
    (state) + 4 (e^{2Psi} - 1) + 8 (rho) in the energy pass, 8 + 8 for the R2C at one
    read and one write, 8 for the pass over the half-complex modes: 52 B."""
    import torch
    out = torch.empty(ctx.info.s2_bins, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    for _ in range(2):
        ctx.density_spectrum_s2(st, t, out)
    torch.cuda.synchronize()
    ctx.profile(True)
    ctx.profile_reset()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        ctx.density_spectrum_s2(st, t, out)
    e1.record(stream)
    torch.cuda.synchronize()
    prof = ctx.profile_read()
    ctx.profile(False)
    ms = e0.elapsed_time(e1) / reps
    N = ctx.N
    peak, kind = load_peaks()
    gbs = 52 * N ** 3 / (ms * 1e-3) / 1e9
    return {"N": N, "ms": ms, "algorithmic_bytes_per_site": 52, "achieved_gbs": gbs, "hbm_frac": gbs / peak,
            "peak_kind": kind, "launches_per_spectrum": sum(v[0] for v in prof.values()) / reps}


def config1_bench():
    """Configuration 1: KleinGordonEquationInFRW, N = 256, L = 256, m = 1, radiation era,
    RK4 dt = 0.05 for 1000 steps from t = 1, from the seeded input of the committed
    fixture tests/golden/config1_kgfrw_n256.npz (made by the reference's own CPU
    build).  Times the 1000 steps in FP64 and FP32-comp and compares the density and
    mode power spectra after them with the fixture: per bin over the bins >= 1e-10 of
    the largest, and norm-wise."""
    import numpy as np
    import torch

    import cfb200
    from cfb200 import fields
    g = dict(np.load(os.path.join(ROOT, "tests", "golden", "config1_kgfrw_n256.npz")))
    N, L, m, dt, t0, nsteps = int(g["N"]), float(g["L"]), float(g["m"]), float(g["dt"]), float(g["t0"]), int(g["nsteps"])
    x0 = fields.initial_state(N, L, float(g["k_star"]), seed=int(g["seed"]))
    chk = np.array([x0.sum(), (x0 * x0).sum()])
    res = {"N": N, "steps": nsteps, "dt": dt, "input_matches_fixture": bool(np.allclose(chk, g["input_checksum"],
                                                                                      rtol=1e-12, atol=0))}

    def per_bin(a, b):
        big = np.abs(b) >= 1e-10 * np.abs(b).max()
        return float(np.max(np.abs(a[big] - b[big]) / np.abs(b[big])))

    for name, prec in (("fp64", cfb200.FP64), ("fp32comp", cfb200.FP32_COMP)):
        ctx = cfb200.Context(N, L, m=m, equation=cfb200.EQ_KG_FRW, precision=prec, stencil=7, **FRW)
        st = torch.empty(ctx.info.state_bytes // 8, dtype=torch.float64, device="cuda")
        ctx.upload(st, x0)
        warm = torch.empty_like(st)
        warm.copy_(st)
        ctx.rk4_steps(warm, t0, dt, 5)  # warm-up on a copy
        del warm
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.rk4_steps(st, t0, dt, nsteps)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        t1 = t0 + nsteps * dt
        rho = torch.empty(ctx.info.s2_bins, dtype=torch.float64, device="cuda")
        mode = torch.empty_like(rho)
        ctx.density_spectrum_s2(st, t1, rho)
        ctx.mode_power_spectrum_s2(st, cfb200.a_of_t(FRW["a1"], FRW["H1"], FRW["t1"], t1), mode)
        r, md = rho.cpu().numpy(), mode.cpu().numpy()
        res[name] = {"ms_per_step": ms / nsteps, "site_updates_per_s": N ** 3 * nsteps / (ms * 1e-3),
                     "density_spectrum_vs_reference": {
                         "per_bin_max": per_bin(r, g["rho_s2_final"]),
                         "normwise": float(np.linalg.norm(r - g["rho_s2_final"]) / np.linalg.norm(g["rho_s2_final"]))},
                     "mode_spectrum_vs_reference_per_bin_max": per_bin(md, g["varphi_plus_s2_final"])}
        ctx.close()
        del st
    if "floor_rho_s2_final" in g:
        res["reference_own_floor_per_bin"] = {"rho": float(g["floor_rho_s2_final"]),
                                              "varphi_plus": float(g["floor_varphi_plus_s2_final"])}
    torch.cuda.empty_cache()
    return res


def time_steps(ctx, st, steps, warmup, profile=False):
    import torch
    W = WORKLOAD
    stream = torch.cuda.current_stream()
    ctx.rk4_steps(st, W["t0"], W["dt"], warmup, step0=0)
    torch.cuda.synchronize()
    if profile:
        ctx.profile(True)
        ctx.profile_reset()
    l0 = ctx.launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.rk4_steps(st, W["t0"], W["dt"], steps, step0=warmup)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    prof = ctx.profile_read() if profile else None
    if profile:
        ctx.profile(False)
    return ms, ctx.launches - l0, prof


def run_product(args):
    import numpy as np
    import torch

    import cfb200
    world, rank, local, pg = dist_setup()
    torch.cuda.set_device(local)
    W = WORKLOAD
    N, L = W["N"], W["L"]
    peak, peak_kind = load_peaks()

    # ---- headline: FP32-comp comoving, 7-point (--quick --fp64: the FP64 stepper on it)
    prec = "fp64" if args.quick and args.fp64 else "fp32comp"
    ctx, st = make_case(N, L, prec, 7, True)
    barrier(pg)
    with ClockSampler(local) as clk:
        ms, launches, prof = time_steps(ctx, st, args.steps, args.warmup, profile=True)
    clocks = clk.summary()
    ms = max_over_ranks(ms, pg)
    value = world * N ** 3 * args.steps / (ms * 1e-3)

    import cfb200
    stage_ms = sum(prof[k][1] for k in cfb200.STEP_KINDS)
    stage_launches = sum(prof[k][0] for k in cfb200.STEP_KINDS)
    bps = stage_bytes_per_site(prec, True, "step")
    achieved = bps * N ** 3 * args.steps / (stage_ms * 1e-3) / 1e9
    # DRAM bytes per site-update of the whole-step pass from an ncu capture at N = 256
    # (inputs 10x L2), scaled by the sites a launch processes
    traffic = traffic_from_profiles("step_kernel_n256.md") if prec == "fp32comp" else None
    roofline = {"bound": "hbm",
                "kernel": f"k_step (one pass per RK4 step, {'FP32-comp' if prec == 'fp32comp' else 'FP64'}, "
                          "comoving, 7-point)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind,
                "traffic": (traffic * N ** 3 * args.steps / stage_launches) if traffic else None,
                "traffic_unit": "bytes per launch",
                "algorithmic_bytes_per_site_update": bps,
                "time_share": {k: v[1] / max(1e-9, sum(x[1] for x in prof.values())) for k, v in prof.items()
                               if v[0]},
                "time_share_note": "per-kind CUDA-event intervals; the Psi refreshes run on a side stream beside "
                                   "the step passes, so their intervals overlap the step's and include time "
                                   "queued behind it"}
    if args.quick:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "config": WORKLOAD, "storage": prec,
                "roofline": roofline, "gpu_launches": launches, "clocks": clocks}
        if args.spectrum:
            line["spectrum"] = spectrum_bench(ctx, st, W["t0"] + (args.steps + args.warmup) * W["dt"], reps=2)
        if rank == 0:
            print(json.dumps(line))
        if pg is not None:
            pg.destroy_process_group()
        return

    # ---- the FP64 stepper on the same workload (throughput)
    ctx64, st64 = make_case(N, L, "fp64", 7, True)
    t64_ms, _, prof64 = time_steps(ctx64, st64, args.steps, args.warmup, profile=True)
    fp64_value = world * N ** 3 * args.steps / (max_over_ranks(t64_ms, pg) * 1e-3)
    del ctx64, st64
    torch.cuda.empty_cache()
    # ---- accuracy: FP32-comp against FP64 over 1000 steps, spectra every dt_save = 5
    accuracy = accuracy_run(N, L, 1000 if not args.quick else 100, 100)
    s32 = torch.empty(ctx.info.s2_bins, dtype=torch.float64, device="cuda")

    # ---- secondary variants (same workload shape)
    secondary = {"fp64_comoving_7pt": {"value": fp64_value, "ms_per_step": t64_ms / args.steps}}
    ks = max(5, args.steps // 4)
    for name, prec, stencil, com in (("fp32comp_comoving_13pt", "fp32comp", 13, True),
                                     ("fp32comp_kgfrw_7pt", "fp32comp", 7, False),
                                     ("fp64_kgfrw_7pt", "fp64", 7, False)):
        c2, s2_ = make_case(N, L, prec, stencil, com)
        t2, _, p2 = time_steps(c2, s2_, ks, args.warmup, profile=True)
        sm = sum(p2[k][1] for k in cfb200.STEP_KINDS)
        bb = stage_bytes_per_site(prec, com, "step" if stencil == 7 else "pair")
        secondary[name] = {"value": world * N ** 3 * ks / (max_over_ranks(t2, pg) * 1e-3),
                           "ms_per_step": t2 / ks,
                           "stage_kernels_gbs": bb * N ** 3 * ks / (sm * 1e-3) / 1e9}
        del c2, s2_
        torch.cuda.empty_cache()

    # ---- config 3: ensemble of uneven N, one captured graph per observer interval
    try:
        secondary["ensemble_config3"] = ensemble_bench(steps=500, per_segment=50)
    except Exception as e:  # reported, not hidden
        secondary["ensemble_config3"] = {"error": str(e)}
    # ---- config 4: adjoint gradient of the shell-spectrum loss
    try:
        secondary["adjoint_config4"] = adjoint_bench()
    except Exception as e:  # reported, not hidden
        secondary["adjoint_config4"] = {"error": str(e)}

    # ---- end to end through the C ABI with host buffers: one observer interval
    # (dt_save = 5 -> 100 RK4 steps) per e2e step: upload the state from pinned
    # host memory, step, density spectrum, download the spectrum.
    n_inner = 100
    host_state = torch.empty(2 * N ** 3, dtype=torch.float64).pin_memory()
    tmp = torch.empty(2 * N ** 3, dtype=torch.float64, device="cuda")
    ctx.export_f64(tmp, st)
    host_state.copy_(tmp.cpu())
    del tmp
    host_spec = [torch.empty(ctx.info.s2_bins, dtype=torch.float64).pin_memory() for _ in range(2)]
    e2e_steps = 4
    stream = torch.cuda.current_stream()
    # Double-buffered: the upload of step k + 1's state runs on a copy stream into the
    # other device state while step k steps; every upload and every spectrum read-back
    # stays inside the timed region.
    copy_stream = torch.cuda.Stream()
    states = [st, torch.empty_like(st)]
    uploaded = [torch.cuda.Event() for _ in range(2)]
    released = [torch.cuda.Event() for _ in range(2)]

    def e2e_upload(k):
        b = k & 1
        copy_stream.wait_event(released[b])
        ctx.upload(states[b], host_state.data_ptr(), stream=copy_stream)
        uploaded[b].record(copy_stream)

    def e2e_compute(k):
        b = k & 1
        stream.wait_event(uploaded[b])
        ctx.rk4_steps(states[b], W["t0"], W["dt"], n_inner, step0=k * n_inner)
        ctx.density_spectrum_s2(states[b], W["t0"] + (k + 1) * n_inner * W["dt"], s32)
        host_spec[b].copy_(s32, non_blocking=True)
        released[b].record(stream)

    for b in range(2):
        released[b].record(stream)
    e2e_upload(0)
    e2e_compute(0)
    torch.cuda.synchronize()
    barrier(pg)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    copy_stream.wait_event(e0)
    e2e_upload(1)
    for k in range(1, e2e_steps + 1):
        if k < e2e_steps:
            e2e_upload(k + 1)
        e2e_compute(k)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), pg)
    e2e_value = world * N ** 3 * n_inner * e2e_steps / (e2e_ms * 1e-3)
    states_last = states[e2e_steps & 1]
    del states

    # ---- the spectrum step at N = 512 on the state of the last e2e step (its Psi slot is cached)
    t_spec = W["t0"] + (e2e_steps + 1) * n_inner * W["dt"]
    try:
        secondary["spectrum_n512"] = spectrum_bench(ctx, states_last, t_spec)
    except Exception as e:  # reported, not hidden
        secondary["spectrum_n512"] = {"error": str(e)}
    del states_last
    # ---- configuration 1 (N = 256, 1000 steps) timed, and checked against the reference's run
    try:
        config1 = config1_bench()
        secondary["config1_kgfrw_n256"] = config1
    except Exception as e:  # reported, not hidden
        config1 = None
        secondary["config1_kgfrw_n256"] = {"error": str(e)}
    # ---- the reference's own GPU stepping path (FP64), a reported baseline
    if world == 1 and rank == 0:
        secondary["reference_gpu"] = reference_gpu_bench()

    # ---- CPU baseline: the reference's own CPU path, bounded sample, rank 0 at N=1
    cpu = None
    if world == 1 and rank == 0:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        if O.ref_available():
            cores = os.cpu_count() or 1
            r, el = cpu_reference_rate(N, 1, cores)
            cpu = {"value": r, "unit": UNIT, "cores": cores, "kind": "reference",
                   "sample": f"reference CPU path (ComovingCurvatureEquationInFRW, Eigen, Boost.odeint RK4) on "
                             f"the workload itself, N={N}, 1 RK4 step ({el:.1f} s); the stepping is "
                             f"single-threaded as shipped, its FFTs (FFTW3 restatement) use {cores} threads"}

    # ---- config 2 at N = 1024 (the headline workload, 8x the sites)
    try:
        del ctx, st
        torch.cuda.empty_cache()
        c2, s2_ = make_case(1024, 1024.0, "fp32comp", 7, True)
        t2, _, p2 = time_steps(c2, s2_, 10, 3, profile=True)
        secondary["fp32comp_comoving_7pt_n1024"] = {
            "value": world * 1024 ** 3 * 10 / (max_over_ranks(t2, pg) * 1e-3), "ms_per_step": t2 / 10,
            "psi_route": int(c2.info.psi_route)}
        del c2, s2_
        torch.cuda.empty_cache()
    except Exception as e:  # reported, not hidden
        secondary["fp32comp_comoving_7pt_n1024"] = {"error": str(e)}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "fp32comp",
                "storage": "f32 hi + f32 lo; stage arithmetic f32 with hi + lo coefficients; f64 reductions",
                "data": "synthetic",
                "config": dict(WORKLOAD, precision="fp32comp", stencil=7, parallelism=f"replicas x{world}",
                               l2="inputs larger than L2 (state 1.07 GB, RK4 buffers 3.2 GB); no flush"),
                "fp32comp_vs_fp64": value / fp64_value,
                "density_spectrum_err_vs_fp64": accuracy,
                "density_spectrum_err_vs_reference": (
                    {"config": "configuration 1 (KG-FRW, N=256, 1000 steps) against the reference's own CPU run",
                     "fp32comp": config1["fp32comp"]["density_spectrum_vs_reference"],
                     "fp64": config1["fp64"]["density_spectrum_vs_reference"]} if config1 else None),
                "roofline": roofline, "cpu_baseline": cpu,
                "e2e": {"value": e2e_value, "unit": UNIT,
                        "h2d_bytes_per_step": int(host_state.numel() * 8),
                        "d2h_bytes_per_step": int(host_spec[0].numel() * 8),
                        "steps": e2e_steps, "ms": e2e_ms,
                        "step": f"upload state + {n_inner} RK4 steps + density spectrum + download spectrum",
                        "pipeline": "two device states: step k+1's upload (copy stream) overlaps step k's "
                                    "stepping; the first upload is not overlapped"},
                "gpu_launches": launches, "clocks": clocks, "secondary": secondary}
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="cfb200", choices=["cfb200", "reference"])
    ap.add_argument("--n", type=int, default=None,
                    help="lattice size override (profiling a smaller case of the same workload)")
    ap.add_argument("--quick", action="store_true",
                    help="headline measurement only (no accuracy check, variants, e2e or CPU baseline)")
    ap.add_argument("--spectrum", action="store_true",
                    help="with --quick: also time the observer's density spectrum on the stepped state")
    ap.add_argument("--fp64", action="store_true",
                    help="with --quick: the FP64 stepper on the headline workload instead of FP32-comp")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.fp64 and not args.quick:
        ap.error("--fp64 goes with --quick")
    if args.fp64:
        WORKLOAD["workload"] = WORKLOAD["workload"].replace("FP32-comp", "FP64")
    if args.n:
        WORKLOAD["N"] = args.n
        WORKLOAD["L"] = float(args.n)
        WORKLOAD["workload"] = WORKLOAD["workload"].replace("N=512^3, L=512", f"N={args.n}^3, L={args.n}")
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_product(args)


if __name__ == "__main__":
    main()
