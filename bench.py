#!/usr/bin/env python
"""Benchmark: GFM Poisson solves/s at relative residual 1e-8 on the 256^2
two-phase droplet workload (plus level-set Mcells/s on the 128^2 level-set
workload), one JSON line on stdout.

A step is one complete GFM pressure solve: curvature + GFM assembly from the
level set, H and divergence, then the solve to a relative residual <= 1e-8
(FP64 recurrence residual; the true FP64 residual is reported), then ps/p
written back.  The measured solver is the mixed-precision one: FP64 flexible
CG preconditioned by an FP32 multigrid V-cycle.  The plain FP64 GPU
Jacobi-PCG (the reference's method, cluster-resident) is timed on the same
system in the same run for the "vs FP64 CG" comparison of the metric.  The system is the one a 256^2
droplet (density ratio 1000, viscosity ratio 100, sigma 0.0728, no-slip
walls) produces after a few steps of the full two-phase step from rest.
Inputs are resident in HBM when the timed region starts; L2 is flushed
(256 MB write) between timed steps because the working set fits in L2.

e2e: the same solves through the C ABI with host buffers: upload ls, H and
div from pinned host memory, assemble, solve, download ps -- all inside the
timed region.

Multi-GPU: the path does not shard (one pressure system per droplet); N
ranks run N independent replicas, value = total solves/s over all ranks with
the time taken as the max over ranks.

--impl reference: the CPU implementation of the same solve on the host's
cores (the C restatement of the reference, one single-threaded process per
core on the same system, since the reference's own all-Neumann solve pins
cell 0 with mis-indexed CSR edits, src/mac2d.cpp:1585-1607, and cannot
converge).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

TOL = 1e-8
N_GRID = 256
LS_GRID = 128
PREP_STEPS = 3
BYTES_PER_UNKNOWN_ITER = 112  # Jacobi-PCG: 14 FP64 streams per iteration (two fused sweeps)
# MG-FCG iteration: FCG sweeps 13 FP64 streams (104 B) + level-0 V-cycle passes
# (pre: r 8 + diag/ce/cn 12 + e 4 = 24 B; post: r 8 + coefficients 12 + e 4 +
# q 8 + z 8 = 40 B) + coarse levels (~1/3 of level 0's 36 FP32 bytes, 12 B)
MG_BYTES_PER_UNKNOWN_ITER = 180
# DRAM bytes (read + write) of one MG-FCG iteration at 256^2, measured: ncu
# --metrics dram__bytes_read.sum,dram__bytes_write.sum --cache-control none on
# 5 iterations (35 launches) of the bench's own solve: 2.3 KB read and 4.56 MB
# written in total
MG_ITER_DRAM_BYTES_256 = 913408
# the same for the one-launch solve (k_mgfcg_persist): DRAM bytes read +
# written by one launch (2.19008 MB + 13.3 KB, 15 iterations) divided by its
# iterations, from one ncu capture of the 256^2 headline solve
MG_PERSIST_DRAM_BYTES_PER_ITER_256 = 146893


METRIC = "GFM Poisson solves/s @resid 1e-8: learned-PC mixed CG vs FP64 CG; LS Mcells/s"


def metric_name():
    return METRIC


def headline_config(n, world):
    """The workload of the headline line, the same for both arms."""
    return {"workload": f"GFM pressure solve (assembly + solve) of a {n}x{n} two-phase droplet (rho ratio 1000, "
                        f"mu ratio 100, sigma 0.0728, no-slip walls) after {PREP_STEPS} full steps, solved to "
                        f"rel. residual {TOL:g}",
            "grid": [n, n], "tol": TOL, "l2": "flushed (256 MB device write) between timed GPU steps",
            "parallelism": "replicas" if world > 1 else "none"}


# ---------------------------------------------------------------- clocks --
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.rows.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=6)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ------------------------------------------------------------- workloads --
def _mg_levels(nx, ny):
    dims = [(nx, ny)]
    while dims[-1][0] * dims[-1][1] > 64:
        a, b = dims[-1]
        dims.append(((a + 1) // 2, (b + 1) // 2))
    return dims


def droplet_params(case):
    from asd2_b200 import api
    return api.Params.from_case(case)


def prepare_state(n, seed, stream):
    """Run a few full droplet steps from rest and return the session and the
    snapshot (ls, H, div, dt) that defines the benchmark's GFM system."""
    from asd2_b200 import api
    from asd2_b200 import workloads as W
    c = W.droplet(n, seed=seed)
    s = api.Session(droplet_params(c), stream=stream)
    s.upload("ls", c.ls)
    s.upload("u", c.u)
    s.upload("v", c.v)
    s.apply_bc("ls", "P")
    dt = s.update_dt()
    for _ in range(PREP_STEPS):
        r = s.droplet_step(dt, tol=1e-10, maxit=500000)
        dt = r["dt_next"]
    # the step's pressure system: kappa/H/div/ls as left by the last step
    snap = {k: s.download(k) for k in ("ls", "H", "div", "kappa")}
    return c, s, snap, dt


LS_MIXED_GRID = 2048       # above L2 for the FP32 level-set working set (6 FP32 + 1 FP64 padded arrays)
LS_MIXED_BYTES = 244       # 55 FP32 streams (220 B) + FP64 -> FP32 -> FP64 conversion of phi (24 B), per cell
LS_FP64_BYTES = 440        # 55 FP64 streams per cell
# FP32 advection part of the step, per cell: the three WENO5/TVD-RK3 stages
# (16 + 20 + 20 B: phi_in, tu, tv, phi_n read, out written; stage 1 reads phi
# once), velocity centring (16 B FP64 faces in, 8 B out), FP64 -> FP32 -> FP64
# of phi (12 + 12 B) and the lsInit copy (8 B)
LS_ADV_BYTES = 112
CFG3_GRID, CFG3_STEPS = 1024, 50


def level_set_rates(sh, stream, flush, peak):
    """Level-set step (WENO5/TVD-RK3 + 5 MinRK2 pseudo-steps with the Sussman
    constraint) at LS_MIXED_GRID in FP32 (mixed session) and FP64: Mcells/s,
    and algorithmic GB/s against the HBM peak.  L2 is flushed before each
    timed step; each step is timed alone with CUDA events on the session's
    stream."""
    import torch
    from asd2_b200 import api
    from asd2_b200 import workloads as W
    lc = W.perturbed_circle(LS_MIXED_GRID, seed=0)
    cells = lc.nx * lc.ny

    def step_time(prec, reps, max_atime=0.0):
        p = api.Params(lc.nx, lc.ny, lc.dx, lc.dy, bc_u=lc.bc_u, bc_v=lc.bc_v, bc_p=lc.bc_p, precision=prec,
                       ls_max_atime=max_atime)
        ss = api.Session(p, stream=sh)
        ss.upload("ls", lc.ls)
        ss.upload("u", lc.u)
        ss.upload("v", lc.v)
        for _ in range(3):
            ss.ls_step(lc.dt, api.REINIT_MINRK2_SUSSMAN)
        ts = []
        for _ in range(reps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            ss.ls_step(lc.dt, api.REINIT_MINRK2_SUSSMAN)
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
        ss.close()
        return float(np.median(ts))

    out = {}
    for prec, bytes_cell, name in ((api.PRECISION_MIXED, LS_MIXED_BYTES, "fp32"), (api.PRECISION_FP64,
                                                                                 LS_FP64_BYTES, "fp64")):
        t = step_time(prec, 10 if prec == api.PRECISION_MIXED else 4)
        gbs = bytes_cell * cells / t / 1e9
        out[name] = {"mcells_per_s": cells / t / 1e6, "ms_per_step": t * 1e3, "achieved_gbs": gbs,
                     "frac_of_measured_hbm": gbs / peak, "bytes_per_cell": bytes_cell}
    # the FP32 step split into advection and one reinitialisation pseudo-step:
    # the same step with one pseudo-step (reinit pseudo-time below one
    # increment) instead of five
    n_ps = 5
    t1 = step_time(api.PRECISION_MIXED, 10, max_atime=0.25 * min(lc.dx, lc.dy))
    t5 = out["fp32"]["ms_per_step"] / 1e3
    t_ps = (t5 - t1) / (n_ps - 1)
    t_adv = t1 - t_ps
    adv_gbs = LS_ADV_BYTES * cells / t_adv / 1e9
    out["fp32_split"] = {"advection_ms": t_adv * 1e3, "pseudo_step_ms": t_ps * 1e3,
                         "advection_gbs": adv_gbs, "advection_frac_of_measured_hbm": adv_gbs / peak,
                         "advection_bytes_per_cell": LS_ADV_BYTES,
                         "method": "t(1 pseudo-step) and t(5 pseudo-steps), CUDA events, L2 flushed"}
    out["grid"] = [LS_MIXED_GRID, LS_MIXED_GRID]
    out["l2"] = "flushed (256 MB write) before each timed step"
    return out


STENCIL_GRID = 2048          # momentum / assembly rooflines: every array (32 MB FP64) above L2
MOM_BYTES_PER_CELL = 192     # 3 RK stages x (read u, v, phi, HS, u^n, v^n; write u, v) = 24 FP64 streams
ASM_BYTES_PER_UNKNOWN = 64   # read phi, kappa, H, div; write diag, ce, cn, rhs = 8 FP64 streams


def stencil_rooflines(sh, stream, flush, peak, n=STENCIL_GRID, reps=10):
    """The momentum step (GetIntermediateVel: three RK3 stages of convection
    + viscosity + gravity, k_mom_stage) and the GFM assembly (k_assemble) on
    an n x n droplet with a smooth random velocity field: CUDA-event time per
    call with L2 flushed before each, algorithmic GB/s against the HBM peak."""
    import torch
    from asd2_b200 import api
    from asd2_b200 import workloads as W
    c = W.droplet(n, seed=0)
    rng = np.random.default_rng(0)
    out = {}
    with api.Session(api.Params.from_case(c), stream=sh) as ss:
        ss.upload("ls", c.ls)
        ss.upload("u", W.smooth_field(n, n, rng, amplitude=0.05))
        ss.upload("v", W.smooth_field(n, n, rng, amplitude=0.05))
        ss.apply_bc("ls", "P")
        ss.apply_bc("u", "U")
        ss.apply_bc("v", "V")
        ss.heaviside()
        ss.kappa()
        ss.upload("div", W.smooth_field(n, n, rng))
        dt = 1e-5

        def timed(fn):
            ts = []
            for k in range(reps + 3):
                with torch.cuda.stream(stream):
                    flush.fill_(1.0)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                fn()
                e1.record(stream)
                e1.synchronize()
                if k >= 3:
                    ts.append(e0.elapsed_time(e1) / 1e3)
            return float(np.median(ts))
        t_mom = timed(lambda: ss.intermediate_vel(dt, "HS"))
        t_asm = timed(lambda: ss.assemble_gfm(dt, recompute_kappa=False))
    N = n * n
    for name, t, b, what in (("momentum", t_mom, MOM_BYTES_PER_CELL, "3 x k_mom_stage + U/V ghost fills"),
                             ("gfm_assembly", t_asm, ASM_BYTES_PER_UNKNOWN, "k_assemble")):
        gbs = b * N / t / 1e9
        out[name] = {"ms": t * 1e3, "kernels": what, "bytes_per_cell": b, "achieved_gbs": gbs,
                     "frac_of_measured_hbm": gbs / peak, "mcells_per_s": N / t / 1e6}
    return {"grid": [n, n], "l2": "flushed (256 MB write) before each timed call", **out}


def ls_cpu_baseline(budget_s=8.0):
    """The reference's own level-set step (Solve_LevelSet_2D + Reinit_MinRK2_2D
    with the Sussman constraint, compiled unmodified in oracle/_ref) on the
    128^2 perturbed circle, one core, for a bounded number of steps; the C
    restatement when the reference build is absent."""
    from asd2_b200 import workloads as W
    from oracle.pyoracle import GridSpec, Oracle, Reference, have_reference
    lc = W.perturbed_circle(LS_GRID, seed=0)
    g = GridSpec(lc.nx, lc.ny, lc.dx, lc.dy, bc_u=lc.bc_u, bc_v=lc.bc_v, bc_p=lc.bc_p)
    a = lc.ls.copy()
    if have_reference():
        R, kind = Reference(g), "reference"

        def step():
            R.ls_advect(a, lc.u, lc.v, lc.dt)
            R.reinit(4, a)
    else:
        O, kind = Oracle(), "port"

        def step():
            O.ls_advect(g, a, lc.u, lc.v, lc.dt)
            O.reinit(g, 4, a)
    t0 = time.perf_counter()
    n = 0
    while n < 3 or time.perf_counter() - t0 < budget_s:
        step()
        n += 1
        if n >= lc.steps:
            break
    t = time.perf_counter() - t0
    return {"value": lc.nx * lc.ny * n / t / 1e6, "unit": "Mcells/s", "cores": 1, "kind": kind,
            "sample": f"{n} level-set steps (WENO5/TVD-RK3 + 5 MinRK2 pseudo-steps with the Sussman constraint) "
                      f"of the {lc.nx}x{lc.ny} perturbed circle in {t:.1f} s"
                      + (", oracle/_ref (the reference's sources compiled unmodified, -O2)" if kind == "reference"
                         else ", oracle/asd2_oracle.c -O2")}


def mixed_precision_errors(sh):
    """The 1024^2 two-phase droplet for 50 steps in FP64 (Jacobi-PCG) and in
    mixed precision (FP32 level set, MG-FCG with an FP32 V-cycle): relative
    max and L2 errors of phi and p against the FP64 run, volume check, and the
    wall time of each run (device synchronised)."""
    from asd2_b200 import api
    from asd2_b200 import workloads as W
    c = W.droplet(CFG3_GRID, seed=0)
    res = {}
    for prec, solver in ((api.PRECISION_FP64, api.PCG), (api.PRECISION_MIXED, api.MGPCG)):
        ss = api.Session(api.Params.from_case(c, precision=prec), stream=sh)
        ss.upload("ls", c.ls)
        ss.upload("u", c.u)
        ss.upload("v", c.v)
        ss.apply_bc("ls", "P")
        dt = ss.update_dt()
        vol0 = ss.volume()
        ss.sync()
        t0 = time.perf_counter()
        its = 0
        for _ in range(CFG3_STEPS):
            r = ss.droplet_step(dt, reinit_mode=api.REINIT_MINRK2, solver=solver, tol=1e-10, maxit=500000)
            if r["status"] != 0:
                raise SystemExit(f"bench: droplet step failed: {r}")
            dt = r["dt_next"]
            its += r["iters"]
        ss.sync()
        el = time.perf_counter() - t0
        res[prec] = dict(**{k: ss.download(k)[3:-3, 3:-3] for k in ("ls", "u", "v", "p", "kappa")}, t=el, its=its,
                         vol0=vol0, vol=ss.last_volume())
        ss.close()
    # the same mixed run device-resident: one graph per step, one synchronisation
    ss = api.Session(api.Params.from_case(c, precision=api.PRECISION_MIXED), stream=sh)
    ss.upload("ls", c.ls)
    ss.upload("u", c.u)
    ss.upload("v", c.v)
    ss.apply_bc("ls", "P")
    dt = ss.update_dt()
    ss.run_steps(0, dt, reinit_mode=api.REINIT_MINRK2, tol=1e-10, maxit=500000)  # builds the step graph
    ss.sync()
    t0 = time.perf_counter()
    r = ss.run_steps(CFG3_STEPS, dt, reinit_mode=api.REINIT_MINRK2, tol=1e-10, maxit=500000)
    t_dev = time.perf_counter() - t0
    if r["status"] != 0:
        raise SystemExit(f"bench: device-resident run failed: {r}")
    same = bool(np.array_equal(ss.download("ls")[3:-3, 3:-3], res[api.PRECISION_MIXED]["ls"]) and
                np.array_equal(ss.download("p")[3:-3, 3:-3], res[api.PRECISION_MIXED]["p"]))
    ss.close()
    a, b = res[api.PRECISION_MIXED], res[api.PRECISION_FP64]
    err = {}
    for k in ("ls", "u", "v", "p", "kappa"):
        d = a[k] - b[k]
        err[k] = {"rel_max": float(np.abs(d).max() / np.abs(b[k]).max()),
                  "rel_l2": float(np.sqrt((d ** 2).mean() / (b[k] ** 2).mean()))}
    # area: the smoothed-Heaviside volume of each run, relative to the FP64 run's
    err["area"] = {"rel": float(abs(a["vol"][1] - b["vol"][1]) / b["vol"][1])}
    return {"workload": f"{CFG3_GRID}x{CFG3_GRID} droplet (rho ratio 1000, mu ratio 100), {CFG3_STEPS} full steps, "
                        "pressure to rel. residual 1e-10",
            "error_vs_fp64": err,
            "volume_rel_change": {"fp64": (b["vol"][1] - b["vol0"][1]) / b["vol0"][1],
                                  "mixed": (a["vol"][1] - a["vol0"][1]) / a["vol0"][1]},
            "seconds": {"fp64": b["t"], "mixed": a["t"], "mixed_device_resident": t_dev},
            "device_resident_identical": same,
            "pressure_iterations": {"fp64_jacobi_pcg": b["its"], "mixed_mg_fcg": a["its"]}}


BATCH_COUNT = 256


def batched_solves(sh, stream, flush, count=BATCH_COUNT):
    """The 256-droplet batch (grid side uniform in {64, 96, ..., 512}, radius
    in [0.08, 0.2], density ratio log-uniform in [1, 1000], viscosity ratio
    log-uniform in [1, 100]): each instance's GFM system is taken after one
    full FP64 droplet step from rest.  Timed: the batched assembly + solve of
    all systems to the FP64-verified rel. residual 1e-8 (one launch per
    phase), against the same systems solved one after another by the FP64
    Jacobi-PCG (the plain FP64 GPU CG) and by the single-system MG-FCG."""
    import torch
    from asd2_b200 import api
    from asd2_b200 import workloads as W
    cases = W.droplet_batch(count, seed=0)
    states, t_cg, t_mg, its_cg, its_mg = [], 0.0, 0.0, [], []

    def timed(fn):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        r = fn()
        e1.record(stream)
        e1.synchronize()
        return r, e0.elapsed_time(e1) / 1e3

    for c in cases:
        with api.Session(api.Params.from_case(c), stream=sh) as ss:
            ss.upload("ls", c.ls)
            ss.upload("u", c.u)
            ss.upload("v", c.v)
            ss.apply_bc("ls", "P")
            dt = ss.update_dt()
            r = ss.droplet_step(dt, solver=api.MGPCG, tol=1e-10, maxit=500000)
            if r["status"] != 0:
                raise SystemExit(f"bench: batch preparation step failed: {r}")
            snap = {k: ss.download(k) for k in ("ls", "H", "kappa", "div")}
            states.append((snap, dt))

            def solve(sv):
                ss.assemble_gfm(dt, recompute_kappa=False)
                return ss.solve_pressure(sv, tol=TOL, maxit=500000, dt=dt)
            solve(api.PCG)
            rc, t = timed(lambda: solve(api.PCG))
            if rc["status"] != 0:
                raise SystemExit(f"bench: FP64 CG did not converge: {rc}")
            t_cg += t
            its_cg.append(rc["iters"])
            solve(api.MGPCG)
            rm, t = timed(lambda: solve(api.MGPCG))
            t_mg += t
            its_mg.append(rm["iters"])
    b = api.Batch([api.Params.from_case(c) for c in cases], stream=sh)
    for k, (snap, _) in enumerate(states):
        for f in ("ls", "H", "kappa", "div"):
            b.upload(k, f, snap[f])
    dts = np.array([dt for _, dt in states])

    def batch_once():
        b.assemble(dts)
        return b.solve(tol=TOL, maxit=10000)
    for _ in range(2):
        batch_once()
    times, res = [], None
    for _ in range(5):
        res, t = timed(batch_once)
        if res["status"] != 0:
            raise SystemExit(f"bench: batched solve did not converge: {res['status']}")
        times.append(t)
    (trow, tcol), trial_ms = b.tile_shape()
    learned = batched_learned(b, dts, timed)
    b.close()
    t_b = float(np.median(times))
    cells = int(sum(c.nx * c.ny for c in cases))
    peak = 6650.0
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak = json.load(f).get("hbm_gbs", peak)
    except Exception:
        pass
    # algorithmic bytes: assembly 64 B/unknown + MG-FCG 180 B/unknown/iteration (instances' own counts)
    alg = float(sum((64 + MG_BYTES_PER_UNKNOWN_ITER * int(it)) * c.nx * c.ny for c, it in zip(cases, res["iters"])))
    return {"workload": f"{count} droplets, grid side uniform in {{64, 96, ..., 512}} ({cells / 1e6:.1f} M unknowns), "
                        "radius [0.08, 0.2], density ratio log-U[1, 1000], viscosity ratio log-U[1, 100]; "
                        "each system after one full step from rest",
            "value": count / t_b, "unit": "GFM Poisson solves/s", "ms_per_batch": t_b * 1e3,
            "tol": TOL, "max_true_rel_residual": float(np.max(res["resid"])),
            "iters": {"batched_max": int(np.max(res["iters"])), "batched_mean": float(np.mean(res["iters"])),
                      "fp64_cg_mean": float(np.mean(its_cg)), "single_mg_mean": float(np.mean(its_mg))},
            "fp64_cg_sequential": {"value": count / t_cg, "unit": "GFM Poisson solves/s",
                                   "solver": "FP64 Jacobi-PCG per system, one system after another"},
            "single_mg_sequential": {"value": count / t_mg, "unit": "GFM Poisson solves/s"},
            "speedup_vs_fp64_cg": t_cg / t_b,
            "mg_tile": {"shape": [trow, tcol], "trial_ms": {"16x32": trial_ms[0], "32x32": trial_ms[1],
                                                           "16x64": trial_ms[2]}},
            "roofline": {"bound": "hbm", "achieved": alg / t_b / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / t_b / 1e9 / peak,
                         "bytes": "assembly 64 B + MG-FCG 180 B per unknown and iteration of each instance"},
            "learned_pc": learned,
            "l2": "flushed (256 MB write) before each timed batch / system"}


def batched_learned(b, dts, timed):
    """The same batch solved with the learned two-level preconditioner
    (asd2g_batch_solve_with(..., ASD2G_SOLVER_UNET), trained weights; one
    network pass per grid-size group): assembly + solve to rel. residual 1e-8,
    median of five after two untimed."""
    from asd2_b200 import api
    from asd2_b200 import train_unet as T
    if not os.path.exists(T.DEFAULT_WEIGHTS):
        return {"unavailable": "no trained preconditioner weights in the package"}
    params, _ = T.load_params()
    net = api.UNet(1, 64, 64)
    net.set_params(params)
    b.set_preconditioner_net(net)
    net.close()

    def once():
        b.assemble(dts)
        return b.solve(tol=TOL, maxit=10000, solver=api.UNET)
    for _ in range(2):
        once()
    times, res = [], None
    for _ in range(5):
        res, t = timed(once)
        if res["status"] != 0:
            raise SystemExit(f"bench: batched learned solve did not converge: {res['status']}")
        times.append(t)
    t = float(np.median(times))
    return {"value": len(dts) / t, "unit": "GFM Poisson solves/s", "ms_per_batch": t * 1e3,
            "iters": {"max": int(np.max(res["iters"])), "mean": float(np.mean(res["iters"]))},
            "max_true_rel_residual": float(np.max(res["resid"])), "fallback": bool(res["fallback"]),
            "solver": "FP64 truncated flexible CG, preconditioner = FP32 V-cycle + U-Net correction (BF16 "
                      "tcgen05 convolutions, one pass per grid-size group) with the A-norm optimal step"}


def learned_pc_512(sh, stream, flush, weights=None, n=512, counts=tuple(range(1, 9)), cpu_baseline=True):
    """The learned-preconditioner evaluation: eight 512^2 GFM systems with
    1 to 8 droplets (radius [0.05, 0.15], density ratio log-uniform in
    [1, 1000]), each taken after one full FP64 droplet step from rest (gravity
    and surface tension drive the flow).  Timed per system (assembly + solve
    to the FP64 relative residual 1e-8): the learned two-level preconditioner
    (ASD2G_SOLVER_UNET, trained weights), the FP64 Jacobi-PCG (plain FP64 GPU
    CG) and the MG-FCG.  The pressure error of the learned solve is measured
    against an FP64 MG-FCG solve to 1e-12."""
    import torch
    from asd2_b200 import api
    from asd2_b200 import workloads as W
    from asd2_b200 import train_unet as T
    path = weights or T.DEFAULT_WEIGHTS
    if not os.path.exists(path):
        return {"unavailable": f"no trained preconditioner weights at {os.path.relpath(path, ROOT)}"}
    params, meta = T.load_params(path)
    net = api.UNet(1, n, n, stream=sh)
    net.set_params(params)
    rng = np.random.Generator(np.random.PCG64(5))

    def timed(fn):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        r = fn()
        e1.record(stream)
        e1.synchronize()
        return r, e0.elapsed_time(e1) / 1e3

    rows, tot, snaps = [], {"unet": 0.0, "cg": 0.0, "mg": 0.0}, []
    for count in counts:
        ratio = float(10 ** rng.uniform(0.0, 3.0))
        c = W.multi_droplet(n, seed=int(rng.integers(1 << 30)), count=count, rho_ratio=ratio)
        with api.Session(api.Params.from_case(c), stream=sh) as ss:
            ss.upload("ls", c.ls)
            ss.upload("u", c.u)
            ss.upload("v", c.v)
            ss.apply_bc("ls", "P")
            dt = ss.update_dt()
            r = ss.droplet_step(dt, solver=api.MGPCG, tol=1e-10, maxit=100000)
            if r["status"] != 0:
                raise SystemExit(f"bench: learned-PC preparation step failed: {r}")
            ss.assemble_gfm(dt, recompute_kappa=False)  # the step's own system (its kappa, H and divergence)
            ref = ss.solve_pressure(api.MGPCG, tol=1e-12, maxit=100000, dt=dt)
            p_ref = ss.download("ps")
            ss.set_preconditioner_net(net)

            def solve(sv):
                ss.assemble_gfm(dt, recompute_kappa=False)
                return ss.solve_pressure(sv, tol=TOL, maxit=100000, dt=dt)
            out = {"droplets": count, "rho_ratio": ratio}
            for key, sv in (("unet", api.UNET), ("cg", api.PCG), ("mg", api.MGPCG)):
                solve(sv)
                res, t = timed(lambda: solve(sv))
                if res["status"] != 0:
                    raise SystemExit(f"bench: {key} solve did not converge: {res}")
                tot[key] += t
                out[key] = {"ms": t * 1e3, "iters": res["iters"], "true_rel_residual": ss.true_residual()}
                if key == "unet":
                    out[key]["fallback"] = bool(ss.last_fallback())
                    ps = ss.download("ps")
                    inner = (slice(3, -3), slice(3, -3))
                    out[key]["p_rel_err_max"] = float(np.abs(ps[inner] - p_ref[inner]).max()
                                                      / np.abs(p_ref[inner]).max())
            out["ref_resid"] = ref["resid"]
            rows.append(out)
            snaps.append(dict(grid=dict(nx=c.nx, ny=c.ny, dx=c.dx, dy=c.dy, bc_u=c.bc_u, bc_v=c.bc_v, bc_p=c.bc_p),
                              fluid=dict(c.fluid), dt=dt, budget_s=0.0, max_solves=1,
                              **{kk: ss.download(kk) for kk in ("ls", "H", "div", "kappa")}))
    k = len(rows)
    net.close()
    cpu = learned_cpu_baseline(snaps) if cpu_baseline else None
    return {"workload": f"{k} GFM systems of {n}x{n} with 1..{max(counts)} droplets (radius [0.05, 0.15], density "
                        "ratio log-U[1, 1000]) after one full FP64 step from rest; assembly + solve to rel. residual "
                        f"{TOL:g}",
            "value": k / tot["unet"], "unit": "GFM Poisson solves/s",
            "solver": "FP64 flexible CG (directions A-orthogonalised against the previous three), preconditioner "
                      "= FP32 V-cycle + U-Net correction (BF16 tcgen05 convolutions) with the A-norm optimal step",
            "fp64_cg": {"value": k / tot["cg"], "unit": "GFM Poisson solves/s"},
            "mg_fcg": {"value": k / tot["mg"], "unit": "GFM Poisson solves/s"},
            "speedup_vs_fp64_cg": tot["cg"] / tot["unet"],
            "fallbacks": int(sum(r["unet"]["fallback"] for r in rows)),
            "max_true_rel_residual": float(max(r["unet"]["true_rel_residual"] for r in rows)),
            "max_p_rel_err": float(max(r["unet"]["p_rel_err_max"] for r in rows)),
            "cpu_baseline": cpu,
            "training": {kk: meta.get(kk) for kk in ("samples", "epochs", "loss", "grid", "seconds_total")},
            "systems": rows, "l2": "flushed (256 MB write) before each timed solve"}


def unet_forward(sh, stream, shapes=((1, 256), (1, 512), (22, 192)), reps=20):
    """Forward pass of the learned preconditioner's U-Net (random weights, B
    images of n x n with the 4 feature channels; 22 x 192² is one size group
    of the 256-droplet batch): CUDA-event time per pass after 3 warm-up
    passes, and the convolution FLOPs it performs."""
    import torch
    from asd2_b200 import api
    lay, _ = api.UNet.layout()
    out = {}
    for B, n in shapes:
        net = api.UNet(B, n, n, stream=sh)
        net.init(1)
        f = torch.randn(B, n, n, 4, device="cuda")
        o = torch.empty(B, n, n, device="cuda")
        for _ in range(3):
            net.forward(f, o, B, n, n)
        with torch.cuda.stream(stream):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        for _ in range(reps):
            net.forward(f, o, B, n, n)
        e1.record(stream)
        e1.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / reps
        # 2 * 9 * cin * cout per output pixel; layer i of the layout works at level (i // 2) for the
        # encoder (i < 8), 2 - (i - 8) // 2 for the decoder, 0 for the output layer
        flops = 0
        for i, (wo, bo, cin, cout, relu) in enumerate(lay):
            lv = i // 2 if i < 8 else (2 - (i - 8) // 2 if i < 14 else 0)
            flops += 2 * 9 * cin * cout * B * (n >> lv) ** 2
        out[str(n) if B == 1 else f"{B}x{n}"] = {"us_per_forward": t * 1e6, "gflop": flops / 1e9, "tflops": flops / t / 1e12,
                       "finite": bool(torch.isfinite(o).all())}
        net.close()
    return {"workload": "U-Net forward (15 tcgen05 convolutions, BF16), batch 1", "sizes": out}


def batched_steps(sh, stream, count=BATCH_COUNT, steps=10):
    """cfg 4 as a whole step: the 256-droplet batch (sides 64..512, radius
    [0.08, 0.2], density ratio log-U[1, 1000], viscosity ratio log-U[1, 100])
    advanced `steps` full droplet steps from rest by asd2g_batch_step (every
    phase one launch for the whole batch, MG-FCG pressure to 1e-8), against the
    same first step run instance by instance through sessions (MG-FCG)."""
    import torch
    from asd2_b200 import api
    from asd2_b200 import workloads as W
    cases = W.droplet_batch(count, seed=0)
    params = [api.Params.from_case(c) for c in cases]
    init, dts, t_seq, its_seq = [], [], 0.0, []
    for c, p in zip(cases, params):
        with api.Session(p, stream=sh) as ss:
            ss.upload("ls", c.ls)
            ss.upload("u", c.u)
            ss.upload("v", c.v)
            ss.apply_bc("ls", "P")
            init.append({k: ss.download(k) for k in ("ls", "u", "v")})
            dt = ss.update_dt()
            dts.append(dt)
            r = ss.droplet_step(dt, solver=api.MGPCG, tol=TOL, maxit=100000)  # first step: set-up, untimed
            ss.sync()
            with torch.cuda.stream(stream):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            r = ss.droplet_step(r["dt_next"], solver=api.MGPCG, tol=TOL, maxit=100000)
            e1.record(stream)
            e1.synchronize()
            if r["status"] != 0:
                raise SystemExit(f"bench: session step failed: {r}")
            t_seq += e0.elapsed_time(e1) / 1e3
            its_seq.append(r["iters"])
    b = api.Batch(params, stream=sh)
    for i, st in enumerate(init):
        for k, a in st.items():
            b.upload(i, k, a)
    b.sync()
    dt = np.array(dts)
    times, its, worst = [], [], 0.0
    for _ in range(steps):
        with torch.cuda.stream(stream):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        r = b.step(dt, tol=TOL, maxit=100000)
        e1.record(stream)
        e1.synchronize()
        if r["status"] != 0:
            raise SystemExit(f"bench: batched step failed: {r['status']}")
        times.append(e0.elapsed_time(e1) / 1e3)
        its.append(float(np.mean(r["iters"])))
        worst = max(worst, float(np.max(r["resid"])))
        dt = r["dt_next"]
    b.close()
    # the same batch with every instance in mixed precision (FP32 level-set
    # advection and reinitialisation); steps 2.. timed
    bm = api.Batch([api.Params.from_case(c, precision=api.PRECISION_MIXED) for c in cases], stream=sh)
    for i, st in enumerate(init):
        for k, a in st.items():
            bm.upload(i, k, a)
    dtm = np.array(dts)
    tm = []
    for k in range(steps):
        with torch.cuda.stream(stream):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        r = bm.step(dtm, tol=TOL, maxit=100000)
        e1.record(stream)
        e1.synchronize()
        if r["status"] != 0:
            raise SystemExit(f"bench: batched mixed step failed: {r['status']}")
        if k > 0:
            tm.append(e0.elapsed_time(e1) / 1e3)
        dtm = r["dt_next"]
    bm.close()
    mixed = {"value": count * len(tm) / float(sum(tm)), "unit": "droplet steps/s",
             "ms_per_batch_step": 1e3 * float(np.mean(tm)), "steps_timed": len(tm),
             "precision": "mixed (FP32 level-set advection and reinitialisation, packed kernels over the batch)"}
    cells = int(sum(c.nx * c.ny for c in cases))
    t_b = float(sum(times))
    return {"mixed_precision": mixed,
            "workload": f"{count} droplets, grid side uniform in {{64, 96, ..., 512}} ({cells / 1e6:.1f} M cells), "
                        f"radius [0.08, 0.2], density ratio log-U[1, 1000], viscosity ratio log-U[1, 100]; {steps} "
                        f"full steps from rest, pressure to rel. residual {TOL:g}",
            "value": count * steps / t_b, "unit": "droplet steps/s",
            "mcells_per_s": cells * steps / t_b / 1e6, "ms_per_batch_step": 1e3 * t_b / steps,
            "ms_per_batch_step_each": [1e3 * t for t in times],
            "iters_mean_per_step": its, "max_rel_residual": worst,
            "sessions_one_by_one": {"value": count / t_seq, "unit": "droplet steps/s",
                                    "iters_mean": float(np.mean(its_seq)),
                                    "note": "second step of every instance, asd2g_droplet_step with the MG-FCG"},
            "speedup_vs_sessions_second_step": t_seq / times[1]}


def full_steps_256(sh, stream, n=N_GRID, steps=20):
    """cfg 2 as whole steps: the 256^2 droplet (density ratio 1000, viscosity
    ratio 100) advanced `steps` full droplet steps from the state after the
    warm-up steps, pressure to rel. residual 1e-10 (the configuration's
    tolerance): FP64 with the FP64 Jacobi-PCG (the reference's method), FP64
    with the MG-FCG, the same device-resident (asd2g_run_steps), and mixed
    precision device-resident."""
    import torch
    from asd2_b200 import api
    from asd2_b200 import workloads as W
    c = W.droplet(n, seed=0)
    out = {}
    for name, prec, solver, device in (("fp64_jacobi_pcg", api.PRECISION_FP64, api.PCG, False),
                                       ("fp64_mg_fcg", api.PRECISION_FP64, api.MGPCG, False),
                                       ("fp64_mg_fcg_device_resident", api.PRECISION_FP64, api.MGPCG, True),
                                       ("mixed_device_resident", api.PRECISION_MIXED, api.MGPCG, True)):
        with api.Session(api.Params.from_case(c, precision=prec), stream=sh) as ss:
            ss.upload("ls", c.ls)
            ss.upload("u", c.u)
            ss.upload("v", c.v)
            ss.apply_bc("ls", "P")
            dt = ss.update_dt()
            for _ in range(3):  # warm-up steps (set-up, graph capture)
                r = ss.droplet_step(dt, solver=solver, tol=1e-10, maxit=500000)
                dt = r["dt_next"]
            if device:
                ss.run_steps(0, dt, tol=1e-10, maxit=500000)
            ss.sync()
            with torch.cuda.stream(stream):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            its = 0
            if device:
                r = ss.run_steps(steps, dt, tol=1e-10, maxit=500000)
                its = r["iters"]
                ok = r["status"] == 0
            else:
                ok = True
                for _ in range(steps):
                    r = ss.droplet_step(dt, solver=solver, tol=1e-10, maxit=500000)
                    ok = ok and r["status"] == 0
                    its += r["iters"]
                    dt = r["dt_next"]
            e1.record(stream)
            e1.synchronize()
            if not ok:
                raise SystemExit(f"bench: full step {name} failed")
            t = e0.elapsed_time(e1) / 1e3
            out[name] = {"steps_per_s": steps / t, "ms_per_step": 1e3 * t / steps,
                         "pressure_iters_per_step": its / steps, "mcells_per_s": n * n * steps / t / 1e6}
    return {"workload": f"{n}x{n} droplet (rho ratio 1000, mu ratio 100), {steps} full steps after 3, "
                        "pressure to rel. residual 1e-10", **out,
            "speedup_mg_device_vs_jacobi": out["fp64_jacobi_pcg"]["ms_per_step"] /
                                           out["fp64_mg_fcg_device_resident"]["ms_per_step"]}


AXI_GRIDS = ((64, 128), (256, 512), (1024, 2048))


def axisym_steps(sh, stream, grids=AXI_GRIDS, steps=10, cpu=True):
    """The axisymmetric MAC step (asd2g_axi_step) on the stationary bubble of
    the reference's axisymmetric driver, at its 64 x 128 grid and two finer
    grids of the same domain: level set (WENO5 + MinRK2), curvature, the
    implicit viscous uhat / vhat (a Thomas solve per grid line), the r-weighted
    GFM assembly and the pressure solve to rel. residual 1e-10 with the FP64
    Jacobi-PCG (the reference's method) or the MG-FCG; `steps` steps after 2
    warm-up steps, CUDA events on the session's stream (each step ends with its
    host read of dt).  CPU baseline: the oracle's restatement of the same step
    (bit-exact to the reference function by function) at 64 x 128, one core."""
    import torch
    from asd2_b200 import api
    from asd2_b200 import workloads as W
    out = {}
    for nr, nz in grids:
        c = W.axisym_bubble(nr, nz)
        res = {}
        for name, solver in (("fp64_jacobi_pcg", api.PCG), ("fp64_mg_fcg", api.MGPCG)):
            with api.Session(api.Params.from_case(c), stream=sh) as ss:
                ss.upload("ls", c.ls)
                ss.upload("u", c.u)
                ss.upload("v", c.v)
                dt = c.dt
                for _ in range(2):
                    r = ss.axi_step(dt, ls_bc=c.meta["bc_ls"], solver=solver, tol=1e-10, maxit=500000)
                    dt = r["dt_next"]
                ss.sync()
                with torch.cuda.stream(stream):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                its, ok = 0, True
                for _ in range(steps):
                    r = ss.axi_step(dt, ls_bc=c.meta["bc_ls"], solver=solver, tol=1e-10, maxit=500000)
                    ok = ok and r["status"] == 0
                    its += r["iters"]
                    dt = r["dt_next"]
                e1.record(stream)
                e1.synchronize()
                if not ok:
                    raise SystemExit(f"bench: axisymmetric step {nr}x{nz} {name} failed")
                t = e0.elapsed_time(e1) / 1e3
                res[name] = {"steps_per_s": steps / t, "ms_per_step": 1e3 * t / steps,
                             "pressure_iters_per_step": its / steps, "mcells_per_s": nr * nz * steps / t / 1e6}
        out[f"{nr}x{nz}"] = res
    rep = {"workload": f"axisymmetric stationary bubble (rho 1000 / 1.226, sigma 0.0728), {steps} steps after 2, "
                       "pressure to rel. residual 1e-10", **out}
    if cpu:
        rep["cpu_baseline"] = axisym_cpu_baseline()
        g0 = f"{grids[0][0]}x{grids[0][1]}"
        rep["speedup_vs_cpu_" + g0] = out[g0]["fp64_mg_fcg"]["steps_per_s"] / rep["cpu_baseline"]["value"]
    return rep


def axisym_cpu_baseline(nr=64, nz=128, steps=5):
    """CPU baseline of axisym_steps: the oracle's axisymmetric step, one core."""
    from asd2_b200 import workloads as W
    from oracle.pyoracle import FluidSpec, GridSpec, Oracle
    O = Oracle()
    c = W.axisym_bubble(nr, nz)
    g = GridSpec(nr, nz, c.dx, c.dy, bc_u=c.bc_u, bc_v=c.bc_v, bc_p=c.bc_p)
    lg = GridSpec(nr, nz, c.dx, c.dy, bc_u=c.bc_u, bc_v=c.bc_v, bc_p=c.meta["bc_ls"])
    f = FluidSpec(**c.fluid)
    st = dict(ls=c.ls.copy(), u=c.u.copy(), v=c.v.copy(), kappa=np.zeros_like(c.ls), dt=c.dt)
    O.axi_step(g, f, st, ls_grid=lg, tol=1e-10)
    t0 = time.perf_counter()
    for _ in range(steps):
        O.axi_step(g, f, st, ls_grid=lg, tol=1e-10)
    t = time.perf_counter() - t0
    return {"value": steps / t, "unit": "axisymmetric steps/s", "cores": 1, "kind": "port",
            "sample": f"{steps} steps of the {nr}x{nz} bubble after 1, pressure by the oracle's FP64 Jacobi-PCG "
                      "to 1e-10"}


def run_ours(args):
    import torch
    from asd2_b200 import api
    from asd2_b200 import workloads as W

    from asd2_b200 import replicas as R
    rank, world, local = R.rank_env()
    torch.cuda.set_device(local)
    dist = R.init_group("nccl")
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream

    c, s, snap, dt = prepare_state(args.n, args.seed + rank, sh)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    solver = api.MGPCG

    def solve_once(sv=solver):
        s.assemble_gfm(dt, recompute_kappa=True)
        return s.solve_pressure(sv, tol=TOL, maxit=500000, dt=dt)

    def timed_solves(sv, k):
        ts, its = [], []
        for _ in range(k):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            r = solve_once(sv)
            e1.record(stream)
            e1.synchronize()
            if r["status"] != 0 or not 0 < r["iters"] <= 500000:
                raise SystemExit(f"bench: pressure solve did not converge: {r}")
            ts.append(e0.elapsed_time(e1) / 1e3)
            its.append(r["iters"])
        return ts, its

    # warm-up
    for _ in range(args.warmup):
        r = solve_once()
    s.sync()
    # timed: device-resident inputs, L2 flushed between steps
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        times, iters = timed_solves(solver, args.steps)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    one_launch = s.last_solve_one_launch()
    true_res = s.true_residual()
    if not true_res <= 10 * TOL:
        raise SystemExit(f"bench: true relative residual {true_res:.3e} above {10 * TOL:g}")
    t_total = R.job_time(float(sum(times)), dist, "cuda")
    value = R.job_rate(args.steps, world, t_total)

    # assembly alone (to split the iteration time out of the solve time)
    ta = []
    for _ in range(max(3, args.steps)):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        s.assemble_gfm(dt, recompute_kappa=True)
        e1.record(stream)
        e1.synchronize()
        ta.append(e0.elapsed_time(e1) / 1e3)
    t_asm = float(np.median(ta))
    it_mean = float(np.mean(iters))
    t_iter = max((t_total / args.steps - t_asm) / it_mean, 1e-12)
    N = args.n * args.n
    achieved = MG_BYTES_PER_UNKNOWN_ITER * N / t_iter / 1e9

    # the plain FP64 GPU CG (Jacobi-PCG, the reference's method) on the same system
    solve_once(api.PCG)
    cg_times, cg_iters = timed_solves(api.PCG, max(2, args.steps // 2))
    cg_value = len(cg_times) / float(sum(cg_times))

    # e2e through host buffers (pinned), copies inside the timed region
    G = (args.n + 6) ** 2
    pin = {k: torch.from_numpy(snap[k]).pin_memory() for k in ("ls", "H", "div")}
    out = torch.empty((args.n + 6, args.n + 6), dtype=torch.float64).pin_memory()
    host = {k: v.numpy() for k, v in pin.items()}
    e2e_t = []
    for k in range(args.warmup + args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        for f in ("ls", "H", "div"):
            s.upload_async(f, host[f])  # pinned buffers, unchanged until the solve synchronises
        s.assemble_gfm(dt, recompute_kappa=True)
        r = s.solve_pressure(solver, tol=TOL, maxit=500000, dt=dt)
        s.L.asd2g_download(s.h, api.PS, out.numpy())
        e1.record(stream)
        e1.synchronize()
        if k >= args.warmup:
            e2e_t.append(e0.elapsed_time(e1) / 1e3)
    e2e_total = R.job_time(float(sum(e2e_t)), dist, "cuda")
    e2e_value = R.job_rate(args.steps, world, e2e_total)

    # the same copies overlapped with the computation of the neighbouring
    # steps: staged transfers on the session's copy stream (step k+1's
    # uploads beside step k's solve, step k's download beside step k+1's
    # assembly), all K steps in one timed region (inputs re-uploaded each
    # step, no L2 flush inside the region)
    outs = [torch.empty((args.n + 6, args.n + 6), dtype=torch.float64).pin_memory().numpy() for _ in range(2)]

    def overlapped(nsteps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        for f in ("ls", "H", "div"):
            s.upload_staged(f, host[f])
        for k in range(nsteps):
            s.join_copies(1)  # this step's inputs have landed
            s.assemble_gfm(dt, recompute_kappa=True)
            if k + 1 < nsteps:
                for f in ("ls", "H", "div"):
                    s.upload_staged(f, host[f])  # the next step's inputs, after this assembly read them
            if k > 0:
                s.join_copies(2)  # the previous step's ps has been read before this solve rewrites it
            r = s.solve_pressure(solver, tol=TOL, maxit=500000, dt=dt)
            if r["status"] != 0:
                raise SystemExit(f"bench: overlapped e2e solve failed: {r}")
            s.download_staged("ps", outs[k % 2])
        s.join_copies(2)
        e1.record(stream)
        e1.synchronize()
        s.sync_copies()
        return e0.elapsed_time(e1) / 1e3

    overlapped(max(3, args.warmup))
    ov_total = R.job_time(overlapped(args.steps), dist, "cuda")
    e2e_overlapped = {"value": R.job_rate(args.steps, world, ov_total), "unit": "GFM Poisson solves/s",
                      "h2d_bytes_per_step": 3 * G * 8, "d2h_bytes_per_step": G * 8,
                      "how": "staged copies on the session's copy stream overlapping the neighbouring steps' "
                             "computation; all steps in one timed region, no L2 flush inside it"}

    # level-set Mcells/s on the 128^2 perturbed-circle workload
    lc = W.perturbed_circle(LS_GRID, seed=args.seed)
    ls_s = api.Session(api.Params(lc.nx, lc.ny, lc.dx, lc.dy, bc_u=lc.bc_u, bc_v=lc.bc_v, bc_p=lc.bc_p), stream=sh)
    ls_s.upload("ls", lc.ls)
    ls_s.upload("u", lc.u)
    ls_s.upload("v", lc.v)
    for _ in range(3):
        ls_s.ls_step(lc.dt, api.REINIT_MINRK2_SUSSMAN)
    ls_s.sync()
    nls = 200
    with torch.cuda.stream(stream):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
    for _ in range(nls):
        ls_s.ls_step(lc.dt, api.REINIT_MINRK2_SUSSMAN)
    e1.record(stream)
    e1.synchronize()
    t_ls = e0.elapsed_time(e1) / 1e3 / nls
    ls_mcells = lc.nx * lc.ny / t_ls / 1e6
    ls_s.close()

    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    ls_rates = level_set_rates(sh, stream, flush, peak) if not args.no_extra else None
    stencils = stencil_rooflines(sh, stream, flush, peak) if not args.no_extra else None
    batched = batched_solves(sh, stream, flush) if not args.no_extra else None
    mixed = mixed_precision_errors(sh) if not args.no_extra else None
    learned = (learned_pc_512(sh, stream, flush, args.weights, cpu_baseline=rank == 0 and not args.no_cpu)
               if not args.no_extra else None)
    bsteps = batched_steps(sh, stream) if not args.no_extra else None
    fsteps = full_steps_256(sh, stream) if not args.no_extra else None
    axi = axisym_steps(sh, stream, cpu=rank == 0 and not args.no_cpu) if not args.no_extra else None
    if one_launch:
        # per solve: dt, curvature, P ghost fill, k_assemble; dt, solver scalars, k_mgfcg_persist, ps and p
        launches = 9 * args.steps
    else:
        nlev = len(_mg_levels(args.n, args.n))
        per_iter = 2 + 2 * (nlev - 1) + 1
        launches = int(sum(4 + (1 + nlev) + (1 + per_iter - 2) + 8 * per_iter * math.ceil(i / 8) + 3 for i in iters))

    line = {
        "metric": metric_name(),
        "value": value,
        "unit": "GFM Poisson solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * t_total / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": headline_config(args.n, world),
        "solver": "mixed precision: FP64 flexible CG + FP32 multigrid V(1,1) preconditioner "
                  "(Galerkin 2x2 aggregation, red-black GS), " +
                  ("the whole solve as one cooperative kernel launch" if one_launch else "per-phase kernels"),
        "solver_iters_mean": it_mean,
        "fp64_cg": {"value": cg_value, "unit": "GFM Poisson solves/s", "iters_mean": float(np.mean(cg_iters)),
                    "solver": "FP64 Jacobi-PCG (the reference's method), one cooperative launch per solve on all SMs"},
        "speedup_vs_fp64_cg": value / world / cg_value,
        "true_rel_residual": true_res,
        "ls_mcells_per_s": ls_mcells,
        "ls_config": {"workload": f"{LS_GRID}x{LS_GRID} perturbed circle, WENO5/TVD-RK3 + 5 MinRK2 subcell "
                                  "pseudo-steps with the Sussman constraint, FP64", "ms_per_step": t_ls * 1e3},
        "ls_cpu_baseline": ls_cpu_baseline() if rank == 0 and not args.no_cpu else None,
        "roofline": {"bound": "hbm",
                     "kernel": ("k_mgfcg_persist (the whole MG-FCG solve, one cooperative launch)" if one_launch
                                else "MG-FCG iteration (k_fcg_a, k_fcg_b, k_mg_pre/post, k_mg_cta_cycle)"),
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": (MG_PERSIST_DRAM_BYTES_PER_ITER_256 if one_launch else MG_ITER_DRAM_BYTES_256)
                     if args.n == 256 else None,
                     "traffic_note": "DRAM bytes read + written per FCG iteration from one ncu capture of the "
                                     "solve (--cache-control none); the hierarchy stays in L2",
                     "bytes_per_unknown_iter": MG_BYTES_PER_UNKNOWN_ITER,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback",
                     "note": "working set is L2-resident at 256^2; iteration time from CUDA events "
                             "(solve minus assembly) / iterations"},
        "batched_256": batched,
        "ls_large": ls_rates,
        "stencils_2048": stencils,
        "mixed_precision_1024": mixed,
        "learned_pc_512": learned,
        "batched_steps_256": bsteps,
        "full_steps_256": fsteps,
        "axisym_steps": axi,
        "e2e_overlapped": e2e_overlapped,
        "e2e": {"value": e2e_value, "unit": "GFM Poisson solves/s",
                "h2d_bytes_per_step": 3 * G * 8, "d2h_bytes_per_step": G * 8},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(snap, c, dt, args)
        try:  # a reported side figure: its failure must not cost the bench line
            line["cpu_reference_cg"] = cg_blas_baseline(snap, c, dt, line["cpu_baseline"]["pcg_iterations"])
        except Exception as e:  # noqa: BLE001
            line["cpu_reference_cg"] = {"error": f"{type(e).__name__}: {e}"[:300]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    s.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ----------------------------------------------------------- CPU baseline --
def _cpu_worker(payload):
    sys.path.insert(0, ROOT)
    from oracle.pyoracle import FluidSpec, GridSpec, Oracle
    g = GridSpec(**payload["grid"])
    f = FluidSpec(**payload["fluid"])
    O = Oracle()
    budget = payload["budget_s"]
    t0 = time.perf_counter()
    n = 0
    while True:
        kap = payload["kappa"].copy()
        sysd = O.gfm_assemble(g, f, payload["dt"], payload["ls"], kap, payload["H"], payload["div"],
                              recompute_kappa=True)
        _, it, _, tres = O.pcg(g, sysd, tol=TOL, maxit=500000)
        n += 1
        if time.perf_counter() - t0 > budget or n >= payload["max_solves"]:
            break
    return n, time.perf_counter() - t0, it, tres


def cpu_baseline(snap, case, dt, args, procs=1, budget_s=None):
    """The C restatement of the reference's solve (single-threaded, fixed
    summation order) on a bounded sample of the same workload."""
    import multiprocessing as mp
    budget = budget_s if budget_s is not None else args.cpu_budget
    payload = dict(grid=dict(nx=case.nx, ny=case.ny, dx=case.dx, dy=case.dy, bc_u=case.bc_u, bc_v=case.bc_v,
                             bc_p=case.bc_p),
                   fluid={k: v for k, v in case.fluid.items()}, dt=dt, budget_s=budget, max_solves=10 ** 6,
                   **{k: snap[k] for k in ("ls", "H", "div", "kappa")})
    if procs == 1:
        n, t, it, tres = _cpu_worker(payload)
        total, tmax = n, t
    else:
        ctx = mp.get_context("spawn")
        with ctx.Pool(procs) as pool:
            res = pool.map(_cpu_worker, [payload] * procs)
        total = sum(r[0] for r in res)
        tmax = max(r[1] for r in res)
        it, tres = res[0][2], res[0][3]
    return {"value": total / tmax, "unit": "GFM Poisson solves/s", "cores": procs, "kind": "port",
            "sample": f"{total} solves of the same {case.nx}x{case.ny} GFM system ({it} PCG iterations each, "
                      f"true rel. residual {tres:.1e}) in {tmax:.1f} s, oracle/asd2_oracle.c built -O2",
            "pcg_iterations": it}


def _quiet_call(fn):
    """fn() with the process's stdout (fd 1) sent to a pipe; returns (fn's
    result, what it printed).  The reference's solvers print one status line
    per solve, which must not reach the bench's JSON line."""
    import ctypes
    sys.stdout.flush()
    libc = ctypes.CDLL(None)
    r, w = os.pipe()
    chunks = []

    def drain():  # read while fn runs, so that no amount of output fills the pipe
        with os.fdopen(r, "rb") as f:
            for block in iter(lambda: f.read1(65536), b""):
                chunks.append(block)
    reader = threading.Thread(target=drain, daemon=True)
    reader.start()
    saved = os.dup(1)
    try:
        os.dup2(w, 1)
        out = fn()
        libc.fflush(None)
    finally:
        os.dup2(saved, 1)
        os.close(saved)
        os.close(w)
        reader.join()
    return out, b"".join(chunks).decode(errors="replace")


def _isolated_entry(conn, fn, payload):
    try:
        conn.send(("ok", fn(payload)))
    except BaseException as e:  # noqa: BLE001 (reported to the parent)
        conn.send(("error", f"{type(e).__name__}: {e}"))
    finally:
        conn.close()


def _run_isolated(fn, payload, timeout):
    """fn(payload) in a fresh spawned process: its result, or an exception
    when it raises, dies (an abort in native code) or runs past `timeout`
    seconds (then it is terminated).  The bench never waits on it for good."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    recv, send = ctx.Pipe(duplex=False)
    proc = ctx.Process(target=_isolated_entry, args=(send, fn, payload), daemon=True)
    proc.start()
    send.close()
    try:
        if not recv.poll(timeout):
            raise TimeoutError(f"worker ran past {timeout} s")
        status, value = recv.recv()
    except EOFError:
        proc.join(5)
        raise RuntimeError(f"worker died (exit code {proc.exitcode})") from None
    finally:
        if proc.is_alive():
            proc.terminate()
        proc.join(5)
        recv.close()
    if status != "ok":
        raise RuntimeError(value)
    return value


def _cg_worker(payload):
    """One build of the reference's CG timed in a fresh process (its BLAS and
    OpenMP thread counts come from the environment it was started with)."""
    sys.path.insert(0, ROOT)
    from oracle.pyoracle import FluidSpec, GridSpec, Reference
    g = GridSpec(**payload["grid"])
    R = Reference(g, FluidSpec(**payload["fluid"]), path=payload["path"])
    a, ia, ja = payload["csr"]
    best, printed = float("inf"), ""
    for _ in range(payload["reps"]):
        t0 = time.perf_counter()
        _, printed = _quiet_call(lambda: R.cg(payload["rhs"], (a, ia, ja), payload["mdiag"], payload["iters"]))
        best = min(best, time.perf_counter() - t0)
    R.close()
    ran = [ln.split() for ln in printed.splitlines() if ln.startswith("CG :")]
    return best, (int(ran[-1][2]) if ran else None)


def cg_blas_baseline(snap, case, dt, its_to_tol, iters=200, reps=3):
    """The reference's own CG_2FUniformP_2D (poisson2d.cpp:230-401) timed per
    iteration on the same GFM system, in its two CPU builds: the serial
    fixed-order BLAS shim (oracle/_ref/libasd2ref.so, one core) and OpenBLAS
    BLAS-1 with the CSR SpMV split over OpenMP threads (libasd2ref_blas.so) at
    three splits of the host cores between the two (passive OpenMP waits: with
    both spinning on every core the two thread pools starve each other).
    The system is the restatement's correctly pinned CSR (the reference's own
    pin is mis-indexed and its CG does not converge on it); `iters`
    iterations per timed call, below the count at which its 1e-6 stop could
    end the call early.  Solves/s = 1 / (time per iteration x the Jacobi-PCG
    iterations to the bench's tolerance, its_to_tol)."""
    from oracle.pyoracle import REF_SO, FluidSpec, GridSpec, Oracle
    blas_so = os.path.join(os.path.dirname(REF_SO), "libasd2ref_blas.so")
    if not os.path.exists(REF_SO):
        return None
    grid = dict(nx=case.nx, ny=case.ny, dx=case.dx, dy=case.dy, bc_u=case.bc_u, bc_v=case.bc_v, bc_p=case.bc_p)
    g, f = GridSpec(**grid), FluidSpec(**case.fluid)
    O = Oracle()
    kap = snap["kappa"].copy()
    sysd = O.gfm_assemble(g, f, dt, snap["ls"], kap, snap["H"], snap["div"], recompute_kappa=True)
    a, ia, ja, b = O.gfm_to_csr(g, sysd)
    rows = len(ia) - 1
    mdiag = np.array([a[ia[r]:ia[r + 1]][ja[ia[r]:ia[r + 1]] == r][0] for r in range(rows)])
    rhs = g.zeros()
    nat = np.concatenate([[0.0], b]) if rows == g.nx * g.ny - 1 else b
    rhs[3:-3, 3:-3] = nat.reshape(g.ny, g.nx).T
    iters = int(min(iters, max(2, its_to_tol // 2)))
    out = {"system": f"{case.nx}x{case.ny} GFM, {rows} unknowns", "iterations_per_call": iters,
           "iterations_to_tol": int(its_to_tol)}
    # a 65k-row system gains nothing from more threads than this, and an
    # OpenBLAS asked for more threads than it was built for may abort
    cores = min(os.cpu_count() or 1, 32)
    runs = [("serial_shim", REF_SO, 1, 1)]
    if os.path.exists(blas_so):
        half = max(1, cores // 2)
        runs += [(f"openblas_{bt}_openmp_{ot}", blas_so, bt, ot) for bt, ot in ((1, cores), (half, half), (cores, 1))]

    saved = {k: os.environ.get(k) for k in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "OMP_WAIT_POLICY")}
    best_name, best_ms = None, float("inf")
    try:
        for name, path, bt, ot in runs:
            os.environ.update(OPENBLAS_NUM_THREADS=str(bt), OMP_NUM_THREADS=str(ot), OMP_WAIT_POLICY="passive")
            payload = dict(grid=grid, fluid=dict(case.fluid), path=path, csr=(a, ia, ja), mdiag=mdiag, rhs=rhs,
                           iters=iters, reps=reps)
            t, done = _run_isolated(_cg_worker, payload, timeout=300)
            ms_it = 1e3 * t / (done or iters)
            out[name] = {"openblas_threads": bt, "openmp_threads": ot, "ms_per_iteration": ms_it,
                         "iterations_run": done, "solves_per_s": 1e3 / (ms_it * its_to_tol)}
            if ms_it < best_ms:
                best_name, best_ms = name, ms_it
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    out["best"] = best_name
    return out


def learned_cpu_baseline(snaps):
    """The C restatement's Jacobi-PCG (the reference's method) on the same
    GFM systems, assembly + solve to rel. residual 1e-8, one single-threaded
    process per system (up to the host's cores) running at the same time."""
    import multiprocessing as mp
    procs = max(1, min(len(snaps), os.cpu_count() or 1))
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_cpu_worker, snaps)
    span = max(r[1] for r in res)  # the processes solve at the same time; start-up is not counted
    its = [r[2] for r in res]
    return {"value": len(snaps) / span, "unit": "GFM Poisson solves/s", "cores": procs, "kind": "port",
            "sample": f"the {len(snaps)} systems once each ({min(its)}-{max(its)} PCG iterations, max true rel. "
                      f"residual {max(r[3] for r in res):.1e}), {procs} processes at once, longest {span:.1f} s; "
                      "oracle/asd2_oracle.c -O2"}


def run_reference(args):
    """Reference arm: CPU implementation of the same solves on all host cores."""
    from asd2_b200 import replicas as R
    if not R.reference_rank_runs(R.rank_env()[0]):
        return
    # Inputs: the same GFM system, generated on the CPU by the restatement's
    # own droplet steps (no GPU is needed for this arm).
    from asd2_b200 import workloads as W
    from oracle.pyoracle import FluidSpec, GridSpec, Oracle
    c = W.droplet(args.n, seed=args.seed)
    g = GridSpec(c.nx, c.ny, c.dx, c.dy, bc_u=c.bc_u, bc_v=c.bc_v, bc_p=c.bc_p)
    f = FluidSpec(**c.fluid)
    O = Oracle()
    st = dict(ls=c.ls.copy(), u=c.u.copy(), v=c.v.copy(), kappa=g.zeros())
    O.bc(g, "p", st["ls"])
    st["dt"] = O.update_dt(g, f, st["u"], st["v"])
    for _ in range(PREP_STEPS):
        info = O.droplet_step(g, f, st, tol=1e-10)
    snap = dict(ls=st["ls"], H=info["H"], div=info["div"], kappa=st["kappa"])
    cores = os.cpu_count() or 1
    per_step = max(args.cpu_budget / max(args.steps, 1), 1.0)
    vals = []
    for k in range(args.warmup + args.steps):
        cb = cpu_baseline(snap, c, st["dt_used"], args, procs=cores, budget_s=per_step)
        if k >= args.warmup:
            vals.append(cb["value"])
    value = float(np.mean(vals))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    line = {"impl": "reference", "metric": metric_name(), "value": value, "unit": "GFM Poisson solves/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": headline_config(args.n, world),
            "solver": "FP64 Jacobi-PCG (the reference's CG_2FUniformP_2D method), C restatement, one process "
                      "per core",
            "cpu_baseline": {"value": value, "unit": "GFM Poisson solves/s", "cores": cores, "kind": "port",
                             "sample": cb["sample"] + f"; {cores} processes"},
            "e2e": {"value": value, "unit": "GFM Poisson solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_GRID)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the 2048^2 level-set and 1024^2 mixed-precision reports")
    ap.add_argument("--weights", default=None, help="learned-preconditioner weights (default: the committed ones)")
    ap.add_argument("--batch-count", type=int, default=BATCH_COUNT,
                    help="droplets of the batched sections (default 256; smaller for profiling)")
    ap.add_argument("--section", default=None,
                    choices=["ls_large", "mixed_1024", "batched", "batched_steps", "learned_pc", "unet_forward",
                             "full_steps", "stencils", "axisym"],
                    help="run only this report (its JSON object on stdout), e.g. to profile it")
    args = ap.parse_args()
    if args.section:
        run_section(args.section, args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


def run_section(name, args):
    import torch
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    if name == "ls_large":
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        peak = 6650.0
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
                peak = json.load(f).get("hbm_gbs", peak)
        except Exception:
            pass
        out = level_set_rates(stream.cuda_stream, stream, flush, peak)
    elif name == "batched":
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        out = batched_solves(stream.cuda_stream, stream, flush, count=args.batch_count)
    elif name == "stencils":
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        peak = 6650.0
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
                peak = json.load(f).get("hbm_gbs", peak)
        except Exception:
            pass
        out = stencil_rooflines(stream.cuda_stream, stream, flush, peak, n=args.n if args.n != N_GRID
                                else STENCIL_GRID)
    elif name == "full_steps":
        out = full_steps_256(stream.cuda_stream, stream)
    elif name == "axisym":
        out = axisym_steps(stream.cuda_stream, stream, cpu=not args.no_cpu)
    elif name == "batched_steps":
        out = batched_steps(stream.cuda_stream, stream, count=args.batch_count)
    elif name == "unet_forward":
        out = unet_forward(stream.cuda_stream, stream)
    elif name == "learned_pc":
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        out = learned_pc_512(stream.cuda_stream, stream, flush, args.weights, cpu_baseline=not args.no_cpu)
    else:
        out = mixed_precision_errors(stream.cuda_stream)
    print(json.dumps({"section": name, **out}), flush=True)


if __name__ == "__main__":
    main()
