#!/usr/bin/env python
"""Benchmark of the B200 hot path (one JSON line on rank 0).

Workload "dns" (default): the DNS shear layer on the 512x256x512
staggered grid (domain 4pi x 2pi x 20, periodic x/y, free-slip z walls, z
tanh-stretched), Re=4000, Pr=1, Ri=0.08, seeded perturbation 1e-3, time
step from CFL 0.5 (calcdt); every sub-step projects with the mixed-precision
multigrid (FP32 V-cycles inside FP64 defect correction; z-line Gauss-Seidel
with x/y semi-coarsening unless --smoother rbpgs) to a true relative
residual of 1e-10.  One step = one full RK3 time step (three sub-steps,
three projections).  Fields are FP64.

  value    -- cell-updates/s: interior cells x steps / device time, state
              resident in HBM (CUDA events on the step stream, max over ranks)
  e2e      -- the same through the C-ABI with the state in pinned host
              memory: every step copies u, v, w, p, rho host->device, runs
              the step and copies them back
  roofline -- the dominant kernel (finest-level smoother of the pressure
              solves): algorithmic bytes per launch / mean launch time
              (CUDA events on its stream)

Workload "poisson": standalone pressure solves of the same grid (one step
= one solve to 1e-10 from phi0 = 0).

--impl reference times the CPU restatement of the reference's algorithm
(FP64, red-black point Gauss-Seidel; the Fortran reference cannot be built
here) on the host cores instead.
N > 1 GPUs (torchrun): independent replicas, no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    # name: kind, (nx, ny, nz), MG levels, physics
    "dns": ("dns", (512, 256, 512), (9, 8, 9), dict(Re=4000.0, g=-0.08, amp=1e-3, cfl=0.5)),
    "dns256": ("dns", (256, 256, 256), (8, 8, 8), dict(Re=4000.0, g=-0.08, amp=1e-3, cfl=0.5)),
    "dns_small": ("dns", (64, 32, 64), (6, 5, 6), dict(Re=1000.0, g=-0.12, amp=1e-3, cfl=0.5)),
    # LES shear layer: constant-coefficient Smagorinsky (Cs^2 = 0.0289, f_damp = 1),
    # eddy diffusivity with Pr_sgs = 0.7
    "les": ("dns", (768, 384, 384), (9, 8, 8), dict(Re=50000.0, g=-0.1, amp=1e-2, cfl=0.5, les=True)),
    "les_small": ("dns", (96, 48, 48), (6, 5, 5), dict(Re=50000.0, g=-0.1, amp=1e-2, cfl=0.5, les=True)),
    # the 768x384x384 LES grid with the reference runfile's dynamic models (DSM,
    # DSMrho, DSMscal1; TestGrid_ratio sqrt(6), filters in x, y, z)
    "les_dsm": ("dns", (768, 384, 384), (9, 8, 8), dict(Re=50000.0, g=-0.1, amp=1e-2, cfl=0.5, les=True,
                                                       dsm=True)),
    # one member of the serving stream, for the CPU baseline of "serve"
    "dns64": ("dns", (64, 64, 64), (6, 6, 6), dict(Re=1000.0, g=-0.12, amp=1e-3, cfl=0.5)),
    # ensemble serving: a Poisson stream of shear-layer members (sizes below)
    "serve": ("serve", (256, 256, 256), None, {}),
    "poisson": ("poisson", (512, 256, 512), (9, 8, 9), {}),
    "poisson256": ("poisson", (256, 256, 256), (8, 8, 8), {}),
    "poisson_small": ("poisson", (64, 32, 64), (6, 5, 6), {}),
    # serving-bucket sizes, for the batched solve (--members)
    "poisson64": ("poisson", (64, 64, 64), (6, 6, 6), {}),
    "poisson128": ("poisson", (128, 128, 128), (7, 7, 7), {}),
    # profiling case: 134 MB per FP32 field (above L2), ~1.5 GB on the device
    "poisson_prof": ("poisson", (512, 128, 512), (9, 7, 9), {}),
}
TOL = 1e-10


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(key):
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get(key)
    return None


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.f is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().splitlines() if r.strip()]
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


SMOOTHER = {"smoother": "rbpgs", "pre": 2, "post": 2}


def mg_params(lv, precision, mode=None, smoother=None):
    """V(2,2) cycles, metric operator, true-residual stop.  With the ZLINE
    smoother the z direction is not coarsened (horizontal semi-coarsening).
    `smoother` ("zline" | "rbpgs") overrides the run's choice."""
    from anelastic_solve_b200 import abi

    zl = (smoother or SMOOTHER["smoother"]) == "zline"
    levels = (lv[0], lv[1], 1) if zl else lv
    pre, post = (SMOOTHER["pre"], SMOOTHER["post"]) if smoother is None else (2, 2)
    fine = (SMOOTHER.get("fine_pre"), SMOOTHER.get("fine_post")) if smoother is None else (None, None)
    if fine != (None, None):
        # per-level counts (coarsest -> finest), the finest level's own
        ng = max(levels)
        pre = [pre] * (ng - 1) + [pre if fine[0] is None else fine[0]]
        post = [post] * (ng - 1) + [post if fine[1] is None else fine[1]]
    return abi.make_mg_params(levels, maxcy=400, tolmax=TOL, pre=pre, post=post,
                              tbc=(0, 1, 0, 1, 0, 0), precision=precision,
                              smoother=abi.SMOOTHER_ZLINE if zl else abi.SMOOTHER_RBPGS,
                              mode=abi.MODE_METRIC if mode is None else mode, stop=abi.STOP_RESID)


def fine_note(args):
    """The finest level's own sweep counts, when set, for the config line."""
    if args.fine_pre is None and args.fine_post is None:
        return ""
    fp = args.pre if args.fine_pre is None else args.fine_pre
    fq = args.post if args.fine_post is None else args.fine_post
    return f" (finest level V({fp},{fq}))"


def ns_params(phys, pguess=0):
    """pguess 1: each sub-step's pressure solve starts from the linear
    extrapolation of the member's solutions of that sub-step in the last
    two steps (an extension; 0 = the reference's start from the current p)."""
    from anelastic_solve_b200 import abi

    # DeltaT_max large: the CFL condition sets the step (calcdt)
    dsm = phys.get("dsm", False)
    return abi.make_ns_params(Re=phys["Re"], Pr=1.0, g=phys["g"], cfl=phys["cfl"], dtmax=1e9,
                              ew=1, scal1_on=0, les=phys.get("les", False), ssm_const=0.0289,
                              pr_sgs=0.7, les_damp=abi.DAMP_NONE, les_start=0, les_freq=1,
                              models=(abi.MODEL_DSM,) * 3 if dsm else None, stretched=(0, 0, 1),
                              interp=abi.DIAG_CORRECTED, pguess=pguess)


def poisson_rhs(g, seed=1):
    """Seeded N(0,1) right-hand side with the volume mean removed (the
    compatibility condition of the Neumann/periodic problem)."""
    rng = np.random.default_rng(seed)
    f = rng.standard_normal(g.ghosted[::-1])  # (Z,Y,X) C-order == Fortran (X,Y,Z)
    vol = (g.z.dxc[1:-1, None, None] * g.y.dxc[None, 1:-1, None] * g.x.dxc[None, None, 1:-1])
    inner = f[1:-1, 1:-1, 1:-1]
    inner -= (inner * vol).sum() / vol.sum()
    return f


def initial_state(g, phys):
    from anelastic_solve_b200 import shear

    return shear.shear_layer_fields(g, amp=phys["amp"], seed=12345)


STATE = ("u", "v", "w", "p", "rho")


# ------------------------------------------------------------ multi-rank
def combine_ranks(world, device, maxes=(), sums=()):
    """Replicas: the max over ranks of each timing in `maxes` and the sum
    of each count in `sums` (every rank takes the same collective steps in
    the same order).  Returns (maxes, sums) as lists."""
    maxes, sums = [float(v) for v in maxes], [float(v) for v in sums]
    if world <= 1:
        return maxes, sums
    import torch
    import torch.distributed as dist

    if maxes:
        t = torch.tensor(maxes, dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        maxes = t.tolist()
    if sums:
        t = torch.tensor(sums, dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        sums = t.tolist()
    return maxes, sums


def weak_value(world, cells, ms_step):
    """Whole-job throughput of N replicas: every rank advanced `cells` in
    the slowest rank's time."""
    return world * cells / (ms_step / 1e3)


# ---------------------------------------------------------------- ours: dns
def run_dns(args, rank, world, local_rank):
    import torch

    from anelastic_solve_b200 import _lib, abi
    from anelastic_solve_b200 import grid as G
    from anelastic_solve_b200.mg import MGSolver
    from anelastic_solve_b200.ns import NSSolver

    kind, n, lv, phys = WORKLOADS[args.workload]
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    g = G.shear_layer_grid(*n, stretched=True)
    N = g.x.n * g.y.n * g.z.n
    prec = abi.PREC_MIXED if args.prec == "mixed" else abi.PREC_FP64
    s = NSSolver(g, mg_params(lv, prec), ns_params(phys, args.pguess if args.prec == "mixed" else 0),
                 device=local_rank)
    f = initial_state(g, phys)
    s.set_fields({k: f[k] for k in ("u", "v", "w", "p", "rho", "scal1", "r", "densityBG")})
    del f
    s.project()
    st = torch.cuda.Stream(device=dev)
    h = st.cuda_stream

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    for _ in range(args.warmup):
        s.step(1, stream=h)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = []
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        torch.cuda.nvtx.range_push("timed")
        ev0.record(st)
        for _ in range(args.steps):
            reps.append(s.step(1, stream=h))
        ev1.record(st)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    barrier()
    ms_step = ev0.elapsed_time(ev1) / args.steps
    # one more step with the smoother launches timed by events (profiling
    # runs the V-cycles launch by launch), for the roofline of the smoother
    s.set_profiling(True)
    prep = s.step(1, stream=h)
    s.set_profiling(False)
    diag_ms = None
    if args.diag:
        # the driver's per-step plane statistics (stretched z, corrected
        # interpolation), timed by the step report after their own warm-up
        s.set_diagnostics(True, abi.DIAG_CORRECTED, (0, 0, 1))
        s.step(1, stream=h)
        dreps = [s.step(1, stream=h) for _ in range(2)]
        s.set_diagnostics(False, abi.DIAG_CORRECTED, (0, 0, 1))
        diag_ms = float(np.mean([r.diag_ms for r in dreps]))
    out = {"N": N, "ms_step": ms_step, "clocks": clk.summary(),
           "diag_ms_step": diag_ms,
           "launches": int(sum(r.launches for r in reps)),
           "sweeps": int(prep.fine_sweeps),
           "sweep_ms": float(prep.fine_sweep_ms),
           "mg_ms_step": float(np.mean([r.mg_ms for r in reps])),
           "mg_iters": [list(r.mg_iter) for r in reps],
           "dt": reps[-1].dt, "max_div": reps[-1].max_div,
           "umax": None}
    # e2e: the state lives in pinned host memory; every step copies it in,
    # runs through the C-ABI and copies it back
    if not args.no_e2e:
        host = {k: np.asfortranarray(torch.zeros(g.ghosted[::-1], dtype=torch.float64)
                                     .pin_memory().numpy().T) for k in STATE}
        s.get_into(host)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ne = max(1, args.steps // 2)
        torch.cuda.synchronize()
        e0.record(st)
        for _ in range(ne):
            # host state in, one step, host state out (copies overlapped
            # with the step where the data allow)
            s.step_host(host, host, 1, stream=h)
        e1.record(st)
        torch.cuda.synchronize()
        out["e2e_ms"] = e0.elapsed_time(e1) / ne
        nb = len(STATE) * int(np.prod(g.ghosted)) * 8
        out["bytes_io"] = (nb, nb)
    # mixed vs FP64 multigrid on this workload's pressure equation: cold
    # solves (phi0 = 0) of the last sub-step's right-hand side, with this
    # run's multigrid and with the plain FP64 path (the reference's
    # red-black point smoother, full coarsening: the one-for-one mg_solver
    # replacement)
    if rank == 0 and not args.no_fp64:
        fld = s.get_fields(("psrc",))
        rhs = torch.from_numpy(np.ascontiguousarray(fld["psrc"].T)).to(dev)
        mg = {}
        for name, pr, sm in (("mixed", abi.PREC_MIXED, None), (f"fp64_{args.smoother}", abi.PREC_FP64, None),
                             ("fp64_rbpgs", abi.PREC_FP64, "rbpgs")):
            if name in mg:
                continue
            m = MGSolver(g, mg_params(lv, pr, smoother=sm), device=local_rank)
            phi = torch.zeros_like(rhs)
            m.solve(phi, rhs, stream=h)
            phi.zero_()
            m.solve(phi, rhs, stream=h)
            r = m.last_report
            mg[name] = {"ms": round(r.ms, 3), "iter": r.iter, "resid": r.resid}
            m.close()
        del rhs
        out["mg_cold"] = mg
    # the plain FP64 GPU path (FP64 multigrid, red-black point Gauss-Seidel,
    # full coarsening) on the same state: whole steps timed like the main
    # run, so that mixed vs plain FP64 is measured in the same process
    if not args.no_fp64 and kind == "dns":
        names = ("u", "v", "w", "p", "rho", "scal1", "nuT", "kappaT", "nappaT")
        st_now = s.get_fields(names)
        s64 = NSSolver(g, mg_params(lv, abi.PREC_FP64, smoother="rbpgs"), ns_params(phys), device=local_rank)
        s64.set_fields({k: st_now[k] for k in ("u", "v", "w", "p", "rho", "scal1")})
        one = np.ones(g.ghosted, order="F")
        s64.set_fields({"r": one, "densityBG": one})
        del one
        s64.step(1, stream=h)
        torch.cuda.synchronize()
        n64 = 3
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        reps64 = [s64.step(1, stream=h) for _ in range(n64)]
        e1.record(st)
        torch.cuda.synchronize()
        out["fp64_plain"] = {"ms_per_step": e0.elapsed_time(e1) / n64, "steps": n64,
                             "mg_iters": [list(x.mg_iter) for x in reps64],
                             "mg_ms_per_step": float(np.mean([x.mg_ms for x in reps64]))}
        s64.close()
        del st_now
    fu = s.get_fields(("u", "v", "w"))
    out["umax"] = float(max(np.abs(fu[k][1:-1, 1:-1, 1:-1]).max() for k in ("u", "v", "w")))
    out["dzmin"] = float(g.z.dxc[1:-1].min())
    # the benchmarked sub-step against the FP64 oracle at full size, from
    # this run's state after its timed steps: the GPU's sub-step (this
    # run's multigrid) and the oracle's (FP64, the reference's red-black
    # point smoother) from the same fields.  The oracle's time is the CPU
    # baseline (one steady-state sub-step on the host cores, x3 per step).
    if rank == 0 and world == 1 and not args.no_cpu and kind == "dns":
        out["oracle_leg"] = oracle_leg(s, g, lv, phys, os.cpu_count() or 1, h)
    s.close()
    out["tuning"] = _lib.tuning_report().splitlines()
    keys = [k for k in ("ms_step", "e2e_ms") if k in out]
    out.update(zip(keys, combine_ranks(world, dev, maxes=[out[k] for k in keys])[0]))
    return out


# ------------------------------------------------------------ ours: poisson
def run_poisson(args, rank, world, local_rank):
    import torch

    from anelastic_solve_b200 import _lib, abi
    from anelastic_solve_b200 import grid as G
    from anelastic_solve_b200.mg import MGSolver

    kind, n, lv, phys = WORKLOADS[args.workload]
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    g = G.shear_layer_grid(*n, stretched=True)
    N = g.x.n * g.y.n * g.z.n
    prec = abi.PREC_MIXED if args.prec == "mixed" else abi.PREC_FP64
    s = MGSolver(g, mg_params(lv, prec), device=local_rank)
    st = torch.cuda.Stream(device=dev)
    f = poisson_rhs(g)
    dsrc = torch.from_numpy(f).to(dev)
    dphi = torch.zeros_like(dsrc)
    for _ in range(args.warmup):
        with torch.cuda.stream(st):
            dphi.zero_()
        s.solve(dphi, dsrc, stream=st.cuda_stream)
    st.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    iters = []
    launches0 = _lib.launch_count()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        torch.cuda.nvtx.range_push("timed")
        ev0.record(st)
        for _ in range(args.steps):
            with torch.cuda.stream(st):
                dphi.zero_()
            s.solve(dphi, dsrc, stream=st.cuda_stream)
            iters.append(s.last_report.iter)
        ev1.record(st)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    launches = _lib.launch_count() - launches0
    # one more solve with the smoother launches timed by events, for the
    # roofline of the smoother
    s.set_profiling(True)
    with torch.cuda.stream(st):
        dphi.zero_()
    s.solve(dphi, dsrc, stream=st.cuda_stream)
    sweep_ms, sweeps = s.last_report.fine_sweep_ms, s.last_report.fine_sweeps
    s.set_profiling(False)
    out = {"N": N, "ms_step": ev0.elapsed_time(ev1) / args.steps, "clocks": clk.summary(),
           "launches": launches, "sweeps": sweeps, "sweep_ms": sweep_ms,
           "iters": iters, "resid": s.last_report.resid}
    if not args.no_e2e:
        ph = np.asfortranarray(torch.zeros(dsrc.shape, dtype=torch.float64).pin_memory().numpy().T)
        fh = np.asfortranarray(torch.from_numpy(f).pin_memory().numpy().T)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ne = max(1, args.steps // 2)
        e0.record(st)
        for _ in range(ne):
            ph[...] = 0.0
            s.solve(ph, fh, stream=st.cuda_stream)
        e1.record(st)
        torch.cuda.synchronize()
        out["e2e_ms"] = e0.elapsed_time(e1) / ne
        out["bytes_io"] = (2 * dsrc.numel() * 8, dsrc.numel() * 8)
    if args.members > 1:
        out["batched"] = batched_solves(s, g, args, st, dev)
    s.close()
    out["tuning"] = _lib.tuning_report().splitlines()
    keys = [k for k in ("ms_step", "e2e_ms") if k in out]
    out.update(zip(keys, combine_ranks(world, dev, maxes=[out[k] for k in keys])[0]))
    return out


def batched_solves(s, g, args, st, dev):
    """B = args.members independent right-hand sides (seeds 1..B) of this
    grid: solved one after another (solve_device each, CUDA events around
    all B) and as one batched solve (solve_batch); the batched solutions
    must equal the one-by-one ones bit for bit."""
    import torch

    B = args.members
    rhs = [torch.from_numpy(poisson_rhs(g, seed=1 + b)).to(dev) for b in range(B)]
    one = [torch.zeros_like(rhs[0]) for _ in range(B)]
    bat = [torch.zeros_like(rhs[0]) for _ in range(B)]
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]

    def alone():
        for b in range(B):
            with torch.cuda.stream(st):
                one[b].zero_()
            s.solve(one[b], rhs[b], stream=st.cuda_stream)

    def together():
        with torch.cuda.stream(st):
            for b in range(B):
                bat[b].zero_()
        return s.solve_batch(bat, rhs, stream=st.cuda_stream)

    alone()
    together()  # warm-up of both (graphs built)
    torch.cuda.synchronize()
    ev[0].record(st)
    alone()
    ev[1].record(st)
    ev[2].record(st)
    reps = together()
    ev[3].record(st)
    torch.cuda.synchronize()
    t1, tb = ev[0].elapsed_time(ev[1]), ev[2].elapsed_time(ev[3])
    same = all(torch.equal(one[b], bat[b]) for b in range(B))
    return {"members": B, "ms_one_by_one": round(t1, 3), "ms_batched": round(tb, 3),
            "speedup": round(t1 / tb, 3), "cycles": [r.iter for r in reps], "bitwise_equal": same}


# ------------------------------------------------------------ CPU samples
def oracle_fields(g, state):
    """Fortran-ordered host fields for the oracle: every array of
    abi.FIELD_NAMES (zeros), r = densityBG = 1, then the given state."""
    from anelastic_solve_b200 import abi

    f = {n: np.zeros(g.ghosted, order="F") for n in abi.FIELD_NAMES}
    f["r"][...] = 1.0
    f["densityBG"][...] = 1.0
    for k, v in state.items():
        f[k][...] = v
    return f


def cpu_reference_step(workload, threads):
    """The reference's algorithm on the host cores at the full workload
    size: the oracle restatement, FP64, red-black point Gauss-Seidel with
    full coarsening, metric operator, stop at a true relative residual of
    1e-10.  Untimed warm-up: the initial projection and one whole RK3 step
    (its first sub-step, from the projected state, needs about three times
    the cycles of a steady one).  Timed: the next whole step.  Returns a
    dict with the seconds of the timed step, its cycles per sub-step, the
    warm-up's cycles and the interior cell count."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from anelastic_solve_b200 import abi
    from anelastic_solve_b200 import grid as G
    from oracle.pyoracle import OracleNS

    kind, n, lv, phys = WORKLOADS[workload]
    g = G.shear_layer_grid(*n, stretched=True)
    f = initial_state(g, phys)
    o = OracleNS(g, mg_params(lv, abi.PREC_FP64, smoother="rbpgs"), ns_params(phys), f)
    for name, vt in (("u", 0), ("v", 1), ("w", 2), ("rho", 4), ("scal1", 12)):
        o.ghost(f[name], vt)
    pit, _ = o.project()
    warm = o.step()
    t = time.perf_counter()
    rep = o.step()
    sec = time.perf_counter() - t
    return {"seconds": sec, "cycles": list(rep.mg_iter), "warm_cycles": [pit] + list(warm.mg_iter),
            "cells": g.x.n * g.y.n * g.z.n}


def oracle_leg(s, g, lv, phys, threads, stream):
    """One RK3 sub-step (the first of a step) from the GPU run's current
    state, on the GPU with the run's own multigrid and on the host with the
    FP64 oracle (the reference's red-black point smoother, full
    coarsening, to the same 1e-10 residual).  Returns the oracle's time
    and cycles (the CPU baseline sample) and the relative L2 error of each
    GPU field against the oracle's (pressure after removing the volume
    mean)."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from anelastic_solve_b200 import abi
    from anelastic_solve_b200.ns import RK3
    from oracle.pyoracle import OracleNS

    names = ("u", "v", "w", "p", "rho", "scal1", "nuT", "kappaT", "nappaT")
    state = s.get_fields(names)
    dt = cfl_dt(g, state, phys["cfl"])
    a1, a2, a3, ec, fr = RK3[0]
    it_g, _ = s.substep(a1, a2, a3, fr * dt, dt, stream=stream)
    gpu = s.get_fields(("u", "v", "w", "p", "rho"))
    f = oracle_fields(g, state)
    del state
    o = OracleNS(g, mg_params(lv, abi.PREC_FP64, smoother="rbpgs"), ns_params(phys), f)
    t = time.perf_counter()
    it_o, _ = o.substep(a1, a2, a3, fr * dt, dt)
    sec = time.perf_counter() - t

    def rel(a, b):
        a, b = a[1:-1, 1:-1, 1:-1], b[1:-1, 1:-1, 1:-1]
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    def vmean(a):
        vol = g.x.dxc[1:-1, None, None] * g.y.dxc[None, 1:-1, None] * g.z.dxc[None, None, 1:-1]
        inner = a[1:-1, 1:-1, 1:-1]
        return inner - (inner * vol).sum() / vol.sum()

    err = {k: rel(gpu[k], f[k]) for k in ("u", "v", "w", "rho")}
    num = sum(np.linalg.norm((gpu[k] - f[k])[1:-1, 1:-1, 1:-1]) ** 2 for k in "uvw")
    den = sum(np.linalg.norm(f[k][1:-1, 1:-1, 1:-1]) ** 2 for k in "uvw")
    err["velocity"] = float(np.sqrt(num / den))
    pg, po = vmean(gpu["p"]), vmean(f["p"])
    err["p"] = float(np.linalg.norm(pg - po) / np.linalg.norm(po))
    return {"seconds": sec, "oracle_cycles": it_o, "gpu_cycles": it_g, "err": err, "dt": dt}


def cfl_dt(g, f, cfl):
    """calcdt (Routines.F90:221-240) on host arrays."""
    u, v, w = (f[k] for k in ("u", "v", "w"))
    au = np.abs(0.5 * (u[1:-1, 1:-1, 1:-1] + u[:-2, 1:-1, 1:-1])) * g.x.rdxc[1:-1, None, None]
    aw = np.abs(0.5 * (w[1:-1, 1:-1, 1:-1] + w[1:-1, 1:-1, :-2])) * g.z.rdxc[None, None, 1:-1]
    av = np.abs(0.5 * (v[1:-1, 1:-1, 1:-1] + v[1:-1, :-2, 1:-1])) * g.y.rdxc[None, 1:-1, None]
    return cfl / float((au + aw + av).max())


def cpu_sample_poisson(workload, threads):
    """One whole pressure solve of the workload on the host cores: the
    oracle restatement, FP64, the reference's red-black point Gauss-Seidel
    with full coarsening, from phi0 = 0 to a true relative residual of
    1e-10.  Returns (seconds, cycles, interior cells)."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from anelastic_solve_b200 import abi
    from anelastic_solve_b200 import grid as G
    from oracle.pyoracle import OracleMG

    kind, n, lv, phys = WORKLOADS[workload]
    g = G.shear_layer_grid(*n, stretched=True)
    fF = np.asfortranarray(poisson_rhs(g).T)
    o = OracleMG(g, mg_params(lv, abi.PREC_FP64, smoother="rbpgs"))
    phi = np.zeros(g.ghosted, order="F")
    t = time.perf_counter()
    it, _ = o.solve(phi, fF.copy(order="F"))
    return time.perf_counter() - t, it, g.x.n * g.y.n * g.z.n


# ------------------------------------------------------------ ours: serve
SERVE_SIZES = [(32, 32, 32), (64, 64, 64), (96, 48, 96), (128, 128, 128), (192, 96, 192),
               (256, 256, 256)]


def levels_of(n):
    """Level count per direction: halve while the coarse size stays >= 2."""
    L = 1
    while n % 2 == 0 and n // 2 >= 2:
        n //= 2
        L += 1
    return L


def serve_stream(n_req, seed, rate):
    """Seeded request stream: Poisson arrivals at `rate`/s, grid uniform
    over SERVE_SIZES, Ri ~ U[0.05, 0.3], Re log-uniform on [500, 4000], a
    perturbation seed per request."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n_req))
    size = rng.integers(0, len(SERVE_SIZES), n_req)
    Ri = rng.uniform(0.05, 0.3, n_req)
    Re = np.exp(rng.uniform(math.log(500.0), math.log(4000.0), n_req))
    sd = rng.integers(1, 2 ** 31 - 1, n_req)
    return [dict(t=float(t[q]), size=SERVE_SIZES[int(size[q])], Ri=float(Ri[q]), Re=float(Re[q]),
                 seed=int(sd[q])) for q in range(n_req)]


def run_serve(args, rank, world, local_rank):
    import torch

    from anelastic_solve_b200 import _lib, abi
    from anelastic_solve_b200 import grid as G
    from anelastic_solve_b200.serve import ServeEngine

    torch.cuda.set_device(local_rank)
    grids = {n: G.shear_layer_grid(*n, stretched=True) for n in SERVE_SIZES}
    mgp = {}
    for n in SERVE_SIZES:
        SMOOTHER.update(smoother=args.smoother, pre=args.pre, post=args.post)
        mgp[n] = mg_params(tuple(levels_of(v) for v in n),
                           abi.PREC_MIXED if args.prec == "mixed" else abi.PREC_FP64)

    def nsp(Re, Ri):
        return abi.make_ns_params(Re=Re, Pr=1.0, g=-Ri, cfl=0.5, dtmax=1e9, ew=1, scal1_on=0)

    e = ServeEngine(int(args.budget_gb * 1e9), max_active=args.workers, device=local_rank)
    # warm-up: one member of every size (contexts of every bucket created)
    for n in SERVE_SIZES:
        e.submit(grids[n], mgp[n], nsp(1000.0, 0.12), nsteps=1, seed=1)
    e.drain()
    e.poll(cap=1024)
    reqs = serve_stream(args.requests, 7 + rank, args.rate)
    res = []
    launches0 = _lib.launch_count()
    with ClockSampler(local_rank) as clk:
        t0 = time.perf_counter()
        for r in reqs:
            while True:
                now = time.perf_counter() - t0
                if now >= r["t"]:
                    break
                res += e.poll(wait_ms=max(1, int(1000 * (r["t"] - now))))
            e.submit(grids[r["size"]], mgp[r["size"]], nsp(r["Re"], r["Ri"]), nsteps=args.serve_steps,
                     seed=r["seed"], amp=1e-3)
        e.drain()
        t1 = time.perf_counter()
        while len(res) < len(reqs):
            res += e.poll(wait_ms=100, cap=1024)
    st = e.stats()
    e.close()
    ok = [x for x in res if x["status"] == abi.OK]
    lat = np.array([x["latency_ms"] for x in ok])
    cu = float(sum(x["cells"] * x["nsteps"] for x in ok))
    meta = np.array([sum(n[0] * n[1] * n[2] for n in [r["size"]]) for r in reqs])
    out = {"makespan_s": t1 - t0, "cell_updates": cu, "ok": len(ok), "failed": len(res) - len(ok),
           "lat": lat, "queue": np.array([x["queue_ms"] for x in ok]),
           "run": np.array([x["run_ms"] for x in ok]), "stats": st, "clocks": clk.summary(),
           "launches": _lib.launch_count() - launches0,
           "h2d": int(sum(8 * 6 * (2 * (r["size"][0] + r["size"][1] + r["size"][2]) + 6) for r in reqs)),
           "d2h": 8 * 8 * len(reqs), "arrival_span_s": reqs[-1]["t"], "mean_cells": float(meta.mean())}
    (out["makespan_s"],), (out["cell_updates"],) = combine_ranks(
        world, torch.device("cuda", local_rank), maxes=(out["makespan_s"],), sums=(out["cell_updates"],))
    return out


def main_serve(args, rank, world, local_rank, threads):
    sizes = "{" + ", ".join("x".join(map(str, n)) for n in SERVE_SIZES) + "}"
    metric = "cell-updates/s (ensemble serving, aggregate)"
    unit = "cell-updates/s"
    config = {"workload": f"serving stream: {args.requests} shear-layer requests, Poisson arrivals at "
                          f"{args.rate:g}/s, grid uniform over {sizes}, Ri~U[0.05,0.3], Re "
                          f"log-uniform [500,4000], {args.serve_steps} RK3 steps each",
              "hbm_budget_gb": args.budget_gb, "workers": args.workers,
              "mg": f"{args.smoother.upper()} V({args.pre},{args.post}){fine_note(args)}, metric, {args.prec}, to 1e-10",
              "parallelism": f"replicas x{world}", "l2": "mixed sizes (32^3 .. 256^3)"}
    if args.impl == "reference":
        if rank != 0:
            return
        c = cpu_reference_step("dns64", threads)
        t, N = c["seconds"], c["cells"]
        value = N / t
        sample = (f"one 64^3 member, oracle restatement: one steady RK3 step ({t:.2f} s, "
                  f"MG V-cycles per sub-step {c['cycles']}) after the initial projection and one "
                  f"warm-up step; members run one after another")
        line = {"impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": 0,
                "steps": 1, "warmup": 1, "requested_steps": args.requests, "ms_per_step": t * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": dict(config, mg="RBPGS V(2,2), metric, fp64 (host)"),
                "cpu_baseline": {"value": value, "unit": unit, "cores": threads, "kind": "port",
                                 "sample": sample},
                "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))
    r = run_serve(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank != 0:
        return
    value = r["cell_updates"] / r["makespan_s"]
    pct = lambda a, q: float(np.percentile(a, q)) if len(a) else None  # noqa: E731
    cpu = None
    if not args.no_cpu:
        c = cpu_reference_step("dns64", threads)
        cpu = {"value": c["cells"] / c["seconds"], "unit": unit, "cores": threads, "kind": "port",
               "sample": f"one 64^3 member, oracle restatement (FP64 RBPGS): one steady RK3 step "
                         f"({c['seconds']:.2f} s, MG V-cycles per sub-step {c['cycles']}) after the "
                         f"initial projection and one warm-up step"}
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.requests,
            "warmup": len(SERVE_SIZES), "ms_per_step": 1e3 * r["makespan_s"] / max(1, args.requests),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (MG f32-in-f64)" if args.prec == "mixed" else "f64", "data": "synthetic",
            "config": config,
            "latency_ms": {"p50": pct(r["lat"], 50), "p99": pct(r["lat"], 99),
                           "queue_p50": pct(r["queue"], 50), "queue_p99": pct(r["queue"], 99),
                           "run_p50": pct(r["run"], 50), "run_p99": pct(r["run"], 99)},
            "requests_ok": r["ok"], "requests_failed": r["failed"],
            "makespan_s": r["makespan_s"], "arrival_span_s": r["arrival_span_s"],
            "peak_active": r["stats"]["peak_active"], "peak_bytes": r["stats"]["peak_bytes"],
            "contexts": r["stats"]["contexts"],
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": r["h2d"] // max(1, args.requests),
                    "d2h_bytes_per_step": r["d2h"] // max(1, args.requests),
                    "note": "serving is timed end to end on the host clock: submit through the "
                            "C-ABI (grid copied in, state generated on the device from the seed) "
                            "to the member's result record"},
            "roofline": None, "cpu_baseline": cpu, "clocks": r["clocks"],
            "gpu_launches": r["launches"]}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="dns", choices=sorted(WORKLOADS))
    ap.add_argument("--prec", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--smoother", default="zline", choices=["rbpgs", "zline"],
                    help="zline: z-line GS with x/y semi-coarsening (default); rbpgs: the "
                         "reference's red-black point GS with full coarsening")
    ap.add_argument("--pre", type=int, default=2, help="pre-smoothing sweeps per level")
    ap.add_argument("--post", type=int, default=2, help="post-smoothing sweeps per level")
    ap.add_argument("--fine-pre", type=int, default=None, help="pre-smoothing sweeps on the finest level")
    ap.add_argument("--fine-post", type=int, default=None, help="post-smoothing sweeps on the finest level")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 multigrid companion")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--pguess", type=int, default=0, choices=[0, 1],
                    help="mixed runs: 1 = each sub-step's pressure solve starts from the linear "
                         "extrapolation of that sub-step's last two solutions; 0 = from the current "
                         "p, as the reference (default)")
    ap.add_argument("--members", type=int, default=1,
                    help="poisson workloads: also time this many solves one by one and batched")
    ap.add_argument("--requests", type=int, default=2000, help="serve: requests in the stream")
    ap.add_argument("--rate", type=float, default=50.0, help="serve: arrivals per second")
    ap.add_argument("--serve-steps", type=int, default=10, help="serve: RK3 steps per request")
    ap.add_argument("--workers", type=int, default=8, help="serve: members in flight")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serve: HBM budget (GB)")
    ap.add_argument("--diag", action="store_true",
                    help="dns/les: also time the per-step plane statistics (outside the timed steps)")
    args = ap.parse_args()
    SMOOTHER.update(smoother=args.smoother, pre=args.pre, post=args.post, fine_pre=args.fine_pre,
                    fine_post=args.fine_post)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if WORKLOADS[args.workload][0] == "serve":
        main_serve(args, rank, world, local_rank, os.cpu_count() or 1)
        return
    kind, n, lv, phys = WORKLOADS[args.workload]
    nx, ny, nz = n
    field_mb = (nx + 2) * (ny + 2) * (nz + 2) * 8 / 1e6
    l2note = (f"inputs larger than L2 ({field_mb:.0f} MB per FP64 field)" if field_mb > 126
              else f"small ({field_mb:.1f} MB per FP64 field)")
    if kind == "dns":
        metric = "cell-updates/s (RK3 step incl. 3 projections)"
        unit = "cell-updates/s"
        if phys.get("dsm"):
            model = "LES (DSM/DSMrho/DSMscal1 every step, test ratio sqrt(6), x-y averaged)"
        else:
            model = "LES (SSM, Cs^2=0.0289, Pr_sgs=0.7)" if phys.get("les") else "DNS"
        config = {"workload": f"{model} shear layer {nx}x{ny}x{nz}: Re={phys['Re']:g}, Pr=1, "
                              f"Ri={-phys['g']:g}, amp {phys['amp']:g}, CFL {phys['cfl']:g}, "
                              f"MG to ||f-A p||/||f|| <= {TOL:g} each sub-step",
                  "grid": [nx, ny, nz], "mg_levels": list(lv), "mg": f"{args.smoother.upper()} V({args.pre},{args.post}){fine_note(args)}, metric, {args.prec}",
                  "p_guess": ("2 p(n-1) - p(n-2) per sub-step (extension)"
                              if args.pguess and args.prec == "mixed" else "current p (reference)"),
                  "ew": 1, "scal1": "off (zero)", "parallelism": f"replicas x{args.gpus}",
                  "l2": l2note}
    else:
        metric = "MG solve throughput to 1e-10 relative residual (cell-solves/s)"
        unit = "cell-solves/s"
        config = {"workload": f"pressure-Poisson solve {nx}x{ny}x{nz}, tanh-stretched z, periodic "
                              f"x/y, Neumann z, to ||f-A phi||/||f|| <= {TOL:g} from phi0 = 0",
                  "grid": [nx, ny, nz], "mg_levels": list(lv), "mg": f"{args.smoother.upper()} V({args.pre},{args.post}){fine_note(args)}, metric, {args.prec}",
                  "parallelism": f"replicas x{args.gpus}",
                  "l2": l2note}
    threads = os.cpu_count() or 1
    if args.impl == "reference":
        if rank != 0:
            return
        # the reference's own algorithm: red-black point GS, full coarsening
        config = dict(config, mg=f"RBPGS V(2,2), metric, fp64 (the reference's algorithm on the host)")
        if kind == "dns":
            c = cpu_reference_step(args.workload, threads)
            t, N = c["seconds"], c["cells"]
            value = N / t
            sample = (f"oracle restatement at full size: one steady RK3 step ({t:.1f} s, MG V-cycles "
                      f"per sub-step {c['cycles']}) after the untimed initial projection and one "
                      f"warm-up step (cycles {c['warm_cycles']})")
            ms, steps, warm = t * 1e3, 1, 1
        else:
            t, it, N = cpu_sample_poisson(args.workload, threads)
            value = N / t
            sample = f"oracle restatement at full size: one whole solve from phi0 = 0 ({t:.1f} s, {it} V-cycles)"
            ms, steps, warm = t * 1e3, 1, 0
        line = {"impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": 0,
                "steps": steps, "warmup": warm, "requested_steps": args.steps, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": config,
                "cpu_baseline": {"value": value, "unit": unit, "cores": threads, "kind": "port",
                                 "sample": sample},
                "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    r = run_dns(args, rank, world, local_rank) if kind == "dns" else run_poisson(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank != 0:
        return
    peak, peak_kind = load_peaks()
    N = r["N"]
    value = weak_value(world, N, r["ms_step"])
    # smoother bytes per cell and launch (one colour): reads of the other
    # colour's phi (the neighbours, half the cells), f of this colour and
    # the write of this colour's phi -> 12 B FP64, 6 B FP32.  The FP64
    # z-line (Thomas) kernel also writes and re-reads the elimination values
    # in place (+4 B); the FP32 partitioned z-line kernel keeps them on chip.
    zl = args.smoother == "zline"
    bpc = 6.0 if args.prec == "mixed" else (16.0 if zl else 12.0)
    if zl and args.prec == "mixed" and nz % 32 == 0 and nz // 32 in (2, 3, 4, 6, 8, 12, 16):
        # the column-layout FP32 cycle (one warp per z-line)
        kernel = f"k_col_sweep<{nz // 32}>"
    elif zl and args.prec == "mixed" and nz % 16 == 0 and 32 <= nz <= 512:
        kernel = "k_zline_seg<float,16,32>"
    else:
        kname = "k_zline" if zl else "k_rb_sweep"
        kernel = f"{kname}<float>" if args.prec == "mixed" else f"{kname}<double>"
    roof = None
    if r["sweeps"]:
        t_launch = r["sweep_ms"] / r["sweeps"] / 1e3
        achieved = bpc * N / t_launch / 1e9
        roof = {"bound": "hbm", "kernel": kernel, "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": load_traffic(f"{args.workload}:{kernel}"),
                "peak_kind": f"{peak_kind} hbm_gbs", "algorithmic_bytes_per_launch": bpc * N,
                "mean_launch_ms": round(t_launch * 1e3, 4),
                "share_note": "finest-level smoother launches only; share of step time in profiles/"}
    cpu = None
    if not args.no_cpu:
        if kind == "dns" and "oracle_leg" in r:
            c = r["oracle_leg"]
            cpu = {"value": N / (3.0 * c["seconds"]), "unit": unit, "cores": threads, "kind": "port",
                   "sample": f"one steady RK3 sub-step at full size from this run's state after its "
                             f"timed steps: oracle restatement, FP64 RBPGS ({c['seconds']:.1f} s, "
                             f"{c['oracle_cycles']} MG V-cycles), x3 per step"}
        elif kind == "poisson":
            t, it, _ = cpu_sample_poisson(args.workload, threads)
            cpu = {"value": N / t, "unit": unit, "cores": threads, "kind": "port",
                   "sample": f"one whole FP64 RBPGS solve of the oracle restatement at full size "
                             f"({t:.1f} s, {it} V-cycles)"}
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (MG f32-in-f64)" if args.prec == "mixed" else "f64", "data": "synthetic",
            "config": config}
    if kind == "dns":
        line["mg_ms_per_step"] = round(r["mg_ms_step"], 3)
        if r.get("diag_ms_step") is not None:
            line["diag_ms_per_step"] = round(r["diag_ms_step"], 3)
        line["mg_iters_last_step"] = r["mg_iters"][-1]
        line["dt"] = r["dt"]
        line["max_div"] = r["max_div"]
        line["div_bound"] = 1e-10 * r["umax"] / r["dzmin"]
        if "mg_cold" in r:
            line["mg_solve_ms"] = r["mg_cold"]
        if "fp64_plain" in r:
            fp = r["fp64_plain"]
            line["fp64_plain"] = {"ms_per_step": round(fp["ms_per_step"], 3),
                                  "mg_ms_per_step": round(fp["mg_ms_per_step"], 3),
                                  "mg_iters": fp["mg_iters"], "steps": fp["steps"],
                                  "mg": "RBPGS V(2,2), metric, fp64, full coarsening (the one-for-one "
                                        "mg_solver replacement)",
                                  "speedup_of_this_run": round(fp["ms_per_step"] / r["ms_step"], 3)}
        if "oracle_leg" in r:
            c = r["oracle_leg"]
            line["err_vs_fp64_oracle"] = dict(
                {k: float(f"{v:.3e}") for k, v in c["err"].items()},
                sample="one RK3 sub-step at full size from this run's state after its timed steps: "
                       "this run's multigrid on the GPU vs the FP64 oracle (RBPGS) on the host, both "
                       "to 1e-10; relative L2 over the interior, p after removing the volume mean",
                gpu_cycles=c["gpu_cycles"], oracle_cycles=c["oracle_cycles"])
    else:
        line["mg_iters"] = r["iters"][-1]
        line["resid"] = r["resid"]
        if "batched" in r:
            line["batched"] = r["batched"]
    if "e2e_ms" in r:
        line["e2e"] = {"value": world * N / (r["e2e_ms"] / 1e3), "unit": unit,
                       "h2d_bytes_per_step": r["bytes_io"][0], "d2h_bytes_per_step": r["bytes_io"][1],
                       "ms_per_step": r["e2e_ms"]}
    line.update({"roofline": roof, "cpu_baseline": cpu, "clocks": r["clocks"],
                 "gpu_launches": r["launches"], "tuning": r.get("tuning")})
    print(json.dumps(line))


if __name__ == "__main__":
    main()
