#!/usr/bin/env python
"""Benchmark of the B200 hot path (one JSON line on rank 0).

Workload "poisson" (default): standalone pressure-Poisson solves on the
512x256x512 staggered shear-layer grid (domain 4pi x 2pi x 20, periodic
x/y, Neumann z walls, z tanh-stretched), right-hand side = divergence-like
seeded N(0,1) field with the volume mean removed, phi0 = 0, solved to a
true relative residual ||f - A phi||/||f|| <= 1e-10.  One step = one solve.

  value  -- cell-solves/s: interior cells x solves / device time, inputs
            resident in HBM (CUDA events on the solve stream, max over ranks)
  e2e    -- the same through the C-ABI with host (pinned) buffers: the
            host->device copy of phi0 and f and the device->host copy of
            phi are inside the timed region
  roofline -- the dominant kernel (finest-level red-black smoother):
            algorithmic bytes per launch / mean launch time (CUDA events)

--impl reference times the CPU restatement of the same algorithm (the
reference cannot be built here) on the host cores instead.
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
    # name: (nx, ny, nz, levels)
    "poisson": (512, 256, 512, (9, 8, 9)),
    "poisson256": (256, 256, 256, (8, 8, 8)),
    "poisson_small": (64, 32, 64, (6, 5, 6)),
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


def make_problem(workload):
    from anelastic_solve_b200 import grid as G

    nx, ny, nz, lv = WORKLOADS[workload]
    g = G.shear_layer_grid(nx, ny, nz, stretched=True)
    rng = np.random.default_rng(1)
    f = rng.standard_normal(g.ghosted[::-1])  # (Z,Y,X) C-order == Fortran (X,Y,Z)
    vol = (g.z.dxc[1:-1, None, None] * g.y.dxc[None, 1:-1, None] * g.x.dxc[None, None, 1:-1])
    inner = f[1:-1, 1:-1, 1:-1]
    inner -= (inner * vol).sum() / vol.sum()
    return g, lv, f


def mg_params(lv, precision, mode):
    from anelastic_solve_b200 import abi

    return abi.make_mg_params(lv, maxcy=400, tolmax=TOL, pre=2, post=2, tbc=(0, 1, 0, 1, 0, 0),
                              precision=precision, mode=mode, stop=abi.STOP_RESID)


# ----------------------------------------------------------------- ours
def run_ours(args, rank, world, local_rank):
    import torch

    from anelastic_solve_b200 import _lib, abi
    from anelastic_solve_b200.mg import MGSolver

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    g, lv, f = make_problem(args.workload)
    N = g.x.n * g.y.n * g.z.n
    prec = abi.PREC_MIXED if args.prec == "mixed" else abi.PREC_FP64
    mode = abi.MODE_METRIC if args.mode == "metric" else abi.MODE_LITERAL
    s = MGSolver(g, mg_params(lv, prec, mode), device=local_rank)
    st = torch.cuda.Stream(device=dev)
    dsrc = torch.from_numpy(f).to(dev)
    dphi = torch.zeros_like(dsrc)

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    # warm-up
    with torch.cuda.stream(st):
        for _ in range(args.warmup):
            dphi.zero_()
            s.solve(dphi, dsrc, stream=st.cuda_stream)
    st.synchronize()
    # timed region (device-resident inputs)
    s.set_profiling(True)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    iters, resids, sweep_ms, sweeps = [], [], 0.0, 0
    launches0 = _lib.launch_count()
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        with torch.cuda.stream(st):
            ev0.record(st)
            for _ in range(args.steps):
                dphi.zero_()
                s.solve(dphi, dsrc, stream=st.cuda_stream)
                r = s.last_report
                iters.append(r.iter)
                resids.append(r.resid)
                sweep_ms += r.fine_sweep_ms
                sweeps += r.fine_sweeps
            ev1.record(st)
        torch.cuda.synchronize()
    barrier()
    launches = _lib.launch_count() - launches0
    s.set_profiling(False)
    ms = ev0.elapsed_time(ev1)
    # e2e: reference-facing call with host buffers (pinned), copies inside
    if args.no_e2e:
        return {"ms_step": ms / args.steps, "e2e_ms": float("nan"), "N": N, "iters": iters,
                "resids": resids, "sweep_ms": sweep_ms, "sweeps": sweeps, "launches": launches,
                "clocks": clk.summary(), "bytes_io": (2 * dsrc.numel() * 8, dsrc.numel() * 8)}
    ph = torch.zeros(dsrc.shape, dtype=torch.float64).pin_memory()
    fh = torch.from_numpy(f).pin_memory()
    phn = np.asfortranarray(ph.numpy().T)
    fhn = np.asfortranarray(fh.numpy().T)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(st):
        s.solve(phn, fhn, stream=st.cuda_stream)  # warm
        st.synchronize()
        e0.record(st)
        for _ in range(max(1, args.steps // 2)):
            phn[...] = 0.0
            s.solve(phn, fhn, stream=st.cuda_stream)
        e1.record(st)
    torch.cuda.synchronize()
    e2e_steps = max(1, args.steps // 2)
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    ms_step = ms / args.steps
    # max over ranks
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([ms_step, e2e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_step, e2e_ms = float(t[0]), float(t[1])
    out = {
        "ms_step": ms_step, "e2e_ms": e2e_ms, "N": N, "iters": iters, "resids": resids,
        "sweep_ms": sweep_ms, "sweeps": sweeps, "launches": launches,
        "clocks": clk.summary(), "bytes_io": (2 * dsrc.numel() * 8, dsrc.numel() * 8),
    }
    # FP64 companion solve (mixed vs FP64 pair of the metric), rank 0 only
    if rank == 0 and prec == abi.PREC_MIXED and not args.no_fp64:
        s64 = MGSolver(g, mg_params(lv, abi.PREC_FP64, mode), device=local_rank)
        with torch.cuda.stream(st):
            dphi.zero_()
            s64.solve(dphi, dsrc, stream=st.cuda_stream)
            dphi.zero_()
            s64.solve(dphi, dsrc, stream=st.cuda_stream)
        torch.cuda.synchronize()
        out["fp64"] = {"ms": s64.last_report.ms, "iter": s64.last_report.iter,
                       "resid": s64.last_report.resid}
        s64.close()
    s.close()
    return out


def cpu_sample(workload, mode, threads):
    """One FP64 V-cycle of the oracle restatement on the host cores, at the
    full workload size; returns seconds per V-cycle."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from anelastic_solve_b200 import abi
    from oracle.pyoracle import OracleMG

    g, lv, f = make_problem(workload)
    fF = np.asfortranarray(f.T)
    p = mg_params(lv, abi.PREC_FP64, abi.MODE_METRIC if mode == "metric" else abi.MODE_LITERAL)
    p.maxcy = 1
    p.tolmax = 0.0
    o = OracleMG(g, p)
    phi = np.zeros(g.ghosted, order="F")
    o.solve(phi, fF.copy(order="F"))  # warm (first touch)
    t = time.perf_counter()
    o.solve(phi, fF.copy(order="F"))
    return time.perf_counter() - t, g.x.n * g.y.n * g.z.n


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="poisson", choices=sorted(WORKLOADS))
    ap.add_argument("--prec", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--mode", default="metric", choices=["metric", "literal"])
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    nx, ny, nz, lv = WORKLOADS[args.workload]
    config = {"workload": f"pressure-Poisson solve {nx}x{ny}x{nz}, tanh-stretched z, periodic x/y, "
                          f"Neumann z, to ||f-A phi||/||f|| <= {TOL:g}",
              "grid": [nx, ny, nz], "mg_levels": list(lv), "smoother": "RBPGS V(2,2)",
              "mode": args.mode, "precision": args.prec,
              "parallelism": f"replicas x{args.gpus}",
              "l2": "inputs larger than L2 (545 MB per FP64 field)" if args.workload == "poisson"
              else "small workload"}
    metric = "MG solve throughput to 1e-10 relative residual (cell-solves/s)"
    if args.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        sec_cyc, N = cpu_sample(args.workload, args.mode, threads)
        cyc = FP64_CYCLES.get((args.workload, args.mode))
        steps = []
        for _ in range(args.warmup + args.steps):
            t, _ = cpu_sample(args.workload, args.mode, threads)
            steps.append(t)
        sec_cyc = float(np.mean(steps[args.warmup:]))
        value = N / (sec_cyc * cyc) if cyc else None
        line = {"impl": "reference", "metric": metric, "value": value, "unit": "cell-solves/s",
                "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": sec_cyc * cyc * 1e3 if cyc else None, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": config,
                "cpu_baseline": {"value": value, "unit": "cell-solves/s", "cores": threads,
                                 "kind": "port",
                                 "sample": f"1 FP64 V-cycle of the oracle restatement per step at "
                                           f"full size, x {cyc} V-cycles (the FP64 cycle count of "
                                           f"this workload)"},
                "e2e": {"value": value, "unit": "cell-solves/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    r = run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank != 0:
        return
    peak, peak_kind = load_peaks()
    N = r["N"]
    value = world * N / (r["ms_step"] / 1e3)
    e2e_value = world * N / (r["e2e_ms"] / 1e3)
    # roofline of the finest-level smoother: one colour per launch reads phi
    # (8 or 4 B: the neighbours), f (half the cells) and writes half the
    # cells -> 12 B/cell FP64, 6 B/cell FP32, per launch
    bpc = 6.0 if args.prec == "mixed" else 12.0
    kernel = "k_rb_sweep<float>" if args.prec == "mixed" else "k_rb_sweep<double>"
    roof = None
    if r["sweeps"]:
        t_launch = r["sweep_ms"] / r["sweeps"] / 1e3
        achieved = bpc * N / t_launch / 1e9
        traffic = load_traffic(f"{args.workload}:{kernel}")
        roof = {"bound": "hbm", "kernel": kernel, "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                "peak_kind": f"{peak_kind} (hbm_gbs)", "algorithmic_bytes_per_launch": bpc * N,
                "mean_launch_ms": round(t_launch * 1e3, 4)}
    cpu = None
    if not args.no_cpu:
        threads = os.cpu_count() or 1
        sec_cyc, _ = cpu_sample(args.workload, args.mode, threads)
        cyc = FP64_CYCLES.get((args.workload, args.mode)) or (r.get("fp64") or {}).get("iter")
        if cyc:
            cpu = {"value": N / (sec_cyc * cyc), "unit": "cell-solves/s", "cores": threads,
                   "kind": "port",
                   "sample": f"1 FP64 V-cycle of the oracle restatement at full size "
                             f"({sec_cyc:.2f} s) x {cyc} V-cycles"}
    line = {
        "metric": metric, "value": value, "unit": "cell-solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32-in-f64" if args.prec == "mixed" else "f64", "data": "synthetic",
        "config": config,
        "mg_solve_ms": {args.prec: r["ms_step"], **({"fp64": r["fp64"]["ms"]} if "fp64" in r else {})},
        "mg_iters": {args.prec: r["iters"][-1], **({"fp64": r["fp64"]["iter"]} if "fp64" in r else {})},
        "resid": max(r["resids"]),
        "e2e": {"value": e2e_value, "unit": "cell-solves/s",
                "h2d_bytes_per_step": r["bytes_io"][0], "d2h_bytes_per_step": r["bytes_io"][1],
                "ms_per_step": r["e2e_ms"]},
        "roofline": roof, "cpu_baseline": cpu, "clocks": r["clocks"],
        "gpu_launches": r["launches"],
    }
    print(json.dumps(line))


# FP64 V-cycles of the oracle/GPU FP64 algorithm (bit-identical) to reach
# the 1e-10 true residual on each workload; measured on the GPU path.
FP64_CYCLES = {}

if __name__ == "__main__":
    main()
