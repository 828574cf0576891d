#!/usr/bin/env python
"""Benchmark of the B200 path: time-steps/s (and p-solve ms) with every linear solve
taken to a 1e-8 true relative residual, on one GPU per rank.

Default workload: 3-D lid-driven cavity, 128^3 cells, Re = 400, PISO (1 inner iteration,
2 pressure corrections), central convection, Jacobi-BiCGStab momentum, Jacobi-PCG
pressure correction, dt = 1e-3, synthetic (no dataset involved), plain FP64.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--workload c2|c1|c3|c5] [--p-form fp64|mixed|...] [--size n]

One JSON line on rank 0.  --impl reference times the CPU restatement of the reference
path (the reference itself cannot be built here: it needs MPI, PETSc and Boost) on the
host cores, on the same workload.
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

_ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, _ROOT)

import numpy as np  # noqa: E402

from caffe_old_b200 import cases as C  # noqa: E402

HBM_FALLBACK = 6650.0
# algorithmic bytes per matrix row and Krylov iteration of the dominant kernel
# (fused Jacobi-PCG iteration: SpMV 72 + preconditioner 24 + x/r/p updates 64 + dot 8)
PCG_BYTES_PER_ROW = 168.0
BICGSTAB_BYTES_PER_ROW = 344.0


def peaks():
    path = os.path.join(_ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK, "fallback"


def workload(name: str, size: int | None, p_form: str):
    if name == "c1":
        nodes, spec, _ = C.config1_cavity2d(n=size or 64)
        label = f"simple_lid_cavity2d_{size or 64}^2_re100_upwind_jacobi_bicgstab"
    elif name == "c2":
        n = size or 128
        nodes, spec, _ = C.config2_cavity3d(n=n)
        label = f"piso_lid_cavity3d_{n}^3_re400_central_jacobi_pcg"
    elif name == "c3":
        n = size or 128
        nodes, spec, _ = C.config3_skewed(n=n, p_form=p_form)
        label = f"piso_skewed_cavity3d_{n}^3_re400_nonorth"
    elif name == "c5":
        dims = (384, 256, 256) if not size else (size * 3 // 2, size, size)
        nodes, spec, _ = C.config5_sphere(dims=dims, p_form=p_form)
        label = f"ibpiso_sphere_{dims[0]}x{dims[1]}x{dims[2]}_re300"
    else:
        raise SystemExit(f"unknown workload {name}")
    spec = spec.replace(p_form=p_form)
    return nodes, spec, label + f"_{p_form}"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def cpu_baseline(nodes, spec, steps: int = 1) -> dict:
    """The CPU restatement of the reference path (oracle) on the host cores, same workload."""
    from oracle import oracle as O
    O.build()
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    s = O.OracleSolver(nodes, spec)
    t = time.perf_counter()
    for _ in range(steps):
        s.solve()
    dt = time.perf_counter() - t
    st = s.stats()
    s.close()
    return {"value": steps / dt, "unit": "time-steps/s", "cores": threads, "kind": "port",
            "sample": f"{steps} time step(s) from rest of the same workload, oracle restatement (C++ -O2, OpenMP), "
                      f"{dt:.1f} s, p' iterations in the last step {int(st['p_iters_total'])}"}


def run_reference(args, world, rank, pg):
    if rank != 0:
        return
    nodes, spec, label = workload(args.workload, args.size, "fp64")
    from oracle import oracle as O
    O.build()
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    s = O.OracleSolver(nodes, spec)
    budget = float(os.environ.get("CAFFE_REF_BUDGET_S", "150"))
    for _ in range(min(args.warmup, 1)):
        s.solve()
    times = []
    t_all = time.perf_counter()
    for _ in range(args.steps):
        t = time.perf_counter()
        s.solve()
        times.append(time.perf_counter() - t)
        if time.perf_counter() - t_all > budget:
            break
    total = sum(times)
    value = len(times) / total
    line = {
        "impl": "reference", "metric": "time-steps/s at 1e-8 true relative residual", "value": value,
        "unit": "time-steps/s", "n_gpus": args.gpus, "steps": len(times), "warmup": min(args.warmup, 1),
        "ms_per_step": 1e3 * total / len(times), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "config": {"workload": label, "cells": int(np.prod([d - 1 for d in nodes.shape[:3]]))},
        "cpu_baseline": {"value": value, "unit": "time-steps/s", "cores": threads, "kind": "port",
                         "sample": f"{len(times)} of {args.steps} requested steps (time-bounded at {budget:.0f} s), "
                                   "CPU restatement of the reference path; the reference binary needs MPI, PETSc and Boost, "
                                   "absent on this image"},
        "e2e": {"value": value, "unit": "time-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_b200(args, world, rank, local, pg):
    import torch
    from caffe_old_b200.solver import make_solver
    torch.cuda.set_device(local)
    nodes, spec, label = workload(args.workload, args.size, args.p_form)
    dev = make_solver(nodes, spec, device=local)
    N = dev.ncells
    stream = torch.cuda.ExternalStream(dev.stream, device=local)

    for _ in range(args.warmup):
        dev.solve()
    dev.synchronize()
    barrier(pg)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    p_ms, p_iters, p_solves, mom_ms, mom_iters, status = 0.0, 0, 0, 0.0, 0, 0
    conts = []
    t0.record(stream)
    for _ in range(args.steps):
        conts.append(dev.solve())
        st = dev.last_stats
        p_ms += st["p_ms"]; p_iters += st["p_iters_total"]; p_solves += st["p_solves"]
        mom_ms += st["mom_ms"]; mom_iters += sum(st["mom_iters"]); status = max(status, st["status"])
    t1.record(stream)
    t1.synchronize()
    clocks = sampler.stop()
    elapsed_ms = t0.elapsed_time(t1)
    elapsed_ms = max_over_ranks(pg, elapsed_ms)
    ms_per_step = elapsed_ms / args.steps
    value = world * args.steps / (elapsed_ms / 1e3)

    # roofline of the dominant kernel: the pressure-correction Krylov solve
    hbm, peak_kind = peaks()
    per_row = PCG_BYTES_PER_ROW if spec.p_method == "cg_jacobi" else BICGSTAB_BYTES_PER_ROW
    rows = N - (dev.last_stats.get("n_ghost", 0) * 0)
    bytes_p = per_row * rows * p_iters
    achieved = bytes_p / (p_ms / 1e3) / 1e9 if p_ms > 0 else None
    roofline = {"bound": "hbm", "kernel": "cg_kernel (pressure-correction Jacobi-PCG, persistent)"
                if spec.p_method == "cg_jacobi" else "bicgstab_kernel (pressure correction)",
                "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": (achieved / hbm) if achieved else None,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "traffic": None, "bytes_per_row_iteration": per_row,
                "launch_ms_avg": p_ms / max(p_solves, 1), "iterations_per_launch": p_iters / max(p_solves, 1)}

    # end to end through the C ABI with host buffers: per step, upload the solver state
    # (u, p, face mass fluxes) from pinned memory, solve, read u and p back
    e2e = None
    if not args.no_e2e:
        sizes = {nm: dev.size_of(nm) for nm in ("u", "p", "massFlowI", "massFlowJ", "massFlowK")}
        host = {nm: torch.empty(n, dtype=torch.float64, pin_memory=True) for nm, n in sizes.items()}
        for nm in sizes:
            dev.get_to_ptr(nm, host[nm].data_ptr(), sizes[nm])
        up = ("u", "p", "massFlowI", "massFlowJ", "massFlowK")
        down = ("u", "p")
        dev.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        ke = args.steps
        e0.record(stream)
        for _ in range(ke):
            for nm in up:
                dev.set_from_ptr(nm, host[nm].data_ptr(), sizes[nm])
            dev.solve()
            for nm in down:
                dev.get_to_ptr(nm, host[nm].data_ptr(), sizes[nm])
        e1.record(stream)
        e1.synchronize()
        e_ms = max_over_ranks(pg, e0.elapsed_time(e1))
        e2e = {"value": world * ke / (e_ms / 1e3), "unit": "time-steps/s",
               "h2d_bytes_per_step": 8 * sum(sizes[nm] for nm in up),
               "d2h_bytes_per_step": 8 * sum(sizes[nm] for nm in down) + 128,
               "api": "caffe_dev_array (pinned host buffers) + caffe_dev_solve, per step"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(nodes, spec.replace(p_form="fp64"), steps=1)

    launches_per_step = 3 + 2 + (6 * spec.n_pcorr if spec.kind != "simple" else 6) + 3
    if rank == 0:
        working_set = N * 8 * 60
        line = {
            "metric": "time-steps/s at 1e-8 true relative residual", "value": value, "unit": "time-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded mesh and case, no dataset)",
            "config": {"workload": label, "cells": N, "p_form": args.p_form, "parallelism": f"replicas x{world}",
                       "l2": f"inputs larger than L2: working set ~{working_set / 2**30:.1f} GiB > 126 MB"},
            "p_solve_ms": p_ms / args.steps, "momentum_solve_ms": mom_ms / args.steps,
            "p_iters_per_step": p_iters / args.steps, "mom_iters_per_step": mom_iters / args.steps,
            "continuity_last": conts[-1], "solver_status": status,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
            "gpu_launches": launches_per_step * args.steps,
        }
        print(json.dumps(line), flush=True)
    dev.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=("b200", "reference"))
    ap.add_argument("--workload", default="c2", choices=("c1", "c2", "c3", "c5"))
    ap.add_argument("--p-form", default="fp64", choices=tuple(C.P_FORMS))
    ap.add_argument("--size", type=int, default=None)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "b200":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    world, rank, local, pg = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank, pg)
        else:
            run_b200(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.barrier()
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
