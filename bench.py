#!/usr/bin/env python
"""Benchmark of the B200 path: time-steps/s and p-solve ms with every pressure-correction
solve taken to a 1e-8 true relative residual (FP64), on one GPU per rank.

Default workload: flow over an immersed-boundary sphere, 384 x 256 x 256 = 25.2M cells,
Re = 300, IB-PISO (2 inner iterations, 3 pressure corrections), dt = 2e-3, synthetic
(seeded mesh and case, no dataset), pressure correction in the learned + mixed-precision form:
FP32 flexible Krylov (FGMRES) preconditioned by the level pyramid with the trained BF16
tensor-core network, inside FP64 iterative refinement; a solve whose network stage stalls
continues with the pyramid alone (counted as a cascade), and only then with plain FP64 (counted
as a fallback).  The same steps from rest are also run with the plain FP64 pressure solve
(--compare-fp64 steps) and both are reported.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--workload c5|c2|c1|c3] [--p-form learned_mixed|fp64|mixed|learned]
                  [--precond network|levels|jacobi] [--inner auto|fcg|bicgstab|fgmres]
                  [--params file.npy] [--size n] [--compare-fp64 K]

One JSON line on rank 0.  The CPU numbers (--impl reference, and cpu_baseline in the GPU line)
time the CPU restatement of the reference path (the reference itself needs MPI, PETSc and Boost,
which this image lacks) on the host cores.  A step of the 25.2M-cell case does not fit a CPU
budget of minutes (about 57,000 FP64 Krylov iterations per step), so they time whole steps of the
same case on a smaller lattice and say so; nothing is extrapolated.  The GPU line adds the GPU on
that same smaller lattice, and a fully measured 128^3 cavity (configuration 2) on both.
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


# the CPU sample of the immersed-sphere case: the same case on a lattice of 72 x 48 x 48 cells
# (1/152 of the 25.2M cells), small enough for whole plain-FP64 steps on the host cores
CPU_SAMPLE_SIZE = 48


def sample_workload(name: str, size: int | None):
    """The same case on the smaller lattice the CPU times fully."""
    if name == "c5":
        return workload(name, CPU_SAMPLE_SIZE, "fp64")
    if name in ("c2", "c3"):
        return workload(name, max(8, (size or 128) // 4), "fp64")
    return workload(name, size or 64, "fp64")


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


def _oracle_steps(nodes, spec, steps: int, budget_s: float):
    """Whole steps of the CPU restatement (plain FP64 solves) from rest, on every host core;
    stops after `steps` or once `budget_s` is spent (at least one step)."""
    from oracle import oracle as O
    O.build()
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    s = O.OracleSolver(nodes, spec)
    times, iters = [], []
    t_all = time.perf_counter()
    for _ in range(steps):
        t = time.perf_counter()
        s.solve()
        times.append(time.perf_counter() - t)
        iters.append(int(s.stats()["p_iters_total"]))
        if time.perf_counter() - t_all > budget_s:
            break
    s.close()
    return times, iters, threads


def measured_cpu(args, steps: int, budget_s: float) -> dict:
    """The CPU restatement timed on whole steps of the same case on the smaller CPU lattice:
    measured, not scaled."""
    nodes, spec, label = sample_workload(args.workload, args.size)
    cells = int(np.prod([d - 1 for d in nodes.shape[:3]]))
    times, iters, threads = _oracle_steps(nodes, spec, steps, budget_s)
    t_step = sum(times) / len(times)
    return {"value": 1.0 / t_step, "unit": "time-steps/s", "cores": threads, "kind": "port",
            "workload": label, "cells": cells,
            "sample": f"{len(times)} whole step(s) from rest of the same case on a {nodes.shape[2]-1}x{nodes.shape[1]-1}x"
                      f"{nodes.shape[0]-1} lattice ({cells} cells), plain FP64 solves to 1e-8: {t_step:.2f} s/step, p' "
                      f"iterations/step {iters}; measured on that lattice, not scaled to the full one "
                      f"(oracle restatement, C++ -O2, OpenMP on {threads} threads)",
            "s_per_step": t_step}


def case_label(args) -> str:
    if args.workload == "c5":
        dims = (384, 256, 256) if not args.size else (args.size * 3 // 2, args.size, args.size)
        return f"ibpiso_sphere_{dims[0]}x{dims[1]}x{dims[2]}_re300_{args.p_form}"
    return workload(args.workload, args.size, args.p_form)[2]


def run_reference(args, world, rank, pg):
    """The CPU restatement of the reference path (plain FP64) on the host cores.  Rank 0 alone
    measures; the other ranks exit without work."""
    if rank != 0:
        return
    budget = float(os.environ.get("CAFFE_REF_BUDGET_S", "60"))
    cpu = measured_cpu(args, max(1, args.steps), budget)
    value = cpu["value"]
    line = {
        "impl": "reference", "metric": "time-steps/s at 1e-8 true relative residual", "value": value,
        "unit": "time-steps/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": 0,
        "ms_per_step": 1e3 / value, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": case_label(args), "reference_path": "plain FP64 (CPU restatement of the reference, oracle)",
                   "timed_lattice": cpu["workload"], "timed_cells": cpu["cells"],
                   "note": "whole steps measured on the smaller lattice of the same case; a step of the full lattice "
                           "does not fit a CPU budget of minutes; not scaled"},
        "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": value, "unit": "time-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def gpu_steps(nodes, spec, steps: int, local: int, precond_args=None) -> dict:
    """Steps from rest on the GPU, each timed on the device (the handle's own CUDA events)."""
    from caffe_old_b200.solver import make_solver
    dev = make_solver(nodes, spec, device=local)
    if precond_args is not None:
        configure_precond(dev, precond_args)
    rows = []
    for _ in range(steps):
        dev.solve()
        st = dev.last_stats
        rows.append({"step_ms": st["step_ms"], "p_iters": st["p_iters_total"], "fallbacks": st["fallbacks"],
                     "cascades": st["cascades"], "status": st["status"]})
    dev.close()
    return {"s_per_step": sum(r["step_ms"] for r in rows) / len(rows) / 1e3, "rows": rows}


def same_inputs_comparison(args, local: int, cpu: dict) -> dict:
    """GPU and CPU on the identical smaller lattice of the default case: the GPU's plain FP64 and
    learned forms against the CPU restatement's measured steps (cpu_baseline's run)."""
    nodes, spec, label = sample_workload(args.workload, args.size)
    out = {"workload": label, "cpu_s_per_step": cpu["s_per_step"]}
    fp64 = gpu_steps(nodes, spec.replace(p_form="fp64"), 3, local)
    out["gpu_fp64_s_per_step"] = fp64["s_per_step"]
    out["gpu_fp64_over_cpu_time_steps_per_s"] = cpu["s_per_step"] / fp64["s_per_step"]
    if args.p_form.startswith("learned"):
        lrn = gpu_steps(nodes, spec.replace(p_form=args.p_form), 3, local, args)
        out["gpu_learned_s_per_step"] = lrn["s_per_step"]
        out["gpu_learned_over_cpu_time_steps_per_s"] = cpu["s_per_step"] / lrn["s_per_step"]
        out["gpu_learned_rows"] = lrn["rows"]
    return out


def c2_full_line(local: int, cpu_budget_s: float) -> dict:
    """Configuration 2 (128^3 lid-driven cavity, PISO, central, Jacobi-PCG, plain FP64) measured in
    full on both: steps from rest on the GPU and on the CPU restatement, compared over the same
    steps."""
    nodes, spec, _ = C.config2_cavity3d(n=128)
    cpu_times, cpu_iters, threads = _oracle_steps(nodes, spec, 3, cpu_budget_s)
    k = len(cpu_times)
    gpu = gpu_steps(nodes, spec, max(3, k), local)
    g = [r["step_ms"] / 1e3 for r in gpu["rows"][:k]]
    c = sum(cpu_times) / k
    return {"workload": "piso_lid_cavity3d_128^3_re400_central_jacobi_pcg_fp64", "steps_from_rest": k,
            "cpu_s_per_step": c, "cpu_cores": threads, "cpu_p_iters": cpu_iters,
            "gpu_s_per_step": sum(g) / k, "gpu_p_iters": [r["p_iters"] for r in gpu["rows"][:k]],
            "gpu_over_cpu_time_steps_per_s": c / (sum(g) / k)}


# algorithmic bytes per cell and inner iteration of the learned solve (FP32 vectors, the
# level pyramid's restriction reads and the prolonged term's reads included; coarse levels
# excluded): flexible BiCGStab 170 B (two preconditioner applications), flexible CG 110 B
LEARNED_BYTES = {"bicgstab": 170.0, "fcg": 110.0}


def fgmres_bytes_per_cell(m: int) -> float:
    """Algorithmic bytes per cell of one FGMRES(m) iteration j (FP32 vectors), averaged over a full
    cycle j = 0 .. m-1: network scale of v_j 9 + restriction to level 1 9 + z_j = M(v_j) 13.5 +
    w = A z_j 24 + two classical Gram-Schmidt passes, each reading w and v_0..v_j for the dots and
    again for the update and writing w (12 (j+1) + 8) + v_(j+1) = w / h 8."""
    return 79.5 + 12.0 * (m + 1)
# DRAM bytes per cell and inner BiCGStab iteration of the fine-lattice kernels, from one ncu
# capture (dram__bytes_read.sum + dram__bytes_write.sum of the 240x160x160 case, per cell);
# traffic grows with the cell count
LEARNED_TRAFFIC_PER_CELL = {"bicgstab": 143.0}


def configure_precond(dev, args):
    from caffe_old_b200 import precond as P
    if not args.p_form.startswith("learned"):
        return None
    params = None
    if args.params:
        params = np.load(args.params).astype(np.float32)
    elif args.precond == "network":
        params = P.load_default()
        if params is None:
            params = P.identity_params(0)
    if params is not None:
        P.set_params(dev, params)
    P.set_mode(dev, args.precond)
    net_from = args.net_from if args.net_from is not None else int(P.default_info().get("net_from", 1) if not args.params else 1)
    args.net_from = net_from
    P.set_options(dev, args.inner, net_from, args.restart)
    # the network runs only on levels whose level channel it was trained on
    net_to = args.net_to if args.net_to is not None else (P.trained_last_level() if not args.params else None)
    P.set_net_levels(dev, net_from, net_to)
    args.net_to = net_to
    return params


def inner_method(spec, args):
    if args.inner != "auto":
        return args.inner
    if spec.kind != "ibpiso":
        return "fcg"
    return "fgmres" if args.precond == "network" else "bicgstab"


def run_b200(args, world, rank, local, pg):
    import torch
    from caffe_old_b200 import _lib
    from caffe_old_b200.solver import make_solver
    torch.cuda.set_device(local)
    nodes, spec, label = workload(args.workload, args.size, args.p_form)
    dev = make_solver(nodes, spec, device=local)
    configure_precond(dev, args)
    N = dev.ncells
    stream = torch.cuda.ExternalStream(dev.stream, device=local)
    per_step = []

    def record(tag):
        st = dev.last_stats
        per_step.append({"phase": tag, "p_ms": round(st["p_ms"], 2), "p_iters": st["p_iters_total"], "p_solves": st["p_solves"],
                         "fallbacks": st["fallbacks"], "cascades": st["cascades"], "net_iters": st["net_iters"],
                         "step_ms": round(st["step_ms"], 2),
                         "p_res_max": st["p_res_max"]})

    for _ in range(args.warmup):
        dev.solve()
        record("warmup")
    dev.synchronize()
    # the state the timed steps start from (every field a step reads from the one before: u, p,
    # grad p, d, the face and cell mass fluxes, p's boundary patches), kept in pinned host memory:
    # the end-to-end run below replays the same steps from it through the C ABI
    state = ("u", "p", "gradP", "d", "massFlowI", "massFlowJ", "massFlowK", "massFlow") + tuple(f"pPatch{f}" for f in range(6))
    sizes, host = {}, {}
    if not args.no_e2e:
        sizes = {nm: dev.size_of(nm) for nm in state}
        host = {nm: torch.empty(n, dtype=torch.float64, pin_memory=True) for nm, n in sizes.items()}
        for nm in state:
            dev.get_to_ptr(nm, host[nm].data_ptr(), sizes[nm])
        dev.synchronize()
    barrier(pg)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    p_ms, p_iters, p_solves, mom_ms, mom_iters, status, fallbacks, res_max = 0.0, 0, 0, 0.0, 0, 0, 0, 0.0
    cascades = net_iters = 0
    conts = []
    l0 = _lib.lib().caffe_launch_count()
    t0.record(stream)
    for _ in range(args.steps):
        conts.append(dev.solve())
        st = dev.last_stats
        record("timed")
        p_ms += st["p_ms"]; p_iters += st["p_iters_total"]; p_solves += st["p_solves"]
        mom_ms += st["mom_ms"]; mom_iters += sum(st["mom_iters"]); status = max(status, st["status"])
        fallbacks += st["fallbacks"]; res_max = max(res_max, st["p_res_max"]); cascades += st["cascades"]
        net_iters += st["net_iters"]
    t1.record(stream)
    t1.synchronize()
    launches = _lib.lib().caffe_launch_count() - l0
    clocks = sampler.stop()
    elapsed_ms = t0.elapsed_time(t1)
    elapsed_ms = max_over_ranks(pg, elapsed_ms)
    ms_per_step = elapsed_ms / args.steps
    value = world * args.steps / (elapsed_ms / 1e3)

    # roofline of the dominant kernel group: the pressure-correction Krylov iterations
    hbm, peak_kind = peaks()
    learned = args.p_form.startswith("learned")
    method = inner_method(spec, args) if learned else ("pcg" if spec.p_method == "cg_jacobi" else "bicgstab64")
    bytes_total = None
    if learned:
        per_row = LEARNED_BYTES.get(method) if method != "fgmres" else fgmres_bytes_per_cell(args.restart)
        kname = {"bicgstab": "learned inner flexible BiCGStab iteration (FP32, level pyramid)",
                 "fcg": "learned inner flexible CG iteration (FP32, level pyramid)"}.get(
            method, f"learned inner iterations: FGMRES({args.restart}) with the network (FP32, CGS2), then flexible "
                    "BiCGStab with the pyramid once the network stage hands over")
        if method == "fgmres":
            # the network stage's FGMRES iterations, then the pyramid stage's iterations after a cascade
            after = LEARNED_BYTES["bicgstab" if spec.kind == "ibpiso" else "fcg"]
            bytes_total = (per_row * net_iters + after * (p_iters - net_iters)) * N
            per_row = bytes_total / (N * p_iters) if p_iters > 0 else per_row
    else:
        per_row = PCG_BYTES_PER_ROW if method == "pcg" else BICGSTAB_BYTES_PER_ROW
        kname = "cg1_kernel (persistent Jacobi-PCG, FP64)" if method == "pcg" else "bicgstab_kernel (persistent Jacobi-BiCGStab, FP64)"
    achieved = per_row * N * p_iters / (p_ms / 1e3) / 1e9 if (p_ms > 0 and per_row) else None
    # DRAM traffic from the ncu capture of the pyramid BiCGStab iteration; with the network stage
    # it describes the iterations after the hand-over, which are most of them
    traffic_key = "bicgstab" if (method == "fgmres" and spec.kind == "ibpiso") else method
    traffic_unit = ("bytes per pyramid-stage BiCGStab iteration (the iterations after the network stage hands over; "
                    "ncu capture, scaled by cells)" if method == "fgmres"
                    else "bytes per inner iteration (ncu capture, scaled by cells)")
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": (achieved / hbm) if achieved else None,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "traffic": (LEARNED_TRAFFIC_PER_CELL[traffic_key] * N if learned and traffic_key in LEARNED_TRAFFIC_PER_CELL
                            else None),
                "traffic_unit": traffic_unit,
                "bytes_per_row_iteration": per_row,
                "network_stage_iterations_per_step": (net_iters / args.steps) if learned else None,
                "p_solve_ms_per_step": p_ms / args.steps, "iterations_per_step": p_iters / args.steps}

    # end to end through the C ABI with host buffers: per step, upload the solver state
    # (u, p, face mass fluxes) from pinned memory, solve, read u and p back
    e2e = None
    if not args.no_e2e:
        # the timed steps again, end to end: every step uploads its state from pinned host memory,
        # solves, and reads the new state back, starting from the state the timed steps started
        # from, so the steps and their iterations are the same
        dev.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        ke = max(1, args.e2e_steps if args.e2e_steps is not None else args.steps)
        e_iters = []
        e0.record(stream)
        for _ in range(ke):
            for nm in state:
                dev.set_from_ptr(nm, host[nm].data_ptr(), sizes[nm])
            dev.solve()
            e_iters.append(dev.last_stats["p_iters_total"])
            for nm in state:
                dev.get_to_ptr(nm, host[nm].data_ptr(), sizes[nm])
        e1.record(stream)
        e1.synchronize()
        e_ms = max_over_ranks(pg, e0.elapsed_time(e1))
        timed_iters = [r["p_iters"] for r in per_step if r["phase"] == "timed"]
        e2e = {"value": world * ke / (e_ms / 1e3), "unit": "time-steps/s", "steps": ke,
               "h2d_bytes_per_step": 8 * sum(sizes[nm] for nm in state),
               "d2h_bytes_per_step": 8 * sum(sizes[nm] for nm in state) + 128,
               "p_iters": e_iters, "same_steps_as_timed": e_iters == timed_iters[:ke],
               "api": "caffe_dev_array (pinned host buffers) + caffe_dev_solve, per step, replaying the timed steps"}
    dev.close()

    # the same steps from rest with the plain FP64 pressure-correction solve
    compare = None
    if args.compare_fp64 > 0 and learned and rank == 0:
        ref = make_solver(nodes, spec.replace(p_form="fp64"), device=local)
        rows = []
        for k in range(args.compare_fp64):
            ref.solve()
            st = ref.last_stats
            rows.append({"step": k + 1, "p_ms": round(st["p_ms"], 2), "p_iters": st["p_iters_total"], "step_ms": round(st["step_ms"], 2),
                         "p_res_max": st["p_res_max"]})
        ref.close()
        same = per_step[:args.compare_fp64]
        pf = sum(r["p_ms"] for r in rows) / len(rows)
        pl = sum(r["p_ms"] for r in same) / len(same)
        itf = sum(r["p_iters"] for r in rows) / len(rows)
        itl = sum(r["p_iters"] for r in same) / len(same)
        sf = sum(r["step_ms"] for r in rows) / len(rows)
        sl = sum(r["step_ms"] for r in same) / len(same)
        compare = {"plain_fp64_steps_from_rest": rows, "learned_same_steps": same,
                   "p_solve_ms_ratio_fp64_over_learned": pf / pl if pl > 0 else None,
                   "krylov_iterations_ratio_fp64_over_learned": itf / itl if itl > 0 else None,
                   "time_steps_per_s_ratio_learned_over_fp64": sf / sl if sl > 0 else None}

    cpu = None
    same_inputs = None
    c2_line = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu_full = measured_cpu(args, 3, 30.0)
        cpu = {k: cpu_full[k] for k in ("value", "unit", "cores", "kind", "sample")}
        if args.workload == "c5":
            same_inputs = same_inputs_comparison(args, local, cpu_full)
            if not args.no_c2_line:
                c2_line = c2_full_line(local, 60.0)

    if rank == 0:
        working_set = N * 8 * 60
        line = {
            "metric": "time-steps/s at 1e-8 true relative residual", "value": value, "unit": "time-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 fields and outer solve; f32 inner Krylov; bf16 network" if learned else "f64",
            "data": "synthetic (seeded mesh and case, no dataset)",
            "config": {"workload": label, "cells": N, "p_form": args.p_form,
                       "precond": args.precond if learned else None, "inner": method,
                       "net_levels": [args.net_from, args.net_to] if learned and args.precond == "network" else None,
                       "restart": args.restart if method == "fgmres" else None,
                       "parallelism": f"replicas x{world}",
                       "l2": f"inputs larger than L2: working set ~{working_set / 2**30:.1f} GiB > 126 MB"},
            "p_solve_ms": p_ms / args.steps, "momentum_solve_ms": mom_ms / args.steps,
            "p_iters_per_step": p_iters / args.steps, "mom_iters_per_step": mom_iters / args.steps,
            "p_res_max": res_max, "fallbacks": fallbacks, "cascades": cascades,
            "net_iters_per_step": net_iters / args.steps,
            "continuity_last": conts[-1], "solver_status": status,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
            "gpu_launches": launches, "compare": compare, "per_step": per_step,
            "cpu_vs_gpu_same_lattice": same_inputs, "c2_128cubed_fully_measured": c2_line,
        }
        if compare:
            print("compare (same steps from rest): p-solve ms fp64/learned %.2f, Krylov iterations fp64/learned %.2f, "
                  "time-steps/s learned/fp64 %.2f" % (compare["p_solve_ms_ratio_fp64_over_learned"] or 0,
                                                      compare["krylov_iterations_ratio_fp64_over_learned"] or 0,
                                                      compare["time_steps_per_s_ratio_learned_over_fp64"] or 0),
                  file=sys.stderr, flush=True)
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=("b200", "reference"))
    ap.add_argument("--workload", default="c5", choices=("c1", "c2", "c3", "c5"))
    ap.add_argument("--p-form", default="learned_mixed", choices=tuple(C.P_FORMS))
    ap.add_argument("--precond", default="network", choices=("levels", "network", "jacobi"))
    ap.add_argument("--inner", default="auto", choices=("auto", "fcg", "bicgstab", "fgmres"))
    ap.add_argument("--net-from", type=int, default=None, help="first pyramid level that runs the network "
                    "(default: the one the shipped parameters were trained for)")
    ap.add_argument("--net-to", type=int, default=None, help="last pyramid level that runs the network "
                    "(default: the coarsest level the shipped parameters were trained on)")
    ap.add_argument("--restart", type=int, default=5)
    ap.add_argument("--params", default=None, help="network parameters (.npy); default: the shipped ones")
    ap.add_argument("--size", type=int, default=None)
    ap.add_argument("--compare-fp64", type=int, default=1, help="plain FP64 steps from rest to compare with")
    ap.add_argument("--e2e-steps", type=int, default=None, help="end-to-end steps (default: --steps)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-c2-line", action="store_true", help="skip the fully measured 128^3 cavity comparison")
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
