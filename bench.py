#!/usr/bin/env python3
"""Benchmark of the DG right-hand side + SSP-RK3 step on B200.

Workload (N = 1): 2D Euler isentropic vortex (gamma 1.4, beta 5, free stream
(1,1,1,1), centred at (5,5)) on [0,10]^2 cut into 256x256x2 = 131072 seeded
jittered triangles (+-0.15h), P3 orthonormal basis (10 modes x 4 fields), 12-point
volume / 4-point edge rules, Roe flux, exact-solution boundaries, CFL 0.1.
A "step" is one SSP-RK3 step (three stages) over the whole mesh.

Metric: DOF-stage updates/s = cells * fields * modes * 3 * steps / seconds.
`value` times K device-resident steps (dgp_run, CUDA graphs) with CUDA events
on the solver's stream; `e2e` times K steps through the C ABI with the state
copied from pinned host memory before and back after every step.

--gpus N > 1 (torchrun): N independent replicas (the north-star path is one
GPU; there is no data-path collective); barrier + max over ranks of the timed
region, value = total updates of all ranks / that time.

--impl reference: DG-Parallel's own pthreads CPU path (oracle/_ref/ref_driver,
built from the reference sources) on the same mesh and case, all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dg-parallel_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

WORKLOAD = {"workload": "euler2d_isentropic_vortex_256x256x2_P3_roe", "cells": 131072, "order": 3,
            "fields": 4, "modes": 10, "flux": "roe", "cfl": 0.1, "mesh": "tri 256x256x2 jitter 0.15h seed 2",
            "rules": "12-pt volume, 4-pt Gauss-Legendre edges"}
METRIC = "DOF-stage updates/s"
REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
REF_DRIVER_LTS = os.path.join(ROOT, "oracle", "_ref", "ref_driver_lts")


class Ranks:
    """The N > 1 plumbing: one process per GPU (torchrun; NCCL) or CPU ranks
    (gloo, for tests).  Without a process group every call is the identity."""

    def __init__(self, backend: str = "nccl", timeout_s: int = 300):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            from datetime import timedelta
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
            self.dist = dist

    def _reduce(self, x: float, op) -> float:
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x: float) -> float:
        return x if self.dist is None else self._reduce(x, self.dist.ReduceOp.MAX)

    def sum(self, x: float) -> float:
        return x if self.dist is None else self._reduce(x, self.dist.ReduceOp.SUM)

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def shard(n: int, rank: int, world: int) -> list:
    """Instances of a rank when n independent instances spread over world ranks
    (round robin; every instance on exactly one rank)."""
    return list(range(rank, n, world))


def aggregate_rate(units_per_rank: float, seconds_max: float) -> float:
    """Whole-job rate: the units all ranks processed over the slowest rank's time."""
    return units_per_rank / seconds_max


def select_device(index: int):
    """The rank's GPU for torch (events, collectives) and for the library."""
    import torch
    import dgp
    torch.cuda.set_device(index)
    dgp.set_device(index)


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(prefix="clocks", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            self.proc.wait(timeout=10)
        self.out.close()

    def summary(self):
        rows = []
        try:
            for line in open(self.out.name):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        finally:
            os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def make_mesh():
    from dgp import meshgen
    return meshgen.tri_square(256, 256, 0.0, 10.0, 0.0, 10.0, jitter=0.15, seed=2)


def vortex_params():
    import dgp
    return dgp.law_params(velocity=(1.0, 1.0, 0.0), center=(5.0, 5.0, 0.0), gamma=1.4, beta=5.0)


def cpu_reference(mesh, steps: int, warmup: int, threads: int):
    """DG-Parallel's pthreads path (parallel.cc) on this workload; None if not built."""
    from dgp import meshgen
    if not os.path.exists(REF_DRIVER):
        return None
    with tempfile.TemporaryDirectory() as td:
        msh = os.path.join(td, "vortex256.msh")
        meshgen.write_msh_v1(mesh, msh)
        cmd = [REF_DRIVER, "--mesh", msh, "--case", "vortex", "--flux", "roe", "--order", "3",
               "--cfl", "0.1", "--threads", str(threads), "--bench", str(steps), "--warmup", str(warmup)]
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=1800)
    line = next((ln for ln in p.stdout.splitlines() if ln.startswith("BENCH")), None)
    if p.returncode != 0 or line is None:
        return None
    kv = dict(tok.split("=") for tok in line.split()[1:])
    return {"value": float(kv["dof_stage_per_s"]), "seconds": float(kv["seconds"]),
            "steps": int(kv["steps"]), "threads": int(kv["threads"])}


def fused_kernel_bytes(E, M, NP, DIM, tsize, with_u0):
    """Bytes one fused stage-kernel launch must move from and to device memory:
    the stage input read, u_n read (stages 2 and 3), the output written (FP64
    state), J^{-1} (right-hand-side type) and |J| (FP64) per cell; the halo
    rows are neighbours' rows of the same input (counted once)."""
    state = E * M * NP * 8
    return (3 if with_u0 else 2) * state + E * (DIM * DIM * tsize + 8)


def elem_kernel_bytes(E, M, NP, NS, DIM, tsize):
    """Bytes one element-kernel launch must move (solvers whose tiles do not
    fit the fused kernel): state read, u_n read, new state written (FP64), face
    slots read and face-point traces written (right-hand-side type), J^{-1}
    (right-hand-side type) and |J| (FP64) per cell."""
    state = E * M * NP * 8
    return 3 * state + 2 * E * NS * M * tsize + E * (DIM * DIM * tsize + 8)


def stage_formula_bytes(E, F, M, NP, DIM):
    """Algorithmic bytes of one whole stage by the per-element-stage formula of
    the workload's roofline definition: coefficients (2 + 2/3) m Np 8 (FP64
    state), geometry (d^2 + 1) 8, faces (F/E)(8 d + 8 + 2*4 + 2) per element."""
    return E * ((2 + 2.0 / 3.0) * M * NP * 8 + (DIM * DIM + 1) * 8) + F * (8 * DIM + 8 + 2 * 4 + 2)


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    mesh = make_mesh()
    threads = os.cpu_count() or 1
    r = cpu_reference(mesh, args.steps, args.warmup, threads)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_driver not built "
                          "(make -C oracle ref needs the DG-Parallel sources)"}))
        return 0
    line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": "DOF-stage/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * r["seconds"] / r["steps"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(WORKLOAD),
            "run": {"threads": threads, "cpu": cpu_model()},
            "cpu_baseline": {"value": r["value"], "unit": "DOF-stage/s", "cores": threads,
                             "kind": "reference",
                             "sample": f"{args.steps} SSP-RK3 steps of the full workload after "
                                       f"{args.warmup} warm-up steps, DG-Parallel pthreads path "
                                       "(parallel.cc) built from source"},
            "e2e": {"value": r["value"], "unit": "DOF-stage/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="dgp", choices=["dgp", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--no-adjoint", action="store_true",
                    help="leave the discrete-adjoint measurement out of the line")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the untimed runs to t = 2 that state the density L2 errors")
    ap.add_argument("--ensemble", action="store_true",
                    help="only the batched-ensemble measurement (96 Burgers instances to t = 0.5, ~2 min)")
    ap.add_argument("--ensemble-tend", type=float, default=0.5,
                    help="--ensemble: end time of the instances (a short run for launch lists)")
    ap.add_argument("--adjoint", action="store_true",
                    help="only the discrete-adjoint measurement (Euler vortex 128x128x2 P2, 400 steps)")
    ap.add_argument("--decompose", action="store_true",
                    help="only the error decomposition of the mixed form (the vortex to t = 2 with "
                         "groups of terms rounded to FP32, ~3 min)")
    ap.add_argument("--configs", action="store_true",
                    help="only the other workloads: scalar P2 on 2048 triangles (200 steps) and "
                         "Maxwell P2 on 663552 tets (one TM110 period), both forms, ~2 min")
    ap.add_argument("--lts", action="store_true",
                    help="only the local time stepping measurement (Euler vortex P3 on 256x256x2 graded "
                         "triangles, 4 size bins, against SSP-RK3 on the same mesh, ~1 min)")
    ap.add_argument("--profile-case", choices=["fp64", "mixed", "maxwell", "limiter", "lts", "adjoint"], default=None,
                    help="only set up the workload and run --warmup + --steps steps (for ncu)")
    ap.add_argument("--tensor-cores", action="store_true",
                    help="--profile-case mixed: the volume contraction on the tensor cores")
    ap.add_argument("--block", type=int, default=0, choices=[0, 64, 128, 256],
                    help="--profile-case: tile shape (threads) of the element and face kernels "
                         "(0: the autotuner's pick, as the bench line)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.profile_case:
        return profile_case(args)
    if args.adjoint:
        select_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps({"adjoint": adjoint_bench()}))
        return 0
    if args.ensemble:
        ranks = Ranks("nccl")
        select_device(ranks.local)
        out = ensemble_bench(tend=args.ensemble_tend, ranks=ranks)
        if ranks.rank == 0:
            print(json.dumps({"ensemble": out}))
        ranks.close()
        return 0
    if args.decompose:
        select_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps({"decompose": decompose_bench()}))
        return 0
    if args.configs:
        select_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps({"configs": configs_bench()}))
        return 0
    if args.lts:
        select_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps({"lts": lts_bench(steps=args.steps if args.steps != 300 else 16)}))
        return 0

    import numpy as np
    import torch
    import dgp

    ranks = Ranks("nccl")
    world, rank, local = ranks.world, ranks.rank, ranks.local
    select_device(local)

    mesh_np = make_mesh()
    prm = vortex_params()
    mesh = dgp.Mesh.from_arrays(2, mesh_np.vertices, mesh_np.cells, 100, mesh_np.bfaces, mesh_np.btags)
    law = dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, prm)
    E = mesh.ncells
    units_per_step = E * 4 * 10 * 3

    def barrier():
        ranks.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return ranks.max(x)

    def timed_run(solver, steps, warmup, sampler=None):
        solver.project(0.0)
        t, _ = solver.run(0.0, 0.0, 0.1, warmup)
        stream = torch.cuda.ExternalStream(solver.stream())
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        ctx = sampler if sampler is not None else _Null()
        with ctx:
            ev0.record(stream)
            t_end, n = solver.run(t, 0.0, 0.1, steps)
            ev1.record(stream)
            ev1.synchronize()
        barrier()
        return max_over_ranks(ev0.elapsed_time(ev1) / 1e3), t_end, n

    results = {}
    clocks = None
    tiles = {}
    for name, prec, tc in (("fp64", dgp.FP64, False), ("mixed", dgp.MIXED, False),
                           ("mixed_tc", dgp.MIXED, True)):
        # tile shape of the stage kernel from the autotuner (untimed; a few
        # steps of each built shape on this mesh); the tensor-core variant of
        # the mixed form has 128-thread tiles
        if tc:
            dgp.tune_set(dgp.LAW_EULER2D, dgp.FLUX_ROE, 2, 3, prec, E, 128)
        else:
            best, cand = dgp.autotune(mesh, law, 3, prec, 0, iters=5)
            tiles[name] = {"block": best, "ms_per_step_64_128_256": cand}
        s = dgp.Solver(mesh, law, 3, prec)
        if tc:
            s.set_tensor_cores(True)
        sampler = ClockSampler(local) if (name == "fp64" and rank == 0) else None
        sec, t_end, n = timed_run(s, args.steps, args.warmup, sampler)
        if sampler is not None:
            clocks = sampler.summary()
        assert n == args.steps
        err = s.l2_error(t_end, 0)
        kern = s.profile_kernels(20)
        launches = s.launches_per_step() * 8 * ((args.steps + 7) // 8) + 1  # graphs of 8 steps + first CFL
        results[name] = {"seconds": sec, "value": aggregate_rate(units_per_step * args.steps * world, sec),
                         "gpu_launches": launches,
                         "t_end": t_end, "density_l2_vs_exact": err, "kernel_ms": kern.tolist(),
                         "solver": s}
    fp64, mixed, mixed_tc = results["fp64"], results["mixed"], results["mixed_tc"]
    # mixed vs FP64 at the same time: density L2 difference
    c64 = fp64["solver"].get_state()
    c32 = mixed["solver"].get_state()
    mixed["density_coeff_rel_diff_vs_fp64"] = float(np.abs(c32[:, 0] - c64[:, 0]).max() / np.abs(c64[:, 0]).max())
    # the workload's full run (isentropic vortex to t = 2, CFL 0.1), untimed:
    # density L2 error against the exact solution for both forms
    accuracy = None
    if not args.no_accuracy:
        accuracy = {}
        for name in ("fp64", "mixed", "mixed_tc"):
            s = results[name]["solver"]
            s.project(0.0)
            w0 = time.perf_counter()
            t_end, n = s.run(0.0, 2.0, 0.1)
            accuracy[name] = {"t": t_end, "steps": n, "density_l2_vs_exact": s.l2_error(t_end, 0),
                              "wall_s": time.perf_counter() - w0}
        accuracy["mixed_over_fp64_l2"] = (accuracy["mixed"]["density_l2_vs_exact"] /
                                          accuracy["fp64"]["density_l2_vs_exact"])
        accuracy["mixed_tc_over_fp64_l2"] = (accuracy["mixed_tc"]["density_l2_vs_exact"] /
                                             accuracy["fp64"]["density_l2_vs_exact"])
        c64 = results["fp64"]["solver"].get_state()
        c32 = results["mixed"]["solver"].get_state()
        accuracy["mixed_density_coeff_rel_diff_vs_fp64"] = float(
            np.abs(c32[:, 0] - c64[:, 0]).max() / np.abs(c64[:, 0]).max())

    # end to end through the C ABI with host buffers: per step, state H2D from
    # pinned memory, one SSP-RK3 step, state D2H
    s = fp64["solver"]
    host = torch.empty(s.shape, dtype=torch.float64, pin_memory=True).numpy()
    host[...] = s.get_state()
    nbytes = host.nbytes
    t = fp64["t_end"]
    barrier()
    w0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        s.set_state(host)
        t, _ = s.run(t, 0.0, 0.1, 1)
        s.get_state(out=host)
    torch.cuda.synchronize()
    e2e_sec = max_over_ranks(time.perf_counter() - w0)
    e2e_value = units_per_step * args.e2e_steps * world / e2e_sec

    # the adjoint of the discrete operator on its own workload (untimed here;
    # its own CUDA-event times): gradient cost against a forward solve
    adjoint = None
    if not args.no_adjoint:
        adjoint = adjoint_bench()

    if rank == 0:
        peaks, peak_src = load_peaks()
        # the fused stage kernel (one launch a stage): stage 1, stage 2 and
        # the last stage with its CFL reduction (and the one-CTA finalize)
        s1_ms, s2_ms, s3_ms = fp64["kernel_ms"]
        stage_ms = (s1_ms + s2_ms + s3_ms) / 3.0
        M, NP = 4, 10
        F = mesh.nfaces
        # algorithmic bytes of a stage by the workload's per-element-stage
        # formula (coefficients (2 + 2/3) m Np 8, geometry, face data): the
        # roofline's numerator
        st_bytes = stage_formula_bytes(E, F, M, NP, 2)
        achieved = st_bytes / (stage_ms * 1e-3) / 1e9
        kname = "stage_kernel (faces + volume + lift + SSP-RK3 stage, fused; mean of the three stages)"
        # the bytes the fused kernel itself moves per launch (secondary)
        own_bytes = (fused_kernel_bytes(E, M, NP, 2, 8, False) + 2 * fused_kernel_bytes(E, M, NP, 2, 8, True)) / 3.0
        traffic = None
        tfile = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tfile):
            tr = json.load(open(tfile))
            traffic = tr.get("stage_kernel")
        ms_per_step = fp64["seconds"] / args.steps * 1e3
        cpu = None
        if not args.no_cpu_baseline:
            r = cpu_reference(mesh_np, 3, 1, os.cpu_count() or 1)
            if r is not None:
                cpu = {"value": r["value"], "unit": "DOF-stage/s", "cores": r["threads"], "kind": "reference",
                       "sample": "3 SSP-RK3 steps (after 1 warm-up) of the full 131072-cell workload, "
                                 "DG-Parallel pthreads path built from source, " + cpu_model()}
                # the same path on one thread (1 step after 1 warm-up)
                r1 = cpu_reference(mesh_np, 1, 1, 1)
                if r1 is not None:
                    cpu["value_1_thread"] = r1["value"]
        line = {
            "metric": METRIC, "value": fp64["value"], "unit": "DOF-stage/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": dict(WORKLOAD),
            "run": {"parallelism": f"replicas{world}", "tiles": tiles,
                    "l2": "working set 290 MB > 126 MB L2; each step streams ~1 GB"},
            "mixed": {"value": mixed["value"],
                      "dtype": "f32 RHS (traces, fluxes, contractions, face slots); f64 state, "
                               "RK update, inverse mass, time, totals",
                      "speedup_vs_fp64": mixed["value"] / fp64["value"],
                      "density_l2_vs_exact": mixed["density_l2_vs_exact"],
                      "density_coeff_rel_diff_vs_fp64": mixed["density_coeff_rel_diff_vs_fp64"],
                      "kernel_ms": mixed["kernel_ms"],
                      "tensor_cores": {"value": mixed_tc["value"],
                                       "contraction": "tcgen05.mma kind::tf32, split high/low operands",
                                       "speedup_vs_fp64": mixed_tc["value"] / fp64["value"],
                                       "density_l2_vs_exact": mixed_tc["density_l2_vs_exact"],
                                       "kernel_ms": mixed_tc["kernel_ms"]}},
            "fp64_density_l2_vs_exact": fp64["density_l2_vs_exact"],
            "accuracy_t2": accuracy,
            "kernel_ms": {"stage1": s1_ms, "stage2": s2_ms, "stage3_cfl": s3_ms},
            "roofline": {"kernel": kname, "bound": "hbm", "achieved": achieved,
                         "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                         "frac": achieved / peaks.get("hbm_gbs"), "traffic": traffic,
                         "peak_source": peak_src,
                         "algorithmic_bytes_per_launch": st_bytes,
                         "bytes_per_dof_stage": st_bytes / (E * M * NP),
                         "kernel_own_bytes_per_launch": own_bytes,
                         "kernel_own_frac": own_bytes / (stage_ms * 1e-3) / 1e9 / peaks.get("hbm_gbs")},
            "adjoint": adjoint,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "DOF-stage/s", "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes, "steps": args.e2e_steps,
                    "timing": "host wall clock, synchronized, C ABI with pinned host state"},
            "gpu_launches": fp64["gpu_launches"],
            "clocks": clocks,
        }
        print(json.dumps(line))
    for r in results.values():
        r["solver"].close()
    ranks.close()
    return 0


def decompose_bench(tend=2.0):
    """Error decomposition of the mixed form on the bench workload (the vortex
    to t = 2): the FP64 solver with one group of terms rounded to FP32 at a
    time (dgp_set_rounding_probe), every group together, and the mixed form
    itself; density L2 error against the exact vortex for each."""
    import dgp
    m = make_mesh()
    mesh = dgp.Mesh.from_arrays(2, m.vertices, m.cells, 100, m.bfaces, m.btags)
    law = dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, vortex_params())
    dgp.tune_set(dgp.LAW_EULER2D, dgp.FLUX_ROE, 2, 3, dgp.FP64, m.cells.shape[0], 128)
    names = {0: "fp64", 1: "geometry", 2: "face traces", 4: "volume values", 8: "volume flux products",
             16: "face slots", 32: "contraction result", 64: "tables", 127: "all of the above"}
    rows = []
    for mask, name in names.items():
        s = dgp.Solver(mesh, law, 3, dgp.FP64)
        s.set_rounding_probe(mask)
        s.project(0.0)
        t, n = s.run(0.0, tend, 0.1)
        rows.append({"rounded_to_fp32": name, "mask": mask, "steps": n, "density_l2_vs_exact": s.l2_error(t, 0)})
        s.close()
    for name, tc in (("mixed form (FP32 right-hand side)", False), ("mixed form, tensor-core contraction", True)):
        s = dgp.Solver(mesh, law, 3, dgp.MIXED)
        if tc:
            s.set_tensor_cores(True)
        s.project(0.0)
        t, n = s.run(0.0, tend, 0.1)
        rows.append({"rounded_to_fp32": name, "steps": n, "density_l2_vs_exact": s.l2_error(t, 0)})
        s.close()
    base = rows[0]["density_l2_vs_exact"]
    for r in rows:
        r["over_fp64"] = r["density_l2_vs_exact"] / base
    return {"workload": WORKLOAD["workload"], "t": tend, "rows": rows}


def ensemble_bench(n=96, seed=6, tend=0.5, ranks=None):
    """Batched ensemble: n independent Burgers2D instances (Lax-Friedrichs flux,
    far-field boundaries) on seeded jittered triangle meshes whose sizes are
    log-uniform in [2k, 128k] cells, orders uniform in P1-P4, initial state
    0.5 + A sin(2 pi (x + y)) with A uniform in [0.5, 1.5], moment limiter on,
    run to t = 0.5 (past shock formation) in the mixed form (FP32 right-hand
    side, FP64 state and conserved totals).  Tile shapes per group come from the
    autotuner.  The run is timed by the device clock from the common start to
    each instance's last step.  Under torchrun the instances spread over the
    ranks round robin (no communication): the rate is the updates of all ranks
    over the slowest rank's device time."""
    import numpy as np
    import dgp
    from dgp import meshgen
    ranks = ranks or Ranks("nccl")
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(2000.0), np.log(128000.0), n))
    orders_all = rng.integers(1, 5, size=n)
    amps = rng.uniform(0.5, 1.5, size=n)
    mine = shard(n, ranks.rank, ranks.world)
    orders = orders_all[mine]
    t_setup = time.time()
    meshes, laws = [], []
    for i in mine:
        side = max(4, int(round(np.sqrt(counts[i] / 2.0))))
        m = meshgen.tri_square(side, side, 0.0, 1.0, 0.0, 1.0, jitter=0.15, seed=1000 + i)
        meshes.append(dgp.Mesh.from_arrays(2, m.vertices, m.cells, m.domain_tag, m.bfaces, m.btags))
        laws.append(dgp.Law(dgp.LAW_BURGERS2D, dgp.FLUX_LLF, dgp.FIELD_SINE, dgp.law_params(amplitude=amps[i])))
    n_all, n = n, len(mine)
    setup_s = time.time() - t_setup
    t_tune = time.time()
    dgp.autotune_ensemble(meshes, laws, orders.tolist(), dgp.MIXED, dgp.LIMITER_MOMENT, iters=3)
    tune_s = time.time() - t_tune
    ens = dgp.Ensemble(meshes, laws, orders.tolist(), dgp.MIXED, dgp.LIMITER_MOMENT)
    ens.project(0.0)
    ens.run(0.0, 0.0, 0.1, max_steps=8)  # warm-up: graph capture
    ens.project(0.0)
    tot0 = np.array([ens.totals(i)[0] for i in range(n)])
    t_wall = time.time()
    t, steps, ms, total_ms = ens.run(0.0, tend, 0.1)
    wall_s = time.time() - t_wall
    tot1 = np.array([ens.totals(i)[0] for i in range(n)])
    dofs = np.array([ens.shapes[i][0] * ens.shapes[i][1] * ens.shapes[i][2] for i in range(n)], dtype=np.float64)
    updates = float((dofs * 3 * steps).sum())
    # whole-run algorithmic bytes by the per-element-stage formula (FP64 state
    # coefficients, geometry, face data), every instance's cells x 3 stages x steps
    stage_bytes = 0.0
    for i in range(n):
        stage_bytes += 3.0 * float(steps[i]) * stage_formula_bytes(meshes[i].ncells, meshes[i].nfaces,
                                                                   ens.shapes[i][1], ens.shapes[i][2], 2)
    peaks, peak_src = load_peaks()
    # every rank's work over the slowest rank's device time
    ranks.barrier()
    total_ms = ranks.max(total_ms)
    updates = ranks.sum(updates)
    stage_bytes = ranks.sum(stage_bytes)
    achieved = stage_bytes / (total_ms * 1e-3) / 1e9
    finite = all(np.isfinite(ens.get_state(i)).all() for i in range(n))
    groups = {}
    for g in sorted(set(ens.groups)):
        b, te = ens.group_block(g)
        members = [i for i in range(n) if ens.groups[i] == g]
        groups[f"P{int(orders[members[0]])}"] = {"instances": len(members), "block": b, "cells_per_tile": te,
                                                  "cells": int(sum(ens.shapes[i][0] for i in members))}
    out = {
        "metric": "aggregate DOF-stage updates/s", "value": aggregate_rate(updates, total_ms * 1e-3),
        "unit": "DOF-stage/s", "instances": n_all, "ranks": ranks.world, "instances_rank0": n,
        "cells_total_rank0": int(sum(ens.shapes[i][0] for i in range(n))),
        "dofs_total": int(dofs.sum()), "steps_total": int(steps.sum()),
        "steps_min_max": [int(steps.min()), int(steps.max())],
        "device_ms_total": total_ms, "wall_s": wall_s,
        "instance_ms_p50": float(np.percentile(ms, 50)), "instance_ms_p99": float(np.percentile(ms, 99)),
        "all_reached_t_end": bool(np.allclose(t, tend, atol=1e-12)), "finite": bool(finite),
        "total_change_rel_max": float(np.max(np.abs(tot1 - tot0) / np.maximum(np.abs(tot0), 1e-300))),
        "groups": groups, "launches_per_step_all_groups": ens.launches_per_step(),
        "roofline": {"bound": "hbm", "formula": "per-element-stage bytes (coefficients, geometry, faces) "
                                                 "summed over every instance's stages, over the run's device time",
                     "bytes": stage_bytes, "achieved": achieved, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                     "frac": achieved / peaks.get("hbm_gbs"), "peak_source": peak_src},
        "precision": "f32 RHS, f64 state, time and totals", "limiter": "triangle moment limiter",
        "flux": "Lax-Friedrichs, far-field boundaries", "setup_s": setup_s, "autotune_s": tune_s,
        "config": {"sizes": "log-uniform 2k-128k cells", "orders": "P1-P4 uniform", "A": "U[0.5,1.5]",
                   "t_end": tend, "cfl": 0.1, "seed": seed},
    }
    ens.close()
    return out


def configs_bench(steps=200):
    """The other workloads, both forms, CUDA events on the solver's stream:

    scalar: u_t + a.grad u = 0, a = (1, 0.5), Gaussian (centre (0.3, 0.3),
      s = 0.01) on the unit square cut into 32x32x2 = 2048 jittered triangles
      (seed 1), P2, upwind, exact-solution inflow, CFL 0.1, 200 steps; also
      DG-Parallel's pthreads path on all host cores and on one.
    llf: the vortex workload (131072 triangles, P3) with the local
      Lax-Friedrichs flux, to t = 2 for the density error.
    maxwell: 3D Maxwell (eps = mu = 1), upwind flux, PEC walls, TM110 cavity
      mode on the unit cube cut into 48^3 x 6 = 663552 jittered tets (seed 3),
      P2, CFL 0.1; `steps` timed steps, then one full period (T = sqrt 2) for
      the Ez L2 error against the exact mode.  The reference has no 3D Maxwell
      law (its field storage caps at 5 fields), so there is no CPU reference.
    Roofline: the whole stage against the per-element-stage formula, and the
    bytes the stage kernel itself moves (fused_kernel_bytes; elem_kernel_bytes
    for the element kernel of a solver that is not fused) over its CUDA-event
    time."""
    import numpy as np
    import torch
    import dgp
    from dgp import meshgen
    peaks, peak_src = load_peaks()
    hbm = peaks.get("hbm_gbs")

    def timed(s, nsteps):
        s.project(0.0)
        t, _ = s.run(0.0, 0.0, 0.1, 8)
        stream = torch.cuda.ExternalStream(s.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        t_end, n = s.run(t, 0.0, 0.1, nsteps)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3, t_end, n

    def measure(mesh, law, order, M, NP, NS, DIM, field, t_full=None, rule=0):
        E, F = mesh.ncells, mesh.nfaces
        res = {"cells": E, "faces": F, "dofs": E * M * NP,
               "quadrature": "the workloads' point counts" if rule else "DG-Parallel's rules"}
        for name, prec, tsize in (("fp64", dgp.FP64, 8), ("mixed", dgp.MIXED, 4)):
            s = dgp.Solver(mesh, law, order, prec, rule=rule)
            sec, t_end, n = timed(s, steps)
            kern = s.profile_kernels(10)
            sb = stage_formula_bytes(E, F, M, NP, DIM)
            if s.fused:
                # one fused launch a stage: stage 1, stage 2, last stage + CFL
                stage_ms = float(kern.mean())
                kb = (fused_kernel_bytes(E, M, NP, DIM, tsize, False) +
                      2 * fused_kernel_bytes(E, M, NP, DIM, tsize, True)) / 3.0
                kname, kms = "stage_kernel (mean of the three stages)", stage_ms
                kern_named = {"stage1": kern[0], "stage2": kern[1], "stage3_cfl": kern[2]}
            else:
                stage_ms = float(kern[0] + kern[1])
                kb = elem_kernel_bytes(E, M, NP, NS, DIM, tsize)
                kname, kms = "elem_kernel", float(kern[1])
                kern_named = {"face": kern[0], "elem": kern[1], "elem_cfl": kern[2]}
            r = {"value": E * M * NP * 3 * n / sec, "unit": "DOF-stage/s", "steps": n,
                 "ms_per_step": sec / n * 1e3, "kernel_ms": {k: float(v) for k, v in kern_named.items()},
                 "roofline": {"kernel": kname, "bound": "hbm",
                              "basis": "whole stage against the per-element-stage formula",
                              "algorithmic_bytes_per_launch": sb,
                              "achieved": sb / (stage_ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                              "frac": sb / (stage_ms * 1e-3) / 1e9 / hbm, "peak_source": peak_src,
                              "kernel_own_bytes_per_launch": kb,
                              "kernel_own_frac": kb / (kms * 1e-3) / 1e9 / hbm},
                 "l2_vs_exact_after_timed_steps": s.l2_error(t_end, field)}
            if t_full is not None:
                s.project(0.0)
                w = time.perf_counter()
                t_f, n_f = s.run(0.0, t_full, 0.1)
                r["full_run"] = {"t": t_f, "steps": n_f, "wall_s": time.perf_counter() - w,
                                 "l2_vs_exact": s.l2_error(t_f, field)}
            s.close()
            res[name] = r
        res["mixed_over_fp64"] = res["mixed"]["value"] / res["fp64"]["value"]
        return res

    out = {}
    m1 = meshgen.tri_square(32, 32, 0.0, 1.0, 0.0, 1.0, jitter=0.15, seed=1)
    mesh1 = dgp.Mesh.from_arrays(2, m1.vertices, m1.cells, m1.domain_tag, m1.bfaces, m1.btags)
    law1 = dgp.Law(dgp.LAW_SCALAR, dgp.FLUX_UPWIND, dgp.FIELD_GAUSS,
                   dgp.law_params(velocity=(1.0, 0.5, 0.0), center=(0.3, 0.3, 0.0), width=0.01))
    out["scalar_p2_2048tri"] = measure(mesh1, law1, 2, 1, 6, 3 * 3, 2, 0)
    out["scalar_p2_2048tri"]["note"] = "launch/latency bound (12288 DOFs); not roofline-graded"
    # the workload's stated quadrature: 7-point volume rule (degree 5)
    out["scalar_p2_2048tri_7pt"] = measure(mesh1, law1, 2, 1, 6, 3 * 3, 2, 0, rule=dgp.RULE_WORKLOAD)
    if os.path.exists(REF_DRIVER):
        cpu = {}
        with tempfile.TemporaryDirectory() as td:
            msh = os.path.join(td, "scalar32.msh")
            meshgen.write_msh_v1(m1, msh)
            for thr in (os.cpu_count() or 1, 1):
                cmd = [REF_DRIVER, "--mesh", msh, "--case", "gauss", "--order", "2", "--cfl", "0.1",
                       "--ax", "1", "--ay", "0.5", "--cx", "0.3", "--cy", "0.3", "--s", "0.01",
                       "--threads", str(thr), "--bench", str(steps), "--warmup", "3"]
                p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
                line = next((ln for ln in p.stdout.splitlines() if ln.startswith("BENCH")), None)
                if p.returncode == 0 and line:
                    kv = dict(tok.split("=") for tok in line.split()[1:])
                    cpu[f"threads_{thr}"] = float(kv["dof_stage_per_s"])
        out["scalar_p2_2048tri"]["cpu_reference_dof_stage_per_s"] = cpu
    m3 = meshgen.tet_cube(48, 0.0, 1.0, jitter=0.1, seed=3, boundary_tag=40000)
    mesh3 = dgp.Mesh.from_arrays(3, m3.vertices, m3.cells, m3.domain_tag, m3.bfaces, m3.btags)
    law3 = dgp.Law(dgp.LAW_MAXWELL3D, dgp.FLUX_UPWIND, dgp.FIELD_TM110, dgp.law_params(cavity=1.0))
    out["maxwell3d_p2_663552tet"] = measure(mesh3, law3, 2, 6, 10, 4 * 7, 3, 2, t_full=np.sqrt(2.0))
    # the workload's stated quadrature: 11-point volume, 6-point face rules
    out["maxwell3d_p2_663552tet_11pt"] = measure(mesh3, law3, 2, 6, 10, 4 * 6, 3, 2, t_full=np.sqrt(2.0),
                                                 rule=dgp.RULE_WORKLOAD)
    # the vortex workload with the local Lax-Friedrichs flux (to t = 2 for the
    # density error)
    m2 = make_mesh()
    mesh2 = dgp.Mesh.from_arrays(2, m2.vertices, m2.cells, 100, m2.bfaces, m2.btags)
    law2 = dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_LLF, dgp.FIELD_VORTEX, vortex_params())
    out["euler2d_p3_vortex256_llf"] = measure(mesh2, law2, 3, 4, 10, 3 * 4, 2, 0, t_full=2.0)
    return out


def lts_mesh(n=256, ratio=1.0098):
    """[0,10]^2 cut into n x n x 2 triangles with node lines spaced
    geometrically (ratio 1.0098 per line: cell sizes span ~12x, 4 size bins,
    every bin ~70 cells thick)."""
    from dgp import meshgen
    return meshgen.tri_graded(n, n, ratio, 0.0, 10.0, 0.0, 10.0)


def lts_bench(n=256, ratio=1.0098, steps=16):
    """Local time stepping (DGAnalysis mode 5: DGAnalysis::sortCellsBySize +
    RungeKuttaTVD2adaptive) on the Euler vortex (beta 5 at (5, 5), Roe, P3,
    FP64, exact-solution boundary) over lts_mesh(), CFL 0.1.  Timed with CUDA
    events on the solver's stream: `steps` steps of DT (bin 0's step, the CFL
    minimum times 2^(bins-1)) through dgp_run, then SSP-RK3 on the same mesh
    from the same state to the same end time at the CFL step.  Units: a cell of
    bin b takes 2^b sub-steps of two stages, M Np DOFs each (DOF-substage/s).
    CPU: the reference's own binning and integrator (oracle/_ref/
    ref_driver_lts, range helpers with the whole-mesh bodies) for one step on
    one thread."""
    import numpy as np
    import torch
    import dgp
    m = lts_mesh(n, ratio)
    mesh = dgp.Mesh.from_arrays(2, m.vertices, m.cells, 100, m.bfaces, m.btags)
    law = dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, vortex_params())
    M, NP = 4, 10

    def timed_run(s, t0, tend, nmax):
        stream = torch.cuda.ExternalStream(s.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        t_end, k = s.run(t0, tend, 0.1, nmax)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3, t_end, k

    s = dgp.Solver(mesh, law, 3, dgp.FP64)
    s.set_p0_fallback(False)  # local time stepping runs without the P0 fallback
    nb = s.set_time_stepping(dgp.STEPPING_LOCAL)
    bins, role = s.lts_bins()
    E = mesh.ncells
    units = float(np.sum(M * NP * 2 * (2.0 ** bins)))
    t_w, _ = s.run(0.0, 0.0, 0.1, 3)  # warm-up (graph capture)
    state_w = s.get_state()
    DT = s.cfl_dt(0.1)
    sec, t_end, k = timed_run(s, t_w, 0.0, steps)
    launches = s.launches_per_step()
    l2_lts = s.l2_error(t_end, 0)
    rk = dgp.Solver(mesh, law, 3, dgp.FP64)
    rk.set_state(state_w)
    rk.run(t_w, 0.0, 0.1, 3)  # warm-up (graph capture), then back to the same state
    rk.set_state(state_w)
    dt_rk = rk.cfl_dt(0.1)
    sec_rk, t_rk, k_rk = timed_run(rk, t_w, t_end, 0)
    out = {"workload": f"Euler vortex P3 Roe FP64, {n}x{n}x2 graded triangles on [0,10]^2 "
                       f"(node spacing ratio {ratio})", "cells": E, "bins": nb,
           "cells_per_bin": np.bincount(bins, minlength=nb).tolist(),
           "interface_cells": int(np.count_nonzero(role)),
           "steps": k, "DT": DT, "t": [t_w, t_end], "ms_per_step": sec / k * 1e3,
           "value": units * k / sec, "unit": "DOF-substage/s", "gpu_launches_per_step": launches,
           "l2_density_vs_exact": l2_lts,
           "ssprk3_same_mesh": {"steps": k_rk, "dt": dt_rk, "ms_per_step": sec_rk / k_rk * 1e3,
                                "seconds_to_same_t": sec_rk, "l2_density_vs_exact": rk.l2_error(t_rk, 0)},
           "seconds_to_same_t": sec, "speedup_over_ssprk3": sec_rk / sec}
    # roofline by the per-element-stage formula, one element-stage per cell
    # sub-stage (the accumulator, copy slot and saved state the integrator adds
    # are not counted)
    peaks, peak_src = load_peaks()
    hbm = peaks.get("hbm_gbs")
    sb = stage_formula_bytes(E, mesh.nfaces, M, NP, 2) / E * (units / (M * NP))
    ach = sb / (sec / k) / 1e9
    out["roofline"] = {"bound": "hbm", "basis": "per-element-stage formula x cell sub-stages per step",
                       "algorithmic_bytes_per_step": sb, "achieved": ach, "peak": hbm, "unit": "GB/s",
                       "frac": ach / hbm, "peak_source": peak_src}
    rk.close()
    s.close()
    if os.path.exists(REF_DRIVER_LTS):
        with tempfile.TemporaryDirectory() as td:
            msh = os.path.join(td, "graded.msh")
            from dgp import meshgen
            meshgen.write_msh_v1(m, msh)
            cmd = [REF_DRIVER_LTS, "--mesh", msh, "--lts", "1", "--case", "vortex", "--flux", "roe",
                   "--order", "3", "--cfl", "0.1", "--bench", "1", "--warmup", "0"]
            p = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
            line = next((ln for ln in p.stdout.splitlines() if ln.startswith("BENCH")), None)
            if p.returncode == 0 and line:
                kv = dict(tok.split("=") for tok in line.split()[1:])
                out["cpu_baseline"] = {"value": units / float(kv["seconds"]), "unit": "DOF-substage/s",
                                       "cores": 1, "kind": "reference",
                                       "sample": "one step of the same mesh (ref_driver_lts, 1 thread)"}
    return out


def adjoint_bench(n=128, order=2, nsteps=400, every=20, nrec=64, ndir=16, eps=1e-3):
    """Discrete adjoint on the Euler vortex: 128x128x2 jittered triangles on
    [0,10]^2, P2, Roe flux, nsteps SSP-RK3 steps of a fixed dt (half the CFL
    0.1 step of the initial state), checkpoint every `every` steps.
    J = sum over nrec seeded uniform receivers of (rho(x_r, T) - rho_obs)^2 with
    rho_obs from a forward run with vortex strength 5.5.  The gradient with
    respect to every initial coefficient is computed in the mixed form (FP32
    right-hand side and adjoint arithmetic) and in FP64, and checked by central
    differences (step eps along ndir seeded Gaussian directions of unit 2-norm)
    of the FP64 forward map.  Times are CUDA-event times on the solver's stream."""
    import numpy as np
    import torch
    import dgp
    from dgp import meshgen
    m = meshgen.tri_square(n, n, 0.0, 10.0, 0.0, 10.0, jitter=0.15, seed=2)
    mesh = dgp.Mesh.from_arrays(2, m.vertices, m.cells, m.domain_tag, m.bfaces, m.btags)
    prm = vortex_params()
    prm_obs = prm.copy()
    prm_obs[8] = 5.5
    pts = np.random.default_rng(4).uniform(0.5, 9.5, size=(nrec, 2))
    so = dgp.Solver(mesh, dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, prm_obs), order, dgp.FP64)
    so.project(0.0)
    dt = 0.5 * so.cfl_dt(0.1)
    so.set_receivers(pts, np.zeros(nrec))
    so.forward_checkpointed(0.0, dt, nsteps, every)
    obs, _ = so.receiver_values()
    so.close()
    law = dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, prm)
    out = {"workload": f"euler2d vortex {n}x{n}x2 P{order} roe, {nsteps} steps, checkpoint every {every}",
           "cells": 2 * n * n, "receivers": nrec, "dt": dt}
    grads = {}
    for name, prec in (("fp64", dgp.FP64), ("mixed", dgp.MIXED)):
        s = dgp.Solver(mesh, law, order, prec)
        s.project(0.0)
        s.set_receivers(pts, obs)
        u0 = s.get_state()
        stream = torch.cuda.ExternalStream(s.stream())

        def timed(fn):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            r = fn()
            e1.record(stream)
            e1.synchronize()
            return r, e0.elapsed_time(e1)

        # warm-up of both modes: every buffer (checkpoints, the recorded
        # stage states, adjoint vectors) is allocated outside the timed runs
        s.forward_checkpointed(0.0, dt, nsteps, every)
        s.backward()
        s.set_state(u0)
        s.forward_checkpointed(0.0, dt, nsteps, 0)
        s.backward()
        # plain forward solve: the same nsteps fixed-dt steps, no checkpoints
        s.set_state(u0)
        _, t_plain = timed(lambda: s.forward_checkpointed(0.0, dt, nsteps, nsteps))
        s.set_state(u0)
        J, t_fwd = timed(lambda: s.forward_checkpointed(0.0, dt, nsteps, every))
        g, t_bwd = timed(lambda: s.backward())
        grads[name] = g
        # every stage state kept in HBM (3 x nsteps states), no recompute
        s.set_state(u0)
        _, t_fwd_rec = timed(lambda: s.forward_checkpointed(0.0, dt, nsteps, 0))
        g_rec, t_bwd_rec = timed(lambda: s.backward())
        out[name] = {"J": J, "forward_ms": t_plain, "forward_checkpointed_ms": t_fwd, "backward_ms": t_bwd,
                     "gradient_over_forward": (t_fwd + t_bwd) / t_plain, "backward_over_forward": t_bwd / t_plain,
                     "recorded": {"stage_states_gb": 3 * nsteps * u0.nbytes / 1e9, "forward_ms": t_fwd_rec,
                                  "backward_ms": t_bwd_rec, "backward_over_forward": t_bwd_rec / t_plain,
                                  "gradient_over_forward": (t_fwd_rec + t_bwd_rec) / t_plain,
                                  "gradient_equals_checkpointed": bool(np.array_equal(g_rec, g)),
                                  "gradient_max_rel_diff": float(np.abs(g_rec - g).max() / np.abs(g).max())}}
        s.close()
    # central differences of the FP64 forward map
    s = dgp.Solver(mesh, law, order, dgp.FP64)
    s.project(0.0)
    s.set_receivers(pts, obs)
    u0 = s.get_state()
    rng = np.random.default_rng(5)
    err64, err32 = [], []
    for _ in range(ndir):
        d = rng.standard_normal(u0.shape)
        d /= np.linalg.norm(d)  # unit direction in coefficient space
        s.set_state(u0 + eps * d)
        jp = s.forward_checkpointed(0.0, dt, nsteps, nsteps)
        s.set_state(u0 - eps * d)
        jm = s.forward_checkpointed(0.0, dt, nsteps, nsteps)
        fd = (jp - jm) / (2 * eps)
        for g, lst in ((grads["fp64"], err64), (grads["mixed"], err32)):
            ad = float(np.sum(g * d))
            lst.append(abs(fd - ad) / max(abs(fd), abs(ad)))
    s.close()
    out["fd_check"] = {"eps": eps, "directions": ndir, "max_rel_err_fp64": max(err64),
                       "max_rel_err_mixed": max(err32),
                       "mixed_vs_fp64_gradient_rel": float(np.abs(grads["mixed"] - grads["fp64"]).max()
                                                           / np.abs(grads["fp64"]).max())}
    return out


def profile_case(args):
    """The bench workload alone: setup, --warmup steps, then --steps steps
    ("maxwell": the Maxwell P2 workload of --configs, FP64)."""
    import dgp
    if args.profile_case == "limiter":
        # Burgers P4, Lax-Friedrichs, 0.5 + sin(2 pi (x + y)) on 300x300x2
        # triangles, mixed form, moment limiter after every stage
        from dgp import meshgen
        m = meshgen.tri_square(300, 300, 0.0, 1.0, 0.0, 1.0, jitter=0.15, seed=1000)
        mesh = dgp.Mesh.from_arrays(2, m.vertices, m.cells, m.domain_tag, m.bfaces, m.btags)
        law = dgp.Law(dgp.LAW_BURGERS2D, dgp.FLUX_LLF, dgp.FIELD_SINE, dgp.law_params(amplitude=1.0))
        s = dgp.Solver(mesh, law, 4, dgp.MIXED, dgp.LIMITER_MOMENT)
        s.project(0.0)
        t, n = s.run(0.0, 0.0, 0.1, args.warmup + args.steps)
        s.synchronize()
        print(f"profile case limiter: {n} steps, t = {t:.6e}")
        return 0
    if args.profile_case == "adjoint":
        # the adjoint bench's mesh and law: --steps recorded steps (every = 0)
        # and one backward pass, FP64
        import numpy as np
        from dgp import meshgen
        m = meshgen.tri_square(128, 128, 0.0, 10.0, 0.0, 10.0, jitter=0.15, seed=2)
        mesh = dgp.Mesh.from_arrays(2, m.vertices, m.cells, m.domain_tag, m.bfaces, m.btags)
        law = dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, vortex_params())
        s = dgp.Solver(mesh, law, 2, dgp.FP64)
        s.project(0.0)
        s.set_receivers(np.random.default_rng(4).uniform(0.5, 9.5, size=(64, 2)), np.zeros(64))
        dt = 0.5 * s.cfl_dt(0.1)
        J = s.forward_checkpointed(0.0, dt, args.steps, 0)
        g = s.backward()
        s.synchronize()
        print(f"profile case adjoint: {args.steps} steps, J = {J:.6e}, |g|max = {np.abs(g).max():.6e}")
        return 0
    if args.profile_case == "lts":
        # lts_bench's workload: local time stepping steps only
        m = lts_mesh()
        mesh = dgp.Mesh.from_arrays(2, m.vertices, m.cells, 100, m.bfaces, m.btags)
        law = dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, vortex_params())
        s = dgp.Solver(mesh, law, 3, dgp.FP64)
        s.set_p0_fallback(False)
        nb = s.set_time_stepping(dgp.STEPPING_LOCAL)
        t, n = s.run(0.0, 0.0, 0.1, args.warmup + args.steps)
        s.synchronize()
        print(f"profile case lts: {nb} bins, {n} steps, t = {t:.6e}, {s.launches_per_step()} launches per step")
        return 0
    if args.profile_case == "maxwell":
        from dgp import meshgen
        m3 = meshgen.tet_cube(48, 0.0, 1.0, jitter=0.1, seed=3, boundary_tag=40000)
        mesh3 = dgp.Mesh.from_arrays(3, m3.vertices, m3.cells, m3.domain_tag, m3.bfaces, m3.btags)
        law3 = dgp.Law(dgp.LAW_MAXWELL3D, dgp.FLUX_UPWIND, dgp.FIELD_TM110, dgp.law_params(cavity=1.0))
        s = dgp.Solver(mesh3, law3, 2, dgp.FP64)
        t, _ = s.run(0.0, 0.0, 0.1, args.warmup)
        t, n = s.run(t, 0.0, 0.1, args.steps)
        s.synchronize()
        print(f"profile case maxwell: {n} steps, t = {t:.6e}, block {s.block()[0]}")
        return 0
    m = make_mesh()
    mesh = dgp.Mesh.from_arrays(2, m.vertices, m.cells, 100, m.bfaces, m.btags)
    law = dgp.Law(dgp.LAW_EULER2D, dgp.FLUX_ROE, dgp.FIELD_VORTEX, vortex_params())
    prec = dgp.FP64 if args.profile_case == "fp64" else dgp.MIXED
    if args.block:
        dgp.tune_set(dgp.LAW_EULER2D, dgp.FLUX_ROE, 2, 3, prec, m.cells.shape[0], args.block)
    else:
        dgp.autotune(mesh, law, 3, prec, 0, iters=5)
    s = dgp.Solver(mesh, law, 3, prec)
    if args.tensor_cores:
        s.set_tensor_cores(True)
    t, _ = s.run(0.0, 0.0, 0.1, args.warmup)
    t, n = s.run(t, 0.0, 0.1, args.steps)
    s.synchronize()
    print(f"profile case {args.profile_case}: {n} steps, t = {t:.6e}, block {s.block()[0]}")
    return 0


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


if __name__ == "__main__":
    sys.exit(main())
