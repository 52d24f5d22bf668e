"""Benchmark: TeaLeaf 2D FP64 drop-in on B200 (solver iterations/s, HBM GB/s).

Workload (default): the 4096^2 drop-in case -- 8 seeded rectangles + 4
circles on [0,10]^2, reciprocal-density conductivity, CG to eps 1e-15,
dt 0.004 (tealeaf_b200.problems.dropin_2d). A "step" is one implicit
timestep (solve(), 2d/diffuse.c:22-80) of that problem.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--size 4096] [--solver cg|cheby|ppcg] [--workload ...]

B200 arm: value = solver iterations/s of the whole job (independent replicas
on N GPUs: the path does not shard), fields resident in HBM, timesteps run by
the device-resident solver loop (tl2d_solve_step). e2e = the same metric
through the C ABI with the step's inputs copied from pinned host buffers and
the energy field copied back every step; e2e_kernel_interface = the same,
with the timestep driven through the run_* kernel interface the way the
reference drivers call it.
At N=1 the line also carries the other configurations, each driver-measured
in the same run: `refine` (FP32 storage + FP64 refinement against FP64 at
8192^2), `dropin_8192` and `dropin_3d_256` (the FP64 CG drop-in at 8192^2 and
at 256^3), `adjoint` (the 3D adjoint at 256^3 with the 64^3 CPU-adjoint
check), `batch` (64 uneven problems in one launch against 64 sequential
FP64 solves) and `precond` (plain CG against the Jacobi-preconditioned CGs
at the headline size).
Reference arm (--impl reference): the reference omp3 CPU program on this
host's cores, bounded samples of the same workload: each timed timestep
capped at --cpu-cap CG iterations, warm-up timesteps at --warm-cap.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

# Compulsory bytes per interior cell of each kernel (each operand read or
# written once): w=Ap reads p,kx,ky writes w; u/r update reads u,p,r,w writes
# u,r; p update reads p,r writes p; ...
KERNEL_BYTES_PER_CELL = {
    "k_cg_w_fused": 48,      # reads p_old, r, kx, ky; writes p, w
    "k_cg_ur_fused": 48,     # reads u, p, r, w; writes u, r
    "k_cheby_trip": 56,      # reads u, p, u0, kx, ky; writes u, p (w, r only on norm trips)
    "k_ppcg_step": 64,       # reads sd, r, kx, ky, u; writes sd, r, u
    "k_blocked<cheby>": 56,  # per launch of L Chebyshev trips: reads u, p, u0, kx, ky; writes u, p
    "k_blocked<ppcg>": 64,   # per launch of L PPCG inner steps: reads sd, r, u, kx, ky; writes sd, r, u
    "k3_cg_w": 56,           # 3D: reads p_old, r, kx, ky, kz; writes p, w
    "k3_cg_ur": 48,          # 3D: reads u, p, r, w; writes u, r
    "k3_cheby_trip": 64,     # 3D: reads u, p, u0, kx, ky, kz; writes u, p
    "k3_ppcg_step": 72,      # 3D: reads sd, r, u, kx, ky, kz; writes sd, r, u
    "k3_blocked<cheby>": 64,  # 3D, per launch of L Chebyshev trips: reads u, p, u0, kx, ky, kz; writes u, p
    "k3_blocked<ppcg>": 72,   # 3D, per launch of L PPCG inner steps: reads sd, r, u, kx, ky, kz; writes sd, r, u
    "k_cg_calc_w": 32, "k_cg_calc_ur": 48, "k_cg_calc_p": 24,
    "k_cheby_sweep": 64, "k_add_p": 24, "k_ppcg_inner_a": 56, "k_ppcg_inner_b": 24,
    "k_norm2": 8, "k_residual": 40,
}
# Algorithmic bytes of one CG iteration per interior cell (12 FP64 streams:
# sweep 1 r,p,kx,ky -> p,w; sweep 2 u,p,r,w -> u,r).
CG_BYTES_PER_CELL_ITER = 96
FALLBACK_HBM_GBS = 6650.0


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_sample(tea_in: str, steps: int, cap: int, threads: int, dims: int = 2, warm_steps: int = 0,
                         warm_cap: int = 20):
    """Reference omp3 program (stock flags) on this host: per timed step
    (iterations, seconds). The deck must hold warm_steps + steps timesteps; the
    first warm_steps run capped at warm_cap iterations and are not returned,
    the others are capped at `cap`."""
    from oracle.oracle import run_reference  # the CPU baseline leg only
    res = run_reference(tea_in, dims=dims, suite="omp3", threads=threads, fast=True, max_iters=cap,
                        warm=(warm_steps, warm_cap) if warm_steps > 0 else None)
    out = []
    for s in res[warm_steps:warm_steps + steps]:
        it = sum(s.iterations.values())
        out.append((it, s.seconds))
    return out


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_info() -> dict:
    """The host CPU as lscpu reports it: model name and physical cores."""
    info = {"cpu_model": None, "physical_cores": None, "logical_cpus": os.cpu_count()}
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=20).stdout
        kv = {}
        for line in out.splitlines():
            if ":" in line:
                k, v = line.split(":", 1)
                kv.setdefault(k.strip(), v.strip())
        info["cpu_model"] = kv.get("Model name")
        cores, sockets = int(kv.get("Core(s) per socket", "0")), int(kv.get("Socket(s)", "0"))
        if cores and sockets:
            info["physical_cores"] = cores * sockets
    except Exception:
        pass
    return info


def workload_config(args) -> dict:
    """`config` of the drop-in line, identical on both arms."""
    n = args.size
    return {"workload": "dropin_2d_%d_%s" % (n, args.solver), "cells": n * n, "solver": args.solver,
            "eps": 1e-15, "dt": 0.004, "parallelism": "replicas",
            "l2": l2_note(8 * (n + 4) ** 2 * 8)}


def l2_note(working_set_bytes: float) -> str:
    if working_set_bytes > 126e6:
        return "no flush: working set %.2f GB > 126 MB L2" % (working_set_bytes / 1e9)
    return "no flush: working set %.1f MB fits in the 126 MB L2 (timings include L2 reuse)" % (working_set_bytes / 1e6)


def cpu_baseline_record(value, threads, sample) -> dict:
    d = {"value": value, "unit": "iter/s", "cores": threads, "kind": "reference", "sample": sample}
    d.update(cpu_info())
    return d


def bench_reference(args, rank, world):
    from tealeaf_b200 import problems
    if rank != 0:
        return None
    prob = problems.dropin_2d(args.size, seed=2, steps=args.warmup + args.steps, solver=args.solver)
    threads = host_threads()
    t0 = time.time()
    timed = cpu_reference_sample(prob.tea_in(), args.steps, args.cpu_cap, threads, warm_steps=args.warmup,
                                 warm_cap=args.warm_cap)
    iters = sum(i for i, _ in timed)
    secs = sum(t for _, t in timed)
    value = iters / secs if secs > 0 else 0.0
    cells = args.size * args.size
    sample = ("reference omp3 (oracle/_ref/harness2d_omp3_fast, stock flags, OMP_NUM_THREADS=%d): %d timed "
              "timesteps of the same deck, each capped at %d CG iterations, after %d warm-up timesteps capped "
              "at %d" % (threads, len(timed), args.cpu_cap, args.warmup, args.warm_cap))
    line = {
        "metric": "solver_iterations_per_s", "value": value, "unit": "iter/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * secs / max(1, len(timed)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded tea.in generator, dropin_2d seed 2)", "impl": "reference",
        "config": workload_config(args),
        "driver": "reference host, drivers and omp3 kernels (timestep loop of oracle/ref_harness.c)",
        "cells_iterations_per_s": value * cells,
        "cpu_baseline": cpu_baseline_record(value, threads, sample),
        "e2e": {"value": value, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": round(time.time() - t0, 2),
    }
    return line


def bench_b200(args, rank, world, local_rank):
    import ctypes as C

    import numpy as np
    import torch
    import torch.distributed as dist

    from tealeaf_b200 import abi, problems, replicas
    from tealeaf_b200.host import Host

    torch.cuda.set_device(local_rank)
    lib = abi.load(2)
    lib.tl2d_set_device(local_rank)
    prob = problems.dropin_2d(args.size, seed=2, steps=args.warmup + 2 * args.steps + 8, solver=args.solver)
    h = Host(prob.tea_in(), dims=2)
    if args.no_temporal_blocking:
        h.lib.tl2d_set_temporal_blocking(C.byref(h.chunk), 0)
    if args.no_tma:
        h.lib.tl2d_set_tma(C.byref(h.chunk), 0)
    stream = torch.cuda.ExternalStream(h.lib.tl2d_stream(C.byref(h.chunk)))
    cells = args.size * args.size
    interior_launch_cells = cells

    summary_every = h.cfg.summary_frequency

    def step(t):
        # the reference's solve() takes the field summary every summary_frequency steps
        if args.driver == "device":
            return h.solve_device(t, summary=(t % summary_every == 0))
        return h.solve(t)

    tt = 0
    for _ in range(args.warmup):
        step(tt)
        tt += 1
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()

    def timed_pass(profile):
        """K timesteps between two events on the suite stream; per-kernel
        event pairs only when `profile` (they cost the launch overlap)."""
        nonlocal tt
        h.lib.tl2d_profile_reset(C.byref(h.chunk))
        h.lib.tl2d_profile_enable(C.byref(h.chunk), 1 if profile else 0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        its = 0
        n0 = h.lib.tl2d_launch_count(C.byref(h.chunk))
        e0.record(stream)
        for _ in range(min(args.steps, args.profile_steps) if profile else args.steps):
            r = step(tt)
            its += sum(r.iterations.values())
            tt += 1
        e1.record(stream)
        torch.cuda.synchronize()
        n_launch = h.lib.tl2d_launch_count(C.byref(h.chunk)) - n0
        prof = {}
        idx = 0
        name = C.create_string_buffer(128)
        calls, kms = C.c_longlong(), C.c_double()
        while profile and h.lib.tl2d_profile_read(C.byref(h.chunk), idx, name, 128, C.byref(calls), C.byref(kms)):
            if calls.value:
                prof[name.value.decode()] = (calls.value, kms.value)
            idx += 1
        h.lib.tl2d_profile_enable(C.byref(h.chunk), 0)
        return e0.elapsed_time(e1), its, n_launch, prof

    # the headline: K steps, no per-kernel instrumentation, clocks sampled
    sampler = ClockSampler(local_rank)
    with sampler:
        ms, iters, launches, _ = timed_pass(False)
    # the per-kernel breakdown and roofline: the next K steps again, with
    # CUDA events around every launch on the suite stream
    if world > 1:
        dist.barrier()
    ms_prof, iters_prof, _, prof = timed_pass(True)

    # whole-job aggregate: max device time over ranks, iterations summed
    ms_max, iters_all = replicas.aggregate(ms, iters, world)
    value = iters_all / (ms_max / 1000.0)

    # e2e through the C ABI with host buffers: every step uploads the step's
    # inputs (density, energy) from pinned host memory, runs the timestep and
    # reads the energy field and the field summary back.
    init = Host(prob.tea_in(), dims=2)
    dens_h = torch.from_numpy(init.download("density")).pin_memory()
    en_h = torch.from_numpy(init.download("energy")).pin_memory()
    init.finalise()
    out_h = torch.empty_like(en_h).pin_memory()
    n = dens_h.numel()
    fn_up, fn_down = h.lib.tl2d_upload_field, h.lib.tl2d_download_field
    nsteps_e2e = max(1, min(args.steps, args.e2e_steps))

    def e2e(step_fn):
        its = 0
        ev = [torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        for _ in range(nsteps_e2e):
            fn_up(C.byref(h.chunk), C.byref(h.settings), 1, C.c_void_p(dens_h.data_ptr()), n)
            fn_up(C.byref(h.chunk), C.byref(h.settings), 3, C.c_void_p(en_h.data_ptr()), n)
            r = step_fn(0)
            # the step's result: the energy field back to pinned host memory
            fn_down(C.byref(h.chunk), C.byref(h.settings), 3, C.c_void_p(out_h.data_ptr()), n)
            abi.check(h.lib, 2)
            its += sum(r.iterations.values())
        ev[1].record(stream)
        torch.cuda.synchronize()
        return replicas.throughput(ev[0].elapsed_time(ev[1]), its, world)

    e2e_device = e2e(lambda t: h.solve_device(t, summary=False))
    e2e_kernel_interface = e2e(h.solve) if args.e2e_kernel_interface else None
    h.finalise()

    if rank != 0:
        return None
    peak, peak_kind = measured_peaks()
    # dominant kernel of the timed region
    dom = max(prof.items(), key=lambda kv: kv[1][1]) if prof else None
    roofline = None
    if dom:
        kname, (kcalls, kms_tot) = dom
        base = kname.split("<")[0]
        bpc = KERNEL_BYTES_PER_CELL.get(kname, KERNEL_BYTES_PER_CELL.get(base))
        if bpc:
            avg_s = kms_tot / kcalls / 1000.0
            achieved = bpc * interior_launch_cells / avg_s / 1e9
            roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                        "unit": "GB/s", "frac": achieved / peak, "traffic": traffic_per_launch(kname, cells),
                        "bytes_per_launch": bpc * interior_launch_cells, "avg_launch_ms": kms_tot / kcalls,
                        "timing": "CUDA events around every launch on the suite stream, over a second timed "
                                  "pass of %d steps (%.1f iter/s with the events in place)"
                                  % (min(args.steps, args.profile_steps), iters_prof / (ms_prof / 1000.0)),
                        "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                        else "fallback 6650 GB/s"}
    total_kernel_ms = sum(v[1] for v in prof.values())
    eff_gbs = CG_BYTES_PER_CELL_ITER * cells * value / max(1, world) / 1e9
    line = {
        "metric": "solver_iterations_per_s", "value": value, "unit": "iter/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded tea.in generator, dropin_2d seed 2)",
        "config": workload_config(args),
        "driver": "device-resident solver loop (tl2d_solve_step)" if args.driver == "device"
        else "host mirror of the reference drivers over run_*",
        "cells_iterations_per_s": value * cells,
        "hbm_effective_gbs_per_gpu": eff_gbs,
        "hbm_effective_frac_per_gpu": eff_gbs / peak,
        "roofline": roofline,
        "kernels": {k: {"calls": c, "ms": round(m, 3), "share": round(m / total_kernel_ms, 4)}
                    for k, (c, m) in sorted(prof.items(), key=lambda kv: -kv[1][1])},
        "gpu_launches": launches,
        "e2e": {"value": e2e_device, "unit": "iter/s",
                "h2d_bytes_per_step": 2 * n * 8, "d2h_bytes_per_step": n * 8 + 32, "steps": nsteps_e2e,
                "path": "C ABI: tl2d_upload_field (pinned host density, energy) -> tl2d_solve_step -> "
                        "tl2d_download_field (energy)"},
        "e2e_kernel_interface": None if e2e_kernel_interface is None else {
            "value": e2e_kernel_interface, "unit": "iter/s",
            "path": "same, timestep driven through the run_* kernel interface by the host mirror of "
                    "the reference drivers (two synchronous reductions per CG iteration)"},
        "clocks": sampler.summary(),
    }
    if world == 1 and args.refine_size > 0:
        line["refine"] = bench_refine(args.refine_size, peak)
    if world == 1 and not args.no_cpu_baseline:
        try:
            threads = host_threads()
            sprob = problems.dropin_2d(args.size, seed=2, steps=3, solver=args.solver)
            samples = cpu_reference_sample(sprob.tea_in(), 2, args.cpu_cap, threads, warm_steps=1,
                                           warm_cap=args.warm_cap)
            it_s = sum(i for i, _ in samples) / sum(t for _, t in samples)
            line["cpu_baseline"] = cpu_baseline_record(
                it_s, threads, "reference omp3 (stock flags) on this host: 2 timesteps of the same workload, "
                               "each capped at %d CG iterations, after 1 warm-up timestep" % args.cpu_cap)
        except Exception as exc:  # baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "error": str(exc)[:200]}
    if world == 1 and not args.no_extras:
        extras = (("dropin_8192", lambda: extra_dropin(8192, 2, peak)),
                  ("dropin_3d_256", lambda: extra_dropin(256, 3, peak)),
                  ("adjoint", lambda: adjoint_object(256, fd_cells=0, cpu_size=args.adjoint_cpu_size)),
                  ("batch", lambda: bench_batch(args)),
                  ("precond", lambda: precond_object(args.size, peak)))
        for key, fn in extras:
            try:
                line[key] = fn()
            except Exception as exc:   # an extra is reported, never required for the headline
                line[key] = {"error": str(exc)[:300]}
    return line


def extra_dropin(n: int, dims: int, peak: float, steps: int = 2, warm_cap: int = 50) -> dict:
    """The FP64 CG drop-in at another size (2D: the 8 rectangle + 4 circle
    deck; 3D: the 6-box deck of the adjoint configuration): one warm-up
    timestep capped at `warm_cap` iterations, then `steps` full timesteps of
    the device-resident loop to eps 1e-15, timed with CUDA events on the
    suite stream; the fraction counts 96 (2D) / 104 (3D) algorithmic bytes
    per cell and iteration."""
    import ctypes as C

    import torch

    from tealeaf_b200 import problems
    from tealeaf_b200.host import Host
    prob = (problems.dropin_2d(n, seed=2, steps=steps + 1, solver="cg") if dims == 2
            else problems.adjoint_3d(n, seed=4, steps=steps + 1))
    h = Host(prob.tea_in(), dims=dims)
    per_step = []
    try:
        stream = torch.cuda.ExternalStream(getattr(h.lib, "tl%dd_stream" % dims)(C.byref(h.chunk)))
        full = h.settings.max_iters
        h.settings.max_iters = warm_cap
        h.solve_device(0, summary=False)
        h.settings.max_iters = full
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(0)
        with sampler:
            e0.record(stream)
            for tt in range(1, steps + 1):
                per_step.append(sum(h.solve_device(tt, summary=False).iterations.values()))
            e1.record(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
    finally:
        h.finalise()
    cells = n ** dims
    value = sum(per_step) / (ms / 1000.0)
    bpc = CG_BYTES_PER_CELL_ITER if dims == 2 else 104
    gbs = bpc * cells * value / 1e9
    return {"metric": "solver_iterations_per_s", "value": value, "unit": "iter/s", "dtype": "f64",
            "workload": "dropin_%dd_%d_cg" % (dims, n), "cells": cells, "eps": prob.eps, "steps": steps,
            "iterations_per_step": per_step, "ms_per_step": ms / steps, "cells_iterations_per_s": value * cells,
            "bytes_per_cell_iteration": bpc, "hbm_effective_gbs": gbs, "frac_of_measured_hbm": gbs / peak,
            "warmup": "1 timestep capped at %d iterations" % warm_cap, "clocks": sampler.summary()}


def bench_dropin3d(args) -> dict:
    """The 3D FP64 drop-in: device-resident timesteps (tl3d_solve_step) of the
    seeded 3D case (6 boxes on [0,10]^3, recip-conductivity, eps 1e-15 on
    sqrt(r.r) as the reference 3D driver tests it), iterations/s; per-kernel
    breakdown from a second profiled pass; e2e through the C ABI with the
    step's density/energy uploaded from pinned host memory and the energy read
    back; the reference omp3 3D program as CPU baseline."""
    import ctypes as C

    import torch

    from tealeaf_b200 import problems
    from tealeaf_b200.host import Host
    n = args.size
    cells = n ** 3
    prob = problems.adjoint_3d(n, seed=4, steps=args.warmup + 2 * args.steps + 4).with_(solver=args.solver)
    h = Host(prob.tea_in(), dims=3)
    lib = h.lib
    if args.no_tma:
        lib.tl3d_set_tma(C.byref(h.chunk), 0)
    if args.no_temporal_blocking:
        lib.tl3d_set_temporal_blocking(C.byref(h.chunk), 0)
    stream = torch.cuda.ExternalStream(lib.tl3d_stream(C.byref(h.chunk)))
    tt = 0
    for _ in range(args.warmup):
        h.solve_device(tt, summary=False)
        tt += 1
    torch.cuda.synchronize()

    def timed(profile):
        nonlocal tt
        lib.tl3d_profile_reset(C.byref(h.chunk))
        lib.tl3d_profile_enable(C.byref(h.chunk), 1 if profile else 0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        its = 0
        n0 = lib.tl3d_launch_count(C.byref(h.chunk))
        e0.record(stream)
        for _ in range(args.steps):
            r = h.solve_device(tt, summary=(tt % h.cfg.summary_frequency == 0))
            its += sum(r.iterations.values())
            tt += 1
        e1.record(stream)
        torch.cuda.synchronize()
        launches = lib.tl3d_launch_count(C.byref(h.chunk)) - n0
        prof, idx = {}, 0
        name = C.create_string_buffer(128)
        calls, kms = C.c_longlong(), C.c_double()
        while profile and lib.tl3d_profile_read(C.byref(h.chunk), idx, name, 128, C.byref(calls), C.byref(kms)):
            if calls.value:
                prof[name.value.decode()] = (calls.value, kms.value)
            idx += 1
        lib.tl3d_profile_enable(C.byref(h.chunk), 0)
        return e0.elapsed_time(e1), its, launches, prof

    sampler = ClockSampler(0)
    with sampler:
        ms, iters, launches, _ = timed(False)
    ms_p, iters_p, _, prof = timed(True)
    value = iters / (ms / 1000.0)
    peak, peak_kind = measured_peaks()
    kname, (kc, kms_tot) = max(prof.items(), key=lambda kv: kv[1][1])
    bpc = KERNEL_BYTES_PER_CELL.get(kname, KERNEL_BYTES_PER_CELL.get(kname.split("<")[0]))
    roofline = None
    if bpc:
        achieved = bpc * cells / (kms_tot / kc / 1000.0) / 1e9
        roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "traffic": traffic_per_launch(kname, cells),
                    "bytes_per_launch": bpc * cells, "avg_launch_ms": kms_tot / kc,
                    "timing": "CUDA events around every launch on the suite stream, second timed pass of "
                              "%d steps (%.1f iter/s with the events in place)" % (args.steps, iters_p / (ms_p / 1e3)),
                    "peak_source": peak_kind}
    # e2e: host buffers in, energy out, every step
    init = Host(prob.tea_in(), dims=3)
    dens_h = torch.from_numpy(init.download("density")).pin_memory()
    en_h = torch.from_numpy(init.download("energy")).pin_memory()
    init.finalise()
    out_h = torch.empty_like(en_h).pin_memory()
    nel = dens_h.numel()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    its_e = 0
    for _ in range(max(1, min(args.steps, args.e2e_steps))):
        lib.tl3d_upload_field(C.byref(h.chunk), C.byref(h.settings), 1, C.c_void_p(dens_h.data_ptr()), nel)
        lib.tl3d_upload_field(C.byref(h.chunk), C.byref(h.settings), 3, C.c_void_p(en_h.data_ptr()), nel)
        r = h.solve_device(0, summary=False)
        lib.tl3d_download_field(C.byref(h.chunk), C.byref(h.settings), 3, C.c_void_p(out_h.data_ptr()), nel)
        its_e += sum(r.iterations.values())
    e1.record(stream)
    torch.cuda.synchronize()
    e2e = its_e / (e0.elapsed_time(e1) / 1000.0)
    h.finalise()
    tot = sum(v[1] for v in prof.values())
    line = {
        "metric": "solver_iterations_per_s", "value": value, "unit": "iter/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded tea.in generator, adjoint_3d seed 4)",
        "config": {"workload": "dropin_3d_%d_%s" % (n, args.solver), "cells": cells, "solver": args.solver,
                   "eps": prob.eps, "dt": 0.004, "parallelism": "replicas",
                   "l2": "no flush: working set %.2f GB > 126 MB L2" % (8 * (n + 4) ** 3 * 8 / 1e9),
                   "driver": "device-resident solver loop (tl3d_solve_step)"},
        "cells_iterations_per_s": value * cells,
        "roofline": roofline,
        "kernels": {k: {"calls": c, "ms": round(m, 3), "share": round(m / tot, 4)}
                    for k, (c, m) in sorted(prof.items(), key=lambda kv: -kv[1][1])},
        "gpu_launches": launches,
        "e2e": {"value": e2e, "unit": "iter/s", "h2d_bytes_per_step": 2 * nel * 8, "d2h_bytes_per_step": nel * 8,
                "path": "C ABI: tl3d_upload_field -> tl3d_solve_step -> tl3d_download_field"},
        "clocks": sampler.summary(),
    }
    if not args.no_cpu_baseline:
        try:
            threads = host_threads()
            sprob = prob.with_(end_step=3)
            samples = cpu_reference_sample(sprob.tea_in(), 2, args.cpu_cap, threads, dims=3, warm_steps=1,
                                           warm_cap=args.warm_cap)
            it_s = sum(i for i, _ in samples) / sum(t for _, t in samples)
            line["cpu_baseline"] = cpu_baseline_record(
                it_s, threads, "reference omp3 3D (stock flags): 2 timesteps of the same workload, each capped "
                               "at %d iterations, after 1 warm-up timestep" % args.cpu_cap)
        except Exception as exc:
            line["cpu_baseline"] = {"value": None, "error": str(exc)[:200]}
    return line


def bench_refine(n: int, peak: float) -> dict:
    """The iterative-refinement form against FP64 on identical inputs: one
    timestep of the seeded mixed-precision case (16 rectangles, seed 3), each
    solved to the relative FP64 residual 1e-10 (tl2d_refine_solve_step), with
    CG and with PPCG (presteps 30, 10 inner steps; the deck's switch test and
    an early switch)."""
    from tealeaf_b200 import problems
    from tealeaf_b200.host import Host
    tol = 1e-10
    prob = problems.mixed_2d(n, seed=3, steps=1)
    out = {"workload": "mixed_2d_%d (16 rectangles, seed 3), timestep 1" % n, "rel_tol": tol,
           "metric": "device time of the timestep to rel_tol (ms)"}

    def run(p, prec):
        h = Host(p.tea_in(), dims=2)
        try:
            return h.refine_step(0, tol, prec)
        finally:
            h.finalise()

    temps = {}
    for prec in (64, 32):
        r = run(prob, prec)
        bpc = 96 if prec == 64 else 48
        gbs = bpc * n * n * r.iterations / (r.device_ms / 1000.0) / 1e9
        out["fp%d" % prec] = {"ms": r.device_ms, "iterations": r.iterations,
                              "residual_updates": r.residual_updates, "rel_residual": r.rel_residual,
                              "converged": r.converged, "cg_gbs_effective": gbs, "cg_frac_of_peak": gbs / peak}
        temps[prec] = r.summary[3]
    out["time_ratio_fp32_over_fp64"] = out["fp32"]["ms"] / out["fp64"]["ms"]
    out["temp_rel_diff_fp32_vs_fp64"] = temps[32] / temps[64] - 1.0
    # PPCG with the deck's switch test (presteps 30, r.r < 1), and with
    # errswitch and epslim 1e30 (the switch after 21 CG trips)
    for key, p in (("ppcg", prob.with_(solver="ppcg")),
                   ("ppcg_errswitch", prob.with_(solver="ppcg", error_switch=True, eps_lim=1e30))):
        pp = {}
        for prec in (64, 32):
            r = run(p, prec)
            pp["fp%d" % prec] = {"ms": r.device_ms, "iterations": r.iterations, "cg_trips": r.cg_trips,
                                 "residual_updates": r.residual_updates, "rel_residual": r.rel_residual,
                                 "converged": r.converged}
            temps[key + str(prec)] = r.summary[3]
        pp["time_ratio_fp32_over_fp64"] = pp["fp32"]["ms"] / pp["fp64"]["ms"]
        pp["temp_rel_diff_fp32_vs_fp64_cg"] = temps[key + "32"] / temps[64] - 1.0
        out[key] = pp
    return out


def bench_adjoint(args) -> dict:
    """The 3D adjoint form at `--size`^3 (see adjoint_object)."""
    return adjoint_object(args.size, args.fd_cells, args.adjoint_cpu_size)


def adjoint_object(n: int, fd_cells: int, cpu_size: int) -> dict:
    """The 3D adjoint form: dJ/dlog(density) for J = sum over [6,9]^3 of
    volume*density*u after 20 CG timesteps (checkpoints every 5) on the seeded
    adjoint case, timed on the device; checked against central differences
    (h = 1e-6) at `fd_cells` seeded cells of the same mesh and against the
    oracle's FP64 CPU adjoint at `cpu_size`^3."""
    import numpy as np

    from tealeaf_b200 import problems
    from tealeaf_b200.config import read_config
    from tealeaf_b200.host import Host
    steps, every, tol, h = 20, 5, 1e-12, 1e-6
    box = [6.0, 9.0, 6.0, 9.0, 6.0, 9.0]
    prob = problems.adjoint_3d(n, seed=4, steps=steps)
    host = Host(prob.tea_in(), dims=3)
    hd = host.cfg.halo_depth
    rho0, e0 = host.download("density"), host.download("energy")
    J, g, st = host.adjoint_gradient(steps, every, box, tol)
    line = {"metric": "adjoint_gradient_seconds", "value": st.device_ms / 1000.0, "unit": "s",
            "higher_is_better": False, "n_gpus": 1, "dtype": "f64", "data": "synthetic (seeded tea.in generator, "
            "adjoint_3d seed 4)",
            "config": {"workload": "adjoint_3d_%d" % n, "cells": n ** 3, "steps": steps, "checkpoint_every": every,
                       "box": box, "adjoint_rel_tol": tol, "forward_eps": prob.eps},
            "J": J, "forward_steps": st.forward_steps, "forward_iters": st.forward_iters,
            "adjoint_iters": st.adjoint_iters, "checkpoints": st.checkpoints,
            "cg_cells_iterations_per_s": n ** 3 * (st.forward_iters + st.adjoint_iters) / (st.device_ms / 1000.0)}
    gf = g.ravel()

    def objective(cell, scale):
        rho = rho0.copy()
        k, j, i = cell % n, (cell // n) % n, cell // (n * n)
        rho[i + hd, j + hd, k + hd] *= np.exp(scale)
        host.upload("density", rho)
        host.upload("energy", e0)
        for tt in range(steps):
            host.solve_device(tt, summary=False)
        u, v, d = host.download("u"), host.download("volume"), host.download("density")
        c = host.cfg
        sl = (slice(hd, hd + n),) * 3
        xs = c.grid_x_min + c.dx * (np.arange(n) + 0.5)
        inb = (xs >= box[0]) & (xs <= box[1])
        m = inb[:, None, None] & inb[None, :, None] & inb[None, None, :]
        return float(np.sum((v[sl] * d[sl] * u[sl])[m]))

    if fd_cells > 0:
        rng = np.random.default_rng(4)
        top = np.argsort(-np.abs(gf))[: max(1, gf.size // 100)]
        cells = list(rng.choice(top, fd_cells // 2, replace=False)) + \
            list(rng.integers(0, gf.size, fd_cells - fd_cells // 2))
        noise = 8.0 * np.finfo(float).eps * abs(J) / (2 * h)
        rows = []
        for c in cells:
            fd = (objective(int(c), h) - objective(int(c), -h)) / (2 * h)
            rows.append((int(c), float(gf[c]), fd, abs(fd - gf[c]) / abs(gf[c]) if gf[c] else float("inf")))
        strong = [r for r in rows if abs(r[1]) > 1e4 * noise]
        line["fd_check"] = {"h": h, "cells": len(rows), "noise_floor_abs": noise,
                            "max_rel_err_strong_cells": max((r[3] for r in strong), default=None),
                            "strong_cells": len(strong),
                            "max_abs_err_over_noise": max(abs(r[2] - r[1]) / noise for r in rows),
                            "per_cell": [{"cell": r[0], "adjoint": r[1], "fd": r[2], "rel": r[3]} for r in rows]}
    host.finalise()
    if cpu_size > 0:
        m = cpu_size
        small = problems.adjoint_3d(m, seed=4, steps=steps)
        hs = Host(small.tea_in(), dims=3)
        try:
            Jg, gg, _ = hs.adjoint_gradient(steps, every, box, tol)
        finally:
            hs.finalise()
        from oracle.oracle import OracleLib  # the CPU adjoint comparison only
        cfg, states = read_config(small.tea_in(), 3)
        t0 = time.time()
        Jc, gc = OracleLib().adjoint3d(cfg, states, box, tol)
        line["cpu_adjoint_check"] = {"mesh": m, "J_rel_diff": Jg / Jc - 1.0,
                                     "grad_rel_norm_diff": float(np.linalg.norm(gg - gc) / np.linalg.norm(gc)),
                                     "cpu_seconds": time.time() - t0}
    return line


def bench_batch(args) -> dict:
    """The batched form: one timestep of 64 seeded 2D problems (sides
    log-uniform in [128, 2048], 3 rectangles each, CG to eps 1e-12) as one
    graph-captured persistent launch with the autotuned tile shape, against
    the same 64 timesteps solved one after another by the FP64 device driver."""
    import ctypes as C

    import torch

    from tealeaf_b200 import problems
    from tealeaf_b200.batch import Batch
    from tealeaf_b200.host import Host
    probs = problems.batched_2d(args.batch_count, seed=5)
    cells = sum(p.cells[0] * p.cells[1] for p in probs)
    b = Batch([p.tea_in() for p in probs])
    try:
        tuned = b.tune(trial_iters=args.tune_iters)
        st = b.step()
        it, rr, conv = b.results()
        sums = b.summaries()
    finally:
        b.close()
    seq_ms, seq_iters, worst = 0.0, 0, 0.0
    for p, s in zip(probs, sums):
        h = Host(p.tea_in(), dims=2)
        try:
            stream = torch.cuda.ExternalStream(h.lib.tl2d_stream(C.byref(h.chunk)))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            r = h.solve_device(0, summary=False)
            e1.record(stream)
            torch.cuda.synchronize()
            seq_ms += e0.elapsed_time(e1)
            seq_iters += r.iterations["CG"]
            ref = h.field_summary()
            worst = max(worst, abs(s[3] / ref[3] - 1.0))
        finally:
            h.finalise()
    # algorithmic bytes of the FP32 CG sweeps: 24 B per cell in w = A p (r, p, kx, ky -> p, w) and 24 in the
    # u/r update (xs, p, r, w -> xs, r), per problem over its own iterations; the occasional FP64 fold and
    # residual replacement are left out, so this is a lower bound on the bytes moved
    alg = sum(48.0 * p.cells[0] * p.cells[1] * int(n) for p, n in zip(probs, it))
    peak, peak_kind = measured_peaks()
    achieved = alg / (st.device_ms * 1e-3) / 1e9
    return {"metric": "batched_timestep_ms", "value": st.device_ms, "unit": "ms", "higher_is_better": False,
            "roofline": {"bound": "hbm", "kernel": "k_batch_cg", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "algorithmic_bytes": alg,
                         "bytes_rule": "48 B per cell-iteration (FP32 w and u/r sweeps), per problem over its "
                                       "own iterations, over the batched step's device time",
                         "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else "fallback 6650 GB/s"},
            "n_gpus": 1, "dtype": "f32 vectors, f64 reductions/solution", "data": "synthetic (seeded tea.in "
            "generator, batched_2d seed 5)",
            "config": {"workload": "batched_2d_%d" % len(probs), "problems": len(probs), "cells": cells,
                       "eps": 1e-12, "graph": bool(st.graph)},
            "autotuner": tuned, "converged": st.converged, "max_iterations": st.max_iterations,
            "total_iterations": st.total_iterations, "kernel_iterations": st.kernel_iterations,
            "max_fp64_rr": float(rr.max()),
            "sequential_fp64": {"ms": seq_ms, "total_iterations": seq_iters,
                                "path": "tl2d_solve_step per problem, one after another"},
            "speedup_vs_sequential": seq_ms / st.device_ms,
            "temp_max_rel_diff_vs_sequential": worst}


def precond_object(n: int, peak: float, steps: int = 1, warm_cap: int = 50) -> dict:
    """The Jacobi preconditioners of the device-resident CG against plain CG
    on the drop-in deck at n^2: per variant, a warm-up timestep capped at
    `warm_cap` iterations on a throwaway chunk, then the first `steps`
    timesteps of a fresh chunk (the same initial state for every variant) to
    eps 1e-15, timed with CUDA events on the suite stream (iterations, ms per
    timestep, and the temperature against plain CG's)."""
    import ctypes as C

    import torch

    from tealeaf_b200 import problems
    from tealeaf_b200.host import Host
    out = {"workload": "dropin_2d_%d_cg, preconditioner none / jac_diag / jac_block" % n, "cells": n * n,
           "bytes_per_cell_iteration": {"none": 96, "jac_diag": 112, "jac_block": 120}}
    for pc in ("none", "jac_diag", "jac_block"):
        prob = problems.dropin_2d(n, seed=2, steps=steps, solver="cg").with_(preconditioner=pc)
        w = Host(prob.tea_in(), dims=2)
        try:
            w.settings.max_iters = warm_cap
            w.solve_device(0, summary=False)
        finally:
            w.finalise()
        h = Host(prob.tea_in(), dims=2)
        try:
            stream = torch.cuda.ExternalStream(h.lib.tl2d_stream(C.byref(h.chunk)))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            its = []
            e0.record(stream)
            for tt in range(steps):
                its.append(h.solve_device(tt, summary=False).iterations["CG"])
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            temp = h.field_summary()[3]
        finally:
            h.finalise()
        bpc = out["bytes_per_cell_iteration"][pc]
        out[pc] = {"ms_per_step": ms, "iterations_per_step": its, "temp": temp,
                   "hbm_effective_gbs": bpc * n * n * sum(its) / steps / (ms / 1000.0) / 1e9}
    for pc in ("jac_diag", "jac_block"):
        out[pc]["temp_rel_diff_vs_none"] = abs(out[pc]["temp"] / out["none"]["temp"] - 1.0)
        out[pc]["time_ratio_vs_none"] = out[pc]["ms_per_step"] / out["none"]["ms_per_step"]
        out[pc]["iteration_ratio_vs_none"] = sum(out[pc]["iterations_per_step"]) / sum(out["none"]["iterations_per_step"])
    return out


def bench_refine_case(args) -> dict:
    """One refinement timestep of the mixed-precision deck (16 rectangles,
    seed 3) at `--size`, solved to the FP64 relative residual 1e-10 in
    `--precision` 32 or 64, with `--solver` cg or ppcg (`--errswitch`: the
    switch after 21 CG trips, epslim 1e30) and an optional `--max-iters` cap.
    The case the refinement profiles are captured on."""
    import ctypes as C

    from tealeaf_b200 import problems
    from tealeaf_b200.host import Host
    prob = problems.mixed_2d(args.size, seed=3, steps=1).with_(solver=args.solver)
    if args.errswitch:
        prob = prob.with_(error_switch=True, eps_lim=1e30)
    if args.max_iters > 0:
        prob = prob.with_(max_iters=args.max_iters)
    h = Host(prob.tea_in(), dims=2)
    try:
        if args.no_tma:
            h.lib.tl2d_set_tma(C.byref(h.chunk), 0)
        r = h.refine_step(0, 1e-10, args.precision)
    finally:
        h.finalise()
    return {"metric": "refine_timestep_ms", "value": r.device_ms, "unit": "ms", "higher_is_better": False,
            "n_gpus": 1, "dtype": "f%d storage, f64 reductions/solution" % args.precision,
            "data": "synthetic (seeded tea.in generator, mixed_2d seed 3)",
            "config": {"workload": "mixed_2d_%d_%s%s" % (args.size, args.solver, "_errswitch" if args.errswitch else ""),
                       "rel_tol": 1e-10, "max_iters": prob.max_iters, "precision": args.precision},
            "iterations": r.iterations, "cg_trips": r.cg_trips, "residual_updates": r.residual_updates,
            "rel_residual": r.rel_residual, "converged": r.converged}


def traffic_per_launch(kernel: str, cells: int):
    """DRAM bytes per launch from the committed ncu summary (scaled per cell), if any."""
    p = REPO / "profiles" / "ncu_traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
        per_cell = d["bytes_per_cell"].get(kernel, d["bytes_per_cell"].get(kernel.split("<")[0]))
        return None if per_cell is None else per_cell * cells
    except Exception:
        return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=4096)
    ap.add_argument("--solver", default="cg", choices=["cg", "cheby", "ppcg"])
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-cap", type=int, default=1000,
                    help="reference CPU samples: CG iterations per timed timestep")
    ap.add_argument("--warm-cap", type=int, default=20,
                    help="reference CPU samples: CG iterations per warm-up timestep")
    ap.add_argument("--profile-steps", type=int, default=5,
                    help="timesteps of the second pass with per-launch events (kernel shares, roofline)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="default line without the 8192^2 / 3D 256^3 drop-in, adjoint and batch objects")
    ap.add_argument("--refine-size", type=int, default=8192,
                    help="mesh of the FP32-refinement vs FP64 comparison (0: skip)")
    ap.add_argument("--driver", default="device", choices=["device", "run"])
    ap.add_argument("--workload", default="dropin", choices=["dropin", "dropin3d", "adjoint", "batch", "refine", "precond"],
                    help="dropin: the 2D FP64 drop-in line (default); adjoint: the 3D adjoint form; "
                         "batch: the batched form; refine: one refinement timestep (--precision, --errswitch); "
                         "precond: plain CG against the Jacobi-preconditioned CGs")
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--errswitch", action="store_true")
    ap.add_argument("--max-iters", type=int, default=0)
    ap.add_argument("--batch-count", type=int, default=64)
    ap.add_argument("--tune-iters", type=int, default=30)
    ap.add_argument("--fd-cells", type=int, default=32)
    ap.add_argument("--adjoint-cpu-size", type=int, default=64)
    ap.add_argument("--e2e-kernel-interface", type=int, default=1)
    ap.add_argument("--no-temporal-blocking", action="store_true",
                    help="Chebyshev/PPCG: one launch per trip instead of shared-memory blocks")
    ap.add_argument("--no-tma", action="store_true",
                    help="stencil sweeps read their operands with per-thread loads instead of TMA tile loads")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "batch":
        line = bench_batch(args) if rank == 0 else None
    elif args.workload == "refine":
        line = bench_refine_case(args) if rank == 0 else None
    elif args.workload == "precond":
        line = precond_object(args.size, measured_peaks()[0], steps=args.steps) if rank == 0 else None
    elif args.workload == "dropin3d":
        if args.size == 4096:
            args.size = 256
        line = bench_dropin3d(args) if rank == 0 else None
    elif args.workload == "adjoint":
        if args.size == 4096:
            args.size = 256
        line = bench_adjoint(args) if rank == 0 else None
    elif args.impl == "reference":
        line = bench_reference(args, rank, world)
    else:
        if world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        line = bench_b200(args, rank, world, local_rank)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
