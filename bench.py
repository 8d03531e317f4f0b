#!/usr/bin/env python
"""Throughput of the multiphase-field time step on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: 256^3 periodic grain growth with driving force -- 2000 seeded Voronoi grains, eta = 6 dx,
per-grain-pair sigma ~ U[0.8, 1.2], mu = 1, per-grain dG ~ U[0, 0.05], D3Q27 (LB) Laplacian,
dt = 0.08 (synthetic, seeded; the grid does not fit any public dataset).  One "step" is one full
time step of the grid; W untimed steps from the Voronoi start, then K timed steps (steps W+1..W+K).

`value` is voxel-updates/s of the FP64 form (the parity drop-in, the reference's own precision)
with the state resident in HBM; `e2e` is the same metric through the C ABI from pinned host
buffers: upload of the initial state, per step the driving-force upload and the grain-volume
download, and the final state download.  The FP32 form is measured the same way under "fp32",
with its error against the FP64 form after the same W+K steps ("fp32.error").

`--impl reference` times the reference's own OpenMP implementation (oracle/_ref, OpenPhase built
from its sources) on all host threads over the same step window W+1..W+K.

Multi-GPU (torchrun, one rank per GPU): the grid is cut into x-slabs, one per rank, with an NCCL
halo-plane exchange and an all-reduce of the grain volumes every step (strong scaling of the same
workload); the timed region is bracketed by barriers and the device time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "voxel-updates/s & HBM% peak: FP32 vs FP64 GPU at |Δφ|≤1e-4; adjoint/fwd ratio"
UNIT = "voxel-updates/s"


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(precision):
    """DRAM bytes per launch of the step kernel from the committed ncu summary, if present."""
    p = ROOT / "profiles" / "step_kernel_traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
        return d.get(precision)
    except (ValueError, KeyError):
        return None


class ClockSampler:
    """Samples SM clock and clock-event reasons through NVML while the timed region runs."""

    REASONS = {
        0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
        0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
        0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting",
    }

    def __init__(self, device_index):
        self.samples = []
        self.reasons = 0
        self.max_mhz = None
        self._stop = threading.Event()
        self._thread = None
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nvml = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:  # noqa: BLE001 - clocks are reported as unavailable
            self.ok = False

    def _run(self):
        nv = self._nvml
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                self.reasons |= int(nv.nvmlDeviceGetCurrentClocksEventReasons(self._h))
            except Exception:  # noqa: BLE001
                pass
            time.sleep(0.005)

    def __enter__(self):
        if self.ok:
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._thread:
            self._thread.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unavailable"]}
        names = [n for b, n in self.REASONS.items() if self.reasons & b and n != "gpu_idle"]
        return {"sm_mhz": float(statistics.median(self.samples)), "sm_max_mhz": self.max_mhz,
                "reasons": names, "samples": len(self.samples)}


def build_inputs(case, threads=0):
    t = time.time()
    state = case.initial_state(threads)
    sigma = case.pair_sigma()
    dg = case.driving_force()
    return state, sigma, dg, time.time() - t


def device_run(case, precision, k_slots, steps, warmup, device, state, sigma, dg, dist, keep_final=False):
    """Device-resident throughput: W warm-up steps, then exactly K timed steps.  keep_final: also
    return the final state and grain volumes (downloaded after the clock stopped)."""
    import torch
    from openphase_b200.context import Context

    ctx = Context(case.nx, case.ny, case.nz, dx=case.dx, iwidth=case.iwidth, stencil=case.stencil,
                  gradient_stencil=case.gradient_stencil, precision=precision, k_slots=k_slots, device=device)
    ctx.set_model([[case.sigma]], [[case.mu]], limit=[[case.limit]], limiting=case.limiting,
                  regularization=case.regularization)
    ctx.set_grains(case.ngrains)
    ctx.set_pair_table(sigma, None)
    ctx.set_driving_force(dg)
    ctx.upload(*state)
    ctx.finalize_initialization()
    ctx.step(case.dt, warmup)
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    s0 = ctx.stats()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(device)
    ctx.set_timing(True)
    with ClockSampler(device) as clk:
        e0.record(stream)
        ctx.step_async(case.dt, steps)
        e1.record(stream)
        torch.cuda.synchronize(device)
    status = ctx.sync()
    if dist is not None:
        dist.barrier()
    elapsed_ms = e0.elapsed_time(e1)
    s1 = ctx.stats()
    ctx.set_timing(False)
    entries_in = s1["entries_in_total"] - s0["entries_in_total"]
    entries_out = s1["entries_out_total"] - s0["entries_out_total"]
    wide = s1["wide_total"] - s0["wide_total"]
    final = (ctx.download(), ctx.grains()["volume"]) if keep_final else None
    ctx.close()
    return {"final": final,
        "elapsed_ms": elapsed_ms, "kernel_ms": s1["timed_kernel_ms"], "timed_steps": s1["timed_launches"],
        "classify_ms": s1["timed_classify_ms"], "gpu_launches": s1["kernel_launches"] - s0["kernel_launches"],
        "entries_in": entries_in, "entries_out": entries_out, "wide": wide, "status": status | s1["status"],
        "clocks": clk.summary(),
    }


def slab_run(case, precision, k_slots, steps, warmup, device, state, sigma, dg, dist):
    """Slab decomposition over the ranks (NCCL halo exchange and grain-volume all-reduce): strong
    scaling of the workload; the timed region is bracketed by barriers, CUDA events on the rank's
    step stream."""
    import torch
    from openphase_b200 import slab

    comm = slab.DistComm(dist)
    st = slab.SlabStepper(case, comm.rank, comm.world, precision=precision, k_slots=k_slots, device=device,
                          state=state, sigma=sigma, dg=dg)
    slab.initialize(st, comm)
    slab.step(st, comm, case.dt, warmup)
    ctx = st.ctx
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0 = ctx.stats()
    dist.barrier()
    torch.cuda.synchronize(device)
    ctx.set_timing(True)
    with ClockSampler(device) as clk:
        e0.record(stream)
        status = slab.step(st, comm, case.dt, steps)
        e1.record(stream)
        torch.cuda.synchronize(device)
    dist.barrier()
    s1 = ctx.stats()
    ctx.set_timing(False)
    out = {
        "elapsed_ms": e0.elapsed_time(e1), "kernel_ms": s1["timed_kernel_ms"], "timed_steps": s1["timed_launches"],
        "classify_ms": s1["timed_classify_ms"], "gpu_launches": s1["kernel_launches"] - s0["kernel_launches"],
        "entries_in": s1["entries_in_total"] - s0["entries_in_total"],
        "entries_out": s1["entries_out_total"] - s0["entries_out_total"],
        "wide": s1["wide_total"] - s0["wide_total"], "status": status | s1["status"], "clocks": clk.summary(),
        "local_voxels": st.nxl * case.ny * case.nz,
    }
    ctx.close()
    return out


def scale_run(steps, warmup, device, k_slots=16, threads=0):
    """The 512^3 scale set-up (134M voxels, 20000 Voronoi grains, eta = 6, sigma ~ U[0.8, 1.2] per
    grain pair generated on the device, dG ~ U[0, 0.05], dt = 0.08): device-resident step time of
    both forms over steps warmup+1 .. warmup+steps.  The checkpointed adjoint is not run at this
    size: sqrt(1000)-interval checkpointing keeps about 65 states of 13 GB (K = 16, FP32)."""
    import torch
    from openphase_b200.cases import scale_512
    from openphase_b200.context import Context

    case = scale_512()
    t = time.time()
    state = case.initial_state(threads)
    t_init = time.time() - t
    dg = case.driving_force()
    lo, span = case.sigma_pairs
    out = {"workload": case.name, "grid": [case.nx, case.ny, case.nz], "grains": case.ngrains, "k_slots": k_slots,
           "pair_energies": "generated on the device (opgpu_set_pair_hash)", "initial_state_seconds": round(t_init, 1),
           "adjoint": "not run: sqrt(1000)-interval checkpointing needs about 65 states of 13 GB (K = 16, FP32)"}
    for precision in ("fp64", "fp32"):
        s = 4 if precision == "fp32" else 8
        ctx = Context(case.nx, case.ny, case.nz, dx=case.dx, iwidth=case.iwidth, stencil=case.stencil,
                      gradient_stencil=case.gradient_stencil, precision=precision, k_slots=k_slots, device=device)
        ctx.set_model([[case.sigma]], [[case.mu]], limit=[[case.limit]], limiting=case.limiting,
                      regularization=case.regularization)
        ctx.set_grains(case.ngrains)
        ctx.set_pair_hash(case.seed, lo, span)
        ctx.set_driving_force(dg)
        ctx.upload(*state)
        ctx.finalize_initialization()
        ctx.step(case.dt, warmup)
        stream = torch.cuda.ExternalStream(ctx.stream, device=device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0 = ctx.stats()
        torch.cuda.synchronize(device)
        with ClockSampler(device) as clk:
            e0.record(stream)
            ctx.step_async(case.dt, steps)
            e1.record(stream)
            torch.cuda.synchronize(device)
        status = ctx.sync()
        ms = e0.elapsed_time(e1)
        s1 = ctx.stats()
        wide = (s1["wide_total"] - s0["wide_total"]) / steps
        ctx.close()
        out[precision] = {"value": case.n * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps,
                          "state_bytes_per_buffer": case.n * (1 + k_slots * (2 + s)),
                          "wide_fraction": wide / case.n, "status": int(status), "clocks": clk.summary(),
                          "roofline_frac": (wide * 2 * (1 + 8 * (2 + s)) + case.n) / (ms / steps / 1e3) / 1e9
                                           / measured_peaks()[0]}
    out["fp32_over_fp64"] = out["fp32"]["value"] / out["fp64"]["value"]
    return out


def e2e_run(case, precision, k_slots, steps, device, state, sigma, dg):
    """End to end through the C ABI with pinned host buffers; host<->device copies inside the clock."""
    import torch
    from openphase_b200.context import Context

    counts, idx, val = state
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    h_counts, h_idx, h_val, h_dg = pin(counts.astype(np.int32)), pin(idx.astype(np.int32)), pin(val), pin(dg)
    h_vol = torch.empty(case.ngrains, dtype=torch.float64).pin_memory().numpy()
    # pinned buffers for the final state (its entry count stays below 1.5x the initial one here;
    # a larger state is downloaded into fresh host memory inside the clock)
    cap = int(1.5 * idx.size) + 4096
    h_out = (torch.empty(case.n, dtype=torch.int32).pin_memory().numpy(),
             torch.empty(cap, dtype=torch.int32).pin_memory().numpy(),
             torch.empty(cap, dtype=torch.float64).pin_memory().numpy())
    ctx = Context(case.nx, case.ny, case.nz, dx=case.dx, iwidth=case.iwidth, stencil=case.stencil,
                  gradient_stencil=case.gradient_stencil, precision=precision, k_slots=k_slots, device=device)
    ctx.set_model([[case.sigma]], [[case.mu]], limit=[[case.limit]], limiting=case.limiting,
                  regularization=case.regularization)
    ctx.set_grains(case.ngrains)
    ctx.set_pair_table(sigma, None)
    torch.cuda.synchronize(device)
    from openphase_b200._lib import lib, ptr
    L = lib()
    t0 = time.perf_counter()
    ctx.set_driving_force(h_dg)
    ctx.upload(h_counts, h_idx, h_val)
    ctx.finalize_initialization()
    for _ in range(steps):
        ctx.set_driving_force(h_dg)                       # the step's input: per-grain driving forces
        ctx.step(case.dt, 1)
        L.opgpu_grains(ctx.h, ptr(h_vol), None, None, None, None)   # the step's result: grain volumes
    final = ctx.download(out=h_out if ctx.total_entries() <= cap else None)
    t1 = time.perf_counter()
    ctx.close()
    h2d = h_counts.nbytes + h_idx.nbytes + h_val.nbytes + (steps + 1) * h_dg.nbytes
    d2h = steps * h_vol.nbytes + final[0].nbytes + final[1].nbytes + final[2].nbytes
    return {"seconds": t1 - t0, "h2d_per_step": h2d / steps, "d2h_per_step": d2h / steps}


def adjoint_run(device):
    """Cost of the checkpointed adjoint against the forward on the calibration rollout: 128^3,
    256 grains, FP32 states, 200 steps, checkpoints every 16 steps, loss sum_g (V_g(T) - V*_g)^2."""
    import torch
    from openphase_b200.adjoint import Rollout
    from openphase_b200.cases import adjoint_calibration_128
    from openphase_b200.context import Context

    case = adjoint_calibration_128()
    G = case.ngrains
    state = case.initial_state()
    ctx = Context.from_case(case, precision="fp32", k_slots=16, device=device, state=state)
    mu = np.ones((G, G))
    R = Rollout(ctx, case.dt, case.nsteps, interval=16)
    R.set_parameters(case.pair_sigma(), mu, case.driving_force())
    target = R.forward()
    R.set_parameters(np.full((G, G), 1.0), mu, np.zeros(G))
    R.forward()                                   # warm-up of both passes
    R.backward(np.ones(G))
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    V = R.forward()
    torch.cuda.synchronize(device)
    t1 = time.perf_counter()
    R.backward(2.0 * (V - target))
    torch.cuda.synchronize(device)
    t2 = time.perf_counter()
    ctx.close()
    return {"workload": case.name, "steps": case.nsteps, "checkpoint_interval": 16, "dtype": "f32 states, f64 adjoint",
            "forward_ms": 1e3 * (t1 - t0), "adjoint_ms": 1e3 * (t2 - t1), "adjoint_over_forward": (t2 - t1) / (t1 - t0),
            "status": int(R.adjoint_status)}


def host_cpu():
    """CPU model, logical and physical core counts of this host."""
    model = "unknown"
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    try:
        import psutil
        physical = psutil.cpu_count(logical=False)
    except Exception:  # noqa: BLE001 - reported as unknown
        physical = None
    return {"cpu_model": model, "logical_cpus": os.cpu_count(), "physical_cores": physical}


def reference_steps(case, state, warmup, steps, threads):
    """Time the reference's own CPU implementation (oracle/_ref, built from the reference sources)
    on the host cores: warmup + steps full-grid steps from the same initial state, per-step seconds
    of the last `steps` (omp_get_wtime around each step of the reference driver), thread count."""
    from oracle.bridge import reference_available, run_reference
    if not reference_available():
        return None
    res, stats = run_reference(case, *state, [], threads=threads, nsteps=warmup + steps, proc_bind="close")
    per_step = stats["step_seconds"]
    per_step = per_step if isinstance(per_step, list) else [per_step]
    return per_step[warmup:warmup + steps], int(stats["threads"])


def oracle_port_steps(case, state, warmup, steps, threads):
    from oracle.bridge import Oracle
    ora = Oracle(case, *state, cap=16, threads=threads)
    ora.step(warmup)
    out = []
    for _ in range(steps):
        t = time.perf_counter()
        ora.step(1)
        out.append(time.perf_counter() - t)
    return out, threads


def cpu_timing(case, state, warmup, steps, threads):
    r = reference_steps(case, state, warmup, steps, threads)
    kind = "reference"
    if r is None:
        r = oracle_port_steps(case, state, warmup, steps, threads)
        kind = "port"
    per_step, cores = r
    value = case.n * len(per_step) / sum(per_step)
    info = host_cpu()
    return value, per_step, {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                             "omp_proc_bind": "close", **info}


def cpu_baseline(case, state, threads, warmup, steps=3):
    """A bounded sample (about half a minute of host time): the first `steps` steps of the GPU's
    timed window (steps warmup+1 ..), after the same `warmup` steps."""
    value, per_step, d = cpu_timing(case, state, warmup, steps, threads)
    d["sample"] = (f"steps {warmup + 1}-{warmup + len(per_step)} (the first {len(per_step)} of the timed window) "
                   f"of the same {case.nx}^3 workload after {warmup} untimed steps, OpenMP on {d['cores']} "
                   f"host threads")
    return d


def build_record():
    """Which library ran: its build stamp, and whether that is the hash of the sources in this tree."""
    from openphase_b200 import build_ext
    from openphase_b200._lib import lib
    info = lib().opgpu_build_info().decode()
    tree = build_ext.source_hash()
    return {"library": info, "tree_source_hash": tree, "built_from_this_tree": info.endswith(tree)}


def workload_config(case, k_slots, world):
    """The `config` object of both arms' lines."""
    return {"workload": case.name, "grid": [case.nx, case.ny, case.nz], "grains": case.ngrains,
            "eta_cells": case.iwidth, "dt": case.dt, "stencil": "D3Q27 (LB)", "k_slots": k_slots,
            "parallelism": f"x-slabs x{world} (NCCL halo exchange + volume all-reduce)" if world > 1
            else "single GPU",
            "l2": "inputs larger than L2 (the K-slot state is >126 MB)"}


def run_reference_arm(args, case, rank, world):
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    state, sigma, dg, _ = build_inputs(case, threads)
    # the same window as the GPU arm: W untimed steps, then K timed steps
    value, per_step, cpu = cpu_timing(case, state, args.warmup, args.steps, threads)
    cpu["sample"] = (f"steps {args.warmup + 1}-{args.warmup + len(per_step)} of the workload after "
                     f"{args.warmup} untimed steps (the GPU arm's timed window), OpenMP on {cpu['cores']} "
                     f"host threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": len(per_step), "warmup": args.warmup, "ms_per_step": 1e3 * sum(per_step) / len(per_step),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(case, args.k_slots, world),
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--k-slots", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-fp32-error", action="store_true")
    ap.add_argument("--no-scale", action="store_true")
    ap.add_argument("--workload", default="grain_growth_dg_256")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    from openphase_b200 import cases
    case = getattr(cases, args.workload)()

    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local_rank = _env_int("LOCAL_RANK", 0)

    if args.impl == "reference":
        return run_reference_arm(args, case, rank, world)

    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as td
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = td

    threads = max(1, (os.cpu_count() or 1) // max(1, world))
    state, sigma, dg, t_init = build_inputs(case, threads)

    runs = {}
    for precision in ("fp64", "fp32"):
        if world > 1:
            runs[precision] = slab_run(case, precision, args.k_slots, args.steps, args.warmup, local_rank,
                                       state, sigma, dg, dist)
        else:
            runs[precision] = device_run(case, precision, args.k_slots, args.steps, args.warmup, local_rank,
                                         state, sigma, dg, dist, keep_final=not args.no_fp32_error)

    def agg(ms):
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local_rank}")
        if dist is not None:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    peak, peak_kind = measured_peaks()
    out = {}
    for precision, r in runs.items():
        ms = agg(r["elapsed_ms"])
        s = 4 if precision == "fp32" else 8
        # one global grid, split into slabs (strong scaling) when world > 1
        value = case.n * args.steps / (ms / 1e3)
        nsteps_timed = max(1, r["timed_steps"])
        kernel_ms = r["kernel_ms"] / nsteps_timed
        classify_ms = r["classify_ms"] / nsteps_timed
        # algorithmic bytes of one step (the K = 8 slot record of every wide-interface voxel read
        # and written once, plus one count byte per voxel for the flag/worklist pass)
        wide_per_step = r["wide"] / args.steps
        bytes_per_launch = wide_per_step * 2 * (1 + 8 * (2 + s)) + r.get("local_voxels", case.n)
        # the same with only the stored entries counted (what the sparse slot layout moves)
        sparse_bytes = 2 * case.n + (r["entries_in"] + r["entries_out"]) * (2 + s) / args.steps
        achieved = bytes_per_launch / (kernel_ms / 1e3) / 1e9
        traffic = profiled_traffic(precision)
        out[precision] = {
            "value": value, "ms_per_step": ms / args.steps, "status": r["status"], "clocks": r["clocks"],
            "gpu_launches": r["gpu_launches"],
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "step: tile_classify_kernel + bucket_scan_kernel + list_compute_kernel<N=2..8> + warp_general_kernel + grains_update_kernel",
                         "kernel_ms": kernel_ms, "classify_ms": classify_ms,
                         "algorithmic_bytes_per_launch": bytes_per_launch,
                         "algorithmic_bytes_rule": "|W| * 2 * (1 + 8*(2+s)) + N^3 (K = 8 slot records; the run stores K = "
                                                   f"{args.k_slots} slots but touches only the ones a voxel holds)",
                         "sparse_bytes_per_launch": sparse_bytes,
                         "sparse_achieved": sparse_bytes / (kernel_ms / 1e3) / 1e9,
                         "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
                         else "fallback 6.65 TB/s"},
            "wide_fraction": r["wide"] / (case.n * args.steps),
        }

    fp32_error = None
    if runs["fp64"].get("final") and runs["fp32"].get("final"):
        from openphase_b200.compare import precision_error
        (st64, v64), (st32, v32) = runs["fp64"]["final"], runs["fp32"]["final"]
        fp32_error = precision_error(st32, v32, st64, v64, case.ngrains)
        fp32_error["after_steps"] = args.warmup + args.steps
        fp32_error["against"] = "FP64 form of this library from the same initial state (the FP64 form matches the reference)"
        fp32_error["bar"] = {"max_dphi": 1e-4, "volume_rel_max": 1e-3,
                             "met": bool(fp32_error["max_dphi"] <= 1e-4 and fp32_error["volume_rel_max"] <= 1e-3)}
        for r in runs.values():
            r["final"] = None

    e2e = {}
    if not args.no_e2e and world == 1:
        for precision in ("fp64", "fp32"):
            er = e2e_run(case, precision, args.k_slots, args.steps, local_rank, state, sigma, dg)
            sec = agg(er["seconds"] * 1e3) / 1e3
            e2e[precision] = {"value": world * case.n * args.steps / sec, "unit": UNIT,
                              "h2d_bytes_per_step": int(er["h2d_per_step"]),
                              "d2h_bytes_per_step": int(er["d2h_per_step"])}

    adjoint = None
    if not args.no_adjoint and world == 1:
        adjoint = adjoint_run(local_rank)

    scale = None
    if not args.no_scale and world == 1 and args.workload == "grain_growth_dg_256":
        scale = scale_run(args.steps, args.warmup, local_rank, threads=threads)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(case, state, os.cpu_count() or 1, args.warmup)

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    f32, f64 = out["fp32"], out["fp64"]
    line = {
        "metric": METRIC, "value": f64["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": f64["ms_per_step"], "higher_is_better": True,
        "scaling": "strong" if world > 1 else "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(case, args.k_slots, world),
        "clocks": f64["clocks"],
        "e2e": e2e.get("fp64"),
        "gpu_launches": f64["gpu_launches"],
        "roofline": f64["roofline"],
        "cpu_baseline": cpu,
        "fp32": {"value": f32["value"], "ms_per_step": f32["ms_per_step"], "e2e": e2e.get("fp32"),
                 "roofline": f32["roofline"], "clocks": f32["clocks"], "status": f32["status"],
                 "gpu_launches": f32["gpu_launches"], "error": fp32_error},
        "fp32_over_fp64": f32["value"] / f64["value"],
        "adjoint": adjoint,
        "scale_512": scale,
        "status": {"fp32": f32["status"], "fp64": f64["status"]},
        "wide_fraction": f64["wide_fraction"],
        "initial_state_seconds": round(t_init, 2),
        "build": build_record(),
    }
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
