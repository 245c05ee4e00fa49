"""Benchmark of the B200 finite-volume time step.

Workload: the first-order acoustic wave system on 128^3 uniform cells over
[0,1]^3 (c = 1, Gaussian pressure pulse sigma 0.05 at the centre, reflective
walls, CFL 0.4), 500 time steps per bench step, FP32 fused path (one
TMA-staged sweep kernel per time step, replayed from a CUDA graph).  Metric:
cell-updates/s = cells x time steps / device time.

Per rank one replica runs on its own GPU (the solver is single-GPU, so
--gpus N runs N independent replicas: weak scaling, no collective on the data
path).  Between timed bench steps the L2 is flushed by writing a 512 MB
buffer and the state is reset (both outside the CUDA-event brackets).

--impl reference times the CPU restatement of the same workload (the
reference itself cannot be built here) on the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "cell-updates/s"
ALG_BYTES = 32  # FP32 wave: 4 fields read + written once per cell-update


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="native", choices=["native", "reference"])
    p.add_argument("--n", type=int, default=128, help="cells per edge")
    p.add_argument("--tsteps", type=int, default=500, help="time steps per bench step")
    p.add_argument("--no-extras", action="store_true", help="skip the FP64, large-mesh and CPU side measurements")
    return p.parse_args()


def workload_config(n, tsteps):
    return {"workload": f"wave3d_rusanov_{n}^3_x{tsteps}_steps", "mesh": [n, n, n], "time_steps_per_bench_step": tsteps,
            "fields": 4, "path": "fused_tma_sweep", "cfl": 0.4, "c": 1.0,
            "l2": "flushed between bench steps (512 MB write); the 67 MB ping-pong working set stays L2-resident within a solve",
            "parallelism": "replica per GPU"}


# ---------------------------------------------------------------------------
class ClockSampler:
    """Samples SM clock and clock-event reasons through NVML while running."""

    def __init__(self, device_index, period=0.01):
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self.period = period
        self._stop = threading.Event()
        self._t = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:  # NVML unavailable: report no clocks
            self.nv = None

    def _run(self):
        nv = self.nv
        names = {
            "hw_slowdown": getattr(nv, "nvmlClocksEventReasonHwSlowdown", 0x8),
            "hw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
            "sw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
            "sw_power_cap": getattr(nv, "nvmlClocksEventReasonSwPowerCap", 0x4),
            "hw_power_brake_slowdown": getattr(nv, "nvmlClocksEventReasonHwPowerBrakeSlowdown", 0x80),
        }
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                try:
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                except AttributeError:
                    r = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                for k, bit in names.items():
                    if r & bit:
                        self.reasons.add(k)
            except Exception:
                pass
            time.sleep(self.period)

    def start(self):
        if self.nv:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()

    def stop(self):
        if self._t:
            self._stop.set()
            self._t.join()
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples), "source": "nvml"}


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(name):
    """DRAM bytes per launch recorded from an ncu capture in profiles/."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch_at_bench_size:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
def cpu_restatement_rate(n, tsteps_cap=400, budget_s=10.0, threads=None):
    """Cell-updates/s of the CPU restatement (FP32, operator-by-operator passes)
    on the bench workload, timed on this host's cores."""
    import numpy as np
    from oracle import oracle as O
    from cfdarcov2_b200.workloads import wave_config
    if threads:
        O.set_threads(threads)
    cfg = wave_config(n=n)
    m = O.Mesh(n, n, n, cfg["dx"], cfg["dx"], cfg["dx"], dtype=np.float32)
    done, secs = 0, 0.0
    while secs < budget_s and done < tsteps_cap:
        secs += m.wave_time(cfg["q0"], cfg["dt"], 2, faithful=True)
        done += 2
    return n ** 3 * done / secs, done, O.max_threads()


def run_reference(args, rank):
    if rank != 0:
        return
    import numpy as np
    from oracle import oracle as O
    from cfdarcov2_b200.workloads import wave_config
    n = args.n
    cfg = wave_config(n=n)
    m = O.Mesh(n, n, n, cfg["dx"], cfg["dx"], cfg["dx"], dtype=np.float32)
    per_step = 2  # time steps in one bounded sample
    for _ in range(args.warmup):
        m.wave_time(cfg["q0"], cfg["dt"], per_step, faithful=True)
    t = [m.wave_time(cfg["q0"], cfg["dt"], per_step, faithful=True) for _ in range(args.steps)]
    total = sum(t)
    value = n ** 3 * per_step * args.steps / total
    cores = O.max_threads()
    sample = f"{n}^3 wave, {per_step} time steps per bench step, FP32 operator-by-operator CPU restatement"
    line = {"metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(n, args.tsteps), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference (C++/Eigen/OCCA) cannot be built here; this is the oracle's restatement of its CPU path"}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def run_native(args, rank, world, local_rank):
    import numpy as np
    import torch
    import torch.distributed as dist

    import cfdarcov2_b200 as cfdb
    from cfdarcov2_b200.workloads import wave_config

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ctx = cfdb.Context(local_rank)
    stream = torch.cuda.current_stream(dev)
    n, T = args.n, args.tsteps
    cfg = wave_config(n=n, steps=T)
    cells = n ** 3
    mesh = cfdb.Mesh.structured(ctx, n, n, n, cfg["dx"], cfg["dx"], cfg["dx"])
    q0_host = torch.tensor(cfg["q0"], dtype=torch.float32).pin_memory()
    q0 = q0_host.to(dev)
    a = torch.empty_like(q0)
    b = torch.empty_like(q0)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def solve():
        return ctx.wave_run(mesh, a, b, cfg["dt"], T, c_const=cfg["c"], path=cfdb.FUSED, use_graph=True)

    def barrier():
        if world > 1:
            dist.barrier()

    # warm-up (untimed)
    for _ in range(args.warmup):
        a.copy_(q0)
        solve()
    torch.cuda.synchronize()

    sampler = ClockSampler(local_rank)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    wall0 = time.perf_counter()
    for k in range(args.steps):
        flush.zero_()
        a.copy_(q0)
        ev[k][0].record(stream)
        solve()
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    barrier()
    wall = time.perf_counter() - wall0
    clocks = sampler.stop()
    dev_ms = sum(s.elapsed_time(e) for s, e in ev)
    t_max = torch.tensor([dev_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    dev_ms = float(t_max.item())
    value = world * cells * T * args.steps / (dev_ms * 1e-3)

    # end to end through the C ABI with host buffers: H2D of the initial state,
    # the solve, D2H of the final state, every step
    out_host = torch.empty_like(q0_host).pin_memory()
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    for k in range(args.steps):
        flush.zero_()
        ev2[k][0].record(stream)
        a.copy_(q0_host, non_blocking=True)
        fin = solve()
        out_host.copy_(fin, non_blocking=True)
        ev2[k][1].record(stream)
    torch.cuda.synchronize()
    e2e_ms = sum(s.elapsed_time(e) for s, e in ev2)
    t2 = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t2, op=dist.ReduceOp.MAX)
    e2e_ms = float(t2.item())
    e2e_value = world * cells * T * args.steps / (e2e_ms * 1e-3)

    peak, peak_kind = measured_peak_hbm()
    launch_ms = dev_ms / (args.steps * T)
    achieved = ALG_BYTES * cells / (launch_ms * 1e-3) / 1e9
    traffic = profiled_traffic("wave_sweep_128.txt")
    line = {
        "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Gaussian pulse)",
        "config": workload_config(n, T),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)",
                     "kernel": "stencil::sweep_kernel<WavePhys<false>,128,8,3,4>",
                     "algorithmic_bytes_per_cell_update": ALG_BYTES},
        "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": int(q0_host.numel() * 4),
                "d2h_bytes_per_step": int(out_host.numel() * 4)},
        "gpu_launches": args.steps * T,
        "clocks": clocks,
        "wall_s": wall,
    }

    if not args.no_extras and rank == 0:
        line.update(extras(ctx, cfdb, mesh, cfg, q0, a, b, flush, dev, n, T, peak, world))
        line["speedup_fused_fp32_vs_plain_fp64"] = (value / world) / line["fp64_plain"]["value"]
    if rank == 0:
        if world == 1 and not args.no_extras:
            rate, done, cores = cpu_restatement_rate(n)
            line["cpu_baseline"] = {"value": rate, "unit": "cell-updates/s", "cores": cores, "kind": "port",
                                    "sample": f"{n}^3 wave, {done} time steps, FP32 operator-by-operator CPU restatement"}
        print(json.dumps(line), flush=True)


def extras(ctx, cfdb, mesh, cfg, q0, a, b, flush, dev, n, T, peak, world):
    """FP64 plain-path speed and accuracy on the same workload, and the fused
    kernel's HBM efficiency on a mesh larger than L2."""
    import numpy as np
    import torch
    from cfdarcov2_b200.workloads import wave_state
    out = {}
    stream = torch.cuda.current_stream(dev)
    # fused FP32 final state
    a.copy_(q0)
    f32 = ctx.wave_run(mesh, a, b, cfg["dt"], T, c_const=cfg["c"], path=cfdb.FUSED).double().cpu().numpy()
    # FP64 plain path: speed + reference solution
    a64 = q0.double()
    b64 = torch.empty_like(a64)
    ctx.wave_run(mesh, a64, b64, cfg["dt"], 4, c_const=cfg["c"], path=cfdb.PLAIN)  # geometry upload + warm-up
    a64.copy_(q0.double())
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flush.zero_()
    s.record(stream)
    f64t = ctx.wave_run(mesh, a64, b64, cfg["dt"], T, c_const=cfg["c"], path=cfdb.PLAIN)
    e.record(stream)
    torch.cuda.synchronize()
    ms64 = s.elapsed_time(e)
    f64 = f64t.cpu().numpy()
    rate64 = n ** 3 * T / (ms64 * 1e-3)
    l2 = float(np.linalg.norm(f32 - f64) / np.linalg.norm(f64))
    linf = float(np.abs(f32 - f64).max() / np.abs(f64).max())
    out["fp64_plain"] = {"value": rate64, "unit": "cell-updates/s", "path": "plain per-operator kernels, FP64, N x 6 geometry"}
    out["accuracy_vs_fp64"] = {"l2_rel": l2, "linf_rel": linf, "bar_l2": 1e-5}
    del a64, b64
    # fused kernel on a mesh well beyond L2 (state 2 x 226 MB at 384^3)
    N = 384
    big = cfdb.Mesh.structured(ctx, N, N, N, 1.0 / N, 1.0 / N, 1.0 / N)
    qa = torch.tensor(wave_state(N), dtype=torch.float32, device=dev)
    qb = torch.empty_like(qa)
    dt = 0.4 / (3 * N)
    ctx.wave_run(big, qa, qb, dt, 4)
    torch.cuda.synchronize()
    steps = 40
    s.record(stream)
    ctx.wave_run(big, qa, qb, dt, steps)
    e.record(stream)
    torch.cuda.synchronize()
    ms = s.elapsed_time(e) / steps
    ach = ALG_BYTES * N ** 3 / (ms * 1e-3) / 1e9
    out["roofline_beyond_l2"] = {"mesh": [N, N, N], "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                 "ms_per_launch": ms, "cell_updates_per_s": N ** 3 / (ms * 1e-3)}
    return out


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_native(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
