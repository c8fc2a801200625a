"""Benchmark: implicit time steps of the 1D1V Vlasov-Poisson midpoint scheme.

Workload (the single-instance FP64 configuration): nonlinear two-stream
f0 = v^2 exp(-v^2/2)/sqrt(2 pi) (1 + 0.05 cos(0.5 x)), x in [0, 4 pi) with
nx = 512, v in [-8, 8] with nv = 1024, dt = 0.05, Arakawa J4, FFT
tensor-product kinetic preconditioner, GMRES(30) with ksp_rtol 1e-4,
Picard tolerance 1e-10 (runspec defaults).  A "step" is one implicit time
step (Picard loop with one GMRES solve per pass).  The metric is
Gcell-steps/s = nx*nv*steps / seconds.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value : device time of K steps (CUDA events on the solver's stream, L2
        flushed between steps outside the timed intervals), state resident
        in HBM.
e2e   : the same steps through the public API with the distribution
        function copied host->device (pinned) before and device->host after
        every step.
--impl reference : the CPU restatement of the reference algorithm (the C
        port under oracle/, all host threads) on the same workload, a
        bounded number of steps.
Multi-GPU: independent replicas, one per rank (scaling "weak"); the time is
the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX, NV = 512, 1024
L = 4 * np.pi
VMIN, VMAX = -8.0, 8.0
HT = 0.05
KSP_RTOL, SNES_ATOL = 1e-4, 1e-10
METRIC = "Gcell-steps/s"
WORKLOAD = "two-stream 512x1024 FP64, J4, dt=0.05, GMRES(30)+tensor_kinetic PC"
JVP_BYTES_PER_CELL = 16      # read X, write Y (FP64); h regenerated from 1-D profiles


def f0_twostream(x, v):
    return v ** 2 * np.exp(-v ** 2 / 2.) / np.sqrt(2. * np.pi) * (1. + 0.05 * np.cos(0.5 * x))


def config_dict():
    return {"grid": {"nx": NX, "nv": NV, "L": L, "vmin": VMIN, "vmax": VMAX, "ht": HT, "nt": 1},
            "solver": {"method": "matrixfree", "poisson_bracket": "ArakawaJ4", "preconditioner_type": "tensor",
                       "preconditioner_scheme": "tensor_kinetic", "petsc_ksp_rtol": KSP_RTOL,
                       "petsc_snes_atol": SNES_ATOL},
            "initial_data": {"charge": -1.0}}


def initial_field():
    hx = L / NX
    hv = (VMAX - VMIN) / (NV - 1)
    x = np.arange(NX) * hx
    v = VMIN + np.arange(NV) * hv
    X, V = np.meshgrid(x, v, indexing="xy")
    f = f0_twostream(X, V)
    f[:2, :] = 0.
    f[NV - 2:, :] = 0.
    return np.ascontiguousarray(f)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per JVP launch from the committed ncu summary (or None)."""
    p = os.path.join(ROOT, "profiles", "jvp_traffic.json")
    if os.path.exists(p):
        with open(p) as fh:
            return json.load(fh).get("bytes_per_launch_full_size")
    return None


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        with open(self.file.name) as fh:
            rows = [r.strip().split(",") for r in fh if r.strip()]
        os.unlink(self.file.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[0]))
                smax = float(r[1])
                for k, nm in enumerate(names):
                    if r[4 + k].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def flush_l2(buf):
    buf.add_(1.0)   # 256 MB write, larger than the 126 MB L2


def run_gpu(args, rank, world):
    import torch
    import ctypes as C
    from vivlasov1d_b200.run import Run
    from vivlasov1d_b200 import _lib

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    f0 = torch.from_numpy(initial_field())
    run = Run(config_dict(), f0=f0, device=dev)
    ctx = run.ctx
    stream = torch.cuda.current_stream(dev)
    flush = torch.zeros(32 * 1024 * 1024, dtype=torch.float64, device=dev)
    for _ in range(args.warmup):
        run.step()
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    sampler = ClockSampler(dev.index) if rank == 0 else None
    if sampler:
        sampler.start()
    # ---- value: resident state ----
    launches0 = ctx.launch_count()
    picard = gmres = 0
    total_ms = 0.0
    for _ in range(args.steps):
        flush_l2(flush)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        r = run.step()
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
        picard += r["picard_its"]
        gmres += sum(r["gmres_its"])
    launches = ctx.launch_count() - launches0
    # dominant-kernel timing on the workload's own buffers (the last GMRES
    # basis vector 0 and the solver's Hamiltonian), CUDA events on the
    # solver's stream, 200 back-to-back launches in one graph
    jvp_s = ctx.time_kernel(0, reps=200)
    pc_s = ctx.time_kernel(2, reps=50)
    # ---- e2e: host buffers through the public API ----
    host = torch.empty((NV, NX), dtype=torch.float64).pin_memory()
    host.copy_(run.fc.cpu())
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush_l2(flush)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        run.fc.copy_(host, non_blocking=True)
        run.calculate_moments()
        run.step()
        host.copy_(run.fc, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
    clocks = sampler.stop() if sampler else None
    t_value = total_ms / 1e3
    t_e2e = e2e_ms / 1e3
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([t_value, t_e2e], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_value, t_e2e = float(t[0]), float(t[1])
    inv = run.invariants()
    return dict(t_value=t_value, t_e2e=t_e2e, picard=picard, gmres=gmres, launches=launches,
                jvp_s=jvp_s, pc_s=pc_s, clocks=clocks, invariants=inv)


def cpu_baseline_sample(seconds=20.0):
    """Time the oracle port on the host, bounded to about `seconds`."""
    try:
        from oracle.c import CPort
        port = CPort(NX, NV, L, VMIN, VMAX, HT, ksp_rtol=KSP_RTOL, snes_atol=SNES_ATOL)
        port.set_f(initial_field())
        t0 = time.perf_counter()
        steps = 0
        while True:
            port.step()
            steps += 1
            if time.perf_counter() - t0 > seconds or steps >= 50:
                break
        dt = time.perf_counter() - t0
        return {"value": NX * NV * steps / dt / 1e9, "unit": METRIC, "cores": port.threads,
                "kind": "port", "sample": "%d steps of the workload from t=0 (C port, OpenMP)" % steps}
    except ImportError:
        pass
    from oracle import vlasov_oracle as vo
    g = vo.Grid(NX, NV, L, VMAX, VMIN, ht=HT)
    f0 = vo.from_flat(initial_field()).copy()
    t0 = time.perf_counter()
    orun = vo.Run(g, f0, ksp_rtol=KSP_RTOL, snes_atol=SNES_ATOL)
    steps = 0
    while True:
        orun.step()
        steps += 1
        if time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": NX * NV * steps / dt / 1e9, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": "%d steps of the workload from t=0 (numpy oracle, incl. set-up)" % steps}


def reference_arm(steps, warmup, budget=240.0):
    """W warm-up + K timed steps of the C port on all host threads; stops
    early (and says so) if the timed steps would exceed `budget` seconds."""
    from oracle.c import CPort
    port = CPort(NX, NV, L, VMIN, VMAX, HT, ksp_rtol=KSP_RTOL, snes_atol=SNES_ATOL)
    port.set_f(initial_field())
    for _ in range(warmup):
        port.step()
    t0 = time.perf_counter()
    done = 0
    for _ in range(steps):
        port.step()
        done += 1
        if time.perf_counter() - t0 > budget:
            break
    dt = time.perf_counter() - t0
    return {"value": NX * NV * done / dt / 1e9, "cores": port.threads, "kind": "port",
            "sample": "%d timed steps after %d warm-up steps (C port of the oracle, OpenMP)" % (done, warmup)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    config = {"workload": WORKLOAD, "nx": NX, "nv": NV, "dt": HT, "bracket": "arakawaj4",
              "preconditioner": "tensor_kinetic", "ksp_rtol": KSP_RTOL, "snes_atol": SNES_ATOL,
              "instances_per_gpu": 1, "parallelism": "replicas x%d" % args.gpus,
              "l2": "flushed between timed steps (256 MB write)"}

    if args.impl == "reference":
        if rank != 0:
            return
        cb = reference_arm(args.steps, args.warmup)
        line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": METRIC,
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (analytic initial condition)", "config": config,
                "cpu_baseline": {"value": cb["value"], "unit": METRIC, "cores": cb["cores"], "kind": cb["kind"],
                                 "sample": cb["sample"]},
                "e2e": {"value": cb["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    res = run_gpu(args, rank, world)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    cells = NX * NV
    value = cells * args.steps * world / res["t_value"] / 1e9
    e2e = cells * args.steps * world / res["t_e2e"] / 1e9
    peak, peak_kind = measured_peaks()
    avg_s = res["jvp_s"]
    achieved = JVP_BYTES_PER_CELL * cells / avg_s / 1e9
    roofline = {"kernel": "k_bracket_wide<4,JVP> (Jacobian-vector product stencil)", "bound": "hbm",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind, "traffic": profiled_traffic(),
                "algorithmic_bytes_per_launch": JVP_BYTES_PER_CELL * cells,
                "avg_launch_us": avg_s * 1e6,
                "note": "4 MiB operands are L2-resident at this size; see DESIGN.md for the HBM-resident figure",
                "pc_apply_us": res["pc_s"] * 1e6}
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["t_value"] * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (analytic two-stream initial condition)", "config": config,
            "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": cells * 8, "d2h_bytes_per_step": cells * 8},
            "gpu_launches": res["launches"], "roofline": roofline, "clocks": res["clocks"],
            "iterations": {"picard_per_step": res["picard"] / args.steps, "gmres_per_step": res["gmres"] / args.steps},
            "field_energy_end": res["invariants"]["field_energy"]}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(seconds=20.0)
    print(json.dumps(line))


if __name__ == "__main__":
    main()
