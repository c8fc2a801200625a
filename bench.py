"""Benchmark: batched mixed-precision implicit steps of a seeded parameter sweep
against the plain FP64 step, on one B200.

Workload (the metric's configuration): 256 independent runs drawn from the
seed 20261203 -- Landau, two-stream and bump-on-tail initial data, k ~ U[0.3,
0.6], amplitude log-uniform in [1e-3, 0.5], nx in {64, 128, 256}, nv in
{128, 256, 512, 1024}, v in [-10, 10], L = 2 pi / k, dt = 0.1, Arakawa J4,
FFT tensor-product kinetic preconditioner, GMRES(30) with ksp_rtol 1e-4,
Picard tolerance 1e-12 on every arm (SNES_ATOL; about 17.5 M cells in all).  A "step" advances every
instance by one implicit time step.  Gcell-steps/s = sum(nx nv) * steps / s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value       : batched + mixed precision -- every kernel launched once for the
              instance table, lockstep Picard/GMRES loops with per-instance
              masks, one CUDA graph per step; FP32 GMRES basis, Jacobian and
              preconditioner, FP64 residual, Picard loop, moments, Poisson and
              invariants; one lockstep table.
              Device time of K steps (CUDA events), state resident in HBM
              (the working set is far larger than L2).
plain_fp64  : the same instances in FP64, each advanced by its own vv_step
              one after another -- how the reference runs a sweep.
field_energy: after W+K steps, |E - E_oracle| / |E_oracle| per instance for
              every GPU arm against the FP64 oracle (the C port run for the
              same W+K steps, which is also the timed cpu_baseline), and
              the batched mixed arm against the plain FP64 GPU arm.
e2e         : the batched mixed step through Batch.step(host=...), which
              copies every instance's f host->device (one pinned buffer)
              before and device->host after each step, in four pieces each
              way, a step's pieces in waiting only for the previous step's
              same piece out (the two directions overlap).
batched_fp64: the same table through the batch in FP64 (ksp_rtol 1e-4): the
              gain of batching alone, apart from the FP32 inner solves.  After
              the first warm-up step it runs as two tables at once on two
              streams (the eighth of the instances that needed the most GMRES
              iterations, and the rest), 8% faster than one table in FP64;
              in mixed precision one table is 3% faster than two.
step_roofline: algorithmic bytes of the timed steps (from the logged
              Picard and GMRES counts) over their device time.
--impl reference : the CPU restatement of the reference algorithm (the C
              port under oracle/) on the same instances, spread over all host
              threads (each instance single-threaded, as separate runs of a
              sweep use a many-core host); also reported: the port stepping
              one instance after the other with OpenMP inside each.
Multi-GPU: independent replicas, one sweep per rank with its own seed
(scaling "weak"); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gcell-steps/s"
N_INSTANCES = 256
WORKLOAD = ("sweep: 256 seeded instances (Landau/two-stream/bump-on-tail, nx 64-256, nv 128-1024), "
            "J4, dt=0.1, GMRES(30)+tensor_kinetic, batched + mixed precision vs plain FP64")
MDOT_IT = 4   # Arnoldi index of the roofline launch of the multi-dot
# Picard tolerance (petsc_snes_atol) of every arm, GPU and CPU.  The runspec
# default 1e-10 lets two FP64 runs of the same step stop at points of the
# residual ball that differ in field energy by up to 1e-8 relative on the
# strongly damped instances within 25 steps (measured between the FP32-inner
# and FP64 arms; 3e-7 between 1e-10 and 1e-12 themselves at 200 steps); the
# metric's 1e-9 field-energy bound is kept by tightening every arm alike
SNES_ATOL = 1e-12


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(name):
    """DRAM bytes per whole-table launch of a kernel from its committed ncu summary (or None)."""
    p = os.path.join(ROOT, "profiles", name)
    if os.path.exists(p):
        with open(p) as fh:
            return json.load(fh).get("bytes_per_launch")
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


def specs_for(rank):
    from vivlasov1d_b200 import workloads as W
    return W.sweep_specs(N_INSTANCES, seed=W.SWEEP_SEED + rank)


def reduce_over_ranks(maxes, sums, device):
    """Max over ranks of the times and sum over ranks of the work (one
    all-reduce each; every rank calls it the same way)."""
    import torch
    import torch.distributed as dist
    tm = torch.tensor(maxes, dtype=torch.float64, device=device)
    ts = torch.tensor(sums, dtype=torch.float64, device=device)
    dist.all_reduce(tm, op=dist.ReduceOp.MAX)
    dist.all_reduce(ts, op=dist.ReduceOp.SUM)
    return [float(x) for x in tm], [float(x) for x in ts]


def step_algorithmic_bytes(specs, reps, mixed, restart=30):
    """Algorithmic HBM bytes of the timed steps from the logged iteration
    counts: per instance and step, cells x [N_pic (24 + 16 + 8) + N_gmres
    (16 + 48) + sum over Arnoldi steps (16 k + 40)] in FP64 (residual, its
    norm and the moments per Picard pass; Jacobian product and the 3-pass
    preconditioner per GMRES iteration; Gram-Schmidt against the k basis
    vectors of the cycle).  The mixed mode runs the Jacobian product, the
    preconditioner and Gram-Schmidt in FP32: those terms are halved."""
    inner = 0.5 if mixed else 1.0
    total = 0.0
    for rep in reps:                      # one list of instance reports per step
        for s, r in zip(specs, rep):
            cells = s["nx"] * s["nv"]
            npic = r["picard_its"]
            gm = sum(r["gmres_its"])
            gs = 0.0
            for m in r["gmres_its"]:
                for it in range(m):
                    k = it % restart + 1
                    gs += 16 * k + 40
            total += cells * (npic * 48 + inner * (gm * 64 + gs))
    return total


def time_steps(fn, k, stream):
    import torch
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = [fn() for _ in range(k)]
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3, out


def run_gpu(args, rank, world):
    import torch
    from vivlasov1d_b200 import workloads as W
    from vivlasov1d_b200.batch import Batch

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    specs = specs_for(rank)
    cells = sum(s["nx"] * s["nv"] for s in specs)
    mode_rows = sum((s["nx"] // 2 + 1) * s["nv"] for s in specs)   # complex unknowns of the tridiagonal stage
    mixed = W.sweep_runs(specs=specs, device=dev, precision="mixed", snes_atol=SNES_ATOL)
    plain = W.sweep_runs(specs=specs, device=dev, precision="fp64", snes_atol=SNES_ATOL)
    bfp64 = W.sweep_runs(specs=specs, device=dev, precision="fp64", snes_atol=SNES_ATOL)
    # mixed: one lockstep table; batched FP64: the first warm-up step whole,
    # the later steps with the slowest eighth of the instances as a second
    # table beside the rest
    batch = Batch(mixed)
    batch64 = Batch(bfp64, split="auto")
    # ---- warm-up (every arm advances W steps from the same initial state) ----
    for _ in range(args.warmup):
        batch.step()
        batch64.step()
        for r in plain:
            r.step()
    torch.cuda.synchronize()
    # the harness's own objects (three arms of 256 runs, their contexts and
    # tensors: about 200k objects that Python's cyclic collector tracks) are
    # frozen out of the collector: its full passes over them landed inside
    # the timed steps and stalled the host between two launches by about
    # 2 ms per step (measured: 27.5 against 25.5 ms per sweep step)
    gc.collect()
    gc.freeze()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    sampler = ClockSampler(dev.index) if rank == 0 else None
    if sampler:
        sampler.start()
    # the state the timed steps start from (the e2e steps repeat them)
    snapshot = [r.fc.clone() for r in mixed]
    # ---- value: batched + mixed, resident state ----
    batch.launch_count(reset=True)
    t_value, reps = time_steps(batch.step, args.steps, stream)
    launches = batch.launch_count()
    clocks = sampler.stop() if sampler else None
    picard = sum(r["picard_its"] for rep in reps for r in rep) / (args.steps * len(specs))
    gmres = sum(sum(r["gmres_its"]) for rep in reps for r in rep) / (args.steps * len(specs))
    # ---- batched FP64: the same table and tolerances in FP64 (separates the
    # gain of batching from the gain of the FP32 inner solves) ----
    t_b64, reps64 = time_steps(batch64.step, args.steps, stream)
    # ---- plain FP64, one instance after the other ----
    t_plain, _ = time_steps(lambda: [r.step() for r in plain], args.steps, stream)
    fe_m, fe_p, fe_b = W.field_energies(mixed), W.field_energies(plain), W.field_energies(bfp64)
    fe_rel = np.abs(fe_m - fe_p) / np.abs(fe_p)
    fe_rel_b64 = np.abs(fe_b - fe_p) / np.abs(fe_p)
    step_bytes = step_algorithmic_bytes(specs, reps, mixed=True)
    step_bytes64 = step_algorithmic_bytes(specs, reps64, mixed=False)
    # ---- roofline kernels on the whole table (between steps, on the timed
    # batch itself: the same kernel shapes; the launches overwrite its GMRES
    # scratch, which every step re-initialises) ----
    mdot_s = batch.time_kernel(0, it=MDOT_IT, reps=20)
    maxpy_s = batch.time_kernel(3, it=MDOT_IT, reps=20)
    pc_s = batch.time_kernel(1, it=MDOT_IT, reps=10)
    jvp_s = batch.time_kernel(2, it=MDOT_IT, reps=20)
    tri_s = batch.time_kernel(4, it=MDOT_IT, reps=10)
    op_s = batch.time_kernel(5, it=MDOT_IT, reps=10)
    # ---- e2e: host buffers through the public API, the same K steps again ----
    # one pinned host buffer with every instance's f back to back
    hosts = torch.empty(sum(r.fc.numel() for r in mixed), dtype=mixed[0].fc.dtype).pin_memory()
    off = 0
    for snap, r in zip(snapshot, mixed):
        k = snap.numel()
        hosts[off:off + k].copy_(snap.reshape(-1))
        off += k
        r.fc.copy_(snap)
        r.calculate_moments()
    del snapshot

    # every instance's f copied in from the host buffer before the step and
    # back out after it (Batch.step(host=...): one copy each way in pieces,
    # the next step's pieces in overlapping this step's pieces out)
    t_e2e, _ = time_steps(lambda: batch.step(host=hosts), args.steps, stream)
    total_cells = cells
    if world > 1:
        (t_value, t_plain, t_e2e, t_b64), (total_cells,) = reduce_over_ranks([t_value, t_plain, t_e2e, t_b64],
                                                                             [cells], dev)
    return dict(cells=cells, total_cells=total_cells, t_value=t_value, t_plain=t_plain, t_e2e=t_e2e, t_b64=t_b64,
                launches=launches, clocks=clocks, picard=picard, gmres=gmres, fe_rel=fe_rel, fe_rel_b64=fe_rel_b64,
                fe_m=fe_m, fe_p=fe_p, fe_b=fe_b,
                mdot_s=mdot_s, maxpy_s=maxpy_s, pc_s=pc_s, jvp_s=jvp_s, tri_s=tri_s, op_s=op_s, mode_rows=mode_rows,
                step_bytes=step_bytes, step_bytes64=step_bytes64, specs=specs)


def port_runs(specs):
    """C-port instances of the sweep (FP64, all host threads)."""
    from oracle.c import CPort
    from vivlasov1d_b200 import workloads as W
    runs = []
    for s in specs:
        p = CPort(s["nx"], s["nv"], s["L"], -10.0, 10.0, 0.1, ksp_rtol=1e-4, snes_atol=SNES_ATOL)
        hx, hv = s["L"] / s["nx"], 20.0 / (s["nv"] - 1)
        x = np.arange(s["nx"]) * hx
        v = -10.0 + np.arange(s["nv"]) * hv
        X, V = np.meshgrid(x, v, indexing="xy")
        f = W.FAMILIES[s["family"]](s["amp"], s["k"])(X, V)
        f[:2, :] = 0.
        f[s["nv"] - 2:, :] = 0.
        p.set_f(f)
        runs.append(p)
    return runs


def _largest_first(specs):
    return sorted(range(len(specs)), key=lambda i: -specs[i]["nx"] * specs[i]["nv"])


def port_sweep_step(runs, order, mode):
    """One sweep step of the C port.  mode "instances": the runs spread over
    the host threads, each single-threaded inside (how a sweep of separate
    runs uses a many-core host; largest instances first); mode "inside": one
    run after the other, each parallel inside its kernels."""
    from oracle.c import step_many
    if mode == "instances":
        step_many(runs, order)
    else:
        for p in runs:
            p.step()


def cpu_sample(specs, seconds, mode):
    """The C port on the host: whole sweep steps (every instance once) from
    t=0 until about `seconds` have passed, at least one."""
    runs = port_runs(specs)
    order = _largest_first(specs)
    cells = sum(s["nx"] * s["nv"] for s in specs)
    t0 = time.perf_counter()
    steps = 0
    while True:
        port_sweep_step(runs, order, mode)
        steps += 1
        if time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    what = ("instances spread over the threads, each single-threaded" if mode == "instances"
            else "one instance after the other, OpenMP inside each")
    return {"value": cells * steps / dt / 1e9, "unit": METRIC, "cores": runs[0].threads, "kind": "port",
            "sample": "%d step(s) of all %d sweep instances from t=0 (C port of the oracle, %s)"
                      % (steps, len(specs), what)}


def port_field_energy(p, s):
    """Field energy of a C-port run (potential.pyx:54-59, charge -1)."""
    phi = p.phi()
    d = np.roll(phi, -1) - phi
    return 0.5 * -1.0 * float((d * d).sum()) / (s["L"] / s["nx"])


def cpu_baseline_run(specs, steps):
    """The C port (the oracle's FP64 step, instances spread over the host
    threads) for exactly `steps` sweep steps from t=0: the timed CPU
    baseline, and the FP64 oracle's field energies after those steps."""
    runs = port_runs(specs)
    order = _largest_first(specs)
    cells = sum(s["nx"] * s["nv"] for s in specs)
    t0 = time.perf_counter()
    for _ in range(steps):
        port_sweep_step(runs, order, "instances")
    dt = time.perf_counter() - t0
    fe = np.array([port_field_energy(p, s) for p, s in zip(runs, specs)])
    return {"value": cells * steps / dt / 1e9, "unit": METRIC, "cores": runs[0].threads, "kind": "port",
            "sample": "%d step(s) of all %d sweep instances from t=0 (C port of the oracle, instances spread over "
                      "the threads, each single-threaded); the same steps as the GPU arms" % (steps, len(specs))}, fe


def reference_arm(steps, warmup, budget=240.0):
    """W warm-up + K timed sweep steps of the C port, the instances spread over
    all host threads; stops early (and says so) if the timed steps would
    exceed `budget` s.  A second figure: the port stepping one instance after
    the other with OpenMP inside each, on a bounded sample."""
    specs = specs_for(0)
    runs = port_runs(specs)
    order = _largest_first(specs)
    cells = sum(s["nx"] * s["nv"] for s in specs)
    for _ in range(warmup):
        port_sweep_step(runs, order, "instances")
    t0 = time.perf_counter()
    done = 0
    for _ in range(steps):
        port_sweep_step(runs, order, "instances")
        done += 1
        if time.perf_counter() - t0 > budget:
            break
    dt = time.perf_counter() - t0
    inside = cpu_sample(specs, 15.0, "inside")
    return {"value": cells * done / dt / 1e9, "cores": runs[0].threads, "kind": "port",
            "sample": "%d timed sweep steps (all %d instances) after %d warm-up steps (C port of the oracle; "
                      "instances spread over the host threads, each single-threaded)" % (done, len(specs), warmup),
            "inside_parallel": inside}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    config = {"workload": WORKLOAD, "instances": N_INSTANCES, "seed": 20261203, "precision": "mixed",
              "mixed_inner_rtol": 1e-2, "ksp_rtol": 1e-4, "snes_atol": SNES_ATOL, "dt": 0.1,
              "bracket": "arakawaj4", "preconditioner": "tensor_kinetic", "parallelism": "replicas x%d" % args.gpus,
              "tables": "one lockstep table (batched FP64: the slowest eighth of the instances and the rest, "
                        "stepped concurrently on two streams)",
              "l2": "working set far larger than L2 (17.5 M cells x ~40 fields); no flush",
              "host": "the harness's setup objects frozen out of Python's cyclic GC before the timed steps"}

    if args.impl == "reference":
        if rank != 0:
            return
        cb = reference_arm(args.steps, args.warmup)
        line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": METRIC,
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded analytic initial data)", "config": config,
                "cpu_baseline": {"value": cb["value"], "unit": METRIC, "cores": cb["cores"], "kind": cb["kind"],
                                 "sample": cb["sample"]},
                "one_instance_at_a_time": cb["inside_parallel"],
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
    cells = res["cells"]                      # this rank's sweep (for the per-launch roofline)
    work = res["total_cells"] * args.steps    # every rank's cells, every timed step
    value = work / res["t_value"] / 1e9
    plain = work / res["t_plain"] / 1e9
    e2e = work / res["t_e2e"] / 1e9
    b64 = work / res["t_b64"] / 1e9
    peak, peak_kind = measured_peaks()
    step_roofline = {
        "what": "algorithmic bytes of the whole timed steps (per instance: cells x [N_pic x 48 + N_gmres x 64 + "
                "sum over Arnoldi steps (16 k + 40)] B in FP64, the FP32 inner terms halved) from the logged "
                "Picard/GMRES counts, over the device time of the steps",
        "bytes_per_step": res["step_bytes"] / args.steps,
        "achieved": res["step_bytes"] / res["t_value"] / 1e9, "peak": peak, "unit": "GB/s",
        "frac": res["step_bytes"] / res["t_value"] / 1e9 / peak,
        "batched_fp64_achieved": res["step_bytes64"] / res["t_b64"] / 1e9,
        "batched_fp64_frac": res["step_bytes64"] / res["t_b64"] / 1e9 / peak}
    mdot_bytes = cells * (MDOT_IT + 2) * 4      # w and V_0..V_it read in FP32
    maxpy_bytes = cells * (MDOT_IT + 3) * 4     # w and V_0..V_it read, w written
    # the tridiagonal stage: read the FP32 complex spectrum and the LU
    # reciprocals, write the solution (3 x 8 B per mode and row)
    tri_bytes = res["mode_rows"] * 24
    achieved = mdot_bytes / res["mdot_s"] / 1e9
    tri_gbps = tri_bytes / res["tri_s"] / 1e9
    roofline = {"kernel": "multi-dot of the Gram-Schmidt step (k_b_gm_mdot_p, whole table at Arnoldi index %d; "
                          "the largest share of the step's launch list)" % MDOT_IT,
                "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind, "traffic": profiled_traffic("batch_mdot_traffic.json"),
                "algorithmic_bytes_per_launch": mdot_bytes, "avg_launch_us": res["mdot_s"] * 1e6,
                "others": {"tridiagonal_us": res["tri_s"] * 1e6, "tridiagonal_achieved_GBps": tri_gbps,
                           "tridiagonal_frac": tri_gbps / peak, "tridiagonal_bytes_per_launch": tri_bytes,
                           "tridiagonal_traffic": profiled_traffic("batch_tridiag_traffic.json"),
                           "multiaxpy_us": res["maxpy_s"] * 1e6,
                           "multiaxpy_achieved_GBps": maxpy_bytes / res["maxpy_s"] / 1e9,
                           "multiaxpy_frac": maxpy_bytes / res["maxpy_s"] / 1e9 / peak,
                           "preconditioner_3_kernels_us": res["pc_s"] * 1e6,
                           "preconditioner_achieved_GBps": cells * 24 / res["pc_s"] / 1e9,
                           "jacobian_stencil_us": res["jvp_s"] * 1e6,
                           "jacobian_achieved_GBps": cells * 8 / res["jvp_s"] / 1e9,
                           # P^-1 J as the step applies it (the stencil fused into the x-FFT when tuned so):
                           # x read and the result written (4 B each per cell), the half spectrum written
                           # by the x-FFT and read by the inverse (8 B each per complex unknown), the
                           # tridiagonal stage (24 B per complex unknown)
                           "gmres_operator_us": res["op_s"] * 1e6,
                           "gmres_operator_achieved_GBps": (cells * 8 + res["mode_rows"] * 40) / res["op_s"] / 1e9}}
    fe = res["fe_rel"]
    cpu = None
    fe_err = {"steps": args.warmup + args.steps, "max": float(fe.max()), "median": float(np.median(fe)),
              "vs": "plain FP64 GPU step"}
    if not args.no_cpu_baseline:
        cpu, fe_o = cpu_baseline_run(specs_for(0), args.warmup + args.steps)
        specs = res["specs"]

        def err(a):
            e = np.abs(a - fe_o) / np.abs(fe_o)
            i = int(np.argmax(e))
            return {"max": float(e.max()), "median": float(np.median(e)),
                    "worst": {"instance": i, "family": specs[i]["family"], "nx": specs[i]["nx"],
                              "nv": specs[i]["nv"], "amp": specs[i]["amp"], "k": specs[i]["k"],
                              "field_energy": float(fe_o[i])}}
        fe_err = {"steps": args.warmup + args.steps, "max": None, "median": None,
                  "vs": "FP64 oracle (the C port, same instances, same steps)",
                  "batched_mixed": err(res["fe_m"]), "plain_fp64_gpu": err(res["fe_p"]),
                  "batched_fp64": err(res["fe_b"]),
                  "batched_mixed_vs_plain_fp64_gpu": {"max": float(fe.max()), "median": float(np.median(fe))}}
        fe_err["max"] = fe_err["batched_mixed"]["max"]
        fe_err["median"] = fe_err["batched_mixed"]["median"]
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["t_value"] * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 inner / f64 outer (mixed)",
            "data": "synthetic (seeded analytic initial data)", "config": config,
            "plain_fp64": {"value": plain, "unit": METRIC, "ms_per_step": res["t_plain"] * 1e3 / args.steps,
                           "ratio_batched_mixed": value / plain},
            "batched_fp64": {"value": b64, "unit": METRIC, "ms_per_step": res["t_b64"] * 1e3 / args.steps,
                             "ratio_vs_plain": b64 / plain, "ratio_batched_mixed_vs_this": value / b64,
                             "ksp_rtol": 1e-4, "field_energy_rel_err_vs_plain_max": float(res["fe_rel_b64"].max())},
            "step_roofline": step_roofline,
            "field_energy_rel_err": fe_err,
            "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": cells * 8, "d2h_bytes_per_step": cells * 8},
            "gpu_launches": res["launches"], "roofline": roofline, "clocks": res["clocks"],
            "iterations": {"picard_per_step_mean": res["picard"], "gmres_per_step_mean": res["gmres"]}}
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line))


if __name__ == "__main__":
    main()
