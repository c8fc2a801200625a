"""Trajectories of the single-run workloads at their full lengths, against the
C port of the oracle (a test-side script; it writes the records under
results/).

  landau_linear     64 x 256, f0 = (1 + 0.01 cos 0.5x) M(v), L = 4 pi,
                    v in [-10, 10], dt 0.1, 100 steps, Picard 1e-12, FP64:
                    every invariant against the port at every step.
  twostream         512 x 1024, f0 = v^2 M(v) (1 + 0.05 cos 0.5x), v in [-8, 8],
                    dt 0.05, 400 steps, FP64: invariant drift and the
                    field-energy trace, against the port every 10 steps.
  landau_nonlinear  1024 x 2048, f0 = (1 + 0.5 cos 0.5x) M(v), v in [-10, 10],
                    dt 0.05, 1000 steps: mixed precision and FP64 on the GPU,
                    field energy and mass / L2 / energy / entropy against the
                    FP64 port every 10 steps.

M(v) = exp(-v^2/2)/sqrt(2 pi); J4 bracket, tensor_kinetic preconditioner,
GMRES(30) with ksp_rtol 1e-4, Picard tolerance 1e-10 unless stated.

    python tests/baseline_configs.py gpu  --config twostream --out DIR   # GPU part (npz)
    python tests/baseline_configs.py port --config twostream --out DIR   # C port part (npz, host)
    python tests/baseline_configs.py record --config twostream --out DIR # results/<config>.json

The GPU and host parts can run on different machines: the record step reads
both npz files.
"""
import argparse
import json
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

CONFIGS = {
    "landau_linear": dict(nx=64, nv=256, vmax=10.0, ht=0.1, amp=0.01, family="landau", steps=100, atol=1e-12,
                          every=1, precisions=("fp64",)),
    "twostream": dict(nx=512, nv=1024, vmax=8.0, ht=0.05, amp=0.05, family="twostream", steps=400, atol=1e-10,
                      every=10, precisions=("fp64",)),
    "landau_nonlinear": dict(nx=1024, nv=2048, vmax=10.0, ht=0.05, amp=0.5, family="landau", steps=1000,
                             atol=1e-10, every=10, precisions=("mixed", "fp64")),
}
NAMES = ("mass", "L1", "L2", "entropy", "E_kin", "E_pot", "energy", "momentum", "field_energy")
L = 4 * math.pi
K = 0.5


def initial_f(c):
    """(nv, nx) initial data before normalisation, band rows zeroed."""
    x = np.arange(c["nx"]) * (L / c["nx"])
    v = -c["vmax"] + np.arange(c["nv"]) * (2 * c["vmax"] / (c["nv"] - 1))
    X, V = np.meshgrid(x, v, indexing="xy")
    m = np.exp(-V ** 2 / 2) / math.sqrt(2 * math.pi)
    f = (V ** 2 * m if c["family"] == "twostream" else m) * (1 + c["amp"] * np.cos(K * X))
    f[:2] = 0.
    f[-2:] = 0.
    return np.ascontiguousarray(f)


def gpu_part(name, out):
    import torch
    from bench import ClockSampler
    from vivlasov1d_b200 import workloads as W
    c = CONFIGS[name]
    res = {}
    for prec in c["precisions"]:
        cfg = W.config(c["nx"], c["nv"], L, -c["vmax"], c["vmax"], c["ht"], snes_atol=c["atol"])
        from vivlasov1d_b200.run import Run
        run = Run(cfg, f0=torch.from_numpy(initial_f(c)), precision=prec)
        inv = [run.invariants()]
        pic, gm = [], []
        sampler = ClockSampler(0)
        sampler.start()
        torch.cuda.synchronize()
        t_dev = 0.0
        for k in range(1, c["steps"] + 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            r = run.step()
            e1.record()
            e1.synchronize()
            t_dev += e0.elapsed_time(e1) / 1e3
            pic.append(r["picard_its"])
            gm.append(sum(r["gmres_its"]))
            if k % c["every"] == 0:
                inv.append(run.invariants())
        clocks = sampler.stop()
        res[prec] = dict(inv=np.array([[d[n] for n in NAMES] for d in inv]), picard=np.array(pic),
                         gmres=np.array(gm), seconds=t_dev, clocks=json.dumps(clocks))
        del run
    np.savez(os.path.join(out, "%s_gpu.npz" % name),
             **{"%s_%s" % (p, k): v for p, d in res.items() for k, v in d.items()})


def port_part(name, out):
    from oracle.c import CPort
    from oracle import vlasov_oracle as vo
    c = CONFIGS[name]
    og = vo.Grid(c["nx"], c["nv"], L, c["vmax"], -c["vmax"], ht=c["ht"])
    p = CPort(c["nx"], c["nv"], L, -c["vmax"], c["vmax"], c["ht"], ksp_rtol=1e-4, snes_atol=c["atol"])
    p.set_f(initial_f(c))

    def inv():
        d = vo.invariants(vo.from_flat(p.f()), p.phi(), og)
        return [d[n] for n in NAMES]
    rows = [inv()]
    pic, gm = [], []
    t0 = time.perf_counter()
    for k in range(1, c["steps"] + 1):
        a, b = p.step()
        pic.append(a)
        gm.append(b)
        if k % c["every"] == 0:
            rows.append(inv())
    np.savez(os.path.join(out, "%s_port.npz" % name), inv=np.array(rows), picard=np.array(pic), gmres=np.array(gm),
             seconds=time.perf_counter() - t0, threads=p.threads)


def rel_err(a, b):
    """|a - b| / |b| per recorded step and invariant; the momentum of these
    symmetric initial data is zero up to round-off, so its error is taken
    relative to the mass instead."""
    den = np.maximum(np.abs(b), 1e-300)
    e = np.abs(a - b) / den
    k, m = NAMES.index("momentum"), NAMES.index("mass")
    e[:, k] = np.abs(a[:, k] - b[:, k]) / np.abs(b[:, m])
    return e


def record(name, out):
    c = CONFIGS[name]
    g = np.load(os.path.join(out, "%s_gpu.npz" % name))
    o = np.load(os.path.join(out, "%s_port.npz" % name))
    cells = c["nx"] * c["nv"]
    t = np.arange(0, c["steps"] + 1, c["every"]) * c["ht"]
    rec = {"config": name, "grid": [c["nx"], c["nv"]], "steps": c["steps"], "dt": c["ht"], "amp": c["amp"],
           "family": c["family"], "picard_atol": c["atol"], "ksp_rtol": 1e-4, "recorded_every": c["every"],
           "commands": ["python tests/baseline_configs.py gpu --config %s --out DIR" % name,
                        "python tests/baseline_configs.py port --config %s --out DIR" % name,
                        "python tests/baseline_configs.py record --config %s --out DIR" % name],
           "port": {"note": "host timing of the check run (its threads shared with other host work): not a "
                            "benchmark figure",
                    "seconds": float(o["seconds"]), "threads": int(o["threads"]),
                    "picard_mean": float(o["picard"].mean()), "gmres_mean": float(o["gmres"].mean()),
                    "Gcell_steps_per_s": cells * c["steps"] / float(o["seconds"]) / 1e9}}
    oi = o["inv"]
    rec["port"]["drift"] = {n: float(abs(oi[-1, k] - oi[0, k]) / abs(oi[0, k]))
                            for k, n in enumerate(NAMES) if n in ("mass", "L2", "energy", "entropy")}
    for prec in c["precisions"]:
        gi = g["%s_inv" % prec]
        e = rel_err(gi, oi)
        d = {"ms_per_step": float(g["%s_seconds" % prec]) * 1e3 / c["steps"],
             "Gcell_steps_per_s": cells * c["steps"] / float(g["%s_seconds" % prec]) / 1e9,
             "picard_mean": float(g["%s_picard" % prec].mean()), "gmres_mean": float(g["%s_gmres" % prec].mean()),
             "picard_steps_equal_to_port": int((g["%s_picard" % prec] == o["picard"]).sum()),
             "clocks": json.loads(str(g["%s_clocks" % prec])),
             "rel_err_vs_port": {n: {"max": float(e[:, k].max()), "median": float(np.median(e[:, k])),
                                     "at_end": float(e[-1, k])} for k, n in enumerate(NAMES)},
             "drift": {n: float(abs(gi[-1, k] - gi[0, k]) / abs(gi[0, k]))
                       for k, n in enumerate(NAMES) if n in ("mass", "L2", "energy", "entropy")}}
        rec[prec] = d
    if "mixed" in c["precisions"] and "fp64" in c["precisions"]:
        e = rel_err(g["mixed_inv"], g["fp64_inv"])
        rec["mixed_vs_fp64_gpu"] = {n: {"max": float(e[:, k].max()), "median": float(np.median(e[:, k]))}
                                    for k, n in enumerate(NAMES)}
    fe = NAMES.index("field_energy")
    stride = max(1, len(t) // 50)
    key = "fp64" if "fp64" in c["precisions"] else c["precisions"][0]
    rec["field_energy_trace"] = {"t": [float(x) for x in t[::stride]],
                                 "gpu": [float(x) for x in g["%s_inv" % key][::stride, fe]],
                                 "port": [float(x) for x in oi[::stride, fe]]}
    os.makedirs(os.path.join(ROOT, "results"), exist_ok=True)
    path = os.path.join(ROOT, "results", "%s.json" % name)
    with open(path, "w") as fh:
        json.dump(rec, fh, indent=1)
    print(path)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("part", choices=["gpu", "port", "record"])
    ap.add_argument("--config", required=True, choices=sorted(CONFIGS))
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    {"gpu": gpu_part, "port": port_part, "record": record}[a.part](a.config, a.out)


if __name__ == "__main__":
    main()
