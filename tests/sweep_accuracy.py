"""Field-energy accuracy of the batched sweep over its full length (a
test-side script; it writes results/sweep_accuracy.json).

The 256-instance seeded sweep of bench.py (Landau / two-stream /
bump-on-tail, nx 64-256, nv 128-1024, dt 0.1, J4, GMRES(30) +
tensor_kinetic, ksp_rtol 1e-4) for 200 steps at one Picard tolerance:
batched mixed precision, batched FP64 and per-instance FP64 on the GPU, and
the C port of the oracle (FP64) on the host.  Field energies are recorded at
checkpoints; the record gives, per checkpoint, the relative error of every
GPU arm against the oracle and of the mixed arm against the FP64 GPU arm
(max, median, the worst instance), and the same errors relative to each
instance's initial field energy.

    python tests/sweep_accuracy.py gpu  --atol 1e-12 --out DIR
    python tests/sweep_accuracy.py port --atol 1e-12 --out DIR
    python tests/sweep_accuracy.py record --atol 1e-12 --out DIR
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

STEPS = 200
CHECKPOINTS = (5, 10, 25, 50, 100, 150, 200)


def gpu_part(atol, out):
    import torch
    from vivlasov1d_b200 import workloads as W
    from vivlasov1d_b200.batch import Batch
    specs = W.sweep_specs()
    rec = {}
    for arm in ("mixed", "batched_fp64", "plain_fp64"):
        runs = W.sweep_runs(specs=specs, precision="mixed" if arm == "mixed" else "fp64", snes_atol=atol)
        rec["%s_fe_0" % arm] = W.field_energies(runs)
        batch = Batch(runs) if arm != "plain_fp64" else None
        pic, gm = [], []
        t0 = time.perf_counter()
        for k in range(1, STEPS + 1):
            reps = batch.step() if batch else [r.step() for r in runs]
            pic.append([r["picard_its"] for r in reps])
            gm.append([sum(r["gmres_its"]) for r in reps])
            if k in CHECKPOINTS:
                rec["%s_fe_%d" % (arm, k)] = W.field_energies(runs)
        torch.cuda.synchronize()
        rec["%s_seconds" % arm] = time.perf_counter() - t0
        rec["%s_picard" % arm] = np.array(pic)
        rec["%s_gmres" % arm] = np.array(gm)
        del batch, runs
    np.savez(os.path.join(out, "sweep_gpu_%g.npz" % atol), **rec)


def port_part(atol, out):
    from oracle.c import CPort, step_many
    from vivlasov1d_b200 import workloads as W
    specs = W.sweep_specs()
    runs = []
    for s in specs:
        p = CPort(s["nx"], s["nv"], s["L"], -10.0, 10.0, 0.1, ksp_rtol=1e-4, snes_atol=atol)
        hx, hv = s["L"] / s["nx"], 20.0 / (s["nv"] - 1)
        X, V = np.meshgrid(np.arange(s["nx"]) * hx, -10.0 + np.arange(s["nv"]) * hv, indexing="xy")
        f = W.FAMILIES[s["family"]](s["amp"], s["k"])(X, V)
        f[:2, :] = 0.
        f[s["nv"] - 2:, :] = 0.
        p.set_f(f)
        runs.append(p)
    order = sorted(range(len(specs)), key=lambda i: -specs[i]["nx"] * specs[i]["nv"])

    def fe():
        out_ = []
        for p, s in zip(runs, specs):
            phi = p.phi()
            d = np.roll(phi, -1) - phi
            out_.append(0.5 * -1.0 * (d * d).sum() / (s["L"] / s["nx"]))
        return np.array(out_)
    rec = {"oracle_fe_0": fe()}
    pic, gm = [], []
    for k in range(1, STEPS + 1):
        a, b = step_many(runs, order)
        pic.append(a)
        gm.append(b)
        if k in CHECKPOINTS:
            rec["oracle_fe_%d" % k] = fe()
    rec["oracle_picard"], rec["oracle_gmres"] = np.array(pic), np.array(gm)
    np.savez(os.path.join(out, "sweep_port_%g.npz" % atol), **rec)


def record(atol, out):
    from vivlasov1d_b200 import workloads as W
    specs = W.sweep_specs()
    g = np.load(os.path.join(out, "sweep_gpu_%g.npz" % atol))
    o = np.load(os.path.join(out, "sweep_port_%g.npz" % atol))

    def stats(a, b, b0):
        e = np.abs(a - b) / np.abs(b)
        e0 = np.abs(a - b) / np.abs(b0)
        i = int(np.argmax(e))
        s = specs[i]
        return {"max": float(e.max()), "median": float(np.median(e)),
                "max_rel_to_initial_field_energy": float(e0.max()),
                "worst": {"instance": i, "family": s["family"], "nx": s["nx"], "nv": s["nv"], "amp": s["amp"],
                          "k": s["k"], "field_energy": float(b[i]), "initial_field_energy": float(b0[i])}}
    rec = {"what": "field-energy error of the 256-instance sweep over 200 steps (dt 0.1, J4, ksp_rtol 1e-4)",
           "picard_atol": atol, "checkpoints": {},
           "commands": ["python tests/sweep_accuracy.py %s --atol %g --out DIR" % (p, atol)
                        for p in ("gpu", "port", "record")],
           "gpu_seconds_200_steps": {a: float(g["%s_seconds" % a]) for a in ("mixed", "batched_fp64", "plain_fp64")},
           "iterations_per_step": {a: {"picard": float(g["%s_picard" % a].mean()), "gmres": float(g["%s_gmres" % a].mean())}
                                   for a in ("mixed", "batched_fp64", "plain_fp64")}}
    rec["iterations_per_step"]["oracle"] = {"picard": float(o["oracle_picard"].mean()),
                                            "gmres": float(o["oracle_gmres"].mean())}
    o0 = o["oracle_fe_0"]
    p0 = g["plain_fp64_fe_0"]
    for k in CHECKPOINTS:
        ok = o["oracle_fe_%d" % k]
        rec["checkpoints"][str(k)] = {
            "mixed_vs_oracle": stats(g["mixed_fe_%d" % k], ok, o0),
            "batched_fp64_vs_oracle": stats(g["batched_fp64_fe_%d" % k], ok, o0),
            "plain_fp64_vs_oracle": stats(g["plain_fp64_fe_%d" % k], ok, o0),
            "mixed_vs_plain_fp64_gpu": stats(g["mixed_fe_%d" % k], g["plain_fp64_fe_%d" % k], p0)}
    os.makedirs(os.path.join(ROOT, "results"), exist_ok=True)
    path = os.path.join(ROOT, "results", "sweep_accuracy.json")
    with open(path, "w") as fh:
        json.dump(rec, fh, indent=1)
    print(path)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("part", choices=["gpu", "port", "record"])
    ap.add_argument("--atol", type=float, default=1e-12)
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    {"gpu": gpu_part, "port": port_part, "record": record}[a.part](a.atol, a.out)


if __name__ == "__main__":
    main()
