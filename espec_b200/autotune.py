"""Autotuner of the batched split-operator kernels.

For every packet size and arithmetic form it times each kernel variant
(radix plan, location of the per-point tables, register budget) on a batch
large enough to fill the GPU, and reports the fastest.  The library's
built-in defaults (default_variant in spo1d.cu) are the result of this run
on B200; `tuned_variants()` returns a saved table for SpoBatch users who
retune on other parts.

    python -m espec_b200.autotune [--steps 300] [--out tuned.json]
"""
import argparse
import json
import os
import time

import numpy as np

from . import _native as N
from . import workloads as W
from .spo import SpoBatch

SIZES = (256, 384, 512, 768, 1024, 1536, 2048, 4096)


def time_variant(n, variant, precision, npk, nsteps, reps=3):
    import torch

    w = W.morse_scan(npk=npk, nsteps=nsteps, sizes=(n,), seed=3)
    b = SpoBatch(w["n"], w["sh"], w["sm"], w["dt_fs"], precision=precision)
    b.set_variant(n, variant)
    dev = torch.device("cuda")
    v = torch.from_numpy(w["vpot"]).to(dev)
    p = torch.from_numpy(w["psi"]).to(dev)
    z = torch.zeros_like(p)
    s = torch.cuda.current_stream().cuda_stream
    b.load(v, (p, z), stream=s)
    b.run(nsteps, stream=s)  # warm-up (also sizes the C(t) buffer)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        b.run(nsteps, stream=s)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    b.close()
    return float(w["off"][-1]) * nsteps / (ms * 1e-3) / 1e9  # G gridpt*steps/s


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--out", default=None)
    ap.add_argument("--sizes", default=None)
    args = ap.parse_args()
    nvar = N.load().espec_spo_variant_count()
    sizes = [int(x) for x in args.sizes.split(",")] if args.sizes else SIZES
    res = {}
    for prec in ("mixed", "fp64"):
        res[prec] = {}
        for n in sizes:
            npk = max(148 * 8, 148 * 8 * 1024 // n)  # several waves of CTAs
            rates = []
            for v in range(nvar):
                try:
                    rates.append(time_variant(n, v, prec, npk, args.steps))
                except Exception as e:  # a variant may not launch (resources)
                    rates.append(0.0)
                    print(f"  {prec} n={n} v={v}: {e}")
            best = int(np.argmax(rates))
            res[prec][n] = {"best": best, "gpts": rates}
            print(f"{prec:5s} n={n:5d} " + " ".join(f"v{i}:{r:7.1f}" for i, r in enumerate(rates))
                  + f"  -> v{best}", flush=True)
    if args.out:
        with open(args.out, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
