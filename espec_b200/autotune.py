"""Autotuner of the batched split-operator kernels.

For every packet size and arithmetic form it times each kernel variant
(radix plan, location of the per-point tables, register budget; for
256-point mixed packets also the tensor-core DFT variant) on a batch large
enough to fill the GPU, and reports the fastest.  The library's built-in
defaults (default_variant in spo1d.cu) are the result of this run on B200.

Packing (--packing): the persistent launch groups the packets of one size
into items that fill a CTA and claims them longest first; the tuner times
one item of every size (a batch of that size alone in the persistent
kernel, time x CTA slots / items), then the whole scan with the default
item costs, with the measured costs and with the per-class launch, and
reports the fastest shape.  `SpoBatch.set_item_cost` applies a measured
table.

    python -m espec_b200.autotune [--steps 300] [--out tuned.json] [--packing]
"""
import argparse
import json

import numpy as np

from . import _native as N
from . import workloads as W
from .spo import SpoBatch

SIZES = (256, 384, 512, 768, 1024, 1536, 2048, 4096)
# packets per persistent item: 256 threads over the threads one packet of
# each size takes in the persistent kernel's plan
ITEM_PACKETS = {256: 8, 384: 8, 512: 4, 768: 4, 1024: 2, 1536: 2, 2048: 1}


def _timed_runs(b, nsteps, reps=3):
    import torch

    s = torch.cuda.current_stream().cuda_stream
    b.run(nsteps, stream=s)  # warm-up (also sizes the C(t) buffer)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        b.run(nsteps, stream=s)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def time_variant(n, variant, precision, npk, nsteps, reps=3):
    w = W.morse_scan(npk=npk, nsteps=nsteps, sizes=(n,), seed=3)
    b = SpoBatch(w["n"], w["sh"], w["sm"], w["dt_fs"], precision=precision)
    b.set_variant(n, variant)
    b.load(w["vpot"], w["psi"])
    ms = _timed_runs(b, nsteps, reps)
    b.close()
    return float(w["off"][-1]) * nsteps / (ms * 1e-3) / 1e9  # G gridpt*steps/s


def item_costs(precision, nsteps, sms=148):
    """ms of one persistent item of each size (4 waves of items on the GPU)."""
    out = {}
    for n, g in ITEM_PACKETS.items():
        nitems = 4 * sms
        w = W.morse_scan(npk=g * nitems, nsteps=nsteps, sizes=(n,), seed=4)
        b = SpoBatch(w["n"], w["sh"], w["sm"], w["dt_fs"], precision=precision)
        b.set_launch("persistent")
        b.load(w["vpot"], w["psi"])
        out[n] = _timed_runs(b, nsteps) * sms / nitems
        b.close()
    return out


def scan_shapes(precision, nsteps, costs):
    """The 4096-packet scan in each launch shape: G gridpt*steps/s."""
    w = W.morse_scan(nsteps=nsteps)
    res = {}
    for name in ("classes", "persistent_default", "persistent_measured"):
        b = SpoBatch(w["n"], w["sh"], w["sm"], w["dt_fs"], precision=precision)
        b.set_launch("classes" if name == "classes" else "persistent")
        if name == "persistent_measured":
            for n, c in costs.items():
                b.set_item_cost(n, c)
        b.load(w["vpot"], w["psi"])
        res[name] = float(w["off"][-1]) * nsteps / (_timed_runs(b, nsteps) * 1e-3) / 1e9
        b.close()
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--out", default=None)
    ap.add_argument("--sizes", default=None)
    ap.add_argument("--packing", action="store_true")
    args = ap.parse_args()
    res = {}
    if args.packing:
        for prec in ("fp64", "mixed"):
            costs = item_costs(prec, args.steps)
            res[prec] = {"item_ms": costs, "scan_gpts": scan_shapes(prec, args.steps, costs)}
            print(prec, json.dumps(res[prec]), flush=True)
    else:
        nvar = N.load().espec_spo_variant_count()
        sizes = [int(x) for x in args.sizes.split(",")] if args.sizes else SIZES
        for prec in ("mixed", "fp64"):
            res[prec] = {}
            for n in sizes:
                npk = max(148 * 8, 148 * 8 * 1024 // n)  # several waves of CTAs
                variants = list(range(nvar))
                if prec == "mixed" and n == 256:
                    variants.append(N.VARIANT_TC)
                rates = []
                for v in variants:
                    try:
                        rates.append(time_variant(n, v, prec, npk, args.steps))
                    except Exception as e:  # a variant may not launch (resources)
                        rates.append(0.0)
                        print(f"  {prec} n={n} v={v}: {e}")
                best = variants[int(np.argmax(rates))]
                res[prec][n] = {"best": best, "gpts": dict(zip(variants, rates))}
                print(f"{prec:5s} n={n:5d} "
                      + " ".join(f"v{v}:{r:7.1f}" for v, r in zip(variants, rates))
                      + f"  -> v{best}", flush=True)
    if args.out:
        with open(args.out, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
