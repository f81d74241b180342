"""Launch-shape autotuner: measures the team size (CTAs per problem) of batched solves per
problem class and writes the table the library applies (rb_set_launch_rules).

A class is a representative set of problems (the configurations' shapes and the serving stream's
size bins), measured at two batch sizes (a small batch and a full one: the best team depends on
how many problems share the GPU). For each (class, batch size) the tuner uploads the batch once,
times rb_solve_batch at every candidate team size (a rule covering exactly that batch, wall clock
around the synchronised launch, best of `reps` after a warm-up solve) and keeps the fastest.
Rules are written small batches first, then in increasing order of work, each covering the
problems up to its class's largest direction count and work and batches up to its size, so a
batch takes the rule of the smallest class and batch size that contain it.

    python -m radiant_b200.autotune --out radiant_b200/launch_rules.json
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import workloads as W
from ._abi import Context, PackedProblem


def work_of(tabs: dict) -> float:
    """The library's work estimate of a problem (problem_work in rb_capi.cu)."""
    ncell = int(np.prod(tabs["ns"]))
    return float(tabs["ng"]) * tabs["nd"] * ncell * tabs["nm"][4] * (2.0 if tabs["solver_type"] >= 2 else 1.0)


SMALL_BATCH, FULL_BATCH = 24, 150


def default_classes(seed: int = 1) -> dict:
    """Representative 1D problem sets of FULL_BATCH problems: the two slab configurations and
    three size bins of the serving stream's slab requests (by work)."""
    c1 = [W.c1_tables(seed=s) for s in range(1, FULL_BATCH + 1)]
    c2 = [W.c2_tables(seed=s, particle=p) for s in range(1, FULL_BATCH // 3 + 1)
          for p in ("photon", "electron", "positron")]
    rng = np.random.default_rng(seed)
    slabs = [W.random_slab_tables(int(rng.integers(0, 2 ** 31 - 1))) for _ in range(3 * FULL_BATCH)]
    slabs.sort(key=work_of)
    k = len(slabs) // 3
    return {"serving slabs, small": slabs[:k], "serving slabs, medium": slabs[k:2 * k],
            "serving slabs, large": slabs[2 * k:], "1D photon slab (200 cells, S16)": c1,
            "1D coupled slab (300 cells, 80 groups, S32)": c2}


def time_batch(ctx: Context, handles: list, reps: int) -> float:
    """Seconds per rb_solve_batch of the handles (best of `reps`, after one warm-up solve)."""
    import torch

    ctx.solve_batch(handles)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.solve_batch(handles)
        torch.cuda.synchronize()
        best = min(best, time.perf_counter() - t0)
    return best


def tune(classes: dict, candidates=(2, 4, 8, 16), reps: int = 2, sizes=(SMALL_BATCH, FULL_BATCH)) -> dict:
    """Measures every class at every batch size and candidate team size; returns the table and
    the timings."""
    ctx = Context(0, 0, launch_rules=None)
    entries = []
    for name, probs in classes.items():
        nd_max = max(t["nd"] for t in probs)
        wmax = max(work_of(t) for t in probs)
        for size in sizes:
            # a seeded sample that keeps the set's composition (particles, sizes)
            pick = np.sort(np.random.default_rng(size).choice(len(probs), size=min(size, len(probs)), replace=False))
            batch = [probs[i] for i in pick]
            handles = [ctx.upload(PackedProblem(t)) for t in batch]
            times = {}
            for c in candidates:
                ctx.set_launch_rules([{"ndims": batch[0]["ndims"], "nd_max": nd_max, "work_max": int(wmax) + 1,
                                       "batch_max": len(batch), "cluster": c}])
                times[c] = time_batch(ctx, handles, reps)
            for h in handles:
                ctx.release(h)
            ctx.set_launch_rules([])
            best = min(times, key=times.get)
            entries.append({"class": name, "ndims": int(batch[0]["ndims"]), "nd_max": int(nd_max),
                            "work_max": int(wmax) + 1, "batch_max": len(batch) if size != sizes[-1] else 2 ** 31 - 1,
                            "cluster": int(best), "problems": len(batch),
                            "seconds": {str(c): round(t, 5) for c, t in times.items()}})
    ctx.close()
    entries.sort(key=lambda e: (e["batch_max"], e["work_max"]))
    rules = [{k: e[k] for k in ("ndims", "nd_max", "work_max", "batch_max", "cluster")} for e in entries]
    return {"rules": rules, "measured": entries}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None, help="where to write the table (JSON)")
    ap.add_argument("--reps", type=int, default=2)
    args = ap.parse_args()
    table = tune(default_classes(), reps=args.reps)
    text = json.dumps(table, indent=1)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text + "\n")
    print(text)


if __name__ == "__main__":
    main()
