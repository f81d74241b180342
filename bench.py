#!/usr/bin/env python
"""Benchmark of the SN transport solve: cell-direction-group updates per second.

Workload (one step): a batch of independent 1D slab coupled-BFP particle solves with the
shapes of the 1D coupled Boltzmann Fokker-Planck configuration -- water 0-3 cm / cortical
bone 3-5 cm / water 5-15 cm, 300 voxels, 80 log groups 1 keV-20 MeV, S32 Gauss-Legendre,
P15, linear DG in x (and in E for the charged particles), Galerkin angular Fokker-Planck,
normal beam in the 6 MeV group -- one photon (BTE), one electron (BFP) and one positron
(BFP) solve per seed, `--seeds` seeds. Cross sections are seeded synthetic tables with the
configuration's shapes (the reference's physics generator is not available here).

  value  updates/s over the batch, inputs resident in HBM, one persistent launch per step
  e2e    the same through the C ABI with host buffers: upload (H2D) + solve + download (D2H)
  unit   of work: one (cell, direction) visit inside one transport pass of one group;
         updates = Σ passes × cells × directions, passes as counted by the reference.

`--impl reference` times the oracle port of the reference's CPU solve (the reference is
Julia, unavailable here) on all host cores over a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "radiant.jl_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "cell-dir-group updates/s"
# DRAM bytes per update of solve_local1d_kernel, from one ncu capture (dram__bytes_read.sum +
# dram__bytes_write.sum) of 18 electron solves of this workload reduced to 8 groups, FP64;
# traffic grows in proportion to the updates, so a launch's traffic is this times its updates.
TRAFFIC_BYTES_PER_UPDATE = 399.8
PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")


def kernel_name(workload="c2"):
    """The persistent kernel the workload runs on: every 1D problem of the benchmark's workloads
    takes the local (cell-split) pass, whose batches run on their own kernel; a 3D problem runs on
    the whole GPU as one cooperative launch."""
    if workload == "c4g1":
        return "solve_grid_kernel"
    return "solve_batch_kernel" if os.environ.get("RB_LOCAL1D", "1") == "0" else "solve_local1d_kernel"


def peaks():
    try:
        with open(PEAKS_PATH) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload_tables(seeds, precision, workload="c2"):
    from radiant_b200 import workloads as W

    tabs = []
    if workload == "c1":  # small case (profiling): the 1D photon BTE slab, one solve per seed
        return [W.c1_tables(seed=s, precision=precision) for s in seeds]
    if workload == "c2e8":  # small case (profiling): the electron BFP solve of the workload, 8 groups
        return [W.c2_tables(seed=s, precision=precision, ng=8) for s in seeds]
    if workload == "c4g1":  # small case (profiling): the C4-shaped 3D photon solve, one group
        return [W.c4_tables(seed=s, ng=1) for s in seeds]
    for s in seeds:
        for part in ("photon", "electron", "positron"):
            t = W.c2_tables(seed=s * 3 + {"photon": 0, "electron": 1, "positron": 2}[part], precision=precision,
                            particle="photon" if part == "photon" else "electron")
            t["particle"] = part
            tabs.append(t)
    return tabs


def algorithmic_bytes(t, passes, w=8):
    """Minimal HBM traffic of a fused pass (per pass: read Qlout and 𝚽, write 𝚽, the material
    id; energy-face fluxes in and out for CSD) × passes."""
    ncell = int(np.prod(t["ns"]))
    nm5, np_, nd = t["nm"][4], t["np"], t["nd"]
    b = ncell * (3 * np_ * nm5 * w + 4)
    if t["solver_type"] >= 2:
        b += ncell * nd * 2 * t["nm"][3] * w
    return b * passes


def max_over_ranks(value: float, world: int, device: str = "cuda") -> float:
    """The largest value over all ranks (every rank gets it): timings are max over ranks."""
    if world <= 1:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                parts = [p.strip() for p in out.stdout.strip().split(",")]
                if len(parts) >= 7:
                    self.samples.append(parts)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=6)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[3 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ------------------------------------------------------------------------------------------
# our arm
# ------------------------------------------------------------------------------------------
def run_ours(args, rank, world):
    import torch

    from radiant_b200._abi import Context, PackedProblem, ResultBuffers

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    seeds = [1 + rank * 1000 + k for k in range(args.seeds)]
    tabs = workload_tables(seeds, args.precision, args.workload)
    ctx = Context(dev, 0)
    packs = [PackedProblem(t) for t in tabs]
    handles = [ctx.upload(p) for p in packs]
    # a dedicated stream: the library launches on it and the CUDA events are recorded on it
    stream = torch.cuda.Stream(dev)
    sptr = stream.cuda_stream
    rbs = [ResultBuffers(p) for p in packs]

    def step():
        ctx.solve_batch(handles, sptr)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # passes per problem (identical every step: the solve is deterministic)
    for h, rb in zip(handles, rbs):
        ctx.download(h, rb)
    updates = sum(rb.passes * int(np.prod(t["ns"])) * t["nd"] for rb, t in zip(rbs, tabs))
    abytes = sum(algorithmic_bytes(t, rb.passes, 8 if args.precision == "fp64" else 4) for rb, t in zip(rbs, tabs))
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, world)
    value = updates * world / (ms / 1e3)

    # e2e through the C ABI with host buffers: upload + solve + download per step
    h2d = sum(p_bytes(t) for t in tabs)
    d2h = sum(rb.flux.nbytes + (rb.flux_cutoff.nbytes if rb.flux_cutoff is not None else 0)
              + rb.rho.nbytes + rb.group_iters.nbytes + rb.group_resid.nbytes + rb.group_converged.nbytes
              for rb in rbs)
    for h in handles:
        ctx.release(h)
    e2e_steps = max(1, min(args.steps, 2))

    def e2e_step():
        hs = [ctx.upload(p) for p in packs]
        ctx.solve_batch(hs, sptr)
        for h, rb in zip(hs, rbs):
            ctx.download(h, rb)
        for h in hs:
            ctx.release(h)

    e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / e2e_steps, world)

    # the mixed-precision form on the same batch (FP32 angular work, FP64 Krylov; 1e-5 contract)
    mixed = None
    if args.precision == "fp64" and not args.no_mixed:
        mtabs = workload_tables(seeds, "mixed", args.workload)
        mpacks = [PackedProblem(t) for t in mtabs]
        mh = [ctx.upload(p) for p in mpacks]
        for _ in range(max(1, args.warmup)):
            ctx.solve_batch(mh, sptr)
        torch.cuda.synchronize()
        mrbs = [ResultBuffers(p) for p in mpacks]
        for h, rb in zip(mh, mrbs):
            ctx.download(h, rb)
        mupd = sum(rb.passes * int(np.prod(t["ns"])) * t["nd"] for rb, t in zip(mrbs, mtabs))
        err = max(float(np.linalg.norm(a.flux - b.flux) / max(np.linalg.norm(b.flux), 1e-300)) for a, b in zip(mrbs, rbs))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            ctx.solve_batch(mh, sptr)
        e1.record(stream)
        torch.cuda.synchronize()
        mms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
        for h in mh:
            ctx.release(h)
        mixed = {"value": mupd * world / (mms / 1e3), "unit": "updates/s", "ms_per_step": mms,
                 "solves_per_s": len(mtabs) * world / (mms / 1e3), "fp64_solves_per_s": len(tabs) * world / (ms / 1e3),
                 "max_rel_l2_vs_fp64": err, "passes": int(sum(rb.passes for rb in mrbs)),
                 "fp64_passes": int(sum(rb.passes for rb in rbs))}

    serving = run_serving(args, ctx, dev) if (args.serve > 0 and rank == 0) else None
    ctx.close()

    peak, pk = peaks()
    achieved = abytes / (ms / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic (seeded cross-section tables with the configuration's shapes)",
        "config": {"workload": "1D slab coupled BFP: 300 voxels (water/bone/water), 80 groups, S32, P15, "
                               "linear DG in x and E, Galerkin angular FP, 6 MeV beam; photon+electron+positron "
                               f"solves x {args.seeds} seeds per GPU", "problems_per_gpu": len(tabs),
                   "precision": args.precision, "accel": "gmres(30)", "tol": 1e-8,
                   "l2": "per-step working set (flux + Krylov vectors of every problem) exceeds the 126 MB L2",
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": TRAFFIC_BYTES_PER_UPDATE * updates if args.workload == "c2" and args.precision == "fp64" else None,
                     "traffic_note": "bytes per launch, scaled from an ncu capture of the reduced workload",
                     "algorithmic_bytes": abytes, "peak_source": pk, "kernel": kernel_name(args.workload)},
        "e2e": {"value": updates * world / (e2e_ms / 1e3), "unit": "updates/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
    }
    if mixed:
        line["mixed_form"] = mixed
    if serving:
        line["serving"] = serving
    return line


def run_serving(args, ctx, dev):
    """A bounded serving run: a seeded Poisson stream of requests from the serving mix through
    rb_submit / rb_poll (continuous batching, mixed form for 1D requests), against plain FP64
    per-request solves of the same requests, one at a time."""
    from radiant_b200 import serving as S
    from radiant_b200 import workloads as W
    from radiant_b200._abi import PackedProblem, ResultBuffers

    n = args.serve
    reqs_t = W.serving_stream(n, seed=2024, precision="mixed", max_cells=args.serve_cells,
                              max_groups=args.serve_groups, max_side=args.serve_side)
    arrivals = S.poisson_arrivals(n, args.serve_rate, seed=7)
    # warm the request path once
    S.ServingLoop(ctx).run([S.Request(0, reqs_t[0], 0.0)])
    reqs = [S.Request(i, t, float(a)) for i, (t, a) in enumerate(zip(reqs_t, arrivals))]
    S.ServingLoop(ctx).run(reqs)
    served = S.latency_summary(reqs)
    upd = sum(r.result.passes * int(np.prod(r.tables["ns"])) * r.tables["nd"] for r in reqs)
    span = max(r.finished for r in reqs) - min(r.arrival for r in reqs)
    served["updates_per_s"] = upd / span
    # plain FP64, one request at a time (per-request drop-in solves)
    base_t = [dict(t, precision="fp64") for t in reqs_t]
    lat = []
    t_all = time.perf_counter()
    bupd = 0
    for t in base_t:
        pp = PackedProblem(t)
        rb = ResultBuffers(pp)
        t0 = time.perf_counter()
        h = ctx.upload(pp)
        ctx.solve(h)
        ctx.download(h, rb)
        ctx.release(h)
        lat.append(time.perf_counter() - t0)
        bupd += rb.passes * int(np.prod(t["ns"])) * t["nd"]
    t_all = time.perf_counter() - t_all
    lat = np.array(lat)
    return {"requests": n, "arrival_rate_per_s": args.serve_rate, "mix": "70% 1D slabs / 30% 2D grids (seeded)",
            "served": served,
            "fp64_per_request": {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                                 "solves_per_s": n / t_all, "updates_per_s": bupd / t_all}}


def p_bytes(t):
    """Bytes of the host tables rb_upload copies for one problem."""
    tot = 0
    for k, v in t.items():
        if isinstance(v, np.ndarray) and k not in ("w", "pm", "omega"):
            tot += v.nbytes
        elif isinstance(v, list):
            tot += sum(a.nbytes for a in v if isinstance(a, np.ndarray))
    return tot


# ------------------------------------------------------------------------------------------
# CPU legs (the oracle port of the reference's CPU solve)
# ------------------------------------------------------------------------------------------
def _cpu_one(args_):
    seed, particle = args_
    sys.path.insert(0, os.path.join(ROOT, "radiant.jl_b200"))
    sys.path.insert(0, ROOT)
    from oracle import run as orun
    from radiant_b200 import workloads as W

    t = W.c2_tables(seed=seed, particle="photon" if particle == "photon" else "electron")
    t0 = time.perf_counter()
    rb = orun.solve(t)
    dt = time.perf_counter() - t0
    return rb.passes * int(np.prod(t["ns"])) * t["nd"], dt


def cpu_baseline_single():
    """~10-15 s of single-thread CPU work: one photon and one electron solve."""
    u1, t1 = _cpu_one((1, "photon"))
    u2, t2 = _cpu_one((2, "electron"))
    return {"value": (u1 + u2) / (t1 + t2), "unit": "updates/s", "cores": 1, "kind": "port",
            "sample": "one photon (BTE) and one electron (BFP) solve of the workload, single thread, "
                      f"{t1 + t2:.1f} s of CPU work"}


def run_reference(args):
    ncores = os.cpu_count() or 1
    jobs = [(k + 1, "photon" if k % 3 == 0 else "electron") for k in range(ncores)]
    ctxmp = mp.get_context("spawn")
    with ctxmp.Pool(ncores) as pool:
        for _ in range(args.warmup):
            pool.map(_cpu_one, jobs[:ncores])
        vals = []
        t_all = 0.0
        for _ in range(args.steps):
            t0 = time.perf_counter()
            res = pool.map(_cpu_one, jobs)
            dt = time.perf_counter() - t0
            t_all += dt
            vals.append(sum(u for u, _ in res) / dt)
    value = statistics.mean(vals)
    line = {
        "metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_all * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "impl": "reference",
        "data": "synthetic (seeded cross-section tables with the configuration's shapes)",
        "config": {"workload": "1D slab coupled BFP (same shapes as our arm); one photon or electron solve "
                               "per host core per step", "precision": "fp64"},
        "cpu_baseline": {"value": value, "unit": "updates/s", "cores": ncores, "kind": "port",
                         "sample": f"{len(jobs)} solves per step on {ncores} processes (C restatement of the "
                                   "reference's Julia solve; Julia is not installed)"},
        "e2e": {"value": value, "unit": "updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--seeds", type=int, default=50)
    ap.add_argument("--workload", default="c2", choices=["c2", "c1", "c2e8", "c4g1"],
                    help="c2: the benchmark workload; c1 / c2e8 / c4g1: small cases for profiling captures")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cluster", type=int, default=0, help="CTAs per problem team (0: library default)")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision form")
    ap.add_argument("--serve", type=int, default=60, help="requests of the serving run (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=200.0, help="Poisson arrival rate (requests/s)")
    ap.add_argument("--serve-cells", type=int, default=2000)
    ap.add_argument("--serve-groups", type=int, default=120)
    ap.add_argument("--serve-side", type=int, default=128)
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.cluster:
        os.environ["RB_CLUSTER_SIZE"] = str(args.cluster)
    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(run_reference(args)))
        return 0
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    line = run_ours(args, rank, world)
    if rank == 0:
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_single()
        print(json.dumps(line))
    if world > 1:
        import torch

        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
