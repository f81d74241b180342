#!/usr/bin/env python
"""Benchmark of the SN transport solve: cell-direction-group updates per second.

Headline workload (one step; --workload c4, the default): the 3D Cartesian photon-electron
configuration -- 64^3 voxels over a 16 cm cube, water with a seeded 16^3-voxel bone block,
40 photon + 40 electron groups (10 keV - 6 MeV), level-symmetric S8 (80 directions, Galerkin
basis: 80 moments), P3, diamond difference, reflective Z-, isotropic volume source in the top
group inside the central 8^3 voxels, BiCGStab to 1e-6 -- in the configuration's mixed form
(FP32 sweeps, split-TF32 tensor-core moment products, FP64 Krylov and defect correction): the
photon and the electron solve of one seed per GPU, each on the whole GPU (one cooperative
launch per problem). The plain FP64 form of the same problems runs beside it, with the mixed
form's error against it. Cross sections are seeded synthetic tables with the configuration's
shapes (the reference's physics generator is not available here).

  value  updates/s of the step, inputs resident in HBM
  e2e    the same through the C ABI with page-locked host buffers: upload (H2D) + solve +
         download (D2H) of every problem per step, the next problem's upload and the previous
         problem's download overlapping the current solve
  unit   of work: one (cell, direction) visit inside one transport pass of one group;
         updates = sum of passes x cells x directions, passes as the reference counts them.

Second section: the 1D coupled-BFP batch (150 slab solves of the 1D configuration's shapes in
one persistent launch), FP64 and mixed. Third: a bounded serving run.

`--impl reference` times the oracle (the C restatement of the reference's Julia solve; Julia
is not installed) on all host cores over a bounded sample of the same 3D workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
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
# DRAM bytes per update of the workloads' dominant kernels, each from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum) of a reduced case; traffic grows in
# proportion to the updates, so a launch's traffic is this times its updates:
#   solve_local1d_kernel, 18 electron solves of the 1D batch reduced to 8 groups, FP64;
#   solve_grid_kernel, the 3D photon problem reduced to one group, mixed and FP64 forms.
TRAFFIC_BYTES_PER_UPDATE = {("c2", "fp64"): 399.8, ("c4", "mixed"): 140.9, ("c4", "fp64"): 158.2}
PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")


def kernel_name(workload="c4"):
    """The persistent kernel the workload runs on: every 1D problem of the benchmark's workloads
    takes the local (cell-split) pass, whose batches run on their own kernel; a 3D problem runs on
    the whole GPU as one cooperative launch."""
    if workload in ("c4", "c4g1"):
        return "solve_grid_kernel"
    return "solve_batch_kernel" if os.environ.get("RB_LOCAL1D", "1") == "0" else "solve_local1d_kernel"


def peaks():
    try:
        with open(PEAKS_PATH) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload_tables(seeds, precision, workload="c4", groups=None):
    from radiant_b200 import workloads as W

    tabs = []
    if workload in ("c4", "c4g1"):  # the 3D configuration: photon and electron solve per seed
        ng = 1 if workload == "c4g1" else (groups or 40)
        for s in seeds:
            for part in ("photon", "electron"):
                t = W.c4_tables(seed=s, particle=part, precision=precision, ng=ng)
                t["particle"] = part
                tabs.append(t)
        return tabs
    if workload == "c1":  # small case (profiling): the 1D photon BTE slab, one solve per seed
        return [W.c1_tables(seed=s, precision=precision) for s in seeds]
    if workload == "c2e8":  # small case (profiling): the electron BFP solve of the workload, 8 groups
        return [W.c2_tables(seed=s, precision=precision, ng=8) for s in seeds]
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
def updates_of(rbs, tabs):
    return sum(rb.passes * int(np.prod(t["ns"])) * t["nd"] for rb, t in zip(rbs, tabs))


def deposition(tabs, rbs):
    """Energy deposition summed over the particles (energy_deposition.jl:36-78), from the
    downloaded fluxes through rb_energy_deposition."""
    import ctypes as C

    from radiant_b200._abi import load_library

    lib = load_library()
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int32)
    tot = None
    for t, rb in zip(tabs, rbs):
        xs = t["xs"]
        ncell = int(np.prod(t["ns"]))
        mat = np.asfortranarray(t["mat"].astype(np.int32))
        se, rho = np.asfortranarray(xs.sigma_e), np.asfortranarray(xs.density)
        out = np.zeros(ncell)
        cf = rb.flux_cutoff if t["solver_type"] >= 2 else None
        st = lib.rb_energy_deposition(t["ng"], t["np"], t["nm"][4], ncell, t["nmat"], mat.ctypes.data_as(ip),
                                      rb.flux.ctypes.data_as(dp), None if cf is None else cf.ctypes.data_as(dp),
                                      se.ctypes.data_as(dp), rho.ctypes.data_as(dp), 1.0, out.ctypes.data_as(dp))
        assert st == 0
        tot = out if tot is None else tot + out
    return tot


def rel_l2(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def time_steps(ctx, handles, sptr, stream, steps):
    import torch

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        ctx.solve_batch(handles, sptr)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def run_ours(args, rank, world):
    import torch

    from radiant_b200._abi import Context, PackedProblem, ResultBuffers

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    seeds = [1 + rank * 1000 + k for k in range(args.seeds)]
    prec = args.precision or ("mixed" if args.workload in ("c4", "c4g1") else "fp64")
    tabs = workload_tables(seeds, prec, args.workload, args.groups)
    ctx = Context(dev, 0)
    # host tables and results in page-locked memory (rb_host_alloc), as a caller that streams
    # problems keeps them: the e2e copies then run at the host link's speed
    packs = [PackedProblem(t, pinned=True) for t in tabs]
    handles = [ctx.upload(p) for p in packs]
    # a dedicated stream: the library launches on it and the CUDA events are recorded on it
    stream = torch.cuda.Stream(dev)
    sptr = stream.cuda_stream
    rbs = [ResultBuffers(p, pinned=True) for p in packs]

    for _ in range(args.warmup):
        ctx.solve_batch(handles, sptr)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        ms = max_over_ranks(time_steps(ctx, handles, sptr, stream, args.steps), world)
    # passes per problem (identical every step: the solve is deterministic)
    for h, rb in zip(handles, rbs):
        ctx.download(h, rb)
    updates = updates_of(rbs, tabs)
    w = 8 if prec == "fp64" else 4
    abytes = sum(algorithmic_bytes(t, rb.passes, w) for rb, t in zip(rbs, tabs))
    value = updates * world / (ms / 1e3)
    for h in handles:
        ctx.release(h)

    # the plain FP64 form of the same problems (the drop-in), and the chosen form's error
    # against it on the flux moments and on the energy deposition
    plain = None
    if prec != "fp64" and not args.no_fp64:
        ftabs = workload_tables(seeds, "fp64", args.workload, args.groups)
        fpacks = [PackedProblem(t) for t in ftabs]
        fh = [ctx.upload(p) for p in fpacks]
        ctx.solve_batch(fh, sptr)
        torch.cuda.synchronize()
        frbs = [ResultBuffers(p) for p in fpacks]
        for h, rb in zip(fh, frbs):
            ctx.download(h, rb)
        fms = max_over_ranks(time_steps(ctx, fh, sptr, stream, max(1, min(args.steps, 2))), world)
        for h in fh:
            ctx.release(h)
        fupd = updates_of(frbs, ftabs)
        err_flux = max(rel_l2(a.flux, b.flux) for a, b in zip(rbs, frbs))
        err_cut = max((rel_l2(a.flux_cutoff, b.flux_cutoff) for a, b, t in zip(rbs, frbs, tabs)
                       if t["solver_type"] >= 2), default=0.0)
        err_dep = rel_l2(deposition(tabs, rbs), deposition(ftabs, frbs)) if "xs" in tabs[0] else None
        plain = {"value": fupd * world / (fms / 1e3), "unit": "updates/s", "ms_per_step": fms,
                 "solves_per_s": len(ftabs) * world / (fms / 1e3), "passes": int(sum(rb.passes for rb in frbs)),
                 "chosen_form_solves_per_s": len(tabs) * world / (ms / 1e3),
                 "chosen_form_speedup_solves": fms / ms, "chosen_form_passes": int(sum(rb.passes for rb in rbs)),
                 "chosen_form_max_rel_l2_flux": err_flux, "chosen_form_max_rel_l2_cutoff": err_cut,
                 "chosen_form_rel_l2_energy_deposition": err_dep}

    # e2e through the C ABI with host buffers: upload + solve + download per step
    h2d = sum(p_bytes(t) for t in tabs)
    d2h = sum(rb.flux.nbytes + (rb.flux_cutoff.nbytes if rb.flux_cutoff is not None else 0)
              + rb.rho.nbytes + rb.group_iters.nbytes + rb.group_resid.nbytes + rb.group_converged.nbytes
              for rb in rbs)
    e2e_steps = max(5, args.steps)

    def pipelined(upload):
        # problem k+1's tables cross the host link while problem k solves (rb_upload's copies run
        # on the context's stream, the solve on sptr); problem k's results cross back while
        # problem k+1 solves (rb_download_async queues the layout change right behind solve k
        # and the copies on the context's copy stream)
        hs = [upload(0)]
        for k in range(len(packs)):
            ctx.solve(hs[k], sptr)
            if k + 1 < len(packs):
                hs.append(upload(k + 1))
            if k > 0:
                ctx.download_wait(hs[k - 1])
                ctx.release(hs[k - 1])
            ctx.download_async(hs[k], rbs[k])
        ctx.download_wait(hs[-1])
        ctx.release(hs[-1])

    def e2e_step():
        pipelined(lambda k: ctx.upload(packs[k]))

    e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / e2e_steps, world)

    # the same e2e step with the fixed sources as definitions (rb_upload_sources): the volume
    # sources are built on the device instead of crossing the host link as dense arrays
    e2e_src = None
    if all("sources" in t for t in tabs):
        from radiant_b200.workloads import without_dense_sources

        bare = [without_dense_sources(t) for t in tabs]
        bpacks = [PackedProblem(b, pinned=True) for b, _ in bare]
        ssets = [ss for _, ss in bare]
        h2d_src = sum(p_bytes(b) for b, _ in bare) + sum(
            sum(p.nbytes for p in ss.positions) + C.sizeof(ss.boxes) + C.sizeof(ss.beams) + sum(b.nbytes for b in ss.bases)
            for ss in ssets)

        def e2e_src_step():
            pipelined(lambda k: ctx.upload_sources(bpacks[k], ssets[k])[0])

        e2e_src_step()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_src_step()
        torch.cuda.synchronize()
        src_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / e2e_steps, world)
        e2e_src = {"value": updates * world / (src_ms / 1e3), "unit": "updates/s", "h2d_bytes_per_step": h2d_src,
                   "d2h_bytes_per_step": d2h, "ms_per_step": src_ms, "steps": e2e_steps,
                   "entry": "rb_upload_sources (Volume_Source / Surface_Source definitions, arrays built on the device)"}
        del bpacks

    c2 = run_c2_section(args, ctx, sptr, stream, rank, world) if args.workload == "c4" and not args.no_c2 else None
    serving = run_serving(args, ctx, dev) if (args.serve > 0 and rank == 0) else None
    ctx.close()

    peak, pk = peaks()
    achieved = abytes / (ms / 1e3) / 1e9
    tpu = TRAFFIC_BYTES_PER_UPDATE.get((args.workload, prec))
    if args.workload == "c4":
        cfg = {"workload": "3D 64^3 photon-electron: 16 cm water cube with a 16^3 bone block, 40+40 groups, "
                           "S8 (80 directions, Galerkin 80 moments), P3, DD, reflective Z-, central 8^3 volume "
                           f"source, BiCGStab 1e-6; photon + electron solve x {args.seeds} seed(s) per GPU",
               "groups_per_particle": args.groups or 40, "problems_per_gpu": len(tabs), "precision": prec,
               "l2": "per-step working set (flux, Krylov vectors, angular flux of each problem) exceeds the 126 MB L2",
               "parallelism": f"replicas x{world}", "launches": "one cooperative launch per problem (whole GPU)"}
    else:
        cfg = {"workload": args.workload, "problems_per_gpu": len(tabs), "precision": prec,
               "parallelism": f"replicas x{world}"}
    line = {
        "metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == "fp64" else "f32 sweep + tf32x3 tensor-core products + f64 Krylov",
        "data": "synthetic (seeded cross-section tables with the configuration's shapes)",
        "config": cfg,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": tpu * updates / len(tabs) if tpu else None,
                     "traffic_note": "DRAM bytes per launch, scaled from an ncu capture of the reduced case",
                     "algorithmic_bytes_per_launch": abytes / len(tabs), "peak_source": pk,
                     "kernel": kernel_name(args.workload)},
        "e2e": {"value": updates * world / (e2e_ms / 1e3), "unit": "updates/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms, "steps": e2e_steps},
        "e2e_source_definitions": e2e_src,
        "updates_per_step": updates,
        "gpu_launches": args.steps * (len(tabs) if args.workload in ("c4", "c4g1") else 1),
        "clocks": clk.summary(),
    }
    if plain:
        line["plain_fp64_form"] = plain
    if c2:
        line["c2_batch"] = c2
    if serving:
        line["serving"] = serving
    return line


def run_c2_section(args, ctx, sptr, stream, rank, world):
    """The 1D coupled-BFP batch: 150 slab solves (photon BTE, electron and positron BFP; 300
    voxels, 80 groups, S32, P15, linear DG in x and E) in one persistent launch, FP64 and mixed."""
    from radiant_b200._abi import PackedProblem, ResultBuffers

    seeds = [1 + rank * 1000 + k for k in range(50)]
    out = {"workload": "1D slab coupled BFP (300 voxels, 80 groups, S32, P15, linear DG x and E, Galerkin FP, "
                       "6 MeV beam): photon+electron+positron x 50 seeds, one persistent launch",
           "kernel": kernel_name("c2")}
    rbs_by = {}
    for prec in ("fp64", "mixed"):
        tabs = workload_tables(seeds, prec, "c2")
        packs = [PackedProblem(t) for t in tabs]
        hs = [ctx.upload(p) for p in packs]
        ctx.solve_batch(hs, sptr)
        import torch

        torch.cuda.synchronize()
        rbs = [ResultBuffers(p) for p in packs]
        for h, rb in zip(hs, rbs):
            ctx.download(h, rb)
        ms = max_over_ranks(time_steps(ctx, hs, sptr, stream, 2), world)
        for h in hs:
            ctx.release(h)
        upd = updates_of(rbs, tabs)
        rbs_by[prec] = rbs
        out[prec] = {"value": upd * world / (ms / 1e3), "unit": "updates/s", "ms_per_step": ms,
                     "solves_per_s": len(tabs) * world / (ms / 1e3)}
        if prec == "fp64":
            ab = sum(algorithmic_bytes(t, rb.passes, 8) for rb, t in zip(rbs, tabs))
            peak, pk = peaks()
            out["fp64"]["roofline_frac"] = ab / (ms / 1e3) / 1e9 / peak
    out["mixed"]["max_rel_l2_vs_fp64"] = max(rel_l2(a.flux, b.flux) for a, b in zip(rbs_by["mixed"], rbs_by["fp64"]))
    # the team size: the packaged launch rules (radiant_b200/autotune.py) where one covers the
    # batch, else the built-in choice
    from radiant_b200.autotune import work_of
    tabs = workload_tables(seeds[:1], "fp64", "c2")
    wmax = max(work_of(t) for t in tabs)
    rule = next((r for r in ctx.launch_rules if r["ndims"] == 1 and r["nd_max"] >= tabs[0]["nd"]
                 and r["work_max"] >= wmax), None)
    out["launch_team"] = (f"{rule['cluster']} CTAs per problem (tuned rule)" if rule
                          else "built-in shape choice (no tuned rule covers the batch)")
    return out


def run_serving(args, ctx, dev):
    """A bounded serving run: the first `--serve` requests of the seeded serving stream (70 % 1D
    slabs / 30 % 2D grids, photon-only or photon+electron+positron sets, 10-`--serve-groups`
    groups, log-uniform beam energy 0.1-20 MeV), Poisson arrivals, through rb_submit / rb_poll
    (continuous batching: every admitted solve runs at once beside the others). The same stream
    is served in the mixed form and in the plain FP64 form at the same arrivals and admission
    (equal concurrency); plain FP64 per-request solves one at a time are timed on a prefix."""
    from radiant_b200 import serving as S
    from radiant_b200 import workloads as W
    from radiant_b200._abi import PackedProblem, ResultBuffers

    n = args.serve
    arrivals = S.poisson_arrivals(n, args.serve_rate, seed=7)
    out = {"requests": n, "arrival_rate_per_s": args.serve_rate,
           "stream": f"seeded serving stream: 70% 1D slabs (50-{args.serve_cells} cells, S8-S64, P1-P9, 1-5 layers "
                     f"of 4 materials) / 30% 2D grids (side 32-{args.serve_side}, S4-S12); 10-{args.serve_groups} "
                     "groups per particle; photon-only or photon+electron+positron sets with p=1/2; beam energy "
                     "log-uniform 0.1-20 MeV"}

    def solves_updates(reqs):
        return sum(rb.passes * int(np.prod(t["ns"])) * t["nd"] for r in reqs for rb, t in zip(r.results, r.parts))

    for prec in ("mixed", "fp64"):
        reqs_t = W.c5_stream(n, 2024, prec, args.serve_cells, args.serve_groups, args.serve_side)
        S.ServingLoop(ctx).run([S.Request(0, reqs_t[0], 0.0)])  # warm the request path
        reqs = [S.Request(i, t, float(a)) for i, (t, a) in enumerate(zip(reqs_t, arrivals))]
        S.ServingLoop(ctx).run(reqs)
        summ = S.latency_summary(reqs)
        span = max(r.finished for r in reqs) - min(r.arrival for r in reqs)
        summ["updates_per_s"] = solves_updates(reqs) / span
        out["served_" + prec] = summ
        if prec == "mixed":
            served_mixed = reqs
        else:
            out["mixed_vs_fp64_max_rel_l2"] = max(
                float(np.linalg.norm(a.flux - b.flux) / max(np.linalg.norm(b.flux), 1e-300))
                for ra, rb_ in zip(served_mixed, reqs) for a, b in zip(ra.results, rb_.results))
    out["mixed_over_fp64"] = {"solves_per_s": out["served_mixed"]["solves_per_s"] / out["served_fp64"]["solves_per_s"],
                              "p50": out["served_mixed"]["p50_ms"] / out["served_fp64"]["p50_ms"],
                              "p99": out["served_mixed"]["p99_ms"] / out["served_fp64"]["p99_ms"]}
    # plain FP64 per-request solves, one request at a time (no overlap), on a prefix of the stream
    m = min(n, args.serve_sequential)
    base_t = W.c5_stream(m, 2024, "fp64", args.serve_cells, args.serve_groups, args.serve_side)
    lat, nsolves = [], 0
    t_all = time.perf_counter()
    for parts in base_t:
        t0 = time.perf_counter()
        for t in parts:
            pp = PackedProblem(t)
            rb = ResultBuffers(pp)
            h = ctx.upload(pp)
            ctx.solve(h)
            ctx.download(h, rb)
            ctx.release(h)
            nsolves += 1
        lat.append(time.perf_counter() - t0)
    t_all = time.perf_counter() - t_all
    lat = np.array(lat)
    out["fp64_one_at_a_time"] = {"requests": m, "p50_ms": float(np.percentile(lat, 50) * 1e3),
                                 "p99_ms": float(np.percentile(lat, 99) * 1e3), "requests_per_s": m / t_all,
                                 "solves_per_s": nsolves / t_all}
    return out


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
# CPU legs (the oracle: the C restatement of the reference's CPU solve, on all host cores)
# ------------------------------------------------------------------------------------------
CPU_SAMPLE_ITERS = 3


def cpu_sample_tables():
    """The bounded sample of the 3D workload the CPU legs time: the photon problem of the 3D
    configuration (64^3, S8, 80 moments, reflective Z-, BiCGStab) reduced to one group and at
    most CPU_SAMPLE_ITERS BiCGStab iterations: the same shapes, passes and per-update work."""
    from radiant_b200 import workloads as W

    t = W.c4_tables(seed=1, particle="photon", ng=1)
    t["max_iter"] = CPU_SAMPLE_ITERS
    return t


def cpu_sample(tabs):
    from oracle import run as orun

    t0 = time.perf_counter()
    rb = orun.solve(tabs)
    dt = time.perf_counter() - t0
    return rb.passes * int(np.prod(tabs["ns"])) * tabs["nd"], dt, rb.passes


def cpu_baseline_single():
    """One bounded sample on the host's cores (the oracle threads over the directions)."""
    t = cpu_sample_tables()
    upd, dt, passes = cpu_sample(t)
    ncores = os.cpu_count() or 1
    return {"value": upd / dt, "unit": "updates/s", "cores": ncores, "kind": "port",
            "sample": f"the 3D photon problem (64^3, S8, 80 moments) reduced to one group, {passes} passes "
                      f"({CPU_SAMPLE_ITERS} BiCGStab iterations at most), {dt:.1f} s on {ncores} threads"}


def run_reference(args):
    ncores = os.cpu_count() or 1
    t = cpu_sample_tables()
    for _ in range(args.warmup):
        cpu_sample(t)
    vals, t_all, passes = [], 0.0, 0
    for _ in range(args.steps):
        upd, dt, passes = cpu_sample(t)
        t_all += dt
        vals.append(upd / dt)
    value = statistics.mean(vals)
    sample = (f"the 3D photon problem (64^3, S8, 80 moments, reflective Z-, BiCGStab) reduced to one group and "
              f"{CPU_SAMPLE_ITERS} iterations ({passes} passes) per step, {ncores} threads (C restatement of the "
              "reference's Julia solve; Julia is not installed)")
    line = {
        "metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_all * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "impl": "reference",
        "data": "synthetic (seeded cross-section tables with the configuration's shapes)",
        "config": {"workload": "3D 64^3 photon-electron configuration (same shapes as our arm); bounded sample: "
                               "the photon problem, one group, 3 BiCGStab iterations per step", "precision": "fp64"},
        "cpu_baseline": {"value": value, "unit": "updates/s", "cores": ncores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed"],
                    help="arithmetic form of the headline (default: mixed for c4, fp64 otherwise)")
    ap.add_argument("--seeds", type=int, default=1, help="seeds per GPU (c4: one photon + one electron solve each)")
    ap.add_argument("--groups", type=int, default=None, help="groups per particle (c4; default 40)")
    ap.add_argument("--workload", default="c4", choices=["c4", "c2", "c1", "c2e8", "c4g1"],
                    help="c4: the benchmark workload; c2: the 1D batch alone; c1 / c2e8 / c4g1: small cases "
                         "for profiling captures")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cluster", type=int, default=0, help="CTAs per problem team (0: library default)")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 form beside the chosen one")
    ap.add_argument("--no-c2", action="store_true", help="skip the 1D batch section")
    ap.add_argument("--serve", type=int, default=100,
                    help="requests of the serving run (0: skip); the full serving configuration is 2000")
    ap.add_argument("--serve-rate", type=float, default=50.0, help="Poisson arrival rate (requests/s)")
    ap.add_argument("--serve-cells", type=int, default=2000, help="largest 1D request (cells)")
    ap.add_argument("--serve-groups", type=int, default=120, help="most groups per particle")
    ap.add_argument("--serve-side", type=int, default=64,
                    help="largest 2D request side (the configuration draws up to 128)")
    ap.add_argument("--serve-sequential", type=int, default=30,
                    help="requests of the one-at-a-time FP64 control")
    args = ap.parse_args()
    if args.workload == "c2" and args.seeds == 1:
        args.seeds = 50
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
