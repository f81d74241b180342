"""GPU parity of the two 1D passes and of the launch shapes.

A 1D problem whose cells and angular flux fit in shared memory takes the cell-split (local)
pass: each CTA of the cluster owns a cell range, keeps ψ of its cells on chip and exchanges
face maps with the other CTAs; the others take the team-wide pass. These tests pin both passes
to the oracle (1e-10 relative L2 and identical pass counts, as every FP64 parity test), at each
cluster size (including clusters with more CTAs than cells, whose trailing CTAs own none), on
meshes with more (material, width) kinds than a CTA factors ahead of time, and in batches that
mix shapes in one launch.
"""
import os

import numpy as np
import pytest

from oracle import run as oracle_run
from radiant_b200 import workloads as W
from radiant_b200._abi import Context, PackedProblem, ResultBuffers

from test_gpu_parity_1d import TOL, check, rel_l2, small_slab

pytestmark = pytest.mark.gpu


def make_ctx(**env):
    """A context created under the given RB_* settings (read once, when the context is made)."""
    old = {k: os.environ.get(k) for k in env}
    os.environ.update({k: str(v) for k, v in env.items()})
    try:
        return Context(0, 0)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


@pytest.fixture(scope="module")
def teamwide_ctx():
    ctx = make_ctx(RB_LOCAL1D=0)
    yield ctx
    ctx.close()


@pytest.mark.parametrize("solver,order,eorder", [("BTE", 2, 1), ("BFP", 2, 2), ("BFP", 1, 1)])
def test_teamwide_pass(teamwide_ctx, solver, order, eorder):
    check(teamwide_ctx, small_slab(solver=solver, scheme="DG", order=order, escheme="DG", eorder=eorder))


def test_teamwide_c2_photon(teamwide_ctx):
    check(teamwide_ctx, W.c2_tables(seed=2, particle="photon", ng=12))


@pytest.mark.parametrize("cluster", [1, 2, 4, 8, 16])
def test_local_pass_cluster_sizes(cluster):
    ctx = make_ctx(RB_CLUSTER_SIZE=cluster)
    try:
        # 13 cells: not a multiple of the cluster size; on 16 CTAs three own no cell
        check(ctx, small_slab(solver="BFP", scheme="DG", order=2, escheme="DG", eorder=2, nx=13, bc=(1, 0)))
        check(ctx, small_slab(solver="BTE", nx=13, bc=(2, 2), beam=None, volume=1))
    finally:
        ctx.close()


def test_local_pass_many_cell_kinds(gpu_ctx):
    # every cell its own width: more (material, width) kinds per CTA than are factored ahead,
    # so the local sweep solves each cell system as it goes
    rng = np.random.default_rng(5)
    widths = rng.uniform(0.05, 0.15, 40)
    check(gpu_ctx, small_slab(solver="BFP", scheme="DG", order=2, escheme="DG", eorder=2, nx=40, widths=widths))


def test_local_pass_mixed_form_many_kinds(gpu_ctx):
    rng = np.random.default_rng(6)
    t = small_slab(solver="BFP", scheme="DG", order=2, escheme="DG", eorder=2, nx=40,
                   widths=rng.uniform(0.05, 0.15, 40))
    ref = oracle_run.solve(t)
    pp = PackedProblem(dict(t, precision="mixed"))
    rb = ResultBuffers(pp)
    h = gpu_ctx.upload(pp)
    gpu_ctx.solve(h)
    gpu_ctx.download(h, rb)
    gpu_ctx.release(h)
    assert rel_l2(rb.flux, ref.flux) <= 1e-5


def test_batch_of_mixed_shapes(gpu_ctx):
    # BTE and BFP problems of different sizes in one launch: one persistent kernel, one team
    # per problem at a time, each result equal to the oracle's
    tabs = [small_slab(solver="BTE", nx=30, seed=7),
            small_slab(solver="BFP", scheme="DG", order=2, escheme="DG", eorder=2, nx=50, seed=8),
            W.c2_tables(seed=3, particle="photon", ng=10),
            small_slab(solver="BFP", nx=7, seed=9)]
    packs = [PackedProblem(t) for t in tabs]
    bufs = [ResultBuffers(p) for p in packs]
    hs = [gpu_ctx.upload(p) for p in packs]
    gpu_ctx.solve_batch(hs)
    for t, h, rb in zip(tabs, hs, bufs):
        gpu_ctx.download(h, rb)
        gpu_ctx.release(h)
        ref = oracle_run.solve(t)
        assert rel_l2(rb.flux, ref.flux) <= TOL
        assert rb.passes == ref.passes


@pytest.mark.gpu
@pytest.mark.parametrize("cluster", [2, 16])
def test_launch_rules_set_the_team_and_keep_parity(cluster):
    """rb_set_launch_rules: a batch covered by a rule runs with the rule's team size, and the
    results still match the oracle within the parity tolerance."""
    from oracle import run as orun
    from radiant_b200._abi import Context, PackedProblem, ResultBuffers
    from radiant_b200.autotune import work_of
    batch = [W.c1_tables(seed=s) for s in (1, 2)]
    ctx = Context(0, 0, launch_rules=[{"ndims": 1, "nd_max": 64, "work_max": int(max(work_of(t) for t in batch)) + 1,
                                       "batch_max": 8, "cluster": cluster}])
    pps = [PackedProblem(t) for t in batch]
    hs = [ctx.upload(p) for p in pps]
    ctx.solve_batch(hs)
    for h, p, t in zip(hs, pps, batch):
        rb = ResultBuffers(p)
        ctx.download(h, rb)
        ref = orun.solve(t)
        assert np.linalg.norm(rb.flux - ref.flux) / np.linalg.norm(ref.flux) <= 1e-10
        assert rb.passes == ref.passes
    ctx.close()
