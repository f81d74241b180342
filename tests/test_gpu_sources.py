"""Fixed sources built on the device (rb_upload_sources) against the dense host arrays of the
same Volume_Source / Surface_Source definitions (volume_source.jl:21-122, surface_source.jl:
22-330, Source.add_source): the solve gives the same bits, the normalization factors are the
same numbers, and the dense path itself is within 1e-10 of the oracle. 1D, 2D and 3D, with
overlapping boxes in several groups and several beams on one face.
"""
import math

import numpy as np
import pytest

from oracle import run as oracle_run
from radiant_b200 import sources as S
from radiant_b200 import workloads as W
from radiant_b200._abi import RB_ERR_INVALID, Context, PackedProblem, RadiantError, ResultBuffers
from radiant_b200.sn_flux import SNSettings, prepare_sn_tables

pytestmark = pytest.mark.gpu


def _unit(v):
    v = np.asarray(v, dtype=float)
    return tuple(v / np.linalg.norm(v))


def build(ndims, ns, sn, ng, volume, surface, seed=3, csd=False, bc=None):
    """(dense tables, tables without sources, SourceSet, normalization factors)."""
    nmat = 2
    xs = W.synthetic_xs(ng, nmat, sn.legendre_order, seed, csd=csd)
    ds = [np.linspace(0.15, 0.35, n) for n in ns]
    pos = [S.positions_of(d) for d in ds]
    rng = np.random.default_rng(seed)
    full = list(ns) + [1] * (3 - ndims)
    mats = rng.integers(1, nmat + 1, size=full).astype(np.int32)
    bc = bc or [0] * (2 * ndims)
    vol, surf, norms = S.dense_sources(sn, ndims, ng, ns, ds, pos, volume, surface)
    dense = prepare_sn_tables(xs, ndims, ns, ds, mats, bc, sn, volume_sources=vol, surface_sources=surf)
    bare = prepare_sn_tables(xs, ndims, ns, ds, mats, bc, sn)
    sset = S.SourceSet(sn, ndims, pos, volume, surface, np_surf=bare["np_surf"])
    bare["np_source"] = sset.np_source
    assert sset.np_source == dense["np_source"]
    return dense, bare, sset, norms


def _sn(ndims, solver="BTE", quad="carlson", order=4, L=3, btype="galerkin-d"):
    axes = "xyz"[:ndims]
    st = {a: "DD" for a in axes}
    so = {a: 1 for a in axes}
    if solver != "BTE":
        st["E"], so["E"] = "DD", 1
    return SNSettings(solver_type=solver, quadrature_type=quad, quadrature_order=order, legendre_order=L,
                      scheme_type=st, scheme_order=so, acceleration="gmres", convergence_criterion=1e-11,
                      angular_boltzmann=btype, angular_fokker_planck="galerkin")


CASES = {
    "1d": dict(ndims=1, ns=[40], sn=_sn(1, quad="gauss-legendre", order=16, L=5, btype="standard"), ng=4,
               volume=[S.VolumeSource(2, {"x": (1.0, 4.0)}, 2.0), S.VolumeSource(2, {"x": (3.0, 9.0)}, 0.5),
                       S.VolumeSource(4, {"x": (0.0, 2.0)}, 1.0)],
               surface=[S.SurfaceSource(1, "X-", (0.9, 0.0, 0.0), intensity=1.3),
                        S.SurfaceSource(1, "X-", (0.3, 0.0, 0.0), legendre_order=2),
                        S.SurfaceSource(3, "X+", (-0.7, 0.0, 0.0), intensity=0.4)]),
    "2d": dict(ndims=2, ns=[14, 11], sn=_sn(2), ng=3,
               volume=[S.VolumeSource(1, {"x": (0.5, 2.0), "y": (0.5, 1.5)}, 1.5),
                       S.VolumeSource(1, {"x": (1.0, 3.0), "y": (0.0, 1.0)}, 0.7)],
               surface=[S.SurfaceSource(1, "X-", _unit((0.8, 0.4, 0.2)), {"y": (0.3, 1.6)}, 1.1),
                        S.SurfaceSource(2, "Y-", _unit((0.3, 0.9, -0.2)), {"x": (0.0, 2.0)}),
                        S.SurfaceSource(2, "Y-", _unit((-0.3, 0.9, 0.1)), {"x": (1.0, 3.5)}, 0.6),
                        S.SurfaceSource(1, "X+", _unit((0.8, 0.4, 0.2)), {"y": (0.0, 9.0)})]),  # leaves
    "3d_bfp": dict(ndims=3, ns=[7, 6, 5], sn=_sn(3, solver="BFP"), ng=3, csd=True, bc=[0, 0, 0, 0, 1, 0],
                   volume=[S.VolumeSource(1, {"x": (0.3, 1.0), "y": (0.2, 0.9), "z": (0.0, 0.6)}, 1.0),
                           S.VolumeSource(2, {"x": (0.0, 9.0), "y": (0.0, 9.0), "z": (0.0, 9.0)}, 0.01)],
                   surface=[S.SurfaceSource(1, "Z+", _unit((0.2, 0.3, -0.9)), {"x": (0.2, 1.2), "y": (0.3, 1.0)}),
                            S.SurfaceSource(1, "Z+", _unit((-0.2, 0.1, -0.95)), {"x": (0.0, 0.8), "y": (0.0, 1.5)},
                                            0.5),
                            S.SurfaceSource(3, "X-", _unit((0.7, 0.5, 0.5)), {"y": (0.0, 1.0), "z": (0.2, 0.9)})]),
}


@pytest.fixture(scope="module")
def ctx():
    c = Context(0, 0)
    yield c
    c.close()


def _solve(ctx, h, pp):
    rb = ResultBuffers(pp)
    ctx.solve(h)
    ctx.download(h, rb)
    ctx.release(h)
    return rb


@pytest.mark.parametrize("name", list(CASES))
def test_device_sources_give_the_dense_bits(ctx, name):
    case = dict(CASES[name])
    dense, bare, sset, norms = build(case.pop("ndims"), case.pop("ns"), case.pop("sn"), case.pop("ng"),
                                     case.pop("volume"), case.pop("surface"), csd=case.pop("csd", False),
                                     bc=case.pop("bc", None))
    pd = PackedProblem(dense)
    a = _solve(ctx, ctx.upload(pd), pd)
    pb = PackedProblem(bare)
    h, got_norms = ctx.upload_sources(pb, sset)
    b = _solve(ctx, h, pb)
    assert np.array_equal(a.flux, b.flux)
    if a.flux_cutoff is not None:
        assert np.array_equal(a.flux_cutoff, b.flux_cutoff)
    assert a.passes == b.passes
    assert np.array_equal(got_norms, np.asarray(norms))
    assert np.abs(a.flux).max() > 0
    ref = oracle_run.solve(dense)
    e = np.linalg.norm(a.flux - ref.flux) / np.linalg.norm(ref.flux)
    assert e <= 1e-10, e


def test_rejections(ctx):
    case = CASES["2d"]
    dense, bare, sset, _ = build(2, case["ns"], case["sn"], case["ng"], case["volume"], case["surface"])
    with pytest.raises(RadiantError) as ei:
        ctx.upload_sources(PackedProblem(dense), sset)  # dense arrays and definitions together
    assert ei.value.status == RB_ERR_INVALID
    bad = S.SourceSet(case["sn"], 2, sset.positions, [S.VolumeSource(9, {})], [])
    with pytest.raises(RadiantError) as ei:
        ctx.upload_sources(PackedProblem(bare), bad)  # group beyond ng
    assert ei.value.status == RB_ERR_INVALID and "energy group" in str(ei.value)
    beam = S.SurfaceSource(1, "X-", _unit((0.8, 0.4, 0.2)))
    bad = S.SourceSet(case["sn"], 2, sset.positions, [], [beam], np_surf=bare["np_surf"])
    bad.beams[0].face = 4  # Z- on a 2D grid
    with pytest.raises(RadiantError) as ei:
        ctx.upload_sources(PackedProblem(bare), bad)
    assert ei.value.status == RB_ERR_INVALID and "face" in str(ei.value)
    t0 = dict(bare)
    t0["np_source"] = 0
    with pytest.raises(RadiantError) as ei:
        ctx.upload_sources(PackedProblem(t0), sset)  # beams but no surface moments read
    assert ei.value.status == RB_ERR_INVALID
