"""GPU parity, 2D and 3D: the CUDA library (wavefront sweeps, grid and cluster teams) against
the oracle on the same seeded inputs. FP64 tolerance 1e-10 relative L2; identical pass counts."""
import os

import numpy as np
import pytest

from oracle import run as oracle_run
from radiant_b200 import workloads as W
from radiant_b200._abi import Context, PackedProblem, ResultBuffers
from radiant_b200.sn_flux import SNSettings

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel_l2(a, b):
    a = np.asarray(a).ravel(); b = np.asarray(b).ravel()
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


@pytest.fixture(scope="module", params=["grid", "cluster"])
def md_ctx(request):
    old = os.environ.get("RB_MD_TEAM")
    os.environ["RB_MD_TEAM"] = request.param
    ctx = Context(0, 0)
    if old is None:
        del os.environ["RB_MD_TEAM"]
    else:
        os.environ["RB_MD_TEAM"] = old
    yield ctx
    ctx.close()


def check(ctx, tabs, tol=TOL):
    ref = oracle_run.solve(tabs)
    pp = PackedProblem(tabs)
    got = ResultBuffers(pp)
    h = ctx.upload(pp)
    ctx.solve(h)
    ctx.download(h, got)
    ctx.release(h)
    e = rel_l2(got.flux, ref.flux)
    assert e <= tol, f"flux rel L2 {e:.3e}"
    if ref.flux_cutoff is not None:
        assert rel_l2(got.flux_cutoff, ref.flux_cutoff) <= tol
    assert got.passes == ref.passes, (got.passes, ref.passes)
    np.testing.assert_array_equal(got.group_iters, ref.group_iters)
    return ref, got


def sn2(solver="BTE", accel="gmres", order=1, boltz="standard", N=4, L=2, fc=True, orderE=1):
    st, so = {"x": "DD", "y": "DD", "z": "DD"}, {"x": order, "y": order, "z": order}
    if solver != "BTE":
        st["E"] = "DD"
        so["E"] = orderE
    return SNSettings(solver_type=solver, quadrature_type="carlson", quadrature_order=N, legendre_order=L,
                      scheme_type=st, scheme_order=so, acceleration=accel, convergence_criterion=1e-9,
                      angular_boltzmann=boltz, angular_fokker_planck="galerkin", is_full_coupling=fc,
                      maximum_iteration=400)


def grid2d(sn, nx=6, ny=5, bc=(0, 0, 0, 0, 0, 0), beam=True, volume=False, ng=4, csd=False, seed=7):
    mats = np.ones((nx, ny), dtype=np.int32)
    mats[2:4, 1:3] = 2
    b = ("X-", 0, (0.8, 0.6, 0.0), {1: (0.2, 0.8)}) if beam else None
    v = (0, {0: (0.0, 0.4), 1: (0.0, 0.5)}) if volume else None
    return W.grid_tables(2, [nx, ny], [np.full(nx, 0.2), np.full(ny, 0.2)], mats, ng, 2, seed, sn, sn.legendre_order,
                         beam=b, volume=v, bc=bc, csd=csd)


def grid3d(sn, n=(4, 3, 3), bc=(0, 0, 0, 0, 1, 0), ng=3, csd=False, seed=9):
    mats = np.ones(n, dtype=np.int32)
    mats[1:3, 1, 1] = 2
    v = (0, {0: (0.0, 0.5), 1: (0.0, 0.5), 2: (0.0, 0.5)})
    return W.grid_tables(3, list(n), [np.full(k, 0.25) for k in n], mats, ng, 2, seed, sn, sn.legendre_order,
                         volume=v, bc=bc, csd=csd)


@pytest.mark.parametrize("accel", ["gmres", "bicgstab", "livolant"])
def test_2d_beam(md_ctx, accel):
    check(md_ctx, grid2d(sn2(accel=accel)))


@pytest.mark.parametrize("bc", [(1, 0, 0, 0, 0, 0), (1, 1, 1, 1, 0, 0), (2, 2, 0, 0, 0, 0), (0, 0, 2, 2, 0, 0)])
def test_2d_boundaries(md_ctx, bc):
    check(md_ctx, grid2d(sn2(), bc=bc, beam=False, volume=True))


def test_2d_galerkin_basis(md_ctx):
    check(md_ctx, grid2d(sn2(boltz="galerkin-d", N=4)))


def test_2d_high_order_full_coupling(md_ctx):
    check(md_ctx, grid2d(sn2(order=2)))


def test_2d_high_order_partial_coupling(md_ctx):
    check(md_ctx, grid2d(sn2(order=2, fc=False)))


def test_2d_bfp(md_ctx):
    check(md_ctx, grid2d(sn2(solver="BFP"), csd=True))


def test_2d_rows_beyond_threads(md_ctx):
    check(md_ctx, grid2d(sn2(accel="gmres"), nx=3, ny=300, ng=2))


@pytest.mark.parametrize("accel", ["gmres", "bicgstab"])
def test_3d_reflective_z(md_ctx, accel):
    check(md_ctx, grid3d(sn2(accel=accel)))


def test_3d_bfp_periodic(md_ctx):
    check(md_ctx, grid3d(sn2(solver="BFP"), bc=(2, 2, 0, 0, 0, 0), csd=True))


# ---- the configurations' own shapes -------------------------------------------------------
# 128² with level-symmetric S12 and the Galerkin-d basis (168 directions, 168 moments), and 64³
# with S8 (80 directions, 80 moments), BiCGStab and a reflective Z- face: the sizes at which the
# product tiles, the octant tiles of the 3D sweep and the 2D wavefront run in the benchmark.
# The grid team only (one problem on the whole GPU); fewer groups than the configurations.

@pytest.fixture(scope="module")
def grid_ctx():
    ctx = Context(0, 0)
    yield ctx
    ctx.close()


def test_c3_shape_fp64(grid_ctx):
    tabs = W.c3_tables(1, "photon", ng=2)
    assert tabs["nd"] == 168 and tabs["np"] == 168 and tabs["ns"][:2] == [128, 128]
    check(grid_ctx, tabs)


def test_c4_shape_fp64(grid_ctx):
    tabs = W.c4_tables(1, "photon", ng=1)
    assert tabs["nd"] == 80 and tabs["np"] == 80 and tabs["ns"] == [64, 64, 64] and tabs["bc"][4] == 1
    assert tabs["accel"] == "bicgstab"
    check(grid_ctx, tabs)


# ---- the mixed form in 2D and 3D: FP32 sweeps and products, FP64 Krylov and defect correction;
# contract 1e-5 relative L2 against the FP64 oracle
MIXED_TOL = 1e-5


def check_mixed(ctx, tabs, tol=MIXED_TOL):
    ref = oracle_run.solve(tabs)
    t2 = dict(tabs)
    t2["precision"] = "mixed"
    pp = PackedProblem(t2)
    got = ResultBuffers(pp)
    h = ctx.upload(pp)
    ctx.solve(h)
    ctx.download(h, got)
    ctx.release(h)
    e = rel_l2(got.flux, ref.flux)
    assert e <= tol, f"mixed flux rel L2 {e:.3e}"
    if ref.flux_cutoff is not None:
        ec = rel_l2(got.flux_cutoff, ref.flux_cutoff)
        assert ec <= tol, f"mixed cutoff rel L2 {ec:.3e}"
    assert np.all(got.group_converged == 1)
    return e


@pytest.mark.parametrize("accel", ["gmres", "bicgstab"])
def test_2d_mixed(md_ctx, accel):
    check_mixed(md_ctx, grid2d(sn2(accel=accel, boltz="galerkin-d")))


def test_2d_bfp_mixed(md_ctx):
    check_mixed(md_ctx, grid2d(sn2(solver="BFP"), csd=True))


@pytest.mark.parametrize("accel", ["gmres", "bicgstab"])
def test_3d_mixed(md_ctx, accel):
    check_mixed(md_ctx, grid3d(sn2(accel=accel)))


def test_3d_bfp_mixed(md_ctx):
    check_mixed(md_ctx, grid3d(sn2(solver="BFP"), bc=(2, 2, 0, 0, 0, 0), csd=True))


def test_2d_high_order_mixed_runs_fp64(md_ctx):
    """Order-2 cells have no FP32 sweep: their mixed-form passes run in FP64."""
    check_mixed(md_ctx, grid2d(sn2(order=2)))


def test_c3_shape_mixed(grid_ctx):
    check_mixed(grid_ctx, W.c3_tables(1, "photon", ng=2))


def test_c4_shape_mixed(grid_ctx):
    check_mixed(grid_ctx, W.c4_tables(1, "photon", ng=1))



def _sn_fd(N=4, L=2):
    """The reference's default angular Fokker-Planck ("finite-difference") on the product
    Gauss-Legendre-Chebychev quadrature."""
    return SNSettings(solver_type="BFP", quadrature_type="gauss-legendre-chebychev", quadrature_order=N,
                      legendre_order=L, scheme_type={"x": "DD", "y": "DD", "z": "DD", "E": "DD"},
                      scheme_order={"x": 1, "y": 1, "z": 1, "E": 1}, acceleration="gmres",
                      convergence_criterion=1e-9, angular_boltzmann="standard", maximum_iteration=400)


def test_2d_bfp_finite_difference_fokker_planck(md_ctx):
    check(md_ctx, grid2d(_sn_fd(), csd=True))


def test_3d_bfp_finite_difference_fokker_planck(md_ctx):
    check(md_ctx, grid3d(_sn_fd(), csd=True))
