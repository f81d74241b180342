"""GPU parity, 1D: the CUDA library against the oracle on the same seeded inputs.

Tolerance: the FP64 form must match within 1e-10 relative L2 on the flux moments and the
cutoff flux (the acceptance limit of the plain form); pass counts must be identical.
"""
import numpy as np
import pytest

from oracle import run as oracle_run
from radiant_b200 import workloads as W
from radiant_b200._abi import PackedProblem, ResultBuffers
from radiant_b200.sn_flux import SNSettings

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel_l2(a, b):
    a = np.asarray(a).ravel(); b = np.asarray(b).ravel()
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def gpu_solve(ctx, tabs):
    pp = PackedProblem(tabs)
    rb = ResultBuffers(pp)
    h = ctx.upload(pp)
    ctx.solve(h)
    ctx.download(h, rb)
    ctx.release(h)
    return rb


def check(ctx, tabs, tol=TOL):
    ref = oracle_run.solve(tabs)
    got = gpu_solve(ctx, tabs)
    e = rel_l2(got.flux, ref.flux)
    assert e <= tol, f"flux rel L2 {e:.3e}"
    if ref.flux_cutoff is not None:
        ec = rel_l2(got.flux_cutoff, ref.flux_cutoff)
        assert ec <= tol, f"cutoff rel L2 {ec:.3e}"
    assert got.passes == ref.passes, (got.passes, ref.passes)
    np.testing.assert_array_equal(got.group_iters, ref.group_iters)
    return ref, got


def small_slab(solver="BTE", accel="gmres", order=1, scheme="DD", eorder=1, escheme="DD", nx=24, ng=5,
               N=8, L=3, bc=(0, 0), boltz="galerkin-d", afp="galerkin", fc=True, seed=3, volume=None,
               beam=0, widths=None, mats=None, nmat=2):
    st = {"x": scheme}
    so = {"x": order}
    if solver != "BTE":
        st["E"] = escheme
        so["E"] = eorder
    sn = SNSettings(solver_type=solver, quadrature_type="gauss-legendre", quadrature_order=N, legendre_order=L,
                    scheme_type=st, scheme_order=so, acceleration=accel, convergence_criterion=1e-9,
                    angular_boltzmann=boltz, angular_fokker_planck=afp, is_full_coupling=fc, maximum_iteration=400)
    if mats is None:
        mats = np.ones(nx, dtype=np.int32)
        mats[nx // 3: 2 * nx // 3] = 2 if nmat > 1 else 1
    widths = np.full(nx, 0.1) if widths is None else widths
    return W.slab_tables(nx, widths, mats, ng, nmat, seed, sn, L, beam_group=beam, bc=bc,
                         volume_group=volume, csd=(solver != "BTE"))


@pytest.mark.parametrize("accel", ["none", "livolant", "anderson", "gmres", "bicgstab"])
def test_bte_dd_accels(gpu_ctx, accel):
    check(gpu_ctx, small_slab(accel=accel))


@pytest.mark.parametrize("scheme,order", [("DD", 2), ("DG", 2), ("DG", 3), ("DG-", 2), ("DD", 3)])
def test_bte_high_order(gpu_ctx, scheme, order):
    check(gpu_ctx, small_slab(scheme=scheme, order=order))


@pytest.mark.parametrize("bc", [(1, 0), (0, 1), (1, 1), (2, 2)])
def test_bte_boundaries(gpu_ctx, bc):
    check(gpu_ctx, small_slab(bc=bc, volume=0, beam=None))


@pytest.mark.parametrize("boltz", ["standard", "galerkin-m", "galerkin-d"])
def test_bte_bases(gpu_ctx, boltz):
    check(gpu_ctx, small_slab(boltz=boltz, N=9))  # odd N: a tangential direction μ = 0


@pytest.mark.parametrize("accel", ["gmres", "livolant", "bicgstab"])
@pytest.mark.parametrize("orders", [(1, 1), (2, 2), (2, 1), (1, 2)])
def test_bfp(gpu_ctx, accel, orders):
    check(gpu_ctx, small_slab(solver="BFP", accel=accel, scheme="DG", order=orders[0], escheme="DG",
                              eorder=orders[1]))


@pytest.mark.parametrize("solver", ["BCSD", "FP", "CSD", "BFP-EF"])
def test_csd_family(gpu_ctx, solver):
    check(gpu_ctx, small_slab(solver=solver, scheme="DD", order=1, escheme="DD", eorder=1))


def test_bfp_not_fully_coupled(gpu_ctx):
    check(gpu_ctx, small_slab(solver="BFP", scheme="DG", order=2, escheme="DG", eorder=2, fc=False))


def test_bfp_finite_difference_fp(gpu_ctx):
    check(gpu_ctx, small_slab(solver="BFP", afp="finite-difference", scheme="DD", order=1))


def test_zero_source(gpu_ctx):
    t = small_slab(beam=None)
    ref, got = check(gpu_ctx, t)
    assert np.all(got.flux == 0.0) and got.passes == 0


def test_single_cell(gpu_ctx):
    check(gpu_ctx, small_slab(nx=1, mats=np.ones(1, dtype=np.int32), nmat=1))


def test_c1_config(gpu_ctx):
    check(gpu_ctx, W.c1_tables(seed=1))


def test_c2_electron_config(gpu_ctx):
    check(gpu_ctx, W.c2_tables(seed=1))
