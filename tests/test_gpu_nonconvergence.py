"""GPU behaviour when a group does not converge within max_iter.

The reference prints "has not converged" and goes on with the next group
(sn_one_speed.jl:189-193); the library does the same: the solve completes, the group's converged
flag is 0, and the flux is the iterate the accelerator stopped at — the oracle's iterate, within
the FP64 parity tolerance and with the same pass count. The failure is made on the host (a tiny
iteration budget); nothing waits or faults on the device.
"""
import numpy as np
import pytest

from oracle import run as oracle_run
from radiant_b200 import workloads as W
from radiant_b200.sn_flux import SNSettings

from test_gpu_parity_1d import TOL, gpu_solve, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("accel", ["none", "livolant", "gmres", "bicgstab"])
def test_group_hits_max_iter(gpu_ctx, accel):
    sn = SNSettings(solver_type="BFP", quadrature_type="gauss-legendre", quadrature_order=8, legendre_order=3,
                    scheme_type={"x": "DG", "E": "DG"}, scheme_order={"x": 2, "E": 2}, acceleration=accel,
                    convergence_criterion=1e-12, maximum_iteration=3, angular_fokker_planck="galerkin")
    nx = 20
    mats = np.ones(nx, dtype=np.int32)
    mats[7:14] = 2
    t = W.slab_tables(nx, np.full(nx, 0.1), mats, 4, 2, 11, sn, 3, beam_group=0, csd=True)
    ref = oracle_run.solve(t)
    got = gpu_solve(gpu_ctx, t)
    assert not np.asarray(got.group_converged).all()
    np.testing.assert_array_equal(got.group_converged, ref.group_converged)
    assert rel_l2(got.flux, ref.flux) <= TOL
    assert got.passes == ref.passes
