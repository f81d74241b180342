"""Serving on the GPU: requests admitted while others run overlap on the device, and each
result is the same alone and in the mix (bit for bit: reductions do not depend on what shares
the device), and within the FP64 tolerance of the oracle."""
import numpy as np
import pytest

from oracle import run as oracle_run
from radiant_b200 import serving as S
from radiant_b200 import workloads as W
from radiant_b200._abi import RB_ERR_BUDGET, Context, PackedProblem, RadiantError, ResultBuffers
from radiant_b200.sn_flux import SNSettings

pytestmark = pytest.mark.gpu


def mix():
    out = []
    for seed in range(6):
        t = W.random_slab_tables(seed, max_cells=300, max_groups=12)
        out.append(t)
    sn = SNSettings(solver_type="BTE", quadrature_type="carlson", quadrature_order=4, legendre_order=2,
                    scheme_type={"x": "DD", "y": "DD"}, scheme_order={"x": 1, "y": 1}, acceleration="gmres",
                    convergence_criterion=1e-9, angular_boltzmann="standard")
    mats = np.ones((8, 6), dtype=np.int32)
    out.append(W.grid_tables(2, [8, 6], [np.full(8, 0.3), np.full(6, 0.3)], mats, 3, 1, 5, sn, 2,
                             beam=("X-", 0, (0.8, 0.6, 0.0), {1: (0.0, 2.0)})))
    return out


def test_same_alone_and_in_the_mix():
    ctx = Context(0, 0)
    tabs = mix()
    alone = []
    for t in tabs:  # one request at a time
        req = S.Request(0, t, 0.0)
        S.ServingLoop(ctx).run([req])
        alone.append(req.result)
    reqs = [S.Request(i, t, 0.0) for i, t in enumerate(tabs)]  # all at once
    S.ServingLoop(ctx).run(reqs)
    for a, r, t in zip(alone, reqs, tabs):
        assert np.array_equal(a.flux, r.result.flux)
        assert a.passes == r.result.passes
        ref = oracle_run.solve(t)
        assert np.linalg.norm(r.result.flux - ref.flux) <= 1e-10 * np.linalg.norm(ref.flux)
    ctx.close()


def test_budget_refusal_then_admission():
    tabs = mix()[:2]
    import ctypes as C
    from radiant_b200._abi import load_library
    lib = load_library()
    sizes = []
    for t in tabs:
        b = C.c_uint64()
        assert lib.rb_required_bytes(C.byref(PackedProblem(t).P), C.byref(b)) == 0
        sizes.append(b.value)
    ctx = Context(0, max(sizes) + 1024)  # room for one request at a time
    p0, p1 = PackedProblem(tabs[0]), PackedProblem(tabs[1])
    h0 = ctx.submit(p0)
    with pytest.raises(RadiantError) as e:
        ctx.submit(p1)
    assert e.value.status == RB_ERR_BUDGET
    r0 = ResultBuffers(p0)
    while not ctx.poll(h0, r0):
        pass
    h1 = ctx.submit(p1)  # memory freed: admitted now
    r1 = ResultBuffers(p1)
    while not ctx.poll(h1, r1):
        pass
    assert r0.passes > 0 and r1.passes > 0
    ctx.close()
