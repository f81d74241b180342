"""rb_compute_flux_static: the solve without device allocation, checked against rb_compute_flux.

Callers that cannot call cudaMalloc (a process whose GPU memory is held by another allocator's
pool, which cudaMalloc/cudaFree would synchronise and fragment) use this entry point; its
device memory is one static 16 MiB array. Two different problems are solved in a row through
it, each compared with the allocating entry point within the FP64 tolerance of the parity
tests (1e-10 relative L2), so the array's left-over contents from the first call must not
leak into the second. This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

from radiant_b200 import workloads as W
from radiant_b200._abi import PackedProblem, ResultBuffers, RbSnProblem, RbSnResult, load_library
from radiant_b200.sn_flux import SNSettings

pytestmark = pytest.mark.gpu
TOL = 1e-10
RB_ERR_BUDGET = 4


def rel_l2(a, b):
    a = np.asarray(a).ravel(); b = np.asarray(b).ravel()
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def _lib():
    lib = load_library()
    fn = lib.rb_compute_flux_static
    fn.argtypes = [C.POINTER(RbSnProblem), C.POINTER(RbSnResult), C.c_void_p]
    fn.restype = C.c_int32
    return lib


def _bfp_slab():
    sn = SNSettings(solver_type="BFP", quadrature_type="gauss-legendre", quadrature_order=8, legendre_order=3,
                    scheme_type={"x": "DG", "E": "DG"}, scheme_order={"x": 2, "E": 2},
                    angular_fokker_planck="galerkin", acceleration="gmres", convergence_criterion=1e-9)
    nx = 40
    mats = np.ones(nx, dtype=np.int32)
    mats[10:20] = 2
    return W.slab_tables(nx, np.full(nx, 0.1), mats, 12, 2, 11, sn, 3, beam_group=0, csd=True)


def test_static_entry_matches_allocating_entry_twice():
    lib = _lib()
    for tabs in (W.c1_tables(seed=1), _bfp_slab()):
        pp = PackedProblem(tabs)
        ref = ResultBuffers(pp)
        assert lib.rb_compute_flux(0, C.byref(pp.P), C.byref(ref.R)) == 0
        got = ResultBuffers(pp)
        st = lib.rb_compute_flux_static(C.byref(pp.P), C.byref(got.R), None)
        assert st == 0, st
        assert rel_l2(got.flux, ref.flux) <= TOL
        if ref.flux_cutoff is not None:
            assert rel_l2(got.flux_cutoff, ref.flux_cutoff) <= TOL
        assert got.passes == ref.passes
        np.testing.assert_array_equal(got.group_iters, ref.group_iters)


def _grid2d():
    sn = SNSettings(solver_type="BTE", quadrature_type="carlson", quadrature_order=4, legendre_order=2,
                    scheme_type={"x": "DD", "y": "DD"}, scheme_order={"x": 1, "y": 1}, acceleration="gmres",
                    convergence_criterion=1e-9)
    nx, ny = 12, 10
    mats = np.ones((nx, ny), dtype=np.int32)
    mats[3:6, 2:5] = 2
    return W.grid_tables(2, [nx, ny], [np.full(nx, 0.2), np.full(ny, 0.25)], mats, 4, 2, 5, sn, 2,
                         beam=("X-", 0, (0.8, 0.6, 0.0), {1: (0.5, 2.0)}), bc=(0, 0, 1, 0, 0, 0))


def _grid3d_bfp():
    sn = SNSettings(solver_type="BFP", quadrature_type="carlson", quadrature_order=4, legendre_order=2,
                    scheme_type={"x": "DD", "y": "DD", "z": "DD", "E": "DD"},
                    scheme_order={"x": 1, "y": 1, "z": 1, "E": 1}, angular_fokker_planck="galerkin",
                    acceleration="bicgstab", convergence_criterion=1e-9)
    n = [6, 5, 4]
    mats = np.ones(n, dtype=np.int32)
    mats[2:4, 1:3, 1:3] = 2
    v = (0, {0: (0.0, 0.75), 1: (0.0, 0.75), 2: (0.0, 0.75)})
    return W.grid_tables(3, n, [np.full(k, 0.25) for k in n], mats, 3, 2, 9, sn, 2, volume=v,
                         bc=(0, 0, 0, 0, 1, 0), csd=True)


def test_static_entry_2d_and_3d_match_allocating_entry():
    """The 2D wavefront and the 3D octant sweep on the static entry's one-CTA team, against the
    allocating entry (whose 2D/3D problems take the whole GPU), two calls in a row."""
    lib = _lib()
    for tabs in (_grid2d(), _grid3d_bfp()):
        pp = PackedProblem(tabs)
        ref = ResultBuffers(pp)
        assert lib.rb_compute_flux(0, C.byref(pp.P), C.byref(ref.R)) == 0
        got = ResultBuffers(pp)
        assert lib.rb_compute_flux_static(C.byref(pp.P), C.byref(got.R), None) == 0
        assert rel_l2(got.flux, ref.flux) <= TOL
        if ref.flux_cutoff is not None:
            assert rel_l2(got.flux_cutoff, ref.flux_cutoff) <= TOL
        assert got.passes == ref.passes


def test_static_entry_rejects_oversized_problem():
    lib = _lib()
    pp = PackedProblem(W.c2_tables(seed=1))  # ~55 MiB of device memory
    got = ResultBuffers(pp)
    assert lib.rb_compute_flux_static(C.byref(pp.P), C.byref(got.R), None) == RB_ERR_BUDGET
    buf = C.create_string_buffer(512)
    lib.rb_last_error(None, buf, 512)
    assert b"static scratch" in buf.value
