"""Page-locked host buffers (rb_host_alloc / rb_host_free / rb_host_register / rb_host_unregister).

A problem uploaded from page-locked tables and downloaded into page-locked results gives the
bits of the same problem through pageable numpy arrays; an existing array registered in place
serves as a result buffer; the calls reject null pointers and zero sizes with RB_ERR_INVALID.
"""
import ctypes as C

import numpy as np
import pytest

from radiant_b200 import _abi
from radiant_b200 import workloads as W
from radiant_b200._abi import RB_ERR_INVALID, RB_OK, Context, PackedProblem, ResultBuffers, load_library

pytestmark = pytest.mark.gpu


def _solve(ctx, pp, rb, stream=None):
    h = ctx.upload(pp)
    ctx.solve(h, stream)
    ctx.download(h, rb)
    ctx.release(h)
    return rb


def _is_pinned_array(a):
    """cudaPointerGetAttributes: page-locked host memory reads as cudaMemoryTypeHost."""
    from cuda.bindings import runtime as rt
    err, attr = rt.cudaPointerGetAttributes(a.ctypes.data)
    return err == rt.cudaError_t.cudaSuccess and attr.type == rt.cudaMemoryType.cudaMemoryTypeHost


@pytest.mark.parametrize("make", [lambda: W.c1_tables(seed=4),
                                  lambda: W.c4_tables(seed=2, particle="electron", n=16, ng=3)])
def test_pinned_buffers_give_the_same_bits(monkeypatch, make):
    monkeypatch.setattr(_abi, "PINNED_MIN_BYTES", 0)  # every array of the problem page-locked
    tabs = make()
    ctx = Context(0, 0)
    try:
        ref = _solve(ctx, PackedProblem(tabs), ResultBuffers(PackedProblem(tabs)))
        pp = PackedProblem(tabs, pinned=True)
        rb = ResultBuffers(pp, pinned=True)
        assert _is_pinned_array(pp.t["sigma_t"]) and _is_pinned_array(rb.flux)
        got = _solve(ctx, pp, rb)
        assert np.array_equal(got.flux, ref.flux)
        if ref.flux_cutoff is not None:
            assert np.array_equal(got.flux_cutoff, ref.flux_cutoff)
        assert got.passes == ref.passes and np.array_equal(got.group_iters, ref.group_iters)
    finally:
        ctx.close()


def test_registered_result_buffer():
    lib = load_library()
    tabs = W.c1_tables(seed=5)
    ctx = Context(0, 0)
    try:
        ref = _solve(ctx, PackedProblem(tabs), ResultBuffers(PackedProblem(tabs)))
        pp = PackedProblem(tabs)
        rb = ResultBuffers(pp)
        assert lib.rb_host_register(rb.flux.ctypes.data, rb.flux.nbytes) == RB_OK
        try:
            got = _solve(ctx, pp, rb)
        finally:
            assert lib.rb_host_unregister(rb.flux.ctypes.data) == RB_OK
        assert np.array_equal(got.flux, ref.flux)
    finally:
        ctx.close()


def test_host_calls_reject_bad_arguments():
    lib = load_library()
    p = C.c_void_p()
    assert lib.rb_host_alloc(0, C.byref(p)) == RB_ERR_INVALID
    assert lib.rb_host_alloc(64, None) == RB_ERR_INVALID
    assert lib.rb_host_register(None, 64) == RB_ERR_INVALID
    assert lib.rb_host_unregister(None) == RB_ERR_INVALID
    assert lib.rb_host_free(None) == RB_OK
    assert lib.rb_host_alloc(4096, C.byref(p)) == RB_OK and p.value
    C.memset(p.value, 0, 4096)
    assert lib.rb_host_free(p.value) == RB_OK


def test_pinned_empty_lifetime():
    a = _abi.pinned_empty((3, 5, 7))
    assert a.flags["F_CONTIGUOUS"] and a.shape == (3, 5, 7) and a.dtype == np.float64
    a[...] = 1.5
    v = a[1]
    del a
    assert float(v.sum()) == 1.5 * 35  # the view keeps the page-locked block alive


def test_download_async_overlaps_the_next_solve():
    """rb_download_async of one problem while the next one solves gives the bits of rb_download,
    for both problems; a wait with nothing in flight and a second async download of the same
    problem are refused."""
    tabs = [W.c4_tables(seed=3, particle="photon", n=16, ng=2), W.c4_tables(seed=3, particle="electron", n=16, ng=2)]
    ctx = Context(0, 0)
    try:
        refs = [_solve(ctx, PackedProblem(t), ResultBuffers(PackedProblem(t))) for t in tabs]
        packs = [PackedProblem(t, pinned=True) for t in tabs]
        rbs = [ResultBuffers(p, pinned=True) for p in packs]
        hs = [ctx.upload(packs[0])]
        ctx.solve(hs[0])
        hs.append(ctx.upload(packs[1]))
        ctx.download_async(hs[0], rbs[0])
        with pytest.raises(_abi.RadiantError) as ei:
            ctx.download_async(hs[0], rbs[0])
        assert ei.value.status == RB_ERR_INVALID
        ctx.solve(hs[1])
        ctx.download_wait(hs[0])
        with pytest.raises(_abi.RadiantError) as ei:
            ctx.download_wait(hs[0])
        assert ei.value.status == RB_ERR_INVALID
        ctx.download_async(hs[1], rbs[1])
        ctx.download_wait(hs[1])
        for h in hs:
            ctx.release(h)
        for got, ref in zip(rbs, refs):
            assert np.array_equal(got.flux, ref.flux) and got.passes == ref.passes
            assert (got.flux_cutoff is None) == (ref.flux_cutoff is None)
            if ref.flux_cutoff is not None:
                assert np.array_equal(got.flux_cutoff, ref.flux_cutoff)
            assert np.array_equal(got.group_iters, ref.group_iters) and np.array_equal(got.rho, ref.rho)
    finally:
        ctx.close()
