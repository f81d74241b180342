"""The mixed-precision form (FP32 angular flux, sweep and moment<->discrete products; FP64
Krylov vectors, reductions, orthogonalisation and updates) against the FP64 oracle.

Acceptance of the chosen form: flux moments and cutoff flux within 1e-5 relative L2 of the FP64
solution, and the energy deposition computed from them within 1e-5 as well."""
import numpy as np
import pytest

from oracle import run as oracle_run
from radiant_b200 import workloads as W
from radiant_b200._abi import PackedProblem, ResultBuffers, load_library

pytestmark = pytest.mark.gpu
TOL_MIXED = 1e-5


def rel_l2(a, b):
    a = np.asarray(a).ravel(); b = np.asarray(b).ravel()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def solve(ctx, tabs):
    pp = PackedProblem(tabs)
    rb = ResultBuffers(pp)
    h = ctx.upload(pp)
    ctx.solve(h)
    ctx.download(h, rb)
    ctx.release(h)
    return rb


def deposition(tabs, flux, cutoff):
    import ctypes as C
    lib = load_library()
    xs = tabs["xs"]
    ng, np_, nm5 = tabs["ng"], tabs["np"], tabs["nm"][4]
    ncell = int(np.prod(tabs["ns"]))
    mat = np.asfortranarray(tabs["mat"].astype(np.int32))
    out = np.zeros(ncell)
    se = np.asfortranarray(xs.sigma_e)
    rho = np.asfortranarray(xs.density)
    dp = C.POINTER(C.c_double)
    f = np.asfortranarray(flux)
    cf = None if cutoff is None else np.asfortranarray(cutoff)
    st = lib.rb_energy_deposition(ng, np_, nm5, ncell, tabs["nmat"], mat.ctypes.data_as(C.POINTER(C.c_int32)),
                                  f.ctypes.data_as(dp), None if cf is None else cf.ctypes.data_as(dp),
                                  se.ctypes.data_as(dp), rho.ctypes.data_as(dp), 1.0, out.ctypes.data_as(dp))
    assert st == 0
    return out


@pytest.mark.parametrize("name,build", [
    ("c1_photon", lambda: W.c1_tables(seed=1, precision="mixed")),
    ("c2_photon", lambda: W.c2_tables(seed=3, precision="mixed", particle="photon")),
    ("c2_electron", lambda: W.c2_tables(seed=4, precision="mixed")),
])
def test_mixed_form_within_1e5_of_fp64(gpu_ctx, name, build):
    tabs = build()
    ref = oracle_run.solve(dict(tabs, precision="fp64"))
    got = solve(gpu_ctx, tabs)
    e = rel_l2(got.flux, ref.flux)
    assert e <= TOL_MIXED, f"{name}: flux rel L2 {e:.2e}"
    if ref.flux_cutoff is not None:
        assert rel_l2(got.flux_cutoff, ref.flux_cutoff) <= TOL_MIXED
    d_ref = deposition(tabs, ref.flux, ref.flux_cutoff)
    d_got = deposition(tabs, got.flux, got.flux_cutoff)
    assert rel_l2(d_got, d_ref) <= TOL_MIXED


@pytest.mark.parametrize("accel", ["none", "livolant", "anderson", "bicgstab"])
def test_mixed_form_other_accelerators(gpu_ctx, accel):
    tabs = W.c1_tables(seed=2, precision="mixed", accel=accel)
    ref = oracle_run.solve(dict(tabs, precision="fp64"))
    got = solve(gpu_ctx, tabs)
    assert rel_l2(got.flux, ref.flux) <= TOL_MIXED
    assert got.group_converged.all()
