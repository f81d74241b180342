"""Energy deposition (energy_deposition.jl:24-87): the library's rb_energy_deposition against the
oracle's restatement (oracle_energy_deposition) on a CSD slab with three materials and a
non-trivial cutoff flux. Both are host functions; no device is used."""
import ctypes as C

import numpy as np

from oracle import run as orun
from radiant_b200 import workloads as W
from radiant_b200._abi import load_library
from radiant_b200.sn_flux import SNSettings

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


def _deposition(lib, fn, tabs, flux, cutoff, norm):
    xs = tabs["xs"]
    ng, np_, nm5 = tabs["ng"], tabs["np"], tabs["nm"][4]
    ncell = int(np.prod(tabs["ns"]))
    mat = np.asfortranarray(tabs["mat"].astype(np.int32))
    se = np.asfortranarray(xs.sigma_e)
    rho = np.asfortranarray(xs.density)
    f = np.asfortranarray(flux)
    cf = None if cutoff is None else np.asfortranarray(cutoff)
    out = np.zeros(ncell)
    getattr(lib, fn).restype = C.c_int32
    st = getattr(lib, fn)(C.c_int32(ng), C.c_int32(np_), C.c_int32(nm5), C.c_int64(ncell), C.c_int32(tabs["nmat"]),
                          mat.ctypes.data_as(_ip), f.ctypes.data_as(_dp), None if cf is None else cf.ctypes.data_as(_dp),
                          se.ctypes.data_as(_dp), rho.ctypes.data_as(_dp), C.c_double(norm), out.ctypes.data_as(_dp))
    assert st == 0
    return out


def test_energy_deposition_matches_the_oracle_on_a_csd_slab():
    sn = SNSettings(solver_type="BFP", quadrature_order=8, legendre_order=3, scheme_type={"x": "DG", "E": "DG"},
                    scheme_order={"x": 2, "E": 2}, angular_fokker_planck="galerkin", acceleration="gmres",
                    convergence_criterion=1e-10)
    nx = 24
    mats = np.ones(nx, dtype=np.int32)
    mats[6:12] = 2
    mats[15:20] = 3
    tabs = W.slab_tables(nx, np.full(nx, 0.15), mats, 6, 3, 11, sn, 3, beam_group=0, csd=True)
    tabs["xs"].density = np.array([1.0, 1.85, 0.3])
    ref = orun.solve(tabs)
    assert np.linalg.norm(ref.flux_cutoff) > 0
    norm = 2.5
    a = _deposition(load_library(), "rb_energy_deposition", tabs, ref.flux, ref.flux_cutoff, norm)
    b = _deposition(orun.lib(), "oracle_energy_deposition", tabs, ref.flux, ref.flux_cutoff, norm)
    assert np.any(a != 0)
    np.testing.assert_array_equal(a, b)
    # the cutoff term matters on this slab
    c = _deposition(orun.lib(), "oracle_energy_deposition", tabs, ref.flux, None, norm)
    assert np.max(np.abs(b - c)) > 1e-6 * np.max(np.abs(b))
