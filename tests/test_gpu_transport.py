"""rb_transport (the generation loop of transport.jl:21-147 on the device) against the oracle's
generation loop: photon, electron and positron coupled both ways on 1D, 2D and 3D geometries.

Tolerances: 1e-10 relative L2 per particle for the FP64 form (the parity bar of the single
solves); 1e-5 for the mixed form. The number of generations must be the same.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import run as orun
from radiant_b200 import workloads as W
from radiant_b200._abi import RB_ERR_INVALID, PackedProblem, RadiantError, ResultBuffers, \
    load_library
from radiant_b200.transport import transport_tables

pytestmark = pytest.mark.gpu
TOL = 1e-10
TOL_MIXED = 1e-5


def rel_l2(a, b):
    a = np.asarray(a).ravel(); b = np.asarray(b).ravel()
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def _compare(parts, cps, ngen_max, eps_gen, tol):
    ref, n_ref, e_ref = orun.transport(parts, cps, ngen_max=ngen_max, eps_gen=eps_gen)
    got = transport_tables(parts, cps, ngen_max=ngen_max, eps_gen=eps_gen)
    assert got.generations == n_ref
    for k, (g, r) in enumerate(zip(got.fluxes, ref)):
        assert np.linalg.norm(r.flux) > 0, f"particle {k} has no flux"
        e = rel_l2(g.flux, r.flux)
        assert e <= tol, f"particle {k}: flux rel L2 {e:.3e}"
        if r.flux_cutoff is not None:
            assert rel_l2(g.flux_cutoff, r.flux_cutoff) <= tol
    if n_ref > 1 and tol == TOL:
        assert got.eps == pytest.approx(e_ref, rel=1e-5, abs=1e-12)
    return got


@pytest.mark.parametrize("ndims", [1, 2, 3])
def test_coupled_three_particles_match_oracle(ndims):
    parts, cps = W.coupled_particles(ndims, seed=5, ng=6 if ndims > 1 else 10)
    got = _compare(parts, cps, ngen_max=20, eps_gen=1e-7, tol=TOL)
    assert got.generations > 2


def test_coupled_runs_to_the_generation_limit():
    """A loop stopped by Ngen_max: the last generation computes no sources it will not use
    (transport.jl:98-102), and the totals still match."""
    parts, cps = W.coupled_particles(1, seed=6, ng=8)
    got = _compare(parts, cps, ngen_max=3, eps_gen=0.0, tol=TOL)
    assert got.generations == 3


def test_coupled_mixed_form():
    parts, cps = W.coupled_particles(1, seed=7, ng=10, precision="mixed")
    ref_parts = [dict(t, precision="fp64") for t in parts]
    ref, n_ref, _ = orun.transport(ref_parts, cps, ngen_max=20, eps_gen=1e-7)
    got = transport_tables(parts, cps, ngen_max=20, eps_gen=1e-7)
    assert abs(got.generations - n_ref) <= 1
    for g, r in zip(got.fluxes, ref):
        assert rel_l2(g.flux, r.flux) <= TOL_MIXED


def test_zero_coupling_equals_compute_flux():
    parts, _ = W.coupled_particles(1, seed=8, ng=8)
    got = transport_tables(parts[:2], {}, ngen_max=5, eps_gen=1e-12)
    assert got.generations == 2 and got.eps == 0.0
    pp = PackedProblem(parts[0])
    rb = ResultBuffers(pp)
    assert load_library().rb_compute_flux(0, C.byref(pp.P), C.byref(rb.R)) == 0
    np.testing.assert_array_equal(got.fluxes[0].flux, rb.flux)
    assert not got.fluxes[1].flux.any()


def test_rejections():
    parts, cps = W.coupled_particles(1, seed=9, ng=4, n=16)
    with pytest.raises(RadiantError) as e:  # a deposition criterion without its cross sections
        transport_tables(parts, cps, conv_type="energy-deposition")
    assert e.value.status == RB_ERR_INVALID and "deposition" in str(e.value)
    with pytest.raises(ValueError):
        transport_tables(parts, cps, conv_type="dose")
    with pytest.raises(RadiantError) as e:
        transport_tables(parts[1:], {})
    assert e.value.status == RB_ERR_INVALID and "No fixed sources" in str(e.value)


def _dep_tables(parts):
    return [np.asarray(t["xs"].sigma_e, dtype=float) for t in parts], np.asarray(parts[0]["xs"].density, dtype=float)


@pytest.mark.parametrize("conv", ["energy-deposition", "charge-deposition"])
def test_deposition_criteria_match_oracle(conv):
    """The deposition criteria (transport.jl:122-133) on the device against the oracle's loop:
    same generations, same last ϵ, and the summed deposition of the final fluxes within 1e-10.
    (Charge deposition has the energy deposition's formula with Σc; the synthetic tables serve
    as both.)"""
    parts, cps = W.coupled_particles(1, seed=11, ng=8)
    sig, rho = _dep_tables(parts)
    ct = {"energy-deposition": 1, "charge-deposition": 2}[conv]
    ref, n_ref, e_ref, d_ref = orun.transport(parts, cps, ngen_max=20, eps_gen=1e-7, conv_type=ct, sigma_dep=sig,
                                              density=rho, norm=1.7, deposition=True)
    got = transport_tables(parts, cps, ngen_max=20, eps_gen=1e-7, conv_type=conv, sigma_dep=sig, density=rho,
                           norm=1.7, deposition=True)
    assert got.generations == n_ref > 2
    assert got.eps == pytest.approx(e_ref, rel=1e-5, abs=1e-12)
    assert rel_l2(got.deposition, d_ref) <= TOL
    for g, r in zip(got.fluxes, ref):
        assert rel_l2(g.flux, r.flux) <= TOL


@pytest.mark.parametrize("ndims", [1, 3])
def test_device_deposition_of_resident_problems(ndims):
    """rb_deposition (energy_deposition.jl:24-87 on the device, summed over particles) against the
    oracle's per-particle deposition of the downloaded fluxes."""
    from radiant_b200._abi import Context, PackedProblem, ResultBuffers
    parts, _ = W.coupled_particles(ndims, seed=12, ng=5 if ndims == 3 else 8)
    sig, rho = _dep_tables(parts)
    ctx = Context(0, 0)
    hs, rbs = [], []
    for t in parts:
        pp = PackedProblem(t); rb = ResultBuffers(pp)
        h = ctx.upload(pp); ctx.solve(h); ctx.download(h, rb)
        hs.append(h); rbs.append((pp, rb))
    got = ctx.deposition(hs, sig, rho, norm=0.9)
    want = np.zeros_like(got)
    L = orun.lib()
    dp = C.POINTER(C.c_double)
    for (pp, rb), s in zip(rbs, sig):
        t = pp.tables
        one = np.zeros_like(got)
        mat = np.ascontiguousarray(np.asarray(t["mat"]).reshape(-1, order="F"), dtype=np.int32)
        s = np.asfortranarray(s)
        L.oracle_energy_deposition(C.c_int32(t["ng"]), C.c_int32(t["np"]), C.c_int32(t["nm"][4]), C.c_int64(mat.size),
                                   C.c_int32(t["nmat"]), mat.ctypes.data_as(C.POINTER(C.c_int32)),
                                   rb.flux.ctypes.data_as(dp),
                                   rb.flux_cutoff.ctypes.data_as(dp) if rb.flux_cutoff is not None else None,
                                   s.ctypes.data_as(dp), rho.ctypes.data_as(dp), C.c_double(0.9), one.ctypes.data_as(dp))
        want += one
    ctx.close()
    assert np.linalg.norm(want) > 0
    assert rel_l2(got, want) <= TOL
