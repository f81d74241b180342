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
from radiant_b200._abi import RB_ERR_INVALID, RB_ERR_UNSUPPORTED, PackedProblem, RadiantError, ResultBuffers, \
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
    with pytest.raises(RadiantError) as e:
        transport_tables(parts, cps, conv_type="energy-deposition")
    assert e.value.status == RB_ERR_UNSUPPORTED
    with pytest.raises(RadiantError) as e:
        transport_tables(parts[1:], {})
    assert e.value.status == RB_ERR_INVALID and "No fixed sources" in str(e.value)
