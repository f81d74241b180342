"""FMAC-M files (read_fmac_m.jl:16-461, write_fmac_m.jl:16-377): the number fields against hand-
computed values, a written coupled photon-electron-positron library read back (six significant
digits kept, zero transfers kept zero, the cutoff rows of the deposition tables derived as the
reference does), and a solve on tables read from a file.
"""
import numpy as np
import pytest

from oracle import run as orun
from radiant_b200 import fmac as F
from radiant_b200.sn_flux import SNSettings, prepare_sn_tables


def test_number_fields():
    assert F._fmt_float(1.0) == " 1.00000E+00"
    assert F._fmt_float(-0.00123456) == "-1.23456E-03"
    assert F._fmt_float(0.0) == " 0.00000E+00"
    assert F._fmt_float(123456789.0) == " 1.23457E+08"
    assert F._fmt_float(2.5e-30) == " 2.50000E-30"
    assert F._fmt_float(1e-120) == " 0.00000E-00"  # beyond two exponent digits: written as zero
    assert F._fmt_int(42) == "          42" and F._fmt_int(-7) == "          -7"
    line = F._one_space(" 1.00000E+00-1.23456E-03 2.50000E-30")
    assert line == "1.00000E+00-1.23456E-03 2.50000E-30"
    np.testing.assert_allclose(F._floats(line, 3), [1.0, -1.23456e-3, 2.5e-30], rtol=1e-15)
    assert F._one_space("   3   4      5 ") == "3 4 5 "


def _library(seed=3):
    rng = np.random.default_rng(seed)
    parts, ng, nmat, L = ["photon", "electron", "positron"], [5, 4, 4], 2, 3
    lib = F.FmacLibrary(particles=parts, ng=ng, legendre_order=L, nmat=nmat, title="synthetic")
    for n, p in enumerate(parts):
        eb = np.sort(rng.uniform(0.01, 10.0, ng[n] + 1))[::-1]
        lib.e_bounds.append(eb)
        lib.total.append(rng.uniform(0.1, 5.0, (ng[n], nmat)))
        lib.absorption.append(np.zeros((ng[n], nmat)))
        lib.stopping.append(rng.uniform(1.0, 3.0, (ng[n] + 1, nmat)) if p != "photon" else np.zeros((ng[n] + 1, nmat)))
        lib.momentum.append(rng.uniform(0.0, 1.0, (ng[n], nmat)))
        lib.edep.append(rng.uniform(0.0, 1.0, (ng[n] + 1, nmat)))
        lib.cdep.append(rng.uniform(-1.0, 1.0, (ng[n] + 1, nmat)))
    for n in range(3):
        for m in range(3):
            s = np.zeros((nmat, ng[n], ng[m], L + 1))
            for mat in range(nmat):
                for gi in range(ng[n]):
                    for gf in range(gi if n == m else 0, ng[m]):
                        if rng.uniform() < 0.3:
                            continue  # some transfers are zero
                        lmax = int(rng.integers(0, L + 1))
                        s[mat, gi, gf, :lmax + 1] = rng.uniform(-0.5, 1.0, lmax + 1)
            lib.scattering[(n, m)] = s
    return lib


def test_write_then_read_keeps_the_tables(tmp_path):
    lib = _library()
    path = str(tmp_path / "lib.fmac")
    F.write_fmac_m(lib, path)
    got = F.read_fmac_m(path)
    assert got.particles == lib.particles and got.ng == lib.ng and got.nmat == lib.nmat
    assert got.legendre_order == lib.legendre_order
    rt = dict(rtol=5e-6, atol=0.0)
    for n in range(3):
        np.testing.assert_allclose(got.e_bounds[n], lib.e_bounds[n], **rt)
        np.testing.assert_allclose(got.total[n], lib.total[n], **rt)
        np.testing.assert_allclose(got.stopping[n], lib.stopping[n], **rt)
        np.testing.assert_allclose(got.momentum[n], lib.momentum[n], **rt)
        np.testing.assert_allclose(got.edep[n][:-1], lib.edep[n][:-1], **rt)
        np.testing.assert_allclose(got.cdep[n][:-1], lib.cdep[n][:-1], **rt)
        # the cutoff rows come from the stopping power at the cutoff (read_fmac_m.jl:335-337)
        eb, sp = got.e_bounds[n], got.stopping[n][-1]
        q = {"photon": 0.0, "electron": -1.0, "positron": 1.0}[lib.particles[n]]
        np.testing.assert_allclose(got.edep[n][-1], sp * eb[-1] / (eb[-2] - eb[-1]), rtol=1e-15)
        np.testing.assert_allclose(got.cdep[n][-1], sp * (-q) / (eb[-2] - eb[-1]), rtol=1e-15, atol=0.0)
        for m in range(3):
            a, b = got.scattering[(n, m)], lib.scattering[(n, m)]
            np.testing.assert_allclose(a, b, rtol=5e-6, atol=1e-300)
            assert np.array_equal(a == 0.0, b == 0.0)
    sub = F.read_fmac_m(path, particles=["electron", "photon"])
    assert sub.particles == ["photon", "electron"]
    np.testing.assert_array_equal(sub.get_scattering("electron", "photon", 3), got.get_scattering("electron", "photon", 3))


def test_rejects_other_files(tmp_path):
    p = tmp_path / "x.txt"
    p.write_text("NOT-FMAC\n")
    with pytest.raises(ValueError):
        F.read_fmac_m(str(p))


def test_solve_on_tables_read_from_a_file(tmp_path):
    """The electron tables of a written and re-read library feed a BFP slab solve (oracle)."""
    lib = _library(seed=5)
    path = str(tmp_path / "lib.fmac")
    F.write_fmac_m(lib, path)
    xs = F.read_fmac_m(path).multigroup("electron", density=[1.0, 1.8])
    sn = SNSettings(solver_type="BFP", quadrature_order=8, legendre_order=3, scheme_type={"x": "DD", "E": "DD"},
                    scheme_order={"x": 1, "E": 1}, angular_fokker_planck="galerkin", acceleration="gmres",
                    convergence_criterion=1e-9, angular_boltzmann="standard")
    nx = 20
    mats = np.ones((nx, 1, 1), dtype=np.int32)
    mats[8:12] = 2
    vol = np.zeros((xs.ng, 1, 1, nx, 1, 1))
    vol[0, 0, 0, :5] = 1.0
    tabs = prepare_sn_tables(xs, 1, [nx], [np.full(nx, 0.1)], mats, [0] * 6, sn, volume_sources=vol)
    r = orun.solve(tabs)
    assert np.all(np.isfinite(r.flux)) and r.flux[:, 0, 0].sum() > 0


@pytest.mark.gpu
def test_gpu_solve_on_tables_read_from_a_file(tmp_path):
    """The same read-back electron problem on the GPU (rb_compute_flux) against the oracle, 1e-10."""
    import ctypes as C
    from radiant_b200._abi import PackedProblem, ResultBuffers, load_library
    lib = _library(seed=7)
    path = str(tmp_path / "lib.fmac")
    F.write_fmac_m(lib, path)
    xs = F.read_fmac_m(path).multigroup("electron", density=[1.0, 1.8])
    sn = SNSettings(solver_type="BFP", quadrature_order=16, legendre_order=3, scheme_type={"x": "DG", "E": "DG"},
                    scheme_order={"x": 2, "E": 2}, angular_fokker_planck="galerkin", acceleration="gmres",
                    convergence_criterion=1e-10, angular_boltzmann="standard")
    nx = 30
    mats = np.ones((nx, 1, 1), dtype=np.int32)
    mats[10:20] = 2
    vol = np.zeros((xs.ng, 1, 1, nx, 1, 1))
    vol[0, 0, 0, :6] = 1.0
    tabs = prepare_sn_tables(xs, 1, [nx], [np.full(nx, 0.1)], mats, [0] * 6, sn, volume_sources=vol)
    ref = orun.solve(tabs)
    pp = PackedProblem(tabs)
    got = ResultBuffers(pp)
    assert load_library().rb_compute_flux(0, C.byref(pp.P), C.byref(got.R)) == 0
    assert np.linalg.norm(got.flux - ref.flux) / np.linalg.norm(ref.flux) <= 1e-10
    assert np.linalg.norm(got.flux_cutoff - ref.flux_cutoff) / np.linalg.norm(ref.flux_cutoff) <= 1e-10
