"""Host table builders (restating the reference's host functions) against known values."""
import numpy as np
import pytest

from radiant_b200 import tables as T


@pytest.mark.parametrize("N", [2, 3, 8, 9, 16, 32, 64])
def test_gauss_legendre_matches_numpy(N):
    x, w = T.gauss_legendre(N)
    xr, wr = np.polynomial.legendre.leggauss(N)
    order = np.argsort(-x)
    np.testing.assert_allclose(np.sort(x), np.sort(xr), atol=4e-15)
    np.testing.assert_allclose(w[order], wr[::-1], rtol=5e-12)  # the reference formula loses ~1e-12 near |x| = 1
    assert x[0] > x[-1]  # reference order: largest node first (gauss_legendre.jl:20-24)


@pytest.mark.parametrize("btype", ["galerkin-d", "galerkin-m"])
def test_galerkin_bases_are_inverses(btype):
    x, w = T.gauss_legendre(16)
    Np, Mn, Dn, pl, _ = T.angular_polynomial_basis([x, 0 * x, 0 * x], w, 7, btype, 1)
    assert Np == 16 and list(pl) == list(range(16))
    np.testing.assert_allclose(Dn @ Mn, np.eye(16), atol=1e-10)


def test_standard_basis_moments():
    x, w = T.gauss_legendre(8)
    Np, Mn, Dn, pl, _ = T.angular_polynomial_basis([x, 0 * x, 0 * x], w, 3, "standard", 1)
    assert Np == 4
    np.testing.assert_allclose(Dn @ Mn, np.eye(4), atol=1e-12)  # GL8 integrates P_l P_l' exactly


def test_surface_basis_maps():
    x, w = T.gauss_legendre(8)
    Np, Mn, Dn, n2p, p2n, pl, _ = T.surface_angular_polynomial_basis_face([x, 0 * x, 0 * x], w, 64, "galerkin-d", 1, "X-")
    assert Np == 4 and list(n2p) == [1, 2, 3, 4]
    assert list(p2n) == [1, 2, 3, 4, 0, 0, 0, 0]
    np.testing.assert_allclose(Dn @ Mn, np.eye(4), atol=1e-10)


def test_scheme_weights():
    np.testing.assert_array_equal(T.axis_weights("DD", 1), [-1.0, 2.0])
    np.testing.assert_array_equal(T.axis_weights("DD", 2), [1.0, 0.0, 2.0])
    np.testing.assert_array_equal(T.axis_weights("DG", 2), [0.0, 1.0, 1.0])
    np.testing.assert_allclose(T.axis_weights("DG-", 2), [0.0, 1.0, 1 / 3])
    with pytest.raises(ValueError):
        T.axis_weights("DG+", 1)


@pytest.mark.parametrize("j", [(0, 0, 0), (1, 1, 0), (1, 1, 2), (2, 2, 2), (1, 2, 3), (1, 1, 1)])
def test_G6_is_triple_legendre_integral(j):
    x, w = np.polynomial.legendre.leggauss(12)
    P = [np.polynomial.legendre.Legendre.basis(k)(x) for k in range(4)]
    expect = 0.5 * np.sum(w * P[j[0]] * P[j[1]] * P[j[2]])
    assert T.G6(*j) == pytest.approx(expect, abs=1e-14)


def test_fokker_planck_galerkin_preserves_moments():
    x, w = T.gauss_legendre(8)
    Np, Mn, Dn, pl, _ = T.angular_polynomial_basis([x, 0 * x, 0 * x], w, 7, "galerkin-d", 1)
    M, lam0 = T.fokker_planck_galerkin(8, Mn, Dn, pl, Np)
    # eigenvalues of ℳ are -l(l+1) + λ₀ (Galerkin: Dn·(Mn·diag·Dn + λ₀I)·Mn)
    ev = np.sort(np.linalg.eigvals(M).real)
    np.testing.assert_allclose(ev, np.sort([-l * (l + 1) + lam0 for l in pl]), rtol=1e-9, atol=1e-9)
    assert lam0 >= 0


def test_fokker_planck_finite_difference_annihilates_isotropic():
    x, w = T.gauss_legendre(8)
    Np, Mn, Dn, pl, _ = T.angular_polynomial_basis([x, 0 * x, 0 * x], w, 7, "galerkin-d", 1)
    M, lam0 = T.fokker_planck_finite_difference_1d(8, "gauss-legendre", Mn, Dn)
    # the Laplacian part kills the isotropic moment: ℳ e0 = λ₀ e0
    e0 = np.zeros(Np); e0[0] = 1.0
    np.testing.assert_allclose(M @ e0, lam0 * e0, atol=1e-9)


def test_get_schemes_moment_counts():
    _, O, Nm = T.get_schemes({"x": "DG", "E": "DG"}, {"x": 2, "E": 2}, ["x"], True, True)
    assert O == [2, 1, 1, 2] and Nm == [2, 4, 4, 2, 4]
    _, O, Nm = T.get_schemes({"x": "DG", "E": "DG"}, {"x": 2, "E": 2}, ["x"], True, False)
    assert Nm == [2, 3, 3, 2, 3]
