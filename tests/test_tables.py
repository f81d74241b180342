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


def test_gauss_lobatto_and_legendre_chebychev_quadratures():
    x, w = T.gauss_lobatto(7)
    assert x[0] == 1.0 and x[-1] == -1.0
    for k in range(0, 11):  # exact to degree 2N - 3
        np.testing.assert_allclose((w * x ** k).sum(), (1 + (-1) ** k) / (k + 1), atol=1e-14)
    Om, w = T.gauss_legendre_chebychev(6)
    assert len(w) == 2 * 36
    np.testing.assert_allclose(w.sum(), 4 * np.pi, rtol=1e-14)
    for a in range(3):
        np.testing.assert_allclose((w * Om[a] ** 2).sum(), 4 * np.pi / 3, rtol=1e-13)
        np.testing.assert_allclose((w * Om[a]).sum(), 0.0, atol=1e-13)


@pytest.mark.parametrize("Qdims", [2, 3])
def test_finite_difference_fokker_planck_on_the_product_quadrature(Qdims):
    """fokker_planck_finite_difference.jl, product-quadrature branches: every row of ℳ_n − λ₀I sums
    to zero (the operator conserves particles), the shifted diagonal is non-negative, and the
    first-order harmonics are eigenvectors with the Laplace-Beltrami value −l(l+1) = −2 (the scheme
    is moment-preserving): μ and η in 2D (the folded half-range domain), μ, η, ξ in 3D."""
    for N in (4, 8, 16):
        Om, w = T.quadrature(N, "gauss-legendre-chebychev", 3, Qdims)
        Nd = len(w)
        M, lam0 = T.fokker_planck_finite_difference_glc(N, Qdims, np.eye(Nd), np.eye(Nd))
        L = M - lam0 * np.eye(Nd)
        np.testing.assert_allclose(L.sum(axis=1), 0.0, atol=1e-10 * lam0)
        assert np.all(np.diag(M) >= -1e-12) and lam0 > 0
        for a in range(2 if Qdims == 2 else 3):
            f = np.asarray(Om[a])
            np.testing.assert_allclose(L @ f, -2 * f, atol=1e-10)


def test_differential_quadrature_fokker_planck_is_exact_on_legendre_polynomials():
    """fokker_planck_differential_quadrature.jl: the Lagrange-derivative form is exact on
    polynomials below the quadrature order: (ℳ − λ₀I)·P_l(μ) = −l(l+1)·P_l(μ)."""
    N = 8
    mu, w = T.quadrature(N, "gauss-legendre", 1)
    M, lam0 = T.fokker_planck_differential_quadrature(N, "gauss-legendre", np.eye(N), np.eye(N))
    L = M - lam0 * np.eye(N)
    for l in range(N):
        P = np.array([T.legendre_polynomials_up_to_L(l, float(m))[l] for m in mu])
        np.testing.assert_allclose(L @ P, -l * (l + 1) * P, atol=1e-8 * max(1, l * l))


@pytest.mark.parametrize("ndims", [2, 3])
def test_default_fokker_planck_tables_build_in_2d_and_3d(ndims):
    """A BFP problem with the default angular Fokker-Planck ("finite-difference") on the product
    quadrature sets up in 2D and 3D, and the oracle solves it to a finite flux."""
    from oracle import run as orun
    from radiant_b200 import workloads as W
    from radiant_b200.sn_flux import SNSettings
    sn = SNSettings(solver_type="BFP", quadrature_type="gauss-legendre-chebychev", quadrature_order=4,
                    legendre_order=2, scheme_type={"x": "DD", "y": "DD", "z": "DD", "E": "DD"},
                    scheme_order={"x": 1, "y": 1, "z": 1, "E": 1}, acceleration="gmres", convergence_criterion=1e-8,
                    angular_boltzmann="standard")
    n = [5, 4] if ndims == 2 else [4, 3, 3]
    mats = np.ones(n, dtype=np.int32)
    t = W.grid_tables(ndims, n, [np.full(k, 0.25) for k in n], mats, 3, 1, 1, sn, 2,
                      volume=(0, {0: (0.0, 0.5)}), csd=True)
    assert t["fp"] is not None and t["fp"].shape == (t["np"], t["np"])
    r = orun.solve(t)
    assert np.all(np.isfinite(r.flux)) and r.flux.sum() > 0
