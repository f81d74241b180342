"""Coupled transport (transport.jl:21-147) on the CPU: the coupling builders (angular transfer
matrix, moment map) against their definitions, and the oracle's generation loop against an
independent numpy restatement of particle_source and against closed-form known answers.
"""
import numpy as np
import pytest

from oracle import run as orun
from radiant_b200 import workloads as W
from radiant_b200.sn_flux import MultigroupXS, SNSettings, prepare_sn_tables
from radiant_b200.transport import Coupling, angular_transfer_matrix, build_coupling, map_moments


def test_map_moments_known_cases():
    # same orders: identity (map_moments.jl:29-55)
    np.testing.assert_array_equal(map_moments([2, 1, 1, 2], [2, 1, 1, 2], True, True), [1, 2, 3, 4])
    np.testing.assert_array_equal(map_moments([2, 2, 1, 1], [2, 2, 1, 1], False, False), [1, 2, 3])
    # low order into high order: only the average moment is fed
    np.testing.assert_array_equal(map_moments([1, 1, 1, 1], [2, 1, 1, 2], True, True), [1, 0, 0, 0])
    np.testing.assert_array_equal(map_moments([1, 1, 1, 1], [2, 2, 2, 1], False, False), [1, 0, 0, 0])
    # high order into low order: the average moment only
    np.testing.assert_array_equal(map_moments([2, 1, 1, 2], [1, 1, 1, 1], True, True), [1])
    # fully coupled in, decoupled out: (x,E) = (1,2) and (2,1) are moments 2 and 3 of both sets,
    # the coupled (2,2) has no decoupled counterpart (and the reverse leaves it unfed)
    np.testing.assert_array_equal(map_moments([2, 1, 1, 2], [2, 1, 1, 2], True, False), [1, 2, 3])
    np.testing.assert_array_equal(map_moments([2, 1, 1, 2], [2, 1, 1, 2], False, True), [1, 2, 3, 0])


def _sn_tabs(N, L, boltz="standard", qtype="gauss-legendre", ndims=1):
    xs = MultigroupXS(sigma_t=np.ones((1, 1)), sigma_s=np.zeros((1, 1, 1, L + 1)), sigma_a=np.ones((1, 1)),
                      sigma_e=np.ones((2, 1)), e_width=np.ones(1), density=np.ones(1))
    axes = ["x", "y", "z"][:ndims]
    sn = SNSettings(solver_type="BTE", quadrature_type=qtype, quadrature_order=N, legendre_order=L,
                    scheme_type={a: "DD" for a in axes}, scheme_order={a: 1 for a in axes}, angular_boltzmann=boltz)
    ns = [2] * ndims
    return prepare_sn_tables(xs, ndims, ns, [np.ones(2)] * ndims, np.ones(ns + [1] * (3 - ndims), dtype=np.int32),
                             [0] * 6, sn)


def test_transfer_same_quadrature_is_the_moment_identity():
    a, b = _sn_tabs(8, 5), _sn_tabs(8, 3)
    Tm = angular_transfer_matrix(a, b)  # P_out × P_in: (l, m) matched
    assert Tm.shape == (b["np"], a["np"])
    np.testing.assert_array_equal(Tm, np.eye(b["np"], a["np"]))


@pytest.mark.parametrize("ndims,qtype", [(1, "gauss-legendre"), (2, "carlson"), (3, "carlson")])
def test_transfer_between_quadratures_preserves_low_moments(ndims, qtype):
    """Dn_out·M(Ω_out) (particle_source.jl:243-244) maps a moment vector back onto itself for the
    orders both quadratures integrate exactly: the isotropic and linear moments are kept."""
    a, b = _sn_tabs(8, 1, qtype=qtype, ndims=ndims), _sn_tabs(6, 1, qtype=qtype, ndims=ndims)
    Tm = angular_transfer_matrix(a, b)
    assert Tm.shape == (b["np"], a["np"])
    k = min(a["np"], b["np"])
    np.testing.assert_allclose(Tm[:k, :k], np.eye(k), atol=1e-12)


def _numpy_particle_source(ti, tj, cp: Coupling, phi_i):
    """particle_source (particle_source.jl:54-70) written with numpy contractions."""
    mat = np.asarray(ti["mat"]).reshape(-1, order="F") - 1
    ng_j = tj["ng"]
    ncell = mat.size
    phi = phi_i.reshape(ti["ng"], ti["np"], ti["nm"][4], ncell, order="F")
    pl = np.asarray(ti["pl"])
    ss = cp.sigma_s[mat][:, :, :, pl]                 # [c, gi, gf, p]
    ql_in = np.einsum("cigp,ipkc->gpkc", ss, phi)     # [gf, p_in, k_in, c]
    ql_out = np.zeros((ng_j, tj["np"], tj["nm"][4], ncell))
    for k, m in enumerate(cp.moment_map):
        if m:
            ql_out[:, :, k, :] = np.einsum("qp,gpc->gqc", cp.transfer, ql_in[:, :, m - 1, :])
    return ql_out


def test_one_generation_matches_numpy_particle_source():
    """With Ngen_max = 1 the electron is solved once, from the source the photon flux produces
    (transport.jl:98-108): the oracle's loop against compute_flux on a numpy-built source."""
    parts, cps = W.coupled_particles(1, seed=3, ng=6, n=24)
    res, ngen, eps = orun.transport(parts, cps, ngen_max=1)
    assert ngen == 1 and np.isnan(eps)
    ph = orun.solve(parts[0])
    np.testing.assert_array_equal(res[0].flux, ph.flux)
    src = _numpy_particle_source(parts[0], parts[1], cps[(0, 1)], ph.flux)
    te = dict(parts[1])
    ns = list(te["ns"]) + [1] * (3 - len(te["ns"]))
    te["volume_sources"] = np.asfortranarray(src.reshape(te["ng"], te["np"], te["nm"][4], *ns, order="F"))
    el = orun.solve(te)
    den = np.linalg.norm(el.flux)
    assert den > 0
    assert np.linalg.norm(res[1].flux - el.flux) / den < 1e-13


def test_zero_coupling_is_the_single_particle_solve():
    """No coupling: generation 1 solves the photon, generation 2 adds zero and converges."""
    parts, _ = W.coupled_particles(1, seed=2, ng=5, n=20)
    res, ngen, eps = orun.transport(parts[:2], {}, ngen_max=10, eps_gen=1e-12)
    assert ngen == 2 and eps == 0.0
    np.testing.assert_array_equal(res[0].flux, orun.solve(parts[0]).flux)
    assert not res[1].flux.any()


def test_generation_loop_sums_a_geometric_series():
    """Two one-group particles in an infinite medium (reflective slab, pure absorbers), particle 1
    with a uniform isotropic source Q, isotropic production a (1→2) and b (2→1). Generation n adds
    k^(n-1)·Q/Σ₁ to particle 1, k = a·b/(Σ₁Σ₂), and particle 2 follows as a/Σ₂ times particle 1's
    flux of the same generation."""
    Q, s1, s2, a, b, nx = 2.0, 1.5, 0.8, 0.6, 0.5, 10
    sn = SNSettings(solver_type="BTE", quadrature_order=8, legendre_order=0, scheme_type={"x": "DD"},
                    scheme_order={"x": 1}, acceleration="gmres", convergence_criterion=1e-13,
                    angular_boltzmann="standard")

    def xs(st):
        return MultigroupXS(sigma_t=np.full((1, 1), st), sigma_s=np.zeros((1, 1, 1, 1)), sigma_a=np.full((1, 1), st),
                            sigma_e=np.ones((2, 1)), e_width=np.ones(1), density=np.ones(1))

    def slab(st, vol):
        return prepare_sn_tables(xs(st), 1, [nx], [np.full(nx, 0.3)], np.ones((nx, 1, 1), dtype=np.int32),
                                 [1, 1, 0, 0, 0, 0], sn, volume_sources=vol)

    p1 = slab(s1, np.full((1, 1, 1, nx, 1, 1), Q))
    p2 = slab(s2, None)
    cps = {(0, 1): build_coupling(p1, p2, np.full((1, 1, 1, 1), a)),
           (1, 0): build_coupling(p2, p1, np.full((1, 1, 1, 1), b))}
    k = a * b / (s1 * s2)
    for ngen_max in (1, 3, 6):
        res, ngen, _ = orun.transport([p1, p2], cps, ngen_max=ngen_max, eps_gen=0.0)
        assert ngen == ngen_max
        series = sum(k ** g for g in range(ngen_max))
        np.testing.assert_allclose(res[0].flux[0, 0, 0, :, 0, 0], Q / s1 * series, rtol=1e-11)
        np.testing.assert_allclose(res[1].flux[0, 0, 0, :, 0, 0], a / s2 * Q / s1 * series, rtol=1e-11)
    # the flux criterion: generation n changes particle 1 by k^(n-1) / Σ_{g<n} k^g
    res, ngen, eps = orun.transport([p1, p2], cps, ngen_max=50, eps_gen=1e-6)
    n = ngen
    expect = k ** (n - 1) / sum(k ** g for g in range(n))
    assert eps == pytest.approx(expect, rel=1e-9)
    assert eps < 1e-6 and k ** (n - 2) / sum(k ** g for g in range(n - 1)) >= 1e-6


def test_particle_order_starts_at_the_first_sourced_particle():
    """transport.jl:61-74: particles are solved from the first one with fixed sources, wrapping
    around; a loop with no fixed source at all is an error."""
    parts, cps = W.coupled_particles(1, seed=4, ng=4, n=16)
    # photon last in the list: the loop starts at it
    perm = [1, 2, 0]
    pp = [parts[i] for i in perm]
    inv = {old: new for new, old in enumerate(perm)}
    cc = {(inv[i], inv[j]): c for (i, j), c in cps.items()}
    r1, n1, e1 = orun.transport(parts, cps, ngen_max=4, eps_gen=0.0)
    r2, n2, e2 = orun.transport(pp, cc, ngen_max=4, eps_gen=0.0)
    assert n1 == n2
    for new, old in enumerate(perm):
        np.testing.assert_array_equal(r2[new].flux, r1[old].flux)
    with pytest.raises(RuntimeError):
        orun.transport(parts[1:], {}, ngen_max=2)


def test_deposition_criterion_on_the_geometric_series():
    """The energy-deposition criterion (transport.jl:122-127) on the two-particle infinite medium:
    the summed deposition grows like the fluxes, so its relative change per generation is the flux
    criterion's k^(n-1)/Σ_{g<n} k^g and both stop at the same generation; the deposition returned is
    (Σe₁·φ₁ + Σe₂·φ₂)/(ρ·norm)."""
    Q, s1, s2, a, b, nx = 2.0, 1.5, 0.8, 0.6, 0.5, 10
    sn = SNSettings(solver_type="BTE", quadrature_order=8, legendre_order=0, scheme_type={"x": "DD"},
                    scheme_order={"x": 1}, acceleration="gmres", convergence_criterion=1e-13,
                    angular_boltzmann="standard")

    def slab(st, vol):
        xs = MultigroupXS(sigma_t=np.full((1, 1), st), sigma_s=np.zeros((1, 1, 1, 1)), sigma_a=np.full((1, 1), st),
                          sigma_e=np.ones((2, 1)), e_width=np.ones(1), density=np.ones(1))
        return prepare_sn_tables(xs, 1, [nx], [np.full(nx, 0.3)], np.ones((nx, 1, 1), dtype=np.int32),
                                 [1, 1, 0, 0, 0, 0], sn, volume_sources=vol)

    p1, p2 = slab(s1, np.full((1, 1, 1, nx, 1, 1), Q)), slab(s2, None)
    cps = {(0, 1): build_coupling(p1, p2, np.full((1, 1, 1, 1), a)),
           (1, 0): build_coupling(p2, p1, np.full((1, 1, 1, 1), b))}
    se = [np.array([[0.7], [0.0]]), np.array([[0.3], [0.0]])]
    rho, norm = np.array([1.3]), 2.0
    r0, n0, e0 = orun.transport([p1, p2], cps, ngen_max=50, eps_gen=1e-6)
    r1, n1, e1, dep = orun.transport([p1, p2], cps, ngen_max=50, eps_gen=1e-6, conv_type=1, sigma_dep=se,
                                     density=rho, norm=norm, deposition=True)
    assert n1 == n0 and e1 == pytest.approx(e0, rel=1e-9)
    phi1, phi2 = r1[0].flux[0, 0, 0, :, 0, 0], r1[1].flux[0, 0, 0, :, 0, 0]
    np.testing.assert_allclose(dep, (0.7 * phi1 + 0.3 * phi2) / (1.3 * 2.0), rtol=1e-14)
    with pytest.raises(RuntimeError):
        orun.transport([p1, p2], cps, ngen_max=3, conv_type=3, sigma_dep=se, density=rho)
