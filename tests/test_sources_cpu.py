"""Fixed-source builders (radiant_b200.sources) against hand-computed values of
volume_source.jl:21-122, surface_source.jl:22-330 and Source.add_source (Source.jl:129-203):
voxel selection by centre with inclusive bounds, accumulation of overlapping sources, the
normalization factors, the entering-direction rule of a beam and its face-cell area factor.
"""
import math

import numpy as np
import pytest

from radiant_b200 import sources as S
from radiant_b200 import tables as T
from radiant_b200.sn_flux import SNSettings


def sn2d(L=3, order=4):
    return SNSettings(solver_type="BTE", quadrature_type="carlson", quadrature_order=order, legendre_order=L,
                      scheme_type={"x": "DD", "y": "DD"}, scheme_order={"x": 1, "y": 1}, acceleration="gmres",
                      convergence_criterion=1e-10, angular_boltzmann="galerkin-d")


def test_positions_are_voxel_centres():
    np.testing.assert_array_equal(S.positions_of([1.0, 1.0, 2.0, 2.0]), [0.5, 1.5, 3.0, 5.0])


def test_volume_boxes_known_answer():
    wx, wy = np.array([1.0, 1.0, 2.0, 2.0]), np.array([0.5, 0.5, 1.0])
    px, py = S.positions_of(wx), S.positions_of(wy)  # x 0.5 1.5 3 5; y 0.25 0.75 1.5
    a = S.VolumeSource(2, {"x": (0.0, 2.5), "y": (0.6, 2.0)}, intensity=3.0)
    b = S.VolumeSource(2, {"x": (1.5, 3.0), "y": (0.75, 0.75)}, intensity=0.5)  # bounds inclusive
    c = S.VolumeSource(1, {"x": (-1.0, 9.0), "y": (-1.0, 9.0)}, intensity=1.0)
    vol, surf, norms = S.dense_sources(sn2d(), 2, 3, [4, 3], [wx, wy], [px, py], [a, b, c])
    assert surf is None and vol.shape == (3, 1, 1, 4, 3, 1)
    want = np.zeros((4, 3))
    want[0:2, 1:3] += 3.0
    want[1:3, 1] += 0.5
    np.testing.assert_array_equal(vol[1, 0, 0, :, :, 0], want)
    np.testing.assert_array_equal(vol[0, 0, 0, :, :, 0], np.ones((4, 3)))
    assert not vol[2].any()
    # Σ intensity · Δx · Δy over the selected voxels, x outermost
    assert norms[0] == ((0.0 + 3.0 * 1.0 * 0.5) + 3.0 * 1.0 * 1.0 + 3.0 * 1.0 * 0.5) + 3.0 * 1.0 * 1.0
    assert norms[1] == 0.5 * 1.0 * 0.5 + 0.5 * 2.0 * 0.5
    assert norms[2] == pytest.approx(float(np.sum(np.outer(wx, wy))), rel=1e-15)


def test_beam_known_answer_2d():
    sn = sn2d()
    wx, wy = np.array([1.0, 2.0]), np.array([0.5, 0.25, 0.25])
    px, py = S.positions_of(wx), S.positions_of(wy)  # y 0.25 0.625 0.875
    d = (0.6, math.sqrt(1 - 0.6 ** 2 - 0.3 ** 2), 0.3)
    beam = S.SurfaceSource(1, "X-", d, {"y": (0.5, 1.0)}, intensity=2.0)
    basis, pl, pm = S.beam_basis(sn, 2, beam)
    vol, surf, norms = S.dense_sources(sn, 2, 2, [2, 3], [wx, wy], [px, py], surface=[beam])
    assert vol is None and surf[1] is None and surf[0].shape == (2, len(basis), 3)
    for p in range(len(basis)):
        assert surf[0][0, p, 0] == 0.0
        assert surf[0][0, p, 1] == 2.0 * basis[p] * 0.25
        assert surf[0][0, p, 2] == 2.0 * basis[p] * 0.25
    assert not surf[0][1].any()
    assert norms == [2.0 * 0.25 + 2.0 * 0.25]
    # the basis is the half-range harmonics at (|mu|, atan(xi, eta)); the first one is constant
    assert pl[0] == 0 and basis[0] > 0
    # a beam that leaves through its face adds nothing but still counts in its normalization
    out = S.SurfaceSource(1, "X-", (-d[0], d[1], d[2]), {"y": (0.5, 1.0)}, intensity=2.0)
    _, surf2, norms2 = S.dense_sources(sn, 2, 2, [2, 3], [wx, wy], [px, py], surface=[out])
    assert not surf2[0].any() and norms2 == norms


def test_beam_known_answer_1d_and_accumulation():
    sn = SNSettings(solver_type="BTE", quadrature_type="gauss-legendre", quadrature_order=8, legendre_order=5,
                    scheme_type={"x": "DD"}, scheme_order={"x": 1}, acceleration="gmres",
                    convergence_criterion=1e-10, angular_boltzmann="standard")
    w = np.full(4, 0.5)
    p = [S.positions_of(w)]
    b1 = S.SurfaceSource(3, "X-", (0.8, 0.0, 0.0), intensity=1.5)
    b2 = S.SurfaceSource(3, "X-", (0.4, 0.0, 0.0), intensity=0.5, legendre_order=2)
    b3 = S.SurfaceSource(1, "X+", (-1.0, 0.0, 0.0))
    _, surf, norms = S.dense_sources(sn, 1, 3, [4], [w], p, surface=[b1, b2, b3])
    P1 = T.half_range_legendre_polynomials_up_to_L(5, 0.8)
    P2 = T.half_range_legendre_polynomials_up_to_L(5, 0.4)
    n1 = len(S.beam_basis(sn, 1, b1)[0])
    n2 = len(S.beam_basis(sn, 1, b2)[0])
    assert n2 < n1 == surf[0].shape[1]
    for k in range(n1):
        want = 0.0 + 1.5 * P1[k]
        if k < n2:
            want = want + 0.5 * P2[k]
        assert surf[0][2, k, 0] == want
    assert surf[1][0, 0, 0] == 1.0 and norms == [1.5, 0.5, 1.0]


def test_source_set_layout():
    sn = sn2d()
    w = [np.ones(3), np.ones(2)]
    pos = [S.positions_of(a) for a in w]
    beam = S.SurfaceSource(2, "Y+", (0.5, -0.5, math.sqrt(0.5)), {"x": (1.0, 2.0)})
    box = S.VolumeSource(1, {"x": (0.0, 1.0)}, intensity=4.0)
    ss = S.SourceSet(sn, 2, pos, [box], [beam], np_surf=3)
    assert ss.np_source == 3 and ss.S.nvolume == 1 and ss.S.nsurface == 1
    assert ss.beams[0].face == 3 and ss.beams[0].energy_group == 2
    assert ss.boxes[0].lo[1] == -math.inf and ss.boxes[0].hi[0] == 1.0
    np.testing.assert_array_equal(np.ctypeslib.as_array(ss.beams[0].basis, (3,)), S.beam_basis(sn, 2, beam)[0][:3])


def test_workload_definitions_rebuild_the_workload_arrays():
    """The definitions a grid workload keeps (its volume box, its beam) rebuild exactly the dense
    arrays its tables carry, and the tables without them take the definitions' np_source."""
    from radiant_b200 import workloads as W

    for tabs in (W.c4_tables(seed=2, particle="photon", n=8, ng=2), W.random_grid_tables(5)):
        src = tabs["sources"]
        ns = list(tabs["ns"])
        vol, surf, _ = S.dense_sources(src["sn"], tabs["ndims"], tabs["ng"], ns, tabs["ds"], src["positions"],
                                       src["volume"], src["surface"])
        if vol is not None:
            np.testing.assert_array_equal(tabs["volume_sources"][:, :1, :1], vol)
            assert not tabs["volume_sources"][:, 1:].any()
        for f in range(2 * tabs["ndims"]):
            if surf is not None and surf[f] is not None:
                k = tabs["np_source"]
                np.testing.assert_array_equal(tabs["surface_sources"][f], surf[f][:, :k])
        bare, sset = W.without_dense_sources(tabs)
        assert bare["volume_sources"] is None and all(a is None for a in bare["surface_sources"])
        assert sset.np_source == tabs["np_source"]


@pytest.mark.parametrize("ndims", [1, 2, 3])
def test_host_builders_against_the_oracle(ndims):
    """The Python host builders (the dense path) against the oracle's C restatement
    (oracle_sources) on seeded random definitions: identical arrays and normalization factors."""
    from oracle import run as orun

    rng = np.random.default_rng(10 + ndims)
    if ndims == 1:
        sn = SNSettings(solver_type="BTE", quadrature_type="gauss-legendre", quadrature_order=16, legendre_order=5,
                        scheme_type={"x": "DD"}, scheme_order={"x": 1}, acceleration="gmres",
                        convergence_criterion=1e-10, angular_boltzmann="standard")
        ns = [37]
    else:
        sn = SNSettings(solver_type="BTE", quadrature_type="carlson", quadrature_order=4, legendre_order=3,
                        scheme_type={a: "DD" for a in "xyz"[:ndims]}, scheme_order={a: 1 for a in "xyz"[:ndims]},
                        acceleration="gmres", convergence_criterion=1e-10, angular_boltzmann="galerkin-d")
        ns = [9, 7, 5][:ndims]
    ng = 4
    widths = [rng.uniform(0.1, 0.5, n) for n in ns]
    pos = [S.positions_of(w) for w in widths]
    ext = [float(np.sum(w)) for w in widths]

    def box():
        out = {}
        for a in range(ndims):
            lo, hi = np.sort(rng.uniform(-0.1, ext[a] + 0.1, 2))
            out["xyz"[a]] = (float(lo), float(hi))
        return out

    vols = [S.VolumeSource(int(rng.integers(1, ng + 1)), box(), float(rng.uniform(0.1, 3.0))) for _ in range(4)]
    faces = S.FACES[:2 * ndims]
    beams = []
    for _ in range(5):
        f = faces[int(rng.integers(0, len(faces)))]
        d = rng.normal(size=3)
        d = tuple(d / np.linalg.norm(d))
        aperture = {k: v for k, v in box().items() if k != "xyz"[faces.index(f) // 2]}
        beams.append(S.SurfaceSource(int(rng.integers(1, ng + 1)), f, d, aperture, float(rng.uniform(0.2, 2.0)),
                                     legendre_order=int(rng.integers(1, 4))))
    vol, surf, norms = S.dense_sources(sn, ndims, ng, ns, widths, pos, vols, beams)
    sset = S.SourceSet(sn, ndims, pos, vols, beams)
    ovol, osurf, onorms = orun.sources(ndims, ng, ns, widths, pos, sset, sset.np_source)
    np.testing.assert_array_equal(vol.reshape(ng, -1, order="F"), ovol)
    for f in range(2 * ndims):
        assert (surf[f] is None) == (osurf[f] is None)
        if surf[f] is not None:
            np.testing.assert_array_equal(surf[f], osurf[f])
    np.testing.assert_array_equal(np.asarray(norms), onorms)
