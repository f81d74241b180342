"""Seeded synthetic inputs with the shapes of the benchmark configurations.

Radiant.jl generates multigroup cross sections from physics models and bundled data
(src/cross_sections/*). That generator stays outside this library, and it cannot run
where this library is built, so the workloads below use synthetic tables with the same
shapes (groups, materials, Legendre orders) and physically shaped values:
Σt ~ U(0.05, 5)/cm smooth in the group, downscatter-only Σs₀ whose row sums are c·Σt with
c ~ U(0.3, 0.95), Henyey-Greenstein moments Σs_l = Σs₀·g^l with g ~ U(0.3, 0.9)
(Radiant's Mn already carries the (2l+1)/2 factor, so the moments carry none), and positive stopping powers
and momentum transfer smooth in the group. Every table is labelled synthetic.
"""
from __future__ import annotations

import math

import numpy as np

from . import sources as S
from . import tables as T
from .sn_flux import MultigroupXS, SNSettings, prepare_sn_tables


def log_groups(ng: int, e_top: float, e_cut: float):
    """Log-spaced group boundaries, highest energy first (the reference's group order)."""
    eb = np.exp(np.linspace(math.log(e_top), math.log(e_cut), ng + 1))
    e = np.sqrt(eb[:-1] * eb[1:])
    return eb, e, eb[:-1] - eb[1:]


def synthetic_xs(ng: int, nmat: int, L: int, seed: int, csd: bool = False,
                 e_top: float = 2.0, e_cut: float = 0.01, scale: float = 1.0) -> MultigroupXS:
    """Synthetic multigroup tables of one particle (labelled synthetic)."""
    rng = np.random.default_rng(seed)
    g = np.arange(ng)
    sigma_t = np.zeros((ng, nmat))
    sigma_s = np.zeros((nmat, ng, ng, L + 1))
    t_mom = np.zeros((ng, nmat))
    sb = np.zeros((ng + 1, nmat))
    sigma_e = np.zeros((ng + 1, nmat))
    density = np.zeros(nmat)
    for m in range(nmat):
        lo, hi = sorted(rng.uniform(0.05, 5.0, size=2))
        ramp = np.linspace(0.0, 1.0, ng) ** rng.uniform(0.5, 2.0)
        sigma_t[:, m] = scale * (lo + (hi - lo) * ramp)
        c = rng.uniform(0.3, 0.95)
        aniso = rng.uniform(0.3, 0.9)
        for gi in range(ng):
            # downscatter-only row gi -> gf >= gi, geometric fall-off, row sum c·Σt
            k = np.arange(ng - gi)
            prof = np.exp(-k * rng.uniform(0.5, 2.0))
            prof /= prof.sum()
            row = c * sigma_t[gi, m] * prof
            for l in range(L + 1):
                sigma_s[m, gi, gi:, l] = row * aniso ** l
        density[m] = rng.uniform(0.3, 2.0)
        if csd:
            s0 = rng.uniform(1.5, 2.5)
            sb[:, m] = s0 * (1.0 + 0.5 * np.linspace(0.0, 1.0, ng + 1))
            t_mom[:, m] = rng.uniform(0.05, 0.5) * (1.0 + np.linspace(0.0, 2.0, ng))
        sigma_e[:ng, m] = rng.uniform(0.01, 0.1) * (1.0 + g / ng)
        sigma_e[ng, m] = rng.uniform(0.5, 1.5)
    eb, e, de = log_groups(ng, e_top, e_cut)
    return MultigroupXS(sigma_t=sigma_t, sigma_s=sigma_s, sigma_a=sigma_t * 0.2, sb=sb if csd else None,
                        t_mom=t_mom if csd else None, sigma_e=sigma_e, e_width=de, energies=e, e_bounds=eb,
                        density=density)


def surface_source_1d(tabs_np_surf_L: int, L_solver: int, btype: str, Om, w, ng: int, group: int,
                      mu_s: float, intensity: float = 1.0, surface: str = "X-"):
    """Moments of a monodirectional 1D surface beam (surface_source.jl:64-96, Qdims == 1).
    Returns (Q [ng, Np_src, 2 faces], normalisation)."""
    L = min(tabs_np_surf_L, L_solver)
    Np, _, _, _, _, pl, _ = T.surface_angular_polynomial_basis_face(Om, w, L, btype, 1, surface)
    Lmax = int(np.max(pl))
    Pls = T.half_range_legendre_polynomials_up_to_L(Lmax, abs(mu_s))
    Q = np.zeros((ng, Np, 2))
    for p in range(Np):
        l = pl[p]
        if surface == "X-" and mu_s > 0:
            Q[group, p, 0] = intensity * Pls[l]
        elif surface == "X+" and mu_s < 0:
            Q[group, p, 1] = intensity * Pls[l]
    return Q, intensity


def slab_tables(nx: int, widths, mats, ng: int, nmat: int, seed: int, sn: SNSettings, L_xs: int,
                beam_group: int = 0, bc=(0, 0), volume_group=None, csd=False, precision="fp64",
                xs: MultigroupXS | None = None, beam_mu: float = 1.0):
    """A 1D slab: `mats` gives the material id (1-based) of each voxel, `widths` its width."""
    xs = xs or synthetic_xs(ng, nmat, L_xs, seed, csd=csd)
    Qdims = sn.qdims(1)
    Om, w = T.quadrature(sn.quadrature_order, sn.quadrature_type, 1, Qdims)
    surf = None
    if beam_group is not None:
        Q, _ = surface_source_1d(64, sn.legendre_order, sn.angular_boltzmann, [Om, 0 * Om, 0 * Om], w, ng,
                                 beam_group, beam_mu)
        surf = [Q[:, :, 0:1], Q[:, :, 1:2]]
    vol = None
    if volume_group is not None:
        vol = np.zeros((ng, 1, 1, nx, 1, 1))
        vol[volume_group, 0, 0, :, 0, 0] = 1.0
    tabs = prepare_sn_tables(xs, 1, [nx], [np.asarray(widths, dtype=float)], np.asarray(mats).reshape(nx, 1, 1),
                             list(bc) + [0] * 4, sn, volume_sources=vol, surface_sources=surf, precision=precision)
    tabs["xs"] = xs
    return tabs


def c1_tables(seed: int = 1, precision: str = "fp64", accel: str = "gmres"):
    """1D slab BTE, photons: 10 cm, 200 voxels, void/void, 40 groups, S16 Gauss-Legendre,
    P7, diamond difference, GMRES to 1e-8, normal beam at x=0 in the top group."""
    sn = SNSettings(solver_type="BTE", quadrature_type="gauss-legendre", quadrature_order=16,
                    legendre_order=7, scheme_type={"x": "DD"}, scheme_order={"x": 1},
                    acceleration=accel, convergence_criterion=1e-8)
    nx = 200
    return slab_tables(nx, np.full(nx, 10.0 / nx), np.ones(nx, dtype=np.int32), 40, 1, seed, sn, 7,
                       precision=precision)


def c2_tables(seed: int = 1, precision: str = "fp64", accel: str = "gmres", particle: str = "electron",
              ng: int = 80):
    """1D slab BFP: water 0-3 cm / bone 3-5 cm / water 5-15 cm, 300 voxels of 0.05 cm,
    80 groups, S32 Gauss-Legendre, P15, linear DG in x and in E, Galerkin (moment-preserving)
    angular Fokker-Planck, normal beam in the group holding 6 MeV."""
    nx = 300
    mats = np.ones(nx, dtype=np.int32)
    mats[60:100] = 2
    eb, e, de = log_groups(ng, 20.0, 0.001)
    g6 = int(np.nonzero((eb[:-1] >= 6.0) & (eb[1:] < 6.0))[0][0])
    if particle == "photon":
        sn = SNSettings(solver_type="BTE", quadrature_type="gauss-legendre", quadrature_order=32,
                        legendre_order=15, scheme_type={"x": "DG"}, scheme_order={"x": 2},
                        acceleration=accel, convergence_criterion=1e-8)
        csd = False
    else:
        sn = SNSettings(solver_type="BFP", quadrature_type="gauss-legendre", quadrature_order=32,
                        legendre_order=15, scheme_type={"x": "DG", "E": "DG"}, scheme_order={"x": 2, "E": 2},
                        angular_fokker_planck="galerkin", acceleration=accel, convergence_criterion=1e-8)
        csd = True
    xs = synthetic_xs(ng, 2, 15, seed, csd=csd, e_top=20.0, e_cut=0.001)
    return slab_tables(nx, np.full(nx, 0.05), mats, ng, 2, seed, sn, 15, beam_group=g6, csd=csd,
                       precision=precision, xs=xs)


def random_slab_tables(seed: int, precision: str = "fp64", max_cells: int = 2000, max_groups: int = 120):
    """One 1D request of the serving stream: cells U(50, max_cells), groups U(10, max_groups),
    SN order in {8,16,32,64}, P order U(1,9), 1-5 layers of 4 materials, photon (BTE) or
    electron (BFP) with probability 1/2."""
    rng = np.random.default_rng(seed)
    nx = int(rng.integers(50, max_cells + 1))
    ng = int(rng.integers(10, max_groups + 1))
    N = int(rng.choice([8, 16, 32, 64]))
    L = int(rng.integers(1, 10))
    nlay = int(rng.integers(1, 6))
    cuts = np.sort(rng.choice(np.arange(1, nx), size=nlay - 1, replace=False)) if nlay > 1 else []
    mats = np.ones(nx, dtype=np.int32)
    start = 0
    for k, cpos in enumerate(list(cuts) + [nx]):
        mats[start:cpos] = int(rng.integers(1, 5))
        start = cpos
    bfp = bool(rng.integers(0, 2))
    if bfp:
        sn = SNSettings(solver_type="BFP", quadrature_type="gauss-legendre", quadrature_order=N,
                        legendre_order=L, scheme_type={"x": "DD", "E": "DD"}, scheme_order={"x": 1, "E": 1},
                        angular_fokker_planck="galerkin", acceleration="gmres", convergence_criterion=1e-7,
                        angular_boltzmann="standard")
    else:
        sn = SNSettings(solver_type="BTE", quadrature_type="gauss-legendre", quadrature_order=N,
                        legendre_order=L, scheme_type={"x": "DD"}, scheme_order={"x": 1},
                        acceleration="gmres", convergence_criterion=1e-7, angular_boltzmann="standard")
    width = rng.uniform(2.0, 20.0)
    xs = synthetic_xs(ng, 4, L, seed + 7919, csd=bfp)
    return slab_tables(nx, np.full(nx, width / nx), mats, ng, 4, seed, sn, L, beam_group=0, csd=bfp,
                       precision=precision, xs=xs)


def grid_source_definitions(ndims, beam=None, volume=None) -> dict:
    """The Volume_Source / Surface_Source definitions of grid_tables' `beam` = (face, group,
    direction, aperture) and `volume` = (group, {axis: (lo, hi)}) (0-based groups and axes):
    unit intensity, the beam's Legendre order the reference's default (64)."""
    out = {"volume": [], "surface": []}
    if volume is not None:
        group, box = volume
        out["volume"].append(S.VolumeSource(group + 1, {"xyz"[a]: tuple(v) for a, v in box.items()}))
    if beam is not None:
        face, group, direction, aperture = beam
        out["surface"].append(S.SurfaceSource(group + 1, face, tuple(direction),
                                              {"xyz"[a]: tuple(v) for a, v in (aperture or {}).items()}))
    return out


def grid_tables(ndims, ns, widths, mats, ng, nmat, seed, sn: SNSettings, L_xs: int, beam=None, volume=None,
                bc=(0, 0, 0, 0, 0, 0), csd=False, precision="fp64", xs: MultigroupXS | None = None):
    """A 2D/3D Cartesian grid: `widths` per axis, `mats` [nx,ny(,nz)] 1-based; `beam` =
    (face, group, direction, aperture) and `volume` = (group, {axis: (lo, hi)}) as in the
    reference's Surface_Source / Volume_Source."""
    xs = xs or synthetic_xs(ng, nmat, L_xs, seed, csd=csd)
    ns = list(ns)
    ds = [np.asarray(wd, dtype=float) for wd in widths]
    defs = grid_source_definitions(ndims, beam, volume)
    positions = [S.positions_of(d) for d in ds]
    vol, surf, _ = S.dense_sources(sn, ndims, ng, ns, ds, positions, defs["volume"], defs["surface"])
    full = ns + [1] * (3 - ndims)
    tabs = prepare_sn_tables(xs, ndims, ns, ds, np.asarray(mats).reshape(full, order="F"), list(bc), sn,
                             volume_sources=vol, surface_sources=surf, precision=precision)
    tabs["xs"] = xs
    tabs["sources"] = dict(defs, positions=positions, sn=sn)  # the definitions behind vol / surf
    return tabs


def without_dense_sources(tabs: dict):
    """(tables with no dense source arrays, sources.SourceSet of their definitions): the problem as
    rb_upload_sources takes it."""
    src = tabs["sources"]
    sset = S.SourceSet(src["sn"], tabs["ndims"], src["positions"], src["volume"], src["surface"],
                       np_surf=tabs["np_surf"])
    bare = dict(tabs)
    bare["volume_sources"] = None
    bare["surface_sources"] = [None] * 6
    bare["np_source"] = sset.np_source
    return bare, sset


def c3_tables(seed: int = 1, particle: str = "photon", precision: str = "fp64", n: int = 128, ng: int = 60,
              quad: int = 12, accel: str = "gmres"):
    """2D Cartesian photon-electron solve: 128×128 voxels over 20×20 cm, water plus 12 seeded
    circular inclusions (centres uniform, radii U(0.5, 2) cm, bone or 0.3 g/cc water with
    probability 1/2), 60 groups per particle 10 keV-10 MeV, level-symmetric S12 (168
    directions), P5, diamond difference, 2 MeV photon beam on the left face over a 4 cm
    aperture."""
    rng = np.random.default_rng(seed)
    L = 20.0
    dx = L / n
    xc = (np.arange(n) + 0.5) * dx
    mats = np.ones((n, n), dtype=np.int32)
    for _ in range(12):
        cx, cy = rng.uniform(0, L, size=2)
        r = rng.uniform(0.5, 2.0)
        tag = 2 if rng.uniform() < 0.5 else 3
        X, Y = np.meshgrid(xc, xc, indexing="ij")
        mats[(X - cx) ** 2 + (Y - cy) ** 2 <= r * r] = tag
    eb, e, de = log_groups(ng, 10.0, 0.01)
    g2 = int(np.nonzero((eb[:-1] >= 2.0) & (eb[1:] < 2.0))[0][0])
    csd = particle != "photon"
    st = {"x": "DD", "y": "DD"}
    so = {"x": 1, "y": 1}
    if csd:
        st["E"] = "DD"
        so["E"] = 1
    sn = SNSettings(solver_type="BFP" if csd else "BTE", quadrature_type="carlson", quadrature_order=quad,
                    legendre_order=5, scheme_type=st, scheme_order=so, acceleration=accel,
                    convergence_criterion=1e-7, angular_fokker_planck="galerkin")
    xs = synthetic_xs(ng, 3, 5, seed * 11 + (1 if csd else 0), csd=csd, e_top=10.0, e_cut=0.01)
    beam = ("X-", g2, (1.0, 0.0, 0.0), {1: (8.0, 12.0)}) if not csd else None
    vol = None if not csd else (g2, {0: (0.0, 4.0), 1: (8.0, 12.0)})
    return grid_tables(2, [n, n], [np.full(n, dx), np.full(n, dx)], mats, ng, 3, seed, sn, 5, beam=beam,
                       volume=vol, csd=csd, precision=precision, xs=xs)


def c4_tables(seed: int = 1, particle: str = "photon", precision: str = "fp64", n: int = 64, ng: int = 40,
              quad: int = 8):
    """3D Cartesian photon-electron solve: 64³ voxels over a 16 cm cube, water with a seeded
    16³-voxel bone block at a random offset, 40 groups per particle 10 keV-6 MeV,
    level-symmetric S8 (80 directions), P3, reflective at z=0 (Z-), void elsewhere, isotropic
    volume source of unit strength in the top group inside the central 8³ voxels, BiCGStab to
    1e-6."""
    rng = np.random.default_rng(seed)
    L = 16.0
    dx = L / n
    mats = np.ones((n, n, n), dtype=np.int32)
    b = max(1, n // 4)
    o = rng.integers(0, n - b + 1, size=3)
    mats[o[0]:o[0] + b, o[1]:o[1] + b, o[2]:o[2] + b] = 2
    csd = particle != "photon"
    st = {"x": "DD", "y": "DD", "z": "DD"}
    so = {"x": 1, "y": 1, "z": 1}
    if csd:
        st["E"] = "DD"
        so["E"] = 1
    sn = SNSettings(solver_type="BFP" if csd else "BTE", quadrature_type="carlson", quadrature_order=quad,
                    legendre_order=3, scheme_type=st, scheme_order=so, acceleration="bicgstab",
                    convergence_criterion=1e-6, angular_fokker_planck="galerkin")
    xs = synthetic_xs(ng, 2, 3, seed * 13 + (1 if csd else 0), csd=csd, e_top=6.0, e_cut=0.01)
    c = L / 2
    h = 8 * dx / 2
    vol = (0, {0: (c - h, c + h), 1: (c - h, c + h), 2: (c - h, c + h)})
    return grid_tables(3, [n, n, n], [np.full(n, dx)] * 3, mats, ng, 2, seed, sn, 3, volume=vol,
                       bc=(0, 0, 0, 0, 1, 0), csd=csd, precision=precision, xs=xs)


def random_grid_tables(seed: int, precision: str = "fp64", max_side: int = 128):
    """One 2D request of the serving stream: square grid of side U(32, max_side), level-symmetric
    S4-S12, photon transport (BTE), 1-4 materials in vertical layers, beam on the left face."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(32, max_side + 1))
    N = int(rng.choice([4, 6, 8, 10, 12]))
    L = int(rng.integers(1, 4))
    ng = int(rng.integers(10, 41))
    nmat = int(rng.integers(1, 5))
    mats = np.ones((n, n), dtype=np.int32)
    cuts = np.linspace(0, n, nmat + 1).astype(int)
    for k in range(nmat):
        mats[cuts[k]:cuts[k + 1], :] = k + 1
    sn = SNSettings(solver_type="BTE", quadrature_type="carlson", quadrature_order=N, legendre_order=L,
                    scheme_type={"x": "DD", "y": "DD"}, scheme_order={"x": 1, "y": 1}, acceleration="gmres",
                    convergence_criterion=1e-7, angular_boltzmann="standard")
    width = rng.uniform(5.0, 20.0)
    d = width / n
    xs = synthetic_xs(ng, nmat, L, seed + 104729, e_top=10.0, e_cut=0.01)
    return grid_tables(2, [n, n], [np.full(n, d), np.full(n, d)], mats, ng, nmat, seed, sn, L,
                       beam=("X-", 0, (1.0, 0.0, 0.0), {1: (0.25 * width, 0.75 * width)}), precision=precision, xs=xs)


def serving_stream(n: int, seed: int, precision: str = "mixed", max_cells: int = 2000, max_groups: int = 120,
                   max_side: int = 128):
    """The serving request mix: 70 % 1D slabs (random_slab_tables) and 30 % 2D grids
    (random_grid_tables), seeded; 1D requests in `precision`, 2D requests in FP64."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        s = int(rng.integers(0, 2 ** 31 - 1))
        if rng.uniform() < 0.7:
            out.append(random_slab_tables(s, precision=precision, max_cells=max_cells, max_groups=max_groups))
        else:
            out.append(random_grid_tables(s, max_side=max_side))
    return out


# ------------------------------------------------------------------------------------------
# the serving stream (configuration C5)
# ------------------------------------------------------------------------------------------
C5_MATERIALS = 4  # water, cortical bone, lung-density water (0.3 g/cc), aluminium (synthetic tables)


def _beam_group(eb, energy):
    """Index of the group holding `energy` (boundaries highest first)."""
    for g in range(len(eb) - 1):
        if eb[g] >= energy > eb[g + 1]:
            return g
    return 0 if energy > eb[0] else len(eb) - 2


def c5_request(seed: int, precision: str = "mixed", max_cells: int = 2000, max_groups: int = 120,
               max_side: int = 128):
    """One request of the serving stream, as the serving configuration draws it: a 1D slab with
    probability 0.7 (cells U(50, max_cells), SN order in {8,16,32,64}, P order U(1,9), 1-5
    layers of the four materials) or a 2D grid (side U(32, max_side), level-symmetric S4-S12,
    vertical material layers); groups U(10, max_groups) per particle; a normal beam on the X-
    face at an energy log-uniform in 0.1-20 MeV (group structure 20 MeV - 1 keV); particle set
    photon only or photon + electron + positron with probability 1/2. Returns the list of the
    request's particle solves (tables), photon first."""
    rng = np.random.default_rng(seed)
    is1d = rng.uniform() < 0.7
    parts = ["photon"] if rng.uniform() < 0.5 else ["photon", "electron", "positron"]
    energy = math.exp(rng.uniform(math.log(0.1), math.log(20.0)))
    ng = int(rng.integers(10, max_groups + 1))
    eb, _, _ = log_groups(ng, 20.0, 0.001)
    gb = _beam_group(eb, energy)
    L = int(rng.integers(1, 10))
    out = []
    if is1d:
        nx = int(rng.integers(50, max_cells + 1))
        N = int(rng.choice([8, 16, 32, 64]))
        nlay = int(rng.integers(1, 6))
        cuts = sorted(rng.choice(np.arange(1, nx), size=nlay - 1, replace=False)) if nlay > 1 else []
        mats = np.ones(nx, dtype=np.int32)
        start = 0
        for cpos in list(cuts) + [nx]:
            mats[start:cpos] = int(rng.integers(1, C5_MATERIALS + 1))
            start = cpos
        width = rng.uniform(2.0, 20.0)
        for k, part in enumerate(parts):
            bfp = part != "photon"
            if bfp:
                sn = SNSettings(solver_type="BFP", quadrature_type="gauss-legendre", quadrature_order=N,
                                legendre_order=L, scheme_type={"x": "DD", "E": "DD"}, scheme_order={"x": 1, "E": 1},
                                angular_fokker_planck="galerkin", acceleration="gmres", convergence_criterion=1e-7,
                                angular_boltzmann="standard")
            else:
                sn = SNSettings(solver_type="BTE", quadrature_type="gauss-legendre", quadrature_order=N,
                                legendre_order=L, scheme_type={"x": "DD"}, scheme_order={"x": 1},
                                acceleration="gmres", convergence_criterion=1e-7, angular_boltzmann="standard")
            xs = synthetic_xs(ng, C5_MATERIALS, L, seed * 7 + k + 7919, csd=bfp, e_top=20.0, e_cut=0.001)
            t = slab_tables(nx, np.full(nx, width / nx), mats, ng, C5_MATERIALS, seed, sn, L, beam_group=gb,
                            csd=bfp, precision=precision, xs=xs)
            t["particle"] = part
            out.append(t)
        return out
    n = int(rng.integers(32, max_side + 1))
    N = int(rng.choice([4, 6, 8, 10, 12]))
    L2 = min(L, 3)
    nmat = int(rng.integers(1, C5_MATERIALS + 1))
    mats = np.ones((n, n), dtype=np.int32)
    cuts = np.linspace(0, n, nmat + 1).astype(int)
    for k in range(nmat):
        mats[cuts[k]:cuts[k + 1], :] = int(rng.integers(1, C5_MATERIALS + 1))
    width = rng.uniform(5.0, 20.0)
    d = width / n
    for k, part in enumerate(parts):
        bfp = part != "photon"
        st = {"x": "DD", "y": "DD"}
        so = {"x": 1, "y": 1}
        if bfp:
            st["E"] = "DD"
            so["E"] = 1
        sn = SNSettings(solver_type="BFP" if bfp else "BTE", quadrature_type="carlson", quadrature_order=N,
                        legendre_order=L2, scheme_type=st, scheme_order=so, acceleration="gmres",
                        convergence_criterion=1e-7, angular_boltzmann="standard", angular_fokker_planck="galerkin")
        xs = synthetic_xs(ng, C5_MATERIALS, L2, seed * 7 + k + 104729, csd=bfp, e_top=20.0, e_cut=0.001)
        t = grid_tables(2, [n, n], [np.full(n, d), np.full(n, d)], mats, ng, C5_MATERIALS, seed, sn, L2,
                        beam=("X-", gb, (1.0, 0.0, 0.0), {1: (0.25 * width, 0.75 * width)}), csd=bfp,
                        precision=precision, xs=xs)
        t["particle"] = part
        out.append(t)
    return out


def c5_stream(n: int, seed: int, precision: str = "mixed", max_cells: int = 2000, max_groups: int = 120,
              max_side: int = 128):
    """The first `n` requests of the seeded serving stream (c5_request each)."""
    rng = np.random.default_rng(seed)
    seeds = rng.integers(0, 2 ** 31 - 1, size=n)
    return [c5_request(int(s), precision, max_cells, max_groups, max_side) for s in seeds]


# ------------------------------------------------------------------------------------------
# coupled particles (transport())
# ------------------------------------------------------------------------------------------
def synthetic_coupling_xs(ng_in: int, ng_out: int, nmat: int, L: int, seed: int, strength: float) -> np.ndarray:
    """Synthetic production cross sections Σs(i→j) [nmat, ng_in, ng_out, L+1] of a secondary
    particle (labelled synthetic): from group gi into the groups gf ≥ gi of the other particle,
    geometric fall-off, row sum `strength`·U(0.5, 1), anisotropy a^l."""
    rng = np.random.default_rng(seed)
    ss = np.zeros((nmat, ng_in, ng_out, L + 1))
    for m in range(nmat):
        c = strength * rng.uniform(0.5, 1.0)
        aniso = rng.uniform(0.2, 0.8)
        rate = rng.uniform(0.3, 1.5)
        for gi in range(min(ng_in, ng_out)):
            k = np.arange(ng_out - gi)
            prof = np.exp(-k * rate)
            prof /= prof.sum()
            for l in range(L + 1):
                ss[m, gi, gi:, l] = c * prof * aniso ** l
    return ss


COUPLING_STRENGTH = {(0, 1): 0.4, (0, 2): 0.1, (1, 0): 0.05, (2, 0): 0.3}  # γ→e⁻, γ→e⁺, e⁻→γ, e⁺→γ


def coupled_particles(ndims: int = 1, seed: int = 1, precision: str = "fp64", ng: int = 10, n=None,
                      photon_quad: int = 8, positron_quad: int | None = None, L: int = 3, dg_electron: bool = True,
                      tol: float = 1e-9):
    """Photon (BTE), electron and positron (BFP, CSD) on one geometry with the synthetic
    couplings γ→e⁻, γ→e⁺, e⁻→γ, e⁺→γ; photon beam on the X- face in the top group. The electron
    uses the photon's quadrature (identity angular transfer); the positron another order
    (transfer through its Dn); with `dg_electron` the electron carries linear DG moments in x and
    E (a non-trivial cell-moment map). Returns (tables per particle, {(i, j): Coupling})."""
    from .transport import build_coupling

    positron_quad = positron_quad or max(2, photon_quad - 2)
    nmat = 2
    parts = []
    if ndims == 1:
        nx = n or 60
        mats = np.ones(nx, dtype=np.int32)
        mats[nx // 3:nx // 2] = 2
        widths = np.full(nx, 6.0 / nx)
    else:
        n = list(n or ([12, 10] if ndims == 2 else [6, 5, 4]))
        mats = np.ones(n, dtype=np.int32)
        sl = tuple(slice(k // 3, k // 2 + 1) for k in n)
        mats[sl] = 2
        widths = [np.full(k, 3.0 / k) for k in n]
    for k, part in enumerate(("photon", "electron", "positron")):
        bfp = part != "photon"
        quad = positron_quad if part == "positron" else photon_quad
        dg = dg_electron and part == "electron"
        axes = ["x", "y", "z"][:ndims]
        st = {a: "DD" for a in axes}
        so = {a: 1 for a in axes}
        if dg:
            st["x"], so["x"] = "DG", 2
        if bfp:
            st["E"], so["E"] = ("DG", 2) if dg else ("DD", 1)
        sn = SNSettings(solver_type="BFP" if bfp else "BTE",
                        quadrature_type="gauss-legendre" if ndims == 1 else "carlson", quadrature_order=quad,
                        legendre_order=L, scheme_type=st, scheme_order=so, acceleration="gmres",
                        convergence_criterion=tol, angular_fokker_planck="galerkin")
        xs = synthetic_xs(ng, nmat, L, seed * 17 + k, csd=bfp, e_top=6.0, e_cut=0.01)
        if ndims == 1:
            t = slab_tables(nx, widths, mats, ng, nmat, seed, sn, L, beam_group=0 if k == 0 else None, csd=bfp,
                            precision=precision, xs=xs)
        else:
            beam = ("X-", 0, (0.8, 0.6, 0.0), {1: (0.5, 2.5)}) if k == 0 else None
            t = grid_tables(ndims, n, widths, mats, ng, nmat, seed, sn, L, beam=beam, csd=bfp,
                            precision=precision, xs=xs)
        t["particle"] = part
        parts.append(t)
    couplings = {}
    for (i, j), s in COUPLING_STRENGTH.items():
        Li = int(np.max(parts[i]["pl"]))
        ss = synthetic_coupling_xs(ng, ng, nmat, Li, seed * 31 + 3 * i + j, s)
        couplings[(i, j)] = build_coupling(parts[i], parts[j], ss)
    return parts, couplings
