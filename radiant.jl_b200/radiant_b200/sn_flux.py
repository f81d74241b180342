"""compute_flux(::SN): the table set-up of sn_flux.jl:27-147 and the call into the CUDA library.

``prepare_sn_tables`` restates the set-up part of Radiant.jl's
``compute_flux(cross_sections, geometry, solver::SN, source)`` (sn_flux.jl:22-147) on the host,
from plain arrays; ``compute_flux`` then hands the tables to ``libradiant_b200.so`` which runs
the group loop (sn_flux.jl:162-224) on the GPU.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import tables as T
from ._abi import Context, PackedProblem, ResultBuffers

SOLVER_TYPES = {"BTE": 1, "BFP": 2, "BCSD": 3, "FP": 4, "CSD": 5, "BFP-EF": 6}
BC_CODES = {"void": 0, "reflective": 1, "periodic": 2}


@dataclass
class MultigroupXS:
    """Multigroup data of one particle, in the reference's getter shapes
    (src/structures/Cross_Sections.jl:854-1105)."""
    sigma_t: np.ndarray            # [ng,nmat]      get_total
    sigma_s: np.ndarray            # [nmat,ng,ng,L+1] get_scattering(p,p,L)
    sigma_a: np.ndarray | None = None   # [ng,nmat]  get_absorption
    sb: np.ndarray | None = None   # [ng+1,nmat]    get_boundary_stopping_powers
    t_mom: np.ndarray | None = None  # [ng,nmat]    get_momentum_transfer
    sigma_e: np.ndarray | None = None  # [ng+1,nmat] get_energy_deposition
    e_width: np.ndarray | None = None  # [ng]       get_energy_width
    energies: np.ndarray | None = None  # [ng]      get_energies
    e_bounds: np.ndarray | None = None  # [ng+1]    get_energy_boundaries
    density: np.ndarray | None = None   # [nmat]    get_densities

    @property
    def ng(self) -> int:
        return self.sigma_t.shape[0]

    @property
    def nmat(self) -> int:
        return self.sigma_t.shape[1]

    def scattering(self, L: int) -> np.ndarray:
        """get_scattering zero-pads / truncates to L+1 moments (Cross_Sections.jl:928-942)."""
        nmat, ng, _, nl = self.sigma_s.shape
        out = np.zeros((nmat, ng, ng, L + 1))
        k = min(L + 1, nl)
        out[:, :, :, :k] = self.sigma_s[:, :, :, :k]
        return out


@dataclass
class SNSettings:
    """The SN object's fields (src/structures/SN.jl:22-63)."""
    solver_type: str = "BTE"
    quadrature_type: str = "gauss-legendre"
    quadrature_order: int = 8
    quadrature_dimension: int = 0
    legendre_order: int = 64
    angular_fokker_planck: str = "finite-difference"
    angular_boltzmann: str = "galerkin-d"
    convergence_criterion: float = 1e-7
    maximum_iteration: int = 300
    scheme_type: dict = field(default_factory=dict)
    scheme_order: dict = field(default_factory=dict)
    acceleration: str = "none"
    gmres_restart: int = 30
    anderson_depth: int = 3
    is_full_coupling: bool = True

    def qdims(self, Ndims: int) -> int:
        """get_quadrature_dimension (SN.jl:638-659)."""
        q = self.quadrature_dimension
        if self.quadrature_type in ("gauss-legendre", "gauss-lobatto"):
            if q in (2, 3):
                raise ValueError("Quadrature dimension should be 1 with quadrature over the direction cosine.")
            return 1
        if Ndims in (1, 2):
            if q == 1:
                raise ValueError("Quadrature dimension should not be 1 with quadrature over the unit sphere.")
            return 2 if q == 2 else 3
        if q in (1, 2):
            raise ValueError("Quadrature dimension should not be 1 or 2 in 3D geometry.")
        return 3


def _face_cells(ndims, ns, axis):
    if ndims == 1:
        return 1
    if ndims == 2:
        return ns[1] if axis == 0 else ns[0]
    return [ns[1] * ns[2], ns[0] * ns[2], ns[0] * ns[1]][axis]


def prepare_sn_tables(xs: MultigroupXS, ndims: int, ns, ds, mat, bc, sn: SNSettings,
                      volume_sources=None, surface_sources=None, surface_L=None,
                      precision: str = "fp64") -> dict:
    """Everything sn_flux.jl:27-147 builds before its group loop, as a dict of arrays.

    ``mat`` is 1-based [nx,ny,nz]; ``bc`` the six RB_BC codes; ``volume_sources``
    [ng,np,nm5,nx,ny,nz] or None; ``surface_sources`` a list (one per face) of
    [ng, nsrc, face cells] arrays or None.
    """
    ns = [int(v) for v in ns] + [1] * (3 - len(ns))
    Qdims = sn.qdims(ndims)
    Om, w = T.quadrature(sn.quadrature_order, sn.quadrature_type, ndims, Qdims)
    if Qdims == 1:
        Om = [np.asarray(Om), 0 * np.asarray(Om), 0 * np.asarray(Om)]
    Nd = len(w)
    L = sn.legendre_order
    Np, Mn, Dn, pl, pm = T.angular_polynomial_basis(Om, w, L, sn.angular_boltzmann, Qdims)
    Np_surf, Mn_s, Dn_s, _np2n, n_to_np, _pls, _pms = T.surface_angular_polynomial_basis(
        Om, w, L, sn.angular_boltzmann, Qdims, ndims)
    st = SOLVER_TYPES[sn.solver_type.upper()]
    isCSD = st >= 2
    axes = ["x", "y", "z"][:ndims]
    schemes, O, Nm = T.get_schemes(sn.scheme_type, sn.scheme_order, axes, isCSD, sn.is_full_coupling)
    w_axis, Cc, is_adaptive, W = T.scheme_weights(O, schemes, ndims, isCSD)
    ng, nmat = xs.ng, xs.nmat
    # Σtot (sn_flux.jl:69-74)
    if st in (4, 5):
        sigma_t = np.array(xs.sigma_a, dtype=float)
    else:
        sigma_t = np.array(xs.sigma_t, dtype=float)
    Ls = int(np.max(pl))
    sigma_s = np.zeros((nmat, ng, ng, Ls + 1))
    if st not in (4, 5):
        sigma_s = xs.scattering(Ls)
    s_minus = s_plus = s_mom = None
    if isCSD:
        Sb = np.asarray(xs.sb, dtype=float)
        s_minus = np.array(Sb[0:ng, :])
        s_plus = np.array(Sb[1:ng + 1, :])
        s_mom = np.zeros((ng, nmat, O[3]))
        s_mom[:, :, 0] = (s_minus + s_plus) / 2
        if O[3] > 1:
            s_mom[:, :, 1] = (s_minus - s_plus) / (2 * math.sqrt(3))
    t_mom = fp = None
    if st in (2, 4):
        t_mom = np.array(xs.t_mom, dtype=float)
        fp, lam0 = T.fokker_planck_scattering_matrix(sn.quadrature_order, Nd, sn.quadrature_type, ndims,
                                                     sn.angular_fokker_planck, Mn, Dn, pl, Np, Qdims)
        sigma_t = sigma_t + t_mom * lam0
    if st == 6:
        for n in range(nmat):
            for ig in range(ng):
                sigma_t[ig, n] -= sigma_s[n, ig, ig, 0]
    nm5 = Nm[4]
    if volume_sources is None:
        vol = None
    else:
        vol = np.asarray(volume_sources, dtype=float)
        full = np.zeros((ng, Np, nm5, *ns), order="F")  # the reference's column-major layout
        full[:, :vol.shape[1], :vol.shape[2]] = vol.reshape(vol.shape[0], vol.shape[1], vol.shape[2], *ns)
        vol = full
    surf = [None] * 6
    np_source = 0
    if surface_sources is not None:
        nsrc = max((s.shape[1] for s in surface_sources if s is not None), default=0)
        np_source = int(min(Np_surf, nsrc))
        for f in range(2 * ndims):
            s = surface_sources[f] if f < len(surface_sources) else None
            if s is None:
                continue
            arr = np.zeros((ng, np_source, _face_cells(ndims, ns, f // 2)))
            k = min(np_source, s.shape[1])
            arr[:, :k, :] = np.asarray(s, dtype=float).reshape(ng, s.shape[1], -1)[:, :k, :]
            surf[f] = arr
    return dict(
        ndims=ndims, ns=ns[:3], ds=[np.asarray(d, dtype=float) for d in ds], mat=np.asarray(mat).reshape(ns, order="F"),
        nmat=nmat, bc=list(bc) + [0] * (6 - len(bc)),
        nd=Nd, omega=[np.asarray(Om[0]), np.asarray(Om[1]), np.asarray(Om[2])], w=np.asarray(w),
        qdims=Qdims, btype=sn.angular_boltzmann,
        np=Np, mn=Mn, dn=Dn, pl=pl, pm=pm, np_surf=Np_surf, mn_surf=Mn_s, dn_surf=Dn_s, n_to_nplus=n_to_np,
        order=O, nm=Nm, is_fc=sn.is_full_coupling, w_axis=w_axis, cc=Cc, ww=W, is_adaptive=is_adaptive,
        solver_type=st, ng=ng, sigma_t=sigma_t, ls=Ls, sigma_s=sigma_s, s_minus=s_minus, s_plus=s_plus,
        s_mom=s_mom, t_mom=t_mom, fp=fp, e_width=None if xs.e_width is None else np.asarray(xs.e_width, dtype=float),
        volume_sources=vol, np_source=np_source, surface_sources=surf,
        accel=sn.acceleration, tol=float(sn.convergence_criterion), max_iter=int(sn.maximum_iteration),
        gmres_restart=int(sn.gmres_restart), anderson_depth=int(sn.anderson_depth), precision=precision,
    )


@dataclass
class FluxPerParticle:
    """What compute_flux returns (src/structures/Flux_Per_Particle.jl)."""
    flux: np.ndarray
    flux_cutoff: np.ndarray | None
    spectral_radius: np.ndarray
    group_iters: np.ndarray
    group_resid: np.ndarray
    group_converged: np.ndarray
    passes: int


_default_ctx: Context | None = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0, 0)
    return _default_ctx


def compute_flux_tables(tabs: dict, ctx: Context | None = None, verbose: bool = False) -> FluxPerParticle:
    """Run the group loop on the GPU for prepared tables (the drop-in of sn_flux.jl:146-233)."""
    ctx = ctx or default_context()
    pp = PackedProblem(tabs)
    rb = ResultBuffers(pp)
    h = ctx.upload(pp)
    try:
        ctx.solve(h)
        ctx.download(h, rb)
    finally:
        ctx.release(h)
    if verbose:
        for ig in range(tabs["ng"]):
            state = "has converged" if rb.group_converged[ig] else "has not converged"
            print(f">>>Group {ig + 1} {state} ( ϵ = {rb.group_resid[ig]:.4E} , N = {rb.group_iters[ig]} ,"
                  f" ρ = {rb.rho[ig]:.4f} )")
    return FluxPerParticle(rb.flux, rb.flux_cutoff, rb.rho, rb.group_iters, rb.group_resid,
                           rb.group_converged, rb.passes)
