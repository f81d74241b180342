"""Coupled transport of several SN particles: transport() on the GPU (rb_transport).

The generation loop of transport.jl:21-147 runs in the library: every particle's problem, its
accumulated particle source and its running total flux stay on the device, each solve is
followed by the sources it produces for the other particles (device kernels), and only the
summed fluxes come back. This module builds what the library needs for each pair of particles
(the reference builds them inside particle_source, particle_source.jl:23-77): the group-transfer
cross sections Σs(i→j), the angular transfer matrix between the two bases and the map between
their cell moments.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import sphere as S
from . import tables as T
from ._abi import (PackedProblem, RadiantError, RB_OK, RbCoupling, RbSnProblem, RbSnResult, ResultBuffers,
                   _dp, _ip, _ptr, load_library)
from .sn_flux import FluxPerParticle

CONV_TYPES = {"flux": 0, "energy-deposition": 1, "charge-deposition": 2}


def moments_to_directions(pl, pm, Om, Qdims: int) -> np.ndarray:
    """M [Nd, P] rebuilding the angular flux at directions Om from its moments
    (particle_source.jl:196-220): Legendre in 1D angular domains, real spherical harmonics else."""
    P = len(pl)
    Nd = len(Om[0])
    Lmax = int(max(pl))
    M = np.zeros((Nd, P))
    if Qdims == 1:
        for n in range(Nd):
            Pl = T.legendre_polynomials_up_to_L(Lmax, float(Om[0][n]))
            for p in range(P):
                if pm[p] == 0:
                    M[n, p] = (2 * pl[p] + 1) / 2 * Pl[pl[p]]
    else:
        for n in range(Nd):
            Rlm = S.real_spherical_harmonics_up_to_L(Lmax, float(Om[0][n]), math.atan2(Om[2][n], Om[1][n]))
            for p in range(P):
                M[n, p] = (2 * pl[p] + 1) / (4 * math.pi) * Rlm[pl[p]][pl[p] + pm[p]]
    return M


def _same_quadrature(a: dict, b: dict) -> bool:
    return (a["btype"] == b["btype"] and a["qdims"] == b["qdims"] and len(a["w"]) == len(b["w"])
            and np.array_equal(a["w"], b["w"])
            and all(np.array_equal(np.asarray(a["omega"][k]), np.asarray(b["omega"][k])) for k in range(3)))


def angular_transfer_matrix(tabs_in: dict, tabs_out: dict) -> np.ndarray:
    """T [P_out, P_in] (particle_source.jl:239-257): for two SN bases on different quadratures
    (or closures), Dn_out · M(pl_in, pm_in, Ω_out); on the same one, the identity over the
    moments with equal (l, m)."""
    if not _same_quadrature(tabs_in, tabs_out):
        M = moments_to_directions(list(tabs_in["pl"]), list(tabs_in["pm"]), tabs_out["omega"], tabs_out["qdims"])
        return np.asarray(tabs_out["dn"], dtype=float) @ M
    Tm = np.zeros((tabs_out["np"], tabs_in["np"]))
    index_in = {}
    for p in range(tabs_in["np"]):
        index_in[(int(tabs_in["pl"][p]), int(tabs_in["pm"][p]))] = p
    for q in range(tabs_out["np"]):
        p = index_in.get((int(tabs_out["pl"][q]), int(tabs_out["pm"][q])))
        if p is not None:
            Tm[q, p] = 1.0
    return Tm


def _moment_index(o, ix, iy, iz, iE, fc: bool):
    if fc:
        return o[1] * o[0] * o[3] * (iz - 1) + o[0] * o[3] * (iy - 1) + o[3] * (ix - 1) + iE
    high = [ix > 1, iy > 1, iz > 1, iE > 1]
    if sum(high) > 1:
        return None
    i = 1 + (iE - 1) + (ix - 1) + (iy - 1) + (iz - 1)
    if ix > 1:
        i += o[3] - 1
    if iy > 1:
        i += o[3] - 1 + o[0] - 1
    if iz > 1:
        i += o[3] - 1 + o[0] - 1 + o[1] - 1
    return i


def map_moments(oi, of, fc_in: bool, fc_out: bool) -> np.ndarray:
    """map [Nm_out]: the 1-based incoming cell moment feeding each outgoing one, 0 = none
    (map_moments.jl:21-57)."""
    oi = [int(v) for v in oi]
    of = [int(v) for v in of]
    M = {}
    for ix in range(1, oi[0] + 1):
        for iy in range(1, oi[1] + 1):
            for iz in range(1, oi[2] + 1):
                for iE in range(1, oi[3] + 1):
                    i = _moment_index(oi, ix, iy, iz, iE, fc_in)
                    if i is not None:
                        M[(ix, iy, iz, iE)] = i
    nmf = int(np.prod(of)) if fc_out else 1 + sum(v - 1 for v in of)
    mp = np.zeros(nmf, dtype=np.int32)
    for ix in range(1, of[0] + 1):
        for iy in range(1, of[1] + 1):
            for iz in range(1, of[2] + 1):
                for iE in range(1, of[3] + 1):
                    i = _moment_index(of, ix, iy, iz, iE, fc_out)
                    if i is None:
                        continue
                    if ix <= oi[0] and iy <= oi[1] and iz <= oi[2] and iE <= oi[3]:
                        mp[i - 1] = M.get((ix, iy, iz, iE), 0)
    return mp


@dataclass
class Coupling:
    """What particle_source needs for one pair (particle i into particle j)."""
    sigma_s: np.ndarray     # [nmat, ng_i, ng_j, ls+1]
    transfer: np.ndarray    # [np_j, np_i]
    moment_map: np.ndarray  # [nm5_j] int32

    @property
    def ls(self) -> int:
        return self.sigma_s.shape[3] - 1


def build_coupling(tabs_in: dict, tabs_out: dict, sigma_s: np.ndarray) -> Coupling:
    """The coupling of particle `tabs_in` into `tabs_out`. `sigma_s` [nmat, ng_in, ng_out, L+1]
    is get_scattering(particle_in, particle_out, maximum(pl_in)) (particle_source.jl:49); its
    orders above maximum(pl_in) are dropped."""
    ls = int(np.max(tabs_in["pl"]))
    ss = np.asarray(sigma_s, dtype=float)
    if ss.shape[3] < ls + 1:
        raise ValueError(f"coupling cross sections carry order {ss.shape[3] - 1} < {ls}")
    ss = np.asfortranarray(ss[:, :, :, :ls + 1])
    return Coupling(ss, np.asfortranarray(angular_transfer_matrix(tabs_in, tabs_out)),
                    map_moments(tabs_in["order"], tabs_out["order"], bool(tabs_in["is_fc"]), bool(tabs_out["is_fc"])))


class _CouplingPack:
    """rb_coupling array [npart * npart] with the host arrays it points to kept alive."""

    def __init__(self, npart: int, couplings: dict):
        self.arr = (RbCoupling * (npart * npart))()
        self.keep = []
        for (i, j), c in couplings.items():
            if i == j:
                continue
            e = self.arr[i * npart + j]
            ss = np.asfortranarray(c.sigma_s, dtype=float)
            tm = np.asfortranarray(c.transfer, dtype=float)
            mp = np.ascontiguousarray(c.moment_map, dtype=np.int32)
            self.keep += [ss, tm, mp]
            e.sigma_s = _ptr(ss)
            e.ls = c.ls
            e.transfer = _ptr(tm)
            e.moment_map = _ptr(mp, _ip)


@dataclass
class TransportResult:
    fluxes: list            # FluxPerParticle per particle (fluxes summed over the generations)
    generations: int
    eps: float              # the last generation's ϵ (NaN after one generation)
    deposition: np.ndarray | None = None  # summed deposition of the final fluxes [ncell], if asked


class _DepPack:
    """sigma_dep pointer array (one [ng+1, nmat] table per particle) with its arrays kept alive."""

    def __init__(self, sigma_dep):
        self.keep = [np.asfortranarray(x, dtype=float) for x in sigma_dep]
        self.arr = (_dp * len(self.keep))(*[_ptr(x) for x in self.keep])


def transport_tables(parts: list, couplings: dict, ngen_max: int = 50, eps_gen: float = 1e-6,
                     conv_type: str = "flux", device: int = 0, sigma_dep=None, density=None, norm: float = 1.0,
                     deposition: bool = False) -> TransportResult:
    """transport() (transport.jl:21-147) for particles given as prepared tables on one geometry.

    ``couplings[(i, j)]`` is the Coupling of particle i into j (build_coupling). The
    "energy-deposition" and "charge-deposition" criteria need ``sigma_dep`` (one [ng+1, nmat]
    table per particle: Σe or Σc), ``density`` [nmat] and ``norm`` (the sources' normalization
    factor); with ``deposition`` the summed deposition of the final fluxes comes back too."""
    if conv_type not in CONV_TYPES:
        raise ValueError("Unknown convergence type.")
    lib = load_library()
    packs = [PackedProblem(t) for t in parts]
    res = [ResultBuffers(p) for p in packs]
    n = len(parts)
    probs = (C.POINTER(RbSnProblem) * n)(*[C.pointer(p.P) for p in packs])
    results = (C.POINTER(RbSnResult) * n)(*[C.pointer(r.R) for r in res])
    cp = _CouplingPack(n, couplings)
    dp = _DepPack(sigma_dep) if sigma_dep is not None else None
    rho = np.ascontiguousarray(density, dtype=float) if density is not None else None
    dep = np.zeros(int(np.prod(parts[0]["ns"]))) if deposition else None
    ngen = C.c_int32(0)
    eps = C.c_double(0.0)
    st = lib.rb_transport(device, n, probs, cp.arr, int(ngen_max), float(eps_gen), CONV_TYPES[conv_type],
                          dp.arr if dp else None, _ptr(rho), float(norm), results, _ptr(dep), C.byref(ngen),
                          C.byref(eps))
    if st != RB_OK:
        buf = C.create_string_buffer(1024)
        lib.rb_last_error(None, buf, 1024)
        raise RadiantError(st, buf.value.decode(errors="replace"))
    out = [FluxPerParticle(r.flux, r.flux_cutoff, r.rho, r.group_iters, r.group_resid, r.group_converged, r.passes)
           for r in res]
    return TransportResult(out, int(ngen.value), float(eps.value), dep)
