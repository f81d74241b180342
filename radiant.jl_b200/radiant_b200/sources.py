"""Fixed sources of an SN solve: Radiant's Volume_Source and Surface_Source
(src/structures/Volume_Source.jl, Surface_Source.jl), the dense arrays the reference builds from
them on the host, and the definitions rb_upload_sources builds the same arrays from on the device.

- ``VolumeSource`` / ``SurfaceSource``: the fields the reference reads (energy group 1-based,
  intensity, boundaries per axis, direction and location of a beam, Legendre order 64 unless set).
- ``beam_basis``: the half-range basis values of a beam's direction in the order of the surface
  moments (surface_source.jl:103 in 1D with Qdims 1, :137/:195/:284 otherwise).
- ``dense_sources``: volume_source.jl:21-122 and the SN branch of surface_source.jl:22-330,
  added source after source as Source.add_source does (Source.jl:129-203): the volume sources
  [ng,1,1,nx,ny,nz], the per-face surface sources [ng, Np, face cells] and each source's
  normalization factor. This is the host path (arrays handed to rb_upload).
- ``SourceSet``: the same definitions as an rb_source_set (rb_upload_sources).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import tables as T

FACES = ("X-", "X+", "Y-", "Y+", "Z-", "Z+")


@dataclass
class VolumeSource:
    energy_group: int                       # 1-based
    boundaries: dict                        # {"x": (lo, hi), "y": ..., "z": ...}
    intensity: float = 1.0


@dataclass
class SurfaceSource:
    energy_group: int                       # 1-based
    location: str                           # "X-", "X+", "Y-", "Y+", "Z-", "Z+"
    direction: tuple                        # (mu, eta, xi)
    boundaries: dict = field(default_factory=dict)  # in-plane axes of the face (2D/3D)
    intensity: float = 1.0
    legendre_order: int = 64


def positions_of(widths) -> np.ndarray:
    """Voxel centres along one axis from its widths, the axis starting at 0
    (particle_transport/geometry.jl:33-49)."""
    x = np.zeros(len(widths))
    xp = 0.0
    for i, d in enumerate(np.asarray(widths, dtype=float)):
        xp += d
        x[i] = xp - d / 2
    return x


def beam_basis(sn, ndims: int, s: SurfaceSource):
    """(values[Np], pl, pm) of the beam's half-range basis (surface_source.jl:36-45 for the basis,
    :103 / :137 / :195 / :284 for the values)."""
    from .sphere import real_half_range_spherical_harmonics_up_to_L, surface_basis_sphere_face

    L = min(s.legendre_order, sn.legendre_order)
    Qdims = sn.qdims(ndims)
    Om, w = T.quadrature(sn.quadrature_order, sn.quadrature_type, ndims, Qdims)
    if Qdims == 1:
        Om = [np.asarray(Om), 0 * np.asarray(Om), 0 * np.asarray(Om)]
    mus, etas, xis = (float(v) for v in s.direction)
    if ndims == 1 and Qdims == 1:
        Np, _, _, _, _, pl, pm = T.surface_angular_polynomial_basis_face(Om, w, L, sn.angular_boltzmann, 1, s.location)
        Pls = T.half_range_legendre_polynomials_up_to_L(int(np.max(pl)), abs(mus))
        return np.array([Pls[pl[p]] for p in range(Np)]), pl, pm
    Np, _, _, _, _, pl, pm = surface_basis_sphere_face(Om, w, L, sn.angular_boltzmann, Qdims, s.location)
    ps = real_half_range_spherical_harmonics_up_to_L(int(np.max(pl)), abs(mus), math.atan2(xis, etas))
    return np.array([ps[pl[p]][pl[p] + pm[p]] for p in range(Np)]), pl, pm


def _enters(s: SurfaceSource) -> bool:
    f = FACES.index(s.location.upper())
    c = float(s.direction[f // 2])
    return c > 0 if f % 2 == 0 else c < 0


def _face_axes(ndims: int, f: int):
    return [a for a in range(ndims) if a != f // 2]


def dense_sources(sn, ndims: int, ng: int, ns, widths, positions, volume=(), surface=()):
    """The reference's host arrays of the given sources: (volume sources [ng,1,1,nx,ny,nz] or
    None, surface sources [ng, Np, face cells] per face (None for a face no beam enters: the
    reference's zeros), normalization factors [volume sources..., surface sources...])."""
    ns = [int(v) for v in ns] + [1] * (3 - len(ns))
    norms = []
    vol = None
    if volume:
        vol = np.zeros((ng, 1, 1, *ns), order="F")
    for v in volume:
        Q = np.zeros((ng, 1, 1, *ns), order="F")
        norm = 0.0
        g = v.energy_group - 1
        box = [v.boundaries.get(k, (-math.inf, math.inf)) for k in "xyz"]
        for ix in range(ns[0]):
            if not (box[0][0] <= positions[0][ix] <= box[0][1]):
                continue
            for iy in range(ns[1]):
                if ndims >= 2 and not (box[1][0] <= positions[1][iy] <= box[1][1]):
                    continue
                for iz in range(ns[2]):
                    if ndims >= 3 and not (box[2][0] <= positions[2][iz] <= box[2][1]):
                        continue
                    Q[g, 0, 0, ix, iy, iz] += v.intensity
                    term = v.intensity * widths[0][ix]
                    if ndims >= 2:
                        term = term * widths[1][iy]
                    if ndims >= 3:
                        term = term * widths[2][iz]
                    norm = norm + term
        vol[:, 0, 0] += Q[:, 0, 0]
        norms.append(norm)
    surf = None
    if surface:
        bases = [beam_basis(sn, ndims, s)[0] for s in surface]
        npmax = max(1, max(len(b) for b in bases))
        surf = [None] * (2 * ndims)
        for s in surface:
            f = FACES.index(s.location.upper())
            ax = _face_axes(ndims, f)
            ncf = int(np.prod([ns[a] for a in ax])) if ax else 1
            surf[f] = np.zeros((ng, npmax, ncf))
        for s, basis in zip(surface, bases):
            f = FACES.index(s.location.upper())
            ax = _face_axes(ndims, f)
            g = s.energy_group - 1
            Qn = np.zeros_like(surf[f])
            norm = 0.0
            if ndims == 1:
                norm = s.intensity
                if _enters(s):
                    for p in range(len(basis)):
                        Qn[g, p, 0] = s.intensity * basis[p]
            else:
                a = ax[0]
                c = ax[1] if len(ax) > 1 else None
                lo = {k: s.boundaries.get("xyz"[k], (-math.inf, math.inf)) for k in ax}
                for ia in range(ns[a]):
                    if positions[a][ia] < lo[a][0] or positions[a][ia] > lo[a][1]:
                        continue
                    for ic in range(ns[c] if c is not None else 1):
                        if c is not None and (positions[c][ic] < lo[c][0] or positions[c][ic] > lo[c][1]):
                            continue
                        cell = ia + (ns[a] * ic if c is not None else 0)
                        if _enters(s):
                            for p in range(len(basis)):
                                q = s.intensity * basis[p] * widths[a][ia]
                                if c is not None:
                                    q = q * widths[c][ic]
                                Qn[g, p, cell] = q
                        area = s.intensity * widths[a][ia]
                        if c is not None:
                            area = area * widths[c][ic]
                        norm += area
            surf[f] += Qn
            norms.append(norm)
    return vol, surf, norms


# ---- the C ABI form ------------------------------------------------------------------------------
class RbVolumeBox(C.Structure):
    _fields_ = [("energy_group", C.c_int32), ("reserved", C.c_int32), ("intensity", C.c_double),
                ("lo", C.c_double * 3), ("hi", C.c_double * 3)]


class RbSurfaceBeam(C.Structure):
    _fields_ = [("energy_group", C.c_int32), ("face", C.c_int32), ("intensity", C.c_double),
                ("direction", C.c_double * 3), ("lo", C.c_double * 3), ("hi", C.c_double * 3),
                ("basis", C.POINTER(C.c_double))]


class RbSourceSet(C.Structure):
    _fields_ = [("position", C.POINTER(C.c_double) * 3), ("nvolume", C.c_int32), ("nsurface", C.c_int32),
                ("volume", C.POINTER(RbVolumeBox)), ("surface", C.POINTER(RbSurfaceBeam))]


class SourceSet:
    """An rb_source_set of the given definitions, its arrays kept alive by this object.
    ``np_source`` is the number of surface moments the solve reads: min(Np_surf, the largest
    beam basis), the value the dense path's arrays give."""

    def __init__(self, sn, ndims: int, positions, volume=(), surface=(), np_surf: int | None = None):
        self.positions = [np.ascontiguousarray(p, dtype=np.float64) for p in positions[:ndims]]
        bases = [beam_basis(sn, ndims, s)[0] for s in surface]
        npmax = max([len(b) for b in bases] + [1]) if bases else 0
        self.np_source = min(np_surf, npmax) if np_surf else npmax
        self.bases = []
        for b in bases:
            arr = np.zeros(self.np_source)
            k = min(len(b), self.np_source)
            arr[:k] = b[:k]
            self.bases.append(arr)
        S = RbSourceSet()
        for a in range(3):
            S.position[a] = self.positions[a].ctypes.data_as(C.POINTER(C.c_double)) if a < ndims else None
        self.boxes = (RbVolumeBox * max(1, len(volume)))()
        for k, v in enumerate(volume):
            self.boxes[k].energy_group = v.energy_group
            self.boxes[k].intensity = v.intensity
            for a, key in enumerate("xyz"):
                lo, hi = v.boundaries.get(key, (-math.inf, math.inf))
                self.boxes[k].lo[a], self.boxes[k].hi[a] = lo, hi
        self.beams = (RbSurfaceBeam * max(1, len(surface)))()
        for k, s in enumerate(surface):
            B = self.beams[k]
            B.energy_group = s.energy_group
            B.face = FACES.index(s.location.upper())
            B.intensity = s.intensity
            for a, key in enumerate("xyz"):
                B.direction[a] = float(s.direction[a])
                lo, hi = s.boundaries.get(key, (-math.inf, math.inf))
                B.lo[a], B.hi[a] = lo, hi
            B.basis = self.bases[k].ctypes.data_as(C.POINTER(C.c_double))
        S.nvolume, S.nsurface = len(volume), len(surface)
        S.volume = self.boxes if volume else None
        S.surface = self.beams if surface else None
        self.S = S
