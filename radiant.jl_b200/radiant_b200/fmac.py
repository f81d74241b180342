"""FMAC-M multigroup cross-section files: reader and writer.

read_fmac_m follows src/cross_sections/read_fmac_m.jl:16-461 (the records it reads, their
order and the derived quantities), write_fmac_m follows src/cross_sections/write_fmac_m.jl:16-377
(the records Radiant.jl writes, in its fixed-column number format). The file is line based:

  line 1            "FMAC-M ..." identification
  lines 2-6         label, integer and character parameters (not used by the reader)
  Record II + 1     40 integers, 6 per line: [1] cumulative groups G, [2] particles, [15]
                    materials, [17] length of Record II + 2, [20] Legendre order + 1
  Record II + 2     the lengths L[i] of the Records III + i (zero: record absent)
  Records III + i   in increasing i where L[i] ≠ 0: 1 title (one line), 2 groups per particle,
                    3 particle names (GAMA / BETA / POSITR), 4 rest energies, 5 energy
                    boundaries, 6 group velocities, 11/12 transition bounds, 14 scattering moment
                    counts, 15 total, 16 absorption, 35 boundary stopping powers, 36 momentum
                    transfer, 37 energy deposition, 38 charge deposition
  then              per (particle out j, group gf, particle in i, group gi): 3 + Nmat integers
                    (global gi, global gf, −(L_eff+1) or 0 per material, value count) and the
                    Legendre moments of every material's transfer (one 0.0 for a zero transfer)

Numbers are 12-column fields, 6 per line: integers right-aligned, reals as a sign column, a
7-character mantissa, 'E', the exponent's sign and 2 exponent digits. Line numbers count blank
lines too (the label record is two blank lines).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .sn_flux import MultigroupXS

NAMES = {"GAMA": "photon", "BETA": "electron", "POSITR": "positron"}
CODES = {v: k for k, v in NAMES.items()}
CHARGE = {"photon": 0.0, "electron": -1.0, "positron": 1.0}


@dataclass
class FmacLibrary:
    """What read_fmac_m stores in a Cross_Sections object, per particle (file order)."""
    particles: list                 # "photon" / "electron" / "positron"
    ng: list                        # groups per particle
    legendre_order: int
    nmat: int
    title: str = ""
    e_bounds: list = field(default_factory=list)     # [ng+1] per particle, highest first
    total: list = field(default_factory=list)        # [ng, nmat]
    absorption: list = field(default_factory=list)   # [ng, nmat] (zero when the record is absent)
    stopping: list = field(default_factory=list)     # [ng+1, nmat] at the group boundaries
    momentum: list = field(default_factory=list)     # [ng, nmat]
    edep: list = field(default_factory=list)         # [ng+1, nmat], last row: the cutoff term
    cdep: list = field(default_factory=list)         # [ng+1, nmat], last row: the cutoff term
    scattering: dict = field(default_factory=dict)   # (n_in, m_out) -> [nmat, ng_n, ng_m, L+1]

    def index(self, particle: str) -> int:
        if particle not in self.particles:
            raise ValueError("Cross-sections don't contain data for the given particle.")
        return self.particles.index(particle)

    def get_scattering(self, p_in: str, p_out: str, L: int) -> np.ndarray:
        """get_scattering(particle_in, particle_out, L) (Cross_Sections.jl:928-942): zero-padded or
        truncated to L+1 moments."""
        s = self.scattering[(self.index(p_in), self.index(p_out))]
        out = np.zeros(s.shape[:3] + (L + 1,))
        k = min(L + 1, s.shape[3])
        out[..., :k] = s[..., :k]
        return out

    def multigroup(self, particle: str, density) -> MultigroupXS:
        """The particle's tables in the getters' shapes (Cross_Sections.jl:817-1105)."""
        n = self.index(particle)
        eb = np.asarray(self.e_bounds[n], dtype=float)
        charged = particle != "photon"
        return MultigroupXS(sigma_t=self.total[n].copy(), sigma_s=self.scattering[(n, n)].copy(),
                            sigma_a=self.absorption[n].copy(), sb=self.stopping[n].copy() if charged else None,
                            t_mom=self.momentum[n].copy() if charged else None, sigma_e=self.edep[n].copy(),
                            e_width=eb[:-1] - eb[1:], energies=(eb[:-1] + eb[1:]) / 2, e_bounds=eb,
                            density=np.asarray(density, dtype=float))


# ------------------------------------------------------------------------------------------
# number fields
# ------------------------------------------------------------------------------------------
def _one_space(line: str) -> str:
    """Leading blanks removed and runs of blanks collapsed to one (src/tools/one_space.jl:13-31)."""
    out = []
    prev_space = True
    for ch in line:
        if ch.isspace():
            if not prev_space:
                out.append(ch)
            prev_space = True
        else:
            out.append(ch)
            prev_space = False
    return "".join(out)


def _floats(line: str, count: int) -> list:
    """`count` 12-column reals of a line after blank collapsing (read_fmac_m.jl:426-461): a '+'
    is put in front when the line does not start with '-', then each field is sign, 7-character
    mantissa, 'E', exponent sign and two digits."""
    if not line.startswith("-"):
        line = "+" + line
    vals = []
    for i in range(count):
        f = line[12 * i:12 * i + 12]
        sign = -1.0 if f[0] == "-" else 1.0
        mant = sign * float(f[1:8])
        esign = -1.0 if f[9] == "-" else 1.0
        expo = esign * float(f[10:12])
        vals.append(mant * 10.0 ** expo)
    return vals


def _fmt_int(i: int) -> str:
    s = str(int(i))
    return " " * (12 - len(s)) + s


def _fmt_float(x: float) -> str:
    """write_fmac_m.jl:270-303: six significant digits in 12 columns."""
    x = float(x)
    sng = "-" if x < 0 else " "
    e = math.floor(math.log10(abs(x))) if x != 0 else 0
    sng_e = "-" if e < 0 else "+"
    mant = abs(x) / 10.0 ** e
    e = abs(e)
    if e < 10:
        es = "0" + str(e)
    elif e < 99:
        es = str(e)
    else:  # an exponent beyond two digits is written as zero
        es, mant, sng = "00", 0.0, " "
    ms = _julia_round5(mant)
    pad = 7 - len(ms)
    return sng + ms + ("0" * pad if pad > 0 else "") + "E" + sng_e + es


def _julia_round5(m: float) -> str:
    """string(round(m; digits=5)) for 0 ≤ m < 10.5: shortest repr of the rounded double."""
    r = round(m, 5)
    s = repr(float(r))
    if "e" in s or "E" in s:  # tiny mantissas do not occur: m ≥ 1 or m == 0
        s = f"{r:.5f}".rstrip("0")
    return s


def _lines_of(values, fmt) -> list:
    out, cur = [], ""
    for k, v in enumerate(values):
        cur += fmt(v)
        if (k + 1) % 6 == 0:
            out.append(cur)
            cur = ""
    if cur:
        out.append(cur)
    return out


# ------------------------------------------------------------------------------------------
# writer
# ------------------------------------------------------------------------------------------
def write_fmac_m(lib: FmacLibrary, path: str) -> None:
    """write_fmac_m.jl:16-236: the records Radiant.jl writes (title, groups, names, boundaries,
    total, stopping powers, momentum transfer, energy and charge deposition, scattering)."""
    npart, nmat, L = len(lib.particles), lib.nmat, lib.legendre_order
    G = int(sum(lib.ng))
    out = ["FMAC-M                       5", "", ""]
    v0 = [0] * 10
    v0[0] = 1
    out += _lines_of(v0, _fmt_int)
    out.append("NGCAP")
    v1 = [0] * 40
    v1[0], v1[1], v1[14], v1[16], v1[19] = G, npart, nmat, 38, L + 1
    out += _lines_of(v1, _fmt_int)
    v2 = [0] * 38
    v2[0], v2[1], v2[2], v2[4] = 12, npart, npart, G + npart
    v2[14], v2[34], v2[35], v2[36], v2[37] = G * nmat, (G + npart) * nmat, G * nmat, G * nmat, G * nmat
    out += _lines_of(v2, _fmt_int)
    out.append("Coupled multigroup cross-sections produced with Radiant.jl")
    out += _lines_of(lib.ng, _fmt_int)
    out.append("".join(CODES[p] + "  " for p in lib.particles))
    mesh = [v for i in range(npart) for v in lib.e_bounds[i][:-1]]
    mesh += [lib.e_bounds[npart - 1 - i][-1] for i in range(npart)]
    out += _lines_of(mesh, _fmt_float)
    out += _lines_of([lib.total[i][g, n] for i in range(npart) for g in range(lib.ng[i]) for n in range(nmat)],
                     _fmt_float)
    sp = [lib.stopping[i][g, n] for i in range(npart) for g in range(lib.ng[i]) for n in range(nmat)]
    sp += [lib.stopping[npart - 1 - i][-1, n] for i in range(npart) for n in range(nmat)]
    out += _lines_of(sp, _fmt_float)
    for arr in (lib.momentum, lib.edep, lib.cdep):
        out += _lines_of([arr[i][g, n] for i in range(npart) for g in range(lib.ng[i]) for n in range(nmat)],
                         _fmt_float)
    off = np.concatenate([[0], np.cumsum(lib.ng)]).astype(int)
    for j in range(npart):
        for gf in range(lib.ng[j]):
            for i in range(npart):
                dcs = lib.get_scattering(lib.particles[i], lib.particles[j], L)
                for gi in range(lib.ng[i]):
                    p = [0] * (3 + nmat)
                    p[0], p[1] = off[i] + gi + 1, off[j] + gf + 1
                    vals = []
                    for n in range(nmat):
                        row = dcs[n, gi, gf, :]
                        if not np.any(row != 0.0):
                            p[2 + n] = 0
                            p[-1] += 1
                            vals.append(0.0)
                        else:
                            leff = max(l for l in range(L + 1) if row[l] != 0.0)
                            p[2 + n] = -(leff + 1)
                            p[-1] += leff + 1
                            vals += list(row[:leff + 1])
                    out += _lines_of(p, _fmt_int)
                    out += _lines_of(vals, _fmt_float)
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


# ------------------------------------------------------------------------------------------
# reader
# ------------------------------------------------------------------------------------------
def read_fmac_m(path: str, particles=None) -> FmacLibrary:
    """read_fmac_m.jl:16-316. `particles` (names) keeps those of the file's particles, in the
    file's order (None: all). The energy-deposition and charge-deposition tables get the
    reference's cutoff row: S(E_cut)·E_cut/ΔE_G and S(E_cut)·(−q)/ΔE_G (read_fmac_m.jl:335-337)."""
    with open(path) as f:
        raw = f.read().split("\n")
    if raw and raw[-1] == "":
        raw = raw[:-1]
    lines = [_one_space(r) for r in raw]
    if not lines or lines[0][:6] != "FMAC-M":
        raise ValueError("The file is not a FMAC-M format file.")
    k = 6  # 0-based index of the first line of Record II + 1 (line 7)
    P = []
    for li in range(k, k + 7):
        P += [int(x) for x in lines[li].split()]
    G, npart, nmat, n2, L = P[0], P[1], P[14], P[16], P[19] - 1
    k += 7
    Lrec = []
    nl2 = math.ceil(n2 / 6)
    for li in range(k, k + nl2):
        Lrec += [int(x) for x in lines[li].split()]
    k += nl2
    rec = {}
    title, names = "", []
    for i, li_len in enumerate(Lrec, start=1):
        if li_len == 0:
            continue
        if i in (1, 3):  # one line each
            if i == 1:
                title = lines[k]
            else:
                names = lines[k].split()
            k += 1
            continue
        nlin = math.ceil(li_len / 6)
        if i in (2, 11, 12, 14):
            vals = []
            for li in range(k, k + nlin):
                vals += [int(x) for x in lines[li].split()]
        else:
            vals = []
            for q, li in enumerate(range(k, k + nlin)):
                cnt = 6 if q < nlin - 1 else (li_len % 6 or 6)
                vals += _floats(lines[li], cnt)
        rec[i] = vals
        k += nlin
    ng = [int(v) for v in rec[2]]
    off = np.concatenate([[0], np.cumsum(ng)]).astype(int)

    def per_group(i):  # [G·nmat] g-major -> per particle [ng, nmat]
        a = np.asarray(rec[i]).reshape(G, nmat) if i in rec else np.zeros((G, nmat))
        return [a[off[n]:off[n + 1]].copy() for n in range(npart)]

    # energy boundaries: each particle's upper boundaries, then the cutoffs in reversed order
    eb_t = rec.get(5, [])
    e_bounds = [np.array(list(eb_t[off[n]:off[n + 1]]) + [eb_t[len(eb_t) - 1 - n]]) for n in range(npart)]
    total, absorption, momentum = per_group(15), per_group(16), per_group(36)
    ed, cd = per_group(37), per_group(38)
    sp_t = np.asarray(rec.get(35, np.zeros((G + npart) * nmat)))
    stopping = []
    for n in range(npart):
        s = np.zeros((ng[n] + 1, nmat))
        s[:ng[n]] = sp_t[off[n] * nmat:(off[n] + ng[n]) * nmat].reshape(ng[n], nmat)
        s[ng[n]] = sp_t[len(sp_t) - (n + 1) * nmat:len(sp_t) - n * nmat]
        stopping.append(s)
    # scattering records: integers (global gi, global gf, −(L_eff+1) or 0 per material, count),
    # then the values
    scat_in = {}
    while k < len(lines):
        if lines[k] == "":
            k += 1
            continue
        nl_i = math.ceil((3 + nmat) / 6)
        p = []
        for li in range(k, k + nl_i):
            p += [int(x) for x in lines[li].split()]
        k += nl_i
        cnt = p[2 + nmat]
        nl_f = math.ceil(cnt / 6)
        vals = []
        for q, li in enumerate(range(k, k + nl_f)):
            vals += _floats(lines[li], 6 if q < nl_f - 1 else (cnt % 6 or 6))
        k += nl_f
        pos = 0
        for n in range(nmat):
            sz = abs(p[2 + n])
            scat_in[(n, p[1], p[0])] = vals[pos:pos + sz]
            pos += sz if sz else 1
    file_parts = [NAMES[nm] for nm in names[:npart]]
    lib = FmacLibrary(particles=file_parts, ng=ng, legendre_order=L, nmat=nmat, title=title)
    for n in range(npart):
        eb = e_bounds[n]
        dE = eb[-2] - eb[-1]
        cut = stopping[n][-1]
        lib.e_bounds.append(eb)
        lib.total.append(total[n])
        lib.absorption.append(absorption[n])
        lib.stopping.append(stopping[n])
        lib.momentum.append(momentum[n])
        lib.edep.append(np.vstack([ed[n], cut * eb[-1] / dE]))
        lib.cdep.append(np.vstack([cd[n], cut * (-CHARGE[file_parts[n]]) / dE]))
        for m in range(npart):
            s = np.zeros((nmat, ng[n], ng[m], L + 1))
            for mat in range(nmat):
                for gi in range(ng[n]):
                    for gf in range(ng[m]):
                        v = scat_in.get((mat, off[m] + gf + 1, off[n] + gi + 1))
                        if v:
                            s[mat, gi, gf, :len(v)] = v
            lib.scattering[(n, m)] = s
    if particles is not None:
        keep = [i for i, p in enumerate(lib.particles) if p in set(particles)]
        lib = _subset(lib, keep)
    return lib


def _subset(lib: FmacLibrary, keep: list) -> FmacLibrary:
    out = FmacLibrary(particles=[lib.particles[i] for i in keep], ng=[lib.ng[i] for i in keep],
                      legendre_order=lib.legendre_order, nmat=lib.nmat, title=lib.title)
    for a in ("e_bounds", "total", "absorption", "stopping", "momentum", "edep", "cdep"):
        setattr(out, a, [getattr(lib, a)[i] for i in keep])
    out.scattering = {(a, b): lib.scattering[(keep[a], keep[b])] for a in range(len(keep)) for b in range(len(keep))}
    return out
