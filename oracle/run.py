"""Thin ctypes wrapper around the oracle library (test infrastructure only)."""
import ctypes as C

from .build_oracle import build

_lib = None


def lib():
    global _lib
    if _lib is None:
        from radiant_b200._abi import RbSnProblem, RbSnResult

        _lib = C.CDLL(build())
        _lib.oracle_compute_flux.argtypes = [C.POINTER(RbSnProblem), C.POINTER(RbSnResult)]
        _lib.oracle_compute_flux.restype = C.c_int
    return _lib


def solve(tables):
    """Run the oracle on prepared tables; returns the filled ResultBuffers."""
    from radiant_b200._abi import PackedProblem, ResultBuffers

    pp = PackedProblem(tables)
    rb = ResultBuffers(pp)
    st = lib().oracle_compute_flux(C.byref(pp.P), C.byref(rb.R))
    if st != 0:
        raise RuntimeError(f"oracle status {st}")
    return rb


def transport(parts, couplings, ngen_max=50, eps_gen=1e-6, conv_type=0, sigma_dep=None, density=None, norm=1.0,
              deposition=False):
    """oracle_transport on prepared tables of several particles; ``couplings[(i, j)]`` as in
    radiant_b200.transport; conv_type 0/1/2 = flux / energy / charge deposition criterion.
    Returns (ResultBuffers per particle, generations, eps), plus the summed deposition of the final
    fluxes when ``deposition``."""
    import numpy as np

    from radiant_b200._abi import PackedProblem, ResultBuffers, RbCoupling, RbSnProblem, RbSnResult
    from radiant_b200.transport import _CouplingPack, _DepPack

    L = lib()
    if not getattr(L, "_transport_declared", False):
        dp = C.POINTER(C.c_double)
        L.oracle_transport.argtypes = [C.c_int32, C.POINTER(C.POINTER(RbSnProblem)), C.POINTER(RbCoupling),
                                       C.c_int32, C.c_double, C.c_int32, C.POINTER(dp), dp, C.c_double,
                                       C.POINTER(C.POINTER(RbSnResult)), dp, C.POINTER(C.c_int32),
                                       C.POINTER(C.c_double)]
        L.oracle_transport.restype = C.c_int
        L._transport_declared = True
    packs = [PackedProblem(t) for t in parts]
    res = [ResultBuffers(p) for p in packs]
    n = len(parts)
    probs = (C.POINTER(RbSnProblem) * n)(*[C.pointer(p.P) for p in packs])
    results = (C.POINTER(RbSnResult) * n)(*[C.pointer(r.R) for r in res])
    cp = _CouplingPack(n, couplings)
    dpk = _DepPack(sigma_dep) if sigma_dep is not None else None
    rho = np.ascontiguousarray(density, dtype=float) if density is not None else None
    dep = np.zeros(int(np.prod(parts[0]["ns"]))) if deposition else None
    ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None
    ngen = C.c_int32(0)
    eps = C.c_double(0.0)
    st = L.oracle_transport(n, probs, cp.arr, int(ngen_max), float(eps_gen), int(conv_type),
                            dpk.arr if dpk else None, ptr(rho), float(norm), results, ptr(dep), C.byref(ngen),
                            C.byref(eps))
    if st != 0:
        raise RuntimeError(f"oracle status {st}")
    if deposition:
        return res, int(ngen.value), float(eps.value), dep
    return res, int(ngen.value), float(eps.value)


def sources(ndims, ng, ns, widths, positions, source_set, nps):
    """oracle_sources: (volume sources [ng, ncell] or None, per-face surface sources [ng, nps, face
    cells] for the faces beams enter, normalization factors) of an rb_source_set's definitions."""
    import numpy as np

    L = lib()
    dp = C.POINTER(C.c_double)
    S = source_set.S
    ns3 = [int(v) for v in ns] + [1] * (3 - len(ns))
    ncell = int(np.prod(ns3))
    w = [np.ascontiguousarray(widths[a], dtype=np.float64) for a in range(ndims)]
    p = [np.ascontiguousarray(positions[a], dtype=np.float64) for a in range(ndims)]
    nsa = (C.c_int32 * 3)(*ns3)
    wa = (dp * 3)(*[w[a].ctypes.data_as(dp) if a < ndims else None for a in range(3)])
    pa = (dp * 3)(*[p[a].ctypes.data_as(dp) if a < ndims else None for a in range(3)])
    vol = np.zeros((ng, ncell), order="F") if S.nvolume else None
    faces = [None] * 6
    for k in range(S.nsurface):
        f = source_set.beams[k].face
        ax = [a for a in range(ndims) if a != f // 2]
        ncf = int(np.prod([ns3[a] for a in ax])) if ax else 1
        if faces[f] is None:
            faces[f] = np.zeros((ng, nps, ncf), order="F")
    fa = (dp * 6)(*[a.ctypes.data_as(dp) if a is not None else None for a in faces])
    basis = np.concatenate(source_set.bases) if source_set.bases else np.zeros(1)
    norms = np.zeros(max(1, S.nvolume + S.nsurface))
    L.oracle_sources.restype = C.c_int
    st = L.oracle_sources(C.c_int32(ndims), nsa, wa, pa, C.c_int32(ng), C.c_int32(nps), C.c_int32(S.nvolume),
                          C.cast(S.volume, C.c_void_p), C.c_int32(S.nsurface), C.cast(S.surface, C.c_void_p),
                          basis.ctypes.data_as(dp), vol.ctypes.data_as(dp) if vol is not None else None, fa,
                          norms.ctypes.data_as(dp))
    if st != 0:
        raise ValueError("oracle_sources: bad definitions")
    return vol, faces, norms[:S.nvolume + S.nsurface]
