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
