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
