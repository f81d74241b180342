"""Shared test set-up: import paths, the gpu marker, the oracle loader.

`-m "not gpu"` runs the oracle against analytic known answers, the host table builders and
the ABI surface of the library (no compute call). `-m gpu` runs the CUDA library against the
oracle on the same inputs.
"""
import ctypes as C
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "radiant.jl_b200"))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libradiant_b200.so")


@pytest.fixture(scope="session")
def oracle():
    """The C oracle (test infrastructure): oracle_compute_flux(problem, result)."""
    from oracle.build_oracle import build
    from radiant_b200._abi import RbSnProblem, RbSnResult

    lib = C.CDLL(build())
    lib.oracle_compute_flux.argtypes = [C.POINTER(RbSnProblem), C.POINTER(RbSnResult)]
    lib.oracle_compute_flux.restype = C.c_int
    return lib


@pytest.fixture(scope="session")
def gpu_ctx():
    import torch  # noqa: F401  (device memory and streams come from the library itself)
    from radiant_b200._abi import Context

    ctx = Context(0, 0)
    yield ctx
    ctx.close()
