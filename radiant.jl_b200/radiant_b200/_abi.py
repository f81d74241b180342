"""ctypes mirror of include/radiant_b200.h and the loader of the CUDA library.

The product path is libradiant_b200.so (built from csrc/ for sm_100a). There is no CPU
fallback: when the library is missing, loading raises.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libradiant_b200.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)

RB_OK = 0
RB_ERR_INVALID = 1
RB_ERR_UNSUPPORTED = 2
RB_ERR_CUDA = 3
RB_ERR_BUDGET = 4
RB_ERR_TIMEOUT = 5
RB_ERR_NOT_READY = 6
RB_ERR_NOT_FOUND = 7

ACCEL = {"none": 0, "livolant": 1, "anderson": 2, "gmres": 3, "bicgstab": 4}
PRECISION = {"fp64": 0, "mixed": 1}


class RbSnProblem(C.Structure):
    _fields_ = [
        ("ndims", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("dx", _dp), ("dy", _dp), ("dz", _dp),
        ("mat", _ip), ("nmat", C.c_int32), ("bc", C.c_int32 * 6),
        ("nd", C.c_int32), ("mu", _dp), ("eta", _dp), ("xi", _dp),
        ("np", C.c_int32), ("mn", _dp), ("dn", _dp), ("pl", _ip),
        ("np_surf", C.c_int32), ("nd_plus", C.c_int32 * 6),
        ("mn_surf", _dp * 6), ("dn_surf", _dp * 6), ("n_to_nplus", _ip * 6),
        ("order", C.c_int32 * 4), ("nm", C.c_int32 * 5), ("is_fc", C.c_int32),
        ("w_axis", _dp * 4), ("cc", _dp), ("ncc", C.c_int32), ("ww", _dp),
        ("is_adaptive", C.c_int32), ("is_em", C.c_int32),
        ("solver_type", C.c_int32), ("ng", C.c_int32), ("sigma_t", _dp), ("ls", C.c_int32),
        ("sigma_s", _dp), ("s_minus", _dp), ("s_plus", _dp), ("s_mom", _dp), ("t_mom", _dp),
        ("fp", _dp), ("e_width", _dp),
        ("volume_sources", _dp), ("np_source", C.c_int32), ("surface_sources", _dp * 6),
        ("accel", C.c_int32), ("tol", C.c_double), ("max_iter", C.c_int32),
        ("gmres_restart", C.c_int32), ("anderson_depth", C.c_int32),
        ("precision", C.c_int32),
    ]


class RbCoupling(C.Structure):
    _fields_ = [("sigma_s", _dp), ("ls", C.c_int32), ("transfer", _dp), ("moment_map", _ip)]


class RbLaunchRule(C.Structure):
    _fields_ = [("ndims", C.c_int32), ("nd_max", C.c_int32), ("work_max", C.c_int64), ("batch_max", C.c_int32),
                ("cluster", C.c_int32)]


class RbSnResult(C.Structure):
    _fields_ = [
        ("flux", _dp), ("flux_cutoff", _dp), ("rho", _dp), ("group_iters", _ip),
        ("group_resid", _dp), ("group_converged", _ip), ("passes", C.c_int64),
    ]


def _f64(a) -> np.ndarray:
    """Column-major (Fortran-order) float64 copy, the reference's layout."""
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def _i32(a) -> np.ndarray:
    return np.asfortranarray(np.asarray(a, dtype=np.int32))


PINNED_MIN_BYTES = 1 << 20


def pinned_empty(shape, dtype=np.float64, order: str = "F") -> np.ndarray:
    """An uninitialised array in page-locked host memory (rb_host_alloc), given back
    (rb_host_free) when the last view of it is gone."""
    dt = np.dtype(dtype)
    count = int(np.prod(shape))
    if count == 0:
        return np.empty(shape, dtype=dt, order=order)
    lib = load_library()
    p = C.c_void_p()
    if lib.rb_host_alloc(count * dt.itemsize, C.byref(p)) != 0:
        buf = C.create_string_buffer(512)
        lib.rb_last_error(None, buf, 512)
        raise MemoryError(f"rb_host_alloc({count * dt.itemsize} bytes): {buf.value.decode(errors='replace')}")
    buf = (C.c_char * (count * dt.itemsize)).from_address(p.value)
    weakref.finalize(buf, lib.rb_host_free, p.value)
    return np.frombuffer(buf, dtype=dt, count=count).reshape(shape, order=order)


def _pinned_copy(a: np.ndarray) -> np.ndarray:
    if a.nbytes < PINNED_MIN_BYTES:
        return a
    out = pinned_empty(a.shape, a.dtype, "F")
    out[...] = a
    return out


def _ptr(a, kind=_dp):
    if a is None:
        return C.cast(None, kind)
    return a.ctypes.data_as(kind)


class PackedProblem:
    """An rb_sn_problem whose arrays are kept alive by this object. pinned=True puts the arrays
    of PINNED_MIN_BYTES or more in page-locked host memory (the upload's copies then run at the
    host link's speed)."""

    def __init__(self, tables: dict, pinned: bool = False):
        self.t = t = {}

        def f64(a):
            return _pinned_copy(_f64(a)) if pinned else _f64(a)

        def i32(a):
            return _pinned_copy(_i32(a)) if pinned else _i32(a)

        P = RbSnProblem()
        P.ndims = tables["ndims"]
        ns = list(tables["ns"]) + [1] * (3 - len(tables["ns"]))
        P.nx, P.ny, P.nz = ns
        for k, name in enumerate(("dx", "dy", "dz")):
            arr = tables["ds"][k] if k < len(tables["ds"]) else None
            t[name] = None if arr is None else f64(arr)
            setattr(P, name, _ptr(t[name]))
        t["mat"] = i32(tables["mat"])
        P.mat = _ptr(t["mat"], _ip)
        P.nmat = tables["nmat"]
        for f in range(6):
            P.bc[f] = tables["bc"][f] if f < len(tables["bc"]) else 0
        P.nd = tables["nd"]
        for k, name in enumerate(("mu", "eta", "xi")):
            arr = tables["omega"][k] if k < len(tables["omega"]) else None
            t[name] = None if arr is None else f64(arr)
            setattr(P, name, _ptr(t[name]))
        P.np = tables["np"]
        t["mn"], t["dn"], t["pl"] = f64(tables["mn"]), f64(tables["dn"]), i32(tables["pl"])
        P.mn, P.dn, P.pl = _ptr(t["mn"]), _ptr(t["dn"]), _ptr(t["pl"], _ip)
        P.np_surf = tables["np_surf"]
        for f in range(6):
            if f < len(tables["mn_surf"]):
                ms, ds_, nn = f64(tables["mn_surf"][f]), f64(tables["dn_surf"][f]), i32(tables["n_to_nplus"][f])
                t[f"ms{f}"], t[f"ds{f}"], t[f"nn{f}"] = ms, ds_, nn
                P.nd_plus[f] = ms.shape[0]
                P.mn_surf[f], P.dn_surf[f], P.n_to_nplus[f] = _ptr(ms), _ptr(ds_), _ptr(nn, _ip)
            else:
                P.nd_plus[f] = 0
        for a in range(4):
            P.order[a] = tables["order"][a]
            t[f"w{a}"] = f64(tables["w_axis"][a])
            P.w_axis[a] = _ptr(t[f"w{a}"])
        for a in range(5):
            P.nm[a] = tables["nm"][a]
        P.is_fc = int(tables["is_fc"])
        t["cc"], t["ww"] = f64(tables["cc"]), f64(tables["ww"])
        P.cc, P.ncc, P.ww = _ptr(t["cc"]), len(t["cc"]), _ptr(t["ww"])
        P.is_adaptive = int(tables.get("is_adaptive", 0))
        P.is_em = int(tables.get("is_em", 0))
        P.solver_type = tables["solver_type"]
        P.ng = tables["ng"]
        t["sigma_t"], t["sigma_s"] = f64(tables["sigma_t"]), f64(tables["sigma_s"])
        P.sigma_t, P.sigma_s, P.ls = _ptr(t["sigma_t"]), _ptr(t["sigma_s"]), tables["ls"]
        for name in ("s_minus", "s_plus", "s_mom", "t_mom", "fp", "e_width", "volume_sources"):
            arr = tables.get(name)
            t[name] = None if arr is None else f64(arr)
            setattr(P, name, _ptr(t[name]))
        P.np_source = tables["np_source"]
        for f in range(6):
            ss = tables["surface_sources"][f] if f < len(tables["surface_sources"]) else None
            t[f"ss{f}"] = None if ss is None else f64(ss)
            P.surface_sources[f] = _ptr(t[f"ss{f}"])
        P.accel = ACCEL[tables["accel"]] if isinstance(tables["accel"], str) else tables["accel"]
        P.tol = tables["tol"]
        P.max_iter = tables["max_iter"]
        P.gmres_restart = tables["gmres_restart"]
        P.anderson_depth = tables["anderson_depth"]
        P.precision = PRECISION[tables.get("precision", "fp64")] if isinstance(tables.get("precision", "fp64"), str) else tables["precision"]
        self.P = P
        self.tables = tables

    # sizes ---------------------------------------------------------------------------
    @property
    def ncell(self) -> int:
        return int(np.prod(self.tables["ns"]))

    @property
    def flux_shape(self):
        ns = list(self.tables["ns"]) + [1] * (3 - len(self.tables["ns"]))
        return (self.tables["ng"], self.tables["np"], self.tables["nm"][4], *ns)


class ResultBuffers:
    """Caller-owned host buffers of an rb_sn_result (the large ones page-locked when pinned)."""

    def __init__(self, pp: PackedProblem, pinned: bool = False):
        t = pp.tables
        ng = t["ng"]

        def zeros(shape):
            if pinned and int(np.prod(shape)) * 8 >= PINNED_MIN_BYTES:
                a = pinned_empty(shape)
                a[...] = 0.0
                return a
            return np.zeros(shape, order="F")

        self.flux = zeros(pp.flux_shape)
        self.flux_cutoff = zeros(pp.flux_shape[1:]) if t["solver_type"] >= 2 else None
        self.rho = np.zeros(ng)
        self.group_iters = np.zeros(ng, dtype=np.int32)
        self.group_resid = np.zeros(ng)
        self.group_converged = np.zeros(ng, dtype=np.int32)
        R = RbSnResult()
        R.flux = _ptr(self.flux)
        R.flux_cutoff = _ptr(self.flux_cutoff)
        R.rho = _ptr(self.rho)
        R.group_iters = _ptr(self.group_iters, _ip)
        R.group_resid = _ptr(self.group_resid)
        R.group_converged = _ptr(self.group_converged, _ip)
        R.passes = 0
        self.R = R

    @property
    def passes(self) -> int:
        return int(self.R.passes)


# --------------------------------------------------------------------------------------
# the CUDA library
# --------------------------------------------------------------------------------------
_lib = None


def load_library(path: str | None = None):
    """Load libradiant_b200.so and declare its ABI. Raises if it is absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"libradiant_b200.so not built ({p}); run radiant.jl_b200/build.py "
                           "-- there is no CPU fallback for the SN solve")
    lib = C.CDLL(p)
    vp = C.c_void_p
    PP = C.POINTER(RbSnProblem)
    RP = C.POINTER(RbSnResult)
    h64 = C.c_int64
    sig = {
        "rb_create": (C.c_int32, [C.c_int32, C.c_uint64, C.POINTER(vp)]),
        "rb_destroy": (C.c_int32, [vp]),
        "rb_last_error": (C.c_int32, [vp, C.c_char_p, C.c_uint64]),
        "rb_upload": (C.c_int32, [vp, PP, C.POINTER(h64)]),
        "rb_solve": (C.c_int32, [vp, h64, vp]),
        "rb_solve_batch": (C.c_int32, [vp, C.POINTER(h64), C.c_int32, vp]),
        "rb_download": (C.c_int32, [vp, h64, RP]),
        "rb_release": (C.c_int32, [vp, h64]),
        "rb_download_async": (C.c_int32, [vp, h64, RP]),
        "rb_download_wait": (C.c_int32, [vp, h64]),
        "rb_required_bytes": (C.c_int32, [PP, C.POINTER(C.c_uint64)]),
        "rb_compute_flux": (C.c_int32, [C.c_int32, PP, RP]),
        "rb_submit": (C.c_int32, [vp, PP, C.POINTER(h64)]),
        "rb_poll": (C.c_int32, [vp, h64, RP]),
        "rb_energy_deposition": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_int64, C.c_int32, _ip,
                                             _dp, _dp, _dp, _dp, C.c_double, _dp]),
        "rb_transport": (C.c_int32, [C.c_int32, C.c_int32, C.POINTER(PP), C.POINTER(RbCoupling), C.c_int32,
                                     C.c_double, C.c_int32, C.POINTER(_dp), _dp, C.c_double, C.POINTER(RP), _dp,
                                     _ip, _dp]),
        "rb_set_launch_rules": (C.c_int32, [vp, C.POINTER(RbLaunchRule), C.c_int32]),
        "rb_deposition": (C.c_int32, [vp, C.c_int32, C.POINTER(h64), C.POINTER(_dp), _dp, C.c_double, _dp]),
        "rb_upload_sources": (C.c_int32, [vp, PP, vp, C.POINTER(h64), _dp]),
        "rb_host_alloc": (C.c_int32, [C.c_uint64, C.POINTER(vp)]),
        "rb_host_free": (C.c_int32, [vp]),
        "rb_host_register": (C.c_int32, [vp, C.c_uint64]),
        "rb_host_unregister": (C.c_int32, [vp]),
        "rb_version": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


EXPORTED_SYMBOLS = (
    "rb_create", "rb_destroy", "rb_last_error", "rb_upload", "rb_solve", "rb_solve_batch", "rb_download",
    "rb_download_async", "rb_download_wait", "rb_release", "rb_required_bytes", "rb_compute_flux",
    "rb_submit", "rb_poll", "rb_energy_deposition", "rb_transport", "rb_deposition", "rb_set_launch_rules",
    "rb_upload_sources", "rb_host_alloc", "rb_host_free", "rb_host_register", "rb_host_unregister",
    "rb_version",
)


RULES_PATH = os.path.join(_HERE, "launch_rules.json")


def packaged_launch_rules() -> list:
    """The tuning table shipped with the package (empty when there is none)."""
    if not os.path.exists(RULES_PATH):
        return []
    import json

    with open(RULES_PATH) as f:
        return json.load(f)["rules"]


class RadiantError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"radiant_b200 status {status}: {msg}")
        self.status = status


class Context:
    """Owns one rb_context (one device, one HBM budget)."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, launch_rules="packaged"):
        """launch_rules: "packaged" applies the tuning table shipped with the package
        (launch_rules.json, written by radiant_b200.autotune) when present; a list of rule dicts
        applies those; None leaves the built-in shape choice."""
        self.lib = load_library()
        self._ncell = {}  # voxels of each uploaded problem (deposition maps)
        self.h = C.c_void_p()
        st = self.lib.rb_create(device, hbm_budget_bytes, C.byref(self.h))
        if st != RB_OK:
            raise RadiantError(st, self.last_error(None))
        self.launch_rules = []
        if launch_rules == "packaged":
            launch_rules = packaged_launch_rules()
        if launch_rules:
            self.set_launch_rules(launch_rules)

    def set_launch_rules(self, rules):
        """rb_set_launch_rules: rules = [{"ndims", "nd_max", "work_max", "batch_max", "cluster"}, ...]."""
        arr = (RbLaunchRule * max(len(rules), 1))()
        for k, r in enumerate(rules):
            arr[k].ndims, arr[k].nd_max = int(r["ndims"]), int(r["nd_max"])
            arr[k].work_max, arr[k].cluster = int(r["work_max"]), int(r["cluster"])
            arr[k].batch_max = int(r.get("batch_max", 2 ** 31 - 1))
        self.check(self.lib.rb_set_launch_rules(self.h, arr, len(rules)))
        self.launch_rules = [dict(r) for r in rules]

    def last_error(self, h="self") -> str:
        buf = C.create_string_buffer(1024)
        self.lib.rb_last_error(self.h if h == "self" else None, buf, 1024)
        return buf.value.decode(errors="replace")

    def check(self, st: int):
        if st != RB_OK:
            raise RadiantError(st, self.last_error())

    def upload(self, pp: PackedProblem) -> int:
        h = C.c_int64()
        self.check(self.lib.rb_upload(self.h, C.byref(pp.P), C.byref(h)))
        self._ncell[h.value] = int(np.prod(pp.tables["ns"]))
        return h.value

    def upload_sources(self, pp: PackedProblem, sources) -> tuple:
        """rb_upload_sources: the problem with its fixed sources built on the device from
        `sources` (a sources.SourceSet); returns (handle, normalization factors)."""
        h = C.c_int64()
        n = int(sources.S.nvolume + sources.S.nsurface)
        norms = np.zeros(max(n, 1))
        self.check(self.lib.rb_upload_sources(self.h, C.byref(pp.P), C.cast(C.pointer(sources.S), C.c_void_p),
                                              C.byref(h), norms.ctypes.data_as(_dp)))
        self._ncell[h.value] = int(np.prod(pp.tables["ns"]))
        return h.value, norms[:n]

    def solve(self, h: int, stream=None):
        self.check(self.lib.rb_solve(self.h, h, C.c_void_p(stream) if stream else None))

    def solve_batch(self, hs, stream=None):
        arr = (C.c_int64 * len(hs))(*hs)
        self.check(self.lib.rb_solve_batch(self.h, arr, len(hs), C.c_void_p(stream) if stream else None))

    def download(self, h: int, rb: ResultBuffers):
        self.check(self.lib.rb_download(self.h, h, C.byref(rb.R)))

    def download_async(self, h: int, rb: ResultBuffers):
        """rb_download_async: the copies are queued; `rb` must stay alive until download_wait."""
        self.check(self.lib.rb_download_async(self.h, h, C.byref(rb.R)))

    def download_wait(self, h: int):
        self.check(self.lib.rb_download_wait(self.h, h))

    def release(self, h: int):
        self.check(self.lib.rb_release(self.h, h))

    def submit(self, pp: PackedProblem) -> int:
        h = C.c_int64()
        self.check(self.lib.rb_submit(self.h, C.byref(pp.P), C.byref(h)))
        return h.value

    def poll(self, h: int, rb: ResultBuffers) -> bool:
        st = self.lib.rb_poll(self.h, h, C.byref(rb.R))
        if st == RB_ERR_NOT_READY:
            return False
        self.check(st)
        return True

    def deposition(self, handles, sigma_dep, density, norm: float = 1.0) -> np.ndarray:
        """Summed energy (Σe) or charge (Σc) deposition of solved resident problems, on the device
        (rb_deposition); sigma_dep: one [ng+1, nmat] array per handle. Returns [ncell] (x fastest)."""
        n = len(handles)
        sig = [np.asfortranarray(x, dtype=float) for x in sigma_dep]
        rho = np.ascontiguousarray(density, dtype=float)
        arr = (C.c_int64 * n)(*handles)
        ptrs = (_dp * n)(*[_ptr(x) for x in sig])
        out = np.zeros(self._ncell[handles[0]])
        self.check(self.lib.rb_deposition(self.h, n, arr, ptrs, _ptr(rho), float(norm), _ptr(out)))
        return out

    def close(self):
        if self.h:
            self.lib.rb_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
