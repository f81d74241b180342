"""The C-ABI library loads, exports every entry point include/radiant_b200.h declares, and
rejects bad descriptions on the host (no device call is made here)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from radiant_b200 import workloads as W
from radiant_b200._abi import PackedProblem, load_library

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "radiant_b200.h")


def declared_symbols():
    with open(HDR) as f:
        src = f.read()
    return sorted(set(re.findall(r"RB_API\s+[\w\s\*]+?\b(rb_\w+)\s*\(", src)))


def test_header_declares_the_abi():
    syms = declared_symbols()
    for s in ("rb_create", "rb_upload", "rb_solve", "rb_download", "rb_compute_flux", "rb_submit", "rb_poll",
              "rb_last_error"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    lib = load_library()
    for s in declared_symbols():
        assert hasattr(lib, s), s


def _required(tabs):
    lib = load_library()
    pp = PackedProblem(tabs)
    b = C.c_uint64()
    st = lib.rb_required_bytes(C.byref(pp.P), C.byref(b))
    buf = C.create_string_buffer(512)
    lib.rb_last_error(None, buf, 512)
    return st, b.value, buf.value.decode()


def test_required_bytes_of_configs():
    st, b, _ = _required(W.c1_tables(seed=1))
    assert st == 0 and 1 << 20 < b < 8 << 20
    st, b, _ = _required(W.c2_tables(seed=1))
    assert st == 0 and b > 16 << 20


def test_rejects_bad_material_id():
    t = W.c1_tables(seed=1)
    t["mat"] = t["mat"].copy()
    t["mat"].flat[5] = 7
    st, _, msg = _required(t)
    assert st == 1 and "mat[5]=7" in msg


def test_rejects_inconsistent_moments():
    t = W.c1_tables(seed=1)
    t["nm"] = list(t["nm"])
    t["nm"][4] = 3
    st, _, msg = _required(t)
    assert st == 1 and "nm[4]" in msg


def test_rejects_adaptive_and_em():
    for key in ("is_adaptive", "is_em"):
        t = W.c1_tables(seed=1)
        t[key] = 1
        st, _, _ = _required(t)
        assert st == 2


def test_rejects_oversized_restart():
    t = W.c1_tables(seed=1)
    t["gmres_restart"] = 1000
    st, _, msg = _required(t)
    assert st == 1 and "gmres_restart" in msg


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        load_library(str(tmp_path / "nope.so"))


def test_launch_rule_struct_and_table_shape():
    """The launch-rule struct mirrors rb_launch_rule, and the packaged table (when present) holds
    rules the library accepts: dimension 1-3, power-of-two teams up to 16, increasing work."""
    import ctypes as C
    from radiant_b200._abi import RbLaunchRule, packaged_launch_rules
    assert C.sizeof(RbLaunchRule) == 24
    rules = packaged_launch_rules()
    for r in rules:
        assert r["ndims"] in (1, 2, 3) and r["cluster"] in (1, 2, 4, 8, 16) and r["nd_max"] > 0
    keys = [(r["batch_max"], r["work_max"]) for r in rules]
    assert keys == sorted(keys)


def test_ctypes_mirrors_match_the_header_layout(tmp_path):
    """Every struct of the header has the size and field offsets of its ctypes mirror: the C
    compiler's layout (gcc on the header itself) against ctypes'."""
    import shutil
    import subprocess

    from radiant_b200 import _abi as A
    from radiant_b200 import sources as S

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    mirrors = {"rb_sn_problem": A.RbSnProblem, "rb_sn_result": A.RbSnResult, "rb_coupling": A.RbCoupling,
               "rb_launch_rule": A.RbLaunchRule, "rb_volume_box": S.RbVolumeBox,
               "rb_surface_beam": S.RbSurfaceBeam, "rb_source_set": S.RbSourceSet}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HDR}"', 'int main(void) {']
    for cname, py in mirrors.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.check_call([cc, "-std=c99", "-o", str(exe), str(src)])
    got = {}
    for line in subprocess.check_output([str(exe)], text=True).splitlines():
        cname, what, val = line.split()
        got[(cname, what)] = int(val)
    for cname, py in mirrors.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
