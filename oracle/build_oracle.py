"""Builds the oracle (test infrastructure): oracle/_build/liboracle_sn.so from sn_oracle.c.

Plain gcc, FP64, no fast-math and no FMA contraction, so the restatement keeps the
reference's operation order. Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg load the result.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build", "liboracle_sn.so")


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "sn_oracle.c")
    hdr = os.path.join(HERE, "..", "include", "radiant_b200.h")
    if (not force and os.path.exists(OUT)
            and os.path.getmtime(OUT) >= max(os.path.getmtime(src), os.path.getmtime(hdr))):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["gcc", "-O2", "-std=gnu99", "-fPIC", "-shared", "-pthread", "-ffp-contract=off", "-fno-fast-math",
           "-Wall", "-Wno-unused-function", src, "-o", OUT, "-lm"]
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
