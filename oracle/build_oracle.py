"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``cg3m_oracle.c`` into ``oracle/_build/libcg3m_oracle.so`` with every
floating-point operation kept separate (``-ffp-contract=off``, no fast-math).

The reference implementation itself (Ascend C for the Atlas 950PR, built by the
CANN ``bisheng`` toolchain against an ops-blas tree that is not shipped) cannot be
compiled here, so there is no ``oracle/_ref`` build: the C restatement in this
directory is the oracle.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libcg3m_oracle.so")
SRC = os.path.join(HERE, "cg3m_oracle.c")


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = [
        os.environ.get("CC", "gcc"), "-O2", "-std=c11", "-ffp-contract=off", "-fno-fast-math",
        "-fno-builtin-fmaf", "-fPIC", "-shared", "-o", LIB, SRC, "-lm",
    ]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
