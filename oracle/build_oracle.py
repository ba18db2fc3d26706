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
# The CPU-baseline build: same source and operation order without the
# per-operation volatile stores, so the compiler may vectorise across outputs
# (contraction and reassociation stay off).  Used only for timing.
LIB_TIMING = os.path.join(OUT_DIR, "libcg3m_oracle_timing.so")
SRC = os.path.join(HERE, "cg3m_oracle.c")


def _build_one(out, extra, force):
    if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(SRC):
        return out
    cmd = [
        os.environ.get("CC", "gcc"), "-std=c11", "-ffp-contract=off", "-fno-fast-math",
        "-fno-builtin-fmaf", "-fPIC", "-shared", "-o", out, SRC, "-lm",
    ] + extra
    subprocess.check_call(cmd)
    return out


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    _build_one(LIB_TIMING, ["-O3", "-DORACLE_TIMING_BUILD"], force)
    return _build_one(LIB, ["-O2"], force)


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
