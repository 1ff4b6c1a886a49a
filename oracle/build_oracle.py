"""Build the C half of the oracle (``sx_oracle.c``) into ``oracle/_build``.

TEST INFRASTRUCTURE ONLY: the library is the checker and the CPU baseline,
never part of the product path.
"""

from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
SRC = os.path.join(HERE, "sx_oracle.c")
LIB = os.path.join(OUT_DIR, "libsx_oracle.so")


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    tmp = LIB + f".{os.getpid()}.tmp"
    cmd = ["gcc", "-O3", "-std=c11", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
           "-fPIC", "-shared", SRC, "-o", tmp, "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
