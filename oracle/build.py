"""Build the oracle's C restatement into ``oracle/liboracle.so``.

Test infrastructure only: the shared object is loaded by ``oracle`` (the
checker), never by the product package. FMA contraction is disabled so that
floating-point results follow the reference's operation order exactly.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCES = ["cf_laplacian.c", "ichol.c", "foreground.c", "knn.c"]
TARGET = os.path.join(HERE, "liboracle.so")


def build(force=False):
    srcs = [os.path.join(HERE, s) for s in SOURCES]
    if not force and os.path.exists(TARGET):
        t = os.path.getmtime(TARGET)
        if all(os.path.getmtime(s) <= t for s in srcs):
            return TARGET
    cmd = ["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off",
           "-fno-fast-math", "-o", TARGET] + srcs + ["-lm"]
    subprocess.check_call(cmd)
    return TARGET


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
