"""Build recipe of the CPU oracle (test infrastructure): oracle/stencil_oracle.c -> oracle/liboracle.so.

-ffp-contract=off keeps the compiler from fusing anything the reference's nvcc build does not
fuse; the explicit fma()/fmaf() calls in the source are the only fused operations.
-march=x86-64-v3 (AVX2 + FMA) so the library runs on any current x86 host.
"""

from __future__ import annotations

import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "stencil_oracle.c"
LIB_PATH = HERE / "liboracle.so"


def build_oracle(force: bool = False) -> Path:
    if LIB_PATH.exists() and not force and LIB_PATH.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB_PATH
    tmp = str(LIB_PATH) + ".tmp.%d" % os.getpid()
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
           "-std=gnu11", "-shared", "-fPIC", str(SRC), "-o", tmp, "-lm"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + proc.stderr)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build_oracle(force=True))
