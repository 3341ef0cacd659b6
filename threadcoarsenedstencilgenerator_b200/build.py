"""Build step for the engine's native library (in-tree, sm_100a).

Produces ``threadcoarsenedstencilgenerator_b200/libtcs.so``: the C ABI of ``include/tcs.h``,
compiled by nvcc with the static CUDA runtime and linked against NVRTC.  The device header
``csrc/tcs_kernels.cuh`` is embedded into the library as a string (the NVRTC instantiation
source) and is also compiled once by nvcc for sm_100a as a syntax/resource check.

Run ``python -m threadcoarsenedstencilgenerator_b200.build`` (or ``__graft_entry__.build()``).
"""

from __future__ import annotations

import hashlib
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = ROOT / "_build"
LIB = PKG / "libtcs.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

HOST_SOURCES = ["tcs_capi.cpp"]
# NVRTC is linked statically (its symbols kept private): a process that already loaded another
# libnvrtc.so.12 (PyTorch ships one) would otherwise hand the library that NVRTC, whose version
# changes both the generated code and the cubin cache keys.
CUDA_LIB = Path("/usr/local/cuda/lib64")
NVRTC_STATIC = [str(CUDA_LIB / "libnvrtc_static.a"), str(CUDA_LIB / "libnvrtc-builtins_static.a"),
                str(CUDA_LIB / "libnvptxcompiler_static.a")]
CUDA_SOURCES: list[str] = ["tcs_field.cu", "tcs_mlp.cu", "tcs_tc.cu"]  # AOT device code compiled straight into libtcs.so


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(
            "command failed (%d): %s\n%s\n%s" % (proc.returncode, " ".join(cmd), proc.stdout, proc.stderr)
        )


DEVICE_HEADERS = [("tcs_kernels.cuh", "tcs_kernels_src"), ("tcs_tile.cuh", "tcs_tile_src")]


def _embed_kernel_source() -> Path:
    """Write the NVRTC instantiation sources (device headers) as C++ raw string literals."""
    BUILD.mkdir(exist_ok=True)
    text = ""
    for fname, var in DEVICE_HEADERS:
        src = (CSRC / fname).read_text()
        if ")TCSSRC" in src:
            raise RuntimeError("kernel source contains the raw-string delimiter")
        text += "static const char " + var + '[] = R"TCSSRC(' + src + ')TCSSRC";\n'
    inc = BUILD / "tcs_kernels_src.inc"
    if not inc.exists() or inc.read_text() != text:
        inc.write_text(text)
    return inc


def _inputs_digest() -> str:
    h = hashlib.sha256()
    files = [CSRC / f for f, _ in DEVICE_HEADERS] + [INCLUDE / "tcs.h", Path(__file__), CSRC / "tcs_field.h"]
    files += [CSRC / f for f in HOST_SOURCES + CUDA_SOURCES]
    for f in sorted(files):
        h.update(f.name.encode())
        h.update(f.read_bytes())
    return h.hexdigest()


def check_kernel_header() -> None:
    """Compile the device header for sm_100a with nvcc (one representative parameter set)."""
    BUILD.mkdir(exist_ok=True)
    probe = BUILD / "tcs_kernels_check.cu"
    probe.write_text(
        "#define TCS_T double\n#define TCS_DIM 3\n#define TCS_SHAPE 1\n#define TCS_ORIENT 0\n"
        "#define TCS_COEFF 1\n#define TCS_R 4\n#define TCS_CX 2\n#define TCS_CY 2\n#define TCS_CZ 1\n"
        '#include "tcs_kernels.cuh"\n'
    )
    _run(
        [NVCC, *ARCH, "-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-I", str(CSRC), "-c",
         str(probe), "-o", str(BUILD / "tcs_kernels_check.o")]
    )
    # the pipelined sweep and its batched form (3D Star Jacobi r2, 2x2 coarsening, block 16x4)
    for name, extra in (("pipe", ""), ("batch", "#define TCS_BATCH 1\n")):
        probe = BUILD / ("tcs_kernels_check_%s.cu" % name)
        probe.write_text(
            "#define TCS_T double\n#define TCS_DIM 3\n#define TCS_SHAPE 1\n#define TCS_ORIENT 0\n"
            "#define TCS_COEFF 0\n#define TCS_R 2\n#define TCS_CX 2\n#define TCS_CY 2\n#define TCS_CZ 2\n"
            "#define TCS_PIPE 1\n#define TCS_BX 16\n#define TCS_BY 4\n#define TCS_CH 5\n#define TCS_LSHIFT 0\n"
            + extra + '#include "tcs_kernels.cuh"\n'
        )
        _run(
            [NVCC, *ARCH, "-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-I", str(CSRC), "-c",
             str(probe), "-o", str(BUILD / ("tcs_kernels_check_%s.o" % name))]
        )


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile libtcs.so in-tree if its inputs changed; return its path."""
    stamp = BUILD / "libtcs.stamp"
    digest = _inputs_digest()
    if LIB.exists() and stamp.exists() and stamp.read_text() == digest and not force:
        return LIB
    _embed_kernel_source()
    check_kernel_header()
    srcs = [str(CSRC / f) for f in HOST_SOURCES + CUDA_SOURCES]
    cmd = [
        NVCC, *ARCH, "-std=c++17", "-O3", "-lineinfo", "-shared", "-Xcompiler", "-fPIC",
        "-Xcompiler", "-Wall", "-cudart", "static", "-I", str(INCLUDE), "-I", str(BUILD),
        "-I", str(CSRC), *srcs, "-o", str(LIB) + ".tmp", *NVRTC_STATIC, "-Xlinker", "--exclude-libs,ALL", "-ldl", "-lpthread", "-lrt",
        "-Xlinker", "-rpath=/usr/local/cuda/lib64",
    ]
    if verbose:
        print(" ".join(cmd))
    _run(cmd)
    os.replace(str(LIB) + ".tmp", LIB)
    stamp.write_text(digest)
    return LIB


if __name__ == "__main__":
    path = build(force="--force" in sys.argv, verbose=True)
    print(path)
