"""Recipe: build the reference's own generated kernels into oracle/_ref/ (test infrastructure).

For every parameter set of ``ref_configs.ALL`` this runs the reference's generators straight from
the read-only reference tree (cuda/generate2DStencil_cuda.py, cuda/generate3DStencil_cuda.py,
cuda/generateLaunchUpdateGrid.py), writes their output (``kernels.cu``, ``launchUpdateGrid.cu``)
to ``oracle/_ref/<key>/`` and compiles it with ``ref_driver.cu`` into ``oracle/_ref/<key>/libref.so``.

The shipped 3D generator does not run: a comment line in it is not indented under its ``for``
loop (cuda/generate3DStencil_cuda.py:294-295, IndentationError).  The recipe feeds the interpreter
that file's text with that single line re-indented (whitespace only, in memory; nothing of the
reference is copied into the repository).

Compilation uses ``-arch=sm_100a`` (``--shipped`` also builds the reference Makefile's flags: no
-arch, no -O, i.e. default-target SASS + PTX that the driver JIT-compiles on B200).  Both builds
keep nvcc's default -fmad=true, as the reference does.  Nothing here reads the reference at run
time: the GPU box only loads the built ``libref.so`` files.
"""

from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
# The reference tree is named by TCS_REFERENCE_ROOT (or --reference-root): no default, so nothing
# here reads a fixed path; without it the recipe builds nothing.
REF_ROOT = Path(os.environ["TCS_REFERENCE_ROOT"]) if os.environ.get("TCS_REFERENCE_ROOT") else None
REF_CUDA = REF_ROOT / "cuda" if REF_ROOT else None
OUT = HERE / "_ref"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

sys.path.insert(0, str(HERE.parent))
from oracle.ref_configs import ALL, key  # noqa: E402


def set_reference_root(path) -> None:
    """Point the recipe at a reference tree (what TCS_REFERENCE_ROOT does)."""
    global REF_ROOT, REF_CUDA
    REF_ROOT = Path(path)
    REF_CUDA = REF_ROOT / "cuda"


def reference_available() -> bool:
    return REF_CUDA is not None and (REF_CUDA / "generate2DStencil_cuda.py").exists()


def _generator_text(dim: int) -> str:
    path = REF_CUDA / ("generate%dDStencil_cuda.py" % dim)
    text = path.read_text()
    if dim == 3:
        lines = text.split("\n")
        for i, ln in enumerate(lines):
            # the one mis-indented line: directly after `for z in range(0, zCoarsening, 1):`
            if ln.strip().startswith('content += "\\t\\t//slice z = {0}\\n".format(z)') and i > 0 and \
                    lines[i - 1].strip() == "for z in range(0, zCoarsening, 1):":
                lead = len(lines[i - 1]) - len(lines[i - 1].lstrip())
                if len(ln) - len(ln.lstrip()) <= lead:
                    lines[i] = " " * (lead + 4) + ln.lstrip()
        text = "\n".join(lines)
    return text


def _run_generator(text: str, args: list[str], name: str) -> str:
    proc = subprocess.run([sys.executable, "-", *args], input=text, capture_output=True, text=True,
                          cwd=str(REF_CUDA))
    if proc.returncode != 0:
        raise RuntimeError("%s %s failed:\n%s" % (name, " ".join(args), proc.stderr))
    return proc.stdout


def generate(cfg, dest: Path) -> None:
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    dest.mkdir(parents=True, exist_ok=True)
    gargs = [sh, o, c, str(r), str(cx), str(cy)] + ([str(cz)] if d == 3 else [])
    if al != "None":
        gargs += [al, str(cl)]
    kernels = _run_generator(_generator_text(d), gargs, "generate%dDStencil_cuda.py" % d)
    largs = [sh, c, str(r), "%dD" % d] + ([al] if al != "None" else [])
    launcher = _run_generator((REF_CUDA / "generateLaunchUpdateGrid.py").read_text(), largs,
                              "generateLaunchUpdateGrid.py")
    (dest / "kernels.cu").write_text(kernels)
    (dest / "launchUpdateGrid.cu").write_text(launcher)


def compile_one(cfg, shipped: bool = False) -> Path:
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    dest = OUT / key(cfg)
    generate(cfg, dest)
    lib = dest / ("libref_shipped.so" if shipped else "libref.so")
    flags = [] if shipped else ["-gencode", "arch=compute_100a,code=sm_100a", "-O3"]
    cmd = [NVCC, *flags, "-shared", "-Xcompiler", "-fPIC", "-DREF_DIM=%d" % d,
           "-DREF_ALIGNED=%d" % (0 if al == "None" else 1), "-I", str(dest), "-I", str(REF_CUDA),
           str(HERE / "ref_driver.cu"), "-o", str(lib)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s" % (key(cfg), proc.stderr[-4000:]))
    return lib


SHAPES = {"Box": 0, "Star": 1}
ORIENTS = {"Row": 0, "Column": 1}
COEFFS = {"Jacobi": 0, "Variable": 1}
ALIGNS = {"None": 0, "Read": 1, "Write": 2}


def build_shim_bench(cfg) -> Path:
    """Link the reference's unmodified host program (cuda/main.cpp, cuda/benchmark.cpp,
    cuda/primes.cpp) against the engine through launch_update_grid_shim.cpp: the reference's
    `bench` binary for one parameter set, running on libtcs.so.  Output: oracle/_ref/<key>/bench_tcs."""
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    dest = OUT / key(cfg)
    dest.mkdir(parents=True, exist_ok=True)
    pkg = HERE.parent / "threadcoarsenedstencilgenerator_b200"
    exe = dest / "bench_tcs"
    defs = ["-DTCS_SHIM_DIM=%d" % d, "-DTCS_SHIM_SHAPE=%d" % SHAPES[sh], "-DTCS_SHIM_ORIENT=%d" % ORIENTS[o],
            "-DTCS_SHIM_COEFF=%d" % COEFFS[c], "-DTCS_SHIM_R=%d" % r, "-DTCS_SHIM_CX=%d" % cx,
            "-DTCS_SHIM_CY=%d" % cy, "-DTCS_SHIM_CZ=%d" % (cz if d == 3 else 1), "-DTCS_SHIM_ALIGN=%d" % ALIGNS[al],
            "-DTCS_SHIM_CL=%d" % cl]
    rel = "$ORIGIN/../../../threadcoarsenedstencilgenerator_b200"
    cmd = [NVCC, "-O2", *defs, "-I", str(HERE.parent / "include"), "-I", str(REF_CUDA),
           str(REF_CUDA / "main.cpp"), str(REF_CUDA / "benchmark.cpp"), str(REF_CUDA / "primes.cpp"),
           str(pkg / "csrc" / "launch_update_grid_shim.cpp"), "-L", str(pkg), "-ltcs",
           "-Xlinker", "-rpath=" + rel, "-o", str(exe)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("shim bench link failed for %s:\n%s" % (key(cfg), proc.stderr[-4000:]))
    return exe


SHIM_CONFIGS = [
    (2, "Box", "Row", "Jacobi", 1, 1, 1, 1, "None", 0),
    (3, "Star", "Row", "Variable", 4, 2, 2, 1, "Read", 16),
]


def build_ref(configs=None, shipped: bool = False, jobs: int = 8) -> list:
    if not reference_available():
        return []
    configs = list(configs or ALL)
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        libs = list(ex.map(lambda c: compile_one(c, shipped), configs))
    return libs


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--shipped", action="store_true", help="also build with the reference Makefile flags")
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("--reference-root", help="the reference tree (default: $TCS_REFERENCE_ROOT)")
    a = ap.parse_args()
    if a.reference_root:
        set_reference_root(a.reference_root)
    if not reference_available():
        print("reference tree not found at %s; nothing built" % REF_ROOT)
        sys.exit(0)
    libs = build_ref(shipped=False, jobs=a.j)
    if a.shipped:
        libs += build_ref(shipped=True, jobs=a.j)
    libs += [build_shim_bench(c) for c in SHIM_CONFIGS]
    print("built %d reference libraries under %s" % (len(libs), OUT))
