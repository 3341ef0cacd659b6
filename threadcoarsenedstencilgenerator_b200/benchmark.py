"""Port of the reference's benchmark host (`stencilBenchmark`, cuda/benchmark.h:18-124,
cuda/benchmark.cpp) on top of the engine.

Same flow — initGPU, initBenchmark (isotropic 1/S mask, maxPotentialBlockSize, geometry,
two buffers, init pattern), run (exhaustive block-shape sweep through benchmarkUpdateGrid) or
singleRun, printResults — and the same TSV report, so scripts that parse the reference's output
keep working.  torch only owns the two device buffers.
"""

from __future__ import annotations

import math
import sys

from . import _lib
from .launch import LaunchUpdateGrid
from .primes import block_shapes
from .spec import StencilSpec


class StencilBenchmark:
    def __init__(self, neighbourhood: str, dimension: int, alignment: str, cl_size: int, coeff_type: str,
                 orientation: str, stencil_range: int, coarsening, grid_size, max_time: float,
                 precision: str = "f64", mask=None):
        coarsening = tuple(coarsening) + (1,) * (3 - len(coarsening))
        grid_size = tuple(grid_size) + (1,) * (3 - len(grid_size))
        if any(g == 0 for g in grid_size[:dimension]):
            raise ValueError("Grid dimensions have to be greater than zero!")
        if max_time < 0:
            raise ValueError("Time for iterations must be non-negative: %r" % max_time)
        self.spec = StencilSpec(dimension=dimension, neighbourhood=neighbourhood, orientation=orientation,
                                coefficients=coeff_type, range=stencil_range, cx=coarsening[0], cy=coarsening[1],
                                cz=coarsening[2], alignment=alignment, cl_size=cl_size, precision=precision)
        self.grid_size_in = grid_size
        self.max_time = float(max_time)
        self.user_mask = mask
        self.bench_results: list = []
        self.launcher: LaunchUpdateGrid | None = None
        self.stream = None

    # stencilBenchmark::initGPU (cuda/benchmark.cpp:96-118)
    def init_gpu(self, device: int = 0) -> None:
        import torch

        if not torch.cuda.is_available():
            raise _lib.TcsError(_lib.TCS_ERR_NO_DEVICE, "No gpu found, exiting.")
        torch.cuda.set_device(device)
        props = torch.cuda.get_device_properties(device)
        self.gpu_name = props.name
        self.warp_size = 32
        self.max_threads = (1024, 1024, 64)

    # stencilBenchmark::initBenchmark (cuda/benchmark.cpp:120-220)
    def init_benchmark(self) -> None:
        import torch

        spec = self.spec
        self.launcher = LaunchUpdateGrid(spec)
        S = spec.stencil_size
        if spec.coefficients == "Variable":
            mask = self.user_mask if self.user_mask is not None else [1.0 / S] * S
            self.launcher.copyMask(mask, S)
        self.max_threads_per_block = self.launcher.maxPotentialBlockSize()
        nx, ny, nz = self.grid_size_in
        self.geom = spec.geometry(nx, ny, nz)
        dtype = torch.float64 if spec.precision == "f64" else torch.float32
        free, total = torch.cuda.mem_get_info()
        need = 2 * spec.itemsize * self.geom.n_points
        if need > free:
            raise MemoryError("Requested grid size is too big for the GPU (needed/free/total: %d / %d / %d)"
                              % (need, free, total))
        self.d_array0 = torch.zeros(self.geom.shape, dtype=dtype, device="cuda")
        self.d_array1 = torch.zeros(self.geom.shape, dtype=dtype, device="cuda")
        g = self.geom.grid
        if spec.dimension == 2:
            ib = (32, 16, 1)
            ig = (math.ceil(g[0] / ib[0]), math.ceil(g[1] / ib[1]), 1)
        else:
            ib = (16, 16, 4)
            ig = (math.ceil(g[0] / ib[0]), math.ceil(g[1] / ib[1]), math.ceil(g[2] / ib[2]))
        self.launcher.launchInit(g, ib, ig, self.d_array0, self.geom.right_offset)
        self.launcher.launchInit(g, ib, ig, self.d_array1, self.geom.right_offset)
        torch.cuda.synchronize()

    def _grid_blocks(self, block) -> tuple:
        t = self.geom.threads
        gb = [math.ceil(t[i] / block[i]) for i in range(3)]
        if self.spec.dimension == 2:
            gb[2] = 1
        return tuple(gb)

    def _bench_one(self, block) -> None:
        spec = self.spec
        try:
            durations = self.launcher.benchmarkUpdateGrid(
                spec.coefficients, spec.neighbourhood, spec.range, spec.dimension, spec.alignment, self.max_time,
                self.geom.grid, block, self._grid_blocks(block), self.d_array0, self.d_array1,
                self.geom.right_offset)
            self.bench_results.append((durations, tuple(block)))
        except _lib.TcsError:
            print("kernel failed for blockSize: %d\t%d\t%d" % tuple(block), file=sys.stderr)

    # stencilBenchmark::run -> Benchmark2D/Benchmark3D (cuda/benchmark.cpp:208-216,223-251,287-318)
    def run(self) -> None:
        for block in block_shapes(self.spec.dimension, self.max_threads_per_block, self.warp_size,
                                  self.max_threads):
            self._bench_one(block)

    # stencilBenchmark::singleRun (cuda/benchmark.cpp:253-283,320-351)
    def single_run(self, xthreads: int, ythreads: int, zthreads: int = 1) -> None:
        block = (xthreads, ythreads, zthreads if self.spec.dimension == 3 else 1)
        if any(b == 0 for b in block):
            raise ValueError("One of the dimensions of the requested threadblock is 0 %r." % (block,))
        if any(block[i] > self.max_threads[i] for i in range(3)):
            raise ValueError("Requested threadblock dimensions %r bigger than maximal possible %r."
                             % (block, self.max_threads))
        if block[0] * block[1] * block[2] > self.max_threads_per_block:
            raise ValueError("Threadblock %r is too big. Maximum threads per block are %d threads for this kernel."
                             % (block, self.max_threads_per_block))
        self._bench_one(block)

    # stencilBenchmark::printResults (cuda/benchmark.cpp:354-428)
    def results_tsv(self) -> str:
        spec = self.spec
        e = self.geom.elements
        lines = ["#GPU: %s" % self.gpu_name]
        grid_line = "#grid size excluding border: x %d y %d" % (e[0], e[1])
        coarse_line = "#coarsening factors: x %d y %d" % (spec.cx, spec.cy)
        if spec.dimension == 3:
            grid_line += " z %d" % e[2]
            coarse_line += " z %d" % spec.cz
        lines += [grid_line, coarse_line, "#alignment: %s" % spec.alignment]
        if spec.alignment != "None":
            lines.append("#aligned to %d byte" % (spec.cl_size * spec.itemsize))
        lines += ["#orientation: %s" % spec.orientation, "#coefficients: %s" % spec.coefficients,
                  "#neighbourhood: %s" % spec.neighbourhood, "#range: %d" % spec.range,
                  "#dimension: %d" % spec.dimension,
                  "#xthreads\tythreads\tzthreads\tPerf [Flop/s]\tPerf dev [Flop/s]\tPerf [Lup/s]\t"
                  "Perf dev [Lup/s]\titerations\ttotal time[s]"]
        updated = float(self.geom.interior_points)
        flops_per_update = spec.flops_per_update
        for durations, block in self.bench_results:
            if not durations:
                continue
            lups = [updated / t for t in durations]
            mean_lups = sum(lups) / len(lups)
            mean_flops = sum(l * flops_per_update for l in lups) / len(lups)
            sd_lups = math.sqrt(sum((l - mean_lups) ** 2 for l in lups) / len(lups))
            zcol = str(block[2]) if spec.dimension == 3 else "0"
            lines.append("%d\t%d\t%s\t%e\t%e\t%e\t%e\t%d\t%e" % (
                block[0], block[1], zcol, mean_flops, flops_per_update * sd_lups, mean_lups, sd_lups,
                len(durations), sum(durations)))
        return "\n".join(lines) + "\n"

    def print_results(self, file=None) -> None:
        (file or sys.stdout).write(self.results_tsv())
