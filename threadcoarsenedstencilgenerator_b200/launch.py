"""The reference's host interface `launchUpdateGrid.h`, bound to one parameter set.

The reference generates ``launchUpdateGrid.cu`` per parameter set; its four functions
(cuda/launchUpdateGrid.h:13-18) then act on the kernels baked into ``kernels.cu``.
``LaunchUpdateGrid`` is that generated file for one ``StencilSpec``: the same four entry
points, the same argument meaning (gridSize is the padded grid, blockSize/gridBlocks the launch
shape, rightOffset the row padding) and the same error behaviour (a runtime parameter that does
not match the baked-in set raises ``CudaErrorInvalidValue``, the reference's
``throw cudaErrorInvalidValue``).
"""

from __future__ import annotations

from .spec import StencilSpec
from .stencil import Stencil


class LaunchUpdateGrid:
    def __init__(self, spec: StencilSpec, stencil: Stencil | None = None):
        self.spec = spec
        self.stencil = stencil or Stencil(spec)

    # std::vector<double> benchmarkUpdateGrid(...)   cuda/generateLaunchUpdateGrid.py:103-147
    def benchmarkUpdateGrid(self, coeffType: str, stencilType: str, stencilRange: int, dimension: int,
                            alignment: str, maxTime: float, gridSize, blockSize, gridBlocks, d_array0, d_array1,
                            rightOffset: int) -> list:
        return self.stencil.benchmark_update_grid(coeffType, stencilType, stencilRange, dimension, alignment,
                                                  maxTime, gridSize, blockSize, gridBlocks, d_array0, d_array1,
                                                  rightOffset)

    # void launchInit(dim3 gridSize, dim3 blockSize, dim3 gridBlocks, double* d_array, unsigned rightOffset)
    def launchInit(self, gridSize, blockSize, gridBlocks, d_array, rightOffset: int) -> None:
        self.stencil.launch_init(gridSize, blockSize, gridBlocks, d_array, rightOffset)

    # int maxPotentialBlockSize()
    def maxPotentialBlockSize(self) -> int:
        return self.stencil.max_potential_block_size()

    # void copyMask(double* mask, unsigned int maskSize)
    def copyMask(self, mask, maskSize: int | None = None) -> None:
        vals = list(mask)
        if maskSize is not None:
            vals = vals[:maskSize]
        self.stencil.copy_mask(vals)
