// Host build of the engine's per-thread stencil arithmetic (test harness).
//
// Compiles threadcoarsenedstencilgenerator_b200/csrc/tcs_tile.cuh for the CPU with the CUDA
// qualifiers mapped to plain C++ and the __fma_rn intrinsics mapped to std::fma, then runs the
// tcs_direct thread mapping (one thread tile at a time over the whole interior).  Built with
// -ffp-contract=off, so the only fused operations are the explicit ones in the header — the same
// arithmetic the GPU module executes (it is compiled with --fmad=false).  Lets the test suite
// compare the kernel arithmetic with the oracle bit for bit on machines without a GPU.
#include <cmath>
#include <cstring>

#include "host_cuda_shim.h"
#include "tcs_tile.cuh"

extern "C" int tile_sweep(const unsigned grid[3], unsigned left_offset, unsigned right_offset,
                          int aligned, const T* in, T* out, const double* mask) {
  using namespace tcs;
  if (COEFF == 1)
    for (int k = 0; k < S; ++k) tcs_mask[k] = (T)mask[k];
  const long long xdim = grid[0], ydim = grid[1], zdim = DIM == 3 ? grid[2] : 1;
  const long long plane = xdim * ydim;
  const long long x_lim = xdim - R - (aligned ? right_offset : 0);
  const long long y_lim = ydim - R, z_lim = DIM == 3 ? zdim - R : 1;
  const long long z_first = DIM == 3 ? R : 0;
  for (long long z = z_first; DIM == 3 ? (z + CZ - 1 < z_lim) : (z < 1); z += CZ)
    for (long long y = R; y + CY - 1 < y_lim; y += CY)
      for (long long x = R + left_offset; x + CX - 1 < x_lim; x += CX) {
        const long long base = x + y * xdim + z * plane;
        const T* p = in + base;
        auto ld = [&](int gx, int gy, int gz) { return p[gx + gy * xdim + gz * plane]; };
        Acc acc[NE];  // T, or the compensated pair with TCS_COMP
        traverse(ld, acc);
        store(out + base, acc, (tcs_u64)xdim, (tcs_u64)plane);
      }
  return 0;
}
