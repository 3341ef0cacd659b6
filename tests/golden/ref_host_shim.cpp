// Host-CPU harness for the reference's generated kernels (fixture generation only).
//
// make_golden.py compiles this file with g++ after putting one generated `kernels.cu`
// (output of cuda/generate{2,3}DStencil_cuda.py, unmodified) on the include path.  The CUDA
// qualifiers become no-ops and the launch becomes a loop over every block and thread, so the
// generated kernel body runs exactly as written.  g++ -ffp-contract=fast -mfma fuses each
// `resultN += registerM*d_mask[k]` into one fma, as nvcc's default -fmad=true does on the GPU.
#include <cmath>
#include <cstddef>
#include <cstring>

struct tcs_uint3 {
  unsigned x, y, z;
};
static tcs_uint3 blockIdx, threadIdx, blockDim;
#define __global__
#define __constant__

#include "kernels.cu"

extern "C" int shim_sweeps(const unsigned grid[3], const unsigned block[3], const unsigned gblocks[3],
                           unsigned right_offset, const double* mask, unsigned mask_n, double* a,
                           double* b, unsigned nsweeps) {
#ifdef SHIM_VARIABLE
  std::memcpy(d_mask, mask, sizeof(double) * mask_n);
#else
  (void)mask;
  (void)mask_n;
#endif
  (void)right_offset;
  blockDim = {block[0], block[1], block[2]};
  for (unsigned s = 0; s < nsweeps; ++s) {
    for (unsigned bz = 0; bz < gblocks[2]; ++bz)
      for (unsigned by = 0; by < gblocks[1]; ++by)
        for (unsigned bx = 0; bx < gblocks[0]; ++bx)
          for (unsigned tz = 0; tz < block[2]; ++tz)
            for (unsigned ty = 0; ty < block[1]; ++ty)
              for (unsigned tx = 0; tx < block[0]; ++tx) {
                blockIdx = {bx, by, bz};
                threadIdx = {tx, ty, tz};
#if SHIM_DIM == 2
#if SHIM_ALIGNED
                updateGrid(grid[0], grid[1], a, b, right_offset);
#else
                updateGrid(grid[0], grid[1], a, b);
#endif
#else
#if SHIM_ALIGNED
                updateGrid(grid[0], grid[1], grid[2], a, b, right_offset);
#else
                updateGrid(grid[0], grid[1], grid[2], a, b);
#endif
#endif
              }
    double* t = a;
    a = b;
    b = t;
  }
  // result is in `a` (caller swaps accordingly: odd sweep counts end in the second buffer)
  return 0;
}
