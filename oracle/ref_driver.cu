// ref_driver.cu — runs the reference's own generated kernel (test infrastructure).
//
// Compiled by oracle/build_ref.py together with the reference's generated sources: it includes the
// generated `launchUpdateGrid.cu` (cuda/generateLaunchUpdateGrid.py output, which itself includes
// the generated `kernels.cu` and the reference header cuda/launchUpdateGrid.h).  Nothing of the
// reference is modified; this file only drives it:
//   ref_sweeps  — n sweeps through the reference's public entry point benchmarkUpdateGrid with
//                 maxTime = 0, which performs exactly one launch per call
//                 (cuda/generateLaunchUpdateGrid.py:128-139), ping-pong on our side;
//   ref_time    — n back-to-back launches of the generated `updateGrid` kernel timed with CUDA
//                 events (the reference's own kernel without its per-launch host synchronisation).
// Build-time macros: REF_DIM (2|3) and REF_ALIGNED (0|1: Read/Write kernels take rightOffset).
#include "launchUpdateGrid.cu"

#include <cstring>

static int g_last_cuda = 0;

extern "C" int ref_last_cuda_error(void) { return g_last_cuda; }

static int ck(cudaError_t e) {
  if (e != cudaSuccess) {
    g_last_cuda = (int)e;
    return 1;
  }
  return 0;
}

extern "C" int ref_sweeps(const char* coeff, const char* shape, unsigned stencil_range, unsigned dim,
                          const char* align, const unsigned grid[3], const unsigned block[3],
                          const unsigned grid_blocks[3], unsigned right_offset, const double* mask,
                          unsigned mask_n, const double* host_in, double* host_out,
                          unsigned nsweeps) {
  const size_t n = (size_t)grid[0] * grid[1] * (dim == 3 ? grid[2] : 1);
  double *a = nullptr, *b = nullptr;
  if (ck(cudaMalloc(&a, n * sizeof(double))) || ck(cudaMalloc(&b, n * sizeof(double)))) return 2;
  int rc = 0;
  if (ck(cudaMemcpy(a, host_in, n * sizeof(double), cudaMemcpyHostToDevice)) ||
      ck(cudaMemcpy(b, host_in, n * sizeof(double), cudaMemcpyHostToDevice))) {
    rc = 2;
  }
  if (!rc && mask && mask_n) copyMask(const_cast<double*>(mask), mask_n);
  const dim3 gs(grid[0], grid[1], dim == 3 ? grid[2] : 1);
  const dim3 bs(block[0], block[1], block[2]);
  const dim3 gb(grid_blocks[0], grid_blocks[1], grid_blocks[2]);
  for (unsigned s = 0; s < nsweeps && !rc; ++s) {
    try {
      benchmarkUpdateGrid(coeff, shape, stencil_range, dim, align, 0.0, gs, bs, gb, a, b, right_offset);
    } catch (cudaError_t e) {
      g_last_cuda = (int)e;
      rc = 3;
    }
    if (!rc && ck(cudaGetLastError())) rc = 2;
    double* t = a;
    a = b;
    b = t;
  }
  if (!rc && ck(cudaMemcpy(host_out, a, n * sizeof(double), cudaMemcpyDeviceToHost))) rc = 2;
  cudaFree(a);
  cudaFree(b);
  return rc;
}

static void launch_update(const dim3& gs, const dim3& bs, const dim3& gb, double* a, double* b,
                          unsigned right_offset) {
#if REF_DIM == 2
#if REF_ALIGNED
  updateGrid<<<gb, bs>>>(gs.x, gs.y, a, b, right_offset);
#else
  (void)right_offset;
  updateGrid<<<gb, bs>>>(gs.x, gs.y, a, b);
#endif
#else
#if REF_ALIGNED
  updateGrid<<<gb, bs>>>(gs.x, gs.y, gs.z, a, b, right_offset);
#else
  (void)right_offset;
  updateGrid<<<gb, bs>>>(gs.x, gs.y, gs.z, a, b);
#endif
#endif
}

extern "C" int ref_time(unsigned dim, const unsigned grid[3], const unsigned block[3],
                        const unsigned grid_blocks[3], unsigned right_offset, const double* mask,
                        unsigned mask_n, unsigned warmup, unsigned nsweeps, float* ms_total) {
  const size_t n = (size_t)grid[0] * grid[1] * (dim == 3 ? grid[2] : 1);
  double *a = nullptr, *b = nullptr;
  if (ck(cudaMalloc(&a, n * sizeof(double))) || ck(cudaMalloc(&b, n * sizeof(double)))) return 2;
  const dim3 gs(grid[0], grid[1], dim == 3 ? grid[2] : 1);
  const dim3 bs(block[0], block[1], block[2]);
  const dim3 gb(grid_blocks[0], grid_blocks[1], grid_blocks[2]);
  dim3 ib = dim == 3 ? dim3(16, 16, 4) : dim3(32, 16, 1);
  dim3 ig((gs.x + ib.x - 1) / ib.x, (gs.y + ib.y - 1) / ib.y, (gs.z + ib.z - 1) / ib.z);
  launchInit(gs, ib, ig, a, right_offset);
  launchInit(gs, ib, ig, b, right_offset);
  if (mask && mask_n) copyMask(const_cast<double*>(mask), mask_n);
  for (unsigned i = 0; i < warmup; ++i) {
    launch_update(gs, bs, gb, a, b, right_offset);
    double* t = a;
    a = b;
    b = t;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  for (unsigned i = 0; i < nsweeps; ++i) {
    launch_update(gs, bs, gb, a, b, right_offset);
    double* t = a;
    a = b;
    b = t;
  }
  cudaEventRecord(e1);
  int rc = ck(cudaEventSynchronize(e1)) ? 2 : 0;
  if (!rc && ck(cudaGetLastError())) rc = 2;
  float ms = 0.f;
  if (!rc) cudaEventElapsedTime(&ms, e0, e1);
  if (ms_total) *ms_total = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(a);
  cudaFree(b);
  return rc;
}

extern "C" int ref_max_potential_block_size(void) { return maxPotentialBlockSize(); }

// Same as ref_time, but both buffers start from `host_in` instead of the init pattern.
extern "C" int ref_time_data(unsigned dim, const unsigned grid[3], const unsigned block[3],
                             const unsigned grid_blocks[3], unsigned right_offset,
                             const double* mask, unsigned mask_n, const double* host_in,
                             unsigned warmup, unsigned nsweeps, float* ms_total) {
  const size_t n = (size_t)grid[0] * grid[1] * (dim == 3 ? grid[2] : 1);
  double *a = nullptr, *b = nullptr;
  if (ck(cudaMalloc(&a, n * sizeof(double))) || ck(cudaMalloc(&b, n * sizeof(double)))) return 2;
  const dim3 gs(grid[0], grid[1], dim == 3 ? grid[2] : 1);
  const dim3 bs(block[0], block[1], block[2]);
  const dim3 gb(grid_blocks[0], grid_blocks[1], grid_blocks[2]);
  int rc = 0;
  if (ck(cudaMemcpy(a, host_in, n * sizeof(double), cudaMemcpyHostToDevice)) ||
      ck(cudaMemcpy(b, host_in, n * sizeof(double), cudaMemcpyHostToDevice)))
    rc = 2;
  if (!rc && mask && mask_n) copyMask(const_cast<double*>(mask), mask_n);
  for (unsigned i = 0; i < warmup && !rc; ++i) {
    launch_update(gs, bs, gb, a, b, right_offset);
    double* t = a;
    a = b;
    b = t;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  for (unsigned i = 0; i < nsweeps && !rc; ++i) {
    launch_update(gs, bs, gb, a, b, right_offset);
    double* t = a;
    a = b;
    b = t;
  }
  cudaEventRecord(e1);
  if (!rc && ck(cudaEventSynchronize(e1))) rc = 2;
  if (!rc && ck(cudaGetLastError())) rc = 2;
  float ms = 0.f;
  if (!rc) cudaEventElapsedTime(&ms, e0, e1);
  if (ms_total) *ms_total = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(a);
  cudaFree(b);
  return rc;
}
