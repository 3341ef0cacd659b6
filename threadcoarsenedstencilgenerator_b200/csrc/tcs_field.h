// Internal interface between tcs_capi.cpp and the field kernels of tcs_field.cu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// Size of the static scratch array of the allocation-free residual (doubles: 32 KiB), and the
// number of devices whose address of it is cached.
#define TCS_STATIC_SCRATCH_DOUBLES 4096
#define TCS_STATIC_SCRATCH_MAX_DEVICES 64

// Interior box of a grid buffer (units: grid points; xdim is the padded row pitch).
struct TcsFieldGeo {
  uint64_t xdim, ydim;
  uint32_t x0, x_lim, y0, y_lim, z0, z_lim;
};

// Tile grid of the tensor-core sweep of a 2D Box stencil (tcs_tc.cu).
struct TcsTcGeo {
  uint64_t xdim, ydim;     // padded row pitch, rows
  uint32_t x0, x_lim;      // interior columns [x0, x_lim)
  uint32_t y_lim;          // interior rows [R, y_lim)
  uint32_t ntx, nty;       // tiles of 32 columns x 128 rows
  uint32_t R;              // range (1..8)
};

#ifdef __cplusplus
extern "C" {
#endif
// Each returns a cudaError_t value (0 = launched).  `scratch` holds nblocks*2 (defect) or nblocks*4
// (compare) doubles of per-block partials plus 4 doubles for the result, which is written to
// result2/result4 (device pointers).
int tcs_field_launch_defect(const double* x, const double* sx, float* r, TcsFieldGeo g,
                            double* scratch, int nblocks, double* result2, cudaStream_t st);
int tcs_field_launch_compare(const void* a, int a_f32, const double* b, TcsFieldGeo g,
                             double* scratch, int nblocks, double* result4, cudaStream_t st);
int tcs_field_launch_add(double* x, const float* e, TcsFieldGeo g, int nblocks, cudaStream_t st);
// Reduce nblocks per-block partials of width w into result (one block; slot k is a maximum when bit
// k of max_mask is set, a sum otherwise).
int tcs_field_launch_finish(const double* partial, int nblocks, int w, unsigned max_mask, double* result,
                            cudaStream_t st);
// Failure-detection self-test: a bounded wait on a barrier nothing arrives at (at most `limit`
// clock cycles), which then sets bit 0 (value 1) of `status`.  Returns a cudaError_t value.
int tcs_field_launch_wait_probe(unsigned* status, long long limit, cudaStream_t st);
// Device address of the static scratch array in the current context, whose unique id (cuCtxGetId)
// is `ctx_id` (cudaError_t value).
int tcs_field_static_scratch(unsigned long long ctx_id, double** out);
// Tensor-core sweep: dynamic shared memory of a launch for range R, and the launch itself
// (`bops`: the Toeplitz operands built by the host, BF16 high parts of all 2R+1 rows then low
// parts; `nctas` persistent CTAs).  Returns a cudaError_t value.
// `map`: a 2D tensor map of `in` (FP32, box 48 x tcs_tc_box_rows(R)) for the TMA-fed form, or
// NULL for direct loads.
unsigned tcs_tc_smem_bytes(unsigned R);
unsigned tcs_tc_box_rows(unsigned R);
int tcs_tc_launch(const float* in, const float* src, float* out, const void* bops, const void* map, TcsTcGeo g,
                  unsigned* status, int nctas, cudaStream_t st);
// Set the calling thread's message returned by tcs_last_error (for the other .cu files).
void tcs_internal_set_error(const char* msg);
#ifdef __cplusplus
}
#endif
