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
// Device address of the static scratch array on the current device (cudaError_t value).
int tcs_field_static_scratch(double** out);
// Set the calling thread's message returned by tcs_last_error (for the other .cu files).
void tcs_internal_set_error(const char* msg);
#ifdef __cplusplus
}
#endif
