// Field kernels of the mixed-precision path (compiled by nvcc into libtcs.so for sm_100a).
//
// They act on the interior of a grid laid out like the sweep buffers (row pitch xdim, interior
// [x0, x_lim) x [y0, y_lim) x [z0, z_lim)):
//   tcs_k_defect    r = fl32(sx - x), with max |sx - x| and sum (sx - x)^2 in FP64
//   tcs_k_add       x += e                    (FP64 state, FP32 correction)
//   tcs_k_compare   max |a - b|, sum (a - b)^2, max |b|, sum b^2   (a FP32 or FP64, b FP64)
// Reductions are two-pass and deterministic: each block reduces its rows in a fixed order into
// per-block partials (scratch memory), then one block reduces the partials in index order.
#include <cuda_runtime.h>
#include <stdint.h>

#include "tcs_field.h"

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ void row_of(const TcsFieldGeo& g, uint64_t row, uint64_t& y, uint64_t& z) {
  const uint64_t ny = g.y_lim - g.y0;
  y = g.y0 + row % ny;
  z = g.z0 + row / ny;
}

// Block-wide reduction of up to 4 values (max for slots with is_max, sum otherwise).
template <int N>
__device__ void block_reduce(double (&v)[N], const bool (&is_max)[N], double* out) {
  __shared__ double sh[N][kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double a = v[k];
    for (int o = 16; o > 0; o >>= 1) {
      const double b = __shfl_down_sync(0xffffffffu, a, o);
      a = is_max[k] ? fmax(a, b) : a + b;
    }
    if (lane == 0) sh[k][warp] = a;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      double a = sh[k][0];
      for (int w = 1; w < kThreads / 32; ++w) a = is_max[k] ? fmax(a, sh[k][w]) : a + sh[k][w];
      out[k] = a;
    }
  }
}

__global__ void __launch_bounds__(kThreads)
    tcs_k_defect(const double* __restrict__ x, const double* __restrict__ sx, float* __restrict__ r,
                 TcsFieldGeo g, double* __restrict__ partial) {
  const uint64_t rows = (uint64_t)(g.y_lim - g.y0) * (g.z_lim - g.z0);
  double mx = 0.0, ss = 0.0;
  for (uint64_t row = blockIdx.x; row < rows; row += gridDim.x) {
    uint64_t y, z;
    row_of(g, row, y, z);
    const uint64_t base = y * g.xdim + z * g.xdim * g.ydim;
    // unrolled: several loads of a thread in flight at once (two blocks per SM alone do not
    // keep enough bytes in flight to stream at the HBM rate)
#pragma unroll 4
    for (uint32_t xx = g.x0 + threadIdx.x; xx < g.x_lim; xx += kThreads) {
      const double d = sx[base + xx] - x[base + xx];
      r[base + xx] = (float)d;
      mx = fmax(mx, fabs(d));
      ss = fma(d, d, ss);
    }
  }
  double v[2] = {mx, ss};
  const bool is_max[2] = {true, false};
  block_reduce<2>(v, is_max, partial + 2 * blockIdx.x);
}

__global__ void __launch_bounds__(kThreads)
    tcs_k_compare(const void* __restrict__ a, int a_f32, const double* __restrict__ b, TcsFieldGeo g,
                  double* __restrict__ partial) {
  const uint64_t rows = (uint64_t)(g.y_lim - g.y0) * (g.z_lim - g.z0);
  const float* af = static_cast<const float*>(a);
  const double* ad = static_cast<const double*>(a);
  double md = 0.0, sd = 0.0, mb = 0.0, sb = 0.0;
  for (uint64_t row = blockIdx.x; row < rows; row += gridDim.x) {
    uint64_t y, z;
    row_of(g, row, y, z);
    const uint64_t base = y * g.xdim + z * g.xdim * g.ydim;
    // unrolled: several loads of a thread in flight at once (two blocks per SM alone do not
    // keep enough bytes in flight to stream at the HBM rate)
#pragma unroll 4
    for (uint32_t xx = g.x0 + threadIdx.x; xx < g.x_lim; xx += kThreads) {
      const double bv = b[base + xx];
      const double av = a_f32 ? (double)af[base + xx] : ad[base + xx];
      const double d = av - bv;
      md = fmax(md, fabs(d));
      sd = fma(d, d, sd);
      mb = fmax(mb, fabs(bv));
      sb = fma(bv, bv, sb);
    }
  }
  double v[4] = {md, sd, mb, sb};
  const bool is_max[4] = {true, false, true, false};
  block_reduce<4>(v, is_max, partial + 4 * blockIdx.x);
}

// One block: reduce nblocks partials of width w (slot k is a max when bit k of max_mask is set).
__global__ void __launch_bounds__(kThreads)
    tcs_k_finish(const double* __restrict__ partial, int nblocks, int w, unsigned max_mask,
                 double* __restrict__ out) {
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  bool is_max[4];
  for (int k = 0; k < 4; ++k) is_max[k] = (max_mask >> k) & 1u;
  for (int i = threadIdx.x; i < nblocks; i += kThreads)
    for (int k = 0; k < w; ++k) v[k] = is_max[k] ? fmax(v[k], partial[i * w + k]) : v[k] + partial[i * w + k];
  double res[4];
  block_reduce<4>(v, is_max, res);
  if (threadIdx.x == 0)
    for (int k = 0; k < w; ++k) out[k] = res[k];
}

__global__ void __launch_bounds__(kThreads)
    tcs_k_add(double* __restrict__ x, const float* __restrict__ e, TcsFieldGeo g) {
  const uint64_t rows = (uint64_t)(g.y_lim - g.y0) * (g.z_lim - g.z0);
  for (uint64_t row = blockIdx.x; row < rows; row += gridDim.x) {
    uint64_t y, z;
    row_of(g, row, y, z);
    const uint64_t base = y * g.xdim + z * g.xdim * g.ydim;
    // unrolled: several loads of a thread in flight at once (two blocks per SM alone do not
    // keep enough bytes in flight to stream at the HBM rate)
#pragma unroll 4
    for (uint32_t xx = g.x0 + threadIdx.x; xx < g.x_lim; xx += kThreads) x[base + xx] += (double)e[base + xx];
  }
}

}  // namespace

extern "C" int tcs_field_launch_defect(const double* x, const double* sx, float* r, TcsFieldGeo g,
                                       double* scratch, int nblocks, double* result2,
                                       cudaStream_t st) {
  tcs_k_defect<<<nblocks, kThreads, 0, st>>>(x, sx, r, g, scratch);
  tcs_k_finish<<<1, kThreads, 0, st>>>(scratch, nblocks, 2, 1u, result2);
  return (int)cudaGetLastError();
}

extern "C" int tcs_field_launch_finish(const double* partial, int nblocks, int w, unsigned max_mask,
                                       double* result, cudaStream_t st) {
  tcs_k_finish<<<1, kThreads, 0, st>>>(partial, nblocks, w, max_mask, result);
  return (int)cudaGetLastError();
}

extern "C" int tcs_field_launch_compare(const void* a, int a_f32, const double* b, TcsFieldGeo g,
                                        double* scratch, int nblocks, double* result4,
                                        cudaStream_t st) {
  tcs_k_compare<<<nblocks, kThreads, 0, st>>>(a, a_f32, b, g, scratch);
  tcs_k_finish<<<1, kThreads, 0, st>>>(scratch, nblocks, 4, 5u, result4);
  return (int)cudaGetLastError();
}

extern "C" int tcs_field_launch_add(double* x, const float* e, TcsFieldGeo g, int nblocks,
                                    cudaStream_t st) {
  tcs_k_add<<<nblocks, kThreads, 0, st>>>(x, e, g);
  return (int)cudaGetLastError();
}

// ---- failure-detection self-test -----------------------------------------------------------
// One warp waits on a shared-memory mbarrier that expects one arrival and never gets it -- the
// wait of a sweep kernel whose copy never lands -- through the same bounded loop the kernels use:
// after `limit` cycles it gives up, sets bit 0 (value 1, TCS_DEV_TIMEOUT) of `status` and returns.  No copy
// is in flight and nothing else waits on the barrier, so the context stays usable.
namespace {

__global__ void __launch_bounds__(32) tcs_k_wait_probe(unsigned* status, long long limit) {
  __shared__ __align__(8) unsigned long long bar;
  const unsigned b = (unsigned)__cvta_generic_to_shared(&bar);
  if (threadIdx.x == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
  __syncthreads();
  unsigned done = 0;
  const long long t0 = clock64();
  bool expired = false;
  for (;;) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(b)
        : "memory");
    if (done) break;
    if (clock64() - t0 > limit) {
      expired = true;
      break;
    }
  }
  if (__syncthreads_or(expired) && threadIdx.x == 0) atomicOr(status, 1u);
}

}  // namespace

extern "C" int tcs_field_launch_wait_probe(unsigned* status, long long limit, cudaStream_t st) {
  tcs_k_wait_probe<<<1, 32, 0, st>>>(status, limit);
  return (int)cudaGetLastError();
}

// ---- allocation-free residual: scratch in a static device array ------------------------------
// Some callers cannot allocate device memory at the point where they need the residual norm: a
// framework whose caching allocator owns the device memory, a solver loop that must not pay the
// implicit device synchronisation of cudaMalloc/cudaFree, or a process with a fixed memory
// budget.  For them the partial sums live in this array, part of the library image: every GPU
// that loads the library holds it until the process exits.  It is shared by all calls, keeps the
// last call's contents, and calls that overlap on the GPU race on it.  Nothing in it has to start
// at zero: each call writes every partial it later reads.
static __device__ __align__(256) double tcs_static_scratch[TCS_STATIC_SCRATCH_DOUBLES];

#include <mutex>

// Device address of tcs_static_scratch in the current context.  In host code the array's name
// is only a host-side stand-in, so the address is looked up with cudaGetSymbolAddress, with the
// device current, the first time a context of that device is seen: the entry is keyed by the
// context's unique id (cuCtxGetId), so a context recreated after cudaDeviceReset, which may hold
// the array elsewhere, gets a fresh lookup.
extern "C" int tcs_field_static_scratch(unsigned long long ctx_id, double** out) {
  struct Entry {
    unsigned long long ctx_id;
    double* addr;
  };
  static std::mutex mu;
  static Entry cache[TCS_STATIC_SCRATCH_MAX_DEVICES] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= TCS_STATIC_SCRATCH_MAX_DEVICES) return (int)cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(mu);
  if (!cache[dev].addr || cache[dev].ctx_id != ctx_id) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, tcs_static_scratch);
    if (e != cudaSuccess) return (int)e;
    cache[dev].addr = static_cast<double*>(p);
    cache[dev].ctx_id = ctx_id;
  }
  *out = cache[dev].addr;
  return 0;
}
