// Thread-coarsened structured-grid stencil sweeps for sm_100a.
//
// This header is the device half of the engine. The host layer (tcs_capi.cpp) compiles it
// with NVRTC once per stencil parameter set, prepending the TCS_* macros below, exactly as the
// reference bakes one parameter set into one generated `kernels.cu`
// (cuda/generate2DStencil_cuda.py:225-318, cuda/generate3DStencil_cuda.py:245-383).
//
// Required macros (set by the host, one module per parameter set):
//   TCS_T       double | float       element type of the grid
//   TCS_DIM     2 | 3
//   TCS_SHAPE   0 Box | 1 Star       neighbourhood
//   TCS_ORIENT  0 Row | 1 Column     footprint traversal order
//   TCS_COEFF   0 Jacobi | 1 Variable
//   TCS_R       stencil range >= 1
//   TCS_CX, TCS_CY, TCS_CZ           per-thread coarsening factors (TCS_CZ = 1 in 2D)
//
// Arithmetic contract.  Every output point accumulates its S terms in the order in which the
// reference's generated kernel visits them, with the reference's first-term initialisation and
// FMA contraction (the module is compiled with --fmad=false, so only the explicit fma() calls
// below fuse): Jacobi `acc = v0; acc = acc + v_k; out = acc * fl(1/S)`, Variable
// `acc = v0 * m0; acc = fma(v_k, m_k, acc)`.  The FP64 result is therefore bit-identical to the
// reference kernel compiled by nvcc with its default -fmad=true.
//
// Two sweep kernels share that per-thread arithmetic:
//   tcs_direct  one thread per coarsened tile, operands read through L1 (the reference's
//               launch geometry; used for the drop-in grid/block contract and as the
//               fallback when a tile does not fit the TMA constraints);
//   tcs_march   one CTA per (x[,y]) tile column marching along the slowest axis; the input
//               planes stream into a shared-memory ring through TMA
//               (cp.async.bulk.tensor, no multicast) behind mbarriers, so each input element
//               crosses HBM once per sweep and every footprint read is a shared-memory hit.
//
// Every mbarrier wait is bounded (TCS_WAIT_LIMIT cycles).  On expiry the CTA records
// TCS_DEV_TIMEOUT in `tcs_status`, waits (bounded again) for its own bulk copies and returns;
// the host reads `tcs_status` after the sweep.

#ifndef TCS_T
#error "TCS_T must be defined by the instantiation layer"
#endif

#include "tcs_tile.cuh"

#define TCS_DEV_TIMEOUT 1u
#ifndef TCS_WAIT_LIMIT
#define TCS_WAIT_LIMIT 1000000000LL
#endif

// Device-side status word (bit TCS_DEV_TIMEOUT: a bounded wait expired).
__device__ tcs_u32 tcs_status;

// Launch geometry, passed by value.  Units are grid points; xdim is the padded row pitch.
struct TcsGeo {
  tcs_u64 xdim, ydim, zdim;   // gridSize after truncation/alignment (zdim = 1 in 2D)
  tcs_u32 x0, x_lim;          // interior x range [x0, x_lim) = [R + leftOff, xdim - R - rightOff)
  tcs_u32 y_lim, z_lim;       // interior is y < y_lim, z < z_lim (lower bound R)
  tcs_u32 seg;                // tcs_march: outputs along the march axis per CTA
  tcs_u32 nslot;              // tcs_march: ring slots (chunks of one step each)
  tcs_u32 width;              // tcs_march: shared-memory row width W in elements
  tcs_u32 loader;             // tcs_march: 0 = TMA tensor copies, 1 = cp.async element copies
};

// Opaque CUtensorMap (128 bytes, 64-byte aligned), passed as a __grid_constant__ parameter.
struct __align__(64) TcsTmaMap {
  tcs_u64 w[16];
};

namespace tcs {

// ---- mbarrier / TMA primitives (inline PTX) -------------------------------------------------

__device__ __forceinline__ tcs_u32 smem_addr(const void* p) {
  return (tcs_u32)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(tcs_u32 bar, tcs_u32 count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(tcs_u32 bar, tcs_u32 bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(tcs_u32 bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(tcs_u32 bar, tcs_u32 parity) {
  tcs_u32 done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait for the phase with the given parity; returns true when the limit expired.
__device__ __forceinline__ bool mbar_wait_bounded(tcs_u32 bar, tcs_u32 parity, long long limit) {
  if (mbar_try_wait(bar, parity)) return false;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_prefetch_map(const TcsTmaMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<tcs_u64>(map)) : "memory");
}

__device__ __forceinline__ void tma_load_2d(tcs_u32 dst, const TcsTmaMap* map, tcs_u32 bar, int x,
                                            int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<tcs_u64>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tma_load_3d(tcs_u32 dst, const TcsTmaMap* map, tcs_u32 bar, int x,
                                            int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
      "l"(reinterpret_cast<tcs_u64>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

// Element copy global -> shared through the async copy unit (8 or 4 bytes); src_bytes = 0
// writes zeros (the fill for points outside the grid).
__device__ __forceinline__ void cp_async_elem(tcs_u32 dst, const T* src, tcs_u32 src_bytes) {
  if (sizeof(T) == 8) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(src_bytes)
                 : "memory");
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(src_bytes)
                 : "memory");
  }
}

// Copy of E consecutive elements (E * sizeof(T) = 4, 8 or 16 bytes; both addresses aligned to
// that size); src_bytes = 0 writes zeros.
template <int E>
__device__ __forceinline__ void cp_async_vec(tcs_u32 dst, const T* src, tcs_u32 src_bytes) {
  constexpr int B = E * (int)sizeof(T);
  static_assert(B == 4 || B == 8 || B == 16, "cp.async copies 4, 8 or 16 bytes");
  if constexpr (B == 16) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes)
                 : "memory");
  } else if constexpr (B == 8) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(src_bytes)
                 : "memory");
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(src_bytes)
                 : "memory");
  }
}

// The mbarrier receives one arrival once all of this thread's prior cp.async copies landed.
__device__ __forceinline__ void cp_async_arrive(tcs_u32 bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

}  // namespace tcs

#ifndef TCS_PIPE
// ---- tcs_direct: the reference's launch geometry, operands through L1 -------------------------
// Thread origin and tile guard as in cuda/generate2DStencil_cuda.py:78-104 and
// cuda/generate3DStencil_cuda.py:81-114 (x0 already includes the Write left offset).
extern "C" __global__ void tcs_direct(const T* __restrict__ in, T* __restrict__ out,
                                      const T* __restrict__ src, const TcsGeo g) {
  using namespace tcs;
  const tcs_u64 x = (tcs_u64)(blockIdx.x * blockDim.x + threadIdx.x) * CX + g.x0;
  const tcs_u64 y = (tcs_u64)(blockIdx.y * blockDim.y + threadIdx.y) * CY + R;
  const tcs_u64 z = (DIM == 3) ? (tcs_u64)(blockIdx.z * blockDim.z + threadIdx.z) * CZ + R : 0;
  if (x + (CX - 1) < g.x_lim && y + (CY - 1) < g.y_lim &&
      (DIM == 2 || z + (CZ - 1) < g.z_lim)) {
    const tcs_i64 xdim = (tcs_i64)g.xdim;
    const tcs_i64 plane = (tcs_i64)(g.xdim * g.ydim);
    const tcs_u64 base = x + y * g.xdim + z * (tcs_u64)plane;
    const T* __restrict__ p = in + base;
    auto ld = [&](int gx, int gy, int gz) {
      return __ldg(p + (tcs_i64)gx + (tcs_i64)gy * xdim + (tcs_i64)gz * plane);
    };
    Acc acc[NE];
    traverse(ld, acc);
    store(out + base, acc, g.xdim, (tcs_u64)plane, src ? src + base : nullptr);
  }
}

// ---- tcs_march: shared-memory ring fed by TMA (or cp.async), one CTA per tile column ---------
// CTA tile per step: (blockDim.x*CX) x (blockDim.y*CY) in 2D (march along y, step = blockDim.y*CY
// rows) and (blockDim.x*CX) x (blockDim.y*CY) x (blockDim.z*CZ) in 3D (march along z).  Chunk j of
// the ring holds the `step` input planes starting at (segment start - R + j*step), each plane the
// tile plus its halo; a step needs K = 1 + ceil(2R/step) consecutive chunks and the ring keeps
// nslot >= K+1 of them, so the loads of the next nslot-K chunks overlap the arithmetic of a step.
// Loader 0 copies a chunk with one cp.async.bulk.tensor (TMA, issued by thread 0, no multicast);
// loader 1 — for row pitches or base addresses outside the TMA rules — has every thread copy
// elements with cp.async and signal the same mbarrier through cp.async.mbarrier.arrive.
extern "C" __global__ void tcs_march(const __grid_constant__ TcsTmaMap tmap,
                                     const T* __restrict__ in, T* __restrict__ out,
                                     const T* __restrict__ src, const TcsGeo g) {
  using namespace tcs;
  extern __shared__ __align__(128) unsigned char tcs_smem[];
  const tcs_u32 nslot = g.nslot;
  const tcs_u32 W = g.width;
  const tcs_u32 TX = blockDim.x * CX;
  const bool use_tma = (g.loader == 0);
#if TCS_DIM == 2
  const tcs_u32 STEP = blockDim.y * CY;
  const tcs_u32 rows = 1;
  const tcs_u32 mlim = g.y_lim;
  const tcs_u32 ms = R + blockIdx.y * g.seg;
  const tcs_u32 Y0 = 0;
#else
  const tcs_u32 TY = blockDim.y * CY;
  const tcs_u32 STEP = blockDim.z * CZ;
  const tcs_u32 rows = TY + 2 * R;
  const tcs_u32 mlim = g.z_lim;
  const tcs_u32 ms = R + blockIdx.z * g.seg;
  const tcs_u32 Y0 = R + blockIdx.y * TY;
#endif
  const tcs_u32 plane_elems = W * rows;
  if (ms >= mlim) return;
  const tcs_u32 me = min(ms + g.seg, mlim);
  const tcs_u32 nsteps = (me - ms + STEP - 1) / STEP;
  const tcs_u32 nchunks = (me - ms + 2 * R + STEP - 1) / STEP;
  const tcs_u32 K = 1 + (2 * R + STEP - 1) / STEP;
  const tcs_u32 ring_planes = nslot * STEP;
  const tcs_u32 chunk_elems = STEP * plane_elems;
  const tcs_u32 chunk_bytes = chunk_elems * (tcs_u32)sizeof(T);

  const tcs_u32 X0 = g.x0 + blockIdx.x * TX;
  const tcs_u32 xl = (X0 - R) & ~(tcs_u32)(VEC - 1);
  const tcs_u32 nthreads = blockDim.x * blockDim.y * blockDim.z;
  const tcs_u32 tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);

  // Layout: nslot mbarriers, then the ring on a 128-byte boundary (TMA destinations must be
  // 128-byte aligned; the planner makes every chunk a multiple of 128 bytes).
  const tcs_u32 bars = smem_addr(tcs_smem);
  const tcs_u32 bar_bytes = ((nslot * 8u + 127u) / 128u) * 128u;
  const tcs_u32 ring_s = (bars + bar_bytes + 127u) & ~127u;
  T* ring = reinterpret_cast<T*>(tcs_smem + (ring_s - bars));

  // Copy chunk j into its ring slot.  TMA: thread 0 only.  cp.async: every thread.
  auto issue = [&](tcs_u32 j) {
    const tcs_u32 slot = j % nslot;
    const tcs_u32 bar = bars + 8u * slot;
    const tcs_u32 m0 = ms - R + j * STEP;  // first plane of the chunk along the march axis
    if (use_tma) {
      mbar_expect_tx(bar, chunk_bytes);
#if TCS_DIM == 2
      tma_load_2d(ring_s + slot * chunk_bytes, &tmap, bar, (int)xl, (int)m0);
#else
      tma_load_3d(ring_s + slot * chunk_bytes, &tmap, bar, (int)xl, (int)(Y0 - R), (int)m0);
#endif
    } else {
      const tcs_u32 dst0 = ring_s + slot * chunk_bytes;
      for (tcs_u32 q = tid; q < chunk_elems; q += nthreads) {
        const tcs_u32 xx = xl + q % W;
#if TCS_DIM == 2
        const tcs_u64 yy = m0 + q / W;
        const bool inside = xx < g.xdim && yy < g.ydim;
        const tcs_u64 gi = inside ? (tcs_u64)xx + yy * g.xdim : 0;
#else
        const tcs_u64 yy = (Y0 - R) + (q / W) % rows;
        const tcs_u64 zz = m0 + q / plane_elems;
        const bool inside = xx < g.xdim && yy < g.ydim && zz < g.zdim;
        const tcs_u64 gi = inside ? (tcs_u64)xx + yy * g.xdim + zz * g.xdim * g.ydim : 0;
#endif
        cp_async_elem(dst0 + q * (tcs_u32)sizeof(T), in + gi, inside ? (tcs_u32)sizeof(T) : 0u);
      }
      cp_async_arrive(bar);
    }
  };

  if (tid == 0) {
    for (tcs_u32 i = 0; i < nslot; ++i) mbar_init(bars + 8u * i, use_tma ? 1u : nthreads);
    fence_barrier_init();
    if (use_tma) tma_prefetch_map(&tmap);
  }
  __syncthreads();
  {
    const tcs_u32 pro = min(nslot - 1, nchunks);
    if (use_tma) {
      if (tid == 0)
        for (tcs_u32 j = 0; j < pro; ++j) issue(j);
    } else {
      for (tcs_u32 j = 0; j < pro; ++j) issue(j);
    }
  }

  const tcs_u32 x = X0 + threadIdx.x * CX;
  const tcs_u32 col = x - xl;  // ring column of the thread's gx = 0
#if TCS_DIM == 3
  const tcs_u32 y = Y0 + threadIdx.y * CY;
  const tcs_u32 row0 = threadIdx.y * CY + R;  // row in a plane of the thread's gy = 0
  const bool lane_ok = (x + (CX - 1) < g.x_lim) && (y + (CY - 1) < g.y_lim);
  const tcs_u32 tm = threadIdx.z * CZ;
#else
  const bool lane_ok = (x + (CX - 1) < g.x_lim);
  const tcs_u32 tm = threadIdx.y * CY;
#endif
  const tcs_u64 plane_g = g.xdim * g.ydim;

  tcs_u32 ring_base = 0;  // ring plane index of march position (ms - R + s*STEP)
  for (tcs_u32 s = 0; s < nsteps; ++s) {
    const tcs_u32 jlo = (s == 0) ? 0u : s + K - 1;
    const tcs_u32 jhi = min(s + K - 1, nchunks - 1);
    bool expired = false;
    for (tcs_u32 j = jlo; j <= jhi; ++j)
      expired |= mbar_wait_bounded(bars + 8u * (j % nslot), (j / nslot) & 1u, TCS_WAIT_LIMIT);
    if (__syncthreads_or(expired)) {
      if (use_tma) {
        if (tid == 0) {
          atomicOr(&tcs_status, TCS_DEV_TIMEOUT);
          // drain this CTA's own bulk copies in flight (bounded as well)
          const tcs_u32 issued_hi = min(s + nslot - 2, nchunks - 1);
          for (tcs_u32 j = jlo; j <= issued_hi; ++j)
            (void)mbar_wait_bounded(bars + 8u * (j % nslot), (j / nslot) & 1u, TCS_WAIT_LIMIT);
        }
      } else {
        if (tid == 0) atomicOr(&tcs_status, TCS_DEV_TIMEOUT);
        cp_async_wait_all();
      }
      return;
    }
    {
      const tcs_u32 j = s + nslot - 1;
      if (j < nchunks) {
        if (!use_tma)
          issue(j);
        else if (tid == 0)
          issue(j);
      }
    }

    const tcs_u32 m = ms + s * STEP + tm;  // first output of this thread along the march axis
    const bool ok = lane_ok && (m + ((DIM == 3 ? CZ : CY) - 1) < me);
    if (ok) {
      tcs_u32 pb = ring_base + tm;  // ring plane of the thread's footprint start (offset -R)
      if (pb >= ring_planes) pb -= ring_planes;
      Acc acc[NE];
#if TCS_DIM == 2
      auto ld = [&](int gx, int gy, int) {
        tcs_u32 rr = pb + (tcs_u32)(gy + R);
        if (rr >= ring_planes) rr -= ring_planes;
        return ring[rr * W + col + gx];
      };
      traverse(ld, acc);
      const tcs_u64 ob = (tcs_u64)x + (tcs_u64)m * g.xdim;
      store(out + ob, acc, g.xdim, plane_g, src ? src + ob : nullptr);
#else
      auto ld = [&](int gx, int gy, int gz) {
        tcs_u32 pp = pb + (tcs_u32)(gz + R);
        if (pp >= ring_planes) pp -= ring_planes;
        return ring[pp * plane_elems + (row0 + gy) * W + col + gx];
      };
      traverse(ld, acc);
      const tcs_u64 ob = (tcs_u64)x + (tcs_u64)y * g.xdim + (tcs_u64)m * plane_g;
      store(out + ob, acc, g.xdim, plane_g, src ? src + ob : nullptr);
#endif
    }
    ring_base += STEP;
    if (ring_base >= ring_planes) ring_base -= ring_planes;
  }
}


#if defined(TCS_TB) && TCS_DIM == 2
// ---- tcs_tb2: two sweeps in one pass over HBM (temporal blocking, 2D) -------------------------
// Runs on an instance with coarsening CX x CY = 1 x 8 (the thread tile; independent of the
// caller's coarsening).  A CTA loads an input tile into shared memory, computes the first sweep on
// the region of TB_TY x TB_TX outputs plus a range-wide halo into a second tile -- interior points
// with the stencil, every other point keeps its input value (the fixed border, as in the second
// buffer of a ping-pong pair) -- and then the second sweep of its outputs from that.  Both stages
// run the tile arithmetic on CX x CY thread tiles, so every footprint value read from shared
// memory serves all the outputs it touches.  The per-point term order does not depend on the
// tile, so out = S(S(in)) bit for bit; `out` needs in's border (the ping-pong invariant).
constexpr int TB_TX = 128, TB_TY = 256 / (int)sizeof(T), TB_THREADS = 256;  // TB_TY: 32 FP64, 64 FP32

extern "C" __global__ void __launch_bounds__(TB_THREADS)
    tcs_tb2(const T* __restrict__ in, T* __restrict__ out, const TcsGeo g) {
  using namespace tcs;
  static_assert(TB_TX % CX == 0 && TB_TY % CY == 0, "output tile is a multiple of the thread tile");
  extern __shared__ __align__(16) unsigned char tb_smem[];
  constexpr int BW = (TB_TX + 2 * R + CX - 1) / CX * CX;  // first-sweep tile (rounded to thread tiles)
  constexpr int BH = (TB_TY + 2 * R + CY - 1) / CY * CY;
  constexpr int AW = BW + 2 * R, AH = BH + 2 * R;         // input tile
  T* A = reinterpret_cast<T*>(tb_smem);
  T* Bt = A + AW * AH;
  constexpr T c = T(1) / T(S);
  const tcs_i64 xdim = (tcs_i64)g.xdim, ydim = (tcs_i64)g.ydim;
  const tcs_i64 xs = (tcs_i64)g.x0 + (tcs_i64)blockIdx.x * TB_TX;  // first output column
  const tcs_i64 ys = (tcs_i64)R + (tcs_i64)blockIdx.y * TB_TY;     // first output row
  // Input tile through the async copy unit: every thread issues all its copies before waiting, so
  // the whole tile is in flight at once; points outside the grid read as zero.
  const tcs_u32 a_s = (tcs_u32)__cvta_generic_to_shared(A);
  for (int q = threadIdx.x; q < AW * AH; q += TB_THREADS) {
    const int r = q / AW, cc = q - r * AW;
    const tcs_i64 gy = ys - 2 * R + r, gx = xs - 2 * R + cc;
    const bool inside = gy >= 0 && gy < ydim && gx >= 0 && gx < xdim;
    cp_async_elem(a_s + (tcs_u32)q * (tcs_u32)sizeof(T), in + (inside ? gy * xdim + gx : 0),
                  inside ? (tcs_u32)sizeof(T) : 0u);
  }
  cp_async_wait_all();
  __syncthreads();
  constexpr int NT1 = (BW / CX) * (BH / CY);
  for (int t = threadIdx.x; t < NT1; t += TB_THREADS) {
    const int r0 = (t / (BW / CX)) * CY, c0 = (t % (BW / CX)) * CX;  // first-sweep tile coordinates
    const T* p = A + (r0 + R) * AW + (c0 + R);
    auto ld = [&](int dx, int dy, int) { return p[dx + dy * AW]; };
    Acc acc[NE];
    traverse(ld, acc);
    static_for<0, CY>([&](auto ey) {
      static_for<0, CX>([&](auto ex) {
        constexpr int e = decltype(ex)::value + decltype(ey)::value * CX;
        const tcs_i64 gy = ys - R + r0 + decltype(ey)::value, gx = xs - R + c0 + decltype(ex)::value;
        const bool interior = gx >= (tcs_i64)g.x0 && gx < (tcs_i64)g.x_lim && gy >= R && gy < (tcs_i64)g.y_lim;
        const T v = (COEFF == 0) ? acc_value(acc[e]) * c : acc_value(acc[e]);
        Bt[(r0 + decltype(ey)::value) * BW + c0 + decltype(ex)::value] =
            interior ? v : p[decltype(ex)::value + decltype(ey)::value * AW];  // not swept: keeps its value
      });
    });
  }
  __syncthreads();
  constexpr int NT2 = (TB_TX / CX) * (TB_TY / CY);
  for (int t = threadIdx.x; t < NT2; t += TB_THREADS) {
    const int r0 = (t / (TB_TX / CX)) * CY, c0 = (t % (TB_TX / CX)) * CX;  // output tile coordinates
    const T* p = Bt + (r0 + R) * BW + (c0 + R);
    auto ld = [&](int dx, int dy, int) { return p[dx + dy * BW]; };
    Acc acc[NE];
    traverse(ld, acc);
    static_for<0, CY>([&](auto ey) {
      static_for<0, CX>([&](auto ex) {
        constexpr int e = decltype(ex)::value + decltype(ey)::value * CX;
        const tcs_i64 gy = ys + r0 + decltype(ey)::value, gx = xs + c0 + decltype(ex)::value;
        if (gx < (tcs_i64)g.x_lim && gy < (tcs_i64)g.y_lim)
          out[gy * xdim + gx] = (COEFF == 0) ? acc_value(acc[e]) * c : acc_value(acc[e]);
      });
    });
  }
}
#endif

// ---- tcs_init: the reference's initial pattern -----------------------------------------------
// 2D: border columns x < R (right of the Write left offset) and rows y < R are 1.0, else 0.0
// (cuda/generate2DStencil_cuda.py:321-350).  3D: those and planes z < R are 0.75 / 0.25 by the
// parity of the linear index, else 0.0 (cuda/generate3DStencil_cuda.py:386-430).  x_shift is the
// Write left offset (0 otherwise); x_end is xdim - rightOffset for Read/Write and xdim for None.
extern "C" __global__ void tcs_init(T* __restrict__ a, const tcs_u64 xdim, const tcs_u64 ydim,
                                    const tcs_u64 zdim, const tcs_u32 x_shift,
                                    const tcs_u64 x_end) {
  using namespace tcs;
  const tcs_u64 x = (tcs_u64)(blockIdx.x * blockDim.x + threadIdx.x) + x_shift;
  const tcs_u64 y = (tcs_u64)(blockIdx.y * blockDim.y + threadIdx.y);
  const tcs_u64 z = (DIM == 3) ? (tcs_u64)(blockIdx.z * blockDim.z + threadIdx.z) : 0;
  if (x < x_end && y < ydim && z < zdim) {
    const tcs_u64 idx = x + y * xdim + z * xdim * ydim;
    const bool border = (x - x_shift < (tcs_u64)R) || (y < (tcs_u64)R) || (DIM == 3 && z < (tcs_u64)R);
    if (DIM == 2) {
      a[idx] = border ? T(1.0) : T(0.0);
    } else {
      a[idx] = border ? ((idx % 2 == 0) ? T(0.75) : T(0.25)) : T(0.0);
    }
  }
}
#endif  // !TCS_PIPE

#ifdef TCS_PIPE
// ---- tcs_pipe: pipelined streaming sweep -------------------------------------------------------
// Persistent CTAs.  The work is the list of (tile, output plane) pairs, tiles being BX*CX columns
// (2D) or BX*CX x BY*CY columns (3D) and planes running along the slowest axis; each CTA takes an
// equal contiguous share and sweeps it as one or two pieces (tile, [ms, me)).  A piece streams the
// input planes ms-R .. me+R-1 through a shared-memory ring (chunks of TCS_CH planes copied by TMA,
// or by cp.async when the row pitch breaks the TMA rules), and every thread keeps the 2R+1 output
// planes that the current input plane touches in registers: plane p adds its terms to the outputs
// p-R .. p+R (march-axis offset outermost in the reference's per-output order, so each output
// still accumulates in exactly the reference order) and completes output p-R.  Each input element
// is read from HBM once and from shared memory once per thread that needs it; with the plane loop
// unrolled by 2R+1 every register slot and every shared-memory offset is a compile-time constant.
#ifndef TCS_CYCLE
#define TCS_CYCLE 1
#endif
// TCS_STCS: output pairs written with the streaming (evict-first) store, so that the outputs do
// not push the input planes' halo rows out of L2.
#ifndef TCS_STCS
#define TCS_STCS 0
#endif
#ifndef TCS_EPI
#define TCS_EPI 0
#endif
namespace tcs {
// Epilogue of the pipelined sweep (what happens to an output value v once it is complete):
//   0  out = v (+ src)                                      every ordinary sweep
//   1  (FP64) r = fl32(v - x) with x = src, into the float array `aux`, and the running norms
//      max |v - x|, sum (v - x)^2 per thread, reduced per CTA into `partials`: the defect of a
//      defect-correction period without writing S(x) (r bit-identical to a sweep followed by
//      tcs_residual)
//   2  (FP32) x64 += (double)(v (+ src)) with x64 the double array `aux`: the last correction
//      sweep of a period fused with the accumulation into the FP64 state
constexpr int EPI = TCS_EPI;
static_assert(EPI == 0 || (EPI == 1 && sizeof(T) == 8) || (EPI == 2 && sizeof(T) == 4),
              "epilogue 1 needs FP64 sweeps, epilogue 2 FP32 sweeps");
constexpr int BX = TCS_BX;
constexpr int BY = (DIM == 3) ? TCS_BY : 1;
constexpr int CHP = TCS_CH;          // planes per chunk
constexpr int LSHIFT = TCS_LSHIFT;   // (left offset) mod VEC: x position of the tile in its granule
constexpr int TXP = BX * CX;
constexpr int TYP = (DIM == 3) ? BY * CY : 1;
constexpr int ROWS = (DIM == 3) ? TYP + 2 * R : 1;
constexpr int pipe_width() {
  int w = ((TXP + 2 * R + LSHIFT + VEC - 1) / VEC) * VEC;
  while ((CHP * ROWS * w * (int)sizeof(T)) % 128 != 0) w += VEC;
  return w;
}
constexpr int PW = pipe_width();     // shared-memory row width (elements)
constexpr int PLANE = PW * ROWS;     // elements per plane
constexpr int CHUNK = CHP * PLANE;   // elements per ring slot
constexpr int NP2 = 2 * R + 1;       // pipeline depth (output planes in flight)
static_assert(!(DIM == 2 && ORIENT == 1), "2D Column orientation is not pipelined");
static_assert(!COMP || PAIRS, "compensated pipelined sweeps take the packed Box path only");
static_assert(!TCS_SHFL || (BX % 32 == 0 && SHAPE == 1 && (DIM == 2 || ORIENT == 0)),
              "shuffled rows: Star stencils in Row order, block x extent a multiple of the warp");
static_assert(CHP >= 1, "planes per chunk");
static_assert(TXP % VEC == 0, "tile width must be a multiple of the 16-byte granule");

// TCS_TMEM: the ring form of the Star pipeline (tcs::ring_step).  Each thread keeps, in tensor
// memory, R entries of its own centre values (one input plane each) and R entries of output
// accumulators whose in-plane cross is done, instead of 2R+1 output planes in registers: the
// registers hold two output planes, so twice the warps fit on an SM.  A warp reaches the 32 TMEM
// lanes of its quarter (warp % 4); warps w and w + 4k share the lanes and use column groups k.
#ifndef TCS_TMEM
#define TCS_TMEM 0
#endif
constexpr bool TMEM = TCS_TMEM != 0;
constexpr int TM_W = NEP * (int)sizeof(T) / 4;         // 32-bit columns per ring entry
constexpr int TM_THREAD_COLS = 2 * R * TM_W;           // R raw entries + R accumulator entries
constexpr int TM_GROUPS = (BX * BY + 127) / 128;       // column groups (warps per lane quarter)
constexpr int tm_cols() {
  int n = 32;
  while (n < TM_GROUPS * TM_THREAD_COLS) n *= 2;
  return n;
}
constexpr int TM_COLS = tm_cols();                     // allocation: a power of two >= 32
static_assert(!TMEM || (DIM == 3 && SHAPE == 1 && ORIENT == 0 && EPI == 0 && !COMP && !TCS_SHFL),
              "the ring form is built for 3D Star stencils in Row order, plain epilogue");
static_assert(!TMEM || TM_W == 4 || TM_W == 8 || TM_W == 16 || TM_W == 32, "ring entries of 4 to 32 columns");
static_assert(!TMEM || TM_COLS <= 512, "ring exceeds the 512 tensor-memory columns of an SM");
// Columns whose element index is even for every thread: the thread origin sits at ring column
// LSHIFT + R + tx*CX and every row, plane and chunk starts on a 16-byte boundary, so with CX even
// the pair (gx, gx+1) is 16-byte (8-byte for float) aligned exactly when LSHIFT + R + gx is even.
__host__ __device__ constexpr bool pipe_pair_aligned(int gx) { return (CX % 2 == 0) && (((LSHIFT + R + gx) % 2 + 2) % 2 == 0); }

template <class V>
struct PairOf;
template <>
struct PairOf<double> {
  typedef double2 type;
};
template <>
struct PairOf<float> {
  typedef float2 type;
};

// Shared-memory plane reader of one thread (origin `p`, row pitch PW).
struct PipeRing {
  const T* p;
  __host__ __device__ static constexpr bool pair_aligned(int gx) { return pipe_pair_aligned(gx); }
  template <int GX, int GY>
  __device__ __forceinline__ T one() const {
    return p[GY * PW + GX];
  }
  template <int GX, int GY>
  __device__ __forceinline__ void two(T& a, T& b) const {
    const typename PairOf<T>::type v = *reinterpret_cast<const typename PairOf<T>::type*>(p + GY * PW + GX);
    a = v.x;
    b = v.y;
  }
};

#if TCS_TMEM
// tcgen05.ld / st of N consecutive 32-bit columns of this thread's TMEM lane (shape 32x32b).  The
// wait takes the loaded registers as read-write operands, so no use of them moves above it.  The
// statements are volatile (kept in program order among themselves) without a memory clobber:
// they touch no generic memory, and shared-memory loads of the plane may be scheduled across them.
#define TCS_R4(a, o) "=r"(a[o + 0]), "=r"(a[o + 1]), "=r"(a[o + 2]), "=r"(a[o + 3])
#define TCS_W4(a, o) "+r"(a[o + 0]), "+r"(a[o + 1]), "+r"(a[o + 2]), "+r"(a[o + 3])
#define TCS_S4(a, o) "r"(a[o + 0]), "r"(a[o + 1]), "r"(a[o + 2]), "r"(a[o + 3])
template <int N>
__device__ __forceinline__ void tm_ld(tcs_u32 taddr, tcs_u32 (&r)[N]) {
  if constexpr (N == 4) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];" : TCS_R4(r, 0) : "r"(taddr));
  } else if constexpr (N == 8) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : TCS_R4(r, 0), TCS_R4(r, 4) : "r"(taddr));
  } else if constexpr (N == 16) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : TCS_R4(r, 0), TCS_R4(r, 4), TCS_R4(r, 8), TCS_R4(r, 12) : "r"(taddr));
  } else {
    static_assert(N == 32, "4, 8, 16 or 32 columns");
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : TCS_R4(r, 0), TCS_R4(r, 4), TCS_R4(r, 8), TCS_R4(r, 12), TCS_R4(r, 16), TCS_R4(r, 20), TCS_R4(r, 24),
          TCS_R4(r, 28)
        : "r"(taddr));
  }
}
template <int N>
__device__ __forceinline__ void tm_wait_ld(tcs_u32 (&r)[N]) {
  if constexpr (N == 4) {
    asm volatile("tcgen05.wait::ld.sync.aligned;" : TCS_W4(r, 0));
  } else if constexpr (N == 8) {
    asm volatile("tcgen05.wait::ld.sync.aligned;" : TCS_W4(r, 0), TCS_W4(r, 4));
  } else if constexpr (N == 16) {
    asm volatile("tcgen05.wait::ld.sync.aligned;" : TCS_W4(r, 0), TCS_W4(r, 4), TCS_W4(r, 8), TCS_W4(r, 12));
  } else {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : TCS_W4(r, 0), TCS_W4(r, 4), TCS_W4(r, 8), TCS_W4(r, 12), TCS_W4(r, 16), TCS_W4(r, 20),
                   TCS_W4(r, 24), TCS_W4(r, 28));
  }
}
template <int N>
__device__ __forceinline__ void tm_wait_ld2(tcs_u32 (&a)[N], tcs_u32 (&b)[N]) {
  tm_wait_ld<N>(a);
  tm_wait_ld<N>(b);  // nothing left in flight: returns at once, orders b's uses after the wait
}
template <int N>
__device__ __forceinline__ void tm_st(tcs_u32 taddr, const tcs_u32 (&r)[N]) {
  if constexpr (N == 4) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr), TCS_S4(r, 0));
  } else if constexpr (N == 8) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 TCS_S4(r, 0), TCS_S4(r, 4));
  } else if constexpr (N == 16) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};" ::"r"(taddr),
        TCS_S4(r, 0), TCS_S4(r, 4), TCS_S4(r, 8), TCS_S4(r, 12));
  } else {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};" ::"r"(taddr),
        TCS_S4(r, 0), TCS_S4(r, 4), TCS_S4(r, 8), TCS_S4(r, 12), TCS_S4(r, 16), TCS_S4(r, 20), TCS_S4(r, 24),
        TCS_S4(r, 28));
  }
}
#undef TCS_R4
#undef TCS_W4
#undef TCS_S4
__device__ __forceinline__ void tm_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;"); }

// T values <-> 32-bit TMEM columns (a double is two columns: low word, high word).
__device__ __forceinline__ void tm_pack(const T (&v)[NEP], tcs_u32 (&w)[TM_W]) {
#pragma unroll
  for (int e = 0; e < NEP; ++e) {
    if constexpr (sizeof(T) == 8) {
      w[2 * e] = (tcs_u32)__double2loint((double)v[e]);
      w[2 * e + 1] = (tcs_u32)__double2hiint((double)v[e]);
    } else {
      w[e] = __float_as_uint((float)v[e]);
    }
  }
}
__device__ __forceinline__ void tm_unpack(const tcs_u32 (&w)[TM_W], T (&v)[NEP]) {
#pragma unroll
  for (int e = 0; e < NEP; ++e) {
    if constexpr (sizeof(T) == 8)
      v[e] = (T)__hiloint2double((int)w[2 * e + 1], (int)w[2 * e]);
    else
      v[e] = (T)__uint_as_float(w[e]);
  }
}

// The two rings of one thread in tensor memory, addressed relative to input plane c (entry
// e0 = c mod R): raw entries at columns [0, R*TM_W), accumulator entries at [R*TM_W, 2R*TM_W).
struct TmemRing {
  tcs_u32 base;  // this thread's lane quarter and column group
  tcs_u32 e0;
  __device__ __forceinline__ tcs_u32 raw_col(tcs_u32 i) const {
    const tcs_u32 e = e0 + i;
    return base + (e >= (tcs_u32)R ? e - R : e) * TM_W;
  }
  __device__ __forceinline__ void load_first(PipeSlot& s, T (&v)[NEP]) const {
    tm_wait_st();  // the previous plane's stores are in tensor memory
    tcs_u32 w[TM_W], x[TM_W];
    tm_ld<TM_W>(base + (R + e0) * TM_W, w);
    tm_ld<TM_W>(raw_col(0), x);
    tm_wait_ld2<TM_W>(w, x);
    tm_unpack(w, s.v);
    tm_unpack(x, v);
  }
  template <int I>
  __device__ __forceinline__ void load_two(T (&a)[NEP], T (&b)[NEP]) const {
    tcs_u32 w[TM_W], x[TM_W];
    tm_ld<TM_W>(raw_col(I), w);
    if constexpr (I + 1 < R) {
      tm_ld<TM_W>(raw_col(I + 1), x);
      tm_wait_ld2<TM_W>(w, x);
      tm_unpack(x, b);
    } else {
      tm_wait_ld<TM_W>(w);
    }
    tm_unpack(w, a);
  }
  __device__ __forceinline__ void store(const PipeSlot& s, const T (&v)[NEP]) const {
    tcs_u32 a[TM_W], r[TM_W];
    tm_pack(s.v, a);
    tm_pack(v, r);
    tm_st<TM_W>(base + (R + e0) * TM_W, a);
    tm_st<TM_W>(base + e0 * TM_W, r);
  }
};
#endif
}  // namespace tcs

struct TcsPipeGeo {
  tcs_u64 xdim, ydim, zdim;    // padded row pitch, rows, planes (1 in 2D)
  tcs_u64 total;               // work items: tiles * m
  tcs_u64 per_cta;             // work items per CTA
  tcs_u32 x0, x_lim;           // interior x range
  tcs_u32 y_lim, z_lim;        // interior upper bounds in y and z
  tcs_u32 ntx;                 // tiles along x
  tcs_u32 m;                   // output planes along the march axis
  tcs_u32 nslot;               // ring slots
  tcs_u32 loader;              // 0 = TMA, 1 = cp.async by element, 2 = cp.async by pairs
};

// One grid of a batched sweep: an entry of the device-resident grid table (256 bytes).
struct __align__(64) TcsBatchGrid {
  TcsTmaMap map;               // tensor map of `in` (unused with the cp.async loader)
  const T* in;
  T* out;
  const T* src;                // optional source term (nullptr: none)
  tcs_u64 xdim, ydim, zdim;
  tcs_u64 first;               // index of the grid's first work item in the batch
  tcs_u32 x0, x_lim, y_lim, z_lim;
  tcs_u32 ntx, m;
  tcs_u32 loader;
  tcs_u32 pad_;
};

namespace tcs {

// What the pipe body needs to know about the grid a piece belongs to.
struct PipeGridView {
  const TcsTmaMap* map;
  const T* in;
  T* out;
  const T* src;
  tcs_u64 xdim, ydim, zdim;
  tcs_u32 x0, x_lim, y_lim, z_lim, ntx;
  bool use_tma;
  bool cp_pair;  // cp.async loader moves two elements per copy (FP32, even pitch, 8-byte base)
  bool st_pair;  // output pairs stored with one access (even pitch, pair-aligned base)
  void* aux;     // epilogues 1 and 2: the float defect array / the double state (same layout)
  bool src_pair;  // source pairs read with one access (the store's rule for the source's base)
  bool aux_pair;  // epilogue 2: FP64 state pairs with one access (even pitch, 16-byte base)
};

// cp.async fill of one ring chunk: CHP planes of ROWS rows (3D) or CHP rows (2D), PW elements
// each, starting at grid column xl, row y0 (3D) and plane / row m0.  The copies walk the chunk
// row-major in units of E elements, so the row and plane of a copy come from divisions by
// compile-time constants.  Points outside the tensor are filled with zeros, as TMA does.
template <int E>
__device__ __forceinline__ void pipe_copy_chunk(const PipeGridView& G, tcs_u32 dst0, tcs_u32 xl,
                                                tcs_u32 y0, tcs_u32 m0, tcs_u32 tid) {
  constexpr tcs_u32 NTHREADS = BX * BY;
  constexpr tcs_u32 NSEG = PW / E;
  static_assert(PW % E == 0, "ring row width is a multiple of the copy width");
  constexpr tcs_u32 NROW = (DIM == 3) ? CHP * ROWS : CHP;
  for (tcs_u32 q = tid; q < NROW * NSEG; q += NTHREADS) {
    const tcs_u32 row = q / NSEG;
    const tcs_u32 xx = xl + (q - row * NSEG) * E;
#if TCS_DIM == 2
    const tcs_u64 yy = m0 + row;
    const bool inside = xx < G.xdim && yy < G.ydim;
    const tcs_u64 gi = inside ? (tcs_u64)xx + yy * G.xdim : 0;
#else
    const tcs_u32 t = row / ROWS;
    const tcs_u64 yy = y0 + (row - t * ROWS);
    const tcs_u64 zz = m0 + t;
    const bool inside = xx < G.xdim && yy < G.ydim && zz < G.zdim;
    const tcs_u64 gi = inside ? (tcs_u64)xx + (yy + zz * G.ydim) * G.xdim : 0;
#endif
    cp_async_vec<E>(dst0 + q * (tcs_u32)(E * sizeof(T)), G.in + gi,
                    inside ? (tcs_u32)(E * sizeof(T)) : 0u);
  }
}

// Per-CTA streaming state that survives from piece to piece.
struct PipeState {
  tcs_u32 bars, ring_s, nslot, tid, gc;
  tcs_u32 tm;  // TCS_TMEM: this thread's tensor-memory ring base
  T* ring;
  double nmax, nsum;  // epilogue 1: this thread's running defect norms
};

// Sweep one piece: tile `tile` of grid `G`, output planes [R + zs, R + ze) along the march axis.
// Returns false when a bounded wait expired (the CTA must stop).  With MIXED, every barrier
// counts all threads of the CTA, so that pieces loaded by TMA and by cp.async can share the ring:
// for a TMA chunk thread 0 arrives with the byte count and the other threads arrive plainly.
// Every piece consumes all chunks it issues, so the loader may change from piece to piece.
template <bool MIXED>
__device__ __forceinline__ bool pipe_piece(const PipeGridView& G, tcs_u32 tile, tcs_u32 zs,
                                           tcs_u32 ze, PipeState& st, PipeSlot (&acc)[NP2]) {
  constexpr tcs_u32 NTHREADS = BX * BY;
  constexpr tcs_u32 CHUNK_BYTES = CHUNK * (tcs_u32)sizeof(T);
  const tcs_u32 nslot = st.nslot, tid = st.tid, bars = st.bars, gc = st.gc;
  const bool use_tma = G.use_tma;
  const tcs_u32 ms = R + zs;                 // first output plane of the piece
  const tcs_u32 nout = ze - zs;              // output planes of the piece
  const tcs_u32 np = nout + 2 * R;           // input planes streamed
  const tcs_u32 nch = (np + CHP - 1) / CHP;  // chunks of the piece
  const tcs_u32 X0 = G.x0 + (tile % G.ntx) * TXP;
  const tcs_u32 xl = X0 - R - LSHIFT;        // TMA x start, a multiple of VEC
  const tcs_u32 Y0 = (DIM == 3) ? R + (tile / G.ntx) * TYP : 0;

  auto issue = [&](tcs_u32 j) {  // chunk j of the piece -> ring slot (gc + j) % nslot
    const tcs_u32 slot = (gc + j) % nslot;
    const tcs_u32 bar = bars + 8u * slot;
    const tcs_u32 m0 = ms - R + j * CHP;   // first input plane of the chunk
    if (use_tma) {
      if (MIXED && tid != 0) {
        mbar_arrive(bar);
        return;
      }
      mbar_expect_tx(bar, CHUNK_BYTES);
#if TCS_DIM == 2
      tma_load_2d(st.ring_s + slot * CHUNK_BYTES, G.map, bar, (int)xl, (int)m0);
#else
      tma_load_3d(st.ring_s + slot * CHUNK_BYTES, G.map, bar, (int)xl, (int)(Y0 - R), (int)m0);
#endif
    } else {
      const tcs_u32 dst0 = st.ring_s + slot * CHUNK_BYTES;
      const tcs_u32 y0 = (DIM == 3) ? Y0 - R : 0;
      if constexpr (sizeof(T) == 4) {
        if (G.cp_pair)
          pipe_copy_chunk<2>(G, dst0, xl, y0, m0, tid);
        else
          pipe_copy_chunk<1>(G, dst0, xl, y0, m0, tid);
      } else {
        pipe_copy_chunk<1>(G, dst0, xl, y0, m0, tid);
      }
      cp_async_arrive(bar);
    }
  };
  {
    const tcs_u32 pro = min(nslot - 1, nch);
    if (use_tma && !MIXED) {
      if (tid == 0)
        for (tcs_u32 j = 0; j < pro; ++j) issue(j);
    } else {
      for (tcs_u32 j = 0; j < pro; ++j) issue(j);
    }
  }

  const tcs_u32 x = X0 + threadIdx.x * CX;
  const tcs_u32 col0 = LSHIFT + R + threadIdx.x * CX;  // ring column of the thread's gx = 0
#if TCS_DIM == 3
  const tcs_u32 y = Y0 + threadIdx.y * CY;
  const tcs_u32 lane_off = (R + threadIdx.y * CY) * PW + col0;
  const bool lane_ok = (x + (CX - 1) < G.x_lim) && (y + (CY - 1) < G.y_lim);
  const tcs_i64 plane_g = (tcs_i64)(G.xdim * G.ydim);
  T* obase = G.out + (tcs_u64)x + (tcs_u64)y * G.xdim;
#else
  const tcs_u32 lane_off = col0;
  const bool lane_ok = (x + (CX - 1) < G.x_lim);
  const tcs_i64 plane_g = (tcs_i64)G.xdim;
  T* obase = G.out + (tcs_u64)x;
#endif
  // One chunk step consumes one ring chunk: wait for it (bounded), release the slot of the
  // previous chunk to the next copy, then run its CHP planes as straight-line code.  The slot
  // cursor advances by additions only.  Output pi - 2R is complete after input plane pi.
  // Register slot of output plane p: (p - first) mod 2R+1.  When CHP divides 2R+1 the loop runs
  // U = (2R+1)/CHP chunk steps per iteration, a whole cycle of slots, so every slot index stays a
  // compile-time constant without moving registers at the back-edge; otherwise one step per
  // iteration and the slots rotate by CHP at the back-edge.  The cycle is unrolled only while its
  // straight-line code stays near the size of a one-step body (about 2400 terms) and spans at most
  // three chunk steps (more ring waits in one body measured slower than the rotation).
  constexpr int U = (!TMEM && NP2 % CHP == 0 && TCS_CYCLE != 0 && NP2 * S * NEP <= 2400 && NP2 / CHP <= 3)
                        ? NP2 / CHP : 1;
  tcs_u32 tslot = 0;  // TCS_TMEM: ring entry of the current input plane (plane mod R)
  tcs_u32 cur_slot = gc % nslot;
  tcs_u32 cur_par = (gc / nslot) & 1u;
  T* optr = obase + ((tcs_i64)ms - 2 * R) * plane_g;
  // A return from inside this loop costs registers across the whole body: leave it by break.
  bool aborted = false;
  for (tcs_u32 j0 = 0; j0 < nch; j0 += U) {
    static_for<0, U>([&](auto uu) {
      constexpr int u = decltype(uu)::value;
      const tcs_u32 j = j0 + u;
      if (aborted || j >= nch) return;
      const bool expired = mbar_wait_bounded(bars + 8u * cur_slot, cur_par, TCS_WAIT_LIMIT);
      if (__syncthreads_or(expired)) {
        if (use_tma) {
          if (tid == 0) {
            atomicOr(&tcs_status, TCS_DEV_TIMEOUT);
            const tcs_u32 hi = min(j + nslot - 2, nch - 1);
            for (tcs_u32 jj = j; jj <= hi; ++jj)
              (void)mbar_wait_bounded(bars + 8u * ((gc + jj) % nslot), ((gc + jj) / nslot) & 1u,
                                      TCS_WAIT_LIMIT);
          }
        } else {
          if (tid == 0) atomicOr(&tcs_status, TCS_DEV_TIMEOUT);
          cp_async_wait_all();
        }
        aborted = true;
        return;
      }
      if (j + nslot - 1 < nch) {
        if (!use_tma || MIXED)
          issue(j + nslot - 1);
        else if (tid == 0)
          issue(j + nslot - 1);
      }
      const T* pc = st.ring + cur_slot * CHUNK + lane_off;
      const tcs_u32 pbase = j * CHP;  // input plane index (within the piece) of the chunk's first
      static_for<0, CHP>([&](auto tt) {
        constexpr int t = decltype(tt)::value;
        constexpr int tc = u * CHP + t;  // position of the plane in the slot cycle
        const tcs_u32 pi = pbase + t;
        if (pi < np) {
          // A source term is read from global memory when its output row is stored: fetch the rows
          // of the output completed PF planes later into L1 now, so that the store does not wait
          // for the latency of DRAM or L2.
          // (Epilogue 2 reads and writes the FP64 state the same way: its rows too.)
          constexpr int PF = 2;
          if ((G.src || EPI == 2) && lane_ok) {
            const int opf = (int)pi - 2 * R + PF;
            if (opf >= 0 && opf < (int)nout) {
              const tcs_i64 off0 = (optr - G.out) + (tcs_i64)(t + PF) * plane_g;
              static_for<0, (DIM == 3) ? CY : 1>([&](auto ey) {
                const tcs_i64 off = off0 + decltype(ey)::value * (tcs_i64)G.xdim;
                if (G.src) {
                  asm volatile("prefetch.global.L1 [%0];" ::"l"(G.src + off));
                  if constexpr (CX * sizeof(T) > 16) asm volatile("prefetch.global.L1 [%0];" ::"l"(G.src + off + CX - 1));
                }
                if constexpr (EPI == 2) {
                  const double* xq = static_cast<const double*>(G.aux) + off;
                  asm volatile("prefetch.global.L1 [%0];" ::"l"(xq));
                  if constexpr (CX * sizeof(double) > 16) asm volatile("prefetch.global.L1 [%0];" ::"l"(xq + CX - 1));
                }
              });
            }
          }
          const PipeRing ld{pc + t * PLANE};
#if TCS_TMEM
          PipeSlot ring_done;  // the output centred R planes back, complete after this plane
          {
            const TmemRing ring{st.tm, tslot};
            ring_step(ld, ring, ring_done);
            tslot = (tslot + 1u == (tcs_u32)R) ? 0u : tslot + 1u;
          }
#else
          auto slot = [&](auto kk) -> PipeSlot& {
            constexpr int k = decltype(kk)::value;
            return acc[((tc - k) % NP2 + NP2) % NP2];
          };
          pipe_plane(ld, slot);
#endif
          const int op = (int)pi - 2 * R;
          if (EPI != 0 && lane_ok && op >= 0 && op < (int)nout) {
            constexpr T c = T(1) / T(S);
            PipeSlot& done = acc[((tc - 2 * R) % NP2 + NP2) % NP2];
            const tcs_i64 rowoff = (optr - G.out) + (tcs_i64)t * plane_g;
            static_for<0, (DIM == 3) ? CY : 1>([&](auto ey) {
              static_for<0, CX>([&](auto ex) {
                constexpr int e = decltype(ex)::value + decltype(ey)::value * CX;
                const tcs_i64 off = rowoff + decltype(ex)::value + decltype(ey)::value * (tcs_i64)G.xdim;
                T v = (COEFF == 0) ? slot_value<e>(done) * c : slot_value<e>(done);
                if constexpr (EPI == 1) {
                  const double d = (double)v - (double)G.src[off];
                  static_cast<float*>(G.aux)[off] = (float)d;
                  st.nmax = fmax(st.nmax, fabs(d));
                  st.nsum = fma(d, d, st.nsum);
                } else {
                  // the state's pairs with one access each way where the output pair rule holds
                  constexpr bool pair = pipe_pair_aligned(0) && (decltype(ex)::value % 2 == 0);
                  constexpr bool tail = pipe_pair_aligned(0) && (decltype(ex)::value % 2 == 1);
                  double* xg = static_cast<double*>(G.aux);
                  if constexpr (pair) {
                    T v1 = (COEFF == 0) ? slot_value<e + 1>(done) * c : slot_value<e + 1>(done);
                    if (G.src) {
                      v = v + G.src[off];
                      v1 = v1 + G.src[off + 1];
                    }
                    if (G.aux_pair) {
                      double2 x2 = *reinterpret_cast<const double2*>(xg + off);
                      x2.x = x2.x + (double)v;
                      x2.y = x2.y + (double)v1;
                      *reinterpret_cast<double2*>(xg + off) = x2;
                    } else {
                      xg[off] = xg[off] + (double)v;
                      xg[off + 1] = xg[off + 1] + (double)v1;
                    }
                  } else if constexpr (!tail) {
                    if (G.src) v = v + G.src[off];
                    xg[off] = xg[off] + (double)v;
                  }
                }
              });
            });
          }
          if (EPI == 0 && lane_ok && op >= 0 && op < (int)nout) {
            constexpr T c = T(1) / T(S);
#if TCS_TMEM
            PipeSlot& done = ring_done;
#else
            PipeSlot& done = acc[((tc - 2 * R) % NP2 + NP2) % NP2];
#endif
            T* orow = optr + (tcs_i64)t * plane_g;
            // Output x is R + leftOff + an even offset when CX is even: pairs are aligned when
            // R + LSHIFT is even (the shared-memory pair rule at gx = 0).
            static_for<0, (DIM == 3) ? CY : 1>([&](auto ey) {
              static_for<0, CX>([&](auto ex) {
                constexpr int e = decltype(ex)::value + decltype(ey)::value * CX;
                constexpr bool pair = pipe_pair_aligned(0) && (decltype(ex)::value % 2 == 0);
                constexpr bool tail = pipe_pair_aligned(0) && (decltype(ex)::value % 2 == 1);
                T* o = orow + decltype(ex)::value + decltype(ey)::value * (tcs_i64)G.xdim;
                const T* so = G.src ? G.src + (o - G.out) : nullptr;
                if constexpr (pair) {
                  T v0 = (COEFF == 0) ? slot_value<e>(done) * c : slot_value<e>(done);
                  T v1 = (COEFF == 0) ? slot_value<e + 1>(done) * c : slot_value<e + 1>(done);
                  if (so) {
                    if (G.src_pair) {  // the source pair in one access, like the store
                      const typename PairOf<T>::type s2 = *reinterpret_cast<const typename PairOf<T>::type*>(so);
                      v0 = v0 + s2.x;
                      v1 = v1 + s2.y;
                    } else {
                      v0 = v0 + so[0];
                      v1 = v1 + so[1];
                    }
                  }
                  if (G.st_pair) {
                    typename PairOf<T>::type v2;
                    v2.x = v0;
                    v2.y = v1;
                    if constexpr (TCS_STCS)
                      __stcs(reinterpret_cast<typename PairOf<T>::type*>(o), v2);
                    else
                      *reinterpret_cast<typename PairOf<T>::type*>(o) = v2;
                  } else {
                    o[0] = v0;
                    o[1] = v1;
                  }
                } else if constexpr (!tail) {
                  T v = (COEFF == 0) ? slot_value<e>(done) * c : slot_value<e>(done);
                  if (so) v = v + so[0];
                  *o = v;
                }
              });
            });
          }
        }
      });
      // One step per iteration: re-align the register slots with the next chunk (slot m takes
      // what slot (m + CHP) held).
      if constexpr (!TMEM && U == 1 && CHP % NP2 != 0) {
        PipeSlot tmp[NP2];
        static_for<0, NP2>([&](auto m) { tmp[decltype(m)::value] = acc[decltype(m)::value]; });
        static_for<0, NP2>([&](auto m) { acc[decltype(m)::value] = tmp[(decltype(m)::value + CHP) % NP2]; });
      }
      optr += (tcs_i64)CHP * plane_g;
      if (++cur_slot == nslot) {
        cur_slot = 0;
        cur_par ^= 1u;
      }
    });
    if (aborted) break;
  }
  st.gc = gc + nch;
  return !aborted;
}

// Shared-memory layout of both pipe kernels: nslot mbarriers, then the ring on a 128-byte
// boundary.  Thread 0 initialises the barriers (arrival count 1 when only thread 0 arrives, for
// TMA; all threads otherwise).
__device__ __forceinline__ PipeState pipe_setup(tcs_u32 nslot, bool single_arrival) {
  extern __shared__ __align__(128) unsigned char tcs_smem[];
  PipeState st;
  st.nslot = nslot;
  st.tid = threadIdx.x + BX * threadIdx.y;
  st.bars = smem_addr(tcs_smem);
  const tcs_u32 bar_bytes = ((nslot * 8u + 127u) / 128u) * 128u;
  st.ring_s = (st.bars + bar_bytes + 127u) & ~127u;
  st.ring = reinterpret_cast<T*>(tcs_smem + (st.ring_s - st.bars));
  st.gc = 0;
  st.nmax = 0.0;
  st.nsum = 0.0;
  if (st.tid == 0) {
    for (tcs_u32 i = 0; i < nslot; ++i) mbar_init(st.bars + 8u * i, single_arrival ? 1u : BX * BY);
    fence_barrier_init();
  }
  __syncthreads();
  return st;
}

}  // namespace tcs

#if !defined(TCS_BATCH) && !defined(TCS_TB3)
extern "C" __global__ void __launch_bounds__(TCS_BX * ((TCS_DIM == 3) ? TCS_BY : 1))
    tcs_pipe(const __grid_constant__ TcsTmaMap tmap, const T* __restrict__ in,
             T* __restrict__ out, const T* __restrict__ src, const TcsPipeGeo g, void* aux,
             double* __restrict__ partials) {
  using namespace tcs;
  PipeGridView G;
  G.aux = aux;
  G.map = &tmap;
  G.in = in;
  G.out = out;
  G.src = src;
  G.xdim = g.xdim;
  G.ydim = g.ydim;
  G.zdim = g.zdim;
  G.x0 = g.x0;
  G.x_lim = g.x_lim;
  G.y_lim = g.y_lim;
  G.z_lim = g.z_lim;
  G.ntx = g.ntx;
  G.use_tma = (g.loader == 0);
  G.cp_pair = (g.loader == 2);
  // Output pairs are stored with one access only when every row keeps the parity of the first:
  // an even row pitch and a pair-aligned base address.
  G.st_pair = (g.xdim % 2 == 0) && (reinterpret_cast<tcs_u64>(out) % (2 * sizeof(T)) == 0);
  G.src_pair = G.st_pair && (reinterpret_cast<tcs_u64>(src) % (2 * sizeof(T)) == 0);
  G.aux_pair = (g.xdim % 2 == 0) && (reinterpret_cast<tcs_u64>(aux) % 16 == 0);
  if (G.use_tma && threadIdx.x == 0 && threadIdx.y == 0) tma_prefetch_map(&tmap);
  PipeState st = pipe_setup(g.nslot, G.use_tma);
#if TCS_TMEM
  // Warp 0 allocates the CTA's tensor-memory columns (the host limits the CTAs per SM so that
  // their allocations fit the SM's 512 columns) and frees them when the CTA is done, on the
  // error path too.
  __shared__ tcs_u32 tm_base;
  const tcs_u32 warp_id = st.tid >> 5;
  if (warp_id == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tm_base)),
                 "r"((tcs_u32)TM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  st.tm = tm_base + ((32u * (warp_id & 3u)) << 16) + (warp_id >> 2) * (tcs_u32)TM_THREAD_COLS;
#else
  st.tm = 0;
#endif
  PipeSlot acc[NP2];
  const tcs_u64 w_begin = (tcs_u64)blockIdx.x * g.per_cta;
  const tcs_u64 w_end = min(w_begin + g.per_cta, g.total);
  bool ok = true;
  for (tcs_u64 w = w_begin; w < w_end;) {
    const tcs_u32 tile = (tcs_u32)(w / g.m);
    const tcs_u32 zs = (tcs_u32)(w % g.m);
    const tcs_u32 ze = (tcs_u32)min((tcs_u64)g.m, (tcs_u64)zs + (w_end - w));
    w += ze - zs;
    if (!pipe_piece<false>(G, tile, zs, ze, st, acc)) {
      ok = false;
      break;
    }
  }
#if TCS_TMEM
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp_id == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm_base), "r"((tcs_u32)TM_COLS)
                 : "memory");
  }
#endif
  if (!ok) return;
  if constexpr (EPI == 1) {
    // this CTA's defect norms: shuffles within each warp, then one value per warp in shared memory
    __shared__ double red[2][32];
    double mx = st.nmax, ss = st.nsum;
    constexpr tcs_u32 NT = BX * BY;
    const tcs_u32 lane = st.tid & 31u, width = min(32u, NT - (st.tid & ~31u));  // lanes of this warp
    const unsigned lanes = width == 32u ? 0xffffffffu : ((1u << width) - 1u);
    for (tcs_u32 o = 16; o > 0; o >>= 1) {
      const double m2 = __shfl_down_sync(lanes, mx, o), s2 = __shfl_down_sync(lanes, ss, o);
      if (lane + o < width) {
        mx = fmax(mx, m2);
        ss += s2;
      }
    }
    const tcs_u32 warp = st.tid >> 5, nwarps = (NT + 31) / 32;
    if (lane == 0) {
      red[0][warp] = mx;
      red[1][warp] = ss;
    }
    __syncthreads();
    if (st.tid == 0) {
      for (tcs_u32 k = 1; k < nwarps; ++k) {
        mx = fmax(mx, red[0][k]);
        ss += red[1][k];
      }
      partials[2 * blockIdx.x] = mx;
      partials[2 * blockIdx.x + 1] = ss;
    }
  }
}
#endif  // !TCS_BATCH && !TCS_TB3

#ifdef TCS_BATCH
// ---- tcs_pipe_batch: one persistent launch over many grids of the same parameter set ---------
// The work list is the concatenation of every grid's (tile, plane) items; each CTA takes an equal
// contiguous share and sweeps it as pieces of one grid each, reusing its ring, barriers and
// register pipeline from piece to piece.  Grid g's items start at grids[g].first (ascending);
// each grid has its own loader (TMA where its rows and base allow, cp.async otherwise).
extern "C" __global__ void __launch_bounds__(TCS_BX * ((TCS_DIM == 3) ? TCS_BY : 1))
    tcs_pipe_batch(const TcsBatchGrid* __restrict__ grids, const tcs_u32 ngrids,
                   const tcs_u64 total, const tcs_u64 per_cta, const tcs_u32 nslot) {
  using namespace tcs;
  static_assert(EPI == 0, "batched sweeps store plain outputs");
  PipeState st = pipe_setup(nslot, false);
  PipeSlot acc[NP2];
  const tcs_u64 w_begin = (tcs_u64)blockIdx.x * per_cta;
  const tcs_u64 w_end = min(w_begin + per_cta, total);
  tcs_u32 gi = 0;
  {  // last grid whose first item is <= w_begin (binary search)
    tcs_u32 lo = 0, hi = ngrids;
    while (hi - lo > 1) {
      const tcs_u32 mid = (lo + hi) / 2;
      if (grids[mid].first <= w_begin) lo = mid; else hi = mid;
    }
    gi = lo;
  }
  for (tcs_u64 w = w_begin; w < w_end;) {
    while (gi + 1 < ngrids && grids[gi + 1].first <= w) ++gi;
    const TcsBatchGrid& B = grids[gi];
    PipeGridView G;
    G.map = &B.map;
    G.in = B.in;
    G.out = B.out;
    G.src = B.src;
    G.xdim = B.xdim;
    G.ydim = B.ydim;
    G.zdim = B.zdim;
    G.x0 = B.x0;
    G.x_lim = B.x_lim;
    G.y_lim = B.y_lim;
    G.z_lim = B.z_lim;
    G.ntx = B.ntx;
    G.use_tma = (B.loader == 0);
    G.cp_pair = (B.loader == 2);
    G.st_pair = (B.xdim % 2 == 0) && (reinterpret_cast<tcs_u64>(B.out) % (2 * sizeof(T)) == 0);
    G.src_pair = G.st_pair && (reinterpret_cast<tcs_u64>(B.src) % (2 * sizeof(T)) == 0);
    G.aux = nullptr;
    G.aux_pair = false;
    const tcs_u64 local = w - B.first;
    const tcs_u32 tile = (tcs_u32)(local / B.m);
    const tcs_u32 zs = (tcs_u32)(local % B.m);
    const tcs_u32 ze = (tcs_u32)min((tcs_u64)B.m, (tcs_u64)zs + (w_end - w));
    w += ze - zs;
    if (!pipe_piece<true>(G, tile, zs, ze, st, acc)) return;
  }
}
#endif  // TCS_BATCH

#ifdef TCS_TB3
// ---- tcs_tb3: two sweeps in one pass over HBM (temporal blocking, 3D and 2D) -------------------
// The pipelined sweep run twice in the same CTA, stage 2 on the output of stage 1.  A CTA owns an
// extended tile of TB_EX x TB_EY columns (its threads' coverage, CX x CY per thread, with CX = CY
// dividing R) and streams its input planes through the TMA ring as tcs_pipe does.  Stage 1 keeps
// 2R+1 planes of S(in) over the extended tile in registers (pipeline 1); each completed plane of
// S(in) goes to a shared-memory plane buffer (two, used in turn), where points outside the grid's
// interior take the input's value (the fixed border of the ping-pong pair).  Stage 2 applies that
// plane to its own register pipeline (pipeline 2) and stores the completed planes of S(S(in)) for
// the inner (TB_EX - 2R) x (TB_EY - 2R) columns; the outer ring of threads only serves stage 1.
// Both stages use the per-output term order of one sweep, so out = S(S(in)) bit for bit.
// In 2D the march axis is y and a "plane" is one row: the extended tile is a strip of TB_EX
// columns, the plane buffer one row with an R-wide margin, and the output tile the inner
// TB_EX - 2R columns of every row; a thread tile (CX columns) may straddle the output tile's
// edge, so the store tests each column.
namespace tcs {
constexpr int TB_EX = TXP, TB_EY = TYP;                                       // extended tile (stage 1)
constexpr int TB_OX = TB_EX - 2 * R, TB_OY = (DIM == 3) ? TB_EY - 2 * R : 1;  // output tile (stage 2)
// Plane buffer with a range-wide margin; in 2D the left margin TB_ML is rounded up to even and the
// row to an even width, so a thread's column pairs sit on 2-element boundaries (one access each).
constexpr int TB_ML = (DIM == 3) ? R : R + (R & 1);
constexpr int TB_BW = (DIM == 3) ? TB_EX + 2 * R : ((TB_ML + TB_EX + R + 1) / 2) * 2;
constexpr int TB_BH = (DIM == 3) ? TB_EY + 2 * R : 1;
static_assert(TB_OX > 0 && TB_OY > 0 && TB_OX % VEC == 0, "output tile: positive, 16-byte multiple");
static_assert(DIM == 2 || (R % CX == 0 && R % CY == 0), "3D thread tiles must not straddle the output tile's edge");
static_assert(DIM == 3 || CY == 1, "2D strips: one row per thread");
static_assert(!COMP && EPI == 0, "plain sweeps only");

// Reader of a stage-1 plane in the plane buffer at a thread origin (row pitch TB_BW).  Pairs are
// aligned where the buffer column TB_ML + gx is even (the buffer starts on 128 bytes, TB_BW is even).
struct TbPlane {
  const T* p;
  __host__ __device__ static constexpr bool pair_aligned(int gx) {
    return (CX % 2 == 0) && (TB_BW % 2 == 0) && (((TB_ML + gx) % 2 + 2) % 2 == 0);
  }
  template <int GX, int GY>
  __device__ __forceinline__ T one() const {
    return p[GY * TB_BW + GX];
  }
  template <int GX, int GY>
  __device__ __forceinline__ void two(T& a, T& b) const {
    const typename PairOf<T>::type v = *reinterpret_cast<const typename PairOf<T>::type*>(p + GY * TB_BW + GX);
    a = v.x;
    b = v.y;
  }
};

// One piece: tile `tile`, output planes [R + zs, R + ze).  Returns false when a wait expired.
__device__ __forceinline__ bool tb3_piece(const PipeGridView& G, tcs_u32 tile, tcs_u32 zs, tcs_u32 ze,
                                          PipeState& st, PipeSlot (&acc1)[NP2], PipeSlot (&acc2)[NP2],
                                          T* bbuf) {
  constexpr tcs_u32 CHUNK_BYTES = CHUNK * (tcs_u32)sizeof(T);
  const tcs_u32 nslot = st.nslot, tid = st.tid, bars = st.bars, gc = st.gc;
  const bool use_tma = G.use_tma;
  const int ms = R + (int)zs;                       // first output plane
  const int nout = (int)(ze - zs);
  const int np = nout + 4 * R;                      // input planes streamed
  const tcs_u32 nch = (tcs_u32)((np + CHP - 1) / CHP);
  const int m_first = ms - 2 * R;                   // input plane of pi = 0
  const int X0 = (int)G.x0 - R + (int)(tile % G.ntx) * TB_OX;  // extended tile origin
  const int Y0 = (DIM == 3) ? (int)(tile / G.ntx) * TB_OY : 0;  // 3D: = R + ty*TB_OY - R
  const int xl = X0 - R - LSHIFT;                   // TMA x start: a multiple of VEC (may be < 0)
  auto issue = [&](tcs_u32 j) {
    const tcs_u32 slot = (gc + j) % nslot;
    const tcs_u32 bar = bars + 8u * slot;
    const int m0 = m_first + (int)(j * CHP);
    if (use_tma) {
      mbar_expect_tx(bar, CHUNK_BYTES);
#if TCS_DIM == 2
      tma_load_2d(st.ring_s + slot * CHUNK_BYTES, G.map, bar, xl, m0);
#else
      tma_load_3d(st.ring_s + slot * CHUNK_BYTES, G.map, bar, xl, Y0 - R, m0);
#endif
    } else {
      // negative coordinates wrap to large unsigned values and read as zeros
      pipe_copy_chunk<1>(G, st.ring_s + slot * CHUNK_BYTES, (tcs_u32)xl, (tcs_u32)(Y0 - R), (tcs_u32)m0, tid);
      cp_async_arrive(bar);
    }
  };
  {
    const tcs_u32 pro = min(nslot - 1, nch);
    if (use_tma) {
      if (tid == 0)
        for (tcs_u32 j = 0; j < pro; ++j) issue(j);
    } else {
      for (tcs_u32 j = 0; j < pro; ++j) issue(j);
    }
  }
  const int ex0 = (int)threadIdx.x * CX;  // thread tile in the extended tile
  const int ey0 = (DIM == 3) ? (int)threadIdx.y * CY : 0;
  const tcs_u32 lane_off = ((DIM == 3) ? (R + threadIdx.y * CY) * PW : 0u) + LSHIFT + R + threadIdx.x * CX;
  // some column of the thread tile lies in the output tile (3D: all of them)
  const bool inner = ex0 + CX > R && ex0 < TB_EX - R && (DIM == 2 || (ey0 >= R && ey0 < TB_EY - R));
  const tcs_i64 xdim = (tcs_i64)G.xdim;
  const tcs_i64 plane_g = (DIM == 3) ? (tcs_i64)(G.xdim * G.ydim) : xdim;  // stride of the march axis
  const int plane_lim = (DIM == 3) ? (int)G.z_lim : (int)G.y_lim;         // interior bound along it
  const int plane_dim = (DIM == 3) ? (int)G.zdim : (int)G.ydim;
  constexpr T c = T(1) / T(S);
  tcs_u32 cur_slot = gc % nslot;
  tcs_u32 cur_par = (gc / nslot) & 1u;
  bool aborted = false;
  for (tcs_u32 j = 0; j < nch; ++j) {
    const bool expired = mbar_wait_bounded(bars + 8u * cur_slot, cur_par, TCS_WAIT_LIMIT);
    if (__syncthreads_or(expired)) {
      if (use_tma) {
        if (tid == 0) {
          atomicOr(&tcs_status, TCS_DEV_TIMEOUT);
          const tcs_u32 hi = min(j + nslot - 2, nch - 1);
          for (tcs_u32 jj = j; jj <= hi; ++jj)
            (void)mbar_wait_bounded(bars + 8u * ((gc + jj) % nslot), ((gc + jj) / nslot) & 1u, TCS_WAIT_LIMIT);
        }
      } else {
        if (tid == 0) atomicOr(&tcs_status, TCS_DEV_TIMEOUT);
        cp_async_wait_all();
      }
      aborted = true;
      break;
    }
    if (j + nslot - 1 < nch) {
      if (!use_tma)
        issue(j + nslot - 1);
      else if (tid == 0)
        issue(j + nslot - 1);
    }
    const T* pc = st.ring + cur_slot * CHUNK + lane_off;
    static_for<0, CHP>([&](auto tt) {
      constexpr int t = decltype(tt)::value;
      const int pi = (int)(j * CHP) + t;
      if (pi < np) {
        // stage 1: input plane m_first + pi; completes plane q = m_first + pi - R of S(in)
        const PipeRing lda{pc + t * PLANE};
        auto slot1 = [&](auto kk) -> PipeSlot& {
          constexpr int k = decltype(kk)::value;
          return acc1[((t - k) % NP2 + NP2) % NP2];
        };
        pipe_plane(lda, slot1);
        const int q = m_first + pi - R;
        T* bq = bbuf + (pi & 1) * (TB_BW * TB_BH);
        PipeSlot& d1 = acc1[((t - 2 * R) % NP2 + NP2) % NP2];
        static_for<0, CY>([&](auto ey) {
          T vrow[CX];
          static_for<0, CX>([&](auto ex) {
            constexpr int e = decltype(ex)::value + decltype(ey)::value * CX;
            const int gx = X0 + ex0 + decltype(ex)::value, gy = Y0 + ey0 + decltype(ey)::value;
            const bool interior = gx >= (int)G.x0 && gx < (int)G.x_lim &&
                                  (DIM == 2 || (gy >= R && gy < (int)G.y_lim)) && q >= R && q < plane_lim;
            T v = (COEFF == 0) ? slot_value<e>(d1) * c : slot_value<e>(d1);
            if (!interior) {
              const bool in_grid = gx >= 0 && gx < (int)G.xdim && (DIM == 2 || (gy >= 0 && gy < (int)G.ydim)) &&
                                   q >= 0 && q < plane_dim;
              v = in_grid ? G.in[gx + gy * xdim + q * plane_g] : T(0);  // gy = 0 in 2D
            }
            vrow[decltype(ex)::value] = v;
          });
          T* brow = bq + ((DIM == 3) ? (R + ey0 + decltype(ey)::value) * TB_BW : 0) + TB_ML + ex0;
          if constexpr (DIM == 2 && CX % 2 == 0) {
            // TB_ML and ex0 are even: each pair of the thread's row is one aligned access
            static_for<0, CX / 2>([&](auto pp) {
              constexpr int k = 2 * decltype(pp)::value;
              typename PairOf<T>::type v2;
              v2.x = vrow[k];
              v2.y = vrow[k + 1];
              *reinterpret_cast<typename PairOf<T>::type*>(brow + k) = v2;
            });
          } else {
            static_for<0, CX>([&](auto ex) { brow[decltype(ex)::value] = vrow[decltype(ex)::value]; });
          }
        });
        __syncthreads();
        // stage 2: plane q of S(in); completes plane p = q - R of S(S(in)), output pi - 4R
        const TbPlane ldb{bq + ((DIM == 3) ? (R + ey0) * TB_BW : 0) + TB_ML + ex0};
        auto slot2 = [&](auto kk) -> PipeSlot& {
          constexpr int k = decltype(kk)::value;
          return acc2[((t - k) % NP2 + NP2) % NP2];
        };
        pipe_plane(ldb, slot2);
        const int op = pi - 4 * R;
        if (inner && op >= 0 && op < nout) {
          PipeSlot& d2 = acc2[((t - 2 * R) % NP2 + NP2) % NP2];
          const tcs_i64 pz = (tcs_i64)(ms + op) * plane_g;
          if constexpr (DIM == 2 && CX % 2 == 0) {
            // column pairs: one access where both are outputs and the address allows it
            static_for<0, CX / 2>([&](auto pp) {
              constexpr int k = 2 * decltype(pp)::value;
              const int exa = ex0 + k, ox = X0 + exa;
              const T a = (COEFF == 0) ? slot_value<k>(d2) * c : slot_value<k>(d2);
              const T b = (COEFF == 0) ? slot_value<k + 1>(d2) * c : slot_value<k + 1>(d2);
              const bool sa = ox < (int)G.x_lim && exa >= R && exa < TB_EX - R;
              const bool sb = ox + 1 < (int)G.x_lim && exa + 1 >= R && exa + 1 < TB_EX - R;
              T* o = G.out + ox + pz;
              if (sa && sb && G.st_pair && (ox & 1) == 0) {
                typename PairOf<T>::type v2;
                v2.x = a;
                v2.y = b;
                *reinterpret_cast<typename PairOf<T>::type*>(o) = v2;
              } else {
                if (sa) o[0] = a;
                if (sb) o[1] = b;
              }
            });
          } else {
            static_for<0, CY>([&](auto ey) {
              static_for<0, CX>([&](auto ex) {
                constexpr int e = decltype(ex)::value + decltype(ey)::value * CX;
                const int ox = X0 + ex0 + decltype(ex)::value, oy = Y0 + ey0 + decltype(ey)::value;
                constexpr bool EDGE = DIM == 2 && R % CX != 0;  // thread tiles straddling the edge
                const int exx = ex0 + decltype(ex)::value;
                if (ox < (int)G.x_lim && oy < (int)G.y_lim && (!EDGE || (exx >= R && exx < TB_EX - R)))
                  G.out[ox + oy * xdim + pz] = (COEFF == 0) ? slot_value<e>(d2) * c : slot_value<e>(d2);
              });
            });
          }
        }
      }
    });
    if constexpr (CHP % NP2 != 0) {
      PipeSlot tmp[NP2];
      static_for<0, NP2>([&](auto m) { tmp[decltype(m)::value] = acc1[decltype(m)::value]; });
      static_for<0, NP2>([&](auto m) { acc1[decltype(m)::value] = tmp[(decltype(m)::value + CHP) % NP2]; });
      static_for<0, NP2>([&](auto m) { tmp[decltype(m)::value] = acc2[decltype(m)::value]; });
      static_for<0, NP2>([&](auto m) { acc2[decltype(m)::value] = tmp[(decltype(m)::value + CHP) % NP2]; });
    }
    if (++cur_slot == nslot) {
      cur_slot = 0;
      cur_par ^= 1u;
    }
  }
  st.gc = gc + nch;
  return !aborted;
}
}  // namespace tcs

// Work list: (output tile, output plane) items over persistent CTAs, as in tcs_pipe; the plane
// buffer follows the ring in dynamic shared memory.
extern "C" __global__ void __launch_bounds__(TCS_BX * TCS_BY)
    tcs_tb3(const __grid_constant__ TcsTmaMap tmap, const T* __restrict__ in, T* __restrict__ out,
            const TcsPipeGeo g) {
  using namespace tcs;
  PipeGridView G;
  G.map = &tmap;
  G.in = in;
  G.out = out;
  G.src = nullptr;
  G.xdim = g.xdim;
  G.ydim = g.ydim;
  G.zdim = g.zdim;
  G.x0 = g.x0;
  G.x_lim = g.x_lim;
  G.y_lim = g.y_lim;
  G.z_lim = g.z_lim;
  G.ntx = g.ntx;
  G.use_tma = (g.loader == 0);
  G.cp_pair = false;
  // output pairs with one access: even pitch and a pair-aligned base (2D strips)
  G.st_pair = (g.xdim % 2 == 0) && (reinterpret_cast<tcs_u64>(out) % (2 * sizeof(T)) == 0);
  G.src_pair = false;
  G.aux = nullptr;
  if (G.use_tma && threadIdx.x == 0 && threadIdx.y == 0) tma_prefetch_map(&tmap);
  PipeState st = pipe_setup(g.nslot, G.use_tma);
  T* bbuf = st.ring + g.nslot * CHUNK;
  PipeSlot acc1[NP2], acc2[NP2];
  const tcs_u64 w_begin = (tcs_u64)blockIdx.x * g.per_cta;
  const tcs_u64 w_end = min(w_begin + g.per_cta, g.total);
  for (tcs_u64 w = w_begin; w < w_end;) {
    const tcs_u32 tile = (tcs_u32)(w / g.m);
    const tcs_u32 zs = (tcs_u32)(w % g.m);
    const tcs_u32 ze = (tcs_u32)min((tcs_u64)g.m, (tcs_u64)zs + (w_end - w));
    w += ze - zs;
    if (!tb3_piece(G, tile, zs, ze, st, acc1, acc2, bbuf)) return;
  }
}
#endif  // TCS_TB3
#endif  // TCS_PIPE
