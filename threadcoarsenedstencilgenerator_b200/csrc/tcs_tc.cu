// Tensor-core sweep of 2D Box stencils on FP32 grids: the stencil as a banded dense contraction
// on the 5th-generation tensor cores (tcgen05, accumulators in tensor memory).  No counterpart in
// the reference, which sweeps on the FP64 pipe only (cuda/generate2DStencil_cuda.py:146-198).
//
// For an output tile of TM = 128 rows x TN = 32 columns at (y0, x0):
//   out[m][n] = sum_{dy} sum_{k} A_dy[m][k] * B_dy[n][k]
//   A_dy[m][k] = in[y0 + m + dy - R][x0 - R + k]         (k < TN + 2R; zero beyond)
//   B_dy[n][k] = mask[dy][k - n]  for 0 <= k - n <= 2R   (banded Toeplitz; zero elsewhere)
// i.e. one GEMM of M = 128, N = 32, K = (2R+1) * 48 per tile.  Inputs and the mask are split
// into BF16 high and low parts (x = hi + lo + O(2^-17 |x|)); the three products hi*hi, hi*lo and
// lo*hi are accumulated in FP32 in tensor memory.  The Toeplitz operands of all 2R+1 rows are built
// once on the host (tcs_capi.cpp) and stay in shared memory; the A operands of every row offset
// dy are the same shared-memory tile read from a different start row, which the no-swizzle K-major
// operand layout (8-row core matrices with a 16-byte row stride) allows at any row.
//
// Per CTA (persistent, 1 per SM): one warp issues the MMAs; 8 worker warps stage and split the
// input tiles (TMA ring two tiles ahead) and drain finished accumulators (+ source term) through
// a shared transpose buffer, so that a tile's MMAs overlap the previous tile's drain and the next
// tile's staging.  The roles hand tiles over through mbarriers only.  Every mbarrier wait is
// bounded; on expiry the CTA records TCS_DEV_TIMEOUT, waits (bounded) for its MMAs in flight,
// frees its tensor memory and returns.

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "tcs_field.h"

namespace {

constexpr int TM = 128;           // output rows per tile (MMA M)
constexpr int TN = 32;            // output columns per tile (MMA N)
constexpr int KD = 48;            // operand columns per row offset: TN + 2R <= 48 for R <= 8
constexpr int NCH = KD / 8;       // 16-byte core-matrix columns per row offset
constexpr int NTHREADS = 256;
constexpr int TC_MAX_R = 8;
constexpr unsigned DEV_TIMEOUT = 1u;
constexpr long long WAIT_LIMIT = 1000000000ll;  // cycles

// Instruction descriptor, kind::f16: D FP32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1),
// both K-major (bits 15, 16 = 0), N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: no swizzle, K-major.  Start address, LBO (distance between the
// two 16-byte K halves of an MMA) and SBO (distance between 8-row core-matrix groups), all >> 4;
// bits 46-47 = 1 (the descriptor version of sm_100).
__device__ __forceinline__ uint64_t make_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

template <int N>
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
      "}"
      :
      : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc(N)), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void bar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool bar_try(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait; true when the limit expired.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
  if (bar_try(bar, parity)) return false;
  const long long t0 = clock64();
  while (!bar_try(bar, parity))
    if (clock64() - t0 > WAIT_LIMIT) return true;
  return false;
}

// 16 consecutive accumulator columns of this thread's lane (no wait: see tmem_wait_ld).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
      "%13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15])
      : "r"(taddr)
      : "memory");
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 2D TMA tile load (no multicast) completing on an mbarrier.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const void* map, uint32_t bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void bar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 a, __nv_bfloat16 b) {
  return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

// Load the input rows of one tile and store their BF16 high and low parts in the operand layout:
// element (row r, column k) at (k / 8) * cs + r * 16 + (k % 8) * 2 bytes.
__device__ __forceinline__ void load_split(const float* __restrict__ in, const TcsTcGeo& g, unsigned tile,
                                           unsigned char* a_hi, unsigned char* a_lo, unsigned rows,
                                           unsigned cs, unsigned tid) {
  const unsigned R = g.R;
  const unsigned ty = tile / g.ntx, tx = tile - ty * g.ntx;
  const unsigned long long gy0 = (unsigned long long)ty * TM;  // input row of operand row 0
  const unsigned gx0 = g.x0 + tx * TN - R;                       // input column of operand column 0
  const unsigned kvalid = TN + 2 * R;
  for (unsigned q = tid; q < rows * (KD / 4); q += NTHREADS) {
    const unsigned r = q / (KD / 4), grp = q - r * (KD / 4);
    const unsigned k = grp * 4;
    const unsigned long long gy = gy0 + r;
    float v[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const unsigned long long gx = (unsigned long long)gx0 + k + e;
      v[e] = (k + e < kvalid && gy < g.ydim && gx < g.xdim) ? __ldg(in + gy * g.xdim + gx) : 0.f;
    }
    __nv_bfloat16 h[4], l[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      h[e] = __float2bfloat16_rn(v[e]);
      l[e] = __float2bfloat16_rn(v[e] - __bfloat162float(h[e]));
    }
    const unsigned off = (k / 8) * cs + r * 16 + (k % 8) * 2;
    *reinterpret_cast<uint2*>(a_hi + off) = make_uint2(pack_bf16(h[0], h[1]), pack_bf16(h[2], h[3]));
    *reinterpret_cast<uint2*>(a_lo + off) = make_uint2(pack_bf16(l[0], l[1]), pack_bf16(l[2], l[3]));
  }
}

// Split a staged FP32 tile (rows x KD floats, row-major) into the BF16 operand layout.  Columns
// k >= TN + 2R hold real neighbours or TMA's zero fill; their Toeplitz weights are zero.
__device__ __forceinline__ void split_staged(const float* __restrict__ stage, unsigned char* a_hi,
                                             unsigned char* a_lo, unsigned rows, unsigned cs, unsigned tid) {
  for (unsigned q = tid; q < rows * (KD / 4); q += NTHREADS) {
    const unsigned r = q / (KD / 4), k = (q - r * (KD / 4)) * 4;
    const float4 f = *reinterpret_cast<const float4*>(stage + r * KD + k);
    const float v[4] = {f.x, f.y, f.z, f.w};
    __nv_bfloat16 h[4], l[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      h[e] = __float2bfloat16_rn(v[e]);
      l[e] = __float2bfloat16_rn(v[e] - __bfloat162float(h[e]));
    }
    const unsigned off = (k / 8) * cs + r * 16 + (k % 8) * 2;
    *reinterpret_cast<uint2*>(a_hi + off) = make_uint2(pack_bf16(h[0], h[1]), pack_bf16(h[2], h[3]));
    *reinterpret_cast<uint2*>(a_lo + off) = make_uint2(pack_bf16(l[0], l[1]), pack_bf16(l[2], l[3]));
  }
}

struct __align__(64) TcTmaMap {
  uint64_t w[16];
};

// Byte distance between the 16-byte columns of an A operand: the rows (16 bytes each) padded so
// that successive columns start 16 bytes apart modulo 128 -- the split's stores of neighbouring
// columns then fall into different shared-memory banks.  At range 8 the padding would not fit in
// shared memory and the columns stay unpadded.  Either way 24 columns (the 4 operand buffers) are
// a multiple of 128 bytes, which keeps the staging slots behind them aligned for TMA.
__host__ __device__ constexpr unsigned col_stride(unsigned rows) {
  return rows <= 142 ? ((rows * 16 + 127) / 128) * 128 + 16 : rows * 16;
}

constexpr int NWORK = NTHREADS / 32;  // worker warps
constexpr int BLOCK = NTHREADS + 32;  // + the MMA warp
// Successive MMAs into one accumulator wait for each other, and an N = 32 MMA is short: every tile
// spreads its MMAs over NACC independent accumulators -- (hi*hi, hi*lo, lo*hi) x (even, odd row
// offset) -- that the epilogue sums.  Two tiles in flight: 2 x NACC x 32 = 384 of 512 TMEM columns.
constexpr int NACC = 6;
constexpr uint32_t TMEM_COLS = 512;

// Shared state of one CTA.
struct TcShared {
  uint64_t full[2];      // staging slot filled (TMA bytes)
  uint64_t aready[2];    // operand buffer written by all workers
  uint64_t mdone[2];     // MMAs of the accumulator complete (tcgen05.commit)
  uint64_t afree[2];     // accumulator drained by all workers
  uint32_t tmem;         // tensor-memory base of the two accumulators
  volatile uint32_t abort_flag;
};

// Bounded wait that also gives up when another role has aborted; true = give up.
__device__ __forceinline__ bool role_wait(TcShared* S, uint64_t* bar, uint32_t parity, unsigned* status) {
  const uint32_t a = smem_u32(bar);
  if (bar_try(a, parity)) return false;
  const long long t0 = clock64();
  while (!bar_try(a, parity)) {
    if (S->abort_flag) return true;
    if (clock64() - t0 > WAIT_LIMIT) {
      S->abort_flag = 1;
      atomicOr(status, DEV_TIMEOUT);
      return true;
    }
  }
  return false;
}

__device__ __forceinline__ void bar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void workers_sync() {  // named barrier 1 over the worker warps
  asm volatile("bar.sync 1, %0;" ::"r"(NTHREADS) : "memory");
}

// Named barrier 1 with an OR over the worker warps: every worker takes the same branch after it,
// so no worker can be left waiting at a later barrier that the others skip.
__device__ __forceinline__ bool workers_any(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.or.pred p, 1, %2, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(NTHREADS)
      : "memory");
  return r != 0;
}

// Warp-specialised persistent CTA: warps 0-7 stage, split and drain tiles; warp 8 issues the
// tensor-core MMAs.  Tile j of the CTA uses staging slot, operand buffer and accumulator j % 2,
// and the k-th use of a barrier slot waits on parity k & 1.  With USE_TMA the input tiles stream
// through a 2-slot FP32 staging ring filled by TMA two tiles ahead (needs a 16-byte row pitch, base
// and tile start); otherwise the workers load their part of each tile directly.
template <bool USE_TMA>
__global__ void __launch_bounds__(BLOCK, 1)
    tcs_tc_box2d(const __grid_constant__ TcTmaMap tmap, const float* __restrict__ in,
                 const float* __restrict__ src, float* __restrict__ out, const uint4* __restrict__ bops,
                 const TcsTcGeo g, unsigned* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  // TMA destinations need 128-byte alignment: round the base (the launch adds 128 bytes of slack)
  unsigned char* sm = sm_raw + ((128u - (smem_u32(sm_raw) & 127u)) & 127u);
  const unsigned tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const unsigned R = g.R, D = 2 * R + 1, rows = TM + 2 * R;
  const unsigned cs = col_stride(rows);          // A operand: bytes per 16-byte column
  // B operand of row offset dy: 16-byte column c holds rows 0-31 (BF16 high parts of the Toeplitz
  // rows n) then rows 32-63 (low parts), so one N = 64 MMA multiplies A_hi by both.
  const unsigned bcol = 2 * TN * 16;             // 1024 bytes per 16-byte column
  const unsigned bdy = NCH * bcol;               // 6144 bytes per row offset
  TcShared* S = reinterpret_cast<TcShared*>(sm);
  unsigned char* b_ops = sm + 128;
  unsigned char* a_base = b_ops + D * bdy;
  const unsigned abytes = NCH * cs;  // 4 buffers = 24 cs, a multiple of 128
  auto a_hi = [&](unsigned b) { return a_base + (2 * b) * abytes; };
  auto a_lo = [&](unsigned b) { return a_base + (2 * b + 1) * abytes; };
  const unsigned sbytes = ((rows * KD * 4 + 127) / 128) * 128;
  auto stage = [&](unsigned b) { return reinterpret_cast<float*>(a_base + 4 * abytes + b * sbytes); };
  float* obuf = reinterpret_cast<float*>(a_base + 4 * abytes + 2 * sbytes);  // TM x (TN + 1) floats

  const unsigned total = g.ntx * g.nty;
  const unsigned step = gridDim.x;
  const unsigned mine = total > blockIdx.x ? (total - blockIdx.x + step - 1) / step : 0;

  // Toeplitz operands (prebuilt bit patterns, hi then lo) into shared memory.
  for (unsigned i = tid; i < D * bdy / 16; i += BLOCK) reinterpret_cast<uint4*>(b_ops)[i] = bops[i];
  if (tid == 0) {
    for (int k = 0; k < 2; ++k) {
      bar_init(smem_u32(&S->full[k]), 1);
      bar_init(smem_u32(&S->aready[k]), NTHREADS);
      bar_init(smem_u32(&S->mdone[k]), 1);
      bar_init(smem_u32(&S->afree[k]), NTHREADS);
    }
    S->abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == NWORK) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S->tmem)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = S->tmem;

  if (warp == NWORK) {
    // ---- MMA warp: one lane issues every tile's 117 (for R = 6) MMAs ----
    unsigned issued = 0;
    if (lane == 0) {
      // Descriptors differ only in their start-address field (bits 0-13, 16-byte units): advance
      // them by adding offset >> 4 (every operand lies below 256 KB, so the field cannot carry).
      const uint64_t b0 = make_desc(smem_u32(b_ops), bcol, 128);
      for (unsigned j = 0; j < mine; ++j) {
        const unsigned b = j & 1u;
        if (role_wait(S, &S->aready[b], (j >> 1) & 1u, status)) break;
        if (j >= 2 && role_wait(S, &S->afree[b], ((j - 2) >> 1) & 1u, status)) break;
        fence_after();
        const uint64_t ah0 = make_desc(smem_u32(a_hi(b)), cs, 128), al0 = make_desc(smem_u32(a_lo(b)), cs, 128);
        for (unsigned dy = 0; dy < D; ++dy) {
          // accumulators of this row-offset parity: [hi*hi | hi*lo] (64 columns), lo*hi (32)
          const uint32_t d = tmem + (b * NACC + (dy & 1u) * 3) * TN;
#pragma unroll
          for (unsigned s = 0; s < KD / 16; ++s) {
            const uint64_t ao = (2 * s * cs + dy * 16) >> 4;  // start row dy, K columns 2s, 2s+1
            const uint64_t bo = (dy * bdy + 2 * s * bcol) >> 4;
            const uint32_t acc = (dy >= 2 || s > 0) ? 1u : 0u;  // first product of each accumulator
            mma_bf16<2 * TN>(d, ah0 + ao, b0 + bo, acc);
            mma_bf16<TN>(d + 2 * TN, al0 + ao, b0 + bo, acc);
          }
        }
        mma_commit(smem_u32(&S->mdone[b]));
        ++issued;
      }
      if (S->abort_flag) {  // let the MMAs in flight finish before the memory is released
        for (unsigned k = issued >= 2 ? issued - 2 : 0; k < issued; ++k)
          (void)bar_wait(smem_u32(&S->mdone[k & 1u]), (k >> 1) & 1u);
      }
    }
    __syncwarp();
  } else {
    // ---- worker warps ----
    const uint32_t stage_bytes = rows * KD * 4;
    unsigned fetched = 0, consumed = 0;  // TMA tiles issued (thread 0) / waited for
    auto fetch = [&](unsigned j) {  // TMA of this CTA's j-th tile into staging slot j % 2
      if (j >= mine) return;
      fetched = j + 1;
      const unsigned tile = blockIdx.x + j * step;
      const unsigned ty = tile / g.ntx, tx = tile - ty * g.ntx;
      const uint32_t bar = smem_u32(&S->full[j & 1u]);
      bar_expect_tx(bar, stage_bytes);
      tma_load_2d(smem_u32(stage(j & 1u)), &tmap, bar, (int)(g.x0 + tx * TN - R), (int)(ty * TM));
    };
    // Operands of tile j into buffer j % 2, then arrive on aready; false = give up.
    auto prepare = [&](unsigned j) -> bool {
      if (USE_TMA) {
        if (workers_any(role_wait(S, &S->full[j & 1u], (j >> 1) & 1u, status))) return false;
        consumed = j + 1;
        split_staged(stage(j & 1u), a_hi(j & 1u), a_lo(j & 1u), rows, cs, tid);
      } else {
        load_split(in, g, blockIdx.x + j * step, a_hi(j & 1u), a_lo(j & 1u), rows, cs, tid);
      }
      fence_proxy_async();
      bar_arrive(&S->aready[j & 1u]);
      // every worker finished reading staging slot j % 2 and the transpose buffer of the last tile
      workers_sync();
      if (USE_TMA && tid == 0) fetch(j + 2);
      return true;
    };
    bool ok = true;
    if (USE_TMA && tid == 0) {
      fetch(0);
      fetch(1);
    }
    if (mine > 0) ok = prepare(0);
    if (ok && mine > 1) ok = prepare(1);
    for (unsigned j = 0; ok && j < mine; ++j) {
      const unsigned b = j & 1u;
      const unsigned t = blockIdx.x + j * step;
      const unsigned ty = t / g.ntx, tx = t - ty * g.ntx;
      const unsigned x = g.x0 + tx * TN + lane;
      const unsigned long long ybase = (unsigned long long)R + (unsigned long long)ty * TM;
      // the source term of this worker's outputs, loaded while the tensor core works
      float sv[TM / NWORK];
#pragma unroll
      for (unsigned i = 0; i < TM / NWORK; ++i) {
        const unsigned long long y = ybase + warp + i * NWORK;
        sv[i] = (src && x < g.x_lim && y < g.y_lim) ? __ldg(src + y * g.xdim + x) : 0.f;
      }
      if (workers_any(role_wait(S, &S->mdone[b], (j >> 1) & 1u, status))) break;
      fence_after();
      // drain accumulator b: warp w reads TMEM lanes 32 (w % 4) .., columns 16 (w / 4) .. (one
      // output row per thread) into a transpose buffer; then each warp writes whole rows of 32
      // outputs, one coalesced 128-byte access per row (+ the source term, read the same way).
      {
        const unsigned q = warp % 4, h = warp / 4;
        const uint32_t base = tmem + ((32u * q) << 16) + b * NACC * TN + 16u * h;
        uint32_t r[NACC][16];
#pragma unroll
        for (int a = 0; a < NACC; ++a) tmem_ld16(base + a * TN, r[a]);
        tmem_wait_ld();
        float* row = obuf + (32u * q + lane) * (TN + 1) + 16u * h;
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          // (hh + hl + lh) of the even row offsets, then of the odd ones
          const float ev = (__uint_as_float(r[0][e]) + __uint_as_float(r[1][e])) + __uint_as_float(r[2][e]);
          const float od = (__uint_as_float(r[3][e]) + __uint_as_float(r[4][e])) + __uint_as_float(r[5][e]);
          row[e] = ev + od;
        }
      }
      fence_before();
      bar_arrive(&S->afree[b]);  // accumulator b may be overwritten by tile j + 2
      workers_sync();
      if (x < g.x_lim) {
#pragma unroll
        for (unsigned i = 0; i < TM / NWORK; ++i) {
          const unsigned m = warp + i * NWORK;
          const unsigned long long y = ybase + m;
          if (y < g.y_lim) out[y * g.xdim + x] = obuf[m * (TN + 1) + lane] + sv[i];
        }
      }
      // operand buffer b is free (MMAs of tile j done): stage tile j + 2 into it
      if (j + 2 < mine) ok = prepare(j + 2);
      else workers_sync();  // the transpose buffer is rewritten by the next tile
    }
    if (S->abort_flag && USE_TMA && tid == 0) {  // TMA copies in flight land before the CTA leaves
      for (unsigned k = consumed; k < fetched; ++k) (void)bar_wait(smem_u32(&S->full[k & 1u]), (k >> 1) & 1u);
    }
  }
  fence_before();
  __syncthreads();
  if (warp == NWORK) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

}  // namespace

extern "C" unsigned tcs_tc_smem_bytes(unsigned R) {
  const unsigned D = 2 * R + 1, rows = TM + 2 * R, cs = col_stride(rows);
  const unsigned abytes = NCH * cs;  // 4 buffers = 24 cs, a multiple of 128
  const unsigned sbytes = ((rows * KD * 4 + 127) / 128) * 128;
  return 128 + 128 + D * (NCH * 2 * TN * 16) + 4 * abytes + 2 * sbytes + TM * (TN + 1) * 4;
}

extern "C" unsigned tcs_tc_box_rows(unsigned R) { return TM + 2 * R; }

extern "C" int tcs_tc_launch(const float* in, const float* src, float* out, const void* bops, const void* map,
                             TcsTcGeo g, unsigned* status, int nctas, cudaStream_t st) {
  if (g.R < 1 || g.R > TC_MAX_R) return (int)cudaErrorInvalidValue;
  const unsigned smem = tcs_tc_smem_bytes(g.R);
  TcTmaMap m;
  if (map) {
    memcpy(&m, map, sizeof(m));
  } else {
    memset(&m, 0, sizeof(m));
  }
  auto kern = map ? tcs_tc_box2d<true> : tcs_tc_box2d<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return (int)e;
  const unsigned total = g.ntx * g.nty;
  const unsigned grid = (unsigned)nctas < total ? (unsigned)nctas : total;
  kern<<<grid ? grid : 1, BLOCK, smem, st>>>(m, in, src, out, reinterpret_cast<const uint4*>(bops), g, status);
  return (int)cudaGetLastError();
}
