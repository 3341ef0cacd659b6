// Per-thread arithmetic of the thread-coarsened stencil sweep (included by tcs_kernels.cuh).
//
// Everything here is plain C++ on registers: the footprint traversal of one thread tile in the
// reference generator's order, the mask layout, the first-term initialisation and the fused
// multiply-adds.  The caller supplies a loader `ld(gx, gy, gz)` returning the grid value at a
// thread-relative offset (from global memory, a shared-memory ring, ...).  With the TCS_* macros
// fixed at compile time every loop unrolls and every branch folds, which turns this into the
// straight-line register code the reference generates as text
// (cuda/generate2DStencil_cuda.py:107-198, cuda/generate3DStencil_cuda.py:116-218).
//
// The header has no CUDA-only dependencies besides the __device__/__constant__ qualifiers and the
// __fma_rn intrinsics, so a host harness can compile it with those mapped to plain C++.

#pragma once

#ifndef TCS_T
#error "TCS_T must be defined by the instantiation layer"
#endif

typedef unsigned long long tcs_u64;
typedef unsigned int tcs_u32;
typedef long long tcs_i64;
typedef TCS_T T;

namespace tcs {
constexpr int DIM = TCS_DIM;
constexpr int SHAPE = TCS_SHAPE;
constexpr int ORIENT = TCS_ORIENT;
constexpr int COEFF = TCS_COEFF;
constexpr int R = TCS_R;
constexpr int CX = TCS_CX;
constexpr int CY = TCS_CY;
constexpr int CZ = (TCS_DIM == 3) ? TCS_CZ : 1;
constexpr int NE = CX * CY * CZ;            // outputs per thread
constexpr int W1 = 2 * R + 1;
// stencilSize as in cuda/generate2DStencil_cuda.py:63-67 and cuda/generate3DStencil_cuda.py:66-70
constexpr int S = (SHAPE == 0) ? (DIM == 2 ? W1 * W1 : W1 * W1 * W1) : (2 * DIM * R + 1);
constexpr int VEC = 16 / (int)sizeof(T);    // elements per 16-byte TMA granule
#ifndef TCS_COMP
#define TCS_COMP 0
#endif
// Compensated accumulation (FP32 grids, precision TCS_F32C): every output keeps a running sum and
// the rounding errors of its additions (Knuth's two-sum) and of its products (fma(v, m, -v*m)),
// added back at the end.  The terms still arrive in the reference's order.
constexpr bool COMP = TCS_COMP != 0;
struct CompAcc {
  T s, c;
};
template <bool B, class X, class Y>
struct pick {
  typedef X type;
};
template <class X, class Y>
struct pick<false, X, Y> {
  typedef Y type;
};
typedef typename pick<COMP, CompAcc, T>::type Acc;  // one output's accumulator
}  // namespace tcs

// Stencil coefficients (Variable); the reference's `__constant__ double d_mask[S]`.
__constant__ T tcs_mask[tcs::S];

namespace tcs {

__device__ __forceinline__ constexpr int iabs(int v) { return v < 0 ? -v : v; }

// Fused multiply-add with a single rounding, for either element type.
__device__ __forceinline__ double fmat(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fmat(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// Linear mask index of relative offset (rx, ry[, rz]); calcMaskAddress in
// cuda/generate2DStencil_cuda.py:120-144 and cuda/generate3DStencil_cuda.py:132-169.
__device__ __forceinline__ constexpr int mask_index(int rx, int ry, int rz) {
  if (SHAPE == 0) {
    return (DIM == 2) ? (rx + R) + (ry + R) * W1 : (rx + R) + (ry + R) * W1 + (rz + R) * W1 * W1;
  }
  if (DIM == 2) {
    if (rx == 0 && ry < 0) return ry + R;
    if (ry == 0) return rx + 2 * R;
    return ry + 3 * R;  // rx == 0 && ry > 0
  }
  if (rz < 0) return rz + R;
  if (rz == 0 && rx == 0 && ry < 0) return ry + 2 * R;
  if (rz == 0 && ry == 0) return rx + 3 * R;
  if (rz == 0 && rx == 0 && ry > 0) return ry + 4 * R;
  return rz + 5 * R;  // rz > 0
}

// Does the grid point at offset (rx, ry, rz) from an output belong to its neighbourhood?
// (printAdditions, cuda/generate2DStencil_cuda.py:175-186, cuda/generate3DStencil_cuda.py:201-212)
__device__ __forceinline__ constexpr bool contributes(int rx, int ry, int rz) {
  if (SHAPE == 0) return iabs(rx) <= R && iabs(ry) <= R && (DIM == 2 || iabs(rz) <= R);
  if (DIM == 2) return (iabs(rx) <= R && ry == 0) || (iabs(ry) <= R && rx == 0);
  return (iabs(rx) <= R && ry == 0 && rz == 0) || (iabs(ry) <= R && rx == 0 && rz == 0) ||
         (iabs(rz) <= R && rx == 0 && ry == 0);
}

// Is it the first term of that output (initialised, not added)?
// (cuda/generate2DStencil_cuda.py:179,188-195, cuda/generate3DStencil_cuda.py:205,214)
__device__ __forceinline__ constexpr bool is_first(int rx, int ry, int rz) {
  if (SHAPE == 0) return rx == -R && ry == -R && (DIM == 2 || rz == -R);
  if (DIM == 2) return (ORIENT == 1) ? (ry == 0 && rx == -R) : (rx == 0 && ry == -R);
  return rx == 0 && ry == 0 && rz == -R;
}

// The second term of every output in the reference's per-output order (that order does not
// depend on the coarsening factors: it is the traversal of a 1x1[x1] tile).
__device__ __forceinline__ constexpr bool is_second(int rx, int ry, int rz) {
  if (SHAPE == 0) {
    if (DIM == 2)
      return (ORIENT == 0) ? (rx == -R + 1 && ry == -R) : (rx == -R && ry == -R + 1);
    return (ORIENT == 0) ? (rx == -R + 1 && ry == -R && rz == -R) : (rx == -R && ry == -R + 1 && rz == -R);
  }
  if (DIM == 2) {
    if (ORIENT == 0) return (R >= 2) ? (rx == 0 && ry == -R + 1) : (rx == -1 && ry == 0);
    return (R >= 2) ? (rx == -R + 1 && ry == 0) : (rx == 0 && ry == -1);
  }
  if (R >= 2) return rx == 0 && ry == 0 && rz == -R + 1;
  return (ORIENT == 0) ? (rx == 0 && ry == -1 && rz == 0) : (rx == -1 && ry == 0 && rz == 0);
}

// Mask index of the first term of every output.
__device__ __forceinline__ constexpr int first_mask_index() {
  if (SHAPE == 0) return mask_index(-R, -R, -R);
  if (DIM == 2) return (ORIENT == 1) ? mask_index(-R, 0, 0) : mask_index(0, -R, 0);
  return mask_index(0, 0, -R);
}

// Compile-time loops.  Every footprint offset and element index below is a template constant,
// so the traversal is straight-line code by construction (the reference generates it as text);
// relying on #pragma unroll for these deep nests leaves outer loops rolled and turns offsets,
// mask indices and first-term tests into run-time arithmetic.
template <int V>
struct ic {
  static constexpr int value = V;
};

template <int I, int N, class F>
__device__ __forceinline__ void static_for(F&& f) {
  if constexpr (I < N) {
    f(ic<I>{});
    static_for<I + 1, N>(f);
  }
}

// Apply the value v loaded from thread-relative (GX, GY, GZ) to every output it touches.
// Variable stencils keep the first value v0 of an output in its accumulator until the second
// term arrives and then form fma(v0, m0, v1*m1): the nvcc -fmad=true fusion of the reference's
// `result = v0*m0; result += v1*m1;` (an add of two products fuses its left operand).
__device__ __forceinline__ void two_sum_add(CompAcc& a, const T p, const T ep) {
  const T t = a.s + p;
  const T z = t - a.s;
  a.c = a.c + ((a.s - (t - z)) + (p - z) + ep);
  a.s = t;
}
__device__ __forceinline__ T acc_value(const T& a) { return a; }
__device__ __forceinline__ T acc_value(const CompAcc& a) { return a.s + a.c; }
__device__ __forceinline__ void acc_zero(T& a) { a = T(0); }
__device__ __forceinline__ void acc_zero(CompAcc& a) { a.s = T(0); a.c = T(0); }
// First term: the plain accumulator holds v (a Variable product forms at the second term); the
// compensated one starts from v*m and its rounding error (m = 1 for Jacobi).
__device__ __forceinline__ void acc_first(T& a, const T v, const T) { a = v; }
__device__ __forceinline__ void acc_first(CompAcc& a, const T v, const T m) {
  a.s = v * m;
  a.c = fmat(v, m, -a.s);
}
__device__ __forceinline__ void acc_add(T& a, const T v) { a = a + v; }
__device__ __forceinline__ void acc_add(CompAcc& a, const T v) { two_sum_add(a, v, T(0)); }
__device__ __forceinline__ void acc_fma(T& a, const T v, const T m) { a = fmat(v, m, a); }
__device__ __forceinline__ void acc_fma(CompAcc& a, const T v, const T m) {
  const T p = v * m;
  two_sum_add(a, p, fmat(v, m, -p));
}
// Second Variable term: fma(v0, m0, fl(v1*m1)) for the plain accumulator; for the compensated one
// the first product is already formed.
__device__ __forceinline__ void acc_second(T& a, const T m0, const T v, const T m) { a = fmat(a, m0, v * m); }
__device__ __forceinline__ void acc_second(CompAcc& a, const T, const T v, const T m) { acc_fma(a, v, m); }

template <int GX, int GY, int GZ>
__device__ __forceinline__ void apply(Acc (&acc)[NE], const T v) {
  static_for<0, CZ>([&](auto ez) {
    static_for<0, CY>([&](auto ey) {
      static_for<0, CX>([&](auto ex) {
        constexpr int rx = GX - decltype(ex)::value;
        constexpr int ry = GY - decltype(ey)::value;
        constexpr int rz = GZ - decltype(ez)::value;
        constexpr int e = decltype(ex)::value + decltype(ey)::value * CX + decltype(ez)::value * CX * CY;
        if constexpr (contributes(rx, ry, rz)) {
          if constexpr (is_first(rx, ry, rz)) {
            acc_first(acc[e], v, (COEFF == 0) ? T(1) : tcs_mask[mask_index(rx, ry, rz)]);
          } else if constexpr (COEFF == 0) {
            acc_add(acc[e], v);
          } else if constexpr (is_second(rx, ry, rz)) {
            acc_second(acc[e], tcs_mask[first_mask_index()], v, tcs_mask[mask_index(rx, ry, rz)]);
          } else {
            acc_fma(acc[e], v, tcs_mask[mask_index(rx, ry, rz)]);
          }
        }
      });
    });
  });
}

template <int GX, int GY, int GZ, class LD>
__device__ __forceinline__ void point(const LD& ld, Acc (&acc)[NE]) {
  apply<GX, GY, GZ>(acc, ld(GX, GY, GZ));
}

// Footprint traversal of one thread tile in the reference's order
// (cuda/generate2DStencil_cuda.py:244-297, cuda/generate3DStencil_cuda.py:265-360).
// Loops run over [-R, ...) as [0, ...) shifted by R.
template <int GZ, class LD>
__device__ __forceinline__ void traverse_slice(const LD& ld, Acc (&acc)[NE]) {
  // one z slice of a Box stencil (or the whole 2D Box stencil with GZ = 0)
  if constexpr (ORIENT == 1) {
    static_for<0, 2 * R + CX>([&](auto ix) {
      static_for<0, 2 * R + CY>([&](auto iy) {
        point<decltype(ix)::value - R, decltype(iy)::value - R, GZ>(ld, acc);
      });
    });
  } else {
    static_for<0, 2 * R + CY>([&](auto iy) {
      static_for<0, 2 * R + CX>([&](auto ix) {
        point<decltype(ix)::value - R, decltype(iy)::value - R, GZ>(ld, acc);
      });
    });
  }
}

template <int GZ, class LD>
__device__ __forceinline__ void traverse_cross(const LD& ld, Acc (&acc)[NE]) {
  // the in-slice cross of a Star stencil
  if constexpr (ORIENT == 1) {
    static_for<0, R>([&](auto i) {  // gx in [-R, 0)
      static_for<0, CY>([&](auto gy) { point<decltype(i)::value - R, decltype(gy)::value, GZ>(ld, acc); });
    });
    static_for<0, CX>([&](auto gx) {  // gy in [-R, R + CY)
      static_for<0, 2 * R + CY>([&](auto i) { point<decltype(gx)::value, decltype(i)::value - R, GZ>(ld, acc); });
    });
    static_for<0, R>([&](auto i) {  // gx in [CX, CX + R)
      static_for<0, CY>([&](auto gy) { point<CX + decltype(i)::value, decltype(gy)::value, GZ>(ld, acc); });
    });
  } else {
    static_for<0, R>([&](auto i) {  // gy in [-R, 0)
      static_for<0, CX>([&](auto gx) { point<decltype(gx)::value, decltype(i)::value - R, GZ>(ld, acc); });
    });
    static_for<0, CY>([&](auto gy) {  // gx in [-R, R + CX)
      static_for<0, 2 * R + CX>([&](auto i) { point<decltype(i)::value - R, decltype(gy)::value, GZ>(ld, acc); });
    });
    static_for<0, R>([&](auto i) {  // gy in [CY, CY + R)
      static_for<0, CX>([&](auto gx) { point<decltype(gx)::value, CY + decltype(i)::value, GZ>(ld, acc); });
    });
  }
}

template <int GZ, class LD>
__device__ __forceinline__ void traverse_column(const LD& ld, Acc (&acc)[NE]) {
  // the thread's own columns in a z slice outside the centre (Star, 3D)
  if constexpr (ORIENT == 1) {
    static_for<0, CX>([&](auto gx) {
      static_for<0, CY>([&](auto gy) { point<decltype(gx)::value, decltype(gy)::value, GZ>(ld, acc); });
    });
  } else {
    static_for<0, CY>([&](auto gy) {
      static_for<0, CX>([&](auto gx) { point<decltype(gx)::value, decltype(gy)::value, GZ>(ld, acc); });
    });
  }
}

template <class LD>
__device__ __forceinline__ void traverse(const LD& ld, Acc (&acc)[NE]) {
#pragma unroll
  for (int e = 0; e < NE; ++e) acc_zero(acc[e]);
  if constexpr (DIM == 2) {
    if constexpr (SHAPE == 0)
      traverse_slice<0>(ld, acc);
    else
      traverse_cross<0>(ld, acc);
  } else if constexpr (SHAPE == 0) {
    static_for<0, 2 * R + CZ>([&](auto iz) { traverse_slice<decltype(iz)::value - R>(ld, acc); });
  } else {
    static_for<0, R>([&](auto iz) { traverse_column<decltype(iz)::value - R>(ld, acc); });   // in front
    static_for<0, CZ>([&](auto gz) { traverse_cross<decltype(gz)::value>(ld, acc); });      // centre
    static_for<0, R>([&](auto iz) { traverse_column<CZ + decltype(iz)::value>(ld, acc); });  // behind
  }
}

// Write the tile back; Jacobi scales by c = fl(1/S) (cuda/generate2DStencil_cuda.py:300-315).
// An optional source array `src` (same layout, positioned like `o`) is added after the stencil
// value: out = stencil(in) + src.  Sweeps without a source (src == nullptr, every drop-in sweep)
// store the reference's value unchanged.
__device__ __forceinline__ void store(T* __restrict__ o, const Acc (&acc)[NE], tcs_u64 xdim,
                                      tcs_u64 plane, const T* __restrict__ src = nullptr) {
  constexpr T c = T(1) / T(S);
#pragma unroll
  for (int ez = 0; ez < CZ; ++ez)
#pragma unroll
    for (int ey = 0; ey < CY; ++ey)
#pragma unroll
      for (int ex = 0; ex < CX; ++ex) {
        const int e = ex + ey * CX + ez * CX * CY;
        const tcs_i64 off = (tcs_i64)ex + (tcs_i64)ey * (tcs_i64)xdim + (tcs_i64)ez * (tcs_i64)plane;
        T v = (COEFF == 0) ? acc_value(acc[e]) * c : acc_value(acc[e]);
        if (src) v = v + src[off];
        o[off] = v;
      }
}

}  // namespace tcs

// ---- pipeline arithmetic (tcs_pipe) -------------------------------------------------------------
// In the pipelined sweep a thread owns CX x CY (3D) or CX (2D) outputs per plane along the march
// axis and keeps 2R+1 output planes in flight.  The term an input point contributes to the
// output in pipeline slot DZ (the march-axis offset from that output) is (rx, ry, rz) =
// (GX - ex, GY - ey, DZ) in 3D and (GX - ex, DZ, 0) in 2D (the march axis is y there).
namespace tcs {
constexpr int NEP = (DIM == 3) ? CX * CY : CX;  // outputs per thread and plane

// Packed FP32 arithmetic (sm_100 `fma.rn.f32x2`, `add`/`mul` likewise): one instruction applies a
// term to two outputs, each lane rounded exactly as the scalar fmaf/add/mul, so results stay
// bit-identical.  Used for FP32 Box stencils in Row order with an even x coarsening: the outputs
// (2p, 2p+1) of a thread row receive the same term (rx, ry, rz) -- same mask coefficient -- from
// the neighbouring input values (row[2p + rx + R], row[2p + 1 + rx + R]).
#ifndef TCS_PAIRS
#define TCS_PAIRS 1
#endif
constexpr bool PAIRS = (TCS_PAIRS != 0) && sizeof(T) == 4 && SHAPE == 0 && CX % 2 == 0 &&
                       (DIM == 2 || ORIENT == 0);
constexpr int NPAIR = (NEP / 2 > 0) ? NEP / 2 : 1;
}  // namespace tcs

// The packed path's coefficients as pairs (m_k, m_k): a term's broadcast operand of the packed
// fma is one 64-bit constant read instead of a pair assembled in registers.  The host fills it
// from the same mask as tcs_mask (pipelined modules that declare it with S entries).
__constant__ float2 tcs_mask_pairs[tcs::PAIRS ? tcs::S : 1];

namespace tcs {
__device__ __forceinline__ float2 mask_pair(int k) { return tcs_mask_pairs[k]; }

// The accumulators of one output plane of a thread: NEP scalars, or NEP/2 packed pairs (output
// e = ex + ey*CX is lane e%2 of pair e/2).  The compensated form (FP32 grids, TCS_COMP) keeps, per
// pair, the running sum `p` and the collected rounding errors `c`; the value is p + c.
template <bool P, bool C>
struct PipeSlotT {
  T v[NEP];
  template <int E>
  __device__ __forceinline__ T& at() { return v[E]; }
};
template <>
struct PipeSlotT<true, false> {
  float2 p[NPAIR];
  template <int E>
  __device__ __forceinline__ float& at() {
    if constexpr (E % 2 == 0)
      return p[E / 2].x;
    else
      return p[E / 2].y;
  }
  template <int E>
  __device__ __forceinline__ float value() const {
    return (E % 2 == 0) ? p[E / 2].x : p[E / 2].y;
  }
};
template <>
struct PipeSlotT<true, true> {
  float2 p[NPAIR], c[NPAIR];
  template <int E>
  __device__ __forceinline__ float value() const {
    return (E % 2 == 0) ? p[E / 2].x + c[E / 2].x : p[E / 2].y + c[E / 2].y;
  }
};
typedef PipeSlotT<PAIRS, PAIRS && COMP> PipeSlot;

// Value of output e of a slot (the compensated sum where there is one).
template <int E, class SL>
__device__ __forceinline__ T slot_value(SL& s) {
  if constexpr (PAIRS)
    return s.template value<E>();
  else
    return s.template at<E>();
}

template <int GX, int GY, int DZ, class SL>
__device__ __forceinline__ void apply_slot(SL& acc, const T v) {
  static_for<0, (DIM == 3) ? CY : 1>([&](auto ey) {
    static_for<0, CX>([&](auto ex) {
      constexpr int rx = GX - decltype(ex)::value;
      constexpr int ry = (DIM == 3) ? GY - decltype(ey)::value : DZ;
      constexpr int rz = (DIM == 3) ? DZ : 0;
      constexpr int e = decltype(ex)::value + decltype(ey)::value * CX;
      T& a = acc.template at<e>();
      if constexpr (contributes(rx, ry, rz)) {
        if constexpr (is_first(rx, ry, rz)) {
          a = v;
        } else if constexpr (COEFF == 0) {
          a = a + v;
        } else if constexpr (is_second(rx, ry, rz)) {
          a = fmat(a, tcs_mask[first_mask_index()], v * tcs_mask[mask_index(rx, ry, rz)]);
        } else {
          a = fmat(v, tcs_mask[mask_index(rx, ry, rz)], a);
        }
      }
    });
  });
}

// One term (rx, ry, rz) applied to a pair of outputs with the packed instructions; the same
// first-term / second-term rules as apply_slot, lane by lane.
template <int RX, int RY, int RZ>
__device__ __forceinline__ void apply_pair(float2& a, const float2 v) {
  if constexpr (is_first(RX, RY, RZ)) {
    a = v;
  } else if constexpr (COEFF == 0) {
    a = __fadd2_rn(a, v);
  } else {
    const float2 mm = mask_pair(mask_index(RX, RY, RZ));
    if constexpr (is_second(RX, RY, RZ)) {
      a = __ffma2_rn(a, mask_pair(first_mask_index()), __fmul2_rn(v, mm));
    } else {
      a = __ffma2_rn(v, mm, a);
    }
  }
}

// Compensated form: the terms of one footprint row of an output (2R+1 of them, rx ascending) are
// summed with plain packed FMAs into a row partial q (q = v*m, then q = fma(v, m, q); Jacobi: sums
// of the values); the row partial is then added to the running sum p with Knuth's two-sum and its
// rounding error collected in c.  Error: |value - exact| <= u|exact| + gamma_{2R+1} sum|terms|
// + O(u^2) (u = 2^-24), against gamma_S sum|terms| for the plain FP32 sweep.
template <int RX, int RY, int RZ>
__device__ __forceinline__ void row_term_pair(float2& q, const float2 v) {
  if constexpr (RX == -R) {
    if constexpr (COEFF == 0) {
      q = v;
    } else {
      q = __fmul2_rn(v, mask_pair(mask_index(RX, RY, RZ)));
    }
  } else if constexpr (COEFF == 0) {
    q = __fadd2_rn(q, v);
  } else {
    q = __ffma2_rn(v, mask_pair(mask_index(RX, RY, RZ)), q);
  }
}

// Knuth's two-sum of (p, q), lane by lane: p <- fl(p + q), c += the exact rounding error.  The
// differences are fma(x, -1, y) = fl(y - x), one rounding each, as the scalar subtractions.
template <bool FIRST_ROW>
__device__ __forceinline__ void two_sum_pair(float2& p, float2& c, const float2 q) {
  if constexpr (FIRST_ROW) {
    p = q;
    c = make_float2(0.f, 0.f);
  } else {
    const float2 m1 = make_float2(-1.f, -1.f);
    const float2 t = __fadd2_rn(p, q);
    const float2 z = __ffma2_rn(p, m1, t);       // t - p
    const float2 tz = __ffma2_rn(z, m1, t);      // t - z
    const float2 e1 = __ffma2_rn(tz, m1, p);     // p - (t - z)
    const float2 e2 = __ffma2_rn(z, m1, q);      // q - z
    c = __fadd2_rn(c, __fadd2_rn(e1, e2));
    p = t;
  }
}

// Load the row segment gx in [GX0, GX0 + N) of in-plane row GY into registers.  The loader says
// which columns start a pair it can fetch with one 16-byte (8-byte for float) access
// (`pair_aligned(gx)`, a compile-time property of the column parity) and provides `one<gx, gy>()`
// and `two<gx, gy>(a, b)`.
template <int GY, int GX0, int N, class LD>
__device__ __forceinline__ void load_row(const LD& ld, T (&v)[N]) {
  static_for<0, N>([&](auto ii) {
    constexpr int i = decltype(ii)::value;
    constexpr int gx = GX0 + i;
    constexpr bool starts_pair = LD::pair_aligned(gx) && (i + 1 < N);
    constexpr bool second_of_pair = (i > 0) && LD::pair_aligned(gx - 1);
    if constexpr (starts_pair) {
      ld.template two<gx, GY>(v[i], v[i + 1]);
    } else if constexpr (!second_of_pair) {
      v[i] = ld.template one<gx, GY>();
    }
  });
}

// Middle rows of a Star stencil by warp shuffles (pipelined sweep instances built with TCS_SHFL,
// blocks whose x extent is a multiple of 32, so a warp is 32 consecutive thread tiles of one row):
// every lane loads only its own CX values from shared memory; the R-wide halos on either side are
// the own values of the neighbouring lanes, passed with __shfl_up/down_sync, and only the lanes at
// the warp's edges, whose neighbours are outside the warp, read them from shared memory.  Same
// values as load_row<GY, -R, 2R + CX>, less shared-memory traffic.
#ifndef TCS_SHFL
#define TCS_SHFL 0
#endif
template <int GY, class LD>
__device__ __forceinline__ void load_row_shfl(const LD& ld, T (&v)[2 * R + CX]) {
#if TCS_SHFL
  T own[CX];
  load_row<GY, 0, CX>(ld, own);
  static_for<0, CX>([&](auto ex) { v[R + decltype(ex)::value] = own[decltype(ex)::value]; });
  const int lane = (int)(threadIdx.x & 31u);
  constexpr int J = (R + CX - 1) / CX;  // neighbour lanes per side that hold halo values
  static_for<1, J + 1>([&](auto jj) {
    constexpr int j = decltype(jj)::value;
    T l[CX], r[CX];
    static_for<0, CX>([&](auto ex) {
      l[decltype(ex)::value] = __shfl_up_sync(0xffffffffu, own[decltype(ex)::value], j);
      r[decltype(ex)::value] = __shfl_down_sync(0xffffffffu, own[decltype(ex)::value], j);
    });
    static_for<0, CX>([&](auto ex) {
      constexpr int gl = -j * CX + decltype(ex)::value;  // column of l[ex] relative to the thread
      constexpr int gr = j * CX + decltype(ex)::value;   // column of r[ex]
      if constexpr (gl >= -R) {
        if (lane < j) l[decltype(ex)::value] = ld.template one<gl, GY>();
        v[gl + R] = l[decltype(ex)::value];
      }
      if constexpr (gr < CX + R) {
        if (lane >= 32 - j) r[decltype(ex)::value] = ld.template one<gr, GY>();
        v[gr + R] = r[decltype(ex)::value];
      }
    });
  });
#else
  load_row<GY, -R, 2 * R + CX>(ld, v);
#endif
}

// In-plane cross of a Star stencil in Row order into the slot of the outputs centred on this
// plane (DZ = 0): the column segments above (3D), the middle rows -- contiguous segments that
// also hold the thread's own centre points, returned in cv -- and the column segments below.
template <class LD, class SL>
__device__ __forceinline__ void pipe_cross(const LD& ld, SL& s0, T (&cv)[NEP]) {
  constexpr int NY = (DIM == 3) ? CY : 1;
  if constexpr (DIM == 3) {
    static_for<0, R>([&](auto i) {  // gy in [-R, 0): the thread's columns
      constexpr int gy = decltype(i)::value - R;
      T seg[CX];
      load_row<gy, 0, CX>(ld, seg);
      static_for<0, CX>([&](auto gx) { apply_slot<decltype(gx)::value, gy, 0>(s0, seg[decltype(gx)::value]); });
    });
  }
  static_for<0, NY>([&](auto gyc) {  // middle rows: gx in [-R, R + CX)
    constexpr int gy = decltype(gyc)::value;
    T row[2 * R + CX];
    load_row_shfl<gy>(ld, row);
    static_for<0, CX>([&](auto ex) { cv[decltype(ex)::value + gy * CX] = row[R + decltype(ex)::value]; });
    static_for<0, 2 * R + CX>([&](auto ix) {
      apply_slot<decltype(ix)::value - R, gy, 0>(s0, row[decltype(ix)::value]);
    });
  });
  if constexpr (DIM == 3) {
    static_for<0, R>([&](auto i) {  // gy in [CY, CY + R)
      constexpr int gy = CY + decltype(i)::value;
      T seg[CX];
      load_row<gy, 0, CX>(ld, seg);
      static_for<0, CX>([&](auto gx) { apply_slot<decltype(gx)::value, gy, 0>(s0, seg[decltype(gx)::value]); });
    });
  }
}

// The march-axis arm term of each of the thread's outputs: own value v[e] of the plane at offset
// DZ (!= 0) from the output's centre plane.
template <int DZ, class SL>
__device__ __forceinline__ void apply_own(SL& s, const T (&v)[NEP]) {
  static_for<0, (DIM == 3) ? CY : 1>([&](auto ey) {
    static_for<0, CX>([&](auto ex) {
      apply_slot<decltype(ex)::value, decltype(ey)::value, DZ>(s, v[decltype(ex)::value + decltype(ey)::value * CX]);
    });
  });
}

// Ring form of the Star pipeline (3D, Row order; the kernel's TCS_TMEM variant).  Instead of
// 2R+1 output planes in registers, a thread keeps two rings of R entries elsewhere (tensor memory
// in the kernel): the own centre values of the last R input planes, and the accumulators of the
// last R outputs whose in-plane cross is done.  For input plane c, `ring_step`
//   * starts the output centred on c: its R lower arm terms from the own values of planes
//     c-R .. c-1 (ring), then the cross of plane c -- the reference's per-output order;
//   * finishes the output centred on c-R (accumulators from the ring): its R upper arm terms
//     from planes c-R+1 .. c-1 (ring) and c (the centre values just read);
//   * stores the new accumulators and plane c's own values into the ring entries just read.
// RING provides load_first(slot&, v) (the accumulators of the output centred on c-R and the own
// values of plane c-R), load_two<i>(a, b) (own values of planes c-R+i and c-R+i+1; b only when
// i+1 < R) and store(slot, v); its entries are addressed relative to plane c.  Entries come in
// pairs so that the kernel waits for tensor memory once per two entries.
template <class LD, class RING>
__device__ __forceinline__ void ring_step(const LD& ld, RING& ring, PipeSlot& done) {
  PipeSlot cur;
  {
    T v[NEP];
    ring.load_first(done, v);
    apply_own<-R>(cur, v);
  }
  static_for<0, R / 2>([&](auto pp) {
    constexpr int i = 1 + 2 * decltype(pp)::value;  // entries i and i+1 (i+1 < R unless R is even)
    T a[NEP], b[NEP];
    ring.template load_two<i>(a, b);
    apply_own<i - R>(cur, a);
    apply_own<i>(done, a);
    if constexpr (i + 1 < R) {
      apply_own<i + 1 - R>(cur, b);
      apply_own<i + 1>(done, b);
    }
  });
  T cv[NEP];
  pipe_cross(ld, cur, cv);
  apply_own<R>(done, cv);
  ring.store(cur, cv);
}

// Apply input plane (offset DZ relative to pending outputs) held in shared memory to the 2R+1
// pipeline slots.  `ld` reads the plane at in-plane offsets from the thread origin (see load_row);
// `slot(ic<k>)` returns the accumulators of the output at march-axis offset k - R.
template <class LD, class SLOTS>
__device__ __forceinline__ void pipe_plane(const LD& ld, SLOTS&& slot) {
  if constexpr (SHAPE == 0 && PAIRS && COMP) {
    // Box, packed FP32, compensated: per input row and slot, the row partial of each output pair
    // (rx ascending), then one two-sum into the slot's running sum.
    constexpr int NY = (DIM == 3) ? 2 * R + CY : 1;
    constexpr int OY = (DIM == 3) ? R : 0;
    static_for<0, NY>([&](auto iy) {
      constexpr int gy = decltype(iy)::value - OY;
      T row[2 * R + CX];
      load_row<gy, -R, 2 * R + CX>(ld, row);
      static_for<0, 2 * R + 1>([&](auto k) {
        constexpr int dz = decltype(k)::value - R;
        auto& s = slot(k);
        static_for<0, (DIM == 3) ? CY : 1>([&](auto ey) {
          constexpr int ry = (DIM == 3) ? gy - decltype(ey)::value : dz;
          constexpr int rz = (DIM == 3) ? dz : 0;
          if constexpr (contributes(0, ry, rz)) {
            static_for<0, CX / 2>([&](auto pp) {
              constexpr int e = decltype(ey)::value * (CX / 2) + decltype(pp)::value;
              float2 q;
              static_for<0, 2 * R + 1>([&](auto rxi) {
                constexpr int rx = decltype(rxi)::value - R;
                constexpr int j = 2 * decltype(pp)::value + rx + R;
                row_term_pair<rx, ry, rz>(q, make_float2(row[j], row[j + 1]));
              });
              // the first row of an output starts its sum (ry = rz = -R)
              two_sum_pair<(ry == -R && (DIM == 2 || rz == -R))>(s.p[e], s.c[e], q);
            });
          }
        });
      });
    });
  } else if constexpr (SHAPE == 0 && PAIRS) {
    // Box, packed FP32: per input row, every term rx feeds every slot and every output pair.  For a
    // fixed output the terms still arrive row by row and, within a row, rx ascending.
    constexpr int NY = (DIM == 3) ? 2 * R + CY : 1;
    constexpr int OY = (DIM == 3) ? R : 0;
    static_for<0, NY>([&](auto iy) {
      constexpr int gy = decltype(iy)::value - OY;
      T row[2 * R + CX];
      load_row<gy, -R, 2 * R + CX>(ld, row);
      static_for<0, 2 * R + 1>([&](auto rxi) {
        constexpr int rx = decltype(rxi)::value - R;
        static_for<0, 2 * R + 1>([&](auto k) {
          constexpr int dz = decltype(k)::value - R;
          auto& s = slot(k);
          static_for<0, (DIM == 3) ? CY : 1>([&](auto ey) {
            constexpr int ry = (DIM == 3) ? gy - decltype(ey)::value : dz;
            constexpr int rz = (DIM == 3) ? dz : 0;
            if constexpr (contributes(rx, ry, rz)) {
              static_for<0, CX / 2>([&](auto pp) {
                constexpr int j = 2 * decltype(pp)::value + rx + R;  // row index of lane 0's value
                constexpr int e = decltype(ey)::value * (CX / 2) + decltype(pp)::value;
                apply_pair<rx, ry, rz>(s.p[e], make_float2(row[j], row[j + 1]));
              });
            }
          });
        });
      });
    });
  } else if constexpr (SHAPE == 0) {
    // Box: every in-plane footprint point feeds every slot, in the slice traversal order.
    constexpr int NY = (DIM == 3) ? 2 * R + CY : 1;
    constexpr int OY = (DIM == 3) ? R : 0;
    if constexpr (ORIENT == 1 && DIM == 3) {
      static_for<0, 2 * R + CX>([&](auto ix) {
        static_for<0, NY>([&](auto iy) {
          constexpr int gx = decltype(ix)::value - R, gy = decltype(iy)::value - OY;
          const T v = ld.template one<gx, gy>();
          static_for<0, 2 * R + 1>([&](auto k) { apply_slot<gx, gy, decltype(k)::value - R>(slot(k), v); });
        });
      });
    } else {
      static_for<0, NY>([&](auto iy) {
        constexpr int gy = decltype(iy)::value - OY;
        T row[2 * R + CX];
        load_row<gy, -R, 2 * R + CX>(ld, row);
        static_for<0, 2 * R + CX>([&](auto ix) {
          constexpr int gx = decltype(ix)::value - R;
          static_for<0, 2 * R + 1>([&](auto k) {
            apply_slot<gx, gy, decltype(k)::value - R>(slot(k), row[decltype(ix)::value]);
          });
        });
      });
    }
  } else {
    // Star: the thread's own centre points feed the slots DZ != 0; the in-plane cross feeds DZ = 0.
    constexpr int NY = (DIM == 3) ? CY : 1;
    auto& s0 = slot(ic<R>{});
    T cv[NEP];
    if constexpr (ORIENT == 0 || DIM == 2) {
      pipe_cross(ld, s0, cv);
    } else {
      // 3D Column order: columns of the cross, point by point.
      static_for<0, NY>([&](auto ey) {
        static_for<0, CX>([&](auto ex) {
          cv[decltype(ex)::value + decltype(ey)::value * CX] = ld.template one<decltype(ex)::value, decltype(ey)::value>();
        });
      });
      auto ldc = [&](auto gxc, auto gyc) -> T {
        constexpr int gx = decltype(gxc)::value, gy = decltype(gyc)::value;
        if constexpr (gx >= 0 && gx < CX && gy >= 0 && gy < NY)
          return cv[gx + gy * CX];
        else
          return ld.template one<gx, gy>();
      };
      static_for<0, R>([&](auto i) {
        static_for<0, CY>([&](auto gy) {
          constexpr int gx = decltype(i)::value - R, y = decltype(gy)::value;
          apply_slot<gx, y, 0>(s0, ldc(ic<gx>{}, ic<y>{}));
        });
      });
      static_for<0, CX>([&](auto gx) {
        static_for<0, 2 * R + CY>([&](auto i) {
          constexpr int x = decltype(gx)::value, gy = decltype(i)::value - R;
          apply_slot<x, gy, 0>(s0, ldc(ic<x>{}, ic<gy>{}));
        });
      });
      static_for<0, R>([&](auto i) {
        static_for<0, CY>([&](auto gy) {
          constexpr int gx = CX + decltype(i)::value, y = decltype(gy)::value;
          apply_slot<gx, y, 0>(s0, ldc(ic<gx>{}, ic<y>{}));
        });
      });
    }
    // centre points -> slots DZ != 0 (one term each)
    static_for<0, 2 * R + 1>([&](auto k) {
      constexpr int dz = decltype(k)::value - R;
      if constexpr (dz != 0) {
        static_for<0, NY>([&](auto ey) {
          static_for<0, CX>([&](auto ex) {
            apply_slot<decltype(ex)::value, decltype(ey)::value, dz>(
                slot(k), cv[decltype(ex)::value + decltype(ey)::value * CX]);
          });
        });
      }
    });
  }
}
}  // namespace tcs
