// Host build of the pipelined sweep's per-thread arithmetic (test harness).
//
// Drives tcs::pipe_plane (threadcoarsenedstencilgenerator_b200/csrc/tcs_tile.cuh) exactly as the
// tcs_pipe kernel does: every thread tile streams the input planes ms-R .. me+R-1 of its column,
// keeps 2R+1 output planes in flight in the slots (t - k) mod (2R+1), and stores output pi - 2R
// after input plane pi.  Pieces start at arbitrary planes (`piece` splits the march axis) to
// exercise the pipeline restart.  Built with -ffp-contract=off like tile_host.cpp.
#include <cmath>
#include <cstring>

#include "host_cuda_shim.h"
#include "tcs_tile.cuh"

// Run-time element access of a slot (the kernel indexes with compile-time constants).
template <int E = 0>
static T slot_value_rt(tcs::PipeSlot& s, int e) {
  if constexpr (E + 1 < tcs::NEP) {
    if (e != E) return slot_value_rt<E + 1>(s, e);
  }
  return tcs::slot_value<E>(s);
}

// Plane reader with the kernel's interface (pairs are just two scalar loads here).
struct HostPlane {
  const T* b;
  long long pitch;
  static constexpr bool pair_aligned(int gx) { return ((gx % 2) + 2) % 2 == 0; }
  template <int GX, int GY>
  T one() const {
    return b[GX + GY * pitch];
  }
  template <int GX, int GY>
  void two(T& a, T& c) const {
    a = b[GX + GY * pitch];
    c = b[GX + 1 + GY * pitch];
  }
};

extern "C" int pipe_sweep(const unsigned grid[3], unsigned left_offset, unsigned right_offset,
                          int aligned, const T* in, T* out, const double* mask, unsigned piece,
                          unsigned unroll) {
  using namespace tcs;
  constexpr int NP2 = 2 * R + 1;
  if (COEFF == 1)
    for (int k = 0; k < S; ++k) tcs_mask[k] = (T)mask[k];
  if (COEFF == 1 && tcs::PAIRS)
    for (int k = 0; k < S; ++k) tcs_mask_pairs[k] = make_float2((float)mask[k], (float)mask[k]);
  const long long xdim = grid[0], ydim = grid[1], zdim = DIM == 3 ? grid[2] : 1;
  const long long plane = DIM == 3 ? xdim * ydim : xdim;  // stride of the march axis
  const long long x_lim = xdim - R - (aligned ? right_offset : 0);
  const long long y_lim = ydim - R, z_lim = DIM == 3 ? zdim - R : 1;
  const long long m_lim = DIM == 3 ? z_lim : y_lim;       // march-axis interior bound
  const long long y_step = DIM == 3 ? CY : 1;
  const long long y_end = DIM == 3 ? y_lim : R + 1;
  for (long long y = R; DIM == 3 ? (y + CY - 1 < y_end) : (y < y_end); y += y_step)
    for (long long x = R + left_offset; x + CX - 1 < x_lim; x += CX)
      for (long long ms = R; ms < m_lim; ms += piece) {
        const long long me = (ms + piece < m_lim) ? ms + piece : m_lim;
        const long long np = me - ms + 2 * R;
        PipeSlot acc[NP2];
        // super-steps of `unroll` planes; slots re-aligned after each, as in tcs_pipe
        for (long long pi = 0; pi < np; ++pi) {
          const long long p = ms - R + pi;
          const T* base = in + x + (DIM == 3 ? y * xdim : 0) + p * plane;
          const HostPlane ld{base, xdim};
          const int t = (int)(pi % unroll);
          auto slot = [&](auto kk) -> PipeSlot& {
            constexpr int k = decltype(kk)::value;
            return acc[((t - k) % NP2 + NP2) % NP2];
          };
          pipe_plane(ld, slot);
          const long long op = pi - 2 * R;
          if (op >= 0 && op < me - ms) {
            PipeSlot& done = acc[((t - 2 * R) % NP2 + NP2) % NP2];
            constexpr T c = T(1) / T(S);
            T* o = out + x + (DIM == 3 ? y * xdim : 0) + (ms + op) * plane;
            for (int ey = 0; ey < (DIM == 3 ? CY : 1); ++ey)
              for (int ex = 0; ex < CX; ++ex) {
                const int e = ex + ey * CX;
                const T v = slot_value_rt(done, e);
                o[ex + ey * xdim] = (COEFF == 0) ? v * c : v;
              }
          }
          if (t == (int)unroll - 1 && unroll % NP2 != 0) {
            PipeSlot tmp[NP2];
            std::memcpy(tmp, acc, sizeof(acc));
            for (int m = 0; m < NP2; ++m) acc[m] = tmp[(m + unroll) % NP2];
          }
        }
      }
  return 0;
}

// The ring form (tcs::ring_step, the kernel's TCS_TMEM variant) of 3D Star stencils in Row
// order: per input plane c of a piece, the output centred on c - R is completed from the rings and
// stored; the rings are plain arrays here (tensor memory in the kernel), entry (plane mod R).
#if TCS_DIM == 3 && TCS_SHAPE == 1 && TCS_ORIENT == 0
struct HostRing {
  T (*raw)[tcs::NEP];
  tcs::PipeSlot* acc;
  long long c;  // current input plane (piece-relative)
  int entry(long long p) const { return (int)(((p % tcs::R) + tcs::R) % tcs::R); }
  void load_first(tcs::PipeSlot& s, T (&v)[tcs::NEP]) const {
    s = acc[entry(c - tcs::R)];
    std::memcpy(v, raw[entry(c - tcs::R)], sizeof(v));
  }
  template <int I>
  void load_two(T (&a)[tcs::NEP], T (&b)[tcs::NEP]) const {
    std::memcpy(a, raw[entry(c - tcs::R + I)], sizeof(a));
    if (I + 1 < tcs::R) std::memcpy(b, raw[entry(c - tcs::R + I + 1)], sizeof(b));
  }
  void store(const tcs::PipeSlot& s, const T (&v)[tcs::NEP]) {
    acc[entry(c)] = s;
    std::memcpy(raw[entry(c)], v, sizeof(v));
  }
};

extern "C" int pipe_sweep_ring(const unsigned grid[3], unsigned left_offset, unsigned right_offset,
                               int aligned, const T* in, T* out, const double* mask, unsigned piece) {
  using namespace tcs;
  if (COEFF == 1)
    for (int k = 0; k < S; ++k) tcs_mask[k] = (T)mask[k];
  const long long xdim = grid[0], ydim = grid[1], zdim = grid[2];
  const long long plane = xdim * ydim;
  const long long x_lim = xdim - R - (aligned ? right_offset : 0);
  const long long y_lim = ydim - R, z_lim = zdim - R;
  // stale ring contents from the previous piece (or column) must not matter: start from garbage
  T raw[R][NEP];
  PipeSlot acc[R];
  for (int i = 0; i < R; ++i)
    for (int e = 0; e < NEP; ++e) raw[i][e] = (T)NAN;
  std::memset(static_cast<void*>(acc), 0xff, sizeof(acc));
  for (long long y = R; y + CY - 1 < y_lim; y += CY)
    for (long long x = R + left_offset; x + CX - 1 < x_lim; x += CX)
      for (long long ms = R; ms < z_lim; ms += piece) {
        const long long me = (ms + piece < z_lim) ? ms + piece : z_lim;
        const long long np = me - ms + 2 * R;
        for (long long pi = 0; pi < np; ++pi) {
          const long long p = ms - R + pi;
          const HostPlane ld{in + x + y * xdim + p * plane, xdim};
          HostRing ring{raw, acc, pi};
          PipeSlot done;
          ring_step(ld, ring, done);
          const long long op = pi - 2 * R;
          if (op >= 0 && op < me - ms) {
            constexpr T c = T(1) / T(S);
            T* o = out + x + y * xdim + (ms + op) * plane;
            for (int ey = 0; ey < CY; ++ey)
              for (int ex = 0; ex < CX; ++ex) {
                const T v = slot_value_rt(done, ex + ey * CX);
                o[ex + ey * xdim] = (COEFF == 0) ? v * c : v;
              }
          }
        }
      }
  return 0;
}
#else
extern "C" int pipe_sweep_ring(const unsigned*, unsigned, unsigned, int, const T*, T*, const double*, unsigned) {
  return -1;
}
#endif
