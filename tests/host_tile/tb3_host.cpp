// Host build of the two-sweep kernel's control flow (test harness for tcs_tb3, 3D and 2D).
//
// Runs tcs_tb3's per-piece logic for every CTA tile and piece, one thread tile after another:
// stage 1 applies each input plane to pipeline 1 with tcs::pipe_plane (reading the input with zero
// fill outside the grid, as the TMA ring does), writes the completed plane of S(in) into the plane
// buffer -- points outside the interior take the input's value -- and, once every thread of the
// tile has written, stage 2 applies the buffer plane to pipeline 2 and stores the inner thread
// tiles' completed outputs.  Same tile geometry (extended tile, output tile, thread tiles of
// TCS_CX x TCS_CY dividing R in 3D), same plane offsets and slot rotation as the kernel.  In 2D the
// march axis is y: a "plane" is one row, the extended tile a strip of bx * CX columns, the plane
// buffer one row with an R-wide margin.
#include <cstring>
#include <vector>

#include "host_cuda_shim.h"
#include "tcs_tile.cuh"

namespace {
using namespace tcs;

struct GlobalPlane {  // input plane at a thread origin; zero outside the grid
  const T* in;
  long long xdim, ydim, zdim, x, y, z;
  static constexpr bool pair_aligned(int) { return false; }
  template <int GX, int GY>
  T one() const {
    const long long xx = x + GX, yy = y + GY;
    if constexpr (DIM == 2) {  // z is the row
      if (xx < 0 || z < 0 || xx >= xdim || z >= ydim) return T(0);
      return in[xx + z * xdim];
    }
    if (xx < 0 || yy < 0 || z < 0 || xx >= xdim || yy >= ydim || z >= zdim) return T(0);
    return in[xx + yy * xdim + z * xdim * ydim];
  }
  template <int GX, int GY>
  void two(T& a, T& b) const {
    a = one<GX, GY>();
    b = one<GX + 1, GY>();
  }
};

struct BufPlane {
  const T* p;
  long long pitch;
  static constexpr bool pair_aligned(int) { return false; }
  template <int GX, int GY>
  T one() const {
    return p[GY * pitch + GX];
  }
  template <int GX, int GY>
  void two(T& a, T& b) const {
    a = p[GY * pitch + GX];
    b = p[GY * pitch + GX + 1];
  }
};
}  // namespace

// One pass (two sweeps) of in into out; bx, by: threads of the kernel's block; piece: output
// planes per piece (pieces restart both pipelines).
extern "C" int tb3_pass(const unsigned grid[3], unsigned left_offset, unsigned right_offset, int aligned,
                        const T* in, T* out, const double* mask, unsigned bx, unsigned by, unsigned piece,
                        unsigned unroll) {
  constexpr int NP2 = 2 * R + 1;
  if (COEFF == 1)
    for (int k = 0; k < S; ++k) tcs_mask[k] = (T)mask[k];
  if (COEFF == 1 && tcs::PAIRS)
    for (int k = 0; k < S; ++k) tcs_mask_pairs[k] = make_float2((float)mask[k], (float)mask[k]);
  constexpr bool D3 = DIM == 3;
  const long long xdim = grid[0], ydim = grid[1], zdim = D3 ? grid[2] : 1;
  const long long plane = D3 ? xdim * ydim : xdim;  // stride of the march axis
  const long long x0 = R + left_offset;
  const long long x_lim = xdim - R - (aligned ? right_offset : 0), y_lim = ydim - R, z_lim = zdim - R;
  const long long m_lim = D3 ? z_lim : y_lim, m_dim = D3 ? zdim : ydim;  // march axis
  if (!D3) by = 1;
  const int EX = (int)bx * CX, EY = D3 ? (int)by * CY : 1, OX = EX - 2 * R, OY = D3 ? EY - 2 * R : 1;
  const int BW = EX + 2 * R, BH = D3 ? EY + 2 * R : 1;
  if (OX <= 0 || OY <= 0 || (D3 && (R % CX || R % CY)) || (!D3 && CY != 1)) return 1;
  const long long ntx = (x_lim - x0 + OX - 1) / OX, nty = D3 ? (y_lim - R + OY - 1) / OY : 1;
  const int nthr = (int)(bx * by);
  std::vector<T> buf(2 * (size_t)BW * BH, T(0));
  std::vector<PipeSlot> acc1((size_t)nthr * NP2), acc2((size_t)nthr * NP2);
  constexpr T c = T(1) / T(S);
  for (long long tile = 0; tile < ntx * nty; ++tile)
    for (long long zs = 0; zs < m_lim - R; zs += piece) {
      const long long ze = (zs + piece < m_lim - R) ? zs + piece : m_lim - R;
      const long long ms = R + zs, nout = ze - zs, np = nout + 4 * R, m_first = ms - 2 * R;
      const long long X0 = x0 - R + (tile % ntx) * OX, Y0 = (tile / ntx) * OY;
      for (long long pi = 0; pi < np; ++pi) {
        const int t = (int)(pi % unroll);
        const long long m = m_first + pi, q = m - R;
        T* bq = buf.data() + (pi & 1) * (size_t)BW * BH;
        for (int th = 0; th < nthr; ++th) {  // stage 1
          const int ex0 = (th % (int)bx) * CX, ey0 = (th / (int)bx) * CY;
          PipeSlot* a1 = &acc1[(size_t)th * NP2];
          const GlobalPlane ld{in, xdim, ydim, zdim, X0 + ex0, Y0 + ey0, m};
          auto slot1 = [&](auto kk) -> PipeSlot& {
            constexpr int k = decltype(kk)::value;
            return a1[((t - k) % NP2 + NP2) % NP2];
          };
          pipe_plane(ld, slot1);
          PipeSlot& d1 = a1[((t - 2 * R) % NP2 + NP2) % NP2];
          static_for<0, CY>([&](auto ey) {
            static_for<0, CX>([&](auto ex) {
              constexpr int e = decltype(ex)::value + decltype(ey)::value * CX;
              const long long gx = X0 + ex0 + decltype(ex)::value, gy = Y0 + ey0 + decltype(ey)::value;
              const bool interior =
                  gx >= x0 && gx < x_lim && (!D3 || (gy >= R && gy < y_lim)) && q >= R && q < m_lim;
              T v = (COEFF == 0) ? slot_value<e>(d1) * c : slot_value<e>(d1);
              if (!interior) {
                const bool ing = gx >= 0 && gx < xdim && (!D3 || (gy >= 0 && gy < ydim)) && q >= 0 && q < m_dim;
                v = ing ? in[gx + (D3 ? gy * xdim : 0) + q * plane] : T(0);
              }
              bq[(D3 ? (R + ey0 + decltype(ey)::value) * BW : 0) + R + ex0 + decltype(ex)::value] = v;
            });
          });
        }
        for (int th = 0; th < nthr; ++th) {  // stage 2
          const int ex0 = (th % (int)bx) * CX, ey0 = (th / (int)bx) * CY;
          PipeSlot* a2 = &acc2[(size_t)th * NP2];
          const bool inner = ex0 + CX > R && ex0 < EX - R && (!D3 || (ey0 >= R && ey0 < EY - R));
          // edge thread tiles read the buffer's margin (never written); their outputs are discarded
          const BufPlane ldb{bq + (D3 ? (R + ey0) * BW : 0) + R + ex0, BW};
          auto slot2 = [&](auto kk) -> PipeSlot& {
            constexpr int k = decltype(kk)::value;
            return a2[((t - k) % NP2 + NP2) % NP2];
          };
          pipe_plane(ldb, slot2);
          const long long op = pi - 4 * R;
          if (inner && op >= 0 && op < nout) {
            PipeSlot& d2 = a2[((t - 2 * R) % NP2 + NP2) % NP2];
            static_for<0, CY>([&](auto ey) {
              static_for<0, CX>([&](auto ex) {
                constexpr int e = decltype(ex)::value + decltype(ey)::value * CX;
                const long long ox = X0 + ex0 + decltype(ex)::value, oy = Y0 + ey0 + decltype(ey)::value;
                const int exx = ex0 + decltype(ex)::value;  // 2D thread tiles may straddle the edge
                if (ox < x_lim && (!D3 || oy < y_lim) && exx >= R && exx < EX - R)
                  out[ox + (D3 ? oy * xdim : 0) + (ms + op) * plane] =
                      (COEFF == 0) ? slot_value<e>(d2) * c : slot_value<e>(d2);
              });
            });
          }
        }
        if (t == (int)unroll - 1 && unroll % NP2 != 0) {  // slot re-alignment at a chunk's end
          for (int th = 0; th < nthr; ++th)
            for (auto* a : {&acc1[(size_t)th * NP2], &acc2[(size_t)th * NP2]}) {
              PipeSlot tmp[NP2];
              std::memcpy(tmp, a, sizeof(tmp));
              for (int k = 0; k < NP2; ++k) a[k] = tmp[(k + unroll) % NP2];
            }
        }
      }
    }
  return 0;
}
