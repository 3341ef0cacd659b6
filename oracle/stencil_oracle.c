/* stencil_oracle.c — CPU restatement of the reference's stencil sweep.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker of the engine: only the test
 * suite, the smoke check and the CPU-baseline leg of bench.py load it.  The engine never
 * calls it, and nothing here is a fallback for the GPU path.
 *
 * It restates, independently of the engine's CUDA templates, what one kernel generated by the
 * reference computes (MKKnorr/ThreadCoarsenedStencilGenerator):
 *   - thread tiles of cx*cy[*cz] outputs, origin and guard:  cuda/generate2DStencil_cuda.py:78-104,
 *     cuda/generate3DStencil_cuda.py:81-114
 *   - footprint traversal order (Row / Column, Box / Star): cuda/generate2DStencil_cuda.py:244-297,
 *     cuda/generate3DStencil_cuda.py:265-360
 *   - per-point additions and first-term initialisation:   cuda/generate2DStencil_cuda.py:146-198,
 *     cuda/generate3DStencil_cuda.py:171-218
 *   - mask layout (calcMaskAddress):                        cuda/generate2DStencil_cuda.py:120-144,
 *     cuda/generate3DStencil_cuda.py:132-169
 *   - write-back, Jacobi factor c = fl(1/S):                cuda/generate2DStencil_cuda.py:206-211,300-315
 *   - init pattern:                                         cuda/generate2DStencil_cuda.py:321-350,
 *     cuda/generate3DStencil_cuda.py:386-430
 *   - geometry (truncation, Read/Write padding):            cuda/benchmark.cpp:142-179,
 *     cuda/benchmark.h:100-123
 * Arithmetic: the generated kernels are compiled by nvcc with its default -fmad=true, which fuses
 * each `result += register*d_mask[k]` into one fma.  The second term of an output is special:
 * there `result` still holds the bare product v0*m0, the statement is an add of two products,
 * and the compiler fuses the left one, giving fma(v0, m0, fl(v1*m1)); every later term is
 * fma(vk, mk, result).  This file is compiled with -ffp-contract=off and spells exactly those
 * fma()/fmaf() calls, so its FP64 output is bit-identical to the reference kernel's
 * (oracle_set_second_term_mode(0) selects the other fusion, for diagnosis only).
 *
 * The OpenMP loop (oracle_cpu_sweep_*) is the timed CPU baseline: the same per-output term order,
 * x innermost, rows in parallel.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct oracle_spec {
  int dimension;     /* 2 | 3 */
  int neighbourhood; /* 0 Box | 1 Star */
  int orientation;   /* 0 Row | 1 Column */
  int coefficients;  /* 0 Jacobi | 1 Variable */
  int range;
  int cx, cy, cz;
  int alignment;     /* 0 None | 1 Read | 2 Write */
  int cl_size;
} oracle_spec;

typedef struct oracle_geometry {
  unsigned grid[3], elements[3], threads[3];
  unsigned left_offset, right_offset;
  unsigned long long n_points;
} oracle_geometry;

static int iabs_(int v) { return v < 0 ? -v : v; }

/* How the second term of a Variable output is fused (see oracle_set_second_term_mode). */
static int oracle_second_term_mode = 1;

/* 0: acc = fma(v1, m1, fl(v0*m0));  1: acc = fma(v0, m0, fl(v1*m1)). */
void oracle_set_second_term_mode(int mode) { oracle_second_term_mode = mode; }

int oracle_stencil_size(const oracle_spec* s) {
  const int w = 2 * s->range + 1;
  if (s->neighbourhood == 0) return s->dimension == 2 ? w * w : w * w * w;
  return 2 * s->dimension * s->range + 1;
}

unsigned oracle_left_offset(const oracle_spec* s) {
  if (s->alignment != 2) return 0;
  return (s->range % s->cl_size != 0) ? (unsigned)(s->cl_size - s->range % s->cl_size) : 0u;
}

/* cuda/benchmark.cpp:262-303 with cuda/benchmark.h:100-123 */
int oracle_geometry_of(const oracle_spec* s, unsigned nx, unsigned ny, unsigned nz,
                       oracle_geometry* g) {
  const unsigned R = (unsigned)s->range;
  unsigned n[3] = {nx, ny, s->dimension == 3 ? nz : 1u};
  unsigned c[3] = {(unsigned)s->cx, (unsigned)s->cy, s->dimension == 3 ? (unsigned)s->cz : 1u};
  unsigned long long xmem;
  int i;
  memset(g, 0, sizeof(*g));
  for (i = 0; i < s->dimension; ++i) {
    if (n[i] < 2 * R) return 1;
    g->grid[i] = n[i] - (n[i] - 2 * R) % c[i];
    g->elements[i] = g->grid[i] - 2 * R;
    g->threads[i] = g->elements[i] / c[i];
  }
  if (s->dimension == 2) {
    g->grid[2] = 1;
    g->elements[2] = 1;
    g->threads[2] = 1;
  }
  xmem = g->grid[0];
  if (s->alignment == 2) { /* alignXwidthWrite */
    g->left_offset = oracle_left_offset(s);
    xmem += g->left_offset;
    g->right_offset = (xmem % s->cl_size) ? (unsigned)(s->cl_size - xmem % s->cl_size) : 0u;
    xmem += g->right_offset;
  } else if (s->alignment == 1) { /* alignXwidthRead */
    g->right_offset = (xmem % s->cl_size) ? (unsigned)(s->cl_size - xmem % s->cl_size) : 0u;
    xmem += g->right_offset;
  }
  g->grid[0] = (unsigned)xmem;
  g->n_points = (unsigned long long)g->grid[0] * g->grid[1] * g->grid[2];
  return 0;
}

/* calcMaskAddress */
static int mask_address(const oracle_spec* s, int rx, int ry, int rz) {
  const int R = s->range;
  if (s->neighbourhood == 0) {
    const int w = 2 * R + 1;
    if (s->dimension == 2) return (rx + R) + (ry + R) * w;
    return (rx + R) + (ry + R) * w + (rz + R) * w * w;
  }
  if (s->dimension == 2) {
    if (rx == 0 && ry < 0) return ry + R;
    if (ry == 0) return R + (rx + R);
    return (ry + R) + 2 * R;
  }
  if (rz < 0) return rz + R;
  if (rz == 0 && rx == 0 && ry < 0) return (ry + R) + R;
  if (rz == 0 && ry == 0) return (rx + R) + 2 * R;
  if (rz == 0 && rx == 0 && ry > 0) return (ry + R) + 3 * R;
  return (rz + R) + 4 * R;
}

/* Would printAdditions emit a term for element (ex,ey,ez) from grid point (gx,gy,gz)?
 * Returns 0 (no), 1 (initialise), 2 (add). */
static int term_kind(const oracle_spec* s, int gx, int gy, int gz, int ex, int ey, int ez) {
  const int R = s->range;
  if (s->neighbourhood == 0) {
    int in = iabs_(gx - ex) <= R && iabs_(gy - ey) <= R;
    if (s->dimension == 3) in = in && iabs_(gz - ez) <= R;
    if (!in) return 0;
    if (ex - R == gx && ey - R == gy && (s->dimension == 2 || ez - R == gz)) return 1;
    return 2;
  }
  if (s->dimension == 2) {
    if (!((iabs_(gx - ex) <= R && ey == gy) || (iabs_(gy - ey) <= R && ex == gx))) return 0;
    if (s->orientation == 1) return (gy == ey && ex - R == gx) ? 1 : 2;
    return (gx == ex && ey - R == gy) ? 1 : 2;
  }
  if (!((iabs_(gx - ex) <= R && ey == gy && ez == gz) || (iabs_(gy - ey) <= R && ex == gx && ez == gz) ||
        (iabs_(gz - ez) <= R && ex == gx && ey == gy)))
    return 0;
  return (ex == gx && ey == gy && ez - R == gz) ? 1 : 2;
}

/* The generator's traversal of one thread tile: the sequence of grid points (gx,gy,gz) relative
 * to the thread origin, in emission order.  Returns the count; pts holds 3 ints per point. */
static int traversal(const oracle_spec* s, int* pts) {
  const int R = s->range, cx = s->cx, cy = s->cy, cz = s->dimension == 3 ? s->cz : 1;
  int n = 0, x, y, z;
#define EMIT(a, b, c) \
  do {                \
    pts[3 * n] = (a); \
    pts[3 * n + 1] = (b); \
    pts[3 * n + 2] = (c); \
    ++n;              \
  } while (0)
  if (s->dimension == 2) {
    if (s->neighbourhood == 0) {
      if (s->orientation == 1) {
        for (x = -R; x < R + cx; ++x)
          for (y = -R; y < R + cy; ++y) EMIT(x, y, 0);
      } else {
        for (y = -R; y < R + cy; ++y)
          for (x = -R; x < R + cx; ++x) EMIT(x, y, 0);
      }
    } else if (s->orientation == 1) {
      for (x = -R; x < 0; ++x)
        for (y = 0; y < cy; ++y) EMIT(x, y, 0);
      for (x = 0; x < cx; ++x)
        for (y = -R; y < R + cy; ++y) EMIT(x, y, 0);
      for (x = cx; x < R + cx; ++x)
        for (y = 0; y < cy; ++y) EMIT(x, y, 0);
    } else {
      for (y = -R; y < 0; ++y)
        for (x = 0; x < cx; ++x) EMIT(x, y, 0);
      for (y = 0; y < cy; ++y)
        for (x = -R; x < R + cx; ++x) EMIT(x, y, 0);
      for (y = cy; y < R + cy; ++y)
        for (x = 0; x < cx; ++x) EMIT(x, y, 0);
    }
    return n;
  }
  if (s->neighbourhood == 0) {
    for (z = -R; z < R + cz; ++z) {
      if (s->orientation == 1) {
        for (x = -R; x < R + cx; ++x)
          for (y = -R; y < R + cy; ++y) EMIT(x, y, z);
      } else {
        for (y = -R; y < R + cy; ++y)
          for (x = -R; x < R + cx; ++x) EMIT(x, y, z);
      }
    }
    return n;
  }
  for (z = -R; z < 0; ++z) {
    if (s->orientation == 1) {
      for (x = 0; x < cx; ++x)
        for (y = 0; y < cy; ++y) EMIT(x, y, z);
    } else {
      for (y = 0; y < cy; ++y)
        for (x = 0; x < cx; ++x) EMIT(x, y, z);
    }
  }
  for (z = 0; z < cz; ++z) {
    if (s->orientation == 1) {
      for (x = -R; x < 0; ++x)
        for (y = 0; y < cy; ++y) EMIT(x, y, z);
      for (x = 0; x < cx; ++x)
        for (y = -R; y < R + cy; ++y) EMIT(x, y, z);
      for (x = cx; x < R + cx; ++x)
        for (y = 0; y < cy; ++y) EMIT(x, y, z);
    } else {
      for (y = -R; y < 0; ++y)
        for (x = 0; x < cx; ++x) EMIT(x, y, z);
      for (y = 0; y < cy; ++y)
        for (x = -R; x < R + cx; ++x) EMIT(x, y, z);
      for (y = cy; y < R + cy; ++y)
        for (x = 0; x < cx; ++x) EMIT(x, y, z);
    }
  }
  for (z = cz; z < R + cz; ++z) {
    if (s->orientation == 1) {
      for (x = 0; x < cx; ++x)
        for (y = 0; y < cy; ++y) EMIT(x, y, z);
    } else {
      for (y = 0; y < cy; ++y)
        for (x = 0; x < cx; ++x) EMIT(x, y, z);
    }
  }
#undef EMIT
  return n;
}

static int traversal_capacity(const oracle_spec* s) {
  const int R = s->range, cz = s->dimension == 3 ? s->cz : 1;
  return (2 * R + s->cx) * (2 * R + s->cy) * (s->dimension == 3 ? (2 * R + cz) : 1);
}

/* One reference sweep, thread tile by thread tile, exactly as the generated kernel evaluates
 * it.  Arrays are [z][y][x] with row pitch g->grid[0]; only interior points are written. */
#define DEFINE_TILE_SWEEP(NAME, T, FMA)                                                           \
  int NAME(const oracle_spec* s, const unsigned grid[3], unsigned right_offset, const T* in,      \
           T* out, const T* mask) {                                                               \
    const int R = s->range, cx = s->cx, cy = s->cy, cz = s->dimension == 3 ? s->cz : 1;           \
    const int S = oracle_stencil_size(s);                                                         \
    const unsigned long long xdim = grid[0], ydim = grid[1];                                      \
    const unsigned long long zdim = s->dimension == 3 ? grid[2] : 1;                              \
    const unsigned lo = oracle_left_offset(s);                                                    \
    const unsigned long long ro = s->alignment == 0 ? 0 : right_offset;                           \
    const unsigned long long xlim = xdim - R - ro, ylim = ydim - R;                               \
    const unsigned long long zlim = s->dimension == 3 ? zdim - R : 1;                             \
    const unsigned long long plane = xdim * ydim;                                                 \
    const T c = (T)1 / (T)S;                                                                      \
    const int ne = cx * cy * cz;                                                                  \
    int* pts = (int*)malloc(sizeof(int) * 3 * traversal_capacity(s));                             \
    T* acc = (T*)malloc(sizeof(T) * ne);                                                          \
    T* v0 = (T*)malloc(sizeof(T) * ne);                                                           \
    T* m0 = (T*)malloc(sizeof(T) * ne);                                                           \
    int* cnt = (int*)malloc(sizeof(int) * ne);                                                    \
    const int np = traversal(s, pts);                                                             \
    unsigned long long x, y, z;                                                                   \
    for (z = (s->dimension == 3 ? (unsigned long long)R : 0);                                     \
         s->dimension == 3 ? (z + cz - 1 < zlim) : (z < 1); z += cz)                              \
      for (y = R; y + cy - 1 < ylim; y += cy)                                                     \
        for (x = (unsigned long long)R + lo; x + cx - 1 < xlim; x += cx) {                        \
          int p, ex, ey, ez;                                                                      \
          for (p = 0; p < ne; ++p) cnt[p] = 0;                                                    \
          for (p = 0; p < np; ++p) {                                                              \
            const int gx = pts[3 * p], gy = pts[3 * p + 1], gz = pts[3 * p + 2];                  \
            const T v = in[(long long)(x + gx) + (long long)(y + gy) * (long long)xdim +           \
                           (long long)(z + gz) * (long long)plane];                               \
            for (ez = 0; ez < cz; ++ez)                                                           \
              for (ey = 0; ey < cy; ++ey)                                                         \
                for (ex = 0; ex < cx; ++ex) {                                                     \
                  const int k = term_kind(s, gx, gy, gz, ex, ey, ez);                             \
                  const int e = ex + ey * cx + ez * cx * cy;                                      \
                  if (k == 0) continue;                                                           \
                  if (s->coefficients == 0) {                                                     \
                    acc[e] = (k == 1) ? v : acc[e] + v;                                           \
                  } else {                                                                        \
                    const T m = mask[mask_address(s, gx - ex, gy - ey, gz - ez)];                 \
                    if (k == 1) {                                                                 \
                      acc[e] = v * m;                                                             \
                      v0[e] = v;                                                                  \
                      m0[e] = m;                                                                  \
                    } else if (cnt[e] == 1 && oracle_second_term_mode == 1) {                     \
                      acc[e] = FMA(v0[e], m0[e], v * m);                                          \
                    } else {                                                                      \
                      acc[e] = FMA(v, m, acc[e]);                                                 \
                    }                                                                             \
                    cnt[e] += 1;                                                                  \
                  }                                                                               \
                }                                                                                 \
          }                                                                                       \
          for (ez = 0; ez < cz; ++ez)                                                             \
            for (ey = 0; ey < cy; ++ey)                                                           \
              for (ex = 0; ex < cx; ++ex) {                                                       \
                const int e = ex + ey * cx + ez * cx * cy;                                        \
                out[(x + ex) + (y + ey) * xdim + (z + ez) * plane] =                              \
                    (s->coefficients == 0) ? acc[e] * c : acc[e];                                 \
              }                                                                                   \
        }                                                                                         \
    free(pts);                                                                                    \
    free(acc);                                                                                    \
    free(v0);                                                                                     \
    free(m0);                                                                                     \
    free(cnt);                                                                                    \
    return 0;                                                                                     \
  }

DEFINE_TILE_SWEEP(oracle_sweep_f64, double, fma)
DEFINE_TILE_SWEEP(oracle_sweep_f32, float, fmaf)

/* Per-output term order: the traversal of a 1x1[x1] tile (it is independent of the coarsening
 * factors).  Fills offsets (3 ints per term) and mask indices; returns the term count. */
int oracle_term_order(const oracle_spec* s, int* offsets, int* mask_idx) {
  oracle_spec one = *s;
  int n, p;
  one.cx = one.cy = one.cz = 1;
  n = traversal(&one, offsets);
  for (p = 0; p < n; ++p)
    mask_idx[p] = mask_address(&one, offsets[3 * p], offsets[3 * p + 1], offsets[3 * p + 2]);
  return n;
}

/* OpenMP CPU sweep (the timed CPU baseline): for every interior row, terms in the per-output
 * order with x innermost.  Bit-identical to the tile sweep.  nthreads <= 0: all available. */
#define DEFINE_CPU_SWEEP(NAME, T, FMA)                                                            \
  int NAME(const oracle_spec* s, const unsigned grid[3], unsigned right_offset, const T* in,      \
           T* out, const T* mask, int nthreads) {                                                 \
    const int R = s->range;                                                                       \
    const int S = oracle_stencil_size(s);                                                         \
    const long long xdim = grid[0], ydim = grid[1];                                               \
    const long long zdim = s->dimension == 3 ? grid[2] : 1;                                       \
    const long long lo = oracle_left_offset(s);                                                   \
    const long long ro = s->alignment == 0 ? 0 : right_offset;                                    \
    const long long x0 = R + lo, x1 = xdim - R - ro;                                              \
    const long long z0 = s->dimension == 3 ? R : 0, z1 = s->dimension == 3 ? zdim - R : 1;       \
    const long long nxr = x1 - x0, nrows = (ydim - 2 * R) * (z1 - z0);                            \
    const long long plane = xdim * ydim;                                                          \
    const T c = (T)1 / (T)S;                                                                      \
    int* off = (int*)malloc(sizeof(int) * 3 * S);                                                 \
    int* mi = (int*)malloc(sizeof(int) * S);                                                      \
    long long* delta = (long long*)malloc(sizeof(long long) * S);                                 \
    T* mk = (T*)malloc(sizeof(T) * S);                                                            \
    long long row;                                                                                \
    int k;                                                                                        \
    oracle_term_order(s, off, mi);                                                                \
    for (k = 0; k < S; ++k) {                                                                     \
      delta[k] = off[3 * k] + off[3 * k + 1] * xdim + off[3 * k + 2] * plane;                     \
      mk[k] = s->coefficients == 1 ? mask[mi[k]] : (T)0;                                          \
    }                                                                                             \
    if (nthreads <= 0) nthreads = omp_get_max_threads();                                          \
    if (nxr > 0) {                                                                                \
      _Pragma("omp parallel num_threads(nthreads)") {                                             \
        T* acc = (T*)malloc(sizeof(T) * (size_t)nxr);                                             \
        _Pragma("omp for schedule(static)") for (row = 0; row < nrows; ++row) {                   \
          const long long y = R + row % (ydim - 2 * R);                                           \
          const long long z = z0 + row / (ydim - 2 * R);                                          \
          const long long base = x0 + y * xdim + z * plane;                                       \
          const T* src = in + base;                                                               \
          long long i;                                                                            \
          int kk;                                                                                 \
          if (s->coefficients == 0) {                                                             \
            for (i = 0; i < nxr; ++i) acc[i] = src[i + delta[0]];                                 \
            for (kk = 1; kk < S; ++kk) {                                                          \
              const T* q = src + delta[kk];                                                       \
              for (i = 0; i < nxr; ++i) acc[i] = acc[i] + q[i];                                   \
            }                                                                                     \
            for (i = 0; i < nxr; ++i) out[base + i] = acc[i] * c;                                 \
          } else {                                                                                \
            if (oracle_second_term_mode == 1) {                                                   \
              const T* q0 = src + delta[0];                                                       \
              const T* q1 = src + delta[1];                                                       \
              for (i = 0; i < nxr; ++i) acc[i] = FMA(q0[i], mk[0], q1[i] * mk[1]);                \
            } else {                                                                              \
              for (i = 0; i < nxr; ++i) acc[i] = FMA(src[i + delta[1]], mk[1], src[i + delta[0]] * mk[0]); \
            }                                                                                     \
            for (kk = 2; kk < S; ++kk) {                                                          \
              const T* q = src + delta[kk];                                                       \
              const T m = mk[kk];                                                                 \
              for (i = 0; i < nxr; ++i) acc[i] = FMA(q[i], m, acc[i]);                            \
            }                                                                                     \
            for (i = 0; i < nxr; ++i) out[base + i] = acc[i];                                     \
          }                                                                                       \
        }                                                                                         \
        free(acc);                                                                                \
      }                                                                                           \
    }                                                                                             \
    free(off);                                                                                    \
    free(mi);                                                                                     \
    free(delta);                                                                                  \
    free(mk);                                                                                     \
    return 0;                                                                                     \
  }

DEFINE_CPU_SWEEP(oracle_cpu_sweep_f64, double, fma)
DEFINE_CPU_SWEEP(oracle_cpu_sweep_f32, float, fmaf)

/* The reference's init kernel over the whole buffer (cuda/generate2DStencil_cuda.py:321-350,
 * cuda/generate3DStencil_cuda.py:386-430).  Cells the reference never writes keep their value. */
int oracle_init_f64(const oracle_spec* s, const unsigned grid[3], unsigned right_offset,
                    double* a) {
  const unsigned long long xdim = grid[0], ydim = grid[1];
  const unsigned long long zdim = s->dimension == 3 ? grid[2] : 1;
  const unsigned long long lo = oracle_left_offset(s);
  const unsigned long long xend = s->alignment == 0 ? xdim : xdim - right_offset;
  const unsigned long long R = (unsigned long long)s->range;
  unsigned long long x, y, z;
  for (z = 0; z < zdim; ++z)
    for (y = 0; y < ydim; ++y)
      for (x = lo; x < xend; ++x) {
        const unsigned long long idx = x + y * xdim + z * xdim * ydim;
        const int border = (x - lo < R) || (y < R) || (s->dimension == 3 && z < R);
        if (s->dimension == 2)
          a[idx] = border ? 1.0 : 0.0;
        else
          a[idx] = border ? ((idx % 2 == 0) ? 0.75 : 0.25) : 0.0;
      }
  return 0;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
