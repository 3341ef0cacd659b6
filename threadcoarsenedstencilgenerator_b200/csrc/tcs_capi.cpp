// Host half of the B200 stencil engine: the C ABI declared in include/tcs.h.
//
// One `tcs_stencil` handle = one stencil parameter set.  tcs_create instantiates the kernel
// templates of tcs_kernels.cuh for that set with NVRTC (sm_100a cubin, cached on disk keyed by
// a hash of source + options) and loads the module with the CUDA driver API, reached through
// cudaGetDriverEntryPoint so that the library itself links only the static CUDA runtime and
// NVRTC and loads on machines without a GPU driver (host-only entry points work there).
//
// Reference behaviour mirrored here (file:line in the reference project):
//   parameter checks          cuda/benchmark.cpp:430-491, cuda/generate2DStencil_cuda.py:49-60
//   stencilSize / flops       cuda/benchmark.cpp:62-81
//   geometry                  cuda/benchmark.cpp:142-179, cuda/benchmark.h:100-123
//   copyMask                  cuda/generateLaunchUpdateGrid.py:77-82
//   maxPotentialBlockSize     cuda/generateLaunchUpdateGrid.py:84-89
//   benchmarkUpdateGrid       cuda/generateLaunchUpdateGrid.py:103-147
//   launchInit                cuda/generateLaunchUpdateGrid.py:150-158

#include "tcs.h"

#include <cuda.h>
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <chrono>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "tcs_field.h"
#include "tcs_kernels_src.inc"  // tcs_kernels_src[], tcs_tile_src[]: the device headers

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

// ---- driver API through the runtime's entry-point query --------------------------------------
struct Driver {
  decltype(&cuModuleLoadData) ModuleLoadData = nullptr;
  decltype(&cuModuleUnload) ModuleUnload = nullptr;
  decltype(&cuModuleGetFunction) ModuleGetFunction = nullptr;
  decltype(&cuModuleGetGlobal) ModuleGetGlobal = nullptr;
  decltype(&cuFuncSetAttribute) FuncSetAttribute = nullptr;
  decltype(&cuFuncGetAttribute) FuncGetAttribute = nullptr;
  decltype(&cuLaunchKernel) LaunchKernel = nullptr;
  decltype(&cuTensorMapEncodeTiled) TensorMapEncodeTiled = nullptr;
  decltype(&cuOccupancyMaxActiveBlocksPerMultiprocessor) OccMaxActive = nullptr;
  decltype(&cuOccupancyMaxPotentialBlockSize) OccMaxPotential = nullptr;
  decltype(&cuGetErrorString) GetErrorString = nullptr;
  decltype(&cuCtxGetCurrent) CtxGetCurrent = nullptr;
  decltype(&cuCtxGetId) CtxGetId = nullptr;
  bool ok = false;
  std::string why;
};

Driver g_drv;
std::once_flag g_drv_once;

template <class F>
bool entry(const char* name, F& fn, std::string& why) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  cudaError_t e = cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q);
  if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || p == nullptr) {
    why = std::string("driver entry point unavailable: ") + name;
    return false;
  }
  fn = reinterpret_cast<F>(p);
  return true;
}

void load_driver() {
  Driver d;
  bool ok = entry("cuModuleLoadData", d.ModuleLoadData, d.why) &&
            entry("cuModuleUnload", d.ModuleUnload, d.why) &&
            entry("cuModuleGetFunction", d.ModuleGetFunction, d.why) &&
            entry("cuModuleGetGlobal", d.ModuleGetGlobal, d.why) &&
            entry("cuFuncSetAttribute", d.FuncSetAttribute, d.why) &&
            entry("cuFuncGetAttribute", d.FuncGetAttribute, d.why) &&
            entry("cuLaunchKernel", d.LaunchKernel, d.why) &&
            entry("cuTensorMapEncodeTiled", d.TensorMapEncodeTiled, d.why) &&
            entry("cuOccupancyMaxActiveBlocksPerMultiprocessor", d.OccMaxActive, d.why) &&
            entry("cuOccupancyMaxPotentialBlockSize", d.OccMaxPotential, d.why) &&
            entry("cuGetErrorString", d.GetErrorString, d.why) &&
            entry("cuCtxGetCurrent", d.CtxGetCurrent, d.why) && entry("cuCtxGetId", d.CtxGetId, d.why);
  d.ok = ok;
  g_drv = d;
}

std::string cu_msg(CUresult r) {
  const char* s = nullptr;
  if (g_drv.GetErrorString) g_drv.GetErrorString(r, &s);
  return s ? std::string(s) : ("CUresult " + std::to_string((int)r));
}

#define TCS_CU(call)                                                                    \
  do {                                                                                  \
    CUresult r_ = (call);                                                               \
    if (r_ != CUDA_SUCCESS) return fail(TCS_ERR_CUDA, std::string(#call ": ") + cu_msg(r_)); \
  } while (0)

#define TCS_RT(call)                                                                       \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return fail(TCS_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_));         \
  } while (0)

// Make sure a device exists, the primary context is current and the driver table is loaded.
int ensure_cuda() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(TCS_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
  }
  TCS_RT(cudaFree(nullptr));
  std::call_once(g_drv_once, load_driver);
  if (!g_drv.ok) return fail(TCS_ERR_CUDA, g_drv.why);
  return TCS_OK;
}

// ---- parameter logic -------------------------------------------------------------------------
int validate(const tcs_spec* s) {
  if (!s) return fail(TCS_ERR_INVALID_VALUE, "spec is NULL");
  if (s->dimension != 2 && s->dimension != 3)
    return fail(TCS_ERR_INVALID_VALUE, "Unknown dimension: either 2D or 3D");
  if (s->neighbourhood != TCS_BOX && s->neighbourhood != TCS_STAR)
    return fail(TCS_ERR_INVALID_VALUE, "Unknown stencil-neighbourhood: either 'Box' or 'Star'");
  if (s->orientation != TCS_ROW && s->orientation != TCS_COLUMN)
    return fail(TCS_ERR_INVALID_VALUE, "Unknown orientation: either 'Row' or 'Column'");
  if (s->coefficients != TCS_JACOBI && s->coefficients != TCS_VARIABLE)
    return fail(TCS_ERR_INVALID_VALUE, "Unknown coefficients: either 'Jacobi' or 'Variable'");
  if (s->range < 1) return fail(TCS_ERR_INVALID_VALUE, "Stencil range must be greater than zero");
  if (s->cx < 1 || s->cy < 1 || (s->dimension == 3 && s->cz < 1))
    return fail(TCS_ERR_INVALID_VALUE, "Coarsening factors have to be greater than zero");
  if (s->alignment != TCS_ALIGN_NONE && s->alignment != TCS_ALIGN_READ &&
      s->alignment != TCS_ALIGN_WRITE)
    return fail(TCS_ERR_INVALID_VALUE, "Unknown alignment: either 'None', 'Write' or 'Read'");
  if (s->alignment != TCS_ALIGN_NONE && s->cl_size <= 0)
    return fail(TCS_ERR_INVALID_VALUE, "size of alignment has to be > 0 when alignment is given");
  if (s->precision != TCS_F64 && s->precision != TCS_F32 && s->precision != TCS_F32C)
    return fail(TCS_ERR_INVALID_VALUE, "Unknown precision");
  // Practical limits of one instantiation (the reference has none but its unrolled code
  // stops compiling long before these).
  if (s->range > 16) return fail(TCS_ERR_INVALID_VALUE, "range > 16 is not supported");
  const int cz = s->dimension == 3 ? s->cz : 1;
  if (s->cx > 16 || s->cy > 16 || cz > 16 || s->cx * s->cy * cz > 512)
    return fail(TCS_ERR_INVALID_VALUE, "coarsening tile too large (per axis <= 16, product <= 512)");
  return TCS_OK;
}

unsigned stencil_size_of(const tcs_spec& s) {
  const unsigned w = 2u * s.range + 1u;
  if (s.neighbourhood == TCS_BOX) return s.dimension == 2 ? w * w : w * w * w;
  return 2u * s.dimension * s.range + 1u;
}

unsigned left_offset_of(const tcs_spec& s) {
  if (s.alignment != TCS_ALIGN_WRITE) return 0;
  const unsigned cl = (unsigned)s.cl_size, r = (unsigned)s.range;
  return (r % cl != 0) ? cl - r % cl : 0;
}

const char* coeff_str(int c) { return c == TCS_JACOBI ? "Jacobi" : "Variable"; }
const char* shape_str(int s) { return s == TCS_BOX ? "Box" : "Star"; }
const char* align_str(int a) {
  return a == TCS_ALIGN_NONE ? "None" : (a == TCS_ALIGN_READ ? "Read" : "Write");
}

// ---- NVRTC instantiation with an on-disk cubin cache -----------------------------------------
uint64_t fnv1a(const std::string& s, uint64_t h = 1469598103934665603ull) {
  for (unsigned char c : s) {
    h ^= c;
    h *= 1099511628211ull;
  }
  return h;
}

std::string library_dir() {
  Dl_info info;
  if (dladdr(reinterpret_cast<void*>(&tcs_abi_version), &info) && info.dli_fname) {
    std::string p(info.dli_fname);
    const size_t k = p.find_last_of('/');
    if (k != std::string::npos) return p.substr(0, k);
  }
  return ".";
}

std::string cache_dir() {
  const char* env = std::getenv("TCS_KCACHE");
  std::string d = (env && *env) ? std::string(env) : library_dir() + "/_kcache";
  mkdir(d.c_str(), 0775);
  return d;
}

// Compile-time launch shape of a pipelined-sweep module: tcs_pipe (one grid), or tcs_pipe_batch
// (a table of grids) when `batch` is set.
struct PipeKey {
  unsigned bx, by, ch, lshift;
  unsigned batch = 0;
  unsigned epi = 0;  // epilogue mode (tcs_kernels.cuh, TCS_EPI): 0 plain, 1 FP64 defect, 2 FP32 accumulate
  unsigned tb3 = 0;  // tcs_tb3 (two sweeps per pass) with thread tiles tb3 x tb3 (2D: tb3 x 1); 0: tcs_pipe
  unsigned shfl = 0;  // Star middle rows through warp shuffles (TCS_SHFL)
  unsigned tmem = 0;  // ring form in tensor memory (TCS_TMEM)
  bool operator==(const PipeKey& o) const {
    return bx == o.bx && by == o.by && ch == o.ch && lshift == o.lshift && batch == o.batch && epi == o.epi &&
           tb3 == o.tb3 && shfl == o.shfl && tmem == o.tmem;
  }
};

// The ring form (TCS_TMEM, tcs_kernels.cuh): 3D Star stencils in Row order, FP64 or FP32, plain
// epilogue, ring entries of 4, 8, 16 or 32 columns, blocks of whole warps.  Its tensor-memory columns per CTA (the
// allocation, a power of two) or 0 when the form does not apply.
unsigned tmem_cols(const tcs_spec& s, unsigned bx, unsigned by) {
  if (s.dimension != 3 || s.neighbourhood != TCS_STAR || s.orientation != TCS_ROW || s.precision == TCS_F32C)
    return 0;
  if ((bx * by) % 32u != 0) return 0;  // tensor-memory loads and stores are whole-warp instructions
  const unsigned w = (unsigned)(s.cx * s.cy) * (s.precision == TCS_F64 ? 2u : 1u);
  if (w != 4 && w != 8 && w != 16 && w != 32) return 0;
  const unsigned groups = (bx * by + 127u) / 128u;
  const unsigned need = groups * 2u * (unsigned)s.range * w;
  unsigned n = 32;
  while (n < need) n *= 2;
  return n <= 512 ? n : 0;
}

std::string instance_macros(const tcs_spec& s, const PipeKey* pk) {
  std::ostringstream m;
  if (pk)
    m << "#define TCS_PIPE 1\n#define TCS_BX " << pk->bx << "\n#define TCS_BY " << pk->by
      << "\n#define TCS_CH " << pk->ch << "\n#define TCS_LSHIFT " << pk->lshift << "\n";
  if (pk && pk->batch) m << "#define TCS_BATCH 1\n";
  if (pk && pk->epi) m << "#define TCS_EPI " << pk->epi << "\n";
  if (pk && pk->tb3) m << "#define TCS_TB3 1\n";
  if (pk && pk->shfl) m << "#define TCS_SHFL 1\n";
  if (pk && pk->tmem) m << "#define TCS_TMEM 1\n";
  // TCS_PIPE_CYCLE=0 in the environment builds the pipelined kernels with a one-chunk loop body
  // (register slots rotated at the back-edge) instead of one whole slot cycle per iteration
  if (pk) {
    const char* cyc = std::getenv("TCS_PIPE_CYCLE");
    if (cyc && std::string(cyc) == "0") m << "#define TCS_CYCLE 0\n";
    // TCS_PIPE_STREAM_STORES=1: output pairs with streaming (evict-first) stores
    const char* sts = std::getenv("TCS_PIPE_STREAM_STORES");
    if (sts && std::string(sts) == "1") m << "#define TCS_STCS 1\n";
  }
  // the two-sweep kernel has thread tiles of its own (tb3 x tb3 x 1); the term order of every
  // output does not depend on them
  const int cx = (pk && pk->tb3) ? (int)pk->tb3 : s.cx;
  const int cy = (pk && pk->tb3) ? (s.dimension == 3 ? (int)pk->tb3 : 1) : s.cy;
  const int cz = (pk && pk->tb3) ? 1 : (s.dimension == 3 ? s.cz : 1);
  m << "#define TCS_T " << (s.precision == TCS_F64 ? "double" : "float") << "\n"
    << "#define TCS_COMP " << (s.precision == TCS_F32C ? 1 : 0) << "\n"
    << "#define TCS_DIM " << s.dimension << "\n"
    << "#define TCS_SHAPE " << s.neighbourhood << "\n"
    << "#define TCS_ORIENT " << s.orientation << "\n"
    << "#define TCS_COEFF " << s.coefficients << "\n"
    << "#define TCS_R " << s.range << "\n"
    << "#define TCS_CX " << cx << "\n"
    << "#define TCS_CY " << cy << "\n"
    << "#define TCS_CZ " << cz << "\n";
  return m.str();
}

std::atomic<unsigned long long> g_tmp_counter{0};

// NVRTC programs are independent, so instantiations run concurrently (the build step compiles
// many in parallel); a finished cubin is published into the cache by an atomic rename.
int instantiate(const tcs_spec& s, const PipeKey* pk, std::vector<char>& cubin,
                std::string* path_out, const char* extra = nullptr) {
  const std::string src = instance_macros(s, pk) + (extra ? extra : "") + "#include \"tcs_kernels.cuh\"\n";
  const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "--fmad=false",
                        "--device-as-default-execution-space"};
  const int nopts = sizeof(opts) / sizeof(opts[0]);
  int major = 0, minor = 0;
  nvrtcVersion(&major, &minor);
  std::string keysrc = src + "\x01" + tcs_kernels_src + "\x01" + tcs_tile_src + "\x01" +
                       std::to_string(major) + "." + std::to_string(minor);
  for (int i = 0; i < nopts; ++i) keysrc += std::string("\x02") + opts[i];
  char key[32];
  std::snprintf(key, sizeof(key), "%016llx", (unsigned long long)fnv1a(keysrc));
  const std::string path = cache_dir() + "/tcs_" + key + ".cubin";
  if (path_out) *path_out = path;

  {
    std::ifstream f(path, std::ios::binary);
    if (f) {
      cubin.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
      if (!cubin.empty()) return TCS_OK;
    }
  }
  nvrtcProgram prog;
  const char* hdrs[] = {tcs_kernels_src, tcs_tile_src};
  const char* hdr_names[] = {"tcs_kernels.cuh", "tcs_tile.cuh"};
  nvrtcResult r = nvrtcCreateProgram(&prog, src.c_str(), "tcs_instance.cu", 2, hdrs, hdr_names);
  if (r != NVRTC_SUCCESS) return fail(TCS_ERR_COMPILE, nvrtcGetErrorString(r));
  r = nvrtcCompileProgram(prog, nopts, opts);
  if (r != NVRTC_SUCCESS) {
    size_t n = 0;
    nvrtcGetProgramLogSize(prog, &n);
    std::string log(n, '\0');
    nvrtcGetProgramLog(prog, &log[0]);
    nvrtcDestroyProgram(&prog);
    return fail(TCS_ERR_COMPILE, "NVRTC: " + log);
  }
  size_t n = 0;
  nvrtcGetCUBINSize(prog, &n);
  cubin.resize(n);
  nvrtcGetCUBIN(prog, cubin.data());
  nvrtcDestroyProgram(&prog);
  // atomic publish into the cache
  const std::string tmp = path + ".tmp." + std::to_string((long long)getpid()) + "." +
                          std::to_string(g_tmp_counter.fetch_add(1));
  {
    std::ofstream f(tmp, std::ios::binary);
    f.write(cubin.data(), (std::streamsize)cubin.size());
  }
  std::rename(tmp.c_str(), path.c_str());
  return TCS_OK;
}

// Host mirror of the device TcsGeo (same layout).
struct TcsGeo {
  unsigned long long xdim, ydim, zdim;
  unsigned x0, x_lim;
  unsigned y_lim, z_lim;
  unsigned seg;
  unsigned nslot;
  unsigned width;
  unsigned loader;
};
static_assert(sizeof(TcsGeo) == 56, "TcsGeo layout");

// Host mirror of the device TcsPipeGeo (same layout).
struct TcsPipeGeo {
  unsigned long long xdim, ydim, zdim;
  unsigned long long total, per_cta;
  unsigned x0, x_lim;
  unsigned y_lim, z_lim;
  unsigned ntx, m;
  unsigned nslot, loader;
};
static_assert(sizeof(TcsPipeGeo) == 72, "TcsPipeGeo layout");

// One loaded pipelined-sweep module (its own constant mask and status word).
struct PipeMod {
  PipeKey key;
  CUmodule mod = nullptr;
  CUfunction f = nullptr;
  CUdeviceptr mask_ptr = 0;
  size_t mask_bytes = 0;
  CUdeviceptr pairs_ptr = 0;  // tcs_mask_pairs (packed FP32 instances), 0 when absent
  size_t pairs_bytes = 0;
  CUdeviceptr status_ptr = 0;
  int smem_attr = 0;
};

struct MapEntry {
  const void* ptr;
  unsigned long long dims[3];
  unsigned box[3];
  CUtensorMap map;
};

}  // namespace

struct tcs_stencil {
  tcs_spec spec{};
  unsigned S = 0, flops = 0, left_off = 0;
  int device = 0;
  int num_sms = 0;
  int smem_optin = 0;
  CUmodule mod = nullptr;
  CUfunction f_direct = nullptr, f_march = nullptr, f_init = nullptr;
  CUdeviceptr mask_ptr = 0;
  size_t mask_bytes = 0;
  CUdeviceptr status_ptr = 0;
  int march_smem_attr = 0;
  int dropin_variant = TCS_VARIANT_AUTO;  // variant used by tcs_benchmark_update_grid
  unsigned dropin_segments = 0, dropin_depth = 0;
  std::vector<double> mask_host;          // last mask uploaded (copied into new pipe modules)
  std::vector<double> last_durations;     // per-launch durations [s] of the last benchmark loop
  double* scratch = nullptr;              // per-block partials of the field reductions
  size_t scratch_len = 0;                 // in doubles
  std::vector<PipeMod*> pipes;            // pipelined-sweep modules, one per launch shape
  void* tc_bops = nullptr;                // tensor-core Toeplitz operands (built from mask_host)
  CUmodule fringe_mod = nullptr;          // coarsening-1 instance for the ragged fringe of a grid
  CUfunction f_fringe = nullptr;
  CUdeviceptr fringe_mask = 0;
  CUmodule tb_mod = nullptr;              // 1 x 8 instance with tcs_tb2: two sweeps per pass (2D)
  CUfunction f_tb2 = nullptr;
  int tb2_smem_attr = 0;
  CUdeviceptr tb_mask = 0;
  bool tc_stale = true;                   // mask changed since tc_bops was built
  std::mutex mu;
  std::vector<MapEntry> maps;
};

namespace {

struct Resolved {
  int variant = 0;
  TcsGeo geo{};
  TcsPipeGeo pgeo{};
  PipeMod* pipe = nullptr;
  unsigned chunk = 0;
  unsigned grid[3] = {1, 1, 1};
  unsigned block[3] = {1, 1, 1};
  unsigned smem = 0;
  unsigned depth = 0;
  unsigned box[3] = {1, 1, 1};
  int occ = 0;
  bool no_tma = false;  // pipe: tile rows wider than one TMA box, streamed through cp.async
};

int elem_size(const tcs_spec& s) { return s.precision == TCS_F64 ? 8 : 4; }

// Interior geometry from the reference-style (gridSize, rightOffset) pair.
int make_geo(const tcs_stencil* h, const unsigned grid[3], unsigned right_offset, TcsGeo& g) {
  const tcs_spec& s = h->spec;
  const unsigned R = (unsigned)s.range;
  if (!grid) return fail(TCS_ERR_INVALID_VALUE, "grid is NULL");
  const unsigned ro = (s.alignment == TCS_ALIGN_NONE) ? 0u : right_offset;
  const unsigned long long xdim = grid[0], ydim = grid[1];
  const unsigned long long zdim = (s.dimension == 3) ? grid[2] : 1ull;
  if (xdim < 2ull * R + h->left_off + ro || ydim < 2ull * R || (s.dimension == 3 && zdim < 2ull * R))
    return fail(TCS_ERR_INVALID_VALUE, "grid smaller than twice the stencil range plus padding");
  if (xdim > 0xffffffffull || ydim > 0xffffffffull || zdim > 0xffffffffull)
    return fail(TCS_ERR_INVALID_VALUE, "grid extent exceeds 32 bits");
  g = TcsGeo{};
  g.xdim = xdim;
  g.ydim = ydim;
  g.zdim = zdim;
  g.x0 = R + h->left_off;
  g.x_lim = (unsigned)(xdim - R - ro);
  g.y_lim = (unsigned)(ydim - R);
  g.z_lim = (unsigned)(zdim - (s.dimension == 3 ? R : 0));
  return TCS_OK;
}

int check_block(const tcs_stencil* h, const unsigned b[3]) {
  if (b[0] < 1 || b[1] < 1 || b[2] < 1) return fail(TCS_ERR_INVALID_VALUE, "block dimension of 0");
  if (h->spec.dimension == 2 && b[2] != 1)
    return fail(TCS_ERR_INVALID_VALUE, "2D stencils take a block with z = 1");
  if (b[0] > 1024 || b[1] > 1024 || b[2] > 64 || (unsigned long long)b[0] * b[1] * b[2] > 1024)
    return fail(TCS_ERR_INVALID_VALUE, "block exceeds the device thread-block limits");
  return TCS_OK;
}

unsigned cdiv(unsigned long long a, unsigned long long b) { return (unsigned)((a + b - 1) / b); }

int resolve_direct(tcs_stencil* h, const TcsGeo& g, const tcs_launch* L, Resolved& out) {
  const tcs_spec& s = h->spec;
  const unsigned cz = s.dimension == 3 ? (unsigned)s.cz : 1u;
  int maxthr = 0;
  TCS_CU(g_drv.FuncGetAttribute(&maxthr, CU_FUNC_ATTRIBUTE_MAX_THREADS_PER_BLOCK, h->f_direct));
  const unsigned long long nthr = (unsigned long long)L->block[0] * L->block[1] * L->block[2];
  if (nthr > (unsigned long long)maxthr)
    return fail(TCS_ERR_UNSUPPORTED, "block has more threads than the direct kernel supports (" +
                                         std::to_string(maxthr) + ")");
  out.variant = TCS_VARIANT_DIRECT;
  out.geo = g;
  for (int i = 0; i < 3; ++i) out.block[i] = L->block[i];
  if (L->grid_blocks[0] && L->grid_blocks[1] && L->grid_blocks[2]) {
    for (int i = 0; i < 3; ++i) out.grid[i] = L->grid_blocks[i];
  } else {
    const unsigned long long ex = g.x_lim > g.x0 ? g.x_lim - g.x0 : 0;
    const unsigned long long ey = g.y_lim - s.range;
    const unsigned long long ez = s.dimension == 3 ? g.z_lim - s.range : 1;
    const unsigned long long tx = ex / s.cx, ty = ey / s.cy, tz = s.dimension == 3 ? ez / cz : 1;
    out.grid[0] = std::max(1u, cdiv(tx, L->block[0]));
    out.grid[1] = std::max(1u, cdiv(ty, L->block[1]));
    out.grid[2] = std::max(1u, cdiv(tz, L->block[2]));
  }
  if (out.grid[1] > 65535 || out.grid[2] > 65535)
    return fail(TCS_ERR_UNSUPPORTED, "direct launch grid exceeds 65535 blocks in y or z");
  int occ = 0;
  TCS_CU(g_drv.OccMaxActive(&occ, h->f_direct, (int)nthr, 0));
  out.occ = occ;
  out.smem = 0;
  return TCS_OK;
}

int resolve_march(tcs_stencil* h, const TcsGeo& g, const tcs_launch* L, Resolved& out) {
  const tcs_spec& s = h->spec;
  const unsigned R = (unsigned)s.range;
  const unsigned es = (unsigned)elem_size(s);
  const unsigned vec = 16u / es;
  const unsigned cz = s.dimension == 3 ? (unsigned)s.cz : 1u;
  // TMA needs a row pitch that is a multiple of 16 bytes; other pitches use the cp.async loader.
  const unsigned loader = ((g.xdim * es) % 16 == 0) ? 0u : 1u;
  const unsigned TX = L->block[0] * s.cx;
  unsigned STEP, rows;
  if (s.dimension == 2) {
    STEP = L->block[1] * s.cy;
    rows = 1;
  } else {
    STEP = L->block[2] * cz;
    rows = L->block[1] * s.cy + 2 * R;
  }
  // Row width W: the tile plus its halo plus the alignment shift of the TMA x coordinate, in
  // whole 16-byte granules, widened until a chunk (STEP planes of W x rows) is a multiple of
  // 128 bytes: every TMA destination (one chunk per ring slot) must be 128-byte aligned.
  unsigned W = ((TX + 2 * R + vec - 1 + vec - 1) / vec) * vec;
  while ((STEP * W * rows * es) % 128 != 0) W += vec;
  if (W > 256 || STEP > 256 || rows > 256)
    return fail(TCS_ERR_UNSUPPORTED, "tile exceeds the 256-element TMA box limit");
  const unsigned plane = W * rows;
  const unsigned chunk_bytes = STEP * plane * es;
  const unsigned K = 1 + (2 * R + STEP - 1) / STEP;
  unsigned depth = L->depth;
  if (depth == 0) depth = std::max(1u, std::min(4u, cdiv(16384, chunk_bytes)));
  unsigned smem = 0, nslot = 0;
  for (;;) {
    nslot = K + depth;
    // barriers, then 128 bytes of slack so the ring can start on a 128-byte boundary
    smem = ((nslot * 8 + 127) / 128) * 128 + 128 + nslot * chunk_bytes;
    if (smem <= (unsigned)h->smem_optin || depth == 1) break;
    --depth;
  }
  if (smem > (unsigned)h->smem_optin)
    return fail(TCS_ERR_UNSUPPORTED, "ring does not fit in shared memory (" +
                                         std::to_string(smem) + " bytes)");
  const int nthr = (int)(L->block[0] * L->block[1] * L->block[2]);
  int maxthr = 0;
  TCS_CU(g_drv.FuncGetAttribute(&maxthr, CU_FUNC_ATTRIBUTE_MAX_THREADS_PER_BLOCK, h->f_march));
  if (nthr > maxthr)
    return fail(TCS_ERR_UNSUPPORTED, "block has more threads than the march kernel supports (" +
                                         std::to_string(maxthr) + ")");
  {
    std::lock_guard<std::mutex> lock(h->mu);
    if ((int)smem > h->march_smem_attr) {
      TCS_CU(g_drv.FuncSetAttribute(h->f_march, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES,
                                    (int)smem));
      h->march_smem_attr = (int)smem;
    }
  }
  int occ = 0;
  TCS_CU(g_drv.OccMaxActive(&occ, h->f_march, nthr, smem));
  if (occ < 1) return fail(TCS_ERR_UNSUPPORTED, "march kernel cannot be resident at this shape");

  const unsigned long long ex = g.x_lim > g.x0 ? g.x_lim - g.x0 : 0;
  const unsigned long long ey = g.y_lim - R;
  const unsigned nxt = std::max(1u, cdiv(ex, TX));
  unsigned nyt = 1;
  unsigned long long M = ey;
  if (s.dimension == 3) {
    nyt = std::max(1u, cdiv(ey, (unsigned long long)L->block[1] * s.cy));
    M = g.z_lim - R;
  }
  unsigned nseg = L->segments;
  if (nseg == 0) {
    const unsigned long long slots = (unsigned long long)h->num_sms * (unsigned)occ;
    const unsigned long long tiles = (unsigned long long)nxt * nyt;
    nseg = (unsigned)std::max<unsigned long long>(1, slots / std::max<unsigned long long>(1, tiles));
  }
  const unsigned max_seg = std::max(1u, cdiv(M, STEP));
  nseg = std::min(nseg, max_seg);
  unsigned seg = cdiv(std::max<unsigned long long>(M, 1), nseg);
  seg = cdiv(seg, STEP) * STEP;
  nseg = std::max(1u, cdiv(std::max<unsigned long long>(M, 1), seg));

  out.variant = TCS_VARIANT_MARCH;
  out.geo = g;
  out.geo.seg = seg;
  out.geo.nslot = nslot;
  out.geo.width = W;
  out.geo.loader = loader;
  for (int i = 0; i < 3; ++i) out.block[i] = L->block[i];
  if (s.dimension == 2) {
    out.grid[0] = nxt;
    out.grid[1] = nseg;
    out.grid[2] = 1;
    out.box[0] = W;
    out.box[1] = STEP;
    out.box[2] = 1;
  } else {
    out.grid[0] = nxt;
    out.grid[1] = nyt;
    out.grid[2] = nseg;
    out.box[0] = W;
    out.box[1] = rows;
    out.box[2] = STEP;
  }
  if (out.grid[1] > 65535 || out.grid[2] > 65535)
    return fail(TCS_ERR_UNSUPPORTED, "march launch grid exceeds 65535 blocks in y or z");
  out.smem = smem;
  out.depth = depth;
  out.occ = occ;
  return TCS_OK;
}

int upload_mask(tcs_stencil* h, CUdeviceptr dst) {
  const unsigned n = (unsigned)h->mask_host.size();
  if (n == 0 || h->spec.coefficients == TCS_JACOBI) return TCS_OK;
  if (h->spec.precision == TCS_F64) {
    TCS_RT(cudaMemcpy((void*)dst, h->mask_host.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
  } else {
    std::vector<float> f(h->mask_host.begin(), h->mask_host.end());
    TCS_RT(cudaMemcpy((void*)dst, f.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
  }
  return TCS_OK;
}

// The mask of a pipelined module: tcs_mask, and the (m_k, m_k) pairs of packed FP32 instances.
int upload_pipe_mask(tcs_stencil* h, const PipeMod* pm) {
  int rc = upload_mask(h, pm->mask_ptr);
  if (rc) return rc;
  const unsigned n = (unsigned)h->mask_host.size();
  if (!pm->pairs_ptr || n == 0 || h->spec.coefficients == TCS_JACOBI || h->spec.precision == TCS_F64 ||
      pm->pairs_bytes != 2 * sizeof(float) * n)
    return TCS_OK;
  std::vector<float> f(2 * n);
  for (unsigned k = 0; k < n; ++k) f[2 * k] = f[2 * k + 1] = (float)h->mask_host[k];
  TCS_RT(cudaMemcpy((void*)pm->pairs_ptr, f.data(), sizeof(float) * 2 * n, cudaMemcpyHostToDevice));
  return TCS_OK;
}

// Pipelined-sweep module for a launch shape: instantiate (NVRTC, cached) and load on first use.
int pipe_module(tcs_stencil* h, const PipeKey& key, PipeMod** out) {
  std::lock_guard<std::mutex> lock(h->mu);
  for (PipeMod* p : h->pipes)
    if (p->key == key) {
      *out = p;
      return TCS_OK;
    }
  std::vector<char> cubin;
  int rc = instantiate(h->spec, &key, cubin, nullptr);
  if (rc) return rc;
  PipeMod* pm = new PipeMod();
  pm->key = key;
  CUresult cr = g_drv.ModuleLoadData(&pm->mod, cubin.data());
  if (cr != CUDA_SUCCESS) {
    delete pm;
    return fail(TCS_ERR_CUDA, "cuModuleLoadData (pipe): " + cu_msg(cr));
  }
  size_t bytes = 0;
  if ((cr = g_drv.ModuleGetFunction(&pm->f, pm->mod,
                                    key.batch ? "tcs_pipe_batch" : (key.tb3 ? "tcs_tb3" : "tcs_pipe"))) !=
          CUDA_SUCCESS ||
      (cr = g_drv.ModuleGetGlobal(&pm->mask_ptr, &pm->mask_bytes, pm->mod, "tcs_mask")) != CUDA_SUCCESS ||
      (cr = g_drv.ModuleGetGlobal(&pm->status_ptr, &bytes, pm->mod, "tcs_status")) != CUDA_SUCCESS) {
    g_drv.ModuleUnload(pm->mod);
    delete pm;
    return fail(TCS_ERR_CUDA, "pipe module symbols: " + cu_msg(cr));
  }
  if (g_drv.ModuleGetGlobal(&pm->pairs_ptr, &pm->pairs_bytes, pm->mod, "tcs_mask_pairs") != CUDA_SUCCESS) {
    pm->pairs_ptr = 0;
    pm->pairs_bytes = 0;
  }
  cudaMemset((void*)pm->status_ptr, 0, sizeof(unsigned));
  rc = upload_pipe_mask(h, pm);
  if (rc) {
    g_drv.ModuleUnload(pm->mod);
    delete pm;
    return rc;
  }
  h->pipes.push_back(pm);
  *out = pm;
  return TCS_OK;
}

// Default planes per ring chunk, which is also the unroll depth of the pipe kernel's loop body.
// Limits: an instruction budget of about 2000 fused multiply-adds per body (one plane applies S
// terms to each of the thread's NEP outputs) and a chunk small enough that two ring slots fit
// in the shared memory left to each CTA at the occupancy the registers allow.  Among the
// feasible depths, a divisor of 2R+1 (no register permutation at the loop back-edge) is
// preferred unless it is less than half the largest feasible depth.
unsigned pipe_auto_chunk(const tcs_spec& s, unsigned bx, unsigned by) {
  const unsigned es = (unsigned)elem_size(s), vec = 16u / es;
  const unsigned R = (unsigned)s.range;
  const unsigned nep = (unsigned)s.cx * (s.dimension == 3 ? (unsigned)s.cy : 1u);
  const unsigned n = 2u * R + 1u;
  const unsigned S = stencil_size_of(s);
  const unsigned tx = bx * (unsigned)s.cx;
  const unsigned rows = s.dimension == 3 ? by * (unsigned)s.cy + 2u * R : 1u;
  const unsigned plane_bytes = ((tx + 2u * R + 2u * vec) / vec * vec) * rows * es;
  const unsigned threads = bx * (s.dimension == 3 ? by : 1u);
  const unsigned regs = std::min(255u, n * nep * (es / 4u) + 48u);
  const unsigned occ = std::max(1u, 65536u / (((regs + 7u) / 8u * 8u) * threads));
  const unsigned max_chunk = std::min(227u * 1024u, 228u * 1024u / std::min(occ, 8u)) / 2u;
  const unsigned budget = std::max(1u, 2000u / std::max(1u, S * nep));
  unsigned best = 1;
  for (unsigned c = 1; c <= std::min(budget, 4u * n); ++c)
    if (c * plane_bytes <= max_chunk) best = c;
  unsigned div = 1;
  for (unsigned c = 1; c <= best; ++c)
    if (n % c == 0 || c % n == 0) div = c;
  return (2 * div >= best) ? div : best;
}

// Compile-time row width of a pipe instantiation (tcs::pipe_width in tcs_kernels.cuh).
unsigned pipe_width(unsigned tx, unsigned R, unsigned lshift, unsigned vec, unsigned ch,
                    unsigned rows, unsigned es) {
  unsigned w = ((tx + 2 * R + lshift + vec - 1) / vec) * vec;
  while ((ch * rows * w * es) % 128 != 0) w += vec;
  return w;
}

// Loader of the pipe kernel for a row pitch (and input base, when known): 0 = TMA (pitch and
// base on 16 bytes), 2 = cp.async of element pairs (FP32 with an even pitch and an 8-byte base),
// 1 = cp.async of single elements.
// cp.async loaders: pairs of floats where the pitch and the base allow it, else single elements.
unsigned pipe_loader_cp(const tcs_spec& s, unsigned long long xdim, const void* in) {
  const uintptr_t base = reinterpret_cast<uintptr_t>(in);
  if (elem_size(s) == 4 && xdim % 2 == 0 && base % 8 == 0) return 2u;
  return 1u;
}

unsigned pipe_loader(const tcs_spec& s, unsigned long long xdim, const void* in) {
  const unsigned es = (unsigned)elem_size(s);
  const uintptr_t base = reinterpret_cast<uintptr_t>(in);
  if ((xdim * es) % 16 == 0 && base % 16 == 0) return 0u;
  return pipe_loader_cp(s, xdim, in);
}

// The pipelined kernel's compensated FP32 form is the packed-pair Box path (tcs_tile.cuh):
// Box neighbourhood, Row order (or 2D), even x coarsening.
bool pipe_comp_ok(const tcs_spec& s) {
  return s.neighbourhood == TCS_BOX && s.cx % 2 == 0 && (s.dimension == 2 || s.orientation == TCS_ROW);
}

int resolve_pipe(tcs_stencil* h, const TcsGeo& g, const tcs_launch* L, Resolved& out,
                 bool batch = false, unsigned epi = 0) {
  const tcs_spec& s = h->spec;
  if (s.precision == TCS_F32C && !pipe_comp_ok(s))
    return fail(TCS_ERR_UNSUPPORTED,
                "compensated FP32 pipelined sweeps need a Box stencil in Row order with an even x coarsening");
  const unsigned R = (unsigned)s.range;
  const unsigned es = (unsigned)elem_size(s);
  const unsigned vec = 16u / es;
  if (s.dimension == 2 && s.orientation == TCS_COLUMN)
    return fail(TCS_ERR_UNSUPPORTED, "2D Column orientation is not pipelined");
  if (s.dimension == 2 && (L->block[1] != 1 || L->block[2] != 1))
    return fail(TCS_ERR_UNSUPPORTED, "pipe: 2D blocks are (bx, 1, 1)");
  if (s.dimension == 3 && L->block[2] != 1)
    return fail(TCS_ERR_UNSUPPORTED, "pipe: 3D blocks are (bx, by, 1)");
  const unsigned TX = L->block[0] * s.cx;
  if (TX % vec != 0) return fail(TCS_ERR_UNSUPPORTED, "pipe: tile width not a multiple of 16 bytes");
  const unsigned TY = s.dimension == 3 ? L->block[1] * s.cy : 1;
  const unsigned rows = s.dimension == 3 ? TY + 2 * R : 1;
  const unsigned lshift = h->left_off % vec;
  const unsigned ch = L->chunk ? L->chunk : pipe_auto_chunk(s, L->block[0], L->block[1]);
  const unsigned W = pipe_width(TX, R, lshift, vec, ch, rows, es);
  // A TMA box is at most 256 elements per dimension.  A single-grid sweep that asks for the pipe
  // kernel with wider tile rows streams them through cp.async instead (the automatic choice keeps
  // such shapes on the march and direct kernels; the batch's table holds one tensor map per grid).
  if (rows > 256 || ch > 256 || (W > 256 && (batch || L->variant != TCS_VARIANT_PIPE)))
    return fail(TCS_ERR_UNSUPPORTED, "pipe: tile exceeds the 256-element TMA box limit");
  const bool no_tma = W > 256;
  const unsigned chunk_bytes = ch * rows * W * es;
  // Star middle rows through warp shuffles: on request (TCS_LAUNCH_SHUFFLE), where the block's rows
  // are whole warps
  const bool shfl_ok = s.neighbourhood == TCS_STAR && (s.dimension == 2 || s.orientation == TCS_ROW) &&
                       L->block[0] % 32 == 0;
  if ((L->flags & TCS_LAUNCH_SHUFFLE) && !shfl_ok)
    return fail(TCS_ERR_UNSUPPORTED, "pipe: shuffled rows need a Star stencil in Row order and bx % 32 == 0");
  const unsigned shfl = ((L->flags & TCS_LAUNCH_SHUFFLE) && shfl_ok) ? 1u : 0u;
  // the ring form in tensor memory: on request (TCS_LAUNCH_TMEM), plain single-grid sweeps
  const unsigned tm_cols = tmem_cols(s, L->block[0], s.dimension == 3 ? L->block[1] : 1u);
  if ((L->flags & TCS_LAUNCH_TMEM) && (tm_cols == 0 || batch || epi || shfl))
    return fail(TCS_ERR_UNSUPPORTED,
                "pipe: the tensor-memory ring form needs a 3D Star stencil in Row order (FP64 or FP32), "
                "cx*cy*sizeof/4 of 4, 8, 16 or 32, a plain single-grid sweep");
  const unsigned tmem = (L->flags & TCS_LAUNCH_TMEM) ? 1u : 0u;
  PipeKey key{L->block[0], s.dimension == 3 ? L->block[1] : 1u, ch, lshift, batch ? 1u : 0u, epi, 0u, shfl, tmem};
  PipeMod* pm = nullptr;
  int rc = pipe_module(h, key, &pm);
  if (rc) return rc;
  const int nthr = (int)(L->block[0] * L->block[1]);
  int maxthr = 0;
  TCS_CU(g_drv.FuncGetAttribute(&maxthr, CU_FUNC_ATTRIBUTE_MAX_THREADS_PER_BLOCK, pm->f));
  if (nthr > maxthr) return fail(TCS_ERR_UNSUPPORTED, "pipe: block exceeds the kernel's thread limit");
  const unsigned bar_area = 256;  // barriers + alignment slack, rounded
  unsigned depth = L->depth;
  if (depth == 0) {
    // Enough chunks in flight to keep about 96 KB of input moving per SM at the occupancy the
    // registers allow, within the shared memory those CTAs share.
    int occ_r = 0;
    TCS_CU(g_drv.OccMaxActive(&occ_r, pm->f, nthr, 0));
    occ_r = std::max(1, occ_r);
    const unsigned smem_sm = 228u * 1024u;
    depth = 2;
    for (unsigned d = 2; d <= 16; ++d) {
      const unsigned per_cta = bar_area + (1 + d) * chunk_bytes;
      const unsigned fit = std::min<unsigned>((unsigned)occ_r, smem_sm / per_cta);
      if (fit == 0 || per_cta > (unsigned)h->smem_optin) break;
      depth = d;
      if ((unsigned long long)fit * d * chunk_bytes >= 96ull * 1024ull &&
          fit >= std::min<unsigned>((unsigned)occ_r, 2u))
        break;
    }
  }
  unsigned smem = 0, nslot = 0;
  for (;;) {
    nslot = 1 + depth;
    smem = ((nslot * 8 + 127) / 128) * 128 + 128 + nslot * chunk_bytes;
    if (smem <= (unsigned)h->smem_optin || depth == 1) break;
    --depth;
  }
  if (smem > (unsigned)h->smem_optin)
    return fail(TCS_ERR_UNSUPPORTED, "pipe: ring does not fit in shared memory");
  {
    std::lock_guard<std::mutex> lock(h->mu);
    if ((int)smem > pm->smem_attr) {
      TCS_CU(g_drv.FuncSetAttribute(pm->f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)smem));
      pm->smem_attr = (int)smem;
    }
  }
  int occ = 0;
  TCS_CU(g_drv.OccMaxActive(&occ, pm->f, nthr, smem));
  if (occ < 1) return fail(TCS_ERR_UNSUPPORTED, "pipe kernel cannot be resident at this shape");
  if (tmem) {
    // Every resident CTA holds tm_cols tensor-memory columns: no more CTAs on an SM than its 512
    // columns serve (an allocation beyond them would wait for another CTA to finish).  Where the
    // registers and the ring would admit more, the dynamic shared memory grows until they do not.
    const int cap = (int)(512u / tm_cols);
    while (occ > cap) {
      smem = std::min<unsigned>((unsigned)h->smem_optin, smem + 4096u);
      {
        std::lock_guard<std::mutex> lock(h->mu);
        if ((int)smem > pm->smem_attr) {
          TCS_CU(g_drv.FuncSetAttribute(pm->f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)smem));
          pm->smem_attr = (int)smem;
        }
      }
      TCS_CU(g_drv.OccMaxActive(&occ, pm->f, nthr, smem));
      if (smem >= (unsigned)h->smem_optin && occ > cap)
        return fail(TCS_ERR_UNSUPPORTED, "pipe: cannot limit the CTAs per SM to the tensor-memory columns");
    }
    if (occ < 1) return fail(TCS_ERR_UNSUPPORTED, "pipe kernel cannot be resident at this shape");
  }
  const unsigned long long ex = g.x_lim > g.x0 ? g.x_lim - g.x0 : 0;
  const unsigned long long ey = g.y_lim - R;
  const unsigned ntx = std::max(1u, cdiv(ex, TX));
  unsigned nty = 1;
  unsigned long long M = ey;
  if (s.dimension == 3) {
    nty = std::max(1u, cdiv(ey, TY));
    M = g.z_lim - R;
  }
  const unsigned long long total = (unsigned long long)ntx * nty * M;
  unsigned long long nctas = (unsigned long long)h->num_sms * (unsigned)occ;
  if (L->flags & TCS_LAUNCH_LOCKSTEP) {
    // Whole tile columns (or 1/k of one) per CTA, k as large as the resident CTAs allow: every
    // CTA starts at a column's (or a column part's) first plane, so neighbouring tiles sweep the
    // same planes at the same time and their shared halo rows come from L2, not DRAM.
    const unsigned long long tiles = (unsigned long long)ntx * nty;
    const unsigned long long k = std::max<unsigned long long>(1, nctas / tiles);
    nctas = tiles * std::min<unsigned long long>(k, M);
  }
  if (L->segments) nctas = L->segments;  // explicit CTA count
  const unsigned long long per = std::max<unsigned long long>(1, (total + nctas - 1) / nctas);
  const unsigned long long grid = std::max<unsigned long long>(1, (total + per - 1) / per);
  if (grid > 0x7fffffffull) return fail(TCS_ERR_UNSUPPORTED, "pipe grid too large");
  out.variant = TCS_VARIANT_PIPE;
  out.no_tma = no_tma;
  out.geo = g;
  out.geo.width = W;
  out.geo.nslot = nslot;
  out.pipe = pm;
  out.chunk = ch;
  TcsPipeGeo& pg = out.pgeo;
  pg = TcsPipeGeo{};
  pg.xdim = g.xdim;
  pg.ydim = g.ydim;
  pg.zdim = g.zdim;
  pg.total = total;
  pg.per_cta = per;
  pg.x0 = g.x0;
  pg.x_lim = g.x_lim;
  pg.y_lim = g.y_lim;
  pg.z_lim = g.z_lim;
  pg.ntx = ntx;
  pg.m = (unsigned)M;
  pg.nslot = nslot;
  pg.loader = no_tma ? pipe_loader_cp(s, g.xdim, nullptr) : pipe_loader(s, g.xdim, nullptr);
  out.geo.loader = pg.loader;
  out.geo.seg = (unsigned)std::min<unsigned long long>(per, 0xffffffffull);
  out.grid[0] = (unsigned)grid;
  out.grid[1] = 1;
  out.grid[2] = 1;
  out.block[0] = L->block[0];
  out.block[1] = s.dimension == 3 ? L->block[1] : 1;
  out.block[2] = 1;
  if (s.dimension == 2) {
    out.box[0] = W;
    out.box[1] = ch;
    out.box[2] = 1;
  } else {
    out.box[0] = W;
    out.box[1] = rows;
    out.box[2] = ch;
  }
  out.smem = smem;
  out.depth = depth;
  out.occ = occ;
  return TCS_OK;
}

// The two-sweep kernel tcs_tb3.  3D: thread tiles C x C with C = 2 for even ranges and 1 for odd
// ones (C divides R, so a thread tile lies wholly inside or outside the output tile); by default
// an extended tile of 64 x 32 columns (C = 2: 32 x 16 threads) or 32 x 32 (C = 1: 32 x 32
// threads), whose inner (EX - 2R) x (EY - 2R) columns are the output tile.  2D (Row order): a
// strip of EX = bx * 2 columns marching along y, thread tiles 2 x 1 (which may straddle the
// output strip's edge), by default 64 threads (narrower where a TMA box needs it), whose inner
// EX - 2R columns are the output strip.  `L` (may be NULL) gives the block (bx, by), the
// planes (2D: rows) per ring chunk, the chunks in flight and the CTA count.
int resolve_tb3(tcs_stencil* h, const TcsGeo& g, const tcs_launch* L, Resolved& out) {
  const tcs_spec& s = h->spec;
  if (s.precision == TCS_F32C) return fail(TCS_ERR_UNSUPPORTED, "tb3: plain FP64 or FP32 sweeps only");
  if (s.dimension == 2 && s.orientation == TCS_COLUMN)
    return fail(TCS_ERR_UNSUPPORTED, "tb3: 2D stencils in Row order only");
  const bool d3 = s.dimension == 3;
  const unsigned R = (unsigned)s.range;
  const unsigned es = (unsigned)elem_size(s), vec = 16u / es;
  const unsigned C = (R % 2 == 0 || !d3) ? 2u : 1u;
  // 2D: 64 threads (128-column strips) by default; on the 4096^2 Box r1 grid 64, 96, 120 and 126
  // threads measured 514, 500-520, 504 and 503-520 GLup/s
  unsigned bx = d3 ? 32u : 64u, by = d3 ? ((C == 2) ? 16u : 32u) : 1u;
  while (!d3 && bx > 8 && bx * C + 2 * R + vec > 256) bx -= 8;  // 2D: the strip fits a TMA box
  if (L && L->block[0]) {
    bx = L->block[0];
    by = L->block[1] ? L->block[1] : 1u;
  }
  if (!d3 && by != 1) return fail(TCS_ERR_UNSUPPORTED, "tb3: 2D blocks are (bx, 1, 1)");
  const unsigned EX = bx * C, EY = d3 ? by * C : 1u;
  if (EX <= 2 * R || (d3 && EY <= 2 * R)) return fail(TCS_ERR_UNSUPPORTED, "tb3: tile too small for the range");
  const unsigned OX = EX - 2 * R, OY = d3 ? EY - 2 * R : 1u;
  if (OX % vec != 0 || EX % vec != 0)
    return fail(TCS_ERR_UNSUPPORTED, "tb3: extended or output tile width not a multiple of 16 bytes");
  const unsigned lshift = (unsigned)((((int)h->left_off - (int)R) % (int)vec + (int)vec) % (int)vec);
  // 2D rows are short: 8 per chunk by default (a chunk of 8 rows is a multiple of 128 bytes for
  // any row width, so the ring rows need no padding and the TMA box reads no extra columns)
  const unsigned ch = (L && L->chunk) ? L->chunk : (d3 ? 2u : 8u);
  const unsigned rows = d3 ? EY + 2 * R : 1u;
  const unsigned W = pipe_width(EX, R, lshift, vec, ch, rows, es);
  if (W > 256 || rows > 256 || ch > 256)
    return fail(TCS_ERR_UNSUPPORTED, "tb3: tile exceeds the 256-element TMA box limit");
  const unsigned chunk_bytes = ch * rows * W * es;
  // two plane buffers; a 2D row has its left margin rounded up to even and an even width (at
  // most EX + 2R + 2 elements)
  const unsigned buf_bytes = 2u * (d3 ? (EX + 2 * R) * (EY + 2 * R) : EX + 2 * R + 2) * es;
  PipeKey key{bx, by, ch, lshift, 0u, 0u, C};
  PipeMod* pm = nullptr;
  int rc = pipe_module(h, key, &pm);
  if (rc) return rc;
  const int nthr = (int)(bx * by);
  int maxthr = 0;
  TCS_CU(g_drv.FuncGetAttribute(&maxthr, CU_FUNC_ATTRIBUTE_MAX_THREADS_PER_BLOCK, pm->f));
  if (nthr > maxthr) return fail(TCS_ERR_UNSUPPORTED, "tb3: block exceeds the kernel's thread limit");
  // 2D: one chunk in flight by default (the smaller ring admits more CTAs per SM; measured on the
  // 4096^2 Box r1 grid: 520.9 GLup/s against 503.8 with two)
  unsigned nslot = (L && L->depth) ? 1 + L->depth : (d3 ? 3u : 2u), smem = 0;
  for (;; --nslot) {
    smem = ((nslot * 8 + 127) / 128) * 128 + 128 + nslot * chunk_bytes + buf_bytes;
    if (smem <= (unsigned)h->smem_optin || nslot == 2) break;
  }
  if (smem > (unsigned)h->smem_optin) return fail(TCS_ERR_UNSUPPORTED, "tb3: ring does not fit in shared memory");
  {
    std::lock_guard<std::mutex> lock(h->mu);
    if ((int)smem > pm->smem_attr) {
      TCS_CU(g_drv.FuncSetAttribute(pm->f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)smem));
      pm->smem_attr = (int)smem;
    }
  }
  int occ = 0;
  TCS_CU(g_drv.OccMaxActive(&occ, pm->f, nthr, smem));
  if (occ < 1) return fail(TCS_ERR_UNSUPPORTED, "tb3 kernel cannot be resident at this shape");
  const unsigned long long ex = g.x_lim > g.x0 ? g.x_lim - g.x0 : 0;
  const unsigned ntx = std::max(1u, cdiv(ex, OX)), nty = d3 ? std::max(1u, cdiv(g.y_lim - R, OY)) : 1u;
  const unsigned long long M = d3 ? g.z_lim - R : g.y_lim - R;
  const unsigned long long total = (unsigned long long)ntx * nty * M;
  unsigned long long nctas = (unsigned long long)h->num_sms * (unsigned)occ;
  if (!d3) {
    // 2D: three waves of resident CTAs (on the 4096^2 Box r1 grid 1, 1.6, 2.4, 3.2 and 4.8 waves
    // of 128-thread CTAs measured 369, 467, 520, 521 and 521 GLup/s: later waves fill the SMs
    // whose CTAs finish first), but pieces of at least 16 rows (each re-reads 4R rows and
    // recomputes 2R rows of stage 1).
    const unsigned long long cap = std::max<unsigned long long>((unsigned long long)h->num_sms, total / 16);
    nctas = std::min(3 * nctas, cap);
  }
  if (L && L->segments) nctas = L->segments;
  const unsigned long long per = std::max<unsigned long long>(1, (total + nctas - 1) / nctas);
  const unsigned long long grid = std::max<unsigned long long>(1, (total + per - 1) / per);
  out = Resolved{};
  out.variant = TCS_VARIANT_PIPE;
  out.geo = g;
  out.geo.width = W;
  out.geo.nslot = nslot;
  out.pipe = pm;
  out.chunk = ch;
  TcsPipeGeo& pg = out.pgeo;
  pg = TcsPipeGeo{};
  pg.xdim = g.xdim;
  pg.ydim = g.ydim;
  pg.zdim = g.zdim;
  pg.total = total;
  pg.per_cta = per;
  pg.x0 = g.x0;
  pg.x_lim = g.x_lim;
  pg.y_lim = g.y_lim;
  pg.z_lim = g.z_lim;
  pg.ntx = ntx;
  pg.m = (unsigned)M;
  pg.nslot = nslot;
  pg.loader = ((g.xdim * es) % 16 == 0) ? 0u : 1u;
  out.geo.loader = pg.loader;
  out.grid[0] = (unsigned)grid;
  out.block[0] = bx;
  out.block[1] = by;
  out.block[2] = 1;
  out.box[0] = W;
  out.box[1] = d3 ? rows : ch;
  out.box[2] = d3 ? ch : 1u;
  out.smem = smem;
  out.depth = nslot - 1;
  out.occ = occ;
  return TCS_OK;
}

int fill_plan(const tcs_stencil* h, const Resolved& r, tcs_plan* out) {
  if (out) {
    tcs_plan p{};
    p.variant = r.variant;
    for (int i = 0; i < 3; ++i) {
      p.grid_blocks[i] = r.grid[i];
      p.block[i] = r.block[i];
    }
    p.dyn_smem = r.smem;
    p.seg_len = r.geo.seg;
    p.nslot = r.geo.nslot;
    p.width = r.geo.width;
    p.chunk = r.chunk;
    p.depth = r.depth;
    p.loader = r.geo.loader;
    p.ctas_per_sm = r.occ;
    p.num_sms = h->num_sms;
    *out = p;
  }
  return TCS_OK;
}

int resolve(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, const tcs_launch* L,
            Resolved& out) {
  if (!h || !L) return fail(TCS_ERR_INVALID_VALUE, "NULL handle or launch");
  TcsGeo g;
  int rc = make_geo(h, grid, right_offset, g);
  if (rc) return rc;
  rc = check_block(h, L->block);
  if (rc) return rc;
  if (L->variant == TCS_VARIANT_DIRECT) return resolve_direct(h, g, L, out);
  if (L->variant == TCS_VARIANT_MARCH) return resolve_march(h, g, L, out);
  if (L->variant == TCS_VARIANT_PIPE) return resolve_pipe(h, g, L, out);
  if (L->variant != TCS_VARIANT_AUTO) return fail(TCS_ERR_INVALID_VALUE, "unknown variant");
  const std::string saved = g_err;
  rc = resolve_pipe(h, g, L, out);
  if (rc == TCS_OK) return rc;
  if (rc != TCS_ERR_UNSUPPORTED) return rc;
  rc = resolve_march(h, g, L, out);
  if (rc == TCS_OK) return rc;
  if (rc != TCS_ERR_UNSUPPORTED) return rc;
  g_err = saved;
  return resolve_direct(h, g, L, out);
}

// Tiled tensor map of a grid buffer (rank = dimension, x innermost) with the given box.
int encode_map(const tcs_spec& s, const void* ptr, const unsigned long long dims[3],
               const unsigned box_in[3], CUtensorMap* map) {
  if (reinterpret_cast<uintptr_t>(ptr) % 16 != 0)
    return fail(TCS_ERR_INVALID_VALUE, "input buffer is not 16-byte aligned (TMA rule)");
  const unsigned es = (unsigned)elem_size(s);
  const cuuint32_t rank = (cuuint32_t)s.dimension;
  cuuint64_t gdim[3] = {dims[0], dims[1], dims[2]};
  cuuint64_t gstride[2] = {dims[0] * es, dims[0] * dims[1] * es};
  cuuint32_t box[3] = {box_in[0], box_in[1], box_in[2]};
  cuuint32_t estride[3] = {1, 1, 1};
  CUresult cr = g_drv.TensorMapEncodeTiled(
      map, s.precision == TCS_F64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
      rank, const_cast<void*>(ptr), gdim, gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (cr != CUDA_SUCCESS) return fail(TCS_ERR_CUDA, "cuTensorMapEncodeTiled: " + cu_msg(cr));
  return TCS_OK;
}

int tensor_map(tcs_stencil* h, const void* ptr, const Resolved& r, CUtensorMap** out) {
  std::lock_guard<std::mutex> lock(h->mu);
  const unsigned long long dims[3] = {r.geo.xdim, r.geo.ydim, r.geo.zdim};
  for (auto& m : h->maps) {
    if (m.ptr == ptr && std::memcmp(m.dims, dims, sizeof(dims)) == 0 &&
        std::memcmp(m.box, r.box, sizeof(r.box)) == 0) {
      *out = &m.map;
      return TCS_OK;
    }
  }
  MapEntry e;
  e.ptr = ptr;
  std::memcpy(e.dims, dims, sizeof(dims));
  std::memcpy(e.box, r.box, sizeof(r.box));
  int rc = encode_map(h->spec, ptr, dims, r.box, &e.map);
  if (rc) return rc;
  if (h->maps.size() > 64) h->maps.erase(h->maps.begin());
  h->maps.push_back(e);
  *out = &h->maps.back().map;
  return TCS_OK;
}

// ---- ragged grids --------------------------------------------------------------------------
// Every kernel updates whole coarsening tiles only, like the reference's.  When the interior is
// not a multiple of the coarsening (a grid from tcs_compute_geometry_ragged), the points of the
// partial tiles -- the fringe -- are swept by a second instance of the direct kernel with
// coarsening 1 x 1 x 1.  The per-point term order does not depend on the coarsening, so the fringe
// values are the ones a coarsening-1 sweep of the whole grid would give, bit for bit.
int fringe_module(tcs_stencil* h) {
  std::lock_guard<std::mutex> lock(h->mu);
  if (h->fringe_mod) return TCS_OK;
  tcs_spec s1 = h->spec;
  s1.cx = s1.cy = s1.cz = 1;
  std::vector<char> cubin;
  int rc = instantiate(s1, nullptr, cubin, nullptr);
  if (rc) return rc;
  CUmodule mod = nullptr;
  CUresult cr = g_drv.ModuleLoadData(&mod, cubin.data());
  if (cr != CUDA_SUCCESS) return fail(TCS_ERR_CUDA, "cuModuleLoadData (fringe): " + cu_msg(cr));
  size_t bytes = 0;
  if ((cr = g_drv.ModuleGetFunction(&h->f_fringe, mod, "tcs_direct")) != CUDA_SUCCESS ||
      (cr = g_drv.ModuleGetGlobal(&h->fringe_mask, &bytes, mod, "tcs_mask")) != CUDA_SUCCESS) {
    g_drv.ModuleUnload(mod);
    return fail(TCS_ERR_CUDA, "fringe module symbols: " + cu_msg(cr));
  }
  h->fringe_mod = mod;
  return upload_mask(h, h->fringe_mask);
}

// Does a sweep of this geometry leave partial coarsening tiles to the coarsening-1 fringe kernel?
bool has_fringe(const tcs_stencil* h, const TcsGeo& g) {
  const tcs_spec& s = h->spec;
  const bool d3 = s.dimension == 3;
  const unsigned R = (unsigned)s.range;
  const unsigned cz = d3 ? (unsigned)s.cz : 1u;
  const unsigned ex = g.x_lim > g.x0 ? g.x_lim - g.x0 : 0, ey = g.y_lim - R, ez = d3 ? g.z_lim - R : 0;
  return ex % (unsigned)s.cx != 0 || ey % (unsigned)s.cy != 0 || (d3 && ez % cz != 0);
}

int launch_fringe(tcs_stencil* h, const TcsGeo& g, const void* in, void* out, const void* src, CUstream st) {
  const tcs_spec& s = h->spec;
  const bool d3 = s.dimension == 3;
  const unsigned R = (unsigned)s.range;
  const unsigned cz = d3 ? (unsigned)s.cz : 1u;
  const unsigned ex = g.x_lim > g.x0 ? g.x_lim - g.x0 : 0, ey = g.y_lim - R, ez = d3 ? g.z_lim - R : 0;
  const unsigned xf = g.x0 + ex / s.cx * s.cx, yf = R + ey / s.cy * s.cy, zf = d3 ? R + ez / cz * cz : g.z_lim;
  if (xf == g.x0 + ex && yf == g.y_lim && zf == g.z_lim) return TCS_OK;
  int rc = fringe_module(h);
  if (rc) return rc;
  const size_t es = (size_t)elem_size(s);
  // regions [xa, xb) x [ya, yb) x [za, zb): the partial x tiles, then partial y, then partial z
  const unsigned z0 = d3 ? R : 0;
  const unsigned reg[3][6] = {{xf, g.x_lim, R, g.y_lim, z0, g.z_lim},
                              {g.x0, xf, yf, g.y_lim, z0, g.z_lim},
                              {g.x0, xf, R, yf, zf, g.z_lim}};
  for (int k = 0; k < (d3 ? 3 : 2); ++k) {
    const unsigned xa = reg[k][0], xb = reg[k][1], ya = reg[k][2], yb = reg[k][3], za = reg[k][4], zb = reg[k][5];
    if (xa >= xb || ya >= yb || (d3 && za >= zb)) continue;
    // The direct kernel starts at row R and plane R: shift the buffers so that those are ya, za.
    const size_t shift = ((size_t)(ya - R) * g.xdim + (d3 ? (size_t)(za - R) * g.xdim * g.ydim : 0)) * es;
    TcsGeo f = g;
    f.x0 = xa;
    f.x_lim = xb;
    f.y_lim = yb - (ya - R);
    f.z_lim = d3 ? zb - (za - R) : g.z_lim;
    CUdeviceptr pin = (CUdeviceptr)in + shift, pout = (CUdeviceptr)out + shift;
    CUdeviceptr psrc = src ? (CUdeviceptr)src + shift : 0;
    void* args[] = {&pin, &pout, &psrc, &f};
    const unsigned bx = 32, by = 4, bz = d3 ? 2 : 1;
    TCS_CU(g_drv.LaunchKernel(h->f_fringe, cdiv(xb - xa, bx), cdiv(yb - ya, by), d3 ? cdiv(zb - za, bz) : 1, bx, by,
                              bz, 0, st, args, nullptr));
  }
  return TCS_OK;
}

int launch_tb3(tcs_stencil* h, const Resolved& r, const void* in, void* out, CUstream st) {
  TcsPipeGeo pg = r.pgeo;
  if (reinterpret_cast<uintptr_t>(in) % 16 != 0) pg.loader = 1;  // TMA needs a 16-byte aligned base
  alignas(64) CUtensorMap pmap;
  std::memset(&pmap, 0, sizeof(pmap));
  if (pg.loader == 0) {
    CUtensorMap* map = nullptr;
    int rc = tensor_map(h, in, r, &map);
    if (rc) return rc;
    pmap = *map;
  }
  CUdeviceptr pin = (CUdeviceptr)in, pout = (CUdeviceptr)out;
  void* args[] = {&pmap, &pin, &pout, &pg};
  TCS_CU(g_drv.LaunchKernel(r.pipe->f, r.grid[0], 1, 1, r.block[0], r.block[1], 1, r.smem, st, args, nullptr));
  return TCS_OK;
}

// `pre`: an already encoded tensor map of `in` for the pipe kernel (skips the map cache).
int launch_resolved(tcs_stencil* h, const Resolved& r, const void* in, void* out, CUstream st,
                    const void* src = nullptr, const CUtensorMap* pre = nullptr) {
  if (!in || !out) return fail(TCS_ERR_INVALID_VALUE, "NULL device buffer");
  if (in == out) return fail(TCS_ERR_INVALID_VALUE, "input and output must be distinct buffers");
  if (src == out) return fail(TCS_ERR_INVALID_VALUE, "source and output must be distinct buffers");
  CUdeviceptr psrc = (CUdeviceptr)src;
  TcsGeo geo = r.geo;
  if (r.variant == TCS_VARIANT_DIRECT) {
    CUdeviceptr pin = (CUdeviceptr)in, pout = (CUdeviceptr)out;
    void* args[] = {&pin, &pout, &psrc, &geo};
    TCS_CU(g_drv.LaunchKernel(h->f_direct, r.grid[0], r.grid[1], r.grid[2], r.block[0],
                              r.block[1], r.block[2], 0, st, args, nullptr));
    return launch_fringe(h, r.geo, in, out, src, st);
  }
  if (r.variant == TCS_VARIANT_PIPE) {
    TcsPipeGeo pg = r.pgeo;
    pg.loader = r.no_tma ? pipe_loader_cp(h->spec, pg.xdim, in) : pipe_loader(h->spec, pg.xdim, in);
    alignas(64) CUtensorMap pmap;
    std::memset(&pmap, 0, sizeof(pmap));
    if (pg.loader == 0 && pre) {
      pmap = *pre;
    } else if (pg.loader == 0) {
      CUtensorMap* map = nullptr;
      int rc = tensor_map(h, in, r, &map);
      if (rc) return rc;
      pmap = *map;
    }
    CUdeviceptr pin = (CUdeviceptr)in, pout = (CUdeviceptr)out, paux = 0, ppart = 0;
    void* args[] = {&pmap, &pin, &pout, &psrc, &pg, &paux, &ppart};
    TCS_CU(g_drv.LaunchKernel(r.pipe->f, r.grid[0], 1, 1, r.block[0], r.block[1], 1, r.smem, st,
                              args, nullptr));
    return launch_fringe(h, r.geo, in, out, src, st);
  }
  // The TMA loader also needs a 16-byte aligned base address; otherwise copy with cp.async.
  if (geo.loader == 0 && reinterpret_cast<uintptr_t>(in) % 16 != 0) geo.loader = 1;
  alignas(64) CUtensorMap mcopy;
  std::memset(&mcopy, 0, sizeof(mcopy));
  if (geo.loader == 0) {
    CUtensorMap* map = nullptr;
    int rc = tensor_map(h, in, r, &map);
    if (rc) return rc;
    mcopy = *map;
  }
  CUdeviceptr pin = (CUdeviceptr)in, pout = (CUdeviceptr)out;
  void* args[] = {&mcopy, &pin, &pout, &psrc, &geo};
  TCS_CU(g_drv.LaunchKernel(h->f_march, r.grid[0], r.grid[1], r.grid[2], r.block[0], r.block[1],
                            r.block[2], r.smem, st, args, nullptr));
  return launch_fringe(h, r.geo, in, out, src, st);
}

}  // namespace

// =============================================================================================
extern "C" {

int tcs_abi_version(void) { return TCS_ABI_VERSION; }

void tcs_internal_set_error(const char* msg) { g_err = msg ? msg : ""; }

const char* tcs_last_error(void) { return g_err.c_str(); }

int tcs_spec_validate(const tcs_spec* spec) { return validate(spec); }

int tcs_stencil_size(const tcs_spec* spec, unsigned* stencil_size, unsigned* flops_per_update) {
  int rc = validate(spec);
  if (rc) return rc;
  const unsigned S = stencil_size_of(*spec);
  if (stencil_size) *stencil_size = S;
  if (flops_per_update) *flops_per_update = spec->coefficients == TCS_JACOBI ? S : 2 * S - 1;
  return TCS_OK;
}

int tcs_left_offset(const tcs_spec* spec, unsigned* left_offset) {
  int rc = validate(spec);
  if (rc) return rc;
  if (left_offset) *left_offset = left_offset_of(*spec);
  return TCS_OK;
}

}  // extern "C"

namespace {

// The reference's geometry (cuda/benchmark.cpp:142-179); with `ragged` the truncation of the
// interior to a coarsening multiple is skipped (threads then counts partial tiles).
int geometry_impl(const tcs_spec* spec, unsigned nx, unsigned ny, unsigned nz, bool ragged, tcs_geometry* out) {
  int rc = validate(spec);
  if (rc) return rc;
  if (!out) return fail(TCS_ERR_INVALID_VALUE, "geometry output is NULL");
  const tcs_spec& s = *spec;
  const unsigned R = (unsigned)s.range;
  const bool d3 = s.dimension == 3;
  if (nx == 0 || ny == 0 || (d3 && nz == 0))
    return fail(TCS_ERR_INVALID_VALUE, "Grid dimensions have to be greater than zero");
  if (nx < 2 * R || ny < 2 * R || (d3 && nz < 2 * R))
    return fail(TCS_ERR_INVALID_VALUE, "grid smaller than twice the stencil range");
  tcs_geometry g{};
  const unsigned c[3] = {(unsigned)s.cx, (unsigned)s.cy, d3 ? (unsigned)s.cz : 1u};
  const unsigned n[3] = {nx, ny, d3 ? nz : 1u};
  for (int i = 0; i < 3; ++i) {
    if (i == 2 && !d3) {
      g.grid[2] = 1;
      g.elements[2] = 1;
      g.threads[2] = 1;
      continue;
    }
    g.grid[i] = ragged ? n[i] : n[i] - (n[i] - 2 * R) % c[i];
    g.elements[i] = g.grid[i] - 2 * R;
    g.threads[i] = (g.elements[i] + (ragged ? c[i] - 1 : 0)) / c[i];
  }
  unsigned long long xmem = g.grid[0];
  unsigned right = 0, left = 0;
  const unsigned long long cl = (unsigned long long)s.cl_size;
  if (s.alignment == TCS_ALIGN_WRITE) {
    left = left_offset_of(s);
    xmem += left;
    if (xmem % cl != 0) right = (unsigned)(cl - xmem % cl);
    xmem += right;
  } else if (s.alignment == TCS_ALIGN_READ) {
    if (xmem % cl != 0) right = (unsigned)(cl - xmem % cl);
    xmem += right;
  }
  if (xmem > 0xffffffffull) return fail(TCS_ERR_INVALID_VALUE, "padded row exceeds 32 bits");
  g.grid[0] = (unsigned)xmem;
  g.left_offset = left;
  g.right_offset = right;
  g.n_points = (unsigned long long)g.grid[0] * g.grid[1] * g.grid[2];
  *out = g;
  return TCS_OK;
}

}  // namespace

extern "C" {

int tcs_compute_geometry(const tcs_spec* spec, unsigned nx, unsigned ny, unsigned nz, tcs_geometry* out) {
  return geometry_impl(spec, nx, ny, nz, false, out);
}

int tcs_compute_geometry_ragged(const tcs_spec* spec, unsigned nx, unsigned ny, unsigned nz, tcs_geometry* out) {
  return geometry_impl(spec, nx, ny, nz, true, out);
}

int tcs_create(const tcs_spec* spec, tcs_stencil** out) {
  int rc = validate(spec);
  if (rc) return rc;
  if (!out) return fail(TCS_ERR_INVALID_VALUE, "output handle pointer is NULL");
  rc = ensure_cuda();
  if (rc) return rc;
  std::vector<char> cubin;
  tcs_spec canon = *spec;
  if (canon.dimension == 2) canon.cz = 1;
  rc = instantiate(canon, nullptr, cubin, nullptr);
  if (rc) return rc;
  tcs_stencil* h = new tcs_stencil();
  h->spec = canon;
  h->S = stencil_size_of(h->spec);
  h->flops = h->spec.coefficients == TCS_JACOBI ? h->S : 2 * h->S - 1;
  h->left_off = left_offset_of(h->spec);
  h->mask_host.assign(h->S, 0.0);
  auto bail = [&](int code) {
    if (h->mod) g_drv.ModuleUnload(h->mod);
    delete h;
    return code;
  };
  if (cudaGetDevice(&h->device) != cudaSuccess) return bail(fail(TCS_ERR_CUDA, "cudaGetDevice"));
  cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
  cudaDeviceGetAttribute(&h->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
  CUresult cr = g_drv.ModuleLoadData(&h->mod, cubin.data());
  if (cr != CUDA_SUCCESS) return bail(fail(TCS_ERR_CUDA, "cuModuleLoadData: " + cu_msg(cr)));
  if ((cr = g_drv.ModuleGetFunction(&h->f_direct, h->mod, "tcs_direct")) != CUDA_SUCCESS ||
      (cr = g_drv.ModuleGetFunction(&h->f_march, h->mod, "tcs_march")) != CUDA_SUCCESS ||
      (cr = g_drv.ModuleGetFunction(&h->f_init, h->mod, "tcs_init")) != CUDA_SUCCESS)
    return bail(fail(TCS_ERR_CUDA, "cuModuleGetFunction: " + cu_msg(cr)));
  size_t bytes = 0;
  if ((cr = g_drv.ModuleGetGlobal(&h->mask_ptr, &h->mask_bytes, h->mod, "tcs_mask")) !=
          CUDA_SUCCESS ||
      (cr = g_drv.ModuleGetGlobal(&h->status_ptr, &bytes, h->mod, "tcs_status")) != CUDA_SUCCESS)
    return bail(fail(TCS_ERR_CUDA, "cuModuleGetGlobal: " + cu_msg(cr)));
  if (cudaMemset((void*)h->status_ptr, 0, sizeof(unsigned)) != cudaSuccess)
    return bail(fail(TCS_ERR_CUDA, "clearing the status word failed"));
  *out = h;
  return TCS_OK;
}

int tcs_destroy(tcs_stencil* h) {
  if (!h) return TCS_OK;
  if (h->fringe_mod && g_drv.ModuleUnload) g_drv.ModuleUnload(h->fringe_mod);
  if (h->tb_mod && g_drv.ModuleUnload) g_drv.ModuleUnload(h->tb_mod);
  if (h->scratch) cudaFree(h->scratch);
  if (h->tc_bops) cudaFree(h->tc_bops);
  for (PipeMod* p : h->pipes) {
    if (p->mod && g_drv.ModuleUnload) g_drv.ModuleUnload(p->mod);
    delete p;
  }
  if (h->mod && g_drv.ModuleUnload) g_drv.ModuleUnload(h->mod);
  delete h;
  return TCS_OK;
}

int tcs_get_spec(const tcs_stencil* h, tcs_spec* out) {
  if (!h || !out) return fail(TCS_ERR_INVALID_VALUE, "NULL argument");
  *out = h->spec;
  return TCS_OK;
}

int tcs_copy_mask(tcs_stencil* h, const double* mask, unsigned n) {
  if (!h) return fail(TCS_ERR_INVALID_VALUE, "NULL handle");
  if (h->spec.coefficients == TCS_JACOBI) return TCS_OK;  // reference: empty copyMask
  if (!mask && n) return fail(TCS_ERR_INVALID_VALUE, "NULL mask");
  if (n > h->S)
    return fail(TCS_ERR_INVALID_VALUE, "mask larger than the stencil (" + std::to_string(h->S) + ")");
  std::copy(mask, mask + n, h->mask_host.begin());
  h->tc_stale = true;
  int rc = upload_mask(h, h->mask_ptr);
  if (rc) return rc;
  for (PipeMod* p : h->pipes) {
    rc = upload_pipe_mask(h, p);
    if (rc) return rc;
  }
  if (h->fringe_mod && (rc = upload_mask(h, h->fringe_mask))) return rc;
  if (h->tb_mod && (rc = upload_mask(h, h->tb_mask))) return rc;
  TCS_RT(cudaDeviceSynchronize());
  return TCS_OK;
}

int tcs_max_potential_block_size(tcs_stencil* h, int* out) {
  if (!h || !out) return fail(TCS_ERR_INVALID_VALUE, "NULL argument");
  int min_grid = 0, block = 0;
  TCS_CU(g_drv.OccMaxPotential(&min_grid, &block, h->f_direct, nullptr, 0, 0));
  *out = block;
  return TCS_OK;
}

int tcs_plan_launch(tcs_stencil* h, const unsigned grid[3], unsigned right_offset,
                    const tcs_launch* launch, tcs_plan* out) {
  Resolved r;
  int rc = resolve(h, grid, right_offset, launch, r);
  if (rc) return rc;
  return fill_plan(h, r, out);
}

int tcs_update_grid(tcs_stencil* h, const unsigned grid[3], unsigned right_offset,
                    const tcs_launch* launch, const void* in, void* out, void* stream) {
  Resolved r;
  int rc = resolve(h, grid, right_offset, launch, r);
  if (rc) return rc;
  return launch_resolved(h, r, in, out, (CUstream)stream);
}

int tcs_update_grid_source(tcs_stencil* h, const unsigned grid[3], unsigned right_offset,
                           const tcs_launch* launch, const void* in, const void* src, void* out,
                           void* stream) {
  Resolved r;
  int rc = resolve(h, grid, right_offset, launch, r);
  if (rc) return rc;
  if (!src) return fail(TCS_ERR_INVALID_VALUE, "NULL source buffer");
  return launch_resolved(h, r, in, out, (CUstream)stream, src);
}

int tcs_sweeps(tcs_stencil* h, const unsigned grid[3], unsigned right_offset,
               const tcs_launch* launch, void* a, void* b, unsigned n, void* stream,
               int* result_in_b) {
  Resolved r;
  int rc = resolve(h, grid, right_offset, launch, r);
  if (rc) return rc;
  void* src = a;
  void* dst = b;
  for (unsigned i = 0; i < n; ++i) {
    rc = launch_resolved(h, r, src, dst, (CUstream)stream);
    if (rc) return rc;
    std::swap(src, dst);
  }
  if (result_in_b) *result_in_b = (n % 2 == 1) ? 1 : 0;
  return TCS_OK;
}

int tcs_time_sweeps(tcs_stencil* h, const unsigned grid[3], unsigned right_offset,
                    const tcs_launch* launch, void* a, void* b, unsigned n, void* stream,
                    float* ms) {
  Resolved r;
  int rc = resolve(h, grid, right_offset, launch, r);
  if (rc) return rc;
  cudaEvent_t e0, e1;
  TCS_RT(cudaEventCreate(&e0));
  TCS_RT(cudaEventCreate(&e1));
  cudaStream_t st = (cudaStream_t)stream;
  void* src = a;
  void* dst = b;
  cudaEventRecord(e0, st);
  for (unsigned i = 0; i < n; ++i) {
    rc = launch_resolved(h, r, src, dst, (CUstream)stream);
    if (rc) break;
    std::swap(src, dst);
  }
  cudaEventRecord(e1, st);
  cudaError_t se = cudaEventSynchronize(e1);
  float t = 0.f;
  if (rc == TCS_OK && se == cudaSuccess) cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (se != cudaSuccess) return fail(TCS_ERR_CUDA, std::string("sweeps: ") + cudaGetErrorString(se));
  if (ms) *ms = t;
  return TCS_OK;
}

int tcs_sweep_host_jobs(tcs_stencil* h, const unsigned grid[3], unsigned right_offset,
                        const tcs_launch* launch, const void* const* host_in, void* const* host_out,
                        unsigned njobs, unsigned n, void* const* dev_a, void* const* dev_b, unsigned nslots,
                        float* ms) {
  if (!h || !host_in || !host_out || !dev_a || !dev_b) return fail(TCS_ERR_INVALID_VALUE, "NULL argument");
  if (nslots < 1) return fail(TCS_ERR_INVALID_VALUE, "need at least one slot");
  for (unsigned s = 0; s < nslots; ++s)
    if (!dev_a[s] || !dev_b[s] || dev_a[s] == dev_b[s])
      return fail(TCS_ERR_INVALID_VALUE, "every slot needs two distinct device buffers");
  for (unsigned j = 0; j < njobs; ++j)
    if (!host_in[j] || !host_out[j]) return fail(TCS_ERR_INVALID_VALUE, "NULL host buffer");
  Resolved r;
  int rc = resolve(h, grid, right_offset, launch, r);
  if (rc) return rc;
  TcsGeo g;
  if ((rc = make_geo(h, grid, right_offset, g))) return rc;
  const size_t bytes = (size_t)g.xdim * g.ydim * g.zdim * (size_t)elem_size(h->spec);
  std::vector<cudaStream_t> st(nslots, nullptr);
  std::vector<cudaEvent_t> ev(nslots + 1, nullptr);  // ev[0]: start; ev[s]: slot s done (s >= 1)
  for (unsigned s = 0; s < nslots && rc == TCS_OK; ++s) {
    cudaError_t e = cudaStreamCreateWithFlags(&st[s], cudaStreamNonBlocking);
    if (e != cudaSuccess) rc = fail(TCS_ERR_CUDA, std::string("cudaStreamCreateWithFlags: ") + cudaGetErrorString(e));
  }
  for (unsigned k = 0; k <= nslots && rc == TCS_OK; ++k) {
    cudaError_t e = cudaEventCreateWithFlags(&ev[k], k == 0 ? cudaEventDefault : cudaEventDisableTiming);
    if (e != cudaSuccess) rc = fail(TCS_ERR_CUDA, std::string("cudaEventCreate: ") + cudaGetErrorString(e));
  }
  cudaEvent_t end = nullptr;
  if (rc == TCS_OK && cudaEventCreate(&end) != cudaSuccess) rc = fail(TCS_ERR_CUDA, "cudaEventCreate failed");
  // Device-side timing across the slots: every slot stream starts after ev[0] on slot 0, and slot 0
  // records `end` after waiting for every other slot's last download.
  if (rc == TCS_OK) {
    cudaEventRecord(ev[0], st[0]);
    for (unsigned s = 1; s < nslots; ++s) cudaStreamWaitEvent(st[s], ev[0], 0);
  }
  // Job j runs on slot j % nslots: upload, the border copy into b (the ping-pong invariant), n
  // sweeps, download -- all ordered on the slot's stream, so the slot's buffers are reused only
  // after its previous job's download has been issued behind them.
  for (unsigned j = 0; j < njobs && rc == TCS_OK; ++j) {
    const unsigned s = j % nslots;
    cudaError_t e = cudaMemcpyAsync(dev_a[s], host_in[j], bytes, cudaMemcpyHostToDevice, st[s]);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dev_b[s], dev_a[s], bytes, cudaMemcpyDeviceToDevice, st[s]);
    if (e != cudaSuccess) {
      rc = fail(TCS_ERR_CUDA, std::string("host job upload: ") + cudaGetErrorString(e));
      break;
    }
    void* src = dev_a[s];
    void* dst = dev_b[s];
    for (unsigned i = 0; i < n && rc == TCS_OK; ++i) {
      rc = launch_resolved(h, r, src, dst, (CUstream)st[s]);
      std::swap(src, dst);
    }
    if (rc) break;
    e = cudaMemcpyAsync(host_out[j], src, bytes, cudaMemcpyDeviceToHost, st[s]);
    if (e != cudaSuccess) rc = fail(TCS_ERR_CUDA, std::string("host job download: ") + cudaGetErrorString(e));
  }
  if (end && st[0]) {
    for (unsigned s = 1; s < nslots; ++s) {
      if (!st[s] || !ev[s]) continue;
      cudaEventRecord(ev[s], st[s]);
      cudaStreamWaitEvent(st[0], ev[s], 0);
    }
    cudaEventRecord(end, st[0]);
  }
  for (unsigned s = 0; s < nslots; ++s) {
    if (!st[s]) continue;
    cudaError_t e = cudaStreamSynchronize(st[s]);
    if (e != cudaSuccess && rc == TCS_OK) rc = fail(TCS_ERR_CUDA, std::string("host jobs: ") + cudaGetErrorString(e));
  }
  if (rc == TCS_OK && ms) {
    float t = 0.f;
    cudaError_t e = cudaEventElapsedTime(&t, ev[0], end);
    if (e != cudaSuccess) rc = fail(TCS_ERR_CUDA, std::string("host jobs timing: ") + cudaGetErrorString(e));
    *ms = t;
  }
  for (unsigned s = 0; s < nslots; ++s)
    if (st[s]) cudaStreamDestroy(st[s]);
  for (cudaEvent_t e : ev)
    if (e) cudaEventDestroy(e);
  if (end) cudaEventDestroy(end);
  return rc;
}

int tcs_benchmark_update_grid(tcs_stencil* h, const char* coeff_type, const char* neighbourhood,
                              unsigned stencil_range, unsigned dimension, const char* alignment,
                              double max_time, const unsigned grid[3], const unsigned block[3],
                              const unsigned grid_blocks[3], void* d_array0, void* d_array1,
                              unsigned right_offset, double* durations, unsigned cap,
                              unsigned* n_out) {
  if (!h) return fail(TCS_ERR_INVALID_VALUE, "NULL handle");
  // runtime sanity check against the baked-in parameters (generateLaunchUpdateGrid.py:106-119)
  const tcs_spec& s = h->spec;
  bool passed = true;
  if (!coeff_type || std::strcmp(coeff_type, coeff_str(s.coefficients)) != 0) passed = false;
  if (!neighbourhood || std::strcmp(neighbourhood, shape_str(s.neighbourhood)) != 0) passed = false;
  if (stencil_range != (unsigned)s.range) passed = false;
  if (dimension != (unsigned)s.dimension) passed = false;
  if (!alignment || std::strcmp(alignment, align_str(s.alignment)) != 0) passed = false;
  if (!passed)
    return fail(TCS_ERR_INVALID_VALUE,
                "benchmarkUpdateGrid: runtime parameters do not match the instantiated kernel");
  if (max_time < 0) return fail(TCS_ERR_INVALID_VALUE, "maxTime must be non-negative");
  tcs_launch L{};
  for (int i = 0; i < 3; ++i) {
    L.block[i] = block ? block[i] : 0;
    L.grid_blocks[i] = grid_blocks ? grid_blocks[i] : 0;
  }
  L.variant = h->dropin_variant;
  L.segments = h->dropin_segments;
  L.depth = h->dropin_depth;
  Resolved r;
  int rc = resolve(h, grid, right_offset, &L, r);
  if (rc) return rc;
  using clock = std::chrono::steady_clock;
  std::vector<clock::time_point> ts;
  ts.reserve(1024);
  ts.push_back(clock::now());
  double runtime = 0.0;
  void* a0 = d_array0;
  void* a1 = d_array1;
  for (unsigned long long it = 1; runtime <= max_time; it *= 2) {
    for (unsigned long long i = 0; i < it; ++i) {
      rc = launch_resolved(h, r, a0, a1, nullptr);
      if (rc) return rc;
      TCS_RT(cudaDeviceSynchronize());
      std::swap(a0, a1);
      ts.push_back(clock::now());
    }
    runtime = std::chrono::duration<double>(ts.back() - ts.front()).count();
  }
  const unsigned n = (unsigned)(ts.size() - 1);
  h->last_durations.resize(n);
  for (unsigned i = 0; i < n; ++i) h->last_durations[i] = std::chrono::duration<double>(ts[i + 1] - ts[i]).count();
  for (unsigned i = 0; i < n && i < cap && durations; ++i) durations[i] = h->last_durations[i];
  if (n_out) *n_out = n;
  return TCS_OK;
}

int tcs_benchmark_durations(tcs_stencil* h, double* durations, unsigned cap, unsigned* n_out) {
  if (!h || !n_out) return fail(TCS_ERR_INVALID_VALUE, "NULL argument");
  const unsigned n = (unsigned)h->last_durations.size();
  for (unsigned i = 0; i < n && i < cap && durations; ++i) durations[i] = h->last_durations[i];
  *n_out = n;
  return TCS_OK;
}

int tcs_launch_init(tcs_stencil* h, const unsigned grid[3], const unsigned block[3],
                    const unsigned grid_blocks[3], void* d_array, unsigned right_offset) {
  if (!h || !grid || !block || !grid_blocks || !d_array)
    return fail(TCS_ERR_INVALID_VALUE, "NULL argument");
  const tcs_spec& s = h->spec;
  unsigned long long xdim = grid[0], ydim = grid[1], zdim = s.dimension == 3 ? grid[2] : 1;
  unsigned x_shift = h->left_off;
  unsigned long long x_end = (s.alignment == TCS_ALIGN_NONE) ? xdim : xdim - right_offset;
  CUdeviceptr p = (CUdeviceptr)d_array;
  void* args[] = {&p, &xdim, &ydim, &zdim, &x_shift, &x_end};
  TCS_CU(g_drv.LaunchKernel(h->f_init, grid_blocks[0], grid_blocks[1], grid_blocks[2], block[0],
                            block[1], block[2], 0, nullptr, args, nullptr));
  TCS_RT(cudaDeviceSynchronize());
  return TCS_OK;
}

int tcs_device_status(tcs_stencil* h, unsigned* status, int clear) {
  if (!h) return fail(TCS_ERR_INVALID_VALUE, "NULL handle");
  unsigned v = 0, w = 0;
  TCS_RT(cudaMemcpy(&v, (void*)h->status_ptr, sizeof(v), cudaMemcpyDeviceToHost));
  if (clear) TCS_RT(cudaMemset((void*)h->status_ptr, 0, sizeof(unsigned)));
  for (PipeMod* p : h->pipes) {
    TCS_RT(cudaMemcpy(&w, (void*)p->status_ptr, sizeof(w), cudaMemcpyDeviceToHost));
    if (clear) TCS_RT(cudaMemset((void*)p->status_ptr, 0, sizeof(unsigned)));
    v |= w;
  }
  if (status) *status = v;
  return TCS_OK;
}

int tcs_self_test_wait(tcs_stencil* h, long long cycles) {
  if (!h) return fail(TCS_ERR_INVALID_VALUE, "NULL handle");
  if (cycles < 1000 || cycles > 4000000000LL)
    return fail(TCS_ERR_INVALID_VALUE, "self-test wait budget outside [1e3, 4e9] cycles");
  int e = tcs_field_launch_wait_probe(reinterpret_cast<unsigned*>(h->status_ptr), cycles, nullptr);
  if (e != 0) return fail(TCS_ERR_CUDA, std::string("wait probe launch: ") + cudaGetErrorString((cudaError_t)e));
  TCS_RT(cudaDeviceSynchronize());
  unsigned v = 0;
  TCS_RT(cudaMemcpy(&v, (void*)h->status_ptr, sizeof(v), cudaMemcpyDeviceToHost));
  TCS_RT(cudaMemset((void*)h->status_ptr, 0, sizeof(unsigned)));
  if (v & 1u) return fail(TCS_ERR_DEVICE_TIMEOUT, "bounded device wait expired (self-test)");
  return TCS_OK;
}

int tcs_set_dropin_launch(tcs_stencil* h, int variant, unsigned segments, unsigned depth) {
  if (!h) return fail(TCS_ERR_INVALID_VALUE, "NULL handle");
  if (variant != TCS_VARIANT_AUTO && variant != TCS_VARIANT_DIRECT && variant != TCS_VARIANT_MARCH)
    return fail(TCS_ERR_INVALID_VALUE, "unknown variant");
  h->dropin_variant = variant;
  h->dropin_segments = segments;
  h->dropin_depth = depth;
  return TCS_OK;
}

int tcs_precompile(const tcs_spec* spec, char* cubin_path, unsigned path_cap) {
  int rc = validate(spec);
  if (rc) return rc;
  tcs_spec s = *spec;
  if (s.dimension == 2) s.cz = 1;
  std::vector<char> cubin;
  std::string path;
  rc = instantiate(s, nullptr, cubin, &path);
  if (rc) return rc;
  if (cubin_path && path_cap) {
    std::strncpy(cubin_path, path.c_str(), path_cap - 1);
    cubin_path[path_cap - 1] = '\0';
  }
  return TCS_OK;
}

}  // extern "C"

namespace {

int precompile_pipe(const tcs_spec* spec, unsigned bx, unsigned by, unsigned chunk, bool batch,
                    char* cubin_path, unsigned path_cap, unsigned epi = 0, unsigned shfl = 0, unsigned tmem = 0) {
  int rc = validate(spec);
  if (rc) return rc;
  tcs_spec s = *spec;
  if (s.dimension == 2) s.cz = 1;
  if (s.dimension == 2 && s.orientation == TCS_COLUMN)
    return fail(TCS_ERR_UNSUPPORTED, "2D Column orientation is not pipelined");
  if (s.precision == TCS_F32C && !pipe_comp_ok(s))
    return fail(TCS_ERR_UNSUPPORTED, "compensated FP32 pipelined sweeps need the packed Box path");
  const unsigned vec = 16u / (unsigned)elem_size(s);
  if (bx == 0 || (bx * (unsigned)s.cx) % vec != 0)
    return fail(TCS_ERR_UNSUPPORTED, "pipe: unsupported block");
  if (chunk == 0) chunk = pipe_auto_chunk(s, bx, by);
  if (epi > 2 || (epi == 1 && s.precision != TCS_F64) || (epi == 2 && s.precision != TCS_F32) || (epi && batch))
    return fail(TCS_ERR_UNSUPPORTED, "pipe: epilogue not available for this precision");
  if (shfl && !(s.neighbourhood == TCS_STAR && (s.dimension == 2 || s.orientation == TCS_ROW) && bx % 32 == 0))
    return fail(TCS_ERR_UNSUPPORTED, "pipe: shuffled rows need a Star stencil in Row order and bx % 32 == 0");
  if (tmem && (tmem_cols(s, bx, s.dimension == 3 ? by : 1u) == 0 || batch || epi || shfl))
    return fail(TCS_ERR_UNSUPPORTED, "pipe: the tensor-memory ring form does not apply to this instance");
  PipeKey key{bx, s.dimension == 3 ? by : 1u, chunk, left_offset_of(s) % vec, batch ? 1u : 0u, epi, 0u, shfl ? 1u : 0u,
              tmem ? 1u : 0u};
  std::vector<char> cubin;
  std::string path;
  rc = instantiate(s, &key, cubin, &path);
  if (rc) return rc;
  if (cubin_path && path_cap) {
    std::strncpy(cubin_path, path.c_str(), path_cap - 1);
    cubin_path[path_cap - 1] = '\0';
  }
  return TCS_OK;
}

// Interior box of a buffer with the reference geometry (gridSize, rightOffset).
int field_geo(const tcs_stencil* h, const unsigned grid[3], unsigned right_offset, TcsFieldGeo& f) {
  TcsGeo g;
  int rc = make_geo(h, grid, right_offset, g);
  if (rc) return rc;
  const unsigned R = (unsigned)h->spec.range;
  f.xdim = g.xdim;
  f.ydim = g.ydim;
  f.x0 = g.x0;
  f.x_lim = g.x_lim;
  f.y0 = R;
  f.y_lim = g.y_lim;
  f.z0 = h->spec.dimension == 3 ? R : 0;
  f.z_lim = g.z_lim;
  return TCS_OK;
}

int field_blocks(const tcs_stencil* h) { return 2 * std::max(1, h->num_sms); }

// Scratch of the two-pass reductions: nblocks*4 partials + 8 result slots, allocated once.
int ensure_scratch(tcs_stencil* h, size_t need) {
  std::lock_guard<std::mutex> lock(h->mu);
  if (h->scratch_len >= need) return TCS_OK;
  if (h->scratch) cudaFree(h->scratch);
  h->scratch = nullptr;
  h->scratch_len = 0;
  TCS_RT(cudaMalloc(&h->scratch, need * sizeof(double)));
  h->scratch_len = need;
  return TCS_OK;
}

// The residual entry points launch on the calling thread's current device: it must be the device
// the handle (and the buffers) belong to.
int check_current_device(const tcs_stencil* h) {
  int dev = -1;
  TCS_RT(cudaGetDevice(&dev));
  if (dev != h->device)
    return fail(TCS_ERR_INVALID_VALUE, "current device " + std::to_string(dev) + " is not the handle's device " +
                                           std::to_string(h->device));
  return TCS_OK;
}

}  // namespace

extern "C" {

int tcs_precompile_pipe(const tcs_spec* spec, unsigned bx, unsigned by, unsigned chunk,
                        char* cubin_path, unsigned path_cap) {
  return precompile_pipe(spec, bx, by, chunk, false, cubin_path, path_cap);
}

int tcs_precompile_pipe_epilogue(const tcs_spec* spec, unsigned bx, unsigned by, unsigned chunk, unsigned epi,
                                 char* cubin_path, unsigned path_cap) {
  return precompile_pipe(spec, bx, by, chunk, false, cubin_path, path_cap, epi);
}

int tcs_precompile_pipe_flags(const tcs_spec* spec, unsigned bx, unsigned by, unsigned chunk, unsigned flags,
                              char* cubin_path, unsigned path_cap) {
  return precompile_pipe(spec, bx, by, chunk, false, cubin_path, path_cap, 0, (flags & TCS_LAUNCH_SHUFFLE) ? 1u : 0u,
                         (flags & TCS_LAUNCH_TMEM) ? 1u : 0u);
}

int tcs_precompile_batch(const tcs_spec* spec, unsigned bx, unsigned by, unsigned chunk,
                         char* cubin_path, unsigned path_cap) {
  return precompile_pipe(spec, bx, by, chunk, true, cubin_path, path_cap);
}

int tcs_residual(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, const double* x,
                 const double* sx, float* r, double norms[2], void* stream) {
  if (!h || !x || !sx || !r) return fail(TCS_ERR_INVALID_VALUE, "NULL argument");
  int rc = check_current_device(h);
  if (rc) return rc;
  TcsFieldGeo f;
  rc = field_geo(h, grid, right_offset, f);
  if (rc) return rc;
  const int nb = field_blocks(h);
  rc = ensure_scratch(h, (size_t)nb * 4 + 8);
  if (rc) return rc;
  double* res = h->scratch + (size_t)nb * 4;
  const int e = tcs_field_launch_defect(x, sx, r, f, h->scratch, nb, res, (cudaStream_t)stream);
  if (e != 0) return fail(TCS_ERR_CUDA, std::string("defect kernel: ") + cudaGetErrorString((cudaError_t)e));
  if (norms) {
    double host[2];
    TCS_RT(cudaMemcpyAsync(host, res, sizeof(host), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    TCS_RT(cudaStreamSynchronize((cudaStream_t)stream));
    norms[0] = host[0];
    norms[1] = std::sqrt(host[1]);
  }
  return TCS_OK;
}

int tcs_residual_static(tcs_stencil* h, const unsigned grid[3], unsigned right_offset,
                        const double* x, const double* sx, float* r, double norms[2],
                        unsigned nblocks, void* stream) {
  if (!h || !x || !sx || !r) return fail(TCS_ERR_INVALID_VALUE, "NULL argument");
  int rc = check_current_device(h);
  if (rc) return rc;
  TcsFieldGeo f;
  rc = field_geo(h, grid, right_offset, f);
  if (rc) return rc;
  const unsigned nb = nblocks ? nblocks : (unsigned)field_blocks(h);
  const unsigned long long need = 2ull * nb + 2ull;  // two partials per block + two results
  if (need > TCS_STATIC_SCRATCH_DOUBLES)
    return fail(TCS_ERR_INVALID_VALUE,
                "tcs_residual_static: " + std::to_string(nb) + " blocks need " + std::to_string(need) +
                    " doubles of scratch; the static array holds " +
                    std::to_string(TCS_STATIC_SCRATCH_DOUBLES) + " (at most " +
                    std::to_string((TCS_STATIC_SCRATCH_DOUBLES - 2) / 2) + " blocks)");
  // The array's address belongs to the module image loaded into the current context; a context
  // recreated after cudaDeviceReset may place it elsewhere, so the cached address is keyed by the
  // context's unique id.
  CUcontext ctx = nullptr;
  TCS_CU(g_drv.CtxGetCurrent(&ctx));
  if (!ctx) return fail(TCS_ERR_CUDA, "tcs_residual_static: no current CUDA context");
  unsigned long long ctx_id = 0;
  TCS_CU(g_drv.CtxGetId(ctx, &ctx_id));
  double* scratch = nullptr;
  const int se = tcs_field_static_scratch(ctx_id, &scratch);
  if (se != 0)
    return fail(TCS_ERR_CUDA, std::string("static scratch address: ") + cudaGetErrorString((cudaError_t)se));
  double* res = scratch + 2ull * nb;
  const int e = tcs_field_launch_defect(x, sx, r, f, scratch, (int)nb, res, (cudaStream_t)stream);
  if (e != 0) return fail(TCS_ERR_CUDA, std::string("defect kernel: ") + cudaGetErrorString((cudaError_t)e));
  if (norms) {
    double host[2];
    TCS_RT(cudaMemcpyAsync(host, res, sizeof(host), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    TCS_RT(cudaStreamSynchronize((cudaStream_t)stream));
    norms[0] = host[0];
    norms[1] = std::sqrt(host[1]);
  }
  return TCS_OK;
}

int tcs_scratch_bytes(tcs_stencil* h, unsigned long long* bytes) {
  if (!h || !bytes) return fail(TCS_ERR_INVALID_VALUE, "NULL argument");
  *bytes = (unsigned long long)h->scratch_len * sizeof(double);
  return TCS_OK;
}

// ---- fused defect-correction sweeps (pipe kernel epilogues 1 and 2) ---------------------------
}  // extern "C"

namespace {

// Resolve a launch of the pipelined kernel with epilogue `epi`; the fused sweeps run on the pipe
// kernel only and on geometries without a coarsening fringe.
int resolve_epi(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, const tcs_launch* launch,
                unsigned epi, Resolved& r) {
  if (!h || !launch) return fail(TCS_ERR_INVALID_VALUE, "NULL handle or launch");
  int rc = check_current_device(h);
  if (rc) return rc;
  TcsGeo g;
  rc = make_geo(h, grid, right_offset, g);
  if (rc) return rc;
  rc = check_block(h, launch->block);
  if (rc) return rc;
  if (launch->variant != TCS_VARIANT_AUTO && launch->variant != TCS_VARIANT_PIPE)
    return fail(TCS_ERR_UNSUPPORTED, "fused defect-correction sweeps run on the pipelined kernel");
  if (has_fringe(h, g))
    return fail(TCS_ERR_UNSUPPORTED, "fused defect-correction sweeps need a grid of whole coarsening tiles");
  return resolve_pipe(h, g, launch, r, false, epi);
}

int launch_epi(tcs_stencil* h, const Resolved& r, const void* in, const void* src, void* aux, double* partials,
               CUstream st) {
  TcsPipeGeo pg = r.pgeo;
  pg.loader = r.no_tma ? pipe_loader_cp(h->spec, pg.xdim, in) : pipe_loader(h->spec, pg.xdim, in);
  alignas(64) CUtensorMap pmap;
  std::memset(&pmap, 0, sizeof(pmap));
  if (pg.loader == 0) {
    CUtensorMap* map = nullptr;
    int rc = tensor_map(h, in, r, &map);
    if (rc) return rc;
    pmap = *map;
  }
  // `out` only anchors the kernel's output offsets: epilogues 1 and 2 store through `aux`
  CUdeviceptr pin = (CUdeviceptr)in, pout = (CUdeviceptr)in, psrc = (CUdeviceptr)src, paux = (CUdeviceptr)aux,
              ppart = (CUdeviceptr)partials;
  void* args[] = {&pmap, &pin, &pout, &psrc, &pg, &paux, &ppart};
  TCS_CU(g_drv.LaunchKernel(r.pipe->f, r.grid[0], 1, 1, r.block[0], r.block[1], 1, r.smem, st, args, nullptr));
  return TCS_OK;
}

}  // namespace

extern "C" {

int tcs_defect_sweep(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, const tcs_launch* launch,
                     const void* x, float* r, double norms[2], void* stream) {
  if (!h || !x || !r) return fail(TCS_ERR_INVALID_VALUE, "NULL argument");
  if (h->spec.precision != TCS_F64) return fail(TCS_ERR_INVALID_VALUE, "the defect sweep needs an FP64 handle");
  Resolved rs;
  int rc = resolve_epi(h, grid, right_offset, launch, 1, rs);
  if (rc) return rc;
  const unsigned nb = rs.grid[0];
  rc = ensure_scratch(h, 2ull * nb + 8);
  if (rc) return rc;
  double* res = h->scratch + 2ull * nb;
  rc = launch_epi(h, rs, x, x, r, h->scratch, (CUstream)stream);
  if (rc) return rc;
  const int e = tcs_field_launch_finish(h->scratch, (int)nb, 2, 1u, res, (cudaStream_t)stream);
  if (e != 0) return fail(TCS_ERR_CUDA, std::string("finish kernel: ") + cudaGetErrorString((cudaError_t)e));
  if (norms) {
    double host[2];
    TCS_RT(cudaMemcpyAsync(host, res, sizeof(host), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    TCS_RT(cudaStreamSynchronize((cudaStream_t)stream));
    norms[0] = host[0];
    norms[1] = std::sqrt(host[1]);
  }
  return TCS_OK;
}

int tcs_update_grid_accumulate(tcs_stencil* h, const unsigned grid[3], unsigned right_offset,
                               const tcs_launch* launch, const void* in, const void* src, double* x,
                               void* stream) {
  if (!h || !in || !x) return fail(TCS_ERR_INVALID_VALUE, "NULL argument");
  if (h->spec.precision != TCS_F32) return fail(TCS_ERR_INVALID_VALUE, "the accumulating sweep needs an FP32 handle");
  Resolved rs;
  int rc = resolve_epi(h, grid, right_offset, launch, 2, rs);
  if (rc) return rc;
  return launch_epi(h, rs, in, src, x, nullptr, (CUstream)stream);
}

int tcs_accumulate(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, double* x,
                   const float* e, void* stream) {
  if (!h || !x || !e) return fail(TCS_ERR_INVALID_VALUE, "NULL argument");
  TcsFieldGeo f;
  int rc = field_geo(h, grid, right_offset, f);
  if (rc) return rc;
  const int err = tcs_field_launch_add(x, e, f, field_blocks(h), (cudaStream_t)stream);
  if (err != 0) return fail(TCS_ERR_CUDA, std::string("add kernel: ") + cudaGetErrorString((cudaError_t)err));
  return TCS_OK;
}

int tcs_compare(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, const void* a,
                int a_precision, const double* b, double stats[4], void* stream) {
  if (!h || !a || !b || !stats) return fail(TCS_ERR_INVALID_VALUE, "NULL argument");
  if (a_precision != TCS_F64 && a_precision != TCS_F32)
    return fail(TCS_ERR_INVALID_VALUE, "unknown precision");
  TcsFieldGeo f;
  int rc = field_geo(h, grid, right_offset, f);
  if (rc) return rc;
  const int nb = field_blocks(h);
  rc = ensure_scratch(h, (size_t)nb * 4 + 8);
  if (rc) return rc;
  double* res = h->scratch + (size_t)nb * 4;
  const int e = tcs_field_launch_compare(a, a_precision == TCS_F32 ? 1 : 0, b, f, h->scratch, nb, res,
                                         (cudaStream_t)stream);
  if (e != 0) return fail(TCS_ERR_CUDA, std::string("compare kernel: ") + cudaGetErrorString((cudaError_t)e));
  double host[4];
  TCS_RT(cudaMemcpyAsync(host, res, sizeof(host), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  TCS_RT(cudaStreamSynchronize((cudaStream_t)stream));
  stats[0] = host[0];
  stats[1] = std::sqrt(host[1]);
  stats[2] = host[2];
  stats[3] = std::sqrt(host[3]);
  return TCS_OK;
}

int tcs_device_sm_count(int* out) {
  int rc = ensure_cuda();
  if (rc) return rc;
  int dev = 0;
  TCS_RT(cudaGetDevice(&dev));
  TCS_RT(cudaDeviceGetAttribute(out, cudaDevAttrMultiProcessorCount, dev));
  return TCS_OK;
}

}  // extern "C"

// =============================================================================================
// Batched sweeps: many grids of one parameter set in one persistent launch (tcs_pipe_batch).

// Host mirror of the device TcsBatchGrid (same layout: tensor map, then pointers and geometry).
struct alignas(64) TcsBatchGrid {
  CUtensorMap map;
  const void* in;
  void* out;
  const void* src;
  unsigned long long xdim, ydim, zdim;
  unsigned long long first;
  unsigned x0, x_lim, y_lim, z_lim;
  unsigned ntx, m;
  unsigned loader;
  unsigned pad_;
};
static_assert(sizeof(TcsBatchGrid) == 256, "TcsBatchGrid layout");
static_assert(offsetof(TcsBatchGrid, in) == 128 && offsetof(TcsBatchGrid, first) == 176 &&
                  offsetof(TcsBatchGrid, loader) == 208,
              "TcsBatchGrid layout");

struct tcs_batch {
  tcs_stencil* h = nullptr;
  tcs_launch launch{};
  unsigned n = 0;
  std::vector<unsigned> dims;           // 3 per grid
  std::vector<unsigned> right_offsets;  // 1 per grid
  std::vector<void*> a, b;              // the two buffers of each grid
  PipeMod* pm = nullptr;
  unsigned smem = 0, nslot = 0, depth = 0, chunk = 0, width = 0, occ = 0, block[2] = {1, 1};
  unsigned nctas = 0;
  unsigned long long total = 0, per = 0;
  unsigned tma_grids[2] = {0, 0};       // grids loaded by TMA in each direction
  CUdeviceptr table[2] = {0, 0};        // grid tables: a -> b, b -> a
  std::vector<Resolved> single;         // per-grid single-grid launches (filled on first use)
  std::vector<CUtensorMap> maps[2];     // per-grid tensor maps of the input, per direction
  std::vector<TcsGeo> ragged;           // grids whose interior is not a coarsening multiple
  std::vector<unsigned> ragged_ids;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

void batch_free(tcs_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (CUdeviceptr t : b->table)
    if (t) cudaFree((void*)t);
  delete b;
}

int batch_launch(tcs_batch* b, int from_b, CUstream st) {
  CUdeviceptr table = b->table[from_b ? 1 : 0];
  unsigned ngrids = b->n, nslot = b->nslot;
  unsigned long long total = b->total, per = b->per;
  void* args[] = {&table, &ngrids, &total, &per, &nslot};
  TCS_CU(g_drv.LaunchKernel(b->pm->f, b->nctas, 1, 1, b->block[0], b->block[1], 1, b->smem, st, args,
                            nullptr));
  for (size_t k = 0; k < b->ragged.size(); ++k) {  // partial coarsening tiles of ragged grids
    const unsigned i = b->ragged_ids[k];
    int rc = launch_fringe(b->h, b->ragged[k], from_b ? b->b[i] : b->a[i], from_b ? b->a[i] : b->b[i], nullptr, st);
    if (rc) return rc;
  }
  return TCS_OK;
}

int batch_single(tcs_batch* b) {
  if (!b->single.empty()) return TCS_OK;
  std::vector<Resolved> rs(b->n);
  for (unsigned i = 0; i < b->n; ++i) {
    TcsGeo g;
    int rc = make_geo(b->h, &b->dims[3 * i], b->right_offsets[i], g);
    if (rc) return rc;
    tcs_launch L = b->launch;
    L.segments = 0;  // each grid spreads over the whole device
    rc = resolve_pipe(b->h, g, &L, rs[i], false);
    if (rc) return rc;
  }
  b->single.swap(rs);
  return TCS_OK;
}

int batch_launch_separate(tcs_batch* b, int from_b, CUstream st) {
  int rc = batch_single(b);
  if (rc) return rc;
  for (unsigned i = 0; i < b->n; ++i) {
    const void* in = from_b ? b->b[i] : b->a[i];
    void* out = from_b ? b->a[i] : b->b[i];
    rc = launch_resolved(b->h, b->single[i], in, out, st, nullptr, &b->maps[from_b ? 1 : 0][i]);
    if (rc) return rc;
  }
  return TCS_OK;
}

}  // namespace

extern "C" {

int tcs_batch_create(tcs_stencil* h, unsigned ngrids, const unsigned* grids,
                     const unsigned* right_offsets, const tcs_launch* launch, void* const* a,
                     void* const* b, tcs_batch** out) {
  if (!h || !grids || !launch || !a || !b || !out)
    return fail(TCS_ERR_INVALID_VALUE, "NULL argument");
  *out = nullptr;
  if (ngrids == 0) return fail(TCS_ERR_INVALID_VALUE, "a batch needs at least one grid");
  if (launch->variant != TCS_VARIANT_AUTO && launch->variant != TCS_VARIANT_PIPE)
    return fail(TCS_ERR_UNSUPPORTED, "batched sweeps run the pipe kernel only");
  int rc = check_block(h, launch->block);
  if (rc) return rc;
  const tcs_spec& s = h->spec;
  tcs_batch* B = new tcs_batch();
  B->h = h;
  B->launch = *launch;
  B->launch.variant = TCS_VARIANT_PIPE;
  B->n = ngrids;
  B->dims.assign(grids, grids + 3 * (size_t)ngrids);
  B->right_offsets.assign(ngrids, 0u);
  if (right_offsets) B->right_offsets.assign(right_offsets, right_offsets + ngrids);
  B->a.assign(a, a + ngrids);
  B->b.assign(b, b + ngrids);
  std::vector<TcsBatchGrid> tab[2];
  tab[0].resize(ngrids);
  tab[1].resize(ngrids);
  B->maps[0].resize(ngrids);
  B->maps[1].resize(ngrids);
  unsigned long long first = 0;
  for (unsigned i = 0; i < ngrids; ++i) {
    if (!a[i] || !b[i] || a[i] == b[i]) {
      batch_free(B);
      return fail(TCS_ERR_INVALID_VALUE, "grid " + std::to_string(i) + ": NULL or shared buffers");
    }
    TcsGeo g;
    Resolved r;
    if ((rc = make_geo(h, &B->dims[3 * i], B->right_offsets[i], g)) ||
        (rc = resolve_pipe(h, g, &B->launch, r, true))) {
      batch_free(B);
      g_err = "grid " + std::to_string(i) + ": " + g_err;
      return rc;
    }
    if (i == 0) {
      B->pm = r.pipe;
      B->smem = r.smem;
      B->nslot = r.pgeo.nslot;
      B->depth = r.depth;
      B->chunk = r.chunk;
      B->width = r.geo.width;
      B->occ = r.occ;
      B->block[0] = r.block[0];
      B->block[1] = r.block[1];
    }
    const TcsPipeGeo& pg = r.pgeo;
    {
      const unsigned cz = s.dimension == 3 ? (unsigned)s.cz : 1u;
      const bool rx = (g.x_lim - g.x0) % (unsigned)s.cx != 0, ry = (g.y_lim - (unsigned)s.range) % (unsigned)s.cy != 0;
      const bool rz = s.dimension == 3 && (g.z_lim - (unsigned)s.range) % cz != 0;
      if (rx || ry || rz) {
        B->ragged.push_back(g);
        B->ragged_ids.push_back(i);
      }
    }
    for (int d = 0; d < 2; ++d) {
      TcsBatchGrid& e = tab[d][i];
      std::memset(&e, 0, sizeof(e));
      e.in = d ? b[i] : a[i];
      e.out = d ? a[i] : b[i];
      e.src = nullptr;
      e.xdim = pg.xdim;
      e.ydim = pg.ydim;
      e.zdim = pg.zdim;
      e.first = first;
      e.x0 = pg.x0;
      e.x_lim = pg.x_lim;
      e.y_lim = pg.y_lim;
      e.z_lim = pg.z_lim;
      e.ntx = pg.ntx;
      e.m = pg.m;
      // TMA needs a 16-byte row pitch and base; other grids stream through cp.async.
      e.loader = pipe_loader(s, pg.xdim, e.in);
      if (e.loader == 0) {
        const unsigned long long dims[3] = {pg.xdim, pg.ydim, pg.zdim};
        if ((rc = encode_map(s, e.in, dims, r.box, &e.map))) {
          batch_free(B);
          return rc;
        }
        ++B->tma_grids[d];
      }
      B->maps[d][i] = e.map;
    }
    first += pg.total;
  }
  B->total = first;
  unsigned long long nctas = (unsigned long long)h->num_sms * B->occ;
  if (launch->segments) nctas = launch->segments;
  B->per = std::max<unsigned long long>(1, (B->total + nctas - 1) / nctas);
  const unsigned long long grid = std::max<unsigned long long>(1, (B->total + B->per - 1) / B->per);
  if (grid > 0x7fffffffull) {
    batch_free(B);
    return fail(TCS_ERR_UNSUPPORTED, "batch grid too large");
  }
  B->nctas = (unsigned)grid;
  for (int d = 0; d < 2; ++d) {
    cudaError_t e = cudaMalloc((void**)&B->table[d], sizeof(TcsBatchGrid) * ngrids);
    if (e == cudaSuccess)
      e = cudaMemcpy((void*)B->table[d], tab[d].data(), sizeof(TcsBatchGrid) * ngrids,
                     cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      batch_free(B);
      return fail(TCS_ERR_CUDA, std::string("batch table: ") + cudaGetErrorString(e));
    }
  }
  *out = B;
  return TCS_OK;
}

int tcs_batch_plan(const tcs_batch* b, tcs_plan* out) {
  if (!b || !out) return fail(TCS_ERR_INVALID_VALUE, "NULL argument");
  tcs_plan p{};
  p.variant = TCS_VARIANT_PIPE;
  p.grid_blocks[0] = b->nctas;
  p.grid_blocks[1] = p.grid_blocks[2] = 1;
  p.block[0] = b->block[0];
  p.block[1] = b->block[1];
  p.block[2] = 1;
  p.dyn_smem = b->smem;
  p.seg_len = (unsigned)std::min<unsigned long long>(b->per, 0xffffffffull);
  p.nslot = b->nslot;
  p.width = b->width;
  p.chunk = b->chunk;
  p.depth = b->depth;
  p.loader = (b->tma_grids[0] == b->n) ? 0u : 1u;
  p.ctas_per_sm = b->occ;
  p.num_sms = b->h->num_sms;
  *out = p;
  return TCS_OK;
}

int tcs_batch_sweep(tcs_batch* b, int from_b, void* stream) {
  if (!b) return fail(TCS_ERR_INVALID_VALUE, "NULL batch");
  return batch_launch(b, from_b, (CUstream)stream);
}

int tcs_batch_sweep_separate(tcs_batch* b, int from_b, void* stream) {
  if (!b) return fail(TCS_ERR_INVALID_VALUE, "NULL batch");
  return batch_launch_separate(b, from_b, (CUstream)stream);
}

int tcs_batch_graph(tcs_batch* b, unsigned n, int separate) {
  if (!b) return fail(TCS_ERR_INVALID_VALUE, "NULL batch");
  if (n == 0) return fail(TCS_ERR_INVALID_VALUE, "a graph needs at least one sweep");
  int rc = separate ? batch_single(b) : TCS_OK;  // module loads and uploads happen before capture
  if (rc) return rc;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  cudaStream_t cs;
  TCS_RT(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    cudaStreamDestroy(cs);
    return fail(TCS_ERR_CUDA, std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(e));
  }
  for (unsigned i = 0; i < n && rc == TCS_OK; ++i)
    rc = separate ? batch_launch_separate(b, (int)(i & 1u), (CUstream)cs)
                  : batch_launch(b, (int)(i & 1u), (CUstream)cs);
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(cs, &graph);
  cudaStreamDestroy(cs);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess)
    return fail(TCS_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&b->exec, graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    b->exec = nullptr;
    return fail(TCS_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  }
  b->graph = graph;
  return TCS_OK;
}

int tcs_batch_graph_launch(tcs_batch* b, void* stream) {
  if (!b) return fail(TCS_ERR_INVALID_VALUE, "NULL batch");
  if (!b->exec) return fail(TCS_ERR_INVALID_VALUE, "no graph captured (tcs_batch_graph)");
  TCS_RT(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
  return TCS_OK;
}

int tcs_batch_destroy(tcs_batch* b) {
  if (b) batch_free(b);
  return TCS_OK;
}

}  // extern "C"

// =============================================================================================
// Tensor-core sweep of 2D Box stencils on FP32 grids (tcs_tc.cu).

namespace {

uint16_t bf16_bits(float f) {  // round to nearest even
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7F800000u) == 0x7F800000u && (u & 0x007FFFFFu)) return 0x7FC0u;
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

float bf16_value(uint16_t b) {
  uint32_t u = (uint32_t)b << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

int tc_check(const tcs_spec& s) {
  if (s.dimension != 2 || s.neighbourhood != TCS_BOX)
    return fail(TCS_ERR_UNSUPPORTED, "tensor-core sweep: 2D Box stencils only");
  if (s.precision != TCS_F32) return fail(TCS_ERR_UNSUPPORTED, "tensor-core sweep: FP32 grids only");
  if (s.range < 1 || s.range > 8) return fail(TCS_ERR_UNSUPPORTED, "tensor-core sweep: range 1..8");
  return TCS_OK;
}

// Toeplitz operands of the 2R+1 mask rows in the kernel's shared-memory layout: for row offset dy,
// 16-byte column c and output column n, bytes dy*6144 + c*1024 + n*16 hold the BF16 high parts of
// mask[dy][k - n] for k = 8c .. 8c+7 (zero outside 0 <= k - n <= 2R), and bytes
// dy*6144 + c*1024 + (32 + n)*16 the low parts.  Jacobi stencils use the weight 1/S everywhere.
int tc_build(tcs_stencil* h) {
  if (h->tc_bops && !h->tc_stale) return TCS_OK;
  const tcs_spec& s = h->spec;
  const int R = s.range, D = 2 * R + 1;
  const int TN = 32, NCH = 6;
  std::vector<uint16_t> buf((size_t)D * NCH * 2 * TN * 8, 0);
  const double c = 1.0 / (double)h->S;
  for (int dy = 0; dy < D; ++dy)
    for (int ch = 0; ch < NCH; ++ch)
      for (int n = 0; n < TN; ++n)
        for (int e = 0; e < 8; ++e) {
          const int k = 8 * ch + e, j = k - n;
          if (j < 0 || j > 2 * R) continue;
          const double m = s.coefficients == TCS_JACOBI ? c : h->mask_host[(size_t)j + (size_t)dy * D];
          const uint16_t hb = bf16_bits((float)m);
          const uint16_t lb = bf16_bits((float)(m - (double)bf16_value(hb)));
          const size_t at = (((size_t)dy * NCH + ch) * 2 * TN + n) * 8 + e;
          buf[at] = hb;
          buf[at + (size_t)TN * 8] = lb;
        }
  if (!h->tc_bops) TCS_RT(cudaMalloc(&h->tc_bops, buf.size() * sizeof(uint16_t)));
  TCS_RT(cudaMemcpy(h->tc_bops, buf.data(), buf.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
  h->tc_stale = false;
  return TCS_OK;
}

}  // namespace

extern "C" {

int tcs_tc_supported(const tcs_spec* spec) {
  int rc = validate(spec);
  if (rc) return rc;
  return tc_check(*spec);
}

int tcs_tc_update_grid(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, const float* in,
                       const float* src, float* out, void* stream) {
  if (!h) return fail(TCS_ERR_INVALID_VALUE, "NULL handle");
  int rc = tc_check(h->spec);
  if (rc) return rc;
  if (!in || !out) return fail(TCS_ERR_INVALID_VALUE, "NULL device buffer");
  if ((const void*)in == (const void*)out || (const void*)src == (const void*)out)
    return fail(TCS_ERR_INVALID_VALUE, "output must be distinct from input and source");
  TcsGeo g;
  if ((rc = make_geo(h, grid, right_offset, g))) return rc;
  if ((rc = tc_build(h))) return rc;
  const unsigned R = (unsigned)h->spec.range;
  TcsTcGeo tg;
  tg.xdim = g.xdim;
  tg.ydim = g.ydim;
  tg.x0 = g.x0;
  tg.x_lim = g.x_lim;
  tg.y_lim = g.y_lim;
  tg.R = R;
  const unsigned long long ex = g.x_lim > g.x0 ? g.x_lim - g.x0 : 0, ey = g.y_lim - R;
  tg.ntx = std::max(1u, cdiv(ex, 32));
  tg.nty = std::max(1u, cdiv(ey, 128));
  if ((unsigned long long)tg.ntx * tg.nty > 0x7fffffffull) return fail(TCS_ERR_UNSUPPORTED, "grid too large");
  // TMA staging needs a 16-byte row pitch, base and tile start (x0 - R = the left offset).
  const bool tma = (g.xdim * 4) % 16 == 0 && reinterpret_cast<uintptr_t>(in) % 16 == 0 && (g.x0 - R) % 4 == 0;
  alignas(64) CUtensorMap map;
  if (tma) {
    cuuint64_t gdim[2] = {g.xdim, g.ydim};
    cuuint64_t gstride[1] = {g.xdim * 4};
    cuuint32_t box[2] = {48, tcs_tc_box_rows(R)};
    cuuint32_t estride[2] = {1, 1};
    CUresult cr = g_drv.TensorMapEncodeTiled(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(in), gdim,
                                             gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return fail(TCS_ERR_CUDA, "cuTensorMapEncodeTiled: " + cu_msg(cr));
  }
  const int e = tcs_tc_launch(in, src, out, h->tc_bops, tma ? &map : nullptr, tg, (unsigned*)h->status_ptr,
                              h->num_sms, (cudaStream_t)stream);
  if (e) return fail(TCS_ERR_CUDA, std::string("tensor-core sweep: ") + cudaGetErrorString((cudaError_t)e));
  return TCS_OK;
}

}  // extern "C"

// =============================================================================================
// Temporal blocking: two sweeps per pass over the grid (2D; tcs_tb2 in tcs_kernels.cuh).

namespace {

// The tile sizes match tcs_tb2's constants.  Thread tile 1 x 8: a warp reads 32 consecutive points
// of a row (no bank conflicts) and each value loaded serves up to 8 outputs of a column.
constexpr unsigned TB_TX = 128, TB_CX = 1, TB_CY = 8, TB_THREADS = 256;
unsigned tb_ty(unsigned es) { return 256 / es; }  // tile rows: 32 FP64, 64 FP32

// A parameter set's 2D spec with the TB thread tile; every other parameter as given.
tcs_spec tb_spec(const tcs_spec& s) {
  tcs_spec t = s;
  t.cx = TB_CX;
  t.cy = TB_CY;
  t.cz = 1;
  return t;
}

int tb_module(tcs_stencil* h) {
  std::lock_guard<std::mutex> lock(h->mu);
  if (h->tb_mod) return TCS_OK;
  std::vector<char> cubin;
  int rc = instantiate(tb_spec(h->spec), nullptr, cubin, nullptr, "#define TCS_TB 1\n");
  if (rc) return rc;
  CUmodule mod = nullptr;
  CUresult cr = g_drv.ModuleLoadData(&mod, cubin.data());
  if (cr != CUDA_SUCCESS) return fail(TCS_ERR_CUDA, "cuModuleLoadData (tb2): " + cu_msg(cr));
  size_t bytes = 0;
  if ((cr = g_drv.ModuleGetFunction(&h->f_tb2, mod, "tcs_tb2")) != CUDA_SUCCESS ||
      (cr = g_drv.ModuleGetGlobal(&h->tb_mask, &bytes, mod, "tcs_mask")) != CUDA_SUCCESS) {
    g_drv.ModuleUnload(mod);
    return fail(TCS_ERR_CUDA, "tb2 module symbols: " + cu_msg(cr));
  }
  h->tb_mod = mod;
  return upload_mask(h, h->tb_mask);
}

int launch_tb2(tcs_stencil* h, const TcsGeo& g, const void* in, void* out, CUstream st) {
  const unsigned R = (unsigned)h->spec.range;
  const unsigned es = (unsigned)elem_size(h->spec);
  // first-sweep tile rounded up to whole thread tiles, input tile R wider on each side
  const unsigned TB_TY = tb_ty(es);
  const unsigned bw = cdiv(TB_TX + 2 * R, TB_CX) * TB_CX, bh = cdiv(TB_TY + 2 * R, TB_CY) * TB_CY;
  const unsigned smem = ((bw + 2 * R) * (bh + 2 * R) + bw * bh) * es;
  if (smem > (unsigned)h->smem_optin) return fail(TCS_ERR_UNSUPPORTED, "tb2: tile does not fit in shared memory");
  {
    std::lock_guard<std::mutex> lock(h->mu);
    if ((int)smem > h->tb2_smem_attr) {
      TCS_CU(g_drv.FuncSetAttribute(h->f_tb2, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)smem));
      h->tb2_smem_attr = (int)smem;
    }
  }
  const unsigned long long ex = g.x_lim > g.x0 ? g.x_lim - g.x0 : 0, ey = g.y_lim - R;
  const unsigned gx = std::max(1u, cdiv(ex, TB_TX)), gy = std::max(1u, cdiv(ey, TB_TY));
  if (gy > 65535) return fail(TCS_ERR_UNSUPPORTED, "tb2: too many tile rows");
  CUdeviceptr pin = (CUdeviceptr)in, pout = (CUdeviceptr)out;
  TcsGeo geo = g;
  void* args[] = {&pin, &pout, &geo};
  TCS_CU(g_drv.LaunchKernel(h->f_tb2, gx, gy, 1, TB_THREADS, 1, 1, smem, st, args, nullptr));
  return TCS_OK;
}

}  // namespace

extern "C" {

int tcs_sweeps_tb2(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, void* a, void* b, unsigned n,
                   void* stream, int* result_in_b) {
  if (!h) return fail(TCS_ERR_INVALID_VALUE, "NULL handle");
  if (h->spec.dimension != 2) return fail(TCS_ERR_UNSUPPORTED, "tb2: 2D stencils only");
  if (!a || !b || a == b) return fail(TCS_ERR_INVALID_VALUE, "need two distinct buffers");
  TcsGeo g;
  int rc = make_geo(h, grid, right_offset, g);
  if (rc) return rc;
  if ((rc = tb_module(h))) return rc;
  void* src = a;
  void* dst = b;
  for (unsigned i = 0; i + 1 < n; i += 2) {  // pairs of sweeps, one pass each
    if ((rc = launch_tb2(h, g, src, dst, (CUstream)stream))) return rc;
    std::swap(src, dst);
  }
  if (n % 2 == 1) {  // the last odd sweep: one ordinary sweep
    tcs_launch L{};
    L.block[0] = 128;
    L.block[1] = 1;
    L.block[2] = 1;
    L.variant = TCS_VARIANT_AUTO;
    Resolved r;
    if ((rc = resolve(h, grid, right_offset, &L, r))) return rc;
    if ((rc = launch_resolved(h, r, src, dst, (CUstream)stream))) return rc;
    std::swap(src, dst);
  }
  if (result_in_b) *result_in_b = (src == b) ? 1 : 0;
  return TCS_OK;
}

int tcs_sweeps_tb3(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, const tcs_launch* launch,
                   void* a, void* b, unsigned n, void* stream, int* result_in_b) {
  if (!h) return fail(TCS_ERR_INVALID_VALUE, "NULL handle");
  if (!a || !b || a == b) return fail(TCS_ERR_INVALID_VALUE, "need two distinct buffers");
  TcsGeo g;
  int rc = make_geo(h, grid, right_offset, g);
  if (rc) return rc;
  if (has_fringe(h, g)) return fail(TCS_ERR_UNSUPPORTED, "tb3: grids of whole coarsening tiles only");
  Resolved r;
  if ((rc = resolve_tb3(h, g, launch, r))) return rc;
  void* src = a;
  void* dst = b;
  for (unsigned i = 0; i + 1 < n; i += 2) {  // pairs of sweeps, one pass each
    if ((rc = launch_tb3(h, r, src, dst, (CUstream)stream))) return rc;
    std::swap(src, dst);
  }
  if (n % 2 == 1) {  // the last odd sweep: one ordinary sweep
    tcs_launch L{};
    L.block[0] = 32;
    L.block[1] = 4;
    L.block[2] = 1;
    L.variant = TCS_VARIANT_AUTO;
    Resolved r1;
    if ((rc = resolve(h, grid, right_offset, &L, r1))) return rc;
    if ((rc = launch_resolved(h, r1, src, dst, (CUstream)stream))) return rc;
    std::swap(src, dst);
  }
  if (result_in_b) *result_in_b = (src == b) ? 1 : 0;
  return TCS_OK;
}

int tcs_plan_tb3(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, const tcs_launch* launch,
                 tcs_plan* plan) {
  if (!h || !plan) return fail(TCS_ERR_INVALID_VALUE, "NULL argument");
  TcsGeo g;
  int rc = make_geo(h, grid, right_offset, g);
  if (rc) return rc;
  Resolved r;
  if ((rc = resolve_tb3(h, g, launch, r))) return rc;
  return fill_plan(h, r, plan);
}

int tcs_precompile_tb3(const tcs_spec* spec, unsigned bx, unsigned by, unsigned chunk, char* cubin_path,
                       unsigned path_cap) {
  int rc = validate(spec);
  if (rc) return rc;
  const bool d3 = spec->dimension == 3;
  if (!d3 && spec->orientation == TCS_COLUMN) return fail(TCS_ERR_UNSUPPORTED, "tb3: 2D stencils in Row order only");
  const unsigned R = (unsigned)spec->range, vec = 16u / (unsigned)elem_size(*spec);
  const unsigned C = (R % 2 == 0 || !d3) ? 2u : 1u;
  if (bx == 0) {
    bx = d3 ? 32u : 64u;
    by = d3 ? ((C == 2) ? 16u : 32u) : 1u;
    while (!d3 && bx > 8 && bx * C + 2 * R + vec > 256) bx -= 8;
  }
  if (!d3) by = 1;
  if (bx * C <= 2 * R || (d3 && by * C <= 2 * R) || (bx * C - 2 * R) % vec != 0 || (bx * C) % vec != 0)
    return fail(TCS_ERR_UNSUPPORTED, "tb3: no output tile of 16-byte multiples for this range and block");
  const unsigned lshift = (unsigned)((((int)left_offset_of(*spec) - (int)R) % (int)vec + (int)vec) % (int)vec);
  PipeKey key{bx, by, chunk ? chunk : (d3 ? 2u : 8u), lshift, 0u, 0u, C};
  std::vector<char> cubin;
  std::string path;
  if ((rc = instantiate(*spec, &key, cubin, &path))) return rc;
  if (cubin_path && path_cap) {
    std::strncpy(cubin_path, path.c_str(), path_cap - 1);
    cubin_path[path_cap - 1] = '\0';
  }
  return TCS_OK;
}

}  // extern "C"

extern "C" int tcs_precompile_fringe(const tcs_spec* spec, char* cubin_path, unsigned path_cap) {
  int rc = validate(spec);
  if (rc) return rc;
  tcs_spec s1 = *spec;
  s1.cx = s1.cy = s1.cz = 1;
  std::vector<char> cubin;
  std::string path;
  if ((rc = instantiate(s1, nullptr, cubin, &path))) return rc;
  if (s1.dimension == 2 && (rc = instantiate(tb_spec(*spec), nullptr, cubin, nullptr, "#define TCS_TB 1\n")))
    return rc;
  if (cubin_path && path_cap) {
    std::strncpy(cubin_path, path.c_str(), path_cap - 1);
    cubin_path[path_cap - 1] = '\0';
  }
  return TCS_OK;
}
