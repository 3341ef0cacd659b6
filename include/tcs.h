/* tcs.h — C ABI of the B200 thread-coarsened stencil engine (libtcs.so).
 *
 * This is the drop-in boundary for the reference's host interface `launchUpdateGrid.h`
 * (cuda/launchUpdateGrid.h:13-18) and the generated implementation of it
 * (cuda/generateLaunchUpdateGrid.py:71-158).  The reference bakes one stencil parameter set
 * into one generated `kernels.cu`; here a `tcs_stencil` handle plays that role: it is created
 * from a `tcs_spec` (the generators' argv, cuda/generate2DStencil_cuda.py:31-44,
 * cuda/generate3DStencil_cuda.py:32-46) and owns the kernels instantiated for it.
 *
 * Conventions: plain C types only; device buffers are raw device pointers owned by the caller;
 * `stream` is a cudaStream_t (NULL = legacy default stream, as in the reference).  Every call
 * returns a status (TCS_OK or a TCS_ERR_* code) and never throws or exits; the message of the
 * last failure on the calling thread is available from tcs_last_error().
 */
#ifndef TCS_H
#define TCS_H

#ifdef __cplusplus
extern "C" {
#endif

#define TCS_ABI_VERSION 2

/* Status codes. */
#define TCS_OK 0
#define TCS_ERR_INVALID_VALUE 1   /* bad/mismatched argument: the reference throws cudaErrorInvalidValue */
#define TCS_ERR_CUDA 2            /* a CUDA runtime/driver call failed */
#define TCS_ERR_COMPILE 3         /* NVRTC instantiation of the kernel templates failed */
#define TCS_ERR_UNSUPPORTED 4     /* launch shape not supported by the requested kernel variant */
#define TCS_ERR_DEVICE_TIMEOUT 5  /* a bounded device-side wait expired (recorded by the kernel) */
#define TCS_ERR_NO_DEVICE 6       /* no CUDA device is visible */

/* Parameter enumerations (string forms in the reference: 'Box'/'Star', 'Row'/'Column',
 * 'Jacobi'/'Variable', 'None'/'Read'/'Write'). */
#define TCS_BOX 0
#define TCS_STAR 1
#define TCS_ROW 0
#define TCS_COLUMN 1
#define TCS_JACOBI 0
#define TCS_VARIABLE 1
#define TCS_ALIGN_NONE 0
#define TCS_ALIGN_READ 1
#define TCS_ALIGN_WRITE 2
#define TCS_F64 0 /* the reference's arithmetic (double) */
#define TCS_F32 1 /* single-precision grids */
#define TCS_F32C 2 /* single-precision grids, compensated accumulation in the reference's term order.
                      Direct and march kernels: every output also sums the rounding errors of its
                      additions (two-sum) and products (fma(v,m,-v*m)) and adds them at the end;
                      |error| <= 3u|exact| + 4Su^2 sum|m||x| (u = 2^-24).  Pipelined kernel (Box,
                      Row order, even x coarsening): each footprint row's 2R+1 terms are summed with
                      plain FMAs and the row partials combined with two-sum;
                      |error| <= 3u|exact| + (2R+2)u sum|m||x|. */

/* Kernel variants. */
#define TCS_VARIANT_AUTO 0   /* pipe, else march, else direct: the first that supports the shape */
#define TCS_VARIANT_DIRECT 1 /* reference launch geometry, operands through L1 */
#define TCS_VARIANT_MARCH 2  /* TMA-fed shared-memory ring, CTAs march along the slowest axis */
#define TCS_VARIANT_PIPE 3   /* persistent streaming sweep, 2R+1 output planes in flight per thread
                                (3D, and 2D Row orientation; march-axis block dimension 1) */

typedef struct tcs_stencil tcs_stencil; /* opaque handle: one instantiated parameter set */

/* Stencil parameter set (cuda/generate2DStencil_cuda.py:31-44, cuda/generate3DStencil_cuda.py:32-46,
 * cuda/benchmark.h:40-47). */
typedef struct tcs_spec {
  int dimension;     /* 2 or 3 */
  int neighbourhood; /* TCS_BOX | TCS_STAR */
  int orientation;   /* TCS_ROW | TCS_COLUMN */
  int coefficients;  /* TCS_JACOBI | TCS_VARIABLE */
  int range;         /* >= 1 */
  int cx, cy, cz;    /* coarsening factors >= 1 (cz ignored in 2D) */
  int alignment;     /* TCS_ALIGN_NONE | TCS_ALIGN_READ | TCS_ALIGN_WRITE */
  int cl_size;       /* alignment size in grid points (> 0 unless alignment is None) */
  int precision;     /* TCS_F64 | TCS_F32 */
} tcs_spec;

/* Grid geometry after coarsening truncation and alignment padding
 * (cuda/benchmark.cpp:262-308, cuda/benchmark.h:100-123). */
typedef struct tcs_geometry {
  unsigned grid[3];         /* gridSize: x = padded row pitch (xmem), y, z (1 in 2D) */
  unsigned elements[3];     /* gridElements: updated (interior) points per axis (1 for z in 2D) */
  unsigned threads[3];      /* gridThreads = elements / coarsening */
  unsigned left_offset;     /* Write alignment: padding left of every row (baked into kernels) */
  unsigned right_offset;    /* Read/Write alignment: padding right of every row */
  unsigned long long n_points; /* N = grid[0]*grid[1]*grid[2]: elements per buffer */
} tcs_geometry;

/* Launch parameters of one sweep. */
typedef struct tcs_launch {
  unsigned block[3];        /* thread-block shape (z = 1 in 2D) */
  unsigned grid_blocks[3];  /* direct variant: CTA grid; zeros = ceil(gridThreads / block) */
  int variant;              /* TCS_VARIANT_* */
  unsigned segments;        /* march: CTAs along the march axis per tile column (0 = auto) */
  unsigned depth;           /* march/pipe: chunks in flight ahead of the current step (0 = auto) */
  unsigned chunk;           /* pipe: planes per ring chunk (0 = auto) */
  unsigned flags;           /* TCS_LAUNCH_* options (0: the planner's choice) */
} tcs_launch;

/* tcs_launch.flags: the pipelined sweep's middle rows of a Star stencil (Row order, block x extent a
 * multiple of 32) through warp shuffles, or through shared-memory loads only. */
#define TCS_LAUNCH_SHUFFLE 1u
#define TCS_LAUNCH_NO_SHUFFLE 2u
/* tcs_launch.flags: the pipelined sweep of a 3D Star stencil in Row order in its ring form: own
 * centre values and finished crosses in two R-entry rings in tensor memory, two output planes in
 * registers (plain single-grid sweeps; cx*cy*sizeof(element)/4 of 4, 8, 16 or 32). */
#define TCS_LAUNCH_TMEM 4u
/* tcs_launch.flags: the pipelined sweep's persistent CTAs each take one tile column (or an equal
 * part of one): the tiles sweep the march axis in step, so neighbouring tiles' shared halo rows
 * are read from L2 (CTA count = tiles x the largest k the resident CTAs allow). */
#define TCS_LAUNCH_LOCKSTEP 8u

/* Resolved launch of one sweep (what tcs_update_grid will run). */
typedef struct tcs_plan {
  int variant;              /* TCS_VARIANT_DIRECT or TCS_VARIANT_MARCH */
  unsigned grid_blocks[3];
  unsigned block[3];
  unsigned dyn_smem;        /* dynamic shared memory per CTA in bytes */
  unsigned seg_len;         /* march: outputs along the march axis per CTA; pipe: work items per CTA */
  unsigned nslot;           /* march: ring slots */
  unsigned width;           /* march/pipe: shared-memory row width in elements */
  unsigned chunk;           /* pipe: planes per ring chunk */
  unsigned depth;           /* march: chunks in flight */
  unsigned loader;          /* march: 0 = TMA tensor copies, 1 = cp.async element copies */
  int ctas_per_sm;          /* occupancy of the resolved kernel at this shape */
  int num_sms;
} tcs_plan;

/* Library / error state. */
int tcs_abi_version(void);
const char* tcs_last_error(void);

/* Host-only parameter logic (no GPU needed). */
/* Validate a parameter set: stencilBenchmark::checkParameters (cuda/benchmark.cpp:430-491)
 * and the generators' argv checks (cuda/generate2DStencil_cuda.py:49-60). */
int tcs_spec_validate(const tcs_spec* spec);
/* stencilSize and flopsPerUpdate (cuda/benchmark.cpp:62-81). */
int tcs_stencil_size(const tcs_spec* spec, unsigned* stencil_size, unsigned* flops_per_update);
/* Truncation to a coarsening multiple and Read/Write row padding (cuda/benchmark.cpp:142-179). */
int tcs_compute_geometry(const tcs_spec* spec, unsigned nx, unsigned ny, unsigned nz,
                         tcs_geometry* out);
/* The same geometry without the truncation of the interior to a coarsening multiple (no
 * counterpart in the reference, which truncates: cuda/benchmark.cpp:142-166).  Sweeps of such a
 * "ragged" grid update every interior point: the kernels sweep the whole coarsening tiles and a
 * coarsening-1 instance of the direct kernel sweeps the partial tiles at the far x, y and z ends,
 * with the reference's per-point term order (the values equal a coarsening-1 sweep bit for bit).
 * threads[] counts the partial tiles. */
int tcs_compute_geometry_ragged(const tcs_spec* spec, unsigned nx, unsigned ny, unsigned nz,
                                tcs_geometry* out);

/* Left offset baked into Write-aligned kernels (cuda/generate2DStencil_cuda.py:83-85). */
int tcs_left_offset(const tcs_spec* spec, unsigned* left_offset);

/* Handle lifetime.  tcs_create instantiates (or loads from the cubin cache) the kernels of the
 * parameter set on the current device; it is the equivalent of generating and building
 * kernels.cu + launchUpdateGrid.cu (cuda/RunBenchmark.sh:118-129). */
int tcs_create(const tcs_spec* spec, tcs_stencil** out);
int tcs_destroy(tcs_stencil* h);
int tcs_get_spec(const tcs_stencil* h, tcs_spec* out);

/* copyMask (cuda/generateLaunchUpdateGrid.py:77-82): upload `n` <= stencilSize coefficients
 * into the module's constant bank (converted to float for TCS_F32).  Jacobi stencils ignore it,
 * like the reference's empty copyMask. */
int tcs_copy_mask(tcs_stencil* h, const double* mask, unsigned n);

/* maxPotentialBlockSize (cuda/generateLaunchUpdateGrid.py:84-89) of the direct kernel. */
int tcs_max_potential_block_size(tcs_stencil* h, int* out);

/* Resolve a launch without running it. */
int tcs_plan_launch(tcs_stencil* h, const unsigned grid[3], unsigned right_offset,
                    const tcs_launch* launch, tcs_plan* out);

/* One sweep out = stencil(in) over the interior: the `updateGrid<<<gridBlocks, blockSize>>>`
 * launch of cuda/generateLaunchUpdateGrid.py:92-100.  `grid` is the padded gridSize and
 * `right_offset` the row padding, exactly as the reference kernel receives them.  Asynchronous
 * on `stream`. */
int tcs_update_grid(tcs_stencil* h, const unsigned grid[3], unsigned right_offset,
                    const tcs_launch* launch, const void* in, void* out, void* stream);

/* `n` ping-pong sweeps a -> b -> a ...; *result_in_b = 1 when the last sweep wrote b. */
int tcs_sweeps(tcs_stencil* h, const unsigned grid[3], unsigned right_offset,
               const tcs_launch* launch, void* a, void* b, unsigned n, void* stream,
               int* result_in_b);

/* `n` ping-pong sweeps timed with CUDA events on `stream` (synchronises); *ms = elapsed. */
int tcs_time_sweeps(tcs_stencil* h, const unsigned grid[3], unsigned right_offset,
                    const tcs_launch* launch, void* a, void* b, unsigned n, void* stream,
                    float* ms);

/* Sweep `njobs` host-resident grids of one geometry: job j copies host_in[j] to the device, runs
 * `n` ping-pong sweeps and copies the result to host_out[j] (no counterpart in the reference,
 * whose host program allocates one pair of device grids and fills them on the device:
 * cuda/benchmark.cpp:194-196).  Jobs rotate over `nslots` slots, each a pair of
 * device buffers (dev_a[s], dev_b[s], the grid's size) with a stream of its own, so the upload
 * of one job, the sweeps of another and the download of a third overlap; with pinned host
 * buffers the link runs both directions at once.  Every job's result equals the same sweeps run
 * alone, bit for bit.  host_out buffers must not overlap any host_in, nor each other unless the
 * two jobs share a slot (j = j' mod nslots: their downloads run in order).  Returns after every
 * job's download completed; *ms (may be NULL) = device time from the first upload's start to the
 * last download's end, measured with CUDA events joined across the slots' streams. */
int tcs_sweep_host_jobs(tcs_stencil* h, const unsigned grid[3], unsigned right_offset,
                        const tcs_launch* launch, const void* const* host_in, void* const* host_out,
                        unsigned njobs, unsigned n, void* const* dev_a, void* const* dev_b,
                        unsigned nslots, float* ms);

/* benchmarkUpdateGrid (cuda/launchUpdateGrid.h:13, cuda/generateLaunchUpdateGrid.py:103-147):
 * runtime sanity check of the baked-in parameters, then the doubling loop of synchronous
 * launches with host timestamps.  Writes up to `cap` per-launch durations [s]; *n_out is the
 * number measured.  The ping-pong swap is local, as in the reference. */
int tcs_benchmark_update_grid(tcs_stencil* h, const char* coeff_type, const char* neighbourhood,
                              unsigned stencil_range, unsigned dimension, const char* alignment,
                              double max_time, const unsigned grid[3], const unsigned block[3],
                              const unsigned grid_blocks[3], void* d_array0, void* d_array1,
                              unsigned right_offset, double* durations, unsigned cap,
                              unsigned* n_out);

/* Every per-launch duration [s] of the handle's last tcs_benchmark_update_grid loop, however many
 * it measured: writes up to `cap` and sets *n_out to the full count.  The reference's launcher
 * returns them all as a std::vector (cuda/generateLaunchUpdateGrid.py:140-147); a caller sizes its
 * buffer from *n_out of the benchmark call and collects them here. */
int tcs_benchmark_durations(tcs_stencil* h, double* durations, unsigned cap, unsigned* n_out);

/* launchInit (cuda/launchUpdateGrid.h:14, cuda/generateLaunchUpdateGrid.py:150-158): the
 * reference's `init` pattern (cuda/generate2DStencil_cuda.py:321-350,
 * cuda/generate3DStencil_cuda.py:386-430), synchronous. */
int tcs_launch_init(tcs_stencil* h, const unsigned grid[3], const unsigned block[3],
                    const unsigned grid_blocks[3], void* d_array, unsigned right_offset);

/* Failure-detection self-test (no counterpart in the reference, whose launcher only prints CUDA
 * errors: cuda/generateLaunchUpdateGrid.py:62-69).  One warp waits on a barrier that nothing
 * arrives at, through the same bounded wait the sweep kernels use, for at most `cycles` clock
 * cycles (1e3..4e9; 2e6 is about a millisecond), then records the timeout in the handle's device
 * status word as an expired sweep wait does.  The call reads and clears the word and returns
 * TCS_ERR_DEVICE_TIMEOUT when the timeout was recorded -- the expected outcome -- with the
 * context still usable. */
int tcs_self_test_wait(tcs_stencil* h, long long cycles);

/* Read (and optionally clear) the device status word of the handle's kernels. */
int tcs_device_status(tcs_stencil* h, unsigned* status, int clear);

/* Launch used by tcs_benchmark_update_grid (default TCS_VARIANT_AUTO with auto segments/depth;
 * TCS_VARIANT_DIRECT reproduces the reference's own grid geometry exactly). */
int tcs_set_dropin_launch(tcs_stencil* h, int variant, unsigned segments, unsigned depth);

/* Instantiate the kernels of a parameter set into the cubin cache without a GPU (NVRTC only);
 * writes the cache path.  Used by the build step so GPU runs start warm. */
int tcs_precompile(const tcs_spec* spec, char* cubin_path, unsigned path_cap);

/* Same for the pipelined sweep of a launch shape (block bx x by, `chunk` planes per ring slot,
 * 0 = the planner's default). */
int tcs_precompile_pipe(const tcs_spec* spec, unsigned bx, unsigned by, unsigned chunk,
                        char* cubin_path, unsigned path_cap);

/* Same with launch options (TCS_LAUNCH_* flags). */
int tcs_precompile_pipe_flags(const tcs_spec* spec, unsigned bx, unsigned by, unsigned chunk, unsigned flags,
                              char* cubin_path, unsigned path_cap);

/* Same with an epilogue: 1 = the FP64 defect sweep, 2 = the FP32 accumulating sweep. */
int tcs_precompile_pipe_epilogue(const tcs_spec* spec, unsigned bx, unsigned by, unsigned chunk, unsigned epi,
                                 char* cubin_path, unsigned path_cap);

/* Two sweeps per pass over HBM (temporal blocking; no counterpart in the reference, which sweeps
 * once per launch: cuda/generateLaunchUpdateGrid.py:128-139).  n ping-pong sweeps starting from a,
 * in passes of two (tcs_tb3 kernel), an odd last sweep as an ordinary sweep; *result_in_b says
 * which buffer holds the result.  Bit-identical to n tcs_update_grid sweeps.  `launch` (may be
 * NULL) gives the block (bx, by) of the kernel's thread tiles -- 2 x 2 points for even ranges,
 * 1 x 1 for odd ones; in 2D, strips of bx thread tiles of 2 x 1 points marching along y, block
 * (bx, 1, 1) -- the planes (2D: rows) per ring chunk, the chunks in flight and the CTA count
 * (segments).  3D, and 2D in Row order; FP64 and FP32 (FP32: even ranges), grids of whole
 * coarsening tiles; TCS_ERR_UNSUPPORTED otherwise. */
int tcs_sweeps_tb3(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, const tcs_launch* launch,
                   void* a, void* b, unsigned n, void* stream, int* result_in_b);

/* The launch tcs_sweeps_tb3 would make (variant reported as TCS_VARIANT_PIPE). */
int tcs_plan_tb3(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, const tcs_launch* launch,
                 tcs_plan* plan);

/* Instantiate the two-sweep kernel of a parameter set (block bx x by, 0 = the default; chunk 0 =
 * 2 planes in 3D, 8 rows in 2D) into the cubin cache without a GPU. */
int tcs_precompile_tb3(const tcs_spec* spec, unsigned bx, unsigned by, unsigned chunk, char* cubin_path,
                       unsigned path_cap);

/* ---- Mixed-precision helpers (FP64 defect correction of FP32 sweeps) ----
 * All act on the interior of buffers laid out like the sweep buffers (gridSize, rightOffset).
 * They are additions of this engine; the reference computes in FP64 only. */

/* One sweep out = stencil(in) + src (src: same layout and precision).  With src == NULL this is
 * tcs_update_grid. */
int tcs_update_grid_source(tcs_stencil* h, const unsigned grid[3], unsigned right_offset,
                           const tcs_launch* launch, const void* in, const void* src, void* out,
                           void* stream);

/* Fused defect-correction sweeps on the pipelined kernel (variant TCS_VARIANT_AUTO or
 * TCS_VARIANT_PIPE; grids of whole coarsening tiles; TCS_ERR_UNSUPPORTED otherwise).
 * tcs_defect_sweep (FP64 handle): one sweep of x whose epilogue writes the defect
 * r = fl32(S(x) - x) on the interior and, when norms != NULL, the norms {max |S(x) - x|,
 * ||S(x) - x||_2} in FP64 (synchronises `stream`).  S(x) itself is never stored.  r is
 * bit-identical to tcs_update_grid into a buffer sx followed by tcs_residual(x, sx); the 2-norm is
 * summed per thread and per CTA, so its last bits may differ from tcs_residual's.  The per-CTA
 * partials live in the handle's scratch memory.
 * tcs_update_grid_accumulate (FP32 handle): x += (double)(S(in) + src) on the interior, with x the
 * FP64 state (src may be NULL): the last correction sweep of a period and the accumulation into
 * the state in one pass, bit-identical to tcs_update_grid_source into e followed by
 * tcs_accumulate(x, e).  The current device must be the handle's. */
int tcs_defect_sweep(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, const tcs_launch* launch,
                     const void* x, float* r, double norms[2], void* stream);
int tcs_update_grid_accumulate(tcs_stencil* h, const unsigned grid[3], unsigned right_offset,
                               const tcs_launch* launch, const void* in, const void* src, double* x,
                               void* stream);

/* FP64 defect r = fl32(sx - x) (sx = one FP64 sweep of x) and, when norms != NULL, the global
 * residual norms {max |sx - x|, ||sx - x||_2} computed on the GPU in FP64 (synchronises
 * `stream`).  Uses library-allocated scratch memory for the per-block partial sums.  The calling
 * thread's current device must be the handle's (TCS_ERR_INVALID_VALUE otherwise). */
int tcs_residual(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, const double* x,
                 const double* sx, float* r, double norms[2], void* stream);

/* tcs_residual without any allocation.  No counterpart in the reference.
 * For callers that cannot allocate device memory where they need the residual norm: code whose
 * device memory is owned by another allocator (a framework's caching allocator), solver loops
 * that cannot afford the implicit device synchronisation of cudaMalloc/cudaFree, or processes
 * held to a fixed memory budget.  It calls no cudaMalloc, cudaFree or other allocating routine:
 * the per-block partial sums live in a static 32 KiB device array of libtcs.so (4096 doubles),
 * which every GPU that loads the library holds until the process exits.  `nblocks` partial
 * blocks (0 = 2 per SM) need 2*nblocks + 2 doubles, so at most 2047 blocks; larger requests
 * return TCS_ERR_INVALID_VALUE with the limit in the message.  The first call in a context looks
 * up the array's device address (cudaGetSymbolAddress, with that device current), so make that
 * first call before any stream capture; after cudaDeviceReset the recreated context is a new one,
 * and its first call (again before any capture) looks the address up again.  The calling thread's
 * current device must be the handle's (TCS_ERR_INVALID_VALUE otherwise, as for tcs_residual).
 * All calls share the array and it keeps the last call's
 * contents (nothing in it needs to start at zero); calls that overlap on the GPU race on it, so
 * serialise them (one stream, or events).  Outputs and norms are those of tcs_residual. */
int tcs_residual_static(tcs_stencil* h, const unsigned grid[3], unsigned right_offset,
                        const double* x, const double* sx, float* r, double norms[2],
                        unsigned nblocks, void* stream);

/* Bytes of device scratch the handle has allocated for its field reductions (tcs_residual,
 * tcs_compare); 0 until one of them runs.  tcs_residual_static never adds to it. */
int tcs_scratch_bytes(tcs_stencil* h, unsigned long long* bytes);

/* x += e (FP64 state, FP32 correction). */
int tcs_accumulate(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, double* x,
                   const float* e, void* stream);

/* Error statistics of a (TCS_F32 or TCS_F64) against b (FP64): {max |a-b|, ||a-b||_2, max |b|,
 * ||b||_2} over the interior, computed on the GPU (synchronises `stream`). */
int tcs_compare(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, const void* a,
                int a_precision, const double* b, double stats[4], void* stream);

/* Number of SMs of the current device. */
int tcs_device_sm_count(int* out);

/* ---- Batched sweeps over many grids (no counterpart in the reference, which sweeps one grid
 * per launch: cuda/generateLaunchUpdateGrid.py:103-147) ----
 * A batch is a list of grids of ONE parameter set, each with its own extents and its own two
 * buffers (a, b), swept together by ONE persistent launch of the pipelined kernel: the CTAs take
 * equal shares of all grids' (tile, plane) work, so small grids leave no SM idle and there is no
 * per-grid launch or tail.  Each grid's result is bit-identical to tcs_update_grid on that grid.
 * Grids are described like tcs_update_grid's (gridSize x,y,z and rightOffset per grid, or NULL for
 * zeros); `launch` gives the pipe block (bx, by, 1), chunk, depth and, in `segments`, an explicit
 * CTA count (0 = every SM at full occupancy).  Buffers belong to the caller and must outlive the
 * batch; the batch must be destroyed before its stencil handle.  tcs_batch_create allocates the
 * two device grid tables (a->b and b->a; one tensor map per grid and direction). */
typedef struct tcs_batch tcs_batch;
int tcs_batch_create(tcs_stencil* h, unsigned ngrids, const unsigned* grids /* 3 per grid */,
                     const unsigned* right_offsets, const tcs_launch* launch, void* const* a,
                     void* const* b, tcs_batch** out);
/* Launch shape of the batched kernel (grid_blocks[0] CTAs, seg_len work items each). */
int tcs_batch_plan(const tcs_batch* b, tcs_plan* out);
/* One sweep of every grid: a -> b (from_b = 0) or b -> a (from_b = 1), one launch. */
int tcs_batch_sweep(tcs_batch* b, int from_b, void* stream);
/* The same sweep as one single-grid pipe launch per grid (the unbatched comparison). */
int tcs_batch_sweep_separate(tcs_batch* b, int from_b, void* stream);
/* Capture n ping-pong sweeps starting from a (batched, or with separate != 0 one launch per grid
 * per sweep) into a CUDA graph held by the batch, replacing any earlier one. */
int tcs_batch_graph(tcs_batch* b, unsigned n, int separate);
/* Launch the captured graph on `stream`. */
int tcs_batch_graph_launch(tcs_batch* b, void* stream);
int tcs_batch_destroy(tcs_batch* b);
/* Instantiate the batched kernel of a launch shape into the cubin cache (NVRTC only). */
int tcs_precompile_batch(const tcs_spec* spec, unsigned bx, unsigned by, unsigned chunk,
                         char* cubin_path, unsigned path_cap);

/* n ping-pong sweeps starting from `a` with temporal blocking (2D only; no counterpart in the
 * reference): every pair of sweeps is one pass over the grid -- a CTA computes the first sweep on
 * its tile plus a range-wide halo in shared memory and the second from it -- so HBM is read and
 * written once per two sweeps.  Each point's terms keep the reference's order: results equal n
 * ordinary sweeps bit for bit (ragged grids included).  An odd last sweep is an ordinary sweep.
 * *result_in_b tells which buffer holds the result. */
int tcs_sweeps_tb2(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, void* a, void* b,
                   unsigned n, void* stream, int* result_in_b);
/* Instantiate the coarsening-1 instance of a parameter set (fringe of ragged grids) and, for 2D
 * sets, the 1 x 8 temporal-blocking instance into the cubin cache (NVRTC only). */
int tcs_precompile_fringe(const tcs_spec* spec, char* cubin_path, unsigned path_cap);

/* ---- Tensor-core sweep of 2D Box stencils on FP32 grids (no counterpart in the reference, which
 * runs the generated kernel on the FP64 pipe: cuda/generate2DStencil_cuda.py:146-198) ----
 * out = stencil(in) (+ src when src != NULL) over the interior, as a banded dense contraction on the
 * tcgen05 tensor cores: inputs and mask split into BF16 high and low parts, the products hi*hi,
 * hi*lo and lo*hi accumulated in FP32.  Each output has a relative error of a few 1e-5 of
 * sum |mask| |in| (not the reference's bits: this is a precision option, meant for the FP32
 * correction sweeps of FP64 defect correction).  Supported: dimension 2, Box, TCS_F32, range 1..8
 * (any orientation, alignment and coarsening; Jacobi uses the weight 1/S).  The first call after
 * tcs_copy_mask uploads the mask's Toeplitz operands (synchronous). */
int tcs_tc_supported(const tcs_spec* spec);
int tcs_tc_update_grid(tcs_stencil* h, const unsigned grid[3], unsigned right_offset, const float* in,
                       const float* src, float* out, void* stream);

/* ---- Autotuner cost model (no counterpart in the reference, whose block shape is chosen by an
 * exhaustive timed sweep: cuda/benchmark.cpp:223-251, 287-318) ----
 * A 3-layer perceptron n_in -> H -> H -> 1 with ReLU, FP32, trained with Adam on the mean squared
 * error, all on the GPU by this library's own kernels.  Parameters are one packed vector:
 * W1 [n_in x H], b1 [H], W2 [H x H], b2 [H], W3 [H], b3 (row-major, input index first).
 * Inputs x are device arrays of n rows x n_in features; targets t and outputs y have n rows.
 * Reductions run in a fixed order: results are deterministic. */
typedef struct tcs_mlp tcs_mlp;
/* Allocates parameters, Adam state and activation buffers for batches of up to max_batch rows
 * (parameters start at zero: set them). */
int tcs_mlp_create(unsigned n_in, unsigned n_hidden, unsigned max_batch, tcs_mlp** out);
int tcs_mlp_param_count(const tcs_mlp* m, unsigned* count);
/* Host -> model parameters (count values); also clears the Adam moments and step. */
int tcs_mlp_set_params(tcs_mlp* m, const float* host, unsigned count);
int tcs_mlp_get_params(const tcs_mlp* m, float* host, unsigned count);
/* y = model(x) for n rows (any n; processed max_batch rows at a time). */
int tcs_mlp_forward(tcs_mlp* m, const float* x, unsigned n, float* y, void* stream);
/* Gradient of mean((model(x) - t)^2) over n <= max_batch rows into the device vector grad (count
 * values, may be NULL); the loss goes to *loss (host; synchronises the stream) when loss != NULL. */
int tcs_mlp_gradient(tcs_mlp* m, const float* x, const float* t, unsigned n, float* grad, float* loss,
                     void* stream);
/* One Adam step (bias-corrected) on the minibatch (x, t) of n <= max_batch rows. */
int tcs_mlp_adam_step(tcs_mlp* m, const float* x, const float* t, unsigned n, float lr, float beta1,
                      float beta2, float eps, float* loss, void* stream);
int tcs_mlp_destroy(tcs_mlp* m);

#ifdef __cplusplus
}
#endif

#endif /* TCS_H */
