/*
 * fishfry_b200 C ABI -- the drop-in boundary of the B200 Poisson solve.
 *
 * Plain C: pointers, sizes and status codes.  No CUDA or C++ types cross this
 * line (streams travel as void*, i.e. a cudaStream_t or NULL for the legacy
 * default stream).  Every device pointer is caller-owned memory on the
 * current CUDA device.
 *
 * Each entry point replaces one interface of the reference (trey-ornl/fishfry):
 *   ff_plan_create   <- ParisPencil::ParisPencil(n, lo, hi, m, id)     ParisPencil.hpp:23, ParisPencil.cpp:7-82
 *   ff_plan_bytes    <- ParisPencil::bytes()                            ParisPencil.hpp:30
 *   ff_solve         <- ParisPencil::solve(bytes, density, potential,   ParisPencil.hpp:44, ParisPencil.cpp:95-425
 *                        stamps)
 *   ff_plan_destroy  <- ParisPencil::~ParisPencil()                     ParisPencil.cpp:84-93
 *   ff_init_field    <- FishFry init kernel                             FishFry.hpp:14-45 (launch :174)
 *   ff_error_sums    <- FishFry diff kernel + its reductions            FishFry.hpp:47-101 (launches :148, :190;
 *                                                                       MPI_Reduce :153-154, :195-196)
 * The C++ class in ParisPencil.hpp (same directory) wraps these with the
 * reference's exact constructor / bytes() / solve() signatures.
 *
 * Errors: the reference asserts or prints and calls exit() (gpu.hpp:69-87,
 * ParisPencil.cpp:101).  Here every entry point returns an ff_status; the
 * message of the last failure on the calling thread is in ff_last_error().
 */
#ifndef FISHFRY_B200_H
#define FISHFRY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  FF_OK = 0,
  FF_ERR_INVALID = 1,          /* bad argument (null pointer, non-positive size, ...) */
  FF_ERR_UNSUPPORTED = 2,      /* length above FF_MAX_AXIS, or no tile shape fits (or, in the
                                  batched and serving forms, above 574 points) */
  FF_ERR_BYTES = 3,            /* caller buffers smaller than ff_plan_bytes() */
  FF_ERR_CUDA = 4,             /* a CUDA runtime call failed (message has the name) */
  FF_ERR_NOMEM = 5,            /* device allocation failed */
  FF_ERR_TIMEOUT = 6,          /* a bounded device wait gave up */
  FF_ERR_TASKS = 7             /* task grid other than 1x1x1 (single GPU only) */
} ff_status;

enum { FF_FP64 = 0, FF_FP32 = 1 };

/* Longest axis a plan takes.  A strided-pass tile holds whole lines in shared
 * memory: 128-byte rows (8 FP64 / 16 FP32 columns) up to about 1800 / 3600
 * points, narrower rows (64 or 32 bytes) for longer lines.  A length with a
 * prime factor above 7 also needs its Bluestein convolution length M >= 2n-1
 * to fit: up to about 3600 points on x and y (FF_ERR_UNSUPPORTED beyond). */
#define FF_MAX_AXIS 4096

typedef struct ff_plan ff_plan;

/* One Fourier mode of the optional seeded random term of the right-hand side:
 * f += a*cos(kx*x + ky*y + kz*z + theta), exact solution -a/|k|^2 * cos(...). */
typedef struct {
  int kx, ky, kz;
  double a, theta;
} ff_mode;

/* Per-launch device times of one solve, in milliseconds (CUDA events):
 * count = ff_plan_phases(plan) entries of ms are filled. */
#define FF_MAX_PHASES 5
typedef struct {
  int count;
  double ms[FF_MAX_PHASES];
  double total_ms;
} ff_phase_times;

/* Plan a solve of an n[0] x n[1] x n[2] periodic grid (x slowest, z fastest:
 * index (i*n[1]+j)*n[2]+k).  lo/hi are the physical bounds with hi one cell
 * short of the period, as in the reference; they set the wavenumber scale
 * dd = 2*pi*(n-1)/(n*(hi-lo)) (ParisPencil.cpp:9-11).  precision is FF_FP64
 * (the plain method) or FF_FP32 (FP32 butterflies, FP64-generated twiddles and
 * 1/k^2).  Allocates the plan's twiddle and index tables on the current device.
 * Each length must be at most FF_MAX_AXIS.  A length with a prime factor
 * above 7 (cuFFT, the reference's transform library, takes any length) is
 * transformed by Bluestein's algorithm through an M-point convolution, M the
 * smallest 2^a 3^b 5^c 7^d >= 2n-1: its passes run plain-load tiles and
 * cost several times a 2^a 3^b 5^c 7^d length's (radix 8, 4, 2, 5, 3 and 7
 * stages); if no tile of M rows fits in shared memory the plan returns
 * FF_ERR_UNSUPPORTED. */
int ff_plan_create(const int n[3], const double lo[3], const double hi[3], int precision, ff_plan **plan);

/* Bytes each of density and potential must hold (the half spectrum
 * n0*n1*(n2/2+1) complex values, or the real field if larger). */
int ff_plan_bytes(const ff_plan *plan, size_t *bytes);

/* Grid dimensions and precision of a plan. */
int ff_plan_info(const ff_plan *plan, int n[3], int *precision);

/* Number of device launches (phases) of a solve: 5, one per pass (the
 * default), or 3 with the z and y passes fused through L2 (environment
 * FF_PASSES=3 at plan creation).  Name of phase q, built from the reference's stamp names
 * (ParisPencil.cpp:142-424), e.g. "X FFTs and filter". */
int ff_plan_phases(const ff_plan *plan);
const char *ff_phase_name(const ff_plan *plan, int q);

/* Solve lap(phi) = f.  density: device array holding f (FP64 or FP32 per the
 * plan), at least ff_plan_bytes() bytes; it is used as a work array and
 * destroyed.  potential: device array of the same size; receives phi in the
 * same layout as f.  Work is enqueued on `stream` and the call returns without
 * waiting, unless `times` is non-NULL: then it records CUDA events between the
 * passes, waits for the stream and fills the per-pass times. */
int ff_solve(const ff_plan *plan, size_t bytes, void *density, void *potential, void *stream,
             ff_phase_times *times);

/* Diagnostic: enqueues only the first `passes` (1..5) of ff_solve's five
 * passes, so each pass can be checked on its own; every intermediate is in
 * natural order.  After pass 1 potential holds the half spectrum along z,
 * S[i][j][kh] (kh < n2/2+1, row pitch: n2/2+1 complex values FP64, that
 * rounded up to even FP32); after pass 2 that spectrum transformed along y
 * (unnormalised forward DFT); after pass 3 transformed along x, multiplied by
 * the filter -1/(k^2 N) (0 at the zero mode) and transformed back along x
 * (unnormalised inverse DFT); after pass 4 density holds it transformed back
 * along y; pass 5 completes the solve (potential = phi).  No counterpart in
 * the reference, whose phase stamps (ParisPencil.cpp:142-424) time the same
 * steps.  FF_ERR_INVALID for a plan whose passes are fused (FF_PASSES=3). */
int ff_solve_passes(const ff_plan *plan, size_t bytes, void *density, void *potential, void *stream, int passes);

/* Reads and clears the plan's device status word (waits for `stream`).
 * Returns FF_ERR_TIMEOUT if a bounded wait inside a solve kernel gave up since
 * the last check (a TMA tile copy that never completed); that solve's result
 * is invalid.  ff_solve with `times` runs this check itself. */
int ff_plan_check(const ff_plan *plan, void *stream);

/* Test hook for the bounded device waits (no counterpart in the reference,
 * whose CHECK prints and exits, gpu.hpp:69-87, and whose kernels never wait
 * on one another).  iterations: iteration limit of the first wait of every
 * inbound tile copy and of every dependency wait of the fused passes
 * (FF_PASSES=3) in this plan's later solves; 0 restores the built-in limits
 * (about a second each).  target_extra: added to the producer count that each
 * dependency wait of the fused passes waits for (0 normally; 1 makes every
 * such wait run out, so a test can check that the kernels return and that
 * ff_plan_check reports FF_ERR_TIMEOUT).  A block whose wait ran out skips
 * its tile (after waiting, with the built-in limit, for its own copy in
 * flight), so that solve's result is invalid. */
int ff_plan_set_wait_limit(ff_plan *plan, int iterations, int target_extra);

int ff_plan_destroy(ff_plan *plan);

/* ---- Batched form (no counterpart in the reference, which solves one grid
 * per ParisPencil).  `count` independent grids, dims[3g..3g+2] = (ni, nj, nk)
 * of grid g, each axis at most FF_MAX_AXIS; lo/hi (3 per grid) give the
 * physical bounds as ParisPencil's constructor takes them
 * (ParisPencil.hpp:23), or NULL for the reference's domain [-pi, pi - 2pi/n].
 * A solve of the batch runs the same five passes as ff_solve, each pass one
 * persistent kernel launch over the tiles of all grids whose axes are
 * 2^a 3^b 5^c 7^d and at most 574 points, the five launches captured once
 * into a CUDA graph and replayed.  Every other grid (an axis with a prime
 * factor above 7, or longer than the batch tiles hold) is solved by its own
 * single-grid plan (Bluestein passes where needed) after the batched
 * launches, on the same stream. */
typedef struct ff_batch ff_batch;

int ff_batch_create(int count, const int *dims, const double *lo, const double *hi, int precision, ff_batch **batch);

/* Bytes each of grid `index`'s two buffers must hold (as ff_plan_bytes). */
int ff_batch_bytes(const ff_batch *batch, int index, size_t *bytes);

/* Solves every grid: density[g] and potential[g] are device buffers of at
 * least ff_batch_bytes(g) bytes, 16-byte aligned; density is destroyed.
 * Asynchronous on `stream` unless `times` is non-NULL (then times->ms[0..4]
 * are the five batched passes, times->total_ms the whole solve including the
 * grids solved by their own plans).  The first solve, and any solve whose
 * buffer pointers differ from the previous one, uploads the grid descriptors
 * and waits for `stream`; solves of one batch must not overlap each other. */
int ff_batch_solve(ff_batch *batch, void *const *density, void *const *potential, void *stream,
                   ff_phase_times *times);

/* Autotuner: times each pass with every candidate tile shape for each axis
 * length of the batch (z passes: line pairs per tile; strided passes:
 * columns per tile; compile-time or runtime radix plan; for runtime plans, the
 * order of the radices) and keeps the fastest.
 * Results are also remembered for batches created later in this process.
 * The buffers are overwritten (zeroed, then used as scratch); initialise the
 * densities after tuning.  reps: timed launches per candidate (median). */
int ff_batch_tune(ff_batch *batch, void *const *density, void *const *potential, void *stream, int reps);

/* The tile shape pass `kind` (0..4) of grid `index` uses (FF_ERR_UNSUPPORTED
 * for a grid solved by its own plan): W (line pairs for
 * the z passes, columns for the strided ones), ct (1: compile-time plan) and
 * tma (strided passes: 1 = one-plane tiles loaded by TMA boxes, 0 = tiles of
 * the flattened column index read straight from HBM; z passes of runtime
 * lengths: 1 = line blocks moved by bulk copies).  Any pointer may be NULL. */
int ff_batch_shape(const ff_batch *batch, int index, int kind, int *W, int *ct, int *tma);

/* The radix split (DIF stage radices, first stage first) grid `index` uses
 * on axis `axis` (0 = x, 1 = y, 2 = z): the tuner may reorder the radices of a
 * runtime-plan length.  radix has room for 16 entries. */
int ff_batch_radices(const ff_batch *batch, int index, int axis, int radix[16], int *count);

/* As ff_plan_check, for the batch's device status word. */
int ff_batch_check(ff_batch *batch, void *stream);

int ff_batch_destroy(ff_batch *batch);

/* ---- Serving form (no counterpart in the reference).  A request loop on a
 * library thread takes solves of mixed sizes and precisions as they arrive,
 * admits them against an HBM budget, and runs them with continuous batching:
 * every scheduling step carries each admitted request one pass further, all
 * requests at the same pass sharing one persistent launch (the batch
 * kernels), so requests that arrive while others run join the next step.
 * Axis tables stay resident per (length, precision); the device memory of
 * the requests' buffers is one arena of hbm_budget bytes reserved at
 * creation.  Each request's result is bit-identical whether it runs alone or
 * in a mix (its tiles and their arithmetic do not depend on the mix). */
typedef struct ff_server ff_server;

typedef struct {
  size_t hbm_budget; /* bytes reserved for request buffers (2 x ff_plan_bytes per request) */
  int max_active;    /* requests admitted at once (descriptor slots per precision) */
} ff_server_config;

typedef struct {
  double latency_ms; /* submit -> result ready on the device */
  double queue_ms;   /* submit -> admitted (buffers reserved, input copy issued) */
  double run_ms;     /* admitted -> result ready */
} ff_request_info;

typedef struct {
  uint64_t submitted, completed;
  double p50_ms, p99_ms, mean_ms, max_ms; /* latency over completed requests */
  double solves_per_s, points_per_s;      /* completed over first submit .. last completion */
  size_t peak_bytes, budget_bytes;        /* arena high-water mark and budget */
  uint64_t steps, launches;               /* scheduling steps and kernel launches so far */
  int max_active;                         /* most requests on the device at once */
} ff_server_report;

int ff_server_create(const ff_server_config *cfg, ff_server **server);

/* Queues a solve of the real field f (ni*nj*nk values of the precision's
 * type, x slowest) on the reference domain of n.  f is a host pointer
 * (f_on_host = 1; pinned memory avoids a staged copy) or a device pointer,
 * and must stay valid until ff_server_wait reports the request done.  The
 * server copies f on its own stream, ordered after the work queued on the
 * legacy default stream of the server's device before this call; a field
 * produced on another stream must be complete (that stream synchronised)
 * before the call.  FF_ERR_NOMEM if the request alone exceeds the budget. */
int ff_server_submit(ff_server *server, const int n[3], int precision, const void *f, int f_on_host, uint64_t *id);

/* Waits up to timeout_ms (negative, NaN or above 1e12: without limit) for the
 * request; FF_OK when its result is ready, FF_ERR_TIMEOUT otherwise.  info may
 * be NULL. */
int ff_server_wait(ff_server *server, uint64_t id, double timeout_ms, ff_request_info *info);

/* Completion queue: the id (and timings) of the next request that finished
 * and has not been returned by this call before, waiting up to timeout_ms
 * (negative, NaN or above 1e12: without limit); FF_ERR_TIMEOUT if none.  A finished request keeps
 * its buffers until fetched or released, so a client that waits for
 * requests in submission order can hold the budget with finished work while
 * an earlier, larger request waits for memory; taking completions from this
 * queue avoids that. */
int ff_server_next(ff_server *server, double timeout_ms, uint64_t *id, ff_request_info *info);

/* Copies a finished request's potential (ni*nj*nk values) to phi (host or
 * device; phi NULL copies nothing) and releases the request's buffers.  While
 * the copy runs the request is claimed: a fetch or release of the same id from
 * another thread returns FF_ERR_INVALID, and the buffers are not reused. */
int ff_server_fetch(ff_server *server, uint64_t id, void *phi, int phi_on_host);

/* Releases a finished (or not yet admitted) request without copying. */
int ff_server_release(ff_server *server, uint64_t id);

int ff_server_stats(ff_server *server, ff_server_report *stats);

/* Clears the latency record and counters (e.g. after a warm-up). */
int ff_server_reset_stats(ff_server *server);

/* FF_ERR_TIMEOUT if a kernel's bounded wait gave up; the scheduler's error if
 * it stopped. */
int ff_server_check(ff_server *server);

/* Stops the loop (requests still queued are dropped) and frees everything. */
int ff_server_destroy(ff_server *server);

/* ---- Multi-rank solve over an x-slab decomposition: the reference's task
 * grid (P, 1, 1) (ParisPencil.cpp:23-75 with mi = P, mj = mk = 1), one rank
 * per GPU.  Rank r holds planes [r*di, r*di + planes) of the real field,
 * di = ceil(n0/P) (ParisPencil.cpp:54); for the x pencils rank p holds rows
 * [p*djp, p*djp + rows) of the spectrum with every x, djp = ceil(n1/P)
 * (ParisPencil.cpp:61).  A solve is three device phases and two exchanges of
 * equal blocks of di x djp x nhp complex values (the reference's
 * MPI_Alltoall over its commI, ParisPencil.cpp:236, :312; nhp = n2/2+1 FP64,
 * that rounded up to even FP32); the block from rank r to rank p holds r's
 * planes and p's rows, [i - r*di][j - p*djp][kh].  The z and y transforms of
 * the reference's other pencil exchanges are local here.  Lengths must be
 * 2^a 3^b 5^c 7^d, at most FF_MAX_AXIS, with n0 and n1 at least P. */
typedef struct ff_slab ff_slab;

/* Rank `rank` of `nranks` (<= 64) for the grid n on the bounds lo/hi. */
int ff_slab_create(const int n[3], const double lo[3], const double hi[3], int precision, int nranks, int rank,
                   ff_slab **slab);

/* layout[0..7] = {P, rank, di, djp, first_plane, planes, first_row, rows};
 * *bytes = bytes each of density and potential must hold (the slab's real
 * field or spectrum, or P blocks); *block_bytes = bytes of one block.  Any
 * output may be NULL. */
int ff_slab_layout(const ff_slab *slab, int layout[8], size_t *bytes, size_t *block_bytes);

/* Phase 1 ("Real-to-complex FFT in Z", "Forward FFT in Y"): density holds the
 * rank's planes of f (x slowest) and is destroyed; the z pass writes the
 * slab's spectrum to potential, and the y pass stores the values of rank p's
 * rows into the block at dst[p] (p < P, device pointers, 16-byte aligned):
 * the caller's send buffer, or the block's place in rank p's receive buffer
 * if the caller can store into it (peer memory).  Enqueued on stream. */
int ff_slab_forward(const ff_slab *slab, void *density, void *potential, void *const *dst, void *stream);

/* Phase 2 ("X FFTs and filter"): pencils holds the P blocks this rank
 * received, rank 0's first (so [i][j - first_row][kh] for every i); x
 * forward, filter (global wavenumbers, 1/N of the whole grid), x inverse;
 * the values of rank q's planes go to the block at dst[q].  pencils is not
 * written. */
int ff_slab_xpass(const ff_slab *slab, const void *pencils, void *const *dst, void *stream);

/* Phase 3 ("Backward FFT in Y", "Complex-to-real FFT in Z"): packed holds
 * the P blocks this rank received back, rank 0's first; the y inverse writes
 * the slab's spectrum to density, the z pass writes phi for the rank's planes
 * to potential.  packed may be potential (it is read before the z pass
 * writes), not density. */
int ff_slab_backward(const ff_slab *slab, const void *packed, void *density, void *potential, void *stream);

/* As ff_plan_check, for the slab's kernels. */
int ff_slab_check(const ff_slab *slab, void *stream);

int ff_slab_destroy(ff_slab *slab);

/* Harness: write f on the device at x = xlo + i*dx (FishFry.hpp:22-44),
 * plus sum_m a_m cos(k_m.x + theta_m) for the given modes (nmodes may be 0).
 * precision selects a double or float field.  Enqueued on stream. */
int ff_init_field(const int n[3], const double xlo[3], const double dx[3], int nmodes,
                  const ff_mode *modes, int precision, void *f, void *stream);

/* Harness: sums[0..2] = { sum|d|, sum d^2, max|d| } with d = phi_exact - phi
 * (FishFry.hpp:57-101), accumulated in FP64 with a fixed-order (deterministic)
 * two-stage reduction.  phi == NULL gives the phi = 0 pass that the reference
 * uses for its relative-norm scales (FishFry.hpp:146-159).  sums is HOST
 * memory; the call waits for the stream, which must belong to the current
 * device (as every stream passed to this library must). */
int ff_error_sums(const int n[3], const double xlo[3], const double dx[3], int nmodes,
                  const ff_mode *modes, int precision, const void *phi, double sums[3], void *stream);

/* ff_error_sums for callers that cannot allocate device memory (no counterpart
 * in the reference).  Some callers may not allocate at the point where they
 * want the norms: their host application's pool allocator already holds the
 * device memory, cudaMalloc's implicit synchronisation is unacceptable in their
 * loop, or they are plug-ins that may not call the CUDA allocator at all.
 * This entry point calls no cudaMalloc/cudaFree: its partial sums live in a
 * fixed device array inside the library (about 384 KB per GPU, held until the
 * process exits), and grids are limited to 2^30 points (1024^3); larger ones
 * return FF_ERR_UNSUPPORTED.  Same arguments and results as ff_error_sums,
 * summed in a different fixed order (so sums agree to rounding, max exactly).
 * The first call on each device looks up that array's device address and
 * remembers it; make that call before any stream capture, and do not use this
 * entry point after a cudaDeviceReset in the same process (the remembered
 * address is then stale).  The stream must belong to the current device.  All
 * calls share the one array: calls that overlap on the GPU (other streams,
 * other threads) race and must be serialised by the caller.  sums is HOST
 * memory; the call waits for stream. */
int ff_error_sums_noalloc(const int n[3], const double xlo[3], const double dx[3], int nmodes,
                          const ff_mode *modes, int precision, const void *phi, double sums[3], void *stream);

/* Seeded random modes: `count` modes with integer k, 0 < |k| <= kmax and
 * |k_axis| <= kaxis[axis]; amplitude ~ N(0, sigma), phase ~ U[0, 2*pi)
 * (SplitMix64 counter stream + Box-Muller).  Host only. */
int ff_modes_generate(uint64_t seed, int count, int kmax, const int kaxis[3], double sigma, ff_mode *out);

/* Status text and the last error message of the calling thread. */
const char *ff_status_string(int status);
const char *ff_last_error(void);

/* Library version string. */
const char *ff_version(void);

#ifdef __cplusplus
}
#endif

#endif
