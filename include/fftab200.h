/* fftab200.h -- C ABI of libfftab200.so, the sm_100a transform library that
 * stands in for FFTA.jl's complex transform path.
 *
 * FFTA.jl is pure Julia; its entry points are AbstractFFTs methods.  Each
 * function below names the FFTA method it replaces (file:line inside the
 * FFTA.jl repository).  The Julia package julia/FFTAB200 calls these with
 * `ccall`; the Python package ffta_b200 calls them with ctypes.
 *
 * Conventions
 *  - Complex data are interleaved (re, im) pairs: ComplexF32 = 2 x float,
 *    ComplexF64 = 2 x double, the memory layout of Julia's Complex{T}.
 *  - Strides and distances are in elements, not bytes.
 *  - `dir` is FB_FORWARD (-1, FFTA's FFT_FORWARD) or FB_BACKWARD (+1,
 *    FFT_BACKWARD, unnormalised), FFTA src/callgraph.jl:1.
 *  - Every function returns an FB_* status; fb_last_error() gives the
 *    message of the last failure on the calling thread.  Statuses map to the
 *    Julia exception FFTA throws in the same situation.
 *  - There is no CPU fallback: without a CUDA device every plan call fails
 *    with FB_ERR_CUDA.
 */
#ifndef FFTAB200_H
#define FFTAB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fb_plan_s* fb_plan;

enum {
  FB_OK = 0,
  FB_ERR_DIMENSION_MISMATCH = 1, /* Julia DimensionMismatch */
  FB_ERR_ARGUMENT = 2,           /* Julia ArgumentError */
  FB_ERR_DOMAIN = 3,             /* Julia DomainError */
  FB_ERR_CUDA = 4,               /* CUDA runtime failure, or no device */
  FB_ERR_UNSUPPORTED = 5,        /* a length this build has no schedule for */
  FB_ERR_OUT_OF_MEMORY = 6
};

enum { FB_C32 = 0, FB_C64 = 1 };          /* ComplexF32, ComplexF64 */
enum { FB_FORWARD = -1, FB_BACKWARD = 1 };
enum { FB_DEFAULT_BLUESTEIN_CUTOFF = 73 }; /* src/callgraph.jl:44 */

/* Plan flags.
 * FB_FLAG_GENERIC_ONLY: use only the generic line kernel, never the
 *   length-specialised ones (results are bit-identical either way; the flag
 *   exists so tests can check that).
 * FB_FLAG_SAME_SCHEDULE_STRIDED: transform long strided lines (longer than
 *   about 750 elements, e.g. the columns of a large 2-D array) with the
 *   schedule of a contiguous line of that length.  By default such axes use a
 *   four-step split that moves long contiguous runs; its results equal the
 *   contiguous schedule's within rounding but not bit for bit.  With the flag
 *   every strided transform is bit-identical to the same transform of a
 *   contiguous copy (FFTA's `==` property), at lower speed for those axes.
 * FB_FLAG_STREAM: run contiguous lines with the persistent bulk-copy
 *   variant of the specialised kernel where the length has one (bit-identical
 *   results; the autotuner also considers it).
 * FB_FLAG_TENSOR_STAGE: ComplexF32 only -- compute the first radix-16 stage
 *   of each specialised pass whose program starts with 16 on the tensor cores
 *   (tcgen05, split-BF16 operands in three terms, FP32 accumulation) instead
 *   of the FP32 butterflies.  Error stays at the FP32 path's level; results
 *   are not bit-identical to the default path.  No FFTA counterpart (FFTA
 *   computes in the element type only).
 * FB_FLAG_TMA: load the tiles of strided passes (four-step columns, strided
 *   axes) with tensor copies (cp.async.bulk.tensor) into shared memory, two
 *   tiles per persistent block, instead of thread by thread (bit-identical
 *   results).  Opt-in: on B200 the thread-loaded kernel measured faster for
 *   the four-step and 2-D column passes (more warps resident per SM).
 * FB_FLAG_TUNE_RADIX: let fb_plan_autotune also choose the radix program
 *   (the order and sizes of the butterfly stages) of each one-pass length of
 *   the plan among alternatives -- 16/8/4/2 groupings of the factor 2^a,
 *   9/3 of 3^b, powers of two or of three first -- and use the tuned
 *   programs in later plans made with this flag.  A tuned plan's results
 *   are within the usual rounding of the default plan's, not bit-identical to
 *   them.  No FFTA counterpart (FFTA's recursion order is fixed by its call
 *   graph, src/callgraph.jl:76-126). */
enum {
  FB_FLAG_GENERIC_ONLY = 1u,
  FB_FLAG_SAME_SCHEDULE_STRIDED = 2u,
  FB_FLAG_STREAM = 4u,
  FB_FLAG_TENSOR_STAGE = 8u,
  FB_FLAG_TMA = 16u,
  FB_FLAG_TUNE_RADIX = 32u
};

/* Batched 1-D plan: `batch` transforms of length n; element j of transform b
 * is read at in[b*idist + j*istride] and written at out[b*odist + j*ostride].
 * Replaces plan_fft/plan_bfft with a one-dimensional region
 * (src/plan.jl:71-87) together with the 1-D executors mul! for a vector
 * (src/plan.jl:157-167) and for the columns of an array (src/plan.jl:170-207).
 * n <= 0 gives FB_ERR_DIMENSION_MISMATCH ("Array length must be strictly
 * positive", src/callgraph.jl:83-85).  Primes >= bluestein_cutoff go through
 * Bluestein (src/callgraph.jl:95-100). */
int fb_plan_create(fb_plan* plan, int64_t n, int dtype, int dir, int64_t batch, int64_t istride,
                   int64_t idist, int64_t ostride, int64_t odist, int64_t bluestein_cutoff,
                   uint32_t flags);

/* 2-D plan over `batch` contiguous column-major n1 x n2 matrices (dim 1
 * contiguous).  Replaces plan_fft(X) with region 1:2 (src/plan.jl:88-92) and
 * the N-D executor mul! (src/plan.jl:210-257, fft_along_dim! :327-348). */
int fb_plan_create_2d(fb_plan* plan, int64_t n1, int64_t n2, int dtype, int dir, int64_t batch,
                      int64_t bluestein_cutoff, uint32_t flags);

/* General plan over a strided array of `rank` dims: dims[d] elements with
 * element strides istrides[d] (input) and ostrides[d] (output), transformed
 * along the 1-based dims listed in `region` (strictly ascending).  Replaces
 * plan_fft/plan_bfft for any region (src/plan.jl:77-100) and the executors
 * for 1-D, N-D and M<N plans (src/plan.jl:170-325).  A region that is not
 * strictly ascending gives "Region is invalid." and one outside 1..rank
 * "Plan region is outside array dimensions." (src/plan.jl:268-271), both
 * FB_ERR_DIMENSION_MISMATCH. */
int fb_plan_create_nd(fb_plan* plan, int dtype, int dir, int rank, const int64_t* dims,
                      const int64_t* istrides, const int64_t* ostrides, int nregion,
                      const int32_t* region, int64_t bluestein_cutoff, uint32_t flags);

/* Real transforms over a contiguous column-major array.  dir FB_FORWARD is
 * rfft: real input with dims[], complex output whose first region dim holds
 * dims[r]/2+1 entries (AbstractFFTs.plan_rfft, FFTA src/plan.jl:102-125 and
 * the real executors :390-454, :506-542).  dir FB_BACKWARD is brfft: complex
 * input with dims[r]/2+1 entries along the first region dim, real output
 * with dims[] (plan_brfft, src/plan.jl:127-150, :456-504, :544-583); dims[r]
 * is brfft's `len`.  dtype FB_C32 pairs Float32 with ComplexF32, FB_C64
 * Float64 with ComplexF64.  FFTA allows one or two region dims ("only
 * supports 1D and 2D FFTs"); this entry point takes any number.  irfft is
 * brfft scaled by 1/prod(len) (fb_plan_set_scale). */
int fb_plan_create_real(fb_plan* plan, int dtype, int dir, int rank, const int64_t* dims,
                        int nregion, const int32_t* region, int64_t bluestein_cutoff,
                        uint32_t flags);

/* Multiply every output by `scale` (fused into the last kernel).  ifft is
 * bfft scaled by 1/prod(n) (AbstractFFTs ScaledPlan). */
int fb_plan_set_scale(fb_plan plan, double scale);

/* Run the plan on device pointers, enqueued on `stream` (a cudaStream_t; NULL
 * is the legacy default stream).  Input and output may be the same buffer.
 * Replaces LinearAlgebra.mul!(y, p, x) (src/plan.jl:157,170,210,260). */
int fb_execute(fb_plan plan, const void* in, void* out, void* stream);

/* Run a batched 1-D plan (fb_plan_create) on its first `batch` transforms
 * only (0 <= batch <= the plan's batch, else FB_ERR_DIMENSION_MISMATCH), with
 * the plan's strides and distances: LinearAlgebra.mul! on the leading
 * columns of the array, FFTA src/plan.jl:170-207.  Results equal those of
 * the full plan for those columns bit for bit.  Lets a caller keep one plan
 * per length for every batch up to its own (the serving loop does). */
int fb_execute_batch(fb_plan plan, const void* in, void* out, int64_t batch, void* stream);

/* Run the plan on host arrays: copies in, transforms, copies out, and returns
 * when `out` holds the result.  Pinned host memory gives full copy speed.
 * Replaces Base.:*(p, x) on a CPU array (src/plan.jl:374-384). */
int fb_execute_host(fb_plan plan, const void* in, void* out, void* stream);

/* Run one batched 1-D plan over `count` requests in a single kernel launch:
 * request r has batches[r] contiguous transforms of the plan's length n at
 * device pointers ins[r] / outs[r] (distance n; the plan's own batch count is
 * ignored).  The descriptor table is copied to the device on `stream`; calls
 * with the same plan must stay on one stream.  Only plans whose length runs
 * in one specialised pass support this (else FB_ERR_UNSUPPORTED).  No FFTA
 * counterpart: FFTA runs each call's columns serially (src/plan.jl:204-206);
 * this is the work-descriptor launch of the serving loop. */
int fb_execute_grouped(fb_plan plan, int64_t count, const void* const* ins, void* const* outs,
                       const int64_t* batches, void* stream);

/* Serving: continuous batching over work-descriptor launches.  No FFTA
 * counterpart (FFTA is a library of synchronous calls).  A server admits
 * requests in arrival order while their device bytes (input + output + any
 * multi-pass scratch) fit `budget_bytes`, packs all admitted single-pass
 * requests -- any mix of lengths, types and directions -- into one kernel
 * launch per kernel variant, runs multi-pass lengths and large requests
 * (2^18 elements or more) with cached plans, each plan on one of `nstreams`
 * plan streams, and rotates launches over `nstreams` CUDA streams.  A
 * multi-pass request whose (length, type, direction, batch, input, output)
 * recurs is captured into a CUDA graph on its second occurrence and replayed
 * as one graph launch afterwards (at most 1024 graphs per server, least
 * recently used released first); FB_SERVER_NO_GRAPHS in `flags` turns this
 * off.
 * Small requests of length 16..4096 (powers of two) go instead to one
 * resident kernel: the server appends a work descriptor per request to a
 * queue in mapped host memory, and the kernel -- launched when work arrives
 * and none is resident, ending after 100 us without new work -- claims
 * chunks of lines of the queued requests with the specialised stage
 * programs.  Its waits are bounded; a request whose descriptor does not
 * arrive in time completes with done_ms = -1 in fb_server_poll (-2 when its
 * program was missing).  FB_SERVER_NO_PERSISTENT
 * sends those requests to the descriptor launches as well.
 * Multi-pass and large requests run plans kept per (length, type,
 * direction, batch rounded up to a power of two, at least 512) on the
 * request's own batch (fb_execute_batch); the least recently used idle plans
 * are released while the plans' device bytes (their tables) exceed half
 * the budget.  The plans bound to one plan stream share that
 * stream's scratch buffers, and the device blocks of released plans are
 * kept for the next plans (cudaFree would wait for the whole device).
 * FB_SERVER_SERIAL makes the server the plain path it is compared with: one
 * request at a time, each its own plan launch, the next one dispatched only
 * after the previous one completed (no packing, no resident kernel, no
 * graphs, the same plan cache). */
enum { FB_SERVER_NO_GRAPHS = 1u, FB_SERVER_NO_PERSISTENT = 2u, FB_SERVER_SERIAL = 4u };
typedef struct fb_server_s* fb_server;
int fb_server_create(fb_server* srv, double budget_bytes, int nstreams, uint32_t flags);
/* Queue `batch` contiguous transforms of length n (device pointers; the
 * caller keeps them alive until the ticket completes).  Nothing is launched
 * until fb_server_poll / fb_server_wait.  A request whose device bytes
 * (input, output and multi-pass scratch) exceed the whole budget is refused
 * with FB_ERR_OUT_OF_MEMORY; a length the build has no schedule for with
 * FB_ERR_UNSUPPORTED; n <= 0 with FB_ERR_DIMENSION_MISMATCH.  A refused
 * request takes no ticket and leaves the queue as it was. */
int fb_server_submit(fb_server srv, int64_t n, int dtype, int dir, int64_t batch, const void* in,
                     void* out, int64_t* ticket);
/* fb_server_submit for `count` requests given as arrays (one call for every
 * request that arrived since the last poll); stops at the first error. */
int fb_server_submit_many(fb_server srv, int64_t count, const int64_t* n, const int32_t* dtype,
                          const int32_t* dir, const int64_t* batch, const void* const* in,
                          void* const* out, int64_t* tickets);
/* Retire finished launches, dispatch what is queued when a stream is free,
 * and return up to `max` completed tickets with their completion times (ms
 * on the device clock since fb_server_create). */
int fb_server_poll(fb_server srv, int64_t max, int64_t* tickets, double* done_ms, int64_t* count);
/* Withdraw a request that is still waiting (not yet dispatched): it never
 * runs, its output is not written and poll never reports its ticket.
 * FB_ERR_ARGUMENT if the ticket is unknown, already dispatched or done. */
int fb_server_cancel(fb_server srv, int64_t ticket);
/* Diagnostic (failure-path tests): the next request the server sends to its
 * resident kernel is published with a descriptor that never arrives, as if
 * its write had been lost.  The kernel waits for it a bounded time (2 ms),
 * gives up, completes it with done_ms = -1 and goes on with the others.
 * FB_ERR_UNSUPPORTED without a resident kernel. */
int fb_server_drop_next_descriptor(fb_server srv);
/* Dispatch and wait until every submitted request has completed. */
int fb_server_wait(fb_server srv);
/* out[0..12]: requests, launches, descriptor launches, max queue depth, max
 * admitted bytes, resident plans, graph launches, graph captures, cancelled
 * requests, requests served by the resident kernel, requests it gave up on,
 * plans made, plans released (the first `nout` of them). */
int fb_server_stats(fb_server srv, int64_t* out, int nout);
/* Restart the clock of fb_server_poll's completion times (waits until the
 * server's first stream is idle). */
int fb_server_reset_clock(fb_server srv);
int fb_server_destroy(fb_server srv);

/* Base.size(p, i) (src/plan.jl:36-47): the transform length along the i-th
 * region entry, 1 past the last one, FB_ERR_DOMAIN for i < 1. */
int fb_plan_size(fb_plan plan, int i, int64_t* out);

/* Device bytes held by the plan (tables and scratch). */
int fb_plan_device_bytes(fb_plan plan, size_t* out);

/* Human-readable schedule (kernel passes, radices, launch shapes). */
int fb_plan_describe(fb_plan plan, char* buf, size_t len);

int fb_plan_destroy(fb_plan plan);

/* Batched contiguous ComplexF32 transform that allocates no device memory:
 * `batch` transforms of length n, element j of transform b at in[b*n + j] and
 * out[b*n + j] (device pointers), direction dir, enqueued on `stream`.
 * No counterpart in the reference (FFTA allocates its workspace while
 * planning).  It exists for callers that cannot call cudaMalloc when they
 * transform -- allocator callbacks, real-time loops that forbid allocation
 * after start-up, hosts that hand over only the data buffers.  It runs the
 * two-pass (four-step) schedule with its intermediate in a static device
 * array of 4,194,304 complex values (32 MiB, held by every GPU that loads the
 * library until exit) and its tables in a second static array.  Limits:
 * n*batch <= 4194304 (else FB_ERR_ARGUMENT) and n a product of 2s, 3s and 5s
 * (else FB_ERR_UNSUPPORTED); batch < 0 gives FB_ERR_ARGUMENT.  `in` and
 * `out` may be the same buffer.  All calls share the arrays: calls that
 * overlap on the GPU race.  The first call on a device looks up the arrays' addresses
 * (make it before any stream capture).  Errors via fb_last_error(). */
int fb_execute_noalloc_c32(const void* in, void* out, int64_t n, int64_t batch, int dir,
                           void* stream);

/* Autotuner (no FFTA counterpart: FFTA's plans are fixed by its call graph,
 * src/callgraph.jl:76-126).  Runs the plan `iters` times per candidate launch
 * shape -- lines per block of each pass and, on the generic kernel, threads
 * per line -- on the given device buffers (their contents are overwritten),
 * keeps the fastest, and caches it for later plans of this process with the
 * same type, direction, dims, strides and region.  The stage program of a
 * length (its radix order) is not tuned, so results do not change -- unless
 * the plan was made with FB_FLAG_TUNE_RADIX, which also times alternative
 * radix programs of each one-pass length and keeps the fastest. */
int fb_plan_autotune(fb_plan plan, const void* in, void* out, void* stream, int iters);
/* Save / load the process-wide tuning cache (a text file).  Loaded entries
 * are applied only where every shape is valid for the plan's kernels. */
int fb_tune_cache_save(const char* path);
int fb_tune_cache_load(const char* path);

/* Diagnostic: the current device's kernel error flag (0; a radix that a
 * stage program named without a butterfly for it; or -1 when a kernel gave up
 * waiting about a second for one of its bulk copies to land and stopped
 * early, leaving that output partial), optionally reset.  No
 * FFTA counterpart: FFTA raises ArgumentError("kernel not implemented")
 * for an unknown node type (src/algos.jl:31). */
int fb_kernel_error_flag(int* value, int reset);

/* Limit, in nanoseconds, of every wait a kernel makes on its own
 * asynchronous work (the bulk copies of FB_FLAG_STREAM kernels, the products
 * of FB_FLAG_TENSOR_STAGE kernels) for launches made after this call, in
 * every thread of the process.  When a wait runs out the kernel sets the
 * error flag to -1 (fb_kernel_error_flag), stops early and leaves its output
 * partial; before it reuses or frees the memory those copies or products
 * write, it still waits at least the default limit for them.  ns <= 0
 * restores the default (about one second).  No FFTA counterpart: FFTA has no
 * asynchronous work to wait for. */
int fb_set_wait_limit(int64_t ns);

/* Message of the last failing call on this thread ("" if none). */
const char* fb_last_error(void);

/* Library version string. */
const char* fb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* FFTAB200_H */
