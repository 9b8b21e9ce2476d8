// fb_internal.h -- structures shared by the planner (fb_plan.cu) and the
// kernels (fb_kernels.cu).  Not part of the public C ABI.
#pragma once
#include <cuda.h>  // CUtensorMap (types only; the driver is reached through cudart)
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#define FB_MAX_STAGES 24
#define FB_MAX_PRIME 71  // largest prime done by a register butterfly

namespace fb {

// How one side (load or store) of a line kernel addresses memory.
// Line l is split as l0 = l % m0, t = l / m0, l1 = t % m1, l2 = t / m1; its
// base offset is l0*s0 + l1*s1 + l2*s2 elements and element i of the line is at
// base + i*es.  `vn`, `ves`, `vls`: element i of line l is present when
// i*ves + l0*vls < vn (absent loads read zero, absent stores are skipped);
// the same index selects the optional multiplier table `mul`.
struct LineIO {
  int64_t s0, s1, s2, es;
  int64_t vn, ves, vls;
  const void* mul;  // per-element multiplier (chirp) or null
  int mode;         // 0: line-major (a line's threads walk its elements),
                    // 1: element-major (threads walk the G lines of a block first)
  int count;        // elements touched per line (<= L)
};

// A stage program: Stockham passes with the given radices, the per-stage
// twiddle tables at tw + tw_off[s] (entries (r-1)*Ns + k = w_P^(r k),
// P = Ns*R, forward sign).
struct StageProg {
  int L;
  int nst;
  int radix[FB_MAX_STAGES];
  int tw_off[FB_MAX_STAGES];
  const void* tw;
};

struct LineArgs {
  const void* in;
  void* out;
  int64_t nlines, m0, m1;
  LineIO ld, st;
  StageProg prog;
  int dir1;             // direction of the first transform (-1 / +1)
  int dir2;             // direction of the second (only with mid)
  const void* mid;      // pointwise multiplier between the two transforms, or null
  int64_t mid_ls, mid_es;
  // twiddle on store: multiply element k of line l by w_N^(dir * lt * k) where
  // lt is the line's level-`tw_level` index (l0 or l1),
  // w_N^e = hi[e >> shift] * lo[e & (2^shift - 1)].
  int64_t tw_N;         // 0: none
  int tw_dir, tw_shift, tw_level;
  const void* tw_hi;
  const void* tw_lo;
  // or a full table (tw_tab != null, takes precedence): element i of line l
  // is multiplied by tw_tab[i*tw_es + lt*tw_ls] (conjugated when tw_dir > 0)
  const void* tw_tab;
  int64_t tw_es, tw_ls;
  int tw_on_load;       // 1: the twiddle multiplies element i of each line as
                        // it is loaded (before the transform), not on store
  int plain_io;         // 1: no presence window, no tables but tw_tab, and
                        // |strides| * L < 2^31 (the tile kernel's lean I/O)
  double scale;         // applied on store when != 1
  int G, T;             // lines per block, threads per line
  int Lpad;             // smem elements per line
  const void* prime_cs; // cos/sin tables of odd primes (see prime_table_offset)
  int* err;             // device flag: set to the radix when a program names one
                        // this kernel has no butterfly for (never traps)
  const void* tcb;      // tensor-core stage: B tables (forward, then backward)
  int st_stream;        // 1: no later pass of the plan reads the output; the
                        // specialised kernels store it evict-first
  uint64_t wait_ns;     // limit of a wait on the block's own asynchronous
                        // work (tensor-core products); 0: kWaitNsDefault
};

// Shared-memory pitch (elements) of the lines of a tile block.  A warp holds
// G lines x 32/G butterflies, and a 128-byte row of shared memory has
// S = 128/es element slots (16 for ComplexF32, 8 for ComplexF64), served to S
// consecutive lanes at a time.  Those lanes hit distinct slots when
// pitch = S/G (mod S) for G < S (lines interleave with the consecutive
// butterflies) and pitch = 1 (mod S) for G >= S (S lines side by side).
__host__ __device__ constexpr int tile_pitch(int lpad, int G, int es) {
  return lpad + ((((G >= 128 / es ? 1 : (128 / es) / G) - lpad) % (128 / es)) + (128 / es)) %
                    (128 / es);
}

// Longest line whose twiddle slice a tile block stages in shared memory.
constexpr int kStagedTwiddleMax = 1024;

// Arguments of the specialised direct-I/O kernel (fb_fast.cuh): `nlines`
// contiguous lines of length L, line l at in + l*idist / out + l*odist.
struct FastArgs {
  const void* in;
  void* out;
  int64_t nlines, idist, odist;
  const void* tw;
  const void* prime_cs;
  double scale;
  int G;
  // Grouped launch (ndesc > 0): the lines of ndesc requests in one launch.
  // Request r owns lines pre[r] .. pre[r+1]-1, its line l at
  // ins[r] + (l - pre[r])*idist and outs[r] + (l - pre[r])*odist; `in` and
  // `out` are unused.  The descriptor arrays live in device memory.
  int ndesc;
  const int64_t* pre;
  const void* const* ins;
  void* const* outs;
  int* err;  // device flag: kErrWaitTimeout when a bulk-copy wait gave up
  const void* tcb;  // tensor-core stage: B tables (forward, then backward)
  int st_stream;    // 1: store the output evict-first (see LineArgs::st_stream)
  uint64_t wait_ns; // limit of a wait on the block's own bulk copies or
                    // tensor-core products; 0: kWaitNsDefault
};

// Value of the kernel error flag when a wait on a bulk copy or on tensor-core
// products gave up; the kernel then stops early and leaves its output partial.
constexpr int kErrWaitTimeout = -1;
// Default limit of such a wait (ns).  After giving up, a block still waits up
// to this long (never less) for the copies and products it has in flight
// before it touches their shared or tensor memory again, frees it or exits.
constexpr uint64_t kWaitNsDefault = 1000000000ull;
// The limit a launch uses: fb_set_wait_limit's value, 0 for the default.
uint64_t wait_limit_ns();

// Arguments of the half-length real kernel (fast_real_kernel): `nlines`
// contiguous real lines of even length n = 2L.  rfft reads line l as L
// complex values (even samples real, odd ones imaginary) at in + l*idist
// reals, transforms them and splits the result into the n/2+1 outputs at
// out + l*odist complex values; brfft does the reverse (idist complex in,
// odist reals out).  FFTA src/plan.jl:398-442 (rfft) and :466-495 (brfft).
struct RealArgs {
  const void* in;
  void* out;
  int64_t nlines, idist, odist;
  const void* tw;        // stage twiddles of the length-L program
  const void* prime_cs;
  const void* wk;        // exp(-2 pi i k / n), k = 0..L/2, FP64-made, rounded once
  double scale;
  int G;
  int st_stream;
};

// Geometry of a tile pass whose loads are tensor copies (fast_tma_tile_kernel):
// tile k holds lines k*G .. k*G+G-1 (G divides the first batch level, so a
// tile's lines are neighbours in memory), brought into shared memory as
// `nbox` boxes of `boxr` elements x G lines.
struct TmaGeom {
  int nbox, boxr;      // boxes per tile along the line, elements per box
  int units;           // 8-byte units per element (1: ComplexF32, 2: ComplexF64)
  int nbuf;            // tile buffers in flight per block
  uint32_t buf_bytes;  // bytes per buffer (flat tile or padded lines; 1 KB multiple)
  int64_t ntiles;
};

// One specialised length: its radix program, threads per line, launcher and
// padded shared-memory elements per line.
struct FastFn {
  int L, T, nst;
  int radix[8];
  cudaError_t (*launch)(int dir, const FastArgs&, cudaStream_t);
  cudaError_t (*launch_tile)(const LineArgs&, cudaStream_t);
  size_t lpad;
  // persistent bulk-copy variant of `launch` (contiguous, 16-byte aligned
  // lines; see fast_stream_kernel), nullptr where the length has none
  cudaError_t (*launch_stream)(int dir, const FastArgs&, cudaStream_t);
  // the same kernels with the first radix-16 stage on the tensor cores
  // (split-BF16 GEMM, FP32 accumulation); nullptr where not available
  cudaError_t (*launch_tc)(int dir, const FastArgs&, cudaStream_t);
  cudaError_t (*launch_tile_tc)(const LineArgs&, cudaStream_t);
  // threads per block of launch_tile outside Bluestein (G * T at most)
  int tile_threads;
  // the lean tile kernel fed by tensor copies (persistent blocks, `nbuf`
  // tiles in flight); `tmap` is the CUtensorMap of the pass's input;
  // nullptr where the length has none
  cudaError_t (*launch_tile_tma)(const LineArgs&, const void* tmap, const TmaGeom&, cudaStream_t);
  // half-length real transform of lines of length 2L (dir -1: rfft, +1:
  // brfft); nullptr where the length has none
  cudaError_t (*launch_real)(int dir, const RealArgs&, cudaStream_t);
  // threads per block of launch_tile in Bluestein (MID) passes (G * T at most)
  int mid_threads;
};

// Bytes of one direction's B table of the tensor-core radix-16 stage.
constexpr int kTcTableBytesHost = 6144;
// The compiled specialised lengths of a type (dtype 0/1), in `parts` pieces.
int fast_table_parts();
const FastFn* fast_table(int dtype, int part, int* count);

// Set the message fb_last_error() returns on this thread.
void set_last_error(const std::string& msg);

// Details of the last failed launch of a specialised kernel ("" if none).
const char* last_launch_message();

// Offsets (in (cos,sin) pairs) of each odd prime's table inside prime_cs.
int prime_table_offset(int p);
int prime_table_total();

// Kernel launch entry points (fb_kernels.cu).  dtype: 0 = C32, 1 = C64.
cudaError_t launch_line(int dtype, int variant, const LineArgs& a, cudaStream_t s);
size_t line_smem_bytes(int dtype, const LineArgs& a);
// Work-descriptor launch of the generic kernel (see line_kernel_desc).
cudaError_t launch_desc(int dtype, int variant, const LineArgs* descs, const int64_t* bstart,
                        int ndesc, int64_t nblocks, int threads, size_t smem, cudaStream_t s);
int line_max_threads();
// variant bits: 1 = large register budget (32 values/thread), 2 = big primes
cudaError_t gen_stage_twiddles(int dtype, void* out, int R, int64_t Ns, cudaStream_t s);
// out[q] = exp(sign * 2 pi i * ((q*step) mod N) / N) for q < count, sign = -1
cudaError_t gen_roots(int dtype, void* out, int64_t N, int64_t step, int64_t count,
                      cudaStream_t s);
// Full twiddle table: out[i*n_ln + l] = exp(-2 pi i (i*l mod N)/N).
cudaError_t gen_tw_table(int dtype, void* out, int64_t N, int64_t n_el, int64_t n_ln,
                         cudaStream_t s);
// Bluestein chirp pieces for length N, pad M, direction dir (FFTA
// src/algos.jl:344-367: b[n] = exp(i pi sgn n^2 / N), sgn = -dir):
//   pre[n]  = conj(b[n])            n < N
//   post[n] = conj(b[n]) (scaled by 1/M when post_scale)  n < N
//   bext[m] = b[m] (m < N), b[M-m] at M-m (0 < m < N), 0 elsewhere
cudaError_t gen_chirp(int dtype, void* pre, void* post, void* bext_c64, int64_t N, int64_t M,
                      int dir, cudaStream_t s);
// Round a C64 array to the plan's type (copy for C64).
cudaError_t convert_c64(int dtype, void* dst, const void* src_c64, int64_t n, double scale,
                        cudaStream_t s);
cudaError_t gen_prime_tables(void* f32tab, void* f64tab, cudaStream_t s);

// The serving loop's resident kernel and its descriptor queue (fb_serve.cu).
struct PQueue;
enum { kPqStatOk = 0, kPqStatTimeout = 1, kPqStatBadProgram = 2 };
// Program id of contiguous lines of length L (16..4096, powers of two), or -1.
int pq_program_id(int dtype, int dir, int64_t L);
// Queue with its buffers; the kernel ends after `idle_ns` without new work.
cudaError_t pq_create(PQueue** q, uint64_t idle_ns);
void pq_destroy(PQueue* q);
// Register program `id` with its stage twiddle table and odd-prime table.
cudaError_t pq_set_program(PQueue* q, int id, const void* tw, const void* pcs);
bool pq_has_program(const PQueue* q, int id);
int64_t pq_slots();
// Append a request (returns its queue index); pq_publish makes the appended
// ones visible to the kernel; pq_kick launches the kernel if none is resident.
int64_t pq_push(PQueue* q, int prog, const void* in, void* out, int64_t batch, int64_t seq_add);
void pq_publish(PQueue* q);
cudaError_t pq_kick(PQueue* q);
bool pq_running(PQueue* q);
// 1 when request r has completed (time in globaltimer ns, status kPqStat*).
int pq_poll(PQueue* q, int64_t r, int64_t* t_ns, int32_t* status);
// The device globaltimer, read by a one-thread kernel on `s` into mapped
// host memory (device and host addresses of one int64).
cudaError_t pq_clock(cudaStream_t s, int64_t* host_mapped_dev, int64_t* host_mapped);

// Strided copy between two layouts of one array: element k (k_d < dims[d])
// moves from in + sum k_d*is[d] to out + sum k_d*os[d] (strides in elements
// of elem_bytes = 4, 8 or 16).
struct PermCopy {
  int rank;
  int64_t dims[8], is[8], os[8];
  int64_t count;
};
cudaError_t permute_copy(int elem_bytes, const void* in, void* out, const PermCopy& p,
                         cudaStream_t s);

// Real-transform helpers on contiguous column-major arrays (dtype 0: float /
// ComplexF32, 1: double / ComplexF64).
cudaError_t real_to_complex(int dtype, const void* in, void* out, int64_t count, cudaStream_t s);
cudaError_t complex_to_real(int dtype, const void* in, void* out, int64_t count, cudaStream_t s);
cudaError_t extract_half(int dtype, const void* in, void* out, int64_t pre, int64_t n, int64_t h,
                         int64_t post, cudaStream_t s);
cudaError_t herm_extend(int dtype, const void* x, void* z, int rank, const int64_t* dims, int r0,
                        int64_t h, uint32_t region, cudaStream_t s);

}  // namespace fb
