// fb_noalloc.cu -- a batched ComplexF32 transform that allocates no memory.
//
// Who needs it: callers that cannot call cudaMalloc at the point where they
// run a transform -- code running inside a memory pool or allocator callback,
// real-time or signal-processing loops that forbid allocation after start-up,
// and embedding hosts (plugins, firmware-style services) that hand the library
// only the input and output buffers.  The regular plans (fb_plan_create...)
// allocate their twiddle tables and scratch with cudaMalloc; this entry point
// instead runs the two-pass (four-step) schedule with its intermediate in a
// file-scope static __device__ array, and writes its twiddle tables into a
// second static array.  Both arrays exist once per GPU that loads the library
// and stay allocated until the process exits.
//
// Limits: n * batch <= FB_NOALLOC_MAX_ELEMS (4,194,304 complex values, i.e.
// 32 MiB of scratch), and n must be a product of 2s, 3s and 5s (the stage
// programs then need no odd-prime table).  Larger or other lengths are
// rejected with FB_ERR_ARGUMENT / FB_ERR_UNSUPPORTED.
//
// Sharing: every call on a device uses the same two arrays and leaves its
// contents behind.  Nothing in them has to start at zero: each call rewrites
// the tables it reads, and pass 1 writes every scratch element pass 2 reads.
// In place (in == out) is allowed: pass 1 reads all of the input into the
// scratch before pass 2, on the same stream, writes the output.
// Calls whose work overlaps on the GPU (different streams, or different host
// threads without ordering between them) race on the arrays and give wrong
// results; run them on one stream or otherwise serialise them.
//
// Set-up: the first call on a device looks up the arrays' device addresses
// (cudaGetSymbolAddress, with that device current).  Make that first call
// before any stream capture.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "fb_internal.h"
#include "fftab200.h"

namespace fb {

#define FB_NOALLOC_MAX_ELEMS (1 << 22)
#define FB_NOALLOC_TABLE_ELEMS (1 << 16)

// Host code may only take these arrays' device addresses through
// cudaGetSymbolAddress; their names are host-side stand-ins.
static __device__ __align__(256) float2 g_noalloc_scratch[FB_NOALLOC_MAX_ELEMS];
static __device__ __align__(256) float2 g_noalloc_tables[FB_NOALLOC_TABLE_ELEMS];

// Errors go to the library's per-thread message (fb_last_error).
static void noalloc_error(const std::string& msg) { set_last_error(msg); }

struct NoallocDev {
  bool ready = false;
  float2* scratch = nullptr;
  float2* tables = nullptr;
};
static std::mutex g_noalloc_mu;
static NoallocDev g_noalloc_dev[64];

// Radix program of a 2^a 3^b 5^c length, the same rule as the planner's.
static std::vector<int> noalloc_radices(int64_t L) {
  std::vector<int> r;
  int a = 0, b = 0;
  while (L % 2 == 0) {
    L /= 2;
    ++a;
  }
  const int q = a / 4, rem = a % 4;
  if (rem == 1 && q >= 1) {
    for (int i = 0; i < q - 1; ++i) r.push_back(16);
    r.push_back(8);
    r.push_back(4);
  } else {
    for (int i = 0; i < q; ++i) r.push_back(16);
    if (rem == 1) r.push_back(2);
    if (rem == 2) r.push_back(4);
    if (rem == 3) r.push_back(8);
  }
  while (L % 3 == 0) {
    L /= 3;
    ++b;
  }
  for (int i = 0; i < b / 2; ++i) r.push_back(9);
  if (b % 2) r.push_back(3);
  while (L % 5 == 0) {
    L /= 5;
    r.push_back(5);
  }
  return r;
}

static bool smooth235(int64_t n) {
  for (int p : {2, 3, 5})
    while (n % p == 0) n /= p;
  return n == 1;
}

// Threads per line for the generic line kernel with a 16-value register
// budget (variant 0), or 32 values (variant 1).
static bool noalloc_threads(int L, const std::vector<int>& rad, int* T, int* variant) {
  for (int cap : {16, 32}) {
    int tmin = 1;
    for (int R : rad) {
      const int um = R >= cap ? 1 : cap / R;
      tmin = std::max(tmin, (L / R + um - 1) / um);
    }
    if (tmin <= line_max_threads()) {
      int t = 1;
      if (tmin <= 32) {
        while (t < tmin) t <<= 1;
      } else {
        t = (tmin + 31) / 32 * 32;
      }
      *T = t;
      *variant = cap == 32 ? 1 : 0;
      return true;
    }
  }
  return false;
}

static int lpad_len(int L) {
  int lp = (L - 1) + ((L - 1) >> 4) + 1;
  if ((lp & 1) == 0) lp += 1;
  return lp;
}

// Stage-twiddle table of a radix program written at `dst`; returns entries.
static int64_t stage_tables(float2* dst, const std::vector<int>& rad, int* off, cudaStream_t s,
                            cudaError_t* err) {
  int64_t o = 0, Ns = 1;
  for (size_t i = 0; i < rad.size(); ++i) {
    off[i] = (int)o;
    if (*err == cudaSuccess) *err = gen_stage_twiddles(0, dst + o, rad[i], Ns, s);
    o += (int64_t)(rad[i] - 1) * Ns;
    Ns *= rad[i];
  }
  return o;
}

static int noalloc_run(const void* in, void* out, int64_t n, int64_t batch, int dir,
                       cudaStream_t stream) {
  if (n <= 0) {
    noalloc_error("Array length must be strictly positive");
    return FB_ERR_DIMENSION_MISMATCH;
  }
  if (batch < 0) {
    noalloc_error("fb_execute_noalloc_c32: batch must be >= 0, got " + std::to_string(batch));
    return FB_ERR_ARGUMENT;
  }
  if (dir != FB_FORWARD && dir != FB_BACKWARD) {
    noalloc_error("direction must be -1 or +1");
    return FB_ERR_ARGUMENT;
  }
  if (batch == 0) return FB_OK;
  if (n > FB_NOALLOC_MAX_ELEMS / batch) {
    noalloc_error("fb_execute_noalloc_c32: n*batch = " + std::to_string(n) + "*" +
                    std::to_string(batch) + " exceeds the static scratch of " +
                    std::to_string(FB_NOALLOC_MAX_ELEMS) + " complex values");
    return FB_ERR_ARGUMENT;
  }
  if (!smooth235(n)) {
    noalloc_error("fb_execute_noalloc_c32: length " + std::to_string(n) +
                    " is not a product of 2s, 3s and 5s");
    return FB_ERR_UNSUPPORTED;
  }
  if (!in || !out) {
    noalloc_error("null data pointer");
    return FB_ERR_ARGUMENT;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    noalloc_error(std::string("no usable CUDA device: ") + cudaGetErrorString(e));
    cudaGetLastError();
    return FB_ERR_CUDA;
  }
  if (dev >= 64) {
    noalloc_error("fb_execute_noalloc_c32: device index " + std::to_string(dev) +
                  " is beyond the 64 devices whose array addresses it caches");
    return FB_ERR_UNSUPPORTED;
  }
  NoallocDev d;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_dev[dev].ready) {
      void* ps = nullptr;
      void* pt = nullptr;
      e = cudaGetSymbolAddress(&ps, g_noalloc_scratch);
      if (e == cudaSuccess) e = cudaGetSymbolAddress(&pt, g_noalloc_tables);
      if (e != cudaSuccess) {
        noalloc_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        cudaGetLastError();
        return FB_ERR_CUDA;
      }
      g_noalloc_dev[dev].scratch = (float2*)ps;
      g_noalloc_dev[dev].tables = (float2*)pt;
      g_noalloc_dev[dev].ready = true;
    }
    d = g_noalloc_dev[dev];
  }
  // Balanced split n = N1 * N2 (N1 <= N2), both at most 16384 long.
  int64_t N1 = 1;
  for (int64_t f = 1; f * f <= n; ++f)
    if (n % f == 0 && n / f <= 16384) N1 = f;
  const int64_t N2 = n / N1;
  if (N2 > 16384) {
    noalloc_error("fb_execute_noalloc_c32: length " + std::to_string(n) + " has no split");
    return FB_ERR_UNSUPPORTED;
  }
  const std::vector<int> r1 = noalloc_radices(N1), r2 = noalloc_radices(N2);
  int T1, T2, v1, v2;
  if (!noalloc_threads((int)N1, r1, &T1, &v1) || !noalloc_threads((int)N2, r2, &T2, &v2) ||
      r1.size() > FB_MAX_STAGES || r2.size() > FB_MAX_STAGES) {
    noalloc_error("fb_execute_noalloc_c32: no stage program for length " + std::to_string(n));
    return FB_ERR_UNSUPPORTED;
  }
  // Tables in the static table array: stage twiddles of N1 and N2 (a program
  // of length L needs L - 1 entries), then the two-level roots of N (lo:
  // 2^shift entries, hi: ceil(N / 2^shift)).  Sized before anything is written.
  int shift = 0;
  while ((int64_t(1) << (2 * shift)) < n) ++shift;
  const int64_t lo_n = int64_t(1) << shift, hi_n = (n + lo_n - 1) / lo_n;
  if ((N1 - 1) + (N2 - 1) + lo_n + hi_n > FB_NOALLOC_TABLE_ELEMS) {
    noalloc_error("fb_execute_noalloc_c32: tables exceed the static table array");
    return FB_ERR_UNSUPPORTED;
  }
  e = cudaSuccess;
  LineArgs a1, a2;
  memset(&a1, 0, sizeof(a1));
  memset(&a2, 0, sizeof(a2));
  int64_t used = stage_tables(d.tables, r1, a1.prog.tw_off, stream, &e);
  float2* tw2 = d.tables + used;
  used += stage_tables(tw2, r2, a2.prog.tw_off, stream, &e);
  float2* lo = d.tables + used;
  float2* hi = lo + lo_n;
  if (e == cudaSuccess) e = gen_roots(0, lo, n, 1, lo_n, stream);
  if (e == cudaSuccess) e = gen_roots(0, hi, n, lo_n, hi_n, stream);
  // Pass 1: the N2 columns (stride N2) of every transform -> scratch, with
  // the twiddle w_N^(n2 k1) fused into the store.
  a1.in = in;
  a1.out = d.scratch;
  a1.nlines = N2 * batch;
  a1.m0 = N2;
  a1.m1 = batch;
  a1.ld = LineIO{1, n, 0, N2, INT64_MAX, 0, 0, nullptr, 1, (int)N1};
  a1.st = LineIO{1, n, 0, N2, INT64_MAX, 0, 0, nullptr, 1, (int)N1};
  a1.prog.L = (int)N1;
  a1.prog.nst = (int)r1.size();
  for (size_t i = 0; i < r1.size(); ++i) a1.prog.radix[i] = r1[i];
  a1.prog.tw = d.tables;
  a1.dir1 = a1.dir2 = dir;
  a1.tw_N = n;
  a1.tw_dir = dir;
  a1.tw_shift = shift;
  a1.tw_lo = lo;
  a1.tw_hi = hi;
  a1.scale = 1.0;
  a1.T = T1;
  a1.G = std::max(1, std::min(16, line_max_threads() / T1));
  while (a1.G & (a1.G - 1)) --a1.G;  // element-major tiles need a power of two
  a1.Lpad = lpad_len((int)N1);
  // Pass 2: the N1 rows (contiguous) of the scratch -> X[k1 + N1 k2].
  a2.in = d.scratch;
  a2.out = out;
  a2.nlines = N1 * batch;
  a2.m0 = N1;
  a2.m1 = batch;
  a2.ld = LineIO{N2, n, 0, 1, INT64_MAX, 0, 0, nullptr, 0, (int)N2};
  a2.st = LineIO{1, n, 0, N1, INT64_MAX, 0, 0, nullptr, 1, (int)N2};
  a2.prog.L = (int)N2;
  a2.prog.nst = (int)r2.size();
  for (size_t i = 0; i < r2.size(); ++i) a2.prog.radix[i] = r2[i];
  a2.prog.tw = tw2;
  a2.dir1 = a2.dir2 = dir;
  a2.scale = 1.0;
  a2.T = T2;
  a2.G = std::max(1, std::min(16, line_max_threads() / T2));
  while (a2.G & (a2.G - 1)) --a2.G;
  a2.Lpad = lpad_len((int)N2);
  for (LineArgs* a : {&a1, &a2})
    while (a->G > 1 && line_smem_bytes(0, *a) > 200 * 1024) a->G /= 2;
  if (e == cudaSuccess) e = launch_line(0, v1, a1, stream);
  if (e == cudaSuccess) e = launch_line(0, v2, a2, stream);
  if (e != cudaSuccess) {
    noalloc_error(std::string("fb_execute_noalloc_c32: ") + cudaGetErrorString(e));
    cudaGetLastError();
    return FB_ERR_CUDA;
  }
  set_last_error("");
  return FB_OK;
}

}  // namespace fb

extern "C" int fb_execute_noalloc_c32(const void* in, void* out, int64_t n, int64_t batch,
                                      int dir, void* stream) {
  return fb::noalloc_run(in, out, n, batch, dir, (cudaStream_t)stream);
}
