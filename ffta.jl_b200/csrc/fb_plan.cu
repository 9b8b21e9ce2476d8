// fb_plan.cu -- planner, executor and C ABI of libfftab200.so.
//
// FFTA.jl plans a transform by building a call graph (src/callgraph.jl:76-126)
// and runs it with recursive CPU kernels (src/algos.jl).  This planner keeps
// the same inputs and semantics -- length, direction, Bluestein cutoff,
// region -- and maps each transformed axis to a short sequence of line-kernel
// launches (fb_kernels.cu):
//   DIRECT  one kernel: the whole line in shared memory (lengths up to Lmax)
//   BLUE1   one kernel: Bluestein with the pad held in shared memory
//   FOUR    two kernels: N = N1*N2, each pass a DIRECT or BLUE1 line
//           transform, the twiddle fused into the second pass's loads (or,
//           over a contiguous batch, the first pass's stores)
//   BLUE3   three kernels: Bluestein whose pad M = M1*M2 is done four-step,
//           with the chirp spectrum multiply fused between the two halves
// The arithmetic of a length depends only on (length, type, direction,
// cutoff), never on batch or strides, so batched transforms and strided
// one-pass axes are bit-identical to single contiguous ones (long strided
// axes take a four-step split unless FB_FLAG_SAME_SCHEDULE_STRIDED is set).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <thread>
#include <cstdio>
#include <cstring>
#include <functional>
#include <deque>
#include <map>
#include <set>
#include <tuple>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "fb_internal.h"
#include "fftab200.h"

#define FB_VERSION "fftab200 0.1.0 (sm_100a)"

namespace fb {

static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }

// fb_set_wait_limit's value (0: the kernels' default limit).
static std::atomic<uint64_t> g_wait_ns{0};
uint64_t wait_limit_ns() { return g_wait_ns.load(std::memory_order_relaxed); }

struct FbError {
  int code;
  std::string msg;
};
[[noreturn]] static void fail(int code, const std::string& m) { throw FbError{code, m}; }
static void cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  cudaGetLastError();
  if (e == cudaErrorMemoryAllocation)
    fail(FB_ERR_OUT_OF_MEMORY, std::string(what) + ": out of device memory");
  fail(FB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ----------------------------------------------------------- device memory
// A cache of device blocks for plans that a serving loop makes and releases
// by the thousand: a released block goes back to a free list of its size
// class instead of to cudaFree, which waits for the whole device (every plan
// release would drain the GPU).  Blocks are reused only by plans made under
// the same cache, and the server releases only plans whose work has
// completed.  Beyond `cap` cached bytes the least recently freed blocks are
// given back with cudaFree, many at a time.
struct BlockCache {
  std::mutex mu_;
  std::map<size_t, std::set<void*>> free_;      // cached blocks per size class
  std::deque<std::pair<size_t, void*>> order_;  // frees, oldest first (may hold
                                                // entries of blocks reused since)
  size_t cached = 0, nblocks = 0, cap;
  explicit BlockCache(size_t c) : cap(c) {}
  static size_t round(size_t b) {
    if (b <= 4096) return 4096;
    if (b <= (size_t(2) << 20)) {
      size_t r = 4096;
      while (r < b) r *= 2;
      return r;
    }
    return (b + (size_t(2) << 20) - 1) / (size_t(2) << 20) * (size_t(2) << 20);
  }
  void* alloc(size_t b) {
    std::lock_guard<std::mutex> lk(mu_);
    const size_t r = round(b);
    auto it = free_.find(r);
    if (it != free_.end() && !it->second.empty()) {
      void* p = *it->second.begin();
      it->second.erase(it->second.begin());
      cached -= r;
      nblocks -= 1;
      return p;
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, r);
    if (e == cudaErrorMemoryAllocation && cached) {
      cudaGetLastError();
      trim_locked(0);  // give the cached blocks back and try once more
      e = cudaMalloc(&p, r);
    }
    cuda_check(e, "cudaMalloc");
    return p;
  }
  void release(void* p, size_t b) {
    std::lock_guard<std::mutex> lk(mu_);
    const size_t r = round(b);
    free_[r].insert(p);
    order_.emplace_back(r, p);
    cached += r;
    nblocks += 1;
    if (cached > cap) trim_locked(cap / 2);
    if (order_.size() > 4 * nblocks + 1024) {
      // drop the entries of blocks that were reused
      std::deque<std::pair<size_t, void*>> keep;
      for (auto& e : order_) {
        auto f = free_.find(e.first);
        if (f != free_.end() && f->second.count(e.second)) keep.push_back(e);
      }
      order_.swap(keep);
    }
  }
  void trim(size_t to) {
    std::lock_guard<std::mutex> lk(mu_);
    trim_locked(to);
  }
  void trim_locked(size_t to) {
    while (cached > to && !order_.empty()) {
      auto [r, p] = order_.front();
      order_.pop_front();
      auto f = free_.find(r);
      if (f == free_.end() || !f->second.erase(p)) continue;  // reused since
      cudaFree(p);
      cached -= r;
      nblocks -= 1;
    }
  }
  ~BlockCache() { trim(0); }
};
// The cache DevBufs made on this thread draw from (set by the server while it
// makes a plan), or null for plain cudaMalloc / cudaFree.
static thread_local BlockCache* g_block_cache = nullptr;
struct BlockCacheScope {
  BlockCache* saved;
  explicit BlockCacheScope(BlockCache* c) : saved(g_block_cache) { g_block_cache = c; }
  ~BlockCacheScope() { g_block_cache = saved; }
};

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  BlockCache* cache = nullptr;  // where the block goes back to
  DevBuf() = default;
  explicit DevBuf(size_t b) : bytes(b), cache(g_block_cache) {
    if (!b) return;
    if (cache)
      p = cache->alloc(b);
    else
      cuda_check(cudaMalloc(&p, b), "cudaMalloc");
  }
  ~DevBuf() {
    if (!p) return;
    if (cache)
      cache->release(p, bytes);
    else
      cudaFree(p);
  }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

// Internal plan flag (above the public FB_FLAG_* bits): make the plan without
// scratch buffers; its owner binds them (fb_plan_s::ext_s0/1) before use.
constexpr uint32_t kFlagNoScratch = 1u << 30;

// Per-device odd-prime cos/sin tables used by the register DFTs.
struct DeviceTables {
  void* f32 = nullptr;
  void* f64 = nullptr;
  int* err = nullptr;  // kernel error flag (see LineArgs::err)
  void* tc = nullptr;  // B tables of the tensor-core radix-16 stage (made on first use)
};
static std::mutex g_dev_mu;
static std::map<int, DeviceTables> g_dev_tables;

static const DeviceTables& device_tables(int dev) {
  std::lock_guard<std::mutex> lk(g_dev_mu);
  auto it = g_dev_tables.find(dev);
  if (it != g_dev_tables.end()) return it->second;
  DeviceTables t;
  const int total = prime_table_total();
  cuda_check(cudaMalloc(&t.f32, (size_t)total * 2 * sizeof(float)), "cudaMalloc");
  cuda_check(cudaMalloc(&t.f64, (size_t)total * 2 * sizeof(double)), "cudaMalloc");
  cuda_check(cudaMalloc(&t.err, sizeof(int)), "cudaMalloc");
  cuda_check(cudaMemset(t.err, 0, sizeof(int)), "cudaMemset");
  cuda_check(gen_prime_tables(t.f32, t.f64, 0), "prime tables");
  // table work runs on the legacy default stream; waiting for it alone (not
  // the whole device) keeps plan creation independent of a serving loop's
  // resident kernel on its non-blocking stream
  cuda_check(cudaStreamSynchronize(0), "prime tables");
  return g_dev_tables.emplace(dev, t).first->second;
}

// Round to nearest even FP32 -> BF16 (finite inputs).
static uint16_t bf16_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}
static double bf16_value(uint16_t b) {
  const uint32_t u = (uint32_t)b << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

// B operand of the tensor-core radix-16 stage for both directions (forward
// table, then backward): row o < 16 gives Re y_o = sum_n Re(F_on) re_n -
// Im(F_on) im_n, row 16+o gives Im y_o = sum_n Im(F_on) re_n + Re(F_on) im_n,
// F_on = exp(dir 2 pi i (o n mod 16) / 16); each entry split into three BF16
// terms (h, m, l: residuals of the FP64 value) in column blocks 0-31, 32-63,
// 64-95, stored in the K-major canonical shared-memory layout.
static const void* tc_tables(int dev) {
  static std::mutex mu;
  static std::map<int, void*> made;
  std::lock_guard<std::mutex> lk(mu);
  auto it = made.find(dev);
  if (it != made.end()) return it->second;
  const int K = 96;
  std::vector<uint16_t> host(2 * kTcTableBytesHost / 2, 0);
  // cos(pi m / 8) for m = 0..15 with exact zeros and ones
  auto cos8 = [](int m) -> double {
    m &= 15;
    if (m == 0) return 1.0;
    if (m == 8) return -1.0;
    if (m == 4 || m == 12) return 0.0;
    return std::cos(M_PI * m / 8.0);
  };
  for (int d = 0; d < 2; ++d) {
    const int dir = d == 0 ? -1 : 1;
    uint16_t* tab = host.data() + d * (kTcTableBytesHost / 2);
    for (int o = 0; o < 32; ++o) {
      const int k = o & 15;
      for (int c = 0; c < 32; ++c) {
        const int n = c & 15;
        const int m = (k * n) & 15;
        const double fr = cos8(m), fi = dir * cos8(m + 12);  // sin(pi m/8) = cos(pi (m-4)/8)
        double val;
        if (o < 16)
          val = c < 16 ? fr : -fi;
        else
          val = c < 16 ? fi : fr;
        const uint16_t h = bf16_bits((float)val);
        const double r1 = val - bf16_value(h);
        const uint16_t mm = bf16_bits((float)r1);
        const double r2 = r1 - bf16_value(mm);
        const uint16_t l = bf16_bits((float)r2);
        const uint16_t parts[3] = {h, mm, l};
        for (int blk = 0; blk < 3; ++blk) {
          const int kk = blk * 32 + c;
          const size_t off = (size_t)((o >> 3) * (K / 8) * 128 + (kk >> 3) * 128 + (o & 7) * 16 +
                                      (kk & 7) * 2);
          tab[off / 2] = parts[blk];
        }
      }
    }
  }
  void* p = nullptr;
  cuda_check(cudaMalloc(&p, 2 * kTcTableBytesHost), "cudaMalloc");
  cuda_check(cudaMemcpy(p, host.data(), 2 * kTcTableBytesHost, cudaMemcpyHostToDevice),
             "tensor-core tables");
  made[dev] = p;
  return p;
}

// ------------------------------------------------------------ arithmetic
static int64_t ipow2_ceil(int64_t v) {
  int64_t p = 1;
  while (p < v) p <<= 1;
  return p;
}
static std::vector<std::pair<int64_t, int>> factorize(int64_t n) {
  std::vector<std::pair<int64_t, int>> f;
  for (int64_t d = 2; d * d <= n; d += (d == 2 ? 1 : 2)) {
    int c = 0;
    while (n % d == 0) {
      n /= d;
      ++c;
    }
    if (c) f.push_back({d, c});
  }
  if (n > 1) f.push_back({n, 1});
  return f;
}
static bool is_prime(int64_t n) {
  if (n < 2) return false;
  auto f = factorize(n);
  return f.size() == 1 && f[0].second == 1;
}
static int elem_bytes(int dtype) { return dtype == FB_C32 ? 8 : 16; }
static int64_t lmax_for(int dtype) { return dtype == FB_C32 ? 16384 : 8192; }
// Longest contiguous ComplexF32 line done in one pass by a specialised kernel
// (the line and its padding fill up to 167 KB of shared memory).
static const int64_t kLongDirectMax = 19683;

// ------------------------------------------------------ line transforms
// A transform of one line done by one kernel.
struct LineX {
  int kind = 0;  // 0 direct, 1 Bluestein in shared memory
  int64_t n = 0; // logical length
  int L = 0;     // shared-memory transform length (n, or the Bluestein pad)
  std::vector<int> radices;
  int variant = 0;
  int T = 1;
  std::vector<int> tw_off;
  int64_t tw_count = 0;
};

static int um_for(int R, int cap) { return R >= cap ? 1 : cap / R; }

// Radix program for a length whose prime factors are all <= FB_MAX_PRIME:
// powers of two as radix 16 with an 8, 4 or 2 (8*4 in place of 16*2), then
// powers of three as radix 9 with a final 3, then fives and the odd primes
// in ascending order.  The program depends on the length alone -- unless a
// plan made with FB_FLAG_TUNE_RADIX has a tuned program for the length (the
// override below, consulted while such a plan is built).
static thread_local const std::map<int64_t, std::vector<int>>* g_radix_override = nullptr;
// Tuned programs per (type, direction) and length: chosen by fb_plan_autotune
// for plans with FB_FLAG_TUNE_RADIX, used by later such plans.
static std::mutex g_radix_mu;
static std::map<std::pair<int, int>, std::map<int64_t, std::vector<int>>> g_radix_tuned;
// Sets the override for the plan being built and restores the caller's.
struct RadixScope {
  const std::map<int64_t, std::vector<int>>* saved;
  std::map<int64_t, std::vector<int>> own;
  RadixScope(int dtype, int dir, uint32_t flags, const std::map<int64_t, std::vector<int>>* force)
      : saved(g_radix_override) {
    if (force) {
      own = *force;
      g_radix_override = &own;
    } else if (flags & FB_FLAG_TUNE_RADIX) {
      std::lock_guard<std::mutex> lk(g_radix_mu);
      own = g_radix_tuned[{dtype, dir}];
      g_radix_override = &own;
    } else {
      g_radix_override = nullptr;
    }
  }
  ~RadixScope() { g_radix_override = saved; }
};
// An explicit override for the next create_plan on this thread (the tuner's
// candidates).
static thread_local const std::map<int64_t, std::vector<int>>* g_radix_force = nullptr;
static std::vector<int> default_radix_program(int64_t L);
static std::vector<int> radix_program(int64_t L) {
  if (g_radix_override) {
    auto it = g_radix_override->find(L);
    if (it != g_radix_override->end()) return it->second;
  }
  return default_radix_program(L);
}
static std::vector<int> default_radix_program(int64_t L) {
  std::vector<int> r;
  int a = 0;
  while (L % 2 == 0) {
    L /= 2;
    ++a;
  }
  int q = a / 4, rem = a % 4;
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
  int b = 0;
  while (L % 3 == 0) {
    L /= 3;
    ++b;
  }
  for (int i = 0; i < b / 2; ++i) r.push_back(9);
  if (b % 2) r.push_back(3);
  for (auto& pe : factorize(L))
    for (int i = 0; i < pe.second; ++i) r.push_back((int)pe.first);
  return r;
}

// Can `n` be a DIRECT line (all factors by register butterflies) under the
// Bluestein cutoff?  FFTA sends a prime p >= 5 to Bluestein when
// p >= cutoff; 2 and 3 always take the radix kernels (src/callgraph.jl:86-100).
static bool direct_ok(int64_t n, int64_t cutoff, int dtype) {
  if (n < 1 || n > lmax_for(dtype)) return false;
  for (auto& pe : factorize(n)) {
    const int64_t p = pe.first;
    if (p == 2 || p == 3) continue;
    if (p > FB_MAX_PRIME || p >= cutoff) return false;
  }
  return true;
}

// Threads per line and the kernel variant for a radix program.
static bool pick_threads(int L, const std::vector<int>& rad, int* T_out, int* variant_out) {
  bool big = false;
  for (int R : rad) big |= R > 16;
  const int caps[2] = {16, 32};
  for (int ci = 0; ci < 2; ++ci) {
    const int cap = caps[ci];
    if (big && cap != 16) break;
    int tmin = 1;
    for (int R : rad) {
      const int nb = L / R;
      const int need = (nb + um_for(R, cap) - 1) / um_for(R, cap);
      tmin = std::max(tmin, need);
    }
    if (tmin <= line_max_threads()) {
      int T;
      if (tmin <= 32) {
        T = 1;
        while (T < tmin) T <<= 1;
      } else {
        T = (tmin + 31) / 32 * 32;
      }
      *T_out = T;
      *variant_out = (cap == 32 ? 1 : 0) | (big ? 2 : 0);
      return true;
    }
  }
  return false;
}

static bool make_direct(int64_t n, int64_t cutoff, int dtype, LineX* x) {
  if (!direct_ok(n, cutoff, dtype)) return false;
  LineX r;
  r.kind = 0;
  r.n = n;
  r.L = (int)n;
  r.radices = radix_program(n);
  if (!pick_threads(r.L, r.radices, &r.T, &r.variant)) return false;
  *x = r;
  return true;
}

// Lengths with a compile-time-specialised kernel that a Bluestein pad may
// take: 2^a, 2^a*3, 2^a*9 and 3^b, ascending.  FFTA pads to nextpow2(2n-1)
// (src/algos.jl:345); any length >= 2n-1 gives the same transform, and the
// smallest of these is up to 1.9x shorter (e.g. 9216 instead of 16384 for
// n = 4099).
static const std::vector<int64_t>& pad_lengths() {
  static const std::vector<int64_t> v = [] {
    std::vector<int64_t> c;
    for (int64_t p = 16; p <= 16384; p *= 2) c.push_back(p);
    for (int64_t p = 48; p <= 12288; p *= 2) c.push_back(p);
    for (int64_t p = 144; p <= 9216; p *= 2) c.push_back(p);
    for (int64_t p = 27; p <= 6561; p *= 3) c.push_back(p);
    std::sort(c.begin(), c.end());
    return c;
  }();
  return v;
}

// Smallest pad >= need that one kernel transforms (at most lmax), or 0.
static int64_t blue_pad(int64_t need, int64_t lmax, int dtype) {
  for (int64_t c : pad_lengths()) {
    if (c < need) continue;
    if (c > lmax) break;
    LineX t;
    if (make_direct(c, 1 << 30, dtype, &t)) return c;
  }
  return 0;
}

static bool make_blue1(int64_t n, int dtype, LineX* x) {
  const int64_t M = blue_pad(2 * n - 1, lmax_for(dtype), dtype);
  if (M == 0) return false;
  LineX r;
  if (!make_direct(M, 1 << 30, dtype, &r)) return false;
  r.kind = 1;
  r.n = n;
  *x = r;
  return true;
}

// One line transform of length n if one kernel can do it.
static bool make_line(int64_t n, int64_t cutoff, int dtype, LineX* x) {
  if (make_direct(n, cutoff, dtype, x)) return true;
  // Lengths with a factor that needs Bluestein, and primes >= cutoff.
  return make_blue1(n, dtype, x);
}

// Relative cost of one line: work ~ L (log2 L + 4).  With `weighted` (splits
// of lengths that are not powers of two) the work is scaled by how close the
// length's kernels come to copy bandwidth: powers of two from 256 (radix-16
// programs) 1.0, lines shorter than 16 2.0, others 1.25 -- measured on the
// four-step splits of 27648: 1024 x 27 in 0.182 ms, 144 x 192 in 0.226 ms.
// Cost factor of a four-step factor that has no compiled kernel.
static const double kGenericPassCost = 3.0;

static double line_cost(const LineX& x, bool weighted = false) {
  const double L = x.L;
  const double c = L * (std::log2(std::max(2.0, L)) + 4.0);
  double eff = 1.0;
  if (weighted)
    eff = (x.L >= 256 && (x.L & (x.L - 1)) == 0) ? 1.0 : (x.L < 16 ? 2.0 : 1.25);
  return x.kind == 0 ? c * eff : 2.0 * c + 2.0 * L;
}

// ------------------------------------------------------------------ plan
enum BufId { B_IN = 0, B_OUT = 1, B_S0 = 2, B_S1 = 3 };

struct Pass {
  LineArgs a;
  int variant = 0;
  int src = B_IN, dst = B_OUT;
  std::string what;
  const FastFn* fast = nullptr;    // specialised direct-I/O kernel, if any
  FastArgs fa;
  const FastFn* staged = nullptr;  // specialised tile kernel (strided lines, fused I/O)
  int stream = 0;                  // 1: run `fast` as its persistent bulk-copy kernel
  int tc = 0;                      // 1: first radix-16 stage on the tensor cores
  int tma = 0;                     // 1: run `staged` fed by tensor copies (geometry tg)
  TmaGeom tg;
  // the tensor map of the last input this pass ran on, with the box it was
  // encoded for (re-encoded when the input address, the lines per tile or
  // the box rows change -- the autotuner may change the lines per tile)
  CUtensorMap tmap;
  const void* tmap_in = nullptr;
  int tmap_G = 0, tmap_boxr = 0;
};

// The specialised kernel for a radix program, if one is compiled.
static const FastFn* find_fast(int dtype, int L, const std::vector<int>& radices) {
  for (int part = 0; part < fast_table_parts(); ++part) {
    int cnt = 0;
    const FastFn* t = fast_table(dtype, part, &cnt);
    for (int i = 0; i < cnt; ++i) {
      if (t[i].L != L || t[i].nst != (int)radices.size()) continue;
      bool same = true;
      for (int s = 0; s < t[i].nst; ++s) same &= t[i].radix[s] == radices[s];
      if (same) return &t[i];
    }
  }
  return nullptr;
}


struct BDim {
  int64_t n, is, os;
};

struct Axis {
  int64_t n = 0;
  std::string kind;
  std::vector<Pass> passes;
  std::vector<BDim> outer;  // batch dims looped on the host
};

}  // namespace fb

struct fb_plan_s {
  int dtype = 0, dir = -1, device = 0;
  uint32_t flags = 0;  // FB_FLAG_GENERIC_ONLY, FB_FLAG_SAME_SCHEDULE_STRIDED
  int64_t cutoff = 73;
  double scale = 1.0;
  int rank = 0;
  std::vector<int64_t> dims, istrides, ostrides;
  std::vector<int> region;  // 0-based, ascending
  std::vector<fb::Axis> axes;
  std::vector<std::unique_ptr<fb::DevBuf>> bufs;  // tables
  size_t scratch_elems = 0;
  std::unique_ptr<fb::DevBuf> scratch0, scratch1;
  // plans made without scratch (kFlagNoScratch, the server's): the buffers
  // their passes use, bound by the owner before each execution
  bool need_s1 = false;
  void* ext_s0 = nullptr;
  void* ext_s1 = nullptr;
  // host-execution staging
  std::unique_ptr<fb::DevBuf> hin, hout;
  // grouped execution: device copy of the request descriptors
  std::unique_ptr<fb::DevBuf> desc;
  // real transforms (rfft: 1, brfft: 2): a complex plan over the full dims run
  // in place on zbuf, between a conversion in and an extraction out
  int real_kind = 0;
  std::unique_ptr<fb_plan_s> cplan;
  std::unique_ptr<fb::DevBuf> zbuf;
  // half-length real path (even length along the contiguous first dim):
  // the real kernel's length-L program and arguments; cplan then covers the
  // other region dims of the half array (or is null)
  const fb::FastFn* rfn = nullptr;
  fb::RealArgs ra;
  // a strided region dim: the copies that bring it to the front and back
  // (real array and half array) and the contiguous buffers between them
  fb::PermCopy perm_full, perm_half;
  std::unique_ptr<fb::DevBuf> zr, zc;
  int r0 = 0;
  int64_t rh = 0;
  uint32_t region_mask = 0;
  // pipelined host execution: plans for one chunk and the last one, device
  // slots, streams and events
  std::unique_ptr<fb_plan_s> chunk_plan, tail_plan;
  int64_t chunk = 0;
  std::vector<std::unique_ptr<fb::DevBuf>> slots;
  cudaStream_t pstream[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t pev[3][3] = {};
  ~fb_plan_s() {
    for (auto s : pstream)
      if (s) cudaStreamDestroy(s);
    for (auto& row : pev)
      for (auto e : row)
        if (e) cudaEventDestroy(e);
  }
  int64_t in_span = 0, out_span = 0;
  size_t table_bytes = 0;
};

namespace fb {

static int pick_G(const fb_plan_s* P, int L, int T, int Lpad, bool elem_major, int64_t nlines);
static void apply_tuning(fb_plan_s* P);
static void plan_tma(const fb_plan_s* P, Pass& p);
static int lpad_for(int L);

// Lines per block of the tile kernel: by its threads (FastFn::tile_threads),
// and by shared memory -- 100 KB for ComplexF32 (two blocks per SM), up to
// 220 KB where a block takes more than 512 threads (one block per SM anyway);
// ComplexF64 tiles run faster at about 40 KB (more resident blocks per SM,
// measured).
static int tile_thread_cap(const FastFn* ff) { return std::max(1, ff->tile_threads / ff->T); }
static int tile_smem_cap(const FastFn* ff, int es) {
  const size_t budget = es == 8 ? (ff->tile_threads > 512 ? 220 : 100) * 1024 : 40 * 1024;
  return (int)std::max<size_t>(1, budget / ((size_t)(ff->lpad + 15) * es + 32));
}

// Switch a generic pass to the compile-time tile kernel of its length when
// one is compiled (same arithmetic, direct HBM I/O, lines fastest across a
// warp).  Bluestein passes need the forward-then-inverse order it implements.
static void use_tile(const fb_plan_s* P, Pass& p, const std::vector<int>& radices) {
  // lean I/O when nothing but strides, a full twiddle table and a scale is
  // needed and every 32-bit offset fits.  Set for generic passes too: a
  // four-step twiddle on the loads of a lean pass is tw_elem's product in
  // both kernels, so they keep equal bits.
  {
    const int64_t L = p.a.prog.L;
    const bool small = std::llabs(p.a.ld.es) * L < (int64_t(1) << 31) &&
                       std::llabs(p.a.st.es) * L < (int64_t(1) << 31) &&
                       (!p.a.tw_tab || (L * p.a.tw_es + p.a.tw_ls * (int64_t)p.a.nlines) < (int64_t(1) << 31));
    p.a.plain_io = !p.a.mid && !p.a.ld.mul && !p.a.st.mul && p.a.ld.vn == INT64_MAX &&
                   p.a.st.vn == INT64_MAX && !(p.a.tw_N && !p.a.tw_tab) && small &&
                   p.a.ld.count == L && p.a.st.count == L;
  }
  if (P->flags & 1) return;
  const FastFn* ff = find_fast(P->dtype, p.a.prog.L, radices);
  if (!ff || (int)ff->lpad != p.a.Lpad) return;
  if (p.a.mid && (p.a.dir1 > 0 || p.a.dir2 < 0)) return;
  const int es = elem_bytes(P->dtype);
  const int T = ff->T;
  const int thr_cap = tile_thread_cap(ff), smem_cap = tile_smem_cap(ff, es);
  const bool em = p.a.ld.mode == 1 || p.a.st.mode == 1;
  // strided tiles: as many neighbouring lines as the block allows (longer
  // contiguous runs per DRAM page); contiguous lines: 128-thread blocks
  const int want = em ? thr_cap : std::max(1, 128 / T);
  int G = std::min(std::min(thr_cap, smem_cap), want);
  // ComplexF64 strided tiles of long lines: up to 4 lines (80 KB) rather
  // than the 40 KB budget's 2 (four-step columns of 1024: 0.37 -> 0.33 ms
  // per N = 2^20 x 16 step, autotuned); a lean pass that also loads the
  // four-step twiddle takes half the lines (its table loads add latency
  // per line: N = 2^20 C32 pass 2 and the short rows of 27648, 19683)
  if (em && es == 16 && G < 4) {
    const int g80 = (int)((80 * 1024) / ((size_t)(ff->lpad + 15) * es + 32));
    G = std::max(G, std::min(std::min(4, thr_cap), g80));
  }
  if (em && p.a.tw_on_load && p.a.plain_io && G >= 4) G /= 2;
  if (p.a.mid) G = std::min(G, std::max(1, ff->mid_threads / T));
  const int64_t nl = std::max<int64_t>(1, p.a.nlines);
  while (G > 1 && G / 2 >= nl) G /= 2;
  // lines contiguous on load: at least about four blocks per SM when the
  // batch is small (strided loads keep their width for long DRAM runs)
  if (p.a.ld.mode == 0)
    while (G > 1 && nl / G < 4 * 148) G /= 2;
  p.staged = ff;
  p.a.T = T;
  p.a.G = std::max(1, G);
  if ((P->flags & FB_FLAG_TENSOR_STAGE) && ff->launch_tile_tc && p.a.plain_io) {
    // 512 threads per block: four 128-row tiles of the stage's GEMM
    p.tc = 1;
    p.a.G = 512 / T;
    p.a.tcb = tc_tables(P->device);
  }
  p.what += "[tile T=" + std::to_string(T) + " G=" + std::to_string(p.a.G) + "]";
  plan_tma(P, p);
}

// Tensor-copy geometry of a lean tile pass with G lines per tile, or false
// when the pass cannot take tensor copies: its lines must be neighbours in
// memory (element-major loads, line stride 1) and G must divide the first
// batch level (a tile never straddles it), the rows of a box must cover
// whole 32-byte sectors and 16-byte units, and two tiles must fit in shared
// memory.  Shared memory per block: up to ~110 KB (two blocks per SM) when
// two or three buffers fit there, else up to ~220 KB (one block per SM).
static bool tma_geometry(const fb_plan_s* P, const Pass& p, const LineArgs& a, TmaGeom* g) {
  const FastFn* ff = p.staged;
  const int G = a.G;
  if (!ff || !ff->launch_tile_tma || p.tc || !a.plain_io || a.mid) return false;
  if (a.ld.mode != 1 || a.ld.s0 != 1 || G < 2 || G * ff->T > ff->tile_threads) return false;
  const int es = elem_bytes(P->dtype);
  const int L = a.prog.L;
  if (a.m0 % G || a.nlines % G || G * es < 32) return false;
  const int64_t m2 = a.nlines / std::max<int64_t>(1, a.m0 * a.m1);
  if (a.m0 * a.m1 * m2 != a.nlines) return false;
  for (int64_t st : {a.ld.es, a.ld.s1, a.ld.s2})
    if ((st * es) % 16 || std::llabs(st) * es >= (int64_t(1) << 39)) return false;
  if (a.m0 * (es / 8) >= (int64_t(1) << 31) || a.m1 >= (int64_t(1) << 31) || m2 >= (int64_t(1) << 31))
    return false;
  // boxes of at most 256 elements that split the line evenly, each landing
  // 128-byte aligned
  int nbox = (L + 255) / 256;
  while (nbox <= L && (L % nbox || ((size_t)(L / nbox) * G * es) % 128)) ++nbox;
  if (nbox > L || nbox > 64) return false;
  const int boxr = L / nbox;
  const size_t flat = (size_t)L * G * es;
  const size_t padded = (size_t)G * tile_pitch(lpad_for(L), G, es) * es;
  const size_t buf = (std::max(flat, padded) + 1023) / 1024 * 1024;
  // two tiles per block: one computing, one landing (measured: a third
  // buffer costs more in resident blocks than it gains)
  const int nbuf = 2;
  if (nbuf * buf > 220 * 1024) return false;
  g->nbox = nbox;
  g->boxr = boxr;
  g->units = es / 8;
  g->nbuf = nbuf;
  g->buf_bytes = (uint32_t)buf;
  g->ntiles = a.nlines / G;
  return true;
}

// FB_FLAG_TMA: switch a lean tile pass to tensor-copy loads where it
// qualifies, with the lines per tile that leave the most warps resident per
// SM (two tile buffers per block; ties: the wider rows).  Opt-in: on the
// four-step and strided-axis passes measured here the thread-loaded tile
// kernel, with two blocks of 512 threads per SM, was faster.
static void plan_tma(const fb_plan_s* P, Pass& p) {
  if (!(P->flags & FB_FLAG_TMA) || !p.staged) return;
  const int es = elem_bytes(P->dtype);
  int bestG = 0;
  double bw = 0;
  for (int G = 128 / es; G * es >= 32; G /= 2) {
    TmaGeom g;
    LineArgs ag = p.a;
    ag.G = G;
    if (!tma_geometry(P, p, ag, &g)) continue;
    const int thr = G * p.staged->T;
    const int blocks = std::min(std::min((int)((227 * 1024) / (g.nbuf * g.buf_bytes + 256)),
                                         2048 / thr),
                                65536 / (thr * 64));
    const double w = (double)blocks * thr / 32 + G * 1e-3;
    if (w > bw) {
      bw = w;
      bestG = G;
    }
  }
  if (!bestG) return;
  TmaGeom g;
  LineArgs ag = p.a;
  ag.G = bestG;
  tma_geometry(P, p, ag, &g);
  p.tma = 1;
  p.tg = g;
  p.a.G = bestG;
  p.what += "<tma G=" + std::to_string(bestG) + " bufs=" + std::to_string(g.nbuf) + ">";
}

// CUtensorMap of a tensor-copy pass over the input `in` (4-D: lines in
// 8-byte units, elements, the two batch levels) with boxes of G lines x
// g.boxr elements: the box the kernel's copies and byte counts assume.
static bool encode_tma(const fb_plan_s* P, Pass& p, const void* in, int G, const TmaGeom& g) {
  typedef CUresult (*EncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                               const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                               const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                               CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static EncodeFn encode = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &qr) ==
            cudaSuccess &&
        qr == cudaDriverEntryPointSuccess)
      encode = (EncodeFn)fn;
    cudaGetLastError();
  });
  if (!encode || reinterpret_cast<uintptr_t>(in) % 16) return false;
  if (p.tmap_in == in && p.tmap_G == G && p.tmap_boxr == g.boxr) return true;
  const LineArgs& a = p.a;
  const int es = elem_bytes(P->dtype);
  const int64_t m2 = a.nlines / (a.m0 * a.m1);
  const cuuint64_t row = (cuuint64_t)(a.ld.es * es);
  const cuuint64_t dims[4] = {(cuuint64_t)(a.m0 * (es / 8)), (cuuint64_t)a.prog.L,
                              (cuuint64_t)a.m1, (cuuint64_t)m2};
  // strides of extent-1 levels are never used; give them a valid value
  const cuuint64_t s1 = a.m1 > 1 ? (cuuint64_t)(a.ld.s1 * es) : row * a.prog.L;
  const cuuint64_t s2 = m2 > 1 ? (cuuint64_t)(a.ld.s2 * es) : s1 * a.m1;
  const cuuint64_t strides[3] = {row, s1, s2};
  const cuuint32_t box[4] = {(cuuint32_t)(G * (es / 8)), (cuuint32_t)g.boxr, 1, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r =
      encode(&p.tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<void*>(in), dims, strides,
             box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    p.tmap_in = nullptr;
    return false;
  }
  p.tmap_in = in;
  p.tmap_G = G;
  p.tmap_boxr = g.boxr;
  return true;
}

static void* alloc_table(fb_plan_s* P, size_t bytes) {
  P->bufs.emplace_back(new DevBuf(bytes));
  P->table_bytes += bytes;
  return P->bufs.back()->p;
}

static void fill_prog(fb_plan_s* P, LineX& x, StageProg* prog) {
  if ((int)x.radices.size() > FB_MAX_STAGES) fail(FB_ERR_UNSUPPORTED, "too many stages");
  // stage twiddle table: stage s has (R-1)*Ns entries
  int64_t off = 0, Ns = 1;
  x.tw_off.clear();
  for (int R : x.radices) {
    x.tw_off.push_back((int)off);
    off += (int64_t)(R - 1) * Ns;
    Ns *= R;
  }
  x.tw_count = off;
  void* tw = nullptr;
  if (off > 0) {
    tw = alloc_table(P, (size_t)off * elem_bytes(P->dtype));
    Ns = 1;
    for (size_t s = 0; s < x.radices.size(); ++s) {
      const int R = x.radices[s];
      cuda_check(gen_stage_twiddles(P->dtype, (char*)tw + (size_t)x.tw_off[s] * elem_bytes(P->dtype),
                                    R, Ns, 0),
                 "stage twiddles");
      Ns *= R;
    }
  }
  memset(prog, 0, sizeof(*prog));
  prog->L = x.L;
  prog->nst = (int)x.radices.size();
  for (size_t s = 0; s < x.radices.size(); ++s) {
    prog->radix[s] = x.radices[s];
    prog->tw_off[s] = x.tw_off[s];
  }
  prog->tw = tw;
}

static fb_plan_s* create_plan(int dtype, int dir, int rank, const int64_t* dims,
                              const int64_t* istrides, const int64_t* ostrides,
                              const std::vector<int>& region, int64_t cutoff,
                              uint32_t flags = 0);
static void execute_plan(fb_plan_s* P, const void* in, void* out, cudaStream_t s,
                         int64_t nb = -1);

// Chirp spectrum FFT_M(b_ext), forward, computed in FP64 by a C64 plan and
// rounded to the plan type, optionally scaled.
// The chirp spectrum FFT(b_ext) of length M.  With M1 > 0 (three-pass
// Bluestein, M = M1*M2) it is stored transposed, entry k1*M2 + k2 holding
// spectrum element k1 + M1*k2: the middle pass multiplies row k1 by elements
// k2 = 0..M2-1, which are then contiguous instead of M1 entries apart.
static void* chirp_spectrum(fb_plan_s* P, int64_t N, int64_t M, double scale, int64_t M1 = 0) {
  DevBuf bext((size_t)M * 16), spec((size_t)M * 16);
  cuda_check(gen_chirp(P->dtype, nullptr, nullptr, bext.p, N, M, P->dir, 0), "chirp");
  std::vector<int> reg{0};
  int64_t d[1] = {M}, st[1] = {1};
  std::unique_ptr<fb_plan_s> sub(create_plan(FB_C64, FB_FORWARD, 1, d, st, st, reg, 1 << 30));
  execute_plan(sub.get(), bext.p, spec.p, 0);
  const void* src = spec.p;
  if (M1 > 0) {
    PermCopy pc;
    memset(&pc, 0, sizeof(pc));
    pc.rank = 2;
    pc.dims[0] = M / M1;  // k2
    pc.dims[1] = M1;      // k1
    pc.is[0] = M1;
    pc.is[1] = 1;
    pc.os[0] = 1;
    pc.os[1] = M / M1;
    pc.count = M;
    cuda_check(permute_copy(16, spec.p, bext.p, pc, 0), "chirp spectrum layout");
    src = bext.p;
  }
  void* mid = alloc_table(P, (size_t)M * elem_bytes(P->dtype));
  cuda_check(convert_c64(P->dtype, mid, src, M, scale, 0), "chirp spectrum");
  cuda_check(cudaStreamSynchronize(0), "chirp spectrum");
  return mid;
}

// Tables of a Bluestein line: pre = conj(b), post = conj(b)/M, mid = FFT(b_ext).
static void blue_tables(fb_plan_s* P, int64_t N, int64_t M, void** pre, void** post, void** mid) {
  *pre = alloc_table(P, (size_t)N * elem_bytes(P->dtype));
  *post = alloc_table(P, (size_t)N * elem_bytes(P->dtype));
  cuda_check(gen_chirp(P->dtype, *pre, *post, nullptr, N, M, P->dir, 0), "chirp");
  *mid = chirp_spectrum(P, N, M, 1.0);
}

static int pick_G(const fb_plan_s* P, int L, int T, int Lpad, bool elem_major, int64_t nlines) {
  const int es = elem_bytes(P->dtype);
  const int thr_cap = std::max(1, std::max(line_max_threads(), T) / T);
  const size_t line_bytes = (size_t)Lpad * es + 24;
  const size_t budget = 100 * 1024;
  int g_smem = (int)std::max<size_t>(1, budget / line_bytes);
  int want = std::max(1, 256 / T);
  if (elem_major) want = std::max(want, es == 8 ? 16 : 8);
  int G = std::min(std::min(thr_cap, g_smem), want);
  int64_t nl = std::max<int64_t>(1, nlines);
  while (G > 1 && G / 2 >= nl) G /= 2;
  if (elem_major) {
    int p = 1;
    while (p * 2 <= G) p *= 2;
    G = p;
  }
  (void)L;
  return std::max(1, G);
}

static int lpad_for(int L) {
  int lp = (L - 1) + ((L - 1) >> 4) + 1;
  if (lp < 1) lp = 1;
  if ((lp & 1) == 0) lp += 1;
  return lp;
}

static LineIO io_plain(int64_t s0, int64_t s1, int64_t s2, int64_t es, int count) {
  LineIO io;
  memset(&io, 0, sizeof(io));
  io.s0 = s0;
  io.s1 = s1;
  io.s2 = s2;
  io.es = es;
  io.vn = INT64_MAX;
  io.ves = 0;
  io.vls = 0;
  io.mul = nullptr;
  io.mode = 0;
  io.count = count;
  return io;
}

// Base LineArgs for a line transform `x` applied to `nlines` lines.
static void base_args(fb_plan_s* P, LineX& x, LineArgs* a, int dir) {
  memset(a, 0, sizeof(*a));
  fill_prog(P, x, &a->prog);
  a->dir1 = dir;
  a->dir2 = dir;
  a->scale = 1.0;
  a->T = x.T;
  a->Lpad = lpad_for(x.L);
  const DeviceTables& dt = device_tables(P->device);
  a->prime_cs = P->dtype == FB_C32 ? dt.f32 : dt.f64;
  a->err = dt.err;
  a->m0 = 1;
  a->m1 = 1;
}

// Make `x` a Bluestein line on top of base args: pre on load, convolution,
// post on store.  `vls_ld/vls_st`, `ves` describe the element index as in LineIO.
static void attach_blue(fb_plan_s* P, const LineX& x, LineArgs* a) {
  void *pre, *post, *mid;
  blue_tables(P, x.n, x.L, &pre, &post, &mid);
  a->ld.mul = pre;
  a->ld.vn = x.n;
  a->ld.ves = 1;
  a->ld.vls = 0;
  a->ld.count = (int)x.n;
  a->st.mul = post;
  a->st.vn = x.n;
  a->st.ves = 1;
  a->st.vls = 0;
  a->st.count = (int)x.n;
  a->mid = mid;
  a->mid_ls = 0;
  a->mid_es = 1;
  a->dir1 = FB_FORWARD;
  a->dir2 = FB_BACKWARD;
}

// Two-level root tables for w_N^e, e < N: hi[e >> shift] * lo[e & mask].
// Four-step twiddle w_N^(e) for the elements i < n_el of the lines with
// twiddle index lt < n_ln, e = i*lt.  Up to kFullTwiddle entries a full table
// (one coalesced load per element: entry i*n_ln + lt) is made; beyond, the
// two-level tables (hi[e >> shift] * lo[e & mask]).
static const int64_t kFullTwiddle = int64_t(1) << 23;
static const int64_t kBlueFullTwiddle = int64_t(1) << 18;

static void attach_twiddle(fb_plan_s* P, LineArgs* a, int64_t N, int dir, int64_t n_el,
                           int64_t n_ln, bool roots_only = false) {
  a->tw_dir = dir;
  if (n_el * n_ln <= kFullTwiddle && !roots_only) {
    void* tab = alloc_table(P, (size_t)(n_el * n_ln) * elem_bytes(P->dtype));
    cuda_check(gen_tw_table(P->dtype, tab, N, n_el, n_ln, 0), "twiddle table");
    a->tw_tab = tab;
    a->tw_es = n_ln;
    a->tw_ls = 1;
    a->tw_N = 0;
    return;
  }
  int shift = 0;
  while ((int64_t(1) << (2 * shift)) < N) ++shift;  // 2^shift >= sqrt(N)
  const int64_t lo_n = int64_t(1) << shift;
  const int64_t hi_n = (N + lo_n - 1) / lo_n;
  void* lo = alloc_table(P, (size_t)lo_n * elem_bytes(P->dtype));
  void* hi = alloc_table(P, (size_t)hi_n * elem_bytes(P->dtype));
  cuda_check(gen_roots(P->dtype, lo, N, 1, lo_n, 0), "roots");
  cuda_check(gen_roots(P->dtype, hi, N, lo_n, hi_n, 0), "roots");
  a->tw_N = N;
  a->tw_dir = dir;
  a->tw_shift = shift;
  a->tw_lo = lo;
  a->tw_hi = hi;
}

// Collapse batch dims that are contiguous in both input and output, drop
// extent-1 dims, and order them by input stride.
static std::vector<BDim> normalize_batch(std::vector<BDim> bd) {
  std::vector<BDim> v;
  for (auto& b : bd)
    if (b.n != 1) v.push_back(b);
  std::sort(v.begin(), v.end(), [](const BDim& x, const BDim& y) {
    return std::llabs(x.is) < std::llabs(y.is);
  });
  bool merged = true;
  while (merged) {
    merged = false;
    for (size_t i = 0; i + 1 < v.size() && !merged; ++i) {
      BDim& a = v[i];
      BDim& b = v[i + 1];
      if (a.is * a.n == b.is && a.os * a.n == b.os) {
        a.n *= b.n;
        v.erase(v.begin() + i + 1);
        merged = true;
      }
    }
  }
  return v;
}

static int64_t prod_n(const std::vector<BDim>& v, size_t from, size_t to) {
  int64_t p = 1;
  for (size_t i = from; i < to && i < v.size(); ++i) p *= v[i].n;
  return p;
}

// Split batch dims into kernel levels (up to `kl`) and host-looped dims.
static void split_levels(const std::vector<BDim>& bd, size_t kl, std::vector<BDim>* inner,
                         std::vector<BDim>* outer) {
  inner->clear();
  outer->clear();
  for (size_t i = 0; i < bd.size(); ++i) (i < kl ? inner : outer)->push_back(bd[i]);
}

static int64_t level_n(const std::vector<BDim>& v, size_t i) { return i < v.size() ? v[i].n : 1; }
static int64_t level_is(const std::vector<BDim>& v, size_t i) { return i < v.size() ? v[i].is : 0; }
static int64_t level_os(const std::vector<BDim>& v, size_t i) { return i < v.size() ? v[i].os : 0; }

static Axis plan_direct_axis(fb_plan_s* P, int64_t n, LineX& x, int64_t is, int64_t os,
                             const std::vector<BDim>& bd, int src, int dst) {
  Axis ax;
  ax.n = n;
  std::vector<BDim> inner;
  split_levels(bd, 3, &inner, &ax.outer);
  Pass p;
  base_args(P, x, &p.a, P->dir);
  p.variant = x.variant;
  p.src = src;
  p.dst = dst;
  const int64_t nl = prod_n(inner, 0, 3);
  p.a.nlines = nl;
  p.a.m0 = level_n(inner, 0);
  p.a.m1 = level_n(inner, 1);
  p.a.ld = io_plain(level_is(inner, 0), level_is(inner, 1), level_is(inner, 2), is, (int)x.L);
  p.a.st = io_plain(level_os(inner, 0), level_os(inner, 1), level_os(inner, 2), os, (int)x.L);
  if (x.kind == 1) attach_blue(P, x, &p.a);
  const bool ld_em = is != 1 && !inner.empty() && inner[0].is == 1;
  const bool st_em = os != 1 && !inner.empty() && inner[0].os == 1;
  p.a.ld.mode = ld_em ? 1 : 0;
  p.a.st.mode = st_em ? 1 : 0;
  p.a.G = pick_G(P, x.L, x.T, p.a.Lpad, ld_em || st_em, nl);
  ax.kind = x.kind == 0 ? "DIRECT" : "BLUE1";
  // Contiguous lines at one batch stride: the specialised direct-I/O kernel.
  const FastFn* ff = nullptr;
  if (x.kind == 0 && is == 1 && os == 1 && inner.size() <= 1 && !(P->flags & 1))
    ff = find_fast(P->dtype, x.L, x.radices);
  if (ff) {
    p.fast = ff;
    memset(&p.fa, 0, sizeof(p.fa));
    p.fa.nlines = nl;
    p.fa.idist = level_is(inner, 0);
    p.fa.odist = level_os(inner, 0);
    p.fa.tw = p.a.prog.tw;
    p.fa.prime_cs = p.a.prime_cs;
    p.fa.scale = 1.0;
    const int es = elem_bytes(P->dtype);
    // one line per block once a line fills a warp: measured faster than
    // packing several lines into 256-thread blocks (fewer lines wait at each
    // stage barrier); shorter lines share a block up to a warp's worth
    int G = std::max(1, 32 / ff->T);
    while (G > 1 && (size_t)G * ff->lpad * es > 100 * 1024) G /= 2;
    while (G > 1 && G / 2 >= nl) G /= 2;
    p.fa.G = G;
    p.fa.err = p.a.err;
    if ((P->flags & FB_FLAG_TENSOR_STAGE) && ff->launch_tc) {
      p.tc = 1;
      p.fa.G = 1;
      p.fa.tcb = tc_tables(P->device);
    }
    // the persistent bulk-copy variant measured slower than one line per
    // block (it holds fewer warps per SM): used on request or when tuned
    p.stream = ff->launch_stream && (P->flags & FB_FLAG_STREAM) ? 1 : 0;
    std::ostringstream w;
    w << "FAST(L=" << x.L << " radices=";
    for (size_t i = 0; i < x.radices.size(); ++i) w << (i ? "x" : "") << x.radices[i];
    w << " T=" << ff->T << " G=" << G << ")";
    p.what = w.str();
    ax.passes.push_back(p);
    return ax;
  }
  std::ostringstream w;
  w << ax.kind << "(L=" << x.L << " radices=";
  for (size_t i = 0; i < x.radices.size(); ++i) w << (i ? "x" : "") << x.radices[i];
  w << " T=" << x.T << " G=" << p.a.G << " var=" << x.variant << ")";
  p.what = w.str();
  use_tile(P, p, x.radices);
  ax.passes.push_back(p);
  return ax;
}

// Four-step N = N1*N2: pass 1 transforms the N2 strided columns (length N1)
// into scratch with the twiddle w_N^(n2 k1) fused; pass 2 transforms the N1
// rows (length N2) and writes X[k1 + N1 k2].
//
// Line order.  For an axis whose elements are contiguous (is == 1) the lines
// of a pass are ordered (n2 or k1, batch...): neighbouring lines are
// neighbouring in memory.  For a strided axis whose first batch dim is
// contiguous (the columns of a 2-D array) they are ordered (batch0, n2 or
// k1, batch1) instead, the scratch keeps batch0 fastest, and the twiddle's
// line factor is the level-1 index -- again neighbouring lines are
// neighbouring in memory, so both passes move long contiguous runs.
//
// L2 residency.  With contiguous axes the batch is cut into chunks whose
// scratch (N * chunk elements, at most kL2Chunk bytes) stays in L2 between
// pass 1 and pass 2; the chunks run one after the other (host loop).
static const size_t kL2Chunk = 64u << 20;

static Axis plan_four_axis(fb_plan_s* P, int64_t N, int64_t N1, int64_t N2, LineX& x1, LineX& x2,
                           int64_t is, int64_t os, const std::vector<BDim>& bd, int src, int dst) {
  Axis ax;
  ax.n = N;
  ax.kind = "FOUR";
  std::vector<BDim> inner;
  split_levels(bd, 2, &inner, &ax.outer);
  const bool tmode = is != 1 && !inner.empty() && inner[0].is == 1 && inner[0].os == 1 &&
                     inner[0].n > 1;
  const int es = elem_bytes(P->dtype);
  if (!tmode && !inner.empty()) {
    // chunk the first batch dim so that N * chunk elements fit kL2Chunk
    const int64_t B0 = inner[0].n;
    const int64_t per = std::max<int64_t>(1, (int64_t)(kL2Chunk / ((size_t)N * es)));
    if (B0 > per) {
      int64_t chunk = 1;
      for (int64_t c = per; c >= 1; --c)
        if (B0 % c == 0) {
          chunk = c;
          break;
        }
      if (chunk * 4 >= per) {  // only when the chunk is not tiny
        ax.outer.insert(ax.outer.begin(),
                        BDim{B0 / chunk, chunk * inner[0].is, chunk * inner[0].os});
        inner[0].n = chunk;
        ax.kind = "FOUR/L2";
      }
    }
  }
  const int64_t B = prod_n(inner, 0, 2), B0 = level_n(inner, 0), B1 = level_n(inner, 1);
  P->scratch_elems = std::max<size_t>(P->scratch_elems, (size_t)(N * B));
  Pass p1, p2;
  base_args(P, x1, &p1.a, P->dir);
  base_args(P, x2, &p2.a, P->dir);
  p1.variant = x1.variant;
  p2.variant = x2.variant;
  p1.src = src;
  p1.dst = B_S0;
  p2.src = B_S0;
  p2.dst = dst;
  p1.a.nlines = N2 * B;
  p2.a.nlines = N1 * B;
  if (!tmode) {
    // lines (n2, b0, b1); scratch S[b*N + k1*N2 + n2], b = b0 + B0*b1
    p1.a.m0 = N2;
    p1.a.m1 = B0;
    p1.a.ld = io_plain(is, level_is(inner, 0), level_is(inner, 1), N2 * is, x1.L);
    p1.a.st = io_plain(1, N, B0 * N, N2, x1.L);
    p1.a.ld.mode = is == 1 ? 1 : 0;
    p1.a.st.mode = 1;
    // lines (k1, b0, b1)
    p2.a.m0 = N1;
    p2.a.m1 = B0;
    p2.a.ld = io_plain(N2, N, B0 * N, 1, x2.L);
    p2.a.st = io_plain(os, level_os(inner, 0), level_os(inner, 1), N1 * os, x2.L);
    p2.a.ld.mode = 0;
    p2.a.st.mode = os == 1 ? 1 : 0;
  } else {
    // lines (b0, n2, b1); scratch S[b0 + B0*(k1*N2 + n2) + B0*N*b1]
    p1.a.m0 = B0;
    p1.a.m1 = N2;
    p1.a.ld = io_plain(1, is, level_is(inner, 1), N2 * is, x1.L);
    p1.a.st = io_plain(1, B0, B0 * N, B0 * N2, x1.L);
    p1.a.ld.mode = 1;
    p1.a.st.mode = 1;
    // lines (b0, k1, b1)
    p2.a.m0 = B0;
    p2.a.m1 = N1;
    p2.a.ld = io_plain(1, B0 * N2, B0 * N, B0, x2.L);
    p2.a.st = io_plain(1, os, level_os(inner, 1), N1 * os, x2.L);
    p2.a.ld.mode = 1;
    p2.a.st.mode = 1;
    (void)B1;
  }
  if (x1.kind == 1) attach_blue(P, x1, &p1.a);
  if (x2.kind == 1) attach_blue(P, x2, &p2.a);
  // the twiddle w_N^(n2 k1) multiplies the columns' outputs; with a full
  // table it is applied as pass 2 loads them (element n2 of line k1), so its
  // table loads issue with the data loads
  if ((int64_t)N <= kFullTwiddle && x2.kind == 0 && !tmode) {
    attach_twiddle(P, &p2.a, N, P->dir, N2, N1);
    p2.a.tw_on_load = 1;
    p2.a.tw_level = tmode ? 1 : 0;
  } else {
    attach_twiddle(P, &p1.a, N, P->dir, N1, N2);
    p1.a.tw_level = tmode ? 1 : 0;
  }
  p1.a.G = pick_G(P, x1.L, x1.T, p1.a.Lpad, true, p1.a.nlines);
  p2.a.G = pick_G(P, x2.L, x2.T, p2.a.Lpad, p2.a.ld.mode == 1 || p2.a.st.mode == 1,
                  p2.a.nlines);
  std::ostringstream w1, w2;
  w1 << "FOUR" << (tmode ? "T" : "") << ".1(N1=" << N1 << (x1.kind ? " blue" : "")
     << " L=" << x1.L << " T=" << x1.T << " G=" << p1.a.G << ")";
  w2 << "FOUR" << (tmode ? "T" : "") << ".2(N2=" << N2 << (x2.kind ? " blue" : "")
     << " L=" << x2.L << " T=" << x2.T << " G=" << p2.a.G << ")";
  p1.what = w1.str();
  p2.what = w2.str();
  use_tile(P, p1, x1.radices);
  use_tile(P, p2, x2.radices);
  ax.passes.push_back(p1);
  ax.passes.push_back(p2);
  return ax;
}

// Bluestein with the pad M = M1*M2 done four-step in three passes:
//  1. a = x conj(b) (zero beyond N), FFT over n1 (length M1), twiddle, -> S0
//  2. FFT over n2 (M2), times FFT(b_ext), inverse FFT over k2, twiddle, -> S1
//  3. inverse FFT over k1 (M1), times conj(b)/M, store n < N.
static Axis plan_blue3_axis(fb_plan_s* P, int64_t N, int64_t is, int64_t os,
                            const std::vector<BDim>& bd, int src, int dst) {
  // pad M = M1*M2 >= 2N-1: the smallest product of two specialised lengths
  // in [16, 4096] (ties: the more balanced), else FFTA's power of two split
  // in balanced halves
  int64_t M1 = 0, M2 = 0;
  {
    const int64_t need = 2 * N - 1;
    int64_t best = 0;
    double bal = 0;
    for (int64_t a : pad_lengths()) {
      if (a > 4096) break;
      for (int64_t b : pad_lengths()) {
        if (b > 4096) break;
        if (a * b < need) continue;
        const double r = std::fabs(std::log((double)a / (double)b));
        if (best == 0 || a * b < best || (a * b == best && r < bal)) {
          best = a * b;
          bal = r;
          M1 = a;
          M2 = b;
        }
        break;  // larger b only grows the product
      }
    }
    LineX t1, t2;
    if (best == 0 || !make_direct(M1, 1 << 30, P->dtype, &t1) ||
        !make_direct(M2, 1 << 30, P->dtype, &t2)) {
      const int64_t Mp = ipow2_ceil(need);
      int lg = 0;
      while ((int64_t(1) << lg) < Mp) ++lg;
      M1 = int64_t(1) << (lg / 2);
      M2 = Mp / M1;
    }
  }
  const int64_t M = M1 * M2;
  LineX x1, x2;
  if (!make_direct(M1, 1 << 30, P->dtype, &x1) || !make_direct(M2, 1 << 30, P->dtype, &x2))
    fail(FB_ERR_UNSUPPORTED, "length " + std::to_string(N) + " is beyond this build's schedules");
  Axis ax;
  ax.n = N;
  ax.kind = "BLUE3";
  std::vector<BDim> inner;
  split_levels(bd, 2, &inner, &ax.outer);
  if (!inner.empty()) {
    // as in the four-step: the batch in chunks whose scratch (M * chunk
    // elements per buffer) is at most kL2Chunk, one after the other, so the
    // scratch stays bounded (and in L2 between the passes); chunks of up to
    // 2^24 pad elements measured no faster on configuration-5 requests
    const int64_t B0c = inner[0].n;
    const int64_t per =
        std::max<int64_t>(1, (int64_t)(kL2Chunk / ((size_t)M * elem_bytes(P->dtype))));
    if (B0c > per) {
      int64_t chunk = 1;
      for (int64_t c = per; c >= 1; --c)
        if (B0c % c == 0) {
          chunk = c;
          break;
        }
      if (chunk * 4 >= per) {
        ax.outer.insert(ax.outer.begin(),
                        BDim{B0c / chunk, chunk * inner[0].is, chunk * inner[0].os});
        inner[0].n = chunk;
        ax.kind = "BLUE3/L2";
      }
    }
  }
  const int64_t B = prod_n(inner, 0, 2), B0 = level_n(inner, 0);
  P->scratch_elems = std::max<size_t>(P->scratch_elems, (size_t)(M * B));
  void* pre = alloc_table(P, (size_t)N * elem_bytes(P->dtype));
  void* post = alloc_table(P, (size_t)N * elem_bytes(P->dtype));
  cuda_check(gen_chirp(P->dtype, pre, post, nullptr, N, M, P->dir, 0), "chirp");
  // pass 1
  Pass p1;
  base_args(P, x1, &p1.a, FB_FORWARD);
  p1.variant = x1.variant;
  p1.src = src;
  p1.dst = B_S0;
  p1.a.nlines = M2 * B;
  p1.a.m0 = M2;
  p1.a.m1 = B0;
  p1.a.ld = io_plain(is, level_is(inner, 0), level_is(inner, 1), M2 * is, (int)M1);
  p1.a.ld.mul = pre;
  p1.a.ld.vn = N;
  p1.a.ld.ves = M2;
  p1.a.ld.vls = 1;
  p1.a.st = io_plain(1, M, B0 * M, M2, (int)M1);
  // Pads above kBlueFullTwiddle take their twiddles from two small root
  // tables on the passes' stores: a full table would be read from HBM as
  // often as the data itself when the batch is small.
  const bool full_tw = M <= kBlueFullTwiddle;
  if (!full_tw) attach_twiddle(P, &p1.a, M, FB_FORWARD, M1, M2, true);
  p1.a.ld.mode = is == 1 ? 1 : 0;
  p1.a.st.mode = 1;
  p1.a.G = pick_G(P, x1.L, x1.T, p1.a.Lpad, true, p1.a.nlines);
  // pass 2
  Pass p2;
  base_args(P, x2, &p2.a, FB_FORWARD);
  p2.variant = x2.variant;
  p2.src = B_S0;
  p2.dst = B_S1;
  p2.a.nlines = M1 * B;
  p2.a.m0 = M1;
  p2.a.m1 = B0;
  p2.a.ld = io_plain(M2, M, B0 * M, 1, (int)M2);
  p2.a.st = io_plain(1, M, B0 * M, M1, (int)M2);
  p2.a.mid = pre;  // placeholder until the spectrum is made below (never read)
  p2.a.mid_ls = 1;
  p2.a.mid_es = M1;
  p2.a.dir1 = FB_FORWARD;
  p2.a.dir2 = FB_BACKWARD;
  if (full_tw) {
    // pass 1's twiddle w_M^(n2 k1), applied as pass 2 loads (element n2 of line k1)
    attach_twiddle(P, &p2.a, M, FB_FORWARD, M2, M1);
    p2.a.tw_on_load = 1;
  } else {
    attach_twiddle(P, &p2.a, M, FB_BACKWARD, M2, M1, true);
  }
  p2.a.ld.mode = 0;
  p2.a.st.mode = 1;
  p2.a.G = pick_G(P, x2.L, x2.T, p2.a.Lpad, true, p2.a.nlines);
  // pass 3
  Pass p3;
  base_args(P, x1, &p3.a, FB_BACKWARD);
  p3.variant = x1.variant;
  p3.src = B_S1;
  p3.dst = dst;
  p3.a.nlines = M2 * B;
  p3.a.m0 = M2;
  p3.a.m1 = B0;
  p3.a.ld = io_plain(M1, M, B0 * M, 1, (int)M1);
  p3.a.st = io_plain(os, level_os(inner, 0), level_os(inner, 1), M2 * os, (int)M1);
  p3.a.st.mul = post;
  p3.a.st.vn = N;
  p3.a.st.ves = M2;
  p3.a.st.vls = 1;
  p3.a.ld.mode = 0;
  p3.a.st.mode = os == 1 ? 1 : 0;
  if (full_tw) {
    // the conjugate twiddle of pass 2's outputs, applied as pass 3 loads them
    // (element k1 of line m2)
    attach_twiddle(P, &p3.a, M, FB_BACKWARD, M1, M2);
    p3.a.tw_on_load = 1;
  }
  p3.a.G = pick_G(P, x1.L, x1.T, p3.a.Lpad, p3.a.st.mode == 1, p3.a.nlines);
  std::ostringstream w;
  w << "BLUE3(N=" << N << " M=" << M1 << "x" << M2 << ")";
  p1.what = w.str() + ".1";
  p2.what = w.str() + ".2";
  p3.what = w.str() + ".3";
  use_tile(P, p1, x1.radices);
  use_tile(P, p2, x2.radices);
  use_tile(P, p3, x1.radices);
  // The chirp spectrum in the layout the middle pass reads fastest.  With
  // one line per block the threads of a warp walk a row's elements, so the
  // rows are stored contiguous (transposed); with several lines per block
  // neighbouring lanes hold neighbouring rows at the same element, which
  // the natural order already puts side by side.  Measured on one B200:
  // 1000003 x 1 (one line per block) 0.116 -> 0.101 ms transposed, and
  // 65537 x 16 (nine lines per block) 0.096 -> 0.099 ms, so it keeps the
  // natural order.  Either layout gives the same bits.
  const bool rows = p2.staged && p2.a.G == 1;
  p2.a.mid = chirp_spectrum(P, N, M, 1.0, rows ? M1 : 0);
  p2.a.mid_ls = rows ? M2 : 1;
  p2.a.mid_es = rows ? 1 : M1;
  ax.passes.push_back(p1);
  ax.passes.push_back(p2);
  ax.passes.push_back(p3);
  return ax;
}

static Axis plan_axis(fb_plan_s* P, int64_t n, int64_t is, int64_t os, std::vector<BDim> bd,
                      int src, int dst) {
  if (n <= 0) fail(FB_ERR_DIMENSION_MISMATCH, "Array length must be strictly positive");
  bd = normalize_batch(bd);
  LineX x;
  // A strided axis whose neighbouring lines are neighbours in memory: one
  // pass holds only as many lines as fit a block, so a long line gives short
  // contiguous runs per row.  The tile kernel of a compiled length keeps one
  // pass while its block covers a whole 32-byte sector per row (measured: one
  // pass is 10-34 % faster than the split there, and slower below); other
  // lengths want 128-byte runs.  Shorter runs prefer a four-step split whose
  // passes hold many lines (FOURT order, see plan_four_axis).
  const bool strided = is != 1 && !bd.empty() && bd[0].is == 1 && bd[0].os == 1 && bd[0].n > 1;
  bool prefer_split = false;
  if (strided && make_direct(n, P->cutoff, P->dtype, &x)) {
    const int es = elem_bytes(P->dtype);
    const FastFn* ff = (P->flags & FB_FLAG_GENERIC_ONLY) ? nullptr
                                                          : find_fast(P->dtype, x.L, x.radices);
    int lines = std::min(16, std::max(1, (int)((100 * 1024) / ((size_t)lpad_for(x.L) * es))));
    int need = 128;
    if (ff && (int)ff->lpad == lpad_for(x.L) && x.kind == 0) {
      lines = std::min(tile_thread_cap(ff), tile_smem_cap(ff, es));
      need = 32;
    }
    prefer_split = (int64_t)lines * es < need && !(P->flags & FB_FLAG_SAME_SCHEDULE_STRIDED);
  }
  if (!prefer_split && make_direct(n, P->cutoff, P->dtype, &x))
    return plan_direct_axis(P, n, x, is, os, bd, src, dst);
  // Bluestein for a prime in one kernel when its pad fits.
  if (is_prime(n) && make_blue1(n, P->dtype, &x))
    return plan_direct_axis(P, n, x, is, os, bd, src, dst);
  // Contiguous ComplexF32 lines beyond the generic kernel's limit that still
  // fit one SM's shared memory: one pass on their specialised kernel.
  if (P->dtype == FB_C32 && n > lmax_for(FB_C32) && n <= kLongDirectMax && is == 1 && os == 1 &&
      bd.size() <= 1 && !(P->flags & FB_FLAG_GENERIC_ONLY)) {
    LineX lx;
    lx.kind = 0;
    lx.n = n;
    lx.L = (int)n;
    lx.radices = radix_program(n);
    const FastFn* ff = find_fast(P->dtype, lx.L, lx.radices);
    if (ff && ff->launch) {
      lx.T = ff->T;
      lx.variant = 0;
      return plan_direct_axis(P, n, lx, is, os, bd, src, dst);
    }
  }
  // Four-step over the cheapest split into two one-kernel line transforms.
  double best = 1e300;
  int64_t bN1 = 0;
  LineX b1, b2;
  for (int64_t N1 = 2; N1 * N1 <= n; ++N1) {
    if (n % N1) continue;
    const int64_t cand[2] = {N1, n / N1};
    for (int o = 0; o < 2; ++o) {
      const int64_t a = cand[o], b = n / a;
      LineX xa, xb;
      if (!make_line(a, P->cutoff, P->dtype, &xa) || !make_line(b, P->cutoff, P->dtype, &xb)) continue;
      if (prefer_split && (xa.kind != 0 || xb.kind != 0)) continue;
      const bool weighted = (n & (n - 1)) != 0;
      // a factor without a compiled kernel runs on the generic one, about
      // three times slower per element (measured on configuration-5
      // lengths: 200-600 GB/s against 1300-1900 GB/s); decided without
      // FB_FLAG_GENERIC_ONLY so that such plans keep the same split
      const auto gen = [&](const LineX& x) {
        return x.kind == 0 && !find_fast(P->dtype, x.L, x.radices) ? kGenericPassCost : 1.0;
      };
      double c = line_cost(xa, weighted) * gen(xa) * (double)b +
                 line_cost(xb, weighted) * gen(xb) * (double)a;
      // prefer balanced direct splits on ties, and the power-of-two factor
      // as the first pass (the strided columns)
      c *= 1.0 + 1e-9 * std::fabs(std::log((double)a) - std::log((double)b));
      if ((a & (a - 1)) == 0 && (b & (b - 1)) != 0) c *= 1.0 - 1e-6;
      // few neighbouring columns per transform (a short second factor) keep
      // the first pass's tiles narrow: 27648 = 27 x 1024 measured 0.141 ms
      // against 0.161 ms for 1024 x 27 (C32, 606 columns)
      if (is == 1 && b < 128 && a > b) c *= 1.25;
      if (c < best) {
        best = c;
        bN1 = a;
        b1 = xa;
        b2 = xb;
      }
    }
  }
  if (bN1) return plan_four_axis(P, n, bN1, n / bN1, b1, b2, is, os, bd, src, dst);
  if (prefer_split && make_direct(n, P->cutoff, P->dtype, &x))
    return plan_direct_axis(P, n, x, is, os, bd, src, dst);
  return plan_blue3_axis(P, n, is, os, bd, src, dst);
}

static fb_plan_s* create_plan(int dtype, int dir, int rank, const int64_t* dims,
                              const int64_t* istrides, const int64_t* ostrides,
                              const std::vector<int>& region, int64_t cutoff, uint32_t flags) {
  if (dtype != FB_C32 && dtype != FB_C64)
    fail(FB_ERR_ARGUMENT, "element type must be ComplexF32 or ComplexF64");
  if (dir != FB_FORWARD && dir != FB_BACKWARD) fail(FB_ERR_ARGUMENT, "direction must be -1 or +1");
  if (rank < 1) fail(FB_ERR_DIMENSION_MISMATCH, "array must have at least one dimension");
  // radix programs: tuned ones for FB_FLAG_TUNE_RADIX plans, the tuner's
  // candidate while it times one, else the defaults
  const auto* force = g_radix_force;
  g_radix_force = nullptr;
  RadixScope radix_scope(dtype, dir, flags, force);
  for (size_t i = 0; i < region.size(); ++i) {
    if (region[i] < 0 || region[i] >= rank)
      fail(FB_ERR_DIMENSION_MISMATCH, "Plan region is outside array dimensions.");
    if (i && region[i] <= region[i - 1]) fail(FB_ERR_DIMENSION_MISMATCH, "Region is invalid.");
  }
  for (int d = 0; d < rank; ++d) {
    if (dims[d] < 0) fail(FB_ERR_DIMENSION_MISMATCH, "negative dimension");
    if (istrides[d] < 0 || ostrides[d] < 0) fail(FB_ERR_ARGUMENT, "negative strides are not supported");
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    fail(FB_ERR_CUDA, "no CUDA device: this library has no CPU fallback");
  }
  std::unique_ptr<fb_plan_s> P(new fb_plan_s());
  P->dtype = dtype;
  P->dir = dir;
  P->cutoff = cutoff;
  P->flags = flags;
  P->rank = rank;
  P->dims.assign(dims, dims + rank);
  P->istrides.assign(istrides, istrides + rank);
  P->ostrides.assign(ostrides, ostrides + rank);
  P->region = region;
  cuda_check(cudaGetDevice(&P->device), "cudaGetDevice");
  int64_t total = 1;
  for (int d = 0; d < rank; ++d) total *= dims[d];
  for (size_t r = 0; r < region.size(); ++r) {
    const int d = region[r];
    if (dims[d] <= 0) fail(FB_ERR_DIMENSION_MISMATCH, "Array length must be strictly positive");
  }
  P->in_span = P->out_span = 0;
  if (total > 0) {
    int64_t si = 1, so = 1;
    for (int d = 0; d < rank; ++d) {
      si += (dims[d] - 1) * istrides[d];
      so += (dims[d] - 1) * ostrides[d];
    }
    P->in_span = si;
    P->out_span = so;
  }
  if (total > 0) {
    for (size_t r = 0; r < region.size(); ++r) {
      const int d = region[r];
      const bool first = r == 0;
      std::vector<BDim> bd;
      for (int j = 0; j < rank; ++j) {
        if (j == d) continue;
        bd.push_back({dims[j], first ? istrides[j] : ostrides[j], ostrides[j]});
      }
      P->axes.push_back(plan_axis(P.get(), dims[d], first ? istrides[d] : ostrides[d], ostrides[d],
                                  bd, first ? B_IN : B_OUT, B_OUT));
    }
    if (region.empty()) {
      // no transform: a copy (FFTA's mul! copies X into out first)
      std::vector<BDim> bd;
      for (int j = 1; j < rank; ++j) bd.push_back({dims[j], istrides[j], ostrides[j]});
      LineX x;
      make_direct(1, cutoff, dtype, &x);
      bd.insert(bd.begin(), BDim{dims[0], istrides[0], ostrides[0]});
      P->axes.push_back(plan_direct_axis(P.get(), 1, x, 0, 0, bd, B_IN, B_OUT));
    }
  }
  if (P->scratch_elems) {
    bool need1 = false;
    for (auto& ax : P->axes)
      for (auto& p : ax.passes) need1 |= p.src == B_S1 || p.dst == B_S1;
    P->need_s1 = need1;
    if (!(flags & kFlagNoScratch)) {
      P->scratch0.reset(new DevBuf(P->scratch_elems * elem_bytes(dtype)));
      if (need1) P->scratch1.reset(new DevBuf(P->scratch_elems * elem_bytes(dtype)));
    }
  }
  cuda_check(cudaStreamSynchronize(0), "plan tables");
  apply_tuning(P.get());
  return P.release();
}

static void execute_real(fb_plan_s* P, const void* in, void* out, cudaStream_t s);

// Whether a plan is a batched 1-D plan over contiguous-or-strided lines with
// one batch dim (fb_plan_create), which fb_execute_batch can run on fewer
// transforms than it was made for.
static bool batched_1d(const fb_plan_s* P) {
  return !P->real_kind && P->rank == 2 && P->region.size() == 1 && P->region[0] == 0 &&
         P->axes.size() == 1 && P->axes[0].outer.size() <= 1;
}

// nb >= 0 (batched 1-D plans only): run the first nb transforms of the
// batch.  The axis covers Bin transforms per host-loop step (the whole batch,
// or one L2 chunk); every pass's lines are a whole multiple of Bin, so a
// step of bc < Bin transforms runs nlines / Bin * bc lines.
static void execute_plan(fb_plan_s* P, const void* in, void* out, cudaStream_t s,
                         int64_t nb) {
  if (P->real_kind) {
    execute_real(P, in, out, s);
    return;
  }
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev != P->device) fail(FB_ERR_ARGUMENT, "plan was created on another device");
  if (P->scratch_elems && !(P->scratch0 ? P->scratch0->p : P->ext_s0))
    fail(FB_ERR_ARGUMENT, "plan has no scratch buffer bound");
  if (P->need_s1 && !(P->scratch1 ? P->scratch1->p : P->ext_s1))
    fail(FB_ERR_ARGUMENT, "plan has no second scratch buffer bound");
  const int es = elem_bytes(P->dtype);
  for (size_t ai = 0; ai < P->axes.size(); ++ai) {
    Axis& ax = P->axes[ai];
    int64_t nouter = 1;
    for (auto& o : ax.outer) nouter *= o.n;
    int64_t Bin = 0;
    if (nb >= 0) {
      Bin = P->dims[1] / nouter;
      nouter = (nb + Bin - 1) / Bin;
    }
    for (int64_t oi = 0; oi < nouter; ++oi) {
      int64_t offi = 0, offo = 0, t = oi;
      for (auto& o : ax.outer) {
        const int64_t k = t % o.n;
        t /= o.n;
        offi += k * o.is;
        offo += k * o.os;
      }
      const int64_t bc = nb >= 0 ? std::min(Bin, nb - oi * Bin) : 0;
      for (size_t pi = 0; pi < ax.passes.size(); ++pi) {
        Pass& p = ax.passes[pi];
        LineArgs a = p.a;
        if (nb >= 0) {
          a.nlines = p.a.nlines / Bin * bc;
          if (a.nlines <= 0) continue;
        }
        auto resolve = [&](int id, int64_t off) -> void* {
          switch (id) {
            case B_IN: return (char*)in + off * es;
            case B_OUT: return (char*)out + off * es;
            case B_S0: return P->scratch0 ? P->scratch0->p : P->ext_s0;
            default: return P->scratch1 ? P->scratch1->p : P->ext_s1;
          }
        };
        // outer offsets: the source of a first pass is the user input (axis 0)
        // or the output (later axes); both use the axis' own stride set.
        a.in = (void*)resolve(p.src, offi);
        a.out = resolve(p.dst, offo);
        const bool last = ai + 1 == P->axes.size() && pi + 1 == ax.passes.size();
        // the last pass's output is read by no later pass: store it evict-first
        a.st_stream = last ? 1 : 0;
        a.wait_ns = wait_limit_ns();
        if (p.fast) {
          FastArgs fa = p.fa;
          fa.in = a.in;
          fa.out = a.out;
          fa.st_stream = a.st_stream;
          fa.wait_ns = a.wait_ns;
          if (nb >= 0) fa.nlines = p.fa.nlines / Bin * bc;
          if (last) fa.scale = P->scale;
          // the bulk copies need 16-byte aligned line starts
          const bool st = p.stream && p.fast->launch_stream &&
                          reinterpret_cast<uintptr_t>(fa.in) % 16 == 0 && (fa.idist * es) % 16 == 0;
          const cudaError_t e = p.tc ? p.fast->launch_tc(P->dir, fa, s)
                                : st ? p.fast->launch_stream(P->dir, fa, s)
                                     : p.fast->launch(P->dir, fa, s);
          if (e != cudaSuccess) cuda_check(e, last_launch_message());
          continue;
        }
        if (last && P->scale != 1.0) a.scale = P->scale * a.scale;
        if (p.staged) {
          // tensor copies need the geometry for the current lines per tile
          // (the autotuner may have changed them) and a 16-byte aligned input
          TmaGeom tg;
          if (p.tma && tma_geometry(P, p, a, &tg) && encode_tma(P, p, a.in, a.G, tg)) {
            const cudaError_t e = p.staged->launch_tile_tma(a, &p.tmap, tg, s);
            if (e != cudaSuccess) cuda_check(e, last_launch_message());
            continue;
          }
          const cudaError_t e = p.tc ? p.staged->launch_tile_tc(a, s) : p.staged->launch_tile(a, s);
          if (e != cudaSuccess) cuda_check(e, last_launch_message());
          continue;
        }
        cuda_check(launch_line(P->dtype, p.variant, a, s), "line kernel launch");
      }
    }
  }
}

static int guard(const std::function<void()>& f) {
  try {
    f();
    g_last_error.clear();
    return FB_OK;
  } catch (FbError& e) {
    g_last_error = e.msg;
    return e.code;
  } catch (std::bad_alloc&) {
    g_last_error = "host out of memory";
    return FB_ERR_OUT_OF_MEMORY;
  } catch (std::exception& e) {
    g_last_error = e.what();
    return FB_ERR_ARGUMENT;
  }
}

}  // namespace fb

using namespace fb;

extern "C" {

int fb_plan_create_nd(fb_plan* plan, int dtype, int dir, int rank, const int64_t* dims,
                      const int64_t* istrides, const int64_t* ostrides, int nregion,
                      const int32_t* region, int64_t bluestein_cutoff, uint32_t flags) {
  return guard([&] {
    if (!plan) fail(FB_ERR_ARGUMENT, "plan pointer is null");
    *plan = nullptr;
    if (rank < 1 || !dims || !istrides || !ostrides) fail(FB_ERR_ARGUMENT, "bad array description");
    std::vector<int> reg;
    for (int i = 0; i < nregion; ++i) reg.push_back(region[i] - 1);
    *plan = create_plan(dtype, dir, rank, dims, istrides, ostrides, reg, bluestein_cutoff, flags);
  });
}

int fb_plan_create(fb_plan* plan, int64_t n, int dtype, int dir, int64_t batch, int64_t istride,
                   int64_t idist, int64_t ostride, int64_t odist, int64_t bluestein_cutoff,
                   uint32_t flags) {
  return guard([&] {
    if (!plan) fail(FB_ERR_ARGUMENT, "plan pointer is null");
    *plan = nullptr;
    if (n <= 0) fail(FB_ERR_DIMENSION_MISMATCH, "Array length must be strictly positive");
    if (batch < 0) fail(FB_ERR_DIMENSION_MISMATCH, "negative batch");
    int64_t dims[2] = {n, batch}, is[2] = {istride, idist}, os[2] = {ostride, odist};
    std::vector<int> reg{0};
    *plan = create_plan(dtype, dir, 2, dims, is, os, reg, bluestein_cutoff, flags);
  });
}

int fb_plan_create_2d(fb_plan* plan, int64_t n1, int64_t n2, int dtype, int dir, int64_t batch,
                      int64_t bluestein_cutoff, uint32_t flags) {
  return guard([&] {
    if (!plan) fail(FB_ERR_ARGUMENT, "plan pointer is null");
    *plan = nullptr;
    if (n1 <= 0 || n2 <= 0) fail(FB_ERR_DIMENSION_MISMATCH, "Array length must be strictly positive");
    int64_t dims[3] = {n1, n2, batch}, st[3] = {1, n1, n1 * n2};
    std::vector<int> reg{0, 1};
    *plan = create_plan(dtype, dir, 3, dims, st, st, reg, bluestein_cutoff, flags);
  });
}

int fb_plan_set_scale(fb_plan plan, double scale) {
  return guard([&] {
    if (!plan) fail(FB_ERR_ARGUMENT, "null plan");
    plan->scale = scale;
  });
}

int fb_execute(fb_plan plan, const void* in, void* out, void* stream) {
  return guard([&] {
    if (!plan) fail(FB_ERR_ARGUMENT, "null plan");
    if ((!in || !out) && (plan->in_span > 0)) fail(FB_ERR_ARGUMENT, "null data pointer");
    execute_plan(plan, in, out, (cudaStream_t)stream);
  });
}

int fb_execute_batch(fb_plan plan, const void* in, void* out, int64_t batch, void* stream) {
  return guard([&] {
    if (!plan) fail(FB_ERR_ARGUMENT, "null plan");
    if (!batched_1d(plan))
      fail(FB_ERR_UNSUPPORTED, "fb_execute_batch takes a batched 1-D plan (fb_plan_create)");
    if (batch < 0 || batch > plan->dims[1])
      fail(FB_ERR_DIMENSION_MISMATCH, "batch " + std::to_string(batch) +
                                          " is outside the plan's 0.." +
                                          std::to_string(plan->dims[1]));
    if (batch == 0) return;
    if (!in || !out) fail(FB_ERR_ARGUMENT, "null data pointer");
    execute_plan(plan, in, out, (cudaStream_t)stream, batch);
  });
}

// Pipelined host execution of a batched 1-D plan over contiguous columns:
// the batch is cut into chunks of about kHostChunk bytes that rotate through
// three device slots; each chunk is copied in on one stream, transformed in
// place on a second and copied out on a third, so the two copy directions and
// the kernels overlap.  Returns false when the plan is not of that shape.
static const size_t kHostChunk = 32u << 20;

static bool host_pipeline(fb_plan_s* P, const void* in, void* out) {
  if (P->rank != 2 || P->region.size() != 1 || P->region[0] != 0) return false;
  const int64_t n = P->dims[0], B = P->dims[1];
  if (P->istrides[0] != 1 || P->ostrides[0] != 1 || P->istrides[1] != n || P->ostrides[1] != n)
    return false;
  const size_t es = elem_bytes(P->dtype);
  const size_t col = (size_t)n * es;
  if ((size_t)B * col <= 2 * kHostChunk || col > kHostChunk) return false;
  if (!P->chunk_plan) {
    const int64_t chunk = std::max<int64_t>(1, (int64_t)(kHostChunk / col));
    int64_t dims[2] = {n, chunk}, st[2] = {1, n};
    std::vector<int> reg{0};
    P->chunk_plan.reset(create_plan(P->dtype, P->dir, 2, dims, st, st, reg, P->cutoff, P->flags));
    P->chunk_plan->scale = P->scale;
    if (B % chunk) {
      int64_t dt[2] = {n, B % chunk};
      P->tail_plan.reset(create_plan(P->dtype, P->dir, 2, dt, st, st, reg, P->cutoff, P->flags));
      P->tail_plan->scale = P->scale;
    }
    P->chunk = chunk;
    for (int i = 0; i < 3; ++i) {
      P->slots.emplace_back(new DevBuf((size_t)chunk * col));
      cuda_check(cudaStreamCreateWithFlags(&P->pstream[i], cudaStreamNonBlocking), "stream");
      for (int j = 0; j < 3; ++j)
        cuda_check(cudaEventCreateWithFlags(&P->pev[i][j], cudaEventDisableTiming), "event");
    }
  }
  P->chunk_plan->scale = P->scale;
  if (P->tail_plan) P->tail_plan->scale = P->scale;
  const int64_t chunk = P->chunk, nch = (B + chunk - 1) / chunk;
  cudaStream_t h2d = P->pstream[0], comp = P->pstream[1], d2h = P->pstream[2];
  for (int64_t c = 0; c < nch; ++c) {
    const int k = (int)(c % 3);
    const int64_t cols = std::min(chunk, B - c * chunk);
    const size_t bytes = (size_t)cols * col;
    void* slot = P->slots[k]->p;
    // the slot is free once its previous chunk has been copied out
    if (c >= 3) cuda_check(cudaStreamWaitEvent(h2d, P->pev[k][2], 0), "wait");
    cuda_check(cudaMemcpyAsync(slot, (const char*)in + (size_t)c * chunk * col, bytes,
                               cudaMemcpyHostToDevice, h2d), "copy in");
    cuda_check(cudaEventRecord(P->pev[k][0], h2d), "event");
    cuda_check(cudaStreamWaitEvent(comp, P->pev[k][0], 0), "wait");
    execute_plan(cols == chunk ? P->chunk_plan.get() : P->tail_plan.get(), slot, slot, comp);
    cuda_check(cudaEventRecord(P->pev[k][1], comp), "event");
    cuda_check(cudaStreamWaitEvent(d2h, P->pev[k][1], 0), "wait");
    cuda_check(cudaMemcpyAsync((char*)out + (size_t)c * chunk * col, slot, bytes,
                               cudaMemcpyDeviceToHost, d2h), "copy out");
    cuda_check(cudaEventRecord(P->pev[k][2], d2h), "event");
  }
  cuda_check(cudaStreamSynchronize(d2h), "synchronize");
  return true;
}

int fb_execute_host(fb_plan plan, const void* in, void* out, void* stream) {
  return guard([&] {
    if (!plan) fail(FB_ERR_ARGUMENT, "null plan");
    if (plan->in_span == 0) return;
    if (!plan->real_kind && host_pipeline(plan, in, out)) return;
    const int es = elem_bytes(plan->dtype);
    const int ies = plan->real_kind == 1 ? es / 2 : es, oes = plan->real_kind == 2 ? es / 2 : es;
    const size_t ib = (size_t)plan->in_span * ies, ob = (size_t)plan->out_span * oes;
    if (!plan->hin || plan->hin->bytes < ib) plan->hin.reset(new DevBuf(ib));
    if (!plan->hout || plan->hout->bytes < ob) plan->hout.reset(new DevBuf(ob));
    cudaStream_t s = (cudaStream_t)stream;
    cuda_check(cudaMemcpyAsync(plan->hin->p, in, ib, cudaMemcpyHostToDevice, s), "copy in");
    if (!plan->real_kind && (ob > ib || plan->out_span != plan->in_span)) {
      // outputs that no pass writes keep the host's values
      cuda_check(cudaMemcpyAsync(plan->hout->p, out, ob, cudaMemcpyHostToDevice, s), "copy out init");
    }
    execute_plan(plan, plan->hin->p, plan->hout->p, s);
    cuda_check(cudaMemcpyAsync(out, plan->hout->p, ob, cudaMemcpyDeviceToHost, s), "copy out");
    cuda_check(cudaStreamSynchronize(s), "synchronize");
  });
}

int fb_execute_grouped(fb_plan plan, int64_t count, const void* const* ins, void* const* outs,
                       const int64_t* batches, void* stream) {
  return guard([&] {
    if (!plan || (count > 0 && (!ins || !outs || !batches))) fail(FB_ERR_ARGUMENT, "null argument");
    if (count <= 0) return;
    if (plan->axes.size() != 1 || plan->axes[0].passes.size() != 1 ||
        !plan->axes[0].passes[0].fast || !plan->axes[0].outer.empty())
      fail(FB_ERR_UNSUPPORTED, "grouped execution needs a plan of one single-pass batched length");
    const Pass& p = plan->axes[0].passes[0];
    const int64_t n = plan->axes[0].n;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev != plan->device) fail(FB_ERR_ARGUMENT, "plan was created on another device");
    // descriptor block: pre[count+1] | ins[count] | outs[count]
    std::vector<int64_t> blob((size_t)(3 * count + 1));
    int64_t total = 0;
    for (int64_t r = 0; r < count; ++r) {
      if (batches[r] < 0) fail(FB_ERR_DIMENSION_MISMATCH, "negative batch");
      blob[r] = total;
      total += batches[r];
      blob[count + 1 + r] = (int64_t)(uintptr_t)ins[r];
      blob[2 * count + 1 + r] = (int64_t)(uintptr_t)outs[r];
    }
    blob[count] = total;
    if (total == 0) return;
    const size_t bytes = blob.size() * sizeof(int64_t);
    if (!plan->desc || plan->desc->bytes < bytes) plan->desc.reset(new DevBuf(bytes * 2));
    cudaStream_t s = (cudaStream_t)stream;
    cuda_check(cudaMemcpyAsync(plan->desc->p, blob.data(), bytes, cudaMemcpyHostToDevice, s),
               "descriptor copy");
    const int64_t* d = (const int64_t*)plan->desc->p;
    FastArgs fa = p.fa;
    fa.in = nullptr;
    fa.out = nullptr;
    fa.idist = n;  // each request's transforms are contiguous (API contract)
    fa.odist = n;
    fa.nlines = total;
    fa.scale = plan->scale;
    fa.ndesc = (int)count;
    fa.pre = d;
    fa.ins = (const void* const*)(d + count + 1);
    fa.outs = (void* const*)(d + 2 * count + 1);
    const int es = elem_bytes(plan->dtype);
    int G = std::max(1, 256 / p.fast->T);
    while (G > 1 && (size_t)G * p.fast->lpad * es > 100 * 1024) G /= 2;
    fa.G = G;
    const cudaError_t e = p.fast->launch(plan->dir, fa, s);
    if (e != cudaSuccess) cuda_check(e, last_launch_message());
  });
}

int fb_plan_size(fb_plan plan, int i, int64_t* out) {
  return guard([&] {
    if (!plan || !out) fail(FB_ERR_ARGUMENT, "null argument");
    if (i < 1) fail(FB_ERR_DOMAIN, "No non-positive dimensions");
    if (i > (int)plan->region.size())
      *out = 1;
    else
      *out = plan->dims[plan->region[i - 1]];
  });
}

int fb_plan_device_bytes(fb_plan plan, size_t* out) {
  return guard([&] {
    if (!plan || !out) fail(FB_ERR_ARGUMENT, "null argument");
    size_t b = plan->table_bytes;
    if (plan->scratch0) b += plan->scratch0->bytes;
    if (plan->scratch1) b += plan->scratch1->bytes;
    *out = b;
  });
}

int fb_plan_describe(fb_plan plan, char* buf, size_t len) {
  return guard([&] {
    if (!plan || !buf || !len) fail(FB_ERR_ARGUMENT, "null argument");
    std::ostringstream o;
    o << (plan->dtype == FB_C32 ? "C32" : "C64") << (plan->dir < 0 ? " fwd" : " bwd");
    if (plan->real_kind) {
      o << (plan->real_kind == 1 ? " rfft" : " brfft");
      if (plan->rfn)
        o << " | n=" << plan->dims[plan->r0] << " REAL-HALF(L=" << plan->rfn->L
          << " T=" << plan->rfn->T << " G=" << plan->ra.G << (plan->zr ? " strided" : "") << ")";
      else
        o << " | full-length complex plan:";
      if (plan->cplan) {
        char sub[3000];
        if (fb_plan_describe(plan->cplan.get(), sub, sizeof(sub)) == FB_OK) o << " + " << sub;
      }
    }
    for (auto& ax : plan->axes) {
      o << " | n=" << ax.n << " " << ax.kind;
      if (!ax.outer.empty()) o << " (host loop " << ax.outer.size() << " dims)";
      for (auto& p : ax.passes) {
        o << " " << p.what;
        if (p.tc)
          o << "<tc>";
        else if (p.fast)
          o << (p.stream ? "<stream>" : "<G=") << (p.stream ? "" : std::to_string(p.fa.G) + ">");
        else
          o << "<G=" << p.a.G << " T=" << p.a.T << " v=" << p.variant << ">";
      }
    }
    std::string s = o.str();
    std::snprintf(buf, len, "%s", s.c_str());
  });
}

int fb_plan_destroy(fb_plan plan) {
  return guard([&] { delete plan; });
}

int fb_kernel_error_flag(int* value, int reset) {
  return guard([&] {
    if (!value) fail(FB_ERR_ARGUMENT, "null argument");
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    const DeviceTables& dt = device_tables(dev);
    cuda_check(cudaMemcpy(value, dt.err, sizeof(int), cudaMemcpyDeviceToHost), "read flag");
    if (reset) cuda_check(cudaMemset(dt.err, 0, sizeof(int)), "reset flag");
  });
}

int fb_set_wait_limit(int64_t ns) {
  g_wait_ns.store(ns > 0 ? (uint64_t)ns : 0, std::memory_order_relaxed);
  set_last_error("");
  return FB_OK;
}

const char* fb_last_error(void) { return g_last_error.c_str(); }
const char* fb_version(void) { return FB_VERSION; }

}  // extern "C"

// ============================================================ real transforms
// rfft (src/plan.jl:102-125, 390-454, 506-542): the real input becomes the
// complex array x + 0i, the complex plan transforms it, and the first n/2+1
// entries along the first region dim are kept.  brfft (src/plan.jl:127-150,
// 456-504, 544-583): the n/2+1 stored entries are extended to the full
// Hermitian spectrum (mirrored in every region dim), the backward complex
// plan transforms it, and the real part is kept.  FFTA computes even lengths
// through a half-length complex transform and a split; the results agree to
// rounding.
namespace fb {

// FFTA's even-length real transform (src/plan.jl:398-442, :466-495): when
// the first region dim is the contiguous one (dim 1) and has even length
// n = 2L whose half runs on a specialised kernel, one fast_real_kernel pass
// transforms every line at half length with the split fused in, and the
// other region dims (if any) are complex transforms of the n/2+1-long half
// array -- after the real pass for rfft (in place on the output), before it
// for brfft (input -> scratch).  Returns nullptr when the path does not apply.
static fb_plan_s* create_half_real_plan(int dtype, int dir, int rank, const int64_t* dims,
                                        const std::vector<int>& region, int64_t cutoff,
                                        uint32_t flags) {
  if (region.empty() || (flags & FB_FLAG_GENERIC_ONLY)) return nullptr;
  // a single strided region dim is moved to the front (a strided copy in
  // and out), so every 1-D real transform takes the same half-length path
  // as a contiguous vector -- FFTA applies its vector method to each slice
  // (mapslices, src/plan.jl:507-527) -- and gives the same bits
  const int r0 = region[0];
  if (r0 != 0 && region.size() != 1) return nullptr;
  const int64_t n = dims[r0];
  if (n < 4 || n % 2) return nullptr;
  int64_t total = 1;
  for (int d = 0; d < rank; ++d) total *= dims[d];
  if (total <= 0) return nullptr;
  const int64_t L = n / 2;
  LineX x;
  if (!make_direct(L, cutoff, dtype, &x) || x.kind != 0) return nullptr;
  const FastFn* ff = find_fast(dtype, (int)L, x.radices);
  if (!ff || !ff->launch_real || (int)ff->lpad != lpad_for((int)L)) return nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    fail(FB_ERR_CUDA, "no CUDA device: this library has no CPU fallback");
  }
  std::unique_ptr<fb_plan_s> P(new fb_plan_s());
  P->dtype = dtype;
  P->dir = dir;
  P->cutoff = cutoff;
  P->flags = flags;
  P->rank = rank;
  P->dims.assign(dims, dims + rank);
  std::vector<int64_t> st(rank), hd(dims, dims + rank), hst(rank);
  hd[r0] = L + 1;
  int64_t s = 1, hs = 1;
  for (int d = 0; d < rank; ++d) {
    st[d] = s;
    hst[d] = hs;
    s *= dims[d];
    hs *= hd[d];
  }
  P->istrides = st;
  P->ostrides = st;
  P->region = region;
  cuda_check(cudaGetDevice(&P->device), "cudaGetDevice");
  P->real_kind = dir == FB_FORWARD ? 1 : 2;
  P->r0 = r0;
  P->rh = L + 1;
  for (int r : region) P->region_mask |= 1u << r;
  const int64_t half = total / n * (L + 1);
  if (r0 != 0) {
    // dims in the order (r0, the others): the kernel's contiguous lines
    std::vector<int> perm{r0};
    for (int d = 0; d < rank; ++d)
      if (d != r0) perm.push_back(d);
    PermCopy full, hp;
    memset(&full, 0, sizeof(full));
    memset(&hp, 0, sizeof(hp));
    full.rank = hp.rank = rank;
    full.count = total;
    hp.count = half;
    int64_t cf = 1, ch = 1;
    for (int d = 0; d < rank; ++d) {
      full.dims[d] = dims[perm[d]];
      hp.dims[d] = hd[perm[d]];
      // real array: `st` (user layout) <-> contiguous (cf); half: hst <-> ch
      full.is[d] = P->real_kind == 1 ? st[perm[d]] : cf;
      full.os[d] = P->real_kind == 1 ? cf : st[perm[d]];
      hp.is[d] = P->real_kind == 1 ? ch : hst[perm[d]];
      hp.os[d] = P->real_kind == 1 ? hst[perm[d]] : ch;
      cf *= full.dims[d];
      ch *= hp.dims[d];
    }
    P->perm_full = full;
    P->perm_half = hp;
    P->zr.reset(new DevBuf((size_t)total * elem_bytes(dtype) / 2));
    P->zc.reset(new DevBuf((size_t)half * elem_bytes(dtype)));
  }
  P->in_span = P->real_kind == 1 ? total : half;
  P->out_span = P->real_kind == 1 ? half : total;
  // the length-L program and the split's twiddles w^k = exp(-2 pi i k / n)
  StageProg prog;
  fill_prog(P.get(), x, &prog);
  void* wk = alloc_table(P.get(), (size_t)(L / 2 + 1) * elem_bytes(dtype));
  cuda_check(gen_roots(dtype, wk, n, 1, L / 2 + 1, 0), "real split twiddles");
  RealArgs& a = P->ra;
  memset(&a, 0, sizeof(a));
  a.nlines = total / n;
  a.idist = P->real_kind == 1 ? n : L + 1;
  a.odist = P->real_kind == 1 ? L + 1 : n;
  a.tw = prog.tw;
  const DeviceTables& dt = device_tables(P->device);
  a.prime_cs = dtype == FB_C32 ? dt.f32 : dt.f64;
  a.wk = wk;
  a.scale = 1.0;
  // lines per block as for the complex direct kernel: up to a warp's worth
  // of threads, within 100 KB of shared memory
  int G = std::max(1, 32 / ff->T);
  while (G > 1 && (size_t)G * ff->lpad * elem_bytes(dtype) > 100 * 1024) G /= 2;
  while (G > 1 && G / 2 >= a.nlines) G /= 2;
  a.G = G;
  P->rfn = ff;
  if (region.size() > 1) {
    std::vector<int> reg(region.begin() + 1, region.end());
    P->cplan.reset(create_plan(dtype, dir, rank, hd.data(), hst.data(), hst.data(), reg, cutoff,
                               flags));
    if (P->real_kind == 2) P->zbuf.reset(new DevBuf((size_t)half * elem_bytes(dtype)));
  }
  cuda_check(cudaStreamSynchronize(0), "real plan tables");
  return P.release();
}

static fb_plan_s* create_real_plan(int dtype, int dir, int rank, const int64_t* dims,
                                   const std::vector<int>& region, int64_t cutoff, uint32_t flags) {
  if (region.empty()) fail(FB_ERR_ARGUMENT, "a real transform needs at least one region dim");
  std::vector<int64_t> st(rank);
  int64_t total = 1;
  for (int d = 0; d < rank; ++d) {
    if (dims[d] < 0) fail(FB_ERR_DIMENSION_MISMATCH, "negative dimension");
    st[d] = total;
    total *= dims[d];
  }
  if (auto* H = create_half_real_plan(dtype, dir, rank, dims, region, cutoff, flags)) return H;
  std::unique_ptr<fb_plan_s> C(create_plan(dtype, dir, rank, dims, st.data(), st.data(), region,
                                           cutoff, flags));
  std::unique_ptr<fb_plan_s> P(new fb_plan_s());
  P->dtype = dtype;
  P->dir = dir;
  P->cutoff = cutoff;
  P->flags = flags;
  P->rank = rank;
  P->dims.assign(dims, dims + rank);
  P->istrides = st;
  P->ostrides = st;
  P->region = region;
  P->device = C->device;
  P->real_kind = dir == FB_FORWARD ? 1 : 2;
  P->r0 = region[0];
  P->rh = dims[P->r0] / 2 + 1;
  for (int r : region) P->region_mask |= 1u << r;
  const int64_t half = total / std::max<int64_t>(1, dims[P->r0]) * P->rh;
  // spans counted in elements of each side's own type (real or complex)
  P->in_span = P->real_kind == 1 ? total : half;
  P->out_span = P->real_kind == 1 ? half : total;
  if (total > 0) P->zbuf.reset(new DevBuf((size_t)total * elem_bytes(dtype)));
  P->cplan = std::move(C);
  return P.release();
}

static void execute_real(fb_plan_s* P, const void* in, void* out, cudaStream_t s) {
  int64_t total = 1, pre = 1, post = 1;
  for (int d = 0; d < P->rank; ++d) {
    total *= P->dims[d];
    if (d < P->r0) pre *= P->dims[d];
    if (d > P->r0) post *= P->dims[d];
  }
  if (total == 0) return;
  if (P->rfn && P->zr) {
    // strided region dim: copy to (r0, others) order, transform, copy back
    RealArgs a = P->ra;
    const int es = elem_bytes(P->dtype);
    a.scale = P->scale;
    a.st_stream = 0;
    if (P->real_kind == 1) {
      cuda_check(permute_copy(es / 2, in, P->zr->p, P->perm_full, s), "real gather");
      a.in = P->zr->p;
      a.out = P->zc->p;
    } else {
      cuda_check(permute_copy(es, in, P->zc->p, P->perm_half, s), "half gather");
      a.in = P->zc->p;
      a.out = P->zr->p;
    }
    const cudaError_t e = P->rfn->launch_real(P->real_kind == 1 ? FB_FORWARD : FB_BACKWARD, a, s);
    if (e != cudaSuccess) cuda_check(e, last_launch_message());
    if (P->real_kind == 1)
      cuda_check(permute_copy(es, P->zc->p, out, P->perm_half, s), "half scatter");
    else
      cuda_check(permute_copy(es / 2, P->zr->p, out, P->perm_full, s), "real scatter");
    return;
  }
  if (P->rfn) {
    RealArgs a = P->ra;
    fb_plan_s* C = P->cplan.get();
    if (P->real_kind == 1) {
      a.in = in;
      a.out = out;
      a.scale = C ? 1.0 : P->scale;
      a.st_stream = C ? 0 : 1;
      const cudaError_t e = P->rfn->launch_real(FB_FORWARD, a, s);
      if (e != cudaSuccess) cuda_check(e, last_launch_message());
      if (C) {
        C->scale = P->scale;
        execute_plan(C, out, out, s);
      }
    } else {
      const void* src = in;
      if (C) {
        C->scale = 1.0;
        execute_plan(C, in, P->zbuf->p, s);
        src = P->zbuf->p;
      }
      a.in = src;
      a.out = out;
      a.scale = P->scale;
      a.st_stream = 1;
      const cudaError_t e = P->rfn->launch_real(FB_BACKWARD, a, s);
      if (e != cudaSuccess) cuda_check(e, last_launch_message());
    }
    return;
  }
  P->cplan->scale = P->scale;
  void* z = P->zbuf->p;
  if (P->real_kind == 1) {
    cuda_check(real_to_complex(P->dtype, in, z, total, s), "real to complex");
    execute_plan(P->cplan.get(), z, z, s);
    cuda_check(extract_half(P->dtype, z, out, pre, P->dims[P->r0], P->rh, post, s), "extract");
  } else {
    cuda_check(herm_extend(P->dtype, in, z, P->rank, P->dims.data(), P->r0, P->rh,
                           P->region_mask, s), "hermitian extension");
    execute_plan(P->cplan.get(), z, z, s);
    cuda_check(complex_to_real(P->dtype, z, out, total, s), "complex to real");
  }
}

}  // namespace fb

extern "C" int fb_plan_create_real(fb_plan* plan, int dtype, int dir, int rank,
                                   const int64_t* dims, int nregion, const int32_t* region,
                                   int64_t bluestein_cutoff, uint32_t flags) {
  return guard([&] {
    if (!plan) fail(FB_ERR_ARGUMENT, "plan pointer is null");
    *plan = nullptr;
    if (rank < 1 || rank > 8 || !dims) fail(FB_ERR_ARGUMENT, "bad array description");
    std::vector<int> reg;
    for (int i = 0; i < nregion; ++i) reg.push_back(region[i] - 1);
    *plan = create_real_plan(dtype, dir, rank, dims, reg, bluestein_cutoff, flags);
  });
}

// ===================================================================== server
// Continuous batching over work-descriptor launches.  Requests (n, type,
// direction, batch, device in/out) wait in arrival order; dispatch() admits
// them while their bytes fit the budget and
//  * packs every admitted request whose length runs in one pass and that has
//    fewer than kPackedMaxElems elements into work-descriptor launches of the
//    generic kernel (one per kernel variant, block size and shared-memory
//    class) -- requests of different lengths and directions share a launch;
//  * runs multi-pass lengths (four-step, three-pass Bluestein) and large
//    requests with a cached per-(n, type, direction, batch) plan, each plan
//    bound to one plan stream, so that a plan's scratch is never used by two
//    requests at once while different plans overlap.
// Launches rotate over the server's streams; poll() retires completed ones
// and dispatches what has arrived since, so new requests join as earlier
// ones finish.
namespace fb {

// Descriptor-launch shape of a single-pass template plan: its line
// arguments with the thread shape and shared-memory class filled in.
struct SrvShape {
  LineArgs a;
  int var = 0, threads = 0, cls = 0, G = 1;
};

struct SrvReq {
  int64_t ticket, n, batch;
  int dtype, dir;
  const void* in;
  void* out;
  double bytes;
  const SrvShape* shape;  // nullptr: multi-pass length
  bool drop = false;      // fault injection: its descriptor never arrives
};

struct SrvLaunch {
  cudaEvent_t ev;
  std::vector<int64_t> tickets;
  double bytes;
  int slot;  // descriptor slot, or -1
};

struct SrvSlot {
  std::unique_ptr<DevBuf> buf;
  void* host = nullptr;  // pinned staging of the descriptor table
  size_t host_bytes = 0;
  cudaEvent_t last = nullptr;  // the launch that last read this slot
};

}  // namespace fb

struct fb_server_s {
  // device blocks of the plans this server makes and releases (declared
  // first: destroyed after every plan that holds one)
  std::unique_ptr<fb::BlockCache> cache;
  // scratch of the multi-pass plans, one pair of buffers per plan stream
  struct Arena {
    std::unique_ptr<fb::DevBuf> s0, s1;
  };
  std::vector<Arena> arena;
  int device = 0;
  double budget = 100e9;
  std::vector<cudaStream_t> streams;
  // multi-pass plans: each plan keeps one of these streams (its scratch is
  // then never used by two launches at once); different plans run side by side
  std::vector<cudaStream_t> multi_streams;
  std::map<const fb_plan_s*, int> multi_stream_of;
  int next_multi_stream = 0;
  cudaEvent_t start = nullptr;
  int next_stream = 0, next_slot = 0;
  std::map<std::tuple<int64_t, int, int>, std::unique_ptr<fb_plan_s>> templ;
  // plans of multi-pass and large requests, one per (n, type, direction,
  // batch bucket) -- the bucket is the smallest power of two >= the batch,
  // at least kSrvMinBucket -- run on a request's batch with the plan's
  // variable-batch execution; least recently used plans are released while
  // their device bytes exceed multi_cap
  struct MultiPlan {
    std::unique_ptr<fb_plan_s> P;
    int64_t used = 0;
    cudaEvent_t ev = nullptr;  // after its last launch
    size_t bytes = 0;
  };
  std::map<std::tuple<int64_t, int, int, int64_t>, MultiPlan> multi;
  size_t multi_bytes = 0, multi_cap = 0;
  int64_t multi_clock = 0, st_plans_made = 0, st_plans_released = 0;
  bool serial = false;  // FB_SERVER_SERIAL: one request at a time
  std::deque<fb::SrvReq> pending;
  std::deque<fb::SrvLaunch> inflight;
  std::vector<fb::SrvSlot> slots;
  double admitted = 0;
  int64_t next_ticket = 0;
  std::deque<std::pair<int64_t, double>> done;
  // per template plan: its descriptor launch shape, computed once
  std::map<const fb_plan_s*, fb::SrvShape> shapes;
  // CUDA graphs of multi-pass plans keyed by (plan, input, output): a request
  // shape that recurs on the same buffers is captured on its second
  // occurrence and replayed as one graph launch from then on
  typedef std::tuple<const fb_plan_s*, const void*, void*, int64_t> GraphKey;
  struct Graph {
    cudaGraphExec_t exec;
    cudaStream_t st;
    int64_t used;
  };
  bool graphs = true;
  std::map<GraphKey, int> seen;
  std::map<GraphKey, Graph> graph_of;
  // released graphs, destroyed once the event after their last launch is done
  std::vector<std::pair<cudaEvent_t, cudaGraphExec_t>> graph_retiring;
  int64_t graph_clock = 0, st_graph_launches = 0, st_graph_captures = 0;
  int64_t st_launches = 0, st_desc_launches = 0, st_requests = 0, st_max_queue = 0;
  int64_t st_cancelled = 0, st_resident = 0, st_failed = 0;
  // the resident kernel's descriptor queue (small requests of served
  // lengths), its outstanding requests, and the device clock origin
  struct PqDeleter {
    void operator()(fb::PQueue* q) const { fb::pq_destroy(q); }
  };
  std::unique_ptr<fb::PQueue, PqDeleter> pq;
  struct PqReq {
    int64_t r, ticket;
    double bytes;
  };
  std::vector<PqReq> pq_out;
  int64_t* clk_host = nullptr;  // mapped pinned: globaltimer at the clock origin
  int64_t* clk_dev = nullptr;
  int64_t clk0_ns = 0;
  bool drop_next = false;  // fault injection (tests): the next request's descriptor never arrives
  double st_max_admitted = 0;
  ~fb_server_s() {
    for (auto& g : graph_of) cudaGraphExecDestroy(g.second.exec);
    for (auto& g : graph_retiring) {
      cudaEventDestroy(g.first);
      cudaGraphExecDestroy(g.second);
    }
    for (auto& l : inflight) cudaEventDestroy(l.ev);
    for (auto& sl : slots) {
      if (sl.last) cudaEventDestroy(sl.last);
      if (sl.host) cudaFreeHost(sl.host);
    }
    pq.reset();
    for (auto& m : multi)
      if (m.second.ev) cudaEventDestroy(m.second.ev);
    if (clk_host) cudaFreeHost(clk_host);
    for (auto s : streams) cudaStreamDestroy(s);
    for (auto s : multi_streams) cudaStreamDestroy(s);
    if (start) cudaEventDestroy(start);
  }
};

namespace fb {

static bool srv_single_pass(const fb_plan_s* P);

static fb_plan_s* srv_template(fb_server_s* S, int64_t n, int dtype, int dir) {
  auto key = std::make_tuple(n, dtype, dir);
  auto it = S->templ.find(key);
  if (it != S->templ.end()) return it->second.get();
  if (n > lmax_for(dtype)) {
    // beyond the generic kernel's line: never one generic pass
    S->templ[key].reset();
    return nullptr;
  }
  // two contiguous transforms: the batch level of the lines is level 0 with
  // stride n, which the descriptors rewrite per request
  int64_t dims[2] = {n, 2}, st[2] = {1, n};
  std::vector<int> reg{0};
  BlockCacheScope scope(S->cache.get());
  fb_plan_s* P = create_plan(dtype, dir, 2, dims, st, st, reg, FB_DEFAULT_BLUESTEIN_CUTOFF,
                             FB_FLAG_GENERIC_ONLY);
  if (!srv_single_pass(P)) {
    // multi-pass lengths run their bucket plans; only the single-pass answer is kept
    // (tens of thousands of distinct lengths would otherwise hold their
    // tables and scratch for good)
    delete P;
    P = nullptr;
  }
  S->templ[key].reset(P);
  return P;
}

static bool srv_single_pass(const fb_plan_s* P) {
  return P && P->axes.size() == 1 && P->axes[0].passes.size() == 1 && P->axes[0].outer.empty() &&
         P->axes[0].passes[0].a.ld.mode == 0 && P->axes[0].passes[0].a.st.mode == 0;
}

static const int64_t kSrvMinBucket = 512;
// Bytes of each scratch buffer a plan stream shares among its plans: the L2
// chunk the four-step and Bluestein schedules cut their batch into, so every
// plan of the served lengths fits (larger needs get their own).
static const size_t kSrvArenaBytes = kL2Chunk;
// Bind the scratch of plan P (made without its own) to the buffers of plan
// stream si.  Plans of one stream never run at once, so they share them.
static void srv_bind_scratch(fb_server_s* S, fb_plan_s* P, int si) {
  if (!P->scratch_elems || P->scratch0) return;
  auto& ar = S->arena[si];
  if (!ar.s0) {
    ar.s0.reset(new DevBuf(kSrvArenaBytes));
    ar.s1.reset(new DevBuf(kSrvArenaBytes));
  }
  P->ext_s0 = ar.s0->p;
  P->ext_s1 = ar.s1->p;
}
static int64_t srv_bucket(int64_t batch) {
  int64_t b = kSrvMinBucket;
  while (b < batch) b *= 2;
  return b;
}
static size_t plan_scratch_bytes(const fb_plan_s* P);
static void srv_release_plan(fb_server_s* S, const fb_plan_s* P);
static void srv_trim_multi(fb_server_s* S, size_t cap);

static fb_plan_s* srv_multi(fb_server_s* S, int64_t n, int dtype, int dir, int64_t batch) {
  auto key = std::make_tuple(n, dtype, dir, srv_bucket(batch));
  auto it = S->multi.find(key);
  if (it != S->multi.end()) {
    it->second.used = ++S->multi_clock;
    return it->second.P.get();
  }
  srv_trim_multi(S, S->multi_cap);
  int64_t dims[2] = {n, srv_bucket(batch)}, st[2] = {1, n};
  std::vector<int> reg{0};
  fb_plan_s* P = nullptr;
  BlockCacheScope scope(S->cache.get());
  try {
    P = create_plan(dtype, dir, 2, dims, st, st, reg, FB_DEFAULT_BLUESTEIN_CUTOFF, kFlagNoScratch);
  } catch (const FbError& e) {
    if (e.code != FB_ERR_OUT_OF_MEMORY) throw;
    // device memory is short (other users of the device): release every
    // idle plan and try once more
    srv_trim_multi(S, 0);
    S->cache->trim(0);
    P = create_plan(dtype, dir, 2, dims, st, st, reg, FB_DEFAULT_BLUESTEIN_CUTOFF, kFlagNoScratch);
  }
  // scratch above a plan stream's shared buffers: the plan's own
  const size_t need = P->scratch_elems * elem_bytes(dtype);
  if (need > kSrvArenaBytes) {
    P->scratch0.reset(new DevBuf(need));
    if (P->need_s1) P->scratch1.reset(new DevBuf(need));
  }
  fb_server_s::MultiPlan& m = S->multi[key];
  m.P.reset(P);
  m.used = ++S->multi_clock;
  m.bytes = P->table_bytes + plan_scratch_bytes(P);
  S->multi_bytes += m.bytes;
  S->st_plans_made += 1;
  return P;
}

// Release idle multi-pass plans, least recently used first, while their
// device bytes exceed `cap`.
static void srv_trim_multi(fb_server_s* S, size_t cap) {
  while (S->multi_bytes > cap && !S->multi.empty()) {
    auto lru = S->multi.end();
    for (auto m = S->multi.begin(); m != S->multi.end(); ++m) {
      if (m->second.ev && cudaEventQuery(m->second.ev) == cudaErrorNotReady) {
        cudaGetLastError();
        continue;
      }
      if (lru == S->multi.end() || m->second.used < lru->second.used) lru = m;
    }
    if (lru == S->multi.end()) break;  // every plan is busy
    srv_release_plan(S, lru->second.P.get());
    S->multi_bytes -= lru->second.bytes;
    if (lru->second.ev) cudaEventDestroy(lru->second.ev);
    S->multi.erase(lru);
    S->st_plans_released += 1;
  }
}

static size_t plan_scratch_bytes(const fb_plan_s* P) {
  size_t b = 0;
  if (P->scratch0) b += P->scratch0->bytes;
  if (P->scratch1) b += P->scratch1->bytes;
  return b;
}

// Forget everything that refers to an idle plan about to be released: its
// CUDA graphs (their launches have completed), its occurrence counts and its
// plan stream.
static void srv_release_plan(fb_server_s* S, const fb_plan_s* P) {
  for (auto g = S->graph_of.begin(); g != S->graph_of.end();) {
    if (std::get<0>(g->first) == P) {
      cudaGraphExecDestroy(g->second.exec);
      g = S->graph_of.erase(g);
    } else {
      ++g;
    }
  }
  for (auto k = S->seen.begin(); k != S->seen.end();)
    k = std::get<0>(k->first) == P ? S->seen.erase(k) : std::next(k);
  S->multi_stream_of.erase(P);
}

// Graphs kept per server; the least recently used one is released first.
static const size_t kGraphCacheMax = 1024;

// Destroy the released graphs whose last launch has finished.
static void srv_sweep_graphs(fb_server_s* S) {
  auto& v = S->graph_retiring;
  for (size_t i = 0; i < v.size();) {
    const cudaError_t q = cudaEventQuery(v[i].first);
    if (q == cudaErrorNotReady) {
      ++i;
      continue;
    }
    cuda_check(q, "graph release");
    cudaEventDestroy(v[i].first);
    cudaGraphExecDestroy(v[i].second);
    v[i] = v.back();
    v.pop_back();
  }
}

// Run multi-pass plan P on (in, out) in stream st: plain launches the first
// time a (plan, in, out) key is seen, a captured graph from the second time.
// Capture only records the launches (relaxed mode, nothing runs), so the
// graph's kernels and arguments are exactly those of execute_plan.
static void srv_run_plan(fb_server_s* S, fb_plan_s* P, const void* in, void* out,
                         int64_t batch, cudaStream_t st) {
  if (!S->graphs) {
    execute_plan(P, in, out, st, batch);
    return;
  }
  const fb_server_s::GraphKey key(P, in, out, batch);
  auto g = S->graph_of.find(key);
  if (g == S->graph_of.end()) {
    if (S->seen.size() >= 16 * kGraphCacheMax) S->seen.clear();
    if (++S->seen[key] < 2) {
      execute_plan(P, in, out, st, batch);
      return;
    }
    if (S->graph_of.size() >= kGraphCacheMax) {
      auto lru = S->graph_of.begin();
      for (auto it = S->graph_of.begin(); it != S->graph_of.end(); ++it)
        if (it->second.used < lru->second.used) lru = it;
      // released after its last launch: an event behind it on its stream
      cudaEvent_t ev = nullptr;
      cuda_check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
      cuda_check(cudaEventRecord(ev, lru->second.st), "event record");
      S->graph_retiring.push_back({ev, lru->second.exec});
      S->graph_of.erase(lru);
      srv_sweep_graphs(S);
    }
    cudaGraph_t graph = nullptr;
    cuda_check(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed), "graph capture");
    try {
      execute_plan(P, in, out, st, batch);
    } catch (...) {
      cudaStreamEndCapture(st, &graph);
      if (graph) cudaGraphDestroy(graph);
      throw;
    }
    cuda_check(cudaStreamEndCapture(st, &graph), "graph capture");
    cudaGraphExec_t exec = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    cuda_check(e, "graph instantiate");
    g = S->graph_of.emplace(key, fb_server_s::Graph{exec, st, 0}).first;
    S->seen.erase(key);
    S->st_graph_captures += 1;
  }
  g->second.used = ++S->graph_clock;
  g->second.st = st;
  cuda_check(cudaGraphLaunch(g->second.exec, st), "graph launch");
  S->st_graph_launches += 1;
}

// Completed requests of the resident kernel's queue; relaunches the kernel
// while requests are outstanding and none is resident (it ends when idle).
// Completion times come from the device globaltimer; a request the kernel
// gave up on (kPqStat*) completes with time -1.
static void srv_reap_resident(fb_server_s* S) {
  if (S->pq_out.empty()) return;
  size_t keep = 0;
  for (size_t i = 0; i < S->pq_out.size(); ++i) {
    const auto& q = S->pq_out[i];
    int64_t t = 0;
    int32_t st = 0;
    if (pq_poll(S->pq.get(), q.r, &t, &st)) {
      // failed: -1 when the descriptor never arrived, -2 without a program
      S->done.push_back({q.ticket, st == kPqStatOk
                                       ? (double)(t - S->clk0_ns) * 1e-6
                                       : (st == kPqStatTimeout ? -1.0 : -2.0)});
      if (st != kPqStatOk) S->st_failed += 1;
      S->admitted -= q.bytes;
    } else {
      S->pq_out[keep++] = q;
    }
  }
  S->pq_out.resize(keep);
  if (!S->pq_out.empty()) cuda_check(pq_kick(S->pq.get()), "resident kernel launch");
}

static void srv_retire(fb_server_s* S, bool block) {
  if (!S->graph_retiring.empty()) srv_sweep_graphs(S);
  srv_reap_resident(S);
  while (!S->inflight.empty()) {
    bool done_any = false;
    for (auto it = S->inflight.begin(); it != S->inflight.end();) {
      cudaError_t q = block ? cudaEventSynchronize(it->ev) : cudaEventQuery(it->ev);
      if (q == cudaErrorNotReady) {
        ++it;
        continue;
      }
      cuda_check(q, "server launch");
      float ms = 0;
      cuda_check(cudaEventElapsedTime(&ms, S->start, it->ev), "event time");
      for (int64_t t : it->tickets) S->done.push_back({t, (double)ms});
      S->admitted -= it->bytes;
      cudaEventDestroy(it->ev);
      it = S->inflight.erase(it);
      done_any = true;
    }
    if (!block || !done_any) break;
  }
}

// Shared-memory classes of descriptor launches (bytes per block).
static const size_t kSmemClass[4] = {16u << 10, 48u << 10, 100u << 10, 220u << 10};

// The descriptor-launch shape of template T (made once per template).
static const SrvShape* srv_shape(fb_server_s* S, const fb_plan_s* T, int dtype) {
  auto it = S->shapes.find(T);
  if (it != S->shapes.end()) return &it->second;
  const Pass& p = T->axes[0].passes[0];
  SrvShape sh;
  sh.a = p.a;
  int Tt = sh.a.T, var = p.variant;
  std::vector<int> rad(sh.a.prog.radix, sh.a.prog.radix + sh.a.prog.nst);
  if (!pick_threads(sh.a.prog.L, rad, &Tt, &var)) fail(FB_ERR_UNSUPPORTED, "no thread shape");
  sh.threads = Tt > 256 ? 512 : 256;
  const size_t line_bytes = (size_t)sh.a.Lpad * elem_bytes(dtype) + 4 * sizeof(int64_t);
  int cls = 0;
  while (cls < 3 && line_bytes > kSmemClass[cls]) ++cls;
  int G = std::max(1, sh.threads / Tt);
  while (G > 1 && (size_t)G * line_bytes > kSmemClass[cls]) --G;
  sh.a.T = Tt;
  sh.a.G = G;
  sh.var = var;
  sh.cls = cls;
  sh.G = G;
  return &(S->shapes[T] = sh);
}

// Requests one dispatch takes at most: a burst is cut into several launches
// so building the next one's descriptors overlaps the GPU running this one.
static const size_t kDispatchMax = 384;
// Requests of at least this many elements are not packed into descriptor
// launches of the generic kernel but run through their own cached plan.
static const int64_t kPackedMaxElems = int64_t(1) << 18;

static void srv_dispatch(fb_server_s* S) {
  std::vector<SrvReq> batch;
  // serial mode: one request, and only once the previous one has completed
  const size_t most = S->serial ? (S->inflight.empty() && S->pq_out.empty() ? 1 : 0) : kDispatchMax;
  while (!S->pending.empty() && batch.size() < most) {
    const SrvReq& r = S->pending.front();
    if (S->admitted + r.bytes > S->budget && (S->admitted > 0 || !batch.empty())) break;
    S->admitted += r.bytes;
    batch.push_back(r);
    S->pending.pop_front();
  }
  S->st_max_admitted = std::max(S->st_max_admitted, S->admitted);
  if (batch.empty()) return;
  // groups of descriptors keyed by (dtype, variant, threads, smem class)
  struct Group {
    std::vector<LineArgs> descs;
    std::vector<int64_t> bstart{0};
    std::vector<int64_t> tickets;
    double bytes = 0;
    size_t smem = 0;
  };
  std::map<std::tuple<int, int, int, int>, Group> groups;
  bool resident = false;
  for (const SrvReq& r : batch) {
    // small requests of a served length go to the resident kernel's queue
    const int pid = r.shape && S->pq ? pq_program_id(r.dtype, r.dir, r.n) : -1;
    if (pid >= 0 && (int64_t)S->pq_out.size() < pq_slots() - 1) {
      if (!pq_has_program(S->pq.get(), pid)) {
        const Pass& tp = srv_template(S, r.n, r.dtype, r.dir)->axes[0].passes[0];
        cuda_check(pq_set_program(S->pq.get(), pid, tp.a.prog.tw, tp.a.prime_cs),
                   "resident program table");
      }
      // a dropped descriptor carries a sequence number no request ever has
      const int64_t q =
          pq_push(S->pq.get(), pid, r.in, r.out, r.batch, r.drop ? int64_t(1) << 41 : 0);
      S->pq_out.push_back({q, r.ticket, r.bytes});
      S->st_resident += 1;
      resident = true;
      continue;
    }
    if (!r.shape || S->serial) {
      fb_plan_s* P = srv_multi(S, r.n, r.dtype, r.dir, r.batch);
      auto ms = S->multi_stream_of.find(P);
      if (ms == S->multi_stream_of.end())
        ms = S->multi_stream_of
                 .emplace(P, (int)(S->next_multi_stream++ % S->multi_streams.size()))
                 .first;
      cudaStream_t mst = S->multi_streams[ms->second];
      srv_bind_scratch(S, P, ms->second);
      srv_run_plan(S, P, r.in, r.out, r.batch, mst);
      {
        fb_server_s::MultiPlan& m =
            S->multi[std::make_tuple(r.n, r.dtype, r.dir, srv_bucket(r.batch))];
        if (!m.ev) cuda_check(cudaEventCreateWithFlags(&m.ev, cudaEventDisableTiming), "event");
        cuda_check(cudaEventRecord(m.ev, mst), "event record");
      }
      SrvLaunch l;
      cuda_check(cudaEventCreateWithFlags(&l.ev, cudaEventDefault), "event");
      cuda_check(cudaEventRecord(l.ev, mst), "event record");
      l.tickets.push_back(r.ticket);
      l.bytes = r.bytes;
      l.slot = -1;
      S->inflight.push_back(std::move(l));
      S->st_launches += 1;
      continue;
    }
    const SrvShape& sh = *r.shape;
    LineArgs a = sh.a;
    const int var = sh.var, threads = sh.threads, cls = sh.cls;
    int G = sh.G;
    while (G > 1 && G / 2 >= r.batch) G /= 2;
    a.G = G;
    a.in = r.in;
    a.out = r.out;
    a.nlines = r.batch;
    a.m0 = r.batch;
    a.m1 = 1;
    a.scale = 1.0;
    Group& g = groups[std::make_tuple(r.dtype, var, threads, cls)];
    g.descs.push_back(a);
    g.bstart.push_back(g.bstart.back() + (r.batch + G - 1) / G);
    g.tickets.push_back(r.ticket);
    g.bytes += r.bytes;
    g.smem = std::max(g.smem, line_smem_bytes(r.dtype, sh.a));
  }
  if (resident) {
    pq_publish(S->pq.get());
    cuda_check(pq_kick(S->pq.get()), "resident kernel launch");
  }
  for (auto& kv : groups) {
    Group& g = kv.second;
    const int dtype = std::get<0>(kv.first), var = std::get<1>(kv.first);
    const int threads = std::get<2>(kv.first);
    const int nd = (int)g.descs.size();
    // descriptor slot (reused once its previous launch has finished)
    const int si = S->next_slot++ % (int)S->slots.size();
    SrvSlot& slot = S->slots[si];
    if (slot.last) {
      cuda_check(cudaEventSynchronize(slot.last), "slot reuse");
      cudaEventDestroy(slot.last);
      slot.last = nullptr;
    }
    const size_t bytes = nd * sizeof(LineArgs) + (nd + 1) * sizeof(int64_t);
    if (!slot.buf || slot.buf->bytes < bytes) slot.buf.reset(new DevBuf(bytes * 2));
    if (slot.host_bytes < bytes) {
      if (slot.host) cudaFreeHost(slot.host);
      slot.host = nullptr;
      slot.host_bytes = 0;
      cuda_check(cudaMallocHost(&slot.host, bytes * 2), "pinned staging");
      slot.host_bytes = bytes * 2;
    }
    unsigned char* host = (unsigned char*)slot.host;
    memcpy(host, g.descs.data(), nd * sizeof(LineArgs));
    memcpy(host + nd * sizeof(LineArgs), g.bstart.data(), (nd + 1) * sizeof(int64_t));
    cudaStream_t st = S->streams[S->next_stream++ % S->streams.size()];
    cuda_check(cudaMemcpyAsync(slot.buf->p, host, bytes, cudaMemcpyHostToDevice, st),
               "descriptor copy");
    const LineArgs* dd = (const LineArgs*)slot.buf->p;
    const int64_t* db = (const int64_t*)((char*)slot.buf->p + nd * sizeof(LineArgs));
    cuda_check(launch_desc(dtype, var, dd, db, nd, g.bstart.back(), threads, g.smem, st),
               "descriptor launch");
    SrvLaunch l;
    cuda_check(cudaEventCreateWithFlags(&l.ev, cudaEventDefault), "event");
    cuda_check(cudaEventRecord(l.ev, st), "event record");
    cuda_check(cudaEventCreateWithFlags(&slot.last, cudaEventDisableTiming), "event");
    cuda_check(cudaEventRecord(slot.last, st), "event record");
    l.tickets = std::move(g.tickets);
    l.bytes = g.bytes;
    l.slot = si;
    S->inflight.push_back(std::move(l));
    S->st_launches += 1;
    S->st_desc_launches += 1;
  }
}

}  // namespace fb

extern "C" {

int fb_server_create(fb_server* srv, double budget_bytes, int nstreams, uint32_t flags) {
  return guard([&] {
    if (!srv) fail(FB_ERR_ARGUMENT, "null argument");
    *srv = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      fail(FB_ERR_CUDA, "no CUDA device: this library has no CPU fallback");
    }
    std::unique_ptr<fb_server_s> S(new fb_server_s());
    cuda_check(cudaGetDevice(&S->device), "cudaGetDevice");
    S->budget = budget_bytes > 0 ? budget_bytes : 100e9;
    S->serial = (flags & FB_SERVER_SERIAL) != 0;
    S->graphs = !(flags & FB_SERVER_NO_GRAPHS) && !S->serial;
    S->multi_cap = (size_t)std::max(S->budget / 2, 1e9);
    S->cache.reset(new BlockCache(size_t(4) << 30));
    const int ns = std::max(1, std::min(nstreams, 16));
    for (int i = 0; i < ns; ++i) {
      cudaStream_t st;
      cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
      S->streams.push_back(st);
    }
    for (int i = 0; i < ns; ++i) {
      cudaStream_t st;
      cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
      S->multi_streams.push_back(st);
    }
    S->arena.resize(S->multi_streams.size());
    // descriptor slots sized for the largest dispatch up front: growing one
    // later frees device memory (which synchronises the device) and
    // allocates pinned memory in the middle of serving
    S->slots.resize(4 * ns);
    const size_t slot_bytes = kDispatchMax * sizeof(LineArgs) + (kDispatchMax + 1) * sizeof(int64_t);
    for (SrvSlot& sl : S->slots) {
      sl.buf.reset(new DevBuf(slot_bytes));
      cuda_check(cudaMallocHost(&sl.host, slot_bytes), "pinned staging");
      sl.host_bytes = slot_bytes;
    }
    cuda_check(cudaEventCreate(&S->start), "event");
    cuda_check(cudaEventRecord(S->start, S->streams[0]), "event record");
    cuda_check(cudaEventSynchronize(S->start), "event sync");
    if (!(flags & (FB_SERVER_NO_PERSISTENT | FB_SERVER_SERIAL))) {
      PQueue* q = nullptr;
      // the resident kernel ends after 100 us without work, so that it does
      // not hold SMs that the plan launches of other requests need
      cuda_check(pq_create(&q, 100000ull), "persistent queue");
      S->pq.reset(q);
      cuda_check(cudaHostAlloc((void**)&S->clk_host, sizeof(int64_t), cudaHostAllocMapped),
                 "clock");
      cuda_check(cudaHostGetDevicePointer((void**)&S->clk_dev, S->clk_host, 0), "clock");
      cuda_check(pq_clock(S->streams[0], S->clk_dev, S->clk_host), "clock");
      S->clk0_ns = *(volatile int64_t*)S->clk_host;
    }
    *srv = S.release();
  });
}

int fb_server_submit(fb_server srv, int64_t n, int dtype, int dir, int64_t batch, const void* in,
                     void* out, int64_t* ticket) {
  return guard([&] {
    if (!srv || !ticket) fail(FB_ERR_ARGUMENT, "null argument");
    if (n <= 0) fail(FB_ERR_DIMENSION_MISMATCH, "Array length must be strictly positive");
    if (dtype != FB_C32 && dtype != FB_C64)
      fail(FB_ERR_ARGUMENT, "element type must be ComplexF32 or ComplexF64");
    if (dir != FB_FORWARD && dir != FB_BACKWARD) fail(FB_ERR_ARGUMENT, "direction must be -1 or +1");
    if (batch < 1 || !in || !out) fail(FB_ERR_ARGUMENT, "bad batch or data pointer");
    // plans are made at submission (tables resident); bytes = data + scratch
    double bytes = 2.0 * (double)n * (double)batch * elem_bytes(dtype);
    auto refuse = [&]() {
      std::ostringstream m;
      m << "request needs " << (int64_t)bytes << " device bytes (input, output, scratch), above "
        << "the server's budget of " << (int64_t)srv->budget;
      fail(FB_ERR_OUT_OF_MEMORY, m.str());
    };
    if (bytes > srv->budget) refuse();  // before any plan (and its scratch) is made
    fb_plan_s* T = srv_template(srv, n, dtype, dir);
    // large single-pass requests run their own plan (specialised kernels) on
    // a plan stream; small ones are packed into descriptor launches
    const bool packed = srv_single_pass(T) && n * batch < kPackedMaxElems;
    const SrvShape* shape = packed ? srv_shape(srv, T, dtype) : nullptr;
    if (!shape || srv->serial) {
      // the scratch this batch uses in its plan: one host-loop step's share
      // of the plan's scratch per transform, at most the whole of it
      const fb_plan_s* M = srv_multi(srv, n, dtype, dir, batch);
      int64_t steps = 1;
      for (auto& o : M->axes[0].outer) steps *= o.n;
      const double per = (double)plan_scratch_bytes(M) / (double)(M->dims[1] / steps);
      bytes += std::min((double)plan_scratch_bytes(M), per * (double)batch);
    }
    // a request that could never be admitted is refused now, not queued for good
    if (bytes > srv->budget) refuse();
    SrvReq r{srv->next_ticket++, n, batch, dtype, dir, in, out, bytes, shape, srv->drop_next};
    srv->drop_next = false;
    srv->pending.push_back(r);
    srv->st_requests += 1;
    srv->st_max_queue = std::max<int64_t>(srv->st_max_queue, (int64_t)srv->pending.size());
    *ticket = r.ticket;
  });
}

int fb_server_submit_many(fb_server srv, int64_t count, const int64_t* n, const int32_t* dtype,
                          const int32_t* dir, const int64_t* batch, const void* const* in,
                          void* const* out, int64_t* tickets) {
  for (int64_t i = 0; i < count; ++i) {
    const int rc = fb_server_submit(srv, n[i], dtype[i], dir[i], batch[i], in[i], out[i],
                                    tickets + i);
    if (rc != FB_OK) return rc;
  }
  return FB_OK;
}

int fb_server_poll(fb_server srv, int64_t max, int64_t* tickets, double* done_ms, int64_t* count) {
  return guard([&] {
    if (!srv || !count) fail(FB_ERR_ARGUMENT, "null argument");
    srv_retire(srv, false);
    // keep at most one launch per stream (plus multi-pass work) in flight:
    // whatever arrived meanwhile goes out together in the next dispatch
    if ((int64_t)srv->inflight.size() < (int64_t)srv->streams.size()) srv_dispatch(srv);
    int64_t k = 0;
    while (k < max && !srv->done.empty()) {
      tickets[k] = srv->done.front().first;
      done_ms[k] = srv->done.front().second;
      srv->done.erase(srv->done.begin());
      ++k;
    }
    *count = k;
  });
}

int fb_server_drop_next_descriptor(fb_server srv) {
  return guard([&] {
    if (!srv) fail(FB_ERR_ARGUMENT, "null argument");
    if (!srv->pq) fail(FB_ERR_UNSUPPORTED, "the server has no resident kernel");
    srv->drop_next = true;
  });
}

int fb_server_cancel(fb_server srv, int64_t ticket) {
  return guard([&] {
    if (!srv) fail(FB_ERR_ARGUMENT, "null argument");
    for (auto it = srv->pending.begin(); it != srv->pending.end(); ++it) {
      if (it->ticket != ticket) continue;
      srv->pending.erase(it);
      srv->st_cancelled += 1;
      return;
    }
    fail(FB_ERR_ARGUMENT, "ticket " + std::to_string(ticket) +
                              " is not waiting: unknown, already dispatched or completed");
  });
}

int fb_server_wait(fb_server srv) {
  return guard([&] {
    if (!srv) fail(FB_ERR_ARGUMENT, "null argument");
    // requests of the resident kernel complete in host memory: poll them,
    // giving up (an error) after 30 s without any completing
    auto last = std::chrono::steady_clock::now();
    size_t outstanding = (size_t)-1;
    while (!srv->pending.empty() || !srv->inflight.empty() || !srv->pq_out.empty()) {
      srv_dispatch(srv);
      srv_retire(srv, srv->pq_out.empty());
      if (srv->pq_out.empty()) continue;
      const size_t n = srv->pq_out.size() + srv->pending.size() + srv->inflight.size();
      if (n != outstanding) {
        outstanding = n;
        last = std::chrono::steady_clock::now();
      } else if (std::chrono::steady_clock::now() - last > std::chrono::seconds(30)) {
        fail(FB_ERR_CUDA, "resident kernel made no progress for 30 s");
      }
      std::this_thread::yield();
    }
  });
}

int fb_server_stats(fb_server srv, int64_t* out, int nout) {
  return guard([&] {
    if (!srv || !out) fail(FB_ERR_ARGUMENT, "null argument");
    const int64_t v[13] = {srv->st_requests, srv->st_launches, srv->st_desc_launches,
                           srv->st_max_queue, (int64_t)srv->st_max_admitted,
                           (int64_t)(srv->templ.size() + srv->multi.size()),
                           srv->st_graph_launches, srv->st_graph_captures, srv->st_cancelled,
                           srv->st_resident, srv->st_failed, srv->st_plans_made,
                           srv->st_plans_released};
    for (int i = 0; i < nout && i < 13; ++i) out[i] = v[i];
  });
}

int fb_server_reset_clock(fb_server srv) {
  return guard([&] {
    if (!srv) fail(FB_ERR_ARGUMENT, "null argument");
    cuda_check(cudaEventRecord(srv->start, srv->streams[0]), "event record");
    cuda_check(cudaEventSynchronize(srv->start), "event sync");
    if (srv->clk_host) {
      cuda_check(pq_clock(srv->streams[0], srv->clk_dev, srv->clk_host), "clock");
      srv->clk0_ns = *(volatile int64_t*)srv->clk_host;
    }
  });
}

int fb_server_destroy(fb_server srv) {
  return guard([&] {
    if (!srv) return;
    srv->pq.reset();  // asks the resident kernel to stop and waits for it
    cudaDeviceSynchronize();
    delete srv;
  });
}

}  // extern "C"

// ================================================================= autotuner
// Launch shapes -- lines per block (G) of every pass and, for passes on the
// generic kernel, its register budget (16 or 32 values per thread, which sets
// the threads per line) -- are timed on the caller's buffers and the fastest
// kept.  Winners are cached per plan key (type, direction, dims, strides,
// region: i.e. per length, batch and layout) for later plans in the process,
// and can be saved to / loaded from a text file.  The stage program of a
// length is never tuned: it fixes the arithmetic, which must not depend on the
// batch (batched and single transforms stay bit-identical).
namespace fb {

struct TuneEntry {
  std::vector<int> G, T, variant;
};
static std::mutex g_tune_mu;
static std::map<std::string, TuneEntry> g_tune;

static std::string plan_key(const fb_plan_s* P) {
  std::ostringstream k;
  k << P->dtype << ":" << P->dir << ":" << P->cutoff << ":" << P->flags << ":";
  for (int d = 0; d < P->rank; ++d)
    k << P->dims[d] << "/" << P->istrides[d] << "/" << P->ostrides[d] << ",";
  k << ":";
  for (int r : P->region) k << r << ",";
  return k.str();
}

static std::vector<Pass*> all_passes(fb_plan_s* P) {
  std::vector<Pass*> v;
  for (auto& ax : P->axes)
    for (auto& p : ax.passes) v.push_back(&p);
  return v;
}

static int& pass_G(Pass& p) { return p.fast ? p.fa.G : p.a.G; }

// Candidate shapes of a pass that its kernel accepts.
struct Shape {
  int G, T, variant;
};

static std::vector<Shape> pass_shapes(const fb_plan_s* P, const Pass& p) {
  if (p.tc) return {};  // the tensor-core stage fixes its block shape
  // lines per block: the planner's choice and a geometric ladder around it
  std::vector<int> gs;
  const int G0 = p.fast ? p.fa.G : p.a.G;
  gs.push_back(G0);
  for (int g = 1; g <= 1024; g = g < 4 ? g + 1 : g + g / 2) gs.push_back(g);
  std::sort(gs.begin(), gs.end());
  gs.erase(std::unique(gs.begin(), gs.end()), gs.end());
  std::vector<Shape> out;
  const int es = elem_bytes(P->dtype);
  const int64_t nl = std::max<int64_t>(1, p.fast ? p.fa.nlines : p.a.nlines);
  const size_t smem_max = 200 * 1024;
  if (p.fast) {
    // variant 1: the persistent bulk-copy kernel (one line per block)
    const int T = p.fast->T, cap = std::max(1, (T >= 256 ? T : 256) / T);
    if (p.fast->launch_stream) out.push_back({1, T, 1});
    for (int G : gs)
      if (G <= cap && (G == G0 || G <= nl) && (size_t)G * p.fast->lpad * es <= smem_max)
        out.push_back({G, T, 0});
  } else if (p.staged) {
    const int T = p.staged->T;
    const int cap = p.a.mid ? std::max(1, p.staged->mid_threads / T) : tile_thread_cap(p.staged);
    for (int G : gs)
      if (G <= cap && (G == G0 || G <= nl) &&
          (size_t)G * (tile_pitch((int)p.staged->lpad, G, es) * es + 32) <= smem_max)
        out.push_back({G, T, 0});
  } else {
    // generic kernel: both register budgets, each with the line-count ladder
    std::vector<int> rad(p.a.prog.radix, p.a.prog.radix + p.a.prog.nst);
    bool big = false;
    for (int R : rad) big |= R > 16;
    const bool em = p.a.ld.mode == 1 || p.a.st.mode == 1;
    for (int cap : {16, 32}) {
      if (big && cap == 32) continue;
      int tmin = 1;
      for (int R : rad) tmin = std::max(tmin, (p.a.prog.L / R + um_for(R, cap) - 1) / um_for(R, cap));
      if (tmin > line_max_threads()) continue;
      int T = 1;
      if (tmin <= 32) {
        while (T < tmin) T <<= 1;
      } else {
        T = (tmin + 31) / 32 * 32;
      }
      const int variant = (cap == 32 ? 1 : 0) | (big ? 2 : 0);
      for (int G : gs) {
        if (em && (G & (G - 1))) continue;  // element-major tiles take powers of two
        if (G * T > line_max_threads() || (G != G0 && G > nl)) continue;
        LineArgs a = p.a;
        a.G = G;
        a.T = T;
        if (line_smem_bytes(P->dtype, a) > smem_max) continue;
        out.push_back({G, T, variant});
      }
    }
  }
  return out;
}

static void set_shape(Pass& p, const Shape& s) {
  pass_G(p) = s.G;
  if (p.fast) {
    p.stream = s.variant;
  } else if (!p.staged) {
    p.a.T = s.T;
    p.variant = s.variant;
  }
}

static int pass_variant(const Pass& p) { return p.fast ? p.stream : p.variant; }

// A cached entry is applied only when every one of its shapes is one the
// pass's kernel accepts (a file may come from another build or be edited).
static void apply_tuning(fb_plan_s* P) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(plan_key(P));
  if (it == g_tune.end()) return;
  auto ps = all_passes(P);
  const TuneEntry& e = it->second;
  if (ps.size() != e.G.size()) return;
  std::vector<Shape> pick(ps.size());
  for (size_t i = 0; i < ps.size(); ++i) {
    const bool generic = !ps[i]->fast && !ps[i]->staged;
    bool ok = false;
    for (const Shape& s : pass_shapes(P, *ps[i]))
      if (s.G == e.G[i] && s.variant == e.variant[i] && (!generic || s.T == e.T[i])) {
        ok = true;
        pick[i] = s;
      }
    if (!ok) return;
  }
  for (size_t i = 0; i < ps.size(); ++i) set_shape(*ps[i], pick[i]);
}

// Alternative radix programs of a one-pass length L: groupings of the factor
// 2^a into radices 16/8/4/2 (largest first; fewest stages first), of 3^b into
// 9/3, the other primes ascending; the powers of two first, or (when both
// are present) the powers of three first.  The default program comes first;
// at most 12, each one a program the kernels can run.
static std::vector<std::vector<int>> radix_candidates(int64_t L, int dtype) {
  int a = 0, b = 0;
  int64_t m = L;
  while (m % 2 == 0) {
    m /= 2;
    ++a;
  }
  while (m % 3 == 0) {
    m /= 3;
    ++b;
  }
  std::vector<int> rest;
  for (auto& pe : factorize(m))
    for (int i = 0; i < pe.second; ++i) rest.push_back((int)pe.first);
  std::vector<std::vector<int>> p2;
  std::vector<int> cur;
  std::function<void(int, int)> part = [&](int left, int maxlg) {
    if (left == 0) {
      p2.push_back(cur);
      return;
    }
    for (int lg = std::min(maxlg, left); lg >= 1; --lg) {
      cur.push_back(1 << lg);
      part(left - lg, lg);
      cur.pop_back();
    }
  };
  part(a, 4);
  std::stable_sort(p2.begin(), p2.end(),
                   [](const std::vector<int>& x, const std::vector<int>& y) { return x.size() < y.size(); });
  if (p2.size() > 5) p2.resize(5);
  std::vector<std::vector<int>> p3;
  for (int i = b / 2; i >= 0 && p3.size() < 2; --i) {
    std::vector<int> v(i, 9);
    v.insert(v.end(), b - 2 * i, 3);
    p3.push_back(v);
  }
  std::vector<std::vector<int>> out{default_radix_program(L)};
  auto add = [&](std::vector<int> v) {
    v.insert(v.end(), rest.begin(), rest.end());
    int T, var;
    if ((int)v.size() > FB_MAX_STAGES || !pick_threads((int)L, v, &T, &var)) return;
    if (std::find(out.begin(), out.end(), v) == out.end() && out.size() < 12) out.push_back(v);
  };
  for (auto& x : p2)
    for (auto& y : p3) {
      std::vector<int> v = x;
      v.insert(v.end(), y.begin(), y.end());
      add(v);
      if (!x.empty() && !y.empty()) {
        std::vector<int> w = y;
        w.insert(w.end(), x.begin(), x.end());
        add(w);
      }
    }
  (void)dtype;
  return out;
}

static double time_plan(fb_plan_s* P, const void* in, void* out, cudaStream_t st, int iters) {
  cudaEvent_t e0, e1;
  cuda_check(cudaEventCreate(&e0), "event");
  cuda_check(cudaEventCreate(&e1), "event");
  execute_plan(P, in, out, st);  // warm (attributes, caches)
  cuda_check(cudaEventRecord(e0, st), "event");
  for (int i = 0; i < iters; ++i) execute_plan(P, in, out, st);
  cuda_check(cudaEventRecord(e1, st), "event");
  cuda_check(cudaEventSynchronize(e1), "event sync");
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms / std::max(1, iters);
}

// FB_FLAG_TUNE_RADIX: for every one-pass length of the plan, build the plan
// with each candidate program for that length, time it on the caller's
// buffers and keep the fastest (its schedule replaces the plan's own); the
// choice is recorded for later plans with the flag.
static void tune_radix(fb_plan_s* P, const void* in, void* out, cudaStream_t st, int iters) {
  std::vector<int64_t> Ls;
  for (auto& ax : P->axes)
    if (ax.kind == "DIRECT" && ax.passes.size() == 1 && ax.n > 3 &&
        std::find(Ls.begin(), Ls.end(), ax.n) == Ls.end())
      Ls.push_back(ax.n);
  std::map<int64_t, std::vector<int>> chosen;
  {
    std::lock_guard<std::mutex> lk(g_radix_mu);
    chosen = g_radix_tuned[{P->dtype, P->dir}];
  }
  for (int64_t L : Ls) {
    const auto cands = radix_candidates(L, P->dtype);
    if (cands.size() < 2) continue;
    double tbest = time_plan(P, in, out, st, iters);
    std::unique_ptr<fb_plan_s> best;
    std::vector<int> bestc;
    for (const auto& c : cands) {
      std::map<int64_t, std::vector<int>> ov = chosen;
      ov[L] = c;
      g_radix_force = &ov;
      std::unique_ptr<fb_plan_s> Q(create_plan(P->dtype, P->dir, P->rank, P->dims.data(),
                                               P->istrides.data(), P->ostrides.data(), P->region,
                                               P->cutoff, P->flags));
      Q->scale = P->scale;
      const double t = time_plan(Q.get(), in, out, st, iters);
      if (t < tbest) {
        tbest = t;
        best = std::move(Q);
        bestc = c;
      }
    }
    if (best) {
      chosen[L] = bestc;
      std::swap(P->axes, best->axes);
      std::swap(P->bufs, best->bufs);
      std::swap(P->table_bytes, best->table_bytes);
      std::swap(P->scratch_elems, best->scratch_elems);
      std::swap(P->scratch0, best->scratch0);
      std::swap(P->scratch1, best->scratch1);
      P->chunk_plan.reset();  // the host pipeline's plans are made again
      P->tail_plan.reset();
    }
  }
  std::lock_guard<std::mutex> lk(g_radix_mu);
  auto& g = g_radix_tuned[{P->dtype, P->dir}];
  for (auto& kv : chosen) g[kv.first] = kv.second;
}

}  // namespace fb

extern "C" {

int fb_plan_autotune(fb_plan plan, const void* in, void* out, void* stream, int iters) {
  return guard([&] {
    if (!plan) fail(FB_ERR_ARGUMENT, "null plan");
    if (plan->real_kind) fail(FB_ERR_UNSUPPORTED, "autotune a real plan through its complex plan");
    if (plan->in_span == 0) return;
    if (!in || !out) fail(FB_ERR_ARGUMENT, "null data pointer");
    cudaStream_t st = (cudaStream_t)stream;
    iters = std::max(1, iters);
    if (plan->flags & FB_FLAG_TUNE_RADIX) tune_radix(plan, in, out, st, iters);
    auto ps = all_passes(plan);
    for (Pass* p : ps) {
      auto shapes = pass_shapes(plan, *p);
      if (shapes.size() < 2) continue;
      Shape best{pass_G(*p), p->a.T, pass_variant(*p)};
      double tbest = time_plan(plan, in, out, st, iters);
      for (const Shape& s : shapes) {
        set_shape(*p, s);
        const double t = time_plan(plan, in, out, st, iters);
        if (t < tbest) {
          tbest = t;
          best = s;
        }
      }
      set_shape(*p, best);
    }
    TuneEntry e;
    for (Pass* p : ps) {
      e.G.push_back(pass_G(*p));
      e.T.push_back(p->a.T);
      e.variant.push_back(pass_variant(*p));
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[plan_key(plan)] = e;
  });
}

int fb_tune_cache_save(const char* path) {
  return guard([&] {
    if (!path) fail(FB_ERR_ARGUMENT, "null path");
    std::lock_guard<std::mutex> lk(g_tune_mu);
    FILE* f = std::fopen(path, "w");
    if (!f) fail(FB_ERR_ARGUMENT, std::string("cannot write ") + path);
    std::fprintf(f, "# fftab200 tuning cache v1: key|G,T,variant;...  and  radix|type:dir:L|r.r.r\n");
    for (auto& kv : g_tune) {
      std::fprintf(f, "%s|", kv.first.c_str());
      for (size_t i = 0; i < kv.second.G.size(); ++i)
        std::fprintf(f, "%d,%d,%d;", kv.second.G[i], kv.second.T[i], kv.second.variant[i]);
      std::fprintf(f, "\n");
    }
    std::lock_guard<std::mutex> lr(g_radix_mu);
    for (auto& td : g_radix_tuned)
      for (auto& kv : td.second) {
        std::fprintf(f, "radix|%d:%d:%lld|", td.first.first, td.first.second, (long long)kv.first);
        for (size_t i = 0; i < kv.second.size(); ++i)
          std::fprintf(f, "%s%d", i ? "." : "", kv.second[i]);
        std::fprintf(f, "\n");
      }
    std::fclose(f);
  });
}

int fb_tune_cache_load(const char* path) {
  return guard([&] {
    if (!path) fail(FB_ERR_ARGUMENT, "null path");
    FILE* f = std::fopen(path, "r");
    if (!f) fail(FB_ERR_ARGUMENT, std::string("cannot read ") + path);
    char line[8192];
    std::lock_guard<std::mutex> lk(g_tune_mu);
    while (std::fgets(line, sizeof(line), f)) {
      std::string l(line);
      if (l.empty() || l[0] == '#') continue;
      if (l.compare(0, 6, "radix|") == 0) {
        // a tuned radix program: kept only if it multiplies to its length
        int dt, dr;
        long long L;
        if (std::sscanf(l.c_str() + 6, "%d:%d:%lld|", &dt, &dr, &L) != 3) continue;
        std::istringstream rs(l.substr(l.find('|', 6) + 1));
        std::vector<int> prog;
        std::string tok;
        int64_t prod = 1;
        while (std::getline(rs, tok, '.')) {
          const int r = std::atoi(tok.c_str());
          if (r < 2 || r > FB_MAX_PRIME) break;
          prog.push_back(r);
          prod *= r;
        }
        if (prod == L && !prog.empty() && prog.size() <= FB_MAX_STAGES) {
          std::lock_guard<std::mutex> lr(g_radix_mu);
          g_radix_tuned[{dt, dr}][L] = prog;
        }
        continue;
      }
      const size_t bar = l.find('|');
      if (bar == std::string::npos) continue;
      TuneEntry e;
      std::istringstream rest(l.substr(bar + 1));
      std::string item;
      while (std::getline(rest, item, ';')) {
        int G, T, v;
        if (std::sscanf(item.c_str(), "%d,%d,%d", &G, &T, &v) == 3) {
          e.G.push_back(G);
          e.T.push_back(T);
          e.variant.push_back(v);
        }
      }
      g_tune[l.substr(0, bar)] = e;
    }
    std::fclose(f);
  });
}

}  // extern "C"
