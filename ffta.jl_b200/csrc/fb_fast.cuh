// fb_fast.cuh -- compile-time-specialised line kernels for the common lengths.
//
// The stage program (radices) is a template parameter, so every index, stride
// and twiddle offset is a constant and each stage's registers die before the
// next stage starts.  The first stage reads its butterfly inputs straight
// from HBM into registers and the last stage writes its outputs straight from
// registers to HBM; only the exchanges between stages go through shared
// memory.  A length-4096 line with radices 16x16x16 makes one HBM read, two
// shared-memory round trips and one HBM write per element.
//
// Two kernels share the stage code:
//   fast_direct_kernel  batched contiguous lines: consecutive threads own
//                       consecutive butterflies of one line (coalesced along
//                       the line);
//   fast_tile_kernel    G lines of any stride per block, lines fastest across
//                       the threads of a warp, so adjacent lines (the columns
//                       of a four-step pass, the rows of a 2-D axis) coalesce;
//                       fuses the Bluestein chirp on load, the four-step
//                       twiddle, the chirp and a scale on store, and (MID) the
//                       Bluestein spectrum multiply between a forward and an
//                       inverse program.
//
// The arithmetic -- twiddle table entries, twiddle multiply (tw_elem's
// product for the four-step twiddle on a lean-I/O pass's loads), butterflies,
// order of stages -- is exactly that of the generic line kernel
// (fb_line.cuh), so all of them produce the same bits for the same length.
#pragma once
#include <cstdio>
#include <cstring>
#include <type_traits>

#include "fb_line.cuh"
#include "fb_tc.cuh"

namespace fb {

// Text of the last launch failure in the specialised kernels (read by the
// planner to build its error message).
extern thread_local char g_launch_msg[512];

template <int... Rs> struct RList {
  static constexpr int n = sizeof...(Rs);
  static constexpr int r[n] = {Rs...};
};

template <class RL, int S> __host__ __device__ constexpr int ns_before() {
  int p = 1;
  for (int i = 0; i < S; ++i) p *= RL::r[i];
  return p;
}
template <class RL, int S> __host__ __device__ constexpr int tw_offset() {
  int off = 0, ns = 1;
  for (int i = 0; i < S; ++i) {
    off += (RL::r[i] - 1) * ns;
    ns *= RL::r[i];
  }
  return off;
}
template <class RL> __host__ __device__ constexpr int prog_len() {
  int p = 1;
  for (int i = 0; i < RL::n; ++i) p *= RL::r[i];
  return p;
}
__host__ __device__ constexpr int lpad_of(int L) {
  return (((L - 1) + ((L - 1) >> 4) + 1) & 1) ? (L - 1) + ((L - 1) >> 4) + 1
                                               : (L - 1) + ((L - 1) >> 4) + 2;
}

// Shared-memory slot of element e of a line.  Power-of-two strides would hit
// the same banks, so even lengths skip one slot every 16 (padi); odd lengths
// (powers of three and 5-smooth odd lengths) have only odd strides, which
// spread over the banks by themselves, and are stored flat.
template <class RL> __device__ __forceinline__ int pidx(int e) {
  if constexpr (prog_len<RL>() % 2 == 1)
    return e;
  else
    return padi(e);
}

// ---------------------------------------------------------------- I/O
// A stage's input or output is shared memory (SmemIO) or a functor that
// loads element i of the line / stores element i of the line.
struct SmemIO {};

// Input functors load element i in two steps: raw(i) issues the memory load,
// fin(i, v) applies what depends on the element (tables, twiddles).  A stage
// issues all of its raw loads before any fin, so every data load is in flight
// before the table loads take registers.
//
// Cache hints.  A pass reads each input element once, so data loads are
// streaming (evict-first in L2): the misses of a pass then displace each
// other rather than the lines of its input that are still resident (the
// previous pass's output).  Stores are evict-first only in a plan's last pass
// (`cs`); an earlier pass leaves its output in L2 for the next one.
template <typename R> __device__ __forceinline__ void store(cplx<R>* p, cplx<R> v, bool cs) {
  if (cs)
    __stcs(p, v);
  else
    *p = v;
}
template <typename R> struct DirectIn {
  const cplx<R>* __restrict__ g;
  bool ok;
  __device__ __forceinline__ cplx<R> raw(int i) const {
    return ok ? __ldcs(g + i) : Sc<R>::mk(R(0), R(0));
  }
  __device__ __forceinline__ cplx<R> fin(int, cplx<R> v) const { return v; }
};
template <typename R> struct DirectOut {
  cplx<R>* __restrict__ g;
  bool ok;
  R scale;
  bool cs;
  __device__ __forceinline__ void operator()(int i, cplx<R> v) const {
    if (ok) store<R>(g + i, scale == R(1) ? v : cscale<R>(v, scale), cs);
  }
};

// Element i of a strided line, present when i*ves + voff < vn; the optional
// table `mul` (the chirp) is indexed by that same value.
template <typename R> struct TileIn {
  const cplx<R>* __restrict__ base;
  int64_t es;
  const cplx<R>* __restrict__ mul;
  int64_t vn, ves, voff;
  bool ok;
  const cplx<R>* __restrict__ tab;  // twiddle on load (LineArgs::tw_on_load)
  int64_t tab_es, tab_off;
  int tw_dir;
  __device__ __forceinline__ cplx<R> raw(int i) const {
    const int64_t vi = (int64_t)i * ves + voff;
    if (!ok || vi >= vn) return Sc<R>::mk(R(0), R(0));
    return __ldcs(base + (int64_t)i * es);
  }
  __device__ __forceinline__ cplx<R> fin(int i, cplx<R> v) const {
    const int64_t vi = (int64_t)i * ves + voff;
    if (!ok || vi >= vn) return v;
    if (mul) v = cmul<R>(v, __ldg(mul + vi));
    if (tab) {
      const cplx<R> w = __ldg(tab + (int64_t)i * tab_es + tab_off);
      v = tw_dir < 0 ? cmul<R>(v, w) : cmulc<R>(v, w);
    }
    return v;
  }
};
// Store with, in order: the table `mul` (chirp), the twiddle w_N^(dir*l0*i)
// (hi/lo root tables), the scale.
// prefetch.global.L1: a hint that brings the line into L1 (no register is
// written; the address is one the kernel reads later).
__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

template <typename R> struct TileOut {
  cplx<R>* __restrict__ base;
  int64_t es;
  const cplx<R>* __restrict__ mul;
  int64_t vn, ves, voff;
  int64_t l0;
  const cplx<R>* __restrict__ tw_hi;
  const cplx<R>* __restrict__ tw_lo;
  int tw_shift, tw_dir;
  R scale;
  bool ok;
  const cplx<R>* __restrict__ tab;  // full twiddle table (precedence over hi/lo)
  int64_t tab_es, tab_off;
  bool cs;
  __device__ __forceinline__ void operator()(int i, cplx<R> v) const {
    const int64_t vi = (int64_t)i * ves + voff;
    if (!ok || vi >= vn) return;
    if (mul) v = cmul<R>(v, __ldg(mul + vi));
    if (tab) {
      const cplx<R> w = __ldg(tab + (int64_t)i * tab_es + tab_off);
      v = tw_dir < 0 ? cmul<R>(v, w) : cmulc<R>(v, w);
    } else if (tw_hi) {
      const int64_t e = l0 * (int64_t)i;
      const cplx<R> w = cmul<R>(__ldg(tw_hi + (e >> tw_shift)),
                                __ldg(tw_lo + (e & ((int64_t(1) << tw_shift) - 1))));
      v = tw_dir < 0 ? cmul<R>(v, w) : cmulc<R>(v, w);
    }
    if (scale != R(1)) v = cscale<R>(v, scale);
    store<R>(base + (int64_t)i * es, v, cs);
  }
  // Bring the per-element tables element i's store will read (chirp, full
  // twiddle table) into L1 ahead of time; the same presence test as above.
  __device__ __forceinline__ void prefetch(int i) const {
    const int64_t vi = (int64_t)i * ves + voff;
    if (!ok || vi >= vn) return;
    if (mul) prefetch_l1(mul + vi);
    if (tab) prefetch_l1(tab + (int64_t)i * tab_es + tab_off);
  }
};

// Lean I/O for the common case (LineArgs::plain_io): every element present,
// no chirp tables, 32-bit strides, twiddle (if any) from a full table.  The
// line index is clamped to a valid line, so loads need no predicate.
// `tab` is a generic pointer: the twiddle table in global memory, or the
// line's slice of it staged in shared memory (then tab_es = 1, tab_off = 0).
//
// TW fixes at compile time what a functor multiplies by: kTwRuntime tests
// `tab` and `tw_dir` at every element; kTwNone has no table; -1 / +1 always
// apply the table, as w (forward) or conj(w) (backward).  PlainOut's SCALE =
// false leaves out the scale (a scale of 1).  The four-step and 2-D passes
// take the fixed forms, so their unrolled stages carry no per-element tests
// of launch-wide values; the arithmetic is the same in every form.
constexpr int kTwRuntime = 0, kTwNone = 2;
template <typename R, int TW = kTwRuntime> struct PlainIn {
  const cplx<R>* __restrict__ base;
  int es;
  const cplx<R>* tab;  // twiddle on load (LineArgs::tw_on_load)
  int tab_es, tab_off, tw_dir;
  __device__ __forceinline__ bool has_tab() const {
    return TW == kTwRuntime ? tab != nullptr : TW != kTwNone;
  }
  __device__ __forceinline__ cplx<R> twm(cplx<R> v, cplx<R> w) const {
    if constexpr (TW == -1)
      return cmul<R>(v, w);
    else if constexpr (TW == 1)
      return cmulc<R>(v, w);
    else
      return tw_dir < 0 ? cmul<R>(v, w) : cmulc<R>(v, w);
  }
  __device__ __forceinline__ cplx<R> raw(int i) const { return __ldcs(base + (int64_t)(i * es)); }
  __device__ __forceinline__ cplx<R> fin(int i, cplx<R> v) const {
    if (has_tab()) v = twm(v, tab[i * tab_es + tab_off]);
    return v;
  }
  // The twiddles of butterfly j's inputs i = j + r*nb (tw_elem's product):
  // ceil(RAD/4) entries of its own plus the line's steps t(c*nb), c = 1..3.
  template <int RAD>
  __device__ __forceinline__ void fin_bfly(int j, int nb, cplx<R>* v) const {
    if (!has_tab()) return;
    if constexpr (RAD < 4) {
#pragma unroll
      for (int r = 0; r < RAD; ++r) v[r] = fin(j + r * nb, v[r]);
    } else {
      cplx<R> s[4];
#pragma unroll
      for (int c = 1; c < 4; ++c) s[c] = tab[c * nb * tab_es + tab_off];
#pragma unroll
      for (int a = 0; a < RAD; a += 4) {
        const cplx<R> b = tab[(j + a * nb) * tab_es + tab_off];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (a + c < RAD) {
            const cplx<R> w = c == 0 ? b : cmul<R>(b, s[c]);
            v[a + c] = twm(v[a + c], w);
          }
        }
      }
    }
  }
};
template <class In> struct InHasBfly : std::false_type {};
template <typename R, int TW> struct InHasBfly<PlainIn<R, TW>> : std::true_type {};
template <typename R, int TW = kTwRuntime, bool SCALE = true> struct PlainOut {
  cplx<R>* __restrict__ base;
  int es;
  const cplx<R>* tab;
  int tab_es, tab_off, tw_dir;
  R scale;
  bool ok;
  bool cs;
  __device__ __forceinline__ void operator()(int i, cplx<R> v) const {
    if (TW == kTwRuntime ? tab != nullptr : TW != kTwNone) {
      const cplx<R> w = tab[i * tab_es + tab_off];
      if constexpr (TW == -1)
        v = cmul<R>(v, w);
      else if constexpr (TW == 1)
        v = cmulc<R>(v, w);
      else
        v = tw_dir < 0 ? cmul<R>(v, w) : cmulc<R>(v, w);
    }
    if (SCALE && scale != R(1)) v = cscale<R>(v, scale);
    if (ok) store<R>(base + (int64_t)(i * es), v, cs);
  }
};

// Element i of a line held flat (unpadded) in shared memory: the landing
// buffer of a bulk copy (fast_stream_kernel).  Stage 0 then overwrites the
// same buffer in the padded layout, after a barrier.
template <typename R> struct FlatIn {
  const cplx<R>* p;
  __device__ __forceinline__ cplx<R> raw(int i) const { return p[i]; }
  __device__ __forceinline__ cplx<R> fin(int, cplx<R> v) const { return v; }
};
template <class In> struct InIsSmem : std::false_type {};
template <typename R> struct InIsSmem<FlatIn<R>> : std::true_type {};

// ------------------------------------------------------------- stages
// Stage S of program RL on one line held at `buf` (padded layout).  Thread u
// of T owns butterflies j = u + q*T.  The first stage takes its inputs from
// `in` unless it is SmemIO; the last stage gives its outputs to `out` unless
// it is SmemIO.
// TC: stage 0 is the radix-16 DFT on the tensor cores (tc::tc_dft16, context
// *tcx) instead of the FP32 butterfly.
template <typename R, int DIR, class RL, int S, int T, class In, class Out, bool TC = false>
__device__ __forceinline__ void fast_stage(cplx<R>* buf, const In& in, const Out& out,
                                           const cplx<R>* __restrict__ tw, const R* pcs, int u,
                                           const tc::TcCtx* tcx = nullptr) {
  constexpr int L = prog_len<RL>();
  constexpr int RAD = RL::r[S];
  constexpr int Ns = ns_before<RL, S>();
  constexpr int nb = L / RAD;
  constexpr int UM = (nb + T - 1) / T;
  constexpr bool GIN = S == 0 && !std::is_same<In, SmemIO>::value;
  constexpr bool GOUT = S == RL::n - 1 && !std::is_same<Out, SmemIO>::value;
  static_assert(!TC || (S == 0 && RAD == 16 && UM == 1 && nb == T && std::is_same<R, float>::value),
                "the tensor-core stage is a first radix-16 stage, one butterfly per thread");
  cplx<R> v[UM][RAD];
#pragma unroll
  for (int q = 0; q < UM; ++q) {
    const int j = u + q * T;
    if (nb % T == 0 || j < nb) {
#pragma unroll
      for (int r = 0; r < RAD; ++r) {
        if constexpr (GIN)
          v[q][r] = in.raw(j + r * nb);
        else
          v[q][r] = buf[pidx<RL>(j + r * nb)];
      }
    }
  }
  if constexpr (GIN) {
#pragma unroll
    for (int q = 0; q < UM; ++q) {
      const int j = u + q * T;
      if (nb % T == 0 || j < nb) {
        if constexpr (InHasBfly<In>::value) {
          in.template fin_bfly<RAD>(j, nb, v[q]);
        } else {
#pragma unroll
          for (int r = 0; r < RAD; ++r) v[q][r] = in.fin(j + r * nb, v[q][r]);
        }
      }
    }
  }
  // in place: all reads of the line finish before any write, unless one side
  // is global memory
  if constexpr ((!GIN || InIsSmem<In>::value) && !GOUT) __syncthreads();
#pragma unroll
  for (int q = 0; q < UM; ++q) {
    const int j = u + q * T;
    if (nb % T == 0 || j < nb) {
      const int k = (Ns == 1) ? 0 : j % Ns;
      if constexpr (Ns > 1) {
        const cplx<R>* w = tw + tw_offset<RL, S>() + k;  // entry (r-1)*Ns + k
#pragma unroll
        for (int r = 1; r < RAD; ++r) v[q][r] = ctw<R, DIR>(v[q][r], __ldg(w + (r - 1) * Ns));
      }
      if constexpr (TC)
        tc::tc_dft16(v[q], *tcx);
      else
        butterfly<R, RAD, DIR>(v[q], pcs);
      const int base = (j - k) * RAD + k;
#pragma unroll
      for (int r = 0; r < RAD; ++r) {
        if constexpr (GOUT)
          out(base + r * Ns, v[q][r]);
        else
          buf[pidx<RL>(base + r * Ns)] = v[q][r];
      }
    }
  }
  if constexpr (!GOUT) __syncthreads();
}

template <typename R, int DIR, class RL, int T, class In, class Out, int S = 0, bool TC = false>
__device__ __forceinline__ void fast_prog(cplx<R>* buf, const In& in, const Out& out,
                                          const cplx<R>* tw, const R* pcs, int u,
                                          const tc::TcCtx* tcx = nullptr) {
  fast_stage<R, DIR, RL, S, T, In, Out, TC && S == 0>(buf, in, out, tw, pcs, u, tcx);
  if constexpr (S + 1 < RL::n)
    fast_prog<R, DIR, RL, T, In, Out, S + 1, TC>(buf, in, out, tw, pcs, u, tcx);
}

// Prefetch the store-time tables of the elements thread u stores in the last
// stage (the index pattern of fast_stage's last stage), so that their loads
// overlap the first loads and the stages: in a launch of about one wave every
// block reaches its stores at the same time, and the table loads there would
// otherwise wait out the memory latency with nothing else to run.
template <typename R, class RL, int T>
__device__ __forceinline__ void prefetch_store_tables(const TileOut<R>& o, int u) {
  if (!o.ok || !(o.mul || o.tab)) return;
  constexpr int S = RL::n - 1;
  constexpr int RAD = RL::r[S];
  constexpr int Ns = ns_before<RL, S>();
  constexpr int nb = prog_len<RL>() / RAD;
  constexpr int UM = (nb + T - 1) / T;
#pragma unroll
  for (int q = 0; q < UM; ++q) {
    const int j = u + q * T;
    if (nb % T == 0 || j < nb) {
      const int k = (Ns == 1) ? 0 : j % Ns;
      const int base = (j - k) * RAD + k;
#pragma unroll
      for (int r = 0; r < RAD; ++r) o.prefetch(base + r * Ns);
    }
  }
}

// ------------------------------------------------------ direct kernel
// Blocks hold 256 threads (G = 256/T lines) for T <= 256, one line otherwise.
// ComplexF32 blocks of 256 threads are held to 64 registers so four fit per
// SM; ComplexF64 needs twice the registers per value.
template <typename R, int T> struct DirectBounds {
  static constexpr int threads = T >= 256 ? T : 256;
  static constexpr int min_blocks = T >= 512 ? 1 : (sizeof(R) == 4 ? 4 : 2);
};

template <typename R, int DIR, class RL, int T>
__global__ void __launch_bounds__(DirectBounds<R, T>::threads, DirectBounds<R, T>::min_blocks)
    fast_direct_kernel(const FastArgs a) {
  typedef cplx<R> C;
  constexpr int LPAD = lpad_of(prog_len<RL>());
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw + threadIdx.y * LPAD;
  const int64_t line = (int64_t)blockIdx.x * a.G + threadIdx.y;
  const bool ok = line < a.nlines;
  const int64_t l = ok ? line : 0;
  const C* gin = (const C*)a.in + l * a.idist;
  C* gout = (C*)a.out + l * a.odist;
  if (a.ndesc > 0) {
    // grouped launch: find the request owning this line (binary search)
    int lo = 0, hi = a.ndesc - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(a.pre + mid) <= l)
        lo = mid;
      else
        hi = mid - 1;
    }
    const int64_t k = l - __ldg(a.pre + lo);
    gin = (const C*)a.ins[lo] + k * a.idist;
    gout = (C*)a.outs[lo] + k * a.odist;
  }
  const DirectIn<R> in{gin, ok};
  const DirectOut<R> out{gout, ok, (R)a.scale, a.st_stream != 0};
  fast_prog<R, DIR, RL, T>(buf, in, out, (const C*)a.tw, (const R*)a.prime_cs, threadIdx.x);
}

// ------------------------------------------------------ stream kernel
// Persistent variant of the direct kernel for contiguous lines whose bytes
// start on 16-byte boundaries.  Block b transforms lines b, b + gridDim.x, ...
// One thread keeps NBUF-1 lines ahead in flight as bulk asynchronous copies
// (cp.async.bulk global -> shared, completion counted in bytes on one
// mbarrier per buffer), so HBM reads continue while the block computes.
// Stage 0 reads the flat copy, the later stages the padded layout in the same
// buffer, and the last stage stores to HBM from registers.  The arithmetic is
// that of the other kernels.  Every wait is bounded: after about a second the
// block sets kErrWaitTimeout, waits (again bounded) for its copies in flight
// and returns.

template <typename R, class RL> struct StreamShape {
  static constexpr int L = prog_len<RL>();
  static constexpr uint32_t bytes = (uint32_t)(L * sizeof(cplx<R>));
  // buffer stride: the padded line, rounded to 128 bytes
  static constexpr size_t stride = ((size_t)lpad_of(L) * sizeof(cplx<R>) + 127) / 128 * 128;
  static constexpr int nbuf = 2;
  static constexpr size_t smem = 128 + nbuf * stride;
  // lines of at least 4 KB, whole 16-byte units, two blocks per SM
  static constexpr bool ok = bytes >= 4096 && bytes % 16 == 0 && smem <= 110 * 1024;
};
// Resident blocks per SM asked of the compiler: as many as shared memory
// allows (227 KB, 1 KB reserved per block), at most 2048 threads, and never
// below 64 registers per thread.
template <typename R, class RL, int T> struct StreamBounds {
  static constexpr int by_smem = (int)(232448 / (StreamShape<R, RL>::smem + 1024));
  static constexpr int by_thr = 2048 / T;
  static constexpr int by_reg = 65536 / (T * 64);
  static constexpr int m0 = by_smem < by_thr ? by_smem : by_thr;
  static constexpr int m1 = m0 < by_reg ? m0 : by_reg;
  static constexpr int min_blocks = m1 < 1 ? 1 : m1;
};

template <typename R, int DIR, class RL, int T>
__global__ void __launch_bounds__(T, StreamBounds<R, RL, T>::min_blocks)
    fast_stream_kernel(const FastArgs a) {
  typedef cplx<R> C;
  typedef StreamShape<R, RL> SS;
  constexpr int NBUF = SS::nbuf;
  extern __shared__ __align__(16) unsigned char smraw[];
  uint64_t* bar = (uint64_t*)smraw;
  auto buffer = [&](int b) { return (C*)(smraw + 128 + (size_t)b * SS::stride); };
  const int u = threadIdx.x;
  const int64_t first = blockIdx.x, step = gridDim.x;
  const int64_t nmine = first < a.nlines ? (a.nlines - 1 - first) / step + 1 : 0;
  const C* gin = (const C*)a.in;
  C* gout = (C*)a.out;
  if (u == 0) {
    for (int b = 0; b < NBUF; ++b) mbar_init(bar + b, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int b = 0; b < NBUF - 1 && b < nmine; ++b) {
      mbar_expect_tx(bar + b, SS::bytes);
      bulk_load(buffer(b), gin + (first + b * step) * a.idist, SS::bytes, bar + b);
    }
  }
  __syncthreads();
  int64_t i = 0;
  for (; i < nmine; ++i) {
    const int b = (int)(i % NBUF);
    const bool got = mbar_wait(bar + b, (uint32_t)((i / NBUF) & 1), a.wait_ns);
    // this thread's writes to line i-1's buffer are ordered before the copy
    // that refills it, and every thread has finished line i-1
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (!__syncthreads_and(got)) break;
    const int64_t nx = i + NBUF - 1;
    if (u == 0 && nx < nmine) {
      const int bb = (int)(nx % NBUF);
      mbar_expect_tx(bar + bb, SS::bytes);
      bulk_load(buffer(bb), gin + (first + nx * step) * a.idist, SS::bytes, bar + bb);
    }
    C* buf = buffer(b);
    const FlatIn<R> in{buf};
    const DirectOut<R> out{gout + (first + i * step) * a.odist, true, (R)a.scale,
                           a.st_stream != 0};
    fast_prog<R, DIR, RL, T>(buf, in, out, (const C*)a.tw, (const R*)a.prime_cs, u);
  }
  if (i < nmine && u == 0) {
    // gave up on line i: flag it, then let the copies still in flight land
    // (waiting at least the default limit, whatever the launch's limit)
    if (a.err) atomicExch(a.err, kErrWaitTimeout);
    for (int64_t k = i; k < nmine && k < i + NBUF - 1; ++k)
      mbar_wait(bar + (int)(k % NBUF), (uint32_t)((k / NBUF) & 1), drain_limit(a.wait_ns));
  }
}

// -------------------------------------------------------- tile kernel
// Most complex values one thread holds in any stage of program RL on T threads.
template <class RL, int T> __host__ __device__ constexpr int max_values() {
  int m = 0;
  for (int i = 0; i < RL::n; ++i) {
    const int nb = prog_len<RL>() / RL::r[i];
    const int v = (nb + T - 1) / T * RL::r[i];
    m = v > m ? v : m;
  }
  return m;
}
// Threads per tile block: up to 512, or 1024 for ComplexF32 lines of 256
// threads outside Bluestein (four lines per block, so that a block covers a
// whole 32-byte sector of each row of a strided axis).
// The Bluestein MID variant (two programs and a product per line) takes at
// most 256 threads per block (or T) at up to 80 registers, three blocks per
// SM: with 512-thread bounds it took 128 registers and a 2048-point line's
// 128-thread blocks ran four per SM.
// The ComplexF32 2048-point MID variant (T = 128) takes one line per block
// at up to 72 registers, seven blocks per SM: the 1024 middle-pass blocks of
// a 2^21-point Bluestein pad then fit one wave of 148 SMs (six blocks per SM
// at 80 registers made it 1.15 waves).
template <typename R, int T> struct MidOneLine {
  static constexpr bool value = sizeof(R) == 4 && T == 128;
};
template <typename R, int T, bool MID> struct TileThreads {
  static constexpr int value = MID ? (T > 256 ? T : (MidOneLine<R, T>::value ? T : 256))
                                   : ((sizeof(R) == 4 && T == 256) ? 1024 : (T > 512 ? T : 512));
};
template <typename R, class RL, int T, bool MID, bool PLAIN> struct TileBounds {
  static constexpr int min_blocks =
      MID ? (MidOneLine<R, T>::value ? 7 : (T <= 256 ? 3 : 1))
          : ((TileThreads<R, T, MID>::value <= 512 && T <= 512 &&
              max_values<RL, T>() <= (sizeof(R) == 4 ? 18 : 9))
                 ? 2
                 : 1);
};
// Whether a tile launch reserves shared memory for a staged twiddle slice:
// only four-step passes whose slice follows the second batch level.
__host__ __device__ inline bool stages_twiddles(const LineArgs& a, int L) {
  return a.tw_tab && a.tw_level == 1 && L <= kStagedTwiddleMax;
}
// Lines of one block that share their twiddle slice (four-step passes over a
// contiguous batch: the slice depends on the line's second batch level only)
// read it from shared memory: stage entries tab[i*tw_es + lt*tw_ls], i < L,
// into `dst` when the block's first and last lines agree on lt.  Returns dst,
// or nullptr (and stages nothing) otherwise.  Every thread calls it.
template <typename C>
__device__ __forceinline__ const C* stage_twiddles(const LineArgs& a, const int64_t* lt_of,
                                                   int G, int L, C* dst, int tid, int nthreads) {
  if (!stages_twiddles(a, L)) return nullptr;
  const int64_t left = a.nlines - (int64_t)blockIdx.x * G;
  const int last = (int)(left < G ? left : G) - 1;
  const int64_t lt = lt_of[0];
  if (lt_of[last] != lt) return nullptr;
  const C* __restrict__ tab = (const C*)a.tw_tab + lt * a.tw_ls;
  for (int i = tid; i < L; i += nthreads) dst[i] = __ldg(tab + (int64_t)i * a.tw_es);
  __syncthreads();
  return dst;
}

// G lines per block addressed like the generic kernel (LineArgs: three batch
// levels, element strides, presence window, tables).  Thread (g, u) is
// threadIdx.x = g, threadIdx.y = u, so a warp spans 32/G butterflies of G
// lines.  MID: forward program, multiply by a.mid, inverse program.
template <typename R, class RL, int T, bool MID, bool PLAIN>
// Blocks of up to 512 threads (except the Bluestein MID variant) are held to
// 64 registers so two fit per SM -- measured faster than one block with more
// registers, also where the full-I/O variant then spills a little -- unless a
// thread holds more than 18 ComplexF32 or 9 ComplexF64 values in some stage.
// 1024-thread blocks (TileThreads) get the same 64 registers.
__global__ void __launch_bounds__(TileThreads<R, T, MID>::value,
                                  TileBounds<R, RL, T, MID, PLAIN>::min_blocks)
    fast_tile_kernel(const LineArgs a) {
  typedef cplx<R> C;
  constexpr int L = prog_len<RL>();
  constexpr int LPAD = lpad_of(L);
  extern __shared__ __align__(16) unsigned char smraw[];
  const int g = threadIdx.x, u = threadIdx.y;
  const int G = a.G, P = tile_pitch(LPAD, G, (int)sizeof(C));
  C* buf = (C*)smraw + g * P;
  // one thread per line splits its index into the batch levels (64-bit
  // divisions) and leaves the results in shared memory for the others
  // (four arrays of G entries, so a warp's reads are consecutive)
  int64_t* lb = (int64_t*)((C*)smraw + (size_t)G * P);
  const int64_t line = (int64_t)blockIdx.x * G + g;
  const bool ok = line < a.nlines;
  if (u == 0) {
    const int64_t l = ok ? line : 0;
    const int64_t q0 = l % a.m0, t = l / a.m0;
    const int64_t q1 = t % a.m1, q2 = t / a.m1;
    lb[g] = q0;
    lb[G + g] = q0 * a.ld.s0 + q1 * a.ld.s1 + q2 * a.ld.s2;
    lb[2 * G + g] = q0 * a.st.s0 + q1 * a.st.s1 + q2 * a.st.s2;
    lb[3 * G + g] = a.tw_level ? q1 : q0;
  }
  __syncthreads();
  const int64_t l0 = lb[g], lt = lb[3 * G + g];
  const C* tw = (const C*)a.prog.tw;
  const R* pcs = (const R*)a.prime_cs;
  const C* ib = (const C*)a.in + lb[G + g];
  C* ob = (C*)a.out + lb[2 * G + g];
  if constexpr (PLAIN && !MID) {
    const C* tin = a.tw_on_load ? (const C*)a.tw_tab : nullptr;
    const C* tout = a.tw_on_load ? nullptr : (const C*)a.tw_tab;
    const C* st = stage_twiddles<C>(a, lb + 3 * G, G, L, (C*)(lb + 4 * G), g + G * u, G * T);
    const int tes = st ? 1 : (int)a.tw_es, toff = st ? 0 : (int)(lt * a.tw_ls);
    const C* ti = tin ? (st ? st : tin) : nullptr;
    const C* to = tout ? (st ? st : tout) : nullptr;
    const int ies = (int)a.ld.es, oes = (int)a.st.es;
    const bool cs = a.st_stream != 0;
    // The lean passes of the four-step and 2-D schedules -- no twiddle, or a
    // twiddle on the loads or on the stores in the transform's direction,
    // and no scale -- run with those choices fixed at compile time; any other
    // lean launch takes the run-time form.
    const bool fixed = (R)a.scale == R(1) && !(ti && to) && (!(ti || to) || a.tw_dir == a.dir1);
    if (fixed && !ti && !to) {
      const PlainIn<R, kTwNone> in{ib, ies, nullptr, 0, 0, 0};
      const PlainOut<R, kTwNone, false> out{ob, oes, nullptr, 0, 0, 0, R(1), ok, cs};
      if (a.dir1 < 0)
        fast_prog<R, -1, RL, T>(buf, in, out, tw, pcs, u);
      else
        fast_prog<R, 1, RL, T>(buf, in, out, tw, pcs, u);
    } else if (fixed && ti) {
      const PlainOut<R, kTwNone, false> out{ob, oes, nullptr, 0, 0, 0, R(1), ok, cs};
      if (a.dir1 < 0)
        fast_prog<R, -1, RL, T>(buf, PlainIn<R, -1>{ib, ies, ti, tes, toff, -1}, out, tw, pcs, u);
      else
        fast_prog<R, 1, RL, T>(buf, PlainIn<R, 1>{ib, ies, ti, tes, toff, 1}, out, tw, pcs, u);
    } else if (fixed) {
      const PlainIn<R, kTwNone> in{ib, ies, nullptr, 0, 0, 0};
      if (a.dir1 < 0)
        fast_prog<R, -1, RL, T>(buf, in, PlainOut<R, -1, false>{ob, oes, to, tes, toff, -1, R(1), ok, cs},
                                tw, pcs, u);
      else
        fast_prog<R, 1, RL, T>(buf, in, PlainOut<R, 1, false>{ob, oes, to, tes, toff, 1, R(1), ok, cs},
                               tw, pcs, u);
    } else {
      const PlainIn<R> in{ib, ies, ti, tes, toff, a.tw_dir};
      const PlainOut<R> out{ob, oes, to, tes, toff, a.tw_dir, (R)a.scale, ok, cs};
      if (a.dir1 < 0)
        fast_prog<R, -1, RL, T>(buf, in, out, tw, pcs, u);
      else
        fast_prog<R, 1, RL, T>(buf, in, out, tw, pcs, u);
    }
  } else {
    const C* tin = a.tw_on_load ? (const C*)a.tw_tab : nullptr;
    const C* tout = a.tw_on_load ? nullptr : (const C*)a.tw_tab;
    const TileIn<R> in{ib, a.ld.es, (const C*)a.ld.mul, a.ld.vn, a.ld.ves, l0 * a.ld.vls, ok,
                       tin, a.tw_es, lt * a.tw_ls, a.tw_dir};
    const TileOut<R> out{ob, a.st.es, (const C*)a.st.mul, a.st.vn, a.st.ves, l0 * a.st.vls, lt,
                         a.tw_N ? (const C*)a.tw_hi : nullptr, (const C*)a.tw_lo, a.tw_shift,
                         a.tw_dir, (R)a.scale, ok, tout, a.tw_es, lt * a.tw_ls,
                         a.st_stream != 0};
    prefetch_store_tables<R, RL, T>(out, u);
    if constexpr (MID) {
      const C* __restrict__ mid = (const C*)a.mid;
      if (ok)
        for (int k = u; k < L; k += T) prefetch_l1(mid + l0 * a.mid_ls + (int64_t)k * a.mid_es);
      fast_prog<R, -1, RL, T>(buf, in, SmemIO{}, tw, pcs, u);
      for (int k = u; k < L; k += T)
        buf[pidx<RL>(k)] = cmul<R>(buf[pidx<RL>(k)], __ldg(mid + l0 * a.mid_ls + (int64_t)k * a.mid_es));
      __syncthreads();
      fast_prog<R, 1, RL, T>(buf, SmemIO{}, out, tw, pcs, u);
    } else {
      if (a.dir1 < 0)
        fast_prog<R, -1, RL, T>(buf, in, out, tw, pcs, u);
      else
        fast_prog<R, 1, RL, T>(buf, in, out, tw, pcs, u);
    }
  }
}

// ------------------------------------------------------- real kernel
// Half-length real transforms of contiguous lines of even length n = 2L, as
// FFTA computes them (src/plan.jl:398-442 and :466-495, after Sorensen et
// al.): rfft reads the real line as L complex values z[m] = x[2m] + i x[2m+1]
// (no conversion pass), transforms them with the length-L program into
// shared memory and splits Z into the n/2+1 outputs
//   X[k]   = XX + w^k XY,  X[L-k] = conj(XX - w^k XY),
//   XX = (Z[k] + conj Z[L-k]) / 2,  XY = i (conj Z[L-k] - Z[k]) / 2,
//   X[0] = Re Z[0] + Im Z[0],  X[L] = Re Z[0] - Im Z[0],  w = exp(-2 pi i / n);
// brfft builds Zb[k] = XX + i XY, Zb[L-k] = conj(XX - i XY) with
// XX = Y[k] + conj Y[L-k], XY = w^-k (Y[k] - conj Y[L-k]) and
// Zb[0] = (Re Y[0] + Re Y[L]) + i (Re Y[0] - Re Y[L]) in shared memory,
// runs the inverse program and stores the L complex results as the 2L reals.
// One HBM read and one write per element, as in the complex kernel, at half
// its length.  w^k comes from a table computed in FP64 and rounded once.
template <typename R, int DIR, class RL, int T>
__global__ void __launch_bounds__(DirectBounds<R, T>::threads, DirectBounds<R, T>::min_blocks)
    fast_real_kernel(const RealArgs a) {
  typedef cplx<R> C;
  typedef Sc<R> S;
  constexpr int L = prog_len<RL>();
  constexpr int LPAD = lpad_of(L);
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw + threadIdx.y * LPAD;
  const int64_t line = (int64_t)blockIdx.x * a.G + threadIdx.y;
  const bool ok = line < a.nlines;
  const int64_t l = ok ? line : 0;
  const int u = threadIdx.x;
  const C* tw = (const C*)a.tw;
  const R* pcs = (const R*)a.prime_cs;
  const C* __restrict__ wk = (const C*)a.wk;
  const R h = R(0.5), sc = (R)a.scale;
  const bool cs = a.st_stream != 0;
  if constexpr (DIR < 0) {
    const DirectIn<R> in{(const C*)((const R*)a.in + l * a.idist), ok};
    fast_prog<R, -1, RL, T>(buf, in, SmemIO{}, tw, pcs, u);
    if (!ok) return;  // (no barrier follows)
    C* o = (C*)a.out + l * a.odist;
    for (int k = u; k <= L / 2; k += T) {
      if (k == 0) {
        const C z = buf[pidx<RL>(0)];
        store<R>(o, S::mk(S::mul(S::add(z.x, z.y), sc), R(0)), cs);
        store<R>(o + L, S::mk(S::mul(S::sub(z.x, z.y), sc), R(0)), cs);
        continue;
      }
      const C A = buf[pidx<RL>(k)], B = buf[pidx<RL>(L - k)];
      const C xx = S::mk(S::mul(h, S::add(A.x, B.x)), S::mul(h, S::sub(A.y, B.y)));
      // XY = i * (conj B - A) / 2
      const C xy = S::mk(S::mul(h, S::add(B.y, A.y)), S::mul(h, S::sub(B.x, A.x)));
      const C wxy = cmul<R>(__ldg(wk + k), xy);
      store<R>(o + k, cscale<R>(cadd<R>(xx, wxy), sc), cs);
      if (k != L - k) {
        const C d = csub<R>(xx, wxy);
        store<R>(o + (L - k), cscale<R>(S::mk(d.x, -d.y), sc), cs);
      }
    }
  } else {
    const C* __restrict__ y = (const C*)a.in + l * a.idist;
    for (int k = u; k <= L / 2; k += T) {
      if (k == 0) {
        const R a0 = ok ? __ldcs(y).x : R(0), aL = ok ? __ldcs(y + L).x : R(0);
        buf[pidx<RL>(0)] = S::mk(S::add(a0, aL), S::sub(a0, aL));
        continue;
      }
      const C A = ok ? __ldcs(y + k) : S::mk(R(0), R(0));
      const C B = ok ? __ldcs(y + (L - k)) : S::mk(R(0), R(0));
      const C xx = S::mk(S::add(A.x, B.x), S::sub(A.y, B.y));
      const C dd = S::mk(S::sub(A.x, B.x), S::add(A.y, B.y));
      const C xy = cmulc<R>(dd, __ldg(wk + k));  // w^-k (Y[k] - conj Y[L-k])
      const C ixy = S::mk(-xy.y, xy.x);
      buf[pidx<RL>(k)] = cadd<R>(xx, ixy);
      if (k != L - k) {
        const C d = csub<R>(xx, ixy);
        buf[pidx<RL>(L - k)] = S::mk(d.x, -d.y);
      }
    }
    __syncthreads();
    const DirectOut<R> out{(C*)((R*)a.out + l * a.odist), ok, sc, cs};
    fast_prog<R, 1, RL, T>(buf, SmemIO{}, out, tw, pcs, u);
  }
}

// ------------------------------------------------------ TMA tile kernel
// The lean tile kernel for passes whose lines are neighbours in memory
// (four-step columns, strided 2-D axes): instead of each thread loading its
// butterfly's inputs from HBM (short strided segments whose latency the
// block then waits out), one thread issues tensor copies
// (cp.async.bulk.tensor) of whole tiles -- G neighbouring lines x L elements
// -- into shared memory, `nbuf` tiles ahead, each completing on an mbarrier.
// Blocks are persistent: block b transforms tiles b, b + gridDim.x, ...  So
// HBM keeps streaming the next tiles while the block computes this one.
// The first stage reads the landed tile (element i of line g at t[i*G + g]),
// then every stage runs as in fast_tile_kernel, in the same buffer, and the
// last stage stores to HBM from registers; the arithmetic is the same, so
// results equal the other kernels' bit for bit.  Tensor maps cover this GPU's
// own memory only, and each copy lands in its own block's shared memory.
// Every wait is bounded: a block that gives up sets kErrWaitTimeout, drains
// its copies in flight (at least the default limit) and returns.

// One box of a 4-D tensor map (x: lines in 8-byte units, y: elements of the
// line, z/w: batch levels) into shared memory, completing on *bar.
__device__ __forceinline__ void tma_load_4d(void* dst, const void* tmap, int x, int y, int z,
                                            int w, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(z), "r"(w),
      "r"(smem_addr(bar))
      : "memory");
}

// Element i of line g read from a landed tile (this thread's line: t + g,
// stride G); the four-step twiddle on the loads as PlainIn applies it.
template <typename R> struct TmaIn : PlainIn<R> {
  __device__ __forceinline__ cplx<R> raw(int i) const { return this->base[i * this->es]; }
};
template <typename R> struct InHasBfly<TmaIn<R>> : std::true_type {};
template <typename R> struct InIsSmem<TmaIn<R>> : std::true_type {};

template <typename R, class RL, int T>
__global__ void __launch_bounds__(TileThreads<R, T, false>::value,
                                  TileBounds<R, RL, T, false, true>::min_blocks)
    fast_tma_tile_kernel(const LineArgs a, const __grid_constant__ CUtensorMap tm,
                         const TmaGeom q) {
  typedef cplx<R> C;
  constexpr int L = prog_len<RL>();
  constexpr int LPAD = lpad_of(L);
  // the buffers start 128-byte aligned (tensor copies land there); the
  // launch reserves 128 bytes for the adjustment
  extern __shared__ __align__(16) unsigned char smtma[];
  unsigned char* smraw = smtma + ((128u - (smem_addr(smtma) & 127u)) & 127u);
  const int g = threadIdx.x, u = threadIdx.y, G = a.G;
  const int tid = g + G * u;
  const int P = tile_pitch(LPAD, G, (int)sizeof(C));
  uint64_t* bar = (uint64_t*)(smraw + (size_t)q.nbuf * q.buf_bytes);
  const int64_t first = blockIdx.x, step = gridDim.x;
  const int64_t nmine = first < q.ntiles ? (q.ntiles - 1 - first) / step + 1 : 0;
  const uint32_t tile_bytes = (uint32_t)(L * G * (int)sizeof(C));
  const uint32_t box_bytes = (uint32_t)(q.boxr * G * (int)sizeof(C));
  // the copies of this block's k-th tile into buffer b (thread 0 only)
  auto issue = [&](int64_t k, int b) {
    const int64_t line = (first + k * step) * G;
    const int64_t q0 = line % a.m0, t = line / a.m0;
    const int64_t q1 = t % a.m1, q2 = t / a.m1;
    unsigned char* dst = smraw + (size_t)b * q.buf_bytes;
    mbar_expect_tx(bar + b, tile_bytes);
    for (int r = 0; r < q.nbox; ++r)
      tma_load_4d(dst + (size_t)r * box_bytes, &tm, (int)(q0 * q.units), r * q.boxr, (int)q1,
                  (int)q2, bar + b);
  };
  if (tid == 0) {
    for (int b = 0; b < q.nbuf; ++b) mbar_init(bar + b, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int b = 0; b < q.nbuf - 1 && b < nmine; ++b) issue(b, b);
  }
  __syncthreads();
  const C* tw = (const C*)a.prog.tw;
  const R* pcs = (const R*)a.prime_cs;
  const C* tin = a.tw_on_load ? (const C*)a.tw_tab : nullptr;
  const C* tout = a.tw_on_load ? nullptr : (const C*)a.tw_tab;
  int64_t k = 0;
  for (; k < nmine; ++k) {
    const int b = (int)(k % q.nbuf);
    const bool got = mbar_wait(bar + b, (uint32_t)((k / q.nbuf) & 1), a.wait_ns);
    // this thread's writes to tile k-1's buffer (its stage exchanges) are
    // ordered before the tensor copy that refills it ...
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    // ... and every thread has finished tile k-1
    if (!__syncthreads_and(got)) break;
    const int64_t nx = k + q.nbuf - 1;
    if (tid == 0 && nx < nmine) issue(nx, (int)(nx % q.nbuf));
    const int64_t line = (first + k * step) * G + g;
    const int64_t q0 = line % a.m0, t = line / a.m0;
    const int64_t q1 = t % a.m1, q2 = t / a.m1;
    const int64_t lt = a.tw_level ? q1 : q0;
    C* tile = (C*)(smraw + (size_t)b * q.buf_bytes);
    TmaIn<R> in;
    in.base = tile + g;
    in.es = G;
    in.tab = tin;
    in.tab_es = (int)a.tw_es;
    in.tab_off = (int)(lt * a.tw_ls);
    in.tw_dir = a.tw_dir;
    const PlainOut<R> out{(C*)a.out + q0 * a.st.s0 + q1 * a.st.s1 + q2 * a.st.s2, (int)a.st.es,
                          tout, (int)a.tw_es, (int)(lt * a.tw_ls), a.tw_dir, (R)a.scale, true,
                          a.st_stream != 0};
    if (a.dir1 < 0)
      fast_prog<R, -1, RL, T>(tile + g * P, in, out, tw, pcs, u);
    else
      fast_prog<R, 1, RL, T>(tile + g * P, in, out, tw, pcs, u);
  }
  if (k < nmine && tid == 0) {
    // gave up on tile k: flag it, then let the copies still in flight land
    if (a.err) atomicExch(a.err, kErrWaitTimeout);
    for (int64_t j = k; j < nmine && j < k + q.nbuf - 1; ++j)
      mbar_wait(bar + (int)(j % q.nbuf), (uint32_t)((j / q.nbuf) & 1), drain_limit(a.wait_ns));
  }
}

// ------------------------------------------------ tensor-core variants
// The direct kernel and the lean-I/O tile kernel with their first radix-16
// stage on the tensor cores (tc::tc_dft16).  Shared memory: the stage's A
// operand and the line buffers share the first region (lines are written
// only after the products complete), then (tile kernel) the per-line
// offsets, the B table, the mbarrier and the tensor-memory address.
template <class RL, int T> struct TcShape {
  static constexpr int L = prog_len<RL>();
  __host__ __device__ static constexpr size_t line_bytes(int G) {
    return (size_t)tile_pitch(lpad_of(L), G, 8) * 8;
  }
  static constexpr bool first16 = RL::r[0] == 16 && L / 16 == T;  // one butterfly per thread
  static constexpr bool direct_ok = first16 && T % 128 == 0 && T <= 512;
  static constexpr bool tile_ok = first16 && T <= 512 && 512 % T == 0;
  __host__ __device__ static constexpr size_t region(int G) {
    return ((((size_t)G * line_bytes(G) > (size_t)G * T * tc::kTcRowBytes)
                 ? (size_t)G * line_bytes(G)
                 : (size_t)G * T * tc::kTcRowBytes) +
            127) / 128 * 128;
  }
  __host__ __device__ static constexpr size_t direct_smem() {
    return region(1) + tc::kTcTableBytes + 16;
  }
  __host__ __device__ static constexpr size_t tile_smem(int G, bool staged) {
    return region(G) + (size_t)G * 32 + tc::kTcTableBytes + 16 + (staged ? (size_t)L * 8 : 0);
  }
  static constexpr int direct_blocks =
      (int)(232448 / (direct_smem() + 1024)) < 1 ? 1 : (int)(232448 / (direct_smem() + 1024));
};

template <int DIR, class RL, int T>
__global__ void __launch_bounds__(T, TcShape<RL, T>::direct_blocks)
    fast_tc_direct_kernel(const FastArgs a) {
  typedef cplx<float> C;
  typedef TcShape<RL, T> TS;
  extern __shared__ __align__(16) unsigned char smraw[];
  unsigned char* b = smraw + TS::region(1);
  uint64_t* bar = (uint64_t*)(b + tc::kTcTableBytes);
  uint32_t* slot = (uint32_t*)(bar + 1);
  const int u = threadIdx.x;
  const tc::TcCtx c =
      tc::tc_begin(smraw, b, bar, slot,
                   (const unsigned char*)a.tcb + (DIR < 0 ? 0 : tc::kTcTableBytes), a.err, u, T,
                   a.wait_ns);
  const int64_t line = blockIdx.x;  // grid = lines
  const DirectIn<float> in{(const C*)a.in + line * a.idist, true};
  const DirectOut<float> out{(C*)a.out + line * a.odist, true, (float)a.scale, a.st_stream != 0};
  fast_prog<float, DIR, RL, T, DirectIn<float>, DirectOut<float>, 0, true>(
      (C*)smraw, in, out, (const C*)a.tw, (const float*)a.prime_cs, u, &c);
  tc::tc_end(c);
}

template <class RL, int T>
__global__ void __launch_bounds__(512, 2) fast_tc_tile_kernel(const LineArgs a) {
  typedef cplx<float> C;
  typedef TcShape<RL, T> TS;
  constexpr int LPAD = lpad_of(prog_len<RL>());
  extern __shared__ __align__(16) unsigned char smraw[];
  const int g = threadIdx.x, u = threadIdx.y, G = a.G;
  const size_t reg = TS::region(G);
  int64_t* lb = (int64_t*)(smraw + reg);
  unsigned char* b = smraw + reg + (size_t)G * 32;
  uint64_t* bar = (uint64_t*)(b + tc::kTcTableBytes);
  uint32_t* slot = (uint32_t*)(bar + 1);
  C* buf = (C*)smraw + g * tile_pitch(LPAD, G, 8);
  const int64_t line = (int64_t)blockIdx.x * G + g;
  const bool ok = line < a.nlines;
  if (u == 0) {
    const int64_t l = ok ? line : 0;
    const int64_t q0 = l % a.m0, t = l / a.m0;
    const int64_t q1 = t % a.m1, q2 = t / a.m1;
    lb[G + g] = q0 * a.ld.s0 + q1 * a.ld.s1 + q2 * a.ld.s2;
    lb[2 * G + g] = q0 * a.st.s0 + q1 * a.st.s1 + q2 * a.st.s2;
    lb[3 * G + g] = a.tw_level ? q1 : q0;
  }
  // (tc_begin's barrier publishes lb)
  const tc::TcCtx c = tc::tc_begin(
      smraw, b, bar, slot, (const unsigned char*)a.tcb + (a.dir1 < 0 ? 0 : tc::kTcTableBytes),
      a.err, g + G * u, G * T, a.wait_ns);
  const int64_t lt = lb[3 * G + g];
  const C* tin = a.tw_on_load ? (const C*)a.tw_tab : nullptr;
  const C* tout = a.tw_on_load ? nullptr : (const C*)a.tw_tab;
  const C* st = stage_twiddles<C>(a, lb + 3 * G, G, prog_len<RL>(), (C*)(slot + 2), g + G * u,
                                  G * T);
  const int tes = st ? 1 : (int)a.tw_es, toff = st ? 0 : (int)(lt * a.tw_ls);
  const PlainIn<float> in{(const C*)a.in + lb[G + g], (int)a.ld.es,
                          tin ? (st ? st : tin) : nullptr, tes, toff, a.tw_dir};
  const PlainOut<float> out{(C*)a.out + lb[2 * G + g], (int)a.st.es,
                            tout ? (st ? st : tout) : nullptr, tes, toff, a.tw_dir,
                            (float)a.scale, ok, a.st_stream != 0};
  const C* tw = (const C*)a.prog.tw;
  const float* pcs = (const float*)a.prime_cs;
  if (a.dir1 < 0)
    fast_prog<float, -1, RL, T, PlainIn<float>, PlainOut<float>, 0, true>(buf, in, out, tw, pcs,
                                                                          u, &c);
  else
    fast_prog<float, 1, RL, T, PlainIn<float>, PlainOut<float>, 0, true>(buf, in, out, tw, pcs,
                                                                         u, &c);
  tc::tc_end(c);
}

// Refuse a tensor-core launch whose resident blocks could ask for more than
// the SM's 512 tensor-memory columns (an allocation would then wait).
template <typename K> static cudaError_t tc_check_columns(K k, int threads, size_t smem, uint32_t cols) {
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem);
  if (e != cudaSuccess) return e;
  return (per_sm >= 1 && (uint32_t)per_sm * cols <= 512u) ? cudaSuccess
                                                          : cudaErrorInvalidConfiguration;
}

// ---------------------------------------------------------- launching
// Raise a kernel's dynamic shared-memory limit when a launch needs more than
// the default 48 KB.  `set` is the caller's per-kernel, per-device record.
template <typename K> static cudaError_t configure(K k, size_t smem, int* set) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (smem <= 48 * 1024 || (dev < 64 && set[dev] >= (int)smem)) return cudaSuccess;
  e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess && dev < 64) set[dev] = (int)smem;
  return e;
}

// Describe a failed launch: the launch shape and the kernel's attributes.
template <typename K>
static void launch_failure(K k, const char* what, int L, int T, int G, size_t smem, cudaError_t e) {
  cudaFuncAttributes fa;
  memset(&fa, 0, sizeof(fa));
  cudaFuncGetAttributes(&fa, k);
  snprintf(g_launch_msg, sizeof(g_launch_msg),
           "%s L=%d T=%d G=%d smem=%zu: %s (kernel maxThreads=%d regs=%d maxDynSmem=%d)", what, L,
           T, G, smem, cudaGetErrorString(e), fa.maxThreadsPerBlock, fa.numRegs,
           fa.maxDynamicSharedSizeBytes);
}

template <typename R, class RL, int T> struct FastEntry {
  static constexpr int L = prog_len<RL>();
  static constexpr int LPAD = lpad_of(L);
  static constexpr int TILE_THREADS = TileThreads<R, T, false>::value;
  static cudaError_t launch(int dir, const FastArgs& a, cudaStream_t s) {
    static int set_fwd[64] = {0}, set_bwd[64] = {0};
    const size_t smem = (size_t)a.G * LPAD * sizeof(cplx<R>);
    auto k = dir < 0 ? fast_direct_kernel<R, -1, RL, T> : fast_direct_kernel<R, 1, RL, T>;
    if (a.G * T > DirectBounds<R, T>::threads) {
      launch_failure(k, "direct launch shape", L, T, a.G, smem, cudaErrorInvalidValue);
      return cudaErrorInvalidValue;
    }
    cudaError_t e = configure(k, smem, dir < 0 ? set_fwd : set_bwd);
    if (e != cudaSuccess) {
      launch_failure(k, "direct smem attribute", L, T, a.G, smem, e);
      return e;
    }
    const int64_t nblk = (a.nlines + a.G - 1) / a.G;
    if (nblk <= 0) return cudaSuccess;
    k<<<dim3((unsigned)nblk), dim3(T, a.G), smem, s>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) launch_failure(k, "direct launch", L, T, a.G, smem, e);
    return e;
  }
  // Persistent launch: as many blocks as fit on the device at once (or one
  // per line, if fewer).
  static cudaError_t launch_stream(int dir, const FastArgs& a, cudaStream_t s) {
    if constexpr (!StreamShape<R, RL>::ok) {
      snprintf(g_launch_msg, sizeof(g_launch_msg), "no stream kernel for L=%d", L);
      return cudaErrorNotSupported;
    } else {
      static int set_fwd[64] = {0}, set_bwd[64] = {0}, occ[2][64] = {{0}};
      constexpr size_t smem = StreamShape<R, RL>::smem;
      auto k = dir < 0 ? fast_stream_kernel<R, -1, RL, T> : fast_stream_kernel<R, 1, RL, T>;
      int dev = 0;
      cudaError_t e = cudaGetDevice(&dev);
      if (e == cudaSuccess) e = configure(k, smem, dir < 0 ? set_fwd : set_bwd);
      int* o = dev < 64 ? &occ[dir < 0 ? 0 : 1][dev] : nullptr;
      int per_sm = o ? *o : 0;
      if (e == cudaSuccess && per_sm == 0) {
        int nsm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, T, smem);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        per_sm = per_sm * nsm;
        if (o) *o = per_sm;
      }
      if (e != cudaSuccess || per_sm <= 0) {
        if (e == cudaSuccess) e = cudaErrorInvalidConfiguration;
        launch_failure(k, "stream set-up", L, T, 1, smem, e);
        return e;
      }
      if (a.nlines <= 0) return cudaSuccess;
      const int64_t nblk = a.nlines < per_sm ? a.nlines : per_sm;
      k<<<dim3((unsigned)nblk), dim3(T), smem, s>>>(a);
      e = cudaGetLastError();
      if (e != cudaSuccess) launch_failure(k, "stream launch", L, T, 1, smem, e);
      return e;
    }
  }
  // Half-length real kernel: lines of 2L for L up to 8192 (one block of at
  // most 512 threads per line).
  static constexpr bool has_real = L >= 2 && T <= 512;
  static cudaError_t launch_real(int dir, const RealArgs& a, cudaStream_t s) {
    if constexpr (!has_real) {
      snprintf(g_launch_msg, sizeof(g_launch_msg), "no real kernel for L=%d", L);
      return cudaErrorNotSupported;
    } else {
      static int set_fwd[64] = {0}, set_bwd[64] = {0};
      const size_t smem = (size_t)a.G * LPAD * sizeof(cplx<R>);
      auto k = dir < 0 ? fast_real_kernel<R, -1, RL, T> : fast_real_kernel<R, 1, RL, T>;
      if (a.G < 1 || a.G * T > DirectBounds<R, T>::threads) {
        launch_failure(k, "real launch shape", L, T, a.G, smem, cudaErrorInvalidValue);
        return cudaErrorInvalidValue;
      }
      cudaError_t e = configure(k, smem, dir < 0 ? set_fwd : set_bwd);
      if (e != cudaSuccess) {
        launch_failure(k, "real smem attribute", L, T, a.G, smem, e);
        return e;
      }
      const int64_t nblk = (a.nlines + a.G - 1) / a.G;
      if (nblk <= 0) return cudaSuccess;
      k<<<dim3((unsigned)nblk), dim3(T, a.G), smem, s>>>(a);
      e = cudaGetLastError();
      if (e != cudaSuccess) launch_failure(k, "real launch", L, T, a.G, smem, e);
      return e;
    }
  }
  // Tensor-copy tile kernel: lengths 8..4096 (longer lines leave no room for
  // a second tile buffer).  As many persistent blocks as fit at once, at most
  // one per tile.
  static constexpr bool has_tma = L >= 8 && L <= 4096;
  static cudaError_t launch_tile_tma(const LineArgs& a, const void* tmap, const TmaGeom& q,
                                     cudaStream_t s) {
    if constexpr (!has_tma) {
      snprintf(g_launch_msg, sizeof(g_launch_msg), "no tensor-copy tile kernel for L=%d", L);
      return cudaErrorNotSupported;
    } else {
      static int set[64] = {0};
      const size_t smem = (size_t)q.nbuf * q.buf_bytes + 64 + 128;
      auto k = fast_tma_tile_kernel<R, RL, T>;
      if (a.G * T > TILE_THREADS || a.mid || !a.plain_io || q.nbuf < 2) {
        launch_failure(k, "tensor-copy tile shape", L, T, a.G, smem, cudaErrorInvalidValue);
        return cudaErrorInvalidValue;
      }
      int dev = 0, per_sm = 0, nsm = 0;
      cudaError_t e = cudaGetDevice(&dev);
      if (e == cudaSuccess) e = configure(k, smem, set);
      if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, a.G * T, smem);
      if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      if (e == cudaSuccess && per_sm < 1) e = cudaErrorInvalidConfiguration;
      if (e != cudaSuccess) {
        launch_failure(k, "tensor-copy tile set-up", L, T, a.G, smem, e);
        return e;
      }
      if (q.ntiles <= 0) return cudaSuccess;
      const int64_t cap = (int64_t)per_sm * nsm;
      const int64_t nblk = q.ntiles < cap ? q.ntiles : cap;
      k<<<dim3((unsigned)nblk), dim3(a.G, T), smem, s>>>(a, *(const CUtensorMap*)tmap, q);
      e = cudaGetLastError();
      if (e != cudaSuccess) launch_failure(k, "tensor-copy tile launch", L, T, a.G, smem, e);
      return e;
    }
  }
  static constexpr bool has_stream = StreamShape<R, RL>::ok;
  static constexpr bool has_tc = std::is_same<R, float>::value && TcShape<RL, T>::direct_ok;
  static constexpr bool has_tile_tc = std::is_same<R, float>::value && TcShape<RL, T>::tile_ok;
  static cudaError_t launch_tc(int dir, const FastArgs& a, cudaStream_t s) {
    if constexpr (!has_tc) {
      snprintf(g_launch_msg, sizeof(g_launch_msg), "no tensor-core stage for L=%d", L);
      return cudaErrorNotSupported;
    } else {
      static int set_fwd[64] = {0}, set_bwd[64] = {0};
      constexpr size_t smem = TcShape<RL, T>::direct_smem();
      auto k = dir < 0 ? fast_tc_direct_kernel<-1, RL, T> : fast_tc_direct_kernel<1, RL, T>;
      cudaError_t e = configure(k, smem, dir < 0 ? set_fwd : set_bwd);
      if (e == cudaSuccess) e = tc_check_columns(k, T, smem, tc::tc_cols(T));
      if (e != cudaSuccess) {
        launch_failure(k, "tensor-core direct set-up", L, T, 1, smem, e);
        return e;
      }
      if (a.nlines <= 0) return cudaSuccess;
      k<<<dim3((unsigned)a.nlines), dim3(T), smem, s>>>(a);
      e = cudaGetLastError();
      if (e != cudaSuccess) launch_failure(k, "tensor-core direct launch", L, T, 1, smem, e);
      return e;
    }
  }
  static cudaError_t launch_tile_tc(const LineArgs& a, cudaStream_t s) {
    if constexpr (!has_tile_tc) {
      snprintf(g_launch_msg, sizeof(g_launch_msg), "no tensor-core tile stage for L=%d", L);
      return cudaErrorNotSupported;
    } else {
      static int set[64] = {0};
      const size_t smem = TcShape<RL, T>::tile_smem(a.G, stages_twiddles(a, L));
      auto k = fast_tc_tile_kernel<RL, T>;
      const int nt = a.G * T;
      if (nt % 128 != 0 || nt > 512 || a.mid || !a.plain_io) {
        launch_failure(k, "tensor-core tile shape", L, T, a.G, smem, cudaErrorInvalidValue);
        return cudaErrorInvalidValue;
      }
      cudaError_t e = configure(k, smem, set);
      if (e == cudaSuccess) e = tc_check_columns(k, nt, smem, tc::tc_cols(nt));
      if (e != cudaSuccess) {
        launch_failure(k, "tensor-core tile set-up", L, T, a.G, smem, e);
        return e;
      }
      const int64_t nblk = (a.nlines + a.G - 1) / a.G;
      if (nblk <= 0) return cudaSuccess;
      k<<<dim3((unsigned)nblk), dim3(a.G, T), smem, s>>>(a);
      e = cudaGetLastError();
      if (e != cudaSuccess) launch_failure(k, "tensor-core tile launch", L, T, a.G, smem, e);
      return e;
    }
  }
  static cudaError_t launch_tile(const LineArgs& a, cudaStream_t s) {
    static int set_plain[64] = {0}, set_mid[64] = {0}, set_full[64] = {0};
    const size_t smem = (size_t)a.G * tile_pitch(LPAD, a.G, (int)sizeof(cplx<R>)) * sizeof(cplx<R>) +
                        (size_t)a.G * 4 * sizeof(int64_t) +
                        (stages_twiddles(a, L) ? (size_t)L * sizeof(cplx<R>) : 0);
    const bool mid = a.mid != nullptr;
    auto k = mid ? fast_tile_kernel<R, RL, T, true, false>
                 : (a.plain_io ? fast_tile_kernel<R, RL, T, false, true>
                               : fast_tile_kernel<R, RL, T, false, false>);
    int* set = mid ? set_mid : (a.plain_io ? set_plain : set_full);
    const int max_threads = mid ? TileThreads<R, T, true>::value : TILE_THREADS;
    if (a.G * T > max_threads || (mid && (a.dir1 > 0 || a.dir2 < 0))) {
      launch_failure(k, "tile launch shape", L, T, a.G, smem, cudaErrorInvalidValue);
      return cudaErrorInvalidValue;
    }
    cudaError_t e = configure(k, smem, set);
    if (e != cudaSuccess) {
      launch_failure(k, "tile smem attribute", L, T, a.G, smem, e);
      return e;
    }
    const int64_t nblk = (a.nlines + a.G - 1) / a.G;
    if (nblk <= 0) return cudaSuccess;
    k<<<dim3((unsigned)nblk), dim3(a.G, T), smem, s>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) launch_failure(k, "tile launch", L, T, a.G, smem, e);
    return e;
  }
};

}  // namespace fb
