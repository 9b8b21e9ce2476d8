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
// The arithmetic -- twiddle table entries, twiddle multiply, butterflies,
// order of stages -- is exactly that of the generic line kernel
// (fb_line.cuh), so all of them produce the same bits for the same length.
#pragma once
#include <cstdio>
#include <cstring>
#include <type_traits>

#include "fb_line.cuh"

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

// ---------------------------------------------------------------- I/O
// A stage's input or output is shared memory (SmemIO) or a functor that
// loads element i of the line / stores element i of the line.
struct SmemIO {};

template <typename R> struct DirectIn {
  const cplx<R>* __restrict__ g;
  bool ok;
  __device__ __forceinline__ cplx<R> operator()(int i) const {
    return ok ? g[i] : Sc<R>::mk(R(0), R(0));
  }
};
template <typename R> struct DirectOut {
  cplx<R>* __restrict__ g;
  bool ok;
  R scale;
  __device__ __forceinline__ void operator()(int i, cplx<R> v) const {
    if (ok) g[i] = scale == R(1) ? v : cscale<R>(v, scale);
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
  __device__ __forceinline__ cplx<R> operator()(int i) const {
    const int64_t vi = (int64_t)i * ves + voff;
    if (!ok || vi >= vn) return Sc<R>::mk(R(0), R(0));
    cplx<R> v = base[(int64_t)i * es];
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
    base[(int64_t)i * es] = v;
  }
};

// Lean I/O for the common case (LineArgs::plain_io): every element present,
// no chirp tables, 32-bit strides, twiddle (if any) from a full table.  The
// line index is clamped to a valid line, so loads need no predicate.
template <typename R> struct PlainIn {
  const cplx<R>* __restrict__ base;
  int es;
  const cplx<R>* __restrict__ tab;  // twiddle on load (LineArgs::tw_on_load)
  int tab_es, tab_off, tw_dir;
  __device__ __forceinline__ cplx<R> operator()(int i) const {
    cplx<R> v = base[(int64_t)(i * es)];
    if (tab) {
      const cplx<R> w = __ldg(tab + (i * tab_es + tab_off));
      v = tw_dir < 0 ? cmul<R>(v, w) : cmulc<R>(v, w);
    }
    return v;
  }
};
template <typename R> struct PlainOut {
  cplx<R>* __restrict__ base;
  int es;
  const cplx<R>* __restrict__ tab;
  int tab_es, tab_off, tw_dir;
  R scale;
  bool ok;
  __device__ __forceinline__ void operator()(int i, cplx<R> v) const {
    if (tab) {
      const cplx<R> w = __ldg(tab + (i * tab_es + tab_off));
      v = tw_dir < 0 ? cmul<R>(v, w) : cmulc<R>(v, w);
    }
    if (scale != R(1)) v = cscale<R>(v, scale);
    if (ok) base[(int64_t)(i * es)] = v;
  }
};

// ------------------------------------------------------------- stages
// Stage S of program RL on one line held at `buf` (padded layout).  Thread u
// of T owns butterflies j = u + q*T.  The first stage takes its inputs from
// `in` unless it is SmemIO; the last stage gives its outputs to `out` unless
// it is SmemIO.
template <typename R, int DIR, class RL, int S, int T, class In, class Out>
__device__ __forceinline__ void fast_stage(cplx<R>* buf, const In& in, const Out& out,
                                           const cplx<R>* __restrict__ tw, const R* pcs, int u) {
  constexpr int L = prog_len<RL>();
  constexpr int RAD = RL::r[S];
  constexpr int Ns = ns_before<RL, S>();
  constexpr int nb = L / RAD;
  constexpr int UM = (nb + T - 1) / T;
  constexpr bool GIN = S == 0 && !std::is_same<In, SmemIO>::value;
  constexpr bool GOUT = S == RL::n - 1 && !std::is_same<Out, SmemIO>::value;
  cplx<R> v[UM][RAD];
#pragma unroll
  for (int q = 0; q < UM; ++q) {
    const int j = u + q * T;
    if (nb % T == 0 || j < nb) {
#pragma unroll
      for (int r = 0; r < RAD; ++r) {
        if constexpr (GIN)
          v[q][r] = in(j + r * nb);
        else
          v[q][r] = buf[padi(j + r * nb)];
      }
    }
  }
  // in place: all reads of the line finish before any write, unless one side
  // is global memory
  if constexpr (!GIN && !GOUT) __syncthreads();
#pragma unroll
  for (int q = 0; q < UM; ++q) {
    const int j = u + q * T;
    if (nb % T == 0 || j < nb) {
      const int k = (Ns == 1) ? 0 : j % Ns;
      if constexpr (Ns > 1) {
        const cplx<R>* w = tw + tw_offset<RL, S>() + k * (RAD - 1) - 1;
#pragma unroll
        for (int r = 1; r < RAD; ++r) v[q][r] = ctw<R, DIR>(v[q][r], __ldg(w + r));
      }
      butterfly<R, RAD, DIR>(v[q], pcs);
      const int base = (j - k) * RAD + k;
#pragma unroll
      for (int r = 0; r < RAD; ++r) {
        if constexpr (GOUT)
          out(base + r * Ns, v[q][r]);
        else
          buf[padi(base + r * Ns)] = v[q][r];
      }
    }
  }
  if constexpr (!GOUT) __syncthreads();
}

template <typename R, int DIR, class RL, int T, class In, class Out, int S = 0>
__device__ __forceinline__ void fast_prog(cplx<R>* buf, const In& in, const Out& out,
                                          const cplx<R>* tw, const R* pcs, int u) {
  fast_stage<R, DIR, RL, S, T, In, Out>(buf, in, out, tw, pcs, u);
  if constexpr (S + 1 < RL::n) fast_prog<R, DIR, RL, T, In, Out, S + 1>(buf, in, out, tw, pcs, u);
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
  const DirectOut<R> out{gout, ok, (R)a.scale};
  fast_prog<R, DIR, RL, T>(buf, in, out, (const C*)a.tw, (const R*)a.prime_cs, threadIdx.x);
}

// -------------------------------------------------------- tile kernel
// G lines per block addressed like the generic kernel (LineArgs: three batch
// levels, element strides, presence window, tables).  Thread (g, u) is
// threadIdx.x = g, threadIdx.y = u, so a warp spans 32/G butterflies of G
// lines.  MID: forward program, multiply by a.mid, inverse program.
template <typename R, class RL, int T, bool MID, bool PLAIN>
__global__ void __launch_bounds__(T > 512 ? T : 512) fast_tile_kernel(const LineArgs a) {
  typedef cplx<R> C;
  constexpr int L = prog_len<RL>();
  constexpr int LPAD = lpad_of(L);
  extern __shared__ __align__(16) unsigned char smraw[];
  const int g = threadIdx.x, u = threadIdx.y;
  C* buf = (C*)smraw + g * LPAD;
  // one thread per line splits its index into the batch levels (64-bit
  // divisions) and leaves the results in shared memory for the others
  int64_t* lb = (int64_t*)((C*)smraw + (size_t)a.G * LPAD);
  const int64_t line = (int64_t)blockIdx.x * a.G + g;
  const bool ok = line < a.nlines;
  if (u == 0) {
    const int64_t l = ok ? line : 0;
    const int64_t q0 = l % a.m0, t = l / a.m0;
    const int64_t q1 = t % a.m1, q2 = t / a.m1;
    lb[4 * g + 0] = q0;
    lb[4 * g + 1] = q0 * a.ld.s0 + q1 * a.ld.s1 + q2 * a.ld.s2;
    lb[4 * g + 2] = q0 * a.st.s0 + q1 * a.st.s1 + q2 * a.st.s2;
    lb[4 * g + 3] = a.tw_level ? q1 : q0;
  }
  __syncthreads();
  const int64_t l0 = lb[4 * g + 0], lt = lb[4 * g + 3];
  const C* tw = (const C*)a.prog.tw;
  const R* pcs = (const R*)a.prime_cs;
  const C* ib = (const C*)a.in + lb[4 * g + 1];
  C* ob = (C*)a.out + lb[4 * g + 2];
  if constexpr (PLAIN && !MID) {
    const C* tin = a.tw_on_load ? (const C*)a.tw_tab : nullptr;
    const C* tout = a.tw_on_load ? nullptr : (const C*)a.tw_tab;
    const PlainIn<R> in{ib, (int)a.ld.es, tin, (int)a.tw_es, (int)(lt * a.tw_ls), a.tw_dir};
    const PlainOut<R> out{ob, (int)a.st.es, tout, (int)a.tw_es, (int)(lt * a.tw_ls), a.tw_dir,
                          (R)a.scale, ok};
    if (a.dir1 < 0)
      fast_prog<R, -1, RL, T>(buf, in, out, tw, pcs, u);
    else
      fast_prog<R, 1, RL, T>(buf, in, out, tw, pcs, u);
  } else {
    const C* tin = a.tw_on_load ? (const C*)a.tw_tab : nullptr;
    const C* tout = a.tw_on_load ? nullptr : (const C*)a.tw_tab;
    const TileIn<R> in{ib, a.ld.es, (const C*)a.ld.mul, a.ld.vn, a.ld.ves, l0 * a.ld.vls, ok,
                       tin, a.tw_es, lt * a.tw_ls, a.tw_dir};
    const TileOut<R> out{ob, a.st.es, (const C*)a.st.mul, a.st.vn, a.st.ves, l0 * a.st.vls, lt,
                         a.tw_N ? (const C*)a.tw_hi : nullptr, (const C*)a.tw_lo, a.tw_shift,
                         a.tw_dir, (R)a.scale, ok, tout, a.tw_es, lt * a.tw_ls};
    if constexpr (MID) {
      fast_prog<R, -1, RL, T>(buf, in, SmemIO{}, tw, pcs, u);
      const C* __restrict__ mid = (const C*)a.mid;
      for (int k = u; k < L; k += T)
        buf[padi(k)] = cmul<R>(buf[padi(k)], __ldg(mid + l0 * a.mid_ls + (int64_t)k * a.mid_es));
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
  static cudaError_t launch_tile(const LineArgs& a, cudaStream_t s) {
    static int set_plain[64] = {0}, set_mid[64] = {0}, set_full[64] = {0};
    const size_t smem = (size_t)a.G * LPAD * sizeof(cplx<R>) + (size_t)a.G * 4 * sizeof(int64_t);
    const bool mid = a.mid != nullptr;
    auto k = mid ? fast_tile_kernel<R, RL, T, true, false>
                 : (a.plain_io ? fast_tile_kernel<R, RL, T, false, true>
                               : fast_tile_kernel<R, RL, T, false, false>);
    int* set = mid ? set_mid : (a.plain_io ? set_plain : set_full);
    if (a.G * T > (T > 512 ? T : 512) || (mid && (a.dir1 > 0 || a.dir2 < 0))) {
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
