// fb_fast.cuh -- compile-time-specialised line kernels for the common lengths.
//
// The stage program (radices) is a template parameter, so every index, stride
// and twiddle offset is a constant and each stage's registers die before the
// next stage starts.  For batched contiguous lines ("direct" I/O) the first
// stage reads its butterfly inputs straight from HBM into registers and the
// last stage writes its outputs straight from registers to HBM, both fully
// coalesced (consecutive threads own consecutive butterflies); only the
// exchanges between stages go through shared memory.  A length-4096 line
// with radices 16x16x16 thus makes one HBM read, two shared-memory round trips
// and one HBM write per element.
//
// The arithmetic -- twiddle table entries, twiddle multiply, butterflies,
// order of stages -- is exactly that of the generic line kernel
// (fb_line.cuh), so both produce the same bits for the same length.
#pragma once
#include "fb_line.cuh"

namespace fb {

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
template <class RL> __host__ __device__ constexpr int max_radix() {
  int m = 1;
  for (int i = 0; i < RL::n; ++i) m = RL::r[i] > m ? RL::r[i] : m;
  return m;
}

// Stage S of program RL on one line.  DIN: the first stage reads the line
// from global memory (`gin`, contiguous); DOUT: the last stage writes it to
// global memory (`gout`).  Otherwise the stage works in shared memory.  `ok`
// is false for the padding lines of the last block (no global access).
template <typename R, int DIR, class RL, int S, int T, bool DIN, bool DOUT>
__device__ __forceinline__ void fast_stage(cplx<R>* buf, const cplx<R>* __restrict__ gin,
                                           cplx<R>* __restrict__ gout,
                                           const cplx<R>* __restrict__ tw, const R* pcs, int u,
                                           bool ok, R scale) {
  constexpr int L = prog_len<RL>();
  constexpr int RAD = RL::r[S];
  constexpr int Ns = ns_before<RL, S>();
  constexpr int nb = L / RAD;
  constexpr int UM = (nb + T - 1) / T;
  constexpr bool GIN = DIN && S == 0, GOUT = DOUT && S == RL::n - 1;
  cplx<R> v[UM][RAD];
#pragma unroll
  for (int q = 0; q < UM; ++q) {
    const int j = u + q * T;
    if (nb % T == 0 || j < nb) {
#pragma unroll
      for (int r = 0; r < RAD; ++r) {
        if constexpr (GIN)
          v[q][r] = ok ? gin[j + r * nb] : Sc<R>::mk(R(0), R(0));
        else
          v[q][r] = buf[padi(j + r * nb)];
      }
    }
  }
  // in-place: all reads of the line finish before any write, unless one side
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
        if constexpr (GOUT) {
          if (ok) gout[base + r * Ns] = scale == R(1) ? v[q][r] : cscale<R>(v[q][r], scale);
        } else {
          buf[padi(base + r * Ns)] = v[q][r];
        }
      }
    }
  }
  if constexpr (!GOUT) __syncthreads();
}

template <typename R, int DIR, class RL, int T, bool DIN, bool DOUT, int S = 0>
__device__ __forceinline__ void fast_prog(cplx<R>* buf, const cplx<R>* gin, cplx<R>* gout,
                                          const cplx<R>* tw, const R* pcs, int u, bool ok,
                                          R scale) {
  fast_stage<R, DIR, RL, S, T, DIN, DOUT>(buf, gin, gout, tw, pcs, u, ok, scale);
  if constexpr (S + 1 < RL::n)
    fast_prog<R, DIR, RL, T, DIN, DOUT, S + 1>(buf, gin, gout, tw, pcs, u, ok, scale);
}

template <typename R, int DIR, class RL, int T>
__global__ void __launch_bounds__(512) fast_direct_kernel(const FastArgs a) {
  typedef cplx<R> C;
  constexpr int L = prog_len<RL>();
  constexpr int LP = (L - 1) + ((L - 1) >> 4) + 1;
  constexpr int LPAD = (LP & 1) ? LP : LP + 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw + threadIdx.y * LPAD;
  const int64_t line = (int64_t)blockIdx.x * a.G + threadIdx.y;
  const bool ok = line < a.nlines;
  const int64_t l = ok ? line : 0;
  const C* gin = (const C*)a.in + l * a.idist;
  C* gout = (C*)a.out + l * a.odist;
  fast_prog<R, DIR, RL, T, true, true>(buf, gin, gout, (const C*)a.tw, (const R*)a.prime_cs,
                                       threadIdx.x, ok, (R)a.scale);
}

// Staged variant: the generic kernel's loads and stores (strided tiles,
// chirp, four-step twiddle, scale; fb_line.cuh) around a compile-time stage
// program, run twice with a pointwise multiply between when `a.mid` is set
// (Bluestein).  `a.Lpad` equals LPAD below (the planner's lpad_for).
template <typename R, class RL, int T>
__global__ void __launch_bounds__(512) fast_staged_kernel(const LineArgs a) {
  typedef cplx<R> C;
  constexpr int L = prog_len<RL>();
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = (C*)smraw;
  const int G = a.G;
  const int u = threadIdx.x, g = threadIdx.y;
  const int tid = g * T + u, nthr = G * T;
  const int64_t line0 = (int64_t)blockIdx.x * G;
  int64_t* lb = (int64_t*)(sm + (size_t)G * a.Lpad);
  if (tid < G) {
    const int64_t l = line0 + tid;
    const int64_t l0 = l % a.m0, t = l / a.m0;
    const int64_t l1 = t % a.m1, l2 = t / a.m1;
    lb[tid] = l0 * a.ld.s0 + l1 * a.ld.s1 + l2 * a.ld.s2;
    lb[G + tid] = l0 * a.st.s0 + l1 * a.st.s1 + l2 * a.st.s2;
    lb[2 * G + tid] = l0;
  }
  __syncthreads();
  load_lines<R>(a, sm, lb, line0, tid, nthr);
  __syncthreads();
  C* buf = sm + g * a.Lpad;
  const C* tw = (const C*)a.prog.tw;
  const R* pcs = (const R*)a.prime_cs;
  const int npass = a.mid ? 2 : 1;
#pragma unroll 1
  for (int ps = 0; ps < npass; ++ps) {
    if ((ps == 0 ? a.dir1 : a.dir2) < 0)
      fast_prog<R, -1, RL, T, false, false>(buf, nullptr, nullptr, tw, pcs, u, true, R(1));
    else
      fast_prog<R, 1, RL, T, false, false>(buf, nullptr, nullptr, tw, pcs, u, true, R(1));
    if (ps == 0 && a.mid) {
      const C* __restrict__ mid = (const C*)a.mid;
      const int64_t l0 = lb[2 * G + g];
      for (int k = u; k < L; k += T)
        buf[padi(k)] = cmul<R>(buf[padi(k)], __ldg(mid + l0 * a.mid_ls + (int64_t)k * a.mid_es));
      __syncthreads();
    }
  }
  store_lines<R>(a, sm, lb, line0, tid, nthr);
}

template <typename R, class RL, int T> struct FastEntry {
  static constexpr int L = prog_len<RL>();
  static constexpr int LP = (L - 1) + ((L - 1) >> 4) + 1;
  static constexpr int LPAD = (LP & 1) ? LP : LP + 1;
  static cudaError_t launch(int dir, const FastArgs& a, cudaStream_t s) {
    const size_t smem = (size_t)a.G * LPAD * sizeof(cplx<R>);
    auto k = dir < 0 ? fast_direct_kernel<R, -1, RL, T> : fast_direct_kernel<R, 1, RL, T>;
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem);
      if (e != cudaSuccess) return e;
    }
    const int64_t nblk = (a.nlines + a.G - 1) / a.G;
    if (nblk <= 0) return cudaSuccess;
    k<<<dim3((unsigned)nblk), dim3(T, a.G), smem, s>>>(a);
    return cudaGetLastError();
  }
  static cudaError_t launch_staged(const LineArgs& a, cudaStream_t s) {
    const size_t smem = (size_t)a.G * LPAD * sizeof(cplx<R>) + (size_t)3 * a.G * sizeof(int64_t);
    if (a.Lpad != LPAD || a.T != T) return cudaErrorInvalidValue;
    auto k = fast_staged_kernel<R, RL, T>;
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem);
      if (e != cudaSuccess) return e;
    }
    const int64_t nblk = (a.nlines + a.G - 1) / a.G;
    if (nblk <= 0) return cudaSuccess;
    k<<<dim3((unsigned)nblk), dim3(T, a.G), smem, s>>>(a);
    return cudaGetLastError();
  }
};

}  // namespace fb
