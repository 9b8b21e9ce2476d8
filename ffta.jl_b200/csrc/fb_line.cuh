// fb_kernels.cu -- the line kernel and the FP64 table generators.
//
// A "line" is one 1-D transform of length L held in shared memory.  A block
// holds G lines; each line is processed by T threads.  The kernel
//   1. loads its lines (gathering strided elements, zero-filling absent ones,
//      multiplying by an optional per-element table -- the Bluestein chirp),
//   2. runs a Stockham stage program in shared memory (radix 2/3/4/5/8/16
//      and odd-prime butterflies up to 71), in place: every stage reads its
//      butterflies into registers, synchronises, then writes,
//   3. optionally multiplies by a pointwise table and runs a second program in
//      the opposite direction (the Bluestein convolution in one kernel),
//   4. stores, fusing the four-step twiddle, an optional per-element table
//      and a scale factor.
// The same kernel serves batched 1-D columns, strided N-D axes, both passes
// of the four-step and all three passes of the multi-pass Bluestein.
//
// The reference computes all of this on the CPU with recursive radix-4 /
// radix-3 / DFT / Bluestein functions (FFTA src/algos.jl:51-424) and a
// Singleton twiddle recurrence (src/singleton_twiddle.jl:25-39); here every
// twiddle comes from a table computed in FP64 and rounded once.
#pragma once
#include <cuda_runtime.h>

#include "fb_device.cuh"
#include "fb_internal.h"

namespace fb {

__host__ __device__ __forceinline__ int padi(int e) { return e + (e >> 4); }

// compile-time offsets (must match prime_table_offset)
template <int P> struct POff;
#define FB_POFF(p, o) \
  template <> struct POff<p> { static constexpr int v = o; };
FB_POFF(7, 0)
FB_POFF(11, 7)
FB_POFF(13, 18)
FB_POFF(17, 31)
FB_POFF(19, 48)
FB_POFF(23, 67)
FB_POFF(29, 90)
FB_POFF(31, 119)
FB_POFF(37, 150)
FB_POFF(41, 187)
FB_POFF(43, 228)
FB_POFF(47, 271)
FB_POFF(53, 318)
FB_POFF(59, 371)
FB_POFF(61, 430)
FB_POFF(67, 491)
FB_POFF(71, 558)
#undef FB_POFF

// ---------------------------------------------------------------- stages
template <typename R, int RAD, int DIR>
__device__ __forceinline__ void butterfly(cplx<R>* v, const R* pcs) {
  if constexpr (RAD == 2) {
    bf2<R, DIR>(v[0], v[1]);
  } else if constexpr (RAD == 3) {
    dft3<R, DIR>(v);
  } else if constexpr (RAD == 4) {
    dft4<R, DIR>(v);
  } else if constexpr (RAD == 5) {
    dft5<R, DIR>(v);
  } else if constexpr (RAD == 8) {
    dft8<R, DIR>(v);
  } else if constexpr (RAD == 9) {
    dft9<R, DIR>(v);
  } else if constexpr (RAD == 16) {
    dft16<R, DIR>(v);
  } else {
    dftp<R, DIR, RAD>(v, pcs + 2 * POff<RAD>::v);
  }
}

// One Stockham stage of radix RAD on a line of length L held in `buf`
// (padded layout).  Ns is the product of the radices already applied.
// Butterfly j (k = j mod Ns) reads x[j + r*L/RAD], twiddles input r by
// w_{Ns*RAD}^(r k), and writes y[(j-k)*RAD + k + r*Ns].
template <typename R, int RAD, int DIR, int CAP>
__device__ __noinline__ void stage(cplx<R>* buf, int L, int Ns, const cplx<R>* __restrict__ tw,
                                      const R* pcs, int u, int T) {
  constexpr int UM = (RAD >= CAP) ? 1 : CAP / RAD;
  const int nb = L / RAD;
  cplx<R> v[UM][RAD];
#pragma unroll
  for (int q = 0; q < UM; ++q) {
    const int j = u + q * T;
    if (j < nb) {
#pragma unroll
      for (int r = 0; r < RAD; ++r) v[q][r] = buf[padi(j + r * nb)];
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < UM; ++q) {
    const int j = u + q * T;
    if (j < nb) {
      const int k = j % Ns;
      if (Ns > 1) {
        const cplx<R>* w = tw + k;  // entry (r-1)*Ns + k
#pragma unroll
        for (int r = 1; r < RAD; ++r) v[q][r] = ctw<R, DIR>(v[q][r], __ldg(w + (r - 1) * Ns));
      }
      butterfly<R, RAD, DIR>(v[q], pcs);
      const int base = (j - k) * RAD + k;
#pragma unroll
      for (int r = 0; r < RAD; ++r) buf[padi(base + r * Ns)] = v[q][r];
    }
  }
  __syncthreads();
}

template <typename R, int DIR, int CAP, bool BIG>
__device__ __forceinline__ void run_prog(cplx<R>* buf, const StageProg& p, const R* pcs, int u,
                                         int T, int* err) {
  const cplx<R>* twb = (const cplx<R>*)p.tw;
  int Ns = 1;
  const int L = p.L;
  for (int s = 0; s < p.nst; ++s) {
    const int rad = p.radix[s];
    const cplx<R>* tw = twb + p.tw_off[s];
    switch (rad) {
      case 2: stage<R, 2, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
      case 3: stage<R, 3, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
      case 4: stage<R, 4, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
      case 5: stage<R, 5, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
      case 7: stage<R, 7, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
      case 8: stage<R, 8, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
      case 9: stage<R, 9, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
      case 11: stage<R, 11, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
      case 13: stage<R, 13, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
      case 16: stage<R, 16, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
      default:
        if constexpr (BIG) {
          switch (rad) {
            case 17: stage<R, 17, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
            case 19: stage<R, 19, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
            case 23: stage<R, 23, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
            case 29: stage<R, 29, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
            case 31: stage<R, 31, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
            case 37: stage<R, 37, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
            case 41: stage<R, 41, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
            case 43: stage<R, 43, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
            case 47: stage<R, 47, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
            case 53: stage<R, 53, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
            case 59: stage<R, 59, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
            case 61: stage<R, 61, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
            case 67: stage<R, 67, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
            case 71: stage<R, 71, DIR, CAP>(buf, L, Ns, tw, pcs, u, T); break;
            default:
              if (threadIdx.x == 0 && threadIdx.y == 0 && err) atomicExch(err, rad);
          }
        } else {
          if (threadIdx.x == 0 && threadIdx.y == 0 && err) atomicExch(err, rad);
        }
    }
    Ns *= rad;
  }
}

// ------------------------------------------------------------ load / store
// Four-step twiddle of element i on a pass's loads (line twiddle index lt):
// a lean-I/O pass forms tw_elem's product over the first stage's radix, as the
// specialised tile kernel does; other passes read the table entry itself.
template <typename R>
__device__ __forceinline__ cplx<R> tw_on_load_elem(const LineArgs& a, int64_t lt, int i) {
  const cplx<R>* __restrict__ t = (const cplx<R>*)a.tw_tab + lt * a.tw_ls;
  auto at = [&](int k) { return __ldg(t + (int64_t)k * a.tw_es); };
  if (!a.plain_io) return at(i);
  const int rad = a.prog.radix[0];
  return tw_elem<R>(at, i, a.prog.L / rad, rad);
}

template <typename R>
__device__ __forceinline__ void load_lines(const LineArgs& a, cplx<R>* sm, const int64_t* lb,
                                           int64_t line0, int tid, int nthr, int u, int gl) {
  typedef cplx<R> C;
  const C* __restrict__ in = (const C*)a.in;
  const LineIO& io = a.ld;
  const C* __restrict__ mul = (const C*)io.mul;
  const int L = a.prog.L, G = a.G, cnt = io.count, Lp = a.Lpad;
  const C zero = Sc<R>::mk(R(0), R(0));
  if (io.mode == 1) {
    const int gs = __ffs(G) - 1;
    for (int f = tid; f < G * L; f += nthr) {
      const int g = f & (G - 1), i = f >> gs;
      C v = zero;
      if (line0 + g < a.nlines && i < cnt) {
        const int64_t vi = (int64_t)i * io.ves + lb[2 * G + g] * io.vls;
        if (vi < io.vn) {
          v = in[lb[g] + (int64_t)i * io.es];
          if (mul) v = cmul<R>(v, __ldg(mul + vi));
          if (a.tw_on_load) {
            const C w = tw_on_load_elem<R>(a, lb[3 * G + g], i);
            v = (a.tw_dir < 0) ? cmul<R>(v, w) : cmulc<R>(v, w);
          }
        }
      }
      sm[g * Lp + padi(i)] = v;
    }
  } else {
    const int g = gl, T = a.T;
    const bool ok = line0 + g < a.nlines;
    const int64_t base = lb[g], l0 = lb[2 * G + g];
    for (int i = u; i < L; i += T) {
      C v = zero;
      if (ok && i < cnt) {
        const int64_t vi = (int64_t)i * io.ves + l0 * io.vls;
        if (vi < io.vn) {
          v = in[base + (int64_t)i * io.es];
          if (mul) v = cmul<R>(v, __ldg(mul + vi));
          if (a.tw_on_load) {
            const C w = tw_on_load_elem<R>(a, lb[3 * G + g], i);
            v = (a.tw_dir < 0) ? cmul<R>(v, w) : cmulc<R>(v, w);
          }
        }
      }
      sm[g * Lp + padi(i)] = v;
    }
  }
}

template <typename R>
__device__ __forceinline__ cplx<R> finish(const LineArgs& a, cplx<R> v, int64_t tfac, int i,
                                          int64_t vi) {
  typedef cplx<R> C;
  if (a.st.mul) v = cmul<R>(v, __ldg((const C*)a.st.mul + vi));
  if (a.tw_tab && !a.tw_on_load) {
    const C w = __ldg((const C*)a.tw_tab + (int64_t)i * a.tw_es + tfac * a.tw_ls);
    v = (a.tw_dir < 0) ? cmul<R>(v, w) : cmulc<R>(v, w);
  } else if (a.tw_N) {
    const int64_t e = tfac * (int64_t)i;
    const C hi = __ldg((const C*)a.tw_hi + (e >> a.tw_shift));
    const C lo = __ldg((const C*)a.tw_lo + (e & ((int64_t(1) << a.tw_shift) - 1)));
    const C w = cmul<R>(hi, lo);
    v = (a.tw_dir < 0) ? cmul<R>(v, w) : cmulc<R>(v, w);
  }
  if (a.scale != 1.0) v = cscale<R>(v, (R)a.scale);
  return v;
}

template <typename R>
__device__ __forceinline__ void store_lines(const LineArgs& a, const cplx<R>* sm,
                                            const int64_t* lb, int64_t line0, int tid, int nthr,
                                            int u, int gl) {
  typedef cplx<R> C;
  C* __restrict__ out = (C*)a.out;
  const LineIO& io = a.st;
  const int G = a.G, cnt = io.count, Lp = a.Lpad;
  if (io.mode == 1) {
    const int gs = __ffs(G) - 1;
    for (int f = tid; f < G * cnt; f += nthr) {
      const int g = f & (G - 1), i = f >> gs;
      if (line0 + g >= a.nlines) continue;
      const int64_t l0 = lb[2 * G + g];
      const int64_t vi = (int64_t)i * io.ves + l0 * io.vls;
      if (vi >= io.vn) continue;
      out[lb[G + g] + (int64_t)i * io.es] = finish<R>(a, sm[g * Lp + padi(i)], lb[3 * G + g], i, vi);
    }
  } else {
    const int g = gl, T = a.T;
    if (line0 + g >= a.nlines) return;
    const int64_t base = lb[G + g], l0 = lb[2 * G + g], tfac = lb[3 * G + g];
    for (int i = u; i < cnt; i += T) {
      const int64_t vi = (int64_t)i * io.ves + l0 * io.vls;
      if (vi >= io.vn) continue;
      out[base + (int64_t)i * io.es] = finish<R>(a, sm[g * Lp + padi(i)], tfac, i, vi);
    }
  }
}

// ----------------------------------------------------------------- kernel
// One block's work: lines block*G .. block*G + G-1 of `a`.  Thread (u, g) is
// butterfly lane u of line g; tid = g*T + u.  Threads of a block beyond T*G
// pass u = kIdle (no butterflies, no elements) and tid = T*G, and only take
// part in the barriers.
constexpr int kIdle = 1 << 29;

template <typename R, int CAP, bool BIG>
__device__ __forceinline__ void line_body(const LineArgs& a, int64_t block, int u, int g, int tid,
                                          unsigned char* smraw) {
  typedef cplx<R> C;
  C* sm = (C*)smraw;
  const int T = a.T, G = a.G;
  const int nthr = G * T;
  const int64_t line0 = block * G;
  int64_t* lb = (int64_t*)(sm + (size_t)G * a.Lpad);
  if (tid < G) {
    const int64_t l = line0 + tid;
    const int64_t l0 = l % a.m0, t = l / a.m0;
    const int64_t l1 = t % a.m1, l2 = t / a.m1;
    lb[tid] = l0 * a.ld.s0 + l1 * a.ld.s1 + l2 * a.ld.s2;
    lb[G + tid] = l0 * a.st.s0 + l1 * a.st.s1 + l2 * a.st.s2;
    lb[2 * G + tid] = l0;
    lb[3 * G + tid] = a.tw_level ? l1 : l0;
  }
  __syncthreads();
  load_lines<R>(a, sm, lb, line0, tid, nthr, u, g);
  __syncthreads();
  C* buf = sm + g * a.Lpad;
  const R* pcs = (const R*)a.prime_cs;
  // One program, or (Bluestein) program -> pointwise multiply -> program in
  // the other direction.  The loop keeps one inlined copy per direction.
  const int npass = a.mid ? 2 : 1;
#pragma unroll 1
  for (int ps = 0; ps < npass; ++ps) {
    if ((ps == 0 ? a.dir1 : a.dir2) < 0)
      run_prog<R, -1, CAP, BIG>(buf, a.prog, pcs, u, T, a.err);
    else
      run_prog<R, 1, CAP, BIG>(buf, a.prog, pcs, u, T, a.err);
    if (ps == 0 && a.mid) {
      const C* __restrict__ mid = (const C*)a.mid;
      const int64_t l0 = lb[2 * G + g];
      for (int k = u; k < a.prog.L; k += T)
        buf[padi(k)] = cmul<R>(buf[padi(k)], __ldg(mid + l0 * a.mid_ls + (int64_t)k * a.mid_es));
      __syncthreads();
    }
  }
  store_lines<R>(a, sm, lb, line0, tid, nthr, u, g);
}

template <typename R, int CAP, bool BIG>
__global__ void __launch_bounds__(512) line_kernel(const LineArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int u = threadIdx.x, g = threadIdx.y;
  line_body<R, CAP, BIG>(a, blockIdx.x, u, g, g * a.T + u, smraw);
}

// Work-descriptor launch: many line transforms -- different lengths,
// directions, pointers -- in one grid.  Descriptor r owns blocks
// bstart[r] .. bstart[r+1]-1 and is run by the generic body with its own
// T x G shape inside the launch's one-dimensional block.
template <typename R, int CAP, bool BIG>
__global__ void __launch_bounds__(512)
    line_kernel_desc(const LineArgs* __restrict__ descs, const int64_t* __restrict__ bstart,
                     int ndesc) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ LineArgs sa;
  __shared__ int64_t sblock;
  if (threadIdx.x == 0) {
    int lo = 0, hi = ndesc - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(bstart + mid) <= (int64_t)blockIdx.x)
        lo = mid;
      else
        hi = mid - 1;
    }
    sa = descs[lo];
    sblock = (int64_t)blockIdx.x - __ldg(bstart + lo);
  }
  __syncthreads();
  const int nthr = sa.T * sa.G;
  const bool active = (int)threadIdx.x < nthr;
  const int u = active ? (int)threadIdx.x % sa.T : kIdle;
  const int g = active ? (int)threadIdx.x / sa.T : 0;
  line_body<R, CAP, BIG>(sa, sblock, u, g, active ? (int)threadIdx.x : nthr, smraw);
}

}  // namespace fb
