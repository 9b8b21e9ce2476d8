// fb_kernels.cu -- line-kernel dispatch and the FP64 table generators.
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
#include <cuda_runtime.h>

#include <cstring>

#include "fb_device.cuh"
#include "fb_internal.h"

namespace fb {

// ------------------------------------------------------------ prime tables
static const int kPrimes[] = {7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71};
static const int kNumPrimes = sizeof(kPrimes) / sizeof(kPrimes[0]);

int prime_table_offset(int p) {
  int off = 0;
  for (int i = 0; i < kNumPrimes; ++i) {
    if (kPrimes[i] == p) return off;
    off += kPrimes[i];
  }
  return -1;
}
int prime_table_total() {
  int off = 0;
  for (int i = 0; i < kNumPrimes; ++i) off += kPrimes[i];
  return off;
}

const FastFn* fast_table_f32_0(int*);
const FastFn* fast_table_f32_1(int*);
const FastFn* fast_table_f32_2(int*);
const FastFn* fast_table_f32_3(int*);
const FastFn* fast_table_f64_0(int*);
const FastFn* fast_table_f64_1(int*);
const FastFn* fast_table_f64_2(int*);
const FastFn* fast_table_f64_3(int*);

int fast_table_parts() { return 4; }
const FastFn* fast_table(int dtype, int part, int* count) {
  typedef const FastFn* (*Get)(int*);
  static const Get f32[4] = {fast_table_f32_0, fast_table_f32_1, fast_table_f32_2,
                             fast_table_f32_3};
  static const Get f64[4] = {fast_table_f64_0, fast_table_f64_1, fast_table_f64_2,
                             fast_table_f64_3};
  if (part < 0 || part >= 4) {
    *count = 0;
    return nullptr;
  }
  return (dtype == 0 ? f32 : f64)[part](count);
}

#define FB_DESC_DECL(tag)                                                                 \
  cudaError_t launch_desc_##tag(const LineArgs*, const int64_t*, int, int64_t, int, size_t, \
                                cudaStream_t);
FB_DESC_DECL(f32_c16)
FB_DESC_DECL(f32_c32)
FB_DESC_DECL(f32_big)
FB_DESC_DECL(f64_c16)
FB_DESC_DECL(f64_c32)
FB_DESC_DECL(f64_big)
#undef FB_DESC_DECL

cudaError_t launch_desc(int dtype, int variant, const LineArgs* descs, const int64_t* bstart,
                        int ndesc, int64_t nblocks, int threads, size_t smem, cudaStream_t s) {
  const bool cap32 = variant & 1, big = variant & 2;
  if (dtype == 0) {
    if (big) return launch_desc_f32_big(descs, bstart, ndesc, nblocks, threads, smem, s);
    return cap32 ? launch_desc_f32_c32(descs, bstart, ndesc, nblocks, threads, smem, s)
                 : launch_desc_f32_c16(descs, bstart, ndesc, nblocks, threads, smem, s);
  }
  if (big) return launch_desc_f64_big(descs, bstart, ndesc, nblocks, threads, smem, s);
  return cap32 ? launch_desc_f64_c32(descs, bstart, ndesc, nblocks, threads, smem, s)
               : launch_desc_f64_c16(descs, bstart, ndesc, nblocks, threads, smem, s);
}

cudaError_t launch_line_f32_c16(const LineArgs&, size_t, cudaStream_t);
cudaError_t launch_line_f32_c32(const LineArgs&, size_t, cudaStream_t);
cudaError_t launch_line_f32_big(const LineArgs&, size_t, cudaStream_t);
cudaError_t launch_line_f64_c16(const LineArgs&, size_t, cudaStream_t);
cudaError_t launch_line_f64_c32(const LineArgs&, size_t, cudaStream_t);
cudaError_t launch_line_f64_big(const LineArgs&, size_t, cudaStream_t);

thread_local char g_launch_msg[512] = {0};
const char* last_launch_message() { return g_launch_msg; }

size_t line_smem_bytes(int dtype, const LineArgs& a) {
  const size_t es = dtype == 0 ? 8 : 16;
  return (size_t)a.G * a.Lpad * es + (size_t)4 * a.G * sizeof(int64_t);
}
int line_max_threads() { return 512; }

cudaError_t launch_line(int dtype, int variant, const LineArgs& a, cudaStream_t s) {
  const size_t smem = line_smem_bytes(dtype, a);
  const bool cap32 = variant & 1, big = variant & 2;
  if (dtype == 0) {
    if (big) return launch_line_f32_big(a, smem, s);
    return cap32 ? launch_line_f32_c32(a, smem, s) : launch_line_f32_c16(a, smem, s);
  }
  if (big) return launch_line_f64_big(a, smem, s);
  return cap32 ? launch_line_f64_c32(a, smem, s) : launch_line_f64_c16(a, smem, s);
}

// ------------------------------------------------------------ FP64 tables
// exp(-2 pi i m / N) for integer m, computed in FP64: the index is reduced
// exactly to a quadrant and a fraction <= 1/2 of it, then CUDA's sincospi.
__device__ double2 root_fp64(int64_t m, int64_t N) {
  m %= N;
  if (m < 0) m += N;
  const int64_t m4 = 4 * m;
  const int q = (int)(m4 / N);
  const int64_t rem = m4 - (int64_t)q * N;  // theta = (pi/2)(q + rem/N)
  const bool flip = 2 * rem > N;
  const int64_t rr = flip ? N - rem : rem;
  const double x = (double)rr / (double)N;  // in [0, 1/2]
  double s, c;
  sincospi(0.5 * x, &s, &c);
  const double cq = flip ? s : c, sq = flip ? c : s;  // cos, sin of (pi/2) rem/N
  double ct, st;
  switch (q) {
    case 0: ct = cq; st = sq; break;
    case 1: ct = -sq; st = cq; break;
    case 2: ct = -cq; st = -sq; break;
    default: ct = sq; st = -cq; break;
  }
  return make_double2(ct, -st);
}

template <typename C> __device__ __forceinline__ C from_d2(double2 v);
template <> __device__ __forceinline__ float2 from_d2<float2>(double2 v) {
  return make_float2((float)v.x, (float)v.y);
}
template <> __device__ __forceinline__ double2 from_d2<double2>(double2 v) { return v; }

template <typename C>
__global__ void k_stage_tw(C* out, int R, int64_t Ns, int64_t count) {
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < count;
       idx += (int64_t)gridDim.x * blockDim.x) {
    // r-major: the R-1 twiddles of butterfly k sit Ns apart, so the threads
    // of a warp (consecutive k) read consecutive entries
    const int64_t r = idx / Ns + 1;
    const int64_t k = idx % Ns;
    out[idx] = from_d2<C>(root_fp64(r * k, Ns * R));
  }
}

// out[i*n_ln + l] = exp(-2 pi i (i*l mod N) / N) for i < n_el, l < n_ln.
template <typename C>
__global__ void k_tw_table(C* out, int64_t N, int64_t n_el, int64_t n_ln) {
  const int64_t count = n_el * n_ln;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < count;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = q / n_ln, l = q % n_ln;
    const unsigned __int128 e = (unsigned __int128)i * (unsigned __int128)l;
    out[q] = from_d2<C>(root_fp64((int64_t)(e % (unsigned __int128)N), N));
  }
}

template <typename C>
__global__ void k_roots(C* out, int64_t N, int64_t step, int64_t count) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < count;
       q += (int64_t)gridDim.x * blockDim.x) {
    const unsigned __int128 e = (unsigned __int128)q * (unsigned __int128)step;
    out[q] = from_d2<C>(root_fp64((int64_t)(e % (unsigned __int128)N), N));
  }
}

// b[n] = exp(i pi sgn p / N), p = n^2 mod 2N (exact), sgn = -dir.
// exp(-i pi p / N) = root(p, 2N); sgn > 0 takes the conjugate.
__device__ double2 chirp_b(int64_t n, int64_t N, int dir) {
  const unsigned __int128 p = ((unsigned __int128)n * (unsigned __int128)n) % (unsigned __int128)(2 * N);
  double2 r = root_fp64((int64_t)p, 2 * N);
  if (-dir > 0) r.y = -r.y;
  return r;
}

template <typename C>
__global__ void k_chirp(C* pre, C* post, double2* bext, int64_t N, int64_t M, int dir) {
  const double invM = 1.0 / (double)M;
  for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < M;
       m += (int64_t)gridDim.x * blockDim.x) {
    if (m < N) {
      const double2 b = chirp_b(m, N, dir);
      if (pre) pre[m] = from_d2<C>(make_double2(b.x, -b.y));
      if (post) post[m] = from_d2<C>(make_double2(b.x * invM, -b.y * invM));
    }
    if (bext) {
      double2 v = make_double2(0.0, 0.0);
      if (m < N)
        v = chirp_b(m, N, dir);
      else if (M - m < N)
        v = chirp_b(M - m, N, dir);
      bext[m] = v;
    }
  }
}

template <typename C>
__global__ void k_convert(C* dst, const double2* src, int64_t n, double scale) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double2 v = src[i];
    dst[i] = from_d2<C>(make_double2(v.x * scale, v.y * scale));
  }
}

__global__ void k_prime_tables(float* f32, double* f64, int total) {
  // walk the prime list: entry e belongs to prime p at offset off
  const int primes[] = {7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71};
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    int off = 0, p = 0;
    for (int i = 0; i < 17; ++i) {
      if (e < off + primes[i]) { p = primes[i]; break; }
      off += primes[i];
    }
    const int m = e - off;
    const double2 r = root_fp64(m, p);  // (cos, -sin)
    f64[2 * e] = r.x;
    f64[2 * e + 1] = -r.y;
    f32[2 * e] = (float)r.x;
    f32[2 * e + 1] = (float)(-r.y);
  }
}

static unsigned grid_for(int64_t n) {
  int64_t b = (n + 255) / 256;
  if (b < 1) b = 1;
  if (b > 65535) b = 65535;
  return (unsigned)b;
}

cudaError_t gen_stage_twiddles(int dtype, void* out, int R, int64_t Ns, cudaStream_t s) {
  const int64_t count = (int64_t)(R - 1) * Ns;
  if (count <= 0) return cudaSuccess;
  if (dtype == 0)
    k_stage_tw<float2><<<grid_for(count), 256, 0, s>>>((float2*)out, R, Ns, count);
  else
    k_stage_tw<double2><<<grid_for(count), 256, 0, s>>>((double2*)out, R, Ns, count);
  return cudaGetLastError();
}

cudaError_t gen_roots(int dtype, void* out, int64_t N, int64_t step, int64_t count,
                      cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  if (dtype == 0)
    k_roots<float2><<<grid_for(count), 256, 0, s>>>((float2*)out, N, step, count);
  else
    k_roots<double2><<<grid_for(count), 256, 0, s>>>((double2*)out, N, step, count);
  return cudaGetLastError();
}

cudaError_t gen_tw_table(int dtype, void* out, int64_t N, int64_t n_el, int64_t n_ln,
                         cudaStream_t s) {
  const int64_t count = n_el * n_ln;
  if (count <= 0) return cudaSuccess;
  if (dtype == 0)
    k_tw_table<float2><<<grid_for(count), 256, 0, s>>>((float2*)out, N, n_el, n_ln);
  else
    k_tw_table<double2><<<grid_for(count), 256, 0, s>>>((double2*)out, N, n_el, n_ln);
  return cudaGetLastError();
}

cudaError_t gen_chirp(int dtype, void* pre, void* post, void* bext_c64, int64_t N, int64_t M,
                      int dir, cudaStream_t s) {
  if (dtype == 0)
    k_chirp<float2><<<grid_for(M), 256, 0, s>>>((float2*)pre, (float2*)post, (double2*)bext_c64,
                                                N, M, dir);
  else
    k_chirp<double2><<<grid_for(M), 256, 0, s>>>((double2*)pre, (double2*)post,
                                                 (double2*)bext_c64, N, M, dir);
  return cudaGetLastError();
}

cudaError_t convert_c64(int dtype, void* dst, const void* src_c64, int64_t n, double scale,
                        cudaStream_t s) {
  if (dtype == 0)
    k_convert<float2><<<grid_for(n), 256, 0, s>>>((float2*)dst, (const double2*)src_c64, n, scale);
  else
    k_convert<double2><<<grid_for(n), 256, 0, s>>>((double2*)dst, (const double2*)src_c64, n,
                                                   scale);
  return cudaGetLastError();
}

// ------------------------------------------------------ real transforms
// Column-major arrays; `dims` (rank <= 8) are the full (complex) dims.
struct RealGeom {
  int rank, r0;
  int64_t dims[8];
  int64_t h;        // n/2 + 1 along r0
  uint32_t region;  // bit d: dim d is transformed
};

template <typename R>
__global__ void k_real_to_complex(const R* __restrict__ in, cplx<R>* __restrict__ out,
                                  int64_t count) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = Sc<R>::mk(in[i], R(0));
}

template <typename R>
__global__ void k_complex_to_real(const cplx<R>* __restrict__ in, R* __restrict__ out,
                                  int64_t count) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[i].x;
}

// out (dims with r0 cut to h) <- in (full dims): the first h entries along r0
template <typename R>
__global__ void k_extract_half(const cplx<R>* __restrict__ in, cplx<R>* __restrict__ out,
                               int64_t pre, int64_t n, int64_t h, int64_t post) {
  const int64_t count = pre * h * post;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < count;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = q % pre, t = q / pre, k = t % h, b = t / h;
    out[q] = in[a + pre * (k + n * b)];
  }
}

// z (full dims) <- Hermitian extension of x (r0 cut to h): entries with index
// k < h along r0 are copied; the others are conj(x at the mirrored index
// (-k mod n) in every transformed dim), the symmetry of a real signal's
// spectrum.
template <typename R>
__global__ void k_herm_extend(const cplx<R>* __restrict__ x, cplx<R>* __restrict__ z,
                              RealGeom g) {
  int64_t total = 1;
  for (int d = 0; d < g.rank; ++d) total *= g.dims[d];
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    int64_t idx[8];
    int64_t t = q;
    for (int d = 0; d < g.rank; ++d) {
      idx[d] = t % g.dims[d];
      t /= g.dims[d];
    }
    const bool mirror = idx[g.r0] >= g.h;
    if (mirror)
      for (int d = 0; d < g.rank; ++d)
        if ((g.region >> d) & 1) idx[d] = idx[d] ? g.dims[d] - idx[d] : 0;
    int64_t src = 0, stride = 1;
    for (int d = 0; d < g.rank; ++d) {
      src += idx[d] * stride;
      stride *= d == g.r0 ? g.h : g.dims[d];
    }
    const cplx<R> v = x[src];
    z[q] = mirror ? Sc<R>::mk(v.x, -v.y) : v;
  }
}

cudaError_t real_to_complex(int dtype, const void* in, void* out, int64_t count, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  if (dtype == 0)
    k_real_to_complex<float><<<grid_for(count), 256, 0, s>>>((const float*)in, (float2*)out, count);
  else
    k_real_to_complex<double><<<grid_for(count), 256, 0, s>>>((const double*)in, (double2*)out,
                                                               count);
  return cudaGetLastError();
}

cudaError_t complex_to_real(int dtype, const void* in, void* out, int64_t count, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  if (dtype == 0)
    k_complex_to_real<float><<<grid_for(count), 256, 0, s>>>((const float2*)in, (float*)out, count);
  else
    k_complex_to_real<double><<<grid_for(count), 256, 0, s>>>((const double2*)in, (double*)out,
                                                              count);
  return cudaGetLastError();
}

cudaError_t extract_half(int dtype, const void* in, void* out, int64_t pre, int64_t n, int64_t h,
                         int64_t post, cudaStream_t s) {
  const int64_t count = pre * h * post;
  if (count <= 0) return cudaSuccess;
  if (dtype == 0)
    k_extract_half<float><<<grid_for(count), 256, 0, s>>>((const float2*)in, (float2*)out, pre, n,
                                                          h, post);
  else
    k_extract_half<double><<<grid_for(count), 256, 0, s>>>((const double2*)in, (double2*)out, pre,
                                                           n, h, post);
  return cudaGetLastError();
}

cudaError_t herm_extend(int dtype, const void* x, void* z, int rank, const int64_t* dims, int r0,
                        int64_t h, uint32_t region, cudaStream_t s) {
  RealGeom g;
  memset(&g, 0, sizeof(g));
  g.rank = rank;
  g.r0 = r0;
  g.h = h;
  g.region = region;
  int64_t total = 1;
  for (int d = 0; d < rank; ++d) {
    g.dims[d] = dims[d];
    total *= dims[d];
  }
  if (total <= 0) return cudaSuccess;
  if (dtype == 0)
    k_herm_extend<float><<<grid_for(total), 256, 0, s>>>((const float2*)x, (float2*)z, g);
  else
    k_herm_extend<double><<<grid_for(total), 256, 0, s>>>((const double2*)x, (double2*)z, g);
  return cudaGetLastError();
}

// out[sum_d k_d * os[d]] = in[sum_d k_d * is[d]] for every index (k_d < dims[d]):
// a strided copy that moves an array between two layouts (rank <= 8).
template <typename E>
__global__ void k_permute(const E* __restrict__ in, E* __restrict__ out, PermCopy p) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < p.count;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t t = i, oi = 0, oo = 0;
    for (int d = 0; d < p.rank; ++d) {
      const int64_t k = t % p.dims[d];
      t /= p.dims[d];
      oi += k * p.is[d];
      oo += k * p.os[d];
    }
    out[oo] = in[oi];
  }
}

cudaError_t permute_copy(int elem_bytes, const void* in, void* out, const PermCopy& p,
                         cudaStream_t s) {
  if (p.count <= 0) return cudaSuccess;
  switch (elem_bytes) {
    case 4: k_permute<float><<<grid_for(p.count), 256, 0, s>>>((const float*)in, (float*)out, p); break;
    case 8: k_permute<float2><<<grid_for(p.count), 256, 0, s>>>((const float2*)in, (float2*)out, p); break;
    case 16: k_permute<double2><<<grid_for(p.count), 256, 0, s>>>((const double2*)in, (double2*)out, p); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t gen_prime_tables(void* f32tab, void* f64tab, cudaStream_t s) {
  const int total = prime_table_total();
  k_prime_tables<<<grid_for(total), 256, 0, s>>>((float*)f32tab, (double*)f64tab, total);
  return cudaGetLastError();
}

}  // namespace fb
