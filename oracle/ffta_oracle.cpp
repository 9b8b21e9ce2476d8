// ffta_oracle.cpp -- CPU restatement of FFTA.jl's complex transform path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library in
// ffta.jl_b200/csrc: only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg may load it.  The product never links or calls it.
//
// It restates, in C++ templated on the working precision (float, double,
// __float128), the algorithm of FFTA.jl v0.3.1 (Project.toml:3):
//   * call graph ............ src/callgraph.jl:76-126 (CallGraphNode!), :133-138
//   * dispatcher ............ src/algos.jl:5-34 (fft!)
//   * Cooley-Tukey composite  src/algos.jl:51-118 (fft_composite!)
//   * O(N^2) DFT leaf ....... src/algos.jl:135-160 (fft_dft!, complex input)
//   * radix-4 pow2 .......... src/algos.jl:207-280 (fft_pow2_radix4!)
//   * radix-3 pow3 .......... src/algos.jl:299-341 (fft_pow3!)
//   * Bluestein ............. src/algos.jl:344-367 (prealloc_blue), :389-424
//   * Singleton twiddles .... src/singleton_twiddle.jl:25-39
//   * batched / N-D drivers . src/plan.jl:194-207 (_mul_loop!), :210-257 and
//                             :327-348 (mul! ND, fft_along_dim!)
//
// Julia's Complex arithmetic is mirrored: products are (ac-bd, ad+bc) with no
// fused multiply-add, except where FFTA writes @muladd (fft_pow3!), which maps
// to fma.  The file is compiled with -ffp-contract=off so that the compiler
// adds no contractions of its own.  Julia's sincospi/cispi are evaluated in
// __float128 after an exact argument reduction and rounded once to the working
// type, which matches a correctly rounded sincospi.
//
// Run in __float128 the same algorithm is the high-precision (113-bit) oracle.
#include <quadmath.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace {

typedef __float128 f128;

// ---------------------------------------------------------------- scalar ops
template <typename R> struct Ops;
template <> struct Ops<float> {
  static float fma(float a, float b, float c) { return fmaf(a, b, c); }
};
template <> struct Ops<double> {
  static double fma(double a, double b, double c) { return ::fma(a, b, c); }
};
template <> struct Ops<f128> {
  static f128 fma(f128 a, f128 b, f128 c) { return fmaq(a, b, c); }
};

template <typename R> struct Cx {
  R re, im;
};
template <typename R> inline Cx<R> operator+(Cx<R> a, Cx<R> b) { return {a.re + b.re, a.im + b.im}; }
template <typename R> inline Cx<R> operator-(Cx<R> a, Cx<R> b) { return {a.re - b.re, a.im - b.im}; }
template <typename R> inline Cx<R> operator-(Cx<R> a) { return {-a.re, -a.im}; }
// Julia: *(z::Complex, w::Complex) = Complex(zr*wr - zi*wi, zr*wi + zi*wr)
template <typename R> inline Cx<R> operator*(Cx<R> a, Cx<R> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename R> inline Cx<R> conj(Cx<R> a) { return {a.re, -a.im}; }
// Julia Base muladd(z::Complex, w::Complex, x::Complex): the form LLVM may
// fuse; restated with explicit fma.
template <typename R> inline Cx<R> muladd(Cx<R> z, Cx<R> w, Cx<R> x) {
  typedef Ops<R> O;
  return {O::fma(z.re, w.re, -O::fma(z.im, w.im, -x.re)),
          O::fma(z.re, w.im, O::fma(z.im, w.re, x.im))};
}
// Multiplication by the Complex{Int} constant `minusi = -dir*im`
// (src/algos.jl:224): (x + iy) * (0 + i s) = (x*0 - y*s) + i (x*s + y*0).
template <typename R> inline Cx<R> mul_i(Cx<R> a, int s) {
  const R z = R(0), sr = R(s);
  return {a.re * z - a.im * sr, a.re * sr + a.im * z};
}

// sincospi(x) evaluated in __float128 after exact reduction, rounded once.
// Multiples of 1/2 give exact 0/+-1 results as Julia's sincospi does.
inline void sincospi_q(f128 x, f128* s, f128* c) {
  f128 r = fmodq(x, (f128)2);  // exact
  if (r < 0) r += 2;           // [0, 2)
  f128 n = roundq(2 * r);      // quadrant index 0..4
  f128 f = r - n / 2;          // [-1/4, 1/4], exact
  f128 s0 = 0, c0 = 1;
  if (f != 0) {
    s0 = sinq(M_PIq * f);
    c0 = cosq(M_PIq * f);
  }
  int q = ((int)n) & 3;
  switch (q) {
    case 0: *s = s0; *c = c0; break;
    case 1: *s = c0; *c = -s0; break;
    case 2: *s = -s0; *c = -c0; break;
    default: *s = -c0; *c = s0; break;
  }
}
template <typename R> inline void sincospi_T(R x, R* s, R* c) {
  f128 sq, cq;
  sincospi_q((f128)x, &sq, &cq);
  *s = (R)sq;
  *c = (R)cq;
}
template <typename R> inline Cx<R> cispi_T(R x) {
  R s, c;
  sincospi_T(x, &s, &c);
  return {c, s};
}

// src/singleton_twiddle.jl:25-30
template <typename R> inline Cx<R> singleton_params(R hfreq) {
  R s_h, c_h;
  sincospi_T<R>(-hfreq, &s_h, &c_h);
  R alpha = R(2) * s_h * s_h;
  R beta = R(2) * s_h * c_h;
  return {alpha, beta};
}
// src/singleton_twiddle.jl:36-39 : w - z*w
template <typename R> inline Cx<R> singleton_step(Cx<R> w, Cx<R> z) { return w - z * w; }

// ------------------------------------------------------------- call graph
enum FFTEnum { COMPOSITE_FFT = 0, DFT = 1, POW3_FFT = 2, POW2RADIX4_FFT = 3, BLUESTEIN = 4 };

struct Node {
  int64_t left, right;
  int type;
  int64_t sz, s_in, s_out;
};

bool is_prime(int64_t n) {
  if (n < 2) return false;
  if (n % 2 == 0) return n == 2;
  for (int64_t d = 3; d * d <= n; d += 2)
    if (n % d == 0) return false;
  return true;
}
// Primes.factor restated: ascending (prime, exponent) pairs.
std::vector<std::pair<int64_t, int>> factor(int64_t n) {
  std::vector<std::pair<int64_t, int>> f;
  for (int64_t d = 2; d * d <= n; d += (d == 2 ? 1 : 2)) {
    int c = 0;
    while (n % d == 0) { n /= d; ++c; }
    if (c) f.push_back({d, c});
  }
  if (n > 1) f.push_back({n, 1});
  return f;
}
int64_t isqrt64(int64_t n) {
  int64_t r = (int64_t)std::sqrt((double)n);
  while (r * r > n) --r;
  while ((r + 1) * (r + 1) <= n) ++r;
  return r;
}
bool is_pow3(int64_t n) {  // N % 3 == 0 && nextpow(3, N) == N
  if (n % 3 != 0) return false;
  while (n % 3 == 0) n /= 3;
  return n == 1;
}

struct DimMismatch : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// src/callgraph.jl:76-126
int64_t callgraph_node(std::vector<Node>& nodes, std::vector<int64_t>& ws_len, int64_t N,
                       int64_t cutoff, int64_t s_in, int64_t s_out) {
  if (N <= 0) throw DimMismatch("Array length must be strictly positive");
  if ((N % 2 == 0) && ((N & (N - 1)) == 0)) {
    ws_len.push_back(0);
    nodes.push_back({0, 0, POW2RADIX4_FFT, N, s_in, s_out});
    return 1;
  } else if (is_pow3(N)) {
    ws_len.push_back(0);
    nodes.push_back({0, 0, POW3_FFT, N, s_in, s_out});
    return 1;
  } else if (N == 1 || is_prime(N)) {
    ws_len.push_back(0);
    nodes.push_back({0, 0, N < cutoff ? DFT : BLUESTEIN, N, s_in, s_out});
    return 1;
  }
  auto fzn = factor(N);
  int64_t Nf1 = fzn[0].first;
  int Nf1_cnt = fzn[0].second;
  int64_t N1;
  if (Nf1 == 2 || Nf1 == 3) {
    N1 = 1;
    for (int i = 0; i < Nf1_cnt; ++i) N1 *= Nf1;
  } else {
    std::vector<int64_t> cp;
    int64_t acc = 1;
    for (auto& pe : fzn)
      for (int i = 0; i < pe.second; ++i) { acc *= pe.first; cp.push_back(acc); }
    double N_fsqrt = std::sqrt((double)N);
    int64_t N_isqrt = isqrt64(N);
    // searchsortedlast: last index with cp[idx] <= N_isqrt
    size_t idx = 0;
    for (size_t i = 0; i < cp.size(); ++i)
      if (cp[i] <= N_isqrt) idx = i;
    N1 = cp[idx];
    if (idx != cp.size() - 1 && ((double)cp[idx + 1] - N_fsqrt < (N_fsqrt - (double)N1)))
      N1 = cp[idx + 1];
  }
  int64_t N2 = N / N1;
  nodes.push_back({0, 0, DFT, N, s_in, s_out});
  size_t sz = nodes.size();  // 1-based index of this node
  ws_len.push_back(N);
  int64_t left_len = callgraph_node(nodes, ws_len, N1, cutoff, N2, N2 * s_out);
  int64_t right_len = callgraph_node(nodes, ws_len, N2, cutoff, N1 * s_in, 1);
  nodes[sz - 1] = {1, 1 + left_len, COMPOSITE_FFT, N, s_in, s_out};
  return 1 + left_len + right_len;
}

template <typename R> struct CallGraph {
  std::vector<Node> nodes;
  std::vector<std::vector<Cx<R>>> workspace;
  int64_t cutoff;
  CallGraph(int64_t N, int64_t cut) : cutoff(cut) {
    std::vector<int64_t> ws;
    callgraph_node(nodes, ws, N, cut, 1, 1);
    for (auto l : ws) workspace.emplace_back((size_t)l);
  }
};

// -------------------------------------------------------------- kernels
// All indices below are 0-based; FFTA's are 1-based.  `dir` is -1 (forward)
// or +1 (backward), src/callgraph.jl:1.

// src/algos.jl:135-160
template <typename R>
void fft_dft(Cx<R>* out, const Cx<R>* in, int64_t N, int64_t so0, int64_t sout, int64_t si0,
             int64_t sin_, int dir) {
  Cx<R> tmp = in[si0];
  for (int64_t j = 1; j < N; ++j) tmp = tmp + in[si0 + j * sin_];
  out[so0] = tmp;
  for (int64_t j = 1; j < N; ++j) {
    tmp = in[si0];
    Cx<R> zj = singleton_params<R>(R(dir) * R(j) / R(N));
    Cx<R> wk = {R(1), R(0)};
    for (int64_t k = 1; k < N; ++k) {
      wk = singleton_step(wk, zj);
      tmp = tmp + wk * in[si0 + k * sin_];
    }
    out[so0 + j * sout] = tmp;
  }
}

// src/algos.jl:207-280
template <typename R>
void fft_pow2_radix4(Cx<R>* out, const Cx<R>* in, int64_t N, int64_t so0, int64_t sout,
                     int64_t si0, int64_t sin_, int dir) {
  if (N == 2) {
    Cx<R> a = in[si0], b = in[si0 + sin_];
    out[so0] = a + b;
    out[so0 + sout] = a - b;
    return;
  }
  const int minusi = -dir;  // minusi = -dir * im
  if (N == 4) {
    Cx<R> xee = in[si0], xoe = in[si0 + sin_], xeo = in[si0 + 2 * sin_], xoo = in[si0 + 3 * sin_];
    Cx<R> xee_p_xeo = xee + xeo, xee_m_xeo = xee - xeo;
    Cx<R> xoe_p_xoo = xoe + xoo;
    Cx<R> xoe_m_xoo = mul_i(-(xoe - xoo), minusi);
    out[so0] = xee_p_xeo + xoe_p_xoo;
    out[so0 + sout] = xee_m_xeo + xoe_m_xoo;
    out[so0 + 2 * sout] = xee_p_xeo - xoe_p_xoo;
    out[so0 + 3 * sout] = xee_m_xeo - xoe_m_xoo;
    return;
  }
  int64_t m = N / 4;
  fft_pow2_radix4(out, in, m, so0, sout, si0, sin_ * 4, dir);
  fft_pow2_radix4(out, in, m, so0 + m * sout, sout, si0 + sin_, sin_ * 4, dir);
  fft_pow2_radix4(out, in, m, so0 + 2 * m * sout, sout, si0 + 2 * sin_, sin_ * 4, dir);
  fft_pow2_radix4(out, in, m, so0 + 3 * m * sout, sout, si0 + 3 * sin_, sin_ * 4, dir);
  Cx<R> z1 = singleton_params<R>(R(dir) * R(1) / R(N));
  Cx<R> z2 = singleton_params<R>(R(dir) * R(2) / R(N));
  Cx<R> z3 = singleton_params<R>(R(dir) * R(3) / R(N));
  Cx<R> wkoe = {1, 0}, wkeo = {1, 0}, wkoo = {1, 0};
  for (int64_t k = 0; k < m; ++k) {
    int64_t kee = so0 + k * sout, koe = so0 + (k + m) * sout;
    int64_t keo = so0 + (k + 2 * m) * sout, koo = so0 + (k + 3 * m) * sout;
    Cx<R> y_kee = out[kee], y_koe = out[koe], y_keo = out[keo], y_koo = out[koo];
    Cx<R> t_koe = y_koe * wkoe, t_keo = y_keo * wkeo, t_koo = y_koo * wkoo;
    Cx<R> a = y_kee + t_keo, b = y_kee - t_keo;
    Cx<R> c = t_koe + t_koo;
    Cx<R> d = mul_i(-(t_koe - t_koo), minusi);
    out[kee] = a + c;
    out[koe] = b + d;
    out[keo] = a - c;
    out[koo] = b - d;
    wkoe = singleton_step(wkoe, z1);
    wkeo = singleton_step(wkeo, z2);
    wkoo = singleton_step(wkoo, z3);
  }
}

// src/algos.jl:299-341 (@muladd sums restated with fma)
template <typename R>
void fft_pow3(Cx<R>* out, const Cx<R>* in, int64_t N, int64_t so0, int64_t sout, int64_t si0,
              int64_t sin_, Cx<R> minus120, int dir) {
  Cx<R> plus120 = conj(minus120);
  if (N == 3) {
    Cx<R> a = in[si0], b = in[si0 + sin_], c = in[si0 + 2 * sin_];
    out[so0] = a + b + c;
    out[so0 + sout] = muladd(c, minus120, muladd(b, plus120, a));
    out[so0 + 2 * sout] = muladd(c, plus120, muladd(b, minus120, a));
    return;
  }
  int64_t Np = N / 3;
  fft_pow3(out, in, Np, so0, sout, si0, sin_ * 3, minus120, dir);
  fft_pow3(out, in, Np, so0 + Np * sout, sout, si0 + sin_, sin_ * 3, minus120, dir);
  fft_pow3(out, in, Np, so0 + 2 * Np * sout, sout, si0 + 2 * sin_, sin_ * 3, minus120, dir);
  Cx<R> z1 = singleton_params<R>(R(dir) * R(1) / R(N));
  Cx<R> z2 = singleton_params<R>(R(dir) * R(2) / R(N));
  Cx<R> wk1 = {1, 0}, wk2 = {1, 0};
  for (int64_t k = 0; k < Np; ++k) {
    int64_t k0 = so0 + sout * k, k1 = so0 + sout * (k + Np), k2 = so0 + sout * (k + 2 * Np);
    Cx<R> y0 = out[k0], y1 = out[k1], y2 = out[k2];
    out[k0] = muladd(y2, wk2, muladd(y1, wk1, y0));
    out[k1] = muladd(y2 * wk2, minus120, muladd(y1 * wk1, plus120, y0));
    out[k2] = muladd(y2 * wk2, plus120, muladd(y1 * wk1, minus120, y0));
    wk1 = singleton_step(wk1, z1);
    wk2 = singleton_step(wk2, z2);
  }
}

// src/algos.jl:344-367
template <typename R> struct BlueScratch {
  std::vector<Cx<R>> tmp, a, b;
  int64_t pad;
};
int64_t nextpow2(int64_t v) {
  int64_t p = 1;
  while (p < v) p <<= 1;
  return p;
}
template <typename R> BlueScratch<R> prealloc_blue(int64_t N, int dir) {
  BlueScratch<R> s;
  s.pad = nextpow2(2 * N - 1);
  s.tmp.assign(s.pad, {0, 0});
  s.a.assign(s.pad, {0, 0});
  s.b.assign(s.pad, {0, 0});
  int sgn = -dir;
  int64_t p = 0;  // n^2 reduced into (-N, N]
  for (int64_t i = 1; i <= N; ++i) {
    // cispi(sgn * p / N): Int/Int is a Float64 division, cispi in Float64,
    // then converted to the element type on assignment.
    double x = (double)(sgn * p) / (double)N;
    Cx<double> v = cispi_T<double>(x);
    s.b[i - 1] = {(R)v.re, (R)v.im};
    p += 2 * i - 1;
    if (p > N) p -= 2 * N;
  }
  for (int64_t j = 0; j < N; ++j) s.b[s.pad - 1 - j] = s.b[1 + j];
  return s;
}
// For __float128 the chirp is evaluated in full quad precision instead of
// through Float64, so that the high-precision oracle stays accurate.
template <> BlueScratch<f128> prealloc_blue<f128>(int64_t N, int dir) {
  BlueScratch<f128> s;
  s.pad = nextpow2(2 * N - 1);
  s.tmp.assign(s.pad, {0, 0});
  s.a.assign(s.pad, {0, 0});
  s.b.assign(s.pad, {0, 0});
  int sgn = -dir;
  int64_t p = 0;
  for (int64_t i = 1; i <= N; ++i) {
    s.b[i - 1] = cispi_T<f128>((f128)(sgn * p) / (f128)N);
    p += 2 * i - 1;
    if (p > N) p -= 2 * N;
  }
  for (int64_t j = 0; j < N; ++j) s.b[s.pad - 1 - j] = s.b[1 + j];
  return s;
}

// src/algos.jl:389-424
template <typename R>
void fft_bluestein(Cx<R>* out, const Cx<R>* in, int dir, int64_t N, int64_t so0, int64_t sout,
                   int64_t si0, int64_t sin_, BlueScratch<R>& s) {
  (void)dir;  // the direction is carried by the chirp, as in FFTA
  const int64_t pad = s.pad;
  for (int64_t i = N; i < pad; ++i) { s.a[i] = {0, 0}; s.tmp[i] = {0, 0}; }
  for (int64_t i = 0; i < N; ++i) s.a[i] = in[si0 + i * sin_] * conj(s.b[i]);
  fft_pow2_radix4<R>(s.tmp.data(), s.a.data(), pad, 0, 1, 0, 1, +1);  // FFT_BACKWARD
  fft_pow2_radix4<R>(s.a.data(), s.b.data(), pad, 0, 1, 0, 1, +1);    // FFT_BACKWARD
  for (int64_t i = 0; i < pad; ++i) s.tmp[i] = s.tmp[i] * s.a[i];
  fft_pow2_radix4<R>(s.a.data(), s.tmp.data(), pad, 0, 1, 0, 1, -1);  // FFT_FORWARD
  for (int64_t i = 0; i < N; ++i) {
    Cx<R> v = conj(s.b[i]) * s.a[i];
    s.tmp[i] = {v.re / R(pad), v.im / R(pad)};
  }
  for (int64_t i = 0; i < N; ++i) out[so0 + i * sout] = s.tmp[i];
}

template <typename R>
void fft_node(Cx<R>* out, const Cx<R>* in, int64_t so0, int64_t si0, int dir, CallGraph<R>& g,
              int64_t idx);

// src/algos.jl:51-118
template <typename R>
void fft_composite(Cx<R>* out, const Cx<R>* in, int64_t so0, int64_t si0, int dir,
                   CallGraph<R>& g, int64_t idx) {
  const Node root = g.nodes[idx];
  const int64_t left_idx = idx + root.left, right_idx = idx + root.right;
  const Node left = g.nodes[left_idx], right = g.nodes[right_idx];
  const int64_t N = root.sz, N1 = left.sz, N2 = right.sz;
  const int64_t s_in = root.s_in, s_out = root.s_out;
  Cx<R>* tmp = g.workspace[idx].data();
  BlueScratch<R> rblue, lblue;
  if (right.type == BLUESTEIN) rblue = prealloc_blue<R>(N2, dir);
  for (int64_t j1 = 0; j1 < N1; ++j1) {
    int64_t R_start_in = si0 + j1 * s_in;
    int64_t R_start_out = N2 * j1;
    if (right.type == BLUESTEIN)
      fft_bluestein<R>(tmp, in, dir, N2, R_start_out, right.s_out, R_start_in, right.s_in, rblue);
    else
      fft_node<R>(tmp, in, R_start_out, R_start_in, dir, g, right_idx);
    if (j1 > 0) {
      Cx<R> zj1 = singleton_params<R>(R(dir) * R(j1) / R(N));
      Cx<R> wk2 = {1, 0};
      for (int64_t k2 = 1; k2 < N2; ++k2) {
        wk2 = singleton_step(wk2, zj1);
        tmp[R_start_out + k2] = tmp[R_start_out + k2] * wk2;
      }
    }
  }
  if (left.type == BLUESTEIN) lblue = prealloc_blue<R>(N1, dir);
  for (int64_t k2 = 0; k2 < N2; ++k2) {
    int64_t L_start_out = so0 + k2 * s_out;
    int64_t L_start_in = k2;
    if (left.type == BLUESTEIN)
      fft_bluestein<R>(out, tmp, dir, N1, L_start_out, left.s_out, L_start_in, left.s_in, lblue);
    else
      fft_node<R>(out, tmp, L_start_out, L_start_in, dir, g, left_idx);
  }
}

// src/algos.jl:5-34
template <typename R>
void fft_node(Cx<R>* out, const Cx<R>* in, int64_t so0, int64_t si0, int dir, CallGraph<R>& g,
              int64_t idx) {
  const Node& root = g.nodes[idx];
  switch (root.type) {
    case COMPOSITE_FFT: fft_composite<R>(out, in, so0, si0, dir, g, idx); break;
    case DFT: fft_dft<R>(out, in, root.sz, so0, root.s_out, si0, root.s_in, dir); break;
    case POW2RADIX4_FFT:
      fft_pow2_radix4<R>(out, in, root.sz, so0, root.s_out, si0, root.s_in, dir);
      break;
    case POW3_FFT: {
      // _m_120 = cispi(T(2)/3); conj for the backward direction
      Cx<R> m120 = cispi_T<R>(R(2) / R(3));
      if (dir != -1) m120 = conj(m120);
      fft_pow3<R>(out, in, root.sz, so0, root.s_out, si0, root.s_in, m120, dir);
      break;
    }
    case BLUESTEIN: {
      BlueScratch<R> s = prealloc_blue<R>(root.sz, dir);
      fft_bluestein<R>(out, in, dir, root.sz, so0, root.s_out, si0, root.s_in, s);
      break;
    }
    default: throw std::invalid_argument("kernel not implemented");
  }
}

// One transform of a contiguous line: fft!(y, x, 1, 1, dir, t, g, 1).
template <typename R> void fft_line(Cx<R>* y, const Cx<R>* x, int dir, CallGraph<R>& g) {
  fft_node<R>(y, x, 0, 0, dir, g, 0);
}

// ------------------------------------------------------- N-D drivers
// Column-major array with `rank` dims.  Transform along each dim in `region`
// (0-based, ascending), in place on `data`.  This is fft_along_dim! in
// src/plan.jl:327-348: gather a line, transform into obuf, scatter back.
// Lines are split over `nthreads` threads when more than one is asked for.
template <typename R>
void along_dims(Cx<R>* data, int rank, const int64_t* dims, int nreg, const int* region, int dir,
                int64_t cutoff, int nthreads) {
  for (int r = 0; r < nreg; ++r) {
    const int d = region[r];
    const int64_t n = dims[d];
    int64_t pre = 1, post = 1;
    for (int i = 0; i < d; ++i) pre *= dims[i];
    for (int i = d + 1; i < rank; ++i) post *= dims[i];
    const int64_t nlines = pre * post;
    auto worker = [&](int64_t l0, int64_t l1) {
      CallGraph<R> g(n, cutoff);  // per-thread: the workspace is mutable
      std::vector<Cx<R>> ibuf(n), obuf(n);
      for (int64_t l = l0; l < l1; ++l) {
        const int64_t ipre = l % pre, ipost = l / pre;
        Cx<R>* base = data + ipre + ipost * pre * n;
        for (int64_t j = 0; j < n; ++j) ibuf[j] = base[j * pre];
        fft_line<R>(obuf.data(), ibuf.data(), dir, g);
        for (int64_t j = 0; j < n; ++j) base[j * pre] = obuf[j];
      }
    };
    int nt = nthreads < 1 ? 1 : nthreads;
    if (nt > nlines) nt = (int)nlines;
    if (nt <= 1) {
      worker(0, nlines);
    } else {
      std::vector<std::thread> th;
      for (int t = 0; t < nt; ++t) {
        int64_t a = nlines * t / nt, b = nlines * (t + 1) / nt;
        th.emplace_back(worker, a, b);
      }
      for (auto& t : th) t.join();
    }
  }
}

thread_local std::string g_err;

template <typename R>
int run_typed(const double* in, double* out, int rank, const int64_t* dims, int nreg,
              const int* region, int dir, int64_t cutoff, int nthreads) {
  int64_t total = 1;
  for (int i = 0; i < rank; ++i) total *= dims[i];
  if (total <= 0) throw DimMismatch("Array length must be strictly positive");
  std::vector<Cx<R>> buf((size_t)total);
  for (int64_t i = 0; i < total; ++i) buf[i] = {(R)in[2 * i], (R)in[2 * i + 1]};
  along_dims<R>(buf.data(), rank, dims, nreg, region, dir, cutoff, nthreads);
  for (int64_t i = 0; i < total; ++i) {
    out[2 * i] = (double)buf[i].re;
    out[2 * i + 1] = (double)buf[i].im;
  }
  return 0;
}

}  // namespace

extern "C" {

// Status: 0 ok, 1 DimensionMismatch, 2 ArgumentError.
const char* oracle_last_error(void) { return g_err.c_str(); }

// Transform a column-major complex array (interleaved re/im doubles) along
// the 0-based dims in `region` (ascending), like FFTA's mul! for an N-D plan
// (src/plan.jl:210-257) or a 1-D plan on an N-D array (:170-207).
// prec: 0 = float (ComplexF32), 1 = double (ComplexF64), 2 = __float128.
// Inputs and outputs are doubles in every precision; for prec 0 the input is
// rounded to float first and the result widened exactly.
int oracle_fft(int prec, const double* in, double* out, int rank, const int64_t* dims, int nreg,
               const int* region, int dir, int64_t cutoff, int nthreads) {
  try {
    if (dir != -1 && dir != 1) throw std::invalid_argument("direction must be -1 or +1");
    for (int r = 0; r < nreg; ++r)
      if (region[r] < 0 || region[r] >= rank)
        throw DimMismatch("Plan region is outside array dimensions.");
    switch (prec) {
      case 0: return run_typed<float>(in, out, rank, dims, nreg, region, dir, cutoff, nthreads);
      case 1: return run_typed<double>(in, out, rank, dims, nreg, region, dir, cutoff, nthreads);
      case 2: return run_typed<f128>(in, out, rank, dims, nreg, region, dir, cutoff, nthreads);
      default: throw std::invalid_argument("unknown precision");
    }
  } catch (DimMismatch& e) {
    g_err = e.what();
    return 1;
  } catch (std::exception& e) {
    g_err = e.what();
    return 2;
  }
}

// Float32 entry for the CPU baseline: interleaved floats in and out, batched
// contiguous 1D transforms, split over nthreads threads (FFTA itself runs the
// batch serially, src/plan.jl:204-206).
int oracle_fft_batched_f32(const float* in, float* out, int64_t n, int64_t batch, int dir,
                           int64_t cutoff, int nthreads) {
  try {
    typedef Cx<float> C;
    auto worker = [&](int64_t b0, int64_t b1) {
      CallGraph<float> g(n, cutoff);
      for (int64_t b = b0; b < b1; ++b)
        fft_line<float>((C*)out + b * n, (const C*)in + b * n, dir, g);
    };
    int nt = nthreads < 1 ? 1 : nthreads;
    if (nt > batch) nt = (int)batch;
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t) th.emplace_back(worker, batch * t / nt, batch * (t + 1) / nt);
    for (auto& t : th) t.join();
    return 0;
  } catch (DimMismatch& e) {
    g_err = e.what();
    return 1;
  } catch (std::exception& e) {
    g_err = e.what();
    return 2;
  }
}

// Same for ComplexF64 (interleaved doubles).
int oracle_fft_batched_f64(const double* in, double* out, int64_t n, int64_t batch, int dir,
                           int64_t cutoff, int nthreads) {
  try {
    typedef Cx<double> C;
    auto worker = [&](int64_t b0, int64_t b1) {
      CallGraph<double> g(n, cutoff);
      for (int64_t b = b0; b < b1; ++b)
        fft_line<double>((C*)out + b * n, (const C*)in + b * n, dir, g);
    };
    int nt = nthreads < 1 ? 1 : nthreads;
    if (nt > batch) nt = (int)batch;
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t) th.emplace_back(worker, batch * t / nt, batch * (t + 1) / nt);
    for (auto& t : th) t.join();
    return 0;
  } catch (DimMismatch& e) {
    g_err = e.what();
    return 1;
  } catch (std::exception& e) {
    g_err = e.what();
    return 2;
  }
}

// The call graph of src/callgraph.jl:133-138 as rows of 6 int64:
// (left, right, type, sz, s_in, s_out); type is the FFTEnum order of
// src/callgraph.jl:3.  Returns the node count, or -1 on error.
int64_t oracle_callgraph(int64_t n, int64_t cutoff, int64_t* rows, int64_t max_nodes) {
  try {
    std::vector<Node> nodes;
    std::vector<int64_t> ws;
    callgraph_node(nodes, ws, n, cutoff, 1, 1);
    int64_t cnt = (int64_t)nodes.size();
    for (int64_t i = 0; i < cnt && i < max_nodes; ++i) {
      rows[6 * i + 0] = nodes[i].left;
      rows[6 * i + 1] = nodes[i].right;
      rows[6 * i + 2] = nodes[i].type;
      rows[6 * i + 3] = nodes[i].sz;
      rows[6 * i + 4] = nodes[i].s_in;
      rows[6 * i + 5] = nodes[i].s_out;
    }
    return cnt;
  } catch (std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

}  // extern "C"
