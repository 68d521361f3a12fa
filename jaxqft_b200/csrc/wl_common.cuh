// Shared device definitions for the sm_100a SU(3) Wilson-fermion library.
//
// Internal HBM layout (all kernels of the solver path):
//   * even/odd "compact" site order: a site (x,y,z,t) of parity p=(x+y+z+t)&1
//     has compact index c = flat/2 with flat = ((x*Ly+y)*Lz+z)*Lt+t.  With Lt
//     even this equals the reference's ascending-flat-index ordering of the
//     parity-p sites (jaxqft/models/su3_wilson_nf2.py:831-840).
//   * spinors are structure-of-arrays per right-hand side:
//       FP64: double2 [rhs][12][Vh]    (component k = spin*3 + colour)
//       FP32: float4  [rhs][6][Vh]     (two complex components per float4)
//       FP16: uint4   [rhs][3][Vh]     (chunk = one colour, its four spins as half2) + float norm[rhs][Vh]
//     so one warp's load of one chunk is 512 contiguous bytes.
//   * links, split by the parity p of the site they start from:
//       FP64/18: double2 [p][mu][9][Vh]   FP64/12: double2 [p][mu][6][Vh]
//       FP32/12: float4  [p][mu][3][Vh]   FP16/12: uint2  [p][mu][3][Vh]
//     12-real links keep rows 0 and 1; row 2 = conj(row0 x row1) (exact for SU(3)).
//     Boundary phases are NOT folded into stored links; kernels apply them by
//     index (forward hop from x_mu = L_mu-1, backward hop into x_mu = 0).
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>
#include <type_traits>

#define WL_HD __host__ __device__ __forceinline__
#define WL_D __device__ __forceinline__

namespace wl {

// ---------------------------------------------------------------- complex
template <typename T> struct cplx { T re, im; };
template <typename T> WL_HD cplx<T> mk(T r, T i) { return cplx<T>{r, i}; }
template <typename T> WL_HD cplx<T> operator+(cplx<T> a, cplx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <typename T> WL_HD cplx<T> operator-(cplx<T> a, cplx<T> b) { return {a.re - b.re, a.im - b.im}; }
template <typename T> WL_HD cplx<T> operator*(cplx<T> a, cplx<T> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename T> WL_HD cplx<T> operator*(T s, cplx<T> a) { return {s * a.re, s * a.im}; }
template <typename T> WL_HD cplx<T> conj(cplx<T> a) { return {a.re, -a.im}; }
// i*a and -i*a
template <typename T> WL_HD cplx<T> mul_i(cplx<T> a) { return {-a.im, a.re}; }
template <typename T> WL_HD cplx<T> mul_mi(cplx<T> a) { return {a.im, -a.re}; }
// a += b*c ; a += conj(b)*c
template <typename T> WL_HD void fma_(cplx<T>& a, cplx<T> b, cplx<T> c) {
  a.re += b.re * c.re - b.im * c.im;
  a.im += b.re * c.im + b.im * c.re;
}
template <typename T> WL_HD void fmac_(cplx<T>& a, cplx<T> b, cplx<T> c) {
  a.re += b.re * c.re + b.im * c.im;
  a.im += b.re * c.im - b.im * c.re;
}
template <typename T> WL_HD T norm2(cplx<T> a) { return a.re * a.re + a.im * a.im; }

template <typename T> struct Spinor { cplx<T> v[4][3]; };
template <typename T> struct Half { cplx<T> v[2][3]; };
template <typename T> struct Link { cplx<T> m[3][3]; };

template <typename T> WL_D void zero(Spinor<T>& s) {
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) s.v[a][c] = {T(0), T(0)};
}

// ---------------------------------------------------------------- geometry
// Division by a run-time invariant d by multiply-high and shift (Granlund and
// Montgomery, "Division by invariant integers using multiplication", PLDI
// 1994): with l = ceil(log2 d) and the round-up multiplier
// m = ceil(2^(31+l) / d) < 2^32, floor(n/d) = floor(n m / 2^(31+l)) for every
// 0 <= n < 2^31, i.e. __umulhi(n, m) >> (l-1).  d == 1 is flagged by m == 0.
struct FastDiv {
  unsigned d, mul, shr;
};

inline FastDiv make_fastdiv(unsigned d) {
  FastDiv f{d, 0u, 0u};
  if (d <= 1) return f;
  unsigned l = 0;
  while ((1ull << l) < d) ++l;
  f.mul = (unsigned)(((1ull << (31 + l)) + d - 1) / d);
  f.shr = l - 1;
  return f;
}

WL_D unsigned fdiv(const FastDiv& f, unsigned n) { return f.mul ? (__umulhi(n, f.mul) >> f.shr) : n; }

struct Geom {
  int L[4];      // Lx, Ly, Lz, Lt
  int Lth;       // Lt / 2
  int Vh;        // V / 2
  int V;
  int strideRow[3];  // row stride of x, y, z in units of rows: Ly*Lz, Lz, 1
  double ph_re[4], ph_im[4];  // boundary phase per direction
  int ph_on[4];               // phase != 1
  FastDiv fd_lth, fd_l2, fd_l1;  // divisions by Lt/2, Lz, Ly in the compact-index decomposition
  int Ty;                         // y-slab width of the tiled sweep order (a divisor of Ly, <= 8)
  FastDiv fd_ty, fd_l0;           // divisions by Ty and Lx
};

struct Site {
  int c;       // compact index
  int row;     // (x*Ly+y)*Lz+z
  int x[4];    // coordinates
};

// Checking build (-DWL_BOUNDS_CHECK=1): every compact site index that the
// decode, the tiled sweep and the neighbour gathers produce is compared with
// Vh.  An index out of range is counted in g_wl_bounds_errors, the first one is
// kept in g_wl_bounds_first, and 0 is used instead so the access stays inside
// the field (no assert, no trap).  wl_bounds_errors() reads and clears the count.
#ifndef WL_BOUNDS_CHECK
#define WL_BOUNDS_CHECK 0
#endif
#if WL_BOUNDS_CHECK
__device__ unsigned int g_wl_bounds_errors;
__device__ long long g_wl_bounds_first;
WL_D int wl_checked_index(long long v, long long n) {
  if (v < 0 || v >= n) {
    if (atomicAdd(&g_wl_bounds_errors, 1u) == 0u) g_wl_bounds_first = v;
    return 0;
  }
  return (int)v;
}
#define WL_CHECKED(v, n) wl_checked_index((long long)(v), (long long)(n))
#else
#define WL_CHECKED(v, n) (v)
#endif

// Tiled sweep order for kernels whose blocks walk the compact sites in order: the
// logical index enumerates rows as (y-slab, x, y in slab, z) instead of (x, y, z),
// so the x-neighbour rows of a row are Ty*Lz rows away in the sweep (not Ly*Lz)
// and a source row's eight readers fall inside a window that stays in L2 even
// for 16 FP64 RHS per site; a source row at a slab face is read once more by the
// next slab.  Returns the compact index of logical position cl.
WL_D int tiled_compact(const Geom& g, int cl) {
  const int row_l = (int)fdiv(g.fd_lth, (unsigned)cl);
  const int th = cl - row_l * g.Lth;
  const int r1 = (int)fdiv(g.fd_l2, (unsigned)row_l);
  const int z = row_l - r1 * g.L[2];
  const int r2 = (int)fdiv(g.fd_ty, (unsigned)r1);
  const int yi = r1 - r2 * g.Ty;
  const int yb = (int)fdiv(g.fd_l0, (unsigned)r2);
  const int x = r2 - yb * g.L[0];
  const int row = (x * g.L[1] + yb * g.Ty + yi) * g.L[2] + z;
  return WL_CHECKED(row * g.Lth + th, g.Vh);
}

WL_D Site site_from_compact(const Geom& g, int parity, int c) {
  Site s;
  c = WL_CHECKED(c, g.Vh);
  s.c = c;
  const int row = (int)fdiv(g.fd_lth, (unsigned)c);
  const int th = c - row * g.Lth;
  s.row = row;
  const int r2 = (int)fdiv(g.fd_l2, (unsigned)row);
  s.x[2] = row - r2 * g.L[2];
  s.x[0] = (int)fdiv(g.fd_l1, (unsigned)r2);
  s.x[1] = r2 - s.x[0] * g.L[1];
  s.x[3] = 2 * th + ((parity + s.x[0] + s.x[1] + s.x[2]) & 1);
  return s;
}

// compact index (in the opposite-parity field) of the neighbour x + dir*e_mu
WL_D int neighbor(const Geom& g, const Site& s, int mu, int dir) {
  if (mu == 3) {
    int t = s.x[3] + dir;
    t = (t < 0) ? t + g.L[3] : (t >= g.L[3] ? t - g.L[3] : t);
    return WL_CHECKED(s.row * g.Lth + (t >> 1), g.Vh);
  }
  int xm = s.x[mu] + dir;
  int row = s.row + dir * g.strideRow[mu];
  if (xm < 0) row += g.L[mu] * g.strideRow[mu];
  else if (xm >= g.L[mu]) row -= g.L[mu] * g.strideRow[mu];
  return WL_CHECKED(row * g.Lth + (s.x[3] >> 1), g.Vh);
}

// ---------------------------------------------------------------- loads
WL_D double2 ldg(const double2* p) { return __ldg(p); }
WL_D float4 ldg(const float4* p) { return __ldg(p); }
WL_D uint4 ldg(const uint4* p) { return __ldg(p); }
WL_D uint2 ldg(const uint2* p) { return __ldg(p); }
WL_D float ldg(const float* p) { return __ldg(p); }

WL_D float2 h2f(unsigned int u) {
  __half2 h = *reinterpret_cast<__half2*>(&u);
  return __half22float2(h);
}
WL_D unsigned int f2h(float a, float b) {
  __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<unsigned int*>(&h);
}

// ---------------------------------------------------------------- precisions
enum Prec { P_DOUBLE = 0, P_SINGLE = 1, P_HALF = 2 };

// Spinor field in the internal SoA compact layout.
template <int P> struct SpinorField;

// Element (rhs, chunk k, site c) lives at ptr[rhs*rstride + k*kstride + c*cstride]
// (chunk = 16 bytes).  Two layouts use this accessor:
//   site-major   [rhs][k][Vh]: rstride = chunks*Vh*npar, kstride = Vh,   cstride = 1
//   RHS-innermost [k][Vh][nrhs]: rstride = 1, kstride = Vh*nrhs, cstride = nrhs
// The first coalesces when consecutive lanes are consecutive sites, the second
// when consecutive lanes are consecutive RHS of one site.  FP16 norms use
// norm[rhs*nrstride + c*ncstride] likewise.  Offsets are 32-bit unsigned (the
// allocator refuses fields of 2^32 chunks or more), which keeps the address
// arithmetic of the stencil loads to one multiply-add per access.
struct Strides {
  unsigned rstride, kstride, cstride;
  unsigned nrstride, ncstride;
  WL_D unsigned at(int rhs, int k, unsigned c) const { return rhs * rstride + k * kstride + c * cstride; }
  WL_D unsigned nat(int rhs, unsigned c) const { return rhs * nrstride + c * ncstride; }
};

template <> struct SpinorField<P_DOUBLE> : Strides {
  using real = double;
  double2* ptr;
  float* norm;  // unused
  WL_D void load(Spinor<double>& s, int rhs, long long c) const {
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      double2 v = ldg(ptr + at(rhs, k, c));
      s.v[k / 3][k % 3] = {v.x, v.y};
    }
  }
  WL_D void load_plain(Spinor<double>& s, int rhs, long long c) const {  // for read-after-write within a kernel
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      double2 v = ptr[at(rhs, k, c)];
      s.v[k / 3][k % 3] = {v.x, v.y};
    }
  }
  WL_D void store(const Spinor<double>& s, int rhs, long long c) const {
#pragma unroll
    for (int k = 0; k < 12; ++k) ptr[at(rhs, k, c)] = make_double2(s.v[k / 3][k % 3].re, s.v[k / 3][k % 3].im);
  }
};

template <> struct SpinorField<P_SINGLE> : Strides {
  using real = float;
  float4* ptr;
  float* norm;
  template <bool NC>
  WL_D void load_impl(Spinor<float>& s, int rhs, long long c) const {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      float4 v = NC ? ldg(ptr + at(rhs, k, c)) : ptr[at(rhs, k, c)];
      int i0 = 2 * k, i1 = 2 * k + 1;
      s.v[i0 / 3][i0 % 3] = {v.x, v.y};
      s.v[i1 / 3][i1 % 3] = {v.z, v.w};
    }
  }
  WL_D void load(Spinor<float>& s, int rhs, long long c) const { load_impl<true>(s, rhs, c); }
  WL_D void load_plain(Spinor<float>& s, int rhs, long long c) const { load_impl<false>(s, rhs, c); }
  WL_D void store(const Spinor<float>& s, int rhs, long long c) const {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      int i0 = 2 * k, i1 = 2 * k + 1;
      ptr[at(rhs, k, c)] = make_float4(s.v[i0 / 3][i0 % 3].re, s.v[i0 / 3][i0 % 3].im, s.v[i1 / 3][i1 % 3].re,
                                       s.v[i1 / 3][i1 % 3].im);
    }
  }
};

// FP16 record of one (site, rhs): three 16-byte chunks, chunk k = colour k with
// the four spins as half2 (re, im), plus one float norm (value = norm * half).
// The colour-major order lets the tensor-core hop give each lane of an MMA
// group one colour of all four spins with a single 16-byte load.
template <> struct SpinorField<P_HALF> : Strides {
  using real = float;
  uint4* ptr;
  float* norm;
  template <bool NC>
  WL_D void load_impl(Spinor<float>& s, int rhs, long long c) const {
    float nrm = NC ? ldg(norm + nat(rhs, c)) : norm[nat(rhs, c)];
#pragma unroll
    for (int k = 0; k < 3; ++k) {  // chunk k = colour k, spins 0..3
      uint4 v = NC ? ldg(ptr + at(rhs, k, c)) : ptr[at(rhs, k, c)];
      float2 a0 = h2f(v.x), a1 = h2f(v.y), a2 = h2f(v.z), a3 = h2f(v.w);
      s.v[0][k] = {a0.x * nrm, a0.y * nrm};
      s.v[1][k] = {a1.x * nrm, a1.y * nrm};
      s.v[2][k] = {a2.x * nrm, a2.y * nrm};
      s.v[3][k] = {a3.x * nrm, a3.y * nrm};
    }
  }
  WL_D void load(Spinor<float>& s, int rhs, long long c) const { load_impl<true>(s, rhs, c); }
  WL_D void load_plain(Spinor<float>& s, int rhs, long long c) const { load_impl<false>(s, rhs, c); }
  WL_D void store(const Spinor<float>& s, int rhs, long long c) const {
    float mx = 0.f;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) mx = fmaxf(mx, fmaxf(fabsf(s.v[a][cc].re), fabsf(s.v[a][cc].im)));
    // A site whose largest component is below FLT_MIN is stored as zero: 1/mx
    // would overflow to Inf there and turn exact zeros into NaN (0 * Inf).
    // Such sites occur far from a point source, where Krylov vectors decay
    // over tens of lattice spacings.
    const bool keep = mx >= 1.17549435e-38f;
    const float inv = keep ? 1.0f / mx : 0.f;
    norm[nat(rhs, c)] = keep ? mx : 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const cplx<float>& c0 = s.v[0][k];
      const cplx<float>& c1 = s.v[1][k];
      const cplx<float>& c2 = s.v[2][k];
      const cplx<float>& c3 = s.v[3][k];
      uint4 v;
      v.x = f2h(c0.re * inv, c0.im * inv);
      v.y = f2h(c1.re * inv, c1.im * inv);
      v.z = f2h(c2.re * inv, c2.im * inv);
      v.w = f2h(c3.re * inv, c3.im * inv);
      ptr[at(rhs, k, c)] = v;
    }
  }
};

// ---------------------------------------------------------------- packed FP32x2 I/O
// A spinor as 12 float2 (re, im), component k = spin*3 + colour, for the
// sm_100 packed FP32x2 pipe (__ffma2_rn / __fmul2_rn: two lanes per instruction).
WL_D float2 f2(float a, float b) { return make_float2(a, b); }
WL_D float2 swp(float2 v) { return make_float2(v.y, v.x); }
WL_D float2 ffma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
WL_D float2 fmul2(float2 a, float2 b) { return __fmul2_rn(a, b); }

// load: v = stored values, returns the scale (value = scale * v; FP16 per-site norm)
// store: v = values; FP16 stores pick the per-site norm max|v| and pack pairs
template <class SF> struct Packed;

template <> struct Packed<SpinorField<P_SINGLE>> {
  WL_D static float load(const SpinorField<P_SINGLE>& f, int rhs, unsigned c, float2 (&v)[12]) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const float4 q = ldg(f.ptr + f.at(rhs, k, c));
      v[2 * k] = f2(q.x, q.y);
      v[2 * k + 1] = f2(q.z, q.w);
    }
    return 1.0f;
  }
  WL_D static void store(const SpinorField<P_SINGLE>& f, int rhs, unsigned c, const float2 (&v)[12]) {
#pragma unroll
    for (int k = 0; k < 6; ++k) f.ptr[f.at(rhs, k, c)] = make_float4(v[2 * k].x, v[2 * k].y, v[2 * k + 1].x, v[2 * k + 1].y);
  }
};

template <> struct Packed<SpinorField<P_HALF>> {
  WL_D static float load(const SpinorField<P_HALF>& f, int rhs, unsigned c, float2 (&v)[12]) {
    const float n = ldg(f.norm + f.nat(rhs, c));
#pragma unroll
    for (int k = 0; k < 3; ++k) {  // chunk k = colour k, spins 0..3
      const uint4 q = ldg(f.ptr + f.at(rhs, k, c));
      v[k] = h2f(q.x);
      v[3 + k] = h2f(q.y);
      v[6 + k] = h2f(q.z);
      v[9 + k] = h2f(q.w);
    }
    return n;
  }
  WL_D static void store(const SpinorField<P_HALF>& f, int rhs, unsigned c, const float2 (&v)[12]) {
    float mx = 0.f;
#pragma unroll
    for (int k = 0; k < 12; ++k) mx = fmaxf(mx, fmaxf(fabsf(v[k].x), fabsf(v[k].y)));
    // below FLT_MIN the site is stored as zero (1/mx would overflow, 0 * Inf = NaN)
    const bool keep = mx >= 1.17549435e-38f;
    const float inv = keep ? 1.0f / mx : 0.f;
    f.norm[f.nat(rhs, c)] = keep ? mx : 0.f;
    const float2 s = f2(inv, inv);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float2 a0 = fmul2(s, v[k]), a1 = fmul2(s, v[3 + k]);
      const float2 a2 = fmul2(s, v[6 + k]), a3 = fmul2(s, v[9 + k]);
      uint4 q;
      q.x = f2h(a0.x, a0.y);
      q.y = f2h(a1.x, a1.y);
      q.z = f2h(a2.x, a2.y);
      q.w = f2h(a3.x, a3.y);
      f.ptr[f.at(rhs, k, c)] = q;
    }
  }
};

// |v|^2 of a packed spinor, accumulated in FP32 pairs
WL_D double pnorm2(const float2 (&v)[12]) {
  float2 s = f2(0.f, 0.f);
#pragma unroll
  for (int k = 0; k < 12; ++k) s = ffma2(v[k], v[k], s);
  return (double)s.x + (double)s.y;
}

WL_D double pnorm2_4(const float2 (&v)[4]) {
  float2 s = f2(0.f, 0.f);
#pragma unroll
  for (int k = 0; k < 4; ++k) s = ffma2(v[k], v[k], s);
  return (double)s.x + (double)s.y;
}

// One colour of an FP16 record (its four spins), for the tensor-core hop, whose
// lanes hold one colour each: lanes t = 0, 1, 2 of an aligned group of four
// share a record (colour t), lane t = 3 holds none (its values are zero).
struct SliceHalf {
  struct Raw {
    uint4 q;
    float n;
  };
  // the stored chunk and norm (zeros unless `mine`), issued early by the tensor-core hop
  WL_D static Raw load(const SpinorField<P_HALF>& f, int rhs, unsigned c, int t, bool mine) {
    Raw r{make_uint4(0u, 0u, 0u, 0u), 0.f};
    if (mine) {
      r.q = ldg(f.ptr + f.at(rhs, t, c));
      r.n = ldg(f.norm + f.nat(rhs, c));
    }
    return r;
  }
  // v = stored values of colour t; returns the record's norm
  WL_D static float unpack(const Raw& r, float2 (&v)[4]) {
    v[0] = h2f(r.q.x);
    v[1] = h2f(r.q.y);
    v[2] = h2f(r.q.z);
    v[3] = h2f(r.q.w);
    return r.n;
  }
  // Every lane of the warp calls this (the norm is the max over the group's four
  // lanes); `act` is uniform over a group, and only active groups write.
  WL_D static void store(const SpinorField<P_HALF>& f, int rhs, unsigned c, int t, bool act, const float2 (&v)[4]) {
    float mx = 0.f;
#pragma unroll
    for (int k = 0; k < 4; ++k) mx = fmaxf(mx, fmaxf(fabsf(v[k].x), fabsf(v[k].y)));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
    // below FLT_MIN the record is stored as zero (1/mx would overflow, 0 * Inf = NaN)
    const bool keep = mx >= 1.17549435e-38f;
    const float inv = keep ? 1.0f / mx : 0.f;
    if (act && t < 3) {
      const float2 s = f2(inv, inv);
      const float2 a0 = fmul2(s, v[0]), a1 = fmul2(s, v[1]), a2 = fmul2(s, v[2]), a3 = fmul2(s, v[3]);
      uint4 q;
      q.x = f2h(a0.x, a0.y);
      q.y = f2h(a1.x, a1.y);
      q.z = f2h(a2.x, a2.y);
      q.w = f2h(a3.x, a3.y);
      f.ptr[f.at(rhs, t, c)] = q;
    }
    if (act && t == 0) f.norm[f.nat(rhs, c)] = keep ? mx : 0.f;
  }
};

// Spinor field in the reference layout: complex128 [rhs][V][4][3], site = flat index.
struct SpinorRef {
  using real = double;
  double2* ptr;
  long long rstride;  // double2 per rhs (= 12*V)
  int Lt;
  WL_D static int flat(int parity_off_unused, int c) { return c; }
  WL_D void load(Spinor<double>& s, int rhs, long long flat) const {
    const double2* b = ptr + rhs * rstride + flat * 12;
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      double2 v = ldg(b + k);
      s.v[k / 3][k % 3] = {v.x, v.y};
    }
  }
  WL_D void store(const Spinor<double>& s, int rhs, long long flat) const {
    double2* b = ptr + rhs * rstride + flat * 12;
#pragma unroll
    for (int k = 0; k < 12; ++k) b[k] = make_double2(s.v[k / 3][k % 3].re, s.v[k / 3][k % 3].im);
  }
};

// flat index of compact site c of the given parity
WL_D long long flat_of(const Geom& g, int parity, int c) {
  Site s = site_from_compact(g, parity, c);
  return (long long)s.row * g.L[3] + s.x[3];
}

// ---------------------------------------------------------------- links
template <typename T> WL_D void reconstruct_row2(Link<T>& u) {
  // row2 = conj(row0 x row1)
  u.m[2][0] = conj(u.m[0][1] * u.m[1][2] - u.m[0][2] * u.m[1][1]);
  u.m[2][1] = conj(u.m[0][2] * u.m[1][0] - u.m[0][0] * u.m[1][2]);
  u.m[2][2] = conj(u.m[0][0] * u.m[1][1] - u.m[0][1] * u.m[1][0]);
}

enum LinkKind { L_D18 = 0, L_D12 = 1, L_S12 = 2, L_H12 = 3, L_REF = 4 };

template <int K> struct LinkField;

template <> struct LinkField<L_D18> {
  using real = double;
  const double2* ptr;  // [p][mu][9][Vh]
  int vh;
  WL_D void load(Link<double>& u, int p, int mu, int c) const {
    const double2* b = ptr + ((long long)(p * 4 + mu) * 9) * vh + c;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      double2 v = ldg(b + (long long)k * vh);
      u.m[k / 3][k % 3] = {v.x, v.y};
    }
  }
};

template <> struct LinkField<L_D12> {
  using real = double;
  const double2* ptr;  // [p][mu][6][Vh]
  int vh;
  WL_D void load(Link<double>& u, int p, int mu, int c) const {
    const double2* b = ptr + ((long long)(p * 4 + mu) * 6) * vh + c;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      double2 v = ldg(b + (long long)k * vh);
      u.m[k / 3][k % 3] = {v.x, v.y};
    }
    reconstruct_row2(u);
  }
};

template <> struct LinkField<L_S12> {
  using real = float;
  const float4* ptr;  // [p][mu][3][Vh]
  int vh;
  WL_D void load(Link<float>& u, int p, int mu, int c) const {
    const float4* b = ptr + ((long long)(p * 4 + mu) * 3) * vh + c;
    float4 a = ldg(b), bb = ldg(b + vh), cc = ldg(b + 2LL * vh);
    u.m[0][0] = {a.x, a.y};
    u.m[0][1] = {a.z, a.w};
    u.m[0][2] = {bb.x, bb.y};
    u.m[1][0] = {bb.z, bb.w};
    u.m[1][1] = {cc.x, cc.y};
    u.m[1][2] = {cc.z, cc.w};
    reconstruct_row2(u);
  }
};

template <> struct LinkField<L_H12> {
  using real = float;
  const uint2* ptr;  // [p][mu][3][Vh]
  int vh;
  WL_D void load(Link<float>& u, int p, int mu, int c) const {
    const uint2* b = ptr + ((long long)(p * 4 + mu) * 3) * vh + c;
    uint2 a = ldg(b), bb = ldg(b + vh), cc = ldg(b + 2LL * vh);
    float2 t;
    t = h2f(a.x); u.m[0][0] = {t.x, t.y};
    t = h2f(a.y); u.m[0][1] = {t.x, t.y};
    t = h2f(bb.x); u.m[0][2] = {t.x, t.y};
    t = h2f(bb.y); u.m[1][0] = {t.x, t.y};
    t = h2f(cc.x); u.m[1][1] = {t.x, t.y};
    t = h2f(cc.y); u.m[1][2] = {t.x, t.y};
    reconstruct_row2(u);
  }
};

// Links in the reference layout BMXYIJ for one configuration: complex128 [mu][V][3][3].
template <> struct LinkField<L_REF> {
  using real = double;
  const double2* ptr;
  long long V;
  WL_D void load_flat(Link<double>& u, int mu, long long flat) const {
    const double2* b = ptr + ((long long)mu * V + flat) * 9;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      double2 v = ldg(b + k);
      u.m[k / 3][k % 3] = {v.x, v.y};
    }
  }
};

// ---------------------------------------------------------------- reductions
// Deterministic block reduction of NV doubles; result valid in thread 0.
template <int NV>
WL_D void block_sum(double (&v)[NV], double* smem /* >= NV * 32 */) {
  const int lane = (threadIdx.x + threadIdx.y * blockDim.x) & 31;
  const int warp = (threadIdx.x + threadIdx.y * blockDim.x) >> 5;
  const int nwarps = (blockDim.x * blockDim.y + 31) >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double x = v[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    v[i] = x;
  }
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < NV; ++i) smem[i * 32 + warp] = v[i];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double x = lane < nwarps ? smem[i * 32 + lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      v[i] = x;
    }
  }
}

}  // namespace wl
