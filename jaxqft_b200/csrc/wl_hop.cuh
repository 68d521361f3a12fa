// Wilson hopping stencil for sm_100a.
//
// Computes, for every target site x of one parity (or both), and for NR
// right-hand sides per thread that share one link stream,
//     acc(x) = sum_mu [ (1 + cf g_mu) U_mu(x) psi(x+mu) + (1 + cb g_mu) U_mu^dag(x-mu) psi(x-mu) ]
// with cf = -1, cb = +1 for D and cf = +1, cb = -1 for D^dag (the reference's
// `sign` convention, jaxqft/fermions/wilson.py:228-284 with r = 1), and then
// hands acc to an epilogue functor (xpay, CG update, residual, norms).  The
// -1/2 of the Wilson normalisation lives in the epilogue coefficients.
//
// Spin projection uses the rank-2 structure of (1 +- g_mu) in the basis of
// jaxqft/fermions/gamma.py:14-46 (g0 = s1 x s1, g1 = s1 x s2, g2 = s2 x I,
// g3 = s3 x I):
//   mu=0: h0 = s0 + c s3,   h1 = s1 + c s2,   rows 2,3 = ( c h1,  c h0)
//   mu=1: h0 = s0 - ic s3,  h1 = s1 + ic s2,  rows 2,3 = (-ic h1, ic h0)
//   mu=2: h0 = s0 - ic s2,  h1 = s1 - ic s3,  rows 2,3 = ( ic h0, ic h1)
//   mu=3: c=+1: (2 s0, 2 s1, 0, 0);  c=-1: (0, 0, 2 s2, 2 s3)
// so each hop multiplies the link into two colour vectors instead of four.
#pragma once
#include "wl_common.cuh"

namespace wl {

template <int MU, int C, typename T>
WL_D void spin_project(const Spinor<T>& s, Half<T>& h) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (MU == 0) {
      h.v[0][c] = C > 0 ? s.v[0][c] + s.v[3][c] : s.v[0][c] - s.v[3][c];
      h.v[1][c] = C > 0 ? s.v[1][c] + s.v[2][c] : s.v[1][c] - s.v[2][c];
    } else if (MU == 1) {
      h.v[0][c] = C > 0 ? s.v[0][c] + mul_mi(s.v[3][c]) : s.v[0][c] + mul_i(s.v[3][c]);
      h.v[1][c] = C > 0 ? s.v[1][c] + mul_i(s.v[2][c]) : s.v[1][c] + mul_mi(s.v[2][c]);
    } else if (MU == 2) {
      h.v[0][c] = C > 0 ? s.v[0][c] + mul_mi(s.v[2][c]) : s.v[0][c] + mul_i(s.v[2][c]);
      h.v[1][c] = C > 0 ? s.v[1][c] + mul_mi(s.v[3][c]) : s.v[1][c] + mul_i(s.v[3][c]);
    } else {
      h.v[0][c] = C > 0 ? T(2) * s.v[0][c] : T(2) * s.v[2][c];
      h.v[1][c] = C > 0 ? T(2) * s.v[1][c] : T(2) * s.v[3][c];
    }
  }
}

template <int MU, int C, typename T>
WL_D void spin_accum(Spinor<T>& a, const Half<T>& h) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (MU == 0) {
      a.v[0][c] = a.v[0][c] + h.v[0][c];
      a.v[1][c] = a.v[1][c] + h.v[1][c];
      a.v[2][c] = C > 0 ? a.v[2][c] + h.v[1][c] : a.v[2][c] - h.v[1][c];
      a.v[3][c] = C > 0 ? a.v[3][c] + h.v[0][c] : a.v[3][c] - h.v[0][c];
    } else if (MU == 1) {
      a.v[0][c] = a.v[0][c] + h.v[0][c];
      a.v[1][c] = a.v[1][c] + h.v[1][c];
      a.v[2][c] = C > 0 ? a.v[2][c] + mul_mi(h.v[1][c]) : a.v[2][c] + mul_i(h.v[1][c]);
      a.v[3][c] = C > 0 ? a.v[3][c] + mul_i(h.v[0][c]) : a.v[3][c] + mul_mi(h.v[0][c]);
    } else if (MU == 2) {
      a.v[0][c] = a.v[0][c] + h.v[0][c];
      a.v[1][c] = a.v[1][c] + h.v[1][c];
      a.v[2][c] = C > 0 ? a.v[2][c] + mul_i(h.v[0][c]) : a.v[2][c] + mul_mi(h.v[0][c]);
      a.v[3][c] = C > 0 ? a.v[3][c] + mul_i(h.v[1][c]) : a.v[3][c] + mul_mi(h.v[1][c]);
    } else {
      if (C > 0) {
        a.v[0][c] = a.v[0][c] + h.v[0][c];
        a.v[1][c] = a.v[1][c] + h.v[1][c];
      } else {
        a.v[2][c] = a.v[2][c] + h.v[0][c];
        a.v[3][c] = a.v[3][c] + h.v[1][c];
      }
    }
  }
}

// uh = U h  (fwd) or U^dag h (bwd), both spin rows
template <bool DAGU, typename T>
WL_D void color_mul(const Link<T>& u, const Half<T>& h, Half<T>& o) {
#pragma unroll
  for (int s = 0; s < 2; ++s)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      cplx<T> acc = {T(0), T(0)};
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        if (DAGU) fmac_(acc, u.m[b][a], h.v[s][b]);
        else fma_(acc, u.m[a][b], h.v[s][b]);
      }
      o.v[s][a] = acc;
    }
}

template <typename T>
WL_D void phase_mul(Half<T>& h, T re, T im) {
#pragma unroll
  for (int s = 0; s < 2; ++s)
#pragma unroll
    for (int a = 0; a < 3; ++a) h.v[s][a] = h.v[s][a] * cplx<T>{re, im};
}

// Index maps: internal compact layout vs reference flat layout.
struct IdxCompact {
  WL_D static long long self(const Geom&, const Site& s) { return s.c; }
  WL_D static long long nb(const Geom& g, const Site& s, int mu, int dir) { return neighbor(g, s, mu, dir); }
};
struct IdxFlat {
  WL_D static long long self(const Geom& g, const Site& s) { return (long long)s.row * g.L[3] + s.x[3]; }
  WL_D static long long nb(const Geom& g, const Site& s, int mu, int dir) {
    int x[4] = {s.x[0], s.x[1], s.x[2], s.x[3]};
    int v = x[mu] + dir;
    x[mu] = v < 0 ? v + g.L[mu] : (v >= g.L[mu] ? v - g.L[mu] : v);
    return (((long long)x[0] * g.L[1] + x[1]) * g.L[2] + x[2]) * g.L[3] + x[3];
  }
};

// Reference-layout link field adapter with the internal load() signature.
struct LinkRefAdapter {
  using real = double;
  LinkField<L_REF> f;
  WL_D void load(Link<double>& u, int /*p*/, int mu, long long flat) const { f.load_flat(u, mu, flat); }
};
// Reference-layout spinor adapter
struct SpinorRefAdapter {
  using real = double;
  SpinorRef f;
  WL_D void load(Spinor<double>& s, int rhs, long long flat) const { f.load(s, rhs, flat); }
  WL_D void load_plain(Spinor<double>& s, int rhs, long long flat) const { f.load(s, rhs, flat); }
  WL_D void store(const Spinor<double>& s, int rhs, long long flat) const { f.store(s, rhs, flat); }
};

template <int MU, bool DAG, int NR, class IDX, class LF, class SF, typename T>
WL_D void hop_dir(const Geom& g, const LF& links, const SF& src, int parity, const Site& s, int rhs0,
                  const bool (&act)[NR], Spinor<T> (&acc)[NR]) {
  constexpr int CF = DAG ? +1 : -1;
  constexpr int CB = -CF;
  {  // forward: U_mu(x) psi(x+mu), link stored on the target parity
    const long long nb = IDX::nb(g, s, MU, +1);
    Link<T> u;
    links.load(u, parity, MU, IDX::self(g, s));
    const bool ph = g.ph_on[MU] && (s.x[MU] == g.L[MU] - 1);
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      if (!act[r]) continue;
      Spinor<T> p;
      src.load(p, rhs0 + r, nb);
      Half<T> h, uh;
      spin_project<MU, CF>(p, h);
      color_mul<false>(u, h, uh);
      if (ph) phase_mul(uh, T(g.ph_re[MU]), T(g.ph_im[MU]));
      spin_accum<MU, CF>(acc[r], uh);
    }
  }
  {  // backward: U_mu(x-mu)^dag psi(x-mu), link stored on the other parity
    const long long nb = IDX::nb(g, s, MU, -1);
    Link<T> u;
    links.load(u, 1 - parity, MU, nb);
    const bool ph = g.ph_on[MU] && (s.x[MU] == 0);
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      if (!act[r]) continue;
      Spinor<T> p;
      src.load(p, rhs0 + r, nb);
      Half<T> h, uh;
      spin_project<MU, CB>(p, h);
      color_mul<true>(u, h, uh);
      if (ph) phase_mul(uh, T(g.ph_re[MU]), T(-g.ph_im[MU]));
      spin_accum<MU, CB>(acc[r], uh);
    }
  }
}

// Launch-wide reductions: every block writes one partial sum per RHS it
// covers into partials[rhs][block]; reduce_finalize_kernel (launched right
// after, one block per RHS) adds them in a fixed order.  Deterministic run to
// run, no floating-point atomics and no per-block fences.  (Finishing the sum
// in the last block of the launch instead -- a fence, a block counter and one
// block reading every partial -- was measured slower on the 16^3x32 HMC
// solves: the fence before each block's count lengthened every hop by more
// than the finalize launch it saved.)
struct Reduce {
  double* partials;   // [nrhs][nblk]
  unsigned* counter;  // unused (kept for layout stability)
  double* result;     // [nrhs]
  const double* num;  // optional: quot[rhs] = num[rhs] / result[rhs] (0 when result <= 0)
  double* quot;
};

constexpr int kMaxRB = 16;  // RHS per block (BY * NR)

template <int NR>
WL_D void reduce_rhs(const double (&val)[NR], const Reduce& R, int nrhs, const int* mask) {
  __shared__ double sred[kMaxRB * 8];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int lane = tx & 31, wx = tx >> 5, nwx = blockDim.x >> 5;
  const int RB = blockDim.y * NR;
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    double x = val[r];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sred[(ty * NR + r) * 8 + wx] = x;
  }
  __syncthreads();
  const int tid = ty * blockDim.x + tx;
  const int nblk = gridDim.x * gridDim.z;
  const int blk = blockIdx.z * gridDim.x + blockIdx.x;
  const int rbase = blockIdx.y * RB;
  if (tid < RB) {
    double x = 0.0;
    for (int w = 0; w < nwx; ++w) x += sred[tid * 8 + w];
    const int rhs = rbase + tid;
    if (rhs < nrhs) R.partials[(long long)rhs * nblk + blk] = x;
  }
}

// result[rhs] = sum_b partials[rhs][b] in a fixed order, for RHS in `mask`:
// one 1024-thread block per RHS, eight independent accumulators per thread so
// that enough loads are in flight to stream the partials at a useful rate.
constexpr int kFinalizeThreads = 1024;

__global__ void __launch_bounds__(kFinalizeThreads) reduce_finalize_kernel(Reduce R, int nrhs, int nblk,
                                                                            const int* mask) {
  __shared__ double sm[32];
  const int rhs = blockIdx.x;
  if (rhs >= nrhs) return;
  if (mask != nullptr && mask[rhs] == 0) return;  // uniform per block
  const double* p = R.partials + (long long)rhs * nblk;
  double a[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  constexpr int step = 8 * kFinalizeThreads;
  int b = threadIdx.x;
  for (; b + 7 * kFinalizeThreads < nblk; b += step) {
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] += p[b + k * kFinalizeThreads];
  }
  for (; b < nblk; b += kFinalizeThreads) a[0] += p[b];
  double v[1] = {((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]))};
  block_sum<1>(v, sm);
  if (threadIdx.x == 0) {
    R.result[rhs] = v[0];
    if (R.quot) R.quot[rhs] = v[0] > 0.0 ? R.num[rhs] / v[0] : 0.0;
  }
}

// Generic launch parameters
template <class LF, class SF, class EPI>
struct HopArgs {
  Geom g;
  LF links;
  SF src[2];        // indexed by source parity (= 1 - target parity)
  int parity0;      // target parity of blockIdx.z == 0
  int nrhs;
  const int* mask;  // per-RHS gate (nullptr: all)
  EPI epi;
  Reduce red;
};

template <bool DAG, int NR, class IDX, class LF, class SF, class EPI>
__global__ void __launch_bounds__(256) hop_kernel(HopArgs<LF, SF, EPI> A) {
  using T = typename SF::real;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int parity = A.parity0 ^ blockIdx.z;
  const int rhs0 = (blockIdx.y * blockDim.y + threadIdx.y) * NR;
  double red[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) red[r] = 0.0;
  if (c < A.g.Vh) {
    bool act[NR];
    bool any = false;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      act[r] = (rhs0 + r < A.nrhs) && (A.mask == nullptr || A.mask[rhs0 + r] != 0);
      any |= act[r];
    }
    if (any) {
      const Site s = site_from_compact(A.g, parity, c);
      Spinor<T> acc[NR];
#pragma unroll
      for (int r = 0; r < NR; ++r) zero(acc[r]);
      const SF& src = A.src[1 - parity];
      hop_dir<0, DAG, NR, IDX>(A.g, A.links, src, parity, s, rhs0, act, acc);
      hop_dir<1, DAG, NR, IDX>(A.g, A.links, src, parity, s, rhs0, act, acc);
      hop_dir<2, DAG, NR, IDX>(A.g, A.links, src, parity, s, rhs0, act, acc);
      hop_dir<3, DAG, NR, IDX>(A.g, A.links, src, parity, s, rhs0, act, acc);
      const long long self = IDX::self(A.g, s);
#pragma unroll
      for (int r = 0; r < NR; ++r)
        if (act[r]) red[r] = A.epi(rhs0 + r, parity, self, acc[r]);
    }
  }
  if (EPI::kReduce) reduce_rhs<NR>(red, A.red, A.nrhs, A.mask);
}

// ------------------------------------------------------------------ one RHS, two threads per site
// Single-RHS stencil (FP64 or FP32 storage) with a pair of threads per target
// site.  Thread j (j = lane & 1) forms half-spinor row j of every hop,
//   mu=0: h = s_j + c s_{3-j}      mu=1: h = s_j + (1-2j) c' s_{3-j}
//   mu=2: h = s_j + c' s_{2+j}     mu=3: 2 s_j (c = +1) or 2 s_{2+j} (c = -1)
// (c' = -i c), so it loads only the two spin components it needs; both threads
// of a pair read the same link addresses in the same instruction (one memory
// request).  Thread j keeps three colour vectors: its own upper spin A = a_j
// and partial sums X of a_{3-j} and Y of a_{2+j}; one xor-shuffle exchange
// assembles the site in thread 0, which runs the epilogue.  Per thread this
// holds about half the registers of hop_kernel, so twice as many threads per
// SM keep neighbour loads in flight.  FP64 engines of 1-3 slots use it at
// 24^3x48; for FP32 storage it is an autotuner candidate (at 16^3x32 with one
// RHS, an L2-resident working set, the thread-per-site FP32 kernel measured
// faster: 10.3 against 12.3 us per half-lattice hop).

// Spin s (three colours) of an FP32 record: complex z = 3 s + colour sits in
// 16-byte chunk z / 2 (half z % 2), so spin s is chunk (3 s - (s & 1)) / 2 from
// colour 0 (even s: the whole chunk; odd s: its upper half) and the next chunk.
WL_D void pair_spin_load(const SpinorField<P_SINGLE>& f, int rhs, unsigned c, int s, cplx<float> (&v)[3]) {
  const int odd = s & 1;
  const int k0 = (3 * s - odd) >> 1;
  const float4 q0 = ldg(f.ptr + f.at(rhs, k0, c));
  const float4 q1 = ldg(f.ptr + f.at(rhs, k0 + 1, c));
  v[0] = odd ? cplx<float>{q0.z, q0.w} : cplx<float>{q0.x, q0.y};
  v[1] = odd ? cplx<float>{q1.x, q1.y} : cplx<float>{q0.z, q0.w};
  v[2] = odd ? cplx<float>{q1.z, q1.w} : cplx<float>{q1.x, q1.y};
}
WL_D void pair_spin_load(const SpinorField<P_DOUBLE>& f, int rhs, unsigned c, int s, cplx<double> (&v)[3]) {
#pragma unroll
  for (int col = 0; col < 3; ++col) {
    const double2 a = ldg(f.ptr + f.at(rhs, s * 3 + col, c));
    v[col] = {a.x, a.y};
  }
}

template <int MU, int C, class SF, typename T>
WL_D void pair_project(const SF& src, int rhs, unsigned nb, int j, T sg, cplx<T> (&h)[3]) {
  const int s1 = (MU == 3 && C < 0) ? 2 + j : j;
  const int s2 = MU == 2 ? 2 + j : 3 - j;
  cplx<T> a[3], b[3];
  pair_spin_load(src, rhs, nb, s1, a);
  if (MU < 3) pair_spin_load(src, rhs, nb, s2, b);
#pragma unroll
  for (int col = 0; col < 3; ++col) {
    if (MU == 3) {
      h[col] = {T(2) * a[col].re, T(2) * a[col].im};
      continue;
    }
    if (MU == 0) {
      h[col] = C > 0 ? a[col] + b[col] : a[col] - b[col];
    } else {
      const cplx<T> w = C > 0 ? mul_mi(b[col]) : mul_i(b[col]);  // w = -i C b
      if (MU == 1) h[col] = {fma(sg, w.re, a[col].re), fma(sg, w.im, a[col].im)};
      else h[col] = a[col] + w;
    }
  }
}

// Accumulate colour component a of one hop, uh, into A, X, Y (see above).
template <int MU, int C, typename T>
WL_D void pair_accum(int a, cplx<T> uh, T sg, cplx<T> (&A)[3], cplx<T> (&X)[3], cplx<T> (&Y)[3]) {
  if (MU == 3) {
    if (C > 0) A[a] = A[a] + uh;
    else Y[a] = Y[a] + uh;
    return;
  }
  A[a] = A[a] + uh;
  if (MU == 0) {
    X[a] = C > 0 ? X[a] + uh : X[a] - uh;
  } else if (MU == 1) {  // X += (1-2j) (i C) uh
    const cplx<T> w = C > 0 ? mul_i(uh) : mul_mi(uh);
    X[a] = {fma(sg, w.re, X[a].re), fma(sg, w.im, X[a].im)};
  } else {  // Y += (i C) uh
    Y[a] = Y[a] + (C > 0 ? mul_i(uh) : mul_mi(uh));
  }
}

template <int MU, int C, bool DAGU, typename T>
WL_D void pair_hop(const Link<T>& u, const cplx<T> (&h)[3], bool ph, const Geom& g, T sg, cplx<T> (&A)[3],
                   cplx<T> (&X)[3], cplx<T> (&Y)[3]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    cplx<T> uh = {T(0), T(0)};
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      if (DAGU) fmac_(uh, u.m[b][a], h[b]);
      else fma_(uh, u.m[a][b], h[b]);
    }
    if (ph) uh = uh * cplx<T>{T(g.ph_re[MU]), T(DAGU ? -g.ph_im[MU] : g.ph_im[MU])};
    pair_accum<MU, C>(a, uh, sg, A, X, Y);
  }
}

template <int MU, bool DAG, class LF, class SF, typename T>
WL_D void pair_dir(const Geom& g, const LF& links, const SF& src, int parity, const Site& s, int rhs, int j, T sg,
                   cplx<T> (&A)[3], cplx<T> (&X)[3], cplx<T> (&Y)[3]) {
  constexpr int CF = DAG ? +1 : -1;
  constexpr int CB = -CF;
  {
    const unsigned nb = (unsigned)neighbor(g, s, MU, +1);
    Link<T> u;
    links.load(u, parity, MU, s.c);
    cplx<T> h[3];
    pair_project<MU, CF>(src, rhs, nb, j, sg, h);
    pair_hop<MU, CF, false>(u, h, g.ph_on[MU] && (s.x[MU] == g.L[MU] - 1), g, sg, A, X, Y);
  }
  {
    const unsigned nb = (unsigned)neighbor(g, s, MU, -1);
    Link<T> u;
    links.load(u, 1 - parity, MU, (int)nb);
    cplx<T> h[3];
    pair_project<MU, CB>(src, rhs, nb, j, sg, h);
    pair_hop<MU, CB, true>(u, h, g.ph_on[MU] && (s.x[MU] == 0), g, sg, A, X, Y);
  }
}

template <typename T>
WL_D cplx<T> shfl_pair(cplx<T> v) {
  return {__shfl_xor_sync(0xffffffffu, v.re, 1), __shfl_xor_sync(0xffffffffu, v.im, 1)};
}

// Resident 256-thread blocks per SM the pair kernel is compiled for.  FP64: 2
// caps it at 128 registers (no spills); measured at 24^3x48, 1 RHS: 96 us,
// against 148 us at 80 registers (3 blocks, spills) and 103 us for hop_kernel
// (144 registers).  FP32 storage and arithmetic: 3 (80 registers).
#ifndef WL_HOP_PAIR_MINB
#define WL_HOP_PAIR_MINB 2
#endif
#ifndef WL_HOP_PAIR_MINB_S
#define WL_HOP_PAIR_MINB_S 3
#endif
template <class SF> struct PairMinBlocks {
  static constexpr int value = WL_HOP_PAIR_MINB;
};
template <> struct PairMinBlocks<SpinorField<P_SINGLE>> {
  static constexpr int value = WL_HOP_PAIR_MINB_S;
};

template <bool DAG, class LF, class SF, class EPI>
__global__ void __launch_bounds__(256, PairMinBlocks<SF>::value) hop_pair_kernel(HopArgs<LF, SF, EPI> A) {
  using T = typename SF::real;
  static_assert(std::is_same<T, typename LF::real>::value, "links and spinors in the same arithmetic");
  const int c = blockIdx.x * (blockDim.x >> 1) + (threadIdx.x >> 1);
  const int j = threadIdx.x & 1;
  const T sg = T(1) - T(2) * T(j);
  const int parity = A.parity0 ^ blockIdx.z;
  const int rhs = blockIdx.y;
  const bool act = c < A.g.Vh && rhs < A.nrhs && (A.mask == nullptr || A.mask[rhs] != 0);
  cplx<T> Ac[3], Xc[3], Yc[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) Ac[a] = Xc[a] = Yc[a] = {T(0), T(0)};
  Site s{};
  if (act) {
    s = site_from_compact(A.g, parity, c);
    const SF& src = A.src[1 - parity];
    pair_dir<0, DAG>(A.g, A.links, src, parity, s, rhs, j, sg, Ac, Xc, Yc);
    pair_dir<1, DAG>(A.g, A.links, src, parity, s, rhs, j, sg, Ac, Xc, Yc);
    pair_dir<2, DAG>(A.g, A.links, src, parity, s, rhs, j, sg, Ac, Xc, Yc);
    pair_dir<3, DAG>(A.g, A.links, src, parity, s, rhs, j, sg, Ac, Xc, Yc);
  }
  // thread 0 of the pair: a0 = A, a1 = A', a2 = Y + X', a3 = X + Y'
  Spinor<T> acc;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const cplx<T> Ap = shfl_pair(Ac[a]), Xp = shfl_pair(Xc[a]), Yp = shfl_pair(Yc[a]);
    acc.v[0][a] = Ac[a];
    acc.v[1][a] = Ap;
    acc.v[2][a] = Yc[a] + Xp;
    acc.v[3][a] = Xc[a] + Yp;
  }
  double red[1] = {0.0};
  if (act && j == 0) red[0] = A.epi(rhs, parity, s.c, acc);
  if (EPI::kReduce) reduce_rhs<1>(red, A.red, A.nrhs, A.mask);
}

// ------------------------------------------------------------------ epilogues
template <typename T>
WL_D double snorm2(const Spinor<T>& s) {
  double n = 0.0;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) n += (double)norm2(s.v[a][c]);
  return n;
}

template <typename T>
WL_D void axpby(Spinor<T>& o, T a, const Spinor<T>& x, T b, const Spinor<T>& y) {
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int c = 0; c < 3; ++c) o.v[s][c] = a * x.v[s][c] + b * y.v[s][c];
}

// out = a[rhs] * self + b[rhs] * acc, optional |out|^2 reduction.
// self may be absent (has_self = 0).  a/b are per-RHS device arrays.
template <class SF, bool RED>
struct EpiXpay {
  static constexpr bool kReduce = RED;
  SF out[2];
  SF self[2];
  int has_self;
  const double* a;  // per-RHS coefficients, or nullptr to use a0/b0
  const double* b;
  double a0, b0;
  WL_D double operator()(int rhs, int parity, long long idx, Spinor<typename SF::real>& acc) const {
    using T = typename SF::real;
    Spinor<T> o;
    const T bb = T(b ? b[rhs] : b0);
    if (has_self) {
      Spinor<T> x;
      self[parity].load(x, rhs, idx);
      axpby(o, T(a ? a[rhs] : a0), x, bb, acc);
    } else {
#pragma unroll
      for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int c = 0; c < 3; ++c) o.v[s][c] = bb * acc.v[s][c];
    }
    out[parity].store(o, rhs, idx);
    return RED ? snorm2(o) : 0.0;
  }
  // same on packed FP32 pairs (FP16/FP32 fields, RHS-in-lanes kernels)
  WL_D double packed(int rhs, int parity, unsigned idx, float2 (&acc)[12]) const {
    const float bb = float(b ? b[rhs] : b0);
    const float2 b2 = f2(bb, bb);
    if (has_self) {
      float2 x[12];
      const float sx = Packed<SF>::load(self[parity], rhs, idx, x) * float(a ? a[rhs] : a0);
      const float2 s2 = f2(sx, sx);
#pragma unroll
      for (int k = 0; k < 12; ++k) acc[k] = ffma2(b2, acc[k], fmul2(s2, x[k]));
    } else {
#pragma unroll
      for (int k = 0; k < 12; ++k) acc[k] = fmul2(b2, acc[k]);
    }
    Packed<SF>::store(out[parity], rhs, idx, acc);
    return RED ? pnorm2(acc) : 0.0;
  }
  // same on one colour of an FP16 record (tensor-core hop): slice_in issues the loads
  // early, slice_out (called by every lane of the warp) finishes the record
  struct SliceIn {
    SliceHalf::Raw x;
  };
  WL_D SliceIn slice_in(int rhs, int parity, unsigned idx, int t, bool mine) const {
    return SliceIn{SliceHalf::load(self[parity], rhs, idx, t, mine && has_self)};
  }
  WL_D double slice_out(const SliceIn& in, int rhs, int parity, unsigned idx, int t, bool act,
                        float2 (&acc)[4]) const {
    const float bb = act ? float(b ? b[rhs] : b0) : 0.f;
    const float2 b2 = f2(bb, bb);
    if (has_self) {
      float2 x[4];
      const float sx = SliceHalf::unpack(in.x, x) * (act ? float(a ? a[rhs] : a0) : 0.f);
      const float2 s2 = f2(sx, sx);
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[k] = ffma2(b2, acc[k], fmul2(s2, x[k]));
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[k] = fmul2(b2, acc[k]);
    }
    SliceHalf::store(out[parity], rhs, idx, t, act, acc);
    return RED ? pnorm2_4(acc) : 0.0;
  }
};

}  // namespace wl
