// FP64 Wilson hop on reference-layout fermions for the drop-in operators (D,
// D^dag, K, the masked and Schur forms): two threads per target site.
//
// Fermions keep the caller's layout: complex128 [rhs][Lx][Ly][Lz][Lt][4][3],
// 192 contiguous bytes per site.  sm_100 has 256-bit global loads and stores
// (ld.global.v4.f64 / st.global.v4.f64), so a spin (48 bytes) is one 32-byte
// vector and one 16-byte half, and a pair of threads reads a neighbour's
// spinor without shared-memory staging or block barriers.  Links come from the
// gauge object's parity-split SoA copy (double2 [p][mu][9][Vh]), so a warp's
// link load is two contiguous runs (the two parities of 8 compact sites)
// instead of a 144-byte-stride gather.  Neighbour spinors and the second use
// of every link (forward from x, backward from x + mu) are L2 hits: the reuse
// distance is at most one x-slice of the lattice (Ly*Lz*Lt sites).
//
// Thread mapping: with both parities targeted (D, D^dag, K) pair i of the grid
// row owns flat site i, so a warp covers 16 consecutive sites; with one target
// parity p pair i owns compact site i of parity p.
//
// Contract = row_hop_kernel: out = a*self + b*acc on the target sites,
//   acc = sum_mu [(1 + cf g_mu) U_mu(x) psi(x+mu) + (1 + cb g_mu) U_mu^dag(x-mu) psi(x-mu)],
// cf = -1 (D) or +1 (D^dag), cb = -cf, boundary phase on the forward hop from
// x_mu = L_mu - 1 and (conjugated) on the backward hop into x_mu = 0.
//
// Measured at 24^3x48 (1 RHS): 0.217 ms, limited by the L1 data pipe (83-88 % of
// its wavefront rate at 33 % of DRAM bandwidth): every load instruction of a
// warp touches one or two sectors of each of its 16 sites.  A one-thread-per-
// site form (six 32-byte loads per neighbour, 168 registers) timed the same.
#pragma once
#include "wl_hop.cuh"

namespace wl {

struct RefSiteArgs {
  Geom g;
  const double2* U;     // FP64 18-real links [p][mu][9][Vh]
  const double* in;     // [nrhs][V][24] reals
  double* out;          // [nrhs][V][24]
  const double* self;   // [nrhs][V][24] or nullptr
  double a, b;
  int nrhs;
  int parity;           // target parity, or -1 for every site
};

// 32-byte (W = 4) or 16-byte (W = 2) vector accesses of doubles.  The 32-byte
// form needs 32-byte aligned addresses; launchers check the field pointers
// (sites are 192 bytes apart, a multiple of 32).
template <int W>
WL_D void ld_vec(const double* p, double* v) {
  if (W == 4) {
    asm volatile("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
                 : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
                 : "l"(p));
  } else {
    const double2 q = __ldg(reinterpret_cast<const double2*>(p));
    v[0] = q.x;
    v[1] = q.y;
  }
}
template <int W>
WL_D void st_vec(double* p, const double* v) {
  if (W == 4) {
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(v[0]), "d"(v[1]), "d"(v[2]), "d"(v[3])
                 : "memory");
  } else {
    *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
  }
}

constexpr int kRefSiteBlock = 128;

// ---------------------------------------------------------------- two threads per site
// Thread j (j = lane & 1) of a pair forms half-spinor row j of every hop (as
// hop_pair_kernel does on the internal layout):
//   mu=0: h = s_j + c s_{3-j}        mu=1: h = s_j + (1-2j) c' s_{3-j}
//   mu=2: h = s_j + c' s_{2+j}       mu=3: 2 s_j (c = +1) or 2 s_{2+j} (c = -1)
// with c' = -i c.  In the reference layout spin s is reals [6s, 6s+6): one
// 32-byte vector plus one 16-byte half.  The pair's 16-byte halves of spins
// (0, 1) and of spins (2, 3) share a sector and are requested by the same
// instruction (the load offsets depend on the spin's parity arithmetically, so
// the pair does not diverge), so a pair requests every sector of a neighbour's
// spinor exactly once.  Both threads read the same link addresses in the same instruction.
// Thread j keeps its upper spin A = a_j and partial sums X of a_{3-j} and Y of
// a_{2+j} (18 doubles instead of 24); at the end two xor-shuffle rounds give
// thread 0 spins (0, 1) and thread 1 spins (2, 3), and each stores its half of
// the site with three 32-byte stores.

// spin s (6 reals) of one site: the 32-byte vector and the 16-byte half
template <int W>
WL_D void ld_spin(const double* site, int s, double (&v)[6]) {
  const double* p = site + 6 * s;
  if (W == 4) {
    // Even s: reals [6s, 6s+4) are a whole 32-byte vector and [6s+4, 6s+6) the lower half of the
    // next; odd s: [6s, 6s+2) the upper half of a vector and [6s+2, 6s+6) a whole one.  The two
    // threads of a pair have spins of different parity, so the offsets are computed, not branched
    // on: both threads issue the same two load instructions.
    const int odd = s & 1;
    double q[4], h[2];
    ld_vec<4>(p + 2 * odd, q);
    ld_vec<2>(p + 4 - 4 * odd, h);
    v[0] = odd ? h[0] : q[0];
    v[1] = odd ? h[1] : q[1];
    v[2] = odd ? q[0] : q[2];
    v[3] = odd ? q[1] : q[3];
    v[4] = odd ? q[2] : h[0];
    v[5] = odd ? q[3] : h[1];
  } else {
#pragma unroll
    for (int k = 0; k < 6; k += 2) ld_vec<2>(p + k, v + k);
  }
}

// the two spins thread j of a pair projects from: s1 (always) and s2 (mu < 3)
template <int MU, int C>
WL_D int pair_spin1(int j) { return (MU == 3 && C < 0) ? 2 + j : j; }
template <int MU>
WL_D int pair_spin2(int j) { return MU == 2 ? 2 + j : 3 - j; }

// half-spinor row j of (1 + C g_mu) psi from its spins a = s1, b = s2 (6 reals each)
template <int MU, int C>
WL_D void pair_combine(const double (&a)[6], const double (&b)[6], double sg, cplx<double> (&h)[3]) {
  if (MU == 3) {
#pragma unroll
    for (int col = 0; col < 3; ++col) h[col] = {2.0 * a[2 * col], 2.0 * a[2 * col + 1]};
    return;
  }
#pragma unroll
  for (int col = 0; col < 3; ++col) {
    const cplx<double> av{a[2 * col], a[2 * col + 1]}, bv{b[2 * col], b[2 * col + 1]};
    if (MU == 0) {
      h[col] = C > 0 ? av + bv : av - bv;
    } else {
      const cplx<double> w = C > 0 ? mul_mi(bv) : mul_i(bv);  // -i C b
      if (MU == 1) h[col] = {fma(sg, w.re, av.re), fma(sg, w.im, av.im)};
      else h[col] = av + w;
    }
  }
}

// Sector loads (SECT): the pair reads a neighbour's 192 bytes as three 64-byte pieces, one
// 32-byte sector per thread per instruction, each piece inside one 128-byte line (the site is
// 64-byte aligned), so an instruction touches one line per site instead of one or two per
// spin.  Sector k holds complex values z[2k], z[2k+1] (z[3 spin + colour]); thread j takes
// the sector of each piece that holds more of its own spins and the pair swaps the rest with
// xor-shuffles (mask pm: the active pairs of the warp):
//   mu = 0, 1 (spins j, 3 - j): pieces (0,1) (3,2) (5,4); 0 <- z2, z9 of thread 1; 1 <- z6, z7
//   mu = 2 (spins j, 2 + j): pieces (0,1) (3,2) (4,5); 0 <- z2, 1 <- z9
//   mu = 3, C > 0 (spin j): pieces (0,1) (3,2); 0 <- z2
//   mu = 3, C < 0 (spin 2 + j): pieces (3,2) (4,5); 1 <- z9
// (piece (x, y): thread 0 loads sector x, thread 1 sector y).
WL_D void ld_sector(const double* site, int sec, double (&v)[4]) { ld_vec<4>(site + 4 * sec, v); }

WL_D double pick(int j, double x0, double x1) { return j ? x1 : x0; }

template <int MU, int C>
WL_D void ld_pair_spins(const double* site, int j, unsigned pm, double (&a)[6], double (&b)[6]) {
  double r0[4], r1[4], r2[4];
  if (MU < 3) {
    ld_sector(site, j, r0);               // (0, 1)
    ld_sector(site, 3 - j, r1);           // (3, 2)
    if (MU < 2) ld_sector(site, 5 - j, r2);  // (5, 4)
    else ld_sector(site, 4 + j, r2);         // (4, 5)
  } else if (C > 0) {
    ld_sector(site, j, r0);
    ld_sector(site, 3 - j, r1);
  } else {
    ld_sector(site, 3 - j, r1);
    ld_sector(site, 4 + j, r2);
  }
  if (MU < 2) {
    // thread 0 sends z6, z7 (r1); thread 1 sends z2 (r0[0..1]) and z9 (r2[2..3])
    double x[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double snd = j ? (k < 2 ? r0[k] : r2[k]) : r1[k];
      x[k] = __shfl_xor_sync(pm, snd, 1);
    }
    // a: spin j (t0: z0 z1 z2 = r0[0..3], x[0..1]; t1: z3 z4 z5 = r0[2..3], r1[0..3])
    // b: spin 3 - j (t0: z9 z10 z11 = x[2..3], r2[0..3]; t1: z6 z7 z8 = x[0..3], r2[0..1])
    a[0] = pick(j, r0[0], r0[2]);
    a[1] = pick(j, r0[1], r0[3]);
    a[2] = pick(j, r0[2], r1[0]);
    a[3] = pick(j, r0[3], r1[1]);
    a[4] = pick(j, x[0], r1[2]);
    a[5] = pick(j, x[1], r1[3]);
    b[0] = pick(j, x[2], x[0]);
    b[1] = pick(j, x[3], x[1]);
    b[2] = pick(j, r2[0], x[2]);
    b[3] = pick(j, r2[1], x[3]);
    b[4] = pick(j, r2[2], r2[0]);
    b[5] = pick(j, r2[3], r2[1]);
  } else if (MU == 2) {
    // thread 0 sends z9 (r2[2..3]); thread 1 sends z2 (r0[0..1])
    double x[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) x[k] = __shfl_xor_sync(pm, j ? r0[k] : r2[2 + k], 1);
    // a: spin j (t0: z0 z1 z2 = r0, x; t1: z3 z4 z5 = r0[2..3], r1)
    // b: spin 2 + j (t0: z6 z7 z8 = r1, r2[0..1]; t1: z9 z10 z11 = x, r2)
    a[0] = pick(j, r0[0], r0[2]);
    a[1] = pick(j, r0[1], r0[3]);
    a[2] = pick(j, r0[2], r1[0]);
    a[3] = pick(j, r0[3], r1[1]);
    a[4] = pick(j, x[0], r1[2]);
    a[5] = pick(j, x[1], r1[3]);
    b[0] = pick(j, r1[0], x[0]);
    b[1] = pick(j, r1[1], x[1]);
    b[2] = pick(j, r1[2], r2[0]);
    b[3] = pick(j, r1[3], r2[1]);
    b[4] = pick(j, r2[0], r2[2]);
    b[5] = pick(j, r2[1], r2[3]);
  } else if (C > 0) {
    // thread 0 receives z2 (thread 1's r0[0..1]); a = spin j
    double x[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) x[k] = __shfl_xor_sync(pm, r0[k], 1);
    a[0] = pick(j, r0[0], r0[2]);
    a[1] = pick(j, r0[1], r0[3]);
    a[2] = pick(j, r0[2], r1[0]);
    a[3] = pick(j, r0[3], r1[1]);
    a[4] = pick(j, x[0], r1[2]);
    a[5] = pick(j, x[1], r1[3]);
  } else {
    // thread 1 receives z9 (thread 0's r2[2..3]); a = spin 2 + j
    double x[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) x[k] = __shfl_xor_sync(pm, r2[2 + k], 1);
    a[0] = pick(j, r1[0], x[0]);
    a[1] = pick(j, r1[1], x[1]);
    a[2] = pick(j, r1[2], r2[0]);
    a[3] = pick(j, r1[3], r2[1]);
    a[4] = pick(j, r2[0], r2[2]);
    a[5] = pick(j, r2[1], r2[3]);
  }
}

template <int MU, int C, int W, bool SECT>
WL_D void refpair_project(const double* site, int j, double sg, unsigned pm, cplx<double> (&h)[3]) {
  double a[6], b[6];
  if (SECT) {
    ld_pair_spins<MU, C>(site, j, pm, a, b);
  } else {
    ld_spin<W>(site, pair_spin1<MU, C>(j), a);
    if (MU < 3) ld_spin<W>(site, pair_spin2<MU>(j), b);
  }
  pair_combine<MU, C>(a, b, sg, h);
}

// links of one hop: forward U_mu(x) (stored with the target's parity p, compact c) or
// backward U_mu(x - mu) (parity 1 - p, compact index of the neighbour)
WL_D void ld_link(const double2* U, unsigned vh, int p, int mu, int c, Link<double>& u) {
  const double2* lk = U + (size_t)(p * 4 + mu) * 9 * vh + c;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const double2 q = ldg(lk + (size_t)k * vh);
    u.m[k / 3][k % 3] = {q.x, q.y};
  }
}

// the pair's epilogue: assemble spins (0,1) in thread 0 and (2,3) in thread 1
// (a0 = A_0, a1 = A_1, a2 = Y_0 + X_1, a3 = X_0 + Y_1, subscript = thread of the pair:
// round 1 thread 0 sends X_0 and receives A_1, round 2 thread 0 sends Y_0), then
// out = a*self + b*acc for this thread's two spins.  Every lane must call it.
template <int W>
WL_D void pair_store(const RefSiteArgs& A, size_t off, bool act, int j, const cplx<double> (&Ac)[3],
                     const cplx<double> (&Xc)[3], const cplx<double> (&Yc)[3]) {
  cplx<double> lo[3], hi[3];  // thread 0: spins 0, 1; thread 1: spins 2, 3
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const cplx<double> r1 = shfl_pair(j == 0 ? Xc[a] : Ac[a]);
    const cplx<double> r2 = shfl_pair(Yc[a]);
    if (j == 0) {
      lo[a] = Ac[a];
      hi[a] = r1;
    } else {
      lo[a] = r2 + Xc[a];
      hi[a] = r1 + Yc[a];
    }
  }
  if (!act) return;
  double o[12];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    o[2 * a] = A.b * lo[a].re;
    o[2 * a + 1] = A.b * lo[a].im;
    o[6 + 2 * a] = A.b * hi[a].re;
    o[6 + 2 * a + 1] = A.b * hi[a].im;
  }
  if (A.self) {
    double x[12];
#pragma unroll
    for (int k = 0; k < 12; k += W) ld_vec<W>(A.self + off + k, x + k);
#pragma unroll
    for (int k = 0; k < 12; ++k) o[k] = fma(A.a, x[k], o[k]);
  }
#pragma unroll
  for (int k = 0; k < 12; k += W) st_vec<W>(A.out + off + k, o + k);
}

// Sector form of pair_store: after the assembly thread j holds sectors 3j..3j+2 of the site
// (its two spins); one more shuffle swaps sector 1 (thread 0) with sector 4 (thread 1), so
// thread j writes sectors j, 2 + j, 4 + j and every store instruction of the pair covers one
// 64-byte piece, as the loads do; the self term is read in the same pieces.  `site` is the
// site's first double.  Every lane must call it.
WL_D void pair_store_sect(const RefSiteArgs& A, size_t site, bool act, int j, const cplx<double> (&Ac)[3],
                          const cplx<double> (&Xc)[3], const cplx<double> (&Yc)[3]) {
  cplx<double> lo[3], hi[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const cplx<double> r1 = shfl_pair(j == 0 ? Xc[a] : Ac[a]);
    const cplx<double> r2 = shfl_pair(Yc[a]);
    if (j == 0) {
      lo[a] = Ac[a];
      hi[a] = r1;
    } else {
      lo[a] = r2 + Xc[a];
      hi[a] = r1 + Yc[a];
    }
  }
  double o[12];  // sectors 3j, 3j + 1, 3j + 2 of b * acc
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    o[2 * a] = A.b * lo[a].re;
    o[2 * a + 1] = A.b * lo[a].im;
    o[6 + 2 * a] = A.b * hi[a].re;
    o[6 + 2 * a + 1] = A.b * hi[a].im;
  }
#pragma unroll
  for (int k = 4; k < 8; ++k) o[k] = __shfl_xor_sync(0xffffffffu, o[k], 1);  // sector 1 <-> sector 4
  if (!act) return;
  // this thread's sectors j, 2 + j, 4 + j, in that order
  double v[12];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = j ? o[4 + k] : o[k];
    v[4 + k] = j ? o[k] : o[8 + k];
    v[8 + k] = j ? o[8 + k] : o[4 + k];
  }
  if (A.self) {
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      double x[4];
      ld_vec<4>(A.self + site + 8 * p + 4 * j, x);
#pragma unroll
      for (int k = 0; k < 4; ++k) v[4 * p + k] = fma(A.a, x[k], v[4 * p + k]);
    }
  }
#pragma unroll
  for (int p = 0; p < 3; ++p) st_vec<4>(A.out + site + 8 * p + 4 * j, v + 4 * p);
}

// site coordinates of flat index f
WL_D Site site_of_flat(const Geom& g, int f) {
  Site s;
  const int c = f >> 1;
  const int row = (int)fdiv(g.fd_lth, (unsigned)c);
  const int t = f - row * g.L[3];
  const int r2 = (int)fdiv(g.fd_l2, (unsigned)row);
  s.c = WL_CHECKED(c, g.Vh);
  s.row = row;
  s.x[2] = row - r2 * g.L[2];
  s.x[0] = (int)fdiv(g.fd_l1, (unsigned)r2);
  s.x[1] = r2 - s.x[0] * g.L[1];
  s.x[3] = t;
  return s;
}

template <int MU, bool DAG, int W, bool SECT>
WL_D void refpair_mu(const RefSiteArgs& A, const double* base, const Site& s, int parity, int j, double sg,
                     unsigned pm, cplx<double> (&Ac)[3], cplx<double> (&Xc)[3], cplx<double> (&Yc)[3]) {
  constexpr int CF = DAG ? +1 : -1;
  constexpr int CB = -CF;
  const Geom& g = A.g;
  const unsigned vh = (unsigned)g.Vh;
#pragma unroll
  for (int dir = 0; dir < 2; ++dir) {
    const int nb = neighbor(g, s, MU, dir == 0 ? +1 : -1);
    int tn = s.x[3];
    if (MU == 3) tn = dir == 0 ? (tn == g.L[3] - 1 ? 0 : tn + 1) : (tn == 0 ? g.L[3] - 1 : tn - 1);
    const double* src = base + (size_t)(2 * nb + (tn & 1)) * 24;
    Link<double> u;
    if (dir == 0) ld_link(A.U, vh, parity, MU, s.c, u);
    else ld_link(A.U, vh, 1 - parity, MU, nb, u);
    cplx<double> h[3];
    if (dir == 0) {
      refpair_project<MU, CF, W, SECT>(src, j, sg, pm, h);
      pair_hop<MU, CF, false>(u, h, g.ph_on[MU] && s.x[MU] == g.L[MU] - 1, g, sg, Ac, Xc, Yc);
    } else {
      refpair_project<MU, CB, W, SECT>(src, j, sg, pm, h);
      pair_hop<MU, CB, true>(u, h, g.ph_on[MU] && s.x[MU] == 0, g, sg, Ac, Xc, Yc);
    }
  }
}

#ifndef WL_REFPAIR_MINB
#define WL_REFPAIR_MINB 4  // resident 128-thread blocks per SM the pair kernel is compiled for
#endif

template <bool DAG, int W, bool SECT = false>
__global__ void __launch_bounds__(kRefSiteBlock, WL_REFPAIR_MINB) ref_pair_kernel(RefSiteArgs A) {
  static_assert(!SECT || W == 4, "sector loads use 32-byte vectors");
  const Geom& g = A.g;
  const int i = blockIdx.x * (blockDim.x >> 1) + (threadIdx.x >> 1);
  const int j = threadIdx.x & 1;
  const double sg = 1.0 - 2.0 * j;
  const int rhs = blockIdx.y;
  const bool act = i < (A.parity < 0 ? g.V : g.Vh);
  Site s{};
  int parity = 0;
  cplx<double> Ac[3], Xc[3], Yc[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) Ac[a] = Xc[a] = Yc[a] = {0.0, 0.0};
  const size_t field = (size_t)rhs * g.V * 24;
  const unsigned pm = __ballot_sync(0xffffffffu, act);  // both threads of a pair share `act`
  if (act) {
    if (A.parity < 0) {  // every site: i is the flat index
      s = site_of_flat(g, i);
      parity = (s.x[0] + s.x[1] + s.x[2] + s.x[3]) & 1;
    } else {  // one parity: i is the compact index
      parity = A.parity;
      s = site_from_compact(g, parity, i);
    }
    const double* base = A.in + field;
    refpair_mu<0, DAG, W, SECT>(A, base, s, parity, j, sg, pm, Ac, Xc, Yc);
    refpair_mu<1, DAG, W, SECT>(A, base, s, parity, j, sg, pm, Ac, Xc, Yc);
    refpair_mu<2, DAG, W, SECT>(A, base, s, parity, j, sg, pm, Ac, Xc, Yc);
    refpair_mu<3, DAG, W, SECT>(A, base, s, parity, j, sg, pm, Ac, Xc, Yc);
  }
  const size_t flat = (size_t)s.row * g.L[3] + s.x[3];
  if (SECT) pair_store_sect(A, field + flat * 24, act, j, Ac, Xc, Yc);
  else pair_store<W>(A, field + flat * 24 + 12 * j, act, j, Ac, Xc, Yc);  // this thread's two spins
}

}  // namespace wl
