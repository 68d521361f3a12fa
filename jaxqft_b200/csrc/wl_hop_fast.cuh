// Wilson hop for FP32 arithmetic (FP16 or FP32 storage) written for the
// sm_100 packed FP32x2 pipe: every complex value is a float2 (re, im) and
// every complex multiply-add is two __ffma2_rn:
//     c += u * h   ==   c += (u.re, u.re) * (h.re, h.im) + (-u.im, u.im) * (h.im, h.re)
// The FP16 per-site norm, the factor 2 of the mu=3 projector and the +-1 /
// +-i reconstruction coefficients are folded into the accumulation weights, so
// they cost no extra instructions.  Same contract and epilogues as hop_kernel
// (wl_hop.cuh): acc = sum_mu [(1+cf g_mu) U psi(x+mu) + (1+cb g_mu) U^dag psi(x-mu)].
#pragma once
#include "wl_hop.cuh"

namespace wl {

// Raw spinor load: values without the FP16 per-site norm (returned separately).
template <class SF> struct RawLoad;

template <> struct RawLoad<SpinorField<P_SINGLE>> {
  WL_D static float load(const SpinorField<P_SINGLE>& f, int rhs, long long c, float2 (&s)[12]) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      float4 v = ldg(f.ptr + f.at(rhs, k, c));
      s[2 * k] = f2(v.x, v.y);
      s[2 * k + 1] = f2(v.z, v.w);
    }
    return 1.0f;
  }
};

template <> struct RawLoad<SpinorField<P_HALF>> {
  WL_D static float load(const SpinorField<P_HALF>& f, int rhs, long long c, float2 (&s)[12]) {
    const float n = ldg(f.norm + f.nat(rhs, c));
#pragma unroll
    for (int k = 0; k < 3; ++k) {  // chunk k = colour k, spins 0..3
      uint4 v = ldg(f.ptr + f.at(rhs, k, c));
      s[k] = h2f(v.x);
      s[3 + k] = h2f(v.y);
      s[6 + k] = h2f(v.z);
      s[9 + k] = h2f(v.w);
    }
    return n;
  }
};

// Link as packed pairs: R[a][b] = (re, re), I[a][b] = (-im, im) of U_ab.
struct LinkPairs {
  float2 R[3][3], I[3][3];
};

WL_D void make_pairs(const Link<float>& u, LinkPairs& p) {
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      p.R[a][b] = f2(u.m[a][b].re, u.m[a][b].re);
      p.I[a][b] = f2(-u.m[a][b].im, u.m[a][b].im);
    }
}

// h[s*3+a], s in {0,1}: the rank-2 projection (1 + C g_mu) psi, top two rows,
// WITHOUT the factor 2 of mu=3 (folded into the weight).
template <int MU, int C>
WL_D void project2(const float2 (&s)[12], float2 (&h)[6]) {
  const float2 pc = f2((float)C, (float)C);
  const float2 pcm = f2((float)C, -(float)C);   // for -iC x = (C x.im, -C x.re) = pcm * swap(x)
  const float2 pmc = f2(-(float)C, (float)C);   // for  iC x = (-C x.im, C x.re) = pmc * swap(x)
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float2 s0 = s[c], s1 = s[3 + c], s2 = s[6 + c], s3 = s[9 + c];
    if (MU == 0) {
      h[c] = ffma2(pc, s3, s0);
      h[3 + c] = ffma2(pc, s2, s1);
    } else if (MU == 1) {
      h[c] = ffma2(pcm, swp(s3), s0);      // s0 - iC s3
      h[3 + c] = ffma2(pmc, swp(s2), s1);  // s1 + iC s2
    } else if (MU == 2) {
      h[c] = ffma2(pcm, swp(s2), s0);      // s0 - iC s2
      h[3 + c] = ffma2(pcm, swp(s3), s1);  // s1 - iC s3
    } else {
      h[c] = C > 0 ? s0 : s2;
      h[3 + c] = C > 0 ? s1 : s3;
    }
  }
}

// uh = U h (DAGU = false) or U^dag h (DAGU = true), both rows.
template <bool DAGU>
WL_D void color_mul2(const LinkPairs& p, const float2 (&h)[6], float2 (&uh)[6]) {
#pragma unroll
  for (int sp = 0; sp < 2; ++sp) {
    float2 hs[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) hs[b] = swp(h[sp * 3 + b]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float2 acc = f2(0.f, 0.f);
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        if (DAGU) {  // conj(U_ba): (re, re) h + (im, -im) swap(h)
          acc = ffma2(p.R[b][a], h[sp * 3 + b], acc);
          acc = ffma2(f2(-p.I[b][a].x, -p.I[b][a].y), hs[b], acc);
        } else {
          acc = ffma2(p.R[a][b], h[sp * 3 + b], acc);
          acc = ffma2(p.I[a][b], hs[b], acc);
        }
      }
      uh[sp * 3 + a] = acc;
    }
  }
}

// acc += w * full spinor reconstructed from uh (rows 0,1 = uh; rows 2,3 by MU, C).
template <int MU, int C>
WL_D void accum2(float2 (&acc)[12], const float2 (&uh)[6], float w) {
  const float2 ww = f2(w, w);
  const float2 cw = f2(C * w, C * w);
  const float2 pcm = f2(C * w, -C * w);   // -iC w x = pcm * swap(x)
  const float2 pmc = f2(-C * w, C * w);   //  iC w x = pmc * swap(x)
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float2 u0 = uh[c], u1 = uh[3 + c];
    if (MU == 3) {
      if (C > 0) {
        acc[c] = ffma2(ww, u0, acc[c]);
        acc[3 + c] = ffma2(ww, u1, acc[3 + c]);
      } else {
        acc[6 + c] = ffma2(ww, u0, acc[6 + c]);
        acc[9 + c] = ffma2(ww, u1, acc[9 + c]);
      }
      continue;
    }
    acc[c] = ffma2(ww, u0, acc[c]);
    acc[3 + c] = ffma2(ww, u1, acc[3 + c]);
    if (MU == 0) {
      acc[6 + c] = ffma2(cw, u1, acc[6 + c]);
      acc[9 + c] = ffma2(cw, u0, acc[9 + c]);
    } else if (MU == 1) {
      acc[6 + c] = ffma2(pcm, swp(u1), acc[6 + c]);  // -iC u1
      acc[9 + c] = ffma2(pmc, swp(u0), acc[9 + c]);  //  iC u0
    } else {
      acc[6 + c] = ffma2(pmc, swp(u0), acc[6 + c]);  //  iC u0
      acc[9 + c] = ffma2(pmc, swp(u1), acc[9 + c]);  //  iC u1
    }
  }
}

template <int MU, bool DAG, int NR, class LF, class SF>
WL_D void hop_dir_fast(const Geom& g, const LF& links, const SF& src, int parity, const Site& s, int rhs0,
                       const bool (&act)[NR], float2 (&acc)[NR][12]) {
  constexpr int CF = DAG ? +1 : -1;
  constexpr int CB = -CF;
  constexpr float W3 = (MU == 3) ? 2.0f : 1.0f;
#pragma unroll
  for (int dir = 0; dir < 2; ++dir) {
    const long long nb = neighbor(g, s, MU, dir == 0 ? +1 : -1);
    Link<float> u;
    if (dir == 0) links.load(u, parity, MU, s.c);
    else links.load(u, 1 - parity, MU, nb);
    LinkPairs lp;
    make_pairs(u, lp);
    const bool ph = g.ph_on[MU] && (dir == 0 ? (s.x[MU] == g.L[MU] - 1) : (s.x[MU] == 0));
    const float phr = (float)g.ph_re[MU], phi = dir == 0 ? (float)g.ph_im[MU] : -(float)g.ph_im[MU];
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      if (!act[r]) continue;
      float2 sp[12];
      const float n = RawLoad<SF>::load(src, rhs0 + r, nb, sp) * W3;
      float2 h[6], uh[6];
      if (dir == 0) {
        project2<MU, CF>(sp, h);
        color_mul2<false>(lp, h, uh);
      } else {
        project2<MU, CB>(sp, h);
        color_mul2<true>(lp, h, uh);
      }
      if (ph) {
#pragma unroll
        for (int k = 0; k < 6; ++k) uh[k] = ffma2(f2(phr, phr), uh[k], fmul2(f2(-phi, phi), swp(uh[k])));
      }
      if (dir == 0) accum2<MU, CF>(acc[r], uh, n);
      else accum2<MU, CB>(acc[r], uh, n);
    }
  }
}

template <bool DAG, int NR, class LF, class SF, class EPI>
__global__ void __launch_bounds__(256) hop_fast_kernel(HopArgs<LF, SF, EPI> A) {
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
      float2 acc[NR][12];
#pragma unroll
      for (int r = 0; r < NR; ++r)
#pragma unroll
        for (int k = 0; k < 12; ++k) acc[r][k] = f2(0.f, 0.f);
      const SF& src = A.src[1 - parity];
      hop_dir_fast<0, DAG, NR>(A.g, A.links, src, parity, s, rhs0, act, acc);
      hop_dir_fast<1, DAG, NR>(A.g, A.links, src, parity, s, rhs0, act, acc);
      hop_dir_fast<2, DAG, NR>(A.g, A.links, src, parity, s, rhs0, act, acc);
      hop_dir_fast<3, DAG, NR>(A.g, A.links, src, parity, s, rhs0, act, acc);
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        if (!act[r]) continue;
        Spinor<float> o;
#pragma unroll
        for (int k = 0; k < 12; ++k) o.v[k / 3][k % 3] = {acc[r][k].x, acc[r][k].y};
        red[r] = A.epi(rhs0 + r, parity, (long long)c, o);
      }
    }
  }
  if (EPI::kReduce) reduce_rhs<NR>(red, A.red, A.nrhs, A.mask);
}

// ============================================================================
// Multi-RHS hop with RHS in the lanes.  A block of 128 threads covers
// S = 128 / R sites x R right-hand sides (lane = rhs + R * site).  Phase 1:
// each warp reconstructs the 8 links of each of its 32/R sites once into shared
// memory as packed pairs (boundary phase folded in) together with the
// neighbour indices; a warp barrier (not a block barrier) ends the phase.
// Phase 2: every lane runs the stencil for its (site, RHS), reading
// the site's links as shared-memory broadcasts.  Spinor loads stay
// sector-efficient: lanes r of sites c and c+1 read the two 16-byte halves of
// one 32-byte sector.
constexpr int kLaneBlock = 128;
// Resident blocks per SM the FP32-arithmetic lane kernel is compiled for,
// per epilogue: 7 (72 registers, 28 warps per SM) for K_oe p and the fused
// CG hop, 8 (64 registers, 32 warps) for the reducing xpay hop (M p with
// |Mp|^2) and the plain dagger hop (K^dag_oe y).  Enough warps hide the L2
// latency of the neighbour gathers; more registers cut spill and
// rematerialisation work.  Measured at 24^3x48 with 16 FP16 RHS (whole
// batched solve, interleaved runs): this split 344.6-346.2 ms, 7 blocks for
// all four 346.9-347.6 ms; on another box 7 blocks for all 348.5-349.0 ms,
// 8 blocks for all 350.0-350.5 ms, 6 blocks for all 357.5 ms; on a third box
// this split 351.8-352.9 ms, 6 blocks (80 registers) for the CG hop alone or
// for K_oe p alone 356.2-357.0 ms.  Each cap can be overridden with -D.
#ifndef WL_LANE_MIN_BLOCKS
#define WL_LANE_MIN_BLOCKS 7
#endif
#ifndef WL_LANE_MIN_BLOCKS_XPAY_RED
#define WL_LANE_MIN_BLOCKS_XPAY_RED 8
#endif
#ifndef WL_LANE_MIN_BLOCKS_DAG_XPAY
#define WL_LANE_MIN_BLOCKS_DAG_XPAY 8
#endif
#ifndef WL_LANE_MIN_BLOCKS_CG
#define WL_LANE_MIN_BLOCKS_CG WL_LANE_MIN_BLOCKS
#endif
#ifndef WL_LANE_MIN_BLOCKS_XPAY
#define WL_LANE_MIN_BLOCKS_XPAY WL_LANE_MIN_BLOCKS
#endif
// The FP16-accumulation form (HA) holds its sums as half2 and needs fewer registers: 8 blocks
// (64 registers) for every epilogue measured faster than the split above (49.9-50.1 against
// 49.3-49.5 solves/s in interleaved whole-solve runs at 24^3x48 with 16 RHS) and than 9 blocks
// (56 registers, 20-byte spills: 48.7-48.9 against 49.1-49.5).
#ifndef WL_LANE_MIN_BLOCKS_HA
#define WL_LANE_MIN_BLOCKS_HA 8
#endif
template <class SF>
struct EpiCG;  // wl_site.cuh
template <bool DAG, class EPI>
struct LaneMinBlocks {
  static constexpr int value = WL_LANE_MIN_BLOCKS;
};
template <bool DAG, class SF>
struct LaneMinBlocks<DAG, EpiXpay<SF, true>> {
  static constexpr int value = WL_LANE_MIN_BLOCKS_XPAY_RED;
};
template <class SF>
struct LaneMinBlocks<true, EpiXpay<SF, false>> {
  static constexpr int value = WL_LANE_MIN_BLOCKS_DAG_XPAY;
};
template <class SF>
struct LaneMinBlocks<false, EpiXpay<SF, false>> {
  static constexpr int value = WL_LANE_MIN_BLOCKS_XPAY;
};
template <bool DAG, class SF>
struct LaneMinBlocks<DAG, EpiCG<SF>> {
  static constexpr int value = WL_LANE_MIN_BLOCKS_CG;
};

struct LinkSmem {
  float4 p[9];  // (R.x, R.y, I.x, I.y) for element (a, b) = k / 3, k % 3
};

// One site's 8 links; the 16-byte pad makes the per-site stride 1168 B so the
// sites read by one warp fall in different shared-memory banks.
struct SiteLinks {
  LinkSmem l[8];  // q = 2*mu + dir
  float4 pad;
};

template <int R>
struct LaneSmem {
  static constexpr int S = kLaneBlock / R;
  SiteLinks link[S];
  int nb[S][8];
  int ok[S];
};

template <bool DAGU>
WL_D void color_mul_smem(const LinkSmem& L, const float2 (&h)[6], float2 (&uh)[6]) {
#pragma unroll
  for (int sp = 0; sp < 2; ++sp) {
    float2 hs[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) hs[b] = swp(h[sp * 3 + b]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float2 acc = f2(0.f, 0.f);
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const float4 q = DAGU ? L.p[b * 3 + a] : L.p[a * 3 + b];
        acc = ffma2(f2(q.x, q.y), h[sp * 3 + b], acc);
        acc = DAGU ? ffma2(f2(-q.z, -q.w), hs[b], acc) : ffma2(f2(q.z, q.w), hs[b], acc);
      }
      uh[sp * 3 + a] = acc;
    }
  }
}

// FP16 projection: the rank-2 projection is formed on the stored half2 values
// (packed FP16 add/FMA, one rounding to FP16) and only the six projected
// components are converted to FP32, instead of all twelve.  For mu = 3 the
// projection is a selection and the two unused spins are not loaded.
// Measured at 24^3x48, 16 RHS: hop 0.329 -> 0.320 ms at a lower clock, CG
// iteration and reliable-update counts unchanged (156-165, 16).
#ifndef WL_HALF_PROJECT
#define WL_HALF_PROJECT 1
#endif

WL_D __half2 as_h2(unsigned int u) { return *reinterpret_cast<__half2*>(&u); }

// s[spin*3 + colour] of an FP16 record; for mu = 3 the projector keeps two spins
// (0, 1 for C > 0, else 2, 3), so only those 8 bytes of each colour chunk are loaded.
template <int MU, int C>
WL_D void load_half_spins(const SpinorField<P_HALF>& f, int rhs, unsigned c, __half2 (&s)[12]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (MU == 3) {
      const uint2* q = reinterpret_cast<const uint2*>(f.ptr + f.at(rhs, k, c)) + (C > 0 ? 0 : 1);
      const uint2 v = __ldg(q);
      s[(C > 0 ? 0 : 6) + k] = as_h2(v.x);
      s[(C > 0 ? 3 : 9) + k] = as_h2(v.y);
    } else {
      const uint4 v = ldg(f.ptr + f.at(rhs, k, c));
      s[k] = as_h2(v.x);
      s[3 + k] = as_h2(v.y);
      s[6 + k] = as_h2(v.z);
      s[9 + k] = as_h2(v.w);
    }
  }
}

// the projection as half2 values (rows 0, 1 x colours), no conversion and no norm
template <int MU, int C>
WL_D void load_project_half2_raw(const SpinorField<P_HALF>& f, int rhs, unsigned c, __half2 (&h)[6]);

// the projection as half2 values (rows 0, 1 x colours), no conversion; returns the site norm
template <int MU, int C>
WL_D float load_project_half2(const SpinorField<P_HALF>& f, int rhs, unsigned c, __half2 (&h)[6]) {
  const float n = ldg(f.norm + f.nat(rhs, c));
  load_project_half2_raw<MU, C>(f, rhs, c, h);
  return n;
}

template <int MU, int C>
WL_D void load_project_half2_raw(const SpinorField<P_HALF>& f, int rhs, unsigned c, __half2 (&h)[6]) {
  __half2 s[12];
  load_half_spins<MU, C>(f, rhs, c, s);
  const __half2 pcm = __floats2half2_rn((float)C, -(float)C);  // -iC x = pcm * swap(x)
  const __half2 pmc = __floats2half2_rn(-(float)C, (float)C);  //  iC x = pmc * swap(x)
#pragma unroll
  for (int col = 0; col < 3; ++col) {
    const __half2 s0 = s[col], s1 = s[3 + col], s2 = s[6 + col], s3 = s[9 + col];
    if (MU == 0) {
      h[col] = C > 0 ? __hadd2(s0, s3) : __hsub2(s0, s3);
      h[3 + col] = C > 0 ? __hadd2(s1, s2) : __hsub2(s1, s2);
    } else if (MU == 1) {
      h[col] = __hfma2(pcm, __lowhigh2highlow(s3), s0);
      h[3 + col] = __hfma2(pmc, __lowhigh2highlow(s2), s1);
    } else if (MU == 2) {
      h[col] = __hfma2(pcm, __lowhigh2highlow(s2), s0);
      h[3 + col] = __hfma2(pcm, __lowhigh2highlow(s3), s1);
    } else {
      h[col] = C > 0 ? s0 : s2;
      h[3 + col] = C > 0 ? s1 : s3;
    }
  }
}

template <int MU, int C>
WL_D float load_project_half(const SpinorField<P_HALF>& f, int rhs, unsigned c, float2 (&h)[6]) {
  const float n = ldg(f.norm + f.nat(rhs, c));
  __half2 s[12];
  load_half_spins<MU, C>(f, rhs, c, s);
  const __half2 pcm = __floats2half2_rn((float)C, -(float)C);  // -iC x = pcm * swap(x)
  const __half2 pmc = __floats2half2_rn(-(float)C, (float)C);  //  iC x = pmc * swap(x)
#pragma unroll
  for (int col = 0; col < 3; ++col) {
    const __half2 s0 = s[col], s1 = s[3 + col], s2 = s[6 + col], s3 = s[9 + col];
    __half2 h0, h1;
    if (MU == 0) {
      h0 = C > 0 ? __hadd2(s0, s3) : __hsub2(s0, s3);
      h1 = C > 0 ? __hadd2(s1, s2) : __hsub2(s1, s2);
    } else if (MU == 1) {
      h0 = __hfma2(pcm, __lowhigh2highlow(s3), s0);  // s0 - iC s3
      h1 = __hfma2(pmc, __lowhigh2highlow(s2), s1);  // s1 + iC s2
    } else if (MU == 2) {
      h0 = __hfma2(pcm, __lowhigh2highlow(s2), s0);  // s0 - iC s2
      h1 = __hfma2(pcm, __lowhigh2highlow(s3), s1);  // s1 - iC s3
    } else {
      h0 = C > 0 ? s0 : s2;
      h1 = C > 0 ? s1 : s3;
    }
    h[col] = __half22float2(h0);
    h[3 + col] = __half22float2(h1);
  }
  return n;
}

template <int MU, bool DAG, class SF>
WL_D void lane_dir(const SF& src, const LinkSmem* Ls, const int* nbs, int rhs, float2 (&acc)[12]) {
  constexpr int CF = DAG ? +1 : -1;
  constexpr int CB = -CF;
  constexpr float W3 = (MU == 3) ? 2.0f : 1.0f;
  constexpr bool kHalfProject = WL_HALF_PROJECT && std::is_same<SF, SpinorField<P_HALF>>::value;
#pragma unroll
  for (int dir = 0; dir < 2; ++dir) {
    const int q = 2 * MU + dir;
    float2 h[6], uh[6];
    float n;
    if constexpr (kHalfProject) {
      n = (dir == 0 ? load_project_half<MU, CF>(src, rhs, (unsigned)nbs[q], h)
                    : load_project_half<MU, CB>(src, rhs, (unsigned)nbs[q], h)) * W3;
    } else {
      float2 sp[12];
      n = RawLoad<SF>::load(src, rhs, (long long)nbs[q], sp) * W3;
      if (dir == 0) project2<MU, CF>(sp, h);
      else project2<MU, CB>(sp, h);
    }
    if (dir == 0) {
      color_mul_smem<false>(Ls[q], h, uh);
      accum2<MU, CF>(acc, uh, n);
    } else {
      color_mul_smem<true>(Ls[q], h, uh);
      accum2<MU, CB>(acc, uh, n);
    }
  }
}

// Colour multiply in packed FP16 (HFMA2, FP16 accumulation of the three terms), the default
// for FP16 fields: the FP32 pairs of the multiply are what throttles the FMA pipe of the hop
// (math-pipe stalls about as frequent as L2-gather stalls), and an HFMA2 does the same two
// multiply-adds in half the pipe time.  The link element k of a hop is staged as two half2, (re, re) and
// (-im, im) for a forward hop, (re, re) and (im, -im) -- the conjugate -- for a backward one,
// so U h and U^dag h are the same two HFMA2 per complex multiply-add.  h stays in FP16 (no
// conversion); the six products are converted to FP32 for the accumulation.
struct LinkSmemH {
  uint2 p[9];  // (re, re), (-+im, +-im) as half2 pairs
};

// The nine link pairs of a hop, read from the start of its 16-byte aligned LinkSmem
// slot as four 128-bit and one 64-bit shared loads instead of nine 64-bit ones.
WL_D void load_link_pairs(const LinkSmem& slot, uint2 (&e)[9]) {
  const uint4* L4 = reinterpret_cast<const uint4*>(&slot);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint4 v = L4[i];
    e[2 * i] = make_uint2(v.x, v.y);
    e[2 * i + 1] = make_uint2(v.z, v.w);
  }
  e[8] = reinterpret_cast<const LinkSmemH*>(&slot)->p[8];
}

template <bool DAGU>
WL_D void color_mul_half(const LinkSmem& L, const __half2 (&h)[6], float2 (&uh)[6]) {
  uint2 e[9];
  load_link_pairs(L, e);
#pragma unroll
  for (int sp = 0; sp < 2; ++sp) {
    __half2 hs[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) hs[b] = __lowhigh2highlow(h[sp * 3 + b]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      __half2 acc = __float2half2_rn(0.f);
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const uint2 q = DAGU ? e[b * 3 + a] : e[a * 3 + b];
        acc = __hfma2(as_h2(q.x), h[sp * 3 + b], acc);
        acc = __hfma2(as_h2(q.y), hs[b], acc);
      }
      uh[sp * 3 + a] = __half22float2(acc);
    }
  }
}

// Ls: the site's LinkSmem slots; a hop's FP16 pairs sit at the start of its slot
template <int MU, bool DAG>
WL_D void lane_dir_hc(const SpinorField<P_HALF>& src, const LinkSmem* Ls, const int* nbs, int rhs,
                      float2 (&acc)[12]) {
  constexpr int CF = DAG ? +1 : -1;
  constexpr int CB = -CF;
  constexpr float W3 = (MU == 3) ? 2.0f : 1.0f;
#pragma unroll
  for (int dir = 0; dir < 2; ++dir) {
    const int q = 2 * MU + dir;
    __half2 h[6];
    float2 uh[6];
    const float n = (dir == 0 ? load_project_half2<MU, CF>(src, rhs, (unsigned)nbs[q], h)
                              : load_project_half2<MU, CB>(src, rhs, (unsigned)nbs[q], h)) * W3;
    const LinkSmem& L = Ls[q];
    if (dir == 0) {
      color_mul_half<false>(L, h, uh);
      accum2<MU, CF>(acc, uh, n);
    } else {
      color_mul_half<true>(L, h, uh);
      accum2<MU, CB>(acc, uh, n);
    }
  }
}

// FP16 accumulation.  The eight contributions of a site are summed in packed
// FP16 with weights relative to the largest neighbour norm of this (site, RHS):
// w_q = n_q / max n (times the factor 2 of mu = 3), so every weight is in
// [0, 2] and the sums stay far inside the FP16 range (|U h| <= 2 sqrt 3 per
// component); the FP32 result is the FP16 sum times max n.  This drops the six
// half2 -> FP32 conversions per hop, and the accumulation is one HFMA2 per
// complex term with the +-1 / +-i reconstruction folded into the weight pair.
template <bool DAGU>
WL_D void color_mul_hh(const LinkSmem& L, const __half2 (&h)[6], __half2 (&uh)[6]) {
  uint2 e[9];
  load_link_pairs(L, e);
#pragma unroll
  for (int sp = 0; sp < 2; ++sp) {
    __half2 hs[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) hs[b] = __lowhigh2highlow(h[sp * 3 + b]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      __half2 acc = __float2half2_rn(0.f);
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const uint2 q = DAGU ? e[b * 3 + a] : e[a * 3 + b];
        acc = __hfma2(as_h2(q.x), h[sp * 3 + b], acc);
        acc = __hfma2(as_h2(q.y), hs[b], acc);
      }
      uh[sp * 3 + a] = acc;
    }
  }
}

template <int MU, int C>
WL_D void accum2_hh(__half2 (&acc)[12], const __half2 (&uh)[6], float w) {
  const __half2 ww = __float2half2_rn(w);
  const __half2 cw = __float2half2_rn(C * w);
  const __half2 pcm = __floats2half2_rn(C * w, -C * w);  // -iC w x = pcm * swap(x)
  const __half2 pmc = __floats2half2_rn(-C * w, C * w);  //  iC w x = pmc * swap(x)
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const __half2 u0 = uh[c], u1 = uh[3 + c];
    if (MU == 3) {
      if (C > 0) {
        acc[c] = __hfma2(ww, u0, acc[c]);
        acc[3 + c] = __hfma2(ww, u1, acc[3 + c]);
      } else {
        acc[6 + c] = __hfma2(ww, u0, acc[6 + c]);
        acc[9 + c] = __hfma2(ww, u1, acc[9 + c]);
      }
      continue;
    }
    acc[c] = __hfma2(ww, u0, acc[c]);
    acc[3 + c] = __hfma2(ww, u1, acc[3 + c]);
    if (MU == 0) {
      acc[6 + c] = __hfma2(cw, u1, acc[6 + c]);
      acc[9 + c] = __hfma2(cw, u0, acc[9 + c]);
    } else if (MU == 1) {
      acc[6 + c] = __hfma2(pcm, __lowhigh2highlow(u1), acc[6 + c]);  // -iC u1
      acc[9 + c] = __hfma2(pmc, __lowhigh2highlow(u0), acc[9 + c]);  //  iC u0
    } else {
      acc[6 + c] = __hfma2(pmc, __lowhigh2highlow(u0), acc[6 + c]);  //  iC u0
      acc[9 + c] = __hfma2(pmc, __lowhigh2highlow(u1), acc[9 + c]);  //  iC u1
    }
  }
}

// w[q]: the relative weights of the site's eight neighbours for this RHS
template <int MU, bool DAG>
WL_D void lane_dir_hh(const SpinorField<P_HALF>& src, const LinkSmem* Ls, const int* nbs, int rhs,
                      const float (&w)[8], __half2 (&acc)[12]) {
  constexpr int CF = DAG ? +1 : -1;
  constexpr int CB = -CF;
#pragma unroll
  for (int dir = 0; dir < 2; ++dir) {
    const int q = 2 * MU + dir;
    __half2 h[6], uh[6];
    if (dir == 0) load_project_half2_raw<MU, CF>(src, rhs, (unsigned)nbs[q], h);
    else load_project_half2_raw<MU, CB>(src, rhs, (unsigned)nbs[q], h);
    const LinkSmem& L = Ls[q];
    if (dir == 0) {
      color_mul_hh<false>(L, h, uh);
      accum2_hh<MU, CF>(acc, uh, w[q]);
    } else {
      color_mul_hh<true>(L, h, uh);
      accum2_hh<MU, CB>(acc, uh, w[q]);
    }
  }
}

// The whole stencil of one (site, RHS) with FP16 accumulation; acc = FP32 result.
template <bool DAG>
WL_D void lane_site_hh(const SpinorField<P_HALF>& src, const LinkSmem* Ls, const int* nbs, int rhs,
                       float2 (&acc)[12]) {
  float w[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) w[q] = ldg(src.norm + src.nat(rhs, (unsigned)nbs[q]));
  float m = 0.f;
#pragma unroll
  for (int q = 0; q < 8; ++q) m = fmaxf(m, w[q]);
  const float im = m > 0.f ? 1.0f / m : 0.f;
#pragma unroll
  for (int q = 0; q < 8; ++q) w[q] *= (q >= 6 ? 2.0f * im : im);
  __half2 ah[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) ah[k] = __float2half2_rn(0.f);
  lane_dir_hh<0, DAG>(src, Ls, nbs, rhs, w, ah);
  lane_dir_hh<1, DAG>(src, Ls, nbs, rhs, w, ah);
  lane_dir_hh<2, DAG>(src, Ls, nbs, rhs, w, ah);
  lane_dir_hh<3, DAG>(src, Ls, nbs, rhs, w, ah);
  const float2 m2 = f2(m, m);
#pragma unroll
  for (int k = 0; k < 12; ++k) acc[k] = fmul2(m2, __half22float2(ah[k]));
}

// Link q = 2 mu + dir of target site c (compact index, target parity) with the
// boundary phase folded in, staged as FP32 quads (re, re, -im, im) or, for the
// FP16 colour multiply (HC), as two half2 (re, re), (-+im, +-im) (backward hops
// stage the conjugate); returns the compact index of the neighbour it hops to.
template <bool HC, class LF, class DST>
WL_D int stage_link(const Geom& g, const LF& links, int parity, int c, int mu, int dir, DST& dst) {
  const Site s = site_from_compact(g, parity, c);
  const int nb = neighbor(g, s, mu, dir == 0 ? +1 : -1);
  Link<float> u;
  if (dir == 0) links.load(u, parity, mu, c);
  else links.load(u, 1 - parity, mu, nb);
  // the forward hop from x_mu = L-1 uses ph*U; the backward hop into
  // x_mu = 0 uses (ph*U)^dag, i.e. the same phase-multiplied link
  const bool ph = g.ph_on[mu] && (dir == 0 ? (s.x[mu] == g.L[mu] - 1) : (s.x[mu] == 0));
  if (ph) {
    const cplx<float> w{(float)g.ph_re[mu], (float)g.ph_im[mu]};
#pragma unroll
    for (int k = 0; k < 9; ++k) u.m[k / 3][k % 3] = u.m[k / 3][k % 3] * w;
  }
  if constexpr (HC) {
    LinkSmemH* lh = reinterpret_cast<LinkSmemH*>(&dst);
    const float sgn = dir == 0 ? 1.0f : -1.0f;  // backward hops use the conjugate
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const cplx<float> v = u.m[k / 3][k % 3];
      lh->p[k] = make_uint2(f2h(v.re, v.re), f2h(-sgn * v.im, sgn * v.im));
    }
  } else {
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const cplx<float> v = u.m[k / 3][k % 3];
      dst.p[k] = make_float4(v.re, v.re, -v.im, v.im);
    }
  }
  return nb;
}

// Per-block partial sums: xor-shuffles over the sites of a warp leave lanes
// 0..R-1 with the warp's sum for RHS rbase + lane; after one barrier threads
// 0..R-1 add the block's warps in a fixed order and block b writes
// partials[rhs][b].  Every thread of the block must call this.
constexpr int kLaneWarps = kLaneBlock / 32;
static_assert(kLaneWarps == 4, "reduce_lanes adds four warps");

// rbase: first RHS of the block's group (blockIdx.y * R unless a block works through several
// groups); a block that calls it more than once must pass again = true after the first call.
template <int R>
WL_D void reduce_lanes(double v, const Reduce& Rd, int nrhs, const int* /*mask*/, int rbase = -1,
                       bool again = false) {
  __shared__ double sred[kLaneWarps][32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int off = R; off < 32; off <<= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if (again) __syncthreads();  // the previous call's readers are done with sred
  if (lane < R) sred[warp][lane] = v;
  __syncthreads();
  if (tid < R) {
    const double x = (sred[0][tid] + sred[1][tid]) + (sred[2][tid] + sred[3][tid]);
    const int nblk = gridDim.x * gridDim.z;
    const int blk = blockIdx.z * gridDim.x + blockIdx.x;
    const int rhs = (rbase < 0 ? (int)blockIdx.y * R : rbase) + tid;
    if (rhs < nrhs) Rd.partials[(long long)rhs * nblk + blk] = x;
  }
}

template <bool DAG, int R, class LF, class SF, class EPI, bool HC = false, bool HA = false>
__global__ void __launch_bounds__(kLaneBlock, HA ? WL_LANE_MIN_BLOCKS_HA : LaneMinBlocks<DAG, EPI>::value)
    hop_lanes_kernel(HopArgs<LF, SF, EPI> A) {
  static_assert(!HC || std::is_same<SF, SpinorField<P_HALF>>::value, "FP16 colour multiply needs FP16 fields");
  static_assert(!HA || HC, "FP16 accumulation runs behind the FP16 colour multiply");
  constexpr int S = kLaneBlock / R;
  __shared__ LaneSmem<R> sm;
  const int tid = threadIdx.x;
  const int parity = A.parity0 ^ blockIdx.z;
  const int site0 = blockIdx.x * S;
  // ---- phase 1: links (phase-folded packed pairs) and neighbour indices.
  // Each warp stages the links of its own 32/R sites, so only a warp barrier
  // separates the phases and warps of one block do not wait for each other.
  constexpr int SPW = 32 / R;
  const int wsite = (tid >> 5) * SPW;
  for (int j = tid & 31; j < 8 * SPW; j += 32) {
    const int sl = wsite + (j >> 3), q = j & 7, mu = q >> 1, dir = q & 1;
    const int c = site0 + sl;
    if (c < A.g.Vh) {
      sm.nb[sl][q] = stage_link<HC>(A.g, A.links, parity, c, mu, dir, sm.link[sl].l[q]);
      if (q == 0) sm.ok[sl] = 1;
    } else if (q == 0) {
      sm.ok[sl] = 0;
    }
  }
  __syncwarp();
  // ---- phase 2: stencil for (site, rhs) of this lane (a site of this warp)
  const int sl = tid / R;
  const int c = site0 + sl;
  const int rhs = blockIdx.y * R + (tid % R);
  double red = 0.0;
  const bool act = sm.ok[sl] && rhs < A.nrhs && (A.mask == nullptr || A.mask[rhs] != 0);
  if (act) {
    float2 acc[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = f2(0.f, 0.f);
    const SF& src = A.src[1 - parity];
    const int* nbs = sm.nb[sl];
    if constexpr (HA) {
      lane_site_hh<DAG>(src, sm.link[sl].l, nbs, rhs, acc);
    } else if constexpr (HC) {
      const LinkSmem* Ls = sm.link[sl].l;
      lane_dir_hc<0, DAG>(src, Ls, nbs, rhs, acc);
      lane_dir_hc<1, DAG>(src, Ls, nbs, rhs, acc);
      lane_dir_hc<2, DAG>(src, Ls, nbs, rhs, acc);
      lane_dir_hc<3, DAG>(src, Ls, nbs, rhs, acc);
    } else {
      const LinkSmem* Ls = sm.link[sl].l;
      lane_dir<0, DAG>(src, Ls, nbs, rhs, acc);
      lane_dir<1, DAG>(src, Ls, nbs, rhs, acc);
      lane_dir<2, DAG>(src, Ls, nbs, rhs, acc);
      lane_dir<3, DAG>(src, Ls, nbs, rhs, acc);
    }
    red = A.epi.packed(rhs, parity, (unsigned)c, acc);
  }
  if (EPI::kReduce) reduce_lanes<R>(red, A.red, A.nrhs, A.mask);
}

// ============================================================================
#ifndef WL_LANE_D_MIN_BLOCKS
#define WL_LANE_D_MIN_BLOCKS 4  // resident blocks per SM the FP64 lane kernel is compiled for (128 registers)
#endif

// FP64 stencil with RHS in the lanes, for the reliable updates of the batched
// solver (FP64 fields RHS-innermost).  Same two phases as hop_lanes_kernel:
// each site's 8 links are reconstructed once per block into shared memory
// (boundary phase folded in), then every lane applies them to its RHS.  The
// spin projection is fused with the load, one colour at a time, so a full
// FP64 source spinor is never live in registers; for mu = 3 only the two spin
// rows the projector keeps are loaded.
struct SiteLinksD {
  double2 m[8][9];  // q = 2*mu + dir; element (a, b) at a*3 + b
  double2 pad;      // 1168-byte stride: the sites of one warp hit different banks
};

template <int R>
struct LaneSmemD {
  static constexpr int S = kLaneBlock / R;
  SiteLinksD link[S];
  int nb[S][8];
  int ok[S];
  int c[S];  // compact index of each site (tiled sweep order)
};

// h = (1 + C g_mu) psi(nb) rows 0,1 (mu = 3 without its factor 2, applied by the
// caller).  All loads of the direction are issued before any is used (12, or 6
// for mu = 3), so each thread keeps a whole source spinor's worth of requests in
// flight: at 16 warps per SM this is what hides the L2/HBM latency.
template <int MU, int C>
WL_D void load_project_d(const SpinorField<P_DOUBLE>& f, int rhs, unsigned nb, Half<double>& h) {
  constexpr int s_lo = (MU == 3 && C < 0) ? 2 : 0;
  constexpr int s_hi = (MU == 3 && C > 0) ? 2 : 4;
  double2 v[4][3];
#pragma unroll
  for (int sp = s_lo; sp < s_hi; ++sp)
#pragma unroll
    for (int col = 0; col < 3; ++col) v[sp][col] = ldg(f.ptr + f.at(rhs, sp * 3 + col, nb));
#pragma unroll
  for (int col = 0; col < 3; ++col) {
    if (MU == 3) {
      h.v[0][col] = cplx<double>{v[s_lo][col].x, v[s_lo][col].y};
      h.v[1][col] = cplx<double>{v[s_lo + 1][col].x, v[s_lo + 1][col].y};
      continue;
    }
    const cplx<double> s0{v[0][col].x, v[0][col].y}, s1{v[1][col].x, v[1][col].y};
    const cplx<double> s2{v[2][col].x, v[2][col].y}, s3{v[3][col].x, v[3][col].y};
    if (MU == 0) {
      h.v[0][col] = C > 0 ? s0 + s3 : s0 - s3;
      h.v[1][col] = C > 0 ? s1 + s2 : s1 - s2;
    } else if (MU == 1) {
      h.v[0][col] = C > 0 ? s0 + mul_mi(s3) : s0 + mul_i(s3);
      h.v[1][col] = C > 0 ? s1 + mul_i(s2) : s1 + mul_mi(s2);
    } else {
      h.v[0][col] = C > 0 ? s0 + mul_mi(s2) : s0 + mul_i(s2);
      h.v[1][col] = C > 0 ? s1 + mul_mi(s3) : s1 + mul_i(s3);
    }
  }
}

template <bool DAGU>
WL_D void color_mul_smem_d(const double2 (&m)[9], const Half<double>& h, Half<double>& o) {
#pragma unroll
  for (int s = 0; s < 2; ++s)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      cplx<double> acc = {0.0, 0.0};
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const double2 u = DAGU ? m[b * 3 + a] : m[a * 3 + b];
        if (DAGU) fmac_(acc, cplx<double>{u.x, u.y}, h.v[s][b]);
        else fma_(acc, cplx<double>{u.x, u.y}, h.v[s][b]);
      }
      o.v[s][a] = acc;
    }
}

template <int MU, bool DAG>
WL_D void lane_dir_d(const SpinorField<P_DOUBLE>& src, const SiteLinksD& Ls, const int* nbs, int rhs,
                     Spinor<double>& acc) {
  constexpr int CF = DAG ? +1 : -1;
  constexpr int CB = -CF;
#pragma unroll
  for (int dir = 0; dir < 2; ++dir) {
    const int q = 2 * MU + dir;
    Half<double> h, uh;
    if (dir == 0) {
      load_project_d<MU, CF>(src, rhs, (unsigned)nbs[q], h);
      color_mul_smem_d<false>(Ls.m[q], h, uh);
    } else {
      load_project_d<MU, CB>(src, rhs, (unsigned)nbs[q], h);
      color_mul_smem_d<true>(Ls.m[q], h, uh);
    }
    if (MU == 3) {
#pragma unroll
      for (int s = 0; s < 2; ++s)
#pragma unroll
        for (int a = 0; a < 3; ++a) uh.v[s][a] = 2.0 * uh.v[s][a];
    }
    if (dir == 0) spin_accum<MU, CF>(acc, uh);
    else spin_accum<MU, CB>(acc, uh);
  }
}

// G > 1: the block works through G groups of R right-hand sides one after the other on the
// links it staged once (grid.y = ceil(nrhs / (R G))), so each link is read once per launch
// instead of once per group.
template <bool DAG, int R, class LF, class EPI, int G = 1>
__global__ void __launch_bounds__(kLaneBlock, WL_LANE_D_MIN_BLOCKS) hop_lanes_d_kernel(HopArgs<LF, SpinorField<P_DOUBLE>, EPI> A) {
  constexpr int S = kLaneBlock / R;
  __shared__ LaneSmemD<R> sm;
  const int tid = threadIdx.x;
  const int parity = A.parity0 ^ blockIdx.z;
  const int site0 = blockIdx.x * S;
  constexpr int SPW = 32 / R;  // sites per warp: each warp stages its own links
  const int wsite = (tid >> 5) * SPW;
  for (int j = tid & 31; j < 8 * SPW; j += 32) {
    const int sl = wsite + (j >> 3), q = j & 7, mu = q >> 1, dir = q & 1;
    const int cl = site0 + sl;
    if (cl < A.g.Vh) {
      const int c = tiled_compact(A.g, cl);
      const Site s = site_from_compact(A.g, parity, c);
      const int nb = neighbor(A.g, s, mu, dir == 0 ? +1 : -1);
      Link<double> u;
      if (dir == 0) A.links.load(u, parity, mu, c);
      else A.links.load(u, 1 - parity, mu, nb);
      const bool ph = A.g.ph_on[mu] && (dir == 0 ? (s.x[mu] == A.g.L[mu] - 1) : (s.x[mu] == 0));
      if (ph) {
        const cplx<double> w{A.g.ph_re[mu], A.g.ph_im[mu]};
#pragma unroll
        for (int k = 0; k < 9; ++k) u.m[k / 3][k % 3] = u.m[k / 3][k % 3] * w;
      }
#pragma unroll
      for (int k = 0; k < 9; ++k) sm.link[sl].m[q][k] = make_double2(u.m[k / 3][k % 3].re, u.m[k / 3][k % 3].im);
      sm.nb[sl][q] = nb;
      if (q == 0) {
        sm.ok[sl] = 1;
        sm.c[sl] = c;
      }
    } else if (q == 0) {
      sm.ok[sl] = 0;
    }
  }
  __syncwarp();
  const int sl = tid / R;
#pragma unroll 1
  for (int u = 0; u < G; ++u) {
    const int rbase = ((int)blockIdx.y * G + u) * R;
    const int rhs = rbase + (tid % R);
    double red = 0.0;
    const bool act = sm.ok[sl] && rhs < A.nrhs && (A.mask == nullptr || A.mask[rhs] != 0);
    if (act) {
      Spinor<double> acc;
      zero(acc);
      const SpinorField<P_DOUBLE>& src = A.src[1 - parity];
      lane_dir_d<0, DAG>(src, sm.link[sl], sm.nb[sl], rhs, acc);
      lane_dir_d<1, DAG>(src, sm.link[sl], sm.nb[sl], rhs, acc);
      lane_dir_d<2, DAG>(src, sm.link[sl], sm.nb[sl], rhs, acc);
      lane_dir_d<3, DAG>(src, sm.link[sl], sm.nb[sl], rhs, acc);
      red = A.epi(rhs, parity, (long long)sm.c[sl], acc);
    }
    if (EPI::kReduce) reduce_lanes<R>(red, A.red, A.nrhs, A.mask, rbase, u > 0);
  }
}

}  // namespace wl
