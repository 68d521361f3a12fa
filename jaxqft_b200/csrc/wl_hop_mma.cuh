// Wilson hop on the tensor cores for FP16 fields, 8 RHS per block.
//
// For one target site x the hop over 8 RHS is a single real contraction:
//     out[(r, s), (a, ri)] = sum_{d, b, ri'} A[(r, s), (d, b, ri')] * B_d[(b, ri'), (a, ri)]
// where d runs over the 8 hops, r over the RHS, s over the 4 output spins, a, b
// over colours and ri, ri' over (re, im).  The A row for output spin s holds
// the weighted, spin-projected neighbour h' = w_d * R_{d,s} P_d psi(x +- mu):
// rows of spins 0, 1 are the two projected rows, those of spins 2, 3 the +-1 /
// +-i multiples the reconstruction of the projector gives (so the
// reconstruction costs nothing in the contraction), and B_d is the realified
// link U (forward) or U^dag (backward).  Each site is 8 mma.sync m16n8k16 (FP16
// inputs, FP32 accumulation): 2 tiles of 16 rows (tile j: RHS 0-7 for output
// spin 2j, then RHS 0-7 for spin 2j + 1) times 4 k-steps (one per mu: 8
// columns per hop = 3 colours + 1 zero pad, re/im).
//
// Lane (g, t) of a warp (g = lane / 4, t = lane % 4) owns colour t of RHS g: it
// loads exactly the 16-byte chunk (colour t, four spins) of each neighbour
// record (FP16 records are colour-major), forms its A fragments in registers,
// and receives colour t of all four output spins, which is again one chunk of
// the output record.  Lane t = 3 is the pad: zero A and B.
//
// The FP16 records carry per-(site, RHS) norms, which differ between the 8
// neighbours.  They are folded into the A rows relative to the largest of the
// 8 (w_d = n_d / max n, in (0, 1] times the factor 2 of mu = 3), so the FP16
// operand keeps its relative precision; the FP32 result is scaled by max n.
//
// A warp works through 8 consecutive sites; its 32 lanes first stage the 64
// links of those sites into shared memory (two each, FP16 pairs with the
// boundary phase folded in, conjugated for backward hops), then per site each
// lane picks its B element U[a = g / 2][b = t] of each hop.
//
// A per-(site, hop) 3x3 colour multiply fills few MMA rows; here the RHS and
// output spins of one site fill all 16 rows of every tile and the 8 hops fill
// K, so one link element per lane and hop serves 32 output rows.
//
// Measured at 24^3x48 with 16 RHS (two blocks per site along y): 0.60 ms per
// hop against 0.28 ms for the RHS-in-lanes kernel, with identical CG iteration
// counts.  The colour multiply leaves the FMA pipe, but every lane still does
// the projection, weights and epilogue for one colour of one RHS (lane t = 3
// idles), so the per-(site, RHS) instruction count stays close to the lanes
// kernel's while the per-site dependency chain (norms -> weights -> MMAs ->
// epilogue) leaves the kernel latency-bound.  It stays selectable and tested.
#pragma once
#include "wl_site.cuh"

namespace wl {

constexpr int kMmaWarps = 4;
#ifndef WL_MMA_SITES_PER_WARP
#define WL_MMA_SITES_PER_WARP 8
#endif
constexpr int kMmaSitesPerWarp = WL_MMA_SITES_PER_WARP;  // x 8 links staged by the 32 lanes
constexpr int kMmaSites = kMmaWarps * kMmaSitesPerWarp;
constexpr int kMmaRhs = 8;  // RHS per block: one per lane group

#ifndef WL_MMA_MIN_BLOCKS
#define WL_MMA_MIN_BLOCKS 3  // resident 128-thread blocks per SM the kernel is compiled for
#endif

struct MmaSmem {
  LinkSmemH link[kMmaSites][8];
  int nb[kMmaSites][8];
  int ok[kMmaSites];
};

// Epilogues with a per-colour form (SliceHalf records) can run behind this kernel.
template <class EPI> struct HasSlice : std::false_type {};
template <bool RED> struct HasSlice<EpiXpay<SpinorField<P_HALF>, RED>> : std::true_type {};
template <> struct HasSlice<EpiCG<SpinorField<P_HALF>>> : std::true_type {};

WL_D unsigned h2bits(__half2 h) { return *reinterpret_cast<unsigned*>(&h); }
WL_D __half2 hswap(__half2 h) { return __lowhigh2highlow(h); }

// D += A B for one m16n8k16 tile (row-major A, column-major B, FP16 in, FP32 accumulate)
WL_D void mma_16816(float (&d)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3, unsigned b0, unsigned b1) {
  asm(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// A-operand words of one hop for one colour: v = (spin 0..3) of the neighbour's
// colour chunk, w = (w, w); o[s] = h' for output spin s (see the file comment).
// Same projection (1 + C g_mu) and reconstruction as project2 / accum2.
template <int MU, int C>
WL_D void mma_rows(const uint4 v, const __half2 w, unsigned (&o)[4]) {
  const __half2 s0 = as_h2(v.x), s1 = as_h2(v.y), s2 = as_h2(v.z), s3 = as_h2(v.w);
  const __half2 pcm = __floats2half2_rn((float)C, -(float)C);  // -iC x = pcm * swap(x)
  const __half2 pmc = __floats2half2_rn(-(float)C, (float)C);  //  iC x = pmc * swap(x)
  __half2 h0, h1;
  if (MU == 0) {
    h0 = C > 0 ? __hadd2(s0, s3) : __hsub2(s0, s3);
    h1 = C > 0 ? __hadd2(s1, s2) : __hsub2(s1, s2);
  } else if (MU == 1) {
    h0 = __hfma2(pcm, hswap(s3), s0);  // s0 - iC s3
    h1 = __hfma2(pmc, hswap(s2), s1);  // s1 + iC s2
  } else if (MU == 2) {
    h0 = __hfma2(pcm, hswap(s2), s0);  // s0 - iC s2
    h1 = __hfma2(pcm, hswap(s3), s1);  // s1 - iC s3
  } else {
    h0 = C > 0 ? s0 : s2;
    h1 = C > 0 ? s1 : s3;
  }
  h0 = __hmul2(w, h0);
  h1 = __hmul2(w, h1);
  if (MU == 3) {
    const unsigned z = 0u;
    o[0] = C > 0 ? h2bits(h0) : z;
    o[1] = C > 0 ? h2bits(h1) : z;
    o[2] = C > 0 ? z : h2bits(h0);
    o[3] = C > 0 ? z : h2bits(h1);
    return;
  }
  o[0] = h2bits(h0);
  o[1] = h2bits(h1);
  if (MU == 0) {
    o[2] = C > 0 ? h2bits(h1) : h2bits(__hneg2(h1));  // C u1
    o[3] = C > 0 ? h2bits(h0) : h2bits(__hneg2(h0));  // C u0
  } else if (MU == 1) {
    o[2] = h2bits(__hmul2(pcm, hswap(h1)));  // -iC u1
    o[3] = h2bits(__hmul2(pmc, hswap(h0)));  //  iC u0
  } else {
    o[2] = h2bits(__hmul2(pmc, hswap(h0)));  //  iC u0
    o[3] = h2bits(__hmul2(pmc, hswap(h1)));  //  iC u1
  }
}

// What one lane reads for one site: colour t of the 8 neighbour records of its
// RHS (for mu = 3 only the two spins the projector keeps) and their norms.
struct MmaSiteIn {
  uint4 v[8];
  float n[8];
};

template <int Q, bool DAG>
WL_D uint4 mma_chunk(const SpinorField<P_HALF>& f, int rhs, unsigned nb, int t, bool on) {
  uint4 v = make_uint4(0u, 0u, 0u, 0u);
  if (!on) return v;
  if (Q < 6) return ldg(f.ptr + f.at(rhs, t, nb));
  // mu = 3: C > 0 keeps spins 0, 1 (first 8 bytes), C < 0 spins 2, 3 (last 8 bytes)
  constexpr int C = (Q == 6) == DAG ? +1 : -1;
  const uint2 h = __ldg(reinterpret_cast<const uint2*>(f.ptr + f.at(rhs, t, nb)) + (C > 0 ? 0 : 1));
  if (C > 0) {
    v.x = h.x;
    v.y = h.y;
  } else {
    v.z = h.x;
    v.w = h.y;
  }
  return v;
}

template <bool DAG>
WL_D void mma_load_site(const SpinorField<P_HALF>& src, const int* nbs, int r, int t, bool act, MmaSiteIn& in) {
  const bool on = act && t < 3;
#pragma unroll
  for (int q = 0; q < 8; ++q) in.n[q] = act ? ldg(src.norm + src.nat(r, (unsigned)nbs[q])) : 0.f;
  in.v[0] = mma_chunk<0, DAG>(src, r, (unsigned)nbs[0], t, on);
  in.v[1] = mma_chunk<1, DAG>(src, r, (unsigned)nbs[1], t, on);
  in.v[2] = mma_chunk<2, DAG>(src, r, (unsigned)nbs[2], t, on);
  in.v[3] = mma_chunk<3, DAG>(src, r, (unsigned)nbs[3], t, on);
  in.v[4] = mma_chunk<4, DAG>(src, r, (unsigned)nbs[4], t, on);
  in.v[5] = mma_chunk<5, DAG>(src, r, (unsigned)nbs[5], t, on);
  in.v[6] = mma_chunk<6, DAG>(src, r, (unsigned)nbs[6], t, on);
  in.v[7] = mma_chunk<7, DAG>(src, r, (unsigned)nbs[7], t, on);
}

// One k-step: hops q = 2 MU (forward, C = CF) and 2 MU + 1 (backward, C = CB).
// Tile j holds output spins 2j (rows 0-7 = RHS) and 2j + 1 (rows 8-15).
template <int MU, bool DAG>
WL_D void mma_step(const MmaSiteIn& in, const LinkSmemH* Ls, const float (&w)[8], int kf, int kb, bool bval,
                   unsigned sel, float (&d)[2][4]) {
  constexpr int CF = DAG ? +1 : -1;
  constexpr int CB = -CF;
  unsigned f[4], b[4];
  mma_rows<MU, CF>(in.v[2 * MU], __float2half2_rn(w[2 * MU]), f);
  mma_rows<MU, CB>(in.v[2 * MU + 1], __float2half2_rn(w[2 * MU + 1]), b);
  const uint2 xf = Ls[2 * MU].p[kf];
  const uint2 xb = Ls[2 * MU + 1].p[kb];
  const unsigned b0 = bval ? __byte_perm(xf.x, xf.y, sel) : 0u;
  const unsigned b1 = bval ? __byte_perm(xb.x, xb.y, sel) : 0u;
  mma_16816(d[0], f[0], f[1], b[0], b[1], b0, b1);
  mma_16816(d[1], f[2], f[3], b[2], b[3], b0, b1);
}

// The hop of one site for this lane's RHS: o = colour t of spins 0..3.
template <bool DAG>
WL_D void mma_site(const MmaSiteIn& in, const LinkSmemH* Ls, int kf, int kb, bool bval, unsigned sel,
                   float2 (&o)[4]) {
  float m = 0.f;
#pragma unroll
  for (int q = 0; q < 8; ++q) m = fmaxf(m, in.n[q]);
  const float im = m > 0.f ? 1.0f / m : 0.f;
  float w[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) w[q] = in.n[q] * (q >= 6 ? 2.0f * im : im);  // factor 2 of the mu = 3 projector
  float d[2][4];
#pragma unroll
  for (int j = 0; j < 2; ++j) d[j][0] = d[j][1] = d[j][2] = d[j][3] = 0.f;
  mma_step<0, DAG>(in, Ls, w, kf, kb, bval, sel, d);
  mma_step<1, DAG>(in, Ls, w, kf, kb, bval, sel, d);
  mma_step<2, DAG>(in, Ls, w, kf, kb, bval, sel, d);
  mma_step<3, DAG>(in, Ls, w, kf, kb, bval, sel, d);
  o[0] = f2(d[0][0] * m, d[0][1] * m);
  o[1] = f2(d[0][2] * m, d[0][3] * m);
  o[2] = f2(d[1][0] * m, d[1][1] * m);
  o[3] = f2(d[1][2] * m, d[1][3] * m);
}

// Block partials of the RHS each lane group holds (rbase + g): sums over the
// group's four lanes, then over the block's warps in a fixed order.
WL_D void reduce_mma(double v, const Reduce& Rd, int nrhs, int rbase) {
  __shared__ double sred[kMmaWarps][kMmaRhs];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  v += __shfl_xor_sync(0xffffffffu, v, 1);
  v += __shfl_xor_sync(0xffffffffu, v, 2);
  if ((lane & 3) == 0) sred[warp][lane >> 2] = v;
  __syncthreads();
  if (tid < kMmaRhs) {
    const double x = (sred[0][tid] + sred[1][tid]) + (sred[2][tid] + sred[3][tid]);
    const int nblk = gridDim.x * gridDim.z;
    const int blk = blockIdx.z * gridDim.x + blockIdx.x;
    const int rhs = rbase + tid;
    if (rhs < nrhs) Rd.partials[(long long)rhs * nblk + blk] = x;
  }
}

// Each warp walks kMmaSitesPerWarp consecutive sites for the block's 8 RHS.
// The neighbour data of site i + 1 and the epilogue inputs of site i are loaded
// before site i's contraction, so every lane keeps about one site of requests
// in flight while it computes (the loads are the latency the kernel hides).
template <bool DAG, class LF, class EPI>
__global__ void __launch_bounds__(kMmaWarps * 32, WL_MMA_MIN_BLOCKS) hop_mma_kernel(
    HopArgs<LF, SpinorField<P_HALF>, EPI> A) {
  static_assert(kMmaWarps == 4, "reduce_mma adds four warps");
  __shared__ MmaSmem sm;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int parity = A.parity0 ^ blockIdx.z;
  const int rbase = blockIdx.y * kMmaRhs;
  const int wsite = warp * kMmaSitesPerWarp;
  const int site0 = blockIdx.x * kMmaSites + wsite;
  // ---- the warp's sites x 8 links, staged by its lanes
#pragma unroll
  for (int j = lane; j < 8 * kMmaSitesPerWarp; j += 32) {
    const int sl = j >> 3, q = j & 7;
    const int c = site0 + sl;
    if (c < A.g.Vh) {
      sm.nb[wsite + sl][q] = stage_link<true>(A.g, A.links, parity, c, q >> 1, q & 1, sm.link[wsite + sl][q]);
      if (q == 0) sm.ok[wsite + sl] = 1;
    } else if (q == 0) {
      sm.ok[wsite + sl] = 0;
    }
  }
  __syncwarp();
  const int r = rbase + g;
  const bool act = r < A.nrhs && (A.mask == nullptr || A.mask[r] != 0);
  const int ca = g >> 1;  // output colour of this lane's B column (3: pad)
  const bool bval = ca < 3 && t < 3;
  const unsigned sel = (g & 1) ? 0x3276u : 0x5410u;  // im column: (y.hi, x.hi); re column: (x.lo, y.lo)
  const int kf = bval ? ca * 3 + t : 0, kb = bval ? t * 3 + ca : 0;  // U[a][b]; U^dag[a][b] = conj U[b][a]
  const SpinorField<P_HALF>& src = A.src[1 - parity];
  double red = 0.0;
  MmaSiteIn cur;
  if (sm.ok[wsite]) mma_load_site<DAG>(src, sm.nb[wsite], r, t, act, cur);
#pragma unroll
  for (int i = 0; i < kMmaSitesPerWarp; ++i) {
    const int sl = wsite + i;
    if (!sm.ok[sl]) break;  // warp-uniform; the warp's later sites are out of range too
    const unsigned c = (unsigned)(site0 + i);
    MmaSiteIn nxt;
    if (i + 1 < kMmaSitesPerWarp && sm.ok[sl + 1]) mma_load_site<DAG>(src, sm.nb[sl + 1], r, t, act, nxt);
    const typename EPI::SliceIn e = A.epi.slice_in(r, parity, c, t, act && t < 3);
    float2 o[4];
    mma_site<DAG>(cur, sm.link[sl], kf, kb, bval, sel, o);
    red += A.epi.slice_out(e, r, parity, c, t, act, o);
    if (i + 1 < kMmaSitesPerWarp) cur = nxt;
  }
  if (EPI::kReduce) reduce_mma(red, A.red, A.nrhs, rbase);
}

}  // namespace wl
