// Wilson hop on the tensor cores for FP16 fields, 16 RHS per warp.
//
// For one target site x and one mu, the forward and backward hops of 16 RHS
// are four real contractions (m16n8k16, FP16 inputs, FP32 accumulation):
//     D_s[r, (a, ri)] += sum_k A_j[r, k] B[k, (a, ri)]
// Rows r are the 16 RHS.  K holds the weighted, spin-projected neighbours:
// k = 0..5 the forward hop's projected row j (colour b, re/im), k = 8..13 the
// backward hop's, k = 6, 7, 14, 15 zero; A_0 is row 0 of the rank-2
// projection (1 + C g_mu) psi, A_1 row 1.  B is the realified link pair,
// forward U_mu(x) over backward U_mu(x - mu)^dag, with columns (a, re/im) of
// the output colour (6, 7 zero).  The four output spins are four accumulator
// tiles: spins 0, 1 take A_0, A_1 times B_up = [U ; U'^dag]; the lower spins
// are +-1 / +-i times a projected row, and that coefficient kappa is folded
// into B_lo = [kappa U ; -kappa U'^dag] (the backward hop has the opposite
// C), so the reconstruction costs no arithmetic and the accumulators of all
// four mu chain through one set of 16 FP32 registers per lane.
//
// Lane (g, t) (g = lane / 4, t = lane % 4) holds RHS g and g + 8 of colour t:
// its A words are the projections of colour chunk t of those two RHS'
// neighbour records (FP16 records are colour-major, so that is one 16-byte
// chunk each), its accumulators are colour t of all four spins of the same
// two RHS -- again one chunk of each output record.  Lanes t = 3 are the
// zero pad of K and of the output columns.
//
// The FP16 records carry per-(site, RHS) norms that differ between the eight
// neighbours; they are folded into the A rows relative to the largest of the
// eight for that RHS (w = n / max n, times the factor 2 of mu = 3), so the
// FP16 operand keeps its relative precision, and the FP32 result is scaled by
// max n.
//
// Data movement: each warp walks 8 consecutive sites.  The 8 links of its
// sites are staged once (12-real FP16 -> complex half2 with the boundary
// phase folded in) and every lane builds its B words from them with sign and
// swap bit operations.  The neighbour records of site i + 1 (8 hops x 3
// colours x 16 RHS x 16 bytes, plus 128 norms) are fetched with cp.async into
// the warp's second shared-memory slot while site i is contracted, so the
// loads are in flight for a whole site of work without holding registers.
// Chunks are stored at RHS index r ^ 2t, which makes the lanes' 16-byte
// shared reads conflict-free.
#pragma once
#include "wl_site.cuh"

namespace wl {

constexpr int kMmaWarps = 4;
constexpr int kMmaSitesPerWarp = 8;
constexpr int kMmaSites = kMmaWarps * kMmaSitesPerWarp;
constexpr int kMmaRhs = 16;  // RHS per block: rows of every tile

#ifndef WL_MMA_MIN_BLOCKS
#define WL_MMA_MIN_BLOCKS 3  // resident 128-thread blocks per SM the kernel is compiled for
#endif

struct MmaSlot {
  uint4 chunk[8][3][16];  // [hop q][colour t][RHS r ^ 2t]: spins 0..3 as half2
  float norm[16][8];      // [RHS r][hop q]
};

struct MmaWarpSmem {
  MmaSlot slot[2];
  unsigned lk[kMmaSitesPerWarp][8][9];  // link of hop q, element a*3+b, half2 (re, im), phase folded
  int nb[kMmaSitesPerWarp][8];
  int ok[kMmaSitesPerWarp];
};

struct MmaSmem {
  MmaWarpSmem w[kMmaWarps];
  double sred[kMmaWarps][kMmaRhs];
};

// Epilogues with a per-colour form (SliceHalf records) can run behind this kernel.
template <class EPI> struct HasSlice : std::false_type {};
template <bool RED> struct HasSlice<EpiXpay<SpinorField<P_HALF>, RED>> : std::true_type {};
template <> struct HasSlice<EpiCG<SpinorField<P_HALF>>> : std::true_type {};

WL_D unsigned h2bits(__half2 h) { return *reinterpret_cast<unsigned*>(&h); }
WL_D __half2 bits2h(unsigned u) { return *reinterpret_cast<__half2*>(&u); }
WL_D unsigned hswapw(unsigned u) { return __byte_perm(u, 0u, 0x1032); }  // (lo, hi) -> (hi, lo)

// D += A B for one m16n8k16 tile (row-major A, column-major B, FP16 in, FP32 accumulate)
WL_D void mma_16816(float (&d)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3, unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// 16-byte records bypass L1 (.cg): most of the SM's L1/shared storage is the record slots,
// and the streamed records are reused through L2, not L1
WL_D void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? 16 : 0;  // 0: the destination is zero-filled and nothing is read
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
WL_D void cp_async4(void* smem, const void* gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? 4 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
WL_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
WL_D void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Complex half2 word E = (re, im) times kappa in {+1, -1, +i, -i} (K = 0, 1, 2, 3): sign and swap bits.
template <int K>
WL_D unsigned cmul_unit(unsigned e) {
  if (K == 0) return e;
  if (K == 1) return e ^ 0x80008000u;              // -E
  if (K == 2) return hswapw(e) ^ 0x00008000u;      // iE = (-im, re)
  return hswapw(e) ^ 0x80000000u;                  // -iE = (im, -re)
}
// The B word of lane (g, t) for complex link element E: column (a, re) holds (E.re, -E.im) over
// rows (t, re), (t, im); column (a, im) holds (E.im, E.re).
WL_D unsigned bword(unsigned e, bool im_col) { return im_col ? hswapw(e) : (e ^ 0x80000000u); }
WL_D unsigned conjw(unsigned e) { return e ^ 0x80000000u; }

// kappa of the lower spins for mu < 3 (0: +1, 1: -1, 2: +i, 3: -i) given the forward C:
// mu = 0: C, mu = 1: -iC, mu = 2: iC (the lower spin rows of accum2).
template <int MU, int C>
struct LowerKappa {
  static constexpr int value = MU == 0 ? (C > 0 ? 0 : 1) : MU == 1 ? (C > 0 ? 3 : 2) : (C > 0 ? 2 : 3);
};

// rows 0, 1 of (1 + C g_mu) psi for one colour (v = spins 0..3 as half2), times w
template <int MU, int C>
WL_D void mma_project(const uint4 v, const __half2 w, unsigned& r0, unsigned& r1) {
  const __half2 s0 = bits2h(v.x), s1 = bits2h(v.y), s2 = bits2h(v.z), s3 = bits2h(v.w);
  const __half2 pcm = __floats2half2_rn((float)C, -(float)C);  // -iC x = pcm * swap(x)
  const __half2 pmc = __floats2half2_rn(-(float)C, (float)C);  //  iC x = pmc * swap(x)
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
  r0 = h2bits(__hmul2(w, h0));
  r1 = h2bits(__hmul2(w, h1));
}

// Stage the link of hop q = 2 mu + dir of compact site c as complex half2 words with the
// boundary phase folded in (the backward hop stores U(x - mu) itself; lanes take its dagger);
// returns the compact index of the neighbour.
template <class LF>
WL_D int stage_link_cplx(const Geom& g, const LF& links, int parity, int c, int mu, int dir, unsigned (&dst)[9]) {
  const Site s = site_from_compact(g, parity, c);
  const int nb = neighbor(g, s, mu, dir == 0 ? +1 : -1);
  Link<float> u;
  if (dir == 0) links.load(u, parity, mu, c);
  else links.load(u, 1 - parity, mu, nb);
  const bool ph = g.ph_on[mu] && (dir == 0 ? (s.x[mu] == g.L[mu] - 1) : (s.x[mu] == 0));
  if (ph) {
    const cplx<float> w{(float)g.ph_re[mu], (float)g.ph_im[mu]};
#pragma unroll
    for (int k = 0; k < 9; ++k) u.m[k / 3][k % 3] = u.m[k / 3][k % 3] * w;
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) dst[k] = f2h(u.m[k / 3][k % 3].re, u.m[k / 3][k % 3].im);
  return nb;
}

// cp.async of one site's neighbour records for RHS rbase..rbase+15 into a slot.  Lane L copies
// RHS r = L % 16 of hops 4h..4h+3 (h = L / 16): colour chunks m = 0..11 (hop 4h + m / 3, colour
// m % 3; the 16 lanes of a half copy one contiguous 256-byte run of a record chunk) and the
// four norms.  RHS outside `valid` (a bit per RHS) are zero-filled.
WL_D void mma_fetch(const SpinorField<P_HALF>& f, const int* nbq, int rbase, unsigned valid, MmaSlot& S, int lane) {
  const int r = lane & 15, h = lane >> 4;
  const bool v = (valid >> r) & 1u;
  const unsigned rofs = f.at(rbase + r, 0, 0u), nofs = f.nat(rbase + r, 0u);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int q = 4 * h + k;
    const unsigned nb = (unsigned)nbq[q];
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      const uint4* src = v ? f.ptr + (rofs + (unsigned)t * f.kstride + nb * f.cstride) : f.ptr;
      cp_async16(&S.chunk[q][t][r ^ (2 * t)], src, v);
    }
    cp_async4(&S.norm[r][q], v ? f.norm + (nofs + nb * f.ncstride) : f.norm, v);
  }
}

// One mu: four tiles (output spins 0..3) for hops q = 2 mu (forward, C = CF) and 2 mu + 1.
template <int MU, bool DAG>
WL_D void mma_mu(const MmaSlot& S, const unsigned (&lk)[8][9], int g, int t, const __half2 (&w0)[8],
                 const __half2 (&w1)[8], float (&d)[4][4]) {
  constexpr int CF = DAG ? +1 : -1;
  constexpr int CB = -CF;
  constexpr int qf = 2 * MU, qb = 2 * MU + 1;
  // A words: rows g (RHS g) and g + 8, forward then backward hop
  unsigned f0a = 0, f0b = 0, f1a = 0, f1b = 0, b0a = 0, b0b = 0, b1a = 0, b1b = 0;
  if (t < 3) {
    const int ra = g ^ (2 * t), rb = ra + 8;
    mma_project<MU, CF>(S.chunk[qf][t][ra], w0[qf], f0a, f1a);
    mma_project<MU, CF>(S.chunk[qf][t][rb], w1[qf], f0b, f1b);
    mma_project<MU, CB>(S.chunk[qb][t][ra], w0[qb], b0a, b1a);
    mma_project<MU, CB>(S.chunk[qb][t][rb], w1[qb], b0b, b1b);
  }
  // B words: column g = (output colour a, re/im), rows (colour t, re/im) of each hop
  const int a = g >> 1;
  const bool imc = g & 1;
  unsigned uf = 0u, vb = 0u;
  if (a < 3 && t < 3) {
    uf = lk[qf][a * 3 + t];          // U(x)[a][t]
    vb = conjw(lk[qb][t * 3 + a]);   // U(x - mu)^dag [a][t] = conj U(x - mu)[t][a]
  }
  unsigned up0, up1, lo0, lo1;
  if (MU < 3) {
    constexpr int K = LowerKappa<MU, CF>::value;
    up0 = bword(uf, imc);
    up1 = bword(vb, imc);
    lo0 = bword(cmul_unit<K>(uf), imc);
    lo1 = bword(cmul_unit<K ^ 1>(vb), imc);  // -kappa for the backward hop
  } else {  // mu = 3: upper spins from the C > 0 hop, lower from the C < 0 hop
    const unsigned wf = bword(uf, imc), wb = bword(vb, imc);
    up0 = CF > 0 ? wf : 0u;
    up1 = CB > 0 ? wb : 0u;
    lo0 = CF < 0 ? wf : 0u;
    lo1 = CB < 0 ? wb : 0u;
  }
  mma_16816(d[0], f0a, f0b, b0a, b0b, up0, up1);
  mma_16816(d[1], f1a, f1b, b1a, b1b, up0, up1);
  if (MU == 0) {         // spin 2 <- C row 1, spin 3 <- C row 0
    mma_16816(d[2], f1a, f1b, b1a, b1b, lo0, lo1);
    mma_16816(d[3], f0a, f0b, b0a, b0b, lo0, lo1);
  } else if (MU == 1) {  // spin 2 <- -iC row 1, spin 3 <- iC row 0
    mma_16816(d[2], f1a, f1b, b1a, b1b, lo0, lo1);
    mma_16816(d[3], f0a, f0b, b0a, b0b, lo0 ^ 0x80008000u, lo1 ^ 0x80008000u);
  } else {               // mu = 2: spin 2 <- iC row 0, spin 3 <- iC row 1; mu = 3: rows 0, 1
    mma_16816(d[2], f0a, f0b, b0a, b0b, lo0, lo1);
    mma_16816(d[3], f1a, f1b, b1a, b1b, lo0, lo1);
  }
}

// Block partials of the RHS each lane holds (rbase + g, rbase + g + 8): sums over the group's
// four lanes, then over the block's warps in a fixed order.
WL_D void reduce_mma(double v0, double v1, const Reduce& Rd, int nrhs, int rbase, double (&sred)[kMmaWarps][kMmaRhs]) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  v0 += __shfl_xor_sync(0xffffffffu, v0, 1);
  v0 += __shfl_xor_sync(0xffffffffu, v0, 2);
  v1 += __shfl_xor_sync(0xffffffffu, v1, 1);
  v1 += __shfl_xor_sync(0xffffffffu, v1, 2);
  if ((lane & 3) == 0) {
    sred[warp][lane >> 2] = v0;
    sred[warp][(lane >> 2) + 8] = v1;
  }
  __syncthreads();
  if (tid < kMmaRhs) {
    const double x = (sred[0][tid] + sred[1][tid]) + (sred[2][tid] + sred[3][tid]);
    const int nblk = gridDim.x * gridDim.z;
    const int blk = blockIdx.z * gridDim.x + blockIdx.x;
    const int rhs = rbase + tid;
    if (rhs < nrhs) Rd.partials[(long long)rhs * nblk + blk] = x;
  }
}

constexpr size_t kMmaSmemBytes = sizeof(MmaSmem);

// Each warp walks kMmaSitesPerWarp consecutive sites for the block's 16 RHS; the records of
// site i + 1 are in flight (cp.async) while site i is contracted.
template <bool DAG, class LF, class EPI>
__global__ void __launch_bounds__(kMmaWarps * 32, WL_MMA_MIN_BLOCKS) hop_mma_kernel(
    HopArgs<LF, SpinorField<P_HALF>, EPI> A) {
  static_assert(kMmaWarps == 4, "reduce_mma adds four warps");
  extern __shared__ __align__(16) unsigned char mma_dyn[];
  MmaSmem& sm = *reinterpret_cast<MmaSmem*>(mma_dyn);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  MmaWarpSmem& W = sm.w[warp];
  const int parity = A.parity0 ^ blockIdx.z;
  const int rbase = blockIdx.y * kMmaRhs;
  const int site0 = blockIdx.x * kMmaSites + warp * kMmaSitesPerWarp;
  // RHS validity bits (active and unmasked) of the block's 16 RHS
  const int rl = rbase + (lane & 15);
  const bool rv = rl < A.nrhs && (A.mask == nullptr || A.mask[rl] != 0);
  const unsigned valid = __ballot_sync(0xffffffffu, rv && lane < 16) & 0xffffu;
  // ---- links and neighbour indices of the warp's sites
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    const int j = lane + 32 * m;
    const int i = j >> 3, q = j & 7;
    const int c = site0 + i;
    if (c < A.g.Vh) {
      W.nb[i][q] = stage_link_cplx(A.g, A.links, parity, c, q >> 1, q & 1, W.lk[i][q]);
      if (q == 0) W.ok[i] = 1;
    } else if (q == 0) {
      W.ok[i] = 0;
    }
  }
  __syncwarp();
  const SpinorField<P_HALF>& src = A.src[1 - parity];
  const int r0 = rbase + g, r1 = rbase + g + 8;
  const bool act0 = (valid >> g) & 1u, act1 = (valid >> (g + 8)) & 1u;
  double red0 = 0.0, red1 = 0.0;
  if (W.ok[0]) mma_fetch(src, W.nb[0], rbase, valid, W.slot[0], lane);
  cp_async_commit();
#pragma unroll 1
  for (int i = 0; i < kMmaSitesPerWarp; ++i) {
    if (!W.ok[i]) break;  // warp-uniform; the warp's later sites are out of range too
    const unsigned c = (unsigned)(site0 + i);
    if (i + 1 < kMmaSitesPerWarp && W.ok[i + 1]) mma_fetch(src, W.nb[i + 1], rbase, valid, W.slot[(i + 1) & 1], lane);
    cp_async_commit();
    const typename EPI::SliceIn e0 = A.epi.slice_in(r0, parity, c, t, act0 && t < 3);
    const typename EPI::SliceIn e1 = A.epi.slice_in(r1, parity, c, t, act1 && t < 3);
    cp_async_wait1();  // this lane's copies of site i have landed
    __syncwarp();      // and every other lane's
    const MmaSlot& S = W.slot[i & 1];
    // relative weights per RHS: w = n / max n over the eight hops (times 2 for mu = 3)
    float n0[8], n1[8], m0 = 0.f, m1 = 0.f;
    {
      const float4* p0 = reinterpret_cast<const float4*>(S.norm[g]);
      const float4* p1 = reinterpret_cast<const float4*>(S.norm[g + 8]);
      const float4 a0 = p0[0], a1 = p0[1], c0 = p1[0], c1 = p1[1];
      n0[0] = a0.x, n0[1] = a0.y, n0[2] = a0.z, n0[3] = a0.w, n0[4] = a1.x, n0[5] = a1.y, n0[6] = a1.z, n0[7] = a1.w;
      n1[0] = c0.x, n1[1] = c0.y, n1[2] = c0.z, n1[3] = c0.w, n1[4] = c1.x, n1[5] = c1.y, n1[6] = c1.z, n1[7] = c1.w;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      m0 = fmaxf(m0, n0[q]);
      m1 = fmaxf(m1, n1[q]);
    }
    const float i0 = m0 > 0.f ? 1.0f / m0 : 0.f, i1 = m1 > 0.f ? 1.0f / m1 : 0.f;
    __half2 w0[8], w1[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      w0[q] = __float2half2_rn(n0[q] * (q >= 6 ? 2.0f * i0 : i0));
      w1[q] = __float2half2_rn(n1[q] * (q >= 6 ? 2.0f * i1 : i1));
    }
    float d[4][4];
#pragma unroll
    for (int s = 0; s < 4; ++s) d[s][0] = d[s][1] = d[s][2] = d[s][3] = 0.f;
    mma_mu<0, DAG>(S, W.lk[i], g, t, w0, w1, d);
    mma_mu<1, DAG>(S, W.lk[i], g, t, w0, w1, d);
    mma_mu<2, DAG>(S, W.lk[i], g, t, w0, w1, d);
    mma_mu<3, DAG>(S, W.lk[i], g, t, w0, w1, d);
    __syncwarp();  // every lane is done with slot i & 1 before it is refilled
    float2 o0[4], o1[4];  // colour t of spins 0..3 for RHS g and g + 8
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      o0[s] = f2(d[s][0] * m0, d[s][1] * m0);
      o1[s] = f2(d[s][2] * m1, d[s][3] * m1);
    }
    red0 += A.epi.slice_out(e0, r0, parity, c, t, act0, o0);
    red1 += A.epi.slice_out(e1, r1, parity, c, t, act1, o1);
  }
  if (EPI::kReduce) reduce_mma(red0, red1, A.red, A.nrhs, rbase, sm.sred);
}

}  // namespace wl
