// FP64 Wilson hop on reference-layout fermions with the neighbour spinors
// staged in shared memory by TMA, one warp per tile of 16 consecutive sites of
// a t-row (lattices with Lt a multiple of 16, all sites targeted: D, D^dag, K).
//
// Why: read straight from the caller's AoS field (ref_pair_kernel), every load
// instruction of a warp touches one or two 32-byte sectors of each of its 16
// sites, and the L1 data pipe -- about one wavefront per sector -- saturates at a
// third of the DRAM bandwidth.  A tile's neighbours along x, y or z are another
// 16 consecutive sites (3 KB), so one 2D tensor-map copy (cp.async.bulk.tensor,
// 128-byte swizzle) brings each of them into shared memory without the load/store
// unit, and the pair threads then read their spins with conflict-light 16-byte
// shared loads.  Links stay in the parity-split SoA copy and are read with
// ordinary loads (two contiguous runs per warp request).
//
// Per warp four stages per tile, double-buffered across stages and tiles:
// stage 0 = the tile itself (the t hops; the two t-neighbours outside the
// tile are read from global memory), stages 1..3 = the tiles at x -/+ mu_hat for
// mu = 0, 1, 2.  Every warp owns its buffers and mbarriers, so warps never wait
// for each other; each wait is bounded, and a wait that runs out sets the
// context's error flag (wl_ctx_synchronize reports WL_ERR_TIMEOUT), lets the
// copies already issued land (bounded too) and ends the warp.
//
// Contract = ref_pair_kernel with parity = -1.
#pragma once
#include "wl_refsite.cuh"
#include "wl_rowhop.cuh"  // mbarrier / TMA helpers and the 128-byte swizzle address

namespace wl {

constexpr int kTileSites = 16;                                // sites per warp tile
constexpr int kTileWarps = 4;                                 // warps per block
constexpr unsigned kTileBox = 16u * 192u;                     // one tile of spinors (24 lines of 128 B)
constexpr int kTileBufs = 2;                                  // stage buffers per warp
constexpr size_t kTileWarpBytes = (size_t)kTileBufs * 2 * kTileBox;  // 12 KB: two tiles per stage
constexpr int kTileStages = 4;
constexpr long long kTileWaitLimit = 1LL << 24;

WL_HD size_t tile_smem_bytes() { return 128 + 1024 + (size_t)kTileWarps * kTileWarpBytes; }

struct TileStage {
  int rhs, row, t0, q;
};

WL_D TileStage tile_stage(const Geom& g, int tiles_per_rhs, long long wid, long long nw, int k) {
  TileStage s;
  const long long tile = wid + (long long)(k / kTileStages) * nw;
  s.q = k % kTileStages;
  s.rhs = (int)(tile / tiles_per_rhs);
  const int rem = (int)(tile - (long long)s.rhs * tiles_per_rhs);
  const int tpr = g.L[3] / kTileSites;  // tiles per t-row
  s.row = rem / tpr;
  s.t0 = (rem - s.row * tpr) * kTileSites;
  return s;
}

// first 128-byte line of the tile (rhs, row, t0) in the field viewed as lines (1.5 lines per site)
WL_D int tile_line(const Geom& g, int rhs, int row, int t0) {
  return (int)((((long long)rhs * g.V + (long long)row * g.L[3] + t0) * 3) >> 1);
}

WL_D void tile_issue(const Geom& g, const CUtensorMap* map, const TileStage& st, unsigned char* buf,
                     unsigned long long* bar) {
  if (st.q == 0) {
    mbar_expect_tx(bar, kTileBox);
    tma_g2s_2d(buf, map, 0, tile_line(g, st.rhs, st.row, st.t0), bar);
    return;
  }
  const int mu = st.q - 1;
  const int stride = g.strideRow[mu], Lm = g.L[mu];
  const int xm = (st.row / stride) % Lm;
  const int rp = st.row + (xm == Lm - 1 ? -(Lm - 1) * stride : stride);
  const int rm = st.row + (xm == 0 ? (Lm - 1) * stride : -stride);
  mbar_expect_tx(bar, 2 * kTileBox);
  tma_g2s_2d(buf, map, 0, tile_line(g, st.rhs, rp, st.t0), bar);
  tma_g2s_2d(buf + kTileBox, map, 0, tile_line(g, st.rhs, rm, st.t0), bar);
}

// spin s (6 reals) of site i of a swizzled tile in shared memory
WL_D void ld_spin_tile(const unsigned char* tile, int i, int s, double (&v)[6]) {
#pragma unroll
  for (int col = 0; col < 3; ++col) {
    const double2 q = *swz_psi(tile, i, s * 3 + col);
    v[2 * col] = q.x;
    v[2 * col + 1] = q.y;
  }
}

// one hop of thread j for site s: spins from `tile` (site ti) or, with tile == nullptr,
// from the global site `gsite`
template <int MU, int C, bool DAGU>
WL_D void tile_hop(const RefSiteArgs& A, const unsigned char* tile, int ti, const double* gsite, int lp, int lc,
                   bool ph, int j, double sg, cplx<double> (&Ac)[3], cplx<double> (&Xc)[3], cplx<double> (&Yc)[3]) {
  double a[6], b[6];
  if (tile) {
    ld_spin_tile(tile, ti, pair_spin1<MU, C>(j), a);
    if (MU < 3) ld_spin_tile(tile, ti, pair_spin2<MU>(j), b);
  } else {
    ld_spin<4>(gsite, pair_spin1<MU, C>(j), a);
    if (MU < 3) ld_spin<4>(gsite, pair_spin2<MU>(j), b);
  }
  Link<double> u;
  ld_link(A.U, (unsigned)A.g.Vh, lp, MU, lc, u);
  cplx<double> h[3];
  pair_combine<MU, C>(a, b, sg, h);
  pair_hop<MU, C, DAGU>(u, h, ph, A.g, sg, Ac, Xc, Yc);
}

// the hops of direction MU for site s (tile index i); stage buffer `buf`
template <int MU, bool DAG>
WL_D void tile_stage_compute(const RefSiteArgs& A, const unsigned char* buf, const Site& s, int parity, int i,
                             const TileStage& st, int j, double sg, cplx<double> (&Ac)[3], cplx<double> (&Xc)[3],
                             cplx<double> (&Yc)[3]) {
  constexpr int CF = DAG ? +1 : -1;
  constexpr int CB = -CF;
  const Geom& g = A.g;
  const int nbm = neighbor(g, s, MU, -1);
  if (MU == 3) {
    const double* field = A.in + (size_t)st.rhs * g.V * 24;
    const int Lt = g.L[3];
    // t + 1 and t - 1 inside the tile come from shared memory, the two outside it from global memory
    const int tp = s.x[3] == Lt - 1 ? 0 : s.x[3] + 1, tm = s.x[3] == 0 ? Lt - 1 : s.x[3] - 1;
    const bool pin = i < kTileSites - 1, min = i > 0;
    tile_hop<3, CF, false>(A, pin ? buf : nullptr, i + 1, field + ((size_t)s.row * Lt + tp) * 24, parity, s.c,
                           g.ph_on[3] && s.x[3] == Lt - 1, j, sg, Ac, Xc, Yc);
    tile_hop<3, CB, true>(A, min ? buf : nullptr, i - 1, field + ((size_t)s.row * Lt + tm) * 24, 1 - parity, nbm,
                          g.ph_on[3] && s.x[3] == 0, j, sg, Ac, Xc, Yc);
  } else {
    tile_hop<MU, CF, false>(A, buf, i, nullptr, parity, s.c, g.ph_on[MU] && s.x[MU] == g.L[MU] - 1, j, sg, Ac, Xc,
                            Yc);
    tile_hop<MU, CB, true>(A, buf + kTileBox, i, nullptr, 1 - parity, nbm, g.ph_on[MU] && s.x[MU] == 0, j, sg, Ac,
                           Xc, Yc);
  }
}

// all lanes wait (bounded) on the stage's mbarrier and agree on the outcome
WL_D bool tile_wait(unsigned long long* bar, unsigned parity) {
  bool ok = false;
  for (long long n = 0; n < kTileWaitLimit && !ok; ++n) ok = mbar_try_wait(bar, parity);
  return __all_sync(0xffffffffu, ok) != 0;
}

#ifndef WL_REFTILE_MINB
#define WL_REFTILE_MINB 4  // resident blocks per SM the tile kernel is compiled for (128 registers)
#endif

template <bool DAG>
__global__ void __launch_bounds__(32 * kTileWarps, WL_REFTILE_MINB)
    ref_tile_kernel(const __grid_constant__ CUtensorMap psimap, RefSiteArgs A, int* err) {
  extern __shared__ __align__(128) unsigned char smem[];
  const Geom& g = A.g;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = lane >> 1, j = lane & 1;
  const double sg = 1.0 - 2.0 * j;
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem) + warp * kTileBufs;
  // stage buffers from the first 1024-byte boundary past the barriers (swizzle atom)
  unsigned char* base = smem + 128u + ((1024u - ((smem_u32(smem) + 128u) & 1023u)) & 1023u);
  unsigned char* wbuf = base + (size_t)warp * kTileWarpBytes;
  const int tiles_per_rhs = g.V / kTileSites;
  const long long ntiles = (long long)tiles_per_rhs * A.nrhs;
  const long long wid = (long long)blockIdx.x * kTileWarps + warp, nw = (long long)gridDim.x * kTileWarps;
  const int my_tiles = wid < ntiles ? (int)((ntiles - 1 - wid) / nw + 1) : 0;
  const int nst = kTileStages * my_tiles;
  if (lane == 0) {
#pragma unroll
    for (int b = 0; b < kTileBufs; ++b) mbar_init(&bars[b], 1);
    mbar_fence_init();
  }
  __syncwarp();
  if (lane == 0)
    for (int k = 0; k < kTileBufs && k < nst; ++k)
      tile_issue(g, &psimap, tile_stage(g, tiles_per_rhs, wid, nw, k), wbuf + (size_t)k * 2 * kTileBox, &bars[k]);
  cplx<double> Ac[3], Xc[3], Yc[3];
  Site s{};
  int parity = 0;
  for (int k = 0; k < nst; ++k) {
    const TileStage st = tile_stage(g, tiles_per_rhs, wid, nw, k);
    const int slot = k % kTileBufs;
    const unsigned char* buf = wbuf + (size_t)slot * 2 * kTileBox;
    if (!tile_wait(&bars[slot], (unsigned)((k / kTileBufs) & 1))) {
      // record the lost wait, let the copies already issued land (bounded), and stop
      if (lane == 0) {
        atomicExch(err, 1);
        for (int m = k; m < k + kTileBufs && m < nst; ++m)
          for (long long n = 0; n < kTileWaitLimit; ++n)
            if (mbar_try_wait(&bars[m % kTileBufs], (unsigned)((m / kTileBufs) & 1))) break;
      }
      __syncwarp();
      return;
    }
    if (st.q == 0) {
#pragma unroll
      for (int a = 0; a < 3; ++a) Ac[a] = Xc[a] = Yc[a] = {0.0, 0.0};
      s = site_of_flat(g, st.row * g.L[3] + st.t0 + i);
      parity = (s.x[0] + s.x[1] + s.x[2] + s.x[3]) & 1;
    }
    switch (st.q) {
      case 0: tile_stage_compute<3, DAG>(A, buf, s, parity, i, st, j, sg, Ac, Xc, Yc); break;
      case 1: tile_stage_compute<0, DAG>(A, buf, s, parity, i, st, j, sg, Ac, Xc, Yc); break;
      case 2: tile_stage_compute<1, DAG>(A, buf, s, parity, i, st, j, sg, Ac, Xc, Yc); break;
      default: tile_stage_compute<2, DAG>(A, buf, s, parity, i, st, j, sg, Ac, Xc, Yc); break;
    }
    if (st.q == kTileStages - 1) {
      const size_t flat = (size_t)s.row * g.L[3] + s.x[3];
      pair_store<4>(A, (size_t)st.rhs * g.V * 24 + flat * 24 + 12 * j, true, j, Ac, Xc, Yc);
    }
    // the buffer is free once every lane has read it; then refill it
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0 && k + kTileBufs < nst)
      tile_issue(g, &psimap, tile_stage(g, tiles_per_rhs, wid, nw, k + kTileBufs), wbuf + (size_t)slot * 2 * kTileBox,
                 &bars[slot]);
  }
}

}  // namespace wl
