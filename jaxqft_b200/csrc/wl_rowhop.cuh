// FP64 Wilson hop on the reference layout, staged through shared memory by
// 1D TMA bulk copies (cp.async.bulk + mbarrier), for the drop-in operators
// (D, D^dag and the masked / Schur forms built from them).
//
// Layout (reference): fermions [rhs][Lx][Ly][Lz][Lt][4][3] complex128, links
// [mu][Lx][Ly][Lz][Lt][3][3] complex128.  A "row" is the Lt consecutive sites of
// one (x, y, z): the x/y/z neighbours of a row are whole rows, and its t
// neighbours are in the row itself.  So for one row every direction's operands
// are contiguous chunks.  Four stages per row, one per mu, each holding both
// hops of that direction: mu=3 = {own row of psi, own row of U_3}; mu<3 = {rows
// x+mu and x-mu of psi, own row of U_mu, row x-mu of U_mu} (<= 672*Lt bytes).  A
// persistent block walks work items (rhs, row) through the stages with a ring of
// kRowBufs buffers: while it computes stage k, the bulk copies of the next
// kRowBufs-1 stages are in flight.  (Seven single-hop stages per row were
// measured slower: the per-stage barrier then dominates.)  Thread 3*t + a owns output colour a of site t and
// accumulates its four spin components; a site's three threads read the same
// neighbour spinor (shared-memory broadcast).
//
// Contract = hop_kernel with IdxFlat: out = a*self + b*acc on the target
// parities in pmask, acc = sum_mu [(1 + cf g_mu) U psi(x+mu) + (1 + cb g_mu) U^dag psi(x-mu)],
// boundary phase on the forward hop from x_mu = L_mu - 1 and (conjugated) on the
// backward hop into x_mu = 0.  Waits on the mbarriers are bounded; on time-out
// the block records an error flag and stops.
#pragma once
#include <cuda.h>  // CUtensorMap (the map itself is encoded on the host through the driver entry point)

#include "wl_hop.cuh"

namespace wl {

WL_D unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

WL_D void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
WL_D void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
WL_D void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
WL_D bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// global -> shared bulk copy into this CTA's own shared memory, completing on `bar`
WL_D void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  unsigned long long gsrc;
  asm volatile("cvta.to.global.u64 %0, %1;" : "=l"(gsrc) : "l"(src));
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// 2D tensor-map global -> shared copy (box defined by the map) into this CTA's own shared memory,
// completing on `bar`
WL_D void tma_g2s_2d(void* dst, const CUtensorMap* map, int c0, int c1, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}

// The spinor rows are copied with the TMA 128-byte swizzle: viewed as 128-byte
// lines, the 16-byte chunk j of line r lands at chunk j ^ (r mod 8) (buffer
// 1024-byte aligned).  This spreads the components that the sites of one warp
// read at the same time (192-byte site stride: every other site on the same
// banks otherwise) over the bank groups.
WL_D const double2* swz_psi(const unsigned char* chunk, int site, int comp) {
  const unsigned o = (unsigned)site * 192u + (unsigned)comp * 16u;
  const unsigned line = o >> 7;
  const unsigned j = ((o >> 4) & 7u) ^ (line & 7u);
  return reinterpret_cast<const double2*>(chunk + (line << 7) + (j << 4));
}

// order this thread's earlier generic-proxy shared-memory accesses before later async-proxy ones
WL_D void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Links staged in shared memory (1) or read through L1 from global memory (0):
// without them a stage is 384*Lt bytes instead of 672*Lt and twice as many
// blocks fit on an SM, but the link loads then stall the stencil (measured at
// 24^3x48: 0.33 ms against 0.25 ms with staged links).
#ifndef WL_ROW_LINKS_SMEM
#define WL_ROW_LINKS_SMEM 1
#endif
#ifndef WL_ROW_BUFS
#define WL_ROW_BUFS 2
#endif
constexpr int kRowBufs = WL_ROW_BUFS;  // stage buffers per block (kRowBufs - 1 stages prefetched)
constexpr int kRowStages = 4;          // stages per row
// largest Lt whose kRowBufs stages (~672*Lt bytes each, padded) fit in shared memory, 3*Lt threads in a
// block, and a psi row of 1.5*Lt lines in one tensor-map box (<= 256)
constexpr int kRowMaxLt = (220 * 1024) / (672 * kRowBufs) < 148 ? (220 * 1024) / (672 * kRowBufs) : 148;
constexpr long long kRowWaitLimit = 1LL << 24;  // try_wait rounds before a wait is declared lost

struct RowHopArgs {
  Geom g;
  const double2* U;     // [4][V][9]
  const double2* in;    // [nrhs][V][12]
  double2* out;         // [nrhs][V][12]
  const double2* self;  // [nrhs][V][12] or nullptr
  double a, b;
  int nrhs;
  int pmask;            // bit p set: compute target sites of parity p
  int* err;             // set to 1 if a wait ran out
};

struct RowStage {
  int item, mu;
};

// psi chunks padded to 1024 bytes (swizzle atom), link chunks after them
WL_HD size_t row_psi_pad(int Lt) { return (((size_t)192 * Lt + 1023) / 1024) * 1024; }
WL_HD size_t row_stage_bytes(int Lt) {
  return ((2 * row_psi_pad(Lt) + (WL_ROW_LINKS_SMEM ? (size_t)288 * Lt : 0) + 1023) / 1024) * 1024;
}

WL_D RowStage row_stage_of(int k) {
  RowStage s;
  s.item = blockIdx.x + (k / kRowStages) * gridDim.x;
  const int q = k % kRowStages;
  s.mu = q == 0 ? 3 : q - 1;
  return s;
}

// buffer layout of a stage: [psi A | psi B | U fwd | U bwd]: swizzled psi rows (tensor map over the
// field viewed as 128-byte lines, box = one row = 1.5*Lt lines) padded to 1024 bytes, then 144*Lt-byte link rows
WL_D void row_stage_issue(const RowHopArgs& A, const CUtensorMap* psimap, const RowStage& st, unsigned char* buf,
                          unsigned long long* bar) {
  const Geom& g = A.g;
  const int Lt = g.L[3];
  const int nrows = g.V / Lt;
  const int rhs = st.item / nrows, row = st.item - rhs * nrows;
  const size_t spad = row_psi_pad(Lt), lk = (size_t)144 * Lt;
  const unsigned sp = 192u * (unsigned)Lt;
  const int line0 = (int)(((long long)rhs * g.V) * 3 / 2);  // first 128-byte line of this RHS
  const int lpr = Lt * 3 / 2;                               // lines per row (Lt even)
  const unsigned lkb = WL_ROW_LINKS_SMEM ? (unsigned)lk : 0u;
  if (st.mu == 3) {
    mbar_expect_tx(bar, sp + lkb);
    tma_g2s_2d(buf, psimap, 0, line0 + row * lpr, bar);
    if (WL_ROW_LINKS_SMEM) bulk_g2s(buf + 2 * spad, A.U + ((size_t)3 * g.V + (size_t)row * Lt) * 9, (unsigned)lk, bar);
    return;
  }
  // row = (x*Ly + y)*Lz + z ; neighbour rows along mu with periodic wrap
  const int stride = g.strideRow[st.mu];
  const int Lm = g.L[st.mu];
  const int xm = (row / stride) % Lm;
  const int rp = row + (xm == Lm - 1 ? -(Lm - 1) * stride : stride);
  const int rm = row + (xm == 0 ? (Lm - 1) * stride : -stride);
  mbar_expect_tx(bar, 2 * sp + 2 * lkb);
  tma_g2s_2d(buf, psimap, 0, line0 + rp * lpr, bar);
  tma_g2s_2d(buf + spad, psimap, 0, line0 + rm * lpr, bar);
  if (WL_ROW_LINKS_SMEM) {
    bulk_g2s(buf + 2 * spad, A.U + ((size_t)st.mu * g.V + (size_t)row * Lt) * 9, (unsigned)lk, bar);
    bulk_g2s(buf + 2 * spad + lk, A.U + ((size_t)st.mu * g.V + (size_t)rm * Lt) * 9, (unsigned)lk, bar);
  }
}

// One direction for thread (site t, colour a): acc[s] += [(1 + C g_mu) W psi]_s,a with W = ph*U
// (forward) or (ph*U)^dag (backward, DAGU), psi and the link read from shared memory.
template <int MU, int C, bool DAGU>
WL_D void row_dir(const unsigned char* chunk, int site, const double2* u, int a, bool ph, const Geom& g,
                  cplx<double> (&acc)[4]) {
  Half<double> h;
#pragma unroll
  for (int col = 0; col < 3; ++col) {
    auto ld = [&](int sp) {
      const double2 v = *swz_psi(chunk, site, sp * 3 + col);
      return cplx<double>{v.x, v.y};
    };
    if (MU == 3) {
      h.v[0][col] = C > 0 ? 2.0 * ld(0) : 2.0 * ld(2);
      h.v[1][col] = C > 0 ? 2.0 * ld(1) : 2.0 * ld(3);
      continue;
    }
    const cplx<double> s0 = ld(0), s1 = ld(1), s2 = ld(2), s3 = ld(3);
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
  cplx<double> uh[2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
  for (int b = 0; b < 3; ++b) {
#if WL_ROW_LINKS_SMEM
    const double2 w = DAGU ? u[b * 3 + a] : u[a * 3 + b];
#else
    const double2 w = ldg(u + (DAGU ? b * 3 + a : a * 3 + b));
#endif
    const cplx<double> wc{w.x, w.y};
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      if (DAGU) fmac_(uh[s], wc, h.v[s][b]);
      else fma_(uh[s], wc, h.v[s][b]);
    }
  }
  if (ph) {
    const cplx<double> p{g.ph_re[MU], DAGU ? -g.ph_im[MU] : g.ph_im[MU]};
    uh[0] = uh[0] * p;
    uh[1] = uh[1] * p;
  }
  // spin_accum for one colour: rows 0,1 = uh, rows 2,3 reconstructed
  if (MU == 3) {  // (1 + g3) keeps rows 0,1; (1 - g3) rows 2,3
    if (C > 0) {
      acc[0] = acc[0] + uh[0];
      acc[1] = acc[1] + uh[1];
    } else {
      acc[2] = acc[2] + uh[0];
      acc[3] = acc[3] + uh[1];
    }
    return;
  }
  acc[0] = acc[0] + uh[0];
  acc[1] = acc[1] + uh[1];
  if (MU == 0) {
    acc[2] = C > 0 ? acc[2] + uh[1] : acc[2] - uh[1];
    acc[3] = C > 0 ? acc[3] + uh[0] : acc[3] - uh[0];
  } else if (MU == 1) {
    acc[2] = C > 0 ? acc[2] + mul_mi(uh[1]) : acc[2] + mul_i(uh[1]);
    acc[3] = C > 0 ? acc[3] + mul_i(uh[0]) : acc[3] + mul_mi(uh[0]);
  } else {
    acc[2] = C > 0 ? acc[2] + mul_i(uh[0]) : acc[2] + mul_mi(uh[0]);
    acc[3] = C > 0 ? acc[3] + mul_i(uh[1]) : acc[3] + mul_mi(uh[1]);
  }
}

template <int MU, bool DAG>
WL_D void row_stage_compute(const RowHopArgs& A, const unsigned char* buf, int row, int t, int a,
                            cplx<double> (&acc)[4]) {
  constexpr int CF = DAG ? +1 : -1;
  constexpr int CB = -CF;
  const Geom& g = A.g;
  const int Lt = g.L[3];
  const size_t spad = row_psi_pad(Lt), lk = (size_t)144 * Lt;
  const unsigned char* psiA = buf;
  const unsigned char* psiB = buf + spad;
#if WL_ROW_LINKS_SMEM
  const double2* Uf = reinterpret_cast<const double2*>(buf + 2 * spad);
  const double2* Ub = reinterpret_cast<const double2*>(buf + 2 * spad + lk);
#else
  (void)lk;
  const double2* Uf = A.U + ((size_t)MU * g.V + (size_t)row * Lt) * 9;  // own row of U_mu
  const double2* Ub = Uf;
  if (MU < 3) {  // row x - mu of U_mu
    const int stride = g.strideRow[MU], Lm = g.L[MU];
    const int xm_ = (row / stride) % Lm;
    Ub = A.U + ((size_t)MU * g.V + (size_t)(row + (xm_ == 0 ? (Lm - 1) * stride : -stride)) * Lt) * 9;
  }
#endif
  if (MU == 3) {
    const int tp = t == Lt - 1 ? 0 : t + 1, tm = t == 0 ? Lt - 1 : t - 1;
    const bool on = g.ph_on[3] != 0;
    row_dir<3, CF, false>(psiA, tp, Uf + t * 9, a, on && t == Lt - 1, g, acc);
    row_dir<3, CB, true>(psiA, tm, Uf + tm * 9, a, on && t == 0, g, acc);
  } else {
    const int xm = (row / g.strideRow[MU]) % g.L[MU];
    const bool on = g.ph_on[MU] != 0;
    row_dir<MU, CF, false>(psiA, t, Uf + t * 9, a, on && xm == g.L[MU] - 1, g, acc);
    row_dir<MU, CB, true>(psiB, t, Ub + t * 9, a, on && xm == 0, g, acc);
  }
}

// Every thread of the block waits (bounded); the block then agrees on the outcome,
// so that all of its threads leave together if the wait was lost.
WL_D bool row_wait(const RowHopArgs& A, unsigned long long* bar, unsigned parity) {
  bool ok = false;
  for (long long i = 0; i < kRowWaitLimit && !ok; ++i) ok = mbar_try_wait(bar, parity);
  return __syncthreads_and(ok ? 1 : 0) != 0;
}

template <bool DAG>
__global__ void __launch_bounds__(3 * kRowMaxLt) row_hop_kernel(const __grid_constant__ CUtensorMap psimap,
                                                                 RowHopArgs A) {
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem);
  // stage buffers start at the first 1024-byte boundary past the barriers (swizzle atom)
  unsigned char* bufs = smem + 128u + ((1024u - ((smem_u32(smem) + 128u) & 1023u)) & 1023u);
  const Geom& g = A.g;
  const int Lt = g.L[3];
  const int nrows = g.V / Lt;
  const int nitems = nrows * A.nrhs;
  const size_t sbytes = row_stage_bytes(Lt);
  const int tid = threadIdx.x;
  const int t = tid / 3, a = tid - 3 * t;
  const bool worker = tid < 3 * Lt;
  // this block's items: blockIdx.x, blockIdx.x + gridDim.x, ...; kRowStages stages each
  const int my_items = (int)blockIdx.x < nitems ? (nitems - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int nst = kRowStages * my_items;
  if (tid == 0) {
#pragma unroll
    for (int j = 0; j < kRowBufs; ++j) mbar_init(&bars[j], 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (tid == 0)
    for (int k = 0; k < kRowBufs && k < nst; ++k) row_stage_issue(A, &psimap, row_stage_of(k), bufs + k * sbytes, &bars[k]);
  cplx<double> acc[4];
  for (int k = 0; k < nst; ++k) {
    const RowStage s = row_stage_of(k);
    const int slot = k % kRowBufs;
    const unsigned parity = (unsigned)((k / kRowBufs) & 1);
    const unsigned char* buf = bufs + slot * sbytes;
    if (!row_wait(A, &bars[slot], parity)) {
      // record the lost wait, give the copies already issued one more bounded wait
      // (they write into this block's shared memory), and stop
      if (tid == 0) atomicExch(A.err, 1);
      for (int j = k; j < k + kRowBufs && j < nst; ++j)
        for (long long i = 0; i < kRowWaitLimit; ++i)
          if (mbar_try_wait(&bars[j % kRowBufs], (unsigned)((j / kRowBufs) & 1))) break;
      return;
    }
    const int rhs = s.item / nrows, row = s.item - rhs * nrows;
    if (s.mu == 3) {
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = {0.0, 0.0};
    }
    if (worker) {
      switch (s.mu) {
        case 3: row_stage_compute<3, DAG>(A, buf, row, t, a, acc); break;
        case 0: row_stage_compute<0, DAG>(A, buf, row, t, a, acc); break;
        case 1: row_stage_compute<1, DAG>(A, buf, row, t, a, acc); break;
        default: row_stage_compute<2, DAG>(A, buf, row, t, a, acc); break;
      }
    }
    if ((k % kRowStages) == kRowStages - 1 && worker) {  // item done: out = a*self + b*acc on target parities
      const int x2 = row % g.L[2], r2 = row / g.L[2];
      const int x1 = r2 % g.L[1], x0 = r2 / g.L[1];
      const int par = (x0 + x1 + x2 + t) & 1;
      if ((A.pmask >> par) & 1) {
        const size_t site = (size_t)rhs * g.V + (size_t)row * Lt + t;
        double2* o = A.out + site * 12;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          cplx<double> v = A.b * acc[q];
          if (A.self) {
            const double2 sv = A.self[site * 12 + q * 3 + a];
            v = v + A.a * cplx<double>{sv.x, sv.y};
          }
          o[q * 3 + a] = make_double2(v.re, v.im);
        }
      }
    }
    // the buffer is free once every thread has read it; then refill it
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0 && k + kRowBufs < nst) row_stage_issue(A, &psimap, row_stage_of(k + kRowBufs), bufs + slot * sbytes, &bars[slot]);
  }
}

}  // namespace wl
