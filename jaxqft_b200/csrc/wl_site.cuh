// Site-local kernels: layout conversion (reference <-> internal), precision
// conversion, gauge-field compression and the CG vector/scalar updates.
#pragma once
#include "wl_hop_fast.cuh"

namespace wl {

// ------------------------------------------------------------- generic driver
template <class F>
struct SiteArgs {
  int vh;
  int parity0;
  int nrhs;
  const int* mask;
  F f;
  Reduce red;
};

template <int NR, class F>
__global__ void __launch_bounds__(256) site_kernel(SiteArgs<F> A) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int parity = A.parity0 ^ blockIdx.z;
  const int rhs0 = (blockIdx.y * blockDim.y + threadIdx.y) * NR;
  double red[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    red[r] = 0.0;
    const int rhs = rhs0 + r;
    if (c < A.vh && rhs < A.nrhs && (A.mask == nullptr || A.mask[rhs] != 0)) red[r] = A.f(rhs, parity, c);
  }
  if (F::kReduce) reduce_rhs<NR>(red, A.red, A.nrhs, A.mask);
}

// Same functors with RHS in the lanes: lane = rhs + R * site (fields in the
// RHS-innermost layout coalesce this way).
template <int R, class F>
__global__ void __launch_bounds__(kLaneBlock) site_lanes_kernel(SiteArgs<F> A) {
  constexpr int S = kLaneBlock / R;
  const int tid = threadIdx.x;
  const int c = blockIdx.x * S + tid / R;
  const int rhs = blockIdx.y * R + (tid % R);
  const int parity = A.parity0 ^ blockIdx.z;
  double red = 0.0;
  if (c < A.vh && rhs < A.nrhs && (A.mask == nullptr || A.mask[rhs] != 0)) red = A.f(rhs, parity, c);
  if (F::kReduce) reduce_lanes<R>(red, A.red, A.nrhs, A.mask);
}

// -------------------------------------------------------- layout conversion
// reference complex128 [rhs][V][4][3] -> internal compact field of parity p
template <class SF>
struct FPack {
  static constexpr bool kReduce = true;  // returns |psi|^2 of the packed site (FP64 input)
  Geom g;
  SpinorRef in;   // in-field index = rhs - rhs_off
  int rhs_off;
  SF out[2];
  WL_D double operator()(int rhs, int parity, int c) const {
    const long long f = flat_of(g, parity, c);
    Spinor<double> s;
    in.load(s, rhs - rhs_off, f);
    Spinor<typename SF::real> o;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
        o.v[a][b] = {(typename SF::real)s.v[a][b].re, (typename SF::real)s.v[a][b].im};
    out[parity].store(o, rhs, c);
    return snorm2(s);
  }
};

// internal FP64 compact -> reference layout (sites of that parity only)
struct FUnpack {
  static constexpr bool kReduce = false;
  Geom g;
  SpinorField<P_DOUBLE> in[2];
  SpinorRef out;  // out-field index = rhs - rhs_off
  int rhs_off;
  int in_off;     // in-field index = rhs + in_off
  WL_D double operator()(int rhs, int parity, int c) const {
    const long long f = flat_of(g, parity, c);
    Spinor<double> s;
    in[parity].load(s, rhs + in_off, c);
    out.store(s, rhs - rhs_off, f);
    return 0.0;
  }
};

// zero the reference-layout sites of one parity
struct FZeroRef {
  static constexpr bool kReduce = false;
  Geom g;
  SpinorRef out;
  int rhs_off;
  WL_D double operator()(int rhs, int parity, int c) const {
    Spinor<double> z;
    zero(z);
    out.store(z, rhs - rhs_off, flat_of(g, parity, c));
    return 0.0;
  }
};

// precision conversion between internal compact fields, with |src|^2
template <class SFI, class SFO>
struct FConvert {
  static constexpr bool kReduce = true;
  SFI in[2];
  SFO out[2];
  WL_D double operator()(int rhs, int parity, int c) const {
    Spinor<typename SFI::real> s;
    in[parity].load_plain(s, rhs, c);
    Spinor<typename SFO::real> o;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
        o.v[a][b] = {(typename SFO::real)s.v[a][b].re, (typename SFO::real)s.v[a][b].im};
    out[parity].store(o, rhs, c);
    return snorm2(s);
  }
};

// zero an internal field
template <class SF>
struct FZero {
  static constexpr bool kReduce = false;
  SF out[2];
  WL_D double operator()(int rhs, int parity, int c) const {
    Spinor<typename SF::real> z;
    zero(z);
    out[parity].store(z, rhs, c);
    return 0.0;
  }
};

// ------------------------------------------------------------ CG updates
// x64 += xs (converted); xs = 0.  Gated by the reliable-update mask.
template <class SFS>
struct FAccumX {
  static constexpr bool kReduce = false;
  SpinorField<P_DOUBLE> x[2];
  SFS xs[2];
  WL_D double operator()(int rhs, int parity, int c) const {
    Spinor<typename SFS::real> s;
    xs[parity].load_plain(s, rhs, c);
    Spinor<double> xv;
    x[parity].load_plain(xv, rhs, c);
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        xv.v[a][b].re += (double)s.v[a][b].re;
        xv.v[a][b].im += (double)s.v[a][b].im;
      }
    x[parity].store(xv, rhs, c);
    Spinor<typename SFS::real> z;
    zero(z);
    xs[parity].store(z, rhs, c);
    return 0.0;
  }
};

// p = rs + beta * p.  Gated by the active mask.
template <class SFS>
struct FUpdateP {
  static constexpr bool kReduce = false;
  SFS rs[2];
  SFS p[2];
  const double* beta;
  WL_D double operator()(int rhs, int parity, int c) const {
    using T = typename SFS::real;
    if constexpr (std::is_same<T, float>::value) {  // packed FP32 pairs
      float2 r[12], pv[12];
      const float sr = Packed<SFS>::load(rs[parity], rhs, (unsigned)c, r);
      const float sp = Packed<SFS>::load(p[parity], rhs, (unsigned)c, pv) * float(beta[rhs]);
      const float2 r2 = f2(sr, sr), p2 = f2(sp, sp);
#pragma unroll
      for (int k = 0; k < 12; ++k) pv[k] = ffma2(p2, pv[k], fmul2(r2, r[k]));
      Packed<SFS>::store(p[parity], rhs, (unsigned)c, pv);
    } else {
      Spinor<T> r, pv, o;
      rs[parity].load_plain(r, rhs, c);
      p[parity].load_plain(pv, rhs, c);
      axpby(o, T(1), r, T(beta[rhs]), pv);
      p[parity].store(o, rhs, c);
    }
    return 0.0;
  }
};

// ------------------------------------------------------------ CG epilogues
// Last hop of the sloppy normal operator fused with the CG update:
//   Ap = a*y + b*acc ; alpha = r2/pAp ; xs += alpha p ; rs -= alpha Ap ; return |rs|^2
template <class SF>
struct EpiCG {
  static constexpr bool kReduce = true;
  SF y[2], p[2], xs[2], rs[2];
  const double* a;
  const double* b;
  const double* r2;
  const double* pAp;
  const double* alpha;  // r2 / pAp per RHS (written by the pAp reduction), packed path
  WL_D double operator()(int rhs, int parity, long long idx, Spinor<typename SF::real>& acc) const {
    using T = typename SF::real;
    const double den = pAp[rhs];
    const T alpha = (den > 0.0) ? T(r2[rhs] / den) : T(0);
    Spinor<T> yv, pv, xv, rv;
    y[parity].load(yv, rhs, idx);
    p[parity].load_plain(pv, rhs, idx);
    xs[parity].load_plain(xv, rhs, idx);
    rs[parity].load_plain(rv, rhs, idx);
    const T aa = T(a[rhs]), bb = T(b[rhs]);
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cplx<T> ap = aa * yv.v[s][c] + bb * acc.v[s][c];
        xv.v[s][c] = xv.v[s][c] + alpha * pv.v[s][c];
        rv.v[s][c] = rv.v[s][c] - alpha * ap;
      }
    xs[parity].store(xv, rhs, idx);
    rs[parity].store(rv, rhs, idx);
    return snorm2(rv);
  }
  // same on packed FP32 pairs; the order keeps at most two packed spinors live
  WL_D double packed(int rhs, int parity, unsigned idx, float2 (&acc)[12]) const {
    const float al = float(alpha[rhs]);
    const float bb = float(b[rhs]);
    const float2 b2 = f2(bb, bb), nal = f2(-al, -al);
    float2 v[12];
    {  // acc <- Ap = a*y + b*acc
      const float sy = Packed<SF>::load(y[parity], rhs, idx, v) * float(a[rhs]);
      const float2 s2 = f2(sy, sy);
#pragma unroll
      for (int k = 0; k < 12; ++k) acc[k] = ffma2(b2, acc[k], fmul2(s2, v[k]));
    }
    double n;
    {  // rs <- rs - alpha Ap
      const float sr = Packed<SF>::load(rs[parity], rhs, idx, v);
      const float2 s2 = f2(sr, sr);
#pragma unroll
      for (int k = 0; k < 12; ++k) v[k] = ffma2(nal, acc[k], fmul2(s2, v[k]));
      Packed<SF>::store(rs[parity], rhs, idx, v);
      n = pnorm2(v);
    }
    {  // xs <- xs + alpha p
      const float sp = Packed<SF>::load(p[parity], rhs, idx, acc) * al;
      const float sx = Packed<SF>::load(xs[parity], rhs, idx, v);
      const float2 p2 = f2(sp, sp), x2 = f2(sx, sx);
#pragma unroll
      for (int k = 0; k < 12; ++k) v[k] = ffma2(p2, acc[k], fmul2(x2, v[k]));
      Packed<SF>::store(xs[parity], rhs, idx, v);
    }
    return n;
  }
  // same on one colour of an FP16 record (tensor-core hop): slice_in issues the four
  // loads early, slice_out (called by every lane of the warp) finishes the records
  struct SliceIn {
    SliceHalf::Raw y, r, p, x;
  };
  WL_D SliceIn slice_in(int rhs, int parity, unsigned idx, int t, bool mine) const {
    return SliceIn{SliceHalf::load(y[parity], rhs, idx, t, mine), SliceHalf::load(rs[parity], rhs, idx, t, mine),
                   SliceHalf::load(p[parity], rhs, idx, t, mine), SliceHalf::load(xs[parity], rhs, idx, t, mine)};
  }
  WL_D double slice_out(const SliceIn& in, int rhs, int parity, unsigned idx, int t, bool act,
                        float2 (&acc)[4]) const {
    const float al = act ? float(alpha[rhs]) : 0.f;
    const float bb = act ? float(b[rhs]) : 0.f, aa = act ? float(a[rhs]) : 0.f;
    const float2 b2 = f2(bb, bb), nal = f2(-al, -al);
    float2 v[4];
    {  // acc <- Ap = a*y + b*acc
      const float sy = SliceHalf::unpack(in.y, v) * aa;
      const float2 s2 = f2(sy, sy);
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[k] = ffma2(b2, acc[k], fmul2(s2, v[k]));
    }
    double n;
    {  // rs <- rs - alpha Ap
      const float sr = SliceHalf::unpack(in.r, v);
      const float2 s2 = f2(sr, sr);
#pragma unroll
      for (int k = 0; k < 4; ++k) v[k] = ffma2(nal, acc[k], fmul2(s2, v[k]));
      SliceHalf::store(rs[parity], rhs, idx, t, act, v);
      n = pnorm2_4(v);
    }
    {  // xs <- xs + alpha p
      const float sp = SliceHalf::unpack(in.p, acc) * al;
      const float sx = SliceHalf::unpack(in.x, v);
      const float2 p2 = f2(sp, sp), x2 = f2(sx, sx);
#pragma unroll
      for (int k = 0; k < 4; ++k) v[k] = ffma2(p2, acc[k], fmul2(x2, v[k]));
      SliceHalf::store(xs[parity], rhs, idx, t, act, v);
    }
    return n;
  }
};

// Last hop of the FP64 normal operator on x64, giving the true residual:
//   r = bvec - (a*y + b*acc) ; rs = convert(r) ; return |r|^2 (FP64)
template <class SFS>
struct EpiResid {
  static constexpr bool kReduce = true;
  SpinorField<P_DOUBLE> y[2], bvec[2];
  SFS rs[2];
  const double* a;
  const double* b;
  WL_D double operator()(int rhs, int parity, long long idx, Spinor<double>& acc) const {
    Spinor<double> yv, bv;
    y[parity].load(yv, rhs, idx);
    bvec[parity].load(bv, rhs, idx);
    const double aa = a[rhs], bb = b[rhs];
    Spinor<typename SFS::real> o;
    double n = 0.0;
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cplx<double> r = bv.v[s][c] - (aa * yv.v[s][c] + bb * acc.v[s][c]);
        n += norm2(r);
        o.v[s][c] = {(typename SFS::real)r.re, (typename SFS::real)r.im};
      }
    rs[parity].store(o, rhs, idx);
    return n;
  }
};

// ------------------------------------------------------------ gauge upload
// Reference BMXYIJ complex128 [mu][V][3][3] (one configuration) -> internal
// parity-split copies.  Also records max |U U^dag - 1| + |det U - 1| so the
// host knows whether 12-real reconstruction is exact for these links.
struct GaugeOut {
  double2* d18;   // [p][mu][9][Vh]
  double2* d12;   // [p][mu][6][Vh]
  float4* s12;    // [p][mu][3][Vh]
  uint2* h12;     // [p][mu][3][Vh]
  unsigned int* unitarity_err;  // float bits, atomicMax
};

__global__ void gauge_convert_kernel(Geom g, const double2* __restrict__ U, GaugeOut o) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int parity = blockIdx.y;
  const int mu = blockIdx.z;
  if (c >= g.Vh) return;
  const long long f = flat_of(g, parity, c);
  const double2* src = U + ((long long)mu * g.V + f) * 9;
  Link<double> u;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    double2 v = src[k];
    u.m[k / 3][k % 3] = {v.x, v.y};
  }
  const long long base = (long long)(parity * 4 + mu);
  const int vh = g.Vh;
#pragma unroll
  for (int k = 0; k < 9; ++k) o.d18[(base * 9 + k) * vh + c] = make_double2(u.m[k / 3][k % 3].re, u.m[k / 3][k % 3].im);
#pragma unroll
  for (int k = 0; k < 6; ++k) o.d12[(base * 6 + k) * vh + c] = make_double2(u.m[k / 3][k % 3].re, u.m[k / 3][k % 3].im);
  float f12[12];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    f12[2 * k] = (float)u.m[k / 3][k % 3].re;
    f12[2 * k + 1] = (float)u.m[k / 3][k % 3].im;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    o.s12[(base * 3 + k) * vh + c] = make_float4(f12[4 * k], f12[4 * k + 1], f12[4 * k + 2], f12[4 * k + 3]);
    o.h12[(base * 3 + k) * vh + c] = make_uint2(f2h(f12[4 * k], f12[4 * k + 1]), f2h(f12[4 * k + 2], f12[4 * k + 3]));
  }
  // unitarity / determinant check
  double err = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cplx<double> s = {0.0, 0.0};
#pragma unroll
      for (int k = 0; k < 3; ++k) fmac_(s, u.m[j][k], u.m[i][k]);  // (U U^dag)_ij = sum_k U_ik conj(U_jk)
      if (i == j) s.re -= 1.0;
      err = fmax(err, sqrt(norm2(s)));
    }
  cplx<double> det = u.m[0][0] * (u.m[1][1] * u.m[2][2] - u.m[1][2] * u.m[2][1]) -
                     u.m[0][1] * (u.m[1][0] * u.m[2][2] - u.m[1][2] * u.m[2][0]) +
                     u.m[0][2] * (u.m[1][0] * u.m[2][1] - u.m[1][1] * u.m[2][0]);
  det.re -= 1.0;
  err = fmax(err, sqrt(norm2(det)));
  float ef = (float)err;
  // warp max then one atomic per warp
  for (int off = 16; off > 0; off >>= 1) ef = fmaxf(ef, __shfl_down_sync(0xffffffffu, ef, off));
  if ((threadIdx.x & 31) == 0) atomicMax(o.unitarity_err, __float_as_uint(ef));
}

// ------------------------------------------------------------ scalar control
// One block; thread s handles slot s.  See the engine for the state machine.
struct CGScalars {
  double* r2;        // current residual^2 used by alpha
  double* r2_new;    // sloppy residual^2 after the update (reduction target)
  double* pAp;       // |M p|^2 (reduction target)
  double* r2_true;   // true residual^2 from the reliable update (reduction target)
  double* rmax2;     // max residual^2 since the last reliable update
  double* b2;
  double* tol2;
  double* beta;
  int* active;
  int* ru;
  int* iters;
  int* maxiter;
  int* status;
  int* n_ru;
  int* n_active;     // single int
  double delta2;
};

enum SlotStatus { ST_IDLE = 0, ST_RUNNING = 1, ST_CONVERGED = 2, ST_MAXITER = 3, ST_BREAKDOWN = 4, ST_NAN = 5 };

// Decides which slots take a reliable update this iteration.  In a CUDA graph
// with a conditional node (`use_cond`), also switches the node's body (the FP64
// true-residual kernels) on only when at least one slot needs it, and counts
// such iterations in *ru_iters.
// Reliable-update decision per slot.  With `group` set, one slot's trigger
// sends every active slot through the update: the batched FP64 update costs
// the same for one slot as for all, and updating together keeps the slots'
// update schedules aligned instead of staggered over many iterations.
__global__ void cg_decide_kernel(CGScalars S, int n, int use_cond, cudaGraphConditionalHandle cond, int* ru_iters,
                                 int group) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int s = threadIdx.x; s < n; s += blockDim.x) {
    S.ru[s] = 0;
    if (!S.active[s]) continue;
    const double r2n = S.r2_new[s];
    const double pap = S.pAp[s];
    if (!isfinite(r2n) || !isfinite(pap)) {
      S.status[s] = ST_NAN;
      S.active[s] = 0;
      continue;
    }
    if (!(pap > 0.0)) {
      S.status[s] = ST_BREAKDOWN;
      S.active[s] = 0;
      continue;
    }
    const bool trig = (r2n < S.delta2 * S.rmax2[s]) || (r2n <= S.tol2[s] * S.b2[s]) || (S.iters[s] + 1 >= S.maxiter[s]);
    S.ru[s] = trig ? 1 : 0;
    if (trig) atomicOr(&any, 1);
  }
  __syncthreads();
  if (group && any)
    for (int s = threadIdx.x; s < n; s += blockDim.x)
      if (S.active[s]) S.ru[s] = 1;
  if (threadIdx.x == 0) {
    if (any && ru_iters) *ru_iters += 1;
    if (use_cond) cudaGraphSetConditional(cond, any ? 1u : 0u);
  }
}

// The WHILE node of a device-side iteration loop (one iteration per body execution).
// Whole solve (wl_solve): continue while any slot is active and fewer than `cap`
// iterations have run in this launch.  Engine run (wl_engine_run): the cap is read from
// `capd` (set per launch), and the loop also stops as soon as a slot has finished, i.e.
// the active count fell below its value at the start of the launch (`start`), so the
// host can retire it.
struct SolveLoop {
  const int* n_active;  // written by cg_finalize_kernel of the same iteration
  int* count;           // iterations of this launch (zeroed before each launch)
  int cap;
  cudaGraphConditionalHandle handle;
  const int* capd;      // engine run: per-launch cap (else nullptr: cap)
  const int* start;     // engine run: active count at the start of the launch (else nullptr)
  int* total;           // engine run: iterations over all launches (else nullptr)
};

// One step of the loop: count the iteration and set the WHILE condition from the active
// count `na` of this iteration.  Run by thread 0 of cg_finalize_kernel, which computes `na`.
WL_D void solve_loop_step(const SolveLoop& L, int na) {
  const int c = *L.count + 1;
  *L.count = c;
  if (L.total) *L.total += 1;
  const int cap = L.capd ? *L.capd : L.cap;
  const bool more = na > 0 && c < cap && (L.start == nullptr || na >= *L.start);
  cudaGraphSetConditional(L.handle, more ? 1u : 0u);
}

// Per-launch state of an engine run: the cap, the active count at the start, the count reset.
__global__ void run_loop_setup_kernel(int* capd, int cap, int* start, const int* n_active, int* count) {
  *capd = cap;
  *start = *n_active;
  *count = 0;
}

// With L.count set (an iteration captured inside a device-side loop) thread 0 also takes the
// loop's step, so the loop costs no kernel of its own.
__global__ void cg_finalize_kernel(CGScalars S, int n, SolveLoop L) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int local = 0;
  for (int s = threadIdx.x; s < n; s += blockDim.x) {
    if (!S.active[s]) continue;
    double r2n;
    if (S.ru[s]) {
      r2n = S.r2_true[s];
      S.rmax2[s] = r2n;
      S.n_ru[s] += 1;
    } else {
      r2n = S.r2_new[s];
      S.rmax2[s] = fmax(S.rmax2[s], r2n);
    }
    S.iters[s] += 1;
    if (!isfinite(r2n)) {
      S.status[s] = ST_NAN;
      S.active[s] = 0;
      continue;
    }
    S.beta[s] = r2n / S.r2[s];
    S.r2[s] = r2n;
    if (S.ru[s] && r2n <= S.tol2[s] * S.b2[s]) {
      S.status[s] = ST_CONVERGED;
      S.active[s] = 0;
      continue;
    }
    if (S.iters[s] >= S.maxiter[s]) {
      S.status[s] = ST_MAXITER;
      S.active[s] = 0;
      continue;
    }
    local++;
  }
  atomicAdd(&cnt, local);
  __syncthreads();
  if (threadIdx.x == 0) {
    *S.n_active = cnt;
    if (L.count) solve_loop_step(L, cnt);
  }
}

}  // namespace wl
