// libwilson_sm100: C-ABI implementation (contexts, gauge fields, operators,
// batched mixed-precision CG engine, pseudofermion force).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>

#include <cudaTypedefs.h>
#include <nvtx3/nvToolsExt.h>
#include <vector>

#include "../../include/wilson_sm100.h"
#include "wl_force.cuh"
#include "wl_gauge.cuh"
#include "wl_meas.cuh"
#include "wl_reftile.cuh"
#include "wl_rng.cuh"
#include "wl_blas.cuh"
#include "wl_rowhop.cuh"
#include "wl_hop_fast.cuh"
#include "wl_site.cuh"
#include "wl_hop_mma.cuh"

using namespace wl;

// Named host ranges around the entry points (NVTX, header-only and inert
// unless a profiler is attached).  A tool can then attribute kernels to the
// call that launched them, e.g. ncu --nvtx --nvtx-include "wl_solve/".
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// ============================================================== error helpers
struct wl_ctx {
  Geom g;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  // scratch for reference-layout operator chains (temp full fields)
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  // scratch for the gauge-sector reductions (block partials + per-batch results)
  double* red = nullptr;
  size_t red_bytes = 0;
  int* dev_err = nullptr;  // set by kernels whose bounded waits ran out (read at wl_ctx_synchronize)
  int sm_count = 0;
};

struct wl_gauge {
  wl_ctx* ctx = nullptr;
  double2* d18 = nullptr;
  double2* d12 = nullptr;
  float4* s12 = nullptr;
  uint2* h12 = nullptr;
  const double2* ref = nullptr;  // caller's reference-layout links (valid during wl_gauge_create/update only)
  double2* ref_copy = nullptr;   // library-owned copy of the reference layout (for reference-layout kernels)
  unsigned int* uerr = nullptr;  // device float bits
  float unitarity = 0.f;
  unsigned long long id = 0;     // unique per gauge object (graphs capture its buffers)
};
static std::atomic<unsigned long long> g_gauge_ids{1};
extern "C" void wl_release_solve_cache(wl_ctx* ctx);

static thread_local std::string g_static_err;
static std::atomic<long long> g_launches{0};
extern "C" int64_t wl_kernel_launches(void) { return g_launches.load(); }

// Out-of-range site indices counted by a checking build on the current device
// since the last call (and cleared), or -1 in a build without the checks.
extern "C" int64_t wl_bounds_errors(long long* first_bad) {
#if WL_BOUNDS_CHECK
  unsigned int n = 0;
  long long first = 0;
  if (cudaDeviceSynchronize() != cudaSuccess ||
      cudaMemcpyFromSymbol(&n, g_wl_bounds_errors, sizeof(n)) != cudaSuccess ||
      cudaMemcpyFromSymbol(&first, g_wl_bounds_first, sizeof(first)) != cudaSuccess) {
    cudaGetLastError();
    return -2;
  }
  const unsigned int zero = 0;
  if (cudaMemcpyToSymbol(g_wl_bounds_errors, &zero, sizeof(zero)) != cudaSuccess) {
    cudaGetLastError();
    return -2;
  }
  if (first_bad) *first_bad = first;
  return (int64_t)n;
#else
  if (first_bad) *first_bad = 0;
  return -1;
#endif
}

static inline void set_err(wl_ctx* ctx, const std::string& m);
#define WL_FAIL(ctx, code, msg) \
  do {                          \
    set_err((ctx), (msg));      \
    return (code);              \
  } while (0)

#define WL_CUDA(ctx, call)                                                                          \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess) {                                                                        \
      set_err((ctx), std::string(#call) + ": " + cudaGetErrorString(e_));                         \
      return (e_ == cudaErrorMemoryAllocation) ? WL_ERR_OOM : WL_ERR_CUDA;                          \
    }                                                                                               \
  } while (0)

static inline void set_err(wl_ctx* ctx, const std::string& m) {
  if (ctx) ctx->err = m;
  else g_static_err = m;
}

static wl_status check_launch(wl_ctx* ctx, const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    ctx->err = std::string(what) + ": " + cudaGetErrorString(e);
    return WL_ERR_CUDA;
  }
  return WL_OK;
}

// ============================================================== field helpers
static inline long long chunks_of(int prec) { return prec == P_DOUBLE ? 12 : (prec == P_SINGLE ? 6 : 3); }
static inline size_t chunk_bytes() { return 16; }
// bytes of one parity-half of one RHS (data + norm)
static inline size_t half_bytes(int prec, int vh) {
  return (size_t)chunks_of(prec) * chunk_bytes() * vh + (prec == P_HALF ? (size_t)vh * sizeof(float) : 0);
}

// A device field in the internal layout: nrhs x nparity halves, norms stored
// after all data for FP16.
struct IField {
  void* data = nullptr;
  float* norm = nullptr;
  int prec = 0, vh = 0, nrhs = 0, npar = 1;
  bool rhs_inner = false;  // [k][Vh][nrhs] (RHS innermost) instead of [rhs][k][Vh]
  long long rstride() const { return chunks_of(prec) * vh * npar; }  // site-major layout: chunks per rhs
};

template <int P>
static SpinorField<P> sf(const IField& f, int par) {
  SpinorField<P> s;
  using Ptr = decltype(s.ptr);
  const long long ch = chunks_of(P), vh = f.vh, n = f.nrhs;
  if (!f.rhs_inner) {
    s.ptr = reinterpret_cast<Ptr>(f.data) + par * ch * vh;
    s.rstride = (unsigned)(ch * vh * f.npar);
    s.kstride = (unsigned)vh;
    s.cstride = 1;
    s.nrstride = (unsigned)vh;
    s.ncstride = 1;
  } else {
    s.ptr = reinterpret_cast<Ptr>(f.data) + par * ch * vh * n;
    s.rstride = 1;
    s.kstride = (unsigned)(vh * n);
    s.cstride = (unsigned)n;
    s.nrstride = 1;
    s.ncstride = (unsigned)n;
  }
  s.norm = f.norm ? f.norm + par * n * vh : nullptr;
  return s;
}
// field pair indexed by parity; for single-parity fields both entries alias par 0
template <int P>
static void sf2(const IField& f, SpinorField<P> (&o)[2]) {
  o[0] = sf<P>(f, 0);
  o[1] = f.npar == 2 ? sf<P>(f, 1) : o[0];
}

static wl_status alloc_field(wl_ctx* ctx, IField& f, int prec, int vh, int nrhs, int npar, bool rhs_inner = false) {
  f.prec = prec;
  f.vh = vh;
  f.nrhs = nrhs;
  f.npar = npar;
  f.rhs_inner = rhs_inner;
  if ((unsigned long long)chunks_of(prec) * vh * npar * nrhs >= (1ull << 32))
    WL_FAIL(ctx, WL_ERR_ARG, "field of 2^32 or more 16-byte chunks (32-bit offsets): use fewer RHS per engine");
  size_t data = (size_t)chunks_of(prec) * 16 * vh * npar * nrhs;
  size_t nb = data + (prec == P_HALF ? (size_t)vh * npar * nrhs * sizeof(float) : 0);
  WL_CUDA(ctx, cudaMalloc(&f.data, nb));
  WL_CUDA(ctx, cudaMemsetAsync(f.data, 0, nb, ctx->stream));
  f.norm = prec == P_HALF ? reinterpret_cast<float*>(reinterpret_cast<char*>(f.data) + data) : nullptr;
  return WL_OK;
}
static size_t field_bytes(int prec, int vh, int nrhs, int npar) {
  size_t data = (size_t)chunks_of(prec) * 16 * vh * npar * nrhs;
  return data + (prec == P_HALF ? (size_t)vh * npar * nrhs * sizeof(float) : 0);
}
static void free_field(IField& f) {
  if (f.data) cudaFree(f.data);
  f.data = nullptr;
  f.norm = nullptr;
}

static SpinorRef sref(const void* p, const Geom& g) {
  SpinorRef r;
  r.ptr = (double2*)p;
  r.rstride = 12LL * g.V;
  r.Lt = g.L[3];
  return r;
}

// ============================================================== launch helpers
struct Tune {
  int nr = 1, bx = 128, by = 1;
  int lanes = 0;  // > 0: RHS-in-lanes hop (FP16/FP32 storage) with this many RHS lanes per site
  int pair = 0;   // 1: single-RHS stencil with two threads per site (hop_pair_kernel; FP64 or FP32 storage)
  int seq = 1;    // FP64 RHS-in-lanes hop: groups of `lanes` RHS each block works through in turn
  // 1: FP16 hop on the tensor cores (hop_mma_kernel, 16 RHS per warp) where its epilogue
  // allows.  Selected only by WL_FORCE_TUNE: at 24^3x48 with 16 RHS it takes 0.45 ms per hop
  // against 0.28 ms for the 16-lane kernel (same iteration counts).  It moves the colour
  // multiply to the tensor pipe (7 % busy) but executes about 800 warp instructions per site
  // (record fetch, relative weights, per-colour epilogue) against 650 for the lanes kernel, with
  // 12 resident warps per SM instead of 28, so it issues on 46 % of cycles.
  int mma = 0;
};

static dim3 grid_for(const Geom& g, const Tune& t, int nrhs, int npar) {
  if (t.mma) return dim3((g.Vh + kMmaSites - 1) / kMmaSites, (nrhs + kMmaRhs - 1) / kMmaRhs, npar);
  if (t.lanes > 0) {
    const int S = kLaneBlock / t.lanes, per = t.lanes * std::max(1, t.seq);
    return dim3((g.Vh + S - 1) / S, (nrhs + per - 1) / per, npar);
  }
  if (t.pair) return dim3((g.Vh + t.bx / 2 - 1) / (t.bx / 2), nrhs, npar);
  int groups = (nrhs + t.nr - 1) / t.nr;
  return dim3((g.Vh + t.bx - 1) / t.bx, (groups + t.by - 1) / t.by, npar);
}

template <class SF> struct UsesFastHop : std::false_type {};
template <> struct UsesFastHop<SpinorField<P_SINGLE>> : std::true_type {};
template <> struct UsesFastHop<SpinorField<P_HALF>> : std::true_type {};

// The FP16 RHS-in-lanes hop multiplies by the links in packed FP16 (HFMA2); WL_HALF_COLOR=0
// selects FP32 pairs instead (for comparisons).  Measured at 24^3x48, 16 RHS, on one box in
// interleaved runs: 48.1 / 47.9 solves/s against 45.8 / 45.8, hop 0.29-0.33 ms against
// 0.355-0.360, with the same iteration (156-165) and reliable-update (16) counts.
static bool half_color_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("WL_HALF_COLOR");
    return !(e && e[0] == '0');
  }();
  return on;
}

// The 16-lane FP16 hop accumulates its eight contributions in packed FP16 (relative weights,
// lane_site_hh) and is compiled for 8 resident blocks per SM; WL_HALF_ACC=0 selects FP32
// accumulation (per-epilogue register caps) for comparisons.  Measured at 24^3x48 with 16 RHS,
// two interleaved rounds on one box: 49.9-50.1 solves/s against 48.8-49.0 (hop 0.281-0.297 ms
// against 0.296-0.315), 157-165 CG iterations against 156-165, every true residual <= 1e-10.
static bool half_acc_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("WL_HALF_ACC");
    return !(e && e[0] == '0');
  }();
  return on;
}

// The drop-in pair kernel reads neighbour spinors as 64-byte pieces, one 32-byte sector per
// thread, and swaps spins within the pair by shuffles (WL_REF_SECTOR=0: per-spin loads).
static bool ref_sector_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("WL_REF_SECTOR");
    return !(e && e[0] == '0');
  }();
  return on;
}

static bool fast_hop_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("WL_FAST_HOP");
    return !(e && e[0] == '0');
  }();
  return on;
}

// `per_block`: partial sums each block writes per RHS (lane kernels: one per warp)
static void launch_finalize(const Reduce& r, int nrhs, dim3 grid, const int* mask, cudaStream_t st,
                            int per_block = 1) {
  g_launches++;
  reduce_finalize_kernel<<<nrhs, kFinalizeThreads, 0, st>>>(r, nrhs, (int)(grid.x * grid.z) * per_block, mask);
}

template <bool DAG, class IDX, class LF, class SF, class EPI>
static void launch_hop_impl(const Tune& t, const HopArgs<LF, SF, EPI>& a, int npar, cudaStream_t st);

// The tensor-core hop runs for FP16 fields on the compact layout behind epilogues that
// have a per-colour form; any other launch with Tune::mma set uses the lanes kernel.
template <class IDX, class SF, class EPI>
static Tune effective_tune(Tune t) {
  if (t.mma && !(std::is_same<SF, SpinorField<P_HALF>>::value && std::is_same<IDX, IdxCompact>::value &&
                 HasSlice<EPI>::value))
    t.mma = 0;
  return t;
}

template <bool DAG, class IDX, class LF, class SF, class EPI>
static void launch_hop(const Tune& t0, const HopArgs<LF, SF, EPI>& a, int npar, cudaStream_t st) {
  const Tune t = effective_tune<IDX, SF, EPI>(t0);
  launch_hop_impl<DAG, IDX>(t, a, npar, st);
  if (EPI::kReduce) launch_finalize(a.red, a.nrhs, grid_for(a.g, t, a.nrhs, npar), a.mask, st, 1);
}

template <bool DAG, class IDX, class LF, class SF, class EPI>
static void launch_hop_impl(const Tune& t, const HopArgs<LF, SF, EPI>& a, int npar, cudaStream_t st) {
  dim3 grid = grid_for(a.g, t, a.nrhs, npar), block(t.bx, t.by, 1);
  g_launches++;
  if constexpr (std::is_same<SF, SpinorField<P_DOUBLE>>::value && std::is_same<IDX, IdxCompact>::value) {
    if (t.lanes > 0) {  // FP64 fields stored RHS-innermost
      dim3 lb(kLaneBlock, 1, 1);
      switch (t.lanes * 10 + t.seq) {
        case 161: hop_lanes_d_kernel<DAG, 16><<<grid, lb, 0, st>>>(a); break;
        case 81: hop_lanes_d_kernel<DAG, 8><<<grid, lb, 0, st>>>(a); break;
        case 82: hop_lanes_d_kernel<DAG, 8, LF, EPI, 2><<<grid, lb, 0, st>>>(a); break;
        case 42: hop_lanes_d_kernel<DAG, 4, LF, EPI, 2><<<grid, lb, 0, st>>>(a); break;
        case 44: hop_lanes_d_kernel<DAG, 4, LF, EPI, 4><<<grid, lb, 0, st>>>(a); break;
        default: hop_lanes_d_kernel<DAG, 4><<<grid, lb, 0, st>>>(a); break;
      }
      return;
    }
    if (t.pair) {
      hop_pair_kernel<DAG><<<grid, dim3(t.bx, 1, 1), 0, st>>>(a);
      return;
    }
  }
  if constexpr (std::is_same<SF, SpinorField<P_SINGLE>>::value && std::is_same<IDX, IdxCompact>::value &&
                std::is_same<typename LF::real, float>::value) {
    if (t.pair && t.lanes == 0) {
      hop_pair_kernel<DAG><<<grid, dim3(t.bx, 1, 1), 0, st>>>(a);
      return;
    }
  }
  if constexpr (UsesFastHop<SF>::value && std::is_same<IDX, IdxCompact>::value) {
    if constexpr (std::is_same<SF, SpinorField<P_HALF>>::value && HasSlice<EPI>::value) {
      if (t.mma) {
        // 64 KB of dynamic shared memory per block (two record slots and the links of each
        // warp); the opt-in is set once per instantiation
        static const cudaError_t attr = cudaFuncSetAttribute(
            hop_mma_kernel<DAG, LF, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMmaSmemBytes);
        (void)attr;
        hop_mma_kernel<DAG><<<grid, dim3(kMmaWarps * 32, 1, 1), kMmaSmemBytes, st>>>(a);
        return;
      }
    }
    if constexpr (std::is_same<SF, SpinorField<P_HALF>>::value) {
      if (t.lanes > 0 && half_color_enabled()) {  // colour multiply in packed FP16 (HFMA2)
        dim3 lb(kLaneBlock, 1, 1);
        if (t.lanes == 16 && half_acc_enabled()) {
          hop_lanes_kernel<DAG, 16, LF, SF, EPI, true, true><<<grid, lb, 0, st>>>(a);
          return;
        }
        switch (t.lanes) {
          case 16: hop_lanes_kernel<DAG, 16, LF, SF, EPI, true><<<grid, lb, 0, st>>>(a); break;
          case 8: hop_lanes_kernel<DAG, 8, LF, SF, EPI, true><<<grid, lb, 0, st>>>(a); break;
          default: hop_lanes_kernel<DAG, 4, LF, SF, EPI, true><<<grid, lb, 0, st>>>(a); break;
        }
        return;
      }
    }
    if (t.lanes > 0) {
      dim3 lb(kLaneBlock, 1, 1);
      switch (t.lanes) {
        case 16: hop_lanes_kernel<DAG, 16><<<grid, lb, 0, st>>>(a); break;
        case 8: hop_lanes_kernel<DAG, 8><<<grid, lb, 0, st>>>(a); break;
        default: hop_lanes_kernel<DAG, 4><<<grid, lb, 0, st>>>(a); break;
      }
      return;
    }
    if (fast_hop_enabled()) {
      switch (t.nr) {
        case 4: hop_fast_kernel<DAG, 4><<<grid, block, 0, st>>>(a); break;
        case 2: hop_fast_kernel<DAG, 2><<<grid, block, 0, st>>>(a); break;
        default: hop_fast_kernel<DAG, 1><<<grid, block, 0, st>>>(a); break;
      }
      return;
    }
  }
  switch (t.nr) {
    case 4: hop_kernel<DAG, 4, IDX><<<grid, block, 0, st>>>(a); break;
    case 2: hop_kernel<DAG, 2, IDX><<<grid, block, 0, st>>>(a); break;
    default: hop_kernel<DAG, 1, IDX><<<grid, block, 0, st>>>(a); break;
  }
}

template <class F>
static void launch_site(const Tune& t, const Geom& g, int parity0, int npar, int nrhs, const int* mask, const F& f,
                        Reduce red, cudaStream_t st) {
  SiteArgs<F> a;
  a.vh = g.Vh;
  a.parity0 = parity0;
  a.nrhs = nrhs;
  a.mask = mask;
  a.f = f;
  a.red = red;
  dim3 grid = grid_for(g, t, nrhs, npar), block(t.bx, t.by, 1);
  g_launches++;
  switch (t.nr) {
    case 4: site_kernel<4><<<grid, block, 0, st>>>(a); break;
    case 2: site_kernel<2><<<grid, block, 0, st>>>(a); break;
    default: site_kernel<1><<<grid, block, 0, st>>>(a); break;
  }
  if (F::kReduce) launch_finalize(red, nrhs, grid, mask, st);
}

// Site functor over (site, RHS) with RHS in the lanes (for fields in the
// RHS-innermost layout).
template <class F>
static void launch_site_lanes(int R, const Geom& g, int parity0, int npar, int nrhs, const int* mask, const F& f,
                              Reduce red, cudaStream_t st) {
  SiteArgs<F> a;
  a.vh = g.Vh;
  a.parity0 = parity0;
  a.nrhs = nrhs;
  a.mask = mask;
  a.f = f;
  a.red = red;
  const int S = kLaneBlock / R;
  dim3 grid((g.Vh + S - 1) / S, (nrhs + R - 1) / R, npar), block(kLaneBlock, 1, 1);
  g_launches++;
  switch (R) {
    case 16: site_lanes_kernel<16><<<grid, block, 0, st>>>(a); break;
    case 8: site_lanes_kernel<8><<<grid, block, 0, st>>>(a); break;
    default: site_lanes_kernel<4><<<grid, block, 0, st>>>(a); break;
  }
  if (F::kReduce) launch_finalize(red, nrhs, grid, mask, st, 1);
}

// ============================================================== context
extern "C" int wl_version(void) { return 1; }

extern "C" wl_status wl_ctx_create(const wl_geometry* geom, int device, wl_ctx** out) {
  if (!geom || !out) WL_FAIL(nullptr, WL_ERR_ARG, "null argument");
  for (int mu = 0; mu < 4; ++mu)
    if (geom->dims[mu] < 2 || (geom->dims[mu] & 1))
      WL_FAIL(nullptr, WL_ERR_ARG, "every lattice extent must be even and >= 2");
  long long V = (long long)geom->dims[0] * geom->dims[1] * geom->dims[2] * geom->dims[3];
  if (V > (1LL << 30)) WL_FAIL(nullptr, WL_ERR_ARG, "lattice too large for 32-bit site indices");
  WL_CUDA(nullptr, cudaSetDevice(device));
  wl_ctx* c = new wl_ctx();
  c->device = device;
  Geom& g = c->g;
  for (int mu = 0; mu < 4; ++mu) g.L[mu] = geom->dims[mu];
  g.V = (int)V;
  g.Vh = (int)(V / 2);
  g.Lth = g.L[3] / 2;
  g.strideRow[0] = g.L[1] * g.L[2];
  g.strideRow[1] = g.L[2];
  g.strideRow[2] = 1;
  g.fd_lth = make_fastdiv((unsigned)g.Lth);
  g.fd_l2 = make_fastdiv((unsigned)g.L[2]);
  g.fd_l1 = make_fastdiv((unsigned)g.L[1]);
  g.Ty = 1;
  for (int d = 8; d >= 1; --d)
    if (g.L[1] % d == 0) {
      g.Ty = d;
      break;
    }
  g.fd_ty = make_fastdiv((unsigned)g.Ty);
  g.fd_l0 = make_fastdiv((unsigned)g.L[0]);
  for (int mu = 0; mu < 4; ++mu) {
    g.ph_re[mu] = geom->bc_re[mu];
    g.ph_im[mu] = geom->bc_im[mu];
    g.ph_on[mu] = (std::fabs(geom->bc_re[mu] - 1.0) > 1e-12 || std::fabs(geom->bc_im[mu]) > 1e-12) ? 1 : 0;
  }
  if (cudaMalloc(&c->dev_err, sizeof(int)) != cudaSuccess || cudaMemset(c->dev_err, 0, sizeof(int)) != cudaSuccess ||
      cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
    if (c->dev_err) cudaFree(c->dev_err);
    delete c;
    WL_FAIL(nullptr, WL_ERR_CUDA, "context set-up failed");
  }
  *out = c;
  return WL_OK;
}

extern "C" void wl_ctx_destroy(wl_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  wl_release_solve_cache(ctx);
  if (ctx->tmp) cudaFree(ctx->tmp);
  if (ctx->red) cudaFree(ctx->red);
  if (ctx->dev_err) cudaFree(ctx->dev_err);
  delete ctx;
}

extern "C" const char* wl_last_error(const wl_ctx* ctx) { return ctx ? ctx->err.c_str() : g_static_err.c_str(); }

extern "C" wl_status wl_ctx_set_stream(wl_ctx* ctx, void* stream) {
  if (!ctx) WL_FAIL(nullptr, WL_ERR_ARG, "null context");
  ctx->stream = (cudaStream_t)stream;
  return WL_OK;
}

extern "C" wl_status wl_ctx_synchronize(wl_ctx* ctx) {
  if (!ctx) WL_FAIL(nullptr, WL_ERR_ARG, "null context");
  WL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (ctx->dev_err) {
    int e = 0;
    WL_CUDA(ctx, cudaMemcpy(&e, ctx->dev_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
      WL_CUDA(ctx, cudaMemset(ctx->dev_err, 0, sizeof(int)));
      WL_FAIL(ctx, WL_ERR_TIMEOUT, "a bounded device wait ran out (row-staged operator); its output is invalid");
    }
  }
  return WL_OK;
}

extern "C" wl_status wl_eo_maps(wl_ctx* ctx, int32_t* even, int32_t* odd, int32_t* nbr) {
  if (!ctx) WL_FAIL(nullptr, WL_ERR_ARG, "null context");
  const Geom& g = ctx->g;
  // host restatement of the device index arithmetic (site_from_compact / neighbor)
  for (int p = 0; p < 2; ++p) {
    for (int c = 0; c < g.Vh; ++c) {
      int th = c % g.Lth, row = c / g.Lth;
      int z = row % g.L[2], r2 = row / g.L[2];
      int y = r2 % g.L[1], x = r2 / g.L[1];
      int t = 2 * th + ((p + x + y + z) & 1);
      int flat = row * g.L[3] + t;
      if (p == 0 && even) even[c] = flat;
      if (p == 1 && odd) odd[c] = flat;
      if (!nbr) continue;
      int xs[4] = {x, y, z, t};
      for (int mu = 0; mu < 4; ++mu)
        for (int dir = 0; dir < 2; ++dir) {
          int xx[4] = {xs[0], xs[1], xs[2], xs[3]};
          xx[mu] = (xx[mu] + (dir == 0 ? 1 : -1) + g.L[mu]) % g.L[mu];
          int f2 = ((xx[0] * g.L[1] + xx[1]) * g.L[2] + xx[2]) * g.L[3] + xx[3];
          nbr[((long long)(p * 4 + mu) * 2 + dir) * g.Vh + c] = f2 >> 1;
        }
    }
  }
  return WL_OK;
}

// ============================================================== gauge
static wl_status gauge_fill(wl_gauge* G, const void* U) {
  wl_ctx* ctx = G->ctx;
  const Geom& g = ctx->g;
  WL_CUDA(ctx, cudaMemcpyAsync(G->ref_copy, U, (size_t)4 * g.V * 9 * sizeof(double2), cudaMemcpyDeviceToDevice,
                               ctx->stream));
  WL_CUDA(ctx, cudaMemsetAsync(G->uerr, 0, sizeof(unsigned int), ctx->stream));
  GaugeOut o{G->d18, G->d12, G->s12, G->h12, G->uerr};
  dim3 grid((g.Vh + 127) / 128, 2, 4);
  g_launches++;
  gauge_convert_kernel<<<grid, 128, 0, ctx->stream>>>(g, G->ref_copy, o);
  return check_launch(ctx, "gauge_convert_kernel");
}

extern "C" wl_status wl_gauge_create(wl_ctx* ctx, const void* U, wl_gauge** out) {
  NvtxRange nvtx_range("wl_gauge_create");
  if (!ctx || !U || !out) WL_FAIL(ctx, WL_ERR_ARG, "null argument");
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  const Geom& g = ctx->g;
  wl_gauge* G = new wl_gauge();
  G->ctx = ctx;
  G->id = g_gauge_ids.fetch_add(1);
  size_t n = (size_t)2 * 4 * g.Vh;
  cudaError_t e = cudaSuccess;
  e = e ? e : cudaMalloc(&G->d18, n * 9 * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc(&G->d12, n * 6 * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc(&G->s12, n * 3 * sizeof(float4));
  if (e == cudaSuccess) e = cudaMalloc(&G->h12, n * 3 * sizeof(uint2));
  if (e == cudaSuccess) e = cudaMalloc(&G->ref_copy, (size_t)4 * g.V * 9 * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc(&G->uerr, sizeof(unsigned int));
  if (e != cudaSuccess) {
    wl_gauge_destroy(G);
    ctx->err = std::string("gauge allocation: ") + cudaGetErrorString(e);
    return WL_ERR_OOM;
  }
  wl_status st = gauge_fill(G, U);
  if (st != WL_OK) {
    wl_gauge_destroy(G);
    return st;
  }
  *out = G;
  return WL_OK;
}

extern "C" wl_status wl_gauge_update(wl_gauge* G, const void* U) {
  NvtxRange nvtx_range("wl_gauge_update");
  if (!G || !U) WL_FAIL(nullptr, WL_ERR_ARG, "null argument");
  return gauge_fill(G, U);
}

extern "C" wl_status wl_gauge_unitarity(wl_gauge* G, double* err) {
  if (!G || !err) WL_FAIL(nullptr, WL_ERR_ARG, "null argument");
  wl_ctx* ctx = G->ctx;
  unsigned int bits = 0;
  WL_CUDA(ctx, cudaMemcpyAsync(&bits, G->uerr, sizeof(bits), cudaMemcpyDeviceToHost, ctx->stream));
  WL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  float f;
  std::memcpy(&f, &bits, sizeof(f));
  G->unitarity = f;
  *err = (double)f;
  return WL_OK;
}

extern "C" void wl_gauge_destroy(wl_gauge* G) {
  if (!G) return;
  cudaFree(G->d18);
  cudaFree(G->d12);
  cudaFree(G->s12);
  cudaFree(G->h12);
  cudaFree(G->ref_copy);
  cudaFree(G->uerr);
  delete G;
}

// ============================================================== reference-layout operators
using RefHopArgs = HopArgs<LinkRefAdapter, SpinorRefAdapter, EpiXpay<SpinorRefAdapter, false>>;

static RefHopArgs ref_args(wl_ctx* ctx, wl_gauge* G, const void* in, void* out, const void* self, double a, double b,
                           int nrhs, int parity0) {
  RefHopArgs A;
  std::memset(&A, 0, sizeof(A));
  const Geom& g = ctx->g;
  A.g = g;
  A.links.f.ptr = G->ref_copy;
  A.links.f.V = g.V;
  A.src[0].f = sref(in, g);
  A.src[1].f = A.src[0].f;
  A.parity0 = parity0;
  A.nrhs = nrhs;
  A.mask = nullptr;
  A.epi.out[0].f = sref(out, g);
  A.epi.out[1].f = A.epi.out[0].f;
  A.epi.has_self = self != nullptr;
  if (self) {
    A.epi.self[0].f = sref(self, g);
    A.epi.self[1].f = A.epi.self[0].f;
  }
  A.epi.a = nullptr;
  A.epi.b = nullptr;
  A.epi.a0 = a;
  A.epi.b0 = b;
  return A;
}

static wl_status ensure_tmp(wl_ctx* ctx, size_t bytes) {
  if (ctx->tmp_bytes >= bytes) return WL_OK;
  if (ctx->tmp) {
    WL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    cudaFree(ctx->tmp);
    ctx->tmp = nullptr;
    ctx->tmp_bytes = 0;
  }
  WL_CUDA(ctx, cudaMalloc(&ctx->tmp, bytes));
  ctx->tmp_bytes = bytes;
  return WL_OK;
}

// Kernel for the reference-layout hop: 0 = ref_pair_kernel (two threads per site,
// 256-bit spinor loads, parity-split SoA links; the default), 1 = row_hop_kernel (TMA row
// staging), 2 = hop_kernel on the reference layout, 3 = ref_tile_kernel (warp tiles staged
// by TMA) where it applies (every site targeted, Lt a multiple of 16, 32-byte aligned
// fields), else ref_pair_kernel.  WL_REF_HOP=pair|row|generic|tile selects one (the pair
// kernel measured fastest: 0.199 ms against 0.241 for the tile kernel at 24^3x48).
static int ref_hop_kind() {
  static const int k = [] {
    const char* e = std::getenv("WL_REF_HOP");
    if (!e) return 0;
    if (std::strcmp(e, "row") == 0) return 1;
    if (std::strcmp(e, "generic") == 0) return 2;
    if (std::strcmp(e, "tile") == 0) return 3;
    return 0;
  }();
  return k;
}
static bool row_hop_enabled() { return ref_hop_kind() == 1; }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link needed)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// The spinor field `in` (nrhs fields) as 128-byte lines of 16 doubles for 2D tensor-map copies
// with the 128-byte swizzle, `box_lines` lines per copy.  False if the map cannot be built.
static bool encode_psi_lines_map(const void* in, long long lines, unsigned box_lines, CUtensorMap* map) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc || lines >= (1LL << 31) || ((uintptr_t)in & 15) || box_lines == 0 || box_lines > 256) return false;
  const cuuint64_t dims[2] = {16, (cuuint64_t)lines};
  const cuuint64_t strides[1] = {128};
  const cuuint32_t box[2] = {16, box_lines};
  const cuuint32_t estr[2] = {1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void*>(in), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Row-staged (TMA) FP64 hop for the reference layout; false if the lattice does
// not fit its shared-memory stages or the tensor map cannot be built.
template <bool DAG>
static bool row_hop(wl_ctx* ctx, wl_gauge* G, const void* in, void* out, const void* self, double a, double b,
                    int nrhs, int pmask) {
  const Geom& g = ctx->g;
  const int Lt = g.L[3];
  if (!row_hop_enabled() || Lt > kRowMaxLt) return false;
  const long long lines = (long long)nrhs * g.V * 3 / 2;  // the fields as 128-byte lines
  CUtensorMap map;
  if (!encode_psi_lines_map(in, lines, (unsigned)(Lt * 3 / 2), &map)) return false;
  RowHopArgs A{};
  A.g = g;
  A.U = G->ref_copy;
  A.in = (const double2*)in;
  A.out = (double2*)out;
  A.self = (const double2*)self;
  A.a = a;
  A.b = b;
  A.nrhs = nrhs;
  A.pmask = pmask;
  A.err = ctx->dev_err;
  const int threads = ((3 * Lt + 31) / 32) * 32;
  const size_t smem = 128 + 1024 + (size_t)kRowBufs * row_stage_bytes(Lt);
  int per_sm = 0;
  if (cudaFuncSetAttribute(row_hop_kernel<DAG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, row_hop_kernel<DAG>, threads, smem) != cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();  // fall back to the thread-per-site kernel; clear the error this left
    return false;
  }
  const long long items = (long long)(g.V / Lt) * nrhs;
  const int blocks = (int)std::min<long long>(items, (long long)per_sm * ctx->sm_count);
  g_launches++;
  row_hop_kernel<DAG><<<blocks, threads, smem, ctx->stream>>>(map, A);
  return true;
}

// Warp-tile TMA hop (wl_reftile.cuh): every site targeted, Lt a multiple of 16.
template <bool DAG>
static bool tile_hop_launch(wl_ctx* ctx, const RefSiteArgs& A) {
  const Geom& g = ctx->g;
  if (g.L[3] % kTileSites != 0) return false;
  const long long lines = (long long)A.nrhs * g.V * 3 / 2;
  if (lines >= (1LL << 31) || ((uintptr_t)A.in & 15)) return false;
  CUtensorMap map;
  if (!encode_psi_lines_map(A.in, lines, kTileSites * 3 / 2, &map)) return false;
  const size_t smem = tile_smem_bytes();
  int per_sm = 0;
  if (cudaFuncSetAttribute(ref_tile_kernel<DAG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ref_tile_kernel<DAG>, 32 * kTileWarps, smem) !=
          cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();  // fall back to the pair kernel; clear the error this left
    return false;
  }
  const long long tiles = (long long)(g.V / kTileSites) * A.nrhs;
  const long long want = (tiles + kTileWarps - 1) / kTileWarps;
  const int blocks = (int)std::min<long long>(want, (long long)per_sm * ctx->sm_count);
  g_launches++;
  ref_tile_kernel<DAG><<<blocks, 32 * kTileWarps, smem, ctx->stream>>>(map, A, ctx->dev_err);
  return true;
}

// Site-parallel reference-layout hop (wl_refsite.cuh); parity < 0 targets every site.
template <bool DAG>
static bool site_hop(wl_ctx* ctx, wl_gauge* G, const void* in, void* out, const void* self, double a, double b,
                     int nrhs, int parity) {
  const Geom& g = ctx->g;
  const int kind = ref_hop_kind();
  if ((kind != 0 && kind != 3) || nrhs > 65535) return false;
  RefSiteArgs A{};
  A.g = g;
  A.U = G->d18;
  A.in = (const double*)in;
  A.out = (double*)out;
  A.self = (const double*)self;
  A.a = a;
  A.b = b;
  A.nrhs = nrhs;
  A.parity = parity;
  const bool w32 = (((uintptr_t)in | (uintptr_t)out | (uintptr_t)self) & 31) == 0;
  if (kind == 3 && parity < 0 && w32 && tile_hop_launch<DAG>(ctx, A)) return true;
  const long long n = (parity < 0 ? g.V : g.Vh) * 2LL;  // two threads per target site
  const dim3 grid((unsigned)((n + kRefSiteBlock - 1) / kRefSiteBlock), nrhs);
  g_launches++;
  if (w32 && ref_sector_enabled()) ref_pair_kernel<DAG, 4, true><<<grid, kRefSiteBlock, 0, ctx->stream>>>(A);
  else if (w32) ref_pair_kernel<DAG, 4><<<grid, kRefSiteBlock, 0, ctx->stream>>>(A);
  else ref_pair_kernel<DAG, 2><<<grid, kRefSiteBlock, 0, ctx->stream>>>(A);
  return true;
}

// out(target parities) = a*self + b*hop(in); npar = 2 for both parities, else target parity0 only
template <bool DAG>
static void ref_hop(wl_ctx* ctx, wl_gauge* G, const void* in, void* out, const void* self, double a, double b,
                    int nrhs, int parity0, int npar) {
  if (site_hop<DAG>(ctx, G, in, out, self, a, b, nrhs, npar == 2 ? -1 : parity0)) return;
  if (row_hop<DAG>(ctx, G, in, out, self, a, b, nrhs, npar == 2 ? 3 : (1 << parity0))) return;
  RefHopArgs A = ref_args(ctx, G, in, out, self, a, b, nrhs, parity0);
  Tune t;
  t.nr = 1;
  t.bx = 128;
  t.by = 1;
  launch_hop<DAG, IdxFlat>(t, A, npar, ctx->stream);
}

extern "C" wl_status wl_apply(wl_ctx* ctx, wl_gauge* G, int op, double mass, unsigned flags, const void* in, void* out,
                              int nrhs) {
  NvtxRange nvtx_range("wl_apply");
  if (!ctx || !G || !in || !out) WL_FAIL(ctx, WL_ERR_ARG, "null argument");
  if (in == out) WL_FAIL(ctx, WL_ERR_ARG, "in and out must not alias");
  if (nrhs <= 0) WL_FAIL(ctx, WL_ERR_ARG, "nrhs must be positive");
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  const Geom& g = ctx->g;
  const double m0 = mass + 4.0;
  const size_t fbytes = (size_t)nrhs * g.V * 12 * sizeof(double2);
  const bool norm = (flags & WL_FLAG_NORMALIZED) != 0;
  cudaStream_t st = ctx->stream;
  switch (op) {
    case WL_OP_D: ref_hop<false>(ctx, G, in, out, in, m0, -0.5, nrhs, 0, 2); break;
    case WL_OP_DDAG: ref_hop<true>(ctx, G, in, out, in, m0, -0.5, nrhs, 0, 2); break;
    case WL_OP_HOP: ref_hop<false>(ctx, G, in, out, nullptr, 0.0, -0.5, nrhs, 0, 2); break;
    case WL_OP_HOP_DAG: ref_hop<true>(ctx, G, in, out, nullptr, 0.0, -0.5, nrhs, 0, 2); break;
    case WL_OP_DDAGD: {
      wl_status s = ensure_tmp(ctx, fbytes);
      if (s != WL_OK) return s;
      ref_hop<false>(ctx, G, in, ctx->tmp, in, m0, -0.5, nrhs, 0, 2);
      ref_hop<true>(ctx, G, ctx->tmp, out, ctx->tmp, m0, -0.5, nrhs, 0, 2);
      break;
    }
    case WL_OP_K_OE:
    case WL_OP_K_EO:
    case WL_OP_KDAG_OE:
    case WL_OP_KDAG_EO: {
      const int target = (op == WL_OP_K_OE || op == WL_OP_KDAG_OE) ? 1 : 0;
      WL_CUDA(ctx, cudaMemsetAsync(out, 0, fbytes, st));
      if (op == WL_OP_K_OE || op == WL_OP_K_EO) ref_hop<false>(ctx, G, in, out, nullptr, 0.0, -0.5, nrhs, target, 1);
      else ref_hop<true>(ctx, G, in, out, nullptr, 0.0, -0.5, nrhs, target, 1);
      break;
    }
    case WL_OP_SCHUR_E:
    case WL_OP_SCHUR_E_DAG:
    case WL_OP_SCHUR_O: {
      // t = K_{p'p} x_p (target p' = 1-p); out_p = c0 x_p + c1 * hop(t)
      const int p = (op == WL_OP_SCHUR_O) ? 1 : 0;
      const bool dag = (op == WL_OP_SCHUR_E_DAG);
      wl_status s = ensure_tmp(ctx, fbytes);
      if (s != WL_OK) return s;
      WL_CUDA(ctx, cudaMemsetAsync(out, 0, fbytes, st));
      const double c0 = norm ? 1.0 : m0;
      const double c1 = norm ? 0.5 / (m0 * m0) : 0.5 / m0;
      if (dag) {
        ref_hop<true>(ctx, G, in, ctx->tmp, nullptr, 0.0, -0.5, nrhs, 1 - p, 1);
        ref_hop<true>(ctx, G, ctx->tmp, out, in, c0, c1, nrhs, p, 1);
      } else {
        ref_hop<false>(ctx, G, in, ctx->tmp, nullptr, 0.0, -0.5, nrhs, 1 - p, 1);
        ref_hop<false>(ctx, G, ctx->tmp, out, in, c0, c1, nrhs, p, 1);
      }
      break;
    }
    case WL_OP_SCHUR_E_NORMAL: {
      // out = S^dag S x (normalized or not), via two Schur applications
      wl_status s = ensure_tmp(ctx, 2 * fbytes);
      if (s != WL_OK) return s;
      void* t1 = ctx->tmp;
      void* y = (char*)ctx->tmp + fbytes;
      WL_CUDA(ctx, cudaMemsetAsync(y, 0, fbytes, st));
      WL_CUDA(ctx, cudaMemsetAsync(out, 0, fbytes, st));
      const double c0 = norm ? 1.0 : m0;
      const double c1 = norm ? 0.5 / (m0 * m0) : 0.5 / m0;
      ref_hop<false>(ctx, G, in, t1, nullptr, 0.0, -0.5, nrhs, 1, 1);
      ref_hop<false>(ctx, G, t1, y, in, c0, c1, nrhs, 0, 1);
      ref_hop<true>(ctx, G, y, t1, nullptr, 0.0, -0.5, nrhs, 1, 1);
      ref_hop<true>(ctx, G, t1, out, y, c0, c1, nrhs, 0, 1);
      break;
    }
    default: WL_FAIL(ctx, WL_ERR_ARG, "unknown operator");
  }
  return check_launch(ctx, "wl_apply");
}

// ============================================================== field inner products / combinations
static wl_status ensure_red(wl_ctx* ctx, size_t bytes);

extern "C" wl_status wl_field_dots(wl_ctx* ctx, int npairs, const void* const* a, const void* const* b, int64_t len,
                                   double* out) {
  NvtxRange nvtx_range("wl_field_dots");
  if (!ctx || !a || !b || !out) WL_FAIL(ctx, WL_ERR_ARG, "null argument");
  if (npairs <= 0 || npairs > kMaxFieldPairs) WL_FAIL(ctx, WL_ERR_ARG, "npairs must be in 1..64");
  if (len <= 0) WL_FAIL(ctx, WL_ERR_ARG, "len must be positive");
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  DotsArgs A{};
  for (int k = 0; k < npairs; ++k) {
    if (!a[k] || !b[k]) WL_FAIL(ctx, WL_ERR_ARG, "null field pointer");
    A.a[k] = (const double2*)a[k];
    A.b[k] = (const double2*)b[k];
  }
  A.len = len;
  const int nblk = (int)std::min<long long>((len + kBlasThreads - 1) / kBlasThreads, 4LL * ctx->sm_count);
  wl_status s = ensure_red(ctx, sizeof(double2) * ((size_t)npairs * nblk + npairs));
  if (s != WL_OK) return s;
  A.partials = (double2*)ctx->red;
  A.result = A.partials + (size_t)npairs * nblk;
  g_launches += 2;
  field_dots_kernel<<<dim3(nblk, npairs), kBlasThreads, 0, ctx->stream>>>(A);
  field_dots_finalize_kernel<<<npairs, kBlasThreads, 0, ctx->stream>>>(A, nblk);
  WL_CUDA(ctx, cudaMemcpyAsync(out, A.result, sizeof(double2) * npairs, cudaMemcpyDeviceToHost, ctx->stream));
  WL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return check_launch(ctx, "field_dots_kernel");
}

extern "C" wl_status wl_field_combine(wl_ctx* ctx, int n, const void* const* x, const double* coef, int64_t len,
                                      void* out) {
  NvtxRange nvtx_range("wl_field_combine");
  if (!ctx || !x || !coef || !out) WL_FAIL(ctx, WL_ERR_ARG, "null argument");
  if (n <= 0 || n > kMaxCombine) WL_FAIL(ctx, WL_ERR_ARG, "n must be in 1..32");
  if (len <= 0) WL_FAIL(ctx, WL_ERR_ARG, "len must be positive");
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  CombineArgs A{};
  for (int k = 0; k < n; ++k) {
    if (!x[k]) WL_FAIL(ctx, WL_ERR_ARG, "null field pointer");
    A.x[k] = (const double2*)x[k];
    A.c[k] = make_double2(coef[2 * k], coef[2 * k + 1]);
  }
  A.n = n;
  A.len = len;
  A.out = (double2*)out;
  const int nblk = (int)std::min<long long>((len + kBlasThreads - 1) / kBlasThreads, 8LL * ctx->sm_count);
  g_launches++;
  field_combine_kernel<<<nblk, kBlasThreads, 0, ctx->stream>>>(A);
  return check_launch(ctx, "field_combine_kernel");
}

// ============================================================== random fields
static wl_status launch_rng(wl_ctx* ctx, bool spinor, uint64_t seed, uint64_t stream, int nfield, double scale,
                            void* out) {
  if (!ctx || !out) WL_FAIL(ctx, WL_ERR_ARG, "null argument");
  if (nfield <= 0 || nfield > 65535) WL_FAIL(ctx, WL_ERR_ARG, "field count out of range");
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  RngArgs A{};
  A.seed = seed;
  A.stream = stream;
  A.n_elem = spinor ? (long long)ctx->g.V : 4LL * ctx->g.V;
  A.nfield = nfield;
  A.scale = scale;
  A.out = (double2*)out;
  const dim3 grid((unsigned)((A.n_elem + 255) / 256), (unsigned)nfield);
  g_launches++;
  if (spinor) rng_spinor_kernel<<<grid, 256, 0, ctx->stream>>>(A);
  else rng_algebra_kernel<<<grid, 256, 0, ctx->stream>>>(A);
  return check_launch(ctx, spinor ? "rng_spinor_kernel" : "rng_algebra_kernel");
}

extern "C" wl_status wl_random_spinor(wl_ctx* ctx, uint64_t seed, uint64_t stream, int n, void* out) {
  NvtxRange nvtx_range("wl_random_spinor");
  return launch_rng(ctx, true, seed, stream, n, 1.0, out);
}

extern "C" wl_status wl_random_algebra(wl_ctx* ctx, uint64_t seed, uint64_t stream, int batch, double scale,
                                       void* P) {
  NvtxRange nvtx_range("wl_random_algebra");
  return launch_rng(ctx, false, seed, stream, batch, scale, P);
}

// ============================================================== force
extern "C" wl_status wl_pf_force(wl_ctx* ctx, wl_gauge* G, const void* X, const void* Y, double coef, int accumulate,
                                 void* F) {
  NvtxRange nvtx_range("wl_pf_force");
  if (!ctx || !G || !X || !Y || !F) WL_FAIL(ctx, WL_ERR_ARG, "null argument");
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  const Geom& g = ctx->g;
  ForceArgs A;
  A.g = g;
  A.U.ptr = G->ref_copy;
  A.U.V = g.V;
  A.X = sref(X, g);
  A.Y = sref(Y, g);
  A.F = (double2*)F;
  A.coef = coef;
  A.accumulate = accumulate;
  dim3 grid((g.Vh + 127) / 128, 2, 4);
  g_launches++;
  pf_force_kernel<<<grid, 128, 0, ctx->stream>>>(A);
  return check_launch(ctx, "pf_force_kernel");
}

// ============================================================== gauge sector
static wl_status ensure_red(wl_ctx* ctx, size_t bytes) {
  if (ctx->red_bytes >= bytes) return WL_OK;
  if (ctx->red) {
    cudaFree(ctx->red);
    ctx->red = nullptr;
    ctx->red_bytes = 0;
  }
  WL_CUDA(ctx, cudaMalloc(&ctx->red, bytes));
  ctx->red_bytes = bytes;
  return WL_OK;
}

// Sum of per-block partials [batch][nblk] -> host out[batch] (fixed order).
static wl_status finish_sums(wl_ctx* ctx, int batch, int nblk, double scale, double* out) {
  Reduce r{};
  r.partials = ctx->red;
  r.result = ctx->red + (size_t)batch * nblk;
  g_launches++;
  reduce_finalize_kernel<<<batch, kFinalizeThreads, 0, ctx->stream>>>(r, batch, nblk, nullptr);
  wl_status s = check_launch(ctx, "reduce_finalize_kernel");
  if (s != WL_OK) return s;
  std::vector<double> h(batch);
  WL_CUDA(ctx, cudaMemcpyAsync(h.data(), r.result, sizeof(double) * batch, cudaMemcpyDeviceToHost, ctx->stream));
  WL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int b = 0; b < batch; ++b) out[b] = scale * h[b];
  return WL_OK;
}

static GaugeArgs gauge_args(wl_ctx* ctx, const void* U, const void* P, void* out, int batch, double coef) {
  GaugeArgs A{};
  A.g = ctx->g;
  A.U = (const double2*)U;
  A.P = (const double2*)P;
  A.out = (double2*)out;
  A.batch = batch;
  A.coef = coef;
  A.partials = ctx->red;
  return A;
}

extern "C" wl_status wl_gauge_force(wl_ctx* ctx, const void* U, int batch, double beta, void* F) {
  NvtxRange nvtx_range("wl_gauge_force");
  if (!ctx || !U || !F || batch < 1) WL_FAIL(ctx, WL_ERR_ARG, "null argument or batch < 1");
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  GaugeArgs A = gauge_args(ctx, U, nullptr, F, batch, -beta / 3.0);
  dim3 grid((ctx->g.V + 127) / 128, 4, batch);
  g_launches++;
  gauge_force_kernel<<<grid, 128, 0, ctx->stream>>>(A);
  return check_launch(ctx, "gauge_force_kernel");
}

extern "C" wl_status wl_gauge_evolve(wl_ctx* ctx, const void* P, const void* U, int batch, double dt, void* Uout) {
  NvtxRange nvtx_range("wl_gauge_evolve");
  if (!ctx || !P || !U || !Uout || batch < 1) WL_FAIL(ctx, WL_ERR_ARG, "null argument or batch < 1");
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  GaugeArgs A = gauge_args(ctx, U, P, Uout, batch, dt);
  const long long nl = (long long)batch * 4 * ctx->g.V;
  g_launches++;
  gauge_evolve_kernel<<<(unsigned)((nl + 127) / 128), 128, 0, ctx->stream>>>(A);
  return check_launch(ctx, "gauge_evolve_kernel");
}

extern "C" wl_status wl_gauge_plaquette_sum(wl_ctx* ctx, const void* U, int batch, double* plaq_sum) {
  NvtxRange nvtx_range("wl_gauge_plaquette_sum");
  if (!ctx || !U || !plaq_sum || batch < 1) WL_FAIL(ctx, WL_ERR_ARG, "null argument or batch < 1");
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  const int nblk = (ctx->g.V + 127) / 128;
  wl_status s = ensure_red(ctx, sizeof(double) * ((size_t)batch * nblk + batch));
  if (s != WL_OK) return s;
  GaugeArgs A = gauge_args(ctx, U, nullptr, nullptr, batch, 0.0);
  g_launches++;
  gauge_plaquette_kernel<<<dim3(nblk, 1, batch), 128, 0, ctx->stream>>>(A);
  s = check_launch(ctx, "gauge_plaquette_kernel");
  if (s != WL_OK) return s;
  return finish_sums(ctx, batch, nblk, 1.0, plaq_sum);
}

extern "C" wl_status wl_momentum_kinetic(wl_ctx* ctx, const void* P, int batch, double* kin) {
  NvtxRange nvtx_range("wl_momentum_kinetic");
  if (!ctx || !P || !kin || batch < 1) WL_FAIL(ctx, WL_ERR_ARG, "null argument or batch < 1");
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  const int nblk = (int)((4LL * ctx->g.V + 127) / 128);
  wl_status s = ensure_red(ctx, sizeof(double) * ((size_t)batch * nblk + batch));
  if (s != WL_OK) return s;
  GaugeArgs A = gauge_args(ctx, nullptr, P, nullptr, batch, 0.0);
  g_launches++;
  gauge_kinetic_kernel<<<dim3(nblk, 1, batch), 128, 0, ctx->stream>>>(A);
  s = check_launch(ctx, "gauge_kinetic_kernel");
  if (s != WL_OK) return s;
  return finish_sums(ctx, batch, nblk, 1.0, kin);
}

extern "C" wl_status wl_pion_correlator(wl_ctx* ctx, const void* prop, int ncol, int source_t, double* corr) {
  NvtxRange nvtx_range("wl_pion_correlator");
  if (!ctx || !prop || !corr || ncol < 1) WL_FAIL(ctx, WL_ERR_ARG, "null argument or ncol < 1");
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  const Geom& g = ctx->g;
  const int Lt = g.L[3];
  const int nblk = (g.V / Lt + 127) / 128;
  wl_status s = ensure_red(ctx, sizeof(double) * ((size_t)Lt * nblk + Lt));
  if (s != WL_OK) return s;
  PionArgs A{(const double2*)prop, ncol, g.V, Lt, ctx->red};
  g_launches++;
  pion_kernel<<<dim3(nblk, Lt, 1), 128, 0, ctx->stream>>>(A);
  s = check_launch(ctx, "pion_kernel");
  if (s != WL_OK) return s;
  std::vector<double> c(Lt);
  s = finish_sums(ctx, Lt, nblk, 1.0, c.data());
  if (s != WL_OK) return s;
  const int t0 = ((source_t % Lt) + Lt) % Lt;
  for (int t = 0; t < Lt; ++t) corr[(t - t0 + Lt) % Lt] = c[t];
  return WL_OK;
}

// ============================================================== CG engine
namespace {

struct TuneKey {
  int vh, prec, nslots, op;
  bool operator<(const TuneKey& o) const {
    return std::tie(vh, prec, nslots, op) < std::tie(o.vh, o.prec, o.nslots, o.op);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, Tune> g_tune_cache;

}  // namespace

struct wl_engine {
  wl_ctx* ctx = nullptr;
  wl_gauge* gauge = nullptr;
  unsigned long long gauge_id = 0;  // id of the gauge the graph was captured with
  wl_solve_params prm;
  int n = 0;        // slots
  int npar = 1;     // 1 for EO (even fields), 2 for full lattice
  int sprec = 0;
  bool lanes_mode = false;  // sloppy fields RHS-innermost, sloppy hops with RHS in the lanes
  Tune ts, td, tsite;  // sloppy hop, FP64 hop, site kernels
  // fields
  IField b64, x64, y64, t64;  // FP64
  IField xs, rs, p, y, t1;    // sloppy (t1 reused for t2)
  // scalars (device)
  double* dbl = nullptr;
  int* ints = nullptr;
  double *r2, *r2_new, *pAp, *r2_true, *rmax2, *b2, *tol2, *beta, *one, *neg_half, *half_alpha, *m0, *alpha;
  int *active, *ru, *iters, *maxiter, *status, *n_ru, *n_active, *admit;
  // host mirrors of parameters
  std::vector<double> h_tol2, h_one, h_neg_half, h_half_alpha, h_m0;
  std::vector<int> h_maxiter, h_admit;
  int* h_pinned = nullptr;
  cudaEvent_t poll_ev = nullptr;  // recorded after the copies of wl_engine_poll_async
  bool poll_pending = false;
  // reductions
  double* partials = nullptr;
  unsigned* counters = nullptr;
  // graph
  cudaGraphExec_t gexec = nullptr;
  bool graph_built = false;
  long long graph_kernels = 0;     // unconditional kernel nodes per captured iteration
  long long ru_body_kernels = 0;   // kernels in the conditional reliable-update body
  bool use_cond = false;           // decide kernel drives a graph conditional node
  cudaGraphConditionalHandle cond = 0;
  int* ru_iters = nullptr;         // device: iterations whose conditional body ran
  long long ru_iters_seen = 0;
  // the solve as one graph (WHILE node over the iteration), launched once per wl_solve
  cudaGraphExec_t gloop = nullptr;
  int* loop_count = nullptr;       // device: iterations run by the loop graph's current launch
  long long loop_kernels = 0;      // unconditional kernels per loop iteration
  int loop_cap = 0;                // maxiter the loop graph was built for
  unsigned long long loop_gauge_id = 0;
  bool loop_failed = false;        // the loop graph could not be built: host-driven loop
  const SolveLoop* capture_loop = nullptr;  // set while part 3 of a loop body is captured
  // engine run (wl_engine_run): WHILE node that stops when a slot finishes or at a per-launch cap
  cudaGraphExec_t grun = nullptr;
  int* run_state = nullptr;        // device: [0] cap, [1] active count at launch start, [2] iterations
  long long run_kernels = 0;       // unconditional kernels per run iteration
  long long run_seen = 0;          // run iterations already counted into g_launches
  unsigned long long run_gauge_id = 0;
  bool run_failed = false;
  bool ru_links12 = false;         // FP64 true residual with 12-real links (links unitary to 1e-12)
};

struct EngineStream {
  cudaStream_t st;
};
static std::map<const wl_engine*, cudaStream_t> g_engine_streams;
static std::mutex g_es_mu;

static cudaStream_t engine_stream(const wl_engine* E) {
  std::lock_guard<std::mutex> lk(g_es_mu);
  return g_engine_streams[E];
}

static const int kEngineDoubles = 13;
static const int kEngineInts = 8;

int64_t engine_bytes_impl(const Geom& g, int op, int sprec, int n) {
  const int npar = (op == WL_SOLVE_EO_NORMAL) ? 1 : 2;
  int64_t b = 0;
  b += 3 * (int64_t)field_bytes(P_DOUBLE, g.Vh, n, npar);                // b64, x64, y64
  b += (int64_t)field_bytes(P_DOUBLE, g.Vh, n, op == WL_SOLVE_EO_NORMAL ? 1 : 2);  // t64
  b += 4 * (int64_t)field_bytes(sprec, g.Vh, n, npar);                   // xs, rs, p, y
  b += (int64_t)field_bytes(sprec, g.Vh, n, 1);                          // t1
  b += (int64_t)n * (g.Vh + 64) * sizeof(double) + 4096;
  return b;
}

static int64_t hop_bytes(const Geom& g, int sprec, int nrhs) {
  // one EO hop: 8 links per target site (4 fwd own parity + 4 bwd other) and,
  // per RHS, one source spinor and one output spinor per site.
  const double L = sprec == P_DOUBLE ? 144.0 : (sprec == P_SINGLE ? 48.0 : 24.0);
  const double S = sprec == P_DOUBLE ? 192.0 : (sprec == P_SINGLE ? 96.0 : 52.0);
  return (int64_t)((double)g.Vh * (8.0 * L + nrhs * 2.0 * S));
}

extern "C" int64_t wl_engine_bytes(const wl_ctx* ctx, int op, int inner_prec, int nslots) {
  if (!ctx) return -1;
  return engine_bytes_impl(ctx->g, op, inner_prec, nslots);
}

static Reduce red_to(wl_engine* E, double* result) {
  Reduce r{};
  r.partials = E->partials;
  r.counter = E->counters;
  r.result = result;
  return r;
}

// Site functors that touch only sloppy fields follow the sloppy layout.
template <class F>
static void launch_site_sloppy(wl_engine* E, int parity0, int npar, int nrhs, const int* mask, const F& f, Reduce red,
                               cudaStream_t st) {
  if (E->lanes_mode) launch_site_lanes(E->ts.lanes > 0 ? E->ts.lanes : 16, E->ctx->g, parity0, npar, nrhs, mask, f,
                                       red, st);
  else launch_site(E->tsite, E->ctx->g, parity0, npar, nrhs, mask, f, red, st);
}

__global__ void admit_state_kernel(CGScalars S, const int* admit, int use_x0, int n) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int local = 0;
  for (int s = threadIdx.x; s < n; s += blockDim.x) {
    if (admit[s]) {
      S.iters[s] = 0;
      S.n_ru[s] = 0;
      const double r2 = use_x0 ? S.r2_true[s] : S.b2[s];
      S.r2[s] = r2;
      S.rmax2[s] = r2;
      S.beta[s] = 0.0;
      if (!(S.b2[s] > 0.0) || r2 <= S.tol2[s] * S.b2[s]) {
        S.active[s] = 0;
        S.status[s] = ST_CONVERGED;
      } else if (!isfinite(r2)) {
        S.active[s] = 0;
        S.status[s] = ST_NAN;
      } else {
        S.active[s] = 1;
        S.status[s] = ST_RUNNING;
      }
    }
    local += S.active[s];
  }
  atomicAdd(&cnt, local);
  __syncthreads();
  if (threadIdx.x == 0) *S.n_active = cnt;
}

// Maps admitted slot -> index in the caller's b buffer
struct FPackMapped {
  static constexpr bool kReduce = true;
  Geom g;
  SpinorRef in;
  const int* map;
  SpinorField<P_DOUBLE> out[2];
  WL_D double operator()(int rhs, int parity, int c) const {
    const long long f = flat_of(g, parity, c);
    Spinor<double> s;
    in.load(s, map[rhs], f);
    out[parity].store(s, rhs, c);
    return snorm2(s);
  }
};

static CGScalars scalars_of(wl_engine* E) {
  CGScalars S;
  S.r2 = E->r2;
  S.r2_new = E->r2_new;
  S.pAp = E->pAp;
  S.r2_true = E->r2_true;
  S.rmax2 = E->rmax2;
  S.b2 = E->b2;
  S.tol2 = E->tol2;
  S.beta = E->beta;
  S.active = E->active;
  S.ru = E->ru;
  S.iters = E->iters;
  S.maxiter = E->maxiter;
  S.status = E->status;
  S.n_ru = E->n_ru;
  S.n_active = E->n_active;
  S.delta2 = E->prm.delta * E->prm.delta;
  return S;
}

template <int S> struct SloppyLinks;
template <> struct SloppyLinks<P_DOUBLE> {
  using type = LinkField<L_D18>;
  static type get(wl_gauge* G) { return type{G->d18, G->ctx->g.Vh}; }
};
template <> struct SloppyLinks<P_SINGLE> {
  using type = LinkField<L_S12>;
  static type get(wl_gauge* G) { return type{G->s12, G->ctx->g.Vh}; }
};
template <> struct SloppyLinks<P_HALF> {
  using type = LinkField<L_H12>;
  static type get(wl_gauge* G) { return type{G->h12, G->ctx->g.Vh}; }
};

template <int S>
static void time_hop_impl(wl_engine* E, cudaStream_t st, int reps, float* ms) {
  using SFS = SpinorField<S>;
  using LS = typename SloppyLinks<S>::type;
  HopArgs<LS, SFS, EpiXpay<SFS, false>> A{};
  A.g = E->ctx->g;
  A.links = SloppyLinks<S>::get(E->gauge);
  sf2<S>(E->p, A.src);
  A.parity0 = 1;
  A.nrhs = E->n;
  A.mask = nullptr;
  sf2<S>(E->t1, A.epi.out);
  A.epi.has_self = 0;
  A.epi.b = E->neg_half;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  launch_hop<false, IdxCompact>(E->ts, A, 1, st);
  cudaEventRecord(e0, st);
  for (int i = 0; i < reps; ++i) launch_hop<false, IdxCompact>(E->ts, A, 1, st);
  cudaEventRecord(e1, st);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
}

// The fused CG hop, timed like time_hop_impl: the fourth hop of an iteration (M^dag y for the
// EO operator, D^dag y for the full one) with the CG update in its epilogue (x_s += alpha p,
// r_s -= alpha A p, |r_s|^2 partials) over all slots, the kernel alone (no finalize).  It
// updates x_s and r_s in place, so the slots must be admitted again before they iterate.
template <int S>
static void time_cg_hop_impl(wl_engine* E, cudaStream_t st, int reps, float* ms) {
  using SFS = SpinorField<S>;
  using LS = typename SloppyLinks<S>::type;
  const bool eo = E->prm.op == WL_SOLVE_EO_NORMAL;
  HopArgs<LS, SFS, EpiCG<SFS>> A{};
  A.g = E->ctx->g;
  A.links = SloppyLinks<S>::get(E->gauge);
  sf2<S>(eo ? E->t1 : E->y, A.src);
  A.parity0 = 0;
  A.nrhs = E->n;
  A.mask = nullptr;
  sf2<S>(E->y, A.epi.y);
  sf2<S>(E->p, A.epi.p);
  sf2<S>(E->xs, A.epi.xs);
  sf2<S>(E->rs, A.epi.rs);
  A.epi.a = eo ? E->one : E->m0;
  A.epi.b = eo ? E->half_alpha : E->neg_half;
  A.epi.r2 = E->r2;
  A.epi.pAp = E->pAp;
  A.epi.alpha = E->alpha;
  A.red = red_to(E, E->r2_new);
  const int npar = eo ? 1 : 2;
  const Tune t = effective_tune<IdxCompact, SFS, EpiCG<SFS>>(E->ts);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  launch_hop_impl<true, IdxCompact>(t, A, npar, st);
  cudaEventRecord(e0, st);
  for (int i = 0; i < reps; ++i) launch_hop_impl<true, IdxCompact>(t, A, npar, st);
  cudaEventRecord(e1, st);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
}

// Enqueue the FP64 normal operator on x64 ending in the true residual
// rs = convert(b - A x64), r2_true = |b - A x64|^2, for the slots in `mask`.
template <int S, class LDT>
static void enqueue_true_residual_links(wl_engine* E, const int* mask, cudaStream_t st, const LDT& LD) {
  using SFS = SpinorField<S>;
  using SFD = SpinorField<P_DOUBLE>;
  const Geom& g = E->ctx->g;
  const bool eo = E->prm.op == WL_SOLVE_EO_NORMAL;
  if (eo) {
    {  // t64 = K_oe x64
      HopArgs<LDT, SFD, EpiXpay<SFD, false>> A{};
      A.g = g; A.links = LD; sf2<P_DOUBLE>(E->x64, A.src); A.parity0 = 1; A.nrhs = E->n; A.mask = mask;
      sf2<P_DOUBLE>(E->t64, A.epi.out); A.epi.has_self = 0; A.epi.b = E->neg_half;
      launch_hop<false, IdxCompact>(E->td, A, 1, st);
    }
    {  // y64 = x64 + (alpha/2) hop(t64)
      HopArgs<LDT, SFD, EpiXpay<SFD, false>> A{};
      A.g = g; A.links = LD; sf2<P_DOUBLE>(E->t64, A.src); A.parity0 = 0; A.nrhs = E->n; A.mask = mask;
      sf2<P_DOUBLE>(E->y64, A.epi.out); sf2<P_DOUBLE>(E->x64, A.epi.self); A.epi.has_self = 1;
      A.epi.a = E->one; A.epi.b = E->half_alpha;
      launch_hop<false, IdxCompact>(E->td, A, 1, st);
    }
    {  // t64 = Kdag_oe y64
      HopArgs<LDT, SFD, EpiXpay<SFD, false>> A{};
      A.g = g; A.links = LD; sf2<P_DOUBLE>(E->y64, A.src); A.parity0 = 1; A.nrhs = E->n; A.mask = mask;
      sf2<P_DOUBLE>(E->t64, A.epi.out); A.epi.has_self = 0; A.epi.b = E->neg_half;
      launch_hop<true, IdxCompact>(E->td, A, 1, st);
    }
    {  // rs = b - (y64 + (alpha/2) hopdag(t64))
      HopArgs<LDT, SFD, EpiResid<SFS>> A{};
      A.g = g; A.links = LD; sf2<P_DOUBLE>(E->t64, A.src); A.parity0 = 0; A.nrhs = E->n; A.mask = mask;
      sf2<P_DOUBLE>(E->y64, A.epi.y); sf2<P_DOUBLE>(E->b64, A.epi.bvec); sf2<S>(E->rs, A.epi.rs);
      A.epi.a = E->one; A.epi.b = E->half_alpha;
      A.red = red_to(E, E->r2_true);
      launch_hop<true, IdxCompact>(E->td, A, 1, st);
    }
  } else {
    {  // y64 = D x64
      HopArgs<LDT, SFD, EpiXpay<SFD, false>> A{};
      A.g = g; A.links = LD; sf2<P_DOUBLE>(E->x64, A.src); A.parity0 = 0; A.nrhs = E->n; A.mask = mask;
      sf2<P_DOUBLE>(E->y64, A.epi.out); sf2<P_DOUBLE>(E->x64, A.epi.self); A.epi.has_self = 1;
      A.epi.a = E->m0; A.epi.b = E->neg_half;
      launch_hop<false, IdxCompact>(E->td, A, 2, st);
    }
    {  // rs = b - D^dag y64
      HopArgs<LDT, SFD, EpiResid<SFS>> A{};
      A.g = g; A.links = LD; sf2<P_DOUBLE>(E->y64, A.src); A.parity0 = 0; A.nrhs = E->n; A.mask = mask;
      sf2<P_DOUBLE>(E->y64, A.epi.y); sf2<P_DOUBLE>(E->b64, A.epi.bvec); sf2<S>(E->rs, A.epi.rs);
      A.epi.a = E->m0; A.epi.b = E->neg_half;
      A.red = red_to(E, E->r2_true);
      launch_hop<true, IdxCompact>(E->td, A, 2, st);
    }
  }
}

template <int S>
static void enqueue_true_residual(wl_engine* E, const int* mask, cudaStream_t st) {
  const Geom& g = E->ctx->g;
  if (E->ru_links12) enqueue_true_residual_links<S>(E, mask, st, LinkField<L_D12>{E->gauge->d12, g.Vh});
  else enqueue_true_residual_links<S>(E, mask, st, LinkField<L_D18>{E->gauge->d18, g.Vh});
}

// One CG iteration for all active slots, in three parts: (1) the sloppy
// normal operator with the fused CG update and the reliable-update decision,
// (2) the reliable update (x += x_s; r = b - A x in FP64) for the slots that
// take one, (3) convergence bookkeeping and p = r + beta p.  In a CUDA graph,
// part 2 sits in a conditional node that runs only when some slot needs it.
template <int S>
static void enqueue_iteration(wl_engine* E, cudaStream_t st, int part) {
  using SFS = SpinorField<S>;
  using LS = typename SloppyLinks<S>::type;
  const Geom& g = E->ctx->g;
  LS L = SloppyLinks<S>::get(E->gauge);
  const bool eo = E->prm.op == WL_SOLVE_EO_NORMAL;
  const int n = E->n;
  CGScalars Sc = scalars_of(E);
  if (part == 2) {
    {  // x64 += xs ; xs = 0  (reliable-update slots)
      FAccumX<SFS> f;
      sf2<P_DOUBLE>(E->x64, f.x);
      sf2<S>(E->xs, f.xs);
      launch_site_sloppy(E, 0, E->npar, n, E->ru, f, Reduce{}, st);
    }
    enqueue_true_residual<S>(E, E->ru, st);
    return;
  }
  if (part == 3) {
    g_launches++;
    cg_finalize_kernel<<<1, 128, 0, st>>>(Sc, n, E->capture_loop ? *E->capture_loop : SolveLoop{});
    FUpdateP<SFS> f;  // p = rs + beta p
    sf2<S>(E->rs, f.rs);
    sf2<S>(E->p, f.p);
    f.beta = E->beta;
    launch_site_sloppy(E, 0, E->npar, n, E->active, f, Reduce{}, st);
    return;
  }
  if (eo) {
    {  // t1 = K_oe p
      HopArgs<LS, SFS, EpiXpay<SFS, false>> A{};
      A.g = g; A.links = L; sf2<S>(E->p, A.src); A.parity0 = 1; A.nrhs = n; A.mask = E->active;
      sf2<S>(E->t1, A.epi.out); A.epi.has_self = 0; A.epi.b = E->neg_half;
      launch_hop<false, IdxCompact>(E->ts, A, 1, st);
    }
    {  // y = p + (alpha/2) hop(t1) = M p ; pAp = |y|^2
      HopArgs<LS, SFS, EpiXpay<SFS, true>> A{};
      A.g = g; A.links = L; sf2<S>(E->t1, A.src); A.parity0 = 0; A.nrhs = n; A.mask = E->active;
      sf2<S>(E->y, A.epi.out); sf2<S>(E->p, A.epi.self); A.epi.has_self = 1;
      A.epi.a = E->one; A.epi.b = E->half_alpha;
      A.red = red_to(E, E->pAp);
      A.red.num = E->r2;
      A.red.quot = E->alpha;  // alpha = r2 / pAp for the fused CG update
      launch_hop<false, IdxCompact>(E->ts, A, 1, st);
    }
    {  // t2 = Kdag_oe y
      HopArgs<LS, SFS, EpiXpay<SFS, false>> A{};
      A.g = g; A.links = L; sf2<S>(E->y, A.src); A.parity0 = 1; A.nrhs = n; A.mask = E->active;
      sf2<S>(E->t1, A.epi.out); A.epi.has_self = 0; A.epi.b = E->neg_half;
      launch_hop<true, IdxCompact>(E->ts, A, 1, st);
    }
    {  // Ap = M^dag y ; CG update
      HopArgs<LS, SFS, EpiCG<SFS>> A{};
      A.g = g; A.links = L; sf2<S>(E->t1, A.src); A.parity0 = 0; A.nrhs = n; A.mask = E->active;
      sf2<S>(E->y, A.epi.y); sf2<S>(E->p, A.epi.p); sf2<S>(E->xs, A.epi.xs); sf2<S>(E->rs, A.epi.rs);
      A.epi.a = E->one; A.epi.b = E->half_alpha; A.epi.r2 = E->r2; A.epi.pAp = E->pAp; A.epi.alpha = E->alpha;
      A.red = red_to(E, E->r2_new);
      launch_hop<true, IdxCompact>(E->ts, A, 1, st);
    }
  } else {
    {  // y = D p ; pAp = |y|^2
      HopArgs<LS, SFS, EpiXpay<SFS, true>> A{};
      A.g = g; A.links = L; sf2<S>(E->p, A.src); A.parity0 = 0; A.nrhs = n; A.mask = E->active;
      sf2<S>(E->y, A.epi.out); sf2<S>(E->p, A.epi.self); A.epi.has_self = 1;
      A.epi.a = E->m0; A.epi.b = E->neg_half;
      A.red = red_to(E, E->pAp);
      A.red.num = E->r2;
      A.red.quot = E->alpha;  // alpha = r2 / pAp for the fused CG update
      launch_hop<false, IdxCompact>(E->ts, A, 2, st);
    }
    {  // Ap = D^dag y ; CG update
      HopArgs<LS, SFS, EpiCG<SFS>> A{};
      A.g = g; A.links = L; sf2<S>(E->y, A.src); A.parity0 = 0; A.nrhs = n; A.mask = E->active;
      sf2<S>(E->y, A.epi.y); sf2<S>(E->p, A.epi.p); sf2<S>(E->xs, A.epi.xs); sf2<S>(E->rs, A.epi.rs);
      A.epi.a = E->m0; A.epi.b = E->neg_half; A.epi.r2 = E->r2; A.epi.pAp = E->pAp; A.epi.alpha = E->alpha;
      A.red = red_to(E, E->r2_new);
      launch_hop<true, IdxCompact>(E->ts, A, 2, st);
    }
  }
  g_launches++;
  cg_decide_kernel<<<1, 128, 0, st>>>(Sc, n, E->use_cond ? 1 : 0, E->cond, E->use_cond ? E->ru_iters : nullptr,
                                      E->lanes_mode ? 1 : 0);
}

template <int S>
static void enqueue_admit(wl_engine* E, const void* b, int use_x0, const void* x0, const int* map_dev,
                          cudaStream_t st) {
  using SFS = SpinorField<S>;
  using SFD = SpinorField<P_DOUBLE>;
  const Geom& g = E->ctx->g;
  const int n = E->n;
  const int* adm = E->admit;
  const int par0 = 0;
  {  // b64 <- b ; b2
    FPackMapped f;
    f.g = g;
    f.in = sref(b, g);
    f.map = map_dev;
    sf2<P_DOUBLE>(E->b64, f.out);
    launch_site(E->tsite, g, par0, E->npar, n, adm, f, red_to(E, E->b2), st);
  }
  if (use_x0) {
    FPackMapped f;
    f.g = g;
    f.in = sref(x0, g);
    f.map = map_dev;
    sf2<P_DOUBLE>(E->x64, f.out);
    launch_site(E->tsite, g, par0, E->npar, n, adm, f, red_to(E, E->r2_true), st);
    enqueue_true_residual<S>(E, adm, st);
  } else {
    FZero<SFD> z;
    sf2<P_DOUBLE>(E->x64, z.out);
    launch_site(E->tsite, g, par0, E->npar, n, adm, z, Reduce{}, st);
    FConvert<SFD, SFS> cv;
    sf2<P_DOUBLE>(E->b64, cv.in);
    sf2<S>(E->rs, cv.out);
    launch_site(E->tsite, g, par0, E->npar, n, adm, cv, red_to(E, E->r2_true), st);
  }
  {  // p = rs ; xs = 0
    FConvert<SFS, SFS> cv;
    sf2<S>(E->rs, cv.in);
    sf2<S>(E->p, cv.out);
    launch_site_sloppy(E, par0, E->npar, n, adm, cv, red_to(E, E->pAp), st);
    FZero<SFS> z;
    sf2<S>(E->xs, z.out);
    launch_site_sloppy(E, par0, E->npar, n, adm, z, Reduce{}, st);
  }
  g_launches++;
  admit_state_kernel<<<1, 128, 0, st>>>(scalars_of(E), adm, use_x0, n);
}

// Debug/test path: apply the sloppy operator to one field via slot 0.
template <int S>
static void debug_apply_impl(wl_engine* E, int stage, double mass, const void* in, void* out, cudaStream_t st) {
  using SFS = SpinorField<S>;
  using SFD = SpinorField<P_DOUBLE>;
  using LS = typename SloppyLinks<S>::type;
  const Geom& g = E->ctx->g;
  LS L = SloppyLinks<S>::get(E->gauge);
  const double m0 = mass + 4.0;
  std::vector<double> coef = {1.0, -0.5, 0.5 / (m0 * m0), m0};
  double* dc = E->r2_true;  // scratch: 4 doubles (engine has >= 1 slot; r2_true has n entries)
  double* tmp;
  cudaMalloc(&tmp, 4 * sizeof(double));
  cudaMemcpyAsync(tmp, coef.data(), 4 * sizeof(double), cudaMemcpyHostToDevice, st);
  cudaStreamSynchronize(st);
  (void)dc;
  const double *one = tmp, *nh = tmp + 1, *ha = tmp + 2, *mm = tmp + 3;
  const int npar = E->npar;
  const int par0 = 0;
  // in -> b64 (slot 0) -> p (sloppy)
  {
    FPack<SFD> f;
    f.g = g;
    f.in = sref(in, g);
    f.rhs_off = 0;
    sf2<P_DOUBLE>(E->b64, f.out);
    launch_site(E->tsite, g, par0, npar, 1, nullptr, f, red_to(E, E->r2_true), st);
    FConvert<SFD, SFS> cv;
    sf2<P_DOUBLE>(E->b64, cv.in);
    sf2<S>(E->p, cv.out);
    launch_site(E->tsite, g, par0, npar, 1, nullptr, cv, red_to(E, E->r2_true), st);
  }
  IField* res = &E->y;
  int res_par = 0, res_np = npar;
  if (E->prm.op == WL_SOLVE_EO_NORMAL) {
    HopArgs<LS, SFS, EpiXpay<SFS, false>> A{};
    A.g = g; A.links = L; A.nrhs = 1;
    sf2<S>(E->p, A.src); A.parity0 = 1; sf2<S>(E->t1, A.epi.out); A.epi.b = nh;
    launch_hop<false, IdxCompact>(E->ts, A, 1, st);
    if (stage == 0) {
      res = &E->t1;
      res_par = 1;
      res_np = 1;
    } else {
      HopArgs<LS, SFS, EpiXpay<SFS, false>> B{};
      B.g = g; B.links = L; B.nrhs = 1;
      sf2<S>(E->t1, B.src); B.parity0 = 0; sf2<S>(E->y, B.epi.out); sf2<S>(E->p, B.epi.self);
      B.epi.has_self = 1; B.epi.a = one; B.epi.b = ha;
      launch_hop<false, IdxCompact>(E->ts, B, 1, st);
      if (stage >= 2) {
        HopArgs<LS, SFS, EpiXpay<SFS, false>> C{};
        C.g = g; C.links = L; C.nrhs = 1;
        sf2<S>(E->y, C.src); C.parity0 = 1; sf2<S>(E->t1, C.epi.out); C.epi.b = nh;
        launch_hop<true, IdxCompact>(E->ts, C, 1, st);
        HopArgs<LS, SFS, EpiXpay<SFS, false>> D{};
        D.g = g; D.links = L; D.nrhs = 1;
        sf2<S>(E->t1, D.src); D.parity0 = 0; sf2<S>(E->xs, D.epi.out); sf2<S>(E->y, D.epi.self);
        D.epi.has_self = 1; D.epi.a = one; D.epi.b = ha;
        launch_hop<true, IdxCompact>(E->ts, D, 1, st);
        res = &E->xs;
      }
    }
  } else {
    HopArgs<LS, SFS, EpiXpay<SFS, false>> A{};
    A.g = g; A.links = L; A.nrhs = 1;
    sf2<S>(E->p, A.src); A.parity0 = 0; sf2<S>(E->y, A.epi.out); sf2<S>(E->p, A.epi.self);
    A.epi.has_self = 1; A.epi.a = mm; A.epi.b = nh;
    if (stage == 5) launch_hop<true, IdxCompact>(E->ts, A, 2, st);  // D^dag x
    else launch_hop<false, IdxCompact>(E->ts, A, 2, st);            // D x
    if (stage == 4) {
      HopArgs<LS, SFS, EpiXpay<SFS, false>> B{};
      B.g = g; B.links = L; B.nrhs = 1;
      sf2<S>(E->y, B.src); B.parity0 = 0; sf2<S>(E->xs, B.epi.out); sf2<S>(E->y, B.epi.self);
      B.epi.has_self = 1; B.epi.a = mm; B.epi.b = nh;
      launch_hop<true, IdxCompact>(E->ts, B, 2, st);
      res = &E->xs;
    }
  }
  // result (sloppy) -> FP64 (x64 slot 0, or t64 for odd) -> reference layout
  IField dst = res_np == 1 && res_par == 1 ? E->t64 : E->x64;
  {
    IField srcv = *res;
    FConvert<SFS, SFD> cv;
    sf2<S>(srcv, cv.in);
    sf2<P_DOUBLE>(dst, cv.out);
    launch_site(E->tsite, g, res_np == 1 ? res_par : 0, res_np, 1, nullptr, cv, red_to(E, E->r2_true), st);
  }
  cudaMemsetAsync(out, 0, (size_t)g.V * 12 * sizeof(double2), st);
  {
    FUnpack f;
    f.g = g;
    sf2<P_DOUBLE>(dst, f.in);
    f.in_off = 0;
    f.out = sref(out, g);
    f.rhs_off = 0;
    launch_site(E->tsite, g, res_np == 1 ? res_par : 0, res_np, 1, nullptr, f, Reduce{}, st);
  }
  cudaStreamSynchronize(st);
  cudaFree(tmp);
}

extern "C" wl_status wl_engine_debug_apply(wl_engine* E, int stage, double mass, const void* in, void* out) {
  if (!E || !in || !out) WL_FAIL(nullptr, WL_ERR_ARG, "null argument");
  wl_ctx* ctx = E->ctx;
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  const bool eo = E->prm.op == WL_SOLVE_EO_NORMAL;
  if ((eo && (stage < 0 || stage > 2)) || (!eo && (stage < 3 || stage > 5)))
    WL_FAIL(ctx, WL_ERR_ARG, "stage does not match the engine's operator");
  cudaStream_t st = engine_stream(E);
  switch (E->sprec) {
    case P_HALF: debug_apply_impl<P_HALF>(E, stage, mass, in, out, st); break;
    case P_SINGLE: debug_apply_impl<P_SINGLE>(E, stage, mass, in, out, st); break;
    default: debug_apply_impl<P_DOUBLE>(E, stage, mass, in, out, st); break;
  }
  return check_launch(ctx, "wl_engine_debug_apply");
}

static void enqueue_part(wl_engine* E, cudaStream_t st, int part) {
  switch (E->sprec) {
    case P_HALF: enqueue_iteration<P_HALF>(E, st, part); break;
    case P_SINGLE: enqueue_iteration<P_SINGLE>(E, st, part); break;
    default: enqueue_iteration<P_DOUBLE>(E, st, part); break;
  }
}

static void enqueue_iteration_any(wl_engine* E, cudaStream_t st) {
  enqueue_part(E, st, 1);
  enqueue_part(E, st, 2);
  enqueue_part(E, st, 3);
}

// ------------------------------------------------------------------ autotune
// Times the sloppy hop kernel (the dominant cost) over candidate
// (RHS per thread, sites per block, RHS groups per block) shapes and keeps
// the fastest for this (volume, precision, slot count, operator).
template <int S>
static Tune autotune_hop(wl_engine* E, cudaStream_t st) {
  using SFS = SpinorField<S>;
  using LS = typename SloppyLinks<S>::type;
  const Geom& g = E->ctx->g;
  const int n = E->n;
  std::vector<Tune> cands;
  for (int nr : {1, 2, 4}) {
    if (E->lanes_mode) break;
    if (nr > 1 && nr > n) continue;
    int groups = (n + nr - 1) / nr;
    for (int bx : {64, 128, 256})
      for (int by : {1, 2, 4, 8}) {
        if (bx * by > 256 || by * nr > kMaxRB || (by > 1 && by > groups)) continue;
        cands.push_back(Tune{nr, bx, by});
      }
  }
  if ((S == P_DOUBLE || S == P_SINGLE) && !E->lanes_mode)
    for (int bx : {64, 128, 256}) {
      Tune t;
      t.bx = bx;
      t.pair = 1;
      cands.push_back(t);
    }
  if (E->lanes_mode) {
    for (int lanes : {4, 8, 16}) {
      if (lanes > n && lanes > 4) continue;
      Tune t;
      t.lanes = lanes;
      t.bx = kLaneBlock;
      cands.push_back(t);
    }
  }
  Tune best = cands.front();
  float best_ms = 1e30f;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  HopArgs<LS, SFS, EpiXpay<SFS, false>> A{};
  A.g = g;
  A.links = SloppyLinks<S>::get(E->gauge);
  sf2<S>(E->p, A.src);
  A.parity0 = 1;
  A.nrhs = n;
  A.mask = nullptr;
  sf2<S>(E->t1, A.epi.out);
  A.epi.has_self = 0;
  A.epi.b = E->neg_half;
  const int reps = g.Vh >= 65536 ? 5 : 20;
  for (const Tune& t : cands) {  // best of three timings per candidate (shapes within a few % of each other)
    launch_hop<false, IdxCompact>(t, A, 1, st);
    for (int trial = 0; trial < 3; ++trial) {
      cudaEventRecord(e0, st);
      for (int i = 0; i < reps; ++i) launch_hop<false, IdxCompact>(t, A, 1, st);
      cudaEventRecord(e1, st);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (cudaGetLastError() == cudaSuccess && ms < best_ms) {
        best_ms = ms;
        best = t;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

static float time_update_hop(wl_engine* E, cudaStream_t st, const Tune& t, int reps);

// The FP64 hop of the reliable update in lanes engines: the RHS lanes per site,
// i.e. how many sweeps over the lattice one update hop makes (nslots / lanes),
// is chosen by timing.  With 16 FP64 RHS a site's sources are 3 KB and the
// x-neighbour reuse distance of one sweep (2 Ly Lz Lt/2 sites) outgrows the L2,
// so narrower sweeps can move fewer DRAM bytes even though each re-reads the links.
static Tune pick_update_tune(wl_engine* E, cudaStream_t st) {
  const int n = E->n;
  Tune t;
  t.bx = kLaneBlock;
  t.lanes = n > 8 ? 16 : (n > 4 ? 8 : 4);
  // WL_FORCE_UPDATE_TUNE="lanes[,seq]" pins the shape
  if (const char* f = std::getenv("WL_FORCE_UPDATE_TUNE")) {
    int lanes = 0, seq = 1;
    const int got = std::sscanf(f, "%d,%d", &lanes, &seq);
    const bool ok_seq = seq == 1 || (lanes == 8 && seq == 2) || (lanes == 4 && (seq == 2 || seq == 4));
    if (got >= 1 && (lanes == 4 || lanes == 8 || lanes == 16) && ok_seq) {
      t.lanes = lanes;
      t.seq = seq;
      return t;
    }
  }
  TuneKey k{E->ctx->g.Vh, 100 + (E->ru_links12 ? 1 : 0), n, E->prm.op};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(k);
    if (it != g_tune_cache.end()) return it->second;
  }
  const char* env = std::getenv("WL_AUTOTUNE");
  if (!(env && env[0] == '0')) {
    const int reps = E->ctx->g.Vh >= 65536 ? 3 : 10;
    float best_ms = 1e30f;
    Tune best = t;
    const int shapes[][2] = {{4, 1}, {4, 2}, {4, 4}, {8, 1}, {8, 2}, {16, 1}};
    for (const auto& sh : shapes) {
      const int lanes = sh[0], seq = sh[1];
      if ((lanes > n && lanes > 4) || (seq > 1 && lanes * seq > n)) continue;
      Tune c = t;
      c.lanes = lanes;
      c.seq = seq;
      for (int trial = 0; trial < 3; ++trial) {
        const float ms = time_update_hop(E, st, c, reps);
        if (cudaGetLastError() == cudaSuccess && ms < best_ms) {
          best_ms = ms;
          best = c;
        }
      }
    }
    t = best;
  }
  const char* verb = std::getenv("WL_VERBOSE");
  if (verb && verb[0] == '1')
    std::fprintf(stderr, "[wl] update tune vh=%d links12=%d nslots=%d op=%d -> lanes=%d seq=%d\n", k.vh,
                 (int)E->ru_links12, n, k.op, t.lanes, t.seq);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[k] = t;
  return t;
}

static Tune pick_tune(wl_engine* E, cudaStream_t st) {
  // WL_FORCE_TUNE="nr,bx,by,lanes[,pair[,mma]]" pins the hop shape (tests exercise every shape this way)
  if (const char* f = std::getenv("WL_FORCE_TUNE")) {
    Tune t;
    const int nf = std::sscanf(f, "%d,%d,%d,%d,%d,%d", &t.nr, &t.bx, &t.by, &t.lanes, &t.pair, &t.mma);
    if (nf == 4) t.pair = 0;
    if (nf < 6) t.mma = 0;
    t.mma = t.mma ? 1 : 0;
    if (nf >= 4) {
      const bool lanes_ok = t.lanes == 0 || t.lanes == 4 || t.lanes == 8 || t.lanes == 16;
      const bool nr_ok = t.nr == 1 || t.nr == 2 || t.nr == 4;
      const bool shape_ok = t.bx % 32 == 0 && t.bx >= 64 && t.bx * t.by <= 256 && t.by * t.nr <= kMaxRB;
      if (lanes_ok && nr_ok && (t.lanes > 0 || shape_ok)) {
        if (t.lanes > 0 && !E->lanes_mode) t = Tune{};  // FP64 iteration or < 4 slots: thread-per-site kernel
        if (t.mma && (t.lanes == 0 || E->sprec != P_HALF)) t.mma = 0;  // FP16 lanes engines only
        if (t.lanes > 0) t.bx = kLaneBlock;
        if (t.pair && (E->sprec == P_HALF || E->lanes_mode || t.lanes > 0)) t.pair = 0;  // FP64 / FP32 sites only
        if (t.pair) t.nr = 1, t.by = 1;
        return t;
      }
    }
  }
  TuneKey k{E->ctx->g.Vh, E->sprec * 2 + (E->lanes_mode ? 1 : 0), E->n, E->prm.op};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(k);
    if (it != g_tune_cache.end()) return it->second;
  }
  Tune t;
  const char* env = std::getenv("WL_AUTOTUNE");
  const bool on = !(env && env[0] == '0');
  if (on) {
    switch (E->sprec) {
      case P_HALF: t = autotune_hop<P_HALF>(E, st); break;
      case P_SINGLE: t = autotune_hop<P_SINGLE>(E, st); break;
      default: t = autotune_hop<P_DOUBLE>(E, st); break;
    }
  } else {
    t.nr = E->n >= 2 ? 2 : 1;
    t.bx = 128;
    t.by = std::max(1, std::min(4, (E->n + t.nr - 1) / t.nr));
  }
  const char* verb = std::getenv("WL_VERBOSE");
  if (verb && verb[0] == '1')
    std::fprintf(stderr, "[wl] tune vh=%d prec=%d nslots=%d op=%d -> nr=%d bx=%d by=%d lanes=%d pair=%d mma=%d\n",
                 k.vh, k.prec, k.nslots, k.op, t.nr, t.bx, t.by, t.lanes, t.pair, t.mma);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[k] = t;
  return t;
}

// ------------------------------------------------------------------ engine API
extern "C" void wl_engine_destroy(wl_engine* E) {
  if (!E) return;
  cudaSetDevice(E->ctx->device);
  cudaStream_t st = engine_stream(E);
  if (st) cudaStreamSynchronize(st);
  if (E->gexec) cudaGraphExecDestroy(E->gexec);
  if (E->gloop) cudaGraphExecDestroy(E->gloop);
  if (E->grun) cudaGraphExecDestroy(E->grun);
  IField* fs[] = {&E->b64, &E->x64, &E->y64, &E->t64, &E->xs, &E->rs, &E->p, &E->y, &E->t1};
  for (IField* f : fs) free_field(*f);
  cudaFree(E->dbl);
  cudaFree(E->ints);
  cudaFree(E->partials);
  cudaFree(E->counters);
  cudaFree(E->ru_iters);
  cudaFree(E->loop_count);
  cudaFree(E->run_state);
  if (E->h_pinned) cudaFreeHost(E->h_pinned);
  if (E->poll_ev) cudaEventDestroy(E->poll_ev);
  if (st) cudaStreamDestroy(st);
  {
    std::lock_guard<std::mutex> lk(g_es_mu);
    g_engine_streams.erase(E);
  }
  delete E;
}

extern "C" wl_status wl_engine_create(wl_ctx* ctx, wl_gauge* G, const wl_solve_params* prm, int nslots,
                                      wl_engine** out) {
  NvtxRange nvtx_range("wl_engine_create");
  if (!ctx || !G || !prm || !out) WL_FAIL(ctx, WL_ERR_ARG, "null argument");
  if (nslots <= 0 || nslots > 4096) WL_FAIL(ctx, WL_ERR_ARG, "nslots out of range");
  if (prm->op != WL_SOLVE_NORMAL && prm->op != WL_SOLVE_EO_NORMAL) WL_FAIL(ctx, WL_ERR_ARG, "unknown solve op");
  if (prm->inner_prec < 0 || prm->inner_prec > 2) WL_FAIL(ctx, WL_ERR_ARG, "unknown inner precision");
  if (!(prm->tol > 0.0)) WL_FAIL(ctx, WL_ERR_ARG, "tol must be positive");
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  wl_engine* E = new wl_engine();
  E->ctx = ctx;
  E->gauge = G;
  E->prm = *prm;
  if (E->prm.maxiter <= 0) E->prm.maxiter = 1000;
  if (E->prm.check_every <= 0) E->prm.check_every = 8;
  E->n = nslots;
  E->npar = prm->op == WL_SOLVE_EO_NORMAL ? 1 : 2;
  E->sprec = prm->inner_prec;
  // 12-real reconstruction is exact only for SU(3) links: fall back to FP64
  // 18-real iteration when the uploaded links are not unitary.
  double uerr = 0.0;
  wl_status s0 = wl_gauge_unitarity(G, &uerr);
  if (s0 != WL_OK) {
    delete E;
    return s0;
  }
  if (E->sprec != P_DOUBLE && !(uerr < 1e-4)) E->sprec = P_DOUBLE;
  E->ru_links12 = uerr < 1e-12;
  cudaStream_t st;
  WL_CUDA(ctx, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  {
    std::lock_guard<std::mutex> lk(g_es_mu);
    g_engine_streams[E] = st;
  }
  const Geom& g = ctx->g;
  const int n = nslots;
  {
    // RHS-in-lanes sloppy hops (and the RHS-innermost field layout they need)
    // for FP16/FP32 iteration with 4 or more slots, unless a forced shape or
    // WL_FAST_HOP=0 selects the thread-per-site kernels
    const char* ft = std::getenv("WL_FORCE_TUNE");
    int fnr = 0, fbx = 0, fby = 0, flanes = -1;
    const bool forced = ft && std::sscanf(ft, "%d,%d,%d,%d", &fnr, &fbx, &fby, &flanes) == 4;
    E->lanes_mode = E->sprec != P_DOUBLE && n >= 4 && fast_hop_enabled() && (!forced || flanes > 0);
  }
  wl_status s = WL_OK;
  cudaStream_t keep = ctx->stream;
  ctx->stream = st;
  const int tpar = prm->op == WL_SOLVE_EO_NORMAL ? 1 : 2;
  // in lanes mode the FP64 fields are RHS-innermost too: the reliable update
  // then runs as one RHS-in-lanes FP64 pass over all slots
  const bool li = E->lanes_mode;
  if (s == WL_OK) s = alloc_field(ctx, E->b64, P_DOUBLE, g.Vh, n, E->npar, li);
  if (s == WL_OK) s = alloc_field(ctx, E->x64, P_DOUBLE, g.Vh, n, E->npar, li);
  if (s == WL_OK) s = alloc_field(ctx, E->y64, P_DOUBLE, g.Vh, n, E->npar, li);
  if (s == WL_OK) s = alloc_field(ctx, E->t64, P_DOUBLE, g.Vh, n, tpar, li);
  if (s == WL_OK) s = alloc_field(ctx, E->xs, E->sprec, g.Vh, n, E->npar, li);
  if (s == WL_OK) s = alloc_field(ctx, E->rs, E->sprec, g.Vh, n, E->npar, li);
  if (s == WL_OK) s = alloc_field(ctx, E->p, E->sprec, g.Vh, n, E->npar, li);
  if (s == WL_OK) s = alloc_field(ctx, E->y, E->sprec, g.Vh, n, E->npar, li);
  if (s == WL_OK) s = alloc_field(ctx, E->t1, E->sprec, g.Vh, n, 1, li);
  ctx->stream = keep;
  if (s != WL_OK) {
    wl_engine_destroy(E);
    return s;
  }
  cudaError_t e = cudaMalloc(&E->dbl, sizeof(double) * kEngineDoubles * n);
  if (e == cudaSuccess) e = cudaMalloc(&E->ints, sizeof(int) * (kEngineInts * n + 1));
  // most partial sums per RHS: one per warp of the RHS-in-lanes kernels; at 16 lanes a
  // warp covers 2 sites, so both parities give up to Vh partials
  const size_t nblk = (size_t)g.Vh + 64;
  if (e == cudaSuccess) e = cudaMalloc(&E->partials, sizeof(double) * nblk * n);
  if (e == cudaSuccess) e = cudaMalloc(&E->counters, sizeof(unsigned) * (n + 1));
  if (e == cudaSuccess) e = cudaMallocHost(&E->h_pinned, sizeof(int) * (3 * n + 2));
  if (e == cudaSuccess) e = cudaMalloc(&E->ru_iters, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&E->loop_count, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&E->run_state, 4 * sizeof(int));
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&E->poll_ev, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    ctx->err = std::string("engine allocation: ") + cudaGetErrorString(e);
    wl_engine_destroy(E);
    return WL_ERR_OOM;
  }
  cudaMemsetAsync(E->dbl, 0, sizeof(double) * kEngineDoubles * n, st);
  cudaMemsetAsync(E->ints, 0, sizeof(int) * (kEngineInts * n + 1), st);
  cudaMemsetAsync(E->counters, 0, sizeof(unsigned) * (n + 1), st);
  cudaMemsetAsync(E->ru_iters, 0, sizeof(int), st);
  cudaMemsetAsync(E->run_state, 0, 4 * sizeof(int), st);
  double* d = E->dbl;
  E->r2 = d + 0 * n; E->r2_new = d + 1 * n; E->pAp = d + 2 * n; E->r2_true = d + 3 * n;
  E->rmax2 = d + 4 * n; E->b2 = d + 5 * n; E->tol2 = d + 6 * n; E->beta = d + 7 * n;
  E->one = d + 8 * n; E->neg_half = d + 9 * n; E->half_alpha = d + 10 * n; E->m0 = d + 11 * n;
  E->alpha = d + 12 * n;
  int* I = E->ints;
  E->active = I + 0 * n; E->ru = I + 1 * n; E->iters = I + 2 * n; E->maxiter = I + 3 * n;
  E->status = I + 4 * n; E->n_ru = I + 5 * n; E->admit = I + 6 * n; E->n_active = I + 8 * n;
  // I + 7n .. 8n: slot -> caller index map
  E->h_tol2.assign(n, 0.0);
  E->h_one.assign(n, 1.0);
  E->h_neg_half.assign(n, -0.5);
  E->h_half_alpha.assign(n, 0.0);
  E->h_m0.assign(n, 4.0);
  E->h_maxiter.assign(n, E->prm.maxiter);
  E->ts = pick_tune(E, st);
  E->td = Tune{1, 128, 1};
  E->td.pair = 1;  // FP64 fields site-major: the two-threads-per-site stencil
  if (E->lanes_mode) E->td = pick_update_tune(E, st);
  E->tsite = Tune{1, 128, 1};
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    ctx->err = std::string("engine set-up: ") + cudaGetErrorString(e);
    wl_engine_destroy(E);
    return WL_ERR_CUDA;
  }
  *out = E;
  return WL_OK;
}

static wl_status admit_impl(wl_engine* E, const int* slots, int nadm, const void* b, const void* x0,
                            const double* masses, const double* tols, const int* maxiters) {
  if (!E || !slots || !b || !masses) WL_FAIL(nullptr, WL_ERR_ARG, "null argument");
  wl_ctx* ctx = E->ctx;
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  const int n = E->n;
  std::vector<int> adm(n, 0), map(n, 0);
  for (int i = 0; i < nadm; ++i) {
    int s = slots[i];
    if (s < 0 || s >= n) WL_FAIL(ctx, WL_ERR_ARG, "slot index out of range");
    adm[s] = 1;
    map[s] = i;
    const double m0 = masses[i] + 4.0;
    if (!(std::fabs(m0) > 1e-12)) WL_FAIL(ctx, WL_ERR_ARG, "m0 = mass + 4 must be non-zero");
    const double tol = tols ? tols[i] : E->prm.tol;
    E->h_tol2[s] = tol * tol;
    E->h_m0[s] = m0;
    E->h_half_alpha[s] = 0.5 / (m0 * m0);
    E->h_maxiter[s] = maxiters ? maxiters[i] : E->prm.maxiter;
  }
  cudaStream_t st = engine_stream(E);
  // order after work already queued on the caller's stream (b may have been produced there)
  cudaEvent_t ev;
  WL_CUDA(ctx, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  cudaEventRecord(ev, ctx->stream);
  cudaStreamWaitEvent(st, ev, 0);
  cudaEventDestroy(ev);
  WL_CUDA(ctx, cudaMemcpyAsync(E->admit, adm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  WL_CUDA(ctx, cudaMemcpyAsync(E->ints + 7 * n, map.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  WL_CUDA(ctx, cudaMemcpyAsync(E->tol2, E->h_tol2.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
  WL_CUDA(ctx, cudaMemcpyAsync(E->one, E->h_one.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
  WL_CUDA(ctx, cudaMemcpyAsync(E->neg_half, E->h_neg_half.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
  WL_CUDA(ctx, cudaMemcpyAsync(E->half_alpha, E->h_half_alpha.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
  WL_CUDA(ctx, cudaMemcpyAsync(E->m0, E->h_m0.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
  WL_CUDA(ctx, cudaMemcpyAsync(E->maxiter, E->h_maxiter.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  // host vectors must outlive the async copies
  WL_CUDA(ctx, cudaStreamSynchronize(st));
  const int use_x0 = x0 != nullptr;
  switch (E->sprec) {
    case P_HALF: enqueue_admit<P_HALF>(E, b, use_x0, x0, E->ints + 7 * n, st); break;
    case P_SINGLE: enqueue_admit<P_SINGLE>(E, b, use_x0, x0, E->ints + 7 * n, st); break;
    default: enqueue_admit<P_DOUBLE>(E, b, use_x0, x0, E->ints + 7 * n, st); break;
  }
  return check_launch(ctx, "wl_engine_admit");
}

extern "C" wl_status wl_engine_admit(wl_engine* E, const int* slots, int nadm, const void* b, const double* masses,
                                     const double* tols, const int* maxiters) {
  NvtxRange nvtx_range("wl_engine_admit");
  return admit_impl(E, slots, nadm, b, nullptr, masses, tols, maxiters);
}

static wl_status engine_admit_all(wl_engine* E, const void* b, const void* x0, const double* masses) {
  const int n = E->n;
  std::vector<int> slots(n);
  for (int i = 0; i < n; ++i) slots[i] = i;
  return admit_impl(E, slots.data(), n, b, x0, masses, nullptr, nullptr);
}

// Appends one CG iteration to graph `g` (captured from stream st): part 1, the reliable-update
// body (part 2) inside an IF node on a conditional handle created on g (the decide kernel of
// part 1 sets it), then part 3, whose finalize kernel also drives an enclosing WHILE node
// when `loop` is set.  Counts the unconditional kernels in *uncond and the body's in E->ru_body_kernels.
static cudaError_t capture_iteration(wl_engine* E, cudaStream_t st, cudaGraph_t g, const SolveLoop* loop,
                                     long long* uncond) {
  const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
  cudaGraphConditionalHandle cond = 0;
  cudaError_t e = cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) return e;
  E->cond = cond;  // captured by value into the decide kernel of this iteration
  E->use_cond = true;
  const long long before = g_launches.load();
  e = cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, mode);
  if (e != cudaSuccess) return e;
  enqueue_part(E, st, 1);
  cudaStreamCaptureStatus cs;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  std::vector<cudaGraphNode_t> dv;
  e = cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &deps, &ndeps);
  if (e == cudaSuccess) dv.assign(deps, deps + ndeps);
  cudaGraph_t g1 = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(st, &g1);
  if (e == cudaSuccess) e = e2;
  long long n_uncond = g_launches.load() - before;
  cudaGraphNode_t cond_node = nullptr;
  if (e == cudaSuccess) {
    // cudaGraphNodeParams has no default constructor (it holds a union): zeroed storage
    alignas(cudaGraphNodeParams) unsigned char cpbuf[sizeof(cudaGraphNodeParams)];
    std::memset(cpbuf, 0, sizeof(cpbuf));
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cpbuf);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    e = cudaGraphAddNode(&cond_node, g, dv.data(), dv.size(), &cp);
    if (e == cudaSuccess) {
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      e = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, mode);
      if (e == cudaSuccess) {
        const long long b0 = g_launches.load();
        enqueue_part(E, st, 2);
        E->ru_body_kernels = g_launches.load() - b0;
        cudaGraph_t gb = nullptr;
        e = cudaStreamEndCapture(st, &gb);
      }
    }
  }
  if (e == cudaSuccess) {
    e = cudaStreamBeginCaptureToGraph(st, g, &cond_node, nullptr, 1, mode);
    if (e == cudaSuccess) {
      const long long p3 = g_launches.load();
      E->capture_loop = loop;  // the finalize kernel of part 3 drives the loop
      enqueue_part(E, st, 3);
      E->capture_loop = nullptr;
      n_uncond += g_launches.load() - p3;
      cudaGraph_t g3 = nullptr;
      e = cudaStreamEndCapture(st, &g3);
    }
  }
  g_launches = before;  // captured, not launched
  *uncond = n_uncond;
  return e;
}

static wl_status build_graph(wl_engine* E, cudaStream_t st) {
  wl_ctx* ctx = E->ctx;
  cudaGraph_t graph = nullptr;
  WL_CUDA(ctx, cudaGraphCreate(&graph, 0));
  long long nk = 0;
  cudaError_t e = capture_iteration(E, st, graph, nullptr, &nk);
  E->graph_kernels = nk;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&E->gexec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    E->use_cond = false;
    E->gexec = nullptr;
    ctx->err = std::string("graph build: ") + cudaGetErrorString(e);
    return WL_ERR_CUDA;
  }
  E->graph_built = true;
  return WL_OK;
}

// The whole solve as one graph: a WHILE node whose body is one iteration, whose finalize
// kernel (solve_loop_step) keeps the loop going while any slot is active and fewer than
// `cap` iterations have run (a hard bound on the device loop; slots stop at their maxiter
// long before).  wl_solve launches it once per solve instead of launching an iteration graph
// and synchronising on a status poll every check_every iterations.  On any failure the
// engine keeps the host-driven loop.
static wl_status build_loop_graph(wl_engine* E, cudaStream_t st, bool run_mode = false) {
  wl_ctx* ctx = E->ctx;
  cudaGraph_t graph = nullptr;
  WL_CUDA(ctx, cudaGraphCreate(&graph, 0));
  cudaGraphConditionalHandle wh = 0;
  cudaError_t e = cudaGraphConditionalHandleCreate(&wh, graph, 1, cudaGraphCondAssignDefault);
  cudaGraphNode_t wnode = nullptr;
  cudaGraph_t body = nullptr;
  if (e == cudaSuccess) {
    alignas(cudaGraphNodeParams) unsigned char cpbuf[sizeof(cudaGraphNodeParams)];
    std::memset(cpbuf, 0, sizeof(cpbuf));
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cpbuf);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = wh;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    e = cudaGraphAddNode(&wnode, graph, nullptr, 0, &cp);
    if (e == cudaSuccess) body = cp.conditional.phGraph_out[0];
  }
  long long nk = 0;
  if (e == cudaSuccess) {
    int cap = 0;
    for (int m : E->h_maxiter) cap = std::max(cap, m);
    SolveLoop L{E->n_active, E->loop_count, cap + 8, wh, nullptr, nullptr, nullptr};
    if (run_mode) L = SolveLoop{E->n_active, E->run_state + 2, 0, wh, E->run_state, E->run_state + 1, E->run_state + 3};
    e = capture_iteration(E, st, body, &L, &nk);
  }
  cudaGraphExec_t& exec = run_mode ? E->grun : E->gloop;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    exec = nullptr;
    (run_mode ? E->run_failed : E->loop_failed) = true;
    cudaGetLastError();
    return WL_ERR_CUDA;
  }
  if (run_mode) {
    E->run_kernels = nk;
    return WL_OK;
  }
  E->loop_kernels = nk;
  E->loop_cap = 0;
  for (int m : E->h_maxiter) E->loop_cap = std::max(E->loop_cap, m);
  return WL_OK;
}

// Up to max_iters iterations in one launch of the engine's run graph, stopping on the device
// as soon as a slot finishes (see solve_loop_step); engines without graphs step instead.
extern "C" wl_status wl_engine_run(wl_engine* E, int max_iters) {
  NvtxRange nvtx_range("wl_engine_run");
  if (!E) WL_FAIL(nullptr, WL_ERR_ARG, "null engine");
  if (max_iters <= 0) WL_FAIL(E->ctx, WL_ERR_ARG, "max_iters must be positive");
  wl_ctx* ctx = E->ctx;
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  if (!E->prm.use_graph || E->run_failed) return wl_engine_step(E, max_iters);
  cudaStream_t st = engine_stream(E);
  if (E->grun && E->run_gauge_id != E->gauge->id) {
    cudaGraphExecDestroy(E->grun);
    E->grun = nullptr;
  }
  if (!E->grun) {
    if (build_loop_graph(E, st, true) != WL_OK) {
      ctx->err.clear();
      return wl_engine_step(E, max_iters);
    }
    E->run_gauge_id = E->gauge->id;
  }
  g_launches++;
  run_loop_setup_kernel<<<1, 1, 0, st>>>(E->run_state, max_iters, E->run_state + 1, E->n_active, E->run_state + 2);
  WL_CUDA(ctx, cudaGraphLaunch(E->grun, st));
  return check_launch(ctx, "wl_engine_run");
}

extern "C" wl_status wl_engine_step(wl_engine* E, int iters) {
  NvtxRange nvtx_range("wl_engine_step");
  if (!E) WL_FAIL(nullptr, WL_ERR_ARG, "null engine");
  wl_ctx* ctx = E->ctx;
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = engine_stream(E);
  if (E->prm.use_graph && E->graph_built && E->gauge_id != E->gauge->id) {
    cudaGraphExecDestroy(E->gexec);
    E->gexec = nullptr;
    E->graph_built = false;
  }
  if (E->prm.use_graph && !E->graph_built) {
    E->gauge_id = E->gauge->id;
    wl_status s = build_graph(E, st);
    if (s != WL_OK) return s;
  }
  for (int i = 0; i < iters; ++i) {
    if (E->prm.use_graph) {
      WL_CUDA(ctx, cudaGraphLaunch(E->gexec, st));
      g_launches += E->graph_kernels;
    } else {
      enqueue_iteration_any(E, st);
    }
  }
  return check_launch(ctx, "wl_engine_step");
}

extern "C" void* wl_engine_stream(wl_engine* E) { return E ? (void*)engine_stream(E) : nullptr; }

extern "C" wl_status wl_engine_time_hop(wl_engine* E, int reps, double* ms, double* bytes) {
  if (!E || !ms || !bytes || reps <= 0) WL_FAIL(nullptr, WL_ERR_ARG, "bad argument");
  wl_ctx* ctx = E->ctx;
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = engine_stream(E);
  float t = 0.f;
  switch (E->sprec) {
    case P_HALF: time_hop_impl<P_HALF>(E, st, reps, &t); break;
    case P_SINGLE: time_hop_impl<P_SINGLE>(E, st, reps, &t); break;
    default: time_hop_impl<P_DOUBLE>(E, st, reps, &t); break;
  }
  wl_status s = check_launch(ctx, "wl_engine_time_hop");
  if (s != WL_OK) return s;
  *ms = (double)t / reps;
  *bytes = (double)hop_bytes(ctx->g, E->sprec, E->n);
  return WL_OK;
}

extern "C" wl_status wl_engine_time_cg_hop(wl_engine* E, int reps, double* ms, double* bytes) {
  if (!E || !ms || !bytes || reps <= 0) WL_FAIL(nullptr, WL_ERR_ARG, "bad argument");
  wl_ctx* ctx = E->ctx;
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = engine_stream(E);
  float t = 0.f;
  switch (E->sprec) {
    case P_HALF: time_cg_hop_impl<P_HALF>(E, st, reps, &t); break;
    case P_SINGLE: time_cg_hop_impl<P_SINGLE>(E, st, reps, &t); break;
    default: time_cg_hop_impl<P_DOUBLE>(E, st, reps, &t); break;
  }
  wl_status s = check_launch(ctx, "wl_engine_time_cg_hop");
  if (s != WL_OK) return s;
  *ms = (double)t / reps;
  // per target site: 8 links; per RHS the source record gathered once, the self records of
  // y, p, x_s and r_s read and x_s, r_s written
  const double L = E->sprec == P_DOUBLE ? 144.0 : (E->sprec == P_SINGLE ? 48.0 : 24.0);
  const double S = E->sprec == P_DOUBLE ? 192.0 : (E->sprec == P_SINGLE ? 96.0 : 52.0);
  const double sites = (double)ctx->g.Vh * (E->prm.op == WL_SOLVE_EO_NORMAL ? 1 : 2);
  *bytes = sites * (8.0 * L + E->n * 7.0 * S);
  return WL_OK;
}

// x64 -> t64 = -1/2 K_oe x64 over all slots with the update's links and shape, `reps` launches
// after one warm-up; returns the CUDA-event time of the reps on the engine stream.
template <class LDT>
static float time_update_hop_impl(wl_engine* E, cudaStream_t st, const Tune& t, int reps, const LDT& LD) {
  using SFD = SpinorField<P_DOUBLE>;
  HopArgs<LDT, SFD, EpiXpay<SFD, false>> A{};
  A.g = E->ctx->g;
  A.links = LD;
  sf2<P_DOUBLE>(E->x64, A.src);
  A.parity0 = 1;
  A.nrhs = E->n;
  A.mask = nullptr;
  sf2<P_DOUBLE>(E->t64, A.epi.out);
  A.epi.has_self = 0;
  A.epi.b = E->neg_half;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  launch_hop<false, IdxCompact>(t, A, 1, st);
  cudaEventRecord(e0, st);
  for (int i = 0; i < reps; ++i) launch_hop<false, IdxCompact>(t, A, 1, st);
  cudaEventRecord(e1, st);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms;
}

static float time_update_hop(wl_engine* E, cudaStream_t st, const Tune& t, int reps) {
  if (E->ru_links12) return time_update_hop_impl(E, st, t, reps, LinkField<L_D12>{E->gauge->d12, E->ctx->g.Vh});
  return time_update_hop_impl(E, st, t, reps, LinkField<L_D18>{E->gauge->d18, E->ctx->g.Vh});
}

extern "C" wl_status wl_engine_time_update_hop(wl_engine* E, int reps, double* ms, double* bytes) {
  if (!E || !ms || !bytes || reps <= 0) WL_FAIL(nullptr, WL_ERR_ARG, "bad argument");
  wl_ctx* ctx = E->ctx;
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  const float t = time_update_hop(E, engine_stream(E), E->td, reps);
  wl_status s = check_launch(ctx, "wl_engine_time_update_hop");
  if (s != WL_OK) return s;
  *ms = (double)t / reps;
  const double L = E->ru_links12 ? 96.0 : 144.0;
  *bytes = (double)ctx->g.Vh * (8.0 * L + E->n * 2.0 * 192.0);
  return WL_OK;
}

// Copies of the active count, the per-slot status and the conditional-body counter into the
// engine's pinned host buffer, queued on the engine stream.
static wl_status enqueue_poll_copies(wl_engine* E, cudaStream_t st) {
  wl_ctx* ctx = E->ctx;
  const int n = E->n;
  WL_CUDA(ctx, cudaMemcpyAsync(E->h_pinned, E->n_active, sizeof(int), cudaMemcpyDeviceToHost, st));
  WL_CUDA(ctx, cudaMemcpyAsync(E->h_pinned + 1, E->status, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  WL_CUDA(ctx, cudaMemcpyAsync(E->h_pinned + 1 + n, E->ru_iters, sizeof(int), cudaMemcpyDeviceToHost, st));
  WL_CUDA(ctx, cudaMemcpyAsync(E->h_pinned + 3 + n, E->run_state + 3, sizeof(int), cudaMemcpyDeviceToHost, st));
  return WL_OK;
}

// Read the pinned buffer once its copies have completed.
static void read_poll_copies(wl_engine* E, int* status, int* n_active) {
  const int n = E->n;
  {  // kernels that ran inside the graph's conditional reliable-update body
    const long long seen = E->h_pinned[1 + n];
    g_launches += (seen - E->ru_iters_seen) * E->ru_body_kernels;
    E->ru_iters_seen = seen;
    const long long runs = E->h_pinned[3 + n];  // iterations run by wl_engine_run launches
    g_launches += (runs - E->run_seen) * E->run_kernels;
    E->run_seen = runs;
  }
  if (n_active) *n_active = E->h_pinned[0];
  if (status) std::memcpy(status, E->h_pinned + 1, sizeof(int) * n);
}

extern "C" wl_status wl_engine_poll(wl_engine* E, int* status, int* n_active) {
  if (!E) WL_FAIL(nullptr, WL_ERR_ARG, "null engine");
  wl_ctx* ctx = E->ctx;
  cudaStream_t st = engine_stream(E);
  wl_status s = enqueue_poll_copies(E, st);
  if (s != WL_OK) return s;
  WL_CUDA(ctx, cudaStreamSynchronize(st));
  E->poll_pending = false;
  read_poll_copies(E, status, n_active);
  return WL_OK;
}

extern "C" wl_status wl_engine_poll_async(wl_engine* E) {
  if (!E) WL_FAIL(nullptr, WL_ERR_ARG, "null engine");
  wl_ctx* ctx = E->ctx;
  cudaStream_t st = engine_stream(E);
  wl_status s = enqueue_poll_copies(E, st);
  if (s != WL_OK) return s;
  WL_CUDA(ctx, cudaEventRecord(E->poll_ev, st));
  E->poll_pending = true;
  return WL_OK;
}

extern "C" int wl_engine_poll_ready(wl_engine* E, int* status, int* n_active) {
  if (!E || !E->poll_pending) return -1;
  const cudaError_t q = cudaEventQuery(E->poll_ev);
  if (q == cudaErrorNotReady) return 0;
  if (q != cudaSuccess) {
    E->ctx->err = std::string("wl_engine_poll_ready: ") + cudaGetErrorString(q);
    return -2;
  }
  E->poll_pending = false;
  read_poll_copies(E, status, n_active);
  return 1;
}

static wl_status engine_stats(wl_engine* E, wl_solve_stats* stats, int first, int count) {
  wl_ctx* ctx = E->ctx;
  cudaStream_t st = engine_stream(E);
  const int n = E->n;
  std::vector<int> it(n), sts(n), nru(n);
  std::vector<double> r2(n), b2(n);
  WL_CUDA(ctx, cudaMemcpyAsync(it.data(), E->iters, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  WL_CUDA(ctx, cudaMemcpyAsync(sts.data(), E->status, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  WL_CUDA(ctx, cudaMemcpyAsync(nru.data(), E->n_ru, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  WL_CUDA(ctx, cudaMemcpyAsync(r2.data(), E->r2, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  WL_CUDA(ctx, cudaMemcpyAsync(b2.data(), E->b2, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  WL_CUDA(ctx, cudaStreamSynchronize(st));
  for (int i = 0; i < count; ++i) {
    const int s = first + i;
    stats[i].iters = it[s];
    stats[i].reliable_updates = nru[s];
    stats[i].status = sts[s];
    stats[i].true_res = b2[s] > 0.0 ? std::sqrt(std::max(r2[s], 0.0) / b2[s]) : 0.0;
  }
  return WL_OK;
}

static wl_status engine_unpack(wl_engine* E, int first, int count, void* x) {
  wl_ctx* ctx = E->ctx;
  cudaStream_t st = engine_stream(E);
  const Geom& g = ctx->g;
  FUnpack f;
  f.g = g;
  sf2<P_DOUBLE>(E->x64, f.in);
  f.in_off = first;
  f.out = sref(x, g);
  f.rhs_off = 0;
  launch_site(E->tsite, g, 0, E->npar, count, nullptr, f, Reduce{}, st);
  if (E->npar == 1) {  // zero odd sites of the reference-layout output
    FZeroRef z;
    z.g = g;
    z.out = sref(x, g);
    z.rhs_off = 0;
    launch_site(E->tsite, g, 1, 1, count, nullptr, z, Reduce{}, st);
  }
  wl_status s = check_launch(ctx, "unpack");
  if (s != WL_OK) return s;
  // make the caller's stream wait for the result
  cudaEvent_t ev;
  WL_CUDA(ctx, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  cudaEventRecord(ev, st);
  cudaStreamWaitEvent(ctx->stream, ev, 0);
  cudaEventDestroy(ev);
  return WL_OK;
}

extern "C" wl_status wl_engine_retire(wl_engine* E, int slot, void* x, wl_solve_stats* stats) {
  NvtxRange nvtx_range("wl_engine_retire");
  if (!E || !x) WL_FAIL(nullptr, WL_ERR_ARG, "null argument");
  if (slot < 0 || slot >= E->n) WL_FAIL(E->ctx, WL_ERR_ARG, "slot index out of range");
  wl_status s = engine_unpack(E, slot, 1, x);
  if (s != WL_OK) return s;
  if (stats) {
    s = engine_stats(E, stats, slot, 1);
    if (s != WL_OK) return s;
  }
  // mark idle
  int zero = 0;
  cudaStream_t st = engine_stream(E);
  WL_CUDA(E->ctx, cudaMemcpyAsync(E->status + slot, &zero, sizeof(int), cudaMemcpyHostToDevice, st));
  WL_CUDA(E->ctx, cudaMemcpyAsync(E->active + slot, &zero, sizeof(int), cudaMemcpyHostToDevice, st));
  WL_CUDA(E->ctx, cudaStreamSynchronize(st));
  return WL_OK;
}

// ------------------------------------------------------------------ solve
// One launch of the engine's whole-solve graph (built on first use, rebuilt when the gauge or
// the iteration limit changed); *ran is false when the graph is unavailable and the caller
// drives the iterations from the host instead.
static wl_status run_loop_graph(wl_engine* E, bool* ran) {
  *ran = false;
  if (E->loop_failed) return WL_OK;
  wl_ctx* ctx = E->ctx;
  cudaStream_t st = engine_stream(E);
  int cap = 0;
  for (int m : E->h_maxiter) cap = std::max(cap, m);
  if (E->gloop && (E->loop_gauge_id != E->gauge->id || E->loop_cap != cap)) {
    cudaGraphExecDestroy(E->gloop);
    E->gloop = nullptr;
  }
  if (!E->gloop) {
    if (build_loop_graph(E, st) != WL_OK) {
      ctx->err.clear();
      return WL_OK;
    }
    E->loop_gauge_id = E->gauge->id;
  }
  const int n = E->n;
  WL_CUDA(ctx, cudaMemsetAsync(E->loop_count, 0, sizeof(int), st));
  WL_CUDA(ctx, cudaGraphLaunch(E->gloop, st));
  WL_CUDA(ctx, cudaMemcpyAsync(E->h_pinned + 2 + n, E->loop_count, sizeof(int), cudaMemcpyDeviceToHost, st));
  WL_CUDA(ctx, cudaStreamSynchronize(st));
  g_launches += (long long)E->h_pinned[2 + n] * E->loop_kernels;
  *ran = true;
  return WL_OK;
}

struct SolveKey {
  const wl_ctx* ctx;
  int op, prec, n, graph;
  bool operator<(const SolveKey& o) const {
    return std::tie(ctx, op, prec, n, graph) < std::tie(o.ctx, o.op, o.prec, o.n, o.graph);
  }
};
static std::map<SolveKey, wl_engine*> g_solve_cache;
static std::mutex g_solve_mu;

extern "C" wl_status wl_solve(wl_ctx* ctx, wl_gauge* G, const wl_solve_params* prm, const double* masses,
                              const void* b, void* x, int nrhs, wl_solve_stats* stats) {
  NvtxRange nvtx_range("wl_solve");
  if (!ctx || !G || !prm || !masses || !b || !x) WL_FAIL(ctx, WL_ERR_ARG, "null argument");
  if (nrhs <= 0) WL_FAIL(ctx, WL_ERR_ARG, "nrhs must be positive");
  wl_engine* E = nullptr;
  SolveKey key{ctx, prm->op, prm->inner_prec, nrhs, prm->use_graph};
  {
    std::lock_guard<std::mutex> lk(g_solve_mu);
    auto it = g_solve_cache.find(key);
    if (it != g_solve_cache.end()) {
      E = it->second;
      g_solve_cache.erase(it);
    }
  }
  if (E) {
    E->gauge = G;  // wl_engine_step rebuilds the graph when the gauge id changed
    const bool delta_changed = E->prm.delta != prm->delta;
    E->prm = *prm;
    if (E->prm.maxiter <= 0) E->prm.maxiter = 1000;
    if (E->prm.check_every <= 0) E->prm.check_every = 8;
    E->h_maxiter.assign(E->n, E->prm.maxiter);
    // delta is the only solve parameter captured by value in the graph (per-RHS
    // masses, tolerances and iteration limits live in device arrays)
    if (E->gexec && delta_changed) {
      cudaGraphExecDestroy(E->gexec);
      E->gexec = nullptr;
      E->graph_built = false;
    }
    if (E->gloop && delta_changed) {
      cudaGraphExecDestroy(E->gloop);
      E->gloop = nullptr;
    }
  } else {
    wl_status s = wl_engine_create(ctx, G, prm, nrhs, &E);
    if (s != WL_OK) return s;
  }
  wl_status s = engine_admit_all(E, b, prm->use_x0 ? x : nullptr, masses);
  int n_active = 1;
  long long done_iters = 0;
  const int chunk = E->prm.check_every;
  bool looped = false;
  if (s == WL_OK && E->prm.use_graph) s = run_loop_graph(E, &looped);
  if (looped) s = wl_engine_poll(E, nullptr, &n_active);  // status, counters, wait errors
  while (s == WL_OK && !looped) {
    s = wl_engine_poll(E, nullptr, &n_active);
    if (s != WL_OK || n_active == 0) break;
    if (done_iters > (long long)E->prm.maxiter + 2 * chunk) break;  // host-side guard
    s = wl_engine_step(E, chunk);
    done_iters += chunk;
  }
  if (s == WL_OK) s = engine_unpack(E, 0, nrhs, x);
  std::vector<wl_solve_stats> tmp(nrhs);
  if (s == WL_OK) s = engine_stats(E, stats ? stats : tmp.data(), 0, nrhs);
  if (s != WL_OK) {
    wl_engine_destroy(E);
    return s;
  }
  {
    std::lock_guard<std::mutex> lk(g_solve_mu);
    auto it = g_solve_cache.find(key);
    if (it == g_solve_cache.end()) g_solve_cache[key] = E;
    else wl_engine_destroy(E);
  }
  const wl_solve_stats* S = stats ? stats : tmp.data();
  wl_status rc = WL_OK;
  for (int i = 0; i < nrhs; ++i) {
    if (S[i].status == ST_NAN) return WL_ERR_NAN;
    if (S[i].status != ST_CONVERGED) rc = WL_NOT_CONVERGED;
  }
  if (rc != WL_OK) ctx->err = "one or more right-hand sides did not converge";
  return rc;
}

// Release cached solve engines of a context (called before the context dies).
extern "C" void wl_release_solve_cache(wl_ctx* ctx) {
  std::lock_guard<std::mutex> lk(g_solve_mu);
  for (auto it = g_solve_cache.begin(); it != g_solve_cache.end();) {
    if (it->first.ctx == ctx) {
      wl_engine_destroy(it->second);
      it = g_solve_cache.erase(it);
    } else {
      ++it;
    }
  }
}

// ============================================================== allocation-free Schur normal operator
// Some callers cannot call cudaMalloc: a JAX/XLA custom-call handler runs with
// device memory owned by the framework (JAX preallocates most of the GPU at
// start-up, so an allocation made from inside the handler can fail), and
// latency-critical serving loops avoid the allocator's implicit device
// synchronisation.  wl_apply(WL_OP_SCHUR_E_NORMAL) allocates its two
// intermediate fields on first use; this variant takes them from a fixed
// file-scope device array instead and allocates nothing.
static constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;  // 64 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
static std::mutex g_noalloc_mu;
static void* g_noalloc_ptr[64] = {nullptr};

// Device address of the scratch array for ctx->device.  Resolved once per
// device (with that device current) and cached for the life of the process, so
// the library must not be used across a cudaDeviceReset of that device; host
// code must never use the symbol itself as a device pointer.
static wl_status noalloc_scratch(wl_ctx* ctx, void** out) {
  if (ctx->device < 0 || ctx->device >= 64) WL_FAIL(ctx, WL_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[ctx->device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      ctx->err = std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e);
      return WL_ERR_CUDA;
    }
    g_noalloc_ptr[ctx->device] = p;
  }
  *out = g_noalloc_ptr[ctx->device];
  return WL_OK;
}

extern "C" wl_status wl_apply_schur_normal_noalloc(wl_ctx* ctx, wl_gauge* G, double mass, unsigned flags,
                                                   const void* in, void* out, int nrhs) {
  if (!ctx || !G || !in || !out) WL_FAIL(ctx, WL_ERR_ARG, "null argument");
  if (in == out) WL_FAIL(ctx, WL_ERR_ARG, "in and out must not alias");
  if (nrhs <= 0) WL_FAIL(ctx, WL_ERR_ARG, "nrhs must be positive");
  const Geom& g = ctx->g;
  const size_t fbytes = (size_t)nrhs * g.V * 12 * sizeof(double2);
  if (2 * fbytes > kNoAllocScratchBytes)
    WL_FAIL(ctx, WL_ERR_ARG,
            "wl_apply_schur_normal_noalloc needs " + std::to_string(2 * fbytes) +
                " bytes of scratch (2 * nrhs * volume * 192) but its static scratch holds " +
                std::to_string(kNoAllocScratchBytes) + " bytes (nrhs * volume <= 174762)");
  WL_CUDA(ctx, cudaSetDevice(ctx->device));
  void* scratch = nullptr;
  wl_status s = noalloc_scratch(ctx, &scratch);
  if (s != WL_OK) return s;
  // t1 holds K_oe x on odd sites, y holds M x on even sites; each kernel reads
  // only the sites the previous one wrote, so neither needs clearing.
  void* t1 = scratch;
  void* y = static_cast<char*>(scratch) + fbytes;
  const bool norm = (flags & WL_FLAG_NORMALIZED) != 0;
  const double m0 = mass + 4.0;
  const double c0 = norm ? 1.0 : m0;
  const double c1 = norm ? 0.5 / (m0 * m0) : 0.5 / m0;
  WL_CUDA(ctx, cudaMemsetAsync(out, 0, fbytes, ctx->stream));  // odd sites of the result are zero
  ref_hop<false>(ctx, G, in, t1, nullptr, 0.0, -0.5, nrhs, 1, 1);
  ref_hop<false>(ctx, G, t1, y, in, c0, c1, nrhs, 0, 1);
  ref_hop<true>(ctx, G, y, t1, nullptr, 0.0, -0.5, nrhs, 1, 1);
  ref_hop<true>(ctx, G, t1, out, y, c0, c1, nrhs, 0, 1);
  return check_launch(ctx, "wl_apply_schur_normal_noalloc");
}
