/*
 * wilson_sm100.h -- C-ABI of libwilson_sm100.so, the sm_100a (B200) SU(3)
 * Wilson-fermion hot path: Dirac operator D, D^dag, even-odd Schur blocks,
 * mixed-precision multi-RHS CG, and the Nf=2 pseudofermion force.
 *
 * Conventions (identical to jaxQFT's):
 *   - gauge field: one configuration, complex128 interleaved, layout BMXYIJ
 *     [mu=4][Lx][Ly][Lz][Lt][3][3]  (jaxqft/models/su3_ym.py:246-249)
 *   - fermion field: complex128 [nrhs][Lx][Ly][Lz][Lt][Ns=4][Nc=3], t fastest
 *     (jaxqft/models/su3_wilson_nf2.py:815-817)
 *   - D = (m + 4r) - 1/2 sum_mu [(r - g_mu) U_mu(x) psi(x+mu) + (r + g_mu) U_mu^dag(x-mu) psi(x-mu)]
 *     with the Euclidean gammas of jaxqft/fermions/gamma.py:14-46, r = 1
 *   - boundary phase bc[mu] multiplies U_mu(x) on x_mu = L_mu - 1
 *     (jaxqft/models/su3_wilson_nf2.py:726-759)
 * All field pointers are DEVICE pointers owned by the caller.  Every call is
 * asynchronous on the context's stream unless stated otherwise.  A context is
 * not thread-safe: callers serialise calls on one context.  No C++ exception
 * crosses this boundary; every call returns a wl_status and, on failure,
 * wl_last_error() describes it.
 */
#ifndef WILSON_SM100_H
#define WILSON_SM100_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  WL_OK = 0,
  WL_ERR_ARG = 1,         /* invalid argument (shape, parity, op, null pointer) */
  WL_ERR_OOM = 2,         /* device allocation failed / HBM budget exceeded */
  WL_NOT_CONVERGED = 3,   /* a solve stopped at maxiter (per-RHS status says which) */
  WL_ERR_NAN = 4,         /* a solve produced a non-finite residual */
  WL_ERR_TIMEOUT = 5,     /* a bounded device wait ran out */
  WL_ERR_CUDA = 6,        /* CUDA runtime error */
  WL_ERR_STATE = 7        /* call not valid in the current state */
} wl_status;

typedef enum { WL_PREC_DOUBLE = 0, WL_PREC_SINGLE = 1, WL_PREC_HALF = 2 } wl_prec;

typedef enum {
  /* full-lattice operators (jaxqft/models/su3_wilson_nf2.py:1036-1055, 1101-1105) */
  WL_OP_D = 0,          /* apply_D */
  WL_OP_DDAG = 1,       /* apply_Ddag */
  WL_OP_DDAGD = 2,      /* apply_normal: D^dag (D psi) */
  WL_OP_HOP = 3,        /* apply_offdiag: K = D - m0 */
  WL_OP_HOP_DAG = 4,    /* apply_offdiag_dagger */
  /* masked even/odd blocks on full-lattice fields (1057-1099): input projected
     to the source parity, output zero on the other parity */
  WL_OP_K_OE = 5,       /* apply_K_oe  (even -> odd) */
  WL_OP_K_EO = 6,       /* apply_K_eo  (odd -> even) */
  WL_OP_KDAG_OE = 7,    /* apply_Kdag_oe */
  WL_OP_KDAG_EO = 8,    /* apply_Kdag_eo */
  /* Schur complements (1112-1155): S_e = m0 - (1/m0) K_eo K_oe, normalized = S_e / m0 */
  WL_OP_SCHUR_E = 9,      /* apply_eo_schur_even */
  WL_OP_SCHUR_E_DAG = 10, /* apply_eo_schur_even_dagger */
  WL_OP_SCHUR_O = 11,     /* apply_eo_schur_odd */
  WL_OP_SCHUR_E_NORMAL = 12 /* S_e^dag S_e (the operator solve_eop_even_normal inverts) */
} wl_op;

#define WL_FLAG_NORMALIZED 1u

typedef struct {
  int dims[4];        /* Lx, Ly, Lz, Lt; all even */
  double bc_re[4];    /* boundary phase per direction */
  double bc_im[4];
} wl_geometry;

typedef struct wl_ctx wl_ctx;
typedef struct wl_gauge wl_gauge;
typedef struct wl_engine wl_engine;

/* Library / context ------------------------------------------------------ */
int wl_version(void);
/* Create a context for one lattice geometry on CUDA device `device`.
   Replaces the geometry set-up of SU3WilsonNf2.__post_init__
   (jaxqft/models/su3_wilson_nf2.py:625-709: BC factor, masks, EO maps).
   Every extent must be even and >= 2, else WL_ERR_ARG.  The reference
   accepts odd extents, but there a wrap by one site keeps the parity, so its
   EO neighbour maps (su3_wilson_nf2.py:847-882) hold -1 entries and its EO
   operators and solvers are not defined; only its unpreconditioned D is. */
wl_status wl_ctx_create(const wl_geometry* geom, int device, wl_ctx** out);
void wl_ctx_destroy(wl_ctx* ctx);
const char* wl_last_error(const wl_ctx* ctx);
/* Use `stream` (a cudaStream_t; NULL = legacy default) for subsequent calls. */
wl_status wl_ctx_set_stream(wl_ctx* ctx, void* stream);
wl_status wl_ctx_synchronize(wl_ctx* ctx);

/* Even/odd index maps for bit-exact checks (su3_wilson_nf2.py:831-882):
   even[Vh], odd[Vh] ascending flat indices; nbr[8][2][Vh] = compact index of
   the opposite-parity neighbour x+mu (dir 0) / x-mu (dir 1) of compact site k
   of parity p, laid out [p*4+mu][dir][k].  Host pointers, synchronous. */
wl_status wl_eo_maps(wl_ctx* ctx, int32_t* even, int32_t* odd, int32_t* nbr);

/* Gauge field ------------------------------------------------------------ */
/* Build the internal parity-split FP64 (18- and 12-real), FP32 and FP16
   12-real copies of one configuration.  Replaces _links_with_fermion_bc
   (su3_wilson_nf2.py:751-759), which the kernels apply by index instead.
   `U` stays owned by the caller and is not referenced after the call. */
wl_status wl_gauge_create(wl_ctx* ctx, const void* U, wl_gauge** out);
wl_status wl_gauge_update(wl_gauge* gauge, const void* U);
/* max over links of |U U^dag - 1| and |det U - 1| (synchronous) */
wl_status wl_gauge_unitarity(wl_gauge* gauge, double* err);
void wl_gauge_destroy(wl_gauge* gauge);

/* Operators on reference-layout fields, FP64 ----------------------------- */
/* out = op(in) for nrhs fields.  `mass` is the bare mass m (m0 = m + 4).
   `flags`: WL_FLAG_NORMALIZED for the Schur ops.  in and out must not alias. */
wl_status wl_apply(wl_ctx* ctx, wl_gauge* gauge, int op, double mass, unsigned flags,
                   const void* in, void* out, int nrhs);

/* Solver ------------------------------------------------------------------ */
typedef enum {
  WL_SOLVE_NORMAL = 0,    /* (D^dag D) x = b on the full lattice: solve_normal (1410-1432) */
  WL_SOLVE_EO_NORMAL = 1  /* (M^dag M) x_e = b_e, M = normalized even Schur:
                             solve_eop_even_normal (1370-1392) */
} wl_solve_op;

typedef struct {
  int op;            /* wl_solve_op */
  int inner_prec;    /* wl_prec of the iterated operator; FP64 = plain CG */
  double tol;        /* stop when ||b - A x|| <= tol ||b|| with A in FP64 */
  int maxiter;
  double delta;      /* reliable-update trigger: sloppy ||r|| < delta * max ||r|| since update */
  int use_x0;        /* x holds an initial guess on entry */
  int use_graph;     /* capture each CG iteration in a CUDA graph */
  int check_every;   /* iterations between host convergence polls (0 = default) */
} wl_solve_params;

typedef struct {
  int iters;            /* CG iterations */
  int reliable_updates; /* FP64 true-residual recomputations */
  int status;           /* 2 converged, 3 maxiter, 4 breakdown, 5 nan */
  double true_res;      /* ||b - A x|| / ||b|| in FP64 at exit */
} wl_solve_stats;

/* Solve nrhs independent systems sharing the gauge field, one batched CG
   (links streamed once per iteration for all RHS, converged RHS masked).
   b, x: reference-layout fields.  `masses` holds one bare mass per RHS.
   For WL_SOLVE_EO_NORMAL the odd sites of b are ignored and x is zero there,
   as the reference's _unpack_even_sites does.  Synchronous (returns when all
   RHS have stopped).  Replaces _solve_linear + jax.scipy.sparse.linalg.cg
   (su3_wilson_nf2.py:1243-1269) for the cg/normal forms. */
wl_status wl_solve(wl_ctx* ctx, wl_gauge* gauge, const wl_solve_params* params, const double* masses,
                   const void* b, void* x, int nrhs, wl_solve_stats* stats);

/* Continuous-batching engine: a fixed set of RHS slots that iterate together;
   a slot can be admitted while others are mid-solve and retired when done. */
wl_status wl_engine_create(wl_ctx* ctx, wl_gauge* gauge, const wl_solve_params* params, int nslots,
                           wl_engine** out);
void wl_engine_destroy(wl_engine* eng);
/* Admit `n` RHS into slots[0..n) (b: n consecutive reference-layout fields). */
wl_status wl_engine_admit(wl_engine* eng, const int* slots, int n, const void* b, const double* masses,
                          const double* tols, const int* maxiters);
/* Run `iters` iterations on all active slots (asynchronous). */
wl_status wl_engine_step(wl_engine* eng, int iters);
/* Run up to `max_iters` iterations on all active slots in one launch, stopping
   on the device as soon as a slot finishes (asynchronous; no counterpart in the
   reference, whose solves are synchronous): a host loop driving many engines
   then acts only when a slot can be retired.  Engines created without graphs
   run `max_iters` iterations as wl_engine_step does. */
wl_status wl_engine_run(wl_engine* eng, int max_iters);
/* Synchronise and report per-slot status (0 idle, 1 running, 2..5 stopped). */
wl_status wl_engine_poll(wl_engine* eng, int* status, int* n_active);
/* Non-blocking form of wl_engine_poll, for a host loop that drives many
   engines (no counterpart in the reference, whose solves are synchronous):
   wl_engine_poll_async queues the status copies on the engine stream behind the
   work queued so far and returns at once; wl_engine_poll_ready never blocks and
   returns 1 (status / n_active filled, as wl_engine_poll would), 0 while that
   work is still running, -1 with no poll queued, -2 on a CUDA error. */
wl_status wl_engine_poll_async(wl_engine* eng);
int wl_engine_poll_ready(wl_engine* eng, int* status, int* n_active);
/* Copy the solution of slot `slot` into x (reference layout) and free the slot. */
wl_status wl_engine_retire(wl_engine* eng, int slot, void* x, wl_solve_stats* stats);
/* Size in bytes of the engine's device allocations (for HBM admission). */
int64_t wl_engine_bytes(const wl_ctx* ctx, int op, int inner_prec, int nslots);
/* The cudaStream_t the engine runs on (for events / stream ordering). */
void* wl_engine_stream(wl_engine* eng);

/* Instrumentation (no counterpart in the reference) ----------------------- */
/* Time `reps` launches of the engine's dominant kernel (the iterated-precision
   hop over all slots, as the CG runs it) with CUDA events on the engine stream.
   Writes the mean milliseconds per launch and the algorithmic HBM bytes one
   launch must move (every link and spinor touched once). Synchronous. */
wl_status wl_engine_time_hop(wl_engine* eng, int reps, double* ms_per_launch, double* bytes_per_launch);
/* The same for the FP64 hop of the reliable update (x64 -> K_oe x64 over all
   slots, with the FP64 links and the shape the update uses). */
wl_status wl_engine_time_update_hop(wl_engine* eng, int reps, double* ms_per_launch, double* bytes_per_launch);
/* The same for the fused CG hop, the fourth hop of an iteration with the CG
   update in its epilogue (x_s += alpha p, r_s -= alpha A p, |r_s|^2); bytes =
   8 links per target site plus, per RHS, the gathered source and the y, p, x_s,
   r_s records read and x_s, r_s written.  It changes the slots' iteration
   fields: admit the slots again before stepping them. */
wl_status wl_engine_time_cg_hop(wl_engine* eng, int reps, double* ms_per_launch, double* bytes_per_launch);
/* Apply the engine's iterated (sloppy-precision) operator to one
   reference-layout field through slot 0's buffers, for testing the FP16/FP32
   operators against FP64: stage 0 -> K_oe x_e (odd sites of out), 1 -> M x_e,
   2 -> M^dag M x_e (EO engines; even sites of out), 3 -> D x, 4 -> D^dag D x,
   5 -> D^dag x (full-lattice engines).  Overwrites slot 0's work fields.  Synchronous. */
wl_status wl_engine_debug_apply(wl_engine* eng, int stage, double mass, const void* in, void* out);
/* Number of kernels this library has launched in the process so far
   (graph launches count every kernel node of the graph). */
int64_t wl_kernel_launches(void);

/* Checking builds (no counterpart in the reference; compiled with
   -DWL_BOUNDS_CHECK=1 as libwilson_sm100_check.so): the kernels compare every
   compact site index they decode or gather with the half volume, count the
   ones out of range, keep the first and use site 0 instead, so the access
   stays in bounds.  Returns the count on the current device since the last
   call and clears it (after a device synchronisation), with the first bad
   index in *first_bad; -1 in a build without the checks, -2 on a CUDA error. */
int64_t wl_bounds_errors(long long* first_bad);

/* Allocation-free operator (no counterpart in the reference) -------------- */
/* out = S_e^dag S_e in, exactly what wl_apply(WL_OP_SCHUR_E_NORMAL) computes,
   for callers that cannot call cudaMalloc: a JAX/XLA custom-call handler
   works in device memory the framework already owns (JAX preallocates most
   of the GPU), and latency-critical loops avoid the allocator's implicit
   synchronisation.  The two intermediate fields live in a 64 MiB static
   device array that every GPU loading this library holds until exit, so
   2 * nrhs * volume * 192 bytes must fit (nrhs * volume <= 174762, e.g. one
   16^3x32 field); larger requests return WL_ERR_ARG.  The first call on a
   device resolves the array's address with that device current; make it
   before any stream capture.  The address is kept for the life of the
   process, so the library must not be used across a cudaDeviceReset of that
   device.  All calls share the array: calls that overlap on the GPU
   (different streams or contexts of one device) race. */
wl_status wl_apply_schur_normal_noalloc(wl_ctx* ctx, wl_gauge* gauge, double mass, unsigned flags,
                                        const void* in, void* out, int nrhs);

/* Field inner products and combinations ----------------------------------- */
/* For the chronological initial-guess predictors (su3_wilson_nf2.py:85-194),
   on complex128 device vectors of `len` elements.  `a`, `b`, `x` are HOST
   arrays of device pointers.
   wl_field_dots: out[2k], out[2k+1] = Re, Im of <a_k, b_k> = sum conj(a_k) b_k
   for k < npairs <= 64 (host array; deterministic order of summation;
   synchronises the context stream).
   wl_field_combine: out = sum_k (coef[2k] + i coef[2k+1]) x_k, k < n <= 32;
   out may be one of the x_k.  Asynchronous on the context stream. */
wl_status wl_field_dots(wl_ctx* ctx, int npairs, const void* const* a, const void* const* b, int64_t len,
                        double* out);
wl_status wl_field_combine(wl_ctx* ctx, int n, const void* const* x, const double* coef, int64_t len, void* out);

/* Random fields ----------------------------------------------------------- */
/* Gaussian fields from a counter-based generator (Philox4x32-10 with key =
   seed; every value is a function of (seed, stream, position), so a given
   (seed, stream) always yields the same field).  Asynchronous on the context
   stream.  Replace the jax.random draws of random_fermion
   (jaxqft/models/su3_wilson_nf2.py:1169-1175) and of _sample_algebra /
   refresh_p (jaxqft/models/su3_ym.py:238-244, 339-347); the streams are not
   jax's threefry streams.
   wl_random_spinor: out [n][Lx][Ly][Lz][Lt][4][3] complex128, each component
   (g0 + i g1)/sqrt(2) with g0, g1 standard normal (E|z|^2 = 1).
   wl_random_algebra: P [batch][4][Lx][Ly][Lz][Lt][3][3] complex128 (BMXYIJ),
   P = TA(scale (G1 + i G2)), TA(X) = (X - X^dag)/2 - Tr(X - X^dag)/6. */
wl_status wl_random_spinor(wl_ctx* ctx, uint64_t seed, uint64_t stream, int n, void* out);
wl_status wl_random_algebra(wl_ctx* ctx, uint64_t seed, uint64_t stream, int batch, double scale, void* P);

/* Pseudofermion force ----------------------------------------------------- */
/* F = pseudofermion_force_from_solution(U, X, Y) (su3_wilson_nf2.py:1556-1576):
   F[mu][x] = TA( (c1 - c2)^T ), link-shaped complex128 BMXYIJ.  If
   `accumulate` is non-zero, F += coef * force, else F = coef * force. */
wl_status wl_pf_force(wl_ctx* ctx, wl_gauge* gauge, const void* X, const void* Y, double coef,
                      int accumulate, void* F);

/* Gauge sector (HMC pure-gauge pieces) ------------------------------------ */
/* Links / momenta in the reference layout BMXYIJ: complex128
   [batch][4][Lx][Ly][Lz][Lt][3][3], periodic boundaries (the fermion BC of the
   context does not apply).  All FP64. */

/* F = -(beta/3) TA(U_mu(x) V_mu(x)^dag), V the sum of the six staples
   (jaxqft/models/su3_ym.py:298-327 _staple / force_reference; su3_ym.py:96-123
   the BMXYIJ form).  F has U's shape. */
wl_status wl_gauge_force(wl_ctx* ctx, const void* U, int batch, double beta, void* F);

/* Uout = exp(dt P) U per link (su3_ym.py:349-350 evolve_q_reference with
   exp_method "expm", su3_ym.py:265-272).  Uout may alias U. */
wl_status wl_gauge_evolve(wl_ctx* ctx, const void* P, const void* U, int batch, double dt, void* Uout);

/* plaq_sum[b] = sum_{x, mu<nu} Re Tr U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag
   (host array; su3_ym.py:274-286 action = -(beta/3) plaq_sum, 369-388
   average_plaquette = plaq_sum / (3 V 6)).  Synchronises the context stream. */
wl_status wl_gauge_plaquette_sum(wl_ctx* ctx, const void* U, int batch, double* plaq_sum);

/* kin[b] = -1/2 sum Re Tr P P (host array; su3_ym.py:362-364).  Synchronises. */
wl_status wl_momentum_kinetic(wl_ctx* ctx, const void* P, int batch, double* kin);

/* Measurements -------------------------------------------------------------- */
/* Pion two-point function of point-source propagator columns
   (jaxqft/core/measurements.py:375-390): corr[dt] = sum over the timeslice
   t = source_t + dt (mod Lt) of |S|^2 summed over all `ncol` columns (fermion
   fields [ncol][Lx][Ly][Lz][Lt][4][3] complex128, device) and their spin and
   colour.  corr is a host array of Lt doubles.  Synchronises the context stream. */
wl_status wl_pion_correlator(wl_ctx* ctx, const void* prop, int ncol, int source_t, double* corr);

#ifdef __cplusplus
}
#endif
#endif /* WILSON_SM100_H */
