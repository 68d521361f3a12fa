/*
 * CPU restatement (C99 + pthreads, FP64) of jaxQFT's even-odd preconditioned
 * Wilson normal operator and its CG solve -- TEST INFRASTRUCTURE ONLY.
 *
 * It restates jaxqft/models/su3_wilson_nf2.py:934-988 (compact parity hops
 * and the normalized Schur operator M = 1 - K_eo K_oe / m0^2) and the CG
 * recurrence that jax.scipy.sparse.linalg.cg runs for solve_eop_even_normal
 * (su3_wilson_nf2.py:1370-1392).  Used by tests (parity against the numpy
 * oracle) and as the timed CPU baseline of bench.py; never by the product.
 *
 * Layouts: links as the reference's BMXYIJ complex128 [4][V][3][3]; compact
 * fields complex128 [Vh][4][3] in ascending flat-index order of one parity.
 */
#include <complex.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ---------------------------------------------------------- parallel for */
typedef void (*range_fn)(void* arg, size_t lo, size_t hi, int tid);
typedef struct {
  range_fn fn;
  void* arg;
  size_t lo, hi;
  int tid;
} job_t;

static int g_threads = 0;

int wcpu_threads(void) {
  if (g_threads <= 0) {
    const char* e = getenv("WCPU_THREADS");
    long n = e ? atol(e) : sysconf(_SC_NPROCESSORS_ONLN);
    g_threads = n > 0 ? (int)n : 1;
    if (g_threads > 256) g_threads = 256;
  }
  return g_threads;
}

static void* job_run(void* p) {
  job_t* j = (job_t*)p;
  j->fn(j->arg, j->lo, j->hi, j->tid);
  return NULL;
}

static void par_for(size_t n, range_fn fn, void* arg) {
  int T = wcpu_threads();
  if (T == 1 || n < 4096) {
    fn(arg, 0, n, 0);
    return;
  }
  pthread_t th[256];
  job_t jobs[256];
  for (int t = 0; t < T; ++t) {
    jobs[t].fn = fn;
    jobs[t].arg = arg;
    jobs[t].lo = n * t / T;
    jobs[t].hi = n * (t + 1) / T;
    jobs[t].tid = t;
    if (t > 0) pthread_create(&th[t], NULL, job_run, &jobs[t]);
  }
  job_run(&jobs[0]);
  for (int t = 1; t < T; ++t) pthread_join(th[t], NULL);
}

typedef double complex cplx;

typedef struct {
  int L[4];
  int V, Vh;
  cplx ph[4];
  const cplx* U; /* [4][V][9] */
  double m0;
  int* nbr;      /* [2 parities][4 mu][2 dir][Vh] compact neighbour index */
  int* flat;     /* [2][Vh] flat index of compact site */
} wcpu;

static int flat_of(const int* L, const int* x) { return ((x[0] * L[1] + x[1]) * L[2] + x[2]) * L[3] + x[3]; }

wcpu* wcpu_create(const int* dims, const double* bc_re, const double* bc_im, const void* U, double mass) {
  wcpu* w = (wcpu*)calloc(1, sizeof(wcpu));
  for (int m = 0; m < 4; ++m) {
    w->L[m] = dims[m];
    w->ph[m] = bc_re[m] + I * bc_im[m];
  }
  w->V = dims[0] * dims[1] * dims[2] * dims[3];
  w->Vh = w->V / 2;
  w->U = (const cplx*)U;
  w->m0 = mass + 4.0;
  w->nbr = (int*)malloc(sizeof(int) * 16 * w->Vh);
  w->flat = (int*)malloc(sizeof(int) * 2 * w->Vh);
  int cnt[2] = {0, 0};
  int x[4];
  for (x[0] = 0; x[0] < w->L[0]; ++x[0])
    for (x[1] = 0; x[1] < w->L[1]; ++x[1])
      for (x[2] = 0; x[2] < w->L[2]; ++x[2])
        for (x[3] = 0; x[3] < w->L[3]; ++x[3]) {
          int p = (x[0] + x[1] + x[2] + x[3]) & 1;
          w->flat[p * w->Vh + cnt[p]++] = flat_of(w->L, x);
        }
  for (int p = 0; p < 2; ++p)
    for (int c = 0; c < w->Vh; ++c) {
      int f = w->flat[p * w->Vh + c];
      int y[4] = {f / (w->L[1] * w->L[2] * w->L[3]), (f / (w->L[2] * w->L[3])) % w->L[1], (f / w->L[3]) % w->L[2],
                  f % w->L[3]};
      for (int mu = 0; mu < 4; ++mu)
        for (int d = 0; d < 2; ++d) {
          int z[4] = {y[0], y[1], y[2], y[3]};
          z[mu] = (z[mu] + (d == 0 ? 1 : -1) + w->L[mu]) % w->L[mu];
          /* the compact index of a site is flat/2 when Lt is even */
          w->nbr[((p * 4 + mu) * 2 + d) * w->Vh + c] = flat_of(w->L, z) / 2;
        }
    }
  return w;
}

void wcpu_destroy(wcpu* w) {
  if (!w) return;
  free(w->nbr);
  free(w->flat);
  free(w);
}

/* (1 + c g_mu) psi for the Euclidean basis of jaxqft/fermions/gamma.py:14-46 */
static void gamma_apply(int mu, const cplx* s, cplx* o) {
  /* o = g_mu s (spin index major, 3 colours) */
  for (int c = 0; c < 3; ++c) {
    cplx s0 = s[0 * 3 + c], s1 = s[1 * 3 + c], s2 = s[2 * 3 + c], s3 = s[3 * 3 + c];
    switch (mu) {
      case 0: o[0 * 3 + c] = s3; o[1 * 3 + c] = s2; o[2 * 3 + c] = s1; o[3 * 3 + c] = s0; break;
      case 1: o[0 * 3 + c] = -I * s3; o[1 * 3 + c] = I * s2; o[2 * 3 + c] = -I * s1; o[3 * 3 + c] = I * s0; break;
      case 2: o[0 * 3 + c] = -I * s2; o[1 * 3 + c] = -I * s3; o[2 * 3 + c] = I * s0; o[3 * 3 + c] = I * s1; break;
      default: o[0 * 3 + c] = s0; o[1 * 3 + c] = s1; o[2 * 3 + c] = -s2; o[3 * 3 + c] = -s3; break;
    }
  }
}

/* out_c = -1/2 sum_mu [(1 + sf g) U psi(x+mu) + (1 - sf g) U^dag(x-mu) psi(x-mu)], sf = sign */
typedef struct {
  const wcpu* w;
  int target, sign;
  const cplx* in;
  cplx* out;
} hop_args;

static void hop_range(void* a_, size_t lo, size_t hi, int tid) {
  (void)tid;
  hop_args* a = (hop_args*)a_;
  const wcpu* w = a->w;
  const int target = a->target, sign = a->sign;
  const cplx* in = a->in;
  cplx* out = a->out;
  const int Vh = w->Vh;
  for (int c = (int)lo; c < (int)hi; ++c) {
    cplx acc[12] = {0};
    int f = w->flat[target * Vh + c];
    int x[4] = {f / (w->L[1] * w->L[2] * w->L[3]), (f / (w->L[2] * w->L[3])) % w->L[1], (f / w->L[3]) % w->L[2],
                f % w->L[3]};
    for (int mu = 0; mu < 4; ++mu) {
      for (int d = 0; d < 2; ++d) {
        int nb = w->nbr[((target * 4 + mu) * 2 + d) * Vh + c];
        const cplx* s = in + (size_t)nb * 12;
        cplx us[12], gs[12];
        if (d == 0) {
          const cplx* u = w->U + ((size_t)mu * w->V + f) * 9;
          cplx ph = (x[mu] == w->L[mu] - 1) ? w->ph[mu] : 1.0;
          for (int sp = 0; sp < 4; ++sp)
            for (int a = 0; a < 3; ++a)
              us[sp * 3 + a] = ph * (u[a * 3 + 0] * s[sp * 3 + 0] + u[a * 3 + 1] * s[sp * 3 + 1] + u[a * 3 + 2] * s[sp * 3 + 2]);
        } else {
          int fb = w->flat[(1 - target) * Vh + nb];
          const cplx* u = w->U + ((size_t)mu * w->V + fb) * 9;
          cplx ph = (x[mu] == 0) ? conj(w->ph[mu]) : 1.0;
          for (int sp = 0; sp < 4; ++sp)
            for (int a = 0; a < 3; ++a)
              us[sp * 3 + a] = ph * (conj(u[0 * 3 + a]) * s[sp * 3 + 0] + conj(u[1 * 3 + a]) * s[sp * 3 + 1] +
                                     conj(u[2 * 3 + a]) * s[sp * 3 + 2]);
        }
        gamma_apply(mu, us, gs);
        double cf = (d == 0) ? (double)sign : -(double)sign;
        for (int k = 0; k < 12; ++k) acc[k] += us[k] + cf * gs[k];
      }
    }
    for (int k = 0; k < 12; ++k) out[(size_t)c * 12 + k] = -0.5 * acc[k];
  }
}

static void hop(const wcpu* w, int target, int sign, const cplx* in, cplx* out) {
  hop_args a = {w, target, sign, in, out};
  par_for((size_t)w->Vh, hop_range, &a);
}

/* out = K in on compact fields: target-parity sites of -1/2 sum_mu [...] above
   (sign -1: the hop of D, +1: of D^dag).  Exported for full-size operator checks. */
void wcpu_hop(const wcpu* w, int target, int sign, const void* in, void* out) {
  hop(w, target, sign, (const cplx*)in, (cplx*)out);
}

/* vector kernels */
typedef struct {
  int kind;
  double a, b;
  const cplx *x, *y;
  cplx *u, *v;
  double part[256];
} vec_args;

static void vec_range(void* a_, size_t lo, size_t hi, int tid) {
  vec_args* a = (vec_args*)a_;
  double s = 0.0;
  for (size_t i = lo; i < hi; ++i) {
    switch (a->kind) {
      case 0: a->u[i] = a->x[i] - a->a * a->u[i]; break;            /* u = x - a u */
      case 1: s += creal(conj(a->x[i]) * a->y[i]); break;           /* dot */
      case 2: a->u[i] += a->a * a->x[i]; a->v[i] -= a->a * a->y[i]; break; /* x += a p, r -= a Ap */
      default: a->u[i] = a->x[i] + a->b * a->u[i]; break;           /* p = r + b p */
    }
  }
  a->part[tid] = s;
}

/* M x = x - K_eo K_oe x / m0^2 (dagger: with K^dag blocks) */
static void schur(const wcpu* w, int dag, const cplx* x, cplx* tmp_o, cplx* out) {
  int sign = dag ? +1 : -1;
  hop(w, 1, sign, x, tmp_o);
  hop(w, 0, sign, tmp_o, out);
  vec_args va;
  memset(&va, 0, sizeof(va));
  va.kind = 0;
  va.a = 1.0 / (w->m0 * w->m0);
  va.x = x;
  va.u = out;
  par_for((size_t)w->Vh * 12, vec_range, &va);
}

void wcpu_normal(const wcpu* w, const void* x, void* out) {
  size_t n = (size_t)w->Vh * 12;
  cplx* t = (cplx*)malloc(sizeof(cplx) * n);
  cplx* y = (cplx*)malloc(sizeof(cplx) * n);
  schur(w, 0, (const cplx*)x, t, y);
  schur(w, 1, y, t, (cplx*)out);
  free(t);
  free(y);
}

static double dotr(const cplx* a, const cplx* b, size_t n) {
  vec_args va;
  memset(&va, 0, sizeof(va));
  va.kind = 1;
  va.x = a;
  va.y = b;
  par_for(n, vec_range, &va);
  double s = 0.0;
  int T = (n < 4096) ? 1 : wcpu_threads();
  for (int t = 0; t < T; ++t) s += va.part[t];
  return s;
}

/* CG on M^dag M x = b (x = 0 start) until ||r||^2 <= tol^2 ||b||^2 or maxiter.
   Returns iterations; writes the recursive residual norm ratio to *res. */
int wcpu_cg(const wcpu* w, const void* bv, void* xv, double tol, int maxiter, double* res) {
  size_t n = (size_t)w->Vh * 12;
  const cplx* b = (const cplx*)bv;
  cplx* x = (cplx*)xv;
  cplx* r = (cplx*)malloc(sizeof(cplx) * n);
  cplx* p = (cplx*)malloc(sizeof(cplx) * n);
  cplx* Ap = (cplx*)malloc(sizeof(cplx) * n);
  cplx* t = (cplx*)malloc(sizeof(cplx) * n);
  cplx* y = (cplx*)malloc(sizeof(cplx) * n);
  memset(x, 0, sizeof(cplx) * n);
  memcpy(r, b, sizeof(cplx) * n);
  memcpy(p, b, sizeof(cplx) * n);
  double b2 = dotr(b, b, n), g = b2;
  int k = 0;
  while (g > tol * tol * b2 && k < maxiter) {
    schur(w, 0, p, t, y);
    schur(w, 1, y, t, Ap);
    double alpha = g / dotr(p, Ap, n);
    vec_args va;
    memset(&va, 0, sizeof(va));
    va.kind = 2;
    va.a = alpha;
    va.x = p;
    va.y = Ap;
    va.u = x;
    va.v = r;
    par_for(n, vec_range, &va);
    double g2 = dotr(r, r, n);
    double beta = g2 / g;
    memset(&va, 0, sizeof(va));
    va.kind = 3;
    va.b = beta;
    va.x = r;
    va.u = p;
    par_for(n, vec_range, &va);
    g = g2;
    ++k;
  }
  if (res) *res = sqrt(g / b2);
  free(r);
  free(p);
  free(Ap);
  free(t);
  free(y);
  return k;
}
