// Pure-gauge pieces of the SU(3) HMC on the device, reference layout BMXYIJ
// (links [B][mu][Lx][Ly][Lz][Lt][3][3] complex128, t fastest, periodic):
//   * Wilson plaquette sum  sum_{x, mu<nu} Re Tr U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag
//     (jaxqft/models/su3_ym.py:274-286 action_reference, 369-388 average_plaquette)
//   * gauge force  F_mu(x) = -(beta/3) TA(U_mu(x) V_mu(x)^dag) with the staple
//     V_mu(x) = sum_{nu != mu} U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag + U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu)
//     (su3_ym.py:298-327 _staple / force_reference)
//   * exponential drift  U <- exp(dt P) U  (su3_ym.py:349-350 evolve_q_reference with
//     exp_method "expm", su3_ym.py:265-272)
//   * kinetic term  -1/2 sum Re Tr P P  (su3_ym.py:362-364)
// All FP64.  One thread per link (force, drift, kinetic) or per site (plaquette);
// sums are deterministic block partials finished by reduce_finalize_kernel.
#pragma once
#include "wl_hop.cuh"

namespace wl {

struct M3 {
  cplx<double> m[3][3];
};

WL_D void m3_load(M3& a, const double2* p) {
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const double2 v = ldg(p + k);
    a.m[k / 3][k % 3] = {v.x, v.y};
  }
}

WL_D void m3_store(const M3& a, double2* p) {
#pragma unroll
  for (int k = 0; k < 9; ++k) p[k] = make_double2(a.m[k / 3][k % 3].re, a.m[k / 3][k % 3].im);
}

// c = a b ; c = a b^dag ; c = a^dag b
WL_D void m3_mul(const M3& a, const M3& b, M3& c) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cplx<double> s = {0.0, 0.0};
#pragma unroll
      for (int k = 0; k < 3; ++k) fma_(s, a.m[i][k], b.m[k][j]);
      c.m[i][j] = s;
    }
}
WL_D void m3_mul_nd(const M3& a, const M3& b, M3& c) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cplx<double> s = {0.0, 0.0};
#pragma unroll
      for (int k = 0; k < 3; ++k) fmac_(s, b.m[j][k], a.m[i][k]);  // a_ik conj(b_jk)
      c.m[i][j] = s;
    }
}
WL_D void m3_mul_dn(const M3& a, const M3& b, M3& c) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cplx<double> s = {0.0, 0.0};
#pragma unroll
      for (int k = 0; k < 3; ++k) fmac_(s, a.m[k][i], b.m[k][j]);  // conj(a_ki) b_kj
      c.m[i][j] = s;
    }
}

// Re Tr(a b^dag) = sum_ij Re(a_ij conj(b_ij))
WL_D double m3_retr_nd(const M3& a, const M3& b) {
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) s += a.m[i][j].re * b.m[i][j].re + a.m[i][j].im * b.m[i][j].im;
  return s;
}

// TA(x) = (x - x^dag)/2 - Tr(x - x^dag)/6 * 1   (su3_ym.py:56-67)
WL_D void m3_ta(const M3& x, M3& y, double coef) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      y.m[i][j] = {0.5 * (x.m[i][j].re - x.m[j][i].re), 0.5 * (x.m[i][j].im + x.m[j][i].im)};
  const double tr = (y.m[0][0].im + y.m[1][1].im + y.m[2][2].im) / 3.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) y.m[i][i].im -= tr;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) y.m[i][j] = coef * y.m[i][j];
}

// exp(A) by a degree-14 Taylor polynomial (Horner) after scaling A by 2^-s so that
// its max-row-sum norm is <= 1/2, then s squarings (scaling and squaring, as in
// Moler and Van Loan, "Nineteen dubious ways to compute the exponential of a
// matrix", method 3).  Truncation error <= 0.5^15/15! ~ 2e-17 relative.
WL_D void m3_exp(const M3& A, M3& E) {
  double nrm = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double r = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j) r += fabs(A.m[i][j].re) + fabs(A.m[i][j].im);
    nrm = fmax(nrm, r);
  }
  int s = 0;
  while (nrm > 0.5 && s < 64) {  // bounded: at most 64 halvings
    nrm *= 0.5;
    ++s;
  }
  const double sc = ldexp(1.0, -s);
  M3 a;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) a.m[i][j] = sc * A.m[i][j];
  // E = I + a/1 (I + a/2 (I + ... (I + a/14)))
  M3 t;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) E.m[i][j] = {i == j ? 1.0 : 0.0, 0.0};
#pragma unroll 1
  for (int k = 14; k >= 1; --k) {
    m3_mul(a, E, t);
    const double inv = 1.0 / k;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) E.m[i][j] = {(i == j ? 1.0 : 0.0) + inv * t.m[i][j].re, inv * t.m[i][j].im};
  }
#pragma unroll 1
  for (int q = 0; q < s; ++q) {
    m3_mul(E, E, t);
    E = t;
  }
}

struct GaugeArgs {
  Geom g;
  const double2* U;  // [B][4][V][9]
  const double2* P;  // [B][4][V][9] (drift, kinetic)
  double2* out;      // [B][4][V][9]
  int batch;
  double coef;       // force: -beta/3 ; drift: dt
  double* partials;  // [batch][nblk]
};

WL_D long long gflat(const Geom& g, int x0, int x1, int x2, int x3) {
  return (((long long)x0 * g.L[1] + x1) * g.L[2] + x2) * g.L[3] + x3;
}

WL_D void gcoords(const Geom& g, long long f, int (&x)[4]) {
  x[3] = (int)(f % g.L[3]);
  f /= g.L[3];
  x[2] = (int)(f % g.L[2]);
  f /= g.L[2];
  x[1] = (int)(f % g.L[1]);
  x[0] = (int)(f / g.L[1]);
}

WL_D long long gshift(const Geom& g, const int (&x)[4], int mu, int dmu, int nu, int dnu) {
  int y[4] = {x[0], x[1], x[2], x[3]};
  y[mu] += dmu;
  y[nu] += dnu;
#pragma unroll
  for (int d = 0; d < 4; ++d) y[d] = y[d] < 0 ? y[d] + g.L[d] : (y[d] >= g.L[d] ? y[d] - g.L[d] : y[d]);
  return gflat(g, y[0], y[1], y[2], y[3]);
}

WL_D const double2* glink(const GaugeArgs& A, const double2* base, int b, int mu, long long f) {
  return base + (((long long)b * 4 + mu) * A.g.V + f) * 9;
}

// grid: x over sites, y = mu, z = batch
__global__ void __launch_bounds__(128) gauge_force_kernel(GaugeArgs A) {
  const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int mu = blockIdx.y, b = blockIdx.z;
  if (f >= A.g.V) return;
  int x[4];
  gcoords(A.g, f, x);
  M3 st, t1, t2, u1, u2, u3;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) st.m[i][j] = {0.0, 0.0};
#pragma unroll 1
  for (int nu = 0; nu < 4; ++nu) {
    if (nu == mu) continue;
    // forward: U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag
    m3_load(u1, glink(A, A.U, b, nu, f));
    m3_load(u2, glink(A, A.U, b, mu, gshift(A.g, x, nu, +1, mu, 0)));
    m3_load(u3, glink(A, A.U, b, nu, gshift(A.g, x, mu, +1, nu, 0)));
    m3_mul(u1, u2, t1);
    m3_mul_nd(t1, u3, t2);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) st.m[i][j] = st.m[i][j] + t2.m[i][j];
    // backward: U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu)
    const long long fm = gshift(A.g, x, nu, -1, mu, 0);
    m3_load(u1, glink(A, A.U, b, nu, fm));
    m3_load(u2, glink(A, A.U, b, mu, fm));
    m3_load(u3, glink(A, A.U, b, nu, gshift(A.g, x, nu, -1, mu, +1)));
    m3_mul_dn(u1, u2, t1);
    m3_mul(t1, u3, t2);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) st.m[i][j] = st.m[i][j] + t2.m[i][j];
  }
  m3_load(u1, glink(A, A.U, b, mu, f));
  m3_mul_nd(u1, st, t1);  // U_mu(x) V^dag
  m3_ta(t1, t2, A.coef);
  m3_store(t2, A.out + (((long long)b * 4 + mu) * A.g.V + f) * 9);
}

// out = exp(coef * P) U, one thread per link (grid.x over all B*4*V links)
__global__ void __launch_bounds__(128) gauge_evolve_kernel(GaugeArgs A) {
  const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= (long long)A.batch * 4 * A.g.V) return;
  M3 p, e, u, r;
  m3_load(p, A.P + l * 9);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) p.m[i][j] = A.coef * p.m[i][j];
  m3_exp(p, e);
  m3_load(u, A.U + l * 9);
  m3_mul(e, u, r);
  m3_store(r, A.out + l * 9);
}

// per-site plaquette sums (grid: x over sites, z = batch); partials[b][block]
__global__ void __launch_bounds__(128) gauge_plaquette_kernel(GaugeArgs A) {
  __shared__ double sm[32];
  const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.z;
  double v[1] = {0.0};
  if (f < A.g.V) {
    int x[4];
    gcoords(A.g, f, x);
    M3 um, un, a, c, t;
#pragma unroll 1
    for (int mu = 0; mu < 4; ++mu) {
      m3_load(um, glink(A, A.U, b, mu, f));
#pragma unroll 1
      for (int nu = mu + 1; nu < 4; ++nu) {
        // Re Tr (U_mu(x) U_nu(x+mu)) (U_nu(x) U_mu(x+nu))^dag
        m3_load(t, glink(A, A.U, b, nu, gshift(A.g, x, mu, +1, nu, 0)));
        m3_mul(um, t, a);
        m3_load(un, glink(A, A.U, b, nu, f));
        m3_load(t, glink(A, A.U, b, mu, gshift(A.g, x, nu, +1, mu, 0)));
        m3_mul(un, t, c);
        v[0] += m3_retr_nd(a, c);
      }
    }
  }
  block_sum<1>(v, sm);
  if (threadIdx.x == 0) A.partials[(long long)b * gridDim.x + blockIdx.x] = v[0];
}

// -1/2 Re Tr P P per link (grid: x over links of one configuration, z = batch)
__global__ void __launch_bounds__(128) gauge_kinetic_kernel(GaugeArgs A) {
  __shared__ double sm[32];
  const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.z;
  double v[1] = {0.0};
  if (l < 4LL * A.g.V) {
    M3 p;
    m3_load(p, A.P + ((long long)b * 4 * A.g.V + l) * 9);
    double s = 0.0;  // Re Tr P P = sum_ij Re(p_ij p_ji)
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) s += p.m[i][j].re * p.m[j][i].re - p.m[i][j].im * p.m[j][i].im;
    v[0] = -0.5 * s;
  }
  block_sum<1>(v, sm);
  if (threadIdx.x == 0) A.partials[(long long)b * gridDim.x + blockIdx.x] = v[0];
}

}  // namespace wl
