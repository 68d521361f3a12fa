// Nf=2 pseudofermion link force from a pair of solutions (X, Y), reference layout.
//
// Restates jaxqft/models/su3_wilson_nf2.py:1556-1576 per link (x, mu), with
// the boundary-phased link U = U_mu(x) (phase on x_mu = L_mu - 1):
//   c1_ac = sum_s conj(Y(x))_sa  [ (1 - g_mu) U X(x+mu) ]_sc
//   c2_dc = sum_s conj(U Y(x+mu))_sd [ (1 + g_mu) X(x) ]_sc
//   F_mu(x) = TA( transpose(c1 - c2) ),  TA(k) = (k - k^dag)/2 - tr/3
// (c2 follows from the reference's einsum "sa,st,ad,tc->dc" by moving U^dag
// onto Y(x+mu)).  One thread per (site, mu); output link-shaped BMXYIJ.
#pragma once
#include "wl_hop.cuh"

namespace wl {

template <int MU>
WL_D void force_link(const Geom& g, const LinkField<L_REF>& U, const SpinorRef& X, const SpinorRef& Y, const Site& s,
                     long long f, Link<double>& k) {
  const long long fp = IdxFlat::nb(g, s, MU, +1);
  Link<double> u;
  U.load_flat(u, MU, f);
  if (g.ph_on[MU] && s.x[MU] == g.L[MU] - 1) {
    cplx<double> ph = {g.ph_re[MU], g.ph_im[MU]};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) u.m[i][j] = u.m[i][j] * ph;
  }
  Spinor<double> xp, yx, xx, yp;
  X.load(xp, 0, fp);
  Y.load(yx, 0, f);
  X.load(xx, 0, f);
  Y.load(yp, 0, fp);
  // W = (1 - g) U X(x+mu) ; V = (1 + g) X(x) ; Z = U Y(x+mu)
  Spinor<double> W, V, Z;
  zero(W);
  zero(V);
  {
    Half<double> h, uh;
    spin_project<MU, -1>(xp, h);
    color_mul<false>(u, h, uh);
    spin_accum<MU, -1>(W, uh);
    spin_project<MU, +1>(xx, h);
    spin_accum<MU, +1>(V, h);
  }
#pragma unroll
  for (int sp = 0; sp < 4; ++sp)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      cplx<double> acc = {0.0, 0.0};
#pragma unroll
      for (int b = 0; b < 3; ++b) fma_(acc, u.m[a][b], yp.v[sp][b]);
      Z.v[sp][a] = acc;
    }
  // k_ca = sum_s W_sc conj(Y_sa) - V_sc conj(Z_sa)
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      cplx<double> acc = {0.0, 0.0};
#pragma unroll
      for (int sp = 0; sp < 4; ++sp) {
        fmac_(acc, yx.v[sp][a], W.v[sp][c]);
        cplx<double> t = {0.0, 0.0};
        fmac_(t, Z.v[sp][a], V.v[sp][c]);
        acc = acc - t;
      }
      k.m[c][a] = acc;
    }
}

struct ForceArgs {
  Geom g;
  LinkField<L_REF> U;
  SpinorRef X, Y;
  double2* F;  // [mu][V][3][3]
  double coef;
  int accumulate;
};

template <int MU>
WL_D void force_store(const ForceArgs& A, const Site& s, long long f) {
  Link<double> k;
  force_link<MU>(A.g, A.U, A.X, A.Y, s, f, k);
  // TA projection
  cplx<double> ta[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) ta[i][j] = 0.5 * (k.m[i][j] - conj(k.m[j][i]));
  cplx<double> tr = (1.0 / 3.0) * (ta[0][0] + ta[1][1] + ta[2][2]);
#pragma unroll
  for (int i = 0; i < 3; ++i) ta[i][i] = ta[i][i] - tr;
  double2* o = A.F + ((long long)MU * A.g.V + f) * 9;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double re = A.coef * ta[i][j].re, im = A.coef * ta[i][j].im;
      if (A.accumulate) {
        double2 old = o[i * 3 + j];
        re += old.x;
        im += old.y;
      }
      o[i * 3 + j] = make_double2(re, im);
    }
}

__global__ void __launch_bounds__(128) pf_force_kernel(ForceArgs A) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int parity = blockIdx.y;
  const int mu = blockIdx.z;
  if (c >= A.g.Vh) return;
  const Site s = site_from_compact(A.g, parity, c);
  const long long f = IdxFlat::self(A.g, s);
  switch (mu) {
    case 0: force_store<0>(A, s, f); break;
    case 1: force_store<1>(A, s, f); break;
    case 2: force_store<2>(A, s, f); break;
    default: force_store<3>(A, s, f); break;
  }
}

}  // namespace wl
