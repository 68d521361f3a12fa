// Gaussian random fields on the device from a counter-based generator.
//
// Philox4x32-10 (J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw, "Parallel
// random numbers: as easy as 1, 2, 3", SC 2011): a 128-bit counter is mixed
// with a 64-bit key by ten rounds of two 32x32 -> 64-bit multiplies, with the
// key bumped by two Weyl increments between rounds.  Every output is a pure
// function of (key, counter), so each thread draws its own numbers with no
// state in memory, any launch shape gives the same field, and a stream of
// fields is indexed by a counter word instead of a stored generator state.
//
// Counter words: c0 = element * calls_per_element + call, c1 = field index
// (right-hand side or batch entry), (c2, c3) = the caller's 64-bit stream
// number; key = the caller's 64-bit seed.  Two 32-bit outputs make one uniform
// double in (0, 1) with 53 random bits; two uniforms make two standard normals
// by the Box-Muller transform (G. E. P. Box, M. E. Muller, Ann. Math. Statist.
// 29 (1958) 610), with CUDA's own log, sqrt and sincospi.
#pragma once
#include "wl_common.cuh"

namespace wl {

WL_D void philox4x32_10(uint32_t (&c)[4], uint32_t k0, uint32_t k1) {
  constexpr uint32_t kM0 = 0xD2511F53u, kM1 = 0xCD9E8D57u;  // round multipliers
  constexpr uint32_t kW0 = 0x9E3779B9u, kW1 = 0xBB67AE85u;  // key increments
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(kM0, c[0]), lo0 = kM0 * c[0];
    const uint32_t hi1 = __umulhi(kM1, c[2]), lo1 = kM1 * c[2];
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += kW0;
    k1 += kW1;
  }
}

// uniform in (0, 1): the top 53 bits of (a, b), offset by half a step so 0 never occurs
WL_D double u01(uint32_t a, uint32_t b) {
  const unsigned long long x = (((unsigned long long)a << 32) | b) >> 11;
  return ((double)x + 0.5) * 0x1.0p-53;
}

// two standard normals from one Philox output
WL_D void normal2(uint64_t seed, uint64_t stream, uint32_t ctr, uint32_t field, double& g0, double& g1) {
  uint32_t c[4] = {ctr, field, (uint32_t)stream, (uint32_t)(stream >> 32)};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double u = u01(c[0], c[1]), v = u01(c[2], c[3]);
  const double r = sqrt(-2.0 * log(u));
  double s, co;
  sincospi(2.0 * v, &s, &co);
  g0 = r * co;
  g1 = r * s;
}

struct RngArgs {
  uint64_t seed, stream;
  long long n_elem;  // sites (spinors) or links (algebra) per field
  int nfield;
  double scale;
  double2* out;
};

// Complex Gaussian spinor field, reference layout [field][site][4][3]:
// z = (g0 + i g1) / sqrt(2), E|z|^2 = 1 (random_fermion, su3_wilson_nf2.py:1169-1175).
__global__ void __launch_bounds__(256) rng_spinor_kernel(RngArgs A) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (s >= A.n_elem || f >= A.nfield) return;
  double2* o = A.out + ((long long)f * A.n_elem + s) * 12;
  const double h = 0.70710678118654752440;  // 1/sqrt(2)
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    double g0, g1;
    normal2(A.seed, A.stream, (uint32_t)(s * 12 + k), (uint32_t)f, g0, g1);
    o[k] = make_double2(h * g0, h * g1);
  }
}

// su(3) algebra field, one 3x3 per link, [field][link][3][3]:
// P = TA(scale (G1 + i G2)) with G1, G2 standard normal per entry and
// TA(X) = (X - X^dag)/2 - Tr(X - X^dag)/6 (_sample_algebra / refresh_p,
// jaxqft/models/su3_ym.py:63-67, 238-244, 339-347).
__global__ void __launch_bounds__(256) rng_algebra_kernel(RngArgs A) {
  const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (l >= A.n_elem || f >= A.nfield) return;
  cplx<double> x[3][3];
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    double g0, g1;
    normal2(A.seed, A.stream, (uint32_t)(l * 9 + k), (uint32_t)f, g0, g1);
    x[k / 3][k % 3] = {A.scale * g0, A.scale * g1};
  }
  cplx<double> y[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) y[a][b] = {0.5 * (x[a][b].re - x[b][a].re), 0.5 * (x[a][b].im + x[b][a].im)};
  const double tr = (y[0][0].im + y[1][1].im + y[2][2].im) / 3.0;  // y is anti-Hermitian: its trace is imaginary
  double2* o = A.out + ((long long)f * A.n_elem + l) * 9;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const int a = k / 3, b = k % 3;
    o[k] = make_double2(y[a][b].re, a == b ? y[a][b].im - tr : y[a][b].im);
  }
}

}  // namespace wl
