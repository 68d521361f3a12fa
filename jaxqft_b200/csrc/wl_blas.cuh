// Level-1 kernels on complex128 fields for the chronological initial-guess
// predictors (jaxqft/models/su3_wilson_nf2.py:85-194): batched inner products
// <a_k, b_k> = sum conj(a_k) b_k, and linear combinations sum_k c_k x_k.
// Inner products are deterministic: each block writes one partial per pair, a
// second kernel adds them in a fixed order (no floating-point atomics).
#pragma once
#include "wl_common.cuh"

namespace wl {

constexpr int kMaxFieldPairs = 64;   // inner products per launch
constexpr int kMaxCombine = 32;      // fields per linear combination
constexpr int kBlasThreads = 256;

struct DotsArgs {
  const double2* a[kMaxFieldPairs];
  const double2* b[kMaxFieldPairs];
  long long len;        // complex elements per field
  double2* partials;    // [pair][block]
  double2* result;      // [pair]
};

__global__ void __launch_bounds__(kBlasThreads) field_dots_kernel(DotsArgs A) {
  __shared__ double sm[2 * 32];
  const int k = blockIdx.y;
  const double2* a = A.a[k];
  const double2* b = A.b[k];
  double v[2] = {0.0, 0.0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < A.len;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 x = __ldg(a + i), y = __ldg(b + i);
    v[0] = fma(x.x, y.x, fma(x.y, y.y, v[0]));   // Re conj(x) y
    v[1] = fma(x.x, y.y, fma(-x.y, y.x, v[1]));  // Im conj(x) y
  }
  block_sum<2>(v, sm);
  if (threadIdx.x == 0) A.partials[(long long)k * gridDim.x + blockIdx.x] = make_double2(v[0], v[1]);
}

__global__ void __launch_bounds__(kBlasThreads) field_dots_finalize_kernel(DotsArgs A, int nblk) {
  __shared__ double sm[2 * 32];
  const int k = blockIdx.x;
  double v[2] = {0.0, 0.0};
  for (int j = threadIdx.x; j < nblk; j += blockDim.x) {
    const double2 p = A.partials[(long long)k * nblk + j];
    v[0] += p.x;
    v[1] += p.y;
  }
  block_sum<2>(v, sm);
  if (threadIdx.x == 0) A.result[k] = make_double2(v[0], v[1]);
}

struct CombineArgs {
  const double2* x[kMaxCombine];
  double2 c[kMaxCombine];
  int n;
  long long len;
  double2* out;
};

__global__ void __launch_bounds__(kBlasThreads) field_combine_kernel(CombineArgs A) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < A.len;
       i += (long long)gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int k = 0; k < A.n; ++k) {
      const double2 x = A.x[k][i], c = A.c[k];  // plain load: out may be one of the x
      re = fma(c.x, x.x, fma(-c.y, x.y, re));
      im = fma(c.x, x.y, fma(c.y, x.x, im));
    }
    A.out[i] = make_double2(re, im);
  }
}

}  // namespace wl
