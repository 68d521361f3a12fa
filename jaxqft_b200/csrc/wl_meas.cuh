// Measurement kernels on solver output, reference layout.
//
// Pion two-point function from point-source propagator columns
// (jaxqft/core/measurements.py:375-390):
//     C(dt) = sum_{x in timeslice t0+dt} sum_{columns, spin, colour} |S(x)|^2
// The columns are fermion fields [ncol][Lx][Ly][Lz][Lt][4][3] complex128 (the
// 12 solves of one point source); the sum is over every entry of a timeslice,
// so the column order does not matter.  Block (j, t) adds the sites of rows
// j*128 .. j*128+127 at time t; partials[t][j] are finished in a fixed order.
#pragma once
#include "wl_hop.cuh"

namespace wl {

struct PionArgs {
  const double2* prop;  // [ncol][V][12]
  int ncol;
  int V, Lt;
  double* partials;     // [Lt][gridDim.x]
};

__global__ void __launch_bounds__(128) pion_kernel(PionArgs A) {
  __shared__ double sm[32];
  const int t = blockIdx.y;
  const int rows = A.V / A.Lt;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  double v[1] = {0.0};
  if (r < rows) {
    const long long site = (long long)r * A.Lt + t;
    double s = 0.0;
#pragma unroll 1
    for (int k = 0; k < A.ncol; ++k) {
      const double2* p = A.prop + ((long long)k * A.V + site) * 12;
#pragma unroll
      for (int c = 0; c < 12; ++c) {
        const double2 q = ldg(p + c);
        s += q.x * q.x + q.y * q.y;
      }
    }
    v[0] = s;
  }
  block_sum<1>(v, sm);
  if (threadIdx.x == 0) A.partials[(long long)t * gridDim.x + blockIdx.x] = v[0];
}

}  // namespace wl
