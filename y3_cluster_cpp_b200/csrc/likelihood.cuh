// likelihood.cuh -- the Gaussian likelihood of the counts and tangential
// shear data vector (y3_buzzard/likelihood_cp.py:94-200), evaluated on the
// device by one block per parameter point, in the block that produced the
// point's counts and shear.
#pragma once

#include "common.cuh"

namespace y3b {

// Device copy of a y3b_likelihood, data and inverse covariances already in
// the form likelihood_cp.setup() stores (logged data and the delta-method
// inverse covariance in log space).
struct LikeDev {
  int on, log_space, n_R, nc_dense, sh_dense;
  const double* data_nc;  // [nB]
  const double* ic_nc;    // [nB] or [nB][nB]
  const double* data_sh;  // [nB * n_R]
  const double* ic_sh;    // [nB * n_R] or square
  const double* prj;      // [nB * n_R] projection shear, or null
};

// Residual of one observable: data - theory, or ln data - ln max(theory,
// 1e-300) in log space (likelihood_cp.py:166-177).
__device__ __forceinline__ double
like_resid(const LikeDev& L, double data, double theory)
{
  return L.log_space ? data - log(fmax(theory, 1e-300)) : data - theory;
}

// delta^T C^-1 delta over n entries: diagonal (sum delta^2 ic) or dense
// (likelihood_cp.py:66-72); each thread takes rows t, t + blockDim, ... in
// order and the block sums with a fixed tree, so reruns are bit-identical.
__device__ __forceinline__ double
like_chi2(int n, const double* delta, const double* ic, int dense, double* red)
{
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double row;
    if (dense) {
      row = 0.0;
      const double* r = ic + (size_t)i * n;
      for (int j = 0; j < n; ++j) row += r[j] * delta[j];
    } else {
      row = ic[i] * delta[i];
    }
    acc += delta[i] * row;
  }
  return block_sum<1024>(acc, red);
}

// logL = -0.5 (chi2_NC + chi2_Shear) of one point: nc[nB] are its counts,
// sh[nB * n_R] its N_i-weighted one-halo shear (bin slow, R fast), turned in
// place into the shear residual: theory = (nc_b > 0 ? sh / nc_b : 0) + prj
// (likelihood_cp.py:122-162).  All threads of the block take part; `red`
// holds blockDim.x doubles.  nc is turned into its residual too.
__device__ __forceinline__ double
gaussian_loglike_block(const LikeDev& L, int nB, int n_R, double* nc, double* sh, double* red)
{
  const int nsh = nB * n_R;
  for (int u = threadIdx.x; u < nsh; u += blockDim.x) {
    const double c = nc[u / n_R];
    const double th = (c <= 0.0 ? 0.0 : sh[u] / c) + (L.prj ? L.prj[u] : 0.0);
    sh[u] = like_resid(L, L.data_sh[u], th);
  }
  __syncthreads();  // every shear residual has read its count
  for (int b = threadIdx.x; b < nB; b += blockDim.x) nc[b] = like_resid(L, L.data_nc[b], nc[b]);
  __syncthreads();
  const double chi2_nc = like_chi2(nB, nc, L.ic_nc, L.nc_dense, red);
  const double chi2_sh = nsh ? like_chi2(nsh, sh, L.ic_sh, L.sh_dense, red) : 0.0;
  return -0.5 * (chi2_nc + chi2_sh);
}

}  // namespace y3b
