// Input producer on the GPU: vertical velocity from continuity, fesom_jax/ale.py:309-365
// (``compute_w(mesh, uv, helem)``), the function the reference's step calls right before
// the FCT (fesom_jax/step.py:367) to produce ``w_e``.
//
// One thread per node column: for each level, the edge->node antisymmetric divergence is
// gathered over the node's incident edges in ascending edge id (the order in which the
// reference's segment_sum over the flattened [edge, 2] contributions adds them), then a
// bottom-to-top running sum gives w, divided by ``area`` (safe where 0) and masked to the
// node's interfaces.
#include <algorithm>

#include "fct_div.cuh"
#include "fct_host.h"

using namespace fct;

namespace {

__global__ void __launch_bounds__(128) k_compute_w(const DevMesh* __restrict__ mp,
                                                   const double* __restrict__ uv,
                                                   const double* __restrict__ helem,
                                                   double* __restrict__ w) {
  const DevMesh& m = *mp;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= m.N) return;
  const int L = m.L;
  const int64_t base = int64_t(n) * L;
  const int nzmin = m.nzmin[n], nzmax = m.nzmax[n];
  const int e0 = m.ne_off[n], e1 = m.ne_off[n + 1];
  double acc = 0.0;
  for (int k = L - 1; k >= 0; --k) {
    double div = 0.0;
    for (int j = e0; j < e1; ++j) {
      const int idx = m.ne_idx[j], e = idx >> 1;
      if (k < m.ekmin[e] || k >= m.ekmax[e]) continue;
      const int el1 = m.etri[2 * e], el2 = m.etri[2 * e + 1];
      const double* cr = m.cross + 4 * int64_t(e);
      double t1 = 0.0, t2 = 0.0;
      if (k >= m.eul[el1] && k < m.enl[el1]) {
        const int64_t q = int64_t(el1) * L + k;
        t1 = (uv[2 * q + 1] * cr[0] - uv[2 * q] * cr[1]) * helem[q];
      }
      if (el2 >= 0 && k >= m.eul[el2] && k < m.enl[el2]) {
        const int64_t q = int64_t(el2) * L + k;
        t2 = (uv[2 * q + 1] * cr[2] - uv[2 * q] * cr[3]) * helem[q];
      }
      const double c = t1 - t2;
      div += (idx & 1) ? -c : c;
    }
    acc += div;
    const double a = m.area[base + k];
    w[base + k] = (k >= nzmin && k <= nzmax) ? acc / (a > 0.0 ? a : 1.0) : 0.0;
  }
}

}  // namespace

extern "C" int fct_compute_w(FctPlan* P, const double* uv, const double* helem, double* w,
                             fct_stream_t stream) {
  if (!P || !uv || !helem || !w) return set_error(FCT_ERR_INVALID, "NULL argument");
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != P->device) cudaSetDevice(P->device);
  k_compute_w<<<(P->N + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      P->d_mesh, uv, helem, w);
  cudaError_t e = cudaGetLastError();
  if (prev >= 0 && prev != P->device) cudaSetDevice(prev);
  return e == cudaSuccess ? FCT_OK : cuda_error(e, "compute_w launch");
}

namespace {

// divr (shared-reciprocal division) against the native IEEE division, bit for bit
__global__ void __launch_bounds__(256) k_div_check(const double* __restrict__ x,
                                                   const double* __restrict__ y, int64_t n,
                                                   unsigned long long* result) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const double a = x[i] / y[i];
    const double b = fct::divr(x[i], fct::rcp(y[i]));
    if (__double_as_longlong(a) != __double_as_longlong(b)) {
      atomicAdd(result, 1ull);
      atomicMin(result + 1, static_cast<unsigned long long>(i));
    }
  }
}

}  // namespace

extern "C" int fct_div_check(const double* x, const double* y, int64_t n,
                             unsigned long long* result, fct_stream_t stream) {
  if (!x || !y || !result || n < 0) return set_error(FCT_ERR_INVALID, "invalid argument");
  if (n == 0) return FCT_OK;
  const int64_t blocks = std::min<int64_t>((n + 255) / 256, 148 * 16);
  k_div_check<<<unsigned(blocks), 256, 0, static_cast<cudaStream_t>(stream)>>>(x, y, n, result);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FCT_OK : cuda_error(e, "div_check launch");
}
