// Input producer on the GPU: vertical velocity from continuity, fesom_jax/ale.py:309-365
// (``compute_w(mesh, uv, helem)``), the function the reference's step calls right before
// the FCT (fesom_jax/step.py:367) to produce ``w_e``.
//
// For each node level, the edge->node antisymmetric divergence is gathered over the
// node's incident edges in ascending edge id (the order in which the reference's
// segment_sum over the flattened [edge, 2] contributions adds them), then a bottom-to-top
// running sum gives w, divided by ``area`` (safe where 0) and masked to the node's
// interfaces.
#include <algorithm>

#include "fct_div.cuh"
#include "fct_host.h"

using namespace fct;

namespace {

// One warp per node column, the levels in its lanes (32 at a time, bottom block first):
// every lane gathers its level's divergence, then the bottom-up running sum is added in
// the sequential order (level L-1 first) through shuffles, so the result is the same as a
// per-column loop's.
__device__ __forceinline__ void compute_w_column(const DevMesh& m, const double* __restrict__ uv,
                                                 const double* __restrict__ helem,
                                                 double* __restrict__ w, int n, int lane) {
  if (n >= m.N) return;   // warp-uniform
  const int L = m.L;
  const int64_t base = int64_t(n) * L;
  const int nzmin = __ldg(m.nzmin + n), nzmax = __ldg(m.nzmax + n);
  const int e0 = __ldg(m.ne_off + n), e1 = __ldg(m.ne_off + n + 1);
  double carry = 0.0;
  for (int kb = ((L - 1) / 32) * 32; kb >= 0; kb -= 32) {
    const int k = kb + lane;
    double div = 0.0;
    if (k < L) {
      for (int j = e0; j < e1; ++j) {
        const int idx = __ldg(m.ne_idx + j), e = idx >> 1;
        if (k < __ldg(m.ekmin + e) || k >= __ldg(m.ekmax + e)) continue;
        const int el1 = __ldg(m.etri + 2 * e), el2 = __ldg(m.etri + 2 * e + 1);
        const double* cr = m.cross + 4 * int64_t(e);
        double t1 = 0.0, t2 = 0.0;
        if (k >= __ldg(m.eul + el1) && k < __ldg(m.enl + el1)) {
          const int64_t q = int64_t(el1) * L + k;
          t1 = (__ldg(uv + 2 * q + 1) * __ldg(cr) - __ldg(uv + 2 * q) * __ldg(cr + 1)) *
               __ldg(helem + q);
        }
        if (el2 >= 0 && k >= __ldg(m.eul + el2) && k < __ldg(m.enl + el2)) {
          const int64_t q = int64_t(el2) * L + k;
          t2 = (__ldg(uv + 2 * q + 1) * __ldg(cr + 2) - __ldg(uv + 2 * q) * __ldg(cr + 3)) *
               __ldg(helem + q);
        }
        const double c = t1 - t2;
        div += (idx & 1) ? -c : c;
      }
    }
    double acc = carry, mine = 0.0;
    for (int s = 31; s >= 0; --s) {   // acc += div[kb + s], top of the block last
      const double ds = __shfl_sync(0xffffffffu, div, s);
      if (kb + s < L) acc += ds;
      if (lane == s) mine = acc;
    }
    carry = acc;
    if (k < L) {
      const double a = __ldg(m.area + base + k);
      w[base + k] = (k >= nzmin && k <= nzmax) ? mine / (a > 0.0 ? a : 1.0) : 0.0;
    }
  }
}

__global__ void __launch_bounds__(128) k_compute_w(const DevMesh* __restrict__ mp,
                                                   const double* __restrict__ uv,
                                                   const double* __restrict__ helem,
                                                   double* __restrict__ w) {
  compute_w_column(*mp, uv, helem, w, blockIdx.x * 4 + (threadIdx.x >> 5), threadIdx.x & 31);
}

// batched: instance blockIdx.y of a device table derives its w into w_derived
__global__ void __launch_bounds__(128) k_compute_w_n(const Inst* __restrict__ tab) {
  const Inst& in = tab[blockIdx.y];
  if (!in.w_derived) return;
  compute_w_column(*in.m, in.uv, in.helem, in.w_derived, blockIdx.x * 4 + (threadIdx.x >> 5),
                   threadIdx.x & 31);
}

}  // namespace

namespace fct {

int launch_compute_w_tab(const Inst* tab, int n, int64_t max_nodes, cudaStream_t s) {
  const dim3 g(unsigned(std::max<int64_t>(1, (max_nodes + 3) / 4)), unsigned(n), 1);
  k_compute_w_n<<<g, 128, 0, s>>>(tab);   // 4 warps = 4 node columns per block
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FCT_OK : cuda_error(e, "compute_w (batched) launch");
}

}  // namespace fct

extern "C" int fct_compute_w(FctPlan* P, const double* uv, const double* helem, double* w,
                             fct_stream_t stream) {
  if (!P || !uv || !helem || !w) return set_error(FCT_ERR_INVALID, "NULL argument");
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != P->device) cudaSetDevice(P->device);
  k_compute_w<<<(P->N + 3) / 4, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      P->d_mesh, uv, helem, w);   // 4 warps = 4 node columns per block
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
