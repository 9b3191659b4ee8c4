// Sea-ice FCT advection (fesom_jax/ice_adv.py:37-194, fesom_ice_fct.c): one step of the
// three ice tracers (a_ice, m_ice, m_snow) on the surface mesh.
//
// The reference scatters element contributions to nodes; here every node gathers over
// its cells (node->element CSR in the reference's nod_in_elem2D order, the node's vertex
// index packed in the slot) so sums are deterministic and no atomics are needed. One
// thread per node carries all three tracers: the tracer-independent cell terms (the
// Taylor-Galerkin matrix row, the mass-matrix weight) are formed once per cell.
//
//   k_ice_rhs    _tg_rhs (:47-75), _mm_times (:37-44), _solve_low_order (:78-89),
//                first high-order approximation (:103)
//   k_ice_hi     one high-order residual correction (:104-107), launched twice
//   k_ice_limit  _fem_fct antidiffusive fluxes, cluster bounds, clipping ratios (:126-160)
//   k_ice_apply  _fem_fct limited flux application (:162-172)
#include <algorithm>

#include "fct_host.h"

using namespace fct;

namespace {

constexpr double kIceScaleArea = 2.0e8;   // ice_adv.py:33
constexpr double kIceFluxEps = 1.0e-12;   // ice_adv.py:34
constexpr int B = 128;

struct IceArgs {
  const DevMesh* m;
  const double* X[3];   // a_ice, m_ice, m_snow
  const double *u, *v;
  double* out[3];
  double *rhs, *xl, *d0, *d1, *pp, *pm;   // workspace, each [3][nod2D]
  double dt, gamma, diff;
};

__device__ __forceinline__ int64_t node_index() {
  return int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
}
__device__ __forceinline__ bool cell_on(const DevMesh& m, int el) { return __ldg(m.eul + el) <= 0; }
__device__ __forceinline__ double inv_area(const DevMesh& m, int n) {
  const double a = __ldg(m.area + int64_t(n) * m.L);   // surface level
  return 1.0 / (a > 0.0 ? a : 1.0);
}

__global__ void __launch_bounds__(B) k_ice_rhs(IceArgs A) {
  const DevMesh& m = *A.m;
  const int64_t n = node_index();
  if (n >= m.N) return;
  const int N = m.N;
  double rhs[3] = {0.0, 0.0, 0.0}, mmx[3] = {0.0, 0.0, 0.0};
  const int c0 = __ldg(m.nel_off + n), c1 = __ldg(m.nel_off + n + 1);
  for (int j = c0; j < c1; ++j) {
    const int4 sl = __ldg(m.nel4 + j);
    if (!cell_on(m, sl.x)) continue;   // cavity cells contribute 0
    const int p = (__ldg(m.nelr + j) >> 16) & 3;
    const int vq[3] = {sl.y, sl.z, sl.w};
    const double* gs = m.gsca + 6 * int64_t(sl.x);
    const double dx[3] = {__ldg(gs), __ldg(gs + 1), __ldg(gs + 2)};
    const double dy[3] = {__ldg(gs + 3), __ldg(gs + 4), __ldg(gs + 5)};
    const double vol = __ldg(m.earea + sl.x);
    double U[3], V[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) { U[q] = __ldg(A.u + vq[q]); V[q] = __ldg(A.v + vq[q]); }
    const double um = U[0] + U[1] + U[2], vm = V[0] + V[1] + V[2];
    const double diff = A.diff * sqrt(vol / kIceScaleArea);
    const double dxp = dx[p], dyp = dy[p];
    const double udnp = um * dxp + vm * dyp;
    double E[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const double a = (dxp * (um + U[q]) + dyp * (vm + V[q])) / 12.0;
      const double b = diff * (dxp * dx[q] + dyp * dy[q]);
      const double udnq = um * dx[q] + vm * dy[q];
      const double c = 0.5 * A.dt * (udnp * udnq) / 9.0;
      E[q] = vol * A.dt * (a - b - c);
    }
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      const double x0 = __ldg(A.X[t] + vq[0]), x1 = __ldg(A.X[t] + vq[1]),
                   x2 = __ldg(A.X[t] + vq[2]);
      rhs[t] += E[0] * x0 + E[1] * x1 + E[2] * x2;
      const double xs[3] = {x0, x1, x2};
      mmx[t] += vol / 12.0 * (xs[p] + (x0 + x1 + x2));
    }
  }
  const bool nc = __ldg(m.nzmin + n) <= 0;   // ulevels_nod2D <= 1
  const double ia = inv_area(m, int(n));
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    const double X = __ldg(A.X[t] + n);
    A.rhs[t * N + n] = rhs[t];
    A.d0[t * N + n] = nc ? rhs[t] * ia : 0.0;
    A.xl[t * N + n] = nc ? (rhs[t] + A.gamma * mmx[t]) * ia + (1.0 - A.gamma) * X : X;
  }
}

// d_out = d_in + (rhs - mm d_in) / area on open-water/ice nodes
__global__ void __launch_bounds__(B) k_ice_hi(IceArgs A, const double* __restrict__ din,
                                              double* __restrict__ dout) {
  const DevMesh& m = *A.m;
  const int64_t n = node_index();
  if (n >= m.N) return;
  const int N = m.N;
  double mmd[3] = {0.0, 0.0, 0.0};
  const int c0 = __ldg(m.nel_off + n), c1 = __ldg(m.nel_off + n + 1);
  for (int j = c0; j < c1; ++j) {
    const int4 sl = __ldg(m.nel4 + j);
    if (!cell_on(m, sl.x)) continue;
    const int p = (__ldg(m.nelr + j) >> 16) & 3;
    const double vol = __ldg(m.earea + sl.x);
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      const double x0 = din[t * N + sl.y], x1 = din[t * N + sl.z], x2 = din[t * N + sl.w];
      const double xs[3] = {x0, x1, x2};
      mmd[t] += vol / 12.0 * (xs[p] + (x0 + x1 + x2));
    }
  }
  const bool nc = __ldg(m.nzmin + n) <= 0;
  const double ia = inv_area(m, int(n));
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    const double d = din[t * N + n];
    dout[t * N + n] = nc ? d + (A.rhs[t * N + n] - mmd[t]) * ia : d;
  }
}

// the cell's antidiffusive flux at vertex q: -s_q (vol / area_q) / 12, s_q = sum w - 3 w_q
__device__ __forceinline__ double ice_flux(double sw, double wq, double vol, double iaq) {
  return -(sw - 3.0 * wq) * (vol * iaq) / 12.0;
}

__global__ void __launch_bounds__(B) k_ice_limit(IceArgs A, const double* __restrict__ dv) {
  const DevMesh& m = *A.m;
  const int64_t n = node_index();
  if (n >= m.N) return;
  const int N = m.N;
  const double ia_n = inv_area(m, int(n));
  double fp[3] = {0.0, 0.0, 0.0}, fm[3] = {0.0, 0.0, 0.0};
  double hi[3] = {-INFINITY, -INFINITY, -INFINITY}, lo[3] = {INFINITY, INFINITY, INFINITY};
  const int c0 = __ldg(m.nel_off + n), c1 = __ldg(m.nel_off + n + 1);
  for (int j = c0; j < c1; ++j) {
    const int4 sl = __ldg(m.nel4 + j);
    const bool on = cell_on(m, sl.x);
    const int p = (__ldg(m.nelr + j) >> 16) & 3;
    const int vq[3] = {sl.y, sl.z, sl.w};
    const double vol = __ldg(m.earea + sl.x);
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      double w[3], xl[3], xv[3];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        xv[q] = __ldg(A.X[t] + vq[q]);
        w[q] = A.gamma * xv[q] + dv[t * N + vq[q]];
        xl[q] = A.xl[t * N + vq[q]];
      }
      const double sw = w[0] + w[1] + w[2];
      const double f = on ? ice_flux(sw, w[p], vol, ia_n) : 0.0;
      fp[t] += fmax(f, 0.0);
      fm[t] += fmin(f, 0.0);
      if (on) {
        const double ehi = fmax(fmax(fmax(xl[0], xl[1]), xl[2]), fmax(fmax(xv[0], xv[1]), xv[2]));
        const double elo = fmin(fmin(fmin(xl[0], xl[1]), xl[2]), fmin(fmin(xv[0], xv[1]), xv[2]));
        hi[t] = fmax(hi[t], ehi);
        lo[t] = fmin(lo[t], elo);
      }
    }
  }
  const bool nc = __ldg(m.nzmin + n) <= 0;
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    const double h = isfinite(hi[t]) ? hi[t] : 0.0, l = isfinite(lo[t]) ? lo[t] : 0.0;
    const double xl = A.xl[t * N + n];
    const double tmax = h - xl, tmin = l - xl;
    double pp = fp[t] > 0.0 ? fmin(tmax / (fp[t] > kIceFluxEps ? fp[t] : kIceFluxEps), 1.0) : 0.0;
    double pm = fm[t] < 0.0 ? fmin(tmin / (fm[t] < -kIceFluxEps ? fm[t] : -kIceFluxEps), 1.0) : 0.0;
    A.pp[t * N + n] = nc ? pp : 0.0;
    A.pm[t * N + n] = nc ? pm : 0.0;
  }
}

__global__ void __launch_bounds__(B) k_ice_apply(IceArgs A, const double* __restrict__ dv) {
  const DevMesh& m = *A.m;
  const int64_t n = node_index();
  if (n >= m.N) return;
  const int N = m.N;
  double acc[3] = {0.0, 0.0, 0.0};
  const int c0 = __ldg(m.nel_off + n), c1 = __ldg(m.nel_off + n + 1);
  for (int j = c0; j < c1; ++j) {
    const int4 sl = __ldg(m.nel4 + j);
    if (!cell_on(m, sl.x)) continue;   // limited fluxes of cavity cells are 0
    const int p = (__ldg(m.nelr + j) >> 16) & 3;
    const int vq[3] = {sl.y, sl.z, sl.w};
    const double vol = __ldg(m.earea + sl.x);
    const double ia[3] = {inv_area(m, vq[0]), inv_area(m, vq[1]), inv_area(m, vq[2])};
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      double w[3];
#pragma unroll
      for (int q = 0; q < 3; ++q) w[q] = A.gamma * __ldg(A.X[t] + vq[q]) + dv[t * N + vq[q]];
      const double sw = w[0] + w[1] + w[2];
      double f[3], cand[3];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        f[q] = ice_flux(sw, w[q], vol, ia[q]);
        cand[q] = f[q] >= 0.0 ? A.pp[t * N + vq[q]] : A.pm[t * N + vq[q]];
      }
      const double ae = fmin(fmin(cand[0], cand[1]), cand[2]);
      acc[t] += f[p] * ae;
    }
  }
#pragma unroll
  for (int t = 0; t < 3; ++t) A.out[t][n] = A.xl[t * N + n] + acc[t];
}

}  // namespace

extern "C" int fct_ice_solve(FctPlan* P, const FctIceFields* f, const FctIceConfig* cfg,
                             fct_stream_t stream) {
  if (!P || !f || !cfg) return set_error(FCT_ERR_INVALID, "NULL argument");
  for (int t = 0; t < 3; ++t)
    if (!f->tracer[t] || !f->tracer_new[t])
      return set_error(FCT_ERR_INVALID, "ice tracer %d pointer is NULL", t);
  if (!f->u_ice || !f->v_ice) return set_error(FCT_ERR_INVALID, "ice velocity is NULL");
  if (!(cfg->dt > 0.0)) return set_error(FCT_ERR_INVALID, "dt must be positive");
  const int64_t N = P->N;
  // scratch: 6 fields of 3 x nod2D doubles, carved from the plan workspace's node fields
  // (LO onwards: at least kFusedNodeFields x nod2D x nl doubles per tracer, contiguous in
  // both workspace layouts)
  if (18 * N > kFusedNodeFields * N * P->L * int64_t(P->max_tracers))
    return set_error(FCT_ERR_CAPACITY, "plan workspace too small for the ice step");
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != P->device) cudaSetDevice(P->device);
  IceArgs A{};
  A.m = P->d_mesh;
  for (int t = 0; t < 3; ++t) { A.X[t] = f->tracer[t]; A.out[t] = f->tracer_new[t]; }
  A.u = f->u_ice;
  A.v = f->v_ice;
  double* w = P->ws.lo;
  A.rhs = w; A.xl = w + 3 * N; A.d0 = w + 6 * N; A.d1 = w + 9 * N;
  A.pp = w + 12 * N; A.pm = w + 15 * N;
  A.dt = cfg->dt; A.gamma = cfg->gamma; A.diff = cfg->diff;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const unsigned g = unsigned((N + B - 1) / B);
  int st;
  {
    PlanUse use(P, s);
    st = use.status();
    if (!st) {
      k_ice_rhs<<<g, B, 0, s>>>(A);
      k_ice_hi<<<g, B, 0, s>>>(A, A.d0, A.d1);   // two residual corrections (ice_adv.py:104)
      k_ice_hi<<<g, B, 0, s>>>(A, A.d1, A.d0);
      k_ice_limit<<<g, B, 0, s>>>(A, A.d0);
      k_ice_apply<<<g, B, 0, s>>>(A, A.d0);
      const cudaError_t e = cudaGetLastError();
      st = e == cudaSuccess ? use.release() : cuda_error(e, "ice FCT launch");
    }
  }
  if (prev >= 0 && prev != P->device) cudaSetDevice(prev);
  return st;
}
