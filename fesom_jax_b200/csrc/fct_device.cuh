// Device-side helpers shared by the forward kernels of libfesom_fct: tracer addressing
// in the tracer-major and interleaved layouts, the AB2 extrapolation, the upwind vertical
// flux, element gradients and the health counter.
#pragma once

#include "fct_div.cuh"
#include "fct_host.h"

namespace fct {
namespace {

__device__ __forceinline__ double ab2(double T, double To) { return kAbOld * To + kAbNew * T; }
__device__ __forceinline__ double safe_nz(double x) { return x == 0.0 ? 1.0 : x; }

__device__ __forceinline__ int64_t lane_index() {
  return int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
}

template <class T>
__device__ __forceinline__ T ld(const T* p) { return __ldg(p); }

// Address of tracer t at entity-level q: interleaved q*tg + t (below 2^32: the batch
// engine checks every interleaved array against it), else t*stride + q.
template <bool IL>
__device__ __forceinline__ int64_t tix(uint32_t q, int t, int64_t stride, int tg) {
  return IL ? int64_t(q * uint32_t(tg) + uint32_t(t)) : int64_t(t) * stride + q;
}

// Tracers [t0, t0+NTR) of entity-level q.
template <int NTR, bool IL>
__device__ __forceinline__ void ldn(const double* __restrict__ p, uint32_t q, int t0,
                                    int64_t stride, int tg, double (&v)[NTR]) {
  if constexpr (IL && (NTR % 2 == 0)) {
    const double* b = p + (q * uint32_t(tg) + uint32_t(t0));
    if ((reinterpret_cast<uintptr_t>(b) & 15) == 0) {
#pragma unroll
      for (int i = 0; i < NTR; i += 2) {
        const double2 x = __ldg(reinterpret_cast<const double2*>(b + i));
        v[i] = x.x;
        v[i + 1] = x.y;
      }
      return;
    }
  }
#pragma unroll
  for (int i = 0; i < NTR; ++i) v[i] = __ldg(p + tix<IL>(q, t0 + i, stride, tg));
}

// ldn/stn for the segment kernels: in the interleaved layout with an even NTR the host
// guarantees 16-byte alignment (even tracer strides and offsets, workspace fields on
// 256-byte boundaries), so the tracer pairs load and store as double2 without a test.
template <int NTR, bool IL>
__device__ __forceinline__ void ldv(const double* __restrict__ p, uint32_t q, int t0,
                                    int64_t stride, int tg, double (&v)[NTR]) {
  if constexpr (IL && (NTR % 2 == 0)) {
    const double2* b = reinterpret_cast<const double2*>(p + (q * uint32_t(tg) + uint32_t(t0)));
#pragma unroll
    for (int i = 0; i < NTR; i += 2) {
      const double2 x = __ldg(b + i / 2);
      v[i] = x.x;
      v[i + 1] = x.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < NTR; ++i) v[i] = __ldg(p + tix<IL>(q, t0 + i, stride, tg));
  }
}

template <int NTR, bool IL>
__device__ __forceinline__ void stv(double* __restrict__ p, uint32_t q, int t0, int64_t stride,
                                    int tg, const double (&v)[NTR]) {
  if constexpr (IL && (NTR % 2 == 0)) {
    double2* b = reinterpret_cast<double2*>(p + (q * uint32_t(tg) + uint32_t(t0)));
#pragma unroll
    for (int i = 0; i < NTR; i += 2) b[i / 2] = make_double2(v[i], v[i + 1]);
  } else {
#pragma unroll
    for (int i = 0; i < NTR; ++i) p[tix<IL>(q, t0 + i, stride, tg)] = v[i];
  }
}

template <int NTR, bool IL>
__device__ __forceinline__ void stn(double* __restrict__ p, uint32_t q, int t0, int64_t stride,
                                    int tg, const double (&v)[NTR]) {
  if constexpr (IL && (NTR % 2 == 0)) {
    double* b = p + (q * uint32_t(tg) + uint32_t(t0));
    if ((reinterpret_cast<uintptr_t>(b) & 15) == 0) {
#pragma unroll
      for (int i = 0; i < NTR; i += 2)
        *reinterpret_cast<double2*>(b + i) = make_double2(v[i], v[i + 1]);
      return;
    }
  }
#pragma unroll
  for (int i = 0; i < NTR; ++i) p[tix<IL>(q, t0 + i, stride, tg)] = v[i];
}

// tie counts (bytes) of tracers [t0, t0+NTR) at entity-level q
template <int NTR, bool IL>
__device__ __forceinline__ void stc(uint8_t* __restrict__ p, uint32_t q, int t0, int64_t stride,
                                    int tg, const int (&v)[NTR]) {
#pragma unroll
  for (int i = 0; i < NTR; ++i) p[tix<IL>(q, t0 + i, stride, tg)] = uint8_t(v[i]);
}

// Health counter (the reference's finiteness gate, fesom_jax/diagnostics.py:31-101): add
// the number of non-finite values among ``v`` to ``*counter``. Finite results cost a test
// per value and no atomic.
template <int NTR>
__device__ __forceinline__ void count_nonfinite(unsigned long long* counter,
                                                const double (&v)[NTR]) {
  if (!counter) return;
  unsigned bad = 0;
#pragma unroll
  for (int t = 0; t < NTR; ++t) bad += isfinite(v[t]) ? 0u : 1u;
  if (bad) atomicAdd(counter, static_cast<unsigned long long>(bad));
}

// k in [r & 255, (r >> 8) & 255): the packed level ranges of the fused stages' slots
__device__ __forceinline__ bool in_range(int k, unsigned r) {
  return k >= int(r & 255u) && k < int((r >> 8) & 255u);
}

// ---------------------------------------------------- tracer_gradient_elements
// Gradient of T on cell `el` (nodes v0, v1, v2) at level k; the stored (elem_grad) and the
// recomputed (fused stages) gradients both come from here, so they are the same bits.
template <int NTR>
__device__ __forceinline__ void cell_grad_vals(const Inst& in, int el, const double (&a0)[NTR],
                                               const double (&a1)[NTR], const double (&a2)[NTR],
                                               double (&gx)[NTR], double (&gy)[NTR]) {
  // gradient_sca row of the cell: 48 bytes, 16-byte aligned (3 double2 loads)
  const double2* g = reinterpret_cast<const double2*>(in.m->gsca + 6 * int64_t(el));
  const double2 p = __ldg(g), q = __ldg(g + 1), r = __ldg(g + 2);
  const double g0 = p.x, g1 = p.y, g2 = q.x, g3 = q.y, g4 = r.x, g5 = r.y;
#pragma unroll
  for (int t = 0; t < NTR; ++t) {
    gx[t] = g0 * a0[t] + g1 * a1[t] + g2 * a2[t];
    gy[t] = g3 * a0[t] + g4 * a1[t] + g5 * a2[t];
  }
}

template <int NTR, bool IL>
__device__ __forceinline__ void cell_grad(const Inst& in, int el, int v0, int v1, int v2, int k,
                                          int t0, double (&gx)[NTR], double (&gy)[NTR]) {
  const int L = in.m->L;
  double a0[NTR], a1[NTR], a2[NTR];
  ldn<NTR, IL>(in.T, lq(v0, L, k), t0, in.tstride, in.tg, a0);
  ldn<NTR, IL>(in.T, lq(v1, L, k), t0, in.tstride, in.tg, a1);
  ldn<NTR, IL>(in.T, lq(v2, L, k), t0, in.tstride, in.tg, a2);
  cell_grad_vals<NTR>(in, el, a0, a1, a2, gx, gy);
}

// The same gradient when the tracer values at the lane's own node (vertex `pos` of the
// cell) are already in registers: only the other two vertices are gathered.
template <int NTR, bool IL>
__device__ __forceinline__ void cell_grad_own(const Inst& in, int el, int v0, int v1, int v2,
                                              int pos, const double (&own)[NTR], int k, int t0,
                                              double (&gx)[NTR], double (&gy)[NTR]) {
  const int L = in.m->L;
  double a0[NTR], a1[NTR], a2[NTR];
  if (pos == 0) {
    ldn<NTR, IL>(in.T, lq(v1, L, k), t0, in.tstride, in.tg, a1);
    ldn<NTR, IL>(in.T, lq(v2, L, k), t0, in.tstride, in.tg, a2);
#pragma unroll
    for (int t = 0; t < NTR; ++t) a0[t] = own[t];
  } else if (pos == 1) {
    ldn<NTR, IL>(in.T, lq(v0, L, k), t0, in.tstride, in.tg, a0);
    ldn<NTR, IL>(in.T, lq(v2, L, k), t0, in.tstride, in.tg, a2);
#pragma unroll
    for (int t = 0; t < NTR; ++t) a1[t] = own[t];
  } else {
    ldn<NTR, IL>(in.T, lq(v0, L, k), t0, in.tstride, in.tg, a0);
    ldn<NTR, IL>(in.T, lq(v1, L, k), t0, in.tstride, in.tg, a1);
#pragma unroll
    for (int t = 0; t < NTR; ++t) a2[t] = own[t];
  }
  cell_grad_vals<NTR>(in, el, a0, a1, a2, gx, gy);
}

template <int NTR, bool IL>
__device__ __forceinline__ void cell_grad(const Inst& in, int el, int k, int t0,
                                          double (&gx)[NTR], double (&gy)[NTR]) {
  const int* en = in.m->enodes + 3 * int64_t(el);
  cell_grad<NTR, IL>(in, el, ld(en), ld(en + 1), ld(en + 2), k, t0, gx, gy);
}


// Upwind vertical flux at interface j (layer-masked), tracer_adv.py:108-120, given the
// tracer below (Tb = T[j]) and above (Ta = T[j-1], edge-replicated at j = 0).
__device__ __forceinline__ double vflux_up(double Tb, double Ta, double w, double area) {
  const double aw = fabs(w);
  return -0.5 * (Tb * (w + aw) + Ta * (w - aw)) * area;
}

}  // namespace
}  // namespace fct
