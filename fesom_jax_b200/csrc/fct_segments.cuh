// Segment kernels of the fused forward step: the product path of fct_forward, the
// batched engine and the serving engine (fesom_jax/tracer_adv.py:532-578).
//
// A thread takes a *segment*: a run of up to LPT consecutive levels of one node (or one
// edge) and NTR tracers. The entity's neighbour slots, level range and static geometry
// are decoded once per segment and every neighbour gather issues LPT x NTR independent
// loads (consecutive levels of one column), instead of one level per thread re-decoding
// the same lists. Every quantity is the reference's expression; the arithmetic (below)
// trades correctly rounded quotients for reciprocal products and fused multiply-adds, so
// the results equal the one-kernel-per-stage path's to rounding (a few ulp per step), and
// every mapping and layout of these kernels gives the same bits.
//
// Stages (kernels over the plan's segment lists, fct_internal.cuh DevMesh):
//   seg_node_lo     node layers: LO (compute_fct_lo with adv_flux_hor/ver, :96-120,
//                   :298-313) and adf_v (adv_flux_ver_ho minus the LO vertical flux,
//                   :241-295, :568) on the tops of the layers; the bottom interface's
//                   adf_v is 0 and not stored (readers take 0 there)
//   seg_edge_adf    edge levels where MFCT takes the up/down cells' gradients
//                   (fill_up_dn_grad :344-368, adv_flux_hor_ho :196-225): adf_h
//   edge_fix        the other edge lanes: the node-average gradients (:329-341) of the
//                   two end nodes computed on the fly; at 1-2 % of the edge lanes of an
//                   open-ocean mesh this is cheaper than storing node gradients everywhere
//   seg_node_limit  zalesak_limit a1-a4, b1, b2 (:371-451): cluster bounds over the edge
//                   neighbours, the k-1/k/k+1 window (across runs through shared memory),
//                   the antidiffusive sums and the limiter factors
//   seg_node_final  b3, flux2dtracer_fct, ale_reconstruct (:453-484, :142-151): T_new
#pragma once

#include <algorithm>

#include "fct_device.cuh"

namespace fct {
namespace {

// Arithmetic of the segment kernels. Quotients multiply by the divisor's correctly rounded
// reciprocal (within 1.5 ulp of the quotient; the one-kernel-per-stage path rounds every
// quotient correctly instead), products that feed a sum fuse into FMAs written out in the
// source (--fmad=false keeps the compiler from contracting anything else, so every
// template instantiation rounds alike), and max/min are plain comparisons (the same values
// as fmax/fmin on the finite numbers the scheme carries).
struct Rcq {
  double r;
};
__device__ __forceinline__ Rcq rcpq(double y) { return Rcq{__drcp_rn(y)}; }
__device__ __forceinline__ double divq(double x, const Rcq& c) { return x * c.r; }
__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }
// AB2 extrapolation ttfAB = -0.6*T_old + 1.6*T (tracer_adv.py:59-66)
__device__ __forceinline__ double ab2f(double T, double To) { return fma(kAbNew, T, kAbOld * To); }

// The node kernels' neighbour loops load each slot record one slot ahead, so the next
// slot's gathers do not wait behind its record (2-4% faster per node kernel on the
// CORE2-size batched step)
#define FCT_SLOT_BEGIN(e0, e1) \
  int4 sl_nx = (e0) < (e1) ? __ldg(m.ne4 + (e0)) : make_int4(0, 0, 0, 0);
#define FCT_SLOT_GET(j, e1) \
  const int4 sl = sl_nx;    \
  if ((j) + 1 < (e1)) sl_nx = __ldg(m.ne4 + (j) + 1);

// a level clamped into [0, L - 1]: loads at clamped levels are in bounds and their values
// are discarded by the predicates that follow
__device__ __forceinline__ int kclamp(int k, int L) { return k < 0 ? 0 : (k >= L ? L - 1 : k); }

// ----------------------------------------------------------- LO and adf_v, node runs
template <int NTR, int LPT, bool IL>
__device__ __forceinline__ void seg_node_lo(const Inst& in, int64_t si, int t0, int w0) {
  const DevMesh& m = *in.m;
  constexpr int V = seg_variant(LPT);
  if (si >= m.n_nseg[V]) return;
  const uint32_t sg = __ldg(m.nseg[V] + si);
  const int n = lane_ent(sg), k0 = lane_lev(sg), L = m.L;
  const int4 rec = __ldg(m.nrec + n);
  const unsigned pk = unsigned(rec.z);
  const int nzmin = int(pk & 255u), nzmax = int((pk >> 8) & 255u);
  const int nk = min(LPT, nzmax - k0);   // layers of this run
  const uint32_t base = lq(n, L, 0);
  const int64_t ts = in.tstride;
  const int tg = in.tg;
  const double dt = in.dt;
  // T of the column at levels k0-2 .. k0+LPT (Tw[i] <-> level k0-2+i; the level above
  // the surface reads T[0], the reference's edge-replicated top)
  double Tw[LPT + 3][NTR];
#pragma unroll
  for (int i = 0; i < LPT + 3; ++i)
    ldv<NTR, IL>(in.T, base + uint32_t(kclamp(k0 - 2 + i, L)), t0, ts, tg, Tw[i]);

  // compute_fct_lo: edge->node upwind divergence in ascending edge id
  double div[LPT][NTR];
#pragma unroll
  for (int l = 0; l < LPT; ++l)
#pragma unroll
    for (int t = 0; t < NTR; ++t) div[l][t] = 0.0;
  unsigned long long fl_[LPT];   // the run's node-layer flags (0 beyond the run)
#pragma unroll
  for (int l = 0; l < LPT; ++l) fl_[l] = l < nk ? __ldg(m.nflags + rec.w + (k0 + l - nzmin)) : 0ull;
  const int e0 = rec.x, e1 = rec.x + int((pk >> 16) & 255u);
  FCT_SLOT_BEGIN(e0, e1)
  for (int j = e0; j < e1; ++j) {
    FCT_SLOT_GET(j, e1)
    const int jj = j - e0;
    const bool second = sl.x & 1;
    const double sg1 = second ? -1.0 : 1.0;   // the flux leaves the edge's first node
    const uint32_t qe = lq(sl.x >> 1, L, 0), qo = lq(sl.y, L, 0);
#pragma unroll
    for (int l = 0; l < LPT; ++l) {
      const int kc = kclamp(k0 + l, L);
      const bool on = ((fl_[l] >> jj) & 1ull);
      const double vf = __ldg(in.ws.vflux + qe + kc);
      const double avf = fabs(vf);
      // the reference's face flux -0.5*(T1*(vf+|vf|) + T2*(vf-|vf|)) with the node's own
      // value first (a + b == b + a exactly): the same bits for either end of the edge
      const double cown = second ? vf - avf : vf + avf, coth = second ? vf + avf : vf - avf;
      double To[NTR];
      ldv<NTR, IL>(in.T, qo + uint32_t(kc), t0, ts, tg, To);
#pragma unroll
      for (int t = 0; t < NTR; ++t) {
        const double f = -0.5 * fma(Tw[l + 2][t], cown, To[t] * coth);
        div[l][t] = on ? div[l][t] + sg1 * f : div[l][t];
      }
    }
  }

  // upwind vertical flux at the interfaces k0 .. k0+LPT (layer-masked, tracer_adv.py:108-120)
  double fv[LPT + 1][NTR];
#pragma unroll
  for (int i = 0; i <= LPT; ++i) {
    const int k = k0 + i, kc = kclamp(k, L);
    const bool layer = i <= nk && k < nzmax;
    const double w = __ldg(in.w_e + base + kc), ar = __ldg(m.area + base + kc);
#pragma unroll
    for (int t = 0; t < NTR; ++t)
      fv[i][t] = layer ? vflux_up(Tw[i + 2][t], Tw[i + 1][t], w, ar) : 0.0;
  }
  // LO on the run's layers
#pragma unroll
  for (int l = 0; l < LPT; ++l) {
    if (l >= nk) break;
    const uint32_t qn = base + uint32_t(k0 + l);
    const double hn = __ldg(in.hnode + qn), hnn = __ldg(in.hnode_new + qn);
    const double av = __ldg(m.areasvol + qn);
    const double fdt = dt * __drcp_rn(av);   // dt / areasvol
    const Rcq rhn = rcpq(hnn);
    const bool valid = (hnn > 0.0) && (av > 0.0);
    double lo[NTR];
#pragma unroll
    for (int t = 0; t < NTR; ++t)
      lo[t] = valid ? divq(fma(Tw[l + 2][t], hn, (div[l][t] + (fv[l][t] - fv[l + 1][t])) * fdt),
                           rhn)
                    : 0.0;
    stv<NTR, IL>(in.ws.lo, qn, w0, in.ws.sN, in.wtg, lo);
  }

  // adv_flux_ver_ho (QR4C on ttfAB) minus the LO vertical flux at the layer tops
  double To[LPT + 3][NTR];   // T_old at levels k0-2 .. k0+LPT
#pragma unroll
  for (int i = 0; i < LPT + 3; ++i)
    ldv<NTR, IL>(in.T_old, base + uint32_t(kclamp(k0 - 2 + i, L)), t0, ts, tg, To[i]);
#pragma unroll
  for (int l = 0; l < LPT; ++l) {
    if (l >= nk) break;
    const int k = k0 + l;
    const uint32_t qn = base + uint32_t(k);
    const double w = __ldg(in.w_e + qn);
    const double Wf = in.w_i ? w + __ldg(in.w_i + qn) : w;
    const double area_k = __ldg(m.area + qn);
    double hi[NTR];
    if (k == nzmin) {
#pragma unroll
      for (int t = 0; t < NTR; ++t) hi[t] = -ab2f(Tw[l + 2][t], To[l + 2][t]) * Wf * area_k;
    } else if (k == nzmin + 1 || k == nzmax - 1) {
#pragma unroll
      for (int t = 0; t < NTR; ++t)
        hi[t] = -0.5 * (ab2f(Tw[l + 1][t], To[l + 1][t]) + ab2f(Tw[l + 2][t], To[l + 2][t])) *
                Wf * area_k;
    } else {   // nzmin + 2 <= k <= nzmax - 2
      double Znz, Zm1, Zm2, Zp1, zb;   // QR4C stencil depths (tracer_adv.py:228-238, 265-273)
      if (in.Z3d) {
        const double* Zc = in.Z3d + base;
        Znz = __ldg(Zc + k); Zm1 = __ldg(Zc + k - 1); Zm2 = __ldg(Zc + k - 2);
        Zp1 = __ldg(Zc + (k + 1 < L ? k + 1 : L - 1)); zb = __ldg(in.zbar3 + qn);
      } else {
        Znz = __ldg(m.Zp + k); Zm1 = __ldg(m.Zp + k - 1); Zm2 = __ldg(m.Zp + k - 2);
        Zp1 = __ldg(m.Zp + (k + 1 < L ? k + 1 : L - 1)); zb = __ldg(m.zbar + k);
      }
      const Rcq rdc = rcpq(safe_nz(Zm1 - Znz)), rdu = rcpq(safe_nz(Znz - Zp1)),
                rdd = rcpq(safe_nz(Zm2 - Zm1));
      const double d1 = (zb - Znz) * (1.0 / 3.0), d2 = (zb - Zm1) * (1.0 / 3.0);
      const double wa = -0.5 * Wf * area_k;
#pragma unroll
      for (int t = 0; t < NTR; ++t) {
        const double A0 = ab2f(Tw[l + 2][t], To[l + 2][t]);
        const double Am1 = ab2f(Tw[l + 1][t], To[l + 1][t]);
        const double Am2 = ab2f(Tw[l][t], To[l][t]);
        const double Ap1 = ab2f(Tw[l + 3][t], To[l + 3][t]);
        const double qc = divq(Am1 - A0, rdc);
        const double qu = divq(A0 - Ap1, rdu);
        const double qd = divq(Am2 - Am1, rdd);
        const double Tmean1 = fma(fma(2.0, qc, qu), d1, A0);
        const double Tmean2 = fma(fma(2.0, qc, qd), d2, Am1);
        hi[t] = (Tmean1 + Tmean2) * wa;
      }
    }
    double adf[NTR];
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      const double lo_v = in.w_i ? vflux_up(Tw[l + 2][t], Tw[l + 1][t], Wf, area_k) : fv[l][t];
      adf[t] = hi[t] - lo_v;
    }
    stv<NTR, IL>(in.ws.adfv, qn, w0, in.ws.sN, in.wtg, adf);
  }
}

// ---------------------------------------------- adf_h on a run of up/down-cell levels
template <int NTR, int LPT, bool IL>
__device__ __forceinline__ void seg_edge_adf(const Inst& in, int64_t si, int t0, int w0) {
  const DevMesh& m = *in.m;
  constexpr int V = seg_variant(LPT);
  if (si >= m.n_eseg[V]) return;
  const uint32_t sg = __ldg(m.eseg[V] + si);
  const int e = lane_ent(sg), k0 = lane_lev(sg), L = m.L;
  const int4 er = __ldg(m.erec + e);
  const int nk = min(LPT, int((unsigned(er.z) >> 8) & 255u) - k0);
  const int4 ov = __ldg(m.emf4 + e);
  const double2* wp = reinterpret_cast<const double2*>(m.emfw + 8 * int64_t(e));
  const double2 w01 = __ldg(wp), w23 = __ldg(wp + 1), w45 = __ldg(wp + 2);
  const uint32_t q1 = lq(er.x, L, 0), q2 = lq(er.y, L, 0), qe = lq(e, L, 0);
  const uint32_t qua = lq(ov.x, L, 0), qub = lq(ov.y, L, 0);
  const uint32_t qda = lq(ov.z, L, 0), qdb = lq(ov.w, L, 0);
  const int64_t ts = in.tstride;
  const int tg = in.tg;
#pragma unroll
  for (int l = 0; l < LPT; ++l) {
    const int kc = kclamp(k0 + l, L);
    const double vf = __ldg(in.ws.vflux + qe + kc);
    const double avf = fabs(vf);
    double T1[NTR], T2[NTR], O1[NTR], O2[NTR], ua[NTR], ub[NTR], da[NTR], db[NTR];
    ldv<NTR, IL>(in.T, q1 + kc, t0, ts, tg, T1);
    ldv<NTR, IL>(in.T, q2 + kc, t0, ts, tg, T2);
    ldv<NTR, IL>(in.T_old, q1 + kc, t0, ts, tg, O1);
    ldv<NTR, IL>(in.T_old, q2 + kc, t0, ts, tg, O2);
    ldv<NTR, IL>(in.T, qua + kc, t0, ts, tg, ua);
    ldv<NTR, IL>(in.T, qub + kc, t0, ts, tg, ub);
    ldv<NTR, IL>(in.T, qda + kc, t0, ts, tg, da);
    ldv<NTR, IL>(in.T, qdb + kc, t0, ts, tg, db);
    double adf[NTR];
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      // Tm1 = A1 + (2*(A2 - A1) + edx*a*g_up_x + edy*R*g_up_y)/6 with the up cell's
      // gradient as one weighted vertex sum; Tm2 likewise with the down cell's, minus
      const double A1 = ab2f(T1[t], O1[t]), A2 = ab2f(T2[t], O2[t]);
      const double dA = A2 - A1;
      const double su = fma(w01.y, ua[t], fma(w23.x, ub[t], w01.x * T1[t]));
      const double sd = fma(w23.y, T2[t], fma(w45.x, da[t], w45.y * db[t]));
      const double Tm1 = fma(dA, 1.0 / 3.0, A1) + su;
      const double Tm2 = fma(dA, -1.0 / 3.0, A2) - sd;
      // HO - LO = -0.5*((vf+|vf|)*(Tm1 - T1) + (vf-|vf|)*(Tm2 - T2))
      adf[t] = -0.5 * fma(vf + avf, Tm1 - T1[t], (vf - avf) * (Tm2 - T2[t]));
    }
    if (l < nk) stv<NTR, IL>(in.ws.adfh, qe + uint32_t(kc), w0, in.ws.sEd, in.wtg, adf);
  }
}

// node-average gradient of T at node n, level k (_node_avg_grad, tracer_adv.py:329-341):
// the area-weighted mean over n's cells wet at k, in the node's cell order
template <int NTR, bool IL>
__device__ __forceinline__ void node_avg_grad(const Inst& in, int n, int k, int t0,
                                              double (&nx)[NTR], double (&ny)[NTR]) {
  const DevMesh& m = *in.m;
  const int4 rec = __ldg(m.nrec + n);
  double den = 0.0;
#pragma unroll
  for (int t = 0; t < NTR; ++t) nx[t] = ny[t] = 0.0;
  const int c0 = rec.y, c1 = rec.y + int(unsigned(rec.z) >> 24);
  for (int j = c0; j < c1; ++j) {
    const unsigned r = unsigned(__ldg(m.nelr + j));
    const int4 sl = __ldg(m.nel4 + j);
    if (!in_range(k, r)) continue;
    const double a = __ldg(m.earea + sl.x);
    double gx[NTR], gy[NTR];
    cell_grad<NTR, IL>(in, sl.x, sl.y, sl.z, sl.w, k, t0, gx, gy);
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      nx[t] += gx[t] * a;
      ny[t] += gy[t] * a;
    }
    den += a;
  }
  const Rcp rdd = rcp(den > 0.0 ? den : 1.0);
#pragma unroll
  for (int t = 0; t < NTR; ++t) {
    nx[t] = divr(nx[t], rdd);
    ny[t] = divr(ny[t], rdd);
  }
}

// ----------------------------------------------- adf_h on the remaining edge lanes
template <int NTR, bool IL>
__device__ __forceinline__ void body_edge_fix(const Inst& in, int64_t i, int t0, int w0) {
  const DevMesh& m = *in.m;
  if (i >= m.n_efix) return;
  const uint32_t lane = __ldg(m.efix + i);
  const int e = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int4 er = __ldg(m.erec + e);
  const int n1 = er.x, n2 = er.y;
  const bool use_tri = in_range(k, unsigned(__ldg(m.etr + e)));
  const double vf = __ldg(in.ws.vflux + lq(e, L, k));
  const double avf = fabs(vf);
  const double c1 = __ldg(m.ecoef + 2 * e), c2 = __ldg(m.ecoef + 2 * e + 1);
  const uint32_t q1 = lq(n1, L, k), q2 = lq(n2, L, k);
  const int64_t ts = in.tstride;
  const int tg = in.tg;
  double T1[NTR], T2[NTR], O1[NTR], O2[NTR], g0[NTR], g1[NTR], g2[NTR], g3[NTR];
  ldn<NTR, IL>(in.T, q1, t0, ts, tg, T1);
  ldn<NTR, IL>(in.T, q2, t0, ts, tg, T2);
  ldn<NTR, IL>(in.T_old, q1, t0, ts, tg, O1);
  ldn<NTR, IL>(in.T_old, q2, t0, ts, tg, O2);
  if (use_tri) {   // a mesh whose up/down cells do not hold the edge's nodes
    const int4 cu = __ldg(m.eud4 + 2 * e), cd = __ldg(m.eud4 + 2 * e + 1);
    cell_grad<NTR, IL>(in, cu.x, cu.y, cu.z, cu.w, k, t0, g0, g2);
    cell_grad<NTR, IL>(in, cd.x, cd.y, cd.z, cd.w, k, t0, g1, g3);
  } else {
    node_avg_grad<NTR, IL>(in, n1, k, t0, g0, g2);
    node_avg_grad<NTR, IL>(in, n2, k, t0, g1, g3);
  }
  double adf[NTR];
  const Rcp r6{6.0, 1.0 / 6.0, true};
#pragma unroll
  for (int t = 0; t < NTR; ++t) {
    const double fl = -0.5 * (T1[t] * (vf + avf) + T2[t] * (vf - avf));
    const double A1 = ab2(T1[t], O1[t]), A2 = ab2(T2[t], O2[t]);
    const double diff = A2 - A1;
    const double Tm1 = A1 + divr(2.0 * diff + c1 * g0[t] + c2 * g2[t], r6);
    const double Tm2 = A2 - divr(2.0 * diff + c1 * g1[t] + c2 * g3[t], r6);
    const double ho = -0.5 * ((vf + avf) * Tm1 + (vf - avf) * Tm2);
    adf[t] = ho - fl;
  }
  stn<NTR, IL>(in.ws.adfh, lq(e, L, k), w0, in.ws.sEd, in.wtg, adf);
}

// ---------------------------------------- limiter factors on a node's layer run
// The cluster bound of node n at level k is the max (min) of max(LO, T) (min(LO, T)) over
// the nodes of n's cells that are wet at k, padded with -BIG (+BIG) when one of n's cells
// is dry at k (tracer_adv.py:389-405). Every cell of n has two edges at n, so those nodes
// are n itself (when any cell is wet at k) and the edge neighbours with a wet cell at k;
// max/min are exact, so this equals the per-cell evaluation bit for bit.
// The a4 window (k-1, k, k+1 of the same column) crosses a run's ends: each thread leaves
// the bounds of its run's first and last level in shared memory, and the neighbouring
// runs of the column (the adjacent segment slots of the block: a column's runs are
// consecutive) read them. A block's first and last slot are halo runs that only publish
// their bounds; ``sh`` holds [4][NTR][256] doubles (first-level max, min, last-level max,
// min) and ``S`` is the distance between adjacent slots in threads.
template <int NTR, int LPT, bool IL>
__device__ __forceinline__ void seg_node_limit(const Inst& in, int64_t si, bool core, int t0,
                                               int w0, int tid, int S, double* sh) {
  const DevMesh& m = *in.m;
  constexpr int V = seg_variant(LPT);
  const bool valid = si >= 0 && si < m.n_nseg[V];
  const int L = m.L;
  const int64_t sN = in.ws.sN;
  int n = 0, k0 = 0, nzmin = 0, nzmax = 1, nk = 1;
  uint32_t base = 0;
  double mx[LPT][NTR], mn[LPT][NTR], sp[LPT][NTR], sm[LPT][NTR], lo[LPT][NTR];
#pragma unroll
  for (int l = 0; l < LPT; ++l)
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      mx[l][t] = -INFINITY; mn[l][t] = INFINITY; sp[l][t] = 0.0; sm[l][t] = 0.0;
      lo[l][t] = 0.0;
    }
  if (valid) {
    const uint32_t sg = __ldg(m.nseg[V] + si);
    n = lane_ent(sg);
    k0 = lane_lev(sg);
    const int4 rec = __ldg(m.nrec + n);
    const unsigned pk = unsigned(rec.z);
    nzmin = int(pk & 255u);
    nzmax = int((pk >> 8) & 255u);
    nk = min(LPT, nzmax - k0);
    base = lq(n, L, 0);
    unsigned long long fl_[LPT];   // the run's node-layer flags (0 beyond the run)
#pragma unroll
    for (int l = 0; l < LPT; ++l)
      fl_[l] = l < nk ? __ldg(m.nflags + rec.w + (k0 + l - nzmin)) : 0ull;
    const int e0 = rec.x, e1 = rec.x + int((pk >> 16) & 255u);
    FCT_SLOT_BEGIN(e0, e1)
    for (int j = e0; j < e1; ++j) {
      FCT_SLOT_GET(j, e1)
      const int jj = j - e0;
      const double sg1 = (sl.x & 1) ? -1.0 : 1.0;   // adf_h leaves the edge's first node
      const uint32_t qo = lq(sl.y, L, 0), qe = lq(sl.x >> 1, L, 0);
#pragma unroll
      for (int l = 0; l < LPT; ++l) {
        const int kc = kclamp(k0 + l, L);
        const bool wet = ((fl_[l] >> (kSlotWet + jj)) & 1ull);
        const bool on = ((fl_[l] >> jj) & 1ull);
        double lv[NTR], tv[NTR], a[NTR];
        ldv<NTR, IL>(in.ws.lo, qo + uint32_t(kc), w0, sN, in.wtg, lv);
        ldv<NTR, IL>(in.T, qo + uint32_t(kc), t0, in.tstride, in.tg, tv);
        ldv<NTR, IL>(in.ws.adfh, qe + uint32_t(kc), w0, in.ws.sEd, in.wtg, a);
#pragma unroll
        for (int t = 0; t < NTR; ++t) {
          mx[l][t] = wet ? dmax(mx[l][t], dmax(lv[t], tv[t])) : mx[l][t];
          mn[l][t] = wet ? dmin(mn[l][t], dmin(lv[t], tv[t])) : mn[l][t];
          const double sv = sg1 * a[t];
          sp[l][t] = on ? sp[l][t] + dmax(sv, 0.0) : sp[l][t];
          sm[l][t] = on ? sm[l][t] + dmin(sv, 0.0) : sm[l][t];
        }
      }
    }
    // the node itself, and the padding of dry cells
#pragma unroll
    for (int l = 0; l < LPT; ++l) {
      const int kc = kclamp(k0 + l, L);
      double tv[NTR];
      ldv<NTR, IL>(in.ws.lo, base + uint32_t(kc), w0, sN, in.wtg, lo[l]);
      ldv<NTR, IL>(in.T, base + uint32_t(kc), t0, in.tstride, in.tg, tv);
      const bool ow = (fl_[l] >> kOwnBit) & 1ull, of = (fl_[l] >> kOffBit) & 1ull;
#pragma unroll
      for (int t = 0; t < NTR; ++t) {
        if (ow) {
          mx[l][t] = dmax(mx[l][t], dmax(lo[l][t], tv[t]));
          mn[l][t] = dmin(mn[l][t], dmin(lo[l][t], tv[t]));
        }
        if (of) {
          mx[l][t] = dmax(mx[l][t], -kBig);
          mn[l][t] = dmin(mn[l][t], kBig);
        }
      }
    }
    // publish the first and last level's bounds for the neighbouring runs
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      sh[(0 * NTR + t) * 256 + tid] = mx[0][t];
      sh[(1 * NTR + t) * 256 + tid] = mn[0][t];
    }
#pragma unroll
    for (int l = 0; l < LPT; ++l)
      if (l == nk - 1)
#pragma unroll
        for (int t = 0; t < NTR; ++t) {
          sh[(2 * NTR + t) * 256 + tid] = mx[l][t];
          sh[(3 * NTR + t) * 256 + tid] = mn[l][t];
        }
  }
  __syncthreads();
  if (!valid || !core) return;
  const double dt = in.dt;
#pragma unroll
  for (int l = 0; l < LPT; ++l) {
    if (l >= nk) break;
    const int k = k0 + l;
    const uint32_t qn = base + uint32_t(k);
    const bool interior = k != nzmin && k != nzmax - 1;   // a4: window over k-1, k, k+1
    const double av = __ldg(m.areasvol + qn), hnn = __ldg(in.hnode_new + qn);
    const bool valid_n = (av > 0.0) && (hnn > 0.0);
    const double sa = av > 0.0 ? av : 1.0, sh_ = hnn > 0.0 ? hnn : 1.0;
    const double fdt = dt * __drcp_rn(sa * sh_);   // dt / (areasvol * hnode_new)
    double ft[NTR], fb[NTR];
    ldv<NTR, IL>(in.ws.adfv, qn, w0, sN, in.wtg, ft);
    if (k + 1 < nzmax) {
      ldv<NTR, IL>(in.ws.adfv, qn + 1, w0, sN, in.wtg, fb);
    } else {   // the bottom interface carries no flux
#pragma unroll
      for (int t = 0; t < NTR; ++t) fb[t] = 0.0;
    }
    double pf[NTR], mf[NTR];
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      double wmx = mx[l][t], wmn = mn[l][t];
      if (interior) {
        const double ax = l > 0 ? mx[l - 1][t] : sh[(2 * NTR + t) * 256 + tid - S];
        const double an = l > 0 ? mn[l - 1][t] : sh[(3 * NTR + t) * 256 + tid - S];
        const double bx = l + 1 < nk ? mx[l + 1 < LPT ? l + 1 : l][t]
                                     : sh[(0 * NTR + t) * 256 + tid + S];
        const double bn = l + 1 < nk ? mn[l + 1 < LPT ? l + 1 : l][t]
                                     : sh[(1 * NTR + t) * 256 + tid + S];
        wmx = dmax(dmax(ax, wmx), bx);
        wmn = dmin(dmin(an, wmn), bn);
      }
      const double plus = (dmax(ft[t], 0.0) + dmax(-fb[t], 0.0)) + sp[l][t];
      const double minus = (dmin(ft[t], 0.0) + dmin(-fb[t], 0.0)) + sm[l][t];
      pf[t] = 1.0;
      mf[t] = 1.0;
      if (valid_n) {
        const double flux_pos = fma(plus, fdt, kFluxEps);
        const double flux_neg = fma(minus, fdt, -kFluxEps);
        pf[t] = dmin(1.0, (wmx - lo[l][t]) * __drcp_rn(flux_pos));
        mf[t] = dmin(1.0, (wmn - lo[l][t]) * __drcp_rn(flux_neg));
      }
    }
    stv<NTR, IL>(in.ws.pf, qn, w0, sN, in.wtg, pf);
    stv<NTR, IL>(in.ws.mf, qn, w0, sN, in.wtg, mf);
  }
}

// ------------------- zalesak b3 + flux2dtracer_fct + ale_reconstruct on a layer run
template <int NTR, int LPT, bool IL>
__device__ __forceinline__ void seg_node_final(const Inst& in, int64_t si, int t0, int w0) {
  const DevMesh& m = *in.m;
  constexpr int V = seg_variant(LPT);
  constexpr int NB = LPT + 2;   // factor levels k0-1 .. k0+LPT
  if (si >= m.n_nseg[V]) return;
  const uint32_t sg = __ldg(m.nseg[V] + si);
  const int n = lane_ent(sg), k0 = lane_lev(sg), L = m.L;
  const int4 rec = __ldg(m.nrec + n);
  const unsigned pk = unsigned(rec.z);
  const int nzmin = int(pk & 255u), nzmax = int((pk >> 8) & 255u);
  const int nk = min(LPT, nzmax - k0);
  const uint32_t base = lq(n, L, 0);
  const int64_t sN = in.ws.sN;
  const int tg = in.tg;
  // limited horizontal fluxes, ascending edge id
  double hsc[LPT][NTR];
#pragma unroll
  for (int l = 0; l < LPT; ++l)
#pragma unroll
    for (int t = 0; t < NTR; ++t) hsc[l][t] = 0.0;
  double pfw[NB][NTR], mfw[NB][NTR];   // own factors at levels k0-1 .. k0+LPT
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const uint32_t q = base + uint32_t(kclamp(k0 - 1 + b, L));
    ldv<NTR, IL>(in.ws.pf, q, w0, sN, in.wtg, pfw[b]);
    ldv<NTR, IL>(in.ws.mf, q, w0, sN, in.wtg, mfw[b]);
  }
  unsigned long long fl_[LPT];   // the run's node-layer flags (0 beyond the run)
#pragma unroll
  for (int l = 0; l < LPT; ++l) fl_[l] = l < nk ? __ldg(m.nflags + rec.w + (k0 + l - nzmin)) : 0ull;
  const int e0 = rec.x, e1 = rec.x + int((pk >> 16) & 255u);
  FCT_SLOT_BEGIN(e0, e1)
  for (int j = e0; j < e1; ++j) {
    FCT_SLOT_GET(j, e1)
    const int jj = j - e0;
    const bool second = sl.x & 1;
    const double sg1 = second ? -1.0 : 1.0;   // adf_h leaves the edge's first node
    const uint32_t qo = lq(sl.y, L, 0), qe = lq(sl.x >> 1, L, 0);
#pragma unroll
    for (int l = 0; l < LPT; ++l) {
      const int kc = kclamp(k0 + l, L);
      const bool on = ((fl_[l] >> jj) & 1ull);
      double a[NTR], pfo[NTR], mfo[NTR];
      ldv<NTR, IL>(in.ws.adfh, qe + uint32_t(kc), w0, in.ws.sEd, in.wtg, a);
      ldv<NTR, IL>(in.ws.pf, qo + uint32_t(kc), w0, sN, in.wtg, pfo);
      ldv<NTR, IL>(in.ws.mf, qo + uint32_t(kc), w0, sN, in.wtg, mfo);
#pragma unroll
      for (int t = 0; t < NTR; ++t) {
        // b3 (tracer_adv.py:461-465): adf >= 0 ? min(plus(n1), minus(n2)) : min(minus(n1),
        // plus(n2)); min is exact and symmetric, so in the node's own terms the factor is
        // min(own plus, other minus) when the flux leaves the node, else the other pair
        const double x1 = dmin(pfw[l + 1][t], mfo[t]), x2 = dmin(mfw[l + 1][t], pfo[t]);
        const double ae = ((a[t] >= 0.0) != second) ? x1 : x2;
        const double lim = ae * a[t];
        hsc[l][t] = on ? hsc[l][t] + sg1 * lim : hsc[l][t];
      }
    }
  }
  const double dt = in.dt;
#pragma unroll
  for (int l = 0; l < LPT; ++l) {
    if (l >= nk) break;
    const int k = k0 + l;
    const uint32_t qn = base + uint32_t(k);
    const double av = __ldg(m.areasvol + qn);
    const double sa = av > 0.0 ? av : 1.0;
    const double hn = __ldg(in.hnode + qn), hnn = __ldg(in.hnode_new + qn);
    const double fdt = dt * __drcp_rn(sa);   // dt / areasvol
    const Rcq rhn = rcpq(hnn);
    double ft[NTR], vt[NTR], vb[NTR];
    ldv<NTR, IL>(in.ws.adfv, qn, w0, sN, in.wtg, ft);
    // limited vertical flux at the top interface k (tracer_adv.py:453-459)
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      const double pf0 = pfw[l + 1][t], mf0 = mfw[l + 1][t];
      vt[t] = k == nzmin ? (ft[t] >= 0.0 ? pf0 : mf0) * ft[t]
                         : (ft[t] >= 0.0 ? dmin(mfw[l][t], pf0) : dmin(pfw[l][t], mf0)) * ft[t];
    }
    // limited vertical flux at the bottom interface k+1 (0 at the node's bottom)
    if (k + 1 >= nzmax) {
#pragma unroll
      for (int t = 0; t < NTR; ++t) vb[t] = 0.0;
    } else {
      double fb[NTR];
      ldv<NTR, IL>(in.ws.adfv, qn + 1, w0, sN, in.wtg, fb);
#pragma unroll
      for (int t = 0; t < NTR; ++t)
        vb[t] = (fb[t] >= 0.0 ? dmin(mfw[l + 1][t], pfw[l + 2][t])
                              : dmin(pfw[l + 1][t], mfw[l + 2][t])) * fb[t];
    }
    double Tv[NTR], lo[NTR], out[NTR];
    ldv<NTR, IL>(in.T, qn, t0, in.tstride, tg, Tv);
    ldv<NTR, IL>(in.ws.lo, qn, w0, sN, in.wtg, lo);
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      const double lo_trans = fma(lo[t], hnn, -Tv[t] * hn);
      const double vdiv = av > 0.0 ? (vt[t] - vb[t]) * fdt : 0.0;
      double d = fma(hsc[l][t], fdt, lo_trans + vdiv);
      d = fma(Tv[t], hn - hnn, d);
      out[t] = Tv[t] + (hnn > 0.0 ? divq(d, rhn) : 0.0);
    }
    stv<NTR, IL>(in.T_new, qn, t0, in.tstride, tg, out);
    count_nonfinite<NTR>(in.nonfinite, out);
  }
}

// ------------------------------------------------------------- kernels and launchers
// Kernel wrappers: ``_1`` takes one instance by value (tracer-major layout, the
// single-call path; tracer slice = blockIdx.y), ``_n`` instance blockIdx.y of a device
// table (interleaved layout; 2^lg adjacent threads of a segment take adjacent tracer
// slices, so together they read whole interleaved lines).
// Resident 256-thread blocks per SM the compiler must fit, by the updates a thread
// carries (registers capped accordingly: the gathers are latency-bound, so resident warps
// pay more than the spills a cap may cost). Measured on the CORE2-size batched step: one
// block more per SM than 6/4/3/2/1 made it 5.5% faster (the autotuner then picks other
// mappings), two more 1-9% slower.
__host__ __device__ constexpr int seg_min_blocks(int ntr, int lpt) {
  return ntr * lpt <= 1 ? 7 : ntr * lpt <= 2 ? 5 : ntr * lpt <= 4 ? 4 : ntr * lpt <= 8 ? 3 : 2;
}

#define FCT_SEG_KERNEL(name, body)                                                       \
  template <int NTR, int LPT>                                                            \
  __global__ void __launch_bounds__(256, seg_min_blocks(NTR, LPT))                       \
      name##_1(Inst in, int t0, int w0) {                                                \
    const int sub = int(blockIdx.y) * NTR;                                               \
    body<NTR, LPT, false>(in, lane_index(), t0 + sub, w0 + sub);                         \
  }                                                                                      \
  template <int NTR, int LPT>                                                            \
  __global__ void __launch_bounds__(256, seg_min_blocks(NTR, LPT))                       \
      name##_n(const Inst* __restrict__ tab, int t0, int w0, int lg) {                   \
    const int64_t g = lane_index();                                                      \
    const int sub = int(g & ((int64_t(1) << lg) - 1)) * NTR;                             \
    body<NTR, LPT, true>(tab[blockIdx.y], g >> lg, t0 + sub, w0 + sub);                  \
  }

// The limiter stage: 256-thread blocks of 256/S segment slots (S = 2^lg tracer-slice
// threads per slot in ``_n``, 1 in ``_1``), the first and last slot halo runs.
#define FCT_SEG_LIMIT_KERNEL(name)                                                       \
  template <int NTR, int LPT>                                                            \
  __global__ void __launch_bounds__(256, seg_min_blocks(NTR, LPT))                       \
      name##_1(Inst in, int t0, int w0) {                                                \
    __shared__ double sh[4 * NTR * 256];                                                 \
    const int tid = threadIdx.x;                                                         \
    const int64_t si = int64_t(blockIdx.x) * 254 + tid - 1;                              \
    const int sub = int(blockIdx.y) * NTR;                                               \
    seg_node_limit<NTR, LPT, false>(in, si, tid >= 1 && tid <= 254, t0 + sub, w0 + sub,  \
                                    tid, 1, sh);                                         \
  }                                                                                      \
  template <int NTR, int LPT>                                                            \
  __global__ void __launch_bounds__(256, seg_min_blocks(NTR, LPT))                       \
      name##_n(const Inst* __restrict__ tab, int t0, int w0, int lg) {                   \
    __shared__ double sh[4 * NTR * 256];                                                 \
    const int tid = threadIdx.x;                                                         \
    const int slot = tid >> lg, slots = 256 >> lg;                                       \
    const int64_t si = int64_t(blockIdx.x) * (slots - 2) + slot - 1;                     \
    const int sub = (tid & ((1 << lg) - 1)) * NTR;                                       \
    seg_node_limit<NTR, LPT, true>(tab[blockIdx.y], si, slot >= 1 && slot <= slots - 2,  \
                                   t0 + sub, w0 + sub, tid, 1 << lg, sh);                \
  }

inline unsigned seg_blocks(int64_t lanes) {
  return unsigned(std::max<int64_t>(1, (lanes + 255) / 256));
}
// grids: one thread per segment and slice; the limiter's blocks hold 256/S - 2 core slots
#define FCT_GRID_N(lanes, lg) seg_blocks((lanes) << (lg))
#define FCT_GRID_1(lanes) seg_blocks(lanes)
#define FCT_LIMIT_GRID_N(lanes, lg) \
  unsigned(std::max<int64_t>(1, ((lanes) + (256 >> (lg)) - 3) / ((256 >> (lg)) - 2)))
#define FCT_LIMIT_GRID_1(lanes) unsigned(std::max<int64_t>(1, ((lanes) + 253) / 254))

// Tracers per thread of one launch: the largest of the compiled set (1, 2 or 4 in the
// interleaved layout, 1 when its strides are odd; 1 or 2 tracer-major) that is at most
// ``rem`` and ``per_thread``.
inline int seg_tracers(int rem, int per_thread, bool interleaved, int lpt, bool even) {
  (void)lpt;
  const int lim = std::min(rem, per_thread);
  if (interleaved && !even) return 1;   // tracer pairs would not be 16-byte aligned
  if (interleaved && lim >= 4) return 4;
  return lim >= 2 ? 2 : 1;
}
// the interleaved tracer and workspace strides are even (tracer pairs 16-byte aligned)
inline bool seg_even(const LaunchDims& d) {
  const int chunk = d.chunk > 0 ? d.chunk : d.ntr;
  return d.ntr % 2 == 0 && chunk % 2 == 0;
}

#define FCT_SEG_CASE_N(kern, P, V)                                                       \
  case P * 16 + V:                                                                       \
    kern##_n<P, V><<<g, 256, 0, s>>>(tab, t0, w0, lg);                                   \
    break;
#define FCT_SEG_CASE_1(kern, P, V)                                                       \
  case P * 16 + V:                                                                       \
    kern##_1<P, V><<<g, 256, 0, s>>>(single, t0, w0);                                    \
    break;

// One segment stage over the tracers [c0, c1) of a workspace chunk (workspace index of
// tracer t is t - c0): launches of P tracers x 2^lg slices. ``COUNT(V)`` is the largest
// segment count of the variant over the launch's instances.
#define FCT_SEG_LAUNCHER(fn, kern, COUNT, GRID_N, GRID_1, STAGE)                         \
  int fn(const Inst& single, const Inst* tab, int n, const LaunchDims& d, int c0, int c1, \
         cudaStream_t s) {                                                               \
    const int lpt = d.smap_levels[STAGE], per_thread = d.smap_tracers[STAGE];            \
    const int V = seg_variant(lpt);                                                      \
    const int64_t lanes = COUNT(V);                                                      \
    for (int t0 = c0; t0 < c1;) {                                                        \
      const int rem = c1 - t0;                                                           \
      const int P = seg_tracers(rem, per_thread, tab != nullptr, lpt, seg_even(d));      \
      int lg = 0;                                                                        \
      while (lg < 3 && (P << (lg + 1)) <= rem) ++lg;                                     \
      const int w0 = t0 - c0;                                                            \
      if (tab) {                                                                         \
        const dim3 g(GRID_N(lanes, lg), unsigned(n));                                    \
        switch (P * 16 + lpt) {                                                          \
          FCT_SEG_CASE_N(kern, 1, 1) FCT_SEG_CASE_N(kern, 1, 2)                          \
          FCT_SEG_CASE_N(kern, 1, 4) FCT_SEG_CASE_N(kern, 1, 8)                          \
          FCT_SEG_CASE_N(kern, 2, 1) FCT_SEG_CASE_N(kern, 2, 2)                          \
          FCT_SEG_CASE_N(kern, 2, 4) FCT_SEG_CASE_N(kern, 2, 8)                          \
          FCT_SEG_CASE_N(kern, 4, 1) FCT_SEG_CASE_N(kern, 4, 2)                          \
          FCT_SEG_CASE_N(kern, 4, 4) FCT_SEG_CASE_N(kern, 4, 8)                          \
          default:                                                                       \
            return set_error(FCT_ERR_INVALID, "no segment kernel for %d tracers x %d "  \
                             "levels per thread", P, lpt);                              \
        }                                                                                \
      } else {                                                                           \
        const dim3 g(GRID_1(lanes), 1u << lg);                                           \
        switch (P * 16 + lpt) {                                                          \
          FCT_SEG_CASE_1(kern, 1, 1) FCT_SEG_CASE_1(kern, 1, 2)                          \
          FCT_SEG_CASE_1(kern, 1, 4) FCT_SEG_CASE_1(kern, 1, 8)                          \
          FCT_SEG_CASE_1(kern, 2, 1) FCT_SEG_CASE_1(kern, 2, 2)                          \
          FCT_SEG_CASE_1(kern, 2, 4) FCT_SEG_CASE_1(kern, 2, 8)                          \
          default:                                                                       \
            return set_error(FCT_ERR_INVALID, "no segment kernel for %d tracers x %d "  \
                             "levels per thread", P, lpt);                              \
        }                                                                                \
      }                                                                                  \
      t0 += P << lg;                                                                     \
    }                                                                                    \
    const cudaError_t e = cudaGetLastError();                                            \
    return e == cudaSuccess ? FCT_OK : cuda_error(e, #fn);                               \
  }

}  // namespace
}  // namespace fct
