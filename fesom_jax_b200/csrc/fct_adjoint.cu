// Reverse mode of the FCT step (fct_adjoint) and of compute_w (fct_compute_w_adjoint).
//
// The forward step is recomputed first (the stage kernels of fct_forward write their
// intermediates to the plan workspace); the reverse kernels below then walk the stages
// backwards. Every transpose of a forward scatter is again a deterministic gather over a
// CSR list, so cotangents are bit-identical run to run.
//
// Reverse stage map (forward function in fesom_jax/tracer_adv.py -> reverse kernel):
//   ale_reconstruct (:142-151), flux2dtracer_fct (:469-484)       -> r_seed
//   zalesak_limit b3 (:453-465)                                    -> r_factors
//   zalesak_limit b2 (:441-451), a4 window minus LO (:417-418)     -> r_ratio
//   zalesak_limit a4 vertical window max/min (:412-416)            -> r_window
//   zalesak_limit a3 segment_max/min (:399-405)                    -> r_cluster
//   zalesak_limit a1-a2 (:389-397)                                 -> r_bounds
//   compute_fct_lo (:298-313)                                      -> r_lo
//   adv_flux_hor_ho (:196-225), adv_flux_hor (:96-105), b1 edges   -> r_edge
//   fill_up_dn_grad (:344-368), _node_avg_grad (:329-341)          -> r_gnode, r_tr
//   tracer_gradient_elements (:316-326)                            -> r_grad_t
//   adv_flux_ver_ho (:241-295), adv_flux_ver (:108-120), b1 vertical -> r_vert_a, r_vert_b
//   tracer_ab (:59-66), assembly of dT, dT_old                    -> r_final
//   edge_vflux (:69-93)                                            -> r_uv
//   ale.compute_w (fesom_jax/ale.py:309-365)                       -> r_w_div, r_w_uv
//
// Subgradients follow JAX: maximum/minimum split the cotangent equally at a tie,
// max over an element's vertices and segment_max/min spread it evenly over tied
// entries, abs'(0) = 0 (so d max(x, 0)/dx = 1/2 at x = 0).
#include <algorithm>

#include "fct_host.h"

using namespace fct;

namespace {

constexpr int B = 256;

__device__ __forceinline__ int64_t lane_index() {
  return int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
}
__device__ __forceinline__ double ab2(double T, double To) { return kAbOld * To + kAbNew * T; }
__device__ __forceinline__ double safe_nz(double x) { return x == 0.0 ? 1.0 : x; }
__device__ __forceinline__ double sgn(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }
// share of d max(a, b) that goes to a / to b
__device__ __forceinline__ double smax_a(double a, double b) { return a > b ? 1.0 : (a == b ? 0.5 : 0.0); }
__device__ __forceinline__ double smax_b(double a, double b) { return b > a ? 1.0 : (a == b ? 0.5 : 0.0); }
__device__ __forceinline__ double smin_a(double a, double b) { return a < b ? 1.0 : (a == b ? 0.5 : 0.0); }
__device__ __forceinline__ double smin_b(double a, double b) { return b < a ? 1.0 : (a == b ? 0.5 : 0.0); }
// d max(x, 0)/dx and d min(x, 0)/dx
__device__ __forceinline__ double dmax0(double x) { return x > 0.0 ? 1.0 : (x == 0.0 ? 0.5 : 0.0); }
__device__ __forceinline__ double dmin0(double x) { return x < 0.0 ? 1.0 : (x == 0.0 ? 0.5 : 0.0); }

struct Adj {
  Inst in;               // forward fields + forward workspace (recomputed)
  AdjWorkspace a;
  const double* gTn;     // cotangent of T_new (tracer-major, in.tstride)
  double *gT, *gTo, *guv, *gw;
};

__device__ __forceinline__ bool edge_on(const DevMesh& m, int e, int k) {
  return k >= m.ekmin[e] && k < m.ekmax[e];
}
__device__ __forceinline__ bool elem_on(const DevMesh& m, int el, int k) {
  return k >= m.eul[el] && k < m.enl[el];
}

// cotangent reaching the limited vertical flux at interface j of node column `base`
__device__ __forceinline__ double gvl_at(const DevMesh& m, const double* gdel, int64_t base,
                                        int j, int nzmin, int nzmax, double dt) {
  double g = 0.0;
  if (j >= nzmin && j < nzmax) {
    const double av = m.areasvol[base + j];
    if (av > 0.0) g += gdel[base + j] * dt / av;
  }
  if (j - 1 >= nzmin && j - 1 < nzmax) {
    const double av = m.areasvol[base + j - 1];
    if (av > 0.0) g -= gdel[base + j - 1] * dt / av;
  }
  return g;
}

// ------------------------------------------------------------------ r_seed
__global__ void __launch_bounds__(B) r_seed(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_layer) return;
  const uint32_t lane = m.layer_lanes[i];
  const int n = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int64_t qn = int64_t(n) * L + k;
  const double hn = in.hnode[qn], hnn = in.hnode_new[qn];
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t o = t * A.a.sN;
    const double g = A.gTn[t * in.tstride + qn];
    double gT = g, gdel = 0.0;
    if (hnn > 0.0) {
      gdel = g / hnn;                 // T_new = T + d / hnn
      gT += gdel * (hn - hnn);        // d = del + T (hn - hnn)
    }
    gT += -gdel * hn;                 // lo_trans = -T hn + LO hnn
    A.a.gdel[o + qn] = gdel;
    A.a.gLOd[o + qn] = gdel * hnn;
    A.a.gTd[o + qn] = gT;
  }
}

// --------------------------------------------- r_factors: cotangents of pf, mf
__global__ void __launch_bounds__(B) r_factors(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_layer) return;
  const uint32_t lane = m.layer_lanes[i];
  const int n = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int nzmin = m.nzmin[n], nzmax = m.nzmax[n];
  const int64_t base = int64_t(n) * L, qn = base + k;
  const double dt = in.dt;
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t o = t * in.ws.sN;
    const double* pf = in.ws.pf + o;
    const double* mf = in.ws.mf + o;
    const double* adfv = in.ws.adfv + o;
    const double* gdel = A.a.gdel + t * A.a.sN;
    double gp = 0.0, gm = 0.0;
    // vertical limited flux at interface k (this node's own factors at k)
    {
      const double f = adfv[qn];
      const double g_ae = gvl_at(m, gdel, base, k, nzmin, nzmax, dt) * f;
      if (k == nzmin) {
        if (f >= 0.0) gp += g_ae; else gm += g_ae;
      } else if (f >= 0.0) {
        gp += g_ae * smin_b(mf[qn - 1], pf[qn]);
      } else {
        gm += g_ae * smin_b(pf[qn - 1], mf[qn]);
      }
    }
    // vertical limited flux at interface k+1 (uses this node's factors as the k-1 ones)
    if (k + 1 < nzmax) {
      const double f = adfv[qn + 1];
      const double g_ae = gvl_at(m, gdel, base, k + 1, nzmin, nzmax, dt) * f;
      if (f >= 0.0) gm += g_ae * smin_a(mf[qn], pf[qn + 1]);
      else gp += g_ae * smin_a(pf[qn], mf[qn + 1]);
    }
    // horizontal limited fluxes of the incident edges
    const double av0 = m.areasvol[qn];
    const double ghsc0 = gdel[qn] * dt / (av0 > 0.0 ? av0 : 1.0);
    for (int j = m.ne_off[n]; j < m.ne_off[n + 1]; ++j) {
      const int idx = m.ne_idx[j], e = idx >> 1;
      if (!edge_on(m, e, k)) continue;
      const int64_t qo = int64_t(m.ne_oth[j]) * L + k;
      const double avo = m.areasvol[qo];
      const double ghsco = gdel[qo] * dt / (avo > 0.0 ? avo : 1.0);
      const bool second = idx & 1;
      const double glim = second ? (ghsco - ghsc0) : (ghsc0 - ghsco);
      const double a = in.ws.adfh[t * in.ws.sEd + int64_t(e) * L + k];
      const double g_ae = glim * a;
      const double pf1 = second ? pf[qo] : pf[qn], mf1 = second ? mf[qo] : mf[qn];
      const double pf2 = second ? pf[qn] : pf[qo], mf2 = second ? mf[qn] : mf[qo];
      if (a >= 0.0) {   // ae = min(pf[n1], mf[n2])
        if (!second) gp += g_ae * smin_a(pf1, mf2); else gm += g_ae * smin_b(pf1, mf2);
      } else {          // ae = min(mf[n1], pf[n2])
        if (!second) gm += g_ae * smin_a(mf1, pf2); else gp += g_ae * smin_b(mf1, pf2);
      }
    }
    A.a.gpf[t * A.a.sN + qn] = gp;
    A.a.gmf[t * A.a.sN + qn] = gm;
  }
}

// ------------------------------- r_ratio: pf = min(1, fmax_w / flux_pos), likewise mf
__global__ void __launch_bounds__(B) r_ratio(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_layer) return;
  const uint32_t lane = m.layer_lanes[i];
  const int n = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int nzmin = m.nzmin[n], nzmax = m.nzmax[n];
  const int64_t qn = int64_t(n) * L + k;
  const double av = m.areasvol[qn], hnn = in.hnode_new[qn];
  const bool valid = (av > 0.0) && (hnn > 0.0);
  const double sa = av > 0.0 ? av : 1.0, sh = hnn > 0.0 ? hnn : 1.0;
  const double dt = in.dt;
  const bool use_own = (k == nzmin) || (k == nzmax - 1);
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t o = t * in.ws.sN, oa = t * A.a.sN;
    double gtmax = 0.0, gtmin = 0.0, gplus = 0.0, gminus = 0.0;
    if (valid) {
      const double* tv = in.ws.tvmax + o;
      const double* tn = in.ws.tvmin + o;
      double tmax = tv[qn], tmin = tn[qn];
      if (!use_own) {
        tmax = fmax(fmax(tv[qn - 1], tv[qn]), tv[qn + 1]);
        tmin = fmin(fmin(tn[qn - 1], tn[qn]), tn[qn + 1]);
      }
      const double lo = in.ws.lo[o + qn];
      const double plus = in.ws.fplus[o + qn], minus = in.ws.fminus[o + qn];
      const double fmax_w = tmax - lo, fmin_w = tmin - lo;
      const double flux_pos = plus * dt / sa / sh + kFluxEps;
      const double flux_neg = minus * dt / sa / sh - kFluxEps;
      const double rp = fmax_w / flux_pos, rm = fmin_w / flux_neg;
      const double grp = A.a.gpf[oa + qn] * smin_b(1.0, rp);
      const double grm = A.a.gmf[oa + qn] * smin_b(1.0, rm);
      gtmax = grp / flux_pos;
      gtmin = grm / flux_neg;
      gplus = (-grp * fmax_w / (flux_pos * flux_pos)) * dt / sa / sh;
      gminus = (-grm * fmin_w / (flux_neg * flux_neg)) * dt / sa / sh;
    }
    A.a.gtmax[oa + qn] = gtmax;
    A.a.gtmin[oa + qn] = gtmin;
    A.a.gplus[oa + qn] = gplus;
    A.a.gminus[oa + qn] = gminus;
    A.a.gLOl[oa + qn] = -(gtmax + gtmin);
  }
}

// ------------------------ r_window: tmax(m) = max over tvert at m-1, m, m+1
__global__ void __launch_bounds__(B) r_window(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_layer) return;
  const uint32_t lane = m.layer_lanes[i];
  const int n = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int nzmin = m.nzmin[n], nzmax = m.nzmax[n];
  const int64_t base = int64_t(n) * L;
  for (int t = 0; t < in.ntr; ++t) {
    const double* tv = in.ws.tvmax + t * in.ws.sN + base;
    const double* tn = in.ws.tvmin + t * in.ws.sN + base;
    const double* gx = A.a.gtmax + t * A.a.sN + base;
    const double* gn = A.a.gtmin + t * A.a.sN + base;
    double gvx = 0.0, gvn = 0.0;
    for (int mm = k - 1; mm <= k + 1; ++mm) {
      if (mm < nzmin || mm >= nzmax) continue;
      if (mm == nzmin || mm == nzmax - 1) {
        if (mm == k) { gvx += gx[mm]; gvn += gn[mm]; }
        continue;
      }
      {  // max(max(a, b), c) with a = tv[mm-1], b = tv[mm], c = tv[mm+1]
        const double a = tv[mm - 1], b = tv[mm], c = tv[mm + 1];
        const double inner = fmax(a, b), go = gx[mm];
        const double gi = go * smax_a(inner, c), gc = go * smax_b(inner, c);
        if (k == mm - 1) gvx += gi * smax_a(a, b);
        if (k == mm) gvx += gi * smax_b(a, b);
        if (k == mm + 1) gvx += gc;
      }
      {
        const double a = tn[mm - 1], b = tn[mm], c = tn[mm + 1];
        const double inner = fmin(a, b), go = gn[mm];
        const double gi = go * smin_a(inner, c), gc = go * smin_b(inner, c);
        if (k == mm - 1) gvn += gi * smin_a(a, b);
        if (k == mm) gvn += gi * smin_b(a, b);
        if (k == mm + 1) gvn += gc;
      }
    }
    A.a.gtvmax[t * A.a.sN + base + k] = gvx;
    A.a.gtvmin[t * A.a.sN + base + k] = gvn;
  }
}

// ------------------- r_cluster: segment_max/min over a node's elements (even split)
__global__ void __launch_bounds__(B) r_cluster(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_elem) return;
  const uint32_t lane = m.elem_lanes[i];
  const int e = lane_ent(lane), k = lane_lev(lane), L = m.L;
  for (int t = 0; t < in.ntr; ++t) {
    const double* amax = in.ws.amax + t * in.ws.sE;
    const double* amin = in.ws.amin + t * in.ws.sE;
    const double vx = amax[int64_t(e) * L + k], vn = amin[int64_t(e) * L + k];
    double gx = 0.0, gn = 0.0;
    for (int v = 0; v < 3; ++v) {   // tie counts come from the forward recompute
      const int n = m.enodes[3 * e + v];
      const int64_t qn = int64_t(n) * L + k, qt = t * in.ws.sN + qn;
      if (vx == in.ws.tvmax[qt]) gx += A.a.gtvmax[t * A.a.sN + qn] / int(in.ws.ccx[qt]);
      if (vn == in.ws.tvmin[qt]) gn += A.a.gtvmin[t * A.a.sN + qn] / int(in.ws.ccn[qt]);
    }
    A.a.gamax[t * A.a.sE + int64_t(e) * L + k] = gx;
    A.a.gamin[t * A.a.sE + int64_t(e) * L + k] = gn;
  }
}

// ------------- r_bounds: element max/min over its vertices of max/min(LO, T) (even split)
__global__ void __launch_bounds__(B) r_bounds(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_layer) return;
  const uint32_t lane = m.layer_lanes[i];
  const int n = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int64_t qn = int64_t(n) * L + k;
  for (int t = 0; t < in.ntr; ++t) {
    const double* lo = in.ws.lo + t * in.ws.sN;
    const double* T = in.T + t * in.tstride;
    const double mxv = fmax(lo[qn], T[qn]), mnv = fmin(lo[qn], T[qn]);
    double gx = 0.0, gn = 0.0;
    for (int j = m.nel_off[n]; j < m.nel_off[n + 1]; ++j) {
      const int el = m.nel_idx[j];
      if (!elem_on(m, el, k)) continue;
      const int64_t qe = int64_t(el) * L + k;
      const double ex = in.ws.amax[t * in.ws.sE + qe], en = in.ws.amin[t * in.ws.sE + qe];
      if (mxv != ex && mnv != en) continue;
      const int64_t qc = t * in.ws.sE + qe;   // tie counts from the forward recompute
      if (mxv == ex) gx += A.a.gamax[t * A.a.sE + qe] / int(in.ws.ecx[qc]);
      if (mnv == en) gn += A.a.gamin[t * A.a.sE + qe] / int(in.ws.ecn[qc]);
    }
    const int64_t oa = t * A.a.sN;
    A.a.gLOb[oa + qn] = gx * smax_a(lo[qn], T[qn]) + gn * smin_a(lo[qn], T[qn]);
    A.a.gTb[oa + qn] = gx * smax_b(lo[qn], T[qn]) + gn * smin_b(lo[qn], T[qn]);
  }
}

// ------------------------------------------------------ r_lo: LO = numer / hnn
__global__ void __launch_bounds__(B) r_lo(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_layer) return;
  const uint32_t lane = m.layer_lanes[i];
  const int n = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int64_t qn = int64_t(n) * L + k;
  const double hn = in.hnode[qn], hnn = in.hnode_new[qn], av = m.areasvol[qn];
  const bool valid = (hnn > 0.0) && (av > 0.0);
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t oa = t * A.a.sN;
    const double gLO = A.a.gLOd[oa + qn] + A.a.gLOl[oa + qn] + A.a.gLOb[oa + qn];
    double gdiv = 0.0, gT = A.a.gTd[oa + qn] + A.a.gTb[oa + qn];
    if (valid) {
      const double gnum = gLO / hnn;
      gT += gnum * hn;
      gdiv = gnum * in.dt / av;
    }
    A.a.gdiv[oa + qn] = gdiv;
    A.a.gTp[oa + qn] = gT;
  }
}

// ------------------ r_edge: adf_h = HO - LO flux; cotangents of the edge inputs
__global__ void __launch_bounds__(B) r_edge(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_edge) return;
  const uint32_t lane = m.edge_lanes[i];
  const int e = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int n1 = m.edges[2 * e], n2 = m.edges[2 * e + 1];
  const int up = m.eupdn[2 * e], dn = m.eupdn[2 * e + 1];
  const int kmin = max(m.ulmax[n1], m.ulmax[n2]) - 1;
  const int kmax = min(m.nlmin[n1], m.nlmin[n2]) - 1;
  const bool use_tri = (up >= 0) && (dn >= 0) && k >= kmin && k < kmax;
  const int64_t qe = int64_t(e) * L + k, q1 = int64_t(n1) * L + k, q2 = int64_t(n2) * L + k;
  const double vf = in.ws.vflux[qe], avf = fabs(vf), s = sgn(vf);
  const double c1 = m.ecoef[2 * e], c2 = m.ecoef[2 * e + 1];
  const double av1 = m.areasvol[q1], av2 = m.areasvol[q2];
  const double dt = in.dt;
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t o = t * in.ws.sN, oa = t * A.a.sN, oe = t * A.a.sEd;
    const double* T = in.T + t * in.tstride;
    const double* To = in.T_old + t * in.tstride;
    const double a = in.ws.adfh[t * in.ws.sEd + qe];
    // limited flux lim = ae * a, with hsc(n1) += lim, hsc(n2) -= lim
    const double ghsc1 = A.a.gdel[oa + q1] * dt / (av1 > 0.0 ? av1 : 1.0);
    const double ghsc2 = A.a.gdel[oa + q2] * dt / (av2 > 0.0 ? av2 : 1.0);
    const double glim = ghsc1 - ghsc2;
    const double pf1 = in.ws.pf[o + q1], mf1 = in.ws.mf[o + q1];
    const double pf2 = in.ws.pf[o + q2], mf2 = in.ws.mf[o + q2];
    const double ae = a >= 0.0 ? fmin(pf1, mf2) : fmin(mf1, pf2);
    double ga = glim * ae;
    // fct_plus / fct_minus sums at both ends
    ga += A.a.gplus[oa + q1] * dmax0(a) + A.a.gminus[oa + q1] * dmin0(a);
    ga -= A.a.gplus[oa + q2] * dmax0(-a) + A.a.gminus[oa + q2] * dmin0(-a);
    // adf_h = HO - fl; fl also feeds LO through the divergence
    const double gHO = ga;
    const double gfl = -ga + (A.a.gdiv[oa + q1] - A.a.gdiv[oa + q2]);
    const double T1 = T[q1], T2 = T[q2];
    const double A1 = ab2(T1, To[q1]), A2 = ab2(T2, To[q2]);
    double g0, g1, g2, g3;
    if (use_tri) {
      const int64_t qu = t * in.ws.sE + int64_t(up) * L + k, qd = t * in.ws.sE + int64_t(dn) * L + k;
      g0 = in.ws.gx[qu]; g1 = in.ws.gx[qd]; g2 = in.ws.gy[qu]; g3 = in.ws.gy[qd];
    } else {
      g0 = in.ws.gnx[o + q1]; g1 = in.ws.gnx[o + q2]; g2 = in.ws.gny[o + q1]; g3 = in.ws.gny[o + q2];
    }
    const double diff = A2 - A1;
    const double Tm1 = A1 + (2.0 * diff + c1 * g0 + c2 * g2) / 6.0;
    const double Tm2 = A2 - (2.0 * diff + c1 * g1 + c2 * g3) / 6.0;
    // HO = -0.5 ((vf + |vf|) Tm1 + (vf - |vf|) Tm2); fl = -0.5 (T1 (vf + |vf|) + T2 (vf - |vf|));
    // the per-end terms of Tm1/Tm2 and T1/T2 are re-derived by the consumers (edge_terms)
    double gvf = -0.5 * ((1.0 + s) * Tm1 + (1.0 - s) * Tm2) * gHO;
    gvf += -0.5 * (T1 * (1.0 + s) + T2 * (1.0 - s)) * gfl;
    A.a.gHO[oe + qe] = gHO;
    A.a.gfl[oe + qe] = gfl;
    A.a.gvf[oe + qe] = gvf;
  }
}

// The per-end cotangents of edge e at level k (tracer t), re-derived from the stored
// gHO (of the MFCT flux) and gfl (of the upwind flux) with r_edge's expressions:
//   T1/T2: through the upwind flux; A1/A2: through ttfAB in Tm1/Tm2;
//   g0..g3: through the gradients in Tm1 (g0 = c1 gX1, g2 = c2 gX1) and Tm2 (g1, g3).
struct EdgeTerms {
  double gT1, gT2, gA1, gA2, gg0, gg1, gg2, gg3;
};
__device__ __forceinline__ EdgeTerms edge_terms(const Adj& A, int t, int e, int k) {
  const DevMesh& m = *A.in.m;
  const int64_t qe = int64_t(e) * m.L + k, oe = t * A.a.sEd;
  const double vf = A.in.ws.vflux[qe], avf = fabs(vf);
  const double gHO = A.a.gHO[oe + qe], gfl = A.a.gfl[oe + qe];
  const double c1 = m.ecoef[2 * e], c2 = m.ecoef[2 * e + 1];
  const double gTm1 = -0.5 * (vf + avf) * gHO, gTm2 = -0.5 * (vf - avf) * gHO;
  EdgeTerms r;
  r.gT1 = -0.5 * (vf + avf) * gfl;
  r.gT2 = -0.5 * (vf - avf) * gfl;
  const double gX1 = gTm1 / 6.0, gX2 = -gTm2 / 6.0;
  const double gdiff = 2.0 * gX1 + 2.0 * gX2;
  r.gA1 = gTm1 - gdiff;
  r.gA2 = gTm2 + gdiff;
  r.gg0 = c1 * gX1;
  r.gg2 = c2 * gX1;
  r.gg1 = c1 * gX2;
  r.gg3 = c2 * gX2;
  return r;
}

__device__ __forceinline__ bool use_tri_at(const DevMesh& m, int e, int k) {
  const int n1 = m.edges[2 * e], n2 = m.edges[2 * e + 1];
  const int up = m.eupdn[2 * e], dn = m.eupdn[2 * e + 1];
  const int kmin = max(m.ulmax[n1], m.ulmax[n2]) - 1;
  const int kmax = min(m.nlmin[n1], m.nlmin[n2]) - 1;
  return (up >= 0) && (dn >= 0) && k >= kmin && k < kmax;
}

// ------------- r_gnode: cotangent of the node-average gradient (fill_up_dn_grad else-branch)
__global__ void __launch_bounds__(B) r_gnode(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_layer) return;
  const uint32_t lane = m.layer_lanes[i];
  const int n = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int64_t qn = int64_t(n) * L + k;
  for (int t = 0; t < in.ntr; ++t) {
    double gx = 0.0, gy = 0.0;
    for (int j = m.ne_off[n]; j < m.ne_off[n + 1]; ++j) {
      const int idx = m.ne_idx[j], e = idx >> 1;
      if (!edge_on(m, e, k) || use_tri_at(m, e, k)) continue;
      const EdgeTerms et = edge_terms(A, t, e, k);
      if (idx & 1) { gx += et.gg1; gy += et.gg3; }
      else { gx += et.gg0; gy += et.gg2; }
    }
    A.a.ggnx[t * A.a.sN + qn] = gx;
    A.a.ggny[t * A.a.sN + qn] = gy;
  }
}

// ---------------- r_tr: cotangent of the element gradients (up/dn use + node average)
__global__ void __launch_bounds__(B) r_tr(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_elem) return;
  const uint32_t lane = m.elem_lanes[i];
  const int el = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const double aw = m.earea[el];
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t oa = t * A.a.sN;
    double gx = 0.0, gy = 0.0;
    for (int j = m.eud_off[el]; j < m.eud_off[el + 1]; ++j) {
      const int idx = m.eud_idx[j], e = idx >> 1;
      if (!edge_on(m, e, k) || !use_tri_at(m, e, k)) continue;
      const EdgeTerms et = edge_terms(A, t, e, k);
      if (idx & 1) { gx += et.gg1; gy += et.gg3; }   // down triangle
      else { gx += et.gg0; gy += et.gg2; }           // up triangle
    }
    for (int v = 0; v < 3; ++v) {   // gnode(n) = sum_e a_e tr_e / den(n)
      const int n = m.enodes[3 * el + v];
      const int64_t qn = int64_t(n) * L + k;
      const double dd = in.ws.nden[qn];   // the forward's (safe) denominator
      gx += A.a.ggnx[oa + qn] * aw / dd;
      gy += A.a.ggny[oa + qn] * aw / dd;
    }
    A.a.gtrx[t * A.a.sE + int64_t(el) * L + k] = gx;
    A.a.gtry[t * A.a.sE + int64_t(el) * L + k] = gy;
  }
}

// ------------------------- r_grad_t: tracer_gradient_elements transposed (on T)
__global__ void __launch_bounds__(B) r_grad_t(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_layer) return;
  const uint32_t lane = m.layer_lanes[i];
  const int n = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int64_t qn = int64_t(n) * L + k;
  for (int t = 0; t < in.ntr; ++t) {
    double g = 0.0;
    for (int j = m.nel_off[n]; j < m.nel_off[n + 1]; ++j) {
      const int el = m.nel_idx[j];
      if (!elem_on(m, el, k)) continue;
      const int iv = m.enodes[3 * el] == n ? 0 : (m.enodes[3 * el + 1] == n ? 1 : 2);
      const int64_t qe = t * A.a.sE + int64_t(el) * L + k;
      g += m.gsca[6 * el + iv] * A.a.gtrx[qe] + m.gsca[6 * el + 3 + iv] * A.a.gtry[qe];
    }
    A.a.gTtr[t * A.a.sN + qn] = g;
  }
}

// ------- r_vert_a / r_vert_b: vertical fluxes (QR4C HO, upwind LO) and their limiter terms.
// r_vert_a (one thread per layer interface j of a node): the cotangent gf of adf_v[j]
// (limiter application and the plus/minus sums), ghi = gf and gfv = -gf + gdiv terms,
// stored in the dead r_ratio outputs gtmax / gtmin, and gw[j] complete (only interface
// j feeds it). r_vert_b (one thread per node level k): gT[k] and gA[k] gathered from the
// interfaces j = k-1 .. k+2 in ascending j (the order of a column loop over j that
// scatters into gT / gA), so the per-level sums do not depend on the parallel split.
__device__ __forceinline__ void qr4c_depths(const Inst& in, const DevMesh& m, int64_t base,
                                            int j, double& Znz, double& Zm1, double& Zm2,
                                            double& Zp1, double& zb) {
  const int L = m.L;
  if (in.Z3d) {
    const double* Zc = in.Z3d + base;
    Znz = Zc[j]; Zm1 = Zc[j - 1]; Zm2 = Zc[j - 2]; Zp1 = Zc[j + 1 < L ? j + 1 : L - 1];
    zb = in.zbar3[base + j];
  } else {
    Znz = m.Zp[j]; Zm1 = m.Zp[j - 1]; Zm2 = m.Zp[j - 2]; Zp1 = m.Zp[j + 1 < L ? j + 1 : L - 1];
    zb = m.zbar[j];
  }
}

__global__ void __launch_bounds__(B) r_vert_a(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_layer) return;
  const uint32_t lane = m.layer_lanes[i];
  const int n = lane_ent(lane), j = lane_lev(lane), L = m.L;
  const int nzmin = m.nzmin[n], nzmax = m.nzmax[n];
  const int64_t base = int64_t(n) * L;
  const double dt = in.dt;
  const double w = in.w_e[base + j], area = m.area[base + j];
  const int jm = j > 0 ? j - 1 : 0;
  for (int t = 0; t < in.ntr; ++t) {
    const double* T = in.T + t * in.tstride + base;
    const double* To = in.T_old + t * in.tstride + base;
    const int64_t o = t * in.ws.sN, oa = t * A.a.sN;
    const double* pf = in.ws.pf + o + base;
    const double* mf = in.ws.mf + o + base;
    const double* gplus = A.a.gplus + oa + base;
    const double* gminus = A.a.gminus + oa + base;
    const double* gdiv = A.a.gdiv + oa + base;
    const double f = in.ws.adfv[o + base + j];
    double ae;
    if (j == nzmin) ae = f >= 0.0 ? pf[j] : mf[j];
    else ae = f >= 0.0 ? fmin(mf[j - 1], pf[j]) : fmin(pf[j - 1], mf[j]);
    double gf = gvl_at(m, A.a.gdel + oa, base, j, nzmin, nzmax, dt) * ae;
    gf += gplus[j] * dmax0(f) + gminus[j] * dmin0(f);
    if (j - 1 >= nzmin) gf -= gplus[j - 1] * dmax0(-f) + gminus[j - 1] * dmin0(-f);
    const double ghi = gf;
    double gfv = -gf + gdiv[j];
    if (j - 1 >= nzmin) gfv -= gdiv[j - 1];
    A.a.gtmax[oa + base + j] = ghi;
    A.a.gtmin[oa + base + j] = gfv;
    double gw = 0.0;
    gw += -0.5 * (T[j] * (1.0 + sgn(w)) + T[jm] * (1.0 - sgn(w))) * area * gfv;
    if (j == nzmin) {
      gw += -ab2(T[j], To[j]) * area * ghi;
    } else if (j == nzmin + 1 || j == nzmax - 1) {
      gw += -0.5 * (ab2(T[j - 1], To[j - 1]) + ab2(T[j], To[j])) * area * ghi;
    } else if (j >= nzmin + 2 && j <= nzmax - 2) {
      double Znz, Zm1, Zm2, Zp1, zb;
      qr4c_depths(in, m, base, j, Znz, Zm1, Zm2, Zp1, zb);
      const double dc = safe_nz(Zm1 - Znz), du = safe_nz(Znz - Zp1), dd = safe_nz(Zm2 - Zm1);
      const double A0 = ab2(T[j], To[j]), Am1 = ab2(T[j - 1], To[j - 1]);
      const double Am2 = ab2(T[j - 2], To[j - 2]), Ap1 = ab2(T[j + 1], To[j + 1]);
      const double qc = (Am1 - A0) / dc, qu = (A0 - Ap1) / du, qd = (Am2 - Am1) / dd;
      const double Tmean1 = A0 + (2.0 * qc + qu) * (zb - Znz) / 3.0;
      const double Tmean2 = Am1 + (2.0 * qc + qd) * (zb - Zm1) / 3.0;
      gw += -0.5 * (Tmean1 + Tmean2) * area * ghi;
    }
    A.a.gw[oa + base + j] = gw;
  }
}

// contribution of interface j to gA[k] (QR4C on ttfAB)
__device__ __forceinline__ double ga_term(const Inst& in, const DevMesh& m, int64_t base, int j,
                                         int k, int nzmin, int nzmax, double ghi) {
  const double w = in.w_e[base + j], area = m.area[base + j];
  if (j == nzmin) return k == j ? -w * area * ghi : 0.0;
  if (j == nzmin + 1 || j == nzmax - 1)
    return (k == j - 1 || k == j) ? -0.5 * w * area * ghi : 0.0;
  double Znz, Zm1, Zm2, Zp1, zb;
  qr4c_depths(in, m, base, j, Znz, Zm1, Zm2, Zp1, zb);
  const double dc = safe_nz(Zm1 - Znz), du = safe_nz(Znz - Zp1), dd = safe_nz(Zm2 - Zm1);
  const double gS = -0.5 * w * area * ghi;
  const double gq1 = gS * (zb - Znz) / 3.0, gq2 = gS * (zb - Zm1) / 3.0;
  const double gqc = 2.0 * gq1 + 2.0 * gq2, gqu = gq1, gqd = gq2;
  if (k == j) return gS - gqc / dc + gqu / du;
  if (k == j - 1) return gS + gqc / dc - gqd / dd;
  if (k == j - 2) return gqd / dd;
  return -gqu / du;   // k == j + 1
}

__global__ void __launch_bounds__(B) r_vert_b(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_layer) return;
  const uint32_t lane = m.layer_lanes[i];
  const int n = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int nzmin = m.nzmin[n], nzmax = m.nzmax[n];
  const int64_t base = int64_t(n) * L;
  // Wet layers only: the dry entries of gTv / gAv / gw stay zero from the workspace's
  // one-time clear, except level nzmin - 1 (above a cavity's first layer), which the
  // upwind flux of interface nzmin reaches through jm = nzmin - 1; its thread writes it.
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t oa = t * A.a.sN;
    const double* ghi = A.a.gtmax + oa + base;
    const double* gfv = A.a.gtmin + oa + base;
    double gT = 0.0, gA = 0.0;
    {
      const double w = in.w_e[base + k], area = m.area[base + k];
      gT += -0.5 * (w + fabs(w)) * area * gfv[k];
      if (k == 0) gT += -0.5 * (w - fabs(w)) * area * gfv[k];
    }
    if (k + 1 < nzmax) {
      const double w = in.w_e[base + k + 1], area = m.area[base + k + 1];
      gT += -0.5 * (w - fabs(w)) * area * gfv[k + 1];
    }
    // QR4C terms from interfaces k-1 .. k+2 in ascending j (a term that does not reach
    // k is +0.0; gA starts at +0.0, so adding it changes no bit)
    for (int j = k - 1; j <= k + 2; ++j) {
      if (j < nzmin || j >= nzmax) continue;
      gA += ga_term(in, m, base, j, k, nzmin, nzmax, ghi[j]);
    }
    A.a.gTv[oa + base + k] = gT;
    A.a.gAv[oa + base + k] = gA;
    if (k == nzmin && k > 0) {   // dry level above: only the (w - |w|) term of interface k
      const double w = in.w_e[base + k], area = m.area[base + k];
      double g = 0.0;
      g += -0.5 * (w - fabs(w)) * area * gfv[k];
      A.a.gTv[oa + base + k - 1] = g;
    }
  }
}

// --------------- r_final: assemble dT and dT_old (tracer_ab: ttfAB = -0.6 T_old + 1.6 T)
__global__ void __launch_bounds__(B) r_final(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  const int64_t NL = int64_t(m.N) * m.L;
  if (i >= NL) return;
  const int L = m.L;
  const int n = int(i / L), k = int(i - int64_t(n) * L);
  const bool layer = k >= m.nzmin[n] && k < m.nzmax[n];
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t oa = t * A.a.sN;
    const double gv = A.a.gTv[oa + i];
    double gT, gA = A.a.gAv[oa + i];
    if (!layer) {
      gT = A.gTn[t * in.tstride + i] + gv;   // dry levels: T_new = T
    } else {
      gT = A.a.gTp[oa + i] + A.a.gTtr[oa + i] + gv;
      for (int j = m.ne_off[n]; j < m.ne_off[n + 1]; ++j) {
        const int idx = m.ne_idx[j], e = idx >> 1;
        if (!edge_on(m, e, k)) continue;
        const EdgeTerms et = edge_terms(A, t, e, k);
        if (idx & 1) { gT += et.gT2; gA += et.gA2; }
        else { gT += et.gT1; gA += et.gA1; }
      }
    }
    A.gT[t * in.tstride + i] = gT + kAbNew * gA;
    A.gTo[t * in.tstride + i] = kAbOld * gA;
  }
}

// -------------------------- r_uv: edge_vflux transposed, summed over tracers
__global__ void __launch_bounds__(B) r_uv(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  const int L = m.L;
  if (i >= int64_t(m.E) * L) return;
  const int el = int(i / L), k = int(i - int64_t(el) * L);
  double gU = 0.0, gV = 0.0;
  if (elem_on(m, el, k)) {
    const double h = in.helem[i];
    for (int r = 0; r < 3; ++r) {
      const int ent = m.eedge[3 * el + r];
      if (ent < 0) continue;
      const int e = ent >> 1;
      const double* cr = m.cross + 4 * int64_t(e);
      double gvf = 0.0;
      for (int t = 0; t < in.ntr; ++t) gvf += A.a.gvf[t * A.a.sEd + int64_t(e) * L + k];
      if (ent & 1) {   // t2 = (V dx2 - U dy2) h
        gU += -gvf * cr[3] * h;
        gV += gvf * cr[2] * h;
      } else {         // t1 = (U dy1 - V dx1) h
        gU += gvf * cr[1] * h;
        gV += -gvf * cr[0] * h;
      }
    }
  }
  A.guv[2 * i] = gU;
  A.guv[2 * i + 1] = gV;
}

// ---------------------------------------------- r_wsum: dL/dw_e summed over tracers
__global__ void __launch_bounds__(B) r_wsum(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= int64_t(m.N) * m.L) return;
  double g = 0.0;
  for (int t = 0; t < in.ntr; ++t) g += A.a.gw[t * A.a.sN + i];
  A.gw[i] = g;
}

// --------------------------------- compute_w reverse: w = mask * suffix-sum(div) / area
__global__ void __launch_bounds__(128) r_w_div(const DevMesh* __restrict__ mp,
                                               const double* __restrict__ gw,
                                               double* __restrict__ gdiv) {
  const DevMesh& m = *mp;
  const int64_t n = lane_index();
  if (n >= m.N) return;
  const int L = m.L;
  const int64_t base = n * L;
  const int nzmin = m.nzmin[n], nzmax = m.nzmax[n];
  double acc = 0.0;   // gdiv[j] = sum_{k <= j, k interface} gw[k] / area[k]
  for (int k = 0; k < L; ++k) {
    if (k >= nzmin && k <= nzmax) {
      const double a = m.area[base + k];
      acc += gw[base + k] / (a > 0.0 ? a : 1.0);
    }
    gdiv[base + k] = acc;
  }
}

__global__ void __launch_bounds__(B) r_w_uv(const DevMesh* __restrict__ mp,
                                            const double* __restrict__ gdiv,
                                            const double* __restrict__ helem,
                                            double* __restrict__ guv, int accumulate) {
  const DevMesh& m = *mp;
  const int64_t i = lane_index();
  const int L = m.L;
  if (i >= int64_t(m.E) * L) return;
  const int el = int(i / L), k = int(i - int64_t(el) * L);
  double gU = 0.0, gV = 0.0;
  if (elem_on(m, el, k)) {
    const double h = helem[i];
    for (int r = 0; r < 3; ++r) {
      const int ent = m.eedge[3 * el + r];
      if (ent < 0) continue;
      const int e = ent >> 1;
      const double* cr = m.cross + 4 * int64_t(e);
      // c = t1 - t2 is added to div at n1 and subtracted at n2
      const double gc = gdiv[int64_t(m.edges[2 * e]) * L + k] - gdiv[int64_t(m.edges[2 * e + 1]) * L + k];
      if (ent & 1) {   // t2 = (V dx2 - U dy2) h enters c with a minus sign
        gV += -gc * cr[2] * h;
        gU += gc * cr[3] * h;
      } else {         // t1 = (V dx1 - U dy1) h
        gV += gc * cr[0] * h;
        gU += -gc * cr[1] * h;
      }
    }
  }
  if (accumulate) {
    guv[2 * i] += gU;
    guv[2 * i + 1] += gV;
  } else {
    guv[2 * i] = gU;
    guv[2 * i + 1] = gV;
  }
}

}  // namespace

extern "C" {

int fct_plan_reserve_adjoint(FctPlan* P, int max_tracers) {
  if (!P) return set_error(FCT_ERR_INVALID, "plan is NULL");
  if (max_tracers < 1) return set_error(FCT_ERR_INVALID, "max_tracers must be >= 1");
  if (max_tracers <= P->adj_tracers) return FCT_OK;
  int st = plan_reserve_ws(P, max_tracers, /*full=*/true);   // the recompute keeps every field
  if (st) return st;
  FCT_CUDA(cudaSetDevice(P->device));
  const int64_t sN = int64_t(P->N) * P->L, sE = int64_t(P->E) * P->L, sEd = int64_t(P->Ed) * P->L;
  const int64_t nd = int64_t(max_tracers) * (kAdjNodeFields * sN + kAdjEdgeFields * sEd +
                                             kAdjElemFields * sE);
  double* p = nullptr;
  FCT_CUDA(cudaMalloc(&p, size_t(nd) * sizeof(double)));
  // dry-level entries are never written by the reverse kernels and must read as zero
  FCT_CUDA(cudaMemset(p, 0, size_t(nd) * sizeof(double)));
  if (P->d_adj) cudaFree(P->d_adj);
  P->d_adj = p;
  AdjWorkspace& a = P->aws;
  a.sN = sN; a.sE = sE; a.sEd = sEd;
  auto take = [&](int64_t n) { double* q = p; p += n * max_tracers; return q; };
  double** node[] = {&a.gdel, &a.gLOd, &a.gTd, &a.gpf, &a.gmf, &a.gtmax, &a.gtmin, &a.gplus,
                     &a.gminus, &a.gLOl, &a.gtvmax, &a.gtvmin, &a.gLOb, &a.gTb, &a.gdiv,
                     &a.ggnx, &a.ggny, &a.gTp, &a.gTtr, &a.gTv, &a.gAv, &a.gw};
  static_assert(sizeof(node) / sizeof(node[0]) == kAdjNodeFields, "node field count");
  for (double** f : node) *f = take(sN);
  double** edge[] = {&a.gHO, &a.gfl, &a.gvf};
  static_assert(sizeof(edge) / sizeof(edge[0]) == kAdjEdgeFields, "edge field count");
  for (double** f : edge) *f = take(sEd);
  double** elem[] = {&a.gamax, &a.gamin, &a.gtrx, &a.gtry};
  static_assert(sizeof(elem) / sizeof(elem[0]) == kAdjElemFields, "elem field count");
  for (double** f : elem) *f = take(sE);
  P->adj_tracers = max_tracers;
  return FCT_OK;
}

int fct_adjoint(FctPlan* P, const FctFields* f, const double* gT_new, double dt, int ntr,
                const FctGrads* g, fct_stream_t stream) {
  if (!P || !f || !g || !gT_new) return set_error(FCT_ERR_INVALID, "NULL argument");
  if (ntr < 1) return set_error(FCT_ERR_INVALID, "ntr must be >= 1");
  if (ntr > P->adj_tracers || ntr > P->max_tracers)
    return set_error(FCT_ERR_CAPACITY, "ntr=%d exceeds the reserved adjoint workspace (%d); "
                     "call fct_plan_reserve_adjoint first", ntr, P->adj_tracers);
  if (!f->uv || !f->w_e || !f->helem || !f->hnode || !f->hnode_new || !f->T || !f->T_old)
    return set_error(FCT_ERR_INVALID, "a required field pointer is NULL");
  if (!g->gT || !g->gT_old || !g->guv || !g->gw_e)
    return set_error(FCT_ERR_INVALID, "a gradient output pointer is NULL");
  if (f->w_i) return set_error(FCT_ERR_UNSUPPORTED, "the adjoint does not differentiate w_i");
  if ((f->Z3d == nullptr) != (f->zbar3 == nullptr))
    return set_error(FCT_ERR_INVALID, "Z3d and zbar3 must be given together");
  if (!(dt > 0.0)) return set_error(FCT_ERR_INVALID, "dt must be positive");
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != P->device) cudaSetDevice(P->device);
  auto restore = [&](int st) {
    if (prev >= 0 && prev != P->device) cudaSetDevice(prev);
    return st;
  };
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Adj A{};
  Inst& in = A.in;
  in.m = P->d_mesh;
  in.uv = f->uv; in.w_e = f->w_e; in.helem = f->helem;
  in.hnode = f->hnode; in.hnode_new = f->hnode_new;
  in.T = f->T; in.T_old = f->T_old;
  in.T_new = nullptr;
  in.tstride = f->tracer_stride ? f->tracer_stride : int64_t(P->N) * P->L;
  in.tg = 0;
  in.wtg = ntr;
  in.Z3d = f->Z3d; in.zbar3 = f->zbar3; in.w_i = nullptr;
  in.ws = P->ws;
  in.dt = dt;
  in.ntr = ntr;
  A.a = P->aws;
  A.gTn = gT_new;
  A.gT = g->gT; A.gTo = g->gT_old; A.guv = g->guv; A.gw = g->gw_e;
  // forward recomputation: every stage except the final update (T_new is not needed)
  LaunchDims d{};
  d.max_iface = P->hm.n_iface; d.max_layer = P->hm.n_layer; d.max_edge = P->hm.n_edge;
  d.max_elem = P->hm.n_elem; d.max_dense = int64_t(P->N) * P->L; d.max_nodes = P->N;
  d.ntr = ntr; d.chunk = 0; d.per_thread = 8; d.any_wi = false; d.copy_dry = false;
  d.fused = false;   // the reverse kernels read every stage's intermediates
  int st = launch_forward_stages(in, d, s, /*through_factors=*/true);
  if (st) return restore(st);
  auto grid = [](int64_t lanes, int b) {
    return dim3(unsigned(std::max<int64_t>(1, (lanes + b - 1) / b)));
  };
  const DevMesh& hm = P->hm;
  r_seed<<<grid(hm.n_layer, B), B, 0, s>>>(A);
  r_factors<<<grid(hm.n_layer, B), B, 0, s>>>(A);
  r_ratio<<<grid(hm.n_layer, B), B, 0, s>>>(A);
  r_window<<<grid(hm.n_layer, B), B, 0, s>>>(A);
  r_cluster<<<grid(hm.n_elem, B), B, 0, s>>>(A);
  r_bounds<<<grid(hm.n_layer, B), B, 0, s>>>(A);
  r_lo<<<grid(hm.n_layer, B), B, 0, s>>>(A);
  r_edge<<<grid(hm.n_edge, B), B, 0, s>>>(A);
  r_gnode<<<grid(hm.n_layer, B), B, 0, s>>>(A);
  r_tr<<<grid(hm.n_elem, B), B, 0, s>>>(A);
  r_grad_t<<<grid(hm.n_layer, B), B, 0, s>>>(A);
  r_vert_a<<<grid(hm.n_layer, B), B, 0, s>>>(A);
  r_vert_b<<<grid(hm.n_layer, B), B, 0, s>>>(A);
  r_final<<<grid(int64_t(P->N) * P->L, B), B, 0, s>>>(A);
  r_uv<<<grid(int64_t(P->E) * P->L, B), B, 0, s>>>(A);
  r_wsum<<<grid(int64_t(P->N) * P->L, B), B, 0, s>>>(A);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return restore(cuda_error(e, "adjoint kernel launch"));
  return restore(FCT_OK);
}

int fct_compute_w_adjoint(FctPlan* P, const double* gw, const double* helem, double* guv,
                          int accumulate, fct_stream_t stream) {
  if (!P || !gw || !helem || !guv) return set_error(FCT_ERR_INVALID, "NULL argument");
  if (P->adj_tracers < 1)
    return set_error(FCT_ERR_CAPACITY, "call fct_plan_reserve_adjoint first");
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != P->device) cudaSetDevice(P->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* gdiv = P->aws.gdiv;   // scratch: one node field
  r_w_div<<<unsigned((P->N + 127) / 128), 128, 0, s>>>(P->d_mesh, gw, gdiv);
  const int64_t EL = int64_t(P->E) * P->L;
  r_w_uv<<<unsigned((EL + B - 1) / B), B, 0, s>>>(P->d_mesh, gdiv, helem, guv, accumulate);
  const cudaError_t e = cudaGetLastError();
  if (prev >= 0 && prev != P->device) cudaSetDevice(prev);
  return e == cudaSuccess ? FCT_OK : cuda_error(e, "compute_w adjoint launch");
}

}  // extern "C"
