// FCT forward kernels (sm_100a, FP64): fesom_jax/tracer_adv.py:532-578 split into
// stage kernels over wet-lane lists. Every edge->node or element->node reduction is a
// deterministic gather over a CSR list in ascending edge/element id, so results are
// bit-identical run to run (no atomics).
//
// Stage map (reference function -> kernel):
//   edge_vflux (tracer_adv.py:69-93)                         -> k_vflux      (edge lanes)
//   tracer_gradient_elements (:316-326)                      -> k_elem_grad  (element lanes)
//   adv_flux_hor/adv_flux_ver (:96-120), compute_fct_lo (:298-313),
//   _node_avg_grad (:329-341), adv_flux_ver_ho (:241-295)    -> k_node_lo    (interface lanes)
//   adv_tra_vert_impl (:487-529), w_split only               -> k_vert_impl  (node columns)
//   fill_up_dn_grad (:344-368), adv_flux_hor_ho (:196-225)   -> k_edge_adf   (edge lanes)
//   zalesak_limit a2 (:393-397)                              -> k_elem_bounds(element lanes)
//   zalesak_limit a3 (:399-405)                              -> k_node_cluster (layer lanes)
//   zalesak_limit a4, b1, b2 (:407-451)                      -> k_node_factors (layer lanes)
//   zalesak_limit b3 (:453-465), flux2dtracer_fct (:469-484),
//   ale_reconstruct (:142-151)                               -> k_node_final (layer lanes)
//   invalid lanes keep T (ale_reconstruct)                   -> k_copy_dry   (dense)
#include <algorithm>

#include "fct_host.h"

namespace fct {

namespace {

__device__ __forceinline__ double ab2(double T, double To) { return kAbOld * To + kAbNew * T; }
__device__ __forceinline__ double safe_nz(double x) { return x == 0.0 ? 1.0 : x; }

__device__ __forceinline__ int64_t lane_index() {
  return int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
}

// ---------------------------------------------------------------- edge_vflux
__device__ __forceinline__ void body_vflux(const Inst& in, int64_t i) {
  const DevMesh& m = *in.m;
  if (i >= m.n_edge) return;
  const uint32_t lane = m.edge_lanes[i];
  const int e = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int el1 = m.etri[2 * e], el2 = m.etri[2 * e + 1];
  const double* cr = m.cross + 4 * int64_t(e);
  double t1 = 0.0, t2 = 0.0;
  if (k >= m.eul[el1] && k < m.enl[el1]) {
    const int64_t q = int64_t(el1) * L + k;
    const double U = in.uv[2 * q], V = in.uv[2 * q + 1];
    t1 = (U * cr[1] - V * cr[0]) * in.helem[q];
  }
  if (el2 >= 0 && k >= m.eul[el2] && k < m.enl[el2]) {
    const int64_t q = int64_t(el2) * L + k;
    const double U = in.uv[2 * q], V = in.uv[2 * q + 1];
    t2 = (V * cr[2] - U * cr[3]) * in.helem[q];
  }
  in.ws.vflux[int64_t(e) * L + k] = t1 + t2;
}

// ---------------------------------------------------- tracer_gradient_elements
__device__ __forceinline__ void body_elem_grad(const Inst& in, int64_t i) {
  const DevMesh& m = *in.m;
  if (i >= m.n_elem) return;
  const uint32_t lane = m.elem_lanes[i];
  const int e = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int v0 = m.enodes[3 * e], v1 = m.enodes[3 * e + 1], v2 = m.enodes[3 * e + 2];
  const double* g = m.gsca + 6 * int64_t(e);
  const double g0 = g[0], g1 = g[1], g2 = g[2], g3 = g[3], g4 = g[4], g5 = g[5];
  const int64_t q = int64_t(e) * L + k;
  for (int t = 0; t < in.ntr; ++t) {
    const double* T = in.T + t * in.tstride;
    const double t0 = T[int64_t(v0) * L + k], t1 = T[int64_t(v1) * L + k],
                 t2 = T[int64_t(v2) * L + k];
    in.ws.gx[t * in.ws.sE + q] = g0 * t0 + g1 * t1 + g2 * t2;
    in.ws.gy[t * in.ws.sE + q] = g3 * t0 + g4 * t1 + g5 * t2;
  }
}

// Upwind vertical flux at interface j of a column (layer-masked), tracer_adv.py:108-120.
__device__ __forceinline__ double vflux_up(const double* col, const double* area_col,
                                           double w, int j, bool layer) {
  if (!layer) return 0.0;
  const double aw = fabs(w);
  const double Tb = col[j], Ta = col[j > 0 ? j - 1 : 0];
  return -0.5 * (Tb * (w + aw) + Ta * (w - aw)) * area_col[j];
}

// -------------------------------- LO solution, node-average gradient, adf_v
__device__ __forceinline__ void body_node_lo(const Inst& in, int64_t i) {
  const DevMesh& m = *in.m;
  if (i >= m.n_iface) return;
  const uint32_t lane = m.iface_lanes[i];
  const int n = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int nzmin = m.nzmin[n], nzmax = m.nzmax[n];
  const int64_t base = int64_t(n) * L;
  const bool layer = k < nzmax;
  const bool layer1 = (k + 1) < nzmax;
  const double* area_col = m.area + base;
  const double w = in.w_e[base + k];
  const double w1 = layer1 ? in.w_e[base + k + 1] : 0.0;
  const double Wf = in.w_i ? w + in.w_i[base + k] : w;   // w_full for the HO flux
  const double area_k = area_col[k];
  const double hn = in.hnode[base + k], hnn = in.hnode_new[base + k];
  const double av = m.areasvol[base + k];
  const double dt = in.dt;
  const int e0 = m.ne_off[n], e1 = m.ne_off[n + 1];
  const int c0 = m.nel_off[n], c1 = m.nel_off[n + 1];

  // QR4C stencil depths (tracer_adv.py:228-238, 265-273)
  double Znz, Zm1, Zm2, Zp1, zb;
  if (in.Z3d) {
    const double* Zc = in.Z3d + base;
    Znz = Zc[k]; Zm1 = Zc[k > 0 ? k - 1 : 0]; Zm2 = Zc[k > 1 ? k - 2 : 0];
    Zp1 = Zc[k + 1 < L ? k + 1 : L - 1]; zb = in.zbar3[base + k];
  } else {
    Znz = m.Zp[k]; Zm1 = m.Zp[k > 0 ? k - 1 : 0]; Zm2 = m.Zp[k > 1 ? k - 2 : 0];
    Zp1 = m.Zp[k + 1 < L ? k + 1 : L - 1]; zb = m.zbar[k];
  }

  for (int t = 0; t < in.ntr; ++t) {
    const double* T = in.T + t * in.tstride;
    const double* To = in.T_old + t * in.tstride;
    const double* Tc = T + base;
    const double fvk = vflux_up(Tc, area_col, w, k, layer);
    if (layer) {
      const double fvk1 = vflux_up(Tc, area_col, w1, k + 1, layer1);
      // compute_fct_lo: edge->node upwind divergence, ascending edge id
      double div_h = 0.0;
      for (int j = e0; j < e1; ++j) {
        const int idx = m.ne_idx[j];
        const int e = idx >> 1;
        const double vf = (k >= m.ekmin[e] && k < m.ekmax[e]) ? in.ws.vflux[int64_t(e) * L + k] : 0.0;
        const double avf = fabs(vf);
        const int n1 = m.edges[2 * e], n2 = m.edges[2 * e + 1];
        const double fl = -0.5 * (T[int64_t(n1) * L + k] * (vf + avf) +
                                  T[int64_t(n2) * L + k] * (vf - avf));
        div_h += (idx & 1) ? -fl : fl;
      }
      const bool valid = (hnn > 0.0) && (av > 0.0);
      const double lo = valid ? (Tc[k] * hn + (div_h + (fvk - fvk1)) * dt / av) / hnn : 0.0;
      in.ws.lo[t * in.ws.sN + base + k] = lo;
      // _node_avg_grad: area-weighted mean over the node's active elements
      double nx = 0.0, ny = 0.0, den = 0.0;
      for (int j = c0; j < c1; ++j) {
        const int el = m.nel_idx[j];
        if (k >= m.eul[el] && k < m.enl[el]) {
          const double a = m.earea[el];
          const int64_t q = t * in.ws.sE + int64_t(el) * L + k;
          nx += in.ws.gx[q] * a;
          ny += in.ws.gy[q] * a;
          den += a;
        }
      }
      const double dd = den > 0.0 ? den : 1.0;
      in.ws.gnx[t * in.ws.sN + base + k] = nx / dd;
      in.ws.gny[t * in.ws.sN + base + k] = ny / dd;
    }
    // adv_flux_ver_ho (QR4C on ttfAB) minus the LO vertical flux
    double hi = 0.0;
    if (k == nzmin) {
      hi = -ab2(Tc[k], To[base + k]) * Wf * area_k;
    } else if (k == nzmax) {
      hi = 0.0;
    } else if (k == nzmin + 1 || k == nzmax - 1) {
      const double A0 = ab2(Tc[k], To[base + k]), Am1 = ab2(Tc[k - 1], To[base + k - 1]);
      hi = -0.5 * (Am1 + A0) * Wf * area_k;
    } else if (k >= nzmin + 2 && k <= nzmax - 2) {
      const double A0 = ab2(Tc[k], To[base + k]);
      const double Am1 = ab2(Tc[k - 1], To[base + k - 1]);
      const double Am2 = ab2(Tc[k - 2], To[base + k - 2]);
      const double Ap1 = ab2(Tc[k + 1], To[base + k + 1]);
      const double qc = (Am1 - A0) / safe_nz(Zm1 - Znz);
      const double qu = (A0 - Ap1) / safe_nz(Znz - Zp1);
      const double qd = (Am2 - Am1) / safe_nz(Zm2 - Zm1);
      const double Tmean1 = A0 + (2.0 * qc + qu) * (zb - Znz) / 3.0;
      const double Tmean2 = Am1 + (2.0 * qc + qd) * (zb - Zm1) / 3.0;
      hi = -0.5 * (Tmean1 + Tmean2) * Wf * area_k;
    }
    const double lo_v = in.w_i ? vflux_up(Tc, area_col, Wf, k, layer) : fvk;
    in.ws.adfv[t * in.ws.sN + base + k] = hi - lo_v;
  }
}

// ---------------------------- adv_tra_vert_impl: implicit w_i advection of LO
__device__ __forceinline__ void body_vert_impl(const Inst& in, int64_t n) {
  const DevMesh& m = *in.m;
  if (n >= m.N || !in.w_i) return;
  const int L = m.L;
  const int nzmin = m.nzmin[n], nzmax = m.nzmax[n];
  if (nzmax <= nzmin) return;
  const int64_t base = n * L;
  const double dt = in.dt;
  double cp[kMaxLevels], dp[kMaxLevels];
  for (int t = 0; t < in.ntr; ++t) {
    double* lo = in.ws.lo + t * in.ws.sN + base;
    double cprev = 0.0, dprev = 0.0;
    for (int k = nzmin; k < nzmax; ++k) {
      const double av = m.areasvol[base + k];
      const double sa = av > 0.0 ? av : 1.0;
      const double v_top = dt * m.area[base + k] / sa;
      const double v_bot = dt * (k + 1 < L ? m.area[base + k + 1] : 0.0) / sa;
      const double wu = in.w_i[base + k];
      const double wd = k + 1 < L ? in.w_i[base + k + 1] : 0.0;
      const bool surf = (k == nzmin), bot = (k == nzmax - 1);
      const double a = (surf ? 0.0 : fmin(0.0, wu)) * v_top;
      const double b_top = (surf ? wu : fmax(0.0, wu)) * v_top;
      const double b_bot = (bot ? 0.0 : -fmin(0.0, wd)) * v_bot;
      const double c = (bot ? 0.0 : -fmax(0.0, wd)) * v_bot;
      const double b_adv = b_top + b_bot;
      const double b = in.hnode_new[base + k] + b_adv;
      const double Tm = lo[k > 0 ? k - 1 : 0], T0 = lo[k], Tp = k + 1 < L ? lo[k + 1] : 0.0;
      const double rhs = -(a * Tm + b_adv * T0 + c * Tp);
      const double md = b - a * cprev;
      cprev = c / md;
      dprev = (rhs - a * dprev) / md;
      cp[k] = cprev;
      dp[k] = dprev;
    }
    double x = 0.0;
    for (int k = nzmax - 1; k >= nzmin; --k) {
      x = dp[k] - cp[k] * x;
      dp[k] = x;
    }
    for (int k = nzmin; k < nzmax; ++k) lo[k] = lo[k] + dp[k];
  }
}

// -------------------------- fill_up_dn_grad + adv_flux_hor_ho - LO flux = adf_h
__device__ __forceinline__ void body_edge_adf(const Inst& in, int64_t i) {
  const DevMesh& m = *in.m;
  if (i >= m.n_edge) return;
  const uint32_t lane = m.edge_lanes[i];
  const int e = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int n1 = m.edges[2 * e], n2 = m.edges[2 * e + 1];
  const int up = m.eupdn[2 * e], dn = m.eupdn[2 * e + 1];
  const int kmin = max(m.ulmax[n1], m.ulmax[n2]) - 1;
  const int kmax = min(m.nlmin[n1], m.nlmin[n2]) - 1;
  const bool use_tri = (up >= 0) && (dn >= 0) && k >= kmin && k < kmax;
  const double vf = in.ws.vflux[int64_t(e) * L + k];
  const double avf = fabs(vf);
  const double c1 = m.ecoef[2 * e], c2 = m.ecoef[2 * e + 1];
  const int64_t q1 = int64_t(n1) * L + k, q2 = int64_t(n2) * L + k;
  for (int t = 0; t < in.ntr; ++t) {
    const double* T = in.T + t * in.tstride;
    const double* To = in.T_old + t * in.tstride;
    const double T1 = T[q1], T2 = T[q2];
    const double fl = -0.5 * (T1 * (vf + avf) + T2 * (vf - avf));
    double g0, g1, g2, g3;
    if (use_tri) {
      const int64_t qu = t * in.ws.sE + int64_t(up) * L + k;
      const int64_t qd = t * in.ws.sE + int64_t(dn) * L + k;
      g0 = in.ws.gx[qu]; g1 = in.ws.gx[qd]; g2 = in.ws.gy[qu]; g3 = in.ws.gy[qd];
    } else {
      const int64_t o = t * in.ws.sN;
      g0 = in.ws.gnx[o + q1]; g1 = in.ws.gnx[o + q2]; g2 = in.ws.gny[o + q1]; g3 = in.ws.gny[o + q2];
    }
    const double A1 = ab2(T1, To[q1]), A2 = ab2(T2, To[q2]);
    const double diff = A2 - A1;
    const double Tm1 = A1 + (2.0 * diff + c1 * g0 + c2 * g2) / 6.0;
    const double Tm2 = A2 - (2.0 * diff + c1 * g1 + c2 * g3) / 6.0;
    const double ho = -0.5 * ((vf + avf) * Tm1 + (vf - avf) * Tm2);
    in.ws.adfh[t * in.ws.sEd + int64_t(e) * L + k] = ho - fl;
  }
}

// ------------------------ zalesak a2: element max/min of the LO/T window
__device__ __forceinline__ void body_elem_bounds(const Inst& in, int64_t i) {
  const DevMesh& m = *in.m;
  if (i >= m.n_elem) return;
  const uint32_t lane = m.elem_lanes[i];
  const int e = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int64_t q0 = int64_t(m.enodes[3 * e]) * L + k, q1 = int64_t(m.enodes[3 * e + 1]) * L + k,
                q2 = int64_t(m.enodes[3 * e + 2]) * L + k;
  const int64_t qe = int64_t(e) * L + k;
  for (int t = 0; t < in.ntr; ++t) {
    const double* T = in.T + t * in.tstride;
    const double* lo = in.ws.lo + t * in.ws.sN;
    const double a0 = lo[q0], a1 = lo[q1], a2 = lo[q2];
    const double b0 = T[q0], b1 = T[q1], b2 = T[q2];
    in.ws.amax[t * in.ws.sE + qe] = fmax(fmax(fmax(a0, b0), fmax(a1, b1)), fmax(a2, b2));
    in.ws.amin[t * in.ws.sE + qe] = fmin(fmin(fmin(a0, b0), fmin(a1, b1)), fmin(a2, b2));
  }
}

// ------------------------ zalesak a3: node cluster max/min over elements
__device__ __forceinline__ void body_node_cluster(const Inst& in, int64_t i) {
  const DevMesh& m = *in.m;
  if (i >= m.n_layer) return;
  const uint32_t lane = m.layer_lanes[i];
  const int n = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int c0 = m.nel_off[n], c1 = m.nel_off[n + 1];
  const int64_t qn = int64_t(n) * L + k;
  for (int t = 0; t < in.ntr; ++t) {
    double mx = -INFINITY, mn = INFINITY;
    for (int j = c0; j < c1; ++j) {
      const int el = m.nel_idx[j];
      if (k >= m.eul[el] && k < m.enl[el]) {
        const int64_t q = t * in.ws.sE + int64_t(el) * L + k;
        mx = fmax(mx, in.ws.amax[q]);
        mn = fmin(mn, in.ws.amin[q]);
      } else {   // a cell without this level pads with -+BIG (tracer_adv.py:396-397)
        mx = fmax(mx, -kBig);
        mn = fmin(mn, kBig);
      }
    }
    in.ws.tvmax[t * in.ws.sN + qn] = mx;
    in.ws.tvmin[t * in.ws.sN + qn] = mn;
  }
}

// ------------------- zalesak a4 + b1 + b2: admissible window, sums, factors
__device__ __forceinline__ void body_node_factors(const Inst& in, int64_t i) {
  const DevMesh& m = *in.m;
  if (i >= m.n_layer) return;
  const uint32_t lane = m.layer_lanes[i];
  const int n = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int nzmin = m.nzmin[n], nzmax = m.nzmax[n];
  const int64_t base = int64_t(n) * L, qn = base + k;
  const bool use_own = (k == nzmin) || (k == nzmax - 1);
  const double av = m.areasvol[qn], hnn = in.hnode_new[qn];
  const bool valid = (av > 0.0) && (hnn > 0.0);
  const double sa = av > 0.0 ? av : 1.0, sh = hnn > 0.0 ? hnn : 1.0;
  const double dt = in.dt;
  const int e0 = m.ne_off[n], e1 = m.ne_off[n + 1];
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t o = t * in.ws.sN;
    const double* tvmax = in.ws.tvmax + o + base;
    const double* tvmin = in.ws.tvmin + o + base;
    double tmax, tmin;
    if (use_own) {
      tmax = tvmax[k];
      tmin = tvmin[k];
    } else {
      const int km = k > 0 ? k - 1 : 0;
      const double up_max = k + 1 < L ? tvmax[k + 1] : 0.0;
      const double up_min = k + 1 < L ? tvmin[k + 1] : 0.0;
      tmax = fmax(fmax(tvmax[km], tvmax[k]), up_max);
      tmin = fmin(fmin(tvmin[km], tvmin[k]), up_min);
    }
    const double lo = in.ws.lo[o + qn];
    const double fmax_w = tmax - lo, fmin_w = tmin - lo;
    const double* adfv = in.ws.adfv + o + base;
    const double fvt = adfv[k], fvb = k + 1 < L ? adfv[k + 1] : 0.0;
    const double pos_v = fmax(fvt, 0.0) + fmax(-fvb, 0.0);
    const double neg_v = fmin(fvt, 0.0) + fmin(-fvb, 0.0);
    double sp = 0.0, sm = 0.0;
    for (int j = e0; j < e1; ++j) {
      const int idx = m.ne_idx[j], e = idx >> 1;
      if (k < m.ekmin[e] || k >= m.ekmax[e]) continue;   // no flux on this level
      const double a = in.ws.adfh[t * in.ws.sEd + int64_t(e) * L + k];
      const double s = (idx & 1) ? -a : a;
      sp += fmax(s, 0.0);
      sm += fmin(s, 0.0);
    }
    const double plus = pos_v + sp, minus = neg_v + sm;
    double pf = 1.0, mf = 1.0;
    if (valid) {
      const double flux_pos = plus * dt / sa / sh + kFluxEps;
      const double flux_neg = minus * dt / sa / sh - kFluxEps;
      pf = fmin(1.0, fmax_w / flux_pos);
      mf = fmin(1.0, fmin_w / flux_neg);
    }
    in.ws.pf[o + qn] = pf;
    in.ws.mf[o + qn] = mf;
  }
}

// Limited vertical antidiffusive flux at interface j (tracer_adv.py:453-459).
__device__ __forceinline__ double adfv_lim(const double* adfv, const double* pf,
                                           const double* mf, int j, int nzmin, int nzmax) {
  if (j >= nzmax && j != nzmin) return 0.0;   // adf_v[nzmax] == 0 by construction
  const double f = adfv[j];
  double ae;
  if (j == nzmin) {
    ae = f >= 0.0 ? pf[j] : mf[j];
  } else {
    ae = f >= 0.0 ? fmin(mf[j - 1], pf[j]) : fmin(pf[j - 1], mf[j]);
  }
  return ae * f;
}

// ---------- zalesak b3 + flux2dtracer_fct + ale_reconstruct: T_new on layers
__device__ __forceinline__ void body_node_final(const Inst& in, int64_t i) {
  const DevMesh& m = *in.m;
  if (i >= m.n_layer) return;
  const uint32_t lane = m.layer_lanes[i];
  const int n = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int nzmin = m.nzmin[n], nzmax = m.nzmax[n];
  const int64_t base = int64_t(n) * L, qn = base + k;
  const double av = m.areasvol[qn];
  const double sa = av > 0.0 ? av : 1.0;
  const double hn = in.hnode[qn], hnn = in.hnode_new[qn];
  const double dt = in.dt;
  const int e0 = m.ne_off[n], e1 = m.ne_off[n + 1];
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t o = t * in.ws.sN;
    const double* pf = in.ws.pf + o;
    const double* mf = in.ws.mf + o;
    const double* adfv = in.ws.adfv + o + base;
    const double vt = adfv_lim(adfv, pf + base, mf + base, k, nzmin, nzmax);
    const double vb = adfv_lim(adfv, pf + base, mf + base, k + 1, nzmin, nzmax);
    double hsc = 0.0;
    for (int j = e0; j < e1; ++j) {
      const int idx = m.ne_idx[j];
      const int e = idx >> 1;
      if (k < m.ekmin[e] || k >= m.ekmax[e]) continue;   // no flux on this level
      const double a = in.ws.adfh[t * in.ws.sEd + int64_t(e) * L + k];
      const int64_t p1 = int64_t(m.edges[2 * e]) * L + k, p2 = int64_t(m.edges[2 * e + 1]) * L + k;
      const double ae = a >= 0.0 ? fmin(pf[p1], mf[p2]) : fmin(mf[p1], pf[p2]);
      const double lim = ae * a;
      hsc += (idx & 1) ? -lim : lim;
    }
    const double T = in.T[t * in.tstride + qn];
    const double lo = in.ws.lo[o + qn];
    const double lo_trans = -T * hn + lo * hnn;
    const double vdiv = av > 0.0 ? (vt - vb) * dt / sa : 0.0;
    double d = hsc * dt / sa + (lo_trans + vdiv);
    d = d + T * (hn - hnn);
    in.T_new[t * in.tstride + qn] = T + (hnn > 0.0 ? d / hnn : 0.0);
  }
}

// ------------------------------------------- dry levels keep T (ale_reconstruct)
__device__ __forceinline__ void body_copy_dry(const Inst& in, int64_t i) {
  const DevMesh& m = *in.m;
  const int64_t NL = int64_t(m.N) * m.L;
  if (i >= NL) return;
  const int n = int(i / m.L), k = int(i - int64_t(n) * m.L);
  if (k >= m.nzmin[n] && k < m.nzmax[n]) return;
  for (int t = 0; t < in.ntr; ++t) in.T_new[t * in.tstride + i] = in.T[t * in.tstride + i];
}

#define FCT_KERNEL_PAIR(name, body)                                               \
  __global__ void __launch_bounds__(256) name##_1(Inst in) { body(in, lane_index()); } \
  __global__ void __launch_bounds__(256) name##_n(const Inst* __restrict__ tab) {  \
    body(tab[blockIdx.y], lane_index());                                          \
  }

FCT_KERNEL_PAIR(k_vflux, body_vflux)
FCT_KERNEL_PAIR(k_elem_grad, body_elem_grad)
FCT_KERNEL_PAIR(k_node_lo, body_node_lo)
FCT_KERNEL_PAIR(k_vert_impl, body_vert_impl)
FCT_KERNEL_PAIR(k_edge_adf, body_edge_adf)
FCT_KERNEL_PAIR(k_elem_bounds, body_elem_bounds)
FCT_KERNEL_PAIR(k_node_cluster, body_node_cluster)
FCT_KERNEL_PAIR(k_node_factors, body_node_factors)
FCT_KERNEL_PAIR(k_node_final, body_node_final)
FCT_KERNEL_PAIR(k_copy_dry, body_copy_dry)

}  // namespace

const char* const kStageNames[kNumStages] = {
    "vflux", "elem_grad", "node_lo", "vert_impl", "edge_adf", "elem_bounds",
    "node_cluster", "node_factors", "node_final", "copy_dry"};

int launch_forward_events(const Inst& single, const Inst* tab, int n, const LaunchDims& d,
                          cudaStream_t s, cudaEvent_t* after) {
  constexpr int B = 256;
  auto grid = [&](int64_t lanes) {
    return dim3(unsigned(std::max<int64_t>(1, (lanes + B - 1) / B)), unsigned(n), 1);
  };
  int stage = 0;
  auto mark = [&]() {
    if (after) cudaEventRecord(after[stage], s);
    ++stage;
  };
#define FCT_LAUNCH(name, lanes, enabled)                            \
  do {                                                              \
    if (enabled) {                                                  \
      if (tab) name##_n<<<grid(lanes), B, 0, s>>>(tab);             \
      else name##_1<<<grid(lanes), B, 0, s>>>(single);              \
    }                                                               \
    mark();                                                         \
  } while (0)
  FCT_LAUNCH(k_vflux, d.max_edge, true);
  FCT_LAUNCH(k_elem_grad, d.max_elem, true);
  FCT_LAUNCH(k_node_lo, d.max_iface, true);
  FCT_LAUNCH(k_vert_impl, d.max_nodes, d.any_wi);
  FCT_LAUNCH(k_edge_adf, d.max_edge, true);
  FCT_LAUNCH(k_elem_bounds, d.max_elem, true);
  FCT_LAUNCH(k_node_cluster, d.max_layer, true);
  FCT_LAUNCH(k_node_factors, d.max_layer, true);
  FCT_LAUNCH(k_node_final, d.max_layer, true);
  FCT_LAUNCH(k_copy_dry, d.max_dense, d.copy_dry);
#undef FCT_LAUNCH
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "forward kernel launch");
  return FCT_OK;
}

int launch_forward(const Inst& single, const Inst* tab, int n, const LaunchDims& d,
                   cudaStream_t s) {
  return launch_forward_events(single, tab, n, d, s, nullptr);
}

int launch_copy_dry(const Inst* tab, int n, int64_t max_dense, cudaStream_t s) {
  const dim3 g(unsigned(std::max<int64_t>(1, (max_dense + 255) / 256)), unsigned(n), 1);
  k_copy_dry_n<<<g, 256, 0, s>>>(tab);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FCT_OK : cuda_error(e, "copy_dry launch");
}

}  // namespace fct
