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
//   invalid lanes keep T (ale_reconstruct)                   -> k_copy_dry   (dry lanes)
//
// Each thread owns one lane and NTR tracers (a compile-time chunk of the instance's
// tracers, which share its velocities): mesh indices, geometry and velocity terms are
// loaded once per lane and every neighbour gather issues NTR independent loads (one
// contiguous chunk in the interleaved layout), so the gathers overlap.
#include <algorithm>

#include "fct_device.cuh"

namespace fct {

namespace {

// ---------------------------------------------------------------- edge_vflux
__device__ __forceinline__ void body_vflux(const Inst& in, int64_t i) {
  const DevMesh& m = *in.m;
  if (i >= m.n_edge) return;
  const uint32_t lane = ld(m.edge_lanes + i);
  const int e = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const int4 ec = __ldg(m.ecell4 + e);   // cells and their layer ranges in one load
  const unsigned tr = unsigned(ec.z);
  const double* cr = m.cross + 4 * int64_t(e);
  double t1 = 0.0, t2 = 0.0;
  if (in_range(k, tr & 0xffffu)) {
    const uint32_t q = lq(ec.x, L, k);
    const double2 U = __ldg(reinterpret_cast<const double2*>(in.uv) + q);
    t1 = (U.x * ld(cr + 1) - U.y * ld(cr + 0)) * ld(in.helem + q);
  }
  if (((tr >> 16) & 255u) != kNoCell && in_range(k, tr >> 16)) {
    const uint32_t q = lq(ec.y, L, k);
    const double2 U = __ldg(reinterpret_cast<const double2*>(in.uv) + q);
    t2 = (U.y * ld(cr + 2) - U.x * ld(cr + 3)) * ld(in.helem + q);
  }
  in.ws.vflux[lq(e, L, k)] = t1 + t2;
}

template <int NTR, bool IL>
__device__ __forceinline__ void body_elem_grad(const Inst& in, int64_t i, int t0, int w0) {
  const DevMesh& m = *in.m;
  if (i >= m.n_elem) return;
  const uint32_t lane = ld(m.elem_lanes + i);
  const int e = lane_ent(lane), k = lane_lev(lane), L = m.L;
  double gx[NTR], gy[NTR];
  cell_grad<NTR, IL>(in, e, k, t0, gx, gy);
  const uint32_t q = lq(e, L, k);
  stn<NTR, IL>(in.ws.gx, q, w0, in.ws.sE, in.wtg, gx);
  stn<NTR, IL>(in.ws.gy, q, w0, in.ws.sE, in.wtg, gy);
}

// -------------------------------- LO solution, node-average gradient, adf_v
template <int NTR, bool IL>
__device__ __forceinline__ void body_node_lo(const Inst& in, int64_t i, int t0, int w0) {
  const DevMesh& m = *in.m;
  if (i >= m.n_iface) return;
  const int4 rec = __ldg(m.iface4 + i);
  const unsigned pk = unsigned(rec.w);
  const int n = lane_ent(uint32_t(rec.x)), k = lane_lev(uint32_t(rec.x)), L = m.L;
  const int nzmin = int(pk & 255u), nzmax = int((pk >> 8) & 255u);
  const uint32_t base = lq(n, L, 0), qn = base + uint32_t(k);
  const bool layer = k < nzmax;
  const bool layer1 = (k + 1) < nzmax;
  const int km1 = k > 0 ? k - 1 : 0;
  const double w = ld(in.w_e + qn);
  const double Wf = in.w_i ? w + ld(in.w_i + qn) : w;   // w_full for the HO flux
  const double area_k = ld(m.area + qn);
  const int64_t ts = in.tstride;
  const int tg = in.tg;

  double Tc[NTR], Ta[NTR];   // T[k], T[k-1]
  ldn<NTR, IL>(in.T, qn, t0, ts, tg, Tc);
  ldn<NTR, IL>(in.T, base + km1, t0, ts, tg, Ta);
  double fvk[NTR];
#pragma unroll
  for (int t = 0; t < NTR; ++t) fvk[t] = layer ? vflux_up(Tc[t], Ta[t], w, area_k) : 0.0;

  if (layer) {
    const double hn = ld(in.hnode + qn), hnn = ld(in.hnode_new + qn);
    const double av = ld(m.areasvol + qn);
    const Rcp rav = rcp(av), rhn = rcp(hnn);   // shared by the NTR quotients below
    const double dt = in.dt;
    double fvk1[NTR];
    if (layer1) {
      const double w1 = ld(in.w_e + qn + 1), area1 = ld(m.area + qn + 1);
      double Tb[NTR];
      ldn<NTR, IL>(in.T, qn + 1, t0, ts, tg, Tb);
#pragma unroll
      for (int t = 0; t < NTR; ++t) fvk1[t] = vflux_up(Tb[t], Tc[t], w1, area1);
    } else {
#pragma unroll
      for (int t = 0; t < NTR; ++t) fvk1[t] = 0.0;
    }
    // compute_fct_lo: edge->node upwind divergence in ascending edge id
    double div[NTR];
#pragma unroll
    for (int t = 0; t < NTR; ++t) div[t] = 0.0;
    const int e0 = rec.y, e1 = rec.y + int((pk >> 16) & 255u);
    for (int j = e0; j < e1; ++j) {
      const int idx = ld(m.ne_idx + j), e = idx >> 1;
      if (k < ld(m.ekmin + e) || k >= ld(m.ekmax + e)) continue;   // vflux == 0 there
      const int oth = ld(m.ne_oth + j);
      const double vf = ld(in.ws.vflux + lq(e, L, k));
      const double avf = fabs(vf);
      double To[NTR];
      ldn<NTR, IL>(in.T, lq(oth, L, k), t0, ts, tg, To);
#pragma unroll
      for (int t = 0; t < NTR; ++t) {
        const double T1 = (idx & 1) ? To[t] : Tc[t], T2 = (idx & 1) ? Tc[t] : To[t];
        const double fl = -0.5 * (T1 * (vf + avf) + T2 * (vf - avf));
        div[t] += (idx & 1) ? -fl : fl;
      }
    }
  
    const bool valid = (hnn > 0.0) && (av > 0.0);
    double lo[NTR];
#pragma unroll
    for (int t = 0; t < NTR; ++t)
      lo[t] = valid ? divr(Tc[t] * hn + divr((div[t] + (fvk[t] - fvk1[t])) * dt, rav), rhn)
                    : 0.0;
    stn<NTR, IL>(in.ws.lo, qn, w0, in.ws.sN, in.wtg, lo);
    // _node_avg_grad: area-weighted mean over the node's active elements, at the levels
    // where an edge of the node takes it (kGradBit; its readers, the edge stage's and the
    // reverse pass's node-gradient lanes, read no other level)
    const int fw = __ldg(m.nrec + n).w;
    if ((__ldg(m.nflags + fw + (k - nzmin)) >> kGradBit) & 1ull) {
      double nx[NTR], ny[NTR], den = 0.0;
#pragma unroll
      for (int t = 0; t < NTR; ++t) nx[t] = ny[t] = 0.0;
      const int c0 = rec.z, c1 = rec.z + int(pk >> 24);
      for (int j = c0; j < c1; ++j) {
        const int el = ld(m.nel_idx + j);
        if (k >= ld(m.eul + el) && k < ld(m.enl + el)) {
          const double a = ld(m.earea + el);
          const uint32_t qe = lq(el, L, k);
          double gx[NTR], gy[NTR];
          ldn<NTR, IL>(in.ws.gx, qe, w0, in.ws.sE, in.wtg, gx);
          ldn<NTR, IL>(in.ws.gy, qe, w0, in.ws.sE, in.wtg, gy);
#pragma unroll
          for (int t = 0; t < NTR; ++t) {
            nx[t] += gx[t] * a;
            ny[t] += gy[t] * a;
          }
          den += a;
        }
      }
      const Rcp rdd = rcp(den > 0.0 ? den : 1.0);
      if (w0 == 0) in.ws.nden[qn] = rdd.y;   // kept for the reverse pass (tracer independent)
#pragma unroll
      for (int t = 0; t < NTR; ++t) {
        nx[t] = divr(nx[t], rdd);
        ny[t] = divr(ny[t], rdd);
      }
      stn<NTR, IL>(in.ws.gnx, qn, w0, in.ws.sN, in.wtg, nx);
      stn<NTR, IL>(in.ws.gny, qn, w0, in.ws.sN, in.wtg, ny);
    }
  }

  // adv_flux_ver_ho (QR4C on ttfAB) minus the LO vertical flux (tracer_adv.py:241-295)
  double hi[NTR];
#pragma unroll
  for (int t = 0; t < NTR; ++t) hi[t] = 0.0;
  if (k == nzmin) {
    double To[NTR];
    ldn<NTR, IL>(in.T_old, qn, t0, ts, tg, To);
#pragma unroll
    for (int t = 0; t < NTR; ++t) hi[t] = -ab2(Tc[t], To[t]) * Wf * area_k;
  } else if (k == nzmax) {
    // bottom interface: no flux
  } else if (k == nzmin + 1 || k == nzmax - 1) {
    double To[NTR], Tom[NTR];
    ldn<NTR, IL>(in.T_old, qn, t0, ts, tg, To);
    ldn<NTR, IL>(in.T_old, qn - 1, t0, ts, tg, Tom);
#pragma unroll
    for (int t = 0; t < NTR; ++t)
      hi[t] = -0.5 * (ab2(Ta[t], Tom[t]) + ab2(Tc[t], To[t])) * Wf * area_k;
  } else if (k >= nzmin + 2 && k <= nzmax - 2) {
    double Znz, Zm1, Zm2, Zp1, zb;   // QR4C stencil depths (tracer_adv.py:228-238, 265-273)
    if (in.Z3d) {
      const double* Zc = in.Z3d + base;
      Znz = ld(Zc + k); Zm1 = ld(Zc + k - 1); Zm2 = ld(Zc + k - 2);
      Zp1 = ld(Zc + (k + 1 < L ? k + 1 : L - 1)); zb = ld(in.zbar3 + qn);
    } else {
      Znz = ld(m.Zp + k); Zm1 = ld(m.Zp + k - 1); Zm2 = ld(m.Zp + k - 2);
      Zp1 = ld(m.Zp + (k + 1 < L ? k + 1 : L - 1)); zb = ld(m.zbar + k);
    }
    const Rcp rdc = rcp(safe_nz(Zm1 - Znz)), rdu = rcp(safe_nz(Znz - Zp1)),
              rdd = rcp(safe_nz(Zm2 - Zm1));
    const Rcp r3{3.0, 1.0 / 3.0, true};
    double To[NTR], Tom[NTR], Tm2[NTR], Tom2[NTR], Tp[NTR], Top[NTR];
    ldn<NTR, IL>(in.T_old, qn, t0, ts, tg, To);
    ldn<NTR, IL>(in.T_old, qn - 1, t0, ts, tg, Tom);
    ldn<NTR, IL>(in.T, qn - 2, t0, ts, tg, Tm2);
    ldn<NTR, IL>(in.T_old, qn - 2, t0, ts, tg, Tom2);
    ldn<NTR, IL>(in.T, qn + 1, t0, ts, tg, Tp);
    ldn<NTR, IL>(in.T_old, qn + 1, t0, ts, tg, Top);
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      const double A0 = ab2(Tc[t], To[t]), Am1 = ab2(Ta[t], Tom[t]);
      const double Am2 = ab2(Tm2[t], Tom2[t]), Ap1 = ab2(Tp[t], Top[t]);
      const double qc = divr(Am1 - A0, rdc);
      const double qu = divr(A0 - Ap1, rdu);
      const double qd = divr(Am2 - Am1, rdd);
      const double Tmean1 = A0 + divr((2.0 * qc + qu) * (zb - Znz), r3);
      const double Tmean2 = Am1 + divr((2.0 * qc + qd) * (zb - Zm1), r3);
      hi[t] = -0.5 * (Tmean1 + Tmean2) * Wf * area_k;
    }
  }
  double adf[NTR];
#pragma unroll
  for (int t = 0; t < NTR; ++t) {
    const double lo_v = in.w_i ? (layer ? vflux_up(Tc[t], Ta[t], Wf, area_k) : 0.0) : fvk[t];
    adf[t] = hi[t] - lo_v;
  }
  stn<NTR, IL>(in.ws.adfv, qn, w0, in.ws.sN, in.wtg, adf);
}

// ---------------------------- adv_tra_vert_impl: implicit w_i advection of LO
template <int NTR, bool IL>
__device__ __forceinline__ void body_vert_impl(const Inst& in, int64_t n, int t0, int w0) {
  const DevMesh& m = *in.m;
  if (n >= m.N || !in.w_i) return;
  const int L = m.L;
  const int nzmin = m.nzmin[n], nzmax = m.nzmax[n];
  if (nzmax <= nzmin) return;
  const uint32_t base = lq(int(n), L, 0);
  const double dt = in.dt;
  double cp[kMaxLevels], dp[kMaxLevels];
  for (int tw = w0; tw < w0 + NTR; ++tw) {
    auto LO = [&](int k) -> double& { return in.ws.lo[tix<IL>(base + k, tw, in.ws.sN, in.wtg)]; };
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
      // the neighbours above the surface and below the bottom enter with a zero
      // coefficient; LO is 0 there in the reference, and this step never wrote them
      const double Tm = surf ? 0.0 : LO(k - 1), T0 = LO(k), Tp = bot ? 0.0 : LO(k + 1);
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
    for (int k = nzmin; k < nzmax; ++k) LO(k) = LO(k) + dp[k];
  }
}

// -------------------------- fill_up_dn_grad + adv_flux_hor_ho - LO flux = adf_h
template <int NTR, bool IL>
__device__ __forceinline__ void body_edge_adf(const Inst& in, int64_t i, int t0, int w0) {
  const DevMesh& m = *in.m;
  if (i >= m.n_edge) return;
  const int4 rec = __ldg(m.edge4 + i);
  const int e = lane_ent(uint32_t(rec.x)), k = lane_lev(uint32_t(rec.x)), L = m.L;
  const int n1 = rec.y, n2 = rec.z;
  const bool use_tri = in_range(k, unsigned(rec.w));
  const double vf = ld(in.ws.vflux + lq(e, L, k));
  const double avf = fabs(vf);
  const double c1 = ld(m.ecoef + 2 * e), c2 = ld(m.ecoef + 2 * e + 1);
  const uint32_t q1 = lq(n1, L, k), q2 = lq(n2, L, k);
  const int64_t ts = in.tstride;
  const int tg = in.tg;
  double T1[NTR], T2[NTR], O1[NTR], O2[NTR], g0[NTR], g1[NTR], g2[NTR], g3[NTR];
  ldn<NTR, IL>(in.T, q1, t0, ts, tg, T1);
  ldn<NTR, IL>(in.T, q2, t0, ts, tg, T2);
  ldn<NTR, IL>(in.T_old, q1, t0, ts, tg, O1);
  ldn<NTR, IL>(in.T_old, q2, t0, ts, tg, O2);
  if (use_tri) {
    // both cells are wet at k here (k is above every adjacent cell's bottom)
    const int up = ld(m.eupdn + 2 * e), dn = ld(m.eupdn + 2 * e + 1);
    const uint32_t qu = lq(up, L, k), qd = lq(dn, L, k);
    ldn<NTR, IL>(in.ws.gx, qu, w0, in.ws.sE, in.wtg, g0);
    ldn<NTR, IL>(in.ws.gx, qd, w0, in.ws.sE, in.wtg, g1);
    ldn<NTR, IL>(in.ws.gy, qu, w0, in.ws.sE, in.wtg, g2);
    ldn<NTR, IL>(in.ws.gy, qd, w0, in.ws.sE, in.wtg, g3);
  
  } else {
    ldn<NTR, IL>(in.ws.gnx, q1, w0, in.ws.sN, in.wtg, g0);
    ldn<NTR, IL>(in.ws.gnx, q2, w0, in.ws.sN, in.wtg, g1);
    ldn<NTR, IL>(in.ws.gny, q1, w0, in.ws.sN, in.wtg, g2);
    ldn<NTR, IL>(in.ws.gny, q2, w0, in.ws.sN, in.wtg, g3);
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

// ------------------------ zalesak a2: element max/min of the LO/T window
template <int NTR, bool IL>
__device__ __forceinline__ void body_elem_bounds(const Inst& in, int64_t i, int t0, int w0) {
  const DevMesh& m = *in.m;
  if (i >= m.n_elem) return;
  const uint32_t lane = ld(m.elem_lanes + i);
  const int e = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const uint32_t q[3] = {lq(ld(m.enodes + 3 * e), L, k),
                        lq(ld(m.enodes + 3 * e + 1), L, k),
                        lq(ld(m.enodes + 3 * e + 2), L, k)};
  double mx[NTR], mn[NTR], hi[3][NTR], lw[3][NTR];
#pragma unroll
  for (int t = 0; t < NTR; ++t) { mx[t] = -INFINITY; mn[t] = INFINITY; }
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    double a[NTR], b[NTR];
    ldn<NTR, IL>(in.ws.lo, q[v], w0, in.ws.sN, in.wtg, a);
    ldn<NTR, IL>(in.T, q[v], t0, in.tstride, in.tg, b);
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      hi[v][t] = fmax(a[t], b[t]);
      lw[v][t] = fmin(a[t], b[t]);
      mx[t] = fmax(mx[t], hi[v][t]);
      mn[t] = fmin(mn[t], lw[v][t]);
    }
  }
  const uint32_t qe = lq(e, L, k);
  {   // vertices attaining the bounds (the reverse pass splits cotangents evenly over them)
    int cx[NTR], cn[NTR];
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      cx[t] = (hi[0][t] == mx[t]) + (hi[1][t] == mx[t]) + (hi[2][t] == mx[t]);
      cn[t] = (lw[0][t] == mn[t]) + (lw[1][t] == mn[t]) + (lw[2][t] == mn[t]);
    }
    stc<NTR, IL>(in.ws.ecx, qe, w0, in.ws.sE, in.wtg, cx);
    stc<NTR, IL>(in.ws.ecn, qe, w0, in.ws.sE, in.wtg, cn);
  }
  stn<NTR, IL>(in.ws.amax, qe, w0, in.ws.sE, in.wtg, mx);
  stn<NTR, IL>(in.ws.amin, qe, w0, in.ws.sE, in.wtg, mn);
}

// ------------------------ zalesak a3: node cluster max/min over elements
template <int NTR, bool IL>
__device__ __forceinline__ void body_node_cluster(const Inst& in, int64_t i, int t0, int w0) {
  const DevMesh& m = *in.m;
  if (i >= m.n_layer) return;
  const int4 rec = __ldg(m.layer4 + i);
  const int n = lane_ent(uint32_t(rec.x)), k = lane_lev(uint32_t(rec.x)), L = m.L;
  const int c0 = rec.z, c1 = rec.z + int(unsigned(rec.w) >> 24);
  double mx[NTR], mn[NTR];
#pragma unroll
  for (int t = 0; t < NTR; ++t) { mx[t] = -INFINITY; mn[t] = INFINITY; }
  for (int j = c0; j < c1; ++j) {
    const int el = ld(m.nel_idx + j);
    if (k >= ld(m.eul + el) && k < ld(m.enl + el)) {
      const uint32_t q = lq(el, L, k);
      double a[NTR], b[NTR];
      ldn<NTR, IL>(in.ws.amax, q, w0, in.ws.sE, in.wtg, a);
      ldn<NTR, IL>(in.ws.amin, q, w0, in.ws.sE, in.wtg, b);
#pragma unroll
      for (int t = 0; t < NTR; ++t) {
        mx[t] = fmax(mx[t], a[t]);
        mn[t] = fmin(mn[t], b[t]);
      }
    } else {   // a cell without this level pads with -+BIG (tracer_adv.py:396-397)
#pragma unroll
      for (int t = 0; t < NTR; ++t) {
        mx[t] = fmax(mx[t], -kBig);
        mn[t] = fmin(mn[t], kBig);
      }
    }
  }
  const uint32_t qn = lq(n, L, k);
  stn<NTR, IL>(in.ws.tvmax, qn, w0, in.ws.sN, in.wtg, mx);
  stn<NTR, IL>(in.ws.tvmin, qn, w0, in.ws.sN, in.wtg, mn);
  // cells attaining the cluster bounds (padded values included), for the reverse pass
  int cx[NTR], cn[NTR];
#pragma unroll
  for (int t = 0; t < NTR; ++t) cx[t] = cn[t] = 0;
  for (int j = c0; j < c1; ++j) {
    const int el = ld(m.nel_idx + j);
    double a[NTR], b[NTR];
    if (k >= ld(m.eul + el) && k < ld(m.enl + el)) {
      const uint32_t q = lq(el, L, k);
      ldn<NTR, IL>(in.ws.amax, q, w0, in.ws.sE, in.wtg, a);
      ldn<NTR, IL>(in.ws.amin, q, w0, in.ws.sE, in.wtg, b);
    } else {
#pragma unroll
      for (int t = 0; t < NTR; ++t) { a[t] = -kBig; b[t] = kBig; }
    }
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      cx[t] += a[t] == mx[t];
      cn[t] += b[t] == mn[t];
    }
  }
  stc<NTR, IL>(in.ws.ccx, qn, w0, in.ws.sN, in.wtg, cx);
  stc<NTR, IL>(in.ws.ccn, qn, w0, in.ws.sN, in.wtg, cn);
}

// ------------------- zalesak a4 + b1 + b2: admissible window, sums, factors
template <int NTR, bool IL>
__device__ __forceinline__ void body_node_factors(const Inst& in, int64_t i, int t0, int w0) {
  const DevMesh& m = *in.m;
  if (i >= m.n_layer) return;
  const int4 rec = __ldg(m.layer4 + i);
  const unsigned pk = unsigned(rec.w);
  const int n = lane_ent(uint32_t(rec.x)), k = lane_lev(uint32_t(rec.x)), L = m.L;
  const int nzmin = int(pk & 255u), nzmax = int((pk >> 8) & 255u);
  const uint32_t base = lq(n, L, 0), qn = base + uint32_t(k);
  const bool use_own = (k == nzmin) || (k == nzmax - 1);
  const double av = ld(m.areasvol + qn), hnn = ld(in.hnode_new + qn);
  const bool valid = (av > 0.0) && (hnn > 0.0);
  const double sa = av > 0.0 ? av : 1.0, sh = hnn > 0.0 ? hnn : 1.0;
  const Rcp rsa = rcp(sa), rsh = rcp(sh);
  const double dt = in.dt;
  const int64_t sN = in.ws.sN;
  double tmax[NTR], tmin[NTR];
  ldn<NTR, IL>(in.ws.tvmax, qn, w0, sN, in.wtg, tmax);
  ldn<NTR, IL>(in.ws.tvmin, qn, w0, sN, in.wtg, tmin);
  if (!use_own) {   // interior: max/min over k-1, k, k+1 (all layers of this column)
    double am[NTR], an[NTR], bm[NTR], bn[NTR];
    ldn<NTR, IL>(in.ws.tvmax, qn - 1, w0, sN, in.wtg, am);
    ldn<NTR, IL>(in.ws.tvmin, qn - 1, w0, sN, in.wtg, an);
    ldn<NTR, IL>(in.ws.tvmax, qn + 1, w0, sN, in.wtg, bm);
    ldn<NTR, IL>(in.ws.tvmin, qn + 1, w0, sN, in.wtg, bn);
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      tmax[t] = fmax(fmax(am[t], tmax[t]), bm[t]);
      tmin[t] = fmin(fmin(an[t], tmin[t]), bn[t]);
    }
  }
  double lo[NTR], ft[NTR], fb[NTR];
  ldn<NTR, IL>(in.ws.lo, qn, w0, sN, in.wtg, lo);
  ldn<NTR, IL>(in.ws.adfv, qn, w0, sN, in.wtg, ft);
  ldn<NTR, IL>(in.ws.adfv, qn + 1, w0, sN, in.wtg, fb);   // k+1 <= nzmax < L
  double sp[NTR], sm[NTR];
#pragma unroll
  for (int t = 0; t < NTR; ++t) sp[t] = sm[t] = 0.0;
  const int e0 = rec.y, e1 = rec.y + int((pk >> 16) & 255u);
  for (int j = e0; j < e1; ++j) {
    const int idx = ld(m.ne_idx + j), e = idx >> 1;
    if (k < ld(m.ekmin + e) || k >= ld(m.ekmax + e)) continue;   // no flux on this level
    double a[NTR];
    ldn<NTR, IL>(in.ws.adfh, lq(e, L, k), w0, in.ws.sEd, in.wtg, a);
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      const double s = (idx & 1) ? -a[t] : a[t];
      sp[t] += fmax(s, 0.0);
      sm[t] += fmin(s, 0.0);
    }
  }
  double pf[NTR], mf[NTR], pl[NTR], mi[NTR];
#pragma unroll
  for (int t = 0; t < NTR; ++t) {
    const double plus = (fmax(ft[t], 0.0) + fmax(-fb[t], 0.0)) + sp[t];
    const double minus = (fmin(ft[t], 0.0) + fmin(-fb[t], 0.0)) + sm[t];
    pl[t] = plus;
    mi[t] = minus;
    pf[t] = 1.0;
    mf[t] = 1.0;
    if (valid) {
      const double flux_pos = divr(divr(plus * dt, rsa), rsh) + kFluxEps;
      const double flux_neg = divr(divr(minus * dt, rsa), rsh) - kFluxEps;
      pf[t] = fmin(1.0, (tmax[t] - lo[t]) / flux_pos);
      mf[t] = fmin(1.0, (tmin[t] - lo[t]) / flux_neg);
    }
  }
  stn<NTR, IL>(in.ws.pf, qn, w0, sN, in.wtg, pf);
  stn<NTR, IL>(in.ws.mf, qn, w0, sN, in.wtg, mf);
  stn<NTR, IL>(in.ws.fplus, qn, w0, sN, in.wtg, pl);    // kept for the reverse pass
  stn<NTR, IL>(in.ws.fminus, qn, w0, sN, in.wtg, mi);
}

// ---------- zalesak b3 + flux2dtracer_fct + ale_reconstruct: T_new on layers
template <int NTR, bool IL>
__device__ __forceinline__ void body_node_final(const Inst& in, int64_t i, int t0, int w0) {
  const DevMesh& m = *in.m;
  if (i >= m.n_layer) return;
  const int4 rec = __ldg(m.layer4 + i);
  const unsigned pk = unsigned(rec.w);
  const int n = lane_ent(uint32_t(rec.x)), k = lane_lev(uint32_t(rec.x)), L = m.L;
  const int nzmin = int(pk & 255u), nzmax = int((pk >> 8) & 255u);
  const uint32_t base = lq(n, L, 0), qn = base + uint32_t(k);
  const double av = ld(m.areasvol + qn);
  const double sa = av > 0.0 ? av : 1.0;
  const double hn = ld(in.hnode + qn), hnn = ld(in.hnode_new + qn);
  const Rcp rsa = rcp(sa), rhn = rcp(hnn);
  const double dt = in.dt;
  const int tg = in.tg;
  const int64_t sN = in.ws.sN;
  // own limiter factors at k (and k-1 / k+1 for the vertical fluxes)
  double pf0[NTR], mf0[NTR], ft[NTR];
  ldn<NTR, IL>(in.ws.pf, qn, w0, sN, in.wtg, pf0);
  ldn<NTR, IL>(in.ws.mf, qn, w0, sN, in.wtg, mf0);
  ldn<NTR, IL>(in.ws.adfv, qn, w0, sN, in.wtg, ft);
  // limited vertical flux at the top interface k (tracer_adv.py:453-459)
  double vt[NTR];
  if (k == nzmin) {
#pragma unroll
    for (int t = 0; t < NTR; ++t) vt[t] = (ft[t] >= 0.0 ? pf0[t] : mf0[t]) * ft[t];
  } else {
    double pfa[NTR], mfa[NTR];
    ldn<NTR, IL>(in.ws.pf, qn - 1, w0, sN, in.wtg, pfa);
    ldn<NTR, IL>(in.ws.mf, qn - 1, w0, sN, in.wtg, mfa);
#pragma unroll
    for (int t = 0; t < NTR; ++t)
      vt[t] = (ft[t] >= 0.0 ? fmin(mfa[t], pf0[t]) : fmin(pfa[t], mf0[t])) * ft[t];
  }
  // limited vertical flux at the bottom interface k+1 (0 at the node's bottom)
  double vb[NTR];
  if (k + 1 >= nzmax) {
#pragma unroll
    for (int t = 0; t < NTR; ++t) vb[t] = 0.0;
  } else {
    double fb[NTR], pfb[NTR], mfb[NTR];
    ldn<NTR, IL>(in.ws.adfv, qn + 1, w0, sN, in.wtg, fb);
    ldn<NTR, IL>(in.ws.pf, qn + 1, w0, sN, in.wtg, pfb);
    ldn<NTR, IL>(in.ws.mf, qn + 1, w0, sN, in.wtg, mfb);
#pragma unroll
    for (int t = 0; t < NTR; ++t)
      vb[t] = (fb[t] >= 0.0 ? fmin(mf0[t], pfb[t]) : fmin(pf0[t], mfb[t])) * fb[t];
  }
  // limited horizontal fluxes, ascending edge id
  double hsc[NTR];
#pragma unroll
  for (int t = 0; t < NTR; ++t) hsc[t] = 0.0;
  const int e0 = rec.y, e1 = rec.y + int((pk >> 16) & 255u);
  for (int j = e0; j < e1; ++j) {
    const int idx = ld(m.ne_idx + j), e = idx >> 1;
    if (k < ld(m.ekmin + e) || k >= ld(m.ekmax + e)) continue;   // no flux on this level
    const uint32_t qo = lq(ld(m.ne_oth + j), L, k);
    double a[NTR], pfo[NTR], mfo[NTR];
    ldn<NTR, IL>(in.ws.adfh, lq(e, L, k), w0, in.ws.sEd, in.wtg, a);
    ldn<NTR, IL>(in.ws.pf, qo, w0, sN, in.wtg, pfo);
    ldn<NTR, IL>(in.ws.mf, qo, w0, sN, in.wtg, mfo);
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      // (pf, mf) at the edge's first node n1 and second node n2
      const double pf1 = (idx & 1) ? pfo[t] : pf0[t], mf1 = (idx & 1) ? mfo[t] : mf0[t];
      const double pf2 = (idx & 1) ? pf0[t] : pfo[t], mf2 = (idx & 1) ? mf0[t] : mfo[t];
      const double ae = a[t] >= 0.0 ? fmin(pf1, mf2) : fmin(mf1, pf2);
      const double lim = ae * a[t];
      hsc[t] += (idx & 1) ? -lim : lim;
    }
  }
  double Tv[NTR], lo[NTR], out[NTR];
  ldn<NTR, IL>(in.T, qn, t0, in.tstride, tg, Tv);
  ldn<NTR, IL>(in.ws.lo, qn, w0, sN, in.wtg, lo);
#pragma unroll
  for (int t = 0; t < NTR; ++t) {
    const double lo_trans = -Tv[t] * hn + lo[t] * hnn;
    const double vdiv = av > 0.0 ? divr((vt[t] - vb[t]) * dt, rsa) : 0.0;
    double d = divr(hsc[t] * dt, rsa) + (lo_trans + vdiv);
    d = d + Tv[t] * (hn - hnn);
    out[t] = Tv[t] + (hnn > 0.0 ? divr(d, rhn) : 0.0);
  }
  stn<NTR, IL>(in.T_new, qn, t0, in.tstride, tg, out);
  count_nonfinite<NTR>(in.nonfinite, out);
}

// ------------- implicit vertical diffusion (tracer_diff.py:68-123, ops.py:121-168)
// One thread per node column and NTR tracers: the Thomas algorithm over the column's wet
// layers [nzmin, nzmax) (the reference's padded rows above and below solve to exactly 0,
// so starting and ending the recursions there gives the same numbers). The elimination
// factors m and cp do not depend on the tracer: one reciprocal of m serves c/m and every
// tracer's dp/m. cp goes to workspace slot w0 of adfv, dp to the tracer's slots of lo
// (both free after the FCT stages); the back substitution reads them in reverse.
template <int NTR, bool IL>
__device__ __forceinline__ void body_vdiff(const Inst& in, int64_t n, int t0, int w0) {
  const DevMesh& m = *in.m;
  if (n >= m.N || !in.Kv) return;
  const int L = m.L;
  const int nzmin = ld(m.nzmin + n), nzmax = ld(m.nzmax + n);
  const uint32_t base = lq(int(n), L, 0);
  const int64_t ts = in.tstride, sN = in.ws.sN;
  const int tg = in.tg;
  const double* Tin = in.vd_T;
  if (Tin != in.T_new) {   // out of place: dry levels keep T
    for (int k = 0; k < L; ++k) {
      if (k >= nzmin && k < nzmax) continue;
      double v[NTR];
      ldn<NTR, IL>(Tin, base + k, t0, ts, tg, v);
      stn<NTR, IL>(in.T_new, base + k, t0, ts, tg, v);
    }
  }
  if (nzmax <= nzmin) return;
  const double dt = in.dt;
  const double* Zc = in.vd_Z3d ? in.vd_Z3d + base : m.Zp;
  double cprev = 0.0, dprev[NTR], Tm[NTR], Tc[NTR], Tp[NTR];
#pragma unroll
  for (int t = 0; t < NTR; ++t) dprev[t] = 0.0;
  ldn<NTR, IL>(Tin, base + nzmin, t0, ts, tg, Tc);
  ldn<NTR, IL>(Tin, base + (nzmin > 0 ? nzmin - 1 : 0), t0, ts, tg, Tm);
  for (int k = nzmin; k < nzmax; ++k) {
    const uint32_t q = base + uint32_t(k);
    const bool last = k + 1 >= L;
    if (last) {
#pragma unroll
      for (int t = 0; t < NTR; ++t) Tp[t] = 0.0;
    } else {
      ldn<NTR, IL>(Tin, q + 1, t0, ts, tg, Tp);
    }
    double dzu = k == 0 ? 0.0 : ld(Zc + k - 1) - ld(Zc + k);
    double dzd = ld(Zc + k) - (last ? 0.0 : ld(Zc + k + 1));
    dzu = dzu == 0.0 ? 1.0 : dzu;
    dzd = dzd == 0.0 ? 1.0 : dzd;
    const double av = ld(m.areasvol + q);
    const double sav = av > 0.0 ? av : 1.0;
    const double ar = ld(m.area + q), arp = last ? 0.0 : ld(m.area + q + 1);
    const double kv = ld(in.Kv + q), kvp = last ? 0.0 : ld(in.Kv + q + 1);
    const double a_full = -kv * dt / dzu * (ar / sav);
    const double c_full = -kvp * dt / dzd * (arp / sav);
    const double a = k == nzmin ? 0.0 : a_full;
    const double c = k == nzmax - 1 ? 0.0 : c_full;
    const double b = -a - c + ld(in.hnode_new + q);
    const Rcp rm = rcp(b - a * cprev);
    cprev = divr(c, rm);
    in.ws.adfv[tix<IL>(q, w0, sN, in.wtg)] = cprev;
    double swd = 0.0;
    if (in.sw_3d) {
      const double sw = ld(in.sw_3d + q), swp = last ? 0.0 : ld(in.sw_3d + q + 1);
      swd = (sw - swp * (arp / sav)) * dt;
    }
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      double rhs = a * (Tc[t] - Tm[t]) + c * (Tc[t] - Tp[t]);
      if (in.bc_surf) rhs = rhs + (k == nzmin ? ld(in.bc_surf + (t0 + t) * in.bc_stride + n) : 0.0);
      if (in.sw_3d && t0 + t == in.sw_tracer) rhs = rhs + swd;
      dprev[t] = divr(rhs - a * dprev[t], rm);
      Tm[t] = Tc[t];
      Tc[t] = Tp[t];
    }
    stn<NTR, IL>(in.ws.lo, q, w0, sN, in.wtg, dprev);
  }
  double x[NTR];
#pragma unroll
  for (int t = 0; t < NTR; ++t) x[t] = 0.0;
  for (int k = nzmax - 1; k >= nzmin; --k) {
    const uint32_t q = base + uint32_t(k);
    const double cp = in.ws.adfv[tix<IL>(q, w0, sN, in.wtg)];
    double dp[NTR], Tv[NTR];
    ldn<NTR, IL>(in.ws.lo, q, w0, sN, in.wtg, dp);
    ldn<NTR, IL>(Tin, q, t0, ts, tg, Tv);
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      x[t] = dp[t] - cp * x[t];
      Tv[t] = Tv[t] + x[t];
    }
    stn<NTR, IL>(in.T_new, q, t0, ts, tg, Tv);
  }
}

// ------------------------------------------- dry levels keep T (ale_reconstruct)
template <bool IL>
__device__ __forceinline__ void body_copy_dry(const Inst& in, int64_t i) {
  const DevMesh& m = *in.m;
  if (i >= m.n_dry) return;
  const uint32_t lane = __ldg(m.dry_lanes + i);
  const uint32_t q = lq(lane_ent(lane), m.L, lane_lev(lane));
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t a = tix<IL>(q, t, in.tstride, in.tg);
    in.T_new[a] = in.T[a];
  }
}

// Kernel wrappers: ``_1`` takes one instance by value (tracer-major layout, the
// single-call path); ``_n`` reads instance blockIdx.y of a device table (interleaved
// layout, the batched path). A launch covers S = 2^lg tracer slices of NTR tracers each:
// in ``_n`` the S threads of a lane are adjacent (slice = thread index mod S), so they
// read one contiguous run of S*NTR interleaved tracers together; in ``_1`` the slice is
// blockIdx.y, so lanes stay contiguous along x within each tracer plane.
// Resident 256-thread blocks per SM the compiler must fit (registers capped
// accordingly): latency hiding pays more than the spills it costs (one tracer, the
// adjoint's taped forward on the CORE2-size mesh: 11.1 ms for 10 steps at 6 blocks,
// 10.6 ms at 7, no gain at 8).
template <int NTR>
constexpr int kMinBlocks = NTR == 1 ? 7 : NTR == 2 ? 5 : NTR == 4 ? 4 : 2;

#define FCT_KERNEL_T(name, body)                                                        \
  template <int NTR>                                                                    \
  __global__ void __launch_bounds__(256, kMinBlocks<NTR>) name##_1(Inst in, int t0,     \
                                                                   int w0) {            \
    const int sub = int(blockIdx.y) * NTR;                                              \
    body<NTR, false>(in, lane_index(), t0 + sub, w0 + sub);                             \
  }                                                                                     \
  template <int NTR>                                                                    \
  __global__ void __launch_bounds__(256, kMinBlocks<NTR>) name##_n(                     \
      const Inst* __restrict__ tab, int t0,                                             \
                                                  int w0, int lg) {                     \
    const int64_t g = lane_index();                                                     \
    const int sub = int(g & ((int64_t(1) << lg) - 1)) * NTR;                            \
    body<NTR, true>(tab[blockIdx.y], g >> lg, t0 + sub, w0 + sub);                      \
  }


// unfused stages (every intermediate in the workspace; the reverse pass reads them)
FCT_KERNEL_T(k_elem_grad, body_elem_grad)
FCT_KERNEL_T(k_node_lo, body_node_lo)
FCT_KERNEL_T(k_vert_impl, body_vert_impl)
FCT_KERNEL_T(k_edge_adf, body_edge_adf)
FCT_KERNEL_T(k_elem_bounds, body_elem_bounds)
FCT_KERNEL_T(k_node_cluster, body_node_cluster)
FCT_KERNEL_T(k_node_factors, body_node_factors)
FCT_KERNEL_T(k_node_final, body_node_final)
// implicit vertical diffusion (the epilogue of the batched step and fct_vert_diff)
FCT_KERNEL_T(k_vdiff, body_vdiff)

__global__ void __launch_bounds__(256) k_vflux_1(Inst in) { body_vflux(in, lane_index()); }
__global__ void __launch_bounds__(256) k_vflux_n(const Inst* __restrict__ tab) {
  body_vflux(tab[blockIdx.y], lane_index());
}
__global__ void __launch_bounds__(256) k_copy_dry_1(Inst in) {
  body_copy_dry<false>(in, lane_index());
}
__global__ void __launch_bounds__(256) k_copy_dry_n(const Inst* __restrict__ tab) {
  body_copy_dry<true>(tab[blockIdx.y], lane_index());
}

}  // namespace

const char* const kStageNames[kNumStages] = {
    "vflux", "elem_grad", "node_lo", "vert_impl", "edge_adf", "elem_bounds",
    "node_cluster", "node_factors", "node_final", "copy_dry"};

// One stage over the tracers [c0, c1) of a workspace chunk: launches of S slices x NTR
// tracers, NTR in {8, 4, 2, 1} (largest first, at most d.per_thread) and S the largest
// power of two (at most 8) with S*NTR tracers left; the workspace index of tracer t is
// t - c0.
#define FCT_STAGE_AS(name, lanes, P)                                                    \
  do {                                                                                  \
    if (tab)                                                                            \
      name##_n<P><<<dim3(xblocks(int64_t(lanes) << lg), unsigned(n)), B, 0, s>>>(        \
          tab, t0, w0, lg);                                                             \
    else                                                                                \
      name##_1<P><<<dim3(xblocks(lanes), 1u << lg), B, 0, s>>>(single, t0, w0);          \
  } while (0)

#define FCT_SPLIT(AS, name, lanes)                                                      \
  do {                                                                                  \
    for (int t0 = c0; t0 < c1;) {                                                       \
      const int rem = c1 - t0;                                                          \
      const int lim = std::min(rem, d.per_thread);                                      \
      const int P = lim >= 8 ? 8 : lim >= 4 ? 4 : lim >= 2 ? 2 : 1;                     \
      int lg = 0;                                                                       \
      while (lg < 3 && (P << (lg + 1)) <= rem) ++lg;                                    \
      const int w0 = t0 - c0;                                                           \
      if (P == 8) AS(name, lanes, 8);                                                   \
      else if (P == 4) AS(name, lanes, 4);                                              \
      else if (P == 2) AS(name, lanes, 2);                                              \
      else AS(name, lanes, 1);                                                          \
      t0 += P << lg;                                                                    \
    }                                                                                   \
  } while (0)
#define FCT_STAGE(name, lanes) FCT_SPLIT(FCT_STAGE_AS, name, lanes)

// the fused step's edge stage beside its LO stage when the caller provides a fork
constexpr bool kForkEdge = true;

int fork_create(Fork& f) {
  FCT_CUDA(cudaStreamCreateWithFlags(&f.side, cudaStreamNonBlocking));
  for (auto& e : f.ev) FCT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return FCT_OK;
}

void fork_destroy(Fork& f) {
  if (f.side) {
    cudaStreamSynchronize(f.side);
    cudaStreamDestroy(f.side);
  }
  for (auto& e : f.ev)
    if (e) cudaEventDestroy(e);
  f = Fork{};
}

int launch_forward_events(const Inst& single, const Inst* tab, int n, const LaunchDims& d,
                          cudaStream_t s, cudaEvent_t* after, bool stop_before_final,
                          int chunk_sel) {
  constexpr int B = 256;
  auto xblocks = [&](int64_t lanes) {
    return unsigned(std::max<int64_t>(1, (lanes + B - 1) / B));
  };
  auto grid = [&](int64_t lanes) { return dim3(xblocks(lanes), unsigned(n), 1); };
  const int chunk = d.chunk > 0 ? d.chunk : d.ntr;
  const int nchunks = (d.ntr + chunk - 1) / chunk;
  for (int ci = 0; ci < nchunks; ++ci) {
    if (chunk_sel >= 0 && ci != chunk_sel) continue;
    const int c0 = ci * chunk, c1 = std::min(d.ntr, c0 + chunk);
    int stage = 0;
    auto mark = [&]() {
      if (after) cudaEventRecord(after[stage], s);
      ++stage;
    };
    if (ci == 0) {   // the volume flux is shared by all tracers
      if (tab && d.any_derive_w) {   // producer: w_e from continuity, in the same graph
        const int st = launch_compute_w_tab(tab, n, d.max_nodes, s);
        if (st) return st;
      }
      if (!d.skip_vflux) {
        if (tab) k_vflux_n<<<grid(d.max_edge), B, 0, s>>>(tab);
        else k_vflux_1<<<grid(d.max_edge), B, 0, s>>>(single);
      }
    }
    mark();
    if (d.fused) {
      // segment kernels (fct_seg_*.cu), 5 launches per chunk; the stages folded into
      // others record empty intervals (elem_grad: the node gradients are evaluated only
      // where MFCT needs them, in the edge stage; elem_bounds and node_cluster: the factors
      // stage). With a fork (and no stage timing) the edge stage runs on the side stream
      // beside the LO stage and the limiter waits for both.
      const Fork* fk = (kForkEdge && d.fork && !after) ? d.fork : nullptr;
      mark();
      int st;
      if (fk) {
        FCT_CUDA(cudaEventRecord(fk->ev[0], s));
        FCT_CUDA(cudaStreamWaitEvent(fk->side, fk->ev[0], 0));
        if ((st = launch_seg_edge(single, tab, n, d, c0, c1, fk->side))) return st;
        if ((st = launch_edge_fix(single, tab, n, d, c0, c1, fk->side))) return st;
        FCT_CUDA(cudaEventRecord(fk->ev[1], fk->side));
      }
      if ((st = launch_seg_lo(single, tab, n, d, c0, c1, s))) return st;
      mark();
      if (d.any_wi) FCT_STAGE(k_vert_impl, d.max_nodes);
      mark();
      if (fk) {
        FCT_CUDA(cudaStreamWaitEvent(s, fk->ev[1], 0));
      } else {
        if ((st = launch_seg_edge(single, tab, n, d, c0, c1, s))) return st;
        if ((st = launch_edge_fix(single, tab, n, d, c0, c1, s))) return st;
      }
      mark();
      mark();
      mark();
      if ((st = launch_seg_limit(single, tab, n, d, c0, c1, s))) return st;
      mark();
      if (stop_before_final) continue;
      if ((st = launch_seg_final(single, tab, n, d, c0, c1, s))) return st;
      if (d.any_vdiff) {   // epilogue: implicit vertical diffusion of this chunk, in place
        if (d.copy_dry) {  // the dry levels of T_new must hold T before it runs
          if (tab) k_copy_dry_n<<<grid(d.max_dry), B, 0, s>>>(tab);
          else k_copy_dry_1<<<grid(d.max_dry), B, 0, s>>>(single);
        }
        FCT_STAGE(k_vdiff, d.max_nodes);
      }
      mark();
      continue;
    }
    FCT_STAGE(k_elem_grad, d.max_elem);
    mark();
    FCT_STAGE(k_node_lo, d.max_iface);
    mark();
    if (d.any_wi) FCT_STAGE(k_vert_impl, d.max_nodes);
    mark();
    FCT_STAGE(k_edge_adf, d.max_edge);
    mark();
    FCT_STAGE(k_elem_bounds, d.max_elem);
    mark();
    FCT_STAGE(k_node_cluster, d.max_layer);
    mark();
    FCT_STAGE(k_node_factors, d.max_layer);
    mark();
    if (stop_before_final) continue;
    FCT_STAGE(k_node_final, d.max_layer);
    mark();
  }
  if (d.copy_dry && !stop_before_final && (chunk_sel < 0 || chunk_sel == nchunks - 1)) {
    if (tab) k_copy_dry_n<<<grid(d.max_dry), B, 0, s>>>(tab);
    else k_copy_dry_1<<<grid(d.max_dry), B, 0, s>>>(single);
  }
  if (after) cudaEventRecord(after[kNumStages - 1], s);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "forward kernel launch");
  return FCT_OK;
}

int launch_forward(const Inst& single, const Inst* tab, int n, const LaunchDims& d,
                   cudaStream_t s) {
  return launch_forward_events(single, tab, n, d, s, nullptr, false, -1);
}

int launch_forward_stages(const Inst& single, const LaunchDims& d, cudaStream_t s,
                          bool through_factors) {
  return launch_forward_events(single, nullptr, 1, d, s, nullptr, through_factors, -1);
}

int launch_vdiff(const Inst& single, const LaunchDims& d, cudaStream_t s) {
  constexpr int B = 256;
  auto xblocks = [&](int64_t lanes) {
    return unsigned(std::max<int64_t>(1, (lanes + B - 1) / B));
  };
  const Inst* tab = nullptr;
  const int n = 1;
  const int c0 = 0, c1 = d.ntr;
  FCT_STAGE(k_vdiff, d.max_nodes);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FCT_OK : cuda_error(e, "vertical diffusion launch");
}

int launch_copy_dry(const Inst* tab, int n, int64_t max_dry, cudaStream_t s) {
  const dim3 g(unsigned(std::max<int64_t>(1, (max_dry + 255) / 256)), unsigned(n), 1);
  k_copy_dry_n<<<g, 256, 0, s>>>(tab);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FCT_OK : cuda_error(e, "copy_dry launch");
}

}  // namespace fct
