// Reverse mode of the FCT step (fct_adjoint, fct_adjoint_ex) and of compute_w
// (fct_compute_w_adjoint), plus the forward tape (fct_tape_*, fct_forward_taped).
//
// The reverse kernels read the forward step's intermediates: either recomputed first by
// the unfused stage kernels into the plan workspace (per-step recomputation), or kept
// from the forward call on a tape (one full workspace per recorded step). They walk the
// stages backwards; every transpose of a forward scatter is again a deterministic gather
// over a CSR list, so cotangents are bit-identical run to run, and taped and recomputed
// cotangents are the same bits.
//
// Reverse stage map (forward function in fesom_jax/tracer_adv.py -> reverse kernel):
//   ale_reconstruct (:142-151), flux2dtracer_fct (:469-484)        -> r_seed (divergence),
//                                                                     r_bounds_lo (T, LO),
//                                                                     r_dry (dry levels)
//   zalesak_limit b3 (:453-465), b2 (:441-451), a4 window (:407-418) -> r_ratio_window
//   zalesak_limit a2 (:393-397) over a3's per-cell shares            -> r_cluster
//   zalesak_limit a1 (:389-391), compute_fct_lo (:298-313)          -> r_bounds_lo
//   adv_flux_hor_ho (:196-225), adv_flux_hor (:96-105), b1 edges    -> r_edge
//   fill_up_dn_grad (:344-368) node branch                          -> r_gnode
//   adv_flux_ver_ho (:241-295), adv_flux_ver (:108-120), b1 vertical -> r_vert
//   fill_up_dn_grad triangle branch, _node_avg_grad (:329-341)      -> r_tr
//   tracer_gradient_elements (:316-326), vertical fluxes on T and
//     ttfAB, tracer_ab (:59-66), edge terms; w_e summed over tracers -> r_final
//   edge_vflux (:69-93)                                             -> r_uv
//   ale.compute_w (fesom_jax/ale.py:309-365)                        -> r_w_div, r_w_uv
//
// Subgradients follow JAX: maximum/minimum split the cotangent equally at a tie,
// max over an element's vertices and segment_max/min spread it evenly over tied
// entries, abs'(0) = 0 (so d max(x, 0)/dx = 1/2 at x = 0).
#include <algorithm>
#include <vector>

#include "fct_div.cuh"
#include "fct_host.h"

using namespace fct;

struct FctTape {
  FctPlan* plan = nullptr;
  int ntr = 0, steps = 0;
  double* d = nullptr;
  bool owned = false;   // allocated by fct_tape_create (else caller memory)
  std::vector<Workspace> ws;
  std::vector<char> recorded;
  std::vector<double> dt;
  bool share_vflux = false;   // every slot reads slot 0's volume fluxes (fct_tape_share_vflux)
};

namespace {

constexpr int B = 256;
// Resident 256-thread blocks per SM the reverse kernels' register allocation must allow
// (40 registers; 48 for r_edge). The kernels are latency-bound gathers, so resident warps
// pay more than the spills the cap costs: on the CORE2-size 10-step chain the reverse
// passes took 28.7 ms unconstrained (r_edge at 3 blocks), 23.3 ms at 4 blocks, 20.2 ms at
// 6 (r_edge 5) and 20.0 ms at 8.
constexpr int kRevMinBlocks = 6;
constexpr int kRevEdgeMinBlocks = 5;

__device__ __forceinline__ int64_t lane_index() {
  return int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
}
template <class T>
__device__ __forceinline__ T ld(const T* p) { return __ldg(p); }
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
// k in [r & 255, (r >> 8) & 255) (packed level ranges of the mesh slots)
__device__ __forceinline__ bool in_range(int k, unsigned r) {
  return k >= int(r & 255u) && k < int((r >> 8) & 255u);
}

// accumulate flags of fct_adjoint_ex
constexpr int kAccT = 1, kAccTo = 2, kAccUV = 4, kAccW = 8;
// FCT_ADJ_DEFER_UV: the volume-flux cotangents go into the plan's running sum instead of
// being transposed into guv by this call
constexpr int kDeferUV = 16;

struct Adj {
  Inst in;               // forward fields + forward workspace (recomputed or taped)
  AdjWorkspace a;
  const double* gTn;     // cotangent of T_new (tracer-major, in.tstride)
  double *gT, *gTo, *guv, *gw;
  int acc;               // kAcc* bits: add into the output instead of overwriting it
};

// Cotangent reaching the limited vertical flux at interface j of a node column, from the
// stored divergence cotangents ghsc = gdel * dt / sa (sa = areasvol, 1 where it is 0): the
// flux enters layer j's update with +dt/areasvol and layer j-1's with -dt/areasvol, each
// only where that layer exists and areasvol > 0 (flux2dtracer_fct, tracer_adv.py:476-479).
__device__ __forceinline__ double gvl_at(const DevMesh& m, const double* ghsc, int64_t base,
                                        int j, int nzmin, int nzmax) {
  double g = 0.0;
  if (j >= nzmin && j < nzmax && ld(m.areasvol + base + j) > 0.0) g += ghsc[base + j];
  if (j - 1 >= nzmin && j - 1 < nzmax && ld(m.areasvol + base + j - 1) > 0.0)
    g -= ghsc[base + j - 1];
  return g;
}

// ------------------------------------------------------------------ r_seed
// T_new = T + d / hnn (d = del + T (hn - hnn)) and del holds the flux divergence times
// dt / areasvol: stores the cotangent of a node's flux divergence, gdel * dt / sa.
__global__ void __launch_bounds__(B, kRevMinBlocks) r_seed(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t li = lane_index();
  if (li >= m.n_layer) return;
  const uint32_t lane = ld(m.layer_lanes + li);
  const uint32_t i = lq(lane_ent(lane), m.L, lane_lev(lane));
  const double hnn = ld(in.hnode_new + i), av = ld(m.areasvol + i);
  const double sa = av > 0.0 ? av : 1.0;
  for (int t = 0; t < in.ntr; ++t) {
    const double g = ld(A.gTn + t * in.tstride + i);
    double gdel = 0.0;
    if (hnn > 0.0) gdel = g / hnn;
    A.a.ghsc[t * A.a.sN + i] = gdel * in.dt / sa;
  }
}

// ------------------------------------------------------------------ r_dry
// Dry levels keep T (T_new = T, ale_reconstruct): their outputs depend only on dT_new and
// are final here, except dT at the level above a cavity's first layer, which the upwind
// flux of interface nzmin also reaches (r_final writes it); gw_e is zero there.
__global__ void __launch_bounds__(B, kRevMinBlocks) r_dry(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t li = lane_index();
  const int L = m.L;
  if (li >= m.n_dry) return;
  const uint32_t lane = ld(m.dry_lanes + li);
  const int n = lane_ent(lane), k = lane_lev(lane);
  const int64_t i = lq(n, L, k);
  const int nzmin = ld(m.nzmin + n), nzmax = ld(m.nzmax + n);
  const bool above_cavity = k + 1 == nzmin && nzmin < nzmax;
  const double gA = 0.0;
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t oT = t * in.tstride + i;
    if (!above_cavity) {
      const double vT = (ld(A.gTn + oT) + 0.0) + kAbNew * gA;
      A.gT[oT] = (A.acc & kAccT) ? A.gT[oT] + vT : vT;
    }
    const double vTo = kAbOld * gA;
    A.gTo[oT] = (A.acc & kAccTo) ? A.gTo[oT] + vTo : vTo;
  }
  double g = 0.0;   // dL/dw_e summed over tracers (the workspace's zeros at dry levels)
  for (int t = 0; t < in.ntr; ++t) g += A.a.gw[t * A.a.sN + i];
  A.gw[i] = (A.acc & kAccW) ? A.gw[i] + g : g;
}

// ------------------------------- cotangents of the limiter factors pf, mf at (n, k)
// (zalesak_limit b3, tracer_adv.py:453-465): the limited vertical fluxes at interfaces k
// and k+1 and the limited horizontal fluxes of the incident edges in ascending edge id.
__device__ __forceinline__ void factor_cotangents(const Adj& A, int t, int n, int k, int nzmin,
                                                  int nzmax, int e0, int e1, double& gp,
                                                  double& gm) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int L = m.L;
  const uint32_t base = lq(n, L, 0), qn = base + uint32_t(k);
  const int64_t o = t * in.ws.sN;
  const double* pf = in.ws.pf + o;
  const double* mf = in.ws.mf + o;
  const double* adfv = in.ws.adfv + o;
  const double* ghsc = A.a.ghsc + t * A.a.sN;
  const double pfk = pf[qn], mfk = mf[qn];
  gp = 0.0;
  gm = 0.0;
  // vertical limited flux at interface k (this node's own factors at k)
  {
    const double f = adfv[qn];
    const double g_ae = gvl_at(m, ghsc, base, k, nzmin, nzmax) * f;
    if (k == nzmin) {
      if (f >= 0.0) gp += g_ae; else gm += g_ae;
    } else if (f >= 0.0) {
      gp += g_ae * smin_b(mf[qn - 1], pfk);
    } else {
      gm += g_ae * smin_b(pf[qn - 1], mfk);
    }
  }
  // vertical limited flux at interface k+1 (uses this node's factors as the k-1 ones)
  if (k + 1 < nzmax) {
    const double f = adfv[qn + 1];
    const double g_ae = gvl_at(m, ghsc, base, k + 1, nzmin, nzmax) * f;
    if (f >= 0.0) gm += g_ae * smin_a(mfk, pf[qn + 1]);
    else gp += g_ae * smin_a(pfk, mf[qn + 1]);
  }
  // horizontal limited fluxes of the incident edges, ascending edge id; the loads are
  // unconditional (all in bounds) and edges without a flux at k are selected away
  const double ghsc0 = ghsc[qn];
  const double* adfh = in.ws.adfh + t * in.ws.sEd;
#pragma unroll 2
  for (int j = e0; j < e1; ++j) {
    const int4 sl = __ldg(m.ne4 + j);
    const bool on = in_range(k, unsigned(sl.z));
    const bool second = sl.x & 1;
    const uint32_t qo = lq(sl.y, L, k);
    const double ghsco = ghsc[qo];
    const double glim = second ? (ghsco - ghsc0) : (ghsc0 - ghsco);
    const double a = adfh[lq(sl.x >> 1, L, k)];
    const double g_ae = glim * a;
    const double pfo = pf[qo], mfo = mf[qo];
    const double pf1 = second ? pfo : pfk, mf1 = second ? mfo : mfk;
    const double pf2 = second ? pfk : pfo, mf2 = second ? mfk : mfo;
    double dp = 0.0, dm = 0.0;
    bool tp = false, tm = false;
    if (a >= 0.0) {   // ae = min(pf[n1], mf[n2])
      if (!second) { dp = g_ae * smin_a(pf1, mf2); tp = true; }
      else { dm = g_ae * smin_b(pf1, mf2); tm = true; }
    } else {          // ae = min(mf[n1], pf[n2])
      if (!second) { dm = g_ae * smin_a(mf1, pf2); tm = true; }
      else { dp = g_ae * smin_b(mf1, pf2); tp = true; }
    }
    gp = (on && tp) ? gp + dp : gp;
    gm = (on && tm) ? gm + dm : gm;
  }
}

// ---------------- r_ratio_window: the factor cotangents (b3), pf = min(1, fmax_w /
// flux_pos) and likewise mf (b2), the a4 window (max/min over the cluster bounds at k-1, k,
// k+1 of the same column), and the a3 share of each cell that attains the node's cluster
// bound.
// Blocks of B threads cover B - 2 lanes plus one halo lane on each side: every thread
// computes its lane's window cotangents (gtmax, gtmin) into shared memory, and the core
// lanes spread them back over the window's three levels (lanes i-1, i, i+1).
__global__ void __launch_bounds__(B, kRevMinBlocks) r_ratio_window(Adj A) {
  __shared__ double sx[B], sn[B];
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int tid = threadIdx.x;
  const int64_t lane = int64_t(blockIdx.x) * (B - 2) + tid - 1;
  const bool valid = lane >= 0 && lane < m.n_layer;
  const bool core = valid && tid >= 1 && tid <= B - 2;
  const int L = m.L;
  int n = 0, k = 0, nzmin = 0, nzmax = 0, e0 = 0, e1 = 0;
  uint32_t base = 0, qn = 0;
  bool valid_n = false, use_own = true;
  Rcp rsa{1.0, 1.0, true}, rsh{1.0, 1.0, true};
  if (valid) {
    const int4 rec = __ldg(m.layer4 + lane);
    const unsigned pk = unsigned(rec.w);
    n = lane_ent(uint32_t(rec.x));
    k = lane_lev(uint32_t(rec.x));
    nzmin = int(pk & 255u);
    nzmax = int((pk >> 8) & 255u);
    e0 = rec.y;
    e1 = rec.y + int((pk >> 16) & 255u);
    base = lq(n, L, 0);
    qn = base + uint32_t(k);
    const double av = ld(m.areasvol + qn), hnn = ld(in.hnode_new + qn);
    valid_n = (av > 0.0) && (hnn > 0.0);
    rsa = rcp(av > 0.0 ? av : 1.0);
    rsh = rcp(hnn > 0.0 ? hnn : 1.0);
    use_own = (k == nzmin) || (k == nzmax - 1);
  }
  const double dt = in.dt;
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t o = t * in.ws.sN, oa = t * A.a.sN;
    const double* tv = in.ws.tvmax + o;
    const double* tn = in.ws.tvmin + o;
    double gtmax = 0.0, gtmin = 0.0;
    if (valid) {
      double gpf, gmf;
      factor_cotangents(A, t, n, k, nzmin, nzmax, e0, e1, gpf, gmf);
      double gplus = 0.0, gminus = 0.0;
      if (valid_n) {
        double tmax = tv[qn], tmin = tn[qn];
        if (!use_own) {
          tmax = fmax(fmax(tv[qn - 1], tv[qn]), tv[qn + 1]);
          tmin = fmin(fmin(tn[qn - 1], tn[qn]), tn[qn + 1]);
        }
        const double lo = in.ws.lo[o + qn];
        const double plus = in.ws.fplus[o + qn], minus = in.ws.fminus[o + qn];
        const double fmax_w = tmax - lo, fmin_w = tmin - lo;
        const double flux_pos = divr(divr(plus * dt, rsa), rsh) + kFluxEps;
        const double flux_neg = divr(divr(minus * dt, rsa), rsh) - kFluxEps;
        const Rcp rfp = rcp(flux_pos), rfn = rcp(flux_neg);
        const double rp = divr(fmax_w, rfp), rm = divr(fmin_w, rfn);
        const double grp = gpf * smin_b(1.0, rp);
        const double grm = gmf * smin_b(1.0, rm);
        gtmax = divr(grp, rfp);
        gtmin = divr(grm, rfn);
        gplus = divr(divr(-grp * fmax_w / (flux_pos * flux_pos) * dt, rsa), rsh);
        gminus = divr(divr(-grm * fmin_w / (flux_neg * flux_neg) * dt, rsa), rsh);
      }
      if (core) {
        A.a.gplus[oa + qn] = gplus;
        A.a.gminus[oa + qn] = gminus;
        A.a.gLOl[oa + qn] = -(gtmax + gtmin);
      }
    }
    sx[tid] = gtmax;
    sn[tid] = gtmin;
    __syncthreads();
    if (core) {
      const double* tvc = tv + base;
      const double* tnc = tn + base;
      double gvx = 0.0, gvn = 0.0;
      for (int mm = k - 1; mm <= k + 1; ++mm) {
        if (mm < nzmin || mm >= nzmax) continue;
        const int sl = tid + (mm - k);   // lane of level mm (same column)
        if (mm == nzmin || mm == nzmax - 1) {
          if (mm == k) { gvx += sx[sl]; gvn += sn[sl]; }
          continue;
        }
        {  // max(max(a, b), c) with a = tv[mm-1], b = tv[mm], c = tv[mm+1]
          const double a = tvc[mm - 1], b = tvc[mm], c = tvc[mm + 1];
          const double inner = fmax(a, b), go = sx[sl];
          const double gi = go * smax_a(inner, c), gc = go * smax_b(inner, c);
          if (k == mm - 1) gvx += gi * smax_a(a, b);
          if (k == mm) gvx += gi * smax_b(a, b);
          if (k == mm + 1) gvx += gc;
        }
        {
          const double a = tnc[mm - 1], b = tnc[mm], c = tnc[mm + 1];
          const double inner = fmin(a, b), go = sn[sl];
          const double gi = go * smin_a(inner, c), gc = go * smin_b(inner, c);
          if (k == mm - 1) gvn += gi * smin_a(a, b);
          if (k == mm) gvn += gi * smin_b(a, b);
          if (k == mm + 1) gvn += gc;
        }
      }
      // one tied cell's share of the cluster bound (a3's even split over the cells that
      // attain it; a node layer has at least one such cell)
      const int cx = int(in.ws.ccx[o + qn]), cn = int(in.ws.ccn[o + qn]);
      A.a.gqx[oa + qn] = cx > 0 ? divr(gvx, rcp(double(cx))) : 0.0;
      A.a.gqn[oa + qn] = cn > 0 ? divr(gvn, rcp(double(cn))) : 0.0;
    }
    __syncthreads();
  }
}

// ------- r_cluster: a2 element max/min over its vertices, cotangent spread evenly over
// the tied vertices, of the a3 shares of the vertices whose cluster bound the element
// attains (tie counts come from the forward). Stored already divided by the element's
// vertex tie count: the share of each attaining vertex.
__global__ void __launch_bounds__(B, kRevMinBlocks) r_cluster(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_elem) return;
  const uint32_t lane = ld(m.elem_lanes + i);
  const int e = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const uint32_t qe = lq(e, L, k);
  const uint32_t qv[3] = {lq(ld(m.enodes + 3 * e), L, k),
                         lq(ld(m.enodes + 3 * e + 1), L, k),
                         lq(ld(m.enodes + 3 * e + 2), L, k)};
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t o = t * in.ws.sN, oa = t * A.a.sN, oe = t * in.ws.sE;
    const double vx = in.ws.amax[oe + qe], vn = in.ws.amin[oe + qe];
    double tx[3], tn[3], qx[3], qn[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      tx[v] = in.ws.tvmax[o + qv[v]];
      tn[v] = in.ws.tvmin[o + qv[v]];
      qx[v] = A.a.gqx[oa + qv[v]];
      qn[v] = A.a.gqn[oa + qv[v]];
    }
    double gx = 0.0, gn = 0.0;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      gx = vx == tx[v] ? gx + qx[v] : gx;
      gn = vn == tn[v] ? gn + qn[v] : gn;
    }
    A.a.gax[t * A.a.sE + qe] = divr(gx, rcp(double(int(in.ws.ecx[oe + qe]))));
    A.a.gan[t * A.a.sE + qe] = divr(gn, rcp(double(int(in.ws.ecn[oe + qe]))));
  }
}

// ------- r_bounds_lo: a1 (max/min of LO and T) gathering the element shares of the
// node's cells whose bound this node attains, then LO = numer / hnn and the seed terms
// of T and LO.
__global__ void __launch_bounds__(B, kRevMinBlocks) r_bounds_lo(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_layer) return;
  const int4 rec = __ldg(m.layer4 + i);
  const unsigned pk = unsigned(rec.w);
  const int n = lane_ent(uint32_t(rec.x)), k = lane_lev(uint32_t(rec.x)), L = m.L;
  const uint32_t qn = lq(n, L, k);
  const double hn = ld(in.hnode + qn), hnn = ld(in.hnode_new + qn), av = ld(m.areasvol + qn);
  const bool valid = (hnn > 0.0) && (av > 0.0);
  const int c0 = rec.z, c1 = rec.z + int(pk >> 24);
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t o = t * in.ws.sN, oa = t * A.a.sN, oe = t * in.ws.sE, ae = t * A.a.sE;
    const double lo = in.ws.lo[o + qn], T = ld(in.T + t * in.tstride + qn);
    const double mxv = fmax(lo, T), mnv = fmin(lo, T);
    double gx = 0.0, gn = 0.0;
    // the node's cells in nod_in_elem2D order; loads are unconditional (in bounds) and
    // cells dry at k are selected away
#pragma unroll 2
    for (int j = c0; j < c1; ++j) {
      const bool on = in_range(k, unsigned(ld(m.nelr + j)));
      const uint32_t qe = lq(ld(m.nel_idx + j), L, k);
      const double ex = in.ws.amax[oe + qe], en = in.ws.amin[oe + qe];
      const double sx = A.a.gax[ae + qe], sn = A.a.gan[ae + qe];
      gx = (on && mxv == ex) ? gx + sx : gx;
      gn = (on && mnv == en) ? gn + sn : gn;
    }
    const double gLOb = gx * smax_a(lo, T) + gn * smin_a(lo, T);
    const double gTb = gx * smax_b(lo, T) + gn * smin_b(lo, T);
    // seed: T_new = T + d / hnn, d = (-T hn + LO hnn) + fluxes + T (hn - hnn)
    const double g = ld(A.gTn + t * in.tstride + qn);
    double gTs = g, gdel = 0.0;
    if (hnn > 0.0) {
      gdel = g / hnn;
      gTs += gdel * (hn - hnn);
    }
    gTs += -gdel * hn;
    const double gLO = gdel * hnn + A.a.gLOl[oa + qn] + gLOb;
    double gdiv = 0.0, gT = gTs + gTb;
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
__global__ void __launch_bounds__(B, kRevEdgeMinBlocks) r_edge(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_edge) return;
  const int4 rec = __ldg(m.edge4 + i);
  const int e = lane_ent(uint32_t(rec.x)), k = lane_lev(uint32_t(rec.x)), L = m.L;
  const int n1 = rec.y, n2 = rec.z;
  const bool use_tri = in_range(k, unsigned(rec.w));
  const uint32_t qe = lq(e, L, k), q1 = lq(n1, L, k), q2 = lq(n2, L, k);
  uint32_t qa = q1, qb = q2;   // where the MFCT gradients are read
  if (use_tri) {
    qa = lq(ld(m.eupdn + 2 * e), L, k);
    qb = lq(ld(m.eupdn + 2 * e + 1), L, k);
  }
  const double vf = ld(in.ws.vflux + qe), avf = fabs(vf), s = sgn(vf);
  const double c1 = ld(m.ecoef + 2 * e), c2 = ld(m.ecoef + 2 * e + 1);
  const Rcp r6{6.0, 1.0 / 6.0, true};
  double gvf_t = 0.0;   // summed over tracers in tracer order, as r_uv sums them
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t o = t * in.ws.sN, oa = t * A.a.sN, oe = t * A.a.sEd;
    const double a = in.ws.adfh[t * in.ws.sEd + qe];
    // limited flux lim = ae * a, with hsc(n1) += lim, hsc(n2) -= lim
    const double glim = A.a.ghsc[oa + q1] - A.a.ghsc[oa + q2];
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
    const double* T = in.T + t * in.tstride;
    const double* To = in.T_old + t * in.tstride;
    const double T1 = ld(T + q1), T2 = ld(T + q2);
    const double A1 = ab2(T1, ld(To + q1)), A2 = ab2(T2, ld(To + q2));
    // MFCT gradients: the up/down cells' (use_tri) or the two nodes' averages
    const double* gxp = use_tri ? in.ws.gx + t * in.ws.sE : in.ws.gnx + o;
    const double* gyp = use_tri ? in.ws.gy + t * in.ws.sE : in.ws.gny + o;
    const double g0 = gxp[qa], g1 = gxp[qb], g2 = gyp[qa], g3 = gyp[qb];
    const double diff = A2 - A1;
    const double Tm1 = A1 + divr(2.0 * diff + c1 * g0 + c2 * g2, r6);
    const double Tm2 = A2 - divr(2.0 * diff + c1 * g1 + c2 * g3, r6);
    // HO = -0.5 ((vf + |vf|) Tm1 + (vf - |vf|) Tm2); fl = -0.5 (T1 (vf + |vf|) + T2 (vf - |vf|))
    double gvf = -0.5 * ((1.0 + s) * Tm1 + (1.0 - s) * Tm2) * gHO;
    gvf += -0.5 * (T1 * (1.0 + s) + T2 * (1.0 - s)) * gfl;
    if (!(A.acc & kDeferUV)) A.a.gvf[oe + qe] = gvf;   // r_uv's input (not run when deferred)
    gvf_t += gvf;
    // per-end terms for the node and element gathers: T1/T2 through the upwind flux;
    // ttfAB at the ends through Tm1 = A1 + X1 / 6 and Tm2 = A2 - X2 / 6 with
    // X = 2 (A2 - A1) + c1 gx + c2 gy (so the gradients' factors are c1 gX, c2 gX)
    const double gTm1 = -0.5 * (vf + avf) * gHO, gTm2 = -0.5 * (vf - avf) * gHO;
    const double gX1 = divr(gTm1, r6), gX2 = divr(-gTm2, r6);
    const double gdiff = 2.0 * gX1 + 2.0 * gX2;
    A.a.gT1[oe + qe] = -0.5 * (vf + avf) * gfl;
    A.a.gT2[oe + qe] = -0.5 * (vf - avf) * gfl;
    A.a.gA1[oe + qe] = gTm1 - gdiff;
    A.a.gA2[oe + qe] = gTm2 + gdiff;
    A.a.gX1[oe + qe] = gX1;
    A.a.gX2[oe + qe] = gX2;
  }
  if (A.acc & kDeferUV) A.a.gvf_sum[qe] += gvf_t;   // one thread per edge level: no race
}

// QR4C stencil depths of interface j (tracer_adv.py:228-238, 265-273)
__device__ __forceinline__ void qr4c_depths(const Inst& in, const DevMesh& m, int64_t base,
                                            int j, double& Znz, double& Zm1, double& Zm2,
                                            double& Zp1, double& zb) {
  const int L = m.L;
  if (in.Z3d) {
    const double* Zc = in.Z3d + base;
    Znz = ld(Zc + j); Zm1 = ld(Zc + j - 1); Zm2 = ld(Zc + j - 2);
    Zp1 = ld(Zc + (j + 1 < L ? j + 1 : L - 1));
    zb = ld(in.zbar3 + base + j);
  } else {
    Znz = ld(m.Zp + j); Zm1 = ld(m.Zp + j - 1); Zm2 = ld(m.Zp + j - 2);
    Zp1 = ld(m.Zp + (j + 1 < L ? j + 1 : L - 1));
    zb = ld(m.zbar + j);
  }
}

// ------- r_gnode: cotangent of the node-average gradient (fill_up_dn_grad's node branch),
// gathered over the node's edges in ascending edge id.
__global__ void __launch_bounds__(B, kRevMinBlocks) r_gnode(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_layer) return;
  const int4 rec = __ldg(m.layer4 + i);
  const unsigned pk = unsigned(rec.w);
  const int n = lane_ent(uint32_t(rec.x)), k = lane_lev(uint32_t(rec.x)), L = m.L;
  const uint32_t qn = lq(n, L, k);
  const int e0 = rec.y, e1 = rec.y + int((pk >> 16) & 255u);
  // no edge of the node takes the node-average gradient at k (kGradBit): its cotangent is 0
  const int nzmin = int(pk & 255u);
  const bool grad = (__ldg(m.nflags + __ldg(m.nrec + n).w + (k - nzmin)) >> kGradBit) & 1ull;
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t oa = t * A.a.sN, oe = t * A.a.sEd;
    double gx = 0.0, gy = 0.0;
#pragma unroll 2
    for (int j = grad ? e0 : e1; j < e1; ++j) {   // loads unconditional (in bounds), off edges selected away
      const int4 sl = __ldg(m.ne4 + j);
      const int e = sl.x >> 1;
      const bool on = in_range(k, unsigned(sl.z)) && !in_range(k, unsigned(ld(m.etr + e)));
      const bool second = sl.x & 1;
      const double x = (second ? A.a.gX2 : A.a.gX1)[oe + lq(e, L, k)];
      const double c1 = ld(m.ecoef + 2 * e), c2 = ld(m.ecoef + 2 * e + 1);
      gx = on ? gx + c1 * x : gx;
      gy = on ? gy + c2 * x : gy;
    }
    A.a.ggnx[oa + qn] = gx;
    A.a.ggny[oa + qn] = gy;
  }
}

// ------- r_vert: the vertical fluxes at interface j = k: gf of adf_v[j] (limiter
// application and the plus/minus sums) reaches the QR4C flux (ghi = gf) and the upwind
// flux (gfv = -gf + gdiv terms); gw[j] is complete here (only interface j feeds it), and
// the QR4C flux's terms for ttfAB at levels j, j-1, j-2 and j+1 are stored for r_final to
// gather. Independent of the edge chain (it runs beside r_edge).
__global__ void __launch_bounds__(B, kRevMinBlocks) r_vert(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_layer) return;
  const int4 rec = __ldg(m.layer4 + i);
  const unsigned pk = unsigned(rec.w);
  const int n = lane_ent(uint32_t(rec.x)), j = lane_lev(uint32_t(rec.x)), L = m.L;
  const int nzmin = int(pk & 255u), nzmax = int((pk >> 8) & 255u);
  const uint32_t base = lq(n, L, 0), qn = base + uint32_t(j);
  const double w = ld(in.w_e + qn), area = ld(m.area + qn);
  const int jm = j > 0 ? j - 1 : 0;
  const Rcp r3{3.0, 1.0 / 3.0, true};
  const bool interior = j >= nzmin + 2 && j <= nzmax - 2;
  double Znz = 0.0, Zm1 = 0.0, Zm2 = 0.0, Zp1 = 0.0, zb = 0.0;
  Rcp rdc{1.0, 1.0, true}, rdu{1.0, 1.0, true}, rdd{1.0, 1.0, true};
  if (interior) {
    qr4c_depths(in, m, base, j, Znz, Zm1, Zm2, Zp1, zb);
    rdc = rcp(safe_nz(Zm1 - Znz));
    rdu = rcp(safe_nz(Znz - Zp1));
    rdd = rcp(safe_nz(Zm2 - Zm1));
  }
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t o = t * in.ws.sN, oa = t * A.a.sN;
    const double* T = in.T + t * in.tstride + base;
    const double* To = in.T_old + t * in.tstride + base;
    const double* pf = in.ws.pf + o + base;
    const double* mf = in.ws.mf + o + base;
    const double* gplus = A.a.gplus + oa + base;
    const double* gminus = A.a.gminus + oa + base;
    const double* gdiv = A.a.gdiv + oa + base;
    const double f = in.ws.adfv[o + qn];
    double ae;
    if (j == nzmin) ae = f >= 0.0 ? pf[j] : mf[j];
    else ae = f >= 0.0 ? fmin(mf[j - 1], pf[j]) : fmin(pf[j - 1], mf[j]);
    double gf = gvl_at(m, A.a.ghsc + oa, base, j, nzmin, nzmax) * ae;
    gf += gplus[j] * dmax0(f) + gminus[j] * dmin0(f);
    if (j - 1 >= nzmin) gf -= gplus[j - 1] * dmax0(-f) + gminus[j - 1] * dmin0(-f);
    const double ghi = gf;
    double gfv = -gf + gdiv[j];
    if (j - 1 >= nzmin) gfv -= gdiv[j - 1];
    A.a.gfv[oa + qn] = gfv;
    double gw = 0.0;
    gw += -0.5 * (ld(T + j) * (1.0 + sgn(w)) + ld(T + jm) * (1.0 - sgn(w))) * area * gfv;
    // QR4C (tracer_adv.py:241-295): surface, next-to-surface / next-to-bottom, interior
    double z0 = 0.0, zm1 = 0.0, zm2 = 0.0, zp1 = 0.0;
    if (j == nzmin) {
      gw += -ab2(ld(T + j), ld(To + j)) * area * ghi;
      z0 = -w * area * ghi;
    } else if (j == nzmin + 1 || j == nzmax - 1) {
      gw += -0.5 * (ab2(ld(T + j - 1), ld(To + j - 1)) + ab2(ld(T + j), ld(To + j))) * area * ghi;
      z0 = zm1 = -0.5 * w * area * ghi;
    } else if (interior) {
      const double A0 = ab2(ld(T + j), ld(To + j)), Am1 = ab2(ld(T + j - 1), ld(To + j - 1));
      const double Am2 = ab2(ld(T + j - 2), ld(To + j - 2)), Ap1 = ab2(ld(T + j + 1), ld(To + j + 1));
      const double qc = divr(Am1 - A0, rdc), qu = divr(A0 - Ap1, rdu), qd = divr(Am2 - Am1, rdd);
      const double Tmean1 = A0 + divr((2.0 * qc + qu) * (zb - Znz), r3);
      const double Tmean2 = Am1 + divr((2.0 * qc + qd) * (zb - Zm1), r3);
      gw += -0.5 * (Tmean1 + Tmean2) * area * ghi;
      // Tmean1 = A0 + (2 qc + qu) (zb - Z[j]) / 3, Tmean2 = Am1 + (2 qc + qd) (zb - Z[j-1]) / 3
      const double gS = -0.5 * w * area * ghi;
      const double gq1 = divr(gS * (zb - Znz), r3), gq2 = divr(gS * (zb - Zm1), r3);
      const double gqc = 2.0 * gq1 + 2.0 * gq2, gqu = gq1, gqd = gq2;
      z0 = gS - divr(gqc, rdc) + divr(gqu, rdu);
      zm1 = gS + divr(gqc, rdc) - divr(gqd, rdd);
      zm2 = divr(gqd, rdd);
      zp1 = -divr(gqu, rdu);
    }
    A.a.gw[oa + qn] = gw;
    A.a.gz0[oa + qn] = z0;
    A.a.gzm1[oa + qn] = zm1;
    A.a.gzm2[oa + qn] = zm2;
    A.a.gzp1[oa + qn] = zp1;
  }
}

// ---------------- r_tr: cotangent of the element gradients (up/dn use + node average)
__global__ void __launch_bounds__(B, kRevMinBlocks) r_tr(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t i = lane_index();
  if (i >= m.n_elem) return;
  const uint32_t lane = ld(m.elem_lanes + i);
  const int el = lane_ent(lane), k = lane_lev(lane), L = m.L;
  const double aw = ld(m.earea + el);
  const int u0 = ld(m.eud_off + el), u1 = ld(m.eud_off + el + 1);
  const uint32_t qv[3] = {lq(ld(m.enodes + 3 * el), L, k),
                         lq(ld(m.enodes + 3 * el + 1), L, k),
                         lq(ld(m.enodes + 3 * el + 2), L, k)};
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t oa = t * A.a.sN, oe = t * A.a.sEd;
    double gx = 0.0, gy = 0.0;
#pragma unroll 2
    for (int j = u0; j < u1; ++j) {   // edges using el as up (slot 0) or down (1) cell
      const int idx = ld(m.eud_idx + j), e = idx >> 1;
      const bool on = in_range(k, unsigned(ld(m.etr + e)));
      // the down (slot 1) / up (slot 0) cell's gradient enters Tm2 / Tm1
      const double x = ((idx & 1) ? A.a.gX2 : A.a.gX1)[oe + lq(e, L, k)];
      const double c1 = ld(m.ecoef + 2 * e), c2 = ld(m.ecoef + 2 * e + 1);
      gx = on ? gx + c1 * x : gx;
      gy = on ? gy + c2 * x : gy;
    }
#pragma unroll
    for (int v = 0; v < 3; ++v) {   // gnode(n) = sum_e a_e tr_e / den(n)
      // the cotangent is nonzero only at levels where an edge of the vertex takes the
      // node-average gradient, the only levels whose denominator the forward stored
      const double cx = A.a.ggnx[oa + qv[v]], cy = A.a.ggny[oa + qv[v]];
      if (cx != 0.0 || cy != 0.0) {
        const double dd = in.ws.nden[qv[v]];   // the forward's (safe) denominator
        gx += cx * aw / dd;
        gy += cy * aw / dd;
      }
    }
    A.a.gtrx[t * A.a.sE + lq(el, L, k)] = gx;
    A.a.gtry[t * A.a.sE + lq(el, L, k)] = gy;
  }
}

// --------------- r_final: dT and dT_old at every wet layer (tracer_ab: ttfAB = -0.6 T_old
// + 1.6 T), gathering: the seed/LO/bounds terms (gTp); the element gradients on T over
// the node's cells (tracer_gradient_elements transposed); the vertical upwind flux of
// interfaces k and k+1 on T, and the QR4C fluxes of interfaces k-1 .. k+2 on ttfAB in
// ascending interface order; the edge terms in ascending edge id. Also sums gw_e over the
// tracers, and writes dT at the dry level above a cavity's first layer (only the
// (w - |w|) upwind term of interface nzmin reaches it; r_seed wrote the other dry levels).
__global__ void __launch_bounds__(B, kRevMinBlocks) r_final(Adj A) {
  const Inst& in = A.in;
  const DevMesh& m = *in.m;
  const int64_t li = lane_index();
  if (li >= m.n_layer) return;
  const int4 rec = __ldg(m.layer4 + li);
  const unsigned pk = unsigned(rec.w);
  const int n = lane_ent(uint32_t(rec.x)), k = lane_lev(uint32_t(rec.x)), L = m.L;
  const int64_t i = lq(n, L, k);
  const int nzmin = int(pk & 255u), nzmax = int((pk >> 8) & 255u);
  const int e0 = rec.y, e1 = rec.y + int((pk >> 16) & 255u);
  const int c0 = rec.z, c1 = rec.z + int(pk >> 24);
  for (int t = 0; t < in.ntr; ++t) {
    const int64_t oa = t * A.a.sN;
    const double* gfv = A.a.gfv + oa;
    if (k == nzmin && k > 0) {   // the dry level above a cavity
      const double w = ld(in.w_e + i), area = ld(m.area + i);
      double g = 0.0;
      g += -0.5 * (w - fabs(w)) * area * gfv[i];
      const int64_t oT = t * in.tstride + i - 1;
      const double vT = (ld(A.gTn + oT) + g) + kAbNew * 0.0;
      A.gT[oT] = (A.acc & kAccT) ? A.gT[oT] + vT : vT;
    }
    double gA = 0.0;
    // vertical upwind fluxes of interfaces k and k+1
    double gTv = 0.0;
    {
      const double w = ld(in.w_e + i), area = ld(m.area + i);
      gTv += -0.5 * (w + fabs(w)) * area * gfv[i];
      if (k == 0) gTv += -0.5 * (w - fabs(w)) * area * gfv[i];
    }
    if (k + 1 < nzmax) {
      const double w = ld(in.w_e + i + 1), area = ld(m.area + i + 1);
      gTv += -0.5 * (w - fabs(w)) * area * gfv[i + 1];
    }
    // QR4C terms of interfaces k-1 .. k+2 in ascending order (a term that does not
    // reach k is +0.0; gA starts at +0.0, so adding it changes no bit)
    if (k - 1 >= nzmin) gA += A.a.gzp1[oa + i - 1];
    gA += A.a.gz0[oa + i];
    if (k + 1 < nzmax) gA += A.a.gzm1[oa + i + 1];
    if (k + 2 < nzmax) gA += A.a.gzm2[oa + i + 2];
    // element gradients on T: the node's cells in nod_in_elem2D order
    double gTtr = 0.0;
#pragma unroll 2
    for (int j = c0; j < c1; ++j) {
      const unsigned r = unsigned(ld(m.nelr + j));
      const bool on = in_range(k, r);
      const int el = ld(m.nel_idx + j), iv = int((r >> 16) & 3u);
      const int64_t qe = t * A.a.sE + lq(el, L, k);
      const double v = ld(m.gsca + 6 * el + iv) * A.a.gtrx[qe] +
                       ld(m.gsca + 6 * el + 3 + iv) * A.a.gtry[qe];
      gTtr = on ? gTtr + v : gTtr;
    }
    double gT = A.a.gTp[oa + i] + gTtr + gTv;
#pragma unroll 2
    for (int j = e0; j < e1; ++j) {
      const int4 sl = __ldg(m.ne4 + j);
      const bool on = in_range(k, unsigned(sl.z));
      const bool second = sl.x & 1;
      const int64_t q = t * A.a.sEd + lq(sl.x >> 1, L, k);
      const double vT = (second ? A.a.gT2 : A.a.gT1)[q], vA = (second ? A.a.gA2 : A.a.gA1)[q];
      gT = on ? gT + vT : gT;
      gA = on ? gA + vA : gA;
    }
    const int64_t oT = t * in.tstride + i;
    const double vT = gT + kAbNew * gA, vTo = kAbOld * gA;
    A.gT[oT] = (A.acc & kAccT) ? A.gT[oT] + vT : vT;
    A.gTo[oT] = (A.acc & kAccTo) ? A.gTo[oT] + vTo : vTo;
  }
  double g = 0.0;   // dL/dw_e summed over tracers
  for (int t = 0; t < in.ntr; ++t) g += A.a.gw[t * A.a.sN + i];
  A.gw[i] = (A.acc & kAccW) ? A.gw[i] + g : g;
}

// -------------------------- r_uv: edge_vflux transposed, summed over tracers
// guv at element level i (= el * L + k) from volume-flux cotangents gvf [ntr x Ed*L, sEd
// apart]: the element's three edges in its edge order
__device__ __forceinline__ void uv_transpose(const DevMesh& m, const double* __restrict__ helem,
                                             const double* __restrict__ gvfs, int ntr,
                                             int64_t sEd, double* __restrict__ guv, int acc,
                                             int64_t i) {
  const int L = m.L;
  int el, k;
  split_dense(i, L, el, k);
  double gU = 0.0, gV = 0.0;
  if (k >= ld(m.eul + el) && k < ld(m.enl + el)) {
    const double h = ld(helem + i);
    for (int r = 0; r < 3; ++r) {
      const int ent = ld(m.eedge + 3 * el + r);
      if (ent < 0) continue;
      const int e = ent >> 1;
      const double* cr = m.cross + 4 * int64_t(e);
      double gvf = 0.0;
      for (int t = 0; t < ntr; ++t) gvf += gvfs[t * sEd + lq(e, L, k)];
      if (ent & 1) {   // t2 = (V dx2 - U dy2) h
        gU += -gvf * ld(cr + 3) * h;
        gV += gvf * ld(cr + 2) * h;
      } else {         // t1 = (U dy1 - V dx1) h
        gU += gvf * ld(cr + 1) * h;
        gV += -gvf * ld(cr + 0) * h;
      }
    }
  }
  if (acc & kAccUV) {
    guv[2 * i] += gU;
    guv[2 * i + 1] += gV;
  } else {
    guv[2 * i] = gU;
    guv[2 * i + 1] = gV;
  }
}

__global__ void __launch_bounds__(B, kRevMinBlocks) r_uv(Adj A) {
  const int64_t i = lane_index();
  if (i >= int64_t(A.in.m->E) * A.in.m->L) return;
  uv_transpose(*A.in.m, A.in.helem, A.a.gvf, A.in.ntr, A.a.sEd, A.guv, A.acc, i);
}

// the same transpose of the deferred sum (fct_adjoint_flush_uv)
__global__ void __launch_bounds__(B, kRevMinBlocks) r_uv_sum(const DevMesh* __restrict__ mp,
                                                             const double* __restrict__ helem,
                                                             const double* __restrict__ gvf_sum,
                                                             double* __restrict__ guv,
                                                             int acc) {
  const int64_t i = lane_index();
  if (i >= int64_t(mp->E) * mp->L) return;
  uv_transpose(*mp, helem, gvf_sum, 1, 0, guv, acc, i);
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
  int el, k;
  split_dense(i, L, el, k);
  double gU = 0.0, gV = 0.0;
  if (k >= m.eul[el] && k < m.enl[el]) {
    const double h = helem[i];
    for (int r = 0; r < 3; ++r) {
      const int ent = m.eedge[3 * el + r];
      if (ent < 0) continue;
      const int e = ent >> 1;
      const double* cr = m.cross + 4 * int64_t(e);
      // c = t1 - t2 is added to div at n1 and subtracted at n2
      const double gc = gdiv[lq(m.edges[2 * e], L, k)] - gdiv[lq(m.edges[2 * e + 1], L, k)];
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

// Reverse-pass workspace of `max_tracers` tracers (zeroed: the dry-level entries are
// never written by the reverse kernels and must read as zero).
int reserve_adj_ws(FctPlan* P, int max_tracers) {
  if (max_tracers <= P->adj_tracers) return FCT_OK;
  FCT_CUDA(cudaSetDevice(P->device));
  if (!P->adj_side) {
    FCT_CUDA(cudaStreamCreateWithFlags(&P->adj_side, cudaStreamNonBlocking));
    for (cudaEvent_t& ev : P->adj_ev)
      FCT_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  }
  const int64_t sN = int64_t(P->N) * P->L, sE = int64_t(P->E) * P->L, sEd = int64_t(P->Ed) * P->L;
  const int64_t nd = int64_t(max_tracers) * (kAdjNodeFields * sN + kAdjEdgeFields * sEd +
                                             kAdjElemFields * sE) + sEd;
  double* p = nullptr;
  FCT_CUDA(cudaMalloc(&p, size_t(nd) * sizeof(double)));
  FCT_CUDA(cudaMemset(p, 0, size_t(nd) * sizeof(double)));
  if (P->d_adj) cudaFree(P->d_adj);
  P->d_adj = p;
  AdjWorkspace& a = P->aws;
  a.sN = sN; a.sE = sE; a.sEd = sEd;
  auto take = [&](int64_t n) { double* q = p; p += n * max_tracers; return q; };
  double** node[] = {&a.ghsc, &a.gplus, &a.gminus, &a.gLOl, &a.gqx,
                     &a.gqn, &a.gdiv, &a.gTp, &a.ggnx, &a.ggny, &a.gfv, &a.gw, &a.gz0,
                     &a.gzm1, &a.gzm2, &a.gzp1};
  static_assert(sizeof(node) / sizeof(node[0]) == kAdjNodeFields, "node field count");
  for (double** f : node) *f = take(sN);
  double** edge[] = {&a.gT1, &a.gT2, &a.gA1, &a.gA2, &a.gX1, &a.gX2, &a.gvf};
  static_assert(sizeof(edge) / sizeof(edge[0]) == kAdjEdgeFields, "edge field count");
  for (double** f : edge) *f = take(sEd);
  double** elem[] = {&a.gax, &a.gan, &a.gtrx, &a.gtry};
  static_assert(sizeof(elem) / sizeof(elem[0]) == kAdjElemFields, "elem field count");
  for (double** f : elem) *f = take(sE);
  a.gvf_sum = p;   // zeroed with the rest; fct_adjoint_flush_uv clears it after each use
  P->adj_tracers = max_tracers;
  return FCT_OK;
}

int check_fields(const FctFields* f) {
  if (!f->uv || !f->w_e || !f->helem || !f->hnode || !f->hnode_new || !f->T || !f->T_old)
    return set_error(FCT_ERR_INVALID, "a required field pointer is NULL");
  if (f->w_i) return set_error(FCT_ERR_UNSUPPORTED, "the adjoint does not differentiate w_i");
  if ((f->Z3d == nullptr) != (f->zbar3 == nullptr))
    return set_error(FCT_ERR_INVALID, "Z3d and zbar3 must be given together");
  return FCT_OK;
}

Inst make_inst(const FctPlan* P, const FctFields* f, double dt, int ntr, const Workspace& ws) {
  Inst in{};
  in.m = P->d_mesh;
  in.uv = f->uv; in.w_e = f->w_e; in.helem = f->helem;
  in.hnode = f->hnode; in.hnode_new = f->hnode_new;
  in.T = f->T; in.T_old = f->T_old;
  in.T_new = f->T_new;
  in.tstride = f->tracer_stride ? f->tracer_stride : int64_t(P->N) * P->L;
  in.tg = 0;
  in.wtg = ntr;
  in.Z3d = f->Z3d; in.zbar3 = f->zbar3; in.w_i = nullptr;
  in.ws = ws;
  in.dt = dt;
  in.ntr = ntr;
  return in;
}

LaunchDims unfused_dims(const FctPlan* P, int ntr) {
  LaunchDims d{};
  d.max_iface = P->hm.n_iface; d.max_layer = P->hm.n_layer; d.max_edge = P->hm.n_edge;
  d.max_elem = P->hm.n_elem; d.max_dense = int64_t(P->N) * P->L; d.max_nodes = P->N;
  d.max_dry = P->hm.n_dry;
  d.ntr = ntr; d.chunk = 0; d.per_thread = 8; d.any_wi = false; d.copy_dry = true;
  d.fused = false;   // the reverse kernels read every stage's intermediates
  return d;
}

struct DeviceGuard {
  int prev = -1, dev;
  explicit DeviceGuard(int d) : dev(d) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0 && prev != dev) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" {

int fct_plan_reserve_adjoint(FctPlan* P, int max_tracers) {
  if (!P) return set_error(FCT_ERR_INVALID, "plan is NULL");
  if (max_tracers < 1) return set_error(FCT_ERR_INVALID, "max_tracers must be >= 1");
  int st = plan_reserve_ws(P, max_tracers, /*full=*/true);   // the recompute keeps every field
  if (st) return st;
  return reserve_adj_ws(P, max_tracers);
}

int fct_tape_bytes(const FctPlan* P, int ntr, int steps, int64_t* out) {
  if (!P || !out) return set_error(FCT_ERR_INVALID, "NULL argument");
  if (ntr < 1 || steps < 1) return set_error(FCT_ERR_INVALID, "ntr and steps must be >= 1");
  *out = int64_t(steps) * workspace_doubles(P->N, P->E, P->Ed, P->L, ntr) * int64_t(sizeof(double));
  return FCT_OK;
}

int fct_tape_create(FctPlan* P, int ntr, int steps, void* mem, int64_t bytes, FctTape** out) {
  if (!P || !out) return set_error(FCT_ERR_INVALID, "NULL argument");
  *out = nullptr;
  if (ntr < 1 || steps < 1) return set_error(FCT_ERR_INVALID, "ntr and steps must be >= 1");
  const int64_t per = workspace_doubles(P->N, P->E, P->Ed, P->L, ntr);
  const int64_t need = per * int64_t(steps) * int64_t(sizeof(double));
  if (mem) {
    if (bytes < need)
      return set_error(FCT_ERR_CAPACITY, "tape memory of %lld bytes < %lld needed",
                       (long long)bytes, (long long)need);
    if (reinterpret_cast<uintptr_t>(mem) % 256 != 0)
      return set_error(FCT_ERR_INVALID, "tape memory must be 256-byte aligned");
  }
  DeviceGuard g(P->device);
  int st = reserve_adj_ws(P, ntr);
  if (st) return st;
  double* d = static_cast<double*>(mem);
  if (!d) {
    const cudaError_t e = cudaMalloc(&d, size_t(need));
    if (e != cudaSuccess) {
      cudaGetLastError();
      return set_error(FCT_ERR_CUDA, "tape of %d steps x %d tracers (%.2f GB): %s", steps, ntr,
                       double(need) * 1e-9, cudaGetErrorString(e));
    }
  }
  FctTape* T = new FctTape();
  T->plan = P;
  T->ntr = ntr;
  T->steps = steps;
  T->d = d;
  T->owned = mem == nullptr;
  for (int s = 0; s < steps; ++s)
    T->ws.push_back(carve_workspace(d + per * s, P->N, P->E, P->Ed, P->L, ntr));
  T->recorded.assign(size_t(steps), 0);
  T->dt.assign(size_t(steps), 0.0);
  *out = T;
  return FCT_OK;
}

int fct_tape_share_vflux(FctTape* T) {
  if (!T) return set_error(FCT_ERR_INVALID, "tape is NULL");
  T->share_vflux = true;
  for (size_t s = 1; s < T->ws.size(); ++s) T->ws[s].vflux = T->ws[0].vflux;
  return FCT_OK;
}

int fct_tape_destroy(FctTape* T) {
  if (!T) return FCT_OK;
  DeviceGuard g(T->plan->device);
  if (T->d && T->owned) cudaFree(T->d);
  delete T;
  return FCT_OK;
}

int fct_tape_mark_recorded(FctTape* T, int slot, double dt) {
  if (!T) return set_error(FCT_ERR_INVALID, "tape is NULL");
  if (slot < 0 || slot >= T->steps)
    return set_error(FCT_ERR_INVALID, "slot %d outside the tape's [0, %d)", slot, T->steps);
  if (!(dt > 0.0)) return set_error(FCT_ERR_INVALID, "dt must be positive");
  T->recorded[size_t(slot)] = 1;
  T->dt[size_t(slot)] = dt;
  return FCT_OK;
}

int fct_forward_taped(FctPlan* P, const FctFields* f, double dt, int ntr, FctTape* tape,
                      int slot, fct_stream_t stream) {
  if (!P || !f || !tape) return set_error(FCT_ERR_INVALID, "NULL argument");
  if (tape->plan != P) return set_error(FCT_ERR_INVALID, "the tape belongs to another plan");
  if (ntr < 1 || ntr > tape->ntr)
    return set_error(FCT_ERR_CAPACITY, "ntr=%d outside the tape's [1, %d]", ntr, tape->ntr);
  if (slot < 0 || slot >= tape->steps)
    return set_error(FCT_ERR_INVALID, "slot %d outside the tape's [0, %d)", slot, tape->steps);
  int st = check_fields(f);
  if (st) return st;
  if (!f->T_new) return set_error(FCT_ERR_INVALID, "T_new is NULL");
  if (!(dt > 0.0)) return set_error(FCT_ERR_INVALID, "dt must be positive");
  if (tape->share_vflux && slot > 0 && !tape->recorded[0])
    return set_error(FCT_ERR_INVALID, "a tape sharing its volume fluxes records slot 0 first");
  DeviceGuard g(P->device);
  Inst in = make_inst(P, f, dt, ntr, tape->ws[size_t(slot)]);
  in.nonfinite = P->d_health;
  LaunchDims dims = unfused_dims(P, ntr);
  dims.skip_vflux = tape->share_vflux && slot > 0;   // slot 0's fluxes are this step's
  {
    PlanUse use(P, static_cast<cudaStream_t>(stream));
    st = use.status();
    if (!st) st = launch_forward(in, nullptr, 1, dims, static_cast<cudaStream_t>(stream));
    if (!st) st = use.release();
  }
  if (st) return st;
  tape->recorded[size_t(slot)] = 1;
  tape->dt[size_t(slot)] = dt;
  return FCT_OK;
}

int fct_adjoint_ex(FctPlan* P, const FctFields* f, const double* gT_new, double dt, int ntr,
                   const FctGrads* g, const FctTape* tape, int slot, int accumulate,
                   fct_stream_t stream) {
  if (!P || !f || !g || !gT_new) return set_error(FCT_ERR_INVALID, "NULL argument");
  if (ntr < 1) return set_error(FCT_ERR_INVALID, "ntr must be >= 1");
  if (accumulate & ~(kAccT | kAccTo | kAccUV | kAccW | kDeferUV))
    return set_error(FCT_ERR_INVALID, "unknown accumulate bits 0x%x", accumulate);
  const bool defer_uv = accumulate & kDeferUV;
  if (ntr > P->adj_tracers)
    return set_error(FCT_ERR_CAPACITY, "ntr=%d exceeds the reserved adjoint workspace (%d); "
                     "call fct_plan_reserve_adjoint first", ntr, P->adj_tracers);
  if (tape) {
    if (tape->plan != P) return set_error(FCT_ERR_INVALID, "the tape belongs to another plan");
    if (slot < 0 || slot >= tape->steps)
      return set_error(FCT_ERR_INVALID, "slot %d outside the tape's [0, %d)", slot, tape->steps);
    if (!tape->recorded[size_t(slot)])
      return set_error(FCT_ERR_INVALID, "tape slot %d holds no recorded step", slot);
    if (ntr > tape->ntr)
      return set_error(FCT_ERR_CAPACITY, "ntr=%d exceeds the tape's %d tracers", ntr, tape->ntr);
    if (tape->dt[size_t(slot)] != dt)
      return set_error(FCT_ERR_INVALID, "dt differs from the recorded step's");
  } else if (ntr > P->max_tracers || !P->ws_full) {
    return set_error(FCT_ERR_CAPACITY, "ntr=%d exceeds the reserved recompute workspace; "
                     "call fct_plan_reserve_adjoint first", ntr);
  }
  int st = check_fields(f);
  if (st) return st;
  if (!g->gT || !g->gT_old || (!g->guv && !defer_uv) || !g->gw_e)
    return set_error(FCT_ERR_INVALID, "a gradient output pointer is NULL");
  if (!(dt > 0.0)) return set_error(FCT_ERR_INVALID, "dt must be positive");
  DeviceGuard guard(P->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  PlanUse use(P, s);
  if (use.status()) return use.status();
  Adj A{};
  A.in = make_inst(P, f, dt, ntr, tape ? tape->ws[size_t(slot)] : P->ws);
  A.in.T_new = nullptr;
  A.a = P->aws;
  A.gTn = gT_new;
  A.gT = g->gT; A.gTo = g->gT_old; A.guv = g->guv; A.gw = g->gw_e;
  A.acc = accumulate;
  if (!tape) {   // forward recomputation: every stage except the final update
    LaunchDims d = unfused_dims(P, ntr);
    d.copy_dry = false;
    st = launch_forward_stages(A.in, d, s, /*through_factors=*/true);
    if (st) return st;
  }
  auto grid = [](int64_t lanes, int b) {
    return dim3(unsigned(std::max<int64_t>(1, (lanes + b - 1) / b)));
  };
  const DevMesh& hm = P->hm;
  // Side stream: r_dry (dry levels, needs nothing) from the start; r_vert (needs the
  // node kernels up to r_bounds_lo) beside r_edge; r_uv (needs r_edge's volume-flux
  // cotangents) beside r_gnode / r_tr / r_final. All are latency-bound gathers, so the
  // pairs share the SMs.
  FCT_CUDA(cudaEventRecord(P->adj_ev[0], s));
  FCT_CUDA(cudaStreamWaitEvent(P->adj_side, P->adj_ev[0], 0));
  r_dry<<<grid(hm.n_dry, B), B, 0, P->adj_side>>>(A);
  r_seed<<<grid(hm.n_layer, B), B, 0, s>>>(A);
  r_ratio_window<<<dim3(unsigned(std::max<int64_t>(1, (hm.n_layer + B - 3) / (B - 2)))), B, 0, s>>>(A);
  r_cluster<<<grid(hm.n_elem, B), B, 0, s>>>(A);
  r_bounds_lo<<<grid(hm.n_layer, B), B, 0, s>>>(A);
  FCT_CUDA(cudaEventRecord(P->adj_ev[4], s));
  FCT_CUDA(cudaStreamWaitEvent(P->adj_side, P->adj_ev[4], 0));
  r_vert<<<grid(hm.n_layer, B), B, 0, P->adj_side>>>(A);
  FCT_CUDA(cudaEventRecord(P->adj_ev[1], P->adj_side));
  r_edge<<<grid(hm.n_edge, B), B, 0, s>>>(A);
  if (!defer_uv) {
    FCT_CUDA(cudaEventRecord(P->adj_ev[2], s));
    FCT_CUDA(cudaStreamWaitEvent(P->adj_side, P->adj_ev[2], 0));
    r_uv<<<grid(int64_t(P->E) * P->L, B), B, 0, P->adj_side>>>(A);
  }
  FCT_CUDA(cudaEventRecord(P->adj_ev[3], P->adj_side));
  r_gnode<<<grid(hm.n_layer, B), B, 0, s>>>(A);
  r_tr<<<grid(hm.n_elem, B), B, 0, s>>>(A);
  FCT_CUDA(cudaStreamWaitEvent(s, P->adj_ev[1], 0));
  r_final<<<grid(hm.n_layer, B), B, 0, s>>>(A);
  FCT_CUDA(cudaStreamWaitEvent(s, P->adj_ev[3], 0));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "adjoint kernel launch");
  return use.release();
}

int fct_adjoint(FctPlan* P, const FctFields* f, const double* gT_new, double dt, int ntr,
                const FctGrads* g, fct_stream_t stream) {
  return fct_adjoint_ex(P, f, gT_new, dt, ntr, g, nullptr, 0, 0, stream);
}

int fct_adjoint_flush_uv(FctPlan* P, const double* helem, double* guv, int accumulate,
                         fct_stream_t stream) {
  if (!P || !helem || !guv) return set_error(FCT_ERR_INVALID, "NULL argument");
  if (accumulate != 0 && accumulate != 1)
    return set_error(FCT_ERR_INVALID, "accumulate must be 0 or 1");
  if (P->adj_tracers < 1)
    return set_error(FCT_ERR_CAPACITY, "call fct_plan_reserve_adjoint first");
  DeviceGuard guard(P->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  PlanUse use(P, s);
  if (use.status()) return use.status();
  const int64_t n = int64_t(P->E) * P->L;
  r_uv_sum<<<dim3(unsigned(std::max<int64_t>(1, (n + B - 1) / B))), B, 0, s>>>(
      P->d_mesh, helem, P->aws.gvf_sum, guv, accumulate ? kAccUV : 0);
  FCT_CUDA(cudaMemsetAsync(P->aws.gvf_sum, 0, size_t(P->aws.sEd) * sizeof(double), s));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "uv flush launch");
  return use.release();
}

int fct_compute_w_adjoint(FctPlan* P, const double* gw, const double* helem, double* guv,
                          int accumulate, fct_stream_t stream) {
  if (!P || !gw || !helem || !guv) return set_error(FCT_ERR_INVALID, "NULL argument");
  if (P->adj_tracers < 1)
    return set_error(FCT_ERR_CAPACITY, "call fct_plan_reserve_adjoint first");
  DeviceGuard guard(P->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  PlanUse use(P, s);
  if (use.status()) return use.status();
  double* gdiv = P->aws.gdiv;   // scratch: one node field
  r_w_div<<<unsigned((P->N + 127) / 128), 128, 0, s>>>(P->d_mesh, gw, gdiv);
  const int64_t EL = int64_t(P->E) * P->L;
  r_w_uv<<<unsigned((EL + B - 1) / B), B, 0, s>>>(P->d_mesh, gdiv, helem, guv, accumulate);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? use.release() : cuda_error(e, "compute_w adjoint launch");
}

}  // extern "C"
