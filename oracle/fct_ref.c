/*
 * CPU oracle (test infrastructure only): loop-form C restatement of the reference FCT
 * tracer advection, fesom_jax/tracer_adv.py:532-578, following the stage order of the
 * reference's own loop cross-check fesom_jax/tests/test_tracers.py:325-516.
 *
 * Used as the checker's second opinion (tests compare it with the numpy oracle and the
 * reference-generated golden vectors) and as the timed CPU baseline of bench.py. Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may call it.
 *
 * Parallelism: OpenMP over entities; every edge->node / element->node reduction is a
 * gather over a CSR list in ascending edge/element id, so the sums add the same terms in
 * the same order as the serial edge loop of the reference test, for any thread count.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/fesom_fct.h"

#define R_EARTH 6367500.0      /* fesom_jax/config.py:41 */
#define AB_OLD (-(0.5 + 0.1))  /* tracer_adv.py:44-46 */
#define AB_NEW (1.5 + 0.1)
#define FLUX_EPS 1e-16         /* tracer_adv.py:192 */
#define BIG 1e3                /* tracer_adv.py:193 */

static double dmax(double a, double b) { return a > b ? a : (b > a ? b : a); }
static double dmin(double a, double b) { return a < b ? a : (b < a ? b : a); }
static double safe_nz(double x) { return x == 0.0 ? 1.0 : x; }

typedef struct {
  int *off, *idx; /* node -> incident edges, entry = 2*edge + (node is second) */
} NodeEdges;

static NodeEdges node_edges(const FctMeshDesc* m) {
  NodeEdges r;
  const int N = m->nod2D, Ed = m->edge2D;
  r.off = (int*)calloc((size_t)N + 1, sizeof(int));
  r.idx = (int*)malloc(sizeof(int) * 2 * (size_t)Ed);
  for (int e = 0; e < Ed; ++e) {
    r.off[m->edges[2 * e] + 1]++;
    r.off[m->edges[2 * e + 1] + 1]++;
  }
  for (int n = 0; n < N; ++n) r.off[n + 1] += r.off[n];
  int* fill = (int*)malloc(sizeof(int) * (size_t)N);
  memcpy(fill, r.off, sizeof(int) * (size_t)N);
  for (int e = 0; e < Ed; ++e) {
    r.idx[fill[m->edges[2 * e]]++] = 2 * e;
    r.idx[fill[m->edges[2 * e + 1]]++] = 2 * e + 1;
  }
  free(fill);
  return r;
}

/* One tracer, one FCT step. Z3d/zbar3/w_i may be NULL (the reference's None). */
int oracle_fct_forward(const FctMeshDesc* m, const double* uv, const double* w_e,
                       const double* helem, const double* hnode, const double* hnode_new,
                       const double* T, const double* Told, double* Tnew, double dt,
                       const double* Z3d, const double* zbar3, const double* w_i,
                       int nthreads) {
  const int N = m->nod2D, E = m->elem2D, Ed = m->edge2D, L = m->nl;
  const size_t NL = (size_t)N * L, EL = (size_t)E * L, EdL = (size_t)Ed * L;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  NodeEdges ne = node_edges(m);
  double* ttf = (double*)malloc(sizeof(double) * NL);
  double* vfl = (double*)malloc(sizeof(double) * EdL);
  double* fh = (double*)malloc(sizeof(double) * EdL);
  double* fv = (double*)calloc(NL, sizeof(double));
  double* LO = (double*)calloc(NL, sizeof(double));
  double* tr = (double*)calloc(EL * 2, sizeof(double));
  double* gn = (double*)calloc(NL * 2, sizeof(double));
  double* adfh = (double*)malloc(sizeof(double) * EdL);
  double* adfv = (double*)calloc(NL, sizeof(double));
  double* amax = (double*)malloc(sizeof(double) * EL);
  double* amin = (double*)malloc(sizeof(double) * EL);
  double* tvm = (double*)malloc(sizeof(double) * NL);
  double* tvn = (double*)malloc(sizeof(double) * NL);
  double* pf = (double*)malloc(sizeof(double) * NL);
  double* mf = (double*)malloc(sizeof(double) * NL);
  double* flo = w_i ? (double*)calloc(NL, sizeof(double)) : NULL;
  if (!ttf || !vfl || !fh || !fv || !LO || !tr || !gn || !adfh || !adfv || !amax || !amin ||
      !tvm || !tvn || !pf || !mf || (w_i && !flo))
    return -1;
  double* Zp = (double*)malloc(sizeof(double) * L);
  for (int k = 0; k < L - 1; ++k) Zp[k] = m->Z[k];
  Zp[L - 1] = m->Z[L - 2];

  /* AB2 (tracer_adv.py:59-66) */
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)NL; ++i) ttf[i] = AB_OLD * Told[i] + AB_NEW * T[i];

  /* edge volume flux and LO horizontal flux (tracer_adv.py:69-105) */
#pragma omp parallel for schedule(static)
  for (int e = 0; e < Ed; ++e) {
    const int n1 = m->edges[2 * e], n2 = m->edges[2 * e + 1];
    const int e1 = m->edge_tri[2 * e], e2 = m->edge_tri[2 * e + 1];
    const double* cr = m->edge_cross_dxdy + 4 * (size_t)e;
    for (int k = 0; k < L; ++k) {
      double t1 = 0.0, t2 = 0.0;
      if (e1 >= 0 && k >= m->ulevels[e1] - 1 && k < m->nlevels[e1] - 1) {
        const size_t q = (size_t)e1 * L + k;
        t1 = (uv[2 * q] * cr[1] - uv[2 * q + 1] * cr[0]) * helem[q];
      }
      if (e2 >= 0 && k >= m->ulevels[e2] - 1 && k < m->nlevels[e2] - 1) {
        const size_t q = (size_t)e2 * L + k;
        t2 = (uv[2 * q + 1] * cr[2] - uv[2 * q] * cr[3]) * helem[q];
      }
      const double vf = t1 + t2, av = fabs(vf);
      vfl[(size_t)e * L + k] = vf;
      fh[(size_t)e * L + k] =
          -0.5 * (T[(size_t)n1 * L + k] * (vf + av) + T[(size_t)n2 * L + k] * (vf - av));
    }
  }

  /* LO vertical flux on layers (tracer_adv.py:108-120), LO solution (:298-313) */
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; ++n) {
    const int a = m->ulevels_nod2D[n] - 1, b = m->nlevels_nod2D[n] - 1;
    const size_t o = (size_t)n * L;
    for (int k = a; k < b; ++k) {
      const double w = w_e[o + k], aw = fabs(w);
      fv[o + k] = -0.5 * (T[o + k] * (w + aw) + T[o + (k > 0 ? k - 1 : 0)] * (w - aw)) *
                  m->area[o + k];
    }
    for (int k = a; k < b; ++k) {
      double div = 0.0;
      for (int j = ne.off[n]; j < ne.off[n + 1]; ++j) {
        const int idx = ne.idx[j];
        const double f = fh[(size_t)(idx >> 1) * L + k];
        div += (idx & 1) ? -f : f;
      }
      const double av = m->areasvol[o + k], hn = hnode_new[o + k];
      if (hn > 0.0 && av > 0.0) {
        const double fvb = k + 1 < L ? fv[o + k + 1] : 0.0;
        LO[o + k] = (T[o + k] * hnode[o + k] + (div + (fv[o + k] - fvb)) * dt / av) / hn;
      }
    }
  }

  /* implicit w_i advection of LO (tracer_adv.py:487-529) */
  if (w_i) {
#pragma omp parallel for schedule(static)
    for (int n = 0; n < N; ++n) {
      const int a = m->ulevels_nod2D[n] - 1, b = m->nlevels_nod2D[n] - 1;
      const size_t o = (size_t)n * L;
      double cp[128], dp[128], cprev = 0.0, dprev = 0.0;
      for (int k = a; k < b; ++k) {
        const double av = m->areasvol[o + k], sa = av > 0.0 ? av : 1.0;
        const double vt = dt * m->area[o + k] / sa;
        const double vb = dt * (k + 1 < L ? m->area[o + k + 1] : 0.0) / sa;
        const double wu = w_i[o + k], wd = k + 1 < L ? w_i[o + k + 1] : 0.0;
        const int surf = (k == a), bot = (k == b - 1);
        const double aa = (surf ? 0.0 : dmin(0.0, wu)) * vt;
        const double btop = (surf ? wu : dmax(0.0, wu)) * vt;
        const double bbot = (bot ? 0.0 : -dmin(0.0, wd)) * vb;
        const double cc = (bot ? 0.0 : -dmax(0.0, wd)) * vb;
        const double badv = btop + bbot, bb = hnode_new[o + k] + badv;
        const double Tm = LO[o + (k > 0 ? k - 1 : 0)], Tp = k + 1 < L ? LO[o + k + 1] : 0.0;
        const double rhs = -(aa * Tm + badv * LO[o + k] + cc * Tp);
        const double md = bb - aa * cprev;
        cprev = cc / md;
        dprev = (rhs - aa * dprev) / md;
        cp[k] = cprev;
        dp[k] = dprev;
      }
      double x = 0.0;
      for (int k = b - 1; k >= a; --k) { x = dp[k] - cp[k] * x; dp[k] = x; }
      for (int k = a; k < b; ++k) LO[o + k] += dp[k];
    }
  }

  /* element gradients from T (tracer_adv.py:316-326) */
#pragma omp parallel for schedule(static)
  for (int el = 0; el < E; ++el) {
    const int v0 = m->elem_nodes[3 * el], v1 = m->elem_nodes[3 * el + 1],
              v2 = m->elem_nodes[3 * el + 2];
    const double* g = m->gradient_sca + 6 * (size_t)el;
    for (int k = m->ulevels[el] - 1; k < m->nlevels[el] - 1; ++k) {
      const double t0 = T[(size_t)v0 * L + k], t1 = T[(size_t)v1 * L + k],
                   t2 = T[(size_t)v2 * L + k];
      tr[2 * ((size_t)el * L + k)] = g[0] * t0 + g[1] * t1 + g[2] * t2;
      tr[2 * ((size_t)el * L + k) + 1] = g[3] * t0 + g[4] * t1 + g[5] * t2;
    }
  }
  /* node-average gradient (tracer_adv.py:329-341) */
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; ++n) {
    for (int k = 0; k < L; ++k) {
      double nx = 0.0, ny = 0.0, den = 0.0;
      for (int j = m->nod_in_elem2D_offsets[n]; j < m->nod_in_elem2D_offsets[n + 1]; ++j) {
        const int el = m->nod_in_elem2D[j];
        if (k >= m->ulevels[el] - 1 && k < m->nlevels[el] - 1) {
          const double a = m->elem_area[el];
          nx += tr[2 * ((size_t)el * L + k)] * a;
          ny += tr[2 * ((size_t)el * L + k) + 1] * a;
          den += a;
        }
      }
      const double d = den > 0.0 ? den : 1.0;
      gn[2 * ((size_t)n * L + k)] = nx / d;
      gn[2 * ((size_t)n * L + k) + 1] = ny / d;
    }
  }

  /* up/down gradients + MFCT high-order flux; adf_h = HO - LO (tracer_adv.py:196-225,
   * 344-368, 564) */
#pragma omp parallel for schedule(static)
  for (int e = 0; e < Ed; ++e) {
    const int n1 = m->edges[2 * e], n2 = m->edges[2 * e + 1];
    const int e1 = m->edge_tri[2 * e], e2 = m->edge_tri[2 * e + 1];
    const int up = m->edge_up_dn_tri[2 * e], dn = m->edge_up_dn_tri[2 * e + 1];
    double a = R_EARTH * m->elem_cos[e1 >= 0 ? e1 : 0];
    if (e2 >= 0) a = 0.5 * (a + R_EARTH * m->elem_cos[e2]);
    const double c1 = m->edge_dxdy[2 * e] * a, c2 = m->edge_dxdy[2 * e + 1] * R_EARTH;
    const int kmin = (m->ulevels_nod2D_max[n1] > m->ulevels_nod2D_max[n2]
                          ? m->ulevels_nod2D_max[n1] : m->ulevels_nod2D_max[n2]) - 1;
    const int kmax = (m->nlevels_nod2D_min[n1] < m->nlevels_nod2D_min[n2]
                          ? m->nlevels_nod2D_min[n1] : m->nlevels_nod2D_min[n2]) - 1;
    for (int k = 0; k < L; ++k) {
      const size_t q = (size_t)e * L + k, q1 = (size_t)n1 * L + k, q2 = (size_t)n2 * L + k;
      const int use = up >= 0 && dn >= 0 && k >= kmin && k < kmax;
      const double g0 = use ? tr[2 * ((size_t)up * L + k)] : gn[2 * q1];
      const double g1 = use ? tr[2 * ((size_t)dn * L + k)] : gn[2 * q2];
      const double g2 = use ? tr[2 * ((size_t)up * L + k) + 1] : gn[2 * q1 + 1];
      const double g3 = use ? tr[2 * ((size_t)dn * L + k) + 1] : gn[2 * q2 + 1];
      const double A1 = ttf[q1], A2 = ttf[q2], diff = A2 - A1;
      const double Tm1 = A1 + (2.0 * diff + c1 * g0 + c2 * g2) / 6.0;
      const double Tm2 = A2 - (2.0 * diff + c1 * g1 + c2 * g3) / 6.0;
      const double vf = vfl[q], av = fabs(vf);
      adfh[q] = -0.5 * ((vf + av) * Tm1 + (vf - av) * Tm2) - fh[q];
    }
  }

  /* QR4C high-order vertical flux; adf_v = HO - LO (tracer_adv.py:241-295, 567-572) */
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; ++n) {
    const int a = m->ulevels_nod2D[n] - 1, b = m->nlevels_nod2D[n] - 1;
    const size_t o = (size_t)n * L;
    for (int k = a; k <= b && k < L; ++k) {
      const double W = w_i ? w_e[o + k] + w_i[o + k] : w_e[o + k];
      const double ar = m->area[o + k];
      double hi = 0.0;
      if (k == a) {
        hi = -ttf[o + k] * W * ar;
      } else if (k == b) {
        hi = 0.0;
      } else if (k == a + 1 || k == b - 1) {
        hi = -0.5 * (ttf[o + k - 1] + ttf[o + k]) * W * ar;
      } else if (k >= a + 2 && k <= b - 2) {
        double Znz, Zm1, Zm2, Zp1, zb;
        if (Z3d) {
          const double* Zc = Z3d + o;
          Znz = Zc[k]; Zm1 = Zc[k - 1]; Zm2 = Zc[k - 2]; Zp1 = Zc[k + 1 < L ? k + 1 : L - 1];
          zb = zbar3[o + k];
        } else {
          Znz = Zp[k]; Zm1 = Zp[k - 1]; Zm2 = Zp[k - 2]; Zp1 = Zp[k + 1 < L ? k + 1 : L - 1];
          zb = m->zbar[k];
        }
        const double A0 = ttf[o + k], Am1 = ttf[o + k - 1], Am2 = ttf[o + k - 2],
                     Ap1 = ttf[o + k + 1];
        const double qc = (Am1 - A0) / safe_nz(Zm1 - Znz);
        const double qu = (A0 - Ap1) / safe_nz(Znz - Zp1);
        const double qd = (Am2 - Am1) / safe_nz(Zm2 - Zm1);
        const double Tmean1 = A0 + (2.0 * qc + qu) * (zb - Znz) / 3.0;
        const double Tmean2 = Am1 + (2.0 * qc + qd) * (zb - Zm1) / 3.0;
        hi = -0.5 * (Tmean1 + Tmean2) * W * ar;
      }
      double lo_v = fv[o + k];
      if (w_i) {
        lo_v = 0.0;
        if (k < b) {
          const double aw = fabs(W);
          lo_v = -0.5 * (T[o + k] * (W + aw) + T[o + (k > 0 ? k - 1 : 0)] * (W - aw)) * ar;
        }
      }
      adfv[o + k] = hi - lo_v;
    }
  }

  /* Zalesak limiter a2: element bounds (tracer_adv.py:393-397) */
#pragma omp parallel for schedule(static)
  for (int el = 0; el < E; ++el) {
    const int v[3] = {m->elem_nodes[3 * el], m->elem_nodes[3 * el + 1],
                      m->elem_nodes[3 * el + 2]};
    for (int k = 0; k < L; ++k) {
      double mx = -BIG, mn = BIG;
      if (k >= m->ulevels[el] - 1 && k < m->nlevels[el] - 1) {
        mx = -INFINITY;
        mn = INFINITY;
        for (int i = 0; i < 3; ++i) {
          const size_t q = (size_t)v[i] * L + k;
          mx = dmax(mx, dmax(LO[q], T[q]));
          mn = dmin(mn, dmin(LO[q], T[q]));
        }
      }
      amax[(size_t)el * L + k] = mx;
      amin[(size_t)el * L + k] = mn;
    }
  }
  /* a3: node cluster bounds (tracer_adv.py:399-405) */
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; ++n) {
    for (int k = 0; k < L; ++k) {
      double mx = -INFINITY, mn = INFINITY;
      for (int j = m->nod_in_elem2D_offsets[n]; j < m->nod_in_elem2D_offsets[n + 1]; ++j) {
        const int el = m->nod_in_elem2D[j];
        mx = dmax(mx, amax[(size_t)el * L + k]);
        mn = dmin(mn, amin[(size_t)el * L + k]);
      }
      tvm[(size_t)n * L + k] = mx;
      tvn[(size_t)n * L + k] = mn;
    }
  }
  /* a4 + b1 + b2: window, antidiffusive sums, factors (tracer_adv.py:407-451) */
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; ++n) {
    const int a = m->ulevels_nod2D[n] - 1, b = m->nlevels_nod2D[n] - 1;
    const size_t o = (size_t)n * L;
    for (int k = 0; k < L; ++k) { pf[o + k] = 1.0; mf[o + k] = 1.0; }
    for (int k = a; k < b; ++k) {
      double tmax, tmin;
      if (k == a || k == b - 1) {
        tmax = tvm[o + k];
        tmin = tvn[o + k];
      } else {
        tmax = dmax(dmax(tvm[o + k - 1], tvm[o + k]), tvm[o + k + 1]);
        tmin = dmin(dmin(tvn[o + k - 1], tvn[o + k]), tvn[o + k + 1]);
      }
      const double wmax = tmax - LO[o + k], wmin = tmin - LO[o + k];
      const double ft = adfv[o + k], fb = k + 1 < L ? adfv[o + k + 1] : 0.0;
      const double pv = dmax(ft, 0.0) + dmax(-fb, 0.0);
      const double nv = dmin(ft, 0.0) + dmin(-fb, 0.0);
      double sp = 0.0, sm = 0.0;
      for (int j = ne.off[n]; j < ne.off[n + 1]; ++j) {
        const int idx = ne.idx[j];
        const double f = adfh[(size_t)(idx >> 1) * L + k];
        const double s = (idx & 1) ? -f : f;
        sp += dmax(s, 0.0);
        sm += dmin(s, 0.0);
      }
      const double av = m->areasvol[o + k], hn = hnode_new[o + k];
      if (av > 0.0 && hn > 0.0) {
        const double plus = pv + sp, minus = nv + sm;
        pf[o + k] = dmin(1.0, wmax / (plus * dt / av / hn + FLUX_EPS));
        mf[o + k] = dmin(1.0, wmin / (minus * dt / av / hn - FLUX_EPS));
      }
    }
  }
  /* b3 + flux2dtracer_fct + ale_reconstruct (tracer_adv.py:453-484, 142-151) */
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; ++n) {
    const int a = m->ulevels_nod2D[n] - 1, b = m->nlevels_nod2D[n] - 1;
    const size_t o = (size_t)n * L;
    for (int k = 0; k < L; ++k) Tnew[o + k] = T[o + k];
    for (int k = a; k < b; ++k) {
      double lim[2];
      for (int s = 0; s < 2; ++s) {
        const int j = k + s;
        const double f = adfv[o + j];
        double ae;
        if (j == a) ae = f >= 0.0 ? pf[o + j] : mf[o + j];
        else ae = f >= 0.0 ? dmin(mf[o + j - 1], pf[o + j]) : dmin(pf[o + j - 1], mf[o + j]);
        lim[s] = ae * f;
      }
      double hsc = 0.0;
      for (int j = ne.off[n]; j < ne.off[n + 1]; ++j) {
        const int idx = ne.idx[j], e = idx >> 1;
        const double f = adfh[(size_t)e * L + k];
        const size_t p1 = (size_t)m->edges[2 * e] * L + k, p2 = (size_t)m->edges[2 * e + 1] * L + k;
        const double ae = f >= 0.0 ? dmin(pf[p1], mf[p2]) : dmin(mf[p1], pf[p2]);
        hsc += (idx & 1) ? -(ae * f) : ae * f;
      }
      const double av = m->areasvol[o + k], sa = av > 0.0 ? av : 1.0;
      const double hn = hnode[o + k], hnn = hnode_new[o + k];
      const double vdiv = av > 0.0 ? (lim[0] - lim[1]) * dt / sa : 0.0;
      double d = hsc * dt / sa + ((-T[o + k] * hn + LO[o + k] * hnn) + vdiv);
      d = d + T[o + k] * (hn - hnn);
      Tnew[o + k] = T[o + k] + (hnn > 0.0 ? d / hnn : 0.0);
    }
  }

  free(ne.off); free(ne.idx); free(ttf); free(vfl); free(fh); free(fv); free(LO); free(tr);
  free(gn); free(adfh); free(adfv); free(amax); free(amin); free(tvm); free(tvn); free(pf);
  free(mf); free(flo); free(Zp);
  return 0;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
