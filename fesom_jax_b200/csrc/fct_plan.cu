// Plan construction and the single-instance C-ABI entry points of libfesom_fct.
//
// A plan replaces the reference's per-call Mesh pytree operands (fesom_jax/mesh.py:62-129):
// the mesh is validated and uploaded once, and the derived data the kernels need is
// built on the host here:
//   * node -> incident-edge CSR in ascending edge id (the order in which the reference's
//     edge->node segment_sum accumulates, fesom_jax/ops.py:56-81, so the gathers add the
//     same terms in the same order);
//   * level ranges per node/element and the wet-lane lists the kernels iterate;
//   * per-edge MFCT coefficients (edx*a, edy*R) with a = R*cos averaged over the edge's
//     cells, evaluated with the reference's expression (tracer_adv.py:216-220).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <unordered_set>
#include <vector>

#include "fct_host.h"

namespace fct {

static thread_local std::string g_last_error;

// Plans alive in this process: the custom-call handlers receive a plan as an integer in
// their opaque bytes and check it here before use.
static std::mutex g_plans_mu;
static std::unordered_set<const FctPlan*> g_plans;

bool plan_alive(const FctPlan* P) {
  std::lock_guard<std::mutex> lk(g_plans_mu);
  return g_plans.count(P) != 0;
}

PlanUse::PlanUse(FctPlan* P, cudaStream_t s) : lk_(P->mu), P_(P), s_(s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(s, &cs);
  if (e != cudaSuccess) {   // the legacy stream while another stream captures: treat as
    cudaGetLastError();     // captured (no event work)
    cs = cudaStreamCaptureStatusActive;
  }
  capturing_ = cs != cudaStreamCaptureStatusNone;
  if (!capturing_ && P->ws_used) {
    e = cudaStreamWaitEvent(s, P->ws_ev, 0);
    if (e != cudaSuccess) st_ = cuda_error(e, "workspace order wait");
  }
}

int PlanUse::release() {
  if (st_ || capturing_) return st_;
  const cudaError_t e = cudaEventRecord(P_->ws_ev, s_);
  if (e != cudaSuccess) return cuda_error(e, "workspace order record");
  P_->ws_used = true;
  return FCT_OK;
}

int read_health(unsigned long long* d, int n, cudaStream_t s, int64_t* out) {
  std::vector<unsigned long long> h(size_t(n > 0 ? n : 1), 0ull);
  FCT_CUDA(cudaMemcpyAsync(h.data(), d, size_t(n) * sizeof(*d), cudaMemcpyDeviceToHost, s));
  FCT_CUDA(cudaStreamSynchronize(s));
  FCT_CUDA(cudaMemsetAsync(d, 0, size_t(n) * sizeof(*d), s));
  unsigned long long total = 0;
  for (int i = 0; i < n; ++i) total += h[size_t(i)];
  if (out) *out = int64_t(total);
  if (total)
    return set_error(FCT_ERR_NONFINITE, "%llu non-finite T_new values since the last check",
                     total);
  return FCT_OK;
}

int set_error(int status, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return status;
}

// Every workspace field starts on a 256-byte boundary (whole 32-double blocks), so the
// segment kernels' double2 accesses are aligned.
static int64_t pad32(int64_t n) { return (n + 31) & ~int64_t(31); }

int64_t workspace_doubles(int64_t N, int64_t E, int64_t Ed, int64_t L, int ntr) {
  const int64_t t = ntr;
  return pad32(Ed * L) + 4 * pad32(t * E * L) + 8 * pad32(t * N * L) + pad32(t * Ed * L) +
         pad32(N * L) + 2 * pad32(t * N * L) + pad32((2 * t * (N * L + E * L) + 7) / 8);
}

int64_t workspace_doubles_fused(int64_t N, int64_t Ed, int64_t L, int ntr) {
  const int64_t t = ntr;
  return pad32(Ed * L) + kFusedNodeFields * pad32(t * N * L) + pad32(t * Ed * L);
}

Workspace carve_workspace(double* base, int64_t N, int64_t E, int64_t Ed, int64_t L, int ntr,
                          bool fused) {
  Workspace w{};
  w.sN = N * L;
  w.sE = E * L;
  w.sEd = Ed * L;
  double* p = base;
  auto take = [&](int64_t n) { double* q = p; p += pad32(n); return q; };
  w.vflux = take(Ed * L);
  if (fused) {   // the fused stages keep no element fields, node gradients or cluster bounds
    w.lo = take(ntr * w.sN);
    w.adfv = take(ntr * w.sN);
    w.pf = take(ntr * w.sN);
    w.mf = take(ntr * w.sN);
    w.adfh = take(ntr * w.sEd);
    return w;
  }
  w.gx = take(ntr * w.sE);
  w.gy = take(ntr * w.sE);
  w.amax = take(ntr * w.sE);
  w.amin = take(ntr * w.sE);
  w.lo = take(ntr * w.sN);
  w.gnx = take(ntr * w.sN);
  w.gny = take(ntr * w.sN);
  w.adfv = take(ntr * w.sN);
  w.tvmax = take(ntr * w.sN);
  w.tvmin = take(ntr * w.sN);
  w.pf = take(ntr * w.sN);
  w.mf = take(ntr * w.sN);
  w.adfh = take(ntr * w.sEd);
  w.nden = take(w.sN);
  w.fplus = take(ntr * w.sN);
  w.fminus = take(ntr * w.sN);
  uint8_t* b = reinterpret_cast<uint8_t*>(p);
  w.ccx = b; b += ntr * w.sN;
  w.ccn = b; b += ntr * w.sN;
  w.ecx = b; b += ntr * w.sE;
  w.ecn = b;
  return w;
}

int plan_reserve_ws(FctPlan* P, int ntr, bool full) {
  if (ntr <= P->max_tracers && (P->ws_full || !full)) return FCT_OK;
  ntr = std::max(ntr, P->max_tracers);
  full = full || P->ws_full;
  FCT_CUDA(cudaSetDevice(P->device));
  const int64_t nd = full ? workspace_doubles(P->N, P->E, P->Ed, P->L, ntr)
                          : workspace_doubles_fused(P->N, P->Ed, P->L, ntr);
  double* ws = nullptr;
  FCT_CUDA(cudaMalloc(&ws, size_t(nd) * sizeof(double)));
  Workspace w = carve_workspace(ws, P->N, P->E, P->Ed, P->L, ntr, /*fused=*/!full);
  if (P->d_ws) cudaFree(P->d_ws);
  P->d_ws = ws;
  P->ws = w;
  P->max_tracers = ntr;
  P->ws_full = full;
  return FCT_OK;
}

namespace {

struct Blob {
  std::vector<char> bytes;
  template <class T>
  size_t add(const T* src, size_t n) {
    size_t off = (bytes.size() + 255) & ~size_t(255);
    bytes.resize(off + n * sizeof(T));
    if (n) std::memcpy(bytes.data() + off, src, n * sizeof(T));
    return off;
  }
};

int validate_desc(const FctMeshDesc* d) {
  if (!d) return set_error(FCT_ERR_INVALID, "mesh descriptor is NULL");
  if (d->nod2D <= 0 || d->elem2D <= 0 || d->edge2D <= 0)
    return set_error(FCT_ERR_INVALID, "mesh counts must be positive");
  if (d->nl < 3 || d->nl > kMaxLevels)
    return set_error(FCT_ERR_INVALID, "nl=%d outside [3, %d]", d->nl, kMaxLevels);
  if (int64_t(d->nod2D) >= (int64_t(1) << (32 - kLevelBits)) ||
      int64_t(d->edge2D) >= (int64_t(1) << (32 - kLevelBits)) ||
      int64_t(d->elem2D) >= (int64_t(1) << (32 - kLevelBits)))
    return set_error(FCT_ERR_INVALID, "mesh too large for 25-bit entity ids");
  const void* req[] = {d->edges, d->edge_tri, d->edge_up_dn_tri, d->edge_cross_dxdy,
                       d->edge_dxdy, d->elem_nodes, d->gradient_sca, d->elem_cos,
                       d->elem_area, d->nlevels, d->ulevels, d->nlevels_nod2D,
                       d->nlevels_nod2D_min, d->ulevels_nod2D, d->ulevels_nod2D_max,
                       d->nod_in_elem2D_offsets, d->nod_in_elem2D, d->area, d->areasvol,
                       d->Z, d->zbar};
  for (const void* p : req)
    if (!p) return set_error(FCT_ERR_INVALID, "mesh descriptor has a NULL array");
  const int N = d->nod2D, E = d->elem2D, Ed = d->edge2D, L = d->nl;
  for (int i = 0; i < 2 * Ed; ++i)
    if (d->edges[i] < 0 || d->edges[i] >= N)
      return set_error(FCT_ERR_INVALID, "edges[%d]=%d out of range", i, d->edges[i]);
  for (int e = 0; e < Ed; ++e) {
    if (d->edge_tri[2 * e] < 0 || d->edge_tri[2 * e] >= E)
      return set_error(FCT_ERR_INVALID, "edge_tri[%d,0] must be a valid element", e);
    for (int j = 0; j < 2; ++j) {
      int t = d->edge_tri[2 * e + j], u = d->edge_up_dn_tri[2 * e + j];
      if (t < -1 || t >= E || u < -1 || u >= E)
        return set_error(FCT_ERR_INVALID, "edge %d: element id out of range", e);
    }
  }
  for (int i = 0; i < 3 * E; ++i)
    if (d->elem_nodes[i] < 0 || d->elem_nodes[i] >= N)
      return set_error(FCT_ERR_INVALID, "elem_nodes[%d] out of range", i);
  for (int e = 0; e < E; ++e)
    if (d->ulevels[e] < 1 || d->nlevels[e] > L || d->nlevels[e] < d->ulevels[e])
      return set_error(FCT_ERR_INVALID, "element %d level range invalid", e);
  for (int n = 0; n < N; ++n) {
    if (d->ulevels_nod2D[n] < 1 || d->nlevels_nod2D[n] > L ||
        d->nlevels_nod2D[n] < d->ulevels_nod2D[n] || d->nlevels_nod2D_min[n] > L ||
        d->ulevels_nod2D_max[n] < 1)
      return set_error(FCT_ERR_INVALID, "node %d level range invalid", n);
    if (d->nod_in_elem2D_offsets[n + 1] < d->nod_in_elem2D_offsets[n])
      return set_error(FCT_ERR_INVALID, "nod_in_elem2D_offsets not monotone at %d", n);
  }
  if (d->nod_in_elem2D_offsets[0] != 0)
    return set_error(FCT_ERR_INVALID, "nod_in_elem2D_offsets[0] != 0");
  const int nie = d->nod_in_elem2D_offsets[N];
  for (int i = 0; i < nie; ++i)
    if (d->nod_in_elem2D[i] < 0 || d->nod_in_elem2D[i] >= E)
      return set_error(FCT_ERR_INVALID, "nod_in_elem2D[%d] out of range", i);
  for (int n = 0; n < N; ++n)   // every listed cell has the node as a vertex
    for (int j = d->nod_in_elem2D_offsets[n]; j < d->nod_in_elem2D_offsets[n + 1]; ++j) {
      const int* en = d->elem_nodes + 3 * size_t(d->nod_in_elem2D[j]);
      if (en[0] != n && en[1] != n && en[2] != n)
        return set_error(FCT_ERR_INVALID, "nod_in_elem2D lists element %d for node %d, "
                         "which is not one of its vertices", d->nod_in_elem2D[j], n);
    }
  return FCT_OK;
}

}  // namespace

}  // namespace fct

using namespace fct;

static int plan_build(const FctMeshDesc* d, int device, FctPlan* P) {
  const int N = d->nod2D, E = d->elem2D, Ed = d->edge2D, L = d->nl;
  P->device = device;
  P->N = N; P->E = E; P->Ed = Ed; P->L = L;

  std::vector<int> nzmin(N), nzmax(N), eul(E), enl(E);
  for (int n = 0; n < N; ++n) {
    nzmin[n] = d->ulevels_nod2D[n] - 1;
    nzmax[n] = d->nlevels_nod2D[n] - 1;
  }
  for (int e = 0; e < E; ++e) {
    eul[e] = d->ulevels[e] - 1;
    enl[e] = d->nlevels[e] - 1;
  }
  // node -> edge CSR (ascending edge id per node)
  std::vector<int> ne_off(N + 1, 0), ne_idx(2 * size_t(Ed)), ne_oth(2 * size_t(Ed));
  for (int e = 0; e < Ed; ++e) {
    ne_off[d->edges[2 * e] + 1]++;
    ne_off[d->edges[2 * e + 1] + 1]++;
  }
  for (int n = 0; n < N; ++n) ne_off[n + 1] += ne_off[n];
  {
    std::vector<int> fillp(ne_off.begin(), ne_off.end() - 1);
    for (int e = 0; e < Ed; ++e) {
      const int a = d->edges[2 * e], b = d->edges[2 * e + 1];
      ne_oth[fillp[a]] = b;
      ne_idx[fillp[a]++] = 2 * e;
      ne_oth[fillp[b]] = a;
      ne_idx[fillp[b]++] = 2 * e + 1;
    }
  }
  // per-edge MFCT coefficients, reference expression (tracer_adv.py:216-222)
  std::vector<double> ecoef(2 * size_t(Ed));
  for (int e = 0; e < Ed; ++e) {
    const int el1 = d->edge_tri[2 * e], el2 = d->edge_tri[2 * e + 1];
    double a = kREarth * d->elem_cos[el1 >= 0 ? el1 : 0];
    if (el2 >= 0) a = 0.5 * (a + kREarth * d->elem_cos[el2]);
    ecoef[2 * e] = d->edge_dxdy[2 * e] * a;
    ecoef[2 * e + 1] = d->edge_dxdy[2 * e + 1] * kREarth;
  }
  // element -> its three edges (with its role), element -> edges using it as up/dn
  std::vector<int> eedge(3 * size_t(E), -1), ecount(E, 0);
  std::vector<int> eud_off(E + 1, 0), eud_idx;
  for (int e = 0; e < Ed; ++e)
    for (int r = 0; r < 2; ++r) {
      const int el = d->edge_tri[2 * e + r];
      if (el < 0) continue;
      if (ecount[el] >= 3) return set_error(FCT_ERR_INVALID, "element %d has more than 3 edges", el);
      eedge[3 * size_t(el) + ecount[el]++] = 2 * e + r;
    }
  for (int e = 0; e < Ed; ++e)
    for (int r = 0; r < 2; ++r) {
      const int el = d->edge_up_dn_tri[2 * e + r];
      if (el >= 0) eud_off[el + 1]++;
    }
  for (int el = 0; el < E; ++el) eud_off[el + 1] += eud_off[el];
  eud_idx.assign(size_t(eud_off[E]), 0);
  {
    std::vector<int> fillp(eud_off.begin(), eud_off.end() - 1);
    for (int e = 0; e < Ed; ++e)
      for (int r = 0; r < 2; ++r) {
        const int el = d->edge_up_dn_tri[2 * e + r];
        if (el >= 0) eud_idx[fillp[el]++] = 2 * e + r;
      }
  }
  std::vector<int> ekmin(Ed), ekmax(Ed);
  for (int e = 0; e < Ed; ++e) {
    const int el1 = d->edge_tri[2 * e], el2 = d->edge_tri[2 * e + 1];
    int lo = eul[el1], hi = enl[el1];
    if (el2 >= 0) {
      lo = std::min(lo, eul[el2]);
      hi = std::max(hi, enl[el2]);
    }
    ekmin[e] = std::max(lo, 0);
    ekmax[e] = std::min(hi, L);
  }
  // levels where MFCT takes the up/down cells' gradients (tracer_adv.py:344-368): both
  // cells present and k in [max(ulevels_nod2D_max) - 1, min(nlevels_nod2D_min) - 1) of
  // the two nodes, clipped to the edge's own levels
  std::vector<int> etr(Ed, 0);
  for (int e = 0; e < Ed; ++e) {
    const int n1 = d->edges[2 * e], n2 = d->edges[2 * e + 1];
    if (d->edge_up_dn_tri[2 * e] < 0 || d->edge_up_dn_tri[2 * e + 1] < 0) continue;
    const int lo = std::max({d->ulevels_nod2D_max[n1] - 1, d->ulevels_nod2D_max[n2] - 1,
                             ekmin[e]});
    const int hi = std::min({d->nlevels_nod2D_min[n1] - 1, d->nlevels_nod2D_min[n2] - 1,
                             ekmax[e]});
    if (hi > lo) etr[e] = lo | (hi << 8);
  }
  // packed slots for the fused kernels
  std::vector<int4> ne4(2 * size_t(Ed));
  for (int n = 0; n < N; ++n)
    for (int j = ne_off[n]; j < ne_off[n + 1]; ++j) {
      const int e = ne_idx[j] >> 1;
      const int el1 = d->edge_tri[2 * e], el2 = d->edge_tri[2 * e + 1];
      const unsigned tri = el2 >= 0 ? pack_tri(eul[el1], enl[el1], eul[el2], enl[el2])
                                    : pack_tri(eul[el1], enl[el1], int(kNoCell), 0);
      ne4[j] = make_int4(ne_idx[j], ne_oth[j], ekmin[e] | (ekmax[e] << 8), int(tri));
    }
  const int nie_all = d->nod_in_elem2D_offsets[N];
  std::vector<int4> nel4(std::max(nie_all, 1));
  std::vector<int> nelr(std::max(nie_all, 1));
  for (int n = 0; n < N; ++n)
    for (int j = d->nod_in_elem2D_offsets[n]; j < d->nod_in_elem2D_offsets[n + 1]; ++j) {
      const int el = d->nod_in_elem2D[j];
      const int* en = d->elem_nodes + 3 * size_t(el);
      nel4[j] = make_int4(el, en[0], en[1], en[2]);
      const int pos = en[0] == n ? 0 : (en[1] == n ? 1 : 2);   // n's place in the cell
      nelr[j] = eul[el] | (enl[el] << 8) | (pos << 16);
    }
  std::vector<double> Zp(L);
  for (int k = 0; k < L - 1; ++k) Zp[k] = d->Z[k];
  Zp[L - 1] = d->Z[L - 2];
  // lanes
  std::vector<uint32_t> iface, layer, edgel, eleml, dry;
  for (int n = 0; n < N; ++n) {
    for (int k = std::max(nzmin[n], 0); k <= std::min(nzmax[n], L - 1); ++k) {
      iface.push_back((uint32_t(n) << kLevelBits) | uint32_t(k));
      if (k < nzmax[n]) layer.push_back((uint32_t(n) << kLevelBits) | uint32_t(k));
    }
    for (int k = 0; k < L; ++k)   // the levels that keep T (ale_reconstruct)
      if (!(k >= nzmin[n] && k < nzmax[n])) dry.push_back((uint32_t(n) << kLevelBits) | uint32_t(k));
  }
  int64_t wet_elem = 0;
  for (int e = 0; e < E; ++e)
    for (int k = std::max(eul[e], 0); k < std::min(enl[e], L); ++k) {
      eleml.push_back((uint32_t(e) << kLevelBits) | uint32_t(k));
      ++wet_elem;
    }
  for (int e = 0; e < Ed; ++e)
    for (int k = ekmin[e]; k < ekmax[e]; ++k)
      edgel.push_back((uint32_t(e) << kLevelBits) | uint32_t(k));
  P->n_wet_elem_layers = wet_elem;
  // lane records (fct_internal.cuh): level range, CSR starts and degrees of a node lane,
  // and the end nodes and triangle range of an edge lane, in one 16-byte word
  auto node_rec = [&](uint32_t ln) -> int4 {
    const int n = int(ln >> kLevelBits);
    const int ed = ne_off[n + 1] - ne_off[n];
    const int cd = d->nod_in_elem2D_offsets[n + 1] - d->nod_in_elem2D_offsets[n];
    return make_int4(int(ln), ne_off[n], d->nod_in_elem2D_offsets[n],
                     int(unsigned(nzmin[n]) | (unsigned(nzmax[n]) << 8) | (unsigned(ed) << 16) |
                         (unsigned(cd) << 24)));
  };
  for (int n = 0; n < N; ++n) {
    if (ne_off[n + 1] - ne_off[n] > 255 ||
        d->nod_in_elem2D_offsets[n + 1] - d->nod_in_elem2D_offsets[n] > 255)
      return set_error(FCT_ERR_INVALID, "node %d has more than 255 edges or cells", n);
  }
  std::vector<int4> iface4(std::max<size_t>(iface.size(), 1)), layer4(std::max<size_t>(layer.size(), 1));
  for (size_t i = 0; i < iface.size(); ++i) iface4[i] = node_rec(iface[i]);
  for (size_t i = 0; i < layer.size(); ++i) layer4[i] = node_rec(layer[i]);
  std::vector<int4> eud4(2 * size_t(Ed));
  for (int e = 0; e < Ed; ++e)
    for (int r = 0; r < 2; ++r) {
      const int el = d->edge_up_dn_tri[2 * e + r];
      const int* en = d->elem_nodes + 3 * size_t(el >= 0 ? el : 0);
      eud4[2 * size_t(e) + r] = el >= 0 ? make_int4(el, en[0], en[1], en[2]) : make_int4(0, 0, 0, 0);
    }
  std::vector<int4> ecell4(static_cast<size_t>(Ed));
  for (int e = 0; e < Ed; ++e) {
    const int el1 = d->edge_tri[2 * e], el2 = d->edge_tri[2 * e + 1];
    const unsigned tri = el2 >= 0 ? pack_tri(eul[el1], enl[el1], eul[el2], enl[el2])
                                  : pack_tri(eul[el1], enl[el1], int(kNoCell), 0);
    ecell4[e] = make_int4(el1, el2, int(tri), 0);
  }
  std::vector<int4> edge4(std::max<size_t>(edgel.size(), 1));
  for (size_t i = 0; i < edgel.size(); ++i) {
    const int e = int(edgel[i] >> kLevelBits);
    edge4[i] = make_int4(int(edgel[i]), d->edges[2 * e], d->edges[2 * e + 1], etr[e]);
  }
  // segment kernels (fct_segments.cu): node records, runs of up to kSegLevels[i]
  // consecutive layers of a node, runs of consecutive MFCT up/down-cell levels of an edge
  // (those whose up cell holds the edge's first node and whose down cell its second), and
  // the remaining edge lanes
  // and, per node layer, the flags of the node's edge slots at that level: bit j (slot j
  // has the level: its flux is counted), bit kSlotWet + j (a cell of slot j is wet there),
  // kOwnBit (some cell of the node is wet), kOffBit (some cell of the node is dry) and
  // kGradBit (an edge lane of the node at that level takes the node-average gradients:
  // the only levels where the one-kernel-per-stage forward computes them)
  std::vector<int4> nrec(static_cast<size_t>(N));
  std::vector<unsigned long long> nflags;
  for (int n = 0; n < N; ++n) {
    const int ed = ne_off[n + 1] - ne_off[n];
    const int cd = d->nod_in_elem2D_offsets[n + 1] - d->nod_in_elem2D_offsets[n];
    if (ed > kMaxSlots)
      return set_error(FCT_ERR_INVALID, "node %d has %d edges; at most %d are supported", n,
                       ed, kMaxSlots);
    nrec[n] = make_int4(ne_off[n], d->nod_in_elem2D_offsets[n],
                        int(unsigned(nzmin[n]) | (unsigned(nzmax[n]) << 8) |
                            (unsigned(ed) << 16) | (unsigned(cd) << 24)),
                        int(nflags.size()));
    for (int k = std::max(nzmin[n], 0); k < std::min(nzmax[n], L); ++k) {
      unsigned long long f = 0;
      bool own = false, off = false, grad = false;
      for (int j = ne_off[n]; j < ne_off[n + 1]; ++j) {
        const int4 sl = ne4[j];
        const unsigned rg = unsigned(sl.z), tr = unsigned(sl.w);
        const bool on = k >= int(rg & 255u) && k < int((rg >> 8) & 255u);
        const unsigned et = unsigned(etr[sl.x >> 1]);
        grad = grad || (on && !(k >= int(et & 255u) && k < int((et >> 8) & 255u)));
        const bool has2 = ((tr >> 16) & 255u) != kNoCell;
        const bool c1 = k >= int(tr & 255u) && k < int((tr >> 8) & 255u);
        const bool c2 = has2 && k >= int((tr >> 16) & 255u) && k < int((tr >> 24) & 255u);
        const int jj = j - ne_off[n];
        f |= (unsigned long long)(on) << jj;
        f |= (unsigned long long)(c1 || c2) << (kSlotWet + jj);
        own = own || c1 || c2;
        off = off || !c1 || (has2 && !c2);
      }
      f |= (unsigned long long)(own) << kOwnBit;
      f |= (unsigned long long)(off) << kOffBit;
      f |= (unsigned long long)(grad) << kGradBit;
      nflags.push_back(f);
    }
  }
  std::vector<int4> erec(static_cast<size_t>(Ed)), emf4(static_cast<size_t>(Ed));
  std::vector<double> emfw(8 * size_t(Ed), 0.0);
  std::vector<uint32_t> efix;
  std::vector<int> tlo(Ed, 0), thi(Ed, 0);
  for (int e = 0; e < Ed; ++e) {
    const int n1 = d->edges[2 * e], n2 = d->edges[2 * e + 1];
    const int up = d->edge_up_dn_tri[2 * e], dn = d->edge_up_dn_tri[2 * e + 1];
    auto holds = [&](int el, int n) {
      const int* en = d->elem_nodes + 3 * size_t(el);
      return en[0] == n || en[1] == n || en[2] == n;
    };
    if (etr[e] && holds(up, n1) && holds(dn, n2)) {
      tlo[e] = etr[e] & 255;
      thi[e] = (etr[e] >> 8) & 255;
    }
    erec[e] = make_int4(n1, n2, tlo[e] | (thi[e] << 8), 0);
    if (thi[e] > tlo[e]) {
      // MFCT with the up cell's gradient at n1 and the down cell's at n2
      // (tracer_adv.py:196-225): edx*a*gx + edy*R*gy of a cell is one weighted sum of its
      // vertex values, sum_i (c1*gsca[i] + c2*gsca[3+i]) T_i, scaled here by the scheme's
      // 1/6; vertex order: the edge's own node, then the cell's other two
      const double c1 = ecoef[2 * e], c2 = ecoef[2 * e + 1];
      int other[4];
      for (int r = 0; r < 2; ++r) {
        const int el = d->edge_up_dn_tri[2 * e + r], own = r == 0 ? n1 : n2;
        const int* en = d->elem_nodes + 3 * size_t(el);
        const double* g = d->gradient_sca + 6 * size_t(el);
        const int p = en[0] == own ? 0 : (en[1] == own ? 1 : 2);
        const int a = (p + 1) % 3, bb = (p + 2) % 3;
        const int idx[3] = {p, a, bb};
        for (int i = 0; i < 3; ++i)
          emfw[8 * size_t(e) + 3 * r + i] = (c1 * g[idx[i]] + c2 * g[3 + idx[i]]) / 6.0;
        other[2 * r] = en[a];
        other[2 * r + 1] = en[bb];
      }
      emf4[e] = make_int4(other[0], other[1], other[2], other[3]);
    }
    for (int k = ekmin[e]; k < ekmax[e]; ++k)
      if (k < tlo[e] || k >= thi[e]) efix.push_back((uint32_t(e) << kLevelBits) | uint32_t(k));
  }
  std::vector<uint32_t> nseg[kSegVariants], eseg[kSegVariants];
  for (int v = 0; v < kSegVariants; ++v) {
    const int lpt = kSegLevels[v];
    for (int n = 0; n < N; ++n)
      for (int k = std::max(nzmin[n], 0); k < std::min(nzmax[n], L); k += lpt)
        nseg[v].push_back((uint32_t(n) << kLevelBits) | uint32_t(k));
    for (int e = 0; e < Ed; ++e)
      for (int k = tlo[e]; k < thi[e]; k += lpt)
        eseg[v].push_back((uint32_t(e) << kLevelBits) | uint32_t(k));
  }

  Blob b;
  const int nie = d->nod_in_elem2D_offsets[N];
  size_t o_nzmin = b.add(nzmin.data(), N), o_nzmax = b.add(nzmax.data(), N);
  size_t o_ulmax = b.add(d->ulevels_nod2D_max, N), o_nlmin = b.add(d->nlevels_nod2D_min, N);
  size_t o_neoff = b.add(ne_off.data(), N + 1), o_neidx = b.add(ne_idx.data(), ne_idx.size());
  size_t o_neoth = b.add(ne_oth.data(), ne_oth.size());
  size_t o_neloff = b.add(d->nod_in_elem2D_offsets, N + 1);
  size_t o_nelidx = b.add(d->nod_in_elem2D, nie);
  size_t o_area = b.add(d->area, size_t(N) * L), o_av = b.add(d->areasvol, size_t(N) * L);
  size_t o_en = b.add(d->elem_nodes, 3 * size_t(E));
  size_t o_eul = b.add(eul.data(), E), o_enl = b.add(enl.data(), E);
  size_t o_gs = b.add(d->gradient_sca, 6 * size_t(E)), o_ea = b.add(d->elem_area, E);
  size_t o_edges = b.add(d->edges, 2 * size_t(Ed)), o_etri = b.add(d->edge_tri, 2 * size_t(Ed));
  size_t o_eud = b.add(d->edge_up_dn_tri, 2 * size_t(Ed));
  size_t o_cross = b.add(d->edge_cross_dxdy, 4 * size_t(Ed));
  size_t o_ecoef = b.add(ecoef.data(), ecoef.size());
  size_t o_ekmin = b.add(ekmin.data(), Ed), o_ekmax = b.add(ekmax.data(), Ed);
  size_t o_etr = b.add(etr.data(), Ed);
  size_t o_eedge = b.add(eedge.data(), eedge.size());
  size_t o_eudoff = b.add(eud_off.data(), eud_off.size());
  size_t o_eudidx = b.add(eud_idx.data(), std::max<size_t>(eud_idx.size(), 1));
  size_t o_ne4 = b.add(ne4.data(), ne4.size()), o_nel4 = b.add(nel4.data(), nel4.size());
  size_t o_nelr = b.add(nelr.data(), nelr.size());
  size_t o_Zp = b.add(Zp.data(), L), o_zbar = b.add(d->zbar, L);
  size_t o_if = b.add(iface.data(), iface.size()), o_ly = b.add(layer.data(), layer.size());
  size_t o_dry = b.add(dry.data(), std::max<size_t>(dry.size(), 1));
  size_t o_ed = b.add(edgel.data(), edgel.size()), o_el = b.add(eleml.data(), eleml.size());
  size_t o_if4 = b.add(iface4.data(), iface4.size()), o_ly4 = b.add(layer4.data(), layer4.size());
  size_t o_ed4 = b.add(edge4.data(), edge4.size());
  size_t o_eud4 = b.add(eud4.data(), eud4.size());
  size_t o_ecell4 = b.add(ecell4.data(), ecell4.size());
  size_t o_nrec = b.add(nrec.data(), nrec.size()), o_erec = b.add(erec.data(), erec.size());
  size_t o_emf4 = b.add(emf4.data(), emf4.size()), o_emfw = b.add(emfw.data(), emfw.size());
  size_t o_nflags = b.add(nflags.data(), std::max<size_t>(nflags.size(), 1));
  size_t o_efix = b.add(efix.data(), std::max<size_t>(efix.size(), 1));
  size_t o_nseg[kSegVariants], o_eseg[kSegVariants];
  for (int v = 0; v < kSegVariants; ++v) {
    o_nseg[v] = b.add(nseg[v].data(), std::max<size_t>(nseg[v].size(), 1));
    o_eseg[v] = b.add(eseg[v].data(), std::max<size_t>(eseg[v].size(), 1));
  }

  FCT_CUDA(cudaSetDevice(device));
  FCT_CUDA(cudaMalloc(&P->d_static, b.bytes.size()));
  FCT_CUDA(cudaMemcpy(P->d_static, b.bytes.data(), b.bytes.size(), cudaMemcpyHostToDevice));
  char* base = static_cast<char*>(P->d_static);
  DevMesh& m = P->hm;
  m.N = N; m.E = E; m.Ed = Ed; m.L = L;
  m.nzmin = (const int*)(base + o_nzmin);
  m.nzmax = (const int*)(base + o_nzmax);
  m.ulmax = (const int*)(base + o_ulmax);
  m.nlmin = (const int*)(base + o_nlmin);
  m.ne_off = (const int*)(base + o_neoff);
  m.ne_idx = (const int*)(base + o_neidx);
  m.ne_oth = (const int*)(base + o_neoth);
  m.nel_off = (const int*)(base + o_neloff);
  m.nel_idx = (const int*)(base + o_nelidx);
  m.area = (const double*)(base + o_area);
  m.areasvol = (const double*)(base + o_av);
  m.enodes = (const int*)(base + o_en);
  m.eul = (const int*)(base + o_eul);
  m.enl = (const int*)(base + o_enl);
  m.gsca = (const double*)(base + o_gs);
  m.earea = (const double*)(base + o_ea);
  m.edges = (const int*)(base + o_edges);
  m.etri = (const int*)(base + o_etri);
  m.eupdn = (const int*)(base + o_eud);
  m.cross = (const double*)(base + o_cross);
  m.ecoef = (const double*)(base + o_ecoef);
  m.ekmin = (const int*)(base + o_ekmin);
  m.eedge = (const int*)(base + o_eedge);
  m.eud_off = (const int*)(base + o_eudoff);
  m.eud_idx = (const int*)(base + o_eudidx);
  m.ekmax = (const int*)(base + o_ekmax);
  m.etr = (const int*)(base + o_etr);
  m.ne4 = (const int4*)(base + o_ne4);
  m.nel4 = (const int4*)(base + o_nel4);
  m.nelr = (const int*)(base + o_nelr);
  m.Zp = (const double*)(base + o_Zp);
  m.zbar = (const double*)(base + o_zbar);
  m.iface_lanes = (const uint32_t*)(base + o_if);  m.n_iface = int64_t(iface.size());
  m.layer_lanes = (const uint32_t*)(base + o_ly);  m.n_layer = int64_t(layer.size());
  m.dry_lanes = (const uint32_t*)(base + o_dry);  m.n_dry = int64_t(dry.size());
  m.edge_lanes = (const uint32_t*)(base + o_ed);   m.n_edge = int64_t(edgel.size());
  m.elem_lanes = (const uint32_t*)(base + o_el);   m.n_elem = int64_t(eleml.size());
  m.iface4 = (const int4*)(base + o_if4);
  m.layer4 = (const int4*)(base + o_ly4);
  m.edge4 = (const int4*)(base + o_ed4);
  m.eud4 = (const int4*)(base + o_eud4);
  m.ecell4 = (const int4*)(base + o_ecell4);
  m.nrec = (const int4*)(base + o_nrec);
  m.nflags = (const unsigned long long*)(base + o_nflags);
  m.erec = (const int4*)(base + o_erec);
  m.emf4 = (const int4*)(base + o_emf4);
  m.emfw = (const double*)(base + o_emfw);
  m.efix = (const uint32_t*)(base + o_efix);
  m.n_efix = int64_t(efix.size());
  for (int v = 0; v < kSegVariants; ++v) {
    m.nseg[v] = (const uint32_t*)(base + o_nseg[v]);
    m.n_nseg[v] = int64_t(nseg[v].size());
    m.eseg[v] = (const uint32_t*)(base + o_eseg[v]);
    m.n_eseg[v] = int64_t(eseg[v].size());
  }
  FCT_CUDA(cudaMalloc(&P->d_mesh, sizeof(DevMesh)));
  FCT_CUDA(cudaMemcpy(P->d_mesh, &m, sizeof(DevMesh), cudaMemcpyHostToDevice));
  FCT_CUDA(cudaMalloc(&P->d_health, sizeof(unsigned long long)));
  FCT_CUDA(cudaMemset(P->d_health, 0, sizeof(unsigned long long)));
  FCT_CUDA(cudaEventCreateWithFlags(&P->ws_ev, cudaEventDisableTiming));
  return fork_create(P->fork);
}

extern "C" {

const char* fct_last_error(void) { return fct::g_last_error.c_str(); }

const char* fct_version(void) { return "fesom_fct 0.1.0 (sm_100a, fp64)"; }

int fct_plan_destroy(FctPlan* P) {
  if (!P) return FCT_OK;
  {
    std::lock_guard<std::mutex> lk(fct::g_plans_mu);
    fct::g_plans.erase(P);
  }
  cudaSetDevice(P->device);
  if (P->d_adj) cudaFree(P->d_adj);
  if (P->adj_side) cudaStreamDestroy(P->adj_side);
  for (cudaEvent_t ev : P->adj_ev)
    if (ev) cudaEventDestroy(ev);
  if (P->ws_ev) {
    cudaEventSynchronize(P->ws_ev);
    cudaEventDestroy(P->ws_ev);
  }
  fork_destroy(P->fork);
  if (P->d_health) cudaFree(P->d_health);
  if (P->d_ws) cudaFree(P->d_ws);
  if (P->d_mesh) cudaFree(P->d_mesh);
  if (P->d_static) cudaFree(P->d_static);
  delete P;
  return FCT_OK;
}

int fct_plan_reserve(FctPlan* P, int max_tracers) {
  if (!P) return set_error(FCT_ERR_INVALID, "plan is NULL");
  if (max_tracers < 1) return set_error(FCT_ERR_INVALID, "max_tracers must be >= 1");
  return plan_reserve_ws(P, max_tracers, !P->fused);
}

int fct_plan_create(const FctMeshDesc* desc, int device, int max_tracers, FctPlan** out) {
  if (!out) return set_error(FCT_ERR_INVALID, "out is NULL");
  *out = nullptr;
  int st = validate_desc(desc);
  if (st) return st;
  FctPlan* P = new FctPlan();
  st = plan_build(desc, device, P);
  if (!st) st = fct_plan_reserve(P, max_tracers < 1 ? 1 : max_tracers);
  if (st) { fct_plan_destroy(P); return st; }
  {
    std::lock_guard<std::mutex> lk(fct::g_plans_mu);
    fct::g_plans.insert(P);
  }
  *out = P;
  return FCT_OK;
}

int fct_plan_info(const FctPlan* P, int64_t out[8]) {
  if (!P || !out) return set_error(FCT_ERR_INVALID, "NULL argument");
  out[0] = P->N; out[1] = P->E; out[2] = P->Ed; out[3] = P->L;
  out[4] = P->hm.n_layer; out[5] = P->n_wet_elem_layers; out[6] = P->hm.n_edge;
  out[7] = P->max_tracers;
  return FCT_OK;
}

int fct_plan_set_mapping(FctPlan* P, int tracers_per_thread, int levels_per_thread) {
  if (!P) return set_error(FCT_ERR_INVALID, "NULL plan");
  const int t = tracers_per_thread, l = levels_per_thread;
  if ((t != 1 && t != 2 && t != 4 && t != 8) || (l != 1 && l != 2 && l != 4 && l != 8))
    return set_error(FCT_ERR_INVALID, "tracers and levels per thread must be 1, 2, 4 or 8");
  P->per_thread = t;
  P->lpt = l;
  return FCT_OK;
}

int fct_plan_set_fused(FctPlan* P, int fused) {
  if (!P) return set_error(FCT_ERR_INVALID, "NULL plan");
  if (!fused) {   // the unfused stages need every stage field
    const int st = plan_reserve_ws(P, P->max_tracers, true);
    if (st) return st;
  }
  P->fused = fused != 0;
  return FCT_OK;
}

int fct_vert_diff(FctPlan* P, const FctVdiffFields* f, double dt, int ntr, fct_stream_t stream) {
  if (!P || !f) return set_error(FCT_ERR_INVALID, "NULL plan or fields");
  if (ntr < 1) return set_error(FCT_ERR_INVALID, "ntr must be >= 1");
  if (ntr > P->max_tracers)
    return set_error(FCT_ERR_CAPACITY, "ntr=%d exceeds reserved workspace (%d tracers); "
                     "call fct_plan_reserve first", ntr, P->max_tracers);
  if (!f->T || !f->T_new || !f->Kv || !f->hnode_new)
    return set_error(FCT_ERR_INVALID, "a required field pointer is NULL");
  if (!(dt > 0.0)) return set_error(FCT_ERR_INVALID, "dt must be positive");
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != P->device) cudaSetDevice(P->device);
  Inst in{};
  in.m = P->d_mesh;
  in.hnode_new = f->hnode_new;
  in.T = f->T;
  in.T_new = f->T_new;
  in.vd_T = f->T;
  in.Kv = f->Kv;
  in.vd_Z3d = f->Z3d;
  in.bc_surf = f->bc_surf;
  in.bc_stride = P->N;
  in.sw_3d = f->sw_3d;
  in.sw_tracer = f->sw_3d ? f->sw_tracer : -1;
  in.tstride = f->tracer_stride ? f->tracer_stride : int64_t(P->N) * P->L;
  in.tg = 0;
  in.wtg = ntr;
  in.ws = P->ws;
  in.dt = dt;
  in.ntr = ntr;
  LaunchDims dims{};
  dims.max_nodes = P->N;
  dims.ntr = ntr;
  dims.chunk = 0;
  dims.per_thread = 8;
  int st;
  {
    PlanUse use(P, static_cast<cudaStream_t>(stream));
    st = use.status();
    if (!st) st = launch_vdiff(in, dims, static_cast<cudaStream_t>(stream));
    if (!st) st = use.release();
  }
  if (prev >= 0 && prev != P->device) cudaSetDevice(prev);
  return st;
}

int fct_forward(FctPlan* P, const FctFields* f, double dt, int ntr, fct_stream_t stream) {
  return fct_forward_ex(P, f, dt, ntr, 0, stream);
}

int fct_forward_ex(FctPlan* P, const FctFields* f, double dt, int ntr, int flags,
                   fct_stream_t stream) {
  if (flags & ~FCT_FWD_STAGEWISE) return set_error(FCT_ERR_INVALID, "unknown flags 0x%x", flags);
  const bool stagewise = (flags & FCT_FWD_STAGEWISE) || !P || !P->fused;
  if (P && stagewise && !P->ws_full)
    return set_error(FCT_ERR_CAPACITY, "the stage-by-stage kernels need the full workspace: "
                     "call fct_plan_set_fused(plan, 0) or fct_plan_reserve_adjoint first");
  if (!P || !f) return set_error(FCT_ERR_INVALID, "NULL plan or fields");
  if (ntr < 1) return set_error(FCT_ERR_INVALID, "ntr must be >= 1");
  if (ntr > P->max_tracers)
    return set_error(FCT_ERR_CAPACITY, "ntr=%d exceeds reserved workspace (%d tracers); "
                     "call fct_plan_reserve first", ntr, P->max_tracers);
  if (!f->uv || !f->w_e || !f->helem || !f->hnode || !f->hnode_new || !f->T ||
      !f->T_old || !f->T_new)
    return set_error(FCT_ERR_INVALID, "a required field pointer is NULL");
  if ((f->Z3d == nullptr) != (f->zbar3 == nullptr))
    return set_error(FCT_ERR_INVALID, "Z3d and zbar3 must be given together");
  if (!(dt > 0.0)) return set_error(FCT_ERR_INVALID, "dt must be positive");
  Inst in{};
  in.m = P->d_mesh;
  in.uv = f->uv; in.w_e = f->w_e; in.helem = f->helem;
  in.hnode = f->hnode; in.hnode_new = f->hnode_new;
  in.T = f->T; in.T_old = f->T_old; in.T_new = f->T_new;
  in.tstride = f->tracer_stride ? f->tracer_stride : int64_t(P->N) * P->L;
  in.tg = 0;
  in.wtg = ntr;
  in.Z3d = f->Z3d; in.zbar3 = f->zbar3; in.w_i = f->w_i;
  in.ws = P->ws;
  in.dt = dt;
  in.ntr = ntr;
  in.nonfinite = P->d_health;
  LaunchDims dims{};
  dims_cover(dims, P);
  dims.ntr = ntr;
  dims.chunk = 0;       // one workspace chunk: all ntr tracers
  dims.set_map(P->per_thread, P->lpt);
  dims.any_wi = f->w_i != nullptr;
  dims.copy_dry = true;   // a fresh T_new: dry levels keep T (tracer_adv.py:147-151)
  dims.fused = !stagewise;
  dims.fork = &P->fork;   // used under the plan lock (PlanUse)
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != P->device) cudaSetDevice(P->device);
  int st;
  {
    PlanUse use(P, static_cast<cudaStream_t>(stream));
    st = use.status();
    if (!st) st = launch_forward(in, nullptr, 1, dims, static_cast<cudaStream_t>(stream));
    if (!st) st = use.release();
  }
  if (prev >= 0 && prev != P->device) cudaSetDevice(prev);
  return st;
}

int fct_plan_fill_workspace(FctPlan* P, int byte, fct_stream_t stream) {
  if (!P) return set_error(FCT_ERR_INVALID, "NULL plan");
  if (!P->d_ws) return FCT_OK;
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != P->device) cudaSetDevice(P->device);
  const int64_t nd = P->ws_full ? workspace_doubles(P->N, P->E, P->Ed, P->L, P->max_tracers)
                                : workspace_doubles_fused(P->N, P->Ed, P->L, P->max_tracers);
  int st;
  {
    PlanUse use(P, static_cast<cudaStream_t>(stream));
    st = use.status();
    if (!st) {
      const cudaError_t e = cudaMemsetAsync(P->d_ws, byte & 0xff, size_t(nd) * sizeof(double),
                                            static_cast<cudaStream_t>(stream));
      st = e == cudaSuccess ? use.release() : cuda_error(e, "workspace fill");
    }
  }
  if (prev >= 0 && prev != P->device) cudaSetDevice(prev);
  return st;
}

int fct_plan_health(FctPlan* P, fct_stream_t stream, int64_t* n_nonfinite) {
  if (!P) return set_error(FCT_ERR_INVALID, "NULL plan");
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != P->device) cudaSetDevice(P->device);
  const int st = read_health(P->d_health, 1, static_cast<cudaStream_t>(stream), n_nonfinite);
  if (prev >= 0 && prev != P->device) cudaSetDevice(prev);
  return st;
}

}  // extern "C"
