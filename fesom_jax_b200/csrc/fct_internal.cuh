// Internal device-side structures of libfesom_fct (not part of the public ABI).
//
// Storage: every per-level field is dense row-major [entity, L] float64 (the
// reference layout, fesom_jax/mesh.py:16-20). Kernels walk compact *lane lists*
// (entity, level) that enumerate only wet levels, so dry levels cost no threads and
// no bytes; a lane is packed as (entity << 7) | level (requires L <= 128).
#pragma once

#include <cstdint>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/fesom_fct.h"

namespace fct {

constexpr int kLevelBits = 7;
constexpr int kMaxLevels = 1 << kLevelBits;
constexpr unsigned kLevelMask = kMaxLevels - 1;

constexpr double kREarth = 6367500.0;   // fesom_jax/config.py:41
constexpr double kAbOld = -(0.5 + 0.1);  // tracer_adv.py:44-46
constexpr double kAbNew = (1.5 + 0.1);
constexpr double kFluxEps = 1e-16;       // tracer_adv.py:192
constexpr double kBig = 1e3;             // tracer_adv.py:193

__host__ __device__ inline int lane_ent(uint32_t lane) { return int(lane >> kLevelBits); }
// The layer ranges [eul, enl) of an edge's two cells in one word: cell 1 in the low
// 16 bits, cell 2 in the high 16 (a coast edge has no cell 2: its range is stored as
// [255, 0), empty, and its flag is the eul byte 255).
constexpr unsigned kNoCell = 255u;
__host__ __device__ inline unsigned pack_tri(int ul1, int nl1, int ul2, int nl2) {
  return unsigned(ul1) | (unsigned(nl1) << 8) | (unsigned(ul2) << 16) | (unsigned(nl2) << 24);
}
__host__ __device__ inline int lane_lev(uint32_t lane) { return int(lane & kLevelMask); }
// Dense offset of entity-level (e, k): below 2^32 (entities < 2^25, L <= 128), so it is
// computed in 32 bits (64-bit index products are multi-instruction sequences).
__device__ __forceinline__ uint32_t lq(int e, int L, int k) {
  return uint32_t(e) * uint32_t(L) + uint32_t(k);
}

// (entity, level) of a dense [entity, L] index: entity counts are below 2^25 and L <= 128,
// so the index fits 32 bits and one 32-bit division splits it (a 64-bit integer division
// is a long emulated sequence on the GPU).
__device__ __forceinline__ void split_dense(int64_t i, int L, int& ent, int& k) {
  const uint32_t u = uint32_t(i), q = u / uint32_t(L);
  ent = int(q);
  k = int(u - q * uint32_t(L));
}

// Segment kernels: a thread takes a run of up to kSegLevels[v] consecutive levels of one
// node or edge (variant v), so the entity's neighbour lists and static data are decoded
// once per run instead of once per level.
constexpr int kSegVariants = 4;
// node-layer flag words of the segment kernels (DevMesh::nflags)
constexpr int kMaxSlots = 24;      // edges per node
constexpr int kSlotWet = 24;       // bits 24..47: a cell of the slot's edge is wet
constexpr int kOwnBit = 48;        // some cell of the node is wet at the level
constexpr int kOffBit = 49;        // some cell of the node is dry at the level
constexpr int kGradBit = 50;       // an edge of the node takes the node-average gradients
                                   // at the level (MFCT outside its up/down-cell range)
constexpr int kSegLevels[kSegVariants] = {1, 2, 4, 8};
__host__ __device__ constexpr int seg_variant(int lpt) {
  return lpt == 1 ? 0 : lpt == 2 ? 1 : lpt == 4 ? 2 : 3;
}

// Static mesh on the device (pointers into one plan allocation).
struct DevMesh {
  int N, E, Ed, L;
  // nodes
  const int* nzmin;      // ulevels_nod2D - 1
  const int* nzmax;      // nlevels_nod2D - 1 (exclusive layer bound; bottom interface)
  const int* ulmax;      // ulevels_nod2D_max
  const int* nlmin;      // nlevels_nod2D_min
  const int* ne_off;     // node -> incident edges CSR, ascending edge id
  const int* ne_idx;     //   entry = 2*edge + (node is the edge's second node)
  const int* ne_oth;     //   the edge's other node, aligned with ne_idx
  const int* nel_off;    // node -> elements CSR (nod_in_elem2D, element-ascending)
  const int* nel_idx;
  const double* area;    // [N,L]
  const double* areasvol;
  // elements
  const int* enodes;     // [E,3]
  const int* eul;        // ulevels - 1
  const int* enl;        // nlevels - 1 (exclusive)
  const double* gsca;    // [E,6]
  const double* earea;   // [E]
  // edges
  const int* edges;      // [Ed,2]
  const int* etri;       // [Ed,2]
  const int* eupdn;      // [Ed,2]
  const double* cross;   // [Ed,4]
  const double* ecoef;   // [Ed,2]: edx*a, edy*R  (a = R*cos, averaged over the two cells)
  const int* eedge;      // [E,3] the element's edges: 2*edge + (element is edge_tri[:,1])
  const int* eud_off;    // element -> edges that use it as MFCT up/down triangle (CSR)
  const int* eud_idx;    //   entry = 2*edge + slot (edge_up_dn_tri[edge, slot] == element)
  const int* ekmin;      // [Ed] first level of the edge's lanes (union of its cells' layers)
  const int* ekmax;      // [Ed] one past the last such level
  const int* etr;        // [Ed] levels where MFCT uses the up/down cells' gradients
                         //   (fill_up_dn_grad, tracer_adv.py:344-368), packed
                         //   kmin | kmax << 8 and clipped to [ekmin, ekmax); empty
                         //   when a cell is missing
  // packed CSR slots for the fused stage kernels (one 16-byte load per neighbour)
  const int4* ne4;       // per node->edge slot: {2*edge + second, other node,
                         //   ekmin | ekmax << 8, cell layer ranges (see pack_tri)}
  const int4* nel4;      // per node->element slot: {element, its three nodes}
  const int* nelr;       // per node->element slot: eul | enl << 8 | (node's vertex index) << 16
  // vertical
  const double* Zp;      // [L]  Z padded with Z[L-2] (tracer_adv.py:233)
  const double* zbar;    // [L]
  // lanes
  const uint32_t* iface_lanes;  int64_t n_iface;   // nodes, k in [nzmin, nzmax]
  const uint32_t* layer_lanes;  int64_t n_layer;   // nodes, k in [nzmin, nzmax)
  const uint32_t* dry_lanes;    int64_t n_dry;     // nodes, k outside [nzmin, nzmax)
  const uint32_t* edge_lanes;   int64_t n_edge;    // edges, k in the union of cell layers
  const uint32_t* elem_lanes;   int64_t n_elem;    // elements, k in [eul, enl)
  // lane records of the fused kernels, one 16-byte load per thread:
  //   node lanes {lane, first edge slot, first cell slot,
  //               nzmin | nzmax << 8 | edge count << 16 | cell count << 24}
  //   edge lanes {lane, n1, n2, etr of the edge}
  const int4* iface4;
  const int4* layer4;
  const int4* edge4;
  // per edge, its MFCT up and down cells with their vertices: [2e] = {up, v0, v1, v2},
  // [2e+1] = {dn, v0, v1, v2} (zeros where the cell is missing)
  const int4* eud4;
  // per edge, its two cells and their layer ranges: {el1, el2 (-1 on a coast),
  // ranges packed as in the node->edge slots (pack_tri), 0}
  const int4* ecell4;
  // segment kernels:
  //   nrec per node {first edge slot, first cell slot,
  //                  nzmin | nzmax << 8 | edge count << 16 | cell count << 24,
  //                  index of its first layer in nflags}
  //   erec per edge {n1, n2, lo | hi << 8, 0}: [lo, hi) the levels where MFCT takes the up
  //     and down cells' gradients and the up cell holds n1, the down cell n2 (else empty)
  //   nseg[v] node segments (node << 7 | first layer), runs of kSegLevels[v] layers
  //   eseg[v] edge segments (edge << 7 | first level), runs within [lo, hi)
  //   efix    the edge lanes outside [lo, hi) (node-average gradients, or a mesh whose
  //     up/down cells do not hold the edge's nodes)
  const int4* nrec;
  const unsigned long long* nflags;   // per node layer, at nrec.w + (k - nzmin): bit j the
                                      // slot's edge has level k, bit kSlotWet + j a cell of
                                      // that edge is wet at k, kOwnBit / kOffBit
  const int4* erec;
  // per edge with up/down-cell levels: the up cell's two vertices besides n1 and the down
  // cell's two besides n2, {ua, ub, da, db}, and [8 e ..] the MFCT weights of (n1, ua, ub)
  // and (n2, da, db): (edx*a*gsca_x + edy*R*gsca_y) / 6 of each vertex
  const int4* emf4;
  const double* emfw;
  const uint32_t* nseg[kSegVariants];
  int64_t n_nseg[kSegVariants];
  const uint32_t* eseg[kSegVariants];
  int64_t n_eseg[kSegVariants];
  const uint32_t* efix;
  int64_t n_efix;
};

// A side stream and two events (fork, join) with which the fused step runs its edge stage
// beside the LO stage: both read only the step's inputs and the volume fluxes, and they
// write disjoint workspace fields (adf_h; LO and adf_v), so the two latency-bound kernels
// can share the SMs. Owned by a plan or a batch and used under its lock.
struct Fork {
  cudaStream_t side = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
};

// Per-tracer intermediates of one instance (dense [entity, L]; tracer t at +t*stride).
// Kernels read only entries written earlier in the same step (every reader masks by the
// level range of the entity it reads), so a workspace needs no initial values and may be
// shared by instances of different meshes that run one after another.
// node fields per tracer of the fused workspace: LO, adf_v, the two limiter factors
constexpr int kFusedNodeFields = 4;
struct Workspace {
  double* vflux;                 // [Ed,L] shared by all tracers of the instance
  double *gx, *gy;               // [E,L] element gradients
  double *amax, *amin;           // [E,L] per-element cluster bounds
  double *lo, *gnx, *gny;        // [N,L]
  double* adfv;                  // [N,L] antidiffusive vertical flux (interfaces)
  double *tvmax, *tvmin;         // [N,L]
  double *pf, *mf;               // [N,L] limiter factors
  double* adfh;                  // [Ed,L] antidiffusive horizontal flux
  // kept only by the full workspace (what the reverse pass reads besides the above):
  double* nden;                  // [N,L] node-average denominator (safe), shared by tracers
  double *fplus, *fminus;        // [N,L] limiter sums fct_plus / fct_minus
  uint8_t *ccx, *ccn;            // [N,L] cells attaining the node's cluster max / min
  uint8_t *ecx, *ecn;            // [E,L] vertices attaining the cell's max / min
  int64_t sN, sE, sEd;           // per-tracer strides (doubles, or bytes for the counts)
};

// One FCT instance: a mesh, its per-call fields, and a workspace.
//
// Tracer layouts: tracer-major (the reference's, one [entity, L] array per tracer,
// ``tstride`` doubles apart; ``tg == 0``) or interleaved (``[entity, L, tg]``: the ``tg``
// tracers of one entity-level are contiguous, so a neighbour gather is one contiguous
// chunk). The workspace uses the same convention (interleaved with the same ``tg``).
struct Inst {
  const DevMesh* m;
  const double *uv, *w_e, *helem, *hnode, *hnode_new;
  const double *T, *T_old;
  double* T_new;
  int64_t tstride;
  int tg;
  int wtg;   // tracers held by the workspace (its interleave stride when interleaved)
  // implicit vertical diffusion after the step (fesom_jax/tracer_diff.py:68-123; Kv NULL =
  // off): input vd_T (the FCT result in the batched epilogue), output T_new
  const double *Kv, *vd_T, *vd_Z3d, *bc_surf, *sw_3d;
  int64_t bc_stride;   // doubles between tracers' bc_surf rows
  int sw_tracer;       // tracer that takes the shortwave divergence (-1: none)
  double* w_derived;   // batched producer: w_e = compute_w(uv, helem) written here first
  const double *Z3d, *zbar3, *w_i;
  // health counter: the final stage adds the number of non-finite T_new values it writes
  // (NULL: not counted)
  unsigned long long* nonfinite;
  Workspace ws;
  double dt;
  int ntr;
};

// Reverse-pass intermediates of one instance (tracer-major, dense [entity, L]).
struct AdjWorkspace {
  // node [N, L] per tracer
  double* ghsc;               // cotangent of the node's flux divergence: gdel * dt / areasvol
  double *gplus, *gminus;     // limiter sums
  double* gLOl;               // LO through the limiter window (-(gtmax + gtmin))
  double *gqx, *gqn;          // cluster bounds divided by their tie counts (one cell's share)
  double *gdiv, *gTp;         // LO's divergence; T through the seed, LO and the bounds
  double *ggnx, *ggny;        // node-average gradients
  double *gfv, *gw;           // vertical LO flux, w_e (per tracer)
  double *gz0, *gzm1, *gzm2, *gzp1;  // interface j's QR4C flux into ttfAB at j, j-1, j-2, j+1
  // edge [Ed, L] per tracer: the per-end cotangents of the edge's fluxes (T at the first /
  // second node through the upwind flux, ttfAB through MFCT, the MFCT gradient factor
  // of each end) and of its volume flux
  double *gT1, *gT2, *gA1, *gA2, *gX1, *gX2, *gvf;
  // element [E, L] per tracer: the element bounds' shares (divided by the vertex tie
  // counts) and the element gradients
  double *gax, *gan, *gtrx, *gtry;
  // [Ed, L], once (not per tracer): the volume-flux cotangents of the calls made with
  // FCT_ADJ_DEFER_UV, summed over their tracers and over the calls
  double* gvf_sum;
  int64_t sN, sE, sEd;
};
constexpr int kAdjNodeFields = 16, kAdjEdgeFields = 7, kAdjElemFields = 4;

}  // namespace fct

struct FctPlan {
  int device = 0;
  // the workspace's last user: every call that writes the plan workspace waits for this
  // event on its own stream and records it afterwards, so calls on different streams do
  // not overlap on the workspace (host threads are serialised by ``mu``)
  std::mutex mu;
  cudaEvent_t ws_ev = nullptr;
  bool ws_used = false;
  unsigned long long* d_health = nullptr;   // non-finite T_new values written since the last
                                            // fct_plan_health

  int N = 0, E = 0, Ed = 0, L = 0;
  fct::DevMesh hm{};               // device pointers (host copy)
  fct::DevMesh* d_mesh = nullptr;  // device copy
  void* d_static = nullptr;        // one allocation for all static arrays
  int max_tracers = 0;
  bool fused = true;               // fct_forward runs the fused stage kernels
  int per_thread = 2;              // fused stages: most tracers per thread
  int lpt = 4;                     //   and levels per thread
  bool ws_full = false;            // workspace holds every stage field (unfused / adjoint)
  double* d_ws = nullptr;          // workspace allocation
  fct::Workspace ws{};
  int64_t n_wet_elem_layers = 0;
  double* d_adj = nullptr;         // reverse-pass workspace
  int adj_tracers = 0;
  cudaStream_t adj_side = nullptr;  // reverse pass: kernels independent of the main chain
  cudaEvent_t adj_ev[5] = {};       //   and the events that fork and join it
  fct::Fork fork{};                 // fused forward: the edge stage beside the LO stage
  fct::AdjWorkspace aws{};
};
