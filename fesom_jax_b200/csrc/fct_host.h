// Host-side helpers shared by the libfesom_fct translation units.
#pragma once

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <string>

#include <cuda_runtime.h>

#include "fct_internal.cuh"

namespace fct {

// Record the calling thread's last error and return ``status``.
int set_error(int status, const char* fmt, ...);

inline int cuda_error(cudaError_t e, const char* what) {
  return set_error(FCT_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define FCT_CUDA(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return ::fct::cuda_error(e_, #call); \
  } while (0)

// fused stages with their own thread mapping: LO, edge, limiter, final
constexpr int kFusedStages = 4;
enum { kStageLo = 0, kStageEdge = 1, kStageLimit = 2, kStageFinal = 3 };

// Launch the forward kernel sequence for ``n`` instances. ``single`` is used when
// ``tab`` is null (n == 1), otherwise ``tab`` is a device array of ``n`` instances
// whose lane counts are bounded by the ``max_*`` arguments.
struct LaunchDims {
  int64_t max_iface, max_layer, max_edge, max_elem, max_dense, max_nodes;
  int64_t max_dry = 0;   // dry node levels (kept from T)
  int ntr;           // tracers per instance (every instance of a launch has the same)
  int chunk = 0;     // tracers whose intermediates share the workspace (0 = all ntr);
                     // stages run chunk by chunk
  int per_thread = 8;  // most tracers one thread carries (8, 4, 2 or 1): the tuning knob
  bool any_wi;      // launch the implicit w_i stage
  bool copy_dry;    // launch the dry-level copy
  bool any_vdiff = false;  // launch the implicit vertical diffusion after each chunk
  bool any_derive_w = false;  // derive w_e from uv (compute_w) before the step
  bool skip_vflux = false;    // the workspace already holds this step's volume fluxes
  bool fused = true;  // fused stages (lean workspace); false: every stage kernel writes its
                      // intermediates (what the reverse pass reads)
  // fused (segment) stages: per stage (LO, edge, limiter, final) the most tracers and the
  // levels a thread takes (tuning knobs), and the largest segment counts over the launch's
  // instances
  int smap_tracers[kFusedStages] = {2, 2, 2, 2};
  int smap_levels[kFusedStages] = {4, 4, 4, 4};
  void set_map(int tracers, int levels) {
    for (int i = 0; i < kFusedStages; ++i) {
      smap_tracers[i] = tracers;
      smap_levels[i] = levels;
    }
  }
  int64_t max_nseg[kSegVariants] = {0, 0, 0, 0};
  int64_t max_eseg[kSegVariants] = {0, 0, 0, 0};
  int64_t max_efix = 0;
  // fused path: run the edge stage on fork->side beside the LO stage (null: one stream)
  const Fork* fork = nullptr;
};

// Create / release a Fork on the current device.
int fork_create(Fork& f);
void fork_destroy(Fork& f);

// Grow ``d``'s lane and segment counts to cover a plan's mesh.
inline void dims_cover(LaunchDims& d, const FctPlan* P) {
  const DevMesh& m = P->hm;
  d.max_iface = std::max(d.max_iface, m.n_iface);
  d.max_layer = std::max(d.max_layer, m.n_layer);
  d.max_edge = std::max(d.max_edge, m.n_edge);
  d.max_elem = std::max(d.max_elem, m.n_elem);
  d.max_dense = std::max(d.max_dense, int64_t(P->N) * P->L);
  d.max_dry = std::max(d.max_dry, P->hm.n_dry);
  d.max_nodes = std::max(d.max_nodes, int64_t(P->N));
  for (int v = 0; v < kSegVariants; ++v) {
    d.max_nseg[v] = std::max(d.max_nseg[v], m.n_nseg[v]);
    d.max_eseg[v] = std::max(d.max_eseg[v], m.n_eseg[v]);
  }
  d.max_efix = std::max(d.max_efix, m.n_efix);
}

// The fused stages over the tracers [c0, c1) of a workspace chunk (fct_seg_*.cu).
int launch_seg_lo(const Inst& single, const Inst* tab, int n, const LaunchDims& d, int c0,
                  int c1, cudaStream_t s);
int launch_seg_edge(const Inst& single, const Inst* tab, int n, const LaunchDims& d, int c0,
                    int c1, cudaStream_t s);
int launch_edge_fix(const Inst& single, const Inst* tab, int n, const LaunchDims& d, int c0,
                    int c1, cudaStream_t s);
int launch_seg_limit(const Inst& single, const Inst* tab, int n, const LaunchDims& d, int c0,
                     int c1, cudaStream_t s);
int launch_seg_final(const Inst& single, const Inst* tab, int n, const LaunchDims& d, int c0,
                     int c1, cudaStream_t s);
int launch_forward(const Inst& single, const Inst* tab, int n, const LaunchDims& d,
                   cudaStream_t s);
// Same, recording ``after[i]`` on ``s`` after stage i of a chunk (skipped stages record
// too); ``chunk_sel >= 0`` launches only that workspace chunk.
constexpr int kNumStages = 10;
extern const char* const kStageNames[kNumStages];
int launch_forward_events(const Inst& single, const Inst* tab, int n, const LaunchDims& d,
                          cudaStream_t s, cudaEvent_t* after, bool stop_before_final = false,
                          int chunk_sel = -1);
// Single-instance forward stages; ``through_factors`` stops after the limiter factors
// (everything the reverse pass reads), without writing T_new.
int launch_forward_stages(const Inst& single, const LaunchDims& d, cudaStream_t s,
                          bool through_factors);
// fct_plan_reserve (declared in the public header) is used by the adjoint reservation.

// Copy T's dry levels into T_new for ``n`` instances of ``tab`` (ignores Inst::copy_dry).
int launch_copy_dry(const Inst* tab, int n, int64_t max_dry, cudaStream_t s);
// compute_w of every table instance with w_derived set (fct_producers.cu).
int launch_compute_w_tab(const Inst* tab, int n, int64_t max_nodes, cudaStream_t s);
// Implicit vertical diffusion alone (fct_vert_diff): single instance, tracer-major.
int launch_vdiff(const Inst& single, const LaunchDims& d, cudaStream_t s);

// Workspace of `ntr` tracers: every stage field (the unfused stages, which the reverse
// pass recomputes and reads), or with `fused` only the fields the fused forward keeps.
Workspace carve_workspace(double* base, int64_t N, int64_t E, int64_t Ed, int64_t L, int ntr,
                          bool fused = false);
int64_t workspace_doubles(int64_t N, int64_t E, int64_t Ed, int64_t L, int ntr);
int64_t workspace_doubles_fused(int64_t N, int64_t Ed, int64_t L, int ntr);
// Grow the plan workspace to `ntr` tracers; `full` also makes it hold every stage field.
int plan_reserve_ws(FctPlan* P, int ntr, bool full);
// A plan created by fct_plan_create in this process and not destroyed yet.
bool plan_alive(const FctPlan* P);

// Ordering of the calls that use a plan's workspace: hold ``P->mu`` (PlanUse does), wait
// on stream ``s`` for the previous user, launch, then record the release on ``s``. Both
// are skipped while ``s`` is being captured into a CUDA graph (an event from outside a
// capture cannot be waited on inside it): captured calls are ordered by their graph.
class PlanUse {
 public:
  PlanUse(FctPlan* P, cudaStream_t s);
  // record the release event (call after the launches; returns a status)
  int release();
  int status() const { return st_; }

 private:
  std::lock_guard<std::mutex> lk_;
  FctPlan* P_;
  cudaStream_t s_;
  bool capturing_ = false;
  int st_ = 0;
};

// Copy a device counter to the host on ``s``, wait, zero it, and return FCT_ERR_NONFINITE
// when it was non-zero (``out`` receives the count when not NULL).
int read_health(unsigned long long* d_counter, int n, cudaStream_t s, int64_t* out);

// Launches one stage takes for `csz` tracers of a workspace chunk with at most
// `per_thread` tracers per thread (the split rule of the stage launcher).
inline int stage_launches(int csz, int per_thread) {
  int count = 0;
  for (int t = 0; t < csz;) {
    const int rem = csz - t, lim = rem < per_thread ? rem : per_thread;
    const int P = lim >= 8 ? 8 : lim >= 4 ? 4 : lim >= 2 ? 2 : 1;
    int lg = 0;
    while (lg < 3 && (P << (lg + 1)) <= rem) ++lg;
    t += P << lg;
    ++count;
  }
  return count;
}

}  // namespace fct
