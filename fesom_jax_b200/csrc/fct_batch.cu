// Batched ensemble stepping (fct_batch_* in include/fesom_fct.h).
//
// The reference advances one tracer of one model instance per advect_one_fct call
// (fesom_jax/step.py:409-416, integrate.py:43-169). Here many instances -- ensemble
// members, each with several tracers sharing its velocities, on meshes of different
// sizes -- advance in one launch per stage: blockIdx.y selects the instance from a
// device table, blockIdx.x its lanes. Instances are packed into workspace groups that
// fit a memory budget; groups run back to back on one stream and reuse one arena.
// Multi-step runs are captured once into a CUDA graph and replayed. Tracer buffers and
// workspaces are interleaved ([entity, nl, ntr]): the tracers of one entity-level are
// contiguous, so every gather moves one contiguous chunk; a group holds instances with
// the same ntr.
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <utility>
#include <vector>

#include "fct_host.h"

using namespace fct;

struct FctBatch {
  int device = 0;
  std::vector<FctInstance> insts;
  struct Group {
    int first = 0, count = 0;
    LaunchDims dims{};
    Inst* d_tab[3] = {nullptr, nullptr, nullptr};   // one table per rotation phase
  };
  std::vector<Group> groups;
  double* arena = nullptr;
  int64_t arena_bytes = 0;
  Inst* d_tables = nullptr;
  unsigned long long* d_health = nullptr;   // per-instance non-finite counters
  int64_t total_updates = 0;     // sum over instances of ntr * wet node layers
  std::mutex graph_mu;
  std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
  cudaStream_t cap_stream = nullptr;
  Fork fork{};   // the edge stage beside the LO stage (graph capture and fct_batch_step)
};

static int batch_launch_step(FctBatch* b, int phase, cudaStream_t s) {
  for (auto& g : b->groups) {
    Inst dummy{};
    const int st = launch_forward(dummy, g.d_tab[phase % 3], g.count, g.dims, s);
    if (st) return st;
  }
  return FCT_OK;
}

namespace {

// The kernels index an interleaved array (entity-level x tracer slot) in 32 bits: every
// such array of instance i must hold fewer than 2^32 elements.
int check_interleave(const FctPlan* P, int tg, int wtg, int i) {
  const int64_t ent = std::max({int64_t(P->N), int64_t(P->E), int64_t(P->Ed)});
  if (ent * P->L * std::max(tg, wtg) >= (int64_t(1) << 32))
    return set_error(FCT_ERR_CAPACITY, "instance %d: %lld entity levels x %d tracers exceed "
                     "the 2^32-element interleaved arrays; use fewer tracers per instance", i,
                     (long long)(ent * P->L), std::max(tg, wtg));
  return FCT_OK;
}

}  // namespace

extern "C" {

int fct_batch_create(const FctInstance* insts, int n, int64_t budget, FctBatch** out) {
  if (!out || !insts || n < 1) return set_error(FCT_ERR_INVALID, "bad batch arguments");
  *out = nullptr;
  if (n > 65535) return set_error(FCT_ERR_INVALID, "at most 65535 instances per batch");
  const int dev = insts[0].plan ? insts[0].plan->device : 0;
  std::vector<int64_t> ws_doubles(n);
  std::vector<int> wchunk(n);
  for (int i = 0; i < n; ++i) {
    const FctInstance& q = insts[i];
    if (!q.plan) return set_error(FCT_ERR_INVALID, "instance %d: plan is NULL", i);
    if (q.plan->device != dev)
      return set_error(FCT_ERR_INVALID, "instance %d: all plans must be on one device", i);
    if (q.ntr < 1) return set_error(FCT_ERR_INVALID, "instance %d: ntr < 1", i);
    if (!q.uv || !q.w_e || !q.helem || !q.hnode || !q.hnode_new || !q.buf[0] || !q.buf[1] ||
        !q.buf[2])
      return set_error(FCT_ERR_INVALID, "instance %d: a field pointer is NULL", i);
    if (!(q.dt > 0.0)) return set_error(FCT_ERR_INVALID, "instance %d: dt <= 0", i);
    const FctPlan* P = q.plan;
    // the workspace holds a chunk of the instance's tracers (stages run chunk by chunk):
    // up to 8, halved until one instance fits the budget
    int wc = q.ntr < 8 ? q.ntr : 8;
    while (wc > 1 && workspace_doubles_fused(P->N, P->Ed, P->L, wc) * int64_t(sizeof(double)) > budget)
      wc = (wc + 1) / 2;
    wchunk[i] = wc;
    ws_doubles[i] = workspace_doubles_fused(P->N, P->Ed, P->L, wc);
    const int st = check_interleave(P, q.ntr, wc, i);
    if (st) return st;
  }
  FctBatch* B = new FctBatch();
  B->device = dev;
  B->insts.assign(insts, insts + n);
  // greedy grouping in the given order
  int64_t cur = 0;
  FctBatch::Group g;
  for (int i = 0; i < n; ++i) {
    const int64_t bytes = ws_doubles[i] * int64_t(sizeof(double));
    if (g.count > 0 && (cur + bytes > budget || insts[i].ntr != insts[g.first].ntr ||
                        wchunk[i] != wchunk[g.first])) {
      B->groups.push_back(g);
      g = FctBatch::Group();
      g.first = i;
      cur = 0;
    }
    if (g.count == 0) g.first = i;
    g.count++;
    cur += bytes;
    B->arena_bytes = std::max(B->arena_bytes, cur);
  }
  B->groups.push_back(g);

  auto fail = [&](int st) { fct_batch_destroy(B); return st; };
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(dev);
  cudaError_t e = cudaMalloc(&B->arena, size_t(B->arena_bytes));
  if (e != cudaSuccess) {
    if (prev >= 0) cudaSetDevice(prev);
    return fail(cuda_error(e, "batch workspace cudaMalloc"));
  }
  // host tables: [phase][instance]
  std::vector<Inst> tab(size_t(3) * n);
  for (auto& gr : B->groups) {
    int64_t off = 0;
    LaunchDims d{};
    for (int i = gr.first; i < gr.first + gr.count; ++i) {
      const FctInstance& q = insts[i];
      const FctPlan* P = q.plan;
      const Workspace ws =
          carve_workspace(B->arena + off, P->N, P->E, P->Ed, P->L, wchunk[i], /*fused=*/true);
      off += ws_doubles[i];
      dims_cover(d, P);
      d.ntr = q.ntr;
      d.chunk = wchunk[i];
      B->total_updates += int64_t(q.ntr) * P->hm.n_layer;
      for (int p = 0; p < 3; ++p) {
        Inst& in = tab[size_t(p) * n + i];
        in.m = P->d_mesh;
        in.uv = q.uv; in.w_e = q.w_e; in.helem = q.helem;
        in.hnode = q.hnode; in.hnode_new = q.hnode_new;
        in.T_old = q.buf[p % 3];
        in.T = q.buf[(p + 1) % 3];
        in.T_new = q.buf[(p + 2) % 3];
        in.tstride = 0;
        in.tg = q.ntr;   // interleaved [nod2D, nl, ntr]
        in.wtg = wchunk[i];
        in.Z3d = in.zbar3 = in.w_i = nullptr;
        in.ws = ws;
        in.dt = q.dt;
        in.ntr = q.ntr;
        in.w_derived = q.w_derived;   // optional producer: w_e = compute_w(uv, helem)
        if (q.w_derived) {
          in.w_e = q.w_derived;
          d.any_derive_w = true;
        }
        in.Kv = q.Kv;   // optional diffusion epilogue, in place on T_new
        in.vd_T = in.T_new;
        in.sw_tracer = -1;
        if (q.Kv) d.any_vdiff = true;
      }
    }
    d.any_wi = false;
    d.copy_dry = false;
    d.per_thread = std::min(d.chunk, 2);
    d.set_map(d.per_thread, 4);
    gr.dims = d;
  }
  e = cudaMalloc(&B->d_health, size_t(n) * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(B->d_health, 0, size_t(n) * sizeof(unsigned long long));
  for (int i = 0; i < n && e == cudaSuccess; ++i)
    for (int p = 0; p < 3; ++p)
      tab[size_t(p) * n + i].nonfinite = insts[i].nonfinite ? insts[i].nonfinite
                                                           : B->d_health + i;
  if (e == cudaSuccess) e = cudaMalloc(&B->d_tables, tab.size() * sizeof(Inst));
  if (e == cudaSuccess)
    e = cudaMemcpy(B->d_tables, tab.data(), tab.size() * sizeof(Inst), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&B->cap_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    if (prev >= 0) cudaSetDevice(prev);
    return fail(cuda_error(e, "batch table setup"));
  }
  const int fst = fork_create(B->fork);
  if (prev >= 0) cudaSetDevice(prev);
  if (fst) return fail(fst);
  for (auto& gr : B->groups) gr.dims.fork = &B->fork;
  for (auto& gr : B->groups)
    for (int p = 0; p < 3; ++p) gr.d_tab[p] = B->d_tables + size_t(p) * n + gr.first;
  *out = B;
  return FCT_OK;
}

int fct_batch_destroy(FctBatch* B) {
  if (!B) return FCT_OK;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(B->device);
  for (auto& kv : B->graphs) cudaGraphExecDestroy(kv.second);
  if (B->cap_stream) cudaStreamDestroy(B->cap_stream);
  fork_destroy(B->fork);
  if (B->d_tables) cudaFree(B->d_tables);
  if (B->d_health) cudaFree(B->d_health);
  if (B->arena) cudaFree(B->arena);
  if (prev >= 0) cudaSetDevice(prev);
  delete B;
  return FCT_OK;
}

int fct_batch_set_mapping(FctBatch* B, int tracers_per_thread, int levels_per_thread) {
  if (!B) return set_error(FCT_ERR_INVALID, "batch is NULL");
  const int t = tracers_per_thread, l = levels_per_thread;
  if ((t != 1 && t != 2 && t != 4 && t != 8) || (l != 1 && l != 2 && l != 4 && l != 8))
    return set_error(FCT_ERR_INVALID, "tracers and levels per thread must be 1, 2, 4 or 8");
  std::lock_guard<std::mutex> lk(B->graph_mu);
  for (auto& g : B->groups) {
    g.dims.per_thread = t;
    g.dims.set_map(t, l);
  }
  for (auto& kv : B->graphs) cudaGraphExecDestroy(kv.second);   // recapture with the mapping
  B->graphs.clear();
  return FCT_OK;
}

int fct_batch_set_chunk(FctBatch* B, int chunk) {
  if (!B) return set_error(FCT_ERR_INVALID, "batch is NULL");
  const int lpt = B->groups.empty() ? 4 : B->groups[0].dims.smap_levels[0];
  return fct_batch_set_mapping(B, chunk, lpt);
}

int fct_batch_set_stage_mapping(FctBatch* B, int stage, int tracers_per_thread,
                                int levels_per_thread) {
  if (!B) return set_error(FCT_ERR_INVALID, "batch is NULL");
  if (stage < 0 || stage >= kFusedStages)
    return set_error(FCT_ERR_INVALID, "stage must be 0 (LO), 1 (edge), 2 (limiter) or 3 "
                     "(final)");
  const int t = tracers_per_thread, l = levels_per_thread;
  if ((t != 1 && t != 2 && t != 4 && t != 8) || (l != 1 && l != 2 && l != 4 && l != 8))
    return set_error(FCT_ERR_INVALID, "tracers and levels per thread must be 1, 2, 4 or 8");
  std::lock_guard<std::mutex> lk(B->graph_mu);
  for (auto& g : B->groups) {
    g.dims.smap_tracers[stage] = t;
    g.dims.smap_levels[stage] = l;
  }
  for (auto& kv : B->graphs) cudaGraphExecDestroy(kv.second);   // recapture with the mapping
  B->graphs.clear();
  return FCT_OK;
}

int fct_batch_info(const FctBatch* B, int64_t out[6]) {
  if (!B || !out) return set_error(FCT_ERR_INVALID, "NULL argument");
  out[0] = int64_t(B->insts.size());
  out[1] = int64_t(B->groups.size());
  out[2] = B->arena_bytes;
  out[3] = B->total_updates;
  int64_t wmax = 0, launches = 0;
  for (const auto& g : B->groups) {
    const int chunk = g.dims.chunk > 0 ? g.dims.chunk : g.dims.ntr;
    wmax = std::max<int64_t>(wmax, chunk);
    int64_t per_chunk_launches = 0;
    for (int c0 = 0; c0 < g.dims.ntr; c0 += chunk) {
      const int csz = std::min(chunk, g.dims.ntr - c0);
      per_chunk_launches += stage_launches(csz, g.dims.per_thread);
    }
    const int stages = (g.dims.fused ? 4 + (g.dims.max_efix > 0 ? 1 : 0) : 7) +
                       (g.dims.any_wi ? 1 : 0) + (g.dims.any_vdiff ? 1 : 0);
    launches += 1 + (g.dims.any_derive_w ? 1 : 0) + int64_t(stages) * per_chunk_launches;
  }
  out[4] = wmax;
  out[5] = launches;
  return FCT_OK;
}

int fct_batch_prepare(FctBatch* B, fct_stream_t stream) {
  if (!B) return set_error(FCT_ERR_INVALID, "batch is NULL");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(B->device);
  int st = FCT_OK;
  // phase 0 copies buf[1] -> buf[2]; phase 1 then copies buf[2] -> buf[0]
  for (int p = 0; p < 2 && !st; ++p)
    for (auto& g : B->groups)
      if ((st = launch_copy_dry(g.d_tab[p], g.count, g.dims.max_dry, s))) break;
  if (prev >= 0) cudaSetDevice(prev);
  return st;
}

int fct_batch_step(FctBatch* B, int phase, fct_stream_t stream) {
  if (!B) return set_error(FCT_ERR_INVALID, "batch is NULL");
  if (phase < 0) return set_error(FCT_ERR_INVALID, "phase must be >= 0");
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(B->device);
  const int st = batch_launch_step(B, phase, static_cast<cudaStream_t>(stream));
  if (prev >= 0) cudaSetDevice(prev);
  return st;
}

int fct_batch_run(FctBatch* B, int first_phase, int steps, fct_stream_t stream) {
  if (!B) return set_error(FCT_ERR_INVALID, "batch is NULL");
  if (steps < 1 || first_phase < 0) return set_error(FCT_ERR_INVALID, "bad steps/phase");
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(B->device);
  auto restore = [&](int st) { if (prev >= 0) cudaSetDevice(prev); return st; };
  cudaGraphExec_t exec = nullptr;
  {
    std::lock_guard<std::mutex> lk(B->graph_mu);
    auto key = std::make_pair(first_phase % 3, steps);
    auto it = B->graphs.find(key);
    if (it != B->graphs.end()) {
      exec = it->second;
    } else {
      cudaError_t e = cudaStreamBeginCapture(B->cap_stream, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return restore(cuda_error(e, "cudaStreamBeginCapture"));
      int st = FCT_OK;
      for (int k = 0; k < steps && !st; ++k) st = batch_launch_step(B, first_phase + k, B->cap_stream);
      cudaGraph_t graph = nullptr;
      e = cudaStreamEndCapture(B->cap_stream, &graph);
      if (st) { if (graph) cudaGraphDestroy(graph); return restore(st); }
      if (e != cudaSuccess) return restore(cuda_error(e, "cudaStreamEndCapture"));
      e = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) return restore(cuda_error(e, "cudaGraphInstantiate"));
      B->graphs[key] = exec;
    }
  }
  cudaError_t e = cudaGraphLaunch(exec, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return restore(cuda_error(e, "cudaGraphLaunch"));
  return restore(FCT_OK);
}

int fct_batch_fill_workspace(FctBatch* B, int byte, fct_stream_t stream) {
  if (!B) return set_error(FCT_ERR_INVALID, "batch is NULL");
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(B->device);
  const cudaError_t e = cudaMemsetAsync(B->arena, byte & 0xff, size_t(B->arena_bytes),
                                        static_cast<cudaStream_t>(stream));
  if (prev >= 0) cudaSetDevice(prev);
  return e == cudaSuccess ? FCT_OK : cuda_error(e, "batch workspace fill");
}

int fct_batch_health(FctBatch* B, fct_stream_t stream, int64_t* counts) {
  if (!B) return set_error(FCT_ERR_INVALID, "batch is NULL");
  const int n = int(B->insts.size());
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(B->device);
  auto restore = [&](int st) { if (prev >= 0) cudaSetDevice(prev); return st; };
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  std::vector<unsigned long long> h(size_t(n), 0ull);
  cudaError_t e = cudaMemcpyAsync(h.data(), B->d_health, size_t(n) * sizeof(h[0]),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaMemsetAsync(B->d_health, 0, size_t(n) * sizeof(h[0]), s);
  if (e != cudaSuccess) return restore(cuda_error(e, "batch health read"));
  unsigned long long total = 0;
  int first = -1;
  for (int i = 0; i < n; ++i) {
    if (counts) counts[i] = int64_t(h[size_t(i)]);
    if (h[size_t(i)] && first < 0) first = i;
    total += h[size_t(i)];
  }
  if (total)
    return restore(set_error(FCT_ERR_NONFINITE, "%llu non-finite T_new values since the last "
                             "check (first in instance %d)", total, first));
  return restore(FCT_OK);
}

int fct_batch_profile(FctBatch* B, int phase, double* stage_ms, int max_stages,
                      fct_stream_t stream) {
  if (!B || !stage_ms) return set_error(FCT_ERR_INVALID, "NULL argument");
  if (max_stages < kNumStages)
    return set_error(FCT_ERR_INVALID, "stage_ms needs %d entries", kNumStages);
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(B->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaEvent_t ev[kNumStages + 1];
  for (auto& e : ev) cudaEventCreate(&e);
  for (int i = 0; i < kNumStages; ++i) stage_ms[i] = 0.0;
  int st = FCT_OK;
  for (auto& g : B->groups) {
    const int chunk = g.dims.chunk > 0 ? g.dims.chunk : g.dims.ntr;
    const int nchunks = (g.dims.ntr + chunk - 1) / chunk;
    for (int ci = 0; ci < nchunks && !st; ++ci) {
      Inst dummy{};
      cudaEventRecord(ev[0], s);
      st = launch_forward_events(dummy, g.d_tab[phase % 3], g.count, g.dims, s, ev + 1, false, ci);
      if (st) break;
      cudaError_t e = cudaEventSynchronize(ev[kNumStages]);
      if (e != cudaSuccess) { st = cuda_error(e, "profile synchronize"); break; }
      for (int i = 0; i < kNumStages; ++i) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
        stage_ms[i] += ms;
      }
    }
    if (st) break;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (prev >= 0) cudaSetDevice(prev);
  return st;
}

}  // extern "C"

struct FctServe {
  int device = 0;
  int max_instances = 0;
  double* arena = nullptr;
  int64_t arena_doubles = 0;
  Inst* d_tab = nullptr;      // device instance table (rewritten in stream order per call)
  // pinned staging ring: a call fills the next slot and waits only for that slot's previous
  // upload, so the host can enqueue several calls ahead of the GPU
  static constexpr int kRing = 16;
  Inst* h_tab[kRing] = {};
  cudaEvent_t uploaded[kRing] = {};
  bool pending[kRing] = {};   // an upload from h_tab[i] may still be in flight
  int next = 0;
  unsigned long long* d_health = nullptr;   // non-finite counter of instances without one
};

extern "C" {

int fct_serve_create(int device, int max_instances, int64_t workspace_bytes, FctServe** out) {
  if (!out || max_instances < 1 || workspace_bytes < 0)
    return set_error(FCT_ERR_INVALID, "bad serve arguments");
  *out = nullptr;
  int prev = -1;
  cudaGetDevice(&prev);
  FctServe* S = new FctServe();
  S->device = device;
  S->max_instances = max_instances;
  S->arena_doubles = workspace_bytes / int64_t(sizeof(double));
  auto fail = [&](cudaError_t e, const char* what) {
    const int st = cuda_error(e, what);
    fct_serve_destroy(S);
    if (prev >= 0) cudaSetDevice(prev);
    return st;
  };
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(e, "cudaSetDevice");
  if (S->arena_doubles > 0 &&
      (e = cudaMalloc(&S->arena, size_t(S->arena_doubles) * sizeof(double))) != cudaSuccess)
    return fail(e, "serve workspace cudaMalloc");
  if ((e = cudaMalloc(&S->d_tab, size_t(max_instances) * sizeof(Inst))) != cudaSuccess)
    return fail(e, "serve table cudaMalloc");
  for (int i = 0; i < FctServe::kRing; ++i) {
    if ((e = cudaMallocHost(&S->h_tab[i], size_t(max_instances) * sizeof(Inst))) != cudaSuccess)
      return fail(e, "serve staging cudaMallocHost");
    if ((e = cudaEventCreateWithFlags(&S->uploaded[i], cudaEventDisableTiming)) != cudaSuccess)
      return fail(e, "cudaEventCreate");
  }
  if ((e = cudaMalloc(&S->d_health, sizeof(unsigned long long))) != cudaSuccess ||
      (e = cudaMemset(S->d_health, 0, sizeof(unsigned long long))) != cudaSuccess)
    return fail(e, "serve health counter");
  if (prev >= 0) cudaSetDevice(prev);
  *out = S;
  return FCT_OK;
}

int fct_serve_destroy(FctServe* S) {
  if (!S) return FCT_OK;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(S->device);
  for (int i = 0; i < FctServe::kRing; ++i) {
    if (S->uploaded[i]) {
      cudaEventSynchronize(S->uploaded[i]);
      cudaEventDestroy(S->uploaded[i]);
    }
    if (S->h_tab[i]) cudaFreeHost(S->h_tab[i]);
  }
  if (S->d_tab) cudaFree(S->d_tab);
  if (S->d_health) cudaFree(S->d_health);
  if (S->arena) cudaFree(S->arena);
  if (prev >= 0) cudaSetDevice(prev);
  delete S;
  return FCT_OK;
}

int fct_serve_step(FctServe* S, const FctInstance* insts, const int32_t* phases, int n,
                   fct_stream_t stream) {
  if (!S || (n > 0 && (!insts || !phases))) return set_error(FCT_ERR_INVALID, "NULL argument");
  if (n < 0 || n > S->max_instances)
    return set_error(FCT_ERR_CAPACITY, "%d instances exceed the serve table (%d)", n,
                     S->max_instances);
  if (n == 0) return FCT_OK;
  // order instances by (ntr, mesh): a launch group holds one ntr and one mesh, so its
  // grid is sized for that mesh (a pi-size instance never rides a 1.3M-node grid)
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  auto key = [&](int i) {
    const FctPlan* P = insts[i].plan;
    return std::make_tuple(insts[i].ntr, P ? P->hm.n_layer : 0, reinterpret_cast<uintptr_t>(P));
  };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key(a) < key(b); });
  int64_t need = 0;
  for (int i = 0; i < n; ++i) {
    const FctInstance& q = insts[i];
    if (!q.plan || q.plan->device != S->device || q.ntr < 1 || !q.buf[0] || !q.buf[1] ||
        !q.buf[2] || !q.uv || !q.w_e || !q.helem || !q.hnode || !q.hnode_new || !(q.dt > 0.0))
      return set_error(FCT_ERR_INVALID, "instance %d is invalid", i);
    const int st = check_interleave(q.plan, q.ntr, q.ntr, i);
    if (st) return st;
    need += workspace_doubles_fused(q.plan->N, q.plan->Ed, q.plan->L, q.ntr);
  }
  if (need > S->arena_doubles)
    return set_error(FCT_ERR_CAPACITY, "instances need %lld workspace doubles, arena holds %lld",
                     (long long)need, (long long)S->arena_doubles);
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(S->device);
  auto restore = [&](int st) { if (prev >= 0) cudaSetDevice(prev); return st; };
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int slot = S->next;
  Inst* h_tab = S->h_tab[slot];
  if (S->pending[slot]) {   // that slot's previous upload must have left the staging buffer
    cudaError_t e = cudaEventSynchronize(S->uploaded[slot]);
    if (e != cudaSuccess) return restore(cuda_error(e, "serve staging wait"));
  }
  int64_t off = 0;
  for (int j = 0; j < n; ++j) {
    const FctInstance& q = insts[order[j]];
    const FctPlan* P = q.plan;
    const int p = ((phases[order[j]] % 3) + 3) % 3;
    Inst& in = h_tab[j];
    in = Inst{};
    in.m = P->d_mesh;
    in.uv = q.uv; in.w_e = q.w_e; in.helem = q.helem;
    in.hnode = q.hnode; in.hnode_new = q.hnode_new;
    in.T_old = q.buf[p];
    in.T = q.buf[(p + 1) % 3];
    in.T_new = q.buf[(p + 2) % 3];
    in.tstride = 0;
    in.tg = q.ntr;
    in.wtg = q.ntr;
    in.ws = carve_workspace(S->arena + off, P->N, P->E, P->Ed, P->L, q.ntr, /*fused=*/true);
    off += workspace_doubles_fused(P->N, P->Ed, P->L, q.ntr);
    in.dt = q.dt;
    in.ntr = q.ntr;
    in.nonfinite = q.nonfinite ? q.nonfinite : S->d_health;
    if (q.w_derived) {   // producer: w_e = compute_w(uv, helem) at this step
      in.w_derived = q.w_derived;
      in.w_e = q.w_derived;
    }
  }
  cudaError_t e = cudaMemcpyAsync(S->d_tab, h_tab, size_t(n) * sizeof(Inst),
                                  cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return restore(cuda_error(e, "serve table upload"));
  e = cudaEventRecord(S->uploaded[slot], s);
  if (e != cudaSuccess) return restore(cuda_error(e, "serve event record"));
  S->pending[slot] = true;
  S->next = (slot + 1) % FctServe::kRing;
  for (int j0 = 0; j0 < n;) {
    int j1 = j0;
    LaunchDims d{};
    const int ntr = insts[order[j0]].ntr;
    const FctPlan* P0 = insts[order[j0]].plan;
    while (j1 < n && insts[order[j1]].ntr == ntr && insts[order[j1]].plan == P0) {
      dims_cover(d, insts[order[j1]].plan);
      ++j1;
    }
    d.ntr = ntr;
    d.chunk = 0;
    d.per_thread = P0->per_thread;
    d.set_map(P0->per_thread, P0->lpt);
    for (int j = j0; j < j1; ++j)
      if (insts[order[j]].w_derived) d.any_derive_w = true;
    d.any_wi = false;
    d.copy_dry = false;
    Inst dummy{};
    const int st = launch_forward(dummy, S->d_tab + j0, j1 - j0, d, s);
    if (st) return restore(st);
    j0 = j1;
  }
  return restore(FCT_OK);
}

int fct_serve_health(FctServe* S, fct_stream_t stream, int64_t* n_nonfinite) {
  if (!S) return set_error(FCT_ERR_INVALID, "serve engine is NULL");
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(S->device);
  const int st = read_health(S->d_health, 1, static_cast<cudaStream_t>(stream), n_nonfinite);
  if (prev >= 0) cudaSetDevice(prev);
  return st;
}

const char* fct_stage_name(int i) {
  return (i >= 0 && i < kNumStages) ? kStageNames[i] : "";
}

}  // extern "C"
