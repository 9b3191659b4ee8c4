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
  int64_t total_updates = 0;     // sum over instances of ntr * wet node layers
  std::mutex graph_mu;
  std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
  cudaStream_t cap_stream = nullptr;
};

static int batch_launch_step(FctBatch* b, int phase, cudaStream_t s) {
  for (auto& g : b->groups) {
    Inst dummy{};
    const int st = launch_forward(dummy, g.d_tab[phase % 3], g.count, g.dims, s);
    if (st) return st;
  }
  return FCT_OK;
}

extern "C" {

int fct_batch_create(const FctInstance* insts, int n, int64_t budget, FctBatch** out) {
  if (!out || !insts || n < 1) return set_error(FCT_ERR_INVALID, "bad batch arguments");
  *out = nullptr;
  if (n > 65535) return set_error(FCT_ERR_INVALID, "at most 65535 instances per batch");
  const int dev = insts[0].plan ? insts[0].plan->device : 0;
  std::vector<int64_t> ws_doubles(n);
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
    ws_doubles[i] = workspace_doubles(P->N, P->E, P->Ed, P->L, q.ntr);
  }
  FctBatch* B = new FctBatch();
  B->device = dev;
  B->insts.assign(insts, insts + n);
  // greedy grouping in the given order
  int64_t cur = 0;
  FctBatch::Group g;
  for (int i = 0; i < n; ++i) {
    const int64_t bytes = ws_doubles[i] * int64_t(sizeof(double));
    if (g.count > 0 && (cur + bytes > budget || insts[i].ntr != insts[g.first].ntr)) {
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
      const Workspace ws = carve_workspace(B->arena + off, P->N, P->E, P->Ed, P->L, q.ntr);
      off += ws_doubles[i];
      d.max_iface = std::max(d.max_iface, P->hm.n_iface);
      d.max_layer = std::max(d.max_layer, P->hm.n_layer);
      d.max_edge = std::max(d.max_edge, P->hm.n_edge);
      d.max_elem = std::max(d.max_elem, P->hm.n_elem);
      d.max_dense = std::max(d.max_dense, int64_t(P->N) * P->L);
      d.max_nodes = std::max(d.max_nodes, int64_t(P->N));
      d.ntr = q.ntr;
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
        in.Z3d = in.zbar3 = in.w_i = nullptr;
        in.ws = ws;
        in.dt = q.dt;
        in.ntr = q.ntr;
      }
    }
    d.any_wi = false;
    d.copy_dry = false;
    d.chunk = 8;
    gr.dims = d;
  }
  e = cudaMalloc(&B->d_tables, tab.size() * sizeof(Inst));
  if (e == cudaSuccess)
    e = cudaMemcpy(B->d_tables, tab.data(), tab.size() * sizeof(Inst), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&B->cap_stream, cudaStreamNonBlocking);
  if (prev >= 0) cudaSetDevice(prev);
  if (e != cudaSuccess) return fail(cuda_error(e, "batch table setup"));
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
  if (B->d_tables) cudaFree(B->d_tables);
  if (B->arena) cudaFree(B->arena);
  if (prev >= 0) cudaSetDevice(prev);
  delete B;
  return FCT_OK;
}

int fct_batch_set_chunk(FctBatch* B, int chunk) {
  if (!B) return set_error(FCT_ERR_INVALID, "batch is NULL");
  if (chunk != 1 && chunk != 2 && chunk != 4 && chunk != 8)
    return set_error(FCT_ERR_INVALID, "chunk must be 1, 2, 4 or 8");
  std::lock_guard<std::mutex> lk(B->graph_mu);
  for (auto& g : B->groups) g.dims.chunk = chunk;
  for (auto& kv : B->graphs) cudaGraphExecDestroy(kv.second);   // recapture with the new chunk
  B->graphs.clear();
  return FCT_OK;
}

int fct_batch_info(const FctBatch* B, int64_t out[4]) {
  if (!B || !out) return set_error(FCT_ERR_INVALID, "NULL argument");
  out[0] = int64_t(B->insts.size());
  out[1] = int64_t(B->groups.size());
  out[2] = B->arena_bytes;
  out[3] = B->total_updates;
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
      if ((st = launch_copy_dry(g.d_tab[p], g.count, g.dims.max_dense, s))) break;
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
    Inst dummy{};
    cudaEventRecord(ev[0], s);
    st = launch_forward_events(dummy, g.d_tab[phase % 3], g.count, g.dims, s, ev + 1);
    if (st) break;
    cudaError_t e = cudaEventSynchronize(ev[kNumStages]);
    if (e != cudaSuccess) { st = cuda_error(e, "profile synchronize"); break; }
    for (int i = 0; i < kNumStages; ++i) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
      stage_ms[i] += ms;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (prev >= 0) cudaSetDevice(prev);
  return st;
}

const char* fct_stage_name(int i) {
  return (i >= 0 && i < kNumStages) ? kStageNames[i] : "";
}

}  // extern "C"
