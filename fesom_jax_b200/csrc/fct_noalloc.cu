// fct_forward_noalloc: the FCT forward step with its scratch in a fixed device array.
//
// Who needs it: code that runs where device allocation is not allowed or not safe.
// An XLA/JAX custom-call handler executes inside a runtime that owns (and usually
// preallocates) the GPU's memory, so a cudaMalloc there competes with or fails under
// that pool; a latency-bound serving loop should never block on the allocator. Such
// callers can create a plan once at set-up time, but at call time they can only hand
// over the inputs and outputs they were given.
//
// This entry point runs the fused stage kernels of fct_forward (always the fused ones,
// whatever fct_plan_set_fused chose for the plan), but their intermediates live in
// ``g_fct_static_scratch``, a file-scope __device__ array of kStaticScratchDoubles
// doubles (64 MiB) that every GPU which loads the library holds until the process exits.
// Nothing here calls cudaMalloc, cudaFree or any allocating library routine. Sizes whose
// scratch need exceeds the array are rejected with FCT_ERR_CAPACITY.
//
// The array's name is only a host-side stand-in in host code, so its device address is
// looked up once per device (cudaGetSymbolAddress, with that device current) on the
// first call on that device; make that first call before any stream capture. Every call
// shares the one array and the array keeps the last call's contents: the kernels read
// only scratch entries written earlier in the same call, so nothing needs clearing, but
// two calls that overlap on the GPU (different streams, or different host threads without
// ordering) race on it and corrupt each other's results.
#include <mutex>

#include "fct_host.h"

namespace {

constexpr int64_t kStaticScratchDoubles = int64_t(8) << 20;   // 64 MiB
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_fct_static_scratch[kStaticScratchDoubles];

std::mutex g_scratch_mu;
double* g_scratch_ptr[kMaxDevices] = {};

}  // namespace

using namespace fct;

extern "C" int fct_forward_noalloc(FctPlan* P, const FctFields* f, double dt, int ntr,
                                   fct_stream_t stream) {
  if (!P || !f) return set_error(FCT_ERR_INVALID, "NULL plan or fields");
  if (ntr < 1) return set_error(FCT_ERR_INVALID, "ntr must be >= 1");
  if (!f->uv || !f->w_e || !f->helem || !f->hnode || !f->hnode_new || !f->T ||
      !f->T_old || !f->T_new)
    return set_error(FCT_ERR_INVALID, "a required field pointer is NULL");
  if ((f->Z3d == nullptr) != (f->zbar3 == nullptr))
    return set_error(FCT_ERR_INVALID, "Z3d and zbar3 must be given together");
  if (!(dt > 0.0)) return set_error(FCT_ERR_INVALID, "dt must be positive");
  if (P->device < 0 || P->device >= kMaxDevices)
    return set_error(FCT_ERR_INVALID, "device %d out of range", P->device);
  const int64_t need = workspace_doubles_fused(P->N, P->Ed, P->L, ntr);
  if (need > kStaticScratchDoubles)
    return set_error(FCT_ERR_CAPACITY,
                     "fct_forward_noalloc: %d tracers on this mesh need %lld doubles of "
                     "scratch; the static array holds %lld (64 MiB); use fct_forward",
                     ntr, (long long)need, (long long)kStaticScratchDoubles);
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != P->device) cudaSetDevice(P->device);
  auto restore = [&](int st) {
    if (prev >= 0 && prev != P->device) cudaSetDevice(prev);
    return st;
  };
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[P->device]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_fct_static_scratch);
      if (e != cudaSuccess) return restore(cuda_error(e, "cudaGetSymbolAddress(static scratch)"));
      g_scratch_ptr[P->device] = static_cast<double*>(p);
    }
    scratch = g_scratch_ptr[P->device];
  }
  Inst in{};
  in.m = P->d_mesh;
  in.uv = f->uv; in.w_e = f->w_e; in.helem = f->helem;
  in.hnode = f->hnode; in.hnode_new = f->hnode_new;
  in.T = f->T; in.T_old = f->T_old; in.T_new = f->T_new;
  in.tstride = f->tracer_stride ? f->tracer_stride : int64_t(P->N) * P->L;
  in.tg = 0;
  in.wtg = ntr;
  in.Z3d = f->Z3d; in.zbar3 = f->zbar3; in.w_i = f->w_i;
  in.ws = carve_workspace(scratch, P->N, P->E, P->Ed, P->L, ntr, /*fused=*/true);
  in.dt = dt;
  in.ntr = ntr;
  in.nonfinite = P->d_health;   // allocated with the plan
  LaunchDims dims{};
  dims_cover(dims, P);
  dims.ntr = ntr;
  dims.chunk = 0;
  dims.set_map(P->per_thread, P->lpt);
  dims.any_wi = f->w_i != nullptr;
  dims.copy_dry = true;
  return restore(launch_forward(in, nullptr, 1, dims, static_cast<cudaStream_t>(stream)));
}
