// JAX/XLA custom-call handlers (the legacy GPU custom-call ABI, api_version 0):
// ``void f(cudaStream_t stream, void** buffers, const char* opaque, size_t opaque_len)``,
// registered with jax.ffi.register_ffi_target(name, jax.ffi.pycapsule(f), platform="CUDA",
// api_version=0). They wrap fct_forward and fct_adjoint for the reference's call sites
// (fesom_jax/tracer_adv.py:532-578 under step.py:409-416, and its jax.grad through
// integrate.py:43-169).
//
// XLA owns the device memory and the stream: the handlers allocate nothing (the plan's
// workspaces are reserved when it is built) and never synchronise. The ABI has no error
// return, so each handler writes its FctStatus into a trailing int32 result on the
// stream, which the Python wrapper checks; the message stays in fct_last_error().
// The buffer list has a fixed length (absent optional operands are passed as a
// one-element placeholder and flagged absent in the opaque bytes), so the status result
// is found even when the opaque bytes are malformed.
#include <cstring>

#include "fct_host.h"

namespace {

__global__ void k_put_status(int32_t* p, int32_t v) { *p = v; }

void put_status(void* stream, void* status, int v) {
  if (status) k_put_status<<<1, 1, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<int32_t*>(status), int32_t(v));
}

int parse(const char* opaque, size_t len, FctXlaOpaque* o, FctPlan** P) {
  if (!opaque || len != sizeof(FctXlaOpaque))
    return fct::set_error(FCT_ERR_INVALID, "opaque: %zu bytes, expected %zu", len,
                          sizeof(FctXlaOpaque));
  std::memcpy(o, opaque, sizeof(FctXlaOpaque));
  *P = reinterpret_cast<FctPlan*>(uintptr_t(o->plan));
  if (!fct::plan_alive(*P))
    return fct::set_error(FCT_ERR_INVALID, "opaque names no live plan of this process");
  if (o->flags & ~(FCT_XLA_Z3D | FCT_XLA_WI))
    return fct::set_error(FCT_ERR_INVALID, "unknown opaque flags 0x%x", unsigned(o->flags));
  return FCT_OK;
}

FctFields fields_of(void** b, int32_t flags) {
  FctFields f{};
  f.uv = static_cast<const double*>(b[0]);
  f.w_e = static_cast<const double*>(b[1]);
  f.helem = static_cast<const double*>(b[2]);
  f.hnode = static_cast<const double*>(b[3]);
  f.hnode_new = static_cast<const double*>(b[4]);
  f.T = static_cast<const double*>(b[5]);
  f.T_old = static_cast<const double*>(b[6]);
  f.tracer_stride = 0;
  if (flags & FCT_XLA_Z3D) {
    f.Z3d = static_cast<const double*>(b[7]);
    f.zbar3 = static_cast<const double*>(b[8]);
  }
  return f;
}

}  // namespace

extern "C" {

void fct_xla_forward(void* stream, void** buffers, const char* opaque, size_t opaque_len) {
  if (!buffers) return;
  void* status = buffers[FCT_XLA_FWD_STATUS];
  FctXlaOpaque o;
  FctPlan* P = nullptr;
  int st = parse(opaque, opaque_len, &o, &P);
  if (st == FCT_OK) {
    FctFields f = fields_of(buffers, o.flags);
    if (o.flags & FCT_XLA_WI) f.w_i = static_cast<const double*>(buffers[9]);
    f.T_new = static_cast<double*>(buffers[10]);
    st = fct_forward(P, &f, o.dt, o.ntr, stream);
  }
  put_status(stream, status, st);
}

void fct_xla_adjoint(void* stream, void** buffers, const char* opaque, size_t opaque_len) {
  if (!buffers) return;
  void* status = buffers[FCT_XLA_ADJ_STATUS];
  FctXlaOpaque o;
  FctPlan* P = nullptr;
  int st = parse(opaque, opaque_len, &o, &P);
  if (st == FCT_OK && (o.flags & FCT_XLA_WI))
    st = fct::set_error(FCT_ERR_UNSUPPORTED, "the adjoint does not differentiate w_i");
  if (st == FCT_OK) {
    const FctFields f = fields_of(buffers, o.flags);
    FctGrads g{};
    g.gT = static_cast<double*>(buffers[10]);
    g.gT_old = static_cast<double*>(buffers[11]);
    g.guv = static_cast<double*>(buffers[12]);
    g.gw_e = static_cast<double*>(buffers[13]);
    st = fct_adjoint(P, &f, static_cast<const double*>(buffers[9]), o.dt, o.ntr, &g, stream);
  }
  put_status(stream, status, st);
}

}  // extern "C"
