/*
 * fesom_fct.h -- C ABI of the B200 FCT tracer-advection library (libfesom_fct.so).
 *
 * One FESOM2 FCT (Zalesak flux-corrected transport) tracer-advection step, the
 * function fesom_jax/tracer_adv.py:532-578 ``advect_one_fct(mesh, uv, w_e, helem,
 * hnode, hnode_new, T, T_old, *, dt, exch=None, Z3d=None, zbar3=None, w_i=None)
 * -> (T_new, T_old_new)``, computed in FP64 by CUDA kernels for sm_100a.
 *
 * Layouts are the reference's (fesom_jax/mesh.py:11-20, fesom_jax/state.py:1-19):
 * row-major ``[entity, nl]`` float64 with the level index fastest; element velocities
 * ``uv`` are ``[elem2D, nl, 2]``; indices are 0-based int32 with -1 for a missing
 * neighbour. All field pointers passed to compute entry points are DEVICE pointers;
 * mesh pointers in FctMeshDesc are HOST pointers (copied at plan creation).
 *
 * Every entry point returns FCT_OK (0) or a negative FctStatus; the message of the
 * last failure on the calling thread is returned by fct_last_error().
 * No entry point except fct_plan_create / fct_plan_reserve / fct_plan_reserve_adjoint /
 * fct_batch_create / fct_serve_create / fct_tape_create (without caller memory)
 * allocates device memory, and none but the health checks (fct_*_health) synchronises
 * the stream it is given.
 */
#ifndef FESOM_FCT_H
#define FESOM_FCT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum FctStatus {
  FCT_OK = 0,
  FCT_ERR_INVALID = -1,      /* bad argument, shape or index range */
  FCT_ERR_CUDA = -2,         /* a CUDA runtime call failed */
  FCT_ERR_CAPACITY = -3,     /* more tracers than the plan's reserved workspace */
  FCT_ERR_UNSUPPORTED = -4,  /* option not supported (e.g. a halo exchange) */
  FCT_ERR_NONFINITE = -5     /* a NaN/Inf was detected in an output */
} FctStatus;

/* Opaque CUDA stream handle (a cudaStream_t); NULL is the legacy default stream. */
typedef void* fct_stream_t;

/*
 * Static mesh (HOST pointers; copied at plan creation). Field meanings and shapes
 * follow the reference Mesh dataclass, fesom_jax/mesh.py:70-108.
 */
typedef struct FctMeshDesc {
  int32_t nod2D, elem2D, edge2D, nl;
  const int32_t* edges;                 /* [edge2D,2] node ids */
  const int32_t* edge_tri;              /* [edge2D,2] element ids, [:,1] may be -1 */
  const int32_t* edge_up_dn_tri;        /* [edge2D,2] MFCT up/down triangles, -1 absent */
  const double* edge_cross_dxdy;        /* [edge2D,4] metres */
  const double* edge_dxdy;              /* [edge2D,2] rotated radians */
  const int32_t* elem_nodes;            /* [elem2D,3] */
  const double* gradient_sca;           /* [elem2D,6] */
  const double* elem_cos;               /* [elem2D] */
  const double* elem_area;              /* [elem2D] */
  const int32_t* nlevels;               /* [elem2D] */
  const int32_t* ulevels;               /* [elem2D] */
  const int32_t* nlevels_nod2D;         /* [nod2D] */
  const int32_t* nlevels_nod2D_min;     /* [nod2D] */
  const int32_t* ulevels_nod2D;         /* [nod2D] */
  const int32_t* ulevels_nod2D_max;     /* [nod2D] */
  const int32_t* nod_in_elem2D_offsets; /* [nod2D+1] CSR offsets */
  const int32_t* nod_in_elem2D;         /* [offsets[nod2D]] element ids, ascending */
  const double* area;                   /* [nod2D,nl] */
  const double* areasvol;               /* [nod2D,nl] */
  const double* Z;                      /* [nl-1] mid-layer depths */
  const double* zbar;                   /* [nl] interface depths */
} FctMeshDesc;

/*
 * Per-call fields (DEVICE pointers). ``T``, ``T_old`` and ``T_new`` hold ``ntr``
 * tracers that share the velocities and thicknesses, each ``[nod2D,nl]`` and
 * ``tracer_stride`` doubles apart (ntr = 1 is exactly one reference call; T and S of
 * step.py:409-416 are ntr = 2). ``T_new`` must not alias ``T`` or ``T_old``.
 * Optional (NULL = off, the reference's ``None``): ``Z3d``/``zbar3`` [nod2D,nl] live
 * stencil depths (tracer_adv.py:265-273); ``w_i`` [nod2D,nl] the implicit part of a
 * split vertical velocity (tracer_adv.py:487-529, 557-572).
 */
typedef struct FctFields {
  const double* uv;         /* [elem2D,nl,2] */
  const double* w_e;        /* [nod2D,nl] */
  const double* helem;      /* [elem2D,nl] */
  const double* hnode;      /* [nod2D,nl] */
  const double* hnode_new;  /* [nod2D,nl] */
  const double* T;          /* ntr x [nod2D,nl] */
  const double* T_old;      /* ntr x [nod2D,nl] */
  double* T_new;            /* ntr x [nod2D,nl] (output) */
  int64_t tracer_stride;    /* doubles between consecutive tracers; 0 = nod2D*nl */
  const double* Z3d;        /* optional */
  const double* zbar3;      /* optional */
  const double* w_i;        /* optional */
} FctFields;

typedef struct FctPlan FctPlan;

/* Build a plan for one mesh on ``device``: validates and uploads the mesh, derives the
 * node->edge CSR and lane lists, and reserves workspace for ``max_tracers`` tracers.
 * Replaces the reference's per-call mesh pytree operands (fesom_jax/mesh.py:62-129). */
int fct_plan_create(const FctMeshDesc* mesh, int device, int max_tracers, FctPlan** out);
int fct_plan_destroy(FctPlan* plan);
/* Grow the plan's workspace to ``max_tracers`` (allocates; call outside hot loops). */
int fct_plan_reserve(FctPlan* plan, int max_tracers);
/* Counts: [nod2D, elem2D, edge2D, nl, wet node layers, wet element layers, wet edge
 * layers, max_tracers]. */
int fct_plan_info(const FctPlan* plan, int64_t out[8]);
/* Which stage kernels fct_forward runs: fused (1, the default: 5 launches per tracer
 * chunk over runs of consecutive levels, element gradients and cluster bounds recomputed
 * instead of stored, quotients by reciprocals and explicit FMAs) or one kernel per
 * reference stage (0: 7 launches, every intermediate written to the workspace, every
 * quotient correctly rounded; the form the reverse pass recomputes). The two give the same
 * T_new to rounding (a few ulp per step). */
int fct_plan_set_fused(FctPlan* plan, int fused);
/* Thread mapping of the fused stages of this plan's fct_forward / fct_forward_noalloc and
 * of its instances in fct_serve_step: the most tracers one thread carries and the levels
 * of one node or edge column it takes (each 1, 2, 4 or 8; default 2 and 4). A tuning knob:
 * the results do not depend on it. No reference counterpart (XLA picks its own loop
 * mapping). */
int fct_plan_set_mapping(FctPlan* plan, int tracers_per_thread, int levels_per_thread);

/* One FCT step for ``ntr`` tracers: fesom_jax/tracer_adv.py:532-578 (advect_one_fct),
 * with exch=None. Writes T_new; T_old_new is T itself (the caller keeps the alias).
 * Calls on one plan that use its workspace (fct_forward, fct_forward_taped, fct_adjoint*,
 * fct_vert_diff, fct_ice_solve, fct_compute_w_adjoint, the XLA handlers) are ordered on
 * the GPU even when issued on different streams or host threads: each waits on its stream
 * for the previous one (a plan-owned event; nothing waits on the host). Calls issued while
 * their stream is captured into a CUDA graph skip that ordering. */
int fct_forward(FctPlan* plan, const FctFields* fields, double dt, int ntr,
                fct_stream_t stream);

/* fct_forward with options. FCT_FWD_STAGEWISE runs one kernel per reference stage (the
 * kernels the reverse pass recomputes with, which round every quotient correctly), so a
 * trajectory stepped with it is the one fct_adjoint differentiates bit for bit; it needs
 * the full workspace (fct_plan_reserve_adjoint or fct_plan_set_fused(plan, 0)). The
 * default fused kernels give the same T_new to rounding (a few ulp). */
#define FCT_FWD_STAGEWISE 1
int fct_forward_ex(FctPlan* plan, const FctFields* fields, double dt, int ntr, int flags,
                   fct_stream_t stream);

/* Health check, the finiteness gate of the reference's diagnostics
 * (fesom_jax/diagnostics.py:31-101 state_diagnostics/verdict): the number of non-finite
 * T_new values that fct_forward, fct_forward_taped, fct_forward_noalloc and the XLA
 * forward handler wrote with this plan since the previous check. Synchronises ``stream``
 * (call it between steps, not in a hot loop), resets the counter, stores the count in
 * ``*n_nonfinite`` (may be NULL) and returns FCT_ERR_NONFINITE when it is non-zero. */
int fct_plan_health(FctPlan* plan, fct_stream_t stream, int64_t* n_nonfinite);
/* Debug aid (no reference counterpart): fill the plan's workspace with the byte ``byte``
 * (0xFF makes every double a NaN), ordered like the compute calls. The stage kernels read
 * only workspace entries written earlier in the same step, so a step after a fill gives
 * the same result; tests use it to show that. */
int fct_plan_fill_workspace(FctPlan* plan, int byte, fct_stream_t stream);

/*
 * Implicit vertical tracer diffusion (fesom_jax/tracer_diff.py:68-123 impl_vert_diff_one;
 * :126-141 impl_vert_diff is two tracers with the shortwave on the first): per node
 * column, the tridiagonal system of the diffusivity Kv solved by the Thomas algorithm
 * (ops.py:121-168), the increment added to T on wet layers; dry levels keep T.
 */
typedef struct FctVdiffFields {
  const double* T;          /* ntr x [nod2D, nl], tracer_stride apart */
  double* T_new;            /* ntr x [nod2D, nl] (may equal T: in place) */
  int64_t tracer_stride;    /* 0 = nod2D * nl */
  const double* Kv;         /* [nod2D, nl] diffusivity on interfaces */
  const double* hnode_new;  /* [nod2D, nl] */
  const double* Z3d;        /* optional [nod2D, nl] mid-layer depths (NULL: the mesh's Z) */
  const double* bc_surf;    /* optional ntr x [nod2D] surface-layer RHS increments */
  const double* sw_3d;      /* optional [nod2D, nl] shortwave flux (divergence added) */
  int sw_tracer;            /* which tracer takes sw_3d (the reference: T, 0) */
} FctVdiffFields;
/* Needs a workspace of ntr tracers (fct_plan_reserve); allocates nothing. */
int fct_vert_diff(FctPlan* plan, const FctVdiffFields* fields, double dt, int ntr,
                  fct_stream_t stream);

/*
 * Sea-ice FCT advection (fesom_jax/ice_adv.py:175-194 fct_solve; fesom_ice_fct.c): one
 * step of the three surface ice tracers with the element-based Taylor-Galerkin scheme,
 * the consistent-mass low/high-order solves and the Zalesak limiter. The plan's mesh is
 * used at its surface level; its workspace serves as scratch (allocates nothing).
 */
typedef struct FctIceFields {
  const double* tracer[3];  /* a_ice, m_ice, m_snow: [nod2D] */
  double* tracer_new[3];    /* advected tracers (before cut_off): [nod2D] */
  const double* u_ice;      /* [nod2D] nodal ice velocity */
  const double* v_ice;      /* [nod2D] */
} FctIceFields;
typedef struct FctIceConfig {
  double dt;                /* IceConfig.ice_dt */
  double gamma;             /* IceConfig.ice_gamma_fct (0.5) */
  double diff;              /* IceConfig.ice_diff (10) */
} FctIceConfig;
int fct_ice_solve(FctPlan* plan, const FctIceFields* fields, const FctIceConfig* cfg,
                  fct_stream_t stream);

/*
 * Reverse mode (the reference's autodiff surface: jax.grad through advect_one_fct,
 * fesom_jax/integrate.py:43-169 under jax.grad). Cotangents follow JAX's subgradient
 * conventions: maximum/minimum split equally at a tie, segment_max/min and max over an
 * element's vertices spread evenly over tied entries, abs'(0) = 0.
 */
typedef struct FctGrads {
  double* gT;       /* ntr x [nod2D,nl] cotangent of T (written) */
  double* gT_old;   /* ntr x [nod2D,nl] cotangent of T_old (written) */
  double* guv;      /* [elem2D,nl,2] cotangent of uv, summed over tracers (written) */
  double* gw_e;     /* [nod2D,nl] cotangent of w_e, summed over tracers (written) */
} FctGrads;

/* Reserve the reverse-pass workspace for ``max_tracers`` tracers (allocates). */
int fct_plan_reserve_adjoint(FctPlan* plan, int max_tracers);
/* Vector-Jacobian product of one FCT step (fct_forward's inputs, tracer-major layout):
 * given ``gT_new`` (ntr x [nod2D,nl], same tracer stride as fields->T) write the
 * cotangents of T, T_old, uv and w_e. Recomputes the forward step internally (per-step
 * recomputation checkpointing: only the step's inputs need to be kept). The w_split
 * option (fields->w_i) is not differentiated (FCT_ERR_UNSUPPORTED); Z3d/zbar3 are
 * treated as constants. */
int fct_adjoint(FctPlan* plan, const FctFields* fields, const double* gT_new, double dt,
                int ntr, const FctGrads* grads, fct_stream_t stream);

/* Forward tape: the intermediates of up to ``steps`` recorded FCT steps (one full stage
 * workspace per step, fct_tape_bytes), so that the reverse pass of a recorded step skips
 * the recomputation. The tape keeps intermediates only; the step's inputs (fields) must
 * still be passed to fct_adjoint_ex unchanged. The reference saves its residuals the
 * same way under jax.grad (fesom_jax/integrate.py:43-169). */
typedef struct FctTape FctTape;
int fct_tape_bytes(const FctPlan* plan, int ntr, int steps, int64_t* out);
/* Creates a tape in ``mem`` (device memory of ``bytes`` >= fct_tape_bytes, 256-byte
 * aligned, owned by the caller and kept alive until fct_tape_destroy), or allocates it when
 * ``mem`` is NULL. Also reserves the plan's reverse-pass workspace for ``ntr`` tracers. */
int fct_tape_create(FctPlan* plan, int ntr, int steps, void* mem, int64_t bytes,
                    FctTape** out);
int fct_tape_destroy(FctTape* tape);
/* fct_forward that also records the step's intermediates in tape slot ``slot`` (with the
 * stage-by-stage kernels: T_new is bit-identical to fct_forward_ex with
 * FCT_FWD_STAGEWISE). w_i is not supported (not differentiated). */
int fct_forward_taped(FctPlan* plan, const FctFields* fields, double dt, int ntr,
                      FctTape* tape, int slot, fct_stream_t stream);
/* Declares that ``slot`` of a tape created over caller memory already holds a step
 * recorded by fct_forward_taped with ``dt`` (through another tape over the same memory,
 * e.g. in a separate forward and backward call of a stateless custom-call handler). */
int fct_tape_mark_recorded(FctTape* tape, int slot, double dt);
/* Declares that every step recorded on this tape uses the same uv and helem (a multi-step
 * loss with fixed velocities): slot 0's forward computes the edge volume fluxes
 * (fesom_jax/tracer_adv.py:69-93) and the other slots read them instead of recomputing
 * and storing their own. Slot 0 must be recorded first (FCT_ERR_INVALID otherwise);
 * recording slot 0 again with other velocities changes every slot's fluxes. No reference
 * counterpart (XLA may hoist the loop-invariant flux out of a scan by itself). */
int fct_tape_share_vflux(FctTape* tape);
/* Accumulate bits of fct_adjoint_ex: add into the output instead of overwriting it. */
#define FCT_ACC_T 1
#define FCT_ACC_T_OLD 2
#define FCT_ACC_UV 4
#define FCT_ACC_W 8
/* Bit of fct_adjoint_ex: do not write guv (it may be NULL); add this step's volume-flux
 * cotangents, summed over its tracers, into the plan's running sum instead. The uv
 * cotangent is linear in them with coefficients that depend only on the mesh and helem, so
 * for a chain of steps that share uv and helem one fct_adjoint_flush_uv after the last
 * step gives the sum over the chain of what each call would have added to guv (to
 * rounding: the sum is taken before the transpose). The sum lives in the plan's adjoint
 * workspace: a fct_plan_reserve_adjoint that grows it clears the sum. No reference
 * counterpart (XLA sums the per-step cotangents of the shared uv itself). */
#define FCT_ADJ_DEFER_UV 16
/* fct_adjoint with options: ``tape`` (NULL: recompute the step; else the step recorded
 * in ``slot`` with the same fields and dt) and ``accumulate`` (FCT_ACC_* bits). The
 * cotangents are bit-identical to fct_adjoint's (plus the accumulated contents). */
int fct_adjoint_ex(FctPlan* plan, const FctFields* fields, const double* gT_new, double dt,
                   int ntr, const FctGrads* grads, const FctTape* tape, int slot,
                   int accumulate, fct_stream_t stream);
/*
 * JAX/XLA custom-call handlers, legacy GPU ABI (jax.ffi.register_ffi_target(name,
 * jax.ffi.pycapsule(fn), platform="CUDA", api_version=0)); they replace the reference's
 * in-graph advect_one_fct (fesom_jax/tracer_adv.py:532-578) and its jax.grad.
 * ``opaque`` holds an FctXlaOpaque. ``buffers`` has a fixed layout (absent optional
 * operands are one-element placeholders, flagged absent):
 *   forward: uv, w_e, helem, hnode, hnode_new, T, T_old, Z3d, zbar3, w_i | T_new, status
 *   adjoint: uv, w_e, helem, hnode, hnode_new, T, T_old, Z3d, zbar3, gT_new |
 *            gT, gT_old, guv, gw_e, status
 * ``status`` is an int32 device scalar receiving the FctStatus (the ABI has no error
 * return). No allocation: reserve the plan (fct_plan_reserve; fct_plan_reserve_adjoint for
 * the adjoint) before the first call.
 */
typedef struct FctXlaOpaque {
  uint64_t plan;   /* FctPlan* of this process, as an integer */
  double dt;
  int32_t ntr;     /* tracers in T (tracer-major, [ntr, nod2D, nl]) */
  int32_t flags;   /* FCT_XLA_* */
} FctXlaOpaque;
#define FCT_XLA_Z3D 1   /* Z3d and zbar3 are real operands */
#define FCT_XLA_WI 2    /* w_i is a real operand (forward only) */
#define FCT_XLA_FWD_STATUS 11
#define FCT_XLA_ADJ_STATUS 14
void fct_xla_forward(void* stream, void** buffers, const char* opaque, size_t opaque_len);
void fct_xla_adjoint(void* stream, void** buffers, const char* opaque, size_t opaque_len);

/* guv (+)= the transpose of edge_vflux (fesom_jax/tracer_adv.py:69-93) applied to the
 * running sum of the FCT_ADJ_DEFER_UV calls made since the last flush, with ``helem``
 * [elem2D,nl] (the one those steps used); then clears the sum. ``accumulate`` = 0
 * overwrites guv, 1 adds. Ordered like the other calls on the plan. */
int fct_adjoint_flush_uv(FctPlan* plan, const double* helem, double* guv, int accumulate,
                         fct_stream_t stream);

/* Vector-Jacobian product of fct_compute_w (fesom_jax/ale.py:309-365) w.r.t. uv:
 * guv (+)= J^T gw, [elem2D,nl,2]; ``accumulate`` = 0 overwrites, 1 adds. */
int fct_compute_w_adjoint(FctPlan* plan, const double* gw, const double* helem,
                          double* guv, int accumulate, fct_stream_t stream);

/* The step of fct_forward (its fused stage kernels, whatever fct_plan_set_fused chose) for
 * callers that cannot allocate device memory at call time (an XLA/JAX custom-call handler
 * running inside a runtime that owns the GPU's memory, a serving loop that must not block
 * on the allocator). Its scratch is a 64 MiB file-scope device array instead of the plan's
 * workspace, so the plan may have been created with any max_tracers; sizes whose scratch
 * exceeds the array return FCT_ERR_CAPACITY. No reference counterpart: the reference
 * lets XLA allocate its temporaries. The first call on a device looks up the array's
 * address (make it before any stream capture); all calls share the array, which keeps
 * the last call's contents, so calls that overlap on the GPU race. */
int fct_forward_noalloc(FctPlan* plan, const FctFields* fields, double dt, int ntr,
                        fct_stream_t stream);

/* Vertical velocity at interfaces from continuity, fesom_jax/ale.py:309-365
 * (``compute_w(mesh, uv, helem)``): ``w`` [nod2D,nl] (DEVICE), all levels written. */
int fct_compute_w(FctPlan* plan, const double* uv, const double* helem, double* w,
                  fct_stream_t stream);

/*
 * Batched ensemble stepping: many FCT instances (ensemble members x tracers, on meshes
 * of different sizes) advanced together, one launch per stage for all instances of a
 * workspace group. Each instance owns three rotating tracer buffers of ``ntr`` tracers,
 * INTERLEAVED ``[nod2D, nl, ntr]`` (DEVICE; the tracers of one node-level contiguous);
 * a step of phase p reads T_old = buf[p],
 * T = buf[(p+1)%3] and writes T_new = buf[(p+2)%3], so consecutive phases carry the AB2
 * history (T_old_new = T) without copies. Start with T_old in buf[0], T in buf[1].
 */
typedef struct FctInstance {
  FctPlan* plan;            /* the instance's mesh */
  const double* uv;         /* [elem2D,nl,2] */
  const double* w_e;        /* [nod2D,nl] */
  const double* helem;      /* [elem2D,nl] */
  const double* hnode;      /* [nod2D,nl] */
  const double* hnode_new;  /* [nod2D,nl] */
  double* buf[3];           /* rotating tracer buffers, each [nod2D,nl,ntr] */
  int ntr;
  double dt;
  const double* Kv;         /* optional [nod2D,nl]: implicit vertical diffusion after each
                               step (tracer_diff.py:68-123, step.py:452; NULL = off) */
  double* w_derived;        /* optional [nod2D,nl]: each step first derives w_e =
                               compute_w(uv, helem) (ale.py:309-365, step.py:367) into this
                               buffer and advects with it (w_e is then ignored); NULL = off */
  unsigned long long* nonfinite; /* optional DEVICE counter: each step adds the number of
                               non-finite T_new values it writes (NULL: the batch's own
                               per-instance counter, or the serve engine's counter) */
} FctInstance;

typedef struct FctBatch FctBatch;

/* Group the instances so that each group's workspace fits ``workspace_budget_bytes``
 * (at least one instance per group), allocate one workspace arena (reused by the groups
 * in turn) and the per-phase device instance tables. An instance's interleaved arrays
 * (max(nod2D, elem2D, edge2D) x nl x ntr elements) must hold fewer than 2^32 elements
 * (FCT_ERR_CAPACITY otherwise; the same holds for fct_serve_step). */
int fct_batch_create(const FctInstance* insts, int n, int64_t workspace_budget_bytes,
                     FctBatch** out);
int fct_batch_destroy(FctBatch* b);
/* Tuning: the most tracers one thread carries (1, 2, 4 or 8; default: the workspace
 * chunk, at most 8). Fewer use fewer registers (higher occupancy), more share each
 * gather's index work. Drops cached graphs. */
int fct_batch_set_chunk(FctBatch* b, int chunk);
/* Tuning: tracers per thread (1, 2, 4 or 8; the fused stages carry at most 4) and levels
 * per thread (1, 2, 4 or 8) of the fused stages. Drops cached graphs. */
int fct_batch_set_mapping(FctBatch* b, int tracers_per_thread, int levels_per_thread);
/* The same for one fused stage: 0 LO and adf_v, 1 adf_h, 2 limiter factors, 3 T_new (the
 * stages are separate kernels, so each may take its own mapping). Drops cached graphs. */
int fct_batch_set_stage_mapping(FctBatch* b, int stage, int tracers_per_thread,
                                int levels_per_thread);
/* [instances, groups, workspace bytes, total wet node layers x tracers,
 *  tracers per workspace chunk (largest over groups), kernel launches per step] */
int fct_batch_info(const FctBatch* b, int64_t out[6]);
/* Copy the dry levels of buf[1] into buf[0] and buf[2] (dry levels never change). */
int fct_batch_prepare(FctBatch* b, fct_stream_t stream);
/* One FCT step of every instance with rotation phase ``phase`` (0, 1 or 2). */
int fct_batch_step(FctBatch* b, int phase, fct_stream_t stream);
/* ``steps`` consecutive steps starting at ``first_phase``, captured once into a CUDA
 * graph (cached per (first_phase, steps)) and launched on ``stream``. The instance that
 * holds T after the run is buf[(first_phase + steps + 1) % 3]. */
int fct_batch_run(FctBatch* b, int first_phase, int steps, fct_stream_t stream);

/* Health check of a batch (as fct_plan_health): per-instance counts of non-finite T_new
 * values written since the previous check into ``counts`` (n entries; may be NULL; 0 for
 * instances that count into their own FctInstance.nonfinite). Synchronises ``stream``,
 * resets the counters and returns FCT_ERR_NONFINITE when any count is non-zero. */
int fct_batch_health(FctBatch* b, fct_stream_t stream, int64_t* counts);
/* Debug aid (no reference counterpart), as fct_plan_fill_workspace for the batch's
 * workspace arena, on ``stream``. */
int fct_batch_fill_workspace(FctBatch* b, int byte, fct_stream_t stream);

/*
 * Continuous batching: one FCT step for an arbitrary set of instances that changes from
 * call to call (requests joining and leaving), on any meshes. ``FctServe`` owns a
 * workspace arena (carved per call in instance order; a call whose instances need more
 * returns FCT_ERR_CAPACITY) and a device instance table uploaded from pinned host memory
 * (a ring of 16 staging buffers: a call waits on the host only for the upload of the call
 * sixteen calls back). Instance i steps with rotation phase ``phases[i]`` (same convention as
 * fct_batch_step). Instances are launched in groups of one ntr and one mesh (each group's
 * grid is sized for its mesh). Calls on one FctServe must be ordered on one stream.
 */
typedef struct FctServe FctServe;
int fct_serve_create(int device, int max_instances, int64_t workspace_bytes, FctServe** out);
int fct_serve_destroy(FctServe* s);
int fct_serve_step(FctServe* s, const FctInstance* insts, const int32_t* phases, int n,
                   fct_stream_t stream);
/* Health check of the serve engine's own counter (instances without a counter of their
 * own), as fct_plan_health. */
int fct_serve_health(FctServe* s, fct_stream_t stream, int64_t* n_nonfinite);

/* Self-check of the division the kernels use for quotients that share a divisor (the
 * divisor's reciprocal computed once, then an FMA correction per quotient; see
 * fesom_jax_b200/csrc/fct_div.cuh): compares it with the native IEEE division for the n
 * device pairs x[i] / y[i] and accumulates into the device words result[0] (number of
 * bitwise mismatches, add) and result[1] (smallest mismatching index, min). The caller
 * initialises result to {0, UINT64_MAX}. No reference counterpart (the reference divides
 * with XLA's IEEE division); test infrastructure for the kernels' arithmetic. */
int fct_div_check(const double* x, const double* y, int64_t n, unsigned long long* result,
                  fct_stream_t stream);

/* Profiling aid: run one step of phase ``phase`` stage by stage with CUDA events recorded
 * on ``stream`` between stages, synchronise, and add each stage's time (ms, summed over
 * workspace groups) into ``stage_ms[0..max_stages)`` (needs >= 10 entries). */
int fct_batch_profile(FctBatch* b, int phase, double* stage_ms, int max_stages,
                      fct_stream_t stream);
/* Name of forward stage ``i`` (as reported by fct_batch_profile), "" if out of range. */
const char* fct_stage_name(int i);

/* Last error message on this thread ("" if none). */
const char* fct_last_error(void);
/* Library version string. */
const char* fct_version(void);

#ifdef __cplusplus
}
#endif

#endif /* FESOM_FCT_H */
