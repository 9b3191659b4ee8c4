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
 * No entry point except fct_plan_create / fct_plan_reserve / fct_batch_create
 * allocates device memory, and none synchronises the stream it is given.
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

/* One FCT step for ``ntr`` tracers: fesom_jax/tracer_adv.py:532-578 (advect_one_fct),
 * with exch=None. Writes T_new; T_old_new is T itself (the caller keeps the alias). */
int fct_forward(FctPlan* plan, const FctFields* fields, double dt, int ntr,
                fct_stream_t stream);

/* Last error message on this thread ("" if none). */
const char* fct_last_error(void);
/* Library version string. */
const char* fct_version(void);

#ifdef __cplusplus
}
#endif

#endif /* FESOM_FCT_H */
