"""B200-native FCT tracer advection for fesom_jax (FP64 CUDA for sm_100a behind a C ABI).

Modules:

* ``tracer_adv`` -- ``advect_one_fct`` with the reference's signature, and ``FctPlan``
  (a mesh uploaded to one GPU).
* ``adjoint`` -- step VJPs, the forward ``Tape``, ``chain_loss_and_grad`` and the torch
  autograd functions.
* ``ensemble`` -- many members x tracers x meshes per launch, multi-step CUDA graphs,
  ``autotune``.
* ``serve`` -- the continuous-batching ``ServingEngine``.
* ``tracer_diff``, ``ale``, ``ice_adv`` -- implicit vertical diffusion, ``compute_w``,
  sea-ice FCT on the same plans.
* ``xla`` -- opaque bytes and buffer lists of the JAX/XLA custom-call handlers.
* ``mesh``, ``meshgen``, ``inputs``, ``workloads`` -- meshes, synthetic meshes and inputs.

The C ABI is ``include/fesom_fct.h``; the library is built in place by
``python -m fesom_jax_b200.build``. There is no CPU fallback: the modules raise when the
library or a CUDA GPU is missing.
"""
