"""CPU oracle for the pressure projection -- TEST INFRASTRUCTURE ONLY.

Checkers that live here:
  * ``xfp_oracle.c``   -- this project's FP64 C restatement of xFluid's
    variational pressure projection (assembly, MIC(0), PCG, applyPressure, and
    the adjoint pieces), built into ``oracle/_build/libxfp_oracle.so``.
  * ``oracle/_ref``    -- xFluid's own solver compiled from the reference
    sources by ``build_ref.sh``, and its FluidSimulator by ``build_sim.sh``
    (stepped by ``sim_harness.cpp``), only where the reference checkout exists.
  * ``advect.py``      -- numpy FP64 restatement of the differentiable rollout.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this package, and only as the checker or the timed CPU baseline.  The CUDA
product path never imports it.
"""
from .bindings import (DROPIN_LIB, ORACLE_LIB, REF_LIB, SIM_LIB, Oracle, Reference, RefSim,  # noqa: F401
                       RefSimDropIn, RefSteps, build_oracle, build_reference, dropin_available,
                       oracle_available, reference_available, seed_rand, sim_available)
