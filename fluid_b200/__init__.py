"""B200-native free-surface pressure projection (MAC ghost-fluid MGPCG).

The compute lives in ``fluid_b200/_lib/libfluid_pp.so`` (hand-written CUDA for
sm_100a behind the C ABI of ``include/fluid_pp.h``); this package is the host
mirror of the reference's projection interface plus the seeded workload
generators.  Importing the package does not load the library; the first
projector does, and fails loudly if it was not built.
"""
from .projector import (BatchProjector, FluidError, PipelinedBatchProjector, PressureProjector, batch_tuning,
                        plan_uniform_cm11a_hierarchy, solve_opts)

__all__ = ["PressureProjector", "BatchProjector", "PipelinedBatchProjector", "FluidError", "plan_uniform_cm11a_hierarchy",
           "solve_opts", "batch_tuning"]
