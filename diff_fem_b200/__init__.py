"""diff_fem_b200 — B200-native projective-dynamics step and adjoint.

Drop-in for the hot path of diff_fem (the local-global iterations of one time
step over corotated FEM tets, muscle segments, attachments, cloth springs and
bending, obstacle contact with friction, and the gradient of that step).

* ``diff_fem_b200.engine.Scene``  — handle over the C ABI (include/dfem.h)
* ``diff_fem_b200.scene``         — scene descriptors and workload builders
* ``diff_fem_b200.pydifem``       — the reference's ``pydifem`` module surface
* ``diff_fem_b200.api_diff``      — ``sim_act`` / ``sim_all`` autograd functions
"""
from . import _capi, scene  # noqa: F401
from .engine import Scene, host_factor_solve  # noqa: F401

__all__ = ["Scene", "host_factor_solve", "scene"]
