"""fluidphysics_b200 — B200-native unified-particle step.

The reference (fuugus/fluidphysics, "Slice & Splash") steps soft bodies and
fluid as one particle system: a spatial hash grid, XPBD distance constraints
with plasticity and tearing, double-density fluid relaxation, solid↔fluid
contacts and XSPH, plus slice/pick/grab/hose tools. This package runs that
step as hand-written sm_100a CUDA kernels behind the C ABI of include/upbd.h
(libupbd.so, built in-tree by `python -m fluidphysics_b200.build`).

  sim.Sim      one resident scene (C-ABI handle)
  sim.GpuSim   mirror of the reference's GpuSim (src/gpu/sim.js)
  sim.Solver   mirror of the reference's Solver (src/solver.js)
  scenes       seeded synthetic scenes (deriveOpts, jittered fluid blocks)
"""
from . import _lib, scenes  # noqa: F401

__all__ = ["_lib", "scenes", "sim"]


def __getattr__(name):
    if name == "sim":
        from . import sim
        return sim
    raise AttributeError(name)
