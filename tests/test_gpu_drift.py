"""600-frame drift of the FP32 product build against an FP64 re-run of the
same kernels (oracle O2<double>), on the default GPU scene (20^3 body +
65,536 fluid, slice wedge after frame 60).

The fluid is chaotic, so particle-by-particle positions separate over 600
frames between any two floating-point orders (the FP32 oracle and the FP64
one do too); the check is on per-frame aggregates of the state recorded by
tests/golden/make_drift.py: active fluid count, alive constraints, mean
fluid position, body centre of mass, mean squared speeds. Bounds: three
times the FP32 oracle's own drift from FP64 (its worst frame), with floors
of 1 mm for positions."""
from pathlib import Path

import numpy as np
import pytest

from fluidphysics_b200 import scenes as S
from fluidphysics_b200.sim import sim_from_scene

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def _aggregates():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_drift", GOLDEN / "make_drift.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_drift_600_frames_vs_fp64():
    ref = np.load(GOLDEN / "drift_gpu_default.npz")
    frames = int(ref["frames"])
    md = _aggregates()
    sc = S.gpu_default(frames=frames)
    sim = sim_from_scene(sc, "product")

    def read():
        cons = sim.read_constraints()
        return sim.read_state(), cons[:, 3] != 0

    gpu = md.trajectory(sc, frames, lambda: sim.step(sc.dt, sc.substeps), read, sim.slice)
    num_cons = sim.info.num_cons
    sim.close()
    report = {}
    for key in ("fluid_mean", "body_com"):
        g = np.linalg.norm(gpu[key] - ref[f"fp64_{key}"], axis=1)
        o = np.linalg.norm(ref[f"fp32_{key}"] - ref[f"fp64_{key}"], axis=1)
        report[key] = (float(g.max()), float(g[-1]), float(o.max()))
        assert g.max() <= max(3 * o.max(), 1e-3), f"{key}: drift {g.max():.3g} m vs FP32 oracle {o.max():.3g} m"
    for key in ("fluid_ke", "body_ke"):
        g = np.abs(gpu[key] - ref[f"fp64_{key}"])
        o = np.abs(ref[f"fp32_{key}"] - ref[f"fp64_{key}"])
        report[key] = (float(g.max()), float(g[-1]), float(o.max()))
        assert g.max() <= 3 * o.max() + 1e-4, f"{key}: drift {g.max():.3g} vs FP32 oracle {o.max():.3g}"
    for key, tol in (("fluid_n", 0.001 * sc.desc.max_fluid), ("alive", 0.001 * num_cons)):
        g = np.abs(gpu[key] - ref[f"fp64_{key}"])
        report[key] = (float(g.max()), float(g[-1]), float(np.abs(ref[f"fp32_{key}"] - ref[f"fp64_{key}"]).max()))
        assert g.max() <= tol, f"{key}: differs by {g.max()} (bound {tol})"
    print("drift vs FP64 over", frames, "frames (gpu max, gpu last, fp32-oracle max):", report)
