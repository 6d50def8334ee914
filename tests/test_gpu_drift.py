"""600-frame drift of the FP32 product build on the default GPU scene (20^3
body + 65,536 fluid, slice wedge after frame 60), against two FP64 re-runs
of the same kernels:

  - the CUDA pass bodies themselves instantiated on double
    (libupbd_fp64.so, UPBD_FP64_BUILD), stepped on the GPU beside it;
  - the oracle's restatement of the WGSL kernels in double (O2<double>),
    whose per-frame aggregates tests/golden/make_drift.py recorded, together
    with the FP32 oracle's (O2<float>).

The fluid is chaotic, so particle-by-particle positions separate over 600
frames between any two floating-point orders (the FP32 oracle and the FP64
one do too); the checks are on per-frame aggregates of the state: active
fluid count, alive constraints, mean fluid position, body centre of mass,
mean squared speeds. Bounds: three times the FP32 oracle's own drift from
FP64 (its worst frame), with floors of 1 mm for positions."""
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


def _gpu_trajectory(variant: str, frames: int) -> tuple[dict, int, int]:
    md = _aggregates()
    sc = S.gpu_default(frames=frames)
    sim = sim_from_scene(sc, variant)

    def read():
        cons = sim.read_constraints()
        return sim.read_state(), cons[:, 3] != 0

    tr = md.trajectory(sc, frames, lambda: sim.step(sc.dt, sc.substeps), read, sim.slice)
    num_cons = sim.info.num_cons
    sim.close()
    return tr, num_cons, sc.desc.max_fluid


@pytest.fixture(scope="module")
def runs():
    ref = np.load(GOLDEN / "drift_gpu_default.npz")
    frames = int(ref["frames"])
    fp32, num_cons, max_fluid = _gpu_trajectory("product", frames)
    fp64, _, _ = _gpu_trajectory("fp64", frames)
    return ref, fp32, fp64, num_cons, max_fluid


def _check(a: dict, b: dict, ref, num_cons: int, max_fluid: int, what: str) -> dict:
    """a against b, frame by frame, with the FP32 oracle's drift from the FP64
    oracle as the scale."""
    report = {}
    for key in ("fluid_mean", "body_com"):
        g = np.linalg.norm(a[key] - b[key], axis=1)
        o = np.linalg.norm(ref[f"fp32_{key}"] - ref[f"fp64_{key}"], axis=1)
        report[key] = (float(g.max()), float(g[-1]), float(o.max()))
        assert g.max() <= max(3 * o.max(), 1e-3), f"{what} {key}: drift {g.max():.3g} m vs FP32 oracle {o.max():.3g} m"
    for key in ("fluid_ke", "body_ke"):
        g = np.abs(a[key] - b[key])
        o = np.abs(ref[f"fp32_{key}"] - ref[f"fp64_{key}"])
        report[key] = (float(g.max()), float(g[-1]), float(o.max()))
        assert g.max() <= 3 * o.max() + 1e-4, f"{what} {key}: drift {g.max():.3g} vs FP32 oracle {o.max():.3g}"
    for key, tol in (("fluid_n", 0.001 * max_fluid), ("alive", 0.001 * num_cons)):
        g = np.abs(a[key] - b[key])
        report[key] = (float(g.max()), float(g[-1]), float(np.abs(ref[f"fp32_{key}"] - ref[f"fp64_{key}"]).max()))
        assert g.max() <= tol, f"{what} {key}: differs by {g.max()} (bound {tol})"
    print(what, "over", len(a["fluid_n"]), "frames (max, last, fp32-oracle max):", report)
    return report


def test_drift_600_frames_vs_fp64_oracle(runs):
    ref, fp32, _, num_cons, max_fluid = runs
    oracle64 = {k: ref[f"fp64_{k}"] for k in ("fluid_n", "fluid_mean", "fluid_ke", "body_com", "body_ke", "alive")}
    _check(fp32, oracle64, ref, num_cons, max_fluid, "FP32 product vs O2<double>")


def test_drift_600_frames_vs_gpu_fp64(runs):
    """The FP32 product against the CUDA kernels' own FP64 re-run, and that
    re-run against the oracle's FP64 trajectory (two double-precision runs of
    the same rules: their gap is the floor the FP32 drift is measured on)."""
    ref, fp32, fp64, num_cons, max_fluid = runs
    _check(fp32, fp64, ref, num_cons, max_fluid, "FP32 product vs GPU FP64")
    oracle64 = {k: ref[f"fp64_{k}"] for k in ("fluid_n", "fluid_mean", "fluid_ke", "body_com", "body_ke", "alive")}
    _check(fp64, oracle64, ref, num_cons, max_fluid, "GPU FP64 vs O2<double>")
