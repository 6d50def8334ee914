"""The CUDA library against the reference's own WGSL kernels, executed.

tests/golden/wgsl_passes.npz holds one whole substep of the reference's GPU
schedule (GpuSim.encode's pass order, src/gpu/sim.js:352-385) run by
tests/golden/wgslmini.py on the shader text src/gpu/wgsl.js makes, from a
state of a small scene with every optional pass (tets, the solid contact
cache with a companion cube, solid viscosity; tests/golden/make_golden_wgsl.py).
The GPU steps the same substep from the same state:

  - parity build (--fmad=false): positions within 2e-7 m and velocities
    within 5e-5 m/s of the reference's chain, flags, constraints and tets
    exactly (the bounds the oracle meets: the summation order of the gathers
    is the only difference);
  - product build: the per-substep FP32 tolerance of tests/helpers.py."""
import json
from pathlib import Path

import numpy as np
import pytest

from fluidphysics_b200.sim import sim_from_scene
from helpers import assert_states_close, load_state

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def _golden():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden_wgsl", GOLDEN / "make_golden_wgsl.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    z = np.load(GOLDEN / "wgsl_passes.npz")
    meta = json.loads(bytes(z["meta"]).decode())
    return m.golden_scene(), {k: z[k] for k in z.files if k != "meta"}, meta


def _chain(z, meta, scenario, upto):
    st = {k.split("/")[-1]: v.copy() for k, v in z.items() if k.startswith(f"{scenario}/start/")}
    for e in meta["passes"]:
        if e["scenario"] == scenario and e["index"] < upto:
            for b in e["changed"]:
                st[b] = z[f"{scenario}/{e['index']}/{b}"].copy()
    return st


@pytest.mark.parametrize("variant", ["parity", "product"])
def test_substep_matches_reference_wgsl(variant):
    sc, z, meta = _golden()
    C = meta["C"]
    es = [e for e in meta["passes"] if e["scenario"] == "substep"]
    start = _chain(z, meta, "substep", 0)
    end = _chain(z, meta, "substep", es[-1]["index"] + 1)
    ts, NT = C["TS_TETS"], C["NUM_TETS"]
    sim = sim_from_scene(sc, variant)
    load_state(sim, start, start["cons"])
    sim.write_tets(start["gridS"][ts:ts + NT * 5].reshape(NT, 5))
    sim.substep_partial(es[0]["uniform"]["h"], 1000)
    g = sim.read_state()
    assert np.array_equal(g["flags"], end["flags"])
    assert np.array_equal(sim.read_constraints(), end["cons"])
    assert np.array_equal(sim.read_tets(), end["gridS"][ts:ts + NT * 5].reshape(NT, 5))
    if variant == "parity":
        act = (end["flags"] & 1).astype(bool)
        dp = float(np.abs(g["pos"][act, :3].astype(np.float64) - end["pos"][act, :3]).max())
        dv = float(np.abs(g["vel"][act, :3].astype(np.float64) - end["vel"][act, :3]).max())
        assert dp <= 2e-7 and dv <= 5e-5, f"positions {dp:.3g} m, velocities {dv:.3g} m/s"
    else:
        assert_states_close(g, {k: end[k] for k in ("pos", "prev", "vel", "density", "flags")}, "product substep")
    sim.close()


@pytest.mark.parametrize("variant", ["parity", "product"])
def test_frame_matches_reference_wgsl(variant):
    """One whole frame of the reference's GpuSim.encode (a 32-particle emit,
    five substeps, the queued wedge cut with its tets, the active count), run
    by the WGSL interpreter, against upbd_emit + upbd_slice + upbd_step from
    the same state. Flags, constraints, tets and the active count exactly;
    positions and velocities within 1e-6 m and 1e-4 m/s in the parity build,
    1e-4 m and 1.4e-3 m/s in the product build. The 32 emitted particles get a
    velocity jitter of up to 0.25 m/s per axis from fract(sin(phase * c) * 4e4),
    which turns the last bits of sin()'s argument and result into differences
    of the jitter; they then press on each other for five substeps. Their
    bounds: 1e-3 m and 5e-2 m/s in the parity build, 6e-3 m and 0.2 m/s in the
    product build, whose fused multiply-adds change the argument's last bits
    (measured 2.9e-3 m and 0.094 m/s)."""
    sc, z, meta = _golden()
    C = meta["C"]
    e = next(e for e in meta["passes"] if e["scenario"] == "frame")
    st = {k.split("/")[-1]: v for k, v in z.items() if k.startswith("frame/start/")}
    end = {k.split("/")[-1]: v for k, v in z.items() if k.startswith("frame/end/")}
    ts, NT, S_, F = C["TS_TETS"], C["NUM_TETS"], C["SOLID_N"], C["MAX_FLUID"]
    u = e["uniform"]
    sim = sim_from_scene(sc, variant)
    load_state(sim, st, st["cons"])
    sim.write_tets(st["gridS"][ts:ts + NT * 5].reshape(NT, 5))
    sim.set_fluid_next(int(u["emitStart"]))
    sim.emit(int(u["emitCount"]), u["emitPos"][:3], u["emitDir"][:3], u["emitSide"][:3], u["emitUp"][:3],
             u["emitPos"][3], u["emitDir"][3])
    sim.slice(*e["wedge"])
    sim.step(sc.dt, sc.substeps)
    g = sim.read_state()
    assert np.array_equal(g["flags"], end["flags"])
    assert np.array_equal(sim.read_constraints(), end["cons"])
    assert np.array_equal(sim.read_tets(), end["gridS"][ts:ts + NT * 5].reshape(NT, 5))
    assert sim.active_count() == int(end["gridA"][2 * C["TABLE"] + C["TOTAL"] + 1])
    act = (end["flags"] & 1).astype(bool)
    emitted = np.zeros(C["TOTAL"], bool)
    emitted[S_ + (int(u["emitStart"]) + np.arange(int(u["emitCount"]))) % F] = True
    rest = act & ~emitted
    tol = dict(parity=(1e-6, 1e-4, 1e-3, 5e-2), product=(1e-4, 1.4e-3, 6e-3, 0.2))[variant]

    def err(k, m):
        return float(np.abs(g[k][m, :3].astype(np.float64) - end[k][m, :3]).max())
    assert err("pos", rest) <= tol[0] and err("vel", rest) <= tol[1], (err("pos", rest), err("vel", rest))
    assert err("pos", emitted) <= tol[2] and err("vel", emitted) <= tol[3], (err("pos", emitted), err("vel", emitted))
    sim.close()
