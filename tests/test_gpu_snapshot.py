"""GPU checks of the reference's snapshot and recording formats
(fluidphysics_b200/snapshot.py): a snapshot restores the exact state, and a
recording replays to the exact state of the run it recorded."""
import numpy as np
import pytest

from fluidphysics_b200 import snapshot as SN
from fluidphysics_b200.sim import GpuSim

pytestmark = pytest.mark.gpu

OPTS = {"SOLID_DIM": 8, "MAX_FLUID": 4096, "TABLE": 1 << 14, "substeps": 3, "solidIters": 4,
        "cubeCenter": [0, 0.9, 0]}


def same(a: GpuSim, b: GpuSim, what: str):
    sa, sb = a.sim.read_state(), b.sim.read_state()
    for k in ("pos", "prev", "vel", "density", "flags"):
        assert np.array_equal(sa[k], sb[k]), f"{what}: {k} differs"
    assert np.array_equal(a.sim.read_constraints(), b.sim.read_constraints()), f"{what}: constraints"
    assert np.array_equal(a.sim.read_tets(), b.sim.read_tets()), f"{what}: tets"
    assert a.fluidNext == b.fluidNext


def hose(gs: GpuSim, k: int):
    gs.emit(48, [0.1 * k, 2.0, 0.0], [0, -1, 0], [1, 0, 0], [0, 0, 1], 2.0, 0.3 * k)


def test_snapshot_round_trip_is_exact():
    a = GpuSim(OPTS)
    for k in range(20):
        hose(a, k)
        a.encode()
    a.queueCut([0.05, 5, 0.0], [0.0, -1.0, 0.02], [0.02, -1.0, 0.0])
    a.encode()
    snap = SN.loads(SN.dumps(SN.snapshot(a)))
    assert snap["version"] == 1 and snap["app"] == "slice-splash-gpu"
    assert snap["numCons"] == a.NUM_CONS and snap["opts"]["SOLID_DIM2"] == a.DIM2
    b = SN.load_snapshot(snap)
    same(a, b, "restored")
    for k in range(5):
        hose(a, 20 + k)
        hose(b, 20 + k)
        a.encode()
        b.encode()
    same(a, b, "5 frames after restore")
    a.dispose()
    b.dispose()


def test_standalone_restore_drops_grabs():
    a = GpuSim(OPTS)
    a.encode()
    a.grabAt([0, 0.9, 0], 0.2)
    assert (a.sim.read_state()["flags"] & 2).any()
    snap = SN.snapshot(a)
    assert not (SN.load_snapshot(snap).sim.read_state()["flags"] & 2).any()
    assert (SN.load_snapshot(snap, keep_grabs=True).sim.read_state()["flags"] & 2).any()


def test_recording_replays_exactly():
    a = GpuSim(OPTS)
    for k in range(6):
        hose(a, k)
        a.encode()
    bundle = {"version": 1, "type": "splash-recording", "snapshot": SN.snapshot(a), "actions": []}
    script = {0: [{"emit": [40, 0.0, 2.0, 0.1, 0, -1, 0, 1, 0, 0, 0, 0, 1, 2.5, 0.7]}],
              2: [{"grab": [0.0, 0.9, 0.0, 0.25, 0]}, {"cam": [0.3, 0.2, 6.0]}],
              3: [{"gd": [0.01, 0.02, 0.0]}], 4: [{"gd": [0.01, 0.03, 0.0]}],
              6: [{"rel": 1}], 7: [{"cut": [[0.05, 5, 0.0], [0.0, -1.0, 0.02], [0.02, -1.0, 0.0]]}]}
    tail = 3
    last = max(script)
    for f in range(last + tail + 1):
        for act in script.get(f, []):
            bundle["actions"].append({"f": f, **act})
            SN.apply_action(a, act)
        a.encode()
    b = SN.replay(SN.loads(SN.dumps(bundle)), tail_frames=tail)
    same(a, b, "replay")


def test_reference_written_snapshot_loads_exactly():
    """A snapshot that the reference's own GpuSim.snapshot wrote
    (tests/golden/app_js.json, made by tests/golden/make_golden_app.py from
    seeded buffers) loads into a GpuSim built from its options: every buffer
    lands bit for bit (grab bits dropped, as a standalone restore does), and
    snapshotting the loaded scene writes the same object back."""
    import json
    from pathlib import Path
    gold = Path(__file__).resolve().parent / "golden"
    case = json.loads((gold / "app_js.json").read_text())["cases"]["snapshot"]
    npz = np.load(gold / "app_js.npz")
    snap = case["snapshot"]
    gs = SN.load_snapshot(snap)
    assert (gs.TOTAL, gs.NUM_CONS, gs.NUM_TETS) == (case["total"], case["num_cons"], case["num_tets"])
    st = gs.sim.read_state()
    for k in ("pos", "prev", "vel", "density"):
        assert st[k].tobytes() == npz[k].tobytes(), k
    assert np.array_equal(st["flags"], npz["flags"] & np.uint32(0xFFFFFFFD))
    assert np.array_equal(gs.sim.read_constraints(), npz["cons"])
    assert np.array_equal(gs.sim.read_tets(), npz["tets"])
    assert gs.fluidNext == snap["fluidNext"]
    back = SN.snapshot(gs)
    want = dict(snap)
    want["buffers"] = dict(snap["buffers"])
    want["buffers"]["flags"] = SN.snapshot_from_arrays(
        {}, 0, 0, {**{k: npz[k] for k in ("pos", "prev", "vel", "density")},
                   "flags": npz["flags"] & np.uint32(0xFFFFFFFD)}, npz["cons"], npz["tets"])["buffers"]["flags"]
    assert json.dumps(back) == json.dumps(want)
