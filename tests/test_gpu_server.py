"""GPU checks of the continuous-batching frame server (include/upbd_server.h):
each request's result is the same whether it ran alone or among others that
arrived, ran and left around it; admission follows the HBM budget."""
import numpy as np
import pytest

from fluidphysics_b200 import _lib as L
from fluidphysics_b200 import batch as B
from fluidphysics_b200.server import Server
from fluidphysics_b200.sim import sim_from_scene

pytestmark = pytest.mark.gpu

DT, NSUB = 1 / 60, 5


def alone(sc, frames, variant):
    sim = sim_from_scene(sc, variant)
    for _ in range(frames):
        sim.step(DT, NSUB)
    st = sim.read_state()
    sim.close()
    return st


@pytest.mark.parametrize("variant", ["parity", "product"])
def test_results_same_alone_and_in_the_mix(variant):
    scs = [B.batch_scene(6, 2048, 31), B.batch_scene(9, 5000, 32), B.batch_scene(4, 700, 33),
           B.batch_scene(7, 3000, 34)]
    frames = [9, 4, 6, 3]
    arrivals = [0.0, 0.0, 0.02, 0.05]  # two join a running batch
    with Server(keep_results=True, variant=variant, max_scenes=8) as srv:
        ids = [srv.submit(sc, f, a) for sc, f, a in zip(scs, frames, arrivals)]
        srv.run(120)
        st = srv.stats()
        assert st["completed"] == 4 and st["rejected"] == 0
        assert st["scene_frames"] == sum(frames)
        assert st["peak_scenes"] >= 2  # they did share frames
        for rid, sc, f in zip(ids, scs, frames):
            res = srv.result(rid, with_state=True)
            assert res["state"] == "done" and res["frames_done"] == f
            ref = alone(sc, f, variant)
            assert np.array_equal(res["flags"], ref["flags"])
            assert np.array_equal(res["pos"], ref["pos"]), f"request {rid}: positions differ from the lone run"


def test_admission_follows_the_budget():
    scs = [B.batch_scene(5, 1500, 41 + k) for k in range(4)]
    one = B.Batch.scene_bytes(scs[0].desc)
    big = B.batch_scene(12, 40000, 49)
    with Server(hbm_budget=int(one * 1.5), max_scenes=8) as srv:
        ids = [srv.submit(sc, 3, 0.0) for sc in scs]
        rid_big = srv.submit(big, 2, 0.0)
        srv.run(120)
        st = srv.stats()
        assert st["peak_scenes"] == 1  # one fits at a time
        assert st["peak_bytes"] <= int(one * 1.5)
        assert st["completed"] == 4 and st["rejected"] == 1
        res = srv.result(rid_big)
        assert res["state"] == "rejected" and res["status"] == -8  # UPBD_ERR_CAPACITY
        t = [srv.result(i) for i in ids]
        # served in arrival (submission) order, one after the other
        assert all(t[k]["admit_s"] >= t[k - 1]["done_s"] - 1e-9 for k in range(1, 4))


def test_latency_stats_are_consistent():
    scs = [B.batch_scene(5, 1200, 51 + k) for k in range(3)]
    with Server(max_scenes=8) as srv:
        for k, sc in enumerate(scs):
            srv.submit(sc, 4, 0.01 * k)
        srv.run(120)
        st = srv.stats()
    assert st["scene_frames"] == 12
    assert 0 < st["frame_ms_p50"] <= st["frame_ms_p99"] <= st["frame_ms_max"]
    assert st["batch_frames"] >= 4 and st["device_s"] > 0
    assert st["particle_substeps"] > 0
