"""GPU checks of the scene batch (include/upbd_batch.h).

Every scene of a batch must step exactly as a single-scene handle does: bit
for bit in the parity build (whose single-scene path is pinned to the FP32
oracle by test_gpu_parity.py, and directly here), whatever else is in the
batch, however the persistent grid is shaped, and while scenes join and
leave between frames."""
import ctypes as C

import numpy as np
import pytest

from fluidphysics_b200 import _lib as L
from fluidphysics_b200 import batch as B
from fluidphysics_b200.sim import sim_from_scene
from helpers import assert_states_equal
from oracle.oracle import o2_from_scene

pytestmark = pytest.mark.gpu

DT, NSUB = 1 / 60, 5


def small_scenes():
    """Three uneven scenes (dims 6, 9, 4; 2,048 / 5,000 / 700 fluid)."""
    return [B.batch_scene(6, 2048, 11), B.batch_scene(9, 5000, 12), B.batch_scene(4, 700, 13)]


def run_plain(sc, frames, variant):
    sim = sim_from_scene(sc, variant)
    for _ in range(frames):
        sim.step(DT, NSUB)
    st, cons = sim.read_state(), sim.read_constraints()
    sim.close()
    return st, cons


def step(b, frames):
    for _ in range(frames):
        b.step(DT, NSUB)
    b.sync()


@pytest.mark.parametrize("variant", ["parity", "product"])
def test_batch_matches_single_scene_handles(variant):
    scs = small_scenes()
    with B.Batch(variant=variant, max_scenes=8) as b:
        ids = [b.add_scene(sc) for sc in scs]
        step(b, 12)
        for sid, sc in zip(ids, scs):
            ref, rcons = run_plain(sc, 12, variant)
            assert_states_equal(b.read_state(sid), ref, f"{variant} scene {sid}")
            assert np.array_equal(b.read_constraints(sid), rcons)


def test_batch_scene_matches_oracle_parity_build():
    sc = B.batch_scene(5, 1500, 21)
    o2 = o2_from_scene(sc)
    with B.Batch(variant="parity", max_scenes=4) as b:
        sid = b.add_scene(sc)
        b.add_scene(B.batch_scene(7, 3000, 22))  # a neighbour in the table
        for _ in range(3):
            b.step(DT, NSUB)
            o2.step(DT, NSUB)
        b.sync()
        assert_states_equal(b.read_state(sid), o2.read_state(), "batch vs oracle, 3 frames")


def test_scenes_join_and_leave_without_changing_results():
    scs = small_scenes()
    with B.Batch(variant="parity", max_scenes=4) as b:
        a = b.add_scene(scs[0])
        step(b, 4)
        c = b.add_scene(scs[1])  # joins a running batch
        step(b, 4)
        b.remove_scene(c)
        d = b.add_scene(scs[2])  # takes the freed memory
        step(b, 4)
        assert_states_equal(b.read_state(a), run_plain(scs[0], 12, "parity")[0], "resident scene")
        assert_states_equal(b.read_state(d), run_plain(scs[2], 4, "parity")[0], "late scene")
        assert b.info().scenes == 2


@pytest.mark.parametrize("variant", ["parity", "product"])
def test_grid_shape_does_not_change_results(variant):
    scs = small_scenes()
    out = []
    for bt, cps in ((64, 2), (128, 5), (256, 16)):
        with B.Batch(variant=variant, max_scenes=4, block_threads=bt, ctas_per_sm=cps) as b:
            ids = [b.add_scene(sc) for sc in scs]
            step(b, 6)
            out.append([b.read_state(i) for i in ids])
    for k in (1, 2):
        for g, r in zip(out[k], out[0]):
            assert_states_equal(g, r, f"tuning {k}")


def test_launches_per_frame_do_not_depend_on_scene_count():
    scs = small_scenes()
    counts = []
    for n in (1, 3):
        with B.Batch(max_scenes=4) as b:
            for sc in scs[:n]:
                b.add_scene(sc)
            step(b, 2)
            l0 = b.launches
            step(b, 3)
            counts.append((b.launches - l0) / 3)
    # 5 substeps x (integrate, scan, scatter, rankfix, density, disp,
    # 3 x solve-and-apply, bonds+contacts, apply+bounds+velocity, xsph with
    # its apply) + the active count
    assert counts[0] == counts[1] == 5 * 12 + 1


def test_capacity_and_budget_are_enforced():
    scs = small_scenes()
    need = B.Batch.scene_bytes(scs[1].desc)
    with B.Batch(max_scenes=2, hbm_budget=need + 1) as b:
        b.add_scene(scs[1])
        with pytest.raises(L.UpbdError, match="CAPACITY"):
            b.add_scene(scs[0])  # over the budget
        assert b.info().scenes == 1
        assert b.info().bytes_in_use == need
    with B.Batch(max_scenes=1) as b:
        b.add_scene(scs[2])
        with pytest.raises(L.UpbdError, match="CAPACITY"):
            b.add_scene(scs[2])  # table full
        with pytest.raises(L.UpbdError, match="INVALID"):
            b.remove_scene(999)
    sc = B.batch_scene(5, 1000, 3, iters=2)
    with B.Batch(solid_iters=3) as b:
        with pytest.raises(L.UpbdError, match="INVALID"):
            b.add_scene(sc)  # iteration count differs from the batch's


def test_active_counts_and_nan_health():
    scs = small_scenes()
    with B.Batch(max_scenes=4) as b:
        ids = [b.add_scene(sc) for sc in scs]
        step(b, 2)
        for sid, sc in zip(ids, scs):
            st = b.read_state(sid)
            assert b.active_count(sid) == int((st["flags"][sc.solid_n:] & 1).sum())
        st = b.read_state(ids[1])
        st["vel"][scs[1].solid_n + 3, 0] = np.nan
        b.write_state(ids[1], vel=st["vel"])
        b.step(DT, NSUB)
        with pytest.raises(L.UpbdError, match=f"NAN.*scene {ids[1]}"):
            b.sync()


def test_autotune_leaves_results_unchanged():
    scs = small_scenes()
    with B.Batch(variant="parity", max_scenes=4) as b:
        ids = [b.add_scene(sc) for sc in scs]
        step(b, 2)
        best, table = B.autotune(b, dict(zip(ids, scs)), frames=2, block_threads=(128, 256),
                                 ctas_per_sm=(4, 8), warm_frames=1)
        assert len(table) == 4 and best in table
        info = b.info()
        assert (info.block_threads, info.ctas_per_sm) == (best.block_threads, best.ctas_per_sm)
        step(b, 3)
        for sid, sc in zip(ids, scs):
            assert_states_equal(b.read_state(sid), run_plain(sc, 5, "parity")[0], f"after tuning {sid}")
