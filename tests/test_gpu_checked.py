"""The checked build (libupbd_checked.so: the product sources with
UPBD_CHECKED_BUILD): every index the gathers take from device arrays is
tested against its array's extent before use, and one out of range would set
UPBD_HEALTH_BOUNDS and make upbd_sync / upbd_batch_sync fail. It stands in for
a memory checker here: stepping the workloads of the other tests on it, every
such index stays in range (health word 0, syncs succeed), and its substep
agrees with the product build's within the product tolerance.

Only valid inputs are given: nothing here plants an index out of range on the
GPU."""
import numpy as np
import pytest

from fluidphysics_b200 import _lib as L
from fluidphysics_b200 import batch as B
from fluidphysics_b200 import scenes as S
from fluidphysics_b200.sim import sim_from_scene
from helpers import assert_states_close, load_state, settled_state

pytestmark = pytest.mark.gpu


def _clean(sim, what):
    sim.sync()  # raises on UPBD_HEALTH_BOUNDS (and NaN)
    assert sim.health() == 0, f"{what}: health bits {sim.health():#x}"


def test_default_scene_with_slice():
    sc = S.gpu_default(frames=70)
    sim = sim_from_scene(sc, "checked")
    for f in range(70):
        if f == sc.slice_frame:
            sim.slice(*sc.wedge)
        sim.step(sc.dt, sc.substeps)
    _clean(sim, "gpu_default")
    sim.close()


def test_optional_passes_companion_cube_slice():
    d, p, opts = S.gpu_scene(10, 4096, 40, iters=3, features=L.FEAT_TETS | L.FEAT_SOLID_CONTACTS)
    d.solid_dim2 = 4
    d.cube2_center[:] = [0.25, 0.5 + 3 * d.spacing / 2 + 1.0, 0.1]
    S.set_params(p, dict(solid_viscosity=0.2))
    fp = S.jittered_block(16, 16, 16, 2.2 * 0.04, 1.9, 9)
    sc = S.Scene("feat", d, p, fp, np.zeros_like(fp), opts["fluidMass"], 1 / 60, 5, 24, slice_frame=8,
                 wedge=S.wedge_through(d.cube_center, 5))
    sim = sim_from_scene(sc, "checked")
    for f in range(sc.frames):
        if f == sc.slice_frame:
            sim.slice(*sc.wedge)
        sim.step(sc.dt, sc.substeps)
    _clean(sim, "tets + solid contacts")
    sim.close()


def test_hose_and_grab():
    d, p, opts = S.gpu_scene(12, 16384, 30, iters=3)
    fp = S.jittered_block(32, 8, 32, 2.2 * 0.03, 1.4, 4)
    sc = S.Scene("hose", d, p, fp, np.zeros_like(fp), opts["fluidMass"], 1 / 60, 5, 30,
                 hose_per_frame=120, hose_seed=4)
    sim = sim_from_scene(sc, "checked")
    c = np.array(d.cube_center)
    sim.grab_select([c[0], c[1] + 5 * d.spacing, c[2]], 3 * d.spacing)
    for f, args in enumerate(S.hose_script(sc, sc.frames)):
        sim.emit(120, *args)
        sim.grab_move([0.0, 0.01 * np.sin(f / 3.0), 0.0])
        sim.step(sc.dt, sc.substeps)
    _clean(sim, "hose + grab")
    sim.close()


def test_batch_of_uneven_scenes():
    scs = B.batch_scenes(6, seed0=2000, dims=(5, 12), fluid_log2=(10.0, 13.0), table="compact")
    with B.Batch(max_scenes=8, variant="checked") as b:
        for sc in scs:
            b.add_scene(sc)
        for _ in range(12):
            b.step(1 / 60, 5)
        b.sync()  # raises on UPBD_HEALTH_BOUNDS in any scene


def test_checked_substep_matches_product():
    sc = S.gpu_default(frames=1)
    _, st, cons = settled_state(sc, 3)
    out = {}
    for variant in ("checked", "product"):
        sim = sim_from_scene(sc, variant)
        load_state(sim, st, cons)
        sim.substep_partial(sc.dt / sc.substeps, 1000)
        out[variant] = sim.read_state()
        if variant == "checked":
            _clean(sim, "substep")
        sim.close()
    assert_states_close(out["checked"], out["product"], "checked vs product")
