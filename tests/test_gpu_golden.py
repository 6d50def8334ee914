"""The CUDA library against golden vectors produced by the reference's own
code (src/solver.js and src/gpu/sim.js run unmodified; see
tests/golden/make_golden.py): the scene builder's uploads, the hash grid and
the wedge cut of the GPU default scene, pick rays — all bit for bit."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from fluidphysics_b200 import scenes as S
from fluidphysics_b200.sim import Sim, sim_from_scene

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"
J = json.loads((GOLD / "solver_js.json").read_text())
NPZ = np.load(GOLD / "solver_js_c1.npz")


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", ["small", "default"])
def test_scene_upload_matches_gpusim_build(name):
    b = J["cases"]["gpu_build"][name]
    opts = dict(b["opts"])
    opts["SOLID_DIM"] = int(opts["SOLID_DIM"])
    opts["MAX_FLUID"] = int(opts["MAX_FLUID"])
    opts["SOLID_DIM2"] = b["dim2"]
    sim = Sim(S.desc_from_opts(opts, features=1), S.default_params())
    assert sim.info.num_cons == b["num_cons"] and sim.info.num_tets == b["num_tets"]
    st = sim.read_state()
    assert digest(st["pos"].reshape(-1)) == b["digest"]["pos"]
    assert digest(st["flags"]) == b["digest"]["flags"]
    assert digest(sim.read_constraints().reshape(-1)) == b["digest"]["cons"]
    assert digest(sim.read_adjacency()) == b["digest"]["adj"]
    assert digest(sim.read_tets().reshape(-1)) == b["digest"]["tetData"]


def test_grid_and_cut_of_default_scene_match_solver_js():
    case = J["cases"]["c2_grid_cut"]
    sc = S.gpu_default(frames=1)
    assert sc.params.cell_size == case["cellSize"]
    sim = sim_from_scene(sc)
    assert sim.info.table_size == case["tableSize"]
    sim.rebuild_grid()
    counts, offs, ent = sim.read_grid()
    assert digest(offs.view(np.int32)) == case["digest"]["cellStart"]
    # cellEntries of the reference has `capacity` entries, all filled (every
    # particle is active in this scene)
    assert digest(ent.view(np.int32)) == case["digest"]["cellEntries"]
    o, d1, d2 = sc.wedge
    assert sim.slice_now(o, d1, d2) == case["cut_count"]
    assert digest(sim.read_constraints()[:, 3].astype(np.uint8)) == case["digest"]["consAlive"]


def _c1_tools_sim():
    """A GPU sim of the CPU scene whose body holds the positions the golden
    tool case ran on (the settled substep's output)."""
    sc = S.cpu_scene()
    sim = sim_from_scene(sc)
    # the golden picks ran on the settled-substep output; rebuild that body state
    from oracle.oracle import O1
    o = O1(2600, gravity=-9.8)
    o.add_solid_cube(0, 2.0, 0, 7, 0.18, 0.08)
    fl = sc.fluid_pos.astype(np.float64)
    o.emit_fluid(fl, np.zeros_like(fl), 0.03)
    for k in ("pos", "prev", "vel", "active", "consRest", "consAlive"):
        o.set(k, NPZ[f"c1_settled_in_{k}"])
    o.step(1 / 300, 1)
    assert np.array_equal(o.get("pos"), NPZ["c1_settled_out_pos"])
    st = sim.read_state()
    st["pos"][:, :3] = o.get("pos").reshape(-1, 3)
    sim.write_state(pos=st["pos"])
    return sim


def test_pick_rays_match_solver_js():
    """pickSolid rays of the golden case, on the same body positions."""
    case = J["cases"]["c1_tools"]
    sim = _c1_tools_sim()
    for p in case["picks"]:
        i, t = sim.pick(p["o"], p["d"], p["maxPerp"])
        if p["id"] is None:
            assert i == -1
        else:
            assert i == p["id"] and t == p["t"]


def test_groups_after_cuts_match_solver_js():
    """Solver._recomputeGroups (src/solver.js:488-499) on the GPU after the
    golden case's cuts: the alive flags and every solid's group label equal
    those the unmodified solver.js produced (labels are the roots its
    order of unions leaves, not component minima)."""
    case = J["cases"]["c1_tools"]
    sim = _c1_tools_sim()
    for c in case["cuts"]:
        assert sim.slice_now(c["o"], c["d1"], c["d2"]) == c["count"]
        assert digest(sim.read_constraints()[:, 3].astype(np.uint8)) == c["alive"]
    g = sim.groups()
    assert g.tolist() == case["group"]
    assert len(set(case["group"])) > 1
