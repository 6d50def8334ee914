"""Aggregate physical checks of the default GPU scene, the ones the
reference's app exposes for tuning (window.__sim.metrics and cutLine,
src/gpu/main.js:542-578): after two seconds no non-finite position, the
body above the floor, all fluid active and pooled in the basin; a cutLine
slice through the body queued one segment per frame cuts constraints."""
import numpy as np
import pytest

from fluidphysics_b200 import scenes as S
from fluidphysics_b200.sim import cut_line_segments, sim_from_scene, state_metrics

pytestmark = pytest.mark.gpu


def test_metrics_and_cut_line_on_default_scene():
    sc = S.gpu_default(frames=150)
    sim = sim_from_scene(sc)
    for _ in range(120):
        sim.step(sc.dt, sc.substeps)
    m = state_metrics(sim.read_state(), sc.solid_n)
    r_s = float(sc.params.solid_radius)
    assert m["solid"]["bad"] == 0 and m["fluid"]["bad"] == 0
    assert m["solid"]["minY"] >= r_s * 0.9, m
    assert m["fluid"]["n"] == sc.desc.max_fluid, m
    assert m["fluid"]["pooledPct"] >= 90, m
    alive0 = int(sim.read_constraints()[:, 3].sum())
    c = np.array(sc.desc.cube_center)
    segs = cut_line_segments(float(c[0]), [0.0, 2.5, 4.0])
    for o, d1, d2 in segs:
        sim.slice(o, d1, d2)
    for _ in range(len(segs) + 3):  # one segment per frame
        sim.step(sc.dt, sc.substeps)
    alive1 = int(sim.read_constraints()[:, 3].sum())
    m1 = state_metrics(sim.read_state(), sc.solid_n)
    assert alive1 < alive0, (alive0, alive1)
    assert m1["solid"]["bad"] == 0 and m1["fluid"]["bad"] == 0
    print("metrics", m, "alive", alive0, "->", alive1)
    sim.close()
