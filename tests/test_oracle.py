"""CPU checks of the two oracles against each other and against the
reference's own invariants (no GPU)."""
import math

import numpy as np
import pytest

from fluidphysics_b200 import scenes as S
from oracle.oracle import O1, O2, o1_from_scene, o2_from_scene


def js_toint32(x: float) -> int:
    """ECMAScript ToInt32 written with Python integers."""
    if not math.isfinite(x):
        return 0
    i = int(x)  # trunc
    i &= 0xFFFFFFFF
    return i - (1 << 32) if i >= (1 << 31) else i


def js_hash(xi, yi, zi, T):
    a = js_toint32(xi * 92837111.0)
    b = js_toint32(yi * 689287499.0)
    c = js_toint32(zi * 283923481.0)
    return ((a ^ b ^ c) & 0xFFFFFFFF) & (T - 1)


def test_constraint_counts_match_reference(oracle_lib):
    # 3n^2(n-1) + 6n(n-1)^2 + 4(n-1)^3 lattice bonds; README.md:12 "~94k" at 20^3
    for n, sc in ((7, S.cpu_scene()), (20, S.gpu_default(frames=1))):
        o2 = O2(sc.desc, sc.params)
        assert o2.info.num_cons == 3 * n * n * (n - 1) + 6 * n * (n - 1) ** 2 + 4 * (n - 1) ** 3
        assert o2.info.num_tets == 5 * (n - 1) ** 3
    assert O2(S.gpu_default(frames=1).desc, S.gpu_default(frames=1).params).info.num_cons == 93556


def test_o1_grid_hash_is_js_semantics(oracle_lib):
    sc = S.cpu_scene()
    o1 = o1_from_scene(sc)
    o1.run_pass("grid")
    pos = o1.get("pos").reshape(-1, 3)
    act = o1.get("active")
    T = o1.sizes()["tableSize"]
    inv = 1 / 0.22
    cs = o1.get("cellStart")
    ce = o1.get("cellEntries")
    # every active particle sits in the bucket of its JS hash; buckets list
    # members in descending index order (src/solver.js:182-183)
    for i in np.flatnonzero(act)[::37]:
        h = js_hash(math.floor(float(pos[i, 0]) * inv), math.floor(float(pos[i, 1]) * inv),
                    math.floor(float(pos[i, 2]) * inv), T)
        assert i in ce[cs[h]:cs[h + 1]]
    for h in np.flatnonzero(np.diff(cs) > 1)[:200]:
        b = ce[cs[h]:cs[h + 1]]
        assert np.all(np.diff(b) < 0)
    assert cs[-1] == act.sum()


def test_js_toint32_edges():
    assert js_toint32(2.0 ** 31) == -(2 ** 31)
    assert js_toint32(-1.0) == -1
    assert js_toint32(float("nan")) == 0
    assert js_toint32(2.0 ** 53 + 2) == 2


@pytest.mark.parametrize("mk", [S.cpu_scene, lambda: S.gpu_default(frames=1)])
def test_o1_o2_grids_agree(oracle_lib, mk):
    sc = mk()
    o1 = o1_from_scene(sc)
    o2 = o2_from_scene(sc)
    o1.run_pass("grid")
    o2.rebuild_grid()
    counts, offs, ent = o2.read_grid()
    assert np.array_equal(o1.get("cellStart").astype(np.uint32), offs)
    assert np.array_equal(o1.get("cellEntries")[: offs[-1]].astype(np.uint32), ent)
    assert np.array_equal(np.diff(offs), counts)


def test_o1_o2_cut_and_pick_agree(oracle_lib):
    sc = S.gpu_default(frames=1)
    o1 = o1_from_scene(sc)
    o2 = o2_from_scene(sc)
    o, d1, d2 = sc.wedge
    n1 = o1.cut(o, d1, d2)
    n2 = o2.slice_now(o, d1, d2)
    assert n1 == n2 and n1 > 100
    c2, _ = o2.read_constraints()
    assert np.array_equal(o1.get("consAlive").astype(np.uint32), c2[:, 3])
    rng = np.random.default_rng(7)
    c = np.array(sc.desc.cube_center)
    for _ in range(50):
        ro = c + rng.normal(size=3) * 4
        rd = (c + rng.normal(size=3) * 0.3) - ro
        rd /= np.linalg.norm(rd)
        assert o1.pick(ro, rd, 0.25) == o2.pick(ro, rd, 0.25)


def test_o1_groups_after_cut(oracle_lib):
    sc = S.cpu_scene()
    o1 = o1_from_scene(sc)
    o2 = o2_from_scene(sc)
    # a vertical wedge between two lattice layers (x = 0.09) splits the cube
    # in two; a plane through a layer cuts nothing (sa*sb >= 0 keeps it)
    o = (0.09, 2.0, 10.0)
    d1 = np.array([0.0, 3.0, -10.0]) / np.linalg.norm([0.0, 3.0, -10.0])
    d2 = np.array([0.0, -3.0, -10.0]) / np.linalg.norm([0.0, -3.0, -10.0])
    assert o1.cut(o, d1, d2) == o2.slice_now(o, d1, d2) > 0
    o1.run_pass("groups")
    g1 = o1.get("group")[:343]
    assert np.array_equal(g1, o2.groups())
    assert len(set(g1.tolist())) == 2


def test_o2_float_and_double_stay_close(oracle_lib):
    sc = S.cpu_scene()
    f = o2_from_scene(sc, 0)
    d = o2_from_scene(sc, 1)
    for _ in range(10):
        f.step(1 / 60, 5)
        d.step(1 / 60, 5)
    a, b = f.read_state(), d.read_state()
    assert np.array_equal(a["flags"], b["flags"])
    # the body stays close particle by particle; the fluid is chaotic (single
    # particles part ways within a frame), so it is compared in aggregate
    assert np.abs(a["pos"][:343, :3] - b["pos"][:343, :3]).max() < 1e-4
    fa, fb = a["pos"][343:, :3], b["pos"][343:, :3]
    assert np.abs(fa.mean(0) - fb.mean(0)).max() < 1e-4
    assert np.abs(fa - fb).max() < 5e-2


def test_o2_scene_settles_without_nan(oracle_lib):
    sc = S.cpu_scene()
    o2 = o2_from_scene(sc)
    for _ in range(60):
        o2.step(1 / 60, 5)
    st = o2.read_state()
    assert not np.isnan(st["pos"]).any()
    body = st["pos"][:343, 1]
    assert body.min() > 0.05  # resting on the floor, not through it
    assert o2.active_count() > 2000
    assert o2.health() == 0


def test_o2_reset_solid_rewrites_buffers(oracle_lib):
    sc = S.cpu_scene()
    o2 = o2_from_scene(sc)
    o2.step(1 / 60, 5)
    o2.reset_solid()
    st = o2.read_state()
    # GpuSim.resetSolid rewrites pos/prev of every slot and zeroes every velocity
    assert np.all(st["vel"] == 0)
    assert np.all(st["pos"][343:, :3] == 0)
    assert np.all(st["flags"][:343] == 1)


def test_emit_ring_buffer_wraps(oracle_lib):
    sc = S.cpu_scene()
    o2 = o2_from_scene(sc)
    assert o2.fluid_next() == 0  # 2600 emitted into a 2600 ring
    o2.emit(256, (0, 3, 0), (0, -1, 0), (1, 0, 0), (0, 0, 1), 3.0, 0.0)
    o2.step(1 / 60, 5)
    assert o2.fluid_next() == 256
    assert o2.active_count() <= 2600


def _mark_rule_misses(sc, st, cons=None):
    """Fluid particles that the oracle's contact pass (the reference's
    contacts kernel restated) gives a contact but that the library's contact
    marks would leave unmarked, so that they would skip their contact walk.
    The library marks fluid particle i when (a) its displacement moved it into
    another cell, or (b) some solid j, at its position after the solve, has
    i's grid bucket among the 27 around its own cell and lies within
    (r_s + r_f + 0.35 H) * 1.001 of i's grid position (float32 arithmetic,
    as the kernels do). Returns (misses, contacted fluid, of which by (b) only
    through the widened reach)."""
    from fluidphysics_b200 import _lib as L
    h = sc.dt / sc.substeps
    p = sc.params
    inv = 1.0 / p.cell_size
    T = sc.desc.table_size
    n_s = sc.solid_n
    o2 = O2(sc.desc, sc.params)

    def run(last):
        o2.write_state(**st)
        if cons is not None:
            o2.write_constraints(cons)
        o2.substep_partial(h, last)
        return o2.read_state()

    grid = run(L.PASS["GRID"])["pos"][:, :3].astype(np.float32)
    moved = run(L.PASS["APPLY_FLUID"])["pos"][:, :3].astype(np.float32)
    after = run(L.PASS["CONTACTS"])
    delta = o2.read_delta()
    fin = after["pos"][:n_s, :3].astype(np.float32)
    act = (after["flags"] & 1).astype(bool)
    cell = lambda q: np.floor(q.astype(np.float64) * inv)
    rsum = np.float32(p.solid_radius) + np.float32(p.fluid_radius)
    reach = (rsum + np.float32(0.35) * np.float32(p.fluid_h)) * np.float32(1.001)
    lim2 = reach * reach * np.float32(1.00001)
    fin_cells = cell(fin)
    # the widened reach rests on the displacement pass's clamp (0.35 H)
    fl = np.flatnonzero(act[n_s:]) + n_s
    step = np.linalg.norm(moved[fl].astype(np.float64) - grid[fl].astype(np.float64), axis=1)
    assert step.size == 0 or step.max() <= 0.35 * p.fluid_h * (1 + 1e-5), step.max()
    contacted = np.flatnonzero(act[n_s:] & (delta[n_s:, 3] > 0)) + n_s
    misses, widened = [], 0
    for i in contacted:
        ci = cell(grid[i])
        if (ci != cell(moved[i])).any():
            continue  # (a)
        bi = js_hash(ci[0], ci[1], ci[2], T)
        near = np.flatnonzero(act[:n_s] & (np.abs(fin_cells - ci).max(axis=1) <= 2))
        ok = False
        for j in near:
            d = fin[j] - grid[i]
            if not (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < lim2):
                continue
            fc = fin_cells[j]
            around = {js_hash(fc[0] + a, fc[1] + b, fc[2] + c, T) for a in (-1, 0, 1) for b in (-1, 0, 1)
                      for c in (-1, 0, 1)}
            if bi in around:
                ok = True
                dm = fin[j] - moved[i]
                widened += int(not (float(np.dot(d, d)) < float(rsum) ** 2) and float(np.dot(dm, dm)) < float(rsum) ** 2)
                break
        if not ok:
            misses.append(int(i))
    return misses, len(contacted), widened


@pytest.mark.parametrize("case", ["frame50", "frame60", "crossing"])
def test_contact_mark_rules_cover_every_oracle_contact(oracle_lib, case):
    """The marking rules of the library's contact pass, evaluated on the
    oracle's own substep: every fluid particle the reference's contacts
    kernel gives a contact is marked, in the CPU scene at frames 50 and 60
    (the fluid block landing on the lattice: 170-180 fluid particles in
    contact, some of them reached only through the widened reach) and in
    the crossing case (a particle pushed across a cell boundary into
    contact, which only the cell-change rule marks)."""
    from helpers import crossing_state, settled_state
    sc = S.cpu_scene()
    if case.startswith("frame"):
        _, st, cons = settled_state(sc, int(case[5:]))
    else:
        st, _, _, _ = crossing_state(sc)
        cons = None
    misses, n, widened = _mark_rule_misses(sc, st, cons)
    print(case, "contacted fluid", n, "reached only through the widened reach", widened)
    assert n > 0
    assert not misses, misses[:8]
