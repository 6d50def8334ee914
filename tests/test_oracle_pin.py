"""Pins O2's floating-point passes to the reference's executed arithmetic.

O2 (oracle/o2_sim.cpp) restates the WGSL kernels (src/gpu/wgsl.js); the CUDA
parity build matches it bit for bit. O1 (oracle/o1_solver.cpp) restates the
CPU solver (src/solver.js) and reproduces that file's own execution bit for
bit (tests/test_golden.py, through tests/golden/jsmini.py). Where the two
reference implementations compute the same per-particle rule, this file runs
the O1 pass and the O2 pass from one identical state and requires the results
to agree to within the difference of their arithmetic: O1 computes in double
and rounds to float32 on every typed-array store (JavaScript), O2 in float32
throughout. So the GPU parity chain reaches the reference's executed
arithmetic for:
  - fluid density rho / rho_near  src/solver.js:296-320  vs src/gpu/wgsl.js:254-279
  - the DDR displacement + apply  src/solver.js:323-353  vs src/gpu/wgsl.js:281-323
  - floor / walls / cull          src/solver.js:389-427  vs src/gpu/wgsl.js:663-697
  - velocity, damping, clamp      src/solver.js:219-234  vs src/gpu/wgsl.js:700-710
  - the XSPH blend, at the same neighbour set
                                  src/solver.js:431-454  vs src/gpu/wgsl.js:745-778
  - solid-fluid contact push with the CPU solver's pair scale 1, on isolated
    pairs (where Gauss-Seidel and Jacobi coincide)
                                  src/solver.js:246-279  vs src/gpu/wgsl.js:609-660
Both solvers sum the same terms over the pairs within H, so away from hash
collisions the only differences are rounding. At a hash collision (two of a
particle's 27 neighbour cells in one bucket) the two reference
implementations differ by rule: the CPU solver visits pair (i, j), i < j, as
often as j's bucket occurs among i's 27 buckets and adds the term that many
times to both ends (src/solver.js:302-319); the WGSL gather uses each
particle's own 27 buckets (src/gpu/wgsl.js:262-275). The CUDA path follows
the WGSL rule. The gather comparisons therefore leave out the particles that
a collision reaches (`_collision_reach`; a few per cent at most, asserted).

Tolerances (max-norm): density 2e-6 relative to the largest density;
displacement 1e-5 relative to the largest displacement plus two float32 ulps
of the coordinate (both sides round the moved position once); positions after
bounds and contacts 1e-6 m; velocities 1e-6 relative to maxSpeed (14 m/s) or
the largest speed; xsph velocities 1e-5 relative to the largest speed.
"""
import numpy as np
import pytest

from fluidphysics_b200 import scenes as S
from oracle.oracle import o1_from_scene, o2_from_scene

GOLDEN = np.load(__import__("pathlib").Path(__file__).resolve().parent / "golden" / "solver_js_c1.npz")
PASS_GRID, PASS_DENSITY, PASS_DISP, PASS_APPLY_FLUID = 2, 3, 4, 5
PASS_CONTACTS, PASS_APPLY_ALL, PASS_BOUNDS, PASS_VELOCITY, PASS_XSPH, PASS_XSPH_APPLY = 9, 10, 11, 12, 14, 15
H_SUB = 1 / 300


def _pair(scene, pos3, prev3=None, vel3=None, active=None):
    """O1 and O2 holding the same scene and the same state."""
    o1, o2 = o1_from_scene(scene), o2_from_scene(scene)
    n = scene.total
    pos3 = np.asarray(pos3, np.float32).reshape(n, 3)
    prev3 = pos3 if prev3 is None else np.asarray(prev3, np.float32).reshape(n, 3)
    vel3 = np.zeros((n, 3), np.float32) if vel3 is None else np.asarray(vel3, np.float32).reshape(n, 3)
    active = np.ones(n, np.uint8) if active is None else np.asarray(active, np.uint8)
    o1.set("pos", pos3)
    o1.set("prev", prev3)
    o1.set("vel", vel3)
    o1.set("active", active)
    st = o2.read_state()
    p4, pv4, v4 = st["pos"].copy(), st["prev"].copy(), st["vel"].copy()
    p4[:, :3], pv4[:, :3], v4[:, :3] = pos3, prev3, vel3
    pv4[:, 3] = 0.0
    v4[:, 3] = 0.0
    o2.write_state(pos=p4, prev=pv4, vel=v4, flags=active.astype(np.uint32))
    return o1, o2


def _c1_settled():
    sc = S.cpu_scene()
    return sc, dict(pos3=GOLDEN["c1_settled_in_pos"], prev3=GOLDEN["c1_settled_in_prev"],
                    vel3=GOLDEN["c1_settled_in_vel"], active=GOLDEN["c1_settled_in_active"])


def _c1_frame1():
    sc = S.cpu_scene()
    return sc, dict(pos3=GOLDEN["c1_frame1_pos"], vel3=GOLDEN["c1_frame1_vel"], active=GOLDEN["c1_frame1_active"])


def _c2_settling():
    """The 73,536-particle GPU scene two frames in (O2 FP32): a falling,
    compressing block with pressure everywhere."""
    sc = S.gpu_default(frames=1)
    o2 = o2_from_scene(sc)
    for _ in range(2):
        o2.step(sc.dt, sc.substeps)
    st = o2.read_state()
    return sc, dict(pos3=st["pos"][:, :3], prev3=st["prev"][:, :3], vel3=st["vel"][:, :3],
                    active=(st["flags"] & 1).astype(np.uint8))


STATES = {"c1_settled": _c1_settled, "c1_frame1": _c1_frame1, "c2_settling": _c2_settling}


@pytest.fixture(scope="module", params=sorted(STATES))
def state(request, oracle_lib):
    return STATES[request.param]()


PRIMES = (92837111, 689287499, 283923481)


def _dup27(pos, scene):
    """Per particle: True when two of its 27 neighbour cells share a hash
    bucket (Solver._hash: floor(p * (1/cellSize)) in double, products
    wrapped to 32 bits, xor, mask)."""
    inv = 1.0 / scene.params.cell_size
    c = np.floor(np.asarray(pos, np.float32).astype(np.float64) * inv).astype(np.int64)
    T = scene.desc.table_size
    off = np.array([(a, b, d) for a in (-1, 0, 1) for b in (-1, 0, 1) for d in (-1, 0, 1)], np.int64)
    cc = c[:, None, :] + off[None]
    h = ((cc[..., 0] * PRIMES[0]) ^ (cc[..., 1] * PRIMES[1]) ^ (cc[..., 2] * PRIMES[2])) & (T - 1)
    h.sort(axis=1)
    return (np.diff(h, axis=1) == 0).any(axis=1)


def _collision_reach(pos, scene, active, hops):
    """Fluid particles within `hops` neighbour steps (pairs closer than H,
    with a 1e-5 margin) of a particle whose 27 buckets collide."""
    from scipy.spatial import cKDTree
    idx = np.flatnonzero(_fluid_mask(scene, active))
    p = np.asarray(pos, np.float64).reshape(-1, 3)
    dirty = np.zeros(len(p), bool)
    dirty[idx] = _dup27(p[idx], scene)
    pairs = cKDTree(p[idx]).query_pairs(scene.params.fluid_h * (1 + 1e-5), output_type="ndarray")
    a, b = idx[pairs[:, 0]], idx[pairs[:, 1]]
    for _ in range(hops):
        nxt = dirty.copy()
        nxt[a[dirty[b]]] = True
        nxt[b[dirty[a]]] = True
        dirty = nxt
    return dirty


def _fluid_mask(scene, active):
    m = np.asarray(active, bool).copy()
    m[: scene.solid_n] = False
    return m


def test_density_matches_cpu_solver(state):
    sc, st = state
    o1, o2 = _pair(sc, **st)
    o1.run_pass("grid")
    o1.run_pass("fluid")
    sz = o1.sizes()
    assert sz["pairCount"] < sz["maxPairs"], "pair cap hit: the CPU solver would drop pairs"
    o2.run_pass(PASS_GRID)
    o2.run_pass(PASS_DENSITY)
    d2 = o2.read_state()["density"]
    m = _fluid_mask(sc, st["active"])
    reach = _collision_reach(st["pos3"], sc, st["active"], 1)
    assert reach[m].mean() < 0.05, reach[m].mean()
    m &= ~reach
    rho1, rn1 = o1.get("rho")[m].astype(np.float64), o1.get("rhoNear")[m].astype(np.float64)
    rho2, rn2 = d2[m, 0], d2[m, 1]
    assert rho1.max() > 0.5  # neighbours present
    assert np.abs(rho1 - rho2).max() <= 2e-6 * rho1.max()
    assert np.abs(rn1 - rn2).max() <= 2e-6 * rn1.max()


def test_displacement_matches_cpu_solver(state):
    sc, st = state
    o1, o2 = _pair(sc, **st)
    x0 = np.asarray(st["pos3"], np.float64).reshape(-1, 3)
    o1.run_pass("grid")
    o1.run_pass("fluid")
    x1 = o1.get("pos").astype(np.float64).reshape(-1, 3)
    o2.run_pass(PASS_GRID)
    o2.run_pass(PASS_DENSITY)
    o2.run_pass(PASS_DISP)
    o2.run_pass(PASS_APPLY_FLUID)
    x2 = o2.read_state()["pos"][:, :3]
    m = _fluid_mask(sc, st["active"])
    reach = _collision_reach(x0, sc, st["active"], 2)  # neighbours' densities enter the pressure
    assert reach[m].mean() < 0.08, reach[m].mean()
    m &= ~reach
    d1, d2 = (x1 - x0)[m], (x2 - x0)[m]
    scale = np.abs(d1).max()
    assert scale > 1e-6  # pressure moved the fluid
    # plus two float32 ulps of the coordinate: both round the moved position once
    ulp = np.spacing(np.abs(x0[m]).astype(np.float32)).astype(np.float64)
    assert (np.abs(d1 - d2) <= 1e-5 * scale + 2 * ulp).all(), np.abs(d1 - d2).max() / scale
    # solids untouched by both
    assert np.array_equal(x1[: sc.solid_n], x0[: sc.solid_n].astype(np.float32).astype(np.float64))


def _bounds_state(sc, seed):
    """Positions placed at the floor, inside and outside both walls, over the
    wall height, and past the cull limits, with previous positions offset so
    that floor friction acts."""
    rng = np.random.default_rng(seed)
    p = sc.params
    n = sc.total
    pos = np.zeros((n, 3))
    k = np.arange(n) % 8
    pos[:, 0] = rng.uniform(-3.0, 3.0, n)
    pos[:, 2] = rng.uniform(-3.0, 3.0, n)
    pos[:, 1] = rng.uniform(0.2, 2.0, n)
    below = k == 0
    pos[below, 1] = rng.uniform(-0.1, 0.05, below.sum())                    # under the floor
    wx = k == 1
    pos[wx, 0] = rng.choice([-1, 1], wx.sum()) * (p.wall_x + rng.uniform(-0.15, 0.15, wx.sum()))
    pos[wx, 1] = rng.uniform(0.0, p.wall_h + 0.2, wx.sum())                  # near the x walls
    wz = k == 2
    pos[wz, 2] = rng.choice([-1, 1], wz.sum()) * (p.wall_z + rng.uniform(-0.15, 0.15, wz.sum()))
    pos[wz, 1] = rng.uniform(0.0, p.wall_h + 0.2, wz.sum())                  # near the z walls
    corner = k == 3
    pos[corner, 0] = np.sign(rng.normal(size=corner.sum())) * (p.wall_x + rng.uniform(-0.1, 0.1, corner.sum()))
    pos[corner, 2] = np.sign(rng.normal(size=corner.sum())) * (p.wall_z + rng.uniform(-0.1, 0.1, corner.sum()))
    pos[corner, 1] = rng.uniform(-0.05, 0.5, corner.sum())
    cull = k == 4
    pos[cull, 0] = rng.uniform(6.0, 8.0, cull.sum())                        # near the cull radius
    pos[cull, 1] = rng.uniform(-3.5, 3.0, cull.sum())
    prev = pos + rng.normal(scale=0.01, size=pos.shape)
    return pos.astype(np.float32), prev.astype(np.float32)


@pytest.mark.parametrize("seed", [1, 2])
def test_bounds_match_cpu_solver(oracle_lib, seed):
    sc = S.cpu_scene()
    pos, prev = _bounds_state(sc, seed)
    o1, o2 = _pair(sc, pos, prev3=prev)
    o1.run_pass("bounds")
    o2.run_pass(PASS_BOUNDS)
    x1 = o1.get("pos").astype(np.float64).reshape(-1, 3)
    st = o2.read_state()
    moved = np.abs(x1 - pos).max(axis=1) > 0
    assert moved.sum() > 0.2 * sc.total  # the floor, walls and friction acted
    assert np.abs(x1 - st["pos"][:, :3]).max() <= 1e-6
    culled1 = o1.get("active") == 0
    assert culled1.sum() > 0
    assert np.array_equal(culled1, (st["flags"] & 1) == 0)


def test_velocity_update_matches_cpu_solver(state):
    sc, st = state
    rng = np.random.default_rng(3)
    n = sc.total
    pos = np.asarray(st["pos3"], np.float32).reshape(n, 3)
    # previous positions spread over speeds up to 1.5 x maxSpeed, so the clamp acts
    step = rng.normal(size=(n, 3))
    step *= (rng.uniform(0, 1.5 * sc.params.max_speed, n) * H_SUB / np.linalg.norm(step, axis=1))[:, None]
    prev = (pos - step).astype(np.float32)
    o1, o2 = _pair(sc, pos, prev3=prev, active=st["active"])
    o1.run_pass("velocity", H_SUB)
    o2.run_pass(PASS_VELOCITY, H_SUB)
    a = np.asarray(st["active"], bool)
    v1 = o1.get("vel").astype(np.float64).reshape(-1, 3)[a]
    v2 = o2.read_state()["vel"][a, :3]
    sp = np.linalg.norm(v1, axis=1)
    assert sp.max() <= sc.params.max_speed * (1 + 1e-6) and (sp > 0.99 * sc.params.max_speed).any()
    assert np.abs(v1 - v2).max() <= 1e-6 * sc.params.max_speed


def _borderline(pos, idx, H, rel=1e-5):
    """Fluid particles with a neighbour whose distance lies within `rel` of H:
    float32 and float64 decide those pairs differently."""
    from scipy.spatial import cKDTree
    p = pos[idx].astype(np.float64)
    tree = cKDTree(p)
    pairs = tree.query_pairs(H * (1 + rel), output_type="ndarray")
    d = np.linalg.norm(p[pairs[:, 0]] - p[pairs[:, 1]], axis=1)
    b = pairs[d > H * (1 - rel)]
    out = np.zeros(len(pos), bool)
    out[idx[b.ravel()]] = True
    return out


def test_xsph_matches_cpu_solver_at_the_same_neighbours(state):
    """The CPU solver blends over the pairs its density pass found, the WGSL
    kernel over the neighbours at xsph time: from one position state with no
    move in between, both neighbour sets are the pairs within H."""
    sc, st = state
    rng = np.random.default_rng(4)
    n = sc.total
    vel = rng.normal(scale=1.0, size=(n, 3)).astype(np.float32)
    o1, o2 = _pair(sc, **{**st, "vel3": vel})
    o1.run_pass("grid")
    o1.run_pass("fluid")           # the pair cache at these positions (moves positions,
    o1.set("vel", vel)             # which xsph does not read)
    o1.run_pass("viscosity")
    o2.run_pass(PASS_GRID)
    o2.run_pass(PASS_XSPH)
    o2.run_pass(PASS_XSPH_APPLY)
    m = _fluid_mask(sc, st["active"])
    idx = np.flatnonzero(m)
    pos = np.asarray(st["pos3"], np.float64).reshape(n, 3)
    border = _borderline(pos, idx, sc.params.fluid_h)
    reach = _collision_reach(pos, sc, st["active"], 1)
    keep = m & ~border & ~reach
    assert border[m].mean() < 0.01 and reach[m].mean() < 0.05
    v1 = o1.get("vel").astype(np.float64).reshape(-1, 3)[keep]
    v2 = o2.read_state()["vel"][keep, :3]
    vin = vel.astype(np.float64)[keep]
    assert np.abs(v1 - vin).max() > 0.1  # the blend acted
    assert np.abs(v1 - v2).max() <= 1e-5 * np.abs(vin).max()


def test_isolated_contacts_match_cpu_solver(oracle_lib):
    """Solid-fluid pairs where every particle touches exactly one other: the
    CPU solver's Gauss-Seidel push and the WGSL gather + applyDeltaAll (with
    the CPU pair scale 1) compute the same correction."""
    sc = S.cpu_scene()
    assert sc.params.contact_scale == 1.0
    d, p = sc.desc, sc.params
    n = d.solid_dim
    k = np.arange(sc.solid_n)
    lat = np.stack([k // (n * n), (k // n) % n, k % n], 1)
    spos = np.asarray(d.cube_center[:3]) + (lat - (n - 1) / 2) * d.spacing
    pos = np.zeros((sc.total, 3))
    pos[: sc.solid_n] = spos
    top = np.flatnonzero((lat[:, 1] == n - 1) & (lat[:, 0] % 2 == 0) & (lat[:, 2] % 2 == 0))
    rng = np.random.default_rng(5)
    rsum = p.solid_radius + p.fluid_radius
    active = np.zeros(sc.total, np.uint8)
    active[: sc.solid_n] = 1
    for m, s in enumerate(top):
        f = sc.solid_n + m
        u = np.array([rng.uniform(-0.3, 0.3), 1.0, rng.uniform(-0.3, 0.3)])
        pos[f] = spos[s] + u / np.linalg.norm(u) * rsum * rng.uniform(0.85, 0.97)
        active[f] = 1
    pos[sc.solid_n + len(top):] = [0.0, 9.0, 0.0]  # inactive
    o1, o2 = _pair(sc, pos.astype(np.float32), active=active)
    o1.run_pass("grid")
    o1.run_pass("contacts")
    o2.run_pass(PASS_GRID)
    o2.run_pass(PASS_CONTACTS)
    o2.run_pass(PASS_APPLY_ALL)
    x0 = pos.astype(np.float32).astype(np.float64)
    x1 = o1.get("pos").astype(np.float64).reshape(-1, 3)
    x2 = o2.read_state()["pos"][:, :3]
    a = active.astype(bool)
    push = np.linalg.norm((x1 - x0)[a], axis=1)
    assert (push > 1e-4).sum() == 2 * len(top)  # every pair pushed, both ends
    assert np.abs(x1 - x2)[a].max() <= 1e-6
