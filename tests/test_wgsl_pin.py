"""The oracle's restatement of the WGSL kernels (O2), pass by pass, against
the reference's own WGSL kernels executed on the CPU.

tests/golden/make_golden_wgsl.py ran the shader text that src/gpu/wgsl.js
makes (through tests/golden/jsmini.py) with tests/golden/wgslmini.py, a WGSL
interpreter, on a small scene with every optional pass of the reference's GPU
schedule, and recorded after each pass the buffers it changed
(tests/golden/wgsl_passes.npz). Here each recorded pass's input state is
rebuilt from those buffers, loaded into a fresh oracle, the oracle's pass is
run, and its outputs are compared with the reference's:

  - passes that touch only their own particle or constraint (integrate,
    the applies, bounds, velocity, bond and tet updates, grab select /
    release, the cut of constraints) bit for bit;
  - gathers (density, displacement, solve, tets, solid contacts, contacts,
    solid viscosity, xsph) to the FP32 rounding of a different summation
    order: the reference's atomic scatter leaves a bucket's members in
    ascending index here, the oracle (and the CUDA kernels) in descending
    index, and the oracle deals a gather's terms to lanes;
  - emit, whose sine-hash jitter amplifies the last bit of sin(), to 1e-4 m
    and 2e-2 m/s, the tolerance the GPU's emit test uses.

The GPU parity build reproduces the oracle bit for bit, so these rules of
the CUDA kernels are pinned to the reference's executed WGSL arithmetic."""
import json
from pathlib import Path

import numpy as np
import pytest

from fluidphysics_b200 import _lib as L
from oracle.oracle import o2_from_scene

GOLDEN = Path(__file__).resolve().parent / "golden"


def _gen():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden_wgsl", GOLDEN / "make_golden_wgsl.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


@pytest.fixture(scope="module")
def golden():
    z = np.load(GOLDEN / "wgsl_passes.npz")
    meta = json.loads(bytes(z["meta"]).decode())
    return {k: z[k] for k in z.files if k != "meta"}, meta


@pytest.fixture(scope="module")
def scene():
    return _gen().golden_scene()


def state_before(z, meta, scenario: str, index: int) -> dict:
    st = {k.split("/")[-1]: v.copy() for k, v in z.items() if k.startswith(f"{scenario}/start/")}
    for e in meta["passes"]:
        if e["scenario"] == scenario and e["index"] < index:
            for b in e["changed"]:
                st[b] = z[f"{scenario}/{e['index']}/{b}"].copy()
    return st


def after(z, scenario: str, index: int, st: dict) -> dict:
    out = dict(st)
    for k, v in z.items():
        pre = f"{scenario}/{index}/"
        if k.startswith(pre):
            out[k[len(pre):]] = v
    return out


def load_o2(sc, C: dict, st: dict, grid_state: dict | None = None):
    """A fresh oracle on the scene, its state set to st (and its hash grid
    built from grid_state's positions, as the substep's grid pass would)."""
    o2 = o2_from_scene(sc)
    T, N, S_, NT = C["TABLE"], C["TOTAL"], C["SOLID_N"], C["NUM_TETS"]

    def put(s):
        o2.write_state(pos=s["pos"].astype(np.float64), prev=s["prev"].astype(np.float64),
                       vel=s["vel"].astype(np.float64), density=s["density"].astype(np.float64),
                       flags=s["flags"])
        o2.write_delta(s["delta"].astype(np.float64))
        o2.write_constraints(s["cons"])
        ts = C["TS_TETS"]
        o2.write_tets(s["gridS"][ts:ts + NT * 5].reshape(NT, 5))
        c0 = 2 * T + N + 8
        o2.write_contact_cache(s["gridA"][c0:c0 + S_], s["gridA"][c0 + S_:c0 + S_ + S_ * 40])

    if grid_state is not None:
        put(grid_state)
        o2.run_pass(L.PASS["GRID"])
    put(st)
    return o2


def f32(a):
    return np.asarray(a, dtype=np.float64).astype(np.float32)


def assert_exact(got, want, what):
    g, w = f32(got), np.asarray(want, dtype=np.float32)
    bad = np.flatnonzero(~((g == w) | (np.isnan(g) & np.isnan(w))).reshape(len(g), -1).all(axis=1))
    assert bad.size == 0, f"{what}: differs at {bad[:6]}: oracle {g[bad[:2]]} vs reference {w[bad[:2]]}"


def assert_close(got, want, scale, rtol, what):
    d = np.abs(np.asarray(got, dtype=np.float64) - np.asarray(want, dtype=np.float64))
    err = float(np.nanmax(d)) / scale if d.size else 0.0
    assert err <= rtol, f"{what}: max error {err:.3g} of {scale:g} > {rtol:g}"
    return err


# the oracle's pass for each of the reference's kernels, and how it is compared
KERNELS = {
    "integrate": ("x", "INTEGRATE", "exact"),
    "fluidDensity": ("p", "DENSITY", "gather"),
    "fluidDisp": ("p", "DISP", "gather"),
    "applyDeltaFluid": ("p", "APPLY_FLUID", "exact"),
    "collectContacts": ("x", "COLLECT", "cache"),
    "solidSolve": ("x", "SOLID_SOLVE", "gather"),
    "applyDeltaSolid": ("x", "APPLY_SOLID", "exact"),
    "solveTets": ("x", "SOLVE_TETS", "gather"),
    "applySolidContacts": ("x", "APPLY_SOLID_CONTACTS", "exact"),
    "solidContacts": ("x", "SOLID_CONTACTS", "gather"),
    "bondUpdate": ("x", "BOND_UPDATE", "exact"),
    "tetUpdate": ("x", "TET_UPDATE", "exact"),
    "contacts": ("p", "CONTACTS", "gather"),
    "applyDeltaAll": ("p", "APPLY_ALL", "exact"),
    "bounds": ("p", "BOUNDS", "exact"),
    "velocityUpdate": ("p", "VELOCITY", "exact"),
    "solidVisc": ("x", "SOLID_VISC", "gather"),
    "solidViscApply": ("x", "SOLID_VISC_APPLY", "exact"),
    "xsph": ("p", "XSPH", "gather"),
    "xsphApply": ("p", "XSPH_APPLY", "exact"),
}
GRID_KERNELS = {"fluidDensity", "fluidDisp", "collectContacts", "contacts", "xsph"}


def _passes(meta, scenario):
    return [e for e in meta["passes"] if e["scenario"] == scenario and e["kernel"] in KERNELS]


def _read_o2(o2, C):
    st = o2.read_state()
    T, N, S_, NT = C["TABLE"], C["TOTAL"], C["SOLID_N"], C["NUM_TETS"]
    cc, cl = o2.read_contact_cache()
    return dict(pos=st["pos"], prev=st["prev"], vel=st["vel"], density=st["density"], flags=st["flags"],
                delta=o2.read_delta(), cons=o2.read_constraints()[0], tets=o2.read_tets(), ccount=cc, clist=cl)


def _want(w, C):
    T, N, S_, NT = C["TABLE"], C["TOTAL"], C["SOLID_N"], C["NUM_TETS"]
    ts, c0 = C["TS_TETS"], 2 * T + N + 8
    return dict(pos=w["pos"], prev=w["prev"], vel=w["vel"], density=w["density"], flags=w["flags"],
                delta=w["delta"], cons=w["cons"], tets=w["gridS"][ts:ts + NT * 5].reshape(NT, 5),
                ccount=w["gridA"][c0:c0 + S_], clist=w["gridA"][c0 + S_:c0 + S_ + S_ * 40])


STATE_KEYS = ("pos", "prev", "vel", "density", "flags", "delta", "cons", "tets")


def _compare(kind, kernel, got, want, what):
    """Every state array of the oracle after the pass against the reference's."""
    errs = {}
    for k in STATE_KEYS:
        g, w = got[k], want[k]
        if k in ("flags", "cons", "tets"):
            if k == "tets":  # indices and the sign of the rest volume (dead = negative)
                assert np.array_equal(g[:, :4], w[:, :4]), f"{what}: tet indices"
                gv, wv = g[:, 4].view(np.float32), w[:, 4].view(np.float32)
                assert np.array_equal(gv, wv), f"{what}: tet rest volumes differ at {np.flatnonzero(gv != wv)[:6]}"
            else:
                bad = np.flatnonzero((g != w).reshape(len(g), -1).any(axis=1))
                assert bad.size == 0, f"{what}: {k} differs at {bad[:6]}: {g[bad[:2]]} vs {w[bad[:2]]}"
            continue
        gather_out = kind == "gather" and ((k == "density" and kernel == "fluidDensity") or
                                           (k == "delta" and kernel != "fluidDensity"))
        if gather_out:
            scale = float(np.abs(np.asarray(w, dtype=np.float64)).max()) or 1.0
            errs[k] = assert_close(g, w, scale, 2e-6, f"{what}: {k}")
        else:
            assert_exact(g, w, f"{what}: {k}")
    return errs


def _run(o2, e, h):
    side, name, _ = KERNELS[e["kernel"]]
    if side == "p":
        o2.run_pass(L.PASS[name], h)
    else:
        o2.run_pass_x(name, h, grab_delta_sub=e["uniform"]["grabDelta"][:3])


def test_substep_passes_match_reference_wgsl(golden, scene):
    """Every pass of one whole substep of the reference's GPU schedule
    (GpuSim.encode, src/gpu/sim.js:352-385), each from the reference's own
    state before it."""
    z, meta = golden
    C = meta["C"]
    grid_at = next(e["index"] for e in meta["passes"] if e["scenario"] == "substep" and e["kernel"] == "gridClear")
    grid_state = state_before(z, meta, "substep", grid_at)
    report = {}
    for e in _passes(meta, "substep"):
        st = state_before(z, meta, "substep", e["index"])
        o2 = load_o2(scene, C, st, grid_state)
        _run(o2, e, e["uniform"]["h"])
        got, want = _read_o2(o2, C), _want(after(z, "substep", e["index"], st), C)
        kind = KERNELS[e["kernel"]][2]
        what = f"substep pass {e['index']} {e['kernel']}"
        if kind == "cache":
            # per solid: the same neighbours (the order follows bucket membership)
            assert np.array_equal(got["ccount"], want["ccount"]), f"{what}: counts"
            gl, wl = got["clist"].reshape(-1, 40), want["clist"].reshape(-1, 40)
            for i, n in enumerate(want["ccount"]):
                if n < 40:
                    assert sorted(gl[i, :n]) == sorted(wl[i, :n]), f"{what}: solid {i}"
            kind = "exact"
        report[f"{e['index']} {e['kernel']}"] = _compare(kind, e["kernel"], got, want, what)
    print(report)


@pytest.mark.parametrize("scenario", ["bonds", "bounds"])
def test_rule_passes_match_reference_wgsl(golden, scene, scenario):
    """Bond and tet updates on a stretched state (plasticity, clamping,
    tearing of bonds and tets: src/gpu/wgsl.js:383-404, 472-491), and
    applyDeltaAll / bounds / velocityUpdate with particles under the floor,
    in the walls and past the cull radius (src/gpu/wgsl.js:648-710)."""
    z, meta = golden
    C = meta["C"]
    for e in _passes(meta, scenario):
        st = state_before(z, meta, scenario, e["index"])
        o2 = load_o2(scene, C, st)
        _run(o2, e, e["uniform"]["h"])
        got, want = _read_o2(o2, C), _want(after(z, scenario, e["index"], st), C)
        _compare("exact", e["kernel"], got, want, f"{scenario} pass {e['index']} {e['kernel']}")
    changed = {b for e in meta["passes"] if e["scenario"] == scenario for b in e["changed"]}
    assert changed, f"{scenario}: the reference's passes changed nothing"


def test_grab_passes_match_reference_wgsl(golden, scene):
    """grabSelect (src/gpu/wgsl.js:843-866), three integrates with a grab
    motion (the spring, its 5 cm cap and the 1 m slip, src/gpu/wgsl.js:
    121-160), grabRelease (src/gpu/wgsl.js:868-871): bit for bit."""
    z, meta = golden
    C = meta["C"]
    es = [e for e in meta["passes"] if e["scenario"] == "grab"]
    assert [e["kernel"] for e in es] == ["grabSelect", "integrate", "integrate", "integrate", "grabRelease"]
    for e in es:
        st = state_before(z, meta, "grab", e["index"])
        o2 = load_o2(scene, C, st)
        u = e["uniform"]
        if e["kernel"] == "grabSelect":
            o2.grab_select(u["grabC"][:3], u["grabC"][3], int(u["grabLattice"]))
        elif e["kernel"] == "grabRelease":
            o2.release()
        else:
            _run(o2, e, u["h"])
        got, want = _read_o2(o2, C), _want(after(z, "grab", e["index"], st), C)
        _compare("exact", e["kernel"], got, want, f"grab pass {e['index']} {e['kernel']}")
    sel = after(z, "grab", 0, state_before(z, meta, "grab", 0))
    assert int((sel["flags"][:C["SOLID_N"]] & L.F_GRABBED).sum()) > 0, "the grab selected nothing"
    assert "flags" in es[3]["changed"], "the last pull slipped no grip"


def test_emit_matches_reference_wgsl(golden, scene):
    """The hose emit kernel (src/gpu/wgsl.js:781-801): ring-buffer slots,
    golden-angle disc, sine-hash jitter."""
    z, meta = golden
    C = meta["C"]
    e = next(e for e in meta["passes"] if e["scenario"] == "emit")
    st = state_before(z, meta, "emit", e["index"])
    o2 = load_o2(scene, C, st)
    u = e["uniform"]
    assert int(o2.info.fluid_next) == int(u["emitStart"])
    o2.emit(int(u["emitCount"]), u["emitPos"][:3], u["emitDir"][:3], u["emitSide"][:3], u["emitUp"][:3],
            u["emitPos"][3], u["emitDir"][3])
    o2.run_pass_x("EMIT", u["h"])
    got, want = _read_o2(o2, C), _want(after(z, "emit", e["index"], st), C)
    S_, F = C["SOLID_N"], C["MAX_FLUID"]
    slots = S_ + (int(u["emitStart"]) + np.arange(int(u["emitCount"]))) % F
    other = np.setdiff1d(np.arange(C["TOTAL"]), slots)
    for k in ("pos", "prev", "vel", "density", "flags"):
        assert_exact(got[k][other], want[k][other], f"emit: untouched {k}")
    assert_close(got["pos"][slots, :3], want["pos"][slots, :3], 1.0, 1e-4, "emit: positions (m)")
    assert_close(got["prev"][slots, :3], want["prev"][slots, :3], 1.0, 1e-4, "emit: previous positions (m)")
    assert_close(got["vel"][slots, :3], want["vel"][slots, :3], 1.0, 2e-2, "emit: velocities (m/s)")
    assert_exact(got["pos"][slots, 3], want["pos"][slots, 3], "emit: inverse masses")


def test_tools_match_reference_wgsl(golden, scene):
    """cut + cutTets (src/gpu/wgsl.js:494-519, 804-823), pick
    (src/gpu/wgsl.js:826-840) and countActive (src/gpu/wgsl.js:874-879). The
    oracle cuts and picks in the CPU solver's double precision
    (src/solver.js:458-515) where the reference's kernels use f32: the same
    constraints and tets die, and each pick finds the reference's particle
    or one within the millimetre its packed result resolves."""
    z, meta = golden
    C = meta["C"]
    T, N, S_ = C["TABLE"], C["TOTAL"], C["SOLID_N"]
    es = {e["label"]: e for e in meta["passes"] if e["scenario"] == "tools"}
    st = state_before(z, meta, "tools", es["cut"]["index"])
    o2 = load_o2(scene, C, st)
    u = es["cut"]["uniform"]
    n = o2.slice_now(u["cutO"][:3], u["cutD1"][:3], u["cutD2"][:3])
    got = _read_o2(o2, C)
    want = _want(after(z, "tools", es["cutTets"]["index"],
                       after(z, "tools", es["cut"]["index"], st)), C)
    assert np.array_equal(got["cons"], want["cons"]), "cut: alive flags"
    assert np.array_equal(got["tets"], want["tets"]), "cutTets: tets"
    assert n == int((st["cons"][:, 3] != 0).sum() - (want["cons"][:, 3] != 0).sum()) and n > 0
    s_pick = 2 * T + N
    for k in range(5):
        e = es[f"pick {k}"]
        u = e["uniform"]
        packed = int(z[f"tools/{e['index']}/gridA"][s_pick])
        o2 = load_o2(scene, C, state_before(z, meta, "tools", e["index"]))
        i, t = o2.pick(u["pickO"][:3], u["pickD"][:3], u["pickO"][3])
        if packed == 0xFFFFFFFF:
            assert i < 0, f"pick {k}: the reference found nothing"
            continue
        mm, idx = packed >> 16, packed & 0xFFFF
        assert i == idx or abs(t * 1000.0 - mm) <= 1.0, f"pick {k}: oracle {i} at {t} vs reference {idx} at {mm} mm"
    e = es["countActive"]
    cnt = int(z[f"tools/{e['index']}/gridA"][s_pick + 1])
    o2 = load_o2(scene, C, state_before(z, meta, "tools", e["index"]))
    assert o2.active_count() == cnt


def test_whole_substep_matches_reference_schedule(golden, scene):
    """The oracle's own substep (its pass order and iteration count) from the
    reference's start state, against the end of the reference's chain of
    kernels in GpuSim.encode's order: the schedule, not only the passes.
    Summation orders differ along the way: positions agree to 2e-7 m and
    velocities to 5e-5 m/s (measured: 3e-8 m and 9e-6 m/s, 1,010 of 1,043
    positions bit for bit), every flag, constraint and tet exactly."""
    z, meta = golden
    C = meta["C"]
    es = [e for e in meta["passes"] if e["scenario"] == "substep"]
    st = state_before(z, meta, "substep", 0)
    end = state_before(z, meta, "substep", es[-1]["index"] + 1)
    o2 = load_o2(scene, C, st)
    o2.substep_partial(es[0]["uniform"]["h"], 1000)
    got, want = _read_o2(o2, C), _want(end, C)
    act = (want["flags"] & 1).astype(bool)
    assert np.array_equal(got["flags"], want["flags"])
    assert np.array_equal(got["cons"], want["cons"])
    assert np.array_equal(got["tets"], want["tets"])
    assert_close(got["pos"][act, :3], want["pos"][act, :3], 1.0, 2e-7, "substep positions (m)")
    assert_close(got["vel"][act, :3], want["vel"][act, :3], 1.0, 5e-5, "substep velocities (m/s)")


def test_whole_frame_matches_reference_encode(golden, scene):
    """One whole frame as GpuSim.encode runs it (src/gpu/sim.js:333-392): a
    32-particle emit, five substeps, the queued wedge cut (cut + cutTets) and
    the active count, against the oracle's frame with the same emit and a
    queued slice. Five substeps of different summation orders: positions
    within 1e-6 m, velocities within 1e-4 m/s (measured 1.2e-7 m, 7.6e-6 m/s;
    the emitted particles, whose sine-hash jitter differs in its last bits,
    within 1e-4 m and 5e-3 m/s), every flag, constraint and tet exactly."""
    z, meta = golden
    C = meta["C"]
    e = next(e for e in meta["passes"] if e["scenario"] == "frame")
    st = {k.split("/")[-1]: v for k, v in z.items() if k.startswith("frame/start/")}
    end = {k.split("/")[-1]: v for k, v in z.items() if k.startswith("frame/end/")}
    o2 = load_o2(scene, C, st)
    u = e["uniform"]
    o2.emit(int(u["emitCount"]), u["emitPos"][:3], u["emitDir"][:3], u["emitSide"][:3], u["emitUp"][:3],
            u["emitPos"][3], u["emitDir"][3])
    o2.slice(*e["wedge"])
    o2.step(scene.dt, scene.substeps)
    got, want = _read_o2(o2, C), _want(end, C)
    assert np.array_equal(got["flags"], want["flags"])
    assert np.array_equal(got["cons"], want["cons"])
    assert np.array_equal(got["tets"], want["tets"])
    act = (want["flags"] & 1).astype(bool)
    S_, F = C["SOLID_N"], C["MAX_FLUID"]
    emitted = np.zeros(C["TOTAL"], bool)
    emitted[S_ + (int(u["emitStart"]) + np.arange(int(u["emitCount"]))) % F] = True
    rest = act & ~emitted
    assert_close(got["pos"][rest, :3], want["pos"][rest, :3], 1.0, 1e-6, "frame positions (m)")
    assert_close(got["vel"][rest, :3], want["vel"][rest, :3], 1.0, 1e-4, "frame velocities (m/s)")
    assert_close(got["pos"][emitted, :3], want["pos"][emitted, :3], 1.0, 1e-4, "emitted positions (m)")
    assert_close(got["vel"][emitted, :3], want["vel"][emitted, :3], 1.0, 5e-3, "emitted velocities (m/s)")
    assert o2.active_count() == int(end["gridA"][2 * C["TABLE"] + C["TOTAL"] + 1])
