"""Generate the golden vectors in tests/golden/ from the reference itself.

The reference ships no unit tests, fixtures or known-answer vectors, and no
JavaScript engine exists on this machine, so its files are executed
unmodified by tests/golden/jsmini.py:
  - src/solver.js (class Solver): frames and substeps of the CPU solver,
    its hash grid, wedge cut, union-find groups, pick and grab pull;
  - src/gpu/sim.js (GpuSim.prototype._buildHostData): the lattice,
    constraint, CSR adjacency and tet data the GPU solver uploads.
Inputs are seeded (numpy PCG64, the same generators the scenes use); one
input state is produced by the C++ restatement O1 (30 frames of settling) so
that contacts, plasticity and the pair cap are exercised — its output is
still produced by the reference code.

Run from the repository root, naming the reference checkout (its directory
holding src/solver.js) with --ref or the UPBD_REFERENCE environment variable:
    python tests/golden/make_golden.py --ref <path to the reference>
Writes tests/golden/solver_js.json (digests and small arrays) and
tests/golden/solver_js_c1.npz (full C1 arrays).
"""
from __future__ import annotations

import hashlib
import json
import math
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(ROOT))

import jsmini as J  # noqa: E402



def _reference_dir() -> Path:
    import os
    args = sys.argv[1:]
    if "--ref" in args and args.index("--ref") + 1 < len(args):
        ref = args[args.index("--ref") + 1]
    else:
        ref = os.environ.get("UPBD_REFERENCE", "")
    if not ref:
        raise SystemExit("name the reference checkout: --ref <dir> or UPBD_REFERENCE=<dir>")
    d = Path(ref)
    if not (d / "src" / "solver.js").exists():
        raise SystemExit(f"{d} does not hold src/solver.js")
    return d


REF = _reference_dir() if __name__ == "__main__" else Path(".")


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def solver_class():
    mod = J.run_source((REF / "src/solver.js").read_text())
    return mod.lookup("Solver")


def js_get(o, name):
    v = J.get_member(o, name)
    if isinstance(v, J.TypedArray):
        return J.typed_to_numpy(v)
    if isinstance(v, J.JSArray):
        return np.array([J.to_number(x) for x in v.items], dtype=np.float64)
    return v


def js_state(s) -> dict:
    out = {k: js_get(s, k) for k in ("pos", "prev", "vel", "active", "group", "cellStart", "cellEntries",
                                     "rho", "rhoNear")}
    out["consRest"] = js_get(s, "consRest")
    out["consAlive"] = js_get(s, "consAlive").astype(np.uint8)
    out["pairCount"] = float(J.get_member(s, "pairCount"))
    out["fluidNext"] = float(J.get_member(s, "fluidNext"))
    return out


def new_c1_solver(Solver, fluid):
    s = J.new(Solver, {"maxFluid": 2600})
    J.set_member(s, "gravity", -9.8)
    J.method(s, "addSolidCube", 0, 2.0, 0, 7, 0.18)
    for p in fluid:
        J.method(s, "emitFluid", float(p[0]), float(p[1]), float(p[2]), 0.0, 0.0, 0.0)
    return s


def load_state(s, st):
    for k in ("pos", "prev", "vel"):
        J.numpy_into_typed(J.get_member(s, k), st[k].astype(np.float32))
    J.numpy_into_typed(J.get_member(s, "active"), st["active"].astype(np.uint8))
    rest = J.get_member(s, "consRest")
    rest.items = [float(x) for x in st["consRest"]]
    alive = J.get_member(s, "consAlive")
    alive.items = [float(x) for x in st["consAlive"]]
    ps = J.get_member(s, "pairSet")
    ps.s.clear()
    a = js_get(s, "consA")
    b = js_get(s, "consB")
    cap = J.get_member(s, "capacity")
    for c in range(len(a)):
        if st["consAlive"][c]:
            ps.s.add(int(a[c] * cap + b[c]))
    J.set_member(s, "fluidNext", float(st["fluidNext"]))


def main():
    from fluidphysics_b200 import scenes as S
    from oracle.oracle import O1

    t0 = time.time()
    Solver = solver_class()
    out = {"generator": "tests/golden/make_golden.py (reference files run by tests/golden/jsmini.py)",
           "reference_files": ["src/solver.js", "src/gpu/sim.js"], "cases": {}}
    npz = {}

    # ---- C1: one frame of the CPU solver's own scene from a seeded block
    c1 = S.cpu_scene()
    fluid = c1.fluid_pos.astype(np.float64)
    s = new_c1_solver(Solver, fluid)
    J.method(s, "_buildGrid")
    g0 = js_state(s)
    case = {"desc": "C1 initial grid: Solver({maxFluid:2600}), gravity -9.8, addSolidCube(0,2,0,7,0.18), "
                    "2600 fluid from jittered_block(20,10,13,0.165,2.8,seed=1); _buildGrid()",
            "digest": {k: digest(g0[k]) for k in ("cellStart", "cellEntries")}}
    out["cases"]["c1_grid0"] = case
    J.method(s, "step", 1 / 60, 5)
    st = js_state(s)
    out["cases"]["c1_frame1"] = {
        "desc": "C1 after step(1/60, 5) from the initial state",
        "digest": {k: digest(st[k]) for k in ("pos", "prev", "vel", "active", "group", "cellStart",
                                              "cellEntries", "rho", "rhoNear", "consRest", "consAlive")},
        "pairCount": st["pairCount"]}
    for k in ("pos", "vel", "active", "rho"):
        npz[f"c1_frame1_{k}"] = st[k]
    print(f"c1_frame1 done {time.time() - t0:.0f}s", flush=True)

    # ---- C1 settled: O1 state after 30 frames, then one substep by the reference
    o1 = O1(2600, gravity=-9.8)
    o1.add_solid_cube(0, 2.0, 0, 7, 0.18, 0.08)
    o1.emit_fluid(fluid, np.zeros_like(fluid), 0.03)
    for _ in range(30):
        o1.step(1 / 60, 5)
    st_in = {k: o1.get(k) for k in ("pos", "prev", "vel", "active", "consRest", "consAlive")}
    st_in["fluidNext"] = o1.sizes()["fluidNext"]
    for k, v in st_in.items():
        if k != "fluidNext":
            npz[f"c1_settled_in_{k}"] = v
    s2 = new_c1_solver(Solver, fluid)
    load_state(s2, st_in)
    J.method(s2, "step", 1 / 300, 1)
    st2 = js_state(s2)
    out["cases"]["c1_settled_substep"] = {
        "desc": "C1: the O1 state after 30 frames (arrays c1_settled_in_*), then step(1/300, 1)",
        "digest": {k: digest(st2[k]) for k in ("pos", "prev", "vel", "active", "group", "cellStart",
                                               "cellEntries", "rho", "rhoNear", "consRest", "consAlive")},
        "pairCount": st2["pairCount"]}
    for k in ("pos", "vel"):
        npz[f"c1_settled_out_{k}"] = st2[k]
    print(f"c1_settled done {time.time() - t0:.0f}s", flush=True)

    # ---- tools on the settled output: pick rays, wedge cuts, groups
    rng = np.random.default_rng(21)
    picks = []
    p = st2["pos"].reshape(-1, 3)[:343].astype(np.float64)
    cen = p.mean(0)
    for _ in range(24):
        ro = cen + rng.normal(size=3) * 3
        rd = cen + rng.normal(size=3) * 0.3 - ro
        rd /= np.linalg.norm(rd)
        r = J.method(s2, "pickSolid", *ro, *rd, 0.2)
        picks.append({"o": ro.tolist(), "d": rd.tolist(), "maxPerp": 0.2,
                      "id": None if r is None else int(J.get_member(r, "id")),
                      "t": None if r is None else J.get_member(r, "t")})
    cuts = []
    for k in range(3):
        o, d1, d2 = S.wedge_through(cen + rng.normal(size=3) * 0.05, 100 + k)
        n = J.method(s2, "cut", *o, *d1, *d2)
        cuts.append({"o": o.tolist(), "d1": d1.tolist(), "d2": d2.tolist(), "count": int(n),
                     "alive": digest(js_get(s2, "consAlive").astype(np.uint8))})
    J.method(s2, "_recomputeGroups")
    grp = js_get(s2, "group")[:343]
    out["cases"]["c1_tools"] = {"desc": "pickSolid rays, three wedge cuts and _recomputeGroups on the "
                                        "c1_settled_substep output", "picks": picks, "cuts": cuts,
                                "group": grp.astype(int).tolist()}
    print(f"c1_tools done {time.time() - t0:.0f}s", flush=True)

    # ---- grab pull: 30 body particles with offset targets, one substep
    s3 = new_c1_solver(Solver, fluid)
    load_state(s3, st_in)
    top = np.argsort(-st_in["pos"].reshape(-1, 3)[:343, 1], kind="stable")[:30]
    grabs = []
    for i in sorted(top.tolist()):
        q = st_in["pos"].reshape(-1, 3)[i].astype(np.float64)
        grabs.append({"i": float(i), "x": float(q[0] + 0.1), "y": float(q[1] + 0.3), "z": float(q[2])})
    J.get_member(s3, "grabs").items = [J.py_to_js(g) for g in grabs]
    J.method(s3, "step", 1 / 300, 1)
    st3 = js_state(s3)
    out["cases"]["c1_grab_substep"] = {
        "desc": "c1_settled input, grabs (the 30 highest body particles pulled to +0.1x +0.3y), step(1/300, 1)",
        "grabs": grabs, "digest": {k: digest(st3[k]) for k in ("pos", "prev", "vel")}}
    print(f"c1_grab done {time.time() - t0:.0f}s", flush=True)

    # ---- C2-size grid and cut (the GPU default scene's body and fluid)
    c2 = S.gpu_default(frames=1)
    s4 = J.new(Solver, {"maxFluid": 65536})
    d = c2.desc
    J.method(s4, "addSolidCube", d.cube_center[0], d.cube_center[1], d.cube_center[2], d.solid_dim, d.spacing,
             d.solid_mass)
    J.set_member(s4, "cellSize", c2.params.cell_size)
    for q in c2.fluid_pos.astype(np.float64):
        J.method(s4, "emitFluid", float(q[0]), float(q[1]), float(q[2]), 0.0, 0.0, 0.0, c2.fluid_mass)
    J.method(s4, "_buildGrid")
    o, d1, d2 = c2.wedge
    n = J.method(s4, "cut", *o, *d1, *d2)
    out["cases"]["c2_grid_cut"] = {
        "desc": "GPU default scene (20^3 body, 65,536 fluid) in Solver with cellSize = H: _buildGrid, then the "
                "scene's wedge cut", "cellSize": c2.params.cell_size,
        "tableSize": J.get_member(s4, "tableSize"),
        "digest": {"cellStart": digest(js_get(s4, "cellStart")), "cellEntries": digest(js_get(s4, "cellEntries")),
                   "consAlive": digest(js_get(s4, "consAlive").astype(np.uint8)),
                   "pos": digest(js_get(s4, "pos"))},
        "cut_count": int(n)}
    print(f"c2 done {time.time() - t0:.0f}s", flush=True)

    # ---- GpuSim._buildHostData (lattices, constraints, CSR, tets)
    mod = J.run_source((REF / "src/gpu/sim.js").read_text())
    GpuSim = mod.lookup("GpuSim")
    builds = {}
    for name, dim, dim2, maxf in (("small", 6, None, 64), ("default", 20, None, 65536)):
        o = J.JSObject(proto=GpuSim.proto)
        opts = {"SOLID_DIM": float(dim), "MAX_FLUID": float(maxf), "spacing": 0.065, "solidMass": 0.004,
                "fluidMass": 0.0015, "cubeCenter": [0.0, 1.8, 0.0]}
        # SOLID_DIM2 ?? Math.max(2, Math.round((SOLID_DIM - 1) / Math.cbrt(20)) + 1), src/gpu/sim.js:83
        d2_ = max(2, int(math.floor((dim - 1) / 20 ** (1 / 3) + 0.5)) + 1) if dim2 is None else dim2
        J.set_member(o, "o", J.py_to_js(opts))
        J.set_member(o, "DIM2", float(d2_))
        J.set_member(o, "N1", float(dim ** 3))
        J.set_member(o, "SOLID_N", float(dim ** 3 + d2_ ** 3))
        J.set_member(o, "TOTAL", float(dim ** 3 + d2_ ** 3 + maxf))
        J.method(o, "_buildHostData")
        init = J.get_member(o, "init")
        tets = J.get_member(o, "initTets")
        arr = {"pos": js_get(init, "pos"), "flags": js_get(init, "flags"), "cons": js_get(init, "cons"),
               "adj": js_get(init, "adj"), "tetData": js_get(tets, "tetData"), "tetAdj": js_get(tets, "tetAdj")}
        builds[name] = {"opts": opts, "dim2": int(d2_), "num_cons": int(J.get_member(o, "NUM_CONS")),
                        "num_tets": int(J.get_member(o, "NUM_TETS")),
                        "digest": {k: digest(v) for k, v in arr.items()}}
        if name == "small":
            for k, v in arr.items():
                npz[f"build_small_{k}"] = v
        print(f"build {name} done {time.time() - t0:.0f}s", flush=True)
    out["cases"]["gpu_build"] = builds

    (HERE / "solver_js.json").write_text(json.dumps(out, indent=1))
    np.savez_compressed(HERE / "solver_js_c1.npz", **npz)
    print(f"wrote golden vectors in {time.time() - t0:.0f}s")


if __name__ == "__main__":
    main()
