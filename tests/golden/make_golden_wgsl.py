"""Golden vectors of the reference's WGSL kernels, executed pass by pass.

The reference's GPU solver is WGSL (src/gpu/wgsl.js); no WebGPU runtime
exists on this machine. This script evaluates the unmodified
makeShaderSource of src/gpu/wgsl.js with tests/golden/jsmini.py, with the
constants GpuSim._buildGpu passes it (src/gpu/sim.js:243-249), and runs the
resulting WGSL module with tests/golden/wgslmini.py, on buffers laid out as
GpuSim._buildGpu lays them out (src/gpu/sim.js:215-236) and a uniform block
filled as GpuSim._writeParams fills it (src/gpu/sim.js:300-330).

Scenarios, on a small scene with every optional pass of the reference's GPU
schedule (6^3 body + 3^3 companion cube, 800 fluid, tets, the solid contact
cache, solid viscosity), first stepped 40 frames by the oracle (a slice at
frame 4) so that fluid, bodies, the floor and the cut faces are in contact:

  substep  one whole substep in GpuSim.encode's pass order
           (src/gpu/sim.js:352-385), the hash grid built by gridClear,
           gridCount and gridScatter (its prefix scan, the one kernel group
           that synchronizes workgroups, computed directly);
  bonds    bondUpdate and tetUpdate on a stretched copy of the state (some
           bonds past the plastic threshold, some bonds and tets past the
           tear gap);
  bounds   applyDeltaAll, bounds and velocityUpdate on a copy with particles
           moved under the floor, into the walls and past the cull radius;
  grab     grabSelect, three integrates with grab motions (the spring, its
           cap, the slip), grabRelease;
  emit     the hose emit kernel (96 particles);
  tools    cut + cutTets with a wedge through the body, pick on five rays,
           countActive;
  frame    one whole frame: a 32-particle emit, five substeps, a queued cut
           and the active count (only the end state is kept).

For every pass the file keeps the buffers the pass changed, so a test can
rebuild the state before each pass and compare the oracle's pass on it.

Usage (from the repository root):
    python tests/golden/make_golden_wgsl.py --ref <reference checkout>
Writes tests/golden/wgsl_passes.npz.
"""
from __future__ import annotations

import json
import math
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(ROOT))

import jsmini as J  # noqa: E402
import wgslmini as W  # noqa: E402
from fluidphysics_b200 import scenes as S  # noqa: E402
from oracle.oracle import o2_from_scene  # noqa: E402

OUT = HERE / "wgsl_passes.npz"
MUTABLE = ("pos", "prev", "vel", "flags", "delta", "density", "cons", "gridA", "gridS")


def reference_dir() -> Path:
    args = sys.argv[1:]
    ref = args[args.index("--ref") + 1] if "--ref" in args else os.environ.get("UPBD_REFERENCE", "")
    if not ref:
        raise SystemExit("name the reference checkout: --ref <dir> or UPBD_REFERENCE=<dir>")
    d = Path(ref)
    if not (d / "src" / "gpu" / "wgsl.js").exists():
        raise SystemExit(f"{d} does not hold src/gpu/wgsl.js")
    return d


def golden_scene() -> S.Scene:
    """The scene all scenarios start from (also rebuilt by the test)."""
    d, p, opts = S.gpu_scene(6, 800, 40, iters=2, features=3)
    d.solid_dim2 = 3
    d.cube2_center[:] = [0.22, d.cube_center[1] + 3.2 * d.spacing, 0.05]
    d.table_size = 4096
    S.set_params(p, dict(solid_viscosity=0.3))
    fp = S.jittered_block(10, 8, 10, 2.2 * 0.04, d.cube_center[1] - 0.1, 11)
    return S.Scene("wgsl_pin", d, p, fp, np.zeros_like(fp), opts["fluidMass"], 1 / 60, 5, 40,
                   slice_frame=4, wedge=S.wedge_through(d.cube_center, 11))


def settled(sc: S.Scene):
    o2 = o2_from_scene(sc)
    for f in range(sc.frames):
        if f == sc.slice_frame:
            o2.slice_now(*sc.wedge)
        o2.step(sc.dt, sc.substeps)
    return o2


def shader(ref: Path, o2) -> str:
    """makeShaderSource(C) of src/gpu/wgsl.js, with GpuSim._buildGpu's C."""
    mod = J.run_source((ref / "src" / "gpu" / "wgsl.js").read_text())
    info = o2.info
    T = int(info.table_size)
    C = {"SOLID_N": int(info.solid_n), "SOLID_DIM": int(info.dim1), "N1": int(info.n1),
         "SOLID_DIM2": int(info.dim2), "MAX_FLUID": int(info.max_fluid), "TOTAL": int(info.total),
         "TABLE": T, "NUM_CONS": int(info.num_cons), "SCAN_BLOCKS": T // 256,
         "NUM_TETS": int(info.num_tets), "TS_TETS": T + 1 + T // 256}
    return J.call(mod.vars["makeShaderSource"], J.UNDEF, [J.py_to_js(C)]), C


def buffers(o2, C: dict) -> dict:
    """GpuSim's storage buffers (src/gpu/sim.js:222-233) from the oracle's state."""
    st = o2.read_state()
    N, S_, T, NT = C["TOTAL"], C["SOLID_N"], C["TABLE"], C["NUM_TETS"]
    gridS = np.zeros(T + 1 + T // 256 + NT * 5 + S_ + 1 + NT * 4, np.uint32)
    ts = C["TS_TETS"]
    gridS[ts:ts + NT * 5] = o2.read_tets().reshape(-1)
    gridS[ts + NT * 5:] = o2.read_tet_adjacency()
    gridA = np.zeros(T * 2 + N + 8 + S_ * 41, np.uint32)
    cc, cl = o2.read_contact_cache()
    c_count = 2 * T + N + 8
    gridA[c_count:c_count + S_] = cc
    gridA[c_count + S_:c_count + S_ + S_ * 40] = cl
    return {
        "pos": st["pos"].astype(np.float32), "prev": st["prev"].astype(np.float32),
        "vel": st["vel"].astype(np.float32), "flags": st["flags"].astype(np.uint32),
        "delta": o2.read_delta().astype(np.float32), "density": st["density"].astype(np.float32),
        "cons": o2.read_constraints()[0].astype(np.uint32), "adj": o2.read_adjacency().astype(np.uint32),
        "gridA": gridA, "gridS": gridS,
    }


def uniforms(sc: S.Scene, **pend) -> dict:
    """The Params block as GpuSim._writeParams writes it (src/gpu/sim.js:300-330)."""
    p, d = sc.params, sc.desc
    g = lambda k: float(getattr(p, k))  # noqa: E731
    u = {"h": sc.dt / sc.substeps, "gravity": g("gravity"), "solidRadius": g("solid_radius"),
         "fluidRadius": g("fluid_radius"), "cellSize": g("cell_size"), "fluidH": g("fluid_h"),
         "restDensity": g("rest_density"), "stiffness": g("stiffness"), "nearStiffness": g("near_stiffness"),
         "viscosity": g("viscosity"), "compliance": g("compliance"), "omega": g("omega"),
         "plasticThreshold": g("plastic_threshold"), "plasticRate": g("plastic_rate"), "tearGap": g("tear_gap"),
         "maxSpeed": g("max_speed"), "wallX": g("wall_x"), "wallZ": g("wall_z"), "wallH": g("wall_h"),
         "wallT": g("wall_t"), "cullR": g("cull_r"), "dampSolid": g("damp_solid"), "dampFluid": g("damp_fluid"),
         "frictionSolid": g("friction_solid"), "frictionFluid": g("friction_fluid"), "grabK": g("grab_k"),
         "sleepSpeed": g("sleep_speed"), "spacing": float(d.spacing),
         "emitCount": 0, "emitStart": 0, "solidViscosity": g("solid_viscosity"), "grabLattice": 0xffff,
         "emitPos": [0, 0, 0, 0], "emitDir": [0, 0, 0, 0], "emitSide": [0, 0, 0, 0], "emitUp": [0, 0, 0, 0],
         "grabDelta": [0, 0, 0, 0], "cutO": [0, 0, 0, 0], "cutD1": [0, 0, 0, 0], "cutD2": [0, 0, 0, 0],
         "pickO": [0, 0, 0, 0.25], "pickD": [0, 0, 1, 0], "grabC": [0, 0, 0, 0]}
    u.update(pend)
    return u


class Recorder:
    """Runs WGSL passes on one set of buffers and keeps, per pass, the
    buffers it changed."""

    def __init__(self, mod: W.Module, bufs: dict, tag: str, out: dict, meta: list):
        self.m, self.b, self.tag, self.out, self.meta = mod, bufs, tag, out, meta
        for k, v in bufs.items():
            mod.bind(k, v)
        for k in MUTABLE:
            out[f"{tag}/start/{k}"] = bufs[k].copy()

    def run(self, kernel: str, n_invocations: int, uniform: dict, wg_size: int = 256, label: str | None = None):
        self.m.set_uniform("P", uniform)
        before = {k: self.b[k].copy() for k in MUTABLE}
        t = time.time()
        self.m.dispatch(kernel, max(1, math.ceil(n_invocations / wg_size)))
        k = sum(1 for e in self.meta if e["scenario"] == self.tag)
        name = label or kernel
        changed = [b for b in MUTABLE if not np.array_equal(before[b], self.b[b])]
        for b in changed:
            self.out[f"{self.tag}/{k}/{b}"] = self.b[b].copy()
        self.meta.append({"scenario": self.tag, "index": k, "kernel": kernel, "label": name,
                          "changed": changed, "uniform": {u: (list(map(float, v)) if isinstance(v, list) else float(v))
                                                          for u, v in uniform.items()}})
        print(f"  {self.tag}/{k} {name}: {time.time() - t:.1f} s, changed {changed}", flush=True)

    def grid(self, C: dict, uniform: dict):
        """gridClear, gridCount, the exclusive scan of the counts, gridScatter
        (src/gpu/wgsl.js:163-245)."""
        T = C["TABLE"]
        self.run("gridClear", T, uniform)
        self.run("gridCount", C["TOTAL"], uniform)
        counts = self.b["gridA"][:T].astype(np.uint64)
        scan = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.uint32)
        before = self.b["gridS"].copy()
        self.b["gridS"][:T] = scan
        self.b["gridS"][T] = 0  # scanApply leaves gridS[TABLE] = 0 (src/gpu/wgsl.js:230-236)
        k = sum(1 for e in self.meta if e["scenario"] == self.tag)
        self.out[f"{self.tag}/{k}/gridS"] = self.b["gridS"].copy()
        self.meta.append({"scenario": self.tag, "index": k, "kernel": "scan", "label": "scan (exclusive prefix sum)",
                          "changed": ["gridS"] if not np.array_equal(before, self.b["gridS"]) else [],
                          "uniform": {}})
        self.run("gridScatter", C["TOTAL"], uniform)


def substep(r, C: dict, u: dict, iters: int) -> None:
    """One substep in GpuSim.encode's pass order (src/gpu/sim.js:352-385)."""
    S_, F, N = C["SOLID_N"], C["MAX_FLUID"], C["TOTAL"]
    r.run("integrate", N, u)
    r.grid(C, u)
    for k in ("fluidDensity", "fluidDisp", "applyDeltaFluid"):
        r.run(k, F, u)
    r.run("collectContacts", S_, u)
    for it in range(iters):
        r.run("solidSolve", S_, u)
        r.run("applyDeltaSolid", S_, u)
        r.run("solveTets", S_, u)
        r.run("applySolidContacts", S_, u)
        r.run("solidContacts", S_, u)
        r.run("applySolidContacts", S_, u)
    r.run("bondUpdate", C["NUM_CONS"], u)
    r.run("tetUpdate", C["NUM_TETS"], u)
    for k in ("contacts", "applyDeltaAll", "bounds", "velocityUpdate"):
        r.run(k, N, u)
    if u["solidViscosity"] > 0:
        r.run("solidVisc", S_, u)
        r.run("solidViscApply", S_, u)
    r.run("xsph", F, u)
    r.run("xsphApply", F, u)


class Runner(Recorder):
    """Runs passes without recording them (whole frames: only the end state
    is kept)."""

    def __init__(self, mod: W.Module, bufs: dict):
        self.m, self.b = mod, bufs
        for k, v in bufs.items():
            mod.bind(k, v)
        self.meta, self.tag, self.out = [], "", {}

    def run(self, kernel: str, n_invocations: int, uniform: dict, wg_size: int = 256, label: str | None = None):
        self.m.set_uniform("P", uniform)
        self.m.dispatch(kernel, max(1, math.ceil(n_invocations / wg_size)))


def main():
    ref = reference_dir()
    sc = golden_scene()
    o2 = settled(sc)
    src, C = shader(ref, o2)
    out, meta = {}, []
    S_, F, N = C["SOLID_N"], C["MAX_FLUID"], C["TOTAL"]
    NC, NT = C["NUM_CONS"], C["NUM_TETS"]
    iters = int(sc.desc.solid_iters)
    base = uniforms(sc)

    # ---- one whole substep (GpuSim.encode, src/gpu/sim.js:352-385)
    print("substep", flush=True)
    m = W.Module(src)
    r = Recorder(m, buffers(o2, C), "substep", out, meta)
    substep(r, C, base, iters)

    # ---- bond and tet rules on a stretched state
    print("bonds", flush=True)
    b = buffers(o2, C)
    rng = np.random.default_rng(12)
    hs = float(sc.desc.spacing)
    kick = rng.uniform(-0.6, 0.6, size=(S_, 3)).astype(np.float32) * np.float32(hs)
    kick[rng.random(S_) < 0.85] *= np.float32(0.25)
    kick[rng.random(S_) < 0.05] *= np.float32(3.0)
    b["pos"][:S_, :3] += kick
    m = W.Module(src)
    r = Recorder(m, b, "bonds", out, meta)
    r.run("bondUpdate", NC, base)
    r.run("tetUpdate", NT, base)

    # ---- floor, walls and cull
    print("bounds", flush=True)
    b = buffers(o2, C)
    wx, wz, cr = float(sc.params.wall_x), float(sc.params.wall_z), float(sc.params.cull_r)
    fl = np.arange(S_, N)[b["flags"][S_:] & 1 == 1]
    pick_f = rng.choice(fl, size=min(60, len(fl)), replace=False)
    b["pos"][pick_f[:15], 1] = np.float32(-0.01)                       # under the floor
    b["pos"][pick_f[15:30], 0] = np.float32(wx) + rng.uniform(-0.03, 0.03, 15).astype(np.float32)  # in the x walls
    b["pos"][pick_f[30:45], 2] = -np.float32(wz) + rng.uniform(-0.03, 0.03, 15).astype(np.float32)  # z walls
    b["pos"][pick_f[45:55], 0] = np.float32(cr + 0.5)                   # past the cull radius
    b["pos"][pick_f[55:], 1] = np.float32(-3.5)                         # fallen out
    b["pos"][:2, 1] = np.float32(-0.02)                                 # solids under the floor
    b["delta"][:, :3] = rng.normal(scale=0.004, size=(N, 3)).astype(np.float32)
    b["delta"][pick_f[:5], :3] = np.float32(0.2)                        # clamped to the radius
    m = W.Module(src)
    r = Recorder(m, b, "bounds", out, meta)
    for k in ("applyDeltaAll", "bounds", "velocityUpdate"):
        r.run(k, N, base)

    # ---- grab: select, integrate with a grab motion, release
    print("grab", flush=True)
    m = W.Module(src)
    r = Recorder(m, buffers(o2, C), "grab", out, meta)
    st = o2.read_state()
    top = st["pos"][:S_][np.argmax(st["pos"][:S_, 1])]
    gc = [float(top[0]), float(top[1]), float(top[2]), 2.5 * hs]
    r.run("grabSelect", S_, uniforms(sc, grabC=gc, grabLattice=0))
    # a small pull, one past the spring's 5 cm cap, one that slips every grip (over 1 m)
    for gd in ([0.0, 0.004, 0.0, 0.0], [0.0, 0.25, 0.05, 0.0], [0.0, 1.6, 0.0, 0.0]):
        r.run("integrate", N, uniforms(sc, grabDelta=gd))
    r.run("grabRelease", S_, base)

    # ---- emit (the hose)
    print("emit", flush=True)
    m = W.Module(src)
    r = Recorder(m, buffers(o2, C), "emit", out, meta)
    d = np.array([0.3, -0.8, 0.2])
    d /= np.linalg.norm(d)
    side = np.cross(d, [0.0, 1.0, 0.0])
    side /= np.linalg.norm(side)
    up = np.cross(side, d)
    start = int(o2.info.fluid_next)
    r.run("emit", 96, uniforms(sc, emitCount=96, emitStart=start, emitPos=[0.2, 1.6, -0.1, 3.0],
                                emitDir=[*d, 0.7], emitSide=[*side, 0.0], emitUp=[*up, 0.0]), wg_size=64)

    # ---- tools: cut + cutTets, pick, countActive
    print("tools", flush=True)
    m = W.Module(src)
    r = Recorder(m, buffers(o2, C), "tools", out, meta)
    o, d1, d2 = S.wedge_through(sc.desc.cube_center, 21)
    cut_u = uniforms(sc, cutO=[*o, 0.0], cutD1=[*d1, 0.0], cutD2=[*d2, 0.0])
    r.run("cut", NC, cut_u)
    r.run("cutTets", NT, cut_u)
    cc = np.array(sc.desc.cube_center)
    for k in range(5):
        ro = cc + rng.normal(size=3) * 0.6 + np.array([0.0, 2.0, 3.0])
        rd = cc + rng.normal(size=3) * 0.08 - ro
        rd /= np.linalg.norm(rd)
        b = r.b
        b["gridA"][C["TABLE"] * 2 + N] = 0xFFFFFFFF  # S_PICK reset, as GpuSim.pick does before dispatching
        r.run("pick", S_, uniforms(sc, pickO=[*ro, 0.3], pickD=[*rd, 0.0]), label=f"pick {k}")
    r.run("countActive", F, base)

    # ---- one whole frame: emit, the substeps, the queued cut, the active count
    # (GpuSim.encode, src/gpu/sim.js:333-392)
    print("frame", flush=True)
    b = buffers(o2, C)
    for k in MUTABLE:
        out[f"frame/start/{k}"] = b[k].copy()
    r = Runner(W.Module(src), b)
    emit_u = dict(emitCount=32, emitStart=int(o2.info.fluid_next), emitPos=[-0.15, 1.5, 0.2, 2.5],
                  emitDir=[0.0, -1.0, 0.0, 0.3], emitSide=[1.0, 0.0, 0.0, 0.0], emitUp=[0.0, 0.0, 1.0, 0.0])
    ow, d1w, d2w = S.wedge_through(sc.desc.cube_center, 31)
    frame_u = uniforms(sc, cutO=[*ow, 0.0], cutD1=[*d1w, 0.0], cutD2=[*d2w, 0.0], **emit_u)
    r.run("emit", 32, frame_u, wg_size=64)
    for k in range(sc.substeps):
        substep(r, C, frame_u, iters)
    r.run("cut", NC, frame_u)
    r.run("cutTets", NT, frame_u)
    r.run("countActive", F, frame_u)
    for k in MUTABLE:
        out[f"frame/end/{k}"] = b[k].copy()
    meta.append({"scenario": "frame", "index": 0, "kernel": "frame", "label": "frame", "changed": [],
                 "uniform": {u: (list(map(float, v)) if isinstance(v, list) else float(v)) for u, v in frame_u.items()},
                 "wedge": [list(map(float, ow)), list(map(float, d1w)), list(map(float, d2w))]})

    out["meta"] = np.frombuffer(json.dumps({"C": C, "passes": meta}).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, f"{OUT.stat().st_size / 1e3:.0f} kB")


if __name__ == "__main__":
    main()
