"""The reference app's snapshot and recording files, on libupbd.

  snapshot(gs)            GpuSim.snapshot (src/gpu/sim.js:493-513)
  restore(gs, snap)       GpuSim.restore (src/gpu/sim.js:526-545)
  load_snapshot(snap)     window.__sim.loadSnapshot (src/gpu/main.js:520-535):
                          a new GpuSim from the snapshot's options, then restore
  replay(bundle)          window.__sim.replay + applyReplay (src/gpu/main.js:
                          342-361, 510-518): restore keeping grab bits, then
                          re-apply the action log at its frame indices

A snapshot is a JSON object {version: 1, app: 'slice-splash-gpu', opts,
fluidNext, numCons, buffers}; every buffer is the base64 of its raw
little-endian bytes: pos, prev, vel (4 x f32 per particle), flags (u32),
density (2 x f32), cons (4 x u32 per constraint), tets (5 x u32 per tet:
four vertex ids and the rest-volume bits, negative = dead). A recording is
{version: 1, type: 'splash-recording', snapshot, actions: [{f, grab | rel |
cut | gd | emit | cam}]}. Files written by the reference load here and the
other way round, for scenes of the same options.
"""
from __future__ import annotations

import base64
import json

import numpy as np

from . import _lib as L
from .sim import GpuSim


def _b64(a: np.ndarray) -> str:
    return base64.b64encode(np.ascontiguousarray(a).tobytes()).decode("ascii")


def _unb64(s: str, dtype, cols: int | None = None) -> np.ndarray:
    a = np.frombuffer(base64.b64decode(s), dtype=np.dtype(dtype).newbyteorder("<")).astype(dtype)
    return a.reshape(-1, cols) if cols else a


def js_numbers(v):
    """A JSON-able value with every integral float as an int: JavaScript
    numbers have one type, and JSON.stringify prints 3.0 as 3."""
    if isinstance(v, dict):
        return {k: js_numbers(x) for k, x in v.items()}
    if isinstance(v, (list, tuple)):
        return [js_numbers(x) for x in v]
    if isinstance(v, float) and v.is_integer() and abs(v) < 2.0 ** 53:
        return int(v)
    return v


def snapshot_from_arrays(opts: dict, fluid_next: int, num_cons: int, state: dict, cons: np.ndarray,
                         tets: np.ndarray) -> dict:
    """The snapshot object of GpuSim.snapshot (src/gpu/sim.js:493-513) for
    host arrays: the same keys in the same order, each buffer the base64
    (b64encode, src/gpu/sim.js:3-9) of its raw little-endian bytes."""
    return {
        "version": 1,
        "app": "slice-splash-gpu",
        "opts": js_numbers(json.loads(json.dumps(opts))),
        "fluidNext": int(fluid_next),
        "numCons": int(num_cons),
        "buffers": {
            "pos": _b64(np.asarray(state["pos"]).astype("<f4")),
            "prev": _b64(np.asarray(state["prev"]).astype("<f4")),
            "vel": _b64(np.asarray(state["vel"]).astype("<f4")),
            "flags": _b64(np.asarray(state["flags"]).astype("<u4")),
            "density": _b64(np.asarray(state["density"]).astype("<f4")),
            "cons": _b64(np.asarray(cons).astype("<u4")),
            "tets": _b64(np.asarray(tets).astype("<u4")),
        },
    }


def snapshot(gs: GpuSim) -> dict:
    """The full particle state of a GpuSim as the reference's snapshot."""
    return snapshot_from_arrays(gs.o, gs.fluidNext, gs.NUM_CONS, gs.sim.read_state(),
                                gs.sim.read_constraints(), gs.sim.read_tets())


def decode_buffers(snap: dict, total: int, num_tets: int, keep_grabs: bool = False) -> dict:
    """The arrays GpuSim.restore (src/gpu/sim.js:515-545) writes from a
    snapshot of a scene with `total` particles and `num_tets` tets: pos,
    prev, vel, density, flags (grab bits cleared unless keep_grabs), cons,
    and tets when the snapshot holds exactly num_tets of them (older files
    have none, and keep the scene's own). Missing buffers are left out."""
    b = snap["buffers"]
    out = {}
    for name, cols in (("pos", 4), ("prev", 4), ("vel", 4), ("density", 2)):
        if name in b:
            a = _unb64(b[name], np.float32, cols)
            if a.shape[0] != total:
                raise ValueError(f"snapshot {name} holds {a.shape[0]} particles, the scene {total}")
            out[name] = a
    if "flags" in b:
        f = _unb64(b["flags"], np.uint32)
        if f.shape[0] != total:
            raise ValueError(f"snapshot flags hold {f.shape[0]} particles, the scene {total}")
        if not keep_grabs:
            f = f & np.uint32(~L.F_GRABBED & 0xFFFFFFFF)
        out["flags"] = f
    if "cons" in b:
        out["cons"] = _unb64(b["cons"], np.uint32, 4)
    if "tets" in b:
        t = _unb64(b["tets"], np.uint32)
        if num_tets and t.size == num_tets * 5:
            out["tets"] = t.reshape(-1, 5)
    return out


def restore(gs: GpuSim, snap: dict, keep_grabs: bool = False) -> None:
    """Writes a snapshot's buffers into a GpuSim built with the same options.
    Standalone snapshots drop the grab bits (no release will come); a
    recording keeps them, since the grab targets live in the buffers. A
    snapshot without tets (older files) leaves the tets as they are."""
    a = decode_buffers(snap, gs.TOTAL, gs.NUM_TETS, keep_grabs)
    kw = {k: a[k] for k in ("pos", "prev", "vel", "density", "flags") if k in a}
    gs.sim.write_state(**kw)
    if "cons" in a:
        gs.sim.write_constraints(a["cons"])
    if "tets" in a:
        gs.sim.write_tets(a["tets"])
    gs.sim.set_fluid_next(int(snap.get("fluidNext", 0)))


def load_snapshot(snap: dict, keep_grabs: bool = False, variant: str = "product") -> GpuSim:
    """A new GpuSim from the snapshot's options, restored to its state."""
    opts = dict(snap["opts"])
    if opts.get("SOLID_DIM2") is None:  # files from before the second cube
        opts["SOLID_DIM2"] = 0
    gs = GpuSim(opts, variant=variant)
    restore(gs, snap, keep_grabs)
    return gs


def apply_action(gs: GpuSim, a: dict) -> None:
    """One recorded input (the dispatch of applyReplay, src/gpu/main.js:344-352).
    Camera entries have no effect on the simulation."""
    if "grab" in a:
        g = a["grab"]
        gs.grabAt(g[:3], g[3], g[4] if len(g) > 4 and g[4] is not None else 0xFFFF)
    if a.get("rel"):
        gs.release()
    if "cut" in a:
        gs.queueCut(*a["cut"])
    if "gd" in a:
        gs.moveGrab(a["gd"])  # the frame's grab motion (pending.grabDelta starts at zero)
    if "emit" in a:
        e = a["emit"]
        gs.emit(int(e[0]), e[1:4], e[4:7], e[7:10], e[10:13], e[13], e[14])


def replay(bundle: dict, variant: str = "product", tail_frames: int = 120) -> GpuSim:
    """Plays a recording: restore (keeping grabs), then per frame the actions
    whose index has come, then the frame; ends `tail_frames` frames after the
    last action, as the reference's replay does."""
    gs = load_snapshot(bundle.get("snapshot", bundle), keep_grabs=True, variant=variant)
    actions = bundle.get("actions", [])
    last = actions[-1]["f"] if actions else 0
    frame, idx = 0, 0
    while True:
        while idx < len(actions) and actions[idx]["f"] <= frame:
            apply_action(gs, actions[idx])
            idx += 1
        frame += 1
        gs.encode()
        if idx >= len(actions) and frame > last + tail_frames:
            break
    return gs


def dumps(obj: dict) -> str:
    return json.dumps(obj, separators=(",", ":"))


def loads(s: str) -> dict:
    return json.loads(s)
