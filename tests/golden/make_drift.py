"""Reference trajectories for the 600-frame drift check (test_gpu_drift.py).

Runs the restated GPU kernels on the CPU (oracle O2) in FP64 and in FP32 over
600 frames of the default GPU scene (20^3 body + 65,536 fluid, slice wedge
after frame 60) and records per-frame aggregates of the state, so a GPU run
can be compared frame by frame without storing 600 states:

  fluid_n      active fluid particles
  fluid_mean   mean position of the active fluid (x, y, z)
  fluid_ke     mean squared speed of the active fluid
  body_com     mean position of the body particles (x, y, z)
  body_ke      mean squared speed of the body
  alive        alive constraints

Usage: python tests/golden/make_drift.py [frames]   (about 20-40 min on 8 cores)
"""
from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from fluidphysics_b200 import scenes as S  # noqa: E402
from oracle.oracle import o2_from_scene  # noqa: E402

KEYS = ("fluid_n", "fluid_mean", "fluid_ke", "body_com", "body_ke", "alive")


def aggregates(st: dict, cons_alive: np.ndarray, solid_n: int) -> dict:
    f = st["flags"][solid_n:] & 1 > 0
    fp = st["pos"][solid_n:, :3][f].astype(np.float64)
    fv = st["vel"][solid_n:, :3][f].astype(np.float64)
    bp = st["pos"][:solid_n, :3].astype(np.float64)
    bv = st["vel"][:solid_n, :3].astype(np.float64)
    return dict(fluid_n=float(f.sum()), fluid_mean=fp.mean(axis=0) if len(fp) else np.zeros(3),
                fluid_ke=float((fv ** 2).sum(axis=1).mean()) if len(fv) else 0.0,
                body_com=bp.mean(axis=0), body_ke=float((bv ** 2).sum(axis=1).mean()),
                alive=float(cons_alive.sum()))


def trajectory(scene: S.Scene, frames: int, step, read, slice_fn) -> dict:
    out = {k: [] for k in KEYS}
    for k in range(frames):
        if k == scene.slice_frame:
            slice_fn(*scene.wedge)
        step()
        st, alive = read()
        a = aggregates(st, alive, scene.solid_n)
        for key in KEYS:
            out[key].append(a[key])
    return {k: np.asarray(v) for k, v in out.items()}


def oracle_trajectory(scene: S.Scene, frames: int, precision: int) -> dict:
    o = o2_from_scene(scene, precision)

    def read():
        cons, _ = o.read_constraints()
        return o.read_state(), cons[:, 3] != 0

    return trajectory(scene, frames, lambda: o.step(scene.dt, scene.substeps), read, o.slice)


def main():
    frames = int(sys.argv[1]) if len(sys.argv) > 1 else 600
    sc = S.gpu_default(frames=frames)
    res = {}
    for prec, tag in ((1, "fp64"), (0, "fp32")):
        t = time.time()
        tr = oracle_trajectory(sc, frames, prec)
        for k, v in tr.items():
            res[f"{tag}_{k}"] = v
        print(tag, f"{time.time() - t:.0f} s", flush=True)
    out = Path(__file__).resolve().parent / "drift_gpu_default.npz"
    np.savez_compressed(out, frames=frames, **res)
    print(out)


if __name__ == "__main__":
    main()
