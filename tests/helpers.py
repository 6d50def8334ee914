"""Shared helpers for the parity tests (CPU oracle vs CUDA library)."""
from __future__ import annotations

import numpy as np

from fluidphysics_b200 import scenes as S

# Per-substep tolerances of the FMA product build against the FP32 oracle
# (O2<float>), as max-norm errors relative to a scale: positions relative to
# the basin extent (10 m), velocities relative to maxSpeed (14 m/s).
POS_SCALE = 10.0
VEL_SCALE = 14.0
POS_RTOL = 1e-5
VEL_RTOL = 1e-4


def settled_state(scene: S.Scene, frames: int, precision: int = 0):
    """Run the FP32 oracle `frames` frames from the scene's initial state and
    return (oracle, state, cons) — a state with live contacts and pressure."""
    from oracle.oracle import o2_from_scene
    o2 = o2_from_scene(scene, precision)
    for _ in range(frames):
        o2.step(scene.dt, scene.substeps)
    st = o2.read_state()
    cons, _ = o2.read_constraints()
    return o2, st, cons


def load_state(sim, st, cons=None):
    sim.write_state(pos=st["pos"].astype(np.float32), prev=st["prev"].astype(np.float32),
                    vel=st["vel"].astype(np.float32), density=st["density"].astype(np.float32),
                    flags=st["flags"].astype(np.uint32))
    if cons is not None:
        sim.write_constraints(cons)


def max_rel(a: np.ndarray, b: np.ndarray, scale: float, mask=None) -> float:
    d = np.abs(a.astype(np.float64) - b.astype(np.float64))
    if mask is not None:
        d = d[mask]
    return float(d.max() / scale) if d.size else 0.0


def assert_states_equal(g: dict, r: dict, what: str = "") -> None:
    """Bit-exact comparison of GPU float32 state with the FP32 oracle's."""
    for k in ("pos", "prev", "vel", "density"):
        a = g[k]
        b = r[k].astype(np.float32)
        bad = np.flatnonzero(~((a == b) | (np.isnan(a) & np.isnan(b))).all(axis=1))
        assert bad.size == 0, f"{what}: {k} differs at {bad[:8]} (gpu {a[bad[:2]]} vs oracle {b[bad[:2]]})"
    assert np.array_equal(g["flags"], r["flags"]), f"{what}: flags differ"


def assert_states_close(g: dict, r: dict, what: str = "", pos_rtol=POS_RTOL, vel_rtol=VEL_RTOL) -> dict:
    assert np.array_equal(g["flags"], r["flags"]), f"{what}: flags differ"
    act = (g["flags"] & 1).astype(bool)
    ep = max_rel(g["pos"][:, :3], r["pos"][:, :3], POS_SCALE, act)
    ev = max_rel(g["vel"][:, :3], r["vel"][:, :3], VEL_SCALE, act)
    assert ep <= pos_rtol, f"{what}: position error {ep:.3g} > {pos_rtol}"
    assert ev <= vel_rtol, f"{what}: velocity error {ev:.3g} > {vel_rtol}"
    return dict(pos=ep, vel=ev)


def crossing_state(sc, cluster=12):
    """The CPU scene with its lattice moved so that a surface solid j sits
    1 mm below a cell boundary in x, every fluid particle inactive but one,
    i, 2 mm into the cell two cells beyond j's, and a packed cluster right
    behind i whose pressure pushes i back towards the lattice by the
    displacement limit (0.35 H) within one substep: i crosses into the cell
    next to j's and ends within contact range of j. Rows are float32-exact."""
    from oracle.oracle import o2_from_scene
    o2 = o2_from_scene(sc)
    st = o2.read_state()
    pos, flags = st["pos"].copy(), st["flags"].copy()
    n_s, c = sc.solid_n, sc.params.cell_size
    sol = pos[:n_s, :3]
    ctr = sol.mean(axis=0)
    j = int(np.argmax(sol[:, 0] - 1e-3 * (np.abs(sol[:, 1] - ctr[1]) + np.abs(sol[:, 2] - ctr[2]))))
    Y = np.floor(sol[j, 0] / c) + 3
    pos[:n_s, 0] += (Y + 1) * c - 0.001 - sol[j, 0]
    flags[n_s:] = 0
    i = n_s
    pos[i, :3] = [(Y + 2) * c + 0.002, pos[j, 1], pos[j, 2]]
    flags[i] = 1
    for m in range(cluster):
        a = 2 * np.pi * m / cluster
        pos[i + 1 + m, :3] = [pos[i, 0] + 0.04, pos[j, 1] + 0.01 * np.cos(a), pos[j, 2] + 0.01 * np.sin(a)]
        flags[i + 1 + m] = 1
    f32 = lambda a: a.astype(np.float32).astype(np.float64)
    return dict(pos=f32(pos), prev=f32(st["prev"]), vel=np.zeros_like(st["vel"]), density=f32(st["density"]),
                flags=flags), i, j, Y
