"""Continuous-batching frame server (include/upbd_server.h) and its served
workload.

  Server            handle over upbd_server_*: submit scene requests with
                    arrival times, run, read per-request results and the
                    p50/p99 frame latencies
  served_requests   the seeded served workload: Poisson arrivals (mean
                    rate 200/s), total particles log-uniform in [1k, 262k],
                    body fraction uniform in [0, 0.3], 1-60 frames each

The reference has no server; each request is a scene of the reference's GPU
setup (deriveOpts at 30 mm, src/gpu/main.js:30-54) stepped for its frames
by the same passes a single-scene handle runs.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from . import batch as B
from . import scenes as S

REQ_STATES = {0: "queued", 1: "preparing", 2: "ready", 3: "running", 4: "done", 5: "rejected"}


ServerDesc, Request, RequestResult, ServerStats = L.ServerDesc, L.Request, L.RequestResult, L.ServerStats


class Server:
    """One upbd_server handle (one batch on one GPU)."""

    def __init__(self, dt: float = 1 / 60, substeps: int = 5, solid_iters: int = 3, features: int = 0,
                 hbm_budget: int = 0, max_scenes: int = 4096, block_threads: int = 256, ctas_per_sm: int = 8,
                 builders: int = 4, keep_results: bool = False, device: int = 0, variant: str = "product"):
        self.lib = L.load(variant)
        d = ServerDesc()
        self.lib.upbd_server_default_desc(C.byref(d))
        d.batch.device, d.batch.solid_iters, d.batch.features = device, solid_iters, features
        d.batch.max_scenes, d.batch.hbm_budget = max_scenes, hbm_budget
        d.batch.block_threads, d.batch.ctas_per_sm = block_threads, ctas_per_sm
        d.dt, d.substeps, d.builders, d.keep_results = dt, substeps, builders, 1 if keep_results else 0
        h = C.c_void_p()
        rc = self.lib.upbd_server_create(C.byref(d), C.byref(h))
        if rc != L.UPBD_OK:
            raise L.UpbdError(rc, (self.lib.upbd_server_last_error(None) or b"").decode())
        self.h = h
        self._keep = []  # arrays referenced by submitted requests until submit returns

    def _ck(self, rc: int) -> None:
        if rc != L.UPBD_OK:
            raise L.UpbdError(rc, (self.lib.upbd_server_last_error(self.h) or b"").decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.upbd_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, scene: S.Scene, frames: int, arrival_s: float = 0.0) -> int:
        r = Request()
        r.desc, r.params = scene.desc, scene.params
        r.frames, r.arrival_s = frames, arrival_s
        fp = np.ascontiguousarray(scene.fluid_pos, dtype=np.float32).reshape(-1)
        r.n_fluid, r.fluid_mass = len(fp) // 3, float(scene.fluid_mass)
        r.fluid_pos3 = L.fptr(fp) if len(fp) else None
        fv = None
        if scene.fluid_vel is not None and np.any(scene.fluid_vel):
            fv = np.ascontiguousarray(scene.fluid_vel, dtype=np.float32).reshape(-1)
            r.fluid_vel3 = L.fptr(fv)
        rid = C.c_int64()
        self._ck(self.lib.upbd_server_submit(self.h, C.byref(r), C.byref(rid)))  # copies the arrays
        return rid.value

    def run(self, max_seconds: float = 600.0) -> None:
        self._ck(self.lib.upbd_server_run(self.h, max_seconds))

    def stats(self) -> dict:
        s = ServerStats()
        self._ck(self.lib.upbd_server_get_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_ if not k.startswith("reserved")}

    def result(self, rid: int, slots: int | None = None, with_state: bool = False) -> dict:
        res = RequestResult()
        pos = flags = None
        if with_state:
            self._ck(self.lib.upbd_server_result(self.h, rid, C.byref(res), None, None))
            pos = np.empty((res.slots, 4), np.float32)
            flags = np.empty(res.slots, np.uint32)
        self._ck(self.lib.upbd_server_result(self.h, rid, C.byref(res), L.fptr(pos.reshape(-1)) if with_state
                                             else None, L.uptr(flags) if with_state else None))
        out = {k: getattr(res, k) for k, _ in RequestResult._fields_ if not k.startswith("reserved")}
        out["state"] = REQ_STATES.get(res.state, res.state)
        if with_state:
            out["pos"], out["flags"] = pos, flags
        return out


# ------------------------------------------------------------------ workload
@dataclass
class ServedRequest:
    scene: S.Scene
    frames: int
    arrival_s: float


def served_requests(window_s: float = 2.0, rate: float = 200.0, seed: int = 5, radius_mm: float = 30,
                    iters: int = 3, total_range=(1024, 262144), body_frac=(0.0, 0.3),
                    frames_range=(1, 60)) -> list[ServedRequest]:
    """Requests arriving in [0, window_s): exponential inter-arrival times of
    mean 1/rate; total particles log-uniform in total_range; body fraction
    uniform in body_frac -> body dim = round(cbrt(body)), fluid = the rest;
    frames uniform in frames_range. numpy PCG64(seed) draws the stream; each
    scene's fluid block is seeded by its request index."""
    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    k = 0
    lo, hi = math.log(total_range[0]), math.log(total_range[1])
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= window_s:
            break
        total = int(round(math.exp(rng.uniform(lo, hi))))
        frac = rng.uniform(*body_frac)
        dim = int(round((frac * total) ** (1 / 3)))
        fluid = max(0, total - dim ** 3)
        frames = int(rng.integers(frames_range[0], frames_range[1] + 1))
        sc = B.batch_scene(dim, fluid, seed * 100000 + k, radius_mm=radius_mm, iters=iters)
        out.append(ServedRequest(sc, frames, t))
        k += 1
    return out
