"""Many independent scenes stepped together (libupbd's scene batch).

  Batch           handle over upbd_batch_* (include/upbd_batch.h)
  batch_scenes    the seeded uneven-scene workload: body lattice dim uniform
                  in {6..20}, fluid count log-uniform in [2k, 65k],
                  deriveOpts at 30 mm (src/gpu/main.js:30-54), one seed per
                  scene
  autotune        picks the persistent grid's block size and CTAs per SM
                  (and optionally the hash cell size) by timing frames of
                  the live batch, then restores its state

The reference has no batch: every scene is a GpuSim of its own
(src/gpu/sim.js:76-584). A batch runs that same per-scene pass order with
one launch per pass for all scenes, so each scene's results match a
single-scene handle's (tests/test_gpu_batch.py checks that bit for bit).
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from . import scenes as S


class Batch:
    """One upbd_batch handle."""

    def __init__(self, solid_iters: int = 3, features: int = 0, max_scenes: int = 1024,
                 block_threads: int = 256, ctas_per_sm: int = 8, hbm_budget: int = 0, device: int = 0,
                 variant: str = "product"):
        self.lib = L.load(variant)
        d = L.BatchDesc()
        self.lib.upbd_batch_default_desc(C.byref(d))
        d.device, d.solid_iters, d.features, d.max_scenes = device, solid_iters, features, max_scenes
        d.block_threads, d.ctas_per_sm, d.hbm_budget = block_threads, ctas_per_sm, hbm_budget
        h = C.c_void_p()
        rc = self.lib.upbd_batch_create(C.byref(d), C.byref(h))
        if rc != L.UPBD_OK:
            msg = self.lib.upbd_batch_last_error(None)
            raise L.UpbdError(rc, msg.decode() if msg else "")
        self.h = h
        self.ids: list[int] = []

    def _ck(self, rc: int) -> None:
        L.check_batch(self.lib, self.h, rc)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.upbd_batch_destroy(self.h)
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

    # ------------------------------------------------------------ scenes
    def add_scene(self, scene: S.Scene) -> int:
        fp = np.ascontiguousarray(scene.fluid_pos, dtype=np.float32)
        fv = np.ascontiguousarray(scene.fluid_vel, dtype=np.float32)
        sid = C.c_int32()
        self._ck(self.lib.upbd_batch_add_scene(self.h, C.byref(scene.desc), C.byref(scene.params), len(fp),
                                               L.fptr(fp.reshape(-1)), L.fptr(fv.reshape(-1)),
                                               float(scene.fluid_mass), C.byref(sid)))
        self.ids.append(sid.value)
        return sid.value

    def remove_scene(self, sid: int) -> None:
        self._ck(self.lib.upbd_batch_remove_scene(self.h, sid))
        self.ids.remove(sid)

    def set_params(self, sid: int, p: L.Params) -> None:
        self._ck(self.lib.upbd_batch_set_params(self.h, sid, C.byref(p)))

    def scene_info(self, sid: int) -> L.Info:
        i = L.Info()
        self._ck(self.lib.upbd_batch_scene_info(self.h, sid, C.byref(i)))
        return i

    def info(self) -> L.BatchInfo:
        i = L.BatchInfo()
        self._ck(self.lib.upbd_batch_get_info(self.h, C.byref(i)))
        return i

    @staticmethod
    def scene_bytes(desc: L.SceneDesc, variant: str = "product") -> int:
        lib = L.load(variant)
        b = C.c_uint64()
        rc = lib.upbd_batch_scene_bytes(C.byref(desc), C.byref(b))
        if rc != L.UPBD_OK:
            raise L.UpbdError(rc, (lib.upbd_batch_last_error(None) or b"").decode())
        return b.value

    # ------------------------------------------------------------ frames
    def step(self, dt: float, substeps: int) -> None:
        self._ck(self.lib.upbd_batch_step(self.h, dt, substeps))

    def sync(self) -> None:
        self._ck(self.lib.upbd_batch_sync(self.h))

    def set_stream(self, stream_ptr: int | None) -> None:
        self._ck(self.lib.upbd_batch_set_stream(self.h, C.c_void_p(stream_ptr or 0)))

    def set_tuning(self, block_threads: int, ctas_per_sm: int) -> None:
        self._ck(self.lib.upbd_batch_set_tuning(self.h, block_threads, ctas_per_sm))

    @property
    def launches(self) -> int:
        return int(self.info().launches)

    def active_count(self, sid: int) -> int:
        n = C.c_uint32()
        self._ck(self.lib.upbd_batch_active_count(self.h, sid, C.byref(n)))
        return n.value

    def profile_frame(self, dt: float, substeps: int) -> tuple[np.ndarray, np.ndarray]:
        ms = (C.c_double * L.KERNEL_KINDS)()
        ln = (C.c_uint32 * L.KERNEL_KINDS)()
        self._ck(self.lib.upbd_batch_profile_frame(self.h, dt, substeps, ms, ln))
        return np.array(ms[:]), np.array(ln[:])

    # ------------------------------------------------------------ state
    def read_state(self, sid: int) -> dict:
        """pos, prev, vel (N x 4), density (N x 2) and flags of one scene."""
        n = self.scene_info(sid).total
        pos = np.empty((n, 4), np.float32)
        prev = np.empty((n, 4), np.float32)
        vel = np.empty((n, 4), np.float32)
        dens = np.empty((n, 2), np.float32)
        flags = np.empty(n, np.uint32)
        self._ck(self.lib.upbd_batch_read_state(self.h, sid, L.fptr(pos.reshape(-1)), L.fptr(prev.reshape(-1)),
                                                L.fptr(vel.reshape(-1)), L.fptr(dens.reshape(-1)), L.uptr(flags)))
        return dict(pos=pos, prev=prev, vel=vel, density=dens, flags=flags)

    def write_state(self, sid: int, pos=None, prev=None, vel=None, density=None, flags=None) -> None:
        def f(a):
            return None if a is None else L.fptr(np.ascontiguousarray(a, dtype=np.float32).reshape(-1))
        fl = None if flags is None else np.ascontiguousarray(flags, dtype=np.uint32)
        self._ck(self.lib.upbd_batch_write_state(self.h, sid, f(pos), f(prev), f(vel), f(density), L.uptr(fl)))

    def read_constraints(self, sid: int) -> np.ndarray:
        c = np.empty((self.scene_info(sid).num_cons, 4), np.uint32)
        self._ck(self.lib.upbd_batch_read_constraints(self.h, sid, L.uptr(c.reshape(-1))))
        return c

    def write_constraints(self, sid: int, cons: np.ndarray) -> None:
        c = np.ascontiguousarray(cons, dtype=np.uint32)
        self._ck(self.lib.upbd_batch_write_constraints(self.h, sid, L.uptr(c.reshape(-1))))


# ------------------------------------------------------------------ workload
def fluid_block(n: int, r: float, y0: float, seed: int) -> np.ndarray:
    """n fluid particles: the first n points of a jittered lattice block of
    16 layers at 2.2 r spacing (the emit spacing, src/gpu/wgsl.js:787),
    square in x/z and centred on the body."""
    ny = 16
    nx = max(1, math.ceil(math.sqrt(n / ny)))
    return S.jittered_block(nx, ny, nx, 2.2 * r, y0, seed)[:n]


def compact_table(n: int) -> int:
    """A hash table of the next power of two >= 2n buckets (at least 4,096):
    deriveOpts's sizing rule without its 2^18 floor (src/gpu/main.js:30-54),
    which only the reference's 256-wide scan passes needed."""
    return max(4096, 1 << math.ceil(math.log2(max(2 * n, 2))))


def batch_scene(dim: int, n_fluid: int, seed: int, radius_mm: float = 30, iters: int = 3,
                gravity: float = -9.8, table: str = "reference") -> S.Scene:
    """One scene of the uneven batch: deriveOpts(dim, n_fluid, radius_mm) with
    the fluid block above the body. table "compact" sizes the hash table by
    compact_table instead of deriveOpts's rule."""
    d, p, opts = S.gpu_scene(dim, n_fluid, radius_mm, gravity=gravity, iters=iters)
    if table == "compact":
        d.table_size = compact_table(dim ** 3 + n_fluid)
    r = radius_mm / 1000
    top = opts["cubeCenter"][1] + (dim - 1) * opts["spacing"] / 2
    fp = fluid_block(n_fluid, r, max(1.7, top + 3 * r), seed)
    return S.Scene(f"batch_{seed}", d, p, fp, np.zeros_like(fp), opts["fluidMass"], 1 / 60, 5, 300,
                   extra=dict(seed=seed))


def batch_scenes(n: int = 256, seed0: int = 1000, iters: int = 3, dims=(6, 20),
                 fluid_log2=(11.0, 16.0), table: str = "reference") -> list[S.Scene]:
    """The uneven batch: scene k draws its body dim uniformly from dims and
    its fluid count as floor(2^U(fluid_log2)) from numpy PCG64(seed0 + k)."""
    out = []
    for k in range(n):
        rng = np.random.default_rng(seed0 + k)
        dim = int(rng.integers(dims[0], dims[1] + 1))
        nf = int(math.floor(2.0 ** rng.uniform(*fluid_log2)))
        out.append(batch_scene(dim, nf, seed0 + k, iters=iters, table=table))
    return out


# ------------------------------------------------------------------ tuning
@dataclass
class Tuning:
    block_threads: int
    ctas_per_sm: int
    cell_scale: float
    ms_per_frame: float


def autotune(batch: Batch, scenes: dict[int, S.Scene], dt: float = 1 / 60, substeps: int = 5,
             frames: int = 6, block_threads=(128, 256), ctas_per_sm=(4, 8, 16),
             cell_scales=(1.0,), warm_frames: int = 2) -> tuple[Tuning, list[Tuning]]:
    """Times `frames` frames of the live batch for every candidate and keeps
    the fastest. Scene state is saved first and restored after each
    candidate (and at the end), so tuning leaves the batch where it was.
    Cell scales multiply every scene's hash cell size (>= 1 keeps the 27-cell
    neighbourhood complete); the chosen one stays applied."""
    saved = {sid: (batch.read_state(sid), batch.read_constraints(sid)) for sid in scenes}

    def restore():
        for sid, (st, cons) in saved.items():
            batch.write_state(sid, **st)
            batch.write_constraints(sid, cons)

    base = {sid: sc.params for sid, sc in scenes.items()}
    results = []
    for cs in cell_scales:
        for sid, p in base.items():
            q = L.Params.from_buffer_copy(p)
            q.cell_size = p.cell_size * cs
            batch.set_params(sid, q)
        for bt in block_threads:
            for cps in ctas_per_sm:
                batch.set_tuning(bt, cps)
                for _ in range(warm_frames):
                    batch.step(dt, substeps)
                batch.sync()
                t0 = time.perf_counter()
                for _ in range(frames):
                    batch.step(dt, substeps)
                batch.sync()
                ms = (time.perf_counter() - t0) * 1e3 / frames
                results.append(Tuning(bt, cps, cs, ms))
                restore()
    best = min(results, key=lambda t: t.ms_per_frame)
    for sid, p in base.items():
        q = L.Params.from_buffer_copy(p)
        q.cell_size = p.cell_size * best.cell_scale
        batch.set_params(sid, q)
    batch.set_tuning(best.block_threads, best.ctas_per_sm)
    restore()
    return best, results
