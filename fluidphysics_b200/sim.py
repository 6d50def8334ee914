"""Host-side mirror of the reference's solver surfaces over libupbd.so.

  Sim      thin handle over the C ABI (one resident scene on one GPU)
  GpuSim   the surface of class GpuSim, src/gpu/sim.js:76-584
  Solver   the surface of class Solver, src/solver.js:8-516

Both mirrors run the B200 kernels; nothing here computes physics on the CPU.
Method names and argument meanings follow the reference; readbacks are
synchronous (the reference's async mapAsync readbacks become plain calls).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib as L
from . import scenes as S


class Sim:
    """One upbd_sim handle."""

    def __init__(self, desc: L.SceneDesc, params: L.Params, variant: str = "product"):
        self.lib = L.load(variant)
        self.variant = variant
        h = C.c_void_p()
        rc = self.lib.upbd_create(C.byref(desc), C.byref(params), C.byref(h))
        if rc != L.UPBD_OK:
            msg = self.lib.upbd_last_error(None)
            raise L.UpbdError(rc, msg.decode() if msg else "")
        self.h = h
        self.info = self.get_info()

    # ------------------------------------------------------------ plumbing
    def _ck(self, rc: int) -> None:
        L.check(self.lib, self.h, rc)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.upbd_destroy(self.h)
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

    def get_info(self) -> L.Info:
        info = L.Info()
        self._ck(self.lib.upbd_get_info(self.h, C.byref(info)))
        return info

    def set_params(self, p: L.Params) -> None:
        self._ck(self.lib.upbd_set_params(self.h, C.byref(p)))

    def get_params(self) -> L.Params:
        p = L.Params()
        self._ck(self.lib.upbd_get_params(self.h, C.byref(p)))
        return p

    def set_stream(self, stream_ptr: int | None) -> None:
        self._ck(self.lib.upbd_set_stream(self.h, C.c_void_p(stream_ptr or 0)))

    def device_ptrs(self) -> L.DevicePtrs:
        d = L.DevicePtrs()
        self._ck(self.lib.upbd_get_device_ptrs(self.h, C.byref(d)))
        return d

    def set_graphs(self, on: bool) -> None:
        self._ck(self.lib.upbd_set_graphs(self.h, 1 if on else 0))

    @property
    def launches(self) -> int:
        return int(self.lib.upbd_launch_count(self.h))

    def graph_floor(self, dt: float, substeps: int, reps: int = 200) -> tuple[float, int]:
        """(ms per replay, kernel nodes) of the frame graph with every kernel
        replaced by an empty one of the same grid: the frame's launch floor."""
        import ctypes as C
        ms = C.c_double()
        nk = C.c_uint32()
        self._ck(self.lib.upbd_profile_graph_floor(self.h, float(dt), int(substeps), int(reps), C.byref(ms),
                                                   C.byref(nk)))
        return float(ms.value), int(nk.value)

    # ------------------------------------------------------------ stepping
    def step(self, dt: float, substeps: int) -> None:
        self._ck(self.lib.upbd_step(self.h, float(dt), int(substeps)))

    def frame(self) -> None:
        self._ck(self.lib.upbd_frame(self.h))

    def sync(self) -> None:
        self._ck(self.lib.upbd_sync(self.h))

    def health(self) -> int:
        b = C.c_uint32()
        self._ck(self.lib.upbd_health(self.h, C.byref(b)))
        return b.value

    def clear_health(self) -> None:
        self._ck(self.lib.upbd_clear_health(self.h))

    def substep_partial(self, h: float, last_pass: int) -> None:
        self._ck(self.lib.upbd_substep_partial(self.h, float(h), int(last_pass)))

    def rebuild_grid(self) -> None:
        self._ck(self.lib.upbd_rebuild_grid(self.h))

    # ------------------------------------------------------------ tools
    def reset_solid(self) -> None:
        self._ck(self.lib.upbd_reset_solid(self.h))

    def drain(self) -> None:
        self._ck(self.lib.upbd_drain(self.h))

    def active_count(self) -> int:
        n = C.c_uint32()
        self._ck(self.lib.upbd_active_count(self.h, C.byref(n)))
        return n.value

    def emit(self, count, pos, dir, side, up, speed, phase) -> None:
        self._ck(self.lib.upbd_emit(self.h, int(count), L.f3(pos), L.f3(dir), L.f3(side), L.f3(up),
                                    float(speed), float(phase)))

    def emit_particles(self, pos3: np.ndarray, vel3: np.ndarray, mass: float) -> None:
        p = np.ascontiguousarray(pos3, dtype=np.float32).reshape(-1, 3)
        v = np.ascontiguousarray(vel3, dtype=np.float32).reshape(-1, 3)
        assert p.shape == v.shape
        self._ck(self.lib.upbd_emit_particles(self.h, p.shape[0], L.fptr(p), L.fptr(v), float(mass)))

    def slice(self, o, d1, d2) -> None:
        self._ck(self.lib.upbd_slice(self.h, L.d3(o), L.d3(d1), L.d3(d2)))

    def slice_now(self, o, d1, d2) -> int:
        n = C.c_uint32()
        self._ck(self.lib.upbd_slice_now(self.h, L.d3(o), L.d3(d1), L.d3(d2), C.byref(n)))
        return n.value

    def pick(self, ro, rd, max_perp: float):
        i = C.c_int32()
        t = C.c_double()
        self._ck(self.lib.upbd_pick(self.h, L.d3(ro), L.d3(rd), float(max_perp), C.byref(i), C.byref(t)))
        return (i.value, t.value) if i.value >= 0 else (-1, math.inf)

    def grab_select(self, center, radius: float, lattice: int = 0xFFFF) -> None:
        self._ck(self.lib.upbd_grab_select(self.h, L.f3(center), float(radius), int(lattice)))

    def grab_indices(self, idx, weight=None, targets=None) -> None:
        ix = np.ascontiguousarray(idx, dtype=np.uint32)
        w = None if weight is None else np.ascontiguousarray(weight, dtype=np.float32)
        t = None if targets is None else np.ascontiguousarray(targets, dtype=np.float32).reshape(-1)
        self._ck(self.lib.upbd_grab_indices(self.h, L.uptr(ix), ix.size, L.fptr(w), L.fptr(t)))

    def grab_move(self, delta) -> None:
        self._ck(self.lib.upbd_grab_move(self.h, L.f3(delta)))

    def release(self) -> None:
        self._ck(self.lib.upbd_release(self.h))

    # ------------------------------------------------------------ state
    def read_state(self):
        n = self.info.total
        pos = np.empty((n, 4), np.float32)
        prev = np.empty((n, 4), np.float32)
        vel = np.empty((n, 4), np.float32)
        dens = np.empty((n, 2), np.float32)
        flags = np.empty(n, np.uint32)
        self._ck(self.lib.upbd_read_state(self.h, L.fptr(pos), L.fptr(prev), L.fptr(vel), L.fptr(dens),
                                          L.uptr(flags)))
        return dict(pos=pos, prev=prev, vel=vel, density=dens, flags=flags)

    def read_state_async(self, pos, flags) -> None:
        """Starts copying positions (float32[total, 4]) and flags (uint32[total])
        into the given host arrays (pinned for an asynchronous copy) as they
        stand after the work enqueued so far; read_wait() before using them."""
        self._ck(self.lib.upbd_read_state_async(self.h, L.fptr(pos), L.uptr(flags)))

    def read_wait(self) -> None:
        self._ck(self.lib.upbd_read_wait(self.h))

    def write_state(self, pos=None, prev=None, vel=None, density=None, flags=None) -> None:
        n = self.info.total

        def f(a, k):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float32)
            assert a.size == n * k
            return a

        u = None if flags is None else np.ascontiguousarray(flags, dtype=np.uint32)
        arrs = [f(pos, 4), f(prev, 4), f(vel, 4), f(density, 2)]
        self._ck(self.lib.upbd_write_state(self.h, *[L.fptr(a) for a in arrs], L.uptr(u)))

    def read_constraints(self) -> np.ndarray:
        c = np.empty((max(self.info.num_cons, 0), 4), np.uint32)
        self._ck(self.lib.upbd_read_constraints(self.h, L.uptr(c)))
        return c

    def write_constraints(self, cons: np.ndarray) -> None:
        c = np.ascontiguousarray(cons, dtype=np.uint32)
        self._ck(self.lib.upbd_write_constraints(self.h, L.uptr(c)))

    def read_adjacency(self) -> np.ndarray:
        a = np.empty(self.info.solid_n + 1 + 2 * self.info.num_cons, np.uint32)
        self._ck(self.lib.upbd_read_adjacency(self.h, L.uptr(a)))
        return a

    def read_grid(self):
        T = self.info.table_size
        counts = np.empty(T, np.uint32)
        offsets = np.empty(T + 1, np.uint32)
        entries = np.empty(self.info.total, np.uint32)
        n = C.c_uint32()
        self._ck(self.lib.upbd_read_grid(self.h, L.uptr(counts), L.uptr(offsets), L.uptr(entries),
                                         C.byref(n)))
        return counts, offsets, entries[: n.value].copy()

    def read_tets(self) -> np.ndarray:
        t = np.empty((max(self.info.num_tets, 0), 5), np.uint32)
        if self.info.num_tets:
            self._ck(self.lib.upbd_read_tets(self.h, L.uptr(t)))
        return t

    def write_tets(self, tets5: np.ndarray) -> None:
        t = np.ascontiguousarray(tets5, dtype=np.uint32)
        self._ck(self.lib.upbd_write_tets(self.h, L.uptr(t)))

    def set_fluid_next(self, k: int) -> None:
        self._ck(self.lib.upbd_set_fluid_next(self.h, int(k)))

    def groups(self) -> np.ndarray:
        """Solver._recomputeGroups (src/solver.js:488-499): the root label of
        every solid after the union-find over the alive constraints."""
        g = np.empty(self.info.solid_n, np.int32)
        self._ck(self.lib.upbd_groups(self.h, g.ctypes.data_as(C.POINTER(C.c_int32))))
        return g

    def groups_device(self, out_ptr: int) -> None:
        """The same labels into device memory (solid_n int32 at out_ptr), on
        the simulation's stream, with no host synchronisation."""
        self._ck(self.lib.upbd_groups_device(self.h, C.c_void_p(out_ptr)))


def sim_from_scene(scene: S.Scene, variant: str = "product") -> Sim:
    """Create a Sim for a Scene and load its initial fluid block."""
    s = Sim(scene.desc, scene.params, variant)
    if len(scene.fluid_pos):
        s.emit_particles(scene.fluid_pos, scene.fluid_vel, scene.fluid_mass)
    return s


class GpuSim:
    """Mirror of class GpuSim (src/gpu/sim.js:76-584) on libupbd.so.

    opts follow the reference (SOLID_DIM, SOLID_DIM2, MAX_FLUID, TABLE,
    spacing, solidMass, fluidMass, cubeCenter, substeps, solidIters,
    params={...}); `features` selects the optional passes (tets, solid
    contact cache) of the reference's full schedule."""

    def __init__(self, opts: dict | None = None, features: int = L.FEAT_TETS | L.FEAT_SOLID_CONTACTS,
                 device: int = 0, variant: str = "product"):
        opts = dict(opts or {})
        self.desc = S.desc_from_opts(opts, features=features, device=device)
        self.params = S.default_params()
        S.set_params(self.params, opts.get("params", {}))
        self.sim = Sim(self.desc, self.params, variant)
        # the merged options of the constructor (src/gpu/sim.js:78-84), with
        # the companion cube's size resolved: what a snapshot carries
        self.o = S.merge_gpu_opts(opts)
        i = self.sim.info
        self.SOLID_N, self.N1, self.TOTAL = i.solid_n, i.n1, i.total
        self.DIM2, self.NUM_CONS, self.NUM_TETS = i.dim2, i.num_cons, i.num_tets
        self.substeps, self.solidIters = i.substeps, i.solid_iters

    @property
    def fluidNext(self) -> int:
        return self.sim.get_info().fluid_next

    @property
    def frame(self) -> int:
        return self.sim.get_info().frames

    def setParam(self, key: str, value: float) -> None:
        S.set_params(self.params, {key: value})
        self.sim.set_params(self.params)

    def encode(self) -> None:
        """One frame (GpuSim.encode)."""
        self.sim.frame()

    def emit(self, count, pos, dir, side, up, speed, phase) -> None:
        self.sim.emit(count, pos, dir, side, up, speed, phase)

    def queueCut(self, o, d1, d2) -> None:
        self.sim.slice(o, d1, d2)

    def pick(self, ro, rd, maxPerp: float = 0.25):
        i, t = self.sim.pick(ro, rd, maxPerp)
        return None if i < 0 else {"id": i, "t": t}

    def grabAt(self, center, radius, lattice: int = 0xFFFF) -> None:
        self.sim.grab_select(center, radius, lattice)

    def moveGrab(self, delta) -> None:
        self.sim.grab_move(delta)

    def release(self) -> None:
        self.sim.release()

    def resetSolid(self) -> None:
        self.sim.reset_solid()

    def clearFluid(self) -> None:
        self.sim.drain()

    def readActiveCount(self) -> int:
        return self.sim.active_count()

    def readState(self) -> dict:
        s = self.sim.read_state()
        return {"pos": s["pos"], "vel": s["vel"], "flags": s["flags"]}

    def readConsAlive(self) -> dict:
        c = self.sim.read_constraints()
        return {"alive": int(c[:, 3].sum()), "total": self.NUM_CONS}

    def metrics(self) -> dict:
        """The app's health probe, window.__sim.metrics() (src/gpu/main.js:542-567)."""
        return state_metrics(self.readState(), self.SOLID_N)

    def cutLine(self, x: float, eye) -> None:
        """window.__sim.cutLine(x) (src/gpu/main.js:568-578): a vertical slice
        through the body at world x, queued as wedge segments from the eye
        (the app's camera position) to targets (x, 0.6 + t, 0), t = -1.4 ..
        1.4 by 0.1, one segment applied per frame."""
        for o, d1, d2 in cut_line_segments(x, eye):
            self.queueCut(o, d1, d2)

    def dispose(self) -> None:
        self.sim.close()


def cut_line_segments(x: float, eye) -> list:
    """The wedge segments of window.__sim.cutLine(x) (src/gpu/main.js:568-578)
    from an eye position: (origin, previous direction, direction) for the
    targets (x, 0.6 + t, 0), t = -1.4, -1.3, ... (the app's loop bound
    t <= 1.4 on the double sum: 28 targets, 27 segments)."""
    o = np.asarray(eye, dtype=np.float64)
    out, prev = [], None
    t = -1.4
    while t <= 1.4:
        d = np.array([x, 0.6 + t, 0.0]) - o
        d /= np.linalg.norm(d)
        if prev is not None:
            out.append((o, prev, d))
        prev = d
        t += 0.1
    return out


def state_metrics(st: dict, solid_n: int) -> dict:
    """Aggregates of window.__sim.metrics() (src/gpu/main.js:542-567) over a
    state read back as upbd_read_state returns it: the body's lowest and
    highest y, non-finite count and mean speed; the active fluid's count,
    non-finite count, highest y, percentage below y = 0.5 (pooled) and mean
    speed."""
    pos = st["pos"].astype(np.float64)
    vel = st["vel"].astype(np.float64)
    sy = pos[:solid_n, 1]
    sok = np.isfinite(sy)
    ssp = np.sqrt((vel[:solid_n, :3] ** 2).sum(axis=1))
    act = (st["flags"][solid_n:] & 1) == 1
    fy = pos[solid_n:, 1][act]
    fok = np.isfinite(fy)
    fsp = np.sqrt((vel[solid_n:, :3][act][fok] ** 2).sum(axis=1))
    fn = int(fok.sum())
    return {
        "solid": {"minY": float(sy[sok].min()) if sok.any() else 1e9,
                  "maxY": float(sy[sok].max()) if sok.any() else -1e9,
                  "bad": int((~sok).sum()), "avgSpeed": float(ssp[sok].sum() / max(solid_n, 1))},
        "fluid": {"n": fn, "bad": int((~fok).sum()), "maxY": float(fy[fok].max()) if fn else -1e9,
                  "pooledPct": int(np.floor(100 * (fy[fok] < 0.5).sum() / fn + 0.5)) if fn else 0,
                  "avgSpeed": float(fsp.mean()) if fn else 0.0},
        "gpu": None,
    }


class Solver:
    """Mirror of class Solver (src/solver.js:8-516) on libupbd.so.

    The substep is the GPU pass chain (Jacobi gathers), configured with the
    CPU solver's constants and its order-independent rules (strain tearing,
    unclamped plasticity, full contact push). `grabs` entries {i, x, y, z}
    become spring targets of the integrate pass with grip 1 and stiffness
    grabStiffness."""

    FLUID, SOLID = 0, 1

    def __init__(self, maxFluid: int = 2600, iters: int = 3, device: int = 0, variant: str = "product"):
        self.maxFluid = maxFluid
        self.iters = iters
        self.device = device
        self.variant = variant
        self.solidCount = 0
        self.capacity = 0
        # tuning, src/solver.js:14-36
        self.gravity = -10.0
        self.solidRadius, self.fluidRadius = 0.09, 0.075
        self.compliance = 2.5e-4
        self.plasticThreshold, self.plasticRate, self.breakStrain = 0.32, 0.04, 2.6
        self.fluidH, self.restDensity, self.stiffness, self.nearStiffness = 0.19, 6.0, 0.002, 0.008
        self.viscosity, self.solidDamping = 0.3, 1.2
        self.floorFrictionSolid, self.floorFrictionFluid = 0.4, 0.04
        self.wall = {"x": 3.5, "z": 3.5, "height": 0.92, "halfThick": 0.07}
        self.cullRadius, self.maxSpeed = 7.0, 14.0
        self.grabs: list[dict] = []
        self.grabStiffness = 0.3
        self.cellSize = 0.22
        self.sim: Sim | None = None
        self._grabbed: list[int] = []

    def _params(self, h: float) -> L.Params:
        p = S.solver_params(self.gravity)
        S.set_params(p, dict(h=h, solidRadius=self.solidRadius, fluidRadius=self.fluidRadius,
                             compliance=self.compliance, plasticThreshold=self.plasticThreshold,
                             plasticRate=self.plasticRate, breakStrain=self.breakStrain,
                             fluidH=self.fluidH, restDensity=self.restDensity,
                             stiffness=self.stiffness, nearStiffness=self.nearStiffness,
                             viscosity=self.viscosity, dampSolid=self.solidDamping,
                             frictionSolid=self.floorFrictionSolid,
                             frictionFluid=self.floorFrictionFluid, wallX=self.wall["x"],
                             wallZ=self.wall["z"], wallH=self.wall["height"],
                             wallT=self.wall["halfThick"], cullR=self.cullRadius,
                             maxSpeed=self.maxSpeed, grabK=self.grabStiffness,
                             cellSize=self.cellSize))
        return p

    def addSolidCube(self, cx, cy, cz, n: int = 7, spacing: float = 0.18, particleMass: float = 0.08):
        d = L.SceneDesc()
        S._fill_default_desc(d)
        d.solid_dim, d.solid_dim2, d.max_fluid = n, 0, self.maxFluid
        cap = n ** 3 + self.maxFluid
        d.table_size = 1 << math.ceil(math.log2(2 * cap))  # src/solver.js:51
        d.substeps, d.solid_iters, d.device = 5, self.iters, self.device
        d.spacing, d.solid_mass, d.fluid_mass = spacing, particleMass, 0.03
        d.cube_center[:] = [cx, cy, cz]
        self.sim = Sim(d, self._params(1 / 300), self.variant)
        self.solidCount = n ** 3
        self.capacity = cap

    def step(self, dt: float, substeps: int = 5) -> None:
        self._sync_grabs()
        self.sim.set_params(self._params(dt / substeps))
        self.sim.step(dt, substeps)

    def _sync_grabs(self) -> None:
        ids = [g["i"] for g in self.grabs]
        if ids != self._grabbed:
            self.sim.release()
            if ids:
                tg = np.array([[g["x"], g["y"], g["z"]] for g in self.grabs], np.float32)
                self.sim.grab_indices(np.array(ids, np.uint32), None, tg)
            self._grabbed = ids

    def emitFluid(self, x, y, z, vx, vy, vz, mass: float = 0.03) -> None:
        self.sim.emit_particles(np.array([[x, y, z]], np.float32), np.array([[vx, vy, vz]], np.float32),
                                mass)

    def clearFluid(self) -> None:
        self.sim.drain()

    def resetSolid(self) -> None:
        """Solver.resetSolid keeps the fluid; the GPU reset rewrites whole
        buffers, so the fluid state is carried across it."""
        st = self.sim.read_state()
        self.sim.reset_solid()
        s = self.solidCount
        fresh = self.sim.read_state()
        for k in ("pos", "prev", "vel", "density", "flags"):
            fresh[k][s:] = st[k][s:]
        self.sim.write_state(**fresh)
        self.grabs = []
        self._grabbed = []

    def fluidCount(self) -> int:
        return self.sim.active_count()

    def cut(self, ox, oy, oz, d1x, d1y, d1z, d2x, d2y, d2z) -> int:
        return self.sim.slice_now((ox, oy, oz), (d1x, d1y, d1z), (d2x, d2y, d2z))

    def pickSolid(self, ox, oy, oz, dx, dy, dz, maxPerp: float = 0.2):
        i, t = self.sim.pick((ox, oy, oz), (dx, dy, dz), maxPerp)
        return None if i < 0 else {"id": i, "t": t}

    # typed-array views of the reference (read back on access)
    @property
    def pos(self) -> np.ndarray:
        return self.sim.read_state()["pos"][:, :3].reshape(-1).copy()

    @property
    def vel(self) -> np.ndarray:
        return self.sim.read_state()["vel"][:, :3].reshape(-1).copy()

    @property
    def active(self) -> np.ndarray:
        return (self.sim.read_state()["flags"] & L.F_ACTIVE).astype(np.uint8)

    @property
    def type(self) -> np.ndarray:
        t = np.zeros(self.capacity, np.uint8)
        t[: self.solidCount] = self.SOLID
        return t

    @property
    def group(self) -> np.ndarray:
        g = np.zeros(self.capacity, np.int32)
        g[: self.solidCount] = self.sim.groups()
        return g
