"""ORACLE — test infrastructure only.

ctypes wrapper of oracle/_build/liboracle.so: O1 (restatement of the CPU
solver src/solver.js) and O2 (restatement of the WGSL kernels of
src/gpu/wgsl.js in the pass order of src/gpu/sim.js, float or double).
Only tests/, the smoke check and bench.py's CPU-baseline leg use this module,
as the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
_lib = None


def build() -> Path:
    res = subprocess.run(["make", "-s", "-C", str(HERE)], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    lib = C.CDLL(str(LIB))
    P, D, F, U, I = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_uint32), C.c_int
    sigs = {
        "o1_create": (P, [I]), "o1_destroy": (None, [P]), "o1_set_param": (I, [P, C.c_char_p, C.c_double]),
        "o1_add_solid_cube": (None, [P, C.c_double, C.c_double, C.c_double, I, C.c_double, C.c_double]),
        "o1_emit_fluid": (None, [P, I, D, D, C.c_double]), "o1_sizes": (None, [P, C.POINTER(C.c_int)]),
        "o1_len": (C.c_long, [P, C.c_char_p]), "o1_get": (I, [P, C.c_char_p, P]),
        "o1_set": (I, [P, C.c_char_p, P]), "o1_step": (None, [P, C.c_double, I]),
        "o1_pass": (I, [P, I, C.c_double]), "o1_cut": (I, [P, D, D, D]),
        "o1_pick": (I, [P, D, D, C.c_double, D]), "o1_set_grabs": (None, [P, I, C.POINTER(C.c_int), D]),
        "o1_reset_solid": (None, [P]), "o1_clear_fluid": (None, [P]), "o1_fluid_count": (I, [P]),
        "o1_components_dirty": (I, [P]),
        "o2_create": (P, [P, P, I]), "o2_destroy": (None, [P]), "o2_info": (None, [P, P]),
        "o2_set_params": (None, [P, P]), "o2_step": (None, [P, C.c_double, I]), "o2_frame": (None, [P]),
        "o2_substep_partial": (None, [P, C.c_double, I]), "o2_rebuild_grid": (None, [P]),
        "o2_run_pass": (I, [P, I, C.c_double]),
        "o2_set_iters": (None, [P, I]),
        "o2_read_state": (None, [P, D, D, D, D, U]), "o2_write_state": (None, [P, D, D, D, D, U]),
        "o2_read_delta": (None, [P, D]), "o2_read_constraints": (None, [P, U, D]),
        "o2_write_constraints": (None, [P, U]), "o2_read_adjacency": (None, [P, U]),
        "o2_read_grid": (None, [P, U, U, U]), "o2_read_tets": (None, [P, U]),
        "o2_read_tet_adjacency": (None, [P, U]),
        "o2_run_pass_x": (I, [P, I, C.c_double, F]), "o2_write_delta": (None, [P, D]),
        "o2_read_contact_cache": (None, [P, U, U]), "o2_write_contact_cache": (None, [P, U, U]),
        "o2_write_tets": (None, [P, U]),
        "o2_emit": (None, [P, I, F, F, F, F, C.c_float, C.c_float]),
        "o2_emit_particles": (None, [P, I, F, F, C.c_double]),
        "o2_slice_now": (C.c_uint32, [P, D, D, D]), "o2_slice": (None, [P, D, D, D]),
        "o2_pick": (I, [P, D, D, C.c_double, D]), "o2_grab_select": (None, [P, F, C.c_float, C.c_uint32]),
        "o2_grab_indices": (None, [P, U, I, F, F]), "o2_grab_move": (None, [P, F]),
        "o2_release": (None, [P]), "o2_drain": (None, [P]), "o2_active_count": (C.c_uint32, [P]),
        "o2_reset_solid": (None, [P]), "o2_groups": (None, [P, C.POINTER(C.c_int32)]),
        "o2_health": (C.c_uint32, [P]), "o2_fluid_next": (I, [P]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _d(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))


def _d3(v):
    return (C.c_double * 3)(*[float(x) for x in v])


def _f3(v):
    return (C.c_float * 3)(*[float(x) for x in v])


class O1:
    """Restatement of class Solver (src/solver.js)."""

    F32 = ("pos", "prev", "vel", "invMass", "rho", "rhoNear", "press", "pressNear",
           "dispX", "dispY", "dispZ", "pairD")
    I32 = ("group", "cellStart", "cellEntries", "pairI", "pairJ", "nbrCnt", "consA", "consB")
    U8 = ("active", "type", "consAlive")
    PASSES = dict(integrate=0, grab=1, grid=2, contacts=3, fluid=4, constraints=5, bounds=6,
                  velocity=7, viscosity=8, groups=9)

    def __init__(self, max_fluid: int = 2600, **tuning):
        self.lib = load()
        self.h = self.lib.o1_create(max_fluid)
        for k, v in tuning.items():
            self.set_param(k, v)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.o1_destroy(self.h)
            self.h = None

    def set_param(self, name: str, v: float) -> None:
        if self.lib.o1_set_param(self.h, name.encode(), float(v)) != 0:
            raise KeyError(name)

    def add_solid_cube(self, cx, cy, cz, n=7, spacing=0.18, mass=0.08) -> None:
        self.lib.o1_add_solid_cube(self.h, cx, cy, cz, n, spacing, mass)

    def emit_fluid(self, pos3, vel3, mass=0.03) -> None:
        p = np.ascontiguousarray(pos3, dtype=np.float64).reshape(-1, 3)
        v = np.ascontiguousarray(vel3, dtype=np.float64).reshape(-1, 3)
        self.lib.o1_emit_fluid(self.h, p.shape[0], _d(p), _d(v), mass)

    def sizes(self) -> dict:
        out = (C.c_int * 7)()
        self.lib.o1_sizes(self.h, out)
        return dict(zip(("solidCount", "capacity", "tableSize", "numCons", "maxPairs", "fluidNext",
                         "pairCount"), list(out)))

    def get(self, name: str) -> np.ndarray:
        n = self.lib.o1_len(self.h, name.encode())
        if n < 0:
            raise KeyError(name)
        dt = np.float32 if name in self.F32 else np.int32 if name in self.I32 else \
            np.uint8 if name in self.U8 else np.float64
        a = np.empty(n, dt)
        self.lib.o1_get(self.h, name.encode(), a.ctypes.data_as(C.c_void_p))
        return a

    def set(self, name: str, a: np.ndarray) -> None:
        n = self.lib.o1_len(self.h, name.encode())
        dt = np.float32 if name in self.F32 else np.int32 if name in self.I32 else \
            np.uint8 if name in self.U8 else np.float64
        b = np.ascontiguousarray(a, dtype=dt).reshape(-1)
        assert b.size == n, (name, b.size, n)
        self.lib.o1_set(self.h, name.encode(), b.ctypes.data_as(C.c_void_p))

    def step(self, dt: float, substeps: int) -> None:
        self.lib.o1_step(self.h, dt, substeps)

    def run_pass(self, name: str, h: float = 1 / 300) -> None:
        self.lib.o1_pass(self.h, self.PASSES[name], h)

    def cut(self, o, d1, d2) -> int:
        return self.lib.o1_cut(self.h, _d3(o), _d3(d1), _d3(d2))

    def pick(self, o, d, max_perp):
        t = C.c_double()
        i = self.lib.o1_pick(self.h, _d3(o), _d3(d), max_perp, C.byref(t))
        return i, t.value

    def set_grabs(self, idx, xyz) -> None:
        ix = np.ascontiguousarray(idx, dtype=np.int32)
        p = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1)
        self.lib.o1_set_grabs(self.h, ix.size, ix.ctypes.data_as(C.POINTER(C.c_int)), _d(p))

    def reset_solid(self) -> None:
        self.lib.o1_reset_solid(self.h)

    def clear_fluid(self) -> None:
        self.lib.o1_clear_fluid(self.h)

    def fluid_count(self) -> int:
        return self.lib.o1_fluid_count(self.h)


class O2:
    """Restatement of the WGSL kernels in GpuSim.encode order; precision 0 =
    float, 1 = double."""

    def __init__(self, desc, params, precision: int = 0):
        self.lib = load()
        self.h = self.lib.o2_create(C.byref(desc), C.byref(params), precision)
        if not self.h:
            raise ValueError("invalid scene descriptor")
        self.precision = precision
        from fluidphysics_b200 import _lib as L  # struct layouts only (no library load)
        info = L.Info()
        self.lib.o2_info(self.h, C.byref(info))
        self.info = info

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.o2_destroy(self.h)
            self.h = None

    def refresh_info(self):
        self.lib.o2_info(self.h, C.byref(self.info))
        return self.info

    def set_params(self, p) -> None:
        self.lib.o2_set_params(self.h, C.byref(p))

    def step(self, dt, substeps) -> None:
        self.lib.o2_step(self.h, dt, substeps)

    def frame(self) -> None:
        self.lib.o2_frame(self.h)

    def substep_partial(self, h, last) -> None:
        self.lib.o2_substep_partial(self.h, h, last)

    def rebuild_grid(self) -> None:
        self.lib.o2_rebuild_grid(self.h)

    def run_pass(self, pass_id: int, h: float = 1 / 300) -> None:
        """One pass (UPBD_PASS_* id) on the current state."""
        if self.lib.o2_run_pass(self.h, pass_id, h) != 0:
            raise ValueError(f"pass {pass_id} cannot run alone")

    def read_state(self) -> dict:
        n = self.info.total
        pos, prev, vel = (np.empty((n, 4)) for _ in range(3))
        dens = np.empty((n, 2))
        flags = np.empty(n, np.uint32)
        self.lib.o2_read_state(self.h, pos.ctypes.data_as(C.POINTER(C.c_double)),
                               prev.ctypes.data_as(C.POINTER(C.c_double)),
                               vel.ctypes.data_as(C.POINTER(C.c_double)),
                               dens.ctypes.data_as(C.POINTER(C.c_double)),
                               flags.ctypes.data_as(C.POINTER(C.c_uint32)))
        return dict(pos=pos, prev=prev, vel=vel, density=dens, flags=flags)

    def write_state(self, pos=None, prev=None, vel=None, density=None, flags=None) -> None:
        keep = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (pos, prev, vel, density)]
        fl = None if flags is None else np.ascontiguousarray(flags, dtype=np.uint32)
        ptrs = [None if a is None else a.ctypes.data_as(C.POINTER(C.c_double)) for a in keep]
        self.lib.o2_write_state(self.h, *ptrs, None if fl is None else fl.ctypes.data_as(C.POINTER(C.c_uint32)))

    def read_delta(self) -> np.ndarray:
        d = np.empty((self.info.total, 4))
        self.lib.o2_read_delta(self.h, d.ctypes.data_as(C.POINTER(C.c_double)))
        return d

    def read_constraints(self):
        c = np.empty((self.info.num_cons, 4), np.uint32)
        r = np.empty(self.info.num_cons)
        self.lib.o2_read_constraints(self.h, c.ctypes.data_as(C.POINTER(C.c_uint32)),
                                     r.ctypes.data_as(C.POINTER(C.c_double)))
        return c, r

    def write_constraints(self, cons) -> None:
        c = np.ascontiguousarray(cons, dtype=np.uint32)
        self.lib.o2_write_constraints(self.h, c.ctypes.data_as(C.POINTER(C.c_uint32)))

    # single passes outside o2_run_pass's set (the oracle's own ids)
    PASS_X = dict(INTEGRATE=101, COLLECT=102, SOLID_SOLVE=103, APPLY_SOLID=104, SOLVE_TETS=105,
                  APPLY_SOLID_CONTACTS=106, SOLID_CONTACTS=107, BOND_UPDATE=108, TET_UPDATE=109,
                  SOLID_VISC=110, SOLID_VISC_APPLY=111, EMIT=112)

    def run_pass_x(self, name: str, h: float, grab_delta_sub=None) -> None:
        g = None if grab_delta_sub is None else (C.c_float * 3)(*[float(x) for x in grab_delta_sub])
        if self.lib.o2_run_pass_x(self.h, self.PASS_X[name], h, g) != 0:
            raise ValueError(f"pass {name} cannot run alone")

    def write_delta(self, d4) -> None:
        d = np.ascontiguousarray(d4, dtype=np.float64)
        self.lib.o2_write_delta(self.h, d.ctypes.data_as(C.POINTER(C.c_double)))

    def read_contact_cache(self):
        S = self.info.solid_n
        cc = np.empty(S, np.uint32)
        cl = np.empty(S * 40, np.uint32)
        self.lib.o2_read_contact_cache(self.h, cc.ctypes.data_as(C.POINTER(C.c_uint32)),
                                       cl.ctypes.data_as(C.POINTER(C.c_uint32)))
        return cc, cl

    def write_contact_cache(self, ccount, clist) -> None:
        cc = np.ascontiguousarray(ccount, dtype=np.uint32)
        cl = np.ascontiguousarray(clist, dtype=np.uint32)
        self.lib.o2_write_contact_cache(self.h, cc.ctypes.data_as(C.POINTER(C.c_uint32)),
                                        cl.ctypes.data_as(C.POINTER(C.c_uint32)))

    def write_tets(self, tets5) -> None:
        t = np.ascontiguousarray(tets5, dtype=np.uint32)
        self.lib.o2_write_tets(self.h, t.ctypes.data_as(C.POINTER(C.c_uint32)))

    def read_adjacency(self) -> np.ndarray:
        a = np.empty(self.info.solid_n + 1 + 2 * self.info.num_cons, np.uint32)
        self.lib.o2_read_adjacency(self.h, a.ctypes.data_as(C.POINTER(C.c_uint32)))
        return a

    def read_grid(self):
        T = self.info.table_size
        counts = np.empty(T, np.uint32)
        offs = np.empty(T + 1, np.uint32)
        ent = np.empty(self.info.total, np.uint32)
        u = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint32))
        self.lib.o2_read_grid(self.h, u(counts), u(offs), u(ent))
        return counts, offs, ent[: offs[T]].copy()

    def read_tets(self) -> np.ndarray:
        t = np.empty((self.info.num_tets, 5), np.uint32)
        self.lib.o2_read_tets(self.h, t.ctypes.data_as(C.POINTER(C.c_uint32)))
        return t

    def read_tet_adjacency(self) -> np.ndarray:
        a = np.empty(self.info.solid_n + 1 + 4 * self.info.num_tets, np.uint32)
        self.lib.o2_read_tet_adjacency(self.h, a.ctypes.data_as(C.POINTER(C.c_uint32)))
        return a

    def emit(self, count, pos, dir, side, up, speed, phase) -> None:
        self.lib.o2_emit(self.h, count, _f3(pos), _f3(dir), _f3(side), _f3(up), speed, phase)

    def emit_particles(self, pos3, vel3, mass) -> None:
        p = np.ascontiguousarray(pos3, dtype=np.float32).reshape(-1, 3)
        v = np.ascontiguousarray(vel3, dtype=np.float32).reshape(-1, 3)
        self.lib.o2_emit_particles(self.h, p.shape[0], p.ctypes.data_as(C.POINTER(C.c_float)),
                                   v.ctypes.data_as(C.POINTER(C.c_float)), mass)

    def slice_now(self, o, d1, d2) -> int:
        return int(self.lib.o2_slice_now(self.h, _d3(o), _d3(d1), _d3(d2)))

    def slice(self, o, d1, d2) -> None:
        self.lib.o2_slice(self.h, _d3(o), _d3(d1), _d3(d2))

    def pick(self, ro, rd, max_perp):
        t = C.c_double()
        i = self.lib.o2_pick(self.h, _d3(ro), _d3(rd), max_perp, C.byref(t))
        return i, t.value

    def grab_select(self, c, r, lattice=0xFFFF) -> None:
        self.lib.o2_grab_select(self.h, _f3(c), r, lattice)

    def grab_indices(self, idx, weight=None, targets=None) -> None:
        ix = np.ascontiguousarray(idx, dtype=np.uint32)
        w = None if weight is None else np.ascontiguousarray(weight, dtype=np.float32)
        t = None if targets is None else np.ascontiguousarray(targets, dtype=np.float32).reshape(-1)
        fp = lambda a: None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))
        self.lib.o2_grab_indices(self.h, ix.ctypes.data_as(C.POINTER(C.c_uint32)), ix.size, fp(w), fp(t))

    def grab_move(self, d) -> None:
        self.lib.o2_grab_move(self.h, _f3(d))

    def release(self) -> None:
        self.lib.o2_release(self.h)

    def drain(self) -> None:
        self.lib.o2_drain(self.h)

    def active_count(self) -> int:
        return int(self.lib.o2_active_count(self.h))

    def reset_solid(self) -> None:
        self.lib.o2_reset_solid(self.h)

    def groups(self) -> np.ndarray:
        g = np.empty(self.info.solid_n, np.int32)
        self.lib.o2_groups(self.h, g.ctypes.data_as(C.POINTER(C.c_int32)))
        return g

    def health(self) -> int:
        return int(self.lib.o2_health(self.h))

    def fluid_next(self) -> int:
        return int(self.lib.o2_fluid_next(self.h))


def o1_from_scene(scene, tuning_from_params: bool = True) -> O1:
    """An O1 solver holding the same scene as `scene` (body lattice + fluid),
    with the scene's constants mapped onto Solver's tuning fields."""
    d, p = scene.desc, scene.params
    o = O1(d.max_fluid)
    if tuning_from_params:
        for k, v in dict(gravity=p.gravity, solidRadius=p.solid_radius, fluidRadius=p.fluid_radius,
                         compliance=p.compliance, plasticThreshold=p.plastic_threshold,
                         plasticRate=p.plastic_rate, breakStrain=p.break_strain, fluidH=p.fluid_h,
                         restDensity=p.rest_density, stiffness=p.stiffness,
                         nearStiffness=p.near_stiffness, viscosity=p.viscosity,
                         solidDamping=p.damp_solid, fluidDamping=p.damp_fluid,
                         floorFrictionSolid=p.friction_solid, floorFrictionFluid=p.friction_fluid,
                         wallX=p.wall_x, wallZ=p.wall_z, wallHeight=p.wall_h, wallHalfThick=p.wall_t,
                         cullRadius=p.cull_r, maxSpeed=p.max_speed, grabStiffness=p.grab_k,
                         cellSize=p.cell_size).items():
            o.set_param(k, v)
        o.set_param("tableSizeOverride", d.table_size)
    o.add_solid_cube(d.cube_center[0], d.cube_center[1], d.cube_center[2], d.solid_dim, d.spacing,
                     d.solid_mass)
    if len(scene.fluid_pos):
        o.emit_fluid(scene.fluid_pos.astype(np.float64), scene.fluid_vel.astype(np.float64),
                     scene.fluid_mass)
    return o


def o2_from_scene(scene, precision: int = 0) -> O2:
    o = O2(scene.desc, scene.params, precision)
    if len(scene.fluid_pos):
        o.emit_particles(scene.fluid_pos, scene.fluid_vel, scene.fluid_mass)
    return o
