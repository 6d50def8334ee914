"""Seeded synthetic scenes for the unified-particle step.

Scene parameters follow the reference's own derivations:
  - `derive_opts` is deriveOpts (src/gpu/main.js:30-54): one particle radius
    drives spacing, H, cell size, masses, stiffness and the table size;
  - `solver_params` are the CPU solver's constants (src/solver.js:14-36,50).

Scenes (sizes from the reference: README.md:12-13, src/gpu/sim.js:20-33):
  cpu_scene      7^3 body (343) + 2,600 fluid, the CPU solver's scene
  gpu_default    20^3 body (8,000; 93,556 constraints) + 65,536 fluid,
                 one wedge slice through the body centre at frame 60
  large          24^3 body (13,824) + 262,144 fluid, a hose of 120
                 particles/frame and 64 grabbed body particles on a
                 sinusoidal path
  batch_scenes   many independent scenes of uneven size (see batch.py)

Fluid starts as a jittered lattice block (uniform jitter of +-10% of the
spacing per axis, numpy PCG64 seeded per scene), so every run is
reproducible bit for bit. There are no datasets: the reference ships none.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


def js_round(x: float) -> int:
    """Math.round (half up)."""
    return int(math.floor(x + 0.5))


def derive_opts(dim: int, max_fluid: int, radius_mm: float) -> dict:
    """deriveOpts(dim, maxFluid, radiusMm), src/gpu/main.js:30-54."""
    r = radius_mm / 1000
    H = 2.6 * r
    spacing = 1.91 * r
    return dict(
        SOLID_DIM=dim,
        MAX_FLUID=max_fluid,
        TABLE=max(1 << 18, 1 << math.ceil(math.log2(2 * (max_fluid + dim ** 3)))),
        substeps=min(10, max(5, js_round(0.2 / r))),
        spacing=spacing,
        solidMass=100 * r ** 3,
        fluidMass=12 * r ** 3,
        cubeCenter=[0, (dim - 1) * spacing / 2 + 0.5, 0],
        params=dict(
            solidRadius=r, fluidRadius=r, fluidH=H, cellSize=H,
            stiffness=0.0015 * (H / 0.13), nearStiffness=0.006 * (H / 0.13),
        ),
    )


# camelCase (reference) -> snake_case (C ABI)
PARAM_NAMES = {
    "h": "h", "gravity": "gravity", "solidRadius": "solid_radius", "fluidRadius": "fluid_radius",
    "cellSize": "cell_size", "fluidH": "fluid_h", "restDensity": "rest_density",
    "stiffness": "stiffness", "nearStiffness": "near_stiffness", "viscosity": "viscosity",
    "compliance": "compliance", "omega": "omega", "plasticThreshold": "plastic_threshold",
    "plasticRate": "plastic_rate", "tearGap": "tear_gap", "maxSpeed": "max_speed",
    "wallX": "wall_x", "wallZ": "wall_z", "wallH": "wall_h", "wallT": "wall_t", "cullR": "cull_r",
    "dampSolid": "damp_solid", "dampFluid": "damp_fluid", "frictionSolid": "friction_solid",
    "frictionFluid": "friction_fluid", "grabK": "grab_k", "sleepSpeed": "sleep_speed",
    "solidViscosity": "solid_viscosity", "breakStrain": "break_strain",
    "contactScale": "contact_scale", "tearMode": "tear_mode", "plasticClamp": "plastic_clamp",
}


# GpuSim DEFAULTS, src/gpu/sim.js:20-63, in the reference's own keys (the
# schema of a snapshot's `opts`)
GPU_DEFAULTS = {
    "SOLID_DIM": 20, "SOLID_DIM2": None, "MAX_FLUID": 65536, "TABLE": 1 << 18,
    "spacing": 0.065, "solidMass": 0.004, "fluidMass": 0.0015, "cubeCenter": [0, 1.8, 0],
    "substeps": 5, "solidIters": 8,
    "params": {
        "h": 1 / 300, "gravity": -10, "solidRadius": 0.034, "fluidRadius": 0.05, "cellSize": 0.13,
        "fluidH": 0.13, "restDensity": 3.0, "stiffness": 0.0015, "nearStiffness": 0.006,
        "viscosity": 0.3, "compliance": 5e-4, "omega": 1.5, "plasticThreshold": 0.38,
        "plasticRate": 0.04, "tearGap": 1.3, "maxSpeed": 14, "wallX": 3.5, "wallZ": 3.5,
        "wallH": 0.92, "wallT": 0.07, "cullR": 7.0, "dampSolid": 1.2, "dampFluid": 0.6,
        "frictionSolid": 0.4, "frictionFluid": 0.04, "grabK": 0.6, "sleepSpeed": 0,
        "solidViscosity": 0,
    },
}


def merge_gpu_opts(opts: dict) -> dict:
    """The options object of the GpuSim constructor (src/gpu/sim.js:78-84):
    DEFAULTS overlaid with opts, params merged the same way, and SOLID_DIM2
    resolved (opts' value, else the companion cube's edge (SOLID_DIM - 1) /
    cbrt(20), rounded, + 1, at least 2) — what a snapshot's `opts` holds,
    with the keys in the reference's order."""
    o = {**GPU_DEFAULTS, **{k: v for k, v in opts.items() if k != "params"}}
    o["params"] = {**GPU_DEFAULTS["params"], **opts.get("params", {})}
    dim2 = o.get("SOLID_DIM2")
    if dim2 is None:
        dim2 = max(2, js_round((o["SOLID_DIM"] - 1) / 20 ** (1 / 3)) + 1)
    o["SOLID_DIM2"] = int(dim2)
    return o


def default_desc() -> L.SceneDesc:
    d = L.SceneDesc()
    _fill_default_desc(d)
    return d


def _fill_default_desc(d: L.SceneDesc) -> None:
    # GpuSim DEFAULTS, src/gpu/sim.js:20-33 (mirrors upbd_default_desc)
    d.solid_dim, d.solid_dim2, d.max_fluid, d.table_size = 20, 0, 65536, 1 << 18
    d.substeps, d.solid_iters, d.features, d.device = 5, 8, 0, 0
    d.spacing, d.solid_mass, d.fluid_mass = 0.065, 0.004, 0.0015
    d.cube_center[:] = [0, 1.8, 0]
    d.cube2_center[:] = [1.1, 0.5, 0.7]


def default_params() -> L.Params:
    """GpuSim DEFAULTS.params, src/gpu/sim.js:34-63 (mirrors upbd_default_params)."""
    p = L.Params()
    vals = dict(h=1 / 300, gravity=-10, solid_radius=0.034, fluid_radius=0.05, cell_size=0.13,
                fluid_h=0.13, rest_density=3.0, stiffness=0.0015, near_stiffness=0.006,
                viscosity=0.3, compliance=5e-4, omega=1.5, plastic_threshold=0.38,
                plastic_rate=0.04, tear_gap=1.3, max_speed=14, wall_x=3.5, wall_z=3.5,
                wall_h=0.92, wall_t=0.07, cull_r=7.0, damp_solid=1.2, damp_fluid=0.6,
                friction_solid=0.4, friction_fluid=0.04, grab_k=0.6, sleep_speed=0,
                solid_viscosity=0, break_strain=2.6, contact_scale=0.5)
    for k, v in vals.items():
        setattr(p, k, float(v))
    p.tear_mode = 0
    p.plastic_clamp = 1
    return p


def set_params(p: L.Params, overrides: dict) -> L.Params:
    for k, v in overrides.items():
        name = PARAM_NAMES.get(k, k)
        if name in ("tear_mode", "plastic_clamp"):
            setattr(p, name, int(v))
        else:
            setattr(p, name, float(v))
    return p


def desc_from_opts(opts: dict, *, solid_iters: int | None = None, substeps: int | None = None,
                   features: int = 0, device: int = 0) -> L.SceneDesc:
    """GpuSim constructor options (src/gpu/sim.js:77-95) -> upbd_scene_desc."""
    d = L.SceneDesc()
    _fill_default_desc(d)
    d.solid_dim = int(opts.get("SOLID_DIM", 20))
    dim2 = opts.get("SOLID_DIM2", None)
    if dim2 is None:  # companion cube: edge / cbrt(20), src/gpu/sim.js:83
        dim2 = max(2, js_round((d.solid_dim - 1) / 20 ** (1 / 3)) + 1)
    d.solid_dim2 = int(dim2)
    d.max_fluid = int(opts.get("MAX_FLUID", 65536))
    d.table_size = int(opts.get("TABLE", 1 << 18))
    d.substeps = int(substeps if substeps is not None else opts.get("substeps", 5))
    d.solid_iters = int(solid_iters if solid_iters is not None else opts.get("solidIters", 8))
    d.features = int(features)
    d.device = int(device)
    d.spacing = float(opts.get("spacing", 0.065))
    d.solid_mass = float(opts.get("solidMass", 0.004))
    d.fluid_mass = float(opts.get("fluidMass", 0.0015))
    d.cube_center[:] = [float(x) for x in opts.get("cubeCenter", [0, 1.8, 0])]
    n2 = d.solid_dim2
    d.cube2_center[:] = [1.1, (n2 - 1) * d.spacing / 2 + 0.5, 0.7]  # src/gpu/sim.js:171
    return d


def jittered_block(nx: int, ny: int, nz: int, spacing: float, y0: float, seed: int,
                   jitter: float = 0.1, center_xz=(0.0, 0.0)) -> np.ndarray:
    """A lattice block of fluid centred on x/z with its lowest layer at y0,
    each coordinate jittered by U(-jitter, +jitter) * spacing. float32 (n, 3)."""
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    p = np.stack([ix, iy, iz], axis=-1).reshape(-1, 3).astype(np.float64) * spacing
    p[:, 0] += center_xz[0] - (nx - 1) * spacing / 2
    p[:, 1] += y0
    p[:, 2] += center_xz[1] - (nz - 1) * spacing / 2
    rng = np.random.default_rng(seed)
    p += rng.uniform(-jitter, jitter, size=p.shape) * spacing
    return p.astype(np.float32)


def wedge_through(center, seed: int, dist: float = 10.0, half_width: float = 3.0):
    """A slice wedge whose plane passes through `center` with a normal drawn
    uniformly on the sphere: o = c + dist*u, d1,2 = normalize(c - o +- hw*w),
    u perpendicular to n, w = n x u, so d1 x d2 is parallel to n."""
    rng = np.random.default_rng(seed)
    n = rng.normal(size=3)
    n /= np.linalg.norm(n)
    a = np.array([1.0, 0, 0]) if abs(n[0]) < 0.9 else np.array([0, 1.0, 0])
    u = np.cross(n, a)
    u /= np.linalg.norm(u)
    w = np.cross(n, u)
    c = np.asarray(center, dtype=np.float64)
    o = c + dist * u
    d1 = c - o + half_width * w
    d2 = c - o - half_width * w
    return o, d1 / np.linalg.norm(d1), d2 / np.linalg.norm(d2)


@dataclass
class Scene:
    """A fully specified workload: descriptor, constants, initial fluid and
    the per-frame tool script."""
    name: str
    desc: L.SceneDesc
    params: L.Params
    fluid_pos: np.ndarray          # float32 (n, 3)
    fluid_vel: np.ndarray          # float32 (n, 3)
    fluid_mass: float
    dt: float
    substeps: int
    frames: int
    slice_frame: int = -1
    wedge: tuple | None = None
    hose_per_frame: int = 0
    hose_seed: int = 0
    grab_count: int = 0
    grab_amp: float = 0.0
    grab_freq_hz: float = 0.0
    extra: dict = field(default_factory=dict)

    @property
    def solid_n(self) -> int:
        return self.desc.solid_dim ** 3 + self.desc.solid_dim2 ** 3

    @property
    def total(self) -> int:
        return self.solid_n + self.desc.max_fluid


def solver_params(gravity: float = -9.8) -> L.Params:
    """The CPU solver's constants (src/solver.js:14-36,50) with its rules
    where they are independent of solve order: strain tearing, unclamped
    plasticity, full mass-weighted contact push."""
    p = default_params()
    set_params(p, dict(h=1 / 300, gravity=gravity, solidRadius=0.09, fluidRadius=0.075,
                       cellSize=0.22, fluidH=0.19, restDensity=6.0, stiffness=0.002,
                       nearStiffness=0.008, viscosity=0.3, compliance=2.5e-4,
                       plasticThreshold=0.32, plasticRate=0.04, breakStrain=2.6,
                       maxSpeed=14.0, wallX=3.5, wallZ=3.5, wallH=0.92, wallT=0.07, cullR=7.0,
                       dampSolid=1.2, dampFluid=0.6, frictionSolid=0.4, frictionFluid=0.04,
                       grabK=0.3, tearMode=1, plasticClamp=0, contactScale=1.0))
    return p


def cpu_scene(gravity: float = -9.8, seed: int = 1, iters: int = 3, frames: int = 120) -> Scene:
    """The CPU solver's own scene: new Solver({maxFluid: 2600}) +
    addSolidCube(0, 2.0, 0, 7, 0.18) (src/main.js:8-9); 2,600 fluid on a
    20x10x13 block at 2.2*r_f spacing, lowest layer at y = 2.8."""
    d = L.SceneDesc()
    _fill_default_desc(d)
    d.solid_dim, d.solid_dim2, d.max_fluid = 7, 0, 2600
    n = 7 ** 3 + 2600
    d.table_size = 1 << math.ceil(math.log2(2 * n))  # src/solver.js:51
    d.substeps, d.solid_iters = 5, iters
    d.spacing, d.solid_mass, d.fluid_mass = 0.18, 0.08, 0.03
    d.cube_center[:] = [0.0, 2.0, 0.0]
    p = solver_params(gravity)
    fp = jittered_block(20, 10, 13, 2.2 * 0.075, 2.8, seed)
    return Scene("cpu_scene", d, p, fp, np.zeros_like(fp), 0.03, 1 / 60, 5, frames)


def gpu_scene(dim: int, max_fluid: int, radius_mm: float = 30, *, gravity: float = -9.8,
              iters: int = 3, substeps: int = 5, features: int = 0) -> tuple[L.SceneDesc, L.Params, dict]:
    opts = derive_opts(dim, max_fluid, radius_mm)
    opts["SOLID_DIM2"] = 0
    d = desc_from_opts(opts, solid_iters=iters, substeps=substeps, features=features)
    p = default_params()
    set_params(p, opts["params"])
    set_params(p, dict(gravity=gravity, h=1 / 60 / substeps))
    return d, p, opts


def gpu_default(gravity: float = -9.8, seed: int = 2, frames: int = 600, iters: int = 3) -> Scene:
    """20^3 body + 65,536 fluid at 30 mm (deriveOpts(20, 65536, 30)); 5
    substeps x 3 iterations; one slice through the body centre at frame 60."""
    d, p, opts = gpu_scene(20, 65536, 30, gravity=gravity, iters=iters)
    r = 0.030
    fp = jittered_block(64, 16, 64, 2.2 * r, 1.7, seed)
    c = opts["cubeCenter"]
    return Scene("gpu_default", d, p, fp, np.zeros_like(fp), opts["fluidMass"], 1 / 60, 5, frames,
                 slice_frame=60, wedge=wedge_through(c, seed))


def large(gravity: float = -9.8, seed: int = 3, frames: int = 600, iters: int = 3) -> Scene:
    """24^3 body + 262,144 fluid at 30 mm; hose 120/frame at 3 m/s from a
    seeded nozzle over the box top; 64 grabbed body particles moved on
    y0 + 0.3*sin(pi*t)."""
    d, p, opts = gpu_scene(24, 262144, 30, gravity=gravity, iters=iters)
    r = 0.030
    fp = jittered_block(64, 64, 64, 2.2 * r, 2.0, seed)
    return Scene("large", d, p, fp, np.zeros_like(fp), opts["fluidMass"], 1 / 60, 5, frames,
                 hose_per_frame=120, hose_seed=seed, grab_count=64, grab_amp=0.3, grab_freq_hz=0.5)


def hose_script(scene: Scene, frames: int):
    """Per-frame emit arguments (pos, dir, side, up, speed, phase): nozzle
    uniform on x,z in [-3.5, 3.5] at y = 3.0, aimed at a uniform point of
    the basin floor, 3 m/s; side/up as sprayStep builds them
    (src/gpu/main.js:441-452), phase advanced by count * golden angle."""
    rng = np.random.default_rng(scene.hose_seed)
    phase = 0.0
    out = []
    for _ in range(frames):
        nz = np.array([rng.uniform(-3.5, 3.5), 3.0, rng.uniform(-3.5, 3.5)])
        tgt = np.array([rng.uniform(-3.5, 3.5), 0.0, rng.uniform(-3.5, 3.5)])
        dr = tgt - nz
        dr /= np.linalg.norm(dr)
        side = np.cross(dr, [0.0, 1.0, 0.0])
        side /= np.linalg.norm(side)
        up = np.cross(side, dr)
        up /= np.linalg.norm(up)
        out.append((nz.astype(np.float32), dr.astype(np.float32), side.astype(np.float32),
                    up.astype(np.float32), 3.0, phase))
        phase = (phase + scene.hose_per_frame * 2.39996) % (2 * math.pi)
    return out


def grab_set(init_pos: np.ndarray, solid_n: int, dim: int, count: int) -> np.ndarray:
    """The `count` body particles nearest the centre of the lattice's top face
    (ties broken by index)."""
    p = init_pos[:solid_n, :3].astype(np.float64)
    top = p[:, 1].max()
    c = np.array([p[:, 0].mean(), top, p[:, 2].mean()])
    d2 = ((p - c) ** 2).sum(axis=1)
    order = np.lexsort((np.arange(solid_n), d2))
    return np.sort(order[:count]).astype(np.uint32)
