"""Golden vectors for the GPU app's option table and snapshot files, made by
executing the reference's own code with tests/golden/jsmini.py:

  - deriveOpts (src/gpu/main.js:30-54): its function text is cut out of
    main.js (a browser module whose other parts need a DOM) and run as is,
    for the scene sizes the benchmarks and tests use and a spread of others;
  - new GpuSim(device, opts) (src/gpu/sim.js:76-97): the constructor runs
    unmodified on an object whose prototype is GpuSim's with _buildGpu (the
    WebGPU device setup) replaced by a no-op, so the option merge, the
    companion-cube size and _buildHostData all run as shipped;
  - GpuSim.snapshot (src/gpu/sim.js:493-513) with b64encode (sim.js:3-9):
    run unmodified on that object, its buffer reads (_readBuffer,
    _readBufferAt) answered from seeded host arrays instead of a GPU.

jsmini computes in IEEE doubles; `**`, Math.log2 and Math.cbrt use the
host's libm, which can differ from a browser engine's in the last ulp.

Run from the repository root, naming the reference checkout (its directory
holding src/gpu/main.js) with --ref or the UPBD_REFERENCE environment
variable:
    python tests/golden/make_golden_app.py --ref <path to the reference>
Writes tests/golden/app_js.json and tests/golden/app_js.npz (the host
arrays the snapshot was made from).
"""
from __future__ import annotations

import json
import math
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

import jsmini as J  # noqa: E402

# (dim, maxFluid, radiusMm): the GPU default scene, the large scene, the
# small scenes of the tests, and the UI's slider ends (dim 2..32, fluid up to
# 2^20, size 20..80 mm)
DERIVE_CASES = [(20, 65536, 30), (24, 262144, 30), (10, 4096, 40), (6, 64, 30), (5, 64, 40),
                (32, 1 << 20, 20), (2, 1024, 80), (12, 8192, 55), (16, 32768, 25), (28, 524288, 33)]
# the snapshot's scene: deriveOpts(5, 64, 40), small enough for a fixture
SNAP_CASE = (5, 64, 40)


def _reference_dir() -> Path:
    args = sys.argv[1:]
    if "--ref" in args and args.index("--ref") + 1 < len(args):
        ref = args[args.index("--ref") + 1]
    else:
        ref = os.environ.get("UPBD_REFERENCE", "")
    if not ref:
        raise SystemExit("name the reference checkout: --ref <dir> or UPBD_REFERENCE=<dir>")
    d = Path(ref)
    if not (d / "src" / "gpu" / "main.js").exists():
        raise SystemExit(f"{d} does not hold src/gpu/main.js")
    return d


def function_text(src: str, name: str) -> str:
    """The text of `function name(...) { ... }` in src, braces matched
    (strings and comments in it hold no braces)."""
    start = src.index(f"function {name}(")
    depth, i = 0, src.index("{", start)
    while True:
        ch = src[i]
        if ch == "{":
            depth += 1
        elif ch == "}":
            depth -= 1
            if depth == 0:
                return src[start:i + 1]
        i += 1


def js_to_py(v):
    """A JS value as plain Python, object key order kept (integral numbers
    as int, the way JSON.stringify prints them)."""
    if isinstance(v, J.JSObject):
        return {k: js_to_py(x) for k, x in v.props.items()}
    if isinstance(v, J.JSArray):
        return [js_to_py(x) for x in v.items]
    if isinstance(v, float):
        return int(v) if math.isfinite(v) and v == int(v) and abs(v) < 2 ** 53 else v
    if v is J.UNDEF:
        return None
    return v


def new_host_gpusim(GpuSim, opts_js):
    """new GpuSim(null, opts) with the WebGPU setup (_buildGpu) a no-op: the
    reference constructor and _buildHostData run unmodified."""
    proto = J.JSObject(proto=GpuSim.proto)
    proto.set("_buildGpu", J.Fn(lambda this, args: J.UNDEF))
    obj = J.JSObject(proto=proto)
    GpuSim.ctor.call(obj, [None, opts_js])
    return obj


def seeded_state(total: int, init_flags: np.ndarray, cons0: np.ndarray, tets0: np.ndarray, seed: int = 7):
    """Host arrays standing in for the GPU buffers of a running scene: every
    field filled with seeded values of the right kind (grab bits set on
    some particles, some constraints dead, some tets dead)."""
    rng = np.random.default_rng(seed)
    st = {
        "pos": rng.normal(0, 1.5, size=(total, 4)).astype(np.float32),
        "prev": rng.normal(0, 1.5, size=(total, 4)).astype(np.float32),
        "vel": rng.normal(0, 2.0, size=(total, 4)).astype(np.float32),
        "density": rng.uniform(0, 6, size=(total, 2)).astype(np.float32),
    }
    f = init_flags.astype(np.uint32).copy()
    f[rng.random(total) < 0.2] |= np.uint32(2)            # grabbed
    f[rng.random(total) < 0.1] &= np.uint32(0xFFFFFFFE)   # inactive
    st["flags"] = f
    c = cons0.reshape(-1, 4).astype(np.uint32).copy()
    c[:, 2] = rng.uniform(0.02, 0.2, size=len(c)).astype(np.float32).view(np.uint32)  # rest lengths
    c[:, 3] = (rng.random(len(c)) > 0.15).astype(np.uint32)                           # alive
    st["cons"] = c
    t = tets0.reshape(-1, 5).astype(np.uint32).copy()
    vol = rng.uniform(1e-5, 1e-3, size=len(t)).astype(np.float32)
    vol[rng.random(len(t)) < 0.2] *= -1                     # dead tets carry a negative volume
    t[:, 4] = vol.view(np.uint32)
    st["tets"] = t
    return st


def array_buffer(a: np.ndarray) -> J.ArrayBuffer:
    b = np.ascontiguousarray(a).tobytes()
    ab = J.ArrayBuffer(len(b))
    ab.buf[:] = b
    return ab


def main():
    ref = _reference_dir()
    main_js = (ref / "src/gpu/main.js").read_text()
    scope = J.run_source(function_text(main_js, "deriveOpts"))
    derive = scope.lookup("deriveOpts")
    out = {"generator": "tests/golden/make_golden_app.py",
           "reference_files": ["src/gpu/main.js", "src/gpu/sim.js"], "cases": {}}
    cases = []
    for dim, maxf, rmm in DERIVE_CASES:
        o = J.call(derive, J.UNDEF, [float(dim), float(maxf), float(rmm)])
        cases.append({"args": [dim, maxf, rmm], "opts": js_to_py(o)})
    out["cases"]["derive_opts"] = cases

    # ---- a GpuSim built from deriveOpts, its snapshot over seeded buffers
    mod = J.run_source((ref / "src/gpu/sim.js").read_text())
    GpuSim = mod.lookup("GpuSim")
    opts_js = J.call(derive, J.UNDEF, [float(x) for x in SNAP_CASE])
    gs = new_host_gpusim(GpuSim, opts_js)
    total = int(J.get_member(gs, "TOTAL"))
    num_cons = int(J.get_member(gs, "NUM_CONS"))
    num_tets = int(J.get_member(gs, "NUM_TETS"))
    init = J.get_member(gs, "init")
    st = seeded_state(total, J.typed_to_numpy(J.get_member(init, "flags")),
                      J.typed_to_numpy(J.get_member(init, "cons")),
                      J.typed_to_numpy(J.get_member(J.get_member(gs, "initTets"), "tetData")))
    bufs = {k: array_buffer(st[k]) for k in ("pos", "prev", "vel", "flags", "density", "cons")}
    ts_tets = 3  # any offset of the tet block inside gridS
    grid_s = np.zeros(ts_tets + num_tets * 5 + 7, np.uint32)
    grid_s[ts_tets:ts_tets + num_tets * 5] = st["tets"].reshape(-1)
    bufs["gridS"] = array_buffer(grid_s)
    J.set_member(gs, "buf", J.JSObject(dict(bufs)))
    J.set_member(gs, "TS_TETS", float(ts_tets))
    J.set_member(gs, "fluidNext", 37.0)

    def read_buffer(this, args):  # _readBuffer(buf, size) -> a then-able over its first size bytes
        b, size = args[0], int(J.to_number(args[1]))
        ab = J.ArrayBuffer(size)
        ab.buf[:] = b.buf[:size]
        then = J.JSObject()
        then.set("then", J.Fn(lambda t, a: J.call(a[0], J.UNDEF, [ab])))
        return then

    def read_buffer_at(this, args):  # _readBufferAt(buf, offset, size) -> ArrayBuffer
        b, off, size = args[0], int(J.to_number(args[1])), int(J.to_number(args[2]))
        ab = J.ArrayBuffer(size)
        ab.buf[:] = b.buf[off:off + size]
        return ab
    J.set_member(gs, "_readBuffer", J.Fn(read_buffer))
    J.set_member(gs, "_readBufferAt", J.Fn(read_buffer_at))
    snap = js_to_py(J.method(gs, "snapshot"))
    out["cases"]["snapshot"] = {
        "args": list(SNAP_CASE), "total": total, "num_cons": num_cons, "num_tets": num_tets,
        "constructed_opts": js_to_py(J.get_member(gs, "o")), "snapshot": snap}
    (HERE / "app_js.json").write_text(json.dumps(out, indent=1))
    np.savez_compressed(HERE / "app_js.npz", **st)
    print("wrote app_js.json / app_js.npz:", len(cases), "deriveOpts cases; snapshot of", total,
          "particles,", num_cons, "constraints,", num_tets, "tets")


if __name__ == "__main__":
    main()
