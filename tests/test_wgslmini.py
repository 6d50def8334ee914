"""The WGSL interpreter that executes the reference's kernels for the golden
vectors (tests/golden/wgslmini.py): its arithmetic follows WGSL's types.
Small kernels written here, no reference files needed."""
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import wgslmini as W  # noqa: E402

SRC = """
const K: u32 = 3u;
struct Params { a: f32, b: f32, v: vec4f, n: u32, }
@group(0) @binding(0) var<storage, read_write> outf: array<f32>;
@group(0) @binding(1) var<storage, read_write> outu: array<u32>;
@group(0) @binding(2) var<storage, read_write> outi: array<i32>;
@group(0) @binding(3) var<storage, read_write> rows: array<vec4f>;
@group(0) @binding(4) var<storage, read_write> ctr: array<atomic<u32>>;
@group(0) @binding(5) var<uniform> P: Params;

fn sq(x: f32) -> f32 { return x * x; }

@compute @workgroup_size(4)
fn main(@builtin(global_invocation_id) g: vec3u) {
  let i = g.x;
  if (i >= P.n) { return; }
  // f32: every operation rounds to float32
  outf[i] = P.a + P.b * f32(i);
  // u32 wraps, integer division truncates, shifts
  outu[i] = (0xffffffffu + i + 2u) * 3u / K + (1u << 4u);
  // i32: truncation toward zero, remainder with the dividend's sign, saturating conversion
  var s = -7 / 2 + (-7 % 3);
  s += i32(-3.9) + i32(1e20);
  outi[i] = s;
  // vectors, swizzles, component assignment, builtins
  var v = rows[i].xyz * 2.0;
  v.y = sqrt(sq(v.y));
  rows[i] = vec4f(v, length(vec2f(3.0, 4.0)) + select(0.0, 1.0, i == 1u));
  rows[i].w += dot(P.v.xyz, vec3f(1.0));
  atomicAdd(&ctr[0], i);
  atomicMax(&ctr[1], i * 10u);
}
"""


def test_wgsl_types_and_builtins():
    m = W.Module(SRC)
    outf = np.zeros(6, np.float32)
    outu = np.zeros(6, np.uint32)
    outi = np.zeros(6, np.int32)
    rows = np.arange(24, dtype=np.float32).reshape(6, 4) * np.float32(0.1)
    rows0 = rows.copy()
    ctr = np.zeros(2, np.uint32)
    for k, v in dict(outf=outf, outu=outu, outi=outi, rows=rows, ctr=ctr).items():
        m.bind(k, v)
    m.set_uniform("P", dict(a=0.1, b=0.3, v=[1.0, 2.0, 3.0, 4.0], n=5))
    m.dispatch("main", 2)  # 8 invocations, 5 active
    i = np.arange(5)
    want_f = np.float32(0.1) + np.float32(0.3) * i.astype(np.float32)
    assert np.array_equal(outf[:5], want_f.astype(np.float32)) and outf[5] == 0
    want_u = ((((0xFFFFFFFF + i + 2) & 0xFFFFFFFF) * 3 & 0xFFFFFFFF) // 3 + 16).astype(np.uint32)
    assert np.array_equal(outu[:5], want_u)
    assert np.all(outi[:5] == -3 + -1 + -3 + 2147483647)
    v = rows0[:5, :3] * np.float32(2.0)
    assert np.array_equal(rows[:5, :3], v)
    assert np.array_equal(rows[:5, 3], np.float32(5.0) + (i == 1) + np.float32(6.0))
    assert np.array_equal(rows[5], rows0[5])
    assert ctr[0] == 0 + 1 + 2 + 3 + 4 and ctr[1] == 40


def test_template_list_and_constants():
    m = W.Module("const A: u32 = 8u;\nconst B: u32 = A * A + 1u;\n"
                 "@group(0) @binding(0) var<storage, read_write> g: array<atomic<u32>>;\n"
                 "@compute @workgroup_size(1) fn f() { atomicStore(&g[0], B); }\n")
    g = np.zeros(1, np.uint32)
    m.bind("g", g)
    m.dispatch("f", 1)
    assert int(m.consts["B"]) == 65 and g[0] == 65
