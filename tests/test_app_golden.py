"""The GPU app's option table and snapshot format against golden vectors
that the reference's own code produced (tests/golden/make_golden_app.py runs
src/gpu/main.js's deriveOpts, the GpuSim constructor and GpuSim.snapshot
unmodified under tests/golden/jsmini.py). CPU only."""
import json
from pathlib import Path

import numpy as np
import pytest

from fluidphysics_b200 import _lib as L
from fluidphysics_b200 import scenes as S
from fluidphysics_b200 import snapshot as SN

GOLD = Path(__file__).resolve().parent / "golden"
J = json.loads((GOLD / "app_js.json").read_text())
NPZ = np.load(GOLD / "app_js.npz")
SNAP = J["cases"]["snapshot"]


def same(a, b) -> bool:
    """Equal JSON values (numbers as JavaScript has them) and equal key order
    at every level."""
    return json.dumps(SN.js_numbers(a)) == json.dumps(SN.js_numbers(b))


@pytest.mark.parametrize("case", J["cases"]["derive_opts"], ids=lambda c: "x".join(map(str, c["args"])))
def test_derive_opts_matches_main_js(case):
    """scenes.derive_opts equals deriveOpts (src/gpu/main.js:30-54) as run:
    every number bit for bit, keys in the same order."""
    dim, maxf, rmm = case["args"]
    got = S.derive_opts(dim, maxf, rmm)
    assert same(got, case["opts"]), (got, case["opts"])


def test_constructor_options_match_gpusim():
    """The options a GpuSim holds (and a snapshot carries): DEFAULTS merged
    with deriveOpts' output and the companion cube resolved, as the
    reference's constructor left them."""
    opts = S.derive_opts(*SNAP["args"])
    assert same(S.merge_gpu_opts(opts), SNAP["constructed_opts"])
    d = S.desc_from_opts(opts)
    assert d.solid_dim ** 3 + d.solid_dim2 ** 3 + d.max_fluid == SNAP["total"]


def _state():
    return {k: NPZ[k] for k in ("pos", "prev", "vel", "density", "flags")}


def test_snapshot_writer_matches_gpusim_snapshot():
    """snapshot_from_arrays writes, for the same buffers, exactly the object
    GpuSim.snapshot (src/gpu/sim.js:493-513) wrote: keys, order, options,
    counters and every base64 buffer."""
    snap = SN.snapshot_from_arrays(SNAP["constructed_opts"], SNAP["snapshot"]["fluidNext"],
                                   SNAP["num_cons"], _state(), NPZ["cons"], NPZ["tets"])
    assert same(snap, SNAP["snapshot"])


@pytest.mark.parametrize("keep_grabs", [False, True])
def test_snapshot_reader_decodes_gpusim_snapshot(keep_grabs):
    """decode_buffers reads the reference-written snapshot back to the exact
    buffers it was made from (grab bits cleared for a standalone restore,
    src/gpu/sim.js:526-531)."""
    a = SN.decode_buffers(SNAP["snapshot"], SNAP["total"], SNAP["num_tets"], keep_grabs)
    for k in ("pos", "prev", "vel", "density"):
        assert a[k].tobytes() == NPZ[k].tobytes(), k
    f = NPZ["flags"] if keep_grabs else NPZ["flags"] & np.uint32(~L.F_GRABBED & 0xFFFFFFFF)
    assert np.array_equal(a["flags"], f)
    assert np.any(NPZ["flags"] & L.F_GRABBED)
    assert np.array_equal(a["cons"], NPZ["cons"])
    assert np.array_equal(a["tets"], NPZ["tets"])


def test_snapshot_reader_rejects_other_sizes_and_skips_old_tets():
    with pytest.raises(ValueError):
        SN.decode_buffers(SNAP["snapshot"], SNAP["total"] + 1, SNAP["num_tets"])
    a = SN.decode_buffers(SNAP["snapshot"], SNAP["total"], SNAP["num_tets"] + 1)
    assert "tets" not in a  # a tet block of another size is not this scene's
