"""CPU checks of the snapshot format helpers (no GPU): buffers are the
base64 of raw little-endian arrays, as the reference's b64encode writes them
(src/gpu/sim.js:3-15)."""
import base64

import numpy as np

from fluidphysics_b200 import snapshot as SN


def test_base64_buffers_round_trip():
    pos = np.arange(24, dtype=np.float32).reshape(6, 4) * 0.5
    s = SN._b64(pos.astype("<f4"))
    assert base64.b64decode(s) == pos.astype("<f4").tobytes()
    assert np.array_equal(SN._unb64(s, np.float32, 4), pos)
    flags = np.array([1, 3, 0, 2], np.uint32)
    assert np.array_equal(SN._unb64(SN._b64(flags), np.uint32), flags)


def test_js_btoa_compatible():
    # btoa over the byte string of a Uint8Array: standard alphabet with padding
    raw = bytes(range(7))
    assert SN._b64(np.frombuffer(raw, np.uint8)) == "AAECAwQFBg=="
