"""CPU checks of the frame server's host side: the served workload generator
and the error path of create (no GPU here)."""
import ctypes as C

import numpy as np
import pytest

from fluidphysics_b200 import _lib as L
from fluidphysics_b200 import server as SV


def test_served_requests_follow_the_workload():
    reqs = SV.served_requests(window_s=0.5, seed=5)
    again = SV.served_requests(window_s=0.5, seed=5)
    assert len(reqs) == len(again) and 40 <= len(reqs) <= 170  # Poisson(100)
    arr = np.array([r.arrival_s for r in reqs])
    assert np.all(np.diff(arr) > 0) and arr[-1] < 0.5
    tot = np.array([r.scene.total for r in reqs])
    assert tot.min() >= 1000 and tot.max() <= 262144 + 1
    for r, q in zip(reqs, again):
        assert r.frames == q.frames and 1 <= r.frames <= 60
        assert np.array_equal(r.scene.fluid_pos, q.scene.fluid_pos)
        body = r.scene.desc.solid_dim ** 3
        assert body <= 0.3 * r.scene.total * 1.35 + 30


def test_server_create_without_gpu_reports_error(built_libs):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    lib = L.load("product")
    d = L.ServerDesc()
    assert lib.upbd_server_default_desc(C.byref(d)) == 0
    assert d.substeps == 5 and d.builders >= 1
    h = C.c_void_p()
    assert lib.upbd_server_create(C.byref(d), C.byref(h)) in (-7, -3)
    assert lib.upbd_server_last_error(None)
    d.builders = 0
    assert lib.upbd_server_create(C.byref(d), C.byref(h)) == -1


def test_server_struct_layouts_match_c(tmp_path):
    import subprocess
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "upbd_server.h"\n'
                   'int main(){printf("%zu %zu %zu %zu %zu\\n", sizeof(upbd_server_desc), sizeof(upbd_request),'
                   ' sizeof(upbd_request_result), sizeof(upbd_server_stats), offsetof(upbd_request, arrival_s));'
                   ' return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", str(root / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got == [C.sizeof(L.ServerDesc), C.sizeof(L.Request), C.sizeof(L.RequestResult),
                   C.sizeof(L.ServerStats), L.Request.arrival_s.offset]
