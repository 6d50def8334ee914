"""CPU checks of the scene batch's host side: the uneven workload generator,
the arena size query (no device needed) and the error path of create."""
import ctypes as C

import numpy as np
import pytest

from fluidphysics_b200 import _lib as L
from fluidphysics_b200 import batch as B


def test_batch_scenes_are_seeded_and_uneven():
    a = B.batch_scenes(24)
    b = B.batch_scenes(24)
    assert [s.desc.solid_dim for s in a] == [s.desc.solid_dim for s in b]
    for x, y in zip(a, b):
        assert np.array_equal(x.fluid_pos, y.fluid_pos)
    dims = np.array([s.desc.solid_dim for s in a])
    fl = np.array([s.desc.max_fluid for s in a])
    assert dims.min() >= 6 and dims.max() <= 20
    assert fl.min() >= 2048 and fl.max() < 65536
    assert len(set(dims.tolist())) > 4 and len(set(fl.tolist())) == len(fl)
    for s in a:
        assert s.fluid_pos.shape == (s.desc.max_fluid, 3)
        # the fluid block starts above the body's top layer
        top = s.desc.cube_center[1] + (s.desc.solid_dim - 1) * s.desc.spacing / 2
        assert s.fluid_pos[:, 1].min() > top


def test_scene_bytes_without_device(built_libs):
    small = B.batch_scene(6, 2048, 1)
    big = B.batch_scene(20, 65536, 2)
    nb_small = B.Batch.scene_bytes(small.desc)
    nb_big = B.Batch.scene_bytes(big.desc)
    assert 0 < nb_small < nb_big
    # per-particle state dominates the big scene: at least ~150 B per slot
    assert nb_big > 150 * (20 ** 3 + 65536)


def test_batch_create_without_gpu_reports_error(built_libs):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    lib = L.load("product")
    d = L.BatchDesc()
    assert lib.upbd_batch_default_desc(C.byref(d)) == 0
    assert (d.block_threads, d.ctas_per_sm, d.solid_iters) == (256, 8, 3)
    h = C.c_void_p()
    rc = lib.upbd_batch_create(C.byref(d), C.byref(h))
    assert rc in (-7, -3)
    assert lib.upbd_batch_last_error(None)
    d.block_threads = 100
    assert lib.upbd_batch_create(C.byref(d), C.byref(h)) == -1


def test_batch_struct_layouts_match_c(tmp_path):
    import subprocess
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "upbd_batch.h"\n'
                   'int main(){printf("%zu %zu %zu\\n", sizeof(upbd_batch_desc), sizeof(upbd_batch_info),'
                   ' offsetof(upbd_batch_info, block_threads)); return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", str(root / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got == [C.sizeof(L.BatchDesc), C.sizeof(L.BatchInfo), L.BatchInfo.block_threads.offset]
