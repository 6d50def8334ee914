"""The allocation-free hash-grid build against the pooled one.

upbd_grid_build_noalloc exists for callers that cannot allocate device
memory: hosts whose GPU memory is owned and accounted by an embedding runtime
that refuses foreign cudaMalloc calls, and frame loops that must not stall on
an allocation. Its scratch is a fixed array inside the library, shared by
every call. This test feeds both entry points the same device arrays and
requires identical grids (bit for bit, as every integer output here) on two
consecutive calls with different sizes, so stale scratch from the first call
would show up in the second. It runs last in the suite (file name) and also
passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from fluidphysics_b200 import _lib as L
from fluidphysics_b200 import scenes as S

pytestmark = pytest.mark.gpu


def _grid(torch, lib, fn, pos, flags, n, T, cell, with_counts=True):
    dev = pos.device
    off = torch.full((T + 1,), -1, dtype=torch.int32, device=dev)
    ent = torch.full((max(n, 1),), -1, dtype=torch.int32, device=dev)
    cnt = torch.full((T,), -1, dtype=torch.int32, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = fn(C.c_void_p(pos.data_ptr()), C.c_void_p(flags.data_ptr()), n, T, cell,
            C.c_void_p(cnt.data_ptr()) if with_counts else None,
            C.c_void_p(off.data_ptr()), C.c_void_p(ent.data_ptr()), stream)
    assert rc == 0, lib.upbd_last_error(None)
    torch.cuda.synchronize()
    o = off.cpu().numpy().view(np.uint32)
    return o, ent.cpu().numpy().view(np.uint32)[: o[-1]], cnt.cpu().numpy().view(np.uint32)


def _inputs(torch, scene, jitter_seed):
    p = np.zeros((scene.total, 4), np.float32)
    d = scene.desc
    k = np.arange(scene.solid_n)
    n = d.solid_dim
    p[: scene.solid_n, 0] = d.cube_center[0] + (k // (n * n) - (n - 1) / 2) * d.spacing
    p[: scene.solid_n, 1] = d.cube_center[1] + ((k // n) % n - (n - 1) / 2) * d.spacing
    p[: scene.solid_n, 2] = d.cube_center[2] + (k % n - (n - 1) / 2) * d.spacing
    p[scene.solid_n:, :3] = scene.fluid_pos
    rng = np.random.default_rng(jitter_seed)
    p[:, :3] += rng.normal(scale=0.01, size=(scene.total, 3)).astype(np.float32)
    flags = np.ones(scene.total, np.int32)
    flags[rng.random(scene.total) < 0.05] = 0  # some inactive slots
    return (torch.from_numpy(p).cuda(), torch.from_numpy(flags).cuda())


def test_noalloc_grid_matches_pooled_build_twice():
    torch = pytest.importorskip("torch")
    lib = L.load()
    big, small = S.gpu_default(frames=1), S.cpu_scene()
    for scene, seed in ((big, 1), (small, 2)):  # two calls in a row, sizes shrink
        pos, flags = _inputs(torch, scene, seed)
        n, T, cell = scene.total, scene.desc.table_size, scene.params.cell_size
        ref = _grid(torch, lib, lib.upbd_grid_build, pos, flags, n, T, cell)
        got = _grid(torch, lib, lib.upbd_grid_build_noalloc, pos, flags, n, T, cell)
        for a, b, what in zip(got, ref, ("offsets", "entries", "counts")):
            assert np.array_equal(a, b), f"{what} differ (n={n}, T={T})"
        assert got[0][-1] == int(flags.sum().item())
        # counts are optional: without them the offsets and members are the same
        off, ent, cnt = _grid(torch, lib, lib.upbd_grid_build_noalloc, pos, flags, n, T, cell, with_counts=False)
        assert np.array_equal(off, ref[0]) and np.array_equal(ent, ref[1])
        assert (cnt.view(np.int32) == -1).all(), "counts written although none were asked for"


def test_noalloc_rejects_sizes_beyond_its_array():
    lib = L.load()
    rc = lib.upbd_grid_build_noalloc(C.c_void_p(1), C.c_void_p(1), (1 << 18) + 1, 1 << 10, 0.1, None,
                                     C.c_void_p(1), C.c_void_p(1), None)
    assert rc == -8  # UPBD_ERR_CAPACITY, before any device work
    assert b"262144" in lib.upbd_last_error(None)
