"""CPU checks of the C-ABI boundary: the library loads, exports every symbol
include/upbd.h declares, and its structs have the layout the ctypes mirror
assumes. No compute call is made (no GPU here)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from fluidphysics_b200 import _lib as L

ROOT = Path(__file__).resolve().parents[1]
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_symbols() -> set[str]:
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"^\s*(?:[\w\s\*]+?)\b(upbd_\w+)\s*\(", text, flags=re.M))
    return names


def test_headers_declare_entry_points():
    names = declared_symbols()
    for must in ("upbd_create", "upbd_step", "upbd_slice", "upbd_pick", "upbd_emit", "upbd_drain",
                 "upbd_grid_build", "upbd_read_grid"):
        assert must in names


@pytest.mark.parametrize("variant", ["product", "parity", "checked", "fp64"])
def test_library_exports_every_declared_symbol(built_libs, variant):
    lib = C.CDLL(str(L.lib_path(variant)))
    declared = sorted(declared_symbols())
    if variant == "fp64":  # the single-scene library only
        declared = [n for n in declared if not n.startswith(("upbd_batch_", "upbd_server_"))]
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes table covers the header exactly
    assert set(L.EXPORTED) == declared_symbols()


def test_grid_scratch_layout_alignment(tmp_path):
    """The stateless grid builds carve bucket counts, tickets, cells, the
    scatter, the scan tile counters and a params block (which holds a double)
    from one base. For every particle count, odd ones included, the params
    block starts on a 256-byte boundary and the regions do not overlap."""
    src = tmp_path / "lay.cpp"
    src.write_text(
        '#include <cstdio>\n#include "upbd_grid_layout.h"\nusing namespace upbd;\n'
        "int main(){ const size_t ns[] = {1, 2, 3, 2943, 73535, 73536, 262143, 262144};\n"
        " const size_t ts[] = {1, 1024, 8192, 262144, 1u << 20};\n"
        " for (size_t n : ns) for (size_t t : ts) { GridScratchLayout L = grid_scratch_layout(n, t, 304);\n"
        "  size_t tiles = (t + SCAN_TILE - 1) / SCAN_TILE;\n"
        "  printf(\"%zu %zu %zu %zu %zu %zu %zu %zu %zu %d\\n\", n, t, L.counts, L.ticket, L.cell, L.tmp, L.tiles,"
        " L.params, L.words, tile_words((int)tiles)); }\n return 0; }\n")
    exe = tmp_path / "lay"
    subprocess.run(["g++", "-std=c++17", "-I", str(ROOT / "fluidphysics_b200" / "csrc"), str(src), "-o", str(exe)],
                   check=True)
    rows = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    rows = [list(map(int, r.split())) for r in rows if r.strip()]
    assert len(rows) == 40
    for n, t, counts, ticket, cell, tmp, tiles, params, words, tw in rows:
        assert counts == 0 and ticket == t and cell == ticket + n and tmp == cell + n and tiles == tmp + n
        assert params >= tiles + tw and params % 64 == 0, (n, t)  # 256-byte boundary (double inside)
        assert words == params + 304 // 4


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "upbd.h"\n'
        "int main(){printf(\"%zu %zu %zu %zu %zu %zu\\n\", sizeof(upbd_scene_desc), sizeof(upbd_params),"
        " sizeof(upbd_info), sizeof(upbd_device_ptrs), offsetof(upbd_params, tear_mode),"
        " offsetof(upbd_scene_desc, spacing)); return 0;}\n")
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    got = [int(x) for x in out]
    want = [C.sizeof(L.SceneDesc), C.sizeof(L.Params), C.sizeof(L.Info), C.sizeof(L.DevicePtrs),
            L.Params.tear_mode.offset, L.SceneDesc.spacing.offset]
    assert got == want


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(L, "HERE", tmp_path)
    monkeypatch.setattr(L, "_libs", {})
    with pytest.raises(RuntimeError, match="not built"):
        L.load("product")


def test_create_without_gpu_reports_error(built_libs):
    """On a machine without a CUDA device the create call fails with a
    status code and a message, never a crash."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    lib = L.load("product")
    from fluidphysics_b200 import scenes as S
    sc = S.cpu_scene()
    h = C.c_void_p()
    rc = lib.upbd_create(C.byref(sc.desc), C.byref(sc.params), C.byref(h))
    assert rc in (-7, -3)  # NO_DEVICE (or a CUDA error from a driver stub)
    assert lib.upbd_last_error(None)
