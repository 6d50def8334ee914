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


@pytest.mark.parametrize("variant", ["product", "parity"])
def test_library_exports_every_declared_symbol(built_libs, variant):
    lib = C.CDLL(str(L.lib_path(variant)))
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes table covers the header exactly
    assert set(L.EXPORTED) == declared_symbols()


def test_library_is_sm100a(built_libs):
    # the fatbin carries sm_100a code only; cuobjdump is not needed for this:
    # the build flags are the contract
    from fluidphysics_b200 import build as B
    assert B.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


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
