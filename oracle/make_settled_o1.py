"""The CPU solver's own settled state of the default GPU scene, for the
bench's reference arm.

bench.py times the GPU path on the settled pool of the default scene (frames
300..599, slice wedge at frame 60). Its reference arm times the reference's
CPU implementation of the path (O1, the restatement of src/solver.js) on the
host's cores; for the two to time the same kind of state, the arm starts from
the CPU solver's own trajectory at frame 300, which this script produces by
running O1 (one thread, about four minutes): 300 frames of 5 substeps from
the scene's initial state, the wedge cut at frame 60. Between frames the
solver's state is its positions, velocities, active flags and constraint
rests and alive flags (prev is rewritten from pos at the start of every
substep, src/solver.js:194-197).

Usage: python oracle/make_settled_o1.py   (writes oracle/data/gpu_default_o1_frame300.npz)
"""
from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path[0] = str(HERE.parent)  # the repository root, not this directory (it holds oracle.py)

from fluidphysics_b200 import scenes as S  # noqa: E402
from oracle.oracle import o1_from_scene  # noqa: E402

OUT = HERE / "data" / "gpu_default_o1_frame300.npz"
FRAMES = 300


def main() -> None:
    sc = S.gpu_default(frames=FRAMES)
    o1 = o1_from_scene(sc)
    t = time.time()
    for f in range(FRAMES):
        if f == sc.slice_frame:
            o1.cut(*sc.wedge)
        o1.step(sc.dt, sc.substeps)
        if f % 50 == 0:
            print(f"frame {f}: {time.time() - t:.0f} s", flush=True)
    OUT.parent.mkdir(exist_ok=True)
    np.savez_compressed(OUT, frames=FRAMES, pos=o1.get("pos"), vel=o1.get("vel"), active=o1.get("active"),
                        consRest=o1.get("consRest"), consAlive=o1.get("consAlive"))
    print("wrote", OUT, f"{OUT.stat().st_size / 1e6:.2f} MB in {time.time() - t:.0f} s")


if __name__ == "__main__":
    main()
