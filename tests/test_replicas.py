"""The multi-GPU path of bench.py is replicas only: each rank steps its own
scene and the ranks meet only to agree on the job's time (max over ranks)
and work (sum over ranks). Checked here with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    t, u = bench.reduce_over_ranks(dist, ms=10.0 * (rank + 1), units=1000.0 * (rank + 1), device="cpu")
    out.put((rank, t, u))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_max_time_sum_units():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(0, 20.0, 3000.0), (1, 20.0, 3000.0)]


def test_single_process_is_identity():
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import bench
    assert bench.reduce_over_ranks(None, 5.0, 7.0, "cpu") == (5.0, 7.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = type("A", (), {"steps": 1, "warmup": 0, "gpus": 2})()
    bench.run_reference(args)  # returns at once, prints nothing
    assert capsys.readouterr().out == ""


def test_reference_arm_line(monkeypatch, capsys):
    """Rank 0 of the reference arm prints one JSON line with the base
    contract's keys, its CPU baseline and an e2e block without copies."""
    import json
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import bench
    monkeypatch.setenv("RANK", "0")
    monkeypatch.setenv("WORLD_SIZE", "1")
    args = type("A", (), {"steps": 1, "warmup": 0, "gpus": 1})()
    bench.run_reference(args)
    lines = [l for l in capsys.readouterr().out.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "particle-substeps/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
