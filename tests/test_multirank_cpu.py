"""The N > 1 host logic of ``bench.py`` on CPU ranks (gloo, world size 2).

The path does not shard: every rank solves its own replica batch and the only
collectives are the barrier and the max-over-ranks timing.  These tests run
that logic as two gloo processes: the timing maximum reaches both ranks, the
replicas differ by rank, and under torchrun the reference arm runs on rank 0
alone while the other rank exits 0 without work.
"""

import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        result = {"max": bench.rank_max(float(rank + 1), world, device="cpu")}
        lps = bench.make_batch(seed=1000 + rank)
        result["first_lp"] = lps[0].problem.name
        args = type("Args", (), {"cpu_budget": 0.5, "warmup": 1, "steps": 1})()
        buf = io.StringIO()
        with redirect_stdout(buf):
            rc = bench.run_reference(args, rank, world)
        result["rc"] = rc
        result["printed"] = buf.getvalue()
        dist.barrier()
    finally:
        dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as fh:
        json.dump(result, fh)


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    r0 = json.loads((tmp_path / "rank0.json").read_text())
    r1 = json.loads((tmp_path / "rank1.json").read_text())
    assert r0["max"] == r1["max"] == 2.0                 # max over ranks, on every rank
    assert r0["first_lp"] != r1["first_lp"]              # each rank its own replica batch
    assert r0["rc"] == r1["rc"] == 0
    assert r1["printed"] == ""                           # rank 1: no work, no line
    line = json.loads(r0["printed"].strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["e2e"]["h2d_bytes_per_step"] == 0
