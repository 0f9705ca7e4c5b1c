"""The multi-rank path of bench.py on the CPU: two gloo ranks, as torchrun
launches them (RANK / WORLD_SIZE / LOCAL_RANK / MASTER_* from the
environment, rendezvous on 127.0.0.1).

The hot path does not shard one problem (replicas only), so the only
exchanges are scalars: the whole-job value is the units of all ranks over the
slowest rank's time (sum and max over ranks), and the reference arm runs on
rank 0 alone while the other ranks exit without work.
"""
import json
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import contextlib
    import io

    import bench
    w, r, local, pg = bench.dist_setup()
    try:
        device_ms = 10.0 * (r + 1)        # this replica's timed region
        updates = 1000.0 * (r + 1)        # this replica's voxel updates
        slowest = bench.max_over_ranks(pg, device_ms)
        total = bench.sum_over_ranks(pg, updates)
        bench.barrier(pg)
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            if r != 0:  # the reference arm: ranks other than 0 return at once, printing nothing
                bench.run_reference_arm(None, r)
        with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
            json.dump({"world": w, "rank": r, "local": local, "slowest": slowest, "total": total,
                       "value": total / (slowest / 1e3), "printed": buf.getvalue()}, f)
    finally:
        pg.destroy_process_group()


def test_two_gloo_replicas_reduce_value_and_time(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r, d in enumerate(res):
        assert d["world"] == world and d["rank"] == r and d["local"] == r
        assert d["slowest"] == pytest.approx(20.0)      # max over ranks
        assert d["total"] == pytest.approx(3000.0)      # sum over ranks
        assert d["value"] == pytest.approx(3000.0 / 0.020)
    assert res[1]["printed"] == ""


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK") if k in os.environ}
    try:
        world, rank, local, pg = bench.dist_setup()
        assert (world, rank, local, pg) == (1, 0, 0, None)
        assert bench.max_over_ranks(pg, 3.5) == 3.5 and bench.sum_over_ranks(pg, 2.0) == 2.0
    finally:
        os.environ.update(env)
