"""The multi-rank path of bench.py on CPU: two processes over gloo (the
bench uses NCCL on GPUs; the reduction is the same collective). Each rank
is an independent replica of the whole workload: the timed value is the
slowest rank's, every rank sees it, the whole-job throughput counts every
rank's units, and the reference arm runs and prints on rank 0 only."""
import contextlib
import io
import json
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    ms = 10.0 + 5.0 * rank  # rank 1 is the slower replica
    slowest = bench.max_over_ranks(ms, world, torch.device("cpu"))
    value = bench.replicas_throughput(1000, 4, world, slowest)
    # the reference arm: rank 0 alone runs it and prints its line
    import argparse
    args = argparse.Namespace(n=2000, steps=1, warmup=0, gpus=world, impl="reference")
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.run_reference(args)
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"slowest": slowest, "value": value, "stdout": buf.getvalue()}, f)


def test_two_replicas_over_gloo(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    results = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    assert [r["slowest"] for r in results] == [15.0, 15.0]
    # 2 replicas x 1000 units x 4 steps in the slowest rank's 15 ms
    assert results[0]["value"] == pytest.approx(2 * 1000 * 4 / 0.015 / 1e6)
    assert results[1]["stdout"] == ""
    line = json.loads(results[0]["stdout"].strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == world and line["value"] > 0
