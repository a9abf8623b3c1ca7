"""The multi-rank plumbing of bench.py (one process per GPU, weak scaling:
independent builds, no data-path collective) on CPU with the gloo backend,
world size 2: max-over-ranks timing, barrier, whole-job value, and the
reference arm running on rank 0 only."""
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


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, w, lr = bench.dist_info()
        ms = 2.0 + 3.0 * rank  # the slower rank decides the job time
        ms_max = bench.max_over_ranks(ms, w)
        bench.barrier(w)
        out[rank] = (r, w, lr, ms_max, bench.weak_value(1_000_000, ms_max, w))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_time_as_the_slowest_and_sum_units():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    assert sorted(res) == [0, 1]
    for rank, (r, w, lr, ms_max, value) in res.items():
        assert (r, w, lr) == (rank, 2, rank)
        assert ms_max == 5.0
        assert value == pytest.approx(2 * 1_000_000 / 5.0 / 1e3)


def test_reference_arm_is_rank0_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = bench.argparse.Namespace(gpus=2, steps=1, warmup=0, impl="reference", n=1000, no_components=True,
                                    only_build=False)
    assert bench.run_reference(args) is None  # returns at once, prints nothing
