"""The multi-rank plumbing of bench.py (one process per GPU under torchrun:
rendezvous, the barrier around the timed region, the max over ranks of
the timings, the shared config object), run as two gloo ranks on the CPU;
on a GPU box the same functions run over NCCL."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    w, r, local = bench.dist_setup()
    bench.barrier(w)
    slowest = bench.max_over_ranks(1.5 * (r + 1), w, local)
    cfg = bench.bench_config(bench.workload("box64"), w)
    bench.barrier(w)
    dist.destroy_process_group()
    q.put((r, w, slowest, cfg["parallelism"], cfg["cells_per_gpu"]))


def test_two_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, 2, 3.0, "replicas", 64 ** 3), (1, 2, 3.0, "replicas", 64 ** 3)]


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    """Under torchrun every rank launches `--impl reference`; ranks other
    than 0 exit without work or output."""
    sys.path.insert(0, ROOT)
    import argparse

    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = argparse.Namespace(config="box64", steps=1, warmup=3, cpu_omp_steps=0)
    assert bench.run_reference(args) is None
    assert capsys.readouterr().out == ""
