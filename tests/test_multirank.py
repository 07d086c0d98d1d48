"""The N-GPU bench path on CPU: world_size 2 over gloo.

bench.py runs one replica of the frame per GPU (the path has no data
exchange) and reports the summed rate with the time taken as the maximum
over ranks.  These checks run its rank helpers in two processes on the
gloo backend: the max-over-ranks reduction and the barrier."""
import os

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _worker(rank, world, port, results):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import torch
    t = torch.tensor([float(10 + rank)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    results[rank] = float(t.item())
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    results = mgr.dict()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, results)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert results[0] == results[1] == 11.0


def test_bench_replica_accounting():
    # value = rays x steps x world / max-over-ranks time (weak scaling)
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "bench", os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.launches_per_frame(0) == 1
