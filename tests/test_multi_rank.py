"""The N > 1 path of bench.py on CPU: two gloo ranks (world size 2) over 127.0.0.1.

The encoder shards by texture with no collective on the data path; the only cross-rank step is the max over ranks
of the timed region, and the reference arm runs on rank 0 alone.
"""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, world, device="cpu")
    value = bench.job_value(ms, world, steps=4, mpix_per_step=4.194304)
    buf = io.StringIO()

    class Args:
        steps, warmup = 1, 0
    with redirect_stdout(buf):
        bench.run_reference(Args, world, rank) if rank != 0 else None
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, ms, value, buf.getvalue()))


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, value, printed in results:
        assert ms == pytest.approx(15.0)  # the max over ranks, seen identically by every rank
        assert value == pytest.approx(2 * 4 * 4.194304 / 0.015)
        if rank == 1:
            assert printed == ""  # the reference arm prints on rank 0 only
