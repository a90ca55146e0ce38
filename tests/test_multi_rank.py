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


def test_reference_arm_under_torchrun_prints_once(tmp_path):
    """`bench.py --impl reference` launched by torchrun with two ranks: rank 0 alone times the reference and prints
    one JSON line, the other rank exits 0 without work, and no process group is needed (no GPU here)."""
    import json
    import subprocess
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libzapref.so")):
        pytest.skip("the reference library is not built here")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1 and lines[0]["impl"] == "reference" and lines[0]["value"] > 0
    assert lines[0]["e2e"]["h2d_bytes_per_step"] == 0 and lines[0]["cpu_baseline"]["kind"] == "reference"
