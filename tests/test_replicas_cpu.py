"""The multi-GPU form of bench.py is replicas: every rank advances its own
ensemble (a different seed per rank), and the job's throughput is all
ranks' work over the slowest rank's time.  Checked with two gloo ranks on
the CPU (the reductions bench.py makes), no GPU needed."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        units, steps, seconds = 1000 * (rank + 1), 10, 2.0 + rank
        v = bench.replica_throughput(units, steps, seconds, world, device="cpu")
        t = bench.reduce_over_ranks(seconds, world, "max", device="cpu")
        out[rank] = (v, t)
    finally:
        dist.destroy_process_group()


def test_replica_throughput_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        expect = (1000 * 10 + 2000 * 10) / 3.0
        for r in range(2):
            v, t = out[r]
            assert v == pytest.approx(expect) and t == 3.0


def test_replicas_draw_their_own_ensembles():
    a = bench.make_cases("ensemble", rank=0, first=3)
    b = bench.make_cases("ensemble", rank=1, first=3)
    assert [c["nkn"] for c in a] != [c["nkn"] for c in b]
