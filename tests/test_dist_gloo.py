"""Multi-process host logic of replicated runs, world size 2 on the gloo backend
(CPU only): rendezvous, max-over-ranks timing, whole-job throughput, and row
sharding that covers a matrix exactly once."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from matvans_b200 import dist as mvd
    r, w = mvd.init("gloo", timeout_s=60)
    assert (r, w) == (rank, world)
    mvd.barrier()
    # rank 1 is the slow one: the job time is its time
    secs = 0.5 if rank == 0 else 2.0
    value, t = mvd.aggregate_throughput(1000.0, secs)
    spans = [mvd.shard_rows(11008, k, world) for k in range(world)]
    out[rank] = (value, t, spans)
    mvd.shutdown()


@pytest.mark.timeout(180)
def test_replicated_timing_world2():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(150)
        assert p.exitcode == 0
    for r in range(2):
        value, t, spans = out[r]
        assert t == 2.0 and value == 2 * 1000.0 / 2.0
    spans = out[0][2]
    assert spans[0][0] == 0 and spans[-1][1] == 11008
    assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
    assert all((s[1] - s[0]) % 32 == 0 or s[1] == 11008 for s in spans)


def test_single_process_is_a_noop():
    from matvans_b200 import dist as mvd
    assert mvd.max_over_ranks(3.5) == 3.5
    assert mvd.aggregate_throughput(10.0, 2.0) == (5.0, 2.0)
