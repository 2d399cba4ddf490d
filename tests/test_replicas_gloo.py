"""The multi-GPU launch of bench.py ("replicas only": one process per GPU,
each running BFS from its own roots, no collective on the data path) checked
on CPU with world_size-2 gloo process groups: the roots are dealt to the
ranks without overlap, the timed region's barrier holds, and the job's time
is the max over ranks while its work is the sum over ranks."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    try:
        wsz, r, _ = bench.dist_setup(None, backend="gloo")
        roots = np.arange(64, dtype=np.uint32) * 7 + 3
        seq = bench.replica_roots(roots, wsz, r, 3 + 32)  # warm-up + timed steps
        bench.barrier(wsz)
        t_ms = 10.0 + rank  # this rank's timed region
        half_edges = 1000.0 * (rank + 1)
        q.put((rank, seq, bench.max_over_ranks(t_ms, wsz), bench.sum_over_ranks(half_edges, wsz)))
    finally:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()


def test_replica_ranks_with_gloo():
    mp = pytest.importorskip("torch.multiprocessing")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in procs:
        rank, seq, tmax, esum = q.get(timeout=120)
        res[rank] = (seq, tmax, esum)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # timed steps of the two ranks: disjoint roots, together the first 64 dealt in order
    timed = [res[r][0][3:] for r in (0, 1)]
    assert not set(timed[0][:32]) & set(timed[1][:32])
    roots = list(np.arange(64) * 7 + 3)
    assert sorted(timed[0][:32] + timed[1][:32]) == sorted(roots[(3 * 2) % 64:] + roots[:(3 * 2) % 64])
    # every rank sees the max time and the summed work
    assert res[0][1] == res[1][1] == 11.0
    assert res[0][2] == res[1][2] == 3000.0
