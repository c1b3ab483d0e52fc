"""The N>1 path on CPU: world-size-2 gloo ranks, sharding and the timing reduction."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, sizes, out):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "dada2-rs_b200"))
    import datetime

    import torch.distributed as dist

    from dada2_b200 import multi

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    mine = multi.shard_samples(sizes, rank, world)
    secs, comps = multi.reduce_run(1.0 + rank, 100 * (rank + 1))
    out.put((rank, mine, secs, comps))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shard_and_reduce():
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp

    sizes = [5637, 1975, 10356, 924, 477, 6232, 1996, 12127, 8685, 1738, 5994]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    owned = res[0][1] + res[1][1]
    assert sorted(owned) == list(range(len(sizes)))  # complete and disjoint
    loads = [sum(sizes[i] for i in r[1]) for r in res]
    assert max(loads) - min(loads) <= max(sizes)
    for _, _, secs, comps in res:
        assert secs == 2.0 and comps == 300
    _ = torch


def test_single_process_reduce_is_identity():
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "dada2-rs_b200"))
    from dada2_b200 import multi

    assert multi.reduce_run(3.5, 7) == (3.5, 7)
    assert multi.shard_samples([3, 1, 2], 0, 1) == [0, 1, 2]


def test_request_router_balances_outstanding_work():
    """Service requests go to the device with the least outstanding work and
    their work is returned when collected."""
    from dada2_b200.multi import RequestRouter

    r = RequestRouter(3)
    assert [r.assign(k, w) for k, w in enumerate([100, 50, 50, 10, 200])] == [0, 1, 2, 1, 2]
    assert r.load == [100, 60, 250]
    assert r.release(0) == 0 and r.load == [0, 60, 250]
    assert r.assign(9, 5) == 0


def _gather_worker(rank, world, port, out):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "dada2-rs_b200"))
    import ctypes as C
    import datetime

    import numpy as np
    import torch.distributed as dist

    import dada2_b200
    from dada2_b200 import multi

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    fn = dada2_b200._c_gather(multi.torch_gather(), world)
    got = []
    for nbytes in (56, 24 * 37, 56):  # a head, a comp block, a head: the sharded run's exchange sizes
        send = (np.arange(nbytes, dtype=np.uint32) * (rank + 3) % 251).astype(np.uint8)
        recv = np.zeros(world * nbytes, np.uint8)
        rc = fn(None, C.c_void_p(send.ctypes.data), nbytes, C.c_void_p(recv.ctypes.data))
        got.append((rc, recv.tobytes()))
    # a gather that raises, or answers with the wrong size, reports nonzero
    bad = dada2_b200._c_gather(lambda b: (_ for _ in ()).throw(RuntimeError("peer gone")), world)
    short = dada2_b200._c_gather(lambda b: b, world)
    one = np.zeros(8, np.uint8)
    sink = np.zeros(8 * world, np.uint8)
    rc_bad = bad(None, C.c_void_p(one.ctypes.data), 8, C.c_void_p(sink.ctypes.data))
    rc_short = short(None, C.c_void_p(one.ctypes.data), 8, C.c_void_p(sink.ctypes.data))
    out.put((rank, got, rc_bad, rc_short))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharded_exchange_gather():
    """The all-gather a sharded run calls through its C callback
    (dgpu_allgather_fn over torch.distributed): every rank receives every
    rank's block in rank order, at the head and comp-block sizes."""
    pytest.importorskip("torch")
    import numpy as np
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for nb_i, nbytes in enumerate((56, 24 * 37, 56)):
        want = b"".join((np.arange(nbytes, dtype=np.uint32) * (r + 3) % 251).astype(np.uint8).tobytes()
                        for r in range(2))
        for rank, got, _, _ in res:
            assert got[nb_i] == (0, want)
    for _, _, rc_bad, rc_short in res:
        assert rc_bad != 0 and rc_short != 0
