"""One sample with its compare calls split over ranks (dgpu_dada_sharded).

Every rank's result must equal dada_uniques' on the same sample bit for bit,
with the FP32-decision mode and the transition counts too.
The ranks here are threads of one process on the one visible GPU, exchanging
through an in-process all-gather: the kernels of different ranks never wait
on one another, only the host exchange does. The cross-process exchange over
torch.distributed is covered on CPU by test_multi_rank.py, and the exchange
protocol itself (shares, rank-order merge, failure lockstep) by
test_host_loop.py."""
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import dada2_b200 as D
from dada2_b200 import synth

pytestmark = pytest.mark.gpu

SKIP = {"times"}


class ThreadGather:
    """All-gather among `world` threads: deposit, meet, read, meet again."""

    def __init__(self, world):
        self.blocks = [None] * world
        self.bar = threading.Barrier(world, timeout=300)

    def for_rank(self, rank):
        def gather(block):
            self.blocks[rank] = block
            self.bar.wait()
            out = np.concatenate(self.blocks)
            self.bar.wait()
            return out

        return gather


def _same(a, b):
    assert a["nclust"] == b["nclust"]
    assert set(a) == set(b)
    for k, v in a.items():
        if k in SKIP or k == "clusters":
            continue
        if k == "counters":
            # nalign, nshroud and the kernel counters are sums over the
            # shares; ns_* are the host phases' nanoseconds
            for ck, cv in v.items():
                if not ck.startswith("ns_"):
                    assert cv == b[k][ck], ck
        elif isinstance(v, np.ndarray):
            assert v.tobytes() == b[k].tobytes(), k
        else:
            assert v == b[k], k


def _sharded(s, w, params, world):
    g = ThreadGather(world)
    with ThreadPoolExecutor(world) as ex:
        futs = [ex.submit(D.dada_uniques_sharded, s.seqs, s.abund, w.err, w.ncol, params, quals=s.quals, rank=r,
                          world=world, gather=g.for_rank(r)) for r in range(world)]
        return [f.result(timeout=600) for f in futs]


@pytest.mark.parametrize("case,world,extra", [("small41", 1, {}), ("small41", 2, {}), ("config0", 3, {}),
                                              ("small41", 2, {"transitions": True, "lambda_fp32": True})])
def test_sharded_run_equals_the_one_device_run(case, world, extra):
    w = synth.config0() if case == "config0" else synth.small_illumina(41, nvariants=7, nreads=4000, L=150)
    s = w.samples[0]
    params = D.DadaParams(**extra)
    want = D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, params, quals=s.quals)
    for got in _sharded(s, w, params, world):
        _same(got, want)
