"""dgpu_align_pairs_noalloc: alignments without any device allocation.

Some callers cannot call cudaMalloc: a host whose device memory is already
reserved by its own pool allocator (a new cudaMalloc fails or fragments that
pool), or a latency-bound pipeline that cannot afford the device-wide
synchronisation of cudaFree. The entry point takes caller-owned device
buffers for inputs and outputs and keeps its scratch in a static device
array, so it allocates nothing. This file checks it against the oracle's
alignments (the CPU restatement of the reference's aligners) on two calls in
a row, that an oversize request is refused, and that a pair longer than the
stated maximum is refused on the device while the other pairs still align.
It runs last in a suite so that a failure here leaves every other test run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pairs(seed, n, lmin, lmax):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        L = int(rng.integers(lmin, lmax + 1))
        a = rng.integers(1, 5, size=L).astype(np.uint8)
        b = list(a)
        for _ in range(int(rng.integers(0, 7))):
            p = int(rng.integers(0, len(b)))
            op = int(rng.integers(0, 3))
            if op == 0:
                b[p] = int(rng.integers(1, 5))
            elif op == 1:
                b.insert(p, b[p])
            elif len(b) > 10:
                b.pop(p)
        out.append((a, np.array(b, np.uint8)))
    return out


def _noalloc(which, pairs, params, end_gap, max_len, keep_outputs=False):
    """Calls the entry point with device buffers the caller (this test) owns."""
    import torch

    import dada2_b200 as D
    from dada2_b200 import _lib

    s1 = [a for a, _ in pairs]
    s2 = [b for _, b in pairs]
    l1 = np.array([len(s) for s in s1], np.uint32)
    l2 = np.array([len(s) for s in s2], np.uint32)
    o1 = np.concatenate([[0], np.cumsum(l1)[:-1]]).astype(np.uint32)
    o2 = np.concatenate([[0], np.cumsum(l2)[:-1]]).astype(np.uint32)
    cap = l1.astype(np.int64) + l2
    ao = np.concatenate([[0], np.cumsum(cap)[:-1]]).astype(np.uint32)
    dev = torch.device("cuda", 0)

    def up(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    t = {k: up(v) for k, v in (("s1", np.concatenate(s1)), ("o1", o1), ("l1", l1), ("s2", np.concatenate(s2)),
                                ("o2", o2), ("l2", l2), ("ao", ao))}
    a0 = torch.zeros(int(cap.sum()) + 1, dtype=torch.uint8, device=dev)
    a1 = torch.zeros_like(a0)
    al = torch.zeros(len(pairs), dtype=torch.int32, device=dev)
    L = _lib.lib()
    fn = L.dgpu_align_pairs_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 6 + [C.POINTER(_lib.AlignParamsC), C.c_int] + \
        [C.c_void_p] * 5
    pc = params.c()
    torch.cuda.synchronize()
    p = lambda x: C.c_void_p(x.data_ptr())  # noqa: E731
    rc = fn(which, len(pairs), max_len, p(t["s1"]), p(t["o1"]), p(t["l1"]), p(t["s2"]), p(t["o2"]), p(t["l2"]),
            C.byref(pc), end_gap, p(a0), p(a1), p(t["ao"]), p(al), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    if rc != 0 and not keep_outputs:
        return rc, L.dgpu_last_error().decode()
    err = L.dgpu_last_error().decode() if rc != 0 else ""
    torch.cuda.synchronize()
    a0h, a1h, alh = a0.cpu().numpy(), a1.cpu().numpy(), al.cpu().numpy().astype(np.int64)
    out = [(a0h[o:o + n].copy(), a1h[o:o + n].copy()) for o, n in zip(ao, alh)]
    return rc, ((out, err) if rc != 0 else out)


@pytest.mark.parametrize("which,band,end_gap,hg", [(0, 16, 0, -8), (0, -1, -8, -8), (1, 32, 0, -1), (2, 16, 0, -8)])
def test_noalloc_matches_the_oracle_twice(which, band, end_gap, hg):
    pytest.importorskip("torch")
    import dada2_b200 as D
    from oracle import oracle as O

    params = D.AlignParams(band=band, homo_gap_p=hg)
    owhich = {0: O.ALIGN_VECTORIZED, 1: O.ALIGN_HOMO, 2: O.ALIGN_ENDSFREE}[which]
    for call, seed in enumerate((101, 202)):  # two calls in a row share the static scratch
        pairs = _pairs(seed + which, 150, 30, 260)
        rc, got = _noalloc(which, pairs, params, end_gap, max_len=270)
        assert rc == 0, got
        for (a, b), (g0, g1) in zip(pairs, got):
            w0, w1 = O.align(owhich, a, b, homo_gap=hg, end_gap=end_gap, band=band)
            assert np.array_equal(g0, w0) and np.array_equal(g1, w1), (call, which, band, len(a), len(b))


def test_noalloc_refuses_a_pair_longer_than_max_len():
    pytest.importorskip("torch")
    import dada2_b200 as D
    from dada2_b200._lib import DGPU_E_DEVICE
    from oracle import oracle as O

    pairs = _pairs(303, 40, 30, 120)
    long_a = np.tile(np.array([1, 2, 3, 4], np.uint8), 33)  # 132 nt, one past max_len = 131
    pairs[17] = (long_a, long_a.copy())
    rc, msg = _noalloc(0, pairs, D.AlignParams(band=16), 0, max_len=131, keep_outputs=True)
    assert rc == DGPU_E_DEVICE, msg
    got, err = msg
    assert "max_len" in err
    for i, ((a, b), (g0, g1)) in enumerate(zip(pairs, got)):
        if i == 17:
            assert len(g0) == 0  # refused: its length slot stays as the caller set it
            continue
        w0, w1 = O.align(O.ALIGN_VECTORIZED, a, b, band=16)
        assert np.array_equal(g0, w0) and np.array_equal(g1, w1), i


def test_noalloc_rejects_sizes_beyond_its_scratch():
    pytest.importorskip("torch")
    import dada2_b200 as D
    from dada2_b200._lib import DGPU_E_INVALID

    pairs = _pairs(7, 4, 20, 40)
    rc, msg = _noalloc(0, pairs, D.AlignParams(band=-1), 0, max_len=3500)
    assert rc == DGPU_E_INVALID
    assert "16 MiB" in msg
