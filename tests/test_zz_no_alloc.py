"""dgpu_align_pairs_noalloc: alignments without any device allocation.

Some callers cannot call cudaMalloc -- code that runs while a CUDA stream is
being captured into a graph (allocation is not capturable), or a host whose
device memory is handed out by another allocator. The entry point takes
caller-owned device buffers for inputs and outputs and keeps its scratch in a
static device array, so it allocates nothing. This file checks it against the
allocating entry point (dgpu_align_debug) on two calls in a row, and that an
oversize request is refused. It is named to run last in a suite.
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


def _noalloc(which, pairs, params, end_gap, max_len):
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
    if rc != 0:
        return rc, L.dgpu_last_error().decode()
    a0h, a1h, alh = a0.cpu().numpy(), a1.cpu().numpy(), al.cpu().numpy().astype(np.int64)
    return rc, [(a0h[o:o + n].copy(), a1h[o:o + n].copy()) for o, n in zip(ao, alh)]


@pytest.mark.parametrize("which,band,end_gap,hg", [(0, 16, 0, -8), (0, -1, -8, -8), (1, 32, 0, -1), (2, 16, 0, -8)])
def test_noalloc_matches_allocating_entry_twice(which, band, end_gap, hg):
    pytest.importorskip("torch")
    import dada2_b200 as D

    params = D.AlignParams(band=band, homo_gap_p=hg)
    for call, seed in enumerate((101, 202)):  # two calls in a row share the static scratch
        pairs = _pairs(seed + which, 150, 30, 260)
        rc, got = _noalloc(which, pairs, params, end_gap, max_len=270)
        assert rc == 0, got
        want = D.align_pairs(which, pairs, params, end_gap=end_gap)
        for (g0, g1), (w0, w1) in zip(got, want):
            assert np.array_equal(g0, w0) and np.array_equal(g1, w1), (call, which, band)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    pytest.importorskip("torch")
    import dada2_b200 as D
    from dada2_b200._lib import DGPU_E_INVALID

    pairs = _pairs(7, 4, 20, 40)
    rc, msg = _noalloc(0, pairs, D.AlignParams(band=-1), 0, max_len=3500)
    assert rc == DGPU_E_INVALID
    assert "16 MiB" in msg
