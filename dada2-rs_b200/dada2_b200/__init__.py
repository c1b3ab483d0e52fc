"""B200 (sm_100a) implementation of the compare step of dada2-rs `dada`.

The compare kernels and the clustering loop live in libdada2_b200.so (C ABI:
include/dada2_b200.h). This module is a thin Python mirror of the reference's
interface for the path:

* :class:`CompareContext` -- uniques resident on one GPU; ``compare`` is the map
  of ``b_compare_parallel`` (src/cluster.rs:279-330) and ``b_compare_parallel``
  is map + store (src/cluster.rs:239-423).
* :func:`dada_uniques` -- one sample end to end (src/dada.rs:225-592).
* :func:`dada_uniques_batch` -- many independent samples in one pass.

Sequences are ASCII (A/C/G/T/U, either case); qualities are per-position Phred
SUMS over the reads of each unique, as the reference's derep produces them.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._lib import (AlignParamsC, CountersC, DadaOutC, DadaParamsC, DgpuError, ErrFunC, InvalidInput, KernelStatsC,
                   TuningC, check, device_count, lib, ptr)

__all__ = ["AlignParams", "DadaParams", "CompareContext", "dada_uniques", "dada_uniques_batch", "dada_uniques_sharded",
           "ResidentBatch", "PackedBatch", "DenoiseService", "pack_sample", "Derep", "derep_fastq", "dada_fastq", "align_pairs", "stats_reset", "stats_timing", "stats_read",
           "DgpuError", "InvalidInput", "device_count", "METHOD_NAMES", "KERNEL_NAMES", "TUNING_KEYS",
           "tuning_get", "tuning_set", "tuning_load", "tuning_save", "tuning_reset", "length_class",
           "ErrFun", "errfun_apply", "learn_errors"]

KERNEL_NAMES = ["profiles", "screen", "align", "store"]

METHOD_NAMES = {0: "none", 1: "gapless", 2: "vectorized", 3: "homo", 4: "endsfree"}
COUNTER_KEYS = ["nalign", "compare_calls", "cmp_scanned", "screened", "aligned", "stored",
                "gapless", "vectorized", "homo", "endsfree", "shuffle_calls", "shuffle_moves",
                "nshroud", "ns_shuffle", "ns_pupdate", "ns_bud"]


@dataclass
class AlignParams:
    """AlignParams (src/nwalign.rs:63-90); defaults from src/main.rs:4393-4433."""
    match_score: int = 5
    mismatch: int = -4
    gap_p: int = -8
    homo_gap_p: int = -8
    use_kmers: bool = True
    kdist_cutoff: float = 0.42
    kmer_size: int = 5
    band: int = 16
    vectorized: bool = True
    gapless: bool = True

    def c(self) -> AlignParamsC:
        return AlignParamsC(int(self.match_score), int(self.mismatch), int(self.gap_p),
                            int(self.homo_gap_p), int(bool(self.use_kmers)), float(self.kdist_cutoff),
                            int(self.kmer_size), int(self.band), int(bool(self.vectorized)),
                            int(bool(self.gapless)))


@dataclass
class DadaParams:
    """The DadaParams fields the clustering loop reads (src/dada.rs:54-101)."""
    align: AlignParams = field(default_factory=AlignParams)
    omega_a: float = 1e-40
    omega_p: float = 1e-4
    omega_c: float = 1e-40
    detect_singletons: bool = False
    max_clust: int = 0
    min_fold: float = 1.0
    min_hamming: int = 1
    min_abund: int = 1
    use_quals: bool = True
    greedy: bool = True
    host_threads: int = 0
    transitions: bool = False  # also return DadaAux.transitions (src/error.rs:194-249)
    # decisions from the FP32 compensated log-sum lambda, FP64 within 1e3x of the thresholds
    lambda_fp32: bool = False

    def c(self) -> DadaParamsC:
        return DadaParamsC(self.align.c(), float(self.omega_a), float(self.omega_p), float(self.omega_c),
                           int(bool(self.detect_singletons)), int(self.max_clust), float(self.min_fold),
                           int(self.min_hamming), int(self.min_abund), int(bool(self.use_quals)),
                           int(bool(self.greedy)), int(self.host_threads), int(bool(self.transitions)),
                           int(bool(self.lambda_fp32)))


def _counters(c: CountersC) -> dict:
    return {n: int(getattr(c, n)) for n, _ in CountersC._fields_}


class CompareContext:
    """Uniques resident on one device; the drop-in for b_compare_parallel.

    ``seqs`` are arrays of codes 1..4; ``quals`` rounded mean Phred (u8) or None.
    """

    def __init__(self, params: AlignParams, err: np.ndarray, ncol: int, use_quals: bool = True,
                 device: int = 0):
        self.h = C.c_void_p()
        self._err = np.ascontiguousarray(err, np.float64)
        pc = params.c()
        check(lib().dgpu_ctx_create(device, C.byref(pc), ptr(self._err), int(ncol), int(bool(use_quals)),
                                    C.byref(self.h)))
        self.n = 0

    def upload(self, seqs, reads, quals=None):
        seqs = [np.ascontiguousarray(s, np.uint8) for s in seqs]
        lens = np.array([len(s) for s in seqs], np.uint32)
        offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.uint32)
        cat = np.concatenate(seqs).astype(np.uint8)
        qcat = None if quals is None else np.concatenate(
            [np.ascontiguousarray(q, np.uint8) for q in quals]).astype(np.uint8)
        rd = np.ascontiguousarray(reads, np.uint32)
        check(lib().dgpu_upload_raws(self.h, len(seqs), ptr(cat), ptr(offs), ptr(lens), ptr(qcat), ptr(rd)))
        self.n = len(seqs)

    def set_locks(self, lock):
        lk = np.ascontiguousarray(lock, np.uint8)
        check(lib().dgpu_set_locks(self.h, ptr(lk)))

    def reset_e_minmax(self):
        check(lib().dgpu_reset_e_minmax(self.h))

    def e_minmax(self) -> np.ndarray:
        out = np.zeros(self.n, np.float64)
        check(lib().dgpu_get_e_minmax(self.h, ptr(out)))
        return out

    def compare(self, center: int, kdist_cutoff: float, greedy: bool = True):
        """The map: per-raw (lambda, hamming or UINT32_MAX, skipped)."""
        lam = np.zeros(self.n, np.float64)
        ham = np.zeros(self.n, np.uint32)
        skp = np.zeros(self.n, np.uint8)
        cnt = CountersC()
        check(lib().dgpu_compare(self.h, int(center), float(kdist_cutoff), int(bool(greedy)), ptr(lam), ptr(ham),
                                 ptr(skp), C.byref(cnt)))
        return lam, ham, skp.astype(bool), _counters(cnt)

    def b_compare_parallel(self, center: int, cluster_i: int, kdist_cutoff: float, greedy: bool = True):
        """Map + store: the stored comparisons in ascending raw order."""
        idx = np.zeros(self.n, np.uint32)
        lam = np.zeros(self.n, np.float64)
        ham = np.zeros(self.n, np.uint32)
        ns = C.c_int(0)
        self_ = C.c_double(0.0)
        cnt = CountersC()
        check(lib().dgpu_compare_store(self.h, int(center), int(cluster_i), float(kdist_cutoff), int(bool(greedy)),
                                       ptr(idx), ptr(lam), ptr(ham), C.byref(ns), C.byref(self_), C.byref(cnt)))
        k = ns.value
        return {"index": idx[:k].copy(), "lambda": lam[:k].copy(), "hamming": ham[:k].copy(),
                "self": self_.value, "counters": _counters(cnt)}

    def methods(self) -> np.ndarray:
        """The aligner each raw took in the latest compare (codes of METHOD_NAMES)."""
        out = np.zeros(self.n, np.uint8)
        check(lib().dgpu_get_methods(self.h, ptr(out)))
        return out

    def set_lambda32(self, enable: bool = True):
        """Also form ln(lambda) in compensated FP32 on later compares (precision report)."""
        check(lib().dgpu_ctx_set_lambda32(self.h, int(bool(enable))))

    def loglambda32(self) -> np.ndarray:
        """FP32 ln(lambda) of the latest compare (-inf where the pair was not aligned)."""
        out = np.zeros(self.n, np.float32)
        check(lib().dgpu_get_loglambda32(self.h, ptr(out)))
        return out

    def close(self):
        if self.h:
            lib().dgpu_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _pack(seqs, abund, quals=None, prior=None):
    enc = [s.encode("ascii") if isinstance(s, str) else bytes(s) for s in seqs]
    lens = np.array([len(s) for s in enc], np.uint32)
    offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.uint32)
    cat = np.frombuffer(b"".join(enc), np.uint8).copy()
    ab = np.ascontiguousarray(abund, np.uint32)
    qcat = None
    if quals is not None:
        qcat = np.concatenate([np.ascontiguousarray(q, np.uint32) for q in quals]).astype(np.uint32)
    pr = None if prior is None else np.ascontiguousarray(prior, np.uint8)
    return cat, offs, lens, ab, qcat, pr


def _read_result(h) -> dict:
    sizes = np.zeros(4, np.int64)
    check(lib().dgpu_result_sizes(h, ptr(sizes)))
    ncl, nraw, nmem, nseq = (int(x) for x in sizes)
    a = {
        "cl_reads": np.zeros(ncl, np.uint32), "cl_birth_type": np.zeros(ncl, np.int32),
        "cl_birth_from": np.zeros(ncl, np.uint32), "cl_birth_pval": np.zeros(ncl, np.float64),
        "cl_birth_fold": np.zeros(ncl, np.float64), "cl_birth_e": np.zeros(ncl, np.float64),
        "cl_birth_hamming": np.zeros(ncl, np.uint32), "cl_seq_off": np.zeros(ncl + 1, np.uint32),
        "cl_seq": np.zeros(max(nseq, 1), np.uint8), "cl_mem_off": np.zeros(ncl + 1, np.uint32),
        "mem_raw": np.zeros(max(nmem, 1), np.uint32), "mem_hamming": np.zeros(max(nmem, 1), np.uint32),
        "mem_lambda": np.zeros(max(nmem, 1), np.float64), "mem_pval": np.zeros(max(nmem, 1), np.float64),
        "map": np.zeros(max(nraw, 1), np.int32), "pvals": np.zeros(max(nraw, 1), np.float64),
        "counters": np.zeros(16, np.uint64), "times": np.zeros(6, np.float64),
    }
    o = DadaOutC(*[ptr(a[n]) for n, _ in DadaOutC._fields_])
    check(lib().dgpu_result_fill(h, C.byref(o)))
    res = {"nclust": ncl, "nraw": nraw, **a}
    res["map"] = a["map"][:nraw]
    res["pvals"] = a["pvals"][:nraw]
    res["counters"] = {k: int(v) for k, v in zip(COUNTER_KEYS, a["counters"])}
    res["clusters"] = ClusterList(a, ncl)
    f32 = np.zeros(2, np.uint64)
    check(lib().dgpu_result_fp32_stats(h, ptr(f32)))
    res["fp32"] = {"pvalues": int(f32[0]), "fallbacks": int(f32[1])}
    mg = np.zeros(3, np.float64)
    check(lib().dgpu_result_margins(h, ptr(mg)))
    res["margins"] = {"omega_a": float(mg[0]), "omega_p": float(mg[1]), "omega_c": float(mg[2])}
    tncol = lib().dgpu_result_transitions(h, None)
    if tncol > 0:
        tr = np.zeros(16 * tncol, np.uint32)
        lib().dgpu_result_transitions(h, ptr(tr))
        res["transitions"] = tr.reshape(16, tncol)
    return res


class ClusterList:
    """Per-cluster views of a result's flat arrays (``cl_*``, ``mem_*``), built
    on access: ``len``, indexing and iteration give one dict per cluster with
    its center ``sequence`` (codes 1..4), ``reads``, ``members`` (raw indices in
    membership order) with their ``hammings``, ``lambdas`` and ``pvals``, and
    the ``birth_*`` statistics."""

    def __init__(self, a: dict, n: int):
        self._a = a
        self._n = n

    def __len__(self):
        return self._n

    def __getitem__(self, ci):
        if isinstance(ci, slice):
            return [self[k] for k in range(*ci.indices(self._n))]
        if ci < 0:
            ci += self._n
        if not 0 <= ci < self._n:
            raise IndexError(ci)
        a = self._a
        s0, s1 = a["cl_seq_off"][ci], a["cl_seq_off"][ci + 1]
        m0, m1 = a["cl_mem_off"][ci], a["cl_mem_off"][ci + 1]
        return {
            "sequence": a["cl_seq"][s0:s1].copy(), "reads": int(a["cl_reads"][ci]),
            "members": a["mem_raw"][m0:m1].copy(), "hammings": a["mem_hamming"][m0:m1].copy(),
            "lambdas": a["mem_lambda"][m0:m1].copy(), "pvals": a["mem_pval"][m0:m1].copy(),
            "birth_type": int(a["cl_birth_type"][ci]), "birth_from": int(a["cl_birth_from"][ci]),
            "birth_pval": float(a["cl_birth_pval"][ci]), "birth_fold": float(a["cl_birth_fold"][ci]),
            "birth_e": float(a["cl_birth_e"][ci]), "birth_hamming": int(a["cl_birth_hamming"][ci]),
        }

    def __iter__(self):
        for ci in range(self._n):
            yield self[ci]


def pack_sample(seqs, abund, quals=None, prior=None):
    """A sample's host buffers in the C ABI's layout, for repeated calls."""
    return _pack(seqs, abund, quals, prior)


def dada_uniques(seqs, abund, err, ncol, params: DadaParams | None = None, quals=None, prior=None,
                 device: int = 0, packed=None, read_result: bool = True) -> dict:
    """Denoise one sample on the GPU (src/dada.rs:225-592). ``packed`` (from
    ``pack_sample``) replaces seqs/abund/quals/prior; without ``read_result``
    the result carries its sizes and counters only."""
    params = params or DadaParams()
    cat, offs, lens, ab, qcat, pr = packed if packed is not None else _pack(seqs, abund, quals, prior)
    err = np.ascontiguousarray(err, np.float64)
    pc = params.c()
    h = C.c_void_p()
    check(lib().dgpu_dada(device, C.byref(pc), len(lens), ptr(cat), ptr(offs), ptr(lens), ptr(ab), ptr(pr),
                          ptr(qcat), ptr(err), int(ncol), C.byref(h)))
    try:
        return _read_result(h) if read_result else _read_counters(h)
    finally:
        lib().dgpu_result_free(h)


def _c_gather(gather, world: int):
    """A dgpu_allgather_fn over the Python callable ``gather`` (uint8 block ->
    the world's blocks back to back). A raised exception or a wrong size
    returns nonzero, which fails the sharded run on this rank."""
    from ._lib import ALLGATHER_FN

    def cb(user, send, nbytes, recv):
        try:
            block = np.frombuffer((C.c_uint8 * nbytes).from_address(send), np.uint8).copy()
            out = np.ascontiguousarray(gather(block), np.uint8).reshape(-1)
            if out.size != nbytes * world:
                return 1
            C.memmove(recv, out.ctypes.data, out.size)
            return 0
        except Exception:  # noqa: BLE001 - any failure is reported to the C side as nonzero
            return 1

    return ALLGATHER_FN(cb)


def dada_uniques_sharded(seqs, abund, err, ncol, params: DadaParams | None = None, quals=None, prior=None, *,
                         rank: int, world: int, gather, device: int = 0, packed=None) -> dict:
    """``dada_uniques`` with the compare calls split over ``world`` ranks, this
    one on ``device`` (dgpu_dada_sharded): every rank passes the same sample
    and parameters and gets the same result, dada_uniques' own. ``gather``
    all-gathers a uint8 block among the ranks (``multi.torch_gather`` for a
    process group; all ranks' blocks concatenated in rank order)."""
    params = params or DadaParams()
    cat, offs, lens, ab, qcat, pr = packed if packed is not None else _pack(seqs, abund, quals, prior)
    err = np.ascontiguousarray(err, np.float64)
    pc = params.c()
    h = C.c_void_p()
    fn = _c_gather(gather, int(world))
    check(lib().dgpu_dada_sharded(device, C.byref(pc), len(lens), ptr(cat), ptr(offs), ptr(lens), ptr(ab), ptr(pr),
                                  ptr(qcat), ptr(err), int(ncol), int(rank), int(world), fn, None, C.byref(h)))
    try:
        return _read_result(h)
    finally:
        lib().dgpu_result_free(h)


class PackedBatch:
    """Host buffers of a batch, packed once so repeated runs time only the call."""

    def __init__(self, samples, with_quals=True):
        seqs, ab, qs = [], [], []
        starts = [0]
        for s in samples:
            seqs.extend(s.seqs)
            ab.append(np.asarray(s.abund, np.uint32))
            if with_quals:
                qs.extend(s.quals)
            starts.append(starts[-1] + len(s.seqs))
        self.cat, self.offs, self.lens, self.ab, self.qcat, self.pr = _pack(
            seqs, np.concatenate(ab), qs if with_quals else None, None)
        self.starts = np.array(starts, np.uint32)
        self.nsamples = len(samples)
        self.h2d_bytes = int(self.cat.nbytes + self.offs.nbytes + self.lens.nbytes + self.ab.nbytes +
                             (self.qcat.nbytes if self.qcat is not None else 0) + self.starts.nbytes)


def dada_uniques_batch(samples, err, ncol, params: DadaParams | None = None, device: int = 0,
                       packed: PackedBatch | None = None, read_results: bool = True):
    """Denoise many independent samples in one pass. ``samples`` are objects
    with ``seqs``, ``abund`` and ``quals`` (sums) attributes."""
    params = params or DadaParams()
    pb = packed or PackedBatch(samples)
    err = np.ascontiguousarray(err, np.float64)
    pc = params.c()
    hs = (C.c_void_p * pb.nsamples)()
    check(lib().dgpu_dada_batch(device, C.byref(pc), pb.nsamples, ptr(pb.starts), ptr(pb.cat), ptr(pb.offs),
                                ptr(pb.lens), ptr(pb.ab), ptr(pb.pr), ptr(pb.qcat), ptr(err), int(ncol),
                                C.cast(hs, C.c_void_p)))
    out = []
    try:
        for i in range(pb.nsamples):
            out.append(_read_result(hs[i]) if read_results else None)
    finally:
        for i in range(pb.nsamples):
            if hs[i]:
                lib().dgpu_result_free(hs[i])
    return out


class ResidentBatch:
    """Samples validated, encoded and uploaded once (inputs resident in HBM);
    ``run`` executes the whole clustering loop and may be repeated."""

    def __init__(self, samples, err, ncol, params: DadaParams | None = None, device: int = 0,
                 packed: PackedBatch | None = None):
        self.params = params or DadaParams()
        self.pb = packed or PackedBatch(samples)
        self._err = np.ascontiguousarray(err, np.float64)
        pc = self.params.c()
        self.h = C.c_void_p()
        pb = self.pb
        check(lib().dgpu_batch_prepare(device, C.byref(pc), pb.nsamples, ptr(pb.starts), ptr(pb.cat), ptr(pb.offs),
                                       ptr(pb.lens), ptr(pb.ab), ptr(pb.pr), ptr(pb.qcat), ptr(self._err), int(ncol),
                                       C.byref(self.h)))

    def run(self, read_results: bool = True):
        n = self.pb.nsamples
        hs = (C.c_void_p * n)()
        rc = lib().dgpu_batch_run(self.h, C.cast(hs, C.c_void_p))
        out = []
        try:
            check(rc)
            for i in range(n):
                out.append(_read_result(hs[i]) if read_results else _read_counters(hs[i]))
        finally:
            for i in range(n):
                if hs[i]:
                    lib().dgpu_result_free(hs[i])
        return out

    def close(self):
        if self.h:
            lib().dgpu_batch_free(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _read_counters(h) -> dict:
    cnt = np.zeros(16, np.uint64)
    tm = np.zeros(6, np.float64)
    o = DadaOutC(*[None] * len(DadaOutC._fields_))
    o.counters = ptr(cnt)
    o.times = ptr(tm)
    check(lib().dgpu_result_fill(h, C.byref(o)))
    sizes = np.zeros(4, np.int64)
    check(lib().dgpu_result_sizes(h, ptr(sizes)))
    mg = np.zeros(3, np.float64)
    check(lib().dgpu_result_margins(h, ptr(mg)))
    return {"nclust": int(sizes[0]), "nraw": int(sizes[1]),
            "counters": {k: int(v) for k, v in zip(COUNTER_KEYS, cnt)}, "times": tm,
            "margins": {"omega_a": float(mg[0]), "omega_p": float(mg[1]), "omega_c": float(mg[2])}}


class DenoiseService:
    """Requests (one sample each) submitted at any time and served on one
    device: pending requests of one length class are batched in arrival order
    within a device-memory budget and denoised together, so each result is
    ``dada_uniques``' on that sample. ``wait`` returns (result, latency in s)."""

    def __init__(self, err, ncol, params: DadaParams | None = None, device: int = 0, hbm_budget: int = 0):
        self.params = params or DadaParams()
        self._err = np.ascontiguousarray(err, np.float64)
        pc = self.params.c()
        self._live = {}
        self.h = C.c_void_p()
        check(lib().dgpu_service_create(device, C.byref(pc), ptr(self._err), int(ncol), int(hbm_budget),
                                        C.byref(self.h)))

    def submit(self, seqs=None, abund=None, quals=None, prior=None, packed=None) -> int:
        """Queue one sample; ``packed`` (from ``pack_sample``) skips packing.
        The packed buffers are held until the ticket's ``wait``."""
        pk = packed if packed is not None else _pack(seqs, abund, quals, prior)
        cat, offs, lens, ab, qcat, pr = pk
        t = C.c_uint64(0)
        check(lib().dgpu_service_submit(self.h, len(lens), ptr(cat), ptr(offs), ptr(lens), ptr(ab), ptr(pr),
                                        ptr(qcat), C.byref(t)))
        self._live[int(t.value)] = pk
        return int(t.value)

    def wait(self, ticket: int, read_result: bool = True):
        """(result, latency from submit to completion in s); without
        ``read_result`` the result carries its sizes and counters only."""
        h = C.c_void_p()
        lat = C.c_double(0.0)
        rc = lib().dgpu_service_wait(self.h, int(ticket), C.byref(h), C.byref(lat))
        self._live.pop(int(ticket), None)
        try:
            check(rc)
            return (_read_result(h) if read_result else _read_counters(h)), float(lat.value)
        finally:
            if h:
                lib().dgpu_result_free(h)

    def hold(self, held: bool = True):
        """While held no new batch starts; what is submitted meanwhile is
        batched together on release (``hold(False)``)."""
        check(lib().dgpu_service_hold(self.h, int(held)))

    def stats(self) -> dict:
        b, n = C.c_uint64(0), C.c_uint64(0)
        check(lib().dgpu_service_stats(self.h, C.byref(b), C.byref(n)))
        return {"batches": int(b.value), "served": int(n.value)}

    def close(self):
        if self.h:
            lib().dgpu_service_destroy(self.h)  # serves what is pending before the buffers go
            self.h = C.c_void_p()
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class Derep:
    """Uniques of a FASTQ file (src/derep.rs:43-240): ``seqs`` (str) by read
    count descending, ties by sequence; ``abund`` their counts; ``quals`` the
    per-position Phred sums (u32); ``map`` each read's unique."""
    seqs: list
    abund: np.ndarray
    quals: list
    map: np.ndarray


def derep_fastq(path, phred_offset: int = 33, nthreads: int = 0) -> Derep:
    """Dereplicate a FASTQ file (plain or gzip) on the host."""
    h = C.c_void_p()
    check(lib().dgpu_derep_fastq(str(path).encode(), int(phred_offset), int(nthreads), C.byref(h)))
    try:
        sz = np.zeros(3, np.int64)
        check(lib().dgpu_derep_sizes(h, ptr(sz)))
        nu, nr, nb = (int(x) for x in sz)
        cat = np.zeros(max(nb, 1), np.uint8)
        offs = np.zeros(max(nu, 1), np.uint32)
        lens = np.zeros(max(nu, 1), np.uint32)
        cnt = np.zeros(max(nu, 1), np.uint64)
        qs = np.zeros(max(nb, 1), np.uint32)
        mp = np.zeros(max(nr, 1), np.uint32)
        check(lib().dgpu_derep_fill(h, ptr(cat), ptr(offs), ptr(lens), ptr(cnt), ptr(qs), ptr(mp)))
    finally:
        lib().dgpu_derep_free(h)
    raw = cat.tobytes()
    seqs = [raw[o:o + n].decode("ascii", "replace") for o, n in zip(offs[:nu], lens[:nu])]
    quals = [qs[o:o + n].copy() for o, n in zip(offs[:nu], lens[:nu])]
    return Derep(seqs, cnt[:nu].copy(), quals, mp[:nr].copy())


def dada_fastq(path, err, ncol, params: DadaParams | None = None, phred_offset: int = 33, device: int = 0) -> dict:
    """FASTQ -> derep -> dada on the GPU: the `dada` subcommand's per-sample
    path (src/main.rs:1139-1257) up to its result tables."""
    d = derep_fastq(path, phred_offset)
    if np.any(d.abund > np.iinfo(np.uint32).max):
        raise InvalidInput(-1, "a unique has more than 2^32 - 1 reads")
    res = dada_uniques(d.seqs, d.abund.astype(np.uint32), err, ncol, params, quals=d.quals, device=device)
    res["derep"] = d
    return res


def calc_pA(reads: int, e_reads: float, prior: bool = False) -> float:
    """calc_pA (src/pval.rs:208-241), the library's FP64 p-value."""
    return float(lib().dgpu_calc_pA(int(reads), float(e_reads), int(bool(prior))))


def cache_release(device: int = -1) -> int:
    """Frees the device and pinned host blocks finished pools left for reuse
    (all devices when ``device`` < 0); returns the bytes given back."""
    n = C.c_uint64(0)
    check(lib().dgpu_cache_release(int(device), C.byref(n)))
    return int(n.value)


@dataclass
class ErrFun:
    """The error-model fit of learn-errors (src/learn_errors.rs:67-100):
    kind "loess" (surface "direct", the dada2-rs default, or "interpolate"
    with ``cell``, R's default), "noqual" (``pseudocount``), "binned"
    (piecewise linear between the anchor qualities ``bins``), "pacbio"
    (LOESS, with a maximum-likelihood Q93 column) or "external" (the command
    ``cmd`` fits the matrix from TSV files); off-diagonal rates clamped to
    [min_error_rate, max_error_rate]."""
    kind: str = "loess"
    surface: str = "direct"
    cell: float = 0.2
    max_error_rate: float = 0.25
    min_error_rate: float = 1e-7
    pseudocount: float = 1.0
    bins: tuple = ()
    cmd: str = ""

    def c(self) -> ErrFunC:
        kinds = {"loess": 0, "noqual": 1, "binned": 2, "pacbio": 3, "external": 4}
        surfaces = {"direct": 0, "interpolate": 1}
        b = np.ascontiguousarray(self.bins, np.float64)
        ef = ErrFunC(kinds[self.kind], surfaces[self.surface], float(self.cell), float(self.max_error_rate),
                     float(self.min_error_rate), float(self.pseudocount), b.ctypes.data if len(b) else None,
                     int(len(b)), self.cmd.encode() if self.cmd else None)
        ef._bins = b  # the anchors stay alive with the structure
        return ef


def errfun_apply(trans, nq: int, errfun: ErrFun | None = None) -> np.ndarray:
    """The 16 x nq error-rate matrix fitted to a 16 x nq transition matrix (host)."""
    t = np.ascontiguousarray(trans, np.uint32).reshape(-1)
    out = np.zeros(16 * nq, np.float64)
    ef = (errfun or ErrFun()).c()
    check(lib().dgpu_errfun_apply(C.byref(ef), ptr(t), int(nq), ptr(out)))
    return out.reshape(16, nq)


def learn_errors(samples, params: DadaParams | None = None, errfun: ErrFun | None = None, max_consist: int = 10,
                 device: int = 0) -> dict:
    """learn_errors (src/learn_errors.rs:739-1020): the self-consistent error
    model of the samples (objects with .seqs, .abund and .quals as Phred
    sums). Every pass denoises all samples together on the device and counts
    their transitions there. Returns nq, passes, converged and the last pass's
    trans, err_in and err_out (16 x nq)."""
    params = params or DadaParams()
    seqs = [q for s in samples for q in s.seqs]
    abund = np.concatenate([np.asarray(s.abund, np.uint32) for s in samples])
    quals = [q for s in samples for q in s.quals]
    cat, offs, lens, ab, qcat, _ = _pack(seqs, abund, quals, None)
    start = np.concatenate([[0], np.cumsum([len(s.seqs) for s in samples])]).astype(np.uint32)
    pc = params.c()
    ef = (errfun or ErrFun()).c()
    h = C.c_void_p()
    check(lib().dgpu_learn_errors(int(device), C.byref(pc), C.byref(ef), int(max_consist), len(samples), ptr(start),
                                  ptr(cat), ptr(offs), ptr(lens), ptr(ab), ptr(qcat), C.byref(h)))
    try:
        info = np.zeros(3, np.int32)
        check(lib().dgpu_learn_read(h, ptr(info), None, None, None))
        nq = int(info[0])
        tr = np.zeros(16 * nq, np.uint32)
        ei = np.zeros(16 * nq, np.float64)
        eo = np.zeros(16 * nq, np.float64)
        check(lib().dgpu_learn_read(h, ptr(info), ptr(tr), ptr(ei), ptr(eo)))
        return {"nq": nq, "passes": int(info[1]), "converged": bool(info[2]), "trans": tr.reshape(16, nq),
                "err_in": ei.reshape(16, nq), "err_out": eo.reshape(16, nq)}
    finally:
        lib().dgpu_learn_free(h)


TUNING_KEYS = [n for n, _ in TuningC._fields_]


def length_class(max_len: int) -> int:
    """The tuning table's read-length class: 0 up to 200 nt, 1 up to 600, 2 longer."""
    return 0 if max_len <= 200 else (1 if max_len <= 600 else 2)


def tuning_get(max_len: int) -> dict:
    """The launch shape a pool whose longest unique has ``max_len`` bases uses."""
    t = TuningC()
    check(lib().dgpu_tuning_get(int(max_len), C.byref(t)))
    return {k: int(getattr(t, k)) for k in TUNING_KEYS}


def tuning_set(cls: int, setting: dict):
    """Sets read-length class ``cls``'s launch shape (pools created later use it)."""
    t = TuningC(*[int(setting[k]) for k in TUNING_KEYS])
    check(lib().dgpu_tuning_set(int(cls), C.byref(t)))


def tuning_load(path: str):
    check(lib().dgpu_tuning_load(str(path).encode()))


def tuning_save(path: str):
    check(lib().dgpu_tuning_save(str(path).encode()))


def tuning_reset():
    """Back to the built-in table (no tuning file is read afterwards)."""
    check(lib().dgpu_tuning_reset())


def stats_reset():
    check(lib().dgpu_stats_reset())


def stats_timing(every):
    """Per-kernel device timing of every ``every``-th compare call (True = every
    call, False/0 = off)."""
    check(lib().dgpu_stats_timing(int(every)))


def stats_latencies() -> np.ndarray:
    """Per compare call latency (ms) since the last reset."""
    n = lib().dgpu_stats_latencies(None, 0)
    out = np.zeros(max(n, 1), np.float64)
    n = lib().dgpu_stats_latencies(ptr(out), len(out))
    return out[:n]


def stats_read() -> dict:
    s = KernelStatsC()
    check(lib().dgpu_stats_read(C.byref(s)))
    return {"launches": {k: int(s.launches[i]) for i, k in enumerate(KERNEL_NAMES)},
            "ms": {k: float(s.ms[i]) for i, k in enumerate(KERNEL_NAMES)},
            "rounds": int(s.rounds), "compares": int(s.compares), "screened": int(s.screened),
            "screen_bytes": int(s.screen_bytes), "timed_rounds": int(s.timed_rounds),
            "timed_screen_bytes": int(s.timed_screen_bytes), "timed_compares": int(s.timed_compares),
            "h2d_bytes": int(s.h2d_bytes),
            "batch_ms": {k: float(s.batch_ms[i]) for i, k in enumerate(("before", "loop", "after"))},
            "prepare_ms": {k: float(s.prepare_ms[i]) for i, k in enumerate(("encode", "upload", "slots", "copy_wait"))}}


ALIGN_VECTORIZED, ALIGN_HOMO, ALIGN_ENDSFREE = 0, 1, 2


def align_pairs(which: int, pairs, params: AlignParams | None = None, end_gap: int = 0, device: int = 0):
    """Run one of the GPU aligners on (s1, s2) code arrays; returns (al0, al1) rows."""
    params = params or AlignParams()
    s1 = [np.ascontiguousarray(a, np.uint8) for a, _ in pairs]
    s2 = [np.ascontiguousarray(b, np.uint8) for _, b in pairs]
    l1 = np.array([len(s) for s in s1], np.uint32)
    l2 = np.array([len(s) for s in s2], np.uint32)
    o1 = np.concatenate([[0], np.cumsum(l1)[:-1]]).astype(np.uint32)
    o2 = np.concatenate([[0], np.cumsum(l2)[:-1]]).astype(np.uint32)
    cap = l1.astype(np.int64) + l2
    ao = np.concatenate([[0], np.cumsum(cap)[:-1]]).astype(np.uint32)
    a0 = np.zeros(int(cap.sum()) + 1, np.uint8)
    a1 = np.zeros(int(cap.sum()) + 1, np.uint8)
    alen = np.zeros(len(pairs), np.uint32)
    c1, c2 = np.concatenate(s1), np.concatenate(s2)
    pc = params.c()
    check(lib().dgpu_align_debug(device, which, len(pairs), ptr(c1), ptr(o1), ptr(l1), ptr(c2), ptr(o2), ptr(l2),
                                 C.byref(pc), int(end_gap), ptr(a0), ptr(a1), ptr(ao), ptr(alen)))
    return [(a0[o:o + n].copy(), a1[o:o + n].copy()) for o, n in zip(ao, alen)]
