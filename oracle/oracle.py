"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py``; never by the product package. The oracle is a C++ restatement of
the Rust reference (HPCBio/dada2-rs 0.2.0): see ``dada_oracle.hpp``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_dada.so")
_lib = None

NT_CODE = {"A": 1, "C": 2, "G": 3, "T": 4, "U": 4, "N": 5}
METHOD_NAMES = {0: "none", 1: "gapless", 2: "vectorized", 3: "homo", 4: "endsfree"}


def build(force: bool = False) -> str:
    """Compile liboracle_dada.so with the committed Makefile (make rebuilds it
    only when a source is newer)."""
    if force and os.path.exists(_LIB_PATH):
        os.unlink(_LIB_PATH)
    if force or not os.path.exists(_LIB_PATH) or any(
            os.path.getmtime(os.path.join(_HERE, f)) > os.path.getmtime(_LIB_PATH)
            for f in os.listdir(_HERE) if f.endswith((".cpp", ".hpp"))):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class AlignParamsC(C.Structure):
    _fields_ = [
        ("match_score", C.c_int32), ("mismatch", C.c_int32), ("gap_p", C.c_int32),
        ("homo_gap_p", C.c_int32), ("use_kmers", C.c_int32), ("kdist_cutoff", C.c_double),
        ("kmer_size", C.c_int32), ("band", C.c_int32), ("vectorized", C.c_int32),
        ("gapless", C.c_int32),
    ]


class DadaParamsC(C.Structure):
    _fields_ = [
        ("align", AlignParamsC), ("omega_a", C.c_double), ("omega_p", C.c_double),
        ("omega_c", C.c_double), ("detect_singletons", C.c_int32), ("max_clust", C.c_int32),
        ("min_fold", C.c_double), ("min_hamming", C.c_uint32), ("min_abund", C.c_uint32),
        ("use_quals", C.c_int32), ("greedy", C.c_int32), ("nthreads", C.c_int32),
        ("transitions", C.c_int32),
    ]


class ErrFunC(C.Structure):
    _fields_ = [("kind", C.c_int32), ("surface", C.c_int32), ("cell", C.c_double),
                ("max_error_rate", C.c_double), ("min_error_rate", C.c_double), ("pseudocount", C.c_double),
                ("bins", C.c_void_p), ("nbins", C.c_int32)]


_P = C.c_void_p


class DadaOutC(C.Structure):
    _fields_ = [(n, _P) for n in (
        "cl_reads", "cl_birth_type", "cl_birth_from", "cl_birth_pval", "cl_birth_fold",
        "cl_birth_e", "cl_birth_hamming", "cl_seq_off", "cl_seq", "cl_mem_off", "mem_raw",
        "mem_hamming", "mem_lambda", "mem_pval", "map", "pvals", "counters", "times")]


@dataclass
class AlignParams:
    """src/nwalign.rs:63-90 (defaults from src/main.rs:4393-4433)."""
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


@dataclass
class DadaParams:
    """src/dada.rs:54-101, the fields the compare loop reads."""
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
    nthreads: int = 1
    transitions: bool = False  # also return the DadaAux transition counts (src/error.rs:194-249)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise RuntimeError(f"oracle library missing: {_LIB_PATH} (run `make -C oracle`)")
        _lib = C.CDLL(_LIB_PATH)
        d = C.c_double
        _lib.orc_c_kmer_dist8.restype = d
        _lib.orc_c_kmer_dist.restype = d
        _lib.orc_c_kmer_dist8_sparse.restype = d
        _lib.orc_c_kord_dist.restype = d
        _lib.orc_c_calc_pA.restype = d
        _lib.orc_c_calc_pA.argtypes = [C.c_uint32, d, C.c_int]
        _lib.orc_c_gamma_lr.restype = d
        _lib.orc_c_gamma_lr.argtypes = [d, d]
        _lib.orc_c_ln_gamma.restype = d
        _lib.orc_c_ln_gamma.argtypes = [d]
        _lib.orc_c_get_pA.restype = d
        _lib.orc_c_get_pA.argtypes = [C.c_uint32, C.c_int, d, C.c_uint32, C.c_uint32, C.c_int]
        _lib.orc_c_assign_kmer8_sparse.restype = C.c_size_t
        _lib.orc_c_b_new.restype = C.c_void_p
        _lib.orc_c_b_new.argtypes = [C.c_int, _P, _P, _P, _P, _P, _P, C.c_int, C.c_int, d, d, C.c_int]
        _lib.orc_c_b_free.argtypes = [C.c_void_p]
        _lib.orc_c_b_center.argtypes = [C.c_void_p, C.c_int]
        _lib.orc_c_b_set_center.argtypes = [C.c_void_p, C.c_int, C.c_int]
        _lib.orc_c_b_set_lock.argtypes = [C.c_void_p, C.c_int, C.c_int]
        _lib.orc_c_b_add_center.argtypes = [C.c_void_p, C.c_int]
        _lib.orc_c_compare_map.argtypes = [C.c_void_p, C.c_int, _P, C.c_int, C.POINTER(AlignParamsC),
                                           C.c_int, C.c_int, _P, _P, _P, _P]
        _lib.orc_c_b_compare.argtypes = [C.c_void_p, C.c_int, _P, C.c_int, C.POINTER(AlignParamsC),
                                         C.c_int, C.c_int, _P, _P, _P, _P, _P, _P]
        _lib.orc_c_errfun_apply.restype = C.c_int
        _lib.orc_c_errfun_apply.argtypes = [C.POINTER(ErrFunC), _P, C.c_int, _P, C.c_char_p, C.c_int]
        _lib.orc_c_learn_errors.restype = C.c_int
        _lib.orc_c_learn_errors.argtypes = [C.c_int, _P, _P, _P, _P, _P, _P, C.POINTER(DadaParamsC),
                                            C.POINTER(ErrFunC), C.c_int, C.c_int, _P, _P, _P, _P, C.c_char_p,
                                            C.c_int]
        _lib.orc_c_dada.restype = C.c_void_p
        _lib.orc_c_dada.argtypes = [C.c_int, _P, _P, _P, _P, _P, _P, C.POINTER(DadaParamsC), _P,
                                    C.c_int, C.c_char_p, C.c_int]
        _lib.orc_c_dada_free.argtypes = [C.c_void_p]
        _lib.orc_c_dada_sizes.argtypes = [C.c_void_p, _P]
        _lib.orc_c_dada_fill.argtypes = [C.c_void_p, C.POINTER(DadaOutC)]
        _lib.orc_c_dada_transitions.argtypes = [C.c_void_p, _P]
        _lib.orc_c_dada_transitions.restype = C.c_int
    return _lib


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def encode(seq: str) -> np.ndarray:
    """ASCII -> 1..5 codes (the test helper at src/nwalign.rs:1858-1868)."""
    return np.array([NT_CODE.get(ch.upper(), 5) for ch in seq], dtype=np.uint8)


def align_params_c(p) -> AlignParamsC:
    return AlignParamsC(int(p.match_score), int(p.mismatch), int(p.gap_p), int(p.homo_gap_p),
                        int(bool(p.use_kmers)), float(p.kdist_cutoff), int(p.kmer_size),
                        int(p.band), int(bool(p.vectorized)), int(bool(p.gapless)))


def dada_params_c(p) -> DadaParamsC:
    return DadaParamsC(align_params_c(p.align), float(p.omega_a), float(p.omega_p),
                       float(p.omega_c), int(bool(p.detect_singletons)), int(p.max_clust),
                       float(p.min_fold), int(p.min_hamming), int(p.min_abund),
                       int(bool(p.use_quals)), int(bool(p.greedy)), int(p.nthreads),
                       int(bool(getattr(p, "transitions", False))))


# ---------------- kmers ----------------
def assign_kmer(seq: np.ndarray, k: int) -> np.ndarray:
    out = np.zeros(4 ** k, np.uint16)
    seq = np.ascontiguousarray(seq, np.uint8)
    lib().orc_c_assign_kmer(_ptr(seq), C.c_size_t(len(seq)), k, _ptr(out))
    return out


def assign_kmer8(seq: np.ndarray, k: int) -> np.ndarray:
    out = np.zeros(4 ** k, np.uint8)
    seq = np.ascontiguousarray(seq, np.uint8)
    lib().orc_c_assign_kmer8(_ptr(seq), C.c_size_t(len(seq)), k, _ptr(out))
    return out


def assign_kmer8_sparse(seq: np.ndarray, k: int):
    idx = np.zeros(4 ** k, np.uint16)
    cnt = np.zeros(4 ** k, np.uint8)
    seq = np.ascontiguousarray(seq, np.uint8)
    n = lib().orc_c_assign_kmer8_sparse(_ptr(seq), C.c_size_t(len(seq)), k, _ptr(idx), _ptr(cnt))
    return idx[:n].copy(), cnt[:n].copy()


def assign_kmer_order(seq: np.ndarray, k: int) -> np.ndarray:
    out = np.zeros(max(len(seq) - k + 1, 0), np.uint16)
    seq = np.ascontiguousarray(seq, np.uint8)
    lib().orc_c_assign_kmer_order(_ptr(seq), C.c_size_t(len(seq)), k, _ptr(out))
    return out


def kmer_dist8(a, l1, b, l2, k) -> float:
    return lib().orc_c_kmer_dist8(_ptr(a), C.c_size_t(l1), _ptr(b), C.c_size_t(l2), k)


def kmer_dist(a, l1, b, l2, k) -> float:
    return lib().orc_c_kmer_dist(_ptr(a), C.c_size_t(l1), _ptr(b), C.c_size_t(l2), k)


def kmer_dist8_sparse(sa, l1, sb, l2, k) -> float:
    (ia, ca), (ib, cb) = sa, sb
    return lib().orc_c_kmer_dist8_sparse(_ptr(ia), _ptr(ca), C.c_size_t(len(ia)), C.c_size_t(l1),
                                         _ptr(ib), _ptr(cb), C.c_size_t(len(ib)), C.c_size_t(l2), k)


def kord_dist(a, l1, b, l2, k) -> float:
    return lib().orc_c_kord_dist(_ptr(a), C.c_size_t(l1), _ptr(b), C.c_size_t(l2), k)


# ---------------- aligners ----------------
ALIGN_VECTORIZED, ALIGN_VECTORIZED_FULL, ALIGN_ENDSFREE, ALIGN_HOMO, ALIGN_GAPLESS = range(5)


def align(which: int, s1, s2, match=5, mismatch=-4, gap=-8, homo_gap=-8, end_gap=0, band=16):
    s1 = np.ascontiguousarray(s1, np.uint8)
    s2 = np.ascontiguousarray(s2, np.uint8)
    cap = len(s1) + len(s2) + 1
    a0 = np.zeros(cap, np.uint8)
    a1 = np.zeros(cap, np.uint8)
    n = lib().orc_c_align(which, _ptr(s1), C.c_size_t(len(s1)), _ptr(s2), C.c_size_t(len(s2)),
                          match, mismatch, gap, homo_gap, end_gap, band, _ptr(a0), _ptr(a1))
    return a0[:n].copy(), a1[:n].copy()


def align_vectorized_reuse(pairs, match=5, mismatch=-4, gap=-8, end_gap=0, band=16):
    s1s = [np.ascontiguousarray(a, np.uint8) for a, _ in pairs]
    s2s = [np.ascontiguousarray(b, np.uint8) for _, b in pairs]
    s1cat = np.concatenate(s1s)
    s2cat = np.concatenate(s2s)
    l1 = np.array([len(s) for s in s1s], np.uint32)
    l2 = np.array([len(s) for s in s2s], np.uint32)
    o1 = np.concatenate([[0], np.cumsum(l1)[:-1]]).astype(np.uint32)
    o2 = np.concatenate([[0], np.cumsum(l2)[:-1]]).astype(np.uint32)
    cap = int(l1.sum() + l2.sum()) + 1
    a0 = np.zeros(cap, np.uint8)
    a1 = np.zeros(cap, np.uint8)
    alen = np.zeros(len(pairs), np.uint32)
    lib().orc_c_align_vectorized_reuse(len(pairs), _ptr(s1cat), _ptr(o1), _ptr(l1), _ptr(s2cat),
                                       _ptr(o2), _ptr(l2), match, mismatch, gap, end_gap, band,
                                       _ptr(a0), _ptr(a1), _ptr(alen))
    out, w = [], 0
    for n in alen:
        out.append((a0[w:w + n].copy(), a1[w:w + n].copy()))
        w += int(n)
    return out


def raw_align(s1, s2, params):
    """Screen + dispatch; returns (method_name, al0, al1, kdist, kodist)."""
    s1 = np.ascontiguousarray(s1, np.uint8)
    s2 = np.ascontiguousarray(s2, np.uint8)
    cap = len(s1) + len(s2) + 1
    a0 = np.zeros(cap, np.uint8)
    a1 = np.zeros(cap, np.uint8)
    alen = C.c_int(0)
    kd = C.c_double(0)
    kod = C.c_double(0)
    pc = align_params_c(params)
    m = lib().orc_c_raw_align(_ptr(s1), C.c_size_t(len(s1)), _ptr(s2), C.c_size_t(len(s2)),
                              C.byref(pc), _ptr(a0), _ptr(a1), C.byref(alen), C.byref(kd),
                              C.byref(kod))
    n = alen.value
    return METHOD_NAMES[m], a0[:n].copy(), a1[:n].copy(), kd.value, kod.value


def al2subs(al0, al1):
    al0 = np.ascontiguousarray(al0, np.uint8)
    al1 = np.ascontiguousarray(al1, np.uint8)
    n = len(al0)
    len0 = C.c_uint32(0)
    mp = np.zeros(n + 1, np.uint16)
    pos = np.zeros(n + 1, np.uint16)
    nt0 = np.zeros(n + 1, np.uint8)
    nt1 = np.zeros(n + 1, np.uint8)
    ns = lib().orc_c_al2subs(_ptr(al0), _ptr(al1), n, C.byref(len0), _ptr(mp), _ptr(pos),
                             _ptr(nt0), _ptr(nt1))
    return {"len0": len0.value, "map": mp[:len0.value].copy(), "pos": pos[:ns].copy(),
            "nt0": nt0[:ns].copy(), "nt1": nt1[:ns].copy()}


def calc_pA(reads: int, e_reads: float, prior: bool) -> float:
    return lib().orc_c_calc_pA(reads, e_reads, int(prior))


def gamma_lr(a: float, x: float) -> float:
    return lib().orc_c_gamma_lr(a, x)


def ln_gamma(x: float) -> float:
    """lnGamma as statrs 0.18.0 computes it (Lanczos, Pugh's r = 10.900511)."""
    return lib().orc_c_ln_gamma(x)


def get_pA(reads, prior, lam, hamming, bi_reads, detect_singletons=False) -> float:
    return lib().orc_c_get_pA(reads, int(prior), lam, hamming, bi_reads, int(detect_singletons))


def score_alignment(al0, al1, match=5, mismatch=-4, gap=-8) -> int:
    """Ends-free score of an alignment (the test helper at src/nwalign.rs:1814-1855)."""
    gap_b = ord("-")
    n = len(al0)
    score = 0
    for k in range(n):
        g0 = al0[k] == gap_b
        g1 = al1[k] == gap_b
        if not g0 and not g1:
            score += match if al0[k] == al1[k] else mismatch
        elif g0:
            at_start = all(b == gap_b for b in al0[:k])
            at_end = all(b == gap_b for b in al0[k + 1:])
            if not at_start and not at_end:
                score += gap
        else:
            at_start = all(b == gap_b for b in al1[:k])
            at_end = all(b == gap_b for b in al1[k + 1:])
            if not at_start and not at_end:
                score += gap
    return score


# ---------------- compare session ----------------
class Session:
    """A `B` holding encoded raws with every raw in cluster 0 (src/containers.rs:337-390)."""

    def __init__(self, seqs, reads, quals=None, prior=None, k=5, use_kmers=True,
                 omega_a=1e-40, omega_p=1e-4, use_quals=True):
        self.n = len(seqs)
        seqs = [np.ascontiguousarray(s, np.uint8) for s in seqs]
        lens = np.array([len(s) for s in seqs], np.uint32)
        offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.uint32)
        cat = np.concatenate(seqs).astype(np.uint8)
        qcat = None if quals is None else np.concatenate(
            [np.ascontiguousarray(q, np.uint8) for q in quals]).astype(np.uint8)
        rd = np.ascontiguousarray(reads, np.uint32)
        pr = None if prior is None else np.ascontiguousarray(prior, np.uint8)
        self._keep = (cat, qcat, rd, pr, lens, offs)
        self.h = lib().orc_c_b_new(self.n, _ptr(cat), _ptr(offs), _ptr(lens), _ptr(qcat), _ptr(rd),
                                   _ptr(pr), k, int(use_kmers), omega_a, omega_p, int(use_quals))

    def close(self):
        if self.h:
            lib().orc_c_b_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def center(self, ci=0) -> int:
        return lib().orc_c_b_center(self.h, ci)

    def set_center(self, ci, center):
        lib().orc_c_b_set_center(self.h, ci, center)

    def set_lock(self, raw, lock=True):
        lib().orc_c_b_set_lock(self.h, raw, int(lock))

    def add_center(self, center) -> int:
        return lib().orc_c_b_add_center(self.h, center)

    def compare_map(self, ci, err, ncol, params, greedy=True, nthreads=1):
        err = np.ascontiguousarray(err, np.float64)
        lam = np.zeros(self.n, np.float64)
        ham = np.zeros(self.n, np.uint32)
        skp = np.zeros(self.n, np.uint8)
        meth = np.zeros(self.n, np.int32)
        pc = align_params_c(params)
        lib().orc_c_compare_map(self.h, ci, _ptr(err), ncol, C.byref(pc), int(greedy), nthreads,
                                _ptr(lam), _ptr(ham), _ptr(skp), _ptr(meth))
        return lam, ham, skp.astype(bool), meth

    def compare(self, ci, err, ncol, params, greedy=True, nthreads=1):
        err = np.ascontiguousarray(err, np.float64)
        idx = np.zeros(self.n, np.uint32)
        lam = np.zeros(self.n, np.float64)
        ham = np.zeros(self.n, np.uint32)
        emm = np.zeros(self.n, np.float64)
        self_ = C.c_double(0)
        cnt = np.zeros(9, np.uint64)
        pc = align_params_c(params)
        ns = lib().orc_c_b_compare(self.h, ci, _ptr(err), ncol, C.byref(pc), int(greedy), nthreads,
                                   _ptr(idx), _ptr(lam), _ptr(ham), _ptr(emm), C.byref(self_),
                                   _ptr(cnt))
        keys = ["nalign", "nshroud", "screened", "aligned", "stored", "gapless", "vectorized",
                "homo", "endsfree"]
        return {"index": idx[:ns].copy(), "lambda": lam[:ns].copy(), "hamming": ham[:ns].copy(),
                "e_minmax": emm, "self": self_.value,
                "counters": {k: int(v) for k, v in zip(keys, cnt)}}


# ---------------- full dada ----------------
COUNTER_KEYS = ["nalign", "compare_calls", "cmp_scanned", "screened", "aligned", "stored",
                "gapless", "vectorized", "homo", "endsfree", "shuffle_calls", "shuffle_moves",
                "nshroud"]


def pack_inputs(seqs, abund, quals=None, prior=None):
    """Concatenate ASCII uniques (+ optional per-position Phred sums)."""
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


def unpack_result(sizes, fill_fn):
    """Shared reader for the flat result layout (oracle and product use the same one)."""
    ncl, nraw, nmem, nseq = (int(x) for x in sizes)
    arrs = {
        "cl_reads": np.zeros(ncl, np.uint32), "cl_birth_type": np.zeros(ncl, np.int32),
        "cl_birth_from": np.zeros(ncl, np.uint32), "cl_birth_pval": np.zeros(ncl, np.float64),
        "cl_birth_fold": np.zeros(ncl, np.float64), "cl_birth_e": np.zeros(ncl, np.float64),
        "cl_birth_hamming": np.zeros(ncl, np.uint32), "cl_seq_off": np.zeros(ncl + 1, np.uint32),
        "cl_seq": np.zeros(max(nseq, 1), np.uint8), "cl_mem_off": np.zeros(ncl + 1, np.uint32),
        "mem_raw": np.zeros(max(nmem, 1), np.uint32), "mem_hamming": np.zeros(max(nmem, 1), np.uint32),
        "mem_lambda": np.zeros(max(nmem, 1), np.float64), "mem_pval": np.zeros(max(nmem, 1), np.float64),
        "map": np.zeros(max(nraw, 1), np.int32), "pvals": np.zeros(max(nraw, 1), np.float64),
        "counters": np.zeros(16, np.uint64), "times": np.zeros(4, np.float64),
    }
    fill_fn(arrs)
    res = {"nclust": ncl, "nraw": nraw}
    res.update({k: v for k, v in arrs.items()})
    res["map"] = arrs["map"][:nraw]
    res["pvals"] = arrs["pvals"][:nraw]
    res["counters"] = {k: int(v) for k, v in zip(COUNTER_KEYS, arrs["counters"])}
    res["clusters"] = []
    for ci in range(ncl):
        s0, s1 = arrs["cl_seq_off"][ci], arrs["cl_seq_off"][ci + 1]
        m0, m1 = arrs["cl_mem_off"][ci], arrs["cl_mem_off"][ci + 1]
        res["clusters"].append({
            "sequence": arrs["cl_seq"][s0:s1].copy(), "reads": int(arrs["cl_reads"][ci]),
            "members": arrs["mem_raw"][m0:m1].copy(), "hammings": arrs["mem_hamming"][m0:m1].copy(),
            "lambdas": arrs["mem_lambda"][m0:m1].copy(), "pvals": arrs["mem_pval"][m0:m1].copy(),
            "birth_type": int(arrs["cl_birth_type"][ci]), "birth_from": int(arrs["cl_birth_from"][ci]),
            "birth_pval": float(arrs["cl_birth_pval"][ci]), "birth_fold": float(arrs["cl_birth_fold"][ci]),
            "birth_e": float(arrs["cl_birth_e"][ci]), "birth_hamming": int(arrs["cl_birth_hamming"][ci]),
        })
    return res


def dada(seqs, abund, err, ncol, params: DadaParams, quals=None, prior=None):
    """dada_uniques (src/dada.rs:225-592) on ASCII uniques. Raises ValueError on bad input."""
    cat, offs, lens, ab, qcat, pr = pack_inputs(seqs, abund, quals, prior)
    err = np.ascontiguousarray(err, np.float64)
    pc = dada_params_c(params)
    eb = C.create_string_buffer(512)
    h = lib().orc_c_dada(len(lens), _ptr(cat), _ptr(offs), _ptr(lens), _ptr(ab), _ptr(pr),
                         _ptr(qcat), C.byref(pc), _ptr(err), ncol, eb, 512)
    if not h:
        raise ValueError(eb.value.decode())
    try:
        sizes = np.zeros(4, np.int64)
        lib().orc_c_dada_sizes(h, _ptr(sizes))

        def fill(a):
            o = DadaOutC(*[_ptr(a[n]) for n, _ in DadaOutC._fields_])
            lib().orc_c_dada_fill(h, C.byref(o))

        res = unpack_result(sizes, fill)
        tncol = lib().orc_c_dada_transitions(h, None)
        if tncol:
            tr = np.zeros(16 * tncol, np.uint32)
            lib().orc_c_dada_transitions(h, _ptr(tr))
            res["transitions"] = tr.reshape(16, tncol)
        return res
    finally:
        lib().orc_c_dada_free(h)


ERRFUN_LOESS, ERRFUN_NOQUAL, ERRFUN_BINNED, ERRFUN_PACBIO = 0, 1, 2, 3


def errfun_c(kind=ERRFUN_LOESS, surface=0, cell=0.2, max_error_rate=0.25, min_error_rate=1e-7, pseudocount=1.0,
             bins=None):
    """kind 0 LOESS, 1 noqual, 2 binned quality (anchors `bins`), 3 PacBio. The
    returned structure keeps the anchors' array alive as `_bins`."""
    b = np.ascontiguousarray(bins if bins is not None else [], np.float64)
    ef = ErrFunC(int(kind), int(surface), float(cell), float(max_error_rate), float(min_error_rate),
                 float(pseudocount), b.ctypes.data if len(b) else None, int(len(b)))
    ef._bins = b
    return ef


def errfun_apply(trans, nq, **kw) -> np.ndarray:
    """The error-model fit (loess_errfun / noqual_errfun) of a 16 x nq
    transition matrix; raises ValueError when LOESS fails everywhere."""
    t = np.ascontiguousarray(trans, np.uint32).reshape(-1)
    out = np.zeros(16 * nq, np.float64)
    eb = C.create_string_buffer(256)
    ef = errfun_c(**kw)
    if lib().orc_c_errfun_apply(C.byref(ef), _ptr(t), int(nq), _ptr(out), eb, 256) != 0:
        raise ValueError(eb.value.decode())
    return out.reshape(16, nq)


def learn_errors(samples, params: DadaParams, max_consist=10, **errfun_kw) -> dict:
    """learn_errors (src/learn_errors.rs:739-1020) over samples (objects with
    .seqs, .abund, .quals as Phred sums)."""
    seqs = [q for s in samples for q in s.seqs]
    abund = np.concatenate([np.asarray(s.abund, np.uint32) for s in samples])
    quals = [q for s in samples for q in s.quals]
    cat, offs, lens, ab, qcat, _ = pack_inputs(seqs, abund, quals, None)
    start = np.concatenate([[0], np.cumsum([len(s.seqs) for s in samples])]).astype(np.uint32)
    pc = dada_params_c(params)
    ef = errfun_c(**errfun_kw)
    cap = 256
    info = np.zeros(3, np.int32)
    tr = np.zeros(16 * cap, np.uint32)
    ei = np.zeros(16 * cap, np.float64)
    eo = np.zeros(16 * cap, np.float64)
    eb = C.create_string_buffer(512)
    nq = lib().orc_c_learn_errors(len(samples), _ptr(start), _ptr(cat), _ptr(offs), _ptr(lens), _ptr(ab), _ptr(qcat),
                                  C.byref(pc), C.byref(ef), int(max_consist), cap, _ptr(info), _ptr(tr), _ptr(ei),
                                  _ptr(eo), eb, 512)
    if nq < 0:
        raise ValueError(eb.value.decode())
    return {"nq": int(info[0]), "passes": int(info[1]), "converged": bool(info[2]),
            "trans": tr[:16 * nq].reshape(16, nq).copy(), "err_in": ei[:16 * nq].reshape(16, nq).copy(),
            "err_out": eo[:16 * nq].reshape(16, nq).copy()}


def hardware_threads() -> int:
    return int(lib().orc_c_hardware_threads())


# ---------------- derep (pure Python restatement) ----------------

def read_fastq_records(path):
    """Four-line FASTQ records (plain or gzip) as (sequence bytes, quality bytes)."""
    import gzip

    with open(path, "rb") as f:
        head = f.read(2)
    opener = gzip.open if head == b"\x1f\x8b" else open
    with opener(path, "rb") as f:
        lines = f.read().split(b"\n")
    if lines and lines[-1] == b"":
        lines.pop()
    lines = [ln[:-1] if ln.endswith(b"\r") else ln for ln in lines]
    recs = []
    for i in range(0, len(lines), 4):
        h, s, p, q = (lines[i:i + 4] + [b"", b"", b""])[:4]
        if not h.startswith(b"@") or not p.startswith(b"+") or len(s) != len(q):
            raise ValueError(f"record {i // 4}: malformed")
        recs.append((s, q))
    return recs


def derep(records, phred_offset: int = 33):
    """src/derep.rs:84-240: group identical sequences in first-seen order,
    count reads and sum (quality - offset) per position, store round(sum) as
    u32 (negative -> 0), then order by count descending, ties by sequence
    bytes ascending; map gives each read's unique."""
    index, seqs, counts, sums, local = {}, [], [], [], []
    for s, q in records:
        j = index.get(s)
        if j is None:
            j = len(seqs)
            index[s] = j
            seqs.append(s)
            counts.append(0)
            sums.append([0] * len(q))
        counts[j] += 1
        local.append(j)
        row = sums[j]
        if len(q) > len(row):
            row.extend([0] * (len(q) - len(row)))
        for p, c in enumerate(q):
            row[p] += c - phred_offset
    order = sorted(range(len(seqs)), key=lambda t: (-counts[t], seqs[t]))
    new = {old: k for k, old in enumerate(order)}
    return ([seqs[t].decode() for t in order], np.array([counts[t] for t in order], np.uint64),
            [np.array([max(v, 0) for v in sums[t]], np.uint32) for t in order],
            np.array([new[j] for j in local], np.uint32))
