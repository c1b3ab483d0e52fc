"""Pin the oracle's k-mer screen, compare store and p-values to the reference.

K-mer cases restate src/kmers.rs:330-401; the compare pool restates
src/cluster.rs:1786-1922; tie rules src/cluster.rs:1697-1777. calc_pA has no
reference test (statrs 0.18 is not vendored), so it is checked against
scipy's regularised incomplete gamma instead.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O

MASK64 = (1 << 64) - 1


def make_seq(n, seed, kt):
    s, out = seed, []
    for _ in range(n):
        s = (s * kt["mul"] + kt["add"]) & MASK64
        out.append(((s >> 33) % 4) + 1)
    return np.array(out, np.uint8)


def test_sparse_reconstructs_dense(refvec):
    kt = refvec["kmer_tests"]
    for k in kt["ks"]:
        for seed in range(kt["reconstruct_seeds"]):
            seq = make_seq(kt["reconstruct_len"], seed, kt)
            dense = O.assign_kmer8(seq, k)
            idx, cnt = O.assign_kmer8_sparse(seq, k)
            assert np.all(np.diff(idx.astype(np.int64)) > 0)
            rec = np.zeros(4 ** k, np.uint8)
            rec[idx] = cnt
            assert np.array_equal(dense, rec)


def test_sparse_dist_matches_dense(refvec):
    kt = refvec["kmer_tests"]
    for k in kt["ks"]:
        for seed in range(kt["dist_seeds"]):
            a = make_seq(kt["dist_len"], seed, kt)
            b = make_seq(kt["dist_len"], seed + kt["dist_seed_offset"], kt)
            d = O.kmer_dist8(O.assign_kmer8(a, k), len(a), O.assign_kmer8(b, k), len(b), k)
            s = O.kmer_dist8_sparse(O.assign_kmer8_sparse(a, k), len(a), O.assign_kmer8_sparse(b, k), len(b), k)
            assert np.float64(d).tobytes() == np.float64(s).tobytes()
            sa = O.assign_kmer8_sparse(a, k)
            assert O.kmer_dist8_sparse(sa, len(a), sa, len(a), k) == 0.0


def test_overflow_returns_minus_one(refvec):
    kt = refvec["kmer_tests"]
    k = kt["overflow_k"]
    seq = np.full(kt["overflow_len"], kt["overflow_nt"], np.uint8)
    dense = O.assign_kmer8(seq, k)
    assert O.kmer_dist8(dense, len(seq), dense, len(seq), k) == -1.0
    sp = O.assign_kmer8_sparse(seq, k)
    assert O.kmer_dist8_sparse(sp, len(seq), sp, len(seq), k) == -1.0
    # the u16 fallback is exact: identical sequences are at distance 0
    v = O.assign_kmer(seq, k)
    assert O.kmer_dist(v, len(seq), v, len(seq), k) == 0.0


def test_kord_dist_lengths():
    a = O.encode("ACGTACGTACGTAAC")
    b = O.encode("ACGTACGTACGTAAG")
    k = 5
    ka, kb = O.assign_kmer_order(a, k), O.assign_kmer_order(b, k)
    assert O.kord_dist(ka, len(a), kb, len(b), k) == pytest.approx(1.0 - 10.0 / 11.0)
    c = O.encode("ACGTACGTACGTAA")
    assert O.kord_dist(ka, len(a), O.assign_kmer_order(c, k), len(c), k) == -1.0


def pool_session(refvec):
    pl = refvec["compare_pool"]
    base = list(pl["base"])
    nxt = {"A": "C", "C": "G", "G": "T"}
    seqs, reads = [], []
    for n, r in pl["n_reads"]:
        s = list(base)
        for p in range(n):
            idx = (p * pl["mut_mul"] + pl["mut_add"]) % len(s)
            s[idx] = nxt.get(s[idx], "A")
        seqs.append(O.encode("".join(s)))
        reads.append(r)
    sess = O.Session(seqs, reads, k=pl["k"], use_quals=False)
    sess.set_center(0, pl["center"])
    params = O.AlignParams(homo_gap_p=pl["homo_gap_p"], kdist_cutoff=pl["kdist_cutoff"],
                           kmer_size=pl["k"], band=pl["band"])
    err = np.full(16 * pl["ncol"], pl["err_flat"])
    return sess, params, err, pl["ncol"]


def test_compare_pool_folded_counters(refvec):
    for greedy in (False, True):
        sess, params, err, ncol = pool_session(refvec)
        out = sess.compare(0, err, ncol, params, greedy=greedy, nthreads=4)
        c = out["counters"]
        assert c["screened"] == c["nalign"]
        assert c["screened"] - c["aligned"] == c["nshroud"]
        assert c["stored"] == len(out["index"])
        assert c["screened"] <= sess.n
        assert c["aligned"] > 0 and c["nshroud"] > 0 and c["stored"] > 0
        if greedy:
            assert c["screened"] < sess.n
        sess.close()


def test_compare_pool_parallel_matches_serial(refvec):
    for greedy in (False, True):
        a, params, err, ncol = pool_session(refvec)
        b, _, _, _ = pool_session(refvec)
        pa = a.compare(0, err, ncol, params, greedy=greedy, nthreads=4)
        sb = b.compare(0, err, ncol, params, greedy=greedy, nthreads=1)
        assert pa["counters"] == sb["counters"]
        assert np.array_equal(pa["index"], sb["index"])
        assert np.array_equal(pa["hamming"], sb["hamming"])
        assert pa["lambda"].tobytes() == sb["lambda"].tobytes()


def test_compare_pool_uses_homopolymer_aligner(refvec):
    sess, params, err, ncol = pool_session(refvec)
    lam, ham, skp, meth = sess.compare_map(0, err, ncol, params, greedy=False)
    names = {O.METHOD_NAMES[int(m)] for m in meth}
    assert "gapless" in names and "none" in names


def fold_beats(cands):
    """Pairwise `beats` (src/cluster.rs:781-783) folded in the given order."""
    e_cur, ci_cur = -math.inf, 2 ** 32 - 1
    for e, ci in cands:
        if e > e_cur or (e == e_cur and ci < ci_cur):
            e_cur, ci_cur = e, ci
    return ci_cur


def test_tie_rules(refvec):
    for case in refvec["tie_cases"]:
        cands = [(e, int(ci)) for e, ci in case["cands"]]
        assert fold_beats(cands) == case["winner"]
        srt = sorted(cands, key=lambda t: t[1])
        best_e, best = -math.inf, None
        for e, ci in srt:
            if e > best_e:
                best_e, best = e, ci
        assert best == case["winner"]


@pytest.mark.parametrize("reads", [1, 2, 3, 5, 10, 37, 100, 1000, 20000])
@pytest.mark.parametrize("lam", [1e-3, 0.05, 0.7, 1.0, 3.5, 12.0, 150.0, 999.0, 25000.0])
def test_calc_pA_matches_incomplete_gamma(reads, lam):
    sp = pytest.importorskip("scipy.special")
    want = float(sp.gammainc(reads, lam))  # P(X >= reads | Poisson(lam))
    got = O.calc_pA(reads, lam, True)
    if want > 1e-280:
        assert got == pytest.approx(want, rel=1e-11, abs=0.0)
    norm = 1.0 - math.exp(-lam)
    if norm >= 1e-7:
        assert O.calc_pA(reads, lam, False) == pytest.approx(got / norm, rel=1e-15)


def test_ln_gamma_is_the_lanczos_form_statrs_documents():
    """statrs 0.18.0 computes lnGamma by the Lanczos approximation with Pugh's
    r = 10.900511 and eleven coefficients (accurate to about 16 digits), not
    by the C library: it agrees with lgamma to ~1e-15 relative but not to the
    bit (lnGamma(1) is -4.4e-16 there, a known property of that form)."""
    for x in (0.5, 0.75, 1.0, 1.5, 2.0, 3.0, 7.5, 10.0, 41.0, 100.0, 999.5, 12345.0, 65535.0, 1e6):
        got, want = O.ln_gamma(x), math.lgamma(x)
        assert got == pytest.approx(want, rel=2e-14, abs=2e-15), x
    assert O.ln_gamma(1.0) == -4.440892098500626e-16
    assert O.ln_gamma(2.0) == 0.0
    # ln(k!) = lnGamma(k + 1) over the read counts the p-values see
    acc = 0.0
    for k in range(1, 3000):
        acc += math.log(k)
        assert O.ln_gamma(k + 1.0) == pytest.approx(acc, rel=1e-13, abs=1e-14)


def test_gamma_lr_answers_zero_within_statrs_accuracy_of_zero():
    """statrs' gamma_lr returns 0.0 for x within its default accuracy
    (10 * 2^-53) of zero, so calc_pA takes the log-space tail
    (src/pval.rs:219-226) for such tiny expected abundances."""
    assert O.gamma_lr(3.0, 1e-15) == 0.0
    assert O.gamma_lr(1.0, 1.2e-15) > 0.0
    for reads in (1, 2, 4):
        p = O.calc_pA(reads, 5e-16, True)
        ln_want = reads * math.log(5e-16) - 5e-16 - math.lgamma(reads + 1)
        assert math.log(p) == pytest.approx(ln_want, rel=1e-12)


def test_calc_pA_tiny_lambda_fallback():
    sp = pytest.importorskip("scipy.special")
    for reads in (2, 5, 40):
        for lam in (1e-30, 1e-12, 1e-8):
            got = O.calc_pA(reads, lam, True)
            ln_want = reads * math.log(lam) - lam - math.lgamma(reads + 1)
            if ln_want < -700.0:
                assert got == 0.0  # below the smallest normal double
                continue
            assert got > 0.0
            assert math.log(got) == pytest.approx(ln_want, rel=1e-9)
    assert O.calc_pA(3, 0.0, True) == 1.0
    # conditioning normaliser switches to E - E^2/2 below 1e-7 (src/pval.rs:233-239)
    e = 1e-9
    assert O.calc_pA(1, e, False) == pytest.approx(O.calc_pA(1, e, True) / (e - 0.5 * e * e), rel=1e-15)
    _ = sp


def test_get_pA_sentinels():
    assert O.get_pA(1, False, 0.5, 3, 100) == 1.0
    assert O.get_pA(5, False, 0.5, 0, 100) == 1.0
    assert O.get_pA(5, False, 0.0, 3, 100) == 0.0
    assert O.get_pA(5, False, 1e-3, 3, 100) == O.calc_pA(5, 0.1, False)
