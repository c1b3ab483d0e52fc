"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Integer outputs (alignments, hamming, membership, counters) must be identical;
FP64 outputs (lambda, p-values, birth statistics) must be bit-identical -- the
kernels restate the reference's ordered, separately-rounded arithmetic.
"""
import numpy as np
import pytest

import dada2_b200 as D
from dada2_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MASK64 = (1 << 64) - 1


def xorshift(x):
    x ^= (x << 13) & MASK64
    x ^= x >> 7
    x ^= (x << 17) & MASK64
    return x & MASK64


def fuzz_pairs(fz):
    """The reference's rolling-vs-full fuzz inputs (src/nwalign.rs:2873-2952)."""
    state = fz["seed"]
    out = []
    for l1, l2 in fz["length_pairs"]:
        for band in fz["bands"]:
            for trial in range(fz["trials"]):
                s1 = []
                for _ in range(l1):
                    state = xorshift(state)
                    s1.append(1 + state % 4)
                if trial == 0 and l1 == l2:
                    s2 = list(s1)
                else:
                    v = list(s1[:min(l2, l1)]) if l2 <= l1 else list(s1)
                    v = (v + [1] * l2)[:l2]
                    for t in range(len(v)):
                        state = xorshift(state)
                        if state % 16 < trial:
                            state = xorshift(state)
                            v[t] = 1 + state % 4
                    s2 = v
                out.append((band, np.array(s1, np.uint8), np.array(s2, np.uint8)))
    return out


def test_vectorized_aligner_matches_oracle_on_reference_fuzz(refvec):
    pairs = fuzz_pairs(refvec["rolling_fuzz"])
    for egp in refvec["rolling_fuzz"]["end_gap_ps"]:
        by_band = {}
        for band, a, b in pairs:
            by_band.setdefault(band, []).append((a, b))
        n = 0
        for band, ps in by_band.items():
            got = D.align_pairs(D.ALIGN_VECTORIZED, ps, D.AlignParams(band=band), end_gap=egp)
            for (a, b), (g0, g1) in zip(ps, got):
                w0, w1 = O.align(O.ALIGN_VECTORIZED, a, b, end_gap=egp, band=band)
                assert np.array_equal(g0, w0) and np.array_equal(g1, w1), (len(a), len(b), band, egp)
                n += 1
        assert n == len(pairs)


def random_pairs(seed, n, lmin, lmax, indel=True):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        L = int(rng.integers(lmin, lmax + 1))
        a = rng.integers(1, 5, size=L).astype(np.uint8)
        b = list(a)
        for _ in range(int(rng.integers(0, 6))):
            p = int(rng.integers(0, len(b)))
            op = int(rng.integers(0, 3 if indel else 1))
            if op == 0:
                b[p] = int(rng.integers(1, 5))
            elif op == 1:
                b.insert(p, b[p])  # homopolymer-style insertion
            elif len(b) > 8:
                b.pop(p)
        out.append((a, np.array(b, np.uint8)))
    return out


@pytest.mark.parametrize("match,mismatch,gap,egp", [
    (5, -4, -8, 0),      # default scores: the add-max register form
    (5, -4, -8, -8),     # end gaps as costly as inner gaps (no ends-free recalc)
    (200, -4, -8, 0),    # match * (L + 1) past 32767: the exact saturating form
    (5, -4, -8, 3),      # positive end gap: the exact saturating form
    (40, -30, -60, -9),  # large penalties, lower saturation reached in band corners
])
@pytest.mark.parametrize("band", [-1, 8, 16, 40, 100])
def test_vectorized_register_forms_match_oracle(band, match, mismatch, gap, egp):
    pairs = random_pairs(7 + band + match, 60, 20, 330)
    p = D.AlignParams(band=band, match_score=match, mismatch=mismatch, gap_p=gap, homo_gap_p=gap)
    got = D.align_pairs(D.ALIGN_VECTORIZED, pairs, p, end_gap=egp)
    for (a, b), (g0, g1) in zip(pairs, got):
        w0, w1 = O.align(O.ALIGN_VECTORIZED, a, b, match=match, mismatch=mismatch, gap=gap, homo_gap=gap,
                         end_gap=egp, band=band)
        assert np.array_equal(g0, w0) and np.array_equal(g1, w1), (len(a), len(b), band, match, egp)
    # the swapped orientation (first sequence longer) takes the other tie rule
    got_sw = D.align_pairs(D.ALIGN_VECTORIZED, [(b, a) for a, b in pairs], p, end_gap=egp)
    for (a, b), (g0, g1) in zip(pairs, got_sw):
        w0, w1 = O.align(O.ALIGN_VECTORIZED, b, a, match=match, mismatch=mismatch, gap=gap, homo_gap=gap,
                         end_gap=egp, band=band)
        assert np.array_equal(g0, w0) and np.array_equal(g1, w1), ("swapped", len(a), len(b), band, match, egp)


@pytest.mark.parametrize("band", [-1, 0, 3, 16, 32])
def test_rowmajor_aligners_match_oracle(band):
    pairs = random_pairs(100 + band, 120, 20, 180)
    for which, owhich, hg in ((D.ALIGN_HOMO, O.ALIGN_HOMO, -1), (D.ALIGN_ENDSFREE, O.ALIGN_ENDSFREE, -8)):
        p = D.AlignParams(band=band, homo_gap_p=hg)
        got = D.align_pairs(which, pairs, p)
        for (a, b), (g0, g1) in zip(pairs, got):
            w0, w1 = O.align(owhich, a, b, homo_gap=hg, band=band)
            assert np.array_equal(g0, w0) and np.array_equal(g1, w1), (which, band, len(a), len(b))


def test_homopolymer_dispatch_pair_on_gpu(refvec):
    hd = refvec["homo_dispatch"]
    s1, s2 = O.encode(hd["s1"]), O.encode(hd["s2"])
    (g0, g1), = D.align_pairs(D.ALIGN_HOMO, [(s1, s2)], D.AlignParams(homo_gap_p=hd["homo_gap_p"]))
    w0, w1 = O.align(O.ALIGN_HOMO, s1, s2, homo_gap=hd["homo_gap_p"], band=16)
    assert np.array_equal(g0, w0) and np.array_equal(g1, w1)


def pool(refvec):
    pl = refvec["compare_pool"]
    nxt = {"A": "C", "C": "G", "G": "T"}
    seqs, reads = [], []
    for n, r in pl["n_reads"]:
        s = list(pl["base"])
        for p in range(n):
            idx = (p * pl["mut_mul"] + pl["mut_add"]) % len(s)
            s[idx] = nxt.get(s[idx], "A")
        seqs.append(O.encode("".join(s)))
        reads.append(r)
    return pl, seqs, reads


def test_compare_pool_matches_oracle(refvec):
    pl, seqs, reads = pool(refvec)
    err = np.full(16 * pl["ncol"], pl["err_flat"])
    for greedy in (False, True):
        op = O.AlignParams(homo_gap_p=pl["homo_gap_p"], kdist_cutoff=pl["kdist_cutoff"], kmer_size=pl["k"],
                           band=pl["band"])
        sess = O.Session(seqs, reads, k=pl["k"], use_quals=False)
        sess.set_center(0, pl["center"])
        wl, wh, ws, _ = sess.compare_map(0, err, pl["ncol"], op, greedy=greedy)
        want = sess.compare(0, err, pl["ncol"], op, greedy=greedy)
        gp = D.AlignParams(homo_gap_p=pl["homo_gap_p"], kdist_cutoff=pl["kdist_cutoff"], kmer_size=pl["k"],
                           band=pl["band"])
        with D.CompareContext(gp, err, pl["ncol"], use_quals=False) as ctx:
            ctx.upload(seqs, reads)
            gl, gh, gs, gc = ctx.compare(pl["center"], pl["kdist_cutoff"], greedy=greedy)
            assert gl.tobytes() == wl.tobytes()
            assert np.array_equal(gh, wh) and np.array_equal(gs, ws)
            got = ctx.b_compare_parallel(pl["center"], 0, pl["kdist_cutoff"], greedy=greedy)
            assert np.array_equal(got["index"], want["index"])
            assert got["lambda"].tobytes() == want["lambda"].tobytes()
            assert np.array_equal(got["hamming"], want["hamming"])
            assert got["self"] == want["self"]
            c, w = got["counters"], want["counters"]
            assert (c["screened"], c["aligned"], c["shrouded"], c["stored"]) == (
                w["screened"], w["aligned"], w["nshroud"], w["stored"])
            assert np.array_equal(ctx.e_minmax(), want["e_minmax"])


def _rounded_quals(sample):
    return [np.floor(np.asarray(q, np.float64) / a + 0.5).astype(np.uint8) for q, a in zip(sample.quals, sample.abund)]


def _extend(err, ncol, quals):
    """Repeat the last column up to the largest quality (src/dada.rs:337-384)."""
    qmax = max(int(q.max()) for q in quals)
    if qmax < ncol:
        return err, ncol
    m = np.asarray(err).reshape(16, ncol)
    ext = np.concatenate([m, np.repeat(m[:, -1:], qmax + 1 - ncol, axis=1)], axis=1)
    return ext.reshape(-1).copy(), qmax + 1


@pytest.mark.parametrize("seed", [11, 12])
@pytest.mark.parametrize("k", [5, 8])  # k = 8: the sparse screen (src/kmers.rs:280-308)
def test_compare_many_centers_matches_oracle(seed, k):
    w = synth.small_illumina(seed, nvariants=6, nreads=1500, L=120)
    s = w.samples[0]
    seqs = [O.encode(x) for x in s.seqs]
    quals = _rounded_quals(s)
    err, ncol = _extend(w.err, w.ncol, quals)
    sess = O.Session(seqs, s.abund, quals=quals, k=k, use_quals=True)
    with D.CompareContext(D.AlignParams(kmer_size=k), err, ncol) as ctx:
        ctx.upload(seqs, s.abund, quals=quals)
        for center in (0, 1, 2, 5, len(seqs) // 2, len(seqs) - 1):
            ci = sess.add_center(center)
            for cutoff in (0.42, 1.0):
                pa = O.AlignParams(kdist_cutoff=cutoff, kmer_size=k)
                wl, wh, ws, wm = sess.compare_map(ci, err, ncol, pa, greedy=True)
                gl, gh, gs, _ = ctx.compare(center, cutoff, greedy=True)
                assert gl.tobytes() == wl.tobytes(), (center, cutoff)
                assert np.array_equal(gh, wh) and np.array_equal(gs, ws)


def assert_same_dada(got, want):
    assert got["nclust"] == want["nclust"]
    assert np.array_equal(got["map"], want["map"])
    assert got["pvals"].tobytes() == want["pvals"].tobytes()
    for k in ("nalign", "nshroud", "compare_calls", "cmp_scanned", "screened", "aligned", "stored",
              "gapless", "vectorized", "homo", "endsfree", "shuffle_calls", "shuffle_moves"):
        assert got["counters"][k] == want["counters"][k], k
    for g, w in zip(got["clusters"], want["clusters"]):
        assert np.array_equal(g["sequence"], w["sequence"])
        assert g["reads"] == w["reads"]
        assert np.array_equal(g["members"], w["members"])
        assert np.array_equal(g["hammings"], w["hammings"])
        assert g["lambdas"].tobytes() == w["lambdas"].tobytes()
        assert g["pvals"].tobytes() == w["pvals"].tobytes()
        for k in ("birth_type", "birth_from", "birth_hamming"):
            assert g[k] == w[k]
        for k in ("birth_pval", "birth_fold", "birth_e"):
            assert np.float64(g[k]).tobytes() == np.float64(w[k]).tobytes(), k


@pytest.mark.parametrize("seed", [21, 22, 23])
def test_dada_small_matches_oracle(seed):
    w = synth.small_illumina(seed)
    s = w.samples[0]
    want = O.dada(s.seqs, s.abund, w.err, w.ncol, O.DadaParams(nthreads=4), quals=s.quals)
    got = D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, D.DadaParams(), quals=s.quals)
    assert want["nclust"] > 3
    assert_same_dada(got, want)


def test_dada_config0_matches_oracle():
    w = synth.config0()
    s = w.samples[0]
    want = O.dada(s.seqs, s.abund, w.err, w.ncol, O.DadaParams(nthreads=8), quals=s.quals)
    got = D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, D.DadaParams(), quals=s.quals)
    assert_same_dada(got, want)
    # the map's decision margin is the closest final p-value to omega_c
    # among the non-centers (a center is not tested against omega_c)
    index = {q: i for i, q in enumerate(s.seqs)}
    noncenter = np.ones(len(s.seqs), bool)
    for c in got["clusters"]:
        noncenter[index["".join("ACGT"[x - 1] for x in np.asarray(c["sequence"]))]] = False
    omega_c = D.DadaParams().omega_c
    pv = got["pvals"]
    with np.errstate(divide="ignore"):
        rel = np.abs(pv[noncenter] - omega_c) / np.minimum(pv[noncenter], omega_c)
    assert got["margins"]["omega_c"] == float(np.min(rel))
    assert got["margins"]["omega_a"] > 1e-6


def test_dada_config2_full_size_matches_oracle():
    """PacBio 16S at the full configured size: 5,000 uniques of 1,400-1,550 nt
    from 60 variants, indel-heavy errors, band 32 and homopolymer gap -1 (the
    row-major i32 homopolymer aligner, src/nwalign.rs:435-528), qualities up
    to Q93 (the error matrix extends by its last column)."""
    w = synth.config2(seed=1002)
    s = w.samples[0]
    assert len(s.seqs) == 5000
    import os

    op = O.DadaParams(align=O.AlignParams(band=32, homo_gap_p=-1), nthreads=max(2, os.cpu_count() or 2))
    dp = D.DadaParams(align=D.AlignParams(band=32, homo_gap_p=-1))
    want = O.dada(s.seqs, s.abund, w.err, w.ncol, op, quals=s.quals)
    got = D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, dp, quals=s.quals)
    assert want["counters"]["homo"] > 10000
    assert_same_dada(got, want)


@pytest.fixture(scope="module")
def config3_prefix():
    import os

    w = synth.config3(seed=1003)
    s = w.samples[0]
    n = 30000
    sub = synth.Sample(s.seqs[:n], np.asarray(s.abund[:n]), s.quals[:n], 0, name="config3[:30000]")
    op = O.DadaParams(align=O.AlignParams(band=w.band, homo_gap_p=w.homo_gap_p, kmer_size=w.kmer_size),
                      nthreads=max(2, os.cpu_count() or 2))
    want = O.dada(sub.seqs, sub.abund, w.err, w.ncol, op, quals=sub.quals)
    return w, sub, want


def test_dada_config3_pooled_prefix_matches_oracle(config3_prefix):
    """The pooled workload (200 samples pooled in first-seen order, 3,000
    variants x 150 nt): its first 30,000 pooled uniques as one sample --
    about 2,700 clusters -- equal the oracle's run_dada bit for bit, with
    FP64 lambda and with decisions from the FP32 log-sum lambda."""
    w, s, want = config3_prefix
    dp = D.DadaParams(align=D.AlignParams(band=w.band, homo_gap_p=w.homo_gap_p, kmer_size=w.kmer_size))
    got = D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, dp, quals=s.quals)
    assert want["nclust"] > 1000
    assert_same_dada(got, want)
    dp32 = D.DadaParams(align=dp.align, lambda_fp32=True)
    got32 = D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, dp32, quals=s.quals)
    assert got32["nclust"] == want["nclust"]
    assert np.array_equal(got32["map"], want["map"])


def test_pivot_bound_excludes_profiles_and_keeps_results(config3_prefix):
    """The screen's pivot bound (a far unique is shrouded from its best dot
    with an earlier center, without reading its profile) forced on for every
    compare launch: the run still equals the oracle's bit for bit, counters
    included, and it read fewer profile bytes than the run without it."""
    w, s, want = config3_prefix
    dp = D.DadaParams(align=D.AlignParams(band=w.band, homo_gap_p=w.homo_gap_p, kmer_size=w.kmer_size))
    keep = D.tuning_get(150)
    try:
        D.tuning_set(0, {**keep, "pivot_min_items": 0})
        D.stats_reset()
        off = D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, dp, quals=s.quals)
        bytes_off = D.stats_read()["screen_bytes"]
        D.tuning_set(0, {**keep, "pivot_min_items": 1})
        D.stats_reset()
        on = D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, dp, quals=s.quals)
        bytes_on = D.stats_read()["screen_bytes"]
    finally:
        D.tuning_set(0, keep)
    assert_same_dada(off, want)
    assert_same_dada(on, want)
    assert bytes_on < 0.5 * bytes_off, (bytes_on, bytes_off)


def test_dada_batch_matches_per_sample_oracle():
    ws = [synth.small_illumina(30 + i, nvariants=4 + i, nreads=800 + 300 * i, L=100 + 20 * (i % 3)) for i in range(5)]
    err, ncol = ws[0].err, ws[0].ncol
    samples = [w.samples[0] for w in ws]
    got = D.dada_uniques_batch(samples, err, ncol, D.DadaParams(host_threads=3))
    for s, g in zip(samples, got):
        want = O.dada(s.seqs, s.abund, err, ncol, O.DadaParams(nthreads=4), quals=s.quals)
        assert_same_dada(g, want)


def test_dada_homopolymer_long_reads_matches_oracle():
    w = synth.config2(seed=77, nuniques=120)
    s = w.samples[0]
    op = O.DadaParams(align=O.AlignParams(band=32, homo_gap_p=-1), nthreads=8)
    dp = D.DadaParams(align=D.AlignParams(band=32, homo_gap_p=-1))
    want = O.dada(s.seqs, s.abund, w.err, w.ncol, op, quals=s.quals)
    got = D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, dp, quals=s.quals)
    assert want["counters"]["homo"] > 0
    assert_same_dada(got, want)


@pytest.mark.parametrize("variant", ["band0", "no_kmers", "no_quals", "no_greedy", "unbanded", "kmer3", "kmer8"])
def test_dada_parameter_variants_match_oracle(variant):
    w = synth.small_illumina(41, nvariants=5, nreads=1200, L=90)
    s = w.samples[0]
    oa, da = O.AlignParams(), D.AlignParams()
    okw, dkw = {}, {}
    quals = s.quals
    if variant == "band0":
        oa.band = da.band = 0
    elif variant == "no_kmers":
        oa.use_kmers = da.use_kmers = False
    elif variant == "no_quals":
        quals = None
    elif variant == "no_greedy":
        okw["greedy"] = dkw["greedy"] = False
    elif variant == "unbanded":
        oa.band = da.band = -1
    elif variant == "kmer3":
        oa.kmer_size = da.kmer_size = 3
    elif variant == "kmer8":  # sparse screen (src/kmers.rs:213-221, 280-308)
        oa.kmer_size = da.kmer_size = 8
    want = O.dada(s.seqs, s.abund, w.err, w.ncol, O.DadaParams(align=oa, nthreads=4, **okw), quals=quals)
    got = D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, D.DadaParams(align=da, **dkw), quals=quals)
    assert_same_dada(got, want)


def test_invalid_inputs_are_rejected_like_the_reference():
    err = np.full(16 * 41, 0.01)
    with pytest.raises(D.InvalidInput, match="non-ACGT"):
        D.dada_uniques(["ACGTNACGTA", "ACGTACGTAA"], [3, 2], err, 41)
    with pytest.raises(D.InvalidInput, match="longer than the k-mer"):
        D.dada_uniques(["ACGT", "ACGTACGTAA"], [3, 2], err, 41)
    with pytest.raises(D.InvalidInput):
        D.dada_uniques([], [], err, 41)


class _S:
    def __init__(self, seqs, abund):
        self.seqs, self.abund = seqs, np.array(abund, np.uint32)
        self.quals = [np.full(len(x), 30 * a, np.uint32) for x, a in zip(seqs, abund)]


def test_batch_reports_the_first_failing_sample_in_input_order():
    """Samples are validated in order (src/dada.rs:248-317): the first sample
    with a structural error or a non-ACGT base reports, and within a sample
    the length checks come before the base scan."""
    err = np.full(16 * 41, 0.01)
    good = _S(["ACGTACGTAA", "ACGTACGTAC"], [3, 2])
    bad_base = _S(["ACGTACGTAA", "ACGTACNTAC", "ACGTXCGTAC"], [3, 2, 1])
    too_short = _S(["ACGTACGTAA", "ACG"], [3, 2])
    with pytest.raises(D.InvalidInput, match=r"sample 1: Sequence 1 contains a non-ACGT base at position 6"):
        D.dada_uniques_batch([good, bad_base, too_short], err, 41)
    with pytest.raises(D.InvalidInput, match=r"sample 1: All input sequences must be longer"):
        D.dada_uniques_batch([good, too_short, bad_base], err, 41)
    both = _S(["ACGTNCGTAA", "ACG"], [3, 2])  # structural failure wins inside one sample
    with pytest.raises(D.InvalidInput, match=r"sample 0: All input sequences must be longer"):
        D.dada_uniques_batch([both, good], err, 41)


def test_resident_batch_runs_repeat_identically():
    ws = [synth.small_illumina(60 + i, nvariants=5, nreads=900 + 400 * i, L=110) for i in range(3)]
    err, ncol = ws[0].err, ws[0].ncol
    samples = [w.samples[0] for w in ws]
    with D.ResidentBatch(samples, err, ncol, D.DadaParams(host_threads=4)) as rb:
        first = rb.run()
        second = rb.run()
    for s, a, b in zip(samples, first, second):
        assert_same_dada(a, b)
        want = O.dada(s.seqs, s.abund, err, ncol, O.DadaParams(nthreads=4), quals=s.quals)
        assert_same_dada(a, want)


def test_kernel_stats_count_launches():
    w = synth.small_illumina(71, nvariants=4, nreads=800, L=100)
    s = w.samples[0]
    D.stats_reset()
    D.stats_timing(True)
    r = D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, D.DadaParams(), quals=s.quals)
    D.stats_timing(False)
    st = D.stats_read()
    assert st["rounds"] == r["counters"]["compare_calls"]
    assert st["launches"]["screen"] == st["rounds"] and st["launches"]["profiles"] == 1
    assert st["compares"] == r["counters"]["cmp_scanned"]
    assert st["ms"]["screen"] > 0.0
    assert len(D.stats_latencies()) == st["rounds"]


@pytest.mark.parametrize("k", [5, 8])
def test_saturated_kmers_take_the_exact_distance(k):
    """Profiles with a k-mer counted >= 255 in both sequences (src/nwalign.rs:1270-1277)."""
    rng = np.random.default_rng(5)
    seqs, reads = [], []
    for t in range(12):
        run = 262 + int(rng.integers(0, 40))  # the all-A 5-mer occurs run-4 >= 258 times
        tail = rng.integers(1, 5, size=40 + int(rng.integers(0, 30))).astype(np.uint8)
        s = np.concatenate([np.full(run, 1, np.uint8), tail])
        if t % 3 == 1:
            s[run + 5] = 1 + (s[run + 5] % 4)
        seqs.append(s)
        reads.append(50 - 3 * t)
    err = np.full(16 * 41, 0.01)
    op = O.AlignParams(kdist_cutoff=0.42, kmer_size=k)
    sess = O.Session(seqs, reads, k=k, use_quals=False)
    with D.CompareContext(D.AlignParams(kmer_size=k), err, 41, use_quals=False) as ctx:
        ctx.upload(seqs, reads)
        for center in (0, 3, 7):
            ci = sess.add_center(center)
            wl, wh, ws, _ = sess.compare_map(ci, err, 41, op, greedy=False)
            gl, gh, gs, _ = ctx.compare(center, 0.42, greedy=False)
            assert gl.tobytes() == wl.tobytes()
            assert np.array_equal(gh, wh) and np.array_equal(gs, ws)


def _assert_same_transitions(got, want):
    assert "transitions" in got and "transitions" in want
    assert got["transitions"].shape == want["transitions"].shape
    assert np.array_equal(got["transitions"], want["transitions"])


@pytest.mark.parametrize("variant", ["default", "band0", "no_quals", "unbanded"])
def test_transition_counts_match_oracle(variant):
    """DadaAux.transitions: every correct raw realigned to its center with the
    k-mer screen off (src/dada.rs:609-673), counted by transition and quality
    (src/error.rs:194-249)."""
    w = synth.small_illumina(52, nvariants=6, nreads=1500, L=120)
    s = w.samples[0]
    oa, da = O.AlignParams(), D.AlignParams()
    quals = s.quals
    if variant == "band0":
        oa.band = da.band = 0
    elif variant == "no_quals":
        quals = None
    elif variant == "unbanded":
        oa.band = da.band = -1
    want = O.dada(s.seqs, s.abund, w.err, w.ncol, O.DadaParams(align=oa, nthreads=4, transitions=True), quals=quals)
    got = D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, D.DadaParams(align=da, transitions=True), quals=quals)
    assert_same_dada(got, want)
    _assert_same_transitions(got, want)
    if quals is None:
        assert got["transitions"].shape == (16, 1)
    assert int(got["transitions"].sum()) > 0


def test_transition_counts_homopolymer_path_match_oracle():
    w = synth.config2(seed=78, nuniques=80)
    s = w.samples[0]
    op = O.DadaParams(align=O.AlignParams(band=32, homo_gap_p=-1), nthreads=8, transitions=True)
    dp = D.DadaParams(align=D.AlignParams(band=32, homo_gap_p=-1), transitions=True)
    want = O.dada(s.seqs, s.abund, w.err, w.ncol, op, quals=s.quals)
    got = D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, dp, quals=s.quals)
    _assert_same_transitions(got, want)


def test_transition_counts_in_a_batch_use_each_samples_width():
    """In a batch the error matrix is extended to the largest quality of any
    sample, but each sample's counts keep the width its own run would have."""
    ws = [synth.small_illumina(60 + i, nvariants=4, nreads=900, L=110) for i in range(3)]
    err, ncol = ws[0].err, ws[0].ncol
    samples = [w.samples[0] for w in ws]
    # lift one sample's qualities past the error matrix so the widths differ
    boosted = samples[1]
    boosted.quals = [np.asarray(q, np.uint32) + np.uint32(8) * np.uint32(a) for q, a in zip(boosted.quals, boosted.abund)]
    got = D.dada_uniques_batch(samples, err, ncol, D.DadaParams(host_threads=2, transitions=True))
    widths = set()
    for s, g in zip(samples, got):
        want = O.dada(s.seqs, s.abund, err, ncol, O.DadaParams(nthreads=4, transitions=True), quals=s.quals)
        assert_same_dada(g, want)
        _assert_same_transitions(g, want)
        widths.add(g["transitions"].shape[1])
    assert len(widths) > 1


@pytest.mark.parametrize("L", [150, 250])
def test_fp32_log_lambda_tracks_fp64(L):
    """Precision variant: ln(lambda) as a compensated FP32 sum beside the FP64
    product. Tolerances: |ln32 - ln64| <= 1e-5 * max(1, |ln64|); lambda's
    relative error <= 1e-4 where FP64 lambda is normal; outside 1e3x of
    omega_a the p-value decision p < omega_a agrees with FP64's."""
    w = synth.small_illumina(70 + L, nvariants=8, nreads=2500, L=L)
    s = w.samples[0]
    seqs = [O.encode(x) for x in s.seqs]
    quals = _rounded_quals(s)
    err, ncol = _extend(w.err, w.ncol, quals)
    reads = np.asarray(s.abund, np.uint32)
    total = float(reads.sum())
    omega_a = 1e-40
    with D.CompareContext(D.AlignParams(), err, ncol) as ctx:
        ctx.upload(seqs, reads, quals=quals)
        ctx.set_lambda32(True)
        n_band = n_all = 0
        for center in (0, 3, len(seqs) // 2):
            lam, ham, skp, cnt = ctx.compare(center, 1.0, greedy=False)
            ll32 = ctx.loglambda32().astype(np.float64)
            aligned = np.isfinite(ll32)
            assert aligned.sum() == cnt["aligned"]
            # FP64 lambda is only exact to its relative precision while it is a
            # normal double; below that the product itself has underflowed
            normal = aligned & (lam > 1e-300)
            ll64 = np.log(lam[normal])
            assert np.all(np.abs(ll32[normal] - ll64) <= 1e-5 * np.maximum(1.0, np.abs(ll64)))
            rel = np.abs(np.exp(ll32[normal]) - lam[normal]) / lam[normal]
            assert rel.max() <= 1e-4
            assert np.all(ll32[aligned & ~normal] < np.log(1e-300) + 1e-3)
            for r in np.nonzero(aligned)[0]:
                p64 = D.calc_pA(int(reads[r]), float(lam[r]) * total)
                p32 = D.calc_pA(int(reads[r]), float(np.exp(ll32[r])) * total)
                n_all += 1
                if omega_a / 1e3 <= p32 <= omega_a * 1e3:
                    n_band += 1  # where the FP32 variant falls back to FP64
                else:
                    assert (p32 < omega_a) == (p64 < omega_a)
        assert n_all > 0


def _service_reqs():
    return [synth.small_illumina(80, nvariants=5, nreads=1500, L=150).samples[0],
            synth.small_illumina(81, nvariants=6, nreads=3000, L=150).samples[0],
            synth.small_illumina(84, nvariants=3, nreads=500, L=140).samples[0],
            synth.small_illumina(82, nvariants=4, nreads=900, L=250).samples[0],
            synth.small_illumina(83, nvariants=3, nreads=400, L=700).samples[0]]


@pytest.mark.parametrize("transitions", [False, True])
def test_service_results_match_single_sample_calls(transitions):
    """Requests of three length classes, submitted together, come back as the
    single-sample path's results on each sample and the oracle's: one batch per
    class, each request released as soon as its own sample finishes (or, with
    transition counts, after the batch's final-subs pass)."""
    reqs = _service_reqs()
    w = synth.small_illumina(80)
    err, ncol = w.err, w.ncol
    prm = D.DadaParams(host_threads=4, transitions=transitions)
    with D.DenoiseService(err, ncol, prm) as svc:
        svc.hold()
        tickets = [svc.submit(s.seqs, s.abund, quals=s.quals) for s in reqs]
        svc.hold(False)
        got = [svc.wait(t) for t in tickets]
        assert svc.stats() == {"batches": 3, "served": 5}
    for s, (g, lat) in zip(reqs, got):
        assert lat > 0.0
        want = D.dada_uniques(s.seqs, s.abund, err, ncol, prm, quals=s.quals)
        assert_same_dada(g, want)
        if transitions:
            assert np.array_equal(g["transitions"], want["transitions"])
        else:
            assert_same_dada(g, O.dada(s.seqs, s.abund, err, ncol, O.DadaParams(nthreads=4), quals=s.quals))


def test_service_isolates_an_invalid_request():
    """An invalid request in a batch gets its own error while its batch-mates
    are served with their single-sample results."""
    reqs = _service_reqs()[:2]
    w = synth.small_illumina(80)
    bad = _S(["ACGTACGTAA" * 15, "ACGTACNTAC" * 15], [3, 2])
    with D.DenoiseService(w.err, w.ncol, D.DadaParams()) as svc:
        svc.hold()
        t0 = svc.submit(reqs[0].seqs, reqs[0].abund, quals=reqs[0].quals)
        tbad = svc.submit(bad.seqs, bad.abund, quals=bad.quals)
        t1 = svc.submit(reqs[1].seqs, reqs[1].abund, quals=reqs[1].quals)
        svc.hold(False)
        got = [svc.wait(t0)[0], svc.wait(t1)[0]]
        with pytest.raises(D.InvalidInput, match="non-ACGT"):
            svc.wait(tbad)
        assert svc.stats() == {"batches": 1, "served": 3}
    for s, g in zip(reqs, got):
        assert_same_dada(g, D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, D.DadaParams(), quals=s.quals))


def test_service_budget_splits_batches():
    """A device-memory budget below two requests' footprint serves them one
    batch each, with results unchanged."""
    reqs = [synth.small_illumina(90 + i, nvariants=4, nreads=800, L=150).samples[0] for i in range(3)]
    w = synth.small_illumina(90, nvariants=4, nreads=800, L=150)
    with D.DenoiseService(w.err, w.ncol, D.DadaParams(), hbm_budget=1) as svc:
        svc.hold()
        ts = [svc.submit(s.seqs, s.abund, quals=s.quals) for s in reqs]
        svc.hold(False)
        got = [svc.wait(t)[0] for t in ts]
        assert svc.stats() == {"batches": 3, "served": 3}
    for s, g in zip(reqs, got):
        assert_same_dada(g, D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, D.DadaParams(), quals=s.quals))


@pytest.mark.parametrize("seed", [21, 22, 23, 1000])
def test_fp32_lambda_decisions_keep_the_partition(seed):
    """Decisions from the FP32 compensated log-sum lambda (FP64 within 1e3x of
    the thresholds) give the FP64 drop-in's partition: the same clusters, the
    same map, member lambdas within 1e-4 relative where the FP64 lambda is
    normal."""
    w = synth.config0() if seed == 1000 else synth.small_illumina(seed)
    s = w.samples[0]
    a = D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, D.DadaParams(), quals=s.quals)
    b = D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, D.DadaParams(lambda_fp32=True), quals=s.quals)
    assert a["fp32"] == {"pvalues": 0, "fallbacks": 0}
    assert b["fp32"]["pvalues"] > 0
    assert b["nclust"] == a["nclust"]
    assert np.array_equal(b["map"], a["map"])
    for ga, gb in zip(a["clusters"], b["clusters"]):
        assert np.array_equal(ga["sequence"], gb["sequence"])
        assert np.array_equal(np.sort(ga["members"]), np.sort(gb["members"]))
        la = ga["lambdas"][np.argsort(ga["members"])]
        lb = gb["lambdas"][np.argsort(gb["members"])]
        normal = la > 1e-300
        assert np.all(np.abs(lb[normal] - la[normal]) <= 1e-4 * la[normal])


def test_dada_from_fastq_matches_the_oracle(tmp_path):
    """FASTQ -> derep -> dada: the library's dereplication feeds the GPU loop
    and the result equals the oracle's on the oracle's own dereplication."""
    import gzip

    w = synth.small_illumina(31, nvariants=5, nreads=2000, L=150)
    rng = np.random.default_rng(31)
    recs = []
    for s, a, q in zip(w.samples[0].seqs, w.samples[0].abund, w.samples[0].quals):
        mean = np.rint(np.asarray(q, np.float64) / a).astype(np.int64)
        for _ in range(int(a)):
            qq = np.clip(mean + rng.integers(-2, 3, size=len(mean)), 2, 41)
            recs.append((s.encode(), (qq + 33).astype(np.uint8).tobytes()))
    order = rng.permutation(len(recs))
    recs = [recs[i] for i in order]
    path = tmp_path / "s.fastq.gz"
    with gzip.open(path, "wb") as f:
        f.write(b"".join(b"@r%d\n%s\n+\n%s\n" % (i, s, q) for i, (s, q) in enumerate(recs)))
    got = D.dada_fastq(path, w.err, w.ncol, D.DadaParams())
    seqs, counts, quals, mp = O.derep(recs)
    assert got["derep"].seqs == seqs and np.array_equal(got["derep"].map, mp)
    want = O.dada(seqs, counts.astype(np.uint32), w.err, w.ncol, O.DadaParams(nthreads=4), quals=quals)
    assert_same_dada(got, want)
    import json

    from dada2_b200 import output
    doc = json.loads(output.dada_json(got, D.DadaParams(), path))
    assert doc["sample"] == "s" and doc["num_asvs"] == want["nclust"]
    assert doc["total_reads"] == len(recs)
    assert doc["map"] == [None if m < 0 else int(m) for m in want["map"]]


def test_multi_device_service_matches_single_sample_calls():
    """The service sharded over the node's devices (here, those visible) gives
    each request the single-sample result."""
    from dada2_b200.multi import MultiDeviceService

    reqs = _service_reqs()[:3]
    w = synth.small_illumina(80)
    devs = list(range(D.device_count()))
    with MultiDeviceService(w.err, w.ncol, D.DadaParams(), devices=devs) as svc:
        ts = [svc.submit(s.seqs, s.abund, quals=s.quals) for s in reqs]
        got = [svc.wait(t)[0] for t in ts]
    for s, g in zip(reqs, got):
        assert_same_dada(g, D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, D.DadaParams(), quals=s.quals))


@pytest.mark.parametrize("kind,surface", [("loess", "direct"), ("loess", "interpolate"), ("noqual", "direct"),
                                          ("binned", "direct"), ("pacbio", "direct")])
def test_learn_errors_matches_the_oracle(kind, surface):
    """learn_errors (src/learn_errors.rs:739-1020) on three Illumina-style
    samples: the init pass, every self-consistency pass (all samples denoised
    together on the device, transitions counted there) and the fits give the
    oracle's nq, pass count, convergence, summed transitions and input/output
    error matrices bit for bit."""
    ws = [synth.small_illumina(60 + i, nvariants=6 + 2 * i, nreads=3000 + 500 * i, L=150) for i in range(3)]
    samples = [w.samples[0] for w in ws]
    bins = (0.0, 10.0, 20.0, 30.0, 40.0, 93.0) if kind == "binned" else ()
    ef = D.ErrFun(kind=kind, surface=surface, bins=bins)
    got = D.learn_errors(samples, D.DadaParams(), ef, max_consist=6)
    want = O.learn_errors(samples, O.DadaParams(nthreads=8), max_consist=6,
                          kind={"loess": 0, "noqual": 1, "binned": 2, "pacbio": 3}[kind],
                          surface=0 if surface == "direct" else 1, bins=list(bins) or None)
    assert (got["nq"], got["passes"], got["converged"]) == (want["nq"], want["passes"], want["converged"])
    assert got["passes"] >= 1
    assert np.array_equal(got["trans"], want["trans"])
    assert got["trans"].sum() > 0
    assert got["err_in"].tobytes() == want["err_in"].tobytes()
    assert got["err_out"].tobytes() == want["err_out"].tobytes()


@pytest.fixture(scope="module")
def config1_full():
    return synth.config1(seed=1001)


def test_config1_largest_samples_match_the_oracle(config1_full):
    """The 40-sample workload at full size: its two largest samples (16,124
    and 15,475 uniques, about 400 clusters each) denoised in one batch equal
    the oracle's run_dada on each."""
    w = config1_full
    big = sorted(w.samples, key=lambda s: -len(s.seqs))[:2]
    got = D.dada_uniques_batch(big, w.err, w.ncol, D.DadaParams())
    import os

    nt = max(2, (os.cpu_count() or 2))
    for s, g in zip(big, got):
        assert_same_dada(g, O.dada(s.seqs, s.abund, w.err, w.ncol, O.DadaParams(nthreads=nt), quals=s.quals))


def test_config1_batched_equals_single_sample_path(config1_full):
    """All 40 samples batched (six slots, one dedicated, up to four samples a
    launch) give each sample exactly what the single-sample path gives it."""
    w = config1_full
    pb = D.PackedBatch(w.samples)
    got = D.dada_uniques_batch(w.samples, w.err, w.ncol, D.DadaParams(), packed=pb)
    for s, g in zip(w.samples, got):
        assert_same_dada(g, D.dada_uniques(s.seqs, s.abund, w.err, w.ncol, D.DadaParams(), quals=s.quals))
