"""Pin the oracle's aligners to the reference's own nwalign.rs unit tests.

Inputs, seeds and expected values come from tests/golden/reference_vectors.json,
extracted from the reference test source (src/nwalign.rs:1810-3189).
"""
import numpy as np
import pytest

from oracle import oracle as O

MASK64 = (1 << 64) - 1


def xorshift(state):
    """src/nwalign.rs:2862-2869"""
    x = state
    x ^= (x << 13) & MASK64
    x ^= x >> 7
    x ^= (x << 17) & MASK64
    return x & MASK64


def lcg_seq(n, seed, mul, add):
    s, out = seed, []
    for _ in range(n):
        s = (s * mul + add) & MASK64
        out.append(((s >> 33) % 4) + 1)
    return np.array(out, np.uint8)


def test_endsfree_known_answers(refvec):
    for kat in refvec["endsfree_kats"]:
        a0, a1 = O.align(O.ALIGN_ENDSFREE, O.encode(kat["s1"]), O.encode(kat["s2"]), band=kat["band"])
        assert O.score_alignment(a0, a1) == kat["expected"], kat


def test_vectorized_matches_endsfree_score(refvec):
    pairs = [(O.encode(p["s1"]), O.encode(p["s2"])) for p in refvec["vec_parity_pairs"]]
    mul, add = refvec["lcg_mul"], refvec["lcg_add"]
    seeds = {d["test"]: d["seed"] for d in refvec["vec_parity_lcg_seeds"]}
    s1 = lcg_seq(240, seeds["test_vectorized_vs_endsfree_equal_length_240"], mul, add)
    s2 = s1.copy()
    s2[239] ^= 3
    pairs += [(s1, s1.copy()), (s1, s2)]
    s1 = lcg_seq(240, seeds["test_vectorized_vs_endsfree_divergent_240"], mul, add)
    s2 = s1.copy()
    nts = [1, 2, 3, 4]
    for i in range(0, 240, 50):
        s2[i] = nts[(int(s2[i]) % 4) ^ 1]
    pairs.append((s1, s2))
    # 230 then 240 drawn from one continuing stream (src/nwalign.rs:3051-3061)
    st = seeds["test_vectorized_vs_endsfree_different_lengths"]
    both = lcg_seq(470, st, mul, add)
    pairs.append((both[:230], both[230:]))
    for a, b in pairs:
        ef = O.align(O.ALIGN_ENDSFREE, a, b, band=16)
        ve = O.align(O.ALIGN_VECTORIZED, a, b, band=16)
        assert O.score_alignment(*ef) == O.score_alignment(*ve)


def test_rolling_matches_full_matrix_fuzz(refvec):
    fz = refvec["rolling_fuzz"]
    state = fz["seed"]
    checked = 0
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
                a = np.array(s1, np.uint8)
                b = np.array(s2, np.uint8)
                for egp in fz["end_gap_ps"]:
                    r = O.align(O.ALIGN_VECTORIZED, a, b, end_gap=egp, band=band)
                    f = O.align(O.ALIGN_VECTORIZED_FULL, a, b, end_gap=egp, band=band)
                    assert np.array_equal(r[0], f[0]) and np.array_equal(r[1], f[1]), (l1, l2, band, trial, egp)
                    checked += 1
    assert checked > fz["min_checked"]


def test_rolling_survives_buffer_reuse(refvec):
    br = refvec["buffer_reuse"]
    state = br["seed"]
    pairs = []
    for n in br["lens"]:
        s1 = []
        for _ in range(n):
            state = xorshift(state)
            s1.append(1 + state % 4)
        s2 = list(s1)
        for k in range(0, n, br["step"]):
            s2[k] = 1 + (s2[k] % 4)
        pairs.append((np.array(s1, np.uint8), np.array(s2, np.uint8)))
    reused = O.align_vectorized_reuse(pairs)
    for (a, b), (r0, r1) in zip(pairs, reused):
        f0, f1 = O.align(O.ALIGN_VECTORIZED, a, b)
        assert np.array_equal(r0, f0) and np.array_equal(r1, f1)


def test_homopolymer_gap_routes_to_homopolymer_aligner(refvec):
    hd = refvec["homo_dispatch"]
    s1, s2 = O.encode(hd["s1"]), O.encode(hd["s2"])
    want = O.align(O.ALIGN_HOMO, s1, s2, homo_gap=hd["homo_gap_p"], band=16)
    vec = O.align(O.ALIGN_VECTORIZED, s1, s2, band=16)
    assert not (np.array_equal(vec[0], want[0]) and np.array_equal(vec[1], want[1]))
    p = O.AlignParams(homo_gap_p=hd["homo_gap_p"])
    method, a0, a1, _, _ = O.raw_align(s1, s2, p)
    assert method == "homo"
    assert np.array_equal(a0, want[0]) and np.array_equal(a1, want[1])


def test_vectorized_parity_sweep():
    """Reduced form of the ignored sweep_vectorized_parity (src/nwalign.rs:3069-3118)."""
    st = 0x9E3779B97F4A7C15
    nts = [1, 2, 3, 4]

    def rng(m):
        nonlocal st
        st = (st * 6364136223846793005 + 1) & MASK64
        return (st >> 33) % m

    fails = 0
    for _ in range(600):
        n = 5 + rng(60)
        s1 = [nts[rng(4)] for _ in range(n)]
        s2 = list(s1)
        for _ in range(rng(5)):
            if not s2:
                break
            p = rng(len(s2))
            op = rng(3)
            if op == 0:
                s2[p] = nts[rng(4)]
            elif op == 1:
                s2.insert(p, nts[rng(4)])
            else:
                s2.pop(p)
        if len(s2) < 3:
            continue
        a, b = np.array(s1, np.uint8), np.array(s2, np.uint8)
        for band in (8, 16, 32):
            ef = O.align(O.ALIGN_ENDSFREE, a, b, band=band)
            ve = O.align(O.ALIGN_VECTORIZED, a, b, band=band)
            if O.score_alignment(*ef) != O.score_alignment(*ve):
                fails += 1
    assert fails == 0


def test_al2subs_and_gapless():
    s1 = O.encode("ACGTACGTAC")
    s2 = O.encode("ACGTTCGTACGG")
    a0, a1 = O.align(O.ALIGN_GAPLESS, s1, s2)
    assert len(a0) == 12 and a0[10] == ord("-") and a0[11] == ord("-")
    sub = O.al2subs(a0, a1)
    assert sub["len0"] == 10
    assert list(sub["pos"]) == [4]
    assert list(sub["map"]) == list(range(10))
    # a gap in the reference row leaves map entries untouched; a gap in the query maps to 9999
    a0 = np.array([1, 2, ord("-"), 3], np.uint8)
    a1 = np.array([1, ord("-"), 4, 3], np.uint8)
    sub = O.al2subs(a0, a1)
    assert list(sub["map"]) == [0, 9999, 2]


@pytest.mark.parametrize("k", [3, 5, 7])
def test_raw_align_screen_cutoff_strict(k):
    s = O.encode("ACGTTGCAAGCTTAGCGATCGATCGGCTAGCTAGCATCGACTGACTAGC")
    p = O.AlignParams(kmer_size=k, kdist_cutoff=0.0)
    m, *_ = O.raw_align(s, s.copy(), p)
    assert m == "gapless"  # kdist == 0.0 is not > 0.0
