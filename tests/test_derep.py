"""FASTQ dereplication (src/derep.rs) through the library against the oracle's
restatement: ordering, counts, per-position Phred sums, the read map, gzip
input and malformed files. Host only: no GPU."""
import gzip

import numpy as np
import pytest

import dada2_b200 as D
from oracle import oracle as O


def _reads(seed, nvar=6, nreads=3000, L=120, sub=0.01):
    rng = np.random.default_rng(seed)
    var = rng.integers(0, 4, size=(nvar, L))
    w = np.arange(1, nvar + 1, dtype=float) ** -1.5
    vid = rng.choice(nvar, size=nreads, p=w / w.sum())
    seqs = var[vid].copy()
    hit = rng.random(seqs.shape) < sub
    seqs[hit] = rng.integers(0, 4, size=int(hit.sum()))
    quals = rng.integers(2, 42, size=seqs.shape)
    nt = np.frombuffer(b"ACGT", np.uint8)
    return [(nt[s].tobytes(), (q + 33).astype(np.uint8).tobytes()) for s, q in zip(seqs, quals)]


def _write(path, recs, gz=False, crlf=False):
    nl = b"\r\n" if crlf else b"\n"
    body = b"".join(b"@r%d" % i + nl + s + nl + b"+" + nl + q + nl for i, (s, q) in enumerate(recs))
    if gz:
        with gzip.open(path, "wb") as f:
            f.write(body)
    else:
        path.write_bytes(body)


def _same(got, want):
    seqs, counts, quals, mp = want
    assert got.seqs == seqs
    assert np.array_equal(got.abund, counts)
    assert len(got.quals) == len(quals)
    for a, b in zip(got.quals, quals):
        assert np.array_equal(a, b)
    assert np.array_equal(got.map, mp)


@pytest.mark.parametrize("gz,crlf,threads", [(False, False, 0), (True, False, 3), (False, True, 1)])
def test_derep_matches_the_restatement(tmp_path, gz, crlf, threads):
    recs = _reads(5)
    path = tmp_path / ("r.fastq.gz" if gz else "r.fastq")
    _write(path, recs, gz=gz, crlf=crlf)
    got = D.derep_fastq(path, nthreads=threads)
    _same(got, O.derep(recs))
    assert got.abund.sum() == len(recs)
    assert list(got.abund) == sorted(got.abund, reverse=True)


def test_derep_orders_ties_by_sequence_and_clamps_negative_sums(tmp_path):
    # equal counts order by sequence bytes; scores below the offset sum below
    # zero and are stored as 0 (checked_qual_sum, src/derep.rs:25-39)
    recs = [(b"TTTT", b"IIII"), (b"AAAA", b"!!!!"), (b"CCCC", b"IIII"), (b"AAAA", b"!!!!")]
    path = tmp_path / "t.fastq"
    _write(path, recs)
    got = D.derep_fastq(path, phred_offset=64)
    assert got.seqs == ["AAAA", "CCCC", "TTTT"]
    assert list(got.abund) == [2, 1, 1]
    assert list(got.quals[0]) == [0, 0, 0, 0]
    assert list(got.quals[1]) == [73 - 64] * 4
    assert list(got.map) == [2, 0, 1, 0]
    _same(got, O.derep(recs, 64))


def test_derep_of_an_empty_file(tmp_path):
    path = tmp_path / "e.fastq"
    path.write_bytes(b"")
    got = D.derep_fastq(path)
    assert got.seqs == [] and len(got.map) == 0


def test_derep_rejects_malformed_records(tmp_path):
    path = tmp_path / "m.fastq"
    path.write_bytes(b"@r0\nACGT\n+\nIII\n")
    with pytest.raises(D.InvalidInput, match="quality length"):
        D.derep_fastq(path)
    path.write_bytes(b"r0\nACGT\n+\nIIII\n")
    with pytest.raises(D.InvalidInput, match="header"):
        D.derep_fastq(path)
    with pytest.raises(D.InvalidInput, match="cannot open"):
        D.derep_fastq(tmp_path / "missing.fastq")
