"""Error-model fits of learn-errors (CPU only).

The product's fit (dgpu_errfun_apply, host code in the library) and the
oracle's restatement are each held to the reference's own errfun tests
(src/error_models.rs tests: an empty matrix is an error, one populated
quality column fits a constant (11 / 10,030), binned-quality schemes fit,
the diagonal is 1 minus the off-diagonals), and to each other bit for bit on
random transition matrices, for LOESS on both surfaces and for noqual.
"""
import re
import sys

import numpy as np
import pytest

import dada2_b200 as D
from oracle import oracle as O

KINDS = [({}, D.ErrFun()), ({"surface": 1}, D.ErrFun(surface="interpolate")), ({"kind": 1}, D.ErrFun(kind="noqual"))]


def both(trans, nq, okw, ef):
    return O.errfun_apply(trans, nq, **okw), D.errfun_apply(trans, nq, ef)


def test_empty_matrix_is_an_error():
    """src/error_models.rs: loess_errfun_errors_on_an_empty_transition_matrix."""
    nq = 40
    t = np.zeros((16, nq), np.uint32)
    with pytest.raises(ValueError, match="all 12 transitions"):
        O.errfun_apply(t, nq)
    with pytest.raises(D.DgpuError, match="all 12 transitions"):
        D.errfun_apply(t, nq)


def test_single_populated_column_fits_a_constant():
    """src/error_models.rs: loess_errfun_single_populated_column_fits_a_constant."""
    nq = 40
    t = np.zeros((16, nq), np.uint32)
    for i in range(4):
        for j in range(4):
            t[i * 4 + j, 30] = 10_000 if i == j else 10
    for okw, ef in KINDS[:2]:
        a, b = both(t, nq, okw, ef)
        assert a.tobytes() == b.tobytes()
        assert np.all(np.abs(a[1] - 11.0 / 10_030.0) < 1e-12)


@pytest.mark.parametrize("bins", [[12, 24, 38], [2, 12, 23, 37]])
def test_binned_quality_schemes_fit(bins):
    """src/error_models.rs: loess_errfun_fits_binned_quality_schemes."""
    nq = 40
    t = np.zeros((16, nq), np.uint32)
    for rank, q in enumerate(bins):
        for i in range(4):
            for j in range(4):
                t[i * 4 + j, q] = 10_000 * (rank + 1) if i == j else 100 // (rank + 1) + 1
    for okw, ef in KINDS[:2]:
        a, b = both(t, nq, okw, ef)
        assert a.tobytes() == b.tobytes()
        off = np.array([a[i * 4 + j] for i in range(4) for j in range(4) if i != j])
        assert np.any(off > 1e-7)
        assert np.all((a >= 0.0) & (a <= 1.0))


def test_diagonal_is_one_minus_the_off_diagonals():
    """src/error_models.rs: test_expand_err_matrix_diagonal, through a flat
    noqual fit: every off-diagonal equal gives diagonal 1 - 3 x rate."""
    nq = 3
    t = np.full((16, nq), 1000, np.uint32)
    a, b = both(t, nq, {"kind": 1}, D.ErrFun(kind="noqual"))
    assert a.tobytes() == b.tobytes()
    rate = (3000 + 1.0) / (4 * 3001.0)
    for i in range(4):
        assert np.allclose(a[i * 5], 1.0 - 3 * rate, atol=1e-12)


def test_rates_are_clamped():
    nq = 20
    t = np.zeros((16, nq), np.uint32)
    t[0] = 1_000_000  # A: no errors at all
    t[1] = 1_000_000  # C from A as often as A itself
    t[5] = 1000
    t[10] = 1000
    t[15] = 1000
    for okw, ef in KINDS:
        a, b = both(t, nq, okw, ef)
        assert a.tobytes() == b.tobytes()
        off = np.array([a[i * 4 + j] for i in range(4) for j in range(4) if i != j])
        assert off.min() >= 1e-7 and off.max() <= 0.25


@pytest.mark.parametrize("seed", range(6))
def test_product_fit_equals_the_oracle_bit_for_bit(seed):
    rng = np.random.default_rng(seed)
    for _ in range(40):
        nq = int(rng.integers(3, 60))
        t = rng.integers(0, int(10 ** rng.uniform(0, 5)), size=(16, nq)).astype(np.uint32)
        for i in range(4):
            t[i * 5] *= int(rng.integers(1, 2000))
        t[:, rng.random(nq) < 0.2] = 0
        for okw, ef in KINDS:
            try:
                a = O.errfun_apply(t, nq, **okw)
            except ValueError:
                with pytest.raises(D.DgpuError):
                    D.errfun_apply(t, nq, ef)
                continue
            b = D.errfun_apply(t, nq, ef)
            assert a.tobytes() == b.tobytes(), (nq, okw)


def _binned_case(rng, nq):
    bins = np.sort(rng.choice(np.arange(nq), size=int(rng.integers(2, min(6, nq + 1))), replace=False)).astype(np.float64)
    t = np.zeros((16, nq), np.uint32)
    lo, hi = int(bins[0]), int(bins[-1])
    cols = rng.integers(lo, hi + 1, size=int(rng.integers(1, 8)))
    for q in cols:
        t[:, q] = rng.integers(0, 2000, size=16)
        for i in range(4):
            t[i * 5, q] += int(rng.integers(1000, 50000))
    return t, bins


@pytest.mark.parametrize("seed", range(6))
def test_binned_fit_equals_the_oracle_bit_for_bit(seed):
    """binned_qual_errfun (src/error_models.rs:263-396), product against oracle."""
    rng = np.random.default_rng(100 + seed)
    for _ in range(30):
        nq = int(rng.integers(4, 50))
        t, bins = _binned_case(rng, nq)
        try:
            a = O.errfun_apply(t, nq, kind=2, bins=bins)
        except ValueError as e:
            with pytest.raises(D.DgpuError, match=re.escape(str(e))):
                D.errfun_apply(t, nq, D.ErrFun(kind="binned", bins=tuple(bins)))
            continue
        b = D.errfun_apply(t, nq, D.ErrFun(kind="binned", bins=tuple(bins)))
        assert a.tobytes() == b.tobytes(), (nq, bins)


def test_binned_fit_interpolates_between_anchors():
    """The observed rate at each anchor, linear between them, flat outside."""
    nq = 41
    bins = (10.0, 20.0, 40.0)
    t = np.zeros((16, nq), np.uint32)
    for q, e in ((10, 100), (20, 300), (40, 50)):
        for i in range(4):
            for j in range(4):
                t[i * 4 + j, q] = 100_000 if i == j else e
    got = D.errfun_apply(t, nq, D.ErrFun(kind="binned", bins=bins))
    r = {q: e / (100_000 + 3 * e) for q, e in ((10, 100), (20, 300), (40, 50))}
    assert got[1, 10] == r[10] and got[1, 20] == r[20] and got[1, 40] == r[40]
    assert got[1, 0] == r[10]  # flat below the first anchor
    assert abs(got[1, 15] - (r[10] * 0.5 + r[20] * 0.5)) < 1e-18
    assert abs(got[1, 30] - (r[20] * 0.5 + r[40] * 0.5)) < 1e-18
    assert np.allclose(got[0], 1.0 - got[1] - got[2] - got[3])


def test_binned_fit_errors():
    """No observations, and observed qualities outside the anchors, are errors."""
    nq = 30
    t = np.zeros((16, nq), np.uint32)
    for ef, kw in ((D.ErrFun(kind="binned", bins=(5.0, 20.0)), {"kind": 2, "bins": [5.0, 20.0]}),):
        with pytest.raises(ValueError, match="No observed transitions"):
            O.errfun_apply(t, nq, **kw)
        with pytest.raises(D.DgpuError, match="No observed transitions"):
            D.errfun_apply(t, nq, ef)
        t2 = t.copy()
        t2[0, 25] = 10
        with pytest.raises(ValueError, match="quality score 25 higher than max binned value 20"):
            O.errfun_apply(t2, nq, **kw)
        with pytest.raises(D.DgpuError, match="quality score 25 higher than max binned value 20"):
            D.errfun_apply(t2, nq, ef)
        t3 = t.copy()
        t3[0, 2] = 10
        with pytest.raises(D.DgpuError, match="quality score 2 lower than min binned value 5"):
            D.errfun_apply(t3, nq, ef)


def _pacbio_trans(rng, nq):
    t = rng.integers(0, 300, size=(16, nq)).astype(np.uint32)
    for i in range(4):
        t[i * 5] += rng.integers(5_000, 90_000, size=nq).astype(np.uint32)
    t[:, rng.random(nq) < 0.15] = 0
    return t


@pytest.mark.parametrize("seed", range(3))
def test_pacbio_fit(seed):
    """pacbio_errfun (src/error_models.rs:408-462): with a Q93 column (nq = 94)
    LOESS below it and (count + 1) / (total + 4) in it; otherwise LOESS."""
    rng = np.random.default_rng(200 + seed)
    nq = 94
    t = _pacbio_trans(rng, nq)
    a = O.errfun_apply(t, nq, kind=3)
    b = D.errfun_apply(t, nq, D.ErrFun(kind="pacbio"))
    assert a.tobytes() == b.tobytes()
    below = D.errfun_apply(np.ascontiguousarray(t[:, :93]), 93, D.ErrFun())
    assert b[:, :93].tobytes() == below.tobytes()
    for i in range(4):
        tot = float(t[i * 4:i * 4 + 4, 93].sum())
        for j in range(4):
            assert b[i * 4 + j, 93] == (float(t[i * 4 + j, 93]) + 1.0) / (tot + 4.0)
    t2 = _pacbio_trans(rng, 60)
    assert D.errfun_apply(t2, 60, D.ErrFun(kind="pacbio")).tobytes() == D.errfun_apply(t2, 60, D.ErrFun()).tobytes()
    assert O.errfun_apply(t2, 60, kind=3).tobytes() == D.errfun_apply(t2, 60, D.ErrFun(kind="pacbio")).tobytes()


def _script(tmp_path, name, body):
    p = tmp_path / name
    p.write_text("#!/bin/sh\n" + body)
    return f"/bin/sh {p}"


def _ext(cmd):
    return D.ErrFun(kind="external", cmd=cmd)


def test_external_fit_round_trip(tmp_path, monkeypatch):
    """external_errfun (src/error_models.rs:650-705): the command reads the
    transitions' TSV and writes the error matrix's (the reference's
    test_external_errfun_roundtrip: a constant 0.01 comes back)."""
    monkeypatch.setenv("TMPDIR", str(tmp_path))
    cmd = _script(tmp_path, "const.sh", "awk -F'\\t' 'NR==1{print; n=NF-1; next} "
                  "{s=$1; for(i=1;i<=n;i++) s=s \"\\t0.01\"; print s}' \"$1\" > \"$2\"\n")
    nq = 4
    t = np.arange(16 * nq, dtype=np.uint32).reshape(16, nq)
    got = D.errfun_apply(t, nq, _ext(cmd))
    assert np.all(got == 0.01)
    assert [p.name for p in tmp_path.iterdir() if p.name.startswith("dada2-rs-errfun")] == []  # folder removed


def test_external_fit_reads_the_transitions(tmp_path, monkeypatch):
    """The command sees the layout of R's read.table (header of a tab and
    0..nq-1, rows A2A..T2T) and its numbers come back exactly."""
    monkeypatch.setenv("TMPDIR", str(tmp_path))
    prog = tmp_path / "fit.py"
    prog.write_text(
        "import sys\n"
        "rows = open(sys.argv[1]).read().split('\\n')\n"
        "out = [rows[0]]\n"
        "for r in rows[1:17]:\n"
        "    f = r.split('\\t')\n"
        "    out.append('\\t'.join([f[0]] + [repr((int(x) + 1) / 1000.0) for x in f[1:]]))\n"
        "open(sys.argv[2], 'w').write('\\n'.join(out) + '\\n')\n")
    nq = 7
    rng = np.random.default_rng(3)
    t = rng.integers(0, 999, size=(16, nq)).astype(np.uint32)
    got = D.errfun_apply(t, nq, _ext(f"{sys.executable} {prog}"))
    assert got.tobytes() == ((t.astype(np.float64) + 1.0) / 1000.0).tobytes()
    head = "\t" + "\t".join(str(q) for q in range(nq))
    labels = [a + "2" + b for a in "ACGT" for b in "ACGT"]
    echo = _script(tmp_path, "echo.sh", "cp \"$1\" \"$TMPDIR/seen.tsv\"; awk -F'\\t' 'NR==1{print; n=NF-1; next} "
                   "{s=$1; for(i=1;i<=n;i++) s=s \"\\t0\"; print s}' \"$1\" > \"$2\"\n")
    D.errfun_apply(t, nq, _ext(echo))
    lines = (tmp_path / "seen.tsv").read_text().split("\n")
    assert lines[0] == head and [ln.split("\t")[0] for ln in lines[1:17]] == labels
    assert [[int(x) for x in ln.split("\t")[1:]] for ln in lines[1:17]] == t.tolist()


def test_external_fit_errors(tmp_path, monkeypatch):
    """A failing command's status and standard error, an invalid probability
    (the reference's test_external_errfun_propagates_nonzero_exit and
    test_external_errfun_rejects_invalid_probability), an empty command and a
    malformed table are errors."""
    monkeypatch.setenv("TMPDIR", str(tmp_path))
    t = np.zeros((16, 4), np.uint32)
    fail = _script(tmp_path, "fail.sh", "echo 'oops' >&2\nexit 7\n")
    with pytest.raises(D.DgpuError, match=r"exited with exit status: 7\n--- stderr ---\noops"):
        D.errfun_apply(t, 4, _ext(fail))
    bad = _script(tmp_path, "bad.sh", "awk -F'\\t' 'NR==1{print; n=NF-1; next} "
                  "{s=$1 \"\\t1.5\"; for(i=2;i<=n;i++) s=s \"\\t0.01\"; print s}' \"$1\" > \"$2\"\n")
    with pytest.raises(D.DgpuError, match=re.escape("err[A2A][0] = 1.5 is not a valid probability in [0, 1]")):
        D.errfun_apply(t, 4, _ext(bad))
    with pytest.raises(D.DgpuError, match="--errfun-cmd is empty"):
        D.errfun_apply(t, 4, _ext("   "))
    word = _script(tmp_path, "word.sh", "awk -F'\\t' 'NR==1{print; n=NF-1; next} "
                   "{s=$1 \"\\tabc\"; for(i=2;i<=n;i++) s=s \"\\t0\"; print s}' \"$1\" > \"$2\"\n")
    with pytest.raises(D.DgpuError, match=re.escape('row 1 column 0 ("abc"): invalid float literal')):
        D.errfun_apply(t, 4, _ext(word))
    short = _script(tmp_path, "short.sh", "head -n 5 \"$1\" > \"$2\"\n")
    with pytest.raises(D.DgpuError, match="err TSV has 4 data rows, expected 16"):
        D.errfun_apply(t, 4, _ext(short))
    with pytest.raises(D.DgpuError, match="failed to spawn"):
        D.errfun_apply(t, 4, _ext(str(tmp_path / "no-such-program")))
    assert [p.name for p in tmp_path.iterdir() if p.name.startswith("dada2-rs-errfun")] == []
