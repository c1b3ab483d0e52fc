"""Seeded synthetic amplicon samples with the shapes of the benchmark configs.

No public dataset is named for these workloads and the reference's real
datasets are not available, so every input is generated here, deterministically
from ``seed = 1000 + config``:

* true variants are uniform-random ACGT;
* reads are drawn from the variants with the stated abundance law;
* substitutions follow a 16 x nq transition-by-quality error matrix whose rows
  are ``ref*4 + query`` (A=0..T=3) and whose columns are Phred Q, the layout the
  compare step reads (error rate 10^(-Q/10), transitions twice as likely as
  transversions, off-diagonals clamped to [1e-7, 0.25], diagonal = 1 - sum);
* reads are dereplicated the way the reference's derep does it
  (src/derep.rs:179-185): uniques by abundance descending, ties by sequence
  ascending, with per-position integer Phred SUMS (u32).

The same matrix is handed to the denoiser as its error model.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

NT = np.frombuffer(b"ACGT", np.uint8)
# transitions A<->G and C<->T weigh 2, transversions 1 (per reference base)
_W = np.array([[0, 1, 2, 1], [1, 0, 1, 2], [2, 1, 0, 1], [1, 2, 1, 0]], np.float64)


@dataclass
class Sample:
    """One dereplicated sample: ASCII uniques, abundances and Phred sums."""
    seqs: list
    abund: np.ndarray
    quals: list
    nreads: int = 0
    name: str = ""


@dataclass
class Workload:
    config: int
    name: str
    samples: list
    err: np.ndarray   # flat 16 x ncol, row-major
    ncol: int
    band: int = 16
    homo_gap_p: int = -8
    kmer_size: int = 5
    notes: dict = field(default_factory=dict)


def error_matrix(nq: int, floor: float = 0.0) -> np.ndarray:
    """16 x nq matrix: err[(ref*4+qry), Q]."""
    q = np.arange(nq, dtype=np.float64)
    e = np.maximum(10.0 ** (-q / 10.0), floor)
    m = np.zeros((16, nq))
    for a in range(4):
        off = np.clip(np.outer(_W[a] / 4.0, e), 1e-7, 0.25)
        off[a] = 0.0
        for b in range(4):
            m[a * 4 + b] = off[b]
        m[a * 4 + a] = 1.0 - off.sum(axis=0)
    return m.reshape(-1)


def _random_variants(rng, n, lengths):
    return [rng.integers(0, 4, size=int(L)).astype(np.uint8) for L in lengths[:n]]


def _apply_subs(rng, reads_codes, quals, errm, ncol):
    """Substitute per position with probability 1 - err[diag, Q]; draw the
    replacement base proportionally to the off-diagonal rates."""
    n, L = reads_codes.shape
    e = errm.reshape(16, ncol)
    diag_rows = reads_codes.astype(np.int64) * 5  # row a*4+a
    p_err = 1.0 - e[diag_rows, quals]
    hit = rng.random((n, L)) < p_err
    if not hit.any():
        return reads_codes
    ri, ci = np.nonzero(hit)
    ref = reads_codes[ri, ci].astype(np.int64)
    qv = quals[ri, ci]
    w = np.stack([e[ref * 4 + b, qv] for b in range(4)], axis=1)
    w[np.arange(len(ref)), ref] = 0.0
    w /= w.sum(axis=1, keepdims=True)
    u = rng.random(len(ref))[:, None]
    newb = (u > np.cumsum(w, axis=1)).sum(axis=1)
    out = reads_codes.copy()
    out[ri, ci] = np.minimum(newb, 3).astype(np.uint8)
    return out


def _derep(seq_rows, qual_rows):
    """Group identical reads: returns ASCII uniques sorted by (-count, seq)."""
    keys = {}
    counts = []
    qsums = []
    order = []
    for s, q in zip(seq_rows, qual_rows):
        k = s.tobytes()
        j = keys.get(k)
        if j is None:
            keys[k] = len(counts)
            counts.append(1)
            qsums.append(q.astype(np.uint32).copy())
            order.append(k)
        else:
            counts[j] += 1
            qsums[j] += q
    ascii_seqs = [NT[np.frombuffer(k, np.uint8)].tobytes().decode() for k in order]
    idx = sorted(range(len(order)), key=lambda t: (-counts[t], ascii_seqs[t]))
    return ([ascii_seqs[t] for t in idx], np.array([counts[t] for t in idx], np.uint32),
            [qsums[t] for t in idx])


def illumina_sample(rng, nvariants, nreads, L, errm, ncol, abund_exp=1.5, qhi=38, qlo=25,
                    qsd=2.0, qmin=2, qmax=41, chunk=20000):
    variants = _random_variants(rng, nvariants, [L] * nvariants)
    w = np.arange(1, nvariants + 1, dtype=np.float64) ** (-abund_exp)
    w /= w.sum()
    vidx = rng.choice(nvariants, size=nreads, p=w)
    prof = np.linspace(qhi, qlo, L)
    vmat = np.stack(variants)
    # reads may carry Q above the model's last column (the denoiser then extends
    # the model by repeating that column, src/dada.rs:337-384); draw their
    # errors from the un-truncated rate law
    gen = error_matrix(qmax + 1) if qmax + 1 > ncol else errm
    gcol = max(qmax + 1, ncol)
    seq_rows, qual_rows = [], []
    for lo in range(0, nreads, chunk):
        hi = min(nreads, lo + chunk)
        n = hi - lo
        q = np.clip(np.rint(prof[None, :] + rng.normal(0.0, qsd, size=(n, L))), qmin, qmax).astype(np.int64)
        codes = _apply_subs(rng, vmat[vidx[lo:hi]], q, gen, gcol)
        seq_rows.extend(codes)
        qual_rows.extend(q.astype(np.uint32))
    seqs, abund, quals = _derep(seq_rows, qual_rows)
    return Sample(seqs, abund, quals, nreads)


def _homopolymer_mask(codes):
    n = len(codes)
    m = np.zeros(n, bool)
    s = 0
    while s < n:
        e = s + 1
        while e < n and codes[e] == codes[s]:
            e += 1
        if e - s >= 3:
            m[s:e] = True
        s = e
    return m


def pacbio_sample(rng, nvariants, nuniques, lmin, lmax, errm, ncol, sub_rate=2e-3, indel_rate=5e-3,
                  qbins=(40, 50, 60, 70, 80, 93)):
    lengths = rng.integers(lmin, lmax + 1, size=nvariants)
    variants = _random_variants(rng, nvariants, lengths)
    masks = [_homopolymer_mask(v) for v in variants]
    w = np.arange(1, nvariants + 1, dtype=np.float64) ** (-1.0)
    w /= w.sum()
    qb = np.array(qbins)
    seq_rows, qual_rows = {}, {}
    uniques = set()
    nreads = 0
    while len(uniques) < nuniques:
        v = int(rng.choice(nvariants, p=w))
        base = variants[v]
        L = len(base)
        # homopolymer indels: inside runs of >= 3, a base is dropped or doubled
        hit = (rng.random(L) < indel_rate) & masks[v]
        ins = rng.random(L) < 0.5
        codes = []
        for t in range(L):
            if not hit[t]:
                codes.append(base[t])
            elif ins[t]:
                codes.extend((base[t], base[t]))  # run extended by one
        codes = np.array(codes, np.uint8)
        sub = rng.random(len(codes)) < sub_rate
        if sub.any():
            codes[sub] = (codes[sub] + rng.integers(1, 4, size=int(sub.sum()))) % 4
        q = qb[rng.integers(0, len(qb), size=len(codes))].astype(np.uint32)
        k = codes.tobytes()
        nreads += 1
        if k in seq_rows:
            seq_rows[k][1] += 1
            qual_rows[k] += q
        else:
            seq_rows[k] = [codes, 1]
            qual_rows[k] = q.copy()
            uniques.add(k)
    keys = list(seq_rows.keys())
    ascii_seqs = {k: NT[np.frombuffer(k, np.uint8)].tobytes().decode() for k in keys}
    keys.sort(key=lambda k: (-seq_rows[k][1], ascii_seqs[k]))
    return Sample([ascii_seqs[k] for k in keys], np.array([seq_rows[k][1] for k in keys], np.uint32),
                  [qual_rows[k] for k in keys], nreads)


def config0(seed: int = 1000) -> Workload:
    """Plain single-sample Illumina: 20 variants x 250 nt, 20,000 reads, Zipf 1.5."""
    rng = np.random.default_rng(seed)
    ncol = 41
    errm = error_matrix(ncol)
    s = illumina_sample(rng, 20, 20000, 250, errm, ncol)
    s.name = "config0"
    return Workload(0, "plain single-sample Illumina (20 variants x 250 nt, 20k reads)", [s], errm, ncol)


def config1(seed: int = 1001, nsamples: int = 40, umin: int = 500, umax: int = 30000) -> Workload:
    """40 samples, uniques log-uniform in [500, 30000], 250/220 nt alternating,
    50-400 variants each."""
    rng = np.random.default_rng(seed)
    ncol = 41
    errm = error_matrix(ncol)
    samples = []
    for si in range(nsamples):
        target = int(np.exp(rng.uniform(np.log(umin), np.log(umax))))
        nvar = int(rng.integers(50, 401))
        L = 250 if si % 2 == 0 else 220
        # ~16% of reads carry an error at this quality profile and nearly all of
        # those are unique, so size the read count to land near the target
        nreads = max(int((target - nvar) / 0.155), 2 * nvar)
        s = illumina_sample(rng, nvar, nreads, L, errm, ncol)
        s.name = f"config1.s{si}"
        samples.append(s)
    return Workload(1, "batched 40-sample Illumina (250/220 nt, 500-30k uniques)", samples, errm, ncol)


def config2(seed: int = 1002, nuniques: int = 5000) -> Workload:
    """PacBio full-length 16S: 60 variants of 1400-1550 nt, indel-heavy."""
    rng = np.random.default_rng(seed)
    ncol = 94
    errm = error_matrix(ncol, floor=1e-3)
    s = pacbio_sample(rng, 60, nuniques, 1400, 1550, errm, ncol)
    s.name = "config2"
    return Workload(2, "PacBio full-length 16S (1400-1550 nt, band 32, homopolymer gap -1)", [s], errm,
                    ncol, band=32, homo_gap_p=-1)


def small_illumina(seed: int, nvariants=8, nreads=3000, L=150) -> Workload:
    """A seconds-scale Illumina sample for parity tests."""
    rng = np.random.default_rng(seed)
    ncol = 41
    errm = error_matrix(ncol)
    s = illumina_sample(rng, nvariants, nreads, L, errm, ncol)
    s.name = f"small{seed}"
    return Workload(-1, "small Illumina parity case", [s], errm, ncol)


def _pooled_part(seed: int, vmat: np.ndarray, weights: np.ndarray, nreads: int, qhi=38, qlo=25, qsd=2.0,
                 qmin=2, qmax=41, chunk=20000):
    """One sample of the pooled workload, dereplicated (src/derep.rs:179-185)."""
    rng = np.random.default_rng(seed)
    nvar, L = vmat.shape
    vidx = rng.choice(nvar, size=nreads, p=weights)
    prof = np.linspace(qhi, qlo, L)
    gen = error_matrix(qmax + 1)
    seq_rows, qual_rows = [], []
    for lo in range(0, nreads, chunk):
        hi = min(nreads, lo + chunk)
        q = np.clip(np.rint(prof[None, :] + rng.normal(0.0, qsd, size=(hi - lo, L))), qmin, qmax).astype(np.int64)
        seq_rows.extend(_apply_subs(rng, vmat[vidx[lo:hi]], q, gen, qmax + 1))
        qual_rows.extend(q.astype(np.uint32))
    return _derep(seq_rows, qual_rows)


def pool_samples(parts):
    """Pooled uniques in first-seen order over the samples in input order, each
    sample's uniques in its derep order; counts and per-position Phred sums add
    up (src/main.rs:1355-1398)."""
    index, seqs, counts, quals = {}, [], [], []
    for s_seqs, s_counts, s_quals in parts:
        for sq, c, q in zip(s_seqs, s_counts, s_quals):
            j = index.get(sq)
            if j is None:
                index[sq] = len(seqs)
                seqs.append(sq)
                counts.append(int(c))
                quals.append(np.array(q, np.uint32))
            else:
                counts[j] += int(c)
                quals[j] += q
    return seqs, np.array(counts, np.uint32), quals


def config3(seed: int = 1003, nsamples: int = 200, nvariants: int = 3000, L: int = 150,
            reads_per_sample: int = 38000, workers: int | None = None) -> Workload:
    """Pooled mode: 3,000 variants x 150 nt with log-normal (sigma 2) abundances,
    200 samples of Illumina-style reads (Q38->25 + N(0,2)) dereplicated and
    pooled in first-seen order into about 400,000 uniques. Samples are
    generated in a spawn-started process pool."""
    import concurrent.futures as cf
    import multiprocessing as mp
    import os

    rng = np.random.default_rng(seed)
    vmat = np.stack(_random_variants(rng, nvariants, [L] * nvariants))
    w = np.exp(rng.normal(0.0, 2.0, size=nvariants))
    w /= w.sum()
    seeds = [seed * 1000 + i for i in range(nsamples)]
    nw = workers or max(1, min(nsamples, (os.cpu_count() or 2) // 2))
    if nw > 1:
        with cf.ProcessPoolExecutor(nw, mp_context=mp.get_context("spawn")) as ex:
            parts = list(ex.map(_pooled_part, seeds, [vmat] * nsamples, [w] * nsamples,
                                [reads_per_sample] * nsamples, chunksize=4))
    else:
        parts = [_pooled_part(sd, vmat, w, reads_per_sample) for sd in seeds]
    seqs, counts, quals = pool_samples(parts)
    s = Sample(seqs, counts, quals, nsamples * reads_per_sample, name="config3.pooled")
    return Workload(3, f"pooled {nsamples}-sample Illumina ({nvariants} variants x {L} nt, "
                       f"{len(seqs)} pooled uniques)", [s], error_matrix(41), 41)


# fraction of reads that end up unique at each length under the Q38->Q25
# profile (measured on this generator), used to size a request's read count
_UNIQUE_FRAC = {150: 0.076, 250: 0.145, 1450: 0.78}


def service_request(seed: int, L: int, target: int, nvar: int) -> Sample:
    """One request of the service trace: an Illumina-style sample of length L
    with about ``target`` uniques from ``nvar`` variants (the error model is the
    service's resident 16 x 41 matrix)."""
    rng = np.random.default_rng(seed)
    ncol = 41
    errm = error_matrix(ncol)
    nreads = max(int(target / _UNIQUE_FRAC[L]), 2 * nvar)
    s = illumina_sample(rng, nvar, nreads, L, errm, ncol)
    s.name = f"req{seed}"
    return s


def config4(seed: int = 1004, nrequests: int = 48, rate: float = 20.0, workers: int | None = None) -> Workload:
    """Denoising-service trace: Poisson arrivals at ``rate``/s; uniques per
    request log-normal with median 5,000 (sigma 1) clipped to [1,000, 50,000];
    lengths 150 / 250 / 1,450 nt drawn 60 / 30 / 10 %; 50-200 variants each.
    Requests are generated in a spawn-started process pool."""
    import concurrent.futures as cf
    import multiprocessing as mp
    import os

    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=nrequests))
    arrivals -= arrivals[0]
    lengths = rng.choice([150, 250, 1450], size=nrequests, p=[0.6, 0.3, 0.1])
    targets = np.clip(np.rint(np.exp(rng.normal(np.log(5000.0), 1.0, size=nrequests))), 1000, 50000).astype(int)
    nvars = rng.integers(50, 201, size=nrequests)
    seeds = [seed * 1000 + i for i in range(nrequests)]
    nw = workers or max(1, min(nrequests, (os.cpu_count() or 2) // 2))
    args = list(zip(seeds, lengths.tolist(), targets.tolist(), nvars.tolist()))
    if nw > 1:
        with cf.ProcessPoolExecutor(nw, mp_context=mp.get_context("spawn")) as ex:
            samples = list(ex.map(service_request, *zip(*args)))
    else:
        samples = [service_request(*a) for a in args]
    return Workload(4, f"denoising service ({nrequests} requests, Poisson {rate:g}/s, 150/250/1450 nt 60/30/10%)",
                    samples, error_matrix(41), 41,
                    notes={"arrivals": arrivals, "lengths": lengths, "targets": targets, "rate": rate})


CONFIGS = {0: config0, 1: config1, 2: config2, 3: config3, 4: config4}
