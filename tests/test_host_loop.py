"""The product's clustering loop on the CPU: SampleState's absorb, shuffle,
p-update (floors, zero set), bud and final pass, driven by the oracle's
compare instead of the GPU kernels (tests/host_loop_driver.cpp), must give
the oracle's own run_dada result bit for bit. Host only: no GPU.

The sharded cases run the loop as W ranks (threads) of dgpu_dada_sharded's
exchange: each rank keeps only its own share's comps, and the product's
shard_exchange must rebuild the one-device store on every rank."""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

from dada2_b200 import synth
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _cuda_home():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return os.path.dirname(os.path.dirname(os.path.realpath(nvcc)))


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    cuda = _cuda_home()
    lib = os.path.join(cuda, "lib64")
    out = str(tmp_path_factory.mktemp("hostloop") / "driver")
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", os.path.join(ROOT, "dada2-rs_b200", "csrc"),
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"),
           os.path.join(ROOT, "tests", "host_loop_driver.cpp"), os.path.join(ROOT, "oracle", "dada_oracle.cpp"),
           os.path.join(ROOT, "oracle", "oracle_capi.cpp"), os.path.join(ROOT, "oracle", "oracle_learn.cpp"),
           os.path.join(ROOT, "dada2-rs_b200", "csrc", "dgpu_errfun.cpp"),
           os.path.join(ROOT, "dada2-rs_b200", "csrc", "dgpu_errfun_external.cpp"), "-o", out, "-L", lib,
           f"-Wl,-rpath,{lib}", "-lcudart", "-lpthread"]
    subprocess.run(cmd, check=True, capture_output=True)
    return out


def _run(driver, tmp_path, s, err, ncol, world=1, params=None, prior=None, fp32=False):
    enc = [x.encode() for x in s.seqs]
    lens = np.array([len(x) for x in enc], np.uint32)
    q = np.concatenate([np.asarray(a, np.uint32) for a in s.quals])
    path = tmp_path / "sample.bin"
    with open(path, "wb") as f:
        f.write(struct.pack("<iii", len(enc), int(lens.sum()), ncol))
        f.write(lens.tobytes())
        f.write(b"".join(enc))
        f.write(np.asarray(s.abund, np.uint32).tobytes())
        f.write(q.tobytes())
        f.write(np.ascontiguousarray(err, np.float64).tobytes())
        if params is not None:
            f.write(struct.pack("<dddd", params.omega_a, params.omega_p, params.omega_c, params.min_fold))
            f.write(struct.pack("<iiiiii", int(params.detect_singletons), int(params.greedy), params.min_hamming,
                                params.min_abund, params.max_clust, int(fp32)))
            pr = np.zeros(len(enc), np.uint8) if prior is None else np.asarray(prior, np.uint8)
            f.write(pr.tobytes())
    out = subprocess.run([driver, str(path), str(world)], check=True, capture_output=True, text=True).stdout
    rows = {}
    for line in out.splitlines():
        k, *v = line.split()
        rows[k] = v
    return rows


def _f64(hexes):
    return np.array([int(h, 16) for h in hexes], np.uint64).view(np.float64)


@pytest.mark.parametrize("case,world", [("small41", 1), ("small42", 1), ("config0", 1), ("pooled4", 1),
                                        ("small41", 2), ("config0", 3), ("pooled4", 4)])
def test_host_loop_matches_the_oracle(driver, tmp_path, case, world):
    if case == "config0":
        w = synth.config0()
    elif case == "pooled4":
        w = synth.config3(nsamples=4, nvariants=300, reads_per_sample=6000, workers=1)
    else:
        w = synth.small_illumina(int(case[-2:]), nvariants=7, nreads=4000, L=150)
    s = w.samples[0]
    got = _run(driver, tmp_path, s, w.err, w.ncol, world)
    want = O.dada(s.seqs, s.abund, w.err, w.ncol, O.DadaParams(nthreads=4), quals=s.quals)
    assert int(got["nclust"][0]) == want["nclust"]
    assert np.array_equal(np.array(got["map"], np.int64), want["map"].astype(np.int64))
    assert _f64(got["pvals"]).tobytes() == want["pvals"].tobytes()
    assert [int(x) for x in got["cl_reads"]] == [c["reads"] for c in want["clusters"]]
    assert [int(x) for x in got["cl_birth_type"]] == [c["birth_type"] for c in want["clusters"]]
    off = [int(x) for x in got["cl_mem_off"]]
    raws = np.array(got["mem_raw"], np.int64)
    lam, pv = _f64(got["mem_lambda"]), _f64(got["mem_pval"])
    bp, bf, be = _f64(got["cl_birth_pval"]), _f64(got["cl_birth_fold"]), _f64(got["cl_birth_e"])
    for ci, c in enumerate(want["clusters"]):
        a, b = off[ci], off[ci + 1]
        assert np.array_equal(raws[a:b], c["members"].astype(np.int64))
        assert lam[a:b].tobytes() == c["lambdas"].tobytes()
        assert pv[a:b].tobytes() == c["pvals"].tobytes()
        assert np.float64(bp[ci]).tobytes() == np.float64(c["birth_pval"]).tobytes()
        assert np.float64(bf[ci]).tobytes() == np.float64(c["birth_fold"]).tobytes()
        assert np.float64(be[ci]).tobytes() == np.float64(c["birth_e"]).tobytes()


@pytest.mark.parametrize("world,fail", [(2, "1:0"), (3, "0:5"), (3, "2:3")])
def test_sharded_failure_stops_every_rank_at_the_same_exchange(driver, tmp_path, world, fail):
    """A rank whose compare fails reports it in its exchange head; every rank
    leaves the loop at that exchange with an error (none waits for good)."""
    w = synth.small_illumina(41, nvariants=7, nreads=4000, L=150)
    s = w.samples[0]
    _run(driver, tmp_path, s, w.err, w.ncol, world)  # writes sample.bin
    res = subprocess.run([driver, str(tmp_path / "sample.bin"), str(world), fail], capture_output=True, text=True,
                         timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
    call = fail.split(":")[1]
    lines = res.stdout.splitlines()
    assert len(lines) == world
    bad = int(fail.split(":")[0])
    for r, line in enumerate(lines):
        assert line.startswith(f"rank {r} rc 6 failed at call {call}:")
        if r != bad:
            assert f"rank {bad} of the sharded run failed" in line


def _check(got, want):
    assert int(got["nclust"][0]) == want["nclust"]
    assert np.array_equal(np.array(got["map"], np.int64), want["map"].astype(np.int64))
    assert _f64(got["pvals"]).tobytes() == want["pvals"].tobytes()
    assert [int(x) for x in got["cl_reads"]] == [c["reads"] for c in want["clusters"]]
    assert [int(x) for x in got["cl_birth_type"]] == [c["birth_type"] for c in want["clusters"]]
    assert [int(x) for x in got["cl_birth_from"]] == [c["birth_from"] for c in want["clusters"]]
    off = [int(x) for x in got["cl_mem_off"]]
    raws = np.array(got["mem_raw"], np.int64)
    lam, pv = _f64(got["mem_lambda"]), _f64(got["mem_pval"])
    for ci, c in enumerate(want["clusters"]):
        a, b = off[ci], off[ci + 1]
        assert np.array_equal(raws[a:b], c["members"].astype(np.int64))
        assert lam[a:b].tobytes() == c["lambdas"].tobytes()
        assert pv[a:b].tobytes() == c["pvals"].tobytes()


# parameter regimes of the host phases: singleton detection, priors (omega_p,
# the prior bud), no greedy skip, fold and hamming filters, a cluster cap, an
# abundance floor; each also as two sharded ranks
# (on this sample the default run gives 9 clusters; these give 52, 10, 9 with
# a Prior birth, 13 and 3)
REGIMES = {
    "singletons": dict(detect_singletons=True, omega_a=0.5),
    "min_abund": dict(detect_singletons=True, omega_a=0.5, min_abund=2),
    "priors": dict(omega_p=1e-2),
    "nogreedy_fold_ham": dict(detect_singletons=True, omega_a=0.5, greedy=False, min_fold=4.0, min_hamming=3),
    "max_clust": dict(max_clust=3),
}


@pytest.mark.parametrize("world", [1, 2])
@pytest.mark.parametrize("regime", sorted(REGIMES))
def test_host_loop_parameter_regimes_match_the_oracle(driver, tmp_path, regime, world):
    w = synth.small_illumina(43, nvariants=9, nreads=5000, L=150)
    s = w.samples[0]
    params = O.DadaParams(nthreads=4, **REGIMES[regime])
    prior = None
    if regime == "priors":
        rng = np.random.default_rng(7)
        prior = np.zeros(len(s.seqs), np.uint8)
        prior[rng.choice(len(s.seqs), size=min(25, len(s.seqs)), replace=False)] = 1
    got = _run(driver, tmp_path, s, w.err, w.ncol, world, params=params, prior=prior)
    want = O.dada(s.seqs, s.abund, w.err, w.ncol, params, quals=s.quals,
                  prior=None if prior is None else prior.astype(bool))
    _check(got, want)


@pytest.mark.parametrize("world", [1, 2])
@pytest.mark.parametrize("case", ["small41", "singletons"])
def test_host_loop_fp32_decisions_keep_the_partition(driver, tmp_path, case, world):
    """FP32-decision mode (exp of the FP32 ln lambda, FP64 within 1e3x of the
    thresholds): the partition equals the oracle's FP64 run."""
    w = synth.small_illumina(41 if case == "small41" else 43, nvariants=7 if case == "small41" else 9,
                             nreads=4000 if case == "small41" else 5000, L=150)
    s = w.samples[0]
    params = O.DadaParams(nthreads=4, **({} if case == "small41" else REGIMES["singletons"]))
    got = _run(driver, tmp_path, s, w.err, w.ncol, world, params=params, fp32=True)
    want = O.dada(s.seqs, s.abund, w.err, w.ncol, params, quals=s.quals)
    assert int(got["fp32"][0]) > 0
    assert int(got["nclust"][0]) == want["nclust"]
    assert np.array_equal(np.array(got["map"], np.int64), want["map"].astype(np.int64))
    assert [int(x) for x in got["cl_reads"]] == [c["reads"] for c in want["clusters"]]
    off = [int(x) for x in got["cl_mem_off"]]
    raws = np.array(got["mem_raw"], np.int64)
    for ci, c in enumerate(want["clusters"]):
        assert np.array_equal(np.sort(raws[off[ci]:off[ci + 1]]), np.sort(c["members"].astype(np.int64)))
