"""Extract the inline known-answer vectors of the reference's own unit tests.

The reference (HPCBio/dada2-rs, Rust) cannot be built in this image, so its
tests are read as text: this script pulls the literal inputs, seeds and
expected values out of the `#[cfg(test)]` modules and writes them, each with
the file:line it came from, to ``reference_vectors.json`` beside this file.
The parity tests load that JSON; nothing reads the reference tree at test time.

Usage: python tests/golden/extract_reference_vectors.py REFERENCE_ROOT

REFERENCE_ROOT is the top of a dada2-rs 0.2.0 source tree (the directory
holding src/nwalign.rs).
"""
from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _read(root, rel):
    with open(os.path.join(root, rel), encoding="utf-8") as f:
        return f.read().split("\n")


def _find(lines, pattern, start=0):
    rx = re.compile(pattern)
    for i in range(start, len(lines)):
        m = rx.search(lines[i])
        if m:
            return i, m
    raise LookupError(pattern)


def _rust_int(tok: str) -> int:
    tok = tok.strip().replace("_", "")
    for suf in ("u64", "usize", "i32", "i16", "u32"):
        if tok.endswith(suf):
            tok = tok[: -len(suf)]
    return int(tok, 0)


def _safe_eval(expr: str) -> int:
    if not re.fullmatch(r"[0-9\s\*\+\-\(\)]+", expr):
        raise ValueError(expr)
    return int(eval(expr, {"__builtins__": {}}, {}))  # arithmetic literal only


def extract(root: str) -> dict:
    nw = "src/nwalign.rs"
    L = _read(root, nw)
    out: dict = {"source": "HPCBio/dada2-rs 0.2.0 unit tests (read as text)"}

    # Ends-free known-answer scores (src/nwalign.rs:2345-2363).
    kats = []
    for name in ("test_align_endsfree_identical_short", "test_align_endsfree_one_sub",
                 "test_align_endsfree_one_gap"):
        i, _ = _find(L, rf"fn {name}\(")
        seqs = []
        j = i
        while len(seqs) < 2 and j < i + 8:
            m = re.search(r'encode\("([ACGT]+)"\)', L[j])
            if m:
                seqs.append(m.group(1))
            j += 1
        k, m = _find(L, r"check_endsfree_score\(&(\w+), &(\w+), ([^,]+), \"([^\"]+)\"\)", i)
        if len(seqs) == 1:
            seqs = [seqs[0], seqs[0]]
        kats.append({"s1": seqs[0], "s2": seqs[1], "expected": _safe_eval(m.group(3)),
                     "label": m.group(4), "band": 16, "where": f"{nw}:{k + 1}"})
    # Unbanded known answer: free leading gap, score 255 (src/nwalign.rs:2244-2254).
    i, _ = _find(L, r"fn wfa_endsfree_known_divergence\(")
    s = [re.search(r'encode\("([ACGT]+)"\)', L[j]).group(1) for j in range(i, i + 6)
         if re.search(r'encode\("([ACGT]+)"\)', L[j])]
    k, m = _find(L, r"sef, (\d+),", i)
    kats.append({"s1": s[0], "s2": s[1], "expected": int(m.group(1)), "label": "free-leading-gap",
                 "band": -1, "where": f"{nw}:{k + 1}"})
    out["endsfree_kats"] = kats

    # Vectorized-vs-ends-free score parity pairs (src/nwalign.rs:2989-3062).
    par = []
    for name in ("test_vectorized_vs_endsfree_identical", "test_vectorized_vs_endsfree_one_sub",
                 "test_vectorized_vs_endsfree_one_gap", "test_vectorized_vs_endsfree_different_lengths"):
        i, _ = _find(L, rf"fn {name}\(")
        seqs = []
        for j in range(i, i + 6):
            m = re.search(r'encode\("([ACGT]+)"\)', L[j])
            if m:
                seqs.append(m.group(1))
        if len(seqs) == 1:
            seqs = [seqs[0], seqs[0]]
        par.append({"s1": seqs[0], "s2": seqs[1], "where": f"{nw}:{i + 1}"})
    out["vec_parity_pairs"] = par
    lcg = []
    for name in ("test_vectorized_vs_endsfree_equal_length_240",
                 "test_vectorized_vs_endsfree_divergent_240",
                 "test_vectorized_vs_endsfree_different_lengths"):
        i, _ = _find(L, rf"fn {name}\(")
        k, m = _find(L, r"let mut state: u64 = (\d+);", i)
        lcg.append({"test": name, "seed": int(m.group(1)), "where": f"{nw}:{k + 1}"})
    out["vec_parity_lcg_seeds"] = lcg
    i, m = _find(L, r"\.wrapping_mul\((\d+)\)", _find(L, r"fn test_vectorized_vs_endsfree_equal_length_240")[0])
    out["lcg_mul"] = int(m.group(1))
    i, m = _find(L, r"\.wrapping_add\((\d+)\)", i)
    out["lcg_add"] = int(m.group(1))

    # Rolling-vs-full-matrix fuzz (src/nwalign.rs:2873-2952).
    i, _ = _find(L, r"fn rolling_d16_matches_full_matrix\(")
    k, m = _find(L, r"let mut state = (0x[0-9A-Fa-f_]+u64);", i)
    fuzz = {"seed": _rust_int(m.group(1)), "where": f"{nw}:{k + 1}"}
    j0, _ = _find(L, r"for &\(l1, l2\) in &\[", i)
    j1, _ = _find(L, r"\] \{", j0)
    body = " ".join(L[j0:j1 + 1])
    fuzz["length_pairs"] = [[int(a), int(b)] for a, b in re.findall(r"\((\d+)(?:usize)?, (\d+)(?:usize)?\)", body)]
    k, m = _find(L, r"for &band in &\[([^\]]+)\]", j1)
    fuzz["bands"] = [_rust_int(t) for t in m.group(1).split(",")]
    k, m = _find(L, r"for trial in 0\.\.(\d+)", k)
    fuzz["trials"] = int(m.group(1))
    k, m = _find(L, r"for &end_gap_p in &\[([^\]]+)\]", k)
    fuzz["end_gap_ps"] = [_rust_int(t) for t in m.group(1).split(",")]
    k, m = _find(L, r"assert!\(checked > (\d+)", k)
    fuzz["min_checked"] = int(m.group(1))
    out["rolling_fuzz"] = fuzz

    # Buffer reuse (src/nwalign.rs:2959-2987).
    i, _ = _find(L, r"fn rolling_d16_survives_buffer_reuse\(")
    k, m = _find(L, r"let mut state = (0x[0-9A-Fa-f_]+u64);", i)
    reuse = {"seed": _rust_int(m.group(1)), "where": f"{nw}:{k + 1}"}
    k, m = _find(L, r"for &len in &\[([^\]]+)\]", k)
    reuse["lens"] = [_rust_int(t) for t in m.group(1).split(",")]
    k, m = _find(L, r"step_by\((\d+)\)", k)
    reuse["step"] = int(m.group(1))
    out["buffer_reuse"] = reuse

    # Homopolymer dispatch pair (src/nwalign.rs:3124-3188).
    i, _ = _find(L, r"fn homo_gap_penalty_routes_to_homopolymer_aligner\(")
    seqs = []
    for j in range(i, i + 12):
        m = re.search(r'encode\("([ACGT]+)"\)', L[j])
        if m:
            seqs.append(m.group(1))
    k, m = _find(L, r"homo_gap_p: (-?\d+),", i)
    out["homo_dispatch"] = {"s1": seqs[0], "s2": seqs[1], "homo_gap_p": int(m.group(1)),
                            "where": f"{nw}:{i + 1}"}

    # Compare-level pool (src/cluster.rs:1786-1922).
    cl = "src/cluster.rs"
    L = _read(root, cl)
    i, m = _find(L, r'let base = b"([ACGT]+)";')
    pool = {"base": m.group(1), "where": f"{cl}:{i + 1}"}
    j0, _ = _find(L, r"for \(n, reads\) in \[", i)
    j1, _ = _find(L, r"\] \{", j0)
    body = " ".join(L[j0:j1 + 1])
    pool["n_reads"] = [[int(a), int(b)] for a, b in re.findall(r"\((\d+)(?:usize)?, (\d+)(?:u32)?\)", body)]
    k, m = _find(L, r"let idx = \(p \* (\d+) \+ (\d+)\) % seq\.len\(\);", j1)
    pool["mut_mul"], pool["mut_add"] = int(m.group(1)), int(m.group(2))
    k, m = _find(L, r"const K: usize = (\d+);")
    pool["k"] = int(m.group(1))
    k, m = _find(L, r"homo_gap_p: (-?\d+),", j1)
    pool["homo_gap_p"] = int(m.group(1))
    k, m = _find(L, r"kdist_cutoff: ([0-9.]+),", j1)
    pool["kdist_cutoff"] = float(m.group(1))
    k, m = _find(L, r"band: (\d+),", j1)
    pool["band"] = int(m.group(1))
    k, m = _find(L, r"b\.clusters\[0\]\.center = Some\((\d+)\);", j1)
    pool["center"] = int(m.group(1))
    k, m = _find(L, r"let err = vec!\[([0-9.]+)f64; 16 \* (\d+)\];", k)
    pool["err_flat"], pool["ncol"] = float(m.group(1)), int(m.group(2))
    out["compare_pool"] = pool

    # Tie rules (src/cluster.rs:1735-1777).
    i, _ = _find(L, r"fn exact_ties_resolve_to_lowest_ci\(")
    ties = []
    for j in range(i, i + 12):
        m = re.search(r"assert_eq!\(fold_beats\(&\[(.+)\]\), (\d+)\);", L[j])
        if m:
            cands = [[float(a), int(b)] for a, b in re.findall(r"\(([0-9.]+), (\d+)\)", m.group(1))]
            ties.append({"cands": cands, "winner": int(m.group(2)), "where": f"{cl}:{j + 1}"})
    out["tie_cases"] = ties

    # K-mer sparse/dense tests (src/kmers.rs:330-401).
    km = "src/kmers.rs"
    L = _read(root, km)
    i, _ = _find(L, r"fn make_seq\(")
    k, m = _find(L, r"\.wrapping_mul\((\d+)\)", i)
    kt = {"mul": int(m.group(1))}
    k, m = _find(L, r"\.wrapping_add\((\d+)\)", k)
    kt["add"] = int(m.group(1))
    k, m = _find(L, r"for &k in &\[([^\]]+)\]", k)
    kt["ks"] = [_rust_int(t) for t in m.group(1).split(",")]
    k, m = _find(L, r"for seed in 0\.\.(\d+)", k)
    kt["reconstruct_seeds"] = int(m.group(1))
    k, m = _find(L, r"make_seq\((\d+), seed\)", k)
    kt["reconstruct_len"] = int(m.group(1))
    k, m = _find(L, r"for seed in 0\.\.(\d+)", k)
    kt["dist_seeds"] = int(m.group(1))
    k, m = _find(L, r"make_seq\((\d+), seed\)", k)
    kt["dist_len"] = int(m.group(1))
    k, m = _find(L, r"make_seq\(\d+, seed \+ (\d+)\)", k)
    kt["dist_seed_offset"] = int(m.group(1))
    k, m = _find(L, r"let k = (\d+);", k)
    kt["overflow_k"] = int(m.group(1))
    k, m = _find(L, r"vec!\[(\d+)u8; (\d+)\]", k)
    kt["overflow_nt"], kt["overflow_len"] = int(m.group(1)), int(m.group(2))
    kt["where"] = f"{km}:{i + 1}"
    out["kmer_tests"] = kt
    return out


def main():
    if len(sys.argv) != 2:
        raise SystemExit("usage: extract_reference_vectors.py REFERENCE_ROOT")
    root = sys.argv[1]
    data = extract(root)
    path = os.path.join(HERE, "reference_vectors.json")
    with open(path, "w", encoding="utf-8") as f:
        json.dump(data, f, indent=1, sort_keys=True)
        f.write("\n")
    print(f"wrote {path}")


if __name__ == "__main__":
    main()
