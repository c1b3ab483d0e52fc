"""The `dada` subcommand's JSON output (DadaOutput, src/main.rs:1139-1257).

``dada_json(result, ...)`` writes a denoising result in the reference's
layout: the command tag and version first (Tagged, src/misc.rs:122-137), then
sample, input_file, num_asvs, total_reads, the ASVs (AsvEntry,
src/main.rs:4776-4817), stats (nalign, nshroud), the run parameters
(DadaRunParams, src/main.rs:142-172, filled as src/main.rs:4522-4545) and the
map (null for raws left out of every cluster). Field order is the structs'
declaration order, as serde writes it; floats are printed shortest
round-trip with no '+' in the exponent and non-finite values as null, as
serde_json does. The optional `aux` block (cluster_stats, cluster_quality,
birth_subs) is not produced.
"""
from __future__ import annotations

import math
import os

import numpy as np

VERSION = "0.2.0"
BIRTH_TYPES = {0: "Initial", 1: "Abundance", 2: "Prior", 3: "Singleton"}
NT_DECODE = {1: "A", 2: "C", 3: "G", 4: "T", 5: "N", 45: "-"}


def _num(x) -> str:
    if isinstance(x, (bool, np.bool_)):
        return "true" if x else "false"
    if isinstance(x, (int, np.integer)):
        return str(int(x))
    x = float(x)
    if not math.isfinite(x):
        return "null"
    r = repr(x)
    if "e" in r:
        mant, exp = r.split("e")
        r = mant + "e" + str(int(exp))
    return r


def _dump(v, indent, level) -> str:
    if v is None:
        return "null"
    if isinstance(v, str):
        return '"' + v.replace("\\", "\\\\").replace('"', '\\"') + '"'
    if isinstance(v, (bool, np.bool_, int, float, np.integer, np.floating)):
        return _num(v)
    nl = "" if indent is None else "\n"
    pad = "" if indent is None else " " * (indent * (level + 1))
    end = "" if indent is None else " " * (indent * level)
    sep = ":" if indent is None else ": "
    if isinstance(v, dict):
        if not v:
            return "{}"
        items = [pad + _dump(k, indent, level + 1) + sep + _dump(x, indent, level + 1) for k, x in v.items()]
        return "{" + nl + ("," + nl).join(items) + nl + end + "}"
    items = list(v)
    if not items:
        return "[]"
    return "[" + nl + ("," + nl).join(pad + _dump(x, indent, level + 1) for x in items) + nl + end + "]"


def fastq_stem(path) -> str:
    """The sample name from a FASTQ path (src/main.rs:5175-5186)."""
    name = os.path.basename(str(path)) or "unknown"
    for suffix in (".fastq.gz", ".fq.gz", ".fastq", ".fq"):
        if name.endswith(suffix):
            return name[: -len(suffix)]
    return name


def dada_json(result: dict, params, input_file, sample: str | None = None, n_prior: int = 0,
              compact: bool = False) -> str:
    """``result`` as returned by ``dada_uniques`` / ``dada_fastq``; ``params``
    the DadaParams it ran with."""
    clusters = list(result["clusters"])
    asvs = [{"sequence": "".join(NT_DECODE.get(int(b), "?") for b in c["sequence"]),
             "abundance": int(c["reads"]), "birth_type": BIRTH_TYPES.get(c["birth_type"], "Initial"),
             "birth_pval": float(c["birth_pval"]), "birth_fold": float(c["birth_fold"]),
             "birth_e": float(c["birth_e"])} for c in clusters]
    a = params.align
    run = {"omega_a": float(params.omega_a), "omega_c": float(params.omega_c), "omega_p": float(params.omega_p),
           "min_fold": float(params.min_fold), "min_hamming": int(params.min_hamming),
           "min_abund": int(params.min_abund), "detect_singletons": bool(params.detect_singletons),
           "band": int(a.band), "homo_gap_p": int(a.homo_gap_p), "gap_p": int(a.gap_p),
           "match_score": int(a.match_score), "mismatch": int(a.mismatch), "max_clust": int(params.max_clust),
           "greedy": bool(params.greedy), "use_quals": bool(params.use_quals), "kdist_cutoff": float(a.kdist_cutoff),
           "kmer_size": int(a.kmer_size), "use_kmers": bool(a.use_kmers), "pool": False, "n_prior": int(n_prior)}
    out = {"dada2_rs_command": "dada", "dada2_rs_version": VERSION,
           "sample": sample if sample is not None else fastq_stem(input_file),
           "input_file": os.path.basename(str(input_file)) or "unknown",
           "num_asvs": len(asvs), "total_reads": int(sum(c["reads"] for c in clusters)), "asvs": asvs,
           "stats": {"nalign": int(result["counters"]["nalign"]), "nshroud": int(result["counters"]["nshroud"])},
           "params": run, "map": [None if int(m) < 0 else int(m) for m in result["map"]]}
    return _dump(out, None if compact else 2, 0)
