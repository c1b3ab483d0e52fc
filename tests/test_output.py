"""The `dada` JSON writer (DadaOutput, src/main.rs:1139-1257): field order,
serde_json's number formatting, nulls in the map. Host only."""
import json

import numpy as np

import dada2_b200 as D
from dada2_b200 import output


def _result():
    clusters = [
        {"sequence": np.array([1, 2, 3, 4, 5], np.uint8), "reads": 90, "birth_type": 0, "birth_pval": 0.0,
         "birth_fold": 1.0, "birth_e": 96.0},
        {"sequence": np.array([4, 3, 2, 1], np.uint8), "reads": 6, "birth_type": 1, "birth_pval": 1.5e-300,
         "birth_fold": 2.5e+20, "birth_e": float("inf")},
    ]
    return {"clusters": clusters, "counters": {"nalign": 7, "nshroud": 3},
            "map": np.array([0, 1, -1, 0], np.int32)}


def test_dada_json_layout_and_numbers():
    p = D.DadaParams()
    text = output.dada_json(_result(), p, "/data/run1/sampleA.fastq.gz", compact=True)
    doc = json.loads(text)
    assert list(doc) == ["dada2_rs_command", "dada2_rs_version", "sample", "input_file", "num_asvs",
                         "total_reads", "asvs", "stats", "params", "map"]
    assert doc["dada2_rs_command"] == "dada" and doc["sample"] == "sampleA"
    assert doc["input_file"] == "sampleA.fastq.gz"
    assert doc["num_asvs"] == 2 and doc["total_reads"] == 96
    assert doc["asvs"][0]["sequence"] == "ACGTN" and doc["asvs"][1]["birth_type"] == "Abundance"
    assert list(doc["asvs"][0]) == ["sequence", "abundance", "birth_type", "birth_pval", "birth_fold", "birth_e"]
    assert doc["map"] == [0, 1, None, 0]
    assert list(doc["params"])[:3] == ["omega_a", "omega_c", "omega_p"]
    assert list(doc["params"])[-2:] == ["pool", "n_prior"]
    # serde_json: shortest round trip, no '+' in exponents, non-finite as null
    assert '"birth_pval":1.5e-300' in text and '"birth_fold":2.5e20' in text and '"birth_e":null' in text
    assert '"omega_a":1e-40' in text and '"birth_pval":0.0' in text and '"kdist_cutoff":0.42' in text


def test_dada_json_pretty_matches_compact():
    p = D.DadaParams()
    pretty = output.dada_json(_result(), p, "x.fq", sample="S1")
    assert pretty.startswith('{\n  "dada2_rs_command": "dada",\n')
    assert json.loads(pretty) == json.loads(output.dada_json(_result(), p, "x.fq", sample="S1", compact=True))
    assert json.loads(pretty)["sample"] == "S1"
