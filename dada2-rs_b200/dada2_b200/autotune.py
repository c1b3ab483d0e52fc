"""Autotuner of the compare step's launch shape, per read-length class.

The reference schedules its compare map on rayon with one knob, the grain
DADA2_RS_PAR_GRAIN (src/cluster.rs:19-28). Here the launch shape has eight
knobs (include/dada2_b200.h, dgpu_tuning): concurrent launch slots, samples
per launch, slots dedicated to the longest chains, resident alignment CTAs
per SM (pairs in flight), the screen's largest chunk and its blocks per SM,
the launch size from which the screen's pivot bound runs, and whether the
alignment and store kernels launch as programmatic dependents.
Their best values depend on read length: short reads give many cheap
compare calls, long reads few expensive alignments.

For each class (150, 250/220 and 1,450 nt) the tuner denoises a seeded
production-sized synthetic workload of that class with inputs resident on the device
(ResidentBatch) and descends one knob at a time: every value of a knob is
timed with the others fixed, and a value is kept only when it is at least
2 % faster than the best so far; two passes over the knobs. Each timing is
the best of ``reps`` runs. Results never depend on the setting, so the tuner
only measures time. The chosen table is written to ``tuning.txt`` beside
the library, which loads it at first use.

Usage: python -m dada2_b200.autotune [--device N] [--classes 0,1,2] [--out PATH]
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import DadaParams, AlignParams, ResidentBatch, PackedBatch, TUNING_KEYS, tuning_get, tuning_set, tuning_save
from . import _lib, synth

# candidate values of each knob, in the order the descent visits them
SPACE = {
    "launch_slots": [2, 3, 4, 6, 8],
    "samples_per_launch": [1, 2, 4, 8],
    "dedicated_slots": [0, 1, 2],
    "align_ctas_per_sm": [2, 3, 4],
    "screen_chunk_max": [16, 32],
    "screen_blocks_per_sm": [2, 3, 4],
    "pivot_min_items": [0, 8192, 32768, 131072],
    "programmatic_launch": [0, 1],
}

# representative read length of each class
CLASS_LENGTH = {0: 150, 1: 250, 2: 1450}


def class_workload(cls: int, seed: int = 4242):
    """A seeded synthetic workload of read-length class ``cls``, sized like
    production batches: for 250/220 nt the 40-sample shape (uniques
    log-uniform in [500, 30,000], 50-400 variants, alternating lengths), for
    150 nt 24 such samples of up to 15,000 uniques, for long reads eight
    PacBio-style 16S samples of 800 uniques at 1,400-1,550 nt (band 32,
    homopolymer gap -1), enough samples that the slot knobs matter. The seeds differ from the benchmark's."""
    rng = np.random.default_rng(seed + cls)
    if cls == 2:
        errm = synth.error_matrix(94, floor=1e-3)
        samples = [synth.pacbio_sample(rng, 30, 800, 1400, 1550, errm, 94) for _ in range(8)]
        return synth.Workload(2, "tuning: PacBio-style 16S x8", samples, errm, 94, band=32, homo_gap_p=-1)
    if cls == 1:
        w = synth.config1(seed=seed + 1)
        w.name = "tuning: 40 Illumina-style samples at 250/220 nt"
        return w
    errm = synth.error_matrix(41)
    samples = []
    for si in range(24):
        target = int(np.exp(rng.uniform(np.log(500), np.log(15000))))
        nvar = int(rng.integers(50, 401))
        nreads = max(int((target - nvar) / 0.076), 2 * nvar)
        samples.append(synth.illumina_sample(rng, nvar, nreads, 150, errm, 41))
    return synth.Workload(0, "tuning: 24 Illumina-style samples at 150 nt", samples, errm, 41)


def time_setting(w, params, packed, device: int, reps: int) -> float:
    """Seconds of the fastest of ``reps`` resident denoisings of the workload
    (the pool is created after the setting, so it takes effect)."""
    best = float("inf")
    with ResidentBatch(w.samples, w.err, w.ncol, params, device=device, packed=packed) as rb:
        rb.run(read_results=False)  # warm-up
        for _ in range(reps):
            t0 = time.perf_counter()
            rb.run(read_results=False)
            best = min(best, time.perf_counter() - t0)
    return best


def tune_class(cls: int, device: int = 0, reps: int = 3, passes: int = 2, log=print) -> dict:
    w = class_workload(cls)
    params = DadaParams(align=AlignParams(band=w.band, homo_gap_p=w.homo_gap_p))
    packed = PackedBatch(w.samples)
    cur = tuning_get(CLASS_LENGTH[cls])
    best_t = time_setting(w, params, packed, device, reps)
    start_t = best_t
    trials = 1
    log(f"class {cls}: start {cur} {1e3 * best_t:.1f} ms")
    for _ in range(passes):
        changed = False
        for knob, values in SPACE.items():
            for v in values:
                if v == cur[knob]:
                    continue
                cand = {**cur, knob: v}
                tuning_set(cls, cand)
                t = time_setting(w, params, packed, device, reps)
                trials += 1
                if t < 0.98 * best_t:
                    cur, best_t, changed = cand, t, True
                    log(f"class {cls}: {knob}={v} -> {1e3 * t:.1f} ms")
            tuning_set(cls, cur)
        if not changed:
            break
    tuning_set(cls, cur)
    return {"setting": cur, "ms": 1e3 * best_t, "ms_built_in": 1e3 * start_t, "trials": trials,
            "workload": w.name, "uniques": int(sum(len(s.seqs) for s in w.samples))}


def autotune(device: int = 0, classes=(0, 1, 2), out: str | None = None, reps: int = 3, log=print) -> dict:
    """Tunes each class in turn and saves the table (default: tuning.txt beside
    the library). Returns the per-class report."""
    report = {}
    for cls in classes:
        report[str(cls)] = tune_class(cls, device=device, reps=reps, log=log)
    path = out or os.path.join(os.path.dirname(_lib.LIB_PATH), "tuning.txt")
    tuning_save(path)
    report["path"] = path
    return report


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--classes", default="0,1,2")
    ap.add_argument("--out", default=None)
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    classes = [int(c) for c in a.classes.split(",") if c.strip()]
    rep = autotune(a.device, classes, a.out, a.reps)
    print(json.dumps(rep))


if __name__ == "__main__":
    main()
