"""SHA-256 digests of every stage result and stream the oracle computes on
full-size blocks, for the GPU tests that check the CUDA path at sizes the
oracle takes minutes for (tests/test_fullsize_gpu.py).  CPU only; about half
an hour on 8 cores.

Cases: the paired-end 150 bp benchmark block (10M pairs from a 50 Mbp genome
with 5% repeats, preserved order), and full-scale blocks of the batched
workload (64 single-end blocks from different genomes) chosen to cover each
read length in {75, 100, 150, 250} from low to very deep coverage.

    python tests/golden/make_fullsize_digests.py [--cases a,b]
"""
import argparse
import hashlib
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from curc_b200 import synth  # noqa: E402
from tests.oracle_lib import STAGE_RESULTS, OracleBlock, stream_dtype, stream_names  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "fullsize_digests.json")
BATCH_SEED = 2
# batched-workload blocks: (block, reads, read length, coverage) at scale 1.0
BATCH_BLOCKS = [1, 41, 14, 39, 5, 55]


def cases():
    c = {"pe150_10M_pairs": lambda: synth.paired_repeats(seed=1, pairs=10_000_000, read_len=150,
                                                         genome_len=50_000_000, preserve_order=True)}
    specs = synth.batched_specs(BATCH_SEED, 64, 1.0)
    for b in BATCH_BLOCKS:
        c[f"batch{b}"] = (lambda b=b: synth.batched_block(BATCH_SEED, b, specs[b]))
    return c


def digests(get, read_len):
    """name -> sha256 of the result's bytes, for every stage result and stream."""
    out = {}
    for name, dt in STAGE_RESULTS.items():
        out[name] = hashlib.sha256(get(name, dt).tobytes()).hexdigest()
    for name in stream_names(read_len):
        out[name] = hashlib.sha256(get(name, stream_dtype(name)).tobytes()).hexdigest()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", default=",".join(cases()))
    a = ap.parse_args()
    out = json.load(open(OUT)) if os.path.exists(OUT) else {}
    all_cases = cases()
    for name in a.cases.split(","):
        w = all_cases[name]()
        seqs = w.sequences()
        t = time.time()
        o = OracleBlock(seqs, w.preserve_order, w.mate2 is not None, threads=os.cpu_count() or 8)
        dt = time.time() - t
        out[name] = {"workload": w.name, "reads": int(seqs.shape[0]), "read_len": w.read_len,
                     "preserve_order": w.preserve_order, "paired_end": w.mate2 is not None,
                     "oracle_seconds": round(dt, 1), "sha256": digests(o.get, w.read_len)}
        del o
        print(name, seqs.shape, f"{dt:.0f} s", flush=True)
        json.dump(out, open(OUT, "w"), indent=1)


if __name__ == "__main__":
    main()
