"""Runs the unmodified reference `curc -c` (oracle/_ref/curc_shared, built
from the reference sources by oracle/ref.mk) on seeded synthetic inputs and
stores its archives as golden fixtures.  Needs a GPU.  The zero-filling
cudaMalloc shim oracle/_ref/libzero_alloc.so is preloaded (see
oracle/ref_zero_alloc.c for why).  Each case runs `--repeat` times to record
whether the reference is deterministic.

    python tests/golden/make_golden.py OUTDIR [--repeat 3]
"""
import argparse
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from curc_b200 import synth  # noqa: E402

REF_DIR = os.path.join(ROOT, "oracle", "_ref")

CASES = {
    # the 100k x 100 bp single-end case of the benchmark configs
    "c0_se100_n100k": lambda: synth.small_single(seed=0, n_reads=100_000, read_len=100, genome_len=1_000_000),
    "se75_n20k": lambda: synth.small_single(seed=21, n_reads=20_000, read_len=75, genome_len=150_000, err=0.003),
    "se250_n8k": lambda: synth.small_single(seed=22, n_reads=8_000, read_len=250, genome_len=300_000, err=0.002),
    "pe150_po_p8k": lambda: synth.paired_repeats(seed=23, pairs=8_000, genome_len=400_000, preserve_order=True),
    "pe150_p8k": lambda: synth.paired_repeats(seed=24, pairs=8_000, genome_len=400_000, preserve_order=False),
}


def run_ref(files, po, wd, name):
    env = dict(os.environ)
    env["LD_PRELOAD"] = os.path.join(REF_DIR, "libzero_alloc.so")
    cmd = [os.path.join(REF_DIR, "curc_shared"), "-c", "-i", ",".join(files), "-o", name, "--working_dir", wd]
    if po:
        cmd.append("--preserve_order")
    t = time.time()
    r = subprocess.run(cmd, cwd=REF_DIR, env=env, capture_output=True, text=True, timeout=600)
    dt = time.time() - t
    if r.returncode != 0:
        raise RuntimeError(f"reference failed ({r.returncode}): {r.stdout[-2000:]} {r.stderr[-2000:]}")
    return os.path.join(wd, name + ".curc"), dt, r.stdout


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("outdir")
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--cases", default=",".join(CASES))
    a = ap.parse_args()
    os.makedirs(a.outdir, exist_ok=True)
    meta = {}
    for name in a.cases.split(","):
        w = CASES[name]()
        with tempfile.TemporaryDirectory() as td:
            files = w.write(os.path.join(td, name))
            digests, times = [], []
            for rep in range(a.repeat):
                path, dt, out = run_ref(files, w.preserve_order, td, f"{name}_{rep}")
                data = open(path, "rb").read()
                digests.append(hashlib.sha256(data).hexdigest())
                times.append(dt)
                if rep == 0:
                    shutil.copy(path, os.path.join(a.outdir, name + ".curc"))
            meta[name] = {"sha256": digests, "seconds": times, "bases": w.bases,
                          "deterministic": len(set(digests)) == 1, "stdout_tail": out[-400:]}
            print(name, meta[name]["deterministic"], [d[:12] for d in digests], times, flush=True)
    json.dump(meta, open(os.path.join(a.outdir, "golden_meta.json"), "w"), indent=1)


if __name__ == "__main__":
    main()
