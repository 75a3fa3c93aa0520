"""Random-configuration sweep of the CUDA path against the oracle (needs a GPU).

Not collected by pytest: a longer search than the fixed parity cases, run by
hand.  Each case draws a read length (1-511), single or paired end, preserved
order or not, an error and an N rate, and a block size; the block goes through
the CUDA path (`curc_block_run`) and the oracle, and every stage result and
stream must be equal.  A mismatching case is printed with the parameters that
rebuild it.

    python tests/sweep_gpu.py [--seed S] [--cases N] [--max-reads R]
"""
import argparse
import os
import random
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from curc_b200 import Context, synth  # noqa: E402
from tests.oracle_lib import OracleBlock, STAGE_RESULTS, stream_dtype, stream_names  # noqa: E402


def draw(rnd, max_reads):
    L = rnd.choice([rnd.randint(1, 40), rnd.randint(41, 160), rnd.randint(161, 511)])
    pe, po = rnd.random() < 0.5, rnd.random() < 0.5
    n = rnd.randint(1, max_reads)
    kw = dict(err=rnd.choice([0.0, 0.001, 0.01]), n_rate=rnd.choice([0.0, 0.0001, 0.003, 0.02]))
    seed = rnd.randint(0, 10**6)
    if pe:
        w = synth.paired_repeats(seed=seed, pairs=max(1, n // 2), read_len=L,
                                 genome_len=rnd.randint(3 * L + 20_000, 200_000), preserve_order=po, **kw)
    else:
        w = synth.small_single(seed=seed, n_reads=n, read_len=L, genome_len=rnd.randint(2 * L + 1000, 200_000), **kw)
        w.preserve_order = po
    return w, dict(L=L, pe=pe, po=po, n=n, seed=seed, **kw)


def compare(ctx, w):
    seqs = w.sequences()
    pe = w.mate2 is not None
    ora = OracleBlock(seqs, w.preserve_order, pe)
    ctx.block_run(seqs, w.preserve_order, pe)
    bad = []
    names = list(STAGE_RESULTS.items()) + [(s, stream_dtype(s)) for s in stream_names(seqs.shape[1])]
    for name, dt in names:
        a, b = ctx.get(name, dt), ora.get(name, dt)
        if a.shape != b.shape or not np.array_equal(a, b):
            bad.append(name)
    return bad


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--cases", type=int, default=200)
    ap.add_argument("--max-reads", type=int, default=4000)
    a = ap.parse_args()
    rnd = random.Random(a.seed)
    failures = 0
    with Context(0) as ctx:
        for i in range(a.cases):
            w, params = draw(rnd, a.max_reads)
            bad = compare(ctx, w)
            if bad:
                failures += 1
                print(f"case {i}: {params} differs in {bad}", flush=True)
    print(f"{a.cases} cases, {failures} differing")
    return 1 if failures else 0


if __name__ == "__main__":
    sys.exit(main())
