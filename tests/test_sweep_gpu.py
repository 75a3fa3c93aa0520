"""Random-configuration sweep of the CUDA path against the oracle.

Each case draws a read length (1-511), single or paired end, preserved order
or not, an error and an N rate, and a block size, from a fixed list of
seeds; the block goes through the CUDA path (`curc_block_run`) and the
oracle, and every stage result and stream must be equal.  A mismatching case
is reported with the parameters that rebuild it."""
import random

import numpy as np
import pytest

from curc_b200 import synth
from tests.oracle_lib import OracleBlock, STAGE_RESULTS, stream_dtype, stream_names

pytestmark = pytest.mark.gpu

SEEDS = [1, 2, 3, 4, 5, 6]
CASES_PER_SEED = 24
MAX_READS = 1500


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


@pytest.fixture(scope="module")
def ctx():
    from curc_b200 import Context
    with Context(0) as c:
        yield c


@pytest.mark.parametrize("seed", SEEDS)
def test_random_configurations(ctx, seed):
    rnd = random.Random(seed)
    bad_cases = []
    # seeds 4-6 run the full-match loop as one persistent kernel, the
    # others in the library's default form
    default = ctx.tuning()
    ctx.set_tuning(**dict(default, fm_loop=2 if seed > 3 else default["fm_loop"]))
    for i in range(CASES_PER_SEED):
        w, params = draw(rnd, MAX_READS)
        seqs = w.sequences()
        pe = w.mate2 is not None
        ora = OracleBlock(seqs, w.preserve_order, pe)
        ctx.block_run(seqs, w.preserve_order, pe)
        names = list(STAGE_RESULTS.items()) + [(s, stream_dtype(s)) for s in stream_names(seqs.shape[1])]
        bad = [nm for nm, dt in names
               if not np.array_equal(ctx.get(nm, dt), ora.get(nm, dt))]
        if bad:
            bad_cases.append(f"case {i} {params}: {bad}")
    ctx.set_tuning(**default)
    assert not bad_cases, "\n".join(bad_cases)
