"""The autotuner's knobs change no result, on a B200.

Every knob value (overlap bucket table factor, presence-bitmap bits,
passes between link-count reads, mapping threads per block, full-match
pass loop as a launch per kernel, one graph or one persistent kernel) runs
the same blocks; every stage result and stream must equal the default setting's, and
the default setting's must equal the oracle's.  Then curc_autotune picks a
setting on a block, caches it per (read length, read-count bucket), and a
second call takes it from the cache."""
import numpy as np
import pytest

from tests.cases import CASES
from tests.oracle_lib import OracleBlock, STAGE_RESULTS, stream_dtype, stream_names

pytestmark = pytest.mark.gpu

KNOB_VALUES = {"table_factor": [1, 2, 8], "bitmap_bits": [8, 32], "check_every": [2, 16], "map_threads": [64, 256],
               "fm_loop": [0, 1, 2]}


def _results(ctx, L):
    names = list(STAGE_RESULTS.items()) + [(s, stream_dtype(s)) for s in stream_names(L)]
    return {n: ctx.get(n, dt) for n, dt in names}


@pytest.mark.parametrize("case", ["se100_deep", "pe150_po", "se75_20k"])
def test_every_knob_value_gives_the_same_streams(case):
    from curc_b200 import Context
    seqs, po, pe = CASES[case]()
    L = seqs.shape[1]
    with Context(0) as ctx:
        default = ctx.tuning()
        ctx.block_run(seqs, po, pe)
        base = _results(ctx, L)
        ora = OracleBlock(seqs, po, pe)
        for n, dt in list(STAGE_RESULTS.items())[:3]:
            assert np.array_equal(base[n], ora.get(n, dt)), n
        bad = []
        for knob, values in KNOB_VALUES.items():
            for v in values:
                ctx.set_tuning(**dict(default, **{knob: v}))
                ctx.block_run(seqs, po, pe)
                got = _results(ctx, L)
                diff = [n for n in base if not np.array_equal(base[n], got[n])]
                if diff:
                    bad.append(f"{knob}={v}: {diff}")
        ctx.set_tuning(**default)
    assert not bad, "\n".join(bad)


def test_autotune_caches_per_bucket(tmp_path):
    import torch
    from curc_b200 import Context
    seqs, po, pe = CASES["pe150_po_100k"]()
    n, L = seqs.shape
    d = torch.from_numpy(seqs.reshape(-1).copy()).cuda()
    cache = str(tmp_path / "tune.txt")
    with Context(0) as ctx:
        ctx.block_run(seqs, po, pe)
        base = _results(ctx, L)
        t1, hit1 = ctx.autotune(d.data_ptr(), n, L, po, pe, cache)
        t2, hit2 = ctx.autotune(d.data_ptr(), n, L, po, pe, cache)
        ctx.block_run(seqs, po, pe)
        got = _results(ctx, L)
    assert not hit1 and hit2 and t1 == t2
    line = open(cache).read().split()
    assert [int(x) for x in line[:2]] == [L, int(np.log2(n))]
    assert all(np.array_equal(base[k], got[k]) for k in base)
