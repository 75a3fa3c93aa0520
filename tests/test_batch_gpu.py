"""The batched path (curc_batch_submit / curc_batch_drain): blocks of
different read lengths and sizes queued on one context and run by one or
several concurrent block pipelines give, block by block, exactly the
streams of one-at-a-time curc_block_run calls."""
import numpy as np
import pytest

from curc_b200 import synth
from tests.cases import CASES
from tests.oracle_lib import stream_dtype, stream_names

pytestmark = pytest.mark.gpu


def _blocks():
    out = []
    for w in synth.batched_blocks(seed=5, count=5, scale=0.02):
        out.append((np.ascontiguousarray(w.mate1), False, False))
    for name in ("pe150_po", "se150_hiN"):
        out.append(CASES[name]())
    return out


def _streams(ctx, L):
    return {n: ctx.get(n, stream_dtype(n)).copy() for n in stream_names(L)}


@pytest.mark.parametrize("workers", [1, 3])
def test_batch_equals_single_blocks(workers):
    from curc_b200 import Context
    blocks = _blocks()
    with Context(0) as ctx:
        ctx.keep_intermediates(False)
        ctx.batch_workers(workers)
        single = []
        for seqs, po, pe in blocks:
            ctx.block_run(seqs, po, pe)
            single.append(_streams(ctx, seqs.shape[1]))
        got = {}
        tickets = [ctx.batch_submit(seqs, po, pe) for seqs, po, pe in blocks]
        ctx.batch_drain(lambda t: got.__setitem__(t, _streams(ctx, blocks[tickets.index(t)][0].shape[1])))
        assert sorted(got) == tickets
        for t, ref in zip(tickets, single):
            for name, a in ref.items():
                b = got[t][name]
                assert a.shape == b.shape and np.array_equal(a, b), f"block {t} stream {name}"
        # a second drain on the same context (slots reused)
        got2 = {}
        t2 = [ctx.batch_submit(seqs, po, pe) for seqs, po, pe in blocks[:2]]
        ctx.batch_drain(lambda t: got2.__setitem__(t, _streams(ctx, blocks[t2.index(t)][0].shape[1])))
        for t, ref in zip(t2, single[:2]):
            for name, a in ref.items():
                assert np.array_equal(a, got2[t][name]), f"second drain block {t} stream {name}"
