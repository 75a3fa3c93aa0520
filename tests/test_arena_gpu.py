"""Device memory of a block pipeline stays bounded across blocks of changing
sizes, on a B200.

A pipeline's arena keeps its chunks between blocks.  A block larger than
the last one used to add a chunk even when a free chunk later in the list
was large enough, so blocks of alternating sizes (the batched workload, the
autotuner's reruns) grew device memory until allocation failed.  Here blocks
of alternating sizes run many times; after two rounds of sizes the free
device memory must not keep shrinking, and every run's streams equal
the first run of the same block."""
import numpy as np
import pytest

from tests.oracle_lib import stream_dtype, stream_names

pytestmark = pytest.mark.gpu


def _reads(n, L, seed):
    rng = np.random.default_rng(seed)
    genome = np.frombuffer(b"ACGT", dtype=np.uint8)[rng.integers(0, 4, size=max(4 * L, n * 2))]
    starts = rng.integers(0, genome.size - L, size=n)
    return np.ascontiguousarray(genome[starts[:, None] + np.arange(L)[None, :]])


def _digest(ctx, L):
    import hashlib
    h = hashlib.sha256()
    for nm in stream_names(L):
        h.update(ctx.get(nm, stream_dtype(nm)).tobytes())
    return h.hexdigest()


def test_alternating_block_sizes_do_not_grow_device_memory():
    import torch
    from curc_b200 import Context
    blocks = [_reads(n, L, s) for s, (n, L) in enumerate([(20_000, 100), (400_000, 150), (60_000, 250),
                                                           (800_000, 100), (10_000, 75)])]
    with Context(0) as ctx:
        ctx.keep_intermediates(False)
        first = []
        for b in blocks:
            ctx.block_run(b)
            first.append(_digest(ctx, b.shape[1]))
        for b in blocks:  # one more round to settle the chunk order
            ctx.block_run(b)
        torch.cuda.synchronize()
        free_after_first = torch.cuda.mem_get_info(0)[0]
        for _ in range(4):
            for i, b in enumerate(blocks):
                ctx.block_run(b)
                assert _digest(ctx, b.shape[1]) == first[i]
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info(0)[0]
    # no new chunks once every size has been seen (a little slack for
    # allocations outside the arena)
    assert free_after_first - free_after < (256 << 20), (free_after_first, free_after)


def test_trim_frees_device_memory_and_keeps_results():
    import torch
    from curc_b200 import Context
    b = _reads(400_000, 150, 7)
    with Context(0) as ctx:
        ctx.keep_intermediates(False)
        ctx.block_run(b)
        d0 = _digest(ctx, 150)
        torch.cuda.synchronize()
        before = torch.cuda.mem_get_info(0)[0]
        ctx.trim()
        after = torch.cuda.mem_get_info(0)[0]
        assert _digest(ctx, 150) == d0  # the last run's results stay readable
        assert after > before
        ctx.block_run(b)
        assert _digest(ctx, 150) == d0


def test_autotune_runs_do_not_accumulate_device_memory():
    """curc_autotune runs the block about thirty times: each run starts from
    an empty arena, so device memory after it is what one run needs."""
    import torch
    from curc_b200 import Context
    b = _reads(300_000, 150, 9)
    d = torch.from_numpy(b.reshape(-1).copy()).cuda()
    with Context(0) as ctx:
        ctx.keep_intermediates(False)
        ctx.block_run_device(d.data_ptr(), b.shape[0], b.shape[1], False, False)
        torch.cuda.synchronize()
        before = torch.cuda.mem_get_info(0)[0]
        ctx.autotune(d.data_ptr(), b.shape[0], b.shape[1], False, False)
        torch.cuda.synchronize()
        after = torch.cuda.mem_get_info(0)[0]
    assert before - after < (1 << 30), (before, after)
