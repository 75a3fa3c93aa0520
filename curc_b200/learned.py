"""Training and evaluation of the learned mismatch coder on the
position-dependent-error workload (paired-end 150 bp; substitution rate
rising from 0.1% at base 1 to 1.0% at base 150; transitions twice as likely
as each transversion).  Training and evaluation seeds are disjoint."""
from __future__ import annotations

import numpy as np

from . import synth
from ._native import Context, Learner, general_mismatch_bytes, plain_mismatch_bytes


def workload(seed: int, pairs: int, genome_len: int):
    return synth.paired_repeats(seed=seed, pairs=pairs, read_len=150, genome_len=genome_len,
                                err=synth.position_ramp(150, 0.001, 0.010), ti_tv=2.0, preserve_order=True)


def train_and_evaluate(train_seeds, eval_seeds, pairs=200_000, genome_len=2_000_000, epochs=3, batch=4096,
                       lr=2e-3, device=0, eval_pairs=None, eval_genome_len=None, general=None):
    """Trains on blocks of the training seeds and codes the mismatch streams of
    the evaluation seeds both ways.  Returns a dict with bytes and bits/base of
    the plain and the learned coding, the training loss, and whether every
    learned stream decoded back to its block's mismatches.  Evaluation blocks
    may be larger than the training blocks (eval_pairs, eval_genome_len).
    With `general` = (bsc executable, scratch dir), the same mismatch streams
    are also coded with fast-lzma2 level 10 and libbsc."""
    eval_pairs = eval_pairs or pairs
    eval_genome_len = eval_genome_len or genome_len
    with Context(device) as ctx, Learner(device) as lrn:
        ctx.keep_intermediates(False)
        for s in train_seeds:
            w = workload(s, pairs, genome_len)
            ctx.block_run(w.sequences(), True, True)
            lrn.add_block(ctx)
        loss = lrn.train(epochs=epochs, batch=batch, lr=lr, seed=1)
        res = {"train_anchors": lrn.anchors, "loss": loss, "bases": 0, "plain": [0, 0, 0], "learned": 0,
               "lossless": True, "general": [0, 0], "model_bytes": len(lrn.model())}
        for s in eval_seeds:
            w = workload(s, eval_pairs, eval_genome_len)
            seqs = w.sequences()
            del w
            ctx.block_run(seqs, True, True)
            cnt, base, off = plain_mismatch_bytes(ctx)
            stream = lrn.encode(ctx)
            res["lossless"] &= lrn.decode_check(ctx, stream)
            res["plain"] = [a + b for a, b in zip(res["plain"], (cnt, base, off))]
            res["learned"] += len(stream)
            res["bases"] += seqs.size
            if general:
                g = general_mismatch_bytes(ctx, *general)
                res["general"] = [a + b for a, b in zip(res["general"], g)]
        cnt, base, off = res["plain"]
        res["plain_bits_per_base"] = 8.0 * (cnt + base + off) / res["bases"]
        res["learned_bits_per_base"] = 8.0 * (cnt + res["learned"]) / res["bases"]
        res["gaps_and_bases_ratio"] = res["learned"] / max(1, base + off)
        res["mismatch_streams_ratio"] = (cnt + res["learned"]) / max(1, cnt + base + off)
        if general:
            res["fl2_level10_bits_per_base"] = 8.0 * res["general"][0] / res["bases"]
            res["libbsc_bits_per_base"] = 8.0 * res["general"][1] / res["bases"]
        return res
