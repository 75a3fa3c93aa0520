"""Learned mode of `curc -c` on a B200: the learned mismatch coder as a
per-block coder choice inside the .curc archive.

A model trained on two seeds of the position-dependent-error workload codes
a block of a disjoint seed.  The writer keeps, per block, the smaller of the
plain coding (the reference's PPMd / range-coder streams) and the learned
one, marking a learned block in its mismatch-base container; the product
decoder must give back every read, in order.  Plain mode stays the
reference's format: with the model cleared, the archive is byte for byte the
one written before any model was set."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

pytestmark = pytest.mark.gpu

BSC = os.path.join(ROOT, "curc_b200", "_build", "bsc")
NAME = b"synthetic_read_"


def _rows(path, n, L):
    a = np.fromfile(path, dtype=np.uint8).reshape(n, L + 1)
    return a[:, :L]


def test_learned_blocks_roundtrip_and_plain_mode_unchanged(tmp_path):
    from curc_b200 import Context, Learner, archive_info, decompress_file
    from curc_b200.learned import workload
    with Context(0) as ctx, Learner(0) as lrn:
        ctx.keep_intermediates(False)
        for s in (501, 502):
            w = workload(s, 200_000, 2_000_000)
            ctx.block_run(w.sequences(), True, True)
            lrn.add_block(ctx)
        lrn.train(epochs=2, batch=4096)
        model = lrn.model()
        # large block (learned expected to win) and small block (the model's
        # own bytes outweigh its gain: plain expected)
        results = {}
        for tag, pairs, glen in (("large", 1_000_000, 5_000_000), ("small", 20_000, 200_000)):
            w = workload(601, pairs, glen)
            files = w.write(str(tmp_path / tag), name=NAME)
            plain = str(tmp_path / f"{tag}_plain.curc")
            learned = str(tmp_path / f"{tag}_learned.curc")
            plain2 = str(tmp_path / f"{tag}_plain2.curc")
            ctx.compress_files(files, plain, 1.0, True, BSC, str(tmp_path))
            ctx.set_mismatch_model(model)
            ctx.compress_files(files, learned, 1.0, True, BSC, str(tmp_path))
            kept = ctx.stage_ms("files.learned_blocks")
            kb = (ctx.stage_ms("files.mismatch_plain_kb"), ctx.stage_ms("files.mismatch_learned_kb"))
            ctx.set_mismatch_model(None)
            ctx.compress_files(files, plain2, 1.0, True, BSC, str(tmp_path))
            for f in files:
                os.remove(f)
            assert open(plain, "rb").read() == open(plain2, "rb").read()
            n, L = w.mate1.shape
            out = str(tmp_path / f"{tag}_out")
            assert decompress_file(learned, out, BSC, str(tmp_path)) == 2 * n
            assert np.array_equal(_rows(out + "_1.seq", n, L), w.mate1)
            assert np.array_equal(_rows(out + "_2.seq", n, L), w.mate2)
            results[tag] = (kept, kb, os.path.getsize(plain), os.path.getsize(learned))
            assert len(archive_info(learned)["block_bytes"]) == 1
    kept, (kb_plain, kb_learned), size_plain, size_learned = results["large"]
    assert kept == 1 and kb_learned < kb_plain and size_learned < size_plain, results
    kept, (kb_plain, kb_learned), size_plain, size_learned = results["small"]
    assert kept == 0 and size_learned == size_plain, results
