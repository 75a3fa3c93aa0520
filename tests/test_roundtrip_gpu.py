"""Lossless round trip at the benchmark's full size, on a B200.

The paired-end 150 bp workload of the benchmark (10M pairs, 3 Gbases,
--preserve_order, one block) goes through the whole-file compressor (FASTQ
files to a .curc archive: ingest, device path, stream coders) and back
through the product decoder; every read must come back, in order.  At this
size the oracle cannot run, so the round trip is the size-independent check;
the stage-by-stage comparison with the oracle is done on the smaller cases of
test_parity_gpu.py."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

pytestmark = pytest.mark.gpu

BSC = os.path.join(ROOT, "curc_b200", "_build", "bsc")


def _rows(path, n, L):
    a = np.fromfile(path, dtype=np.uint8)
    assert a.size == n * (L + 1)
    a = a.reshape(n, L + 1)
    assert np.all(a[:, L] == ord("\n"))
    return a[:, :L]


def test_full_size_roundtrip(tmp_path):
    import bench
    from curc_b200 import Context, decompress_file
    w = bench.workload(10_000_000, 50_000_000, seed=1)
    files = w.write(str(tmp_path / "in"), name=bench.FASTQ_NAME)
    archive = str(tmp_path / "full.curc")
    with Context(0) as ctx:
        reads, blocks = ctx.compress_files(files, archive, 1.0, True, BSC, str(tmp_path))
    for f in files:
        os.remove(f)
    n, L = w.mate1.shape
    assert reads == 2 * n and blocks == 1
    outs = [str(tmp_path / "out_1.seq"), str(tmp_path / "out_2.seq")]
    try:
        assert decompress_file(archive, str(tmp_path / "out"), BSC, str(tmp_path)) == 2 * n
        assert np.array_equal(_rows(outs[0], n, L), w.mate1)
        assert np.array_equal(_rows(outs[1], n, L), w.mate2)
    finally:
        for f in outs + [archive]:
            if os.path.exists(f):
                os.remove(f)
