"""The drop-in `curc -c` (curc_b200/_build/curc) on a B200.

Its archives must equal the oracle's byte for byte (same streams, same
coders), equal the reference's own archive where the reference is
deterministic, and decode with the reference's `curc -d` back to the input
reads.  A multi-block input (block_ratio < 1 over two 50 MB windows) checks
the block split."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_golden  # noqa: E402
from curc_b200 import synth  # noqa: E402
from tests.oracle_lib import REF_DIR, lib  # noqa: E402

pytestmark = pytest.mark.gpu
CLI = os.path.join(ROOT, "curc_b200", "_build", "curc")
GOLDEN = os.path.join(ROOT, "tests", "golden")
META = json.load(open(os.path.join(GOLDEN, "golden_meta.json")))


def run_cli(files, po, wd, name, ratio=1.0):
    cmd = [CLI, "-c", "-i", ",".join(files), "-o", name, "--working_dir", str(wd), "--block_ratio", str(ratio)]
    if po:
        cmd.append("--preserve_order")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    return open(os.path.join(wd, name + ".curc"), "rb").read(), r.stdout


def oracle(files, po, wd, ratio=1.0):
    rc = lib().oracle_compress_files(files[0].encode(), files[1].encode() if len(files) > 1 else None,
                                     str(wd).encode(), b"oracle", ratio, int(po),
                                     os.path.join(REF_DIR, "bsc").encode(), 8)
    assert rc == 0
    return open(os.path.join(wd, "oracle.curc"), "rb").read()


def decode_matches(archive_path, w, wd):
    r = subprocess.run([os.path.join(REF_DIR, "curc"), "-d", "-i", archive_path, "-o", "dec", "--working_dir", str(wd)],
                       cwd=REF_DIR, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    L = w.read_len

    def lines(p):
        return np.frombuffer(b"".join(open(p, "rb").read().split(b"\n")[:-1]), dtype=np.uint8).reshape(-1, L)

    if w.mate2 is None:
        got = lines(os.path.join(wd, "dec.seq"))
        if w.preserve_order:
            return np.array_equal(got, w.mate1)
        return np.array_equal(np.sort(got.view(f"S{L}").ravel()), np.sort(w.mate1.view(f"S{L}").ravel()))
    g1, g2 = lines(os.path.join(wd, "dec_1.seq")), lines(os.path.join(wd, "dec_2.seq"))
    if w.preserve_order:
        return np.array_equal(g1, w.mate1) and np.array_equal(g2, w.mate2)
    gp = np.concatenate([g1, g2], axis=1).view(f"S{2 * L}").ravel()
    ep = np.concatenate([w.mate1, w.mate2], axis=1).view(f"S{2 * L}").ravel()
    return np.array_equal(np.sort(gp), np.sort(ep))


@pytest.mark.parametrize("name", sorted(make_golden.CASES))
def test_cli_archive(name, tmp_path):
    w = make_golden.CASES[name]()
    files = w.write(str(tmp_path / name))
    mine, out = run_cli(files, w.preserve_order, tmp_path, "prod")
    assert "archive size" in out
    # the CUDA set-up runs while the input is parsed; its line still comes first
    assert out.index("gpu context init finish") < out.index("reads count")
    assert mine == oracle(files, w.preserve_order, tmp_path)
    if META[name]["deterministic"] and name != "pe150_po_p8k":
        assert mine == open(os.path.join(GOLDEN, name + ".curc"), "rb").read()
    assert decode_matches(os.path.join(tmp_path, "prod.curc"), w, tmp_path)


def test_cli_multiblock(tmp_path):
    w = synth.small_single(seed=31, n_reads=300_000, read_len=100, genome_len=800_000)
    files = w.write(str(tmp_path / "mb"), name=b"synthetic_read_")
    assert os.path.getsize(files[0]) > 50_000_000
    mine, _ = run_cli(files, False, tmp_path, "prod", ratio=0.3)
    assert mine[4] >= 2  # blocks
    assert mine == oracle(files, False, tmp_path, ratio=0.3)
    assert decode_matches(os.path.join(tmp_path, "prod.curc"), w, tmp_path)


def test_deferred_context_compresses_alike(tmp_path):
    """curc_ctx_create_deferred: the FASTQ windows parsed before the CUDA
    set-up has finished wait in host memory and reach the device in order;
    the archive is the oracle's, over several windows and blocks."""
    from curc_b200 import Context
    w = synth.small_single(seed=32, n_reads=300_000, read_len=100, genome_len=800_000)
    files = w.write(str(tmp_path / "df"), name=b"synthetic_read_")
    bsc = os.path.join(ROOT, "curc_b200", "_build", "bsc")
    arc = str(tmp_path / "deferred.curc")
    with Context(0, deferred=True) as ctx:
        ctx.compress_files(files, arc, 0.3, False, bsc, str(tmp_path))
    mine = open(arc, "rb").read()
    assert mine[4] >= 2  # blocks
    assert mine == oracle(files, False, tmp_path, ratio=0.3)
