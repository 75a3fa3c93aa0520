"""FASTQ ingest and block split (`curc_fastq_blocks`) on the CPU.

The product's parallel reader must cut the same blocks as the reference's
process() (preprocess.cpp:66-254), restated by the oracle's split_fastq: the
same block count, the same reads per block, the same read order (mates
interleaved), and the same errors."""
import ctypes
import os

import numpy as np
import pytest

from curc_b200 import synth
from tests.oracle_lib import lib as oracle_lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BLOCK_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64,
                            ctypes.c_uint16)
CURC_OK, CURC_ERR_STATE, CURC_ERR_IO = 0, -3, -4


def _lib():
    L = ctypes.CDLL(os.path.join(ROOT, "curc_b200", "libcurc_b200.so"))
    L.curc_fastq_blocks.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double, BLOCK_FN, ctypes.c_void_p,
                                    ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint32)]
    L.curc_last_error.restype = ctypes.c_char_p
    L.curc_last_error.argtypes = [ctypes.c_void_p]
    return L


def product_blocks(files, ratio, stop_at=None):
    got = []

    def cb(_user, index, seqs, n, L):
        got.append((index, L, ctypes.string_at(seqs, n * L) if n else b""))
        return 1 if stop_at is not None and index == stop_at else 0

    fn = BLOCK_FN(cb)
    reads, blocks = ctypes.c_uint64(), ctypes.c_uint32()
    L = _lib()
    rc = L.curc_fastq_blocks(files[0].encode(), files[1].encode() if len(files) > 1 else None, ratio, fn, None,
                             ctypes.byref(reads), ctypes.byref(blocks))
    return rc, got, reads.value, blocks.value, L.curc_last_error(None).decode()


def oracle_blocks(files, ratio):
    O = oracle_lib()
    O.oracle_split_fastq.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double,
                                     ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_void_p),
                                     ctypes.POINTER(ctypes.c_uint64)]
    nb, L = ctypes.c_uint32(), ctypes.c_int()
    counts = (ctypes.c_uint64 * 256)()
    out, size = ctypes.c_void_p(), ctypes.c_uint64()
    rc = O.oracle_split_fastq(files[0].encode(), files[1].encode() if len(files) > 1 else None, ratio,
                              ctypes.byref(nb), ctypes.byref(L), counts, ctypes.byref(out), ctypes.byref(size))
    data = ctypes.string_at(out, size.value) if rc == 0 else ctypes.string_at(out).decode()
    O.oracle_buf_free(out)
    if rc != 0:
        return None, data
    return (L.value, [int(counts[i]) for i in range(nb.value)], data), None


CASES = {
    "se_one_block": lambda: (synth.small_single(seed=51, n_reads=20_000, read_len=100, genome_len=100_000), 1.0),
    "pe_one_block": lambda: (synth.paired_repeats(seed=52, pairs=10_000, read_len=150, genome_len=200_000), 1.0),
    # above one 50 MB window (25 MB per mate for paired end), several blocks
    "se_blocks": lambda: (synth.small_single(seed=53, n_reads=300_000, read_len=100, genome_len=400_000), 0.3),
    "pe_blocks": lambda: (synth.paired_repeats(seed=54, pairs=150_000, read_len=100, genome_len=400_000), 0.25),
    "se_odd_length": lambda: (synth.small_single(seed=55, n_reads=5_000, read_len=37, genome_len=50_000), 1.0),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_blocks_match_oracle(name, tmp_path):
    w, ratio = CASES[name]()
    files = w.write(str(tmp_path / name), name=b"synthetic_read_")
    rc, got, reads, blocks, err = product_blocks(files, ratio)
    assert rc == CURC_OK, err
    ref, why = oracle_blocks(files, ratio)
    assert ref is not None, why
    L, counts, data = ref
    assert blocks == len(counts) == len(got)
    assert [i for i, _, _ in got] == list(range(blocks))
    assert all(l == L == w.read_len for _, l, _ in got)
    assert [len(s) // L for _, _, s in got] == counts
    assert b"".join(s for _, _, s in got) == data
    assert reads == sum(counts)
    # block order is the files' order, mates interleaved
    assert np.array_equal(np.frombuffer(data, dtype=np.uint8).reshape(-1, L), w.sequences())
    if name.endswith("_blocks"):
        assert blocks >= 2


def test_callback_stops(tmp_path):
    w, ratio = CASES["se_blocks"]()
    files = w.write(str(tmp_path / "s"), name=b"synthetic_read_")
    rc, got, _, _, err = product_blocks(files, ratio, stop_at=0)
    assert rc == CURC_ERR_STATE and len(got) == 1, err


def test_bad_inputs(tmp_path):
    w = synth.paired_repeats(seed=56, pairs=200, read_len=50, genome_len=20_000)
    f1, f2 = w.write(str(tmp_path / "p"))
    # mate files of different sizes
    with open(f2, "ab") as f:
        f.write(b"@x\nACGT\n+\nIIII\n")
    rc, _, _, _, err = product_blocks([f1, f2], 1.0)
    assert rc == CURC_ERR_IO and "size" in err
    # a read of another length
    s = synth.small_single(seed=57, n_reads=100, read_len=40, genome_len=10_000)
    (p,) = s.write(str(tmp_path / "s"))
    data = open(p, "rb").read().split(b"\n")
    data[5] = data[5][:-1]
    data[7] = data[7][:-1]
    open(p, "wb").write(b"\n".join(data))
    rc, _, _, _, err = product_blocks([p], 1.0)
    assert rc == CURC_ERR_IO and "length" in err
    rc, _, _, _, err = product_blocks([str(tmp_path / "missing.fastq")], 1.0)
    assert rc == CURC_ERR_IO


def test_python_wrappers(tmp_path):
    from curc_b200 import archive_info, fastq_blocks
    w, ratio = CASES["pe_blocks"]()
    files = w.write(str(tmp_path / "p"), name=b"synthetic_read_")
    blocks = fastq_blocks(files[0], files[1], ratio)
    assert len(blocks) >= 2
    assert np.array_equal(np.concatenate(blocks), w.sequences())
    info = archive_info(os.path.join(ROOT, "tests", "golden", "pe150_po_p8k.curc"))
    assert info["paired_end"] and info["preserve_order"] and info["read_len"] == 150
    assert info["block_reads"] == [16000]
