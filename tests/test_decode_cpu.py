"""The product decoder (`curc_decompress_file`, `curc -d`) on the CPU.

Archives come from the golden fixtures (written by the reference's own
`curc -c` on a GPU machine) and from the oracle's archive writer, whose
archives the GPU tests pin byte for byte to the CUDA path's.  Every decode
must give back the input reads (in input order with preserved order, as the
same multiset otherwise) and, where the reference decoder was built here
(oracle/_ref/curc), equal its output byte for byte."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_golden  # noqa: E402
from curc_b200 import synth  # noqa: E402
from tests.oracle_lib import REF_DIR, lib as oracle_lib  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")
BSC = os.path.join(ROOT, "curc_b200", "_build", "bsc")
REF_CURC = os.path.join(REF_DIR, "curc")
CURC_OK, CURC_ERR_IO, CURC_ERR_STATE = 0, -4, -3


def _lib():
    L = ctypes.CDLL(os.path.join(ROOT, "curc_b200", "libcurc_b200.so"))
    L.curc_decompress_file.argtypes = [ctypes.c_char_p] * 4 + [ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)]
    L.curc_last_error.restype = ctypes.c_char_p
    L.curc_last_error.argtypes = [ctypes.c_void_p]
    return L


def decode(archive, wd, name="mine", threads=0):
    L = _lib()
    n = ctypes.c_uint64()
    rc = L.curc_decompress_file(str(archive).encode(), os.path.join(str(wd), name).encode(), BSC.encode(),
                                str(wd).encode(), threads, ctypes.byref(n))
    return rc, n.value, L.curc_last_error(None).decode()


def outputs(wd, name, pe):
    files = [f"{name}_1.seq", f"{name}_2.seq"] if pe else [f"{name}.seq"]
    return [open(os.path.join(str(wd), f), "rb").read() for f in files]


def rows(data, L):
    return np.frombuffer(b"".join(data.split(b"\n")[:-1]), dtype=np.uint8).reshape(-1, L)


def same_reads(outs, w):
    L = w.read_len
    if w.mate2 is None:
        got = rows(outs[0], L)
        if w.preserve_order:
            return np.array_equal(got, w.mate1)
        return np.array_equal(np.sort(got.view(f"S{L}").ravel()), np.sort(w.mate1.view(f"S{L}").ravel()))
    g1, g2 = rows(outs[0], L), rows(outs[1], L)
    if w.preserve_order:
        return np.array_equal(g1, w.mate1) and np.array_equal(g2, w.mate2)
    gp = np.concatenate([g1, g2], axis=1).view(f"S{2 * L}").ravel()
    ep = np.concatenate([w.mate1, w.mate2], axis=1).view(f"S{2 * L}").ravel()
    return np.array_equal(np.sort(gp), np.sort(ep))


def reference_outputs(archive, wd, pe):
    if not os.path.exists(REF_CURC):
        return None
    r = subprocess.run([REF_CURC, "-d", "-i", str(archive), "-o", "ref", "--working_dir", str(wd)], cwd=REF_DIR,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return outputs(wd, "ref", pe)


def check(archive, w, wd):
    rc, n, err = decode(archive, wd)
    assert rc == CURC_OK, err
    pe = w.mate2 is not None
    assert n == w.mate1.shape[0] * (2 if pe else 1)
    mine = outputs(wd, "mine", pe)
    assert same_reads(mine, w)
    ref = reference_outputs(archive, wd, pe)
    if ref is not None:
        assert mine == ref


# The golden pe150_p8k archive is left out: the reference writes a different
# archive on every run for that case, and its own decoder crashes on the
# stored one; the same input is covered below through the oracle's archive.
@pytest.mark.parametrize("name", ["c0_se100_n100k", "se75_n20k", "se250_n8k", "pe150_po_p8k"])
def test_decode_golden(name, tmp_path):
    check(os.path.join(GOLDEN, name + ".curc"), make_golden.CASES[name](), tmp_path)


ORACLE_CASES = {
    "pe150_p8k": lambda: make_golden.CASES["pe150_p8k"](),
    "se100_po": lambda: _po(synth.small_single(seed=41, n_reads=20_000, read_len=100, genome_len=200_000)),
    "se150_manyN": lambda: synth.small_single(seed=42, n_reads=10_000, read_len=150, genome_len=100_000,
                                             err=0.004, n_rate=0.003),
    "se33_odd": lambda: synth.small_single(seed=43, n_reads=20_000, read_len=33, genome_len=60_000),
    "se251_po": lambda: _po(synth.small_single(seed=44, n_reads=4_000, read_len=251, genome_len=200_000)),
    "pe100_po_manyN": lambda: synth.paired_repeats(seed=45, pairs=5_000, read_len=100, genome_len=300_000,
                                                   n_rate=0.002, preserve_order=True),
    "pe75": lambda: synth.paired_repeats(seed=46, pairs=6_000, read_len=75, genome_len=200_000,
                                         preserve_order=False),
    # a RefMatcher probe past the last full 36-mer of a pseudogenome, where the
    # reference's length arithmetic breaks: found by a random sweep
    "pe133_po_tail": lambda: synth.paired_repeats(seed=551869, pairs=1585, read_len=133, genome_len=63594,
                                                  err=0.001, n_rate=0.003, preserve_order=True),
}


def _po(w):
    w.preserve_order = True
    return w


@pytest.mark.parametrize("name", sorted(ORACLE_CASES))
def test_decode_oracle_archive(name, tmp_path):
    w = ORACLE_CASES[name]()
    files = w.write(str(tmp_path / name))
    rc = oracle_lib().oracle_compress_files(files[0].encode(), files[1].encode() if len(files) > 1 else None,
                                            str(tmp_path).encode(), b"oracle", 1.0, int(w.preserve_order),
                                            os.path.join(REF_DIR, "bsc").encode(), 8)
    assert rc == 0
    check(tmp_path / "oracle.curc", w, tmp_path)


def test_decode_threads_agree(tmp_path):
    archive = os.path.join(GOLDEN, "se75_n20k.curc")
    assert decode(archive, tmp_path, "one", threads=1)[0] == CURC_OK
    assert decode(archive, tmp_path, "all", threads=0)[0] == CURC_OK
    assert outputs(tmp_path, "one", False) == outputs(tmp_path, "all", False)


def test_decode_errors(tmp_path):
    rc, _, err = decode(tmp_path / "missing.curc", tmp_path)
    assert rc == CURC_ERR_IO and "missing.curc" in err
    data = open(os.path.join(GOLDEN, "se75_n20k.curc"), "rb").read()
    for cut in (3, 40, len(data) // 2, len(data) - 1):
        p = tmp_path / f"cut{cut}.curc"
        p.write_bytes(data[:cut])
        rc, _, err = decode(p, tmp_path)
        assert rc == CURC_ERR_STATE, (cut, err)
    p = tmp_path / "extra.curc"
    p.write_bytes(data + b"\0")
    rc, _, err = decode(p, tmp_path)
    assert rc == CURC_ERR_STATE and "after the last block" in err


def test_decode_multiblock(tmp_path):
    # two blocks: above one 50 MB window, cut at block_ratio 0.3
    w = synth.small_single(seed=31, n_reads=300_000, read_len=100, genome_len=800_000)
    files = w.write(str(tmp_path / "mb"), name=b"synthetic_read_")
    rc = oracle_lib().oracle_compress_files(files[0].encode(), None, str(tmp_path).encode(), b"oracle", 0.3, 0,
                                            os.path.join(REF_DIR, "bsc").encode(), 8)
    assert rc == 0
    archive = tmp_path / "oracle.curc"
    assert archive.read_bytes()[4] >= 2
    check(archive, w, tmp_path)


def test_cli_decompress(tmp_path):
    cli = os.path.join(ROOT, "curc_b200", "_build", "curc")
    archive = os.path.join(GOLDEN, "pe150_po_p8k.curc")
    r = subprocess.run([cli, "-d", "-i", archive, "-o", "cli", "--working_dir", str(tmp_path)], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout == ""  # as the reference's decoder
    assert decode(archive, tmp_path)[0] == CURC_OK
    assert outputs(tmp_path, "cli", True) == outputs(tmp_path, "mine", True)
    assert not [f for f in os.listdir(tmp_path) if f.startswith("curc_tmp_")]
    # an output directory that cannot be written
    rc, _, err = decode(archive, tmp_path / "no" / "such" / "dir")
    assert rc == CURC_ERR_IO, err


def test_python_wrapper(tmp_path):
    from curc_b200 import CurcError, decompress_file
    archive = os.path.join(GOLDEN, "se250_n8k.curc")
    assert decompress_file(archive, str(tmp_path / "py"), tmpdir=str(tmp_path)) == 8000
    assert decode(archive, tmp_path)[0] == CURC_OK
    assert outputs(tmp_path, "py", False) == outputs(tmp_path, "mine", False)
    with pytest.raises(CurcError):
        decompress_file(str(tmp_path / "missing.curc"), str(tmp_path / "x"), tmpdir=str(tmp_path))


def test_corrupt_payloads_do_not_end_the_process(tmp_path):
    from tests.archive import split_archive
    data = bytearray(open(os.path.join(GOLDEN, "se75_n20k.curc"), "rb").read())
    blk = split_archive(bytes(data))["blocks"][0]
    # the mismatch-count container: decoded size, coded size, coder (PPMd), then the model order
    c = blk["mismatch_count"]
    at = bytes(data).find(c)
    assert at > 0 and data[at + 16] == 3
    bad = bytearray(data)
    bad[at + 17] = 1  # model order below the minimum
    p = tmp_path / "order.curc"
    p.write_bytes(bytes(bad))
    rc, _, err = decode(p, tmp_path)
    assert rc == CURC_ERR_STATE and "PPMd" in err
    # flipped bytes inside coded payloads: an error or some output, never an exit
    rng = np.random.default_rng(5)
    for name in ("mismatch_base", "ref_off_map", "mismatch_count"):
        s = blk[name]
        at = bytes(data).find(s)
        for _ in range(3):
            bad = bytearray(data)
            k = at + 22 + int(rng.integers(0, max(1, len(s) - 22)))
            bad[k] ^= 0x5A
            p = tmp_path / f"flip_{name}.curc"
            p.write_bytes(bytes(bad))
            rc, _, err = decode(p, tmp_path)
            assert rc in (CURC_OK, CURC_ERR_STATE), err


def test_archive_info(tmp_path):
    from tests.archive import split_archive
    L = _lib()
    L.curc_archive_info.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_uint16), ctypes.POINTER(ctypes.c_uint32),
                                    ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint32)]
    for name in ["c0_se100_n100k", "pe150_po_p8k", "pe150_p8k"]:
        path = os.path.join(GOLDEN, name + ".curc")
        data = open(path, "rb").read()
        ref = split_archive(data)
        po, pe, rl, nb = ctypes.c_int(), ctypes.c_int(), ctypes.c_uint16(), ctypes.c_uint32()
        sizes, reads = (ctypes.c_uint64 * 256)(), (ctypes.c_uint32 * 256)()
        assert L.curc_archive_info(path.encode(), ctypes.byref(po), ctypes.byref(pe), ctypes.byref(rl),
                                   ctypes.byref(nb), sizes, reads) == CURC_OK
        assert (bool(po.value), bool(pe.value), rl.value) == (bool(ref["preserve_order"]), bool(ref["paired_end"]),
                                                              ref["read_len"])
        assert nb.value == len(ref["blocks"])
        assert [reads[i] for i in range(nb.value)] == [b["reads_count"] for b in ref["blocks"]]
        assert 5 + sum(sizes[i] for i in range(nb.value)) == len(data)
    p = tmp_path / "cut.curc"
    p.write_bytes(data[:-3])
    assert L.curc_archive_info(str(p).encode(), None, None, None, None, None, None) == CURC_ERR_STATE


def test_device_count_without_gpu():
    import torch
    L = _lib()
    n = ctypes.c_int(-1)
    rc = L.curc_device_count(ctypes.byref(n))
    if torch.cuda.is_available():
        assert rc == CURC_OK and n.value >= 1
    else:
        assert rc in (CURC_OK, -2) and n.value == 0


def test_random_corruptions_are_errors_or_output(tmp_path):
    # seeded multi-byte corruptions and truncations of every golden archive: each
    # decode returns an error code or writes reads, and this process survives
    rng = np.random.default_rng(11)
    for name in sorted(f for f in os.listdir(GOLDEN) if f.endswith(".curc")):
        data = open(os.path.join(GOLDEN, name), "rb").read()
        for t in range(6):
            bad = bytearray(data)
            if t % 3 == 2:
                bad = bad[:int(rng.integers(1, len(bad)))]
            else:
                for k in rng.integers(0, len(bad), size=int(rng.integers(1, 12))):
                    bad[int(k)] = int(rng.integers(0, 256))
            p = tmp_path / f"bad_{name}_{t}.curc"
            p.write_bytes(bytes(bad))
            rc, _, err = decode(p, tmp_path)
            assert rc in (CURC_OK, CURC_ERR_STATE), (name, t, err)


def _random_case(rnd):
    L = rnd.choice([rnd.randint(20, 40), rnd.randint(41, 160), rnd.randint(161, 511)])
    pe, po = rnd.random() < 0.5, rnd.random() < 0.5
    n = rnd.randint(50, 2000)
    kw = dict(err=rnd.choice([0.0, 0.001, 0.01]), n_rate=rnd.choice([0.0, 0.0001, 0.003, 0.02]))
    seed = rnd.randint(0, 10**6)
    if pe:
        return synth.paired_repeats(seed=seed, pairs=n, read_len=L, genome_len=rnd.randint(3 * L + 20_000, 100_000),
                                    preserve_order=po, **kw)
    w = synth.small_single(seed=seed, n_reads=n, read_len=L, genome_len=rnd.randint(2 * L + 1000, 100_000), **kw)
    w.preserve_order = po
    return w


@pytest.mark.parametrize("sweep_seed", range(12))
def test_random_small_archives(sweep_seed, tmp_path):
    # random read lengths (20-511), ends, order, error and N rates: the oracle's
    # archive must decode, with the product decoder and the reference's, to the
    # input reads (this sweep found the RefMatcher tail rule)
    import random
    w = _random_case(random.Random(1000 + sweep_seed))
    files = w.write(str(tmp_path / "in"))
    pe = w.mate2 is not None
    rc = oracle_lib().oracle_compress_files(files[0].encode(), files[1].encode() if pe else None,
                                            str(tmp_path).encode(), b"oracle", 1.0, int(w.preserve_order),
                                            os.path.join(REF_DIR, "bsc").encode(), 8)
    assert rc == 0
    check(tmp_path / "oracle.curc", w, tmp_path)
