"""The product's block writer (`curc_encode_block`, `curc_archive_header`) on
the CPU.

Given the oracle's streams of a block, the product's coders must write the
same block body as the oracle's writer, byte for byte (the reference's block
layout, compress.cu:1364-2146); header plus body must then decode, with the
product decoder, back to the block's reads."""
import ctypes
import os

import numpy as np
import pytest

from curc_b200 import synth
from tests.oracle_lib import OracleBlock
from tests.test_decode_cpu import decode, outputs, same_reads, CURC_OK

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BSC = os.path.join(ROOT, "curc_b200", "_build", "bsc")
CURC_ERR_STATE = -3


def _lib():
    L = ctypes.CDLL(os.path.join(ROOT, "curc_b200", "libcurc_b200.so"))
    L.curc_encode_block.argtypes = [ctypes.c_uint32, ctypes.c_uint16, ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_void_p),
                                    ctypes.POINTER(ctypes.c_uint64), ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p),
                                    ctypes.POINTER(ctypes.c_uint64)]
    L.curc_buffer_free.argtypes = [ctypes.c_void_p]
    L.curc_archive_header.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint16, ctypes.c_uint32, ctypes.c_char_p]
    L.curc_last_error.restype = ctypes.c_char_p
    L.curc_last_error.argtypes = [ctypes.c_void_p]
    return L


def stream_names(L, po, pe):
    names = ["decoder_table", "sizes", "strand", "ref", "unmap_ref", "unmap_n_ref", "mis_cnt", "mis_base",
             "ref_off", "ref_len_map", "unmap_ref_off", "unmap_ref_len", "unmap_n_ref_off", "unmap_n_ref_len"]
    if po:
        names.append("id_to_pos")
    else:
        names += ["read_off", "unmap_read_off", "unmap_n_read_off"] + (["pe_order"] if pe else [])
    return names + [f"mis_off_{m}" for m in range(1, L // 5 + 1)]


def encode(n, L, po, pe, streams, tmpdir, drop=None):
    lib = _lib()
    items = [(k, v) for k, v in streams.items() if k != drop]
    keep = [np.ascontiguousarray(v) for _, v in items]
    names = (ctypes.c_char_p * len(items))(*[k.encode() for k, _ in items])
    ptrs = (ctypes.c_void_p * len(items))(*[a.ctypes.data if a.size else None for a in keep])
    sizes = (ctypes.c_uint64 * len(items))(*[a.nbytes for a in keep])
    out, nb = ctypes.c_void_p(), ctypes.c_uint64()
    rc = lib.curc_encode_block(n, L, int(po), int(pe), names, ptrs, sizes, len(items), 10, 16, BSC.encode(),
                               str(tmpdir).encode(), ctypes.byref(out), ctypes.byref(nb))
    if rc != CURC_OK:
        return rc, lib.curc_last_error(None).decode()
    body = ctypes.string_at(out, nb.value)
    lib.curc_buffer_free(out)
    return rc, body


CASES = {
    "se100": lambda: synth.small_single(seed=61, n_reads=20_000, read_len=100, genome_len=200_000),
    "se100_po": lambda: _po(synth.small_single(seed=62, n_reads=20_000, read_len=100, genome_len=200_000)),
    "se150_manyN": lambda: synth.small_single(seed=63, n_reads=10_000, read_len=150, genome_len=100_000, err=0.004,
                                             n_rate=0.003),
    "se37": lambda: synth.small_single(seed=64, n_reads=10_000, read_len=37, genome_len=40_000),
    "pe150": lambda: synth.paired_repeats(seed=65, pairs=8_000, read_len=150, genome_len=300_000,
                                          preserve_order=False),
    "pe150_po": lambda: synth.paired_repeats(seed=66, pairs=8_000, read_len=150, genome_len=300_000,
                                             preserve_order=True),
    # enough pairs for the position coder's threads to split the work, and
    # mates far enough apart for its delta streams
    "pe150_po_150k": lambda: synth.paired_repeats(seed=67, pairs=150_000, read_len=150, genome_len=2_000_000,
                                                  preserve_order=True),
}


def _po(w):
    w.preserve_order = True
    return w


@pytest.mark.parametrize("name", sorted(CASES))
def test_block_body_matches_oracle(name, tmp_path):
    w = CASES[name]()
    seqs = w.sequences()
    n, L = seqs.shape
    po, pe = w.preserve_order, w.mate2 is not None
    ora = OracleBlock(seqs, po, pe)
    streams = {k: ora.get(k) for k in stream_names(L, po, pe)}
    rc, body = encode(n, L, po, pe, streams, tmp_path)
    assert rc == CURC_OK, body
    assert body == ora.encode(str(tmp_path))
    # header + body is an archive that decodes back to the reads
    hdr = ctypes.create_string_buffer(5)
    assert _lib().curc_archive_header(int(po), int(pe), L, 1, hdr) == CURC_OK
    archive = tmp_path / "one.curc"
    archive.write_bytes(hdr.raw + body)
    rc, count, err = decode(archive, tmp_path)
    assert rc == CURC_OK and count == n, err
    assert same_reads(outputs(tmp_path, "mine", pe), w)


def test_missing_stream(tmp_path):
    w = CASES["se37"]()
    seqs = w.sequences()
    n, L = seqs.shape
    ora = OracleBlock(seqs, False, False)
    streams = {k: ora.get(k) for k in stream_names(L, False, False)}
    rc, err = encode(n, L, False, False, streams, tmp_path, drop="mis_base")
    assert rc == CURC_ERR_STATE and "mis_base" in err


@pytest.mark.parametrize("sweep_seed", range(8))
def test_random_block_bodies_match_oracle(sweep_seed, tmp_path):
    # random read lengths (20-511), ends, order, error and N rates
    import random
    from tests.test_decode_cpu import _random_case
    w = _random_case(random.Random(2000 + sweep_seed))
    seqs = w.sequences()
    n, L = seqs.shape
    po, pe = w.preserve_order, w.mate2 is not None
    ora = OracleBlock(seqs, po, pe)
    streams = {k: ora.get(k) for k in stream_names(L, po, pe)}
    rc, body = encode(n, L, po, pe, streams, tmp_path)
    assert rc == CURC_OK, body
    assert body == ora.encode(str(tmp_path))
