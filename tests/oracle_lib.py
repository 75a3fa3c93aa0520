"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so) -- the
checker for the CUDA path.  Test infrastructure only."""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"{ORACLE_SO} missing: run `make -f oracle/ref.mk REF=<reference source root> && make -C oracle REF=<reference source root>`")
        L = ctypes.CDLL(ORACLE_SO)
        L.oracle_block_new.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int]
        L.oracle_block_new.restype = ctypes.c_void_p
        L.oracle_block_new_picks.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64]
        L.oracle_block_new_picks.restype = ctypes.c_void_p
        L.oracle_block_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p),
                                       ctypes.POINTER(ctypes.c_uint64)]
        L.oracle_block_encode.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p,
                                          ctypes.POINTER(ctypes.c_void_p)]
        L.oracle_block_encode.restype = ctypes.c_uint64
        L.oracle_buf_free.argtypes = [ctypes.c_void_p]
        L.oracle_block_free.argtypes = [ctypes.c_void_p]
        L.oracle_compress_files.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                            ctypes.c_double, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        _lib = L
    return _lib


class OracleBlock:
    """One block through the oracle.  `picks`, a list of (overlap pass,
    suffix read id), replays another serialisation of the contested overlap
    runs: in that pass the suffix is visited before the others (the order a
    GPU run of the reference may take; the default is list order)."""

    def __init__(self, seqs: np.ndarray, preserve_order=False, paired_end=False, threads=8, picks=()):
        seqs = np.ascontiguousarray(seqs, dtype=np.uint8)
        n, L = seqs.shape
        self.L = L
        pk = np.ascontiguousarray(np.array(list(picks), dtype=np.uint32).reshape(-1, 2))
        self._h = lib().oracle_block_new_picks(seqs.ctypes.data, n, L, int(preserve_order), int(paired_end), threads,
                                               pk.ctypes.data, len(pk))

    def contests(self):
        """Members of contested overlap runs: rows of (pass, run, suffix,
        prefix taken in that pass or 0xFFFFFFFF), in visiting order per run."""
        return self.get("contests", np.uint32).reshape(-1, 4)

    def get(self, name, dtype=np.uint8):
        p, nb = ctypes.c_void_p(), ctypes.c_uint64()
        if lib().oracle_block_get(self._h, name.encode(), ctypes.byref(p), ctypes.byref(nb)) != 0:
            raise KeyError(name)
        if nb.value == 0:
            return np.zeros(0, dtype=dtype)
        return np.frombuffer(bytes((ctypes.c_uint8 * nb.value).from_address(p.value)), dtype=dtype)

    def encode(self, tmpdir, bsc=os.path.join(REF_DIR, "bsc")):
        out = ctypes.c_void_p()
        n = lib().oracle_block_encode(self._h, tmpdir.encode(), bsc.encode(), ctypes.byref(out))
        data = bytes((ctypes.c_uint8 * n).from_address(out.value))
        lib().oracle_buf_free(out)
        return data

    def __del__(self):
        try:
            lib().oracle_block_free(self._h)
        except Exception:
            pass


# name -> dtype of every stage result both implementations expose
STAGE_RESULTS = {
    "packed": np.uint64, "has_n": np.uint8, "sorted_ids": np.uint32,
    "next": np.uint32, "prev": np.uint32, "offset": np.uint16,
    "ref_ids": np.uint32, "unmatch_ids": np.uint32,
    "hq_seq": np.uint8, "hq_records": np.uint8,
    "map_mm": np.uint8, "map_strand": np.uint8, "map_pos": np.uint64,
}

# every stream of a block (before entropy coding), both implementations
STREAMS = {
    "strand": np.uint8, "mis_cnt": np.uint8, "mis_base": np.uint8, "decoder_table": np.uint8,
    "read_off": np.uint16, "unmap_read_off": np.uint16, "unmap_n_read_off": np.uint16,
    "pe_order": np.uint32, "id_to_pos": np.uint64,
    "ref": np.uint8, "unmap_ref": np.uint8, "unmap_n_ref": np.uint8,
    "ref_off": np.uint8, "ref_len_map": np.uint8, "unmap_ref_off": np.uint8, "unmap_ref_len": np.uint8,
    "unmap_n_ref_off": np.uint8, "unmap_n_ref_len": np.uint8, "sizes": np.uint64,
}


def stream_names(read_len):
    return list(STREAMS) + [f"mis_off_{m}" for m in range(1, read_len // 5 + 1)]


def stream_dtype(name):
    return np.uint16 if name.startswith("mis_off_") else STREAMS[name]


def _setup_decoders():
    L = lib()
    L.oracle_read_compressed.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]
    L.oracle_read_compressed.restype = ctypes.c_uint64
    L.oracle_decode_ref.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_char_p,
                                    ctypes.POINTER(ctypes.c_void_p)]
    L.oracle_decode_ref.restype = ctypes.c_uint64
    L.oracle_decode_offsets.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                        ctypes.c_void_p]
    L.oracle_decode_offsets.restype = ctypes.c_uint64
    return L


def read_compressed(payload: bytes) -> bytes:
    """Raw bytes of a writeCompressed payload (LZMA / PPMd7 container)."""
    L = _setup_decoders()
    out = ctypes.c_void_p()
    n = L.oracle_read_compressed(payload, len(payload), ctypes.byref(out))
    data = bytes((ctypes.c_uint8 * n).from_address(out.value)) if n else b""
    L.oracle_buf_free(out)
    return data


def decode_ref(payload: bytes, total: int, tmpdir: str) -> bytes:
    L = _setup_decoders()
    out = ctypes.c_void_p()
    n = L.oracle_decode_ref(payload, len(payload), total, tmpdir.encode(), ctypes.byref(out))
    data = bytes((ctypes.c_uint8 * n).from_address(out.value))
    L.oracle_buf_free(out)
    return data


def decode_offsets(payload: bytes, read_len: int, m: int, records: int) -> np.ndarray:
    L = _setup_decoders()
    width = 2 if m == 1 else (3 if m == 2 else m + 2)
    out = np.zeros(records * width, dtype=np.uint16)
    L.oracle_decode_offsets(payload, len(payload), read_len, m, records, out.ctypes.data)
    return out
