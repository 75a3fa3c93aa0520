"""ctypes binding of libcurc_b200.so (include/curc_b200.h).

The CUDA library is the only implementation: there is no Python or CPU
fallback, and loading fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcurc_b200.so")

_lib = None


BLOCK_DONE = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C curc_b200 REF=<reference source root>` "
                               "(or __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        c_p, c_u64, c_int = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int
        L.curc_ctx_create.argtypes = [c_int, ctypes.POINTER(c_p)]
        L.curc_ctx_create_deferred.argtypes = [c_int, ctypes.POINTER(c_p)]
        L.curc_ctx_wait.argtypes = [c_p]
        L.curc_ctx_destroy.argtypes = [c_p]
        L.curc_ctx_destroy.restype = None
        L.curc_last_error.argtypes = [c_p]
        L.curc_last_error.restype = ctypes.c_char_p
        L.curc_pack_device.argtypes = [c_p, c_p, c_u64, ctypes.c_uint16, c_p, c_p, c_p]
        L.curc_block_run.argtypes = [c_p, c_p, c_u64, ctypes.c_uint16, c_int, c_int]
        L.curc_block_run_device.argtypes = [c_p, c_p, c_u64, ctypes.c_uint16, c_int, c_int]
        L.curc_block_get.argtypes = [c_p, ctypes.c_char_p, ctypes.POINTER(c_p), ctypes.POINTER(c_u64)]
        L.curc_block_stage_ms.argtypes = [c_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_float)]
        L.curc_ctx_keep_intermediates.argtypes = [c_p, c_int]
        L.curc_ctx_trim.argtypes = [c_p]
        L.curc_ctx_set_mismatch_model.argtypes = [c_p, c_p, c_u64]
        L.curc_ctx_set_tuning.argtypes = [c_p, c_p]
        L.curc_ctx_get_tuning.argtypes = [c_p, c_p]
        L.curc_ctx_use_tuning_cache.argtypes = [c_p, ctypes.c_char_p]
        L.curc_autotune.argtypes = [c_p, c_p, c_u64, ctypes.c_uint16, c_int, c_int, ctypes.c_char_p,
                                    ctypes.POINTER(c_int)]
        L.curc_kernel_launches.argtypes = []
        L.curc_batch_submit.argtypes = [c_p, c_p, c_u64, ctypes.c_uint16, c_int, c_int,
                                        ctypes.POINTER(ctypes.c_uint32)]
        L.curc_batch_drain.argtypes = [c_p, BLOCK_DONE, c_p]
        L.curc_batch_workers.argtypes = [c_p, c_int]
        L.curc_learn_create.argtypes = [c_int, ctypes.POINTER(c_p)]
        L.curc_learn_destroy.argtypes = [c_p]
        L.curc_learn_error.argtypes = [c_p]
        L.curc_learn_error.restype = ctypes.c_char_p
        L.curc_learn_add_block.argtypes = [c_p, c_p]
        L.curc_learn_anchors.argtypes = [c_p]
        L.curc_learn_anchors.restype = c_u64
        L.curc_learn_train.argtypes = [c_p, c_int, c_int, ctypes.c_float, c_u64, ctypes.POINTER(ctypes.c_float)]
        L.curc_learn_model.argtypes = [c_p, ctypes.POINTER(c_p), ctypes.POINTER(c_u64)]
        L.curc_learn_set_model.argtypes = [c_p, c_p, c_u64]
        L.curc_learn_encode.argtypes = [c_p, c_p, ctypes.POINTER(c_p), ctypes.POINTER(c_u64)]
        L.curc_learn_decode_check.argtypes = [c_p, c_p, c_p, c_u64, ctypes.POINTER(c_int)]
        L.curc_learn_infer_check.argtypes = [c_p, c_p, ctypes.POINTER(c_u64), ctypes.POINTER(c_u64)]
        L.curc_learn_param_count.argtypes = []
        L.curc_learn_param_count.restype = c_u64
        L.curc_learn_grad.argtypes = [c_p, c_p, c_p, c_p, c_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_float), c_p]
        L.curc_plain_mismatch_bytes.argtypes = [c_p, c_p]
        L.curc_mismatch_general_bytes.argtypes = [c_p, ctypes.c_char_p, ctypes.c_char_p, c_p]
        L.curc_compress_files.argtypes = [c_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double,
                                          c_int, c_int, c_int, ctypes.c_char_p, ctypes.c_char_p,
                                          ctypes.POINTER(c_u64), ctypes.POINTER(ctypes.c_uint32)]
        L.curc_decompress_file.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, c_int,
                                           ctypes.POINTER(c_u64)]
        L.curc_archive_info.argtypes = [ctypes.c_char_p, ctypes.POINTER(c_int), ctypes.POINTER(c_int),
                                        ctypes.POINTER(ctypes.c_uint16), ctypes.POINTER(ctypes.c_uint32),
                                        ctypes.POINTER(c_u64), ctypes.POINTER(ctypes.c_uint32)]
        L.curc_fastq_blocks.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double, FASTQ_BLOCK, c_p,
                                        ctypes.POINTER(c_u64), ctypes.POINTER(ctypes.c_uint32)]
        L.curc_kernel_launches.restype = ctypes.c_uint64
        _lib = L
    return _lib


def kernel_launches() -> int:
    return int(lib().curc_kernel_launches())


class CurcError(RuntimeError):
    pass


FASTQ_BLOCK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64,
                               ctypes.c_uint16)


def archive_info(archive: str) -> dict:
    """Layout of a .curc archive without decoding it: flags, read length,
    and per block its body size and read count."""
    po, pe, L, nb = ctypes.c_int(), ctypes.c_int(), ctypes.c_uint16(), ctypes.c_uint32()
    sizes, reads = (ctypes.c_uint64 * 256)(), (ctypes.c_uint32 * 256)()
    rc = lib().curc_archive_info(archive.encode(), ctypes.byref(po), ctypes.byref(pe), ctypes.byref(L),
                                 ctypes.byref(nb), sizes, reads)
    if rc != 0:
        raise CurcError(f"curc_archive_info: {lib().curc_last_error(None).decode()} (code {rc})")
    return {"preserve_order": bool(po.value), "paired_end": bool(pe.value), "read_len": L.value,
            "block_bytes": [int(sizes[i]) for i in range(nb.value)],
            "block_reads": [int(reads[i]) for i in range(nb.value)]}


def fastq_blocks(f1: str, f2: str | None = None, block_ratio: float = 1.0) -> list:
    """The reference's block split of FASTQ file(s), host only: a list of
    (n, L) uint8 arrays of ASCII reads in block order (mates interleaved)."""
    out = []

    def cb(_user, _index, seqs, n, L):
        out.append(np.frombuffer(ctypes.string_at(seqs, n * L), dtype=np.uint8).reshape(n, L).copy() if n
                   else np.zeros((0, L), dtype=np.uint8))
        return 0

    fn = FASTQ_BLOCK(cb)
    rc = lib().curc_fastq_blocks(f1.encode(), f2.encode() if f2 else None, block_ratio, fn, None, None, None)
    if rc != 0:
        raise CurcError(f"curc_fastq_blocks: {lib().curc_last_error(None).decode()} (code {rc})")
    return out


def decompress_file(archive: str, out_prefix: str, bsc: str | None = None, tmpdir: str = "/tmp",
                    threads: int = 0) -> int:
    """`curc -d`: a .curc archive to <out_prefix>.seq (single end) or
    <out_prefix>_1.seq / _2.seq (paired end), byte for byte the reference
    decoder's output.  Host only (no GPU).  Returns the read count."""
    if bsc is None:
        bsc = os.path.join(os.path.dirname(LIB_PATH), "_build", "bsc")
    n = ctypes.c_uint64()
    rc = lib().curc_decompress_file(archive.encode(), out_prefix.encode(), bsc.encode(), tmpdir.encode(), threads,
                                    ctypes.byref(n))
    if rc != 0:
        raise CurcError(f"curc_decompress_file: {lib().curc_last_error(None).decode()} (code {rc})")
    return n.value


class Context:
    """One CUDA stream and device arena on one GPU (curc_ctx)."""

    def __init__(self, device: int = 0, deferred: bool = False):
        """deferred: the CUDA set-up runs on a thread of its own
        (curc_ctx_create_deferred); compress_files parses its input
        meanwhile, every other call waits for it."""
        self._h = ctypes.c_void_p()
        create = lib().curc_ctx_create_deferred if deferred else lib().curc_ctx_create
        rc = create(device, ctypes.byref(self._h))
        if rc != 0:
            raise CurcError(f"curc_ctx_create: {lib().curc_last_error(None).decode()}")

    def wait(self):
        """Waits for a deferred context's CUDA set-up (curc_ctx_wait)."""
        self._check(lib().curc_ctx_wait(self._h), "curc_ctx_wait")

    def _check(self, rc: int, what: str):
        if rc != 0:
            raise CurcError(f"{what}: {lib().curc_last_error(self._h).decode()} (code {rc})")

    def close(self):
        if self._h:
            lib().curc_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def block_run(self, seqs: np.ndarray, preserve_order: bool = False, paired_end: bool = False):
        """seqs: (n, L) uint8 ASCII reads in block order, host memory."""
        seqs = np.ascontiguousarray(seqs, dtype=np.uint8)
        n, L = seqs.shape
        self._check(lib().curc_block_run(self._h, seqs.ctypes.data, n, L, int(preserve_order), int(paired_end)),
                    "curc_block_run")

    def block_run_device(self, ptr: int, n: int, L: int, preserve_order=False, paired_end=False):
        self._check(lib().curc_block_run_device(self._h, ctypes.c_void_p(ptr), n, L, int(preserve_order),
                                                int(paired_end)), "curc_block_run_device")

    def get(self, name: str, dtype=np.uint8) -> np.ndarray:
        p, nb = ctypes.c_void_p(), ctypes.c_uint64()
        self._check(lib().curc_block_get(self._h, name.encode(), ctypes.byref(p), ctypes.byref(nb)),
                    f"curc_block_get({name})")
        if nb.value == 0:
            return np.zeros(0, dtype=dtype)
        buf = (ctypes.c_uint8 * nb.value).from_address(p.value)
        return np.frombuffer(bytes(buf), dtype=dtype)

    def keep_intermediates(self, keep: bool):
        self._check(lib().curc_ctx_keep_intermediates(self._h, int(keep)), "curc_ctx_keep_intermediates")

    def trim(self):
        """Frees the device memory the context keeps between blocks (arena,
        batch pipelines); the last run's results stay readable."""
        self._check(lib().curc_ctx_trim(self._h), "curc_ctx_trim")

    def stage_ms(self, stage: str) -> float:
        v = ctypes.c_float()
        self._check(lib().curc_block_stage_ms(self._h, stage.encode(), ctypes.byref(v)), "curc_block_stage_ms")
        return float(v.value)

    def batch_submit(self, seqs: np.ndarray, preserve_order: bool = False, paired_end: bool = False) -> int:
        """Queue a block ((n, L) uint8 ASCII, host memory kept alive by the
        caller until the drain returns); returns its ticket."""
        assert seqs.flags["C_CONTIGUOUS"] and seqs.dtype == np.uint8
        n, L = seqs.shape
        t = ctypes.c_uint32()
        self._check(lib().curc_batch_submit(self._h, ctypes.c_void_p(seqs.ctypes.data), n, L, int(preserve_order),
                                            int(paired_end), ctypes.byref(t)), "curc_batch_submit")
        return t.value

    def batch_workers(self, workers: int):
        """Number of block pipelines of the drain (1..16, default 2)."""
        self._check(lib().curc_batch_workers(self._h, workers), "curc_batch_workers")

    def batch_drain(self, on_block=None):
        """Run the queued blocks (those of at least 2^28 bases first, one at a
        time with the next one's reads already crossing to the device; the
        rest on concurrent pipelines); on_block(ticket) is called after each,
        in completion order, while get() returns that block's results."""
        err = []

        def cb(_user, ticket):
            try:
                if on_block:
                    on_block(ticket)
                return 0
            except Exception as e:  # stop the drain, re-raised below
                err.append(e)
                return 1

        fn = BLOCK_DONE(cb)
        rc = lib().curc_batch_drain(self._h, fn, None)
        if err:
            raise err[0]
        self._check(rc, "curc_batch_drain")

    def compress_files(self, files, archive: str, block_ratio: float = 1.0, preserve_order: bool = False,
                       bsc: str = "", tmpdir: str = "/tmp", flzma2_level: int = 10, flzma2_threads: int = 16):
        """`curc -c` through the library: FASTQ file(s) to a .curc archive.
        Returns (reads, blocks)."""
        reads, blocks = ctypes.c_uint64(), ctypes.c_uint32()
        f2 = files[1].encode() if len(files) > 1 else None
        self._check(lib().curc_compress_files(self._h, files[0].encode(), f2, archive.encode(), block_ratio,
                                              int(preserve_order), flzma2_level, flzma2_threads, bsc.encode(),
                                              tmpdir.encode(), ctypes.byref(reads), ctypes.byref(blocks)),
                    "curc_compress_files")
        return reads.value, blocks.value

    TUNING_KNOBS = ("table_factor", "bitmap_bits", "check_every", "map_threads", "fm_loop")

    def tuning(self) -> dict:
        k = (ctypes.c_int32 * len(self.TUNING_KNOBS))()
        self._check(lib().curc_ctx_get_tuning(self._h, k), "curc_ctx_get_tuning")
        return dict(zip(self.TUNING_KNOBS, list(k)))

    def set_tuning(self, **knobs):
        cur = self.tuning()
        cur.update(knobs)
        k = (ctypes.c_int32 * len(self.TUNING_KNOBS))(*[cur[n] for n in self.TUNING_KNOBS])
        self._check(lib().curc_ctx_set_tuning(self._h, k), "curc_ctx_set_tuning")

    def autotune(self, ptr: int, n: int, L: int, preserve_order=False, paired_end=False, cache: str | None = None):
        """Autotunes on a block already in device memory; returns (tuning,
        whether it came from the cache)."""
        fc = ctypes.c_int(0)
        self._check(lib().curc_autotune(self._h, ctypes.c_void_p(ptr), n, L, int(preserve_order), int(paired_end),
                                        cache.encode() if cache else None, ctypes.byref(fc)), "curc_autotune")
        return self.tuning(), bool(fc.value)

    def use_tuning_cache(self, path: str | None):
        """Per-block tuning from an autotune cache file (None: stop)."""
        self._check(lib().curc_ctx_use_tuning_cache(self._h, path.encode() if path else None),
                    "curc_ctx_use_tuning_cache")

    def set_mismatch_model(self, model: bytes | None):
        """Learned mode of compress_files (model bytes from Learner.model()),
        or plain mode with None."""
        if model:
            self._check(lib().curc_ctx_set_mismatch_model(self._h, model, len(model)), "curc_ctx_set_mismatch_model")
        else:
            self._check(lib().curc_ctx_set_mismatch_model(self._h, None, 0), "curc_ctx_set_mismatch_model")

    def pack_device(self, seqs_ptr: int, n: int, L: int, packed_ptr: int, has_n_ptr: int, stream: int = 0):
        self._check(lib().curc_pack_device(self._h, ctypes.c_void_p(seqs_ptr), n, L, ctypes.c_void_p(packed_ptr),
                                           ctypes.c_void_p(has_n_ptr), ctypes.c_void_p(stream)), "curc_pack_device")


class Learner:
    """The learned mismatch coder (curc_learn_* in include/curc_b200.h)."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        rc = lib().curc_learn_create(device, ctypes.byref(h))
        if rc != 0:
            raise CurcError(f"curc_learn_create: {lib().curc_last_error(None).decode()}")
        self._h = h

    def _check(self, rc: int, what: str):
        if rc != 0:
            raise CurcError(f"{what}: {lib().curc_learn_error(self._h).decode()}")

    def close(self):
        if self._h:
            lib().curc_learn_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add_block(self, ctx: "Context"):
        self._check(lib().curc_learn_add_block(self._h, ctx.handle), "curc_learn_add_block")

    @property
    def anchors(self) -> int:
        return int(lib().curc_learn_anchors(self._h))

    def train(self, epochs=2, batch=4096, lr=2e-3, seed=1) -> float:
        loss = ctypes.c_float()
        self._check(lib().curc_learn_train(self._h, epochs, batch, lr, seed, ctypes.byref(loss)), "curc_learn_train")
        return float(loss.value)

    def model(self) -> bytes:
        p, n = ctypes.c_void_p(), ctypes.c_uint64()
        self._check(lib().curc_learn_model(self._h, ctypes.byref(p), ctypes.byref(n)), "curc_learn_model")
        return ctypes.string_at(p.value, n.value)

    def set_model(self, blob: bytes):
        self._check(lib().curc_learn_set_model(self._h, blob, len(blob)), "curc_learn_set_model")

    def encode(self, ctx: "Context") -> bytes:
        p, n = ctypes.c_void_p(), ctypes.c_uint64()
        self._check(lib().curc_learn_encode(self._h, ctx.handle, ctypes.byref(p), ctypes.byref(n)),
                    "curc_learn_encode")
        return ctypes.string_at(p.value, n.value)

    def infer_check(self, ctx: "Context"):
        """(anchors, anchors whose tensor-core frequencies differ from the
        host model's) over the context's last block."""
        n, bad = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(lib().curc_learn_infer_check(self._h, ctx.handle, ctypes.byref(n), ctypes.byref(bad)),
                    "curc_learn_infer_check")
        return n.value, bad.value

    def decode_check(self, ctx: "Context", stream: bytes) -> bool:
        ok = ctypes.c_int()
        self._check(lib().curc_learn_decode_check(self._h, ctx.handle, stream, len(stream), ctypes.byref(ok)),
                    "curc_learn_decode_check")
        return ok.value == 1

    def grad(self, params: np.ndarray, x: np.ndarray, tb: np.ndarray, tg: np.ndarray):
        params = np.ascontiguousarray(params, dtype=np.float32)
        x = np.ascontiguousarray(x, dtype=np.float32)
        tb = np.ascontiguousarray(tb, dtype=np.int8)
        tg = np.ascontiguousarray(tg, dtype=np.int8)
        g = np.zeros_like(params)
        loss = ctypes.c_float()
        self._check(lib().curc_learn_grad(self._h, params.ctypes.data, x.ctypes.data, tb.ctypes.data, tg.ctypes.data,
                                          x.shape[0], ctypes.byref(loss), g.ctypes.data), "curc_learn_grad")
        return float(loss.value), g


def learn_param_count() -> int:
    return int(lib().curc_learn_param_count())


def plain_mismatch_bytes(ctx: "Context"):
    """Coded sizes (counts, bases, offsets) of the last block's mismatch
    streams with the plain coders."""
    out = (ctypes.c_uint64 * 3)()
    rc = lib().curc_plain_mismatch_bytes(ctx.handle, out)
    if rc != 0:
        raise CurcError(f"curc_plain_mismatch_bytes: {lib().curc_last_error(ctx.handle).decode()}")
    return tuple(int(v) for v in out)


def general_mismatch_bytes(ctx: "Context", bsc: str, tmpdir: str = "/tmp"):
    """(fast-lzma2 level 10, libbsc) bytes of the last block's mismatch
    streams (counts, bases, offsets, each coded on its own)."""
    out = (ctypes.c_uint64 * 2)()
    rc = lib().curc_mismatch_general_bytes(ctx.handle, bsc.encode(), tmpdir.encode(), out)
    if rc != 0:
        raise CurcError(f"curc_mismatch_general_bytes: {lib().curc_last_error(ctx.handle).decode()}")
    return int(out[0]), int(out[1])
