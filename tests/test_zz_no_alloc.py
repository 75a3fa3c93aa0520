"""curc_pack_split_noalloc: packing and N split without device allocation.

The entry point exists for callers that cannot call cudaMalloc: a host
application that manages all device memory through its own pool, or one that
cannot take the device synchronisation an allocation may cause.  It keeps its
scratch in a fixed array inside the library instead of a context arena.

This test calls it twice in a row through the C-ABI (the second call smaller
than the first, so stale scratch from the first call would show) and checks
each result bit for bit against the regular entry point curc_pack_device:
the packed words and N flags must be equal, and the two id lists must be
exactly the reads without / with an N flag in ascending order.  Integer
outputs, so the tolerance is zero.  The test allocates its own buffers; only
the entry point under test must not."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind():
    from curc_b200 import lib
    L = lib()
    f = L.curc_pack_split_noalloc
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint16, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return L, f


def _reads(seed, n, read_len, n_rate):
    from curc_b200 import synth
    rng = np.random.default_rng(seed)
    g = synth.random_genome(rng, 200_000)
    return synth.sample_single(rng, g, n, read_len, 0.002, n_rate)


def test_noalloc_matches_regular_entry_point_on_two_calls():
    import torch
    from curc_b200 import Context

    L, noalloc = _bind()
    cases = [(1, 30_011, 100, 0.002), (2, 4_097, 151, 0.004)]
    results = []
    for seed, n, rl, n_rate in cases:
        seqs = _reads(seed, n, rl, n_rate)
        d_seq = torch.from_numpy(seqs.reshape(-1).copy()).cuda()
        w = (rl + 31) // 32
        packed = torch.full((n * w,), -1, dtype=torch.int64, device="cuda")
        has_n = torch.full((n,), 7, dtype=torch.uint8, device="cuda")
        rid = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        nid = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        counts = torch.full((2,), -1, dtype=torch.int32, device="cuda")
        rc = noalloc(0, d_seq.data_ptr(), n, rl, packed.data_ptr(), has_n.data_ptr(), rid.data_ptr(),
                     nid.data_ptr(), counts.data_ptr(), None)
        assert rc == 0, L.curc_last_error(None).decode()
        torch.cuda.synchronize()
        results.append((seqs, d_seq, packed.cpu().numpy(), has_n.cpu().numpy(), rid.cpu().numpy(),
                        nid.cpu().numpy(), counts.cpu().numpy()))

    with Context(0) as ctx:
        for (seqs, d_seq, packed, has_n, rid, nid, counts), (_, n, rl, _r) in zip(results, cases):
            w = (rl + 31) // 32
            ref_packed = torch.empty(n * w, dtype=torch.int64, device="cuda")
            ref_hn = torch.empty(n, dtype=torch.uint8, device="cuda")
            ctx.pack_device(d_seq.data_ptr(), n, rl, ref_packed.data_ptr(), ref_hn.data_ptr())
            torch.cuda.synchronize()
            ref_hn = ref_hn.cpu().numpy()
            assert np.array_equal(packed, ref_packed.cpu().numpy())
            assert np.array_equal(has_n, ref_hn)
            exp_r = np.flatnonzero(ref_hn == 0)
            exp_n = np.flatnonzero(ref_hn != 0)
            assert 0 < len(exp_n) < n
            assert counts[0] == len(exp_r) and counts[1] == len(exp_n)
            assert np.array_equal(rid[:counts[0]], exp_r)
            assert np.array_equal(nid[:counts[1]], exp_n)


def test_noalloc_rejects_calls_above_its_scratch_limit():
    L, noalloc = _bind()
    too_many = (1 << 27) + 1
    rc = noalloc(0, 1, too_many, 100, 1, 1, 1, 1, 1, None)
    assert rc != 0
    assert "2^27" in L.curc_last_error(None).decode()
