"""curc_pack_split_noalloc: packing and N split without device allocation.

The entry point exists for callers that cannot call cudaMalloc: a host
application that manages all device memory through its own pool, or one that
cannot take the device synchronisation an allocation may cause.  It keeps its
scratch in a fixed array inside the library instead of a context arena.

This test calls it several times in a row through the C-ABI and checks each
result bit for bit against the regular entry point curc_pack_device: the
packed words and N flags must be equal, and the two id lists must be exactly
the reads without / with an N flag in ascending order.  Integer outputs, so
the tolerance is zero.  The calls cover a second call smaller than the first
(stale scratch from the first would show), a call of more than 1024 tiles of
2048 reads (the scan's path where one thread sums several tiles), and input
that starts one byte past an aligned address (the packing's path without
bulk copies).  Around one call the device's free memory is read: it must not
change, which is the property the entry point exists for.  The test
allocates its own buffers beforehand; only the entry point must not."""
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


class _Call:
    """Device input (optionally starting `shift` bytes into its buffer) and
    output buffers of one call, all allocated up front."""

    def __init__(self, seed, n, rl, n_rate, shift=0):
        import torch
        self.n, self.rl = n, rl
        self.seqs = _reads(seed, n, rl, n_rate)
        self.buf = torch.zeros(n * rl + 16, dtype=torch.uint8, device="cuda")
        self.buf[shift:shift + n * rl] = torch.from_numpy(self.seqs.reshape(-1).copy()).cuda()
        self.ptr = self.buf.data_ptr() + shift
        w = (rl + 31) // 32
        self.packed = torch.full((n * w,), -1, dtype=torch.int64, device="cuda")
        self.has_n = torch.full((n,), 7, dtype=torch.uint8, device="cuda")
        self.rid = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        self.nid = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        self.counts = torch.full((2,), -1, dtype=torch.int32, device="cuda")

    def run(self, L, noalloc):
        rc = noalloc(0, self.ptr, self.n, self.rl, self.packed.data_ptr(), self.has_n.data_ptr(),
                     self.rid.data_ptr(), self.nid.data_ptr(), self.counts.data_ptr(), None)
        assert rc == 0, L.curc_last_error(None).decode()

    def check(self, ctx):
        import torch
        n, rl = self.n, self.rl
        w = (rl + 31) // 32
        ref_packed = torch.empty(n * w, dtype=torch.int64, device="cuda")
        ref_hn = torch.empty(n, dtype=torch.uint8, device="cuda")
        ctx.pack_device(self.ptr, n, rl, ref_packed.data_ptr(), ref_hn.data_ptr())
        torch.cuda.synchronize()
        ref_hn = ref_hn.cpu().numpy()
        counts = self.counts.cpu().numpy()
        assert np.array_equal(self.packed.cpu().numpy(), ref_packed.cpu().numpy())
        assert np.array_equal(self.has_n.cpu().numpy(), ref_hn)
        exp_r = np.flatnonzero(ref_hn == 0)
        exp_n = np.flatnonzero(ref_hn != 0)
        assert 0 < len(exp_n) < n
        assert counts[0] == len(exp_r) and counts[1] == len(exp_n)
        assert np.array_equal(self.rid.cpu().numpy()[:counts[0]], exp_r)
        assert np.array_equal(self.nid.cpu().numpy()[:counts[1]], exp_n)


def test_noalloc_matches_regular_entry_point_on_calls_in_a_row():
    import torch
    from curc_b200 import Context

    L, noalloc = _bind()
    calls = [_Call(1, 30_011, 100, 0.002), _Call(2, 4_097, 151, 0.004), _Call(3, 2_200_000, 100, 0.0005),
             _Call(4, 9_999, 75, 0.003, shift=1)]
    torch.cuda.synchronize()
    calls[0].run(L, noalloc)  # the first call on the device loads the module and sets up the scratch address
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    calls[1].run(L, noalloc)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"device free memory changed by {free0 - free1} bytes during a call"
    for c in calls[2:]:
        c.run(L, noalloc)
    torch.cuda.synchronize()
    with Context(0) as ctx:
        for c in calls:
            c.check(ctx)


def test_noalloc_rejects_calls_above_its_scratch_limit():
    L, noalloc = _bind()
    too_many = (1 << 27) + 1
    rc = noalloc(0, 1, too_many, 100, 1, 1, 1, 1, 1, None)
    assert rc != 0
    assert "2^27" in L.curc_last_error(None).decode()
