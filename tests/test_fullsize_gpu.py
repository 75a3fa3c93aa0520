"""Stage and stream parity with the oracle at full size, on a B200.

The oracle takes minutes on the benchmark block (10M pairs x 150 bp, 3
Gbases) and on full-scale blocks of the batched workload, so it was run once
on the CPU and the SHA-256 of every stage result and stream it computed is
committed (tests/golden/fullsize_digests.json, made by
tests/golden/make_fullsize_digests.py).  Here the same seeded inputs go
through the CUDA path and every result must hash to the oracle's digest:
bit-exact at the benchmark's size."""
import hashlib
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
from tests.oracle_lib import STAGE_RESULTS, stream_dtype, stream_names  # noqa: E402

pytestmark = pytest.mark.gpu

DIGESTS = json.load(open(os.path.join(ROOT, "tests", "golden", "fullsize_digests.json")))


@pytest.fixture(scope="module")
def ctx():
    from curc_b200 import Context
    with Context(0) as c:
        c.keep_intermediates(True)
        yield c


@pytest.mark.parametrize("case", sorted(DIGESTS))
def test_fullsize_digests(ctx, case):
    import make_fullsize_digests
    spec = DIGESTS[case]
    w = make_fullsize_digests.cases()[case]()
    seqs = w.sequences()
    assert seqs.shape == (spec["reads"], spec["read_len"])
    ctx.block_run(seqs, spec["preserve_order"], spec["paired_end"])
    del seqs
    bad = []
    names = list(STAGE_RESULTS) + stream_names(spec["read_len"])
    for name in names:
        dt = STAGE_RESULTS.get(name) or stream_dtype(name)
        got = hashlib.sha256(ctx.get(name, dt).tobytes()).hexdigest()
        if got != spec["sha256"][name]:
            bad.append(name)
    assert not bad, f"{case}: differs from the oracle in {bad}"
