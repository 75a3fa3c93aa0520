"""Stage-by-stage parity of the CUDA path against the CPU oracle.

Every comparison is bit-exact: the path is integer/byte work only."""
import numpy as np
import pytest

from tests.cases import CASES
from tests.oracle_lib import OracleBlock, STAGE_RESULTS, stream_dtype, stream_names

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from curc_b200 import Context
    with Context(0) as c:
        yield c


def _first_diff(a, b):
    n = min(len(a), len(b))
    d = np.nonzero(a[:n] != b[:n])[0]
    return int(d[0]) if len(d) else n


@pytest.mark.parametrize("case", sorted(CASES))
def test_stage_parity(ctx, case):
    seqs, po, pe = CASES[case]()
    ora = OracleBlock(seqs, po, pe)
    ctx.block_run(seqs, po, pe)
    bad = []
    for name, dt in STAGE_RESULTS.items():
        a = ctx.get(name, dt)
        b = ora.get(name, dt)
        if a.shape != b.shape or not np.array_equal(a, b):
            bad.append(f"{name}: gpu {a.shape} oracle {b.shape} first diff at {_first_diff(a, b)}")
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("case", sorted(CASES))
def test_stream_parity(ctx, case):
    seqs, po, pe = CASES[case]()
    ora = OracleBlock(seqs, po, pe)
    ctx.block_run(seqs, po, pe)
    bad = []
    for name in stream_names(seqs.shape[1]):
        dt = stream_dtype(name)
        a, b = ctx.get(name, dt), ora.get(name, dt)
        if a.shape != b.shape or not np.array_equal(a, b):
            bad.append(f"{name}: gpu {a.shape} oracle {b.shape} first diff at {_first_diff(a, b)}")
    assert not bad, "\n".join(bad)
