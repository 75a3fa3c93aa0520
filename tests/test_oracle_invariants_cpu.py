"""Invariant of the assembled pseudogenome, on the oracle (the checker).

The reference's unused self-check check_binary_ref (compress.cu:85-105),
restated: every record of the main pseudogenome names a different read, and
that read's bases equal the pseudogenome at the record's position.  It holds
at any size; here it pins the oracle's assembly on seeded cases, including
exact duplicates and periodic reads (chain cycles)."""
import numpy as np
import pytest

from curc_b200 import record_dtype
from tests.cases import CASES
from tests.oracle_lib import OracleBlock


@pytest.mark.parametrize("case", ["se100_20k", "se75_20k", "se250_8k", "pe150", "dups"])
def test_records_match_pseudogenome(case):
    seqs, po, pe = CASES[case]()
    n, L = seqs.shape
    ora = OracleBlock(seqs, po, pe)
    hq = ora.get("hq_seq")
    rec = np.frombuffer(ora.get("hq_records").tobytes(), dtype=record_dtype())
    assert len(rec) > 0
    ids = rec["read_id"].astype(np.int64)
    assert len(np.unique(ids)) == len(ids)          # no read placed twice
    assert ids.max() < n
    pos = rec["pos"].astype(np.int64)
    assert pos.min() >= 0 and pos.max() + L <= len(hq)
    # the read's bases at its position
    windows = hq[pos[:, None] + np.arange(L)[None, :]]
    assert np.array_equal(windows, seqs[ids])


@pytest.mark.parametrize("case", ["se100_20k", "se250_8k", "pe150", "dups"])
def test_oracle_results_do_not_depend_on_threads(case):
    """The oracle searches overlap passes, RefMatcher probe groups and the
    mapping in parallel but links and takes matches in order: one thread and
    eight give the same stage results and streams."""
    from tests.oracle_lib import STAGE_RESULTS, stream_dtype, stream_names
    seqs, po, pe = CASES[case]()
    one = OracleBlock(seqs, po, pe, threads=1)
    many = OracleBlock(seqs, po, pe, threads=8)
    names = list(STAGE_RESULTS.items()) + [(s, stream_dtype(s)) for s in stream_names(seqs.shape[1])]
    bad = [nm for nm, dt in names if not np.array_equal(one.get(nm, dt), many.get(nm, dt))]
    assert not bad, bad
