"""Finds, for each golden archive, the contested overlap links that the
reference's GPU run resolved differently from the oracle's list order, and
writes them to tests/golden/contested_links.json.  CPU only.

In one overlap pass (compress.cu:1473-1532) every suffix read is a GPU
thread; suffixes whose [off, L) equal the same run of prefixes race for the
run's free prefixes with atomicCAS (compress.cu:1518).  The oracle lets them
take prefixes in list order.  Any other serialisation is an equally valid
run of the reference, so an archive of the reference is explained when some
other visiting order of a few contested runs makes the oracle write it byte
for byte.  The search:

1. while the joined pseudogenome stream differs, try each suffix that did
   not win its contested run as the run's first visitor and keep the pick
   that lengthens the common prefix with the reference's stream most;
2. then, for each pair of adjacent records whose mismatch counts are
   swapped (two reads at one position, one exact and one with mismatches),
   pick the loser of the contested run that holds both reads;
3. stop when the archive is identical, or when no pick helps (the case is
   then recorded with the streams that still differ).

    python tests/golden/find_contested_links.py [--cases a,b]
"""
import argparse
import concurrent.futures as cf
import json
import multiprocessing
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_golden  # noqa: E402
from tests.archive import split_archive  # noqa: E402
from tests.oracle_lib import OracleBlock, decode_ref, read_compressed  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")
INVALID = 0xFFFFFFFF


def archive_of(w, picks):
    o = OracleBlock(w.sequences(), w.preserve_order, w.mate2 is not None, picks=picks)
    with tempfile.TemporaryDirectory() as td:
        body = o.encode(td)
    hdr = bytes([int(w.preserve_order), int(w.mate2 is not None), w.read_len & 255, w.read_len >> 8, 1])
    return o, hdr + body


def joined_ref(block):
    with tempfile.TemporaryDirectory() as td:
        return np.frombuffer(decode_ref(block["ref"], sum(block["sizes"]), td), np.uint8)


def common_prefix(a, b):
    n = min(len(a), len(b))
    d = np.nonzero(a[:n] != b[:n])[0]
    return int(d[0]) if len(d) else n


def _score(args):
    name, picks, ref_joined = args
    w = make_golden.CASES[name]()
    _, data = archive_of(w, picks)
    return picks, common_prefix(joined_ref(split_archive(data)["blocks"][0]), ref_joined)


def search(name, pool):
    w = make_golden.CASES[name]()
    golden = open(os.path.join(GOLDEN, name + ".curc"), "rb").read()
    gb = split_archive(golden)["blocks"][0]
    g_ref = joined_ref(gb)
    g_cnt = np.frombuffer(read_compressed(gb["mismatch_count"]), np.uint8)
    picks = []
    while True:
        o, data = archive_of(w, picks)
        if data == golden:
            return picks, []
        b = split_archive(data)["blocks"][0]
        if common_prefix(joined_ref(b), g_ref) < max(len(g_ref), len(joined_ref(b))):
            c = o.contests()
            base = common_prefix(joined_ref(b), g_ref)
            cands = [picks + [(int(p), int(s))] for p, _, s, pr in c if pr == INVALID and (int(p), int(s)) not in picks]
            best = max(pool.map(_score, [(name, cd, g_ref) for cd in cands]), key=lambda t: t[1], default=(None, base))
            if best[1] <= base:
                return picks, sorted(k for k in gb if b[k] != gb[k])
            picks = best[0]
            continue
        # pseudogenomes equal: swapped mismatch counts of records at one position
        cnt = o.get("mis_cnt")
        rec = o.get("records").reshape(-1, 16)
        rid = rec[:, 0:4].copy().view(np.uint32).ravel()
        c = o.contests()
        added = False
        if len(cnt) == len(g_cnt):
            d = np.nonzero(cnt != g_cnt)[0]
            for i in d:
                if i + 1 < len(cnt) and cnt[i] == g_cnt[i + 1] and cnt[i + 1] == g_cnt[i]:
                    x, y = int(rid[i]), int(rid[i + 1])
                    for p, run in {(int(r[0]), int(r[1])) for r in c if int(r[2]) in (x, y)}:
                        members = [int(r[2]) for r in c if int(r[0]) == p and int(r[1]) == run]
                        if x in members and y in members:
                            loser = y if members.index(x) < members.index(y) else x
                            if (p, loser) not in picks:
                                picks.append((p, loser))
                                added = True
        if not added:
            return picks, sorted(k for k in gb if b[k] != gb[k])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", default=",".join(sorted(make_golden.CASES)))
    ap.add_argument("--out", default=os.path.join(GOLDEN, "contested_links.json"))
    a = ap.parse_args()
    out = json.load(open(a.out)) if os.path.exists(a.out) else {}
    with cf.ProcessPoolExecutor(8, mp_context=multiprocessing.get_context("spawn")) as pool:
        for name in a.cases.split(","):
            picks, still = search(name, pool)
            w = make_golden.CASES[name]()
            o, _ = archive_of(w, [])
            c = o.contests()
            runs = {(int(r[0]), int(r[1])) for r in c}
            entry = {"picks": [list(p) for p in picks], "contested_runs": len(runs), "still_differ": still}
            out[name] = {**out.get(name, {}), **entry}
            print(name, entry, flush=True)
    json.dump(out, open(a.out, "w"), indent=1)


if __name__ == "__main__":
    main()
