#!/usr/bin/env python
"""Benchmark of the B200 pseudogenome path on the paired-end 150 bp workload.

Workload (seeded synthetic, no public dataset): 10M read pairs x 150 bp
(3 Gbases) from a 50 Mbp genome at 40% GC, 5% of it covered by 1-5 kbp
repeat copies at 1% divergence, insert size Normal(400, 50), 0.2%
substitutions, 0.01% N, --preserve_order, block_ratio 1 (one block).

One step = one block through the whole device path (pack ... repeat removal),
streams returned to the host.  `value` is Mbases/s with the ASCII reads
already in HBM (CUDA events).  `e2e` is the whole `curc -c` a user runs: the
product binary, one process per step, from the FASTQ files to the closed
archive (parse, copies to and from the device, device path, stream coders,
archive write) -- the same work, on the same files, that the reference arm
times for the reference's own `curc -c`.  With --ref-sample-pairs both
binaries are also timed on the first pairs of those files
(`e2e_same_sample`).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
    python bench.py --impl reference --ref-sample-pairs 1000000   # the reference on a sample

Under torchrun every rank compresses its own block (independent blocks, no
collective: weak scaling); the time is the max over ranks.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
METRIC = "Mbases/s on 1 B200, batched vs plain; bits/base learned vs plain; lossless"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--pairs", type=int, default=10_000_000)
    ap.add_argument("--genome", type=int, default=50_000_000)
    ap.add_argument("--cpu-sample-pairs", type=int, default=300_000,
                    help="pairs of the CPU-baseline sample, drawn at the workload's coverage (genome scaled alike)")
    ap.add_argument("--ref-sample-pairs", type=int, default=0,
                    help="reference arm: time the first pairs of the workload's FASTQ files instead of the whole "
                         "workload (0: the whole workload, the files the headline e2e is timed on); the product's "
                         "curc -c is then also timed on that sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cli", action="store_true", help="skip the whole-file `curc -c` measurement")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-vs-plain measurement")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-coder evaluation")
    ap.add_argument("--learned-pairs", type=int, default=1_000_000, help="pairs per training seed")
    ap.add_argument("--learned-eval-pairs", type=int, default=10_000_000, help="pairs per evaluation seed")
    ap.add_argument("--workload", default="pe150", choices=["pe150", "large", "batched"],
                    help="large: the single-end 250 bp case (40M reads, 200 Mbp genome), device throughput, "
                         "whole-file round trip and learned-coder bytes; batched: the 64 mixed blocks at full "
                         "scale, one block at a time against the batched drain, default against autotuned "
                         "launch choices, streams compared; each prints one JSON line")
    ap.add_argument("--fm-loop", type=int, default=None, choices=[0, 1, 2],
                    help="full-match pass loop: 0 a launch per kernel, 1 one CUDA graph, 2 one persistent "
                         "cooperative kernel (default: the library's)")
    ap.add_argument("--large-reads", type=int, default=40_000_000)
    ap.add_argument("--batched-blocks", type=int, default=16)
    ap.add_argument("--batched-scale", type=float, default=0.1)
    return ap.parse_args()


def hbm_peak():
    try:
        return float(json.load(open(PEAKS_PATH))["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._proc = None

    def wait_first(self, timeout=5.0):
        """Block until the first sample has arrived (nvidia-smi takes a moment
        to start), so that the timed region is sampled."""
        t = time.perf_counter()
        while self._proc and not self.samples and time.perf_counter() - t < timeout:
            time.sleep(0.02)

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={q}",
                                           "--format=csv,noheader,nounits", "-lms", "200"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self._proc:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def workload(pairs, genome, seed):
    from curc_b200 import synth
    return synth.paired_repeats(seed=seed, pairs=pairs, read_len=150, genome_len=genome, preserve_order=True)


# Algorithmic HBM bytes of the pack kernel per read: L ASCII bytes in,
# ceil(L/32) packed words and one N flag out.
def pack_bytes(n, L):
    return n * (L + 8 * ((L + 31) // 32) + 1)


# Algorithmic bytes of the overlap probe kernel (its launches over all
# passes), with one 32-byte sector per random access: per listed suffix its
# k-mer (32); per bucket searched the bucket range (32); per prefix
# comparison the prefix entry (32) and the prefix's row (32 * ceil(8W/32),
# counted as rows read); per hit the run slot (32).  Counts come from the
# kernel's own counters.
def probe_bytes(st, L):
    row = 32 * -(-8 * ((L + 31) // 32) // 32)
    return (32 * st["overlap_probes"] + 32 * st["overlap_searched"] + 32 * st["overlap_compares"]
            + row * st.get("overlap_rows", 0) + 32 * st["overlap_hits"])


# Algorithmic bytes of the first-word read sort (sub-stage sort_dedupe.radix):
# per non-N read one 32-byte sector for its first packed word, then 8 LSD
# passes of 8-bit digits that each read and write a 12-byte (key, id) pair.
# The lower bound of any sort (each read's words read once, ids in and out)
# is 8W + 8 per read.
def sort_bytes(m, L):
    return m * (32 + 8 * 2 * 12)


def sort_lower_bound_bytes(m, L):
    return m * (8 * ((L + 31) // 32) + 8)


# Algorithmic bytes of the overlap resolve kernel (its launches over all
# passes): per hit its 16-byte record, its run slot (32), the prefix id and
# the prefix's predecessor (32 each) and one prefix row (32 * ceil(8W/32));
# per link 10 bytes of next/prev/offset and the bucket's free word (32).
def resolve_bytes(st, L):
    row = 32 * -(-8 * ((L + 31) // 32) // 32)
    return st["overlap_hits"] * (16 + 32 + 64 + row) + st["overlap_links"] * (10 + 32)


# Algorithmic bytes of the mapping kernels (forward and reverse complement):
# per read searched its packed row (8W); per k-mer probe the bucket range,
# one 32-byte sector; per candidate its pos_array slot (32) and the
# pseudogenome window, 32 * (ceil((2L + 62) / 256) + 1).
def map_bytes(st, L, strand):
    win = 32 * (-(-(2 * L + 62) // 256) + 1)
    return (st[f"map_reads_{strand}"] * 8 * ((L + 31) // 32) + st[f"map_probes_{strand}"] * 32
            + st[f"map_candidates_{strand}"] * (32 + win))


# Algorithmic bytes of the full-match pass loop (stage a6), per list entry
# per pass, from the loop's own counters: a suffix entry has its 32-base key
# gathered (one 32-byte sector of its row), moves through two merge levels
# (12 bytes read and 12 written each), is read once by the pairing (12) and
# is compacted (4 read, its link word's sector 32, 4 written); a prefix
# entry is compacted with its key (12 read, link sector 32, 12 written).
# The pairing's binary searches over the prefix keys are not counted, so
# this is a lower bound.
def full_match_bytes(st):
    return st.get("fm_suffix_entries", 0) * (32 + 2 * 24 + 12 + 40) + st.get("fm_prefix_entries", 0) * 56


# DRAM bytes per listed suffix of the probe kernel, from ncu
# (dram__bytes_read.sum + dram__bytes_write.sum over its 96 launches) on the
# 2M-pair case of the same generator: 5.767e9 bytes / 20.21e6 probes.  The
# traffic of a launch at full size is this times its probes.
PROBE_DRAM_BYTES_PER_PROBE = 5.767e9 / 20.207e6


STAT_NAMES = ["reads", "non_n", "n_reads", "pseudogenome_reads", "unmatched", "mapped", "unmapped",
              "unmapped_n", "overlap_passes", "contested", "records", "mismatches",
              "overlap_suffixes", "overlap_active_sum", "overlap_probes", "overlap_hits",
              "overlap_searched", "overlap_compares", "overlap_links", "map_reads_fwd", "map_probes_fwd",
              "map_candidates_fwd", "map_reads_rc", "map_probes_rc", "map_candidates_rc", "overlap_rows",
              "fm_passes", "fm_suffix_entries", "fm_prefix_entries"]


def block_stats(ctx):
    """The last block run's counters (the library's "stats" result)."""
    return dict(zip(STAT_NAMES, [int(x) for x in ctx.get("stats", np.uint64)]))


def rank_seed(rank):
    """Seed of a rank's block: every rank compresses its own block of the same
    generator (independent blocks, weak scaling)."""
    return 1 + 1000 * rank


def init_dist(world):
    """One process per GPU; NCCL when the ranks have GPUs, gloo otherwise (the
    CPU tests of this plumbing).  A short timeout ends a rank that waits for
    one that is gone."""
    if world <= 1:
        return
    import datetime
    import torch
    backend = "nccl" if torch.cuda.is_available() else "gloo"
    torch.distributed.init_process_group(backend, timeout=datetime.timedelta(seconds=600))


def reduce_max(values, world, device="cpu"):
    """Each value's maximum over the ranks (the step time of a weak-scaling run
    is the slowest rank's); the values unchanged on one rank."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def run_ours(a, rank, world):
    import torch
    from curc_b200 import Context, kernel_launches

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    w = workload(a.pairs, a.genome, seed=rank_seed(rank))
    seqs = w.sequences()
    n, L = seqs.shape
    bases = n * L
    # pinned host copy of the reads (e2e input) and a device copy (value input)
    host = torch.empty(seqs.size, dtype=torch.uint8, pin_memory=True)
    host.numpy()[:] = seqs.reshape(-1)
    dseq = host.to(f"cuda:{dev}")
    ctx = Context(dev)
    ctx.keep_intermediates(False)
    if a.fm_loop is not None:
        ctx.set_tuning(fm_loop=a.fm_loop)

    def dev_step():
        ctx.block_run_device(dseq.data_ptr(), n, L, True, True)
        return ctx.stage_ms("total")

    def e2e_step():
        ctx.block_run(host.numpy().reshape(n, L), True, True)

    for _ in range(a.warmup):
        dev_step()
    stage_names = ["pack", "sort_dedupe", "overlap", "chain_filter", "full_match", "assembly", "mapping", "emit",
                   "unmapped_refs", "refmatch"]
    sub_names = ["pack.kernel", "sort_dedupe.first_word", "sort_dedupe.radix", "overlap.index", "overlap.index_sort", "overlap.index_mask",
                 "overlap.probe_resolve", "overlap.filter", "overlap.probe", "overlap.resolve", "overlap.compact",
                 "full_match.resort", "full_match.groups", "full_match.compact", "full_match.graph", "assembly.ranking", "assembly.walk", "assembly.jump",
                 "assembly.order_place", "mapping.index_fwd", "mapping.map_fwd", "mapping.index_rc", "mapping.map_rc",
                 "refmatch.index", "refmatch.probe_unmapped", "refmatch.probe_self", "refmatch.sort_unique",
                 "refmatch.accept"]
    stage_tot = {k: 0.0 for k in stage_names}
    sub_tot = {}
    l0 = kernel_launches()
    with ClockSampler(dev) as clocks:
        clocks.wait_first()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dev_ms = 0.0
        for _ in range(a.steps):
            dev_ms += dev_step()
            for k in stage_names:
                stage_tot[k] += ctx.stage_ms(k)
            for k in sub_names:
                try:
                    sub_tot[k] = sub_tot.get(k, 0.0) + ctx.stage_ms(k)
                except Exception:
                    pass
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    launches = (kernel_launches() - l0) // max(1, a.steps)
    # e2e through the C-ABI from pinned host memory: one call per step
    # (curc_block_run: copy in, run, copy out), and the batched path
    # (curc_batch_submit / curc_batch_drain: every step's reads still cross to
    # the device inside the timed region, overlapped with the previous step)
    for _ in range(1):
        e2e_step()
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for _ in range(a.steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_plain_s = (time.perf_counter() - t1) / a.steps
    hv = host.numpy().reshape(n, L)
    for _ in range(2):  # warm both block pipelines (their device and pinned memory)
        ctx.batch_submit(hv, True, True)
    ctx.batch_drain()
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for _ in range(a.steps):
        ctx.batch_submit(hv, True, True)
    ctx.batch_drain()
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t1) / a.steps
    d2h = sum(ctx.get(k).nbytes for k in ["strand", "mis_cnt", "mis_base", "id_to_pos", "ref", "unmap_ref",
                                           "unmap_n_ref", "ref_off", "ref_len_map", "unmap_ref_off", "unmap_ref_len",
                                           "unmap_n_ref_off", "unmap_n_ref_len"])
    d2h += sum(ctx.get(f"mis_off_{m}").nbytes for m in range(1, L // 5 + 1))
    stats = block_stats(ctx)
    stats.update(dict(zip(["hq_len", "unmap_len", "unmap_n_len"], [int(x) for x in ctx.get("sizes", np.uint64)[:3]])))
    step_s = dev_ms / 1000.0 / a.steps
    step_s, e2e_s, e2e_plain_s = reduce_max([step_s, e2e_s, e2e_plain_s], world, f"cuda:{dev}")
    batched = None
    if not a.no_batched and rank == 0:
        batched = batched_vs_plain(ctx, a)
    cli = None
    if not a.no_cli and world == 1:
        cli = cli_measure(ctx, w, a, dev)
    res = dict(bases=bases, n=n, L=L, step_s=step_s, e2e_s=e2e_s, wall=wall, launches=launches, stats=stats,
               stage_ms={k: v / a.steps for k, v in stage_tot.items()},
               substage_ms={k: round(v / a.steps, 3) for k, v in sub_tot.items()}, clocks=clocks.summary(),
               h2d=int(seqs.size), d2h=int(d2h), cli=cli, e2e_plain_s=e2e_plain_s, batched=batched)
    ctx.close()
    return res


def cpu_baseline(a):
    """The CPU oracle (a restatement whose overlap searches, mapping and
    RefMatcher probes run on OpenMP threads) on a bounded sample of the same
    workload: fewer pairs from a genome scaled
    by the same factor, so that the coverage, and with it the share of reads
    that overlap, map or stay unmapped, is the workload's (a few pairs from
    the whole genome would leave most reads unmapped and time the unmapped
    full match instead)."""
    from tests.oracle_lib import OracleBlock
    genome = max(100_000, int(a.genome * a.cpu_sample_pairs / a.pairs))
    w = workload(a.cpu_sample_pairs, genome, seed=1)
    seqs = w.sequences()
    threads = os.cpu_count() or 1
    t = time.perf_counter()
    OracleBlock(seqs, True, True, threads=threads)
    dt = time.perf_counter() - t
    # the same on one core, for the scaling of the restatement with cores
    t = time.perf_counter()
    OracleBlock(seqs, True, True, threads=1)
    dt1 = time.perf_counter() - t
    return {"value": seqs.size / dt / 1e6, "unit": "Mbases/s", "cores": threads, "kind": "port",
            "value_1_core": seqs.size / dt1 / 1e6,
            "sample": f"{a.cpu_sample_pairs} pairs x 150 bp of the same generator from a {genome / 1e6:g} Mbp genome "
                      f"(the workload's coverage; {seqs.size / 1e6:.0f} Mbases), "
                      f"block streams without the entropy coders, {dt:.1f} s on {threads} threads, {dt1:.1f} s on "
                      "one (OpenMP in the overlap searches, the mapping and the RefMatcher probes; links made in order)"}


# Record headers long enough for the reference's block-boundary heuristic
# (it matches more than 5 bytes of the first header at a line start).
FASTQ_NAME = b"synthetic_read_"
CURC_EXE = os.path.join(ROOT, "curc_b200", "_build", "curc")
BSC_EXE = os.path.join(ROOT, "curc_b200", "_build", "bsc")
HOST_STAGES = ["files.total", "files.ingest", "files.device", "files.snapshot", "files.until_last_block",
               "files.coder_tail", "files.coders", "coder.id_pos", "coder.strand", "coder.ref", "coder.maps",
               "coder.mis_cnt", "coder.mis_base", "coder.mis_off", "coder.read_off", "coder.pe_order",
               "coder.id_pos.fl2_base", "coder.id_pos.order", "coder.id_pos.split", "coder.id_pos.ppmd"]


def sample_of(w, pairs):
    """The first `pairs` pairs of a workload: its FASTQ files are the first
    records of the workload's own files, byte for byte."""
    from curc_b200 import synth
    return synth.Workload(w.name + f"_first{pairs}", w.read_len, w.mate1[:pairs],
                          None if w.mate2 is None else w.mate2[:pairs], w.preserve_order)


def timed_runs(cmd, cwd, steps, warmup, env=None, archive=None, timeout=900):
    """Runs `cmd` warmup + steps times; per timed run its wall time and the
    arrival time of each stdout line (line-buffered)."""
    runs = []
    for i in range(warmup + steps):
        t = time.perf_counter()
        p = subprocess.Popen(["stdbuf", "-oL"] + cmd, cwd=cwd, env=env, stdout=subprocess.PIPE,
                             stderr=subprocess.PIPE, text=True)
        lines = []
        for line in p.stdout:
            lines.append((time.perf_counter() - t, line.rstrip("\n")))
        err = p.stderr.read()
        rc = p.wait(timeout=timeout)
        dt = time.perf_counter() - t
        if rc != 0:
            raise RuntimeError(f"{cmd[0]} exited {rc}: {lines[-3:]} {err[-300:]}")
        if archive and os.path.exists(archive):
            size = os.path.getsize(archive)
            os.remove(archive)
        else:
            size = None
        if i >= warmup:
            runs.append({"s": dt, "lines": lines, "archive_bytes": size})
    return runs


def line_stages(runs):
    """Mean time between the progress lines `curc -c` prints (the reference's
    preprocess.cpp:69-279 and the same lines from the product's CLI): CUDA
    context set-up, FASTQ parse and block split (with the packing), block
    compression (device path and stream coders), archive write, exit."""
    marks = [("init", "gpu context init finish"), ("parse_split", "waiting block compress"),
             ("block_compress", "compress finish"), ("archive_write", "archive size")]
    out = {}
    for name, key in marks:
        ts = [next((t for t, l in r["lines"] if key in l), None) for r in runs]
        if all(x is not None for x in ts):
            out[name] = sum(ts) / len(ts)
    prev, res = 0.0, {}
    for name, _ in marks:
        if name in out:
            res[name + "_s"] = round(out[name] - prev, 4)
            prev = out[name]
    res["exit_s"] = round(sum(r["s"] for r in runs) / len(runs) - prev, 4)
    return res


def curc_runs(files, td, steps, warmup, dev, tag):
    archive = os.path.join(td, tag + ".curc")
    cmd = [CURC_EXE, "-c", "-i", ",".join(files), "-o", tag, "--working_dir", td, "--preserve_order",
           "--device", str(dev)]
    return timed_runs(cmd, td, steps, warmup, archive=archive)


def cli_measure(ctx, w, a, dev):
    """`curc -c` of the workload: the product binary, one process per step
    (the headline e2e), on the whole workload and on the reference arm's
    sample; plus one in-process whole-file call for the host-stage split."""
    with tempfile.TemporaryDirectory() as td:
        files = w.write(os.path.join(td, "full"), name=FASTQ_NAME)
        t = time.perf_counter()
        ctx.compress_files(files, os.path.join(td, "inproc.curc"), 1.0, True, BSC_EXE, td)
        t_in = time.perf_counter() - t
        os.remove(os.path.join(td, "inproc.curc"))
        host_ms = {}
        for k in HOST_STAGES:
            try:
                host_ms[k] = round(ctx.stage_ms(k), 3)
            except Exception:
                pass
        full = curc_runs(files, td, a.steps, a.warmup, dev, "full")
        for f in files:
            os.remove(f)
        sample = None
        if a.ref_sample_pairs:
            ws = sample_of(w, a.ref_sample_pairs)
            sfiles = ws.write(os.path.join(td, "sample"), name=FASTQ_NAME)
            runs = curc_runs(sfiles, td, a.steps, a.warmup, dev, "sample")
            smean = sum(r["s"] for r in runs) / len(runs)
            sample = {"value": ws.bases / smean / 1e6, "s": smean, "pairs": a.ref_sample_pairs,
                      "archive_bytes": runs[0]["archive_bytes"], "line_stages": line_stages(runs)}
    mean = sum(r["s"] for r in full) / len(full)
    return {"s": mean, "value": w.bases / mean / 1e6, "archive_bytes": full[0]["archive_bytes"],
            "archive_bits_per_base": 8.0 * full[0]["archive_bytes"] / w.bases,
            "line_stages": line_stages(full), "in_process_s": t_in, "host_stage_ms": host_ms, "sample": sample}


def batched_vs_plain(ctx, a):
    """Independent single-end blocks of mixed size and read length (the
    batched workload's generator, scaled down): one curc_block_run call per
    block from pageable host memory, against all blocks queued and drained."""
    from curc_b200 import synth
    blocks = [np.ascontiguousarray(w.mate1) for w in synth.batched_blocks(seed=2, count=a.batched_blocks,
                                                                          scale=a.batched_scale)]
    bases = sum(b.size for b in blocks)
    ctx.block_run(blocks[0])  # warm
    ctx.batch_workers(4)  # small blocks: more pipelines to fill the GPU
    for b in blocks:  # warm the block pipelines of the batched path
        ctx.batch_submit(b)
    ctx.batch_drain()
    t = time.perf_counter()
    for b in blocks:
        ctx.block_run(b)
    plain = time.perf_counter() - t
    t = time.perf_counter()
    for b in blocks:
        ctx.batch_submit(b)
    ctx.batch_drain()
    batched = time.perf_counter() - t
    ctx.batch_workers(2)
    return {"workload": f"{len(blocks)} single-end blocks from different random genomes, read counts log-uniform "
                        f"in [50k, 5M] x {a.batched_scale}, read lengths from {{75, 100, 150, 250}}, errors 0.1-0.5%",
            "bases": int(bases), "plain": bases / plain / 1e6, "batched": bases / batched / 1e6, "pipelines": 4,
            "unit": "Mbases/s", "includes": "host reads to host streams (copies and device work), no coders"}


def learned_eval(a):
    """Bits/base of the mismatch streams, learned vs plain coders and vs
    fast-lzma2 level 10 and libbsc on the same streams, on the
    position-dependent-error workload at the benchmark block's shape
    (paired-end 150 bp, error rising 0.1% -> 1.0% along the read, transitions
    2:1): trained on 8 seeds (blocks of the same coverage), evaluated on 2
    disjoint seeds of 10M pairs from 50 Mbp genomes, every learned stream
    decoded back and checked."""
    from curc_b200.learned import train_and_evaluate
    t = time.perf_counter()
    with tempfile.TemporaryDirectory() as td:
        r = train_and_evaluate(train_seeds=list(range(301, 309)), eval_seeds=[401, 402], pairs=a.learned_pairs,
                               genome_len=a.learned_pairs * 5, epochs=2, batch=4096,
                               eval_pairs=a.learned_eval_pairs, eval_genome_len=a.genome,
                               general=(BSC_EXE, td))
    return {"workload": f"paired-end 150 bp, substitutions 0.1% -> 1.0% along the read, Ti:Tv 2:1; training: 8 seeds "
                        f"of {a.learned_pairs} pairs from {a.learned_pairs * 5 / 1e6:.0f} Mbp genomes; evaluation: "
                        f"2 seeds of {a.learned_eval_pairs} pairs from {a.genome / 1e6:.0f} Mbp genomes",
            "plain_bits_per_base": r["plain_bits_per_base"], "learned_bits_per_base": r["learned_bits_per_base"],
            "fl2_level10_bits_per_base": r.get("fl2_level10_bits_per_base"),
            "libbsc_bits_per_base": r.get("libbsc_bits_per_base"),
            "plain_bytes": {"counts": r["plain"][0], "bases": r["plain"][1], "offsets": r["plain"][2]},
            "learned_bytes": {"counts (plain)": r["plain"][0], "gaps and bases": r["learned"],
                              "model (stored once per learned block)": r["model_bytes"]},
            "gaps_and_bases_vs_plain": r["gaps_and_bases_ratio"],
            "mismatch_streams_vs_plain": r["mismatch_streams_ratio"], "lossless": r["lossless"],
            "train_anchors": r["train_anchors"], "final_loss": r["loss"], "s": time.perf_counter() - t}


def run_reference(a):
    """The reference `curc -c` (built from its sources, oracle/_ref), one
    process per step, on the workload's own FASTQ files (the files the
    product's headline e2e is timed on), or on their first pairs with
    --ref-sample-pairs, on this box."""
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    exe = os.path.join(ref_dir, "curc_shared")
    if not os.path.exists(exe):
        return None, "reference build missing (oracle/_ref/curc_shared)"
    w = workload(a.pairs, a.genome, seed=1)
    ws = sample_of(w, a.ref_sample_pairs) if a.ref_sample_pairs else w
    steps, warmup = a.steps, a.warmup
    with tempfile.TemporaryDirectory() as td:
        files = ws.write(os.path.join(td, "in"), name=FASTQ_NAME)
        del w
        shim_log = os.path.join(td, "shim.log")
        env = dict(os.environ, LD_PRELOAD=os.path.join(ref_dir, "libzero_alloc.so"), CURC_SHIM_LOG=shim_log)
        cmd = [exe, "-c", "-i", ",".join(files), "-o", "out", "--working_dir", td, "--preserve_order"]
        try:
            runs = timed_runs(cmd, ref_dir, steps, warmup, env=env, archive=os.path.join(td, "out.curc"),
                              timeout=3600)
        except RuntimeError as e:
            return None, str(e)[:300]
        # one line per process that loaded the shim: the reference's own runs
        # (their allocations filled), and the bsc processes it starts (none)
        fills = [tuple(float(x) for x in l.split()) for l in open(shim_log)] if os.path.exists(shim_log) else []
    fills = [f for f in fills if f[0] > 0][warmup:]
    mean = sum(r["s"] for r in runs) / len(runs)
    return {"bases": ws.bases, "pairs": ws.mate1.shape[0], "s": mean, "steps": len(runs),
            "archive_bytes": runs[0]["archive_bytes"], "line_stages": line_stages(runs),
            "zero_fill": {"allocations": fills[0][0] if fills else None,
                          "s": sum(f[1] for f in fills) / len(fills) if fills else None}}, None


def run_large(a):
    """The single-end 250 bp case: 40M reads (10 Gbases) from a 200 Mbp genome
    (45% GC, 8% repeats of 0.5-10 kbp at 0.5-2% divergence), substitutions
    0.1% -> 1.5% along the read, N 0.02%, preserved order, one block.  Device
    throughput (reads in HBM), the whole-file `curc -c` in learned mode (a
    model trained on a disjoint small seed of the same generator; per block
    the smaller of plain and learned coding), and the round trip of that
    archive through the product decoder, read for read."""
    import torch
    from curc_b200 import Context, Learner, decompress_file, synth
    t0 = time.perf_counter()
    w = synth.large_combined(seed=4, n_reads=a.large_reads)
    gen_s = time.perf_counter() - t0
    seqs = w.mate1
    n, L = seqs.shape
    peak, peak_kind = hbm_peak()
    out = {"workload": f"single-end {L} bp, {n} reads ({n * L / 1e9:.1f} Gbases) from a 200 Mbp genome (45% GC, 8% "
                       "repeats of 0.5-10 kbp at 0.5-2% divergence), substitutions 0.1% -> 1.5% along the read, "
                       "N 0.02%, --preserve_order, block_ratio 1", "generate_s": gen_s}
    with Context(0) as ctx, Learner(0) as lrn:
        # a model from a disjoint seed of the same generator (1M reads)
        ws = synth.large_combined(seed=40, n_reads=1_000_000, genome_len=5_000_000)
        ctx.block_run(ws.mate1, True, False)
        lrn.add_block(ctx)
        lrn.train(epochs=2, batch=4096)
        model = lrn.model()
        del ws
        ctx.keep_intermediates(False)
        d = torch.from_numpy(seqs.reshape(-1)).cuda()
        for _ in range(a.warmup):
            ctx.block_run_device(d.data_ptr(), n, L, True, False)
        ms = []
        with ClockSampler(0) as clocks:
            clocks.wait_first()
            for _ in range(a.steps):
                ctx.block_run_device(d.data_ptr(), n, L, True, False)
                ms.append(ctx.stage_ms("total"))
        stage = {k: ctx.stage_ms(k) for k in ["pack", "sort_dedupe", "overlap", "chain_filter", "full_match",
                                              "assembly", "mapping", "emit", "unmapped_refs", "refmatch"]}
        out["block_stats"] = block_stats(ctx)
        out["substage_ms"] = {k: round(ctx.stage_ms(k), 3) for k in
                              ["mapping.index_fwd", "mapping.map_fwd", "mapping.index_rc", "mapping.map_rc",
                               "overlap.index", "overlap.index_mask", "overlap.filter", "overlap.probe",
                               "overlap.resolve", "overlap.compact", "refmatch.index", "refmatch.probe_self",
                               "refmatch.sort_unique", "refmatch.accept", "full_match.graph",
                               "assembly.ranking", "assembly.order_place"]
                              if _has_stage(ctx, k)}
        pack_ms = stage["pack"]
        del d
        torch.cuda.empty_cache()
        step = sum(ms) / len(ms)
        out.update({"value": n * L / (step / 1000.0) / 1e6, "unit": "Mbases/s", "ms_per_step": step,
                    "steps": a.steps, "stage_ms": stage, "clocks": clocks.summary(),
                    "roofline_pack": {"achieved": pack_bytes(n, L) / (pack_ms / 1000.0) / 1e9, "peak": peak,
                                      "peak_kind": peak_kind, "unit": "GB/s",
                                      "frac": pack_bytes(n, L) / (pack_ms / 1000.0) / 1e9 / peak}})
        try:
            out.update(_large_files(ctx, w, seqs, model))
        except Exception as e:  # e.g. no room for the 21 GB FASTQ file
            out["e2e_learned_mode"] = {"error": str(e)[:300]}
    return out


def _large_files(ctx, w, seqs, model):
    """Whole-file `curc -c` of the large workload in learned mode, then the
    product decoder, compared read for read."""
    from curc_b200 import decompress_file
    n, L = seqs.shape
    out = {}
    with tempfile.TemporaryDirectory() as td:
        files = w.write(os.path.join(td, "large"), name=FASTQ_NAME)
        arc = os.path.join(td, "large.curc")
        ctx.set_mismatch_model(model)
        t = time.perf_counter()
        ctx.compress_files(files, arc, 1.0, True, BSC_EXE, td)
        e2e_s = time.perf_counter() - t
        out["e2e_learned_mode"] = {"value": n * L / e2e_s / 1e6, "unit": "Mbases/s", "s": e2e_s,
                                   "archive_bytes": os.path.getsize(arc),
                                   "archive_bits_per_base": 8.0 * os.path.getsize(arc) / (n * L),
                                   "mismatch_plain_kb": ctx.stage_ms("files.mismatch_plain_kb"),
                                   "mismatch_learned_kb": ctx.stage_ms("files.mismatch_learned_kb"),
                                   "learned_blocks": ctx.stage_ms("files.learned_blocks"),
                                   "host_stage_ms": {k: round(ctx.stage_ms(k), 1) for k in HOST_STAGES
                                                     if _has_stage(ctx, k)}}
        ctx.set_mismatch_model(None)
        for f in files:
            os.remove(f)
        t = time.perf_counter()
        got = decompress_file(arc, os.path.join(td, "dec"), BSC_EXE, td)
        dec_s = time.perf_counter() - t
        ok = got == n
        if ok:
            rows = np.memmap(os.path.join(td, "dec.seq"), dtype=np.uint8, mode="r").reshape(n, L + 1)
            for c0 in range(0, n, 1_000_000):
                ok &= bool(np.array_equal(rows[c0:c0 + 1_000_000, :L], seqs[c0:c0 + 1_000_000]))
            del rows
        out["roundtrip"] = {"lossless": ok, "decode_s": dec_s, "reads": got}
    return out


def run_batched(a):
    """The batched workload at full scale: 64 independent single-end blocks
    from 64 seeded random genomes (2-20 Mbp), read counts log-uniform in
    50k-5M, read lengths from {75, 100, 150, 250}, errors 0.1-0.5%.  Times
    (host reads to host streams, no coders) one curc_block_run per block,
    then the batched drain (concurrent block pipelines, large blocks
    double-buffered), then the drain again with each block's launch choices
    autotuned for its (read length, read-count bucket) on one block of that
    bucket.  Every block's streams must be the same in all three runs."""
    import hashlib
    from curc_b200 import Context, synth
    from tests.oracle_lib import stream_dtype, stream_names
    t0 = time.perf_counter()
    specs = synth.batched_specs(2, 64, 1.0)
    blocks = [np.ascontiguousarray(synth.batched_block(2, b, sp).mate1) for b, sp in enumerate(specs)]
    gen_s = time.perf_counter() - t0
    bases = int(sum(b.size for b in blocks))

    def digest(ctx, L):
        h = hashlib.sha256()
        for nm in stream_names(L):
            h.update(ctx.get(nm, stream_dtype(nm)).tobytes())
        return h.hexdigest()

    out = {"workload": "64 single-end blocks from 64 seeded random genomes (2-20 Mbp), read counts log-uniform in "
                       "50k-5M, read lengths from {75, 100, 150, 250}, errors 0.1-0.5%",
           "blocks": len(blocks), "reads": int(sum(b.shape[0] for b in blocks)), "bases": bases,
           "generate_s": gen_s, "unit": "Mbases/s",
           "includes": "host reads to host streams (H2D, device path, D2H), no stream coders"}
    with tempfile.TemporaryDirectory() as td, Context(0) as ctx:
        ctx.keep_intermediates(False)
        ctx.block_run(blocks[0])  # warm
        plain = []
        t = time.perf_counter()
        for b in blocks:
            ctx.block_run(b)
            plain.append(digest(ctx, b.shape[1]))
        # the digests are taken inside the timed loop here too, as in the drains
        out["one_block_at_a_time"] = bases / (time.perf_counter() - t) / 1e6

        # batched drain: digests per ticket
        tickets = []
        for b in blocks:
            tickets.append(ctx.batch_submit(b))
        dig = {}
        t = time.perf_counter()
        ctx.batch_workers(4)
        ctx.batch_drain(lambda tk: dig.__setitem__(tk, digest(ctx, blocks[tickets.index(tk)].shape[1])))
        out["batched"] = bases / (time.perf_counter() - t) / 1e6
        out["batched_streams_equal"] = all(dig[tk] == plain[i] for i, tk in enumerate(tickets))
        ctx.trim()  # the drain's pipelines are made again by the next drain
        # autotune one block per (read length, read-count bucket), then drain with per-block choices
        import torch
        cache = os.path.join(td, "tune.txt")
        seen = {}
        t = time.perf_counter()
        for i, b in enumerate(blocks):
            key = (b.shape[1], int(np.floor(np.log2(b.shape[0]))))
            if key in seen:
                continue
            d = torch.from_numpy(b.reshape(-1)).cuda()
            print(f"autotune bucket L={key[0]} 2^{key[1]} on {b.shape[0]} reads", file=sys.stderr, flush=True)
            seen[key] = ctx.autotune(d.data_ptr(), b.shape[0], b.shape[1], False, False, cache)[0]
            del d
        out["autotune_s"] = time.perf_counter() - t
        ctx.trim()
        torch.cuda.empty_cache()
        out["tuned_buckets"] = {f"L{k[0]}_2^{k[1]}": v for k, v in seen.items()}
        ctx.set_tuning(table_factor=4, bitmap_bits=16, check_every=8, map_threads=128)
        ctx.use_tuning_cache(cache)
        tickets = [ctx.batch_submit(b) for b in blocks]
        dig = {}
        t = time.perf_counter()
        ctx.batch_drain(lambda tk: dig.__setitem__(tk, digest(ctx, blocks[tickets.index(tk)].shape[1])))
        out["batched_autotuned"] = bases / (time.perf_counter() - t) / 1e6
        out["autotuned_streams_equal"] = all(dig[tk] == plain[i] for i, tk in enumerate(tickets))
        ctx.use_tuning_cache(None)
    return out


def _has_stage(ctx, k):
    try:
        ctx.stage_ms(k)
        return True
    except Exception:
        return False


def finish_dist(world):
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


def main():
    a = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    init_dist(world)
    cfg = {"workload": f"paired-end 150 bp, {a.pairs} pairs ({2 * a.pairs * 150 / 1e9:.1f} Gbases) from a "
                       f"{a.genome / 1e6:.0f} Mbp genome (40% GC, 5% repeats at 1% divergence), insert N(400,50), "
                       "0.2% substitutions, 0.01% N, --preserve_order, block_ratio 1",
           "global_batch": a.pairs * 2 * world, "read_len": 150, "parallelism": f"independent blocks x{world}",
           "l2_flush": "inputs (3 GB ASCII per block) are larger than L2"}
    if a.workload in ("large", "batched"):
        print(json.dumps(run_large(a) if a.workload == "large" else run_batched(a)))
        finish_dist(world)
        return
    if a.impl == "reference":
        if rank != 0:
            finish_dist(world)
            return
        ref, why = run_reference(a)
        if ref is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            finish_dist(world)
            return
        v = ref["bases"] / ref["s"] / 1e6
        what = (f"the first {ref['pairs']} pairs of the workload's FASTQ files ({ref['bases'] / 1e6:.0f} Mbases) "
                "per step" if a.ref_sample_pairs else
                f"the workload's FASTQ files ({ref['bases'] / 1e6:.0f} Mbases) per step")
        out = {"metric": METRIC, "value": v, "unit": "Mbases/s", "n_gpus": 1, "steps": ref["steps"],
               "warmup": a.warmup, "ms_per_step": ref["s"] * 1000, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic", "impl": "reference",
               "config": cfg,
               "cpu_baseline": {"value": v, "unit": "Mbases/s", "cores": os.cpu_count(), "kind": "reference",
                                "sample": f"reference curc -c end to end, one process per step (CUDA set-up, "
                                          f"FASTQ parse, GPU stages, host coders, archive write) on {what}"},
               "e2e": {"value": v, "unit": "Mbases/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
               "line_stages": ref["line_stages"], "archive_bytes": ref["archive_bytes"],
               "zero_fill": dict(ref["zero_fill"], note="LD_PRELOAD shim that zero-fills each cudaMalloc "
                                                        "(cudaMemset + cudaDeviceSynchronize): mean seconds per "
                                                        "run, included in the time above")}
        print(json.dumps(out))
        finish_dist(world)
        return
    r = run_ours(a, rank, world)
    if rank != 0:
        finish_dist(world)
        return
    peak, peak_kind = hbm_peak()
    pack_ms = r["substage_ms"].get("pack.kernel") or r["stage_ms"]["pack"]
    dominant = max(r["stage_ms"], key=r["stage_ms"].get)
    achieved = pack_bytes(r["n"], r["L"]) / (pack_ms / 1000.0) / 1e9 if pack_ms > 0 else None
    st = r["stats"]
    probe_ms = r["substage_ms"].get("overlap.probe", 0.0)
    passes = max(1, st["overlap_passes"])
    probe_ach = probe_bytes(st, r["L"]) / (probe_ms / 1000.0) / 1e9 if probe_ms > 0 else None
    def roof(kernel, nbytes, ms, launches, extra=None):
        ach = nbytes / (ms / 1000.0) / 1e9 if ms > 0 else None
        d = {"kernel": kernel, "bound": "hbm", "achieved": ach, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
             "frac": ach / peak if ach else None, "traffic": None,
             "algorithmic_bytes_per_launch": nbytes / max(1, launches), "launches": launches,
             "ms_per_launch": ms / max(1, launches)}
        d.update(extra or {})
        return d

    sub = r["substage_ms"]
    m_reads = st["non_n"]
    out = {
        "metric": METRIC,
        "value": r["bases"] * world / r["step_s"] / 1e6,
        "unit": "Mbases/s",
        "n_gpus": world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": r["step_s"] * 1000,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8",
        "data": "synthetic",
        "config": cfg,
        "e2e": ({"value": r["cli"]["value"], "unit": "Mbases/s", "h2d_bytes_per_step": r["h2d"],
                 "d2h_bytes_per_step": r["d2h"],
                 "api": "the product's curc -c binary, one process per step, FASTQ files (page cache) to the "
                        "closed archive: parse, H2D, device path, D2H, stream coders, archive write",
                 "s_per_step": r["cli"]["s"]} if r["cli"] else
                {"value": r["bases"] * world / r["e2e_s"] / 1e6, "unit": "Mbases/s",
                 "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"],
                 "api": "curc_batch_submit/curc_batch_drain, one block per step from pinned host memory "
                        "(no stream coders)"}),
        "e2e_batched_device_path": {"value": r["bases"] * world / r["e2e_s"] / 1e6, "unit": "Mbases/s",
                                    "api": "curc_batch_submit/curc_batch_drain from pinned host memory, streams "
                                           "back to the host, no stream coders",
                                    "one_call_per_step": r["bases"] * world / r["e2e_plain_s"] / 1e6},
        "roofline": {"kernel": "probe_kernel (overlap passes, stage a4; the memory-bound kernel with the largest share of the launch list: map_kernel<0> has a slightly larger share but is issue-bound, see roofline_map)",
                     "bound": "hbm", "achieved": probe_ach, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": probe_ach / peak if probe_ach else None,
                     "traffic": PROBE_DRAM_BYTES_PER_PROBE * st["overlap_probes"] / passes,
                     "algorithmic_bytes_per_launch": probe_bytes(st, r["L"]) / passes, "launches": passes,
                     "ms_per_launch": probe_ms / passes,
                     "traffic_source": "ncu dram bytes per probe on the 2M-pair case, times this launch's probes"},
        "roofline_pack": {"kernel": "pack_kernel (stage a1, sub-stage pack.kernel)", "bound": "hbm",
                          "achieved": achieved, "peak": peak,
                          "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak if achieved else None,
                          "traffic": None},
        "roofline_sort": roof("first-word LSD radix sort of the reads (gather + 8 passes, sub-stage "
                              "sort_dedupe.first_word, stage a2)",
                              sort_bytes(m_reads, r["L"]), sub.get("sort_dedupe.first_word", 0.0), 1,
                              {"frac_of_lower_bound": (sort_lower_bound_bytes(m_reads, r["L"]) /
                                                       (sub["sort_dedupe.first_word"] / 1000.0) / 1e9 / peak)
                               if sub.get("sort_dedupe.first_word") else None,
                               "whole_sort_ms": sub.get("sort_dedupe.radix")}),
        "roofline_resolve": roof("resolve_kernel (overlap passes, stage a4)", resolve_bytes(st, r["L"]),
                                 sub.get("overlap.resolve", 0.0), passes),
        "roofline_full_match": roof("full-match pass loop (stage a6: key gather, two merge levels, pairing, "
                                    "two compactions per pass; one CUDA graph, or per-launch with --fm-loop 0)",
                                    full_match_bytes(st), r["stage_ms"].get("full_match", 0.0),
                                    max(1, st.get("fm_passes", 0)), {"passes": st.get("fm_passes", 0)}),
        "roofline_map": roof("map_kernel forward + reverse complement (stage a9)",
                             map_bytes(st, r["L"], "fwd") + map_bytes(st, r["L"], "rc"),
                             sub.get("mapping.map_fwd", 0.0) + sub.get("mapping.map_rc", 0.0), 2),
        "stage_ms": r["stage_ms"],
        "substage_ms": r["substage_ms"],
        "block_stats": r["stats"],
        "dominant_stage": dominant,
        "clocks": r["clocks"],
        "gpu_launches": r["launches"],
    }
    if r["cli"]:
        out["cli"] = r["cli"]
        if r["cli"]["sample"]:
            out["e2e_same_sample"] = dict(r["cli"]["sample"], unit="Mbases/s",
                                          note="the product's curc -c on the same files as the reference arm's steps")
    if r["batched"]:
        out["batched"] = r["batched"]
    if not a.no_learned and rank == 0:
        try:
            out["learned_coder"] = learned_eval(a)
        except Exception as e:  # reported, the rest of the line stands
            out["learned_coder"] = {"error": str(e)[:300]}
    if not a.no_cpu_baseline and world == 1:
        out["cpu_baseline"] = cpu_baseline(a)
    print(json.dumps(out))
    finish_dist(world)


if __name__ == "__main__":
    main()
