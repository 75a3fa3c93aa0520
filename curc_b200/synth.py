"""Seeded synthetic FASTQ workloads.

No public sequencing dataset is used.  Each generator draws a random genome
(optionally GC-biased, with diverged repeat copies), samples fixed-length reads
from it, applies substitution errors and N bases, and writes FASTQ records
with headers ``@r<i>`` (single end) or ``@r<i>/1`` / ``@r<i>/2`` (paired end,
so that both mate files have identical byte layouts, which the block splitter
requires), and a constant quality line of ``I``.

All arrays are uint8 ASCII; records are assembled with vectorised numpy so
that multi-gigabase inputs generate in seconds.
"""
from __future__ import annotations

import dataclasses
import numpy as np

ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)
_COMP = np.zeros(256, dtype=np.uint8)
for a, b in zip(b"ACGTN", b"TGCAN"):
    _COMP[a] = b


def revcomp(seqs: np.ndarray) -> np.ndarray:
    """Reverse complement of each row of a 2-D uint8 ASCII array."""
    return _COMP[seqs[..., ::-1]]


def random_genome(rng: np.random.Generator, length: int, gc: float = 0.5,
                  repeat_frac: float = 0.0, repeat_len=(1000, 5000),
                  repeat_div=(0.01, 0.01)) -> np.ndarray:
    """i.i.d. genome with GC fraction ``gc``; then ``repeat_frac`` of it is
    overwritten by copies of other genome segments (lengths uniform in
    ``repeat_len``) carrying substitutions at a rate uniform in ``repeat_div``."""
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    g = ACGT[rng.choice(4, size=length, p=p).astype(np.uint8)]
    covered = 0
    target = int(repeat_frac * length)
    while covered < target:
        ln = int(rng.integers(repeat_len[0], repeat_len[1] + 1))
        src = int(rng.integers(0, length - ln))
        dst = int(rng.integers(0, length - ln))
        seg = g[src:src + ln].copy()
        div = rng.uniform(repeat_div[0], repeat_div[1])
        m = rng.random(ln) < div
        seg[m] = _substitute(rng, seg[m])
        g[dst:dst + ln] = seg
        covered += ln
    return g


def _substitute(rng: np.random.Generator, bases: np.ndarray, ti_tv: float | None = None) -> np.ndarray:
    """Replace each base by a different base: uniform over the other three, or
    with transitions (A<->G, C<->T) ``ti_tv`` times as likely as each of the
    two transversions."""
    code = np.searchsorted(ACGT, bases)
    if ti_tv is None:
        shift = rng.integers(1, 4, size=code.shape)
        return ACGT[(code + shift) % 4]
    # transition partner of A C G T is G T A C
    ti = np.array([2, 3, 0, 1])
    p_ti = ti_tv / (ti_tv + 2.0)
    u = rng.random(code.shape)
    out = ti[code]
    tv = u >= p_ti
    # the two transversions of a purine are C/T, of a pyrimidine A/G
    tv_choices = np.array([[1, 3], [0, 2], [1, 3], [0, 2]])
    pick = rng.integers(0, 2, size=code.shape)
    out = np.where(tv, tv_choices[code, pick], out)
    return ACGT[out]


DENSE_LIMIT = 20_000_000  # bases; above it errors are drawn sparsely


def _apply_errors(rng, reads: np.ndarray, err, n_rate: float, ti_tv=None) -> None:
    """In place: substitutions with per-position rate ``err`` (scalar or array
    of read length) and N bases at ``n_rate``.  Small inputs draw one uniform
    per base; large ones draw the number of events per read position
    (binomial) and their reads uniformly, which has the same distribution."""
    n, L = reads.shape
    if reads.size > DENSE_LIMIT:
        rate = np.broadcast_to(np.asarray(err, dtype=np.float64), (L,))
        for j in range(L):
            k = rng.binomial(n, rate[j])
            if k:
                rows = rng.choice(n, size=k, replace=False) if k < n // 4 else np.nonzero(rng.random(n) < rate[j])[0]
                reads[rows, j] = _substitute(rng, reads[rows, j], ti_tv)
        if n_rate > 0:
            k = rng.binomial(reads.size, n_rate)
            flat = rng.integers(0, reads.size, size=k)
            reads.reshape(-1)[flat] = ord("N")
        return
    rate = np.broadcast_to(np.asarray(err, dtype=np.float64), (L,))
    m = rng.random((n, L)) < rate[None, :]
    if m.any():
        reads[m] = _substitute(rng, reads[m], ti_tv)
    if n_rate > 0:
        mn = rng.random((n, L)) < n_rate
        reads[mn] = ord("N")


def sample_single(rng, genome: np.ndarray, n: int, L: int, err, n_rate: float,
                  rc_frac: float = 0.5, ti_tv=None) -> np.ndarray:
    starts = rng.integers(0, len(genome) - L + 1, size=n)
    reads = np.lib.stride_tricks.sliding_window_view(genome, L)[starts]
    rc = rng.random(n) < rc_frac
    reads[rc] = revcomp(reads[rc])
    _apply_errors(rng, reads, err, n_rate, ti_tv)
    return reads


def sample_paired(rng, genome: np.ndarray, pairs: int, L: int, err, n_rate: float,
                  insert_mean=400.0, insert_sd=50.0, ti_tv=None):
    ins = np.clip(np.rint(rng.normal(insert_mean, insert_sd, size=pairs)), L, None).astype(np.int64)
    starts = rng.integers(0, len(genome) - ins + 1)
    win = np.lib.stride_tricks.sliding_window_view(genome, L)
    m1 = win[starts]
    m2 = revcomp(win[starts + ins - L])
    flip = rng.random(pairs) < 0.5  # fragment from the reverse strand
    t1 = m1[flip].copy()
    m1[flip] = m2[flip]
    m2[flip] = t1
    _apply_errors(rng, m1, err, n_rate, ti_tv)
    _apply_errors(rng, m2, err, n_rate, ti_tv)
    return m1, m2


def fastq_bytes(reads: np.ndarray, suffix: bytes = b"", name: bytes = b"r") -> bytes:
    """FASTQ text: ``@<name><i><suffix>`` / sequence / ``+`` / ``I`` * L."""
    n, L = reads.shape
    out = []
    lo = 0
    digits = 1
    while lo < n:
        hi = min(n, 10 ** digits)
        if hi > lo:
            cnt = hi - lo
            hl = 1 + len(name) + digits + len(suffix)  # '@' name digits suffix
            rec = hl + 1 + L + 1 + 2 + L + 1
            buf = np.empty((cnt, rec), dtype=np.uint8)
            buf[:, 0] = ord("@")
            for j, ch in enumerate(name):
                buf[:, 1 + j] = ch
            ids = np.arange(lo, hi, dtype=np.int64)
            h0 = 1 + len(name)
            for d in range(digits):
                buf[:, h0 + d] = ord("0") + (ids // 10 ** (digits - 1 - d)) % 10
            for j, ch in enumerate(suffix):
                buf[:, h0 + digits + j] = ch
            buf[:, hl] = ord("\n")
            buf[:, hl + 1:hl + 1 + L] = reads[lo:hi]
            p = hl + 1 + L
            buf[:, p] = ord("\n")
            buf[:, p + 1] = ord("+")
            buf[:, p + 2] = ord("\n")
            buf[:, p + 3:p + 3 + L] = ord("I")
            buf[:, p + 3 + L] = ord("\n")
            out.append(buf.reshape(-1))
        lo = hi
        digits += 1
    return np.concatenate(out).tobytes() if out else b""


@dataclasses.dataclass
class Workload:
    name: str
    read_len: int
    mate1: np.ndarray            # (n, L) uint8 ASCII
    mate2: np.ndarray | None     # paired end: (n, L)
    preserve_order: bool

    @property
    def bases(self) -> int:
        n = self.mate1.shape[0] * (2 if self.mate2 is not None else 1)
        return n * self.read_len

    def sequences(self) -> np.ndarray:
        """Reads in the order the block splitter numbers them (mates interleaved)."""
        if self.mate2 is None:
            return self.mate1
        n, L = self.mate1.shape
        s = np.empty((2 * n, L), dtype=np.uint8)
        s[0::2] = self.mate1
        s[1::2] = self.mate2
        return s

    def write(self, prefix: str, name: bytes = b"r") -> list[str]:
        """Writes the FASTQ file(s); headers are ``@<name><i>`` (``/1``, ``/2``
        for mates).  Inputs above one 50 MB window need a header of at least 6
        bytes for the block splitter's record-boundary test."""
        if self.mate2 is None:
            p = prefix + ".fastq"
            with open(p, "wb") as f:
                f.write(fastq_bytes(self.mate1, name=name))
            return [p]
        p1, p2 = prefix + "_1.fastq", prefix + "_2.fastq"
        with open(p1, "wb") as f:
            f.write(fastq_bytes(self.mate1, b"/1", name))
        with open(p2, "wb") as f:
            f.write(fastq_bytes(self.mate2, b"/2", name))
        return [p1, p2]


def small_single(seed: int = 0, n_reads: int = 100_000, read_len: int = 100,
                 genome_len: int = 1_000_000, err: float = 0.001,
                 n_rate: float = 0.0001) -> Workload:
    """Single end, uniform i.i.d. genome, 50% reverse complement: the 100k x 100 bp
    case at its default sizes."""
    rng = np.random.default_rng(seed)
    g = random_genome(rng, genome_len)
    r = sample_single(rng, g, n_reads, read_len, err, n_rate)
    return Workload(f"se{read_len}_n{n_reads}_g{genome_len}_s{seed}", read_len, r, None, False)


def paired_repeats(seed: int = 1, pairs: int = 10_000_000, read_len: int = 150,
                   genome_len: int = 50_000_000, err=0.002, n_rate: float = 0.0001,
                   preserve_order: bool = True, ti_tv=None) -> Workload:
    """Paired end, 40% GC genome with 5% covered by 1-5 kbp repeat copies at 1%
    divergence, insert size Normal(400, 50): the 10M-pair x 150 bp case at its
    default sizes."""
    rng = np.random.default_rng(seed)
    g = random_genome(rng, genome_len, gc=0.4, repeat_frac=0.05,
                      repeat_len=(1000, 5000), repeat_div=(0.01, 0.01))
    m1, m2 = sample_paired(rng, g, pairs, read_len, err, n_rate, ti_tv=ti_tv)
    return Workload(f"pe{read_len}_p{pairs}_g{genome_len}_s{seed}", read_len, m1, m2, preserve_order)


def large_combined(seed: int = 4, n_reads: int = 40_000_000, read_len: int = 250,
                   genome_len: int = 200_000_000) -> Workload:
    """Single end, 45% GC genome with 8% covered by 0.5-10 kbp repeat copies at
    0.5-2% divergence, substitutions rising from 0.1% at base 1 to 1.5% at the
    last base, N at 0.02%, preserved order: the 40M x 250 bp case at its
    default sizes."""
    rng = np.random.default_rng(seed)
    g = random_genome(rng, genome_len, gc=0.45, repeat_frac=0.08, repeat_len=(500, 10_000),
                      repeat_div=(0.005, 0.02))
    r = sample_single(rng, g, n_reads, read_len, position_ramp(read_len, 0.001, 0.015), 0.0002)
    return Workload(f"se{read_len}_n{n_reads}_g{genome_len}_s{seed}", read_len, r, None, True)


def position_ramp(read_len: int, lo: float, hi: float) -> np.ndarray:
    """Per-position error rate rising linearly from ``lo`` at base 1 to ``hi``
    at the last base."""
    return np.linspace(lo, hi, read_len)


def batched_specs(seed: int = 2, count: int = 64, scale: float = 1.0):
    """(genome length, read count, read length, error rate) of each block of
    :func:`batched_blocks`, without generating any reads."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        glen = int(rng.integers(2_000_000, 20_000_001) * scale) + 10_000
        n = max(1000, int(np.exp(rng.uniform(np.log(50_000), np.log(5_000_000))) * scale))
        L = int(rng.choice([75, 100, 150, 250]))
        e = float(rng.uniform(0.001, 0.005))
        out.append((glen, n, L, e))
    return out


def batched_block(seed: int, b: int, spec) -> Workload:
    """Block ``b`` of :func:`batched_blocks` from its spec (each block has
    its own generator, so one block can be drawn alone)."""
    glen, n, L, e = spec
    brng = np.random.default_rng([seed, b])
    g = random_genome(brng, glen)
    r = sample_single(brng, g, n, L, e, 0.0001)
    return Workload(f"batch{b}_se{L}_n{n}", L, r, None, False)


def batched_blocks(seed: int = 2, count: int = 64, scale: float = 1.0):
    """Independent single-end blocks from different random genomes (2-20 Mbp),
    read counts log-uniform in [50k, 5M] x ``scale``, read lengths from
    {75, 100, 150, 250}, error rates uniform in [0.1%, 0.5%]."""
    return [batched_block(seed, b, sp) for b, sp in enumerate(batched_specs(seed, count, scale))]
