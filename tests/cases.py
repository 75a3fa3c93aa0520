"""Seeded synthetic parity cases (small enough for the CPU oracle)."""
import numpy as np

from curc_b200 import synth


def se(seed, n, L, glen, err=0.001, n_rate=0.0001):
    w = synth.small_single(seed=seed, n_reads=n, read_len=L, genome_len=glen, err=err, n_rate=n_rate)
    return w.sequences(), False, False


def pe(seed, pairs, L, glen, po):
    w = synth.paired_repeats(seed=seed, pairs=pairs, read_len=L, genome_len=glen, preserve_order=po)
    return w.sequences(), po, True


def duplicates(seed=7, n=3000, L=100):
    """Many exact duplicates and periodic reads (self overlaps, cycles)."""
    rng = np.random.default_rng(seed)
    base = synth.ACGT[rng.integers(0, 4, size=(n // 10, L))]
    reads = base[rng.integers(0, len(base), size=n)]
    period = np.tile(synth.ACGT[rng.integers(0, 4, size=7)], L // 7 + 1)[:L]
    reads[: n // 20] = period
    return reads.copy(), False, False


CASES = {
    "se100_20k": lambda: se(11, 20_000, 100, 200_000),
    "se75_20k": lambda: se(12, 20_000, 75, 150_000, err=0.003),
    "se150_hiN": lambda: se(13, 10_000, 150, 100_000, err=0.004, n_rate=0.002),
    "se250_8k": lambda: se(14, 8_000, 250, 300_000, err=0.002),
    # a RefMatcher probe in the tail of the last 4-probe segment of the
    # unmapped pseudogenome matches into the zero padding: it must take no hit
    "pe133_po_tail": lambda: (lambda w: (w.sequences(), True, True))(
        synth.paired_repeats(seed=551869, pairs=1585, read_len=133, genome_len=63594, err=0.001, n_rate=0.003,
                             preserve_order=True)),
    # long reads: 10 and 16 words per read
    "se300_4k": lambda: se(19, 4_000, 300, 200_000, err=0.002),
    "se511_2k": lambda: se(20, 2_000, 511, 200_000, err=0.002),
    "pe150_po": lambda: pe(15, 8_000, 150, 400_000, True),
    "pe150": lambda: pe(16, 8_000, 150, 400_000, False),
    "dups": lambda: duplicates(),
    # high coverage: long chains and chain cycles in the assembly, many
    # contested overlap runs
    "se100_deep": lambda: se(18, 100_000, 100, 250_000, err=0.001),
    "pe150_po_100k": lambda: pe(17, 100_000, 150, 2_000_000, True),
}
