"""The `curc` command line's argument checks on the CPU (they run before any
GPU work): the same messages and exit codes as the reference's CLI
(src/main.cpp:53-161), compared with the reference binary where it was built
here, and with its messages otherwise."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "curc_b200", "_build", "curc")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
REF = os.path.join(REF_DIR, "curc")


def _cases(d):
    fq, txt = os.path.join(d, "a.fastq"), os.path.join(d, "a.txt")
    return {
        "missing_fastq": (["-c", "-i", os.path.join(d, "missing.fastq"), "-o", "x", "--working_dir", d],
                          "please check the first fastq path (filename extension is .fastq or .fq)"),
        "bad_extension": (["-c", "-i", txt, "-o", "x", "--working_dir", d],
                          "please check the first fastq path (filename extension is .fastq or .fq)"),
        "bad_second": (["-c", "-i", f"{fq},{txt}", "-o", "x", "--working_dir", d],
                       "please check the second fastq path (filename extension is .fastq or .fq)"),
        "three_inputs": (["-c", "-i", f"{fq},{fq},{fq}", "-o", "x", "--working_dir", d], "invalid input path number"),
        "both_modes": (["-c", "-d", "-i", fq, "-o", "x"], "compression and decompression options conflict"),
        "no_dir": (["-c", "-i", fq, "-o", "x", "--working_dir", os.path.join(d, "nodir")], "invalid working dir"),
        "bad_ratio": (["-c", "-i", fq, "-o", "x", "--working_dir", d, "--block_ratio", "1.5"],
                      "block ratio is a float number in the range (0,1]"),
        "archive_extension": (["-d", "-i", fq, "-o", "x", "--working_dir", d],
                              "please check the archive path (filename extension is .curc)"),
        "two_archives": (["-d", "-i", f"{d}/a.curc,{d}/b.curc", "-o", "x", "--working_dir", d],
                         "invalid input path number"),
        "version": (["-v"], "v1.0.0"),
    }


@pytest.mark.parametrize("name", sorted(_cases("/d")))
def test_cli_checks_match_reference(name, tmp_path):
    d = str(tmp_path)
    with open(os.path.join(d, "a.fastq"), "w") as f:
        f.write("@r\nACGT\n+\nIIII\n")
    with open(os.path.join(d, "a.txt"), "w") as f:
        f.write("@r\nACGT\n+\nIIII\n")
    args, message = _cases(d)[name]
    mine = subprocess.run([CLI] + args, capture_output=True, text=True, timeout=60)
    assert mine.returncode == 0
    assert mine.stdout.strip() == message
    if os.path.exists(REF):
        ref = subprocess.run([REF] + args, cwd=REF_DIR, capture_output=True, text=True, timeout=60)
        assert (mine.returncode, mine.stdout) == (ref.returncode, ref.stdout)
