"""The parallel stable order of the paired-end position coder and decoder
(curc_b200/csrc/host/stable_order.hpp) is the permutation std::stable_sort
gives, on CPU (tests/helpers/stable_order_check.cpp)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_stable_order_equals_stable_sort(tmp_path):
    exe = str(tmp_path / "stable_order_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-I", os.path.join(ROOT, "curc_b200", "csrc"), "-o", exe,
                    os.path.join(ROOT, "tests", "helpers", "stable_order_check.cpp")], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "stable order ok" in r.stdout
