"""The learned coder's host parts, no GPU: the range coder round trip
(tests/helpers/rc_roundtrip.cpp) and the learned stream written from its
coding rules with the host integer model and read back by the decoder the
product uses for learned archive blocks, on random models, pseudogenomes
and records at 75, 150 and 250 bp, corrupt streams included
(tests/helpers/learned_roundtrip.cpp), both against learned_model.hpp."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_range_coder_round_trip(tmp_path):
    exe = str(tmp_path / "rc")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "curc_b200", "csrc"), "-o", exe,
                    os.path.join(ROOT, "tests", "helpers", "rc_roundtrip.cpp")], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "round trips ok" in r.stdout


def test_learned_stream_round_trip(tmp_path):
    exe = str(tmp_path / "lrt")
    subprocess.run(["g++", "-std=c++17", "-O2", "-fopenmp", "-I", os.path.join(ROOT, "curc_b200", "csrc"), "-o", exe,
                    os.path.join(ROOT, "tests", "helpers", "learned_roundtrip.cpp")], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "learned round trips ok" in r.stdout


def test_host_network_form_gives_the_same_frequencies(tmp_path):
    """The decoder's int16 form of the network (model_freqs_host) against the
    integer model on full-range random weights (tests/helpers/host_model_check.cpp)."""
    exe = str(tmp_path / "host_model_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-fopenmp", "-I", os.path.join(ROOT, "curc_b200", "csrc"), "-o", exe,
                    os.path.join(ROOT, "tests", "helpers", "host_model_check.cpp")], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "host model ok" in r.stdout
