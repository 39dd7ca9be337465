"""The restated C-library generator (csrc/crand.h) that draws the HMIS
tie-break weights equals srand/rand of the C library, value for value."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_crand_sequence_equals_rand(tmp_path):
    exe = str(tmp_path / "crand_check")
    subprocess.run(["g++", "-O2", "-I", os.path.join(ROOT, "blood_network_b200", "csrc"), "-o",
                    exe, os.path.join(ROOT, "tests", "c", "crand_check.cpp")], check=True)
    out = subprocess.run([exe, "2000000"], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
