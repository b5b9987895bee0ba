"""The one-division minmod and superbee limited gradient used by the sweeps
is bit-identical to the reference's two-division formula
(computeAndLimitGradPhi, UtilesRemap.cc:325-357): a host program built by
nvcc from the same device header compares both on about 22 million slope
pairs, random and adversarial (tests/host/limiter_check.cu).  No GPU."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def test_one_division_limiter_is_bit_identical():
    exe = os.path.join(HERE, "host", "_build", "limiter_check")
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "host"), exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mismatches 0" in r.stdout
