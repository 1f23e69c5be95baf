"""bench.py's reference arm on the CPU: one JSON line in the contract's
shape for the compact-FD workload (a small grid, two steps), and the
`unavailable` line for the FFT engines, whose FFTW calls the reference
harness can only answer with DFT sums."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(*args):
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", *args], cwd=ROOT, capture_output=True,
                         text=True, timeout=600, check=True).stdout.strip().splitlines()
    return json.loads(out[-1])


def test_reference_arm_line():
    line = _bench("--steps", "2", "--warmup", "1", "--scale", "0.1")
    assert line["impl"] == "reference" and line["unit"] == "Gpts/s" and line["value"] > 0
    assert line["higher_is_better"] is True and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["cores"] >= 1


@pytest.mark.parametrize("workload", ["vti_r2c", "vti_r2r"])
def test_reference_arm_fft_engines_unavailable(workload):
    line = _bench("--workload", workload, "--steps", "2", "--warmup", "1", "--scale", "0.1")
    assert line["impl"] == "reference" and "FFTW" in line["unavailable"]
