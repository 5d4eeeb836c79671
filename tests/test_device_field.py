"""The device field arithmetic, compiled as host code with nvcc, agrees with
the host field on random and extreme operands (no GPU needed)."""
import json
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent


def nvcc():
    for cand in ("/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    return None


@pytest.mark.skipif(nvcc() is None, reason="nvcc not available")
@pytest.mark.parametrize("source", ["device_field_check.cu", "device_field_check_kb.cu"])
def test_device_field_matches_host_field(tmp_path, source):
    exe = tmp_path / "device_field_check"
    subprocess.run([nvcc(), "-std=c++17", "-O2", "--expt-relaxed-constexpr", "-Xcompiler", "-ffp-contract=off",
                    str(ROOT / source), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert r.returncode == 0 and out["mismatches"] == 0, out
    assert out["checked"] > 1_000_000
