"""Host check of the mbarrier parity bookkeeping of the warm-start network's tensor-core kernel
(csrc/mma_phases.h): tests/cpp/mma_phase_check.cpp is compiled with g++ and run. After a bounded wait
gives up at any of the three layers of any tile, the drain before the tensor memory is freed must wait
for exactly the MMA group still in flight."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")


def test_mma_drain_parity_for_every_give_up(tmp_path):
    exe = tmp_path / "mma_phase_check"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
                    str(ROOT / "tests" / "cpp" / "mma_phase_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "of 34 cases pass" in r.stdout
