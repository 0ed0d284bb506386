"""Host logic of the symmetric form's work plan, built against
libinti_b200.so and run on the CPU (no device): every unordered pair of node
blocks covered by exactly one work item across the panels, per-panel row
lists consistent, panel widths within the partial budget
(tests/symm_plan_check.cpp)."""
import shutil
import subprocess
from pathlib import Path

from inti_b200 import _lib as L

ROOT = Path(__file__).resolve().parents[1]


def test_symmetric_plan_and_panels(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    assert cxx, "a C++ compiler is needed"
    exe = tmp_path / "symm_plan_check"
    libdir = L.LIB_PATH.parent
    subprocess.run([cxx, "-O1", "-std=c++17", str(ROOT / "tests" / "symm_plan_check.cpp"), "-L", str(libdir),
                    "-linti_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True, capture_output=True,
                   text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failures" in r.stdout
