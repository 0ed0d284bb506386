"""The C ABI from a plain C host (tests/abi_driver.c, built with gcc against
include/inti_b200.h and linked to libinti_b200.so): what a foreign-function
caller such as Julia's ccall sees.  Without a device the driver must build,
link, load and report "no device" through the status/message path; on the
GPU it checks a 2D Laplace double layer with a 1-based CSC correction over 3
padded columns and a 3D Helmholtz single layer off the surface against its
own direct loops, and a refused shape."""
import shutil
import subprocess
from pathlib import Path

import pytest

from inti_b200 import _lib as L

ROOT = Path(__file__).resolve().parents[1]


def _build(tmp_path) -> Path:
    cc = shutil.which("gcc") or shutil.which("cc")
    assert cc, "a C compiler is needed for the ABI driver"
    exe = tmp_path / "abi_driver"
    libdir = L.LIB_PATH.parent
    cmd = [cc, "-O2", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"),
           str(ROOT / "tests" / "abi_driver.c"), "-L", str(libdir), "-linti_b200", f"-Wl,-rpath,{libdir}", "-lm",
           "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_c_driver_builds_links_and_reports_status(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert "ABI version 1" in r.stdout
    if r.returncode == 77:  # no usable device here: the failure came back as a status and a message
        assert "no context (status 3)" in r.stdout
    else:
        assert r.returncode == 0 and "PASS" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_c_driver_on_device(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "PASS" in r.stdout, r.stdout + r.stderr
