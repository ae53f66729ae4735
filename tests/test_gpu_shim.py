"""GPU test of the C++ drop-in header (include/vine/cspp.hpp): the
reference's call sequence compiled against it and run on the device."""
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def test_cpp_shim_known_answers(tmp_path):
    exe = tmp_path / "shim_main"
    cmd = ["g++", "-std=c++17", "-O2", f"-I{ROOT / 'include'}", str(ROOT / "tests" / "cpp" / "shim_main.cpp"),
           "-o", str(exe), f"-L{ROOT / 'vine_b200'}", "-lvine", f"-Wl,-rpath,{ROOT / 'vine_b200'}"]
    subprocess.run(cmd, check=True)
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
    assert res.stdout.startswith("OK")
