"""The C++ RenderingAlgo adapter over the C ABI, compiled and run as a host program (GPU)."""
import subprocess

import pytest

from naivetrace_b200 import abi

pytestmark = pytest.mark.gpu


def test_cpp_adapter_runs(gpu_lib, tmp_path):
    root = abi.PKG_DIR.parent
    exe = tmp_path / "algo_driver"
    lib_dir = abi.lib_path().parent
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(root / "include"), str(root / "tests" / "cpp" / "algo_driver.cpp"),
                    "-L", str(lib_dir), "-ltoytrace_gpu", f"-Wl,-rpath,{lib_dir}", "-lpthread", "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "complete=3 incomplete=1" in out.stdout
