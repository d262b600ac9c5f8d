"""The C++ adapter (include/ses_gpu.hpp) compiled as a reference-style caller
and run against the device, checked against the FP64 oracle."""

import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.gpu
def test_cpp_adapter_end_to_end(tmp_path):
    exe = tmp_path / "adapter_test"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", str(ROOT / "include"), "-I", str(ROOT / "oracle"),
           str(ROOT / "tests" / "cpp" / "adapter_test.cpp"),
           "-L", str(ROOT / "shoeridingerequationsolver_b200"), "-l:libses_b200.so",
           "-L", str(ROOT / "oracle"), "-l:libses_oracle.so",
           f"-Wl,-rpath,{ROOT / 'shoeridingerequationsolver_b200'}:{ROOT / 'oracle'}", "-o", str(exe)]
    subprocess.run(cmd, check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "FAIL" not in r.stdout


def test_cpp_adapter_compiles(tmp_path):
    obj = tmp_path / "adapter_test.o"
    subprocess.run(["g++", "-std=c++17", "-O0", "-Wall", "-Werror", "-c", "-I", str(ROOT / "include"),
                    "-I", str(ROOT / "oracle"), str(ROOT / "tests" / "cpp" / "adapter_test.cpp"),
                    "-o", str(obj)], check=True)
    assert obj.exists()
