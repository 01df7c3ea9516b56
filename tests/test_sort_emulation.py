"""The device sort emulation (csrc/sort_emul.cuh) compiled as host code must
reproduce libstdc++ std::sort's permutation exactly (CPU only)."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_sort_emulation_matches_std_sort(tmp_path):
    exe = tmp_path / "sort_emul_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe),
                    os.path.join(HERE, "cpp", "sort_emul_check.cpp")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("OK"), out.stdout
    assert "heap=1" in out.stdout  # the depth-limit heapsort path was exercised
