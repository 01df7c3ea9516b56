"""The drop-in C++ entry points (include/dd_vamana.hpp) compile against types
shaped like the reference's PointRange / Graph / BuildParams / QueryParams /
dataset_para and link the library; run here (no GPU) the program checks the
error path: dd_create fails and reaches the caller's handler."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")
def test_dropin_header_compiles_links_and_reports_errors(tmp_path):
    from distributed_diskann_b200 import _lib

    lib = _lib.load()._name
    exe = tmp_path / "dd_vamana_check"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "dd_vamana_check.cpp"), lib,
                    f"-Wl,-rpath,{os.path.dirname(lib)}", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), str(tmp_path / "graph.bin")], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK"), r.stdout
