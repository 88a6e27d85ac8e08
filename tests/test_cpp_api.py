"""The C++ host API (hpg_b200/cpp, libhpg.so) on the device: builds
tests/cpp/test_hpg_api.cc against it and runs it (known-answer gridding,
degridding, FFT/shift round trip, copies and error values)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "hpg_b200", "lib")


def build_test_program(out_dir):
    from hpg_b200 import build as b
    b.build()
    exe = os.path.join(out_dir, "test_hpg_api")
    subprocess.run(
        ["g++", "-std=c++17", "-O1", "-Wall",
         "-I" + os.path.join(ROOT, "hpg_b200", "cpp", "include"),
         "-I" + os.path.join(ROOT, "include"),
         os.path.join(ROOT, "tests", "cpp", "test_hpg_api.cc"),
         "-L" + LIB, "-lhpg", "-lhpgb", "-Wl,-rpath," + LIB, "-o", exe],
        check=True)
    return exe


def test_cpp_api_builds(tmp_path):
    assert os.access(build_test_program(str(tmp_path)), os.X_OK)


@pytest.mark.gpu
def test_cpp_api_on_device(tmp_path):
    exe = build_test_program(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("OK")


def test_cpp_indexer(tmp_path):
    """hpgb::CFSimpleIndexer (header only) against the reference's cases."""
    exe = str(tmp_path / "test_indexing")
    subprocess.run(
        ["g++", "-std=c++17", "-O1", "-Wall",
         "-I" + os.path.join(ROOT, "hpg_b200", "cpp", "include"),
         os.path.join(ROOT, "tests", "cpp", "test_indexing.cc"), "-o", exe],
        check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "OK"
