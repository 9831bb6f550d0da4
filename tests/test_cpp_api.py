"""The C++ mirror of the Swift API (metalfft_b200/MetalFFT.hpp) compiles
against include/mfft.h and, on a GPU, runs the reference-style checks of
tests/cpp/test_api.cpp through libmfft.so."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_api.cpp")
LIBDIR = os.path.join(ROOT, "metalfft_b200")


def _build(tmp_path):
    exe = str(tmp_path / "test_api")
    subprocess.run(["g++", "-std=c++17", "-O1", SRC, "-o", exe, "-L" + LIBDIR, "-lmfft",
                    "-Wl,-rpath," + LIBDIR], check=True)
    return exe


def test_cpp_mirror_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_cpp_mirror_runs(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "OK"
