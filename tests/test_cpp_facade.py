"""The C++ facade (include/exafmm_b200.hpp) compiles against the reference's call sequence
(examples/serial.cxx) and, on a GPU, reproduces the direct sum."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "exafmm-dev_b200")


def build(tmp_path):
    exe = tmp_path / "serial_example"
    subprocess.check_call(["/usr/bin/g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "native", "serial_example.cpp"),
                           "-L", LIBDIR, "-lexafmm_b200", "-Wl,-rpath," + LIBDIR, "-o", str(exe)])
    return exe


def test_facade_compiles_and_links(tmp_path):
    assert build(tmp_path).exists()


@pytest.mark.gpu
def test_facade_serial_sequence(tmp_path):
    exe = build(tmp_path)
    r = subprocess.run([str(exe), "30000"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "pot" in r.stdout
