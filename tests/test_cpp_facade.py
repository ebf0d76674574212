"""The C++ facade (include/exafmm_b200.hpp) compiles against the reference's call sequences
(examples/serial.cxx; examples/kernel.cxx through namespace kernel) and, on a GPU,
reproduces the direct sum and the reference's kernel-chain errors."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "exafmm-dev_b200")


def build(tmp_path, name="serial_example"):
    exe = tmp_path / name
    subprocess.check_call(["/usr/bin/g++", "-O2", "-std=c++17", "-Wall", "-Werror",
                           "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "native", name + ".cpp"),
                           "-L", LIBDIR, "-lexafmm_b200", "-Wl,-rpath," + LIBDIR, "-o", str(exe)])
    return exe


def test_facade_compiles_and_links(tmp_path):
    assert build(tmp_path).exists()
    assert build(tmp_path, "kernel_example").exists()


@pytest.mark.gpu
def test_facade_kernel_chain(tmp_path):
    """examples/kernel.cxx through namespace kernel: the reference's chain errors
    (tests/golden/kernel_chain.json) for spherical P = 4..10 and Cartesian P = 4..6."""
    exe = build(tmp_path, "kernel_example")
    with open(os.path.join(ROOT, "tests", "golden", "kernel_chain.json")) as f:
        gold = json.load(f)
    for key, val in sorted(gold.items()):
        basis, P = key.split("_p")
        r = subprocess.run([str(exe), basis, P, "f64"], capture_output=True, text=True,
                           timeout=120)
        assert r.returncode == 0, r.stdout + r.stderr
        p, err = r.stdout.split()
        assert int(p) == int(P) and abs(float(err) - val) <= 2e-3 * val, (key, err, val)


@pytest.mark.gpu
def test_facade_serial_sequence(tmp_path):
    exe = build(tmp_path)
    r = subprocess.run([str(exe), "30000"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "pot" in r.stdout
