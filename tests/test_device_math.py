"""The device translation operators, built for the host from the same headers the CUDA
kernels use (tests/native/math_host.cpp), against the oracle's single operators.
FP64 both sides: agreement to rounding (1e-11 of the largest coefficient)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from oracle import CARTESIAN, SPHERICAL, Oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def hostlib(tmp_path_factory):
    out = tmp_path_factory.mktemp("mathhost") / "libmathhost.so"
    subprocess.check_call(["/usr/bin/g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-w",
                           "-I", os.path.join(ROOT, "exafmm-dev_b200", "csrc"),
                           os.path.join(ROOT, "tests", "native", "math_host.cpp"), "-o", str(out)])
    lib = C.CDLL(str(out))
    lib.host_op.restype = C.c_int
    lib.host_op.argtypes = [C.c_int] * 3 + [C.c_void_p] * 3 + [C.c_int] + [C.c_void_p] * 2
    return lib


@pytest.fixture(scope="module")
def olib():
    lib = Oracle("f64").lib
    v, i = C.c_void_p, C.c_int
    lib.oracle_op_m2l.argtypes = [i, i, v, v, v, v]
    lib.oracle_op_m2m.argtypes = [i, i, v, v, v, v]
    lib.oracle_op_l2l.argtypes = [i, i, v, v, v, v]
    lib.oracle_op_p2m.argtypes = [i, i, v, i, v, v]
    lib.oracle_op_l2p.argtypes = [i, i, v, v, i, v, v]
    return lib


def p(a):
    return a.ctypes.data_as(C.c_void_p)


def ncoef(basis, P):
    return P * (P + 1) if basis == SPHERICAL else P * (P + 1) * (P + 2) // 6


ORDERS = [(SPHERICAL, P) for P in (4, 5, 6, 7, 8, 9, 10, 12)] + \
         [(CARTESIAN, P) for P in (3, 4, 5, 6, 7)]


def rand_expansion(rng, basis, P):
    e = rng.standard_normal(ncoef(basis, P))
    if basis == SPHERICAL:
        e[1] = 0.0  # M[0] / L[0] real, as P2M and M2M leave them
    return e


@pytest.mark.parametrize("basis,P", ORDERS)
def test_translation_operators(basis, P, hostlib, olib):
    rng = np.random.default_rng(P + 10 * basis)
    nc = ncoef(basis, P)
    for trial in range(4):
        Xa = rng.uniform(-1, 1, 3)
        Xb = Xa + rng.uniform(2, 3, 3) * rng.choice([-1, 1], 3)
        Xc = Xa + rng.uniform(-0.3, 0.3, 3)
        M = rand_expansion(rng, basis, P)
        for op, (fo, A, B) in enumerate([(olib.oracle_op_m2l, Xa, Xb), (olib.oracle_op_m2m, Xa, Xc),
                                         (olib.oracle_op_l2l, Xc, Xa)]):
            ref = np.zeros(nc)
            got = np.zeros(nc)
            fo(basis, P, p(np.ascontiguousarray(A)), p(np.ascontiguousarray(B)), p(M), p(ref))
            rc = hostlib.host_op(basis, P, op, p(np.ascontiguousarray(A)),
                                 p(np.ascontiguousarray(B)), p(M), 0, None, p(got))
            assert rc == 0
            scale = np.abs(ref).max()
            assert np.abs(got - ref).max() <= 1e-11 * scale, (op, np.abs(got - ref).max() / scale)
        # P2M and L2P with bodies around the cell centre
        nb = 7
        xq = np.zeros((nb, 4))
        xq[:, :3] = Xa + rng.uniform(-0.5, 0.5, (nb, 3))
        xq[:, 3] = rng.uniform(0.1, 1, nb)
        ref = np.zeros(nc)
        got = np.zeros(nc)
        olib.oracle_op_p2m(basis, P, p(np.ascontiguousarray(Xa)), nb, p(xq), p(ref))
        hostlib.host_op(basis, P, 3, p(np.ascontiguousarray(Xa)), None, None, nb, p(xq), p(got))
        assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max()
        x = np.ascontiguousarray(xq[:, :3])
        ref = np.zeros((nb, 4))
        got = np.zeros((nb, 4))
        olib.oracle_op_l2p(basis, P, p(np.ascontiguousarray(Xa)), p(M), nb, p(x), p(ref))
        hostlib.host_op(basis, P, 4, p(np.ascontiguousarray(Xa)), None, p(M), nb, p(x), p(got))
        assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max(), np.abs(got - ref).max()
