"""Separate target and source sets on the CUDA path: examples/serial.cxx with IneJ (two
trees on the box of their common bounds) and the PetIGA wrapper (each tree on its own box).

The traversal runs from (target root, source root).  Lists are bit-exact against the oracle and the reference's
golden lists (use_ropt = 1 may flip a handful of borderline pairs through powf, as for one
tree); potentials and gradients of the targets within 2e-5 (FP32) / 1e-10 (FP64) of the
oracle and within the method's error of an FP64 direct sum.
"""
import importlib
import json
import os

import numpy as np
import pytest

from oracle import CARTESIAN, SPHERICAL, Oracle, rel_l2

pytestmark = pytest.mark.gpu
fmm = importlib.import_module("exafmm-dev_b200")


def gpu_lists_in_source_tree(s):
    """Lists with the source cells renumbered from the source tree's root (cell 0 there)."""
    roots, _ = s.roots()
    m2l, p2p = s.lists()
    j0 = int(roots[1]) if len(roots) > 1 else 0
    def shift(a):
        return ((a >> 32) << 32) | ((a & 0xffffffff) - j0)
    return np.sort(shift(m2l)), np.sort(shift(p2p))


@pytest.mark.parametrize("basis,P,prec,common", [("spherical", 6, "f64", 1),
                                                 ("spherical", 10, "f32", 1),
                                                 ("cartesian", 5, "f32", 1),
                                                 ("spherical", 8, "f32", 0)])
def test_ij_matches_oracle(basis, P, prec, common, datasets):
    xt, qt = datasets.make("cube", 4000, seed=3, precision=prec)
    xs, qs = datasets.make("plummer", 6000, seed=4, precision=prec)
    xt = xt * 0.5 + 0.25
    kw = dict(ncrit=32, theta=0.4, use_ropt=0)
    s = fmm.Solver(basis=basis, P=P, precision=prec, **kw)
    got = s.solve_ij(xt, qt, xs, qs, common_box=common)
    o = Oracle(prec).run_ij(xt, qt, xs, qs, basis=SPHERICAL if basis == "spherical" else CARTESIAN,
                            P=P, kahan=int(prec == "f32"), common_box=common, **kw)
    m2l, p2p = gpu_lists_in_source_tree(s)
    assert np.array_equal(m2l, np.sort(o.m2l()))
    assert np.array_equal(p2p, np.sort(o.p2p()))
    pot, acc = rel_l2(got, o.trg())
    tol = 2e-5 if prec == "f32" else 1e-10
    assert pot < tol and acc < tol, (pot, acc)
    d = Oracle("f64").direct(xt[:128], xs, qs)
    gp, ga = rel_l2(got[:128], d)
    op, oa = rel_l2(o.trg()[:128], d)
    assert gp < 1.05 * op + 2e-6 and ga < 1.05 * oa + 2e-6, (gp, ga, op, oa)


def test_ij_golden_reference(golden_dir):
    g = np.load(os.path.join(golden_dir, "sph_p8_f32k_ij.npz"))
    p = json.loads(str(g["params"]))
    s = fmm.Solver(P=8, theta=p["theta"], ncrit=p["ncrit"], use_ropt=p["use_ropt"])
    got = s.solve_ij(g["xt"], g["qt"], g["xs"], g["qs"])
    m2l, p2p = gpu_lists_in_source_tree(s)
    diff = len(np.setxor1d(m2l, g["m2l"])) + len(np.setxor1d(p2p, g["p2p"]))
    assert diff <= 2, diff
    pot, acc = rel_l2(got, g["trg"])
    assert pot < 5e-5 and acc < 5e-5, (pot, acc)


def test_ij_edge_cases_and_device_entry(datasets):
    s = fmm.Solver(P=6, theta=0.4, ncrit=16, use_ropt=0, precision="f64")
    xt, qt = datasets.make("cube", 500, seed=5, precision="f64")
    xs, qs = datasets.make("cube", 700, seed=6, precision="f64")
    # no sources: zero field; no targets: nothing
    assert np.array_equal(s.solve_ij(xt, qt, xs[:0], qs[:0]), np.zeros((500, 4)))
    assert s.solve_ij(xt[:0], qt[:0], xs, qs).shape == (0, 4)
    # targets that coincide with sources: the coincident pairs are skipped (r^2 = 0)
    got = s.solve_ij(xs[:300], qs[:300], xs, qs)
    ref = fmm.Solver(P=6, theta=0.4, ncrit=16, use_ropt=0, precision="f64")
    d = Oracle("f64").direct(xs[:300], xs, qs)
    assert rel_l2(got, d)[0] < 1e-3
    # device entry: bitwise the host entry
    import torch
    dt = torch.tensor(np.concatenate([xt, qt[:, None]], 1), dtype=torch.float64, device="cuda")
    ds = torch.tensor(np.concatenate([xs, qs[:, None]], 1), dtype=torch.float64, device="cuda")
    out = torch.empty_like(dt)
    lib = fmm.load_library()
    assert lib.fmm_b200_solve_ij_device(ref.h, len(qt), dt.data_ptr(), len(qs), ds.data_ptr(),
                                        1, out.data_ptr()) == fmm.FMM_OK
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), ref.solve_ij(xt, qt, xs, qs))
    with pytest.raises(fmm.FmmError) as e:
        fmm.Solver(P=6, images=1).solve_ij(xt, qt, xs, qs)
    assert e.value.code == fmm.FMM_ERR_NOT_SUPPORTED


def test_petiga_wrapper(datasets):
    """wrappers/petiga.cxx through libexafmm_b200_petiga.so: each interaction adds the
    potential per unit target charge of the one-tree (B2B, V2B) or two-tree (V2B, B2V, each
    tree on its own box) solve, bitwise what the C ABI gives for the same configuration."""
    import ctypes as C
    lib = C.CDLL(os.path.join(os.path.dirname(fmm.LIB_PATH), "libexafmm_b200_petiga.so"))
    D = C.POINTER(C.c_double)
    xb, qb = datasets.make("cube", 3000, seed=11, precision="f32")
    xv, qv = datasets.make("plummer", 2000, seed=12, precision="f32")
    xv = xv * 0.3
    cols = lambda a: [np.ascontiguousarray(a[:, d]) for d in range(3)]
    bx, vx = cols(xb), cols(xv)
    ptr = lambda a: a.ctypes.data_as(D)
    lib.FMM_Init.argtypes = [C.c_double, C.c_int, C.c_int, C.c_int] + [D] * 4 + [C.c_int] + [D] * 4
    lib.FMM_Init(0.0, 32, 1, len(qb), *map(ptr, bx), ptr(qb), len(qv), *map(ptr, vx), ptr(qv))
    nb, nv = C.c_int(0), C.c_int(0)
    outb = [np.zeros(len(qb)) for _ in range(4)]
    outv = [np.zeros(len(qv)) for _ in range(4)]
    lib.FMM_Partition(C.byref(nb), *map(ptr, outb), C.byref(nv), *map(ptr, outv))
    assert nb.value == len(qb) and np.array_equal(outb[0], bx[0]) and np.array_equal(outv[3], qv)
    lib.FMM_BuildTree()
    vi_b, vb, vv, vi_v = np.ones(len(qb)), np.zeros(len(qb)), np.zeros(len(qv)), np.ones(len(qv))
    lib.FMM_B2B(ptr(vi_b), ptr(qb), C.c_bool(False))
    lib.FMM_V2B(ptr(vb), ptr(qv), C.c_bool(False))
    lib.FMM_B2V(ptr(vv), ptr(qb), C.c_bool(False))
    lib.FMM_V2V(ptr(vi_v), ptr(qv), C.c_bool(False))
    vd = np.zeros(100)
    lib.Direct(100, *map(ptr, cols(xb[:100])), ptr(vd), len(qv), *map(ptr, vx), ptr(qv))
    lib.FMM_Finalize()
    s = fmm.Solver(P=10, theta=0.4, ncrit=32, nspawn=1000, use_rmax=1, use_ropt=1)
    assert np.array_equal(vi_b, 1 + s.solve(xb, qb)[:, 0])
    assert np.array_equal(vi_v, 1 + s.solve(xv, qv)[:, 0])
    assert np.array_equal(vb, s.solve_ij(xb, np.ones(len(qb)), xv, qv, common_box=False)[:, 0])
    assert np.array_equal(vv, s.solve_ij(xv, np.ones(len(qv)), xb, qb, common_box=False)[:, 0])
    assert np.allclose(vd, fmm.direct(xb[:100], xv, qv)[:, 0], rtol=1e-13, atol=0)
    assert rel_l2(np.stack([vb] * 4, 1), np.stack([Oracle("f64").direct(xb, xv, qv)[:, 0]] * 4, 1))[0] < 1e-4
