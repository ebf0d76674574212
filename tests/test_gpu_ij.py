"""Separate target and source sets (examples/serial.cxx with IneJ) on the CUDA path.

Targets and sources are two trees on the box of their common bounds; the traversal runs
from (target root, source root).  Lists are bit-exact against the oracle and the reference's
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


@pytest.mark.parametrize("basis,P,prec", [("spherical", 6, "f64"), ("spherical", 10, "f32"),
                                          ("cartesian", 5, "f32")])
def test_ij_matches_oracle(basis, P, prec, datasets):
    xt, qt = datasets.make("cube", 4000, seed=3, precision=prec)
    xs, qs = datasets.make("plummer", 6000, seed=4, precision=prec)
    xt = xt * 0.5 + 0.25
    kw = dict(ncrit=32, theta=0.4, use_ropt=0)
    s = fmm.Solver(basis=basis, P=P, precision=prec, **kw)
    got = s.solve_ij(xt, qt, xs, qs)
    o = Oracle(prec).run_ij(xt, qt, xs, qs, basis=SPHERICAL if basis == "spherical" else CARTESIAN,
                            P=P, kahan=int(prec == "f32"), **kw)
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
                                        out.data_ptr()) == fmm.FMM_OK
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), ref.solve_ij(xt, qt, xs, qs))
    with pytest.raises(fmm.FmmError) as e:
        fmm.Solver(P=6, images=1).solve_ij(xt, qt, xs, qs)
    assert e.value.code == fmm.FMM_ERR_NOT_SUPPORTED
