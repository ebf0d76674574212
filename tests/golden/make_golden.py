"""Generate the committed golden fixtures from the reference exafmm-dev CPU FMM.

Runs the reference compiled from its own sources (oracle/_ref/parity/*.so, built by
``make -C oracle``) on small seeded workloads and stores what it produced:

* ``kernel_chain.json``: rel-L2 potential error of the P2M -> M2M -> M2L -> L2L -> L2P
  chain against P2P (examples/kernel.cxx) per basis and P, from drand48's unseeded state.
* ``<case>.npz``: bodies, tree cells, body order, M2L / P2P pair lists (sorted) and the
  potential + gradient per body, for each case in CASES.

Usage (needs the reference build): python tests/golden/make_golden.py [case ...]
(no case names: the kernel chain and every case; ``<case>.npz`` of an IneJ case holds the
targets xt, qt, the sources xs, qs, the sorted lists and the targets' potential + gradient)
"""
import importlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)
from oracle import Reference  # noqa: E402

datasets = importlib.import_module("exafmm-dev_b200.datasets")

# name: (reference config, working precision, distribution, n, run kwargs)
CASES = {
    "sph_p6_f64_cube": ("sph_p6_f64", "f64", "cube", 4096,
                        dict(ncrit=64, theta=0.4, use_ropt=0)),
    "sph_p10_f32k_plummer": ("sph_p10_f32k_mass", "f32", "plummer", 8192,
                             dict(ncrit=64, theta=0.35, use_ropt=1)),
    "cart_p5_f32_sphere": ("cart_p5_f32", "f32", "sphere", 8192,
                           dict(ncrit=32, theta=0.5, use_ropt=0)),
    # periodic: the cube [-1, 1]^3 as the unit cell of period 2, three image levels
    "sph_p6_f64_periodic": ("sph_p6_f64", "f64", "cube", 4096,
                            dict(ncrit=32, theta=0.4, use_ropt=0, images=3, cycle=2.0)),
}

# separate target and source sets (examples/serial.cxx IneJ): targets from a cube moved to
# x in [0, 1], sources from a Plummer sphere moved to x in [-1, 0]
IJ_CASES = {
    "sph_p8_f32k_ij": ("sph_p8_f32k_mass", "f32", 3000, 5000,
                       dict(ncrit=32, theta=0.4, use_ropt=1)),
}

CHAIN = [("sph_p4_f64", "spherical", 4), ("sph_p6_f64", "spherical", 6),
         ("sph_p8_f64", "spherical", 8), ("sph_p10_f64", "spherical", 10),
         ("cart_p4_f64", "cartesian", 4), ("cart_p5_f64", "cartesian", 5),
         ("cart_p6_f64", "cartesian", 6)]


def main(names):
    if not names:
        chain = {}
        for cfg, basis, P in CHAIN:
            chain["%s_p%d" % (basis, P)] = Reference(cfg).kernel_chain(-1)
        with open(os.path.join(HERE, "kernel_chain.json"), "w") as f:
            json.dump(chain, f, indent=1, sort_keys=True)
    for name, (cfg, prec, dist, n, kw) in CASES.items():
        if names and name not in names:
            continue
        x, q = datasets.make(dist, n, precision=prec)
        run = Reference(cfg).run(x, q, **kw)
        cells = run.cells()
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"), x=x, q=q, order=run.order(),
            m2l=np.sort(run.m2l()), p2p=np.sort(run.p2p()), trg=run.trg(),
            params=json.dumps(dict(config=cfg, precision=prec, dist=dist, n=n, **kw)),
            **{"cell_" + k: v for k, v in cells.items()})
        print(name, run.num_cells, "cells", len(run.m2l()), "M2L", len(run.p2p()), "P2P")


def ij_bodies(nt, ns, precision):
    xt, qt = datasets.make("cube", nt, seed=1, precision=precision)
    xs, qs = datasets.make("plummer", ns, seed=2, precision=precision)
    xt = xt.copy()
    xs = xs.copy()
    xt[:, 0] = (xt[:, 0] + 1) * 0.5
    xs[:, 0] = (xs[:, 0] - 1) * 0.5
    if precision == "f32":
        xt = xt.astype(np.float32).astype(np.float64)
        xs = xs.astype(np.float32).astype(np.float64)
    return xt, qt, xs, qs


def main_ij(names):
    for name, (cfg, prec, nt, ns, kw) in IJ_CASES.items():
        if names and name not in names:
            continue
        xt, qt, xs, qs = ij_bodies(nt, ns, prec)
        run = Reference(cfg).run_ij(xt, qt, xs, qs, **kw)
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"), xt=xt, qt=qt, xs=xs, qs=qs,
            m2l=np.sort(run.m2l()), p2p=np.sort(run.p2p()), trg=run.trg(),
            params=json.dumps(dict(config=cfg, precision=prec, nt=nt, ns=ns, **kw)))
        print(name, len(run.m2l()), "M2L", len(run.p2p()), "P2P")


if __name__ == "__main__":
    names = sys.argv[1:]
    if not names:
        main([])
        main_ij([])
    else:
        if any(a in CASES for a in names):
            main([a for a in names if a in CASES])
        if any(a in IJ_CASES for a in names):
            main_ij([a for a in names if a in IJ_CASES])
