"""Generate the committed golden fixtures from the reference exafmm-dev CPU FMM.

Runs the reference compiled from its own sources (oracle/_ref/parity/*.so, built by
``make -C oracle``) on small seeded workloads and stores what it produced:

* ``kernel_chain.json``: rel-L2 potential error of the P2M -> M2M -> M2L -> L2L -> L2P
  chain against P2P (examples/kernel.cxx) per basis and P, from drand48's unseeded state.
* ``<case>.npz``: bodies, tree cells, body order, M2L / P2P pair lists (sorted) and the
  potential + gradient per body, for each case in CASES.

Usage (needs the reference build): python tests/golden/make_golden.py [case ...]
(no case names: the kernel chain and every case)
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


if __name__ == "__main__":
    main(sys.argv[1:])
