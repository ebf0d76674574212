"""Test infrastructure only: ctypes access to the checkers.

* ``Oracle``: the CPU restatement (``liboracle_f32.so`` / ``liboracle_f64.so``) of the
  exafmm-dev Laplace FMM hot path, built from ``fmm_oracle.c`` by ``oracle/Makefile``.
* ``Reference``: the reference exafmm-dev CPU FMM compiled from its own sources into
  ``oracle/_ref/<flavour>/ref_<config>.so`` (only where the reference tree was present at
  build time; the built files travel with the repository snapshot).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this module;
the product path never does.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SPHERICAL, CARTESIAN = 0, 1
TREE_ADAPTIVE, TREE_UNIFORM = 0, 1


class _Params(C.Structure):
    _fields_ = [("basis", C.c_int), ("P", C.c_int), ("theta", C.c_double),
                ("ncrit", C.c_int), ("nspawn", C.c_int), ("use_rmax", C.c_int),
                ("use_ropt", C.c_int), ("mass", C.c_int), ("kahan", C.c_int),
                ("eps2", C.c_double), ("images", C.c_int), ("cycle", C.c_double),
                ("mutual", C.c_int), ("tree", C.c_int)]


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _bind(lib, prefix):
    vp, i, d, ll = C.c_void_p, C.c_int, C.c_double, C.c_longlong
    sig = {
        "num_cells": (i, [vp]), "maxlevel": (i, [vp]), "free": (None, [vp]),
        "get_cells": (None, [vp] + [vp] * 10), "get_order": (None, [vp, vp]),
        "get_expansion": (None, [vp, i, vp]), "get_trg": (None, [vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, prefix + name)
        f.restype, f.argtypes = res, args
    return lib


class _Run:
    """Common accessors over a handle of either checker."""

    def __init__(self, lib, prefix, h, n, nterm, spherical):
        self.lib, self.prefix, self.h, self.n = lib, prefix, h, n
        self.nterm, self.spherical = nterm, spherical

    def _f(self, name):
        return getattr(self.lib, self.prefix + name)

    def __del__(self):
        if getattr(self, "h", None):
            self._f("free")(self.h)
            self.h = None

    @property
    def num_cells(self):
        return self._f("num_cells")(self.h)

    @property
    def maxlevel(self):
        return self._f("maxlevel")(self.h)

    def cells(self):
        nc = self.num_cells
        out = dict(iparent=np.zeros(nc, np.int32), ichild=np.zeros(nc, np.int32),
                   nchild=np.zeros(nc, np.int32), ibody=np.zeros(nc, np.int32),
                   nbody=np.zeros(nc, np.int32), icell=np.zeros(nc, np.uint64),
                   level=np.zeros(nc, np.int32), X=np.zeros((nc, 3)),
                   R_built=np.zeros(nc), R=np.zeros(nc))
        self._f("get_cells")(self.h, *[_ptr(out[k]) for k in
                                       ("iparent", "ichild", "nchild", "ibody", "nbody",
                                        "icell", "level", "X", "R_built", "R")])
        return out

    def order(self):
        o = np.zeros(self.n, np.int32)
        self._f("get_order")(self.h, _ptr(o))
        return o

    def expansion(self, which):
        """which: 0 = M, 1 = L. Spherical -> complex (nc, nterm); Cartesian -> (nc, nterm)."""
        w = 2 if self.spherical else 1
        a = np.zeros(self.num_cells * self.nterm * w)
        self._f("get_expansion")(self.h, which, _ptr(a))
        if self.spherical:
            a = a.reshape(-1, 2)
            return (a[:, 0] + 1j * a[:, 1]).reshape(self.num_cells, self.nterm)
        return a.reshape(self.num_cells, self.nterm)

    def trg(self):
        t = np.zeros(4 * self.n)
        self._f("get_trg")(self.h, _ptr(t))
        return t.reshape(self.n, 4)


class Oracle:
    """The CPU restatement in one working precision ('f32' or 'f64')."""

    def __init__(self, precision="f64"):
        path = os.path.join(HERE, "liboracle_%s.so" % ("f32" if precision == "f32" else "f64"))
        self.lib = _bind(C.CDLL(path), "oracle_")
        L = self.lib
        L.oracle_new.restype = C.c_void_p
        L.oracle_new.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.POINTER(_Params)]
        L.oracle_uniform_level.restype = C.c_int
        L.oracle_uniform_level.argtypes = [C.c_int, C.c_int]
        for f in ("build_tree", "upward", "traverse", "downward", "solve"):
            getattr(L, "oracle_" + f).restype = C.c_int
            getattr(L, "oracle_" + f).argtypes = [C.c_void_p]
        for f in ("num_m2l", "num_p2p"):
            getattr(L, "oracle_" + f).restype = C.c_longlong
            getattr(L, "oracle_" + f).argtypes = [C.c_void_p]
        for f in ("get_m2l", "get_p2p", "get_box"):
            getattr(L, "oracle_" + f).restype = None
            getattr(L, "oracle_" + f).argtypes = [C.c_void_p, C.c_void_p]
        L.oracle_direct.restype = None
        L.oracle_direct.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                    C.c_double, C.c_void_p]
        L.oracle_solve_ij.restype = C.c_int
        L.oracle_solve_ij.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.oracle_direct_periodic.restype = None
        L.oracle_direct_periodic.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                             C.c_void_p, C.c_double, C.c_int, C.c_double,
                                             C.c_void_p]
        L.oracle_rel_l2.restype = None
        L.oracle_rel_l2.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_kernel_chain.restype = C.c_double
        L.oracle_kernel_chain.argtypes = [C.c_int, C.c_int, C.c_int, C.c_long]
        L.oracle_real_bytes.restype = C.c_int
        for f in ("m2l", "m2m", "l2l"):
            getattr(L, "oracle_op_" + f).restype = None
            getattr(L, "oracle_op_" + f).argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 4
        L.oracle_op_p2m.restype = None
        L.oracle_op_p2m.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                    C.c_void_p]
        L.oracle_op_l2p.restype = None
        L.oracle_op_l2p.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                    C.c_void_p, C.c_void_p]
        self.precision = precision

    def run(self, x, q, basis=SPHERICAL, P=6, theta=0.4, ncrit=64, nspawn=1000, use_rmax=1,
            use_ropt=0, mass=0, kahan=0, eps2=0.0, stages=15, images=0, cycle=2 * np.pi,
            mutual=0, tree=TREE_ADAPTIVE):
        x = np.ascontiguousarray(x, np.float64)
        q = np.ascontiguousarray(q, np.float64)
        n = len(q)
        prm = _Params(basis, P, theta, ncrit, nspawn, use_rmax, use_ropt, mass, kahan, eps2,
                      images, cycle, mutual, tree)
        h = self.lib.oracle_new(n, _ptr(x), _ptr(q), C.byref(prm))
        nterm = P * (P + 1) // 2 if basis == SPHERICAL else P * (P + 1) * (P + 2) // 6
        run = OracleRun(self.lib, "oracle_", h, n, nterm, basis == SPHERICAL)
        steps = [(1, "build_tree"), (2, "upward"), (4, "traverse"), (8, "downward")]
        for bit, f in steps:
            if stages & bit:
                rc = getattr(self.lib, "oracle_" + f)(h)
                assert rc == 0, f
        return run

    def direct(self, xt, xs, qs, eps2=0.0):
        xt = np.ascontiguousarray(xt, np.float64)
        xs = np.ascontiguousarray(xs, np.float64)
        qs = np.ascontiguousarray(qs, np.float64)
        out = np.zeros((len(xt), 4))
        self.lib.oracle_direct(len(xt), _ptr(xt), len(xs), _ptr(xs), _ptr(qs), eps2, _ptr(out))
        return out

    def run_ij(self, xt, qt, xs, qs, basis=SPHERICAL, P=6, theta=0.4, ncrit=64, nspawn=1000,
               use_rmax=1, use_ropt=0, mass=0, kahan=0, eps2=0.0, common_box=1):
        """Targets and sources in two trees (oracle_solve_ij); the returned run holds the
        targets' tree, lists (source cells of the source tree) and results."""
        xt = np.ascontiguousarray(xt, np.float64)
        qt = np.ascontiguousarray(qt, np.float64)
        xs = np.ascontiguousarray(xs, np.float64)
        qs = np.ascontiguousarray(qs, np.float64)
        prm = _Params(basis, P, theta, ncrit, nspawn, use_rmax, use_ropt, mass, kahan, eps2, 0,
                      2 * np.pi, 0, TREE_ADAPTIVE)
        hi = self.lib.oracle_new(len(qt), _ptr(xt), _ptr(qt), C.byref(prm))
        hj = self.lib.oracle_new(len(qs), _ptr(xs), _ptr(qs), C.byref(prm))
        nterm = P * (P + 1) // 2 if basis == SPHERICAL else P * (P + 1) * (P + 2) // 6
        run = OracleRun(self.lib, "oracle_", hi, len(qt), nterm, basis == SPHERICAL)
        run._jsrc = OracleRun(self.lib, "oracle_", hj, len(qs), nterm, basis == SPHERICAL)
        assert self.lib.oracle_solve_ij(hi, hj, common_box) == 0
        return run

    def direct_periodic(self, xt, xs, qs, images, cycle, eps2=0.0):
        """FP64 direct sum over the periodic images Traversal::direct visits."""
        xt = np.ascontiguousarray(xt, np.float64)
        xs = np.ascontiguousarray(xs, np.float64)
        qs = np.ascontiguousarray(qs, np.float64)
        out = np.zeros((len(xt), 4))
        self.lib.oracle_direct_periodic(len(xt), _ptr(xt), len(xs), _ptr(xs), _ptr(qs), eps2,
                                        images, cycle, _ptr(out))
        return out

    def kernel_chain(self, basis, P, mass=0, seed=-1):
        return self.lib.oracle_kernel_chain(basis, P, mass, seed)

    # single operators (kernel::M2L / M2M / L2L / P2M / L2P on hand-made cells, unnormalised
    # multipoles); expansions as flat doubles (spherical: re, im per coefficient)
    def op_m2l(self, basis, P, Xi, Xj, Mj, Li):
        Li = np.array(Li, np.float64)
        self.lib.oracle_op_m2l(basis, P, _ptr(np.asarray(Xi, np.float64)),
                               _ptr(np.asarray(Xj, np.float64)),
                               _ptr(np.ascontiguousarray(Mj, np.float64)), _ptr(Li))
        return Li

    def op_m2m(self, basis, P, Xp, Xc, Mc, Mp):
        Mp = np.array(Mp, np.float64)
        self.lib.oracle_op_m2m(basis, P, _ptr(np.asarray(Xp, np.float64)),
                               _ptr(np.asarray(Xc, np.float64)),
                               _ptr(np.ascontiguousarray(Mc, np.float64)), _ptr(Mp))
        return Mp

    def op_l2l(self, basis, P, Xc, Xp, Lp, Lc):
        Lc = np.array(Lc, np.float64)
        self.lib.oracle_op_l2l(basis, P, _ptr(np.asarray(Xc, np.float64)),
                               _ptr(np.asarray(Xp, np.float64)),
                               _ptr(np.ascontiguousarray(Lp, np.float64)), _ptr(Lc))
        return Lc

    def op_p2m(self, basis, P, Xc, xq, M):
        M = np.array(M, np.float64)
        xq = np.ascontiguousarray(xq, np.float64)
        self.lib.oracle_op_p2m(basis, P, _ptr(np.asarray(Xc, np.float64)), len(xq), _ptr(xq),
                               _ptr(M))
        return M

    def op_l2p(self, basis, P, Xc, L, x):
        x = np.ascontiguousarray(x, np.float64)
        out = np.zeros((len(x), 4))
        self.lib.oracle_op_l2p(basis, P, _ptr(np.asarray(Xc, np.float64)),
                               _ptr(np.ascontiguousarray(L, np.float64)), len(x), _ptr(x),
                               _ptr(out))
        return out

    def uniform_level(self, n, ncrit):
        """Depth of the uniform Morton tree (include/build_tree_omp.h:218)."""
        return self.lib.oracle_uniform_level(n, ncrit)


class OracleRun(_Run):
    def box(self):
        b = np.zeros(4)
        self.lib.oracle_get_box(self.h, _ptr(b))
        return b

    def m2l(self):
        n = self.lib.oracle_num_m2l(self.h)
        a = np.zeros(n, np.int64)
        self.lib.oracle_get_m2l(self.h, _ptr(a))
        return a

    def p2p(self):
        n = self.lib.oracle_num_p2p(self.h)
        a = np.zeros(n, np.int64)
        self.lib.oracle_get_p2p(self.h, _ptr(a))
        return a


def rel_l2(trg, ref):
    """Relative L2 error of potential and gradient (include/verify.h:18-83)."""
    trg = np.asarray(trg, np.float64)
    ref = np.asarray(ref, np.float64)
    pot = np.sqrt(((trg[:, 0] - ref[:, 0]) ** 2).sum() / (ref[:, 0] ** 2).sum())
    acc = np.sqrt(((trg[:, 1:] - ref[:, 1:]) ** 2).sum() / (ref[:, 1:] ** 2).sum())
    return pot, acc


# ----------------------------------------------------------------------------- reference
def reference_path(config, flavour="parity"):
    return os.path.join(HERE, "_ref", flavour, "ref_%s.so" % config)


def have_reference(config="sph_p6_f64", flavour="parity"):
    return os.path.exists(reference_path(config, flavour))


class Reference:
    """The reference exafmm-dev CPU FMM for one compile-time configuration, e.g.
    'sph_p10_f32k_mass' (oracle/Makefile CONFIGS)."""

    _cache = {}

    def __init__(self, config, flavour="parity"):
        key = (config, flavour)
        if key not in Reference._cache:
            lib = _bind(C.CDLL(reference_path(config, flavour)), "ref_")
            lib.ref_run.restype = C.c_void_p
            lib.ref_run.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                    C.c_double, C.c_int, C.c_int, C.c_double, C.c_int,
                                    C.c_int, C.c_int, C.c_int, C.c_int, C.c_double]
            for f in ("P", "nterm", "fp64", "spherical", "mass", "kahan", "uniform"):
                getattr(lib, "ref_" + f).restype = C.c_int
                getattr(lib, "ref_" + f).argtypes = []
            lib.ref_run_ij.restype = C.c_void_p
            lib.ref_run_ij.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                       C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int,
                                       C.c_int, C.c_double, C.c_int]
            lib.ref_num_m2l.restype = C.c_longlong
            lib.ref_num_p2p.restype = C.c_longlong
            lib.ref_get_m2l.argtypes = [C.c_void_p]
            lib.ref_get_p2p.argtypes = [C.c_void_p]
            lib.ref_times.argtypes = [C.c_void_p, C.c_void_p]
            lib.ref_kernel_chain.restype = C.c_double
            lib.ref_kernel_chain.argtypes = [C.c_long]
            Reference._cache[key] = lib
        self.lib = Reference._cache[key]
        L = self.lib
        self.P, self.nterm = L.ref_P(), L.ref_nterm()
        self.fp64, self.spherical = bool(L.ref_fp64()), bool(L.ref_spherical())
        self.mass, self.kahan = bool(L.ref_mass()), bool(L.ref_kahan())
        self.uniform = bool(L.ref_uniform())

    def run(self, x, q, ncrit=64, nspawn=1000, theta=0.4, use_rmax=1, use_ropt=0, eps2=0.0,
            stages=15, record=True, threads=0, images=0, cycle=2 * np.pi, mutual=0):
        x = np.ascontiguousarray(x, np.float64)
        q = np.ascontiguousarray(q, np.float64)
        h = self.lib.ref_run(len(q), _ptr(x), _ptr(q), ncrit, nspawn, theta, use_rmax,
                             use_ropt, eps2, mutual, stages, 1 if record else 0, threads, images,
                             cycle)
        run = RefRun(self.lib, "ref_", h, len(q), self.nterm, self.spherical)
        if record:
            run._m2l = np.zeros(self.lib.ref_num_m2l(), np.int64)
            run._p2p = np.zeros(self.lib.ref_num_p2p(), np.int64)
            self.lib.ref_get_m2l(_ptr(run._m2l))
            self.lib.ref_get_p2p(_ptr(run._p2p))
        return run

    def run_ij(self, xt, qt, xs, qs, ncrit=64, nspawn=1000, theta=0.4, use_rmax=1, use_ropt=0,
               eps2=0.0, common_box=1):
        """Targets and sources in two trees (examples/serial.cxx IneJ); the run's getters
        read the targets."""
        xt = np.ascontiguousarray(xt, np.float64)
        qt = np.ascontiguousarray(qt, np.float64)
        xs = np.ascontiguousarray(xs, np.float64)
        qs = np.ascontiguousarray(qs, np.float64)
        h = self.lib.ref_run_ij(len(qt), _ptr(xt), _ptr(qt), len(qs), _ptr(xs), _ptr(qs), ncrit,
                                nspawn, theta, use_rmax, use_ropt, eps2, common_box)
        run = RefRun(self.lib, "ref_", h, len(qt), self.nterm, self.spherical)
        run._m2l = np.zeros(self.lib.ref_num_m2l(), np.int64)
        run._p2p = np.zeros(self.lib.ref_num_p2p(), np.int64)
        self.lib.ref_get_m2l(_ptr(run._m2l))
        self.lib.ref_get_p2p(_ptr(run._p2p))
        return run

    def kernel_chain(self, seed=-1):
        return self.lib.ref_kernel_chain(seed)


class RefRun(_Run):
    def m2l(self):
        return self._m2l

    def p2p(self):
        return self._p2p

    def times(self):
        t = np.zeros(6)
        self.lib.ref_times(self.h, _ptr(t))
        return dict(zip(("bounds", "tree", "upward", "traverse", "downward", "total"), t))
