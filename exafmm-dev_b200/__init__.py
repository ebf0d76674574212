"""exafmm-dev_b200: Python binding of the B200 Laplace FMM (libexafmm_b200.so).

The solver runs entirely on the GPU through the C ABI declared in include/exafmm_b200.h;
this module only marshals arrays.  It mirrors the reference's single-node API surface
(examples/serial.cxx:46-60):

    s = Solver(basis="spherical", P=10, theta=0.35, ncrit=64, precision="f32")
    s.set_bodies(x, q)                 # Bodies (include/types.h:66-72)
    s.build_tree()                     # BoundBox::getBounds + BuildTree::buildTree
    s.upward_pass()                    # UpDownPass::upwardPass
    s.traverse()                       # Traversal::dualTreeTraversal (M2L + P2P)
    s.downward_pass()                  # UpDownPass::downwardPass
    trg = s.trg()                      # (n, 4): phi, dphi/dx, dphi/dy, dphi/dz

or ``s.solve(x, q)`` for the whole sequence.  There is no CPU fallback: without the
built library or a B200 every call raises FmmError.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libexafmm_b200.so")

FMM_OK, FMM_ERR_INVALID, FMM_ERR_CUDA, FMM_ERR_NOT_SUPPORTED = 0, 1, 2, 3
FMM_ERR_NO_MEMORY, FMM_ERR_STATE, FMM_ERR_NO_DEVICE, FMM_ERR_DEVICE = 4, 5, 6, 7
SPHERICAL, CARTESIAN = 0, 1
FP32, FP64 = 0, 1
TREE_ADAPTIVE, TREE_UNIFORM = 0, 1
PHASES = ("bounds", "tree", "upward", "traverse", "m2l", "p2p", "downward", "total")


class FmmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("exafmm_b200 error %d: %s" % (code, msg))
        self.code = code


class Config(C.Structure):
    """fmm_b200_config (include/exafmm_b200.h)."""
    _fields_ = [("basis", C.c_int), ("P", C.c_int), ("theta", C.c_double),
                ("ncrit", C.c_int), ("nspawn", C.c_int), ("use_rmax", C.c_int),
                ("use_ropt", C.c_int), ("precision", C.c_int), ("eps2", C.c_double),
                ("images", C.c_int), ("device", C.c_int), ("cycle", C.c_double),
                ("mutual", C.c_int), ("tree", C.c_int)]


# every entry point of include/exafmm_b200.h with its ctypes signature
_vp, _i, _d, _ll = C.c_void_p, C.c_int, C.c_double, C.c_longlong
SIGNATURES = {
    "fmm_b200_default_config": (_i, [_vp]),
    "fmm_b200_create": (_i, [_vp, _vp]),
    "fmm_b200_destroy": (_i, [_vp]),
    "fmm_b200_set_stream": (_i, [_vp, _vp]),
    "fmm_b200_trim": (_i, [_vp]),
    "fmm_b200_set_periodic": (_i, [_vp, _i, _d]),
    "fmm_b200_set_mutual": (_i, [_vp, _i]),
    "fmm_b200_set_partition": (_i, [_vp, _i, _i]),
    "fmm_b200_get_partition": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "fmm_b200_autotune_ncrit": (_i, [_vp, _vp, _i, _i, _vp, _vp]),
    "fmm_b200_autotune_p2p": (_i, [_vp, _vp, _vp, _i, _i, _vp, _vp]),
    "fmm_b200_solve_ij_host": (_i, [_vp, _i, _vp, _vp, _i, _vp, _vp, _i, _vp, _vp]),
    "fmm_b200_solve_ij_device": (_i, [_vp, _i, _vp, _i, _vp, _i, _vp]),
    "fmm_b200_last_error": (C.c_char_p, [_vp]),
    "fmm_b200_supported_orders": (_i, [_i, _vp, _i]),
    "fmm_b200_solve_device": (_i, [_vp, _i, _vp, _vp]),
    "fmm_b200_solve_host": (_i, [_vp, _i, _vp, _vp, _vp, _vp]),
    "fmm_b200_set_bodies_host": (_i, [_vp, _i, _vp, _vp]),
    "fmm_b200_solve_batch_device": (_i, [_vp, _i, _vp, _vp, _vp]),
    "fmm_b200_solve_batch_host": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp]),
    "fmm_b200_set_bodies_batch_device": (_i, [_vp, _i, _vp, _vp]),
    "fmm_b200_get_roots": (_i, [_vp, _vp, _vp, _vp]),
    "fmm_b200_set_bodies_device": (_i, [_vp, _i, _vp]),
    "fmm_b200_build_tree": (_i, [_vp]),
    "fmm_b200_upward_pass": (_i, [_vp]),
    "fmm_b200_traverse": (_i, [_vp]),
    "fmm_b200_downward_pass": (_i, [_vp]),
    "fmm_b200_get_trg_host": (_i, [_vp, _vp]),
    "fmm_b200_get_trg_device": (_i, [_vp, _vp]),
    "fmm_b200_num_cells": (_i, [_vp, _vp, _vp]),
    "fmm_b200_get_cells": (_i, [_vp] + [_vp] * 9),
    "fmm_b200_get_order": (_i, [_vp, _vp]),
    "fmm_b200_get_box": (_i, [_vp, _vp]),
    "fmm_b200_get_expansion": (_i, [_vp, _i, _vp]),
    "fmm_b200_num_lists": (_i, [_vp, _vp, _vp, _vp]),
    "fmm_b200_get_lists": (_i, [_vp, _vp, _vp]),
    "fmm_b200_get_timings": (_i, [_vp, _vp]),
    "fmm_b200_kernel_set_cells": (_i, [_vp, _i] + [_vp] * 7),
    "fmm_b200_kernel_set_expansion": (_i, [_vp, _i, _vp]),
    "fmm_b200_kernel_set_trg": (_i, [_vp, _vp]),
    "fmm_b200_kernel_get_trg": (_i, [_vp, _vp]),
    "fmm_b200_kernel_p2m": (_i, [_vp, _i, _vp]),
    "fmm_b200_kernel_m2m": (_i, [_vp, _i, _vp]),
    "fmm_b200_kernel_m2l": (_i, [_vp, _i, _vp, _vp, _vp, _i]),
    "fmm_b200_kernel_l2l": (_i, [_vp, _i, _vp]),
    "fmm_b200_kernel_l2p": (_i, [_vp, _i, _vp]),
    "fmm_b200_kernel_p2p": (_i, [_vp, _i, _vp, _vp, _vp, _i, _d]),
    "fmm_b200_server_create": (_i, [_vp, _d, _i, _i, _vp]),
    "fmm_b200_server_submit": (_i, [_vp, _i, _vp, _vp, _i, _vp]),
    "fmm_b200_server_set_theta": (_i, [_vp, _i, _d]),
    "fmm_b200_server_poll": (_i, [_vp, _ll, _vp]),
    "fmm_b200_server_wait": (_i, [_vp, _ll, _vp, _vp, _vp, _vp]),
    "fmm_b200_server_stats": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "fmm_b200_server_profile": (_i, [_vp, _vp, _vp, _vp]),
    "fmm_b200_server_destroy": (_i, [_vp]),
    "fmm_b200_server_trim": (_i, [_vp]),
    "fmm_b200_direct": (_i, [_i, _i, _vp, _i, _vp, _vp, _d, _vp]),
    "fmm_b200_direct_noalloc": (_i, [_i, _i, _vp, _i, _vp, _vp, _d, _vp]),
    "fmm_b200_fp32_peak": (_i, [_i, _vp]),
    "fmm_b200_kernel_launches": (_ll, []),
    "fmm_b200_device_allocations": (_ll, []),
    "FMM_Init": (None, [_i]),
    "FMM_Finalize": (None, []),
    "FMM_Partition": (None, [_vp, _vp, _vp, _vp, _d]),
    "FMM_Coulomb": (None, [_i, _vp, _vp, _vp, _vp, _d]),
    "fmm_init_": (None, [_vp, _vp, _vp]),
    "fmm_finalize_": (None, []),
    "fmm_partition_": (None, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "fmm_coulomb_": (None, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
}

_lib = None


def load_library(path=LIB_PATH):
    """Load libexafmm_b200.so (built by __graft_entry__.build() / make -C csrc)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise FmmError(FMM_ERR_NO_DEVICE, "libexafmm_b200.so is not built (%s)" % path)
        lib = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype, f.argtypes = res, args
        _lib = lib
    return _lib


def supported_orders(basis=SPHERICAL):
    lib = load_library()
    buf = (C.c_int * 64)()
    n = lib.fmm_b200_supported_orders(basis, buf, 64)
    return list(buf[:n])


def direct(xt, xs, qs, eps2=0.0, device=0):
    """FP64 direct sum on the GPU (Traversal::direct + normalize): (nt, 4) phi, grad phi."""
    lib = load_library()
    xt = np.ascontiguousarray(xt, np.float64).reshape(-1, 3)
    xs = np.ascontiguousarray(xs, np.float64).reshape(-1, 3)
    qs = np.ascontiguousarray(qs, np.float64).reshape(-1)
    out = np.zeros((len(xt), 4))
    rc = lib.fmm_b200_direct(device, len(xt), _p(xt), len(xs), _p(xs), _p(qs), eps2, _p(out))
    if rc != FMM_OK:
        raise FmmError(rc, "direct sum failed: " + lib.fmm_b200_last_error(None).decode())
    return out


def _header_define(name, header=os.path.join(HERE, "..", "include", "exafmm_b200.h")):
    """Integer value of a #define in the C header (the one place the C limits are set)."""
    with open(header) as fh:
        for line in fh:
            parts = line.split()
            if len(parts) >= 3 and parts[0] == "#define" and parts[1] == name:
                return int(parts[2])
    raise FmmError(FMM_ERR_INVALID, "%s is not defined in %s" % (name, header))


DIRECT_NOALLOC_MAX_TARGETS = _header_define("FMM_DIRECT_NOALLOC_MAX_TARGETS")
DIRECT_NOALLOC_MAX_SOURCES = _header_define("FMM_DIRECT_NOALLOC_MAX_SOURCES")


def direct_noalloc(xt, xs, qs, eps2=0.0, device=0):
    """direct() for callers that cannot allocate device memory (fmm_b200_direct_noalloc):
    the same result, staged through a static 3.75 MiB device array instead of per-call
    allocations.  At most DIRECT_NOALLOC_MAX_TARGETS targets and DIRECT_NOALLOC_MAX_SOURCES
    sources; calls on one device share the array and must not overlap."""
    lib = load_library()
    xt = np.ascontiguousarray(xt, np.float64).reshape(-1, 3)
    xs = np.ascontiguousarray(xs, np.float64).reshape(-1, 3)
    qs = np.ascontiguousarray(qs, np.float64).reshape(-1)
    out = np.zeros((len(xt), 4))
    rc = lib.fmm_b200_direct_noalloc(device, len(xt), _p(xt), len(xs), _p(xs), _p(qs), eps2,
                                     _p(out))
    if rc != FMM_OK:
        raise FmmError(rc, lib.fmm_b200_last_error(None).decode())
    return out


def device_allocations():
    """cudaMalloc calls of the solver handles so far (fmm_b200_device_allocations)."""
    return load_library().fmm_b200_device_allocations()


def fp32_peak_tflops(device=0):
    lib = load_library()
    t = C.c_double()
    rc = lib.fmm_b200_fp32_peak(device, C.byref(t))
    if rc != FMM_OK:
        raise FmmError(rc, "fp32 peak probe failed")
    return t.value


def kernel_launches():
    return load_library().fmm_b200_kernel_launches()


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _basis(b):
    if isinstance(b, str):
        return {"spherical": SPHERICAL, "cartesian": CARTESIAN}[b.lower()]
    return int(b)


def _prec(p):
    if isinstance(p, str):
        return {"f32": FP32, "fp32": FP32, "f64": FP64, "fp64": FP64}[p.lower()]
    return int(p)


class Solver:
    """One device-resident FMM solver handle (re-entrant per instance)."""

    def __init__(self, basis="spherical", P=10, theta=0.4, ncrit=64, nspawn=1000, use_rmax=1,
                 use_ropt=1, precision="f32", eps2=0.0, images=0, device=0,
                 cycle=2 * np.pi, mutual=0, tree="adaptive"):
        """tree: "adaptive" (BuildTree of include/build_tree_tbb.h) or "uniform" (the uniform
        Morton tree of include/build_tree_omp.h)."""
        self.lib = load_library()
        cfg = Config()
        self.lib.fmm_b200_default_config(C.byref(cfg))
        cfg.basis, cfg.P, cfg.theta, cfg.ncrit = _basis(basis), P, theta, ncrit
        cfg.nspawn, cfg.use_rmax, cfg.use_ropt = nspawn, use_rmax, use_ropt
        cfg.precision, cfg.eps2, cfg.images, cfg.device = _prec(precision), eps2, images, device
        cfg.cycle, cfg.mutual = cycle, mutual
        cfg.tree = {"adaptive": TREE_ADAPTIVE, "uniform": TREE_UNIFORM}[tree]
        self.cfg = cfg
        self.h = C.c_void_p()
        rc = self.lib.fmm_b200_create(C.byref(cfg), C.byref(self.h))
        if rc != FMM_OK:
            raise FmmError(rc, self.lib.fmm_b200_last_error(None).decode())
        self.n = 0
        spherical = cfg.basis == SPHERICAL
        self.nterm = P * (P + 1) // 2 if spherical else P * (P + 1) * (P + 2) // 6
        self.spherical = spherical
        self.dtype = np.float32 if cfg.precision == FP32 else np.float64

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.fmm_b200_destroy(h)
            self.h = None

    def close(self):
        self.__del__()

    def trim(self):
        """Free the device buffers the solver has grown out of (fmm_b200_trim)."""
        self._check(self.lib.fmm_b200_trim(self.h))

    def _check(self, rc):
        if rc != FMM_OK:
            raise FmmError(rc, self.lib.fmm_b200_last_error(self.h).decode())

    # ---- configuration
    def autotune_p2p(self, candidates=((8, 16), (4, 16), (0, 16), (8, 8), (4, 8), (0, 0)),
                     repeats=5):
        """On the lists of the last solve, time the P2P at each (lanes4_max, lanes2_max) leaf-size
        threshold pair; the fastest becomes the solver's.  Returns (best pair, {pair: ms})."""
        g4 = np.ascontiguousarray([c[0] for c in candidates], np.int32)
        g2 = np.ascontiguousarray([c[1] for c in candidates], np.int32)
        ms = np.zeros(len(candidates))
        best = C.c_int()
        self._check(self.lib.fmm_b200_autotune_p2p(self.h, _p(g4), _p(g2), len(candidates),
                                                   repeats, C.byref(best), _p(ms)))
        return tuple(candidates[best.value]), {tuple(c): float(t) for c, t in zip(candidates, ms)}

    def autotune_ncrit(self, x=None, q=None, candidates=(16, 32, 48, 64, 96, 128), repeats=3):
        """Time solves of these bodies at each ncrit; the fastest becomes the solver's ncrit.
        Without x, q: the bodies the solver last held (a batch of solves included).
        Returns (best ncrit, {ncrit: median ms})."""
        if x is not None:
            self.set_bodies(x, q)
        cand = np.ascontiguousarray(candidates, np.int32)
        times = np.zeros(len(cand))
        best = C.c_int()
        self._check(self.lib.fmm_b200_autotune_ncrit(self.h, _p(cand), len(cand), repeats,
                                                      C.byref(best), _p(times)))
        self.cfg.ncrit = best.value
        return best.value, dict(zip(cand.tolist(), times.tolist()))

    def set_periodic(self, images, cycle):
        self._check(self.lib.fmm_b200_set_periodic(self.h, images, cycle))

    def set_partition(self, part, nparts):
        """Compute only part `part` of nparts of each following solve (fmm_b200_set_partition):
        the results of the other parts' bodies are 0, and the sum over the nparts handles of
        one node's GPUs, given the same bodies, is the whole solve's result."""
        self._check(self.lib.fmm_b200_set_partition(self.h, part, nparts))

    def partition(self):
        """(part, nparts, first body, end body): this part's bodies in tree order after a solve."""
        v = [C.c_int() for _ in range(4)]
        self._check(self.lib.fmm_b200_get_partition(self.h, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def set_stream(self, stream_handle):
        """Issue work on a cudaStream_t (an int handle, e.g. torch.cuda.Stream.cuda_stream)."""
        self._check(self.lib.fmm_b200_set_stream(self.h, C.c_void_p(stream_handle)))

    # ---- stages
    def set_bodies(self, x, q):
        x = np.ascontiguousarray(x, np.float64).reshape(-1, 3)
        q = np.ascontiguousarray(q, np.float64).reshape(-1)
        self.n = len(q)
        self._check(self.lib.fmm_b200_set_bodies_host(self.h, self.n, _p(x), _p(q)))

    def set_bodies_device(self, n, dev_ptr):
        self.n = n
        self._check(self.lib.fmm_b200_set_bodies_device(self.h, n, C.c_void_p(dev_ptr)))

    def build_tree(self):
        self._check(self.lib.fmm_b200_build_tree(self.h))

    def upward_pass(self):
        self._check(self.lib.fmm_b200_upward_pass(self.h))

    def traverse(self):
        self._check(self.lib.fmm_b200_traverse(self.h))

    def downward_pass(self):
        self._check(self.lib.fmm_b200_downward_pass(self.h))

    def trg(self):
        out = np.zeros((self.n, 4))
        if self.n:
            self._check(self.lib.fmm_b200_get_trg_host(self.h, _p(out)))
        return out

    # ---- whole solves
    def solve(self, x, q):
        """Host arrays in, (n, 4) potential + gradient out (FMM_Coulomb-style call)."""
        x = np.ascontiguousarray(x, np.float64).reshape(-1, 3)
        q = np.ascontiguousarray(q, np.float64).reshape(-1)
        n = len(q)
        p = np.zeros(n)
        f = np.zeros((n, 3))
        self._check(self.lib.fmm_b200_solve_host(self.h, n, _p(x), _p(q), _p(p), _p(f)))
        self.n = n
        return np.concatenate([p[:, None], f], axis=1)

    def solve_ij(self, xt, qt, xs, qs, common_box=True):
        """Targets (xt, qt) against sources (xs, qs) in two trees (examples/serial.cxx IneJ
        with common_box, the petiga wrapper's trees without): (nt, 4) potential and
        gradient per unit target charge."""
        xt = np.ascontiguousarray(xt, np.float64).reshape(-1, 3)
        qt = np.ascontiguousarray(qt, np.float64).reshape(-1)
        xs = np.ascontiguousarray(xs, np.float64).reshape(-1, 3)
        qs = np.ascontiguousarray(qs, np.float64).reshape(-1)
        p = np.zeros(len(qt))
        f = np.zeros((len(qt), 3))
        self._check(self.lib.fmm_b200_solve_ij_host(self.h, len(qt), _p(xt), _p(qt), len(qs),
                                                     _p(xs), _p(qs), int(common_box), _p(p),
                                                     _p(f)))
        self.n = len(qt) + len(qs)
        return np.concatenate([p[:, None], f], axis=1)

    def solve_batch(self, xs, qs):
        """Several independent solves in one batch: lists of (n_s, 3) positions and (n_s,)
        charges; returns a list of (n_s, 4) results."""
        counts = np.array([len(q) for q in qs], np.int32)
        x = np.ascontiguousarray(np.concatenate([np.asarray(a, np.float64).reshape(-1, 3) for a in xs]))
        q = np.ascontiguousarray(np.concatenate([np.asarray(a, np.float64).reshape(-1) for a in qs]))
        n = len(q)
        p = np.zeros(n)
        f = np.zeros((n, 3))
        self._check(self.lib.fmm_b200_solve_batch_host(self.h, len(counts), _p(counts), _p(x),
                                                       _p(q), _p(p), _p(f)))
        self.n = n
        out = np.concatenate([p[:, None], f], axis=1)
        return np.split(out, np.cumsum(counts)[:-1])

    def solve_batch_device(self, counts, bodies_ptr, trg_ptr):
        counts = np.ascontiguousarray(counts, np.int32)
        self.n = int(counts.sum())
        self._check(self.lib.fmm_b200_solve_batch_device(self.h, len(counts), _p(counts),
                                                         C.c_void_p(bodies_ptr),
                                                         C.c_void_p(trg_ptr)))

    def roots(self):
        nr = C.c_int()
        self._check(self.lib.fmm_b200_get_roots(self.h, C.byref(nr), None, None))
        cells = np.zeros(nr.value, np.int32)
        solves = np.zeros(nr.value, np.int32)
        self._check(self.lib.fmm_b200_get_roots(self.h, C.byref(nr), _p(cells), _p(solves)))
        return cells, solves

    def solve_host_ptrs(self, n, x_ptr, q_ptr, p_ptr, f_ptr):
        """solve_host on raw host pointers (pinned buffers for end-to-end timing)."""
        self.n = n
        self._check(self.lib.fmm_b200_solve_host(self.h, n, C.c_void_p(x_ptr), C.c_void_p(q_ptr),
                                                 C.c_void_p(p_ptr), C.c_void_p(f_ptr)))

    def solve_device(self, n, bodies_ptr, trg_ptr):
        """Device 4-vectors (x, y, z, q) in, device 4-vectors out, working precision."""
        self.n = n
        self._check(self.lib.fmm_b200_solve_device(self.h, n, C.c_void_p(bodies_ptr),
                                                   C.c_void_p(trg_ptr)))

    # ---- introspection
    def num_cells(self):
        nc, ml = C.c_int(), C.c_int()
        self._check(self.lib.fmm_b200_num_cells(self.h, C.byref(nc), C.byref(ml)))
        return nc.value, ml.value

    def cells(self):
        nc, _ = self.num_cells()
        out = dict(iparent=np.zeros(nc, np.int32), ichild=np.zeros(nc, np.int32),
                   nchild=np.zeros(nc, np.int32), ibody=np.zeros(nc, np.int32),
                   nbody=np.zeros(nc, np.int32), icell=np.zeros(nc, np.uint64),
                   level=np.zeros(nc, np.int32), X=np.zeros((nc, 3)), R=np.zeros(nc))
        if nc:
            self._check(self.lib.fmm_b200_get_cells(
                self.h, *[_p(out[k]) for k in ("iparent", "ichild", "nchild", "ibody", "nbody",
                                                 "icell", "level", "X", "R")]))
        return out

    def order(self):
        o = np.zeros(self.n, np.int32)
        if self.n:
            self._check(self.lib.fmm_b200_get_order(self.h, _p(o)))
        return o

    def box(self):
        b = np.zeros(4)
        self._check(self.lib.fmm_b200_get_box(self.h, _p(b)))
        return b

    def expansion(self, which):
        """which: 0 = M, 1 = L.  Spherical -> complex (nc, nterm), Cartesian -> (nc, nterm)."""
        nc, _ = self.num_cells()
        w = 2 if self.spherical else 1
        a = np.zeros(nc * self.nterm * w)
        if nc:
            self._check(self.lib.fmm_b200_get_expansion(self.h, which, _p(a)))
        if self.spherical:
            a = a.reshape(-1, 2)
            return (a[:, 0] + 1j * a[:, 1]).reshape(nc, self.nterm)
        return a.reshape(nc, self.nterm)

    # ---- single operators (namespace kernel, include/kernel.h:6-14) -----------------------
    def kernel_set_cells(self, X, R, ibody, nbody, ichild, nchild, iparent):
        """Cells by hand over the bodies of set_bodies (in their given order)."""
        X = np.ascontiguousarray(X, np.float64).reshape(-1, 3)
        arr = [np.ascontiguousarray(a, np.int32) for a in (ibody, nbody, ichild, nchild, iparent)]
        R = np.ascontiguousarray(R, np.float64)
        self._check(self.lib.fmm_b200_kernel_set_cells(self.h, len(X), _p(X), _p(R),
                                                       *[_p(a) for a in arr]))

    def kernel_set_expansion(self, which, values):
        """which 0: M, 1: L; values in the layout expansion() returns (None: zero)."""
        if values is None:
            self._check(self.lib.fmm_b200_kernel_set_expansion(self.h, which, None))
            return
        v = np.asarray(values)
        if self.spherical:
            v = np.stack([v.real, v.imag], axis=-1)
        v = np.ascontiguousarray(v, np.float64)
        self._check(self.lib.fmm_b200_kernel_set_expansion(self.h, which, _p(v)))

    def kernel_set_trg(self, trg=None):
        t = None if trg is None else np.ascontiguousarray(trg, np.float64)
        self._check(self.lib.fmm_b200_kernel_set_trg(self.h, None if t is None else _p(t)))

    def kernel_trg(self):
        """(n, 4) targets of the bodies in cell order."""
        t = np.zeros((self.n, 4))
        self._check(self.lib.fmm_b200_kernel_get_trg(self.h, _p(t)))
        return t

    def _cells(self, name, cells):
        c = np.ascontiguousarray(cells, np.int32)
        self._check(getattr(self.lib, "fmm_b200_kernel_" + name)(self.h, len(c), _p(c)))

    def kernel_p2m(self, cells):
        self._cells("p2m", cells)

    def kernel_m2m(self, cells):
        self._cells("m2m", cells)

    def kernel_l2l(self, cells):
        self._cells("l2l", cells)

    def kernel_l2p(self, cells):
        self._cells("l2p", cells)

    def _pairs(self, ci, cj, image):
        ci = np.ascontiguousarray(ci, np.int32)
        cj = np.ascontiguousarray(cj, np.int32)
        im = None if image is None else np.ascontiguousarray(image, np.int32)
        return ci, cj, im

    def kernel_m2l(self, ci, cj, image=None, mutual=0):
        ci, cj, im = self._pairs(ci, cj, image)
        self._check(self.lib.fmm_b200_kernel_m2l(self.h, len(ci), _p(ci), _p(cj),
                                                 None if im is None else _p(im), mutual))

    def kernel_p2p(self, ci, cj, image=None, mutual=0, eps2=0.0):
        ci, cj, im = self._pairs(ci, cj, image)
        self._check(self.lib.fmm_b200_kernel_p2p(self.h, len(ci), _p(ci), _p(cj),
                                                 None if im is None else _p(im), mutual, eps2))

    def list_counts(self):
        a, b, c = C.c_longlong(), C.c_longlong(), C.c_longlong()
        self._check(self.lib.fmm_b200_num_lists(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def lists(self):
        nm2l, np2p, _ = self.list_counts()
        m2l = np.zeros(nm2l, np.int64)
        p2p = np.zeros(np2p, np.int64)
        self._check(self.lib.fmm_b200_get_lists(self.h, _p(m2l), _p(p2p)))
        return m2l, p2p

    def timings(self):
        t = np.zeros(len(PHASES))
        self._check(self.lib.fmm_b200_get_timings(self.h, _p(t)))
        return dict(zip(PHASES, t))


class Server:
    """Continuous-batching serving loop (fmm_b200_server_*): submit solves of any size and
    order P from any thread; results come back per request with their latency."""

    def __init__(self, basis="spherical", theta=0.4, ncrit=64, nspawn=1000, use_rmax=1,
                 use_ropt=1, precision="f32", hbm_budget_gb=32.0, workers=2, max_batch=256,
                 device=0):
        self.lib = load_library()
        cfg = Config()
        self.lib.fmm_b200_default_config(C.byref(cfg))
        cfg.basis, cfg.theta, cfg.ncrit, cfg.nspawn = _basis(basis), theta, ncrit, nspawn
        cfg.use_rmax, cfg.use_ropt, cfg.precision, cfg.device = use_rmax, use_ropt, _prec(precision), device
        self.h = C.c_void_p()
        rc = self.lib.fmm_b200_server_create(C.byref(cfg), hbm_budget_gb * 1e9, workers, max_batch,
                                             C.byref(self.h))
        if rc != FMM_OK:
            raise FmmError(rc, self.lib.fmm_b200_last_error(None).decode())
        self._n = {}

    def trim(self):
        """Free the buffers the workers' handles grew out of (fmm_b200_server_trim)."""
        rc = self.lib.fmm_b200_server_trim(self.h)
        if rc != FMM_OK:
            raise FmmError(rc, "server trim failed")

    def set_theta(self, P, theta):
        """Opening angle of the requests of order P submitted from now on."""
        rc = self.lib.fmm_b200_server_set_theta(self.h, P, theta)
        if rc != FMM_OK:
            raise FmmError(rc, "set_theta(%r, %r) rejected" % (P, theta))

    def submit(self, x, q, P):
        x = np.ascontiguousarray(x, np.float64).reshape(-1, 3)
        q = np.ascontiguousarray(q, np.float64).reshape(-1)
        rid = C.c_longlong()
        rc = self.lib.fmm_b200_server_submit(self.h, len(q), _p(x), _p(q), P, C.byref(rid))
        if rc != FMM_OK:
            raise FmmError(rc, "submit rejected")
        self._n[rid.value] = len(q)
        return rid.value

    def done(self, rid):
        d = C.c_int()
        rc = self.lib.fmm_b200_server_poll(self.h, rid, C.byref(d))
        if rc != FMM_OK:
            raise FmmError(rc, "unknown request")
        return bool(d.value)

    def wait(self, rid):
        """(n, 4) result, latency seconds, queueing seconds."""
        n = self._n.pop(rid)
        p = np.zeros(n)
        f = np.zeros((n, 3))
        lat, que = C.c_double(), C.c_double()
        rc = self.lib.fmm_b200_server_wait(self.h, rid, _p(p), _p(f), C.byref(lat), C.byref(que))
        if rc != FMM_OK:
            raise FmmError(rc, "request failed")
        return np.concatenate([p[:, None], f], axis=1), lat.value, que.value

    def stats(self):
        a, b, c, d = C.c_longlong(), C.c_longlong(), C.c_longlong(), C.c_int()
        self.lib.fmm_b200_server_stats(self.h, C.byref(a), C.byref(b), C.byref(c), C.byref(d))
        return dict(completed=a.value, bodies=b.value, batches=c.value, pending=d.value)

    def profile(self):
        """Worker seconds: staging inputs, batched solves, copying results out."""
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        self.lib.fmm_b200_server_profile(self.h, C.byref(a), C.byref(b), C.byref(c))
        return dict(stage_s=a.value, solve_s=b.value, unstage_s=c.value)

    def close(self):
        if getattr(self, "h", None):
            self.lib.fmm_b200_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
