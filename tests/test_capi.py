"""The C ABI without a GPU: the library loads, exports every entry point that
include/exafmm_b200.h declares, and reports a missing device with a status code."""
import ctypes as C
import importlib
import os
import re

import numpy as np
import pytest

fmm = importlib.import_module("exafmm-dev_b200")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions(header="exafmm_b200.h"):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"^\s*(?:const\s+)?(?:(?:unsigned|long)\s+)*[A-Za-z_][A-Za-z0-9_]*\**\s+\**([A-Za-z_][A-Za-z0-9_]*)\s*\(",
                           src, flags=re.M))
    return sorted(n for n in names if n not in ("defined",))


def test_library_built():
    assert os.path.exists(fmm.LIB_PATH), "run __graft_entry__.build() first"


def test_exports_every_header_symbol():
    lib = C.CDLL(fmm.LIB_PATH)
    names = header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(fmm.SIGNATURES), set(names) ^ set(fmm.SIGNATURES)


def test_defaults_and_orders():
    lib = fmm.load_library()
    cfg = fmm.Config()
    assert lib.fmm_b200_default_config(C.byref(cfg)) == fmm.FMM_OK
    assert (cfg.basis, cfg.P, cfg.ncrit, cfg.nspawn, cfg.use_rmax, cfg.use_ropt) == (0, 10, 64, 1000, 1, 1)
    assert abs(cfg.theta - 0.4) < 1e-15 and cfg.images == 0 and abs(cfg.cycle - 2 * np.pi) < 1e-15
    assert {4, 6, 8, 10} <= set(fmm.supported_orders(fmm.SPHERICAL))
    assert 5 in fmm.supported_orders(fmm.CARTESIAN)
    assert lib.fmm_b200_default_config(None) == fmm.FMM_ERR_INVALID


def test_create_validates_before_touching_a_device():
    lib = fmm.load_library()
    cfg = fmm.Config()
    lib.fmm_b200_default_config(C.byref(cfg))
    h = C.c_void_p()
    cfg.images = 1
    cfg.basis = fmm.CARTESIAN
    cfg.P = 2
    assert lib.fmm_b200_create(C.byref(cfg), C.byref(h)) == fmm.FMM_ERR_INVALID
    assert b"expansion order" in lib.fmm_b200_last_error(None)
    cfg.basis = fmm.SPHERICAL
    cfg.P = 10
    cfg.cycle = 0.0
    assert lib.fmm_b200_create(C.byref(cfg), C.byref(h)) == fmm.FMM_ERR_INVALID
    cfg.images = -1
    cfg.cycle = 1.0
    assert lib.fmm_b200_create(C.byref(cfg), C.byref(h)) == fmm.FMM_ERR_INVALID
    cfg.images = 0
    cfg.P = 99
    assert lib.fmm_b200_create(C.byref(cfg), C.byref(h)) == fmm.FMM_ERR_INVALID
    cfg.P = 10
    cfg.theta = 1.0
    assert lib.fmm_b200_create(C.byref(cfg), C.byref(h)) == fmm.FMM_ERR_INVALID
    for call in ("fmm_b200_build_tree", "fmm_b200_upward_pass", "fmm_b200_traverse",
                 "fmm_b200_downward_pass", "fmm_b200_destroy"):
        assert getattr(lib, call)(None) == fmm.FMM_ERR_INVALID


def test_no_device_is_an_error_not_a_fallback():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(fmm.FmmError) as e:
        fmm.Solver(P=10)
    assert e.value.code == fmm.FMM_ERR_NO_DEVICE


def test_petiga_wrapper_library_exports_its_header():
    """The PetIGA wrapper ABI is its own library (its FMM_* names are the gromacs
    wrapper's); it loads next to libexafmm_b200.so and exports what its header declares."""
    path = os.path.join(os.path.dirname(fmm.LIB_PATH), "libexafmm_b200_petiga.so")
    assert os.path.exists(path)
    lib = C.CDLL(path)
    names = header_functions("exafmm_b200_petiga.h")
    assert set(names) >= {"FMM_Init", "FMM_B2B", "FMM_V2B", "FMM_B2V", "FMM_V2V", "Direct"}
    assert not [n for n in names if not hasattr(lib, n)]
