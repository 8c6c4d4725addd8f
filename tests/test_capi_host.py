"""The C-ABI library loads and exports every entry point of
include/apirl_b200.h; host-only entry points against golden vectors; argument
checks that fail before any device call.  CPU only."""
import ctypes
import json
import os
import re
import hashlib

import numpy as np
import pytest

import apirl_b200 as ap
from apirl_b200 import _lib, workloads
from apirl_b200.projector import _img_c, _sino3d_c, _sino2d_c

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "apirl_b200.h")
G = np.load(os.path.join(ROOT, "tests", "golden", "golden_small.npz"))
with open(os.path.join(ROOT, "tests", "golden", "golden_c2.json")) as f:
    C2 = json.load(f)


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(apirl_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    return _lib.load()


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"


def test_version(lib):
    assert b"sm_100a" in lib.apirl_version()


def test_lor_table_matches_reference(lib):
    ig, sg = workloads.c1_geometry()
    out = np.zeros((sg.n_proj, sg.n_r, 4), np.float32)
    _lib.check(lib.apirl_lor_table(sg.n_proj, sg.n_r, sg.r_fov, sg.r_scanner, out.ctypes.data_as(ctypes.c_void_p)))
    assert np.array_equal(out.view(np.uint32), G["lor_c1"].view(np.uint32))
    ig, sg = workloads.c2_geometry()
    out = np.zeros((sg.n_proj, sg.n_r, 4), np.float32)
    _lib.check(lib.apirl_lor_table(sg.n_proj, sg.n_r, sg.r_fov, sg.r_scanner, out.ctypes.data_as(ctypes.c_void_p)))
    assert hashlib.sha256(out.tobytes()).hexdigest() == C2["lor_table_sha256"]


def test_ring_z_matches_oracle(lib, oracle):
    for ig, sg in [workloads.c2_geometry(),
                   (None, ap.Sino3DGeom(12, 20, 6, 30.0, 24.0, 100.0, [0, -2, 2], [1, -1, 3]))]:
        sc = _sino3d_c(sg)
        n = lib.apirl_sino3d_ring_z(ctypes.byref(sc), None)
        assert n == sg.n_sinos
        z = np.zeros((n, 2), np.float32)
        lib.apirl_sino3d_ring_z(ctypes.byref(sc), z.ctypes.data_as(ctypes.c_void_p))
        z1, z2 = oracle.sino3d_z(sg)
        assert np.array_equal(z[:, 0].view(np.uint32), z1.view(np.uint32))
        assert np.array_equal(z[:, 1].view(np.uint32), z2.view(np.uint32))


def test_invalid_geometry_is_rejected_without_a_device(lib):
    h = ctypes.c_void_p()
    bad = _lib.ImageGeomC(0, 10, 10, 1.0, 1.0, 1.0)
    sg = _sino2d_c(ap.Sino2DGeom(10, 10, 5.0, 20.0))
    st = lib.apirl_projector_create_2d(ctypes.byref(bad), ctypes.byref(sg), 0, ctypes.byref(h))
    assert st == _lib.APIRL_ERR_INVALID and not h.value
    assert b"image" in lib.apirl_last_error()
    ig = _img_c(ap.ImageGeom(8, 8, 1, 1.0, 1.0, 1.0))
    sg = _sino2d_c(ap.Sino2DGeom(10, 10, 50.0, 20.0))  # rFov beyond the ring
    assert lib.apirl_projector_create_2d(ctypes.byref(ig), ctypes.byref(sg), 0, ctypes.byref(h)) == _lib.APIRL_ERR_INVALID
    s3 = ap.Sino3DGeom(10, 10, 4, 5.0, 10.0, 20.0, [1], [0])  # min > max
    sc = _sino3d_c(s3)
    assert lib.apirl_projector_create_3d(ctypes.byref(ig), ctypes.byref(sc), 0, ctypes.byref(h)) == _lib.APIRL_ERR_INVALID
    assert lib.apirl_projector_num_bins(None, -1, 1) == -1
    with pytest.raises(ap.ApirlError):
        _lib.check(lib.apirl_em_pass(None, None, 0, 0, None, None, None, None, None, 0.0, 1, 0, 1, None, None))
    assert lib.apirl_inverse_divide(-1, None, None, None) == _lib.APIRL_ERR_INVALID
    assert lib.apirl_lor_table(0, 4, 1.0, 2.0, None) == _lib.APIRL_ERR_INVALID


def test_product_never_links_the_oracle():
    """The product library and package do not reference oracle/ code."""
    so = open(_lib.LIB_PATH, "rb").read()
    assert b"liboracle" not in so and b"or_project" not in so and b"ref_harness" not in so
    pkg = os.path.join(ROOT, "apirl_b200")
    for dirpath, _, files in os.walk(pkg):
        for fn in files:
            if fn.endswith((".py", ".cu", ".cuh", ".cpp", ".h")):
                txt = open(os.path.join(dirpath, fn)).read()
                assert "oracle" not in txt.replace("the oracle", ""), os.path.join(dirpath, fn)
