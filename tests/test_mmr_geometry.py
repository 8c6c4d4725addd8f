"""Siemens Biograph mMR geometry against the reference compiled from its
sources (Sinogram3DSiemensMmr / Sinogram2DinSiemensMmr,
data/src/Sinogram3DSiemensMmr.cpp, data/src/Sinogram2DinSiemensMmr.cpp).

* the LOR end-point table built on the host by the library
  (apirl_mmr_lor_table) equals the reference's getPointsFromLor bit for bit,
  and the end-point z equal the reference's, for full-size and reduced mMR
  sinograms;
* the oracle's table-driven projector on those tables equals the reference's
  projection (masked loops) bit for bit, and its serial backprojection the
  reference's SiddonProjector::Backproject.

CPU only; runs where oracle/_ref was built.
"""
import ctypes
import os

import numpy as np
import pytest

from apirl_b200.geometry import ImageGeom, Sino3DGeom

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "apirl_b200", "_build", "libapirl_b200.so")


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a, np.float32).view(np.uint32),
                          np.ascontiguousarray(b, np.float32).view(np.uint32))


def lib_tables(sg):
    L = ctypes.CDLL(LIB)
    lor = np.zeros((sg.n_proj, sg.n_r, 4), np.float32)
    assert L.apirl_mmr_lor_table(sg.n_proj, sg.n_r, lor.ctypes.data_as(ctypes.c_void_p)) == 0
    mn = (ctypes.c_int * sg.n_segments)(*sg.min_rd)
    mx = (ctypes.c_int * sg.n_segments)(*sg.max_rd)

    class G(ctypes.Structure):
        _fields_ = [("n_proj", ctypes.c_int), ("n_r", ctypes.c_int), ("n_rings", ctypes.c_int),
                    ("n_segments", ctypes.c_int), ("r_fov", ctypes.c_float), ("axial_fov", ctypes.c_float),
                    ("r_scanner", ctypes.c_float), ("min_ring_diff", ctypes.POINTER(ctypes.c_int)),
                    ("max_ring_diff", ctypes.POINTER(ctypes.c_int)), ("scanner", ctypes.c_int)]
    g = G(sg.n_proj, sg.n_r, sg.n_rings, sg.n_segments, 297.0, 260.0, 328.0,
          ctypes.cast(mn, ctypes.POINTER(ctypes.c_int)), ctypes.cast(mx, ctypes.POINTER(ctypes.c_int)), 1)
    z = np.zeros((sg.n_sinos, 2), np.float32)
    L.apirl_sino3d_ring_z.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    assert L.apirl_sino3d_ring_z(ctypes.byref(g), z.ctypes.data_as(ctypes.c_void_p)) == sg.n_sinos
    return lor, z


@pytest.mark.parametrize("n_proj,n_r,rings,span,maxrd", [(252, 344, 64, 11, 60), (42, 86, 16, 5, 12),
                                                         (21, 344, 8, 1, 3)])
def test_mmr_tables_equal_reference(ref, n_proj, n_r, rings, span, maxrd):
    sg = Sino3DGeom.mmr(n_proj, n_r, rings, span, maxrd)
    h = ref.mmr_sino3d(sg)
    want_lor, want_z = ref.mmr_tables(h, sg)
    lor, z = lib_tables(sg)
    assert bits_equal(lor, want_lor)
    assert bits_equal(z, want_z)


def test_mmr_projection_oracle_equals_reference(oracle, ref):
    sg = Sino3DGeom.mmr(36, 86, 8, 3, 4)
    ig = ImageGeom(72, 72, 16, 8.35, 8.35, 16.25)  # the 594 mm x 260 mm field of view, coarse voxels
    rng = np.random.default_rng(3)
    img = rng.random(ig.n_voxels, dtype=np.float32)
    h = ref.mmr_sino3d(sg)
    lor, z = ref.mmr_tables(h, sg)
    assert bits_equal(oracle.project_3d_tables(lor, z, ig, img), ref.mmr_project(h, sg, ig, img))
    v = rng.random(sg.n_bins, dtype=np.float32)
    v[rng.random(v.size) < 0.3] = 0
    ref.set_threads(1)
    try:
        assert bits_equal(oracle.backproject_3d_tables(lor, z, ig, v), ref.mmr_backproject(h, sg, ig, v))
    finally:
        ref.set_threads(os.cpu_count() or 1)
