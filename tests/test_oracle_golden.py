"""The oracle restatement against golden vectors produced by the reference
APIRL code itself (tests/golden/make_golden.py).  CPU only."""
import hashlib
import json
import os

import numpy as np
import pytest

from apirl_b200 import workloads
from apirl_b200.geometry import ImageGeom, Sino3DGeom

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "golden_small.npz"))
with open(os.path.join(HERE, "golden", "golden_c2.json")) as f:
    C2 = json.load(f)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def bits_equal(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def small_3d():
    return ImageGeom(48, 48, 9, 2.08, 2.08, 2.03), Sino3DGeom.span1(25, 48, 5, 72.0, 5 * 4.054, 150.0, 3)


def test_lor_table_c1(oracle):
    ig, sg = workloads.c1_geometry()
    assert bits_equal(oracle.lor_points_2d(sg.n_proj, sg.n_r, sg.r_fov, sg.r_scanner), G["lor_c1"])


def test_lor_table_c2_hash(oracle):
    ig, sg = workloads.c2_geometry()
    assert sha(oracle.lor_points_2d(sg.n_proj, sg.n_r, sg.r_fov, sg.r_scanner)) == C2["lor_table_sha256"]


def test_phantoms_are_the_golden_ones():
    ig, _ = workloads.c1_geometry()
    assert np.array_equal(workloads.disc_phantom_2d(ig, seed=0), G["c1_phantom"])
    ig, _ = workloads.c2_geometry()
    assert sha(workloads.cylinder_phantom_3d(ig, seed=2)) == C2["phantom_sha256"]


def test_c1_project_bit_exact(oracle):
    ig, sg = workloads.c1_geometry()
    assert bits_equal(oracle.project_2d(sg, ig, G["c1_phantom"]), G["c1_project"])


def test_c1_backproject_bit_exact_serial(oracle):
    ig, sg = workloads.c1_geometry()
    got = oracle.backproject_2d(sg, ig, np.ones(sg.n_bins, np.float32), threads=1)
    assert bits_equal(got, G["c1_backproject_ones"])


def test_c1_mlem60_bit_exact_serial(oracle):
    ig, sg = workloads.c1_geometry()
    img, lik, sens = oracle.mlem_2d(sg, ig, np.ones(ig.n_voxels, np.float32), G["c1_meas"], 60, threads=1)
    assert bits_equal(sens, G["c1_sens"])
    assert bits_equal(img, G["c1_mlem60"])
    assert bits_equal(lik, G["c1_mlem60_lik"])


@pytest.mark.parametrize("sub,ns", [(-1, 1), (0, 4), (3, 4), (2, 5)])
def test_small3d_project_backproject_bit_exact(oracle, sub, ns):
    ig, sg = small_3d()
    key = f"s3_project_{sub}_{ns}".replace("-", "m")
    assert bits_equal(oracle.project_3d(sg, ig, G["s3_image"], sub, ns), G[key])
    v = G[key.replace("project", "bpvalues")]
    got = oracle.backproject_3d(sg, ig, v, sub, ns, threads=1)
    assert bits_equal(got, G[key.replace("project", "backproject")])


def test_small3d_ring_z(oracle):
    ig, sg = small_3d()
    z1, z2 = oracle.sino3d_z(sg)
    rz = G["s3_ringz"]
    rw = np.float32(sg.axial_fov) / np.float32(sg.n_rings)
    za = (rz[:, 0] + rz[:, 1]) / np.float32(2)
    zb = (rz[:, 2] + rz[:, 3]) / np.float32(2)
    # P.Z = z - rw/2 + rw/2 + 0*rw, all in float (SiddonProjector.cpp:394-395)
    za = ((za - rw / np.float32(2)) + rw / np.float32(2)) + np.float32(0) * rw
    zb = ((zb - rw / np.float32(2)) + rw / np.float32(2)) + np.float32(0) * rw
    assert bits_equal(z1, za) and bits_equal(z2, zb)


def test_small3d_osem_bit_exact_serial(oracle):
    ig, sg = small_3d()
    img, lik, sens0 = oracle.osem_3d(sg, ig, np.ones(ig.n_voxels, np.float32), G["s3_meas"], 2, 4, threads=1)
    assert bits_equal(sens0, G["s3_osem_sens0"])
    assert bits_equal(img, G["s3_osem"])
    assert bits_equal(lik, G["s3_osem_lik"])


@pytest.mark.slow
def test_c2_subset0_projection_hash(oracle):
    """Full-size geometry: the oracle's projection of the cylinder phantom for
    subset 0 of 21 (6,779,136 bins, ~2.1e9 Siddon segments) has the same bytes
    as the reference's."""
    ig, sg = workloads.c2_geometry()
    ph = workloads.cylinder_phantom_3d(ig, seed=2)
    p = oracle.project_3d(sg, ig, ph, 0, 21)
    assert p.size == C2["subset0_bins"]
    assert sha(p) == C2["project_phantom_subset0_of21_sha256"]
    ones = oracle.project_3d(sg, ig, np.ones(ig.n_voxels, np.float32), 0, 21)
    assert sha(ones) == C2["project_ones_subset0_of21_sha256"]
