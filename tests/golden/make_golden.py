"""Generates the golden fixtures in this directory from the reference APIRL CPU
code itself (oracle/_ref/libapirl_ref_harness.so, built from the reference
sources by oracle/ref/Makefile).  Run from the repository root where the
reference tree is available:

    python tests/golden/make_golden.py

Outputs
  golden_small.npz  -- reference outputs on small seeded cases (2D at the full
                       2D-MLEM size, 3D on a 48x48x9 image), all float32.
  golden_c2.json    -- size-independent facts of the full 3D OSEM geometry
                       (256x256x81 image, 1261 sinograms of 336x336): SHA-256
                       of the reference LOR table and sinogram z, of the
                       reference projection of the cylinder phantom for
                       subset 0 of 21, and its sums.

The reference's backprojection accumulates with OpenMP atomics; the harness
runs it single-threaded here so the fixtures are reproducible.
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle_lib import RefHarness  # noqa: E402
from apirl_b200.geometry import ImageGeom, Sino2DGeom, Sino3DGeom  # noqa: E402
from apirl_b200 import workloads  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def small_3d_case():
    """A 3D geometry whose sinogram covers the whole square image (no
    zero-sensitivity corners), with an odd angle count for uneven subsets."""
    ig = ImageGeom(48, 48, 9, 2.08, 2.08, 2.03)
    sg = Sino3DGeom.span1(25, 48, 5, 72.0, 5 * 4.054, 150.0, 3)
    return ig, sg


def main():
    R = RefHarness()
    out = {}
    # ---- 2D at the 2D-MLEM size -------------------------------------------
    ig, sg = workloads.c1_geometry()
    out["lor_c1"] = R.lor_points_2d(sg.n_proj, sg.n_r, sg.r_fov, sg.r_scanner)
    x = workloads.disc_phantom_2d(ig, seed=0)
    out["c1_phantom"] = x
    R.set_threads(1)
    out["c1_project"] = R.project_2d(sg, ig, x)
    ones = np.ones(sg.n_bins, np.float32)
    out["c1_backproject_ones"] = R.backproject_2d(sg, ig, ones)
    meas = workloads.poisson_counts(out["c1_project"], 1e6, seed=0).astype(np.float32)
    out["c1_meas"] = meas
    init = np.ones(ig.n_voxels, np.float32)
    t0 = time.time()
    img, lik, sens = R.mlem_2d(sg, ig, init, meas, 60)
    print(f"reference 2D MLEM 60 iterations: {time.time() - t0:.2f} s")
    out["c1_mlem60"] = img
    out["c1_mlem60_lik"] = lik
    out["c1_sens"] = sens

    # ---- small 3D ----------------------------------------------------------
    ig3, sg3 = small_3d_case()
    rng = np.random.default_rng(7)
    x3 = (rng.random(ig3.n_voxels, dtype=np.float32) + 0.25).astype(np.float32)
    out["s3_image"] = x3
    h = R.sino3d(sg3)
    (z1f, z1l, z2f, z2l), nz = R.ring_z(h, sg3.n_sinos)
    out["s3_ringz"] = np.stack([z1f, z1l, z2f, z2l], 1)
    for sub, ns in [(-1, 1), (0, 4), (3, 4), (2, 5)]:
        key = f"s3_project_{sub}_{ns}".replace("-", "m")
        out[key] = R.project_3d(h, sg3, ig3, x3, sub, ns)
        v = rng.random(out[key].size, dtype=np.float32)
        v[rng.random(v.size) < 0.2] = 0
        out[key.replace("project", "bpvalues")] = v
        out[key.replace("project", "backproject")] = R.backproject_3d(h, sg3, ig3, v, sub, ns)
    # OSEM, 2 iterations x 4 subsets, from counts of the random image
    meas3 = rng.poisson(R.project_3d(h, sg3, ig3, x3) * 3.0).astype(np.float32)
    out["s3_meas"] = meas3
    h2 = R.sino3d(sg3, meas3)
    img3, lik3, sens3 = R.osem_3d(h2, ig3, np.ones(ig3.n_voxels, np.float32), 2, 4)
    out["s3_osem"] = img3
    out["s3_osem_lik"] = lik3
    out["s3_osem_sens0"] = sens3
    R.set_threads(os.cpu_count() or 1)
    np.savez_compressed(os.path.join(HERE, "golden_small.npz"), **out)

    # ---- interfile files written by the reference's own writers ---------------
    iodir = os.path.join(HERE, "ref_io")
    os.makedirs(iodir, exist_ok=True)
    sgio = Sino3DGeom(8, 6, 3, 20.0, 12.0, 60.0, [0, 1, -1], [0, 1, -1])
    vals = (np.arange(sgio.n_bins, dtype=np.float32) * 0.5 - 7).astype(np.float32)
    hio = R.sino3d(sgio, vals)
    R.write_sino3d(hio, os.path.join(iodir, "sino3d"))
    igio = ImageGeom(8, 6, 3, 2.5, 2.0, 3.25)
    R.write_image(igio, (np.arange(igio.n_voxels, dtype=np.float32) * 0.25 + 1).astype(np.float32),
                  os.path.join(iodir, "image"))
    # medcon writes the data file's absolute path; keep the fixture relocatable.
    hp = os.path.join(iodir, "image.h33")
    txt = open(hp, "rb").read().replace(os.path.join(iodir, "image.i33").encode(), b"image.i33")
    open(hp, "wb").write(txt)

    # ---- full 3D OSEM geometry ----------------------------------------------
    ig, sg = workloads.c2_geometry()
    lor = R.lor_points_2d(sg.n_proj, sg.n_r, sg.r_fov, sg.r_scanner)
    t0 = time.time()
    hc = R.sino3d(sg)
    (z1f, z1l, z2f, z2l), nz = R.ring_z(hc, sg.n_sinos)
    ph = workloads.cylinder_phantom_3d(ig, seed=2)
    t1 = time.time()
    proj0 = R.project_3d(hc, sg, ig, ph, 0, 21)
    t2 = time.time()
    ones0 = R.project_3d(hc, sg, ig, np.ones(ig.n_voxels, np.float32), 0, 21)
    print(f"reference full-size subset-0 projection: {t2 - t1:.2f} s")
    facts = {
        "geometry": {"image": [ig.nx, ig.ny, ig.nz, ig.dx, ig.dy, ig.dz],
                     "n_proj": sg.n_proj, "n_r": sg.n_r, "n_rings": sg.n_rings, "r_fov": sg.r_fov,
                     "axial_fov": sg.axial_fov, "r_scanner": sg.r_scanner, "min_rd": sg.min_rd, "max_rd": sg.max_rd,
                     "n_sinos": sg.n_sinos},
        "lor_table_sha256": sha(lor),
        "ringz_first_last_sha256": sha(np.stack([z1f, z1l, z2f, z2l], 1)),
        "phantom_sha256": sha(ph),
        "project_phantom_subset0_of21_sha256": sha(proj0),
        "project_phantom_subset0_of21_sum": float(proj0.astype(np.float64).sum()),
        "project_ones_subset0_of21_sha256": sha(ones0),
        "project_ones_subset0_of21_sum": float(ones0.astype(np.float64).sum()),
        "subset0_bins": int(proj0.size),
    }
    with open(os.path.join(HERE, "golden_c2.json"), "w") as f:
        json.dump(facts, f, indent=1)
    print(json.dumps(facts, indent=1))


if __name__ == "__main__":
    main()
