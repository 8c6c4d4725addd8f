"""Oracle against the reference compiled from its sources, on fresh random
cases (runs only where oracle/_ref was built).  CPU only."""
import os

import numpy as np
import pytest

from apirl_b200.geometry import ImageGeom, Sino2DGeom, Sino3DGeom


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a, np.float32).view(np.uint32),
                          np.ascontiguousarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_2d(oracle, ref, seed):
    rng = np.random.default_rng(seed)
    nx = int(rng.integers(16, 80))
    ig = ImageGeom(nx, nx, 1, float(rng.uniform(1.0, 3.0)), 0.0, 1.0)
    ig.dy = ig.dx
    rimg = ig.dx * nx / 2
    sg = Sino2DGeom(int(rng.integers(8, 64)), int(rng.integers(8, 96)), float(rimg * rng.uniform(0.6, 1.6)),
                    float(rimg * 3))
    img = rng.random(ig.n_voxels, dtype=np.float32)
    assert bits_equal(oracle.project_2d(sg, ig, img), ref.project_2d(sg, ig, img))
    v = rng.random(sg.n_bins, dtype=np.float32)
    ref.set_threads(1)
    try:
        assert bits_equal(oracle.backproject_2d(sg, ig, v, threads=1), ref.backproject_2d(sg, ig, v))
    finally:
        ref.set_threads(os.cpu_count() or 1)


@pytest.mark.parametrize("seed", [4, 5])
def test_random_3d(oracle, ref, seed):
    rng = np.random.default_rng(seed)
    nx = int(rng.integers(16, 40))
    nz = int(rng.integers(3, 12))
    ig = ImageGeom(nx, nx, nz, 2.0, 2.0, float(rng.uniform(1.5, 3.0)))
    rings = int(rng.integers(2, 7))
    sg = Sino3DGeom.span1(int(rng.integers(6, 20)), int(rng.integers(10, 40)), rings,
                          float(nx * 2.0 / 2 * rng.uniform(0.7, 1.5)), float(ig.dz * nz * rng.uniform(0.8, 1.0)),
                          150.0, int(rng.integers(0, rings)))
    img = rng.random(ig.n_voxels, dtype=np.float32)
    h = ref.sino3d(sg)
    ns = int(rng.integers(1, 4))
    for sub in range(-1, ns):
        a = oracle.project_3d(sg, ig, img, sub, ns)
        b = ref.project_3d(h, sg, ig, img, sub, ns)
        assert bits_equal(a, b)
        v = rng.random(a.size, dtype=np.float32)
        ref.set_threads(1)
        try:
            assert bits_equal(oracle.backproject_3d(sg, ig, v, sub, ns, threads=1), ref.backproject_3d(h, sg, ig, v, sub, ns))
        finally:
            ref.set_threads(os.cpu_count() or 1)
