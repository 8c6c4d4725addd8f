"""Sampled LORs (several rays per bin): the oracle against the reference
compiled from its sources.  Covers SiddonProjector(nSamples, nAxialSamples)
(recon/src/SiddonProjector.cpp:28-32, 346-397) and
Projector::setMultipleLorsPerBin (recon/inc/Projector.h:54-60) on span-1 and
span-3 sinograms, for Project, Backproject and DivideAndBackproject.  CPU only;
runs where oracle/_ref was built."""
import os

import numpy as np
import pytest

from apirl_b200.geometry import ImageGeom, Sino3DGeom


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a, np.float32).view(np.uint32),
                          np.ascontiguousarray(b, np.float32).view(np.uint32))


def _case(seed, span):
    rng = np.random.default_rng(seed)
    nx = int(rng.integers(16, 36))
    nz = int(rng.integers(5, 12))
    ig = ImageGeom(nx, nx, nz, 2.0, 2.0, float(rng.uniform(1.5, 3.0)))
    rings = int(rng.integers(4, 8))
    rfov = float(nx * 2.0 / 2 * rng.uniform(0.7, 1.2))
    afov = float(ig.dz * nz * rng.uniform(0.8, 1.0))
    nproj, nr = int(rng.integers(6, 16)), int(rng.integers(10, 30))
    if span == 1:
        sg = Sino3DGeom.span1(nproj, nr, rings, rfov, afov, 150.0, int(rng.integers(1, rings)))
    else:
        sg = Sino3DGeom.span(nproj, nr, rings, rfov, afov, 150.0, span, rings - 1)
    return rng, ig, sg


# (ns, nas, multi): the rule for which end points are used differs between
# Project/Backproject (oversampled when ns != 1) and DivideAndBackproject
# (oversampled unless ns == nas == 1); (1, 2, *) exercises that difference.
SAMPLINGS = [(2, 1, 0), (1, 2, 0), (3, 2, 0), (1, 1, 1), (2, 2, 1), (1, 2, 1)]


@pytest.mark.parametrize("span", [1, 3])
@pytest.mark.parametrize("ns,nas,multi", SAMPLINGS)
def test_sampled_vs_reference(oracle, ref, span, ns, nas, multi):
    rng, ig, sg = _case(10 * span + ns + 3 * nas + 7 * multi, span)
    h = ref.sino3d(sg)
    img = rng.random(ig.n_voxels, dtype=np.float32)
    ref.set_threads(1)
    try:
        for sub, nsub in ((-1, 1), (1, 3)):
            a = oracle.sampled_3d(sg, ig, 0, ns, nas, multi, img, subset=sub, nsub=nsub)
            b = ref.sampled_3d(h, sg, ig, 0, ns, nas, multi, img, subset=sub, nsub=nsub)
            assert bits_equal(a, b)
            v = rng.random(a.size, dtype=np.float32)
            v[rng.random(a.size) < 0.2] = 0
            e = rng.random(a.size, dtype=np.float32)
            e[rng.random(a.size) < 0.2] = 0
            bo = oracle.sampled_3d(sg, ig, 1, ns, nas, multi, v, subset=sub, nsub=nsub, threads=1)
            br = ref.sampled_3d(h, sg, ig, 1, ns, nas, multi, v, subset=sub, nsub=nsub)
            assert bits_equal(bo, br)
            do = oracle.sampled_3d(sg, ig, 2, ns, nas, multi, v, e, subset=sub, nsub=nsub, threads=1)
            dr = ref.sampled_3d(h, sg, ig, 2, ns, nas, multi, v, e, subset=sub, nsub=nsub)
            assert bits_equal(do, dr)
    finally:
        ref.set_threads(os.cpu_count() or 1)


def test_single_sample_is_plain(oracle):
    """ns = nas = 1 without multiple LORs is the plain projector, bit for bit."""
    rng, ig, sg = _case(99, 1)
    img = rng.random(ig.n_voxels, dtype=np.float32)
    assert bits_equal(oracle.sampled_3d(sg, ig, 0, 1, 1, 0, img), oracle.project_3d(sg, ig, img))
