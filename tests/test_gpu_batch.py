"""Batched and served OSEM (C ABI apirl_batch_*): every job's result in the
mix equals its result run alone through the plain driver (apirl_osem_3d),
within the reconstruction tolerance 1e-4 relative L2 (the only difference is
the order of fp32 atomic additions)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import apirl_b200 as ap  # noqa: E402
from apirl_b200 import workloads  # noqa: E402
from apirl_b200.batch import Batch, Job, serve  # noqa: E402

DEV = torch.device("cuda:0")


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(np.asarray(b, np.float64)))


def make_jobs(specs):
    jobs = []
    for s in specs:
        ig, sg = workloads.job_geometry(s["n"], s["z"])
        rng = np.random.default_rng(s["seed"])
        x = workloads.random_phantom(ig, rng)
        P = ap.SiddonProjector(ig, sg)
        est = torch.empty(P.num_bins(), dtype=torch.float32, device=DEV)
        P.project(torch.from_numpy(x).to(DEV), est)
        counts = workloads.poisson_counts(est.cpu().numpy(), s["counts"], seed=s["seed"])
        P.close()
        jobs.append(Job(ig, sg, counts, s["iters"], s["nsubsets"], tag=s))
    return jobs


@pytest.fixture(scope="module")
def small_jobs():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    specs = workloads.mixed_job_specs(10, seed=40, sizes=(32, 64), slices=(1, 9, 17), iters=(1, 3), subsets=(3, 7),
                                      counts=(1e4, 1e6))
    return make_jobs(specs)


def test_batch_matches_solo(small_jobs):
    b = Batch(0, budget_bytes=8 << 30)
    res = b.run_all(small_jobs)
    b.close()
    for j, (img, lik) in zip(small_jobs, res):
        solo, solo_lik, _ = ap.osem_3d(j.image_geom, j.sino_geom, j.counts.astype(np.float32),
                                       np.ones(j.image_geom.n_voxels, np.float32), j.iters, j.nsubsets)
        assert np.isfinite(img).all()
        assert rel(img, solo) <= 1e-4, j.tag
        assert np.allclose(lik, solo_lik, rtol=1e-6), j.tag


def test_batch_admission_respects_budget(small_jobs):
    """A budget that holds only the largest job at a time still finishes every
    job, each with the same result."""
    fp = [j.footprint() for j in small_jobs]
    b = Batch(0, budget_bytes=max(fp))
    res = b.run_all(small_jobs[:4])
    b.close()
    b2 = Batch(0, budget_bytes=8 << 30)
    res2 = b2.run_all(small_jobs[:4])
    b2.close()
    for (a, _), (c, _) in zip(res, res2):
        assert rel(a, c) <= 1e-4


def test_oversized_job_is_rejected(small_jobs):
    b = Batch(0, budget_bytes=1024)
    with pytest.raises(ap.ApirlError):
        b.submit(small_jobs[0])
    b.close()


def test_serve_continuous_batching(small_jobs):
    arrivals = np.cumsum(np.random.default_rng(5).exponential(1 / 20.0, len(small_jobs)))
    res, lat, makespan = serve(small_jobs, arrivals, budget_bytes=8 << 30)
    assert (lat > 0).all() and makespan > 0
    for j, (img, _) in zip(small_jobs, res):
        solo, _, _ = ap.osem_3d(j.image_geom, j.sino_geom, j.counts.astype(np.float32),
                                np.ones(j.image_geom.n_voxels, np.float32), j.iters, j.nsubsets)
        assert rel(img, solo) <= 1e-4


def test_batch_big_job_matches_solo():
    """A job whose passes run on their own (2^20 or more bins per pass) and has
    no multiplicative or additive sinogram takes the geometry-image sparse
    pass, beside a small job in the shared launch; both match their solo runs
    (which take the same pass form)."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    specs = [dict(n=128, z=41, seed=7, counts=3e6, iters=2, nsubsets=3),
             dict(n=32, z=9, seed=8, counts=1e5, iters=2, nsubsets=3)]
    jobs = make_jobs(specs)
    P = ap.SiddonProjector(jobs[0].image_geom, jobs[0].sino_geom)
    assert P.num_bins(0, 3) >= 1 << 20
    P.close()
    b = Batch(0, budget_bytes=16 << 30)
    res = b.run_all(jobs)
    b.close()
    for j, (img, lik) in zip(jobs, res):
        solo, solo_lik, _ = ap.osem_3d(j.image_geom, j.sino_geom, j.counts.astype(np.float32),
                                       np.ones(j.image_geom.n_voxels, np.float32), j.iters, j.nsubsets)
        finite = np.isfinite(solo)
        assert np.array_equal(np.isfinite(img), finite), j.tag
        assert rel(img[finite], solo[finite]) <= 1e-4, j.tag
        assert np.allclose(lik[:-1], solo_lik[:-1], rtol=1e-6), j.tag


def test_batch_jobs_with_factors_match_solo():
    """A job with a multiplicative sinogram (its own sensitivity A_s^T a,
    beside the shared G_s of the likelihood) and one with an additive sinogram
    (the likelihood's additive sums per subset), next to a plain one: each
    equals its solo run through apirl_osem_3d."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    specs = [dict(n=32, z=9, seed=11, counts=2e5, iters=2, nsubsets=3),
             dict(n=32, z=9, seed=12, counts=2e5, iters=2, nsubsets=4),
             dict(n=32, z=1, seed=13, counts=5e4, iters=3, nsubsets=5)]
    jobs = make_jobs(specs)
    rng = np.random.default_rng(14)
    jobs[0].mult = (rng.random(jobs[0].counts.size, dtype=np.float32) * 0.5 + 0.5).astype(np.float32)
    jobs[1].add = (rng.random(jobs[1].counts.size, dtype=np.float32) * 0.1).astype(np.float32)
    b = Batch(0, budget_bytes=8 << 30)
    res = b.run_all(jobs)
    b.close()
    for j, (img, lik) in zip(jobs, res):
        solo, solo_lik, _ = ap.osem_3d(j.image_geom, j.sino_geom, j.counts.astype(np.float32),
                                       np.ones(j.image_geom.n_voxels, np.float32), j.iters, j.nsubsets,
                                       mult=j.mult, add=j.add)
        finite = np.isfinite(solo)
        assert np.array_equal(np.isfinite(img), finite), j.tag
        assert rel(img[finite], solo[finite]) <= 1e-4, j.tag
        assert np.allclose(lik, solo_lik, rtol=1e-6), j.tag


def test_batch_shares_geometry_between_subset_splits():
    """Jobs of one geometry with different subset counts (their sensitivity
    images summed from the shared per-angle images) and the same job twice:
    each equals its solo run."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    specs = [dict(n=48, z=9, seed=21 + k, counts=3e5, iters=2, nsubsets=ns) for k, ns in enumerate((3, 5, 7, 5))]
    jobs = make_jobs(specs)
    b = Batch(0, budget_bytes=8 << 30)
    res = b.run_all(jobs)
    res2 = b.run_all(jobs[:2])  # the same geometry again, images already cached
    b.close()
    for j, (img, lik) in zip(jobs + jobs[:2], res + res2):
        solo, solo_lik, _ = ap.osem_3d(j.image_geom, j.sino_geom, j.counts.astype(np.float32),
                                       np.ones(j.image_geom.n_voxels, np.float32), j.iters, j.nsubsets)
        finite = np.isfinite(solo)
        assert np.array_equal(np.isfinite(img), finite), j.tag
        assert rel(img[finite], solo[finite]) <= 1e-4, j.tag
        assert np.allclose(lik, solo_lik, rtol=1e-6), j.tag


def test_job_without_counts_in_a_batch(small_jobs):
    """Empty input in the batch: a job whose counts are all zero (every
    subset's list of bins empty) runs beside jobs with counts, and each
    result equals its solo run (the empty job: the same images, NaN where
    the reference's rule divides 0 by a zero sensitivity, and likelihoods)."""
    ig, sg = workloads.job_geometry(32, 9)
    empty = Job(ig, sg, np.zeros(sg.n_bins, np.uint32), 2, 3, tag="no counts")
    jobs = [small_jobs[0], empty, small_jobs[1]]
    b = Batch(0, budget_bytes=8 << 30)
    res = b.run_all(jobs)
    b.close()
    for j, (img, lik) in zip(jobs, res):
        solo, solo_lik, _ = ap.osem_3d(j.image_geom, j.sino_geom, j.counts.astype(np.float32),
                                       np.ones(j.image_geom.n_voxels, np.float32), j.iters, j.nsubsets)
        assert np.array_equal(np.isnan(img), np.isnan(solo)), j.tag
        fin = ~np.isnan(solo)
        if j is empty:
            assert not img[fin].any() and not solo[fin].any()
        else:
            assert rel(img[fin], solo[fin]) <= 1e-4, j.tag
        assert np.allclose(lik, solo_lik, rtol=1e-6), j.tag


def test_update_rule_positive_sens(small_jobs):
    """update_positive_sens in the batch equals apirl_osem_3d_ex's: the update
    only where sens > 0, so a split whose angles leave voxels uncrossed gives
    finite images (a 24^2 image, 31 angles in 15 subsets of two or three
    angles) where the reference's sens >= 0 gives NaN, in both arms alike."""
    ig, sg = workloads.job_geometry(24, 1)
    rng = np.random.default_rng(9)
    x = workloads.random_phantom(ig, rng)
    P = ap.SiddonProjector(ig, sg)
    est = torch.empty(P.num_bins(), dtype=torch.float32, device=DEV)
    P.project(torch.from_numpy(x).to(DEV), est)
    counts = workloads.poisson_counts(est.cpu().numpy(), 1e5, seed=9)
    P.close()
    nsub = min(15, sg.n_proj)
    jobs = [Job(ig, sg, counts, 2, nsub, update_positive_sens=pos) for pos in (False, True)]
    b = Batch(0, budget_bytes=8 << 30)
    res = b.run_all(jobs + [small_jobs[2]])
    b.close()
    for j, (img, lik) in zip(jobs, res):
        solo, solo_lik, _ = ap.osem_3d(ig, sg, counts.astype(np.float32), np.ones(ig.n_voxels, np.float32), 2, nsub,
                                       update_positive_sens=j.update_positive_sens)
        assert np.array_equal(np.isfinite(img), np.isfinite(solo))
        if j.update_positive_sens:
            assert np.isfinite(img).all()
            assert rel(img, solo) <= 1e-4
            assert np.allclose(lik, solo_lik, rtol=1e-6)


def test_sensitivity_images_returned_as_asked(small_jobs):
    """apirl_recon_options.n_sens_out: the driver writes the first n subsets'
    sensitivity images (osem_3d asks for subset 0's alone unless all_sens),
    the same images as when all are returned, and the same reconstruction
    (two runs: equal up to the order of the fp32 atomic adds)."""
    j = small_jobs[3]
    c = j.counts.astype(np.float32)
    x0 = np.ones(j.image_geom.n_voxels, np.float32)
    img1, lik1, s0 = ap.osem_3d(j.image_geom, j.sino_geom, c, x0, j.iters, j.nsubsets, update_positive_sens=True)
    img2, lik2, sall = ap.osem_3d(j.image_geom, j.sino_geom, c, x0, j.iters, j.nsubsets, update_positive_sens=True,
                                  all_sens=True)
    assert sall.shape == (j.nsubsets, j.image_geom.n_voxels)
    assert s0.shape == sall[0].shape and s0.any()
    assert rel(s0, sall[0]) <= 1e-6
    assert rel(img1, img2) <= 1e-6 and np.allclose(lik1, lik2, rtol=1e-7)
