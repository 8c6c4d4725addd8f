"""The full-size 3D workload against the oracle (256x256x81 image; 1261
sinograms of 336 angles x 336 r; 21 subsets; attenuation in the
sensitivity; 5e8 Poisson counts as uint32).

* The benchmarked pass, as bench.py runs it: the projector's defaults
  (padded two-layout walk, persistent warps), the geometry image
  G_s = A_s^T 1, the list of the subset's bins with counts, uint32 counts,
  update where sens > 0.  One sub-iteration each for subsets 0, 10 and 20,
  chained on the GPU's own images (each pass starts from the image the
  previous one left), each against the oracle's sub-iteration from the same
  image:
    projection of the input image ...... bit-identical to the oracle's
    sensitivity A_s^T a and G_s ........ rel L2 <= 1e-5 (fp32 atomics' order)
    updated image ...................... rel L2 <= 1e-5
    FP64 likelihood of the full pass ... rel <= 1e-9 against the FP64 sum of
                                         m log e - e over e != 0 of the oracle's
                                         estimates (the same estimates summed
                                         in FP64 in another order)
    FP64 likelihood of the listed pass . rel <= 1e-6 against the same (the sum
                                         over e of the bins without counts
                                         comes from x . G_s, so its rounding
                                         differs)
* The whole job: 3 iterations x 21 subsets through apirl_osem_3d (sensitivity
  A_s^T a, update where sens > 0) against the oracle's OSEM with the same
  rule: rel L2 <= 1e-4.
* The batch engine on the same job (1 iteration x 21 subsets) against
  apirl_osem_3d: rel L2 <= 1e-4, likelihoods to 1e-6.

Marked slow: the oracle runs on the host cores (about a minute for the
sub-iterations, a few minutes for the whole job on 16 threads).
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.slow]

import apirl_b200 as ap  # noqa: E402
from apirl_b200 import _lib, workloads  # noqa: E402

DEV = torch.device("cuda:0")
NSUB = 21


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a, np.float32).view(np.uint32),
                          np.ascontiguousarray(b, np.float32).view(np.uint32))


def fp64_likelihood(est, meas):
    """sum of m log e - e over e != 0, in FP64 (Sinogram3D::getLikelihoodValue,
    data/src/Sinogram3D.cpp:584-606, with an FP64 accumulator)."""
    e = est.astype(np.float64)
    m = meas.astype(np.float64)
    nz = e != 0
    return float(np.sum(m[nz] * np.log(e[nz]) - e[nz]))


@pytest.fixture(scope="module")
def c2():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ap.load_library()
    ig, sg = workloads.c2_geometry()
    P = ap.SiddonProjector(ig, sg)
    atten, counts = workloads.c2_device_arrays(P, DEV)
    torch.cuda.synchronize()
    yield dict(P=P, ig=ig, sg=sg, atten=atten, counts=counts,
               counts_np=counts.view(torch.int32).cpu().numpy().view(np.uint32),
               atten_np=atten.cpu().numpy())
    P.close()


def _subset(a, sg, s):
    return np.ascontiguousarray(a.reshape(sg.n_sinos, sg.n_proj, sg.n_r)[:, s::NSUB, :]).reshape(-1)


def test_headline_pass_matches_oracle(oracle, c2):
    P, ig, sg = c2["P"], c2["ig"], c2["sg"]
    threads = os.cpu_count() or 1
    x = torch.ones(ig.n_voxels, dtype=torch.float32, device=DEV)
    for s in (0, 10, 20):
        a_s = _subset(c2["atten_np"], sg, s)
        m_s = _subset(c2["counts_np"], sg, s).astype(np.float32)
        x_in = x.cpu().numpy()
        # sensitivity and geometry image, as the bench makes them
        sens = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        P.backproject(torch.from_numpy(a_s).to(DEV), sens, s, NSUB)
        ap.force_positive(sens)
        gimg = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        P.backproject_ones(gimg, s, NSUB)
        est = torch.zeros(P.num_bins(s, NSUB), dtype=torch.float32, device=DEV)
        P.project(x, est, s, NSUB)
        # the full pass (every bin walked) and the listed geometry-image pass
        bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        x_full = x.clone()
        lik_full = torch.zeros(1, dtype=torch.float64, device=DEV)
        P.em_pass(c2["counts"], x_full, bp, sens, s, NSUB, ge=False, lik=lik_full)
        P.set_option(_lib.APIRL_OPT_SPARSE_IMAGE, _lib.APIRL_SPARSE_GEOMETRY)
        lik = torch.zeros(1, dtype=torch.float64, device=DEV)
        P.em_pass_sparse(c2["counts"], x, bp, sens, gimg, s, NSUB, ge=False, lik=lik)
        torch.cuda.synchronize()
        sens_np = sens.cpu().numpy()

        want_est = oracle.project_3d(sg, ig, x_in, s, NSUB, threads=threads)
        assert bits_equal(est.cpu().numpy(), want_est), f"subset {s}: projection differs"
        want_sens = np.maximum(oracle.backproject_3d(sg, ig, a_s, s, NSUB, threads=threads), 0)
        assert rel(sens_np, want_sens) <= 1e-5
        want_g = oracle.backproject_3d(sg, ig, np.ones_like(a_s), s, NSUB, threads=threads)
        assert rel(gimg.cpu().numpy(), want_g) <= 1e-5
        want_lik = fp64_likelihood(want_est, m_s)
        ratio = oracle.inverse_divide(m_s, want_est)
        bp_ref = oracle.backproject_3d(sg, ig, ratio, s, NSUB, threads=threads)
        want_x = oracle.update(x_in, bp_ref, sens_np, 0.0, False)
        assert np.all(np.isfinite(want_x))
        got_full, got = x_full.cpu().numpy(), x.cpu().numpy()
        assert rel(got_full, want_x) <= 1e-5, f"subset {s}: full pass {rel(got_full, want_x):.3e}"
        assert rel(got, want_x) <= 1e-5, f"subset {s}: listed pass {rel(got, want_x):.3e}"
        assert abs(lik_full.item() - want_lik) <= 1e-9 * abs(want_lik)
        assert abs(lik.item() - want_lik) <= 1e-6 * abs(want_lik)


def test_whole_job_matches_oracle(oracle, c2):
    ig, sg = c2["ig"], c2["sg"]
    meas = c2["counts_np"].astype(np.float32)
    init = np.ones(ig.n_voxels, np.float32)
    got, lik, sens = ap.osem_3d(ig, sg, meas, init, 3, NSUB, mult=c2["atten_np"], update_positive_sens=True)
    want, want_lik, want_sens0 = oracle.osem_3d(sg, ig, init, meas, 3, NSUB, mult=c2["atten_np"],
                                                threads=os.cpu_count() or 1, ge=False)
    assert np.all(np.isfinite(got)) and np.all(np.isfinite(want))
    assert rel(sens, want_sens0) <= 1e-5
    r = rel(got, want)
    assert r <= 1e-4, f"reconstruction rel L2 {r:.3e}"
    # the likelihoods are FP64 sums here and float sums of 6.8 million terms
    # in the oracle (the reference's accumulator), whose rounding reaches
    # ~1e-4: they are checked per pass against an FP64 sum above
    assert np.all(np.isfinite(lik))


def test_full_size_job_in_a_batch(c2):
    """The batch engine at full size: the job with its attenuation factors
    (the batch walks its own sensitivity A_s^T a) as the only job of a batch,
    1 iteration x 21 subsets, update where sens > 0, against the same job
    through apirl_osem_3d: image rel L2 <= 1e-4 (the order of the fp32 atomic
    adds), likelihoods to 1e-6."""
    from apirl_b200.batch import Batch, Job
    ig, sg = c2["ig"], c2["sg"]
    b = Batch(0, budget_bytes=32 << 30)
    (img, lik), = b.run_all([Job(ig, sg, c2["counts_np"], 1, NSUB, mult=c2["atten_np"], update_positive_sens=True)])
    b.close()
    solo, solo_lik, _ = ap.osem_3d(ig, sg, c2["counts_np"].astype(np.float32), np.ones(ig.n_voxels, np.float32), 1,
                                   NSUB, mult=c2["atten_np"], update_positive_sens=True)
    assert np.all(np.isfinite(img)) and np.all(np.isfinite(solo))
    assert rel(img, solo) <= 1e-4, f"batch vs driver rel L2 {rel(img, solo):.3e}"
    assert np.allclose(lik, solo_lik, rtol=1e-6, atol=0)


def test_precision_first_subiteration():
    """The precision study's bounds on the first sub-iteration of the full
    workload, against the FP64 oracle (bench.precision_study):
      reference float arithmetic ....... image rel L2 <= 2e-2, likelihood <= 1e-4
      FP64 walk geometry ............... image rel L2 <= 2e-6, likelihood <= 1e-6
      uint16 counts .................... bit-exact round trip, image equal to uint32's
                                         up to the atomics' order (rel L2 <= 1e-6)
      one ratio backprojection ......... against the FP64 sum of the float walk's own
                                         contributions: compensated atomics better
                                         than plain atomics, and <= 1e-7 relative L2
      adjoint residual of the operators  <= 1e-6"""
    import bench
    r = bench.precision_study(1, lambda m: None)
    row = r["subiterations"][0]
    assert r["u16_round_trip"] and row["u16_vs_f32_rel_l2"] <= 1e-6
    assert row["f32"]["rel_l2"] <= 2e-2 and row["f32"]["lik_rel"] <= 1e-4
    assert row["f64alpha"]["rel_l2"] <= 2e-6 and row["f64alpha"]["lik_rel"] <= 1e-6
    for form in ("f32_warp", "f32_comp"):
        assert row[form]["rel_l2"] <= 2e-2
        assert abs(row[form]["rel_l2"] - row["f32"]["rel_l2"]) <= 1e-5
    acc = r["backprojection_accumulation"]
    assert acc["gpu_compensated_rel_l2"] < acc["gpu_atomic_rel_l2"] and acc["gpu_compensated_rel_l2"] <= 1e-7
    assert all(v <= 1e-6 for v in r["adjoint_residual"].values())
