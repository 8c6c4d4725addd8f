"""Parity of the CUDA path with the oracle (and, through the golden fixtures,
with the reference APIRL code).  Every call goes through the C ABI.

Tolerances
  forward projection ..... bit-exact (same float operations, same order)
  backprojection ......... rel L2 <= 1e-5 (fp32 atomics accumulate in another order)
  adjoint <Ax,y> vs <x,A^T y> ... rel <= 1e-6 (FP64 dot products of fp32 results)
  reconstructions ........ rel L2 <= 1e-4 after the stated iterations
  likelihood (FP64) ...... rel <= 1e-9 against the oracle's FP64 sum of the GPU estimates
"""
import hashlib
import json
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import apirl_b200 as ap  # noqa: E402
from apirl_b200 import workloads  # noqa: E402
from apirl_b200.geometry import ImageGeom, Sino2DGeom, Sino3DGeom  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "golden_small.npz"))
with open(os.path.join(HERE, "golden", "golden_c2.json")) as f:
    C2 = json.load(f)
DEV = torch.device("cuda:0")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def t(a, dtype=None):
    return torch.from_numpy(np.ascontiguousarray(a if dtype is None else a.astype(dtype))).to(DEV)


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a, np.float32).view(np.uint32),
                          np.ascontiguousarray(b, np.float32).view(np.uint32))


def small_3d():
    return ImageGeom(48, 48, 9, 2.08, 2.08, 2.03), Sino3DGeom.span1(25, 48, 5, 72.0, 5 * 4.054, 150.0, 3)


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ap.load_library()


# ---------------------------------------------------------------------------
def test_tables_equal_reference():
    ig, sg = workloads.c1_geometry()
    P = ap.SiddonProjector(ig, sg)
    lor, _ = P.tables()
    assert bits_equal(lor, G["lor_c1"])


def test_2d_project_bit_exact_vs_reference():
    ig, sg = workloads.c1_geometry()
    P = ap.SiddonProjector(ig, sg)
    out = torch.zeros(sg.n_bins, dtype=torch.float32, device=DEV)
    P.project(t(G["c1_phantom"]), out)
    torch.cuda.synchronize()
    assert bits_equal(out.cpu().numpy(), G["c1_project"])


def test_2d_backproject_vs_reference():
    ig, sg = workloads.c1_geometry()
    P = ap.SiddonProjector(ig, sg)
    img = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    P.backproject(torch.ones(sg.n_bins, dtype=torch.float32, device=DEV), img)
    assert rel(img.cpu().numpy(), G["c1_backproject_ones"]) <= 1e-5


def test_2d_divide_and_backproject(oracle):
    ig, sg = workloads.c1_geometry()
    rng = np.random.default_rng(3)
    m = rng.poisson(5, sg.n_bins).astype(np.float32)
    e = rng.random(sg.n_bins, dtype=np.float32)
    e[::5] = 0
    P = ap.SiddonProjector(ig, sg)
    img = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    P.divide_and_backproject(t(m), t(e), img)
    assert rel(img.cpu().numpy(), oracle.divide_and_backproject_2d(sg, ig, m, e)) <= 1e-5


@pytest.mark.parametrize("sub,ns", [(-1, 1), (0, 4), (3, 4), (2, 5)])
def test_3d_project_bit_exact_backproject_close_vs_reference(sub, ns):
    ig, sg = small_3d()
    P = ap.SiddonProjector(ig, sg)
    key = f"s3_project_{sub}_{ns}".replace("-", "m")
    out = torch.zeros(P.num_bins(sub, ns), dtype=torch.float32, device=DEV)
    P.project(t(G["s3_image"]), out, sub, ns)
    assert bits_equal(out.cpu().numpy(), G[key])
    img = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    P.backproject(t(G[key.replace("project", "bpvalues")]), img, sub, ns)
    assert rel(img.cpu().numpy(), G[key.replace("project", "backproject")]) <= 1e-5


def test_3d_divide_and_backproject(oracle):
    ig, sg = small_3d()
    rng = np.random.default_rng(5)
    nb = sg.subset_bins(1, 3)
    m = rng.poisson(3, nb).astype(np.float32)
    e = rng.random(nb, dtype=np.float32)
    e[::4] = 0
    P = ap.SiddonProjector(ig, sg)
    img = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    P.divide_and_backproject(t(m), t(e), img, 1, 3)
    assert rel(img.cpu().numpy(), oracle.divide_and_backproject_3d(sg, ig, m, e, 1, 3)) <= 1e-5


@pytest.mark.parametrize("which", ["2d", "3d"])
def test_adjoint_identity(which):
    if which == "2d":
        ig, sg = workloads.c1_geometry()
        sg = Sino2DGeom(sg.n_proj, sg.n_r, 130.0, sg.r_scanner)  # every ray valid and inside
    else:
        ig, sg = small_3d()
    P = ap.SiddonProjector(ig, sg)
    rng = np.random.default_rng(11)
    x = rng.random(ig.n_voxels, dtype=np.float32)
    y = rng.random(P.num_bins(), dtype=np.float32)
    ax = torch.zeros(P.num_bins(), dtype=torch.float32, device=DEV)
    P.project(t(x), ax)
    aty = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    P.backproject(t(y), aty)
    lhs = float(np.dot(ax.cpu().numpy().astype(np.float64), y.astype(np.float64)))
    rhs = float(np.dot(x.astype(np.float64), aty.cpu().numpy().astype(np.float64)))
    assert abs(lhs - rhs) / abs(rhs) <= 1e-6


# ---------------------------------------------------------------------------
def _oracle_osem_pass(oracle, sg, ig, x, meas_full, sens, subset, ns):
    meas_sub = meas_full.reshape(sg.n_sinos, sg.n_proj, sg.n_r)[:, subset::ns, :].reshape(-1) if subset >= 0 \
        else meas_full
    est = oracle.project_3d(sg, ig, x, subset, ns)
    est64 = est.astype(np.float64)
    nz = est != 0
    lik = float(np.sum(meas_sub[nz].astype(np.float64) * np.log(est64[nz]) - est64[nz]))
    ratio = oracle.inverse_divide(meas_sub, est)
    bp = oracle.backproject_3d(sg, ig, ratio, subset, ns, threads=1)
    return oracle.update(x, bp, sens, np.float32(0), True), lik, meas_sub


@pytest.mark.parametrize("dtype", ["float32", "uint32", "uint16"])
def test_em_pass_vs_oracle(oracle, dtype):
    ig, sg = small_3d()
    rng = np.random.default_rng(21)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    meas = rng.poisson(oracle.project_3d(sg, ig, x0) * 2).astype(np.float32)
    sens = (rng.random(ig.n_voxels, dtype=np.float32) + 1).astype(np.float32)
    subset, ns = 2, 5
    want_x, want_lik, meas_sub = _oracle_osem_pass(oracle, sg, ig, x0, meas, sens, subset, ns)
    P = ap.SiddonProjector(ig, sg)
    from apirl_b200 import _lib
    for packed, block in ((False, 128), (True, 128), (False, 64), (True, 256), (False, 96)):
        P.set_option(_lib.APIRL_OPT_EM_BLOCK, block)
        x = t(x0)
        bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        lik = torch.zeros(1, dtype=torch.float64, device=DEV)
        counts = t((meas_sub if packed else meas).astype(dtype))
        P.em_pass(counts, x, bp, t(sens), subset, ns, lik=lik, counts_packed=packed)
        torch.cuda.synchronize()
        assert rel(x.cpu().numpy(), want_x) <= 1e-5
        assert float(bp.abs().max()) == 0.0  # cleared for the next pass
        assert abs(lik.item() - want_lik) <= 1e-9 * abs(want_lik)


def test_em_pass_host_matches_device(oracle):
    ig, sg = small_3d()
    rng = np.random.default_rng(22)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    meas = rng.poisson(oracle.project_3d(sg, ig, x0) * 2).astype(np.uint32)
    sens = np.ones(ig.n_voxels, np.float32)
    subset, ns = 1, 4
    want_x, want_lik, meas_sub = _oracle_osem_pass(oracle, sg, ig, x0, meas.astype(np.float32), sens, subset, ns)
    P = ap.SiddonProjector(ig, sg)
    import ctypes
    from apirl_b200 import _lib
    x = t(x0)
    bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    stage = torch.zeros(meas_sub.size, dtype=torch.int32, device=DEV)
    h_counts = np.ascontiguousarray(meas_sub.astype(np.uint32))
    h_x = np.zeros(ig.n_voxels, np.float32)
    h_lik = np.zeros(1, np.float64)
    st = t(sens)
    _lib.check(P.lib.apirl_em_pass_host(P.h, h_counts.ctypes.data_as(ctypes.c_void_p), _lib.APIRL_U32,
                                        ctypes.c_void_p(stage.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                        ctypes.c_void_p(bp.data_ptr()), ctypes.c_void_p(st.data_ptr()), None, None,
                                        0.0, 1,
                                        subset, ns, h_x.ctypes.data_as(ctypes.c_void_p),
                                        h_lik.ctypes.data_as(ctypes.c_void_p), None))
    assert rel(h_x, want_x) <= 1e-5
    assert abs(h_lik[0] - want_lik) <= 1e-9 * abs(want_lik)


def test_update_threshold_and_force_positive(oracle):
    rng = np.random.default_rng(4)
    n = 1001
    sens = rng.random(n, dtype=np.float32)
    sens[::7] = 0
    sens[3] = -0.5
    x = rng.random(n, dtype=np.float32)
    bp = rng.random(n, dtype=np.float32)
    thr = ap.mlem_threshold(t(sens))
    assert thr.item() == oracle.mlem_threshold(sens)
    for ge in (True, False):
        xt, bpt = t(x), t(bp)
        ap.update_pixels(xt, bpt, t(sens), thr=thr, ge=ge, zero_bp=True)
        torch.cuda.synchronize()
        assert bits_equal(xt.cpu().numpy(), oracle.update(x, bp, sens, np.float32(thr.item()), ge))
        assert float(bpt.abs().max()) == 0.0
    s2 = t(sens)
    ap.force_positive(s2)
    assert s2.min().item() >= 0
    e = t(x)
    ap.inverse_divide(t(bp), e)
    assert bits_equal(e.cpu().numpy(), oracle.inverse_divide(bp, x))
    lik = ap.likelihood(t(x), t(bp))
    want = float(np.sum(bp.astype(np.float64) * np.log(x.astype(np.float64)) - x.astype(np.float64)))
    assert abs(lik.item() - want) <= 1e-12 * abs(want)


# ---------------------------------------------------------------------------
def test_osem_driver_vs_reference(oracle):
    ig, sg = small_3d()
    init = np.ones(ig.n_voxels, np.float32)
    img, lik, sens0 = ap.osem_3d(ig, sg, G["s3_meas"], init, 2, 4)
    assert rel(sens0, G["s3_osem_sens0"]) <= 1e-5
    assert rel(img, G["s3_osem"]) <= 1e-4
    # likelihood: reference accumulates in float, we in FP64
    assert np.allclose(lik[:-1], G["s3_osem_lik"][:-1].astype(np.float64), rtol=1e-5)


def test_fp64_alpha_osem_vs_fp64_oracle(oracle):
    """Precision study form: OSEM with the FP64-alpha walk against the FP64
    oracle's OSEM, <= 1e-4 relative L2 (the float walk of the reference differs
    from FP64 by percents on some edge voxels: its segment count comes from
    float floors, Siddon.cpp:177-182, 220)."""
    ig, sg = small_3d()
    nsub, iters = 4, 2
    P = ap.SiddonProjector(ig, sg)
    P.set_alpha_precision(True)
    meas = t(G["s3_meas"])
    sens = []
    for s in range(nsub):
        im = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        P.backproject(torch.ones(P.num_bins(s, nsub), dtype=torch.float32, device=DEV), im, s, nsub)
        ap.force_positive(im)
        sens.append(im)
    x = torch.ones(ig.n_voxels, dtype=torch.float32, device=DEV)
    bp = torch.zeros_like(x)
    for _ in range(iters):
        for s in range(nsub):
            P.em_pass(meas, x, bp, sens[s], s, nsub)
    o64, _, s64 = oracle.osem_3d(sg, ig, np.ones(ig.n_voxels), G["s3_meas"], iters, nsub, dtype=np.float64)
    assert rel(sens[0].cpu().numpy(), s64) <= 1e-6
    assert rel(x.cpu().numpy(), o64) <= 1e-4


def test_mlem2d_driver_60_iterations_vs_reference():
    ig, sg = workloads.c1_geometry()
    init = np.ones(ig.n_voxels, np.float32)
    img, lik, sens = ap.mlem_2d(ig, sg, G["c1_meas"], init, 60)
    assert rel(sens, G["c1_sens"]) <= 1e-5
    assert rel(img, G["c1_mlem60"]) <= 1e-4
    assert np.allclose(lik, G["c1_mlem60_lik"].astype(np.float64), rtol=1e-4)


def test_mlem3d_driver_vs_oracle(oracle):
    ig, sg = small_3d()
    init = np.ones(ig.n_voxels, np.float32)
    img, lik, sens = ap.mlem_3d(ig, sg, G["s3_meas"], init, 3)
    # oracle MLEM 3D = OSEM with one subset and the MLEM threshold
    x = init.copy()
    sens_o = oracle.backproject_3d(sg, ig, np.ones(sg.n_bins, np.float32), threads=1)
    assert rel(sens, sens_o) <= 1e-5
    thr = oracle.mlem_threshold(sens_o)
    for _ in range(3):
        est = oracle.project_3d(sg, ig, x)
        bp = oracle.backproject_3d(sg, ig, oracle.inverse_divide(G["s3_meas"], est), threads=1)
        x = oracle.update(x, bp, sens_o, thr, True)
    assert rel(img, x) <= 1e-4


# ---------------------------------------------------------------------------
@pytest.mark.slow
def test_c2_full_size_projection_bytes_equal_reference():
    """Subset 0 of 21 at full size: the GPU projection of the cylinder phantom
    has exactly the reference's bytes (SHA-256 recorded from the reference)."""
    ig, sg = workloads.c2_geometry()
    P = ap.SiddonProjector(ig, sg)
    ph = t(workloads.cylinder_phantom_3d(ig, seed=2))
    out = torch.empty(P.num_bins(0, 21), dtype=torch.float32, device=DEV)
    P.project(ph, out, 0, 21)
    assert sha(out.cpu().numpy()) == C2["project_phantom_subset0_of21_sha256"]
    P.project(torch.ones(ig.n_voxels, dtype=torch.float32, device=DEV), out, 0, 21)
    assert sha(out.cpu().numpy()) == C2["project_ones_subset0_of21_sha256"]
    steps = P.count_steps(0, 21)
    assert int(steps.sum().item()) == 2144070812  # Siddon segments of subset 0


@pytest.mark.slow
def test_c2_full_size_backprojection_vs_oracle(oracle):
    ig, sg = workloads.c2_geometry()
    P = ap.SiddonProjector(ig, sg)
    rng = np.random.default_rng(9)
    v = rng.random(P.num_bins(5, 21), dtype=np.float32)
    v[rng.random(v.size) < 0.3] = 0
    img = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    P.backproject(t(v), img, 5, 21)
    assert rel(img.cpu().numpy(), oracle.backproject_3d(sg, ig, v, 5, 21)) <= 1e-5


@pytest.mark.slow
def test_c2_em_pass_properties():
    """Full-size fused pass: the image update is invariant to the counts' storage
    type, and a pass with measured = A x leaves x unchanged where sens = A^T 1."""
    ig, sg = workloads.c2_geometry()
    P = ap.SiddonProjector(ig, sg)
    x0 = t(workloads.cylinder_phantom_3d(ig, seed=2) + 0.5)
    ns, s = 21, 4
    est = torch.empty(P.num_bins(s, ns), dtype=torch.float32, device=DEV)
    P.project(x0, est, s, ns)
    sens = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    P.backproject(torch.ones_like(est), sens, s, ns)
    x = x0.clone()
    bp = torch.zeros_like(x)
    P.em_pass(est, x, bp, sens, s, ns, counts_packed=True)
    hit = sens > 0
    # m == A x makes every ratio 1, so bp == sens and x is unchanged up to rounding
    assert float(((x - x0).abs()[hit] / x0[hit]).max()) <= 1e-4
    c = torch.poisson(est * 2.0, generator=torch.Generator(device=DEV).manual_seed(0))
    xs = []
    for cc in (c, c.to(torch.int32).view(torch.uint32), c.to(torch.int32).to(torch.int16).view(torch.uint16)):
        xi = x0.clone()
        bp.zero_()
        P.em_pass(cc, xi, bp, sens, s, ns, counts_packed=True)
        xs.append(xi.cpu().numpy())
    assert rel(xs[0], xs[1]) <= 1e-5 and rel(xs[0], xs[2]) <= 1e-5


# ---------------------------------------------------------------------------
def test_fp64_alpha_mode_against_fp64_oracle(oracle):
    """Precision study: with FP64 alphas the projection error against the FP64
    oracle is at the fp32-accumulation level; the reference's float walk is
    checked to be no better."""
    ig, sg = small_3d()
    x = G["s3_image"]
    want = oracle.project_3d(sg, ig, x.astype(np.float64), 3, 4, dtype=np.float64)
    P = ap.SiddonProjector(ig, sg)
    out = torch.zeros(P.num_bins(3, 4), dtype=torch.float32, device=DEV)
    P.project(t(x), out, 3, 4)
    err32 = rel(out.cpu().numpy(), want)
    P.set_alpha_precision(True)
    P.project(t(x), out, 3, 4)
    err64 = rel(out.cpu().numpy(), want)
    assert err64 <= 1e-6
    assert err64 <= err32
    v = np.ones(out.numel(), np.float32)
    img = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    P.backproject(t(v), img, 3, 4)
    want_bp = oracle.backproject_3d(sg, ig, v.astype(np.float64), 3, 4, dtype=np.float64)
    assert rel(img.cpu().numpy(), want_bp) <= 1e-6
    P.set_alpha_precision(False)
    P.project(t(x), out, 3, 4)
    assert bits_equal(out.cpu().numpy(), G["s3_project_3_4"])


def test_generate_acf_and_multiplicative_additive_osem(oracle):
    """generateACFs on the GPU, then OSEM with the multiplicative (1/ACF) and an
    additive sinogram against the oracle's OSEM with the same terms."""
    ig, sg = small_3d()
    mu = np.full(ig.n_voxels, 0.0096, np.float32)
    P = ap.SiddonProjector(ig, sg)
    acf = torch.zeros(sg.n_bins, dtype=torch.float32, device=DEV)
    P.generate_acf(t(mu), acf)
    line = oracle.project_3d(sg, ig, mu)
    want = np.where(line != 0, np.exp(line.astype(np.float64)), 1.0)
    got = acf.cpu().numpy()
    assert np.max(np.abs(got - want) / want) <= 1e-6
    mult = (1.0 / got).astype(np.float32)
    add = np.full(sg.n_bins, 0.05, np.float32)
    init = np.ones(ig.n_voxels, np.float32)
    img, lik, sens0 = ap.osem_3d(ig, sg, G["s3_meas"], init, 2, 4, mult=mult, add=add)
    o, olik, osens0 = oracle.osem_3d(sg, ig, init, G["s3_meas"], 2, 4, mult=mult, add=add)
    assert rel(sens0, osens0) <= 1e-5
    assert rel(img, o) <= 1e-4
    assert np.allclose(lik, olik.astype(np.float64), rtol=1e-4)


def test_multiplicative_only_drivers_take_geometry_pass(oracle):
    """With a multiplicative sinogram and no additive one, the drivers walk
    the sensitivity A_s^T a and the geometry image A_s^T 1 together and then
    run the geometry sparse pass: same sensitivities and reconstruction as the
    oracle, and the same likelihood (1e-7 relative) as the full pass that
    given sensitivities take."""
    ig, sg = small_3d()
    rng = np.random.default_rng(47)
    mult = (rng.random(sg.n_bins, dtype=np.float32) * 0.7 + 0.3).astype(np.float32)
    init = np.ones(ig.n_voxels, np.float32)
    meas = G["s3_meas"]
    assert (meas == 0).any() and (meas != 0).any()
    img, lik, sens = ap.osem_3d(ig, sg, meas, init, 2, 4, mult=mult, all_sens=True)
    o, olik, osens0 = oracle.osem_3d(sg, ig, init, meas, 2, 4, mult=mult)
    assert rel(sens[0], osens0) <= 1e-5
    assert rel(img, o) <= 1e-4
    assert np.allclose(lik, olik.astype(np.float64), rtol=1e-4)
    img2, lik2, _ = ap.osem_3d(ig, sg, meas, init, 2, 4, mult=mult, sens=sens)
    assert rel(img, img2) <= 1e-5
    assert np.allclose(lik, lik2, rtol=1e-7)
    m, mlik, msens = ap.mlem_3d(ig, sg, meas, init, 3, mult=mult)
    m2, mlik2, _ = ap.mlem_3d(ig, sg, meas, init, 3, mult=mult, sens=msens)
    assert rel(m, m2) <= 1e-5
    assert np.allclose(mlik, mlik2, rtol=1e-7)


def test_sparse_likelihood_with_voxels_outside_every_ray(oracle):
    """End slices of an image longer than the scanner's axial FOV have zero
    sensitivity in every subset; the reference's >= 0 update turns them into
    0/0 = NaN, which no ray reaches.  The sparse passes' image dot products
    skip voxels of zero weight, so their likelihoods stay finite and equal the
    full pass's and the oracle's."""
    ig, sg = ImageGeom(48, 48, 13, 2.08, 2.08, 2.03), Sino3DGeom.span1(25, 48, 5, 72.0, 5 * 4.054, 150.0, 3)
    rng = np.random.default_rng(53)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    meas = rng.poisson(oracle.project_3d(sg, ig, x0) * 0.5).astype(np.float32)
    assert (meas == 0).any()
    init = np.ones(ig.n_voxels, np.float32)
    mult = (rng.random(sg.n_bins, dtype=np.float32) * 0.7 + 0.3).astype(np.float32)
    for m in (None, mult):
        img, lik, sens = ap.osem_3d(ig, sg, meas, init, 2, 4, mult=m, all_sens=True)
        assert (sens[0] == 0).any() and np.isnan(img).any()
        img2, lik2, _ = ap.osem_3d(ig, sg, meas, init, 2, 4, mult=m, sens=sens)
        o, olik, _ = oracle.osem_3d(sg, ig, init, meas, 2, 4, mult=m)
        assert np.all(np.isfinite(lik)) and np.allclose(lik, lik2, rtol=1e-7)
        assert np.allclose(lik, olik.astype(np.float64), rtol=1e-4)
        assert np.array_equal(np.isnan(img), np.isnan(o))
        ok = ~np.isnan(o)
        assert rel(img[ok], o[ok]) <= 1e-4


def test_dual_layout_pass_equals_single_layout(oracle):
    """The transposed-copy walk (default) changes only the order of fp32
    additions in the backprojection; projections and the likelihood are
    bit-identical."""
    from apirl_b200 import _lib
    ig, sg = ImageGeom(40, 36, 7, 2.08, 2.08, 2.03), Sino3DGeom.span1(30, 44, 4, 60.0, 4 * 4.06, 150.0, 2)
    rng = np.random.default_rng(31)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    meas = rng.poisson(oracle.project_3d(sg, ig, x0) * 2).astype(np.float32)
    sens = (rng.random(ig.n_voxels, dtype=np.float32) + 1).astype(np.float32)
    outs = []
    for dual in (0, 1):
        P = ap.SiddonProjector(ig, sg)
        P.set_option(_lib.APIRL_OPT_DUAL_LAYOUT, dual)
        x = t(x0)
        bp = torch.zeros_like(x)
        lik = torch.zeros(1, dtype=torch.float64, device=DEV)
        P.em_pass(t(meas), x, bp, t(sens), 1, 3, lik=lik)
        bp2 = torch.zeros_like(x)
        P.em_project_backproject(t(meas), t(x0), bp2, 2, 3)
        torch.cuda.synchronize()
        assert float(bp.abs().max()) == 0.0
        outs.append((x.cpu().numpy(), lik.item(), bp2.cpu().numpy()))
    assert rel(outs[1][0], outs[0][0]) <= 1e-6
    assert outs[1][1] == outs[0][1]
    assert rel(outs[1][2], outs[0][2]) <= 1e-6


@pytest.mark.parametrize("dual", [1, 0])
def test_sparse_pass_equals_full_pass(oracle, dual):
    """apirl_em_pass_sparse (zero-count bins not walked, their likelihood terms
    from the zero-count image) against apirl_em_pass and the oracle."""
    from apirl_b200 import _lib
    ig, sg = small_3d()
    rng = np.random.default_rng(77)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    meas = rng.poisson(oracle.project_3d(sg, ig, x0) * 0.3).astype(np.float32)
    meas[rng.random(meas.size) < 0.3] = 0  # plenty of zero-count bins
    add = (rng.random(meas.size, dtype=np.float32) * 0.1).astype(np.float32)
    sens = (rng.random(ig.n_voxels, dtype=np.float32) + 1).astype(np.float32)
    subset, ns = 3, 5
    P = ap.SiddonProjector(ig, sg)
    P.set_option(_lib.APIRL_OPT_DUAL_LAYOUT, dual)
    for use_add in (False, True):
        a = t(add) if use_add else None
        for dtype, packed in ((np.float32, False), (np.uint32, False), (np.uint16, True)):
            counts_np = meas.reshape(sg.n_sinos, sg.n_proj, sg.n_r)[:, subset::ns, :].reshape(-1) if packed else meas
            counts = t(counts_np.astype(dtype))
            ad = a
            if use_add and packed:
                ad = t(add.reshape(sg.n_sinos, sg.n_proj, sg.n_r)[:, subset::ns, :].reshape(-1))
            zimg = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
            zadd = torch.zeros(1, dtype=torch.float64, device=DEV)
            P.zero_count_image(counts, zimg, subset, ns, add=ad, counts_packed=packed, zero_add=zadd)
            x_full, x_sp = t(x0), t(x0)
            bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
            lik_full = torch.zeros(1, dtype=torch.float64, device=DEV)
            lik_sp = torch.zeros(1, dtype=torch.float64, device=DEV)
            P.em_pass(counts, x_full, bp, t(sens), subset, ns, add=ad, lik=lik_full, counts_packed=packed)
            P.em_pass_sparse(counts, x_sp, bp, t(sens), zimg, subset, ns, add=ad, zero_add=zadd, lik=lik_sp,
                             counts_packed=packed)
            torch.cuda.synchronize()
            assert rel(x_sp.cpu().numpy(), x_full.cpu().numpy()) <= 1e-6
            assert float(bp.abs().max()) == 0.0
            assert abs(lik_sp.item() - lik_full.item()) <= 1e-6 * abs(lik_full.item())
    # the oracle's zero-count image: backprojection of the zero indicator
    sub = meas.reshape(sg.n_sinos, sg.n_proj, sg.n_r)[:, subset::ns, :].reshape(-1)
    want = oracle.backproject_3d(sg, ig, (sub == 0).astype(np.float32), subset, ns)
    zimg = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    P.zero_count_image(t(meas), zimg, subset, ns)
    assert rel(zimg.cpu().numpy(), want) <= 1e-5


def test_osem_driver_sparse_long_job_vs_oracle(oracle):
    """Four iterations: the driver runs the sparse pass (zero-count images)."""
    ig, sg = small_3d()
    rng = np.random.default_rng(41)
    truth = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    meas = rng.poisson(oracle.project_3d(sg, ig, truth) * 0.5).astype(np.float32)
    init = np.ones(ig.n_voxels, np.float32)
    img, lik, _ = ap.osem_3d(ig, sg, meas, init, 4, 4)
    want, want_lik, _ = oracle.osem_3d(sg, ig, init, meas, 4, 4)
    assert rel(img, want) <= 1e-4
    assert np.allclose(lik[:-1], want_lik[:-1].astype(np.float64), rtol=1e-5)


def test_persistent_pass_equals_plain_pass(oracle):
    """APIRL_OPT_PERSISTENT: same bins per warp-chunk, same likelihood partials."""
    from apirl_b200 import _lib
    ig, sg = small_3d()
    rng = np.random.default_rng(23)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    meas = rng.poisson(oracle.project_3d(sg, ig, x0) * 2).astype(np.uint32)
    sens = (rng.random(ig.n_voxels, dtype=np.float32) + 1).astype(np.float32)
    P = ap.SiddonProjector(ig, sg)
    out = {}
    for persistent in (0, 1):
        P.set_option(_lib.APIRL_OPT_PERSISTENT, persistent)
        for block in (64, 128, 256):
            P.set_option(_lib.APIRL_OPT_EM_BLOCK, block)
            x = t(x0)
            bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
            lik = torch.zeros(1, dtype=torch.float64, device=DEV)
            P.em_pass(t(meas), x, bp, t(sens), 3, 5, lik=lik)
            torch.cuda.synchronize()
            out[(persistent, block)] = (x.cpu().numpy(), lik.item())
    ref_x, ref_lik = out[(0, 128)]
    for k, (x, lik) in out.items():
        assert rel(x, ref_x) <= 1e-6
        assert lik == ref_lik  # per-chunk partials summed in the same order


def test_staged_counts_host_pass(oracle):
    """apirl_stage_counts + apirl_em_pass_host, and the same passes queued
    back to back with apirl_em_pass_host_async (likelihoods into page-locked
    slots, read after one synchronisation), equal the unstaged host pass."""
    ig, sg = small_3d()
    rng = np.random.default_rng(24)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    meas = rng.poisson(oracle.project_3d(sg, ig, x0) * 2).astype(np.uint32).reshape(sg.n_sinos, sg.n_proj, sg.n_r)
    ns = 4
    host = [np.ascontiguousarray(meas[:, s::ns, :].reshape(-1)) for s in range(ns)]
    sens = t(np.ones(ig.n_voxels, np.float32))
    P = ap.SiddonProjector(ig, sg)
    stages = [torch.zeros(host[0].size, dtype=torch.int32, device=DEV) for _ in range(2)]
    res = []
    for staged, wait in ((False, True), (True, True), (True, False)):
        x = t(x0)
        bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        slots = torch.full((ns,), float("nan"), dtype=torch.float64).pin_memory().numpy()
        if staged:
            P.stage_counts(host[0], stages[0], 0, ns)
        for s in range(ns):
            if staged and s + 1 < ns:
                P.stage_counts(host[s + 1], stages[(s + 1) % 2], s + 1, ns)
            P.em_pass_host(host[s], stages[s % 2], x, bp, sens, s, ns, None, slots[s:s + 1], wait=wait)
        torch.cuda.synchronize()
        res.append((x.cpu().numpy(), slots.copy()))
    for x, liks in res[1:]:
        assert rel(x, res[0][0]) <= 1e-6
        assert liks[0] == res[0][1][0]  # later passes see images that differ in fp32 atomic order
        assert np.allclose(liks, res[0][1], rtol=1e-7)


def test_drivers_with_given_sensitivity(oracle):
    """apirl_osem_3d_ex / apirl_mlem_3d_ex / apirl_mlem_2d_ex: every subset's
    sensitivity comes back, and given back in place of the computed ones they
    give the same reconstruction (the atomics' order aside); a given image
    that differs changes it."""
    ig, sg = small_3d()
    rng = np.random.default_rng(31)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    meas = rng.poisson(oracle.project_3d(sg, ig, x0) * 2).astype(np.float32)
    init = np.ones(ig.n_voxels, np.float32)
    img, lik, sens_all = ap.osem_3d(ig, sg, meas, init, 2, 4, all_sens=True)
    assert sens_all.shape == (4, ig.n_voxels)
    _, _, sens0 = ap.osem_3d(ig, sg, meas, init, 0, 4)
    assert rel(sens_all[0], sens0) <= 1e-6  # fp32 atomics: equal up to the order of additions
    img2, lik2, back = ap.osem_3d(ig, sg, meas, init, 2, 4, sens=sens_all, all_sens=True)
    assert np.array_equal(back.view(np.uint32), sens_all.view(np.uint32))
    # computed sensitivities without factors let the driver take the
    # geometry-image pass, whose likelihood sums in another order
    assert rel(img2, img) <= 1e-6 and abs(lik2[0] - lik[0]) <= 1e-7 * abs(lik[0])
    img3, _, _ = ap.osem_3d(ig, sg, meas, init, 2, 4, sens=sens_all * np.float32(2))
    assert rel(img3, img) > 1e-3
    m_img, m_lik, m_sens = ap.mlem_3d(ig, sg, meas, init, 2)
    m_img2, m_lik2, _ = ap.mlem_3d(ig, sg, meas, init, 2, sens=m_sens)
    assert rel(m_img2, m_img) <= 1e-6 and abs(m_lik2[0] - m_lik[0]) <= 1e-7 * abs(m_lik[0])
    ig2 = ImageGeom(32, 32, 1, 2.08, 2.08, 1.0)
    sg2 = Sino2DGeom(40, 48, 49.92, 300.0)
    x2 = (rng.random(ig2.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    P2 = ap.SiddonProjector(ig2, sg2)
    est = torch.zeros(sg2.n_bins, dtype=torch.float32, device=DEV)
    P2.project(t(x2), est)
    meas2 = rng.poisson(est.cpu().numpy()).astype(np.float32)
    a, _, s2 = ap.mlem_2d(ig2, sg2, meas2, np.ones(ig2.n_voxels, np.float32), 3)
    b, _, _ = ap.mlem_2d(ig2, sg2, meas2, np.ones(ig2.n_voxels, np.float32), 3, sens=s2)
    assert rel(b, a) <= 1e-6


@pytest.mark.parametrize("dual,persistent", [(1, 1), (1, 0), (0, 0)])
def test_nonzero_pass_with_geometry_image(oracle, dual, persistent):
    """APIRL_OPT_SPARSE_IMAGE = APIRL_SPARSE_GEOMETRY: the sparse pass given
    G_s = A_s^T 1 (apirl_backproject_ones) and the sum of every bin's additive
    term equals the full pass: the image up to the atomics' order, the
    likelihood to 1e-6 relative (sum of m log e over bins with counts minus
    x . G_s minus that sum)."""
    from apirl_b200 import _lib
    ig, sg = small_3d()
    rng = np.random.default_rng(78)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    meas = rng.poisson(oracle.project_3d(sg, ig, x0) * 0.3).astype(np.float32)
    meas[rng.random(meas.size) < 0.3] = 0
    add = (rng.random(meas.size, dtype=np.float32) * 0.1).astype(np.float32)
    sens = (rng.random(ig.n_voxels, dtype=np.float32) + 1).astype(np.float32)
    subset, ns = 2, 5
    P = ap.SiddonProjector(ig, sg)
    P.set_option(_lib.APIRL_OPT_DUAL_LAYOUT, dual)
    P.set_option(_lib.APIRL_OPT_PERSISTENT, persistent)
    gimg = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    P.backproject_ones(gimg, subset, ns)
    ones = np.ones(sg.subset_bins(subset, ns), np.float32)
    assert rel(gimg.cpu().numpy(), oracle.backproject_3d(sg, ig, ones, subset, ns)) <= 1e-5
    v = np.random.default_rng(79).random(ones.size, dtype=np.float32)
    vimg = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    g2 = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    P.backproject_and_ones(t(v), vimg, g2, subset, ns)
    assert rel(vimg.cpu().numpy(), oracle.backproject_3d(sg, ig, v, subset, ns)) <= 1e-5
    assert rel(g2.cpu().numpy(), gimg.cpu().numpy()) <= 1e-6
    add_sub = add.reshape(sg.n_sinos, sg.n_proj, sg.n_r)[:, subset::ns, :].reshape(-1)
    for use_add in (False, True):
        a = t(add) if use_add else None
        add_sum = torch.tensor([float(add_sub.astype(np.float64).sum()) if use_add else 0.0],
                               dtype=torch.float64, device=DEV)
        x_full, x_nz = t(x0), t(x0)
        bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        lik_full = torch.zeros(1, dtype=torch.float64, device=DEV)
        lik_nz = torch.zeros(1, dtype=torch.float64, device=DEV)
        P.set_option(_lib.APIRL_OPT_SPARSE_IMAGE, _lib.APIRL_SPARSE_ZERO_COUNT)
        P.em_pass(t(meas), x_full, bp, t(sens), subset, ns, add=a, lik=lik_full)
        P.set_option(_lib.APIRL_OPT_SPARSE_IMAGE, _lib.APIRL_SPARSE_GEOMETRY)
        P.em_pass_sparse(t(meas), x_nz, bp, t(sens), gimg, subset, ns, add=a, zero_add=add_sum, lik=lik_nz)
        torch.cuda.synchronize()
        assert rel(x_nz.cpu().numpy(), x_full.cpu().numpy()) <= 1e-6
        assert abs(lik_nz.item() - lik_full.item()) <= 1e-6 * abs(lik_full.item())
    with pytest.raises(ap.ApirlError):
        P.set_option(_lib.APIRL_OPT_SPARSE_IMAGE, 7)



@pytest.mark.parametrize("kind", ["span3", "mmr"])
def test_geometry_pass_other_sinograms(oracle, kind):
    """The listed geometry-image pass on a span-3 sinogram (several ring pairs
    per sinogram) and on the Siemens mMR geometry, against the full pass:
    image rel L2 <= 1e-6, likelihood 1e-6 relative; twice in a row (the bin
    list is rebuilt every pass)."""
    from apirl_b200 import _lib
    if kind == "span3":
        ig, sg = ImageGeom(48, 48, 9, 2.08, 2.08, 2.03), Sino3DGeom.span(25, 48, 5, 72.0, 5 * 4.054, 150.0, 3, 4)
    else:
        ig, sg = ImageGeom(72, 72, 16, 8.35, 8.35, 16.25), Sino3DGeom.mmr(36, 86, 8, 3, 4)
    P = ap.SiddonProjector(ig, sg)
    rng = np.random.default_rng(91)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    est = torch.zeros(P.num_bins(), dtype=torch.float32, device=DEV)
    P.project(t(x0), est)
    meas = rng.poisson(est.cpu().numpy() * 0.2).astype(np.uint32)
    sens = (rng.random(ig.n_voxels, dtype=np.float32) + 1).astype(np.float32)
    subset, ns = 1, 4
    gimg = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    P.backproject_ones(gimg, subset, ns)
    x_full, x_nz = t(x0), t(x0)
    for _ in range(2):
        bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        lik_full = torch.zeros(1, dtype=torch.float64, device=DEV)
        lik_nz = torch.zeros(1, dtype=torch.float64, device=DEV)
        P.set_option(_lib.APIRL_OPT_SPARSE_IMAGE, _lib.APIRL_SPARSE_ZERO_COUNT)
        P.em_pass(t(meas), x_full, bp, t(sens), subset, ns, lik=lik_full)
        P.set_option(_lib.APIRL_OPT_SPARSE_IMAGE, _lib.APIRL_SPARSE_GEOMETRY)
        P.em_pass_sparse(t(meas), x_nz, bp, t(sens), gimg, subset, ns, lik=lik_nz)
        torch.cuda.synchronize()
        assert rel(x_nz.cpu().numpy(), x_full.cpu().numpy()) <= 1e-6
        assert abs(lik_nz.item() - lik_full.item()) <= 1e-6 * abs(lik_full.item())
