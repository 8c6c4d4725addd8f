"""Odd geometries on the GPU against the oracle: non-square images, a single
slice, one radial bin, more subsets than a few angles, rays along the axes
(angle 0 and 90 degrees), image larger and smaller than the sinogram field of
view, extreme ring differences, voxels of unequal size.  Projection
bit-exact, backprojection and one fused pass rel L2 <= 1e-5 (NaN-aware where
voxels have zero sensitivity)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import apirl_b200 as ap  # noqa: E402
from apirl_b200 import _lib  # noqa: E402
from apirl_b200.geometry import ImageGeom, Sino3DGeom  # noqa: E402

DEV = torch.device("cuda:0")


def t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    m = np.isfinite(a) & np.isfinite(b)
    assert np.array_equal(np.isfinite(a), np.isfinite(b))
    return float(np.linalg.norm(a[m] - b[m]) / max(np.linalg.norm(b[m]), 1e-300))


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a, np.float32).view(np.uint32),
                          np.ascontiguousarray(b, np.float32).view(np.uint32))


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ap.load_library()


CASES = {
    "non_square": (ImageGeom(40, 24, 6, 2.5, 3.1, 2.0), Sino3DGeom.span1(18, 40, 4, 60.0, 4 * 3.0, 150.0, 3)),
    "single_slice": (ImageGeom(32, 32, 1, 2.0, 2.0, 4.0), Sino3DGeom.span1(16, 32, 1, 40.0, 4.0, 150.0, 0)),
    "one_radial_bin": (ImageGeom(16, 16, 4, 2.0, 2.0, 2.0), Sino3DGeom.span1(8, 1, 3, 20.0, 6.0, 150.0, 2)),
    "image_beyond_fov": (ImageGeom(64, 64, 5, 3.0, 3.0, 2.0), Sino3DGeom.span1(20, 30, 5, 40.0, 10.0, 120.0, 4)),
    "small_image": (ImageGeom(8, 8, 3, 1.0, 1.0, 3.0), Sino3DGeom.span1(12, 40, 3, 50.0, 9.0, 150.0, 2)),
    "span3": (ImageGeom(24, 24, 9, 2.0, 2.0, 2.0), Sino3DGeom.span(10, 24, 9, 24.0, 18.0, 150.0, 3, 8)),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("dual", [1, 0])
def test_edge_geometry(oracle, name, dual):
    ig, sg = CASES[name]
    rng = np.random.default_rng(len(name))
    img = rng.random(ig.n_voxels, dtype=np.float32)
    P = ap.SiddonProjector(ig, sg)
    P.set_option(_lib.APIRL_OPT_DUAL_LAYOUT, dual)
    nsub = min(sg.n_proj, 7)
    for sub, ns in ((-1, 1), (nsub - 1, nsub)):
        want = oracle.project_3d(sg, ig, img, sub, ns)
        out = torch.zeros(P.num_bins(sub, ns), dtype=torch.float32, device=DEV)
        P.project(t(img), out, sub, ns)
        assert bits_equal(out.cpu().numpy(), want)
        v = rng.random(want.size, dtype=np.float32)
        bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        P.backproject(t(v), bp, sub, ns)
        assert rel(bp.cpu().numpy(), oracle.backproject_3d(sg, ig, v, sub, ns)) <= 1e-5
    # one fused pass (persistent and plain kernels)
    meas = rng.poisson(oracle.project_3d(sg, ig, img) * 3).astype(np.uint32)
    sens = (rng.random(ig.n_voxels, dtype=np.float32) + 1).astype(np.float32)
    s = nsub - 1
    m_sub = meas.reshape(sg.n_sinos, sg.n_proj, sg.n_r)[:, s::nsub, :].reshape(-1).astype(np.float32)
    est = oracle.project_3d(sg, ig, img, s, nsub)
    want_x = oracle.update(img, oracle.backproject_3d(sg, ig, oracle.inverse_divide(m_sub, est), s, nsub, threads=1),
                           sens, np.float32(0), True)
    for persistent in (1, 0):
        P.set_option(_lib.APIRL_OPT_PERSISTENT, persistent)
        x = t(img)
        bpd = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        P.em_pass(t(meas), x, bpd, t(sens), s, nsub)
        torch.cuda.synchronize()
        assert rel(x.cpu().numpy(), want_x) <= 1e-5


def test_invalid_geometries_rejected():
    ig = ImageGeom(16, 16, 4, 2.0, 2.0, 2.0)
    with pytest.raises(ap.ApirlError):
        ap.SiddonProjector(ig, Sino3DGeom.span1(8, 16, 3, 200.0, 6.0, 150.0, 2))  # rFov beyond the scanner
    with pytest.raises(ap.ApirlError):
        ap.SiddonProjector(ImageGeom(16, 16, 4, 0.0, 2.0, 2.0), Sino3DGeom.span1(8, 16, 3, 20.0, 6.0, 150.0, 2))
    P = ap.SiddonProjector(ig, Sino3DGeom.span1(8, 16, 3, 20.0, 6.0, 150.0, 2))
    out = torch.zeros(P.num_bins(0, 4), dtype=torch.float32, device=DEV)
    for sub, ns in ((4, 4), (0, 9), (-1, 0)):
        if sub >= 0:
            with pytest.raises(ap.ApirlError):
                P.project(t(np.ones(ig.n_voxels, np.float32)), out, sub, ns)
    P.set_shard(2, 4)  # 9 sinograms: a valid shard
    P.set_shard(0, 9)
    for first, n in ((5, 5), (-1, 2), (0, 0)):
        with pytest.raises(ap.ApirlError):
            P.set_shard(first, n)


@pytest.mark.parametrize("dtype", [np.uint32, np.uint16, np.float32])
def test_listed_pass_with_no_counts(oracle, dtype):
    """Empty input: a subset whose counts are all zero gives the listed pass
    (geometry image) an empty list of bins.  The update equals the oracle's
    (every ratio 0: x becomes 0 where the sensitivity passes) and the FP64
    likelihood is -x . G_s, the reference's sum of m log e - e over e != 0
    with m = 0 (against the FP64 sum of the oracle's float estimates, 1e-6).
    The next subset, with counts, on the same projector (its list grows back
    from empty) matches the oracle too."""
    ig, sg = CASES["non_square"]
    rng = np.random.default_rng(6)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    ns = 3
    m3 = rng.poisson(oracle.project_3d(sg, ig, x0) * 2).astype(dtype).reshape(sg.n_sinos, sg.n_proj, sg.n_r)
    m3[:, 0::ns, :] = 0  # subset 0 without counts
    meas = m3.reshape(-1)
    sens = (rng.random(ig.n_voxels, dtype=np.float32) + 1).astype(np.float32)
    P = ap.SiddonProjector(ig, sg)
    P.set_option(_lib.APIRL_OPT_SPARSE_IMAGE, _lib.APIRL_SPARSE_GEOMETRY)
    for s in (0, 1):
        gimg = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        P.backproject_ones(gimg, s, ns)
        x = t(x0)
        bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        lik = torch.zeros(1, dtype=torch.float64, device=DEV)
        P.em_pass_sparse(t(meas), x, bp, t(sens), gimg, s, ns, lik=lik)
        torch.cuda.synchronize()
        m_sub = m3[:, s::ns, :].reshape(-1).astype(np.float32)
        est = oracle.project_3d(sg, ig, x0, s, ns)
        want_x = oracle.update(x0, oracle.backproject_3d(sg, ig, oracle.inverse_divide(m_sub, est), s, ns,
                                                         threads=1), sens, np.float32(0), True)
        got = x.cpu().numpy()
        if s == 0:
            assert not m_sub.any()
            assert np.array_equal(got, want_x) and not got.any()
        else:
            assert rel(got, want_x) <= 1e-5
        e = est.astype(np.float64)
        nz = est != 0
        want_lik = float(np.sum(m_sub[nz].astype(np.float64) * np.log(e[nz]) - e[nz]))
        assert abs(lik.item() - want_lik) <= 1e-6 * abs(want_lik)
