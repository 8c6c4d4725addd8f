"""The Siemens mMR geometry on the GPU (apirl_projector_create_3d_mmr)
against the oracle's table-driven projector, fed with the tables the library
builds (tests/test_mmr_geometry.py pins those to the reference's
Sinogram2DinSiemensMmr bit for bit).  Projection bit-exact, backprojection
and one fused OSEM pass rel L2 <= 1e-5."""
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
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a, np.float32).view(np.uint32),
                          np.ascontiguousarray(b, np.float32).view(np.uint32))


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ap.load_library()


def case():
    sg = Sino3DGeom.mmr(36, 86, 8, 3, 4)
    ig = ImageGeom(72, 72, 16, 8.35, 8.35, 16.25)
    return ig, sg


def test_mmr_projection_and_backprojection(oracle):
    ig, sg = case()
    P = ap.SiddonProjector(ig, sg)
    lor, z = P.tables()
    rng = np.random.default_rng(5)
    img = rng.random(ig.n_voxels, dtype=np.float32)
    for sub, ns in ((-1, 1), (2, 4)):
        out = torch.zeros(P.num_bins(sub, ns), dtype=torch.float32, device=DEV)
        P.project(t(img), out, sub, ns)
        want = oracle.project_3d_tables(lor, z, ig, img, sub, ns)
        assert bits_equal(out.cpu().numpy(), want)
        v = rng.random(want.size, dtype=np.float32)
        bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        P.backproject(t(v), bp, sub, ns)
        assert rel(bp.cpu().numpy(), oracle.backproject_3d_tables(lor, z, ig, v, sub, ns)) <= 1e-5


def test_mmr_em_pass(oracle):
    ig, sg = case()
    P = ap.SiddonProjector(ig, sg)
    lor, z = P.tables()
    rng = np.random.default_rng(6)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    meas = rng.poisson(oracle.project_3d_tables(lor, z, ig, x0) * 0.5).astype(np.uint32)
    sens = (rng.random(ig.n_voxels, dtype=np.float32) + 1).astype(np.float32)
    subset, ns = 1, 4
    m_sub = meas.reshape(sg.n_sinos, sg.n_proj, sg.n_r)[:, subset::ns, :].reshape(-1).astype(np.float32)
    est = oracle.project_3d_tables(lor, z, ig, x0, subset, ns)
    ratio = oracle.inverse_divide(m_sub, est)
    bp = oracle.backproject_3d_tables(lor, z, ig, ratio, subset, ns)
    want = oracle.update(x0, bp, sens, np.float32(0), True)
    for dual in (1, 0):
        P.set_option(_lib.APIRL_OPT_DUAL_LAYOUT, dual)
        x = t(x0)
        bpd = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        P.em_pass(t(meas), x, bpd, t(sens), subset, ns)
        torch.cuda.synchronize()
        assert rel(x.cpu().numpy(), want) <= 1e-5
    with pytest.raises(ap.ApirlError):
        P.set_alpha_precision(True)
    with pytest.raises(ap.ApirlError):
        P.set_sampling(2, 1, False)
