"""Accumulation forms of the backprojection scatter (APIRL_OPT_ACCUMULATE):
plain fp32 atomics, warp-aggregated atomics, and compensated atomics (each
add's rounding error kept in a second padded pair).

Tolerances
  backprojection, fused pass (any form) vs the oracle ..... rel L2 <= 1e-5
  compensated backprojection vs the FP64 sum of the same float contributions
  (float walk, float segment * value, summed in double):
    no worse than plain atomics, and <= 1e-7 relative L2
  forms that a projector's path cannot take are refused (APIRL_ERR_NOT_SUPPORTED)
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import apirl_b200 as ap  # noqa: E402
from apirl_b200 import _lib  # noqa: E402
from apirl_b200.geometry import ImageGeom, Sino3DGeom  # noqa: E402

DEV = torch.device("cuda:0")
FORMS = [_lib.APIRL_ACC_ATOMIC, _lib.APIRL_ACC_WARP, _lib.APIRL_ACC_COMPENSATED]


def t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def geometry():
    return ImageGeom(64, 64, 13, 2.08, 2.08, 2.03), Sino3DGeom.span1(40, 72, 7, 72.0, 7 * 4.054, 200.0, 6)


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ap.load_library()


@pytest.mark.parametrize("form", FORMS)
def test_backprojection_forms(oracle, form):
    ig, sg = geometry()
    sub, ns = 2, 5
    rng = np.random.default_rng(3 + form)
    v = rng.random(sg.subset_bins(sub, ns), dtype=np.float32)
    P = ap.SiddonProjector(ig, sg)
    P.set_option(_lib.APIRL_OPT_ACCUMULATE, form)
    img = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    P.backproject(t(v), img, sub, ns)
    ones = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    P.backproject_ones(ones, sub, ns)
    torch.cuda.synchronize()
    got = img.cpu().numpy()
    assert rel(got, oracle.backproject_3d(sg, ig, v, sub, ns)) <= 1e-5
    assert rel(ones.cpu().numpy(), oracle.backproject_3d(sg, ig, np.ones_like(v), sub, ns)) <= 1e-5
    exact = oracle.backproject_3d_exact_sum(sg, ig, v, sub, ns)
    err = rel(got, exact)
    if form == _lib.APIRL_ACC_COMPENSATED:
        Pa = ap.SiddonProjector(ig, sg)
        plain = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        Pa.backproject(t(v), plain, sub, ns)
        torch.cuda.synchronize()
        assert err <= rel(plain.cpu().numpy(), exact) and err <= 1e-7


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("listed", [False, True])
def test_fused_pass_forms(oracle, form, listed):
    """One OSEM sub-iteration through the fused pass (every bin, or the listed
    geometry-image form) in each accumulation form, against the oracle."""
    ig, sg = geometry()
    sub, ns = 1, 4
    rng = np.random.default_rng(11)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    meas = rng.poisson(oracle.project_3d(sg, ig, x0) * 0.5).astype(np.uint32)
    sens = (rng.random(ig.n_voxels, dtype=np.float32) + 1).astype(np.float32)
    m_sub = meas.reshape(sg.n_sinos, sg.n_proj, sg.n_r)[:, sub::ns, :].reshape(-1).astype(np.float32)
    est = oracle.project_3d(sg, ig, x0, sub, ns)
    want = oracle.update(x0, oracle.backproject_3d(sg, ig, oracle.inverse_divide(m_sub, est), sub, ns), sens, 0.0,
                         True)
    P = ap.SiddonProjector(ig, sg)
    P.set_option(_lib.APIRL_OPT_ACCUMULATE, form)
    x = t(x0)
    bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    if listed:
        P.set_option(_lib.APIRL_OPT_SPARSE_IMAGE, _lib.APIRL_SPARSE_GEOMETRY)
        g = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        P.backproject_ones(g, sub, ns)
        for _ in range(2):  # the second pass starts from the first's cleared pairs
            xx = t(x0)
            P.em_pass_sparse(t(meas), xx, bp, t(sens), g, sub, ns)
        x = xx
    else:
        for _ in range(2):
            xx = t(x0)
            P.em_pass(t(meas), xx, bp, t(sens), sub, ns)
        x = xx
    torch.cuda.synchronize()
    assert rel(x.cpu().numpy(), want) <= 1e-5


def test_forms_refused_off_the_padded_layouts():
    ig, sg = geometry()
    P = ap.SiddonProjector(ig, sg)
    P.set_alpha_precision(True)
    with pytest.raises(ap.ApirlError) as ei:
        P.set_option(_lib.APIRL_OPT_ACCUMULATE, _lib.APIRL_ACC_WARP)
    assert ei.value.code == _lib.APIRL_ERR_NOT_SUPPORTED
    Q = ap.SiddonProjector(ig, sg)
    Q.set_option(_lib.APIRL_OPT_ACCUMULATE, _lib.APIRL_ACC_COMPENSATED)
    Q.set_alpha_precision(True)  # the FP64 walk has no padded layouts
    img = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    with pytest.raises(ap.ApirlError):
        Q.backproject(torch.ones(sg.subset_bins(0, 2), device=DEV), img, 0, 2)
    with pytest.raises(ap.ApirlError):
        P.set_option(_lib.APIRL_OPT_ACCUMULATE, 9)
