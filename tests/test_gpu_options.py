"""Projector options that change how the padded passes run, not what they
compute: the L2 persisting window (APIRL_OPT_L2_PERSIST) and the order of the
sparse passes' list of bins (APIRL_OPT_LIST_ORDER, by walk length within
groups).  Each gives the default's image to the atomics' order (rel L2 <=
1e-6) and likelihood to 1e-7 relative (the geometry image of each run is its
own atomics' sum), over two passes in a row."""
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


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ap.load_library()


def run_passes(option, value, sparse):
    ig, sg = ImageGeom(64, 64, 13, 2.08, 2.08, 2.03), Sino3DGeom.span1(40, 72, 7, 66.56, 7 * 4.054, 200.0, 6)
    rng = np.random.default_rng(21)
    P = ap.SiddonProjector(ig, sg)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    est = torch.zeros(P.num_bins(), dtype=torch.float32, device=DEV)
    P.project(t(x0), est)
    meas = rng.poisson(est.cpu().numpy() * 0.3).astype(np.uint32)
    if option is not None:
        P.set_option(option, value)
    sub, ns = 1, 4
    g = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    P.backproject_ones(g, sub, ns)
    x = t(x0)
    bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    liks = []
    P.set_option(_lib.APIRL_OPT_SPARSE_IMAGE, _lib.APIRL_SPARSE_GEOMETRY)
    for _ in range(2):
        lik = torch.zeros(1, dtype=torch.float64, device=DEV)
        if sparse:
            P.em_pass_sparse(t(meas), x, bp, g, g, sub, ns, lik=lik)
        else:
            P.em_pass(t(meas), x, bp, g, sub, ns, lik=lik)
        torch.cuda.synchronize()
        liks.append(lik.item())
    return x.cpu().numpy(), np.array(liks)


@pytest.mark.parametrize("sparse", [False, True])
def test_l2_window_changes_nothing(sparse):
    ref, lref = run_passes(None, 0, sparse)
    got, lgot = run_passes(_lib.APIRL_OPT_L2_PERSIST, 1, sparse)
    assert rel(got, ref) <= 1e-6 and np.allclose(lgot, lref, rtol=1e-7, atol=0)


def _persisting_l2_limit():
    """The context's cudaLimitPersistingL2CacheSize (enum value 6)."""
    import ctypes
    rt = ctypes.CDLL("libcudart.so.12")
    v = ctypes.c_size_t(0)
    assert rt.cudaDeviceGetLimit(ctypes.byref(v), 6) == 0
    return v.value


def test_l2_window_puts_the_limit_back():
    """The option raises the context's persisting-L2 limit and puts the value
    it found back when it is turned off and when the projector goes."""
    ig, sg = ImageGeom(32, 32, 5, 2.08, 2.08, 2.03), Sino3DGeom.span1(16, 32, 3, 33.28, 3 * 4.054, 150.0, 2)
    before = _persisting_l2_limit()
    P = ap.SiddonProjector(ig, sg)
    P.set_option(_lib.APIRL_OPT_L2_PERSIST, 1)
    assert _persisting_l2_limit() > 0
    P.set_option(_lib.APIRL_OPT_L2_PERSIST, 0)
    assert _persisting_l2_limit() == before
    P.set_option(_lib.APIRL_OPT_L2_PERSIST, 1)
    P.close()
    assert _persisting_l2_limit() == before


@pytest.mark.parametrize("group", [32, 256, 2048])
def test_list_order_changes_nothing(group):
    ref, lref = run_passes(None, 0, True)
    got, lgot = run_passes(_lib.APIRL_OPT_LIST_ORDER, group, True)
    assert rel(got, ref) <= 1e-6 and np.allclose(lgot, lref, rtol=1e-7, atol=0)


def test_list_order_rejects_other_sizes():
    ig, sg = ImageGeom(16, 16, 3, 2.0, 2.0, 2.0), Sino3DGeom.span1(8, 16, 3, 16.0, 3 * 4.0, 100.0, 1)
    P = ap.SiddonProjector(ig, sg)
    for bad in (16, 100, 4096, -1):
        with pytest.raises(ap.ApirlError):
            P.set_option(_lib.APIRL_OPT_LIST_ORDER, bad)


@pytest.mark.parametrize("unroll", [4, 6, 8])
@pytest.mark.parametrize("sparse", [False, True])
def test_gather_unroll_changes_nothing(unroll, sparse):
    ref, lref = run_passes(None, 0, sparse)
    got, lgot = run_passes(_lib.APIRL_OPT_GATHER_UNROLL, unroll, sparse)
    assert rel(got, ref) <= 1e-6 and np.allclose(lgot, lref, rtol=1e-7, atol=0)


def test_autotune_shape_keeps_the_fastest_and_the_image():
    """apirl_projector_autotune_ex on the listed pass: a block size and gather
    depth from the candidates, a positive time, the input image unchanged;
    passes afterwards equal the default's."""
    ig, sg = ImageGeom(64, 64, 13, 2.08, 2.08, 2.03), Sino3DGeom.span1(40, 72, 7, 66.56, 7 * 4.054, 200.0, 6)
    rng = np.random.default_rng(21)
    P = ap.SiddonProjector(ig, sg)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    est = torch.zeros(P.num_bins(), dtype=torch.float32, device=DEV)
    P.project(t(x0), est)
    meas = t(rng.poisson(est.cpu().numpy() * 0.3).astype(np.uint32))
    P.set_option(_lib.APIRL_OPT_SPARSE_IMAGE, _lib.APIRL_SPARSE_GEOMETRY)
    g = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    P.backproject_ones(g, 1, 4)
    x = t(x0)
    block, unroll, ms = P.autotune_shape(meas, x, zimg=g, subset=1, nsubsets=4)
    torch.cuda.synchronize()
    assert block in (64, 96, 128, 192, 256) and unroll in (4, 6, 8) and ms > 0
    assert np.array_equal(x.cpu().numpy(), x0)
    bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    lik = torch.zeros(1, dtype=torch.float64, device=DEV)
    P.em_pass_sparse(meas, x, bp, g, g, 1, 4, lik=lik)
    Q = ap.SiddonProjector(ig, sg)
    Q.set_option(_lib.APIRL_OPT_SPARSE_IMAGE, _lib.APIRL_SPARSE_GEOMETRY)
    xq = t(x0)
    lq = torch.zeros(1, dtype=torch.float64, device=DEV)
    Q.em_pass_sparse(meas, xq, bp, g, g, 1, 4, lik=lq)
    torch.cuda.synchronize()
    assert rel(x.cpu().numpy(), xq.cpu().numpy()) <= 1e-6
    assert abs(lik.item() - lq.item()) <= 1e-9 * abs(lq.item())
