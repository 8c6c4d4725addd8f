"""Buffers that outlive a call, and CUDA errors that must not go unreported.

* One projector takes the one-walk backprojection (A_s^T v and A_s^T 1 along
  the same walks, into a second padded pair it allocates on first use), then
  sparse passes that grow its list of bins with counts twice, then the
  one-walk backprojection again: both images still match the oracle, and the
  projector's destruction leaves no CUDA error behind.
* The same on sinogram shards (apirl_projector_set_shard): the shards' images
  sum to the oracle's whole backprojections.
* The drivers with a multiplicative sinogram (which take that one-walk
  sensitivity and then size the list) run twice in a row with nothing left
  pending.
* An error left pending by someone else's launch is reported by the next
  entry point as APIRL_ERR_CUDA, not discarded, and the call after that runs.

Tolerances: backprojections rel L2 <= 1e-5 against the oracle (fp32 atomics
in another order); images of the same walks rel L2 <= 1e-6.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import apirl_b200 as ap  # noqa: E402
from apirl_b200 import _lib  # noqa: E402
from apirl_b200.geometry import ImageGeom, Sino3DGeom  # noqa: E402
from apirl_b200.sharded import shard_ranges  # noqa: E402

DEV = torch.device("cuda:0")


def t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def geometry():
    # 25 angles: 4 subsets of 7, 6, 6, 6 angles; 2 subsets of 13 and 12
    return ImageGeom(48, 48, 9, 2.08, 2.08, 2.03), Sino3DGeom.span1(25, 48, 5, 72.0, 5 * 4.054, 150.0, 3)


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ap.load_library()


def _cudart():
    return ctypes.CDLL("libcudart.so.12")


def assert_nothing_pending():
    """No CUDA error pending on this thread (read through the runtime, which
    also clears it), and a torch launch after it runs."""
    torch.cuda.synchronize()
    rt = _cudart()
    rt.cudaPeekAtLastError.restype = ctypes.c_int
    assert rt.cudaPeekAtLastError() == 0
    z = torch.ones(1024, device=DEV) * 2
    torch.cuda.synchronize()
    assert float(z.sum().item()) == 2048.0


def one_walk_sequence(oracle, P, ig, sg, v_full, sinos, counts):
    """backproject_and_ones, two sparse passes growing the list, then
    backproject_and_ones again; returns both rounds' images (numpy)."""
    sub, ns = 3, 4
    nb = P.num_bins(sub, ns)
    out = []
    v = v_full.reshape(sg.n_sinos, sg.n_proj, sg.n_r)[sinos][:, sub::ns, :].reshape(-1)
    assert v.size == nb
    x = t(np.ones(ig.n_voxels, np.float32))
    bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    sens = t(np.ones(ig.n_voxels, np.float32))
    P.set_option(_lib.APIRL_OPT_SPARSE_IMAGE, _lib.APIRL_SPARSE_GEOMETRY)
    for rnd in range(2):
        img = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        gimg = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        P.backproject_and_ones(t(v), img, gimg, sub, ns)
        torch.cuda.synchronize()
        out.append((img.cpu().numpy(), gimg.cpu().numpy()))
        if rnd == 0:
            # lists of 6 angles (subset 3 of 4), then 13 (subset 0 of 2): the
            # projector's list grows on each
            for s2, n2 in ((3, 4), (0, 2)):
                g2 = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
                P.backproject_ones(g2, s2, n2)
                lik = torch.zeros(1, dtype=torch.float64, device=DEV)
                P.em_pass_sparse(t(counts), x, bp, sens, g2, s2, n2, lik=lik)
                torch.cuda.synchronize()
                assert np.isfinite(lik.item())
    return out


def test_one_walk_backprojection_survives_list_growth(oracle):
    ig, sg = geometry()
    rng = np.random.default_rng(5)
    v_full = rng.random(sg.n_sinos * sg.n_proj * sg.n_r, dtype=np.float32)
    counts = rng.poisson(2.0, sg.n_sinos * sg.n_proj * sg.n_r).astype(np.uint32)
    P = ap.SiddonProjector(ig, sg)
    rounds = one_walk_sequence(oracle, P, ig, sg, v_full, np.arange(sg.n_sinos), counts)
    sub, ns = 3, 4
    v_sub = v_full.reshape(sg.n_sinos, sg.n_proj, sg.n_r)[:, sub::ns, :].reshape(-1)
    want_v = oracle.backproject_3d(sg, ig, v_sub, sub, ns)
    want_1 = oracle.backproject_3d(sg, ig, np.ones_like(v_sub), sub, ns)
    for img, gimg in rounds:
        assert rel(img, want_v) <= 1e-5
        assert rel(gimg, want_1) <= 1e-5
    assert rel(rounds[1][0], rounds[0][0]) <= 1e-6
    P.close()
    assert_nothing_pending()


@pytest.mark.parametrize("world", [2, 3])
def test_one_walk_backprojection_on_shards(oracle, world):
    ig, sg = geometry()
    rng = np.random.default_rng(50 + world)
    v_full = rng.random(sg.n_sinos * sg.n_proj * sg.n_r, dtype=np.float32)
    counts = rng.poisson(2.0, sg.n_sinos * sg.n_proj * sg.n_r).astype(np.uint32)
    sub, ns = 3, 4
    v_sub = v_full.reshape(sg.n_sinos, sg.n_proj, sg.n_r)[:, sub::ns, :]
    sums = [np.zeros(ig.n_voxels, np.float64), np.zeros(ig.n_voxels, np.float64)]
    sums2 = [np.zeros(ig.n_voxels, np.float64), np.zeros(ig.n_voxels, np.float64)]
    for first, n in shard_ranges(sg.n_sinos, world):
        P = ap.SiddonProjector(ig, sg)
        P.set_shard(first, n)
        rounds = one_walk_sequence(oracle, P, ig, sg, v_full, np.arange(first, first + n), counts)
        for k in range(2):
            sums[k] += rounds[0][k]
            sums2[k] += rounds[1][k]
        P.close()
        assert_nothing_pending()
    want_v = oracle.backproject_3d(sg, ig, v_sub.reshape(-1), sub, ns)
    want_1 = oracle.backproject_3d(sg, ig, np.ones(v_sub.size, np.float32), sub, ns)
    for s in (sums, sums2):
        assert rel(s[0], want_v) <= 1e-5
        assert rel(s[1], want_1) <= 1e-5


def test_drivers_with_factors_twice(oracle):
    """apirl_osem_3d with a multiplicative sinogram (one-walk sensitivity,
    then the list sized for the passes) twice in a row, then a plain call:
    equal results, nothing pending after either."""
    ig, sg = geometry()
    rng = np.random.default_rng(17)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    mult = (rng.random(sg.n_sinos * sg.n_proj * sg.n_r, dtype=np.float32) * 0.5 + 0.5).astype(np.float32)
    meas = rng.poisson(oracle.project_3d(sg, ig, x0) * mult * 2).astype(np.float32)
    init = np.ones(ig.n_voxels, np.float32)
    a, la, _ = ap.osem_3d(ig, sg, meas, init, 2, 4, mult=mult)
    assert_nothing_pending()
    b, lb, _ = ap.osem_3d(ig, sg, meas, init, 2, 4, mult=mult)
    assert_nothing_pending()
    assert rel(b, a) <= 1e-6 and abs(lb[0] - la[0]) <= 1e-9 * abs(la[0])
    c, _, _ = ap.mlem_3d(ig, sg, meas, init, 2, mult=mult)
    assert np.all(np.isfinite(c))
    assert_nothing_pending()


def test_pending_error_is_reported_not_discarded():
    """A failed runtime call of someone else's (cudaSetDevice of a device that
    does not exist, rejected on the host) leaves a non-sticky error pending;
    the next entry point returns APIRL_ERR_CUDA naming it and does no work;
    the one after runs."""
    rt = _cudart()
    rt.cudaSetDevice.restype = ctypes.c_int
    rt.cudaPeekAtLastError.restype = ctypes.c_int
    x = torch.full((1000,), -1.0, dtype=torch.float32, device=DEV)
    torch.cuda.synchronize()
    assert rt.cudaSetDevice(ctypes.c_int(1 << 20)) != 0
    assert rt.cudaPeekAtLastError() != 0
    with pytest.raises(ap.ApirlError) as ei:
        ap.force_positive(x)
    assert "pending" in str(ei.value)
    torch.cuda.synchronize()
    assert float(x.min().item()) == -1.0  # the refused call did nothing
    ap.force_positive(x)  # negative values become 0 (Image::forcePositive)
    torch.cuda.synchronize()
    assert float(x.min().item()) == 0.0 and float(x.max().item()) == 0.0
    assert_nothing_pending()
