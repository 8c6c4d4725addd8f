"""LOR shards on the GPU (apirl_projector_set_shard, apirl_b200.sharded):
shard projections are the matching sinograms of the whole projection (bit
for bit), shard backprojections and likelihoods sum to the whole ones, and
the sharded OSEM on one rank equals the plain driver.  Several shards in one
process stand in for several ranks (their partial images summed here); the
collective logic itself is covered by tests/test_sharded.py on CPU."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import apirl_b200 as ap  # noqa: E402
from apirl_b200.geometry import ImageGeom, Sino3DGeom  # noqa: E402
from apirl_b200.sharded import shard_ranges, ShardedOsem, GpuShard  # noqa: E402

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


def geometry():
    return ImageGeom(48, 48, 9, 2.08, 2.08, 2.03), Sino3DGeom.span1(25, 48, 5, 72.0, 5 * 4.054, 150.0, 3)


@pytest.mark.parametrize("world", [2, 3])
def test_shards_partition_the_operators(oracle, world):
    ig, sg = geometry()
    rng = np.random.default_rng(world)
    img = rng.random(ig.n_voxels, dtype=np.float32)
    sub, ns = 1, 5
    full = oracle.project_3d(sg, ig, img, sub, ns).reshape(sg.n_sinos, -1)
    v = rng.random(full.size, dtype=np.float32).reshape(sg.n_sinos, -1)
    bp_sum = np.zeros(ig.n_voxels, np.float64)
    for first, n in shard_ranges(sg.n_sinos, world):
        P = ap.SiddonProjector(ig, sg)
        P.set_shard(first, n)
        assert P.num_bins(sub, ns) == n * full.shape[1]
        out = torch.zeros(P.num_bins(sub, ns), dtype=torch.float32, device=DEV)
        P.project(t(img), out, sub, ns)
        got = out.cpu().numpy().reshape(n, -1)
        assert np.array_equal(got.view(np.uint32), full[first:first + n].view(np.uint32))
        bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        P.backproject(t(v[first:first + n]), bp, sub, ns)
        bp_sum += bp.cpu().numpy()
    assert rel(bp_sum, oracle.backproject_3d(sg, ig, v.reshape(-1), sub, ns)) <= 1e-5


def test_sharded_pass_sums_to_whole_pass(oracle):
    ig, sg = geometry()
    rng = np.random.default_rng(9)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    counts = t(rng.poisson(oracle.project_3d(sg, ig, x0) * 2).astype(np.uint32))
    sub, ns = 2, 5
    P = ap.SiddonProjector(ig, sg)
    bp_full = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    lik_full = torch.zeros(1, dtype=torch.float64, device=DEV)
    P.em_project_backproject(counts, t(x0), bp_full, sub, ns, lik=lik_full)
    bp_sum = torch.zeros_like(bp_full)
    lik_sum = 0.0
    for first, n in shard_ranges(sg.n_sinos, 3):
        b = GpuShard(ig, sg, counts, ns, first, n)
        bp = b.zeros_image()
        lik = b.scalar()
        b.em_pass(t(x0), bp, sub, lik)
        bp_sum += bp
        lik_sum += lik.item()
    torch.cuda.synchronize()
    assert rel(bp_sum.cpu().numpy(), bp_full.cpu().numpy()) <= 1e-6
    assert abs(lik_sum - lik_full.item()) <= 1e-9 * abs(lik_full.item())


def test_sharded_osem_one_rank_equals_driver(oracle):
    ig, sg = geometry()
    rng = np.random.default_rng(10)
    truth = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    meas = rng.poisson(oracle.project_3d(sg, ig, truth) * 0.5).astype(np.float32)
    job = ShardedOsem(GpuShard(ig, sg, t(meas), 4, 0, sg.n_sinos), 4)
    x = torch.ones(ig.n_voxels, dtype=torch.float32, device=DEV)
    liks = job.run(x, 2)
    want, want_lik, _ = ap.osem_3d(ig, sg, meas, np.ones(ig.n_voxels, np.float32), 2, 4)
    assert rel(x.cpu().numpy(), want) <= 1e-5
    # the driver (no multiplicative or additive term) takes the geometry-image
    # pass, whose likelihood sums the same terms in another order
    assert np.allclose(liks, want_lik[:-1], rtol=1e-7)


def test_geometry_sparse_shards_sum_to_whole_pass(oracle):
    """Shards taking the geometry-image sparse pass (each with its own
    G_s = A_s^T 1): their backprojections and likelihoods sum to the whole
    full pass's."""
    ig, sg = geometry()
    rng = np.random.default_rng(12)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    counts = t(rng.poisson(oracle.project_3d(sg, ig, x0) * 0.5).astype(np.uint32))
    sub, ns = 1, 5
    P = ap.SiddonProjector(ig, sg)
    bp_full = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    lik_full = torch.zeros(1, dtype=torch.float64, device=DEV)
    P.em_project_backproject(counts, t(x0), bp_full, sub, ns, lik=lik_full)
    bp_sum = torch.zeros_like(bp_full)
    lik_sum = 0.0
    for first, n in shard_ranges(sg.n_sinos, 3):
        b = GpuShard(ig, sg, counts, ns, first, n, geometry_sparse=True)
        bp = b.zeros_image()
        lik = b.scalar()
        b.em_pass(t(x0), bp, sub, lik)
        bp_sum += bp
        lik_sum += lik.item()
    torch.cuda.synchronize()
    assert rel(bp_sum.cpu().numpy(), bp_full.cpu().numpy()) <= 1e-6
    assert abs(lik_sum - lik_full.item()) <= 1e-6 * abs(lik_full.item())
