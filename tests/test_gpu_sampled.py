"""Several rays per bin on the GPU against the oracle: radial and axial
oversampling (SiddonProjector(nSamples, nAxialSamples),
recon/src/SiddonProjector.cpp:16-32, 346-397) and one ray per ring pair
(Projector::setMultipleLorsPerBin, recon/inc/Projector.h:54-60), on span-1 and
span-3 sinograms.  The oracle's sampled projectors are pinned to the reference
by tests/test_oracle_sampled.py.

Tolerances as in test_gpu_parity.py: projection bit-exact, backprojections
rel L2 <= 1e-5, one OSEM iteration rel L2 <= 1e-4, FP64 likelihood rel 1e-9
against the oracle's FP64 sum of the same estimates.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import apirl_b200 as ap  # noqa: E402
from apirl_b200 import _lib  # noqa: E402
from apirl_b200.geometry import ImageGeom, Sino3DGeom  # noqa: E402

DEV = torch.device("cuda:0")

SAMPLINGS = [(2, 1, 0), (1, 2, 0), (3, 2, 0), (1, 1, 1), (2, 2, 1), (1, 2, 1)]


def t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a, np.float32).view(np.uint32),
                          np.ascontiguousarray(b, np.float32).view(np.uint32))


def geometry(span):
    ig = ImageGeom(48, 48, 9, 2.08, 2.08, 2.03)
    if span == 1:
        return ig, Sino3DGeom.span1(25, 48, 5, 72.0, 5 * 4.054, 150.0, 3)
    return ig, Sino3DGeom.span(25, 48, 5, 72.0, 5 * 4.054, 150.0, 3, 4)


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ap.load_library()


@pytest.mark.parametrize("span", [1, 3])
@pytest.mark.parametrize("ns,nas,multi", SAMPLINGS)
def test_sampled_projectors_vs_oracle(oracle, span, ns, nas, multi):
    ig, sg = geometry(span)
    rng = np.random.default_rng(100 + 10 * span + ns + 3 * nas + 7 * multi)
    img = rng.random(ig.n_voxels, dtype=np.float32)
    P = ap.SiddonProjector(ig, sg)
    P.set_sampling(ns, nas, multi)
    for sub, nsub in ((-1, 1), (2, 5)):
        want = oracle.sampled_3d(sg, ig, 0, ns, nas, multi, img, subset=sub, nsub=nsub)
        out = torch.zeros(P.num_bins(sub, nsub), dtype=torch.float32, device=DEV)
        P.project(t(img), out, sub, nsub)
        assert bits_equal(out.cpu().numpy(), want)
        v = rng.random(want.size, dtype=np.float32)
        v[rng.random(want.size) < 0.2] = 0
        e = rng.random(want.size, dtype=np.float32)
        e[rng.random(want.size) < 0.2] = 0
        bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        P.backproject(t(v), bp, sub, nsub)
        assert rel(bp.cpu().numpy(), oracle.sampled_3d(sg, ig, 1, ns, nas, multi, v, subset=sub, nsub=nsub)) <= 1e-5
        db = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        P.divide_and_backproject(t(v), t(e), db, sub, nsub)
        want_db = oracle.sampled_3d(sg, ig, 2, ns, nas, multi, v, e, subset=sub, nsub=nsub)
        assert rel(db.cpu().numpy(), want_db) <= 1e-5


@pytest.mark.parametrize("span", [1, 3])
def test_sampled_em_pass_vs_oracle(oracle, span):
    ns, nas, multi = 2, 2, 1
    ig, sg = geometry(span)
    rng = np.random.default_rng(7 + span)
    x0 = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    full = oracle.sampled_3d(sg, ig, 0, ns, nas, multi, x0)
    meas = rng.poisson(full * 0.5).astype(np.float32)
    sens = (rng.random(ig.n_voxels, dtype=np.float32) + 1).astype(np.float32)
    subset, nsub = 1, 5
    meas_sub = meas.reshape(sg.n_sinos, sg.n_proj, sg.n_r)[:, subset::nsub, :].reshape(-1)
    est = oracle.sampled_3d(sg, ig, 0, ns, nas, multi, x0, subset=subset, nsub=nsub)
    nz = est != 0
    e64 = est.astype(np.float64)
    want_lik = float(np.sum(meas_sub[nz].astype(np.float64) * np.log(e64[nz]) - e64[nz]))
    ratio = oracle.inverse_divide(meas_sub, est)
    bp_want = oracle.sampled_3d(sg, ig, 1, ns, nas, multi, ratio, subset=subset, nsub=nsub, threads=1)
    want_x = oracle.update(x0, bp_want, sens, np.float32(0), True)
    P = ap.SiddonProjector(ig, sg)
    P.set_sampling(ns, nas, multi)
    for dtype, packed in ((np.float32, False), (np.uint32, True), (np.uint16, False)):
        x = t(x0)
        bp = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
        lik = torch.zeros(1, dtype=torch.float64, device=DEV)
        counts = t((meas_sub if packed else meas).astype(dtype))
        P.em_pass(counts, x, bp, t(sens), subset, nsub, lik=lik, counts_packed=packed)
        torch.cuda.synchronize()
        assert rel(x.cpu().numpy(), want_x) <= 1e-5
        assert float(bp.abs().max()) == 0.0
        assert abs(lik.item() - want_lik) <= 1e-9 * abs(want_lik)


def _oracle_osem(oracle, sg, ig, meas, x, iters, nsub, samp):
    ns, nas, multi = samp
    sens = []
    for s in range(nsub):
        ones = np.ones(sg.subset_bins(s, nsub), np.float32)
        sens.append(np.maximum(oracle.sampled_3d(sg, ig, 1, ns, nas, multi, ones, subset=s, nsub=nsub), 0))
    m3 = meas.reshape(sg.n_sinos, sg.n_proj, sg.n_r)
    for _ in range(iters):
        for s in range(nsub):
            est = oracle.sampled_3d(sg, ig, 0, ns, nas, multi, x, subset=s, nsub=nsub)
            ratio = oracle.inverse_divide(m3[:, s::nsub, :].reshape(-1), est)
            bp = oracle.sampled_3d(sg, ig, 1, ns, nas, multi, ratio, subset=s, nsub=nsub, threads=1)
            x = oracle.update(x, bp, sens[s], np.float32(0), True)
    return x, sens[0]


@pytest.mark.parametrize("samp", [(2, 1, 0), (1, 1, 1)])
def test_sampled_osem_driver_vs_oracle(oracle, samp):
    ig, sg = geometry(3)
    rng = np.random.default_rng(31)
    truth = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    meas = rng.poisson(oracle.sampled_3d(sg, ig, 0, *samp, truth) * 0.5).astype(np.float32)
    init = np.ones(ig.n_voxels, np.float32)
    want, want_sens0 = _oracle_osem(oracle, sg, ig, meas, init, 1, 3, samp)
    img, lik, sens0 = ap.osem_3d(ig, sg, meas, init, 1, 3, sampling=samp)
    assert rel(sens0, want_sens0) <= 1e-5
    # Voxels no ray of a subset crosses have zero sensitivity; with threshold 0
    # and >= the reference's update gives 0 * 0 / 0 = NaN there
    # (OsemSinogram3d.cpp:24-33, :217-237), and so must the GPU.
    nan = np.isnan(want)
    assert np.array_equal(np.isnan(img), nan)
    assert rel(img[~nan], want[~nan]) <= 1e-4
    assert np.isfinite(lik[0])  # later passes project those NaN voxels, as the reference does


def test_sampling_reset_and_validation(oracle):
    ig, sg = geometry(1)
    rng = np.random.default_rng(3)
    img = rng.random(ig.n_voxels, dtype=np.float32)
    P = ap.SiddonProjector(ig, sg)
    plain = torch.zeros(P.num_bins(), dtype=torch.float32, device=DEV)
    P.project(t(img), plain)
    steps_plain = int(P.count_steps().sum().item())
    P.set_sampling(3, 2, 1)
    steps_s = int(P.count_steps().sum().item())
    assert steps_s > 3 * steps_plain  # six rays per bin walk about six times the segments
    P.set_sampling(1, 1, 0)  # back to one ray per bin: the plain tables again
    again = torch.zeros_like(plain)
    P.project(t(img), again)
    assert bits_equal(again.cpu().numpy(), plain.cpu().numpy())
    assert int(P.count_steps().sum().item()) == steps_plain
    for bad in ((0, 1, 0), (1, 0, 0), (_lib.APIRL_MAX_SAMPLES + 1, 1, 0)):
        with pytest.raises(ap.ApirlError):
            P.set_sampling(*bad)
    P.set_sampling(2, 1, 0)
    with pytest.raises(ap.ApirlError):
        P.set_alpha_precision(True)
    P2 = ap.SiddonProjector(*geometry(1))
    P2.set_alpha_precision(True)
    with pytest.raises(ap.ApirlError):
        P2.set_sampling(2, 1, 0)
