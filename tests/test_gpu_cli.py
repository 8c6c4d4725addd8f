"""The .par commands (MLEM, OSEM, project, backproject) end to end on the GPU:
interfile inputs written here, outputs read back and compared with the same
operations through the Python front end."""
import os
import subprocess

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import apirl_b200 as ap  # noqa: E402
from apirl_b200.geometry import ImageGeom, Sino3DGeom, Sino2DGeom  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "apirl_b200", "_build", "bin")
DEV = torch.device("cuda:0")


@pytest.fixture(autouse=True)
def _needs_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def write_image(path, ig, px):
    with open(path + ".h33", "w") as f:
        f.write("!INTERFILE :=\n!name of data file := %s.i33\n" % os.path.basename(path))
        f.write("!matrix size [1] := %d\n!matrix size [2] := %d\n!matrix size [3] := %d\n" % (ig.nx, ig.ny, ig.nz))
        f.write("scaling factor (mm/pixel) [1] := %r\nscaling factor (mm/pixel) [2] := %r\n" % (ig.dx, ig.dy))
        f.write("scaling factor (mm/pixel) [3] := %r\n!number format := short float\n" % ig.dz)
        f.write("!number of bytes per pixel := 4\n!END OF INTERFILE :=\n")
    np.asarray(px, np.float32).tofile(path + ".i33")


def write_sino3d(path, sg, vals):
    with open(path + ".h33", "w") as f:
        f.write("!INTERFILE :=\n!name of data file := %s.i33\nnumber of dimensions := 4\n" % os.path.basename(path))
        f.write("matrix axis label [4] := segment\n!matrix size [4] := %d\n" % sg.n_segments)
        f.write("matrix axis label [3] := axial coordinate\n!matrix size [3] := {%s}\n"
                % ",".join(str(n) for n in sg.sinos_per_segment))
        f.write("minimum ring difference per segment := {%s}\n" % ",".join(map(str, sg.min_rd)))
        f.write("maximum ring difference per segment := {%s}\n" % ",".join(map(str, sg.max_rd)))
        f.write("matrix axis label [2] := view\n!matrix size [2] := %d\n" % sg.n_proj)
        f.write("matrix axis label [1] := tangential coordinate\n!matrix size [1] := %d\n" % sg.n_r)
        f.write("number of rings := %d\n!END OF INTERFILE :=\n" % sg.n_rings)
    np.asarray(vals, np.float32).tofile(path + ".i33")


def write_sino2d(path, sg, vals):
    with open(path + ".h33", "w") as f:
        f.write("!INTERFILE :=\n!name of data file := %s.i33\n" % os.path.basename(path))
        f.write("!matrix size [1] := %d\n!matrix size [2] := %d\n!END OF INTERFILE :=\n" % (sg.n_r, sg.n_proj))
    np.asarray(vals, np.float32).tofile(path + ".i33")


def read_data(path, n):
    return np.fromfile(path + ".i33", dtype=np.float32, count=n)


def run(cmd, parfile, cwd):
    r = subprocess.run([os.path.join(BIN, cmd), parfile], cwd=cwd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    d = tmp_path_factory.mktemp("cli")
    ig = ImageGeom(40, 40, 7, 2.08, 2.08, 2.03)
    sg = Sino3DGeom.span1(18, 52, 4, 59.0, 4 * 2 * 2.03, 150.0, 2)
    rng = np.random.default_rng(3)
    x = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    P = ap.SiddonProjector(ig, sg)
    est = torch.zeros(sg.n_bins, dtype=torch.float32, device=DEV)
    P.project(torch.from_numpy(x).to(DEV), est)
    meas = rng.poisson(est.cpu().numpy() * 2).astype(np.float32)
    write_image(str(d / "x"), ig, x)
    write_image(str(d / "ones"), ig, np.ones(ig.n_voxels, np.float32))
    write_sino3d(str(d / "meas"), sg, meas)
    return d, ig, sg, x, meas, P, est.cpu().numpy()


def test_project_command(case):
    d, ig, sg, x, meas, P, est = case
    keys = {"input file": "x.h33", "output type": "Sinogram3D", "projector": "Siddon",
            "output filename": "proj", "output projection": "meas.h33"}
    keys.update({"cylindrical pet radius (in mm)": sg.r_scanner, "radius fov (in mm)": sg.r_fov,
                 "axial fov (in mm)": sg.axial_fov})
    with open(d / "proj.par", "w") as f:
        f.write("Projection Parameters :=\n" + "".join(f"{k} := {v}\n" for k, v in keys.items()) + "END :=\n")
    run("project", str(d / "proj.par"), d)
    got = read_data(str(d / "proj"), sg.n_bins)
    assert np.array_equal(got.view(np.uint32), est.view(np.uint32))


def test_backproject_command(case):
    d, ig, sg, x, meas, P, est = case
    keys = {"input type": "Sinogram3D", "input file": "meas.h33", "backprojector": "Siddon",
            "output image": "x.h33", "output filename": "bp", "number of subsets": 3, "subset index": 1}
    keys.update({"cylindrical pet radius (in mm)": sg.r_scanner, "radius fov (in mm)": sg.r_fov,
                 "axial fov (in mm)": sg.axial_fov})
    with open(d / "bp.par", "w") as f:
        f.write("Backproject Parameters :=\n" + "".join(f"{k} := {v}\n" for k, v in keys.items()) + "END :=\n")
    run("backproject", str(d / "bp.par"), d)
    got = read_data(str(d / "bp"), ig.n_voxels)
    sub = meas.reshape(sg.n_sinos, sg.n_proj, sg.n_r)[:, 1::3, :].reshape(-1)
    img = torch.zeros(ig.n_voxels, dtype=torch.float32, device=DEV)
    P.backproject(torch.from_numpy(sub).to(DEV), img, 1, 3)
    want = img.cpu().numpy()
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-5


def test_osem_command(case):
    d, ig, sg, x, meas, P, est = case
    keys = {"input type": "Sinogram3D", "input file": "meas.h33", "initial estimate": "ones.h33",
            "output filename prefix": "rec", "number of iterations": 2, "number of subsets": 3,
            "forwardprojector": "Siddon", "backprojector": "Siddon"}
    keys.update({"cylindrical pet radius (in mm)": sg.r_scanner, "radius fov (in mm)": sg.r_fov,
                 "axial fov (in mm)": sg.axial_fov})
    with open(d / "osem.par", "w") as f:
        f.write("OSEM Parameters :=\n" + "".join(f"{k} := {v}\n" for k, v in keys.items()) + "END :=\n")
    out = run("OSEM", str(d / "osem.par"), d)
    assert "iterations" in out
    got = read_data(str(d / "rec_final"), ig.n_voxels)
    want, _, _ = ap.osem_3d(ig, sg, meas, np.ones(ig.n_voxels, np.float32), 2, 3)
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-5
    assert os.path.exists(d / "rec.log")


def test_project_command_with_samples(case):
    """`siddon number of samples on the detector` (getSiddonProjectorParameters,
    data/src/readParameters.cpp:162-203) reaches the projector."""
    d, ig, sg, x, meas, P, est = case
    keys = {"input file": "x.h33", "output type": "Sinogram3D", "projector": "Siddon",
            "output filename": "proj_s", "output projection": "meas.h33",
            "siddon number of samples on the detector": 2,
            "siddon number of axial samples on the detector": 3}
    keys.update({"cylindrical pet radius (in mm)": sg.r_scanner, "radius fov (in mm)": sg.r_fov,
                 "axial fov (in mm)": sg.axial_fov})
    with open(d / "proj_s.par", "w") as f:
        f.write("Projection Parameters :=\n" + "".join(f"{k} := {v}\n" for k, v in keys.items()) + "END :=\n")
    run("project", str(d / "proj_s.par"), d)
    got = read_data(str(d / "proj_s"), sg.n_bins)
    Ps = ap.SiddonProjector(ig, sg)
    Ps.set_sampling(2, 3, False)
    want = torch.zeros(sg.n_bins, dtype=torch.float32, device=DEV)
    Ps.project(torch.from_numpy(x).to(DEV), want)
    want = want.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert not np.array_equal(got.view(np.uint32), est.view(np.uint32))


def test_osem_command_with_samples(case):
    d, ig, sg, x, meas, P, est = case
    keys = {"input type": "Sinogram3D", "input file": "meas.h33", "initial estimate": "ones.h33",
            "output filename prefix": "rec_s", "number of iterations": 1, "number of subsets": 3,
            "forwardprojector": "Siddon", "backprojector": "Siddon",
            "siddon number of samples on the detector": 2}
    keys.update({"cylindrical pet radius (in mm)": sg.r_scanner, "radius fov (in mm)": sg.r_fov,
                 "axial fov (in mm)": sg.axial_fov})
    with open(d / "osem_s.par", "w") as f:
        f.write("OSEM Parameters :=\n" + "".join(f"{k} := {v}\n" for k, v in keys.items()) + "END :=\n")
    run("OSEM", str(d / "osem_s.par"), d)
    got = read_data(str(d / "rec_s_final"), ig.n_voxels)
    want, _, _ = ap.osem_3d(ig, sg, meas, np.ones(ig.n_voxels, np.float32), 1, 3, sampling=(2, 1, False))
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-5


def test_mlem2d_command(tmp_path):
    ig = ImageGeom(64, 64, 1, 2.08, 2.08, 1.0)
    sg = Sino2DGeom(60, 80, 83.2, 300.0)
    rng = np.random.default_rng(8)
    x = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    P = ap.SiddonProjector(ig, sg)
    est = torch.zeros(sg.n_bins, dtype=torch.float32, device=DEV)
    P.project(torch.from_numpy(x).to(DEV), est)
    meas = rng.poisson(est.cpu().numpy()).astype(np.float32)
    write_image(str(tmp_path / "ones"), ig, np.ones(ig.n_voxels, np.float32))
    write_sino2d(str(tmp_path / "m2"), sg, meas)
    keys = {"input type": "Sinogram2D", "input file": "m2.h33", "initial estimate": "ones.h33",
            "output filename prefix": "r2", "number of iterations": 5, "cylindrical pet radius (in mm)": 300.0,
            "radius fov (in mm)": sg.r_fov}
    with open(tmp_path / "mlem.par", "w") as f:
        f.write("MLEM Parameters :=\n" + "".join(f"{k} := {v}\n" for k, v in keys.items()) + "END :=\n")
    run("MLEM", str(tmp_path / "mlem.par"), tmp_path)
    got = read_data(str(tmp_path / "r2_final"), ig.n_voxels)
    want, _, _ = ap.mlem_2d(ig, sg, meas, np.ones(ig.n_voxels, np.float32), 5)
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-5


def test_osem_command_mmr(tmp_path):
    """input type := Sinogram3DSiemensMmr (cmd/src/OSEM.cpp:416-425)."""
    d = tmp_path
    sg = Sino3DGeom.mmr(36, 86, 8, 3, 4)
    # every voxel crossed by rays of every subset (no zero sensitivity, which
    # with the reference's threshold 0 and >= would give NaN)
    ig = ImageGeom(48, 48, 14, 8.35, 8.35, 16.25)
    rng = np.random.default_rng(8)
    x = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    P = ap.SiddonProjector(ig, sg)
    est = torch.zeros(sg.n_bins, dtype=torch.float32, device=DEV)
    P.project(torch.from_numpy(x).to(DEV), est)
    meas = rng.poisson(est.cpu().numpy() * 0.2).astype(np.float32)
    write_image(str(d / "ones"), ig, np.ones(ig.n_voxels, np.float32))
    write_sino3d(str(d / "meas"), sg, meas)
    keys = {"input type": "Sinogram3DSiemensMmr", "input file": "meas.h33", "initial estimate": "ones.h33",
            "output filename prefix": "rec", "number of iterations": 2, "number of subsets": 4,
            "forwardprojector": "Siddon", "backprojector": "Siddon"}
    with open(d / "osem.par", "w") as f:
        f.write("OSEM Parameters :=\n" + "".join(f"{k} := {v}\n" for k, v in keys.items()) + "END :=\n")
    run("OSEM", str(d / "osem.par"), d)
    got = read_data(str(d / "rec_final"), ig.n_voxels)
    want, _, _ = ap.osem_3d(ig, sg, meas, np.ones(ig.n_voxels, np.float32), 2, 4)
    assert np.all(np.isfinite(want))
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-5


CUDA_KEYS = {"forwardprojector": "CuSiddonProjector", "backprojector": "CuSiddonProjector",
             "projector block size": "{128,1,1}", "backprojector block size": "{128,1,1}",
             "pixel update block size": "{512,1,1}", "gpu id": 0}


def test_cumlem_command(case):
    """cuMLEM (cmdGPU/src/cuMLEM.cpp) with a Sinogram3D: ML-EM through
    CuMlemSinogram3d; a subset count is ignored for this input type, as in the
    reference (:401-420)."""
    d, ig, sg, x, meas, P, est = case
    keys = {"input type": "Sinogram3D", "input file": "meas.h33", "initial estimate": "ones.h33",
            "output filename prefix": "cu", "number of iterations": 3, "number of subsets": 3}
    keys.update(CUDA_KEYS)
    keys.update({"cylindrical pet radius (in mm)": sg.r_scanner, "radius fov (in mm)": sg.r_fov,
                 "axial fov (in mm)": sg.axial_fov})
    with open(d / "cumlem.par", "w") as f:
        f.write("MLEM Parameters :=\n" + "".join(f"{k} := {v}\n" for k, v in keys.items()) + "END :=\n")
    out = run("cuMLEM", str(d / "cumlem.par"), d)
    assert "iterations" in out
    got = read_data(str(d / "cu_final"), ig.n_voxels)
    want, _, _ = ap.mlem_3d(ig, sg, meas, np.ones(ig.n_voxels, np.float32), 3)
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-5
    assert os.path.exists(d / "cu_sensitivity.h33")


def test_cumlem_command_mmr_subsets(tmp_path):
    """cuMLEM with a Sinogram3DSiemensMmr and a subset count runs
    CuOsemSinogram3d (cuMLEM.cpp:421-432)."""
    d = tmp_path
    sg = Sino3DGeom.mmr(36, 86, 8, 3, 4)
    ig = ImageGeom(48, 48, 14, 8.35, 8.35, 16.25)
    rng = np.random.default_rng(9)
    x = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    P = ap.SiddonProjector(ig, sg)
    est = torch.zeros(sg.n_bins, dtype=torch.float32, device=DEV)
    P.project(torch.from_numpy(x).to(DEV), est)
    meas = rng.poisson(est.cpu().numpy() * 0.2).astype(np.float32)
    write_image(str(d / "ones"), ig, np.ones(ig.n_voxels, np.float32))
    write_sino3d(str(d / "meas"), sg, meas)
    keys = {"input type": "Sinogram3DSiemensMmr", "input file": "meas.h33", "initial estimate": "ones.h33",
            "output filename prefix": "rec", "number of iterations": 2, "number of subsets": 4}
    keys.update(CUDA_KEYS)
    with open(d / "cumlem.par", "w") as f:
        f.write("MLEM Parameters :=\n" + "".join(f"{k} := {v}\n" for k, v in keys.items()) + "END :=\n")
    run("cuMLEM", str(d / "cumlem.par"), d)
    got = read_data(str(d / "rec_final"), ig.n_voxels)
    want, _, _ = ap.osem_3d(ig, sg, meas, np.ones(ig.n_voxels, np.float32), 2, 4)
    assert np.all(np.isfinite(want))
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-5


def _expf(v):
    import ctypes
    libm = ctypes.CDLL("libm.so.6")
    libm.expf.restype = ctypes.c_float
    libm.expf.argtypes = [ctypes.c_float]
    return np.array([libm.expf(float(a)) for a in np.asarray(v, np.float32)], np.float32)


def test_generate_acfs_command(case):
    """generateACFs (cmd/src/generateACFs.cpp): the map in 1/cm is divided by
    10, projected, and every non-zero bin becomes expf(bin), the others 1; the
    template sinogram times the factors goes to <output>_attCorrected."""
    d, ig, sg, x, meas, P, est = case
    rng = np.random.default_rng(11)
    mu_cm = (rng.random(ig.n_voxels, dtype=np.float32) * 0.096).astype(np.float32)
    mu_cm[: ig.nx * ig.ny] = 0  # a slice of zeros: bins that miss the map keep 1
    write_image(str(d / "mu"), ig, mu_cm)
    keys = {"input file": "mu.h33", "output type": "Sinogram3D", "output filename": "acf",
            "output projection": "meas.h33", "projector": "CuSiddonProjector",
            "projector block size": "{128,1,1}", "gpu id": 0,
            "cylindrical pet radius (in mm)": sg.r_scanner, "radius fov (in mm)": sg.r_fov,
            "axial fov (in mm)": sg.axial_fov}
    with open(d / "acf.par", "w") as f:
        f.write("generateACFs Parameters :=\n" + "".join(f"{k} := {v}\n" for k, v in keys.items()) + "END :=\n")
    run("generateACFs", str(d / "acf.par"), d)
    got = read_data(str(d / "acf"), sg.n_bins)
    proj = torch.zeros(sg.n_bins, dtype=torch.float32, device=DEV)
    P.project(torch.from_numpy(mu_cm / np.float32(10)).to(DEV), proj)
    proj = proj.cpu().numpy()
    want = np.where(proj != 0, _expf(proj), np.float32(1)).astype(np.float32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert (got == 1).any() and (got > 1).any()
    corrected = read_data(str(d / "acf_attCorrected"), sg.n_bins)
    assert np.array_equal(corrected.view(np.uint32), (meas * want).astype(np.float32).view(np.uint32))


def test_osem_command_saves_iterations(case):
    """save estimates at iteration intervals (OsemSinogram3d.cpp:266-276):
    <prefix>_iter_<t> after iterations t = 0, 2, ...; the last saved image
    equals the final one."""
    d, ig, sg, x, meas, P, est = case
    keys = {"input type": "Sinogram3D", "input file": "meas.h33", "initial estimate": "ones.h33",
            "output filename prefix": "rsave", "number of iterations": 3, "number of subsets": 3,
            "forwardprojector": "Siddon", "backprojector": "Siddon", "save estimates at iteration intervals": 2}
    keys.update({"cylindrical pet radius (in mm)": sg.r_scanner, "radius fov (in mm)": sg.r_fov,
                 "axial fov (in mm)": sg.axial_fov})
    with open(d / "osem_save.par", "w") as f:
        f.write("OSEM Parameters :=\n" + "".join(f"{k} := {v}\n" for k, v in keys.items()) + "END :=\n")
    run("OSEM", str(d / "osem_save.par"), d)
    assert os.path.exists(d / "rsave_iter_0.h33") and os.path.exists(d / "rsave_iter_2.h33")
    assert not os.path.exists(d / "rsave_iter_1.h33")
    final = read_data(str(d / "rsave_final"), ig.n_voxels)
    assert np.array_equal(read_data(str(d / "rsave_iter_2"), ig.n_voxels).view(np.uint32), final.view(np.uint32))
    want1, _, _ = ap.osem_3d(ig, sg, meas, np.ones(ig.n_voxels, np.float32), 1, 3)
    got1 = read_data(str(d / "rsave_iter_0"), ig.n_voxels)
    assert np.linalg.norm(got1 - want1) / np.linalg.norm(want1) <= 1e-5


def test_iteration_hook_c_abi(case):
    """apirl_set_iteration_hook (apirl_b200.set_iteration_hook): the driver
    hands the image after every interval-th iteration to the callback;
    removed, it calls nothing."""
    d, ig, sg, x, meas, P, est = case
    seen = []
    ap.set_iteration_hook(lambda t, img: seen.append((t, img)), 1)
    try:
        img, _, _ = ap.mlem_3d(ig, sg, meas, np.ones(ig.n_voxels, np.float32), 2)
    finally:
        ap.set_iteration_hook()
    assert [t for t, _ in seen] == [0, 1]
    assert np.array_equal(seen[1][1].view(np.uint32), img.view(np.uint32))
    seen.clear()
    ap.mlem_3d(ig, sg, meas, np.ones(ig.n_voxels, np.float32), 1)
    assert seen == []
    from apirl_b200 import _lib
    assert _lib.load().apirl_set_iteration_hook(None, -1, None) != 0


def test_osem_command_sensitivity_from_file(case):
    """sensitivity filename (OsemSinogram3d.cpp:84-116): every subset's
    computed sensitivity is written as <prefix>_sensitivity_subset_<s>, and a
    run given "<prefix>_sensitivity" reads them back instead of computing."""
    d, ig, sg, x, meas, P, est = case
    base = {"input type": "Sinogram3D", "input file": "meas.h33", "initial estimate": "ones.h33",
            "number of iterations": 2, "number of subsets": 3, "forwardprojector": "Siddon",
            "backprojector": "Siddon", "cylindrical pet radius (in mm)": sg.r_scanner,
            "radius fov (in mm)": sg.r_fov, "axial fov (in mm)": sg.axial_fov}
    for name, extra in (("sa", {}), ("sb", {"sensitivity filename": "sa_sensitivity"})):
        keys = dict(base, **{"output filename prefix": name}, **extra)
        with open(d / f"{name}.par", "w") as f:
            f.write("OSEM Parameters :=\n" + "".join(f"{k} := {v}\n" for k, v in keys.items()) + "END :=\n")
        run("OSEM", str(d / f"{name}.par"), d)
    for s in range(3):
        assert os.path.exists(d / f"sa_sensitivity_subset_{s}.h33")
        assert not os.path.exists(d / f"sb_sensitivity_subset_{s}.h33")
    _, _, sens_all = ap.osem_3d(ig, sg, meas, np.ones(ig.n_voxels, np.float32), 0, 3, all_sens=True)
    for s in range(3):
        got = read_data(str(d / f"sa_sensitivity_subset_{s}"), ig.n_voxels)
        assert np.linalg.norm(got - sens_all[s]) / np.linalg.norm(sens_all[s]) <= 1e-6
    a = read_data(str(d / "sa_final"), ig.n_voxels)
    b = read_data(str(d / "sb_final"), ig.n_voxels)
    assert np.linalg.norm(a - b) / np.linalg.norm(a) <= 1e-6
