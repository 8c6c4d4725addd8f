"""The reference's GPU-side C++ API on the GPU (tests/cu_api_check.cpp):

* CuSiddonProjector's device-buffer calls (reconGPU/inc/CuProjector.h:98-105)
  equal its host-buffer calls: projection bit for bit (whole sinogram and a
  subset), backprojection and divide-and-backprojection rel L2 <= 1e-6 (fp32
  atomics), adding into the caller's device image, copyResult filling the
  host object, the estimate left unchanged;
* CuProjectorInterface (reconGPU/inc/CuProjectorInterface.h:53-172) around a
  CuSiddonProjector equals the plain projector, overwrites its output, returns
  false for Sinogram2D; around a CuProjector of the caller's own it passes the
  per-sinogram axial end points and the grid (ceil(nProj*nR/x), sinograms, 1);
* CuMlemSinogram3d / CuOsemSinogram3d (reconGPU/inc/CuMlemSinogram3d.h,
  CuOsemSinogram3d.h) equal MlemSinogram3d / OsemSinogram3d (rel L2 <= 1e-5),
  and reject the hexagonal kind, a GPU index that does not exist and
  projectors that are not CuSiddonProjector.
"""
import os
import subprocess

import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "apirl_b200", "_build")


@pytest.fixture(scope="module")
def results(tmp_path_factory):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    tmp = tmp_path_factory.mktemp("cuapi")
    exe = str(tmp / "cu_api_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-o", exe, os.path.join(ROOT, "tests", "cu_api_check.cpp"),
                    "-I/usr/local/cuda/include", f"-L{BUILD}", "-lapirl_b200_host", "-lapirl_b200",
                    "-L/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{BUILD}"], check=True)
    r = subprocess.run([exe, str(tmp)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    res = {}
    for line in r.stdout.splitlines():
        k, _, v = line.partition(" ")
        res[k] = v.split()
    return res


def flag(res, k):
    return res[k] == ["1"]


def test_device_buffer_projection(results):
    assert flag(results, "dev_project_ok")
    assert flag(results, "dev_project_bits_equal")
    assert flag(results, "dev_project_buffer_bits_equal")
    assert flag(results, "dev_project_subset_bits_equal")
    assert flag(results, "dev_null_buffer_false")


def test_device_buffer_backprojection(results):
    ok, r = results["dev_backproject_rel"]
    assert ok == "1" and float(r) <= 1e-6
    assert float(results["dev_backproject_accumulates_rel"][0]) <= 1e-6
    ok, r = results["dev_divide_rel"]
    assert ok == "1" and float(r) <= 1e-6
    assert flag(results, "dev_divide_estimate_unchanged")


def test_projector_interface(results):
    assert flag(results, "iface_project_bits_equal")
    assert flag(results, "iface_project_subset_bits_equal")
    for k in ("iface_backproject_rel", "iface_divide_rel"):
        ok, r = results[k]
        assert ok == "1" and float(r) <= 1e-6
    assert flag(results, "iface_2d_false")
    assert flag(results, "iface_bad_gpu_false")


def test_projector_interface_with_own_projector(results):
    assert flag(results, "iface_rings_equal")
    n_sinos = int(results["iface_sinograms"][0])
    gx, gy, gz, bx = map(int, results["iface_grid"])
    assert (gx, gy, gz, bx) == (-(-18 * 52 // 64), n_sinos, 1, 64)
    assert flag(results, "iface_foreign_false")


def test_cu_reconstructors(results):
    assert results["cumlem_block"] == ["256", "1", "1"]
    ok, r = results["cumlem_rel"]
    assert ok == "1" and float(r) <= 1e-5
    assert float(results["cumlem_likelihood_rel"][0]) <= 1e-9
    ok, r = results["cuosem_rel"]
    assert ok == "1" and float(r) <= 1e-5
    assert int(results["cuosem_likelihoods"][0]) == 2 * 3 + 1
    assert flag(results, "cumlem_hexagonal_false")
    assert flag(results, "cumlem_bad_gpu_false")
    assert flag(results, "cumlem_foreign_false")
    assert results["cuda_error"] == ["0"]
