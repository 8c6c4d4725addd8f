"""The cuMLEM command's parameter-file handling (cmdGPU/src/cuMLEM.cpp:159-330,
reconGPU/src/readCudaParameters.cpp), CPU only: every case here stops before
the first CUDA call.

* the file must end in .par (cuMLEM.cpp:176-183);
* the block-size keys are required and must read {x,y,z}
  (ProcessBlockSizeString, readCudaParameters.cpp:22-48);
* the projectors must be CuSiddonProjector (cuMLEM.cpp:280-323);
* the input type must be Sinogram3D or Sinogram3DSiemensMmr.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "apirl_b200", "_build", "bin", "cuMLEM")

BASE = {"input type": "Sinogram3D", "input file": "meas.h33", "initial estimate": "ones.h33",
        "output filename prefix": "rec", "number of iterations": 1,
        "forwardprojector": "CuSiddonProjector", "backprojector": "CuSiddonProjector",
        "projector block size": "{128,1,1}", "backprojector block size": "{128,1,1}",
        "pixel update block size": "{512,1,1}", "gpu id": 0}


@pytest.fixture(scope="module", autouse=True)
def _built():
    if not os.path.exists(EXE):
        pytest.skip("cuMLEM not built")


def run(tmp_path, keys, name="c.par"):
    p = tmp_path / name
    p.write_text("MLEM Parameters :=\n" + "".join(f"{k} := {v}\n" for k, v in keys.items()) + "END :=\n")
    return subprocess.run([EXE, str(p)], cwd=tmp_path, capture_output=True, text=True, timeout=60)


def test_needs_par_extension(tmp_path):
    r = run(tmp_path, BASE, "c.txt")
    assert r.returncode != 0 and ".par" in r.stderr


@pytest.mark.parametrize("k", ["projector block size", "backprojector block size", "pixel update block size"])
def test_block_sizes_required(tmp_path, k):
    keys = dict(BASE)
    del keys[k]
    r = run(tmp_path, keys)
    assert r.returncode != 0 and k in r.stderr


@pytest.mark.parametrize("bad", ["128,1,1", "{128,1}", "{}"])
def test_block_size_format(tmp_path, bad):
    keys = dict(BASE, **{"projector block size": bad})
    r = run(tmp_path, keys)
    assert r.returncode != 0 and "projector block size" in r.stderr


def test_projector_names(tmp_path):
    r = run(tmp_path, dict(BASE, forwardprojector="RotationBasedProjector"))
    assert r.returncode != 0 and "RotationBasedProjector" in r.stderr
    r = run(tmp_path, dict(BASE, backprojector="Siddon"))
    assert r.returncode != 0 and "Siddon" in r.stderr


def test_required_keys(tmp_path):
    keys = dict(BASE)
    del keys["number of iterations"]
    r = run(tmp_path, keys)
    assert r.returncode != 0 and "number of iterations" in r.stderr


def test_input_type(tmp_path):
    # the initial estimate is read before the input type is checked
    (tmp_path / "ones.h33").write_text(
        "!INTERFILE :=\n!name of data file := ones.i33\n!matrix size [1] := 2\n!matrix size [2] := 2\n"
        "!matrix size [3] := 1\nscaling factor (mm/pixel) [1] := 1\nscaling factor (mm/pixel) [2] := 1\n"
        "scaling factor (mm/pixel) [3] := 1\n!number format := short float\n!number of bytes per pixel := 4\n"
        "!END OF INTERFILE :=\n")
    (tmp_path / "ones.i33").write_bytes(b"\0" * 16)
    r = run(tmp_path, dict(BASE, **{"input type": "Michelogram"}))
    assert r.returncode != 0 and "Michelogram" in r.stderr
