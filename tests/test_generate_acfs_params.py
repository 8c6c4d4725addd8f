"""The generateACFs command's parameter-file handling
(cmd/src/generateACFs.cpp:180-275), CPU only: every case here stops before
the first CUDA call."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "apirl_b200", "_build", "bin", "generateACFs")

BASE = {"input file": "mu.h33", "output type": "Sinogram3D", "output filename": "acf",
        "output projection": "tmpl.h33", "projector": "Siddon"}


@pytest.fixture(scope="module", autouse=True)
def _built():
    if not os.path.exists(EXE):
        pytest.skip("generateACFs not built")


def run(tmp_path, keys, section="generateACFs"):
    p = tmp_path / "a.par"
    p.write_text(f"{section} Parameters :=\n" + "".join(f"{k} := {v}\n" for k, v in keys.items()) + "END :=\n")
    return subprocess.run([EXE, str(p)], cwd=tmp_path, capture_output=True, text=True, timeout=60)


def write_map(tmp_path):
    (tmp_path / "mu.h33").write_text(
        "!INTERFILE :=\n!name of data file := mu.i33\n!matrix size [1] := 2\n!matrix size [2] := 2\n"
        "!matrix size [3] := 1\nscaling factor (mm/pixel) [1] := 1\nscaling factor (mm/pixel) [2] := 1\n"
        "scaling factor (mm/pixel) [3] := 1\n!number format := short float\n!number of bytes per pixel := 4\n"
        "!END OF INTERFILE :=\n")
    (tmp_path / "mu.i33").write_bytes(b"\0" * 16)


@pytest.mark.parametrize("k", ["input file", "output type", "output filename", "output projection", "projector"])
def test_required_keys(tmp_path, k):
    keys = dict(BASE)
    del keys[k]
    r = run(tmp_path, keys)
    assert r.returncode != 0 and k in r.stderr


def test_wrong_section(tmp_path):
    r = run(tmp_path, BASE, section="MLEM")
    assert r.returncode != 0


def test_cuda_projector_needs_block_size(tmp_path):
    write_map(tmp_path)
    r = run(tmp_path, dict(BASE, projector="CuSiddonProjector"))
    assert r.returncode != 0 and "projector block size" in r.stderr


def test_output_type(tmp_path):
    write_map(tmp_path)
    r = run(tmp_path, dict(BASE, **{"output type": "Michelogram"}))
    assert r.returncode != 0 and "Michelogram" in r.stderr
