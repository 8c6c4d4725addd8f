"""The C++ host layer's file formats (CPU only): reading interfile files written
by the reference's own writers (tests/golden/ref_io, made by make_golden.py),
writing files the reference reads back, and the .par reader's error codes
(data/inc/ParametersFile.h:34-39)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden", "ref_io")
BUILD = os.path.join(ROOT, "apirl_b200", "_build")


@pytest.fixture(scope="module")
def results(tmp_path_factory):
    tmp = tmp_path_factory.mktemp("hostio")
    exe = str(tmp / "host_io_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-o", exe, os.path.join(ROOT, "tests", "host_io_check.cpp"),
                    "-I/usr/local/cuda/include", f"-L{BUILD}", "-lapirl_b200_host", "-lapirl_b200",
                    "-L/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{BUILD}"], check=True)
    out = subprocess.run([exe, GOLD, str(tmp)], check=True, capture_output=True, text=True).stdout
    res = {}
    for line in out.splitlines():
        k, _, v = line.partition(" ")
        res[k] = v.split()
    res["_tmp"] = str(tmp)
    return res


def test_reads_reference_image(results):
    assert results["image_read"] == ["1"]
    nx, ny, nz, dx, dy, dz = results["image_size"]
    assert (int(nx), int(ny), int(nz)) == (8, 6, 3)
    assert (float(dx), float(dy), float(dz)) == (2.5, 2.0, 3.25)
    px = np.arange(144, dtype=np.float32) * 0.25 + 1
    assert float(results["image_checksum"][0]) == pytest.approx(float(np.sum(px.astype(np.float64) * np.arange(1, 145))))
    assert results["image_roundtrip"][0] == "1"
    assert results["image_roundtrip"][1] == results["image_checksum"][0]


def test_reads_reference_sinogram3d(results):
    r = results["sino_segments"]
    assert r == ["3", "sinograms", "7", "proj", "8", "r", "6", "bins", "336"]
    vals = np.arange(336, dtype=np.float32) * 0.5 - 7
    assert float(results["sino_checksum"][0]) == pytest.approx(float(np.sum(vals.astype(np.float64) * np.arange(1, 337))))
    # subset 1 of 3: angles 1, 4, 7 of each of the 7 sinograms
    sub = vals.reshape(7, 8, 6)[:, 1::3, :].reshape(-1).astype(np.float64)
    assert results["subset_bins"][0] == str(sub.size)
    assert float(results["subset_bins"][2]) == pytest.approx(float(np.sum(sub * np.arange(1, sub.size + 1))))
    assert results["sino_roundtrip"] == ["336", results["sino_checksum"][0]]


def test_par_reader_error_codes(results):
    assert results["par_subsets"] == ["0", "21"]
    # repeated key -> 1, key not found (comment line) -> 2, wrong command -> 5, no file -> 3
    assert results["par_errors"] == ["1", "2", "5", "3"]


def test_reference_reads_our_files(results, ref):
    from apirl_b200.geometry import Sino3DGeom
    dims, pix, px = ref.read_image(os.path.join(results["_tmp"], "image_ours.h33"))
    assert list(dims) == [8, 6, 3] and list(pix) == [2.5, 2.0, 3.25]
    assert np.array_equal(px, np.arange(144, dtype=np.float32) * 0.25 + 1)
    sg = Sino3DGeom(8, 6, 3, 20.0, 12.0, 60.0, [0, 1, -1], [0, 1, -1])
    vals, nseg = ref.read_sino3d(os.path.join(results["_tmp"], "sino_ours.h33"), sg)
    assert nseg == 3 and np.array_equal(vals, np.arange(336, dtype=np.float32) * 0.5 - 7)
