"""Precision study on the full 3D workload (test infrastructure; needs a GPU).

    python tests/precision_study.py [--subiters K] > precision.json

The first K OSEM sub-iterations of the 256x256x81 / 1261x336x336 job (the
bench workload: attenuation in the sensitivity, 5e8 uint32 counts, 21 subsets,
from an image of ones) run through the CUDA path in several arithmetic forms
and, on the host, through the FP64 oracle (double Siddon walk, double LOR
geometry, double accumulation).  Per sub-iteration it prints the relative L2
and max-abs error of each GPU image against the FP64 image, and of the FP64
likelihood of each form against the FP64 oracle's.  Forms:

  f32       the reference's float arithmetic (bit-identical to the reference's
            own Siddon projector), uint32 counts
  u16       the same with the counts stored as uint16 (checked to round-trip
            bit-exactly first)
  f64alpha  FP64 walk geometry (LOR end points, alphas, crossings), fp32
            projection and accumulation

It also compares the backprojection of one ratio sinogram accumulated with
fp32 atomics on the GPU, and accumulated serially in float in the reference's
order (the oracle's float path), against the FP64 backprojection, and reports
the adjoint residual |<Ax,y> - <x,A^T y>| / |<Ax,y>| of the GPU operators.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    m = np.isfinite(a) & np.isfinite(b)
    return float(np.linalg.norm(a[m] - b[m]) / max(np.linalg.norm(b[m]), 1e-300))


def max_abs(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    m = np.isfinite(a) & np.isfinite(b)
    return float(np.max(np.abs(a[m] - b[m])))


def main():
    ap_ = argparse.ArgumentParser()
    ap_.add_argument("--subiters", type=int, default=4)
    args = ap_.parse_args()

    import torch
    import apirl_b200 as ap
    from oracle_lib import Oracle
    import bench

    dev = torch.device("cuda:0")
    log = lambda m: print(f"[precision] {m}", file=sys.stderr, flush=True)  # noqa: E731
    w = bench.setup_workload(dev, log)
    P, ig, sg = w["P"], w["ig"], w["sg"]
    nsub = bench.NSUB
    nv = ig.n_voxels
    orc = Oracle()

    counts32 = w["counts"]
    counts_np = counts32.view(torch.int32).cpu().numpy().astype(np.int64)
    assert counts_np.max() < 65536
    counts16 = torch.from_numpy(counts_np.astype(np.uint16)).to(dev)
    assert np.array_equal(counts16.cpu().numpy().astype(np.int64), counts_np)  # uint16 round trip
    meas64 = counts_np.astype(np.float64).reshape(sg.n_sinos, sg.n_proj, sg.n_r)
    atten64 = w["atten"].cpu().numpy().astype(np.float64).reshape(sg.n_sinos, sg.n_proj, sg.n_r)

    # GPU forms: each its own image, all from ones.
    P64 = ap.SiddonProjector(ig, sg)
    P64.set_alpha_precision(True)
    sens64 = torch.zeros((nsub, nv), dtype=torch.float32, device=dev)
    for s in range(nsub):
        a_s = w["atten"].view(sg.n_sinos, sg.n_proj, sg.n_r)[:, s::nsub, :].contiguous().view(-1)
        P64.backproject(a_s, sens64[s], s, nsub)
        ap.force_positive(sens64[s])
    forms = {
        "f32": dict(P=P, counts=counts32, sens=w["sens"]),
        "u16": dict(P=P, counts=counts16, sens=w["sens"]),
        "f64alpha": dict(P=P64, counts=counts32, sens=sens64),
    }
    for f in forms.values():
        f["x"] = torch.ones(nv, dtype=torch.float32, device=dev)
        f["bp"] = torch.zeros(nv, dtype=torch.float32, device=dev)
        f["lik"] = torch.zeros(1, dtype=torch.float64, device=dev)

    x64 = np.ones(nv, np.float64)
    rows = []
    for s in range(args.subiters):
        t0 = time.time()
        # FP64 oracle sub-iteration (OsemSinogram3d.cpp:159-237 in double).
        a_s = np.ascontiguousarray(atten64[:, s::nsub, :]).reshape(-1)
        sens_s = orc.backproject_3d(sg, ig, a_s, s, nsub, dtype=np.float64)
        est = orc.project_3d(sg, ig, x64, s, nsub, dtype=np.float64)
        m_s = np.ascontiguousarray(meas64[:, s::nsub, :]).reshape(-1)
        nz = est != 0
        lik64 = float(np.sum(m_s[nz] * np.log(est[nz]) - est[nz]))
        ratio = np.where((m_s != 0) & nz, m_s / np.where(nz, est, 1.0), 0.0)
        bp64 = orc.backproject_3d(sg, ig, ratio, s, nsub, dtype=np.float64)
        with np.errstate(invalid="ignore", divide="ignore"):
            x64 = np.where(sens_s >= 0, x64 * bp64 / sens_s, 0.0)
        row = {"subiteration": s, "oracle_s": round(time.time() - t0, 1)}
        for name, f in forms.items():
            f["P"].em_pass(f["counts"], f["x"], f["bp"], f["sens"][s], s, nsub, lik=f["lik"])
            torch.cuda.synchronize(dev)
            xg = f["x"].cpu().numpy()
            row[name] = {"rel_l2": rel(xg, x64), "max_abs": max_abs(xg, x64),
                         "lik_rel": abs(f["lik"].item() - lik64) / abs(lik64)}
        log(json.dumps(row))
        rows.append(row)

    # Backprojection accumulation order: one ratio sinogram of subset 0.
    s = 0
    x1 = forms["f32"]["x"].cpu().numpy()
    est32 = orc.project_3d(sg, ig, x1, s, nsub)
    m_s = np.ascontiguousarray(meas64[:, s::nsub, :]).reshape(-1).astype(np.float32)
    ratio32 = orc.inverse_divide(m_s, est32)
    bp_exact = orc.backproject_3d(sg, ig, ratio32.astype(np.float64), s, nsub, dtype=np.float64)
    bp_serial = orc.backproject_3d(sg, ig, ratio32, s, nsub, threads=1)
    bp_gpu = torch.zeros(nv, dtype=torch.float32, device=dev)
    P.backproject(torch.from_numpy(ratio32).to(dev), bp_gpu, s, nsub)
    acc = {"gpu_fp32_atomics_rel_l2": rel(bp_gpu.cpu().numpy(), bp_exact),
           "reference_order_fp32_rel_l2": rel(bp_serial, bp_exact)}

    # Adjoint residual of the GPU operators (FP64 dot products).
    rng = np.random.default_rng(0)
    xa = rng.random(nv, dtype=np.float32)
    ya = rng.random(sg.subset_bins(s, nsub), dtype=np.float32)
    adj = {}
    for name, PP in (("f32", P), ("f64alpha", P64)):
        Ax = torch.zeros(ya.size, dtype=torch.float32, device=dev)
        PP.project(torch.from_numpy(xa).to(dev), Ax, s, nsub)
        Aty = torch.zeros(nv, dtype=torch.float32, device=dev)
        PP.backproject(torch.from_numpy(ya).to(dev), Aty, s, nsub)
        lhs = float(np.dot(Ax.cpu().numpy().astype(np.float64), ya.astype(np.float64)))
        rhs = float(np.dot(xa.astype(np.float64), Aty.cpu().numpy().astype(np.float64)))
        adj[name] = abs(lhs - rhs) / abs(lhs)

    print(json.dumps({"study": "precision", "workload": bench.WORKLOAD, "subiterations": rows,
                      "backprojection_accumulation": acc, "adjoint_residual": adj}))


if __name__ == "__main__":
    main()
