"""LOR-sharded OSEM (apirl_b200.sharded) on CPU: world_size-2 gloo ranks with
a stand-in backend that computes its shard's operations with the oracle; the
sharded reconstruction equals the oracle's single-process OSEM.  This covers
the host logic (partition, all-reduce of the backprojection, the likelihood
and the sensitivity images, update order); the CUDA backend is checked on a
GPU by tests/test_gpu_sharded.py."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from apirl_b200.geometry import ImageGeom, Sino3DGeom
from apirl_b200.sharded import shard_ranges, ShardedOsem

NSUB, ITERS = 3, 2


def geometry():
    return ImageGeom(24, 24, 7, 2.08, 2.08, 2.03), Sino3DGeom.span1(12, 30, 4, 36.0, 4 * 4.054, 150.0, 3)


def data(oracle):
    ig, sg = geometry()
    rng = np.random.default_rng(12)
    truth = (rng.random(ig.n_voxels, dtype=np.float32) + 0.5).astype(np.float32)
    meas = rng.poisson(oracle.project_3d(sg, ig, truth) * 0.7).astype(np.float32)
    return ig, sg, meas


class OracleShard:
    """Stand-in backend: the shard's operations through the oracle (whole
    subset computed, bins outside the shard set to zero)."""

    def __init__(self, oracle, ig, sg, meas, first, n):
        self.o, self.ig, self.sg, self.meas = oracle, ig, sg, meas
        self.first, self.n = first, n

    def _mask(self, s):
        nk = self.sg.subset_nproj(s, NSUB)
        m = np.zeros((self.sg.n_sinos, nk, self.sg.n_r), bool)
        m[self.first:self.first + self.n] = True
        return m.reshape(-1)

    def zeros_image(self):
        return torch.zeros(self.ig.n_voxels, dtype=torch.float32)

    def scalar(self):
        return torch.zeros(1, dtype=torch.float64)

    def sensitivity(self, s, out):
        ones = self._mask(s).astype(np.float32)
        out += torch.from_numpy(self.o.backproject_3d(self.sg, self.ig, ones, s, NSUB, threads=1))

    def em_pass(self, x, bp, s, lik):
        mask = self._mask(s)
        est = self.o.project_3d(self.sg, self.ig, x.numpy(), s, NSUB, threads=1)
        m = self.meas.reshape(self.sg.n_sinos, self.sg.n_proj, self.sg.n_r)[:, s::NSUB, :].reshape(-1)
        sel = mask & (est != 0)
        e = est[sel].astype(np.float64)
        lik[0] = float(np.sum(m[sel].astype(np.float64) * np.log(e) - e))
        ratio = np.where(mask, self.o.inverse_divide(m, est), 0).astype(np.float32)
        bp += torch.from_numpy(self.o.backproject_3d(self.sg, self.ig, ratio, s, NSUB, threads=1))

    def force_positive(self, img):
        img.clamp_(min=0)

    def update(self, x, bp, sens):
        x.copy_(torch.from_numpy(self.o.update(x.numpy(), bp.numpy(), sens.numpy(), np.float32(0), True)))
        bp.zero_()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import datetime
    import sys
    import torch.distributed as dist
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    sys.path.insert(0, here)
    from oracle_lib import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        oracle = Oracle()
        ig, sg, meas = data(oracle)
        first, n = shard_ranges(sg.n_sinos, world)[rank]
        job = ShardedOsem(OracleShard(oracle, ig, sg, meas, first, n), NSUB, dist)
        x = torch.ones(ig.n_voxels, dtype=torch.float32)
        liks = job.run(x, ITERS)
        q.put((rank, x.numpy().copy(), liks))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_shard_ranges():
    for n, w in ((75, 2), (1261, 8), (7, 7), (100, 3)):
        r = shard_ranges(n, w)
        assert sum(c for _, c in r) == n
        assert all(r[i][0] + r[i][1] == r[i + 1][0] for i in range(w - 1))
        assert max(c for _, c in r) - min(c for _, c in r) <= 1
    with pytest.raises(ValueError):
        shard_ranges(3, 4)


def test_two_rank_sharded_osem_equals_single_process(oracle):
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=240) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    ig, sg, meas = data(oracle)
    want, want_lik, _ = oracle.osem_3d(sg, ig, np.ones(ig.n_voxels, np.float32), meas, ITERS, NSUB, threads=1)
    for rank, x, liks in res:
        assert np.linalg.norm(x - want) / np.linalg.norm(want) <= 1e-5
        assert np.allclose(liks, want_lik[:-1].astype(np.float64), rtol=1e-5)
    assert np.array_equal(res[0][1], res[1][1])  # every rank holds the same image
