"""Batched / served 3D OSEM on one GPU (the C ABI's apirl_batch_*).

``Batch`` queues jobs of any geometry and advances every admitted job by one
pass per ``step()`` in shared launches; ``serve()`` replays an arrival stream
against it (continuous batching: jobs join as memory frees up) and reports
per-job latency.
"""
import ctypes
import time

import numpy as np

from . import _lib
from ._lib import check, JobDescC
from .projector import _img_c, _sino3d_c

_DT = {np.dtype(np.float32): _lib.APIRL_F32, np.dtype(np.uint32): _lib.APIRL_U32,
       np.dtype(np.uint16): _lib.APIRL_U16}


class Job:
    def __init__(self, image_geom, sino_geom, counts, iters, nsubsets, mult=None, add=None, init=None, tag=None,
                 update_positive_sens=False):
        """update_positive_sens: update only where sens > 0 (else the reference's
        sens >= 0, which gives NaN where no ray of a subset crosses a voxel)."""
        self.image_geom, self.sino_geom = image_geom, sino_geom
        self.update_positive_sens = bool(update_positive_sens)
        self.counts = np.ascontiguousarray(counts)
        if self.counts.dtype not in _DT:
            raise TypeError("counts must be float32, uint32 or uint16")
        f32 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float32)
        self.mult, self.add, self.init = f32(mult), f32(add), f32(init)
        self.iters, self.nsubsets, self.tag = iters, nsubsets, tag

    def desc(self):
        sc = _sino3d_c(self.sino_geom)
        p = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)
        d = JobDescC(_img_c(self.image_geom), sc, p(self.counts), _DT[self.counts.dtype], p(self.mult), p(self.add),
                     p(self.init), self.iters, self.nsubsets, int(self.update_positive_sens))
        d._keep = (sc,)
        return d

    def footprint(self):
        return int(_lib.load().apirl_job_footprint(ctypes.byref(self.desc())))


class Batch:
    def __init__(self, device=0, budget_bytes=64 << 30):
        self.lib = _lib.load()
        h = ctypes.c_void_p()
        check(self.lib.apirl_batch_create(device, int(budget_bytes), ctypes.byref(h)))
        self.h = h
        self.jobs = {}

    def close(self):
        if self.h:
            self.lib.apirl_batch_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, job):
        jid = ctypes.c_int64()
        d = job.desc()
        check(self.lib.apirl_batch_submit(self.h, ctypes.byref(d), ctypes.byref(jid)))
        self.jobs[jid.value] = job
        return jid.value

    def step(self):
        na, nq = ctypes.c_int(), ctypes.c_int()
        check(self.lib.apirl_batch_step(self.h, ctypes.byref(na), ctypes.byref(nq)))
        return na.value, nq.value

    def result(self, jid):
        job = self.jobs[jid]
        out = np.zeros(job.image_geom.n_voxels, np.float32)
        lik = np.zeros(job.iters * job.nsubsets + 1, np.float64)
        done = ctypes.c_int()
        check(self.lib.apirl_batch_result(self.h, jid, out.ctypes.data_as(ctypes.c_void_p),
                                          lik.ctypes.data_as(ctypes.c_void_p), ctypes.byref(done)))
        if not done.value:
            return None
        del self.jobs[jid]
        return out, lik

    def run_all(self, jobs):
        """Submits every job and steps until all are done.  Returns results in order."""
        ids = [self.submit(j) for j in jobs]
        res = {}
        while len(res) < len(ids):
            na, nq = self.step()
            if len(ids) - na - nq > len(res):  # some job finished since the last look
                for i in ids:
                    if i not in res:
                        r = self.result(i)
                        if r is not None:
                            res[i] = r
        return [res[i] for i in ids]


def serve(jobs, arrivals_s, device=0, budget_bytes=64 << 30):
    """Continuous batching against an arrival schedule (seconds from start).

    Jobs are submitted when their arrival time has passed; every step advances
    all admitted jobs.  Returns (results, latency_s per job, makespan_s)."""
    b = Batch(device, budget_bytes)
    order = np.argsort(arrivals_s)
    t0 = time.perf_counter()
    ids, submitted_at, done_at, results = {}, {}, {}, {}
    nxt = 0
    while len(done_at) < len(jobs):
        now = time.perf_counter() - t0
        while nxt < len(jobs) and arrivals_s[order[nxt]] <= now:
            k = int(order[nxt])
            ids[b.submit(jobs[k])] = k
            submitted_at[k] = arrivals_s[k]
            nxt += 1
        if len(ids) == len(done_at):
            # nothing in flight: wait for the next arrival
            time.sleep(max(0.0, arrivals_s[order[nxt]] - (time.perf_counter() - t0)))
            continue
        na, nq = b.step()
        now = time.perf_counter() - t0
        if len(ids) - na - nq > len(done_at):  # some job finished since the last look
            for jid, k in list(ids.items()):
                if k in done_at:
                    continue
                r = b.result(jid)
                if r is not None:
                    results[k] = r
                    done_at[k] = now
    b.close()
    lat = np.array([done_at[k] - submitted_at[k] for k in range(len(jobs))])
    return [results[k] for k in range(len(jobs))], lat, max(done_at.values())
