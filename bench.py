"""Benchmark: 3D OSEM sub-iterations per second on the full 3D workload.

Workload (one "step" = one OSEM sub-iteration): image 256x256x81 (2.08 x 2.08 x
2.03 mm), 41 rings, span-1 sinograms of all ring pairs with |ring difference|
<= 20 (1261 sinograms of 336 r x 336 angles, 142,361,856 bins), 21 subsets of
16 angles; water cylinder with 6 hot spheres, attenuation factors in the
sensitivity, 5e8 Poisson counts stored as uint32.  Steps cycle through the
21 subsets as an OSEM iteration does.

Arms
  default            the CUDA path (fused projection/ratio/backprojection kernel
                     + pixel update), counts and images resident in HBM.
  --impl reference   the reference APIRL CPU code (oracle/_ref, compiled from the
                     reference sources) on the host cores, or the oracle
                     restatement where the reference was not built; each step is
                     one sub-iteration restricted to a sample of segments.

Multi-GPU: the job does not exchange data between GPUs; each rank runs its own
replica of the reconstruction and `value` sums the ranks' sub-iterations over
the slowest rank's time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "OSEM subiters/s (256²×81)"
UNIT = "subiter/s"
NSUB = 21
TOTAL_COUNTS = 5e8
# Pixel update of the timed passes: x <- x * bp / sens where sens > 0, else 0.
# The reference's OSEM rule (threshold 0 with >=, OsemSinogram3d.cpp:24-33,
# :217-237, kept by the library's drivers) gives 0 * 0 / 0 = NaN at voxels
# that no ray of a subset crosses; this workload has 4 such voxels in subset
# 3 and 2 in subset 16 (image corners), and the NaN reaches every voxel
# within three more passes.  The passes do the same work either way.
UPDATE_GE = False
L2_FLUSH_BYTES = 256 << 20
# DRAM bytes (read + write) per fused-kernel launch of the full workload,
# mean of the four timed launches captured with ncu --metrics dram__bytes_read.sum,
# dram__bytes_write.sum (one pass; profiles/k_em_pass_osem3d_256x256x81.md).
FULL_TRAFFIC_BYTES = 2.603e8
# The same for the nonzero pass (the default): mean of the three timed
# launches inside the capture's first 400 launches.
NONZERO_TRAFFIC_BYTES = 1.498e8
WORKLOAD = ("3D OSEM 256x256x81 image, 41 rings span-1 |rd|<=20: 1261 sinograms x 336 angles x 336 r, "
            "21 subsets, attenuation in sensitivity, 5e8 counts uint32")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock / throttle samples taken while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"apirl_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # nvidia-smi takes a moment to start: wait for its first sample, so
        # that sampling runs through the whole timed region that follows.
        deadline = time.time() + 5.0
        while time.time() < deadline and self.proc.poll() is None:
            try:
                if os.path.getsize(self.path) > 0:
                    break
            except OSError:
                pass
            time.sleep(0.01)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def setup_workload(dev, log, max_ring_diff=None, alpha="f32"):
    """Builds the resident state of the 3D OSEM job on `dev` (outside timing).
    max_ring_diff < 20 keeps only the segments |rd| <= max_ring_diff (a smaller
    case of the same kernels, used for profiler captures)."""
    import torch
    import apirl_b200 as ap
    from apirl_b200 import workloads
    from apirl_b200.geometry import Sino3DGeom

    ig, sg = workloads.c2_geometry()
    if max_ring_diff is not None and max_ring_diff < 20:
        sg = Sino3DGeom.span1(sg.n_proj, sg.n_r, sg.n_rings, sg.r_fov, sg.axial_fov, sg.r_scanner, max_ring_diff)
    P = ap.SiddonProjector(ig, sg, device=dev.index)
    if alpha == "f64":
        P.set_alpha_precision(True)  # precision-study mode: FP64 walk geometry
    nb = P.num_bins()
    t0 = time.time()
    atten, counts = workloads.c2_device_arrays(P, dev)
    nv = ig.n_voxels
    sens = torch.zeros((NSUB, nv), dtype=torch.float32, device=dev)
    for s in range(NSUB):
        # OsemSinogram3d::computeSensitivity with the multiplicative term:
        # sens_s = A_s^T (attenuation of subset s), then forcePositive.
        a_s = atten.view(sg.n_sinos, sg.n_proj, sg.n_r)[:, s::NSUB, :].contiguous().view(-1)
        P.backproject(a_s, sens[s], s, NSUB)
        ap.force_positive(sens[s])
    x = torch.ones(nv, dtype=torch.float32, device=dev)
    bp = torch.zeros(nv, dtype=torch.float32, device=dev)
    # Siddon segments per subset (all bins: forward; bins with counts: backward).
    fwd, bwd = [], []
    cv = counts.view(torch.int32).view(sg.n_sinos, sg.n_proj, sg.n_r)
    for s in range(NSUB):
        st = P.count_steps(s, NSUB).view(sg.n_sinos, -1, sg.n_r).long()
        fwd.append(int(st.sum().item()))
        bwd.append(int(st[cv[:, s::NSUB, :] != 0].sum().item()))
    torch.cuda.synchronize(dev)
    log(f"setup {time.time() - t0:.1f} s: {nb} bins, counts {int(counts.view(torch.int32).sum().item())}, "
        f"fwd segments/subset {statistics.mean(fwd):.4g}, bwd {statistics.mean(bwd):.4g}")
    return dict(P=P, ig=ig, sg=sg, counts=counts, sens=sens, x=x, bp=bp, fwd=fwd, bwd=bwd, atten=atten)


def step_bytes(w, s, sparse=False):
    """Algorithmic HBM bytes of one sub-iteration: fp32 voxel read per forward
    segment, read-modify-write per backward segment, the uint32 count per bin
    (fused kernel), and 20 B per voxel for the update (x r/w, bp r, sens r, bp
    clear).  The sparse and nonzero passes walk forward only the bins with
    counts, whose segments are the backward ones, and read x and the
    per-subset image for the likelihood's dot product (8 B per voxel)."""
    nbins = w["sg"].n_sinos * w["sg"].subset_nproj(s, NSUB) * w["sg"].n_r
    fwd = w["bwd"][s] if sparse else w["fwd"][s]
    kern = 4 * fwd + 8 * w["bwd"][s] + 4 * nbins + (8 * w["ig"].n_voxels if sparse else 0)
    return kern, kern + 20 * w["ig"].n_voxels


def whole_job_value(steps, local_ms, world, dist=None, device=None):
    """Whole-job throughput of `world` replicas that each ran `steps` steps in
    `local_ms` of device time: steps * world / (max over ranks of the time).
    Every rank takes part in the same all-reduce."""
    total_ms = float(local_ms)
    if dist is not None and world > 1:
        import torch
        t = torch.tensor([total_ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    return steps * world / (total_ms / 1e3), total_ms


def run_sharded(args):
    """--shard: ONE reconstruction split over the ranks by LOR shards
    (apirl_b200.sharded): each sub-iteration is the fused pass over the rank's
    sinograms, an NCCL all-reduce of the backprojection image and of the
    likelihood, and the pixel update.  value = the job's sub-iterations over
    the slowest rank's time (strong scaling)."""
    import datetime
    import torch
    import torch.distributed as dist
    from apirl_b200.sharded import shard_ranges, ShardedOsem, GpuShard
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device(f"cuda:{local}")
    log = (lambda m: print(f"[bench] {m}", file=sys.stderr, flush=True)) if rank == 0 else (lambda m: None)
    import apirl_b200 as ap
    from apirl_b200 import _lib as _l
    ap.load_library()
    w = setup_workload(dev, log)
    ig, sg = w["ig"], w["sg"]
    first, n = shard_ranges(sg.n_sinos, world)[rank]
    nonzero = args.pass_form == "nonzero"
    backend = GpuShard(ig, sg, w["counts"], NSUB, first, n, device=local, mult=w["atten"], ge=UPDATE_GE,
                       geometry_sparse=nonzero)
    backend.P.set_option(_l.APIRL_OPT_KERNEL_TIMING, 1)
    job = ShardedOsem(backend, NSUB, dist if world > 1 else None)
    job.compute_sensitivity()
    if nonzero:
        for s_ in range(NSUB):
            backend.geometry_image(s_)  # the shard's G_s, at set-up like the sensitivity images
    # algorithmic bytes of the fused kernel on this rank's shard, per subset
    cv = w["counts"].view(torch.int32).view(sg.n_sinos, sg.n_proj, sg.n_r)[first:first + n]
    shard_bytes = []
    for s_ in range(NSUB):
        st = backend.P.count_steps(s_, NSUB).view(n, -1, sg.n_r).long()
        fwd, bwd = int(st.sum().item()), int(st[cv[:, s_::NSUB, :] != 0].sum().item())
        shard_bytes.append(4 * (bwd if nonzero else fwd) + 8 * bwd + 4 * st.numel()
                           + (8 * ig.n_voxels if nonzero else 0))
    x = torch.ones(ig.n_voxels, dtype=torch.float32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    for i in range(args.warmup):
        job.subiteration(x, i % NSUB)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
    kern = []
    for i in range(args.steps):
        flush.zero_()
        evs[i][0].record()
        job.subiteration(x, (args.warmup + i) % NSUB)
        evs[i][1].record()
        kern.append(backend.P.last_kernel_ms())
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clock = clocks.stop()
    local_ms = sum(e[0].elapsed_time(e[1]) for e in evs)
    t = torch.tensor([local_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    value = args.steps / (total_ms / 1e3)
    if rank == 0:
        peak, peak_kind = peaks()
        subs = [(args.warmup + i) % NSUB for i in range(args.steps)]
        achieved = statistics.mean(shard_bytes[s_] for s_ in subs) / (statistics.mean(kern) / 1e3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded phantom, Poisson counts)",
            "config": {"workload": WORKLOAD, "subsets": NSUB, "counts_dtype": "uint32",
                       "parallelism": f"LOR shards x{world} (sinograms {first}..{first + n - 1} on rank 0), "
                                      "NCCL all-reduce of the backprojection image and likelihood",
                       "l2": "flushed between timed steps (256 MB write outside the timed events)",
                       "pass": ("nonzero: each shard walks its bins with counts, its likelihood part from its "
                                "geometry images A_s^T 1 (set-up)") if nonzero else "full: every bin walked",
                       "update": "x*bp/sens where sens > 0"},
            "roofline": {"bound": "hbm", "kernel": "k_em_pass on rank 0's shard",
                         "kernel_ms": statistics.mean(kern), "peak": peak, "unit": "GB/s",
                         "peak_source": f"{peak_kind} hbm_gbs",
                         "achieved": achieved, "frac": achieved / peak, "traffic": None},
            "e2e": None, "cpu_baseline": None, "gpu_launches": (9 if nonzero else 5) * args.steps, "clocks": clock,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_gpu(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    log = (lambda m: print(f"[bench] {m}", file=sys.stderr, flush=True)) if rank == 0 else (lambda m: None)

    import apirl_b200 as ap
    ap.load_library()
    if args.alpha == "f64":
        args.pass_form = "full"  # the sparse pass takes the float walk
    w = setup_workload(dev, log, args.max_ring_diff, args.alpha)
    P, counts, sens, x, bp = w["P"], w["counts"], w["sens"], w["x"], w["bp"]
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    lik = torch.zeros(1, dtype=torch.float64, device=dev)

    from apirl_b200 import _lib as _l
    # autotuner: fused-kernel block size, timed on this job's own data (outside the timed region)
    if args.em_block:
        P.set_option(_l.APIRL_OPT_EM_BLOCK, args.em_block)
        best_block = args.em_block
    else:
        best_block = P.autotune(counts, x, 0, NSUB, repeats=2, stream=stream)
    bp.zero_()
    torch.cuda.synchronize(dev)
    log(f"autotuned fused-kernel block size: {best_block}")
    P.set_option(_l.APIRL_OPT_KERNEL_TIMING, 1)
    P.set_option(_l.APIRL_OPT_PERSISTENT, args.persistent)
    if args.l2_persist:
        P.set_option(_l.APIRL_OPT_L2_PERSIST, 1)
    if args.list_order:
        P.set_option(_l.APIRL_OPT_LIST_ORDER, args.list_order)
    if args.accumulate != "atomic":
        P.set_option(_l.APIRL_OPT_ACCUMULATE, {"warp": _l.APIRL_ACC_WARP,
                                               "compensated": _l.APIRL_ACC_COMPENSATED}[args.accumulate])

    sparse = args.pass_form == "sparse"
    nonzero = args.pass_form == "nonzero"
    skipz = sparse or nonzero  # zero-count bins not walked
    zimg = torch.zeros((NSUB, w["ig"].n_voxels), dtype=torch.float32, device=dev) if skipz else None
    if nonzero:
        # G_s = A_s^T 1 per subset: geometry alone (column sums of the subset's
        # system matrix), made once per scanner geometry at set-up like the
        # LOR tables and the sensitivity images.
        P.set_option(_l.APIRL_OPT_SPARSE_IMAGE, _l.APIRL_SPARSE_GEOMETRY)
        gev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        gev[0].record(stream)
        for s_ in range(NSUB):
            P.backproject_ones(zimg[s_], s_, NSUB, stream=stream)
        gev[1].record(stream)
        torch.cuda.synchronize(dev)
        geometry_ms = gev[0].elapsed_time(gev[1])
    # The listed pass's launch shape (block size and gather segments in
    # flight), tuned on this job's own data and geometry image, outside the
    # timed region (apirl_projector_autotune_ex).
    gather_unroll = None
    if (nonzero and not args.em_block and args.persistent and args.alpha == "f32" and args.accumulate == "atomic"
            and args.max_ring_diff is None):
        best_block, gather_unroll, tune_ms = P.autotune_shape(counts, x, zimg=zimg[0], subset=0, nsubsets=NSUB,
                                                              repeats=2, stream=stream)
        bp.zero_()
        torch.cuda.synchronize(dev)
        log(f"autotuned listed pass: {best_block} threads per block, {gather_unroll} segments in flight, "
            f"{tune_ms:.3f} ms")

    def zero_images():
        # Per-subset zero-count images of the sparse pass (once per
        # reconstruction, like the sensitivity images): Z_s = A_s^T 1[m == 0].
        zimg.zero_()
        for s in range(NSUB):
            P.zero_count_image(counts, zimg[s], s, NSUB, stream=stream)

    def step(s, evs=None):
        if evs:
            evs[0].record(stream)
        # one OSEM sub-iteration through the C ABI: layout copy, fused
        # projection / ratio / backprojection kernel, likelihood sum, update
        if skipz:
            P.em_pass_sparse(counts, x, bp, sens[s], zimg[s], s, NSUB, thr_value=0.0, ge=UPDATE_GE, lik=lik,
                             stream=stream)
        else:
            P.em_pass(counts, x, bp, sens[s], s, NSUB, thr_value=0.0, ge=UPDATE_GE, lik=lik, stream=stream)
        if evs:
            evs[1].record(stream)

    with torch.cuda.stream(stream):
        if sparse:
            zero_images()
        for i in range(args.warmup):
            step(i % NSUB)
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        clocks = ClockSampler(local)
        clocks.start()
        pre = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        if sparse:
            # the zero-count images are part of the timed job: computed again
            # here and amortized over the timed sub-iterations
            flush.zero_()
            pre[0].record(stream)
            zero_images()
            pre[1].record(stream)
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
        subs = [(args.warmup + i) % NSUB for i in range(args.steps)]
        kern_ms = []
        for i in range(args.steps):
            flush.zero_()                      # L2 flush between timed steps, outside the events
            step(subs[i], evs[i])
            kern_ms.append(P.last_kernel_ms())  # events the library records around the fused kernel
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        clock = clocks.stop()
        # The same sub-iterations walking every bin (the full pass), timed
        # the same way right after, reported beside the headline.
        full_cmp = None
        if nonzero:
            fev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
            fkern = []
            for i in range(args.steps):
                flush.zero_()
                fev[i][0].record(stream)
                P.em_pass(counts, x, bp, sens[subs[i]], subs[i], NSUB, thr_value=0.0, ge=UPDATE_GE, lik=lik,
                          stream=stream)
                fev[i][1].record(stream)
                fkern.append(P.last_kernel_ms())
            torch.cuda.synchronize(dev)
            if world > 1:
                dist.barrier()
            f_value, _ = whole_job_value(args.steps, sum(fev[i][0].elapsed_time(fev[i][1])
                                                         for i in range(args.steps)),
                                         world, dist if world > 1 else None, dev)
            fb = statistics.mean(step_bytes(w, s_, False)[0] for s_ in subs)
            f_ach = fb / (statistics.mean(fkern) / 1e3) / 1e9
            full_cmp = {"value": f_value, "unit": UNIT, "kernel_ms": statistics.mean(fkern),
                        "roofline_achieved": f_ach, "roofline_frac": f_ach / peaks()[0],
                        "traffic": FULL_TRAFFIC_BYTES if args.max_ring_diff is None else None,
                        "pass": "full: every bin walked, every estimate summed (--pass full)"}
    step_ms = [evs[i][0].elapsed_time(evs[i][1]) for i in range(args.steps)]
    pre_ms = pre[0].elapsed_time(pre[1]) if sparse else 0.0
    value, total_ms = whole_job_value(args.steps, sum(step_ms) + pre_ms, world, dist if world > 1 else None, dev)

    kb = [step_bytes(w, s, skipz) for s in subs]
    kern_bytes = statistics.mean(k for k, _ in kb)
    kern_s = statistics.mean(kern_ms) / 1e3
    peak, peak_kind = peaks()
    achieved = kern_bytes / kern_s / 1e9
    walked = sum((2 * w["bwd"][s]) if skipz else (w["fwd"][s] + w["bwd"][s]) for s in subs)
    if sparse:
        walked += sum(w["fwd"][s] - w["bwd"][s] for s in range(NSUB))  # the zero-count images' segments
    gsteps = walked / (total_ms / 1e3) / 1e9 * world

    # End-to-end through the C ABI with host buffers: the sub-iteration's packed
    # counts go host->device from pinned memory, the updated image and the
    # likelihood come back, every step.
    e2e = None
    if rank == 0 or world > 1:
        sg = w["sg"]
        import torch as _t
        cv = counts.view(_t.int32).view(sg.n_sinos, sg.n_proj, sg.n_r)
        host_counts = [cv[:, s::NSUB, :].contiguous().view(-1).cpu().pin_memory().numpy().view(np.uint32)
                       for s in range(NSUB)]
        stage = _t.empty(host_counts[0].size, dtype=_t.int32, device=dev)
        stages = [stage, _t.empty(host_counts[0].size, dtype=_t.int32, device=dev)]
        h_x_t = _t.empty(w["ig"].n_voxels, dtype=_t.float32).pin_memory()
        h_x = h_x_t.numpy()
        h_lik = np.zeros(1, np.float64)
        # one page-locked likelihood slot per timed step (filled asynchronously)
        h_liks = _t.zeros(max(args.steps, 1), dtype=_t.float64).pin_memory().numpy()
        ev = [_t.cuda.Event(enable_timing=True) for _ in range(2)]

        def e2e_zero_images():
            # the zero-count images from the host counts: each subset's counts
            # host->device, then its image (sparse pass only)
            zimg.zero_()
            for s in range(NSUB):
                stage.copy_(_t.from_numpy(host_counts[s].view(np.int32)), non_blocking=True)
                P.zero_count_image(stage.view(_t.uint32), zimg[s], s, NSUB, counts_packed=True, stream=stream)

        def e2e_step(s):
            # the sub-iteration's counts in, its likelihood out; the image
            # stays resident and comes back once, at the end of the job
            P.em_pass_host(host_counts[s], stage, x, bp, sens[s], s, NSUB, None, h_lik, ge=UPDATE_GE, stream=stream,
                           zimg=zimg[s] if skipz else None)

        with _t.cuda.stream(stream):
            if sparse:
                e2e_zero_images()
            for i in range(min(args.warmup, 3)):
                e2e_step(i % NSUB)
            torch.cuda.synchronize(dev)
            e_ms = 0.0
            if sparse:
                ev[0].record(stream)
                e2e_zero_images()
                ev[1].record(stream)
                ev[1].synchronize()
                e_ms += ev[0].elapsed_time(ev[1])
            # Each pass's counts go up on the library's copy stream while the
            # previous pass computes (apirl_stage_counts, two stages); each
            # pass's likelihood comes back into its own page-locked slot
            # without a host round trip between passes
            # (apirl_em_pass_host_async), all within the timed region.
            subs_e = [(args.warmup + i) % NSUB for i in range(args.steps)]
            h_liks[:] = np.nan
            ev[0].record(stream)
            P.stage_counts(host_counts[subs_e[0]], stages[0], subs_e[0], NSUB, stream=stream)
            for i, s in enumerate(subs_e):
                if i + 1 < args.steps:
                    P.stage_counts(host_counts[subs_e[i + 1]], stages[(i + 1) % 2], subs_e[i + 1], NSUB,
                                   stream=stream)
                P.em_pass_host(host_counts[s], stages[i % 2], x, bp, sens[s], s, NSUB, None, h_liks[i:i + 1],
                               ge=UPDATE_GE, stream=stream, zimg=zimg[s] if skipz else None, wait=False)
            h_x_t.copy_(x, non_blocking=True)  # the reconstructed image, once
            ev[1].record(stream)
            ev[1].synchronize()
            e_ms += ev[0].elapsed_time(ev[1])
            if not np.all(np.isfinite(h_liks[:args.steps])):
                raise RuntimeError("e2e: a pass's likelihood did not arrive")
        e_value, e_ms = whole_job_value(args.steps, e_ms, world, dist if world > 1 else None, dev)
        h2d = host_counts[0].nbytes + (sum(h.nbytes for h in host_counts) / args.steps if sparse else 0)
        e2e = {"value": e_value, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(8 + h_x.nbytes / args.steps),
               "api": "apirl_em_pass_host_async (C ABI): each sub-iteration's uint32 counts host->device from pinned "
                      "memory (apirl_stage_counts: the next pass's copy overlaps the current pass) and its FP64 "
                      "likelihood back; the image host<-device once at the end (counted per step above)"
                      + ("; the zero-count images from host counts inside the timed region" if sparse else "")}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(w, log, budget_s=args.cpu_seconds, threads=args.cpu_threads, first_subset=args.warmup)

    # The batched and served forms of the same path, on their mixed-job
    # workloads, beside the single-job headline (one GPU, rank 0).
    mixed = {}
    if rank == 0 and world == 1 and not args.no_mixed:
        del w, P, counts, sens, x, bp, flush
        torch.cuda.synchronize(dev)
        torch.cuda.empty_cache()
        for kind in ("batched", "served"):
            mixed[kind] = mixed_jobs(args, kind == "served", log)
            log(f"{kind}: {mixed[kind]['value']:.0f} recon/h, {mixed[kind]['speedup_vs_plain']:.2f}x the plain driver")

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded phantom, Poisson counts)",
            "config": {"workload": WORKLOAD if args.max_ring_diff is None else
                       WORKLOAD + f" (profiling case: segments |rd| <= {args.max_ring_diff} only)",
                       "subsets": NSUB, "counts_dtype": "uint32", "em_block": best_block,
                       "gather_unroll": gather_unroll if gather_unroll is not None else "default (6 listed, 4 full)",
                       "alpha": args.alpha, "persistent": args.persistent, "accumulate": args.accumulate,
                       "l2_persist": bool(args.l2_persist), "list_order": args.list_order,
                       "pass": ("sparse: bins with zero counts not walked, their likelihood terms -x.Z_s from "
                                "per-subset zero-count images Z_s = A_s^T 1[m=0], all 21 computed inside the "
                                "timed region and amortized over the timed sub-iterations") if sparse else
                               ("nonzero: bins with zero counts not walked; likelihood = sum over bins with counts "
                                "of m log e - x.G_s, G_s = A_s^T 1 per subset (geometry only: made once per "
                                "scanner geometry at set-up, like the LOR tables; the 21 images took "
                                f"{geometry_ms:.1f} ms)") if nonzero else
                               "full: every bin walked",
                       "l2": "flushed between timed steps (256 MB write outside the timed events)",
                       "update": "x*bp/sens where sens > 0 (the reference's >= 0 gives NaN at the 6 voxels "
                                 "no ray of subsets 3 and 16 crosses)",
                       "parallelism": f"replicas x{world}"},
            "siddon_gsteps_per_s": gsteps,
            "full_pass": full_cmp,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": args.traffic_bytes if args.traffic_bytes is not None else
                         ({"full": FULL_TRAFFIC_BYTES, "nonzero": NONZERO_TRAFFIC_BYTES}.get(args.pass_form)
                          if args.max_ring_diff is None else None),
                         "kernel": ("k_em_pass_persist" if args.persistent and args.alpha == "f32" else "k_em_pass")
                                   + " (fused projection / ratio / backprojection)",
                         "timing": "CUDA events recorded by the library on the launching stream around the fused "
                                   "kernel and its two small likelihood-sum kernels",
                         "algorithmic_bytes_per_launch": kern_bytes, "kernel_ms": kern_s * 1e3,
                         "peak_source": f"{peak_kind} hbm_gbs"},
            "e2e": e2e,
            "cpu_baseline": cpu,
            # per step: layout copy, fused kernel, (zero-count dot,) two-level
            # likelihood sum, reduce/update; plus one zero-count kernel per subset
            # per pass: layout copy, [list: tiles, scan, write], fused kernel,
            # [dot product], two-level sum, update
            "gpu_launches": (9 * args.steps + NSUB) if sparse else (9 * args.steps if nonzero else 5 * args.steps),
            "clocks": clock,
        }
        if mixed:
            line["batched"] = mixed["batched"]
            line["served"] = mixed["served"]
            line["served_p50_s"] = mixed["served"]["p50_latency_s"]
            line["served_p99_s"] = mixed["served"]["p99_latency_s"]
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# CPU side: the reference APIRL code on whole sub-iterations of the same job.
class CpuSubiterations:
    """Whole OSEM sub-iterations of the full workload (all 1261 sinograms) on
    the host cores: the reference code compiled from its sources
    (oracle/_ref: getSubset, Project, getLikelihoodValue, inverseDivideBinToBin,
    Backproject, then the pixel update of OsemSinogram3d.cpp:217-237 with the
    bench's rule, update where sens > 0), or the oracle restatement where the
    reference was not built.  Subsets and sensitivity images are those the GPU
    arm uses."""

    def __init__(self, counts_full, log, threads=None):
        """counts_full: the whole sinogram's counts (any integer or float array)."""
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle_lib import RefHarness, Oracle, REF_SO
        from apirl_b200 import workloads
        self.ig, self.sg = workloads.c2_geometry()
        counts = np.ascontiguousarray(counts_full, np.float32)
        self.cores = threads or os.cpu_count() or 1
        if os.path.exists(REF_SO):
            self.kind = "reference"
            self.R = RefHarness()
            self.R.set_threads(self.cores)
            t0 = time.perf_counter()
            self.h = self.R.sino3d(self.sg, counts)
            log(f"reference sinogram loaded ({counts.size} bins) in {time.perf_counter() - t0:.1f} s")
        else:
            self.kind = "port"
            self.R = None
            self.oracle = Oracle()
            self.counts = counts
        self.x = np.ones(self.ig.n_voxels, np.float32)

    def set_threads(self, n):
        self.cores = n
        if self.R is not None:
            self.R.set_threads(n)

    def run(self, subset, sens):
        """One whole sub-iteration of `subset`, in place on self.x; seconds."""
        sens = np.ascontiguousarray(sens, np.float32)
        t0 = time.perf_counter()
        if self.R is not None:
            self.R.osem_subiteration(self.h, self.ig, subset, NSUB, self.x, sens, ge=UPDATE_GE)
        else:
            o, sg, ig = self.oracle, self.sg, self.ig
            est = o.project_3d(sg, ig, self.x, subset, NSUB, threads=self.cores)
            m = self.counts.reshape(sg.n_sinos, sg.n_proj, sg.n_r)[:, subset::NSUB, :].reshape(-1)
            ratio = o.inverse_divide(m, est)
            bp = o.backproject_3d(sg, ig, ratio, subset, NSUB, threads=self.cores)
            self.x = o.update(self.x, bp, sens, np.float32(0), UPDATE_GE)
        return time.perf_counter() - t0

    def describe(self, subsets):
        src = ("the reference APIRL CPU code compiled from its sources (oracle/_ref)" if self.kind == "reference"
               else "the oracle restatement of the reference (oracle/)")
        return (f"whole OSEM sub-iterations of the full workload (all 1261 sinograms), subsets {subsets}, through "
                f"{src}: getSubset, Project, likelihood, ratio, Backproject, pixel update; wall time per "
                "sub-iteration")


def cpu_baseline(w, log, budget_s=15.0, threads=None, first_subset=0):
    """The reference CPU code on whole sub-iterations of the GPU arm's job (its
    counts and sensitivity images), subsets in the GPU arm's order, until
    `budget_s` of CPU time (at least one sub-iteration)."""
    import torch
    counts_full = w["counts"].view(torch.int32).cpu().numpy().view(np.uint32)
    cs = CpuSubiterations(counts_full, log, threads)
    del counts_full
    times, subs = [], []
    while not times or (sum(times) < budget_s and len(times) < NSUB):
        s = (first_subset + len(times)) % NSUB
        times.append(cs.run(s, w["sens"][s].cpu().numpy()))
        subs.append(s)
    total = sum(times)
    return {"value": len(times) / total, "unit": UNIT, "cores": cs.cores, "kind": cs.kind,
            "sample": cs.describe(subs) + f"; {len(times)} sub-iterations in {total:.2f} s"}


def _reference_job(log, o, needed_subsets):
    """The job's counts and the needed subsets' sensitivity images, made on
    the host exactly as the GPU arm makes them: the oracle's projection of the
    phantom (bit-identical to the GPU's), the same attenuation factors, the
    same per-sinogram Poisson seeds; sensitivity = A_s^T a then forcePositive."""
    from apirl_b200 import workloads
    ig, sg = workloads.c2_geometry()
    t0 = time.perf_counter()
    proj = o.project_3d(sg, ig, workloads.cylinder_phantom_3d(ig, seed=2))
    lor = o.lor_points_2d(sg.n_proj, sg.n_r, sg.r_fov, sg.r_scanner)
    z1, z2 = o.sino3d_z(sg)
    atten = np.exp(-workloads.MU_WATER_PER_MM *
                   workloads.cylinder_chords(lor, np.stack([z1, z2], 1).astype(np.float32))).astype(np.float32)
    atten = atten.reshape(-1)
    proj *= atten
    counts = workloads.c2_counts(proj, range(sg.n_sinos), sg.n_proj * sg.n_r)
    del proj
    sens = {}
    for s in sorted(set(needed_subsets)):
        a_s = np.ascontiguousarray(atten.reshape(sg.n_sinos, sg.n_proj, sg.n_r)[:, s::NSUB, :]).reshape(-1)
        sens[s] = np.maximum(o.backproject_3d(sg, ig, a_s, s, NSUB), np.float32(0))
    log(f"job made on the host in {time.perf_counter() - t0:.1f} s: {int(counts.sum())} counts, "
        f"{len(sens)} sensitivity images")
    return counts, sens


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    log = lambda m: print(f"[bench-ref] {m}", file=sys.stderr, flush=True)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Oracle
    o = Oracle()
    warm = [i % NSUB for i in range(args.warmup)]
    timed = [(args.warmup + i) % NSUB for i in range(args.steps)]
    one_thread_subset = (args.warmup + args.steps) % NSUB
    counts, sens = _reference_job(log, o, warm + timed + [one_thread_subset])
    cs = CpuSubiterations(counts, log, args.cpu_threads)
    del counts
    for s in warm:
        cs.run(s, sens[s])
    times = [cs.run(s, sens[s]) for s in timed]
    total = sum(times)
    value = args.steps / total
    log(f"{args.steps} sub-iterations on {cs.cores} threads: {total:.2f} s")
    one = None
    if not args.no_one_thread:
        threads = cs.cores
        cs.set_threads(1)
        t1 = cs.run(one_thread_subset, sens[one_thread_subset])
        cs.set_threads(threads)
        one = {"value": 1.0 / t1, "unit": UNIT, "cores": 1, "sample": f"one whole sub-iteration (subset "
               f"{one_thread_subset}) on 1 host thread, {t1:.2f} s"}
        log(f"1 thread: {t1:.2f} s")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded phantom, Poisson counts)",
        "config": {"workload": WORKLOAD, "subsets": NSUB, "update": "x * bp / sens where sens > 0, else 0",
                   "parallelism": f"{cs.cores} host threads (OpenMP)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cs.cores, "kind": cs.kind,
                         "sample": cs.describe(timed) + f"; {args.steps} sub-iterations in {total:.2f} s"},
        "one_thread": one,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Batched and served forms (not the headline): many OSEM jobs of mixed size.
def _make_jobs(specs, dev, log, c2_every=0):
    import torch
    import apirl_b200 as ap
    from apirl_b200 import workloads
    from apirl_b200.batch import Job
    jobs = []
    for i, s in enumerate(specs):
        if c2_every and i % c2_every == c2_every - 1:
            ig, sg = workloads.c2_geometry()
            x = workloads.cylinder_phantom_3d(ig, seed=2)
        else:
            ig, sg = workloads.job_geometry(s["n"], s["z"])
            x = workloads.random_phantom(ig, np.random.default_rng(s["seed"]))
        P = ap.SiddonProjector(ig, sg, device=dev.index)
        est = torch.empty(P.num_bins(), dtype=torch.float32, device=dev)
        P.project(torch.from_numpy(x).to(dev), est)
        est.mul_(s["counts"] / float(est.double().sum().item()))
        g = torch.Generator(device=dev).manual_seed(s["seed"])
        counts = torch.poisson(est, generator=g).to(torch.int32).cpu().numpy().view(np.uint32)
        P.close()
        jobs.append(Job(ig, sg, counts, s["iters"], s["nsubsets"], tag=dict(s, geometry=(ig.nx, ig.nz, sg.n_sinos)),
                        update_positive_sens=True))
    torch.cuda.synchronize(dev)
    log(f"made {len(jobs)} jobs, {sum(j.counts.size for j in jobs) / 1e6:.0f} M bins")
    return jobs


def _plain(jobs, dev):
    """The same jobs one after another through the plain driver (apirl_osem_3d,
    float32 counts: converted before the clock starts).  Returns the images,
    the total time and each job's own time."""
    import apirl_b200 as ap
    counts = [j.counts.astype(np.float32) for j in jobs]
    init = [np.ones(j.image_geom.n_voxels, np.float32) for j in jobs]
    t0 = time.perf_counter()
    outs, each = [], []
    for j, c, x0 in zip(jobs, counts, init):
        ts = time.perf_counter()
        img, lik, _ = ap.osem_3d(j.image_geom, j.sino_geom, c, x0, j.iters, j.nsubsets, device=dev.index,
                                 update_positive_sens=j.update_positive_sens)
        each.append(time.perf_counter() - ts)
        outs.append(img)
    return outs, time.perf_counter() - t0, np.array(each)


def _fifo(arrivals, service):
    """Latencies and finish times of one server taking jobs in arrival order,
    each for its measured service time: the plain driver serving the stream."""
    order = np.argsort(arrivals)
    finish = np.zeros(len(arrivals))
    t = -np.inf
    for k in order:
        t = max(t, arrivals[k]) + service[k]
        finish[k] = t
    return finish - arrivals, finish


def mixed_jobs(args, served, log):
    """Batched (all jobs at once) or served (Poisson arrivals) OSEM jobs of
    mixed geometry against the same jobs through the plain driver, one at a
    time.  Returns the JSON fields of the comparison."""
    import torch
    from apirl_b200 import workloads
    from apirl_b200.batch import Batch, serve
    dev = torch.device("cuda:0")
    n = args.jobs
    specs = workloads.mixed_job_specs(n, seed=5 if served else 4)
    jobs = _make_jobs(specs, dev, log, c2_every=10 if served else 0)
    torch.cuda.empty_cache()
    budget = int(args.budget_gb * (1 << 30))
    if args.no_plain:  # (profiler captures of the batched form alone)
        ref, t_plain, each = None, float("nan"), np.full(len(jobs), np.nan)
    else:
        ref, t_plain, each = _plain(jobs, dev)
    if served:
        arrivals = np.cumsum(np.random.default_rng(5).exponential(1.0 / args.rate, len(jobs)))
        res, lat, makespan = serve(jobs, arrivals, budget_bytes=budget)
        t_new = makespan - float(arrivals[0])
        plain_lat, plain_finish = _fifo(arrivals, each)
        plain_stream = float(plain_finish.max() - arrivals.min())
    else:
        b = Batch(0, budget_bytes=budget)
        t0 = time.perf_counter()
        res = b.run_all(jobs)
        t_new = time.perf_counter() - t0
        b.close()
    errs = []
    for r, p in zip(res, ref if ref is not None else []):
        fin = np.isfinite(p)
        if not np.array_equal(np.isfinite(r[0]), fin):
            raise RuntimeError("a batched job's image is not finite where its solo run's is")
        d = float(np.linalg.norm(r[0][fin].astype(np.float64) - p[fin]))
        n = float(np.linalg.norm(p[fin].astype(np.float64)))
        errs.append(d / n if n > 0 else d)
    out = {
        "value": len(jobs) / t_new * 3600, "unit": "recon/h",
        "plain_value": len(jobs) / t_plain * 3600, "speedup_vs_plain": t_plain / t_new,
        "max_rel_l2_vs_plain": max(errs) if errs else None,
        "nonfinite_images": int(sum(not np.isfinite(r[0]).all() for r in res)),
        "workload": ("Poisson arrivals at %.0f jobs/s of " % args.rate if served else "all at once: ") +
                    f"{len(jobs)} mixed OSEM jobs: images {{64,128,256}}^2 x {{1,41,81}} slices, 1.3N r/angles, "
                    "span 1, 2-4 iterations x 7-21 subsets, 1e5-1e8 counts uint32" +
                    ("; every 10th job the full 256x256x81 / 1261x336x336 geometry" if served else "") +
                    "; update where sens > 0 in both arms (the reference's sens >= 0 turns 12 of these 64 "
                    "reconstructions entirely NaN: subsets of a few angles leave voxels no ray crosses)",
        "plain": "the same jobs one after another through apirl_osem_3d (float32 counts made before the clock)",
        "budget_gb": args.budget_gb,
    }
    if served:
        out.update({"p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
                    "makespan_s": float(t_new),
                    "plain_p50_latency_s": float(np.percentile(plain_lat, 50)),
                    "plain_p99_latency_s": float(np.percentile(plain_lat, 99)),
                    "plain_stream_value": len(jobs) / plain_stream * 3600,
                    "speedup_vs_plain_stream": plain_stream / t_new,
                    "plain_stream": "the plain driver serving the same arrivals in order, one job at a time "
                                    "(each job's measured time; latency = finish - arrival)",
                    "arrival_span_s": float(arrivals.max() - arrivals.min())})
    return out


def run_mlem2d(args):
    """--workload mlem2d: the 2D configuration (128x128 image, 192x192
    sinogram, disc phantom with 6 hot points, 1e6 counts, 60 MLEM iterations)
    through the whole-reconstruction driver (host buffers in and out, one CUDA
    graph per iteration), against the reference's Mlem2d on the host cores."""
    import torch
    import apirl_b200 as ap
    from apirl_b200 import workloads
    ap.load_library()
    ig, sg = workloads.c1_geometry()
    x = workloads.disc_phantom_2d(ig, seed=0)
    P = ap.SiddonProjector(ig, sg)
    est = torch.zeros(sg.n_bins, dtype=torch.float32, device="cuda:0")
    P.project(torch.from_numpy(x).cuda(), est)
    meas = workloads.poisson_counts(est.cpu().numpy(), 1e6, seed=0).astype(np.float32)
    init = np.ones(ig.n_voxels, np.float32)
    iters = 60
    for _ in range(max(args.warmup, 1)):
        ap.mlem_2d(ig, sg, meas, init, iters)
    times = []
    for _ in range(max(args.steps, 1)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ap.mlem_2d(ig, sg, meas, init, iters)
        times.append(time.perf_counter() - t0)
    gpu = iters / statistics.median(times)
    cpu = None
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import RefHarness, REF_SO
    if os.path.exists(REF_SO) and not args.no_cpu_baseline:
        R = RefHarness()
        cores = R.set_threads(args.cpu_threads or os.cpu_count() or 1)
        # the reference prints its progress on stdout: send it to stderr, so
        # that stdout carries only the JSON line
        sys.stdout.flush()
        saved = os.dup(1)
        os.dup2(2, 1)
        try:
            t0 = time.perf_counter()
            R.mlem_2d(sg, ig, init, meas, iters)
            sec = time.perf_counter() - t0
        finally:
            os.dup2(saved, 1)
            os.close(saved)
        cpu = {"value": iters / sec, "unit": "iter/s", "cores": cores, "kind": "reference",
               "sample": "the whole 60-iteration Mlem2d reconstruction"}
    print(json.dumps({"metric": "2D MLEM iterations/s (128x128, 192x192 sinogram)", "value": gpu, "unit": "iter/s",
                      "n_gpus": 1, "higher_is_better": True, "ms_per_reconstruction": 1e3 * statistics.median(times),
                      "dtype": "f32", "data": "synthetic (disc phantom, 1e6 Poisson counts)",
                      "config": {"workload": "2D MLEM 60 iterations, whole driver with host buffers (e2e)"},
                      "cpu_baseline": cpu}), flush=True)


def run_batched_c2(args):
    """--workload batched-c2: the 3D OSEM job of the default line (or its
    --max-ring-diff profiling case), 1 iteration x 21 subsets, as the only job
    of a batch, for comparing the batched walk with the single-job kernel on
    the same counts (profiler captures).  Prints the batch's wall time."""
    import torch
    import apirl_b200 as ap
    from apirl_b200 import workloads
    from apirl_b200.batch import Batch, Job
    from apirl_b200.geometry import Sino3DGeom
    dev = torch.device("cuda:0")
    ap.load_library()
    ig, sg = workloads.c2_geometry()
    if args.max_ring_diff is not None and args.max_ring_diff < 20:
        sg = Sino3DGeom.span1(sg.n_proj, sg.n_r, sg.n_rings, sg.r_fov, sg.axial_fov, sg.r_scanner, args.max_ring_diff)
    P = ap.SiddonProjector(ig, sg, device=dev.index)
    _, counts = workloads.c2_device_arrays(P, dev)
    h = counts.view(torch.int32).cpu().numpy().view(np.uint32)
    P.close()
    del counts
    torch.cuda.synchronize(dev)
    b = Batch(0, budget_bytes=int(args.budget_gb * (1 << 30)))
    t0 = time.perf_counter()
    b.run_all([Job(ig, sg, h, 1, NSUB, update_positive_sens=True)])
    sec = time.perf_counter() - t0
    b.close()
    print(json.dumps({"metric": "batch of one 3D OSEM job (1 iteration x 21 subsets)", "value": sec, "unit": "s",
                      "n_gpus": 1, "higher_is_better": False,
                      "config": {"workload": WORKLOAD if args.max_ring_diff is None else
                                 WORKLOAD + f" (profiling case: segments |rd| <= {args.max_ring_diff} only)"}}),
          flush=True)


def run_batched(args, served=False):
    log = lambda m: print(f"[bench] {m}", file=sys.stderr, flush=True)
    r = mixed_jobs(args, served, log)
    line = {"metric": "served OSEM reconstructions/hour" if served else "batched OSEM reconstructions/hour",
            "value": r.pop("value"), "unit": r.pop("unit"), "n_gpus": 1, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic (seeded phantoms, Poisson counts)",
            "config": {"workload": r.pop("workload"), "budget_gb": r.pop("budget_gb")}}
    line.update(r)
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Precision study: the full workload's first sub-iterations in several
# arithmetic forms against the FP64 oracle.
def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    m = np.isfinite(a) & np.isfinite(b)
    return float(np.linalg.norm(a[m] - b[m]) / max(np.linalg.norm(b[m]), 1e-300))


def _max_abs(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    m = np.isfinite(a) & np.isfinite(b)
    return float(np.max(np.abs(a[m] - b[m])))


def precision_study(subiters, log, threads=None):
    """The first `subiters` OSEM sub-iterations of the 3D workload (from an
    image of ones) in several GPU forms and in the FP64 oracle (double LOR
    geometry, double walk, double accumulation).  Returns a dict: per
    sub-iteration the relative L2 and max-abs error of each form's image
    against the FP64 image and the relative error of its FP64 likelihood;
    one ratio sinogram's backprojection in each accumulation form (and the
    reference's serial float order) against its FP64 backprojection; the
    adjoint residual of the GPU operators.  Forms:
      f32          the reference's float arithmetic, fp32 atomics (uint32 counts)
      f32_warp     the same, warp-aggregated atomics (APIRL_ACC_WARP)
      f32_comp     the same, compensated atomics (APIRL_ACC_COMPENSATED)
      u16          uint16 counts (round trip checked bit for bit first)
      f64alpha     FP64 walk geometry, fp32 projection and accumulation"""
    import torch
    import apirl_b200 as ap
    from apirl_b200 import _lib as _l
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Oracle
    dev = torch.device("cuda:0")
    w = setup_workload(dev, log)
    P, ig, sg = w["P"], w["ig"], w["sg"]
    nv = ig.n_voxels
    orc = Oracle()
    thr = threads or os.cpu_count() or 1
    counts32 = w["counts"]
    counts_np = counts32.view(torch.int32).cpu().numpy().astype(np.int64)
    if counts_np.max() >= 65536:
        raise RuntimeError("counts do not fit uint16")
    counts16 = torch.from_numpy(counts_np.astype(np.uint16)).to(dev)
    u16_round_trip = bool(np.array_equal(counts16.cpu().numpy().astype(np.int64), counts_np))
    meas64 = counts_np.astype(np.float64).reshape(sg.n_sinos, sg.n_proj, sg.n_r)
    atten64 = w["atten"].cpu().numpy().astype(np.float64).reshape(sg.n_sinos, sg.n_proj, sg.n_r)

    def projector(acc=None, f64=False):
        Q = ap.SiddonProjector(ig, sg)
        if f64:
            Q.set_alpha_precision(True)
        if acc is not None:
            Q.set_option(_l.APIRL_OPT_ACCUMULATE, acc)
        return Q

    P64 = projector(f64=True)
    Pw = projector(_l.APIRL_ACC_WARP)
    Pc = projector(_l.APIRL_ACC_COMPENSATED)
    sens64 = torch.zeros((NSUB, nv), dtype=torch.float32, device=dev)
    for s in range(subiters):
        a_s = w["atten"].view(sg.n_sinos, sg.n_proj, sg.n_r)[:, s::NSUB, :].contiguous().view(-1)
        P64.backproject(a_s, sens64[s], s, NSUB)
        ap.force_positive(sens64[s])
    forms = {"f32": dict(P=P, counts=counts32, sens=w["sens"]),
             "f32_warp": dict(P=Pw, counts=counts32, sens=w["sens"]),
             "f32_comp": dict(P=Pc, counts=counts32, sens=w["sens"]),
             "u16": dict(P=P, counts=counts16, sens=w["sens"]),
             "f64alpha": dict(P=P64, counts=counts32, sens=sens64)}
    for f in forms.values():
        f["x"] = torch.ones(nv, dtype=torch.float32, device=dev)
        f["bp"] = torch.zeros(nv, dtype=torch.float32, device=dev)
        f["lik"] = torch.zeros(1, dtype=torch.float64, device=dev)
    x64 = np.ones(nv, np.float64)
    rows = []
    for s in range(subiters):
        t0 = time.time()
        # FP64 oracle sub-iteration (OsemSinogram3d.cpp:159-237 in double), update where sens > 0.
        a_s = np.ascontiguousarray(atten64[:, s::NSUB, :]).reshape(-1)
        sens_s = orc.backproject_3d(sg, ig, a_s, s, NSUB, dtype=np.float64, threads=thr)
        est = orc.project_3d(sg, ig, x64, s, NSUB, dtype=np.float64, threads=thr)
        m_s = np.ascontiguousarray(meas64[:, s::NSUB, :]).reshape(-1)
        nz = est != 0
        lik64 = float(np.sum(m_s[nz] * np.log(est[nz]) - est[nz]))
        ratio = np.where((m_s != 0) & nz, m_s / np.where(nz, est, 1.0), 0.0)
        bp64 = orc.backproject_3d(sg, ig, ratio, s, NSUB, dtype=np.float64, threads=thr)
        with np.errstate(invalid="ignore", divide="ignore"):
            x64 = np.where(sens_s > 0, x64 * bp64 / np.where(sens_s > 0, sens_s, 1.0), 0.0)
        row = {"subiteration": s, "oracle_s": round(time.time() - t0, 1)}
        for name, f in forms.items():
            f["P"].em_pass(f["counts"], f["x"], f["bp"], f["sens"][s], s, NSUB, ge=UPDATE_GE, lik=f["lik"])
            torch.cuda.synchronize(dev)
            xg = f["x"].cpu().numpy()
            row[name] = {"rel_l2": _rel(xg, x64), "max_abs": _max_abs(xg, x64),
                         "lik_rel": abs(f["lik"].item() - lik64) / abs(lik64)}
        # same arithmetic; only the atomics' order differs between the two runs
        row["u16_vs_f32_rel_l2"] = _rel(forms["u16"]["x"].cpu().numpy(), forms["f32"]["x"].cpu().numpy())
        log(json.dumps(row))
        rows.append(row)

    # One ratio sinogram of subset 0, backprojected in each accumulation form,
    # against the exact (FP64) sum of the float contributions the float walk
    # makes, so that only the accumulation's rounding is measured (against the
    # FP64 walk, the geometry's 1e-2 would hide it).
    s = 0
    x1 = forms["f32"]["x"].cpu().numpy()
    est32 = orc.project_3d(sg, ig, x1, s, NSUB, threads=thr)
    m32 = np.ascontiguousarray(meas64[:, s::NSUB, :]).reshape(-1).astype(np.float32)
    ratio32 = orc.inverse_divide(m32, est32)
    bp_exact = orc.backproject_3d_exact_sum(sg, ig, ratio32, s, NSUB, threads=thr)
    bp_fp64walk = orc.backproject_3d(sg, ig, ratio32.astype(np.float64), s, NSUB, dtype=np.float64, threads=thr)
    acc = {"reference_serial_fp32_rel_l2": _rel(orc.backproject_3d(sg, ig, ratio32, s, NSUB, threads=1), bp_exact),
           "fp64_walk_vs_float_walk_rel_l2": _rel(bp_fp64walk, bp_exact),
           "against": "the FP64 sum of the float walk's own contributions"}
    r_dev = torch.from_numpy(ratio32).to(dev)
    for name, Q in (("atomic", P), ("warp", Pw), ("compensated", Pc)):
        bpg = torch.zeros(nv, dtype=torch.float32, device=dev)
        Q.backproject(r_dev, bpg, s, NSUB)
        torch.cuda.synchronize(dev)
        acc[f"gpu_{name}_rel_l2"] = _rel(bpg.cpu().numpy(), bp_exact)
        acc[f"gpu_{name}_max_abs"] = _max_abs(bpg.cpu().numpy(), bp_exact)

    # Adjoint residual of the GPU operators (FP64 dot products).
    rng = np.random.default_rng(0)
    xa = rng.random(nv, dtype=np.float32)
    ya = rng.random(sg.subset_bins(s, NSUB), dtype=np.float32)
    adj = {}
    for name, Q in (("f32", P), ("f64alpha", P64), ("f32_comp", Pc)):
        Ax = torch.zeros(ya.size, dtype=torch.float32, device=dev)
        Q.project(torch.from_numpy(xa).to(dev), Ax, s, NSUB)
        Aty = torch.zeros(nv, dtype=torch.float32, device=dev)
        Q.backproject(torch.from_numpy(ya).to(dev), Aty, s, NSUB)
        lhs = float(np.dot(Ax.cpu().numpy().astype(np.float64), ya.astype(np.float64)))
        rhs = float(np.dot(xa.astype(np.float64), Aty.cpu().numpy().astype(np.float64)))
        adj[name] = abs(lhs - rhs) / abs(lhs)
    for Q in (P64, Pw, Pc):
        Q.close()
    return {"subiterations": rows, "u16_round_trip": u16_round_trip, "backprojection_accumulation": acc,
            "adjoint_residual": adj, "oracle_threads": thr}


def run_precision(args):
    log = lambda m: print(f"[precision] {m}", file=sys.stderr, flush=True)
    r = precision_study(args.precision_subiters, log, args.cpu_threads)
    first = r["subiterations"][0]
    print(json.dumps({"metric": "rel L2 vs FP64 oracle after the first sub-iteration (f32, reference arithmetic)",
                      "value": first["f32"]["rel_l2"], "unit": "relative L2", "higher_is_better": False,
                      "n_gpus": 1, "dtype": "f32", "data": "synthetic (seeded phantom, Poisson counts)",
                      "config": {"workload": WORKLOAD, "subiterations": args.precision_subiters,
                                 "update": "x*bp/sens where sens > 0"},
                      **r}), flush=True)


def main():
    ap_ = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap_.add_argument("--gpus", type=int, default=1)
    ap_.add_argument("--steps", type=int, default=63,
                     help="timed sub-iterations (63: the job's 3 iterations x 21 subsets)")
    ap_.add_argument("--warmup", type=int, default=5)
    ap_.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap_.add_argument("--no-cpu-baseline", action="store_true")
    ap_.add_argument("--no-mixed", action="store_true",
                     help="default workload: skip the batched and served mixed-job runs after the headline")
    ap_.add_argument("--cpu-seconds", type=float, default=15.0)
    ap_.add_argument("--pass", dest="pass_form", default="nonzero", choices=["sparse", "nonzero", "full"],
                     help="nonzero: bins with zero counts are not walked, the likelihood from per-subset geometry "
                          "images A_s^T 1 made at set-up; sparse: the same walk, the likelihood from per-subset "
                          "zero-count images computed inside the timed region; full: every bin walked")
    ap_.add_argument("--em-block", type=int, default=0,
                     help="threads per block of the fused kernel (0: autotuned on the job's own data)")
    ap_.add_argument("--persistent", type=int, default=1, choices=[0, 1],
                     help="1: the fused pass as a persistent kernel whose warps pull 32-bin chunks")
    ap_.add_argument("--shard", action="store_true",
                     help="one job split over the ranks by LOR shards (strong scaling) instead of replicas")
    ap_.add_argument("--alpha", default="f32", choices=["f32", "f64"],
                     help="walk geometry: f32 = the reference's float arithmetic (headline); f64 = precision mode")
    ap_.add_argument("--no-one-thread", action="store_true",
                     help="reference arm: skip the extra one-thread sub-iteration")
    ap_.add_argument("--l2-persist", action="store_true",
                     help="L2 persisting window over the padded images (APIRL_OPT_L2_PERSIST)")
    ap_.add_argument("--list-order", type=int, default=0,
                     help="sparse passes: list entries by walk length within groups of this size (0: bin order)")
    ap_.add_argument("--accumulate", default="atomic", choices=["atomic", "warp", "compensated"],
                     help="how the backprojection scatter accumulates (APIRL_OPT_ACCUMULATE)")
    ap_.add_argument("--cpu-threads", type=int, default=None,
                     help="host threads of the CPU baseline / reference arm (default: all)")
    ap_.add_argument("--workload", default="osem3d",
                     choices=["osem3d", "batched", "served", "mlem2d", "precision", "batched-c2"])
    ap_.add_argument("--precision-subiters", type=int, default=4,
                     help="precision workload: sub-iterations compared with the FP64 oracle")
    ap_.add_argument("--max-ring-diff", type=int, default=None,
                     help="profiling: keep segments |rd| <= this (smaller case of the same kernels)")
    ap_.add_argument("--jobs", type=int, default=64)
    ap_.add_argument("--no-plain", action="store_true",
                     help="batched / served workloads: skip the plain-driver comparison (profiler captures)")
    ap_.add_argument("--rate", type=float, default=20.0, help="served: mean arrivals per second")
    ap_.add_argument("--budget-gb", type=float, default=96.0)
    ap_.add_argument("--traffic-bytes", type=float, default=None,
                     help="DRAM bytes per fused-kernel launch from an ncu capture, reported as roofline.traffic "
                          f"(default for the full workload: {FULL_TRAFFIC_BYTES:.3g})")
    args = ap_.parse_args()
    if args.warmup < 3 and args.impl != "reference":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.shard:
        run_sharded(args)
    elif args.workload == "mlem2d":
        run_mlem2d(args)
    elif args.workload == "precision":
        run_precision(args)
    elif args.workload in ("batched", "served"):
        run_batched(args, served=args.workload == "served")
    elif args.workload == "batched-c2":
        run_batched_c2(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
