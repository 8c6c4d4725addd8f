"""One OSEM reconstruction split over several GPUs by LOR shards.

Each rank (one process per GPU, torch.distributed over NCCL) owns a
contiguous range of sinograms.  A sub-iteration is

  1. the fused projection / ratio / backprojection over the rank's bins
     (apirl_em_project_backproject on a projector restricted to the shard,
     apirl_projector_set_shard), giving a partial backprojection image and a
     partial FP64 likelihood;
  2. one all-reduce (sum) of the backprojection image and of the likelihood;
  3. the same pixel update on every rank (threshold 0, >=; OsemSinogram3d.cpp:217-237).

The per-subset sensitivity images are the all-reduced sums of the shards'
backprojections of the multiplicative term (or ones), with forcePositive
applied afterwards (OsemSinogram3d.cpp:101-116).  Every rank takes the same
collective steps in the same order.  The reference runs OSEM on one device
only; this is the scale-out of the same algorithm, its results equal to the
single-device ones up to the order of fp32 additions.

The per-rank work goes through a backend object, so that the collective
logic is the same for the GPU backend (`GpuShard`) and for stand-ins.
"""
from .geometry import subset_nproj


def shard_ranges(n_sinos, world):
    """Contiguous sinogram ranges (first, count) of `world` ranks; the counts
    differ by at most one."""
    if world < 1 or n_sinos < world:
        raise ValueError(f"cannot split {n_sinos} sinograms over {world} ranks")
    base, extra = divmod(n_sinos, world)
    out, first = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((first, n))
        first += n
    return out


class ShardedOsem:
    """OSEM over LOR shards.  backend provides, for its own shard:
    zeros_image(), scalar(), sensitivity(s, out) (out += A_s^T (mult or 1)),
    em_pass(x, bp, s, lik) (bp += A_s^T ratio, lik[0] = shard likelihood),
    force_positive(img), update(x, bp, sens) (x *= bp / sens, bp cleared)."""

    def __init__(self, backend, nsubsets, dist=None):
        self.b = backend
        self.nsub = nsubsets
        self.dist = dist if (dist is not None and dist.is_initialized() and dist.get_world_size() > 1) else None
        self.sens = []
        self.bp = backend.zeros_image()
        self.lik = backend.scalar()

    def _sum(self, t):
        if self.dist is not None:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)

    def compute_sensitivity(self):
        self.sens = []
        for s in range(self.nsub):
            img = self.b.zeros_image()
            self.b.sensitivity(s, img)
            self._sum(img)
            self.b.force_positive(img)
            self.sens.append(img)

    def subiteration(self, x, s):
        """One sub-iteration on every rank; returns the whole job's likelihood
        of this pass (a 1-element FP64 tensor, the same on every rank)."""
        self.b.em_pass(x, self.bp, s, self.lik)
        self._sum(self.bp)
        self._sum(self.lik)
        self.b.update(x, self.bp, self.sens[s])
        return self.lik

    def run(self, x, iters):
        if not self.sens:
            self.compute_sensitivity()
        liks = []
        for _ in range(iters):
            for s in range(self.nsub):
                liks.append(float(self.subiteration(x, s).item()))
        return liks


class GpuShard:
    """The CUDA backend: a projector restricted to sinograms [first, first + n),
    the whole job's counts (and multiplicative term) resident on `device`."""

    def __init__(self, image_geom, sino_geom, counts, nsubsets, first, n, device=0, mult=None, stream=None,
                 ge=True, geometry_sparse=False):
        import torch
        from .projector import SiddonProjector
        self.torch = torch
        self.dev = torch.device(f"cuda:{device}")
        self.P = SiddonProjector(image_geom, sino_geom, device=device)
        self.P.set_shard(first, n)
        self.ig, self.sg = image_geom, sino_geom
        self.counts = counts          # whole sinogram, [sinogram][angle][r]
        self.mult = mult              # whole sinogram or None
        self.first, self.n = first, n
        self.nsub = nsubsets
        self.stream = stream
        self.ge = ge                  # update where sens >= 0 (the reference's OSEM rule) or > 0
        # geometry_sparse: passes walk only the shard's bins with counts, the
        # likelihood from the shard's geometry images G_s = A_s^T 1 (made on
        # first use, per subset); summed over the shards as the rest is.
        self.gimg = {} if geometry_sparse else None
        if geometry_sparse:
            from . import _lib
            self.P.set_option(_lib.APIRL_OPT_SPARSE_IMAGE, _lib.APIRL_SPARSE_GEOMETRY)

    def zeros_image(self):
        return self.torch.zeros(self.ig.n_voxels, dtype=self.torch.float32, device=self.dev)

    def scalar(self):
        return self.torch.zeros(1, dtype=self.torch.float64, device=self.dev)

    def sensitivity(self, s, out):
        sg = self.sg
        if self.mult is None:
            vals = self.torch.ones(self.n * subset_nproj(sg.n_proj, s, self.nsub) * sg.n_r, dtype=self.torch.float32,
                                   device=self.dev)
        else:
            m = self.mult.view(sg.n_sinos, sg.n_proj, sg.n_r)[self.first:self.first + self.n, s::self.nsub, :]
            vals = m.contiguous().view(-1)
        self.P.backproject(vals, out, s, self.nsub, stream=self.stream)

    def geometry_image(self, s):
        if s not in self.gimg:
            img = self.zeros_image()
            self.P.backproject_ones(img, s, self.nsub, stream=self.stream)
            self.gimg[s] = img
        return self.gimg[s]

    def em_pass(self, x, bp, s, lik):
        zimg = self.geometry_image(s) if self.gimg is not None else None
        self.P.em_project_backproject(self.counts, x, bp, s, self.nsub, lik=lik, stream=self.stream, zimg=zimg)

    def force_positive(self, img):
        from .projector import force_positive
        force_positive(img, stream=self.stream)

    def update(self, x, bp, sens):
        from .projector import update_pixels
        update_pixels(x, bp, sens, thr_value=0.0, ge=self.ge, zero_bp=True, stream=self.stream)
