"""Seeded synthetic workloads.

No measured data set ships with the reference, so every input is generated:

* ``c1_2d()``  -- 2D MLEM: 128x128 image of 2.08 mm pixels; sinogram 192 r x
  192 angles over 180 deg, 2.08 mm bin pitch (rFov 199.68 mm), ring radius
  443 mm; uniform disc r = 100 mm (1.0) plus 6 single-pixel point sources
  (10.0) uniformly placed in r < 90 mm (seed 0); 1e6 Poisson counts (seed 0).
* ``c2_3d()``  -- 3D OSEM: 256x256x81 image, 2.08x2.08x2.03 mm voxels; 41
  rings of 4.054 mm pitch (axial FOV 166.214 mm), ring radius 443 mm;
  span-1 sinograms of every ring pair with |ring difference| <= 20 (41
  segments, 1261 sinograms) of 336 r x 336 angles, sinogram rFov = image
  rFov = 266.24 mm (1.58476 mm pitch); water cylinder r = 100 mm over the
  axial FOV (1.0) with 6 spheres r = 5 mm at 4.0 (seed 2); attenuation
  factors exp(-0.0096/mm x chord through the cylinder); 5e8 Poisson counts.

Voxel centres follow the reference's image coordinates: x = -rFov + (i+1/2)dx
(data/src/Images.cpp:435-451) and, because Siddon places the first slice at
z = dz/2 (recon/src/Siddon.cpp:162), z = dz/2 + (k+1/2)dz.
"""
import math

import numpy as np

from .geometry import ImageGeom, Sino2DGeom, Sino3DGeom

MU_WATER_PER_MM = 0.0096


def c1_geometry():
    ig = ImageGeom(128, 128, 1, 2.08, 2.08, 1.0)
    sg = Sino2DGeom(192, 192, 199.68, 443.0)
    return ig, sg


def c2_geometry():
    ig = ImageGeom(256, 256, 81, 2.08, 2.08, 2.03)
    sg = Sino3DGeom.span1(336, 336, 41, 266.24, 41 * 4.054, 443.0, 20)
    return ig, sg


def voxel_centres(ig):
    rfov_x = ig.dx * ig.nx / 2.0
    rfov_y = ig.dy * ig.ny / 2.0
    x = -rfov_x + (np.arange(ig.nx) + 0.5) * ig.dx
    y = -rfov_y + (np.arange(ig.ny) + 0.5) * ig.dy
    z = ig.dz / 2.0 + (np.arange(ig.nz) + 0.5) * ig.dz
    return x, y, z


def disc_phantom_2d(ig, seed=0, radius=100.0, n_points=6, point_value=10.0, point_r=90.0):
    x, y, _ = voxel_centres(ig)
    X, Y = np.meshgrid(x, y)
    img = (X ** 2 + Y ** 2 < radius ** 2).astype(np.float32)
    rng = np.random.default_rng(seed)
    for _ in range(n_points):
        r = point_r * math.sqrt(rng.random())
        th = 2 * math.pi * rng.random()
        px, py = r * math.cos(th), r * math.sin(th)
        i = int(np.argmin(np.abs(x - px)))
        j = int(np.argmin(np.abs(y - py)))
        img[j, i] = point_value
    return img.reshape(-1)


def cylinder_phantom_3d(ig, seed=2, radius=100.0, n_spheres=6, sphere_r=5.0, contrast=4.0, centre_r=90.0):
    x, y, z = voxel_centres(ig)
    Y, X = np.meshgrid(y, x, indexing="ij")
    disc = (X ** 2 + Y ** 2 < radius ** 2)
    img = np.repeat(disc[None, :, :], ig.nz, axis=0).astype(np.float32)
    rng = np.random.default_rng(seed)
    zlo, zhi = z[0], z[-1]
    Z = z[:, None, None]
    for _ in range(n_spheres):
        r = centre_r * math.sqrt(rng.random())
        th = 2 * math.pi * rng.random()
        cx, cy = r * math.cos(th), r * math.sin(th)
        cz = zlo + (zhi - zlo) * rng.random()
        m = (X[None] - cx) ** 2 + (Y[None] - cy) ** 2 + (Z - cz) ** 2 < sphere_r ** 2
        img[m] = contrast
    return img.reshape(-1)


def cylinder_chords(lor, z, radius=100.0):
    """FP64 chord length of every LOR of a 3D sinogram through an axially
    unbounded cylinder of `radius` (the LOR end points lie inside the axial
    FOV, so the cylinder spanning that FOV is unbounded for them).

    lor: [n_proj, n_r, 4] end points; z: [n_sinos, 2].  Returns [n_sinos, n_proj, n_r]."""
    p1 = lor[..., :2].astype(np.float64)
    p2 = lor[..., 2:].astype(np.float64)
    d = p2 - p1
    dxy = np.sqrt((d ** 2).sum(-1))
    # Distance of the line from the axis.
    cross = np.abs(p1[..., 0] * d[..., 1] - p1[..., 1] * d[..., 0]) / dxy
    chord_xy = 2.0 * np.sqrt(np.clip(radius ** 2 - cross ** 2, 0.0, None))
    dz = (z[:, 1] - z[:, 0]).astype(np.float64)
    scale = np.sqrt(1.0 + (dz[:, None, None] / dxy[None]) ** 2)
    return chord_xy[None] * scale


# Expected counts per unit of attenuated projection of the 3D workload:
# 5e8 / 1.7491305e9, the sum of (A x_phantom) * attenuation over all
# 142,361,856 bins, so that the job holds 5e8 expected counts.  A constant, so
# that any set of sinograms can be drawn again on its own.
C2_COUNTS_PER_UNIT = np.float32(5e8 / 1749130543.7612033)


def c2_counts(expected, sino_index, n_per_sino, seed=0):
    """Poisson counts (uint32) of the 3D workload.  expected: float32
    (A x_phantom) * attenuation of the listed sinograms, [len(sino_index) *
    n_per_sino]; sino_index: each sinogram's index in the whole sinogram.
    Sinogram g draws from numpy's default_rng([seed, g]), so a sample of
    sinograms gets the same counts as in the whole job."""
    lam = np.asarray(expected, np.float32).reshape(len(sino_index), n_per_sino) * C2_COUNTS_PER_UNIT
    out = np.empty(lam.shape, np.uint32)
    for i, g in enumerate(sino_index):
        out[i] = np.random.default_rng([seed, int(g)]).poisson(lam[i])
    return out.reshape(-1)


def c2_device_arrays(P, dev):
    """The 3D workload's attenuation factors (float32) and Poisson counts
    (uint32 stored in an int32 tensor viewed as uint32), whole sinogram, on
    `dev`.  P: a SiddonProjector of c2_geometry() (its LOR tables give the
    chords; its projection of the phantom times the attenuation gives the
    expected counts)."""
    import torch
    ig, sg = P.image_geom, P.sino_geom
    lor, z = P.tables()
    phantom = torch.from_numpy(cylinder_phantom_3d(ig, seed=2)).to(dev)
    chords = cylinder_chords(lor, z)                      # FP64 on the host
    atten = torch.from_numpy(np.exp(-MU_WATER_PER_MM * chords).astype(np.float32).reshape(-1)).to(dev)
    del chords
    expected = torch.empty(P.num_bins(), dtype=torch.float32, device=dev)
    P.project(phantom, expected)
    expected.mul_(atten)
    # Poisson draws per sinogram on the host (seeded by sinogram index), so
    # that a sample of sinograms can be drawn again identically on its own.
    counts = torch.from_numpy(c2_counts(expected.cpu().numpy(), range(sg.n_sinos),
                                        sg.n_proj * sg.n_r).view(np.int32)).to(dev).view(torch.uint32)
    return atten, counts


def poisson_counts(expected, total, seed=0):
    """Scale `expected` to sum `total` and draw Poisson counts (uint32), numpy."""
    lam = expected.astype(np.float64) * (total / float(expected.sum()))
    rng = np.random.default_rng(seed)
    return rng.poisson(lam).astype(np.uint32)


# ---------------------------------------------------------------------------
# Batched / served jobs: images drawn from {64^2, 128^2, 256^2} x {1, 41, 81}
# slices, radial bins = angles = round(1.3 N) at the voxel pitch, span 1 with
# max ring difference floor(Z/4), (Z+1)/2 rings of pitch 2 dz, random disc +
# sphere phantoms, total counts log-uniform in [1e5, 1e8], 2-4 iterations of
# 7-21 subsets.
def job_geometry(n, z, dxy=2.08, dz=2.03, r_scanner=443.0):
    ig = ImageGeom(n, n, z, dxy, dxy, dz)
    nr = int(round(1.3 * n))
    rings = (z + 1) // 2
    sg = Sino3DGeom.span1(nr, nr, rings, nr * dxy / 2.0, rings * 2 * dz, r_scanner, z // 4)
    return ig, sg


def random_phantom(ig, rng):
    x, y, z = voxel_centres(ig)
    Y, X = np.meshgrid(y, x, indexing="ij")
    w = ig.nx * ig.dx
    rad = w * rng.uniform(0.3, 0.45)
    img = np.repeat(((X ** 2 + Y ** 2) < rad ** 2)[None], ig.nz, axis=0).astype(np.float32)
    Z = z[:, None, None]
    for _ in range(int(rng.integers(1, 4))):
        r = 0.8 * rad * math.sqrt(rng.random())
        th = 2 * math.pi * rng.random()
        cz = z[0] + (z[-1] - z[0]) * rng.random()
        sr = rng.uniform(5.0, 10.0)
        m = (X[None] - r * math.cos(th)) ** 2 + (Y[None] - r * math.sin(th)) ** 2 + (Z - cz) ** 2 < sr ** 2
        img[m] = 4.0
    return img.reshape(-1)


def mixed_job_specs(n_jobs, seed=4, sizes=(64, 128, 256), slices=(1, 41, 81), iters=(2, 4), subsets=(7, 21),
                    counts=(1e5, 1e8)):
    """Seeded list of dicts: n, z, iters, nsubsets, total counts, phantom seed."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_jobs):
        specs.append(dict(n=int(rng.choice(sizes)), z=int(rng.choice(slices)),
                          iters=int(rng.integers(iters[0], iters[1] + 1)),
                          nsubsets=int(rng.integers(subsets[0], subsets[1] + 1)),
                          counts=float(10 ** rng.uniform(math.log10(counts[0]), math.log10(counts[1]))),
                          seed=int(rng.integers(1 << 30))))
    return specs
