"""Scanner, sinogram and image geometry descriptors.

These mirror the reference's geometry objects field by field:

* ``ImageGeom``   -- ``SizeImage`` (data/inc/Images.h:53-61); voxels [z][y][x],
  field-of-view radius ``dx * nx / 2`` (data/src/Images.cpp:55).
* ``Sino2DGeom``  -- ``Sinogram2DinCylindrical3Dpet(nProj, nR, rFov, rScanner)``
  (data/src/Sinogram2DinCylindrical3Dpet.cpp:29-64); bins [angle][r].
* ``Sino3DGeom``  -- ``Sinogram3DCylindricalPet`` as read from an interfile
  header (data/src/Sinogram3D.cpp:106-471): segments with a ring-difference
  range each, sinograms per segment ordered as the reference builds them,
  bins [segment][sinogram][angle][r].
"""
from dataclasses import dataclass, field
from typing import List
import math


@dataclass
class ImageGeom:
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float

    @property
    def n_voxels(self):
        return self.nx * self.ny * self.nz

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)


@dataclass
class Sino2DGeom:
    n_proj: int
    n_r: int
    r_fov: float
    r_scanner: float

    @property
    def n_bins(self):
        return self.n_proj * self.n_r


def subset_nproj(n_proj, subset, nsub):
    """Angles in subset ``subset`` of ``nsub`` (Sinogram3DCylindricalPet.cpp:164-171)."""
    if subset < 0:
        return n_proj
    n = int(math.floor(float(n_proj) / float(nsub)))
    if n_proj % nsub > subset:
        n += 1
    return n


@dataclass
class Sino3DGeom:
    n_proj: int
    n_r: int
    n_rings: int
    r_fov: float
    axial_fov: float
    r_scanner: float
    min_rd: List[int]
    max_rd: List[int]
    sinos_per_segment: List[int] = field(default_factory=list)
    scanner: str = "cylindrical"   # or "mmr" (Siemens Biograph mMR geometry)

    def __post_init__(self):
        if not self.sinos_per_segment:
            self.sinos_per_segment = [self._count(mn, mx) for mn, mx in zip(self.min_rd, self.max_rd)]

    def _count(self, mn, mx):
        # Same enumeration as Sinogram3D::readFromInterfile (Sinogram3D.cpp:396-433).
        n = 0
        R = self.n_rings
        for z1 in range(2 * R):
            hit = False
            z1a = z1
            for z2 in range(R):
                if mn <= z1a - z2 <= mx and 0 <= z1a < R and 0 <= z2 < R:
                    hit = True
                z1a -= 1
            n += hit
        return n

    @classmethod
    def span1(cls, n_proj, n_r, n_rings, r_fov, axial_fov, r_scanner, max_ring_diff):
        """Span-1 sinogram with segments ordered 0, +1, -1, +2, -2, ..."""
        rds = [0]
        for d in range(1, max_ring_diff + 1):
            rds += [d, -d]
        return cls(n_proj, n_r, n_rings, r_fov, axial_fov, r_scanner, rds, list(rds))

    @classmethod
    def span(cls, n_proj, n_r, n_rings, r_fov, axial_fov, r_scanner, span, max_ring_diff):
        """Axially compressed sinogram of odd span S: segment 0 covers ring
        differences -(S-1)/2..(S-1)/2, then +1, -1, +2, -2, ... each the next S
        differences, up to max_ring_diff; several ring pairs share a sinogram."""
        if span < 1 or span % 2 == 0:
            raise ValueError("span must be odd")
        h = (span - 1) // 2
        mn, mx = [-h], [h]
        lo = h + 1
        while lo <= max_ring_diff:
            hi = min(lo + span - 1, max_ring_diff)
            mn += [lo, -hi]
            mx += [hi, -lo]
            lo = hi + 1
        return cls(n_proj, n_r, n_rings, r_fov, axial_fov, r_scanner, mn, mx)

    @classmethod
    def mmr(cls, n_proj=252, n_r=344, n_rings=64, span=11, max_ring_diff=60):
        """Siemens Biograph mMR sinogram (Sinogram3DSiemensMmr): r_fov 297,
        axial fov 260, radius 328 mm are the scanner's constants."""
        g = cls.span(n_proj, n_r, n_rings, 297.0, 260.0, 328.0, span, max_ring_diff) if span > 1 else \
            cls.span1(n_proj, n_r, n_rings, 297.0, 260.0, 328.0, max_ring_diff)
        g.scanner = "mmr"
        return g

    @property
    def n_segments(self):
        return len(self.min_rd)

    @property
    def n_sinos(self):
        return sum(self.sinos_per_segment)

    @property
    def n_bins(self):
        return self.n_sinos * self.n_proj * self.n_r

    def subset_nproj(self, subset, nsub):
        return subset_nproj(self.n_proj, subset, nsub)

    def subset_bins(self, subset, nsub):
        return self.n_sinos * self.subset_nproj(subset, nsub) * self.n_r

    def subset_angles(self, subset, nsub):
        if subset < 0:
            return list(range(self.n_proj))
        return [subset + nsub * k for k in range(self.subset_nproj(subset, nsub))]
