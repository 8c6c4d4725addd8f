"""ctypes bindings for the test-only CPU checkers.

* ``Oracle`` wraps ``oracle/_build/liboracle.so``: the C++ restatement of the
  reference Siddon projector and EM loops (float path bit-faithful to the
  reference, double path = FP64 oracle).
* ``RefHarness`` wraps ``oracle/_ref/libapirl_ref_harness.so``: the reference
  APIRL CPU code compiled from its own sources, present only where it was
  built (it needs the reference tree at build time).

Nothing in the product imports this module.
"""
import ctypes
import os
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libapirl_ref_harness.so")

_i = ctypes.c_int
_l = ctypes.c_long
_f = ctypes.c_float
_d = ctypes.c_double
_vp = ctypes.c_void_p


def _p(a):
    return a.ctypes.data_as(_vp) if a is not None else None


class OrSino3d(ctypes.Structure):
    _fields_ = [("nProj", _i), ("nR", _i), ("nRings", _i), ("nSeg", _i),
                ("rFov", _f), ("axialFov", _f), ("rScanner", _f),
                ("minRD", ctypes.POINTER(_i)), ("maxRD", ctypes.POINTER(_i))]


def _sino3d_struct(g):
    """g: apirl_b200.geometry.Sino3DGeom"""
    mn = np.ascontiguousarray(g.min_rd, dtype=np.int32)
    mx = np.ascontiguousarray(g.max_rd, dtype=np.int32)
    s = OrSino3d(g.n_proj, g.n_r, g.n_rings, len(mn), g.r_fov, g.axial_fov, g.r_scanner,
                 mn.ctypes.data_as(ctypes.POINTER(_i)), mx.ctypes.data_as(ctypes.POINTER(_i)))
    s._keep = (mn, mx)
    return s


def _img_args(ig):
    return (ig.nx, ig.ny, ig.nz, ig.dx, ig.dy, ig.dz)


class Oracle:
    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run __graft_entry__.build() or make -f oracle/Makefile")
        self.L = ctypes.CDLL(path)
        L = self.L
        for suf, T in (("f32", _f), ("f64", _d)):
            getattr(L, f"or_project_3d_{suf}").argtypes = [_vp, _i, _i, _i, _i, _i, _f, _f, _f, _vp, _vp, _i]
            getattr(L, f"or_backproject_3d_{suf}").argtypes = [_vp, _i, _i, _i, _i, _i, _f, _f, _f, _vp, _vp, _i]
            getattr(L, f"or_divide_and_backproject_3d_{suf}").argtypes = [_vp, _i, _i, _i, _i, _i, _f, _f, _f,
                                                                          _vp, _vp, _vp, _i]
            getattr(L, f"or_project_2d_{suf}").argtypes = [_i, _i, _f, _f, _vp, _i, _i, _f, _f, _vp, _i]
            getattr(L, f"or_backproject_2d_{suf}").argtypes = [_i, _i, _f, _f, _vp, _i, _i, _f, _f, _vp, _i]
            getattr(L, f"or_divide_and_backproject_2d_{suf}").argtypes = [_i, _i, _f, _f, _vp, _i, _i, _f, _f,
                                                                          _vp, _vp, _i]
            getattr(L, f"or_mlem_2d_{suf}").argtypes = [_i, _i, _f, _f, _vp, _i, _i, _f, _f, _vp, _vp, _vp, _i,
                                                        _vp, _vp, _vp, _i]
            getattr(L, f"or_osem_3d_{suf}").argtypes = [_vp, _i, _i, _i, _f, _f, _f, _vp, _vp, _vp, _vp, _i, _i,
                                                        _vp, _vp, _vp, _i]
            getattr(L, f"or_osem_3d_rule_{suf}").argtypes = [_vp, _i, _i, _i, _f, _f, _f, _vp, _vp, _vp, _vp, _i,
                                                             _i, _vp, _vp, _vp, _i, _i]
            getattr(L, f"or_likelihood_{suf}").argtypes = [_l, _vp, _vp, _i]
            getattr(L, f"or_likelihood_{suf}").restype = T
            getattr(L, f"or_inverse_divide_{suf}").argtypes = [_l, _vp, _vp]
            getattr(L, f"or_mlem_threshold_{suf}").argtypes = [_l, _vp]
            getattr(L, f"or_mlem_threshold_{suf}").restype = T
            getattr(L, f"or_update_{suf}").argtypes = [_l, _vp, _vp, _vp, T, _i]
        L.or_backproject_3d_f32_acc64.argtypes = [_vp, _i, _i, _i, _i, _i, _f, _f, _f, _vp, _vp, _i]
        for suf in ("f32", "f64"):
            getattr(L, f"or_sampled_3d_{suf}").argtypes = [_vp, _i, _i, _i, _i, _i, _i, _i, _i, _i, _f, _f, _f,
                                                           _vp, _vp, _vp, _i]
        L.or_project_3d_tables_f32.argtypes = [_i, _i, _i, _vp, _vp, _i, _i, _i, _i, _i, _f, _f, _f, _vp, _vp, _i]
        L.or_backproject_3d_tables_f32.argtypes = [_i, _i, _i, _vp, _vp, _i, _i, _i, _i, _i, _f, _f, _f, _vp, _vp]
        L.or_lor_points_2d.argtypes = [_i, _i, _f, _f, _vp]
        L.or_sino3d_z.argtypes = [_vp, _vp, _vp]
        L.or_siddon3d_f32.argtypes = [_f, _f, _f, _f, _f, _f, _i, _i, _i, _f, _f, _f, _vp, _vp, _i]
        L.or_count_steps_3d.argtypes = [_vp, _i, _i, _i, _i, _i, _f, _f, _f, _i]
        L.or_count_steps_3d.restype = _l
        self.threads = os.cpu_count() or 1

    @staticmethod
    def _suf(dtype):
        return "f64" if np.dtype(dtype) == np.float64 else "f32"

    # ---- geometry ------------------------------------------------------
    def lor_points_2d(self, n_proj, n_r, r_fov, r_scanner):
        out = np.zeros((n_proj, n_r, 4), np.float32)
        self.L.or_lor_points_2d(n_proj, n_r, r_fov, r_scanner, _p(out))
        return out

    def sino3d_z(self, sg):
        s = _sino3d_struct(sg)
        z1 = np.zeros(sg.n_sinos, np.float32)
        z2 = np.zeros(sg.n_sinos, np.float32)
        n = self.L.or_sino3d_z(ctypes.byref(s), _p(z1), _p(z2))
        assert n == sg.n_sinos
        return z1, z2

    def siddon3d(self, p1, p2, ig, cap=4096):
        ijk = np.zeros((cap, 3), np.int32)
        w = np.zeros(cap, np.float32)
        n = self.L.or_siddon3d_f32(*[float(v) for v in p1], *[float(v) for v in p2], *_img_args(ig),
                                   _p(ijk), _p(w), cap)
        return ijk[:min(n, cap)], w[:min(n, cap)], n

    def count_steps_3d(self, sg, ig, subset=-1, nsub=1):
        s = _sino3d_struct(sg)
        return self.L.or_count_steps_3d(ctypes.byref(s), subset, nsub, *_img_args(ig), self.threads)

    # ---- 3D ------------------------------------------------------------
    def project_3d(self, sg, ig, img, subset=-1, nsub=1, dtype=np.float32, threads=None):
        dt = np.dtype(dtype)
        img = np.ascontiguousarray(img, dtype=dt)
        out = np.zeros(sg.subset_bins(subset, nsub), dt)
        s = _sino3d_struct(sg)
        getattr(self.L, f"or_project_3d_{self._suf(dt)}")(ctypes.byref(s), subset, nsub, *_img_args(ig), _p(img),
                                                         _p(out), threads or self.threads)
        return out

    def backproject_3d(self, sg, ig, values, subset=-1, nsub=1, dtype=np.float32, threads=None, out=None):
        dt = np.dtype(dtype)
        values = np.ascontiguousarray(values, dtype=dt)
        img = np.zeros(ig.n_voxels, dt) if out is None else out
        s = _sino3d_struct(sg)
        getattr(self.L, f"or_backproject_3d_{self._suf(dt)}")(ctypes.byref(s), subset, nsub, *_img_args(ig),
                                                             _p(values), _p(img), threads or self.threads)
        return img

    def backproject_3d_exact_sum(self, sg, ig, values, subset=-1, nsub=1, threads=None):
        """The float backprojection's own contributions (float walk, float
        segment * value) summed in double: what a float accumulation of them
        would give without rounding."""
        values = np.ascontiguousarray(values, dtype=np.float32)
        img = np.zeros(ig.n_voxels, np.float64)
        s = _sino3d_struct(sg)
        self.L.or_backproject_3d_f32_acc64(ctypes.byref(s), subset, nsub, *_img_args(ig), _p(values), _p(img),
                                           threads or self.threads)
        return img

    def divide_and_backproject_3d(self, sg, ig, vin, vest, subset=-1, nsub=1, dtype=np.float32, threads=None):
        dt = np.dtype(dtype)
        vin = np.ascontiguousarray(vin, dtype=dt)
        vest = np.ascontiguousarray(vest, dtype=dt)
        img = np.zeros(ig.n_voxels, dt)
        s = _sino3d_struct(sg)
        getattr(self.L, f"or_divide_and_backproject_3d_{self._suf(dt)}")(
            ctypes.byref(s), subset, nsub, *_img_args(ig), _p(vin), _p(vest), _p(img), threads or self.threads)
        return img

    def sampled_3d(self, sg, ig, mode, ns, nas, multi, vin, vest=None, subset=-1, nsub=1, dtype=np.float32,
                   threads=None):
        """Projectors with several rays per bin.  mode 0: Project (vin = image),
        1: Backproject, 2: DivideAndBackproject (vin / vest sinograms)."""
        dt = np.dtype(dtype)
        vin = np.ascontiguousarray(vin, dtype=dt)
        vest = None if vest is None else np.ascontiguousarray(vest, dtype=dt)
        out = np.zeros(sg.subset_bins(subset, nsub) if mode == 0 else ig.n_voxels, dt)
        s = _sino3d_struct(sg)
        rc = getattr(self.L, f"or_sampled_3d_{self._suf(dt)}")(
            ctypes.byref(s), ns, nas, int(multi), mode, subset, nsub, *_img_args(ig), _p(vin), _p(vest), _p(out),
            threads or self.threads)
        assert rc == 0
        return out

    def project_3d_tables(self, lor, z, ig, img, subset=-1, nsub=1, threads=None):
        """Projection over given tables: lor [n_proj, n_r, 4], z [n_sinos, 2] (float32)."""
        lor = np.ascontiguousarray(lor, np.float32)
        z = np.ascontiguousarray(z, np.float32)
        n_proj, n_r = lor.shape[0], lor.shape[1]
        n_sinos = z.shape[0]
        img = np.ascontiguousarray(img, np.float32)
        nk = len(range(subset, n_proj, nsub)) if subset >= 0 else n_proj
        out = np.zeros(n_sinos * nk * n_r, np.float32)
        self.L.or_project_3d_tables_f32(n_sinos, n_proj, n_r, _p(lor), _p(z), subset, nsub, *_img_args(ig), _p(img),
                                        _p(out), threads or self.threads)
        return out

    def backproject_3d_tables(self, lor, z, ig, values, subset=-1, nsub=1):
        lor = np.ascontiguousarray(lor, np.float32)
        z = np.ascontiguousarray(z, np.float32)
        values = np.ascontiguousarray(values, np.float32)
        img = np.zeros(ig.n_voxels, np.float32)
        self.L.or_backproject_3d_tables_f32(z.shape[0], lor.shape[0], lor.shape[1], _p(lor), _p(z), subset, nsub,
                                            *_img_args(ig), _p(values), _p(img))
        return img

    def osem_3d(self, sg, ig, init, meas, iters, nsub, mult=None, add=None, dtype=np.float32, threads=None,
                ge=True):
        """ge=False: update only where sens > 0 (else 0) instead of the reference's sens >= 0."""
        dt = np.dtype(dtype)
        cv = lambda a: None if a is None else np.ascontiguousarray(a, dtype=dt)
        init, meas, mult, add = cv(init), cv(meas), cv(mult), cv(add)
        out = np.zeros(ig.n_voxels, dt)
        lik = np.zeros(iters * nsub + 1, dt)
        sens0 = np.zeros(ig.n_voxels, dt)
        s = _sino3d_struct(sg)
        getattr(self.L, f"or_osem_3d_rule_{self._suf(dt)}")(ctypes.byref(s), *_img_args(ig), _p(init), _p(meas),
                                                           _p(mult), _p(add), iters, nsub, _p(out), _p(lik),
                                                           _p(sens0), threads or self.threads, int(bool(ge)))
        return out, lik, sens0

    # ---- 2D ------------------------------------------------------------
    def project_2d(self, sg, ig, img, dtype=np.float32, threads=None, out=None):
        dt = np.dtype(dtype)
        img = np.ascontiguousarray(img, dtype=dt)
        out = np.zeros(sg.n_bins, dt) if out is None else out
        getattr(self.L, f"or_project_2d_{self._suf(dt)}")(ig.nx, ig.ny, ig.dx, ig.dy, _p(img), sg.n_proj, sg.n_r,
                                                         sg.r_fov, sg.r_scanner, _p(out), threads or self.threads)
        return out

    def backproject_2d(self, sg, ig, values, dtype=np.float32, threads=None):
        dt = np.dtype(dtype)
        values = np.ascontiguousarray(values, dtype=dt)
        img = np.zeros(ig.n_voxels, dt)
        getattr(self.L, f"or_backproject_2d_{self._suf(dt)}")(ig.nx, ig.ny, ig.dx, ig.dy, _p(img), sg.n_proj,
                                                             sg.n_r, sg.r_fov, sg.r_scanner, _p(values),
                                                             threads or self.threads)
        return img

    def divide_and_backproject_2d(self, sg, ig, vin, vest, dtype=np.float32, threads=None):
        dt = np.dtype(dtype)
        vin = np.ascontiguousarray(vin, dtype=dt)
        vest = np.ascontiguousarray(vest, dtype=dt)
        img = np.zeros(ig.n_voxels, dt)
        getattr(self.L, f"or_divide_and_backproject_2d_{self._suf(dt)}")(
            ig.nx, ig.ny, ig.dx, ig.dy, _p(img), sg.n_proj, sg.n_r, sg.r_fov, sg.r_scanner, _p(vin), _p(vest),
            threads or self.threads)
        return img

    def mlem_2d(self, sg, ig, init, meas, iters, mult=None, add=None, dtype=np.float32, threads=None):
        dt = np.dtype(dtype)
        cv = lambda a: None if a is None else np.ascontiguousarray(a, dtype=dt)
        init, meas, mult, add = cv(init), cv(meas), cv(mult), cv(add)
        out = np.zeros(ig.n_voxels, dt)
        lik = np.zeros(iters + 1, dt)
        sens = np.zeros(ig.n_voxels, dt)
        getattr(self.L, f"or_mlem_2d_{self._suf(dt)}")(ig.nx, ig.ny, ig.dx, ig.dy, _p(init), sg.n_proj, sg.n_r,
                                                      sg.r_fov, sg.r_scanner, _p(meas), _p(mult), _p(add), iters,
                                                      _p(out), _p(lik), _p(sens), threads or self.threads)
        return out, lik, sens

    # ---- bin / pixel steps ---------------------------------------------
    def likelihood(self, est, meas, gt0=False):
        dt = est.dtype
        return getattr(self.L, f"or_likelihood_{self._suf(dt)}")(est.size, _p(est), _p(meas.astype(dt)), int(gt0))

    def inverse_divide(self, meas, est):
        est = est.copy()
        getattr(self.L, f"or_inverse_divide_{self._suf(est.dtype)}")(est.size, _p(meas.astype(est.dtype)), _p(est))
        return est

    def mlem_threshold(self, sens):
        return getattr(self.L, f"or_mlem_threshold_{self._suf(sens.dtype)}")(sens.size, _p(sens))

    def update(self, x, bp, sens, thr, ge):
        x = x.copy()
        getattr(self.L, f"or_update_{self._suf(x.dtype)}")(x.size, _p(x), _p(bp), _p(sens), thr, int(ge))
        return x


class RefHarness:
    """The reference APIRL CPU code, compiled from its own sources."""

    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.L = ctypes.CDLL(path)
        L = self.L
        L.ref_set_threads.argtypes = [_i]
        L.ref_lor_points_2d.argtypes = [_i, _i, _f, _f, _vp]
        L.ref_siddon3d.argtypes = [_f, _f, _f, _f, _f, _f, _i, _i, _i, _f, _f, _f, _vp, _vp, _i]
        L.ref_project_2d.argtypes = [_i, _i, _f, _f, _vp, _i, _i, _f, _f, _vp]
        L.ref_backproject_2d.argtypes = [_i, _i, _f, _f, _vp, _i, _i, _f, _f, _vp]
        L.ref_mlem_2d.argtypes = [_i, _i, _f, _f, _vp, _i, _i, _f, _f, _vp, _i, ctypes.c_char_p, _vp, _vp, _vp]
        L.ref_sino3d_create.argtypes = [ctypes.c_char_p, _i, _i, _i, _f, _f, _f, _i, _vp, _vp, _vp, _vp]
        L.ref_sino3d_create.restype = _vp
        L.ref_sino3d_destroy.argtypes = [_vp]
        L.ref_sino3d_num_bins.argtypes = [_vp]
        L.ref_sino3d_num_bins.restype = _l
        L.ref_sino3d_ring_z.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp]
        L.ref_project_3d.argtypes = [_vp, _i, _i, _i, _i, _i, _f, _f, _f, _vp, _vp]
        L.ref_backproject_3d.argtypes = [_vp, _i, _i, _i, _i, _i, _f, _f, _f, _vp, _vp]
        L.ref_osem_3d_subiteration.argtypes = [_vp, _i, _i, _i, _i, _i, _f, _f, _f, _vp, _vp, _vp]
        L.ref_osem_3d_subiteration_rule.argtypes = [_vp, _i, _i, _i, _i, _i, _f, _f, _f, _vp, _vp, _vp, _i]
        L.ref_osem_3d.argtypes = [_vp, _i, _i, _i, _f, _f, _f, _vp, _i, _i, ctypes.c_char_p, _vp, _vp, _vp]
        L.ref_sino3d_write.argtypes = [_vp, ctypes.c_char_p]
        L.ref_image_write.argtypes = [_i, _i, _i, _f, _f, _f, _vp, ctypes.c_char_p]
        L.ref_image_read.argtypes = [ctypes.c_char_p, _vp, _vp, _vp, _l]
        L.ref_sino3d_read.argtypes = [ctypes.c_char_p, _f, _f, _f, _vp, _l, _vp]
        L.ref_sino3d_read.restype = _l
        L.ref_sampled_3d.argtypes = [_vp, _i, _i, _i, _i, _i, _i, _i, _i, _i, _f, _f, _f, _vp, _vp, _vp]
        L.ref_mmr_sino3d_create.argtypes = [ctypes.c_char_p, _i, _i, _i, _i, _vp, _vp, _vp, _vp]
        L.ref_mmr_sino3d_create.restype = _vp
        L.ref_mmr_tables.argtypes = [_vp, _vp, _vp]
        L.ref_mmr_project.argtypes = [_vp, _i, _i, _i, _f, _f, _f, _vp, _vp]
        L.ref_mmr_backproject.argtypes = [_vp, _i, _i, _i, _f, _f, _f, _vp, _vp]
        self._tmp = tempfile.mkdtemp(prefix="apirl_ref_")

    def set_threads(self, n):
        return self.L.ref_set_threads(n)

    def lor_points_2d(self, n_proj, n_r, r_fov, r_scanner):
        out = np.zeros((n_proj, n_r, 4), np.float32)
        self.L.ref_lor_points_2d(n_proj, n_r, r_fov, r_scanner, _p(out))
        return out

    def siddon3d(self, p1, p2, ig, cap=4096):
        ijk = np.zeros((cap, 3), np.int32)
        w = np.zeros(cap, np.float32)
        n = self.L.ref_siddon3d(*[float(v) for v in p1], *[float(v) for v in p2], *_img_args(ig), _p(ijk), _p(w), cap)
        return ijk[:min(n, cap)], w[:min(n, cap)], n

    def project_2d(self, sg, ig, img):
        img = np.ascontiguousarray(img, np.float32)
        out = np.zeros(sg.n_bins, np.float32)
        self.L.ref_project_2d(ig.nx, ig.ny, ig.dx, ig.dy, _p(img), sg.n_proj, sg.n_r, sg.r_fov, sg.r_scanner, _p(out))
        return out

    def backproject_2d(self, sg, ig, values):
        values = np.ascontiguousarray(values, np.float32)
        img = np.zeros(ig.n_voxels, np.float32)
        self.L.ref_backproject_2d(ig.nx, ig.ny, ig.dx, ig.dy, _p(img), sg.n_proj, sg.n_r, sg.r_fov, sg.r_scanner,
                                  _p(values))
        return img

    def mlem_2d(self, sg, ig, init, meas, iters):
        init = np.ascontiguousarray(init, np.float32)
        meas = np.ascontiguousarray(meas, np.float32)
        out = np.zeros(ig.n_voxels, np.float32)
        lik = np.zeros(iters + 1, np.float32)
        sens = np.zeros(ig.n_voxels, np.float32)
        d = tempfile.mkdtemp(dir=self._tmp)
        rc = self.L.ref_mlem_2d(ig.nx, ig.ny, ig.dx, ig.dy, _p(init), sg.n_proj, sg.n_r, sg.r_fov, sg.r_scanner,
                                _p(meas), iters, d.encode(), _p(out), _p(lik), _p(sens))
        assert rc == 0
        return out, lik, sens

    def sino3d(self, sg, data=None):
        d = tempfile.mkdtemp(dir=self._tmp)
        nsin = np.ascontiguousarray(sg.sinos_per_segment, np.int32)
        mn = np.ascontiguousarray(sg.min_rd, np.int32)
        mx = np.ascontiguousarray(sg.max_rd, np.int32)
        dat = None if data is None else np.ascontiguousarray(data, np.float32)
        h = self.L.ref_sino3d_create(d.encode(), sg.n_proj, sg.n_r, sg.n_rings, sg.r_fov, sg.axial_fov,
                                     sg.r_scanner, len(mn), _p(nsin), _p(mn), _p(mx), _p(dat))
        if not h:
            raise RuntimeError("reference failed to read the sinogram header")
        return h

    def ring_z(self, h, n_sinos):
        a = [np.zeros(n_sinos, np.float32) for _ in range(4)]
        nz = np.zeros(n_sinos, np.int32)
        self.L.ref_sino3d_ring_z(h, *[_p(x) for x in a], _p(nz))
        return a, nz

    def project_3d(self, h, sg, ig, img, subset=-1, nsub=1):
        img = np.ascontiguousarray(img, np.float32)
        out = np.zeros(sg.subset_bins(subset, nsub), np.float32)
        self.L.ref_project_3d(h, subset, nsub, *_img_args(ig), _p(img), _p(out))
        return out

    def backproject_3d(self, h, sg, ig, values, subset=-1, nsub=1):
        values = np.ascontiguousarray(values, np.float32)
        img = np.zeros(ig.n_voxels, np.float32)
        self.L.ref_backproject_3d(h, subset, nsub, *_img_args(ig), _p(values), _p(img))
        return img

    def sampled_3d(self, h, sg, ig, mode, ns, nas, multi, vin, vest=None, subset=-1, nsub=1):
        vin = np.ascontiguousarray(vin, np.float32)
        vest = None if vest is None else np.ascontiguousarray(vest, np.float32)
        out = np.zeros(sg.subset_bins(subset, nsub) if mode == 0 else ig.n_voxels, np.float32)
        assert self.L.ref_sampled_3d(h, ns, nas, int(multi), mode, subset, nsub, *_img_args(ig), _p(vin), _p(vest),
                                     _p(out)) == 0
        return out

    # ---- Siemens mMR (whole sinogram only) ------------------------------------
    def mmr_sino3d(self, sg, data=None):
        d = tempfile.mkdtemp(dir=self._tmp)
        nsin = np.ascontiguousarray(sg.sinos_per_segment, np.int32)
        mn = np.ascontiguousarray(sg.min_rd, np.int32)
        mx = np.ascontiguousarray(sg.max_rd, np.int32)
        dat = None if data is None else np.ascontiguousarray(data, np.float32)
        h = self.L.ref_mmr_sino3d_create(d.encode(), sg.n_proj, sg.n_r, sg.n_rings, len(mn), _p(nsin), _p(mn),
                                         _p(mx), _p(dat))
        if not h:
            raise RuntimeError("reference failed to read the mMR sinogram header")
        return h

    def mmr_tables(self, h, sg):
        lor = np.zeros((sg.n_proj, sg.n_r, 4), np.float32)
        z = np.zeros((sg.n_sinos, 2), np.float32)
        assert self.L.ref_mmr_tables(h, _p(lor), _p(z)) == sg.n_sinos
        return lor, z

    def mmr_project(self, h, sg, ig, img):
        img = np.ascontiguousarray(img, np.float32)
        out = np.zeros(sg.n_bins, np.float32)
        self.L.ref_mmr_project(h, *_img_args(ig), _p(img), _p(out))
        return out

    def mmr_backproject(self, h, sg, ig, values):
        values = np.ascontiguousarray(values, np.float32)
        img = np.zeros(ig.n_voxels, np.float32)
        self.L.ref_mmr_backproject(h, *_img_args(ig), _p(values), _p(img))
        return img

    def osem_subiteration(self, h, ig, subset, nsub, x, sens, ge=True):
        """One OSEM sub-iteration in place on x; ge=False updates only where sens > 0."""
        lik = np.zeros(1, np.float32)
        self.L.ref_osem_3d_subiteration_rule(h, subset, nsub, *_img_args(ig), _p(x), _p(sens), _p(lik), int(bool(ge)))
        return float(lik[0])

    def write_sino3d(self, h, path_no_ext):
        assert self.L.ref_sino3d_write(h, path_no_ext.encode()) == 0

    def write_image(self, ig, px, path_no_ext):
        px = np.ascontiguousarray(px, np.float32)
        assert self.L.ref_image_write(*_img_args(ig), _p(px), path_no_ext.encode()) == 0

    def read_image(self, header, cap=1 << 24):
        dims = np.zeros(3, np.int32)
        pix = np.zeros(3, np.float32)
        out = np.zeros(cap, np.float32)
        if self.L.ref_image_read(header.encode(), _p(dims), _p(pix), _p(out), cap) != 0:
            raise RuntimeError("reference could not read " + header)
        return dims, pix, out[:int(np.prod(dims))]

    def read_sino3d(self, header, sg, cap=1 << 26):
        out = np.zeros(cap, np.float32)
        nseg = np.zeros(1, np.int32)
        n = self.L.ref_sino3d_read(header.encode(), sg.r_fov, sg.axial_fov, sg.r_scanner, _p(out), cap, _p(nseg))
        return out[:n], int(nseg[0])

    def osem_3d(self, h, ig, init, iters, nsub):
        init = np.ascontiguousarray(init, np.float32)
        out = np.zeros(ig.n_voxels, np.float32)
        lik = np.zeros(iters * nsub + 1, np.float32)
        sens0 = np.zeros(ig.n_voxels, np.float32)
        d = tempfile.mkdtemp(dir=self._tmp)
        rc = self.L.ref_osem_3d(h, *_img_args(ig), _p(init), iters, nsub, d.encode(), _p(out), _p(lik), _p(sens0))
        assert rc == 0
        return out, lik, sens0
