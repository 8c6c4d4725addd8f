"""Python front end over the C ABI.

``SiddonProjector`` mirrors the reference's ``SiddonProjector`` /
``CuSiddonProjector`` operations (Project, Backproject, DivideAndBackproject;
recon/inc/SiddonProjector.h:25-68) on device-resident torch tensors, plus the
fused EM pass.  ``osem_3d`` / ``mlem_3d`` / ``mlem_2d`` mirror the
``OsemSinogram3d`` / ``MlemSinogram3d`` / ``Mlem2d`` drivers on host arrays.
torch provides device memory and streams only; every operation runs in the
CUDA library.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, ImageGeomC, Sino2DGeomC, Sino3DGeomC
from .geometry import ImageGeom, Sino2DGeom, Sino3DGeom


def _img_c(ig):
    return ImageGeomC(ig.nx, ig.ny, ig.nz, ig.dx, ig.dy, ig.dz)


def _sino3d_c(sg):
    mn = (ctypes.c_int * sg.n_segments)(*sg.min_rd)
    mx = (ctypes.c_int * sg.n_segments)(*sg.max_rd)
    c = Sino3DGeomC(sg.n_proj, sg.n_r, sg.n_rings, sg.n_segments, sg.r_fov, sg.axial_fov, sg.r_scanner,
                    ctypes.cast(mn, ctypes.POINTER(ctypes.c_int)), ctypes.cast(mx, ctypes.POINTER(ctypes.c_int)),
                    _lib.APIRL_SCANNER_MMR if getattr(sg, "scanner", "cylindrical") == "mmr"
                    else _lib.APIRL_SCANNER_CYLINDRICAL)
    c._keep = (mn, mx)
    return c


def _sino2d_c(sg):
    return Sino2DGeomC(sg.n_proj, sg.n_r, sg.r_fov, sg.r_scanner)


def _ptr(t):
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


_DT = {"float32": _lib.APIRL_F32, "uint32": _lib.APIRL_U32, "uint16": _lib.APIRL_U16}


def _counts_dtype(t):
    name = str(t.dtype).replace("torch.", "")
    if name not in _DT:
        raise TypeError(f"counts must be float32, uint32 or uint16, not {t.dtype}")
    return _DT[name]


class SiddonProjector:
    """Siddon projector bound to one image geometry and one sinogram geometry."""

    def __init__(self, image_geom: ImageGeom, sino_geom, device=0):
        self.lib = _lib.load()
        self.image_geom = image_geom
        self.sino_geom = sino_geom
        self.device = device
        h = ctypes.c_void_p()
        ig = _img_c(image_geom)
        if isinstance(sino_geom, Sino3DGeom):
            self._sc = _sino3d_c(sino_geom)
            check(self.lib.apirl_projector_create_3d(ctypes.byref(ig), ctypes.byref(self._sc), device,
                                                     ctypes.byref(h)))
            self.is3d = True
        elif isinstance(sino_geom, Sino2DGeom):
            self._sc = _sino2d_c(sino_geom)
            check(self.lib.apirl_projector_create_2d(ctypes.byref(ig), ctypes.byref(self._sc), device,
                                                     ctypes.byref(h)))
            self.is3d = False
        else:
            raise TypeError("sino_geom must be Sino2DGeom or Sino3DGeom")
        self.h = h

    def close(self):
        if self.h:
            self.lib.apirl_projector_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- sizes / tables ------------------------------------------------
    def num_bins(self, subset=-1, nsubsets=1):
        return int(self.lib.apirl_projector_num_bins(self.h, subset, nsubsets))

    @property
    def num_sinograms(self):
        return int(self.lib.apirl_projector_num_sinograms(self.h))

    def tables(self):
        sg = self.sino_geom
        lor = np.zeros((sg.n_proj, sg.n_r, 4), np.float32)
        z = np.zeros((self.num_sinograms, 2), np.float32) if self.is3d else None
        check(self.lib.apirl_projector_tables(self.h, lor.ctypes.data_as(ctypes.c_void_p),
                                              None if z is None else z.ctypes.data_as(ctypes.c_void_p)))
        return lor, z

    def set_alpha_precision(self, fp64):
        """fp64=False: the reference's float walk (default); True: FP64 alphas (precision study)."""
        check(self.lib.apirl_projector_set_alpha_precision(self.h, _lib.APIRL_ALPHA_F64 if fp64 else _lib.APIRL_ALPHA_F32))

    def set_sampling(self, n_samples=1, n_axial_samples=1, multiple_lors_per_bin=False):
        """Rays per bin: SiddonProjector(nSamples, nAxialSamples) and setMultipleLorsPerBin (3D)."""
        check(self.lib.apirl_projector_set_sampling(self.h, int(n_samples), int(n_axial_samples),
                                                    int(bool(multiple_lors_per_bin))))

    def set_shard(self, first_sinogram, n_sinograms):
        """Restrict every operation to sinograms [first, first + n) of the whole sinogram."""
        check(self.lib.apirl_projector_set_shard(self.h, int(first_sinogram), int(n_sinograms)))

    def set_option(self, option, value):
        check(self.lib.apirl_projector_set_option(self.h, int(option), int(value)))

    def autotune(self, counts, x, subset=0, nsubsets=1, repeats=2, stream=None):
        """Picks the fused kernel's block size by timing the candidates; returns it."""
        best = ctypes.c_int()
        check(self.lib.apirl_projector_autotune(self.h, _ptr(counts), _counts_dtype(counts), _ptr(x), subset, nsubsets,
                                                repeats, ctypes.byref(best), _stream(stream)))
        return best.value

    def autotune_shape(self, counts, x, zimg=None, subset=0, nsubsets=1, repeats=2, stream=None):
        """apirl_projector_autotune_ex: block size and gather segments in flight
        of the fused pass (the sparse pass over bins with counts when zimg is
        given), timed on these counts; the projector keeps the fastest.
        Returns (block, unroll, ms per pass)."""
        out = _lib.TuneC()
        check(self.lib.apirl_projector_autotune_ex(self.h, _ptr(counts), _counts_dtype(counts), _ptr(x), _ptr(zimg),
                                                   subset, nsubsets, repeats, ctypes.byref(out), _stream(stream)))
        return out.block, out.unroll, out.ms

    def last_kernel_ms(self):
        """CUDA-event duration of the last fused kernel (needs APIRL_OPT_KERNEL_TIMING)."""
        ms = ctypes.c_double()
        check(self.lib.apirl_projector_kernel_ms(self.h, ctypes.byref(ms)))
        return ms.value

    def count_steps(self, subset=-1, nsubsets=1, stream=None):
        import torch
        out = torch.empty(self.num_bins(subset, nsubsets), dtype=torch.int32, device=f"cuda:{self.device}")
        check(self.lib.apirl_count_steps(self.h, subset, nsubsets, _ptr(out), _stream(stream)))
        return out

    # ---- projector operations (device tensors) ------------------------
    def project(self, image, sino, subset=-1, nsubsets=1, stream=None):
        """sino = A image (3D: sino is overwritten; 2D: bins with r > rFov untouched)."""
        check(self.lib.apirl_project(self.h, _ptr(image), _ptr(sino), subset, nsubsets, _stream(stream)))
        return sino

    def backproject_ones(self, image, subset=-1, nsubsets=1, stream=None):
        """image += A_s^T 1 (the unweighted sensitivity; G_s of the sparse pass
        with APIRL_SPARSE_GEOMETRY)."""
        check(self.lib.apirl_backproject_ones(self.h, _ptr(image), subset, nsubsets, _stream(stream)))
        return image

    def backproject_and_ones(self, sino, image, ones_image, subset=-1, nsubsets=1, stream=None):
        """image += A_s^T sino and ones_image += A_s^T 1 along one set of walks
        (a sensitivity with a multiplicative sinogram and G_s together)."""
        check(self.lib.apirl_backproject_and_ones(self.h, _ptr(sino), _ptr(image), _ptr(ones_image), subset, nsubsets,
                                                  _stream(stream)))
        return image, ones_image

    def backproject(self, sino, image, subset=-1, nsubsets=1, stream=None):
        """image += A^T sino."""
        check(self.lib.apirl_backproject(self.h, _ptr(sino), _ptr(image), subset, nsubsets, _stream(stream)))
        return image

    def divide_and_backproject(self, meas, est, image, subset=-1, nsubsets=1, stream=None):
        """image += A^T (meas / est) with the reference's zero rules."""
        check(self.lib.apirl_divide_and_backproject(self.h, _ptr(meas), _ptr(est), _ptr(image), subset, nsubsets,
                                                    _stream(stream)))
        return image

    def generate_acf(self, mu, acf, subset=-1, nsubsets=1, stream=None):
        """acf = exp(A mu) where A mu != 0, else 1 (generateACFs)."""
        check(self.lib.apirl_generate_acf(self.h, _ptr(mu), _ptr(acf), subset, nsubsets, _stream(stream)))
        return acf

    def em_pass(self, counts, x, bp, sens, subset=-1, nsubsets=1, add=None, thr=None, thr_value=0.0, ge=True,
                counts_packed=False, lik=None, stream=None):
        """One fused EM pass (OSEM sub-iteration / MLEM iteration); x is updated in place."""
        check(self.lib.apirl_em_pass(self.h, _ptr(counts), _counts_dtype(counts), int(counts_packed), _ptr(add),
                                     _ptr(x), _ptr(bp), _ptr(sens), _ptr(thr), float(thr_value), int(ge), subset,
                                     nsubsets, _ptr(lik), _stream(stream)))
        return x

    def zero_count_image(self, counts, zimg, subset=-1, nsubsets=1, add=None, counts_packed=False, zero_add=None,
                         stream=None):
        """zimg += A_s^T 1[counts == 0]; zero_add (device double) = sum of add over those bins."""
        check(self.lib.apirl_zero_count_image(self.h, _ptr(counts), _counts_dtype(counts), int(counts_packed),
                                              _ptr(add), _ptr(zimg), _ptr(zero_add), subset, nsubsets,
                                              _stream(stream)))
        return zimg

    def em_pass_sparse(self, counts, x, bp, sens, zimg, subset=-1, nsubsets=1, add=None, zero_add=None, thr=None,
                       thr_value=0.0, ge=True, counts_packed=False, lik=None, stream=None):
        """em_pass walking only bins with counts; zimg / zero_add from zero_count_image."""
        check(self.lib.apirl_em_pass_sparse(self.h, _ptr(counts), _counts_dtype(counts), int(counts_packed),
                                            _ptr(add), _ptr(x), _ptr(bp), _ptr(sens), _ptr(zimg), _ptr(zero_add),
                                            _ptr(thr), float(thr_value), int(ge), subset, nsubsets, _ptr(lik),
                                            _stream(stream)))
        return x

    def em_project_backproject(self, counts, x, bp, subset=-1, nsubsets=1, add=None, counts_packed=False, lik=None,
                               stream=None, zimg=None, zero_add=None):
        """The fused kernel of em_pass alone (bp += A^T (m / (A x + add))); x is
        not updated.  With zimg: the sparse form (apirl_em_project_backproject_sparse)."""
        if zimg is not None:
            check(self.lib.apirl_em_project_backproject_sparse(
                self.h, _ptr(counts), _counts_dtype(counts), int(counts_packed), _ptr(add), _ptr(x), _ptr(bp),
                _ptr(zimg), _ptr(zero_add), subset, nsubsets, _ptr(lik), _stream(stream)))
            return bp
        check(self.lib.apirl_em_project_backproject(self.h, _ptr(counts), _counts_dtype(counts), int(counts_packed),
                                                    _ptr(add), _ptr(x), _ptr(bp), subset, nsubsets, _ptr(lik),
                                                    _stream(stream)))
        return bp

    def stage_counts(self, h_counts_subset, stage, subset, nsubsets, stream=None):
        """Copy a pass's host counts to `stage` ahead of em_pass_host, beside the current work."""
        dt = {"float32": _lib.APIRL_F32, "uint32": _lib.APIRL_U32, "uint16": _lib.APIRL_U16}[str(h_counts_subset.dtype)]
        check(self.lib.apirl_stage_counts(self.h, ctypes.c_void_p(h_counts_subset.ctypes.data), dt, _ptr(stage),
                                          subset, nsubsets, _stream(stream)))

    def em_pass_host(self, h_counts_subset, stage, x, bp, sens, subset, nsubsets, h_x_out, h_lik=None,
                     thr_value=0.0, ge=True, stream=None, zimg=None, zero_add=None, wait=True):
        """em_pass (em_pass_sparse when zimg is given) from host counts (packed
        subset, numpy) to a host image; blocks until done, or with wait=False
        returns once queued (apirl_em_pass_host_async: h_x_out / h_lik, which
        should be page-locked, are filled when the stream gets there)."""
        dt = {"float32": _lib.APIRL_F32, "uint32": _lib.APIRL_U32, "uint16": _lib.APIRL_U16}[str(h_counts_subset.dtype)]
        fn = self.lib.apirl_em_pass_host if wait else self.lib.apirl_em_pass_host_async
        check(fn(self.h, ctypes.c_void_p(h_counts_subset.ctypes.data), dt, _ptr(stage),
                                          _ptr(x), _ptr(bp), _ptr(sens), _ptr(zimg), _ptr(zero_add),
                                          float(thr_value), int(ge), subset, nsubsets,
                                          None if h_x_out is None else ctypes.c_void_p(h_x_out.ctypes.data),
                                          None if h_lik is None else ctypes.c_void_p(h_lik.ctypes.data),
                                          _stream(stream)))
        return h_x_out


# ---- iteration hook of the whole-reconstruction drivers -------------------
_ITER_CB = ctypes.CFUNCTYPE(None, ctypes.c_int, ctypes.POINTER(ctypes.c_float), ctypes.c_int64, ctypes.c_void_p)
_iter_hook = None  # the installed ctypes callback, kept alive while installed


def set_iteration_hook(callback=None, interval=0):
    """apirl_set_iteration_hook: osem_3d / mlem_3d / mlem_2d called afterwards
    on this thread call callback(t, image) (numpy copy) after every iteration t
    with t % interval == 0.  No arguments: remove it."""
    global _iter_hook
    lib = _lib.load()
    if callback is None or interval <= 0:
        check(lib.apirl_set_iteration_hook(None, 0, None))
        _iter_hook = None
        return

    def trampoline(t, img, n, user):
        callback(t, np.ctypeslib.as_array(img, shape=(n,)).copy())

    cb = _ITER_CB(trampoline)
    check(lib.apirl_set_iteration_hook(ctypes.cast(cb, ctypes.c_void_p), int(interval), None))
    _iter_hook = cb


# ---- bin-wise / pixel-wise steps (device tensors) -------------------------
def inverse_divide(meas, est, stream=None):
    lib = _lib.load()
    check(lib.apirl_inverse_divide(est.numel(), _ptr(meas), _ptr(est), _stream(stream)))
    return est


def add_bins(add, est, stream=None):
    lib = _lib.load()
    check(lib.apirl_add_bins(est.numel(), _ptr(add), _ptr(est), _stream(stream)))
    return est


def likelihood(est, meas, gt0=False, stream=None):
    import torch
    lib = _lib.load()
    out = torch.zeros(1, dtype=torch.float64, device=est.device)
    check(lib.apirl_likelihood(est.numel(), _ptr(est), _ptr(meas), int(gt0), _ptr(out), _stream(stream)))
    return out


def mlem_threshold(sens, stream=None):
    import torch
    lib = _lib.load()
    out = torch.zeros(1, dtype=torch.float32, device=sens.device)
    check(lib.apirl_mlem_threshold(sens.numel(), _ptr(sens), _ptr(out), _stream(stream)))
    return out


def update_pixels(x, bp, sens, thr=None, thr_value=0.0, ge=True, zero_bp=False, stream=None):
    lib = _lib.load()
    check(lib.apirl_update_pixels(x.numel(), _ptr(x), _ptr(bp), _ptr(sens), _ptr(thr), float(thr_value), int(ge),
                                  int(zero_bp), _stream(stream)))
    return x


def force_positive(x, stream=None):
    lib = _lib.load()
    check(lib.apirl_force_positive(x.numel(), _ptr(x), _stream(stream)))
    return x


# ---- whole reconstructions (host arrays) ----------------------------------
def _np_ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def _sampling_c(sampling):
    """sampling: None (one ray per bin) or (n_samples, n_axial_samples, multiple_lors_per_bin)."""
    if sampling is None:
        return None
    ns, nas, multi = sampling
    return ctypes.byref(_lib.SamplingC(int(ns), int(nas), int(bool(multi))))


def _recon_opts(sampling, sens_in, sens_out, update_positive_sens=False, n_sens_out=0):
    """apirl_recon_options; the ctypes objects are returned with it so they stay alive."""
    smp = None
    if sampling is not None:
        ns, nas, multi = sampling
        smp = _lib.SamplingC(int(ns), int(nas), int(bool(multi)))
    o = _lib.ReconOptionsC(ctypes.pointer(smp) if smp is not None else None,
                           _np_ptr(sens_in) if sens_in is not None else None,
                           _np_ptr(sens_out) if sens_out is not None else None,
                           int(bool(update_positive_sens)), int(n_sens_out))
    return o, smp


def osem_3d(image_geom, sino_geom, meas, init, iters, nsubsets, mult=None, add=None, device=0, sampling=None,
            sens=None, all_sens=False, update_positive_sens=False):
    """OsemSinogram3d::Reconstruct on the GPU.  Returns (image,
    likelihood[iters*nsubsets+1], sensitivity): subset 0's image, or all
    nsubsets images [subset, voxel] with all_sens.  sens: given sensitivity
    images [subset, voxel] instead of A_s^T (mult or 1) (forcePositive applied).
    update_positive_sens: update where sens > 0 (else 0) instead of the
    reference's sens >= 0 (NaN where no ray of a subset reaches a voxel)."""
    lib = _lib.load()
    meas, init, mult, add = _f32(meas), _f32(init), _f32(mult), _f32(add)
    nv = image_geom.n_voxels
    out = np.zeros(nv, np.float32)
    lik = np.zeros(iters * nsubsets + 1, np.float64)
    ig, sc = _img_c(image_geom), _sino3d_c(sino_geom)
    if sens is None and not all_sens and not update_positive_sens:
        sens0 = np.zeros(nv, np.float32)
        check(lib.apirl_osem_3d(ctypes.byref(ig), ctypes.byref(sc), _np_ptr(meas), _np_ptr(mult), _np_ptr(add),
                                _np_ptr(init), iters, nsubsets, device, _np_ptr(out), _np_ptr(lik), _np_ptr(sens0),
                                _sampling_c(sampling)))
        return out, lik, sens0
    sens_in = None if sens is None else np.ascontiguousarray(sens, np.float32).reshape(-1)
    if sens_in is not None and sens_in.size != nsubsets * nv:
        raise ValueError("sens must hold nsubsets images")
    # all subsets' sensitivity images back only when asked for (a C2-size job's are 446 MB)
    sens_out = np.zeros((nsubsets if all_sens else 1, nv), np.float32)
    opts, _keep = _recon_opts(sampling, sens_in, sens_out, update_positive_sens, 0 if all_sens else 1)
    check(lib.apirl_osem_3d_ex(ctypes.byref(ig), ctypes.byref(sc), _np_ptr(meas), _np_ptr(mult), _np_ptr(add),
                               _np_ptr(init), iters, nsubsets, device, _np_ptr(out), _np_ptr(lik), ctypes.byref(opts)))
    return out, lik, (sens_out if all_sens else sens_out[0].copy())


def mlem_3d(image_geom, sino_geom, meas, init, iters, mult=None, add=None, device=0, sampling=None, sens=None):
    """MlemSinogram3d::Reconstruct on the GPU; sens: a given sensitivity image."""
    lib = _lib.load()
    meas, init, mult, add = _f32(meas), _f32(init), _f32(mult), _f32(add)
    out = np.zeros(image_geom.n_voxels, np.float32)
    lik = np.zeros(iters + 1, np.float64)
    sens_out = np.zeros(image_geom.n_voxels, np.float32)
    ig, sc = _img_c(image_geom), _sino3d_c(sino_geom)
    sens_in = None if sens is None else np.ascontiguousarray(sens, np.float32).reshape(-1)
    opts, _keep = _recon_opts(sampling, sens_in, sens_out)
    check(lib.apirl_mlem_3d_ex(ctypes.byref(ig), ctypes.byref(sc), _np_ptr(meas), _np_ptr(mult), _np_ptr(add),
                               _np_ptr(init), iters, device, _np_ptr(out), _np_ptr(lik), ctypes.byref(opts)))
    return out, lik, sens_out


def mlem_2d(image_geom, sino_geom, meas, init, iters, mult=None, add=None, device=0, sens=None):
    """Mlem2d::Reconstruct on the GPU; sens: a given sensitivity image."""
    lib = _lib.load()
    meas, init, mult, add = _f32(meas), _f32(init), _f32(mult), _f32(add)
    out = np.zeros(image_geom.n_voxels, np.float32)
    lik = np.zeros(iters + 1, np.float64)
    sens_out = np.zeros(image_geom.n_voxels, np.float32)
    ig, sc = _img_c(image_geom), _sino2d_c(sino_geom)
    sens_in = None if sens is None else np.ascontiguousarray(sens, np.float32).reshape(-1)
    opts, _keep = _recon_opts(None, sens_in, sens_out)
    check(lib.apirl_mlem_2d_ex(ctypes.byref(ig), ctypes.byref(sc), _np_ptr(meas), _np_ptr(mult), _np_ptr(add),
                               _np_ptr(init), iters, device, _np_ptr(out), _np_ptr(lik), ctypes.byref(opts)))
    return out, lik, sens_out
