// Whole reconstructions with host buffers: the MLEM / OSEM drivers of the
// reference (recon/src/Mlem2d.cpp, MlemSinogram3d.cpp, OsemSinogram3d.cpp)
// on device-resident state.  Each EM pass is captured once as a CUDA graph
// (fused projection/ratio/backprojection kernel, likelihood sum, pixel update)
// and replayed every iteration.
#include <cuda_runtime.h>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>
#include "internal.h"
#include "../../include/apirl_b200.h"

using apirl::SubsetSel;

namespace {

// Small RAII set for device buffers, graphs and the stream of one driver call.
struct Res {
  std::vector<void*> bufs;
  std::vector<cudaGraphExec_t> execs;
  std::vector<cudaGraph_t> graphs;
  cudaStream_t st = nullptr;
  apirl_projector* p = nullptr;
  ~Res() {
    if (st) cudaStreamSynchronize(st);
    for (auto e : execs) cudaGraphExecDestroy(e);
    for (auto g : graphs) cudaGraphDestroy(g);
    for (void* b : bufs) cudaFree(b);
    if (st) cudaStreamDestroy(st);
    if (p) apirl_projector_destroy(p);
  }
  template <typename T> cudaError_t alloc(T** ptr, size_t n) {
    cudaError_t e = cudaMalloc((void**)ptr, n * sizeof(T));
    if (e == cudaSuccess) bufs.push_back(*ptr);
    return e;
  }
};

apirl_status set_err(apirl_status code, const char* what, cudaError_t e) {
  char buf[256];
  snprintf(buf, sizeof buf, "%s: %s", what, e == cudaSuccess ? "invalid argument" : cudaGetErrorString(e));
  return apirl_internal_fail(code, buf);
}

#define DK(call)                                                                                \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      return set_err(e_ == cudaErrorMemoryAllocation ? APIRL_ERR_OOM : APIRL_ERR_CUDA, #call, e_); \
  } while (0)
#define DS(call)                          \
  do {                                    \
    apirl_status s_ = (call);             \
    if (s_ != APIRL_OK) return s_;        \
  } while (0)

// One EM pass (fused kernel + update) recorded into a graph on `st`.
// d_zimg set: the sparse pass (apirl_em_pass_sparse) with that zero-count image.
apirl_status capture_pass(Res& r, apirl_projector* p, const float* d_meas, const float* d_add, float* d_x, float* d_bp,
                          const float* d_sens, const float* d_thr, float thr, int ge, int subset, int nsub,
                          double* d_lik_slot, const float* d_zimg = nullptr, const double* d_zero_add = nullptr) {
  cudaGraph_t g = nullptr;
  DK(cudaStreamBeginCapture(r.st, cudaStreamCaptureModeThreadLocal));
  apirl_status s = d_zimg ? apirl_em_pass_sparse(p, d_meas, APIRL_F32, 0, d_add, d_x, d_bp, d_sens, d_zimg,
                                                 d_zero_add, d_thr, thr, ge, subset, nsub, d_lik_slot, r.st)
                          : apirl_em_pass(p, d_meas, APIRL_F32, 0, d_add, d_x, d_bp, d_sens, d_thr, thr, ge, subset,
                                          nsub, d_lik_slot, r.st);
  cudaError_t e = cudaStreamEndCapture(r.st, &g);
  if (s != APIRL_OK) { if (g) cudaGraphDestroy(g); return s; }
  DK(e);
  r.graphs.push_back(g);
  cudaGraphExec_t ex = nullptr;
  DK(cudaGraphInstantiate(&ex, g, 0));
  r.execs.push_back(ex);
  return APIRL_OK;
}

// The drivers walk only bins with counts (the sparse pass) when the job runs
// at least four passes per subset: a zero-count image (a scatter over the
// zero-count bins) costs about three passes' worth of the forward walks it
// saves (measured on the 256x256x81 / 1261-sinogram job: 2.7 ms per image,
// 0.9 ms saved per pass).
bool use_sparse(const apirl_projector* p, int passes_per_subset) {
  return passes_per_subset >= 4 && p->is3d && !p->t.lor_s && !p->pg.enabled;
}

// With neither a multiplicative nor an additive term, and sensitivities the
// driver computed, each sensitivity image is A_s^T 1 = G_s, the geometry
// image of the sparse pass (APIRL_SPARSE_GEOMETRY): the passes then walk only
// bins with counts at no set-up cost, for any number of passes.
bool use_geometry_sparse(const apirl_projector* p, const float* h_mult, const float* h_add, const float* h_sens_in) {
  return !h_mult && !h_add && !h_sens_in && p->is3d && !p->t.lor_s && !p->pg.enabled;
}

// With a multiplicative term (and no additive one), the sensitivity A_s^T a
// and the geometry image G_s = A_s^T 1 come out of one set of walks
// (apirl::backproject_sino_and_ones): the passes are then the geometry sparse
// pass with G_s beside the sensitivity.
bool use_geometry_mult(const apirl_projector* p, const float* h_mult, const float* h_add, const float* h_sens_in) {
  return h_mult && !h_add && !h_sens_in && p->is3d && !p->t.lor_s && !p->pg.enabled;
}

// Zero-count images and their additive sums of `nsub` subsets of d_meas.
apirl_status zero_images(Res& r, apirl_projector* p, const float* d_meas, const float* d_add, int nsub, int n_proj,
                         float* d_zimg, double* d_zero_add) {
  const int64_t nv = (int64_t)p->g.nx * p->g.ny * p->g.nz;
  DK(cudaMemsetAsync(d_zimg, 0, (size_t)nv * nsub * sizeof(float), r.st));
  for (int s = 0; s < nsub; s++) {
    SubsetSel ss;
    ss.subset = nsub > 1 ? s : -1; ss.nsub = nsub; ss.nk = apirl::subset_nproj(n_proj, ss.subset, nsub);
    DK(apirl::launch_zero_bins(p->g, p->t, ss, d_meas, APIRL_F32, 0, d_add, d_zimg + nv * s, p->d_partials,
                               d_zero_add + s, r.st, p->dual_layout ? p->pad : apirl::PadBuffers()));
  }
  return APIRL_OK;
}

// The calling thread's iteration hook (apirl_set_iteration_hook).
struct IterationHook {
  apirl_iteration_cb cb = nullptr;
  int interval = 0;
  void* user = nullptr;
};
thread_local IterationHook g_hook;

// After iteration t: when the hook asks for it, the image comes to the host
// (the stream's work so far finished) and goes to the callback.
apirl_status iteration_done(Res& r, int t, const float* d_x, int64_t nv, std::vector<float>& h_tmp) {
  if (!g_hook.cb || g_hook.interval <= 0 || t % g_hook.interval != 0) return APIRL_OK;
  h_tmp.resize((size_t)nv);
  DK(cudaMemcpyAsync(h_tmp.data(), d_x, nv * sizeof(float), cudaMemcpyDeviceToHost, r.st));
  DK(cudaStreamSynchronize(r.st));
  g_hook.cb(t, h_tmp.data(), nv, g_hook.user);
  return APIRL_OK;
}

}  // namespace

extern "C" {

apirl_status apirl_set_iteration_hook(apirl_iteration_cb cb, int interval, void* user) {
  if (interval < 0) return set_err(APIRL_ERR_INVALID, "iteration hook interval must be >= 0", cudaSuccess);
  g_hook.cb = cb;
  g_hook.interval = interval;
  g_hook.user = user;
  return APIRL_OK;
}

}  // extern "C"

namespace {

// h_sens_in: nsubsets given sensitivity images (or NULL: computed);
// h_sens_out: receives the first n_sens_out of them.
apirl_status osem_3d(const apirl_image_geom* img, const apirl_sino3d_geom* sino, const float* h_meas,
                     const float* h_mult, const float* h_add, const float* h_init, int iters, int nsubsets,
                     int device, float* h_out, double* h_lik, const float* h_sens_in, float* h_sens_out,
                     int n_sens_out, const apirl_sampling* sampling, int update_positive_sens = 0) {
  if (!h_meas || !h_init || !h_out || iters < 0 || nsubsets <= 0)
    return set_err(APIRL_ERR_INVALID, "apirl_osem_3d arguments", cudaSuccess);
  Res r;
  DS(apirl_projector_create_3d(img, sino, device, &r.p));
  if (sampling)
    DS(apirl_projector_set_sampling(r.p, sampling->n_samples, sampling->n_axial_samples,
                                    sampling->multiple_lors_per_bin));
  int prev = 0;
  cudaGetDevice(&prev);
  DK(cudaSetDevice(device));
  struct Restore { int d; ~Restore() { cudaSetDevice(d); } } restore{prev};
  apirl_projector* p = r.p;
  if (nsubsets > sino->n_proj) return set_err(APIRL_ERR_INVALID, "more subsets than angles", cudaSuccess);
  DK(cudaStreamCreateWithFlags(&r.st, cudaStreamNonBlocking));
  const int64_t nb = apirl_projector_num_bins(p, -1, 1);
  const int64_t nv = (int64_t)img->nx * img->ny * img->nz;
  float *d_meas, *d_mult = nullptr, *d_add = nullptr, *d_x, *d_bp, *d_sens;
  double* d_lik;
  DK(r.alloc(&d_meas, nb));
  if (h_mult) DK(r.alloc(&d_mult, nb));
  if (h_add) DK(r.alloc(&d_add, nb));
  DK(r.alloc(&d_x, nv));
  DK(r.alloc(&d_bp, nv));
  DK(r.alloc(&d_sens, nv * nsubsets));
  DK(r.alloc(&d_lik, (size_t)iters * nsubsets + 1 + nsubsets));
  double* d_slot = d_lik + (size_t)iters * nsubsets + 1;
  DK(cudaMemcpyAsync(d_meas, h_meas, nb * sizeof(float), cudaMemcpyHostToDevice, r.st));
  if (h_mult) DK(cudaMemcpyAsync(d_mult, h_mult, nb * sizeof(float), cudaMemcpyHostToDevice, r.st));
  if (h_add) DK(cudaMemcpyAsync(d_add, h_add, nb * sizeof(float), cudaMemcpyHostToDevice, r.st));
  DK(cudaMemcpyAsync(d_x, h_init, nv * sizeof(float), cudaMemcpyHostToDevice, r.st));
  DK(cudaMemsetAsync(d_bp, 0, nv * sizeof(float), r.st));
  DK(cudaMemsetAsync(d_sens, 0, nv * nsubsets * sizeof(float), r.st));
  float* d_geom = nullptr;
  if (use_geometry_mult(p, h_mult, h_add, h_sens_in)) {
    DK(r.alloc(&d_geom, nv * nsubsets));
    DK(cudaMemsetAsync(d_geom, 0, nv * nsubsets * sizeof(float), r.st));
  }
  // Per-subset sensitivity: A_s^T (mult or 1), or the given images, then
  // forcePositive (OsemSinogram3d.cpp:84-116, :327-346).
  for (int s = 0; s < nsubsets; s++) {
    if (h_sens_in) {
      DK(cudaMemcpyAsync(d_sens + nv * s, h_sens_in + nv * s, nv * sizeof(float), cudaMemcpyHostToDevice, r.st));
    } else {
      SubsetSel ss;
      ss.subset = s; ss.nsub = nsubsets; ss.nk = apirl::subset_nproj(sino->n_proj, s, nsubsets);
      if (d_geom)
        DS(apirl::backproject_sino_and_ones(p, ss, d_mult, 1, d_sens + nv * s, d_geom + nv * s, r.st));
      else
        DK(apirl::backproject_sino(p, ss, d_mult, d_mult ? 1 : 2, d_sens + nv * s, r.st));
    }
    DK(apirl::launch_force_positive(nv, d_sens + nv * s, r.st));
  }
  float* d_zimg = nullptr;
  double* d_zadd = nullptr;
  if (use_geometry_sparse(p, h_mult, h_add, h_sens_in) || d_geom) {
    DS(apirl_projector_set_option(p, APIRL_OPT_SPARSE_IMAGE, APIRL_SPARSE_GEOMETRY));
    d_zimg = d_geom ? d_geom : d_sens;
  } else if (use_sparse(p, iters)) {
    DK(r.alloc(&d_zimg, nv * nsubsets));
    DK(r.alloc(&d_zadd, nsubsets));
    DS(zero_images(r, p, d_meas, d_add, nsubsets, sino->n_proj, d_zimg, d_zadd));
  }
  // Room for the list of bins with counts, made before the passes are
  // captured (subset 0 has the most angles).
  if (d_zimg) DS(apirl::prepare_nz_list(p, apirl_projector_num_bins(p, nsubsets > 1 ? 0 : -1, nsubsets)));
  for (int s = 0; s < nsubsets; s++)
    DS(capture_pass(r, p, d_meas, d_add, d_x, d_bp, d_sens + nv * s, nullptr, 0.f, update_positive_sens ? 0 : 1, s,
                    nsubsets, d_slot + s,
                    d_zimg ? d_zimg + nv * s : nullptr, d_zadd ? d_zadd + s : nullptr));
  std::vector<float> h_tmp;
  for (int t = 0; t < iters; t++) {
    for (int s = 0; s < nsubsets; s++) {
      DK(cudaGraphLaunch(r.execs[s], r.st));
      DK(cudaMemcpyAsync(d_lik + (size_t)t * nsubsets + s, d_slot + s, sizeof(double), cudaMemcpyDeviceToDevice,
                         r.st));
    }
    DS(iteration_done(r, t, d_x, nv, h_tmp));
  }
  // Final likelihood on the whole-sinogram projection of the result (:291-293).
  SubsetSel all;
  all.subset = -1; all.nsub = 1; all.nk = sino->n_proj;
  DK(apirl::launch_em_pass(p->g, p->t, all, d_meas, APIRL_F32, 0, d_add, d_x, d_bp, 0, 0, p->d_partials,
                           d_lik + (size_t)iters * nsubsets, r.st));
  DK(cudaMemcpyAsync(h_out, d_x, nv * sizeof(float), cudaMemcpyDeviceToHost, r.st));
  if (h_lik) DK(cudaMemcpyAsync(h_lik, d_lik, ((size_t)iters * nsubsets + 1) * sizeof(double), cudaMemcpyDeviceToHost, r.st));
  if (h_sens_out && n_sens_out > 0)
    DK(cudaMemcpyAsync(h_sens_out, d_sens, nv * (n_sens_out < nsubsets ? n_sens_out : nsubsets) * sizeof(float),
                       cudaMemcpyDeviceToHost, r.st));
  DK(cudaStreamSynchronize(r.st));
  return APIRL_OK;
}

// h_sens_in: the given sensitivity image (or NULL: computed).
apirl_status mlem_3d(const apirl_image_geom* img, const apirl_sino3d_geom* sino, const float* h_meas,
                     const float* h_mult, const float* h_add, const float* h_init, int iters, int device,
                     float* h_out, double* h_lik, const float* h_sens_in, float* h_sens,
                     const apirl_sampling* sampling) {
  if (!h_meas || !h_init || !h_out || iters < 0) return set_err(APIRL_ERR_INVALID, "apirl_mlem_3d arguments", cudaSuccess);
  Res r;
  DS(apirl_projector_create_3d(img, sino, device, &r.p));
  if (sampling)
    DS(apirl_projector_set_sampling(r.p, sampling->n_samples, sampling->n_axial_samples,
                                    sampling->multiple_lors_per_bin));
  int prev = 0;
  cudaGetDevice(&prev);
  DK(cudaSetDevice(device));
  struct Restore { int d; ~Restore() { cudaSetDevice(d); } } restore{prev};
  apirl_projector* p = r.p;
  DK(cudaStreamCreateWithFlags(&r.st, cudaStreamNonBlocking));
  const int64_t nb = apirl_projector_num_bins(p, -1, 1);
  const int64_t nv = (int64_t)img->nx * img->ny * img->nz;
  float *d_meas, *d_mult = nullptr, *d_add = nullptr, *d_x, *d_bp, *d_sens, *d_thr;
  double* d_lik;
  DK(r.alloc(&d_meas, nb));
  if (h_mult) DK(r.alloc(&d_mult, nb));
  if (h_add) DK(r.alloc(&d_add, nb));
  DK(r.alloc(&d_x, nv));
  DK(r.alloc(&d_bp, nv));
  DK(r.alloc(&d_sens, nv));
  DK(r.alloc(&d_thr, 1));
  DK(r.alloc(&d_lik, (size_t)iters + 2));
  DK(cudaMemcpyAsync(d_meas, h_meas, nb * sizeof(float), cudaMemcpyHostToDevice, r.st));
  if (h_mult) DK(cudaMemcpyAsync(d_mult, h_mult, nb * sizeof(float), cudaMemcpyHostToDevice, r.st));
  if (h_add) DK(cudaMemcpyAsync(d_add, h_add, nb * sizeof(float), cudaMemcpyHostToDevice, r.st));
  DK(cudaMemcpyAsync(d_x, h_init, nv * sizeof(float), cudaMemcpyHostToDevice, r.st));
  DK(cudaMemsetAsync(d_bp, 0, nv * sizeof(float), r.st));
  DK(cudaMemsetAsync(d_sens, 0, nv * sizeof(float), r.st));
  SubsetSel all;
  all.subset = -1; all.nsub = 1; all.nk = sino->n_proj;
  // Sensitivity A^T (mult or 1), or the given image (MlemSinogram3d.cpp:132-151).
  float* d_geom = nullptr;
  if (use_geometry_mult(p, h_mult, h_add, h_sens_in)) {
    DK(r.alloc(&d_geom, nv));
    DK(cudaMemsetAsync(d_geom, 0, nv * sizeof(float), r.st));
  }
  if (h_sens_in)
    DK(cudaMemcpyAsync(d_sens, h_sens_in, nv * sizeof(float), cudaMemcpyHostToDevice, r.st));
  else if (d_geom)
    DS(apirl::backproject_sino_and_ones(p, all, d_mult, 1, d_sens, d_geom, r.st));
  else
    DK(apirl::backproject_sino(p, all, d_mult, d_mult ? 1 : 2, d_sens, r.st));
  DS(apirl_mlem_threshold(nv, d_sens, d_thr, r.st));
  double* d_slot = d_lik + iters + 1;
  float* d_zimg = nullptr;
  double* d_zadd = nullptr;
  if (use_geometry_sparse(p, h_mult, h_add, h_sens_in) || d_geom) {
    DS(apirl_projector_set_option(p, APIRL_OPT_SPARSE_IMAGE, APIRL_SPARSE_GEOMETRY));
    d_zimg = d_geom ? d_geom : d_sens;
  } else if (use_sparse(p, iters)) {
    DK(r.alloc(&d_zimg, nv));
    DK(r.alloc(&d_zadd, 1));
    DS(zero_images(r, p, d_meas, d_add, 1, sino->n_proj, d_zimg, d_zadd));
  }
  if (d_zimg) DS(apirl::prepare_nz_list(p, apirl_projector_num_bins(p, -1, 1)));
  DS(capture_pass(r, p, d_meas, d_add, d_x, d_bp, d_sens, d_thr, 0.f, 1, -1, 1, d_slot, d_zimg, d_zadd));
  std::vector<float> h_tmp;
  for (int t = 0; t < iters; t++) {
    DK(cudaGraphLaunch(r.execs[0], r.st));
    DK(cudaMemcpyAsync(d_lik + t, d_slot, sizeof(double), cudaMemcpyDeviceToDevice, r.st));
    DS(iteration_done(r, t, d_x, nv, h_tmp));
  }
  DK(apirl::launch_em_pass(p->g, p->t, all, d_meas, APIRL_F32, 0, d_add, d_x, d_bp, 0, 0, p->d_partials,
                           d_lik + iters, r.st));
  DK(cudaMemcpyAsync(h_out, d_x, nv * sizeof(float), cudaMemcpyDeviceToHost, r.st));
  if (h_lik) DK(cudaMemcpyAsync(h_lik, d_lik, ((size_t)iters + 1) * sizeof(double), cudaMemcpyDeviceToHost, r.st));
  if (h_sens) DK(cudaMemcpyAsync(h_sens, d_sens, nv * sizeof(float), cudaMemcpyDeviceToHost, r.st));
  DK(cudaStreamSynchronize(r.st));
  return APIRL_OK;
}

apirl_status mlem_2d(const apirl_image_geom* img, const apirl_sino2d_geom* sino, const float* h_meas,
                     const float* h_mult, const float* h_add, const float* h_init, int iters, int device,
                     float* h_out, double* h_lik, const float* h_sens_in, float* h_sens) {
  if (!h_meas || !h_init || !h_out || iters < 0) return set_err(APIRL_ERR_INVALID, "apirl_mlem_2d arguments", cudaSuccess);
  Res r;
  DS(apirl_projector_create_2d(img, sino, device, &r.p));
  int prev = 0;
  cudaGetDevice(&prev);
  DK(cudaSetDevice(device));
  struct Restore { int d; ~Restore() { cudaSetDevice(d); } } restore{prev};
  apirl_projector* p = r.p;
  DK(cudaStreamCreateWithFlags(&r.st, cudaStreamNonBlocking));
  const int64_t nb = apirl_projector_num_bins(p, -1, 1);
  const int64_t nv = (int64_t)img->nx * img->ny * img->nz;
  float *d_meas, *d_mult = nullptr, *d_add = nullptr, *d_x, *d_xprev, *d_bp, *d_sens, *d_thr;
  double* d_lik;
  DK(r.alloc(&d_meas, nb));
  if (h_mult) DK(r.alloc(&d_mult, nb));
  if (h_add) DK(r.alloc(&d_add, nb));
  DK(r.alloc(&d_x, nv));
  DK(r.alloc(&d_xprev, nv));
  DK(r.alloc(&d_bp, nv));
  DK(r.alloc(&d_sens, nv));
  DK(r.alloc(&d_thr, 1));
  DK(r.alloc(&d_lik, (size_t)iters + 2));
  DK(cudaMemcpyAsync(d_meas, h_meas, nb * sizeof(float), cudaMemcpyHostToDevice, r.st));
  if (h_mult) DK(cudaMemcpyAsync(d_mult, h_mult, nb * sizeof(float), cudaMemcpyHostToDevice, r.st));
  if (h_add) DK(cudaMemcpyAsync(d_add, h_add, nb * sizeof(float), cudaMemcpyHostToDevice, r.st));
  DK(cudaMemcpyAsync(d_x, h_init, nv * sizeof(float), cudaMemcpyHostToDevice, r.st));
  DK(cudaMemsetAsync(d_bp, 0, nv * sizeof(float), r.st));
  DK(cudaMemsetAsync(d_sens, 0, nv * sizeof(float), r.st));
  SubsetSel all;
  all.subset = -1; all.nsub = 1; all.nk = sino->n_proj;
  // Sensitivity A^T (mult or 1), or the given image (Mlem2d.cpp:95-112).
  if (h_sens_in)
    DK(cudaMemcpyAsync(d_sens, h_sens_in, nv * sizeof(float), cudaMemcpyHostToDevice, r.st));
  else
    DK(apirl::launch_backproject(p->g, p->t, all, d_mult, d_mult ? 1 : 2, nullptr, 0, d_sens, r.st));
  DS(apirl_mlem_threshold(nv, d_sens, d_thr, r.st));
  double* d_slot = d_lik + iters + 1;
  DS(capture_pass(r, p, d_meas, d_add, d_x, d_bp, d_sens, d_thr, 0.f, 0, -1, 1, d_slot));
  std::vector<float> h_tmp;
  for (int t = 0; t < iters; t++) {
    if (t == iters - 1) DK(cudaMemcpyAsync(d_xprev, d_x, nv * sizeof(float), cudaMemcpyDeviceToDevice, r.st));
    DK(cudaGraphLaunch(r.execs[0], r.st));
    DK(cudaMemcpyAsync(d_lik + t, d_slot, sizeof(double), cudaMemcpyDeviceToDevice, r.st));
    DS(iteration_done(r, t, d_x, nv, h_tmp));
  }
  // Mlem2d.cpp:228 evaluates the last value on the ratio sinogram of the last
  // iteration: recompute that ratio from the image before the last update.
  if (iters > 0)
    DK(apirl::launch_em_pass(p->g, p->t, all, d_meas, APIRL_F32, 0, d_add, d_xprev, d_bp, 0, 2, p->d_partials,
                             d_lik + iters, r.st));
  else
    DK(cudaMemsetAsync(d_lik, 0, sizeof(double), r.st));
  DK(cudaMemcpyAsync(h_out, d_x, nv * sizeof(float), cudaMemcpyDeviceToHost, r.st));
  if (h_lik) DK(cudaMemcpyAsync(h_lik, d_lik, ((size_t)iters + 1) * sizeof(double), cudaMemcpyDeviceToHost, r.st));
  if (h_sens) DK(cudaMemcpyAsync(h_sens, d_sens, nv * sizeof(float), cudaMemcpyDeviceToHost, r.st));
  DK(cudaStreamSynchronize(r.st));
  return APIRL_OK;
}

}  // namespace

extern "C" {

apirl_status apirl_osem_3d(const apirl_image_geom* img, const apirl_sino3d_geom* sino, const float* h_meas,
                           const float* h_mult, const float* h_add, const float* h_init, int iters, int nsubsets,
                           int device, float* h_out, double* h_lik, float* h_sens0, const apirl_sampling* sampling) {
  return osem_3d(img, sino, h_meas, h_mult, h_add, h_init, iters, nsubsets, device, h_out, h_lik, nullptr, h_sens0,
                 1, sampling);
}

apirl_status apirl_osem_3d_ex(const apirl_image_geom* img, const apirl_sino3d_geom* sino, const float* h_meas,
                              const float* h_mult, const float* h_add, const float* h_init, int iters, int nsubsets,
                              int device, float* h_out, double* h_lik, const apirl_recon_options* opts) {
  const apirl_recon_options o = opts ? *opts : apirl_recon_options{nullptr, nullptr, nullptr, 0, 0};
  const int n_out = o.n_sens_out > 0 && o.n_sens_out < nsubsets ? o.n_sens_out : nsubsets;
  return osem_3d(img, sino, h_meas, h_mult, h_add, h_init, iters, nsubsets, device, h_out, h_lik, o.h_sens_in,
                 o.h_sens_out, n_out, o.sampling, o.update_positive_sens);
}

apirl_status apirl_mlem_3d(const apirl_image_geom* img, const apirl_sino3d_geom* sino, const float* h_meas,
                           const float* h_mult, const float* h_add, const float* h_init, int iters, int device,
                           float* h_out, double* h_lik, float* h_sens, const apirl_sampling* sampling) {
  return mlem_3d(img, sino, h_meas, h_mult, h_add, h_init, iters, device, h_out, h_lik, nullptr, h_sens, sampling);
}

apirl_status apirl_mlem_3d_ex(const apirl_image_geom* img, const apirl_sino3d_geom* sino, const float* h_meas,
                              const float* h_mult, const float* h_add, const float* h_init, int iters, int device,
                              float* h_out, double* h_lik, const apirl_recon_options* opts) {
  const apirl_recon_options o = opts ? *opts : apirl_recon_options{nullptr, nullptr, nullptr, 0, 0};
  return mlem_3d(img, sino, h_meas, h_mult, h_add, h_init, iters, device, h_out, h_lik, o.h_sens_in, o.h_sens_out,
                 o.sampling);
}

apirl_status apirl_mlem_2d(const apirl_image_geom* img, const apirl_sino2d_geom* sino, const float* h_meas,
                           const float* h_mult, const float* h_add, const float* h_init, int iters, int device,
                           float* h_out, double* h_lik, float* h_sens) {
  return mlem_2d(img, sino, h_meas, h_mult, h_add, h_init, iters, device, h_out, h_lik, nullptr, h_sens);
}

apirl_status apirl_mlem_2d_ex(const apirl_image_geom* img, const apirl_sino2d_geom* sino, const float* h_meas,
                              const float* h_mult, const float* h_add, const float* h_init, int iters, int device,
                              float* h_out, double* h_lik, const apirl_recon_options* opts) {
  const apirl_recon_options o = opts ? *opts : apirl_recon_options{nullptr, nullptr, nullptr, 0, 0};
  if (o.sampling) return set_err(APIRL_ERR_NOT_SUPPORTED, "2D reconstructions walk one ray per bin", cudaSuccess);
  return mlem_2d(img, sino, h_meas, h_mult, h_add, h_init, iters, device, h_out, h_lik, o.h_sens_in, o.h_sens_out);
}

}  // extern "C"
