// The C ABI declared in include/apirl_b200.h: projector objects, argument
// checks, error reporting, and the MLEM / OSEM drivers.
#include <cuda_runtime.h>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <climits>

#include "internal.h"
#include "../../include/apirl_b200.h"

using apirl::HostTables;
using apirl::ImgGeom;
using apirl::LorTable;
using apirl::SubsetSel;

namespace {

thread_local std::string g_err;

}  // namespace

apirl_status apirl_internal_fail(apirl_status code, const char* msg) {
  g_err = msg;
  return code;
}

// A CUDA error left pending by an earlier launch (this library's or the
// caller's) is reported by the next entry point instead of being discarded:
// that call returns APIRL_ERR_CUDA naming the error and does no work.
// Reading the error resets a non-sticky one, as cudaGetLastError() does for
// any caller, so the call after it runs normally.
apirl_status apirl_internal_pending(void) {
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return APIRL_OK;
  char buf[384];
  snprintf(buf, sizeof buf, "a CUDA error was pending before this call (left by an earlier launch): %s: %s",
           cudaGetErrorName(e), cudaGetErrorString(e));
  g_err = buf;
  return e == cudaErrorMemoryAllocation ? APIRL_ERR_OOM : APIRL_ERR_CUDA;
}

namespace {

apirl_status fail(apirl_status code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

apirl_status cuda_fail(cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation) return fail(APIRL_ERR_OOM, "%s: %s", what, cudaGetErrorString(e));
  return fail(APIRL_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call)                                                  \
  do {                                                            \
    cudaError_t e_ = (call);                                      \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);           \
  } while (0)

// Makes `dev` current for the scope and restores the caller's device after.
struct DeviceScope {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit DeviceScope(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) err = cudaSetDevice(dev);
  }
  ~DeviceScope() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// Also refuses to run over an error pending from an earlier launch
// (apirl_internal_pending), so that the cudaGetLastError() after each of our
// launches reports that launch only.
#define DEVICE_SCOPE(dev)                                                       \
  DeviceScope scope_(dev);                                                      \
  if (scope_.err != cudaSuccess) return cuda_fail(scope_.err, "cudaSetDevice"); \
  if (apirl_status pend_ = apirl_internal_pending()) return pend_
#define NO_PENDING()                                         \
  do {                                                       \
    if (apirl_status pend_ = apirl_internal_pending()) return pend_; \
  } while (0)

// The accumulation form set on a projector applies to its padded passes; a
// projector that no longer takes them (FP64 walk, sampling, dual layout off)
// refuses to backproject with another form than plain atomics.
apirl_status check_acc(const apirl_projector* p) {
  const bool dual = p->is3d && p->dual_layout && !p->pg.enabled && p->pad.pA && !p->t.lor_s;
  if (p->pad.acc != APIRL_ACC_ATOMIC && !dual)
    return fail(APIRL_ERR_NOT_SUPPORTED, "the accumulation form needs the padded 3D layouts");
  return APIRL_OK;
}

bool valid_img(const apirl_image_geom* g) {
  return g && g->nx > 0 && g->ny > 0 && g->nz > 0 && g->dx > 0 && g->dy > 0 && g->dz > 0 &&
         (int64_t)g->nx * g->ny * g->nz < (int64_t)1 << 31;
}

// Bounds the length of every Siddon walk: a LOR spans at most the scanner
// diameter, so it records at most about 2 R / d segments per axis.  Geometries
// that would give walks of more than ~1e5 segments per axis are rejected.
bool walk_bounded(const apirl_image_geom* g, float r_scanner, float axial) {
  const float d = fminf(g->dx, fminf(g->dy, g->dz));
  const float span = fmaxf(2.f * r_scanner, axial);
  return span / d < 1.0e5f && (float)g->nx * g->dx < 1.0e6f && (float)g->nz * g->dz < 1.0e6f;
}

SubsetSel make_subset(const apirl_projector* p, int subset, int nsub) {
  SubsetSel s;
  s.subset = subset < 0 ? -1 : subset;
  s.nsub = subset < 0 ? 1 : nsub;
  s.nk = apirl::subset_nproj(p->t.n_proj, s.subset, s.nsub);
  return s;
}

apirl_status check_subset(const apirl_projector* p, int subset, int nsub) {
  if (!p) return fail(APIRL_ERR_INVALID, "null projector");
  if (subset >= 0 && (nsub <= 0 || subset >= nsub || nsub > p->t.n_proj))
    return fail(APIRL_ERR_INVALID, "subset %d of %d is out of range (%d angles)", subset, nsub, p->t.n_proj);
  return APIRL_OK;
}

// The padded two-layout buffers of the fused 3D pass, allocated with the
// projector so that no pass allocates (passes may be captured into CUDA
// graphs).  Volumes whose padded size does not fit a 32-bit index keep the
// single unpadded layout.
apirl_status alloc_pad(apirl_projector* p) {
  if (p->pad.pA) return APIRL_OK;
  const int64_t pv = (int64_t)(p->g.nx + 2 * apirl::kPad) * (p->g.ny + 2 * apirl::kPad) * (p->g.nz + 2 * apirl::kPad);
  if (pv > INT_MAX) return APIRL_OK;
  // One block for the four images (an L2 access policy window can then
  // cover them all: APIRL_OPT_L2_PERSIST).
  float* b = nullptr;
  cudaError_t e = cudaMalloc(&b, 4 * pv * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(b, 0, 4 * pv * sizeof(float));
  if (e != cudaSuccess) {
    cudaFree(b);
    return cuda_fail(e, "padded layout buffers");
  }
  p->pad.pA = b;
  p->pad.pT = b + pv;
  p->pad.bA = b + 2 * pv;
  p->pad.bT = b + 3 * pv;
  p->pad.lim = (unsigned)pv;
  return APIRL_OK;
}

apirl_status finish_create(apirl_projector* p, apirl_projector** out) {
  const size_t nl = p->host.lor.size() / 4;
  CK(cudaMalloc(&p->d_lor, nl * sizeof(float4)));
  CK(cudaMemcpy(p->d_lor, p->host.lor.data(), nl * sizeof(float4), cudaMemcpyHostToDevice));
  CK(cudaMalloc(&p->d_z, p->host.z.size() / 2 * sizeof(float2)));
  CK(cudaMemcpy(p->d_z, p->host.z.data(), p->host.z.size() * sizeof(float), cudaMemcpyHostToDevice));
  CK(cudaMalloc(&p->d_ok, p->host.ok.size()));
  CK(cudaMemcpy(p->d_ok, p->host.ok.data(), p->host.ok.size(), cudaMemcpyHostToDevice));
  p->t.lor = p->d_lor;
  p->t.z = p->d_z;
  p->t.ok = p->d_ok;
  SubsetSel all = make_subset(p, -1, 1);
  p->n_partials = apirl::em_pass_blocks(p->t, all);
  const int64_t lb = apirl::likelihood_blocks((int64_t)p->t.n_sinos * p->t.n_proj * p->t.n_r);
  if (lb > p->n_partials) p->n_partials = lb;
  CK(cudaMalloc(&p->d_partials, p->n_partials * sizeof(double)));
  CK(cudaMalloc(&p->d_minmax, 2 * sizeof(unsigned)));
  CK(cudaMalloc(&p->d_scalars, 8 * sizeof(double)));
  CK(cudaMalloc(&p->d_chunk, sizeof(unsigned long long)));
  if (p->is3d) CK(apirl::prepare_em_kernels(p->em_block));
  if (p->is3d && p->dual_layout) {
    const apirl_status st = alloc_pad(p);
    if (st) return st;
  }
  *out = p;
  return APIRL_OK;
}

}  // namespace

namespace apirl {
// The host half of a 3D projector: checks the image and sinogram geometry
// (cylindrical or Siemens mMR) and builds the LOR and end-point tables into p
// (g, host, t's sizes, the geometry as given), touching no device.
apirl_status setup_3d(const apirl_image_geom* img, const apirl_sino3d_geom* sino, apirl_projector* p) {
  if (!sino) return fail(APIRL_ERR_INVALID, "invalid 3D sinogram geometry");
  if (sino->scanner != APIRL_SCANNER_CYLINDRICAL && sino->scanner != APIRL_SCANNER_MMR)
    return fail(APIRL_ERR_INVALID, "unknown scanner %d", sino->scanner);
  const bool mmr = sino->scanner == APIRL_SCANNER_MMR;
  if (!valid_img(img)) return fail(APIRL_ERR_INVALID, "invalid image geometry");
  if (mmr) {
    if (sino->n_proj < 2 || sino->n_r <= 0 || sino->n_rings <= 0 || sino->n_segments <= 0 || !sino->min_ring_diff ||
        !sino->max_ring_diff)
      return fail(APIRL_ERR_INVALID, "invalid mMR sinogram geometry (need n_proj >= 2, n_r, n_rings, segments)");
    if (!walk_bounded(img, apirl::kMmrRadius + apirl::kMmrDoi, apirl::kMmrAxialFov))
      return fail(APIRL_ERR_INVALID, "voxels too small for the scanner size (walks above 1e5 segments)");
  } else {
    if (sino->n_proj <= 0 || sino->n_r <= 0 || sino->n_rings <= 0 || sino->n_segments <= 0 ||
        !sino->min_ring_diff || !sino->max_ring_diff || !(sino->r_fov > 0) || !(sino->axial_fov > 0) ||
        !(sino->r_scanner > sino->r_fov))
      return fail(APIRL_ERR_INVALID, "invalid 3D sinogram geometry");
    if (!walk_bounded(img, sino->r_scanner, sino->axial_fov))
      return fail(APIRL_ERR_INVALID, "voxels too small for the scanner size (walks above 1e5 segments)");
  }
  for (int i = 0; i < sino->n_segments; i++)
    if (sino->min_ring_diff[i] > sino->max_ring_diff[i])
      return fail(APIRL_ERR_INVALID, "segment %d: minimum ring difference above maximum", i);
  p->is3d = 1;
  p->scanner = sino->scanner;
  p->g = make_img_geom(img->nx, img->ny, img->nz, img->dx, img->dy, img->dz);
  const bool built = mmr ? build_tables_mmr(sino->n_proj, sino->n_r, sino->n_rings, sino->n_segments,
                                            sino->min_ring_diff, sino->max_ring_diff, p->host)
                         : build_tables_3d(sino->n_proj, sino->n_r, sino->n_rings, sino->r_fov, sino->axial_fov,
                                           sino->r_scanner, sino->n_segments, sino->min_ring_diff,
                                           sino->max_ring_diff, p->host);
  if (!built) return fail(APIRL_ERR_INVALID, "segment table yields no sinograms");
  p->t.n_proj = sino->n_proj;
  p->t.n_r = sino->n_r;
  p->t.n_sinos = p->host.n_sinos;
  p->t.is3d = 1;
  p->n_rings = sino->n_rings;
  p->r_fov = mmr ? kMmrRFov : sino->r_fov;
  p->axial_fov = mmr ? kMmrAxialFov : sino->axial_fov;
  p->r_scanner = mmr ? kMmrRadius : sino->r_scanner;
  p->min_rd.assign(sino->min_ring_diff, sino->min_ring_diff + sino->n_segments);
  p->max_rd.assign(sino->max_ring_diff, sino->max_ring_diff + sino->n_segments);
  if ((int64_t)p->t.n_sinos * p->t.n_proj * p->t.n_r >= ((int64_t)1 << 40))
    return fail(APIRL_ERR_INVALID, "sinogram too large");
  return APIRL_OK;
}
}  // namespace apirl

extern "C" {

const char* apirl_last_error(void) { return g_err.c_str(); }
const char* apirl_version(void) { return "apirl_b200 0.1 (sm_100a)"; }

apirl_status apirl_lor_table(int n_proj, int n_r, float r_fov, float r_scanner, float* h_lor) {
  if (n_proj <= 0 || n_r <= 0 || !h_lor || !(r_scanner > r_fov)) return fail(APIRL_ERR_INVALID, "bad arguments");
  HostTables t;
  apirl::build_tables_2d(n_proj, n_r, r_fov, r_scanner, t);
  memcpy(h_lor, t.lor.data(), t.lor.size() * sizeof(float));
  return APIRL_OK;
}

int apirl_sino3d_ring_z(const apirl_sino3d_geom* sino, float* h_z) {
  if (!sino || sino->n_rings <= 0 || sino->n_segments <= 0 || !sino->min_ring_diff || !sino->max_ring_diff) {
    fail(APIRL_ERR_INVALID, "invalid 3D sinogram geometry");
    return -1;
  }
  HostTables t;
  const float afov = sino->scanner == APIRL_SCANNER_MMR ? apirl::kMmrAxialFov : sino->axial_fov;
  if (!apirl::build_tables_3d(1, 1, sino->n_rings, 1.f, afov, 2.f, sino->n_segments,
                              sino->min_ring_diff, sino->max_ring_diff, t))
    return 0;
  if (h_z) memcpy(h_z, t.z.data(), t.z.size() * sizeof(float));
  return t.n_sinos;
}

apirl_status apirl_projector_create_2d(const apirl_image_geom* img, const apirl_sino2d_geom* sino, int device,
                                       apirl_projector** out) {
  if (!out) return fail(APIRL_ERR_INVALID, "null output pointer");
  *out = nullptr;
  if (!valid_img(img)) return fail(APIRL_ERR_INVALID, "invalid image geometry");
  if (!sino || sino->n_proj <= 0 || sino->n_r <= 0 || !(sino->r_fov > 0) || !(sino->r_scanner > sino->r_fov))
    return fail(APIRL_ERR_INVALID, "invalid 2D sinogram geometry (need n_proj, n_r > 0 and 0 < r_fov < r_scanner)");
  if (!walk_bounded(img, sino->r_scanner, 0.f))
    return fail(APIRL_ERR_INVALID, "voxels too small for the scanner radius (walks above 1e5 segments)");
  DEVICE_SCOPE(device);
  apirl_projector* p = new apirl_projector;
  p->device = device;
  p->is3d = 0;
  p->g = apirl::make_img_geom(img->nx, img->ny, img->nz, img->dx, img->dy, img->dz);
  apirl::build_tables_2d(sino->n_proj, sino->n_r, sino->r_fov, sino->r_scanner, p->host);
  p->t.n_proj = sino->n_proj;
  p->t.n_r = sino->n_r;
  p->t.n_sinos = 1;
  p->t.is3d = 0;
  apirl_status st = finish_create(p, out);
  if (st != APIRL_OK) { std::string m = g_err; apirl_projector_destroy(p); g_err = m; }
  return st;
}

apirl_status apirl_mmr_lor_table(int n_proj, int n_r, float* h_lor) {
  if (n_proj < 2 || n_r <= 0 || !h_lor) return fail(APIRL_ERR_INVALID, "bad arguments");
  std::vector<float> lor;
  apirl::mmr_lor_table(n_proj, n_r, lor);
  memcpy(h_lor, lor.data(), lor.size() * sizeof(float));
  return APIRL_OK;
}

apirl_status apirl_projector_create_3d_mmr(const apirl_image_geom* img, int n_proj, int n_r, int n_rings,
                                           int n_segments, const int* min_ring_diff, const int* max_ring_diff,
                                           int device, apirl_projector** out) {
  apirl_sino3d_geom sino;
  memset(&sino, 0, sizeof sino);
  sino.n_proj = n_proj;
  sino.n_r = n_r;
  sino.n_rings = n_rings;
  sino.n_segments = n_segments;
  sino.min_ring_diff = min_ring_diff;
  sino.max_ring_diff = max_ring_diff;
  sino.scanner = APIRL_SCANNER_MMR;
  return apirl_projector_create_3d(img, &sino, device, out);
}

apirl_status apirl_projector_create_3d(const apirl_image_geom* img, const apirl_sino3d_geom* sino, int device,
                                       apirl_projector** out) {
  if (!out) return fail(APIRL_ERR_INVALID, "null output pointer");
  *out = nullptr;
  apirl_projector* p = new apirl_projector;
  apirl_status st = apirl::setup_3d(img, sino, p);
  if (st != APIRL_OK) {
    delete p;
    return st;
  }
  {
    DEVICE_SCOPE(device);
    p->device = device;
    st = finish_create(p, out);
  }
  if (st != APIRL_OK) { std::string m = g_err; apirl_projector_destroy(p); g_err = m; }
  return st;
}

void apirl_projector_destroy(apirl_projector* p) {
  if (!p) return;
  DeviceScope scope(p->device);
  if (p->l2_limit_set) cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, p->l2_limit_prev);
  cudaFree(p->d_lor);
  cudaFree(p->d_z);
  cudaFree(p->d_ok);
  cudaFree(p->d_partials);
  cudaFree(p->d_minmax);
  cudaFree(p->d_scalars);
  cudaFree(p->d_chunk);
  cudaFree(p->pad2.bA);
  cudaFree(p->pad2.bT);
  cudaFree(p->nz.list);
  cudaFree(p->nz.tiles);
  cudaFree(p->nz.n_list);
  cudaFree(p->d_lor64);
  cudaFree(p->d_z64);
  for (int k = 0; k < 2; k++) {
    cudaFree(p->d_lor_s[k]);
    cudaFree(p->d_zs[k]);
    cudaFree(p->d_zoff[k]);
  }
  cudaFree(p->pad.pA);  // the block of all four padded images
  cudaFree(p->pad.eA);
  cudaFree(p->pad.eT);
  if (p->ev0) cudaEventDestroy(p->ev0);
  if (p->ev1) cudaEventDestroy(p->ev1);
  if (p->copy_ready) cudaEventDestroy(p->copy_ready);
  for (auto& e : p->staged)
    if (e.done) cudaEventDestroy(e.done);
  if (p->copy_stream) cudaStreamDestroy(p->copy_stream);
  delete p;
}

int64_t apirl_projector_num_bins(const apirl_projector* p, int subset, int nsubsets) {
  if (!p || (subset >= 0 && (nsubsets <= 0 || subset >= nsubsets))) return -1;
  SubsetSel s = make_subset(p, subset, nsubsets);
  return (int64_t)p->t.n_sinos * s.nk * p->t.n_r;
}

int apirl_projector_num_sinograms(const apirl_projector* p) { return p ? p->host.n_sinos : -1; }

apirl_status apirl_projector_tables(const apirl_projector* p, float* h_lor, float* h_z) {
  if (!p) return fail(APIRL_ERR_INVALID, "null projector");
  if (h_lor) memcpy(h_lor, p->host.lor.data(), p->host.lor.size() * sizeof(float));
  if (h_z && p->is3d) memcpy(h_z, p->host.z.data(), p->host.z.size() * sizeof(float));
  return APIRL_OK;
}

apirl_status apirl_projector_set_alpha_precision(apirl_projector* p, int mode) {
  if (!p) return fail(APIRL_ERR_INVALID, "null projector");
  if (mode != APIRL_ALPHA_F32 && mode != APIRL_ALPHA_F64) return fail(APIRL_ERR_INVALID, "unknown alpha mode %d", mode);
  if (mode == APIRL_ALPHA_F64 && !p->is3d)
    return fail(APIRL_ERR_NOT_SUPPORTED, "the FP64-alpha walk is implemented for 3D projectors");
  if (mode == APIRL_ALPHA_F64 && p->scanner != APIRL_SCANNER_CYLINDRICAL)
    return fail(APIRL_ERR_NOT_SUPPORTED, "the FP64-alpha tables are built for the cylindrical scanner");
  if (mode == APIRL_ALPHA_F64 && p->t.lor_s)
    return fail(APIRL_ERR_NOT_SUPPORTED, "the FP64-alpha walk takes one ray per bin (sampling is set)");
  DEVICE_SCOPE(p->device);
  if (mode == APIRL_ALPHA_F64 && !p->d_lor64) {
    std::vector<double> lor, z;
    apirl::build_tables_3d_f64(p->t.n_proj, p->t.n_r, p->n_rings, p->r_fov, p->axial_fov, p->r_scanner,
                               (int)p->min_rd.size(), p->min_rd.data(), p->max_rd.data(), lor, z);
    CK(cudaMalloc(&p->d_lor64, lor.size() * sizeof(double)));
    CK(cudaMemcpy(p->d_lor64, lor.data(), lor.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&p->d_z64, z.size() * sizeof(double)));
    CK(cudaMemcpy(p->d_z64, z.data(), z.size() * sizeof(double), cudaMemcpyHostToDevice));
    p->pg.lor = p->d_lor64;
    p->pg.z = p->d_z64;
    p->pg.nx = p->g.nx; p->pg.ny = p->g.ny; p->pg.nz = p->g.nz;
    p->pg.dx = p->g.dx; p->pg.dy = p->g.dy; p->pg.dz = p->g.dz;
    p->pg.rfov = ((double)p->g.dx * p->g.nx) / 2;
    p->pg.offz = (double)p->g.dz / 2;
  }
  p->alpha_mode = mode;
  p->pg.enabled = mode == APIRL_ALPHA_F64;
  return APIRL_OK;
}

apirl_status apirl_projector_set_sampling(apirl_projector* p, int n_samples, int n_axial_samples,
                                         int multiple_lors_per_bin) {
  if (!p) return fail(APIRL_ERR_INVALID, "null projector");
  if (n_samples < 1 || n_axial_samples < 1 || n_samples > APIRL_MAX_SAMPLES || n_axial_samples > APIRL_MAX_SAMPLES)
    return fail(APIRL_ERR_INVALID, "samples per bin must be 1..%d (got %d radial, %d axial)", APIRL_MAX_SAMPLES,
                n_samples, n_axial_samples);
  const bool plain = n_samples == 1 && n_axial_samples == 1 && !multiple_lors_per_bin;
  if (!p->is3d && !plain)
    return fail(APIRL_ERR_NOT_SUPPORTED, "2D projectors take one ray per bin (the reference's 2D loops ignore "
                                         "the sample counts)");
  if (p->scanner != APIRL_SCANNER_CYLINDRICAL && !plain)
    return fail(APIRL_ERR_NOT_SUPPORTED, "sampled rays are built for the cylindrical scanner");
  if (!plain && p->alpha_mode == APIRL_ALPHA_F64)
    return fail(APIRL_ERR_NOT_SUPPORTED, "sampling is not combined with the FP64-alpha walk");
  if (!plain && p->t.n_r < 2 && (n_samples > 1 || n_axial_samples > 1))
    return fail(APIRL_ERR_INVALID, "oversampling needs at least 2 radial bins (getDeltaR)");
  DEVICE_SCOPE(p->device);
  // Drop any previous sampled tables.
  for (int k = 0; k < 2; k++) {
    cudaFree(p->d_lor_s[k]);
    cudaFree(p->d_zs[k]);
    cudaFree(p->d_zoff[k]);
    p->d_lor_s[k] = nullptr;
    p->d_zs[k] = nullptr;
    p->d_zoff[k] = nullptr;
  }
  p->t.lor_s = nullptr; p->t.zs = nullptr; p->t.zoff = nullptr; p->t.n_rs = 1; p->t.n_as = 1;
  p->t_dab = p->t;
  p->n_samples = 1; p->n_axial_samples = 1; p->multi_lors = 0;
  if (plain) return APIRL_OK;
  LorTable* dst[2] = {&p->t, &p->t_dab};
  for (int k = 0; k < 2; k++) {
    apirl::RayTables rt;
    if (!apirl::build_rays_3d(p->t.n_proj, p->t.n_r, p->n_rings, p->r_fov, p->axial_fov, p->r_scanner,
                              (int)p->min_rd.size(), p->min_rd.data(), p->max_rd.data(), n_samples, n_axial_samples,
                              multiple_lors_per_bin != 0, k == 1, rt))
      return fail(APIRL_ERR_INVALID, "a sampled ray end point is not finite (sample outside the scanner radius)");
    if ((int)rt.zoff.size() != p->t.n_sinos + 1) return fail(APIRL_ERR_INVALID, "ring-pair table mismatch");
    CK(cudaMalloc(&p->d_lor_s[k], rt.lor.size() * sizeof(float)));
    CK(cudaMemcpy(p->d_lor_s[k], rt.lor.data(), rt.lor.size() * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&p->d_zs[k], rt.zs.size() * sizeof(float)));
    CK(cudaMemcpy(p->d_zs[k], rt.zs.data(), rt.zs.size() * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&p->d_zoff[k], rt.zoff.size() * sizeof(int)));
    CK(cudaMemcpy(p->d_zoff[k], rt.zoff.data(), rt.zoff.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  for (int k = 0; k < 2; k++) {
    dst[k]->lor_s = p->d_lor_s[k];
    dst[k]->zs = p->d_zs[k];
    dst[k]->zoff = p->d_zoff[k];
    dst[k]->n_rs = n_samples;
    dst[k]->n_as = n_axial_samples;
  }
  p->n_samples = n_samples;
  p->n_axial_samples = n_axial_samples;
  p->multi_lors = multiple_lors_per_bin != 0;
  return APIRL_OK;
}

apirl_status apirl_projector_set_shard(apirl_projector* p, int first_sinogram, int n_sinograms) {
  if (!p) return fail(APIRL_ERR_INVALID, "null projector");
  const int total = p->host.n_sinos;
  if (first_sinogram < 0 || n_sinograms < 1 || first_sinogram + n_sinograms > total)
    return fail(APIRL_ERR_INVALID, "shard %d + %d outside the %d sinograms", first_sinogram, n_sinograms, total);
  p->t.g0 = first_sinogram;
  p->t.n_sinos = n_sinograms;
  p->t_dab.g0 = first_sinogram;
  p->t_dab.n_sinos = n_sinograms;
  return APIRL_OK;
}

apirl_status apirl_count_steps(apirl_projector* p, int subset, int nsubsets, int32_t* d_steps, void* stream) {
  apirl_status st = check_subset(p, subset, nsubsets);
  if (st) return st;
  if (!d_steps) return fail(APIRL_ERR_INVALID, "null output");
  DEVICE_SCOPE(p->device);
  CK(apirl::launch_count_steps(p->g, p->t, make_subset(p, subset, nsubsets), d_steps, (cudaStream_t)stream));
  return APIRL_OK;
}

apirl_status apirl_project(apirl_projector* p, const float* d_image, float* d_sino, int subset, int nsubsets,
                           void* stream) {
  apirl_status st = check_subset(p, subset, nsubsets);
  if (st) return st;
  if (!d_image || !d_sino) return fail(APIRL_ERR_INVALID, "null image or sinogram");
  DEVICE_SCOPE(p->device);
  CK(apirl::launch_project(p->g, p->t, make_subset(p, subset, nsubsets), d_image, d_sino, (cudaStream_t)stream,
                           p->pg));
  return APIRL_OK;
}

apirl_status apirl_backproject(apirl_projector* p, const float* d_sino, float* d_image, int subset, int nsubsets,
                               void* stream) {
  apirl_status st = check_subset(p, subset, nsubsets);
  if (st) return st;
  if ((st = check_acc(p))) return st;
  if (!d_image || !d_sino) return fail(APIRL_ERR_INVALID, "null image or sinogram");
  DEVICE_SCOPE(p->device);
  CK(apirl::backproject_sino(p, make_subset(p, subset, nsubsets), d_sino, 0, d_image, (cudaStream_t)stream));
  return APIRL_OK;
}

apirl_status apirl_backproject_ones(apirl_projector* p, float* d_image, int subset, int nsubsets, void* stream) {
  apirl_status st = check_subset(p, subset, nsubsets);
  if (st) return st;
  if ((st = check_acc(p))) return st;
  if (!d_image) return fail(APIRL_ERR_INVALID, "null image");
  DEVICE_SCOPE(p->device);
  CK(apirl::backproject_sino(p, make_subset(p, subset, nsubsets), nullptr, 2, d_image, (cudaStream_t)stream));
  return APIRL_OK;
}

apirl_status apirl_backproject_and_ones(apirl_projector* p, const float* d_sino, float* d_image, float* d_ones_image,
                                        int subset, int nsubsets, void* stream) {
  apirl_status st = check_subset(p, subset, nsubsets);
  if (st) return st;
  if (!d_image || !d_sino || !d_ones_image) return fail(APIRL_ERR_INVALID, "null image or sinogram");
  if (d_image == d_ones_image) return fail(APIRL_ERR_INVALID, "the two images must differ");
  DEVICE_SCOPE(p->device);
  return apirl::backproject_sino_and_ones(p, make_subset(p, subset, nsubsets), d_sino, 0, d_image, d_ones_image,
                                          (cudaStream_t)stream);
}

apirl_status apirl_divide_and_backproject(apirl_projector* p, const float* d_meas, const float* d_est,
                                          float* d_image, int subset, int nsubsets, void* stream) {
  apirl_status st = check_subset(p, subset, nsubsets);
  if (st) return st;
  if (!d_image || !d_meas || !d_est) return fail(APIRL_ERR_INVALID, "null image or sinogram");
  DEVICE_SCOPE(p->device);
  CK(apirl::launch_backproject(p->g, p->t_dab.lor_s ? p->t_dab : p->t, make_subset(p, subset, nsubsets), d_meas, 0,
                               d_est, 1, d_image, (cudaStream_t)stream, p->pg));
  return APIRL_OK;
}

apirl_status apirl_generate_acf(apirl_projector* p, const float* d_mu, float* d_acf, int subset, int nsubsets,
                                void* stream) {
  apirl_status st = check_subset(p, subset, nsubsets);
  if (st) return st;
  if (!d_mu || !d_acf) return fail(APIRL_ERR_INVALID, "null image or sinogram");
  DEVICE_SCOPE(p->device);
  SubsetSel ss = make_subset(p, subset, nsubsets);
  const int64_t nb = (int64_t)p->t.n_sinos * ss.nk * p->t.n_r;
  if (!p->is3d) CK(cudaMemsetAsync(d_acf, 0, nb * sizeof(float), (cudaStream_t)stream));
  CK(apirl::launch_project(p->g, p->t, ss, d_mu, d_acf, (cudaStream_t)stream, p->pg));
  CK(apirl::launch_exp_nonzero(nb, d_acf, (cudaStream_t)stream));
  return APIRL_OK;
}

apirl_status apirl_inverse_divide(int64_t n, const float* d_meas, float* d_est, void* stream) {
  if (n < 0 || (n > 0 && (!d_meas || !d_est))) return fail(APIRL_ERR_INVALID, "bad arguments");
  NO_PENDING();
  CK(apirl::launch_inverse_divide(n, d_meas, d_est, (cudaStream_t)stream));
  return APIRL_OK;
}

apirl_status apirl_add_bins(int64_t n, const float* d_add, float* d_est, void* stream) {
  if (n < 0 || (n > 0 && (!d_add || !d_est))) return fail(APIRL_ERR_INVALID, "bad arguments");
  NO_PENDING();
  CK(apirl::launch_add_bins(n, d_add, d_est, (cudaStream_t)stream));
  return APIRL_OK;
}

apirl_status apirl_likelihood(int64_t n, const float* d_est, const float* d_meas, int gt0, double* d_out,
                              void* stream) {
  if (n <= 0 || !d_est || !d_meas || !d_out) return fail(APIRL_ERR_INVALID, "bad arguments");
  NO_PENDING();
  // The per-block partials live in a small allocation owned by this call path.
  const int64_t nb = apirl::likelihood_blocks(n);
  double* part = nullptr;
  CK(cudaMallocAsync(&part, nb * sizeof(double), (cudaStream_t)stream));
  cudaError_t e = apirl::launch_likelihood(n, d_est, d_meas, gt0, part, nb, d_out, (cudaStream_t)stream);
  cudaFreeAsync(part, (cudaStream_t)stream);
  CK(e);
  return APIRL_OK;
}

apirl_status apirl_mlem_threshold(int64_t n, const float* d_sens, float* d_thr, void* stream) {
  if (n <= 0 || !d_sens || !d_thr) return fail(APIRL_ERR_INVALID, "bad arguments");
  NO_PENDING();
  unsigned* mm = nullptr;
  CK(cudaMallocAsync(&mm, 2 * sizeof(unsigned), (cudaStream_t)stream));
  cudaError_t e = apirl::launch_threshold(n, d_sens, mm, d_thr, (cudaStream_t)stream);
  cudaFreeAsync(mm, (cudaStream_t)stream);
  CK(e);
  return APIRL_OK;
}

apirl_status apirl_update_pixels(int64_t n, float* d_x, float* d_bp, const float* d_sens, const float* d_thr,
                                 float thr_value, int ge, int zero_bp, void* stream) {
  if (n < 0 || (n > 0 && (!d_x || !d_bp || !d_sens))) return fail(APIRL_ERR_INVALID, "bad arguments");
  NO_PENDING();
  CK(apirl::launch_update(n, d_x, d_bp, d_sens, d_thr, thr_value, ge, zero_bp, (cudaStream_t)stream));
  return APIRL_OK;
}

apirl_status apirl_force_positive(int64_t n, float* d_x, void* stream) {
  if (n < 0 || (n > 0 && !d_x)) return fail(APIRL_ERR_INVALID, "bad arguments");
  NO_PENDING();
  CK(apirl::launch_force_positive(n, d_x, (cudaStream_t)stream));
  return APIRL_OK;
}

namespace {

bool use_dual(const apirl_projector* p) {
  return p->is3d && p->dual_layout && !p->pg.enabled && p->pad.pA && !p->t.lor_s;
}

// The fused kernel, bracketed by timing events when enabled.
apirl_status fused(apirl_projector* p, SubsetSel ss, const void* d_counts, int dtype, int packed, const float* d_add,
                   const float* d_x, float* d_bp, bool dual, double* d_lik, cudaStream_t s,
                   const float* d_zimg = nullptr, const double* d_zero_add = nullptr) {
  if (p->pad.acc != APIRL_ACC_ATOMIC && !(dual && p->persistent))
    return fail(APIRL_ERR_NOT_SUPPORTED, "the accumulation form needs the persistent pass over the padded layouts");
  if (p->timing) {
    if (!p->ev0) {
      CK(cudaEventCreate(&p->ev0));
      CK(cudaEventCreate(&p->ev1));
    }
    CK(cudaEventRecord(p->ev0, s));
  }
  CK(apirl::launch_em_pass(p->g, p->t, ss, d_counts, dtype, packed, d_add, d_x, d_bp, 1, p->is3d ? 0 : 1,
                           p->d_partials, d_lik, s, p->pg, dual ? p->pad : apirl::PadBuffers(), p->em_block,
                           d_zimg, d_zero_add, p->persistent ? p->d_chunk : nullptr, p->sparse_image, p->nz));
  if (p->timing) {
    CK(cudaEventRecord(p->ev1, s));
    p->timed = 1;
  }
  return APIRL_OK;
}

apirl_status check_em(apirl_projector* p, const void* d_counts, int dtype, const float* d_x, const float* d_bp,
                      int subset, int nsubsets) {
  apirl_status st = check_subset(p, subset, nsubsets);
  if (st) return st;
  if (!d_counts || !d_x || !d_bp) return fail(APIRL_ERR_INVALID, "null buffer");
  if (dtype != APIRL_F32 && dtype != APIRL_U32 && dtype != APIRL_U16)
    return fail(APIRL_ERR_INVALID, "unknown counts dtype %d", dtype);
  return APIRL_OK;
}

}  // namespace

apirl_status apirl_em_pass(apirl_projector* p, const void* d_counts, int counts_dtype, int counts_packed,
                           const float* d_add, float* d_x, float* d_bp, const float* d_sens, const float* d_thr,
                           float thr_value, int ge, int subset, int nsubsets, double* d_lik, void* stream) {
  apirl_status st = check_em(p, d_counts, counts_dtype, d_x, d_bp, subset, nsubsets);
  if (st) return st;
  if (!d_sens) return fail(APIRL_ERR_INVALID, "null sensitivity");
  DEVICE_SCOPE(p->device);
  cudaStream_t s = (cudaStream_t)stream;
  SubsetSel ss = make_subset(p, subset, nsubsets);
  const int64_t nv = (int64_t)p->g.nx * p->g.ny * p->g.nz;
  if (use_dual(p)) {
    CK(apirl::launch_pad_copy(p->g, d_x, p->pad, s));
    st = fused(p, ss, d_counts, counts_dtype, counts_packed, d_add, d_x, d_bp, true, d_lik, s);
    if (st) return st;
    CK(apirl::launch_pad_reduce(p->g, p->pad, 0, d_x, nullptr, d_sens, d_thr, thr_value, ge, s));
    return APIRL_OK;
  }
  st = fused(p, ss, d_counts, counts_dtype, counts_packed, d_add, d_x, d_bp, false, d_lik, s);
  if (st) return st;
  CK(apirl::launch_update(nv, d_x, d_bp, d_sens, d_thr, thr_value, ge, 1, s));
  return APIRL_OK;
}

apirl_status apirl_zero_count_image(apirl_projector* p, const void* d_counts, int counts_dtype, int counts_packed,
                                    const float* d_add, float* d_zimg, double* d_zero_add, int subset, int nsubsets,
                                    void* stream) {
  apirl_status st = check_subset(p, subset, nsubsets);
  if (st) return st;
  if (!d_counts || !d_zimg) return fail(APIRL_ERR_INVALID, "null buffer");
  if (counts_dtype != APIRL_F32 && counts_dtype != APIRL_U32 && counts_dtype != APIRL_U16)
    return fail(APIRL_ERR_INVALID, "unknown counts dtype %d", counts_dtype);
  if (!p->is3d || p->t.lor_s)
    return fail(APIRL_ERR_NOT_SUPPORTED, "the sparse pass needs a 3D projector with one ray per bin");
  DEVICE_SCOPE(p->device);
  CK(apirl::launch_zero_bins(p->g, p->t, make_subset(p, subset, nsubsets), d_counts, counts_dtype, counts_packed,
                             d_add, d_zimg, p->d_partials, d_zero_add, (cudaStream_t)stream,
                             use_dual(p) ? p->pad : apirl::PadBuffers()));
  return APIRL_OK;
}

apirl_status apirl_em_pass_sparse(apirl_projector* p, const void* d_counts, int counts_dtype, int counts_packed,
                                  const float* d_add, float* d_x, float* d_bp, const float* d_sens,
                                  const float* d_zimg, const double* d_zero_add, const float* d_thr, float thr_value,
                                  int ge, int subset, int nsubsets, double* d_lik, void* stream) {
  apirl_status st = check_em(p, d_counts, counts_dtype, d_x, d_bp, subset, nsubsets);
  if (st) return st;
  if (!d_sens || !d_zimg) return fail(APIRL_ERR_INVALID, "null sensitivity or zero-count image");
  if (!p->is3d || p->t.lor_s || p->pg.enabled)
    return fail(APIRL_ERR_NOT_SUPPORTED, "the sparse pass needs a 3D projector with one float ray per bin");
  DEVICE_SCOPE(p->device);
  cudaStream_t s = (cudaStream_t)stream;
  SubsetSel ss = make_subset(p, subset, nsubsets);
  const int64_t nv = (int64_t)p->g.nx * p->g.ny * p->g.nz;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(s, &cs));
  if (cs == cudaStreamCaptureStatusNone) {
    st = apirl::prepare_nz_list(p, apirl_projector_num_bins(p, subset, nsubsets));
    if (st) return st;
  }
  if (use_dual(p)) {
    CK(apirl::launch_pad_copy(p->g, d_x, p->pad, s));
    st = fused(p, ss, d_counts, counts_dtype, counts_packed, d_add, d_x, d_bp, true, d_lik, s, d_zimg, d_zero_add);
    if (st) return st;
    CK(apirl::launch_pad_reduce(p->g, p->pad, 0, d_x, nullptr, d_sens, d_thr, thr_value, ge, s));
    return APIRL_OK;
  }
  st = fused(p, ss, d_counts, counts_dtype, counts_packed, d_add, d_x, d_bp, false, d_lik, s, d_zimg, d_zero_add);
  if (st) return st;
  CK(apirl::launch_update(nv, d_x, d_bp, d_sens, d_thr, thr_value, ge, 1, s));
  return APIRL_OK;
}

apirl_status apirl_em_project_backproject_sparse(apirl_projector* p, const void* d_counts, int counts_dtype,
                                                 int counts_packed, const float* d_add, const float* d_x, float* d_bp,
                                                 const float* d_zimg, const double* d_zero_add, int subset,
                                                 int nsubsets, double* d_lik, void* stream) {
  apirl_status st = check_em(p, d_counts, counts_dtype, d_x, d_bp, subset, nsubsets);
  if (st) return st;
  if (!d_zimg) return fail(APIRL_ERR_INVALID, "null zero-count or geometry image");
  if (!p->is3d || p->t.lor_s || p->pg.enabled)
    return fail(APIRL_ERR_NOT_SUPPORTED, "the sparse pass needs a 3D projector with one float ray per bin");
  DEVICE_SCOPE(p->device);
  cudaStream_t s = (cudaStream_t)stream;
  SubsetSel ss = make_subset(p, subset, nsubsets);
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(s, &cs));
  if (cs == cudaStreamCaptureStatusNone) {
    st = apirl::prepare_nz_list(p, apirl_projector_num_bins(p, subset, nsubsets));
    if (st) return st;
  }
  if (use_dual(p)) {
    CK(apirl::launch_pad_copy(p->g, d_x, p->pad, s));
    st = fused(p, ss, d_counts, counts_dtype, counts_packed, d_add, d_x, d_bp, true, d_lik, s, d_zimg, d_zero_add);
    if (st) return st;
    CK(apirl::launch_pad_reduce(p->g, p->pad, 1, nullptr, d_bp, nullptr, nullptr, 0.f, 0, s));
    return APIRL_OK;
  }
  return fused(p, ss, d_counts, counts_dtype, counts_packed, d_add, d_x, d_bp, false, d_lik, s, d_zimg, d_zero_add);
}

apirl_status apirl_em_project_backproject(apirl_projector* p, const void* d_counts, int counts_dtype,
                                          int counts_packed, const float* d_add, const float* d_x, float* d_bp,
                                          int subset, int nsubsets, double* d_lik, void* stream) {
  apirl_status st = check_em(p, d_counts, counts_dtype, d_x, d_bp, subset, nsubsets);
  if (st) return st;
  DEVICE_SCOPE(p->device);
  cudaStream_t s = (cudaStream_t)stream;
  SubsetSel ss = make_subset(p, subset, nsubsets);
  if (use_dual(p)) {
    CK(apirl::launch_pad_copy(p->g, d_x, p->pad, s));
    st = fused(p, ss, d_counts, counts_dtype, counts_packed, d_add, d_x, d_bp, true, d_lik, s);
    if (st) return st;
    CK(apirl::launch_pad_reduce(p->g, p->pad, 1, nullptr, d_bp, nullptr, nullptr, 0.f, 0, s));
    return APIRL_OK;
  }
  return fused(p, ss, d_counts, counts_dtype, counts_packed, d_add, d_x, d_bp, false, d_lik, s);
}

apirl_status apirl_projector_set_option(apirl_projector* p, int option, int value) {
  if (!p) return fail(APIRL_ERR_INVALID, "null projector");
  switch (option) {
    case APIRL_OPT_DUAL_LAYOUT: {
      p->dual_layout = value != 0;
      if (p->dual_layout && p->is3d) {
        DEVICE_SCOPE(p->device);
        return alloc_pad(p);
      }
      return APIRL_OK;
    }
    case APIRL_OPT_KERNEL_TIMING: p->timing = value != 0; p->timed = 0; return APIRL_OK;
    case APIRL_OPT_PERSISTENT: p->persistent = value != 0; return APIRL_OK;
    case APIRL_OPT_SPARSE_IMAGE:
      if (value != APIRL_SPARSE_ZERO_COUNT && value != APIRL_SPARSE_GEOMETRY)
        return fail(APIRL_ERR_INVALID, "unknown sparse image kind %d", value);
      p->sparse_image = value;
      return APIRL_OK;
    case APIRL_OPT_L2_PERSIST: {
      if (value && !use_dual(p))
        return fail(APIRL_ERR_NOT_SUPPORTED, "the L2 window covers the padded 3D layouts");
      DEVICE_SCOPE(p->device);
      p->pad.window = 0;
      p->pad.hit_ratio = 0.f;
      if (p->l2_limit_set) {
        CK(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, p->l2_limit_prev));
        p->l2_limit_set = false;
      }
      if (value) {
        int max_window = 0, max_persist = 0;
        CK(cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, p->device));
        CK(cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, p->device));
        const size_t want = (size_t)4 * p->pad.lim * sizeof(float);
        const size_t win = want < (size_t)max_window ? want : (size_t)max_window;
        const size_t aside = win < (size_t)max_persist ? win : (size_t)max_persist;
        if (win == 0 || aside == 0) return fail(APIRL_ERR_NOT_SUPPORTED, "this device has no persisting L2");
        // The set-aside is a limit of this process's context on the device.
        CK(cudaDeviceGetLimit(&p->l2_limit_prev, cudaLimitPersistingL2CacheSize));
        CK(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, aside));
        p->l2_limit_set = true;
        p->pad.window = win;
        p->pad.hit_ratio = (float)((double)aside / (double)win);
      }
      return APIRL_OK;
    }
    case APIRL_OPT_GATHER_UNROLL:
      if (value != 0 && value != 4 && value != 6 && value != 8)
        return fail(APIRL_ERR_INVALID, "gather segments in flight: 0, 4, 6 or 8");
      p->pad.unroll = value;
      return APIRL_OK;
    case APIRL_OPT_LIST_ORDER:
      if (value != 0 && (value < 32 || value > apirl::kNzTile || (value & (value - 1))))
        return fail(APIRL_ERR_INVALID, "list order: 0, or a power of two from 32 to %d", apirl::kNzTile);
      p->nz.order = value;
      return APIRL_OK;
    case APIRL_OPT_ACCUMULATE: {
      if (value != APIRL_ACC_ATOMIC && value != APIRL_ACC_WARP && value != APIRL_ACC_COMPENSATED)
        return fail(APIRL_ERR_INVALID, "unknown accumulation form %d", value);
      if (value != APIRL_ACC_ATOMIC && !use_dual(p))  // use_dual: the padded layouts are taken
        return fail(APIRL_ERR_NOT_SUPPORTED, "accumulation forms need the padded 3D layouts (3D, float walk, one ray "
                                             "per bin, dual layout)");
      if (value == APIRL_ACC_COMPENSATED && !p->pad.eA) {
        DEVICE_SCOPE(p->device);
        const size_t pv = (size_t)p->pad.lim;
        CK(cudaMalloc(&p->pad.eA, pv * sizeof(float)));
        CK(cudaMalloc(&p->pad.eT, pv * sizeof(float)));
        CK(cudaMemset(p->pad.eA, 0, pv * sizeof(float)));
        CK(cudaMemset(p->pad.eT, 0, pv * sizeof(float)));
      }
      p->pad.acc = value;
      return APIRL_OK;
    }
    case APIRL_OPT_EM_BLOCK:
      if (value < 32 || value > 256 || value % 32) return fail(APIRL_ERR_INVALID, "block size must be 32..256, x32");
      p->em_block = value;
      if (p->is3d) {
        DEVICE_SCOPE(p->device);
        CK(apirl::prepare_em_kernels(value));
      }
      return APIRL_OK;
    default: return fail(APIRL_ERR_INVALID, "unknown option %d", option);
  }
}

apirl_status apirl_projector_autotune(apirl_projector* p, const void* d_counts, int counts_dtype, const float* d_x,
                                     int subset, int nsubsets, int repeats, int* best_block, void* stream) {
  apirl_status st = check_em(p, d_counts, counts_dtype, d_x, d_x, subset, nsubsets);
  if (st) return st;
  DEVICE_SCOPE(p->device);
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t nv = (int64_t)p->g.nx * p->g.ny * p->g.nz;
  float* bp = nullptr;
  CK(cudaMalloc(&bp, nv * sizeof(float)));
  cudaEvent_t a = nullptr, b = nullptr;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const int cands[] = {64, 96, 128, 192, 256};
  const int saved_timing = p->timing;
  p->timing = 0;
  float best = 1e30f;
  int best_b = p->em_block;
  if (repeats < 1) repeats = 1;
  for (int c : cands) {
    p->em_block = c;
    CK(cudaMemsetAsync(bp, 0, nv * sizeof(float), s));
    st = apirl_em_project_backproject(p, d_counts, counts_dtype, 0, nullptr, d_x, bp, subset, nsubsets, nullptr, s);
    if (st) break;
    cudaEventRecord(a, s);
    for (int r = 0; r < repeats && !st; r++)
      st = apirl_em_project_backproject(p, d_counts, counts_dtype, 0, nullptr, d_x, bp, subset, nsubsets, nullptr, s);
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (ms < best) { best = ms; best_b = c; }
  }
  p->timing = saved_timing;
  p->em_block = best_b;
  if (!st) {
    cudaError_t pe = apirl::prepare_em_kernels(best_b);
    if (pe != cudaSuccess) st = fail(APIRL_ERR_CUDA, "prepare_em_kernels: %s", cudaGetErrorString(pe));
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(bp);
  if (st) return st;
  if (best_block) *best_block = best_b;
  return APIRL_OK;
}

apirl_status apirl_projector_autotune_ex(apirl_projector* p, const void* d_counts, int counts_dtype,
                                        const float* d_x, const float* d_zimg, int subset, int nsubsets, int repeats,
                                        apirl_tune* out, void* stream) {
  apirl_status st = check_em(p, d_counts, counts_dtype, d_x, d_x, subset, nsubsets);
  if (st) return st;
  if (!use_dual(p) || !p->persistent || p->pad.acc != APIRL_ACC_ATOMIC)
    return fail(APIRL_ERR_NOT_SUPPORTED, "the launch shape is tuned for the persistent pass over the padded layouts "
                                         "with plain atomics");
  DEVICE_SCOPE(p->device);
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t nv = (int64_t)p->g.nx * p->g.ny * p->g.nz;
  float* bp = nullptr;
  CK(cudaMalloc(&bp, nv * sizeof(float)));
  cudaEvent_t a = nullptr, b = nullptr;
  cudaError_t ce = cudaEventCreate(&a);
  if (ce == cudaSuccess) ce = cudaEventCreate(&b);
  const int blocks[] = {64, 96, 128, 192, 256};
  const int unrolls[] = {4, 6, 8};
  const int saved_timing = p->timing, saved_block = p->em_block, saved_unroll = p->pad.unroll;
  p->timing = 0;
  float best = 1e30f;
  int best_b = p->em_block, best_u = p->pad.unroll;
  if (repeats < 1) repeats = 1;
  auto pass = [&]() {
    return d_zimg ? apirl_em_project_backproject_sparse(p, d_counts, counts_dtype, 0, nullptr, d_x, bp, d_zimg,
                                                        nullptr, subset, nsubsets, nullptr, s)
                  : apirl_em_project_backproject(p, d_counts, counts_dtype, 0, nullptr, d_x, bp, subset, nsubsets,
                                                 nullptr, s);
  };
  for (int blk : blocks) {
    if (ce != cudaSuccess) break;
    p->em_block = blk;
    if ((ce = apirl::prepare_em_kernels(blk)) != cudaSuccess) break;
    for (int u : unrolls) {
      p->pad.unroll = u;
      if ((ce = cudaMemsetAsync(bp, 0, nv * sizeof(float), s)) != cudaSuccess) break;
      if ((st = pass())) break;  // warm-up (and the list, for the sparse pass)
      if ((ce = cudaEventRecord(a, s)) != cudaSuccess) break;
      for (int r = 0; r < repeats && !st; r++) st = pass();
      if (st) break;
      if ((ce = cudaEventRecord(b, s)) != cudaSuccess || (ce = cudaEventSynchronize(b)) != cudaSuccess) break;
      float ms = 0;
      if ((ce = cudaEventElapsedTime(&ms, a, b)) != cudaSuccess) break;
      if (ms < best) { best = ms; best_b = blk; best_u = u; }
    }
    if (st) break;
  }
  p->timing = saved_timing;
  if (!st && ce == cudaSuccess) {
    p->em_block = best_b;
    p->pad.unroll = best_u;
    ce = apirl::prepare_em_kernels(best_b);
  } else {
    p->em_block = saved_block;
    p->pad.unroll = saved_unroll;
  }
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  cudaFree(bp);
  if (st) return st;
  if (ce != cudaSuccess) return cuda_fail(ce, "autotune");
  if (out) {
    out->block = best_b;
    out->unroll = best_u;
    out->ms = best / repeats;
  }
  return APIRL_OK;
}

apirl_status apirl_projector_kernel_ms(apirl_projector* p, double* ms) {
  if (!p || !ms) return fail(APIRL_ERR_INVALID, "bad arguments");
  if (!p->timed) return fail(APIRL_ERR_INVALID, "no timed pass recorded (enable APIRL_OPT_KERNEL_TIMING)");
  DEVICE_SCOPE(p->device);
  CK(cudaEventSynchronize(p->ev1));
  float f = 0.f;
  CK(cudaEventElapsedTime(&f, p->ev0, p->ev1));
  *ms = f;
  return APIRL_OK;
}

apirl_status apirl_stage_counts(apirl_projector* p, const void* h_counts_subset, int counts_dtype, void* d_counts_stage,
                                int subset, int nsubsets, void* stream) {
  apirl_status st = check_subset(p, subset, nsubsets);
  if (st) return st;
  if (!h_counts_subset || !d_counts_stage) return fail(APIRL_ERR_INVALID, "null buffer");
  if (counts_dtype != APIRL_F32 && counts_dtype != APIRL_U32 && counts_dtype != APIRL_U16)
    return fail(APIRL_ERR_INVALID, "unknown counts dtype %d", counts_dtype);
  const int64_t nb = apirl_projector_num_bins(p, subset, nsubsets);
  const size_t esz = counts_dtype == APIRL_U16 ? 2 : 4;
  DEVICE_SCOPE(p->device);
  if (!p->copy_stream) {
    CK(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&p->copy_ready, cudaEventDisableTiming));
    for (auto& e : p->staged) CK(cudaEventCreateWithFlags(&e.done, cudaEventDisableTiming));
  }
  // A free slot, or the one staging the same device buffer (restaged).
  apirl_projector::Staged* slot = nullptr;
  for (auto& e : p->staged)
    if (e.dev == d_counts_stage) slot = &e;
  for (auto& e : p->staged)
    if (!slot && !e.dev) slot = &e;
  if (!slot) return fail(APIRL_ERR_INVALID, "more than 4 staged copies outstanding");
  // The copy starts after the caller's stream's earlier work (which may still
  // read d_counts_stage) and runs beside its later work.
  CK(cudaEventRecord(p->copy_ready, (cudaStream_t)stream));
  CK(cudaStreamWaitEvent(p->copy_stream, p->copy_ready, 0));
  CK(cudaMemcpyAsync(d_counts_stage, h_counts_subset, nb * esz, cudaMemcpyHostToDevice, p->copy_stream));
  CK(cudaEventRecord(slot->done, p->copy_stream));
  slot->host = h_counts_subset;
  slot->dev = d_counts_stage;
  return APIRL_OK;
}

}  // extern "C"

namespace {
// apirl_em_pass_host and apirl_em_pass_host_async; `wait`: synchronise the
// stream before returning.
apirl_status em_pass_host(apirl_projector* p, const void* h_counts_subset, int counts_dtype, void* d_counts_stage,
                          float* d_x, float* d_bp, const float* d_sens, const float* d_zimg,
                          const double* d_zero_add, float thr_value, int ge, int subset, int nsubsets,
                          float* h_x_out, double* h_lik, void* stream, bool wait) {
  apirl_status st = check_subset(p, subset, nsubsets);
  if (st) return st;
  if (!h_counts_subset || !d_counts_stage) return fail(APIRL_ERR_INVALID, "null buffer");
  const int64_t nb = apirl_projector_num_bins(p, subset, nsubsets);
  const size_t esz = counts_dtype == APIRL_U16 ? 2 : 4;
  DEVICE_SCOPE(p->device);
  cudaStream_t s = (cudaStream_t)stream;
  apirl_projector::Staged* slot = nullptr;
  for (auto& e : p->staged)
    if (e.dev == d_counts_stage && e.host == h_counts_subset) slot = &e;
  if (slot) {
    CK(cudaStreamWaitEvent(s, slot->done, 0));  // staged ahead by apirl_stage_counts
    slot->dev = nullptr;
    slot->host = nullptr;
  } else {
    CK(cudaMemcpyAsync(d_counts_stage, h_counts_subset, nb * esz, cudaMemcpyHostToDevice, s));
  }
  double* d_lik = p->d_scalars;
  if (d_zimg)
    st = apirl_em_pass_sparse(p, d_counts_stage, counts_dtype, 1, nullptr, d_x, d_bp, d_sens, d_zimg, d_zero_add,
                              nullptr, thr_value, ge, subset, nsubsets, h_lik ? d_lik : nullptr, stream);
  else
    st = apirl_em_pass(p, d_counts_stage, counts_dtype, 1, nullptr, d_x, d_bp, d_sens, nullptr, thr_value, ge,
                       subset, nsubsets, h_lik ? d_lik : nullptr, stream);
  if (st) return st;
  const int64_t nv = (int64_t)p->g.nx * p->g.ny * p->g.nz;
  if (h_x_out) CK(cudaMemcpyAsync(h_x_out, d_x, nv * sizeof(float), cudaMemcpyDeviceToHost, s));
  if (h_lik) CK(cudaMemcpyAsync(h_lik, d_lik, sizeof(double), cudaMemcpyDeviceToHost, s));
  if (wait) CK(cudaStreamSynchronize(s));
  return APIRL_OK;
}
}  // namespace

extern "C" {

apirl_status apirl_em_pass_host(apirl_projector* p, const void* h_counts_subset, int counts_dtype,
                                void* d_counts_stage, float* d_x, float* d_bp, const float* d_sens,
                                const float* d_zimg, const double* d_zero_add, float thr_value, int ge, int subset,
                                int nsubsets, float* h_x_out, double* h_lik, void* stream) {
  return em_pass_host(p, h_counts_subset, counts_dtype, d_counts_stage, d_x, d_bp, d_sens, d_zimg, d_zero_add,
                      thr_value, ge, subset, nsubsets, h_x_out, h_lik, stream, true);
}

apirl_status apirl_em_pass_host_async(apirl_projector* p, const void* h_counts_subset, int counts_dtype,
                                      void* d_counts_stage, float* d_x, float* d_bp, const float* d_sens,
                                      const float* d_zimg, const double* d_zero_add, float thr_value, int ge,
                                      int subset, int nsubsets, float* h_x_out, double* h_lik, void* stream) {
  return em_pass_host(p, h_counts_subset, counts_dtype, d_counts_stage, d_x, d_bp, d_sens, d_zimg, d_zero_add,
                      thr_value, ge, subset, nsubsets, h_x_out, h_lik, stream, false);
}

}  // extern "C"

namespace apirl {
apirl_status prepare_nz_list(apirl_projector* p, int64_t total) {
  if (total <= p->nz.cap || !p->is3d) return APIRL_OK;
  DEVICE_SCOPE(p->device);
  cudaFree(p->nz.list);
  cudaFree(p->nz.tiles);
  p->nz.list = nullptr;
  p->nz.tiles = nullptr;
  p->nz.cap = 0;
  if (!p->nz.n_list) CK(cudaMalloc(&p->nz.n_list, sizeof(int)));
  const int64_t n_tiles = (total + apirl::kNzTile - 1) / apirl::kNzTile;
  CK(cudaMalloc(&p->nz.list, (size_t)total * sizeof(int)));
  CK(cudaMalloc(&p->nz.tiles, (size_t)n_tiles * sizeof(int)));
  p->nz.cap = total;
  return APIRL_OK;
}
}  // namespace apirl

namespace apirl {
cudaError_t backproject_sino(apirl_projector* p, SubsetSel ss, const float* vin, int vin_mode, float* img,
                             cudaStream_t st) {
  if (use_dual(p)) return launch_backproject_pad(p->g, p->t, ss, vin, vin_mode, img, p->pad, p->d_chunk, st);
  return launch_backproject(p->g, p->t, ss, vin, vin_mode, nullptr, 0, img, st, p->pg);
}
}  // namespace apirl

namespace apirl {
apirl_status backproject_sino_and_ones(apirl_projector* p, SubsetSel ss, const float* vin, int vin_mode, float* img,
                                       float* gimg, cudaStream_t st) {
  if (!use_dual(p)) {
    CK(backproject_sino(p, ss, vin, vin_mode, img, st));
    CK(backproject_sino(p, ss, nullptr, 2, gimg, st));
    return APIRL_OK;
  }
  if (!p->pad2.bA) {
    const size_t pv = (size_t)p->pad.lim;
    CK(cudaMalloc(&p->pad2.bA, pv * sizeof(float)));
    CK(cudaMalloc(&p->pad2.bT, pv * sizeof(float)));
    CK(cudaMemset(p->pad2.bA, 0, pv * sizeof(float)));
    CK(cudaMemset(p->pad2.bT, 0, pv * sizeof(float)));
    p->pad2.lim = p->pad.lim;
  }
  CK(launch_backproject_pad(p->g, p->t, ss, vin, vin_mode, img, p->pad, p->d_chunk, st, gimg, p->pad2));
  return APIRL_OK;
}
}  // namespace apirl

