// Internal interface between the C ABI (capi.cu), the kernels (kernels.cu) and
// the host-side geometry builder (host_geometry.cpp).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>
#include "geom_types.h"

namespace apirl {

// Device-resident geometry of one sinogram.
struct LorTable {
  const float4* lor;    // [n_proj][n_r] = (p1x, p1y, p2x, p2y)
  const float2* z;      // 3D: [n_sinos] = (z1, z2) end-point z; 2D: unused
  const uint8_t* ok;    // 2D: [n_r] 1 when r <= sinogram rFov (getPointsFromLor); 3D: unused
  int n_proj, n_r, n_sinos;  // n_sinos: sinograms of the shard the kernels cover
  int is3d;
  // First sinogram of the shard (apirl_projector_set_shard): bins cover
  // sinograms g0 .. g0 + n_sinos - 1 of the whole sinogram.
  int g0 = 0;
  // Several rays per bin (3D; set when lor_s is not null): a bin is the sum
  // over its rays, in the order ring pair m, radial sample o, axial sample q,
  // with end points lor_s[(a * n_r + l) * n_rs + o] and zs[zoff[g] + m * n_as + q].
  const float4* lor_s = nullptr;
  const float2* zs = nullptr;
  const int* zoff = nullptr;  // [n_sinos + 1]
  int n_rs = 1, n_as = 1;
};

// Host tables of the sampled rays of every bin.
struct RayTables {
  std::vector<float> lor;  // n_proj * n_r * n_rs * 4
  std::vector<float> zs;   // 2 per (sinogram, ring pair, axial sample)
  std::vector<int> zoff;   // n_sinos + 1
  int n_rs = 1, n_as = 1;
};

// Double-precision geometry for the FP64-alpha precision mode (3D only).
struct PreciseGeom {
  const double4* lor = nullptr;  // [n_proj][n_r]
  const double2* z = nullptr;    // [n_sinos]
  int nx = 0, ny = 0, nz = 0;
  double dx = 0, dy = 0, dz = 0, rfov = 0, offz = 0;
  int enabled = 0;
};

struct SubsetSel {
  int subset;  // < 0: all angles
  int nsub;
  int nk;      // angles in this subset
};

// Host-side tables built with the reference's float expressions.
struct HostTables {
  std::vector<float> lor;   // n_proj * n_r * 4
  std::vector<float> z;     // n_sinos * 2
  std::vector<uint8_t> ok;  // n_r
  int n_sinos = 1;
};
// The same tables in double precision (double trigonometry), for FP64-alpha.
void build_tables_3d_f64(int n_proj, int n_r, int n_rings, float r_fov, float axial_fov, float r_scanner, int n_seg,
                         const int* min_rd, const int* max_rd, std::vector<double>& lor, std::vector<double>& z);
void build_tables_2d(int n_proj, int n_r, float r_fov, float r_scanner, HostTables& t);
bool build_tables_3d(int n_proj, int n_r, int n_rings, float r_fov, float axial_fov, float r_scanner, int n_seg,
                     const int* min_rd, const int* max_rd, HostTables& t);
// Rays of every bin for SiddonProjector(ns, nas) with useMultipleLorsPerBin =
// multi (recon/src/SiddonProjector.cpp:346-397).  dab: DivideAndBackproject's
// rule for when the oversampled end points are used (:628).  Returns false
// when a ray end point is not finite (a sample outside the scanner radius).
bool build_rays_3d(int n_proj, int n_r, int n_rings, float r_fov, float axial_fov, float r_scanner, int n_seg,
                   const int* min_rd, const int* max_rd, int ns, int nas, int multi, bool dab, RayTables& t);
// Siemens mMR tables (LOR end points per data/src/Sinogram2DinSiemensMmr.cpp,
// ring z for its 260 mm axial field of view); the LOR table alone for tests.
bool build_tables_mmr(int n_proj, int n_r, int n_rings, int n_seg, const int* min_rd, const int* max_rd,
                      HostTables& t);
void mmr_lor_table(int n_proj, int n_r, std::vector<float>& lor);
extern const float kMmrRadius, kMmrRFov, kMmrAxialFov, kMmrDoi;
ImgGeom make_img_geom(int nx, int ny, int nz, float dx, float dy, float dz);

int subset_nproj(int n_proj, int subset, int nsub);

// Launchers (kernels.cu).  All return cudaGetLastError() after the launch.
// pg.enabled selects the FP64-alpha walk (3D only).
cudaError_t launch_project(const ImgGeom& g, const LorTable& t, SubsetSel s, const float* img, float* out,
                           cudaStream_t st, const PreciseGeom& pg = PreciseGeom());
// vin_mode: 0 = subset sinogram, 1 = whole sinogram read at the subset's angles, 2 = all ones.
cudaError_t launch_backproject(const ImgGeom& g, const LorTable& t, SubsetSel s, const float* vin, int vin_mode,
                               const float* vest, int divide, float* img, cudaStream_t st,
                               const PreciseGeom& pg = PreciseGeom());
cudaError_t launch_count_steps(const ImgGeom& g, const LorTable& t, SubsetSel s, int32_t* steps, cudaStream_t st);

// Fused EM pass.  partials: >= em_pass_blocks() doubles of scratch.
int64_t em_pass_blocks(const LorTable& t, SubsetSel s);
// Padded two-layout buffers of the fused 3D pass: the image as [z][y][x] (pA)
// and [z][x][y] (pT), and the backprojection likewise (bA, bT), each with a
// kPad (2) voxel zero border; lim = voxels of one padded buffer.
struct PadBuffers {
  float* pA = nullptr;
  float* pT = nullptr;
  float* bA = nullptr;
  float* bT = nullptr;
  unsigned lim = 0;
  // How scatters into bA / bT accumulate (APIRL_ACC_*); eA / eT: the
  // rounding errors of the compensated form, same layouts.
  int acc = 0;
  float* eA = nullptr;
  float* eT = nullptr;
  // window > 0 (APIRL_OPT_L2_PERSIST): the padded kernels launch with an L2
  // access policy window of that many bytes from pA (the four images are one
  // block pA, pT, bA, bT), hit_ratio of it persisting.
  size_t window = 0;
  float hit_ratio = 0.f;
  // Gather segments in flight of the fused pass (APIRL_OPT_GATHER_UNROLL: 4,
  // 6 or 8; 0 = the pass kind's default).
  int unroll = 0;
};
// Bins per tile of the list building (one block each).
constexpr int kNzTile = 2048;
// Room for the list of a subset's bins with counts (sparse passes of the
// persistent kernel): `list` holds cap int32 bin numbers, `tiles` one int per
// kNzTile bins of cap, `n_list` one int.
struct NzList {
  int* list = nullptr;
  int* tiles = nullptr;
  int* n_list = nullptr;
  int64_t cap = 0;
  int order = 0;  // APIRL_OPT_LIST_ORDER: 0 = bin order, else groups of this size by walk length
};
// lik_mode: 0 = over e != 0, 1 = over e > 0, 2 = over ratio > 0.  back = 0: no backprojection.
cudaError_t launch_em_pass(const ImgGeom& g, const LorTable& t, SubsetSel s, const void* counts, int counts_dtype,
                           int counts_packed, const float* add, const float* x, float* bp, int back, int lik_mode,
                           double* partials, double* lik, cudaStream_t st, const PreciseGeom& pg = PreciseGeom(),
                           const PadBuffers& pad = PadBuffers(), int block = 0, const float* zimg = nullptr,
                           const double* zero_add = nullptr, unsigned long long* persist_counter = nullptr,
                           int zimg_all_bins = 0, const NzList& nz = NzList());
// Fits the shared-memory carveout of the persistent fused kernels to `block`
// threads per block (called outside graph capture, when a projector is made
// or its block size changes).
cudaError_t prepare_em_kernels(int block);
// zimg_all_bins: zimg is G_s = A_s^T 1 over all bins and zero_add the sum of
// all bins' additive terms; walked bins then add m log e alone.
// Sparse pass (zimg set, 3D float walk): bins with zero counts are not walked;
// the likelihood subtracts x . zimg + *zero_add instead of their estimates.
// zimg = A_s^T 1[m == 0] and zero_add = sum of those bins' additive terms,
// from launch_zero_bins (img accumulated; partials: em_pass_blocks scratch).
cudaError_t launch_zero_bins(const ImgGeom& g, const LorTable& t, SubsetSel s, const void* counts, int counts_dtype,
                             int counts_packed, const float* add, float* img, double* partials, double* zero_add,
                             cudaStream_t st, const PadBuffers& pad = PadBuffers());
cudaError_t launch_pad_copy(const ImgGeom& g, const float* x, const PadBuffers& pad, cudaStream_t st);
// mode 0: EM update of x from bA + bT (threshold rule); mode 1: bp += bA + bT.  Clears bA, bT.
cudaError_t launch_pad_reduce(const ImgGeom& g, const PadBuffers& pad, int mode, float* x, float* bp,
                              const float* sens, const float* thr_ptr, float thr_value, int ge, cudaStream_t st);
// 3D backprojection img += A^T v through the padded pair (3D float walk, one
// ray per bin): a persistent scatter, then k_pad_reduce folds the pair into
// img and clears it.  `counter` is the projector's chunk counter.
// img2 / pad2 (its bA, bT) set: the same walks also give img2 += A_s^T 1.
cudaError_t launch_backproject_pad(const ImgGeom& g, const LorTable& t, SubsetSel s, const float* vin, int vin_mode,
                                   float* img, const PadBuffers& pad, unsigned long long* counter, cudaStream_t st,
                                   float* img2 = nullptr, const PadBuffers& pad2 = PadBuffers());
cudaError_t launch_inverse_divide(int64_t n, const float* meas, float* est, cudaStream_t st);
cudaError_t launch_add_bins(int64_t n, const float* add, float* est, cudaStream_t st);
cudaError_t launch_likelihood(int64_t n, const float* est, const float* meas, int gt0, double* partials,
                              int64_t n_partials, double* out, cudaStream_t st);
int64_t likelihood_blocks(int64_t n);
cudaError_t launch_threshold(int64_t n, const float* sens, unsigned* minmax_scratch, float* thr, cudaStream_t st);
cudaError_t launch_update(int64_t n, float* x, float* bp, const float* sens, const float* thr_ptr, float thr_value,
                          int ge, int zero_bp, cudaStream_t st);
cudaError_t launch_force_positive(int64_t n, float* x, cudaStream_t st);
cudaError_t launch_fill(int64_t n, float* x, float v, cudaStream_t st);
cudaError_t launch_exp_nonzero(int64_t n, float* v, cudaStream_t st);

// ---- batched reconstructions (batch.cu) ---------------------------------------
// One list of bins with counts walked in a batched step: one job's subset list
// (an EM pass), or one of its subset lists for its final likelihood (back = 0).
// Its chunks of 32 list entries are chunk_begin .. chunk_begin +
// ceil(n_list / 32) - 1 of the step; segments are ordered by chunk_begin.
struct MultiSeg {
  ImgGeom g;
  LorTable t;
  SubsetSel s;
  const void* counts;    // whole sinogram, [sinogram][angle][r]
  const float* add;      // same layout, or null
  PadBuffers pad;        // the job's padded image copies and backprojection pair
  const int* list;       // the subset's bins with counts, in bin order
  int64_t n_list;
  int64_t chunk_begin;
  int counts_dtype;
  int back;
};
// One job's voxel work in a batched step, in 32 x 32 tiles of its slices:
// before the walk, x into the padded copies and -x . gimg; after it, with
// `update`, the EM update of x from the padded backprojection pair; the
// likelihood = the job's chunk partials + its -x . gimg partials - zero_add.
struct MultiVox {
  ImgGeom g;
  PadBuffers pad;
  float* x;
  const float* sens;     // the pass's subset sensitivity (update)
  const float* gimg;     // G_s of the pass's subset, or A^T 1 of all subsets (final likelihood)
  double* lik;           // the likelihood's slot
  int64_t tile_begin;    // first tile of the job in the step's tile launches
  int64_t chunk_begin, n_chunks;  // the job's chunk partials in the walk
  double zero_add;       // sum over all walked subsets' bins of the additive term
  int tiles_x, tiles_y;
  int update, ge;
};
// Tiles (blocks of the copy / update launches) of a job: ceil(nx/32) x ceil(ny/32) x nz.
inline int64_t multi_tiles(const ImgGeom& g) {
  return (int64_t)((g.nx + 31) / 32) * ((g.ny + 31) / 32) * g.nz;
}
// Persistent grid of the batched walk on the current device.
cudaError_t multi_walk_grid(int* blocks);
// Loads the batch engine's kernels into the context (instead of at their
// first launch).
cudaError_t load_batch_kernels();
// One batched step: copies and dot products, the walk over every segment's
// list (counter reset here), the likelihood sums, the updates.
// chunk_partials: >= total_chunks doubles; tile_partials: >= total_tiles.
cudaError_t launch_multi_step(const MultiVox* d_vox, int n_vox, int64_t total_tiles, const MultiSeg* d_segs,
                              int n_segs, int64_t total_chunks, int walk_blocks, unsigned long long* counter,
                              double* chunk_partials, double* tile_partials, cudaStream_t st);
// List of the bins with counts of subset s (bin numbers of the subset, in bin
// order), in two launches per subset: count (tiles: ceil(total / kNzTile)
// ints kept for the write; *n_list) then write.
cudaError_t launch_nz_count(const LorTable& t, SubsetSel s, const void* counts, int counts_dtype, int64_t total,
                            int* tiles, int* n_list, cudaStream_t st);
cudaError_t launch_nz_write(const LorTable& t, SubsetSel s, const void* counts, int counts_dtype, int64_t total,
                            const int* tiles, int* list, cudaStream_t st);
// per_angle[a] += A_a^T 1 for every angle a: n_proj padded images of `lim`
// voxels (PadBuffers' border), [z][x][y] where tr_of[a] else [z][y][x],
// cleared by the caller; one warp per 32 bins in angle order.
cudaError_t launch_scatter_angles(const ImgGeom& g, const LorTable& t, const uint8_t* tr_of, float* per_angle,
                                  unsigned lim, unsigned long long* counter, cudaStream_t st);
// out[s] = the interior sum over the angles a = s, s + nsub, ... of those
// padded images (nsub unpadded images of the geometry).
cudaError_t launch_sum_angles(const float* per_angle, const uint8_t* tr_of, unsigned lim, int n_proj,
                              const ImgGeom& g, int nsub, float* out, cudaStream_t st);
// out[s] = sum over a = s, s + nsub, ... < n_img of img[a] (unpadded images of nvox voxels).
cudaError_t launch_sum_images(const float* img, int n_img, int64_t nvox, int nsub, float* out, cudaStream_t st);
// out[s] = sum over subset s's bins of the additive term (whole-sinogram layout), FP64, fixed order.
cudaError_t launch_subset_sums(const LorTable& t, int nsub, const float* add, double* out, cudaStream_t st);

// Sensitivity of every subset of a job whose sinogram has a multiplicative
// term, in one pass over its whole sinogram: bin (g, a, l) belongs to subset
// a % nsub.
struct SensJob {
  ImgGeom g;
  LorTable t;            // whole sinogram; subset of angle a is a % nsub
  const float* mult;     // null: ones
  float* sens;           // nsub images of nvox
  int64_t blk_begin;
  int64_t nbins;
  int64_t nvox;
  int nsub;
};
cudaError_t launch_sens_batch(const SensJob* d_jobs, int njobs, int64_t nblocks, cudaStream_t st);

}  // namespace apirl

typedef int apirl_status;
struct apirl_image_geom;
struct apirl_sino3d_geom;

// Projector object behind the opaque apirl_projector handle.
struct apirl_projector {
  int device = 0;
  int is3d = 0;
  // The context's persisting-L2 limit before APIRL_OPT_L2_PERSIST raised it
  // (put back when the option is turned off or the projector destroyed).
  bool l2_limit_set = false;
  size_t l2_limit_prev = 0;
  apirl::ImgGeom g{};
  apirl::HostTables host;
  float4* d_lor = nullptr;
  float2* d_z = nullptr;
  uint8_t* d_ok = nullptr;
  apirl::LorTable t{};
  double* d_partials = nullptr;  // per-block likelihood partials, enough for a whole-sinogram pass
  int64_t n_partials = 0;
  unsigned* d_minmax = nullptr;  // threshold reduction keys
  double* d_scalars = nullptr;   // 8 doubles of per-projector scratch (likelihood of host passes)
  int alpha_mode = 0;            // APIRL_ALPHA_F32 (reference arithmetic) or APIRL_ALPHA_F64
  double4* d_lor64 = nullptr;    // FP64-alpha tables, built on first use
  double2* d_z64 = nullptr;
  apirl::PreciseGeom pg;
  int dual_layout = 1;           // fused 3D pass gathers / scatters x-running rays in a transposed copy
  apirl::PadBuffers pad;         // padded two-layout copies of the fused pass (3D), interiors of bA/bT zero
  int timing = 0;                // record CUDA events around the fused kernel
  int em_block = 128;            // threads per block of the fused kernel (APIRL_OPT_EM_BLOCK / autotune)
  int persistent = 1;            // APIRL_OPT_PERSISTENT: warps pull 32-bin chunks (padded 3D pass)
  unsigned long long* d_chunk = nullptr;  // chunk counter of the persistent pass
  int sparse_image = 0;          // APIRL_OPT_SPARSE_IMAGE: 0 = zero-count image Z_s, 1 = geometry image G_s
  apirl::NzList nz;              // list of a subset's bins with counts (sparse passes), grown on demand
  apirl::PadBuffers pad2;        // second padded backprojection pair (bA, bT only), on first use
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // Counts staged ahead of apirl_em_pass_host (apirl_stage_counts): copied on
  // copy_stream; each slot's event is recorded after its copy.
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t copy_ready = nullptr;
  struct Staged {
    const void* host = nullptr;
    void* dev = nullptr;
    cudaEvent_t done = nullptr;
  } staged[4];
  int timed = 0;                 // an event pair has been recorded
  int n_rings = 0;               // 3D geometry as given, for building the FP64 tables
  float r_fov = 0, axial_fov = 0, r_scanner = 0;
  std::vector<int> min_rd, max_rd;
  // Sampled rays (apirl_projector_set_sampling): t carries the rays of
  // Project / Backproject, t_dab those of DivideAndBackproject.
  int scanner = 0;               // APIRL_SCANNER_CYLINDRICAL or APIRL_SCANNER_MMR
  int n_samples = 1, n_axial_samples = 1, multi_lors = 0;
  apirl::LorTable t_dab{};
  float4* d_lor_s[2] = {nullptr, nullptr};
  float2* d_zs[2] = {nullptr, nullptr};
  int* d_zoff[2] = {nullptr, nullptr};
};

// Records `msg` as the calling thread's last error and returns `code`.
apirl_status apirl_internal_fail(apirl_status code, const char* msg);
// APIRL_OK, or APIRL_ERR_CUDA (with the last-error message set) when a CUDA
// error was pending from an earlier launch; reading it resets a non-sticky one.
apirl_status apirl_internal_pending(void);

namespace apirl {
// The host half of apirl_projector_create_3d: geometry checks and host tables
// into p (no device work; p->device and the device tables are not set).
apirl_status setup_3d(const apirl_image_geom* img, const apirl_sino3d_geom* sino, apirl_projector* p);
// Room in p->nz for the list of `total` bins (cudaMalloc: call outside graph
// capture; a captured sparse pass without room walks every bin's chunk).
apirl_status prepare_nz_list(apirl_projector* p, int64_t total);
// img += A_s^T v (vin_mode as load_bin): through the padded pair when the
// projector has it (launch_backproject_pad), else launch_backproject.
cudaError_t backproject_sino(apirl_projector* p, SubsetSel ss, const float* vin, int vin_mode, float* img,
                             cudaStream_t st);
// img += A_s^T v and gimg += A_s^T 1 along one set of walks (a second padded
// backprojection pair, allocated on first use); two backprojections when the
// projector has no padded layout.
apirl_status backproject_sino_and_ones(apirl_projector* p, SubsetSel ss, const float* vin, int vin_mode, float* img,
                                       float* gimg, cudaStream_t st);
}  // namespace apirl

