/*
 * apirl_b200 -- B200-native Siddon projector / backprojector and the MLEM /
 * OSEM update around it, as a C ABI.
 *
 * Every entry point replaces one operation of the reference APIRL CPU path;
 * the reference interface each one stands in for is cited beside it
 * (paths are relative to the APIRL source tree).
 *
 * Conventions
 *  - Status codes: APIRL_OK (0) or one of the APIRL_ERR_* values; the message
 *    of the last failure on the calling thread is apirl_last_error().  Nothing
 *    here calls exit() (the reference's checkCudaErrors does).
 *  - Pointers named d_* are device pointers on the projector's device; h_*
 *    are host pointers.  `stream` is a cudaStream_t passed as void* (NULL =
 *    the legacy default stream).  Device-pointer calls are asynchronous.
 *  - Images are float32 [z][y][x] (Image::pixels, data/inc/Images.h:166).
 *    2D sinograms are float32 [angle][r]; 3D sinograms are
 *    [segment][sinogram][angle][r] with the segment's sinograms in the order
 *    Sinogram3D::readFromInterfile builds them (data/src/Sinogram3D.cpp:396-464).
 *  - Subsets: `subset` in [0, nsubsets) selects angles subset, subset+nsubsets,
 *    ... (Sinogram3DCylindricalPet::getSubset, data/src/Sinogram3DCylindricalPet.cpp:164-197);
 *    subset < 0 means all angles.  A subset sinogram is laid out
 *    [sinogram][subset angle][r] and has apirl_projector_num_bins() bins.
 *  - Voxel indices of Siddon segments are checked against all image bounds.
 *    (The reference checks only one side in its Project: SiddonProjector.cpp:178, :417.)
 *  - A projector owns scratch buffers (likelihood partials, padded image
 *    copies, the persistent pass's chunk counter): the calls made with one
 *    projector must run one after another on the device (one stream, or
 *    streams ordered by the caller).  Different projectors are independent;
 *    calls on different projectors may come from different host threads.
 */
#ifndef APIRL_B200_H
#define APIRL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int apirl_status;
enum {
  APIRL_OK = 0,
  APIRL_ERR_INVALID = 1,       /* bad geometry, size, pointer or argument */
  APIRL_ERR_CUDA = 2,          /* a CUDA runtime call failed */
  APIRL_ERR_OOM = 3,           /* device allocation failed */
  APIRL_ERR_NOT_SUPPORTED = 4, /* option not available on this path */
  APIRL_ERR_ABORTED = 5        /* cancelled or timed out */
};

/* Element type of a measured-counts sinogram. */
enum { APIRL_F32 = 0, APIRL_U32 = 1, APIRL_U16 = 2 };

/* Arithmetic of the Siddon walk (apirl_projector_set_alpha_precision). */
enum { APIRL_ALPHA_F32 = 0, APIRL_ALPHA_F64 = 1 };

/* SizeImage (data/inc/Images.h:53-61). */
typedef struct apirl_image_geom {
  int nx, ny, nz;
  float dx, dy, dz; /* voxel size in mm */
} apirl_image_geom;

/* Sinogram2DinCylindrical3Dpet(nProj, nR, rFov_mm, rScanner_mm)
 * (data/src/Sinogram2DinCylindrical3Dpet.cpp:29-64). */
typedef struct apirl_sino2d_geom {
  int n_proj, n_r;
  float r_fov, r_scanner; /* mm */
} apirl_sino2d_geom;

/* Sinogram3DCylindricalPet(header, rFov_mm, zFov_mm, rScanner_mm) with the
 * header's segment table (data/src/Sinogram3D.cpp:106-471).  scanner =
 * APIRL_SCANNER_MMR selects Sinogram3DSiemensMmr instead, whose r_fov,
 * axial_fov and r_scanner are the scanner's constants (the fields are then
 * ignored); see apirl_projector_create_3d_mmr.  Zero-initialised structs are
 * the cylindrical scanner. */
#define APIRL_SCANNER_CYLINDRICAL 0
#define APIRL_SCANNER_MMR 1
typedef struct apirl_sino3d_geom {
  int n_proj, n_r, n_rings, n_segments;
  float r_fov, axial_fov, r_scanner; /* mm */
  const int* min_ring_diff;          /* n_segments entries */
  const int* max_ring_diff;          /* n_segments entries */
  int scanner;                       /* APIRL_SCANNER_CYLINDRICAL (0) or APIRL_SCANNER_MMR */
} apirl_sino3d_geom;

typedef struct apirl_projector apirl_projector;

const char* apirl_last_error(void);
const char* apirl_version(void);

/* ---- host-only geometry (no device needed) -------------------------------
 * The LOR end-point table [angle][r][p1x,p1y,p2x,p2y] built with the
 * reference's float expressions: r and angle tables of
 * Sinogram2DinCylindrical3Dpet (data/src/Sinogram2DinCylindrical3Dpet.cpp:46-63)
 * and getPointsFromLor (:216-266). */
apirl_status apirl_lor_table(int n_proj, int n_r, float r_fov, float r_scanner, float* h_lor);
/* Number of sinograms of a 3D geometry and, when h_z is not NULL, their
 * end-point z ([sinogram][z1,z2]) as SiddonProjector::Project sets them
 * (recon/src/SiddonProjector.cpp:357-360, :392-396 over the ring pairs of
 * data/src/Sinogram3D.cpp:396-464). */
int apirl_sino3d_ring_z(const apirl_sino3d_geom* sino, float* h_z);

/* ---- projector set-up ---------------------------------------------------
 * SiddonProjector(1, 1) bound to one image and one sinogram geometry
 * (recon/inc/SiddonProjector.h:43-47).  Builds the LOR end-point table on the
 * host with the reference's float expressions
 * (Sinogram2DinCylindrical3Dpet::getPointsFromLor, .cpp:216-266) and keeps it,
 * the per-sinogram ring z and scratch space resident on `device`. */
apirl_status apirl_projector_create_2d(const apirl_image_geom* img, const apirl_sino2d_geom* sino, int device,
                                       apirl_projector** out);
apirl_status apirl_projector_create_3d(const apirl_image_geom* img, const apirl_sino3d_geom* sino, int device,
                                       apirl_projector** out);
/* Siemens Biograph mMR (Sinogram3DSiemensMmr, data/src/Sinogram3DSiemensMmr.cpp;
 * Sinogram2DinSiemensMmr, data/src/Sinogram2DinSiemensMmr.cpp:19-198): scanner
 * radius 328 mm, mean depth of interaction 9.6 mm, 594 mm transaxial and
 * 260 mm axial field of view.  r values are arc-corrected crystal positions
 * (bin 4.0891/2 mm, scaled to 344 bins), angles i * 180 / n_proj, and odd r
 * bins are rotated back by half an angular step; the end points lie on the
 * effective radius 337.6 mm.  The angular step is the whole sinogram's for
 * every subset (the reference's subset sinograms take it from their own
 * angle list, i.e. n_subsets times larger).  Ring pairs and end-point z as for
 * the cylindrical scanner with a 260 mm axial field of view.  Sampling and the
 * FP64-alpha mode are not offered for this geometry.  Equivalent to
 * apirl_projector_create_3d with scanner = APIRL_SCANNER_MMR. */
apirl_status apirl_projector_create_3d_mmr(const apirl_image_geom* img, int n_proj, int n_r, int n_rings,
                                           int n_segments, const int* min_ring_diff, const int* max_ring_diff,
                                           int device, apirl_projector** out);
/* The mMR LOR end-point table on the host ([angle][r][p1x,p1y,p2x,p2y]). */
apirl_status apirl_mmr_lor_table(int n_proj, int n_r, float* h_lor);
void apirl_projector_destroy(apirl_projector* p);
/* Bins of one subset (subset < 0: all angles) of the projector's sinograms
 * (its shard, when one is set). */
int64_t apirl_projector_num_bins(const apirl_projector* p, int subset, int nsubsets);
/* Sinograms of the whole sinogram (independent of a shard). */
int apirl_projector_num_sinograms(const apirl_projector* p);
/* Copies the host-built LOR table ([angle][r][p1x,p1y,p2x,p2y]) and, for 3D,
 * the per-sinogram end-point z ([sinogram][z1,z2]); either may be NULL. */
apirl_status apirl_projector_tables(const apirl_projector* p, float* h_lor, float* h_z);
/* Precision study mode (3D projectors).  APIRL_ALPHA_F32 (default) is the
 * reference's float arithmetic, bit-identical to Siddon.cpp.  APIRL_ALPHA_F64
 * computes LOR end points (double trigonometry), entry/exit alphas, first
 * crossings and the running crossing parameters in FP64 and rounds each
 * segment length to float; projection and accumulation stay FP32.  No
 * counterpart in the reference, whose walk is float only. */
apirl_status apirl_projector_set_alpha_precision(apirl_projector* p, int mode);
/* Several rays per bin (3D projectors):
 * SiddonProjector(nSamplesOnDetector, nAxialSamplesOnDetector)
 * (recon/src/SiddonProjector.cpp:16-32) and
 * Projector::setMultipleLorsPerBin (recon/inc/Projector.h:54-60).  Every bin
 * becomes the sum over multiple_lors_per_bin ? (its ring pairs) : 1 x
 * n_samples radial x n_axial_samples axial rays, in the reference's loop order
 * (SiddonProjector.cpp:346-397): radial samples through
 * getPointsFromOverSampledLor (data/src/Sinogram2DinCylindrical3Dpet.cpp:283-299)
 * at r - dR/2 + (o + 1/2) dR / n_samples, axial samples spread over the ring
 * width.  Project and Backproject use the oversampled end points when
 * n_samples != 1, DivideAndBackproject unless both counts are 1 (:628), as the
 * reference does.  (1, 1, 0) restores one ray per bin.  Sampled projectors run
 * the fused pass on one unpadded layout; the FP64-alpha mode and the batch
 * engine take one ray per bin. */
#define APIRL_MAX_SAMPLES 64
apirl_status apirl_projector_set_sampling(apirl_projector* p, int n_samples, int n_axial_samples,
                                         int multiple_lors_per_bin);
/* Restricts the projector to the sinograms first .. first + n - 1 of the
 * whole sinogram (a LOR shard, for splitting one reconstruction over several
 * GPUs; no counterpart in the reference).  Every operation then covers the
 * shard's bins only: subset and packed sinograms (projections, backprojection
 * inputs, packed counts) hold the shard's sinograms, while whole-sinogram
 * layouts (counts_packed = 0, d_add, multiplicative factors) stay indexed by
 * the global sinogram.  Backprojections and the likelihood are then partial
 * sums over the shard, to be summed over the shards (all-reduce) before the
 * pixel update.  (0, all sinograms) restores the whole sinogram. */
apirl_status apirl_projector_set_shard(apirl_projector* p, int first_sinogram, int n_sinograms);
/* Tuning and instrumentation options (no counterpart in the reference).
 * APIRL_OPT_DUAL_LAYOUT (default 1): the fused 3D pass keeps the image and
 *   the backprojection in two padded layouts, [z][y][x] and [z][x][y], each
 *   with a 2-voxel zero border (4 extra images on the device), and walks rays
 *   running mostly along x in the [z][x][y] one, so that a warp's 32
 *   neighbouring rays touch contiguous memory; rays that stay within the
 *   border skip the per-step bounds tests.  Results equal the 0 setting up to
 *   the order of fp32 additions in the backprojection.
 * APIRL_OPT_KERNEL_TIMING (default 0): record CUDA events around the fused
 *   kernel of every pass; apirl_projector_kernel_ms returns the last one.
 * APIRL_OPT_EM_BLOCK (default 128): threads per block of the fused kernel
 *   (32..256, a multiple of 32).
 * APIRL_OPT_PERSISTENT (default 1): the padded 3D pass runs as a persistent
 *   kernel whose warps pull chunks of 32 bins from a counter (identical
 *   results; the SMs keep their warps busy to the end of the pass).
 * APIRL_OPT_SPARSE_IMAGE (default APIRL_SPARSE_ZERO_COUNT): what the image
 *   and the scalar given to the sparse pass (apirl_em_pass_sparse,
 *   apirl_em_pass_host with d_zimg) hold.  APIRL_SPARSE_ZERO_COUNT: Z_s =
 *   A_s^T 1[m == 0] and the sum of the zero-count bins' additive terms
 *   (apirl_zero_count_image; it depends on the counts).
 *   APIRL_SPARSE_GEOMETRY: G_s = A_s^T 1 over every bin of the subset (a
 *   backprojection of ones, apirl_backproject_ones: the geometry alone, the
 *   sensitivity image itself when there is no multiplicative term) and the
 *   sum of every bin's additive term; the likelihood is then the sum over
 *   bins with counts of m log e, minus x . G_s, minus that sum, which is
 *   sum(m log e - e) over the bins with e != 0 as the reference defines it. */
enum {
  APIRL_OPT_DUAL_LAYOUT = 1,
  APIRL_OPT_KERNEL_TIMING = 2,
  APIRL_OPT_EM_BLOCK = 3,
  APIRL_OPT_PERSISTENT = 4,
  APIRL_OPT_SPARSE_IMAGE = 5,
  APIRL_OPT_ACCUMULATE = 6,
  APIRL_OPT_L2_PERSIST = 7,
  APIRL_OPT_LIST_ORDER = 8,
  APIRL_OPT_GATHER_UNROLL = 9
};
/* APIRL_OPT_GATHER_UNROLL (default 0): segments of a walk whose image loads
 * the persistent fused 3D pass issues before it adds any of them: 4, 6 or 8,
 * or 0 for the pass kind's default (6 over a list of bins, 4 over every bin).
 * Results do not depend on it.  Plain atomics only. */
/* APIRL_OPT_L2_PERSIST (default 0): 1 = the padded 3D passes launch with an L2
 * access policy window over the projector's padded images and
 * backprojections (persisting lines), and the process's persisting-L2 limit
 * on the device is set to that window (as far as the device allows).
 * APIRL_OPT_LIST_ORDER (default 0): order of the sparse passes' list of bins
 * with counts within each tile of 2048 bins.  0 = bin order (neighbouring
 * lanes walk neighbouring rays); n > 0 = within groups of n entries (a power
 * of two, 32..2048) by walk length, longest first (the lanes of a warp walk
 * rays of similar lengths).  Results equal bin order's up to the atomics'
 * order; the likelihood partials then sum in another order. */
enum { APIRL_SPARSE_ZERO_COUNT = 0, APIRL_SPARSE_GEOMETRY = 1 };
/* APIRL_OPT_ACCUMULATE (default APIRL_ACC_ATOMIC): how the 3D passes over the
 * padded layouts (the persistent fused pass, its sparse forms, and
 * apirl_backproject / apirl_backproject_ones) add segment contributions into
 * the backprojection.  APIRL_ACC_ATOMIC: one fp32 atomic add per segment, as
 * the reference's `#pragma omp atomic` (recon/src/SiddonProjector.cpp:547-548).
 * APIRL_ACC_WARP: the lanes of a warp that add to the same voxel in the same
 * step sum their contributions first and one atomic adds the sum.
 * APIRL_ACC_COMPENSATED: every atomic add's rounding error (TwoSum on the
 * value it returns) goes into a second padded pair, folded in when the pass
 * reduces its pair: the backprojection to about twice float precision.  The
 * compensated form allocates two more padded images; set it outside graph
 * capture.  Other paths (2D, FP64 walk, sampled rays, unpadded, the
 * non-persistent pass) accept only APIRL_ACC_ATOMIC. */
enum { APIRL_ACC_ATOMIC = 0, APIRL_ACC_WARP = 1, APIRL_ACC_COMPENSATED = 2 };
apirl_status apirl_projector_set_option(apirl_projector* p, int option, int value);
apirl_status apirl_projector_kernel_ms(apirl_projector* p, double* ms);
/* Autotuner: times the fused kernel (apirl_em_project_backproject, `repeats`
 * runs each, on the caller's counts and image) for block sizes 64..256 and
 * keeps the fastest; its size goes to *best_block.  Allocates one scratch image. */
apirl_status apirl_projector_autotune(apirl_projector* p, const void* d_counts, int counts_dtype, const float* d_x,
                                     int subset, int nsubsets, int repeats, int* best_block, void* stream);
/* The launch shape of the persistent fused 3D pass that runs fastest on this
 * projector's own data: every block size of 64, 96, 128, 192, 256 threads
 * with 4, 6 and 8 gather segments in flight (APIRL_OPT_EM_BLOCK,
 * APIRL_OPT_GATHER_UNROLL), each timed over `repeats` passes of subset
 * `subset` on `stream`: the sparse pass over the bins with counts when
 * d_zimg is given (the zero-count or geometry image, as APIRL_OPT_SPARSE_IMAGE
 * says), else the full pass; the image is not changed.  The projector keeps
 * the fastest; it goes to *out (block, unroll, ms per pass).  Allocates one
 * scratch image.  No counterpart in the reference, whose block sizes come
 * from its .par files (reconGPU/src/CuMlemSinogram3d.cu:157-170). */
typedef struct {
  int block;
  int unroll;
  double ms;
} apirl_tune;
apirl_status apirl_projector_autotune_ex(apirl_projector* p, const void* d_counts, int counts_dtype,
                                        const float* d_x, const float* d_zimg, int subset, int nsubsets, int repeats,
                                        apirl_tune* out, void* stream);
/* Number of Siddon segments of every bin of a subset, written to d_steps (int32). */
apirl_status apirl_count_steps(apirl_projector* p, int subset, int nsubsets, int32_t* d_steps, void* stream);

/* ---- projector operations (device pointers) ------------------------------ */
/* SiddonProjector::Project: d_sino = A d_image (recon/src/SiddonProjector.cpp:322-441
 * for 3D, :146-193 for 2D; 2D bins whose r exceeds the sinogram rFov are left
 * untouched, as the reference leaves them). */
apirl_status apirl_project(apirl_projector* p, const float* d_image, float* d_sino, int subset, int nsubsets,
                           void* stream);
/* SiddonProjector::Backproject: d_image += A^T d_sino (:444-568 for 3D, :34-87
 * for 2D).  Accumulates into d_image, as the reference does. */
apirl_status apirl_backproject(apirl_projector* p, const float* d_sino, float* d_image, int subset, int nsubsets,
                               void* stream);
/* d_image += A^T 1 over the subset's bins: the sensitivity image without
 * multiplicative factors (OsemSinogram3d.cpp:327-346 with no
 * setMultiplicativeProjection), and the geometry image G_s of the sparse pass
 * (APIRL_SPARSE_GEOMETRY).  Needs no sinogram buffer. */
apirl_status apirl_backproject_ones(apirl_projector* p, float* d_image, int subset, int nsubsets, void* stream);
/* apirl_backproject and apirl_backproject_ones along one set of walks:
 * d_image += A^T d_sino and d_ones_image += A^T 1 (the sensitivity image with
 * a multiplicative sinogram, OsemSinogram3d.cpp:327-346, and the geometry
 * image G_s of the sparse pass, for the price of about one backprojection on
 * the 3D padded layout).  The images must be distinct. */
apirl_status apirl_backproject_and_ones(apirl_projector* p, const float* d_sino, float* d_image, float* d_ones_image,
                                        int subset, int nsubsets, void* stream);
/* SiddonProjector::DivideAndBackproject: d_image += A^T (d_meas / d_est)
 * (:571-704 for 3D, :90-144 for 2D, with each reference's zero rules). */
apirl_status apirl_divide_and_backproject(apirl_projector* p, const float* d_meas, const float* d_est,
                                          float* d_image, int subset, int nsubsets, void* stream);

/* generateACFs (cmd/src/generateACFs.cpp:292-330): project an attenuation map
 * (1/mm) and take exp of every non-zero bin, 1 elsewhere: the attenuation
 * correction factors.  Their reciprocals are the multiplicative sinogram of
 * the EM drivers.  exp is CUDA's expf (within 2 ulp of the host's). */
apirl_status apirl_generate_acf(apirl_projector* p, const float* d_mu, float* d_acf, int subset, int nsubsets,
                                void* stream);

/* ---- bin-wise and pixel-wise steps --------------------------------------- */
/* Sinogram3D::inverseDivideBinToBin: d_est = (m != 0 && e != 0) ? m / e : 0
 * (data/src/Sinogram3D.cpp:830-855, Sinogram2D.cpp:245-266). */
apirl_status apirl_inverse_divide(int64_t n, const float* d_meas, float* d_est, void* stream);
/* Sinogram3D::addBinToBin: d_est += d_add (data/src/Sinogram3D.cpp:857-873). */
apirl_status apirl_add_bins(int64_t n, const float* d_add, float* d_est, void* stream);
/* Sinogram{2D,3D}::getLikelihoodValue: sum of m*log(e) - e over bins with
 * e > 0 (gt0 = 1, 2D: Sinogram2D.cpp:565-581) or e != 0 (gt0 = 0, 3D:
 * Sinogram3D.cpp:584-606), accumulated in FP64 and written to *d_out (device double). */
apirl_status apirl_likelihood(int64_t n, const float* d_est, const float* d_meas, int gt0, double* d_out,
                              void* stream);
/* apirl_likelihood without any device allocation.  No counterpart in the
 * reference.  For callers that cannot call cudaMalloc: their device memory is
 * owned by another allocator, or an allocation would stall or fail where they
 * run.  Its scratch is one static device array of 65,536 FP64 partials
 * (512 KiB), so n is limited to APIRL_LIKELIHOOD_NOALLOC_MAX_BINS (larger n:
 * APIRL_ERR_INVALID).  Runs on the calling thread's current device; the first
 * call on a device looks up the array's address there, so make it before any
 * stream capture.  Calls share the array: calls that overlap on the GPU race. */
#define APIRL_LIKELIHOOD_NOALLOC_MAX_BINS ((int64_t)65536 * 4096)
apirl_status apirl_likelihood_noalloc(int64_t n, const float* d_est, const float* d_meas, int gt0, double* d_out,
                                      void* stream);
/* Mlem::updateUpdateThreshold: min over non-zero pixels + 1e-4 (max - min)
 * (recon/src/Mlem.cpp:39-43, data/src/Images.cpp:397-433), written to *d_thr. */
apirl_status apirl_mlem_threshold(int64_t n, const float* d_sens, float* d_thr, void* stream);
/* EM pixel update: x = (sens >= thr | sens > thr) ? x * bp / sens : 0
 * (recon/src/MlemSinogram3d.cpp:228-242 and OsemSinogram3d.cpp:217-237 use >=,
 * Mlem2d.cpp:171-185 uses >).  thr is *d_thr when d_thr is not NULL, else
 * thr_value.  With zero_bp != 0 the kernel also clears d_bp for the next pass. */
apirl_status apirl_update_pixels(int64_t n, float* d_x, float* d_bp, const float* d_sens, const float* d_thr,
                                 float thr_value, int ge, int zero_bp, void* stream);
/* Image::forcePositive (data/src/Images.cpp:383-395). */
apirl_status apirl_force_positive(int64_t n, float* d_x, void* stream);

/* ---- fused EM pass --------------------------------------------------------
 * One OSEM sub-iteration of OsemSinogram3d::Reconstruct
 * (recon/src/OsemSinogram3d.cpp:159-237) -- or one MLEM iteration of
 * Mlem2d::Reconstruct (recon/src/Mlem2d.cpp:146-185) for a 2D projector.
 * One fused kernel does, per bin: project the ray through d_x, add d_add, add
 * the likelihood term, form the ratio m / e and backproject it; a second
 * kernel updates d_x with d_sens (3D projectors with the default layout also
 * copy d_x into their padded layouts first and fold the backprojection back
 * from them; the likelihood is a deterministic two-level FP64 sum).  No
 * estimated sinogram is stored.
 *   d_counts : measured sinogram, element type counts_dtype; counts_packed = 0
 *              means the whole sinogram (angles indexed as in the full
 *              sinogram), 1 means the subset sinogram only.
 *   d_add    : additive term laid out like d_counts (float), or NULL.
 *   d_bp     : zero on entry, zero again on return.
 *   d_lik    : receives the FP64 likelihood of this pass (device double), or NULL.
 *   thr/ge   : as for apirl_update_pixels (d_thr may be NULL).
 */
apirl_status apirl_em_pass(apirl_projector* p, const void* d_counts, int counts_dtype, int counts_packed,
                           const float* d_add, float* d_x, float* d_bp, const float* d_sens, const float* d_thr,
                           float thr_value, int ge, int subset, int nsubsets, double* d_lik, void* stream);

/* Sparse form of apirl_em_pass (3D projectors, one float ray per bin; no
 * counterpart in the reference, whose results it reproduces).  A bin with
 * zero counts has ratio 0, so it adds nothing to the backprojection, and its
 * likelihood term is -e, linear in the image: the sum of those terms is
 * -(x . Z_s) - sum of their additive terms, with Z_s = A_s^T 1[m == 0]
 * fixed by the data.  The pass therefore walks only bins with counts and
 * evaluates the zero-count part as an FP64 dot product.  d_zimg, *d_zero_add:
 * from apirl_zero_count_image for the same counts, subset and additive term
 * (it accumulates into d_zimg: zero it first; d_zero_add may be NULL when
 * there is no additive term).
 * With APIRL_OPT_SPARSE_IMAGE = APIRL_SPARSE_GEOMETRY, d_zimg is instead
 * G_s = A_s^T 1 (apirl_backproject_ones: the geometry alone) and *d_zero_add
 * the sum of every bin's additive term.  Either way the walked bins are
 * listed first (a per-pass list of the bins with counts, in bin order, in a
 * buffer the projector grows outside graph capture), so each warp walks 32
 * bins with counts at a time.
 * The image update equals apirl_em_pass's up to the order of fp32 additions;
 * the FP64 likelihood equals it up to the rounding of the image dot product
 * (~1e-7 relative). */
apirl_status apirl_zero_count_image(apirl_projector* p, const void* d_counts, int counts_dtype, int counts_packed,
                                    const float* d_add, float* d_zimg, double* d_zero_add, int subset, int nsubsets,
                                    void* stream);
apirl_status apirl_em_pass_sparse(apirl_projector* p, const void* d_counts, int counts_dtype, int counts_packed,
                                  const float* d_add, float* d_x, float* d_bp, const float* d_sens,
                                  const float* d_zimg, const double* d_zero_add, const float* d_thr, float thr_value,
                                  int ge, int subset, int nsubsets, double* d_lik, void* stream);

/* The first kernel of apirl_em_pass alone: project, add, likelihood, ratio and
 * backprojection into d_bp, without the pixel update (d_x is only read). */
apirl_status apirl_em_project_backproject(apirl_projector* p, const void* d_counts, int counts_dtype,
                                          int counts_packed, const float* d_add, const float* d_x, float* d_bp,
                                          int subset, int nsubsets, double* d_lik, void* stream);

/* apirl_em_project_backproject as the sparse pass (d_zimg, *d_zero_add as
 * for apirl_em_pass_sparse, per APIRL_OPT_SPARSE_IMAGE): only bins with counts
 * are walked.  For LOR shards, whose backprojections and likelihoods are
 * summed over the shards before the update (each shard with its own Z_s or
 * G_s). */
apirl_status apirl_em_project_backproject_sparse(apirl_projector* p, const void* d_counts, int counts_dtype,
                                                 int counts_packed, const float* d_add, const float* d_x, float* d_bp,
                                                 const float* d_zimg, const double* d_zero_add, int subset,
                                                 int nsubsets, double* d_lik, void* stream);

/* The same pass with HOST inputs and outputs: copies this pass's subset
 * counts (packed, from pinned or pageable host memory) to the device, runs
 * apirl_em_pass on the projector's resident image / sensitivity buffers, and
 * copies the updated image and the likelihood back.  d_x, d_bp, d_sens are
 * device buffers the caller keeps resident between passes.  With d_zimg set
 * the pass is apirl_em_pass_sparse (d_zimg, d_zero_add as there).  h_x_out
 * or h_lik may be NULL (no copy back). */
apirl_status apirl_em_pass_host(apirl_projector* p, const void* h_counts_subset, int counts_dtype, void* d_counts_stage,
                                float* d_x, float* d_bp, const float* d_sens, const float* d_zimg,
                                const double* d_zero_add, float thr_value, int ge, int subset, int nsubsets,
                                float* h_x_out, double* h_lik, void* stream);

/* apirl_em_pass_host without the wait: returns once the pass and its copies
 * are queued on `stream`.  h_x_out and h_lik are written when that work has
 * finished (synchronise the stream or an event recorded after the call);
 * they should be page-locked, since a copy into pageable memory makes the
 * call wait for it.  Queued passes run back to back, with no host round trip
 * between them. */
apirl_status apirl_em_pass_host_async(apirl_projector* p, const void* h_counts_subset, int counts_dtype,
                                      void* d_counts_stage, float* d_x, float* d_bp, const float* d_sens,
                                      const float* d_zimg, const double* d_zero_add, float thr_value, int ge,
                                      int subset, int nsubsets, float* h_x_out, double* h_lik, void* stream);

/* Starts copying a pass's host counts into d_counts_stage on a copy stream of
 * the projector, after the work already queued on `stream` and beside the
 * work queued later, so that the copy for the next pass overlaps the current
 * one.  The next apirl_em_pass_host with the same host pointer and stage
 * waits for this copy instead of copying.  Use two stages, alternating (at
 * most 4 staged copies outstanding per projector). */
apirl_status apirl_stage_counts(apirl_projector* p, const void* h_counts_subset, int counts_dtype, void* d_counts_stage,
                                int subset, int nsubsets, void* stream);

/* ---- whole reconstructions (host buffers) --------------------------------
 * OsemSinogram3d::Reconstruct (recon/src/OsemSinogram3d.cpp:36-325): per-subset
 * sensitivity = A_s^T (h_mult or 1), forcePositive, threshold 0 with >=, then
 * iters x nsubsets fused passes, each captured once as a CUDA graph and
 * replayed.  h_lik receives iters*nsubsets+1 values (the last one for the
 * whole-sinogram projection of the result).  h_mult / h_add may be NULL.
 * sampling: the projector's rays per bin (apirl_projector_set_sampling), or
 * NULL for one ray per bin. */
/* "save estimates at iteration intervals" (OsemSinogram3d.cpp:266-276,
 * MlemSinogram3d.cpp:244-251, Mlem2d.cpp:187-198): the drivers below, when
 * called afterwards on the same thread, hand the image after every iteration
 * t (0-based) with t % interval == 0 to cb (h_image valid during the call).
 * cb NULL or interval 0: no calls (the default). */
typedef void (*apirl_iteration_cb)(int iteration, const float* h_image, int64_t n_voxels, void* user);
apirl_status apirl_set_iteration_hook(apirl_iteration_cb cb, int interval, void* user);

typedef struct {
  int n_samples;             /* numSamplesOnDetector */
  int n_axial_samples;       /* numAxialSamplesOnDetector */
  int multiple_lors_per_bin; /* useMultipleLorsPerBin */
} apirl_sampling;
apirl_status apirl_osem_3d(const apirl_image_geom* img, const apirl_sino3d_geom* sino, const float* h_meas,
                           const float* h_mult, const float* h_add, const float* h_init, int iters, int nsubsets,
                           int device, float* h_out, double* h_lik, float* h_sens0, const apirl_sampling* sampling);
/* MlemSinogram3d::Reconstruct (recon/src/MlemSinogram3d.cpp:89-310): threshold
 * from the sensitivity image, >= update; h_lik gets iters+1 values. */
apirl_status apirl_mlem_3d(const apirl_image_geom* img, const apirl_sino3d_geom* sino, const float* h_meas,
                           const float* h_mult, const float* h_add, const float* h_init, int iters, int device,
                           float* h_out, double* h_lik, float* h_sens, const apirl_sampling* sampling);
/* Mlem2d::Reconstruct (recon/src/Mlem2d.cpp:60-278): > update; h_lik gets
 * iters+1 values, the last evaluated on the ratio sinogram as the reference
 * does (Mlem2d.cpp:228). */
apirl_status apirl_mlem_2d(const apirl_image_geom* img, const apirl_sino2d_geom* sino, const float* h_meas,
                           const float* h_mult, const float* h_add, const float* h_init, int iters, int device,
                           float* h_out, double* h_lik, float* h_sens);

/* The same drivers with the sensitivity images given or returned whole
 * (sensitivityImageFromFile / setSensitivityFilename, Mlem.h:85-119;
 * OsemSinogram3d.cpp:84-116, MlemSinogram3d.cpp:132-151, Mlem2d.cpp:95-112).
 * h_sens_in: OSEM, nsubsets images [subset][voxel], forcePositive applied as
 * the reference does to the images it reads; ML-EM, one image used as is (the
 * threshold is taken from it).  NULL: computed as A^T (mult or 1).
 * h_sens_out: receives every sensitivity image (nsubsets for OSEM), may be
 * NULL.  sampling: as above (NULL: one ray per bin; must be NULL in 2D). */
typedef struct {
  const apirl_sampling* sampling;
  const float* h_sens_in;
  float* h_sens_out;
  /* OSEM pixel update rule.  0: the reference's, x * bp / sens where
   * sens >= 0 with threshold 0 (OsemSinogram3d.cpp:24-33, :217-237), which
   * gives 0 * 0 / 0 = NaN at voxels that no ray of a subset crosses;
   * 1: update where sens > 0, else 0 (those voxels become 0).  Read by
   * apirl_osem_3d_ex only. */
  int update_positive_sens;
  /* Sensitivity images h_sens_out receives: 0 = all of them, n > 0 = the
   * first n subsets' (OSEM). */
  int n_sens_out;
} apirl_recon_options;
apirl_status apirl_osem_3d_ex(const apirl_image_geom* img, const apirl_sino3d_geom* sino, const float* h_meas,
                              const float* h_mult, const float* h_add, const float* h_init, int iters, int nsubsets,
                              int device, float* h_out, double* h_lik, const apirl_recon_options* opts);
apirl_status apirl_mlem_3d_ex(const apirl_image_geom* img, const apirl_sino3d_geom* sino, const float* h_meas,
                              const float* h_mult, const float* h_add, const float* h_init, int iters, int device,
                              float* h_out, double* h_lik, const apirl_recon_options* opts);
apirl_status apirl_mlem_2d_ex(const apirl_image_geom* img, const apirl_sino2d_geom* sino, const float* h_meas,
                              const float* h_mult, const float* h_add, const float* h_init, int iters, int device,
                              float* h_out, double* h_lik, const apirl_recon_options* opts);

/* ---- batched and served reconstructions ---------------------------------
 * Many independent 3D OSEM jobs (OsemSinogram3d::Reconstruct each,
 * recon/src/OsemSinogram3d.cpp:36-325, pixel update sens >= 0 as there) of
 * different geometries advance together: every apirl_batch_step runs one pass
 * of every running job (or its final likelihood) in one persistent walk over
 * all their lists of bins with counts, with the image copies, likelihood sums
 * and updates of all jobs in one launch each.  Jobs are admitted in
 * submission order while their device footprint fits the budget, smaller
 * jobs allowed past one that does not fit; each job's counts are uploaded by
 * a worker thread while other jobs run.  Device memory comes from a pool the
 * batch keeps; finished jobs return theirs to it.  Jobs of one image and
 * sinogram geometry share its tables and A_a^T 1 of every angle (kept, within
 * the budget, while no job needs the room), from which any subset split's
 * sensitivity follows without another walk.  No counterpart in the
 * reference, which reconstructs one sinogram per process. */
typedef struct apirl_batch apirl_batch;
typedef struct apirl_job_desc {
  apirl_image_geom img;
  apirl_sino3d_geom sino;  /* ring-difference arrays are copied by submit */
  const void* h_counts;    /* whole sinogram, element type counts_dtype */
  int counts_dtype;
  const float* h_mult;     /* multiplicative sinogram (sensitivity only) or NULL */
  const float* h_add;      /* additive sinogram or NULL */
  const float* h_init;     /* initial image or NULL (ones) */
  int iters, nsubsets;
  /* 0: the reference's pixel update, sens >= 0 (OsemSinogram3d.cpp:217-237,
   * threshold 0), which gives NaN at voxels no ray of a subset crosses; 1:
   * update only where sens > 0 (apirl_recon_options.update_positive_sens). */
  int update_positive_sens;
} apirl_job_desc;
/* Device bytes a job holds while active (its lists of bins with counts at
 * their largest, and its subset split's sensitivity images, included). */
int64_t apirl_job_footprint(const apirl_job_desc* job);
apirl_status apirl_batch_create(int device, int64_t hbm_budget_bytes, apirl_batch** out);
void apirl_batch_destroy(apirl_batch* b);
/* Queues a job; job ids start at 0.  The host arrays are read after the job
 * is admitted (copied to the device by the batch's worker thread), so they
 * must stay valid until apirl_batch_result reports it done. */
apirl_status apirl_batch_submit(apirl_batch* b, const apirl_job_desc* job, int64_t* job_id);
/* Admits what fits, moves each job whose previous stage has finished on the
 * device to its next one (upload -> lists of bins with counts and
 * sensitivity -> passes -> final likelihood -> result), launches one pass of
 * every running job, retires finished jobs.  Returns once the work is queued
 * (at most two steps are in flight; when nothing could be launched it waits
 * for the oldest outstanding stage).  Counts after the step go to *n_active,
 * *n_queued (either may be NULL). */
apirl_status apirl_batch_step(apirl_batch* b, int* n_active, int* n_queued);
/* *done = 1 and the outputs are filled (image, iters*nsubsets+1 likelihood
 * values) once the job has finished; the job is forgotten afterwards. */
apirl_status apirl_batch_result(apirl_batch* b, int64_t job_id, float* h_out, double* h_lik, int* done);

#ifdef __cplusplus
}
#endif
#endif /* APIRL_B200_H */
