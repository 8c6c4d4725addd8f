// CUDA kernels for sm_100a: Siddon projection, backprojection, the fused EM
// pass and the bin-wise / pixel-wise steps around them.
//
// Layout in HBM
//   image        float [z][y][x]
//   LOR table    float4 [angle][r] (p1x, p1y, p2x, p2y), built on the host
//   ring z       float2 [sinogram] (z1, z2)
//   sinogram     [sinogram][angle][r]; subset sinograms [sinogram][k][r]
//
// Thread mapping: one thread per sinogram bin, consecutive threads on
// consecutive r of the same (sinogram, angle), so that the bin loads and stores
// coalesce and a warp walks 32 near-parallel rays through neighbouring voxels.
#include <cuda_runtime.h>
#include <cstdint>
#include <cfloat>
#include <climits>
#include <atomic>
#include <mutex>
#include <utility>
#include <vector>
#include "internal.h"
#include "siddon.cuh"
#include "../../include/apirl_b200.h"

namespace apirl {

namespace {

constexpr int kBlock = 256;
constexpr int kSumLevel2 = 296;  // first-level blocks of the two-level partial sum (2 per SM)
// Minimum resident 256-thread blocks per SM (register caps).  The
// persistent fused kernel: 6 gives 40 registers (16 B of spill, 48 warps per
// SM), measured 0.9 % faster than 5 (48 registers, 40 warps).  The other
// fused kernels (2D, unpadded 3D, FP64 walk geometry): 5, i.e. 48 registers;
// at 40 the FP64 form spills 184 B and runs at less than half the speed.
#ifndef APIRL_PERSIST_MIN_BLOCKS
#define APIRL_PERSIST_MIN_BLOCKS 6
#endif
#ifndef APIRL_EM_MIN_BLOCKS
#define APIRL_EM_MIN_BLOCKS 5
#endif
constexpr int kPersistMinBlocks = APIRL_PERSIST_MIN_BLOCKS;
// The persistent kernel over a list of the bins with counts (sparse passes)
// is bound by memory latency rather than issue: 5 blocks (48 registers, no
// spill) with six gather segments in flight, measured 0.8 % faster there
// than the full pass's 6 blocks with four segments.
constexpr int kListMinBlocks = 5;
constexpr int kListGatherUnroll = 6;
// The batched walk over many jobs' lists (k_em_multi) reads each segment's
// geometry at run time: at 5 blocks (48 registers) it spilled 48 bytes, at 4
// (64 registers) it does not.
#ifndef APIRL_MULTI_MIN_BLOCKS
#define APIRL_MULTI_MIN_BLOCKS 4
#endif
constexpr int kMultiMinBlocks = APIRL_MULTI_MIN_BLOCKS;
// Gather segments in flight of the batched walk.
#ifndef APIRL_MULTI_UNROLL
#define APIRL_MULTI_UNROLL 6
#endif
constexpr int kMultiGatherUnroll = APIRL_MULTI_UNROLL;
constexpr int kEmMinBlocks = APIRL_EM_MIN_BLOCKS;
// 1: the fused 3D pass sets the walk up a second time for the backprojection
// (fewer live registers during the forward walk).
#ifndef APIRL_EM_RESETUP
#define APIRL_EM_RESETUP 1
#endif

struct BinPos {
  int g, k, l, a;  // sinogram, subset angle, r, full angle
};

__device__ __forceinline__ BinPos decode(int64_t b, const LorTable& t, const SubsetSel& s) {
  BinPos p;
  const int64_t per = (int64_t)s.nk * t.n_r;
  const int gl = (int)(b / per);  // sinogram within the shard
  const int rem = (int)(b - (int64_t)gl * per);
  p.g = t.g0 + gl;
  p.k = rem / t.n_r;
  p.l = rem - p.k * t.n_r;
  p.a = s.subset < 0 ? p.k : s.subset + s.nsub * p.k;
  return p;
}

template <typename CT> __device__ __forceinline__ float load_count(const CT* p, int64_t i);
template <> __device__ __forceinline__ float load_count<float>(const float* p, int64_t i) { return __ldg(p + i); }
template <> __device__ __forceinline__ float load_count<uint32_t>(const uint32_t* p, int64_t i) {
  return (float)__ldg(p + i);
}
template <> __device__ __forceinline__ float load_count<uint16_t>(const uint16_t* p, int64_t i) {
  return (float)__ldg(p + i);
}

// Forward projection of one bin (3D), masked gather of the image.
__device__ __forceinline__ float ray_sum3(const ImgGeom& g, const float4 L, const float2 z, const float* __restrict__ img,
                                          Walk3& w) {
  siddon3_setup(L.x, L.y, z.x, A_SUB(L.z, L.x), A_SUB(L.w, L.y), A_SUB(z.y, z.x), g, w);
  float acc = 0.f;
  siddon3_walk(w, g, [&](bool inb, int idx, float seg) {
    if (inb) acc = A_ADD(acc, A_MUL(seg, __ldg(img + idx)));
  });
  return acc;
}

// Calls f(L, z) for every ray of bin p of a sampled table, in the reference's
// loop order: ring pair, radial sample, axial sample (SiddonProjector.cpp:346-397).
template <class F>
__device__ __forceinline__ void for_rays(const LorTable& t, const BinPos& p, F&& f) {
  const int z0 = __ldg(t.zoff + p.g), nz = __ldg(t.zoff + p.g + 1) - z0;
  const float4* lr = t.lor_s + ((int64_t)p.a * t.n_r + p.l) * t.n_rs;
  for (int mz = 0; mz < nz; mz += t.n_as)
    for (int o = 0; o < t.n_rs; o++) {
      const float4 L = __ldg(lr + o);
      for (int q = 0; q < t.n_as; q++) f(L, __ldg(t.zs + z0 + mz + q));
    }
}

// Forward projection of one bin over all its rays: one running sum, as the
// reference increments the zero-filled bin ray after ray (SiddonProjector.cpp:339,419).
__device__ __forceinline__ float rays_sum3(const ImgGeom& g, const LorTable& t, const BinPos& p,
                                           const float* __restrict__ img) {
  float acc = 0.f;
  for_rays(t, p, [&](const float4 L, const float2 z) {
    Walk3 w;
    siddon3_setup(L.x, L.y, z.x, A_SUB(L.z, L.x), A_SUB(L.w, L.y), A_SUB(z.y, z.x), g, w);
    siddon3_walk(w, g, [&](bool inb, int idx, float seg) {
      if (inb) acc = A_ADD(acc, A_MUL(seg, __ldg(img + idx)));
    });
  });
  return acc;
}

// Scatter of v * segment along every ray of bin p (optionally divided by e).
__device__ __forceinline__ void rays_scatter3(const ImgGeom& g, const LorTable& t, const BinPos& p, float v,
                                              bool divide, float e, float* __restrict__ img) {
  for_rays(t, p, [&](const float4 L, const float2 z) {
    Walk3 w;
    siddon3_setup(L.x, L.y, z.x, A_SUB(L.z, L.x), A_SUB(L.w, L.y), A_SUB(z.y, z.x), g, w);
    siddon3_walk(w, g, [&](bool inb, int idx, float seg) {
      if (!inb) return;
      float val = A_MUL(seg, v);
      if (divide) val = A_DIV(val, e);
      red_add_global(img + idx, val);
    });
  });
}

__device__ __forceinline__ ImgGeomD geom_d(const PreciseGeom& pg) {
  ImgGeomD g;
  g.nx = pg.nx; g.ny = pg.ny; g.nz = pg.nz;
  g.dx = pg.dx; g.dy = pg.dy; g.dz = pg.dz; g.rfov = pg.rfov; g.offz = pg.offz;
  return g;
}

// FP64-alpha forward projection of one bin.
__device__ __forceinline__ float ray_sum3d(const ImgGeomD& g, const double4 L, const double2 z,
                                           const float* __restrict__ img, Walk3D& w) {
  siddon3d_setup(L.x, L.y, z.x, L.z - L.x, L.w - L.y, z.y - z.x, g, w);
  float acc = 0.f;
  siddon3d_walk(w, g, [&](bool inb, int idx, float seg) {
    if (inb) acc = A_ADD(acc, A_MUL(seg, __ldg(img + idx)));
  });
  return acc;
}

__device__ __forceinline__ float ray_sum2(const ImgGeom& g, const float4 L, const float* __restrict__ img, Walk2& w) {
  siddon2_setup(L.x, L.y, A_SUB(L.z, L.x), A_SUB(L.w, L.y), g, w);
  float acc = 0.f;
  siddon2_walk(w, g, [&](bool inb, int idx, float seg) {
    if (inb) acc = A_ADD(acc, A_MUL(seg, __ldg(img + idx)));
  });
  return acc;
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[kBlock / 32];
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double s = 0.0;
  if (wid == 0) {
    s = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  }
  return s;  // valid in thread 0
}

// ---------------------------------------------------------------------------
template <bool F64A>
__global__ void __launch_bounds__(kBlock) k_project3(ImgGeom g, LorTable t, SubsetSel s, PreciseGeom pg,
                                                     const float* __restrict__ img, float* __restrict__ out,
                                                     int64_t total) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= total) return;
  const BinPos p = decode(b, t, s);
  if (F64A) {
    Walk3D w;
    out[b] = ray_sum3d(geom_d(pg), pg.lor[(int64_t)p.a * t.n_r + p.l], pg.z[p.g], img, w);
  } else if (t.lor_s) {
    out[b] = rays_sum3(g, t, p, img);
  } else {
    Walk3 w;
    out[b] = ray_sum3(g, t.lor[(int64_t)p.a * t.n_r + p.l], t.z[p.g], img, w);
  }
}

__global__ void __launch_bounds__(kBlock) k_project2(ImgGeom g, LorTable t, SubsetSel s,
                                                     const float* __restrict__ img, float* __restrict__ out,
                                                     int64_t total) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= total) return;
  const BinPos p = decode(b, t, s);
  if (!t.ok[p.l]) return;  // getPointsFromLor false: the bin is not written (SiddonProjector.cpp:166-173)
  Walk2 w;
  out[b] = ray_sum2(g, t.lor[(int64_t)p.a * t.n_r + p.l], img, w);
}

// divide == 0: Backproject, value = seg * v over bins with v != 0.
// divide == 1: DivideAndBackproject with the 3D zero rules (SiddonProjector.cpp:669-683).
// vin_mode: 0 = vin is a subset sinogram, 1 = vin is the whole sinogram (read at
// this subset's angles), 2 = every bin is 1 (sensitivity of ones).
__device__ __forceinline__ float load_bin(const float* __restrict__ v, int vin_mode, int64_t b, const BinPos& p,
                                          const LorTable& t) {
  if (vin_mode == 2) return 1.f;
  if (vin_mode == 1) return __ldg(v + ((int64_t)p.g * t.n_proj + p.a) * t.n_r + p.l);
  return __ldg(v + b);
}

template <bool F64A>
__global__ void __launch_bounds__(kBlock) k_backproject3(ImgGeom g, LorTable t, SubsetSel s, PreciseGeom pg,
                                                         const float* __restrict__ vin, int vin_mode,
                                                         const float* __restrict__ vest, int divide,
                                                         float* __restrict__ img, int64_t total) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= total) return;
  const BinPos p = decode(b, t, s);
  const float v = load_bin(vin, vin_mode, b, p, t);
  if (v == 0.f) return;
  const float e = divide ? vest[b] : 0.f;
  if (!F64A && t.lor_s) {
    rays_scatter3(g, t, p, v, divide && e != 0.f, e, img);
    return;
  }
  auto scatter = [&](bool inb, int idx, float seg) {
    if (!inb) return;
    float val = A_MUL(seg, v);
    if (divide && e != 0.f) val = A_DIV(val, e);
    red_add_global(img + idx, val);
  };
  if (F64A) {
    const ImgGeomD gd = geom_d(pg);
    const double4 L = pg.lor[(int64_t)p.a * t.n_r + p.l];
    const double2 z = pg.z[p.g];
    Walk3D w;
    siddon3d_setup(L.x, L.y, z.x, L.z - L.x, L.w - L.y, z.y - z.x, gd, w);
    siddon3d_walk(w, gd, scatter);
  } else {
    const float4 L = t.lor[(int64_t)p.a * t.n_r + p.l];
    const float2 z = t.z[p.g];
    Walk3 w;
    siddon3_setup(L.x, L.y, z.x, A_SUB(L.z, L.x), A_SUB(L.w, L.y), A_SUB(z.y, z.x), g, w);
    siddon3_walk(w, g, scatter);
  }
}

// divide == 0: Backproject over every bin (SiddonProjector.cpp:34-87).
// divide == 1: DivideAndBackproject, only bins with e != 0 and m != 0 (:110).
__global__ void __launch_bounds__(kBlock) k_backproject2(ImgGeom g, LorTable t, SubsetSel s,
                                                         const float* __restrict__ vin, int vin_mode,
                                                         const float* __restrict__ vest, int divide,
                                                         float* __restrict__ img, int64_t total) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= total) return;
  const BinPos p = decode(b, t, s);
  const float v = load_bin(vin, vin_mode, b, p, t);
  const float e = divide ? vest[b] : 1.f;
  if (divide && !(e != 0.f && v != 0.f)) return;
  if (v == 0.f) return;  // adding seg * 0 leaves every voxel unchanged
  if (!t.ok[p.l]) return;
  const float4 L = t.lor[(int64_t)p.a * t.n_r + p.l];
  Walk2 w;
  siddon2_setup(L.x, L.y, A_SUB(L.z, L.x), A_SUB(L.w, L.y), g, w);
  siddon2_walk(w, g, [&](bool inb, int idx, float seg) {
    if (!inb) return;
    float val = A_MUL(seg, v);
    if (divide) val = A_DIV(val, e);
    red_add_global(img + idx, val);
  });
}

__global__ void __launch_bounds__(kBlock) k_count_steps(ImgGeom g, LorTable t, SubsetSel s, int32_t* steps,
                                                        int64_t total) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= total) return;
  const BinPos p = decode(b, t, s);
  if (t.is3d && t.lor_s) {
    int n = 0;
    for_rays(t, p, [&](const float4 L, const float2 z) {
      Walk3 w;
      siddon3_setup(L.x, L.y, z.x, A_SUB(L.z, L.x), A_SUB(L.w, L.y), A_SUB(z.y, z.x), g, w);
      n += w.n;
    });
    steps[b] = n;
    return;
  }
  const float4 L = t.lor[(int64_t)p.a * t.n_r + p.l];
  if (t.is3d) {
    const float2 z = t.z[p.g];
    Walk3 w;
    siddon3_setup(L.x, L.y, z.x, A_SUB(L.z, L.x), A_SUB(L.w, L.y), A_SUB(z.y, z.x), g, w);
    steps[b] = w.n;
  } else {
    Walk2 w;
    w.n = 0;
    if (t.ok[p.l]) siddon2_setup(L.x, L.y, A_SUB(L.z, L.x), A_SUB(L.w, L.y), g, w);
    steps[b] = w.n;
  }
}

// A walked bin's likelihood term (Sinogram3D::getLikelihoodValue,
// data/src/Sinogram3D.cpp:584-606: m log e - e over e != 0).  skip_zero:
// 0 = every bin walked; 1 = zero-count bins not walked, their -e supplied by
// -x . Z_s (Z_s = A_s^T 1[m == 0]); 2 = zero-count bins not walked and the
// -e of every bin supplied by -x . G_s - sum(add) (G_s = A_s^T 1, a
// geometry image), so a walked bin adds m log e alone.
__device__ __forceinline__ double lik_term(float m, float e, int skip_zero) {
  return skip_zero == 2 ? (double)m * log((double)e) : (double)m * log((double)e) - (double)e;
}

// ---------------------------------------------------------------------------
// Fused EM pass: project, add, likelihood term, ratio, backproject.
// lik_mode: 0 = term over e != 0 (3D), 1 = over e > 0 (2D), 2 = over the ratio
// r > 0 (the final 2D value, Mlem2d.cpp:228).  back = 0 skips the backprojection.
// pad.pA set (3D): the pass reads the image from the padded two-layout copies
// and scatters into the padded backprojection pair (see PadBuffers); else it
// uses x and bp directly.
template <typename CT, bool IS3D, bool F64A>
__global__ void __launch_bounds__(kBlock, kEmMinBlocks) k_em_pass(ImgGeom g, LorTable t, SubsetSel s, PreciseGeom pg,
                                                    const CT* __restrict__ counts,
                                                    int counts_packed, const float* __restrict__ add,
                                                    const float* __restrict__ x, float* __restrict__ bp,
                                                    PadBuffers pad, int back,
                                                    int lik_mode, double* __restrict__ partials, int64_t total,
                                                    int skip_zero) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double term = 0.0;
  if (b < total) {
    const BinPos p = decode(b, t, s);
    const int64_t row = counts_packed ? ((int64_t)(p.g - t.g0) * s.nk + p.k) : ((int64_t)p.g * t.n_proj + p.a);
    const int64_t ci = row * t.n_r + p.l;
    const float m = load_count<CT>(counts, ci);
    const float4 L = t.lor[(int64_t)p.a * t.n_r + p.l];
    if (skip_zero && m == 0.f) {
      // Sparse pass: a zero-count bin's ratio is 0 and its likelihood term
      // -e is linear in the image; the caller's zero-count or geometry image
      // supplies the sum of those terms (k_neg_dot), so the bin is not walked.
    } else if (IS3D && F64A) {
      const ImgGeomD gd = geom_d(pg);
      Walk3D w;
      float e = ray_sum3d(gd, pg.lor[(int64_t)p.a * t.n_r + p.l], pg.z[p.g], x, w);
      if (add) e = A_ADD(e, __ldg(add + ci));
      const float r = (m != 0.f && e != 0.f) ? A_DIV(m, e) : 0.f;
      if (lik_mode == 2) { if (r > 0.f) term = (double)m * log((double)r) - (double)r; }
      else if (lik_mode == 1 ? (e > 0.f) : (e != 0.f)) term = (double)m * log((double)e) - (double)e;
      if (back && r != 0.f)
        siddon3d_walk(w, gd, [&](bool inb, int idx, float seg) {
          if (inb) red_add_global(bp + idx, A_MUL(seg, r));
        });
    } else if (IS3D && pad.pA) {
      // Two padded layouts: rays running mostly along x use the transposed
      // copy, so that a warp's neighbouring rays touch contiguous addresses.
      const float2 z = t.z[p.g];
      const float vx = A_SUB(L.z, L.x), vy = A_SUB(L.w, L.y);
      const bool tr = fabsf(vx) >= fabsf(vy);
      const int px = g.nx + 2 * kPad, py = g.ny + 2 * kPad;
      const int uz = px * py;
      const int ux = tr ? py : 1, uy = tr ? 1 : px;
      Walk3 w;
      siddon3_setup(L.x, L.y, z.x, vx, vy, A_SUB(z.y, z.x), g, w);
      float e = siddon3_gather_pad(w, g, ux, uy, uz, pad.lim, tr ? pad.pT : pad.pA);
      if (add) e = A_ADD(e, __ldg(add + ci));
      const float r = (m != 0.f && e != 0.f) ? A_DIV(m, e) : 0.f;
      if (lik_mode == 2) { if (r > 0.f) term = (double)m * log((double)r) - (double)r; }
      else if (lik_mode == 1 ? (e > 0.f) : (e != 0.f)) term = lik_term(m, e, skip_zero);
#if APIRL_EM_RESETUP
      // The walk is set up again from the tables for the backprojection
      // instead of keeping the set-up state live through the forward walk.
      if (back && r != 0.f) {
        const float4 L2 = __ldcg(t.lor + (int64_t)p.a * t.n_r + p.l);
        const float2 z2 = __ldcg(t.z + p.g);
        Walk3 w2;
        siddon3_setup(L2.x, L2.y, z2.x, A_SUB(L2.z, L2.x), A_SUB(L2.w, L2.y), A_SUB(z2.y, z2.x), g, w2);
        siddon3_scatter_pad(w2, g, ux, uy, uz, pad.lim, r, tr ? pad.bT : pad.bA);
      }
#else
      if (back && r != 0.f) siddon3_scatter_pad(w, g, ux, uy, uz, pad.lim, r, tr ? pad.bT : pad.bA);
#endif
    } else if (IS3D) {
      Walk3 w;
      float e = ray_sum3(g, L, t.z[p.g], x, w);
      if (add) e = A_ADD(e, __ldg(add + ci));
      const float r = (m != 0.f && e != 0.f) ? A_DIV(m, e) : 0.f;
      if (lik_mode == 2) { if (r > 0.f) term = (double)m * log((double)r) - (double)r; }
      else if (lik_mode == 1 ? (e > 0.f) : (e != 0.f)) term = lik_term(m, e, skip_zero);
      if (back && r != 0.f)
        siddon3_walk(w, g, [&](bool inb, int idx, float seg) {
          if (inb) red_add_global(bp + idx, A_MUL(seg, r));
        });
    } else {
      Walk2 w;
      const bool ray = t.ok[p.l] != 0;
      float e = 0.f;
      if (ray) e = ray_sum2(g, L, x, w);
      if (add) e = A_ADD(e, __ldg(add + ci));
      const float r = (m != 0.f && e != 0.f) ? A_DIV(m, e) : 0.f;
      if (lik_mode == 2) { if (r > 0.f) term = (double)m * log((double)r) - (double)r; }
      else if (lik_mode == 1 ? (e > 0.f) : (e != 0.f)) term = (double)m * log((double)e) - (double)e;
      if (back && ray && r != 0.f)
        siddon2_walk(w, g, [&](bool inb, int idx, float seg) {
          if (inb) red_add_global(bp + idx, A_MUL(seg, r));
        });
    }
  }
  // Warp-level partial, no block barrier: warps whose rays are short retire
  // without waiting for the block's longest ray.
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) term += __shfl_down_sync(0xffffffffu, term, o);
  if ((threadIdx.x & 31) == 0) partials[((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5] = term;
}

// The fused pass for sampled tables (several rays per bin, 3D): the bin's
// estimate is the running sum over its rays, the ratio is scattered along
// every ray.  Single [z][y][x] layout, bounds-tested walks.
template <typename CT>
__global__ void __launch_bounds__(kBlock) k_em_pass_rays(ImgGeom g, LorTable t, SubsetSel s,
                                                         const CT* __restrict__ counts, int counts_packed,
                                                         const float* __restrict__ add, const float* __restrict__ x,
                                                         float* __restrict__ bp, int back, int lik_mode,
                                                         double* __restrict__ partials, int64_t total) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double term = 0.0;
  if (b < total) {
    const BinPos p = decode(b, t, s);
    const int64_t row = counts_packed ? ((int64_t)(p.g - t.g0) * s.nk + p.k) : ((int64_t)p.g * t.n_proj + p.a);
    const int64_t ci = row * t.n_r + p.l;
    const float m = load_count<CT>(counts, ci);
    float e = rays_sum3(g, t, p, x);
    if (add) e = A_ADD(e, __ldg(add + ci));
    const float r = (m != 0.f && e != 0.f) ? A_DIV(m, e) : 0.f;
    if (lik_mode == 2) { if (r > 0.f) term = (double)m * log((double)r) - (double)r; }
    else if (lik_mode == 1 ? (e > 0.f) : (e != 0.f)) term = (double)m * log((double)e) - (double)e;
    if (back && r != 0.f) rays_scatter3(g, t, p, r, false, 0.f, bp);
  }
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) term += __shfl_down_sync(0xffffffffu, term, o);
  if ((threadIdx.x & 31) == 0) partials[((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5] = term;
}

// The warp-aggregated scatter of one bin's ratio r along its ray; every lane
// of the warp calls it (live == false: nothing to add).
__device__ __forceinline__ void scatter_bin_warp(const ImgGeom& g, const LorTable& t, const BinPos& p, bool live,
                                                 float r, const PadBuffers& pad) {
  const int px = g.nx + 2 * kPad, py = g.ny + 2 * kPad;
  Walk3 w;
  w.n = 0;
  bool tr = false;
  if (live) {
    const float4 L = __ldcg(t.lor + (int64_t)p.a * t.n_r + p.l);
    const float2 z = __ldcg(t.z + p.g);
    const float vx = A_SUB(L.z, L.x), vy = A_SUB(L.w, L.y);
    tr = fabsf(vx) >= fabsf(vy);
    siddon3_setup(L.x, L.y, z.x, vx, vy, A_SUB(z.y, z.x), g, w);
  }
  siddon3_scatter_pad_warp(w, g, tr ? py : 1, tr ? 1 : px, px * py, pad.lim, r, tr ? pad.bT : pad.bA, live);
}

// ---- backprojection over the padded pair (3D, one float ray per bin) -------
// The fused pass's scatter alone: warps pull 32-bin chunks from a counter
// and scatter seg * v into the padded backprojection pair (rays running
// mostly along x into the transposed one), which k_pad_reduce then folds
// into the image.  v is the bin's value (vin_mode as load_bin); bins with
// v == 0 are not walked, as SiddonProjector::Backproject skips them
// (SiddonProjector.cpp:496).
// b2A / b2T set: the walk also scatters seg into that second padded pair,
// for every bin (the unweighted image A_s^T 1 beside A_s^T v).
template <int ACC>
__global__ void __launch_bounds__(kBlock, kPersistMinBlocks) k_scatter_persist(
    ImgGeom g, LorTable t, SubsetSel s, const float* __restrict__ vin, int vin_mode, PadBuffers pad, int64_t total,
    unsigned long long* __restrict__ chunk_counter, float* __restrict__ b2A, float* __restrict__ b2T) {
  const int lane = threadIdx.x & 31;
  const int64_t nchunks = (total + 31) >> 5;
  const int px = g.nx + 2 * kPad, py = g.ny + 2 * kPad;
  const int uz = px * py;
  for (;;) {
    unsigned long long c = 0;
    if (lane == 0) c = atomicAdd(chunk_counter, 1ULL);
    c = __shfl_sync(0xffffffffu, c, 0);
    if ((int64_t)c >= nchunks) break;
    const int64_t b = (int64_t)c * 32 + lane;
    if (ACC == 1) {  // warp-aggregated: the whole warp scatters together
      BinPos p{0, 0, 0, 0};
      float v = 0.f;
      if (b < total) {
        p = decode(b, t, s);
        v = load_bin(vin, vin_mode, b, p, t);
      }
      scatter_bin_warp(g, t, p, v != 0.f, v, pad);
      continue;
    }
    if (b < total) {
      const BinPos p = decode(b, t, s);
      const float v = load_bin(vin, vin_mode, b, p, t);
      if (v != 0.f || b2A) {
        const float4 L = t.lor[(int64_t)p.a * t.n_r + p.l];
        const float2 z = t.z[p.g];
        const float vx = A_SUB(L.z, L.x), vy = A_SUB(L.w, L.y);
        const bool tr = fabsf(vx) >= fabsf(vy);
        Walk3 w;
        siddon3_setup(L.x, L.y, z.x, vx, vy, A_SUB(z.y, z.x), g, w);
        if (b2A)
          siddon3_scatter2_pad(w, g, tr ? py : 1, tr ? 1 : px, uz, pad.lim, v, tr ? pad.bT : pad.bA, tr ? b2T : b2A);
        else
          siddon3_scatter_pad<ACC>(w, g, tr ? py : 1, tr ? 1 : px, uz, pad.lim, v, tr ? pad.bT : pad.bA,
                                   tr ? pad.eT : pad.eA);
      }
    }
  }
}

// ---- list of the bins with counts (the sparse pass's persistent form) -----
// Tiles of kNzTile (internal.h) consecutive bins of the subset: k_nz_tiles counts each
// tile's bins with counts, k_nz_scan turns the counts into the tiles' first
// list positions and the list length, k_nz_write writes the bin numbers in
// bin order.  Deterministic: the list depends on the counts alone.
constexpr int kNzBlock = 256;

// The list is used for fewer than 2^31 bins, so bin numbers decode in 32-bit
// integer arithmetic here (decode's 64-bit divisions made these streaming
// kernels instruction-bound).
template <typename CT>
__device__ __forceinline__ bool bin_has_count(int64_t b64, const LorTable& t, const SubsetSel& s, const CT* counts,
                                              int counts_packed) {
  const int b = (int)b64;
  const int per = s.nk * t.n_r;
  const int gl = b / per;
  const int rem = b - gl * per;
  const int k = rem / t.n_r;
  const int l = rem - k * t.n_r;
  const int g = t.g0 + gl;
  const int a = s.subset < 0 ? k : s.subset + s.nsub * k;
  const int64_t row = counts_packed ? ((int64_t)gl * s.nk + k) : ((int64_t)g * t.n_proj + a);
  return load_count<CT>(counts, row * t.n_r + l) != 0.f;
}

// Whether each of a thread's kNzTile / kNzBlock bins of its tile (bins
// base + threadIdx.x + kNzBlock * i) has counts.  The first bin is decoded
// once and the others by stepping (r, then subset angle, then sinogram)
// without dividing, and every count is loaded before any is tested, so that
// the thread's loads are in flight together.
constexpr int kNzPerThread = kNzTile / kNzBlock;
template <typename CT>
__device__ __forceinline__ void tile_has_counts(int64_t base, int64_t total, const LorTable& t, const SubsetSel& s,
                                                const CT* __restrict__ counts, int counts_packed,
                                                bool (&has)[kNzPerThread]) {
  const int per = s.nk * t.n_r;
  const int b0 = (int)base + (int)threadIdx.x;
  int gl = b0 / per;
  int rem = b0 - gl * per;
  int k = rem / t.n_r;
  int l = rem - k * t.n_r;
  float m[kNzPerThread];
  #pragma unroll
  for (int i = 0; i < kNzPerThread; i++) {
    const bool in = base + threadIdx.x + (int64_t)kNzBlock * i < total;
    const int a = s.subset < 0 ? k : s.subset + s.nsub * k;
    const int64_t row = counts_packed ? ((int64_t)gl * s.nk + k) : ((int64_t)(t.g0 + gl) * t.n_proj + a);
    m[i] = in ? load_count<CT>(counts, row * t.n_r + l) : 0.f;
    l += kNzBlock;
    while (l >= t.n_r) {
      l -= t.n_r;
      if (++k == s.nk) { k = 0; ++gl; }
    }
  }
  #pragma unroll
  for (int i = 0; i < kNzPerThread; i++) has[i] = m[i] != 0.f;
}

template <typename CT>
__global__ void __launch_bounds__(kNzBlock) k_nz_tiles(LorTable t, SubsetSel s, const CT* __restrict__ counts,
                                                       int counts_packed, int64_t total, int* __restrict__ tiles) {
  __shared__ int warp_n[kNzBlock / 32];
  const int64_t base = (int64_t)blockIdx.x * kNzTile;
  bool has[kNzPerThread];
  tile_has_counts<CT>(base, total, t, s, counts, counts_packed, has);
  int n = 0;
  #pragma unroll
  for (int i = 0; i < kNzPerThread; i++) n += has[i] ? 1 : 0;
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(0xffffffffu, n, o);
  if ((threadIdx.x & 31) == 0) warp_n[threadIdx.x >> 5] = n;
  __syncthreads();
  if (threadIdx.x == 0) {
    int sum = 0;
    for (int w = 0; w < kNzBlock / 32; w++) sum += warp_n[w];
    tiles[blockIdx.x] = sum;
  }
}

// One block: tiles[i] <- sum of tiles[0..i-1]; *n_list <- sum of all.
__global__ void __launch_bounds__(1024) k_nz_scan(int* __restrict__ tiles, int n_tiles, int* __restrict__ n_list) {
  __shared__ int warp_sum[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int base = 0; base < n_tiles; base += 1024) {
    const int i = base + (int)threadIdx.x;
    const int v = i < n_tiles ? tiles[i] : 0;
    int incl = v;
    #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    if (lane == 31) warp_sum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      int w = warp_sum[lane];
      #pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += u;
      }
      warp_sum[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const int before = carry + (warp > 0 ? warp_sum[warp - 1] : 0) + incl - v;
    if (i < n_tiles) tiles[i] = before;
    __syncthreads();
    if (threadIdx.x == 0) carry += warp_sum[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) *n_list = carry;
}

template <typename CT>
__global__ void __launch_bounds__(kNzBlock) k_nz_write(LorTable t, SubsetSel s, const CT* __restrict__ counts,
                                                       int counts_packed, int64_t total,
                                                       const int* __restrict__ tiles, int* __restrict__ list) {
  // Entries go to the list in bin order: sub-tile q (bins base + kNzBlock q
  // + thread), then warp, then lane.  cnt[q][w]: warp w's entries in sub-tile
  // q, turned into the tile-relative offset of that group in one pass.
  __shared__ int cnt[kNzPerThread][kNzBlock / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t base = (int64_t)blockIdx.x * kNzTile;
  bool hs[kNzPerThread];
  tile_has_counts<CT>(base, total, t, s, counts, counts_packed, hs);
  unsigned mask[kNzPerThread];
  #pragma unroll
  for (int q = 0; q < kNzPerThread; q++) {
    mask[q] = __ballot_sync(0xffffffffu, hs[q]);
    if (lane == 0) cnt[q][warp] = __popc(mask[q]);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = tiles[blockIdx.x];
    for (int q = 0; q < kNzPerThread; q++)
      for (int w = 0; w < kNzBlock / 32; w++) {
        const int c = cnt[q][w];
        cnt[q][w] = run;
        run += c;
      }
  }
  __syncthreads();
  const unsigned below = (1u << lane) - 1u;
  #pragma unroll
  for (int q = 0; q < kNzPerThread; q++)
    if (hs[q]) list[cnt[q][warp] + __popc(mask[q] & below)] = (int)(base + (int64_t)kNzBlock * q + threadIdx.x);
}

// One bin of the padded-layout fused pass: forward walk over the padded copy
// of the image that suits the ray's direction (x-running rays: [z][x][y]),
// the additive term, the likelihood term, the ratio m / e and the scatter of
// seg * ratio into the matching padded backprojection.  ci: the bin's index
// in the counts / additive layout.  Returns the likelihood term (lik_term).
// Accumulation form 1 (warp-aggregated) scatters outside, with the whole
// warp (scatter_bin_warp): the ratio is handed back in *r_out instead.
// Walk start delays (walk_delay) that line up the lanes of a warp: 0 none,
// 1 the scatter walk, 2 the gather walk too.  On B200 both forms made the
// listed pass 4-5 % slower (fewer load sectors, more instructions), so the
// default is 0.
#ifndef APIRL_ALIGN_WALKS
#define APIRL_ALIGN_WALKS 0
#endif
template <int U, int ACC>
__device__ __forceinline__ double em_bin_pad(const ImgGeom& g, const LorTable& t, const BinPos& p, float m,
                                             int64_t ci, const float* __restrict__ add, const PadBuffers& pad,
                                             int back, int skip_zero, float* r_out = nullptr) {
  const int px = g.nx + 2 * kPad, py = g.ny + 2 * kPad;
  const int uz = px * py;
  const float4 L = t.lor[(int64_t)p.a * t.n_r + p.l];
  const float2 z = t.z[p.g];
  const float vx = A_SUB(L.z, L.x), vy = A_SUB(L.w, L.y);
  const bool tr = fabsf(vx) >= fabsf(vy);
  const int ux = tr ? py : 1, uy = tr ? 1 : px;
  Walk3 w;
  const float vz = A_SUB(z.y, z.x);
  siddon3_setup(L.x, L.y, z.x, vx, vy, vz, g, w);
#if APIRL_ALIGN_WALKS >= 2
  const int delay = walk_delay(w, g, L.x, L.y, vx, vy, vz, (unsigned)p.g * 65536u + (unsigned)p.a);
#else
  const int delay = 0;
#endif
  float e = siddon3_gather_pad<U>(w, g, ux, uy, uz, pad.lim, tr ? pad.pT : pad.pA, delay);
  if (add) e = A_ADD(e, __ldg(add + ci));
  const float r = (m != 0.f && e != 0.f) ? A_DIV(m, e) : 0.f;
  const double term = e != 0.f ? lik_term(m, e, skip_zero) : 0.0;
  if (ACC == 1) {
    *r_out = r;
    return term;
  }
  if (back && r != 0.f) {
    const float4 L2 = __ldcg(t.lor + (int64_t)p.a * t.n_r + p.l);
    const float2 z2 = __ldcg(t.z + p.g);
    Walk3 w2;
    const float vx2 = A_SUB(L2.z, L2.x), vy2 = A_SUB(L2.w, L2.y), vz2 = A_SUB(z2.y, z2.x);
    siddon3_setup(L2.x, L2.y, z2.x, vx2, vy2, vz2, g, w2);
#if APIRL_ALIGN_WALKS >= 1
    const int delay2 = walk_delay(w2, g, L2.x, L2.y, vx2, vy2, vz2, (unsigned)p.g * 65536u + (unsigned)p.a);
#else
    const int delay2 = 0;
#endif
    siddon3_scatter_pad<ACC>(w2, g, ux, uy, uz, pad.lim, r, tr ? pad.bT : pad.bA, tr ? pad.eT : pad.eA, delay2);
  }
  return term;
}

// k_nz_write with the tile's entries ordered by walk length (APIRL_OPT_LIST_ORDER):
// the tile's bins with counts are gathered in bin order into shared memory,
// each gets its walk's segment count as key, and every aligned group of
// `group` entries (a power of two <= kNzTile) is sorted, longest walk first
// (ties: lower bin first), by a bitonic network; the entries keep their
// tile's place in the list.
template <typename CT>
__global__ void __launch_bounds__(kNzBlock) k_nz_write_sorted(ImgGeom g, LorTable t, SubsetSel s,
                                                              const CT* __restrict__ counts, int counts_packed,
                                                              int64_t total, const int* __restrict__ tiles,
                                                              int* __restrict__ list, int group) {
  __shared__ int key[kNzTile];
  __shared__ int val[kNzTile];
  __shared__ int warp_n[kNzBlock / 32];
  __shared__ int run;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) run = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kNzTile;
  for (int i = 0; i < kNzTile; i += kNzBlock) {
    const int64_t b = base + i + threadIdx.x;
    const bool has = b < total && bin_has_count<CT>(b, t, s, counts, counts_packed);
    const unsigned mask = __ballot_sync(0xffffffffu, has);
    if (lane == 0) warp_n[warp] = __popc(mask);
    __syncthreads();
    int off = run;
    for (int w = 0; w < warp; w++) off += warp_n[w];
    if (has) val[off + __popc(mask & ((1u << lane) - 1u))] = (int)b;
    __syncthreads();
    if (threadIdx.x == 0) {
      int sum = 0;
      for (int w = 0; w < kNzBlock / 32; w++) sum += warp_n[w];
      run += sum;
    }
    __syncthreads();
  }
  const int cnt = run;
  for (int i = threadIdx.x; i < kNzTile; i += kNzBlock) {
    if (i < cnt) {
      const BinPos p = decode((int64_t)val[i], t, s);
      const float4 L = t.lor[(int64_t)p.a * t.n_r + p.l];
      const float2 z = t.z[p.g];
      Walk3 w;
      siddon3_setup(L.x, L.y, z.x, A_SUB(L.z, L.x), A_SUB(L.w, L.y), A_SUB(z.y, z.x), g, w);
      key[i] = w.n;
    } else {
      key[i] = -1;  // after every real entry of its group
      val[i] = INT_MAX;
    }
  }
  __syncthreads();
  // entry a goes before entry b: the longer walk, then the lower bin
  auto before = [](int ka, int va, int kb, int vb) { return ka > kb || (ka == kb && va < vb); };
  for (int k = 2; k <= group; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < kNzTile; i += kNzBlock) {
        const int l = i ^ j;
        if (l > i) {
          // final stage: every group in the same direction
          const bool fwd = k == group || (i & k) == 0;
          const bool swap = fwd ? before(key[l], val[l], key[i], val[i]) : before(key[i], val[i], key[l], val[l]);
          if (swap) {
            const int tk = key[i], tv = val[i];
            key[i] = key[l]; val[i] = val[l];
            key[l] = tk; val[l] = tv;
          }
        }
      }
      __syncthreads();
    }
  const int off = tiles[blockIdx.x];
  for (int i = threadIdx.x; i < cnt; i += kNzBlock) list[off + i] = val[i];
}

// The padded-layout fused pass as a persistent kernel: each warp takes the
// next chunk of 32 consecutive bins from *chunk_counter until none are left,
// so that warps never wait for the rest of their block and the SM keeps its
// full complement of warps until the end of the pass.  The bins of a chunk
// are those of one warp in k_em_pass, and the chunk's likelihood partial goes
// to partials[chunk]: results are identical to k_em_pass's.
// UNROLL: gather segments in flight (0: the default of the pass kind,
// kListGatherUnroll listed, APIRL_GATHER_UNROLL full).
template <typename CT, bool LIST, int ACC, int UNROLL>
__global__ void __launch_bounds__(kBlock, LIST ? kListMinBlocks : kPersistMinBlocks) k_em_pass_persist(
    ImgGeom g, LorTable t, SubsetSel s, const CT* __restrict__ counts, int counts_packed,
    const float* __restrict__ add, PadBuffers pad, int back, double* __restrict__ partials, int64_t total,
    int skip_zero, unsigned long long* __restrict__ chunk_counter, const int* __restrict__ list,
    const int* __restrict__ n_list) {
  const int lane = threadIdx.x & 31;
  // LIST: the chunks are 32 consecutive entries of the subset's list of bins
  // with counts (k_nz_write), so every lane of a chunk walks.
  const int64_t n_items = LIST ? (int64_t)*n_list : total;
  const int64_t nchunks = (n_items + 31) >> 5;
  for (;;) {
    unsigned long long c = 0;
    if (lane == 0) c = atomicAdd(chunk_counter, 1ULL);
    c = __shfl_sync(0xffffffffu, c, 0);
    if ((int64_t)c >= nchunks) break;
    const int64_t item = (int64_t)c * 32 + lane;
    double term = 0.0;
    BinPos p{0, 0, 0, 0};
    float r = 0.f;
    if (item < n_items) {
      const int64_t b = LIST ? (int64_t)list[item] : item;
      p = decode(b, t, s);
      const int64_t row = counts_packed ? ((int64_t)(p.g - t.g0) * s.nk + p.k) : ((int64_t)p.g * t.n_proj + p.a);
      const int64_t ci = row * t.n_r + p.l;
      const float m = load_count<CT>(counts, ci);
      if (!(skip_zero && m == 0.f))
        term = em_bin_pad<UNROLL ? UNROLL : (LIST ? kListGatherUnroll : APIRL_GATHER_UNROLL), ACC>(
            g, t, p, m, ci, add, pad, back, skip_zero, &r);
    }
    if (ACC == 1) scatter_bin_warp(g, t, p, back && r != 0.f, r, pad);  // the whole warp
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) term += __shfl_down_sync(0xffffffffu, term, o);
    if (lane == 0) partials[c] = term;
  }
}

// Deterministic final sum of per-block partials (one block).
__global__ void k_sum_partials(const double* __restrict__ partials, int64_t n, double* __restrict__ out) {
  double v = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) v += partials[i];
  const double s = block_sum(v);
  if (threadIdx.x == 0) *out = s;
}

// out[b] = - (x . z over block b's contiguous chunk of voxels), FP64, fixed
// order; block 0 also subtracts *zero_add (when given).  The negated
// zero-count-bin estimates of the sparse pass.  Voxels with z == 0 are
// skipped: no walked bin reaches them, so an image value there (NaN where the
// update divided 0 by a zero sensitivity, as the reference's >= 0 test lets
// it) is in no estimate and stays out of the sum.
__global__ void __launch_bounds__(kBlock) k_neg_dot(const float* __restrict__ x, const float* __restrict__ z,
                                                    int64_t n, const double* __restrict__ zero_add,
                                                    double* __restrict__ out) {
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t lo = (int64_t)blockIdx.x * chunk;
  const int64_t hi = lo + chunk < n ? lo + chunk : n;
  double v = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const float zi = z[i];
    if (zi != 0.f) v += (double)x[i] * (double)zi;
  }
  const double s = block_sum(v);
  if (threadIdx.x == 0) out[blockIdx.x] = -s - ((blockIdx.x == 0 && zero_add) ? *zero_add : 0.0);
}

// Zero-count image of a subset for the sparse pass: img += A_s^T 1[m == 0]
// (the reference's 3D bounds test, one ray per bin), and per-warp partials of
// the zero-count bins' additive terms.
// With pad.bA set the scatter goes to the padded two-layout backprojection
// pair (as in the fused pass), to be folded into img by k_pad_reduce.
template <typename CT>
__global__ void __launch_bounds__(kBlock) k_zero_bins(ImgGeom g, LorTable t, SubsetSel s,
                                                      const CT* __restrict__ counts, int counts_packed,
                                                      const float* __restrict__ add, float* __restrict__ img,
                                                      PadBuffers pad, double* __restrict__ partials, int64_t total) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double term = 0.0;
  if (b < total) {
    const BinPos p = decode(b, t, s);
    const int64_t row = counts_packed ? ((int64_t)(p.g - t.g0) * s.nk + p.k) : ((int64_t)p.g * t.n_proj + p.a);
    const int64_t ci = row * t.n_r + p.l;
    if (load_count<CT>(counts, ci) == 0.f) {
      if (add) term = (double)__ldg(add + ci);
      const float4 L = t.lor[(int64_t)p.a * t.n_r + p.l];
      const float2 z = t.z[p.g];
      const float vx = A_SUB(L.z, L.x), vy = A_SUB(L.w, L.y);
      Walk3 w;
      siddon3_setup(L.x, L.y, z.x, vx, vy, A_SUB(z.y, z.x), g, w);
      if (pad.bA) {
        const bool tr = fabsf(vx) >= fabsf(vy);
        const int px = g.nx + 2 * kPad, py = g.ny + 2 * kPad;
        siddon3_scatter_pad(w, g, tr ? py : 1, tr ? 1 : px, px * py, pad.lim, 1.f, tr ? pad.bT : pad.bA);
      } else {
        siddon3_walk(w, g, [&](bool inb, int idx, float seg) {
          if (inb) red_add_global(img + idx, seg);
        });
      }
    }
  }
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) term += __shfl_down_sync(0xffffffffu, term, o);
  if ((threadIdx.x & 31) == 0) partials[((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5] = term;
}

// First level of the two-level sum of many partials: block b sums its
// contiguous chunk in a fixed order (deterministic), out2[b] = chunk sum.
__global__ void __launch_bounds__(kBlock) k_sum_chunks(const double* __restrict__ partials, int64_t n,
                                                       double* __restrict__ out2) {
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t lo = (int64_t)blockIdx.x * chunk;
  const int64_t hi = lo + chunk < n ? lo + chunk : n;
  double v = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) v += partials[i];
  const double s = block_sum(v);
  if (threadIdx.x == 0) out2[blockIdx.x] = s;
}

// ---------------------------------------------------------------------------
__global__ void k_inverse_divide(int64_t n, const float* __restrict__ meas, float* __restrict__ est) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float num = meas[i], den = est[i];
    est[i] = (num != 0.f && den != 0.f) ? A_DIV(num, den) : 0.f;
  }
}

__global__ void k_add_bins(int64_t n, const float* __restrict__ add, float* __restrict__ est) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    est[i] = A_ADD(est[i], add[i]);
}

__global__ void __launch_bounds__(kBlock) k_likelihood(int64_t n, const float* __restrict__ est,
                                                       const float* __restrict__ meas, int gt0,
                                                       double* __restrict__ partials) {
  double v = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float e = est[i];
    if (gt0 ? (e > 0.f) : (e != 0.f)) v += (double)meas[i] * log((double)e) - (double)e;
  }
  const double s = block_sum(v);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__device__ __forceinline__ unsigned fkey(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fkey_inv(unsigned k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__global__ void k_minmax_init(const float* __restrict__ sens, unsigned* mm) {
  mm[0] = fkey(FLT_MAX);
  mm[1] = fkey(sens[0]);
}

// Minimum over non-zero values and maximum over all values.
__global__ void __launch_bounds__(kBlock) k_minmax(int64_t n, const float* __restrict__ v, unsigned* mm) {
  float mn = FLT_MAX, mx = -FLT_MAX;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float f = v[i];
    if (f != 0.f && f < mn) mn = f;
    if (f > mx) mx = f;
  }
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = fminf(mn, __shfl_down_sync(0xffffffffu, mn, o));
    mx = fmaxf(mx, __shfl_down_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(mm, fkey(mn));
    atomicMax(mm + 1, fkey(mx));
  }
}

__global__ void k_threshold(const unsigned* mm, float* thr) {
  const float mn = fkey_inv(mm[0]), mx = fkey_inv(mm[1]);
  *thr = A_ADD(mn, A_MUL(A_SUB(mx, mn), 0.0001f));
}

__global__ void k_update(int64_t n, float* __restrict__ x, float* __restrict__ bp, const float* __restrict__ sens,
                         const float* __restrict__ thr_ptr, float thr_value, int ge, int zero_bp, int vec4) {
  const float thr = thr_ptr ? *thr_ptr : thr_value;
  const int64_t n4 = vec4 ? (n >> 2) : 0;
  float4* x4 = reinterpret_cast<float4*>(x);
  float4* b4 = reinterpret_cast<float4*>(bp);
  const float4* s4 = reinterpret_cast<const float4*>(sens);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
    float4 xv = x4[i], bv = b4[i], sv = __ldg(s4 + i);
    float* xs = &xv.x; const float* bs = &bv.x; const float* ss = &sv.x;
    #pragma unroll
    for (int c = 0; c < 4; c++) {
      const bool okv = ge ? (ss[c] >= thr) : (ss[c] > thr);
      xs[c] = okv ? A_DIV(A_MUL(xs[c], bs[c]), ss[c]) : 0.f;
    }
    x4[i] = xv;
    if (zero_bp) b4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  for (int64_t i = (n4 << 2) + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const bool okv = ge ? (sens[i] >= thr) : (sens[i] > thr);
    x[i] = okv ? A_DIV(A_MUL(x[i], bp[i]), sens[i]) : 0.f;
    if (zero_bp) bp[i] = 0.f;
  }
}

__global__ void k_force_positive(int64_t n, float* __restrict__ x) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (x[i] < 0.f) x[i] = 0.f;
}

// generateACFs (cmd/src/generateACFs.cpp:303-318): exp of every non-zero bin, 1 elsewhere.
__global__ void k_exp_nonzero(int64_t n, float* __restrict__ v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float a = v[i];
    v[i] = a != 0.f ? expf(a) : 1.f;
  }
}

__global__ void k_fill(int64_t n, float* __restrict__ x, float v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = v;
}


// ---------------------------------------------------------------------------
// Batched work over many independent jobs in one launch.
__device__ __forceinline__ float load_count_any(const void* p, int dtype, int64_t i) {
  if (dtype == APIRL_U32) return (float)__ldg((const uint32_t*)p + i);
  if (dtype == APIRL_U16) return (float)__ldg((const uint16_t*)p + i);
  return __ldg((const float*)p + i);
}

// The last of n entries whose first (block, tile or chunk) key(e) is <= k;
// entries are ordered by key.
template <typename J, class Key>
__device__ __forceinline__ int find_entry(const J* __restrict__ e, int n, int64_t k, Key key) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (key(e[mid]) <= k) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <typename J>
__device__ __forceinline__ int find_job(const J* __restrict__ jobs, int njobs, int64_t blk) {
  return find_entry(jobs, njobs, blk, [](const J& j) { return j.blk_begin; });
}

// Sensitivity of every subset of a job in one pass over its whole sinogram:
// bin (g, a, l) belongs to subset a % nsub.  forcePositive is a separate pass.
__global__ void __launch_bounds__(kBlock) k_sens_batch(const SensJob* __restrict__ jobs, int njobs) {
  __shared__ int sj;
  if (threadIdx.x == 0) sj = find_job(jobs, njobs, blockIdx.x);
  __syncthreads();
  const SensJob& J = jobs[sj];
  const int64_t b = ((int64_t)blockIdx.x - J.blk_begin) * kBlock + threadIdx.x;
  if (b >= J.nbins) return;
  SubsetSel all;
  all.subset = -1; all.nsub = 1; all.nk = J.t.n_proj;
  const BinPos p = decode(b, J.t, all);
  const float v = J.mult ? __ldg(J.mult + b) : 1.f;
  if (v == 0.f) return;
  float* sens = J.sens + (int64_t)(p.a % J.nsub) * J.nvox;
  const float4 L = J.t.lor[(int64_t)p.a * J.t.n_r + p.l];
  const float2 z = J.t.z[p.g];
  Walk3 w;
  siddon3_setup(L.x, L.y, z.x, A_SUB(L.z, L.x), A_SUB(L.w, L.y), A_SUB(z.y, z.x), J.g, w);
  siddon3_walk(w, J.g, [&](bool inb, int idx, float seg) {
    if (inb) red_add_global(sens + idx, A_MUL(seg, v));
  });
}

// ---- padded two-layout copies of the fused pass ------------------------------
// A: [z][y][x] and T: [z][x][y], both with a kPad-voxel border on every side.
struct PadDims {
  int nx, ny, nz;
  __device__ __forceinline__ int64_t a(int x, int y, int z) const {
    return ((int64_t)(z + kPad) * (ny + 2 * kPad) + (y + kPad)) * (nx + 2 * kPad) + (x + kPad);
  }
  __device__ __forceinline__ int64_t t(int x, int y, int z) const {
    return ((int64_t)(z + kPad) * (nx + 2 * kPad) + (x + kPad)) * (ny + 2 * kPad) + (y + kPad);
  }
};

// One 32 x 32 tile (x0, y0) of slice z, worked by 256 threads as 32 x 8
// (lx, ly): x ([z][y][x], unpadded) -> the interiors of pA ([z][y][x]) and pT
// ([z][x][y]).  With gimg: returns the thread's FP64 sum of x * gimg over its
// voxels where gimg != 0.
__device__ __forceinline__ double pad_copy_tile(const PadDims& d, const float* __restrict__ x, float* __restrict__ pA,
                                                float* __restrict__ pT, const float* __restrict__ gimg, int x0, int y0,
                                                int z, int lx, int ly, float (*tile)[33]) {
  const int64_t base = (int64_t)z * d.nx * d.ny;
  double dot = 0.0;
  // The tile's loads (x, and gimg for the dot) are all issued before its
  // first store.
  float xv[4], gv[4];
  #pragma unroll
  for (int q = 0; q < 4; q++) {
    const int yy = y0 + ly + 8 * q, xx = x0 + lx;
    xv[q] = gv[q] = 0.f;
    if (xx < d.nx && yy < d.ny) {
      const int64_t i = base + (int64_t)yy * d.nx + xx;
      xv[q] = x[i];
      if (gimg) gv[q] = gimg[i];
    }
  }
  #pragma unroll
  for (int q = 0; q < 4; q++) {
    const int r = ly + 8 * q;
    const int yy = y0 + r, xx = x0 + lx;
    if (xx < d.nx && yy < d.ny) {
      tile[r][lx] = xv[q];
      pA[d.a(xx, yy, z)] = xv[q];
      if (gv[q] != 0.f) dot += (double)xv[q] * (double)gv[q];
    }
  }
  __syncthreads();
  #pragma unroll
  for (int r = ly; r < 32; r += 8) {
    const int xx = x0 + r, yy = y0 + lx;
    if (xx < d.nx && yy < d.ny) pT[d.t(xx, yy, z)] = tile[lx][r];
  }
  return dot;
}

// x ([z][y][x], unpadded) -> interiors of pA and pT (32x32 tiles per slice).
__global__ void __launch_bounds__(256) k_pad_copy(PadDims d, const float* __restrict__ x, float* __restrict__ pA,
                                                  float* __restrict__ pT) {
  __shared__ float tile[32][33];
  pad_copy_tile(d, x, pA, pT, nullptr, blockIdx.x * 32, blockIdx.y * 32, blockIdx.z, threadIdx.x, threadIdx.y, tile);
}

// Sum of the two padded backprojections over one 32 x 32 tile (x0, y0) of
// slice z, [z][y][x] order, interiors cleared; threads as in pad_copy_tile.
// mode 0: EM update of x (threshold rule ge/gt); mode 1: bp += sum.  All
// loads come before the clearing stores (a store to an address whose load is
// still in flight stalls the thread's later memory operations: clearing in
// place made this kernel ~8x slower).
// eA / eT (may be null): the compensated form's rounding errors of bA / bT,
// folded in as (bA + eA) + (bT + eT) and cleared too.
__device__ __forceinline__ void pad_reduce_tile(const PadDims& d, float* __restrict__ bA, float* __restrict__ bT,
                                                int mode, float* __restrict__ x, float* __restrict__ bp,
                                                const float* __restrict__ sens, float thr, int ge, int x0, int y0,
                                                int z, int lx, int ly, float (*tile)[33],
                                                float* __restrict__ eA = nullptr, float* __restrict__ eT = nullptr) {
  const int64_t base = (int64_t)z * d.nx * d.ny;
  // Every load of the tile (both padded backprojections, and x and sens for
  // the update or bp for the sum) is issued before the first barrier, so
  // that all are in flight together.
  float av[4], xv[4], sv[4];
  #pragma unroll
  for (int q = 0; q < 4; q++) {
    const int r = ly + 8 * q;
    {
      const int xx = x0 + r, yy = y0 + lx;  // transposed buffer, read along y
      if (xx < d.nx && yy < d.ny) {
        const int64_t it = d.t(xx, yy, z);
        tile[lx][r] = eT ? A_ADD(bT[it], eT[it]) : bT[it];
      }
    }
    const int yy = y0 + r, xx = x0 + lx;
    av[q] = xv[q] = sv[q] = 0.f;
    if (xx < d.nx && yy < d.ny) {
      const int64_t ia = d.a(xx, yy, z);
      av[q] = eA ? A_ADD(bA[ia], eA[ia]) : bA[ia];
      const int64_t i = base + (int64_t)yy * d.nx + xx;
      if (mode == 0) {
        xv[q] = x[i];
        sv[q] = sens[i];
      } else {
        xv[q] = bp[i];
      }
    }
  }
  __syncthreads();
  float bv[4];
  #pragma unroll
  for (int q = 0; q < 4; q++) bv[q] = A_ADD(av[q], tile[ly + 8 * q][lx]);
  __syncthreads();
  #pragma unroll
  for (int q = 0; q < 4; q++) {
    const int r = ly + 8 * q;
    {
      const int xx = x0 + r, yy = y0 + lx;
      if (xx < d.nx && yy < d.ny) {
        bT[d.t(xx, yy, z)] = 0.f;
        if (eT) eT[d.t(xx, yy, z)] = 0.f;
      }
    }
    const int yy = y0 + r, xx = x0 + lx;
    if (xx < d.nx && yy < d.ny) {
      bA[d.a(xx, yy, z)] = 0.f;
      if (eA) eA[d.a(xx, yy, z)] = 0.f;
      const int64_t i = base + (int64_t)yy * d.nx + xx;
      if (mode == 0) {
        const bool okv = ge ? (sv[q] >= thr) : (sv[q] > thr);
        x[i] = okv ? A_DIV(A_MUL(xv[q], bv[q]), sv[q]) : 0.f;
      } else {
        bp[i] = A_ADD(xv[q], bv[q]);
      }
    }
  }
}

__global__ void __launch_bounds__(256) k_pad_reduce(PadDims d, float* __restrict__ bA, float* __restrict__ bT,
                                                    int mode, float* __restrict__ x, float* __restrict__ bp,
                                                    const float* __restrict__ sens, const float* __restrict__ thr_ptr,
                                                    float thr_value, int ge, float* __restrict__ eA,
                                                    float* __restrict__ eT) {
  __shared__ float tile[32][33];
  const float thr = (mode == 0 && thr_ptr) ? *thr_ptr : thr_value;
  pad_reduce_tile(d, bA, bT, mode, x, bp, sens, thr, ge, blockIdx.x * 32, blockIdx.y * 32, blockIdx.z, threadIdx.x,
                  threadIdx.y, tile, eA, eT);
}

// ---- batched reconstructions: one step for many jobs ----------------------------
// Before the walk: every job's image into its padded copies, and the FP64
// partial -x . gimg of every tile (the likelihood's sum over the bins the
// walk leaves out).  One block per tile; tiles of a job are consecutive.
__global__ void __launch_bounds__(256) k_multi_copy(const MultiVox* __restrict__ jobs, int njobs,
                                                    double* __restrict__ tile_partials) {
  __shared__ float tile[32][33];
  __shared__ int sj;
  if (threadIdx.x == 0) sj = find_entry(jobs, njobs, blockIdx.x, [](const MultiVox& j) { return j.tile_begin; });
  __syncthreads();
  const MultiVox& J = jobs[sj];
  const int64_t tl = (int64_t)blockIdx.x - J.tile_begin;
  const int tx = (int)(tl % J.tiles_x);
  const int64_t q = tl / J.tiles_x;
  const int ty = (int)(q % J.tiles_y), z = (int)(q / J.tiles_y);
  const PadDims d{J.g.nx, J.g.ny, J.g.nz};
  const double dot = pad_copy_tile(d, J.x, J.pad.pA, J.pad.pT, J.gimg, tx * 32, ty * 32, z, threadIdx.x & 31,
                                   threadIdx.x >> 5, tile);
  const double sum = block_sum(dot);
  if (threadIdx.x == 0) tile_partials[blockIdx.x] = -sum;
}

// The walk of a batched step: persistent warps take the next chunk of 32
// entries of the concatenated lists of all segments, find its segment, and
// run the fused pass on each listed bin (geometry form of the likelihood: a
// walked bin adds m log e).  One FP64 partial per chunk, as in
// k_em_pass_persist.
__global__ void __launch_bounds__(kBlock, kMultiMinBlocks) k_em_multi(const MultiSeg* __restrict__ segs, int nseg,
                                                                     int64_t nchunks,
                                                                     unsigned long long* __restrict__ counter,
                                                                     double* __restrict__ partials) {
  // Each warp keeps its chunk's segment in shared memory (the walk reads the
  // geometry from there instead of holding it in registers).
  static_assert(sizeof(MultiSeg) % 8 == 0 && sizeof(MultiSeg) <= 64 * 4, "segment copy");
  __shared__ __align__(16) int seg_raw[kBlock / 32][sizeof(MultiSeg) / 4];
  const int lane = threadIdx.x & 31;
  MultiSeg* S = reinterpret_cast<MultiSeg*>(seg_raw[threadIdx.x >> 5]);
  int cur = -1;
  for (;;) {
    unsigned long long c = 0;
    if (lane == 0) c = atomicAdd(counter, 1ULL);
    c = __shfl_sync(0xffffffffu, c, 0);
    if ((int64_t)c >= nchunks) break;
    const int k = find_entry(segs, nseg, (int64_t)c, [](const MultiSeg& e) { return e.chunk_begin; });
    if (k != cur) {
      __syncwarp();
      const int* src = reinterpret_cast<const int*>(segs + k);
      int* dst = reinterpret_cast<int*>(S);
      for (int i = lane; i < (int)(sizeof(MultiSeg) / 4); i += 32) dst[i] = __ldg(src + i);
      __syncwarp();
      cur = k;
    }
    const int64_t item = ((int64_t)c - S->chunk_begin) * 32 + lane;
    double term = 0.0;
    if (item < S->n_list) {
      const BinPos p = decode((int64_t)__ldg(S->list + item), S->t, S->s);
      const int64_t ci = ((int64_t)p.g * S->t.n_proj + p.a) * S->t.n_r + p.l;
      const float m = load_count_any(S->counts, S->counts_dtype, ci);
      if (m != 0.f) term = em_bin_pad<kMultiGatherUnroll, 0>(S->g, S->t, p, m, ci, S->add, S->pad, S->back, 2);
    }
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) term += __shfl_down_sync(0xffffffffu, term, o);
    if (lane == 0) partials[c] = term;
  }
}

// One block per job: its likelihood, the fixed-order sum of its chunk
// partials and its tile partials, minus its additive sum.
__global__ void __launch_bounds__(256) k_multi_sum(const MultiVox* __restrict__ jobs,
                                                   const double* __restrict__ chunk_partials,
                                                   const double* __restrict__ tile_partials) {
  const MultiVox& J = jobs[blockIdx.x];
  const int64_t ntiles = (int64_t)J.tiles_x * J.tiles_y * J.g.nz;
  double v = 0.0;
  for (int64_t i = threadIdx.x; i < J.n_chunks; i += blockDim.x) v += chunk_partials[J.chunk_begin + i];
  for (int64_t i = threadIdx.x; i < ntiles; i += blockDim.x) v += tile_partials[J.tile_begin + i];
  const double s = block_sum(v);
  if (threadIdx.x == 0 && J.lik) *J.lik = s - J.zero_add;
}

// After the walk: the EM update of every job with `update` from its padded
// backprojection pair (threshold 0, rule ge), the pair cleared.
__global__ void __launch_bounds__(256) k_multi_update(const MultiVox* __restrict__ jobs, int njobs) {
  __shared__ float tile[32][33];
  __shared__ int sj;
  if (threadIdx.x == 0) sj = find_entry(jobs, njobs, blockIdx.x, [](const MultiVox& j) { return j.tile_begin; });
  __syncthreads();
  const MultiVox& J = jobs[sj];
  if (!J.update) return;
  const int64_t tl = (int64_t)blockIdx.x - J.tile_begin;
  const int tx = (int)(tl % J.tiles_x);
  const int64_t q = tl / J.tiles_x;
  const int ty = (int)(q % J.tiles_y), z = (int)(q / J.tiles_y);
  const PadDims d{J.g.nx, J.g.ny, J.g.nz};
  pad_reduce_tile(d, J.pad.bA, J.pad.bT, 0, J.x, nullptr, J.sens, 0.f, J.ge, tx * 32, ty * 32, z, threadIdx.x & 31,
                  threadIdx.x >> 5, tile);
}

// per_angle[a] += A_a^T 1 (Backproject of ones, SiddonProjector.cpp:444-568)
// for every angle a, into padded images (PadBuffers' border and layouts):
// angle a's image is [z][x][y] when tr[a] (its rays run mostly along x), else
// [z][y][x], so that the 32 parallel rays of a warp scatter into neighbouring
// addresses.  Persistent warps take 32-bin chunks in angle order (angle,
// sinogram, r): the warps write one angle's image at a time and it stays in
// L2.  Border voxels receive the scatter of guarded walks (see
// siddon3_gather_pad); nothing reads them.
__global__ void __launch_bounds__(kBlock) k_scatter_angles(ImgGeom g, LorTable t, const uint8_t* __restrict__ tr_of,
                                                           float* __restrict__ per_angle, unsigned lim,
                                                           unsigned long long* __restrict__ counter) {
  const int lane = threadIdx.x & 31;
  const int64_t per_a = (int64_t)t.n_sinos * t.n_r;
  const int64_t total = per_a * t.n_proj;
  const int64_t nchunks = (total + 31) >> 5;
  const int px = g.nx + 2 * kPad, py = g.ny + 2 * kPad;
  for (;;) {
    unsigned long long c = 0;
    if (lane == 0) c = atomicAdd(counter, 1ULL);
    c = __shfl_sync(0xffffffffu, c, 0);
    if ((int64_t)c >= nchunks) break;
    const int64_t b = (int64_t)c * 32 + lane;
    if (b >= total) continue;
    const int a = (int)(b / per_a);
    const int64_t rem = b - (int64_t)a * per_a;
    const int gs = (int)(rem / t.n_r);
    const int l = (int)(rem - (int64_t)gs * t.n_r);
    const float4 L = t.lor[(int64_t)a * t.n_r + l];
    const float2 z = t.z[t.g0 + gs];
    const bool tr = __ldg(tr_of + a) != 0;
    Walk3 w;
    siddon3_setup(L.x, L.y, z.x, A_SUB(L.z, L.x), A_SUB(L.w, L.y), A_SUB(z.y, z.x), g, w);
    siddon3_scatter_pad(w, g, tr ? py : 1, tr ? 1 : px, px * py, lim, 1.f, per_angle + (int64_t)a * lim);
  }
}

// out[s] ([z][y][x], unpadded) = the sum over a = s, s + nsub, ... < n_proj of
// the interiors of the padded per-angle images (layouts as k_scatter_angles),
// added in increasing a.  One block per 32 x 32 tile of a slice and subset.
__global__ void __launch_bounds__(256) k_sum_angles(const float* __restrict__ per_angle, const uint8_t* __restrict__ tr_of,
                                                    unsigned lim, int n_proj, ImgGeom g, int nsub,
                                                    float* __restrict__ out) {
  __shared__ float tile[32][33];
  const int s = blockIdx.y;
  const int tiles_x = (g.nx + 31) / 32, tiles_y = (g.ny + 31) / 32;
  const int tx = blockIdx.x % tiles_x, ty = (blockIdx.x / tiles_x) % tiles_y, z = blockIdx.x / (tiles_x * tiles_y);
  const int x0 = tx * 32, y0 = ty * 32, lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
  const PadDims d{g.nx, g.ny, g.nz};
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  for (int a = s; a < n_proj; a += nsub) {
    const float* P = per_angle + (int64_t)a * lim;
    if (__ldg(tr_of + a)) {
      __syncthreads();
      for (int r = ly; r < 32; r += 8) {  // transposed image, read along y
        const int xx = x0 + r, yy = y0 + lx;
        tile[lx][r] = (xx < d.nx && yy < d.ny) ? __ldg(P + d.t(xx, yy, z)) : 0.f;
      }
      __syncthreads();
      #pragma unroll
      for (int q = 0; q < 4; q++) acc[q] = A_ADD(acc[q], tile[ly + 8 * q][lx]);
    } else {
      #pragma unroll
      for (int q = 0; q < 4; q++) {
        const int xx = x0 + lx, yy = y0 + ly + 8 * q;
        acc[q] = A_ADD(acc[q], (xx < d.nx && yy < d.ny) ? __ldg(P + d.a(xx, yy, z)) : 0.f);
      }
    }
  }
  const int64_t nvox = (int64_t)g.nx * g.ny * g.nz;
  #pragma unroll
  for (int q = 0; q < 4; q++) {
    const int xx = x0 + lx, yy = y0 + ly + 8 * q;
    if (xx < d.nx && yy < d.ny) out[(int64_t)s * nvox + ((int64_t)z * d.ny + yy) * d.nx + xx] = acc[q];
  }
}

// out[s] = sum over images a = s, s + nsub, ... < n_img of img[a] (unpadded
// images of nvox), added in increasing a.
__global__ void __launch_bounds__(kBlock) k_sum_images(const float* __restrict__ img, int n_img, int64_t nvox,
                                                       int nsub, float* __restrict__ out) {
  const int s = blockIdx.y;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += (int64_t)gridDim.x * blockDim.x) {
    float acc = 0.f;
    for (int a = s; a < n_img; a += nsub) acc = A_ADD(acc, __ldg(img + (int64_t)a * nvox + v));
    out[(int64_t)s * nvox + v] = acc;
  }
}

// out[s] = sum of the additive term over subset s's bins (whole-sinogram
// layout), one block per subset, FP64, fixed order.
__global__ void __launch_bounds__(kBlock) k_subset_sums(LorTable t, int nsub, const float* __restrict__ add,
                                                        double* __restrict__ out) {
  SubsetSel s;
  s.subset = blockIdx.x; s.nsub = nsub; s.nk = 0;
  for (int a = s.subset; a < t.n_proj; a += nsub) s.nk++;
  const int64_t total = (int64_t)t.n_sinos * s.nk * t.n_r;
  double v = 0.0;
  for (int64_t b = threadIdx.x; b < total; b += blockDim.x) {
    const BinPos p = decode(b, t, s);
    v += (double)__ldg(add + ((int64_t)p.g * t.n_proj + p.a) * t.n_r + p.l);
  }
  const double r = block_sum(v);
  if (threadIdx.x == 0) out[blockIdx.x] = r;
}

inline unsigned grid_for(int64_t total) { return (unsigned)((total + kBlock - 1) / kBlock); }

// Launch of a kernel over the padded layouts: with pad.window
// (APIRL_OPT_L2_PERSIST), an L2 access policy window over the block of the
// four padded images, hits persisting, misses streaming.
template <typename... KArgs, typename... Args>
cudaError_t pad_launch(const PadBuffers& pad, dim3 grid, dim3 block, cudaStream_t st, void (*kernel)(KArgs...),
                       Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  if (pad.window) {
    at[0].id = cudaLaunchAttributeAccessPolicyWindow;
    at[0].val.accessPolicyWindow.base_ptr = pad.pA;
    at[0].val.accessPolicyWindow.num_bytes = pad.window;
    at[0].val.accessPolicyWindow.hitRatio = pad.hit_ratio;
    at[0].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    at[0].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    cfg.attrs = at;
    cfg.numAttrs = 1;
  }
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// The fused 3D kernels use no shared memory: give the SM's unified L1 /
// shared storage to L1.  Set once per device (function attributes belong to
// the device's context).
cudaError_t prefer_l1() {
  static std::atomic<int> done[64];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64 || done[dev].load()) return cudaSuccess;
  if ((e = cudaFuncSetAttribute(k_em_pass<float, true, false>, cudaFuncAttributePreferredSharedMemoryCarveout, 0)) !=
          cudaSuccess ||
      (e = cudaFuncSetAttribute(k_em_pass<uint32_t, true, false>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                0)) != cudaSuccess ||
      (e = cudaFuncSetAttribute(k_em_pass<uint16_t, true, false>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                0)) != cudaSuccess)
    return e;
  done[dev].store(1);
  return cudaSuccess;
}

// The persistent kernel's carveout: the shared memory that its resident
// blocks need (static, dynamic and the per-block reserve,
// cudaDevAttrReservedSharedMemoryPerBlock), at as many blocks per SM as its
// registers and threads allow, and all the rest for L1.  A preferred carveout
// of 0 can leave room for fewer blocks' reserves than the registers allow
// (with 128 threads per block, 10 blocks fit in the registers at 48 per
// thread, 8 blocks' reserves in the smallest carveout), which costs warps.
// Fitted again when the block size changes (the attribute is per function).
std::mutex g_carve_mu;
struct CarveFit {
  const void* f;
  int dev, block;
};
std::vector<CarveFit> g_carve;

cudaError_t fit_carveout(const void* f, int block, size_t dyn_smem) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_carve_mu);
  CarveFit* slot = nullptr;
  for (CarveFit& c : g_carve)
    if (c.f == f && c.dev == dev) slot = &c;
  if (slot && slot->block == block) return cudaSuccess;
  cudaFuncAttributes fa;
  int per_sm = 0, reserved = 0, max_sm = 0;
  if ((e = cudaFuncGetAttributes(&fa, f)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&max_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess) return e;
  // With every byte offered to shared memory, residency is set by the
  // registers and threads alone.
  if ((e = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, block, dyn_smem)) != cudaSuccess) return e;
  if (max_sm <= 0) return cudaErrorInvalidValue;
  const int64_t need = (int64_t)(per_sm < 1 ? 1 : per_sm) * ((int64_t)fa.sharedSizeBytes + (int64_t)dyn_smem + reserved);
  int pct = (int)((need * 100 + max_sm - 1) / max_sm);
  pct = pct < 1 ? 1 : (pct > 100 ? 100 : pct);
  if ((e = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, pct)) != cudaSuccess) return e;
  if (slot) slot->block = block;
  else g_carve.push_back(CarveFit{f, dev, block});
  return cudaSuccess;
}

// Deterministic sum of n partials into *out.  Above kSumLevel2 * 64 partials
// the sum runs in two levels (kSumLevel2 blocks, then one), the second level's
// kSumLevel2 values stored right after partials[n - 1].
cudaError_t launch_sum(double* partials, int64_t n, double* out, cudaStream_t st) {
  if (n > (int64_t)kSumLevel2 * 64) {
    k_sum_chunks<<<kSumLevel2, kBlock, 0, st>>>(partials, n, partials + n);
    k_sum_partials<<<1, kBlock, 0, st>>>(partials + n, kSumLevel2, out);
  } else {
    k_sum_partials<<<1, kBlock, 0, st>>>(partials, n, out);
  }
  return cudaGetLastError();
}
inline unsigned stream_grid(int64_t n) {
  int64_t g = (n + kBlock - 1) / kBlock;
  const int64_t cap = 148 * 16;  // a few waves over the 148 SMs; the loops stride
  return (unsigned)(g < 1 ? 1 : (g > cap ? cap : g));
}

}  // namespace

// The persistent fused kernel for a counts type, list form, accumulation form
// and gather segments in flight (4, 6 or 8 with plain atomics; 0: default).
template <typename CT, bool LIST>
const void* persist_kernel_l(int acc, int unroll) {
  if (acc == 1) return (const void*)k_em_pass_persist<CT, LIST, 1, 0>;
  if (acc == 2) return (const void*)k_em_pass_persist<CT, LIST, 2, 0>;
  switch (unroll) {
    case 4: return (const void*)k_em_pass_persist<CT, LIST, 0, 4>;
    case 6: return (const void*)k_em_pass_persist<CT, LIST, 0, 6>;
    case 8: return (const void*)k_em_pass_persist<CT, LIST, 0, 8>;
    default: return (const void*)k_em_pass_persist<CT, LIST, 0, 0>;
  }
}
template <typename CT>
const void* persist_kernel(bool list, int acc, int unroll) {
  return list ? persist_kernel_l<CT, true>(acc, unroll) : persist_kernel_l<CT, false>(acc, unroll);
}

cudaError_t prepare_em_kernels(int block) {
  for (int acc = 0; acc < 3; acc++)
    for (int unroll : {0, 4, 6, 8})
      for (bool list : {false, true}) {
        if (acc && unroll) continue;
        for (const void* f : {persist_kernel<float>(list, acc, unroll), persist_kernel<uint32_t>(list, acc, unroll),
                              persist_kernel<uint16_t>(list, acc, unroll)}) {
          cudaError_t e = fit_carveout(f, block, 0);
          if (e != cudaSuccess) return e;
        }
      }
  return cudaSuccess;
}


int64_t em_pass_blocks(const LorTable& t, SubsetSel s) {
  // One likelihood partial per warp for any block size of 32..256 threads
  // (ceil(total / b) * b / 32 <= total / 32 + 8), the zero-count image's
  // partials of the sparse pass, then the second level of the sum.
  return ((int64_t)t.n_sinos * s.nk * t.n_r + 31) / 32 + 8 + 2 * kSumLevel2;
}
int64_t likelihood_blocks(int64_t n) { return stream_grid(n); }

cudaError_t launch_project(const ImgGeom& g, const LorTable& t, SubsetSel s, const float* img, float* out,
                           cudaStream_t st, const PreciseGeom& pg) {
  const int64_t total = (int64_t)t.n_sinos * s.nk * t.n_r;
  if (total == 0) return cudaSuccess;
  if (t.is3d && pg.enabled) k_project3<true><<<grid_for(total), kBlock, 0, st>>>(g, t, s, pg, img, out, total);
  else if (t.is3d) k_project3<false><<<grid_for(total), kBlock, 0, st>>>(g, t, s, pg, img, out, total);
  else k_project2<<<grid_for(total), kBlock, 0, st>>>(g, t, s, img, out, total);
  return cudaGetLastError();
}

cudaError_t launch_backproject(const ImgGeom& g, const LorTable& t, SubsetSel s, const float* vin, int vin_mode,
                               const float* vest, int divide, float* img, cudaStream_t st, const PreciseGeom& pg) {
  const int64_t total = (int64_t)t.n_sinos * s.nk * t.n_r;
  if (total == 0) return cudaSuccess;
  if (t.is3d && pg.enabled)
    k_backproject3<true><<<grid_for(total), kBlock, 0, st>>>(g, t, s, pg, vin, vin_mode, vest, divide, img, total);
  else if (t.is3d)
    k_backproject3<false><<<grid_for(total), kBlock, 0, st>>>(g, t, s, pg, vin, vin_mode, vest, divide, img, total);
  else k_backproject2<<<grid_for(total), kBlock, 0, st>>>(g, t, s, vin, vin_mode, vest, divide, img, total);
  return cudaGetLastError();
}

cudaError_t launch_backproject_pad(const ImgGeom& g, const LorTable& t, SubsetSel s, const float* vin, int vin_mode,
                                   float* img, const PadBuffers& pad, unsigned long long* counter, cudaStream_t st,
                                   float* img2, const PadBuffers& pad2) {
  const int64_t total = (int64_t)t.n_sinos * s.nk * t.n_r;
  if (total == 0) return cudaSuccess;
  int per_sm = 0, dev = 0, sms = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_scatter_persist<0>, 128, 0);
  if (e != cudaSuccess) return e;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  const int64_t resident = (int64_t)(per_sm < 1 ? 1 : per_sm) * sms;
  const int64_t need = ((total + 31) / 32 * 32 + 127) / 128;
  if ((e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st)) != cudaSuccess) return e;
  const bool two = img2 && pad2.bA && pad2.bT;
  const unsigned grid = (unsigned)(need < resident ? need : resident);
  // The second pair (img2) takes plain atomics; so does the first beside it.
  const int acc = two ? 0 : pad.acc;
  float* none = nullptr;
  if (acc == 1)
    e = pad_launch(pad, dim3(grid), dim3(128), st, k_scatter_persist<1>, g, t, s, vin, vin_mode, pad, total, counter,
                   none, none);
  else if (acc == 2)
    e = pad_launch(pad, dim3(grid), dim3(128), st, k_scatter_persist<2>, g, t, s, vin, vin_mode, pad, total, counter,
                   none, none);
  else
    e = pad_launch(pad, dim3(grid), dim3(128), st, k_scatter_persist<0>, g, t, s, vin, vin_mode, pad, total, counter,
                   two ? pad2.bA : none, two ? pad2.bT : none);
  if (e != cudaSuccess) return e;
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (two && (e = launch_pad_reduce(g, pad2, 1, nullptr, img2, nullptr, nullptr, 0.f, 0, st)) != cudaSuccess) return e;
  return launch_pad_reduce(g, pad, 1, nullptr, img, nullptr, nullptr, 0.f, 0, st);
}

cudaError_t launch_count_steps(const ImgGeom& g, const LorTable& t, SubsetSel s, int32_t* steps, cudaStream_t st) {
  const int64_t total = (int64_t)t.n_sinos * s.nk * t.n_r;
  if (total == 0) return cudaSuccess;
  k_count_steps<<<grid_for(total), kBlock, 0, st>>>(g, t, s, steps, total);
  return cudaGetLastError();
}

cudaError_t launch_em_pass(const ImgGeom& g, const LorTable& t, SubsetSel s, const void* counts, int counts_dtype,
                           int counts_packed, const float* add, const float* x, float* bp, int back, int lik_mode,
                           double* partials, double* lik, cudaStream_t st, const PreciseGeom& pg,
                           const PadBuffers& pad, int block, const float* zimg, const double* zero_add,
                           unsigned long long* persist_counter, int zimg_all_bins, const NzList& nz) {
  const int skip = zimg ? (zimg_all_bins ? 2 : 1) : 0;
  const int64_t total = (int64_t)t.n_sinos * s.nk * t.n_r;
  if (block < 32 || block > kBlock || block % 32) block = kBlock;
  const unsigned grid = (unsigned)((total + block - 1) / block);
  if (total == 0) return cudaSuccess;
  // The sparse form walks only bins with counts; it runs on the 3D float
  // walk with one ray per bin.
  if (zimg && (!t.is3d || t.lor_s || pg.enabled || lik_mode != 0)) return cudaErrorInvalidValue;
#define APIRL_EM(CT)                                                                                          \
  do {                                                                                                        \
    if (t.is3d && t.lor_s)                                                                                    \
      k_em_pass_rays<CT><<<grid, block, 0, st>>>(g, t, s, (const CT*)counts, counts_packed, add, x, bp, back,  \
                                                 lik_mode, partials, total);                                  \
    else if (t.is3d && pg.enabled)                                                                            \
      k_em_pass<CT, true, true><<<grid, block, 0, st>>>(g, t, s, pg, (const CT*)counts, counts_packed, add, x, \
                                                         bp, PadBuffers(), back, lik_mode, partials, total, 0); \
    else if (t.is3d)                                                                                          \
      k_em_pass<CT, true, false><<<grid, block, 0, st>>>(g, t, s, pg, (const CT*)counts, counts_packed, add,   \
                                                          x, bp, pad, back, lik_mode, partials, total,        \
                                                          skip);                                   \
    else                                                                                                      \
      k_em_pass<CT, false, false><<<grid, block, 0, st>>>(g, t, s, pg, (const CT*)counts, counts_packed, add,  \
                                                           x, bp, PadBuffers(), back, lik_mode, partials,     \
                                                           total, 0);                                         \
  } while (0)
  if (persist_counter && t.is3d && !t.lor_s && !pg.enabled && pad.pA && lik_mode == 0) {
    if (cudaError_t le = prefer_l1()) return le;
    // Persistent form: as many blocks of this size as fit on the current
    // device's SMs at once (a host-side query of a few microseconds).
    // Sparse passes walk a list of the subset's bins with counts when the
    // projector gives room for one (bin numbers are int32).
    const bool use_list = skip && nz.list && nz.tiles && nz.n_list && total <= nz.cap && total < ((int64_t)1 << 31);
    const void* pf;
    switch (counts_dtype) {
      case APIRL_F32: pf = persist_kernel<float>(use_list, pad.acc, pad.unroll); break;
      case APIRL_U32: pf = persist_kernel<uint32_t>(use_list, pad.acc, pad.unroll); break;
      case APIRL_U16: pf = persist_kernel<uint16_t>(use_list, pad.acc, pad.unroll); break;
      default: return cudaErrorInvalidValue;
    }
    // Fitted here unless the launch is being captured into a graph (the
    // projector fits it ahead for its block size: prepare_em_kernels).
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t fe = cudaStreamIsCapturing(st, &cs);
    if (fe != cudaSuccess) return fe;
    if (cs == cudaStreamCaptureStatusNone && (fe = fit_carveout(pf, block, 0)) != cudaSuccess) return fe;
    int per_sm = 0, dev = 0, sms = 0;
    cudaError_t oe = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pf, block, 0);
    if (oe != cudaSuccess) return oe;
    if ((oe = cudaGetDevice(&dev)) != cudaSuccess) return oe;
    if ((oe = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return oe;
    const int64_t resident = (int64_t)(per_sm < 1 ? 1 : per_sm) * sms;
    const int64_t chunks = (total + 31) / 32;
    const int64_t need = (chunks * 32 + block - 1) / block;
    const unsigned pgrid = (unsigned)(need < resident ? need : resident);
    cudaError_t me = cudaMemsetAsync(persist_counter, 0, sizeof(unsigned long long), st);
    if (me != cudaSuccess) return me;
    if (use_list) {
      // The list, and zeros in the partials of the chunks the list leaves
      // out (the sum below runs over as many partials as the full pass has).
      const unsigned n_tiles = (unsigned)((total + kNzTile - 1) / kNzTile);
      switch (counts_dtype) {
        case APIRL_F32:
          k_nz_tiles<float><<<n_tiles, kNzBlock, 0, st>>>(t, s, (const float*)counts, counts_packed, total, nz.tiles);
          break;
        case APIRL_U32:
          k_nz_tiles<uint32_t><<<n_tiles, kNzBlock, 0, st>>>(t, s, (const uint32_t*)counts, counts_packed, total,
                                                             nz.tiles);
          break;
        default:
          k_nz_tiles<uint16_t><<<n_tiles, kNzBlock, 0, st>>>(t, s, (const uint16_t*)counts, counts_packed, total,
                                                             nz.tiles);
          break;
      }
      k_nz_scan<<<1, 1024, 0, st>>>(nz.tiles, (int)n_tiles, nz.n_list);
      if (nz.order > 0) {
        switch (counts_dtype) {
          case APIRL_F32:
            k_nz_write_sorted<float><<<n_tiles, kNzBlock, 0, st>>>(g, t, s, (const float*)counts, counts_packed, total,
                                                                   nz.tiles, nz.list, nz.order);
            break;
          case APIRL_U32:
            k_nz_write_sorted<uint32_t><<<n_tiles, kNzBlock, 0, st>>>(g, t, s, (const uint32_t*)counts, counts_packed,
                                                                      total, nz.tiles, nz.list, nz.order);
            break;
          default:
            k_nz_write_sorted<uint16_t><<<n_tiles, kNzBlock, 0, st>>>(g, t, s, (const uint16_t*)counts, counts_packed,
                                                                      total, nz.tiles, nz.list, nz.order);
            break;
        }
      } else switch (counts_dtype) {
        case APIRL_F32:
          k_nz_write<float><<<n_tiles, kNzBlock, 0, st>>>(t, s, (const float*)counts, counts_packed, total, nz.tiles,
                                                          nz.list);
          break;
        case APIRL_U32:
          k_nz_write<uint32_t><<<n_tiles, kNzBlock, 0, st>>>(t, s, (const uint32_t*)counts, counts_packed, total,
                                                             nz.tiles, nz.list);
          break;
        default:
          k_nz_write<uint16_t><<<n_tiles, kNzBlock, 0, st>>>(t, s, (const uint16_t*)counts, counts_packed, total,
                                                             nz.tiles, nz.list);
          break;
      }
      if ((me = cudaMemsetAsync(partials, 0, (size_t)chunks * sizeof(double), st)) != cudaSuccess) return me;
    }
#define APIRL_PERSIST_ACC(CT, ACC, U)                                                                           \
  do {                                                                                                          \
    const int* no_list = nullptr;                                                                               \
    if (use_list)                                                                                               \
      le = pad_launch(pad, dim3(pgrid), dim3(block), st, k_em_pass_persist<CT, true, ACC, U>, g, t, s,          \
                      (const CT*)counts, counts_packed, add, pad, back, partials, total, skip, persist_counter,   \
                      (const int*)nz.list, (const int*)nz.n_list);                                              \
    else                                                                                                        \
      le = pad_launch(pad, dim3(pgrid), dim3(block), st, k_em_pass_persist<CT, false, ACC, U>, g, t, s,         \
                      (const CT*)counts, counts_packed, add, pad, back, partials, total, skip, persist_counter,   \
                      no_list, no_list);                                                                        \
  } while (0)
#define APIRL_PERSIST(CT)                                  \
  do {                                                     \
    if (pad.acc == 1) APIRL_PERSIST_ACC(CT, 1, 0);         \
    else if (pad.acc == 2) APIRL_PERSIST_ACC(CT, 2, 0);    \
    else if (pad.unroll == 4) APIRL_PERSIST_ACC(CT, 0, 4); \
    else if (pad.unroll == 6) APIRL_PERSIST_ACC(CT, 0, 6); \
    else if (pad.unroll == 8) APIRL_PERSIST_ACC(CT, 0, 8); \
    else APIRL_PERSIST_ACC(CT, 0, 0);                      \
  } while (0)
    cudaError_t le = cudaSuccess;
    switch (counts_dtype) {
      case APIRL_F32: APIRL_PERSIST(float); break;
      case APIRL_U32: APIRL_PERSIST(uint32_t); break;
      case APIRL_U16: APIRL_PERSIST(uint16_t); break;
      default: return cudaErrorInvalidValue;
    }
#undef APIRL_PERSIST
#undef APIRL_PERSIST_ACC
    if (le != cudaSuccess) return le;
    cudaError_t pe = cudaGetLastError();
    if (pe != cudaSuccess || !lik) return pe;
    int64_t np = chunks;
    if (zimg) {
      const int64_t nv = (int64_t)g.nx * g.ny * g.nz;
      k_neg_dot<<<kSumLevel2, kBlock, 0, st>>>(x, zimg, nv, zero_add, partials + np);
      np += kSumLevel2;
    }
    return launch_sum(partials, np, lik, st);
  }
  if (cudaError_t le = prefer_l1()) return le;
  switch (counts_dtype) {
    case APIRL_F32: APIRL_EM(float); break;
    case APIRL_U32: APIRL_EM(uint32_t); break;
    case APIRL_U16: APIRL_EM(uint16_t); break;
    default: return cudaErrorInvalidValue;
  }
#undef APIRL_EM
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !lik) return e;
  // One partial per 32 bins, whatever the block size (warps past the last
  // bin wrote zeros behind them): the same sum for every block size.
  int64_t np = (total + 31) / 32;
  if (zimg) {
    // - sum of the zero-count bins' estimates: - x . zimg - sum of their additive terms.
    const int64_t nv = (int64_t)g.nx * g.ny * g.nz;
    k_neg_dot<<<kSumLevel2, kBlock, 0, st>>>(x, zimg, nv, zero_add, partials + np);
    np += kSumLevel2;
  }
  return launch_sum(partials, np, lik, st);
}

cudaError_t launch_zero_bins(const ImgGeom& g, const LorTable& t, SubsetSel s, const void* counts, int counts_dtype,
                             int counts_packed, const float* add, float* img, double* partials, double* zero_add,
                             cudaStream_t st, const PadBuffers& pad) {
  const int64_t total = (int64_t)t.n_sinos * s.nk * t.n_r;
  if (!t.is3d || t.lor_s) return cudaErrorInvalidValue;
  if (total == 0) return cudaSuccess;
  const unsigned grid = grid_for(total);
  switch (counts_dtype) {
    case APIRL_F32:
      k_zero_bins<float><<<grid, kBlock, 0, st>>>(g, t, s, (const float*)counts, counts_packed, add, img, pad,
                                                 partials, total);
      break;
    case APIRL_U32:
      k_zero_bins<uint32_t><<<grid, kBlock, 0, st>>>(g, t, s, (const uint32_t*)counts, counts_packed, add, img,
                                                    pad, partials, total);
      break;
    case APIRL_U16:
      k_zero_bins<uint16_t><<<grid, kBlock, 0, st>>>(g, t, s, (const uint16_t*)counts, counts_packed, add, img,
                                                    pad, partials, total);
      break;
    default: return cudaErrorInvalidValue;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (pad.bA) {
    e = launch_pad_reduce(g, pad, 1, nullptr, img, nullptr, nullptr, 0.f, 0, st);
    if (e != cudaSuccess) return e;
  }
  if (!zero_add) return cudaSuccess;
  return launch_sum(partials, (int64_t)grid * (kBlock / 32), zero_add, st);
}

cudaError_t launch_inverse_divide(int64_t n, const float* meas, float* est, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_inverse_divide<<<stream_grid(n), kBlock, 0, st>>>(n, meas, est);
  return cudaGetLastError();
}

cudaError_t launch_add_bins(int64_t n, const float* add, float* est, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_add_bins<<<stream_grid(n), kBlock, 0, st>>>(n, add, est);
  return cudaGetLastError();
}

cudaError_t launch_likelihood(int64_t n, const float* est, const float* meas, int gt0, double* partials,
                              int64_t n_partials, double* out, cudaStream_t st) {
  const unsigned grid = stream_grid(n);
  if ((int64_t)grid > n_partials) return cudaErrorInvalidValue;
  k_likelihood<<<grid, kBlock, 0, st>>>(n, est, meas, gt0, partials);
  k_sum_partials<<<1, kBlock, 0, st>>>(partials, grid, out);
  return cudaGetLastError();
}

cudaError_t launch_threshold(int64_t n, const float* sens, unsigned* mm, float* thr, cudaStream_t st) {
  if (n == 0) return cudaErrorInvalidValue;
  k_minmax_init<<<1, 1, 0, st>>>(sens, mm);
  k_minmax<<<stream_grid(n), kBlock, 0, st>>>(n, sens, mm);
  k_threshold<<<1, 1, 0, st>>>(mm, thr);
  return cudaGetLastError();
}

cudaError_t launch_update(int64_t n, float* x, float* bp, const float* sens, const float* thr_ptr, float thr_value,
                          int ge, int zero_bp, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const int vec4 = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(bp) |
                     reinterpret_cast<uintptr_t>(sens)) & 15u) == 0;
  k_update<<<stream_grid((n + 3) / 4), kBlock, 0, st>>>(n, x, bp, sens, thr_ptr, thr_value, ge, zero_bp, vec4);
  return cudaGetLastError();
}

cudaError_t launch_force_positive(int64_t n, float* x, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_force_positive<<<stream_grid(n), kBlock, 0, st>>>(n, x);
  return cudaGetLastError();
}

cudaError_t launch_pad_copy(const ImgGeom& g, const float* x, const PadBuffers& pad, cudaStream_t st) {
  dim3 grid((g.nx + 31) / 32, (g.ny + 31) / 32, g.nz), block(32, 8);
  PadDims d{g.nx, g.ny, g.nz};
  return pad_launch(pad, grid, block, st, k_pad_copy, d, x, pad.pA, pad.pT);
}

cudaError_t launch_pad_reduce(const ImgGeom& g, const PadBuffers& pad, int mode, float* x, float* bp,
                              const float* sens, const float* thr_ptr, float thr_value, int ge, cudaStream_t st) {
  dim3 grid((g.nx + 31) / 32, (g.ny + 31) / 32, g.nz), block(32, 8);
  PadDims d{g.nx, g.ny, g.nz};
  float* eA = pad.acc == 2 ? pad.eA : nullptr;
  float* eT = pad.acc == 2 ? pad.eT : nullptr;
  return pad_launch(pad, grid, block, st, k_pad_reduce, d, pad.bA, pad.bT, mode, x, bp, sens, thr_ptr, thr_value, ge,
                    eA, eT);
}

cudaError_t launch_exp_nonzero(int64_t n, float* v, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_exp_nonzero<<<stream_grid(n), kBlock, 0, st>>>(n, v);
  return cudaGetLastError();
}

cudaError_t launch_fill(int64_t n, float* x, float v, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_fill<<<stream_grid(n), kBlock, 0, st>>>(n, x, v);
  return cudaGetLastError();
}

// Persistent grid of k_em_multi: as many 256-thread blocks as fit on the
// current device's SMs (its shared-memory carveout fitted to that many).
cudaError_t load_batch_kernels() {
  // CUDA loads a kernel's code at its first launch by default; asking for
  // each kernel's attributes loads it now instead.
  const void* fns[] = {
      (const void*)k_em_multi,          (const void*)k_multi_copy,         (const void*)k_multi_sum,
      (const void*)k_multi_update,      (const void*)k_scatter_angles,     (const void*)k_sum_angles,
      (const void*)k_sum_images,        (const void*)k_subset_sums,        (const void*)k_sens_batch,
      (const void*)k_nz_scan,           (const void*)k_nz_tiles<float>,    (const void*)k_nz_tiles<uint16_t>,
      (const void*)k_nz_tiles<uint32_t>, (const void*)k_nz_write<float>,   (const void*)k_nz_write<uint16_t>,
      (const void*)k_nz_write<uint32_t>};
  for (const void* f : fns) {
    cudaFuncAttributes a;
    const cudaError_t e = cudaFuncGetAttributes(&a, f);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t multi_walk_grid(int* blocks) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e;
  if ((e = fit_carveout((const void*)k_em_multi, kBlock, 0)) != cudaSuccess) return e;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_em_multi, kBlock, 0)) != cudaSuccess) return e;
  *blocks = (per_sm < 1 ? 1 : per_sm) * sms;
  return cudaSuccess;
}

cudaError_t launch_multi_step(const MultiVox* d_vox, int n_vox, int64_t total_tiles, const MultiSeg* d_segs,
                              int n_segs, int64_t total_chunks, int walk_blocks, unsigned long long* counter,
                              double* chunk_partials, double* tile_partials, cudaStream_t st) {
  if (n_vox == 0 || total_tiles == 0) return cudaSuccess;
  cudaError_t e;
  k_multi_copy<<<(unsigned)total_tiles, 256, 0, st>>>(d_vox, n_vox, tile_partials);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (total_chunks > 0 && n_segs > 0) {
    if ((e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st)) != cudaSuccess) return e;
    const int64_t need = (total_chunks * 32 + kBlock - 1) / kBlock;
    const unsigned grid = (unsigned)(need < walk_blocks ? need : walk_blocks);
    k_em_multi<<<grid, kBlock, 0, st>>>(d_segs, n_segs, total_chunks, counter, chunk_partials);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  k_multi_sum<<<n_vox, 256, 0, st>>>(d_vox, chunk_partials, tile_partials);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_multi_update<<<(unsigned)total_tiles, 256, 0, st>>>(d_vox, n_vox);
  return cudaGetLastError();
}

cudaError_t launch_nz_count(const LorTable& t, SubsetSel s, const void* counts, int counts_dtype, int64_t total,
                            int* tiles, int* n_list, cudaStream_t st) {
  if (total <= 0) return cudaMemsetAsync(n_list, 0, sizeof(int), st);
  const unsigned n_tiles = (unsigned)((total + kNzTile - 1) / kNzTile);
  switch (counts_dtype) {
    case APIRL_F32: k_nz_tiles<float><<<n_tiles, kNzBlock, 0, st>>>(t, s, (const float*)counts, 0, total, tiles); break;
    case APIRL_U32:
      k_nz_tiles<uint32_t><<<n_tiles, kNzBlock, 0, st>>>(t, s, (const uint32_t*)counts, 0, total, tiles);
      break;
    case APIRL_U16:
      k_nz_tiles<uint16_t><<<n_tiles, kNzBlock, 0, st>>>(t, s, (const uint16_t*)counts, 0, total, tiles);
      break;
    default: return cudaErrorInvalidValue;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_nz_scan<<<1, 1024, 0, st>>>(tiles, (int)n_tiles, n_list);
  return cudaGetLastError();
}

cudaError_t launch_nz_write(const LorTable& t, SubsetSel s, const void* counts, int counts_dtype, int64_t total,
                            const int* tiles, int* list, cudaStream_t st) {
  if (total <= 0) return cudaSuccess;
  const unsigned n_tiles = (unsigned)((total + kNzTile - 1) / kNzTile);
  switch (counts_dtype) {
    case APIRL_F32:
      k_nz_write<float><<<n_tiles, kNzBlock, 0, st>>>(t, s, (const float*)counts, 0, total, tiles, list);
      break;
    case APIRL_U32:
      k_nz_write<uint32_t><<<n_tiles, kNzBlock, 0, st>>>(t, s, (const uint32_t*)counts, 0, total, tiles, list);
      break;
    case APIRL_U16:
      k_nz_write<uint16_t><<<n_tiles, kNzBlock, 0, st>>>(t, s, (const uint16_t*)counts, 0, total, tiles, list);
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_scatter_angles(const ImgGeom& g, const LorTable& t, const uint8_t* tr_of, float* per_angle,
                                  unsigned lim, unsigned long long* counter, cudaStream_t st) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_scatter_angles, kBlock, 0)) != cudaSuccess)
    return e;
  if ((e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st)) != cudaSuccess) return e;
  const int64_t total = (int64_t)t.n_sinos * t.n_r * t.n_proj;
  const int64_t need = (total + kBlock - 1) / kBlock;
  const int64_t resident = (int64_t)(per_sm < 1 ? 1 : per_sm) * sms;
  k_scatter_angles<<<(unsigned)(need < resident ? need : resident), kBlock, 0, st>>>(g, t, tr_of, per_angle, lim,
                                                                                    counter);
  return cudaGetLastError();
}

cudaError_t launch_sum_angles(const float* per_angle, const uint8_t* tr_of, unsigned lim, int n_proj,
                              const ImgGeom& g, int nsub, float* out, cudaStream_t st) {
  if (nsub <= 0) return cudaSuccess;
  const int64_t tiles = multi_tiles(g);
  k_sum_angles<<<dim3((unsigned)tiles, (unsigned)nsub), 256, 0, st>>>(per_angle, tr_of, lim, n_proj, g, nsub, out);
  return cudaGetLastError();
}

cudaError_t launch_sum_images(const float* img, int n_img, int64_t nvox, int nsub, float* out, cudaStream_t st) {
  if (nvox == 0 || nsub <= 0) return cudaSuccess;
  int64_t bx = (nvox + kBlock - 1) / kBlock;
  if (bx > 2048) bx = 2048;
  k_sum_images<<<dim3((unsigned)bx, (unsigned)nsub), kBlock, 0, st>>>(img, n_img, nvox, nsub, out);
  return cudaGetLastError();
}

cudaError_t launch_subset_sums(const LorTable& t, int nsub, const float* add, double* out, cudaStream_t st) {
  if (nsub <= 0) return cudaSuccess;
  k_subset_sums<<<nsub, kBlock, 0, st>>>(t, nsub, add, out);
  return cudaGetLastError();
}

cudaError_t launch_sens_batch(const SensJob* d_jobs, int njobs, int64_t nblocks, cudaStream_t st) {
  if (njobs == 0 || nblocks == 0) return cudaSuccess;
  k_sens_batch<<<(unsigned)nblocks, kBlock, 0, st>>>(d_jobs, njobs);
  return cudaGetLastError();
}

}  // namespace apirl
