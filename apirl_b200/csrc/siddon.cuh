// Device-side Siddon ray walk for sm_100a.
//
// The walk restates the reference's serial Siddon (recon/src/Siddon.cpp:13-344
// for 3D, :358-643 for 2D) with the same float operations in the same order.
// Every add, multiply, divide and square root that feeds a weight or a voxel
// index is written with the round-to-nearest intrinsics (__fadd_rn, ...), which
// the compiler never contracts into FMAs, so each segment (voxel, length) is
// bit-identical to the reference compiled for x86 without FMA.  Instead of
// materialising a malloc'd segment list per LOR (Siddon.cpp:222) the walk hands
// each segment to a visitor in registers.
#pragma once
#include <cuda_runtime.h>
#include <cfloat>
#include <cstdint>
#include "geom_types.h"

namespace apirl {

#define A_ADD(a, b) __fadd_rn((a), (b))
#define A_SUB(a, b) __fsub_rn((a), (b))
#define A_MUL(a, b) __fmul_rn((a), (b))
#define A_DIV(a, b) __fdiv_rn((a), (b))

__device__ __forceinline__ float fmin_ref(float a, float b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ float fmax_ref(float a, float b) { return (a < b) ? b : a; }  // std::max

// Walk state after the set-up of one LOR.  `n` is the number of segments the
// reference records, |di| + |dj| + |dk| (Siddon.cpp:220).
struct Walk3 {
  float ax, ay, az, axu, ayu, azu, ac, L;
  int i, j, k, iinc, jinc, kinc, n;
  // 1 when the entry and exit voxel indices lie in [-1, n] on every axis
  // (see siddon3_gather_pad).
  int guarded;
};

__device__ __forceinline__ void siddon3_setup(float p0x, float p0y, float p0z, float vx, float vy, float vz,
                                              const ImgGeom& g, Walk3& w) {
  const float rFov = g.rfov;
  float amin, amax;
  if (vx == 0.f) {
    float a1 = A_DIV(A_SUB(-rFov, p0y), vy), a2 = A_DIV(A_SUB(rFov, p0y), vy);
    if (a1 < a2) { amin = a1; amax = a2; } else { amin = a2; amax = a1; }
  } else if (vy == 0.f) {
    float a1 = A_DIV(A_SUB(-rFov, p0x), vx), a2 = A_DIV(A_SUB(rFov, p0x), vx);
    if (a1 < a2) { amin = a1; amax = a2; } else { amin = a2; amax = a1; }
  } else {
    float ax1 = A_DIV(A_SUB(-rFov, p0x), vx), ay1 = A_DIV(A_SUB(-rFov, p0y), vy);
    float ax2 = A_DIV(A_SUB(rFov, p0x), vx), ay2 = A_DIV(A_SUB(rFov, p0y), vy);
    amin = fmax_ref(fmin_ref(ax1, ax2), fmin_ref(ay1, ay2));
    amax = fmin_ref(fmax_ref(ax1, ax2), fmax_ref(ay1, ay2));
  }
  if (amin < 0.f || amin > 1.f) amin = 0.f;
  if (amax > 1.f || amax < 0.f) amax = 1.f;
  const float x1 = A_ADD(p0x, A_MUL(vx, amin)), y1 = A_ADD(p0y, A_MUL(vy, amin)), z1 = A_ADD(p0z, A_MUL(vz, amin));
  const float x2 = A_ADD(p0x, A_MUL(vx, amax)), y2 = A_ADD(p0y, A_MUL(vy, amax)), z2 = A_ADD(p0z, A_MUL(vz, amax));
  const int imin = (int)floorf(A_DIV(A_ADD(x1, rFov), g.dx)), jmin = (int)floorf(A_DIV(A_ADD(y1, rFov), g.dy));
  const int kmin = (int)floorf(A_DIV(A_SUB(z1, g.offz), g.dz));
  const int imax = (int)floorf(A_DIV(A_ADD(x2, rFov), g.dx)), jmax = (int)floorf(A_DIV(A_ADD(y2, rFov), g.dy));
  const int kmax = (int)floorf(A_DIV(A_SUB(z2, g.offz), g.dz));
  w.n = abs(imax - imin) + abs(jmax - jmin) + abs(kmax - kmin);
  // Recorded indices run monotonically from the entry index towards the exit
  // index on each axis, so their range is bounded by the two.
  w.guarded = (min(imin, imax) >= -1) & (max(imin, imax) <= g.nx) & (min(jmin, jmax) >= -1) &
              (max(jmin, jmax) <= g.ny) & (min(kmin, kmax) >= -1) & (max(kmin, kmax) <= g.nz);
  w.iinc = vx > 0.f ? 1 : (vx < 0.f ? -1 : 0);
  w.jinc = vy > 0.f ? 1 : (vy < 0.f ? -1 : 0);
  w.kinc = vz > 0.f ? 1 : (vz < 0.f ? -1 : 0);
  const float ex = A_SUB(A_ADD(p0x, vx), p0x), ey = A_SUB(A_ADD(p0y, vy), p0y), ez = A_SUB(A_ADD(p0z, vz), p0z);
  w.L = __fsqrt_rn(A_ADD(A_ADD(A_MUL(ex, ex), A_MUL(ey, ey)), A_MUL(ez, ez)));
  w.axu = fabsf(A_DIV(g.dx, vx));
  w.ayu = fabsf(A_DIV(g.dy, vy));
  w.azu = fabsf(A_DIV(g.dz, vz));
  w.ax = vx > 0.f ? A_DIV(A_SUB(A_ADD(-rFov, A_MUL((float)(imin + w.iinc), g.dx)), p0x), vx)
       : (vx < 0.f ? A_DIV(A_SUB(A_ADD(-rFov, A_MUL((float)imin, g.dx)), p0x), vx) : FLT_MAX);
  w.ay = vy > 0.f ? A_DIV(A_SUB(A_ADD(-rFov, A_MUL((float)(jmin + w.jinc), g.dy)), p0y), vy)
       : (vy < 0.f ? A_DIV(A_SUB(A_ADD(-rFov, A_MUL((float)jmin, g.dy)), p0y), vy) : FLT_MAX);
  w.az = vz > 0.f ? A_DIV(A_SUB(A_ADD(g.offz, A_MUL((float)(kmin + w.kinc), g.dz)), p0z), vz)
       : (vz < 0.f ? A_DIV(A_SUB(A_ADD(g.offz, A_MUL((float)kmin, g.dz)), p0z), vz) : FLT_MAX);
  w.ac = amin;
  w.i = imin; w.j = jmin; w.k = kmin;
}

// Visits the n recorded segments in order: visit(inb, linear_index, length).
// `inb` is the full six-sided bounds test; linear_index = (k*ny + j)*nx + i is
// only meaningful when inb is true.  Record-then-advance as in Siddon.cpp:310-340.
template <class V>
__device__ __forceinline__ void siddon3_walk(Walk3 w, const ImgGeom& g, V&& visit);

// The next crossing of a walk, min(ax, ay, az) with the reference's tie order
// x, y, z (Siddon.cpp:317-339); cx / cy tell which axis it is.  The crossing
// parameters are never NaN, so min-then-compare selects exactly the
// reference's branch.
#ifndef APIRL_SEL_MINMAX
#define APIRL_SEL_MINMAX 1
#endif
__device__ __forceinline__ float next_crossing(const Walk3& w, bool& cx, bool& cy) {
#if APIRL_SEL_MINMAX
  const float an = fminf(fminf(w.ax, w.ay), w.az);
  cx = w.ax == an;
  cy = !cx & (w.ay == an);
  return an;
#else
  cx = (w.ax <= w.ay) & (w.ax <= w.az);
  cy = !cx & (w.ay <= w.az);
  return cx ? w.ax : (cy ? w.ay : w.az);
#endif
}

// One step of a guarded padded walk past its next crossing (x when cx, y
// when cy, else z): the linear index moves one voxel along that axis and the
// axis's crossing parameter advances by its increment.  APIRL_STEP_SELECT
// computes all three candidate parameters and selects (no divergent branch;
// the same float additions on the same operands, so the walk is unchanged):
// on B200 0.5 % faster on the listed pass and 4 % slower on the full pass
// than the branch, so it is off by default.
#ifndef APIRL_STEP_SELECT
#define APIRL_STEP_SELECT 0
#endif
__device__ __forceinline__ void step_pad(Walk3& w, int& idx, bool cx, bool cy, int sx, int sy, int sz) {
#if APIRL_STEP_SELECT
  const float ax = A_ADD(w.ax, w.axu), ay = A_ADD(w.ay, w.ayu), az = A_ADD(w.az, w.azu);
  idx += cx ? sx : (cy ? sy : sz);
  w.ax = cx ? ax : w.ax;
  w.ay = cy ? ay : w.ay;
  w.az = (cx | cy) ? w.az : az;
#else
  if (cx) { idx += sx; w.ax = A_ADD(w.ax, w.axu); }
  else if (cy) { idx += sy; w.ay = A_ADD(w.ay, w.ayu); }
  else { idx += sz; w.az = A_ADD(w.az, w.azu); }
#endif
}

// Walks over an image padded with a kPad-voxel zero border on every side
// (padded sizes n+2 kPad; unit strides ux, uy, uz of the padded layout; `lim`
// = number of padded voxels).  When w.guarded the entry and exit indices lie
// in [-1, n]; recorded indices run between them, and float ties at the exit
// can add at most one crossing per axis beyond it (the crossing parameters'
// rounding error is orders below one crossing step), so the walk stays in
// [-2, n+1], inside the border: a border segment reads a zero (the sum is
// unchanged; the reference skips it) or scatters into the border, which
// nothing reads.  The three per-axis bounds tests become one clamp of the
// linear index to the padded volume's last voxel (a border voxel), kept as a
// memory-safety net.
// Otherwise the reference's bounds test is applied.
// Segments per iteration of the guarded gather: their voxel loads are all
// issued before any product is added (the additions keep the walk order).
#ifndef APIRL_GATHER_UNROLL
#define APIRL_GATHER_UNROLL 4
#endif
template <int U = APIRL_GATHER_UNROLL>
__device__ __forceinline__ float siddon3_gather_pad(Walk3 w, const ImgGeom& g, int ux, int uy, int uz, unsigned lim,
                                                    const float* __restrict__ img, int delay = 0) {
  const int sx = w.iinc * ux, sy = w.jinc * uy, sz = w.kinc * uz;
  int idx = (w.k + kPad) * uz + (w.j + kPad) * uy + (w.i + kPad) * ux;
  float acc = 0.f;
  if (w.guarded) {
    // `delay` idle iterations first (walk_delay): the segments and their sum
    // order are unchanged.
    int m = -(delay / U) * U;
    for (; m + U <= w.n; m += U) {
      if (m < 0) continue;
      int ia[U];
      float sa[U], va[U];
      #pragma unroll
      for (int u = 0; u < U; u++) {
        bool cx, cy;
        const float an = next_crossing(w, cx, cy);
        sa[u] = A_MUL(A_SUB(an, w.ac), w.L);
        ia[u] = idx;
        w.ac = an;
        step_pad(w, idx, cx, cy, sx, sy, sz);
      }
      #pragma unroll
      for (int u = 0; u < U; u++) va[u] = __ldg(img + min((unsigned)ia[u], lim - 1u));
      #pragma unroll
      for (int u = 0; u < U; u++) acc = A_ADD(acc, A_MUL(sa[u], va[u]));
    }
    for (; m < w.n; m++) {
      bool cx, cy;
      const float an = next_crossing(w, cx, cy);
      const float v = __ldg(img + min((unsigned)idx, lim - 1u));
      acc = A_ADD(acc, A_MUL(A_MUL(A_SUB(an, w.ac), w.L), v));
      w.ac = an;
      step_pad(w, idx, cx, cy, sx, sy, sz);
    }
    return acc;
  }
  for (int m = 0; m < w.n; m++) {
    bool cx, cy;
    const float an = next_crossing(w, cx, cy);
    const float seg = A_MUL(A_SUB(an, w.ac), w.L);
    if (((unsigned)w.i < (unsigned)g.nx) & ((unsigned)w.j < (unsigned)g.ny) & ((unsigned)w.k < (unsigned)g.nz))
      acc = A_ADD(acc, A_MUL(seg, __ldg(img + idx)));
    w.ac = an;
    if (cx) { w.i += w.iinc; idx += sx; w.ax = A_ADD(w.ax, w.axu); }
    else if (cy) { w.j += w.jinc; idx += sy; w.ay = A_ADD(w.ay, w.ayu); }
    else { w.k += w.kinc; idx += sz; w.az = A_ADD(w.az, w.azu); }
  }
  return acc;
}

// Start delay of a walk, in crossings, that lines up the walks of a warp's
// lanes.  The lanes of a warp walk parallel rays side by side (consecutive r
// of one angle and sinogram), but where the rays enter the square field of
// view through different faces, their entries lie rows apart along the main
// axis of travel (y when |vy| > |vx|, else x), and so do their steps m: the
// accesses of one warp step then fall in as many sectors as rows.  A lane
// whose entry lies further along the main axis waits as many crossings as
// separate it from the first-entering lane of its group (the lanes with the
// same `key`): the entry's main-axis coordinate in the direction of travel
// (mm) times the ray's crossings per mm of main-axis travel.  Capped at
// kMaxWalkDelay.  This changes only when a lane issues its steps, never
// which steps or in what order.  All lanes that are converged at the call
// take part.
constexpr int kMaxWalkDelay = 128;
__device__ __forceinline__ int walk_delay(const Walk3& w, const ImgGeom& g, float p0x, float p0y, float vx, float vy,
                                          float vz, unsigned key) {
  const float ax = fabsf(vx), ay = fabsf(vy);
  const bool xmain = ax >= ay;
  const float entry = xmain ? (vx > 0.f ? 1.f : -1.f) * (p0x + vx * w.ac) : (vy > 0.f ? 1.f : -1.f) * (p0y + vy * w.ac);
  const float per_mm = (ax / g.dx + ay / g.dy + fabsf(vz) / g.dz) / (xmain ? ax : ay);
  const int k = __float2int_rn(entry * per_mm);
  const unsigned group = __match_any_sync(__activemask(), key);
  const int kmin = __reduce_min_sync(group, k);
  return min(k - kmin, kMaxWalkDelay);
}

// How a scatter step adds v into img[at] (APIRL_OPT_ACCUMULATE):
//  0  one atomic add per segment (the reference's `#pragma omp atomic` float
//     add, SiddonProjector.cpp:547-548, in the atomics' order);
//  1  warp-aggregated (siddon3_scatter_pad_warp below, not here);
//  2  compensated: the atomic returns the value it added to, so the rounding
//     error of that addition (TwoSum, Knuth) is known exactly and goes into
//     a second image err; img + err is the sum to about twice float precision.
// A float add into global memory whose result nobody reads: a reduction
// (red.global), which the SM issues without waiting for a reply.  Stated
// explicitly because atomicAdd on a pointer the compiler cannot place (one
// read from shared memory, as in the batched walk's per-job descriptors)
// becomes a generic atomic instead.
#ifndef APIRL_RED_GLOBAL
#define APIRL_RED_GLOBAL 1
#endif
__device__ __forceinline__ void red_add_global(float* p, float v) {
#if APIRL_RED_GLOBAL
  asm volatile("red.relaxed.gpu.global.add.f32 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "f"(v) : "memory");
#else
  atomicAdd(p, v);
#endif
}

template <int ACC>
__device__ __forceinline__ void acc_add(float* __restrict__ img, float* __restrict__ err, unsigned at, float v) {
  if (ACC == 2) {
    const float old = atomicAdd(img + at, v);
    const float s = A_ADD(old, v);
    const float bv = A_SUB(s, old);
    const float e = A_ADD(A_SUB(old, A_SUB(s, bv)), A_SUB(v, bv));
    if (e != 0.f) red_add_global(err + at, e);
  } else {
    red_add_global(img + at, v);
  }
}

template <int ACC = 0>
__device__ __forceinline__ void siddon3_scatter_pad(Walk3 w, const ImgGeom& g, int ux, int uy, int uz, unsigned lim,
                                                    float r, float* __restrict__ img,
                                                    float* __restrict__ err = nullptr, int delay = 0) {
  const int sx = w.iinc * ux, sy = w.jinc * uy, sz = w.kinc * uz;
  int idx = (w.k + kPad) * uz + (w.j + kPad) * uy + (w.i + kPad) * ux;
  if (w.guarded) {
    // `delay` idle iterations first (walk_delay); a lane's adds go to
    // distinct voxels, so when they are issued changes nothing but the
    // (already unordered) interleaving with other lanes' adds.
    for (int m = -delay; m < w.n; m++) {
      if (m < 0) continue;
      bool cx, cy;
      const float an = next_crossing(w, cx, cy);
      acc_add<ACC>(img, err, min((unsigned)idx, lim - 1u), A_MUL(A_MUL(A_SUB(an, w.ac), w.L), r));
      w.ac = an;
      step_pad(w, idx, cx, cy, sx, sy, sz);
    }
    return;
  }
  for (int m = 0; m < w.n; m++) {
    bool cx, cy;
    const float an = next_crossing(w, cx, cy);
    const float seg = A_MUL(A_SUB(an, w.ac), w.L);
    if (((unsigned)w.i < (unsigned)g.nx) & ((unsigned)w.j < (unsigned)g.ny) & ((unsigned)w.k < (unsigned)g.nz))
      acc_add<ACC>(img, err, (unsigned)idx, A_MUL(seg, r));
    w.ac = an;
    if (cx) { w.i += w.iinc; idx += sx; w.ax = A_ADD(w.ax, w.axu); }
    else if (cy) { w.j += w.jinc; idx += sy; w.ay = A_ADD(w.ay, w.ayu); }
    else { w.k += w.kinc; idx += sz; w.az = A_ADD(w.az, w.azu); }
  }
}

// The warp-aggregated scatter (accumulation form 1): all 32 lanes of the warp
// call it together, each with its own walk (live == false: a lane that adds
// nothing), and step through their walks in lockstep to the longest one.  At
// each step the lanes whose segments fall on the same address (same image and
// voxel: the lanes of a warp may scatter into different images) sum their
// values in lane order (through a per-lane slot of shared memory; blocks of
// at most 256 threads) and the lowest of them adds the sum with one atomic.
// Bounds: the guarded walk's clamp, else the reference's six-sided test.
__device__ __forceinline__ void siddon3_scatter_pad_warp(Walk3 w, const ImgGeom& g, int ux, int uy, int uz,
                                                         unsigned lim, float r, float* __restrict__ img, bool live) {
  __shared__ float slot[256];
  const int lane = (int)(threadIdx.x & 31), warp0 = (int)threadIdx.x - lane;
  const int n = live ? w.n : 0;
  const int nmax = __reduce_max_sync(0xffffffffu, n);
  const int sx = w.iinc * ux, sy = w.jinc * uy, sz = w.kinc * uz;
  int idx = live ? (w.k + kPad) * uz + (w.j + kPad) * uy + (w.i + kPad) * ux : 0;
  for (int m = 0; m < nmax; m++) {
    unsigned at = lim;  // no voxel: this lane adds nothing this step
    float v = 0.f;
    if (m < n) {
      bool cx, cy;
      const float an = next_crossing(w, cx, cy);
      const float seg = A_MUL(A_SUB(an, w.ac), w.L);
      const bool inb = w.guarded || (((unsigned)w.i < (unsigned)g.nx) & ((unsigned)w.j < (unsigned)g.ny) &
                                     ((unsigned)w.k < (unsigned)g.nz));
      if (inb) {
        at = min((unsigned)idx, lim - 1u);
        v = A_MUL(seg, r);
      }
      w.ac = an;
      if (cx) { w.i += w.iinc; idx += sx; w.ax = A_ADD(w.ax, w.axu); }
      else if (cy) { w.j += w.jinc; idx += sy; w.ay = A_ADD(w.ay, w.ayu); }
      else { w.k += w.kinc; idx += sz; w.az = A_ADD(w.az, w.azu); }
    }
    // the address, or a value no address has (one group per idle lane)
    const unsigned long long key =
        at < lim ? (unsigned long long)(uintptr_t)(img + at) : ~0ull - (unsigned long long)lane;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    slot[threadIdx.x] = v;
    __syncwarp();
    if (at < lim && lane == __ffs(peers) - 1) {
      float sum = 0.f;
      for (unsigned q = peers; q; q &= q - 1u) sum = A_ADD(sum, slot[warp0 + __ffs(q) - 1]);
      red_add_global(img + at, sum);
    }
    __syncwarp();
  }
}

// siddon3_scatter_pad into two images of the same padded layout along one
// walk: seg * r1 into img1 (skipped when r1 == 0) and seg into img2.
__device__ __forceinline__ void siddon3_scatter2_pad(Walk3 w, const ImgGeom& g, int ux, int uy, int uz, unsigned lim,
                                                     float r1, float* __restrict__ img1, float* __restrict__ img2) {
  const int sx = w.iinc * ux, sy = w.jinc * uy, sz = w.kinc * uz;
  int idx = (w.k + kPad) * uz + (w.j + kPad) * uy + (w.i + kPad) * ux;
  const bool first = r1 != 0.f;
  for (int m = 0; m < w.n; m++) {
    bool cx, cy;
    const float an = next_crossing(w, cx, cy);
    const float seg = A_MUL(A_SUB(an, w.ac), w.L);
    const bool inb = w.guarded || (((unsigned)w.i < (unsigned)g.nx) & ((unsigned)w.j < (unsigned)g.ny) &
                                   ((unsigned)w.k < (unsigned)g.nz));
    if (inb) {
      const unsigned at = min((unsigned)idx, lim - 1u);
      if (first) red_add_global(img1 + at, A_MUL(seg, r1));
      red_add_global(img2 + at, seg);
    }
    w.ac = an;
    if (cx) { w.i += w.iinc; idx += sx; w.ax = A_ADD(w.ax, w.axu); }
    else if (cy) { w.j += w.jinc; idx += sy; w.ay = A_ADD(w.ay, w.ayu); }
    else { w.k += w.kinc; idx += sz; w.az = A_ADD(w.az, w.azu); }
  }
}

template <class V>
__device__ __forceinline__ void siddon3_walk(Walk3 w, const ImgGeom& g, V&& visit) {
  const int sx = w.iinc, sy = w.jinc * g.nx, sz = w.kinc * g.nx * g.ny;
  int idx = (w.k * g.ny + w.j) * g.nx + w.i;
  for (int m = 0; m < w.n; m++) {
    bool cx, cy;
    const float an = next_crossing(w, cx, cy);
    const float seg = A_MUL(A_SUB(an, w.ac), w.L);
    const bool inb = ((unsigned)w.i < (unsigned)g.nx) & ((unsigned)w.j < (unsigned)g.ny) &
                     ((unsigned)w.k < (unsigned)g.nz);
    visit(inb, idx, seg);
    w.ac = an;
    if (cx) { w.i += w.iinc; idx += sx; w.ax = A_ADD(w.ax, w.axu); }
    else if (cy) { w.j += w.jinc; idx += sy; w.ay = A_ADD(w.ay, w.ayu); }
    else { w.k += w.kinc; idx += sz; w.az = A_ADD(w.az, w.azu); }
  }
}

// ---------------------------------------------------------------------------
// 2D (Siddon.cpp:358-643).  Differences from 3D: early exit when both end
// indices are outside on one side (:515-519), negative first crossings clamp
// to alpha_min (:596-606), and the weight is multiplied by `factor` (1 here).
struct Walk2 {
  float ax, ay, axu, ayu, ac, L;
  int i, j, iinc, jinc, n;
};

__device__ __forceinline__ void siddon2_setup(float p0x, float p0y, float vx, float vy, const ImgGeom& g, Walk2& w) {
  const float rFov = g.rfov;
  float amin, amax;
  if (vx == 0.f) {
    float a1 = A_DIV(A_SUB(-rFov, p0y), vy), a2 = A_DIV(A_SUB(rFov, p0y), vy);
    if (a1 < a2) { amin = a1; amax = a2; } else { amin = a2; amax = a1; }
  } else if (vy == 0.f) {
    float a1 = A_DIV(A_SUB(-rFov, p0x), vx), a2 = A_DIV(A_SUB(rFov, p0x), vx);
    if (a1 < a2) { amin = a1; amax = a2; } else { amin = a2; amax = a1; }
  } else {
    float ax1 = A_DIV(A_SUB(-rFov, p0x), vx), ay1 = A_DIV(A_SUB(-rFov, p0y), vy);
    float ax2 = A_DIV(A_SUB(rFov, p0x), vx), ay2 = A_DIV(A_SUB(rFov, p0y), vy);
    amin = fmax_ref(fmin_ref(ax1, ax2), fmin_ref(ay1, ay2));
    amax = fmin_ref(fmax_ref(ax1, ax2), fmax_ref(ay1, ay2));
  }
  if (amin < 0.f || amin > 1.f) amin = 0.f;
  if (amax > 1.f || amax < 0.f) amax = 1.f;
  const float x1 = A_ADD(p0x, A_MUL(vx, amin)), y1 = A_ADD(p0y, A_MUL(vy, amin));
  const float x2 = A_ADD(p0x, A_MUL(vx, amax)), y2 = A_ADD(p0y, A_MUL(vy, amax));
  const int imin = (int)floorf(A_DIV(A_ADD(x1, rFov), g.dx)), jmin = (int)floorf(A_DIV(A_ADD(y1, rFov), g.dy));
  const int imax = (int)floorf(A_DIV(A_ADD(x2, rFov), g.dx)), jmax = (int)floorf(A_DIV(A_ADD(y2, rFov), g.dy));
  if ((imin < 0 && imax < 0) || (jmin < 0 && jmax < 0) || (imin >= g.nx && imax >= g.nx) ||
      (jmin >= g.ny && jmax >= g.ny)) {
    w.n = 0;
    return;
  }
  w.n = abs(imax - imin) + abs(jmax - jmin);
  w.iinc = vx > 0.f ? 1 : (vx < 0.f ? -1 : 0);
  w.jinc = vy > 0.f ? 1 : (vy < 0.f ? -1 : 0);
  const float ex = A_SUB(A_ADD(p0x, vx), p0x), ey = A_SUB(A_ADD(p0y, vy), p0y);
  w.L = __fsqrt_rn(A_ADD(A_MUL(ex, ex), A_MUL(ey, ey)));
  w.axu = fabsf(A_DIV(g.dx, vx));
  w.ayu = fabsf(A_DIV(g.dy, vy));
  float ax = vx > 0.f ? A_DIV(A_SUB(A_ADD(-rFov, A_MUL((float)(imin + w.iinc), g.dx)), p0x), vx)
           : (vx < 0.f ? A_DIV(A_SUB(A_ADD(-rFov, A_MUL((float)imin, g.dx)), p0x), vx) : FLT_MAX);
  if (ax < 0.f) ax = amin;
  float ay = vy > 0.f ? A_DIV(A_SUB(A_ADD(-rFov, A_MUL((float)(jmin + w.jinc), g.dy)), p0y), vy)
           : (vy < 0.f ? A_DIV(A_SUB(A_ADD(-rFov, A_MUL((float)jmin, g.dy)), p0y), vy) : FLT_MAX);
  if (ay < 0.f) ay = amin;
  w.ax = ax; w.ay = ay;
  w.ac = amin;
  w.i = imin; w.j = jmin;
}

template <class V>
__device__ __forceinline__ void siddon2_walk(Walk2 w, const ImgGeom& g, V&& visit) {
  const int sy = w.jinc * g.nx;
  int idx = w.j * g.nx + w.i;
  for (int m = 0; m < w.n; m++) {
    const bool cx = (w.ax <= w.ay);
    const float an = cx ? w.ax : w.ay;
    // ((alpha - alpha_c) * L) * factor with factor = 1: the product by 1 is exact.
    const float seg = A_MUL(A_SUB(an, w.ac), w.L);
    const bool inb = ((unsigned)w.i < (unsigned)g.nx) & ((unsigned)w.j < (unsigned)g.ny);
    visit(inb, idx, seg);
    w.ac = an;
    if (cx) { w.i += w.iinc; idx += w.iinc; w.ax = A_ADD(w.ax, w.axu); }
    else { w.j += w.jinc; idx += sy; w.ay = A_ADD(w.ay, w.ayu); }
  }
}

}  // namespace apirl

// ---------------------------------------------------------------------------
// FP64-alpha variant (precision mode, not the reference's arithmetic): ray
// entry/exit, first crossings and the running crossing parameters are kept in
// double so that long oblique rays cannot misorder voxel crossings; each
// segment length is rounded to float once.  End points come from a double
// table built with double trigonometry.
namespace apirl {

struct ImgGeomD {
  int nx, ny, nz;
  double dx, dy, dz, rfov, offz;
};

struct Walk3D {
  double ax, ay, az, axu, ayu, azu, ac, L;
  int i, j, k, iinc, jinc, kinc, n;
};

__device__ __forceinline__ double dmin_ref(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double dmax_ref(double a, double b) { return (a < b) ? b : a; }

__device__ __forceinline__ void siddon3d_setup(double p0x, double p0y, double p0z, double vx, double vy, double vz,
                                               const ImgGeomD& g, Walk3D& w) {
  const double rFov = g.rfov;
  double amin, amax;
  if (vx == 0.0) {
    double a1 = __ddiv_rn(-rFov - p0y, vy), a2 = __ddiv_rn(rFov - p0y, vy);
    if (a1 < a2) { amin = a1; amax = a2; } else { amin = a2; amax = a1; }
  } else if (vy == 0.0) {
    double a1 = __ddiv_rn(-rFov - p0x, vx), a2 = __ddiv_rn(rFov - p0x, vx);
    if (a1 < a2) { amin = a1; amax = a2; } else { amin = a2; amax = a1; }
  } else {
    double ax1 = __ddiv_rn(-rFov - p0x, vx), ay1 = __ddiv_rn(-rFov - p0y, vy);
    double ax2 = __ddiv_rn(rFov - p0x, vx), ay2 = __ddiv_rn(rFov - p0y, vy);
    amin = dmax_ref(dmin_ref(ax1, ax2), dmin_ref(ay1, ay2));
    amax = dmin_ref(dmax_ref(ax1, ax2), dmax_ref(ay1, ay2));
  }
  if (amin < 0.0 || amin > 1.0) amin = 0.0;
  if (amax > 1.0 || amax < 0.0) amax = 1.0;
  const double x1 = __dadd_rn(p0x, __dmul_rn(vx, amin)), y1 = __dadd_rn(p0y, __dmul_rn(vy, amin));
  const double z1 = __dadd_rn(p0z, __dmul_rn(vz, amin));
  const double x2 = __dadd_rn(p0x, __dmul_rn(vx, amax)), y2 = __dadd_rn(p0y, __dmul_rn(vy, amax));
  const double z2 = __dadd_rn(p0z, __dmul_rn(vz, amax));
  const int imin = (int)floor(__ddiv_rn(x1 + rFov, g.dx)), jmin = (int)floor(__ddiv_rn(y1 + rFov, g.dy));
  const int kmin = (int)floor(__ddiv_rn(z1 - g.offz, g.dz));
  const int imax = (int)floor(__ddiv_rn(x2 + rFov, g.dx)), jmax = (int)floor(__ddiv_rn(y2 + rFov, g.dy));
  const int kmax = (int)floor(__ddiv_rn(z2 - g.offz, g.dz));
  w.n = abs(imax - imin) + abs(jmax - jmin) + abs(kmax - kmin);
  w.iinc = vx > 0.0 ? 1 : (vx < 0.0 ? -1 : 0);
  w.jinc = vy > 0.0 ? 1 : (vy < 0.0 ? -1 : 0);
  w.kinc = vz > 0.0 ? 1 : (vz < 0.0 ? -1 : 0);
  const double ex = (p0x + vx) - p0x, ey = (p0y + vy) - p0y, ez = (p0z + vz) - p0z;
  w.L = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)), __dmul_rn(ez, ez)));
  w.axu = fabs(__ddiv_rn(g.dx, vx));
  w.ayu = fabs(__ddiv_rn(g.dy, vy));
  w.azu = fabs(__ddiv_rn(g.dz, vz));
  const double big = 1.7976931348623157e308;
  w.ax = vx > 0.0 ? __ddiv_rn(-rFov + (double)(imin + w.iinc) * g.dx - p0x, vx)
       : (vx < 0.0 ? __ddiv_rn(-rFov + (double)imin * g.dx - p0x, vx) : big);
  w.ay = vy > 0.0 ? __ddiv_rn(-rFov + (double)(jmin + w.jinc) * g.dy - p0y, vy)
       : (vy < 0.0 ? __ddiv_rn(-rFov + (double)jmin * g.dy - p0y, vy) : big);
  w.az = vz > 0.0 ? __ddiv_rn(g.offz + (double)(kmin + w.kinc) * g.dz - p0z, vz)
       : (vz < 0.0 ? __ddiv_rn(g.offz + (double)kmin * g.dz - p0z, vz) : big);
  w.ac = amin;
  w.i = imin; w.j = jmin; w.k = kmin;
}

template <class V>
__device__ __forceinline__ void siddon3d_walk(Walk3D w, const ImgGeomD& g, V&& visit) {
  const int sx = w.iinc, sy = w.jinc * g.nx, sz = w.kinc * g.nx * g.ny;
  int idx = (w.k * g.ny + w.j) * g.nx + w.i;
  for (int m = 0; m < w.n; m++) {
    const bool cx = (w.ax <= w.ay) && (w.ax <= w.az);
    const bool cy = !cx && (w.ay <= w.ax) && (w.ay <= w.az);
    const double an = cx ? w.ax : (cy ? w.ay : w.az);
    const float seg = (float)__dmul_rn(an - w.ac, w.L);
    const bool inb = ((unsigned)w.i < (unsigned)g.nx) & ((unsigned)w.j < (unsigned)g.ny) &
                     ((unsigned)w.k < (unsigned)g.nz);
    visit(inb, idx, seg);
    w.ac = an;
    if (cx) { w.i += w.iinc; idx += sx; w.ax += w.axu; }
    else if (cy) { w.j += w.jinc; idx += sy; w.ay += w.ayu; }
    else { w.k += w.kinc; idx += sz; w.az += w.azu; }
  }
}

}  // namespace apirl
