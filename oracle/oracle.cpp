// Test infrastructure, not product code.
//
// CPU restatement of the reference APIRL Siddon projector, backprojector and
// the MLEM / OSEM loops around them.  It is the checker for the CUDA path: only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.  The
// product library never links or calls it.
//
// Every routine is templated on the arithmetic type T.  With T = float it
// follows the reference's float expressions operation by operation (same
// operand order, no fused multiply-add: build with -ffp-contract=off), so that
// its results are bit-identical to the reference compiled with the same
// compiler on the same inputs.  With T = double it is the FP64 oracle that the
// precision study states errors against.
//
// Semantics restated (reference file:line):
//   Siddon 3D walk ............ recon/src/Siddon.cpp:13-344
//   Siddon 2D walk ............ recon/src/Siddon.cpp:358-643
//   2D Project / Backproject .. recon/src/SiddonProjector.cpp:146-193 / 34-87
//   2D DivideAndBackproject ... recon/src/SiddonProjector.cpp:90-144
//   3D Project / Backproject .. recon/src/SiddonProjector.cpp:322-441 / 444-568
//   3D DivideAndBackproject ... recon/src/SiddonProjector.cpp:571-704
//   sampled LORs (numSamplesOnDetector, numAxialSamplesOnDetector,
//   useMultipleLorsPerBin) ..... recon/src/SiddonProjector.cpp:346-397, 466-510,
//                               626-652; data/src/Sinogram2DinCylindrical3Dpet.cpp:283-299,
//                               data/src/Sinogram2D.cpp:172-187 (getDeltaR)
//   LOR end points ............ data/src/Sinogram2DinCylindrical3Dpet.cpp:216-266
//   r / angle tables .......... data/src/Sinogram2DinCylindrical3Dpet.cpp:46-63
//   ring z, ring pairs ........ data/src/Sinogram3D.cpp:358-464
//   subsets ................... data/src/Sinogram3DCylindricalPet.cpp:164-197
//   ratio ..................... data/src/Sinogram3D.cpp:830-855, Sinogram2D.cpp:245-266
//   likelihood ................ data/src/Sinogram3D.cpp:584-606, Sinogram2D.cpp:565-581
//   EM update, thresholds ..... recon/src/Mlem2d.cpp:171-185, MlemSinogram3d.cpp:228-242,
//                               OsemSinogram3d.cpp:24-33,217-237, recon/src/Mlem.cpp:39-43,
//                               data/src/Images.cpp:383-433
//   drivers ................... recon/src/Mlem2d.cpp:60-278, OsemSinogram3d.cpp:36-346
//
// One deliberate difference from the reference: the voxel index of every
// Siddon segment is checked against all six image bounds before a voxel is
// read or written.  The reference checks only the lower bounds in the 2D
// Project (SiddonProjector.cpp:178) and only the upper bounds in the 3D
// Project and DivideAndBackproject (:417, :666), and so reads or writes outside
// the image for a few rays.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <vector>
#include <algorithm>
#include <omp.h>

namespace {

template <typename T> struct Consts;
template <> struct Consts<float> {
  static float deg_to_rad() { return 0.01745329251994329576f; }  // data/../Geometry.h:10
  static float big() { return std::numeric_limits<float>::max(); }
};
template <> struct Consts<double> {
  static double deg_to_rad() { return 0.017453292519943295769; }
  static double big() { return std::numeric_limits<double>::max(); }
};

template <typename T> inline T tmin(T a, T b) { return (b < a) ? b : a; }  // std::min
template <typename T> inline T tmax(T a, T b) { return (a < b) ? b : a; }  // std::max

template <typename T> struct ImgG {
  int nx, ny, nz;
  T dx, dy, dz;
  T rfov;  // (dx * nx) / 2, data/src/Images.cpp:55
};

template <typename T> ImgG<T> make_img(int nx, int ny, int nz, float dx, float dy, float dz) {
  ImgG<T> g;
  g.nx = nx; g.ny = ny; g.nz = nz;
  g.dx = (T)dx; g.dy = (T)dy; g.dz = (T)dz;
  g.rfov = (g.dx * (T)nx) / (T)2;
  return g;
}

// ---------------------------------------------------------------------------
// Siddon walks.  visit(i, j, k, w) receives every recorded segment in walk order.
template <typename T, typename V>
int siddon3d(T p0x, T p0y, T p0z, T vx, T vy, T vz, const ImgG<T>& g, V&& visit) {
  const T rFov = g.rfov;
  T amin, amax;
  if (vx == 0) {
    T a1 = (-rFov - p0y) / vy, a2 = (rFov - p0y) / vy;
    if (a1 < a2) { amin = a1; amax = a2; } else { amin = a2; amax = a1; }
  } else if (vy == 0) {
    T a1 = (-rFov - p0x) / vx, a2 = (rFov - p0x) / vx;
    if (a1 < a2) { amin = a1; amax = a2; } else { amin = a2; amax = a1; }
  } else {
    T ax1 = (-rFov - p0x) / vx, ay1 = (-rFov - p0y) / vy;
    T ax2 = (rFov - p0x) / vx, ay2 = (rFov - p0y) / vy;
    amin = tmax(tmin(ax1, ax2), tmin(ay1, ay2));
    amax = tmin(tmax(ax1, ax2), tmax(ay1, ay2));
  }
  if (amin < 0 || amin > 1) amin = 0;
  if (amax > 1 || amax < 0) amax = 1;
  T x1 = p0x + vx * amin, y1 = p0y + vy * amin, z1 = p0z + vz * amin;
  T x2 = p0x + vx * amax, y2 = p0y + vy * amax, z2 = p0z + vz * amax;
  const T offZ = g.dz / 2;
  int imin = (int)std::floor((x1 + rFov) / g.dx), jmin = (int)std::floor((y1 + rFov) / g.dy);
  int kmin = (int)std::floor((z1 - offZ) / g.dz);
  int imax = (int)std::floor((x2 + rFov) / g.dx), jmax = (int)std::floor((y2 + rFov) / g.dy);
  int kmax = (int)std::floor((z2 - offZ) / g.dz);
  int n = std::abs(imax - imin) + std::abs(jmax - jmin) + std::abs(kmax - kmin);
  int iinc = vx > 0 ? 1 : (vx < 0 ? -1 : 0);
  int jinc = vy > 0 ? 1 : (vy < 0 ? -1 : 0);
  int kinc = vz > 0 ? 1 : (vz < 0 ? -1 : 0);
  T ex = (p0x + vx) - p0x, ey = (p0y + vy) - p0y, ez = (p0z + vz) - p0z;
  T L = std::sqrt(ex * ex + ey * ey + ez * ez);
  T axu = std::fabs(g.dx / vx), ayu = std::fabs(g.dy / vy), azu = std::fabs(g.dz / vz);
  T ax = vx > 0 ? (-rFov + (T)(imin + iinc) * g.dx - p0x) / vx
       : (vx < 0 ? (-rFov + (T)imin * g.dx - p0x) / vx : Consts<T>::big());
  T ay = vy > 0 ? (-rFov + (T)(jmin + jinc) * g.dy - p0y) / vy
       : (vy < 0 ? (-rFov + (T)jmin * g.dy - p0y) / vy : Consts<T>::big());
  T az = vz > 0 ? (offZ + (T)(kmin + kinc) * g.dz - p0z) / vz
       : (vz < 0 ? (offZ + (T)kmin * g.dz - p0z) / vz : Consts<T>::big());
  // The reference's "if (alpha < 0)" statements here have no effect (Siddon.cpp:267-286).
  T ac = amin;
  int i = imin, j = jmin, k = kmin;
  for (int m = 0; m < n; m++) {
    if (ax <= ay && ax <= az) {
      visit(i, j, k, (ax - ac) * L); i += iinc; ac = ax; ax += axu;
    } else if (ay <= ax && ay <= az) {
      visit(i, j, k, (ay - ac) * L); j += jinc; ac = ay; ay += ayu;
    } else {
      visit(i, j, k, (az - ac) * L); k += kinc; ac = az; az += azu;
    }
  }
  return n;
}

template <typename T, typename V>
int siddon2d(T p0x, T p0y, T vx, T vy, const ImgG<T>& g, T factor, V&& visit) {
  const T rFov = g.rfov;
  T amin, amax;
  if (vx == 0) {
    T a1 = (-rFov - p0y) / vy, a2 = (rFov - p0y) / vy;
    if (a1 < a2) { amin = a1; amax = a2; } else { amin = a2; amax = a1; }
  } else if (vy == 0) {
    T a1 = (-rFov - p0x) / vx, a2 = (rFov - p0x) / vx;
    if (a1 < a2) { amin = a1; amax = a2; } else { amin = a2; amax = a1; }
  } else {
    T ax1 = (-rFov - p0x) / vx, ay1 = (-rFov - p0y) / vy;
    T ax2 = (rFov - p0x) / vx, ay2 = (rFov - p0y) / vy;
    amin = tmax(tmin(ax1, ax2), tmin(ay1, ay2));
    amax = tmin(tmax(ax1, ax2), tmax(ay1, ay2));
  }
  if (amin < 0 || amin > 1) amin = 0;
  if (amax > 1 || amax < 0) amax = 1;
  T x1 = p0x + vx * amin, y1 = p0y + vy * amin;
  T x2 = p0x + vx * amax, y2 = p0y + vy * amax;
  int imin = (int)std::floor((x1 + rFov) / g.dx), jmin = (int)std::floor((y1 + rFov) / g.dy);
  int imax = (int)std::floor((x2 + rFov) / g.dx), jmax = (int)std::floor((y2 + rFov) / g.dy);
  // Early exit when both end indices lie outside on one side (Siddon.cpp:515-519).
  if ((imin < 0 && imax < 0) || (jmin < 0 && jmax < 0) || (imin >= g.nx && imax >= g.nx) ||
      (jmin >= g.ny && jmax >= g.ny))
    return 0;
  int n = std::abs(imax - imin) + std::abs(jmax - jmin);
  int iinc = vx > 0 ? 1 : (vx < 0 ? -1 : 0);
  int jinc = vy > 0 ? 1 : (vy < 0 ? -1 : 0);
  T ex = (p0x + vx) - p0x, ey = (p0y + vy) - p0y;
  T L = std::sqrt(ex * ex + ey * ey);
  T axu = std::fabs(g.dx / vx), ayu = std::fabs(g.dy / vy);
  T ax = vx > 0 ? (-rFov + (T)(imin + iinc) * g.dx - p0x) / vx
       : (vx < 0 ? (-rFov + (T)imin * g.dx - p0x) / vx : Consts<T>::big());
  if (ax < 0) ax = amin;
  T ay = vy > 0 ? (-rFov + (T)(jmin + jinc) * g.dy - p0y) / vy
       : (vy < 0 ? (-rFov + (T)jmin * g.dy - p0y) / vy : Consts<T>::big());
  if (ay < 0) ay = amin;
  T ac = amin;
  int i = imin, j = jmin;
  for (int m = 0; m < n; m++) {
    if (ax <= ay) {
      visit(i, j, 0, ((ax - ac) * L) * factor); i += iinc; ac = ax; ax += axu;
    } else {
      visit(i, j, 0, ((ay - ac) * L) * factor); j += jinc; ac = ay; ay += ayu;
    }
  }
  return n;
}

// ---------------------------------------------------------------------------
// Sinogram geometry.
template <typename T> struct Sino2DG {
  int nProj, nR;
  T rFov, rScanner;
  std::vector<T> r, ang;  // ptrRvalues_mm, ptrAngValues_deg
};

template <typename T> Sino2DG<T> make_sino2d(int nProj, int nR, float rFov, float rScanner) {
  Sino2DG<T> s;
  s.nProj = nProj; s.nR = nR; s.rFov = (T)rFov; s.rScanner = (T)rScanner;
  T rinc = ((T)2 * s.rFov) / (T)nR;
  T phinc = (T)180 / (T)nProj;
  s.r.resize(nR); s.ang.resize(nProj);
  for (int j = 0; j < nR; j++) s.r[j] = rinc / 2 + (T)j * rinc - s.rFov;
  for (int i = 0; i < nProj; i++) s.ang[i] = (T)i * phinc;
  return s;
}

template <typename T> struct Lor { T p1x, p1y, p2x, p2y; };

template <typename T> inline Lor<T> lor_points(T r, T ang_deg, T rScanner) {
  T phi = ang_deg * Consts<T>::deg_to_rad();
  T aux = std::sqrt(rScanner * rScanner - r * r);
  T c = std::cos(phi);
  T s = std::sin(phi);
  Lor<T> L;
  L.p1x = r * c + s * aux; L.p1y = r * s - c * aux;
  L.p2x = r * c - s * aux; L.p2y = r * s + c * aux;
  return L;
}

template <typename T> struct Sino3DG {
  int nProj, nR, nRings, nSeg, nSinos;
  T rFov, axialFov, rScanner;
  std::vector<T> r, ang;
  std::vector<T> z1, z2;  // averaged end-point z per sinogram, before the ring-width shift
  std::vector<std::vector<T>> zl1, zl2;  // z of every ring pair of each sinogram (getAxialValue{1,2}FromList)
  T ringWidth;
};

template <typename T>
Sino3DG<T> make_sino3d(int nProj, int nR, int nRings, float rFov, float axialFov, float rScanner, int nSeg,
                       const int* minRD, const int* maxRD) {
  Sino3DG<T> s;
  s.nProj = nProj; s.nR = nR; s.nRings = nRings; s.nSeg = nSeg;
  s.rFov = (T)rFov; s.axialFov = (T)axialFov; s.rScanner = (T)rScanner;
  Sino2DG<T> base = make_sino2d<T>(nProj, nR, rFov, rScanner);
  s.r = base.r; s.ang = base.ang;
  T zinc = s.axialFov / (T)nRings;
  std::vector<T> ringz(nRings);
  for (int i = 0; i < nRings; i++) ringz[i] = zinc / 2 + (T)i * zinc;
  for (int sg = 0; sg < nSeg; sg++) {
    for (int z1 = 0; z1 < nRings * 2; z1++) {
      std::vector<T> l1, l2;
      int z1a = z1;
      for (int z2 = 0; z2 < nRings; z2++) {
        if ((z1a - z2) <= maxRD[sg] && (z1a - z2) >= minRD[sg] && z1a >= 0 && z2 >= 0 && z1a < nRings &&
            z2 < nRings) {
          l1.push_back(ringz[z1a]); l2.push_back(ringz[z2]);
        }
        z1a = z1a - 1;
      }
      if (!l1.empty()) {
        s.z1.push_back((l1.front() + l1.back()) / 2);
        s.z2.push_back((l2.front() + l2.back()) / 2);
        s.zl1.push_back(l1);
        s.zl2.push_back(l2);
      }
    }
  }
  s.nSinos = (int)s.z1.size();
  s.ringWidth = s.axialFov / (T)nRings;
  return s;
}

inline int subset_nproj(int nProj, int subset, int nsubsets) {
  if (subset < 0) return nProj;
  int n = (int)std::floor((float)nProj / (float)nsubsets);
  if ((nProj % nsubsets) > subset) n++;
  return n;
}
inline int subset_angle(int k, int subset, int nsubsets) { return subset < 0 ? k : subset + nsubsets * k; }

// End-point z of sinogram g (SiddonProjector.cpp:392-396 with one axial sample).
template <typename T> inline void sino_z(const Sino3DG<T>& s, int g, T& za, T& zb) {
  T rw = s.ringWidth, dz = rw / (T)1;
  za = s.z1[g] - rw / 2 + dz / 2 + (T)0 * dz;
  zb = s.z2[g] - rw / 2 + dz / 2 + (T)0 * dz;
}

// Rays per bin of the 3D projectors.  ns = numSamplesOnDetector, nas =
// numAxialSamplesOnDetector (SiddonProjector(int, int), SiddonProjector.cpp:28-32),
// multi = useMultipleLorsPerBin (Projector.h:54-60).
struct Sampling {
  int ns = 1, nas = 1, multi = 0;
};

// Sinogram2D::getDeltaR (data/src/Sinogram2D.cpp:172-187).
template <typename T> inline T delta_r(const Sino3DG<T>& s, int l) {
  if (l > 0 && l < s.nR - 1) return (s.r[l + 1] - s.r[l - 1]) / 2;
  if (l == 0) return s.r[1] - s.r[0];
  return s.r[s.nR - 1] - s.r[s.nR - 2];
}

// Calls f(L, za, zb) for every ray of bin (sinogram g, angle a, r l), in the
// reference's loop order: ring pair m, radial sample o, axial sample p
// (SiddonProjector.cpp:346-397).  `dab` selects DivideAndBackproject's rule for
// when the oversampled end points are used ((ns == 1 && nas == 1) fails,
// :628); Project and Backproject use them when ns != 1 (:374, :486).
// Without useMultipleLorsPerBin the end-point z is overwritten by the mean
// ring-pair z shifted to axial sample p (:390-396).
template <typename T, typename F>
void for_rays(const Sino3DG<T>& s, int g, int a, int l, const Sampling& sm, bool dab, F&& f) {
  const int numZ = sm.multi ? (int)s.zl1[g].size() : 1;
  const T rw = s.ringWidth;
  const T dzo = rw / (T)sm.nas;
  const bool over = dab ? !(sm.ns == 1 && sm.nas == 1) : (sm.ns != 1);
  for (int m = 0; m < numZ; m++)
    for (int o = 0; o < sm.ns; o++)
      for (int p = 0; p < sm.nas; p++) {
        Lor<T> L;
        T za, zb;
        if (!over) {
          // getPointsFromLor (Sinogram2DinCylindrical3Dpet.cpp:216-229)
          L = lor_points<T>(s.r[l], s.ang[a], s.rScanner);
          za = s.zl1[g][m];
          zb = s.zl2[g][m];
        } else {
          // getPointsFromOverSampledLor (:283-299)
          const T inc = delta_r(s, l);
          const T dZ = rw / (T)sm.nas;
          const T r = s.r[l] - (inc / 2) + inc / (T)sm.ns * (T)o + (inc / (T)(2 * sm.ns));
          L = lor_points<T>(r, s.ang[a], s.rScanner);
          za = s.zl1[g][m] - rw / 2 + dZ / 2 + (T)p * dZ;
          zb = s.zl2[g][m] - rw / 2 + dZ / 2 + (T)p * dZ;
        }
        if (!sm.multi) {
          za = s.z1[g] - rw / 2 + dzo / 2 + (T)p * dzo;
          zb = s.z2[g] - rw / 2 + dzo / 2 + (T)p * dzo;
        }
        f(L, za, zb);
      }
}

inline bool inb(const int i, const int j, const int k, int nx, int ny, int nz) {
  return i >= 0 && j >= 0 && k >= 0 && i < nx && j < ny && k < nz;
}

// ---------------------------------------------------------------------------
// 3D projector.  Bins are laid out [sinogram][subset angle][r].
// Each bin accumulates the gathers of all its rays into one sum, in ray order
// (incrementSinogramBin on a zero-filled bin, SiddonProjector.cpp:339,419-420).
template <typename T>
void project3d(const Sino3DG<T>& s, int subset, int nsub, const ImgG<T>& g, const T* img, T* out, int threads,
               const Sampling& sm = Sampling()) {
  const int nk = subset_nproj(s.nProj, subset, nsub);
  const long per = (long)nk * s.nR;
  const long total = per * s.nSinos;
  #pragma omp parallel for schedule(dynamic, 256) num_threads(threads)
  for (long b = 0; b < total; b++) {
    int gsino = (int)(b / per);
    int k = (int)((b % per) / s.nR), l = (int)(b % s.nR);
    int a = subset_angle(k, subset, nsub);
    T acc = 0;
    for_rays(s, gsino, a, l, sm, false, [&](const Lor<T>& L, T za, T zb) {
      siddon3d<T>(L.p1x, L.p1y, za, L.p2x - L.p1x, L.p2y - L.p1y, zb - za, g, [&](int i, int j, int kk, T w) {
        if (inb(i, j, kk, g.nx, g.ny, g.nz)) acc += w * (T)1 * img[((long)kk * g.ny + j) * g.nx + i];
      });
    });
    out[b] = acc;
  }
}

// mode 0: Backproject (skip zero bins, value = w * bin)
// mode 1: DivideAndBackproject (in != 0: est != 0 ? w*in/est : w*in)
template <typename T>
void backproject3d(const Sino3DG<T>& s, int subset, int nsub, const ImgG<T>& g, const T* vin, const T* vest,
                   T* img, int threads, int mode, const Sampling& sm = Sampling()) {
  const int nk = subset_nproj(s.nProj, subset, nsub);
  const long per = (long)nk * s.nR;
  const long total = per * s.nSinos;
  const long nvox = (long)g.nx * g.ny * g.nz;
  if (threads < 1) threads = 1;
  std::vector<std::vector<T>> part(threads > 1 ? threads : 0);
  #pragma omp parallel num_threads(threads)
  {
    int t = omp_get_thread_num();
    T* dst = img;
    if (threads > 1) { part[t].assign(nvox, (T)0); dst = part[t].data(); }
    long lo = total * t / threads, hi = total * (t + 1) / threads;
    for (long b = lo; b < hi; b++) {
      T m = vin[b];
      if (m == 0) continue;
      T est = mode == 1 ? vest[b] : (T)0;
      int gsino = (int)(b / per);
      int k = (int)((b % per) / s.nR), l = (int)(b % s.nR);
      int a = subset_angle(k, subset, nsub);
      for_rays(s, gsino, a, l, sm, mode == 1, [&](const Lor<T>& L, T za, T zb) {
        siddon3d<T>(L.p1x, L.p1y, za, L.p2x - L.p1x, L.p2y - L.p1y, zb - za, g, [&](int i, int j, int kk, T w) {
          if (!inb(i, j, kk, g.nx, g.ny, g.nz)) return;
          T v;
          if (mode == 0) v = w * (T)1 * m;
          else v = est != 0 ? w * (T)1 * m / est : w * (T)1 * m;
          dst[((long)kk * g.ny + j) * g.nx + i] += v;
        });
      });
    }
  }
  if (threads > 1)
    for (int t = 0; t < threads; t++)
      for (long v = 0; v < nvox; v++) img[v] += part[t][v];
}

// Backproject (mode 0) with the float walk and float contributions w * 1 * m
// of backproject3d<float>, summed in double: the exact sum, to double
// rounding, of the very values the float backprojection adds (so that the
// error of a float accumulation can be told apart from the geometry's).
void backproject3d_f32_acc64(const Sino3DG<float>& s, int subset, int nsub, const ImgG<float>& g, const float* vin,
                             double* img, int threads) {
  const int nk = subset_nproj(s.nProj, subset, nsub);
  const long per = (long)nk * s.nR;
  const long total = per * s.nSinos;
  const long nvox = (long)g.nx * g.ny * g.nz;
  if (threads < 1) threads = 1;
  std::vector<std::vector<double>> part(threads);
  #pragma omp parallel num_threads(threads)
  {
    const int t = omp_get_thread_num();
    part[t].assign(nvox, 0.0);
    double* dst = part[t].data();
    const long lo = total * t / threads, hi = total * (t + 1) / threads;
    for (long b = lo; b < hi; b++) {
      const float m = vin[b];
      if (m == 0) continue;
      const int gsino = (int)(b / per);
      const int k = (int)((b % per) / s.nR), l = (int)(b % s.nR);
      const int a = subset_angle(k, subset, nsub);
      for_rays(s, gsino, a, l, Sampling(), false, [&](const Lor<float>& L, float za, float zb) {
        siddon3d<float>(L.p1x, L.p1y, za, L.p2x - L.p1x, L.p2y - L.p1y, zb - za, g, [&](int i, int j, int kk, float w) {
          if (!inb(i, j, kk, g.nx, g.ny, g.nz)) return;
          const float v = w * 1.0f * m;
          dst[((long)kk * g.ny + j) * g.nx + i] += (double)v;
        });
      });
    }
  }
  for (int t = 0; t < threads; t++)
    for (long v = 0; v < nvox; v++) img[v] += part[t][v];
}

// ---------------------------------------------------------------------------
// 2D projector.  Bins [angle][r].
template <typename T>
void project2d(const Sino2DG<T>& s, const ImgG<T>& g, const T* img, T* out, int threads) {
  const long total = (long)s.nProj * s.nR;
  #pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
  for (long b = 0; b < total; b++) {
    int a = (int)(b / s.nR), l = (int)(b % s.nR);
    if (s.r[l] > s.rFov) continue;  // bin left as it was
    Lor<T> L = lor_points<T>(s.r[l], s.ang[a], s.rScanner);
    T acc = 0;
    siddon2d<T>(L.p1x, L.p1y, L.p2x - L.p1x, L.p2y - L.p1y, g, (T)1, [&](int i, int j, int, T w) {
      if (inb(i, j, 0, g.nx, g.ny, 1)) acc += (T)1 * w * img[(long)j * g.nx + i];
    });
    out[b] = acc;
  }
}

// mode 0: Backproject (every bin, value = w * bin * 1)
// mode 1: DivideAndBackproject (only est != 0 and in != 0: 1 * w * in / est)
template <typename T>
void backproject2d(const Sino2DG<T>& s, const ImgG<T>& g, const T* vin, const T* vest, T* img, int threads,
                   int mode) {
  const long total = (long)s.nProj * s.nR;
  const long nvox = (long)g.nx * g.ny;
  if (threads < 1) threads = 1;
  std::vector<std::vector<T>> part(threads > 1 ? threads : 0);
  #pragma omp parallel num_threads(threads)
  {
    int t = omp_get_thread_num();
    T* dst = img;
    if (threads > 1) { part[t].assign(nvox, (T)0); dst = part[t].data(); }
    long lo = total * t / threads, hi = total * (t + 1) / threads;
    for (long b = lo; b < hi; b++) {
      int a = (int)(b / s.nR), l = (int)(b % s.nR);
      T m = vin[b];
      T est = mode == 1 ? vest[b] : (T)0;
      if (mode == 1 && !(est != 0 && m != 0)) continue;
      if (s.r[l] > s.rFov) continue;
      Lor<T> L = lor_points<T>(s.r[l], s.ang[a], s.rScanner);
      siddon2d<T>(L.p1x, L.p1y, L.p2x - L.p1x, L.p2y - L.p1y, g, (T)1, [&](int i, int j, int, T w) {
        if (!inb(i, j, 0, g.nx, g.ny, 1)) return;
        T v = mode == 0 ? w * m * (T)1 : (T)1 * w * m / est;
        dst[(long)j * g.nx + i] += v;
      });
    }
  }
  if (threads > 1)
    for (int t = 0; t < threads; t++)
      for (long v = 0; v < nvox; v++) img[v] += part[t][v];
}

// ---------------------------------------------------------------------------
// Bin-wise and pixel-wise steps.
template <typename T> void inverse_divide(long n, const T* meas, T* est) {
  for (long b = 0; b < n; b++) {
    T num = meas[b], den = est[b];
    est[b] = (num != 0 && den != 0) ? num / den : (T)0;
  }
}

// 3D: e != 0 ; 2D: e > 0.  Accumulated in T, serially, as the reference does.
template <typename T> T likelihood(long n, const T* est, const T* meas, bool gt0) {
  T lik = 0;
  for (long b = 0; b < n; b++) {
    T e = est[b];
    if (gt0 ? (e > 0) : (e != 0)) lik += meas[b] * std::log(e) - e;
  }
  return lik;
}

// Minimum over non-zero pixels (data/src/Images.cpp:397-419).
template <typename T> T min_nonzero(long n, const T* v) {
  T mn = Consts<T>::big();
  for (long i = 0; i < n; i++) {
    if (v[i] != 0 && mn != 0) { if (v[i] < mn) mn = v[i]; }
    else if (v[i] != 0) mn = v[0];
  }
  return mn;
}
template <typename T> T max_value(long n, const T* v) {
  T mx = v[0];
  for (long i = 0; i < n; i++) if (v[i] > mx) mx = v[i];
  return mx;
}
template <typename T> T mlem_threshold(long n, const T* sens) {
  T mn = min_nonzero(n, sens), mx = max_value(n, sens);
  return mn + (mx - mn) * (T)0.0001f;
}

template <typename T> void update(long n, T* x, const T* bp, const T* sens, T thr, bool ge) {
  for (long k = 0; k < n; k++) {
    bool ok = ge ? (sens[k] >= thr) : (sens[k] > thr);
    x[k] = ok ? x[k] * bp[k] / sens[k] : (T)0;
  }
}

// ---------------------------------------------------------------------------
template <typename T>
int mlem2d(int nx, int ny, float dx, float dy, const T* init, int nProj, int nR, float rFov, float rScanner,
           const T* meas, const T* mult, const T* add, int iters, T* out_img, T* out_lik, T* out_sens,
           int threads) {
  ImgG<T> g = make_img<T>(nx, ny, 1, dx, dy, 1.0f);
  Sino2DG<T> s = make_sino2d<T>(nProj, nR, rFov, rScanner);
  long nb = (long)nProj * nR, nv = (long)nx * ny;
  std::vector<T> sens(nv, 0), x(init, init + nv), bp(nv), est(nb, 0);
  if (mult) backproject2d<T>(s, g, mult, nullptr, sens.data(), threads, 0);
  else { std::vector<T> ones(nb, 1); backproject2d<T>(s, g, ones.data(), nullptr, sens.data(), threads, 0); }
  T thr = mlem_threshold<T>(nv, sens.data());
  for (int t = 0; t < iters; t++) {
    project2d<T>(s, g, x.data(), est.data(), threads);
    if (add) for (long b = 0; b < nb; b++) est[b] = est[b] + add[b];
    if (out_lik) out_lik[t] = likelihood<T>(nb, est.data(), meas, true);
    std::fill(bp.begin(), bp.end(), (T)0);
    inverse_divide<T>(nb, meas, est.data());
    backproject2d<T>(s, g, est.data(), nullptr, bp.data(), threads, 0);
    update<T>(nv, x.data(), bp.data(), sens.data(), thr, false);
  }
  // Mlem2d.cpp:228 evaluates the final likelihood on the ratio sinogram left in
  // the estimate buffer; kept as is.
  if (out_lik) out_lik[iters] = likelihood<T>(nb, est.data(), meas, true);
  memcpy(out_img, x.data(), sizeof(T) * nv);
  if (out_sens) memcpy(out_sens, sens.data(), sizeof(T) * nv);
  return 0;
}

template <typename T>
void gather_subset(const Sino3DG<T>& s, int subset, int nsub, const T* full, T* sub) {
  int nk = subset_nproj(s.nProj, subset, nsub);
  for (int gsino = 0; gsino < s.nSinos; gsino++)
    for (int k = 0; k < nk; k++) {
      int a = subset_angle(k, subset, nsub);
      memcpy(sub + ((long)gsino * nk + k) * s.nR, full + ((long)gsino * s.nProj + a) * s.nR, sizeof(T) * s.nR);
    }
}

template <typename T>
int osem3d(const Sino3DG<T>& s, const ImgG<T>& g, const T* init, const T* meas, const T* mult, const T* add,
           int iters, int nsub, T* out_img, T* out_lik, T* out_sens0, int threads, bool ge = true) {
  long nv = (long)g.nx * g.ny * g.nz;
  std::vector<std::vector<T>> sens(nsub, std::vector<T>(nv, 0));
  long maxb = (long)subset_nproj(s.nProj, 0, nsub) * s.nR * s.nSinos;
  std::vector<T> a(maxb), m(maxb), est(maxb), ad(maxb), x(init, init + nv), bp(nv);
  for (int sb = 0; sb < nsub; sb++) {
    long nb = (long)subset_nproj(s.nProj, sb, nsub) * s.nR * s.nSinos;
    if (mult) gather_subset<T>(s, sb, nsub, mult, a.data());
    else std::fill(a.begin(), a.begin() + nb, (T)1);
    backproject3d<T>(s, sb, nsub, g, a.data(), nullptr, sens[sb].data(), threads, 0);
    for (long v = 0; v < nv; v++) if (sens[sb][v] < 0) sens[sb][v] = 0;  // forcePositive
  }
  for (int t = 0; t < iters; t++) {
    for (int sb = 0; sb < nsub; sb++) {
      long nb = (long)subset_nproj(s.nProj, sb, nsub) * s.nR * s.nSinos;
      gather_subset<T>(s, sb, nsub, meas, m.data());
      project3d<T>(s, sb, nsub, g, x.data(), est.data(), threads);
      if (add) { gather_subset<T>(s, sb, nsub, add, ad.data()); for (long b = 0; b < nb; b++) est[b] = est[b] + ad[b]; }
      if (out_lik) out_lik[nsub * t + sb] = likelihood<T>(nb, est.data(), m.data(), false);
      std::fill(bp.begin(), bp.end(), (T)0);
      inverse_divide<T>(nb, m.data(), est.data());
      backproject3d<T>(s, sb, nsub, g, est.data(), nullptr, bp.data(), threads, 0);
      update<T>(nv, x.data(), bp.data(), sens[sb].data(), (T)0, ge);
    }
  }
  if (out_lik) {
    long nb = (long)s.nProj * s.nR * s.nSinos;
    std::vector<T> full(nb);
    project3d<T>(s, -1, 1, g, x.data(), full.data(), threads);
    out_lik[iters * nsub] = likelihood<T>(nb, full.data(), meas, false);
  }
  memcpy(out_img, x.data(), sizeof(T) * nv);
  if (out_sens0) memcpy(out_sens0, sens[0].data(), sizeof(T) * nv);
  return 0;
}

// 3D projector and backprojector over given geometry tables (any scanner):
// lor = [nProj][nR] (p1x, p1y, p2x, p2y), z = [nSinos] (z1, z2), the end
// points SiddonProjector::Project / Backproject hand to Siddon() (:392-400,
// :500-520); loops as project3d / backproject3d (mode 0).
template <typename T>
void project3d_tab(int nSinos, int nProj, int nR, const float* lor, const float* z, int subset, int nsub,
                   const ImgG<T>& g, const T* img, T* out, int threads) {
  const int nk = subset_nproj(nProj, subset, nsub);
  const long per = (long)nk * nR, total = per * nSinos;
  #pragma omp parallel for schedule(dynamic, 256) num_threads(threads)
  for (long b = 0; b < total; b++) {
    const int gs = (int)(b / per), k = (int)((b % per) / nR), l = (int)(b % nR);
    const float* L = lor + ((long)subset_angle(k, subset, nsub) * nR + l) * 4;
    const T za = (T)z[2 * gs], zb = (T)z[2 * gs + 1];
    T acc = 0;
    siddon3d<T>((T)L[0], (T)L[1], za, (T)L[2] - (T)L[0], (T)L[3] - (T)L[1], zb - za, g, [&](int i, int j, int kk, T w) {
      if (inb(i, j, kk, g.nx, g.ny, g.nz)) acc += w * (T)1 * img[((long)kk * g.ny + j) * g.nx + i];
    });
    out[b] = acc;
  }
}

template <typename T>
void backproject3d_tab(int nSinos, int nProj, int nR, const float* lor, const float* z, int subset, int nsub,
                       const ImgG<T>& g, const T* vin, T* img) {
  const int nk = subset_nproj(nProj, subset, nsub);
  const long per = (long)nk * nR, total = per * nSinos;
  for (long b = 0; b < total; b++) {
    const T m = vin[b];
    if (m == 0) continue;
    const int gs = (int)(b / per), k = (int)((b % per) / nR), l = (int)(b % nR);
    const float* L = lor + ((long)subset_angle(k, subset, nsub) * nR + l) * 4;
    const T za = (T)z[2 * gs], zb = (T)z[2 * gs + 1];
    siddon3d<T>((T)L[0], (T)L[1], za, (T)L[2] - (T)L[0], (T)L[3] - (T)L[1], zb - za, g, [&](int i, int j, int kk, T w) {
      if (inb(i, j, kk, g.nx, g.ny, g.nz)) img[((long)kk * g.ny + j) * g.nx + i] += w * (T)1 * m;
    });
  }
}

struct S3 {
  int nProj, nR, nRings, nSeg;
  float rFov, axialFov, rScanner;
  const int* minRD;
  const int* maxRD;
};

template <typename T> Sino3DG<T> mk(const S3* d) {
  return make_sino3d<T>(d->nProj, d->nR, d->nRings, d->rFov, d->axialFov, d->rScanner, d->nSeg, d->minRD, d->maxRD);
}

}  // namespace

extern "C" {

// Layout of the 3D sinogram description passed from Python (ctypes).
typedef S3 or_sino3d;

int or_lor_points_2d(int nProj, int nR, float rFov, float rScanner, float* out4) {
  Sino2DG<float> s = make_sino2d<float>(nProj, nR, rFov, rScanner);
  for (int a = 0; a < nProj; a++)
    for (int l = 0; l < nR; l++) {
      Lor<float> L = lor_points<float>(s.r[l], s.ang[a], s.rScanner);
      float* o = out4 + ((long)a * nR + l) * 4;
      o[0] = L.p1x; o[1] = L.p1y; o[2] = L.p2x; o[3] = L.p2y;
    }
  return 0;
}

int or_sino3d_z(const or_sino3d* d, float* z1, float* z2) {
  Sino3DG<float> s = mk<float>(d);
  for (int g = 0; g < s.nSinos; g++) sino_z(s, g, z1[g], z2[g]);
  return s.nSinos;
}

// Siddon segment list of one 3D LOR (testing the walk itself).  Returns the
// number of recorded segments, writes at most cap of them.
int or_siddon3d_f32(float p1x, float p1y, float p1z, float p2x, float p2y, float p2z, int nx, int ny, int nz,
                    float dx, float dy, float dz, int* ijk, float* w, int cap) {
  ImgG<float> g = make_img<float>(nx, ny, nz, dx, dy, dz);
  int c = 0;
  int n = siddon3d<float>(p1x, p1y, p1z, p2x - p1x, p2y - p1y, p2z - p1z, g, [&](int i, int j, int k, float ww) {
    if (c < cap) { ijk[3 * c] = i; ijk[3 * c + 1] = j; ijk[3 * c + 2] = k; w[c] = ww; }
    c++;
  });
  return n;
}

int or_siddon3d_f64(double p1x, double p1y, double p1z, double p2x, double p2y, double p2z, int nx, int ny, int nz,
                    float dx, float dy, float dz, int* ijk, double* w, int cap) {
  ImgG<double> g = make_img<double>(nx, ny, nz, dx, dy, dz);
  int c = 0;
  int n = siddon3d<double>(p1x, p1y, p1z, p2x - p1x, p2y - p1y, p2z - p1z, g, [&](int i, int j, int k, double ww) {
    if (c < cap) { ijk[3 * c] = i; ijk[3 * c + 1] = j; ijk[3 * c + 2] = k; w[c] = ww; }
    c++;
  });
  return n;
}

int or_lor_points_2d_f64(int nProj, int nR, float rFov, float rScanner, double* out4) {
  Sino2DG<double> s = make_sino2d<double>(nProj, nR, rFov, rScanner);
  for (int a = 0; a < nProj; a++)
    for (int l = 0; l < nR; l++) {
      Lor<double> L = lor_points<double>(s.r[l], s.ang[a], s.rScanner);
      double* o = out4 + ((long)a * nR + l) * 4;
      o[0] = L.p1x; o[1] = L.p1y; o[2] = L.p2x; o[3] = L.p2y;
    }
  return 0;
}

int or_sino3d_z_f64(const or_sino3d* d, double* z1, double* z2) {
  Sino3DG<double> s = mk<double>(d);
  for (int g = 0; g < s.nSinos; g++) sino_z(s, g, z1[g], z2[g]);
  return s.nSinos;
}

#define OR_FWD3(SUF, T)                                                                                      \
  int or_project_3d_##SUF(const or_sino3d* d, int subset, int nsub, int nx, int ny, int nz, float dx,       \
                          float dy, float dz, const T* img, T* out, int threads) {                          \
    Sino3DG<T> s = mk<T>(d);                                                                                 \
    project3d<T>(s, subset, nsub, make_img<T>(nx, ny, nz, dx, dy, dz), img, out, threads);                   \
    return 0;                                                                                                \
  }                                                                                                          \
  int or_backproject_3d_##SUF(const or_sino3d* d, int subset, int nsub, int nx, int ny, int nz, float dx,   \
                              float dy, float dz, const T* vin, T* img, int threads) {                      \
    Sino3DG<T> s = mk<T>(d);                                                                                 \
    backproject3d<T>(s, subset, nsub, make_img<T>(nx, ny, nz, dx, dy, dz), vin, nullptr, img, threads, 0);   \
    return 0;                                                                                                \
  }                                                                                                          \
  int or_divide_and_backproject_3d_##SUF(const or_sino3d* d, int subset, int nsub, int nx, int ny, int nz,  \
                                         float dx, float dy, float dz, const T* vin, const T* vest, T* img, \
                                         int threads) {                                                     \
    Sino3DG<T> s = mk<T>(d);                                                                                 \
    backproject3d<T>(s, subset, nsub, make_img<T>(nx, ny, nz, dx, dy, dz), vin, vest, img, threads, 1);      \
    return 0;                                                                                                \
  }                                                                                                          \
  int or_project_2d_##SUF(int nx, int ny, float dx, float dy, const T* img, int nProj, int nR, float rFov,  \
                          float rScanner, T* out, int threads) {                                            \
    project2d<T>(make_sino2d<T>(nProj, nR, rFov, rScanner), make_img<T>(nx, ny, 1, dx, dy, 1.0f), img, out,  \
                 threads);                                                                                   \
    return 0;                                                                                                \
  }                                                                                                          \
  int or_backproject_2d_##SUF(int nx, int ny, float dx, float dy, T* img, int nProj, int nR, float rFov,    \
                              float rScanner, const T* vin, int threads) {                                  \
    backproject2d<T>(make_sino2d<T>(nProj, nR, rFov, rScanner), make_img<T>(nx, ny, 1, dx, dy, 1.0f), vin,   \
                     nullptr, img, threads, 0);                                                              \
    return 0;                                                                                                \
  }                                                                                                          \
  int or_divide_and_backproject_2d_##SUF(int nx, int ny, float dx, float dy, T* img, int nProj, int nR,     \
                                         float rFov, float rScanner, const T* vin, const T* vest,           \
                                         int threads) {                                                     \
    backproject2d<T>(make_sino2d<T>(nProj, nR, rFov, rScanner), make_img<T>(nx, ny, 1, dx, dy, 1.0f), vin,   \
                     vest, img, threads, 1);                                                                 \
    return 0;                                                                                                \
  }                                                                                                          \
  int or_mlem_2d_##SUF(int nx, int ny, float dx, float dy, const T* init, int nProj, int nR, float rFov,    \
                       float rScanner, const T* meas, const T* mult, const T* add, int iters, T* out_img,    \
                       T* out_lik, T* out_sens, int threads) {                                              \
    return mlem2d<T>(nx, ny, dx, dy, init, nProj, nR, rFov, rScanner, meas, mult, add, iters, out_img,       \
                     out_lik, out_sens, threads);                                                            \
  }                                                                                                          \
  int or_osem_3d_##SUF(const or_sino3d* d, int nx, int ny, int nz, float dx, float dy, float dz,            \
                       const T* init, const T* meas, const T* mult, const T* add, int iters, int nsub,      \
                       T* out_img, T* out_lik, T* out_sens0, int threads) {                                 \
    Sino3DG<T> s = mk<T>(d);                                                                                 \
    return osem3d<T>(s, make_img<T>(nx, ny, nz, dx, dy, dz), init, meas, mult, add, iters, nsub, out_img,    \
                     out_lik, out_sens0, threads);                                                           \
  }                                                                                                          \
  /* ge = 0: the update x * bp / sens only where sens > 0 (else 0) instead of    \
     the reference's sens >= 0 (OsemSinogram3d.cpp:217-237).  */                \
  int or_osem_3d_rule_##SUF(const or_sino3d* d, int nx, int ny, int nz, float dx, float dy, float dz,       \
                            const T* init, const T* meas, const T* mult, const T* add, int iters, int nsub, \
                            T* out_img, T* out_lik, T* out_sens0, int threads, int ge) {                   \
    Sino3DG<T> s = mk<T>(d);                                                                                 \
    return osem3d<T>(s, make_img<T>(nx, ny, nz, dx, dy, dz), init, meas, mult, add, iters, nsub, out_img,    \
                     out_lik, out_sens0, threads, ge != 0);                                                  \
  }                                                                                                          \
  T or_likelihood_##SUF(long n, const T* est, const T* meas, int gt0) {                                      \
    return likelihood<T>(n, est, meas, gt0 != 0);                                                            \
  }                                                                                                          \
  void or_inverse_divide_##SUF(long n, const T* meas, T* est) { inverse_divide<T>(n, meas, est); }           \
  T or_mlem_threshold_##SUF(long n, const T* sens) { return mlem_threshold<T>(n, sens); }                    \
  void or_update_##SUF(long n, T* x, const T* bp, const T* sens, T thr, int ge) {                            \
    update<T>(n, x, bp, sens, thr, ge != 0);                                                                 \
  }

OR_FWD3(f32, float)
OR_FWD3(f64, double)

int or_backproject_3d_f32_acc64(const or_sino3d* d, int subset, int nsub, int nx, int ny, int nz, float dx,
                                float dy, float dz, const float* vin, double* img, int threads) {
  backproject3d_f32_acc64(mk<float>(d), subset, nsub, make_img<float>(nx, ny, nz, dx, dy, dz), vin, img, threads);
  return 0;
}

int or_project_3d_tables_f32(int nSinos, int nProj, int nR, const float* lor, const float* z, int subset, int nsub,
                             int nx, int ny, int nz, float dx, float dy, float dz, const float* img, float* out,
                             int threads) {
  project3d_tab<float>(nSinos, nProj, nR, lor, z, subset, nsub, make_img<float>(nx, ny, nz, dx, dy, dz), img, out,
                       threads);
  return 0;
}

// Serial, in bin order (the reference's order with one thread).
int or_backproject_3d_tables_f32(int nSinos, int nProj, int nR, const float* lor, const float* z, int subset,
                                 int nsub, int nx, int ny, int nz, float dx, float dy, float dz, const float* vin,
                                 float* img) {
  backproject3d_tab<float>(nSinos, nProj, nR, lor, z, subset, nsub, make_img<float>(nx, ny, nz, dx, dy, dz), vin,
                           img);
  return 0;
}

// Sampled-LOR projectors: ns radial and nas axial samples per bin, multi =
// one ray per ring pair of the bin (useMultipleLorsPerBin).  mode 0 =
// Project, 1 = Backproject, 2 = DivideAndBackproject (vest used).
#define OR_SAMPLED3(SUF, T)                                                                                  \
  int or_sampled_3d_##SUF(const or_sino3d* d, int ns, int nas, int multi, int mode, int subset, int nsub,   \
                          int nx, int ny, int nz, float dx, float dy, float dz, const T* in, const T* vest, \
                          T* out, int threads) {                                                            \
    if (ns < 1 || nas < 1 || d->nR < 2) return -1;                                                           \
    Sino3DG<T> s = mk<T>(d);                                                                                 \
    Sampling sm;                                                                                             \
    sm.ns = ns; sm.nas = nas; sm.multi = multi != 0;                                                         \
    ImgG<T> g = make_img<T>(nx, ny, nz, dx, dy, dz);                                                         \
    if (mode == 0) project3d<T>(s, subset, nsub, g, in, out, threads, sm);                                   \
    else backproject3d<T>(s, subset, nsub, g, in, mode == 2 ? vest : nullptr, out, threads, mode == 2 ? 1 : 0, sm); \
    return 0;                                                                                                \
  }
OR_SAMPLED3(f32, float)
OR_SAMPLED3(f64, double)

// Number of recorded Siddon segments per bin of a 3D subset (the step count
// used for the Gsteps/s figure).
long or_count_steps_3d(const or_sino3d* d, int subset, int nsub, int nx, int ny, int nz, float dx, float dy,
                       float dz, int threads) {
  Sino3DG<float> s = mk<float>(d);
  ImgG<float> g = make_img<float>(nx, ny, nz, dx, dy, dz);
  const int nk = subset_nproj(s.nProj, subset, nsub);
  const long per = (long)nk * s.nR, total = per * s.nSinos;
  long steps = 0;
  #pragma omp parallel for schedule(dynamic, 256) num_threads(threads) reduction(+ : steps)
  for (long b = 0; b < total; b++) {
    int gsino = (int)(b / per);
    int k = (int)((b % per) / s.nR), l = (int)(b % s.nR);
    Lor<float> L = lor_points<float>(s.r[l], s.ang[subset_angle(k, subset, nsub)], s.rScanner);
    float za, zb; sino_z(s, gsino, za, zb);
    steps += siddon3d<float>(L.p1x, L.p1y, za, L.p2x - L.p1x, L.p2y - L.p1y, zb - za, g, [](int, int, int, float) {});
  }
  return steps;
}

}  // extern "C"
