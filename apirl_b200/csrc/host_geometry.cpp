// Host-side geometry tables, computed once per projector with the reference's
// own float expressions so that the device walk sees bit-identical LOR end
// points (no device transcendental enters a result):
//   r_j   = RInc/2 + j*RInc - rFov, RInc = (2*rFov)/nR
//   phi_i = i * (180/nProj) degrees     (Sinogram2DinCylindrical3Dpet.cpp:46-63)
//   P1 = (r cos + sin aux, r sin - cos aux), P2 = (r cos - sin aux, r sin + cos aux),
//   aux = sqrt(R^2 - r^2)               (Sinogram2DinCylindrical3Dpet.cpp:216-266)
//   ring z_i = zInc/2 + i*zInc, zInc = axialFov/nRings, ring pairs per segment,
//   end-point z = mean of the first and last pair (Sinogram3D.cpp:358-464,
//   SiddonProjector.cpp:357-360, :392-396).
// Built with g++ -O2 -ffp-contract=off, like the reference's own CPU build.
#include <cmath>
#include <vector>
#include "internal.h"

namespace apirl {

namespace {
const float kDegToRad = 0.01745329251994329576f;  // DEG_TO_RAD, utils/inc/Geometry.h:10

void r_and_angles(int n_proj, int n_r, float r_fov, std::vector<float>& r, std::vector<float>& ang) {
  const float rinc = (2 * r_fov) / (float)n_r;
  const float phinc = (float)180 / (float)n_proj;
  r.resize(n_r);
  ang.resize(n_proj);
  for (int j = 0; j < n_r; j++) r[j] = rinc / 2 + (float)j * rinc - r_fov;
  for (int i = 0; i < n_proj; i++) ang[i] = (float)i * phinc;
}

void lor_table(int n_proj, int n_r, float r_scanner, const std::vector<float>& r, const std::vector<float>& ang,
               std::vector<float>& lor) {
  lor.resize((size_t)n_proj * n_r * 4);
  for (int a = 0; a < n_proj; a++) {
    const float phi = ang[a] * kDegToRad;
    const float c = std::cos(phi);
    const float s = std::sin(phi);
    for (int l = 0; l < n_r; l++) {
      const float rv = r[l];
      const float aux = std::sqrt(r_scanner * r_scanner - rv * rv);
      float* o = &lor[((size_t)a * n_r + l) * 4];
      o[0] = rv * c + s * aux;
      o[1] = rv * s - c * aux;
      o[2] = rv * c - s * aux;
      o[3] = rv * s + c * aux;
    }
  }
}
}  // namespace

ImgGeom make_img_geom(int nx, int ny, int nz, float dx, float dy, float dz) {
  ImgGeom g;
  g.nx = nx; g.ny = ny; g.nz = nz;
  g.dx = dx; g.dy = dy; g.dz = dz;
  g.rfov = (dx * (float)nx) / 2;
  g.offz = dz / 2;
  return g;
}

int subset_nproj(int n_proj, int subset, int nsub) {
  if (subset < 0) return n_proj;
  int n = (int)std::floor((float)n_proj / (float)nsub);
  if ((n_proj % nsub) > subset) n++;
  return n;
}

void build_tables_2d(int n_proj, int n_r, float r_fov, float r_scanner, HostTables& t) {
  std::vector<float> r, ang;
  r_and_angles(n_proj, n_r, r_fov, r, ang);
  lor_table(n_proj, n_r, r_scanner, r, ang, t.lor);
  t.ok.resize(n_r);
  for (int l = 0; l < n_r; l++) t.ok[l] = (r[l] > r_fov) ? 0 : 1;
  t.z.assign(2, 0.f);
  t.n_sinos = 1;
}

bool build_tables_3d(int n_proj, int n_r, int n_rings, float r_fov, float axial_fov, float r_scanner, int n_seg,
                     const int* min_rd, const int* max_rd, HostTables& t) {
  std::vector<float> r, ang;
  r_and_angles(n_proj, n_r, r_fov, r, ang);
  lor_table(n_proj, n_r, r_scanner, r, ang, t.lor);
  t.ok.assign(n_r, 1);
  const float zinc = axial_fov / (float)n_rings;
  std::vector<float> ringz(n_rings);
  for (int i = 0; i < n_rings; i++) ringz[i] = zinc / 2 + (float)i * zinc;
  const float rw = axial_fov / (float)n_rings;
  const float dz = rw / (float)1;
  t.z.clear();
  for (int sg = 0; sg < n_seg; sg++) {
    for (int z1 = 0; z1 < 2 * n_rings; z1++) {
      int cnt = 0;
      float f1 = 0, l1 = 0, f2 = 0, l2 = 0;
      int z1a = z1;
      for (int z2 = 0; z2 < n_rings; z2++) {
        if ((z1a - z2) <= max_rd[sg] && (z1a - z2) >= min_rd[sg] && z1a >= 0 && z2 >= 0 && z1a < n_rings &&
            z2 < n_rings) {
          if (cnt == 0) { f1 = ringz[z1a]; f2 = ringz[z2]; }
          l1 = ringz[z1a]; l2 = ringz[z2];
          cnt++;
        }
        z1a = z1a - 1;
      }
      if (cnt > 0) {
        const float za = (f1 + l1) / 2, zb = (f2 + l2) / 2;
        t.z.push_back(za - rw / 2 + dz / 2 + (float)0 * dz);
        t.z.push_back(zb - rw / 2 + dz / 2 + (float)0 * dz);
      }
    }
  }
  t.n_sinos = (int)(t.z.size() / 2);
  return t.n_sinos > 0;
}

// Siemens Biograph mMR (data/src/Sinogram2DinSiemensMmr.cpp,
// data/src/Sinogram3DSiemensMmr.cpp): arc-corrected r values with the mean
// depth of interaction, angles i * 180 / nProj, odd r bins rotated back by
// half an angular step, end points on the effective radius R + DOI.
const float kMmrRadius = 656.0f / 2.0f;
const float kMmrRFov = 594.0f / 2.0f;
const float kMmrAxialFov = 260.0f;
const float kMmrDoi = 9.6f;
const float kMmrBin = 4.0891f / 2.0f;

void mmr_lor_table(int n_proj, int n_r, std::vector<float>& lor) {
  // Sinogram2DinSiemensMmr(nProj, nR) (:57-81): r values and angles.
  const float bin = n_r == 344 ? kMmrBin : kMmrBin * 344 / n_r;
  std::vector<float> r(n_r), ang(n_proj);
  for (int j = 0; j < n_r; j++) {
    const float lr = bin / 2 + (bin * ((float)j - (float)(n_r / 2)));
    r[j] = (kMmrRadius + kMmrDoi * std::cos(lr / kMmrRadius)) * std::sin(lr / kMmrRadius);
  }
  const float phinc = (float)180 / (float)n_proj;
  for (int i = 0; i < n_proj; i++) ang[i] = (float)i * phinc;
  // getPointsFromLor, 3D form (:174-198).
  const float step = ang[1] - ang[0];
  const float reff = kMmrRadius + kMmrDoi;  // getEffectiveRadioScanner_mm (Sinogram2DinSiemensMmr.h:105)
  lor.resize((size_t)n_proj * n_r * 4);
  for (int a = 0; a < n_proj; a++)
    for (int l = 0; l < n_r; l++) {
      const float phi = (ang[a] - (float)(l % 2) * step / 2) * kDegToRad;
      const float c = std::cos(phi), sn = std::sin(phi);
      const float rv = r[l];
      const float aux = std::sqrt(reff * reff - rv * rv);
      float* o = &lor[((size_t)a * n_r + l) * 4];
      o[0] = rv * c + sn * aux;
      o[1] = rv * sn - c * aux;
      o[2] = rv * c - sn * aux;
      o[3] = rv * sn + c * aux;
    }
}

bool build_tables_mmr(int n_proj, int n_r, int n_rings, int n_seg, const int* min_rd, const int* max_rd,
                      HostTables& t) {
  if (n_proj < 2) return false;
  // Ring pairs and end-point z as for any cylindrical scanner, with the
  // mMR's 260 mm axial field of view (ring width 260 / nRings).
  if (!build_tables_3d(n_proj, n_r, n_rings, kMmrRFov, kMmrAxialFov, kMmrRadius, n_seg, min_rd, max_rd, t))
    return false;
  mmr_lor_table(n_proj, n_r, t.lor);
  return true;
}

bool build_rays_3d(int n_proj, int n_r, int n_rings, float r_fov, float axial_fov, float r_scanner, int n_seg,
                   const int* min_rd, const int* max_rd, int ns, int nas, int multi, bool dab, RayTables& t) {
  std::vector<float> r, ang;
  r_and_angles(n_proj, n_r, r_fov, r, ang);
  // End points: getPointsFromLor, or getPointsFromOverSampledLor with the
  // radial sample o (Sinogram2DinCylindrical3Dpet.cpp:216-229, :283-299) and
  // getDeltaR (data/src/Sinogram2D.cpp:172-187).
  const bool over = dab ? !(ns == 1 && nas == 1) : (ns != 1);
  t.n_rs = ns;
  t.n_as = nas;
  t.lor.resize((size_t)n_proj * n_r * ns * 4);
  bool finite = true;
  for (int a = 0; a < n_proj; a++) {
    const float phi = ang[a] * kDegToRad;
    const float c = std::cos(phi);
    const float s = std::sin(phi);
    for (int l = 0; l < n_r; l++) {
      float inc = 0;
      if (over) {
        if (l > 0 && l < n_r - 1) inc = (r[l + 1] - r[l - 1]) / 2;
        else if (l == 0) inc = r[1] - r[0];
        else inc = r[n_r - 1] - r[n_r - 2];
      }
      for (int o = 0; o < ns; o++) {
        const float rv = over ? r[l] - (inc / 2) + inc / (float)ns * (float)o + (inc / (float)(2 * ns)) : r[l];
        const float aux = std::sqrt(r_scanner * r_scanner - rv * rv);
        float* q = &t.lor[(((size_t)a * n_r + l) * ns + o) * 4];
        q[0] = rv * c + s * aux;
        q[1] = rv * s - c * aux;
        q[2] = rv * c - s * aux;
        q[3] = rv * s + c * aux;
        finite = finite && std::isfinite(q[0]) && std::isfinite(q[1]) && std::isfinite(q[2]) && std::isfinite(q[3]);
      }
    }
  }
  // End-point z per (ring pair m, axial sample q): the pair's ring z, or with
  // oversampling that z shifted to sample q; without useMultipleLorsPerBin the
  // mean pair z shifted to sample q (SiddonProjector.cpp:357-360, :390-396).
  const float zinc = axial_fov / (float)n_rings;
  std::vector<float> ringz(n_rings);
  for (int i = 0; i < n_rings; i++) ringz[i] = zinc / 2 + (float)i * zinc;
  const float rw = axial_fov / (float)n_rings;
  const float dzo = rw / (float)nas;
  t.zs.clear();
  t.zoff.assign(1, 0);
  for (int sg = 0; sg < n_seg; sg++) {
    for (int z1 = 0; z1 < 2 * n_rings; z1++) {
      std::vector<float> l1, l2;
      int z1a = z1;
      for (int z2 = 0; z2 < n_rings; z2++) {
        if ((z1a - z2) <= max_rd[sg] && (z1a - z2) >= min_rd[sg] && z1a >= 0 && z2 >= 0 && z1a < n_rings &&
            z2 < n_rings) {
          l1.push_back(ringz[z1a]);
          l2.push_back(ringz[z2]);
        }
        z1a = z1a - 1;
      }
      if (l1.empty()) continue;
      const float m1 = (l1.front() + l1.back()) / 2, m2 = (l2.front() + l2.back()) / 2;
      const int num_z = multi ? (int)l1.size() : 1;
      for (int m = 0; m < num_z; m++)
        for (int q = 0; q < nas; q++) {
          float za, zb;
          if (!multi) {
            za = m1 - rw / 2 + dzo / 2 + (float)q * dzo;
            zb = m2 - rw / 2 + dzo / 2 + (float)q * dzo;
          } else if (!over) {
            za = l1[m];
            zb = l2[m];
          } else {
            const float dz = rw / (float)nas;
            za = l1[m] - rw / 2 + dz / 2 + (float)q * dz;
            zb = l2[m] - rw / 2 + dz / 2 + (float)q * dz;
          }
          finite = finite && std::isfinite(za) && std::isfinite(zb);
          t.zs.push_back(za);
          t.zs.push_back(zb);
        }
      t.zoff.push_back((int)(t.zs.size() / 2));
    }
  }
  return finite;
}

void build_tables_3d_f64(int n_proj, int n_r, int n_rings, float r_fov, float axial_fov, float r_scanner, int n_seg,
                         const int* min_rd, const int* max_rd, std::vector<double>& lor, std::vector<double>& z) {
  const double rf = r_fov, R = r_scanner, afov = axial_fov;
  const double rinc = (2.0 * rf) / n_r, phinc = 180.0 / n_proj;
  lor.resize((size_t)n_proj * n_r * 4);
  for (int a = 0; a < n_proj; a++) {
    const double phi = (a * phinc) * 0.017453292519943295769;
    const double c = std::cos(phi), s = std::sin(phi);
    for (int l = 0; l < n_r; l++) {
      const double rv = rinc / 2 + l * rinc - rf;
      const double aux = std::sqrt(R * R - rv * rv);
      double* o = &lor[((size_t)a * n_r + l) * 4];
      o[0] = rv * c + s * aux;
      o[1] = rv * s - c * aux;
      o[2] = rv * c - s * aux;
      o[3] = rv * s + c * aux;
    }
  }
  const double zinc = afov / n_rings;
  z.clear();
  for (int sg = 0; sg < n_seg; sg++)
    for (int z1 = 0; z1 < 2 * n_rings; z1++) {
      int cnt = 0;
      double f1 = 0, l1 = 0, f2 = 0, l2 = 0;
      int z1a = z1;
      for (int z2 = 0; z2 < n_rings; z2++, z1a--) {
        if ((z1a - z2) <= max_rd[sg] && (z1a - z2) >= min_rd[sg] && z1a >= 0 && z1a < n_rings) {
          const double za = zinc / 2 + z1a * zinc, zb = zinc / 2 + z2 * zinc;
          if (cnt == 0) { f1 = za; f2 = zb; }
          l1 = za; l2 = zb;
          cnt++;
        }
      }
      if (cnt > 0) {
        z.push_back((f1 + l1) / 2);
        z.push_back((f2 + l2) / 2);
      }
    }
}

}  // namespace apirl
