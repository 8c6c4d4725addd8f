// Test infrastructure, not product code.
//
// extern "C" harness around the reference APIRL CPU reconstruction path,
// compiled from the unmodified reference sources by oracle/ref/Makefile into
// oracle/_ref/libapirl_ref_harness.so.  Tests use it to pin the oracle
// restatement (oracle/oracle.cpp) and to make golden fixtures; bench.py uses it
// as the timed CPU baseline.
//
// What is the reference's own code and what is harness code:
//  * Siddon() (recon/src/Siddon.cpp:13-344, :358-643), SiddonProjector::Backproject
//    (recon/src/SiddonProjector.cpp:34-87, :444-568), the sinogram/image classes,
//    getSubset, inverseDivideBinToBin, getLikelihoodValue and the Mlem2d /
//    OsemSinogram3d drivers are the reference's, called unmodified.
//  * Forward projection goes through MaskedSiddonProjector below: the loops of
//    SiddonProjector::Project (recon/src/SiddonProjector.cpp:146-193 for 2D,
//    :322-441 for 3D) restated with a full bounds mask on the voxel index.  The
//    reference checks only the lower bound in 2D (:178) and only the upper bound
//    in 3D (:417), so its own Project reads outside the image for some rays
//    (undefined behaviour); the masked loop is the semantics both the oracle
//    restatement and the CUDA kernels implement.
//  * Known reference defects worked around here:
//    - Sinogram3DCylindricalPet::getSubset writes the subset angles into the
//      parent's ptrAngValues_deg (data/src/Sinogram3DCylindricalPet.cpp:187),
//      which is a 1-float buffer after construction (data/src/Sinogram2D.cpp:27-36).
//      fix_angle_buffer() grows it to numProj floats before any getSubset.
//    - Sinogram3DCylindricalPet's copy constructor builds its segments before it
//      sets radioScanner_mm (data/src/Sinogram3DCylindricalPet.cpp:67-80), so a
//      Copy() carries an uninitialised scanner radius in its 2D sinograms.  The
//      whole-sinogram projections here use getSubset(0, 1) instead, which builds
//      the same bins with the given radius.  OsemSinogram3d's final likelihood
//      (recon/src/OsemSinogram3d.cpp:291) still goes through Copy().
//    - 3D sinograms are built from an interfile header written to a scratch
//      directory (the numbered constructor leaves ptrAxialvalues_mm unset,
//      data/src/Sinogram3DCylindricalPet.cpp:56-61).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <omp.h>

#include <Images.h>
#include <Geometry.h>
#include <Siddon.h>
#include <SiddonProjector.h>
#include <Projector.h>
#include <Sinogram2D.h>
#include <Sinogram2DinCylindrical3Dpet.h>
#include <Sinogram3D.h>
#include <Sinogram3DCylindricalPet.h>
#include <Sinogram3DSiemensMmr.h>
#include <Mlem2d.h>

namespace {

// Access to Sinogram2D::ptrAngValues_deg (protected) through a derived class's
// pointer-to-member, so the reference classes stay unmodified.
struct AngAccess : public Sinogram2D {
  static float*& ang(Sinogram2D* s) { return s->*(&AngAccess::ptrAngValues_deg); }
};

void fix_angle_buffer(Sinogram3D* s) {
  float*& p = AngAccess::ang(s);
  p = (float*)realloc(p, sizeof(float) * (size_t)(s->getNumProj() > 0 ? s->getNumProj() : 1));
}

SizeImage make_size(int nx, int ny, int nz, float dx, float dy, float dz) {
  SizeImage s;
  s.nDimensions = nz > 1 ? 3 : 2;
  s.nPixelsX = nx; s.nPixelsY = ny; s.nPixelsZ = nz;
  s.sizePixelX_mm = dx; s.sizePixelY_mm = dy; s.sizePixelZ_mm = dz;
  return s;
}

Image* make_image(int nx, int ny, int nz, float dx, float dy, float dz, const float* px) {
  SizeImage s = make_size(nx, ny, nz, dx, dy, dz);
  // Image(SizeImage) only sets nPixelsZ = 1 for 2D sizes; a 3D image with one
  // slice keeps nDimensions = 2, which is what the reference does as well.
  Image* im = new Image(s);
  if (px) memcpy(im->getPixelsPtr(), px, sizeof(float) * (size_t)nx * ny * nz);
  return im;
}

// Forward projection with the reference Siddon() and a full bounds mask.
class MaskedSiddonProjector : public Projector {
 public:
  SiddonProjector* ref;
  MaskedSiddonProjector() { ref = new SiddonProjector(1, 1); }
  ~MaskedSiddonProjector() { delete ref; }

  bool Project(Image* inputImage, Sinogram2D* out) {
    SizeImage sz = inputImage->getSize();
    float* px = inputImage->getPixelsPtr();
    #pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < out->getNumProj(); i++) {
      SiddonSegment* w = NULL;
      for (int j = 0; j < out->getNumR(); j++) {
        Point2D P1, P2; Line2D LOR; float geom; int n = 0;
        if (!out->getPointsFromLor(i, j, &P1, &P2, &geom)) continue;
        LOR.P0 = P1; LOR.Vx = P2.X - P1.X; LOR.Vy = P2.Y - P1.Y;
        Siddon(LOR, inputImage, &w, &n, 1);
        out->setSinogramBin(i, j, 0);
        if (n > 0) {
          for (int l = 0; l < n; l++) {
            if (w[l].IndexX >= 0 && w[l].IndexY >= 0 && w[l].IndexX < sz.nPixelsX && w[l].IndexY < sz.nPixelsY)
              out->incrementSinogramBin(i, j, geom * w[l].Segment * px[w[l].IndexY * sz.nPixelsX + w[l].IndexX]);
          }
          free(w);
        }
      }
    }
    return true;
  }
  bool Backproject(Sinogram2D* in, Image* out) { return ref->Backproject(in, out); }
  bool DivideAndBackproject(Sinogram2D* a, Sinogram2D* b, Image* out) { return ref->DivideAndBackproject(a, b, out); }

  bool Project(Image* inputImage, Sinogram3D* out) {
    SizeImage sz = inputImage->getSize();
    float* px = inputImage->getPixelsPtr();
    float ringWidth_mm = out->getAxialFoV_mm() / out->getNumRings();
    float deltaZ = ringWidth_mm / 1;
    out->FillConstant(0.0);
    for (int i = 0; i < out->getNumSegments(); i++) {
      for (int j = 0; j < out->getSegment(i)->getNumSinograms(); j++) {
        Sinogram2DinCylindrical3Dpet* s2 = out->getSegment(i)->getSinogram2D(j);
        float z1 = (s2->getAxialValue1FromList(0) + s2->getAxialValue1FromList(s2->getNumZ() - 1)) / 2;
        float z2 = (s2->getAxialValue2FromList(0) + s2->getAxialValue2FromList(s2->getNumZ() - 1)) / 2;
        #pragma omp parallel for schedule(dynamic, 1)
        for (int k = 0; k < s2->getNumProj(); k++) {
          SiddonSegment* w = NULL;
          for (int l = 0; l < s2->getNumR(); l++) {
            Point3D P1, P2; Line3D LOR; float geom; int n = 0; int p = 0;
            int ok = s2->getPointsFromLor(k, l, 0, &P1, &P2, &geom);
            P1.Z = z1 - ringWidth_mm / 2 + deltaZ / 2 + p * deltaZ;
            P2.Z = z2 - ringWidth_mm / 2 + deltaZ / 2 + p * deltaZ;
            if (!ok) continue;
            LOR.P0 = P1; LOR.Vx = P2.X - P1.X; LOR.Vy = P2.Y - P1.Y; LOR.Vz = P2.Z - P1.Z;
            Siddon(LOR, inputImage, &w, &n, 1);
            if (n > 0) {
              for (int m = 0; m < n; m++) {
                if (w[m].IndexX >= 0 && w[m].IndexY >= 0 && w[m].IndexZ >= 0 &&
                    w[m].IndexX < sz.nPixelsX && w[m].IndexY < sz.nPixelsY && w[m].IndexZ < sz.nPixelsZ)
                  s2->incrementSinogramBin(k, l, w[m].Segment * geom *
                      px[w[m].IndexZ * (sz.nPixelsX * sz.nPixelsY) + w[m].IndexY * sz.nPixelsX + w[m].IndexX]);
              }
              free(w);
            }
          }
        }
      }
    }
    return true;
  }
  bool Backproject(Sinogram3D* in, Image* out) { return ref->Backproject(in, out); }
  bool DivideAndBackproject(Sinogram3D* a, Sinogram3D* b, Image* out) { return ref->DivideAndBackproject(a, b, out); }
};

// The 3D loops of SiddonProjector::Project and ::DivideAndBackproject with
// several rays per bin (recon/src/SiddonProjector.cpp:322-441, :571-704):
// the reference's own getPointsFromLor / getPointsFromOverSampledLor and
// Siddon(), the loop order and the ray-selection rules unchanged, and a full
// bounds mask on the voxel index (the reference checks only the upper bounds
// at :417 and :666).
struct SampledMasked {
  int ns, nas, multi;

  // Calls f(LOR) for every ray of bin (k, l) of sinogram s2.
  template <class F>
  void rays(Sinogram3D* sino, Sinogram2DinCylindrical3Dpet* s2, int k, int l, bool dab, F&& f) const {
    float ringWidth_mm = sino->getAxialFoV_mm() / sino->getNumRings();
    float deltaZ_oversampling = ringWidth_mm / nas;
    int numZ = multi ? s2->getNumZ() : 1;
    float z1_mm = 0, z2_mm = 0;
    if (!multi) {
      z1_mm = (s2->getAxialValue1FromList(0) + s2->getAxialValue1FromList(s2->getNumZ() - 1)) / 2;
      z2_mm = (s2->getAxialValue2FromList(0) + s2->getAxialValue2FromList(s2->getNumZ() - 1)) / 2;
    }
    const bool plain = dab ? (ns == 1 && nas == 1) : (ns == 1);
    for (int m = 0; m < numZ; m++)
      for (int o = 0; o < ns; o++)
        for (int p = 0; p < nas; p++) {
          Point3D P1, P2; float geom; int ok;
          if (plain) ok = s2->getPointsFromLor(k, l, m, &P1, &P2, &geom);
          else ok = s2->getPointsFromOverSampledLor(k, l, o, ns, m, ringWidth_mm, p, nas, &P1, &P2, &geom);
          if (!multi) {
            P1.Z = z1_mm - ringWidth_mm / 2 + deltaZ_oversampling / 2 + p * deltaZ_oversampling;
            P2.Z = z2_mm - ringWidth_mm / 2 + deltaZ_oversampling / 2 + p * deltaZ_oversampling;
          }
          if (!ok) continue;
          Line3D LOR;
          LOR.P0 = P1; LOR.Vx = P2.X - P1.X; LOR.Vy = P2.Y - P1.Y; LOR.Vz = P2.Z - P1.Z;
          f(LOR, geom);
        }
  }

  void project(Image* im, Sinogram3D* out) const {
    SizeImage sz = im->getSize();
    float* px = im->getPixelsPtr();
    out->FillConstant(0.0);
    for (int i = 0; i < out->getNumSegments(); i++)
      for (int j = 0; j < out->getSegment(i)->getNumSinograms(); j++) {
        Sinogram2DinCylindrical3Dpet* s2 = out->getSegment(i)->getSinogram2D(j);
        #pragma omp parallel for schedule(dynamic, 1)
        for (int k = 0; k < s2->getNumProj(); k++)
          for (int l = 0; l < s2->getNumR(); l++)
            rays(out, s2, k, l, false, [&](Line3D& LOR, float geom) {
              SiddonSegment* w = NULL; int n = 0;
              Siddon(LOR, im, &w, &n, 1);
              if (n <= 0) return;
              for (int q = 0; q < n; q++)
                if (w[q].IndexX >= 0 && w[q].IndexY >= 0 && w[q].IndexZ >= 0 && w[q].IndexX < sz.nPixelsX &&
                    w[q].IndexY < sz.nPixelsY && w[q].IndexZ < sz.nPixelsZ)
                  s2->incrementSinogramBin(k, l, w[q].Segment * geom *
                      px[w[q].IndexZ * (sz.nPixelsX * sz.nPixelsY) + w[q].IndexY * sz.nPixelsX + w[q].IndexX]);
              free(w);
            });
      }
  }

  void divide_and_backproject(Sinogram3D* in, Sinogram3D* est, Image* im) const {
    SizeImage sz = im->getSize();
    float* px = im->getPixelsPtr();
    for (int i = 0; i < in->getNumSegments(); i++) {
      #pragma omp parallel for schedule(dynamic, 1)
      for (int j = 0; j < in->getSegment(i)->getNumSinograms(); j++) {
        Sinogram2DinCylindrical3Dpet* s2 = in->getSegment(i)->getSinogram2D(j);
        Sinogram2D* e2 = est->getSegment(i)->getSinogram2D(j);
        for (int k = 0; k < s2->getNumProj(); k++)
          for (int l = 0; l < s2->getNumR(); l++) {
            const float m = s2->getSinogramBin(k, l), e = e2->getSinogramBin(k, l);
            if (m == 0) continue;
            rays(in, s2, k, l, true, [&](Line3D& LOR, float geom) {
              SiddonSegment* w = NULL; int n = 0;
              Siddon(LOR, im, &w, &n, 1);
              for (int q = 0; q < n; q++) {
                if (!(w[q].IndexX >= 0 && w[q].IndexY >= 0 && w[q].IndexZ >= 0 && w[q].IndexX < sz.nPixelsX &&
                      w[q].IndexY < sz.nPixelsY && w[q].IndexZ < sz.nPixelsZ))
                  continue;
                float v;
                if (e != 0) v = w[q].Segment * geom * m / e;
                else if (m != 0) v = w[q].Segment * geom * m;
                else v = 0;
                #pragma omp atomic
                px[w[q].IndexZ * (sz.nPixelsX * sz.nPixelsY) + w[q].IndexY * sz.nPixelsX + w[q].IndexX] += v;
              }
              if (n != 0) free(w);
            });
          }
      }
    }
  }
};

std::string write_sino3d_header(const char* dir, int nProj, int nR, int nRings, int nSeg,
                                const int* nSinos, const int* minRD, const int* maxRD,
                                const float* data) {
  std::string base = std::string(dir) + "/ref_sino3d";
  std::string hdr = base + ".h33", dat = base + ".i33";
  FILE* f = fopen(hdr.c_str(), "w");
  if (!f) return "";
  fprintf(f, "!INTERFILE :=\n");
  fprintf(f, "!name of data file := %s\n", dat.c_str());
  fprintf(f, "number of dimensions := 4\n");
  fprintf(f, "matrix axis label [4] := segment\n");
  fprintf(f, "!matrix size [4] := %d\n", nSeg);
  fprintf(f, "matrix axis label [3] := axial coordinate\n");
  fprintf(f, "!matrix size [3] := {");
  for (int i = 0; i < nSeg; i++) fprintf(f, i ? ",%d" : "%d", nSinos[i]);
  fprintf(f, "}\n");
  fprintf(f, "minimum ring difference per segment := {");
  for (int i = 0; i < nSeg; i++) fprintf(f, i ? ",%d" : "%d", minRD[i]);
  fprintf(f, "}\n");
  fprintf(f, "maximum ring difference per segment := {");
  for (int i = 0; i < nSeg; i++) fprintf(f, i ? ",%d" : "%d", maxRD[i]);
  fprintf(f, "}\n");
  fprintf(f, "matrix axis label [2] := view\n");
  fprintf(f, "!matrix size [2] := %d\n", nProj);
  fprintf(f, "matrix axis label [1] := tangential coordinate\n");
  fprintf(f, "!matrix size [1] := %d\n", nR);
  fprintf(f, "number of rings := %d\n", nRings);
  fprintf(f, "!END OF INTERFILE :=\n");
  fclose(f);
  long total = 0;
  for (int i = 0; i < nSeg; i++) total += (long)nSinos[i] * nProj * nR;
  FILE* d = fopen(dat.c_str(), "wb");
  if (!d) return "";
  if (data) fwrite(data, sizeof(float), (size_t)total, d);
  else {
    std::vector<float> z((size_t)nProj * nR, 0.f);
    for (long s = 0; s < total / ((long)nProj * nR); s++) fwrite(z.data(), sizeof(float), z.size(), d);
  }
  fclose(d);
  return hdr;
}

struct Sino3DHandle {
  Sinogram3DCylindricalPet* sino;
  float rFov, axialFov, rScanner;
};

void copy_out(Sinogram3D* s, float* out) {
  size_t off = 0;
  for (int i = 0; i < s->getNumSegments(); i++)
    for (int j = 0; j < s->getSegment(i)->getNumSinograms(); j++) {
      Sinogram2D* s2 = s->getSegment(i)->getSinogram2D(j);
      size_t n = (size_t)s2->getNumProj() * s2->getNumR();
      memcpy(out + off, s2->getSinogramPtr(), n * sizeof(float));
      off += n;
    }
}
void copy_in(Sinogram3D* s, const float* in) {
  size_t off = 0;
  for (int i = 0; i < s->getNumSegments(); i++)
    for (int j = 0; j < s->getSegment(i)->getNumSinograms(); j++) {
      Sinogram2D* s2 = s->getSegment(i)->getSinogram2D(j);
      size_t n = (size_t)s2->getNumProj() * s2->getNumR();
      memcpy(s2->getSinogramPtr(), in + off, n * sizeof(float));
      off += n;
    }
}

struct Mlem2dAccess : public Mlem2d {
  using Mlem2d::Mlem2d;
  float* lik() { return likelihoodValues; }
  Image* sens() { return sensitivityImage; }
};

}  // namespace

extern "C" {

int ref_set_threads(int n) { if (n > 0) omp_set_num_threads(n); return omp_get_max_threads(); }

// ---- 2D -------------------------------------------------------------------
static Sinogram2DinCylindrical3Dpet* make_sino2d(int nProj, int nR, float rFov, float rScanner, const float* v) {
  Sinogram2DinCylindrical3Dpet* s = new Sinogram2DinCylindrical3Dpet((unsigned)nProj, (unsigned)nR, rFov, rScanner);
  if (v) memcpy(s->getSinogramPtr(), v, sizeof(float) * (size_t)nProj * nR);
  return s;
}

int ref_project_2d(int nx, int ny, float dx, float dy, const float* img,
                   int nProj, int nR, float rFov, float rScanner, float* out) {
  Image* im = make_image(nx, ny, 1, dx, dy, 1.0f, img);
  Sinogram2DinCylindrical3Dpet* s = make_sino2d(nProj, nR, rFov, rScanner, out);
  MaskedSiddonProjector p;
  p.Project(im, (Sinogram2D*)s);
  memcpy(out, s->getSinogramPtr(), sizeof(float) * (size_t)nProj * nR);
  delete s; delete im;
  return 0;
}

// LOR end points as the reference computes them (getPointsFromLor,
// data/src/Sinogram2DinCylindrical3Dpet.cpp:249-266): [angle][r][p1x,p1y,p2x,p2y].
int ref_lor_points_2d(int nProj, int nR, float rFov, float rScanner, float* out4) {
  Sinogram2DinCylindrical3Dpet* s = make_sino2d(nProj, nR, rFov, rScanner, NULL);
  for (int a = 0; a < nProj; a++)
    for (int l = 0; l < nR; l++) {
      Point2D P1, P2; float geom;
      float* o = out4 + ((size_t)a * nR + l) * 4;
      if (!s->getPointsFromLor(a, l, &P1, &P2, &geom)) { o[0] = o[1] = o[2] = o[3] = 0; continue; }
      o[0] = P1.X; o[1] = P1.Y; o[2] = P2.X; o[3] = P2.Y;
    }
  delete s;
  return 0;
}

// Segment list of one 3D LOR from the reference Siddon().
int ref_siddon3d(float p1x, float p1y, float p1z, float p2x, float p2y, float p2z, int nx, int ny, int nz,
                 float dx, float dy, float dz, int* ijk, float* w, int cap) {
  Image* im = make_image(nx, ny, nz, dx, dy, dz, NULL);
  Line3D L; SiddonSegment* ws = NULL; int n = 0;
  L.P0.X = p1x; L.P0.Y = p1y; L.P0.Z = p1z; L.Vx = p2x - p1x; L.Vy = p2y - p1y; L.Vz = p2z - p1z;
  Siddon(L, im, &ws, &n, 1);
  for (int m = 0; m < n && m < cap; m++) {
    ijk[3 * m] = ws[m].IndexX; ijk[3 * m + 1] = ws[m].IndexY; ijk[3 * m + 2] = ws[m].IndexZ; w[m] = ws[m].Segment;
  }
  if (n > 0) free(ws);
  delete im;
  return n;
}

int ref_backproject_2d(int nx, int ny, float dx, float dy, float* img_inout,
                       int nProj, int nR, float rFov, float rScanner, const float* sino) {
  Image* im = make_image(nx, ny, 1, dx, dy, 1.0f, img_inout);
  Sinogram2DinCylindrical3Dpet* s = make_sino2d(nProj, nR, rFov, rScanner, sino);
  SiddonProjector sp(1, 1);
  sp.Backproject((Sinogram2D*)s, im);
  memcpy(img_inout, im->getPixelsPtr(), sizeof(float) * (size_t)nx * ny);
  delete s; delete im;
  return 0;
}

// Mlem2d::Reconstruct (recon/src/Mlem2d.cpp:60-260) with the masked forward
// projector.  The Mlem2d constructor forces the sinogram rFov to the image rFov
// (recon/src/Mlem2d.cpp:12); the caller's sinogram rFov is restored afterwards
// through the shared pointer, as a user wanting a given bin pitch has to do.
int ref_mlem_2d(int nx, int ny, float dx, float dy, const float* init,
                int nProj, int nR, float rFov, float rScanner, const float* measured,
                int iters, const char* tmpdir, float* out_img, float* out_lik, float* out_sens) {
  Image* x0 = make_image(nx, ny, 1, dx, dy, 1.0f, init);
  Sinogram2DinCylindrical3Dpet* s = make_sino2d(nProj, nR, rFov, rScanner, measured);
  MaskedSiddonProjector* p = new MaskedSiddonProjector();
  std::string prefix = std::string(tmpdir) + "/ref_mlem2d";
  Mlem2dAccess* m = new Mlem2dAccess((Sinogram2D*)s, x0, std::string(tmpdir), prefix, iters, 0, false, false, p, p);
  s->setRadioFov_mm(rFov);
  if (!m->Reconstruct()) return 1;
  memcpy(out_img, m->getReconstructedImage()->getPixelsPtr(), sizeof(float) * (size_t)nx * ny);
  if (out_lik) memcpy(out_lik, m->lik(), sizeof(float) * (size_t)(iters + 1));
  if (out_sens) memcpy(out_sens, m->sens()->getPixelsPtr(), sizeof(float) * (size_t)nx * ny);
  return 0;
}

// ---- interfile output of the reference (format fixtures) -------------------
int ref_sino3d_write(void* hv, const char* path_no_ext) {
  return ((Sino3DHandle*)hv)->sino->writeInterfile(std::string(path_no_ext)) ? 0 : 1;
}

int ref_image_write(int nx, int ny, int nz, float dx, float dy, float dz, const float* px, const char* path_no_ext) {
  Image* im = make_image(nx, ny, nz, dx, dy, dz, px);
  int rc = im->writeInterfile((char*)path_no_ext) ? 0 : 1;
  delete im;
  return rc;
}

// Image::readFromInterfile (medcon); dims = {nx, ny, nz}, pix = {dx, dy, dz}.
int ref_image_read(const char* header, int* dims, float* pix, float* out, long cap) {
  Image* im = new Image();
  if (!im->readFromInterfile((char*)header)) { delete im; return 1; }
  SizeImage s = im->getSize();
  dims[0] = s.nPixelsX; dims[1] = s.nPixelsY; dims[2] = s.nPixelsZ;
  pix[0] = s.sizePixelX_mm; pix[1] = s.sizePixelY_mm; pix[2] = s.sizePixelZ_mm;
  long n = (long)s.nPixelsX * s.nPixelsY * s.nPixelsZ;
  if (out && n <= cap) memcpy(out, im->getPixelsPtr(), sizeof(float) * n);
  return 0;
}

// Sinogram3DCylindricalPet(header, ...) reading; returns bins copied.
long ref_sino3d_read(const char* header, float rFov, float zFov, float rScanner, float* out, long cap,
                     int* nseg_out) {
  Sinogram3DCylindricalPet* s = new Sinogram3DCylindricalPet((char*)header, rFov, zFov, rScanner);
  long n = s->getBinCount();
  *nseg_out = s->getNumSegments();
  if (out && n <= cap) copy_out(s, out);
  return n;
}

// ---- 3D -------------------------------------------------------------------
void* ref_sino3d_create(const char* tmpdir, int nProj, int nR, int nRings, float rFov, float axialFov,
                        float rScanner, int nSeg, const int* nSinos, const int* minRD, const int* maxRD,
                        const float* data) {
  std::string hdr = write_sino3d_header(tmpdir, nProj, nR, nRings, nSeg, nSinos, minRD, maxRD, data);
  if (hdr.empty()) return NULL;
  Sino3DHandle* h = new Sino3DHandle;
  h->sino = new Sinogram3DCylindricalPet((char*)hdr.c_str(), rFov, axialFov, rScanner);
  h->rFov = rFov; h->axialFov = axialFov; h->rScanner = rScanner;
  if (h->sino->getNumSegments() != nSeg) { delete h; return NULL; }
  fix_angle_buffer(h->sino);
  return h;
}

void ref_sino3d_destroy(void* hv) {
  Sino3DHandle* h = (Sino3DHandle*)hv;
  delete h;  // the reference sinogram destructor frees with mismatched free/delete; leak it
}

long ref_sino3d_num_bins(void* hv) { return ((Sino3DHandle*)hv)->sino->getBinCount(); }

// Per-sinogram ring-pair z coordinates as the reference holds them: first and
// last entries of the per-sinogram lists (data/src/Sinogram3D.cpp:396-464).
int ref_sino3d_ring_z(void* hv, float* z1_first, float* z1_last, float* z2_first, float* z2_last, int* numZ) {
  Sinogram3DCylindricalPet* s = ((Sino3DHandle*)hv)->sino;
  int g = 0;
  for (int i = 0; i < s->getNumSegments(); i++)
    for (int j = 0; j < s->getSegment(i)->getNumSinograms(); j++, g++) {
      Sinogram2DinCylindrical3Dpet* s2 = s->getSegment(i)->getSinogram2D(j);
      z1_first[g] = s2->getAxialValue1FromList(0); z1_last[g] = s2->getAxialValue1FromList(s2->getNumZ() - 1);
      z2_first[g] = s2->getAxialValue2FromList(0); z2_last[g] = s2->getAxialValue2FromList(s2->getNumZ() - 1);
      numZ[g] = s2->getNumZ();
    }
  return g;
}

// Projection of one subset (subset < 0: the whole sinogram) into `out`, laid out
// as the subset sinogram [segment][sinogram][angle][r].
int ref_project_3d(void* hv, int subset, int nsubsets, int nx, int ny, int nz, float dx, float dy, float dz,
                   const float* img, float* out) {
  Sinogram3DCylindricalPet* full = ((Sino3DHandle*)hv)->sino;
  Sinogram3D* s = subset >= 0 ? full->getSubset(subset, nsubsets) : full->getSubset(0, 1);
  Image* im = make_image(nx, ny, nz, dx, dy, dz, img);
  MaskedSiddonProjector p;
  p.Project(im, s);
  copy_out(s, out);
  delete im;
  return 0;
}

// SiddonProjector::Backproject (unmodified) of `values` laid out as the subset
// sinogram, accumulated into img_inout.
int ref_backproject_3d(void* hv, int subset, int nsubsets, int nx, int ny, int nz, float dx, float dy, float dz,
                       const float* values, float* img_inout) {
  Sinogram3DCylindricalPet* full = ((Sino3DHandle*)hv)->sino;
  Sinogram3D* s = subset >= 0 ? full->getSubset(subset, nsubsets) : full->getSubset(0, 1);
  copy_in(s, values);
  Image* im = make_image(nx, ny, nz, dx, dy, dz, img_inout);
  SiddonProjector sp(1, 1);
  sp.Backproject(s, im);
  memcpy(img_inout, im->getPixelsPtr(), sizeof(float) * (size_t)nx * ny * nz);
  delete im;
  return 0;
}

// Several rays per bin: ns radial and nas axial samples (SiddonProjector(ns,
// nas)), multi = setMultipleLorsPerBin(true).  mode 0: masked Project into
// `out` (subset sinogram layout); 1: the reference's own
// SiddonProjector::Backproject of `in`, accumulated into `out` (image);
// 2: masked DivideAndBackproject of in / vest, accumulated into `out`.
int ref_sampled_3d(void* hv, int ns, int nas, int multi, int mode, int subset, int nsubsets, int nx, int ny, int nz,
                   float dx, float dy, float dz, const float* in, const float* vest, float* out) {
  Sinogram3DCylindricalPet* full = ((Sino3DHandle*)hv)->sino;
  Sinogram3D* s = subset >= 0 ? full->getSubset(subset, nsubsets) : full->getSubset(0, 1);
  SampledMasked sm{ns, nas, multi};
  if (mode == 0) {
    Image* im = make_image(nx, ny, nz, dx, dy, dz, in);
    sm.project(im, s);
    copy_out(s, out);
    delete im;
    return 0;
  }
  copy_in(s, in);
  Image* im = make_image(nx, ny, nz, dx, dy, dz, out);
  if (mode == 1) {
    SiddonProjector sp(ns, nas);
    // SiddonProjector derives privately from Projector (SiddonProjector.h:25);
    // the reference's callers reach the base with a C-style cast too.
    ((Projector*)&sp)->setMultipleLorsPerBin(multi != 0);
    sp.Backproject(s, im);
  } else {
    Sinogram3D* e = subset >= 0 ? full->getSubset(subset, nsubsets) : full->getSubset(0, 1);
    copy_in(e, vest);
    sm.divide_and_backproject(s, e, im);
  }
  memcpy(out, im->getPixelsPtr(), sizeof(float) * (size_t)nx * ny * nz);
  delete im;
  return 0;
}

// One OSEM sub-iteration in the order of OsemSinogram3d::Reconstruct
// (recon/src/OsemSinogram3d.cpp:159-237): subset copies, projection,
// likelihood, ratio, backprojection and the multiplicative update with
// threshold 0 and >=.  Used as the timed CPU baseline; x_inout is updated.
int ref_osem_3d_subiteration_rule(void* hv, int subset, int nsubsets, int nx, int ny, int nz, float dx, float dy,
                                  float dz, float* x_inout, const float* sens, float* out_lik, int ge);

int ref_osem_3d_subiteration(void* hv, int subset, int nsubsets, int nx, int ny, int nz, float dx, float dy,
                             float dz, float* x_inout, const float* sens, float* out_lik) {
  return ref_osem_3d_subiteration_rule(hv, subset, nsubsets, nx, ny, nz, dx, dy, dz, x_inout, sens, out_lik, 1);
}

// ge = 0: the pixel update only where sens > 0 (else 0) instead of the
// reference's sens >= 0, which divides 0 by 0 at voxels no ray of the subset
// crosses.
int ref_osem_3d_subiteration_rule(void* hv, int subset, int nsubsets, int nx, int ny, int nz, float dx, float dy,
                                  float dz, float* x_inout, const float* sens, float* out_lik, int ge) {
  Sinogram3DCylindricalPet* full = ((Sino3DHandle*)hv)->sino;
  Image* x = make_image(nx, ny, nz, dx, dy, dz, x_inout);
  Image* bp = make_image(nx, ny, nz, dx, dy, dz, NULL);
  Sinogram3D* in = full->getSubset(subset, nsubsets);
  Sinogram3D* est = full->getSubset(subset, nsubsets);
  est->FillConstant(0);
  MaskedSiddonProjector p;
  p.Project(x, est);
  float lik = est->getLikelihoodValue(in);
  bp->fillConstant(0);
  est->inverseDivideBinToBin(in);
  p.Backproject(est, bp);
  float* px = x->getPixelsPtr(); float* pb = bp->getPixelsPtr();
  long n = (long)nx * ny * nz;
  for (long k = 0; k < n; k++) px[k] = (ge ? sens[k] >= 0 : sens[k] > 0) ? px[k] * pb[k] / sens[k] : 0;
  memcpy(x_inout, px, sizeof(float) * n);
  if (out_lik) *out_lik = lik;
  delete x; delete bp;
  return 0;
}

// OsemSinogram3d::Reconstruct (recon/src/OsemSinogram3d.cpp:36-325) step by
// step with the reference's own primitives: per-subset sensitivity as in
// computeSensitivity (:327-346) plus forcePositive (:115), threshold 0 (:24-33),
// then for every iteration and subset the body of ref_osem_3d_subiteration.
// The reference driver itself cannot be run end to end: its final likelihood
// projects onto inputProjection->Copy() (:291), whose 2D sinograms carry an
// uninitialised scanner radius (see the note at the top of this file), and
// that projection crashed here.  The final likelihood below projects the whole
// sinogram through getSubset(0, 1) instead.
int ref_osem_3d(void* hv, int nx, int ny, int nz, float dx, float dy, float dz, const float* init,
                int iters, int nsubsets, const char* tmpdir, float* out_img, float* out_lik, float* out_sens0) {
  (void)tmpdir;
  Sinogram3DCylindricalPet* full = ((Sino3DHandle*)hv)->sino;
  long n = (long)nx * ny * nz;
  std::vector<std::vector<float>> sens(nsubsets);
  SiddonProjector sp(1, 1);
  for (int s = 0; s < nsubsets; s++) {
    Image* si = make_image(nx, ny, nz, dx, dy, dz, NULL);
    si->fillConstant(0);
    Sinogram3D* b = full->getSubset(s, nsubsets);
    b->FillConstant(1);
    sp.Backproject(b, si);
    si->forcePositive();
    sens[s].assign(si->getPixelsPtr(), si->getPixelsPtr() + n);
    delete si;
  }
  std::vector<float> x(init, init + n);
  for (int t = 0; t < iters; t++)
    for (int s = 0; s < nsubsets; s++) {
      float lik = 0;
      ref_osem_3d_subiteration(hv, s, nsubsets, nx, ny, nz, dx, dy, dz, x.data(), sens[s].data(), &lik);
      if (out_lik) out_lik[nsubsets * t + s] = lik;
    }
  if (out_lik) {
    Image* xi = make_image(nx, ny, nz, dx, dy, dz, x.data());
    Sinogram3D* est = full->getSubset(0, 1);
    MaskedSiddonProjector p;
    p.Project(xi, est);
    out_lik[iters * nsubsets] = est->getLikelihoodValue(full);
    delete xi;
  }
  memcpy(out_img, x.data(), sizeof(float) * n);
  if (out_sens0) memcpy(out_sens0, sens[0].data(), sizeof(float) * n);
  return 0;
}

// ---- Siemens mMR ------------------------------------------------------------
// Sinogram3DSiemensMmr read from an interfile header (the reference's own
// constructor, data/src/Sinogram3DSiemensMmr.cpp); no subsets are taken of it
// (getSubset copies nProj angles into a one-float buffer, :184).
void* ref_mmr_sino3d_create(const char* tmpdir, int nProj, int nR, int nRings, int nSeg, const int* nSinos,
                            const int* minRD, const int* maxRD, const float* data) {
  std::string hdr = write_sino3d_header(tmpdir, nProj, nR, nRings, nSeg, nSinos, minRD, maxRD, data);
  if (hdr.empty()) return NULL;
  Sinogram3DSiemensMmr* s = new Sinogram3DSiemensMmr((char*)hdr.c_str());
  if (s->getNumSegments() != nSeg) return NULL;
  return s;
}

// LOR end points of every (angle, r) from the first 2D sinogram
// (getPointsFromLor, Sinogram2DinSiemensMmr.cpp:174-198) and each sinogram's
// end-point z as SiddonProjector::Project sets it (:357-360, :392-396).
int ref_mmr_tables(void* hv, float* lor, float* z) {
  Sinogram3D* s = (Sinogram3D*)hv;
  Sinogram2DinCylindrical3Dpet* s0 = s->getSegment(0)->getSinogram2D(0);
  for (int k = 0; k < s0->getNumProj(); k++)
    for (int l = 0; l < s0->getNumR(); l++) {
      Point3D P1, P2; float geom;
      s0->getPointsFromLor(k, l, 0, &P1, &P2, &geom);
      float* o = lor + ((size_t)k * s0->getNumR() + l) * 4;
      o[0] = P1.X; o[1] = P1.Y; o[2] = P2.X; o[3] = P2.Y;
    }
  float ringWidth_mm = s->getAxialFoV_mm() / s->getNumRings();
  float deltaZ = ringWidth_mm / 1;
  int g = 0;
  for (int i = 0; i < s->getNumSegments(); i++)
    for (int j = 0; j < s->getSegment(i)->getNumSinograms(); j++, g++) {
      Sinogram2DinCylindrical3Dpet* s2 = s->getSegment(i)->getSinogram2D(j);
      float z1 = (s2->getAxialValue1FromList(0) + s2->getAxialValue1FromList(s2->getNumZ() - 1)) / 2;
      float z2 = (s2->getAxialValue2FromList(0) + s2->getAxialValue2FromList(s2->getNumZ() - 1)) / 2;
      int p = 0;
      z[2 * g] = z1 - ringWidth_mm / 2 + deltaZ / 2 + p * deltaZ;
      z[2 * g + 1] = z2 - ringWidth_mm / 2 + deltaZ / 2 + p * deltaZ;
    }
  return g;
}

// Whole-sinogram projection (masked loops of SiddonProjector::Project).
int ref_mmr_project(void* hv, int nx, int ny, int nz, float dx, float dy, float dz, const float* img, float* out) {
  Sinogram3D* s = (Sinogram3D*)hv;
  Image* im = make_image(nx, ny, nz, dx, dy, dz, img);
  MaskedSiddonProjector p;
  p.Project(im, s);
  copy_out(s, out);
  delete im;
  return 0;
}

// SiddonProjector::Backproject (unmodified) of `values`, accumulated into img_inout.
int ref_mmr_backproject(void* hv, int nx, int ny, int nz, float dx, float dy, float dz, const float* values,
                        float* img_inout) {
  Sinogram3D* s = (Sinogram3D*)hv;
  copy_in(s, values);
  Image* im = make_image(nx, ny, nz, dx, dy, dz, img_inout);
  SiddonProjector sp(1, 1);
  sp.Backproject(s, im);
  memcpy(img_inout, im->getPixelsPtr(), sizeof(float) * (size_t)nx * ny * nz);
  delete im;
  return 0;
}

}  // extern "C"
