// C++ host layer over the C ABI (include/apirl_b200.h), keeping the class
// names, constructor arguments and bool/error-string conventions of the
// reference's reconstruction path so that reference callers can switch:
//
//   SizeImage, Image ............ data/inc/Images.h:53-307
//   Sinogram2D(inCylindrical3Dpet) data/inc/Sinogram2D.h:63-297,
//                                 data/inc/Sinogram2DinCylindrical3Dpet.h
//   Sinogram3D(CylindricalPet) .. data/inc/Sinogram3D.h:63-313,
//                                 data/inc/Sinogram3DCylindricalPet.h
//   Projector ................... recon/inc/Projector.h:48-85
//   CuSiddonProjector ........... recon/inc/SiddonProjector.h:25-68 (SiddonProjector)
//                                 and reconGPU/inc/CuSiddonProjector.h:110-158
//   Mlem, Mlem2d, MlemSinogram3d, OsemSinogram3d .. recon/inc/Mlem*.h, OsemSinogram3d.h
//
// Everything is in namespace apirl; `using namespace apirl;` gives the
// reference's spellings.  Compute runs on the GPU through the C ABI; these
// classes hold host copies of images and sinograms as the reference's do.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/apirl_b200.h"

namespace apirl {

struct SizeImage {
  int nDimensions;
  int nPixelsX, nPixelsY, nPixelsZ;
  float sizePixelX_mm, sizePixelY_mm, sizePixelZ_mm;
};

class Image {
 public:
  Image();
  explicit Image(SizeImage size);
  explicit Image(Image* copy);
  explicit Image(const std::string& interfileHeader);
  SizeImage getSize() const { return size; }
  float* getPixelsPtr() { return pixels.data(); }
  const float* getPixelsPtr() const { return pixels.data(); }
  int getPixelCount() const { return (int)pixels.size(); }
  float getFovRadio() const { return fovRadio_mm; }
  float getFovHeight() const { return fovHeight_mm; }
  void fillConstant(float v);
  int forcePositive();
  float getMinValue() const;  // minimum over non-zero pixels (Images.cpp:397-419)
  float getMaxValue() const;
  float getPixelValue(int x, int y, int z) const { return pixels[((size_t)z * size.nPixelsY + y) * size.nPixelsX + x]; }
  void setPixelValue(int x, int y, int z, float v) { pixels[((size_t)z * size.nPixelsY + y) * size.nPixelsX + x] = v; }
  bool readFromInterfile(const char* headerPath);
  bool writeInterfile(const char* pathWithoutExtension) const;
  const char* getError() const { return strError.c_str(); }
  apirl_image_geom geom() const;

 private:
  void init(SizeImage s);
  SizeImage size{};
  std::vector<float> pixels;
  float fovRadio_mm = 0, fovHeight_mm = 0;
  mutable std::string strError;
};

// Common base of the sinogram types (the reference's Projection).
class Sinogram2D {
 public:
  Sinogram2D(int nProj, int nR, float rFov_mm, float rScanner_mm);
  virtual ~Sinogram2D() = default;
  int getNumProj() const { return numProj; }
  int getNumR() const { return numR; }
  float getRadioFov_mm() const { return radioFov_mm; }
  float getRadioScanner_mm() const { return radioScanner_mm; }
  // Sinogram2D::setRadioFov_mm recomputes the r values (Sinogram2D.cpp:190-198).
  void setRadioFov_mm(float rFov_mm) { radioFov_mm = rFov_mm; }
  float getSinogramBin(int a, int r) const { return bins[(size_t)a * numR + r]; }
  void setSinogramBin(int a, int r, float v) { bins[(size_t)a * numR + r] = v; }
  void incrementSinogramBin(int a, int r, float v) { bins[(size_t)a * numR + r] += v; }
  float* getSinogramPtr() { return bins.data(); }
  const float* getSinogramPtr() const { return bins.data(); }
  bool FillConstant(float v);
  void inverseDivideBinToBin(const Sinogram2D* dividend);
  void addBinToBin(const Sinogram2D* add);
  void multiplyBinToBin(const Sinogram2D* factor);
  float getLikelihoodValue(const Sinogram2D* reference) const;  // over bins > 0, FP64 sum
  virtual Sinogram2D* Copy() const { return new Sinogram2D(*this); }
  bool readFromInterfile(const char* headerPath);
  bool writeInterfile(const char* pathWithoutExtension) const;
  const char* getError() const { return strError.c_str(); }
  apirl_sino2d_geom geom() const { return apirl_sino2d_geom{numProj, numR, radioFov_mm, radioScanner_mm}; }

 protected:
  int numProj, numR;
  float radioFov_mm, radioScanner_mm;
  std::vector<float> bins;
  mutable std::string strError;
};

class Sinogram2DinCylindrical3Dpet : public Sinogram2D {
 public:
  Sinogram2DinCylindrical3Dpet(int nProj, int nR, float rFov_mm, float rScanner_mm)
      : Sinogram2D(nProj, nR, rFov_mm, rScanner_mm) {}
  Sinogram2DinCylindrical3Dpet(const char* headerPath, float rFov_mm, float rScanner_mm);
  Sinogram2D* Copy() const override { return new Sinogram2DinCylindrical3Dpet(*this); }
};

// Sinogram3D with the segment table of a cylindrical scanner.  Bins are held
// [segment][sinogram][angle][r] in one array.  A subset sinogram (getSubset)
// holds only the subset's angles and remembers which subset it is, so that
// the projector reads it with the right LORs.
class Sinogram3D {
 public:
  Sinogram3D(int nProj, int nR, int nRings, float rFov_mm, float axialFov_mm, float rScanner_mm,
             const std::vector<int>& minRingDiff, const std::vector<int>& maxRingDiff);
  virtual ~Sinogram3D() = default;
  int getNumProj() const { return numProjSubset; }
  int getNumProjFull() const { return numProj; }
  int getNumR() const { return numR; }
  int getNumRings() const { return numRings; }
  int getNumSegments() const { return (int)minRD.size(); }
  int getNumSinograms() const { return numSinos; }
  int getBinCount() const { return (int)bins.size(); }
  float getRadioFov_mm() const { return radioFov_mm; }
  float getAxialFoV_mm() const { return axialFov_mm; }
  float getRadioScanner_mm() const { return radioScanner_mm; }
  const std::vector<int>& minRingDiff() const { return minRD; }
  const std::vector<int>& maxRingDiff() const { return maxRD; }
  int subsetIndex() const { return subset; }
  int subsetCount() const { return nsubsets; }
  float* getSinogramPtr() { return bins.data(); }
  const float* getSinogramPtr() const { return bins.data(); }
  bool FillConstant(float v);
  void inverseDivideBinToBin(const Sinogram3D* dividend);
  void addBinToBin(const Sinogram3D* add);
  void multiplyBinToBin(const Sinogram3D* factor);
  float getLikelihoodValue(const Sinogram3D* reference) const;  // over bins != 0, FP64 sum
  virtual Sinogram3D* Copy() const { return new Sinogram3D(*this); }
  // Sinogram3DCylindricalPet::getSubset (Sinogram3DCylindricalPet.cpp:164-197).
  virtual Sinogram3D* getSubset(int indexSubset, int numSubsets) const;
  bool readFromInterfile(const char* headerPath);
  bool writeInterfile(const char* pathWithoutExtension) const;
  const char* getError() const { return strError.c_str(); }
  apirl_sino3d_geom geom() const;
  // APIRL_SCANNER_CYLINDRICAL, or APIRL_SCANNER_MMR for Sinogram3DSiemensMmr.
  virtual int scanner() const { return APIRL_SCANNER_CYLINDRICAL; }

 protected:
  int numProj, numProjSubset, numR, numRings, numSinos;
  float radioFov_mm, axialFov_mm, radioScanner_mm;
  std::vector<int> minRD, maxRD, sinosPerSegment;
  int subset = -1, nsubsets = 1;
  std::vector<float> bins;
  mutable std::string strError;
};

class Sinogram3DCylindricalPet : public Sinogram3D {
 public:
  using Sinogram3D::Sinogram3D;
  // Sinogram3DCylindricalPet(header, rFov, zFov, rScanner) (Sinogram3DCylindricalPet.cpp:19-35).
  Sinogram3DCylindricalPet(const char* headerPath, float rFov_mm, float zFov_mm, float rScanner_mm);
  Sinogram3D* Copy() const override { return new Sinogram3DCylindricalPet(*this); }
};

// data/inc/Sinogram3DSiemensMmr.h: the Siemens Biograph mMR's sinograms.
class Sinogram3DSiemensMmr : public Sinogram3D {
 public:
  using Sinogram3D::Sinogram3D;
  explicit Sinogram3DSiemensMmr(const char* headerPath);
  Sinogram3D* Copy() const override { return new Sinogram3DSiemensMmr(*this); }
  int scanner() const override { return APIRL_SCANNER_MMR; }
};

// recon/inc/Projector.h:48-85.
class Projector {
 public:
  virtual ~Projector() = default;
  void setMultipleLorsPerBin(bool enable) { useMultipleLorsPerBin = enable; }
  bool getMultipleLorsPerBin() const { return useMultipleLorsPerBin; }
  virtual bool Project(Image*, Sinogram2D*) { return false; }
  virtual bool Backproject(Sinogram2D*, Image*) { return false; }
  virtual bool DivideAndBackproject(Sinogram2D*, Sinogram2D*, Image*) { return false; }
  virtual bool Project(Image*, Sinogram3D*) { return false; }
  virtual bool Backproject(Sinogram3D*, Image*) { return false; }
  virtual bool DivideAndBackproject(Sinogram3D*, Sinogram3D*, Image*) { return false; }
  const char* getError() const { return strError.c_str(); }

 protected:
  bool useMultipleLorsPerBin = false;
  std::string strError;
};

// The Siddon projector on the GPU, as a Projector: host images and sinograms
// in and out, device buffers and geometry tables cached between calls.
class CuSiddonProjector : public Projector {
 public:
  explicit CuSiddonProjector(int nSamplesOnDetector = 1, int nAxialSamplesOnDetector = 1, int gpuId = 0);
  ~CuSiddonProjector() override;
  bool Project(Image* image, Sinogram2D* projection) override;
  bool Backproject(Sinogram2D* projection, Image* image) override;
  bool DivideAndBackproject(Sinogram2D* in, Sinogram2D* est, Image* out) override;
  bool Project(Image* image, Sinogram3D* projection) override;
  bool Backproject(Sinogram3D* projection, Image* image) override;
  bool DivideAndBackproject(Sinogram3D* in, Sinogram3D* est, Image* out) override;
  int gpuId() const { return device; }
  // The rays per bin this projector walks (SiddonProjector.h:43-47, Projector.h:54).
  apirl_sampling sampling() const { return {numSamplesOnDetector, numAxialSamplesOnDetector, useMultipleLorsPerBin}; }

 private:
  struct State;
  State* st;
  int device;
  int numSamplesOnDetector, numAxialSamplesOnDetector;
  bool prepare2d(const Image* img, const Sinogram2D* s);
  bool prepare3d(const Image* img, const Sinogram3D* s);
  bool run(int op, Image* img, const float* a, const float* b, float* out_sino, size_t nbins, int subset, int nsub);
};

// recon/inc/Mlem.h:82-297.
class Mlem {
 public:
  Mlem(Image* initialEstimate, std::string pathSalida, std::string outputPrefix, int numIterations,
       int saveIterationInterval, bool saveIntermediate, bool sensitivityFromFile, Projector* forwardprojector,
       Projector* backprojector);
  virtual ~Mlem();
  void setNumIterations(int n) { numIterations = n; }
  void setOutputFilenamePrefix(const std::string& p) { outputFilenamePrefix = p; }
  void setSensitivityImageFromFile(bool e) { sensitivityImageFromFile = e; }
  void setSensitivityFilename(const std::string& f) { sensitivityFilename = f; }
  void setSaveIterationInterval(int n) { saveIterationInterval = n; }
  void enableSaveIntermediates(bool f) { saveIntermediate = f; }
  Image* getReconstructedImage() { return reconstructionImage; }
  const std::vector<double>& getLikelihoodValues() const { return likelihood; }
  const char* getError() const { return strError.c_str(); }
  virtual bool setMultiplicativeProjection(const std::string& filename) = 0;
  virtual bool setAdditiveProjection(const std::string& filename) = 0;
  virtual bool Reconstruct() = 0;

 protected:
  void writeLog(const std::string& type, const std::string& inputDesc, double totalMs,
                const std::vector<double>& iterMs) const;
  Image* initialEstimate;
  Image* reconstructionImage = nullptr;
  Image* sensitivityImage = nullptr;
  std::string pathSalida, outputFilenamePrefix, sensitivityFilename;
  int numIterations, saveIterationInterval;
  bool saveIntermediate, sensitivityImageFromFile;
  Projector* forwardprojector;
  Projector* backprojector;
  std::vector<double> likelihood;
  std::string strError;
};

class Mlem2d : public Mlem {
 public:
  // Mlem2d.cpp:5-14: the sinogram's rFov is set to the image's.
  Mlem2d(Sinogram2D* inputProjection, Image* initialEstimate, std::string pathSalida, std::string outputPrefix,
         int numIterations, int saveIterationInterval, bool saveIntermediate, bool sensitivityFromFile,
         Projector* forwardprojector, Projector* backprojector);
  ~Mlem2d() override;
  bool setMultiplicativeProjection(const std::string& filename) override;
  bool setMultiplicativeProjection(Sinogram2D* s);
  bool setAdditiveProjection(const std::string& filename) override;
  bool setAdditiveProjection(Sinogram2D* s);
  bool Reconstruct() override;

 private:
  Sinogram2D* inputProjection;
  Sinogram2D* multiplicative = nullptr;
  Sinogram2D* additive = nullptr;
};

class MlemSinogram3d : public Mlem {
 public:
  MlemSinogram3d(Sinogram3D* inputProjection, Image* initialEstimate, std::string pathSalida,
                 std::string outputPrefix, int numIterations, int saveIterationInterval, bool saveIntermediate,
                 bool sensitivityFromFile, Projector* forwardprojector, Projector* backprojector);
  ~MlemSinogram3d() override;
  bool setMultiplicativeProjection(const std::string& filename) override;
  bool setMultiplicativeProjection(Sinogram3D* s);
  bool setAdditiveProjection(const std::string& filename) override;
  bool setAdditiveProjection(Sinogram3D* s);
  bool Reconstruct() override;

 protected:
  bool deviceResident() const;
  bool sameSampling(apirl_sampling* out);
  Sinogram3D* inputProjection;
  Sinogram3D* multiplicative = nullptr;
  Sinogram3D* additive = nullptr;
};

class OsemSinogram3d : public MlemSinogram3d {
 public:
  OsemSinogram3d(Sinogram3D* inputProjection, Image* initialEstimate, std::string pathSalida,
                 std::string outputPrefix, int numIterations, int saveIterationInterval, bool saveIntermediate,
                 bool sensitivityFromFile, Projector* forwardprojector, Projector* backprojector, int numSubsets);
  bool Reconstruct() override;

 private:
  int numSubsets;
};

// ---- parameter files (.par, data/inc/ParametersFile.h:34-46) -----------------
// Returns 0 on success or the reference's error codes: 1 file not found,
// 2 not a parameter file of `command`, 3 key not found, 4 bad format.
int parametersFile_read(const char* file, const char* command, const char* key, std::string* value);
// Interfile key reader (data/src/Interfile.cpp: interfile_read): 0 ok, 2 key not found, 3 no file, 4 not interfile.
int interfile_read(const char* header, const char* key, std::string* value);

}  // namespace apirl
