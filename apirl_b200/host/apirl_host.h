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
//   CuProjector, TipoProyector .. reconGPU/inc/CuProjector.h:63-110,
//                                 reconGPU/inc/CuSiddonProjector.h:101-106
//   CuProjectorInterface ........ reconGPU/inc/CuProjectorInterface.h:53-172
//   Mlem, Mlem2d, MlemSinogram3d, OsemSinogram3d .. recon/inc/Mlem*.h, OsemSinogram3d.h
//   CuMlemSinogram3d, CuOsemSinogram3d .. reconGPU/inc/CuMlemSinogram3d.h:65-282,
//                                 reconGPU/inc/CuOsemSinogram3d.h:66-146
//
// Everything is in namespace apirl; `using namespace apirl;` gives the
// reference's spellings.  Compute runs on the GPU through the C ABI; these
// classes hold host copies of images and sinograms as the reference's do.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include <vector_types.h>  // dim3, as in the reference's GPU-side signatures

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

// reconGPU/inc/CuSiddonProjector.h:101-106.  Every cylindrical kind runs the
// same exact Siddon walk here (the reference's texture kind sampled the image
// with trilinear interpolation instead); SIDDON_HEXAGONAL_SCANNER is rejected.
typedef enum {
  SIDDON_CYLINDRICAL_SCANNER,
  SIDDON_PROJ_TEXT_CYLINDRICAL_SCANNER,
  SIDDON_BACKPROJ_SURF_CYLINDRICAL_SCANNER,
  SIDDON_HEXAGONAL_SCANNER
} TipoProyector;

// reconGPU/inc/CuProjector.h:63-110: projection between device buffers.  An
// image buffer holds the voxels [z][y][x]; a sinogram buffer holds the bins of
// every sinogram of the Sinogram3D argument in its order, [sinogram][angle][r]
// (the subset's angles only, for a sinogram made by getSubset).  d_ring1 and
// d_ring2 hold one float per sinogram, the axial end points in mm; an
// implementation may take them from the Sinogram3D instead.
class CuProjector {
 public:
  CuProjector();
  CuProjector(unsigned int numThreadsPerBlockX, unsigned int numThreadsPerBlockY, unsigned int numThreadsPerBlockZ,
              unsigned int numBlocksX, unsigned int numBlocksY, unsigned int numBlocksZ);
  virtual ~CuProjector() = default;
  virtual bool Backproject(float* d_inputSinogram, float* d_outputImage, float* d_ring1, float* d_ring2,
                           Sinogram3D* inputSinogram, Image* outputImage, bool copyResult) {
    return false;
  }
  virtual bool DivideAndBackproject(float* d_inputSinogram, float* d_estimatedSinogram, float* d_outputImage,
                                    float* d_ring1, float* d_ring2, Sinogram3D* inputSinogram, Image* outputImage,
                                    bool copyResult) {
    return false;
  }
  virtual bool Project(float* d_image, float* d_projection, float* d_ring1, float* d_ring2, Image* inputImage,
                       Sinogram3D* outputSinogram, bool copyResult) {
    return false;
  }
  virtual void initGpuMemory(Sinogram3D*) {}
  void setKernelConfig(unsigned int numThreadsPerBlockX, unsigned int numThreadsPerBlockY,
                       unsigned int numThreadsPerBlockZ, unsigned int numBlocksX, unsigned int numBlocksY,
                       unsigned int numBlocksZ);
  dim3 getBlockSize() const { return blockSize; }
  dim3 getGridSize() const { return gridSize; }

 protected:
  unsigned int threads_per_block = 0;
  dim3 gridSize, blockSize;
};

// The Siddon projector on the GPU.  As a Projector: host images and sinograms
// in and out, device buffers and geometry tables cached between calls.  As a
// CuProjector: the caller's device buffers in and out.
class CuSiddonProjector : public Projector, public CuProjector {
 public:
  explicit CuSiddonProjector(int nSamplesOnDetector = 1, int nAxialSamplesOnDetector = 1, int gpuId = 0);
  ~CuSiddonProjector() override;
  bool Project(Image* image, Sinogram2D* projection) override;
  bool Backproject(Sinogram2D* projection, Image* image) override;
  bool DivideAndBackproject(Sinogram2D* in, Sinogram2D* est, Image* out) override;
  bool Project(Image* image, Sinogram3D* projection) override;
  bool Backproject(Sinogram3D* projection, Image* image) override;
  bool DivideAndBackproject(Sinogram3D* in, Sinogram3D* est, Image* out) override;
  // reconGPU/inc/CuSiddonProjector.h:140-158, on device buffers of the
  // projector's GPU.  Project overwrites d_projection; Backproject and
  // DivideAndBackproject add into d_outputImage (the caller zeroes it first,
  // as the reference's kernels expect) and leave the sinograms unchanged.
  // copyResult also copies the result into the host object (outputSinogram's
  // bins, outputImage's pixels).  The axial end points come from the
  // Sinogram3D as SiddonProjector computes them, so d_ring1 and d_ring2 are
  // not read and may be NULL.  The work runs on the legacy default stream and
  // is finished when the call returns, like the reference's wrappers.
  bool Project(float* d_image, float* d_projection, float* d_ring1, float* d_ring2, Image* inputImage,
               Sinogram3D* outputSinogram, bool copyResult) override;
  bool Backproject(float* d_inputSinogram, float* d_outputImage, float* d_ring1, float* d_ring2,
                   Sinogram3D* inputSinogram, Image* outputImage, bool copyResult) override;
  bool DivideAndBackproject(float* d_inputSinogram, float* d_estimatedSinogram, float* d_outputImage,
                            float* d_ring1, float* d_ring2, Sinogram3D* inputSinogram, Image* outputImage,
                            bool copyResult) override;
  // reconGPU/src/CuSiddonProjector.cu:34-44.  Nothing is set up ahead: the
  // geometry tables are built by the first call that also knows the image.
  bool InitGpuMemory(Sinogram3D*) { return true; }
  void initGpuMemory(Sinogram3D* s) override { InitGpuMemory(s); }
  int gpuId() const { return device; }
  // Moves the projector to GPU `id`; what was set up on another GPU is freed.
  bool setGpuId(int id);
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
  bool runDevice(int op, const float* d_a, const float* d_b, float* d_out, Image* img, Sinogram3D* s,
                 bool copyResult);
  void release();
};

// reconGPU/inc/CuProjectorInterface.h:53-172: a CuProjector used as a
// Projector, with host images and sinograms in and out and device buffers
// kept between calls (the reference allocated and freed them per call).
// Sinogram3D only: the Sinogram2D calls return false, as the reference's do.
// Project overwrites the sinogram; Backproject and DivideAndBackproject
// overwrite the image (the reference zeroes its device image first).  The
// ring arrays given to the CuProjector are the per-sinogram axial end points,
// apirl_sino3d_ring_z.  The CuProjector stays the caller's.
class CuProjectorInterface : public Projector {
 public:
  explicit CuProjectorInterface(CuProjector* projector);
  ~CuProjectorInterface() override;
  // Block size as given; grid = (ceil(nProj * nR / x), number of sinograms, 1)
  // (CuProjectorInterface.cu:152-172), passed to the CuProjector.
  void setProjectorKernelConfig(unsigned int numThreadsPerBlockX, unsigned int numThreadsPerBlockY,
                                unsigned int numThreadsPerBlockZ, Sinogram3D* sinogram);
  void setProjectorKernelConfig(dim3 blockSize, Sinogram3D* sinogram);
  void setProjectorBlockSizeConfig(dim3 blockSize) { blockSizeProjector = blockSize; }
  bool setGpuId(int id);
  bool Project(Image* image, Sinogram2D* projection) override;
  bool Backproject(Sinogram2D* projection, Image* image) override;
  bool DivideAndBackproject(Sinogram2D* in, Sinogram2D* est, Image* out) override;
  bool Project(Image* image, Sinogram3D* projection) override;
  bool Backproject(Sinogram3D* projection, Image* image) override;
  bool DivideAndBackproject(Sinogram3D* in, Sinogram3D* est, Image* out) override;

 private:
  bool prepare(Sinogram3D* s, Image* img, bool estimate);
  void release();
  CuProjector* projector;
  int gpuId = 0, bufDevice = -1;
  dim3 blockSizeProjector;
  float *d_image = nullptr, *d_projection = nullptr, *d_estimated = nullptr;
  float *d_ring1_mm = nullptr, *d_ring2_mm = nullptr;
  size_t nImage = 0, nBins = 0, nEstimated = 0, nSinos = 0;
};

// recon/inc/Mlem.h:82-297.  saveIterationInterval > 0 writes
// "<prefix>_iter_<t>" after every iteration t with t % interval == 0, as the
// reference does; saveIntermediate (the reference's estimated projections and
// backprojected images at those iterations) is kept but not acted on: the
// fused pass never forms them.
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
  // The fused device driver: ML-EM for numSubsets == 0, else OSEM.
  bool reconstructOnDevice(int numSubsets);
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

// reconGPU/inc/CuMlemSinogram3d.h:65-282: ML-EM with CuProjector pointers.
// Both projectors must be CuSiddonProjector with the same rays per bin; the
// iterations run in MlemSinogram3d's fused device driver.  The kernel
// configuration setters keep the block sizes they are given (getters below)
// and check nothing: launch shapes are the library's.
class CuMlemSinogram3d : public MlemSinogram3d {
 public:
  CuMlemSinogram3d(Sinogram3D* inputProjection, Image* initialEstimate, std::string pathSalida,
                   std::string outputPrefix, int numIterations, int saveIterationInterval, bool saveIntermediate,
                   bool sensitivityFromFile, CuProjector* forwardprojector, CuProjector* backprojector);
  void setProjectorKernelConfig(unsigned int x, unsigned int y, unsigned int z) { blockSizeProjector = dim3(x, y, z); }
  void setBackprojectorKernelConfig(unsigned int x, unsigned int y, unsigned int z) {
    blockSizeBackprojector = dim3(x, y, z);
  }
  void setUpdatePixelKernelConfig(unsigned int x, unsigned int y, unsigned int z) { blockSizeImageUpdate = dim3(x, y, z); }
  void setProjectorKernelConfig(dim3* b) { blockSizeProjector = *b; }
  void setBackprojectorKernelConfig(dim3* b) { blockSizeBackprojector = *b; }
  void setUpdatePixelKernelConfig(dim3* b) { blockSizeImageUpdate = *b; }
  dim3 getProjectorKernelConfig() const { return blockSizeProjector; }
  dim3 getBackprojectorKernelConfig() const { return blockSizeBackprojector; }
  dim3 getUpdatePixelKernelConfig() const { return blockSizeImageUpdate; }
  // On the projectors' GPU.
  bool Reconstruct() override;
  virtual bool Reconstruct(TipoProyector tipoProy);
  // Moves both projectors to GPU indexGpu first (CuMlemSinogram3d.cu:498).
  virtual bool Reconstruct(TipoProyector tipoProy, int indexGpu);

 protected:
  dim3 blockSizeProjector{128, 1, 1}, blockSizeBackprojector{128, 1, 1}, blockSizeImageUpdate{512, 1, 1};
};

// reconGPU/inc/CuOsemSinogram3d.h:66-146: OSEM with CuProjector pointers, run
// by OsemSinogram3d's device driver.
class CuOsemSinogram3d : public CuMlemSinogram3d {
 public:
  CuOsemSinogram3d(Sinogram3D* inputProjection, Image* initialEstimate, std::string pathSalida,
                   std::string outputPrefix, int numIterations, int saveIterationInterval, bool saveIntermediate,
                   bool sensitivityFromFile, CuProjector* forwardprojector, CuProjector* backprojector,
                   int numSubsets);
  using CuMlemSinogram3d::Reconstruct;
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
