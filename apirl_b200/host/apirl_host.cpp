// Implementation of the C++ host layer (apirl_host.h) over the C ABI.
#include "apirl_host.h"

#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>

namespace apirl {

namespace {

std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

// Splits "key := value"; the key keeps a leading '!'.
bool split_line(const std::string& line, std::string* key, std::string* value) {
  size_t p = line.find(":=");
  if (p == std::string::npos) return false;
  *key = trim(line.substr(0, p));
  *value = trim(line.substr(p + 2));
  return true;
}

std::string dir_of(const std::string& path) {
  size_t p = path.find_last_of('/');
  return p == std::string::npos ? std::string() : path.substr(0, p + 1);
}

std::string base_of(const std::string& path) {
  size_t p = path.find_last_of('/');
  return p == std::string::npos ? path : path.substr(p + 1);
}

// Resolves a data-file name relative to its header (Sinogram3D.cpp:117-141).
std::string data_path(const std::string& header, const std::string& name) {
  if (name.find('/') != std::string::npos && name[0] == '/') return name;
  return dir_of(header) + name;
}

std::vector<int> parse_list(const std::string& v) {
  std::vector<int> out;
  size_t a = v.find('{'), b = v.rfind('}');
  std::string body = (a != std::string::npos && b != std::string::npos && b > a) ? v.substr(a + 1, b - a - 1) : v;
  std::stringstream ss(body);
  std::string tok;
  while (std::getline(ss, tok, ',')) {
    tok = trim(tok);
    if (!tok.empty()) out.push_back(atoi(tok.c_str()));
  }
  return out;
}

bool read_floats(const std::string& path, float* dst, size_t n, std::string* err) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) { *err = "cannot open data file " + path; return false; }
  size_t got = fread(dst, sizeof(float), n, f);
  fclose(f);
  if (got != n) { *err = "data file " + path + " is shorter than its header says"; return false; }
  return true;
}

bool write_floats(const std::string& path, const float* src, size_t n) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) return false;
  size_t put = fwrite(src, sizeof(float), n, f);
  fclose(f);
  return put == n;
}

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// "<prefix>_iter_<t>" images at the save interval (OsemSinogram3d.cpp:266-276,
// MlemSinogram3d.cpp:244-251, Mlem2d.cpp:187-198), written from the drivers'
// iteration hook while a reconstruction runs.
struct IterationSaver {
  SizeImage size;
  std::string prefix;
  bool ok = true;
  static void save(int t, const float* h_image, int64_t n, void* user) {
    auto* self = static_cast<IterationSaver*>(user);
    Image img(self->size);
    if ((int64_t)img.getPixelCount() != n) { self->ok = false; return; }
    std::memcpy(img.getPixelsPtr(), h_image, (size_t)n * sizeof(float));
    self->ok = img.writeInterfile((self->prefix + "_iter_" + std::to_string(t)).c_str()) && self->ok;
  }
};

// Installs the saver for the lifetime of one driver call (interval 0: none).
struct HookScope {
  HookScope(IterationSaver* saver, int interval) {
    apirl_set_iteration_hook(interval > 0 ? &IterationSaver::save : nullptr, interval > 0 ? interval : 0, saver);
  }
  ~HookScope() { apirl_set_iteration_hook(nullptr, 0, nullptr); }
};

}  // namespace

// ---- key readers -------------------------------------------------------------
int interfile_read(const char* header, const char* key, std::string* value) {
  std::ifstream in(header);
  if (!in) return 3;
  std::string line;
  if (!std::getline(in, line) || line.compare(0, 10, "!INTERFILE") != 0) return 4;
  int count = 0;
  while (std::getline(in, line)) {
    if (!line.empty() && line[0] == ';') continue;
    std::string k, v;
    if (!split_line(line, &k, &v)) continue;
    if (k.compare(0, 17, "!END OF INTERFILE") == 0) break;
    if (k == key) { *value = v; count++; }
  }
  if (count == 0) return 2;
  return count > 1 ? 1 : 0;
}

int parametersFile_read(const char* file, const char* command, const char* key, std::string* value) {
  std::ifstream in(file);
  if (!in) return 3;
  std::string line;
  if (!std::getline(in, line)) return 4;
  std::string first = std::string(command) + " Parameters :=";
  if (line.compare(0, first.size(), first) != 0) return 5;
  int count = 0;
  while (std::getline(in, line)) {
    std::string l = trim(line);
    if (l.empty() || l[0] == ';') continue;
    std::string k, v;
    if (!split_line(l, &k, &v)) continue;
    if (k == "END") break;
    if (k == key) { *value = v; count++; }
  }
  if (count == 0) return 2;
  return count > 1 ? 1 : 0;
}

// ---- Image -------------------------------------------------------------------
Image::Image() { SizeImage s{2, 1, 1, 1, 1.f, 1.f, 1.f}; init(s); }
Image::Image(SizeImage s) { init(s); }
Image::Image(Image* c) : size(c->size), pixels(c->pixels), fovRadio_mm(c->fovRadio_mm), fovHeight_mm(c->fovHeight_mm) {}
Image::Image(const std::string& header) {
  SizeImage s{2, 1, 1, 1, 1.f, 1.f, 1.f};
  init(s);
  readFromInterfile(header.c_str());
}

void Image::init(SizeImage s) {
  size = s;
  if (size.nDimensions == 2) size.nPixelsZ = 1;  // Images.cpp:40-44
  pixels.assign((size_t)size.nPixelsX * size.nPixelsY * size.nPixelsZ, 0.f);
  fovHeight_mm = size.sizePixelZ_mm * size.nPixelsZ;          // Images.cpp:54
  fovRadio_mm = (size.sizePixelX_mm * size.nPixelsX) / 2;     // Images.cpp:55
}

void Image::fillConstant(float v) { std::fill(pixels.begin(), pixels.end(), v); }

int Image::forcePositive() {
  int n = 0;
  for (float& p : pixels) if (p < 0) { p = 0; n++; }
  return n;
}

float Image::getMinValue() const {
  float mn = std::numeric_limits<float>::max();
  for (float p : pixels) if (p != 0 && p < mn) mn = p;
  return mn;
}

float Image::getMaxValue() const {
  float mx = pixels.empty() ? 0.f : pixels[0];
  for (float p : pixels) if (p > mx) mx = p;
  return mx;
}

apirl_image_geom Image::geom() const {
  return apirl_image_geom{size.nPixelsX, size.nPixelsY, size.nPixelsZ, size.sizePixelX_mm, size.sizePixelY_mm,
                          size.sizePixelZ_mm};
}

// Interfile image: the keys medcon writes for a 3D float image
// (data/medcon/m-intf.c MdcWriteIntfHeader): matrix size / scaling factor per
// axis, short float, 4 bytes per pixel, little endian.
bool Image::readFromInterfile(const char* header) {
  std::string v;
  int nx = 0, ny = 0, nz = 1;
  float dx = 1, dy = 1, dz = 1;
  int e = interfile_read(header, "!matrix size [1]", &v);
  if (e == 3 || e == 4) { strError = std::string("cannot read interfile header ") + header; return false; }
  if (e) { strError = "missing !matrix size [1]"; return false; }
  nx = atoi(v.c_str());
  if (interfile_read(header, "!matrix size [2]", &v)) { strError = "missing !matrix size [2]"; return false; }
  ny = atoi(v.c_str());
  if (!interfile_read(header, "!matrix size [3]", &v)) nz = atoi(v.c_str());
  else if (!interfile_read(header, "!number of slices", &v)) nz = atoi(v.c_str());
  else if (!interfile_read(header, "!total number of images", &v)) nz = atoi(v.c_str());
  if (!interfile_read(header, "scaling factor (mm/pixel) [1]", &v)) dx = (float)atof(v.c_str());
  if (!interfile_read(header, "scaling factor (mm/pixel) [2]", &v)) dy = (float)atof(v.c_str());
  if (!interfile_read(header, "scaling factor (mm/pixel) [3]", &v)) dz = (float)atof(v.c_str());
  if (!interfile_read(header, "!number format", &v) && v != "short float" && v != "float") {
    strError = "only float images are supported (number format " + v + ")";
    return false;
  }
  std::string dataName;
  if (interfile_read(header, "!name of data file", &dataName)) { strError = "missing !name of data file"; return false; }
  if (nx <= 0 || ny <= 0 || nz <= 0) { strError = "bad image size in header"; return false; }
  SizeImage s{nz > 1 ? 3 : 2, nx, ny, nz, dx, dy, dz};
  init(s);
  if (nz == 1) { size.nPixelsZ = 1; size.sizePixelZ_mm = dz; fovHeight_mm = dz; }
  return read_floats(data_path(header, dataName), pixels.data(), pixels.size(), &strError);
}

bool Image::writeInterfile(const char* path) const {
  std::string hdr = std::string(path) + ".h33", dat = std::string(path) + ".i33";
  std::ofstream f(hdr);
  if (!f) { strError = "cannot create " + hdr; return false; }
  f << "!INTERFILE :=\r\n!imaging modality := nucmed\r\n!originating system := apirl_b200\r\n"
    << "!version of keys := 3.3\r\n!name of data file := " << base_of(dat) << "\r\n"
    << "!GENERAL IMAGE DATA :=\r\n!type of data := Tomographic\r\nimagedata byte order := LITTLEENDIAN\r\n"
    << "number of dimensions := 3\r\n"
    << "!matrix size [1] := " << size.nPixelsX << "\r\nmatrix axis label [1] := x\r\n"
    << "scaling factor (mm/pixel) [1] := " << size.sizePixelX_mm << "\r\n"
    << "!matrix size [2] := " << size.nPixelsY << "\r\nmatrix axis label [2] := y\r\n"
    << "scaling factor (mm/pixel) [2] := " << size.sizePixelY_mm << "\r\n"
    << "!matrix size [3] := " << size.nPixelsZ << "\r\nmatrix axis label [3] := z\r\n"
    << "scaling factor (mm/pixel) [3] := " << size.sizePixelZ_mm << "\r\n"
    << "!number format := short float\r\n!number of bytes per pixel := 4\r\n"
    << "!number of slices := " << size.nPixelsZ << "\r\n!END OF INTERFILE :=\r\n";
  f.close();
  if (!write_floats(dat, pixels.data(), pixels.size())) { strError = "cannot write " + dat; return false; }
  return true;
}

// ---- Sinogram2D --------------------------------------------------------------
Sinogram2D::Sinogram2D(int nProj, int nR, float rFov, float rScanner)
    : numProj(nProj), numR(nR), radioFov_mm(rFov), radioScanner_mm(rScanner), bins((size_t)nProj * nR, 0.f) {}

bool Sinogram2D::FillConstant(float v) { std::fill(bins.begin(), bins.end(), v); return true; }

void Sinogram2D::inverseDivideBinToBin(const Sinogram2D* m) {
  for (size_t i = 0; i < bins.size(); i++) {
    float num = m->bins[i], den = bins[i];
    bins[i] = (num != 0 && den != 0) ? num / den : 0.f;
  }
}
void Sinogram2D::addBinToBin(const Sinogram2D* a) { for (size_t i = 0; i < bins.size(); i++) bins[i] = bins[i] + a->bins[i]; }
void Sinogram2D::multiplyBinToBin(const Sinogram2D* a) { for (size_t i = 0; i < bins.size(); i++) bins[i] = bins[i] * a->bins[i]; }

float Sinogram2D::getLikelihoodValue(const Sinogram2D* ref) const {
  double l = 0;
  for (size_t i = 0; i < bins.size(); i++)
    if (bins[i] > 0) l += (double)ref->bins[i] * std::log((double)bins[i]) - (double)bins[i];
  return (float)l;
}

// 2D sinogram interfile: matrix size [1] = r, [2] = angles (Sinogram2D.cpp:415-517).
bool Sinogram2D::readFromInterfile(const char* header) {
  std::string v, dataName;
  if (interfile_read(header, "!matrix size [1]", &v)) { strError = "missing !matrix size [1]"; return false; }
  int nr = atoi(v.c_str());
  if (interfile_read(header, "!matrix size [2]", &v)) { strError = "missing !matrix size [2]"; return false; }
  int np = atoi(v.c_str());
  if (interfile_read(header, "!name of data file", &dataName)) { strError = "missing !name of data file"; return false; }
  numR = nr; numProj = np;
  bins.assign((size_t)nr * np, 0.f);
  return read_floats(data_path(header, dataName), bins.data(), bins.size(), &strError);
}

bool Sinogram2D::writeInterfile(const char* path) const {
  std::string hdr = std::string(path) + ".h33", dat = std::string(path) + ".i33";
  std::ofstream f(hdr);
  if (!f) return false;
  f << "!INTERFILE :=\r\n!imaging modality := nucmed\r\n!originating system := apirl_b200\r\n"
    << "!version of keys := 3.3\r\n!name of data file := " << base_of(dat) << "\r\n"
    << "!GENERAL IMAGE DATA :=\r\n!type of data := Tomographic\r\n!total number of images := 1\r\n"
    << "imagedata byte order := LITTLEENDIAN\r\n!matrix size [1] := " << numR << "\r\n!matrix size [2] := "
    << numProj << "\r\n!number format := short float\r\n!number of bytes per pixel := 4\r\n"
    << "!number of projections := 1\r\n!extent of rotation := 180\r\n!END OF INTERFILE :=\r\n";
  f.close();
  return write_floats(dat, bins.data(), bins.size());
}

Sinogram2DinCylindrical3Dpet::Sinogram2DinCylindrical3Dpet(const char* header, float rFov, float rScanner)
    : Sinogram2D(1, 1, rFov, rScanner) {
  readFromInterfile(header);
}

// ---- Sinogram3D --------------------------------------------------------------
Sinogram3D::Sinogram3D(int nProj, int nR, int nRings, float rFov, float axialFov, float rScanner,
                       const std::vector<int>& mn, const std::vector<int>& mx)
    : numProj(nProj), numProjSubset(nProj), numR(nR), numRings(nRings), numSinos(0), radioFov_mm(rFov),
      axialFov_mm(axialFov), radioScanner_mm(rScanner), minRD(mn), maxRD(mx) {
  apirl_sino3d_geom g = geom();
  numSinos = std::max(0, apirl_sino3d_ring_z(&g, nullptr));
  // Sinograms per segment, enumerated as Sinogram3D::readFromInterfile does.
  sinosPerSegment.clear();
  for (size_t s = 0; s < minRD.size(); s++) {
    int n = 0;
    for (int z1 = 0; z1 < 2 * numRings; z1++) {
      bool hit = false;
      int z1a = z1;
      for (int z2 = 0; z2 < numRings; z2++, z1a--)
        if (z1a - z2 <= maxRD[s] && z1a - z2 >= minRD[s] && z1a >= 0 && z1a < numRings) hit = true;
      n += hit;
    }
    sinosPerSegment.push_back(n);
  }
  bins.assign((size_t)numSinos * numProj * numR, 0.f);
}

apirl_sino3d_geom Sinogram3D::geom() const {
  return apirl_sino3d_geom{numProj, numR, numRings, (int)minRD.size(), radioFov_mm, axialFov_mm, radioScanner_mm,
                           minRD.data(), maxRD.data(), scanner()};
}

bool Sinogram3D::FillConstant(float v) { std::fill(bins.begin(), bins.end(), v); return true; }

void Sinogram3D::inverseDivideBinToBin(const Sinogram3D* m) {
  for (size_t i = 0; i < bins.size(); i++) {
    float num = m->bins[i], den = bins[i];
    bins[i] = (num != 0 && den != 0) ? num / den : 0.f;
  }
}
void Sinogram3D::addBinToBin(const Sinogram3D* a) { for (size_t i = 0; i < bins.size(); i++) bins[i] = bins[i] + a->bins[i]; }
void Sinogram3D::multiplyBinToBin(const Sinogram3D* a) { for (size_t i = 0; i < bins.size(); i++) bins[i] = bins[i] * a->bins[i]; }

float Sinogram3D::getLikelihoodValue(const Sinogram3D* ref) const {
  double l = 0;
  for (size_t i = 0; i < bins.size(); i++)
    if (bins[i] != 0) l += (double)ref->bins[i] * std::log((double)bins[i]) - (double)bins[i];
  return (float)l;
}

Sinogram3D* Sinogram3D::getSubset(int s, int S) const {
  Sinogram3D* o = Copy();  // keeps the scanner type
  int nk = (int)std::floor((float)numProj / (float)S);
  if ((numProj % S) > s) nk++;
  o->numProjSubset = nk;
  o->subset = s;
  o->nsubsets = S;
  o->bins.assign((size_t)numSinos * nk * numR, 0.f);
  for (int g = 0; g < numSinos; g++)
    for (int k = 0; k < nk; k++)
      memcpy(&o->bins[((size_t)g * nk + k) * numR], &bins[((size_t)g * numProj + s + S * k) * numR],
             sizeof(float) * numR);
  return o;
}

// 3D sinogram interfile with the keys Sinogram3D::writeInterfile writes and
// readFromInterfile reads (data/src/Sinogram3D.cpp:106-471, :609-748).
bool Sinogram3D::readFromInterfile(const char* header) {
  std::string v, dataName;
  if (interfile_read(header, "!name of data file", &dataName)) { strError = "missing !name of data file"; return false; }
  if (interfile_read(header, "number of dimensions", &v) || atoi(v.c_str()) != 4) {
    strError = "a 3D sinogram has four dimensions";
    return false;
  }
  if (interfile_read(header, "!matrix size [4]", &v)) { strError = "missing !matrix size [4]"; return false; }
  int nseg = atoi(v.c_str());
  std::vector<int> nsin, mn, mx;
  if (interfile_read(header, "!matrix size [3]", &v)) { strError = "missing !matrix size [3]"; return false; }
  nsin = parse_list(v);
  if (interfile_read(header, "minimum ring difference per segment", &v)) { strError = "missing minimum ring difference"; return false; }
  mn = parse_list(v);
  if (interfile_read(header, "maximum ring difference per segment", &v)) { strError = "missing maximum ring difference"; return false; }
  mx = parse_list(v);
  if ((int)nsin.size() != nseg || (int)mn.size() != nseg || (int)mx.size() != nseg) {
    strError = "segment lists do not match the number of segments";
    return false;
  }
  if (interfile_read(header, "!matrix size [2]", &v)) { strError = "missing !matrix size [2]"; return false; }
  int np = atoi(v.c_str());
  if (interfile_read(header, "!matrix size [1]", &v)) { strError = "missing !matrix size [1]"; return false; }
  int nr = atoi(v.c_str());
  int rings = interfile_read(header, "number of rings", &v) ? (nsin[0] + 1) / 2 : atoi(v.c_str());
  Sinogram3D fresh(np, nr, rings, radioFov_mm, axialFov_mm, radioScanner_mm, mn, mx);
  for (int s = 0; s < nseg; s++)
    if (fresh.sinosPerSegment[s] != nsin[s]) {
      strError = "sinograms per segment do not match the ring differences";
      return false;
    }
  *this = fresh;
  return read_floats(data_path(header, dataName), bins.data(), bins.size(), &strError);
}

bool Sinogram3D::writeInterfile(const char* path) const {
  std::string hdr = std::string(path) + ".h33", dat = std::string(path) + ".i33";
  std::ofstream f(hdr);
  if (!f) return false;
  const char* e = "\r\n";
  f << "!INTERFILE :=" << e << "!imaging modality := nucmed" << e << "!originating system := apirl_b200" << e
    << "!version of keys := 3.3" << e << "!name of data file := " << base_of(dat) << e
    << "!GENERAL IMAGE DATA :=" << e << "!type of data := PET" << e << "!imagedata byte order := LITTLEENDIAN" << e
    << "!number format := short float" << e << "!number of bytes per pixel := 4" << e
    << "number of dimensions := 4" << e << "matrix axis label [4] := segment" << e
    << "!matrix size [4] := " << minRD.size() << e << "matrix axis label [2] := view" << e
    << "!matrix size [2] := " << numProjSubset << e << "matrix axis label [1] := tangential coordinate" << e
    << "!matrix size [1] := " << numR << e << "matrix axis label [3] := axial coordinate" << e
    << "!matrix size [3] := {";
  for (size_t i = 0; i < sinosPerSegment.size(); i++) f << (i ? "," : "") << sinosPerSegment[i];
  f << "}" << e << "minimum ring difference per segment := {";
  for (size_t i = 0; i < minRD.size(); i++) f << (i ? "," : "") << minRD[i];
  f << "}" << e << "maximum ring difference per segment := {";
  for (size_t i = 0; i < maxRD.size(); i++) f << (i ? "," : "") << maxRD[i];
  f << "}" << e << "number of rings := " << numRings << e << "!END OF INTERFILE :=" << e;
  f.close();
  return write_floats(dat, bins.data(), bins.size());
}

Sinogram3DCylindricalPet::Sinogram3DCylindricalPet(const char* header, float rFov, float zFov, float rScanner)
    : Sinogram3D(1, 1, 1, rFov, zFov, rScanner, {0}, {0}) {
  readFromInterfile(header);
}

// Sinogram3DSiemensMmr(header) (data/src/Sinogram3DSiemensMmr.cpp): the mMR's
// fixed field of view (594 mm / 260 mm) and radius (328 mm).
Sinogram3DSiemensMmr::Sinogram3DSiemensMmr(const char* header)
    : Sinogram3D(1, 1, 1, 594.0f / 2.0f, 260.0f, 656.0f / 2.0f, {0}, {0}) {
  readFromInterfile(header);
}

// ---- CuSiddonProjector ---------------------------------------------------------
struct CuSiddonProjector::State {
  apirl_projector* p = nullptr;
  bool is3d = false;
  apirl_image_geom ig{};
  std::vector<int> mn, mx;
  int np = 0, nr = 0, rings = 0;
  float rfov = 0, afov = 0, rsc = 0;
  float *d_img = nullptr, *d_a = nullptr, *d_b = nullptr;
  size_t nimg = 0, nsino = 0;
  cudaStream_t stream = nullptr;
  int ns = 1, nas = 1, multi = 0;  // sampling applied to p
  int scanner = APIRL_SCANNER_CYLINDRICAL;
};

CuSiddonProjector::CuSiddonProjector(int nSamples, int nAxialSamples, int gpuId)
    : st(new State), device(gpuId), numSamplesOnDetector(nSamples), numAxialSamplesOnDetector(nAxialSamples) {}

CuSiddonProjector::~CuSiddonProjector() {
  release();
  delete st;
}

// Frees the projector and buffers set up on `device`; the next call sets up again.
void CuSiddonProjector::release() {
  if (st->p) apirl_projector_destroy(st->p);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  cudaFree(st->d_img);
  cudaFree(st->d_a);
  cudaFree(st->d_b);
  if (st->stream) cudaStreamDestroy(st->stream);
  cudaSetDevice(prev);
  *st = State();
}

bool CuSiddonProjector::setGpuId(int id) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || id < 0 || id >= n) {
    strError = "no GPU with index " + std::to_string(id);
    return false;
  }
  if (id != device) {
    release();
    device = id;
  }
  return true;
}

static bool same_img(const apirl_image_geom& a, const apirl_image_geom& b) {
  return a.nx == b.nx && a.ny == b.ny && a.nz == b.nz && a.dx == b.dx && a.dy == b.dy && a.dz == b.dz;
}

bool CuSiddonProjector::prepare2d(const Image* img, const Sinogram2D* s) {
  apirl_image_geom ig = img->geom();
  apirl_sino2d_geom sg = s->geom();
  if (st->p && !st->is3d && same_img(ig, st->ig) && st->np == sg.n_proj && st->nr == sg.n_r && st->rfov == sg.r_fov &&
      st->rsc == sg.r_scanner)
    return true;
  if (st->p) apirl_projector_destroy(st->p);
  st->p = nullptr;
  if (apirl_projector_create_2d(&ig, &sg, device, &st->p) != APIRL_OK) { strError = apirl_last_error(); return false; }
  st->is3d = false; st->ig = ig; st->np = sg.n_proj; st->nr = sg.n_r; st->rfov = sg.r_fov; st->rsc = sg.r_scanner;
  return true;
}

bool CuSiddonProjector::prepare3d(const Image* img, const Sinogram3D* s) {
  apirl_image_geom ig = img->geom();
  if (!(st->p && st->is3d && same_img(ig, st->ig) && st->np == s->getNumProjFull() && st->nr == s->getNumR() &&
        st->rings == s->getNumRings() && st->rfov == s->getRadioFov_mm() && st->afov == s->getAxialFoV_mm() &&
        st->rsc == s->getRadioScanner_mm() && st->mn == s->minRingDiff() && st->mx == s->maxRingDiff() &&
        st->scanner == s->scanner())) {
    if (st->p) apirl_projector_destroy(st->p);
    st->p = nullptr;
    apirl_sino3d_geom sg = s->geom();
    if (apirl_projector_create_3d(&ig, &sg, device, &st->p) != APIRL_OK) { strError = apirl_last_error(); return false; }
    st->is3d = true; st->ig = ig; st->np = s->getNumProjFull(); st->nr = s->getNumR(); st->rings = s->getNumRings();
    st->rfov = s->getRadioFov_mm(); st->afov = s->getAxialFoV_mm(); st->rsc = s->getRadioScanner_mm();
    st->mn = s->minRingDiff(); st->mx = s->maxRingDiff();
    st->scanner = s->scanner();
    st->ns = 1; st->nas = 1; st->multi = 0;
  }
  // Rays per bin: the constructor's sample counts and the current
  // useMultipleLorsPerBin flag, which callers may change between calls.
  const int multi = useMultipleLorsPerBin ? 1 : 0;
  if (st->ns != numSamplesOnDetector || st->nas != numAxialSamplesOnDetector || st->multi != multi) {
    if (apirl_projector_set_sampling(st->p, numSamplesOnDetector, numAxialSamplesOnDetector, multi) != APIRL_OK) {
      strError = apirl_last_error();
      return false;
    }
    st->ns = numSamplesOnDetector; st->nas = numAxialSamplesOnDetector; st->multi = multi;
  }
  return true;
}

// op: 0 project (a = unused, out_sino written), 1 backproject (a), 2 divide-and-backproject (a / b).
bool CuSiddonProjector::run(int op, Image* img, const float* a, const float* b, float* out_sino, size_t nbins,
                            int subset, int nsub) {
  int prev = 0;
  cudaGetDevice(&prev);
  struct Restore { int d; ~Restore() { cudaSetDevice(d); } } restore{prev};
  if (cudaSetDevice(device) != cudaSuccess) { strError = "cudaSetDevice failed"; return false; }
  if (!st->stream && cudaStreamCreateWithFlags(&st->stream, cudaStreamNonBlocking) != cudaSuccess) {
    strError = "cudaStreamCreate failed";
    return false;
  }
  const size_t nv = (size_t)img->getPixelCount();
  auto grow = [&](float** p, size_t* have, size_t n) {
    if (*have >= n) return true;
    cudaFree(*p);
    *p = nullptr;
    if (cudaMalloc(p, n * sizeof(float)) != cudaSuccess) return false;
    *have = n;
    return true;
  };
  size_t dummy = st->nsino;
  if (!grow(&st->d_img, &st->nimg, nv) || !grow(&st->d_a, &dummy, nbins)) { strError = "device allocation failed"; return false; }
  if (op == 2) {
    size_t have_b = st->d_b ? st->nsino : 0;
    if (!grow(&st->d_b, &have_b, nbins)) { strError = "device allocation failed"; return false; }
  }
  st->nsino = std::max(st->nsino, nbins);
  cudaStream_t s = st->stream;
  apirl_status rc;
  if (op == 0) {
    cudaMemcpyAsync(st->d_img, img->getPixelsPtr(), nv * sizeof(float), cudaMemcpyHostToDevice, s);
    // 2D bins with r > rFov keep their values (SiddonProjector.cpp:166-173).
    cudaMemcpyAsync(st->d_a, out_sino, nbins * sizeof(float), cudaMemcpyHostToDevice, s);
    rc = apirl_project(st->p, st->d_img, st->d_a, subset, nsub, s);
    if (rc == APIRL_OK) cudaMemcpyAsync(out_sino, st->d_a, nbins * sizeof(float), cudaMemcpyDeviceToHost, s);
  } else {
    cudaMemcpyAsync(st->d_img, img->getPixelsPtr(), nv * sizeof(float), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(st->d_a, a, nbins * sizeof(float), cudaMemcpyHostToDevice, s);
    if (op == 2) cudaMemcpyAsync(st->d_b, b, nbins * sizeof(float), cudaMemcpyHostToDevice, s);
    rc = op == 1 ? apirl_backproject(st->p, st->d_a, st->d_img, subset, nsub, s)
                 : apirl_divide_and_backproject(st->p, st->d_a, st->d_b, st->d_img, subset, nsub, s);
    if (rc == APIRL_OK) cudaMemcpyAsync(img->getPixelsPtr(), st->d_img, nv * sizeof(float), cudaMemcpyDeviceToHost, s);
  }
  if (rc != APIRL_OK) { strError = apirl_last_error(); cudaStreamSynchronize(s); return false; }
  if (cudaStreamSynchronize(s) != cudaSuccess) { strError = cudaGetErrorString(cudaGetLastError()); return false; }
  return true;
}

bool CuSiddonProjector::Project(Image* img, Sinogram2D* s) {
  return prepare2d(img, s) && run(0, img, nullptr, nullptr, s->getSinogramPtr(), (size_t)s->getNumProj() * s->getNumR(), -1, 1);
}
bool CuSiddonProjector::Backproject(Sinogram2D* s, Image* img) {
  return prepare2d(img, s) && run(1, img, s->getSinogramPtr(), nullptr, nullptr, (size_t)s->getNumProj() * s->getNumR(), -1, 1);
}
bool CuSiddonProjector::DivideAndBackproject(Sinogram2D* in, Sinogram2D* est, Image* img) {
  return prepare2d(img, in) &&
         run(2, img, in->getSinogramPtr(), est->getSinogramPtr(), nullptr, (size_t)in->getNumProj() * in->getNumR(), -1, 1);
}
bool CuSiddonProjector::Project(Image* img, Sinogram3D* s) {
  return prepare3d(img, s) &&
         run(0, img, nullptr, nullptr, s->getSinogramPtr(), (size_t)s->getBinCount(), s->subsetIndex(), s->subsetCount());
}
bool CuSiddonProjector::Backproject(Sinogram3D* s, Image* img) {
  return prepare3d(img, s) &&
         run(1, img, s->getSinogramPtr(), nullptr, nullptr, (size_t)s->getBinCount(), s->subsetIndex(), s->subsetCount());
}
bool CuSiddonProjector::DivideAndBackproject(Sinogram3D* in, Sinogram3D* est, Image* img) {
  return prepare3d(img, in) && run(2, img, in->getSinogramPtr(), est->getSinogramPtr(), nullptr,
                                   (size_t)in->getBinCount(), in->subsetIndex(), in->subsetCount());
}

// Device-buffer calls (CuProjector).  op: 0 project d_a -> d_out (sinogram),
// 1 backproject d_a into d_out (image), 2 divide d_a by d_b and backproject.
bool CuSiddonProjector::runDevice(int op, const float* d_a, const float* d_b, float* d_out, Image* img,
                                  Sinogram3D* s, bool copyResult) {
  if (!img || !s || !d_a || !d_out || (op == 2 && !d_b)) {
    strError = "null image, sinogram or device buffer";
    return false;
  }
  int prev = 0;
  cudaGetDevice(&prev);
  struct Restore { int d; ~Restore() { cudaSetDevice(d); } } restore{prev};
  if (cudaSetDevice(device) != cudaSuccess) { strError = "cudaSetDevice failed"; return false; }
  if (!prepare3d(img, s)) return false;
  cudaStream_t legacy = 0;
  apirl_status rc;
  if (op == 0)
    rc = apirl_project(st->p, d_a, d_out, s->subsetIndex(), s->subsetCount(), legacy);
  else if (op == 1)
    rc = apirl_backproject(st->p, d_a, d_out, s->subsetIndex(), s->subsetCount(), legacy);
  else
    rc = apirl_divide_and_backproject(st->p, d_a, d_b, d_out, s->subsetIndex(), s->subsetCount(), legacy);
  if (rc != APIRL_OK) { strError = apirl_last_error(); cudaStreamSynchronize(legacy); return false; }
  if (copyResult) {
    cudaError_t e = op == 0 ? cudaMemcpy(s->getSinogramPtr(), d_out, (size_t)s->getBinCount() * sizeof(float),
                                         cudaMemcpyDeviceToHost)
                            : cudaMemcpy(img->getPixelsPtr(), d_out, (size_t)img->getPixelCount() * sizeof(float),
                                         cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { strError = cudaGetErrorString(e); return false; }
  }
  cudaError_t e = cudaStreamSynchronize(legacy);
  if (e != cudaSuccess) { strError = cudaGetErrorString(e); return false; }
  return true;
}

bool CuSiddonProjector::Project(float* d_image, float* d_projection, float*, float*, Image* inputImage,
                                Sinogram3D* outputSinogram, bool copyResult) {
  return runDevice(0, d_image, nullptr, d_projection, inputImage, outputSinogram, copyResult);
}
bool CuSiddonProjector::Backproject(float* d_inputSinogram, float* d_outputImage, float*, float*,
                                    Sinogram3D* inputSinogram, Image* outputImage, bool copyResult) {
  return runDevice(1, d_inputSinogram, nullptr, d_outputImage, outputImage, inputSinogram, copyResult);
}
bool CuSiddonProjector::DivideAndBackproject(float* d_inputSinogram, float* d_estimatedSinogram,
                                             float* d_outputImage, float*, float*, Sinogram3D* inputSinogram,
                                             Image* outputImage, bool copyResult) {
  return runDevice(2, d_inputSinogram, d_estimatedSinogram, d_outputImage, outputImage, inputSinogram, copyResult);
}

// ---- CuProjector / CuProjectorInterface ------------------------------------------
CuProjector::CuProjector() : gridSize(1, 1, 1), blockSize(128, 1, 1) {}

CuProjector::CuProjector(unsigned int bx, unsigned int by, unsigned int bz, unsigned int gx, unsigned int gy,
                         unsigned int gz) {
  setKernelConfig(bx, by, bz, gx, gy, gz);
}

void CuProjector::setKernelConfig(unsigned int bx, unsigned int by, unsigned int bz, unsigned int gx,
                                  unsigned int gy, unsigned int gz) {
  blockSize = dim3(bx, by, bz);
  gridSize = dim3(gx, gy, gz);
  threads_per_block = bx * by * bz;
}

CuProjectorInterface::CuProjectorInterface(CuProjector* p) : projector(p), blockSizeProjector(128, 1, 1) {}

CuProjectorInterface::~CuProjectorInterface() { release(); }

void CuProjectorInterface::release() {
  if (bufDevice >= 0) {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(bufDevice);
    cudaFree(d_image);
    cudaFree(d_projection);
    cudaFree(d_estimated);
    cudaFree(d_ring1_mm);
    cudaFree(d_ring2_mm);
    cudaSetDevice(prev);
  }
  d_image = d_projection = d_estimated = d_ring1_mm = d_ring2_mm = nullptr;
  nImage = nBins = nEstimated = nSinos = 0;
  bufDevice = -1;
}

void CuProjectorInterface::setProjectorKernelConfig(unsigned int x, unsigned int y, unsigned int z,
                                                    Sinogram3D* sinogram) {
  blockSizeProjector = dim3(x, y, z);
  const unsigned int per = (unsigned int)(sinogram->getNumProj() * sinogram->getNumR());
  const unsigned int gx = x ? (per + x - 1) / x : 1;
  if (projector) projector->setKernelConfig(x, y, z, gx, (unsigned int)sinogram->getNumSinograms(), 1);
}

void CuProjectorInterface::setProjectorKernelConfig(dim3 b, Sinogram3D* sinogram) {
  setProjectorKernelConfig(b.x, b.y, b.z, sinogram);
}

bool CuProjectorInterface::setGpuId(int id) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || id < 0 || id >= n) {
    strError = "no GPU with index " + std::to_string(id);
    return false;
  }
  gpuId = id;
  return true;
}

bool CuProjectorInterface::Project(Image*, Sinogram2D*) {
  strError = "CuProjectorInterface projects Sinogram3D only";
  return false;
}
bool CuProjectorInterface::Backproject(Sinogram2D*, Image*) {
  strError = "CuProjectorInterface backprojects Sinogram3D only";
  return false;
}
bool CuProjectorInterface::DivideAndBackproject(Sinogram2D*, Sinogram2D*, Image*) {
  strError = "CuProjectorInterface backprojects Sinogram3D only";
  return false;
}

// Device buffers for `s` and `img` on gpuId (grown, never shrunk), the ring
// arrays filled, the CuProjector on the same GPU and its launch shape set.
bool CuProjectorInterface::prepare(Sinogram3D* s, Image* img, bool estimate) {
  if (!projector || !s || !img) { strError = "null projector, image or sinogram"; return false; }
  if (auto* sp = dynamic_cast<CuSiddonProjector*>(projector)) {
    if (!sp->setGpuId(gpuId)) { strError = sp->getError(); return false; }
  }
  if (bufDevice != gpuId) release();
  if (cudaSetDevice(gpuId) != cudaSuccess) { strError = "cudaSetDevice failed"; return false; }
  bufDevice = gpuId;
  auto grow = [](float** p, size_t* have, size_t n) {
    if (*have >= n) return true;
    cudaFree(*p);
    *p = nullptr;
    *have = 0;
    if (cudaMalloc(p, n * sizeof(float)) != cudaSuccess) return false;
    *have = n;
    return true;
  };
  const size_t nsino = (size_t)s->getNumSinograms();
  const bool newRings = nsino != nSinos || !d_ring1_mm;
  if (!grow(&d_image, &nImage, (size_t)img->getPixelCount()) || !grow(&d_projection, &nBins, (size_t)s->getBinCount()) ||
      (estimate && !grow(&d_estimated, &nEstimated, (size_t)s->getBinCount()))) {
    strError = "device allocation failed";
    return false;
  }
  // Axial end points per sinogram (the reference's d_ring1_mm / d_ring2_mm,
  // CuProjectorInterface.cu:243-275), rebuilt on every call: the geometry
  // may change between calls with the same sinogram count.
  apirl_sino3d_geom g = s->geom();
  std::vector<float> z((size_t)2 * nsino);
  if (apirl_sino3d_ring_z(&g, z.data()) != (int)nsino) { strError = apirl_last_error(); return false; }
  std::vector<float> z1(nsino), z2(nsino);
  for (size_t i = 0; i < nsino; i++) { z1[i] = z[2 * i]; z2[i] = z[2 * i + 1]; }
  if (newRings) {
    cudaFree(d_ring1_mm);
    cudaFree(d_ring2_mm);
    d_ring1_mm = d_ring2_mm = nullptr;
    nSinos = 0;
    if (cudaMalloc(&d_ring1_mm, nsino * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&d_ring2_mm, nsino * sizeof(float)) != cudaSuccess) {
      strError = "device allocation failed";
      return false;
    }
    nSinos = nsino;
  }
  if (cudaMemcpy(d_ring1_mm, z1.data(), nsino * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(d_ring2_mm, z2.data(), nsino * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
    strError = "copy of the ring arrays failed";
    return false;
  }
  setProjectorKernelConfig(blockSizeProjector, s);
  return true;
}

namespace {
const char* projector_error(CuProjector* p) {
  auto* q = dynamic_cast<Projector*>(p);
  return q && q->getError()[0] ? q->getError() : "the CuProjector call failed";
}
}  // namespace

bool CuProjectorInterface::Project(Image* img, Sinogram3D* s) {
  int prev = 0;
  cudaGetDevice(&prev);
  struct Restore { int d; ~Restore() { cudaSetDevice(d); } } restore{prev};
  if (!prepare(s, img, false)) return false;
  const size_t nb = (size_t)s->getBinCount();
  if (cudaMemcpy(d_image, img->getPixelsPtr(), (size_t)img->getPixelCount() * sizeof(float),
                 cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(d_projection, 0, nb * sizeof(float)) != cudaSuccess) {
    strError = "copy to the device failed";
    return false;
  }
  if (!projector->Project(d_image, d_projection, d_ring1_mm, d_ring2_mm, img, s, false)) {
    strError = projector_error(projector);
    return false;
  }
  if (cudaMemcpy(s->getSinogramPtr(), d_projection, nb * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
    strError = "copy from the device failed";
    return false;
  }
  return true;
}

bool CuProjectorInterface::Backproject(Sinogram3D* s, Image* img) { return DivideAndBackproject(s, nullptr, img); }

bool CuProjectorInterface::DivideAndBackproject(Sinogram3D* s, Sinogram3D* est, Image* img) {
  int prev = 0;
  cudaGetDevice(&prev);
  struct Restore { int d; ~Restore() { cudaSetDevice(d); } } restore{prev};
  if (est && est->getBinCount() != (s ? s->getBinCount() : -1)) {
    strError = "the estimated sinogram has another size";
    return false;
  }
  if (!prepare(s, img, est != nullptr)) return false;
  const size_t nb = (size_t)s->getBinCount(), nv = (size_t)img->getPixelCount();
  if (cudaMemcpy(d_projection, s->getSinogramPtr(), nb * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
      (est && cudaMemcpy(d_estimated, est->getSinogramPtr(), nb * sizeof(float), cudaMemcpyHostToDevice) !=
                  cudaSuccess) ||
      cudaMemset(d_image, 0, nv * sizeof(float)) != cudaSuccess) {
    strError = "copy to the device failed";
    return false;
  }
  const bool ok = est ? projector->DivideAndBackproject(d_projection, d_estimated, d_image, d_ring1_mm, d_ring2_mm, s,
                                                        img, false)
                      : projector->Backproject(d_projection, d_image, d_ring1_mm, d_ring2_mm, s, img, false);
  if (!ok) { strError = projector_error(projector); return false; }
  if (cudaMemcpy(img->getPixelsPtr(), d_image, nv * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
    strError = "copy from the device failed";
    return false;
  }
  return true;
}

// ---- Mlem ----------------------------------------------------------------------
Mlem::Mlem(Image* init, std::string path, std::string prefix, int iters, int saveInterval, bool saveInter,
           bool sensFromFile, Projector* fwd, Projector* back)
    : initialEstimate(init), pathSalida(path), outputFilenamePrefix(prefix), numIterations(iters),
      saveIterationInterval(saveInterval), saveIntermediate(saveInter), sensitivityImageFromFile(sensFromFile),
      forwardprojector(fwd), backprojector(back) {
  reconstructionImage = new Image(init->getSize());
  sensitivityImage = new Image(init->getSize());
}

Mlem::~Mlem() {
  delete reconstructionImage;
  delete sensitivityImage;
}

// <prefix>.log with the key/value lines and rows of numbers of Logger
// (data/inc/Logger.h:93-148), wall-clock times instead of clock().
void Mlem::writeLog(const std::string& type, const std::string& input, double totalMs,
                    const std::vector<double>& iterMs) const {
  std::ofstream f(outputFilenamePrefix + ".log");
  if (!f) return;
  f << "######## " << type << " Reconstruction #########\n";
  f << "Name: " << outputFilenamePrefix << "\nType: " << type << "\nIterations: " << numIterations << "\n";
  f << "Input Projections: " << input << "\n";
  SizeImage s = initialEstimate->getSize();
  f << "Image Size: " << s.nPixelsX << "[x] x " << s.nPixelsY << "[y] x " << s.nPixelsZ << "[z]\n";
  f << "Device: GPU (apirl_b200)\n_______RESULTADOS DE RECONSTRUCCION_______\n";
  f << "Tiempo Total de Reconstrucción: " << totalMs << "\n";
  f << "Tiempos de Reconstrucción por Iteración [mseg]\n";
  for (double t : iterMs) f << t << "\t";
  f << "\nLikelihood por Iteración:\n";
  f.precision(12);
  for (double l : likelihood) f << l << "\t";
  f << "\n";
}

// ---- Mlem2d --------------------------------------------------------------------
Mlem2d::Mlem2d(Sinogram2D* in, Image* init, std::string path, std::string prefix, int iters, int saveInterval,
               bool saveInter, bool sensFromFile, Projector* fwd, Projector* back)
    : Mlem(init, path, prefix, iters, saveInterval, saveInter, sensFromFile, fwd, back), inputProjection(in) {
  inputProjection->setRadioFov_mm(init->getFovRadio());  // Mlem2d.cpp:12
}

Mlem2d::~Mlem2d() { delete multiplicative; delete additive; }

bool Mlem2d::setMultiplicativeProjection(const std::string& fn) {
  delete multiplicative;
  multiplicative = inputProjection->Copy();
  return multiplicative->readFromInterfile(fn.c_str());
}
bool Mlem2d::setMultiplicativeProjection(Sinogram2D* s) { delete multiplicative; multiplicative = s->Copy(); return true; }
bool Mlem2d::setAdditiveProjection(const std::string& fn) {
  delete additive;
  additive = inputProjection->Copy();
  return additive->readFromInterfile(fn.c_str());
}
bool Mlem2d::setAdditiveProjection(Sinogram2D* s) { delete additive; additive = s->Copy(); return true; }

bool Mlem2d::Reconstruct() {
  double t0 = now_ms();
  if (!dynamic_cast<CuSiddonProjector*>(forwardprojector) || !dynamic_cast<CuSiddonProjector*>(backprojector)) {
    strError = "Mlem2d runs on the GPU and needs CuSiddonProjector as forward and back projector";
    return false;
  }
  int dev = static_cast<CuSiddonProjector*>(forwardprojector)->gpuId();
  apirl_image_geom ig = initialEstimate->geom();
  apirl_sino2d_geom sg = inputProjection->geom();
  likelihood.assign(numIterations + 1, 0.0);
  // Mlem2d.cpp:95-112: the sensitivity image read from sensitivityFilename
  // (sensitivityImageFromFile), or computed and written.
  Image given;
  if (sensitivityImageFromFile &&
      (!given.readFromInterfile(sensitivityFilename.c_str()) ||
       given.getPixelCount() != initialEstimate->getPixelCount())) {
    strError = "reading the sensitivity image " + sensitivityFilename + " failed";
    return false;
  }
  apirl_recon_options opts{nullptr, sensitivityImageFromFile ? given.getPixelsPtr() : nullptr,
                           sensitivityImage->getPixelsPtr()};
  IterationSaver saver{initialEstimate->getSize(), outputFilenamePrefix};
  HookScope hook(&saver, saveIterationInterval);
  apirl_status rc = apirl_mlem_2d_ex(&ig, &sg, inputProjection->getSinogramPtr(),
                                     multiplicative ? multiplicative->getSinogramPtr() : nullptr,
                                     additive ? additive->getSinogramPtr() : nullptr, initialEstimate->getPixelsPtr(),
                                     numIterations, dev, reconstructionImage->getPixelsPtr(), likelihood.data(), &opts);
  if (rc != APIRL_OK) { strError = apirl_last_error(); return false; }
  if (!saver.ok) { strError = "writing an intermediate image failed"; return false; }
  double t1 = now_ms();
  if (!sensitivityImageFromFile) sensitivityImage->writeInterfile((outputFilenamePrefix + "_sensitivity").c_str());
  reconstructionImage->writeInterfile((outputFilenamePrefix + "_final").c_str());
  writeLog("ML-EM", "2D Sinogram", t1 - t0, {});
  return true;
}

// ---- MlemSinogram3d / OsemSinogram3d -------------------------------------------
MlemSinogram3d::MlemSinogram3d(Sinogram3D* in, Image* init, std::string path, std::string prefix, int iters,
                               int saveInterval, bool saveInter, bool sensFromFile, Projector* fwd, Projector* back)
    : Mlem(init, path, prefix, iters, saveInterval, saveInter, sensFromFile, fwd, back),
      inputProjection(in->Copy()) {}

MlemSinogram3d::~MlemSinogram3d() { delete inputProjection; delete multiplicative; delete additive; }

bool MlemSinogram3d::setMultiplicativeProjection(const std::string& fn) {
  delete multiplicative;
  multiplicative = inputProjection->Copy();
  return multiplicative->readFromInterfile(fn.c_str());
}
bool MlemSinogram3d::setMultiplicativeProjection(Sinogram3D* s) { delete multiplicative; multiplicative = s->Copy(); return true; }
bool MlemSinogram3d::setAdditiveProjection(const std::string& fn) {
  delete additive;
  additive = inputProjection->Copy();
  return additive->readFromInterfile(fn.c_str());
}
bool MlemSinogram3d::setAdditiveProjection(Sinogram3D* s) { delete additive; additive = s->Copy(); return true; }

bool MlemSinogram3d::deviceResident() const {
  return dynamic_cast<CuSiddonProjector*>(forwardprojector) && dynamic_cast<CuSiddonProjector*>(backprojector);
}

// The fused GPU pass walks one set of rays for the projection and the
// backprojection, so both projectors must sample alike.
bool MlemSinogram3d::sameSampling(apirl_sampling* out) {
  const apirl_sampling f = static_cast<CuSiddonProjector*>(forwardprojector)->sampling();
  const apirl_sampling b = static_cast<CuSiddonProjector*>(backprojector)->sampling();
  if (f.n_samples != b.n_samples || f.n_axial_samples != b.n_axial_samples ||
      f.multiple_lors_per_bin != b.multiple_lors_per_bin) {
    strError = "forward and back projectors must use the same samples per bin";
    return false;
  }
  *out = f;
  return true;
}

bool MlemSinogram3d::reconstructOnDevice(int numSubsets) {
  if (!deviceResident()) {
    strError = "the reconstruction runs on the GPU and needs CuSiddonProjector as forward and back projector";
    return false;
  }
  double t0 = now_ms();
  int dev = static_cast<CuSiddonProjector*>(forwardprojector)->gpuId();
  if (static_cast<CuSiddonProjector*>(backprojector)->gpuId() != dev) {
    strError = "forward and back projectors must be on the same GPU";
    return false;
  }
  apirl_image_geom ig = initialEstimate->geom();
  apirl_sino3d_geom sg = inputProjection->geom();
  apirl_sampling sm;
  if (!sameSampling(&sm)) return false;
  const float* mult = multiplicative ? multiplicative->getSinogramPtr() : nullptr;
  const float* add = additive ? additive->getSinogramPtr() : nullptr;
  const int64_t nv = initialEstimate->getPixelCount();
  const int nimg = numSubsets == 0 ? 1 : numSubsets;
  // The sensitivity images: read (sensitivityImageFromFile; OSEM reads
  // "<name>_subset_<s>.h33", OsemSinogram3d.cpp:84-96, ML-EM the named file,
  // MlemSinogram3d.cpp:132-138) or computed by the driver and written.
  std::vector<float> sens((size_t)nimg * nv);
  if (sensitivityImageFromFile) {
    for (int s = 0; s < nimg; s++) {
      const std::string fn =
          numSubsets == 0 ? sensitivityFilename : sensitivityFilename + "_subset_" + std::to_string(s) + ".h33";
      Image im;
      if (!im.readFromInterfile(fn.c_str()) || im.getPixelCount() != nv) {
        strError = "reading the sensitivity image " + fn + " failed";
        return false;
      }
      std::memcpy(sens.data() + (size_t)s * nv, im.getPixelsPtr(), (size_t)nv * sizeof(float));
    }
  }
  apirl_recon_options opts{&sm, sensitivityImageFromFile ? sens.data() : nullptr,
                           sensitivityImageFromFile ? nullptr : sens.data()};
  IterationSaver saver{initialEstimate->getSize(), outputFilenamePrefix};
  HookScope hook(&saver, saveIterationInterval);
  apirl_status rc;
  if (numSubsets == 0) {
    likelihood.assign(numIterations + 1, 0.0);
    rc = apirl_mlem_3d_ex(&ig, &sg, inputProjection->getSinogramPtr(), mult, add, initialEstimate->getPixelsPtr(),
                          numIterations, dev, reconstructionImage->getPixelsPtr(), likelihood.data(), &opts);
  } else {
    likelihood.assign((size_t)numIterations * numSubsets + 1, 0.0);
    rc = apirl_osem_3d_ex(&ig, &sg, inputProjection->getSinogramPtr(), mult, add, initialEstimate->getPixelsPtr(),
                          numIterations, numSubsets, dev, reconstructionImage->getPixelsPtr(), likelihood.data(),
                          &opts);
  }
  if (rc != APIRL_OK) { strError = apirl_last_error(); return false; }
  if (!saver.ok) { strError = "writing an intermediate image failed"; return false; }
  double t1 = now_ms();
  std::memcpy(sensitivityImage->getPixelsPtr(), sens.data(), (size_t)nv * sizeof(float));
  if (!sensitivityImageFromFile) {
    for (int s = 0; s < nimg; s++) {
      Image im(initialEstimate->getSize());
      std::memcpy(im.getPixelsPtr(), sens.data() + (size_t)s * nv, (size_t)nv * sizeof(float));
      im.writeInterfile(
          (outputFilenamePrefix + (numSubsets == 0 ? "_sensitivity" : "_sensitivity_subset_" + std::to_string(s)))
              .c_str());
    }
  }
  reconstructionImage->writeInterfile((outputFilenamePrefix + "_final").c_str());
  writeLog(numSubsets == 0 ? "ML-EM" : "OSEM", "Sinogram3D", t1 - t0, {});
  return true;
}

bool MlemSinogram3d::Reconstruct() { return reconstructOnDevice(0); }

OsemSinogram3d::OsemSinogram3d(Sinogram3D* in, Image* init, std::string path, std::string prefix, int iters,
                               int saveInterval, bool saveInter, bool sensFromFile, Projector* fwd, Projector* back,
                               int nsub)
    : MlemSinogram3d(in, init, path, prefix, iters, saveInterval, saveInter, sensFromFile, fwd, back),
      numSubsets(nsub) {}

bool OsemSinogram3d::Reconstruct() {
  if (numSubsets < 1) { strError = "number of subsets must be >= 1"; return false; }
  return reconstructOnDevice(numSubsets);
}

// ---- CuMlemSinogram3d / CuOsemSinogram3d -----------------------------------------
CuMlemSinogram3d::CuMlemSinogram3d(Sinogram3D* in, Image* init, std::string path, std::string prefix, int iters,
                                   int saveInterval, bool saveInter, bool sensFromFile, CuProjector* fwd,
                                   CuProjector* back)
    : MlemSinogram3d(in, init, path, prefix, iters, saveInterval, saveInter, sensFromFile,
                     dynamic_cast<Projector*>(fwd), dynamic_cast<Projector*>(back)) {}

bool CuMlemSinogram3d::Reconstruct() { return reconstructOnDevice(0); }

bool CuMlemSinogram3d::Reconstruct(TipoProyector tipoProy) {
  if (!deviceResident()) { strError = "CuMlemSinogram3d needs CuSiddonProjector as forward and back projector"; return false; }
  return Reconstruct(tipoProy, static_cast<CuSiddonProjector*>(forwardprojector)->gpuId());
}

bool CuMlemSinogram3d::Reconstruct(TipoProyector tipoProy, int indexGpu) {
  if (tipoProy != SIDDON_CYLINDRICAL_SCANNER && tipoProy != SIDDON_PROJ_TEXT_CYLINDRICAL_SCANNER &&
      tipoProy != SIDDON_BACKPROJ_SURF_CYLINDRICAL_SCANNER) {
    strError = "only the cylindrical-scanner Siddon projector kinds are available";
    return false;
  }
  if (!deviceResident()) { strError = "CuMlemSinogram3d needs CuSiddonProjector as forward and back projector"; return false; }
  auto* f = static_cast<CuSiddonProjector*>(forwardprojector);
  auto* b = static_cast<CuSiddonProjector*>(backprojector);
  if (!f->setGpuId(indexGpu)) { strError = f->getError(); return false; }
  if (!b->setGpuId(indexGpu)) { strError = b->getError(); return false; }
  return Reconstruct();
}

CuOsemSinogram3d::CuOsemSinogram3d(Sinogram3D* in, Image* init, std::string path, std::string prefix, int iters,
                                   int saveInterval, bool saveInter, bool sensFromFile, CuProjector* fwd,
                                   CuProjector* back, int nsub)
    : CuMlemSinogram3d(in, init, path, prefix, iters, saveInterval, saveInter, sensFromFile, fwd, back),
      numSubsets(nsub) {}

bool CuOsemSinogram3d::Reconstruct() {
  if (numSubsets < 1) { strError = "number of subsets must be >= 1"; return false; }
  return reconstructOnDevice(numSubsets);
}

}  // namespace apirl
