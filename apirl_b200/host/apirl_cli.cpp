// The reference's .par-driven commands on the GPU path: MLEM, OSEM, project,
// backproject, generateACFs and cuMLEM (cmd/src/MLEM.cpp, OSEM.cpp,
// project.cpp, backproject.cpp, generateACFs.cpp, cmdGPU/src/cuMLEM.cpp).
// One source; the command is chosen at build time with -DAPIRL_COMMAND=<name>
// (the binary's name).  Each takes one argument, a parameter file ending in
// .par whose first line is "<COMMAND> Parameters :=".
//
// Keys read (as in the reference):
//   MLEM/OSEM  input type, input file, initial estimate, output filename prefix,
//              number of iterations, number of subsets (OSEM), forwardprojector,
//              backprojector, sensitivity filename, save estimates at iteration
//              intervals, save estimated projections and backprojected image,
//              multiplicative sinogram, additive sinogram, cylindrical pet radius
//              (in mm), radius fov (in mm), axial fov (in mm), gpu id
//   project    input file, output type, projector, output filename, output
//              projection, number of subsets, subset index (+ scanner keys)
//   backproject input type, input file, backprojector, output image, output
//              filename, number of subsets, subset index (+ scanner keys)
//   generateACFs input file (attenuation map, 1/cm), output type (Sinogram2D,
//              Sinogram3D, Sinogram3DSiemensMmr), output filename, output
//              projection, projector (Siddon, CuSiddonProjector: + projector
//              block size, gpu id) (+ scanner keys)
//   cuMLEM     section "MLEM": input type (Sinogram3D, Sinogram3DSiemensMmr),
//              input file, initial estimate, output filename prefix, number of
//              iterations, forwardprojector and backprojector (CuSiddonProjector),
//              projector / backprojector / pixel update block size ({x,y,z}),
//              gpu id, number of subsets (OSEM, Sinogram3DSiemensMmr only, as in
//              the reference), multiplicative sinogram, additive sinogram
//              (+ scanner keys)
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <memory>
#include <string>

#include "apirl_host.h"

using namespace apirl;

#ifndef APIRL_COMMAND
#define APIRL_COMMAND "OSEM"
#endif

namespace {

const char* kCmd = APIRL_COMMAND;
std::string g_par;
std::string g_section;

bool key(const char* k, std::string* v, bool required = true) {
  int e = parametersFile_read(g_par.c_str(), g_section.c_str(), k, v);
  if (e == 0) return true;
  if (e == 2 && !required) return false;
  std::cerr << "Error " << e << " reading \"" << k << "\" from " << g_par << std::endl;
  exit(1);
}

float fkey(const char* k, float def) {
  std::string v;
  return key(k, &v, false) ? (float)atof(v.c_str()) : def;
}

int ikey(const char* k, int def) {
  std::string v;
  return key(k, &v, false) ? atoi(v.c_str()) : def;
}

struct Scanner {
  float rScanner, rFov, zFov;
};

Scanner scanner(const Image* img) {
  Scanner s;
  s.rScanner = fkey("cylindrical pet radius (in mm)", 443.f);
  s.rFov = fkey("radius fov (in mm)", img ? img->getFovRadio() : 0.f);
  s.zFov = fkey("axial fov (in mm)", img ? img->getFovHeight() : 0.f);
  return s;
}

std::unique_ptr<CuSiddonProjector> siddon(const std::string& name) {
  if (name != "Siddon" && name != "CuSiddon") {
    std::cerr << "Only the Siddon projector is available on this path (got \"" << name << "\")" << std::endl;
    exit(1);
  }
  // getSiddonProjectorParameters (data/src/readParameters.cpp:162-203); an
  // absent key means one sample.
  int ns = ikey("siddon number of samples on the detector", 1);
  int nas = ikey("siddon number of axial samples on the detector", 1);
  if (ns < 1 || nas < 1 || ns > APIRL_MAX_SAMPLES || nas > APIRL_MAX_SAMPLES) {
    std::cerr << "siddon number of samples must be 1.." << APIRL_MAX_SAMPLES << std::endl;
    exit(1);
  }
  return std::unique_ptr<CuSiddonProjector>(new CuSiddonProjector(ns, nas, ikey("gpu id", 0)));
}

int recon(bool osem) {
  std::string type, input, init, prefix, v;
  key("input type", &type);
  key("input file", &input);
  key("initial estimate", &init);
  key("output filename prefix", &prefix);
  int iters = ikey("number of iterations", 1);
  int subsets = osem ? ikey("number of subsets", 1) : 1;
  std::string fwdName = "Siddon", backName = "Siddon";
  key("forwardprojector", &fwdName, false);
  key("backprojector", &backName, false);
  // getSensitivityFromFile, getSaveIntermidiateIntervals
  // (data/src/readParameters.cpp:25-110).
  std::string sensName;
  const bool sensFromFile = key("sensitivity filename", &sensName, false);
  const int saveInterval = ikey("save estimates at iteration intervals", 0);
  const bool saveInter = saveInterval > 0 && ikey("save estimated projections and backprojected image", 0) != 0;
  if (saveInter)
    std::cout << "save estimated projections and backprojected image: not written (the fused pass does not form "
                 "them); the images of the saved iterations are" << std::endl;
  Image x0;
  if (!x0.readFromInterfile(init.c_str())) {
    std::cerr << "Error reading the initial estimate: " << x0.getError() << std::endl;
    return 1;
  }
  auto fwd = siddon(fwdName);
  auto back = siddon(backName);
  Scanner sc = scanner(&x0);
  std::string mult, add;
  bool hasMult = key("multiplicative sinogram", &mult, false);
  bool hasAdd = key("additive sinogram", &add, false);
  std::unique_ptr<Mlem> m;
  std::unique_ptr<Sinogram2D> s2;
  std::unique_ptr<Sinogram3D> s3;
  if (type == "Sinogram2D") {
    s2.reset(new Sinogram2DinCylindrical3Dpet(input.c_str(), sc.rFov, sc.rScanner));
    if (s2->getNumR() <= 1) { std::cerr << "Error reading " << input << ": " << s2->getError() << std::endl; return 1; }
    if (osem) { std::cerr << "OSEM needs a Sinogram3D input" << std::endl; return 1; }
    m.reset(new Mlem2d(s2.get(), &x0, "", prefix, iters, saveInterval, saveInter, sensFromFile, fwd.get(),
                       back.get()));
    // The reference's Mlem2d forces the sinogram rFov to the image's; an
    // explicit "radius fov (in mm)" restores the sinogram's own bin pitch.
    std::string rf;
    if (key("radius fov (in mm)", &rf, false)) s2->setRadioFov_mm((float)atof(rf.c_str()));
  } else if (type == "Sinogram3D" || type == "Sinogram3DSiemensMmr") {
    // Sinogram3DSiemensMmr carries the mMR's fixed geometry (OSEM.cpp:416-425).
    if (type == "Sinogram3D")
      s3.reset(new Sinogram3DCylindricalPet(input.c_str(), sc.rFov, sc.zFov, sc.rScanner));
    else
      s3.reset(new Sinogram3DSiemensMmr(input.c_str()));
    if (s3->getNumSinograms() <= 0 || s3->getBinCount() <= 1) {
      std::cerr << "Error reading " << input << ": " << s3->getError() << std::endl;
      return 1;
    }
    if (osem)
      m.reset(new OsemSinogram3d(s3.get(), &x0, "", prefix, iters, saveInterval, saveInter, sensFromFile,
                                 fwd.get(), back.get(), subsets));
    else
      m.reset(new MlemSinogram3d(s3.get(), &x0, "", prefix, iters, saveInterval, saveInter, sensFromFile,
                                 fwd.get(), back.get()));
  } else {
    std::cerr << "input type " << type << " is not supported on this path (Sinogram2D, Sinogram3D, "
              << "Sinogram3DSiemensMmr)" << std::endl;
    return 1;
  }
  if (sensFromFile) m->setSensitivityFilename(sensName);
  if (hasMult && !m->setMultiplicativeProjection(mult)) { std::cerr << "Error reading " << mult << std::endl; return 1; }
  if (hasAdd && !m->setAdditiveProjection(add)) { std::cerr << "Error reading " << add << std::endl; return 1; }
  auto t0 = std::chrono::steady_clock::now();
  if (!m->Reconstruct()) { std::cerr << "Reconstruction failed: " << m->getError() << std::endl; return 1; }
  double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::cout << kCmd << ": " << iters << " iterations in " << s << " s, output " << prefix << "_final.h33" << std::endl;
  return 0;
}

int project() {
  std::string input, type, proj, out, tmpl;
  key("input file", &input);
  key("output type", &type);
  key("projector", &proj);
  key("output filename", &out);
  key("output projection", &tmpl);
  int nsub = ikey("number of subsets", 0), subset = ikey("subset index", -1);
  Image img;
  if (!img.readFromInterfile(input.c_str())) { std::cerr << img.getError() << std::endl; return 1; }
  auto p = siddon(proj);
  Scanner sc = scanner(&img);
  auto t0 = std::chrono::steady_clock::now();
  if (type == "Sinogram2D") {
    Sinogram2DinCylindrical3Dpet s(tmpl.c_str(), sc.rFov, sc.rScanner);
    s.FillConstant(0);
    if (!p->Project(&img, &s)) { std::cerr << p->getError() << std::endl; return 1; }
    s.writeInterfile(out.c_str());
  } else if (type == "Sinogram3D" || type == "Sinogram3DSiemensMmr") {
    std::unique_ptr<Sinogram3D> full(type == "Sinogram3D"
                                         ? (Sinogram3D*)new Sinogram3DCylindricalPet(tmpl.c_str(), sc.rFov, sc.zFov,
                                                                                     sc.rScanner)
                                         : (Sinogram3D*)new Sinogram3DSiemensMmr(tmpl.c_str()));
    std::unique_ptr<Sinogram3D> s(nsub > 0 && subset >= 0 ? full->getSubset(subset, nsub) : full->Copy());
    if (!p->Project(&img, s.get())) { std::cerr << p->getError() << std::endl; return 1; }
    s->writeInterfile(out.c_str());
  } else {
    std::cerr << "output type " << type << " is not supported on this path" << std::endl;
    return 1;
  }
  double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::cout << "project: " << sec << " s" << std::endl;
  return 0;
}

int backproject() {
  std::string type, input, proj, outImg, out;
  key("input type", &type);
  key("input file", &input);
  key("backprojector", &proj);
  key("output image", &outImg);
  key("output filename", &out);
  int nsub = ikey("number of subsets", 0), subset = ikey("subset index", -1);
  Image img;
  if (!img.readFromInterfile(outImg.c_str())) { std::cerr << img.getError() << std::endl; return 1; }
  img.fillConstant(0);
  auto p = siddon(proj);
  Scanner sc = scanner(&img);
  auto t0 = std::chrono::steady_clock::now();
  if (type == "Sinogram2D") {
    Sinogram2DinCylindrical3Dpet s(input.c_str(), sc.rFov, sc.rScanner);
    if (!p->Backproject(&s, &img)) { std::cerr << p->getError() << std::endl; return 1; }
  } else if (type == "Sinogram3D" || type == "Sinogram3DSiemensMmr") {
    std::unique_ptr<Sinogram3D> full(type == "Sinogram3D"
                                         ? (Sinogram3D*)new Sinogram3DCylindricalPet(input.c_str(), sc.rFov, sc.zFov,
                                                                                     sc.rScanner)
                                         : (Sinogram3D*)new Sinogram3DSiemensMmr(input.c_str()));
    std::unique_ptr<Sinogram3D> s(nsub > 0 && subset >= 0 ? full->getSubset(subset, nsub) : full->Copy());
    if (!p->Backproject(s.get(), &img)) { std::cerr << p->getError() << std::endl; return 1; }
  } else {
    std::cerr << "input type " << type << " is not supported on this path" << std::endl;
    return 1;
  }
  img.writeInterfile(out.c_str());
  double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::cout << "backproject: " << sec << " s" << std::endl;
  return 0;
}

// Attenuation correction factors in place: exp of every non-zero bin, 1
// elsewhere (generateACFs.cpp:306-320, :500-520), with the host's float exp
// as the reference computes them.
void to_acf(float* bins, size_t n) {
  for (size_t i = 0; i < n; i++) bins[i] = bins[i] != 0.f ? std::exp(bins[i]) : 1.f;
}

bool block_size(const char* k, dim3* out);

// cmd/src/generateACFs.cpp:180-560.
int generate_acfs() {
  std::string input, type, out, tmpl, proj;
  key("input file", &input);
  key("output type", &type);
  key("output filename", &out);
  key("output projection", &tmpl);
  key("projector", &proj);
  Image mu;
  if (!mu.readFromInterfile(input.c_str())) {
    std::cerr << "Error reading the attenuation map: " << mu.getError() << std::endl;
    return -1;
  }
  // "CuSiddonProjector" reads its block size and GPU (generateACFs.cpp:254-271);
  // every name runs the Siddon projector on the GPU here.
  dim3 b;
  if (proj == "CuSiddonProjector" && !block_size("projector block size", &b)) return -1;
  CuSiddonProjector p(1, 1, ikey("gpu id", 0));
  // 1/cm to 1/mm (generateACFs.cpp:275-285).
  float* px = mu.getPixelsPtr();
  for (int i = 0; i < mu.getPixelCount(); i++) px[i] = px[i] / 10;
  Scanner sc = scanner(&mu);
  auto t0 = std::chrono::steady_clock::now();
  if (type == "Sinogram2D") {
    Sinogram2DinCylindrical3Dpet s(tmpl.c_str(), sc.rFov, sc.rScanner);
    if (s.getNumR() <= 1) { std::cerr << "Error reading " << tmpl << ": " << s.getError() << std::endl; return -1; }
    s.FillConstant(0);
    if (!p.Project(&mu, &s)) { std::cerr << p.getError() << std::endl; return 1; }
    to_acf(s.getSinogramPtr(), (size_t)s.getNumProj() * s.getNumR());
    s.writeInterfile(out.c_str());
  } else if (type == "Sinogram3D" || type == "Sinogram3DSiemensMmr") {
    std::unique_ptr<Sinogram3D> s(type == "Sinogram3D"
                                      ? (Sinogram3D*)new Sinogram3DCylindricalPet(tmpl.c_str(), sc.rFov, sc.zFov,
                                                                                  sc.rScanner)
                                      : (Sinogram3D*)new Sinogram3DSiemensMmr(tmpl.c_str()));
    if (s->getNumSinograms() <= 0 || s->getBinCount() <= 1) {
      std::cerr << "Error reading " << tmpl << ": " << s->getError() << std::endl;
      return -1;
    }
    std::unique_ptr<Sinogram3D> in(s->Copy());  // the template's own bins
    if (!p.Project(&mu, s.get())) { std::cerr << p.getError() << std::endl; return 1; }
    to_acf(s->getSinogramPtr(), (size_t)s->getBinCount());
    s->writeInterfile(out.c_str());
    // The template corrected with the factors, "<output>_attCorrected"
    // (generateACFs.cpp:522-545).
    float* a = in->getSinogramPtr();
    const float* f = s->getSinogramPtr();
    for (int i = 0; i < in->getBinCount(); i++) a[i] = a[i] * f[i];
    in->writeInterfile((out + "_attCorrected").c_str());
  } else {
    std::cerr << "output type " << type << " is not supported (Sinogram2D, Sinogram3D, Sinogram3DSiemensMmr)"
              << std::endl;
    return -1;
  }
  double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::cout << "generateACFs: " << sec << " s" << std::endl;
  return 0;
}

// ProcessBlockSizeString (reconGPU/src/readCudaParameters.cpp:22-48): the
// three numbers between the last '{' and the last '}', separated by spaces or
// commas.
bool block_size(const char* k, dim3* out) {
  std::string v;
  key(k, &v);
  size_t a = v.rfind('{'), b = v.rfind('}');
  if (a == std::string::npos || b == std::string::npos || b < a) {
    std::cerr << "\"" << k << "\" must be {x,y,z}" << std::endl;
    return false;
  }
  std::string body = v.substr(a + 1, b - a - 1);
  for (char& c : body)
    if (c == ',') c = ' ';
  unsigned int x = 0, y = 0, z = 0;
  if (sscanf(body.c_str(), "%u %u %u", &x, &y, &z) != 3) {
    std::cerr << "\"" << k << "\" needs three elements" << std::endl;
    return false;
  }
  *out = dim3(x, y, z);
  return true;
}

// cmdGPU/src/cuMLEM.cpp:159-483.
int cumlem() {
  std::string type, input, init, prefix, fwdName, backName;
  key("input type", &type);
  key("input file", &input);
  key("initial estimate", &init);
  key("output filename prefix", &prefix);
  std::string it;
  key("number of iterations", &it);
  const int iters = atoi(it.c_str());
  key("forwardprojector", &fwdName);
  key("backprojector", &backName);
  dim3 bp, bb, bu;
  if (!block_size("projector block size", &bp) || !block_size("backprojector block size", &bb) ||
      !block_size("pixel update block size", &bu))
    return -1;
  int gpu = ikey("gpu id", 0);
  int subsets = ikey("number of subsets", 0);
  const int saveInterval = ikey("save estimates at iteration intervals", 0);
  std::string sensName;
  const bool sensFromFile = key("sensitivity filename", &sensName, false);
  for (const std::string* n : {&fwdName, &backName})
    if (*n != "CuSiddonProjector") {
      std::cerr << "No existe el proyector " << *n << "." << std::endl;
      return 1;
    }
  Image x0;
  if (!x0.readFromInterfile(init.c_str())) {
    std::cerr << "Error reading the initial estimate: " << x0.getError() << std::endl;
    return -1;
  }
  CuSiddonProjector fwd, back;
  std::unique_ptr<Sinogram3D> s3;
  std::unique_ptr<CuMlemSinogram3d> m;
  if (type == "Sinogram3D") {
    Scanner sc = scanner(&x0);
    s3.reset(new Sinogram3DCylindricalPet(input.c_str(), sc.rFov, sc.zFov, sc.rScanner));
  } else if (type == "Sinogram3DSiemensMmr") {
    s3.reset(new Sinogram3DSiemensMmr(input.c_str()));
  } else {
    std::cerr << "input type " << type << " is not supported (Sinogram3D, Sinogram3DSiemensMmr)" << std::endl;
    return -1;
  }
  if (s3->getNumSinograms() <= 0 || s3->getBinCount() <= 1) {
    std::cerr << "Error reading " << input << ": " << s3->getError() << std::endl;
    return 1;
  }
  // The reference runs OSEM for mMR sinograms with a subset count only.
  if (type == "Sinogram3DSiemensMmr" && subsets > 0)
    m.reset(new CuOsemSinogram3d(s3.get(), &x0, "", prefix, iters, saveInterval, false, sensFromFile, &fwd, &back,
                                 subsets));
  else
    m.reset(new CuMlemSinogram3d(s3.get(), &x0, "", prefix, iters, saveInterval, false, sensFromFile, &fwd, &back));
  if (sensFromFile) m->setSensitivityFilename(sensName);
  std::string mult, add;
  if (key("multiplicative sinogram", &mult, false) && !m->setMultiplicativeProjection(mult)) {
    std::cerr << "Error reading " << mult << std::endl;
    return 1;
  }
  if (key("additive sinogram", &add, false) && !m->setAdditiveProjection(add)) {
    std::cerr << "Error reading " << add << std::endl;
    return 1;
  }
  m->setBackprojectorKernelConfig(&bb);
  m->setProjectorKernelConfig(&bp);
  m->setUpdatePixelKernelConfig(&bu);
  auto t0 = std::chrono::steady_clock::now();
  if (!m->Reconstruct(SIDDON_PROJ_TEXT_CYLINDRICAL_SCANNER, gpu)) {
    std::cerr << "Reconstruction failed: " << m->getError() << std::endl;
    return 1;
  }
  double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::cout << kCmd << ": " << iters << " iterations in " << sec << " s, output " << prefix << "_final.h33" << std::endl;
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 2) {
    std::cerr << "usage: " << kCmd << " parameters.par" << std::endl;
    return -1;
  }
  g_par = argv[1];
  if (g_par.size() < 4 || g_par.compare(g_par.size() - 4, 4, ".par") != 0) {
    std::cerr << "The parameter file must have the .par extension" << std::endl;
    return -1;
  }
  std::string cmd = kCmd;
  g_section = cmd == "project" ? "Projection" : (cmd == "backproject" ? "Backproject" : cmd == "cuMLEM" ? "MLEM" : cmd);
  if (cmd == "generateACFs") return generate_acfs();
  if (cmd == "MLEM") return recon(false);
  if (cmd == "OSEM") return recon(true);
  if (cmd == "project") return project();
  if (cmd == "backproject") return backproject();
  if (cmd == "cuMLEM") return cumlem();
  std::cerr << "unknown command " << cmd << std::endl;
  return -1;
}
