// Test program (CPU only): the C++ host layer's interfile and .par readers
// against files written by the reference's own writers, and round trips of its
// own writers.  Prints one "name value" line per check; the pytest driver
// (tests/test_host_io.py) compares them.
#include <cstdio>
#include <string>
#include "../apirl_b200/host/apirl_host.h"

using namespace apirl;

int main(int argc, char** argv) {
  std::string gold = argv[1], tmp = argv[2];
  // image written by the reference (medcon)
  Image im;
  bool ok = im.readFromInterfile((gold + "/image.h33").c_str());
  SizeImage s = im.getSize();
  printf("image_read %d\n", ok ? 1 : 0);
  printf("image_size %d %d %d %.6f %.6f %.6f\n", s.nPixelsX, s.nPixelsY, s.nPixelsZ, s.sizePixelX_mm,
         s.sizePixelY_mm, s.sizePixelZ_mm);
  double sum = 0;
  for (int i = 0; i < im.getPixelCount(); i++) sum += im.getPixelsPtr()[i] * (i + 1);
  printf("image_checksum %.6f\n", sum);
  ok = im.writeInterfile((tmp + "/image_ours").c_str());
  Image back;
  back.readFromInterfile((tmp + "/image_ours.h33").c_str());
  double sum2 = 0;
  for (int i = 0; i < back.getPixelCount(); i++) sum2 += back.getPixelsPtr()[i] * (i + 1);
  printf("image_roundtrip %d %.6f\n", ok ? 1 : 0, sum2);
  // 3D sinogram written by the reference
  Sinogram3DCylindricalPet sino((gold + "/sino3d.h33").c_str(), 20.f, 12.f, 60.f);
  printf("sino_segments %d sinograms %d proj %d r %d bins %d\n", sino.getNumSegments(), sino.getNumSinograms(),
         sino.getNumProj(), sino.getNumR(), sino.getBinCount());
  double ss = 0;
  for (int i = 0; i < sino.getBinCount(); i++) ss += sino.getSinogramPtr()[i] * (i + 1);
  printf("sino_checksum %.6f\n", ss);
  Sinogram3D* sub = sino.getSubset(1, 3);
  double sb = 0;
  for (int i = 0; i < sub->getBinCount(); i++) sb += sub->getSinogramPtr()[i] * (i + 1);
  printf("subset_bins %d checksum %.6f\n", sub->getBinCount(), sb);
  delete sub;
  sino.writeInterfile((tmp + "/sino_ours").c_str());
  Sinogram3DCylindricalPet sino2((tmp + "/sino_ours.h33").c_str(), 20.f, 12.f, 60.f);
  double s2 = 0;
  for (int i = 0; i < sino2.getBinCount(); i++) s2 += sino2.getSinogramPtr()[i] * (i + 1);
  printf("sino_roundtrip %d %.6f\n", sino2.getBinCount(), s2);
  // parameter files
  FILE* f = fopen((tmp + "/t.par").c_str(), "w");
  fprintf(f, "OSEM Parameters :=\ninput type := Sinogram3D\n  number of subsets := 21\n;comment := 3\n"
             "number of iterations := 3\nnumber of iterations := 4\nEND :=\n");
  fclose(f);
  std::string v;
  int e1 = parametersFile_read((tmp + "/t.par").c_str(), "OSEM", "number of subsets", &v);
  printf("par_subsets %d %s\n", e1, v.c_str());
  int e2 = parametersFile_read((tmp + "/t.par").c_str(), "OSEM", "number of iterations", &v);
  int e3 = parametersFile_read((tmp + "/t.par").c_str(), "OSEM", "comment", &v);
  int e4 = parametersFile_read((tmp + "/t.par").c_str(), "MLEM", "number of subsets", &v);
  int e5 = parametersFile_read((tmp + "/none.par").c_str(), "OSEM", "number of subsets", &v);
  printf("par_errors %d %d %d %d\n", e2, e3, e4, e5);
  return 0;
}
