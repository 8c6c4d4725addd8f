// The reference's GPU-side C++ API (reconGPU/inc: CuProjector,
// CuSiddonProjector's device-buffer calls, CuProjectorInterface,
// CuMlemSinogram3d, CuOsemSinogram3d) against the host-buffer calls of the
// same library.  Needs a GPU.  Prints "name value..." lines that
// tests/test_gpu_cuda_api.py checks.
//
//   cu_api_check <output dir>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../apirl_b200/host/apirl_host.h"

using namespace apirl;

namespace {

double rel(const float* a, const float* b, size_t n) {
  double num = 0, den = 0;
  for (size_t i = 0; i < n; i++) {
    const double d = (double)a[i] - (double)b[i];
    num += d * d;
    den += (double)b[i] * (double)b[i];
  }
  return std::sqrt(num / (den > 0 ? den : 1e-300));
}

bool bits_equal(const float* a, const float* b, size_t n) { return std::memcmp(a, b, n * sizeof(float)) == 0; }

float* to_device(const float* h, size_t n) {
  float* d = nullptr;
  cudaMalloc(&d, n * sizeof(float));
  if (h)
    cudaMemcpy(d, h, n * sizeof(float), cudaMemcpyHostToDevice);
  else
    cudaMemset(d, 0, n * sizeof(float));
  return d;
}

std::vector<float> to_host(const float* d, size_t n) {
  std::vector<float> h(n);
  cudaMemcpy(h.data(), d, n * sizeof(float), cudaMemcpyDeviceToHost);
  return h;
}

// A CuProjector of the caller's own: records what CuProjectorInterface hands
// it and fails every backprojection.
class Recorder : public CuProjector {
 public:
  std::vector<float> ring1, ring2;
  bool Project(float*, float* d_projection, float* d_ring1, float* d_ring2, Image*, Sinogram3D* s,
               bool) override {
    ring1 = to_host(d_ring1, (size_t)s->getNumSinograms());
    ring2 = to_host(d_ring2, (size_t)s->getNumSinograms());
    cudaMemset(d_projection, 0, (size_t)s->getBinCount() * sizeof(float));
    return true;
  }
  bool Backproject(float*, float*, float*, float*, Sinogram3D*, Image*, bool) override { return false; }
};

}  // namespace

int main(int argc, char** argv) {
  if (argc != 2) return 2;
  const std::string out = argv[1];
  SizeImage size{};
  size.nPixelsX = 40;
  size.nPixelsY = 40;
  size.nPixelsZ = 7;
  size.sizePixelX_mm = 2.08f;
  size.sizePixelY_mm = 2.08f;
  size.sizePixelZ_mm = 2.03f;
  Image x(size), ones(size);
  for (int i = 0; i < x.getPixelCount(); i++) x.getPixelsPtr()[i] = 0.5f + (float)((i * 7919) % 1000) / 1000.0f;
  ones.fillConstant(1);
  // Span 3, 6 rings: several ring pairs per sinogram, so the axial end
  // points are mean ring positions.  The sinogram's field of view covers the
  // whole image, so no voxel has zero sensitivity (which OSEM's threshold 0
  // would turn into NaN).
  Sinogram3DCylindricalPet sino(18, 52, 6, 59.0f, 6 * 2 * 2.03f, 150.0f, {-1, 2, -4}, {1, 4, -2});
  const size_t nb = (size_t)sino.getBinCount(), nv = (size_t)x.getPixelCount();
  printf("bins %zu\n", nb);

  CuSiddonProjector sp;
  // Host-buffer projection: the reference values for what follows.
  Sinogram3D* est = sino.Copy();
  if (!sp.Project(&x, est)) { printf("host_project_failed %s\n", sp.getError()); return 1; }
  Sinogram3D* meas = sino.Copy();
  for (size_t i = 0; i < nb; i++) meas->getSinogramPtr()[i] = std::floor(est->getSinogramPtr()[i] * 2.0f);

  // ---- CuSiddonProjector on device buffers ---------------------------------
  float* d_x = to_device(x.getPixelsPtr(), nv);
  float* d_p = to_device(nullptr, nb);
  Sinogram3D* got = sino.Copy();
  got->FillConstant(-1);
  bool ok = sp.Project(d_x, d_p, nullptr, nullptr, &x, got, true);
  printf("dev_project_ok %d\n", ok ? 1 : 0);
  printf("dev_project_bits_equal %d\n", bits_equal(got->getSinogramPtr(), est->getSinogramPtr(), nb) ? 1 : 0);
  printf("dev_project_buffer_bits_equal %d\n", bits_equal(to_host(d_p, nb).data(), est->getSinogramPtr(), nb) ? 1 : 0);

  Sinogram3D* sub = sino.getSubset(1, 3);
  Sinogram3D* subHost = sino.getSubset(1, 3);
  sp.Project(&x, subHost);
  float* d_ps = to_device(nullptr, (size_t)sub->getBinCount());
  ok = sp.Project(d_x, d_ps, nullptr, nullptr, &x, sub, false);
  printf("dev_project_subset_bits_equal %d\n",
         ok && bits_equal(to_host(d_ps, (size_t)sub->getBinCount()).data(), subHost->getSinogramPtr(),
                          (size_t)sub->getBinCount())
             ? 1
             : 0);

  Image bpHost(size);
  bpHost.fillConstant(0);
  sp.Backproject(meas, &bpHost);
  float* d_m = to_device(meas->getSinogramPtr(), nb);
  float* d_img = to_device(nullptr, nv);
  Image bpDev(size);
  bpDev.fillConstant(-1);
  ok = sp.Backproject(d_m, d_img, nullptr, nullptr, meas, &bpDev, true);
  printf("dev_backproject_rel %d %.3e\n", ok ? 1 : 0, rel(bpDev.getPixelsPtr(), bpHost.getPixelsPtr(), nv));
  // A second call adds into the same device image.
  sp.Backproject(d_m, d_img, nullptr, nullptr, meas, &bpDev, true);
  std::vector<float> twice(nv);
  for (size_t i = 0; i < nv; i++) twice[i] = 2 * bpHost.getPixelsPtr()[i];
  printf("dev_backproject_accumulates_rel %.3e\n", rel(bpDev.getPixelsPtr(), twice.data(), nv));

  Image dbHost(size);
  dbHost.fillConstant(0);
  sp.DivideAndBackproject(meas, est, &dbHost);
  float* d_e = to_device(est->getSinogramPtr(), nb);
  cudaMemset(d_img, 0, nv * sizeof(float));
  ok = sp.DivideAndBackproject(d_m, d_e, d_img, nullptr, nullptr, meas, &bpDev, false);
  printf("dev_divide_rel %d %.3e\n", ok ? 1 : 0, rel(to_host(d_img, nv).data(), dbHost.getPixelsPtr(), nv));
  printf("dev_divide_estimate_unchanged %d\n", bits_equal(to_host(d_e, nb).data(), est->getSinogramPtr(), nb) ? 1 : 0);
  printf("dev_null_buffer_false %d\n", sp.Project(nullptr, d_p, nullptr, nullptr, &x, got, false) ? 0 : 1);

  // ---- CuProjectorInterface --------------------------------------------------
  CuSiddonProjector wrapped;
  CuProjectorInterface iface(&wrapped);
  Sinogram3D* ip = sino.Copy();
  ip->FillConstant(5);
  ok = iface.Project(&x, ip);
  printf("iface_project_bits_equal %d\n", ok && bits_equal(ip->getSinogramPtr(), est->getSinogramPtr(), nb) ? 1 : 0);
  Image ib(size);
  ib.fillConstant(7);  // overwritten, not added to
  ok = iface.Backproject(meas, &ib);
  printf("iface_backproject_rel %d %.3e\n", ok ? 1 : 0, rel(ib.getPixelsPtr(), bpHost.getPixelsPtr(), nv));
  ib.fillConstant(7);
  ok = iface.DivideAndBackproject(meas, est, &ib);
  printf("iface_divide_rel %d %.3e\n", ok ? 1 : 0, rel(ib.getPixelsPtr(), dbHost.getPixelsPtr(), nv));
  ok = iface.Project(&x, sub);
  printf("iface_project_subset_bits_equal %d\n",
         ok && bits_equal(sub->getSinogramPtr(), subHost->getSinogramPtr(), (size_t)sub->getBinCount()) ? 1 : 0);
  Sinogram2DinCylindrical3Dpet s2(18, 52, 59.0f, 150.0f);
  printf("iface_2d_false %d\n", iface.Project(&x, &s2) || iface.Backproject(&s2, &ib) ? 0 : 1);
  printf("iface_bad_gpu_false %d\n", iface.setGpuId(-1) || iface.setGpuId(4096) ? 0 : 1);

  Recorder rec;
  CuProjectorInterface recIface(&rec);
  recIface.setProjectorBlockSizeConfig(dim3(64, 1, 1));
  Sinogram3D* rp = sino.Copy();
  ok = recIface.Project(&x, rp);
  std::vector<float> z((size_t)2 * sino.getNumSinograms());
  apirl_sino3d_geom g = sino.geom();
  apirl_sino3d_ring_z(&g, z.data());
  bool rings = ok && (int)rec.ring1.size() == sino.getNumSinograms();
  for (int i = 0; rings && i < sino.getNumSinograms(); i++)
    rings = rec.ring1[i] == z[2 * i] && rec.ring2[i] == z[2 * i + 1];
  printf("iface_rings_equal %d\n", rings ? 1 : 0);
  printf("iface_sinograms %d\n", sino.getNumSinograms());
  dim3 gs = rec.getGridSize(), bs = rec.getBlockSize();
  printf("iface_grid %u %u %u %u\n", gs.x, gs.y, gs.z, bs.x);
  Image rb(size);
  printf("iface_foreign_false %d\n", recIface.Backproject(meas, &rb) ? 0 : 1);

  // ---- CuMlemSinogram3d / CuOsemSinogram3d -----------------------------------
  CuSiddonProjector f1, b1, f2, b2;
  MlemSinogram3d plain(meas, &ones, "", out + "/plain", 3, 0, false, false, &f1, &b1);
  CuMlemSinogram3d cu(meas, &ones, "", out + "/cu", 3, 0, false, false, &f2, &b2);
  cu.setProjectorKernelConfig(256, 1, 1);
  dim3 b = cu.getProjectorKernelConfig();
  printf("cumlem_block %u %u %u\n", b.x, b.y, b.z);
  const bool okPlain = plain.Reconstruct();
  ok = cu.Reconstruct(SIDDON_PROJ_TEXT_CYLINDRICAL_SCANNER, 0);
  printf("cumlem_rel %d %.3e\n", okPlain && ok ? 1 : 0,
         rel(cu.getReconstructedImage()->getPixelsPtr(), plain.getReconstructedImage()->getPixelsPtr(), nv));
  const auto& l1 = cu.getLikelihoodValues();
  const auto& l0 = plain.getLikelihoodValues();
  printf("cumlem_likelihood_rel %.3e\n", std::fabs(l1[0] - l0[0]) / std::fabs(l0[0]));
  printf("cumlem_hexagonal_false %d\n", cu.Reconstruct(SIDDON_HEXAGONAL_SCANNER, 0) ? 0 : 1);
  printf("cumlem_bad_gpu_false %d\n", cu.Reconstruct(SIDDON_CYLINDRICAL_SCANNER, 4096) ? 0 : 1);

  CuSiddonProjector f3, b3, f4, b4;
  OsemSinogram3d oplain(meas, &ones, "", out + "/oplain", 2, 0, false, false, &f3, &b3, 3);
  CuOsemSinogram3d ocu(meas, &ones, "", out + "/ocu", 2, 0, false, false, &f4, &b4, 3);
  const bool okO = oplain.Reconstruct();
  ok = ocu.Reconstruct(SIDDON_CYLINDRICAL_SCANNER);
  printf("cuosem_rel %d %.3e\n", okO && ok ? 1 : 0,
         rel(ocu.getReconstructedImage()->getPixelsPtr(), oplain.getReconstructedImage()->getPixelsPtr(), nv));
  printf("cuosem_likelihoods %zu\n", ocu.getLikelihoodValues().size());

  Recorder rf, rb2;
  CuMlemSinogram3d foreign(meas, &ones, "", out + "/foreign", 1, 0, false, false, &rf, &rb2);
  printf("cumlem_foreign_false %d\n", foreign.Reconstruct(SIDDON_CYLINDRICAL_SCANNER, 0) ? 0 : 1);

  cudaFree(d_x); cudaFree(d_p); cudaFree(d_ps); cudaFree(d_m); cudaFree(d_img); cudaFree(d_e);
  delete est; delete meas; delete got; delete sub; delete subHost; delete ip; delete rp;
  printf("cuda_error %d\n", (int)cudaGetLastError());
  return 0;
}
