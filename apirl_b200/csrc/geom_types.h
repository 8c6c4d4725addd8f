// Plain geometry structs shared by host and device code.
#pragma once

namespace apirl {

// Image geometry as the walk needs it.  rfov = (dx * nx) / 2 in float
// (data/src/Images.cpp:55), offz = dz / 2 (Siddon.cpp:162).
struct ImgGeom {
  int nx, ny, nz;
  float dx, dy, dz;
  float rfov, offz;
};

// Border width, in voxels, of the padded image layouts of the fused 3D pass.
constexpr int kPad = 2;

}  // namespace apirl
