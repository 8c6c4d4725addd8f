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

}  // namespace apirl
