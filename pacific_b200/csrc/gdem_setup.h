// gdem_setup.h -- the parts of a Grains3D XML input that the adjoint engine
// needs, read by the same importer as the step library (gdem_host.cu).
#pragma once
#include <string>
#include <vector>

#include "gdem_types.h"

namespace gdem {

struct AdjointSetup {
  std::vector<TypeDesc> types;     // particle classes
  std::vector<WallDesc> walls;     // box obstacles
  ModelDesc models[kMaxMat * kMaxMat];
  double dt = 0.;
  int periodic[3] = {0, 0, 0};
  double origin[3] = {0., 0., 0.}, maxc[3] = {0., 0., 0.};   // the domain box
};

// Throws std::runtime_error on malformed input.
void readAdjointSetup(std::string const& path, AdjointSetup& out);

// gdem_last_error() text.
void setLastError(std::string const& msg);

}  // namespace gdem
