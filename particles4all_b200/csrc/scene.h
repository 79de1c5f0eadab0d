// scene.h — host-side scene setup of Sim.reset (src/scene.js:41-315,
// src/sim.js:255-286): the fluid block, rigid-body samples, boundary shell with
// its psi weights, mass calibration and denomRest. JS numbers are doubles, so the
// math here is double and is rounded to float where the reference stores into
// Float32Arrays.
#pragma once
#include <stdint.h>

#include <vector>

#include "../../include/p4a.h"

namespace p4a {

struct HostScene {
  int n = 0, nFluid = 0, nBody = 0;
  std::vector<float> pos, vel, rest;  // float4 per particle
  std::vector<uint32_t> phase;        // uint4 per particle
  std::vector<double> bodyCentre;     // 3 per body
  std::vector<double> bodyDensity;
  std::vector<int> bodyCount;
  double mass = 0, denomRest = 0, h = 0, d = 0;
};

struct HostBoundary {
  int count = 0;
  std::vector<float> pos;       // float4, sorted by sim cell (sortBoundary)
  std::vector<float> psi;       // sorted like pos
  std::vector<uint32_t> cellStart;  // [nCells+2]
};

// buildScene(params) without the boundary (src/scene.js:159-315).
void build_scene(const p4a_params& p, HostScene& sc);
// Mass calibration / denomRest over the leading nFluid particles (src/scene.js:232-311).
void calibrate_scene(const p4a_params& p, HostScene& sc, bool doMass, bool doDenom);
// boundaryParticles (src/scene.js:76-135) followed by sortBoundary (src/sim.js:255-286)
// on the simulation grid gridDim (cell size h).
void build_boundary(const double box[3], double rho0, double d, double h, const int gridDim[3],
                    HostBoundary& out);
// boundaryParticles alone: shell points (double xyz) and psi, in generation order.
void boundary_points(const double box[3], double rho0, double d, double h, std::vector<double>& pts,
                     std::vector<float>& psi);

}  // namespace p4a
