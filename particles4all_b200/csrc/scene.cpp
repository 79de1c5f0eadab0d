// scene.cpp — host scene setup for Sim.reset (src/scene.js:41-315, src/sim.js:255-286).
//
// Neighbour sums (boundary psi, density for the mass calibration, denomRest) use a
// flat cell grid whose buckets list particles in index order and are visited in
// the reference's (dc, db, da) order, so the double sums are added in the same
// order as the JS Map-of-arrays walk and give the same values. Per-particle sums are
// independent, so they run in parallel (OpenMP).
#include "scene.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace p4a {
namespace {

const double kPi = 3.14159265358979323846;  // Math.PI

// A dense cell grid with per-cell particle lists in index order.
struct CellLists {
  int dim[3] = {1, 1, 1};
  std::vector<uint32_t> first;  // [cells + 1]
  std::vector<uint32_t> ids;    // particle ids grouped by cell
  std::vector<uint32_t> cellOf; // per particle

  void build(const int d3[3], int n, const std::vector<uint32_t>& cell) {
    std::memcpy(dim, d3, sizeof(dim));
    const size_t cells = (size_t)dim[0] * dim[1] * dim[2];
    first.assign(cells + 1, 0u);
    for (int i = 0; i < n; i++) first[cell[i] + 1]++;
    for (size_t c = 0; c < cells; c++) first[c + 1] += first[c];
    ids.resize(n);
    std::vector<uint32_t> at(first.begin(), first.end() - 1);
    for (int i = 0; i < n; i++) ids[at[cell[i]]++] = (uint32_t)i;
    cellOf = cell;
  }
  // Visit the ids in the 27 cells around `c` in the reference's order.
  template <class F>
  void around(int cx, int cy, int cz, F&& f) const {
    for (int dc = -1; dc <= 1; dc++) {
      const int z = cz + dc;
      if (z < 0 || z >= dim[2]) continue;
      for (int db = -1; db <= 1; db++) {
        const int y = cy + db;
        if (y < 0 || y >= dim[1]) continue;
        for (int da = -1; da <= 1; da++) {
          const int x = cx + da;
          if (x < 0 || x >= dim[0]) continue;
          const size_t k = ((size_t)z * dim[1] + y) * dim[0] + x;
          for (uint32_t m = first[k]; m < first[k + 1]; m++) f((int)ids[m]);
        }
      }
    }
  }
};

inline int clampi(double v, int hi) { return (int)std::min<double>(hi, std::max(0.0, v)); }

}  // namespace

// fluidBlock (src/scene.js:43-64) appended to `out` as xyz doubles. The JS LCG
// multiplies in double (a rounded product above 2^53), then ToInt32 & 0x7fffffff.
static void fluid_block(const p4a_params& p, double d, std::vector<double>& out) {
  const double margin = d;
  const double nx = std::max(1.0, std::floor(p.box[0] * 0.35 / d));
  const double nz = std::max(1.0, std::floor((p.box[2] - 2 * margin) / d));
  const double maxLayers = std::max(1.0, std::floor((p.box[1] - 2 * margin) / d));
  const double target = p.target_particle_count;
  const double layers = std::min(std::ceil(target / (nx * nz)), maxLayers);
  double seed = 12345;
  auto jitter = [&]() {
    const double s = seed * 1103515245.0 + 12345.0;
    seed = (double)(int32_t)((uint32_t)(int64_t)s & 0x7fffffffu);
    return (seed / 2147483647.0 - 0.5) * 0.002 * d;
  };
  out.clear();
  for (double iy = 0; iy < layers && out.size() / 3 < target; iy++)
    for (double ix = 0; ix < nx && out.size() / 3 < target; ix++)
      for (double iz = 0; iz < nz && out.size() / 3 < target; iz++) {
        const double x = margin + (ix + 0.5) * d + jitter();
        const double y = margin + (iy + 0.5) * d + jitter();
        const double z = margin + (iz + 0.5) * d + jitter();
        out.push_back(x);
        out.push_back(y);
        out.push_back(z);
      }
}

// sampleBody (src/scene.js:137-157).
static void sample_body(int shape, double size, double d, std::vector<double>& out) {
  double e[3];
  if (shape == P4A_SHAPE_SPHERE) {
    e[0] = e[1] = e[2] = size;
  } else if (shape == P4A_SHAPE_TORUS) {
    e[0] = size + 0.4 * size; e[1] = 0.4 * size; e[2] = size + 0.4 * size;
  } else {
    e[0] = size * 0.9; e[1] = size * 0.7; e[2] = size * 0.9;
  }
  const int sx = (int)std::max(1.0, std::ceil(e[0] / d));
  const int sy = (int)std::max(1.0, std::ceil(e[1] / d));
  const int sz = (int)std::max(1.0, std::ceil(e[2] / d));
  out.clear();
  for (int ix = -sx; ix <= sx; ix++)
    for (int iy = -sy; iy <= sy; iy++)
      for (int iz = -sz; iz <= sz; iz++) {
        const double x = ix * d, y = iy * d, z = iz * d;
        bool in;
        switch (shape) {
          case P4A_SHAPE_SPHERE: in = x * x + y * y + z * z <= size * size; break;
          case P4A_SHAPE_TORUS: {
            const double planar = std::sqrt(x * x + z * z) - size;
            in = planar * planar + y * y <= (0.4 * size) * (0.4 * size);
            break;
          }
          default:
            in = std::fabs(x) <= size * 0.9 && std::fabs(y) <= size * 0.7 && std::fabs(z) <= size * 0.9;
        }
        if (in) {
          out.push_back(x);
          out.push_back(y);
          out.push_back(z);
        }
      }
}

void boundary_points(const double box[3], double rho0, double d, double h, std::vector<double>& pts,
                     std::vector<float>& psi) {
  int nb[3];
  double step[3];
  for (int k = 0; k < 3; k++) {
    nb[k] = (int)std::max(2.0, std::ceil(box[k] / d) + 1);
    step[k] = box[k] / (nb[k] - 1);
  }
  pts.clear();
  for (int ix = 0; ix < nb[0]; ix++)
    for (int iy = 0; iy < nb[1]; iy++)
      for (int iz = 0; iz < nb[2]; iz++) {
        if (ix == 0 || ix == nb[0] - 1 || iy == 0 || iy == nb[1] - 1 || iz == 0 || iz == nb[2] - 1) {
          pts.push_back(ix * step[0]);
          pts.push_back(iy * step[1]);
          pts.push_back(iz * step[2]);
        }
      }
  const int n = (int)(pts.size() / 3);
  // The boundary's own bucket grid uses ceil(size / h) cells (src/scene.js:90).
  int dim[3];
  for (int k = 0; k < 3; k++) dim[k] = (int)std::max(1.0, std::ceil(box[k] / h));
  std::vector<uint32_t> cell(n), cx(n), cy(n), cz(n);
  for (int i = 0; i < n; i++) {
    cx[i] = clampi(std::floor(pts[i * 3] / h), dim[0] - 1);
    cy[i] = clampi(std::floor(pts[i * 3 + 1] / h), dim[1] - 1);
    cz[i] = clampi(std::floor(pts[i * 3 + 2] / h), dim[2] - 1);
    cell[i] = (cz[i] * dim[1] + cy[i]) * dim[0] + cx[i];
  }
  CellLists grid;
  grid.build(dim, n, cell);
  const double coef = 315 / (64 * kPi * std::pow(h, 9)), h2 = h * h;
  psi.assign(std::max(1, n), 0.0f);
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; i++) {
    double sum = 0;
    grid.around((int)cx[i], (int)cy[i], (int)cz[i], [&](int j) {
      const double dx = pts[i * 3] - pts[j * 3];
      const double dy = pts[i * 3 + 1] - pts[j * 3 + 1];
      const double dz = pts[i * 3 + 2] - pts[j * 3 + 2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 >= h2) return;
      const double t = h2 - r2;
      sum += t * t * t;
    });
    sum *= coef;
    psi[i] = (float)(sum > 0 ? rho0 / sum : 0);
  }
}

void build_boundary(const double box[3], double rho0, double d, double h, const int gridDim[3],
                    HostBoundary& out) {
  std::vector<double> pts;
  std::vector<float> psi;
  boundary_points(box, rho0, d, h, pts, psi);
  const int n = (int)(pts.size() / 3);
  const size_t cells = (size_t)gridDim[0] * gridDim[1] * gridDim[2];
  // sortBoundary (src/sim.js:255-286): cells of the float positions, stable.
  std::vector<float> f4((size_t)std::max(1, n) * 4, 0.0f);
  std::vector<uint32_t> cell(n);
  out.cellStart.assign(cells + 2, 0u);
  for (int i = 0; i < n; i++) {
    int c[3];
    for (int k = 0; k < 3; k++) {
      f4[i * 4 + k] = (float)pts[i * 3 + k];
      c[k] = clampi(std::floor((double)f4[i * 4 + k] / h), gridDim[k] - 1);
    }
    cell[i] = (uint32_t)((c[2] * gridDim[1] + c[1]) * gridDim[0] + c[0]);
    out.cellStart[cell[i] + 1]++;
  }
  for (size_t c = 0; c < cells; c++) out.cellStart[c + 1] += out.cellStart[c];
  out.cellStart[cells + 1] = (uint32_t)n;
  std::vector<uint32_t> at(out.cellStart.begin(), out.cellStart.begin() + cells);
  out.pos.assign((size_t)std::max(1, n) * 4, 0.0f);
  out.psi.assign(std::max(1, n), 0.0f);
  for (int i = 0; i < n; i++) {
    const uint32_t o = at[cell[i]]++;
    std::memcpy(&out.pos[o * 4], &f4[i * 4], 3 * sizeof(float));
    out.psi[o] = psi[i];
  }
  out.count = n;
}

void calibrate_scene(const p4a_params& p, HostScene& sc, bool doMass, bool doDenom) {
  const double h = sc.h, d = sc.d, rho0 = p.rest_density;
  const int nF = sc.nFluid;
  const double coef = 315 / (64 * kPi * std::pow(h, 9)), h2 = h * h;
  const double spiky = -45 / (kPi * std::pow(h, 6));
  int dim[3];
  for (int k = 0; k < 3; k++) dim[k] = (int)std::max(1.0, std::floor(p.box[k] / h));
  std::vector<uint32_t> cell(nF);
  std::vector<int> c3((size_t)nF * 3);
  for (int i = 0; i < nF; i++) {
    for (int k = 0; k < 3; k++) c3[i * 3 + k] = clampi(std::floor((double)sc.pos[i * 4 + k] / h), dim[k] - 1);
    cell[i] = (uint32_t)((c3[i * 3 + 2] * dim[1] + c3[i * 3 + 1]) * dim[0] + c3[i * 3]);
  }
  CellLists grid;
  grid.build(dim, nF, cell);
  const float* P = sc.pos.data();
  auto density = [&](int i, double m) {
    double rho = m * coef * h2 * h2 * h2;
    grid.around(c3[i * 3], c3[i * 3 + 1], c3[i * 3 + 2], [&](int j) {
      if (j == i) return;
      const double dx = (double)P[i * 4] - P[j * 4], dy = (double)P[i * 4 + 1] - P[j * 4 + 1],
                   dz = (double)P[i * 4 + 2] - P[j * 4 + 2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 >= h2) return;
      const double t = h2 - r2;
      rho += m * coef * t * t * t;
    });
    return rho;
  };
  if (doMass) {
    double mass = rho0 * d * d * d;
    const double m0 = mass;
    double maxRho = 0;
#pragma omp parallel for reduction(max : maxRho) schedule(dynamic, 512)
    for (int i = 0; i < nF; i++) maxRho = std::max(maxRho, density(i, m0));
    if (maxRho > 0.5 * rho0) mass *= rho0 / maxRho;
    sc.mass = mass;
  }
  if (doDenom) {
    const double volume = sc.mass / rho0;
    double denomRest = 0;
    for (int i = 0; i < nF; i++) {
      if (density(i, sc.mass) < 0.99 * rho0) continue;
      double gx = 0, gy = 0, gz = 0, g2 = 0;
      grid.around(c3[i * 3], c3[i * 3 + 1], c3[i * 3 + 2], [&](int j) {
        if (j == i) return;
        const double rx = (double)P[i * 4] - P[j * 4], ry = (double)P[i * 4 + 1] - P[j * 4 + 1],
                     rz = (double)P[i * 4 + 2] - P[j * 4 + 2];
        const double r2 = rx * rx + ry * ry + rz * rz;
        if (r2 < 1e-12 || r2 >= h2) return;
        const double r = std::sqrt(r2), hr = h - r;
        const double s = volume * spiky * hr * hr / r;
        gx += s * rx;
        gy += s * ry;
        gz += s * rz;
        g2 += s * s * r2;
      });
      denomRest = std::max(denomRest, gx * gx + gy * gy + gz * gz + g2);
      if (i > 2000 && denomRest > 0) break;
    }
    sc.denomRest = denomRest;
  }
}

void build_scene(const p4a_params& p, HostScene& sc) {
  const double d = p.spacing, h = 2 * d;
  const double bx = p.box[0], by = p.box[1], bz = p.box[2];
  std::vector<double> fluid;
  fluid_block(p, d, fluid);
  const int nFluid = (int)(fluid.size() / 3);
  const int nSpec = p.bodies ? p.n_bodies : 0;
  const double size = p.body_size > 0 ? p.body_size : 0.12 * std::min(bx, std::min(by, bz));
  const double step = std::min(2.5 * size, bx * 0.25);
  const double span = step * (nSpec - 1);
  std::vector<double> bodyPts, bodyRest, local;
  std::vector<uint32_t> ids;
  sc = HostScene();
  for (int r = 0; r < nSpec; r++) {
    const p4a_body_spec& sp = p.bodies[r];
    sample_body(sp.shape, size, d, local);
    const int cnt = (int)(local.size() / 3);
    if (!cnt) continue;
    // Number(x) || default (src/scene.js:169-170)
    const double dens = (sp.density != 0 && sp.density == sp.density) ? sp.density : 0.5;
    const double sy = (sp.start_y != 0 && sp.start_y == sp.start_y) ? sp.start_y : 0.75;
    const double centre[3] = {0.5 * bx - 0.5 * span + step * r, by * sy, bz * 0.5};
    double m[3] = {0, 0, 0};
    for (int i = 0; i < cnt; i++)
      for (int k = 0; k < 3; k++) m[k] += local[i * 3 + k];
    for (int k = 0; k < 3; k++) m[k] /= cnt;
    const uint32_t id = (uint32_t)sc.bodyCount.size() + 1;
    for (int i = 0; i < cnt; i++) {
      for (int k = 0; k < 3; k++) {
        bodyPts.push_back(centre[k] + local[i * 3 + k]);
        bodyRest.push_back(local[i * 3 + k] - m[k]);
      }
      ids.push_back(id);
    }
    sc.bodyCentre.insert(sc.bodyCentre.end(), centre, centre + 3);
    sc.bodyDensity.push_back(dens);
    sc.bodyCount.push_back(cnt);
  }
  const int nBody = (int)ids.size();
  sc.n = nFluid + nBody;
  sc.nFluid = nFluid;
  sc.nBody = nBody;
  sc.h = h;
  sc.d = d;
  sc.pos.assign((size_t)sc.n * 4, 0.0f);
  sc.vel.assign((size_t)sc.n * 4, 0.0f);
  sc.rest.assign((size_t)sc.n * 4, 0.0f);
  sc.phase.assign((size_t)sc.n * 4, 0u);
  for (int i = 0; i < nFluid; i++)
    for (int k = 0; k < 3; k++) sc.pos[(size_t)i * 4 + k] = (float)fluid[i * 3 + k];
  for (int i = 0; i < nBody; i++) {
    const size_t o = (size_t)(nFluid + i) * 4;
    for (int k = 0; k < 3; k++) {
      sc.pos[o + k] = (float)bodyPts[i * 3 + k];
      sc.rest[o + k] = (float)bodyRest[i * 3 + k];
    }
    sc.phase[o] = ids[i];
  }
  calibrate_scene(p, sc, true, true);
}

}  // namespace p4a

extern "C" int p4a_build_scene(const p4a_params* params, p4a_scene_counts* counts, float* pos,
                               float* vel, float* rest, uint32_t* phase, double* body_centre,
                               double* body_density) {
  if (!params || !counts || !(params->spacing > 0)) return P4A_ERR_ARG;
  p4a::HostScene sc;
  p4a::build_scene(*params, sc);
  std::vector<double> pts;
  std::vector<float> psi;
  const double h = sc.h;
  // Boundary count only (src/scene.js:78-88).
  int nb = 1;
  int inner = 1;
  for (int k = 0; k < 3; k++) {
    const int m = (int)std::max(2.0, std::ceil(params->box[k] / params->spacing) + 1);
    nb *= m;
    inner *= std::max(0, m - 2);
  }
  counts->n = sc.n;
  counts->n_fluid = sc.nFluid;
  counts->n_body = sc.nBody;
  counts->n_bodies = (int32_t)sc.bodyDensity.size();
  counts->n_boundary = nb - inner;
  counts->mass = sc.mass;
  counts->denom_rest = sc.denomRest;
  counts->h = h;
  if (pos) std::memcpy(pos, sc.pos.data(), sc.pos.size() * sizeof(float));
  if (vel) std::memcpy(vel, sc.vel.data(), sc.vel.size() * sizeof(float));
  if (rest) std::memcpy(rest, sc.rest.data(), sc.rest.size() * sizeof(float));
  if (phase) std::memcpy(phase, sc.phase.data(), sc.phase.size() * sizeof(uint32_t));
  if (body_centre) std::memcpy(body_centre, sc.bodyCentre.data(), sc.bodyCentre.size() * sizeof(double));
  if (body_density) std::memcpy(body_density, sc.bodyDensity.data(), sc.bodyDensity.size() * sizeof(double));
  return P4A_OK;
}
