// p4a_oracle.cpp — CPU restatement of the Particles4All simulation step.
//
// TEST INFRASTRUCTURE (what the product's results are compared against, and the
// timed CPU baseline), never the product.
// PARITY UNPINNED: the reference cannot run here and ships no golden vectors; see
// p4a_oracle.h for what pins this restatement instead.
//
// Structure mirrors the reference one pass at a time, in the reference's schedule:
//   scene setup        src/scene.js:41-315
//   Sim.reset / prime  src/sim.js:66-286
//   uniform packing    src/sim.js:371-413   (Params layout src/wgsl.js:4-40)
//   Sim.step           src/sim.js:415-656
//   passes             src/wgsl.js:43-832
//   anisotropic pass   src/aniso_wgsl.js:3-158 with params src/mesh.js:207-242
// Build with -ffp-contract=off: the only fused multiply-adds are the explicit fmaf
// calls of the arithmetic contract (p4a_oracle.h).
#include "p4a_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct f4 { float x, y, z, w; };
struct u4 { uint32_t x, y, z, w; };
struct f3 { float x, y, z; };

const double kPI = 3.14159265358979323846;  // Math.PI

inline f3 xyz(const f4& v) { return {v.x, v.y, v.z}; }
inline f3 sub3(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline f3 add3(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline f3 mul3(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot3(f3 a, f3 b) { return std::fmaf(a.z, b.z, std::fmaf(a.y, b.y, a.x * b.x)); }
inline f3 fma3(float s, f3 v, f3 acc) {
  return {std::fmaf(s, v.x, acc.x), std::fmaf(s, v.y, acc.y), std::fmaf(s, v.z, acc.z)};
}
inline f3 cross3(f3 b, f3 c) {
  return {b.y * c.z - b.z * c.y, b.z * c.x - b.x * c.z, b.x * c.y - b.y * c.x};
}
inline float length3(f3 a) { return std::sqrt(dot3(a, a)); }

// f32 -> i32 with the semantics of the GPU's cvt.rzi / cvt.rni (saturating, NaN -> 0).
inline int32_t f2i_sat(float f) {
  if (f != f) return 0;
  if (f >= 2147483648.0f) return INT32_MAX;
  if (f <= -2147483648.0f) return INT32_MIN;
  return (int32_t)f;
}
inline uint32_t f2u_sat(float f) {
  if (!(f > 0.0f)) return 0u;
  if (f >= 4294967296.0f) return UINT32_MAX;
  return (uint32_t)f;
}
// i32(round(x)) of WGSL: round half to even, then the saturating conversion.
inline int32_t round_i32(float x) { return f2i_sat(std::nearbyint(x)); }

// Column-major 3x3 (m[c] is column c), as WGSL's mat3x3f.
struct m3 { f3 c[3]; };
inline m3 ident3() { return {{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}}; }
inline float det3(const m3& a) { return dot3(a.c[0], cross3(a.c[1], a.c[2])); }
inline f3 row3(const m3& a, int r) {
  const float* c0 = &a.c[0].x; const float* c1 = &a.c[1].x; const float* c2 = &a.c[2].x;
  return {c0[r], c1[r], c2[r]};
}
inline float& el(m3& a, int c, int r) { return (&a.c[c].x)[r]; }
inline float elc(const m3& a, int c, int r) { return (&a.c[c].x)[r]; }
inline m3 matmul(const m3& A, const m3& B) {  // (A*B)[c][r] = dot3(row r of A, col c of B)
  m3 o;
  for (int c = 0; c < 3; c++)
    for (int r = 0; r < 3; r++) el(o, c, r) = dot3(row3(A, r), B.c[c]);
  return o;
}
inline m3 transpose3(const m3& a) {
  m3 o;
  for (int c = 0; c < 3; c++)
    for (int r = 0; r < 3; r++) el(o, c, r) = elc(a, r, c);
  return o;
}
inline m3 scale3(const m3& a, float s) {
  m3 o;
  for (int c = 0; c < 3; c++) o.c[c] = mul3(a.c[c], s);
  return o;
}

// Cube root by a fixed Newton iteration on the mantissa (x > 0, normal): the
// rigid-body resolve's pow(|det|, 1/3) (src/wgsl.js:730). Only IEEE basic
// operations, so every conforming float32 unit gives the same bits.
float cbrt_newton(float x) {
  if (!(x > 0.0f) || std::isinf(x)) return x;
  uint32_t bits;
  std::memcpy(&bits, &x, 4);
  int e = (int)((bits >> 23) & 0xffu);
  if (e == 0) return 0.0f;  // subnormal: not reached by the callers (|det| >= 1e-12)
  e -= 127;
  int q = (e + 300) / 3 - 100;  // floor(e / 3)
  int r = e - 3 * q;            // 0, 1, 2
  uint32_t mb = (bits & 0x7fffffu) | 0x3f800000u;
  float m;
  std::memcpy(&m, &mb, 4);
  float t = m;  // [1, 2)
  if (r >= 1) t = t * 2.0f;
  if (r >= 2) t = t * 2.0f;  // t in [1, 8)
  float y = 0.75f + 0.1666667f * t;
  for (int it = 0; it < 5; it++) y = (2.0f * y + t / (y * y)) * 0.33333334f;
  uint32_t sb = (uint32_t)(q + 127) << 23;
  float s;
  std::memcpy(&s, &sb, 4);
  return y * s;
}

// The 192-byte uniform (src/wgsl.js:4-40) as float32 / int32.
struct Params {
  float boxMin[3]; float dt;
  float boxMax[3]; float h;
  int32_t gridDim[3]; float h2;
  float clampMin[3]; float poly6;
  float clampMax[3]; float spikyGrad;
  float gravity, mass, rho0, invRho0;
  float cfmEps, sCorrK, sCorrWq, xsphC;
  uint32_t n, nCells, nBoundary, nBodyParts;
  uint32_t nBodies; float bodyScale, covScale, omega;
  uint32_t sorAverage; float invDt, volume, tension;
  float cohes, cohesTerm;
};

int g_threads = 0;
inline void apply_threads() {
#ifdef _OPENMP
  if (g_threads > 0) omp_set_num_threads(g_threads);
#endif
}

// ---------------------------------------------------------------- scene.js
struct Scene {
  int n = 0, nFluid = 0, nBody = 0;
  std::vector<float> pos, vel, rest;  // float4
  std::vector<uint32_t> phase;        // uint4
  std::vector<double> bodyCentre, bodyDensity;
  std::vector<int> bodyCount;
  double mass = 0, denomRest = 0, h = 0, d = 0;
};

inline double poly6Coef(double h) { return 315 / (64 * kPI * std::pow(h, 9)); }

// fluidBlock (src/scene.js:43-64). The LCG runs in float64 like the JS, whose
// seed*1103515245 is a rounded double product, then ToInt32 & 0x7fffffff.
std::vector<double> fluidBlock(const p4a_params& p, double d) {
  const double bx = p.box[0], by = p.box[1], bz = p.box[2];
  const double margin = d;
  const double nx = std::max(1.0, std::floor(bx * 0.35 / d));
  const double nz = std::max(1.0, std::floor((bz - 2 * margin) / d));
  const double maxLayers = std::max(1.0, std::floor((by - 2 * margin) / d));
  const double target = p.target_particle_count;
  const double layers = std::min(std::ceil(target / (nx * nz)), maxLayers);
  std::vector<double> out;
  double seed = 12345;
  auto rnd = [&]() {
    double s = seed * 1103515245.0 + 12345.0;
    int64_t si = (int64_t)s;  // integral, |s| < 2^63
    seed = (double)(int32_t)((uint32_t)si & 0x7fffffffu);
    return (seed / 2147483647.0 - 0.5) * 0.002 * d;
  };
  for (double iy = 0; iy < layers && out.size() / 3 < target; iy++)
    for (double ix = 0; ix < nx && out.size() / 3 < target; ix++)
      for (double iz = 0; iz < nz && out.size() / 3 < target; iz++) {
        double x = margin + (ix + 0.5) * d + rnd();
        double y = margin + (iy + 0.5) * d + rnd();
        double z = margin + (iz + 0.5) * d + rnd();
        out.push_back(x); out.push_back(y); out.push_back(z);
      }
  return out;
}

// sampleBody (src/scene.js:137-157).
std::vector<double> sampleBody(int shape, double size, double d) {
  double ext[3];
  if (shape == P4A_SHAPE_SPHERE) { ext[0] = ext[1] = ext[2] = size; }
  else if (shape == P4A_SHAPE_TORUS) { ext[0] = size + 0.4 * size; ext[1] = 0.4 * size; ext[2] = size + 0.4 * size; }
  else { ext[0] = size * 0.9; ext[1] = size * 0.7; ext[2] = size * 0.9; }
  int steps[3];
  for (int k = 0; k < 3; k++) steps[k] = (int)std::max(1.0, std::ceil(ext[k] / d));
  std::vector<double> local;
  for (int ix = -steps[0]; ix <= steps[0]; ix++)
    for (int iy = -steps[1]; iy <= steps[1]; iy++)
      for (int iz = -steps[2]; iz <= steps[2]; iz++) {
        double x = ix * d, y = iy * d, z = iz * d;
        bool inside;
        if (shape == P4A_SHAPE_SPHERE) inside = x * x + y * y + z * z <= size * size;
        else if (shape == P4A_SHAPE_TORUS) {
          double planar = std::sqrt(x * x + z * z) - size;
          inside = planar * planar + y * y <= (0.4 * size) * (0.4 * size);
        } else inside = std::fabs(x) <= size * 0.9 && std::fabs(y) <= size * 0.7 && std::fabs(z) <= size * 0.9;
        if (inside) { local.push_back(x); local.push_back(y); local.push_back(z); }
      }
  return local;
}

// Cell buckets in insertion (index) order, as the JS Map of arrays keeps them.
struct Buckets {
  std::vector<uint32_t> start, items;
  template <class KeyFn>
  void build(int n, int64_t nkeys, KeyFn key) {
    start.assign((size_t)nkeys + 1, 0u);
    std::vector<int64_t> k(n);
    for (int i = 0; i < n; i++) { k[i] = key(i); start[k[i] + 1]++; }
    for (int64_t c = 0; c < nkeys; c++) start[c + 1] += start[c];
    items.assign(n, 0u);
    std::vector<uint32_t> cur(start.begin(), start.end() - 1);
    for (int i = 0; i < n; i++) items[cur[k[i]]++] = (uint32_t)i;
  }
};

// boundaryParticles (src/scene.js:76-135): shell samples and psi = rho0 / sum W.
void boundaryParticles(const double box[3], double rho0, double d, double h,
                       std::vector<double>& pts, std::vector<float>& psi) {
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
        bool shell = ix == 0 || ix == nb[0] - 1 || iy == 0 || iy == nb[1] - 1 || iz == 0 || iz == nb[2] - 1;
        if (shell) { pts.push_back(ix * step[0]); pts.push_back(iy * step[1]); pts.push_back(iz * step[2]); }
      }
  const int n = (int)(pts.size() / 3);
  int dim[3];
  for (int k = 0; k < 3; k++) dim[k] = (int)std::max(1.0, std::ceil(box[k] / h));
  auto cellOf = [&](double x, double y, double z, int c[3]) {
    c[0] = (int)std::min<double>(dim[0] - 1, std::max(0.0, std::floor(x / h)));
    c[1] = (int)std::min<double>(dim[1] - 1, std::max(0.0, std::floor(y / h)));
    c[2] = (int)std::min<double>(dim[2] - 1, std::max(0.0, std::floor(z / h)));
  };
  auto key = [&](int a, int b, int c) { return ((int64_t)c * dim[1] + b) * dim[0] + a; };
  Buckets buckets;
  buckets.build(n, (int64_t)dim[0] * dim[1] * dim[2], [&](int i) {
    int c[3];
    cellOf(pts[i * 3], pts[i * 3 + 1], pts[i * 3 + 2], c);
    return key(c[0], c[1], c[2]);
  });
  const double coef = poly6Coef(h), h2 = h * h;
  psi.assign(std::max(1, n), 0.0f);
  apply_threads();
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; i++) {
    int c[3];
    cellOf(pts[i * 3], pts[i * 3 + 1], pts[i * 3 + 2], c);
    double sum = 0;
    for (int dc = -1; dc <= 1; dc++) {
      if (c[2] + dc < 0 || c[2] + dc >= dim[2]) continue;
      for (int db = -1; db <= 1; db++) {
        if (c[1] + db < 0 || c[1] + db >= dim[1]) continue;
        for (int da = -1; da <= 1; da++) {
          if (c[0] + da < 0 || c[0] + da >= dim[0]) continue;
          const int64_t kk = key(c[0] + da, c[1] + db, c[2] + dc);
          for (uint32_t m = buckets.start[kk]; m < buckets.start[kk + 1]; m++) {
            const int j = (int)buckets.items[m];
            double dx = pts[i * 3] - pts[j * 3];
            double dy = pts[i * 3 + 1] - pts[j * 3 + 1];
            double dz = pts[i * 3 + 2] - pts[j * 3 + 2];
            double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 >= h2) continue;
            double t = h2 - r2;
            sum += t * t * t;
          }
        }
      }
    }
    sum *= coef;
    psi[i] = (float)(sum > 0 ? rho0 / sum : 0);
  }
}

// Mass calibration and denomRest (src/scene.js:232-311) over the fluid particles
// [0, nFluid) of a float4 position array.
void calibrate(const std::vector<float>& pos, int nFluid, double d, double h, double rho0,
               bool doMass, bool doDenom, double& mass, double& denomRest, const double box[3]) {
  const double coef = poly6Coef(h), h2 = h * h;
  const double spiky = -45 / (kPI * std::pow(h, 6));
  int dim[3];
  for (int k = 0; k < 3; k++) dim[k] = (int)std::max(1.0, std::floor(box[k] / h));
  auto cellOf = [&](int i, int c[3]) {
    for (int k = 0; k < 3; k++)
      c[k] = (int)std::min<double>(dim[k] - 1, std::max(0.0, std::floor((double)pos[i * 4 + k] / h)));
  };
  auto key = [&](int a, int b, int c) { return ((int64_t)c * dim[1] + b) * dim[0] + a; };
  Buckets buckets;
  buckets.build(nFluid, (int64_t)dim[0] * dim[1] * dim[2], [&](int i) {
    int c[3];
    cellOf(i, c);
    return key(c[0], c[1], c[2]);
  });
  auto forEach = [&](int i, auto&& f) {
    int c[3];
    cellOf(i, c);
    for (int dc = -1; dc <= 1; dc++) {
      if (c[2] + dc < 0 || c[2] + dc >= dim[2]) continue;
      for (int db = -1; db <= 1; db++) {
        if (c[1] + db < 0 || c[1] + db >= dim[1]) continue;
        for (int da = -1; da <= 1; da++) {
          if (c[0] + da < 0 || c[0] + da >= dim[0]) continue;
          const int64_t kk = key(c[0] + da, c[1] + db, c[2] + dc);
          for (uint32_t m = buckets.start[kk]; m < buckets.start[kk + 1]; m++) {
            const int j = (int)buckets.items[m];
            if (j != i) f(j);
          }
        }
      }
    }
  };
  auto densityAt = [&](int i, double m) {
    double rho = m * coef * h2 * h2 * h2;
    forEach(i, [&](int j) {
      double dx = (double)pos[i * 4] - pos[j * 4], dy = (double)pos[i * 4 + 1] - pos[j * 4 + 1],
             dz = (double)pos[i * 4 + 2] - pos[j * 4 + 2];
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 >= h2) return;
      double t = h2 - r2;
      rho += m * coef * t * t * t;
    });
    return rho;
  };
  apply_threads();
  if (doMass) {
    mass = rho0 * d * d * d;
    double maxRho = 0;
    const double m0 = mass;
#pragma omp parallel for reduction(max : maxRho) schedule(dynamic, 512)
    for (int i = 0; i < nFluid; i++) maxRho = std::max(maxRho, densityAt(i, m0));
    if (maxRho > 0.5 * rho0) mass *= rho0 / maxRho;
  }
  if (doDenom) {
    denomRest = 0;
    const double volume = mass / rho0;
    for (int i = 0; i < nFluid; i++) {
      if (densityAt(i, mass) < 0.99 * rho0) continue;
      double gx = 0, gy = 0, gz = 0, sumGrad2 = 0;
      forEach(i, [&](int j) {
        double rx = (double)pos[i * 4] - pos[j * 4], ry = (double)pos[i * 4 + 1] - pos[j * 4 + 1],
               rz = (double)pos[i * 4 + 2] - pos[j * 4 + 2];
        double r2 = rx * rx + ry * ry + rz * rz;
        if (r2 < 1e-12 || r2 >= h2) return;
        double r = std::sqrt(r2), hr = h - r;
        double s = volume * spiky * hr * hr / r;
        gx += s * rx; gy += s * ry; gz += s * rz;
        sumGrad2 += s * s * r2;
      });
      denomRest = std::max(denomRest, gx * gx + gy * gy + gz * gz + sumGrad2);
      if (i > 2000 && denomRest > 0) break;
    }
  }
}

// buildScene (src/scene.js:159-315).
void buildScene(const p4a_params& p, Scene& sc) {
  const double d = p.spacing, h = 2 * d;
  const double bx = p.box[0], by = p.box[1], bz = p.box[2];
  std::vector<double> fluid = fluidBlock(p, d);
  const int nFluid = (int)(fluid.size() / 3);
  const double sz = p.body_size > 0 ? p.body_size : 0.12 * std::min(bx, std::min(by, bz));
  const int nspec = p.bodies ? p.n_bodies : 0;
  const double step = std::min(2.5 * sz, bx * 0.25);
  const double span = step * (nspec - 1);
  std::vector<double> bodyPts, bodyRest;
  std::vector<uint32_t> bodyPhase;
  sc.bodyCentre.clear(); sc.bodyDensity.clear(); sc.bodyCount.clear();
  for (int r = 0; r < nspec; r++) {
    const p4a_body_spec& spec = p.bodies[r];
    std::vector<double> local = sampleBody(spec.shape, sz, d);
    const int count = (int)(local.size() / 3);
    if (!count) continue;
    double density = spec.density != 0 && spec.density == spec.density ? spec.density : 0.5;
    double startY = spec.start_y != 0 && spec.start_y == spec.start_y ? spec.start_y : 0.75;
    double centre[3] = {0.5 * bx - 0.5 * span + step * r, by * startY, bz * 0.5};
    double cx = 0, cy = 0, cz = 0;
    for (int i = 0; i < count; i++) { cx += local[i * 3]; cy += local[i * 3 + 1]; cz += local[i * 3 + 2]; }
    cx /= count; cy /= count; cz /= count;
    const uint32_t id = (uint32_t)sc.bodyCount.size() + 1;
    for (int i = 0; i < count; i++) {
      double lx = local[i * 3], ly = local[i * 3 + 1], lz = local[i * 3 + 2];
      bodyPts.push_back(centre[0] + lx); bodyPts.push_back(centre[1] + ly); bodyPts.push_back(centre[2] + lz);
      bodyRest.push_back(lx - cx); bodyRest.push_back(ly - cy); bodyRest.push_back(lz - cz);
      bodyPhase.push_back(id);
    }
    sc.bodyCentre.insert(sc.bodyCentre.end(), centre, centre + 3);
    sc.bodyDensity.push_back(density);
    sc.bodyCount.push_back(count);
  }
  const int nBody = (int)(bodyPts.size() / 3);
  const int n = nFluid + nBody;
  sc.n = n; sc.nFluid = nFluid; sc.nBody = nBody; sc.h = h; sc.d = d;
  sc.pos.assign((size_t)n * 4, 0.0f); sc.vel.assign((size_t)n * 4, 0.0f);
  sc.rest.assign((size_t)n * 4, 0.0f); sc.phase.assign((size_t)n * 4, 0u);
  for (int i = 0; i < nFluid; i++)
    for (int k = 0; k < 3; k++) sc.pos[i * 4 + k] = (float)fluid[i * 3 + k];
  for (int i = 0; i < nBody; i++) {
    size_t o = (size_t)(nFluid + i) * 4;
    for (int k = 0; k < 3; k++) {
      sc.pos[o + k] = (float)bodyPts[i * 3 + k];
      sc.rest[o + k] = (float)bodyRest[i * 3 + k];
    }
    sc.phase[o] = bodyPhase[i];
  }
  calibrate(sc.pos, nFluid, d, h, p.rest_density, true, true, sc.mass, sc.denomRest, p.box);
}

// ------------------------------------------------------------------- Sim
struct SimState;
}  // namespace

struct orc_sim {
  p4a_params params{};
  std::vector<p4a_body_spec> specs;
  Scene sc;
  int n = 0, cap = 0, pourBudget = 0, nBoundary = 0, nBodies = 0, nBodyParts = 0;
  double h = 0;
  int gridDim[3] = {1, 1, 1};
  int nCells = 1;
  std::vector<f4> pos[2], vel[2], pred[2], rest[2];
  std::vector<u4> body[2];
  std::vector<float> lambda, density;
  std::vector<uint32_t> slot;
  std::vector<f4> corr, normal;
  std::vector<uint32_t> cellCount, cellStart, cursor;
  std::vector<f4> bpos;
  std::vector<float> bpsi;
  std::vector<uint32_t> bcellStart;
  std::vector<int32_t> bodyAccum, bodyCov;
  std::vector<f4> bodyCentre, bodyRef, bodyRot, bodyInfo;
  std::vector<uint32_t> bodyIdx;
  uint32_t bodyIdxCount = 0;
  double bodyScale = 0, covScale = 0;
  std::vector<uint32_t> statsOut = std::vector<uint32_t>(8, 0u);
  int parity = 0, predParity = 0, gen = 0;
  double simTime = 0, timeBank = 0, lastAdvanced = 0;
  int lastSubsteps = 0;
  int heldBody = -1;
  double heldTarget[3] = {0, 0, 0}, heldRate = 10, heldLimit = 4;
  Params P{};
  p4a_stats stats{};
  std::vector<f4> smoothPos, anisoG;
  int anisoGen = 0;
  std::vector<float> ssfrEyeZ, ssfrRaw, ssfrThick, ssfrBodyT;
  std::vector<uint32_t> ssfrImage;
  int ssfrDims[6] = {0, 0, 0, 0, 0, 0};
  std::vector<float> meshField, meshNField;
  int meshDim[3] = {0, 0, 0};
  double meshOrigin = 0, meshVoxel = 0;
  std::vector<uint32_t> rayImage;
  int rayDims[2] = {0, 0};
  std::vector<uint32_t> meshVerts;  // 2 words per vertex
  std::vector<uint16_t> envCube;    // 6 faces of envSize^2 texels, 4 halves each
  int envSize = 0;
  int64_t meshTris = 0;
  bool ready = false;
};

namespace {

// uploadParams(dt) (src/sim.js:371-413).
void uploadParams(orc_sim* s, double dt) {
  const p4a_params& p = s->params;
  Params& F = s->P;
  const double h = s->h, d = p.spacing;
  F.boxMin[0] = F.boxMin[1] = F.boxMin[2] = 0;
  F.dt = (float)dt;
  for (int k = 0; k < 3; k++) F.boxMax[k] = (float)p.box[k];
  F.h = (float)h;
  for (int k = 0; k < 3; k++) F.gridDim[k] = s->gridDim[k];
  F.h2 = (float)(h * h);
  const double halfD = 0.5 * d;
  for (int k = 0; k < 3; k++) F.clampMin[k] = (float)halfD;
  const double poly6 = 315 / (64 * kPI * std::pow(h, 9));
  F.poly6 = (float)poly6;
  for (int k = 0; k < 3; k++) F.clampMax[k] = (float)(p.box[k] - halfD);
  F.spikyGrad = (float)(-45 / (kPI * std::pow(h, 6)));
  F.gravity = (float)p.gravity;
  F.mass = (float)s->sc.mass;
  F.rho0 = (float)p.rest_density;
  F.invRho0 = (float)(1 / p.rest_density);
  F.cfmEps = (float)(p.cfm_epsilon_abs > 0 ? p.cfm_epsilon_abs
                                           : std::max(1e-9, p.cfm_epsilon_rel * s->sc.denomRest));
  F.sCorrK = (float)(p.s_corr_k / (s->sc.denomRest * std::max(1, p.iterations)));
  const double rq = p.s_corr_dq * h, tq = h * h - rq * rq;
  const double wq = poly6 * tq * tq * tq;
  F.sCorrWq = (float)(wq > 0 ? 1 / wq : 0);
  F.xsphC = (float)p.xsph_c;
  F.n = (uint32_t)s->n;
  F.nCells = (uint32_t)s->nCells;
  F.nBoundary = p.no_boundary ? 0u : (uint32_t)s->nBoundary;
  F.nBodyParts = (uint32_t)s->nBodyParts;
  F.nBodies = (uint32_t)s->nBodies;
  F.bodyScale = (float)s->bodyScale;
  F.covScale = (float)s->covScale;
  F.omega = (float)p.omega;
  F.sorAverage = p.sor_average ? 1u : 0u;
  F.invDt = (float)(dt > 0 ? 1 / dt : 0);
  F.volume = (float)(s->sc.mass / p.rest_density);
  F.tension = (float)p.surface_tension_k;
  F.cohes = (float)(32 / (kPI * std::pow(h, 9)));
  F.cohesTerm = (float)(std::pow(h, 6) / 64);
}

// cellOf / cellIndex (src/wgsl.js:43-49).
struct I3 { int x, y, z; };
inline I3 cellOf(const Params& P, f3 p) {
  I3 c;
  c.x = f2i_sat(std::floor((p.x - P.boxMin[0]) / P.h));
  c.y = f2i_sat(std::floor((p.y - P.boxMin[1]) / P.h));
  c.z = f2i_sat(std::floor((p.z - P.boxMin[2]) / P.h));
  c.x = std::min(std::max(c.x, 0), P.gridDim[0] - 1);
  c.y = std::min(std::max(c.y, 0), P.gridDim[1] - 1);
  c.z = std::min(std::max(c.z, 0), P.gridDim[2] - 1);
  return c;
}
inline uint32_t cellIndex(const Params& P, I3 c) {
  return (uint32_t)((c.z * P.gridDim[1] + c.y) * P.gridDim[0] + c.x);
}
inline float poly6(const Params& P, float r2) {
  float t = P.h2 - r2;
  return r2 < P.h2 ? P.poly6 * t * t * t : 0.0f;
}

// predict (src/wgsl.js:56-70).
void k_predict(const Params& P, std::vector<f4>& pos, std::vector<f4>& vel, std::vector<f4>& pred) {
  const int n = (int)P.n;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    const float gx = P.dt * 0.0f, gy = P.dt * -P.gravity, gz = P.dt * 0.0f;
    f3 v = {vel[i].x + gx, vel[i].y + gy, vel[i].z + gz};
    vel[i] = {v.x, v.y, v.z, 0.0f};
    pred[i] = {pos[i].x + P.dt * v.x, pos[i].y + P.dt * v.y, pos[i].z + P.dt * v.z, 1.0f};
  }
}

// count + scanBlock + scanBlocks + scanAdd + scatterSlot (src/wgsl.js:352-438) with
// a stable slot order; cellCount/cursor cleared first (src/sim.js:475-476).
void k_sort_slots(const Params& P, const std::vector<f4>& pred, std::vector<uint32_t>& cellCount,
                  std::vector<uint32_t>& cellStart, std::vector<uint32_t>& cursor,
                  std::vector<uint32_t>& slot) {
  const int n = (int)P.n;
  const uint32_t C = P.nCells;
  std::fill(cellCount.begin(), cellCount.end(), 0u);
  std::fill(cursor.begin(), cursor.end(), 0u);
  std::vector<uint32_t> key(n);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) key[i] = cellIndex(P, cellOf(P, xyz(pred[i])));
  for (int i = 0; i < n; i++) cellCount[key[i]]++;
  uint32_t run = 0;
  for (uint32_t c = 0; c < C; c++) { cellStart[c] = run; run += cellCount[c]; }
  cellStart[C] = run;
  for (int i = 0; i < n; i++) slot[i] = cellStart[key[i]] + cursor[key[i]]++;
}

template <class T>
void k_scatter(int n, const std::vector<uint32_t>& slot, const std::vector<T>& src, std::vector<T>& dst) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) dst[slot[i]] = src[i];
}

// lambda (src/wgsl.js:477-543).
void k_lambda(const Params& P, const std::vector<f4>& pred, std::vector<float>& lambda,
              std::vector<float>& density, const std::vector<uint32_t>& cs, const std::vector<f4>& bpos,
              const std::vector<float>& bpsi, const std::vector<uint32_t>& bcs) {
  const int n = (int)P.n;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; i++) {
    const f3 pi = xyz(pred[i]);
    const I3 c = cellOf(P, pi);
    const int x0 = std::max(c.x - 1, 0), x1 = std::min(c.x + 1, P.gridDim[0] - 1);
    float rho = P.mass * poly6(P, 0.0f);
    f3 gradSum = {0, 0, 0};
    float sumGrad2 = 0.0f;
    for (int dz = -1; dz <= 1; dz++) {
      const int z = c.z + dz;
      if (z < 0 || z >= P.gridDim[2]) continue;
      for (int dy = -1; dy <= 1; dy++) {
        const int y = c.y + dy;
        if (y < 0 || y >= P.gridDim[1]) continue;
        const uint32_t rowBase = (uint32_t)((z * P.gridDim[1] + y) * P.gridDim[0]);
        const uint32_t b = cs[rowBase + x0], e = cs[rowBase + x1 + 1];
        for (uint32_t j = b; j < e; j++) {
          if (j == (uint32_t)i) continue;
          const f3 rij = sub3(pi, xyz(pred[j]));
          const float r2 = dot3(rij, rij);
          if (r2 >= P.h2) continue;
          rho = std::fmaf(P.mass, poly6(P, r2), rho);
          if (r2 > 1.0e-12f) {
            const float r = std::sqrt(r2);
            const float hr = P.h - r;
            const float s = P.volume * P.spikyGrad * hr * hr / r;
            const f3 g = mul3(rij, s);
            gradSum = add3(gradSum, g);
            sumGrad2 = sumGrad2 + dot3(g, g);
          }
        }
        if (P.nBoundary > 0u) {
          const uint32_t bb = bcs[rowBase + x0], be = bcs[rowBase + x1 + 1];
          for (uint32_t k = bb; k < be; k++) {
            const f3 rij = sub3(pi, xyz(bpos[k]));
            const float r2 = dot3(rij, rij);
            if (r2 >= P.h2 || r2 < 1.0e-12f) continue;
            rho = std::fmaf(bpsi[k], poly6(P, r2), rho);
            const float r = std::sqrt(r2);
            const float hr = P.h - r;
            const float s = bpsi[k] * P.invRho0 * P.spikyGrad * hr * hr / r;
            gradSum = fma3(s, rij, gradSum);
          }
        }
      }
    }
    density[i] = rho;
    const float C = rho * P.invRho0 - 1.0f;
    if (C > 0.0f) {
      const float den = dot3(gradSum, gradSum) + sumGrad2 + P.cfmEps + 1.0e-12f;
      lambda[i] = -C / den;
    } else {
      lambda[i] = 0.0f;
    }
  }
}

// delta (src/wgsl.js:545-612).
void k_delta(const Params& P, const std::vector<f4>& pred, std::vector<f4>& predOut,
             const std::vector<float>& lambda, const std::vector<uint32_t>& cs,
             const std::vector<f4>& bpos, const std::vector<float>& bpsi,
             const std::vector<uint32_t>& bcs) {
  const int n = (int)P.n;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; i++) {
    const f3 pi = xyz(pred[i]);
    const float li = lambda[i];
    const I3 c = cellOf(P, pi);
    const int x0 = std::max(c.x - 1, 0), x1 = std::min(c.x + 1, P.gridDim[0] - 1);
    f3 d = {0, 0, 0}, dB = {0, 0, 0};
    float nc = 1.0f;
    for (int dz = -1; dz <= 1; dz++) {
      const int z = c.z + dz;
      if (z < 0 || z >= P.gridDim[2]) continue;
      for (int dy = -1; dy <= 1; dy++) {
        const int y = c.y + dy;
        if (y < 0 || y >= P.gridDim[1]) continue;
        const uint32_t rowBase = (uint32_t)((z * P.gridDim[1] + y) * P.gridDim[0]);
        const uint32_t b = cs[rowBase + x0], e = cs[rowBase + x1 + 1];
        for (uint32_t j = b; j < e; j++) {
          if (j == (uint32_t)i) continue;
          const f3 rij = sub3(pi, xyz(pred[j]));
          const float r2 = dot3(rij, rij);
          if (r2 >= P.h2 || r2 < 1.0e-12f) continue;
          const float r = std::sqrt(r2);
          const float hr = P.h - r;
          const float s = P.spikyGrad * hr * hr / r;
          const float t = P.h2 - r2;
          const float ratio = P.poly6 * t * t * t * P.sCorrWq;
          const float r2r = ratio * ratio;
          const float sc = -P.sCorrK * r2r * r2r;
          const float coef = (li + lambda[j] + sc) * s;
          d = fma3(coef, rij, d);
          nc += 1.0f;
        }
        if (P.nBoundary > 0u) {
          const uint32_t bb = bcs[rowBase + x0], be = bcs[rowBase + x1 + 1];
          for (uint32_t k = bb; k < be; k++) {
            const f3 rij = sub3(pi, xyz(bpos[k]));
            const float r2 = dot3(rij, rij);
            if (r2 >= P.h2 || r2 < 1.0e-12f) continue;
            const float r = std::sqrt(r2);
            const float hr = P.h - r;
            const float coef = (li * bpsi[k]) * (P.spikyGrad * hr * hr / r);
            dB = fma3(coef, rij, dB);
          }
        }
      }
    }
    f3 dd = {std::fmaf(dB.x, P.invRho0, d.x * P.volume), std::fmaf(dB.y, P.invRho0, d.y * P.volume),
             std::fmaf(dB.z, P.invRho0, d.z * P.volume)};
    float scale = P.omega;
    if (P.sorAverage == 1u) scale = P.omega / std::max(nc, 1.0f);
    f3 o = fma3(scale, dd, pi);
    o.x = std::min(std::max(o.x, P.clampMin[0]), P.clampMax[0]);
    o.y = std::min(std::max(o.y, P.clampMin[1]), P.clampMax[1]);
    o.z = std::min(std::max(o.z, P.clampMin[2]), P.clampMax[2]);
    predOut[i] = {o.x, o.y, o.z, 1.0f};
  }
}

// velFromPos (src/wgsl.js:72-83).
void k_velFromPos(const Params& P, const std::vector<f4>& pos, std::vector<f4>& vel, const std::vector<f4>& pred) {
  const int n = (int)P.n;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++)
    vel[i] = {(pred[i].x - pos[i].x) * P.invDt, (pred[i].y - pos[i].y) * P.invDt,
              (pred[i].z - pos[i].z) * P.invDt, 0.0f};
}

// xsph (src/wgsl.js:85-123).
void k_xsph(const Params& P, const std::vector<f4>& pred, const std::vector<f4>& vel,
            const std::vector<float>& density, std::vector<f4>& corr, const std::vector<uint32_t>& cs) {
  const int n = (int)P.n;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; i++) {
    const f3 pi = xyz(pred[i]), vi = xyz(vel[i]);
    const I3 c = cellOf(P, pi);
    const int x0 = std::max(c.x - 1, 0), x1 = std::min(c.x + 1, P.gridDim[0] - 1);
    f3 acc = {0, 0, 0};
    for (int dz = -1; dz <= 1; dz++) {
      const int z = c.z + dz;
      if (z < 0 || z >= P.gridDim[2]) continue;
      for (int dy = -1; dy <= 1; dy++) {
        const int y = c.y + dy;
        if (y < 0 || y >= P.gridDim[1]) continue;
        const uint32_t rowBase = (uint32_t)((z * P.gridDim[1] + y) * P.gridDim[0]);
        const uint32_t b = cs[rowBase + x0], e = cs[rowBase + x1 + 1];
        for (uint32_t j = b; j < e; j++) {
          if (j == (uint32_t)i) continue;
          const f3 rij = sub3(pi, xyz(pred[j]));
          const float r2 = dot3(rij, rij);
          if (r2 >= P.h2) continue;
          const float f = P.mass * poly6(P, r2) / std::max(density[j], 0.5f * P.rho0);
          acc = fma3(f, sub3(xyz(vel[j]), vi), acc);
        }
      }
    }
    corr[i] = {P.xsphC * acc.x, P.xsphC * acc.y, P.xsphC * acc.z, 0.0f};
  }
}

// normals (src/wgsl.js:250-288).
void k_normals(const Params& P, const std::vector<f4>& pred, const std::vector<float>& density,
               std::vector<f4>& normal, const std::vector<uint32_t>& cs) {
  const int n = (int)P.n;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; i++) {
    const f3 pi = xyz(pred[i]);
    const I3 c = cellOf(P, pi);
    const int x0 = std::max(c.x - 1, 0), x1 = std::min(c.x + 1, P.gridDim[0] - 1);
    f3 acc = {0, 0, 0};
    for (int dz = -1; dz <= 1; dz++) {
      const int z = c.z + dz;
      if (z < 0 || z >= P.gridDim[2]) continue;
      for (int dy = -1; dy <= 1; dy++) {
        const int y = c.y + dy;
        if (y < 0 || y >= P.gridDim[1]) continue;
        const uint32_t rowBase = (uint32_t)((z * P.gridDim[1] + y) * P.gridDim[0]);
        const uint32_t b = cs[rowBase + x0], e = cs[rowBase + x1 + 1];
        for (uint32_t j = b; j < e; j++) {
          if (j == (uint32_t)i) continue;
          const f3 rij = sub3(pi, xyz(pred[j]));
          const float r2 = dot3(rij, rij);
          if (r2 >= P.h2 || r2 < 1.0e-12f) continue;
          const float r = std::sqrt(r2);
          const float hr = P.h - r;
          const float coef = (P.mass / std::max(density[j], 0.5f * P.rho0)) * (P.spikyGrad * hr * hr / r);
          acc = fma3(coef, rij, acc);
        }
      }
    }
    normal[i] = {P.h * acc.x, P.h * acc.y, P.h * acc.z, 0.0f};
  }
}

// tension (src/wgsl.js:290-335).
void k_tension(const Params& P, const std::vector<f4>& pred, const std::vector<float>& density,
               const std::vector<f4>& normal, std::vector<f4>& corr, const std::vector<uint32_t>& cs) {
  const int n = (int)P.n;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; i++) {
    const f3 pi = xyz(pred[i]), ni = xyz(normal[i]);
    const float rhoi = density[i];
    const I3 c = cellOf(P, pi);
    const int x0 = std::max(c.x - 1, 0), x1 = std::min(c.x + 1, P.gridDim[0] - 1);
    f3 acc = {0, 0, 0};
    for (int dz = -1; dz <= 1; dz++) {
      const int z = c.z + dz;
      if (z < 0 || z >= P.gridDim[2]) continue;
      for (int dy = -1; dy <= 1; dy++) {
        const int y = c.y + dy;
        if (y < 0 || y >= P.gridDim[1]) continue;
        const uint32_t rowBase = (uint32_t)((z * P.gridDim[1] + y) * P.gridDim[0]);
        const uint32_t b = cs[rowBase + x0], e = cs[rowBase + x1 + 1];
        for (uint32_t j = b; j < e; j++) {
          if (j == (uint32_t)i) continue;
          const f3 rij = sub3(pi, xyz(pred[j]));
          const float r2 = dot3(rij, rij);
          if (r2 >= P.h2 || r2 < 1.0e-12f) continue;
          const float r = std::sqrt(r2);
          const float hrr = P.h - r;
          const float k = hrr * hrr * hrr * r * r * r;
          float cw = P.cohes * (2.0f * k - P.cohesTerm);
          if (2.0f * r > P.h) cw = P.cohes * k;
          const float sCoh = -P.tension * P.mass * cw / r;
          const f3 fCoh = mul3(rij, sCoh);
          const f3 fCurv = mul3(sub3(ni, xyz(normal[j])), -P.tension);
          const float w = 2.0f * P.rho0 / (rhoi + density[j]);
          acc = fma3(w, add3(fCoh, fCurv), acc);
        }
      }
    }
    corr[i] = {std::fmaf(P.dt, acc.x, corr[i].x), std::fmaf(P.dt, acc.y, corr[i].y),
               std::fmaf(P.dt, acc.z, corr[i].z), 0.0f};
  }
}

// finalize (src/wgsl.js:337-350).
void k_finalize(const Params& P, std::vector<f4>& pos, std::vector<f4>& vel, const std::vector<f4>& pred,
                const std::vector<f4>& corr) {
  const int n = (int)P.n;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    vel[i] = {vel[i].x + corr[i].x, vel[i].y + corr[i].y, vel[i].z + corr[i].z, 0.0f};
    pos[i] = pred[i];
  }
}

// ---- rigid bodies (src/wgsl.js:159-185, 614-783) ----
void k_bodyClear(orc_sim* s) {
  std::fill(s->bodyAccum.begin(), s->bodyAccum.end(), 0);
  std::fill(s->bodyCov.begin(), s->bodyCov.end(), 0);
  s->bodyIdxCount = 0;
}
void k_bodyCompact(orc_sim* s, const std::vector<u4>& body) {
  for (int i = 0; i < (int)s->P.n; i++)
    if (body[i].x != 0u) s->bodyIdx[s->bodyIdxCount++] = (uint32_t)i;
}
inline void iadd(int32_t& a, int32_t v) { a = (int32_t)((uint32_t)a + (uint32_t)v); }
void k_bodyCentre(orc_sim* s, const std::vector<f4>& pred, const std::vector<u4>& body) {
  const Params& P = s->P;
  for (uint32_t t = 0; t < P.nBodyParts; t++) {
    const uint32_t i = s->bodyIdx[t];
    const uint32_t b = body[i].x;
    if (b == 0u) continue;
    const uint32_t base = (b - 1u) * 4u;
    const f4& c = s->bodyCentre[b - 1u];
    const f3 d = mul3(sub3(xyz(pred[i]), xyz(c)), P.bodyScale);
    iadd(s->bodyAccum[base + 0], round_i32(d.x));
    iadd(s->bodyAccum[base + 1], round_i32(d.y));
    iadd(s->bodyAccum[base + 2], round_i32(d.z));
    iadd(s->bodyAccum[base + 3], 1);
  }
}
// bodySeed with the binding swap of src/sim.js:346: writes bodyRef from bodyCentre.
void k_bodySeed(orc_sim* s) {
  const Params& P = s->P;
  for (uint32_t b = 0; b < P.nBodies; b++) {
    const uint32_t a = b * 4u;
    const float count = (float)s->bodyAccum[a + 3];
    if (count <= 0.0f) continue;
    const f3 r = xyz(s->bodyCentre[b]);
    const float den = P.bodyScale * count;
    const f3 d = {(float)s->bodyAccum[a] / den, (float)s->bodyAccum[a + 1] / den, (float)s->bodyAccum[a + 2] / den};
    s->bodyRef[b] = {r.x + d.x, r.y + d.y, r.z + d.z, 0.0f};
  }
}
void k_bodyRefLoad(orc_sim* s) {
  for (size_t b = 0; b < s->bodyRef.size(); b++) s->bodyCentre[b] = s->bodyRef[b];
}
void k_bodyCov(orc_sim* s, const std::vector<f4>& pred, const std::vector<u4>& body, const std::vector<f4>& rest) {
  const Params& P = s->P;
  for (uint32_t t = 0; t < P.nBodyParts; t++) {
    const uint32_t i = s->bodyIdx[t];
    const uint32_t b = body[i].x;
    if (b == 0u) continue;
    const f3 p = sub3(xyz(pred[i]), xyz(s->bodyRef[b - 1u]));
    const f3 q = xyz(rest[i]);
    int32_t* cv = &s->bodyCov[(b - 1u) * 9u];
    iadd(cv[0], round_i32(p.x * q.x * P.covScale));
    iadd(cv[1], round_i32(p.y * q.x * P.covScale));
    iadd(cv[2], round_i32(p.z * q.x * P.covScale));
    iadd(cv[3], round_i32(p.x * q.y * P.covScale));
    iadd(cv[4], round_i32(p.y * q.y * P.covScale));
    iadd(cv[5], round_i32(p.z * q.y * P.covScale));
    iadd(cv[6], round_i32(p.x * q.z * P.covScale));
    iadd(cv[7], round_i32(p.y * q.z * P.covScale));
    iadd(cv[8], round_i32(p.z * q.z * P.covScale));
  }
}
// mat3x3fInverse (src/wgsl.js:749-760), returned transposed: columns r0/d, r1/d, r2/d.
inline m3 inverseTransposed(const m3& m) {
  const f3 a = m.c[0], b = m.c[1], c = m.c[2];
  const f3 r0 = cross3(b, c), r1 = cross3(c, a), r2 = cross3(a, b);
  const float d = dot3(a, r0);
  const float invd = std::fabs(d) > 1.0e-20f ? 1.0f / d : 0.0f;
  return {{mul3(r0, invd), mul3(r1, invd), mul3(r2, invd)}};
}
void k_bodyResolve(orc_sim* s) {
  const Params& P = s->P;
  for (uint32_t b = 0; b < P.nBodies; b++) {
    const uint32_t a = b * 4u;
    const float count = (float)s->bodyAccum[a + 3];
    if (count <= 0.0f) continue;
    const f3 prev = xyz(s->bodyCentre[b]);
    const float den = P.bodyScale * count;
    f3 delta = {(float)s->bodyAccum[a] / den, (float)s->bodyAccum[a + 1] / den, (float)s->bodyAccum[a + 2] / den};
    const float invRatio = s->bodyInfo[b].x;
    if (invRatio > 0.0f) delta = mul3(delta, invRatio);
    s->bodyCentre[b] = {prev.x + delta.x, prev.y + delta.y, prev.z + delta.z, 0.0f};
    const int32_t* cv = &s->bodyCov[b * 9u];
    m3 A = {{{(float)cv[0], (float)cv[1], (float)cv[2]},
             {(float)cv[3], (float)cv[4], (float)cv[5]},
             {(float)cv[6], (float)cv[7], (float)cv[8]}}};
    A = scale3(A, 1.0f / P.covScale);
    float det = det3(A);
    if (std::fabs(det) < 1.0e-12f) { A = ident3(); det = 1.0f; }
    const float sc = cbrt_newton(std::fabs(det));
    if (sc > 1.0e-6f) A = scale3(A, 1.0f / sc);
    m3 R = A;
    for (int it = 0; it < 8; it++) {
      const m3 inv = inverseTransposed(R);
      m3 next;
      for (int c = 0; c < 3; c++) next.c[c] = mul3(add3(R.c[c], inv.c[c]), 0.5f);
      const f3 d0 = sub3(next.c[0], R.c[0]), d1 = sub3(next.c[1], R.c[1]), d2 = sub3(next.c[2], R.c[2]);
      R = next;
      if (dot3(d0, d0) + dot3(d1, d1) + dot3(d2, d2) < 1.0e-12f) break;
    }
    for (int r = 0; r < 3; r++) {
      const f3 row = row3(R, r);
      s->bodyRot[b * 3u + r] = {row.x, row.y, row.z, 0.0f};
    }
  }
}
void k_bodyProject(orc_sim* s, std::vector<f4>& pred, const std::vector<u4>& body, const std::vector<f4>& rest) {
  const Params& P = s->P;
  for (uint32_t t = 0; t < P.nBodyParts; t++) {
    const uint32_t i = s->bodyIdx[t];
    const uint32_t b = body[i].x;
    if (b == 0u) continue;
    const uint32_t r = (b - 1u) * 3u;
    const f3 q = xyz(rest[i]);
    const f3 p = {dot3(xyz(s->bodyRot[r]), q), dot3(xyz(s->bodyRot[r + 1]), q), dot3(xyz(s->bodyRot[r + 2]), q)};
    const f3 c = xyz(s->bodyCentre[b - 1u]);
    pred[i] = {c.x + p.x, c.y + p.y, c.z + p.z, 1.0f};
  }
}

// bodyDrag (src/wgsl.js:187-214) over the compacted body list.
void k_bodyDrag(orc_sim* s, std::vector<f4>& vel, const std::vector<u4>& body, float blend) {
  const float goal[3] = {(float)s->heldTarget[0], (float)s->heldTarget[1], (float)s->heldTarget[2]};
  const float rate = (float)s->heldRate, limit = (float)s->heldLimit;
  const uint32_t held = (uint32_t)s->heldBody;
  for (uint32_t t = 0; t < (uint32_t)s->nBodyParts; t++) {
    const uint32_t i = s->bodyIdx[t];
    if (body[i].x != held) continue;
    const f4& c = s->bodyCentre[held - 1u];
    f3 vWant = {(goal[0] - c.x) * rate, (goal[1] - c.y) * rate, (goal[2] - c.z) * rate};
    const float sp = length3(vWant);
    if (sp > limit) vWant = mul3(vWant, limit / sp);
    const f3 v = xyz(vel[i]);
    const f3 dv = mul3(sub3(vWant, v), blend);
    vel[i] = {v.x + dv.x, v.y + dv.y, v.z + dv.z, vel[i].w};
  }
}

// stats (src/wgsl.js:785-832): 256-wide workgroup trees, then u32 atomics.
void k_stats(orc_sim* s, const std::vector<float>& density, const std::vector<f4>& vel) {
  const Params& P = s->P;
  const int n = (int)P.n;
  const int groups = std::max(1, (n + 255) / 256);
  std::vector<uint32_t> partial((size_t)groups * 4);
#pragma omp parallel for schedule(static)
  for (int g = 0; g < groups; g++) {
    float sRho[256], sMaxRho[256], sMaxV[256], sKe[256];
    for (int t = 0; t < 256; t++) {
      const int i = g * 256 + t;
      float rho = 0.0f, mrho = 0.0f, mv = 0.0f, ke = 0.0f;
      if (i < n) {
        rho = density[i] * P.invRho0;
        mrho = rho;
        const f3 v = xyz(vel[i]);
        const float v2 = dot3(v, v);
        mv = std::sqrt(v2);
        ke = 0.5f * P.mass * v2;
      }
      sRho[t] = rho; sMaxRho[t] = mrho; sMaxV[t] = mv; sKe[t] = ke;
    }
    for (int off = 128; off > 0; off >>= 1)
      for (int t = 0; t < off; t++) {
        sRho[t] = sRho[t] + sRho[t + off];
        sMaxRho[t] = std::max(sMaxRho[t], sMaxRho[t + off]);
        sMaxV[t] = std::max(sMaxV[t], sMaxV[t + off]);
        sKe[t] = sKe[t] + sKe[t + off];
      }
    partial[g * 4 + 0] = f2u_sat(sRho[0] * 1024.0f);
    partial[g * 4 + 1] = f2u_sat(sMaxRho[0] * 1024.0f);
    partial[g * 4 + 2] = f2u_sat(sMaxV[0] * 1024.0f);
    partial[g * 4 + 3] = f2u_sat(sKe[0] * 1024.0f);
  }
  for (int g = 0; g < groups; g++) {
    s->statsOut[0] += partial[g * 4 + 0];
    s->statsOut[1] = std::max(s->statsOut[1], partial[g * 4 + 1]);
    s->statsOut[2] = std::max(s->statsOut[2], partial[g * 4 + 2]);
    s->statsOut[3] += partial[g * 4 + 3];
  }
}

// ------------------------------------------------------------ Sim host code
// sortBoundary (src/sim.js:255-286).
void sortBoundary(orc_sim* s, const std::vector<double>& pts, const std::vector<float>& psi, int nb) {
  const int* dim = s->gridDim;
  const double h = s->h;
  std::vector<uint32_t> counts(s->nCells + 2, 0u), cell(nb);
  std::vector<float> bp((size_t)std::max(1, nb) * 4, 0.0f);
  for (int i = 0; i < nb; i++)
    for (int k = 0; k < 3; k++) bp[i * 4 + k] = (float)pts[i * 3 + k];
  for (int i = 0; i < nb; i++) {
    int c[3];
    for (int k = 0; k < 3; k++)
      c[k] = (int)std::min<double>(dim[k] - 1, std::max(0.0, std::floor((double)bp[i * 4 + k] / h)));
    cell[i] = (uint32_t)((c[2] * dim[1] + c[1]) * dim[0] + c[0]);
    counts[cell[i]]++;
  }
  s->bcellStart.assign(s->nCells + 2, 0u);
  uint32_t run = 0;
  for (int c = 0; c <= s->nCells; c++) { s->bcellStart[c] = run; run += counts[c]; }
  s->bcellStart[s->nCells + 1] = run;
  std::vector<uint32_t> cursor = s->bcellStart;
  s->bpos.assign(std::max(1, nb), f4{0, 0, 0, 0});
  s->bpsi.assign(std::max(1, nb), 0.0f);
  for (int i = 0; i < nb; i++) {
    const uint32_t o = cursor[cell[i]]++;
    s->bpos[o] = {bp[i * 4], bp[i * 4 + 1], bp[i * 4 + 2], 0.0f};
    s->bpsi[o] = psi[i];
  }
}

void allocCells(orc_sim* s) {
  s->cellCount.assign(s->nCells + 1, 0u);
  s->cellStart.assign(s->nCells + 2, 0u);
  s->cursor.assign(s->nCells + 1, 0u);
}

void setBoundary(orc_sim* s) {
  std::vector<double> pts;
  std::vector<float> psi;
  boundaryParticles(s->params.box, s->params.rest_density, s->params.spacing, s->h, pts, psi);
  s->nBoundary = (int)(pts.size() / 3);
  sortBoundary(s, pts, psi, s->nBoundary);
}

// The grid pass with the predict before it (src/sim.js:473-492), at parity `par`.
void gridPass(orc_sim* s, int par) {
  const int o = par ^ 1;
  const Params& P = s->P;
  k_predict(P, s->pos[par], s->vel[par], s->pred[par]);
  k_sort_slots(P, s->pred[par], s->cellCount, s->cellStart, s->cursor, s->slot);
  const int n = (int)P.n;
  k_scatter(n, s->slot, s->pos[par], s->pos[o]);
  k_scatter(n, s->slot, s->vel[par], s->vel[o]);
  k_scatter(n, s->slot, s->pred[par], s->pred[o]);
  k_scatter(n, s->slot, s->body[par], s->body[o]);
  k_scatter(n, s->slot, s->rest[par], s->rest[o]);
}

// primeGrid (src/sim.js:223-253).
void primeGrid(orc_sim* s) {
  uploadParams(s, 0);
  gridPass(s, s->parity);
  s->parity ^= 1;
  s->predParity = s->parity;
  uploadParams(s, 1.0 / 240);
  // The compacted body list the drag pass reads before the first 'bodies' pass.
  if (s->nBodyParts > 0) { k_bodyClear(s); k_bodyCompact(s, s->body[s->parity]); }
}

int resetCommon(orc_sim* s) {
  Scene& sc = s->sc;
  const p4a_params& p = s->params;
  s->simTime = 0;
  s->gen++;
  const int n = sc.n;
  s->h = sc.h;
  for (int k = 0; k < 3; k++) s->gridDim[k] = (int)std::max(1.0, std::floor(p.box[k] / s->h));
  s->nCells = s->gridDim[0] * s->gridDim[1] * s->gridDim[2];
  const int cap = n + s->pourBudget;
  s->cap = cap;
  for (int t = 0; t < 2; t++) {
    s->pos[t].assign(cap, f4{0, 0, 0, 0}); s->vel[t].assign(cap, f4{0, 0, 0, 0});
    s->pred[t].assign(cap, f4{0, 0, 0, 0}); s->rest[t].assign(cap, f4{0, 0, 0, 0});
    s->body[t].assign(cap, u4{0, 0, 0, 0});
  }
  s->lambda.assign(cap, 0.0f); s->density.assign(cap, 0.0f); s->slot.assign(cap, 0u);
  s->corr.assign(cap, f4{0, 0, 0, 0}); s->normal.assign(cap, f4{0, 0, 0, 0});
  allocCells(s);
  setBoundary(s);
  const int nBodies = (int)sc.bodyDensity.size();
  s->nBodies = nBodies;
  s->nBodyParts = sc.nBody;
  const int nb1 = std::max(1, nBodies);
  s->bodyAccum.assign(nb1 * 4, 0); s->bodyCov.assign(nb1 * 9, 0);
  s->bodyCentre.assign(nb1, f4{0, 0, 0, 0}); s->bodyRef.assign(nb1, f4{0, 0, 0, 0});
  s->bodyRot.assign(nb1 * 3, f4{0, 0, 0, 0}); s->bodyInfo.assign(nb1, f4{0, 0, 0, 0});
  s->bodyIdx.assign(std::max(1, sc.nBody), 0u);
  s->bodyIdxCount = 0;
  for (int i = 0; i < nBodies; i++) {
    s->bodyInfo[i].x = (float)(1 / std::max(1e-6, sc.bodyDensity[i]));
    s->bodyCentre[i] = {(float)sc.bodyCentre[i * 3], (float)sc.bodyCentre[i * 3 + 1], (float)sc.bodyCentre[i * 3 + 2], 0.0f};
    s->bodyRef[i] = s->bodyCentre[i];
    for (int r = 0; r < 3; r++) (&s->bodyRot[i * 3 + r].x)[r] = 1.0f;
  }
  // Fixed-point scales (src/sim.js:163-171).
  double maxCount = 1, maxRest = 1e-3;
  std::vector<int> counts(nBodies, 0);
  for (int i = 0; i < n; i++)
    if (sc.phase[i * 4] >= 1 && (int)sc.phase[i * 4] <= nBodies) counts[sc.phase[i * 4] - 1]++;
  for (int b = 0; b < nBodies; b++) maxCount = std::max(maxCount, (double)counts[b]);
  for (int i = 0; i < n; i++) {
    double r = std::hypot((double)sc.rest[i * 4], (double)sc.rest[i * 4 + 1], (double)sc.rest[i * 4 + 2]);
    if (r > maxRest) maxRest = r;
  }
  const double extent = std::max(p.box[0], std::max(p.box[1], p.box[2]));
  s->bodyScale = 1e9 / (extent * maxCount);
  s->covScale = 1e9 / (extent * maxRest * maxCount);
  std::fill(s->statsOut.begin(), s->statsOut.end(), 0u);
  s->stats = p4a_stats{};
  s->stats.avg_rho = 1; s->stats.max_rho = 1;
  for (int i = 0; i < n; i++) {
    s->pos[0][i] = {sc.pos[i * 4], sc.pos[i * 4 + 1], sc.pos[i * 4 + 2], sc.pos[i * 4 + 3]};
    s->vel[0][i] = {sc.vel[i * 4], sc.vel[i * 4 + 1], sc.vel[i * 4 + 2], sc.vel[i * 4 + 3]};
    s->pred[0][i] = s->pos[0][i];
    s->body[0][i] = {sc.phase[i * 4], sc.phase[i * 4 + 1], sc.phase[i * 4 + 2], sc.phase[i * 4 + 3]};
    s->rest[0][i] = {sc.rest[i * 4], sc.rest[i * 4 + 1], sc.rest[i * 4 + 2], sc.rest[i * 4 + 3]};
  }
  s->n = n;
  s->parity = 0;
  s->predParity = 0;
  s->heldBody = -1;
  s->heldTarget[0] = s->heldTarget[1] = s->heldTarget[2] = 0;
  s->heldRate = 10; s->heldLimit = 4;
  uploadParams(s, 1.0 / 240);
  primeGrid(s);
  s->ready = true;
  return P4A_OK;
}

void copyParams(orc_sim* s, const p4a_params* p) {
  s->params = *p;
  s->specs.assign(p->bodies, p->bodies + (p->bodies ? p->n_bodies : 0));
  s->params.bodies = s->specs.empty() ? nullptr : s->specs.data();
  s->params.n_bodies = (int32_t)s->specs.size();
}

}  // namespace

extern "C" {

orc_sim* orc_create(void) { return new orc_sim(); }
void orc_destroy(orc_sim* s) { delete s; }
void orc_set_threads(int threads) { g_threads = threads; }
int orc_get_threads(void) {
#ifdef _OPENMP
  apply_threads();
  return omp_get_max_threads();
#else
  return 1;
#endif
}
float orc_cbrt_newton(float x) { return cbrt_newton(x); }

int orc_build_scene(const p4a_params* p, p4a_scene_counts* counts, float* pos, float* vel,
                    float* rest, uint32_t* phase, double* body_centre, double* body_density) {
  if (!p || !counts) return P4A_ERR_ARG;
  Scene sc;
  buildScene(*p, sc);
  std::vector<double> pts;
  std::vector<float> psi;
  boundaryParticles(p->box, p->rest_density, p->spacing, sc.h, pts, psi);
  counts->n = sc.n; counts->n_fluid = sc.nFluid; counts->n_body = sc.nBody;
  counts->n_bodies = (int32_t)sc.bodyDensity.size(); counts->n_boundary = (int32_t)(pts.size() / 3);
  counts->mass = sc.mass; counts->denom_rest = sc.denomRest; counts->h = sc.h;
  if (pos) std::memcpy(pos, sc.pos.data(), sc.pos.size() * 4);
  if (vel) std::memcpy(vel, sc.vel.data(), sc.vel.size() * 4);
  if (rest) std::memcpy(rest, sc.rest.data(), sc.rest.size() * 4);
  if (phase) std::memcpy(phase, sc.phase.data(), sc.phase.size() * 4);
  if (body_centre) std::memcpy(body_centre, sc.bodyCentre.data(), sc.bodyCentre.size() * 8);
  if (body_density) std::memcpy(body_density, sc.bodyDensity.data(), sc.bodyDensity.size() * 8);
  return P4A_OK;
}

int orc_boundary(const p4a_params* p, double d, double h, int32_t* count, double* pts, float* psi) {
  std::vector<double> vp;
  std::vector<float> vs;
  boundaryParticles(p->box, p->rest_density, d, h, vp, vs);
  *count = (int32_t)(vp.size() / 3);
  if (pts) std::memcpy(pts, vp.data(), vp.size() * 8);
  if (psi) std::memcpy(psi, vs.data(), (size_t)*count * 4);
  return P4A_OK;
}

int orc_reset(orc_sim* s, const p4a_params* p) {
  if (!s || !p || p->spacing <= 0) return P4A_ERR_ARG;
  copyParams(s, p);
  buildScene(s->params, s->sc);
  s->pourBudget = p->pour ? s->sc.nFluid : 0;
  return resetCommon(s);
}

int orc_reset_scene(orc_sim* s, const p4a_params* p, const p4a_scene_desc* d) {
  if (!s || !p || !d || d->n < 0 || !d->pos || p->spacing <= 0) return P4A_ERR_ARG;
  copyParams(s, p);
  Scene& sc = s->sc;
  sc = Scene();
  sc.n = d->n; sc.d = p->spacing; sc.h = 2 * p->spacing;
  sc.pos.assign(d->pos, d->pos + (size_t)d->n * 4);
  sc.vel = d->vel ? std::vector<float>(d->vel, d->vel + (size_t)d->n * 4) : std::vector<float>((size_t)d->n * 4, 0.0f);
  sc.rest = d->rest ? std::vector<float>(d->rest, d->rest + (size_t)d->n * 4) : std::vector<float>((size_t)d->n * 4, 0.0f);
  sc.phase = d->phase ? std::vector<uint32_t>(d->phase, d->phase + (size_t)d->n * 4) : std::vector<uint32_t>((size_t)d->n * 4, 0u);
  int nFluid = 0;
  for (int i = 0; i < d->n; i++) if (sc.phase[i * 4] == 0) nFluid++;
  // The calibration of scene.js runs over the leading fluid block; an explicit
  // scene lists its fluid first too.
  sc.nFluid = nFluid;
  sc.nBody = d->n - nFluid;
  sc.bodyDensity.assign(d->body_density, d->body_density + d->n_bodies);
  sc.bodyCentre.assign(d->body_centre, d->body_centre + 3 * d->n_bodies);
  sc.mass = d->mass;
  sc.denomRest = d->denom_rest;
  const bool doMass = !(d->mass > 0), doDenom = !(d->denom_rest > 0);
  if (doMass || doDenom)
    calibrate(sc.pos, nFluid, sc.d, sc.h, p->rest_density, doMass, doDenom, sc.mass, sc.denomRest, p->box);
  s->pourBudget = std::max(0, d->pour_budget);
  return resetCommon(s);
}

int orc_step(orc_sim* s, double frameDt, int32_t* substeps_out) {
  if (!s || !s->ready) return P4A_ERR_STATE;
  apply_threads();
  const p4a_params& p = s->params;
  const int base = std::max(1, p.substeps);
  const double dtTarget = (1.0 / 60) / base;
  s->timeBank = s->timeBank + frameDt;
  double subD = std::floor(s->timeBank / dtTarget + 1e-4);
  const double workCap = base * 8;
  if (subD > workCap) { subD = workCap; s->timeBank = 0; }
  else s->timeBank -= subD * dtTarget;
  const int sub = (int)subD;
  s->lastSubsteps = sub;
  s->lastAdvanced = subD * dtTarget;
  if (substeps_out) *substeps_out = sub;
  if (sub < 1) { s->lastAdvanced = 0; return P4A_OK; }
  const double dt = dtTarget;
  uploadParams(s, dt);
  const bool dragging = s->heldBody >= 1 && s->nBodyParts > 0;
  const float blend = (float)(1 - std::exp(-std::max(dt, 0.0) / 0.02));
  const Params& P = s->P;
  for (int st = 0; st < sub; st++) {
    const int par = s->parity;
    if (dragging) k_bodyDrag(s, s->vel[par], s->body[par], blend);
    gridPass(s, par);
    s->parity ^= 1;
    s->predParity = s->parity;
    const int par2 = s->parity;
    int pp = s->predParity;
    if (s->nBodyParts > 0) {
      k_bodyClear(s);
      k_bodyCompact(s, s->body[par2]);
      k_bodyCentre(s, s->pred[pp], s->body[par2]);
      k_bodySeed(s);
      k_bodyRefLoad(s);
    }
    for (int it = 0; it < std::max(1, p.iterations); it++) {
      k_lambda(P, s->pred[pp], s->lambda, s->density, s->cellStart, s->bpos, s->bpsi, s->bcellStart);
      k_delta(P, s->pred[pp], s->pred[pp ^ 1], s->lambda, s->cellStart, s->bpos, s->bpsi, s->bcellStart);
      pp ^= 1;
      if (s->nBodyParts > 0) {
        k_bodyClear(s);
        k_bodyCentre(s, s->pred[pp], s->body[par2]);
        k_bodySeed(s);
        k_bodyCov(s, s->pred[pp], s->body[par2], s->rest[par2]);
        k_bodyResolve(s);
        k_bodyProject(s, s->pred[pp], s->body[par2], s->rest[par2]);
      }
    }
    s->predParity = pp;
    if (s->predParity != s->parity) {
      std::copy(s->pred[s->predParity].begin(), s->pred[s->predParity].begin() + s->n,
                s->pred[s->predParity ^ 1].begin());
      s->predParity = s->parity;
    }
    k_velFromPos(P, s->pos[par2], s->vel[par2], s->pred[par2]);
    k_xsph(P, s->pred[par2], s->vel[par2], s->density, s->corr, s->cellStart);
    if (p.surface_tension_k > 0) {
      k_normals(P, s->pred[par2], s->density, s->normal, s->cellStart);
      k_tension(P, s->pred[par2], s->density, s->normal, s->corr, s->cellStart);
    }
    k_finalize(P, s->pos[par2], s->vel[par2], s->pred[par2], s->corr);
    s->simTime += dt;
  }
  std::fill(s->statsOut.begin(), s->statsOut.end(), 0u);
  k_stats(s, s->density, s->vel[s->parity]);
  const double SCALE = 1024;
  s->stats.avg_rho = s->statsOut[0] / SCALE / std::max(1, s->n);
  s->stats.max_rho = s->statsOut[1] / SCALE;
  s->stats.max_speed = s->statsOut[2] / SCALE;
  s->stats.ke = s->statsOut[3] / SCALE;
  for (int k = 0; k < 4; k++) s->stats.raw[k] = s->statsOut[k];
  s->stats.valid = 1;
  return P4A_OK;
}

int orc_append_fluid(orc_sim* s, const float* pos3, const float* vel3, int32_t count, int32_t* added) {
  if (!s || !s->ready || count < 0) return P4A_ERR_ARG;
  const int room = std::max(0, s->cap - s->n);
  const int c = std::min(count, room);
  if (added) *added = std::max(0, c);
  if (c <= 0) return P4A_OK;
  const int n = s->n, par = s->parity, pp = s->predParity;
  for (int i = 0; i < c; i++) {
    f4 p4 = {pos3[i * 3], pos3[i * 3 + 1], pos3[i * 3 + 2], 1.0f};
    f4 v4 = {vel3[i * 3], vel3[i * 3 + 1], vel3[i * 3 + 2], 0.0f};
    s->pos[par][n + i] = p4;
    s->vel[par][n + i] = v4;
    s->pred[pp][n + i] = p4;
    s->density[n + i] = (float)s->params.rest_density;
    s->lambda[n + i] = 0.0f;
    s->corr[n + i] = f4{0, 0, 0, 0};
    s->normal[n + i] = f4{0, 0, 0, 0};
    for (int t = 0; t < 2; t++) { s->body[t][n + i] = u4{0, 0, 0, 0}; s->rest[t][n + i] = f4{0, 0, 0, 0}; }
  }
  s->n += c;
  return P4A_OK;
}

int orc_apply_ray_impulse(orc_sim* s, const double origin[3], const double dir[3], const double impulse[3],
                          double radius, double speedLimit) {
  if (!s || !s->ready) return P4A_ERR_STATE;
  if (!s->n || radius <= 0) return P4A_OK;
  const double len = std::hypot(impulse[0], impulse[1], impulse[2]);
  if (len <= 0) return P4A_OK;
  double dl = std::hypot(dir[0], dir[1], dir[2]);
  if (!(dl != 0)) dl = 1;
  const f3 o = {(float)origin[0], (float)origin[1], (float)origin[2]};
  const f3 dr = {(float)(dir[0] / dl), (float)(dir[1] / dl), (float)(dir[2] / dl)};
  const f3 im = {(float)impulse[0], (float)impulse[1], (float)impulse[2]};
  const float R = (float)radius, sl = (float)speedLimit;
  std::vector<f4>& pos = s->pos[s->parity];
  std::vector<f4>& vel = s->vel[s->parity];
  // impulse (src/wgsl.js:216-248).
  for (int i = 0; i < s->n; i++) {
    const f3 toP = sub3(xyz(pos[i]), o);
    const float along = dot3(toP, dr);
    if (along <= 0.0f) continue;
    const f3 radial = sub3(toP, mul3(dr, along));
    const float d2 = dot3(radial, radial);
    if (d2 >= R * R) continue;
    const float x = 1.0f - std::sqrt(d2) / R;
    const f3 v = xyz(vel[i]);
    const float oldSpeed = length3(v);
    f3 nv = add3(v, mul3(im, x * x));
    const float ns = length3(nv);
    const float allowed = std::max(oldSpeed, sl);
    if (ns > allowed) nv = mul3(nv, allowed / ns);
    vel[i] = {nv.x, nv.y, nv.z, 0.0f};
  }
  return P4A_OK;
}

int orc_hold_body(orc_sim* s, int32_t body1, const double target[3], double rate, double limit) {
  if (!s) return P4A_ERR_ARG;
  s->heldBody = (body1 >= 1 && body1 <= s->nBodies) ? body1 : -1;
  for (int k = 0; k < 3; k++) s->heldTarget[k] = target[k];
  s->heldRate = rate;
  s->heldLimit = limit;
  return P4A_OK;
}
int orc_release_body(orc_sim* s) {
  if (!s) return P4A_ERR_ARG;
  s->heldBody = -1;
  return P4A_OK;
}

int orc_resize_box(orc_sim* s, const double newBox[3]) {
  if (!s || !s->ready) return P4A_ERR_STATE;
  p4a_params& p = s->params;
  const double oldBox[3] = {p.box[0], p.box[1], p.box[2]};
  bool moved = false;
  for (int a = 0; a < 3; a++) if (std::fabs(newBox[a] - oldBox[a]) > 1e-9) moved = true;
  if (!moved) return P4A_OK;
  for (int a = 0; a < 3; a++) p.box[a] = newBox[a];
  for (int k = 0; k < 3; k++) s->gridDim[k] = (int)std::max(1.0, std::floor(newBox[k] / s->h));
  const int cells = s->gridDim[0] * s->gridDim[1] * s->gridDim[2];
  const bool changed = cells != s->nCells;
  s->nCells = cells;
  if (changed) allocCells(s);
  setBoundary(s);
  s->gen++;
  // resize (src/wgsl.js:125-157) on the live pos.
  const float halfD = (float)(0.5 * p.spacing);
  const float oldSize[3] = {(float)oldBox[0], (float)oldBox[1], (float)oldBox[2]};
  const float newSize[3] = {(float)newBox[0], (float)newBox[1], (float)newBox[2]};
  const float cMin[3] = {halfD, halfD, halfD};
  const float cMax[3] = {(float)(newBox[0] - 0.5 * p.spacing), (float)(newBox[1] - 0.5 * p.spacing),
                         (float)(newBox[2] - 0.5 * p.spacing)};
  std::vector<f4>& pos = s->pos[s->parity];
  for (int i = 0; i < s->n; i++) {
    float* pv = &pos[i].x;
    for (int a = 0; a < 3; a++) {
      if (newSize[a] < oldSize[a]) {
        const float t = std::min(std::max((pv[a] - 0.0f) / oldSize[a], 0.0f), 1.0f);
        pv[a] = 0.0f + t * newSize[a];
      }
      pv[a] = std::min(std::max(pv[a], cMin[a]), cMax[a]);
    }
  }
  return P4A_OK;
}

// Anisotropic kernel (src/aniso_wgsl.js:3-158) with the uniform of src/mesh.js:221-242.
int orc_aniso(orc_sim* s, const p4a_aniso_params* ap) {
  if (!s || !s->ready || !ap) return P4A_ERR_ARG;
  const int n = s->n;
  if (n <= 0) return P4A_OK;
  if (s->smoothPos.size() < (size_t)n) { s->smoothPos.assign(n, f4{0, 0, 0, 0}); s->anisoG.assign(2 * (size_t)n, f4{0, 0, 0, 0}); s->anisoGen++; }
  const double support = s->h;
  const double radiusD = ap->radius_scale * support;
  const int cells = (int)std::ceil(ap->radius_scale);
  const double sigmaBulk = 0.15 * radiusD * radiusD;
  const float lambdaA = (float)ap->lambda, invSupport = (float)(1 / support), sup = (float)support;
  const float radius = (float)radiusD, kr = (float)ap->ratio, kn = (float)ap->lonely;
  const float ks = (float)(ap->ks / sigmaBulk), stretch = (float)ap->stretch, minExtent = (float)ap->min_extent;
  const int neps = ap->min_neighbours;
  const int* G = s->gridDim;
  const std::vector<f4>& pos = s->pos[s->parity];
  const std::vector<uint32_t>& cs = s->cellStart;
  apply_threads();
#pragma omp parallel for schedule(dynamic, 128)
  for (int i = 0; i < n; i++) {
    const f3 xi = xyz(pos[i]);
    I3 c;
    c.x = std::min(std::max(f2i_sat(std::floor((xi.x - 0.0f) * invSupport)), 0), G[0] - 1);
    c.y = std::min(std::max(f2i_sat(std::floor((xi.y - 0.0f) * invSupport)), 0), G[1] - 1);
    c.z = std::min(std::max(f2i_sat(std::floor((xi.z - 0.0f) * invSupport)), 0), G[2] - 1);
    const int x0 = std::max(c.x - cells, 0), x1 = std::min(c.x + cells, G[0] - 1);
    const float r2max = radius * radius;
    const float invR = 1.0f / radius;
    const f3 rel = {xi.x - 0.0f, xi.y - 0.0f, xi.z - 0.0f};
    f3 sd = {0, 0, 0};
    m3 m2 = {{{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}};
    float wsum = 0.0f;
    int nn = 0;
    for (int dz = -cells; dz <= cells; dz++) {
      const int z = c.z + dz;
      if (z < 0 || z >= G[2]) continue;
      const float dzMin = std::max(std::max((float)z * sup - rel.z, rel.z - (float)(z + 1) * sup), 0.0f);
      const float dz2 = dzMin * dzMin;
      if (dz2 >= r2max) continue;
      for (int dy = -cells; dy <= cells; dy++) {
        const int y = c.y + dy;
        if (y < 0 || y >= G[1]) continue;
        const float dyMin = std::max(std::max((float)y * sup - rel.y, rel.y - (float)(y + 1) * sup), 0.0f);
        if (dz2 + dyMin * dyMin >= r2max) continue;
        const uint32_t rowBase = (uint32_t)((z * G[1] + y) * G[0]);
        const uint32_t jb = cs[rowBase + x0], je = cs[rowBase + x1 + 1];
        for (uint32_t j = jb; j < je; j++) {
          const f3 d = sub3(xyz(pos[j]), xi);
          const float r2 = dot3(d, d);
          if (r2 >= r2max) continue;
          const float t = std::sqrt(r2) * invR;
          const float w = 1.0f - t * t * t;
          sd = fma3(w, d, sd);
          m2.c[0] = fma3(d.x * w, d, m2.c[0]);
          m2.c[1] = fma3(d.y * w, d, m2.c[1]);
          m2.c[2] = fma3(d.z * w, d, m2.c[2]);
          wsum = wsum + w;
          nn = nn + 1;
        }
      }
    }
    auto storeG = [&](const m3& Gm, float last) {
      s->anisoG[i * 2 + 0] = {elc(Gm, 0, 0), elc(Gm, 1, 0), elc(Gm, 2, 0), elc(Gm, 1, 1)};
      s->anisoG[i * 2 + 1] = {elc(Gm, 2, 1), elc(Gm, 2, 2), det3(Gm), last};
    };
    if (wsum <= 0.0f) {
      s->smoothPos[i] = {xi.x, xi.y, xi.z, 0.0f};
      storeG(scale3(ident3(), kn / sup), 0.0f);
      continue;
    }
    const f3 dbar = {sd.x / wsum, sd.y / wsum, sd.z / wsum};
    s->smoothPos[i] = {xi.x + dbar.x * lambdaA, xi.y + dbar.y * lambdaA, xi.z + dbar.z * lambdaA, 0.0f};
    m3 cov;
    const float db[3] = {dbar.x, dbar.y, dbar.z};
    for (int k = 0; k < 3; k++) {
      cov.c[k] = {m2.c[k].x / wsum - dbar.x * db[k], m2.c[k].y / wsum - dbar.y * db[k],
                  m2.c[k].z / wsum - dbar.z * db[k]};
    }
    // jacobi (src/aniso_wgsl.js:30-55)
    m3 a = cov, v = ident3();
    for (int sweep = 0; sweep < 6; sweep++)
      for (int pI = 0; pI < 2; pI++)
        for (int qI = pI + 1; qI < 3; qI++) {
          const float apq = elc(a, qI, pI);
          if (std::fabs(apq) < 1.0e-12f) continue;
          const float theta = (elc(a, qI, qI) - elc(a, pI, pI)) / (2.0f * apq);
          const float sgn = theta > 0.0f ? 1.0f : (theta < 0.0f ? -1.0f : 0.0f);
          float t = sgn / (std::fabs(theta) + std::sqrt(theta * theta + 1.0f));
          if (theta == 0.0f) t = 1.0f;
          const float cth = 1.0f / std::sqrt(t * t + 1.0f);
          const float sn = t * cth;
          m3 r = ident3();
          el(r, pI, pI) = cth; el(r, qI, qI) = cth;
          el(r, qI, pI) = sn; el(r, pI, qI) = -sn;
          a = matmul(matmul(transpose3(r), a), r);
          v = matmul(v, r);
        }
    const m3& R = v;
    const f3 sig = {elc(a, 0, 0), elc(a, 1, 1), elc(a, 2, 2)};
    const float s1 = std::max(sig.x, std::max(sig.y, sig.z));
    const float sl = s1 / kr;
    f3 ext = {ks * std::max(sig.x, sl), ks * std::max(sig.y, sl), ks * std::max(sig.z, sl)};
    const float den = std::max(1.0f, std::max(ext.x, std::max(ext.y, ext.z)) / stretch);
    ext = {ext.x / den, ext.y / den, ext.z / den};
    ext = {std::max(ext.x, minExtent), std::max(ext.y, minExtent), std::max(ext.z, minExtent)};
    const f3 inv = {1.0f / (sup * ext.x), 1.0f / (sup * ext.y), 1.0f / (sup * ext.z)};
    m3 D = {{{inv.x, 0, 0}, {0, inv.y, 0}, {0, 0, inv.z}}};
    const m3 Gan = matmul(matmul(R, D), transpose3(R));
    const m3 Giso = scale3(ident3(), kn / sup);
    const float lo = (float)neps * 0.4f, hi = (float)neps * 1.6f;
    float tt = ((float)nn - lo) / (hi - lo);
    tt = std::min(std::max(tt, 0.0f), 1.0f);
    const float w = tt * tt * (3.0f - 2.0f * tt);
    m3 Gm;
    for (int k = 0; k < 3; k++) {
      Gm.c[k] = {Giso.c[k].x * (1.0f - w) + Gan.c[k].x * w, Giso.c[k].y * (1.0f - w) + Gan.c[k].y * w,
                 Giso.c[k].z * (1.0f - w) + Gan.c[k].z * w};
    }
    storeG(Gm, (float)nn);
  }
  return P4A_OK;
}

int orc_get_info(const orc_sim* s, p4a_info* o) {
  if (!s || !o) return P4A_ERR_ARG;
  *o = p4a_info{};
  o->n = s->n; o->n_fluid = s->sc.nFluid; o->n_body_parts = s->nBodyParts; o->n_bodies = s->nBodies;
  o->n_boundary = s->nBoundary; o->cap = s->cap; o->pour_budget = s->pourBudget;
  for (int k = 0; k < 3; k++) o->grid_dim[k] = s->gridDim[k];
  o->n_cells = s->nCells; o->parity = s->parity; o->pred_parity = s->predParity; o->gen = s->gen;
  o->last_substeps = s->lastSubsteps; o->h = s->h; o->mass = s->sc.mass; o->denom_rest = s->sc.denomRest;
  o->sim_time = s->simTime; o->last_advanced = s->lastAdvanced; o->time_bank = s->timeBank;
  o->body_scale = s->bodyScale; o->cov_scale = s->covScale; o->held_body = s->heldBody;
  o->aniso_gen = s->anisoGen;
  return P4A_OK;
}

// ---- surface mesh: SurfaceMesh.configure + generate (src/mesh.js:99-352) ----------
namespace {

struct MeshU {  // the uniform of src/mesh_wgsl.js:3-21 as src/mesh.js:137-153 packs it
  int dim[3];
  float voxel, origin[3], iso, invSupport, support2, poly6, mass, rho0;
  int simDim[3];
  uint32_t maxTris, skipBodies;
};

inline float mesh_at(const std::vector<float>& f, const MeshU& M, int x, int y, int z) {
  x = std::min(std::max(x, 0), M.dim[0] - 1);
  y = std::min(std::max(y, 0), M.dim[1] - 1);
  z = std::min(std::max(z, 0), M.dim[2] - 1);
  return f[(size_t)((z * M.dim[1] + y) * M.dim[0] + x)];
}

// meshSmooth (src/mesh_wgsl.js:71-92) along `axis`, in place over every grid line.
void mesh_blur(std::vector<float>& f, const MeshU& M, int axis) {
  const int len = M.dim[axis];
  const size_t stride = axis == 0 ? 1 : axis == 1 ? (size_t)M.dim[0] : (size_t)M.dim[0] * M.dim[1];
  const int o1 = axis == 0 ? 1 : 0, o2 = axis == 2 ? 1 : 2;
  std::vector<float> a(len), b(len);
  for (int u = 0; u < M.dim[o2]; u++)
    for (int w = 0; w < M.dim[o1]; w++) {
      const size_t base = (size_t)u * (o2 == 1 ? M.dim[0] : (size_t)M.dim[0] * M.dim[1]) +
                          (size_t)w * (o1 == 0 ? 1 : M.dim[0]);
      for (int k = 0; k < len; k++) a[k] = f[base + k * stride];
      for (int k = 0; k < len; k++)
        b[k] = (0.25f * a[std::max(k - 1, 0)] + 0.5f * a[k]) + 0.25f * a[std::min(k + 1, len - 1)];
      for (int k = 0; k < len; k++) f[base + k * stride] = b[k];
    }
}

struct MCorner {
  float d;
  f3 p, g;
};

uint32_t mesh_pack(const MeshU& M, f3 pg, f3 nIn, uint32_t* hi) {
  const float px = std::min(std::max(pg.x / (float)(M.dim[0] - 1), 0.0f), 1.0f);
  const float py = std::min(std::max(pg.y / (float)(M.dim[1] - 1), 0.0f), 1.0f);
  const float pz = std::min(std::max(pg.z / (float)(M.dim[2] - 1), 0.0f), 1.0f);
  const uint32_t qx = f2u_sat(px * 65535.0f + 0.5f), qy = f2u_sat(py * 65535.0f + 0.5f),
                 qz = f2u_sat(pz * 65535.0f + 0.5f);
  const float l1 = std::max((std::fabs(nIn.x) + std::fabs(nIn.y)) + std::fabs(nIn.z), 1.0e-12f);
  const f3 nv = {nIn.x / l1, nIn.y / l1, nIn.z / l1};
  float ex = nv.x, ey = nv.y;
  if (nv.z < 0.0f) {
    ex = (1.0f - std::fabs(nv.y)) * (nv.x >= 0.0f ? 1.0f : -1.0f);
    ey = (1.0f - std::fabs(nv.x)) * (nv.y >= 0.0f ? 1.0f : -1.0f);
  }
  const uint32_t ox = f2u_sat(std::min(std::max(ex * 0.5f + 0.5f, 0.0f), 1.0f) * 255.0f + 0.5f);
  const uint32_t oy = f2u_sat(std::min(std::max(ey * 0.5f + 0.5f, 0.0f), 1.0f) * 255.0f + 0.5f);
  *hi = qz | ((ox | (oy << 8)) << 16);
  return qx | (qy << 16);
}

void mesh_edge(const MeshU& M, const MCorner& a, const MCorner& b, uint32_t out[2]) {
  const float t = (M.iso - a.d) / (b.d - a.d);
  const float s = 1.0f - t;
  const f3 p = {a.p.x * s + b.p.x * t, a.p.y * s + b.p.y * t, a.p.z * s + b.p.z * t};
  const f3 g = {a.g.x * s + b.g.x * t, a.g.y * s + b.g.y * t, a.g.z * s + b.g.z * t};
  out[0] = mesh_pack(M, p, {-g.x, -g.y, -g.z}, &out[1]);
}

struct MeshSink {
  std::vector<uint32_t>* verts;
  uint64_t count = 0, limit = 0;
  void tri(const uint32_t a[2], const uint32_t b[2], const uint32_t c[2]) {
    if (count < limit) {
      uint32_t* o = verts->data() + count * 6;
      o[0] = a[0]; o[1] = a[1]; o[2] = b[0]; o[3] = b[1]; o[4] = c[0]; o[5] = c[1];
    }
    count++;
  }
};

// emitTet / emitLone / emitQuad (src/mesh_wgsl.js:154-196)
void mesh_tet(const MeshU& M, MeshSink& S, const MCorner& a, const MCorner& b, const MCorner& c,
              const MCorner& d) {
  const bool ia = a.d > M.iso, ib = b.d > M.iso, ic = c.d > M.iso, id = d.d > M.iso;
  const int nin = (int)ia + (int)ib + (int)ic + (int)id;
  if (nin == 0 || nin == 4) return;
  auto lone = [&](const MCorner& l, const MCorner& p1, const MCorner& p2, const MCorner& p3) {
    uint32_t e1[2], e2[2], e3[2];
    mesh_edge(M, l, p1, e1);
    mesh_edge(M, l, p2, e2);
    mesh_edge(M, l, p3, e3);
    S.tri(e1, e2, e3);
  };
  auto quad = [&](const MCorner& qa, const MCorner& qb, const MCorner& qc, const MCorner& qd) {
    uint32_t q0[2], q1[2], q2[2], q3[2];
    mesh_edge(M, qa, qc, q0);
    mesh_edge(M, qa, qd, q1);
    mesh_edge(M, qb, qd, q2);
    mesh_edge(M, qb, qc, q3);
    S.tri(q0, q1, q2);
    S.tri(q0, q2, q3);
  };
  if (nin == 1 || nin == 3) {
    const bool look = nin == 1;
    if (ia == look) lone(a, b, c, d);
    else if (ib == look) lone(b, a, c, d);
    else if (ic == look) lone(c, a, b, d);
    else lone(d, a, b, c);
  } else {
    if (ia && ib) quad(a, b, c, d);
    else if (ia && ic) quad(a, c, b, d);
    else if (ia && id) quad(a, d, b, c);
    else if (ib && ic) quad(b, c, a, d);
    else if (ib && id) quad(b, d, a, c);
    else quad(c, d, a, b);
  }
}

}  // namespace

int orc_mesh(orc_sim* s, const p4a_mesh_params* mp, int64_t* triangles) {
  if (!s || !s->ready || !mp || mp->resolution < 1 || mp->max_triangles < 0) return P4A_ERR_ARG;
  const double* box = s->params.box;
  const double longest = std::max(box[0], std::max(box[1], box[2]));
  const double voxel = longest / mp->resolution;
  MeshU M{};
  for (int k = 0; k < 3; k++) {
    M.dim[k] = (int)std::ceil(box[k] / voxel) + 2 + 1;
    M.origin[k] = (float)(0.0 - voxel);
    M.simDim[k] = s->gridDim[k];
  }
  M.voxel = (float)voxel;
  for (int k = 0; k < 3; k++) s->meshDim[k] = M.dim[k];
  s->meshOrigin = -voxel;
  s->meshVoxel = voxel;
  M.iso = (float)mp->iso;
  M.invSupport = (float)(1 / s->h);
  M.support2 = (float)(s->h * s->h);
  M.poly6 = (float)(315 / (64 * kPI * std::pow(s->h, 9)));
  M.mass = s->P.mass;
  M.rho0 = (float)s->params.rest_density;
  M.maxTris = (uint32_t)mp->max_triangles;
  M.skipBodies = s->nBodyParts > 0 ? 1u : 0u;
  const size_t nVerts = (size_t)M.dim[0] * M.dim[1] * M.dim[2];
  const int par = s->parity;
  const std::vector<f4>& pos = s->pos[par];
  const std::vector<u4>& body = s->body[par];
  // meshDensity (src/mesh_wgsl.js:23-69)
  std::vector<float>& F = s->meshField;
  F.assign(nVerts, 0.0f);
  const float rhoMin = 0.5f * M.rho0;
#pragma omp parallel for schedule(dynamic, 1024)
  for (long long idx = 0; idx < (long long)nVerts; idx++) {
    const int vx = (int)(idx % M.dim[0]), vy = (int)((idx / M.dim[0]) % M.dim[1]),
              vz = (int)(idx / ((long long)M.dim[0] * M.dim[1]));
    const f3 p = {M.origin[0] + M.voxel * (float)vx, M.origin[1] + M.voxel * (float)vy,
                  M.origin[2] + M.voxel * (float)vz};
    const int cx = std::min(std::max(f2i_sat(std::floor((p.x - 0.0f) * M.invSupport)), 0), M.simDim[0] - 1);
    const int cy = std::min(std::max(f2i_sat(std::floor((p.y - 0.0f) * M.invSupport)), 0), M.simDim[1] - 1);
    const int cz = std::min(std::max(f2i_sat(std::floor((p.z - 0.0f) * M.invSupport)), 0), M.simDim[2] - 1);
    const int x0 = std::max(cx - 1, 0), x1 = std::min(cx + 1, M.simDim[0] - 1);
    float acc = 0.0f;
    for (int dz = -1; dz <= 1; dz++) {
      const int z = cz + dz;
      if (z < 0 || z >= M.simDim[2]) continue;
      for (int dy = -1; dy <= 1; dy++) {
        const int y = cy + dy;
        if (y < 0 || y >= M.simDim[1]) continue;
        const uint32_t rowBase = (uint32_t)((z * M.simDim[1] + y) * M.simDim[0]);
        const uint32_t b = s->cellStart[rowBase + x0];
        const uint32_t e = std::min(s->cellStart[rowBase + x1 + 1], (uint32_t)s->n);
        for (uint32_t j = b; j < e; j++) {
          if (M.skipBodies != 0u && body[j].x != 0u) continue;
          const float vol = M.mass / std::max(s->density[j], rhoMin);
          const f3 r = sub3(p, xyz(pos[j]));
          const float r2 = dot3(r, r);
          if (r2 >= M.support2) continue;
          const float t = M.support2 - r2;
          acc = std::fmaf(((vol * M.poly6) * t) * t, t, acc);
        }
      }
    }
    F[(size_t)idx] = acc;
  }
  // blur passes, then the normal field
  for (int k = 0; k < 3 * mp->field_passes; k++) mesh_blur(F, M, mp->blur_axes ? k % 3 : 0);
  s->meshNField = F;
  for (int k = 0; k < 3 * mp->normal_passes; k++) mesh_blur(s->meshNField, M, mp->blur_axes ? k % 3 : 0);
  const std::vector<float>& NF = mp->normal_passes > 0 ? s->meshNField : F;
  // meshMarch (src/mesh_wgsl.js:198-238), triangles in voxel order
  const size_t tris = (size_t)mp->max_triangles;
  s->meshVerts.assign(std::max<size_t>(1, tris) * 6, 0u);
  MeshSink sink{&s->meshVerts, 0, tris};
  static const int tets[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7}, {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};
  for (int vz = 0; vz < M.dim[2] - 1; vz++)
    for (int vy = 0; vy < M.dim[1] - 1; vy++)
      for (int vx = 0; vx < M.dim[0] - 1; vx++) {
        MCorner cn[8];
        int mask = 0;
        for (int k = 0; k < 8; k++) {
          const int x = vx + (k & 1), y = vy + ((k >> 1) & 1), z = vz + ((k >> 2) & 1);
          cn[k].d = mesh_at(F, M, x, y, z);
          mask |= (cn[k].d > M.iso ? 1 : 0) << k;
        }
        if (mask == 0 || mask == 255) continue;
        for (int k = 0; k < 8; k++) {
          const int x = vx + (k & 1), y = vy + ((k >> 1) & 1), z = vz + ((k >> 2) & 1);
          cn[k].p = {(float)x, (float)y, (float)z};
          cn[k].g = {mesh_at(NF, M, x + 1, y, z) - mesh_at(NF, M, x - 1, y, z),
                     mesh_at(NF, M, x, y + 1, z) - mesh_at(NF, M, x, y - 1, z),
                     mesh_at(NF, M, x, y, z + 1) - mesh_at(NF, M, x, y, z - 1)};
        }
        for (int t = 0; t < 6; t++) mesh_tet(M, sink, cn[tets[t][0]], cn[tets[t][1]], cn[tets[t][2]], cn[tets[t][3]]);
      }
  s->meshTris = (int64_t)sink.count;
  s->meshVerts.resize((size_t)std::min<uint64_t>(sink.count, tris) * 6);
  if (!(mp->normal_passes > 0)) s->meshNField = F;
  if (triangles) *triangles = s->meshTris;
  return P4A_OK;
}

int orc_stats(const orc_sim* s, p4a_stats* out) {
  if (!s || !out) return P4A_ERR_ARG;
  *out = s->stats;
  return P4A_OK;
}

int orc_buffer(orc_sim* s, int32_t id, int32_t which, void** ptr, size_t* bytes) {
  if (!s || !ptr) return P4A_ERR_ARG;
  const int w = which < 0 ? s->parity : (which & 1);
  auto set = [&](void* p, size_t b) { *ptr = p; if (bytes) *bytes = b; return P4A_OK; };
  switch (id) {
    case P4A_BUF_POS: return set(s->pos[w].data(), s->pos[w].size() * 16);
    case P4A_BUF_VEL: return set(s->vel[w].data(), s->vel[w].size() * 16);
    case P4A_BUF_PRED: return set(s->pred[w].data(), s->pred[w].size() * 16);
    case P4A_BUF_BODY: return set(s->body[w].data(), s->body[w].size() * 16);
    case P4A_BUF_REST: return set(s->rest[w].data(), s->rest[w].size() * 16);
    case P4A_BUF_DENSITY: return set(s->density.data(), s->density.size() * 4);
    case P4A_BUF_LAMBDA: return set(s->lambda.data(), s->lambda.size() * 4);
    case P4A_BUF_CORR: return set(s->corr.data(), s->corr.size() * 16);
    case P4A_BUF_NORMAL: return set(s->normal.data(), s->normal.size() * 16);
    case P4A_BUF_CELL_START: return set(s->cellStart.data(), s->cellStart.size() * 4);
    case P4A_BUF_BPOS: return set(s->bpos.data(), s->bpos.size() * 16);
    case P4A_BUF_BPSI: return set(s->bpsi.data(), s->bpsi.size() * 4);
    case P4A_BUF_BCELL_START: return set(s->bcellStart.data(), s->bcellStart.size() * 4);
    case P4A_BUF_BODY_CENTRE: return set(s->bodyCentre.data(), s->bodyCentre.size() * 16);
    case P4A_BUF_BODY_REF: return set(s->bodyRef.data(), s->bodyRef.size() * 16);
    case P4A_BUF_BODY_ROT: return set(s->bodyRot.data(), s->bodyRot.size() * 16);
    case P4A_BUF_BODY_INFO: return set(s->bodyInfo.data(), s->bodyInfo.size() * 16);
    case P4A_BUF_STATS_OUT: return set(s->statsOut.data(), s->statsOut.size() * 4);
    case P4A_BUF_SMOOTH_POS: return set(s->smoothPos.data(), s->smoothPos.size() * 16);
    case P4A_BUF_ANISO_G: return set(s->anisoG.data(), s->anisoG.size() * 16);
    case P4A_BUF_MESH_FIELD: return set(s->meshField.data(), s->meshField.size() * 4);
    case P4A_BUF_MESH_NFIELD: return set(s->meshNField.data(), s->meshNField.size() * 4);
    case P4A_BUF_MESH_VERTS: return set(s->meshVerts.data(), s->meshVerts.size() * 4);
    default: return P4A_ERR_ARG;
  }
}

int orc_grid_sort(const p4a_grid* grid, int32_t n, float dt, float gravity, const float* pos,
                  const float* vel, const uint32_t* body, const float* rest, float* pos_out,
                  float* vel_out, float* pred_out, uint32_t* body_out, float* rest_out,
                  uint32_t* cell_start, uint32_t* slot_out) {
  if (!grid || n < 0) return P4A_ERR_ARG;
  Params P{};
  for (int k = 0; k < 3; k++) { P.boxMin[k] = grid->box_min[k]; P.gridDim[k] = grid->dim[k]; }
  P.h = grid->h; P.dt = dt; P.gravity = gravity; P.n = (uint32_t)n;
  P.nCells = (uint32_t)(grid->dim[0] * grid->dim[1] * grid->dim[2]);
  std::vector<f4> vp(n), vv(n), vpred(n);
  std::memcpy(vp.data(), pos, (size_t)n * 16);
  std::memcpy(vv.data(), vel, (size_t)n * 16);
  apply_threads();
  k_predict(P, vp, vv, vpred);
  std::vector<uint32_t> cnt(P.nCells + 1), cs(P.nCells + 2, 0u), cur(P.nCells + 1), slot(n);
  k_sort_slots(P, vpred, cnt, cs, cur, slot);
  for (int i = 0; i < n; i++) {
    const uint32_t s = slot[i];
    std::memcpy(pos_out + 4 * (size_t)s, &vp[i], 16);
    std::memcpy(vel_out + 4 * (size_t)s, &vv[i], 16);
    std::memcpy(pred_out + 4 * (size_t)s, &vpred[i], 16);
    if (body && body_out) std::memcpy(body_out + 4 * (size_t)s, body + 4 * (size_t)i, 16);
    if (rest && rest_out) std::memcpy(rest_out + 4 * (size_t)s, rest + 4 * (size_t)i, 16);
    if (slot_out) slot_out[i] = s;
  }
  std::memcpy(cell_start, cs.data(), (P.nCells + 1) * 4);
  return P4A_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Screen-space fluid rendering (src/ssfr.js:173-356, src/ssfr_wgsl.js,
// src/ssfr_composite_wgsl.js). Rasterisation is restated as the pipeline
// defines it: instances drawn in order, each quad covering the pixels whose
// centres lie inside it, the depth test 'less' against 1.0 applied fragment by
// fragment in draw order, the thickness blended additively (summed in 2^-32 fixed
// point: the sum does not depend on order). Matrices column-major; M * v as nested
// fma over columns; dot() as dot3; exp/log by Cody-Waite reduction + Taylor and
// the atanh series (own restatement, see orc_exp / orc_log).
namespace {

struct v4o { float x, y, z, w; };
inline v4o mv4(const float* m, v4o v) {
  return {std::fmaf(m[12], v.w, std::fmaf(m[8], v.z, std::fmaf(m[4], v.y, m[0] * v.x))),
          std::fmaf(m[13], v.w, std::fmaf(m[9], v.z, std::fmaf(m[5], v.y, m[1] * v.x))),
          std::fmaf(m[14], v.w, std::fmaf(m[10], v.z, std::fmaf(m[6], v.y, m[2] * v.x))),
          std::fmaf(m[15], v.w, std::fmaf(m[11], v.z, std::fmaf(m[7], v.y, m[3] * v.x)))};
}
inline f3 mv3(const m3& m, f3 v) { return {dot3(row3(m, 0), v), dot3(row3(m, 1), v), dot3(row3(m, 2), v)}; }
inline f3 nrm3(f3 a) { const float l = std::sqrt(dot3(a, a)); return {a.x / l, a.y / l, a.z / l}; }
inline float clampo(float x, float lo, float hi) { return std::fmin(std::fmax(x, lo), hi); }
inline float sstep(float e0, float e1, float x) {
  const float t = clampo((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
inline f3 mixo(f3 a, f3 b, float t) {
  const float u = 1.0f - t;
  return {a.x * u + b.x * t, a.y * u + b.y * t, a.z * u + b.z * t};
}
inline f3 refl(f3 i, f3 n) { const float d = 2.0f * dot3(n, i); return {i.x - d * n.x, i.y - d * n.y, i.z - d * n.z}; }
inline f3 refr(f3 i, f3 n, float eta) {
  const float ni = dot3(n, i);
  const float k = 1.0f - eta * eta * (1.0f - ni * ni);
  if (k < 0.0f) return {0, 0, 0};
  const float a = eta * ni + std::sqrt(k);
  return {eta * i.x - a * n.x, eta * i.y - a * n.y, eta * i.z - a * n.z};
}
inline float frac1(float x) { return x - std::floor(x); }

float o_bits(uint32_t b) { float f; std::memcpy(&f, &b, 4); return f; }
uint32_t o_ubits(float f) { uint32_t b; std::memcpy(&b, &f, 4); return b; }
float o_scale2(float x, int k) {
  while (k > 127) { x = x * 1.7014118346046923e38f; k -= 127; }
  while (k < -126) { x = x * 1.1754943508222875e-38f; k += 126; }
  return x * o_bits((uint32_t)(k + 127) << 23);
}
// e^x: x = k ln2 + r (ln2 = 0.693145751953125 + 1.4286067653e-6), e^r by its Taylor
// series to r^8 in Horner form, times 2^k.
float orc_exp(float x) {
  if (x != x) return x;
  if (x > 88.72283935546875f) return INFINITY;
  if (x < -103.97208404541016f) return 0.0f;
  const float k = std::rint(x * 1.44269502162933349609375f);
  float r = std::fmaf(-k, 0.693145751953125f, x);
  r = std::fmaf(-k, 1.428606765330187045e-6f, r);
  float p = 2.48015873015873e-5f;
  p = std::fmaf(p, r, 1.984126984126984e-4f);
  p = std::fmaf(p, r, 1.388888888888889e-3f);
  p = std::fmaf(p, r, 8.333333333333333e-3f);
  p = std::fmaf(p, r, 4.166666666666667e-2f);
  p = std::fmaf(p, r, 1.666666666666667e-1f);
  p = std::fmaf(p, r, 0.5f);
  p = std::fmaf(p, r, 1.0f);
  p = std::fmaf(p, r, 1.0f);
  return o_scale2(p, (int)k);
}
// log x = e ln2 + 2 atanh((m - 1) / (m + 1)), m in [sqrt(1/2), sqrt(2)).
float orc_log(float x) {
  if (x != x || x < 0.0f) return NAN;
  if (x == 0.0f) return -INFINITY;
  if (x == INFINITY) return x;
  int e = 0;
  if (x < 1.1754943508222875e-38f) { x = x * 16777216.0f; e = -24; }
  const uint32_t b = o_ubits(x);
  e += (int)((b >> 23) & 0xffu) - 127;
  float m = o_bits((b & 0x7fffffu) | 0x3f800000u);
  if (m > 1.41421353816986083984375f) { m = m * 0.5f; e += 1; }
  const float s = (m - 1.0f) / (m + 1.0f);
  const float z = s * s;
  float p = 0.15384615384615385f;
  p = std::fmaf(p, z, 0.18181818181818182f);
  p = std::fmaf(p, z, 0.22222222222222222f);
  p = std::fmaf(p, z, 0.2857142857142857f);
  p = std::fmaf(p, z, 0.4f);
  p = std::fmaf(p, z, 0.6666666666666666f);
  p = std::fmaf(p, z, 2.0f);
  const float fe = (float)e;
  return std::fmaf(fe, 0.693145751953125f, std::fmaf(s, p, fe * 1.428606765330187045e-6f));
}
float orc_pow(float x, float y) {
  if (x > 0.0f) return orc_exp(y * orc_log(x));
  if (x == 0.0f) return y > 0.0f ? 0.0f : (y == 0.0f ? 1.0f : INFINITY);
  return NAN;
}

struct OSplat {
  const float *view, *proj, *ivp;
  float pv[16];
  float vw, vh, kernelScale, quadRadius, thickRadius, maxNeighbours;
  bool skipBodies;
};
m3 o_kernel_g(const std::vector<f4>& g, size_t i) {
  const f4 a = g[i * 2], b = g[i * 2 + 1];
  m3 m;
  m.c[0] = {a.x, a.y, a.z};
  m.c[1] = {a.y, a.w, b.x};
  m.c[2] = {a.z, b.x, b.y};
  return m;
}
m3 o_kernel_inverse(const std::vector<f4>& gd, size_t i) {
  const m3 m = o_kernel_g(gd, i);
  const float a = elc(m, 0, 0), b = elc(m, 1, 0), c = elc(m, 2, 0);
  const float d = elc(m, 0, 1), e = elc(m, 1, 1), f = elc(m, 2, 1);
  const float g = elc(m, 0, 2), h = elc(m, 1, 2), k = elc(m, 2, 2);
  const float A = e * k - f * h, B = f * g - d * k, C = d * h - e * g;
  const float det = a * A + b * B + c * C;
  const float inv = 1.0f / (std::fabs(det) < 1.0e-20f ? 1.0e-20f : det);
  m3 o;
  o.c[0] = {A * inv, B * inv, C * inv};
  o.c[1] = {(c * h - b * k) * inv, (a * k - c * g) * inv, (b * g - a * h) * inv};
  o.c[2] = {(b * f - c * e) * inv, (c * d - a * f) * inv, (a * e - b * d) * inv};
  return o;
}
// vertex shader (src/ssfr_wgsl.js:48-83) + rasteriser coverage
bool o_quad(const OSplat& S, const orc_sim* s, size_t ii, int& x0, int& x1, int& y0, int& y1) {
  const f4 c = s->smoothPos[ii];
  if (S.skipBodies && s->body[s->parity][ii].x != 0u) return false;
  if (S.maxNeighbours > 0.0f && s->anisoG[ii * 2 + 1].w > S.maxNeighbours) return false;
  const v4o ec = mv4(S.view, {c.x, c.y, c.z, 1.0f});
  const float zeye = std::fmax(-ec.z, 1.0e-4f);
  const v4o clip = mv4(S.proj, ec);
  f3 e;
  if (S.quadRadius > 0.0f) {
    e = {S.quadRadius, S.quadRadius, S.quadRadius};
  } else {
    m3 v3;
    for (int cc = 0; cc < 3; cc++) v3.c[cc] = {S.view[cc * 4], S.view[cc * 4 + 1], S.view[cc * 4 + 2]};
    const m3 M = matmul(v3, scale3(o_kernel_inverse(s->anisoG, ii), S.kernelScale));
    e = {length3(row3(M, 0)), length3(row3(M, 1)), length3(row3(M, 2))};
  }
  const float znear = std::fmax(zeye - e.z, 1.0e-4f);
  const float hx = S.proj[0] * e.x / znear, hy = S.proj[5] * e.y / znear;
  if (!(clip.w > 0.0f) || clip.z < 0.0f || clip.z > clip.w) return false;
  const float lx = clip.x - hx * clip.w, rx = clip.x + hx * clip.w;
  const float ty = clip.y + hy * clip.w, by = clip.y - hy * clip.w;
  const float fx0 = (lx / clip.w * 0.5f + 0.5f) * S.vw, fx1 = (rx / clip.w * 0.5f + 0.5f) * S.vw;
  const float fy0 = (0.5f - ty / clip.w * 0.5f) * S.vh, fy1 = (0.5f - by / clip.w * 0.5f) * S.vh;
  const float a0 = std::fmax(std::ceil(fx0 - 0.5f), 0.0f), a1 = std::fmin(std::ceil(fx1 - 0.5f), S.vw);
  const float b0 = std::fmax(std::ceil(fy0 - 0.5f), 0.0f), b1 = std::fmin(std::ceil(fy1 - 0.5f), S.vh);
  if (!(a0 < a1) || !(b0 < b1)) return false;
  x0 = (int)a0; x1 = (int)a1; y0 = (int)b0; y1 = (int)b1;
  return true;
}
void o_ray(const float* ivp, float nx, float ny, f3& ro, f3& rd) {
  const v4o nh = mv4(ivp, {nx, ny, -1.0f, 1.0f});
  const v4o fh = mv4(ivp, {nx, ny, 1.0f, 1.0f});
  ro = {nh.x / nh.w, nh.y / nh.w, nh.z / nh.w};
  rd = nrm3(sub3({fh.x / fh.w, fh.y / fh.w, fh.z / fh.w}, ro));
}
void o_frag_ray(const OSplat& S, int px, int py, f3& ro, f3& rd) {
  const float fx = (float)px + 0.5f, fy = (float)py + 0.5f;
  o_ray(S.ivp, fx / S.vw * 2.0f - 1.0f, 1.0f - fy / S.vh * 2.0f, ro, rd);
}
// depthFS (src/ssfr_wgsl.js:85-108, 122-139)
bool o_depth_frag(const OSplat& S, const orc_sim* s, size_t ii, int px, int py, float& depth, float& eyeZ) {
  const f4 c4 = s->smoothPos[ii];
  const f3 centre = {c4.x, c4.y, c4.z};
  f3 ro, rd;
  o_frag_ray(S, px, py, ro, rd);
  const m3 G = scale3(o_kernel_g(s->anisoG, ii), 1.0f / S.kernelScale);
  const f3 oc = sub3(ro, centre);
  const f3 ga = mv3(G, rd), gb = mv3(G, oc);
  const float A = dot3(ga, ga), B = 2.0f * dot3(ga, gb), C = dot3(gb, gb) - 1.0f;
  const float disc = B * B - 4.0f * A * C;
  if (disc <= 0.0f || A <= 0.0f) return false;
  const float sq = std::sqrt(disc);
  const float t = (-B - sq) / (2.0f * A);
  if (!(t > 0.0f)) return false;
  const f3 p = {ro.x + rd.x * t, ro.y + rd.y * t, ro.z + rd.z * t};
  const v4o ve = mv4(S.view, {p.x, p.y, p.z, 1.0f});
  const v4o cl = mv4(S.pv, {p.x, p.y, p.z, 1.0f});
  depth = clampo(cl.z / cl.w, 0.0f, 1.0f);
  eyeZ = ve.z;
  return true;
}
float o_fetch(const std::vector<float>& z, int x, int y, int w, int h) {
  if (x < 0 || y < 0 || x >= w || y >= h) return -1.0e4f;
  return z[(size_t)y * w + x];
}
void o_nr(float& z, float& w, float& wo, float& up, float& lo, float lowerClamp, float thr) {
  if (z > up) { w = 0.0f; wo = 0.0f; }
  else if (z < lo) { z = lowerClamp; }
  else { up = std::fmax(up, z + thr); lo = std::fmin(lo, z - thr); }
}
struct OFilt { int dirX, dirY, maxRadius, mode, clean, cleanRadius; float sigmaWorld, proj11, viewH, delta, mu, rangeSigma; };
void o_filter(const OFilt& F, const std::vector<float>& in, std::vector<float>& out, int W, int H) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int py = 0; py < H; py++)
    for (int px = 0; px < W; px++) {
      const float zi = in[(size_t)py * W + px];
      if (zi < -1.0e3f) { out[(size_t)py * W + px] = zi; continue; }
      const float sigma = std::fmax(F.sigmaWorld * F.viewH * F.proj11 / (2.0f * std::fabs(zi)), 0.5f);
      int R = (int)std::fmin(3.0f * sigma, (float)F.maxRadius);
      if (F.clean) R = F.cleanRadius;
      float sg = sigma;
      if (F.clean) sg = std::fmax((float)R / 3.0f, 1.0e-3f);
      const float inv2s2 = 1.0f / (2.0f * sg * sg);
      float upP = zi + F.delta, loP = zi - F.delta, upM = zi + F.delta, loM = zi - F.delta;
      const float lc = zi - F.mu;
      float sum = zi, wsum = 1.0f;
      if (F.clean) {
        float up = zi + F.delta, lo = zi - F.delta;
        for (int dy = 1; dy <= R; dy++)
          for (int dx = 1; dx <= R; dx++) {
            const float g = orc_exp(-(float)(dx * dx + dy * dy) * inv2s2);
            float za = o_fetch(in, px + dx, py + dy, W, H), zb = o_fetch(in, px + dx, py - dy, W, H);
            float zc = o_fetch(in, px - dx, py + dy, W, H), zd = o_fetch(in, px - dx, py - dy, W, H);
            float wa = g, wb = g, wc = g, wd = g;
            o_nr(za, wa, wd, up, lo, lc, F.delta);
            o_nr(zb, wb, wc, up, lo, lc, F.delta);
            o_nr(zc, wc, wb, up, lo, lc, F.delta);
            o_nr(zd, wd, wa, up, lo, lc, F.delta);
            sum = sum + za * wa + zb * wb + zc * wc + zd * wd;
            wsum = wsum + wa + wb + wc + wd;
          }
        for (int t = 1; t <= R; t++) {
          const float g = orc_exp(-(float)(t * t) * inv2s2);
          float zv[4] = {o_fetch(in, px + t, py, W, H), o_fetch(in, px - t, py, W, H),
                         o_fetch(in, px, py + t, W, H), o_fetch(in, px, py - t, W, H)};
          float wv[4] = {g, g, g, g};
          o_nr(zv[0], wv[0], wv[1], up, lo, lc, F.delta);
          o_nr(zv[1], wv[1], wv[0], up, lo, lc, F.delta);
          o_nr(zv[2], wv[2], wv[3], up, lo, lc, F.delta);
          o_nr(zv[3], wv[3], wv[2], up, lo, lc, F.delta);
          for (int k = 0; k < 4; k++) { sum = sum + zv[k] * wv[k]; wsum = wsum + wv[k]; }
        }
      } else {
        for (int t = 1; t <= R; t++) {
          float zj = o_fetch(in, px + F.dirX * t, py + F.dirY * t, W, H);
          float zk = o_fetch(in, px - F.dirX * t, py - F.dirY * t, W, H);
          const float g = orc_exp(-(float)(t * t) * inv2s2);
          float wj = g, wk = g;
          if (F.mode == 2) {
            o_nr(zj, wj, wk, upP, loP, lc, F.delta);
            o_nr(zk, wk, wj, upM, loM, lc, F.delta);
            sum = sum + zj * wj + zk * wk;
            wsum = wsum + wj + wk;
          } else {
            if (!(zj < -1.0e3f)) {
              float w = g;
              if (F.mode == 1) { const float dz = zj - zi; w = w * orc_exp(-dz * dz / (2.0f * F.rangeSigma * F.rangeSigma)); }
              sum = sum + w * zj; wsum = wsum + w;
            }
            if (!(zk < -1.0e3f)) {
              float w = g;
              if (F.mode == 1) { const float dz = zk - zi; w = w * orc_exp(-dz * dz / (2.0f * F.rangeSigma * F.rangeSigma)); }
              sum = sum + w * zk; wsum = wsum + w;
            }
          }
        }
      }
      out[(size_t)py * W + px] = sum / wsum;
    }
}

// composite (src/ssfr_composite_wgsl.js)
// Environment map uniforms (src/ray_wgsl.js:29-31, 46-50): size 0 = none.
struct OEnv {
  const uint16_t* texels;
  int size;
  float intensity, yawCos, yawSin;
};
struct OComp {
  const float *ivp, *iv;
  f3 boxMin, absorb, sunDir;
  float proj00, proj11, ior, sunIntensity, roughness, exposure, groundReflection, thicknessScale;
  int bodyCount, floorPlane, debug;
  const float* bdata;  // 24 floats per body
  OEnv env;
};
// IEEE half to float, exactly.
float o_half_to_float(uint16_t h) {
  const uint32_t sgn = (uint32_t)(h & 0x8000u) << 16, e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
  uint32_t bits;
  if (e == 0) {
    if (m == 0) {
      bits = sgn;
    } else {  // subnormal: m * 2^-24
      const float v = (float)m * 5.9604644775390625e-8f;
      std::memcpy(&bits, &v, 4);
      bits |= sgn;
    }
  } else if (e == 31) {
    bits = sgn | 0x7f800000u | (m << 13);
  } else {
    bits = sgn | ((e + 112u) << 23) | (m << 13);
  }
  float v;
  std::memcpy(&v, &bits, 4);
  return v;
}
// textureSampleLevel(cube, linear clamp-to-edge sampler, d, 0): the face of the
// largest component (x, then y, then z on ties), (s, t) on it, bilinear within the
// face with its edges clamped.
f3 o_cube_sample(const OEnv& E, f3 d) {
  const float ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
  int face;
  float ma, sc, tc;
  if (ax >= ay && ax >= az) {
    face = d.x >= 0.0f ? 0 : 1;
    ma = ax;
    sc = d.x >= 0.0f ? -d.z : d.z;
    tc = -d.y;
  } else if (ay >= az) {
    face = d.y >= 0.0f ? 2 : 3;
    ma = ay;
    sc = d.x;
    tc = d.y >= 0.0f ? d.z : -d.z;
  } else {
    face = d.z >= 0.0f ? 4 : 5;
    ma = az;
    sc = d.z >= 0.0f ? d.x : -d.x;
    tc = -d.y;
  }
  const float n = (float)E.size;
  const float u = std::fmin(std::fmax(0.5f * (sc / ma + 1.0f) * n - 0.5f, -1.0f), n);
  const float v = std::fmin(std::fmax(0.5f * (tc / ma + 1.0f) * n - 0.5f, -1.0f), n);
  const float fu = std::floor(u), fv = std::floor(v);
  const float tx = u - fu, ty = v - fv;
  const int x0 = std::min(std::max((int)fu, 0), E.size - 1), x1 = std::min(std::max((int)fu + 1, 0), E.size - 1);
  const int y0 = std::min(std::max((int)fv, 0), E.size - 1), y1 = std::min(std::max((int)fv + 1, 0), E.size - 1);
  auto texel = [&](int y, int x) {
    const uint16_t* t = E.texels + ((((size_t)face * E.size + y) * E.size) + x) * 4;
    return f3{o_half_to_float(t[0]), o_half_to_float(t[1]), o_half_to_float(t[2])};
  };
  const f3 top = mixo(texel(y0, x0), texel(y0, x1), tx), bot = mixo(texel(y1, x0), texel(y1, x1), tx);
  return mixo(top, bot, ty);
}
// envSample (src/ray_wgsl.js:46-50).
f3 o_env_sample(const OEnv& E, f3 d) {
  const f3 r = {E.yawCos * d.x + E.yawSin * d.z, d.y, -E.yawSin * d.x + E.yawCos * d.z};
  const f3 c = o_cube_sample(E, r);
  return {c.x * E.intensity, c.y * E.intensity, c.z * E.intensity};
}
OEnv o_env_uniform(const orc_sim* s, double intensity, double yaw) {
  OEnv E{};
  E.texels = s->envCube.data();
  E.size = s->envCube.empty() ? 0 : s->envSize;
  E.intensity = (float)intensity;
  const float y = (float)yaw;
  E.yawCos = (float)std::cos((double)y);
  E.yawSin = (float)std::sin((double)y);
  return E;
}
f3 o_bd(const OComp& C, int k) { return {C.bdata[k * 4], C.bdata[k * 4 + 1], C.bdata[k * 4 + 2]}; }
float o_body_dist(const OComp& C, int i, f3 p) {
  const int b = i * 6;
  const f3 centre = o_bd(C, b);
  const int shape = (int)(C.bdata[b * 4 + 3] + 0.5f);
  const f3 h = o_bd(C, b + 1);
  const f3 d0 = sub3(p, centre);
  const f3 q = {dot3(o_bd(C, b + 2), d0), dot3(o_bd(C, b + 3), d0), dot3(o_bd(C, b + 4), d0)};
  if (shape == 1) return length3(q) - h.x;
  if (shape == 2) {
    const float tx = std::sqrt(std::fmaf(q.z, q.z, q.x * q.x)) - h.x, ty = q.y;
    return std::sqrt(std::fmaf(ty, ty, tx * tx)) - h.y;
  }
  const f3 d = {std::fabs(q.x) - h.x, std::fabs(q.y) - h.y, std::fabs(q.z) - h.z};
  return length3({std::fmax(d.x, 0.0f), std::fmax(d.y, 0.0f), std::fmax(d.z, 0.0f)}) +
         std::fmin(std::fmax(d.x, std::fmax(d.y, d.z)), 0.0f);
}
struct OTrace { float t; f3 nrm, col; };
OTrace o_trace(const OComp& C, f3 ro, f3 rd, float tMax) {
  OTrace o{-1.0f, {0, 1, 0}, {0.8f, 0.8f, 0.8f}};
  if (C.bodyCount == 0) return o;
  float t = 1.0e-4f;
  for (int it = 0; it < 128; it++) {
    const f3 p = {ro.x + rd.x * t, ro.y + rd.y * t, ro.z + rd.z * t};
    float dist = 1.0e30f;
    int id = -1;
    for (int i = 0; i < C.bodyCount; i++) {
      const float d = o_body_dist(C, i, p);
      if (d < dist) { dist = d; id = i; }
    }
    if (dist < 5.0e-5f) {
      const float e = 2.0e-4f;
      o.nrm = nrm3({o_body_dist(C, id, {p.x + e, p.y, p.z}) - o_body_dist(C, id, {p.x - e, p.y, p.z}),
                    o_body_dist(C, id, {p.x, p.y + e, p.z}) - o_body_dist(C, id, {p.x, p.y - e, p.z}),
                    o_body_dist(C, id, {p.x, p.y, p.z + e}) - o_body_dist(C, id, {p.x, p.y, p.z - e})});
      o.col = o_bd(C, id * 6 + 5);
      o.t = t;
      return o;
    }
    t += std::fmax(dist, 1.0e-4f);
    if (t > tMax) break;
  }
  return o;
}
const f3 kHazeO = {0.62f, 0.74f, 0.90f};
f3 o_sky(const OComp& C, f3 d) {
  if (C.env.size > 0) return o_env_sample(C.env, d);
  const float h = clampo(d.y, 0.0f, 1.0f);
  f3 c = mixo(kHazeO, {0.25f, 0.48f, 0.85f}, sstep(0.0f, 0.16f, h));
  c = mixo(c, {0.09f, 0.28f, 0.72f}, sstep(0.10f, 0.85f, h));
  const float s = std::fmax(dot3(d, C.sunDir), 0.0f);
  const float p1 = orc_pow(s, 3000.0f), p2 = orc_pow(s, 24.0f);
  c = {c.x + 1.00f * p1 * 14.0f, c.y + 0.96f * p1 * 14.0f, c.z + 0.88f * p1 * 14.0f};
  c = {c.x + 1.00f * p2 * 0.20f, c.y + 0.92f * p2 * 0.20f, c.z + 0.78f * p2 * 0.20f};
  return c;
}
f3 o_floor(f3 p) {
  const float gx = std::fabs(frac1(p.x) - 0.5f), gz = std::fabs(frac1(p.z) - 0.5f);
  const float line = 1.0f - sstep(0.0f, 0.015f, std::fmin(gx, gz));
  f3 c = mixo({0.30f, 0.305f, 0.315f}, {0.50f, 0.51f, 0.52f}, line * 0.8f);
  const float fs = std::floor(p.x) + std::floor(p.z);
  const float chk = fs - 2.0f * std::floor(fs * 0.5f);
  const float m = 0.88f * (1.0f - chk) + 1.10f * chk;
  return {c.x * m, c.y * m, c.z * m};
}
f3 o_background(const OComp& C, f3 o, f3 d) {
  if (C.floorPlane != 0 && d.y < -1.0e-4f) {
    const float t = (C.boxMin.y - o.y) / d.y;
    if (t > 0.0f) {
      const f3 p = {o.x + d.x * t, o.y + d.y * t, o.z + d.z * t};
      const float fade = 1.0f - orc_exp(-0.02f * t);
      return mixo(o_floor(p), C.env.size > 0 ? o_env_sample(C.env, d) : kHazeO, fade);
    }
  }
  return o_sky(C, d);
}
f3 o_shade_body(const OComp& C, f3 n, f3 base, f3 rd, f3 env) {
  const float ndl = std::fmax(dot3(n, C.sunDir), 0.0f);
  const f3 h = nrm3(sub3(C.sunDir, rd));
  const float spec = orc_pow(std::fmax(dot3(n, h), 0.0f), 60.0f);
  const float fres = orc_pow(1.0f - std::fmax(dot3({-rd.x, -rd.y, -rd.z}, n), 0.0f), 4.0f);
  const float k = 0.22f + 0.78f * ndl;
  return {base.x * k + 0.7f * spec + env.x * fres * 0.25f, base.y * k + 0.7f * spec + env.y * fres * 0.25f,
          base.z * k + 0.7f * spec + env.z * fres * 0.25f};
}
f3 o_env_reflect(const OComp& C, f3 d) {
  if (C.env.size > 0) return o_env_sample(C.env, d);
  if (d.y >= 0.0f) return o_sky(C, d);
  return mixo(kHazeO, {0.32f, 0.325f, 0.335f}, clampo(-d.y * 4.0f, 0.0f, 1.0f));
}
f3 o_water_reflect(const OComp& C, f3 d, f3 n) {
  const f3 physical = o_env_reflect(C, d);
  if (d.y >= 0.0f || C.groundReflection >= 1.0f) return physical;
  const float top = sstep(0.819152f, 0.939693f, n.y);
  const float below = sstep(0.0f, 0.10f, -d.y);
  const float suppress = (1.0f - clampo(C.groundReflection, 0.0f, 1.0f)) * top * below;
  const float xzl = std::fmax(std::sqrt(std::fmaf(d.z, d.z, d.x * d.x)), 1.0e-4f);
  return mixo(physical, o_sky(C, {d.x / xzl, 0.0f, d.z / xzl}), suppress);
}
f3 o_scene_color(const OComp& C, f3 o, f3 d) {
  const OTrace b = o_trace(C, o, d, 60.0f);
  if (b.t < 0.0f) return o_background(C, o, d);
  const f3 p = {o.x + d.x * b.t, o.y + d.y * b.t, o.z + d.z * b.t};
  const f3 po = {p.x + b.nrm.x * 1.0e-4f, p.y + b.nrm.y * 1.0e-4f, p.z + b.nrm.z * 1.0e-4f};
  return o_shade_body(C, b.nrm, b.col, d, o_background(C, po, refl(d, b.nrm)));
}
float o_fresnel(float cosI, float n1, float n2) {
  const float eta = n1 / n2;
  const float sinT2 = eta * eta * (1.0f - cosI * cosI);
  if (sinT2 >= 1.0f) return 1.0f;
  const float cosT = std::sqrt(1.0f - sinT2);
  const float rs = (n1 * cosI - n2 * cosT) / (n1 * cosI + n2 * cosT);
  const float rp = (n1 * cosT - n2 * cosI) / (n1 * cosT + n2 * cosI);
  return clampo(0.5f * (rs * rs + rp * rp), 0.0f, 1.0f);
}
float o_ggx(f3 n, f3 v, f3 l, float rough) {
  const float a = std::fmax(rough * rough, 1.0e-4f);
  const f3 h = nrm3(add3(l, v));
  const float ndh = std::fmax(dot3(n, h), 0.0f), ndl = std::fmax(dot3(n, l), 0.0f), ndv = std::fmax(dot3(n, v), 0.0f);
  const float a2 = a * a;
  const float d = ndh * ndh * (a2 - 1.0f) + 1.0f;
  const float ndf = a2 / std::fmax(3.14159265f * d * d, 1.0e-7f);
  const float k = a * 0.5f;
  const float gl = ndl / std::fmax(ndl * (1.0f - k) + k, 1.0e-5f);
  const float gv = ndv / std::fmax(ndv * (1.0f - k) + k, 1.0e-5f);
  return ndf * gl * gv * ndl / std::fmax(4.0f * ndl * ndv, 1.0e-4f);
}
f3 o_tonemap(const OComp& C, f3 c) {
  f3 col = {c.x * C.exposure, c.y * C.exposure, c.z * C.exposure};
  const float m = 1.0f + std::fmax(std::fmax(col.x, col.y), col.z) * 0.35f;
  col = {col.x / m, col.y / m, col.z / m};
  const float g = (float)(1.0 / 2.2);
  return {orc_pow(col.x, g), orc_pow(col.y, g), orc_pow(col.z, g)};
}
uint32_t o_rgba8(f3 c) {
  auto u = [](float v) { return (uint32_t)(int)std::floor(clampo(v, 0.0f, 1.0f) * 255.0f + 0.5f); };
  return u(c.x) | (u(c.y) << 8) | (u(c.z) << 16) | (255u << 24);
}

}  // namespace

extern "C" {

int orc_ssfr(orc_sim* s, const p4a_ssfr_params* sp, const float* bodies, int32_t bodyCount) {
  if (!s || !s->ready || !sp || sp->width < 1 || sp->height < 1 || bodyCount < 0 || (bodyCount > 0 && !bodies))
    return P4A_ERR_ARG;
  if (s->smoothPos.size() < (size_t)s->n) return P4A_ERR_STATE;
  const p4a_ssfr_params& q = *sp;
  apply_threads();
  const double rs = std::min(1.0, std::max(0.25, q.render_scale));
  const int W = std::max(1, (int)std::floor(q.width * rs + 0.5)), H = std::max(1, (int)std::floor(q.height * rs + 0.5));
  const bool half = q.thickness_half_res && q.thickness_filter_size >= 4;
  const int TW = half ? (W + 1) >> 1 : W, TH = half ? (H + 1) >> 1 : H;
  const double kPiD = 3.14159265358979323846;
  const double el = q.sun_elevation * kPiD / 180, az = q.sun_azimuth * kPiD / 180;
  const double sun[3] = {std::cos(el) * std::sin(az), std::sin(el), std::cos(el) * std::cos(az)};
  const double sl = std::sqrt(sun[0] * sun[0] + sun[1] * sun[1] + sun[2] * sun[2]);
  double absorb[3];
  for (int k = 0; k < 3; k++) absorb[k] = q.absorption * -std::log(std::min(1.0, std::max(1e-3, q.transmit[k])));
  const double spacing = s->params.spacing, support = s->h;
  const double r = 0.5 * spacing;
  const float scale = (float)(q.splat_radius * spacing / support);
  const float thickRadius = (float)(q.thickness_radius * spacing);
  OSplat S0{q.view, q.proj, q.inv_view_proj, {}, (float)W, (float)H, scale, 0.0f, thickRadius,
            (float)q.depth_cull_neighbours, s->nBodyParts > 0};
  for (int c = 0; c < 4; c++)
    for (int rr = 0; rr < 4; rr++)
      S0.pv[c * 4 + rr] = std::fmaf(q.proj[12 + rr], q.view[c * 4 + 3],
                                    std::fmaf(q.proj[8 + rr], q.view[c * 4 + 2],
                                              std::fmaf(q.proj[4 + rr], q.view[c * 4 + 1], q.proj[rr] * q.view[c * 4])));
  OSplat S1 = S0;
  S1.vw = (float)TW;
  S1.vh = (float)TH;
  S1.quadRadius = thickRadius;
  S1.maxNeighbours = 0.0f;
  const int n = s->n;
  // depth: instances in order, test 'less' per fragment against the cleared 1.0
  std::vector<float> zbuf((size_t)W * H, 1.0f), eyeZ((size_t)W * H, -1.0e4f);
  for (int ii = 0; ii < n; ii++) {
    int x0, x1, y0, y1;
    if (!o_quad(S0, s, (size_t)ii, x0, x1, y0, y1)) continue;
    for (int py = y0; py < y1; py++)
      for (int px = x0; px < x1; px++) {
        float depth, ez;
        if (!o_depth_frag(S0, s, (size_t)ii, px, py, depth, ez)) continue;
        const size_t o = (size_t)py * W + px;
        if (depth < zbuf[o]) { zbuf[o] = depth; eyeZ[o] = ez; }
      }
  }
  s->ssfrRaw = eyeZ;
  // thickness: additive, in 2^-32 fixed point
  std::vector<uint64_t> acc((size_t)TW * TH, 0);
  const float tr2 = thickRadius * thickRadius;
  for (int ii = 0; ii < n; ii++) {
    int x0, x1, y0, y1;
    if (!o_quad(S1, s, (size_t)ii, x0, x1, y0, y1)) continue;
    const f4 c4 = s->smoothPos[ii];
    const f3 centre = {c4.x, c4.y, c4.z};
    for (int py = y0; py < y1; py++)
      for (int px = x0; px < x1; px++) {
        f3 ro, rd;
        o_frag_ray(S1, px, py, ro, rd);
        const f3 oc = sub3(ro, centre);
        const float b = dot3(oc, rd), c = dot3(oc, oc) - tr2;
        const float disc = b * b - c;
        if (disc <= 0.0f) continue;
        const float chord = 2.0f * std::sqrt(disc);
        acc[(size_t)py * TW + px] += (uint64_t)std::llrint(chord * 4294967296.0f);
      }
  }
  std::vector<float> thick((size_t)TW * TH), tmp((size_t)TW * TH);
  for (size_t i = 0; i < thick.size(); i++) thick[i] = (float)((double)acc[i] * (1.0 / 4294967296.0));
  // thickness blur (src/ssfr_wgsl.js:155-183, src/ssfr.js:227-233)
  if (q.thickness_filter_size > 0) {
    const int size = TW < W ? std::max(1, q.thickness_filter_size >> 1) : q.thickness_filter_size;
    const float sigma = std::fmax((float)size / 3.0f, 1.0e-3f);
    const float two = 2.0f * sigma * sigma;
    for (int p = 0; p < 2; p++) {
      const int dx = p == 0 ? 1 : 0, dy = p == 0 ? 0 : 1;
      const std::vector<float>& src = p == 0 ? thick : tmp;
      std::vector<float>& dst = p == 0 ? tmp : thick;
      for (int py = 0; py < TH; py++)
        for (int px = 0; px < TW; px++) {
          float sum = 0.0f, wsum = 0.0f;
          for (int i = -size; i <= size; i++) {
            const int x = std::min(std::max(px + dx * i, 0), TW - 1), y = std::min(std::max(py + dy * i, 0), TH - 1);
            const float w = orc_exp(-(float)(i * i) / two);
            sum = sum + src[(size_t)y * TW + x] * w;
            wsum = wsum + w;
          }
          dst[(size_t)py * TW + px] = sum / wsum;
        }
    }
  }
  s->ssfrThick = thick;
  // depth filter passes (src/ssfr.js:151-164, 331-338)
  OFilt fl[3];
  for (int k = 0; k < 3; k++) {
    fl[k].dirX = k == 0 ? 1 : 0;
    fl[k].dirY = k == 1 ? 1 : 0;
    fl[k].maxRadius = q.filter_max_radius;
    fl[k].mode = q.filter;
    fl[k].clean = k == 2 ? 1 : 0;
    fl[k].cleanRadius = q.cleanup_radius;
    fl[k].sigmaWorld = (float)(q.filter_sigma * r);
    fl[k].proj11 = q.proj[5];
    fl[k].viewH = (float)H;
    fl[k].delta = (float)(q.narrow_delta * r);
    fl[k].mu = (float)(q.narrow_mu * r);
    fl[k].rangeSigma = (float)std::max(q.bilateral_range * r, 1e-4);
  }
  std::vector<float> zb[2] = {eyeZ, std::vector<float>((size_t)W * H)};
  int src = 0;
  for (int it = 0; it < q.filter_iterations * 2; it++) { o_filter(fl[it % 2], zb[src], zb[1 - src], W, H); src = 1 - src; }
  if (q.cleanup_pass && q.filter_iterations > 0) { o_filter(fl[2], zb[src], zb[1 - src], W, H); src = 1 - src; }
  s->ssfrEyeZ = zb[src];
  // body depth and composite
  OComp C{};
  C.ivp = q.inv_view_proj;
  C.iv = q.inv_view;
  C.boxMin = {0.0f, 0.0f, 0.0f};
  C.absorb = {(float)absorb[0], (float)absorb[1], (float)absorb[2]};
  C.sunDir = {(float)(sun[0] / sl), (float)(sun[1] / sl), (float)(sun[2] / sl)};
  C.proj00 = q.proj[0];
  C.proj11 = q.proj[5];
  C.ior = (float)q.ior;
  C.sunIntensity = (float)q.sun_intensity;
  C.roughness = (float)q.roughness;
  C.exposure = (float)q.exposure;
  C.groundReflection = (float)q.ground_reflection;
  C.env = o_env_uniform(s, q.env_intensity, q.env_yaw);
  C.thicknessScale = (float)q.thickness_scale;
  C.bodyCount = bodyCount;
  C.floorPlane = q.floor_plane ? 1 : 0;
  C.debug = q.debug;
  C.bdata = bodies;
  std::vector<float> bodyT((size_t)W * H, 1.0e30f);
  if (bodyCount > 0) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int py = 0; py < H; py++)
      for (int px = 0; px < W; px++) {
        f3 ro, rd;
        o_ray(q.inv_view_proj, ((float)px + 0.5f) / (float)W * 2.0f - 1.0f,
              1.0f - ((float)py + 0.5f) / (float)H * 2.0f, ro, rd);
        const OTrace b = o_trace(C, ro, rd, 60.0f);
        if (b.t >= 0.0f) bodyT[(size_t)py * W + px] = b.t;
      }
  }
  s->ssfrBodyT = bodyT;
  const std::vector<float>& z = zb[src];
  const float msx = (float)((double)W / std::max(1, q.width)), msy = (float)((double)H / std::max(1, q.height));
  s->ssfrImage.assign((size_t)q.width * q.height, 0u);
#pragma omp parallel for schedule(dynamic, 4)
  for (int y = 0; y < q.height; y++)
    for (int x = 0; x < q.width; x++) {
      const float fx = (float)x + 0.5f, fy = (float)y + 0.5f;
      const float nx = fx / (float)q.width * 2.0f - 1.0f, ny = 1.0f - fy / (float)q.height * 2.0f;
      const float u = nx * 0.5f + 0.5f, v = 0.5f - ny * 0.5f;
      const int ipx = (int)(fx * msx), ipy = (int)(fy * msy);
      const float zi = z[(size_t)ipy * W + ipx];
      const float tu = u * (float)TW - 0.5f, tv = v * (float)TH - 0.5f;
      const float fu = std::floor(tu), fv = std::floor(tv);
      const float au = tu - fu, av = tv - fv;
      const int i0 = std::min(std::max((int)fu, 0), TW - 1), i1 = std::min(std::max((int)fu + 1, 0), TW - 1);
      const int j0 = std::min(std::max((int)fv, 0), TH - 1), j1 = std::min(std::max((int)fv + 1, 0), TH - 1);
      const float top = thick[(size_t)j0 * TW + i0] * (1.0f - au) + thick[(size_t)j0 * TW + i1] * au;
      const float bot = thick[(size_t)j1 * TW + i0] * (1.0f - au) + thick[(size_t)j1 * TW + i1] * au;
      float th = (top * (1.0f - av) + bot * av) * C.thicknessScale;
      f3 ro, rd;
      o_ray(q.inv_view_proj, nx, ny, ro, rd);
      uint32_t out;
      if (C.debug == 3) {
        out = o_rgba8({th, th * 0.25f, 0.0f});
      } else if (C.debug == 2 || C.debug == 4) {
        const float d = C.debug == 4 ? s->ssfrRaw[(size_t)ipy * W + ipx] : zi;
        float sg = 0.0f;
        if (!(d < -1.0e3f)) sg = clampo(-d / 4.0f, 0.0f, 1.0f);
        out = o_rgba8({1.0f - sg, 1.0f - sg, 1.0f - sg});
      } else {
        const float tBody = bodyT[(size_t)ipy * W + ipx];
        if (C.debug == 5) {
          out = tBody > 1.0e29f ? o_rgba8({0.0f, 0.0f, 0.6f}) : o_rgba8({frac1(tBody), frac1(tBody * 0.1f), 0.0f});
        } else {
          const f3 p0 = {-nx * zi / C.proj00, -ny * zi / C.proj11, zi};
          const v4o pw = mv4(C.iv, {p0.x, p0.y, p0.z, 1.0f});
          const f3 p = {pw.x, pw.y, pw.z};
          const bool bodyInFront = tBody < length3(sub3(p, ro));
          if (zi < -1.0e3f || bodyInFront) {
            out = o_rgba8(o_tonemap(C, o_scene_color(C, ro, rd)));
          } else {
            auto vp = [&](float ax, float ay, float zz) { return f3{-ax * zz / C.proj00, -ay * zz / C.proj11, zz}; };
            const float pxs = 2.0f / (float)W, pys = 2.0f / (float)H;
            const float zxp = o_fetch(z, ipx + 1, ipy, W, H), zxm = o_fetch(z, ipx - 1, ipy, W, H);
            const float zyp = o_fetch(z, ipx, ipy - 1, W, H), zym = o_fetch(z, ipx, ipy + 1, W, H);
            const f3 dxr = sub3(vp(nx + pxs, ny, zxp), p0), dxl = sub3(p0, vp(nx - pxs, ny, zxm));
            const f3 dyt = sub3(vp(nx, ny + pys, zyp), p0), dyb = sub3(p0, vp(nx, ny - pys, zym));
            const f3 dpx = std::fabs(dxr.z) < std::fabs(dxl.z) ? dxr : dxl;
            const f3 dpy = std::fabs(dyt.z) < std::fabs(dyb.z) ? dyt : dyb;
            const f3 nView = nrm3(cross3(dpx, dpy));
            m3 iv3;
            for (int cc = 0; cc < 3; cc++) iv3.c[cc] = {C.iv[cc * 4], C.iv[cc * 4 + 1], C.iv[cc * 4 + 2]};
            f3 nn = nrm3(mv3(iv3, nView));
            if (nn.x != nn.x || nn.y != nn.y || nn.z != nn.z) nn = {-rd.x, -rd.y, -rd.z};
            if (dot3(nn, rd) > 0.0f) nn = {-nn.x, -nn.y, -nn.z};
            if (C.debug == 1) {
              out = o_rgba8({nn.x * 0.5f + 0.5f, nn.y * 0.5f + 0.5f, nn.z * 0.5f + 0.5f});
            } else {
              const f3 mrd = {-rd.x, -rd.y, -rd.z};
              const float kS = o_fresnel(std::fmax(dot3(mrd, nn), 0.0f), 1.0f, C.ior);
              const f3 rfl = o_water_reflect(C, refl(rd, nn), nn);
              f3 refrDir = refr(rd, nn, 1.0f / C.ior);
              if (dot3(refrDir, refrDir) < 1.0e-8f) refrDir = refl(rd, nn);
              const f3 ro2 = {p.x + refrDir.x * 1.0e-3f, p.y + refrDir.y * 1.0e-3f, p.z + refrDir.z * 1.0e-3f};
              const OTrace st = o_trace(C, ro2, refrDir, 60.0f);
              f3 hit;
              if (st.t >= 0.0f) {
                hit = o_shade_body(C, st.nrm, st.col, refrDir, o_env_reflect(C, refl(refrDir, st.nrm)));
                th = std::fmin(th, st.t);
              } else {
                hit = o_background(C, ro2, refrDir);
              }
              const f3 trans = {hit.x * orc_exp(-C.absorb.x * th), hit.y * orc_exp(-C.absorb.y * th),
                                hit.z * orc_exp(-C.absorb.z * th)};
              f3 col = mixo(trans, rfl, kS);
              const float gs = o_ggx(nn, mrd, C.sunDir, C.roughness);
              col = {col.x + 1.0f * C.sunIntensity * gs * kS, col.y + 0.97f * C.sunIntensity * gs * kS,
                     col.z + 0.90f * C.sunIntensity * gs * kS};
              out = o_rgba8(o_tonemap(C, col));
            }
          }
        }
      }
      s->ssfrImage[(size_t)y * q.width + x] = out;
    }
  s->ssfrDims[0] = q.width; s->ssfrDims[1] = q.height; s->ssfrDims[2] = W; s->ssfrDims[3] = H;
  s->ssfrDims[4] = TW; s->ssfrDims[5] = TH;
  return P4A_OK;
}

int orc_ssfr_buffer(orc_sim* s, int32_t which, void** ptr, size_t* bytes) {
  if (!s || !ptr || !bytes) return P4A_ERR_ARG;
  switch (which) {
    case P4A_SSFR_EYEZ: *ptr = s->ssfrEyeZ.data(); *bytes = s->ssfrEyeZ.size() * 4; return P4A_OK;
    case P4A_SSFR_RAWZ: *ptr = s->ssfrRaw.data(); *bytes = s->ssfrRaw.size() * 4; return P4A_OK;
    case P4A_SSFR_THICK: *ptr = s->ssfrThick.data(); *bytes = s->ssfrThick.size() * 4; return P4A_OK;
    case P4A_SSFR_IMAGE: *ptr = s->ssfrImage.data(); *bytes = s->ssfrImage.size() * 4; return P4A_OK;
    case P4A_SSFR_BODYT: *ptr = s->ssfrBodyT.data(); *bytes = s->ssfrBodyT.size() * 4; return P4A_OK;
    default: return P4A_ERR_ARG;
  }
}

float orc_expf(float x) { return orc_exp(x); }
float orc_logf(float x) { return orc_log(x); }

}  // extern "C"

// ---------------------------------------------------------------------------
// Ray-marched surface (src/ray.js:30-97, src/ray_wgsl.js): per pixel, the eye ray
// through the density field of the last orc_mesh, the cubic iso crossing per
// cell, shading as the SSFR composite (shared helpers above).
namespace {

struct ORay {
  std::vector<float>* field;
  int dim[3];
  f3 origin;
  float voxel, iso, ior, skin, roughness;
  int thickSteps, debug;
  float cosDeg[4];
};
float o_fget(const ORay& R, int x, int y, int z) {
  x = std::min(std::max(x, 0), R.dim[0] - 1);
  y = std::min(std::max(y, 0), R.dim[1] - 1);
  z = std::min(std::max(z, 0), R.dim[2] - 1);
  return (*R.field)[((size_t)z * R.dim[1] + y) * R.dim[0] + x];
}
struct OCell { float d000, d100, d010, d110, d001, d101, d011, d111; };
OCell o_cell(const ORay& R, int x, int y, int z) {
  return {o_fget(R, x, y, z), o_fget(R, x + 1, y, z), o_fget(R, x, y + 1, z), o_fget(R, x + 1, y + 1, z),
          o_fget(R, x, y, z + 1), o_fget(R, x + 1, y, z + 1), o_fget(R, x, y + 1, z + 1), o_fget(R, x + 1, y + 1, z + 1)};
}
inline float lerpo(float a, float b, float t) { return a * (1.0f - t) + b * t; }
float o_tri_local(const OCell& k, f3 u) {
  const float x00 = lerpo(k.d000, k.d100, u.x), x10 = lerpo(k.d010, k.d110, u.x);
  const float x01 = lerpo(k.d001, k.d101, u.x), x11 = lerpo(k.d011, k.d111, u.x);
  return lerpo(lerpo(x00, x10, u.y), lerpo(x01, x11, u.y), u.z);
}
float o_tri_at(const ORay& R, f3 g) {
  const int cx = (int)std::floor(g.x), cy = (int)std::floor(g.y), cz = (int)std::floor(g.z);
  return o_tri_local(o_cell(R, cx, cy, cz), {clampo(g.x - (float)cx, 0.0f, 1.0f), clampo(g.y - (float)cy, 0.0f, 1.0f),
                                              clampo(g.z - (float)cz, 0.0f, 1.0f)});
}
struct OCubic { float A, B, C, D; };
float o_cubic_at(const OCubic& c, float t) { return ((c.A * t + c.B) * t + c.C) * t + c.D; }
float o_segment(const OCell& k, f3 u0, f3 du, float iso) {
  const float third = (float)(1.0 / 3.0), two = (float)(2.0 / 3.0);
  const float f0 = o_tri_local(k, u0);
  const float f1 = o_tri_local(k, {u0.x + du.x * third, u0.y + du.y * third, u0.z + du.z * third});
  const float f2 = o_tri_local(k, {u0.x + du.x * two, u0.y + du.y * two, u0.z + du.z * two});
  const float f3v = o_tri_local(k, {u0.x + du.x, u0.y + du.y, u0.z + du.z});
  const float g1 = f1 - f0, g2 = f2 - f0, g3 = f3v - f0;
  OCubic c;
  c.A = 4.5f * (3.0f * g1 - 3.0f * g2 + g3);
  c.B = -(27.0f * g1 - 9.0f * g3 + 8.0f * c.A) / 6.0f;
  c.C = g3 - c.A - c.B;
  c.D = f0;
  float e0 = 2.0f, e1 = 2.0f;
  const float a = 3.0f * c.A, b = 2.0f * c.B, cc = c.C;
  if (std::fabs(a) > 1.0e-12f) {
    const float disc = b * b - 4.0f * a * cc;
    if (disc > 0.0f) {
      const float sq = std::sqrt(disc);
      const float r0 = (-b - sq) / (2.0f * a), r1 = (-b + sq) / (2.0f * a);
      e0 = std::fmin(r0, r1);
      e1 = std::fmax(r0, r1);
    }
  } else if (std::fabs(b) > 1.0e-12f) {
    e0 = -cc / b;
  }
  float bounds[4] = {0.0f, 1.0f, 1.0f, 1.0f};
  int n = 1;
  if (e0 > 0.0f && e0 < 1.0f) bounds[n++] = e0;
  if (e1 > 0.0f && e1 < 1.0f && e1 > e0) bounds[n++] = e1;
  bounds[n++] = 1.0f;
  float lo = bounds[0], vlo = o_cubic_at(c, lo) - iso;
  for (int i = 1; i < n; i++) {
    float hi = bounds[i], vhi = o_cubic_at(c, hi) - iso;
    if ((vlo <= 0.0f && vhi >= 0.0f) || (vlo >= 0.0f && vhi <= 0.0f)) {
      float t = lo;
      for (int it = 0; it < 12; it++) {  // solveMonotone
        t = lo + (hi - lo) * (-vlo) / std::fmax(vhi - vlo, 1.0e-9f);
        t = clampo(t, lo, hi);
        const float v = o_cubic_at(c, t) - iso;
        if (v * vlo > 0.0f) { lo = t; vlo = v; } else { hi = t; vhi = v; }
      }
      return t;
    }
    lo = hi;
    vlo = vhi;
  }
  return -1.0f;
}
struct OSlab { bool hit; float t0, t1; };
OSlab o_box(f3 o, f3 d, f3 lo, f3 hi) {
  const f3 inv = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
  const f3 a = {(lo.x - o.x) * inv.x, (lo.y - o.y) * inv.y, (lo.z - o.z) * inv.z};
  const f3 b = {(hi.x - o.x) * inv.x, (hi.y - o.y) * inv.y, (hi.z - o.z) * inv.z};
  OSlab s;
  s.t0 = std::fmax(std::fmax(std::fmin(a.x, b.x), std::fmin(a.y, b.y)), std::fmin(a.z, b.z));
  s.t1 = std::fmin(std::fmin(std::fmax(a.x, b.x), std::fmax(a.y, b.y)), std::fmax(a.z, b.z));
  s.hit = s.t1 > std::fmax(s.t0, 0.0f);
  return s;
}
float o_march(const ORay& R, const OComp& C, f3 ro, f3 rd, float tStart, float tEnd, f3& pos) {
  const f3 g0 = {(ro.x - R.origin.x) / R.voxel, (ro.y - R.origin.y) / R.voxel, (ro.z - R.origin.z) / R.voxel};
  const f3 gd = {rd.x / R.voxel, rd.y / R.voxel, rd.z / R.voxel};
  const f3 p0 = {g0.x + gd.x * tStart, g0.y + gd.y * tStart, g0.z + gd.z * tStart};
  int c[3] = {std::min(std::max((int)std::floor(p0.x), 0), R.dim[0] - 2),
              std::min(std::max((int)std::floor(p0.y), 0), R.dim[1] - 2),
              std::min(std::max((int)std::floor(p0.z), 0), R.dim[2] - 2)};
  auto sgn = [](float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); };
  const float gda[3] = {gd.x, gd.y, gd.z}, g0a[3] = {g0.x, g0.y, g0.z};
  int stp[3];
  float tMax[3], tDelta[3];
  for (int a = 0; a < 3; a++) {
    stp[a] = (int)sgn(gda[a]);
    const float invD = 1.0f / std::fmax(std::fabs(gda[a]), 1.0e-12f);
    const float nextEdge = (float)c[a] + std::fmax((float)stp[a], 0.0f);
    tMax[a] = (nextEdge - g0a[a]) / gda[a];
    tDelta[a] = invD;
    if (gda[a] == 0.0f) { tMax[a] = 1.0e30f; tDelta[a] = 1.0e30f; }
  }
  float t = tStart;
  for (int i = 0; i < 4096; i++) {
    const float tNext = std::fmin(std::fmin(tMax[0], tMax[1]), tMax[2]);
    const float segEnd = std::fmin(tNext, tEnd);
    if (segEnd > t) {
      const OCell k = o_cell(R, c[0], c[1], c[2]);
      const f3 u0 = {g0.x + gd.x * t - (float)c[0], g0.y + gd.y * t - (float)c[1], g0.z + gd.z * t - (float)c[2]};
      const float span = segEnd - t;
      const f3 du = {gd.x * span, gd.y * span, gd.z * span};
      const float s = o_segment(k, u0, du, R.iso);
      if (s >= 0.0f) {
        const float tHit = t + s * (segEnd - t);
        const f3 p = {ro.x + rd.x * tHit, ro.y + rd.y * tHit, ro.z + rd.z * tHit};
        bool inside = false;
        if (C.bodyCount > 0) {
          float dist = 1.0e30f;
          for (int b = 0; b < C.bodyCount; b++) dist = std::fmin(dist, o_body_dist(C, b, p));
          inside = dist < 0.0f;
        }
        if (!inside) { pos = p; return tHit; }
      }
    }
    t = tNext;
    if (t >= tEnd) break;
    if (tMax[0] <= tMax[1] && tMax[0] <= tMax[2]) { c[0] += stp[0]; tMax[0] += tDelta[0]; }
    else if (tMax[1] <= tMax[2]) { c[1] += stp[1]; tMax[1] += tDelta[1]; }
    else { c[2] += stp[2]; tMax[2] += tDelta[2]; }
    if (c[0] < 0 || c[1] < 0 || c[2] < 0 || c[0] > R.dim[0] - 2 || c[1] > R.dim[1] - 2 || c[2] > R.dim[2] - 2) break;
  }
  return -1.0f;
}
float o_optical(const ORay& R, f3 ro, f3 rd, float tMax) {
  const f3 lo = R.origin;
  const f3 hi = {lo.x + R.voxel * (float)(R.dim[0] - 1), lo.y + R.voxel * (float)(R.dim[1] - 1),
                 lo.z + R.voxel * (float)(R.dim[2] - 1)};
  const OSlab s = o_box(ro, rd, lo, hi);
  if (!s.hit) return 0.0f;
  const float a = std::fmax(s.t0, 0.0f), b = std::fmin(std::fmax(s.t1, 0.0f), tMax);
  if (b <= a) return 0.0f;
  const float dt = (b - a) / (float)R.thickSteps;
  float acc = 0.0f;
  for (int i = 0; i < R.thickSteps; i++) {
    const float t = a + ((float)i + 0.5f) * dt;
    acc += sstep(R.iso * 0.55f, R.iso * 1.45f,
                 o_tri_at(R, {(ro.x + rd.x * t - lo.x) / R.voxel, (ro.y + rd.y * t - lo.y) / R.voxel,
                              (ro.z + rd.z * t - lo.z) / R.voxel}));
  }
  return acc * dt;
}

// The mesh surface pass (src/mesh.js:380-396; meshDrawWGSL vs + fsSurf,
// src/mesh_wgsl.js:268-321): the triangles in order into an eye-depth map (-1e4
// where empty) and a normal map (w = 1 where covered). Each triangle is clipped to
// 0 <= z <= w (Sutherland-Hodgman, near plane then far plane, the cut vertices'
// clip coordinates, positions and normals interpolated linearly) and its visible
// part drawn as a fan. A pixel centre inside a fan triangle or on its edge is
// covered; the depth test keeps the least screen depth, ties to the lower
// (triangle * 4 + fan index). World position and normal are interpolated
// perspective-correctly.
struct OSVert {
  v4o c;
  f3 p, n;
};
constexpr int kOClipMax = 5;
OSVert o_lerp_vert(const OSVert& A, const OSVert& B, float t) {
  OSVert o;
  o.c = {A.c.x + t * (B.c.x - A.c.x), A.c.y + t * (B.c.y - A.c.y), A.c.z + t * (B.c.z - A.c.z),
         A.c.w + t * (B.c.w - A.c.w)};
  o.p = {A.p.x + t * (B.p.x - A.p.x), A.p.y + t * (B.p.y - A.p.y), A.p.z + t * (B.p.z - A.p.z)};
  o.n = {A.n.x + t * (B.n.x - A.n.x), A.n.y + t * (B.n.y - A.n.y), A.n.z + t * (B.n.z - A.n.z)};
  return o;
}
int o_clip_plane(const OSVert* in, int m, OSVert* out, int cap, bool far) {
  int k = 0;
  for (int a = 0; a < m; a++) {
    const OSVert& A = in[a];
    const OSVert& B = in[a + 1 < m ? a + 1 : 0];
    const float da = far ? A.c.w - A.c.z : A.c.z, db = far ? B.c.w - B.c.z : B.c.z;
    if (da >= 0.0f && k < cap) out[k++] = A;
    if ((da >= 0.0f) != (db >= 0.0f) && k < cap) out[k++] = o_lerp_vert(A, B, da / (da - db));
  }
  return k;
}
int o_surf_clip(const orc_sim* s, const float* vp, size_t t, OSVert P[kOClipMax]) {
  const float voxel = (float)s->meshVoxel, origin = (float)s->meshOrigin;
  OSVert a[3], b[kOClipMax - 1];
  for (int k = 0; k < 3; k++) {
    const uint32_t vx = s->meshVerts[(3 * t + k) * 2], vy = s->meshVerts[(3 * t + k) * 2 + 1];
    const float px = (float)(vx & 0xFFFFu) / 65535.0f, py = (float)(vx >> 16) / 65535.0f,
                pz = (float)(vy & 0xFFFFu) / 65535.0f;
    a[k].p = {origin + px * (float)(s->meshDim[0] - 1) * voxel, origin + py * (float)(s->meshDim[1] - 1) * voxel,
              origin + pz * (float)(s->meshDim[2] - 1) * voxel};
    const uint32_t oct = vy >> 16;
    const float ex = (float)(oct & 0xFFu) / 255.0f * 2.0f - 1.0f, ey = (float)(oct >> 8) / 255.0f * 2.0f - 1.0f;
    f3 m = {ex, ey, 1.0f - std::fabs(ex) - std::fabs(ey)};
    if (m.z < 0.0f)
      m = {(1.0f - std::fabs(m.y)) * (m.x >= 0.0f ? 1.0f : -1.0f), (1.0f - std::fabs(m.x)) * (m.y >= 0.0f ? 1.0f : -1.0f),
           m.z};
    a[k].n = nrm3(m);
    a[k].c = mv4(vp, {a[k].p.x, a[k].p.y, a[k].p.z, 1.0f});
  }
  const int m = o_clip_plane(a, 3, b, kOClipMax - 1, false);
  return o_clip_plane(b, m, P, kOClipMax, true);
}
struct OSurfTri {
  v4o clip[3];
  float sx[3], sy[3], sz[3], area;
  f3 p[3], n[3];
};
bool o_fan_tri(const OSVert* P, int fan, int W, int H, OSurfTri& T) {
  for (int k = 0; k < 3; k++) {
    const OSVert& v = P[k == 0 ? 0 : fan + k];
    T.clip[k] = v.c;
    T.p[k] = v.p;
    T.n[k] = v.n;
    if (!(v.c.w > 0.0f)) return false;
    T.sx[k] = (v.c.x / v.c.w * 0.5f + 0.5f) * (float)W;
    T.sy[k] = (0.5f - v.c.y / v.c.w * 0.5f) * (float)H;
    T.sz[k] = v.c.z / v.c.w;
  }
  T.area = (T.sx[1] - T.sx[0]) * (T.sy[2] - T.sy[0]) - (T.sx[2] - T.sx[0]) * (T.sy[1] - T.sy[0]);
  return T.area != 0.0f;
}
bool o_surf_bary(const OSurfTri& T, float cx, float cy, float b[3]) {
  float w0 = (T.sx[2] - T.sx[1]) * (cy - T.sy[1]) - (T.sy[2] - T.sy[1]) * (cx - T.sx[1]);
  float w1 = (T.sx[0] - T.sx[2]) * (cy - T.sy[2]) - (T.sy[0] - T.sy[2]) * (cx - T.sx[2]);
  float w2 = (T.sx[1] - T.sx[0]) * (cy - T.sy[0]) - (T.sy[1] - T.sy[0]) * (cx - T.sx[0]);
  float a = T.area;
  if (a < 0.0f) {
    w0 = -w0;
    w1 = -w1;
    w2 = -w2;
    a = -a;
  }
  if (w0 < 0.0f || w1 < 0.0f || w2 < 0.0f) return false;
  b[0] = w0 / a;
  b[1] = w1 / a;
  b[2] = w2 / a;
  return true;
}
void o_surface(const orc_sim* s, const float* view, const float* vp, int W, int H, std::vector<float>& surfZ,
               std::vector<f3>& surfN) {
  const size_t px = (size_t)W * H;
  std::vector<uint64_t> key(px, ~0ull);
  const size_t tris = s->meshVerts.size() / 6;
  for (size_t t = 0; t < tris; t++) {
    OSVert P[kOClipMax];
    const int m = o_surf_clip(s, vp, t, P);
    for (int fan = 0; fan + 2 < m; fan++) {
      OSurfTri T;
      if (!o_fan_tri(P, fan, W, H, T)) continue;
      const float lx = std::fmin(T.sx[0], std::fmin(T.sx[1], T.sx[2])), hx = std::fmax(T.sx[0], std::fmax(T.sx[1], T.sx[2]));
      const float ly = std::fmin(T.sy[0], std::fmin(T.sy[1], T.sy[2])), hy = std::fmax(T.sy[0], std::fmax(T.sy[1], T.sy[2]));
      const int x0 = (int)std::fmin(std::fmax(std::ceil(lx - 0.5f), 0.0f), (float)W);
      const int x1 = (int)std::fmax(std::fmin(std::floor(hx - 0.5f), (float)W - 1.0f), -1.0f);
      const int y0 = (int)std::fmin(std::fmax(std::ceil(ly - 0.5f), 0.0f), (float)H);
      const int y1 = (int)std::fmax(std::fmin(std::floor(hy - 0.5f), (float)H - 1.0f), -1.0f);
      for (int y = y0; y <= y1; y++)
        for (int x = x0; x <= x1; x++) {
          float b[3];
          if (!o_surf_bary(T, (float)x + 0.5f, (float)y + 0.5f, b)) continue;
          const float depth = b[0] * T.sz[0] + b[1] * T.sz[1] + b[2] * T.sz[2] + 0.0f;  // -0 -> +0
          if (!(depth < 1.0f)) continue;
          uint32_t bits;
          memcpy(&bits, &depth, 4);
          const uint64_t k = ((uint64_t)bits << 32) | (uint32_t)(t * 4 + (size_t)fan);
          uint64_t& slot = key[(size_t)y * W + x];
          if (k < slot) slot = k;
        }
    }
  }
  surfZ.assign(px, -1.0e4f);
  surfN.assign(px, f3{0.0f, 0.0f, 0.0f});
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      const size_t o = (size_t)y * W + x;
      if (key[o] == ~0ull) continue;
      const uint32_t id = (uint32_t)(key[o] & 0xffffffffu);
      const int fan = (int)(id & 3u);
      OSVert P[kOClipMax];
      const int m = o_surf_clip(s, vp, id >> 2, P);
      OSurfTri T;
      float b[3];
      if (!(fan + 2 < m) || !o_fan_tri(P, fan, W, H, T) || !o_surf_bary(T, (float)x + 0.5f, (float)y + 0.5f, b))
        continue;
      const float q0 = b[0] / T.clip[0].w, q1 = b[1] / T.clip[1].w, q2 = b[2] / T.clip[2].w;
      const float qs = q0 + q1 + q2;
      const f3 wp = {(q0 * T.p[0].x + q1 * T.p[1].x + q2 * T.p[2].x) / qs,
                     (q0 * T.p[0].y + q1 * T.p[1].y + q2 * T.p[2].y) / qs,
                     (q0 * T.p[0].z + q1 * T.p[1].z + q2 * T.p[2].z) / qs};
      const f3 wn = {(q0 * T.n[0].x + q1 * T.n[1].x + q2 * T.n[2].x) / qs,
                     (q0 * T.n[0].y + q1 * T.n[1].y + q2 * T.n[2].y) / qs,
                     (q0 * T.n[0].z + q1 * T.n[1].z + q2 * T.n[2].z) / qs};
      surfZ[o] = mv4(view, {wp.x, wp.y, wp.z, 1.0f}).z;
      surfN[o] = nrm3(wn);
    }
}

}  // namespace

extern "C" {

int orc_ray(orc_sim* s, const p4a_ray_params* rp, const float* bodies, int32_t bodyCount) {
  if (!s || !s->ready || !rp || rp->width < 1 || rp->height < 1 || bodyCount < 0 || (bodyCount > 0 && !bodies))
    return P4A_ERR_ARG;
  if (s->meshDim[0] < 2 || s->meshField.empty()) return P4A_ERR_STATE;
  const p4a_ray_params& q = *rp;
  apply_threads();
  const double kPiD = 3.14159265358979323846;
  const double el = q.sun_elevation * kPiD / 180, az = q.sun_azimuth * kPiD / 180;
  const double sun[3] = {std::cos(el) * std::sin(az), std::sin(el), std::cos(el) * std::cos(az)};
  const double sl = std::sqrt(sun[0] * sun[0] + sun[1] * sun[1] + sun[2] * sun[2]);
  OComp C{};
  C.ivp = q.inv_view_proj;
  C.iv = q.inv_view;
  C.boxMin = {0.0f, 0.0f, 0.0f};
  double ab[3];
  for (int k = 0; k < 3; k++) ab[k] = q.absorption * -std::log(std::min(1.0, std::max(1e-3, q.transmit[k])));
  C.absorb = {(float)ab[0], (float)ab[1], (float)ab[2]};
  C.sunDir = {(float)(sun[0] / sl), (float)(sun[1] / sl), (float)(sun[2] / sl)};
  C.sunIntensity = (float)q.sun_intensity;
  C.roughness = (float)q.roughness;
  C.exposure = (float)q.exposure;
  C.groundReflection = (float)q.ground_reflection;
  C.env = o_env_uniform(s, q.env_intensity, q.env_yaw);
  C.bodyCount = bodyCount;
  C.floorPlane = q.floor_plane ? 1 : 0;
  C.debug = q.debug;
  C.bdata = bodies;
  ORay R{};
  R.field = &s->meshField;
  for (int k = 0; k < 3; k++) R.dim[k] = s->meshDim[k];
  R.origin = {(float)s->meshOrigin, (float)s->meshOrigin, (float)s->meshOrigin};
  R.voxel = (float)s->meshVoxel;
  R.iso = (float)q.iso;
  R.ior = (float)q.ior;
  R.skin = (float)q.skin_width;
  R.roughness = (float)q.roughness;
  R.thickSteps = q.thickness_steps;
  R.debug = q.debug;
  const double deg[4] = {5.0, 10.0, 20.0, 40.0};
  for (int k = 0; k < 4; k++) R.cosDeg[k] = (float)std::cos(deg[k] * kPiD / 180);
  const f3 eye = {q.eye[0], q.eye[1], q.eye[2]};
  const f3 volLo = R.origin;
  const f3 volHi = {volLo.x + R.voxel * (float)(R.dim[0] - 1), volLo.y + R.voxel * (float)(R.dim[1] - 1),
                    volLo.z + R.voxel * (float)(R.dim[2] - 1)};
  s->rayImage.assign((size_t)q.width * q.height, 0u);
  s->rayDims[0] = q.width;
  s->rayDims[1] = q.height;
  const bool useSurface = q.use_surface != 0;
  std::vector<float> surfZ;
  std::vector<f3> surfN;
  if (useSurface) {
    float vp[16];
    for (int c = 0; c < 4; c++)
      for (int rr = 0; rr < 4; rr++)
        vp[c * 4 + rr] = std::fmaf(q.proj[12 + rr], q.view[c * 4 + 3],
                                   std::fmaf(q.proj[8 + rr], q.view[c * 4 + 2],
                                             std::fmaf(q.proj[4 + rr], q.view[c * 4 + 1], q.proj[rr] * q.view[c * 4])));
    o_surface(s, q.view, vp, q.width, q.height, surfZ, surfN);
  }
  const float proj00 = q.proj[0], proj11 = q.proj[5];
#pragma omp parallel for schedule(dynamic, 2)
  for (int y = 0; y < q.height; y++)
    for (int x = 0; x < q.width; x++) {
      const float nx = ((float)x + 0.5f) / (float)q.width * 2.0f - 1.0f;
      const float ny = 1.0f - ((float)y + 0.5f) / (float)q.height * 2.0f;
      const v4o nh = mv4(q.inv_view_proj, {nx, ny, -1.0f, 1.0f}), fh = mv4(q.inv_view_proj, {nx, ny, 1.0f, 1.0f});
      const f3 nearP = {nh.x / nh.w, nh.y / nh.w, nh.z / nh.w}, farP = {fh.x / fh.w, fh.y / fh.w, fh.z / fh.w};
      const f3 ro = eye, rd = nrm3(sub3(farP, nearP));
      float tHit = -1.0f;
      f3 hit = {0, 0, 0}, meshN = {0, 1, 0};
      if (useSurface) {
        // meshSurfaceHit (src/ray_wgsl.js:397-412)
        const size_t o = (size_t)y * q.width + x;
        const float z = surfZ[o];
        const f3 nv = surfN[o];
        if (!(z < -1.0e3f) && !(dot3(nv, nv) < 1.0e-8f)) {
          const v4o wv = mv4(q.inv_view, {-nx * z / proj00, -ny * z / proj11, z, 1.0f});
          hit = {wv.x, wv.y, wv.z};
          meshN = nrm3(nv);
          tHit = length3(sub3(hit, ro));
        }
      } else {
        const OSlab slab = o_box(ro, rd, volLo, volHi);
        if (slab.hit) tHit = o_march(R, C, ro, rd, std::fmax(slab.t0, 0.0f) + 1.0e-5f, slab.t1, hit);
      }
      float tMaxBody = 60.0f;
      if (tHit >= 0.0f) tMaxBody = tHit + R.skin;
      const OTrace bt = o_trace(C, ro, rd, tMaxBody);
      f3 col = {0, 0, 0}, n = {0, 1, 0};
      float thick = 0.0f;
      if (bt.t >= 0.0f && (tHit < 0.0f || bt.t < tHit + R.skin)) {
        col = o_shade_body(C, bt.nrm, bt.col, rd, o_env_reflect(C, refl(rd, bt.nrm)));
      } else if (tHit < 0.0f) {
        col = o_background(C, ro, rd);
      } else {
        if (useSurface) {
          n = meshN;
        } else {
          const f3 g = {(hit.x - R.origin.x) / R.voxel, (hit.y - R.origin.y) / R.voxel,
                        (hit.z - R.origin.z) / R.voxel};
          const f3 sn = {o_tri_at(R, {g.x + 1.0f, g.y, g.z}) - o_tri_at(R, {g.x - 1.0f, g.y, g.z}),
                         o_tri_at(R, {g.x, g.y + 1.0f, g.z}) - o_tri_at(R, {g.x, g.y - 1.0f, g.z}),
                         o_tri_at(R, {g.x, g.y, g.z + 1.0f}) - o_tri_at(R, {g.x, g.y, g.z - 1.0f})};
          n = nrm3({-sn.x, -sn.y, -sn.z});
        }
        if (dot3(n, rd) > 0.0f) n = {-n.x, -n.y, -n.z};
        const f3 mrd = {-rd.x, -rd.y, -rd.z};
        const float kS = o_fresnel(std::fmax(dot3(mrd, n), 0.0f), 1.0f, R.ior);
        const f3 reflDir = refl(rd, n);
        f3 refrDir = refr(rd, n, 1.0f / R.ior);
        if (dot3(refrDir, refrDir) < 1.0e-8f) refrDir = reflDir;
        const f3 rfl = o_water_reflect(C, reflDir, n);
        const float off = R.voxel * 0.02f;
        const f3 ro2 = {hit.x + refrDir.x * off, hit.y + refrDir.y * off, hit.z + refrDir.z * off};
        const OTrace st = o_trace(C, ro2, refrDir, 60.0f);
        f3 trans = st.t >= 0.0f ? o_shade_body(C, st.nrm, st.col, refrDir, o_env_reflect(C, refl(refrDir, st.nrm)))
                                : o_background(C, ro2, refrDir);
        thick = o_optical(R, ro2, refrDir, st.t >= 0.0f ? st.t : 1.0e30f);
        trans = {trans.x * orc_exp(-C.absorb.x * thick), trans.y * orc_exp(-C.absorb.y * thick),
                 trans.z * orc_exp(-C.absorb.z * thick)};
        col = mixo(trans, rfl, kS);
        const float gs = o_ggx(n, mrd, C.sunDir, R.roughness);
        col = {col.x + 1.0f * C.sunIntensity * gs * kS, col.y + 0.97f * C.sunIntensity * gs * kS,
               col.z + 0.90f * C.sunIntensity * gs * kS};
      }
      if (R.debug == 1) {
        col = tHit < 0.0f ? f3{0, 0, 0} : f3{n.x * 0.5f + 0.5f, n.y * 0.5f + 0.5f, n.z * 0.5f + 0.5f};
      } else if (R.debug == 2) {
        col = tHit < 0.0f ? f3{0, 0, 0} : f3{frac1(tHit), frac1(tHit * 0.1f), 0.0f};
      } else if (R.debug == 3) {
        col = {thick, thick * 0.25f, 0.0f};
      } else if (R.debug == 4) {
        f3 c4 = {0.1f, 0.3f, 1.0f};
        if (refl(rd, n).y < 0.0f) c4 = {1.0f, 0.1f, 0.1f};
        col = tHit < 0.0f ? f3{0, 0, 0} : c4;
      } else if (R.debug == 6) {
        col = tHit < 0.0f ? o_background(C, ro, rd) : o_water_reflect(C, refl(rd, n), n);
      } else if (R.debug == 5) {
        if (tHit < 0.0f) {
          col = {0, 0, 0};
        } else {
          const float a = clampo(std::fabs(n.y), 0.0f, 1.0f);
          if (a > R.cosDeg[0]) col = {0.1f, 0.3f, 1.0f};
          else if (a > R.cosDeg[1]) col = {0.1f, 0.9f, 0.9f};
          else if (a > R.cosDeg[2]) col = {0.2f, 0.9f, 0.2f};
          else if (a > R.cosDeg[3]) col = {0.95f, 0.9f, 0.2f};
          else col = {1.0f, 0.15f, 0.1f};
        }
      }
      s->rayImage[(size_t)y * q.width + x] = o_rgba8(o_tonemap(C, col));
    }
  return P4A_OK;
}

int orc_ray_image(orc_sim* s, void** ptr, size_t* bytes) {
  if (!s || !ptr || !bytes) return P4A_ERR_ARG;
  *ptr = s->rayImage.data();
  *bytes = s->rayImage.size() * 4;
  return P4A_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Environment.load (src/env.js:180-236), restated: the panorama resampled into the
// base level of a cube map in double (the JS number type), each sample rounded to
// float and then to half by toHalf (src/env.js:125-147).
namespace {

uint16_t o_to_half(float v) {
  uint32_t x;
  std::memcpy(&x, &v, 4);
  const uint32_t sgn = (x >> 16) & 0x8000u;
  const int e = (int)((x >> 23) & 0xffu) - 112;
  uint32_t m = x & 0x7fffffu;
  if (e <= 0) {
    if (e < -10) return (uint16_t)sgn;
    m = (m | 0x800000u) >> (1 - e);
    return (uint16_t)(sgn | ((m + 0x1000u) >> 13));
  }
  if (e >= 0x1f) return (uint16_t)(sgn | 0x7c00u);
  return (uint16_t)(sgn | ((uint32_t)e << 10) | ((m + 0x1000u) >> 13));
}

// The panorama's bilinear value in direction (dx, dy, dz) (sampleEquirect, src/env.js:94-113).
void o_equirect(const float* src, int w, int h, double dx, double dy, double dz, float out[3]) {
  const double kPiD = 3.14159265358979323846;
  const double len = std::sqrt(dx * dx + dy * dy + dz * dz);
  dx /= len;
  dy /= len;
  dz /= len;
  const double u = 0.5 + std::atan2(dx, dz) / (2 * kPiD);
  const double v = std::acos(std::min(1.0, std::max(-1.0, dy))) / kPiD;
  const double fx = u * w - 0.5, fy = v * h - 0.5;
  const double x0 = std::floor(fx), y0 = std::floor(fy);
  const double tx = fx - x0, ty = fy - y0;
  auto at = [&](long long x, long long y, int c) -> double {
    x = ((x % w) + w) % w;
    y = std::min<long long>(h - 1, std::max<long long>(0, y));
    return src[(y * w + x) * 3 + c];
  };
  const long long ix = (long long)x0, iy = (long long)y0;
  for (int c = 0; c < 3; c++) {
    const double a = at(ix, iy, c) * (1 - tx) + at(ix + 1, iy, c) * tx;
    const double b = at(ix, iy + 1, c) * (1 - tx) + at(ix + 1, iy + 1, c) * tx;
    out[c] = (float)(a * (1 - ty) + b * ty);
  }
}

}  // namespace

extern "C" {

int orc_set_environment(orc_sim* s, const float* rgb, int32_t w, int32_t h) {
  if (!s) return P4A_ERR_ARG;
  s->envCube.clear();
  s->envSize = 0;
  if (!rgb) return P4A_OK;
  if (w < 2 || h < 1 || w < 2 * h - 2 || w > 2 * h + 2) return P4A_ERR_ARG;
  const int size = std::min(2048, std::max(16, w / 4));
  s->envCube.assign((size_t)6 * size * size * 4, 0);
  const uint16_t one = o_to_half(1.0f);
  for (int f = 0; f < 6; f++)
    for (int y = 0; y < size; y++) {
      const double t = 2 * (y + 0.5) / size - 1;
      for (int x = 0; x < size; x++) {
        const double sv = 2 * (x + 0.5) / size - 1;
        double d[3];  // faceDir (src/env.js:115-124)
        if (f == 0) { d[0] = 1; d[1] = -t; d[2] = -sv; }
        else if (f == 1) { d[0] = -1; d[1] = -t; d[2] = sv; }
        else if (f == 2) { d[0] = sv; d[1] = 1; d[2] = t; }
        else if (f == 3) { d[0] = sv; d[1] = -1; d[2] = -t; }
        else if (f == 4) { d[0] = sv; d[1] = -t; d[2] = 1; }
        else { d[0] = -sv; d[1] = -t; d[2] = -1; }
        float c[3];
        o_equirect(rgb, w, h, d[0], d[1], d[2], c);
        uint16_t* o = &s->envCube[(((size_t)f * size + y) * size + x) * 4];
        o[0] = o_to_half(c[0]);
        o[1] = o_to_half(c[1]);
        o[2] = o_to_half(c[2]);
        o[3] = one;
      }
    }
  s->envSize = size;
  return P4A_OK;
}

int orc_environment(orc_sim* s, const void** ptr, int32_t* size) {
  if (!s || !ptr || !size) return P4A_ERR_ARG;
  *ptr = s->envCube.data();
  *size = s->envSize;
  return P4A_OK;
}

}  // extern "C"
