// environment.cpp — Environment.load (src/env.js:180-236) on the host: an
// equirectangular panorama resampled into the six faces of a cube map stored as
// rgba16float texels. The reference builds the faces in JavaScript on the CPU and
// uploads them; this does the same arithmetic in double (the JS number type),
// rounds each sample to float (the Float32Array it is written to) and then to half
// with the reference's own rounding (toHalf, src/env.js:125-147). Only the base
// level is built: the render passes sample level 0 alone.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "p4a_internal.h"

namespace p4a {

int env_face_size(int width) { return std::min(2048, std::max(16, width / 4)); }

// toHalf's conversion of one float (src/env.js:128-143): the mantissa is rounded
// half-up on the 13 dropped bits, and the rounded mantissa is OR-ed into the
// exponent field as the reference does.
uint16_t env_half(float v) {
  uint32_t x;
  std::memcpy(&x, &v, 4);
  const uint32_t s = (x >> 16) & 0x8000u;
  const int e = (int)((x >> 23) & 0xffu) - 112;
  uint32_t m = x & 0x7fffffu;
  if (e <= 0) {
    if (e < -10) return (uint16_t)s;
    m = (m | 0x800000u) >> (1 - e);
    return (uint16_t)(s | ((m + 0x1000u) >> 13));
  }
  if (e >= 0x1f) return (uint16_t)(s | 0x7c00u);
  return (uint16_t)(s | ((uint32_t)e << 10) | ((m + 0x1000u) >> 13));
}

namespace {

constexpr double kPiD = 3.14159265358979323846;

// faceDir (src/env.js:115-124): the direction through face texel (s, t) in [-1, 1].
void face_dir(int face, double s, double t, double d[3]) {
  switch (face) {
    case 0: d[0] = 1; d[1] = -t; d[2] = -s; break;
    case 1: d[0] = -1; d[1] = -t; d[2] = s; break;
    case 2: d[0] = s; d[1] = 1; d[2] = t; break;
    case 3: d[0] = s; d[1] = -1; d[2] = -t; break;
    case 4: d[0] = s; d[1] = -t; d[2] = 1; break;
    default: d[0] = -s; d[1] = -t; d[2] = -1; break;
  }
}

// sampleEquirect (src/env.js:94-113): bilinear sample of the panorama in direction
// d, wrapping in longitude and clamping in latitude.
void sample_equirect(const float* src, int w, int h, double dx, double dy, double dz, float out[3]) {
  const double len = std::sqrt(dx * dx + dy * dy + dz * dz);
  dx /= len;
  dy /= len;
  dz /= len;
  const double u = 0.5 + std::atan2(dx, dz) / (2 * kPiD);
  const double v = std::acos(std::min(1.0, std::max(-1.0, dy))) / kPiD;
  const double fx = u * w - 0.5, fy = v * h - 0.5;
  const double x0 = std::floor(fx), y0 = std::floor(fy);
  const double tx = fx - x0, ty = fy - y0;
  const long long ix = (long long)x0, iy = (long long)y0;
  auto at = [&](long long x, long long y, int c) -> double {
    x = ((x % w) + w) % w;
    y = std::min<long long>(h - 1, std::max<long long>(0, y));
    return src[(y * w + x) * 3 + c];
  };
  for (int c = 0; c < 3; c++) {
    const double a = at(ix, iy, c) * (1 - tx) + at(ix + 1, iy, c) * tx;
    const double b = at(ix, iy + 1, c) * (1 - tx) + at(ix + 1, iy + 1, c) * tx;
    out[c] = (float)(a * (1 - ty) + b * ty);
  }
}

}  // namespace

void build_env_cube(const float* rgb, int w, int h, int size, uint16_t* out) {
  const uint16_t one = env_half(1.0f);
  auto face_job = [&](int f) {
    double d[3];
    float c[3];
    for (int y = 0; y < size; y++) {
      const double t = 2 * (y + 0.5) / size - 1;
      for (int x = 0; x < size; x++) {
        const double s = 2 * (x + 0.5) / size - 1;
        face_dir(f, s, t, d);
        sample_equirect(rgb, w, h, d[0], d[1], d[2], c);
        uint16_t* o = out + (((size_t)f * size + y) * size + x) * 4;
        o[0] = env_half(c[0]);
        o[1] = env_half(c[1]);
        o[2] = env_half(c[2]);
        o[3] = one;
      }
    }
  };
  std::vector<std::thread> pool;
  for (int f = 0; f < 6; f++) pool.emplace_back(face_job, f);
  for (std::thread& t : pool) t.join();
}

}  // namespace p4a
