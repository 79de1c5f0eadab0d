// kernels_hose.cu — the benchmark hose emitted on the device.
//
// The reference pours with pourStep (src/main.js:106-160): square k x k lattice
// layers with jitter, appended through Sim.appendFluid (src/sim.js:774-809) at
// index n with density rho0 and zero lambda / corr / normal / body / rest. The
// fixed-rate hose of the large workload is the same layered emitter; its jitter
// here comes from a counter-based generator keyed by (seed, emission, slot), so a
// layer is a pure function of its emission index and is written straight into the
// particle arrays by one kernel: no host staging, no copy, no host wait. The host
// restatement (particles4all_b200/configs.py Hose.emit) computes the same bits.
//
// Generator: Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC 2011): counter (emission lo, emission hi,
// slot, 0), key (seed, 0x5eed5eed), ten rounds with the published multipliers and
// Weyl increments. Output word a of the 4 gives axis a's uniform
// u = (word >> 8) * 2^-24 in [0, 1), exact in float; jitter = (2u - 1) * amp.
// Layer slot q sits at row iy = q / k, column iz = q % k:
//   x = nozzle.x + jx
//   y = (nozzle.y + (iy - c) * d) + jy,   z = (nozzle.z + (iz - c) * d) + jz,
// c = (k - 1) / 2, every operation one float32 rounding (no contraction).
#include <cuda_runtime.h>

#include "p4a_internal.h"
#include "p4a_math.cuh"

namespace p4a {

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

__global__ void __launch_bounds__(kBlock) k_hose_emit(HoseEmit H, float4* __restrict__ pos,
                                                      float4* __restrict__ vel, float4* __restrict__ pred,
                                                      float* __restrict__ density, float* __restrict__ lambda,
                                                      float4* __restrict__ corr, float4* __restrict__ normal,
                                                      uint4* __restrict__ body0, uint4* __restrict__ body1,
                                                      float4* __restrict__ rest0, float4* __restrict__ rest1) {
  const uint32_t q = blockIdx.x * kBlock + threadIdx.x;
  if (q >= H.count) return;
  const uint32_t i = H.first + q;
  uint32_t c[4] = {(uint32_t)H.emission, (uint32_t)(H.emission >> 32), q, 0u};
  philox4x32_10(c, H.seed, 0x5eed5eedu);
  float j[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const float u = (float)(c[a] >> 8) * 5.9604644775390625e-8f;  // 2^-24
    j[a] = (u * 2.0f - 1.0f) * H.jitter;
  }
  const float iy = (float)(q / H.k), iz = (float)(q % H.k);
  const float x = H.nozzle[0] + j[0];
  const float y = (H.nozzle[1] + (iy - H.centre) * H.spacing) + j[1];
  const float z = (H.nozzle[2] + (iz - H.centre) * H.spacing) + j[2];
  const float4 p = make_float4(x, y, z, 1.0f);
  pos[i] = p;
  pred[i] = p;
  vel[i] = make_float4(H.speed, 0.0f, 0.0f, 0.0f);
  density[i] = H.rho0;
  lambda[i] = 0.0f;
  corr[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  normal[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  body0[i] = make_uint4(0u, 0u, 0u, 0u);
  body1[i] = make_uint4(0u, 0u, 0u, 0u);
  rest0[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  rest1[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

void launch_hose_emit(const HoseEmit& H, const DevScene& d, int parity, int predParity, cudaStream_t st) {
  k_hose_emit<<<groups(H.count), kBlock, 0, st>>>(H, d.pos[parity], d.vel[parity], d.pred[predParity], d.density,
                                                   d.lambda, d.corr, d.normal, d.body[0], d.body[1], d.rest[0],
                                                   d.rest[1]);
}

}  // namespace p4a
