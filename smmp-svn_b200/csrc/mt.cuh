// MT19937 stream slots on the device (twister.f:64-177): the state words,
// the index mti and a queue of values already generated (kernels that draw
// ahead keep them there).  A slot is kMTWords words in shared or global
// memory; included by every translation unit that draws.
#pragma once
#include <cstdint>

#include "device.cuh"

namespace smmpb200 {
namespace {

__device__ void mt_seed(uint32_t* slot, uint32_t seed) {
  slot[0] = seed;
  for (int i = 1; i < 624; ++i) slot[i] = 69069u * slot[i - 1];
  slot[kMTIdx] = 624;
}
__device__ void mt_twist(uint32_t* mt) {
  const uint32_t MATA = 0x9908B0DFu, UM = 0x80000000u, LM = 0x7fffffffu;
  int kk = 0;
  uint32_t y;
  for (; kk < 624 - 397; ++kk) {
    y = (mt[kk] & UM) | (mt[kk + 1] & LM);
    mt[kk] = mt[kk + 397] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
  }
  for (; kk < 623; ++kk) {
    y = (mt[kk] & UM) | (mt[kk + 1] & LM);
    mt[kk] = mt[kk - 227] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
  }
  y = (mt[623] & UM) | (mt[0] & LM);
  mt[623] = mt[396] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
}
__device__ __forceinline__ double temper(uint32_t y) {
  y ^= (y >> 11);
  y ^= (y << 7) & 0x9D2C5680u;
  y ^= (y << 15) & 0xEFC60000u;
  y ^= (y >> 18);
  return __ddiv_rn((double)y, 4294967295.0);   // twister.f:172-176
}
// grnd() of the state words only (twister.f:104-177).
__device__ double mt_grnd(uint32_t* slot) {
  uint32_t mti = slot[kMTIdx];
  if (mti >= 624) {
    if (mti == 625) mt_seed(slot, 4357u);
    mt_twist(slot);
    mti = 0;
  }
  slot[kMTIdx] = mti + 1;
  return temper(slot[mti]);
}
__device__ __forceinline__ double* qbuf(uint32_t* slot) { return reinterpret_cast<double*>(slot + kQOff); }
// Next number of a stream slot: queued values first, then the state.
__device__ double stream_next(uint32_t* slot) {
  uint32_t h = slot[kQHead], t = slot[kQTail];
  if (h != t) {
    slot[kQHead] = h + 1;
    return qbuf(slot)[h & (kQueue - 1)];
  }
  return mt_grnd(slot);
}
}  // namespace
}  // namespace smmpb200
