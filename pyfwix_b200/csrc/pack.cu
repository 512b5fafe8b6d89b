// Lossy fixed-rate store of wavefields: blocks of 16 consecutive floats (8
// complex samples) keep one shared exponent byte and 16 signed 8-bit mantissas,
// 17 bytes for 64 (8.5 bits per value, 3.76 x smaller).  The reference keeps its
// background wavefields ZFP-compressed at a fixed rate of 8 bits per value
// (propagator/src/WavefieldPool.cpp:23, :52-60); this is this library's own
// format with the same purpose and a comparable rate, not ZFP's bit stream.
//
// Block rule, for the block's largest magnitude m = f 2^E (f in [0.5, 1)):
// q = rint(v 2^(7 - E)) clamped to [-127, 127], exponent byte E + 128; blocks with
// m below 2^-100 are stored as zeros with exponent byte 0.  Decoding is
// v = q 2^(E - 7), so |v - v'| <= 2^(E - 8) <= m 2^-7.  The scaling is by powers
// of two and rint rounds to nearest even, so the packed bytes are exact functions
// of the input (the oracle restates the rule in numpy and the tests compare bytes).
// The exponent byte covers blocks up to m < 2^127; larger (and non-finite) values
// are outside the format (a NaN block reads back as zeros).
//
// Layout of one packed wavefield of n floats, nblk = ceil(n / 16): nblk x 16
// mantissa bytes, then nblk exponent bytes, the whole rounded up to 256 bytes.
#include <cstdint>

#include "internal.h"

namespace fwix {
namespace {

constexpr int kBlk = 16;  // floats per block

// kVec: 16-byte vector loads / stores (both buffers 16-byte aligned), else
// single floats and 4-byte mantissa words (buffers 8- and 4-byte aligned).
template <bool kVec>
__global__ void __launch_bounds__(256) k_pack_rate8(long long n, const float* __restrict__ in,
                                                    uint32_t* __restrict__ mant, uint8_t* __restrict__ exps) {
  const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nblk = (n + kBlk - 1) / kBlk;
  if (b >= nblk) return;
  float v[kBlk];
  const long long f0 = b * kBlk;
  if (kVec && f0 + kBlk <= n) {
    const float4* src = reinterpret_cast<const float4*>(in + f0);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float4 t = src[k];
      v[4 * k] = t.x;
      v[4 * k + 1] = t.y;
      v[4 * k + 2] = t.z;
      v[4 * k + 3] = t.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < kBlk; ++k) v[k] = f0 + k < n ? in[f0 + k] : 0.f;
  }
  float m = 0.f;
#pragma unroll
  for (int k = 0; k < kBlk; ++k) m = fmaxf(m, fabsf(v[k]));
  int E = 0;
  frexpf(m, &E);
  const bool zero = !(m >= 0x1p-100f);
  const float scale = zero ? 0.f : ldexpf(1.f, 7 - E);
  uint32_t w[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    uint32_t word = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float q = rintf(v[4 * k + j] * scale);
      q = fminf(fmaxf(q, -127.f), 127.f);
      word |= ((uint32_t)(uint8_t)(int8_t)(int)q) << (8 * j);
    }
    w[k] = word;
  }
  if (kVec) {
    reinterpret_cast<int4*>(mant)[b] = make_int4((int)w[0], (int)w[1], (int)w[2], (int)w[3]);
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) mant[4 * b + k] = w[k];
  }
  exps[b] = zero ? (uint8_t)0 : (uint8_t)min(max(E + 128, 1), 255);
}

template <bool kVec>
__global__ void __launch_bounds__(256) k_unpack_rate8(long long n, const uint32_t* __restrict__ mant,
                                                      const uint8_t* __restrict__ exps, float* __restrict__ out) {
  const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nblk = (n + kBlk - 1) / kBlk;
  if (b >= nblk) return;
  uint32_t w[4];
  if (kVec) {
    const int4 q4 = reinterpret_cast<const int4*>(mant)[b];
    w[0] = (uint32_t)q4.x;
    w[1] = (uint32_t)q4.y;
    w[2] = (uint32_t)q4.z;
    w[3] = (uint32_t)q4.w;
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) w[k] = mant[4 * b + k];
  }
  const uint8_t e = exps[b];
  const float scale = e == 0 ? 0.f : ldexpf(1.f, (int)e - 128 - 7);
  float v[kBlk];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int j = 0; j < 4; ++j) v[4 * k + j] = (float)(int8_t)(uint8_t)(w[k] >> (8 * j)) * scale;
  const long long f0 = b * kBlk;
  if (kVec && f0 + kBlk <= n) {
    float4* dst = reinterpret_cast<float4*>(out + f0);
#pragma unroll
    for (int k = 0; k < 4; ++k) dst[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
  } else {
#pragma unroll
    for (int k = 0; k < kBlk; ++k)
      if (f0 + k < n) out[f0 + k] = v[k];
  }
}

unsigned blocks_for(long long nblk) { return (unsigned)((nblk + 255) / 256); }

}  // namespace

size_t packed_rate8_bytes(long long nfloat) {
  const long long nblk = (nfloat + kBlk - 1) / kBlk;
  const size_t b = (size_t)nblk * (kBlk + 1);
  return (b + 255) / 256 * 256;
}

static bool aligned16(const void* a, const void* b) { return (((uintptr_t)a | (uintptr_t)b) & 15) == 0; }

cudaError_t launch_pack_rate8(long long nfloat, const float* in, void* packed, cudaStream_t s) {
  const long long nblk = (nfloat + kBlk - 1) / kBlk;
  if (nblk == 0) return cudaSuccess;
  if ((((uintptr_t)in) & 3) || (((uintptr_t)packed) & 3)) return cudaErrorMisalignedAddress;
  uint32_t* mant = reinterpret_cast<uint32_t*>(packed);
  uint8_t* exps = reinterpret_cast<uint8_t*>(packed) + nblk * kBlk;
  if (aligned16(in, packed))
    k_pack_rate8<true><<<blocks_for(nblk), 256, 0, s>>>(nfloat, in, mant, exps);
  else
    k_pack_rate8<false><<<blocks_for(nblk), 256, 0, s>>>(nfloat, in, mant, exps);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_unpack_rate8(long long nfloat, const void* packed, float* out, cudaStream_t s) {
  const long long nblk = (nfloat + kBlk - 1) / kBlk;
  if (nblk == 0) return cudaSuccess;
  if ((((uintptr_t)out) & 3) || (((uintptr_t)packed) & 3)) return cudaErrorMisalignedAddress;
  const uint32_t* mant = reinterpret_cast<const uint32_t*>(packed);
  const uint8_t* exps = reinterpret_cast<const uint8_t*>(packed) + nblk * kBlk;
  if (aligned16(out, packed))
    k_unpack_rate8<true><<<blocks_for(nblk), 256, 0, s>>>(nfloat, mant, exps, out);
  else
    k_unpack_rate8<false><<<blocks_for(nblk), 256, 0, s>>>(nfloat, mant, exps, out);
  count_launch();
  return cudaGetLastError();
}

}  // namespace fwix
