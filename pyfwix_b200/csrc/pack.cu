// Lossy fixed-rate store of wavefields: blocks of 16 consecutive floats (8
// complex samples) keep one shared exponent byte and 16 signed 8-bit mantissas,
// 17 bytes for 64 (8.5 bits per value, 3.76 x smaller), or, at rate 16, 16-bit
// mantissas, 33 bytes for 64 (16.5 bits per value, 1.94 x smaller).  The reference keeps its
// background wavefields ZFP-compressed at a fixed rate of 8 bits per value
// (propagator/src/WavefieldPool.cpp:23, :52-60); this is this library's own
// format with the same purpose and a comparable rate, not ZFP's bit stream.
//
// Block rule, for the block's largest magnitude m = f 2^E (f in [0.5, 1)):
// q = rint(v 2^(B - E)) clamped to [-(2^B - 1), 2^B - 1] with B = 7 (rate 8) or 15
// (rate 16), exponent byte E + 128; blocks with m below 2^-100 are stored as
// zeros with exponent byte 0.  Decoding is v = q 2^(E - B), so
// |v - v'| <= m 2^-B.  The scaling is by powers
// of two and rint rounds to nearest even, so the packed bytes are exact functions
// of the input (the oracle restates the rule in numpy and the tests compare bytes).
// The exponent byte covers blocks up to m < 2^127; larger (and non-finite) values
// are outside the format (a NaN block reads back as zeros).
//
// Layout of one packed wavefield of n floats, nblk = ceil(n / 16): nblk x 16 (or 32)
// mantissa bytes, then nblk exponent bytes, the whole rounded up to 256 bytes.
#include <cstdint>

#include "internal.h"

namespace fwix {
namespace {

constexpr int kBlk = 16;  // floats per block

// BITS = 8 or 16 mantissa bits: a block's mantissas are 4 or 8 32-bit words.
// kVec: 16-byte vector loads / stores (both buffers 16-byte aligned), else
// single floats and 4-byte mantissa words (buffers 4-byte aligned).
template <int BITS, bool kVec>
__global__ void __launch_bounds__(256) k_pack(long long n, const float* __restrict__ in,
                                              uint32_t* __restrict__ mant, uint8_t* __restrict__ exps) {
  constexpr int W = kBlk * BITS / 32;         // mantissa words per block
  constexpr int PER = 32 / BITS;              // mantissas per word
  constexpr int B = BITS - 1;                 // magnitude bits
  constexpr float LIM = (float)((1 << B) - 1);
  const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nblk = (n + kBlk - 1) / kBlk;
  {
    // The bytes after the exponents, up to the 256-byte rounded size, are
    // written as zeros, so that a packed field's bytes depend on its values
    // alone (fewer than 256 of them; the grid has at least 256 threads).
    const long long used = nblk * (kBlk * BITS / 8 + 1);
    if (b < (used + 255) / 256 * 256 - used) exps[nblk + b] = 0;
  }
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
  const float scale = zero ? 0.f : ldexpf(1.f, B - E);
  uint32_t w[W];
#pragma unroll
  for (int k = 0; k < W; ++k) {
    uint32_t word = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      float q = rintf(v[PER * k + j] * scale);
      q = fminf(fmaxf(q, -LIM), LIM);
      const uint32_t bitsq = BITS == 8 ? (uint32_t)(uint8_t)(int8_t)(int)q : (uint32_t)(uint16_t)(int16_t)(int)q;
      word |= bitsq << (BITS * j);
    }
    w[k] = word;
  }
  if (kVec) {
    int4* dst = reinterpret_cast<int4*>(mant) + (long long)b * (W / 4);
#pragma unroll
    for (int k = 0; k < W / 4; ++k)
      dst[k] = make_int4((int)w[4 * k], (int)w[4 * k + 1], (int)w[4 * k + 2], (int)w[4 * k + 3]);
  } else {
#pragma unroll
    for (int k = 0; k < W; ++k) mant[(long long)W * b + k] = w[k];
  }
  exps[b] = zero ? (uint8_t)0 : (uint8_t)min(max(E + 128, 1), 255);
}

template <int BITS, bool kVec>
__global__ void __launch_bounds__(256) k_unpack(long long n, const uint32_t* __restrict__ mant,
                                                const uint8_t* __restrict__ exps, float* __restrict__ out) {
  constexpr int W = kBlk * BITS / 32;
  constexpr int PER = 32 / BITS;
  constexpr int B = BITS - 1;
  const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nblk = (n + kBlk - 1) / kBlk;
  if (b >= nblk) return;
  uint32_t w[W];
  if (kVec) {
    const int4* src = reinterpret_cast<const int4*>(mant) + (long long)b * (W / 4);
#pragma unroll
    for (int k = 0; k < W / 4; ++k) {
      const int4 q4 = src[k];
      w[4 * k] = (uint32_t)q4.x;
      w[4 * k + 1] = (uint32_t)q4.y;
      w[4 * k + 2] = (uint32_t)q4.z;
      w[4 * k + 3] = (uint32_t)q4.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < W; ++k) w[k] = mant[(long long)W * b + k];
  }
  const uint8_t e = exps[b];
  const float scale = e == 0 ? 0.f : ldexpf(1.f, (int)e - 128 - B);
  float v[kBlk];
#pragma unroll
  for (int k = 0; k < W; ++k)
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      const uint32_t raw = w[k] >> (BITS * j);
      const float q = BITS == 8 ? (float)(int8_t)(uint8_t)raw : (float)(int16_t)(uint16_t)raw;
      v[PER * k + j] = q * scale;
    }
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

bool aligned16(const void* a, const void* b) { return (((uintptr_t)a | (uintptr_t)b) & 15) == 0; }

}  // namespace

size_t packed_bytes(long long nfloat, int bits) {
  const long long nblk = (nfloat + kBlk - 1) / kBlk;
  const size_t b = (size_t)nblk * (kBlk * bits / 8 + 1);
  return (b + 255) / 256 * 256;
}

size_t packed_rate8_bytes(long long nfloat) { return packed_bytes(nfloat, 8); }

cudaError_t launch_pack(int bits, long long nfloat, const float* in, void* packed, cudaStream_t s) {
  const long long nblk = (nfloat + kBlk - 1) / kBlk;
  if (bits != 8 && bits != 16) return cudaErrorInvalidValue;
  if (nblk == 0) return cudaSuccess;
  if ((((uintptr_t)in) & 3) || (((uintptr_t)packed) & 3)) return cudaErrorMisalignedAddress;
  uint32_t* mant = reinterpret_cast<uint32_t*>(packed);
  uint8_t* exps = reinterpret_cast<uint8_t*>(packed) + nblk * kBlk * bits / 8;
  const bool vec = aligned16(in, packed);
  if (bits == 8) {
    if (vec) k_pack<8, true><<<blocks_for(nblk), 256, 0, s>>>(nfloat, in, mant, exps);
    else k_pack<8, false><<<blocks_for(nblk), 256, 0, s>>>(nfloat, in, mant, exps);
  } else {
    if (vec) k_pack<16, true><<<blocks_for(nblk), 256, 0, s>>>(nfloat, in, mant, exps);
    else k_pack<16, false><<<blocks_for(nblk), 256, 0, s>>>(nfloat, in, mant, exps);
  }
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_unpack(int bits, long long nfloat, const void* packed, float* out, cudaStream_t s) {
  const long long nblk = (nfloat + kBlk - 1) / kBlk;
  if (bits != 8 && bits != 16) return cudaErrorInvalidValue;
  if (nblk == 0) return cudaSuccess;
  if ((((uintptr_t)out) & 3) || (((uintptr_t)packed) & 3)) return cudaErrorMisalignedAddress;
  const uint32_t* mant = reinterpret_cast<const uint32_t*>(packed);
  const uint8_t* exps = reinterpret_cast<const uint8_t*>(packed) + nblk * kBlk * bits / 8;
  const bool vec = aligned16(out, packed);
  if (bits == 8) {
    if (vec) k_unpack<8, true><<<blocks_for(nblk), 256, 0, s>>>(nfloat, mant, exps, out);
    else k_unpack<8, false><<<blocks_for(nblk), 256, 0, s>>>(nfloat, mant, exps, out);
  } else {
    if (vec) k_unpack<16, true><<<blocks_for(nblk), 256, 0, s>>>(nfloat, mant, exps, out);
    else k_unpack<16, false><<<blocks_for(nblk), 256, 0, s>>>(nfloat, mant, exps, out);
  }
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_pack_rate8(long long nfloat, const float* in, void* packed, cudaStream_t s) {
  return launch_pack(8, nfloat, in, packed, s);
}

cudaError_t launch_unpack_rate8(long long nfloat, const void* packed, float* out, cudaStream_t s) {
  return launch_unpack(8, nfloat, packed, out, s);
}

}  // namespace fwix
