// use the register-resident passes of fast.cuh; every other supported length uses
// the per-warp Stockham passes of spectral.cu.  Rows dispatch on NX, columns on NY.
#include "internal.h"

#define FWIX_FAST_DECL(TAG)                                                                            \
  cudaError_t row_forward_##TAG(const SpecArgs& a, int pre, cudaStream_t s);                           \
  cudaError_t row_inverse_##TAG(const SpecArgs& a, int post, int pt, cudaStream_t s);                  \
  cudaError_t col_type_a_##TAG(const SpecArgs& a, int q, cudaStream_t s);                              \
  cudaError_t col_type_b_##TAG(const SpecArgs& a, int q, cudaStream_t s);                              \
  cudaError_t col_fft_##TAG(const SpecArgs& a, int inv, const float2* in, float2* out, int add, float sc, \
                            cudaStream_t s);

namespace fwix {
namespace fast {
FWIX_FAST_DECL(64)
FWIX_FAST_DECL(96)
FWIX_FAST_DECL(128)
FWIX_FAST_DECL(160)
FWIX_FAST_DECL(192)
FWIX_FAST_DECL(256)
FWIX_FAST_DECL(320)
FWIX_FAST_DECL(384)
FWIX_FAST_DECL(512)
FWIX_FAST_DECL(640)
}  // namespace fast

bool fast_length(int n) {
  switch (n) {
    case 64:
    case 96:
    case 128:
    case 160:
    case 192:
    case 256:
    case 320:
    case 384:
    case 512:
    case 640:
      return true;
    default:
      return false;
  }
}

cudaError_t row_forward(const SpecArgs& a, int pre, cudaStream_t s) {
  switch (a.d.NX) {
    case 64: return fast::row_forward_64(a, pre, s);
    case 96: return fast::row_forward_96(a, pre, s);
    case 128: return fast::row_forward_128(a, pre, s);
    case 160: return fast::row_forward_160(a, pre, s);
    case 192: return fast::row_forward_192(a, pre, s);
    case 256: return fast::row_forward_256(a, pre, s);
    case 320: return fast::row_forward_320(a, pre, s);
    case 384: return fast::row_forward_384(a, pre, s);
    case 512: return fast::row_forward_512(a, pre, s);
    case 640: return fast::row_forward_640(a, pre, s);
    default: return generic_row_forward(a, pre, s);
  }
}

cudaError_t row_inverse(const SpecArgs& a, int post, int post_taper, cudaStream_t s) {
  switch (a.d.NX) {
    case 64: return fast::row_inverse_64(a, post, post_taper, s);
    case 96: return fast::row_inverse_96(a, post, post_taper, s);
    case 128: return fast::row_inverse_128(a, post, post_taper, s);
    case 160: return fast::row_inverse_160(a, post, post_taper, s);
    case 192: return fast::row_inverse_192(a, post, post_taper, s);
    case 256: return fast::row_inverse_256(a, post, post_taper, s);
    case 320: return fast::row_inverse_320(a, post, post_taper, s);
    case 384: return fast::row_inverse_384(a, post, post_taper, s);
    case 512: return fast::row_inverse_512(a, post, post_taper, s);
    case 640: return fast::row_inverse_640(a, post, post_taper, s);
    default: return generic_row_inverse(a, post, post_taper, s);
  }
}

cudaError_t col_type_a(const SpecArgs& a, int qmode, cudaStream_t s) {
  switch (a.d.NY) {
    case 64: return fast::col_type_a_64(a, qmode, s);
    case 96: return fast::col_type_a_96(a, qmode, s);
    case 128: return fast::col_type_a_128(a, qmode, s);
    case 160: return fast::col_type_a_160(a, qmode, s);
    case 192: return fast::col_type_a_192(a, qmode, s);
    case 256: return fast::col_type_a_256(a, qmode, s);
    case 320: return fast::col_type_a_320(a, qmode, s);
    case 384: return fast::col_type_a_384(a, qmode, s);
    case 512: return fast::col_type_a_512(a, qmode, s);
    case 640: return fast::col_type_a_640(a, qmode, s);
    default: return generic_col_type_a(a, qmode, s);
  }
}

cudaError_t col_type_b(const SpecArgs& a, int qmode, cudaStream_t s) {
  switch (a.d.NY) {
    case 64: return fast::col_type_b_64(a, qmode, s);
    case 96: return fast::col_type_b_96(a, qmode, s);
    case 128: return fast::col_type_b_128(a, qmode, s);
    case 160: return fast::col_type_b_160(a, qmode, s);
    case 192: return fast::col_type_b_192(a, qmode, s);
    case 256: return fast::col_type_b_256(a, qmode, s);
    case 320: return fast::col_type_b_320(a, qmode, s);
    case 384: return fast::col_type_b_384(a, qmode, s);
    case 512: return fast::col_type_b_512(a, qmode, s);
    case 640: return fast::col_type_b_640(a, qmode, s);
    default: return generic_col_type_b(a, qmode, s);
  }
}

cudaError_t col_fft(const SpecArgs& a, int inverse, const float2* in, float2* out, int add, float scale,
                    cudaStream_t s) {
  switch (a.d.NY) {
    case 64: return fast::col_fft_64(a, inverse, in, out, add, scale, s);
    case 96: return fast::col_fft_96(a, inverse, in, out, add, scale, s);
    case 128: return fast::col_fft_128(a, inverse, in, out, add, scale, s);
    case 160: return fast::col_fft_160(a, inverse, in, out, add, scale, s);
    case 192: return fast::col_fft_192(a, inverse, in, out, add, scale, s);
    case 256: return fast::col_fft_256(a, inverse, in, out, add, scale, s);
    case 320: return fast::col_fft_320(a, inverse, in, out, add, scale, s);
    case 384: return fast::col_fft_384(a, inverse, in, out, add, scale, s);
    case 512: return fast::col_fft_512(a, inverse, in, out, add, scale, s);
    case 640: return fast::col_fft_640(a, inverse, in, out, add, scale, s);
    default: return generic_col_fft(a, inverse, in, out, add, scale, s);
  }
}

}  // namespace fwix
