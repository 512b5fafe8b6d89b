// Device building blocks: complex arithmetic and a per-warp mixed-radix Stockham
// FFT over one line held in shared memory.
//
// The Stockham autosort form used here (one pass per radix R, input read at
// j + r*n/R, output written at (j/Ns)*Ns*R + j%Ns + r*Ns, twiddle
// exp(-+2*pi*i*(j%Ns)*r/(Ns*R))) is the textbook formulation of Govindaraju et al.,
// "High performance discrete Fourier transforms on graphics processors" (SC'08).
// Each warp owns one line; passes ping-pong between two shared-memory lines and
// only __syncwarp() separates them.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define FWIX_MAX_PASS 12
#define FWIX_MAX_N 1024

struct Fft1D {
  int n;
  int npass;
  int radix[FWIX_MAX_PASS];
};

// Complex arithmetic.  On sm_100 the packed FP32 pair instructions
// (__fadd2_rn / __fmul2_rn / __ffma2_rn) do both components in one
// instruction; each component is rounded exactly as the scalar form would be.
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {  // (ax bx - ay by, ax by + ay bx)
  const float2 t = __fmul2_rn(make_float2(a.x, a.x), b);
  return __ffma2_rn(make_float2(-a.y, a.y), make_float2(b.y, b.x), t);
}
__device__ __forceinline__ float2 cmul_conj(float2 a, float2 b) {  // a * conj(b)
  const float2 t = __fmul2_rn(a, make_float2(b.x, b.x));
  return __ffma2_rn(make_float2(a.y, -a.x), make_float2(b.y, b.y), t);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
#else
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmul_conj(float2 a, float2 b) {  // a * conj(b)
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
#endif
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 rot90(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// Principal complex square root with the conventions of
// propagator/src/prop_kernels.cuh:89-102 (zero maps to zero, the imaginary part
// takes the sign of the input's imaginary part).  The reference forms both parts
// from sqrt((r -+ a)/2); here the smaller part comes from x |y| = |b| / 2, which
// gives the same value without the cancellation of r - a (or r + a) in float.
__device__ __forceinline__ float2 csqrt_ref(float2 z) {
  if (z.x == 0.0f && z.y == 0.0f) return make_float2(0.0f, 0.0f);
  const float r = hypotf(z.x, z.y);
  if (z.x >= 0.0f) {
    const float x = sqrtf(0.5f * (r + z.x));
    return make_float2(x, 0.5f * z.y / x);
  }
  const float ay = sqrtf(0.5f * (r - z.x));
  return make_float2(0.5f * fabsf(z.y) / ay, copysignf(ay, z.y));
}
__device__ __forceinline__ float2 cinv(float2 a) {
  float d = a.x * a.x + a.y * a.y;
  return make_float2(a.x / d, -a.y / d);
}
__device__ __forceinline__ float2 cdiv(float2 a, float2 b) {
  float d = b.x * b.x + b.y * b.y;
  return make_float2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}

// ---------------------------------------------------------------- radix kernels
template <int R, bool INV>
struct Dft;

template <bool INV>
struct Dft<2, INV> {
  static __device__ __forceinline__ void run(float2 (&v)[2]) {
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <bool INV>
struct Dft<4, INV> {
  static __device__ __forceinline__ void run(float2 (&v)[4]) {
    float2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
    float2 s13 = cadd(v[1], v[3]), d13 = rot90<INV>(csub(v[1], v[3]));
    v[0] = cadd(s02, s13);
    v[2] = csub(s02, s13);
    v[1] = cadd(d02, d13);
    v[3] = csub(d02, d13);
  }
};

template <bool INV>
struct Dft<8, INV> {
  static __device__ __forceinline__ void run(float2 (&v)[8]) {
    const float h = 0.70710678118654752440f;
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    Dft<4, INV>::run(e);
    Dft<4, INV>::run(o);
    // o[k] *= w8^k, w8 = exp(-+ i pi/4)
    float2 t1 = INV ? make_float2(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y))
                    : make_float2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
    float2 t2 = rot90<INV>(o[2]);
    float2 t3 = INV ? make_float2(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y))
                    : make_float2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], t1);
    v[5] = csub(e[1], t1);
    v[2] = cadd(e[2], t2);
    v[6] = csub(e[2], t2);
    v[3] = cadd(e[3], t3);
    v[7] = csub(e[3], t3);
  }
};

template <bool INV>
struct Dft<3, INV> {
  static __device__ __forceinline__ void run(float2 (&v)[3]) {
    const float s3 = 0.86602540378443864676f;
    float2 t = cadd(v[1], v[2]);
    float2 u = rot90<INV>(cscale(csub(v[1], v[2]), s3));  // -+ i s3 (v1 - v2)
    float2 m = make_float2(v[0].x - 0.5f * t.x, v[0].y - 0.5f * t.y);
    v[0] = cadd(v[0], t);
    v[1] = cadd(m, u);
    v[2] = csub(m, u);
  }
};

template <bool INV>
struct Dft<5, INV> {
  static __device__ __forceinline__ void run(float2 (&v)[5]) {
    const float c1 = 0.30901699437494742410f;   // cos(2 pi / 5)
    const float c2 = -0.80901699437494742410f;  // cos(4 pi / 5)
    const float s1 = 0.95105651629515357212f;   // sin(2 pi / 5)
    const float s2 = 0.58778525229247312917f;   // sin(4 pi / 5)
    float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    float2 u1 = csub(v[1], v[4]), u2 = csub(v[2], v[3]);
    float2 a1 = make_float2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    float2 a2 = make_float2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    float2 b1 = rot90<INV>(make_float2(s1 * u1.x + s2 * u2.x, s1 * u1.y + s2 * u2.y));
    float2 b2 = rot90<INV>(make_float2(s2 * u1.x - s1 * u2.x, s2 * u1.y - s1 * u2.y));
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = cadd(a1, b1);
    v[4] = csub(a1, b1);
    v[2] = cadd(a2, b2);
    v[3] = csub(a2, b2);
  }
};

// Radix 16 as 4 x 4: n = 4 n1 + n2, k = k1 + 4 k2; radix-4 transforms over n1,
// twiddles W16^(n2 k1), radix-4 transforms over n2.
template <bool INV>
__device__ __forceinline__ float2 tw16(float2 a, float c, float s) {  // a * (c -+ i s)
  return INV ? cmul(a, make_float2(c, s)) : cmul(a, make_float2(c, -s));
}
template <bool INV>
struct Dft<16, INV> {
  static __device__ __forceinline__ void run(float2 (&v)[16]) {
    const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;
    const float h = 0.70710678118654752440f;
    float2 y[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
      float2 u[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
      Dft<4, INV>::run(u);
#pragma unroll
      for (int k1 = 0; k1 < 4; ++k1) y[n2][k1] = u[k1];
    }
    y[1][1] = tw16<INV>(y[1][1], c1, s1);   // W^1
    y[1][2] = tw16<INV>(y[1][2], h, h);     // W^2
    y[1][3] = tw16<INV>(y[1][3], s1, c1);   // W^3
    y[2][1] = tw16<INV>(y[2][1], h, h);     // W^2
    y[2][2] = rot90<INV>(y[2][2]);          // W^4
    y[2][3] = tw16<INV>(y[2][3], -h, h);    // W^6
    y[3][1] = tw16<INV>(y[3][1], s1, c1);   // W^3
    y[3][2] = tw16<INV>(y[3][2], -h, h);    // W^6
    y[3][3] = tw16<INV>(y[3][3], -c1, -s1); // W^9
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      float2 u[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
      Dft<4, INV>::run(u);
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = u[k2];
    }
  }
};

// Radix 4 N2 for N2 = 3, 5 by the prime-factor (Good-Thomas) mapping, which needs
// no twiddles between the two transforms: input n = (N2 n1 + 4 n2) mod N, radix-N2
// transforms over n2, radix-4 transforms over n1, output k = k1 (mod 4),
// k = k2 (mod N2), i.e. k = (A k1 + B k2) mod N with A = N2 (N2^-1 mod 4) and
// B = 4 (4^-1 mod N2): (9, 4) for 12, (5, 16) for 20.
template <int N2, int A, int B, bool INV>
__device__ __forceinline__ void dft_pfa4(float2 (&v)[4 * N2]) {
  constexpr int N = 4 * N2;
  float2 y[4][N2];
#pragma unroll
  for (int n1 = 0; n1 < 4; ++n1) {
    float2 u[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) u[n2] = v[(N2 * n1 + 4 * n2) % N];
    Dft<N2, INV>::run(u);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) y[n1][k2] = u[k2];
  }
#pragma unroll
  for (int k2 = 0; k2 < N2; ++k2) {
    float2 u[4] = {y[0][k2], y[1][k2], y[2][k2], y[3][k2]};
    Dft<4, INV>::run(u);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) v[(A * k1 + B * k2) % N] = u[k1];
  }
}
template <bool INV>
struct Dft<12, INV> {
  static __device__ __forceinline__ void run(float2 (&v)[12]) { dft_pfa4<3, 9, 4, INV>(v); }
};
template <bool INV>
struct Dft<20, INV> {
  static __device__ __forceinline__ void run(float2 (&v)[20]) { dft_pfa4<5, 5, 16, INV>(v); }
};

// Radix 7 from the symmetric pair form y_m = v0 + sum_k cos(2 pi k m/7) t_k -+
// i sum_k sin(2 pi k m/7) u_k with t_k = v_k + v_{7-k}, u_k = v_k - v_{7-k}.
template <bool INV>
struct Dft<7, INV> {
  static __device__ __forceinline__ void run(float2 (&v)[7]) {
    const float C[7] = {1.0f, 0.62348980185873353053f, -0.22252093395631440429f, -0.90096886790241912624f,
                        -0.90096886790241912624f, -0.22252093395631440429f, 0.62348980185873353053f};
    const float S[7] = {0.0f, 0.78183148246802980871f, 0.97492791218182360702f, 0.43388373911755812048f,
                        -0.43388373911755812048f, -0.97492791218182360702f, -0.78183148246802980871f};
    float2 t[4], u[4];
#pragma unroll
    for (int k = 1; k <= 3; ++k) {
      t[k] = cadd(v[k], v[7 - k]);
      u[k] = csub(v[k], v[7 - k]);
    }
    const float2 v0 = v[0];
    v[0] = cadd(v0, cadd(t[1], cadd(t[2], t[3])));
#pragma unroll
    for (int m = 1; m <= 3; ++m) {
      float2 a = v0, b = make_float2(0.f, 0.f);
#pragma unroll
      for (int k = 1; k <= 3; ++k) {
        const int j = (k * m) % 7;
        a = make_float2(a.x + C[j] * t[k].x, a.y + C[j] * t[k].y);
        b = make_float2(b.x + S[j] * u[k].x, b.y + S[j] * u[k].y);
      }
      const float2 rb = rot90<INV>(b);
      v[m] = cadd(a, rb);
      v[7 - m] = csub(a, rb);
    }
  }
};

// One Stockham pass of radix R over a line of n elements at element stride `st`.
template <int R, bool INV>
__device__ __forceinline__ void stockham_pass(const float2* __restrict__ src, float2* __restrict__ dst,
                                              int st, int n, int Ns, const float2* __restrict__ tw,
                                              int lane) {
  const int nb = n / R;
  const int tstep = n / (Ns * R);
  for (int j = lane; j < nb; j += 32) {
    const int q = j / Ns;
    const int k = j - q * Ns;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[(j + r * nb) * st];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 w = tw[k * r * tstep];
        v[r] = INV ? cmul_conj(v[r], w) : cmul(v[r], w);
      }
    }
    Dft<R, INV>::run(v);
    const int base = q * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[(base + r * Ns) * st] = v[r];
  }
}

// Full FFT of one line by one warp.  `a` holds the input; `b` is scratch of the
// same shape.  Returns the buffer holding the result (a or b by pass parity).
// tw[m] = exp(-2 pi i m / n) in shared memory.
template <bool INV>
__device__ __forceinline__ float2* warp_fft(float2* a, float2* b, int st, const Fft1D& p,
                                            const float2* __restrict__ tw, int lane) {
  float2* src = a;
  float2* dst = b;
  int Ns = 1;
  for (int i = 0; i < p.npass; ++i) {
    const int R = p.radix[i];
    switch (R) {
      case 8: stockham_pass<8, INV>(src, dst, st, p.n, Ns, tw, lane); break;
      case 4: stockham_pass<4, INV>(src, dst, st, p.n, Ns, tw, lane); break;
      case 2: stockham_pass<2, INV>(src, dst, st, p.n, Ns, tw, lane); break;
      case 3: stockham_pass<3, INV>(src, dst, st, p.n, Ns, tw, lane); break;
      case 5: stockham_pass<5, INV>(src, dst, st, p.n, Ns, tw, lane); break;
      default: stockham_pass<7, INV>(src, dst, st, p.n, Ns, tw, lane); break;
    }
    __syncwarp();
    float2* t = src;
    src = dst;
    dst = t;
    Ns *= R;
  }
  return src;
}
