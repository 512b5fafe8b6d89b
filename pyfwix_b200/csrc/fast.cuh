// Register-resident row / column passes for line lengths with a compile-time plan.
//
// One group of T lanes (T = 8, 16 or 32; 32 / T groups per warp) owns one line of
// N = T * E samples and keeps E of them per lane in registers.  The line goes
// through the radix stages of its plan (mixed-radix Stockham, Govindaraju et al.,
// SC'08): each stage does E / R radix-R butterflies in registers and, except after
// the last one, exchanges the samples through the line's own shared-memory region,
// so stages are separated by __syncwarp() only.  Sample p of a line lives at
// swz(p) = p ^ ((p >> 3) & 15), which keeps every stage's stores and loads within
// about one wavefront per half-warp.  All index arithmetic except the lane's own
// index is compile-time.
//
// Layouts: before stage 0 (radix R0) lane t holds element e = b*R0 + r at position
// t + T*b + r*N/R0; after the last stage (radix Rk) at t + T*b + r*N/Rk.  The
// inverse runs the stages in reverse order, so its input layout is the forward
// output layout: a spectrum is multiplied and transformed back in registers.
//
// Row passes (lines along x) read and write HBM directly from registers (for a
// fixed element, consecutive lanes touch consecutive samples) and need no CTA
// barrier.  Column passes (lines along y) stage a tile of LX columns x NY rows
// through shared memory so that HBM is read and written in row segments.
#pragma once
#include <cstring>
#include <map>
#include <tuple>
#include <mutex>
#include <utility>

#include "ops.cuh"
#include "tma.cuh"

namespace fwix {
namespace fast {

template <int... Rs>
struct Radices {
  static constexpr int NS = sizeof...(Rs);
  __host__ __device__ static constexpr int get(int s) {
    constexpr int r[] = {Rs...};
    return r[s];
  }
};

// SW selects the sample placement of the line exchanges: 0 puts sample p at
// p ^ ((p >> 3) & 15), 1 at p + (p >> 4) (conflict-free for radix-16 stages on
// 16-lane lines); LINE_EXTRA is the room the second needs past N.
// Placement of each line exchange of a plan, one code per exchange: the forward
// transform's exchanges (after stages 0 .. NS-2) first, then the inverse's.  -1
// keeps the plan's default placement (xswz), 0 is p itself, any other code
// a | m << 4 | mask << 8 places sample p at p ^ (((p >> a) * m) & mask), which
// stays within the aligned block of mask + 1 samples; a plan may only use codes
// that permute 0 .. N-1 (with m = 1 every a does: bit i of the result is bit i
// of p plus bit i + a).  Chosen per exchange so that the stores of one stage and
// the loads of the next hit as few shared-memory banks twice as possible (the
// strides of an exchange depend on its stage).
template <int... Cs>
struct XSw {
  static constexpr int n = sizeof...(Cs);
  __host__ __device__ static constexpr int get(int i) {
    constexpr int c[] = {Cs..., -1};
    return c[i];
  }
};
using NoXSw = XSw<>;
constexpr int xs(int a, int m, int mask) { return a | m << 4 | mask << 8; }  // code of p ^ (((p >> a) * m) & mask)
// Whether every code of XS maps 0 .. N-1 onto itself one to one.
template <int N, class XS>
constexpr bool xsw_permutes() {
  for (int i = 0; i < XS::n; ++i) {
    const int c = XS::get(i);
    if (c <= 0) continue;
    bool seen[N] = {};
    for (int p = 0; p < N; ++p) {
      const int q = p ^ (((p >> (c & 15)) * ((c >> 4) & 15)) & (c >> 8));
      if (q < 0 || q >= N || seen[q]) return false;
      seen[q] = true;
    }
  }
  return true;
}

template <int N_, int E_, class RS, int SW_ = 0, class XS_ = NoXSw>
struct Plan {
  using XS = XS_;
  static constexpr int N = N_;
  static constexpr int E = E_;
  static constexpr int SW = SW_;
  static constexpr int LINE_EXTRA = SW_ == 1 ? N_ / 16 : 0;
  static constexpr int T = N_ / E_;    // lanes per line
  static constexpr int G = 32 / T;     // lines per warp
  static constexpr int NS = RS::NS;
  static_assert(T == 8 || T == 16 || T == 32, "a line takes 8, 16 or 32 lanes");
  static_assert(XS::n == 0 || XS::n == 2 * (NS - 1), "one exchange placement per exchange of each direction");
  static_assert(xsw_permutes<N_, XS_>(), "an exchange placement must permute the line");
  __host__ __device__ static constexpr int radix(int s) { return RS::get(s); }
};

constexpr int kWarps = 8;       // warps per CTA in every pass
constexpr int kMaxHatRefs = 32;  // smooth-step references the row passes stage in shared memory

template <class P, bool REV>
struct Order {
  __host__ __device__ static constexpr int radix(int s) { return REV ? P::radix(P::NS - 1 - s) : P::radix(s); }
  __host__ __device__ static constexpr int span(int s) { return s == 0 ? 1 : span(s - 1) * radix(s - 1); }
};

__device__ __forceinline__ int swz(int p) { return p ^ ((p >> 3) & 15); }
template <class P>
__device__ __forceinline__ int xswz(int p) {  // exchange placement of plan P
  return P::SW == 1 ? p + (p >> 4) : swz(p);
}
// Placement of exchange S of the forward (REV false) or inverse transform.
template <class P, bool REV, int S>
__device__ __forceinline__ int xch(int p) {
  constexpr int c = P::XS::n ? P::XS::get((REV ? P::NS - 1 : 0) + S) : -1;
  if constexpr (c < 0) {
    return xswz<P>(p);
  } else if constexpr (c == 0) {
    return p;
  } else {
    return p ^ (((p >> (c & 15)) * ((c >> 4) & 15)) & (c >> 8));
  }
}

// Twiddles in shared memory, one table per stage and order: stage S (span Ns,
// radix R) reads W_N^(k r N / (Ns R)) for k = j mod Ns and r = 1..R-1 at
// (r - 1) Ns + k, so the lanes of a warp read consecutive entries (no bank
// conflicts).  The forward-order tables come first, then the reversed-order
// (inverse transform) ones; together they hold about 2 N values.
template <class P, bool REV>
struct TwLayout {
  using O = Order<P, REV>;
  __host__ __device__ static constexpr int count(int s) { return O::span(s) > 1 ? (O::radix(s) - 1) * O::span(s) : 0; }
  __host__ __device__ static constexpr int offset(int s) { return s == 0 ? 0 : offset(s - 1) + count(s - 1); }
  __host__ __device__ static constexpr int total() { return offset(P::NS); }
};
template <class P>
constexpr int tw_size() {
  return TwLayout<P, false>::total() + TwLayout<P, true>::total();
}

template <class P, bool REV, int S>
__device__ __forceinline__ void fill_stage_tw(float2* dst, const float2* __restrict__ tw) {
  if constexpr (S < P::NS) {
    using O = Order<P, REV>;
    constexpr int Ns = O::span(S), R = O::radix(S), cnt = TwLayout<P, REV>::count(S);
    constexpr int off = TwLayout<P, REV>::offset(S), tstep = P::N / (Ns * R);
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
      const int r = i / Ns + 1, k = i - (r - 1) * Ns;
      dst[off + i] = tw[k * r * tstep];
    }
    fill_stage_tw<P, REV, S + 1>(dst, tw);
  }
}
// Fills both orders' tables from the plain table tw[m] = exp(-2 pi i m / N).
template <class P>
__device__ __forceinline__ void load_stage_tw(float2* dst, const float2* __restrict__ tw) {
  fill_stage_tw<P, false, 0>(dst, tw);
  fill_stage_tw<P, true, 0>(dst + TwLayout<P, false>::total(), tw);
}

template <class P, int R>
__device__ __forceinline__ int lpos(int t, int e) {
  return t + P::T * (e / R) + (e % R) * (P::N / R);
}
template <class P>
__device__ __forceinline__ int pos_first(int t, int e) {  // input of the forward transform
  return lpos<P, P::radix(0)>(t, e);
}
template <class P>
__device__ __forceinline__ int pos_last(int t, int e) {  // output of the forward transform
  return lpos<P, P::radix(P::NS - 1)>(t, e);
}

template <class P, bool REV, bool INV, int S>
__device__ __forceinline__ void stages(float2 (&v)[P::E], int t, const float2* __restrict__ tw, float2* line) {
  using O = Order<P, REV>;
  constexpr int R = O::radix(S);
  constexpr int Ns = O::span(S);
  constexpr int B = P::E / R;
#pragma unroll
  for (int b = 0; b < B; ++b) {
    float2 u[R];
#pragma unroll
    for (int r = 0; r < R; ++r) u[r] = v[b * R + r];
    if constexpr (Ns > 1) {
      const int j = t + P::T * b;
      const int k = j % Ns;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const float2 w = tw[TwLayout<P, REV>::offset(S) + (r - 1) * Ns + k];
        u[r] = INV ? cmul_conj(u[r], w) : cmul(u[r], w);
      }
    }
    Dft<R, INV>::run(u);
#pragma unroll
    for (int r = 0; r < R; ++r) v[b * R + r] = u[r];
  }
  if constexpr (S + 1 < P::NS) {
    constexpr int R2 = O::radix(S + 1);
    __syncwarp();
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const int j = t + P::T * b;
      const int base = (j / Ns) * Ns * R + (j % Ns);
#pragma unroll
      for (int r = 0; r < R; ++r) line[xch<P, REV, S>(base + r * Ns)] = v[b * R + r];
    }
    __syncwarp();
#pragma unroll
    for (int e = 0; e < P::E; ++e) v[e] = line[xch<P, REV, S>(lpos<P, R2>(t, e))];
    stages<P, REV, INV, S + 1>(v, t, tw, line);
  }
}

template <class P>
__device__ __forceinline__ void fft_fwd(float2 (&v)[P::E], int t, const float2* tw, float2* line) {
  stages<P, false, false, 0>(v, t, tw, line);
}
template <class P>
__device__ __forceinline__ void fft_inv(float2 (&v)[P::E], int t, const float2* tw, float2* line) {
  stages<P, true, true, 0>(v, t, tw + TwLayout<P, false>::total(), line);
}

// Asynchronous 8-byte global -> shared copy (zero-filled when !valid).
__device__ __forceinline__ void cp_async8(float2* dst, const float2* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 8 : 0));
}
// Asynchronous 16-byte global -> shared copy through L2 (both addresses 16-byte aligned).
__device__ __forceinline__ void cp_async16(float2* dst, const float2* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
// Hint that the 128-byte line at p is read soon: it moves into L2 without a
// register waiting on it.
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p)); }
// Prefetches into L2 the input rows of the CTA pf_ctas launch positions after
// this one (row passes: CTA = nchunk row blocks of each launch-local slice);
// base points at the rows of launch-local slice 0 when local, else of slice 0.
template <int N, int ROWS>
__device__ __forceinline__ void prefetch_next_ctas(const SpecArgs& a, const float2* base, bool local, int nchunk) {
  const long long f = (long long)blockIdx.x + a.pf_ctas;
  if (a.pf_ctas <= 0 || f >= gridDim.x || !base) return;
  const long long bl = f / nchunk;
  const int y0 = (int)(f - bl * nchunk) * ROWS;
  const int rows = min(ROWS, a.d.NY - y0);
  const long long row0 = ((local ? bl : a.b0 + bl) * a.d.NY + y0) * N;
  for (int i = threadIdx.x; i < rows * (N / 16); i += blockDim.x) prefetch_l2(base + row0 + 16LL * i);
}
// Prefetches into L2 the rows y0 .. y0 + rows - 1 (rows < ny of the unpadded
// window, x < nx) of slice b of each field laid out like SpecArgs::in, one line
// per thread and step, for the reflection terms a row pass reads (RF).
template <class P>
__device__ __forceinline__ void prefetch_refl_rows(const SpecArgs& a, long long b, int y0, int rows) {
  const int nr = min(rows, a.d.ny - y0);
  const int lines = (a.d.nx * 8 + 127) / 128;  // lines of one row's window
  const float2* fs[2] = {a.rf_f1, a.rf_f2};
  for (int f = 0; f < 2; ++f) {
    if (!fs[f]) continue;
    for (int i = threadIdx.x; i < nr * lines; i += blockDim.x) {
      const int r = i / lines, l = i - r * lines;
      prefetch_l2(fs[f] + (b * a.d.NY + y0 + r) * P::N + l * 16);
    }
  }
}
// The same for the whole padded rows y0 .. y0 + rows - 1 (< NY) of slice b of
// one field laid out like SpecArgs::in (the direct term of W_ONE_DIRECT).
template <class P>
__device__ __forceinline__ void prefetch_full_rows(const SpecArgs& a, const float2* f, long long b, int y0,
                                                   int rows) {
  const int nr = min(rows, a.d.NY - y0);
  for (int i = threadIdx.x; i < nr * (P::N / 16); i += blockDim.x)
    prefetch_l2(f + (b * a.d.NY + y0) * P::N + 16LL * i);
}
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Labels of a lane's samples, four to a 32-bit word (fewer registers than a byte
// array, which the compiler keeps one per register).
template <int E>
struct Labels {
  uint32_t w[(E + 3) / 4];
  __device__ __forceinline__ void set(int e, uint32_t v) {
    w[e / 4] = (e % 4 == 0 ? 0u : w[e / 4]) | ((v & 0xffu) << (8 * (e % 4)));
  }
  __device__ __forceinline__ int get(int e) const { return (int)((w[e / 4] >> (8 * (e % 4))) & 0xffu); }
};

// ---------------------------------------------------------------- row passes (NX = P::N)

template <class P>
struct RowGeo {
  // shared-memory stride between lines
  static constexpr int LINE = P::N + (P::LINE_EXTRA > (P::T < 32 ? 8 : 0) ? P::LINE_EXTRA : (P::T < 32 ? 8 : 0));
  static constexpr int ROWS = kWarps * P::G;                // rows per CTA
  // after the twiddles: the smooth step's references and inverse spans (kMaxHatRefs each)
  static size_t smem() { return ((size_t)kWarps * P::G * LINE + tw_size<P>() + kMaxHatRefs) * sizeof(float2); }
  // Born-weight rows of the CTA staged after the above (16-byte aligned): nterm
  // tables x ROWS rows x N samples, when they fit in 160 KB
  __host__ __device__ static constexpr size_t scat_offset() {
    return ((size_t)kWarps * P::G * LINE + tw_size<P>() + kMaxHatRefs + 1) & ~(size_t)1;
  }
  __host__ __device__ static bool scat_stage(int nterm) { return (size_t)nterm * ROWS * P::N * 8 <= 160 * 1024; }
  static size_t smem_scat(int nterm) { return (scat_offset() + (size_t)nterm * ROWS * P::N) * sizeof(float2); }
};

// Smooth-step references of the row passes, staged in shared memory once per CTA:
// ref[0 .. n) and inv[j] = 1 / (ref[j+1] - ref[j]).  With more references than
// kMaxHatRefs the passes fall back to the per-term weights of row_weight.
template <class P>
__device__ __forceinline__ void stage_hat_refs(const SpecArgs& a, float* ref, float* inv) {
  const int n = a.sm_n;
  if ((int)threadIdx.x < n) {
    const int i = threadIdx.x;
    ref[i] = a.sm_ref[i];
    inv[i] = i + 1 < n ? 1.f / (a.sm_ref[i + 1] - a.sm_ref[i]) : 0.f;
  }
}
// Fractional reference index g of slowness s: the hat weights are 1 - (g - j) on
// reference j and g - j on j + 1, j = min(floor g, n - 2); g = 0 and g = n - 1 are
// the clamped ends (weight 1 on the end reference, derivative 0).  Same
// bracketing as hat_weight.
__device__ __forceinline__ float hat_index(const float* ref, const float* inv, int n, float s) {
  if (n == 1 || s <= ref[0]) return 0.f;
  if (s >= ref[n - 1]) return (float)(n - 1);
  int j = 0;
  while (j < n - 2 && s >= ref[j + 1]) ++j;
  return (float)j + (s - ref[j]) * inv[j];
}
__device__ __forceinline__ unsigned hat_index_support(int n, float g) {
  if (n == 1 || g <= 0.f) return 1u;
  if (g >= (float)(n - 1)) return 1u << (n - 1);
  return 3u << min((int)g, n - 2);
}
// Hat weight (x) and its slowness derivative (y) of reference t at index g.
__device__ __forceinline__ float2 hat_at(const float* inv, int n, int t, float g) {
  if (n == 1 || g <= 0.f) return make_float2(t == 0 ? 1.f : 0.f, 0.f);
  if (g >= (float)(n - 1)) return make_float2(t == n - 1 ? 1.f : 0.f, 0.f);
  const int j = min((int)g, n - 2);
  const float u = g - (float)j;
  if (t == j) return make_float2(1.f - u, -inv[j]);
  if (t == j + 1) return make_float2(u, inv[j]);
  return make_float2(0.f, 0.f);
}
// Reference part of the smooth weight from the hat: w C (W_SMOOTH), w conj(C)
// (W_SMOOTH_CONJ), (w' - i w dz w) C (W_SMOOTH_DERIV).
template <int W>
__device__ __forceinline__ float2 hat_ref_weight(float2 h, float wdz, float2 C) {
  if (W == W_SMOOTH) return cscale(C, h.x);
  if (W == W_SMOOTH_CONJ) return cscale(cconj(C), h.x);
  return cmul(make_float2(h.y, -wdz * h.x), C);
}

// Per-thread view of a row pass: which row, which lane of the line, its smem line.
template <class P>
struct RowCtx {
  int t;
  int y;
  bool live;
  long long bl, b;
  int iw;
  float2* line;
  float2* tw;
  __device__ RowCtx(const SpecArgs& a, float2* smem, int nchunk) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane / P::T;
    t = lane % P::T;
    tw = smem + (size_t)kWarps * P::G * RowGeo<P>::LINE;
    line = smem + (size_t)(warp * P::G + g) * RowGeo<P>::LINE;
    bl = blockIdx.x / nchunk;
    b = a.b0 + bl;
    y = (int)(blockIdx.x - bl * nchunk) * RowGeo<P>::ROWS + warp * P::G + g;
    live = y < a.d.NY;
    iw = (int)(b % a.d.nw);
  }
};

// Resident CTAs per SM the forward row pass's registers are held to: the
// multi-term passes of 12- and 16-sample lanes at two (the scattering adjoint's,
// with one term's weights and no labels, at three), the rest unhinted.
// Compile-time occupancy knobs (defaults as measured best): resident CTAs of the
// multi-term forward and inverse row passes and of the multi-input and the
// single-input column pass with 16-sample lanes, and whether the multi-term
// inverse row pass prefetches the next term's row.
#ifndef FWIX_ROW_MULTI_MINB
#define FWIX_ROW_MULTI_MINB 2
#endif
#ifndef FWIX_ROWINV_PREFETCH
#define FWIX_ROWINV_PREFETCH 1
#endif
#ifndef FWIX_COLB_MINB16
#define FWIX_COLB_MINB16 2
#endif
#ifndef FWIX_COLA_MINB16
#define FWIX_COLA_MINB16 3
#endif
template <class P, int PRE>
constexpr int row_fwd_min_blocks() {
  if (PRE == W_SCAT_CONJ && P::E == 16) return 3;
  return multi_term(PRE) && (P::E == 16 || P::E == 12) ? FWIX_ROW_MULTI_MINB : 0;
}

// t1[term] = F_x(pre_term * in) for each term.  RF: the input is in + the
// reflection term of SpecArgs::rf_at 1 (separate instances, so that the passes
// without it keep their registers).
template <class P, int PRE, bool RF = false>
__global__ void __launch_bounds__(kWarps * 32, row_fwd_min_blocks<P, PRE>()) k_row_fwd(const SpecArgs a, int nchunk) {
  extern __shared__ float2 smem[];
  RowCtx<P> c(a, smem, nchunk);
  prefetch_next_ctas<P::N, RowGeo<P>::ROWS>(a, a.in, false, nchunk);
  if constexpr (RF) prefetch_refl_rows<P>(a, c.b, (int)(blockIdx.x - c.bl * nchunk) * RowGeo<P>::ROWS, RowGeo<P>::ROWS);
  // Born weights (W_SCAT_CONJ) from the per-depth table: the CTA's rows of every
  // transformed term's table copied into shared memory (cp.async) while the input
  // rows load, instead of one L2 read per sample and term in each lane.
  constexpr bool kScatC = PRE == W_SCAT_CONJ;
  const int nterm_s = kScatC ? a.nterm : 0;
  const bool scat_smem = kScatC && a.scat_tab && RowGeo<P>::scat_stage(nterm_s);
  float2* wt = smem + RowGeo<P>::scat_offset();
  const int y0 = (int)(blockIdx.x - c.bl * nchunk) * RowGeo<P>::ROWS;
  if (scat_smem) {
    const int rows = min(RowGeo<P>::ROWS, a.d.NY - y0);
    const int per = rows * (P::N / 2);
    for (int i = threadIdx.x; i < nterm_s * per; i += blockDim.x) {
      const int t = i / per, r = (i - t * per) / (P::N / 2), q = i - t * per - r * (P::N / 2);
      cp_async16(wt + ((size_t)t * RowGeo<P>::ROWS + r) * P::N + 2 * q,
                 a.scat_tab + ((long long)(t + a.term0) * a.d.NY + y0 + r) * P::N + 2 * q);
    }
    cp_async_commit();
  }
  load_stage_tw<P>(c.tw, a.twx);
  if (PRE == W_SMOOTH_CONJ && a.sm_n <= kMaxHatRefs)
    stage_hat_refs<P>(a, reinterpret_cast<float*>(c.tw + tw_size<P>()),
                      reinterpret_cast<float*>(c.tw + tw_size<P>()) + kMaxHatRefs);
  __syncthreads();
  float2 raw[P::E];
  const long long roff = (c.b * a.d.NY + (c.live ? c.y : 0)) * P::N;
  const float2* src = a.in + roff;
#pragma unroll
  for (int e = 0; e < P::E; ++e) raw[e] = c.live ? src[pos_first<P>(c.t, e)] : make_float2(0.f, 0.f);
  if (a.in2 && c.live) {
    const float2* src2 = a.in2 + roff;
#pragma unroll
    for (int e = 0; e < P::E; ++e) raw[e] = cadd(raw[e], src2[pos_first<P>(c.t, e)]);
  }
  if constexpr (RF) {
    if (c.live && c.y < a.d.ny) {
#pragma unroll
      for (int e = 0; e < P::E; ++e) {
        const int x = pos_first<P>(c.t, e);
        if (x < a.d.nx) raw[e] = cadd(raw[e], refl_term(a, roff, c.y, x));
      }
    }
  }
  if constexpr (PRE == W_IC) {
    // the image values load beside the background's samples (one wait for
    // both) and weight them here; the term loop takes the products as they are
    float2 im[P::E];
    const bool rowin = c.live && c.y < a.d.ny;
    const float2* irow = a.image + (long long)c.iw * a.img_w + (long long)(rowin ? c.y : 0) * a.d.nx;
#pragma unroll
    for (int e = 0; e < P::E; ++e) {
      const int x = pos_first<P>(c.t, e);
      im[e] = rowin && x < a.d.nx ? irow[x] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int e = 0; e < P::E; ++e) raw[e] = cmul(raw[e], im[e]);
  }
  const int nterm = multi_term(PRE) ? a.nterm : 1;
  Labels<P::E> lab;
  if (PRE == W_MASK) {
    const uint8_t* lrow = a.lab + (long long)c.iw * a.lab_w + (long long)(c.live ? c.y : 0) * P::N;
#pragma unroll
    for (int e = 0; e < P::E; ++e) lab.set(e, c.live ? lrow[pos_first<P>(c.t, e)] : 255u);
  }
  // smooth weights (references staged in shared memory): each cell's fractional
  // reference index and the cell part conj(B(s)) of every reference's weight,
  // once per cell; terms that no sample of the warp's rows supports are zero rows
  constexpr bool kSmooth = PRE == W_SMOOTH_CONJ;
  unsigned used = 0xffffffffu;
  float g[kSmooth ? P::E : 1];
  const float* href = reinterpret_cast<const float*>(c.tw + tw_size<P>());
  const float* hinv = href + kMaxHatRefs;
  const bool hat_smem = kSmooth && a.sm_n <= kMaxHatRefs;
  if (hat_smem) {
    const float* srow = a.sm_s + (long long)(c.live ? c.y : 0) * P::N;
    unsigned mine = 0;
#pragma unroll
    for (int e = 0; e < P::E; ++e) {
      const float sv = c.live ? srow[pos_first<P>(c.t, e)] : 0.f;
      g[e] = hat_index(href, hinv, a.sm_n, sv);
      if (c.live) {
        mine |= hat_index_support(a.sm_n, g[e]);
        raw[e] = cmul_conj(raw[e], smooth_cell_phase(a, c.iw, sv));
      }
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) mine |= __shfl_xor_sync(0xffffffffu, mine, o);
    used = mine;
  }
  if (scat_smem) {  // the weight rows have landed (the input rows are in registers)
    cp_async_wait<0>();
    __syncthreads();
  }
  for (int term = 0; term < nterm; ++term) {
    float2 v[P::E];
    if (!((used >> (term & 31)) & 1u)) {
      if (c.live) {
        float2* dst = a.t1 + (long long)term * a.tstride + (c.bl * a.d.NY + c.y) * P::N;
#pragma unroll
        for (int e = 0; e < P::E; ++e) dst[pos_last<P>(c.t, e)] = make_float2(0.f, 0.f);
      }
      continue;
    }
    if (hat_smem) {
      const float2 C = smooth_ref_phase(a, c.iw, term);
      const float wdz = a.w[c.iw] * a.dz;
#pragma unroll
      for (int e = 0; e < P::E; ++e)
        v[e] = c.live ? cmul(raw[e], hat_ref_weight<PRE>(hat_at(hinv, a.sm_n, term, g[e]), wdz, C))
                      : make_float2(0.f, 0.f);
    } else if (kScatC && scat_smem) {
      const float f = 0.5f * a.w[c.iw] * a.dz * a.coef[term + a.term0];
      const float2* wrow = wt + ((size_t)term * RowGeo<P>::ROWS + (c.y - y0)) * P::N;
#pragma unroll
      for (int e = 0; e < P::E; ++e)
        v[e] = c.live ? cmul_conj(raw[e], rot90<false>(cscale(wrow[pos_first<P>(c.t, e)], f))) : make_float2(0.f, 0.f);
    } else {
#pragma unroll
      for (int e = 0; e < P::E; ++e) {
        if (PRE == W_MASK)
          v[e] = lab.get(e) == term ? raw[e] : make_float2(0.f, 0.f);
        else if (PRE == W_IC)
          v[e] = c.live ? raw[e] : make_float2(0.f, 0.f);  // weighted at the load
        else
          v[e] = c.live ? row_weight<PRE>(a, term, c.iw, c.y, pos_first<P>(c.t, e), raw[e]) : make_float2(0.f, 0.f);
      }
    }
    fft_fwd<P>(v, c.t, c.tw, c.line);
    if (c.live) {
      float2* dst = a.t1 + (long long)term * a.tstride + (c.bl * a.d.NY + c.y) * P::N;
#pragma unroll
      for (int e = 0; e < P::E; ++e) dst[pos_last<P>(c.t, e)] = v[e];
    }
  }
}

// out (+)= post * sum_term W_term * F_x^-1(t2[term]); the next term's row is
// prefetched while the current one is transformed, and with labels the terms
// that no sample of the warp's rows selects are skipped.  W_SMOOTH_PAIR sums each
// transformed term twice, with the smooth weights into out and with their
// slowness derivatives into out2.  RF (W_ONE, W_MASK): the output gains the
// reflection terms of SpecArgs::rf_at 2 (separate instances, as in the forward
// row pass).
template <class P, int POST, bool RF = false>
__global__ void __launch_bounds__(kWarps * 32, multi_term(POST) && (P::E == 16 || P::E == 12) ? FWIX_ROW_MULTI_MINB
                                                                                              : (RF && POST == W_ONE ? 4 : 0))
    k_row_inv(const SpecArgs a, int nchunk, int post_taper) {
  extern __shared__ float2 smem[];
  RowCtx<P> c(a, smem, nchunk);
  prefetch_next_ctas<P::N, RowGeo<P>::ROWS>(a, a.t2, true, nchunk);  // the first term of a later CTA
  // the reflection fields (the direct term's field) are read in the epilogue:
  // their rows head for L2 now
  if constexpr (RF) prefetch_refl_rows<P>(a, c.b, (int)(blockIdx.x - c.bl * nchunk) * RowGeo<P>::ROWS, RowGeo<P>::ROWS);
  if constexpr (POST == W_ONE_DIRECT)
    if (a.direct)
      prefetch_full_rows<P>(a, a.direct, c.b, (int)(blockIdx.x - c.bl * nchunk) * RowGeo<P>::ROWS, RowGeo<P>::ROWS);
  // Born weights from the per-depth table: the CTA's rows of every term's table
  // are copied into shared memory (cp.async, 16 bytes a thread and instruction)
  // while the first term loads and transforms, and read from there after each
  // transform instead of from L2 behind it.
  // (Staging the scattering adjoint's zeroth term conj(W_0) d the same way,
  // W_0 and d rows, measured slower: 34 -> 40 us per 64 slices at 256, its
  // 64 KB of shared memory halving the resident CTAs of that light pass.)
  constexpr bool kScat = POST == W_SCAT;
  const int nterm = multi_term(POST) ? a.nterm : 1;
  const bool scat_smem = kScat && a.scat_tab && RowGeo<P>::scat_stage(nterm);
  float2* wt = smem + RowGeo<P>::scat_offset();
  const int y0 = (int)(blockIdx.x - c.bl * nchunk) * RowGeo<P>::ROWS;
  if (scat_smem) {
    const int rows = min(RowGeo<P>::ROWS, a.d.NY - y0);
    const int per = rows * (P::N / 2);  // 16-byte chunks of one term's rows
    for (int i = threadIdx.x; i < nterm * per; i += blockDim.x) {
      const int t = i / per, r = (i - t * per) / (P::N / 2), q = i - t * per - r * (P::N / 2);
      cp_async16(wt + ((size_t)t * RowGeo<P>::ROWS + r) * P::N + 2 * q,
                 a.scat_tab + ((long long)(t + a.term0) * a.d.NY + y0 + r) * P::N + 2 * q);
    }
    cp_async_commit();
  }
  bool wt_ready = false;
  load_stage_tw<P>(c.tw, a.twx);
  constexpr bool kPair = POST == W_SMOOTH_PAIR;
  constexpr bool kSmooth = POST == W_SMOOTH || POST == W_SMOOTH_DERIV || kPair;
  const bool hat_smem = kSmooth && a.sm_n <= kMaxHatRefs;
  const float* href = reinterpret_cast<const float*>(c.tw + tw_size<P>());
  const float* hinv = href + kMaxHatRefs;
  if (hat_smem) stage_hat_refs<P>(a, const_cast<float*>(href), const_cast<float*>(hinv));
  __syncthreads();
  float g[kSmooth ? P::E : 1];
  float2 acc[P::E];
  float2 acc2[kPair ? P::E : 1];
#pragma unroll
  for (int e = 0; e < P::E; ++e) acc[e] = make_float2(0.f, 0.f);
  if constexpr (kPair) {
#pragma unroll
    for (int e = 0; e < P::E; ++e) acc2[e] = make_float2(0.f, 0.f);
  }
  Labels<P::E> lab;
  unsigned used = 0xffffffffu;
  if (POST == W_MASK) {
    const uint8_t* lrow = a.lab + (long long)c.iw * a.lab_w + (long long)(c.live ? c.y : 0) * P::N;
    unsigned mine = 0;
#pragma unroll
    for (int e = 0; e < P::E; ++e) {
      const uint32_t l = c.live ? lrow[pos_first<P>(c.t, e)] : 255u;
      lab.set(e, l);
      if (l < 32) mine |= 1u << l;
    }
    // the warp steps through the union of its lines' terms so that it stays converged
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) mine |= __shfl_xor_sync(0xffffffffu, mine, o);
    used = nterm > 32 ? 0xffffffffu : mine;
  } else if (hat_smem) {
    unsigned mine = 0;
    const float* srow = a.sm_s + (long long)(c.live ? c.y : 0) * P::N;
#pragma unroll
    for (int e = 0; e < P::E; ++e) {
      g[e] = hat_index(href, hinv, a.sm_n, c.live ? srow[pos_first<P>(c.t, e)] : 0.f);
      if (c.live) mine |= hat_index_support(a.sm_n, g[e]);
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) mine |= __shfl_xor_sync(0xffffffffu, mine, o);
    used = mine;
  }
  auto next_term = [&](int from) {
    int k = from;
    while (k < nterm && k < 32 && !((used >> k) & 1u)) ++k;
    return k;
  };
  const long long roff = (c.bl * a.d.NY + (c.live ? c.y : 0)) * P::N;
  int term = next_term(0);
  // the next term's row is prefetched, except where the paired sums of 16-sample
  // lanes leave no registers for it (two accumulators, the term and the hat indices)
  constexpr bool kPrefetch = FWIX_ROWINV_PREFETCH && !(kPair && P::E >= 16);
  float2 pre[kPrefetch ? P::E : 1];
  if (kPrefetch && term < nterm) {
    const float2* src = a.t2 + (long long)term * a.tstride + roff;
#pragma unroll
    for (int e = 0; e < P::E; ++e) pre[e] = c.live ? src[pos_last<P>(c.t, e)] : make_float2(0.f, 0.f);
  }
  while (term < nterm) {
    float2 v[P::E];
    if constexpr (kPrefetch) {
#pragma unroll
      for (int e = 0; e < P::E; ++e) v[e] = pre[e];
    } else {
      const float2* src = a.t2 + (long long)term * a.tstride + roff;
#pragma unroll
      for (int e = 0; e < P::E; ++e) v[e] = c.live ? src[pos_last<P>(c.t, e)] : make_float2(0.f, 0.f);
    }
    const int nxt = next_term(term + 1);
    if (kPrefetch && nxt < nterm) {
      const float2* src = a.t2 + (long long)nxt * a.tstride + roff;
#pragma unroll
      for (int e = 0; e < P::E; ++e) pre[e] = c.live ? src[pos_last<P>(c.t, e)] : make_float2(0.f, 0.f);
    }
    fft_inv<P>(v, c.t, c.tw, c.line);
    if (hat_smem) {
      // reference part of the weights here, the cell part B(s) once after the sum
      const float2 C = smooth_ref_phase(a, c.iw, term);
      const float wdz = a.w[c.iw] * a.dz;
#pragma unroll
      for (int e = 0; e < P::E; ++e) {
        if (!c.live) continue;
        const float2 h = hat_at(hinv, a.sm_n, term, g[e]);
        if constexpr (kPair) {
          acc[e] = cadd(acc[e], cmul(v[e], hat_ref_weight<W_SMOOTH>(h, wdz, C)));
          acc2[e] = cadd(acc2[e], cmul(v[e], hat_ref_weight<W_SMOOTH_DERIV>(h, wdz, C)));
        } else {
          acc[e] = cadd(acc[e], cmul(v[e], hat_ref_weight<POST>(h, wdz, C)));
        }
      }
    } else if (kScat && scat_smem) {
      if (!wt_ready) {  // every warp reaches this after its first transform (no term is skipped)
        cp_async_wait<0>();
        __syncthreads();
        wt_ready = true;
      }
      const float f = 0.5f * a.w[c.iw] * a.dz * a.coef[term + a.term0];
      const float2* wrow = wt + ((size_t)term * RowGeo<P>::ROWS + (c.y - y0)) * P::N;
#pragma unroll
      for (int e = 0; e < P::E; ++e)
        if (c.live) acc[e] = cadd(acc[e], cmul(v[e], rot90<false>(cscale(wrow[pos_first<P>(c.t, e)], f))));
    } else {
#pragma unroll
      for (int e = 0; e < P::E; ++e) {
        if (POST == W_MASK) {
          if (lab.get(e) == term) acc[e] = v[e];
        } else if (c.live) {
          if constexpr (kPair) {
            acc[e] = cadd(acc[e], row_weight<W_SMOOTH>(a, term, c.iw, c.y, pos_first<P>(c.t, e), v[e]));
            acc2[e] = cadd(acc2[e], row_weight<W_SMOOTH_DERIV>(a, term, c.iw, c.y, pos_first<P>(c.t, e), v[e]));
          } else {
            acc[e] = cadd(acc[e], row_weight<POST>(a, term, c.iw, c.y, pos_first<P>(c.t, e), v[e]));
          }
        }
      }
    }
    term = nxt;
  }
  if (!c.live) return;
  float2* dst = a.out + (c.b * a.d.NY + c.y) * P::N;
  float2* dst2 = kPair ? a.out2 + (c.b * a.d.NY + c.y) * P::N : nullptr;
  const float ty = post_taper ? a.tapy[c.y] : 1.f;
  const float* srow_out = kSmooth ? a.sm_s + (long long)c.y * P::N : nullptr;
#pragma unroll
  for (int e = 0; e < P::E; ++e) {
    const int x = pos_first<P>(c.t, e);
    float2 v = acc[e];
    float2 cell = make_float2(1.f, 0.f);
    if (hat_smem) {
      cell = smooth_cell_phase(a, c.iw, srow_out[x]);
      v = cmul(v, cell);
    }
    if constexpr (POST == W_ONE_DIRECT) v = cadd(v, scat_direct(a, c.b, c.iw, c.y, x));
    if (post_taper) v = cscale(v, a.tapx[x] * ty);
    if (a.add) v = cadd(dst[x], v);
    // (Loading these terms before the transforms, as the start of the sum, held
    // their registers through the transforms: 39 -> 60 us per 64 slices at 256.)
    if constexpr (RF) {
      if (c.y < a.d.ny && x < a.d.nx) v = cadd(v, refl_term(a, (c.b * a.d.NY + c.y) * P::N, c.y, x));
    }
    dst[x] = v;
    if (a.ic_img && c.y < a.d.ny && x < a.d.nx) {
      // a warp's lanes hold consecutive x for each e: coalesced reductions
      const float2 bg = a.ic_bg[(c.b * a.d.NY + c.y) * P::N + x];
      atomicAdd(a.ic_img + (long long)c.y * a.d.nx + x, bg.x * v.x + bg.y * v.y);
    }
    if constexpr (kPair) {
      float2 u = hat_smem ? cmul(acc2[e], cell) : acc2[e];
      if (post_taper) u = cscale(u, a.tapx[x] * ty);
      if (a.add) u = cadd(dst2[x], u);
      dst2[x] = u;
    }
  }
}

// ---------------------------------------------------------------- column passes (NY = P::N)

template <class P>
struct ColGeo {
  static constexpr int LX = kWarps * P::G;  // columns per CTA
  // Tile stride between columns: with 8 columns a warp's tile copy covers 4
  // rows x 8 columns, conflict-free for a stride of 2 (mod 16) samples; with 16
  // or 32 columns an odd stride is, and 5 also suits the line exchanges.
  static constexpr int LINE = P::N + (LX == 8 ? 2 : 5);
  static size_t smem() { return ((size_t)LX * LINE + tw_size<P>()) * sizeof(float2); }
  // Resident CTAs per SM the register allocation is held to: four for plans of
  // at most 8 samples per lane (64 registers; the few spills stay in L1 and the
  // extra warps hide more latency than they cost), else what fits.
  static constexpr int kMinBlocks = P::E <= 8 ? 4 : P::E <= 16 ? FWIX_COLB_MINB16 : 1;
  // k_col_a holds one spectrum and one term in registers (k_col_b a running sum
  // as well): with 16 samples per lane it fits three CTAs per SM
  static constexpr int kMinBlocksA = P::E <= 8 ? 4 : P::E <= 12 ? 2 : P::E <= 16 ? FWIX_COLA_MINB16 : 1;
  static size_t smem2() { return ((size_t)2 * LX * LINE + tw_size<P>()) * sizeof(float2); }  // tile, tw, tile
};

template <class P>
struct ColCtx {
  int t, col, x, x0;
  long long b;
  int iw;
  float2* tile;
  float2* line;
  float2* tw;
  __device__ ColCtx(const SpecArgs& a, float2* smem, int nxt) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane / P::T;
    t = lane % P::T;
    col = warp * P::G + g;
    tile = smem;
    line = smem + (size_t)col * ColGeo<P>::LINE;
    tw = smem + (size_t)ColGeo<P>::LX * ColGeo<P>::LINE;
    b = blockIdx.x / nxt;
    x0 = (int)(blockIdx.x - b * nxt) * ColGeo<P>::LX;
    x = x0 + col;
    iw = (int)((a.b0 + b) % a.d.nw);
  }
};

// Coalesced copy of the CTA's columns of slice-local b between HBM and the tile.
template <class P>
__device__ __forceinline__ void cols_to_tile(float2* tile, const float2* __restrict__ g, const SpecArgs& a,
                                             long long b, int x0) {
  constexpr int LX = ColGeo<P>::LX, NT = kWarps * 32;
  static_assert((LX * P::N) % NT == 0, "tile is a whole number of CTA sweeps");
  const int cc = threadIdx.x % LX, x = x0 + cc;
  if (x >= a.d.NX) return;
  const float2* src = g + b * a.d.slice + x;
#pragma unroll 4
  for (int k = 0; k < LX * P::N / NT; ++k) {
    const int y = (int)(threadIdx.x + k * NT) / LX;
    tile[cc * ColGeo<P>::LINE + swz(y)] = src[(long long)y * a.d.NX];
  }
}
template <class P>
__device__ __forceinline__ void tile_to_cols(const float2* tile, float2* g, const SpecArgs& a, long long b, int x0,
                                             int add, float scale) {
  constexpr int LX = ColGeo<P>::LX, NT = kWarps * 32;
  const int cc = threadIdx.x % LX, x = x0 + cc;
  if (x >= a.d.NX) return;
  float2* dst = g + b * a.d.slice + x;
#pragma unroll 4
  for (int k = 0; k < LX * P::N / NT; ++k) {
    const int y = (int)(threadIdx.x + k * NT) / LX;
    float2 v = tile[cc * ColGeo<P>::LINE + swz(y)];
    if (scale != 1.f) v = cscale(v, scale);
    float2* q = dst + (long long)y * a.d.NX;
    if (add) v = cadd(*q, v);
    *q = v;
  }
}

// Column multipliers of term t for this lane's spectrum samples (forward-output
// layout), from the phase table when one is bound.
template <class P, int QM>
__device__ __forceinline__ void col_factors(const SpecArgs& a, int t, int iw, int x, int lane_t, float2 (&q)[P::E]) {
  if ((QM == Q_PS_FWD || QM == Q_PS_ADJ) && a.ptab) {
    const QCol qc = qcol<QM>(a, t, iw, x);
#pragma unroll
    for (int e = 0; e < P::E; ++e) q[e] = qcol_get(a, qc, pos_last<P>(lane_t, e));
  } else {
#pragma unroll
    for (int e = 0; e < P::E; ++e) q[e] = qmult<QM>(a, t, iw, x, pos_last<P>(lane_t, e));
  }
}

// t2[term] = F_y^-1(Q_term * F_y(t1[0])); the spectrum stays in registers.
template <class P, int QM>
__global__ void __launch_bounds__(kWarps * 32, ColGeo<P>::kMinBlocksA) k_col_a(const SpecArgs a, int nxt) {
  extern __shared__ float2 smem[];
  ColCtx<P> c(a, smem, nxt);
  load_stage_tw<P>(c.tw, a.twy);
  cols_to_tile<P>(c.tile, a.t1, a, c.b, c.x0);
  __syncthreads();
  // The zeroth Born order's filter (|k| / w)^0 is the identity: its output is the
  // tile itself, scaled as the transform pair would (NY times the normalisation),
  // written before the transform overwrites the tile; the loop starts at order 1.
  int first = 0;
  if constexpr (QM == Q_KPOW) {
    if (a.term0 == 0 && a.nterm > 0) {
      tile_to_cols<P>(c.tile, a.t2, a, c.b, c.x0, 0, a.norm * (float)P::N);
      __syncthreads();
      first = 1;
    }
  }
  float2 psi[P::E];
#pragma unroll
  for (int e = 0; e < P::E; ++e) psi[e] = c.line[swz(pos_first<P>(c.t, e))];
  fft_fwd<P>(psi, c.t, c.tw, c.line);
  const int xq = c.x < a.d.NX ? c.x : 0;
  // Up to 12 samples per lane the next term's factors are fetched while the
  // current term is transformed; with 16 the spectrum, the term and the factors
  // do not fit the two-CTA register budget together, so each term's factors are
  // fetched as they are applied.
  constexpr bool kPrefetch = P::E <= 12;
  float2 q[kPrefetch ? P::E : 1];
  if constexpr (kPrefetch) col_factors<P, QM>(a, first, c.iw, xq, c.t, q);
  for (int term = first; term < a.nterm; ++term) {
    float2 v[P::E];
    if constexpr (kPrefetch) {
#pragma unroll
      for (int e = 0; e < P::E; ++e) v[e] = cmul(psi[e], q[e]);
      if (term + 1 < a.nterm) col_factors<P, QM>(a, term + 1, c.iw, xq, c.t, q);
    } else {
      col_factors<P, QM>(a, term, c.iw, xq, c.t, v);
#pragma unroll
      for (int e = 0; e < P::E; ++e) v[e] = cmul(psi[e], v[e]);
    }
    __syncthreads();  // the previous term's tile has been stored
    fft_inv<P>(v, c.t, c.tw, c.line);
    __syncwarp();
#pragma unroll
    for (int e = 0; e < P::E; ++e) c.line[swz(pos_first<P>(c.t, e))] = v[e];
    __syncthreads();
    tile_to_cols<P>(c.tile, a.t2 + (long long)term * a.tstride, a, c.b, c.x0, 0, 1.f);
  }
}

// Asynchronous copy of the CTA's columns of slice-local b into a tile.
template <class P>
__device__ __forceinline__ void cols_to_tile_async(float2* tile, const float2* __restrict__ g, const SpecArgs& a,
                                                   long long b, int x0) {
  constexpr int LX = ColGeo<P>::LX, NT = kWarps * 32;
  const int cc = threadIdx.x % LX, x = x0 + cc;
  const bool ok = x < a.d.NX;
  const float2* src = g + b * a.d.slice + (ok ? x : 0);
#pragma unroll 4
  for (int k = 0; k < LX * P::N / NT; ++k) {
    const int y = (int)(threadIdx.x + k * NT) / LX;
    cp_async8(tile + cc * ColGeo<P>::LINE + swz(y), src + (long long)y * a.d.NX, ok);
  }
  cp_async_commit();
}

// t2[0] = F_y^-1(sum_term Q_term * F_y(t1[term])).  Two tiles: the copy engine
// fills one with the next term while the warps transform the other.
template <class P, int QM>
__global__ void __launch_bounds__(kWarps * 32, ColGeo<P>::kMinBlocks) k_col_b(const SpecArgs a, int nxt) {
  extern __shared__ float2 smem[];
  ColCtx<P> c(a, smem, nxt);
  float2* tiles[2] = {c.tile, c.tw + tw_size<P>()};
  const long long lineoff = (long long)c.col * ColGeo<P>::LINE;
  load_stage_tw<P>(c.tw, a.twy);
  const int xq = c.x < a.d.NX ? c.x : 0;
  float2 acc[P::E];
#pragma unroll
  for (int e = 0; e < P::E; ++e) acc[e] = make_float2(0.f, 0.f);
  cols_to_tile_async<P>(tiles[0], a.t1, a, c.b, c.x0);
  for (int term = 0; term < a.nterm; ++term) {
    __syncthreads();  // every warp is done with the tile the next copy overwrites
    if (term + 1 < a.nterm) {
      cols_to_tile_async<P>(tiles[(term + 1) & 1], a.t1 + (long long)(term + 1) * a.tstride, a, c.b, c.x0);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    float2 q[P::E];
    col_factors<P, QM>(a, term, c.iw, xq, c.t, q);
    __syncthreads();  // this term's tile is complete
    float2* line = tiles[term & 1] + lineoff;
    float2 v[P::E];
#pragma unroll
    for (int e = 0; e < P::E; ++e) v[e] = line[swz(pos_first<P>(c.t, e))];
    fft_fwd<P>(v, c.t, c.tw, line);
#pragma unroll
    for (int e = 0; e < P::E; ++e) acc[e] = cadd(acc[e], cmul(v[e], q[e]));
  }
  __syncthreads();
  fft_inv<P>(acc, c.t, c.tw, c.line);
  __syncwarp();
#pragma unroll
  for (int e = 0; e < P::E; ++e) c.line[swz(pos_first<P>(c.t, e))] = acc[e];
  __syncthreads();
  tile_to_cols<P>(c.tile, a.t2, a, c.b, c.x0, 0, 1.f);
}

// t2[0] = F_y^-1(sum_term Q_term * F_y(t1[term])) with the tiles moved by TMA
// (plans of 16 columns per CTA, 128 bytes per tile row).  Each term's tile
// arrives in one of two row-major swizzled buffers while the previous term is
// transformed; once every lane holds its column in registers the buffer serves
// as the line-exchange scratch (lines of N samples, column-major); the result
// leaves through a swizzled staging tile and one TMA store per box.  A load
// that does not complete within the bounded wait counts in *a.err and the CTA
// leaves without writing.
template <class P>
struct ColTma {
  static constexpr int LX = ColGeo<P>::LX;
  static constexpr int TILE = P::N * LX;  // samples per tile
  static constexpr int NBOX = P::N <= 256 ? 1 : (P::N % 2 == 0 && P::N / 2 <= 256 ? 2 : 4);
  static constexpr int ROWS = P::N / NBOX;  // rows per box (<= 256)
  static_assert(ROWS * NBOX == P::N && ROWS <= 256, "a tile is a whole number of boxes of at most 256 rows");
  // two tiles, the twiddles, two mbarriers, and room to align the tiles to 1024
  // bytes; with the phase tiles (qt samples each: LX |kx| rows of the cached
  // quarter spectrum) two of those after the term tiles
  static size_t smem(size_t qt = 0) {
    return (size_t)(2 * TILE + 2 * qt) * sizeof(float2) + tw_size<P>() * sizeof(float2) + 16 + 1024;
  }
};

// The CTA's columns x0 .. x0 + LX - 1 read the phase factors of |kx| = min(x, NX - x):
// LX consecutive values from k0 (increasing for x0 < NX / 2, decreasing above; a
// tile never straddles NX / 2 when NX / 2 is a multiple of LX).  Row of column x.
template <class P>
__device__ __forceinline__ int qtile_k0(const SpecArgs& a, int x0) {
  constexpr int LX = ColGeo<P>::LX;
  return x0 < a.d.NX / 2 ? x0 : a.d.NX - x0 - (LX - 1);
}
__device__ __forceinline__ int qtile_row(const SpecArgs& a, int x, int k0, int lx) {
  return min(max(min(x, a.d.NX - x) - k0, 0), lx - 1);
}
// Whether the adjoint phase factor of reference t at frequency iw is conj(P)
// (qcol's rule: the reference keeps P where its b > 0 branch applies).
template <int QM>
__device__ __forceinline__ bool qflip(const SpecArgs& a, int t, int iw) {
  if (QM != Q_PS_ADJ) return false;
  const float2 sr = a.sref[t * a.d.nw + iw];
  return !(a.w2[iw] * (sr.y - a.eps * sr.x) > 0.f);
}

// kQT: the phase factors of each term come as a TMA tile with the term's column
// tile (the cached table of the phase shift modes); else col_factors loads them
// from global memory before the tile wait.
template <class P, int QM, bool kQT>
__global__ void __launch_bounds__(kWarps * 32, ColGeo<P>::kMinBlocks)
    k_col_b_tma(const SpecArgs a, int nxt, const __grid_constant__ CUtensorMap tin,
                const __grid_constant__ CUtensorMap tout, const __grid_constant__ CUtensorMap tq) {
  using C = ColTma<P>;
  static_assert(C::LX == 16 || C::LX == 8, "TMA column tiles are 16 or 8 columns (128- or 64-byte rows)");
  extern __shared__ unsigned char smem_raw[];
  float2* base = reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  float2* tiles[2] = {base, base + C::TILE};
  const int pny = a.ptab_ny;
  const int qt = kQT ? C::LX * pny : 0;  // samples per phase tile (pny even: 128-byte multiples)
  float2* qs[2] = {base + 2 * C::TILE, base + 2 * C::TILE + qt};
  float2* tw = base + 2 * C::TILE + 2 * qt;
  uint64_t* bar = reinterpret_cast<uint64_t*>(tw + tw_size<P>());
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane / P::T, t = lane % P::T, col = warp * P::G + g;
  const long long b = blockIdx.x / nxt;  // launch-local slice
  const int x0 = (int)(blockIdx.x - b * nxt) * C::LX;
  const int iw = (int)((a.b0 + b) % a.d.nw);
  const int x = x0 + col;
  const int xq = x < a.d.NX ? x : 0;
  const int zstride = (int)(a.tstride / a.d.slice);  // slices per term in t1
  const int k0 = qtile_k0<P>(a, x0);
  const int qrow = qtile_row(a, xq, k0, C::LX) * pny;
  if (threadIdx.x == 0) {
    tma::mbar_init(&bar[0], 1);
    tma::mbar_init(&bar[1], 1);
    tma::fence_mbar_init();
  }
  load_stage_tw<P>(tw, a.twy);
  __syncthreads();
  auto issue = [&](int term, int buf) {
    tma::mbar_expect_tx(&bar[buf], (unsigned)((C::TILE + qt) * sizeof(float2)));
#pragma unroll
    for (int k = 0; k < C::NBOX; ++k)
      tma::load_3d(tiles[buf] + k * C::ROWS * C::LX, &tin, x0, k * C::ROWS, term * zstride + (int)b, &bar[buf]);
    if constexpr (kQT) tma::load_3d(qs[buf], &tq, 0, k0, term * a.d.nw + iw, &bar[buf]);
  };
  if (threadIdx.x == 0) issue(0, 0);
  float2 acc[P::E];
#pragma unroll
  for (int e = 0; e < P::E; ++e) acc[e] = make_float2(0.f, 0.f);
  for (int term = 0; term < a.nterm; ++term) {
    const int buf = term & 1;
    if (threadIdx.x == 0 && term + 1 < a.nterm) issue(term + 1, buf ^ 1);
    float2 q[kQT ? 1 : P::E];
    if constexpr (!kQT) col_factors<P, QM>(a, term, iw, xq, t, q);
    const bool ok = tma::mbar_wait(&bar[buf], (unsigned)(term >> 1) & 1u);
    if (!__syncthreads_and(ok)) {
      if (threadIdx.x == 0) {
        atomicAdd(a.err, 1u);
        if (term + 1 < a.nterm) tma::mbar_wait(&bar[buf ^ 1], (unsigned)((term + 1) >> 1) & 1u);
      }
      return;
    }
    float2 v[P::E];
#pragma unroll
    for (int e = 0; e < P::E; ++e) v[e] = tiles[buf][tma::swz_tile<C::LX>(pos_first<P>(t, e), col)];
    __syncthreads();  // the tile is in registers: its buffer is free for the exchanges
    fft_fwd<P>(v, t, tw, tiles[buf] + col * P::N);
    if constexpr (kQT) {
      const float2* qr = qs[buf] + qrow;
      const bool flip = qflip<QM>(a, term, iw);
#pragma unroll
      for (int e = 0; e < P::E; ++e) {
        const int ky = pos_last<P>(t, e);
        const float2 f = qr[min(ky, P::N - ky)];
        acc[e] = cadd(acc[e], cmul(v[e], flip ? cconj(f) : f));
      }
    } else {
#pragma unroll
      for (int e = 0; e < P::E; ++e) acc[e] = cadd(acc[e], cmul(v[e], q[e]));
    }
    tma::fence_proxy_async();  // the exchanges and phase reads precede the next loads into this buffer
    __syncthreads();
  }
  // no load is pending: buffer 0 holds the inverse transform's exchanges, buffer 1 the result
  fft_inv<P>(acc, t, tw, tiles[0] + col * P::N);
#pragma unroll
  for (int e = 0; e < P::E; ++e) tiles[1][tma::swz_tile<C::LX>(pos_first<P>(t, e), col)] = acc[e];
  tma::fence_proxy_async();
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < C::NBOX; ++k) tma::store_3d(&tout, x0, k * C::ROWS, (int)b, tiles[1] + k * C::ROWS * C::LX);
    tma::store_commit();
    tma::store_wait_read();
  }
}

// t2[term] = F_y^-1(Q_term * F_y(t1[0])) with the tiles moved by TMA (plans of 16
// columns per CTA): the input tile arrives once; every term's result goes
// through one swizzled staging tile and a TMA store, the staging tile being
// rewritten only after the previous term's store has read it.  The zeroth Born
// order (Q_KPOW with term0 0, the identity filter) is the input tile scaled,
// stored from the staging tile before the transforms.
template <class P>
struct ColTmaA {
  static constexpr int LX = ColTma<P>::LX, TILE = ColTma<P>::TILE, NBOX = ColTma<P>::NBOX, ROWS = ColTma<P>::ROWS;
  // input tile (then the exchange lines), staging tile, two phase tiles of qt
  // samples (none without them), twiddles, three mbarriers, alignment room
  static size_t smem(size_t qt = 0) {
    return (size_t)(2 * TILE + 2 * qt) * sizeof(float2) + tw_size<P>() * sizeof(float2) + 24 + 1024;
  }
};

// Resident CTAs the single-input TMA pass is held to: with the phase tiles its
// shared memory (two tiles, two phase tiles) leaves room for fewer CTAs than the
// register budget of ColGeo::kMinBlocksA would allow, and registers beyond that
// budget only avoid spills.
template <class P>
constexpr int col_a_tma_min_blocks(bool qtile) {
  constexpr int LX = ColGeo<P>::LX;
  constexpr size_t per = (size_t)(2 * P::N * LX + 2 * LX * ((P::N / 2 + 2) & ~1) + tw_size<P>()) * 8 + 24 + 1024;
  constexpr int fit = (int)((227 * 1024) / per) > 0 ? (int)((227 * 1024) / per) : 1;
  return qtile && fit < ColGeo<P>::kMinBlocksA ? fit : ColGeo<P>::kMinBlocksA;
}

template <class P, int QM, bool kQT>
__global__ void __launch_bounds__(kWarps * 32, col_a_tma_min_blocks<P>(kQT))
    k_col_a_tma(const SpecArgs a, int nxt, const __grid_constant__ CUtensorMap tin,
                const __grid_constant__ CUtensorMap tout, const __grid_constant__ CUtensorMap tq) {
  using C = ColTmaA<P>;
  static_assert(C::LX == 16 || C::LX == 8, "TMA column tiles are 16 or 8 columns (128- or 64-byte rows)");
  extern __shared__ unsigned char smem_raw[];
  float2* in = reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  float2* stage = in + C::TILE;
  const int pny = a.ptab_ny;
  const int qt = kQT ? C::LX * pny : 0;
  float2* const q0 = stage + C::TILE;  // phase slot k at q0 + k * qt
  float2* tw = stage + C::TILE + 2 * qt;
  uint64_t* bar = reinterpret_cast<uint64_t*>(tw + tw_size<P>());  // input, phase slot 0, phase slot 1
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane / P::T, t = lane % P::T, col = warp * P::G + g;
  const long long b = blockIdx.x / nxt;
  const int x0 = (int)(blockIdx.x - b * nxt) * C::LX;
  const int iw = (int)((a.b0 + b) % a.d.nw);
  const int x = x0 + col;
  const int xq = x < a.d.NX ? x : 0;
  const int zstride = (int)(a.tstride / a.d.slice);
  const int k0 = qtile_k0<P>(a, x0);
  const int qrow = qtile_row(a, xq, k0, C::LX) * pny;
  const int nterm = a.nterm;
  if (threadIdx.x == 0) {
    tma::mbar_init(&bar[0], 1);
    tma::mbar_init(&bar[1], 1);
    tma::mbar_init(&bar[2], 1);
    tma::fence_mbar_init();
  }
  load_stage_tw<P>(tw, a.twy);
  __syncthreads();
  auto issue_q = [&](int term) {  // the phase tile of `term` into slot term & 1
    uint64_t* qb = &bar[1 + (term & 1)];
    tma::mbar_expect_tx(qb, (unsigned)(qt * sizeof(float2)));
    tma::load_3d(q0 + (term & 1) * qt, &tq, 0, k0, term * a.d.nw + iw, qb);
  };
  if (threadIdx.x == 0) {
    tma::mbar_expect_tx(&bar[0], (unsigned)(C::TILE * sizeof(float2)));
#pragma unroll
    for (int k = 0; k < C::NBOX; ++k) tma::load_3d(in + k * C::ROWS * C::LX, &tin, x0, k * C::ROWS, (int)b, &bar[0]);
    if constexpr (kQT) {
      if (nterm > 0) issue_q(0);
      if (nterm > 1) issue_q(1);
    }
  }
  // Bounded-wait failure: count it, let the loads in flight land (bounded) and
  // the committed stores read their source, then leave together.
  auto bail = [&](int pending_q) {
    if (threadIdx.x == 0) {
      atomicAdd(a.err, 1u);
      if (kQT && pending_q >= 0 && pending_q < nterm)
        tma::mbar_wait(&bar[1 + (pending_q & 1)], (unsigned)(pending_q >> 1) & 1u);
      tma::store_wait_read();
    }
  };
  const bool ok = tma::mbar_wait(&bar[0], 0u);
  if (!__syncthreads_and(ok)) {
    if (threadIdx.x == 0 && kQT) {
      // the phase loads of terms 0 and 1 may be in flight
      for (int k = 0; k < 2 && k < nterm; ++k) tma::mbar_wait(&bar[1 + k], 0u);
    }
    bail(-1);
    return;
  }
  float2 psi[P::E];
#pragma unroll
  for (int e = 0; e < P::E; ++e) psi[e] = in[tma::swz_tile<C::LX>(pos_first<P>(t, e), col)];
  int first = 0;
  auto store = [&](int term) {  // staging tile -> t2[term]
    tma::fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < C::NBOX; ++k)
        tma::store_3d(&tout, x0, k * C::ROWS, term * zstride + (int)b, stage + k * C::ROWS * C::LX);
      tma::store_commit();
    }
  };
  auto stage_free = [&]() {  // the previous store has read the staging tile
    if (threadIdx.x == 0) tma::store_wait_read();
    __syncthreads();
  };
  if constexpr (QM == Q_KPOW) {
    if (a.term0 == 0 && a.nterm > 0) {
      const float sc = a.norm * (float)P::N;
#pragma unroll
      for (int e = 0; e < P::E; ++e) stage[tma::swz_tile<C::LX>(pos_first<P>(t, e), col)] = cscale(psi[e], sc);
      store(0);
      first = 1;
    }
  }
  __syncthreads();  // every lane holds its column: the input tile becomes the exchange lines
  float2* line = in + col * P::N;
  fft_fwd<P>(psi, t, tw, line);
  for (int term = first; term < nterm; ++term) {
    float2 v[P::E];
    if constexpr (kQT) {
      const bool qok = tma::mbar_wait(&bar[1 + (term & 1)], (unsigned)(term >> 1) & 1u);
      if (!__syncthreads_and(qok)) {
        bail(term + 1);
        return;
      }
      const float2* qr = q0 + (term & 1) * qt + qrow;
      const bool flip = qflip<QM>(a, term, iw);
#pragma unroll
      for (int e = 0; e < P::E; ++e) {
        const int ky = pos_last<P>(t, e);
        const float2 f = qr[min(ky, P::N - ky)];
        v[e] = cmul(psi[e], flip ? cconj(f) : f);
      }
    } else {
      col_factors<P, QM>(a, term, iw, xq, t, v);
#pragma unroll
      for (int e = 0; e < P::E; ++e) v[e] = cmul(psi[e], v[e]);
    }
    fft_inv<P>(v, t, tw, line);
    stage_free();
#pragma unroll
    for (int e = 0; e < P::E; ++e) stage[tma::swz_tile<C::LX>(pos_first<P>(t, e), col)] = v[e];
    store(term);  // also orders this term's phase reads before the slot's next load
    if constexpr (kQT) {
      if (threadIdx.x == 0 && term + 2 < nterm) issue_q(term + 2);
    }
  }
  if (threadIdx.x == 0) tma::store_wait_read();
}

// out (+)= scale * F_y^{-+1}(in): the column half of a plain 2D transform.
template <class P, bool INV>
__global__ void __launch_bounds__(kWarps * 32) k_col_fft(const SpecArgs a, int nxt, const float2* in, float2* out,
                                                          int add, float scale) {
  extern __shared__ float2 smem[];
  ColCtx<P> c(a, smem, nxt);
  load_stage_tw<P>(c.tw, a.twy);
  cols_to_tile<P>(c.tile, in, a, c.b, c.x0);
  __syncthreads();
  float2 v[P::E];
  if (!INV) {
#pragma unroll
    for (int e = 0; e < P::E; ++e) v[e] = c.line[swz(pos_first<P>(c.t, e))];
    fft_fwd<P>(v, c.t, c.tw, c.line);
    __syncwarp();
#pragma unroll
    for (int e = 0; e < P::E; ++e) c.line[swz(pos_last<P>(c.t, e))] = v[e];
  } else {
#pragma unroll
    for (int e = 0; e < P::E; ++e) v[e] = c.line[swz(pos_last<P>(c.t, e))];
    fft_inv<P>(v, c.t, c.tw, c.line);
    __syncwarp();
#pragma unroll
    for (int e = 0; e < P::E; ++e) c.line[swz(pos_first<P>(c.t, e))] = v[e];
  }
  __syncthreads();
  tile_to_cols<P>(c.tile, out, a, c.b, c.x0, add, scale);
}

// ---------------------------------------------------------------- launch helpers

// Sets the shared-memory carveout and, above 48 KB, the dynamic shared-memory limit
// of a kernel, once per (kernel, device, size): the attribute calls cost more host
// time than the launch itself, and the depth loops launch every pass per level.
template <class K>
cudaError_t opt_in_smem(K kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const auto key = std::make_pair((const void*)kernel, dev);
  std::lock_guard<std::mutex> lock(mu);
  auto it = done.find(key);
  if (it != done.end() && it->second >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (e == cudaSuccess && bytes > 48 * 1024)
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) done[key] = bytes;
  return e;
}

#ifndef FWIX_NEXT_WAVE_HINTS
#define FWIX_NEXT_WAVE_HINTS 1
#endif
// CTAs of `kernel` resident on the device at once (cached per kernel, size, device).
template <class K>
int resident_ctas(K kernel, size_t smem) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, size_t, int>, int> done;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  const auto key = std::make_tuple((const void*)kernel, smem, dev);
  std::lock_guard<std::mutex> lock(mu);
  auto it = done.find(key);
  if (it != done.end()) return it->second;
  int per = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kWarps * 32, smem) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    per = 0;
  }
  return done[key] = per * sms;
}

// Launches a row pass with its L2 hint distance: one wave of resident CTAs
// ahead, when the grid has more than one wave (NSPS step at 256 x 256 x 128:
// 0.191 -> 0.187 ms).  The same hint for the TMA column passes' first tile
// measured no faster on the step and 0.4 % slower on the Born step.
template <class K, class... Args>
cudaError_t launch_hinted(K kernel, unsigned grid, size_t sm, cudaStream_t s, const SpecArgs& a, Args... args) {
  cudaError_t e = opt_in_smem(kernel, sm);
  if (e != cudaSuccess) return e;
  SpecArgs b = a;
  b.pf_ctas = 0;
  if (FWIX_NEXT_WAVE_HINTS) {
    const int res = resident_ctas(kernel, sm);
    if (res > 0 && grid > (unsigned)res) b.pf_ctas = res;
  }
  kernel<<<grid, kWarps * 32, sm, s>>>(b, args...);
  return cudaSuccess;
}

template <class P>
cudaError_t row_forward(const SpecArgs& a, int pre, cudaStream_t s) {
  const int nchunk = (a.d.NY + RowGeo<P>::ROWS - 1) / RowGeo<P>::ROWS;
  const unsigned grid = (unsigned)(a.nb * nchunk);
  const size_t sm = pre == W_SCAT_CONJ && a.scat_tab && RowGeo<P>::scat_stage(a.nterm) ? RowGeo<P>::smem_scat(a.nterm)
                                                                                       : RowGeo<P>::smem();
  cudaError_t e;
#define FWIX_FAST_RF(W)                                    \
  case W:                                                  \
    e = launch_hinted(k_row_fwd<P, W>, grid, sm, s, a, nchunk); \
    break;
  if (a.rf_at == 1 && pre != W_ONE && pre != W_MASK) return cudaErrorInvalidValue;
  if (a.rf_at == 1) {
    if (pre == W_ONE)
      e = launch_hinted(k_row_fwd<P, W_ONE, true>, grid, sm, s, a, nchunk);
    else
      e = launch_hinted(k_row_fwd<P, W_MASK, true>, grid, sm, s, a, nchunk);
    if (e == cudaSuccess) count_launch();
    return e != cudaSuccess ? e : cudaGetLastError();
  }
  switch (pre) {
    FWIX_FAST_RF(W_ONE)
    FWIX_FAST_RF(W_TAPER)
    FWIX_FAST_RF(W_MASK)
    FWIX_FAST_RF(W_SCAT_CONJ)
    FWIX_FAST_RF(W_IC)
    FWIX_FAST_RF(W_SMOOTH_CONJ)
    default: return cudaErrorInvalidValue;
  }
#undef FWIX_FAST_RF
  if (e == cudaSuccess) count_launch();
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <class P>
cudaError_t row_inverse(const SpecArgs& a, int post, int post_taper, cudaStream_t s) {
  const int nchunk = (a.d.NY + RowGeo<P>::ROWS - 1) / RowGeo<P>::ROWS;
  const unsigned grid = (unsigned)(a.nb * nchunk);
  const size_t sm = post == W_SCAT && a.scat_tab && RowGeo<P>::scat_stage(a.nterm) ? RowGeo<P>::smem_scat(a.nterm)
                                                                                   : RowGeo<P>::smem();
  cudaError_t e;
#define FWIX_FAST_RI(W)                                                \
  case W:                                                              \
    e = launch_hinted(k_row_inv<P, W>, grid, sm, s, a, nchunk, post_taper); \
    break;
  if (a.rf_at == 2 && post != W_ONE && post != W_MASK) return cudaErrorInvalidValue;
  if (a.rf_at == 2) {
    if (post == W_ONE)
      e = launch_hinted(k_row_inv<P, W_ONE, true>, grid, sm, s, a, nchunk, post_taper);
    else
      e = launch_hinted(k_row_inv<P, W_MASK, true>, grid, sm, s, a, nchunk, post_taper);
    if (e == cudaSuccess) count_launch();
    return e != cudaSuccess ? e : cudaGetLastError();
  }
  switch (post) {
    FWIX_FAST_RI(W_ONE)
    FWIX_FAST_RI(W_ONE_DIRECT)
    FWIX_FAST_RI(W_MASK)
    FWIX_FAST_RI(W_SCAT)
    FWIX_FAST_RI(W_SMOOTH)
    FWIX_FAST_RI(W_SMOOTH_DERIV)
    FWIX_FAST_RI(W_SMOOTH_PAIR)
    default: return cudaErrorInvalidValue;
  }
#undef FWIX_FAST_RI
  if (e == cudaSuccess) count_launch();
  return e != cudaSuccess ? e : cudaGetLastError();
}

// Whether a TMA column pass of plan P takes its phase factors as TMA tiles: the
// phase-shift modes with the cached table, asked for in a.qtile (bit 0 the
// multi-input pass k_col_b, bit 1 the single-input k_col_a), rows of at most 256
// even-length entries, and tiles that never straddle NX / 2 (so that a tile's |kx|
// are consecutive).
template <class P>
bool use_qtile(const SpecArgs& a, int qmode, int bit) {
  constexpr int LX = ColGeo<P>::LX;
  return ((a.qtile >> bit) & 1) && (qmode == Q_PS_FWD || qmode == Q_PS_ADJ) && a.ptab && a.ptab_ny % 2 == 0 &&
         a.ptab_ny <= 256 && (a.d.NX / 2) % LX == 0 && a.ptab_nx >= LX;
}

template <class P>
cudaError_t col_type_a_tma(const SpecArgs& a, int qmode, cudaStream_t s) {
  using C = ColTmaA<P>;
  const int nxt = (a.d.NX + C::LX - 1) / C::LX;
  const unsigned grid = (unsigned)(a.nb * nxt);
  const bool qtile = use_qtile<P>(a, qmode, 1);
  const size_t sm = C::smem(qtile ? (size_t)C::LX * a.ptab_ny : 0);
  CUtensorMap tin, tout, tq;
  std::memset(&tq, 0, sizeof(tq));
  cudaError_t e = tile_map(&tin, a.t1, a.d.NX, a.d.NY, a.nb, C::ROWS, C::LX);
  if (e == cudaSuccess) e = tile_map(&tout, a.t2, a.d.NX, a.d.NY, (a.tstride / a.d.slice) * (a.term0 + a.nterm), C::ROWS, C::LX);
  if (e == cudaSuccess && qtile) e = qtab_map(&tq, a.ptab, a.ptab_ny, a.ptab_nx, (long long)a.nterm * a.d.nw, C::LX);
  if (e != cudaSuccess) return e;
#define FWIX_FAST_CAT(Q, QT)                                                                          \
  e = opt_in_smem(k_col_a_tma<P, Q, QT>, sm);                                                         \
  if (e == cudaSuccess) k_col_a_tma<P, Q, QT><<<grid, kWarps * 32, sm, s>>>(a, nxt, tin, tout, tq);
  switch (qmode) {
    case Q_PS_FWD:
      if (qtile) {
        FWIX_FAST_CAT(Q_PS_FWD, true)
      } else {
        FWIX_FAST_CAT(Q_PS_FWD, false)
      }
      break;
    case Q_PS_ADJ:
      if (qtile) {
        FWIX_FAST_CAT(Q_PS_ADJ, true)
      } else {
        FWIX_FAST_CAT(Q_PS_ADJ, false)
      }
      break;
    case Q_KPOW: FWIX_FAST_CAT(Q_KPOW, false) break;
    case Q_ONE: FWIX_FAST_CAT(Q_ONE, false) break;
    default: return cudaErrorInvalidValue;
  }
#undef FWIX_FAST_CAT
  if (e == cudaSuccess) count_launch();
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <class P>
cudaError_t col_type_a(const SpecArgs& a, int qmode, cudaStream_t s) {
  if constexpr (ColGeo<P>::LX == 16 || ColGeo<P>::LX == 8) {
    if (a.tma && a.err && a.d.NX % 2 == 0) return col_type_a_tma<P>(a, qmode, s);
  }
  const int nxt = (a.d.NX + ColGeo<P>::LX - 1) / ColGeo<P>::LX;
  const unsigned grid = (unsigned)(a.nb * nxt);
  const size_t sm = ColGeo<P>::smem();
  cudaError_t e;
#define FWIX_FAST_CA(Q)                                                           \
  case Q:                                                                         \
    e = opt_in_smem(k_col_a<P, Q>, sm);                                           \
    if (e == cudaSuccess) k_col_a<P, Q><<<grid, kWarps * 32, sm, s>>>(a, nxt);    \
    break;
  switch (qmode) {
    FWIX_FAST_CA(Q_PS_FWD)
    FWIX_FAST_CA(Q_PS_ADJ)
    FWIX_FAST_CA(Q_KPOW)
    FWIX_FAST_CA(Q_ONE)
    default: return cudaErrorInvalidValue;
  }
#undef FWIX_FAST_CA
  if (e == cudaSuccess) count_launch();
  return e != cudaSuccess ? e : cudaGetLastError();
}

// The TMA form of k_col_b: plans of 16 columns per CTA, an even row pitch (the
// tensor map's pitch is a multiple of 16 bytes) and a plan whose error word is set.
template <class P>
cudaError_t col_type_b_tma(const SpecArgs& a, int qmode, cudaStream_t s) {
  using C = ColTma<P>;
  const int nxt = (a.d.NX + C::LX - 1) / C::LX;
  const unsigned grid = (unsigned)(a.nb * nxt);
  const bool qtile = use_qtile<P>(a, qmode, 0);
  const size_t sm = C::smem(qtile ? (size_t)C::LX * a.ptab_ny : 0);
  CUtensorMap tin, tout, tq;
  std::memset(&tq, 0, sizeof(tq));
  cudaError_t e = tile_map(&tin, a.t1, a.d.NX, a.d.NY, (a.tstride / a.d.slice) * a.nterm, C::ROWS, C::LX);
  if (e == cudaSuccess) e = tile_map(&tout, a.t2, a.d.NX, a.d.NY, a.nb, C::ROWS, C::LX);
  if (e == cudaSuccess && qtile) e = qtab_map(&tq, a.ptab, a.ptab_ny, a.ptab_nx, (long long)a.nterm * a.d.nw, C::LX);
  if (e != cudaSuccess) return e;
#define FWIX_FAST_CBT(Q, QT)                                                                          \
  e = opt_in_smem(k_col_b_tma<P, Q, QT>, sm);                                                         \
  if (e == cudaSuccess) k_col_b_tma<P, Q, QT><<<grid, kWarps * 32, sm, s>>>(a, nxt, tin, tout, tq);
  switch (qmode) {
    case Q_PS_FWD:
      if (qtile) {
        FWIX_FAST_CBT(Q_PS_FWD, true)
      } else {
        FWIX_FAST_CBT(Q_PS_FWD, false)
      }
      break;
    case Q_PS_ADJ:
      if (qtile) {
        FWIX_FAST_CBT(Q_PS_ADJ, true)
      } else {
        FWIX_FAST_CBT(Q_PS_ADJ, false)
      }
      break;
    case Q_KPOW: FWIX_FAST_CBT(Q_KPOW, false) break;
    case Q_ONE: FWIX_FAST_CBT(Q_ONE, false) break;
    default: return cudaErrorInvalidValue;
  }
#undef FWIX_FAST_CBT
  if (e == cudaSuccess) count_launch();
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <class P>
cudaError_t col_type_b(const SpecArgs& a, int qmode, cudaStream_t s) {
  if constexpr (ColGeo<P>::LX == 16 || ColGeo<P>::LX == 8) {
    if (a.tma && a.err && a.d.NX % 2 == 0) return col_type_b_tma<P>(a, qmode, s);
  }
  const int nxt = (a.d.NX + ColGeo<P>::LX - 1) / ColGeo<P>::LX;
  const unsigned grid = (unsigned)(a.nb * nxt);
  const size_t sm = ColGeo<P>::smem2();
  cudaError_t e;
#define FWIX_FAST_CB(Q)                                                           \
  case Q:                                                                         \
    e = opt_in_smem(k_col_b<P, Q>, sm);                                           \
    if (e == cudaSuccess) k_col_b<P, Q><<<grid, kWarps * 32, sm, s>>>(a, nxt);    \
    break;
  switch (qmode) {
    FWIX_FAST_CB(Q_PS_FWD)
    FWIX_FAST_CB(Q_PS_ADJ)
    FWIX_FAST_CB(Q_KPOW)
    FWIX_FAST_CB(Q_ONE)
    default: return cudaErrorInvalidValue;
  }
#undef FWIX_FAST_CB
  if (e == cudaSuccess) count_launch();
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <class P>
cudaError_t col_fft(const SpecArgs& a, int inverse, const float2* in, float2* out, int add, float scale,
                    cudaStream_t s) {
  const int nxt = (a.d.NX + ColGeo<P>::LX - 1) / ColGeo<P>::LX;
  const unsigned grid = (unsigned)(a.nb * nxt);
  const size_t sm = ColGeo<P>::smem();
  cudaError_t e;
  if (inverse) {
    e = opt_in_smem(k_col_fft<P, true>, sm);
    if (e == cudaSuccess) k_col_fft<P, true><<<grid, kWarps * 32, sm, s>>>(a, nxt, in, out, add, scale);
  } else {
    e = opt_in_smem(k_col_fft<P, false>, sm);
    if (e == cudaSuccess) k_col_fft<P, false><<<grid, kWarps * 32, sm, s>>>(a, nxt, in, out, add, scale);
  }
  if (e == cudaSuccess) count_launch();
  return e != cudaSuccess ? e : cudaGetLastError();
}

}  // namespace fast
}  // namespace fwix

// One translation unit per line length instantiates the launchers of its plan
// (FWIX_FAST_INSTANTIATE2: one plan for the row passes, another for the columns).
#define FWIX_FAST_INSTANTIATE(PLAN, TAG) FWIX_FAST_INSTANTIATE2(PLAN, PLAN, TAG)
#define FWIX_FAST_INSTANTIATE2(PLAN, CPLAN, TAG)                                                                   \
  namespace fwix {                                                                                          \
  namespace fast {                                                                                          \
  cudaError_t row_forward_##TAG(const SpecArgs& a, int pre, cudaStream_t s) {                               \
    return row_forward<PLAN>(a, pre, s);                                                                    \
  }                                                                                                         \
  cudaError_t row_inverse_##TAG(const SpecArgs& a, int post, int pt, cudaStream_t s) {                      \
    return row_inverse<PLAN>(a, post, pt, s);                                                               \
  }                                                                                                         \
  cudaError_t col_type_a_##TAG(const SpecArgs& a, int q, cudaStream_t s) { return col_type_a<CPLAN>(a, q, s); } \
  cudaError_t col_type_b_##TAG(const SpecArgs& a, int q, cudaStream_t s) { return col_type_b<CPLAN>(a, q, s); } \
  cudaError_t col_fft_##TAG(const SpecArgs& a, int inv, const float2* in, float2* out, int add, float sc,    \
                            cudaStream_t s) {                                                               \
    return col_fft<CPLAN>(a, inv, in, out, add, sc, s);                                                     \
  }                                                                                                         \
  }                                                                                                         \
  }
