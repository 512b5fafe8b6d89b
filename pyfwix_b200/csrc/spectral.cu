// Spectral passes of one depth step.  A 2D unitary transform is split into a row
// pass (one warp per row of NX samples, contiguous in HBM) and a column pass (one
// CTA per tile of TX columns x NY rows, one warp per column).  The per-cell work
// of the reference's separate elementwise kernels -- taper, reference selection,
// Born weights, imaging-condition product, phase shift, k-filters -- is applied
// while the data sits in shared memory, so a PSPI or NSPS step costs three
// kernels instead of 1 + 3*nref elementwise passes plus nref+1 cuFFT calls
// (propagator/src/PSPI.cpp:6-103, propagator/src/NSPS.cpp:6-45).
#include <algorithm>
#include <map>
#include <mutex>
#include <utility>

#include "ops.cuh"

namespace fwix {

namespace {

constexpr int kMaxSmem = 227 * 1024;

// Opt a kernel in to more than 48 KB of dynamic shared memory, once per
// (kernel, device) and size.
template <typename K>
cudaError_t ensure_smem(K kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  auto key = std::make_pair((const void*)kernel, dev);
  auto it = done.find(key);
  if (it != done.end() && it->second >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) done[key] = bytes;
  return e;
}

// ---------------------------------------------------------------- row passes

template <int PRE>
__global__ void __launch_bounds__(256) k_row_forward(const SpecArgs a, int nchunk) {
  extern __shared__ float2 smem[];
  const int NX = a.d.NX;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  float2* tw = smem;
  float2* lineIn = smem + NX + warp * 3 * NX;
  float2* lineA = lineIn + NX;
  float2* lineB = lineA + NX;
  for (int i = threadIdx.x; i < NX; i += blockDim.x) tw[i] = a.twx[i];
  __syncthreads();
  const long long bl = blockIdx.x / nchunk, b = a.b0 + bl;
  const int chunk = blockIdx.x - (int)(bl * nchunk);
  const int iw = (int)(b % a.d.nw);
  const int nterm = multi_term(PRE) ? a.nterm : 1;
  for (int y = chunk * nwarp + warp; y < a.d.NY; y += nchunk * nwarp) {
    const long long roff = (b * a.d.NY + y) * NX;
    const long long loff = (bl * a.d.NY + y) * NX;
    const bool rf = (PRE == W_ONE || PRE == W_MASK) && a.rf_at == 1 && y < a.d.ny;
    for (int x = lane; x < NX; x += 32) {
      float2 v = a.in2 ? cadd(a.in[roff + x], a.in2[roff + x]) : a.in[roff + x];
      if (rf && x < a.d.nx) v = cadd(v, refl_term(a, roff, y, x));
      lineIn[x] = v;
    }
    __syncwarp();
    for (int t = 0; t < nterm; ++t) {
      for (int x = lane; x < NX; x += 32) lineA[x] = row_weight<PRE>(a, t, iw, y, x, lineIn[x]);
      __syncwarp();
      const float2* r = warp_fft<false>(lineA, lineB, 1, a.px, tw, lane);
      float2* o = a.t1 + (long long)t * a.tstride + loff;
      for (int x = lane; x < NX; x += 32) o[x] = r[x];
      __syncwarp();
    }
  }
}

template <int POST>
__global__ void __launch_bounds__(256) k_row_inverse(const SpecArgs a, int nchunk, int post_taper) {
  extern __shared__ float2 smem[];
  const int NX = a.d.NX;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  float2* tw = smem;
  float2* acc = smem + NX + warp * 3 * NX;
  float2* lineA = acc + NX;
  float2* lineB = lineA + NX;
  for (int i = threadIdx.x; i < NX; i += blockDim.x) tw[i] = a.twx[i];
  __syncthreads();
  const long long bl = blockIdx.x / nchunk, b = a.b0 + bl;
  const int chunk = blockIdx.x - (int)(bl * nchunk);
  const int iw = (int)(b % a.d.nw);
  const int nterm = multi_term(POST) ? a.nterm : 1;
  for (int y = chunk * nwarp + warp; y < a.d.NY; y += nchunk * nwarp) {
    const long long roff = (b * a.d.NY + y) * NX;
    const long long loff = (bl * a.d.NY + y) * NX;
    for (int x = lane; x < NX; x += 32) acc[x] = make_float2(0.f, 0.f);
    for (int t = 0; t < nterm; ++t) {
      if (POST == W_MASK) {
        // skip references that no cell of this row selects
        bool hit = false;
        const uint8_t* lrow = a.lab + (long long)iw * a.lab_w + (long long)y * NX;
        for (int x = lane; x < NX; x += 32) hit |= ((int)lrow[x] == t);
        if (!__any_sync(0xffffffffu, hit)) continue;
      }
      const float2* src = a.t2 + (long long)t * a.tstride + loff;
      for (int x = lane; x < NX; x += 32) lineA[x] = src[x];
      __syncwarp();
      const float2* r = warp_fft<true>(lineA, lineB, 1, a.px, tw, lane);
      for (int x = lane; x < NX; x += 32) {
        if (POST == W_MASK) {
          const uint8_t l = a.lab[(long long)iw * a.lab_w + (long long)y * NX + x];
          if ((int)l == t) acc[x] = r[x];
        } else {
          acc[x] = cadd(acc[x], row_weight<POST>(a, t, iw, y, x, r[x]));
        }
      }
      __syncwarp();
    }
    const float ty = post_taper ? a.tapy[y] : 1.f;
    for (int x = lane; x < NX; x += 32) {
      float2 v = acc[x];
      if (post_taper) v = cscale(v, a.tapx[x] * ty);
      if (a.add) v = cadd(a.out[roff + x], v);
      if ((POST == W_ONE || POST == W_MASK) && a.rf_at == 2 && y < a.d.ny && x < a.d.nx)
        v = cadd(v, refl_term(a, roff, y, x));
      a.out[roff + x] = v;
      if (a.ic_img && y < a.d.ny && x < a.d.nx) {
        const float2 bg = a.ic_bg[roff + x];
        atomicAdd(a.ic_img + (long long)y * a.d.nx + x, bg.x * v.x + bg.y * v.y);
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------- column passes

struct ColTiles {
  float2 *tw, *T0, *T1, *T2;
};

__device__ __forceinline__ ColTiles col_tiles(float2* smem, int NY, int TS) {
  ColTiles c;
  c.tw = smem;
  c.T0 = smem + NY;
  c.T1 = c.T0 + NY * TS;
  c.T2 = c.T1 + NY * TS;
  return c;
}

__device__ __forceinline__ void tile_load(float2* T, int TS, const float2* __restrict__ src, int NX,
                                          int NY, int x0, int TX) {
  for (int i = threadIdx.x; i < NY * TX; i += blockDim.x) {
    const int y = i / TX, c = i - y * TX;
    T[y * TS + c] = src[(long long)y * NX + x0 + c];
  }
}

__device__ __forceinline__ void tile_store(const float2* T, int TS, float2* __restrict__ dst, int NX,
                                           int NY, int x0, int TX, int add, float scale) {
  for (int i = threadIdx.x; i < NY * TX; i += blockDim.x) {
    const int y = i / TX, c = i - y * TX;
    float2 v = cscale(T[y * TS + c], scale);
    float2* p = dst + (long long)y * NX + x0 + c;
    if (add) v = cadd(*p, v);
    *p = v;
  }
}

template <int QM>
__global__ void __launch_bounds__(256) k_col_a(const SpecArgs a, int TX, int nxt) {
  extern __shared__ float2 smem[];
  const int NY = a.d.NY, NX = a.d.NX, TS = TX + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  ColTiles s = col_tiles(smem, NY, TS);
  for (int i = threadIdx.x; i < NY; i += blockDim.x) s.tw[i] = a.twy[i];
  const long long b = blockIdx.x / nxt;
  const int x0 = (int)(blockIdx.x - b * nxt) * TX;
  const int iw = (int)((a.b0 + b) % a.d.nw);
  tile_load(s.T0, TS, a.t1 + b * a.d.slice, NX, NY, x0, TX);
  __syncthreads();
  for (int c = warp; c < TX; c += nwarp) warp_fft<false>(s.T0 + c, s.T1 + c, TS, a.py, s.tw, lane);
  const bool odd = a.py.npass & 1;
  float2* F = odd ? s.T1 : s.T0;
  float2* G = odd ? s.T0 : s.T1;
  float2* H = s.T2;
  float2* R = odd ? H : G;
  for (int t = 0; t < a.nterm; ++t) {
    for (int c = warp; c < TX; c += nwarp) {
      const int x = x0 + c;
      for (int y = lane; y < NY; y += 32) G[y * TS + c] = cmul(F[y * TS + c], qmult<QM>(a, t, iw, x, y));
      __syncwarp();
      warp_fft<true>(G + c, H + c, TS, a.py, s.tw, lane);
    }
    __syncthreads();
    tile_store(R, TS, a.t2 + (long long)t * a.tstride + b * a.d.slice, NX, NY, x0, TX, 0, 1.f);
    __syncthreads();
  }
}

template <int QM>
__global__ void __launch_bounds__(256) k_col_b(const SpecArgs a, int TX, int nxt) {
  extern __shared__ float2 smem[];
  const int NY = a.d.NY, NX = a.d.NX, TS = TX + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  ColTiles s = col_tiles(smem, NY, TS);
  for (int i = threadIdx.x; i < NY; i += blockDim.x) s.tw[i] = a.twy[i];
  const long long b = blockIdx.x / nxt;
  const int x0 = (int)(blockIdx.x - b * nxt) * TX;
  const int iw = (int)((a.b0 + b) % a.d.nw);
  float2* Z = s.T2;
  for (int i = threadIdx.x; i < NY * TS; i += blockDim.x) Z[i] = make_float2(0.f, 0.f);
  const bool odd = a.py.npass & 1;
  for (int t = 0; t < a.nterm; ++t) {
    tile_load(s.T0, TS, a.t1 + (long long)t * a.tstride + b * a.d.slice, NX, NY, x0, TX);
    __syncthreads();
    float2* F = odd ? s.T1 : s.T0;
    for (int c = warp; c < TX; c += nwarp) {
      warp_fft<false>(s.T0 + c, s.T1 + c, TS, a.py, s.tw, lane);
      const int x = x0 + c;
      for (int y = lane; y < NY; y += 32)
        Z[y * TS + c] = cadd(Z[y * TS + c], cmul(F[y * TS + c], qmult<QM>(a, t, iw, x, y)));
    }
    __syncthreads();
  }
  for (int c = warp; c < TX; c += nwarp) warp_fft<true>(Z + c, s.T0 + c, TS, a.py, s.tw, lane);
  __syncthreads();
  tile_store(odd ? s.T0 : Z, TS, a.t2 + b * a.d.slice, NX, NY, x0, TX, 0, 1.f);
}

template <bool INV>
__global__ void __launch_bounds__(256) k_col_fft(const SpecArgs a, int TX, int nxt, const float2* in,
                                                 float2* out, int add, float scale) {
  extern __shared__ float2 smem[];
  const int NY = a.d.NY, NX = a.d.NX, TS = TX + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  ColTiles s = col_tiles(smem, NY, TS);
  for (int i = threadIdx.x; i < NY; i += blockDim.x) s.tw[i] = a.twy[i];
  const long long b = blockIdx.x / nxt;
  const int x0 = (int)(blockIdx.x - b * nxt) * TX;
  tile_load(s.T0, TS, in + b * a.d.slice, NX, NY, x0, TX);
  __syncthreads();
  for (int c = warp; c < TX; c += nwarp) warp_fft<INV>(s.T0 + c, s.T1 + c, TS, a.py, s.tw, lane);
  __syncthreads();
  tile_store((a.py.npass & 1) ? s.T1 : s.T0, TS, out + b * a.d.slice, NX, NY, x0, TX, add, scale);
}

// ---------------------------------------------------------------- launch geometry

struct RowGeom {
  int nwarp, nchunk;
  size_t smem;
};

RowGeom row_geom(const Dims& d) {
  RowGeom g;
  const long long per_warp = 3LL * d.NX * (long long)sizeof(float2);
  int nw = 8;
  while (nw > 1 && (size_t)(d.NX * sizeof(float2) + nw * per_warp) > (size_t)kMaxSmem / 2) nw >>= 1;
  g.nwarp = nw;
  g.nchunk = (d.NY + nw - 1) / nw;
  g.smem = d.NX * sizeof(float2) + nw * per_warp;
  return g;
}

struct ColGeom {
  int TX, nxt, nwarp;
  size_t smem;
};

ColGeom col_geom(const Dims& d) {
  ColGeom g;
  int tx = 16;
  while (tx > 1 && (d.NX % tx != 0 ||
                    (size_t)(d.NY + 3LL * d.NY * (tx + 1)) * sizeof(float2) > (size_t)kMaxSmem / 2))
    tx >>= 1;
  g.TX = tx;
  g.nxt = d.NX / tx;
  g.nwarp = std::min(tx, 8);
  g.smem = (size_t)(d.NY + 3LL * d.NY * (tx + 1)) * sizeof(float2);
  return g;
}

long long nblocks(long long slices, long long per) { return slices * per; }

}  // namespace

// ---------------------------------------------------------------- host launchers (generic lengths)

cudaError_t generic_row_forward(const SpecArgs& a, int pre, cudaStream_t s) {
  RowGeom g = row_geom(a.d);
  const long long blocks = nblocks(a.nb, g.nchunk);
  dim3 grid((unsigned)blocks), block(32 * g.nwarp);
  cudaError_t e = cudaSuccess;
#define FWIX_ROWF(W)                                                      \
  case W:                                                                 \
    e = ensure_smem(k_row_forward<W>, g.smem);                            \
    if (e == cudaSuccess) k_row_forward<W><<<grid, block, g.smem, s>>>(a, g.nchunk); \
    break;
  switch (pre) {
    FWIX_ROWF(W_ONE)
    FWIX_ROWF(W_TAPER)
    FWIX_ROWF(W_MASK)
    FWIX_ROWF(W_SCAT_CONJ)
    FWIX_ROWF(W_IC)
    FWIX_ROWF(W_SMOOTH_CONJ)
    default: return cudaErrorInvalidValue;
  }
#undef FWIX_ROWF
  if (e == cudaSuccess) count_launch();
  return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t generic_row_inverse(const SpecArgs& a, int post, int post_taper, cudaStream_t s) {
  RowGeom g = row_geom(a.d);
  const long long blocks = nblocks(a.nb, g.nchunk);
  dim3 grid((unsigned)blocks), block(32 * g.nwarp);
  cudaError_t e = cudaSuccess;
#define FWIX_ROWI(W)                                                                  \
  case W:                                                                             \
    e = ensure_smem(k_row_inverse<W>, g.smem);                                        \
    if (e == cudaSuccess) k_row_inverse<W><<<grid, block, g.smem, s>>>(a, g.nchunk, post_taper); \
    break;
  switch (post) {
    FWIX_ROWI(W_ONE)
    FWIX_ROWI(W_MASK)
    FWIX_ROWI(W_SCAT)
    FWIX_ROWI(W_SMOOTH)
    FWIX_ROWI(W_SMOOTH_DERIV)
    default: return cudaErrorInvalidValue;
  }
#undef FWIX_ROWI
  if (e == cudaSuccess) count_launch();
  return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t generic_col_type_a(const SpecArgs& a, int qmode, cudaStream_t s) {
  ColGeom g = col_geom(a.d);
  dim3 grid((unsigned)(a.nb * g.nxt)), block(32 * g.nwarp);
  cudaError_t e = cudaSuccess;
#define FWIX_COLA(Q)                                                              \
  case Q:                                                                         \
    e = ensure_smem(k_col_a<Q>, g.smem);                                          \
    if (e == cudaSuccess) k_col_a<Q><<<grid, block, g.smem, s>>>(a, g.TX, g.nxt); \
    break;
  switch (qmode) {
    FWIX_COLA(Q_PS_FWD)
    FWIX_COLA(Q_PS_ADJ)
    FWIX_COLA(Q_KPOW)
    FWIX_COLA(Q_ONE)
    default: return cudaErrorInvalidValue;
  }
#undef FWIX_COLA
  if (e == cudaSuccess) count_launch();
  return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t generic_col_type_b(const SpecArgs& a, int qmode, cudaStream_t s) {
  ColGeom g = col_geom(a.d);
  dim3 grid((unsigned)(a.nb * g.nxt)), block(32 * g.nwarp);
  cudaError_t e = cudaSuccess;
#define FWIX_COLB(Q)                                                              \
  case Q:                                                                         \
    e = ensure_smem(k_col_b<Q>, g.smem);                                          \
    if (e == cudaSuccess) k_col_b<Q><<<grid, block, g.smem, s>>>(a, g.TX, g.nxt); \
    break;
  switch (qmode) {
    FWIX_COLB(Q_PS_FWD)
    FWIX_COLB(Q_PS_ADJ)
    FWIX_COLB(Q_KPOW)
    FWIX_COLB(Q_ONE)
    default: return cudaErrorInvalidValue;
  }
#undef FWIX_COLB
  if (e == cudaSuccess) count_launch();
  return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t generic_col_fft(const SpecArgs& a, int inverse, const float2* in, float2* out, int add,
                    float scale, cudaStream_t s) {
  ColGeom g = col_geom(a.d);
  dim3 grid((unsigned)(a.nb * g.nxt)), block(32 * g.nwarp);
  cudaError_t e;
  if (inverse) {
    e = ensure_smem(k_col_fft<true>, g.smem);
    if (e == cudaSuccess) k_col_fft<true><<<grid, block, g.smem, s>>>(a, g.TX, g.nxt, in, out, add, scale);
  } else {
    e = ensure_smem(k_col_fft<false>, g.smem);
    if (e == cudaSuccess) k_col_fft<false><<<grid, block, g.smem, s>>>(a, g.TX, g.nxt, in, out, add, scale);
  }
  if (e == cudaSuccess) count_launch();
  return e != cudaSuccess ? e : cudaGetLastError();
}

}  // namespace fwix

// ---------------------------------------------------------------- single-slice operators
// PhaseShift (phase_shift.cu:7-305), Selector (selector.cu:7-37) and Taper
// (taper.cu:7-77) as standalone operators; inside a depth step they are fused
// into the passes above.

namespace fwix {
namespace {

template <int QM>
__global__ void k_phase_shift(const SpecArgs a, const float2* __restrict__ in, float2* out, int add) {
  const long long n = a.d.wfld;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % a.d.NX);
    const long long r = i / a.d.NX;
    const int y = (int)(r % a.d.NY);
    const int iw = (int)((r / a.d.NY) % a.d.nw);
    float2 v = cmul(in[i], qmult<QM>(a, 0, iw, x, y));
    if (add) v = cadd(out[i], v);
    out[i] = v;
  }
}

template <int W>
__global__ void k_weight(const SpecArgs a, int t, const float2* __restrict__ in, float2* out, int add) {
  const long long n = a.d.wfld;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % a.d.NX);
    const long long r = i / a.d.NX;
    const int y = (int)(r % a.d.NY);
    const int iw = (int)((r / a.d.NY) % a.d.nw);
    float2 v = row_weight<W>(a, t, iw, y, x, in[i]);
    if (add) v = cadd(out[i], v);
    out[i] = v;
  }
}

unsigned grid1d(long long n) {
  long long b = (n + 255) / 256;
  return (unsigned)std::min<long long>(b, 148LL * 32);
}

}  // namespace

cudaError_t launch_phase_shift(const SpecArgs& a, int mode, const float2* sref_w, const float2* in,
                               float2* out, int add, cudaStream_t s) {
  SpecArgs b = a;
  b.sref = sref_w;
  b.norm = 1.f;
  const unsigned g = grid1d(a.d.wfld);
  switch (mode) {
    case Q_PS_FWD: k_phase_shift<Q_PS_FWD><<<g, 256, 0, s>>>(b, in, out, add); break;
    case Q_PS_ADJ: k_phase_shift<Q_PS_ADJ><<<g, 256, 0, s>>>(b, in, out, add); break;
    case Q_PS_INV: k_phase_shift<Q_PS_INV><<<g, 256, 0, s>>>(b, in, out, add); break;
    default: return cudaErrorInvalidValue;
  }
  count_launch();
  return cudaGetLastError();
}

// Forward phase factors x norm of one depth for every (ref, w, |kx|, |ky|): the
// same arithmetic as the in-kernel evaluation (k depends on |index| only).
__global__ void k_phase_table(const SpecArgs a, float2* dst) {
  const long long n = (long long)a.nterm * a.d.nw * a.ptab_nx * a.ptab_ny;
  SpecArgs b = a;
  b.ptab = nullptr;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int kyq = (int)(i % a.ptab_ny);
    long long q = i / a.ptab_ny;
    const int kxq = (int)(q % a.ptab_nx);
    q /= a.ptab_nx;
    const int iw = (int)(q % a.d.nw);
    const int r = (int)(q / a.d.nw);
    dst[i] = qmult<Q_PS_FWD>(b, r, iw, kxq, kyq);
  }
}

cudaError_t launch_phase_table(const SpecArgs& a, float2* dst, cudaStream_t s) {
  const long long n = (long long)a.nterm * a.d.nw * a.ptab_nx * a.ptab_ny;
  k_phase_table<<<grid1d(n), 256, 0, s>>>(a, dst);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_select(const SpecArgs& a, int value, const float2* in, float2* out, int add,
                          cudaStream_t s) {
  k_weight<W_MASK><<<grid1d(a.d.wfld), 256, 0, s>>>(a, value, in, out, add);
  count_launch();
  return cudaGetLastError();
}

__global__ void k_scat_table(const SpecArgs a, float2* dst) {
  const long long n = (long long)a.nterm * a.d.slice;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(i / a.d.slice);
    const long long yx = i - (long long)t * a.d.slice;
    const int y = (int)(yx / a.d.NX), x = (int)(yx - (long long)y * a.d.NX);
    dst[i] = scat_power(a, t, 0, y, x);
  }
}

cudaError_t launch_scat_table(const SpecArgs& a, float2* dst, cudaStream_t s) {
  k_scat_table<<<grid1d((long long)a.nterm * a.d.slice), 256, 0, s>>>(a, dst);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_taper(const SpecArgs& a, const float2* in, float2* out, int add, cudaStream_t s) {
  k_weight<W_TAPER><<<grid1d(a.d.wfld), 256, 0, s>>>(a, 0, in, out, add);
  count_launch();
  return cudaGetLastError();
}

}  // namespace fwix
