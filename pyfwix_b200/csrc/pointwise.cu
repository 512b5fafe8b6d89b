// Per-cell operators of the path that carry no FFT: reflection, imaging
// condition, linearised reflection, injection / recording and the migration
// image.  All are deterministic: a thread owns a (y, x) cell and a fixed set of
// frequencies and loops over shots, and sums over frequencies are reduced in a
// fixed order, so no floating-point atomics are needed where the reference uses them
// (imaging_condition.cu:103-104, lin_reflect.cu:369-384), and the injection is a
// gather over a host-built list instead of the reference's unsynchronised
// read-modify-write (injection.cu:89-92).
#include <algorithm>

#include "internal.h"

namespace fwix {
namespace {

unsigned grid1d(long long n) {
  long long b = (n + 255) / 256;
  return (unsigned)std::max<long long>(1, std::min<long long>(b, 148LL * 32));
}

// Normal-incidence coefficient r = (rho1 sqrt(s0) - rho0 sqrt(s1)) / (rho1 sqrt(s0) + rho0 sqrt(s1))
// (reflect.cu:42-45).
__device__ __forceinline__ float2 refl_coef(float2 s0, float2 s1, float2 r0, float2 r1) {
  const float2 a = cmul(r1, csqrt_ref(s0));
  const float2 b = cmul(r0, csqrt_ref(s1));
  return cdiv(csub(a, b), cadd(a, b));
}

// Block shape of the per-cell kernels: 32 consecutive (y, x) cells of the
// unpadded window by 8 frequency groups.  A thread walks the frequencies
// iw = threadIdx.y, threadIdx.y + 8, ..., so a coefficient that does not depend
// on the frequency (model stride mw == 0) is computed once per thread, and a sum
// over frequencies is finished by a fixed-order reduction of the 8 groups in
// shared memory.
constexpr int kCells = 32, kGroups = 8;

struct Cell {
  int yx, y, x;
  bool ok;
};
__device__ __forceinline__ Cell this_cell(const Dims& d) {
  Cell c;
  c.yx = blockIdx.x * kCells + threadIdx.x;
  c.ok = c.yx < d.ny * d.nx;
  c.y = c.ok ? c.yx / d.nx : 0;
  c.x = c.ok ? c.yx - c.y * d.nx : 0;
  return c;
}
__device__ __forceinline__ long long wf_index(const Dims& d, int s, int iw, const Cell& c) {
  return (((long long)s * d.nw + iw) * d.NY + c.y) * d.NX + c.x;
}

// Sums v over the 8 frequency groups of each cell in a fixed order; thread
// (x, 0) gets the total.
template <int K>
__device__ __forceinline__ void reduce_groups(float2 (&v)[K]) {
  __shared__ float2 red[K][kGroups][kCells];
#pragma unroll
  for (int k = 0; k < K; ++k) red[k][threadIdx.y][threadIdx.x] = v[k];
  __syncthreads();
  if (threadIdx.y == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      float2 t = red[k][0][threadIdx.x];
#pragma unroll
      for (int g = 1; g < kGroups; ++g) t = cadd(t, red[k][g][threadIdx.x]);
      v[k] = t;
    }
  }
}

unsigned cell_blocks(const Dims& d) { return (unsigned)((d.ny * d.nx + kCells - 1) / kCells); }

template <bool S1>
__global__ void __launch_bounds__(kCells * kGroups)
    k_reflect(Dims d, int adjoint, const float2* __restrict__ s0, const float2* __restrict__ s1,
              const float2* __restrict__ r0, const float2* __restrict__ r1, long long mw,
              const float2* __restrict__ in, float2* __restrict__ out) {
  const Cell c = this_cell(d);
  // one model for every frequency: the first group forms each cell's coefficient once
  __shared__ float2 rs[kCells];
  if (mw == 0) {
    if (threadIdx.y == 0 && c.ok) {
      const float2 r = refl_coef(s0[c.yx], s1[c.yx], r0[c.yx], r1[c.yx]);
      rs[threadIdx.x] = adjoint ? cconj(r) : r;
    }
    __syncthreads();
  }
  if (!c.ok) return;
  float2 r = mw == 0 ? rs[threadIdx.x] : make_float2(0.f, 0.f);
  const int ns = S1 ? 1 : d.ns;
#pragma unroll 4
  for (int iw = threadIdx.y; iw < d.nw; iw += kGroups) {
    if (mw != 0) {
      const long long m = iw * mw + c.yx;
      r = refl_coef(s0[m], s1[m], r0[m], r1[m]);
      if (adjoint) r = cconj(r);
    }
    for (int s = 0; s < ns; ++s) {
      const long long k = wf_index(d, s, iw, c);
      out[k] = cadd(out[k], cmul(in[k], r));
    }
  }
}

__global__ void __launch_bounds__(kCells * kGroups)
    k_ic_fwd(Dims d, const float2* __restrict__ bg, const float2* __restrict__ image, long long img_w,
             float2* __restrict__ wfld) {
  const Cell c = this_cell(d);
  if (!c.ok) return;
#pragma unroll 4
  for (int iw = threadIdx.y; iw < d.nw; iw += kGroups) {
    const float2 im = image[iw * img_w + c.yx];
    for (int s = 0; s < d.ns; ++s) {
      const long long k = wf_index(d, s, iw, c);
      wfld[k] = cadd(wfld[k], cmul(bg[k], im));
    }
  }
}

// image[w, y, x] (+)= sum_s conj(bg) wfld; with wsum the frequencies are summed as well
// into image[y, x].
template <bool S1>
__global__ void __launch_bounds__(kCells * kGroups)
    k_ic_adj(Dims d, const float2* __restrict__ bg, const float2* __restrict__ wfld, float2* __restrict__ image,
             int add, int wsum) {
  const Cell c = this_cell(d);
  float2 acc[1] = {make_float2(0.f, 0.f)};
  const int ns = S1 ? 1 : d.ns;
#pragma unroll 4
  for (int iw = threadIdx.y; c.ok && iw < d.nw; iw += kGroups) {
    float2 t = make_float2(0.f, 0.f);
    for (int s = 0; s < ns; ++s) {
      const long long k = wf_index(d, s, iw, c);
      t = cadd(t, cmul_conj(wfld[k], bg[k]));
    }
    if (wsum) {
      acc[0] = cadd(acc[0], t);
    } else {
      float2* o = image + (long long)iw * d.ny * d.nx + c.yx;
      *o = add ? cadd(*o, t) : t;
    }
  }
  if (!wsum) return;
  reduce_groups<1>(acc);
  if (threadIdx.y == 0 && c.ok) image[c.yx] = add ? cadd(image[c.yx], acc[0]) : acc[0];
}

// Coefficients of drefl_forward (lin_reflect.cu:248-292).
struct LinCoef {
  float2 as, bs, ar, br;
};
__device__ __forceinline__ LinCoef lin_coef(float2 s0, float2 s1, float2 r0, float2 r1) {
  const float2 q0 = csqrt_ref(s0), q1 = csqrt_ref(s1);
  const float2 den = cadd(cmul(r1, q0), cmul(r0, q1));
  const float2 inv = cinv(den);
  const float2 inv2 = cmul(inv, inv);
  const float2 s1s2sq = cmul(cmul(r0, r1), inv2);
  const float2 r1r2sq = cmul(cscale(cmul(q0, q1), 2.f), inv2);
  const float2 sc = csqrt_ref(cdiv(q1, q0));
  LinCoef c;
  c.as = cmul(sc, s1s2sq);
  c.bs = cmul(cinv(sc), s1s2sq);
  c.ar = cmul(r0, r1r2sq);
  c.br = cmul(r1, r1r2sq);
  return c;
}

// forward: dr[w, y, x] (+)= as dm0 - bs dm1 + ar dm3 - br dm2.  adjoint: the
// conjugate-transposed sums into dm[w] (dm_w != 0) or into dm shared by every
// frequency (dm_w == 0, summed over w).
// With IC the reflectivity perturbation dr is not stored: the forward adds
// bg * dr to the wavefield wf of every shot (the imaging-condition forward,
// imaging_condition.cu:9-55) and the adjoint takes dr = sum_s conj(bg) wf (its
// adjoint, :57-108), which saves writing and re-reading dr.  IC2 (adjoint, model
// and perturbation shared by every frequency): the same pass also sums the
// imaging-condition adjoint of another pair, dm0 += sum conj(bg2) wf2, so that
// one read of the four fields serves both frequency sums of a level.
template <bool IC, bool S1, bool IC2>
__global__ void __launch_bounds__(kCells * kGroups)
    k_lin_reflect(Dims d, int adjoint, const float2* __restrict__ s0, const float2* __restrict__ s1,
                  const float2* __restrict__ r0, const float2* __restrict__ r1, long long mw, float2* dm0,
                  float2* dm1, float2* dm2, float2* dm3, long long dm_w, float2* dr, int add,
                  const float2* __restrict__ bg, float2* __restrict__ wf, const float2* __restrict__ bg2,
                  const float2* __restrict__ wf2) {
  const Cell c = this_cell(d);
  const int ns = S1 ? 1 : d.ns;
  const long long plane = (long long)d.ny * d.nx;
  const int wsum = adjoint && dm_w == 0;
  LinCoef cf;
  // one model for every frequency: the first group forms each cell's coefficients once
  __shared__ LinCoef cs[kCells];
  if (mw == 0) {
    if (threadIdx.y == 0 && c.ok) cs[threadIdx.x] = lin_coef(s0[c.yx], s1[c.yx], r0[c.yx], r1[c.yx]);
    __syncthreads();
    cf = cs[threadIdx.x];
  }
  float2 g[4] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
  // model and perturbation shared by every frequency (with the imaging condition):
  // dr is one value per cell, and the adjoint's frequency sum commutes with the
  // coefficients, so both are formed once per cell
  if (IC && mw == 0 && dm_w == 0) {
    const long long k = c.yx;
    if (!adjoint) {
      if (!c.ok) return;
      float2 v = csub(cmul(cf.as, dm0[k]), cmul(cf.bs, dm1[k]));
      v = cadd(v, csub(cmul(cf.ar, dm3[k]), cmul(cf.br, dm2[k])));
#pragma unroll 4
      for (int iw = threadIdx.y; iw < d.nw; iw += kGroups)
        for (int sh = 0; sh < ns; ++sh) {
          const long long q = wf_index(d, sh, iw, c);
          wf[q] = cadd(wf[q], cmul(bg[q], v));
        }
      return;
    }
    constexpr int K = IC2 ? 2 : 1;
    float2 gi[K];
#pragma unroll
    for (int j = 0; j < K; ++j) gi[j] = make_float2(0.f, 0.f);
#pragma unroll 4
    for (int iw = threadIdx.y; c.ok && iw < d.nw; iw += kGroups)
      for (int sh = 0; sh < ns; ++sh) {
        const long long q = wf_index(d, sh, iw, c);
        gi[0] = cadd(gi[0], cmul_conj(wf[q], bg[q]));
        if constexpr (IC2) gi[K - 1] = cadd(gi[K - 1], cmul_conj(wf2[q], bg2[q]));
      }
    reduce_groups<K>(gi);  // every thread of the block
    if (threadIdx.y != 0 || !c.ok) return;
    float2 t0 = cmul_conj(gi[0], cf.as);
    const float2 t1 = cscale(cmul_conj(gi[0], cf.bs), -1.f);
    if constexpr (IC2) t0 = cadd(t0, gi[K - 1]);
    const float2 t3 = cmul_conj(gi[0], cf.ar), t2 = cscale(cmul_conj(gi[0], cf.br), -1.f);
    dm0[k] = add ? cadd(dm0[k], t0) : t0;
    dm1[k] = (add || dm1 == dm0) ? cadd(dm1[k], t1) : t1;
    dm2[k] = add ? cadd(dm2[k], t2) : t2;
    dm3[k] = (add || dm3 == dm2) ? cadd(dm3[k], t3) : t3;
    return;
  }
#pragma unroll 4
  for (int iw = threadIdx.y; c.ok && iw < d.nw; iw += kGroups) {
    if (mw != 0) {
      const long long m = iw * mw + c.yx;
      cf = lin_coef(s0[m], s1[m], r0[m], r1[m]);
    }
    const long long i = iw * plane + c.yx, k = iw * dm_w + c.yx;
    if (!adjoint) {
      float2 v = csub(cmul(cf.as, dm0[k]), cmul(cf.bs, dm1[k]));
      v = cadd(v, csub(cmul(cf.ar, dm3[k]), cmul(cf.br, dm2[k])));
      if (IC) {
        for (int sh = 0; sh < ns; ++sh) {
          const long long q = wf_index(d, sh, iw, c);
          wf[q] = cadd(wf[q], cmul(bg[q], v));
        }
      } else {
        dr[i] = add ? cadd(dr[i], v) : v;
      }
      continue;
    }
    float2 gi;
    if (IC) {
      gi = make_float2(0.f, 0.f);
      for (int sh = 0; sh < ns; ++sh) {
        const long long q = wf_index(d, sh, iw, c);
        gi = cadd(gi, cmul_conj(wf[q], bg[q]));
      }
    } else {
      gi = dr[i];
    }
    const float2 t0 = cmul_conj(gi, cf.as), t1 = cscale(cmul_conj(gi, cf.bs), -1.f);
    const float2 t3 = cmul_conj(gi, cf.ar), t2 = cscale(cmul_conj(gi, cf.br), -1.f);
    if (wsum) {
      g[0] = cadd(g[0], t0);
      g[1] = cadd(g[1], t1);
      g[2] = cadd(g[2], t2);
      g[3] = cadd(g[3], t3);
    } else {
      // dm0 and dm1 (dm2 and dm3) alias at the bottom level; the same thread adds both.
      dm0[k] = add ? cadd(dm0[k], t0) : t0;
      dm1[k] = (add || dm1 == dm0) ? cadd(dm1[k], t1) : t1;
      dm2[k] = add ? cadd(dm2[k], t2) : t2;
      dm3[k] = (add || dm3 == dm2) ? cadd(dm3[k], t3) : t3;
    }
  }
  if (!wsum) return;
  reduce_groups<4>(g);
  if (threadIdx.y != 0 || !c.ok) return;
  const long long k = c.yx;
  dm0[k] = add ? cadd(dm0[k], g[0]) : g[0];
  dm1[k] = (add || dm1 == dm0) ? cadd(dm1[k], g[1]) : g[1];
  dm2[k] = add ? cadd(dm2[k], g[2]) : g[2];
  dm3[k] = (add || dm3 == dm2) ? cadd(dm3[k], g[3]) : g[3];
}

// Per-cell reflection coefficients of a model shared by every frequency, for the
// reflections fused into a depth step (SpecArgs::rf_tab): tab[yx] = r (conj(r)
// for the adjoint) and, given a perturbation (dm0 != NULL, one value per cell),
// tab[ny nx + yx] = as dm0 - bs dm1 + ar dm3 - br dm2, the linearised reflection
// that k_lin_reflect's forward forms.
__global__ void __launch_bounds__(256)
    k_refl_table(Dims d, int adjoint, const float2* __restrict__ s0, const float2* __restrict__ s1,
                 const float2* __restrict__ r0, const float2* __restrict__ r1, const float2* __restrict__ dm0,
                 const float2* __restrict__ dm1, const float2* __restrict__ dm2, const float2* __restrict__ dm3,
                 float2* __restrict__ tab) {
  const long long n = (long long)d.ny * d.nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float2 r = refl_coef(s0[i], s1[i], r0[i], r1[i]);
    tab[i] = adjoint ? cconj(r) : r;
    if (dm0) {
      const LinCoef cf = lin_coef(s0[i], s1[i], r0[i], r1[i]);
      float2 v = csub(cmul(cf.as, dm0[i]), cmul(cf.bs, dm1[i]));
      v = cadd(v, csub(cmul(cf.ar, dm3[i]), cmul(cf.br, dm2[i])));
      tab[n + i] = v;
    }
  }
}

template <bool S1>
__global__ void __launch_bounds__(kCells * kGroups)
    k_image_acc(Dims d, const float2* __restrict__ S, const float2* __restrict__ R, float* __restrict__ img,
                int add) {
  const Cell c = this_cell(d);
  float2 acc[1] = {make_float2(0.f, 0.f)};
  const int ns = S1 ? 1 : d.ns;
#pragma unroll 4
  for (int iw = threadIdx.y; c.ok && iw < d.nw; iw += kGroups)
    for (int s = 0; s < ns; ++s) {
      const long long k = wf_index(d, s, iw, c);
      const float2 a = S[k], b = R[k];
      acc[0].x += a.x * b.x + a.y * b.y;  // Re(conj(S) R)
    }
  reduce_groups<1>(acc);
  if (threadIdx.y == 0 && c.ok) img[c.yx] = add ? img[c.yx] + acc[0].x : acc[0].x;
}

// Two correlations of one field S in one pass over the padded window (the
// caller's Dims widened to NY x NX): img1[y][x] (+)= Re sum conj(S) R1 there, and
// img2[y][x] (+)= Re sum conj(S) R2 over the model window ny2 x nx2.
template <bool S1>
__global__ void __launch_bounds__(kCells * kGroups)
    k_image_acc2(Dims d, int ny2, int nx2, const float2* __restrict__ S, const float2* __restrict__ R1,
                 const float2* __restrict__ R2, float* __restrict__ img1, float* __restrict__ img2, int add) {
  const Cell c = this_cell(d);
  float2 acc[1] = {make_float2(0.f, 0.f)};
  const int ns = S1 ? 1 : d.ns;
  const bool in2 = c.ok && c.y < ny2 && c.x < nx2;
#pragma unroll 4
  for (int iw = threadIdx.y; c.ok && iw < d.nw; iw += kGroups)
    for (int s = 0; s < ns; ++s) {
      const long long k = wf_index(d, s, iw, c);
      const float2 a = S[k], b = R1[k];
      acc[0].x += a.x * b.x + a.y * b.y;
      if (in2) {
        const float2 e = R2[k];
        acc[0].y += a.x * e.x + a.y * e.y;
      }
    }
  reduce_groups<1>(acc);
  if (threadIdx.y != 0 || !c.ok) return;
  img1[c.yx] = add ? img1[c.yx] + acc[0].x : acc[0].x;
  if (in2) {
    float* o = img2 + (long long)c.y * nx2 + c.x;
    *o = add ? *o + acc[0].y : acc[0].y;
  }
}

__global__ void k_axpy(long long n, const float2* __restrict__ x, float2* __restrict__ y) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = cadd(y[i], x[i]);
}

// Injection and recording move data between traces [trace][w] (frequency
// fastest) and the wavefield [shot][w][y][x] (x fastest).  A block takes 32
// listed cells (or receivers) x 32 frequencies and transposes through shared
// memory, so that both sides are touched in contiguous runs.  Cells within a
// level's list are distinct, and so are receivers, so no two threads write
// the same element.

// wfld[shot, w, y, x] += sum_k weight_k * traces[trace_k, w] for each listed cell.
__global__ void __launch_bounds__(256) k_inject(Dims d, InjectLevel L, const float2* __restrict__ traces,
                                                float2* wfld) {
  __shared__ float2 tile[32][33];
  const int e0 = blockIdx.x * 32, w0 = blockIdx.y * 32;
  const int iw = w0 + threadIdx.x;
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int e = e0 + k;
    float2 acc = make_float2(0.f, 0.f);
    if (e < L.ncell && iw < d.nw)
      for (int j = L.start[e]; j < L.start[e + 1]; ++j)
        acc = cadd(acc, cscale(traces[(long long)L.trace[j] * d.nw + iw], L.weight[j]));
    tile[k][threadIdx.x] = acc;
  }
  __syncthreads();
  const int e = e0 + threadIdx.x;
  if (e >= L.ncell) return;
  const long long cell = L.cell[e];
  const long long shot = cell / d.slice, yx = cell - shot * d.slice;
  for (int f = threadIdx.y; f < 32 && w0 + f < d.nw; f += 8) {
    const long long k = (shot * d.nw + w0 + f) * d.slice + yx;
    wfld[k] = cadd(wfld[k], tile[threadIdx.x][f]);
  }
}

// traces[t, w] += sum of the four corner weights times the wavefield.
__global__ void __launch_bounds__(256) k_record(Dims d, InjectLevel L, const float2* __restrict__ wfld,
                                                float2* traces) {
  __shared__ float2 tile[32][33];
  const int e0 = blockIdx.x * 32, w0 = blockIdx.y * 32;
  const int e = e0 + threadIdx.x;
  if (e < L.ntr) {
    const long long cell = L.rcell[e];
    const long long shot = cell / d.slice, yx = cell - shot * d.slice;
    const float4 w = L.rw[e];
    for (int f = threadIdx.y; f < 32 && w0 + f < d.nw; f += 8) {
      const float2* p = wfld + (shot * d.nw + w0 + f) * d.slice + yx;
      float2 v = cscale(p[0], w.x);
      v = cadd(v, cscale(p[1], w.y));
      v = cadd(v, cscale(p[d.NX], w.z));
      v = cadd(v, cscale(p[d.NX + 1], w.w));
      tile[f][threadIdx.x] = v;
    }
  }
  __syncthreads();
  const int iw = w0 + threadIdx.x;
  if (iw >= d.nw) return;
  for (int k = threadIdx.y; k < 32 && e0 + k < L.ntr; k += 8) {
    const long long t = (long long)L.rtrace[e0 + k] * d.nw + iw;
    traces[t] = cadd(traces[t], tile[threadIdx.x][k]);
  }
}

}  // namespace

cudaError_t launch_reflect(const Dims& d, int adjoint, const float2* s0, const float2* s1,
                           const float2* r0, const float2* r1, long long mw, const float2* in,
                           float2* out, int add, cudaStream_t s) {
  if (!add) {
    cudaError_t e = cudaMemsetAsync(out, 0, d.wfld * sizeof(float2), s);
    if (e != cudaSuccess) return e;
  }
  if (d.ns == 1)
    k_reflect<true><<<cell_blocks(d), dim3(kCells, kGroups), 0, s>>>(d, adjoint, s0, s1, r0, r1, mw, in, out);
  else
    k_reflect<false><<<cell_blocks(d), dim3(kCells, kGroups), 0, s>>>(d, adjoint, s0, s1, r0, r1, mw, in, out);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_ic_fwd(const Dims& d, const float2* bg, const float2* image, long long img_w,
                          float2* wfld, int add, cudaStream_t s) {
  if (!add) {
    cudaError_t e = cudaMemsetAsync(wfld, 0, d.wfld * sizeof(float2), s);
    if (e != cudaSuccess) return e;
  }
  k_ic_fwd<<<cell_blocks(d), dim3(kCells, kGroups), 0, s>>>(d, bg, image, img_w, wfld);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_ic_adj(const Dims& d, const float2* bg, const float2* wfld, float2* image,
                          long long img_w, int add, cudaStream_t s) {
  if (d.ns == 1)
    k_ic_adj<true><<<cell_blocks(d), dim3(kCells, kGroups), 0, s>>>(d, bg, wfld, image, add, img_w == 0);
  else
    k_ic_adj<false><<<cell_blocks(d), dim3(kCells, kGroups), 0, s>>>(d, bg, wfld, image, add, img_w == 0);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_lin_reflect(const Dims& d, int adjoint, const float2* s0, const float2* s1,
                               const float2* r0, const float2* r1, long long mw, float2* dm0,
                               float2* dm1, float2* dm2, float2* dm3, long long dm_w, float2* dr,
                               int add, cudaStream_t s) {
  k_lin_reflect<false, false, false><<<cell_blocks(d), dim3(kCells, kGroups), 0, s>>>(
      d, adjoint, s0, s1, r0, r1, mw, dm0, dm1, dm2, dm3, dm_w, dr, add, nullptr, nullptr, nullptr, nullptr);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_lin_reflect_ic(const Dims& d, int adjoint, const float2* s0, const float2* s1,
                                  const float2* r0, const float2* r1, long long mw, float2* dm0, float2* dm1,
                                  float2* dm2, float2* dm3, long long dm_w, const float2* bg, float2* wf, int add,
                                  cudaStream_t s, const float2* bg2, const float2* wf2) {
  const dim3 grid(cell_blocks(d)), block(kCells, kGroups);
  if (wf2) {
    if (!adjoint || mw != 0 || dm_w != 0 || !bg2) return cudaErrorInvalidValue;
    if (d.ns == 1)
      k_lin_reflect<true, true, true><<<grid, block, 0, s>>>(d, adjoint, s0, s1, r0, r1, mw, dm0, dm1, dm2, dm3,
                                                             dm_w, nullptr, add, bg, wf, bg2, wf2);
    else
      k_lin_reflect<true, false, true><<<grid, block, 0, s>>>(d, adjoint, s0, s1, r0, r1, mw, dm0, dm1, dm2, dm3,
                                                              dm_w, nullptr, add, bg, wf, bg2, wf2);
  } else if (d.ns == 1) {
    k_lin_reflect<true, true, false><<<grid, block, 0, s>>>(d, adjoint, s0, s1, r0, r1, mw, dm0, dm1, dm2, dm3,
                                                            dm_w, nullptr, add, bg, wf, nullptr, nullptr);
  } else {
    k_lin_reflect<true, false, false><<<grid, block, 0, s>>>(d, adjoint, s0, s1, r0, r1, mw, dm0, dm1, dm2, dm3,
                                                             dm_w, nullptr, add, bg, wf, nullptr, nullptr);
  }
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_refl_table(const Dims& d, int adjoint, const float2* s0, const float2* s1, const float2* r0,
                              const float2* r1, const float2* dm0, const float2* dm1, const float2* dm2,
                              const float2* dm3, float2* tab, cudaStream_t s) {
  k_refl_table<<<grid1d((long long)d.ny * d.nx), 256, 0, s>>>(d, adjoint, s0, s1, r0, r1, dm0, dm1, dm2, dm3, tab);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_image_acc(const Dims& d, const float2* S, const float2* R, float* img, int add,
                             cudaStream_t s) {
  if (d.ns == 1)
    k_image_acc<true><<<cell_blocks(d), dim3(kCells, kGroups), 0, s>>>(d, S, R, img, add);
  else
    k_image_acc<false><<<cell_blocks(d), dim3(kCells, kGroups), 0, s>>>(d, S, R, img, add);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_correlate_padded(const Dims& d, const float2* S, const float2* R, float* img, int add,
                                    cudaStream_t s) {
  Dims full = d;  // iterate over the padded slice: the cell window is the whole NY x NX
  full.nx = d.NX;
  full.ny = d.NY;
  if (d.ns == 1)
    k_image_acc<true><<<cell_blocks(full), dim3(kCells, kGroups), 0, s>>>(full, S, R, img, add);
  else
    k_image_acc<false><<<cell_blocks(full), dim3(kCells, kGroups), 0, s>>>(full, S, R, img, add);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_correlate2_padded(const Dims& d, const float2* S, const float2* R1, const float2* R2,
                                     float* img1, float* img2, int add, cudaStream_t s) {
  Dims full = d;  // the padded slice; img2 covers the model window d.ny x d.nx
  full.nx = d.NX;
  full.ny = d.NY;
  if (d.ns == 1)
    k_image_acc2<true><<<cell_blocks(full), dim3(kCells, kGroups), 0, s>>>(full, d.ny, d.nx, S, R1, R2, img1, img2,
                                                                           add);
  else
    k_image_acc2<false><<<cell_blocks(full), dim3(kCells, kGroups), 0, s>>>(full, d.ny, d.nx, S, R1, R2, img1,
                                                                            img2, add);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_axpy(long long n, const float2* x, float2* y, cudaStream_t s) {
  k_axpy<<<grid1d(n), 256, 0, s>>>(n, x, y);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_inject(const Dims& d, const InjectLevel& L, const float2* traces, float2* wfld,
                          cudaStream_t s) {
  if (L.ncell == 0) return cudaSuccess;
  const dim3 grid((unsigned)((L.ncell + 31) / 32), (unsigned)((d.nw + 31) / 32));
  k_inject<<<grid, dim3(32, 8), 0, s>>>(d, L, traces, wfld);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_record(const Dims& d, const InjectLevel& L, const float2* wfld, float2* traces,
                          cudaStream_t s) {
  if (L.ntr == 0) return cudaSuccess;
  const dim3 grid((unsigned)((L.ntr + 31) / 32), (unsigned)((d.nw + 31) / 32));
  k_record<<<grid, dim3(32, 8), 0, s>>>(d, L, wfld, traces);
  count_launch();
  return cudaGetLastError();
}

}  // namespace fwix
