// Per-cell operators of the path that carry no FFT: reflection, imaging
// condition, linearised reflection, injection / recording and the migration
// image.  All are deterministic: a thread owns one (w, y, x) cell and loops over
// shots, so no floating-point atomics are needed where the reference uses them
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

__global__ void k_reflect(Dims d, int adjoint, const float2* __restrict__ s0, const float2* __restrict__ s1,
                          const float2* __restrict__ r0, const float2* __restrict__ r1, long long mw,
                          const float2* __restrict__ in, float2* __restrict__ out) {
  const long long n = (long long)d.nw * d.ny * d.nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % d.nx);
    const long long q = i / d.nx;
    const int y = (int)(q % d.ny);
    const int iw = (int)(q / d.ny);
    const long long m = iw * mw + (long long)y * d.nx + x;
    float2 r = refl_coef(s0[m], s1[m], r0[m], r1[m]);
    if (adjoint) r = cconj(r);
    for (int s = 0; s < d.ns; ++s) {
      const long long k = (((long long)s * d.nw + iw) * d.NY + y) * d.NX + x;
      out[k] = cadd(out[k], cmul(in[k], r));
    }
  }
}

__global__ void k_ic_fwd(Dims d, const float2* __restrict__ bg, const float2* __restrict__ image,
                         long long img_w, float2* __restrict__ wfld) {
  const long long n = (long long)d.nw * d.ny * d.nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % d.nx);
    const long long q = i / d.nx;
    const int y = (int)(q % d.ny);
    const int iw = (int)(q / d.ny);
    const float2 im = image[iw * img_w + (long long)y * d.nx + x];
    for (int s = 0; s < d.ns; ++s) {
      const long long k = (((long long)s * d.nw + iw) * d.NY + y) * d.NX + x;
      wfld[k] = cadd(wfld[k], cmul(bg[k], im));
    }
  }
}

// image[w, y, x] (+)= sum_s conj(bg) wfld; with wsum the frequencies are summed as well
// into image[y, x].
__global__ void k_ic_adj(Dims d, const float2* __restrict__ bg, const float2* __restrict__ wfld,
                         float2* __restrict__ image, int add, int wsum) {
  const int nwo = wsum ? 1 : d.nw;
  const int nwi = wsum ? d.nw : 1;
  const long long n = (long long)nwo * d.ny * d.nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % d.nx);
    const long long q = i / d.nx;
    const int y = (int)(q % d.ny);
    const int iw0 = (int)(q / d.ny);
    float2 acc = make_float2(0.f, 0.f);
    for (int j = 0; j < nwi; ++j) {
      const int iw = iw0 + j;
      for (int s = 0; s < d.ns; ++s) {
        const long long k = (((long long)s * d.nw + iw) * d.NY + y) * d.NX + x;
        acc = cadd(acc, cmul_conj(wfld[k], bg[k]));
      }
    }
    image[i] = add ? cadd(image[i], acc) : acc;
  }
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

__global__ void k_lin_reflect(Dims d, int adjoint, const float2* __restrict__ s0, const float2* __restrict__ s1,
                              const float2* __restrict__ r0, const float2* __restrict__ r1, long long mw,
                              float2* dm0, float2* dm1, float2* dm2, float2* dm3, long long dm_w, float2* dr,
                              int add) {
  // forward: one thread per (w, y, x) of dr.  adjoint: one thread per (w, y, x) of dm,
  // or per (y, x) with a loop over w when dm is shared by every frequency.
  const int wsum = adjoint && dm_w == 0;
  const int nwo = wsum ? 1 : d.nw;
  const long long n = (long long)nwo * d.ny * d.nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % d.nx);
    const long long q = i / d.nx;
    const int y = (int)(q % d.ny);
    const int iw0 = (int)(q / d.ny);
    const long long yx = (long long)y * d.nx + x;
    if (!adjoint) {
      const long long m = iw0 * mw + yx, k = iw0 * dm_w + yx;
      const LinCoef c = lin_coef(s0[m], s1[m], r0[m], r1[m]);
      float2 v = csub(cmul(c.as, dm0[k]), cmul(c.bs, dm1[k]));
      v = cadd(v, csub(cmul(c.ar, dm3[k]), cmul(c.br, dm2[k])));
      dr[i] = add ? cadd(dr[i], v) : v;
      continue;
    }
    float2 g0 = make_float2(0.f, 0.f), g1 = g0, g2 = g0, g3 = g0;
    for (int j = 0; j < (wsum ? d.nw : 1); ++j) {
      const int iw = iw0 + j;
      const long long m = iw * mw + yx;
      const LinCoef c = lin_coef(s0[m], s1[m], r0[m], r1[m]);
      const float2 g = dr[(long long)iw * d.ny * d.nx + yx];
      g0 = cadd(g0, cmul_conj(g, c.as));
      g1 = csub(g1, cmul_conj(g, c.bs));
      g3 = cadd(g3, cmul_conj(g, c.ar));
      g2 = csub(g2, cmul_conj(g, c.br));
    }
    const long long k = iw0 * dm_w + yx;
    // dm0 and dm1 (dm2 and dm3) alias at the bottom level; the same thread adds both.
    dm0[k] = add ? cadd(dm0[k], g0) : g0;
    dm1[k] = (add || dm1 == dm0) ? cadd(dm1[k], g1) : g1;
    dm2[k] = add ? cadd(dm2[k], g2) : g2;
    dm3[k] = (add || dm3 == dm2) ? cadd(dm3[k], g3) : g3;
  }
}

__global__ void k_image_acc(Dims d, const float2* __restrict__ S, const float2* __restrict__ R,
                            float* __restrict__ img, int add) {
  const long long n = (long long)d.ny * d.nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % d.nx);
    const int y = (int)(i / d.nx);
    float acc = 0.f;
    for (int s = 0; s < d.ns; ++s)
      for (int iw = 0; iw < d.nw; ++iw) {
        const long long k = (((long long)s * d.nw + iw) * d.NY + y) * d.NX + x;
        const float2 a = S[k], b = R[k];
        acc += a.x * b.x + a.y * b.y;  // Re(conj(S) R)
      }
    img[i] = add ? img[i] + acc : acc;
  }
}

__global__ void k_axpy(long long n, const float2* __restrict__ x, float2* __restrict__ y) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = cadd(y[i], x[i]);
}

// wfld[shot, w, y, x] += sum_k weight_k * traces[trace_k, w] for each listed cell.
__global__ void k_inject(Dims d, InjectLevel L, const float2* __restrict__ traces, float2* wfld) {
  const long long n = (long long)L.ncell * d.nw;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int iw = (int)(i % d.nw);
    const int e = (int)(i / d.nw);
    float2 acc = make_float2(0.f, 0.f);
    for (int k = L.start[e]; k < L.start[e + 1]; ++k)
      acc = cadd(acc, cscale(traces[(long long)L.trace[k] * d.nw + iw], L.weight[k]));
    const long long cell = L.cell[e];
    const long long shot = cell / d.slice, yx = cell - shot * d.slice;
    const long long k = (shot * d.nw + iw) * d.slice + yx;
    wfld[k] = cadd(wfld[k], acc);
  }
}

// traces[t, w] += sum of the four corner weights times the wavefield.
__global__ void k_record(Dims d, InjectLevel L, const float2* __restrict__ wfld, float2* traces) {
  const long long n = (long long)L.ntr * d.nw;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int iw = (int)(i % d.nw);
    const int e = (int)(i / d.nw);
    const long long cell = L.rcell[e];
    const long long shot = cell / d.slice, yx = cell - shot * d.slice;
    const float2* p = wfld + (shot * d.nw + iw) * d.slice + yx;
    const float4 w = L.rw[e];
    float2 v = cscale(p[0], w.x);
    v = cadd(v, cscale(p[1], w.y));
    v = cadd(v, cscale(p[d.NX], w.z));
    v = cadd(v, cscale(p[d.NX + 1], w.w));
    const long long t = (long long)L.rtrace[e] * d.nw + iw;
    traces[t] = cadd(traces[t], v);
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
  k_reflect<<<grid1d((long long)d.nw * d.ny * d.nx), 256, 0, s>>>(d, adjoint, s0, s1, r0, r1, mw, in, out);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_ic_fwd(const Dims& d, const float2* bg, const float2* image, long long img_w,
                          float2* wfld, int add, cudaStream_t s) {
  if (!add) {
    cudaError_t e = cudaMemsetAsync(wfld, 0, d.wfld * sizeof(float2), s);
    if (e != cudaSuccess) return e;
  }
  k_ic_fwd<<<grid1d((long long)d.nw * d.ny * d.nx), 256, 0, s>>>(d, bg, image, img_w, wfld);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_ic_adj(const Dims& d, const float2* bg, const float2* wfld, float2* image,
                          long long img_w, int add, cudaStream_t s) {
  const int wsum = img_w == 0;
  k_ic_adj<<<grid1d((long long)(wsum ? 1 : d.nw) * d.ny * d.nx), 256, 0, s>>>(d, bg, wfld, image, add, wsum);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_lin_reflect(const Dims& d, int adjoint, const float2* s0, const float2* s1,
                               const float2* r0, const float2* r1, long long mw, float2* dm0,
                               float2* dm1, float2* dm2, float2* dm3, long long dm_w, float2* dr,
                               int add, cudaStream_t s) {
  const long long n = (long long)((adjoint && dm_w == 0) ? 1 : d.nw) * d.ny * d.nx;
  k_lin_reflect<<<grid1d(n), 256, 0, s>>>(d, adjoint, s0, s1, r0, r1, mw, dm0, dm1, dm2, dm3, dm_w, dr, add);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_image_acc(const Dims& d, const float2* S, const float2* R, float* img, int add,
                             cudaStream_t s) {
  k_image_acc<<<grid1d((long long)d.ny * d.nx), 256, 0, s>>>(d, S, R, img, add);
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
  k_inject<<<grid1d((long long)L.ncell * d.nw), 256, 0, s>>>(d, L, traces, wfld);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_record(const Dims& d, const InjectLevel& L, const float2* wfld, float2* traces,
                          cudaStream_t s) {
  if (L.ntr == 0) return cudaSuccess;
  k_record<<<grid1d((long long)L.ntr * d.nw), 256, 0, s>>>(d, L, wfld, traces);
  count_launch();
  return cudaGetLastError();
}

}  // namespace fwix
