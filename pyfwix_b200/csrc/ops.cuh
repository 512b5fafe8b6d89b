// Per-cell weights and spectral multipliers shared by the generic (spectral.cu)
// and the register-resident (fast.cuh) passes.
#pragma once
#include "internal.h"

namespace fwix {

// Reflection term fused into a row pass (SpecArgs::rf_at) at sample x of the row
// that starts at roff (row y < ny of the unpadded window; the caller checks x < nx).
__device__ __forceinline__ float2 refl_term(const SpecArgs& a, long long roff, int y, int x) {
  const long long yx = (long long)y * a.d.nx + x;
  float2 v = cmul(a.rf_tab[yx], a.rf_f1[roff + x]);
  if (a.rf_f2) v = cadd(v, cmul(a.rf_tab[(long long)a.d.ny * a.d.nx + yx], a.rf_f2[roff + x]));
  return v;
}

// Born weight W_n = (-i w dz / 2) c_n s~^(-1/2-n), s~ = Re s^2 + i (Im s^2 - eps Re s^2),
// read from the unpadded slice with edge replication into the pad
// (scatter.cu:61-106 slow_scale, :155-195 scale_by_iw, :240-277 pad_fwd).
// s~^(-1/2-n) = (1/sqrt(s~)) (1/s~)^n with the principal root.
__device__ __forceinline__ float2 scat_power(const SpecArgs& a, int n, int iw, int y, int x) {
  const int xs = min(x, a.d.nx - 1), ys = min(y, a.d.ny - 1);
  const float2 s2 = a.slow[(long long)iw * a.slow_w + (long long)ys * a.d.nx + xs];
  const float2 st = make_float2(s2.x, s2.y - a.eps_scat * s2.x);
  float2 p = cinv(csqrt_ref(st));
  if (n > 0) {
    const float2 is = cinv(st);
    for (int k = 0; k < n; ++k) p = cmul(p, is);
  }
  return p;
}

__device__ __forceinline__ float2 scat_weight(const SpecArgs& a, int n, int iw, int y, int x) {
  const float f = 0.5f * a.w[iw] * a.dz * a.coef[n];
  if (a.scat_tab) return rot90<false>(cscale(a.scat_tab[((long long)n * a.d.NY + y) * a.d.NX + x], f));
  const int xs = min(x, a.d.nx - 1), ys = min(y, a.d.ny - 1);
  const float2 s2 = a.slow[(long long)iw * a.slow_w + (long long)ys * a.d.nx + xs];
  const float2 st = make_float2(s2.x, s2.y - a.eps_scat * s2.x);
  float2 p = cinv(csqrt_ref(st));
  if (n > 0) {
    const float2 is = cinv(st);
    for (int k = 0; k < n; ++k) p = cmul(p, is);
  }
  return rot90<false>(cscale(p, f));
}

// Zeroth Born term of the scattering adjoint applied directly
// (SpecArgs::direct_mode): conj(W_0) d at cell (y, x) of global slice b.
__device__ __forceinline__ float2 scat_direct(const SpecArgs& a, long long b, int iw, int y, int x) {
  return cmul_conj(a.direct[(b * a.d.NY + y) * a.d.NX + x], scat_weight(a, 0, iw, y, x));
}

// Hat-function interpolation weight of reference t at slowness s and its
// derivative, on references sorted ascending (clamped to the end references
// outside their range, where the derivative is 0).
struct Hat {
  float w, dw;
};
__device__ __forceinline__ Hat hat_weight(const float* ref, int n, int t, float s) {
  Hat h = {0.f, 0.f};
  if (n == 1) {
    h.w = 1.f;
    return h;
  }
  if (s <= ref[0]) {
    h.w = t == 0 ? 1.f : 0.f;
    return h;
  }
  if (s >= ref[n - 1]) {
    h.w = t == n - 1 ? 1.f : 0.f;
    return h;
  }
  int j = 0;
  while (j < n - 2 && s >= ref[j + 1]) ++j;
  const float span = ref[j + 1] - ref[j];
  const float u = (s - ref[j]) / span;
  if (t == j) {
    h.w = 1.f - u;
    h.dw = -1.f / span;
  } else if (t == j + 1) {
    h.w = u;
    h.dw = 1.f / span;
  }
  return h;
}

// Terms whose hat weight or its derivative can be nonzero at slowness s (bit r
// for reference r; only the bracketing pair, or one end reference outside).
__device__ __forceinline__ unsigned hat_support(const float* ref, int n, float s) {
  if (n == 1 || s <= ref[0]) return 1u;
  if (s >= ref[n - 1]) return 1u << (n - 1);
  int j = 0;
  while (j < n - 2 && s >= ref[j + 1]) ++j;
  return 3u << j;
}

// The split-step factor of the smooth step factors into a cell part and a
// reference part: SS_r = exp(-i w (s - s_r) dz) = B(s) C_r with B(s) =
// exp(-i w s dz) and C_r = exp(i w s_r dz).  The register-resident row passes use
// it to take one sine / cosine per cell (B, applied once to the sum over
// references, or once to the input of the adjoint) and one per reference and
// line (C_r) instead of one per cell and reference.
__device__ __forceinline__ float2 smooth_cell_phase(const SpecArgs& a, int iw, float s) {  // B(s)
  float sn, cs;
  sincosf(a.w[iw] * a.dz * s, &sn, &cs);
  return make_float2(cs, -sn);
}
__device__ __forceinline__ float2 smooth_ref_phase(const SpecArgs& a, int iw, int t) {  // C_t
  float sn, cs;
  sincosf(a.w[iw] * a.dz * a.sm_ref[t], &sn, &cs);
  return make_float2(cs, sn);
}
// Reference part of the weight of term t at slowness s: w_t C_t (W_SMOOTH),
// w_t conj(C_t) (W_SMOOTH_CONJ) or (w_t' - i w dz w_t) C_t (W_SMOOTH_DERIV).
template <int W>
__device__ __forceinline__ float2 smooth_ref_weight(const SpecArgs& a, int t, int iw, float s, float2 C) {
  const Hat h = hat_weight(a.sm_ref, a.sm_n, t, s);
  if (W == W_SMOOTH) return cscale(C, h.w);
  if (W == W_SMOOTH_CONJ) return cscale(cconj(C), h.w);
  return cmul(make_float2(h.dw, -a.w[iw] * a.dz * h.w), C);
}

// w_r SS_r (W_SMOOTH), w_r conj(SS_r) (W_SMOOTH_CONJ) or (w_r' - i w dz w_r) SS_r
// (W_SMOOTH_DERIV) for reference t at cell (y, x) of frequency iw.
template <int W>
__device__ __forceinline__ float2 smooth_factor(const SpecArgs& a, int t, int iw, int y, int x) {
  const float s = a.sm_s[(long long)y * a.d.NX + x];
  const Hat h = hat_weight(a.sm_ref, a.sm_n, t, s);
  if (h.w == 0.f && h.dw == 0.f) return make_float2(0.f, 0.f);
  const float wdz = a.w[iw] * a.dz;
  float sn, cs;
  sincosf(wdz * (s - a.sm_ref[t]), &sn, &cs);
  const float2 ss = make_float2(cs, -sn);  // exp(-i w (s - s_t) dz)
  if (W == W_SMOOTH) return cscale(ss, h.w);
  if (W == W_SMOOTH_CONJ) return cscale(cconj(ss), h.w);
  return cmul(make_float2(h.dw, -wdz * h.w), ss);
}

template <int W>
__device__ __forceinline__ float2 row_weight(const SpecArgs& a, int t, int iw, int y, int x, float2 v) {
  if (W == W_SMOOTH || W == W_SMOOTH_CONJ || W == W_SMOOTH_DERIV) return cmul(v, smooth_factor<W>(a, t, iw, y, x));
  if (W == W_ONE || W == W_ONE_DIRECT) return v;
  if (W == W_TAPER) return cscale(v, a.tapx[x] * a.tapy[y]);
  if (W == W_MASK) {
    const uint8_t l = a.lab[(long long)iw * a.lab_w + (long long)y * a.d.NX + x];
    return (int)l == t ? v : make_float2(0.f, 0.f);
  }
  if (W == W_SCAT) return cmul(v, scat_weight(a, t + a.term0, iw, y, x));
  if (W == W_SCAT_CONJ) return cmul_conj(v, scat_weight(a, t + a.term0, iw, y, x));
  // W_IC
  if (y < a.d.ny && x < a.d.nx)
    return cmul(v, a.image[(long long)iw * a.img_w + (long long)y * a.d.nx + x]);
  return make_float2(0.f, 0.f);
}

// Column multiplier for term t at (iw, ky[y], kx[x]), scaled by a.norm.
template <int QM>
__device__ __forceinline__ float2 qmult(const SpecArgs& a, int t, int iw, int x, int y) {
  if (QM == Q_ONE) return make_float2(a.norm, 0.f);
  if (QM == Q_KPOW) {
    // (|k| / w)^(2t) (scatter.cu:49-50), the power by products
    const int n = t + a.term0;
    if (n == 0) return make_float2(a.norm, 0.f);
    const float kx = a.kx[x], ky = a.ky[y];
    const float r2 = (kx * kx + ky * ky) / a.w2[iw];  // (|k| / w)^2
    float p = r2;
    for (int k = 1; k < n; ++k) p *= r2;
    return make_float2(p * a.norm, 0.f);
  }
  const float2 sr = a.sref[t * a.d.nw + iw];
  const float w2 = a.w2[iw];
  if ((QM == Q_PS_FWD || QM == Q_PS_ADJ) && a.ptab) {
    const int kxq = min(x, a.d.NX - x), kyq = min(y, a.d.NY - y);
    const float2 P = a.ptab[(((long long)t * a.d.nw + iw) * a.ptab_nx + kxq) * a.ptab_ny + kyq];
    if (QM == Q_PS_FWD) return P;
    // adjoint factor: conj(P), or P itself where the reference flips Re (b > 0)
    const float bb = w2 * (sr.y - a.eps * sr.x);
    return bb > 0.f ? P : cconj(P);
  }
  const float kx = a.kx[x], ky = a.ky[y];
  const float aa = w2 * sr.x - (kx * kx + ky * ky);
  const float bb = w2 * (sr.y - a.eps * sr.x);
  float re, im;
  if (bb == 0.f) {
    // c = sqrt(a^2) = |a| exactly, so the general branch reduces to one root.
    if (aa >= 0.f) {
      re = sqrtf(aa);
      im = 0.f;
    } else {
      re = 0.f;
      im = -sqrtf(-aa);
    }
  } else {
    // Re = sqrt((c+a)/2), Im = -sqrt((c-a)/2) as phase_shift.cu:38-41, with the
    // smaller of the two taken from Re |Im| = |b| / 2: the same values without
    // the cancellation of c - a (or c + a) in float.
    const float c = sqrtf(aa * aa + bb * bb);
    if (aa >= 0.f) {
      re = sqrtf((c + aa) * 0.5f);
      im = -(fabsf(bb) * 0.5f) / re;
    } else {
      im = -sqrtf((c - aa) * 0.5f);
      re = (fabsf(bb) * 0.5f) / -im;
    }
  }
  if (QM == Q_PS_ADJ && bb > 0.f) re = -re;
  if (QM == Q_PS_INV) {
    im = -im;
    if (bb > 0.f) re = -re;
  }
  const float att = (im == 0.f ? 1.f : expf(im * a.dz)) * a.norm;
  float sn = 0.f, cs = 1.f;
  if (re != 0.f) sincosf(re * a.dz, &sn, &cs);
  return QM == Q_PS_FWD ? make_float2(att * cs, -att * sn) : make_float2(att * cs, att * sn);
}

// Phase-table view of one column (fixed x) for one term: the factors of every
// ky of that column are then one load each (qcol_get).  Only for the cached
// phase-shift path (a.ptab set, Q_PS_FWD / Q_PS_ADJ).
struct QCol {
  const float2* p;
  bool flip;  // adjoint: conj(P) unless the reference's b > 0 branch applies
};
template <int QM>
__device__ __forceinline__ QCol qcol(const SpecArgs& a, int t, int iw, int x) {
  QCol q;
  const int kxq = min(x, a.d.NX - x);
  q.p = a.ptab + (((long long)t * a.d.nw + iw) * a.ptab_nx + kxq) * a.ptab_ny;
  if (QM == Q_PS_ADJ) {
    const float2 sr = a.sref[t * a.d.nw + iw];
    q.flip = !(a.w2[iw] * (sr.y - a.eps * sr.x) > 0.f);
  } else {
    q.flip = false;
  }
  return q;
}
__device__ __forceinline__ float2 qcol_get(const SpecArgs& a, const QCol& q, int y) {
  const float2 P = q.p[min(y, a.d.NY - y)];
  return q.flip ? cconj(P) : P;
}

}  // namespace fwix
