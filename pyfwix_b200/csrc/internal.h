// Internal declarations shared by the translation units of libfwix_b200.so.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "fft_device.cuh"

namespace fwix {

// Number of kernels this library has enqueued (fwix_launch_count).
void count_launch(unsigned n = 1);
// Message returned by fwix_last_error() on the calling thread.
void set_last_error(const std::string& msg);

// Per-cell pre-weights of a forward row pass and post-weights of an inverse row pass.
enum RowWeight {
  W_ONE = 0,        // 1
  W_TAPER = 1,      // separable taper w_x * w_y            (taper.cu:46-63)
  W_MASK = 2,       // labels == term                        (selector.cu:29-35)
  W_SCAT = 3,       // Born weight W_n                       (scatter.cu:61-106,155-195)
  W_SCAT_CONJ = 4,  // conj(W_n)
  W_IC = 5,         // bg * image on the unpadded window      (imaging_condition.cu:39-52)
  // differentiable ("smooth") step, no reference counterpart: per reference r a
  // hat-function weight w_r(s) of the local slowness s between the sorted
  // reference slownesses, times the split-step factor SS_r = exp(-i w (s - s_r) dz)
  W_SMOOTH = 6,       // w_r SS_r
  W_SMOOTH_CONJ = 7,  // w_r conj(SS_r)
  W_SMOOTH_DERIV = 8, // d(w_r SS_r)/ds = (w_r' - i w dz w_r) SS_r
  W_ONE_DIRECT = 9,   // 1, plus the Born adjoint's zeroth term conj(W_0) d (inverse row pass only)
  W_SMOOTH_PAIR = 10  // W_SMOOTH into out and W_SMOOTH_DERIV into out2 from the same
                      // inverse transforms (register-resident inverse row pass only)
};

// Weights that run one pass per term (reference or Taylor term).
__host__ __device__ constexpr bool multi_term(int w) {
  return w == W_MASK || w == W_SCAT || w == W_SCAT_CONJ || w == W_SMOOTH || w == W_SMOOTH_CONJ ||
         w == W_SMOOTH_DERIV || w == W_SMOOTH_PAIR;
}

// Spectral multipliers applied between the column FFTs.
enum ColMult {
  Q_PS_FWD = 0,  // e^{Im dz}(cos - i sin)(Re dz)            (phase_shift.cu:36-55)
  Q_PS_ADJ = 1,  // conjugate with the b>0 branch             (phase_shift.cu:153-178)
  Q_PS_INV = 2,  // growing inverse                           (phase_shift.cu:274-298)
  Q_KPOW = 3,    // (|k| / w)^(2n)                            (scatter.cu:49-55)
  Q_ONE = 4
};

struct Dims {
  int NX, NY;       // wavefield (padded)
  int nx, ny;       // model window
  int nw, ns;       // frequencies, shots
  long long slice;  // NX * NY
  long long wfld;   // ns * nw * NX * NY
};

// Everything a spectral kernel may read.  Passed by value (kernel parameter).
struct SpecArgs {
  Dims d;
  Fft1D px, py;
  const float2* twx;
  const float2* twy;
  // tables
  const float* kx;     // [NX]
  const float* ky;     // [NY]
  const float* w2;     // [nw]
  const float* w;      // [nw]
  const float* tapx;   // [NX]
  const float* tapy;   // [NY]
  // depth-dependent inputs
  const float2* sref;  // [nref][nw] at this depth
  const uint8_t* lab;  // labels at this depth, element (iw, y, x) at lab[iw*lab_w + y*NX + x]
  long long lab_w;
  const float2* slow;  // s^2 at this depth (unpadded), (iw, y, x) at slow[iw*slow_w + y*nx + x]
  long long slow_w;
  // when slow_w == 0: s~^(-1/2-n) of the padded slice, [nterm][NY][NX] (NULL: computed per cell)
  const float2* scat_tab;
  const float2* image; // imaging-condition image, (iw, y, x) at image[iw*img_w + y*nx + x] (W_IC)
  long long img_w;     // ny*nx, or 0 for one image shared by every frequency
  // cached forward phase factors of this depth (x norm), element (ref, iw, |kx|, |ky|)
  // at ptab[((ref*nw + iw)*ptab_nx + kxq)*ptab_ny + kyq], kxq = min(x, NX-x),
  // kyq = min(y, NY-y); ptab_nx = NX/2 + 1, ptab_ny = NY/2 + 1 rounded up to even
  // (16-byte rows for TMA); NULL means evaluate the factors in the kernel
  const float2* ptab;
  int ptab_nx, ptab_ny;
  // smooth step: padded local slowness [NY][NX] and the sorted real reference
  // slownesses [sm_n] of this depth
  const float* sm_s;
  const float* sm_ref;
  int sm_n;
  float dz, eps, eps_scat;
  float coef[5];
  float norm;          // scale folded into the column multiplier
  int nterm;           // references (W_MASK) or Taylor terms (W_SCAT)
  // Born scattering adjoint with the zeroth Taylor term applied directly: its
  // filter (|k| / w)^0 is the identity, so conj(W_0) d needs no transform.  The
  // transformed terms are then orders term0 .. term0 + nterm - 1 (term0 = 1), and
  // the inverse row pass (W_ONE_DIRECT) adds conj(W_0) d, d = direct, to its sum
  // (direct_mode 2; 0 = no direct term).
  int term0;
  int direct_mode;
  const float2* direct;
  // buffers.  A launch covers the slices (shot, frequency) b0 .. b0 + nb - 1: in / out
  // (and the labels, images and tables) are indexed by the global slice b0 + bl,
  // the intermediates t1 / t2 by the launch-local slice bl, term after term tstride
  // elements apart.
  const float2* in;    // row-pass input (W_IC: the background wavefield)
  const float2* in2;   // optional second row-pass input added to `in` (NULL: none)
  float2* out;         // row-pass output
  float2* out2;        // second inverse-row-pass output (W_SMOOTH_PAIR: the derivative)
  int add;
  float2* t1;
  float2* t2;
  long long b0, nb, tstride;
  // column passes: move the tiles with TMA where the plan allows (tma != 0); a
  // bounded wait that runs out adds one to *err (the plan's error word)
  int tma;
  unsigned* err;
  // TMA column passes with the cached phase table: bit 0, the multi-input pass
  // takes each term's phase factors as a TMA tile with the term's column tile;
  // bit 1, the single-input pass likewise (else they are loaded per lane)
  int qtile;
  // inverse row pass image epilogue (the lockstep migration): for every output
  // sample of the unpadded window, ic_img[y][x] += Re(conj(ic_bg[b][y][x]) out)
  // by float atomics (ic_img NULL: none)
  const float2* ic_bg;
  float* ic_img;
  // reflections fused into a depth step (a model shared by every frequency):
  // per-cell coefficients rf_tab [2][ny][nx] and fields laid out like `in`, over
  // the unpadded window.  rf_at 1: the first (forward row) pass steps
  // in + rf_tab[0] rf_f1; rf_at 2: the last (inverse row) pass adds
  // rf_tab[0] rf_f1 (+ rf_tab[1] rf_f2 when rf_f2 != NULL) to its output; 0: none.
  int rf_at;
  const float2* rf_tab;
  const float2* rf_f1;
  const float2* rf_f2;
  // register-resident row passes: each CTA hints into L2 the first input rows
  // of the CTA pf_ctas launch positions later, the one that takes its place
  // once every resident CTA has run (0: none)
  int pf_ctas;
};

// Spectral passes (dispatch.cu: register-resident passes for lengths with a
// compile-time plan, else the generic per-warp passes of spectral.cu).  Each
// returns a CUDA error code.
bool fast_length(int n);
cudaError_t row_forward(const SpecArgs& a, int pre, cudaStream_t s);      // in -> t1[0..nterm)
cudaError_t row_inverse(const SpecArgs& a, int post, int post_taper, cudaStream_t s);  // t2 -> out
cudaError_t col_type_a(const SpecArgs& a, int qmode, cudaStream_t s);     // t1[0] -> t2[0..nterm)
cudaError_t col_type_b(const SpecArgs& a, int qmode, cudaStream_t s);     // t1[0..nterm) -> t2[0]
cudaError_t col_fft(const SpecArgs& a, int inverse, const float2* in, float2* out, int add,
                    float scale, cudaStream_t s);
cudaError_t generic_row_forward(const SpecArgs& a, int pre, cudaStream_t s);
cudaError_t generic_row_inverse(const SpecArgs& a, int post, int post_taper, cudaStream_t s);
cudaError_t generic_col_type_a(const SpecArgs& a, int qmode, cudaStream_t s);
cudaError_t generic_col_type_b(const SpecArgs& a, int qmode, cudaStream_t s);
cudaError_t generic_col_fft(const SpecArgs& a, int inverse, const float2* in, float2* out, int add,
                            float scale, cudaStream_t s);

// Powers s~^(-1/2-n), n < nterm, of the edge-padded slowness slice (slow_w == 0):
// dst [nterm][NY][NX] (spectral.cu).
cudaError_t launch_scat_table(const SpecArgs& a, float2* dst, cudaStream_t s);

// One PSPI / NSPS depth step of 256 x 256 slices in one cluster launch
// (fused256.cu); available when the device runs 8-CTA clusters of it.
bool fused_step_available();
cudaError_t fused_step(const SpecArgs& a, int kind, int dir, cudaStream_t s);

// Phase-factor cache of one depth (spectral.cu): dst [nref][nw][ptab_nx][ptab_ny].
cudaError_t launch_phase_table(const SpecArgs& a, float2* dst, cudaStream_t s);

// Pointwise kernels (pointwise.cu).
cudaError_t launch_phase_shift(const SpecArgs& a, int mode, const float2* sref_w, const float2* in,
                               float2* out, int add, cudaStream_t s);
cudaError_t launch_select(const SpecArgs& a, int value, const float2* in, float2* out, int add,
                          cudaStream_t s);
cudaError_t launch_taper(const SpecArgs& a, const float2* in, float2* out, int add, cudaStream_t s);
cudaError_t launch_reflect(const Dims& d, int adjoint, const float2* s0, const float2* s1,
                           const float2* r0, const float2* r1, long long mw, const float2* in,
                           float2* out, int add, cudaStream_t s);
// image / dm arrays are indexed (iw, y, x) -> iw*img_w + y*nx + x; img_w == 0 means one
// array shared by every frequency, whose adjoint sums over frequency.
cudaError_t launch_ic_fwd(const Dims& d, const float2* bg, const float2* image, long long img_w,
                          float2* wfld, int add, cudaStream_t s);
cudaError_t launch_ic_adj(const Dims& d, const float2* bg, const float2* wfld, float2* image,
                          long long img_w, int add, cudaStream_t s);
cudaError_t launch_lin_reflect(const Dims& d, int adjoint, const float2* s0, const float2* s1,
                               const float2* r0, const float2* r1, long long mw, float2* dm0,
                               float2* dm1, float2* dm2, float2* dm3, long long dm_w, float2* dr,
                               int add, cudaStream_t s);
// Linearised reflection fused with the imaging condition: forward wf (+)= bg * LR(dm)
// on every shot; adjoint dm (+)= LR^H(sum_s conj(bg) wf).  With wf2 (adjoint, mw == 0
// and dm_w == 0 only) the imaging-condition adjoint sum_{s,w} conj(bg2) wf2 is added
// to dm0 in the same pass.
cudaError_t launch_lin_reflect_ic(const Dims& d, int adjoint, const float2* s0, const float2* s1,
                                  const float2* r0, const float2* r1, long long mw, float2* dm0, float2* dm1,
                                  float2* dm2, float2* dm3, long long dm_w, const float2* bg, float2* wf, int add,
                                  cudaStream_t s, const float2* bg2 = nullptr, const float2* wf2 = nullptr);
// Per-cell coefficients of the reflections fused into a depth step (model shared
// by every frequency): tab[0][y][x] = r (conj(r) for the adjoint), and with a
// perturbation dm0..dm3 ([ny][nx] each) tab[1][y][x] = its linearised reflection.
cudaError_t launch_refl_table(const Dims& d, int adjoint, const float2* s0, const float2* s1, const float2* r0,
                              const float2* r1, const float2* dm0, const float2* dm1, const float2* dm2,
                              const float2* dm3, float2* tab, cudaStream_t s);
cudaError_t launch_image_acc(const Dims& d, const float2* S, const float2* R, float* img, int add,
                             cudaStream_t s);
// img[y][x] (+)= Re sum_{s,w} conj(S) R over the padded NY x NX slice.
cudaError_t launch_correlate_padded(const Dims& d, const float2* S, const float2* R, float* img, int add,
                                    cudaStream_t s);
// Both at once for one field S: img1 [NY][NX] (+)= Re sum conj(S) R1 over the
// padded slice, img2 [ny][nx] (+)= Re sum conj(S) R2 over the model window.
cudaError_t launch_correlate2_padded(const Dims& d, const float2* S, const float2* R1, const float2* R2,
                                     float* img1, float* img2, int add, cudaStream_t s);
cudaError_t launch_axpy(long long n, const float2* x, float2* y, cudaStream_t s);
// Fixed-rate lossy wavefield store (pack.cu): bytes of one packed array of nfloat
// floats, and the packing / unpacking launches.
size_t packed_rate8_bytes(long long nfloat);
cudaError_t launch_pack_rate8(long long nfloat, const float* in, void* packed, cudaStream_t s);
cudaError_t launch_unpack_rate8(long long nfloat, const void* packed, float* out, cudaStream_t s);
// The same at 8 or 16 mantissa bits.
size_t packed_bytes(long long nfloat, int bits);
cudaError_t launch_pack(int bits, long long nfloat, const float* in, void* packed, cudaStream_t s);
cudaError_t launch_unpack(int bits, long long nfloat, const void* packed, float* out, cudaStream_t s);

// Acquisition kernels (pointwise.cu).  A depth level's injection is a gather
// list: for each target cell, the (trace, weight) pairs that land on it.
struct InjectLevel {
  int ncell;             // target cells touched at this level
  const int* cell;       // [ncell] flat (shot, y, x) -> shot*NY*NX + y*NX + x, no frequency
  const int* start;      // [ncell + 1] offsets into trace/weight
  const int* trace;      // contributing trace
  const float* weight;   // its weight
  int ntr;               // traces recorded at this level
  const int* rtrace;     // [ntr] trace index
  const int* rcell;      // [ntr] flat (shot, y, x) of the (y, x) corner
  const float4* rw;      // [ntr] the four corner weights
};
cudaError_t launch_inject(const Dims& d, const InjectLevel& L, const float2* traces, float2* wfld,
                          cudaStream_t s);
cudaError_t launch_record(const Dims& d, const InjectLevel& L, const float2* wfld, float2* traces,
                          cudaStream_t s);

}  // namespace fwix
