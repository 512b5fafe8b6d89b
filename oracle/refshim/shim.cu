// Reference-kernel shim: C entry points that run pyfwix's OWN CUDA kernels
// (compiled from the reference sources where they lie, see build.py) on
// caller-owned device buffers, so that the oracle can be checked against the
// reference's actual GPU arithmetic and golden fixtures can be generated.
//
// TEST INFRASTRUCTURE ONLY: used by tests/golden/make_golden.py and the parity
// tests, never by the product library.
//
// The reference kernels read their sizes from `complex_vector` headers in
// managed memory (operator/src/complex_vector.h:33-81,
// operator/src/complex_vector.cpp:5-27); Header below builds such a header
// around a caller pointer (n / o / d fastest axis first) and frees it after
// the launch.  Every entry point synchronises the device before returning and
// returns the CUDA error code (0 = success).
#include <cufft.h>

#include <new>
#include <vector>

#include <complex_vector.h>
#include <prop_kernels.cuh>

namespace {

struct Header {
  complex_vector* v = nullptr;
  Header(const void* mat, std::vector<int> n, std::vector<float> o = {}, std::vector<float> d = {}) {
    void* p = nullptr;
    cudaMallocManaged(&p, sizeof(complex_vector));
    v = new (p) complex_vector();
    const int nd = (int)n.size();
    cudaMallocManaged((void**)&v->n, sizeof(int) * nd);
    cudaMallocManaged((void**)&v->o, sizeof(float) * nd);
    cudaMallocManaged((void**)&v->d, sizeof(float) * nd);
    long long ne = 1;
    for (int i = 0; i < nd; ++i) {
      v->n[i] = n[i];
      v->o[i] = i < (int)o.size() ? o[i] : 0.f;
      v->d[i] = i < (int)d.size() ? d[i] : 1.f;
      ne *= n[i];
    }
    v->nelem = (int)ne;
    v->ndim = nd;
    v->mat = (cuFloatComplex*)mat;
    v->allocated = false;
  }
  ~Header() {
    cudaDeviceSynchronize();
    cudaFree(v->n);
    cudaFree(v->o);
    cudaFree(v->d);
    cudaFree(v);
  }
};

const dim3 kGrid3(8, 8, 16), kBlock3(16, 16, 2);

int done() {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  return (int)e;
}

}  // namespace

extern "C" {

// mode 0: ps_forward, 1: ps_adjoint, 2: ps_inverse; out += factor * in
int refshim_phase_shift(int mode, int NX, int NY, int nw, int ns, const float* w2, const float* kx,
                        const float* ky, const void* sref, float dz, float eps, const void* in, void* out) {
  // ps_forward writes data from model; ps_adjoint / ps_inverse write model from data
  Header a(in, {NX, NY, nw, ns}), b(out, {NX, NY, nw, ns});
  if (mode == 0)
    ps_forward<<<kGrid3, kBlock3>>>(a.v, b.v, w2, kx, ky, (const cuFloatComplex*)sref, dz, eps);
  else
    (mode == 1 ? ps_adjoint : ps_inverse)<<<kGrid3, kBlock3>>>(b.v, a.v, w2, kx, ky, (const cuFloatComplex*)sref,
                                                              dz, eps);
  return done();
}

// out += in where labels[w][y][x] == value (labels int32 [nw][NY][NX])
int refshim_select(int NX, int NY, int nw, int ns, int value, const int* labels, const void* in, void* out) {
  Header m(in, {NX, NY, nw, ns}), d(out, {NX, NY, nw, ns});
  select_forward<<<256, 256>>>(m.v, d.v, value, labels);
  return done();
}

// out += taper * in
int refshim_taper(int NX, int NY, int nw, int ns, int tapx, int tapy, const void* in, void* out) {
  Header m(in, {NX, NY, nw, ns}), d(out, {NX, NY, nw, ns});
  taper_forward<<<kGrid3, kBlock3>>>(m.v, d.v, tapx, tapy);
  return done();
}

// adjoint 0: wfld += inject(traces); 1: traces += record(wfld).  traces [ntrace][nw].
int refshim_inject(int adjoint, int NX, int NY, int nw, int ns, float ox, float oy, float dx, float dy, int ntrace,
                   const float* cx, const float* cy, const float* cz, const int* ids, float oz, float dz, int iz,
                   void* traces, void* wfld) {
  Header m(traces, {nw, ntrace}), d(wfld, {NX, NY, nw, ns}, {ox, oy, 0.f, 0.f}, {dx, dy, 1.f, 1.f});
  const dim3 grid((nw + 15) / 16, (ntrace + 15) / 16), block(16, 16);
  (adjoint ? inj_adjoint : inj_forward)<<<grid, block>>>(m.v, d.v, cx, cy, cz, ids, oz, dz, iz);
  return done();
}

// Reflect at one level: slow2 / den2 are [2][nw][ny][nx] (levels z and z+1).
int refshim_reflect(int adjoint, int NX, int NY, int nx, int ny, int nw, int ns, const void* slow2,
                    const void* den2, void* model, void* data) {
  Header m(model, {NX, NY, nw, ns}), d(data, {NX, NY, nw, ns});
  Header s(slow2, {nx, ny, nw, 2}), r(den2, {nx, ny, nw, 2});
  (adjoint ? refl_adjoint : refl_forward)<<<kGrid3, kBlock3>>>(m.v, d.v, s.v, r.v);
  return done();
}

// Imaging condition: image [nw][ny][nx], wfld / bg [ns][nw][NY][NX].
int refshim_imaging(int adjoint, int NX, int NY, int nx, int ny, int nw, int ns, void* image, void* wfld,
                    const void* bg) {
  Header m(image, {nx, ny, nw}), d(wfld, {NX, NY, nw, ns}), b(bg, {NX, NY, nw, ns});
  (adjoint ? ic_adj : ic_fwd)<<<kGrid3, kBlock3>>>(m.v, d.v, b.v);
  return done();
}

// Linearised reflection: model4 [4][nw][ny][nx] (ds0, ds1, drho0, drho1), dr [nw][ny][nx].
int refshim_lin_reflect(int adjoint, int nx, int ny, int nw, void* model4, void* dr, const void* slow2,
                        const void* den2) {
  Header m(model4, {nx, ny, nw, 4}), d(dr, {nx, ny, nw}), s(slow2, {nx, ny, nw, 2}), r(den2, {nx, ny, nw, 2});
  (adjoint ? drefl_adjoint : drefl_forward)<<<kGrid3, kBlock3>>>(m.v, d.v, s.v, r.v);
  return done();
}

// Scatter pieces (propagator/src/Scatter.cpp:76-133 composes them).
int refshim_mult_kxky(int NX, int NY, int nw, int ns, const float* w, const float* kx, const float* ky, int it,
                      const void* in, void* out) {
  Header m(in, {NX, NY, nw, ns}), d(out, {NX, NY, nw, ns});
  mult_kxky<<<kGrid3, kBlock3>>>(m.v, d.v, w, kx, ky, it);
  return done();
}
int refshim_slow_scale(int adjoint, int NX, int NY, int nw, int ns, const void* slow_pad, float coef, int it,
                       float eps, void* model, void* data) {
  Header m(model, {NX, NY, nw, ns}), d(data, {NX, NY, nw, ns}), s(slow_pad, {NX, NY, nw});
  (adjoint ? slow_scale_adj : slow_scale_fwd)<<<kGrid3, kBlock3>>>(m.v, d.v, s.v, coef, it, eps);
  return done();
}
int refshim_scale_by_iw(int adjoint, int NX, int NY, int nw, int ns, const float* w, float dz, void* model,
                        void* data) {
  Header m(model, {NX, NY, nw, ns}), d(data, {NX, NY, nw, ns});
  (adjoint ? scale_by_iw_adj : scale_by_iw_fwd)<<<kGrid3, kBlock3>>>(m.v, d.v, w, dz);
  return done();
}
int refshim_pad(int nx, int ny, int NX, int NY, int nw, const void* in, void* out) {
  Header m(in, {nx, ny, nw}), d(out, {NX, NY, nw});
  pad_fwd<<<kGrid3, kBlock3>>>(m.v, d.v);
  return done();
}

// PSPI::cu_forward (propagator/src/PSPI.cpp:6-24) replayed with the reference's
// kernels and cuFFT on the default stream, for timing the reference's own GPU
// depth step: data->zero(); taper->cu_forward(0, model, model_k);
// fft2d->cu_forward(model_k); per reference: ps->cu_forward(0, model_k,
// wfld_ref) (zero, then ps_forward); fft2d->cu_adjoint(wfld_ref);
// select->cu_forward(1, wfld_ref, data).  Launch shapes as the reference's
// Propagator hands them to its operators (propagator/src/Propagator.cpp:20-21:
// grid {32, 4, 4}, block {16, 16, 4}; Selector.h: 256-thread blocks over every
// sample).  Two differences, both in the reference's favour: the cuFFT plans
// carry no store callback (operator/src/fft_callback.cu scales every stored
// element by 1/sqrt(NX NY); here the outputs are NX NY times the unitary ones
// and that work is not done), and the per-depth host-to-device copies of the
// labels and reference slownesses (Selector.h set_labels, PhaseShift.h
// set_slow) are not made: labels [nw][NY][NX] int32 and sref [nref][nw] are
// already on the device.  One warm-up step, then `reps` steps between CUDA
// events; *ms receives the mean time per step.
int refshim_pspi_forward_timed(int NX, int NY, int nw, int ns, int nref, const float* w2, const float* kx,
                               const float* ky, const void* sref, const int* labels, float dz, float eps, int tapx,
                               int tapy, const void* in, void* out, void* model_k, void* wfld_ref, int reps,
                               float* ms) {
  Header m(in, {NX, NY, nw, ns}), d(out, {NX, NY, nw, ns}), mk(model_k, {NX, NY, nw, ns}),
      wr(wfld_ref, {NX, NY, nw, ns});
  cufftHandle plan;
  int dims[2] = {NY, NX};
  if (cufftPlanMany(&plan, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2C, nw * ns) != CUFFT_SUCCESS) return -1;
  const size_t bytes = (size_t)NX * NY * nw * ns * sizeof(cuFloatComplex);
  const dim3 g(32, 4, 4), b(16, 16, 4);
  const unsigned sel_grid = (unsigned)(((size_t)NX * NY * nw * ns + 255) / 256);
  cufftComplex* K = (cufftComplex*)model_k;
  cufftComplex* W = (cufftComplex*)wfld_ref;
  auto step = [&]() {
    cudaMemsetAsync(out, 0, bytes);
    cudaMemsetAsync(model_k, 0, bytes);
    taper_forward<<<g, b>>>(m.v, mk.v, tapx, tapy);
    cufftExecC2C(plan, K, K, CUFFT_FORWARD);
    for (int r = 0; r < nref; ++r) {
      cudaMemsetAsync(wfld_ref, 0, bytes);
      ps_forward<<<g, b>>>(mk.v, wr.v, w2, kx, ky, (const cuFloatComplex*)sref + (size_t)r * nw, dz, eps);
      cufftExecC2C(plan, W, W, CUFFT_INVERSE);
      select_forward<<<sel_grid, 256>>>(wr.v, d.v, r, labels);
    }
  };
  step();
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaDeviceSynchronize();
  cudaEventRecord(e0);
  for (int i = 0; i < reps; ++i) step();
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  *ms = t / (float)(reps > 0 ? reps : 1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cufftDestroy(plan);
  return done();
}

// ---------------------------------------------------------------------------
// Whole-shot sweeps with the reference's kernels and cuFFT, composed as the
// reference composes them, for the "plain per-shot GPU path" comparison:
//   PSPI in-place forward  (propagator/src/PSPI.cpp:66-83): taper -> FFT -> per
//     reference: phase shift into a zeroed buffer -> inverse FFT -> select-add;
//   PSPI in-place adjoint  (propagator/src/PSPI.cpp:85-103): per reference:
//     select into a zeroed buffer -> FFT -> adjoint phase shift added -> then
//     inverse FFT -> taper;
//   modelling (propagator/src/Propagator.cpp:121-221): down pass inject source,
//     record, keep the field, step; up pass step, reflect the kept down field,
//     record;
//   migration: the source field of the down pass and the receiver field of the
//     back-scattering adjoint (propagator/src/ExtendedBorn.cpp:391-453: inject
//     the data, imaging condition ic_adj, adjoint step) continued in lockstep.
// Launch shapes are the reference operators' (grid {32,4,4} x block {16,16,4}
// for taper / phase shift / imaging, Reflect's grid over (x, y, w*s) with
// 16x16x4 blocks, Injection's (nw/16, ntrace/16) x 16x16, Selector's 256-thread
// blocks over every sample).  Differences, stated: the kept down fields stay
// in device memory (the reference ZFP-compresses and copies them to the host,
// propagator/src/WavefieldPool.cpp); the per-depth host-to-device copies of
// labels and reference slownesses (Selector.h set_labels, PhaseShift.h
// set_slow) are replaced by a device expansion of one depth's labels to every
// frequency; the plans have no store callback, so the 1/(NX NY) of the unitary
// transform pair (operator/src/fft_callback.cu:7-12) is one scaling pass over
// the step's output; the migration sums its per-frequency image over
// frequency into the float image once per level (k_sum_w).  All but the last
// two make the reference path faster than it is; the scaling pass and the sum
// are one read and write of a wavefield and of an image per level.
}  // extern "C"

namespace {

__global__ void k_scale(cuFloatComplex* x, long long n, float s) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] = make_cuFloatComplex(cuCrealf(x[i]) * s, cuCimagf(x[i]) * s);
}

__global__ void k_expand_labels(const int* lab, int* out, long long plane, int nw) {
  const long long n = plane * nw;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = lab[i % plane];
}

// img[y][x] += sum_w Re img_w[w][y][x]
__global__ void k_sum_w(const cuFloatComplex* img_w, float* img, int nw, long long plane) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane; i += (long long)gridDim.x * blockDim.x) {
    float acc = 0.f;
    for (int w = 0; w < nw; ++w) acc += cuCrealf(img_w[(long long)w * plane + i]);
    img[i] += acc;
  }
}

struct Shot {
  int NX, NY, nx, ny, nw, nref, nz, tapx, tapy;
  float dz, eps;
  const float *w2, *kx, *ky;
  const cuFloatComplex* sref;  // [nz][nref][nw]
  const int* labels;           // [nz][NY][NX]
  int* labw;                   // [nw][NY][NX] scratch
  long long n;                 // NX NY nw
  size_t bytes;
  cufftHandle plan = 0;
  dim3 g{32, 4, 4}, b{16, 16, 4};
  unsigned sel_grid = 1;
  Header *K = nullptr, *W = nullptr;

  int init(void* model_k, void* wfld_ref) {
    n = (long long)NX * NY * nw;
    bytes = (size_t)n * sizeof(cuFloatComplex);
    int dims[2] = {NY, NX};
    if (cufftPlanMany(&plan, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2C, nw) != CUFFT_SUCCESS) return -1;
    sel_grid = (unsigned)((n + 255) / 256);
    K = new Header(model_k, {NX, NY, nw, 1});
    W = new Header(wfld_ref, {NX, NY, nw, 1});
    return 0;
  }
  ~Shot() {
    delete K;
    delete W;
    if (plan) cufftDestroy(plan);
  }
  void labels_at(int iz) {
    k_expand_labels<<<1184, 256>>>(labels + (long long)iz * NX * NY, labw, (long long)NX * NY, nw);
  }
  const cuFloatComplex* refs(int iz, int r) const { return sref + ((long long)iz * nref + r) * nw; }
  void scale(Header& X) { k_scale<<<1184, 256>>>(X.v->mat, n, 1.f / ((float)NX * (float)NY)); }
  // PSPI::cu_forward(model) in place on X
  void fwd(int iz, Header& X) {
    labels_at(iz);
    cudaMemsetAsync(K->v->mat, 0, bytes);
    taper_forward<<<g, b>>>(X.v, K->v, tapx, tapy);
    cufftExecC2C(plan, K->v->mat, K->v->mat, CUFFT_FORWARD);
    cudaMemsetAsync(X.v->mat, 0, bytes);
    for (int r = 0; r < nref; ++r) {
      cudaMemsetAsync(W->v->mat, 0, bytes);
      ps_forward<<<g, b>>>(K->v, W->v, w2, kx, ky, refs(iz, r), dz, eps);
      cufftExecC2C(plan, W->v->mat, W->v->mat, CUFFT_INVERSE);
      select_forward<<<sel_grid, 256>>>(W->v, X.v, r, labw);
    }
    scale(X);
  }
  // PSPI::cu_adjoint(data) in place on X
  void adj(int iz, Header& X) {
    labels_at(iz);
    cudaMemsetAsync(K->v->mat, 0, bytes);
    for (int r = 0; r < nref; ++r) {
      cudaMemsetAsync(W->v->mat, 0, bytes);
      select_forward<<<sel_grid, 256>>>(X.v, W->v, r, labw);
      cufftExecC2C(plan, W->v->mat, W->v->mat, CUFFT_FORWARD);
      ps_adjoint<<<g, b>>>(K->v, W->v, w2, kx, ky, refs(iz, r), dz, eps);
    }
    cufftExecC2C(plan, K->v->mat, K->v->mat, CUFFT_INVERSE);
    cudaMemsetAsync(X.v->mat, 0, bytes);
    taper_forward<<<g, b>>>(K->v, X.v, tapx, tapy);
    scale(X);
  }
};

struct Traces {
  int n;
  const float *cx, *cy, *cz;
  const int* ids;
  Header* h;
};

template <class F>
int timed(F run, int reps, float* ms) {
  run();
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaDeviceSynchronize();
  cudaEventRecord(e0);
  for (int i = 0; i < reps; ++i) run();
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  *ms = t / (float)(reps > 0 ? reps : 1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return done();
}

}  // namespace

extern "C" {

// One in-place PSPI step of X [nw][NY][NX] at one level, as the sweeps below
// take it: PSPI::cu_forward(model) (adjoint 0) or PSPI::cu_adjoint(data)
// (adjoint 1), propagator/src/PSPI.cpp:64-102; sref [nref][nw] and labels
// [NY][NX] of that level.  model_k, wfld_ref: wavefield scratch.
int refshim_pspi_step(int adjoint, int NX, int NY, int nw, int nref, const float* w2, const float* kx,
                      const float* ky, const void* sref, const int* labels, int* labw, float dz, float eps, int tapx,
                      int tapy, void* X, void* model_k, void* wfld_ref) {
  Shot sh;
  sh.NX = NX, sh.NY = NY, sh.nx = NX, sh.ny = NY, sh.nw = nw, sh.nref = nref, sh.nz = 1, sh.tapx = tapx;
  sh.tapy = tapy, sh.dz = dz, sh.eps = eps, sh.w2 = w2, sh.kx = kx, sh.ky = ky;
  sh.sref = (const cuFloatComplex*)sref, sh.labels = labels, sh.labw = labw;
  if (sh.init(model_k, wfld_ref) != 0) return -1;
  Header hX(X, {NX, NY, nw, 1});
  if (adjoint)
    sh.adj(0, hX);
  else
    sh.fwd(0, hX);
  return done();
}

// One shot (ns = 1, no padding: NX = nx, NY = ny).  task 0: modelling, data
// [ntrace][nw] recorded, the down field of every level kept in keep [nz][nw][NY][NX];
// slow2 / den2 are the per-frequency model with one level more,
// [nz + 1][nw][ny][nx], level nz a copy of level nz - 1 (the reference's bottom
// reflection pairs the last level with itself, propagator/src/Reflect.h:20-38),
// so that levels (iz, iz + 1) are the pair each reflection reads.  task 1:
// lockstep migration of `data`, image [nz][ny][nx] (float); img_w [nw][ny][nx]
// scratch; task 2: the same with the receivers injected without the race of
// Injection's launch shape (below).  S, R, model_k, wfld_ref: wavefield
// scratch [nw][NY][NX].  One warm-up run, then `reps` runs between CUDA events
// (the image / data are zeroed before each run); *ms receives the mean time.
int refshim_shot_timed(int task, int NX, int NY, int nw, int nz, int nref, const float* w2, const float* kx,
                       const float* ky, const void* sref, const int* labels, int* labw, float dz, float eps, int tapx,
                       int tapy, float ox, float oy, float oz, float dx, float dy, int nsrc, const float* scx,
                       const float* scy, const float* scz, const int* sids, const void* wavelet, int ntrace,
                       const float* rcx, const float* rcy, const float* rcz, const int* rids, void* data,
                       const void* slow2, const void* den2, void* keep, float* image, void* img_w, void* S,
                       void* R, void* model_k, void* wfld_ref, int reps, float* ms) {
  Shot sh;
  sh.NX = NX, sh.NY = NY, sh.nx = NX, sh.ny = NY, sh.nw = nw, sh.nref = nref, sh.nz = nz, sh.tapx = tapx;
  sh.tapy = tapy, sh.dz = dz, sh.eps = eps, sh.w2 = w2, sh.kx = kx, sh.ky = ky;
  sh.sref = (const cuFloatComplex*)sref, sh.labels = labels, sh.labw = labw;
  if (sh.init(model_k, wfld_ref) != 0) return -1;
  const std::vector<float> o4 = {ox, oy, 0.f, 0.f}, d4 = {dx, dy, 1.f, 1.f};
  Header hS(S, {NX, NY, nw, 1}, o4, d4), hR(R, {NX, NY, nw, 1}, o4, d4);
  Header wav(wavelet, {nw, nsrc}), dat(data, {nw, ntrace});
  const dim3 gs((nw + 15) / 16, (nsrc + 15) / 16), gr((nw + 15) / 16, (ntrace + 15) / 16), b2(16, 16);
  const size_t fb = sh.bytes;
  const long long plane = (long long)NX * NY;
  if (task == 0) {
    // per-level views of the kept fields and of the model's level pairs
    std::vector<Header*> kept, sl, dn;
    for (int iz = 0; iz < nz; ++iz) {
      kept.push_back(new Header((char*)keep + (size_t)iz * fb, {NX, NY, nw, 1}));
      sl.push_back(new Header((const char*)slow2 + (size_t)iz * fb, {NX, NY, nw, 2}));
      dn.push_back(new Header((const char*)den2 + (size_t)iz * fb, {NX, NY, nw, 2}));
    }
    const dim3 rg((NX + 15) / 16, (NY + 15) / 16, (nw + 3) / 4), rb(16, 16, 4);
    auto run = [&]() {
      cudaMemsetAsync(data, 0, (size_t)ntrace * nw * sizeof(cuFloatComplex));
      cudaMemsetAsync(S, 0, fb);
      for (int iz = 0; iz < nz; ++iz) {
        inj_forward<<<gs, b2>>>(wav.v, hS.v, scx, scy, scz, sids, oz, dz, iz);
        inj_adjoint<<<gr, b2>>>(dat.v, hS.v, rcx, rcy, rcz, rids, oz, dz, iz);
        cudaMemcpyAsync(kept[iz]->v->mat, S, fb, cudaMemcpyDeviceToDevice);
        sh.fwd(iz, hS);
      }
      cudaMemsetAsync(R, 0, fb);
      for (int iz = nz - 1; iz >= 0; --iz) {
        sh.fwd(iz, hR);
        refl_forward<<<rg, rb>>>(kept[iz]->v, hR.v, sl[iz]->v, dn[iz]->v);
        inj_adjoint<<<gr, b2>>>(dat.v, hR.v, rcx, rcy, rcz, rids, oz, dz, iz);
      }
    };
    const int st = timed(run, reps, ms);
    for (auto* h : kept) delete h;
    for (auto* h : sl) delete h;
    for (auto* h : dn) delete h;
    return st;
  }
  Header img(img_w, {NX, NY, nw});
  // Task 2 launches the receivers' injection with one thread per frequency, each
  // looping over every trace: inj_forward adds into the wavefield without atomics
  // (injection.cu:89-92), so under Injection's launch shape the traces whose
  // bilinear footprints share a cell (receivers on adjacent nodes) race and some
  // additions are lost.  Same kernel, same arithmetic, no race; slower, so only
  // for parity.
  const dim3 gri = task == 2 ? dim3((nw + 15) / 16, 1) : gr, bri = task == 2 ? dim3(16, 1) : b2;
  auto run = [&]() {
    cudaMemsetAsync(image, 0, (size_t)nz * plane * sizeof(float));
    cudaMemsetAsync(S, 0, fb);
    cudaMemsetAsync(R, 0, fb);
    for (int iz = 0; iz < nz; ++iz) {
      inj_forward<<<gs, b2>>>(wav.v, hS.v, scx, scy, scz, sids, oz, dz, iz);
      inj_forward<<<gri, bri>>>(dat.v, hR.v, rcx, rcy, rcz, rids, oz, dz, iz);
      cudaMemsetAsync(img_w, 0, (size_t)plane * nw * sizeof(cuFloatComplex));
      ic_adj<<<sh.g, sh.b>>>(img.v, hR.v, hS.v);
      k_sum_w<<<(unsigned)((plane + 255) / 256), 256>>>((const cuFloatComplex*)img_w, image + iz * plane, nw, plane);
      if (iz < nz - 1) {
        sh.fwd(iz, hS);
        sh.adj(iz, hR);
      }
    }
  };
  return timed(run, reps, ms);
}

}  // extern "C"
