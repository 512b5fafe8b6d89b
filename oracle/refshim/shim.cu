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

}  // extern "C"
