// fwix_step_noalloc: one PSPI / NSPS depth step that allocates no device memory.
//
// Who needs it: callers that cannot call cudaMalloc.  A typical case is a host
// application (a plugin host, a framework with its own device memory pool, an
// embedded or real-time pipeline) that reserves the GPU's memory up front and
// does not let a library allocate afterwards -- a cudaMalloc there would fail,
// fragment the host's pool, or stall the device at a bad time.  Such callers
// pass inputs and outputs that they own and nothing else.
//
// How: the step's scratch (the wavefield-sized intermediates between the row and
// column passes, and the small wavenumber / twiddle / taper tables) lives in the
// file-scope array below.  Every GPU that loads this library holds it until the
// process exits.  Limits and sharing rules are in include/fwix_b200.h next to the
// declaration.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "fwix_b200.h"
#include "internal.h"

static __device__ __align__(256) unsigned char g_noalloc_scratch[FWIX_NOALLOC_SCRATCH_BYTES];

namespace {

// Device address of g_noalloc_scratch for the current device, looked up once per
// device with that device current (cudaGetSymbolAddress).  The host-side symbol
// itself is not a device address and is never passed to a kernel.  The cached
// address belongs to the device's context as it was at the first call: after a
// cudaDeviceReset the module is loaded again and the array may move, so the
// entry point must not be called on a device after it has been reset.
cudaError_t scratch_address(unsigned char** out) {
  static std::mutex mu;
  static unsigned char* addr[64] = {nullptr};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    addr[dev] = (unsigned char*)p;
  }
  *out = addr[dev];
  return cudaSuccess;
}

bool radix_plan(int n, Fft1D* p) {
  if (n < 1 || n > FWIX_MAX_N) return false;
  p->n = n;
  p->npass = 0;
  int m = n;
  const int radices[6] = {8, 4, 2, 3, 5, 7};
  for (int R : radices)
    while (m % R == 0) {
      if (p->npass >= FWIX_MAX_PASS) return false;
      p->radix[p->npass++] = R;
      m /= R;
    }
  return m == 1;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Tables of the step, written into the scratch header by the device: twiddles
// exp(-2 pi i m / n), wavenumbers (PhaseShift.h:47-57), w and w^2
// (PhaseShift.h:59-70, Scatter.h:544-556) and taper weights (taper.cu:46-60).
__global__ void k_noalloc_tables(int NX, int NY, int nw, float dx, float dy, float ow, float dw, int tapx,
                                 int tapy, float2* twx, float2* twy, float* kx, float* ky, float* w2, float* w,
                                 float* tx, float* ty) {
  const int n = max(max(NX, NY), nw);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (i < NX) {
      double s, c;
      sincospi(-2.0 * (double)i / (double)NX, &s, &c);
      twx[i] = make_float2((float)c, (float)s);
      const float dk = (float)(2 * M_PI / (double)(dx * (float)NX));
      kx[i] = (float)(i <= NX / 2 ? i : i - NX) * dk;
      float t = 1.0f;
      if (i < tapx && tapx > 0) t = 0.5f * (1.0f - cosf((float)(M_PI * i / tapx)));
      else if (i >= NX - tapx) t = 0.5f * (1.0f + cosf((float)(M_PI * (i - NX + tapx) / tapx)));
      tx[i] = t;
    }
    if (i < NY) {
      double s, c;
      sincospi(-2.0 * (double)i / (double)NY, &s, &c);
      twy[i] = make_float2((float)c, (float)s);
      const float dk = (float)(2 * M_PI / (double)(dy * (float)NY));
      ky[i] = (float)(i <= NY / 2 ? i : i - NY) * dk;
      float t = 1.0f;
      if (i < tapy && tapy > 0) t = 0.5f * (1.0f - cosf((float)(M_PI * i / tapy)));
      else if (i >= NY - tapy) t = 0.5f * (1.0f + cosf((float)(M_PI * (i - NY + tapy) / tapy)));
      ty[i] = t;
    }
    if (i < nw) {
      const float f = ow + (float)i * dw;
      const float wf = (float)(2 * M_PI * f);
      w2[i] = wf * wf;
      w[i] = wf;
    }
  }
}

fwix_status fail(fwix_status s, const std::string& m) {
  fwix::set_last_error(m);
  return s;
}

fwix_status cuda_fail(cudaError_t e, const char* what) {
  return fail(FWIX_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

extern "C" fwix_status fwix_step_noalloc(const fwix_desc* desc, int kind, int iz, int dir, const void* sref,
                                         const uint8_t* labels, int64_t labels_z_stride, int64_t labels_w_stride,
                                         const void* in, void* out, int add, void* stream) {
  if (!desc || !sref || !labels || !in || !out) return fail(FWIX_ERR_INVALID, "null argument");
  const fwix_desc& q = *desc;
  if (q.nx < 1 || q.ny < 1 || q.nw < 1 || q.ns < 1 || q.nz < 1 || q.padx < 0 || q.pady < 0)
    return fail(FWIX_ERR_INVALID, "sizes must be positive and pads non-negative");
  if (q.nref < 1 || q.nref > 255) return fail(FWIX_ERR_INVALID, "nref must be in [1, 255]");
  if (q.taperx < 0 || q.tapery < 0) return fail(FWIX_ERR_INVALID, "taper widths must be non-negative");
  if (!(q.dx > 0) || !(q.dy > 0) || !(q.dz > 0)) return fail(FWIX_ERR_INVALID, "sampling must be positive");
  if (kind != FWIX_STEP_PSPI && kind != FWIX_STEP_NSPS) return fail(FWIX_ERR_INVALID, "unknown step kind");
  if (dir != FWIX_FWD && dir != FWIX_ADJ_ADD && dir != FWIX_ADJ_INPL)
    return fail(FWIX_ERR_INVALID, "unknown step direction");
  if (iz < 0 || iz >= q.nz) return fail(FWIX_ERR_INVALID, "depth index out of range");
  if ((long long)q.nx + q.padx > FWIX_MAX_N || (long long)q.ny + q.pady > FWIX_MAX_N)
    return fail(FWIX_ERR_UNSUPPORTED, "wavefield sizes must be 2^a 3^b 5^c 7^d and at most 1024");
  fwix::Dims d;
  d.nx = q.nx;
  d.ny = q.ny;
  d.NX = q.nx + q.padx;
  d.NY = q.ny + q.pady;
  d.nw = q.nw;
  d.ns = q.ns;
  d.slice = (long long)d.NX * d.NY;
  Fft1D px, py;
  if (!radix_plan(d.NX, &px) || !radix_plan(d.NY, &py))
    return fail(FWIX_ERR_UNSUPPORTED, "wavefield sizes must be 2^a 3^b 5^c 7^d and at most 1024");
  // scratch layout: tables, then the row-pass output (t1) and the column-pass output (t2)
  const size_t cap = (size_t)FWIX_NOALLOC_SCRATCH_BYTES;
  const size_t tab = align256(8 * (size_t)(d.NX + d.NY)) + align256(4 * (size_t)(2 * d.NX + 2 * d.NY + 2 * q.nw));
  // (nref + 1) wavefields of ns * nw slices follow the tables.  The factors are
  // checked one at a time against what is left, so no product below can wrap: a
  // slice is at most 1024^2 * 8 bytes, and nw, ns and nref + 1 each at most the
  // number of such units that fit.
  const size_t slice_b = (size_t)d.slice * sizeof(float2);
  const size_t room = tab < cap ? cap - tab : 0;
  const size_t units = room / slice_b;  // slices that fit after the tables
  const bool fits = (size_t)q.nw <= units && (size_t)q.ns <= units / (size_t)q.nw &&
                    (size_t)(q.nref + 1) <= units / ((size_t)q.nw * (size_t)q.ns);
  if (!fits) {
    const double need = (double)tab + (double)(q.nref + 1) * (double)q.ns * (double)q.nw * (double)slice_b;
    return fail(FWIX_ERR_UNSUPPORTED, "fwix_step_noalloc needs " + std::to_string((unsigned long long)need) +
                                          " bytes of scratch; the static scratch holds " + std::to_string(cap) +
                                          " bytes ((nref + 1) wavefields plus tables)");
  }
  d.wfld = d.slice * q.nw * q.ns;
  // one side of the step carries a single wavefield, the other nref of them
  const bool one_in = (kind == FWIX_STEP_PSPI) == (dir == FWIX_FWD);
  unsigned char* base = nullptr;
  cudaError_t e = scratch_address(&base);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(scratch)");
  cudaStream_t s = (cudaStream_t)stream;
  float2* twx = (float2*)base;
  float2* twy = twx + d.NX;
  float* ftab = (float*)(base + align256(8 * (size_t)(d.NX + d.NY)));
  float *kx = ftab, *ky = kx + d.NX, *tx = ky + d.NY, *ty = tx + d.NX, *w2 = ty + d.NY, *w = w2 + q.nw;
  const int nt = std::max(std::max(d.NX, d.NY), q.nw);
  k_noalloc_tables<<<(nt + 255) / 256, 256, 0, s>>>(d.NX, d.NY, q.nw, q.dx, q.dy, q.ow, q.dw, q.taperx, q.tapery,
                                                    twx, twy, kx, ky, w2, w, tx, ty);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "scratch tables");
  fwix::count_launch();
  fwix::SpecArgs a;
  memset(&a, 0, sizeof(a));
  a.d = d;
  a.px = px;
  a.py = py;
  a.twx = twx;
  a.twy = twy;
  a.kx = kx;
  a.ky = ky;
  a.w2 = w2;
  a.w = w;
  a.tapx = tx;
  a.tapy = ty;
  a.dz = q.dz;
  a.eps = q.eps;
  a.eps_scat = q.eps_scat;
  a.norm = 1.0f / ((float)d.NX * (float)d.NY);
  a.nterm = q.nref;
  a.in = (const float2*)in;
  a.out = (float2*)out;
  a.add = add;
  a.t1 = (float2*)(base + tab);
  a.t2 = a.t1 + (long long)(one_in ? 1 : q.nref) * d.wfld;
  a.b0 = 0;
  a.nb = (long long)q.ns * q.nw;
  a.tstride = d.wfld;
  a.sref = (const float2*)sref + (long long)iz * q.nref * q.nw;
  a.lab = labels + iz * labels_z_stride;
  a.lab_w = labels_w_stride;
  if (kind == FWIX_STEP_PSPI) {
    if (dir == FWIX_FWD) {
      if ((e = fwix::row_forward(a, fwix::W_TAPER, s)) != cudaSuccess) return cuda_fail(e, "row pass");
      if ((e = fwix::col_type_a(a, fwix::Q_PS_FWD, s)) != cudaSuccess) return cuda_fail(e, "column pass");
      if ((e = fwix::row_inverse(a, fwix::W_MASK, 0, s)) != cudaSuccess) return cuda_fail(e, "inverse row pass");
    } else {
      if ((e = fwix::row_forward(a, fwix::W_MASK, s)) != cudaSuccess) return cuda_fail(e, "row pass");
      if ((e = fwix::col_type_b(a, fwix::Q_PS_ADJ, s)) != cudaSuccess) return cuda_fail(e, "column pass");
      if ((e = fwix::row_inverse(a, fwix::W_ONE, dir == FWIX_ADJ_INPL, s)) != cudaSuccess)
        return cuda_fail(e, "inverse row pass");
    }
  } else {
    if (dir == FWIX_FWD) {
      if ((e = fwix::row_forward(a, fwix::W_MASK, s)) != cudaSuccess) return cuda_fail(e, "row pass");
      if ((e = fwix::col_type_b(a, fwix::Q_PS_FWD, s)) != cudaSuccess) return cuda_fail(e, "column pass");
      if ((e = fwix::row_inverse(a, fwix::W_ONE, 0, s)) != cudaSuccess) return cuda_fail(e, "inverse row pass");
    } else {
      if ((e = fwix::row_forward(a, fwix::W_ONE, s)) != cudaSuccess) return cuda_fail(e, "row pass");
      if ((e = fwix::col_type_a(a, fwix::Q_PS_ADJ, s)) != cudaSuccess) return cuda_fail(e, "column pass");
      if ((e = fwix::row_inverse(a, fwix::W_MASK, 0, s)) != cudaSuccess) return cuda_fail(e, "inverse row pass");
    }
  }
  return FWIX_OK;
}
