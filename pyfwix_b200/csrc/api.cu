// C ABI of libfwix_b200.so: plans, tables, one-slice operators, acquisition and
// the depth-sweep drivers (Downward / Upward, Propagator::forward, lockstep
// migration, ExtendedBorn forward / adjoint).  Host control flow only; every
// numerical operation is a kernel of spectral.cu / pointwise.cu enqueued on the
// caller's stream.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fwix_b200.h"
#include "internal.h"

using fwix::Dims;
using fwix::SpecArgs;

namespace fwix {
static std::atomic<unsigned long long> g_launches{0};
void count_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
}  // namespace fwix

namespace {

thread_local std::string g_err;

fwix_status fail(fwix_status s, const std::string& msg) {
  g_err = msg;
  return s;
}

#define FWIX_CU(call)                                                                      \
  do {                                                                                     \
    cudaError_t _e = (call);                                                               \
    if (_e != cudaSuccess)                                                                 \
      return fail(FWIX_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e));      \
  } while (0)

#define FWIX_TRY(call)              \
  do {                              \
    fwix_status _s = (call);        \
    if (_s != FWIX_OK) return _s;   \
  } while (0)

bool make_fft_plan(int n, Fft1D* p) {
  if (n < 1 || n > FWIX_MAX_N) return false;
  p->n = n;
  p->npass = 0;
  int m = n;
  const int radices[6] = {8, 4, 2, 3, 5, 7};
  for (int R : radices) {
    while (m % R == 0) {
      if (p->npass >= FWIX_MAX_PASS) return false;
      p->radix[p->npass++] = R;
      m /= R;
    }
  }
  return m == 1;
}

// Wavenumber table of propagator/src/PhaseShift.h:47-57, in the same float
// arithmetic (dk rounded to float, then ik * dk).
std::vector<float> k_table(int n, float d) {
  std::vector<float> k(n);
  const int half = n / 2;
  const float dk = (float)(2 * M_PI / (double)(d * (float)n));
  for (int i = 0; i <= half && i < n; ++i) k[i] = (float)i * dk;
  for (int i = half + 1; i < n; ++i) k[i] = (float)(i - n) * dk;
  return k;
}

// Taper weights of propagator/src/taper.cu:46-60.
std::vector<float> taper_table(int n, int tap) {
  std::vector<float> w(n, 1.0f);
  for (int i = 0; i < n; ++i) {
    if (i < tap && tap > 0)
      w[i] = 0.5f * (1.0f - cosf((float)(M_PI * i / tap)));
    else if (i >= n - tap && i < n)
      w[i] = 0.5f * (1.0f + cosf((float)(M_PI * (i - n + tap) / tap)));
  }
  return w;
}

std::vector<float2> twiddles(int n) {
  std::vector<float2> t(n);
  for (int m = 0; m < n; ++m) {
    const double a = -2.0 * M_PI * (double)m / (double)n;
    t[m] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  return t;
}

template <typename T>
cudaError_t upload(T** dst, const std::vector<T>& v) {
  *dst = nullptr;
  if (v.empty()) return cudaSuccess;
  cudaError_t e = cudaMalloc((void**)dst, v.size() * sizeof(T));
  if (e != cudaSuccess) return e;
  return cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}

}  // namespace

namespace fwix {
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace fwix

struct fwix_plan {
  fwix_desc desc;
  Dims d;
  Fft1D px, py;
  float2 *twx = nullptr, *twy = nullptr;
  float *kx = nullptr, *ky = nullptr, *w2 = nullptr, *w = nullptr, *tapx = nullptr, *tapy = nullptr;
  const float2* sref = nullptr;
  const uint8_t* labels = nullptr;
  long long lab_z = 0, lab_w = 0;
  const float2* slow = nullptr;
  const float2* den = nullptr;
  long long m_z = 0, m_w = 0;
  char* ws = nullptr;
  size_t ws_bytes = 0;
  int nterm_max = 1;
  long long chunk = 1;  // slices per launch: the intermediates of one chunk fit in L2
  bool fused = false;   // 256 x 256 slices: one-launch cluster step (fused256.cu), opt-in
  bool col_tma = true;  // column passes with TMA tiles where the plan allows (FWIX_COL_TMA=0: copies)
  int qtile = 3;        // SpecArgs::qtile bits (FWIX_QTILE): both column passes, measured fastest
  // depth steps in chunks alternating between the caller's stream and lane_s
  // (lanes = 2, set by fwix_plan_autotune), each lane with its own intermediates
  int lanes = 1;
  cudaStream_t lane_s = nullptr;
  cudaEvent_t lane_fork = nullptr, lane_join = nullptr;
  unsigned* err = nullptr;  // device word: bounded waits of the TMA passes that ran out
  float2* scat_tab = nullptr;     // scatter weights of one depth, [taylor+1][NY][NX]
  float2* rf_tab = nullptr;       // coefficients of the reflections fused into a step, [2][ny][nx]
  const float* sm_s = nullptr;    // smooth step: padded slowness [nz][NY][NX]
  const float* sm_ref = nullptr;  // smooth step: sorted real reference slownesses [nz][nref]
  float2* pcache = nullptr;   // phase-factor cache of pslots depths (fwix_plan_set_phase_cache)
  int pslots = 0;             // depth iz lives in slot iz % pslots
  std::vector<int> pslot_iz;  // depth whose current factors a slot holds, -1 for none
  int pq_nx() const { return d.NX / 2 + 1; }
  // ky extent of the phase table rounded up to even: 16-byte rows for the TMA tiles
  int pq_ny() const { return (d.NY / 2 + 2) & ~1; }
  long long pdepth() const { return (long long)desc.nref * d.nw * pq_nx() * pq_ny(); }
  float coef[5] = {1.f, 1.f / 2.f, 3.f / 8.f, 5.f / 16.f, 35.f / 128.f};  // Scatter.h:526

  size_t wbytes() const { return (size_t)d.wfld * sizeof(float2); }
  long long lane_span() const { return (long long)nterm_max * chunk * d.slice; }  // samples of one lane's t1 (or t2)
  size_t tbytes() const { return (size_t)lane_span() * lanes * sizeof(float2); }
  size_t ws_need(int cls) const {
    size_t b = 2 * tbytes();  // t1, t2 for one chunk
    if (cls >= FWIX_WS_SWEEP) b += 3 * wbytes();  // A, B, SC
    if (cls == FWIX_WS_BORN) b += (size_t)desc.nz * wbytes();  // per-level field store
    // packed backgrounds: the second unpacked background and the working level
    // field, then the per-level store packed (256-byte aligned)
    if (cls == FWIX_WS_BORN_PACKED) b += 2 * wbytes() + 256 + (size_t)desc.nz * packed_bytes();
    return b;
  }
  float2* t1() const { return (float2*)ws; }
  float2* t2() const { return (float2*)(ws + tbytes()); }
  float2* wA() const { return (float2*)(ws + 2 * tbytes()); }
  float2* wB() const { return wA() + d.wfld; }
  float2* wSC() const { return wB() + d.wfld; }
  float2* store(int iz) const { return wSC() + d.wfld * (long long)(1 + iz); }
  int pack_bits = 8;  // mantissa bits of the packed store (fwix_plan_set_pack_rate)
  size_t packed_bytes() const { return fwix::packed_bytes(2 * d.wfld, pack_bits); }
  // FWIX_WS_BORN_PACKED layout after A, B, SC: U (second background), X (working
  // level field), then the packed per-level store
  float2* wU() const { return wSC() + d.wfld; }
  float2* wX() const { return wSC() + 2 * d.wfld; }
  unsigned char* pstore(int iz) const {
    const uintptr_t base = ((uintptr_t)(wSC() + 3 * d.wfld) + 255) & ~(uintptr_t)255;
    return (unsigned char*)base + (size_t)iz * packed_bytes();
  }

  SpecArgs args(const float2* in, float2* out, int add) const {
    SpecArgs a;
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
    a.tapx = tapx;
    a.tapy = tapy;
    a.dz = desc.dz;
    a.eps = desc.eps;
    a.eps_scat = desc.eps_scat;
    for (int i = 0; i < 5; ++i) a.coef[i] = coef[i];
    a.norm = 1.0f / ((float)d.NX * (float)d.NY);
    a.nterm = 1;
    a.in = in;
    a.out = out;
    a.add = add;
    a.t1 = t1();
    a.t2 = t2();
    a.b0 = 0;
    a.nb = (long long)d.ns * d.nw;
    a.tstride = chunk * d.slice;
    a.tma = col_tma ? 1 : 0;
    a.err = err;
    a.qtile = qtile;
    return a;
  }
};

struct fwix_traces {
  int ntrace = 0;
  int nlevel = 0;
  std::vector<fwix::InjectLevel> level;
  std::vector<void*> allocs;
};

namespace {

// A trace buffer ([ntrace][nw]) may be null only when its trace set is empty.
bool no_traces(const fwix_traces* t, const void* buf) { return !t || (!buf && t->ntrace > 0); }

fwix_status need_ws(const fwix_plan* p, int cls) {
  if (!p->ws) return fail(FWIX_ERR_STATE, "workspace not bound (fwix_plan_set_workspace)");
  if (p->ws_bytes < p->ws_need(cls))
    return fail(FWIX_ERR_WORKSPACE, "workspace smaller than fwix_plan_workspace_bytes for this call");
  return FWIX_OK;
}

fwix_status need_refs(const fwix_plan* p) {
  if (!p->sref || !p->labels) return fail(FWIX_ERR_STATE, "reference slownesses not bound (fwix_plan_set_refs)");
  return FWIX_OK;
}

fwix_status need_model(const fwix_plan* p) {
  if (!p->slow || !p->den) return fail(FWIX_ERR_STATE, "background model not bound (fwix_plan_set_model)");
  return FWIX_OK;
}

fwix_status check_iz(const fwix_plan* p, int iz) {
  if (iz < 0 || iz >= p->desc.nz) return fail(FWIX_ERR_INVALID, "depth index out of range");
  return FWIX_OK;
}

fwix_status cu(cudaError_t e, const char* what) {
  if (e != cudaSuccess) return fail(FWIX_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return FWIX_OK;
}

// Runs f(args) once per chunk of slices (shot, frequency), each chunk small enough
// that its intermediates stay in L2 between the row and column passes.
template <class F>
fwix_status for_chunks(const fwix_plan* p, SpecArgs a, F f) {
  const long long B = (long long)p->d.ns * p->d.nw;
  for (long long b0 = 0; b0 < B; b0 += p->chunk) {
    a.b0 = b0;
    a.nb = std::min(p->chunk, B - b0);
    a.tstride = p->chunk * p->d.slice;
    FWIX_TRY(f(a));
  }
  return FWIX_OK;
}

// Cached phase factors of depth iz, built on the stream on first use.
fwix_status phase_factors(fwix_plan* p, int iz, SpecArgs& a, cudaStream_t s) {
  a.ptab = nullptr;
  if (!p->pcache) return FWIX_OK;
  const int slot = iz % p->pslots;
  float2* dst = p->pcache + slot * p->pdepth();
  a.ptab_nx = p->pq_nx();
  a.ptab_ny = p->pq_ny();
  if (p->pslot_iz[slot] != iz) {
    SpecArgs b = a;
    b.sref = p->sref + (long long)iz * p->desc.nref * p->d.nw;
    b.nterm = p->desc.nref;
    FWIX_TRY(cu(fwix::launch_phase_table(b, dst, s), "phase-factor cache"));
    p->pslot_iz[slot] = iz;
  }
  a.ptab = dst;
  return FWIX_OK;
}

// One depth step: PSPI (PSPI.cpp:6-103) or NSPS (NSPS.cpp:6-45).
fwix_status step_chunk(fwix_plan* p, int kind, int iz, int dir, SpecArgs a, cudaStream_t s) {
  a.sref = p->sref + (long long)iz * p->desc.nref * p->d.nw;
  a.lab = p->labels + iz * p->lab_z;
  a.lab_w = p->lab_w;
  a.nterm = p->desc.nref;
  if (p->fused && fwix::fused_step_available()) return cu(fwix::fused_step(a, kind, dir, s), "fused step");
  if (kind == FWIX_STEP_PSPI) {
    if (dir == FWIX_FWD) {
      FWIX_TRY(cu(fwix::row_forward(a, fwix::W_TAPER, s), "pspi row pass"));
      FWIX_TRY(cu(fwix::col_type_a(a, fwix::Q_PS_FWD, s), "pspi column pass"));
      FWIX_TRY(cu(fwix::row_inverse(a, fwix::W_MASK, 0, s), "pspi inverse row pass"));
    } else {
      FWIX_TRY(cu(fwix::row_forward(a, fwix::W_MASK, s), "pspi adjoint row pass"));
      FWIX_TRY(cu(fwix::col_type_b(a, fwix::Q_PS_ADJ, s), "pspi adjoint column pass"));
      FWIX_TRY(cu(fwix::row_inverse(a, fwix::W_ONE, dir == FWIX_ADJ_INPL, s), "pspi adjoint inverse row pass"));
    }
  } else {
    if (dir == FWIX_FWD) {
      FWIX_TRY(cu(fwix::row_forward(a, fwix::W_MASK, s), "nsps row pass"));
      FWIX_TRY(cu(fwix::col_type_b(a, fwix::Q_PS_FWD, s), "nsps column pass"));
      FWIX_TRY(cu(fwix::row_inverse(a, fwix::W_ONE, 0, s), "nsps inverse row pass"));
    } else {
      FWIX_TRY(cu(fwix::row_forward(a, fwix::W_ONE, s), "nsps adjoint row pass"));
      FWIX_TRY(cu(fwix::col_type_a(a, fwix::Q_PS_ADJ, s), "nsps adjoint column pass"));
      FWIX_TRY(cu(fwix::row_inverse(a, fwix::W_MASK, 0, s), "nsps adjoint inverse row pass"));
    }
  }
  return FWIX_OK;
}

// Reflections taken into a depth step (SpecArgs::rf_at): at 1 the step's input is
// in + tab[0] f1, at 2 its output gains tab[0] f1 + tab[1] f2.
struct Refl {
  int at;
  const float2* tab;
  const float2* f1;
  const float2* f2;
};

fwix_status do_step(fwix_plan* p, int kind, int iz, int dir, const float2* in, float2* out, int add,
                    cudaStream_t s, const float2* in2 = nullptr, const float2* ic_bg = nullptr,
                    float* ic_img = nullptr, const Refl* rf = nullptr) {
  SpecArgs a0 = p->args(in, out, add);
  a0.in2 = in2;  // the step of in + in2 (linear: one step instead of two)
  // image epilogue of the last (inverse row) pass: ic_img += Re sum conj(ic_bg) out
  a0.ic_bg = ic_bg;
  a0.ic_img = ic_img;
  if (rf) {
    if (p->fused) return fail(FWIX_ERR_STATE, "reflections cannot be fused into the cluster step");
    a0.rf_at = rf->at;
    a0.rf_tab = rf->tab;
    a0.rf_f1 = rf->f1;
    a0.rf_f2 = rf->f2;
  }
  FWIX_TRY(phase_factors(p, iz, a0, s));
  if (p->lanes < 2 || p->fused)
    return for_chunks(p, a0, [&](const SpecArgs& a) { return step_chunk(p, kind, iz, dir, a, s); });
  // Two lanes: chunks alternate between `s` and the plan's lane stream, forked
  // from and joined back into `s` with events, each lane with its own half of the
  // intermediates; one chunk's column pass overlaps the next chunk's row pass.
  FWIX_CU(cudaEventRecord(p->lane_fork, s));
  FWIX_CU(cudaStreamWaitEvent(p->lane_s, p->lane_fork, 0));
  const long long B = (long long)p->d.ns * p->d.nw;
  fwix_status st = FWIX_OK;
  int k = 0;
  for (long long b0 = 0; b0 < B && st == FWIX_OK; b0 += p->chunk, ++k) {
    SpecArgs a = a0;
    a.b0 = b0;
    a.nb = std::min(p->chunk, B - b0);
    a.tstride = p->chunk * p->d.slice;
    const int lane = k & 1;
    a.t1 = p->t1() + lane * p->lane_span();
    a.t2 = p->t2() + lane * p->lane_span();
    st = step_chunk(p, kind, iz, dir, a, lane ? p->lane_s : s);
  }
  // `s` waits for the lane also after a failure
  const cudaError_t e1 = cudaEventRecord(p->lane_join, p->lane_s);
  const cudaError_t e2 = e1 == cudaSuccess ? cudaStreamWaitEvent(s, p->lane_join, 0) : e1;
  if (st != FWIX_OK) return st;
  return cu(e2, "lane join");
}

fwix_status need_smooth(const fwix_plan* p) {
  if (!p->sm_s || !p->sm_ref || !p->sref)
    return fail(FWIX_ERR_STATE, "smooth-step slowness / references not bound (fwix_plan_set_smooth, fwix_plan_set_refs)");
  return FWIX_OK;
}

// Smooth PSPI step (no reference counterpart): forward
//   out (+)= sum_r w_r(s) SS_r F^-1(P_r F(taper in)),
// its exact transpose, and the derivative with respect to the local slowness
//   out (+)= sum_r (w_r' - i w dz w_r) SS_r F^-1(P_r F(taper in)).
// mode kSmoothPair: FWD into a.out and DERIV into a.out2 from one forward row pass
// and one column pass (the inverse row pass of the register-resident plans sums
// each term with both weights; other lengths run two inverse row passes).
constexpr int kSmoothPair = -1;

fwix_status smooth_chunk(fwix_plan* p, int iz, int mode, SpecArgs a, cudaStream_t s) {
  a.sref = p->sref + (long long)iz * p->desc.nref * p->d.nw;
  a.sm_s = p->sm_s + (long long)iz * p->d.slice;
  a.sm_ref = p->sm_ref + (long long)iz * p->desc.nref;
  a.sm_n = p->desc.nref;
  a.nterm = p->desc.nref;
  if (mode == FWIX_SMOOTH_ADJ) {
    FWIX_TRY(cu(fwix::row_forward(a, fwix::W_SMOOTH_CONJ, s), "smooth adjoint row pass"));
    FWIX_TRY(cu(fwix::col_type_b(a, fwix::Q_PS_ADJ, s), "smooth adjoint column pass"));
    return cu(fwix::row_inverse(a, fwix::W_ONE, 1, s), "smooth adjoint inverse row pass");
  }
  FWIX_TRY(cu(fwix::row_forward(a, fwix::W_TAPER, s), "smooth row pass"));
  FWIX_TRY(cu(fwix::col_type_a(a, fwix::Q_PS_FWD, s), "smooth column pass"));
  if (mode == kSmoothPair) {
    if (fwix::fast_length(p->d.NX))
      return cu(fwix::row_inverse(a, fwix::W_SMOOTH_PAIR, 0, s), "smooth pair inverse row pass");
    FWIX_TRY(cu(fwix::row_inverse(a, fwix::W_SMOOTH, 0, s), "smooth inverse row pass"));
    a.out = a.out2;
    return cu(fwix::row_inverse(a, fwix::W_SMOOTH_DERIV, 0, s), "smooth derivative inverse row pass");
  }
  return cu(fwix::row_inverse(a, mode == FWIX_SMOOTH_DERIV ? fwix::W_SMOOTH_DERIV : fwix::W_SMOOTH, 0, s),
            "smooth inverse row pass");
}

SpecArgs scatter_args(const fwix_plan* p, int iz, const float2* in, float2* out, int add) {
  SpecArgs a = p->args(in, out, add);
  a.slow = p->slow + iz * p->m_z;
  a.slow_w = p->m_w;
  a.nterm = p->desc.taylor + 1;
  return a;
}

// Scatter::cu_forward / cu_adjoint (Scatter.cpp:76-133).  With image != NULL the
// forward input is the imaging-condition product bg * image (ImagingCondition fwd,
// imaging_condition.cu:9-55) formed inside the first pass.
fwix_status scatter_chunk(int adjoint, const float2* image, long long img_w, SpecArgs a, cudaStream_t s) {
  if (!adjoint) {
    a.image = image;
    a.img_w = img_w;
    FWIX_TRY(cu(fwix::row_forward(a, image ? fwix::W_IC : fwix::W_ONE, s), "scatter row pass"));
    FWIX_TRY(cu(fwix::col_type_a(a, fwix::Q_KPOW, s), "scatter column pass"));
    FWIX_TRY(cu(fwix::row_inverse(a, fwix::W_SCAT, 0, s), "scatter inverse row pass"));
  } else {
    FWIX_TRY(cu(fwix::row_forward(a, fwix::W_SCAT_CONJ, s), "scatter adjoint row pass"));
    FWIX_TRY(cu(fwix::col_type_b(a, fwix::Q_KPOW, s), "scatter adjoint column pass"));
    FWIX_TRY(cu(fwix::row_inverse(a, a.direct_mode ? fwix::W_ONE_DIRECT : fwix::W_ONE, 0, s),
                "scatter adjoint inverse row pass"));
  }
  return FWIX_OK;
}

fwix_status do_scatter(fwix_plan* p, int iz, int adjoint, const float2* in, float2* out, int add,
                       const float2* image, long long img_w, cudaStream_t s) {
  SpecArgs a0 = scatter_args(p, iz, in, out, add);
  if (p->m_w == 0) {
    // one slowness for every frequency: the powers of s~ are a per-cell table
    FWIX_TRY(cu(fwix::launch_scat_table(a0, p->scat_tab, s), "scatter weights"));
    a0.scat_tab = p->scat_tab;
  }
  if (adjoint && p->desc.taylor >= 1 && fwix::fast_length(p->d.NX) && fwix::fast_length(p->d.NY)) {
    // the zeroth term's filter is the identity: conj(W_0) d is added by the inverse
    // row pass, and only orders 1 .. taylor go through the transforms.  (The
    // forward keeps the zeroth term in the transforms: measured on B200, adding
    // W_0 u in its inverse row pass, which then also reads the background and the
    // image, was slower than transforming the term.)
    a0.term0 = 1;
    a0.nterm = p->desc.taylor;
    a0.direct = in;
    a0.direct_mode = 2;
  }
  return for_chunks(p, a0, [&](const SpecArgs& a) { return scatter_chunk(adjoint, image, img_w, a, s); });
}

int lower_iz(const fwix_plan* p, int iz) { return iz < p->desc.nz - 1 ? iz + 1 : iz; }

fwix_status do_reflect(fwix_plan* p, int iz, int adjoint, const float2* in, float2* out, int add,
                       cudaStream_t s) {
  const int z1 = lower_iz(p, iz);
  return cu(fwix::launch_reflect(p->d, adjoint, p->slow + iz * p->m_z, p->slow + z1 * p->m_z,
                                 p->den + iz * p->m_z, p->den + z1 * p->m_z, p->m_w, in, out, add, s),
            "reflect");
}

const fwix::InjectLevel* level_of(const fwix_traces* tr, int iz) {
  if (!tr || iz < 0 || iz >= tr->nlevel) return nullptr;
  return &tr->level[iz];
}

fwix_status do_inject(fwix_plan* p, const fwix_traces* tr, int iz, const float2* traces, float2* wfld,
                      cudaStream_t s) {
  const fwix::InjectLevel* L = level_of(tr, iz);
  if (!L) return FWIX_OK;
  return cu(fwix::launch_inject(p->d, *L, traces, wfld, s), "inject");
}

fwix_status do_record(fwix_plan* p, const fwix_traces* tr, int iz, const float2* wfld, float2* traces,
                      cudaStream_t s) {
  const fwix::InjectLevel* L = level_of(tr, iz);
  if (!L) return FWIX_OK;
  return cu(fwix::launch_record(p->d, *L, wfld, traces, s), "record");
}

long long mslice(const fwix_plan* p) { return (long long)p->d.nw * p->d.ny * p->d.nx; }

// =============================================================================
// Background wavefields of fwix_born: [nz] full fields, or [nz] packed ones each
// unpacked into `slot` when a depth other than the one it holds is asked for.
struct BgSrc {
  const float2* full = nullptr;
  const unsigned char* packed = nullptr;
  float2* slot = nullptr;
  int held = -1;
  fwix_status get(const fwix_plan* p, int iz, cudaStream_t s, const float2** out) {
    if (full) {
      *out = full + (long long)iz * p->d.wfld;
      return FWIX_OK;
    }
    if (held != iz) {
      FWIX_TRY(cu(fwix::launch_unpack(p->pack_bits, 2 * p->d.wfld, packed + (size_t)iz * p->packed_bytes(),
                                      (float*)slot, s),
                  "unpack background"));
      held = iz;
    }
    *out = slot;
    return FWIX_OK;
  }
};

// Per-level fields of the Born recursions (dD_iz forward, zeta_iz adjoint), read
// back in the opposite sweep for the reflections: [nz] full fields in the
// workspace, or, with packed backgrounds, one working field (the recursion runs
// in place in it) whose every level is kept packed and unpacked when read back.
struct LevelStore {
  fwix_plan* p;
  bool packed;
  float2* field(int iz) const { return packed ? p->wX() : p->store(iz); }
  fwix_status keep(int iz, cudaStream_t s) const {
    if (!packed) return FWIX_OK;
    return cu(fwix::launch_pack(p->pack_bits, 2 * p->d.wfld, (const float*)p->wX(), p->pstore(iz), s),
              "pack level field");
  }
  fwix_status get(int iz, cudaStream_t s, const float2** out) const {
    if (!packed) {
      *out = p->store(iz);
      return FWIX_OK;
    }
    FWIX_TRY(cu(fwix::launch_unpack(p->pack_bits, 2 * p->d.wfld, p->pstore(iz), (float*)p->wX(), s),
                "unpack level field"));
    *out = p->wX();
    return FWIX_OK;
  }
};

// ExtendedBorn::forward / adjoint (ExtendedBorn.cpp:80-453) on backgrounds D, U.
fwix_status born_body(fwix_plan* p, int adjoint, const fwix_traces* rec, BgSrc& D, BgSrc& U, float2* ds,
                      float2* dr, long long mw, float2* data, int add, cudaStream_t s, bool packed = false) {
  const LevelStore Lv{p, packed};
  const int nz = p->desc.nz, k = p->desc.step_kind;
  const long long plane = (long long)p->d.ny * p->d.nx;
  const long long M = mw ? mslice(p) : plane;
  float2* A = p->wA();
  const size_t wb = p->wbytes();
  // The reference runs four sweeps each way (ExtendedBorn.cpp:152-453), every
  // scattered source propagated by a step of its own.  All operators are linear,
  // so sources that feed the same recursion are summed before one step:
  // step(A) + step(scat) = step(A + scat).  The forward keeps one downward and one
  // upward recursion, the adjoint one downward and one upward; the results equal
  // the four-sweep operators up to float rounding.
  float2* SC = p->wSC();
  const bool pspi = k == FWIX_STEP_PSPI;
  // With a model and perturbation shared by every frequency the per-level
  // reflections ride in the depth steps' row passes (a per-cell coefficient table
  // instead of two read-modify-write passes over the field), and the adjoint's two
  // frequency sums of a level share one pass.  The cluster step has no such
  // epilogue: it keeps the separate passes.
  const bool frf = p->m_w == 0 && mw == 0 && !p->fused;
  if (!adjoint) {
    if (!add && rec->ntrace > 0) FWIX_CU(cudaMemsetAsync(data, 0, (size_t)rec->ntrace * p->d.nw * sizeof(float2), s));
    // down scattering (ExtendedBorn.cpp:152-178): store[iz] = dD_iz, the field
    // recorded at iz; dD_iz+1 = S_iz(dD_iz + Scat_iz(bg_down_iz * ds_iz))
    FWIX_CU(cudaMemsetAsync(Lv.field(0), 0, wb, s));
    for (int iz = 0; iz < nz; ++iz) {
      FWIX_TRY(do_record(p, rec, iz, Lv.field(iz), data, s));
      FWIX_TRY(Lv.keep(iz, s));
      if (iz == nz - 1) break;
      const float2* bd;
      FWIX_TRY(D.get(p, iz, s, &bd));
      FWIX_TRY(do_scatter(p, iz, 0, bd, SC, 0, ds + iz * M, mw, s));
      FWIX_TRY(do_step(p, k, iz, FWIX_FWD, Lv.field(iz), Lv.field(iz + 1), 0, s, SC));
    }
    // one upward recursion for the reflected down-scattered field (:210-238), the
    // up scattering (:282-311) and the back scattering (:352-389):
    //   Z_iz = S_iz(Z_iz+1 + Scat_iz(bg_up_iz+1 * ds_iz+1)) + R_iz dD_iz + bg_down_iz * dR_iz
    FWIX_CU(cudaMemsetAsync(A, 0, wb, s));
    for (int iz = nz - 1; iz >= 0; --iz) {
      const int z1 = lower_iz(p, iz);
      if (iz < nz - 1) {
        const float2* bu;
        FWIX_TRY(U.get(p, iz + 1, s, &bu));
        FWIX_TRY(do_scatter(p, iz, 0, bu, SC, 0, ds + (iz + 1) * M, mw, s));
        if (frf) {
          // both reflections of this level added by the step's inverse row pass:
          // Z_iz = S_iz(Z_iz+1 + scat) + r dD_iz + dr bg_down_iz
          const float2 *dz, *bd;
          FWIX_TRY(Lv.get(iz, s, &dz));
          FWIX_TRY(D.get(p, iz, s, &bd));
          FWIX_TRY(cu(fwix::launch_refl_table(p->d, 0, p->slow + iz * p->m_z, p->slow + z1 * p->m_z,
                                              p->den + iz * p->m_z, p->den + z1 * p->m_z, ds + iz * M,
                                              ds + z1 * M, dr + iz * M, dr + z1 * M, p->rf_tab, s),
                      "reflection coefficients"));
          const Refl rf{2, p->rf_tab, dz, bd};
          FWIX_TRY(do_step(p, k, iz, FWIX_FWD, A, A, 0, s, SC, nullptr, nullptr, &rf));
          FWIX_TRY(do_record(p, rec, iz, A, data, s));
          continue;
        }
        FWIX_TRY(do_step(p, k, iz, FWIX_FWD, A, A, 0, s, SC));
      }
      const float2* dz;
      FWIX_TRY(Lv.get(iz, s, &dz));
      FWIX_TRY(do_reflect(p, iz, 0, dz, A, 1, s));
      // The bottom level reflects against a copy of itself (LinReflect.h:30-41):
      // its linearised coefficients cancel exactly (FP32 would leave only their
      // rounding), so nothing is added there, forward or adjoint.
      if (z1 != iz) {
        const float2* bd;
        FWIX_TRY(D.get(p, iz, s, &bd));
        FWIX_TRY(cu(fwix::launch_lin_reflect_ic(p->d, 0, p->slow + iz * p->m_z, p->slow + z1 * p->m_z,
                                                p->den + iz * p->m_z, p->den + z1 * p->m_z, p->m_w, ds + iz * M,
                                                ds + z1 * M, dr + iz * M, dr + z1 * M, mw, bd, A, 1, s),
                    "linearised reflection"));
      }
      FWIX_TRY(do_record(p, rec, iz, A, data, s));
    }
    return FWIX_OK;
  }
  if (!add) {
    FWIX_CU(cudaMemsetAsync(ds, 0, (size_t)nz * M * sizeof(float2), s));
    FWIX_CU(cudaMemsetAsync(dr, 0, (size_t)nz * M * sizeof(float2), s));
  }
  // The scattering adjoints step with the add-version adjoint (no taper,
  // Scattering.cpp:54-61), the recursions with the in-place adjoint (taper last,
  // PSPI.cpp:85-103); for PSPI the second is the taper of the first, so one
  // add-version step serves both.  (NSPS has no taper: the two coincide.)
  SpecArgs ta = p->args(nullptr, nullptr, 0);
  auto taper_into = [&](const float2* u, float2* out) {
    return cu(fwix::launch_taper(ta, u, out, 0, s), "taper");
  };
  // downward: zeta_iz = Rec_iz^H d + S_iz-1^H zeta_iz-1 (the adjoint of the upward
  // recursion), kept in store[iz]; it feeds the up-scattering adjoint (:313-349)
  // and the back-scattering adjoint (:391-453), which needs no steps of its own
  FWIX_CU(cudaMemsetAsync(Lv.field(0), 0, wb, s));
  for (int iz = 0; iz < nz; ++iz) {
    const int z1 = lower_iz(p, iz);
    float2* cur = Lv.field(iz);
    const float2* ic_bu = nullptr;  // imaging-condition pair summed by the reflection pass below
    if (iz > 0) {
      // (with the packed store the previous level and this one are the same
      // working field: the step reads it before the taper or the step writes it)
      if (pspi) {
        FWIX_TRY(do_step(p, k, iz - 1, FWIX_ADJ_ADD, Lv.field(iz - 1), SC, 0, s));
        FWIX_TRY(taper_into(SC, cur));
        FWIX_TRY(do_scatter(p, iz - 1, 1, SC, SC, 0, nullptr, 0, s));
      } else {
        FWIX_TRY(do_step(p, k, iz - 1, FWIX_ADJ_ADD, Lv.field(iz - 1), cur, 0, s));
        FWIX_TRY(do_scatter(p, iz - 1, 1, cur, SC, 0, nullptr, 0, s));
      }
      const float2* bu;
      FWIX_TRY(U.get(p, iz, s, &bu));
      if (frf && z1 != iz)
        ic_bu = bu;
      else
        FWIX_TRY(cu(fwix::launch_ic_adj(p->d, bu, SC, ds + iz * M, mw, 1, s), "imaging adjoint"));
    }
    FWIX_TRY(do_inject(p, rec, iz, data, cur, s));
    if (z1 != iz) {  // nothing at the bottom level (see the forward)
      const float2* bd;
      FWIX_TRY(D.get(p, iz, s, &bd));
      FWIX_TRY(cu(fwix::launch_lin_reflect_ic(p->d, 1, p->slow + iz * p->m_z, p->slow + z1 * p->m_z,
                                              p->den + iz * p->m_z, p->den + z1 * p->m_z, p->m_w, ds + iz * M,
                                              ds + z1 * M, dr + iz * M, dr + z1 * M, mw, bd, cur, 1, s, ic_bu,
                                              ic_bu ? SC : nullptr),
                  "linearised reflection adjoint"));
    }
    FWIX_TRY(Lv.keep(iz, s));
  }
  // upward: eta_iz = Rec_iz^H d + conj(R_iz) zeta_iz + S_iz^H eta_iz+1, the adjoint of
  // the down-scattering recursion (reflected :240-280 and direct :180-208)
  FWIX_CU(cudaMemsetAsync(A, 0, wb, s));
  const float2* pend = nullptr;  // (fused) level field whose reflection the next step takes in
  for (int iz = nz - 1; iz >= 0; --iz) {
    if (iz < nz - 1) {
      const Refl rf{1, p->rf_tab, pend, nullptr};
      const Refl* rfp = pend ? &rf : nullptr;
      if (pspi) {
        FWIX_TRY(do_step(p, k, iz, FWIX_ADJ_ADD, A, SC, 0, s, nullptr, nullptr, nullptr, rfp));
        FWIX_TRY(taper_into(SC, A));
        FWIX_TRY(do_scatter(p, iz, 1, SC, SC, 0, nullptr, 0, s));
      } else {
        FWIX_TRY(do_step(p, k, iz, FWIX_ADJ_ADD, A, A, 0, s, nullptr, nullptr, nullptr, rfp));
        FWIX_TRY(do_scatter(p, iz, 1, A, SC, 0, nullptr, 0, s));
      }
      pend = nullptr;
      const float2* bd;
      FWIX_TRY(D.get(p, iz, s, &bd));
      FWIX_TRY(cu(fwix::launch_ic_adj(p->d, bd, SC, ds + iz * M, mw, 1, s), "imaging adjoint"));
    }
    // eta_0 feeds nothing: the top level's reflection and injection are not formed
    if (iz == 0) break;
    const float2* zz;
    FWIX_TRY(Lv.get(iz, s, &zz));
    const int z1 = lower_iz(p, iz);
    if (frf) {
      // conj(R_iz) zeta_iz is only read by the next step: it enters as that step's
      // input (the bottom level reflects against itself, r = 0, and adds nothing)
      if (z1 != iz) {
        FWIX_TRY(cu(fwix::launch_refl_table(p->d, 1, p->slow + iz * p->m_z, p->slow + z1 * p->m_z,
                                            p->den + iz * p->m_z, p->den + z1 * p->m_z, nullptr, nullptr,
                                            nullptr, nullptr, p->rf_tab, s),
                    "reflection coefficients"));
        pend = zz;
      }
    } else {
      FWIX_TRY(do_reflect(p, iz, 1, zz, A, 1, s));
    }
    FWIX_TRY(do_inject(p, rec, iz, data, A, s));
  }
  return FWIX_OK;
}

}  // namespace

extern "C" {

const char* fwix_last_error(void) { return g_err.c_str(); }

int fwix_version(void) { return 100; }

uint64_t fwix_launch_count(void) { return fwix::g_launches.load(std::memory_order_relaxed); }

fwix_status fwix_plan_create(const fwix_desc* desc, fwix_plan** out) {
  if (!desc || !out) return fail(FWIX_ERR_INVALID, "null descriptor or output");
  *out = nullptr;
  const fwix_desc& q = *desc;
  if (q.nx < 1 || q.ny < 1 || q.nw < 1 || q.ns < 1 || q.nz < 1 || q.padx < 0 || q.pady < 0)
    return fail(FWIX_ERR_INVALID, "sizes must be positive and pads non-negative");
  if (q.nref < 1 || q.nref > 255) return fail(FWIX_ERR_INVALID, "nref must be in [1, 255]");
  if (q.taylor < 0 || q.taylor > 4) return fail(FWIX_ERR_INVALID, "taylor must be in [0, 4]");
  if (q.taperx < 0 || q.tapery < 0) return fail(FWIX_ERR_INVALID, "taper widths must be non-negative");
  if (!(q.dx > 0) || !(q.dy > 0) || !(q.dz > 0)) return fail(FWIX_ERR_INVALID, "sampling must be positive");
  if (q.step_kind != FWIX_STEP_PSPI && q.step_kind != FWIX_STEP_NSPS)
    return fail(FWIX_ERR_INVALID, "unknown step kind");
  fwix_plan* p = new fwix_plan();
  p->desc = q;
  p->d.nx = q.nx;
  p->d.ny = q.ny;
  p->d.NX = q.nx + q.padx;
  p->d.NY = q.ny + q.pady;
  p->d.nw = q.nw;
  p->d.ns = q.ns;
  p->d.slice = (long long)p->d.NX * p->d.NY;
  p->d.wfld = p->d.slice * q.nw * q.ns;
  if (!make_fft_plan(p->d.NX, &p->px) || !make_fft_plan(p->d.NY, &p->py)) {
    delete p;
    return fail(FWIX_ERR_UNSUPPORTED, "wavefield sizes must be 2^a 3^b 5^c 7^d and at most 1024");
  }
  p->nterm_max = std::max(q.nref, q.taylor + 1);
  {
    // One launch covers every slice unless FWIX_CHUNK_SLICES asks for chunks (smaller
    // launches keep the intermediates in L2 but leave SMs idle at these sizes).
    long long c = (long long)q.ns * q.nw;
    if (const char* env = getenv("FWIX_CHUNK_SLICES")) c = atoll(env);
    p->chunk = std::max(1LL, std::min(c, (long long)q.ns * q.nw));
  }
  {
    // The one-launch cluster step is opt-in (FWIX_FUSED=1): measured on B200 it
    // is slower than the three-launch step at these sizes.
    const char* env = getenv("FWIX_FUSED");
    p->fused = p->d.NX == 256 && p->d.NY == 256 && env && env[0] == '1';
    const char* tma = getenv("FWIX_COL_TMA");
    p->col_tma = !(tma && tma[0] == '0');
    if (const char* q = getenv("FWIX_QTILE")) p->qtile = atoi(q) & 3;
  }
  std::vector<float> w2(q.nw), w(q.nw);
  for (int i = 0; i < q.nw; ++i) {
    // PhaseShift.h:59-70 and Scatter.h:544-556 (float f, then 2 pi f in double)
    float f = q.ow + (float)i * q.dw;
    float wf = (float)(2 * M_PI * f);
    w2[i] = wf * wf;
    w[i] = (float)(2 * M_PI * f);
  }
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = upload(&p->twx, twiddles(p->d.NX));
  if (e == cudaSuccess) e = upload(&p->twy, twiddles(p->d.NY));
  if (e == cudaSuccess) e = upload(&p->kx, k_table(p->d.NX, q.dx));
  if (e == cudaSuccess) e = upload(&p->ky, k_table(p->d.NY, q.dy));
  if (e == cudaSuccess) e = upload(&p->w2, w2);
  if (e == cudaSuccess) e = upload(&p->w, w);
  if (e == cudaSuccess) e = upload(&p->tapx, taper_table(p->d.NX, q.taperx));
  if (e == cudaSuccess) e = upload(&p->tapy, taper_table(p->d.NY, q.tapery));
  if (e == cudaSuccess)
    e = cudaMalloc((void**)&p->scat_tab, (size_t)(q.taylor + 1) * p->d.slice * sizeof(float2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&p->rf_tab, (size_t)2 * p->d.nx * p->d.ny * sizeof(float2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&p->err, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(p->err, 0, sizeof(unsigned));
  if (e != cudaSuccess) {
    fwix_plan_destroy(p);
    return fail(FWIX_ERR_CUDA, std::string("plan tables: ") + cudaGetErrorString(e));
  }
  *out = p;
  return FWIX_OK;
}

fwix_status fwix_plan_destroy(fwix_plan* p) {
  if (!p) return FWIX_OK;
  void* ptrs[] = {p->twx, p->twy, p->kx, p->ky, p->w2, p->w, p->tapx, p->tapy, p->scat_tab, p->rf_tab, p->err};
  for (void* v : ptrs)
    if (v) cudaFree(v);
  if (p->lane_fork) cudaEventDestroy(p->lane_fork);
  if (p->lane_join) cudaEventDestroy(p->lane_join);
  if (p->lane_s) cudaStreamDestroy(p->lane_s);
  delete p;
  return FWIX_OK;
}

size_t fwix_plan_workspace_bytes(const fwix_plan* p, int cls) { return p ? p->ws_need(cls) : 0; }

uint64_t fwix_plan_wait_timeouts(const fwix_plan* p) {
  if (!p || !p->err) return 0;
  unsigned v = 0;
  if (cudaMemcpy(&v, p->err, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
  return v;
}

fwix_status fwix_plan_set_workspace(fwix_plan* p, void* ptr, size_t bytes) {
  if (!p) return fail(FWIX_ERR_INVALID, "null plan");
  if (((uintptr_t)ptr) % 16 != 0) return fail(FWIX_ERR_INVALID, "workspace must be 16-byte aligned");
  p->ws = (char*)ptr;
  p->ws_bytes = bytes;
  return FWIX_OK;
}

size_t fwix_plan_phase_cache_bytes(const fwix_plan* p) {
  return p ? (size_t)p->desc.nz * (size_t)p->pdepth() * sizeof(float2) : 0;
}

fwix_status fwix_plan_set_phase_cache(fwix_plan* p, void* ptr, size_t bytes) {
  if (!p) return fail(FWIX_ERR_INVALID, "null plan");
  const size_t depth_bytes = (size_t)p->pdepth() * sizeof(float2);
  if (ptr && bytes < depth_bytes)
    return fail(FWIX_ERR_WORKSPACE, "phase cache smaller than one depth (fwix_plan_phase_cache_bytes / nz)");
  if (((uintptr_t)ptr) % 16 != 0) return fail(FWIX_ERR_INVALID, "phase cache must be 16-byte aligned");
  p->pcache = (float2*)ptr;
  p->pslots = ptr ? (int)std::min<size_t>((size_t)p->desc.nz, bytes / depth_bytes) : 0;
  p->pslot_iz.assign(std::max(p->pslots, 1), -1);
  return FWIX_OK;
}

fwix_status fwix_plan_set_refs(fwix_plan* p, const void* sref, const uint8_t* labels, int64_t z_stride,
                               int64_t w_stride) {
  if (!p || !sref || !labels) return fail(FWIX_ERR_INVALID, "null plan, refs or labels");
  p->pslot_iz.assign(std::max(p->pslots, 1), -1);  // cached factors belong to the previous references
  p->sref = (const float2*)sref;
  p->labels = labels;
  p->lab_z = z_stride;
  p->lab_w = w_stride;
  return FWIX_OK;
}

fwix_status fwix_plan_set_model(fwix_plan* p, const void* slow, const void* den, int64_t z_stride,
                                int64_t w_stride) {
  if (!p || !slow || !den) return fail(FWIX_ERR_INVALID, "null plan or model");
  p->slow = (const float2*)slow;
  p->den = (const float2*)den;
  p->m_z = z_stride;
  p->m_w = w_stride;
  return FWIX_OK;
}

fwix_status fwix_fft2d(fwix_plan* p, int inverse, const void* in, void* out, int add, void* stream) {
  if (!p || !in || !out) return fail(FWIX_ERR_INVALID, "null argument");
  FWIX_TRY(need_ws(p, FWIX_WS_STEP));
  cudaStream_t s = (cudaStream_t)stream;
  SpecArgs a0 = p->args((const float2*)in, (float2*)out, add);
  const float sc = 1.0f / sqrtf((float)p->d.NX * (float)p->d.NY);
  return for_chunks(p, a0, [&](const SpecArgs& a) -> fwix_status {
    const long long off = a.b0 * p->d.slice;
    if (!inverse) {
      FWIX_TRY(cu(fwix::row_forward(a, fwix::W_ONE, s), "fft row pass"));
      FWIX_TRY(cu(fwix::col_fft(a, 0, p->t1(), (float2*)out + off, add, sc, s), "fft column pass"));
    } else {
      FWIX_TRY(cu(fwix::col_fft(a, 1, (const float2*)in + off, p->t2(), 0, sc, s), "ifft column pass"));
      FWIX_TRY(cu(fwix::row_inverse(a, fwix::W_ONE, 0, s), "ifft row pass"));
    }
    return FWIX_OK;
  });
}

fwix_status fwix_phase_shift(fwix_plan* p, int mode, const void* sref_w, const void* in, void* out, int add,
                             void* stream) {
  if (!p || !sref_w || !in || !out) return fail(FWIX_ERR_INVALID, "null argument");
  int q = mode == FWIX_PS_FWD ? fwix::Q_PS_FWD : mode == FWIX_PS_ADJ ? fwix::Q_PS_ADJ
        : mode == FWIX_PS_INV ? fwix::Q_PS_INV : -1;
  if (q < 0) return fail(FWIX_ERR_INVALID, "unknown phase-shift mode");
  SpecArgs a = p->args((const float2*)in, (float2*)out, add);
  return cu(fwix::launch_phase_shift(a, q, (const float2*)sref_w, (const float2*)in, (float2*)out, add,
                                     (cudaStream_t)stream),
            "phase shift");
}

fwix_status fwix_select(fwix_plan* p, int iz, int value, const void* in, void* out, int add, void* stream) {
  if (!p || !in || !out) return fail(FWIX_ERR_INVALID, "null argument");
  FWIX_TRY(need_refs(p));
  FWIX_TRY(check_iz(p, iz));
  SpecArgs a = p->args((const float2*)in, (float2*)out, add);
  a.lab = p->labels + iz * p->lab_z;
  a.lab_w = p->lab_w;
  return cu(fwix::launch_select(a, value, (const float2*)in, (float2*)out, add, (cudaStream_t)stream), "select");
}

fwix_status fwix_taper(fwix_plan* p, const void* in, void* out, int add, void* stream) {
  if (!p || !in || !out) return fail(FWIX_ERR_INVALID, "null argument");
  SpecArgs a = p->args((const float2*)in, (float2*)out, add);
  return cu(fwix::launch_taper(a, (const float2*)in, (float2*)out, add, (cudaStream_t)stream), "taper");
}

fwix_status fwix_step(fwix_plan* p, int kind, int iz, int dir, const void* in, void* out, int add,
                      void* stream) {
  if (!p || !in || !out) return fail(FWIX_ERR_INVALID, "null argument");
  if (kind != FWIX_STEP_PSPI && kind != FWIX_STEP_NSPS) return fail(FWIX_ERR_INVALID, "unknown step kind");
  if (dir != FWIX_FWD && dir != FWIX_ADJ_ADD && dir != FWIX_ADJ_INPL)
    return fail(FWIX_ERR_INVALID, "unknown step direction");
  FWIX_TRY(need_refs(p));
  FWIX_TRY(need_ws(p, FWIX_WS_STEP));
  FWIX_TRY(check_iz(p, iz));
  return do_step(p, kind, iz, dir, (const float2*)in, (float2*)out, add, (cudaStream_t)stream);
}

fwix_status fwix_plan_set_smooth(fwix_plan* p, const float* slow_pad, const float* sref_real) {
  if (!p) return fail(FWIX_ERR_INVALID, "null plan");
  p->sm_s = slow_pad;
  p->sm_ref = sref_real;
  return FWIX_OK;
}

fwix_status fwix_smooth_step(fwix_plan* p, int iz, int mode, const void* in, void* out, int add, void* stream) {
  if (!p || !in || !out) return fail(FWIX_ERR_INVALID, "null argument");
  if (mode != FWIX_SMOOTH_FWD && mode != FWIX_SMOOTH_ADJ && mode != FWIX_SMOOTH_DERIV)
    return fail(FWIX_ERR_INVALID, "unknown smooth-step mode");
  FWIX_TRY(need_smooth(p));
  FWIX_TRY(need_ws(p, FWIX_WS_STEP));
  FWIX_TRY(check_iz(p, iz));
  cudaStream_t s = (cudaStream_t)stream;
  SpecArgs a0 = p->args((const float2*)in, (float2*)out, add);
  FWIX_TRY(phase_factors(p, iz, a0, s));
  return for_chunks(p, a0, [&](const SpecArgs& a) { return smooth_chunk(p, iz, mode, a, s); });
}

fwix_status fwix_smooth_step_pair(fwix_plan* p, int iz, const void* in, void* out, void* deriv, int add,
                                  void* stream) {
  if (!p || !in || !out || !deriv) return fail(FWIX_ERR_INVALID, "null argument");
  if (out == deriv) return fail(FWIX_ERR_INVALID, "out and deriv must be different buffers");
  FWIX_TRY(need_smooth(p));
  FWIX_TRY(need_ws(p, FWIX_WS_STEP));
  FWIX_TRY(check_iz(p, iz));
  cudaStream_t s = (cudaStream_t)stream;
  SpecArgs a0 = p->args((const float2*)in, (float2*)out, add);
  FWIX_TRY(phase_factors(p, iz, a0, s));
  return for_chunks(p, a0, [&](SpecArgs a) {
    a.out2 = (float2*)deriv;
    return smooth_chunk(p, iz, kSmoothPair, a, s);
  });
}

fwix_status fwix_correlate(fwix_plan* p, const void* a, const void* b, float* out, int add, int padded,
                           void* stream) {
  if (!p || !a || !b || !out) return fail(FWIX_ERR_INVALID, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  if (padded)
    return cu(fwix::launch_correlate_padded(p->d, (const float2*)a, (const float2*)b, out, add, s), "correlate");
  return cu(fwix::launch_image_acc(p->d, (const float2*)a, (const float2*)b, out, add, s), "correlate");
}

fwix_status fwix_scatter(fwix_plan* p, int iz, int adjoint, const void* in, void* out, int add, void* stream) {
  if (!p || !in || !out) return fail(FWIX_ERR_INVALID, "null argument");
  FWIX_TRY(need_model(p));
  FWIX_TRY(need_ws(p, FWIX_WS_STEP));
  FWIX_TRY(check_iz(p, iz));
  return do_scatter(p, iz, adjoint, (const float2*)in, (float2*)out, add, nullptr, 0, (cudaStream_t)stream);
}

fwix_status fwix_reflect(fwix_plan* p, int iz, int adjoint, const void* in, void* out, int add, void* stream) {
  if (!p || !in || !out) return fail(FWIX_ERR_INVALID, "null argument");
  FWIX_TRY(need_model(p));
  FWIX_TRY(check_iz(p, iz));
  return do_reflect(p, iz, adjoint, (const float2*)in, (float2*)out, add, (cudaStream_t)stream);
}

// Every-depth FWI sweeps of the smooth step: the level loops of the FWI driver
// (pyfwix_b200/fwi.py, SmoothFWI with every depth stored) enqueued from here, so
// that a sweep's ~10 launches per level leave the host once instead of through
// one binding call each.  Steps whose results nothing reads are not taken: the
// down field's step below the bottom, the up field's step of the zero field
// below the model, and the last adjoint step of nu.
fwix_status fwix_smooth_model_sweep(fwix_plan* p, const fwix_traces* src, const fwix_traces* rec,
                                    const void* wavelet, void* data, void* U, void* Ds, void* dSU, void* stream) {
  if (!p || !U || !Ds || no_traces(src, wavelet) || no_traces(rec, data))
    return fail(FWIX_ERR_INVALID, "null argument");
  FWIX_TRY(need_smooth(p));
  FWIX_TRY(need_model(p));
  FWIX_TRY(need_ws(p, FWIX_WS_STEP));
  cudaStream_t s = (cudaStream_t)stream;
  const int nz = p->desc.nz;
  const size_t wb = p->wbytes();
  const long long W = p->d.wfld;
  float2* u = (float2*)U;
  float2* ds = (float2*)Ds;
  float2* dsu = (float2*)dSU;
  if (rec->ntrace > 0) FWIX_CU(cudaMemsetAsync(data, 0, (size_t)rec->ntrace * p->d.nw * sizeof(float2), s));
  // the down recursion runs through the stored fields themselves: level iz's
  // step writes level iz + 1's slot (no working field, no copies)
  FWIX_CU(cudaMemsetAsync(ds, 0, wb, s));
  for (int iz = 0; iz < nz; ++iz) {
    float2* d = ds + iz * W;
    FWIX_TRY(do_inject(p, src, iz, (const float2*)wavelet, d, s));
    FWIX_TRY(do_record(p, rec, iz, d, (float2*)data, s));
    if (iz + 1 < nz) FWIX_TRY(fwix_smooth_step(p, iz, FWIX_SMOOTH_FWD, d, d + W, 0, s));
  }
  FWIX_CU(cudaMemsetAsync(u, 0, wb, s));
  for (int iz = nz - 1; iz >= 0; --iz) {
    if (iz + 1 < nz) {
      if (dsu)
        FWIX_TRY(fwix_smooth_step_pair(p, iz, u, u, dsu + iz * W, 0, s));
      else
        FWIX_TRY(fwix_smooth_step(p, iz, FWIX_SMOOTH_FWD, u, u, 0, s));
    }
    FWIX_TRY(do_reflect(p, iz, 0, ds + iz * W, u, 1, s));
    FWIX_TRY(do_record(p, rec, iz, u, (float2*)data, s));
  }
  return FWIX_OK;
}

fwix_status fwix_smooth_gradient_sweep(fwix_plan* p, const fwix_traces* rec, const void* res, const void* Ds,
                                       const void* dSU, void* mus, void* nu, void* G, float* gpad, float* crefl,
                                       void* stream) {
  if (!p || !Ds || !mus || !nu || !G || !gpad || !crefl || no_traces(rec, res) || (!dSU && p->desc.nz > 1))
    return fail(FWIX_ERR_INVALID, "null argument");
  FWIX_TRY(need_smooth(p));
  FWIX_TRY(need_model(p));
  FWIX_TRY(need_ws(p, FWIX_WS_STEP));
  cudaStream_t s = (cudaStream_t)stream;
  const int nz = p->desc.nz;
  const size_t wb = p->wbytes();
  const long long W = p->d.wfld, gp = (long long)p->d.NY * p->d.NX, gc = (long long)p->d.ny * p->d.nx;
  const float2* ds = (const float2*)Ds;
  const float2* dsu = (const float2*)dSU;
  const float2* r = (const float2*)res;
  float2* v = (float2*)nu;
  float2* ms = (float2*)mus;
  FWIX_CU(cudaMemsetAsync(gpad, 0, (size_t)nz * gp * sizeof(float), s));
  FWIX_CU(cudaMemsetAsync(crefl, 0, (size_t)nz * gc * sizeof(float), s));
  // mu_iz = Rec_iz^H res + S_iz-1^H mu_iz-1 in its own slot of mus (each step
  // writes the next level's slot), and the terms it meets at iz
  FWIX_CU(cudaMemsetAsync(ms, 0, wb, s));
  for (int iz = 0; iz < nz; ++iz) {
    float2* m = ms + iz * W;
    if (iz > 0) FWIX_TRY(fwix_smooth_step(p, iz - 1, FWIX_SMOOTH_ADJ, m - W, m, 0, s));
    FWIX_TRY(do_inject(p, rec, iz, r, m, s));
    if (iz + 1 < nz)  // mu meets dS_iz(U_iz+1) and D_iz in one pass over mu
      FWIX_TRY(cu(fwix::launch_correlate2_padded(p->d, m, dsu + iz * W, ds + iz * W, gpad + iz * gp, crefl + iz * gc,
                                                 1, s),
                  "correlate"));
  }
  // nu_iz = S_iz^H (nu_iz+1 + conj(R_iz) mu_iz + Rec_iz^H res), met by dS_iz(D_iz)
  FWIX_CU(cudaMemsetAsync(v, 0, wb, s));
  for (int iz = nz - 1; iz >= 0; --iz) {
    if (iz + 1 < nz) {
      FWIX_TRY(fwix_smooth_step(p, iz, FWIX_SMOOTH_DERIV, ds + iz * W, G, 0, s));
      FWIX_TRY(fwix_correlate(p, v, G, gpad + iz * gp, 1, 1, s));
    }
    if (iz == 0) break;
    FWIX_TRY(fwix_smooth_step(p, iz, FWIX_SMOOTH_ADJ, v, v, 0, s));
    FWIX_TRY(do_reflect(p, iz, 1, ms + iz * W, v, 1, s));
    FWIX_TRY(do_inject(p, rec, iz, r, v, s));
  }
  return FWIX_OK;
}

fwix_status fwix_imaging(fwix_plan* p, int adjoint, const void* bg, void* image, void* wfld, int add,
                         void* stream) {
  if (!p || !bg || !image || !wfld) return fail(FWIX_ERR_INVALID, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  const long long iw = (long long)p->d.ny * p->d.nx;
  if (!adjoint)
    return cu(fwix::launch_ic_fwd(p->d, (const float2*)bg, (const float2*)image, iw, (float2*)wfld, add, s),
              "imaging forward");
  return cu(fwix::launch_ic_adj(p->d, (const float2*)bg, (const float2*)wfld, (float2*)image, iw, add, s),
            "imaging adjoint");
}

fwix_status fwix_lin_reflect(fwix_plan* p, int iz, int adjoint, void* dmodel, void* dr, int add, void* stream) {
  if (!p || !dmodel || !dr) return fail(FWIX_ERR_INVALID, "null argument");
  FWIX_TRY(need_model(p));
  FWIX_TRY(check_iz(p, iz));
  const int z1 = lower_iz(p, iz);
  float2* dm = (float2*)dmodel;
  const long long n = mslice(p);
  return cu(fwix::launch_lin_reflect(p->d, adjoint, p->slow + iz * p->m_z, p->slow + z1 * p->m_z,
                                     p->den + iz * p->m_z, p->den + z1 * p->m_z, p->m_w, dm, dm + n,
                                     dm + 2 * n, dm + 3 * n, (long long)p->d.ny * p->d.nx, (float2*)dr, add,
                                     (cudaStream_t)stream),
            "linearised reflection");
}

// ---------------------------------------------------------------- acquisition

fwix_status fwix_traces_create(fwix_plan* p, int ntrace, const float* cx, const float* cy, const float* cz,
                               const int32_t* ids, fwix_traces** out) {
  if (!p || !out || ntrace < 0 || (ntrace > 0 && (!cx || !cy || !cz || !ids)))
    return fail(FWIX_ERR_INVALID, "bad trace arguments");
  *out = nullptr;
  const Dims& d = p->d;
  const float OX = p->desc.ox, OY = p->desc.oy, DX = p->desc.dx, DY = p->desc.dy;
  const float oz = p->desc.oz, dz = p->desc.dz;
  const int nlevel = p->desc.nz;
  // gather entries per level: (cell, trace, weight), grouped by cell below
  struct Entry {
    long long cell;
    int trace;
    float w;
  };
  std::vector<std::vector<Entry>> inj(nlevel);
  std::vector<std::vector<int>> rtr(nlevel), rcell(nlevel);
  std::vector<std::vector<float4>> rw(nlevel);
  for (int t = 0; t < ntrace; ++t) {
    if (ids[t] < 0 || ids[t] >= d.ns) return fail(FWIX_ERR_INVALID, "trace shot id outside [0, ns)");
    // injection.cu:34-53, in float
    const int iy = (int)floorf((cy[t] - OY) / DY);
    const float y = OY + (float)iy * DY;
    const float ly = 1.f - (cy[t] - y) / DY;
    const int ix = (int)floorf((cx[t] - OX) / DX);
    const float x = OX + (float)ix * DX;
    const float lx = 1.f - (cx[t] - x) / DX;
    const int izt = (int)floorf((cz[t] - oz) / dz);
    const float z = oz + (float)izt * dz;
    const float lz = 1.f - (cz[t] - z) / dz;
    if (ix < 0 || ix >= d.NX - 1 || iy < 0 || iy >= d.NY - 1) continue;  // injection.cu:46-48
    for (int lev = izt; lev <= izt + 1; ++lev) {
      if (lev < 0 || lev >= nlevel) continue;
      const float zz = (lev == izt) ? lz : (1 - lz);
      const float w0 = zz * lx * ly, w1 = zz * (1 - lx) * ly, w2 = zz * lx * (1 - ly),
                  w3 = zz * (1 - lx) * (1 - ly);
      const long long base = (long long)ids[t] * d.slice + (long long)iy * d.NX + ix;
      inj[lev].push_back({base, t, w0});
      inj[lev].push_back({base + 1, t, w1});
      inj[lev].push_back({base + d.NX, t, w2});
      inj[lev].push_back({base + d.NX + 1, t, w3});
      rtr[lev].push_back(t);
      rcell[lev].push_back((int)base);
      rw[lev].push_back(make_float4(w0, w1, w2, w3));
    }
  }
  fwix_traces* tr = new fwix_traces();
  tr->ntrace = ntrace;
  tr->nlevel = nlevel;
  tr->level.resize(nlevel);
  // pack all levels into flat host arrays, upload once, then point into them
  std::vector<int> cells, starts, trs, rtrace, rcells;
  std::vector<float> wts;
  std::vector<float4> rws;
  std::vector<long long> off_cell(nlevel), off_start(nlevel), off_tr(nlevel), off_r(nlevel);
  for (int lev = 0; lev < nlevel; ++lev) {
    off_cell[lev] = cells.size();
    off_start[lev] = starts.size();
    off_tr[lev] = trs.size();
    off_r[lev] = rtrace.size();
    // cells ascending, each cell's traces in trace order (a stable sort of the
    // entries, which were appended trace by trace)
    std::vector<Entry>& en = inj[lev];
    std::stable_sort(en.begin(), en.end(), [](const Entry& a, const Entry& b) { return a.cell < b.cell; });
    for (size_t i = 0; i < en.size(); ++i) {
      if (i == 0 || en[i].cell != en[i - 1].cell) {
        if (en[i].cell > 0x7fffffffLL) {
          delete tr;
          return fail(FWIX_ERR_UNSUPPORTED, "wavefield batch too large for 32-bit cell indices");
        }
        cells.push_back((int)en[i].cell);
        starts.push_back((int)(trs.size() - off_tr[lev]));
      }
      trs.push_back(en[i].trace);
      wts.push_back(en[i].w);
    }
    std::vector<Entry>().swap(en);
    starts.push_back((int)(trs.size() - off_tr[lev]));
    for (size_t k = 0; k < rtr[lev].size(); ++k) {
      rtrace.push_back(rtr[lev][k]);
      rcells.push_back(rcell[lev][k]);
      rws.push_back(rw[lev][k]);
    }
  }
  int *dcells = nullptr, *dstarts = nullptr, *dtrs = nullptr, *drtrace = nullptr, *drcells = nullptr;
  float* dwts = nullptr;
  float4* drws = nullptr;
  cudaError_t e = upload(&dcells, cells);
  if (e == cudaSuccess) e = upload(&dstarts, starts);
  if (e == cudaSuccess) e = upload(&dtrs, trs);
  if (e == cudaSuccess) e = upload(&dwts, wts);
  if (e == cudaSuccess) e = upload(&drtrace, rtrace);
  if (e == cudaSuccess) e = upload(&drcells, rcells);
  if (e == cudaSuccess) e = upload(&drws, rws);
  void* allocs[] = {dcells, dstarts, dtrs, dwts, drtrace, drcells, drws};
  for (void* v : allocs)
    if (v) tr->allocs.push_back(v);
  if (e != cudaSuccess) {
    fwix_traces_destroy(tr);
    return fail(FWIX_ERR_CUDA, std::string("trace tables: ") + cudaGetErrorString(e));
  }
  for (int lev = 0; lev < nlevel; ++lev) {
    fwix::InjectLevel& L = tr->level[lev];
    const long long nc = (lev + 1 < nlevel ? off_cell[lev + 1] : (long long)cells.size()) - off_cell[lev];
    L.ncell = (int)nc;
    L.cell = dcells ? dcells + off_cell[lev] : nullptr;
    L.start = dstarts + off_start[lev];
    L.trace = dtrs ? dtrs + off_tr[lev] : nullptr;
    L.weight = dwts ? dwts + off_tr[lev] : nullptr;
    const long long nr = (lev + 1 < nlevel ? off_r[lev + 1] : (long long)rtrace.size()) - off_r[lev];
    L.ntr = (int)nr;
    L.rtrace = drtrace ? drtrace + off_r[lev] : nullptr;
    L.rcell = drcells ? drcells + off_r[lev] : nullptr;
    L.rw = drws ? drws + off_r[lev] : nullptr;
  }
  *out = tr;
  return FWIX_OK;
}

fwix_status fwix_traces_destroy(fwix_traces* tr) {
  if (!tr) return FWIX_OK;
  for (void* v : tr->allocs) cudaFree(v);
  delete tr;
  return FWIX_OK;
}

fwix_status fwix_inject(fwix_plan* p, const fwix_traces* tr, int iz, int adjoint, void* traces, void* wfld,
                        int add, void* stream) {
  if (!p || no_traces(tr, traces) || !wfld) return fail(FWIX_ERR_INVALID, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  if (!adjoint) {
    if (!add) FWIX_CU(cudaMemsetAsync(wfld, 0, p->wbytes(), s));
    return do_inject(p, tr, iz, (const float2*)traces, (float2*)wfld, s);
  }
  if (!add && tr->ntrace > 0) FWIX_CU(cudaMemsetAsync(traces, 0, (size_t)tr->ntrace * p->d.nw * sizeof(float2), s));
  return do_record(p, tr, iz, (const float2*)wfld, (float2*)traces, s);
}

// ---------------------------------------------------------------- sweeps

fwix_status fwix_downward(fwix_plan* p, int adjoint, void* wfld, void* stream) {
  if (!p || !wfld) return fail(FWIX_ERR_INVALID, "null argument");
  FWIX_TRY(need_refs(p));
  FWIX_TRY(need_ws(p, FWIX_WS_STEP));
  cudaStream_t s = (cudaStream_t)stream;
  float2* w = (float2*)wfld;
  const int k = p->desc.step_kind;
  if (!adjoint) {
    for (int iz = 0; iz < p->desc.nz; ++iz) FWIX_TRY(do_step(p, k, iz, FWIX_FWD, w, w, 0, s));
  } else {
    for (int iz = p->desc.nz - 1; iz >= 0; --iz) FWIX_TRY(do_step(p, k, iz, FWIX_ADJ_INPL, w, w, 0, s));
  }
  return FWIX_OK;
}

fwix_status fwix_upward(fwix_plan* p, int adjoint, void* wfld, void* stream) {
  if (!p || !wfld) return fail(FWIX_ERR_INVALID, "null argument");
  FWIX_TRY(need_refs(p));
  FWIX_TRY(need_ws(p, FWIX_WS_STEP));
  cudaStream_t s = (cudaStream_t)stream;
  float2* w = (float2*)wfld;
  const int k = p->desc.step_kind;
  if (!adjoint) {
    for (int iz = p->desc.nz - 1; iz >= 0; --iz) FWIX_TRY(do_step(p, k, iz, FWIX_FWD, w, w, 0, s));
  } else {
    for (int iz = 0; iz < p->desc.nz; ++iz) FWIX_TRY(do_step(p, k, iz, FWIX_ADJ_INPL, w, w, 0, s));
  }
  return FWIX_OK;
}

// Propagator::forward (Propagator.cpp:121-221).  The level-iz checkpoints are the
// working buffers themselves: the step from iz writes straight into slot iz+1.
fwix_status fwix_propagate(fwix_plan* p, const fwix_traces* src, const fwix_traces* rec, const void* wavelet,
                           void* data, int add, void* bg_down, void* bg_up, void* stream) {
  if (!p || no_traces(src, wavelet) || no_traces(rec, data)) return fail(FWIX_ERR_INVALID, "null argument");
  if (!bg_down) return fail(FWIX_ERR_INVALID, "bg_down storage ([nz] wavefields) is required");
  FWIX_TRY(need_refs(p));
  FWIX_TRY(need_model(p));
  FWIX_TRY(need_ws(p, FWIX_WS_SWEEP));
  cudaStream_t s = (cudaStream_t)stream;
  const int nz = p->desc.nz, k = p->desc.step_kind;
  const long long W = p->d.wfld;
  float2* down = (float2*)bg_down;
  float2* up = (float2*)bg_up;
  float2* dat = (float2*)data;
  const float2* wav = (const float2*)wavelet;
  if (!add && rec->ntrace > 0) FWIX_CU(cudaMemsetAsync(dat, 0, (size_t)rec->ntrace * p->d.nw * sizeof(float2), s));
  FWIX_CU(cudaMemsetAsync(down, 0, p->wbytes(), s));
  for (int iz = 0; iz < nz; ++iz) {
    float2* cur = down + iz * W;
    FWIX_TRY(do_inject(p, src, iz, wav, cur, s));
    FWIX_TRY(do_record(p, rec, iz, cur, dat, s));
    if (iz < nz - 1) FWIX_TRY(do_step(p, k, iz, FWIX_FWD, cur, down + (iz + 1) * W, 0, s));
  }
  float2* prev = nullptr;
  for (int iz = nz - 1; iz >= 0; --iz) {
    float2* cur = up ? up + iz * W : ((nz - 1 - iz) % 2 ? p->wB() : p->wA());
    if (prev)
      FWIX_TRY(do_step(p, k, iz, FWIX_FWD, prev, cur, 0, s));
    else
      FWIX_CU(cudaMemsetAsync(cur, 0, p->wbytes(), s));  // stepping the zero field gives zero
    FWIX_TRY(do_reflect(p, iz, 0, down + iz * W, cur, 1, s));
    FWIX_TRY(do_record(p, rec, iz, cur, dat, s));
    prev = cur;
  }
  return FWIX_OK;
}

size_t fwix_plan_packed_bytes(const fwix_plan* p) { return p ? p->packed_bytes() : 0; }

fwix_status fwix_plan_set_pack_rate(fwix_plan* p, int bits) {
  if (!p) return fail(FWIX_ERR_INVALID, "null plan");
  if (bits != 8 && bits != 16) return fail(FWIX_ERR_UNSUPPORTED, "pack rate must be 8 or 16 bits per value");
  p->pack_bits = bits;
  return FWIX_OK;
}

fwix_status fwix_pack_wavefield(fwix_plan* p, const void* wfld, void* packed, void* stream) {
  if (!p || !wfld || !packed) return fail(FWIX_ERR_INVALID, "null argument");
  if (((uintptr_t)wfld) % 4 != 0 || ((uintptr_t)packed) % 4 != 0)
    return fail(FWIX_ERR_INVALID, "wavefield and packed buffers must be 4-byte aligned");
  return cu(fwix::launch_pack(p->pack_bits, 2 * p->d.wfld, (const float*)wfld, packed, (cudaStream_t)stream), "pack");
}

fwix_status fwix_unpack_wavefield(fwix_plan* p, const void* packed, void* wfld, void* stream) {
  if (!p || !wfld || !packed) return fail(FWIX_ERR_INVALID, "null argument");
  if (((uintptr_t)wfld) % 4 != 0 || ((uintptr_t)packed) % 4 != 0)
    return fail(FWIX_ERR_INVALID, "wavefield and packed buffers must be 4-byte aligned");
  return cu(fwix::launch_unpack(p->pack_bits, 2 * p->d.wfld, packed, (float*)wfld, (cudaStream_t)stream),
            "unpack");
}

fwix_status fwix_pack_rate8(fwix_plan* p, const void* wfld, void* packed, void* stream) {
  if (!p || !wfld || !packed) return fail(FWIX_ERR_INVALID, "null argument");
  if (((uintptr_t)wfld) % 4 != 0 || ((uintptr_t)packed) % 4 != 0)
    return fail(FWIX_ERR_INVALID, "wavefield and packed buffers must be 4-byte aligned");
  return cu(fwix::launch_pack_rate8(2 * p->d.wfld, (const float*)wfld, packed, (cudaStream_t)stream), "pack");
}

fwix_status fwix_unpack_rate8(fwix_plan* p, const void* packed, void* wfld, void* stream) {
  if (!p || !wfld || !packed) return fail(FWIX_ERR_INVALID, "null argument");
  if (((uintptr_t)wfld) % 4 != 0 || ((uintptr_t)packed) % 4 != 0)
    return fail(FWIX_ERR_INVALID, "wavefield and packed buffers must be 4-byte aligned");
  return cu(fwix::launch_unpack_rate8(2 * p->d.wfld, packed, (float*)wfld, (cudaStream_t)stream), "unpack");
}

// Propagator::forward (Propagator.cpp:121-221) keeping the down and up fields of
// every depth packed, as the reference keeps them ZFP-compressed in its
// WavefieldPool: D in workspace A, each depth packed after its injection; the up
// pass reflects the unpacked down field of each depth (workspace B).
fwix_status fwix_propagate_packed(fwix_plan* p, const fwix_traces* src, const fwix_traces* rec, const void* wavelet,
                                  void* data, int add, void* packed_down, void* packed_up, void* stream) {
  if (!p || no_traces(src, wavelet) || no_traces(rec, data) || !packed_down)
    return fail(FWIX_ERR_INVALID, "null argument");
  if (((uintptr_t)packed_down) % 4 != 0 || ((uintptr_t)packed_up) % 4 != 0 || p->packed_bytes() % 16 != 0)
    return fail(FWIX_ERR_INVALID, "packed buffers must be 4-byte aligned");
  FWIX_TRY(need_refs(p));
  FWIX_TRY(need_model(p));
  FWIX_TRY(need_ws(p, FWIX_WS_SWEEP));
  cudaStream_t s = (cudaStream_t)stream;
  const int nz = p->desc.nz, k = p->desc.step_kind;
  const long long nf = 2 * p->d.wfld;
  const size_t pb = p->packed_bytes();
  unsigned char* pd = (unsigned char*)packed_down;
  unsigned char* pu = (unsigned char*)packed_up;
  float2* dat = (float2*)data;
  const float2* wav = (const float2*)wavelet;
  float2* D = p->wA();
  float2* R = p->wB();
  if (!add && rec->ntrace > 0) FWIX_CU(cudaMemsetAsync(dat, 0, (size_t)rec->ntrace * p->d.nw * sizeof(float2), s));
  FWIX_CU(cudaMemsetAsync(D, 0, p->wbytes(), s));
  for (int iz = 0; iz < nz; ++iz) {
    FWIX_TRY(do_inject(p, src, iz, wav, D, s));
    FWIX_TRY(do_record(p, rec, iz, D, dat, s));
    FWIX_TRY(cu(fwix::launch_pack(p->pack_bits, nf, (const float*)D, pd + (size_t)iz * pb, s), "pack down field"));
    if (iz < nz - 1) FWIX_TRY(do_step(p, k, iz, FWIX_FWD, D, D, 0, s));
  }
  float2* U = p->wA();  // the down pass is done with it
  for (int iz = nz - 1; iz >= 0; --iz) {
    if (iz == nz - 1)
      FWIX_CU(cudaMemsetAsync(U, 0, p->wbytes(), s));
    else
      FWIX_TRY(do_step(p, k, iz, FWIX_FWD, U, U, 0, s));
    FWIX_TRY(cu(fwix::launch_unpack(p->pack_bits, nf, pd + (size_t)iz * pb, (float*)R, s), "unpack down field"));
    FWIX_TRY(do_reflect(p, iz, 0, R, U, 1, s));
    FWIX_TRY(do_record(p, rec, iz, U, dat, s));
    if (pu)
      FWIX_TRY(cu(fwix::launch_pack(p->pack_bits, nf, (const float*)U, pu + (size_t)iz * pb, s), "pack up field"));
  }
  return FWIX_OK;
}

// Lockstep migration: the source field (Propagator.cpp:155-180) and the receiver
// field of the back-scattering adjoint (ExtendedBorn.cpp:396-408) move down
// together and image[iz] accumulates sum_w Re sum_s conj(S) R
// (imaging_condition.cu:57-108 summed over frequency).
fwix_status fwix_migrate(fwix_plan* p, const fwix_traces* src, const fwix_traces* rec, const void* wavelet,
                         const void* data, float* image, int add, void* stream) {
  if (!p || no_traces(src, wavelet) || no_traces(rec, data) || !image) return fail(FWIX_ERR_INVALID, "null argument");
  FWIX_TRY(need_refs(p));
  FWIX_TRY(need_ws(p, FWIX_WS_SWEEP));
  cudaStream_t s = (cudaStream_t)stream;
  const int nz = p->desc.nz, k = p->desc.step_kind;
  float2* S = p->wA();
  float2* R = p->wB();
  FWIX_CU(cudaMemsetAsync(S, 0, p->wbytes(), s));
  FWIX_CU(cudaMemsetAsync(R, 0, p->wbytes(), s));
  const long long plane = (long long)p->d.ny * p->d.nx;
  // The image of a level is summed by the receiver step that reaches it (the
  // epilogue of its inverse row pass, reading S of that level), except at the
  // first level and at levels where receivers inject: there the field is only
  // complete after the injection, and one correlation pass sums the image.
  // The one-launch cluster step has no such epilogue.
  const bool fuse = !p->fused;
  if (!add) FWIX_CU(cudaMemsetAsync(image, 0, (size_t)nz * plane * sizeof(float), s));
  FWIX_TRY(do_inject(p, src, 0, (const float2*)wavelet, S, s));
  FWIX_TRY(do_inject(p, rec, 0, (const float2*)data, R, s));
  FWIX_TRY(cu(fwix::launch_image_acc(p->d, S, R, image, 1, s), "image"));
  for (int iz = 0; iz + 1 < nz; ++iz) {
    float* img = image + (iz + 1) * plane;
    FWIX_TRY(do_step(p, k, iz, FWIX_FWD, S, S, 0, s));
    FWIX_TRY(do_inject(p, src, iz + 1, (const float2*)wavelet, S, s));
    const fwix::InjectLevel* L = level_of(rec, iz + 1);
    if (fuse && !(L && L->ncell > 0)) {
      FWIX_TRY(do_step(p, k, iz, FWIX_ADJ_INPL, R, R, 0, s, nullptr, S, img));
    } else {
      FWIX_TRY(do_step(p, k, iz, FWIX_ADJ_INPL, R, R, 0, s));
      FWIX_TRY(do_inject(p, rec, iz + 1, (const float2*)data, R, s));
      FWIX_TRY(cu(fwix::launch_image_acc(p->d, S, R, img, 1, s), "image"));
    }
  }
  return FWIX_OK;
}

// ExtendedBorn::forward / adjoint (ExtendedBorn.cpp:80-453).
fwix_status fwix_born(fwix_plan* p, int adjoint, const fwix_traces* rec, const void* bg_down_v,
                      const void* bg_up_v, void* dslow_v, void* dden_v, int64_t model_w_stride, void* data_v,
                      int add, void* stream) {
  if (!p || no_traces(rec, data_v) || !bg_down_v || !bg_up_v || !dslow_v || !dden_v)
    return fail(FWIX_ERR_INVALID, "null argument");
  const long long plane = (long long)p->d.ny * p->d.nx;
  if (model_w_stride != 0 && model_w_stride != plane)
    return fail(FWIX_ERR_INVALID, "model_w_stride must be 0 or ny*nx");
  const long long mw = model_w_stride;
  FWIX_TRY(need_refs(p));
  FWIX_TRY(need_model(p));
  FWIX_TRY(need_ws(p, FWIX_WS_BORN));
  BgSrc D{(const float2*)bg_down_v}, U{(const float2*)bg_up_v};
  return born_body(p, adjoint, rec, D, U, (float2*)dslow_v, (float2*)dden_v, mw, (float2*)data_v, add,
                   (cudaStream_t)stream);
}

fwix_status fwix_born_packed(fwix_plan* p, int adjoint, const fwix_traces* rec, const void* packed_down,
                             const void* packed_up, void* dslow_v, void* dden_v, int64_t model_w_stride,
                             void* data_v, int add, void* stream) {
  if (!p || no_traces(rec, data_v) || !packed_down || !packed_up || !dslow_v || !dden_v)
    return fail(FWIX_ERR_INVALID, "null argument");
  const long long plane = (long long)p->d.ny * p->d.nx;
  if (model_w_stride != 0 && model_w_stride != plane)
    return fail(FWIX_ERR_INVALID, "model_w_stride must be 0 or ny*nx");
  FWIX_TRY(need_refs(p));
  FWIX_TRY(need_model(p));
  FWIX_TRY(need_ws(p, FWIX_WS_BORN_PACKED));
  BgSrc D{nullptr, (const unsigned char*)packed_down, p->wB()};
  BgSrc U{nullptr, (const unsigned char*)packed_up, p->wU()};
  return born_body(p, adjoint, rec, D, U, (float2*)dslow_v, (float2*)dden_v, model_w_stride, (float2*)data_v,
                   add, (cudaStream_t)stream, true);
}


// ---------------------------------------------------------------- runtime tuning
// Times the equivalent implementations of one depth step of this plan on the
// caller's wavefield and keeps the fastest: column tiles moved by per-thread
// cp.async or by TMA; every slice in one launch, or halves / quarters of them
// (the intermediates of a smaller launch stay in L2), also alternating between
// two streams; for 256 x 256 slices the one-launch cluster step.  Each
// candidate runs once untimed (it builds its
// tables), then `reps` steps between CUDA events on `stream`.  Synchronises the
// stream: call it before any capture.
fwix_status fwix_plan_autotune(fwix_plan* p, int kind, int iz, const void* in, void* out, int reps, void* stream,
                               fwix_tuning* result) {
  if (!p || !in || !out) return fail(FWIX_ERR_INVALID, "null argument");
  if (kind != FWIX_STEP_PSPI && kind != FWIX_STEP_NSPS) return fail(FWIX_ERR_INVALID, "unknown step kind");
  FWIX_TRY(need_refs(p));
  FWIX_TRY(need_ws(p, FWIX_WS_STEP));
  FWIX_TRY(check_iz(p, iz));
  if (in == out) return fail(FWIX_ERR_INVALID, "autotune needs distinct in and out buffers");
  cudaStream_t s = (cudaStream_t)stream;
  reps = std::max(1, reps);
  struct Cand {
    bool tma;
    long long chunk;
    bool fused;
    int lanes;
  };
  std::vector<Cand> cands;
  // the workspace holds the intermediates of this many slices (one lane)
  const long long c0 = p->chunk * p->lanes;
  for (long long c : {c0, c0 / 2, c0 / 4}) {
    if (c < 8 && c != c0) continue;
    bool dup = false;
    for (const Cand& k : cands) dup = dup || k.chunk == c;
    if (dup) continue;
    cands.push_back({false, c, false, 1});
    cands.push_back({true, c, false, 1});
  }
  for (long long c : {c0 / 2, c0 / 4, c0 / 8}) {  // two lanes of c slices each
    if (c < 8) continue;
    cands.push_back({false, c, false, 2});
    cands.push_back({true, c, false, 2});
  }
  if (p->d.NX == 256 && p->d.NY == 256 && fwix::fused_step_available()) cands.push_back({false, c0, true, 1});
  bool have_lanes = false;
  for (const Cand& k : cands) have_lanes = have_lanes || k.lanes == 2;
  if (have_lanes && !p->lane_s) {
    FWIX_CU(cudaStreamCreateWithFlags(&p->lane_s, cudaStreamNonBlocking));
    FWIX_CU(cudaEventCreateWithFlags(&p->lane_fork, cudaEventDisableTiming));
    FWIX_CU(cudaEventCreateWithFlags(&p->lane_join, cudaEventDisableTiming));
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  FWIX_CU(cudaEventCreate(&e0));
  FWIX_CU(cudaEventCreate(&e1));
  const bool tma0 = p->col_tma, fused0 = p->fused;
  const long long chunk0 = p->chunk;
  const int lanes0 = p->lanes;
  float best = -1.f;
  Cand pick{tma0, chunk0, fused0, lanes0};
  int tried = 0;
  for (const Cand& k : cands) {
    p->col_tma = k.tma;
    p->chunk = k.chunk;
    p->fused = k.fused;
    p->lanes = k.lanes;
    if (do_step(p, kind, iz, FWIX_FWD, (const float2*)in, (float2*)out, 0, s) != FWIX_OK) {
      cudaGetLastError();  // a candidate this device or size does not run (launch error, not sticky)
      continue;
    }
    fwix_status st = FWIX_OK;
    cudaError_t ce = cudaEventRecord(e0, s);
    for (int r = 0; r < reps && st == FWIX_OK; ++r)
      st = do_step(p, kind, iz, FWIX_FWD, (const float2*)in, (float2*)out, 0, s);
    if (ce == cudaSuccess) ce = cudaEventRecord(e1, s);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
    if (st != FWIX_OK || ce != cudaSuccess) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      p->col_tma = tma0, p->chunk = chunk0, p->fused = fused0, p->lanes = lanes0;
      return st != FWIX_OK ? st : fail(FWIX_ERR_CUDA, std::string("autotune timing: ") + cudaGetErrorString(ce));
    }
    ++tried;
    ms /= (float)reps;
    if (best < 0.f || ms < best) {
      best = ms;
      pick = k;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  p->col_tma = pick.tma;
  p->chunk = pick.chunk;
  p->fused = pick.fused;
  p->lanes = pick.lanes;
  if (tried == 0) return fail(FWIX_ERR_UNSUPPORTED, "autotune: no candidate ran");
  if (result) {
    result->col_tma = pick.tma ? 1 : 0;
    result->fused = pick.fused ? 1 : 0;
    result->slices_per_launch = pick.chunk;
    result->ms = best;
    result->candidates = tried;
    result->streams = pick.lanes;
  }
  return FWIX_OK;
}

// A choice fwix_plan_autotune made earlier (for a plan of the same sizes),
// applied without timing: tile movement, slices per launch, lanes, cluster step.
fwix_status fwix_plan_set_tuning(fwix_plan* p, const fwix_tuning* t) {
  if (!p || !t) return fail(FWIX_ERR_INVALID, "null argument");
  const long long slices = (long long)p->d.ns * p->d.nw;
  if (t->slices_per_launch < 1 || t->slices_per_launch > slices)
    return fail(FWIX_ERR_INVALID, "slices_per_launch must be in [1, ns * nw]");
  if (t->streams != 1 && t->streams != 2) return fail(FWIX_ERR_INVALID, "streams must be 1 or 2");
  if (t->fused && !(p->d.NX == 256 && p->d.NY == 256 && fwix::fused_step_available()))
    return fail(FWIX_ERR_UNSUPPORTED, "the one-launch cluster step needs 256 x 256 slices");
  if (t->streams == 2 && !p->lane_s) {
    FWIX_CU(cudaStreamCreateWithFlags(&p->lane_s, cudaStreamNonBlocking));
    FWIX_CU(cudaEventCreateWithFlags(&p->lane_fork, cudaEventDisableTiming));
    FWIX_CU(cudaEventCreateWithFlags(&p->lane_join, cudaEventDisableTiming));
  }
  p->col_tma = t->col_tma != 0;
  p->chunk = t->slices_per_launch;
  p->fused = t->fused != 0;
  p->lanes = t->streams;
  return FWIX_OK;
}

// ---------------------------------------------------------------- one-call forms
fwix_status fwix_pspi_step(fwix_plan* p, int iz, const void* in, void* out, int adjoint, void* stream) {
  return fwix_step(p, FWIX_STEP_PSPI, iz, adjoint, in, out, 0, stream);
}

fwix_status fwix_nsps_step(fwix_plan* p, int iz, const void* in, void* out, int adjoint, void* stream) {
  return fwix_step(p, FWIX_STEP_NSPS, iz, adjoint, in, out, 0, stream);
}

fwix_status fwix_image_accumulate(fwix_plan* p, const void* S, const void* R, float* image, int add,
                                  void* stream) {
  return fwix_correlate(p, S, R, image, add, 0, stream);
}

// ---------------------------------------------------------------- batched sweeps
namespace {

fwix_status sweep_one(int kind, const fwix_instance& in, void* s) {
  switch (kind) {
    case FWIX_SWEEP_DOWN: return fwix_downward(in.plan, in.adjoint, in.wfld, s);
    case FWIX_SWEEP_UP: return fwix_upward(in.plan, in.adjoint, in.wfld, s);
    case FWIX_SWEEP_MODEL:
      return fwix_propagate(in.plan, in.src, in.rec, in.wavelet, in.data, in.add, in.bg_down, in.bg_up, s);
    case FWIX_SWEEP_IMAGE: return fwix_migrate(in.plan, in.src, in.rec, in.wavelet, in.data, in.image, in.add, s);
    case FWIX_SWEEP_BORN_FWD:
    case FWIX_SWEEP_BORN_ADJ:
      return fwix_born(in.plan, kind == FWIX_SWEEP_BORN_ADJ, in.rec, in.bg_down, in.bg_up, in.dslow, in.dden,
                       in.model_w_stride, in.data, in.add, s);
    default: return fail(FWIX_ERR_INVALID, "unknown sweep kind");
  }
}

}  // namespace

fwix_status fwix_sweep(int kind, const fwix_instance* insts, int ninst, void* const* streams, int nstreams,
                       void* stream) {
  if (ninst < 0 || (ninst > 0 && !insts) || nstreams < 0 || (nstreams > 0 && !streams))
    return fail(FWIX_ERR_INVALID, "null or negative instance / stream list");
  if (kind < FWIX_SWEEP_DOWN || kind > FWIX_SWEEP_BORN_ADJ) return fail(FWIX_ERR_INVALID, "unknown sweep kind");
  for (int i = 0; i < ninst; ++i) {
    if (!insts[i].plan) return fail(FWIX_ERR_INVALID, "instance " + std::to_string(i) + " has no plan");
    for (int j = 0; j < i; ++j)
      if (insts[j].plan == insts[i].plan)
        return fail(FWIX_ERR_INVALID, "instances " + std::to_string(j) + " and " + std::to_string(i) +
                                          " share a plan (its workspace would be used by two streams)");
  }
  if (nstreams == 0) {
    for (int i = 0; i < ninst; ++i) FWIX_TRY(sweep_one(kind, insts[i], stream));
    return FWIX_OK;
  }
  // largest first onto the least loaded stream
  std::vector<int> order(ninst);
  for (int i = 0; i < ninst; ++i) order[i] = i;
  auto cost = [&](int i) {
    const fwix_desc& q = insts[i].plan->desc;
    return (double)insts[i].plan->d.NX * insts[i].plan->d.NY * q.nw * q.ns * q.nz;
  };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
  std::vector<double> load(nstreams, 0.0);
  std::vector<std::vector<int>> lanes(nstreams);
  for (int i : order) {
    const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    lanes[k].push_back(i);
    load[k] += cost(i);
  }
  cudaStream_t main = (cudaStream_t)stream;
  cudaEvent_t fork = nullptr;
  FWIX_CU(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  fwix_status st = FWIX_OK;
  std::vector<cudaEvent_t> joins;
  cudaError_t e = cudaEventRecord(fork, main);
  for (int k = 0; k < nstreams && e == cudaSuccess && st == FWIX_OK; ++k) {
    if (lanes[k].empty()) continue;
    cudaStream_t sk = (cudaStream_t)streams[k];
    e = cudaStreamWaitEvent(sk, fork, 0);
    for (size_t j = 0; j < lanes[k].size() && e == cudaSuccess && st == FWIX_OK; ++j)
      st = sweep_one(kind, insts[lanes[k][j]], sk);
    cudaEvent_t join = nullptr;
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join, cudaEventDisableTiming);
    if (e == cudaSuccess) {
      joins.push_back(join);
      e = cudaEventRecord(join, sk);
    }
  }
  // the caller's stream waits for every lane enqueued so far, also after a failure
  for (cudaEvent_t j : joins) {
    const cudaError_t w = cudaStreamWaitEvent(main, j, 0);
    if (e == cudaSuccess) e = w;
    cudaEventDestroy(j);
  }
  cudaEventDestroy(fork);
  if (st != FWIX_OK) return st;
  if (e != cudaSuccess) return fail(FWIX_ERR_CUDA, std::string("fwix_sweep: ") + cudaGetErrorString(e));
  return FWIX_OK;
}

}  // extern "C"
