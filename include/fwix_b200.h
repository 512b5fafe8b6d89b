/*
 * fwix_b200.h -- C ABI of the B200 (sm_100a) one-way wave-equation depth-stepping
 * library (libfwix_b200.so).
 *
 * Conventions
 *   - Every array argument is a DEVICE pointer owned by the caller, except the
 *     host arrays that fwix_traces_create copies.  Complex values are interleaved
 *     float pairs (complex64).  Layouts are row-major with x fastest:
 *       wavefield  [ns][nw][NY][NX]        NX = nx + padx, NY = ny + pady
 *       model      [nz][nw][ny][nx]        (s^2 = 1/v^2, density), strides given
 *       labels     uint8, [nz][nw][NY][NX] with caller strides (w stride may be 0)
 *       refs       [nz][nref][nw]          complex reference s^2
 *       traces     [ntrace][nw]
 *   - "add" follows the reference operators: add == 0 overwrites the output,
 *     add != 0 accumulates into it.
 *   - Calls are stream ordered on the cudaStream_t passed as `stream` (NULL = the
 *     legacy default stream) and never synchronise the device.
 *   - Errors are negative status codes; fwix_last_error() returns the message
 *     of the last failure on the calling thread.  Nothing calls exit().
 *   - A plan may be used by one host thread at a time.
 *   - Wavefield-sized temporaries come from a caller-provided workspace
 *     (fwix_plan_workspace_bytes / fwix_plan_set_workspace); only small tables
 *     (wavenumbers, twiddles, trace lists) are allocated by the library, at
 *     plan / trace-set creation.
 *
 * Reference interface each entry point replaces (paths inside pyfwix):
 *   operator/src/CudaOperator.h:61-72          cu_forward / cu_adjoint(add, m, d)
 *   operator/src/FFT.cpp:36-69                 cuFFT2d
 *   propagator/src/PhaseShift.cpp:27-41        PhaseShift fwd / adj / inverse
 *   propagator/src/Selector.h:38-45            Selector
 *   propagator/src/Taper.h:30-37               Taper
 *   propagator/src/PSPI.cpp:6-103              PSPI (add and in-place forms)
 *   propagator/src/NSPS.cpp:6-45               NSPS
 *   propagator/src/Injection.cpp:35-44         Injection fwd / adj
 *   propagator/src/Reflect.cpp:45-62           Reflect
 *   propagator/src/Scatter.cpp:76-133          Scatter
 *   propagator/src/ImagingCondition.cpp:33-48  ImagingCondition
 *   propagator/src/LinReflect.cpp:28-40        LinReflect
 *   propagator/src/OneWay.cpp:24-79            Downward / Upward
 *   propagator/src/Propagator.cpp:121-221      Propagator::forward
 *   propagator/src/ExtendedBorn.cpp:80-150     ExtendedBorn::forward / adjoint
 */
#ifndef FWIX_B200_H
#define FWIX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fwix_status {
  FWIX_OK = 0,
  FWIX_ERR_INVALID = -1,     /* bad argument or descriptor                     */
  FWIX_ERR_UNSUPPORTED = -2, /* size or option outside what the kernels cover  */
  FWIX_ERR_CUDA = -3,        /* CUDA runtime error                             */
  FWIX_ERR_STATE = -4,       /* refs / model / workspace not bound yet         */
  FWIX_ERR_WORKSPACE = -5    /* workspace smaller than required                */
} fwix_status;

/* Depth-step kinds (the reference's OneWay always uses PSPI,
 * propagator/src/OneWay.h:24-25). */
enum { FWIX_STEP_PSPI = 0, FWIX_STEP_NSPS = 1 };

/* Directions of a depth step.
 *   FWD      : out (+)= sum_r mask_r F^-1(P_r F(taper in))       PSPI.cpp:6-24 / :66-83
 *   ADJ_ADD  : out (+)= F^-1(sum_r P_r^* F(mask_r in))           PSPI.cpp:26-44 (no taper)
 *   ADJ_INPL : out (+)= taper F^-1(sum_r P_r^* F(mask_r in))     PSPI.cpp:85-103
 * For NSPS the taper never applies (NSPS.cpp:6-45). */
enum { FWIX_FWD = 0, FWIX_ADJ_ADD = 1, FWIX_ADJ_INPL = 2 };

/* PhaseShift modes (phase_shift.cu:7-61, :125-184, :248-305). */
enum { FWIX_PS_FWD = 0, FWIX_PS_ADJ = 1, FWIX_PS_INV = 2 };

/* Smooth-step modes (fwix_smooth_step). */
enum { FWIX_SMOOTH_FWD = 0, FWIX_SMOOTH_ADJ = 1, FWIX_SMOOTH_DERIV = 2 };

/* Workspace classes for fwix_plan_workspace_bytes. */
enum { FWIX_WS_STEP = 0, FWIX_WS_SWEEP = 1, FWIX_WS_BORN = 2, FWIX_WS_BORN_PACKED = 3 };

typedef struct fwix_desc {
  int nx, ny;        /* model lateral size                                   */
  int padx, pady;    /* wavefield = (nx + padx) x (ny + pady)                 */
  int nw;            /* frequencies                                           */
  int ns;            /* shots in the wavefield batch                          */
  int nz;            /* depth levels                                          */
  float ox, oy, oz;  /* origins [m]                                           */
  float dx, dy, dz;  /* sampling [m]                                          */
  float ow, dw;      /* first frequency and step [Hz]                         */
  int nref;          /* reference slownesses per depth ("nref")               */
  float eps;         /* phase-shift damping ("eps")                           */
  int taperx, tapery;/* lateral taper widths ("taperx", "tapery")             */
  float eps_scat;    /* Born damping ("eps_scat", default 0.04)               */
  int taylor;        /* Born Taylor order ("taylor", default 1, max 4)        */
  int step_kind;     /* FWIX_STEP_PSPI or FWIX_STEP_NSPS for the sweeps       */
} fwix_desc;

typedef struct fwix_plan fwix_plan;
typedef struct fwix_traces fwix_traces;

const char* fwix_last_error(void);
int fwix_version(void);
/* Kernels this library has enqueued since it was loaded (all plans, all threads). */
uint64_t fwix_launch_count(void);

/* ---- plan ------------------------------------------------------------------ */
fwix_status fwix_plan_create(const fwix_desc* desc, fwix_plan** plan);
fwix_status fwix_plan_destroy(fwix_plan* plan);
size_t fwix_plan_workspace_bytes(const fwix_plan* plan, int ws_class);
/* Bounded device-side waits of this plan's kernels that ran out of tries (the
 * kernel then skipped its work); 0 in normal operation.  Reads device memory
 * (synchronous). */
uint64_t fwix_plan_wait_timeouts(const fwix_plan* plan);
fwix_status fwix_plan_set_workspace(fwix_plan* plan, void* dev_ptr, size_t bytes);
/* sref: [nz][nref][nw] complex; labels: uint8 label of (iz, iw, y, x) at
 * labels[iz*z_stride + iw*w_stride + y*NX + x] (RefSampler.cpp:27-28, 126-133). */
fwix_status fwix_plan_set_refs(fwix_plan* plan, const void* sref, const uint8_t* labels,
                               int64_t labels_z_stride, int64_t labels_w_stride);
/* Optional phase-factor cache.  The factor of a depth step depends only on
 * (depth, reference, frequency, |kx|, |ky|) (phase_shift.cu:36-55), so with a
 * cache of fwix_plan_phase_cache_bytes bytes bound, each depth's factors are
 * computed once, on the first step at that depth, and every later step there
 * (Born sweeps visit each depth many times) reads them.  A smaller cache of k
 * depths (at least fwix_plan_phase_cache_bytes / nz bytes each) keeps depth iz
 * in slot iz mod k and rebuilds a slot when another depth has taken it: one
 * depth is enough for the two steps per level of a lockstep migration.
 * Binding NULL disables it; fwix_plan_set_refs invalidates it.  Calls that use
 * it must be ordered on one stream (or synchronised), as for the workspace. */
size_t fwix_plan_phase_cache_bytes(const fwix_plan* plan);
fwix_status fwix_plan_set_phase_cache(fwix_plan* plan, void* dev_ptr, size_t bytes);
/* Background s^2 and density, element (iz,iw,y,x) at
 * p[iz*z_stride + iw*w_stride + y*nx + x] (Reflect.h:20-38, Scatter.cpp:68-74). */
fwix_status fwix_plan_set_model(fwix_plan* plan, const void* slow, const void* den,
                                int64_t z_stride, int64_t w_stride);

/* ---- one-slice operators (device -> device) --------------------------------- */
/* Unitary 2D FFT, forward e^{-i} or inverse e^{+i}, x 1/sqrt(NX*NY). */
fwix_status fwix_fft2d(fwix_plan* plan, int inverse, const void* in, void* out, int add, void* stream);
/* Phase shift in the wavenumber domain with per-frequency reference s^2 sref_w[nw]. */
fwix_status fwix_phase_shift(fwix_plan* plan, int mode, const void* sref_w, const void* in,
                             void* out, int add, void* stream);
fwix_status fwix_select(fwix_plan* plan, int iz, int value, const void* in, void* out, int add,
                        void* stream);
fwix_status fwix_taper(fwix_plan* plan, const void* in, void* out, int add, void* stream);
/* One depth step at level iz; in may equal out. */
fwix_status fwix_step(fwix_plan* plan, int kind, int iz, int dir, const void* in, void* out,
                      int add, void* stream);
/* Born scattering at level iz (adjoint != 0 for the transpose). */
fwix_status fwix_scatter(fwix_plan* plan, int iz, int adjoint, const void* in, void* out, int add,
                         void* stream);
/* Reflection at level iz: fwd up (+)= r down, adj down (+)= conj(r) up. */
fwix_status fwix_reflect(fwix_plan* plan, int iz, int adjoint, const void* in, void* out, int add,
                         void* stream);
/* Imaging condition: fwd wfld (+)= bg * image; adj image (+)= sum_s conj(bg) wfld.
 * image is [nw][ny][nx]. */
fwix_status fwix_imaging(fwix_plan* plan, int adjoint, const void* bg, void* image, void* wfld,
                         int add, void* stream);
/* Linearised reflection at level iz: dmodel [4][nw][ny][nx] = (ds2(iz), ds2(iz+1),
 * drho(iz), drho(iz+1)) <-> dr [nw][ny][nx]. */
fwix_status fwix_lin_reflect(fwix_plan* plan, int iz, int adjoint, void* dmodel, void* dr, int add,
                             void* stream);

/* ---- differentiable ("smooth") step ------------------------------------------
 * No reference counterpart: the reference's PSPI selects the nearest reference
 * per cell (propagator/src/selector.cu:29-35), so its output depends on the
 * slowness only through piecewise-constant labels and has no usable gradient.
 * The smooth step interpolates between the two references that bracket the
 * local slowness s (hat functions over the references sorted ascending,
 * clamped at both ends) and applies the split-step correction
 * SS_r = exp(-i w (s - s_r) dz):
 *   FWD   out (+)= sum_r w_r(s) SS_r F^-1(P_r F(taper in))
 *   ADJ   out (+)= its exact transpose
 *   DERIV out (+)= sum_r (w_r'(s) - i w dz w_r(s)) SS_r F^-1(P_r F(taper in))
 *                  (the derivative of FWD with respect to s, cell by cell)
 * P_r are the phase factors of the complex references bound by
 * fwix_plan_set_refs (s_r^2 for every frequency; labels are not used). */
/* slow_pad [nz][NY][NX] (edge-replicated s), sref_real [nz][nref] ascending. */
fwix_status fwix_plan_set_smooth(fwix_plan* plan, const float* slow_pad, const float* sref_real);
fwix_status fwix_smooth_step(fwix_plan* plan, int iz, int mode, const void* in, void* out, int add,
                             void* stream);
/* FWD into out and DERIV into deriv (different buffers; in may be either) from
 * one set of transforms: the forward step and its slowness derivative share the
 * forward row and column passes and each inverse row transform, which the
 * gradient's segment recomputations need together. */
fwix_status fwix_smooth_step_pair(fwix_plan* plan, int iz, const void* in, void* out, void* deriv, int add,
                                  void* stream);
/* out[y][x] (+)= Re sum_{shots, w} conj(a) b over the padded slice (padded != 0,
 * out is [NY][NX]) or the model window (out is [ny][nx]). */
fwix_status fwix_correlate(fwix_plan* plan, const void* a, const void* b, float* out, int add, int padded,
                           void* stream);

/* Every-depth FWI sweeps of the smooth step (no reference counterpart: the
 * reference's gradient is ExtendedBorn's adjoint, propagator/src/ExtendedBorn.cpp:
 * 122-150, whose piecewise-constant reference selection has no slowness
 * derivative).  The level loops of the FWI driver with every depth stored, each
 * on one stream; fields are [ns][nw][NY][NX], field blocks [nz] (dSU [nz-1]) of
 * them.  Needs fwix_plan_set_smooth / set_refs and a model (the reflections).
 * Model sweep: data = recorded down + up fields of the source injection (zeroed
 * first); Ds[iz] = the down field at iz after injection (the down recursion runs
 * in Ds itself); dSU[iz] = dS_iz(U_iz+1), the slowness derivative of the up
 * pass's step (dSU may be NULL); U a working field. */
fwix_status fwix_smooth_model_sweep(fwix_plan* plan, const fwix_traces* src, const fwix_traces* rec,
                                    const void* wavelet, void* data, void* U, void* Ds, void* dSU, void* stream);
/* Gradient sweep for the residual res [ntrace][nw]: gpad [nz][NY][NX] = the
 * slowness-derivative correlations (the padded gradient before folding the pad),
 * crefl [nz][ny][nx] = the correlations with the reflection coefficients, both
 * overwritten; Ds and dSU as the model sweep left them (dSU may be NULL only
 * when nz == 1); mus [nz] receives the mu field of every depth (the mu
 * recursion runs in it); nu, G working fields. */
fwix_status fwix_smooth_gradient_sweep(fwix_plan* plan, const fwix_traces* rec, const void* res, const void* Ds,
                                       const void* dSU, void* mus, void* nu, void* G, float* gpad, float* crefl,
                                       void* stream);

/* ---- acquisition ------------------------------------------------------------ */
/* Host coordinate arrays; ids are dense shot indices in [0, ns).  ntrace may be 0
 * (the arrays may then be NULL); a [ntrace][nw] trace buffer of an empty trace set
 * (wavelet, data) may be NULL in every call that takes one. */
fwix_status fwix_traces_create(fwix_plan* plan, int ntrace, const float* cx, const float* cy,
                               const float* cz, const int32_t* ids, fwix_traces** out);
fwix_status fwix_traces_destroy(fwix_traces* tr);
/* adjoint == 0: wfld (+)= inject(traces) at level iz (inj_forward);
 * adjoint != 0: traces (+)= record(wfld) (inj_adjoint). */
fwix_status fwix_inject(fwix_plan* plan, const fwix_traces* tr, int iz, int adjoint, void* traces,
                        void* wfld, int add, void* stream);

/* ---- depth sweeps ------------------------------------------------------------ */
/* Downward / Upward continuation in place over all nz levels. */
fwix_status fwix_downward(fwix_plan* plan, int adjoint, void* wfld, void* stream);
fwix_status fwix_upward(fwix_plan* plan, int adjoint, void* wfld, void* stream);
/* Nonlinear modelling wavelet -> data.  bg_down: [nz] wavefields, required (the up
 * pass reflects the down field of every depth); on return it holds the down field
 * of every depth.  bg_up: [nz] wavefields receiving the up field of every depth, or
 * NULL when the Born operators are not needed. */
fwix_status fwix_propagate(fwix_plan* plan, const fwix_traces* src, const fwix_traces* rec,
                           const void* wavelet, void* data, int add, void* bg_down, void* bg_up,
                           void* stream);
/* Lockstep migration image[nz][ny][nx] (float) (+)= sum_w Re sum_s conj(S) R.  The
 * sum over frequencies and shots is taken with float atomics in no fixed order:
 * repeated calls agree to rounding, not bit for bit. */
fwix_status fwix_migrate(fwix_plan* plan, const fwix_traces* src, const fwix_traces* rec,
                         const void* wavelet, const void* data, float* image, int add,
                         void* stream);
/* Extended Born: forward (dslow, dden) -> data, adjoint data -> (dslow, dden).
 * dslow/dden element (iz, iw, y, x) at iz*nw'*ny*nx + iw*model_w_stride + y*nx + x
 * with model_w_stride = ny*nx (nw' = nw, the reference domain [nz][nw][ny][nx]) or
 * 0 (nw' = 1: one perturbation per depth shared by every frequency; the adjoint
 * then returns the sum over frequency, the transpose of that broadcast). */
fwix_status fwix_born(fwix_plan* plan, int adjoint, const fwix_traces* rec, const void* bg_down,
                      const void* bg_up, void* dslow, void* dden, int64_t model_w_stride,
                      void* data, int add, void* stream);

/* ---- lossy background store ---------------------------------------------------
 * Replaces the role of the reference's ZFP-compressed background wavefields
 * (propagator/src/WavefieldPool.cpp:13-219, fixed rate "compress_rate" = 8 bits
 * per value) with this library's own fixed-rate format, kept in device memory:
 * blocks of 16 floats share an exponent byte and keep 8-bit mantissas (8.5 bits
 * per value, 3.76 x smaller than complex64; error at most 2^-7 of the block's
 * largest magnitude).  Not ZFP's bit stream.
 *   fwix_plan_set_pack_rate: 8 (default) or 16 mantissa bits per value for the
 *     plan's packed store (16.5 bits per value, 1.94 x smaller than complex64,
 *     error at most 2^-15 of a block's largest magnitude), used by everything
 *     below except the explicitly 8-bit fwix_pack_rate8 / fwix_unpack_rate8.
 *   fwix_plan_packed_bytes: bytes of one packed wavefield [ns][nw][NY][NX] at the
 *     plan's rate; [nz] packed wavefields are nz times that, depth iz at
 *     iz * packed_bytes.
 *   fwix_pack_wavefield / fwix_unpack_wavefield: one wavefield at the plan's rate;
 *   fwix_pack_rate8 / fwix_unpack_rate8: one wavefield at 8 bits (buffers 4-byte
 *     aligned; 16-byte aligned ones take the vector path).
 *   fwix_propagate_packed: fwix_propagate storing the down and up fields of every
 *     depth packed (packed_up may be NULL); the up pass reflects the unpacked down
 *     fields, as the reference's reflects its decompressed ones.
 *   fwix_born_packed: fwix_born reading packed backgrounds, each depth unpacked
 *     when first needed; workspace class FWIX_WS_BORN_PACKED. */
size_t fwix_plan_packed_bytes(const fwix_plan* plan);
fwix_status fwix_plan_set_pack_rate(fwix_plan* plan, int bits);
fwix_status fwix_pack_wavefield(fwix_plan* plan, const void* wfld, void* packed, void* stream);
fwix_status fwix_unpack_wavefield(fwix_plan* plan, const void* packed, void* wfld, void* stream);
fwix_status fwix_pack_rate8(fwix_plan* plan, const void* wfld, void* packed, void* stream);
fwix_status fwix_unpack_rate8(fwix_plan* plan, const void* packed, void* wfld, void* stream);
fwix_status fwix_propagate_packed(fwix_plan* plan, const fwix_traces* src, const fwix_traces* rec,
                                  const void* wavelet, void* data, int add, void* packed_down, void* packed_up,
                                  void* stream);
fwix_status fwix_born_packed(fwix_plan* plan, int adjoint, const fwix_traces* rec, const void* packed_down,
                             const void* packed_up, void* dslow, void* dden, int64_t model_w_stride, void* data,
                             int add, void* stream);

/* ---- one-call forms of the depth steps and the image --------------------------
 * fwix_pspi_step / fwix_nsps_step: PSPI::cu_forward / cu_adjoint
 * (propagator/src/PSPI.cpp:6-103) and NSPS (propagator/src/NSPS.cpp:6-45) at
 * level iz, overwriting psi_out (psi_in may equal psi_out).  adjoint: 0 forward,
 * 1 the add-version adjoint (PSPI.cpp:26-44, no taper), 2 the in-place adjoint
 * (PSPI.cpp:85-103, taper last); the same as fwix_step with that direction. */
fwix_status fwix_pspi_step(fwix_plan* plan, int iz, const void* psi_in, void* psi_out, int adjoint,
                           void* stream);
fwix_status fwix_nsps_step(fwix_plan* plan, int iz, const void* psi_in, void* psi_out, int adjoint,
                           void* stream);
/* Imaging condition of one level summed over frequency and shots
 * (imaging_condition.cu:57-108 with the sum over w of Scattering.cpp:104-111):
 * image[y][x] (+)= sum_w Re sum_s conj(S) R over the unpadded window; S, R are
 * wavefields [ns][nw][NY][NX], image is float [ny][nx]. */
fwix_status fwix_image_accumulate(fwix_plan* plan, const void* S, const void* R, float* image, int add,
                                  void* stream);

/* ---- batched sweeps over many instances --------------------------------------
 * fwix_sweep runs one sweep for each of ninst instances -- shots of their own
 * grid, band, references and buffers, each described by its plan and the
 * arrays below -- the way the reference's StreamingPropagator runs its
 * propagators on TBB threads, one CUDA stream each
 * (propagator/src/StreamingPropagator.cpp).  Instances are assigned largest
 * first (nx*ny*nw*nz*ns) to the least loaded of the nstreams streams given;
 * every stream first waits for the work already enqueued on `stream`, and
 * `stream` waits for all of them at the end, so the call is stream ordered on
 * `stream` like the others (and can be captured into a CUDA graph from it).
 * With nstreams == 0 everything runs on `stream`.  Instances must not share a
 * plan.  Per kind, the instance fields used:
 *   DOWN / UP  : wfld (in place), adjoint        fwix_downward / fwix_upward
 *   MODEL      : src, rec, wavelet, data, add, bg_down, bg_up   fwix_propagate
 *   IMAGE      : src, rec, wavelet, data, image, add            fwix_migrate
 *   BORN_FWD   : rec, bg_down, bg_up, dslow, dden, model_w_stride, data, add
 *   BORN_ADJ   : the same, data in, (dslow, dden) out           fwix_born */
enum { FWIX_SWEEP_DOWN = 0, FWIX_SWEEP_UP = 1, FWIX_SWEEP_MODEL = 2, FWIX_SWEEP_IMAGE = 3,
       FWIX_SWEEP_BORN_FWD = 4, FWIX_SWEEP_BORN_ADJ = 5 };
typedef struct fwix_instance {
  fwix_plan* plan;
  const fwix_traces* src;
  const fwix_traces* rec;
  const void* wavelet;
  void* data;
  void* wfld;
  float* image;
  void* bg_down;
  void* bg_up;
  void* dslow;
  void* dden;
  int64_t model_w_stride;
  int adjoint;
  int add;
} fwix_instance;
fwix_status fwix_sweep(int kind, const fwix_instance* insts, int ninst, void* const* streams, int nstreams,
                       void* stream);

/* ---- runtime tuning ----------------------------------------------------------
 * fwix_plan_autotune times the equivalent implementations of one depth step of
 * kind `kind` at level iz on the caller's wavefield (in -> out, distinct buffers;
 * refs and a FWIX_WS_STEP workspace bound) and keeps the fastest for every later
 * call of the plan: column tiles moved per thread (cp.async) or by TMA; all
 * slices (shot, frequency) in one launch, or halves / quarters of them, on the
 * caller's stream or alternating between it and a second stream of the plan
 * (forked and joined with events, so calls stay ordered on `stream` and can be
 * captured); for 256 x 256 slices the one-launch cluster step.  Each candidate runs once untimed,
 * then `reps` steps between CUDA events on `stream`.  It synchronises `stream`:
 * call it before any stream capture.  `result` (may be NULL) receives the choice. */
typedef struct fwix_tuning {
  int col_tma;                /* 1: TMA column tiles                               */
  int fused;                  /* 1: one-launch cluster step                        */
  int64_t slices_per_launch;  /* slices of one launch of each pass                 */
  float ms;                   /* time per step of the choice                       */
  int candidates;             /* candidates timed                                  */
  int streams;                /* 1, or 2: chunks alternate between two streams     */
} fwix_tuning;
fwix_status fwix_plan_autotune(fwix_plan* plan, int kind, int iz, const void* in, void* out, int reps, void* stream,
                               fwix_tuning* result);
/* fwix_plan_set_tuning applies a choice fwix_plan_autotune returned earlier (for a
 * plan of the same sizes) without timing anything: col_tma, fused,
 * slices_per_launch (1 .. ns * nw) and streams (1 or 2) are read, ms and
 * candidates ignored.  A later call whose workspace is too small for the
 * chosen slices per launch fails with FWIX_ERR_WORKSPACE. */
fwix_status fwix_plan_set_tuning(fwix_plan* plan, const fwix_tuning* tuning);

/* ---- allocation-free depth step ----------------------------------------------
 * fwix_step_noalloc has no counterpart in the reference.  It is fwix_step for
 * callers that cannot call cudaMalloc -- for example a host application or
 * framework that reserves the GPU's memory in its own pool up front and does not
 * let a library allocate (an allocation there would fail, fragment the pool or
 * stall the device).  It takes no plan and no workspace: the descriptor is read on
 * the host and the scratch (tables plus (nref + 1) wavefield-sized intermediates)
 * lives in one static device array of FWIX_NOALLOC_SCRATCH_BYTES that every GPU
 * loading this library holds until the process exits.  Larger problems are
 * rejected with FWIX_ERR_UNSUPPORTED and a message giving the bytes needed.
 * All calls share that array and it keeps the previous call's contents, so two
 * calls that overlap on the GPU (other streams, other host threads) race: order
 * them on one stream.  The first call on each device looks up the array's device
 * address (cudaGetSymbolAddress); make that first call before any stream capture.
 * The address is kept for the life of the process: do not call this entry point
 * on a device after a cudaDeviceReset of it (the array may then have moved).
 * sref / labels / strides are as in fwix_plan_set_refs; in may equal out. */
#define FWIX_NOALLOC_SCRATCH_BYTES (64ull * 1024ull * 1024ull)
fwix_status fwix_step_noalloc(const fwix_desc* desc, int kind, int iz, int dir, const void* sref,
                              const uint8_t* labels, int64_t labels_z_stride,
                              int64_t labels_w_stride, const void* in, void* out, int add,
                              void* stream);

#ifdef __cplusplus
}
#endif
#endif /* FWIX_B200_H */
