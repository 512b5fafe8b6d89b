// One PSPI / NSPS depth step of 256 x 256 slices in a single launch, the slice
// kept on chip: a thread-block cluster of 8 CTAs owns one (shot, frequency)
// slice, CTA r holding rows 32r .. 32r+31 in the row phases and columns
// 32r .. 32r+31 in the column phases.  Rows and columns change hands through
// distributed shared memory: a column pass reads its 256 samples from the 8
// CTAs' row buffers (sample y of a column sits in CTA y / 32 at local row
// y % 32), and the last row pass reads its rows back from the CTAs' column
// buffers.  HBM sees the input once, the output once, the labels and the phase
// factors; the per-reference intermediates never leave the cluster.
//
// Two orders, as in the three-launch passes:
//   kind B (sum in the spectrum: NSPS forward, PSPI adjoint)
//     per term: rows F_x(pre_term in) -> cluster exchange -> columns F_y,
//     times Q_term, summed in registers; then F_y^-1, exchange, F_x^-1, post.
//   kind A (split spectrum: PSPI forward, NSPS adjoint)
//     rows F_x(pre in) -> exchange -> columns F_y kept in registers; per term:
//     F_y^-1(Q_term spectrum) -> exchange -> rows F_x^-1, post_term, summed.
// Exchange buffers are double-buffered so one cluster barrier per term keeps
// every CTA from overwriting a buffer another CTA is still reading (each CTA
// reads buffer k only before it arrives at the barrier that precedes the next
// write of buffer k).  All barriers are the hardware cluster barrier, reached by
// every thread of every CTA the same number of times; there are no spin waits.
#include <cooperative_groups.h>

#include <mutex>

#include "fast.cuh"
#include "fwix_b200.h"

namespace cg = cooperative_groups;

namespace fwix {
namespace fused {

using P = fast::Plan<256, 8, fast::Radices<8, 8, 4>>;
constexpr int kRanks = 8;               // CTAs per cluster
constexpr int kLines = P::N / kRanks;   // rows / columns per CTA (= 32 = lanes per line)
constexpr int kWarps = 16;              // two adjacent lines per warp
constexpr int kPitch = P::N + 2;        // float2 between lines of an exchange buffer
constexpr int kBuf = kLines * kPitch;
static_assert(P::T == kLines, "a lane's samples of a line sit in distinct CTAs");
static_assert(kLines == 2 * kWarps, "two lines per warp");

inline size_t smem_bytes() {
  return (2 * (size_t)kBuf + (size_t)kWarps * P::N + fast::tw_size<P>()) * sizeof(float2);
}

struct Ctx {
  float2* buf0;  // exchange buffer k is buf0 + k * kBuf
  float2* line;
  float2* tw;
  int warp, t, rank;
  long long bl, b;
  int iw;
};

__device__ __forceinline__ Ctx make_ctx(const SpecArgs& a, float2* smem, int rank) {
  Ctx c;
  c.buf0 = smem;
  c.warp = threadIdx.x >> 5;
  c.t = threadIdx.x & 31;
  c.line = smem + 2 * kBuf + c.warp * P::N;
  c.tw = smem + 2 * kBuf + kWarps * P::N;
  c.rank = rank;
  c.bl = blockIdx.x / kRanks;
  c.b = a.b0 + c.bl;
  c.iw = (int)(c.b % a.d.nw);
  return c;
}

// Lanes' samples of local lines 2w and 2w+1 from the 8 CTAs' buffers.  Sample e
// of lane t sits at position t + 32 e in the input layout of a forward
// transform (LAST = false) and at t + 32 (e / 4) + 64 (e % 4) in its output
// layout (LAST = true): t plus a multiple of 32, so it is element (t, pos) of
// CTA (position - t) / 32's buffer, pos being the index of the line pair.
// Shared-memory address of `p` in CTA `rank` of the cluster (mapa), and 8- / 16-byte
// loads through the shared::cluster window (ld.shared::cluster).
__device__ __forceinline__ uint32_t cluster_addr(const void* p, int rank) {
  const uint32_t local = (uint32_t)__cvta_generic_to_shared(p);
  uint32_t remote;
  asm("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(remote) : "r"(local), "r"(rank));
  return remote;
}
__device__ __forceinline__ float4 ld_cluster4(uint32_t addr) {
  float4 v;
  asm volatile("ld.shared::cluster.v4.f32 {%0, %1, %2, %3}, [%4];\n"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"(addr));
  return v;
}
__device__ __forceinline__ float2 ld_cluster2(uint32_t addr) {
  float2 v;
  asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];\n" : "=f"(v.x), "=f"(v.y) : "r"(addr));
  return v;
}

template <bool LAST>
__device__ __forceinline__ void gather_pair(cg::cluster_group& cl, const float2* buf, int pos, int t,
                                            float2 (&v0)[P::E], float2 (&v1)[P::E]) {
  const float2* mine = buf + (size_t)t * kPitch + pos;
  float4 f[P::E];
#pragma unroll
  for (int e = 0; e < P::E; ++e) f[e] = ld_cluster4(cluster_addr(mine, LAST ? (e / 4 + 2 * (e % 4)) : e));
#pragma unroll
  for (int e = 0; e < P::E; ++e) {
    v0[e] = make_float2(f[e].x, f[e].y);
    v1[e] = make_float2(f[e].z, f[e].w);
  }
}

// One line (2w + j) of the pair, 8-byte loads.
template <bool LAST>
__device__ __forceinline__ void gather_one(cg::cluster_group& cl, const float2* buf, int pos, int t,
                                           float2 (&v)[P::E]) {
  const float2* mine = buf + (size_t)t * kPitch + pos;
#pragma unroll
  for (int e = 0; e < P::E; ++e) v[e] = ld_cluster2(cluster_addr(mine, LAST ? (e / 4 + 2 * (e % 4)) : e));
}

// Labels of this lane's samples of a row, four to a word.
__device__ __forceinline__ void load_labels(const SpecArgs& a, int iw, int y, int t, uint32_t (&w)[2]) {
  const uint8_t* lrow = a.lab + (long long)iw * a.lab_w + (long long)y * P::N;
  w[0] = w[1] = 0;
#pragma unroll
  for (int e = 0; e < P::E; ++e) w[e / 4] |= (uint32_t)lrow[fast::pos_first<P>(t, e)] << (8 * (e % 4));
}
__device__ __forceinline__ int label_of(const uint32_t (&w)[2], int e) { return (int)((w[e / 4] >> (8 * (e % 4))) & 0xffu); }

// kind B: out (+)= post F^-1(sum_term Q_term F(pre_term in)).
template <int PRE, int QM>
__global__ void __launch_bounds__(kWarps * 32, 1) k_fused_b(const SpecArgs a, int post_taper) {
  extern __shared__ __align__(16) float2 smem[];
  cg::cluster_group cl = cg::this_cluster();
  Ctx c = make_ctx(a, smem, (int)cl.block_rank());
  fast::load_stage_tw<P>(c.tw, a.twx);
  __syncthreads();
  const int nterm = a.nterm;
  const int yl = 2 * c.warp, y0 = c.rank * kLines + yl;
  uint32_t lab[2][2];
  if (PRE == W_MASK) {
    load_labels(a, c.iw, y0, c.t, lab[0]);
    load_labels(a, c.iw, y0 + 1, c.t, lab[1]);
  }
  const int x0 = c.rank * kLines + 2 * c.warp;  // this warp's two columns
  float2 acc[2][P::E];
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int e = 0; e < P::E; ++e) acc[j][e] = make_float2(0.f, 0.f);
  for (int term = 0; term < nterm; ++term) {
    float2* B = c.buf0 + (term & 1) * kBuf;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      // the rows are read again each term (from L2 after the first)
      const float2* src = a.in + (c.b * a.d.NY + y0 + j) * P::N;
      float2 v[P::E];
#pragma unroll
      for (int e = 0; e < P::E; ++e) {
        const int x = fast::pos_first<P>(c.t, e);
        if (PRE == W_MASK)
          v[e] = label_of(lab[j], e) == term ? src[x] : make_float2(0.f, 0.f);
        else
          v[e] = row_weight<PRE>(a, term, c.iw, y0 + j, x, src[x]);
      }
      fast::fft_fwd<P>(v, c.t, c.tw, c.line);
      __syncwarp();
#pragma unroll
      for (int e = 0; e < P::E; ++e) B[(yl + j) * kPitch + fast::pos_last<P>(c.t, e)] = v[e];
    }
    cl.sync();
    float2 v0[P::E], v1[P::E];
    gather_pair<false>(cl, B, x0, c.t, v0, v1);
    float2 q[P::E];
    fast::fft_fwd<P>(v0, c.t, c.tw, c.line);
    fast::col_factors<P, QM>(a, term, c.iw, x0, c.t, q);
#pragma unroll
    for (int e = 0; e < P::E; ++e) acc[0][e] = cadd(acc[0][e], cmul(v0[e], q[e]));
    __syncwarp();
    fast::fft_fwd<P>(v1, c.t, c.tw, c.line);
    fast::col_factors<P, QM>(a, term, c.iw, x0 + 1, c.t, q);
#pragma unroll
    for (int e = 0; e < P::E; ++e) acc[1][e] = cadd(acc[1][e], cmul(v1[e], q[e]));
    __syncwarp();
  }
  // inverse columns into the column buffer Y (column-major: local column, then row)
  float2* Y = c.buf0 + (nterm & 1) * kBuf;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    fast::fft_inv<P>(acc[j], c.t, c.tw, c.line);
    __syncwarp();
#pragma unroll
    for (int e = 0; e < P::E; ++e) Y[(2 * c.warp + j) * kPitch + fast::pos_first<P>(c.t, e)] = acc[j][e];
  }
  cl.sync();
  float2 v0[P::E], v1[P::E];
  gather_pair<true>(cl, Y, y0, c.t, v0, v1);
  auto finish = [&](float2(&w)[P::E], int j) {
    fast::fft_inv<P>(w, c.t, c.tw, c.line);
    __syncwarp();
    float2* dst = a.out + (c.b * a.d.NY + y0 + j) * P::N;
    const float ty = post_taper ? a.tapy[y0 + j] : 1.f;
#pragma unroll
    for (int e = 0; e < P::E; ++e) {
      const int x = fast::pos_first<P>(c.t, e);
      float2 r = w[e];
      if (post_taper) r = cscale(r, a.tapx[x] * ty);
      if (a.add) r = cadd(dst[x], r);
      dst[x] = r;
    }
  };
  finish(v0, 0);
  finish(v1, 1);
  cl.sync();  // no CTA leaves while another may still read its buffers
}

// kind A: out (+)= sum_term post_term F^-1(Q_term F(pre in)).
template <int PRE, int QM, int POST>
__global__ void __launch_bounds__(kWarps * 32, 1) k_fused_a(const SpecArgs a) {
  extern __shared__ __align__(16) float2 smem[];
  cg::cluster_group cl = cg::this_cluster();
  Ctx c = make_ctx(a, smem, (int)cl.block_rank());
  fast::load_stage_tw<P>(c.tw, a.twx);
  __syncthreads();
  const int nterm = a.nterm;
  const int yl = 2 * c.warp, y0 = c.rank * kLines + yl;
  const int x0 = c.rank * kLines + 2 * c.warp;
  // forward rows into buffer 0
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const float2* src = a.in + (c.b * a.d.NY + y0 + j) * P::N;
    float2 v[P::E];
#pragma unroll
    for (int e = 0; e < P::E; ++e) {
      const int x = fast::pos_first<P>(c.t, e);
      v[e] = row_weight<PRE>(a, 0, c.iw, y0 + j, x, src[x]);
    }
    fast::fft_fwd<P>(v, c.t, c.tw, c.line);
    __syncwarp();
#pragma unroll
    for (int e = 0; e < P::E; ++e) c.buf0[(yl + j) * kPitch + fast::pos_last<P>(c.t, e)] = v[e];
  }
  cl.sync();
  float2 S[2][P::E];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    gather_one<false>(cl, c.buf0, x0 + j, c.t, S[j]);
    fast::fft_fwd<P>(S[j], c.t, c.tw, c.line);
    __syncwarp();
  }
  uint32_t lab[2][2];
  if (POST == W_MASK) {
    load_labels(a, c.iw, y0, c.t, lab[0]);
    load_labels(a, c.iw, y0 + 1, c.t, lab[1]);
  }
  float2 acc[2][P::E];
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int e = 0; e < P::E; ++e) acc[j][e] = make_float2(0.f, 0.f);
  for (int term = 0; term < nterm; ++term) {
    float2* Y = c.buf0 + ((term + 1) & 1) * kBuf;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      float2 q[P::E], v[P::E];
      fast::col_factors<P, QM>(a, term, c.iw, x0 + j, c.t, q);
#pragma unroll
      for (int e = 0; e < P::E; ++e) v[e] = cmul(S[j][e], q[e]);
      fast::fft_inv<P>(v, c.t, c.tw, c.line);
      __syncwarp();
#pragma unroll
      for (int e = 0; e < P::E; ++e) Y[(2 * c.warp + j) * kPitch + fast::pos_first<P>(c.t, e)] = v[e];
    }
    cl.sync();
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      float2 v[P::E];
      gather_one<true>(cl, Y, y0 + j, c.t, v);
      fast::fft_inv<P>(v, c.t, c.tw, c.line);
      __syncwarp();
#pragma unroll
      for (int e = 0; e < P::E; ++e) {
        if (POST == W_MASK) {
          if (label_of(lab[j], e) == term) acc[j][e] = v[e];
        } else {
          acc[j][e] = cadd(acc[j][e], row_weight<POST>(a, term, c.iw, y0 + j, fast::pos_first<P>(c.t, e), v[e]));
        }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    float2* dst = a.out + (c.b * a.d.NY + y0 + j) * P::N;
#pragma unroll
    for (int e = 0; e < P::E; ++e) {
      const int x = fast::pos_first<P>(c.t, e);
      dst[x] = a.add ? cadd(dst[x], acc[j][e]) : acc[j][e];
    }
  }
  cl.sync();  // no CTA leaves while another may still read its buffers
}

template <class K, class... Args>
cudaError_t launch_cluster(K kernel, const SpecArgs& a, cudaStream_t s, Args... args) {
  const size_t sm = smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(a.nb * kRanks));
  cfg.blockDim = dim3(kWarps * 32);
  cfg.dynamicSmemBytes = sm;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kRanks;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  e = cudaLaunchKernelEx(&cfg, kernel, a, args...);
  if (e == cudaSuccess) count_launch();
  return e != cudaSuccess ? e : cudaGetLastError();
}

}  // namespace fused

// Whether this device can run 8-CTA clusters of the fused step (checked once per
// device: a cluster of 8 CTAs with the fused step's shared memory must fit).
bool fused_step_available() {
  static std::mutex mu;
  static int state[64];  // 0 unknown, 1 yes, 2 no
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
  std::lock_guard<std::mutex> lock(mu);
  if (state[dev] == 0) {
    auto k = fused::k_fused_b<W_MASK, Q_PS_FWD>;
    const size_t sm = fused::smem_bytes();
    int n = 0;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(fused::kRanks);
    cfg.blockDim = dim3(fused::kWarps * 32);
    cfg.dynamicSmemBytes = sm;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = fused::kRanks;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    bool ok = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) == cudaSuccess &&
              cudaOccupancyMaxActiveClusters(&n, k, &cfg) == cudaSuccess && n > 0;
    cudaGetLastError();  // clear a refusal so that it does not surface later
    state[dev] = ok ? 1 : 2;
  }
  return state[dev] == 1;
}

// One depth step of 256 x 256 slices (PSPI.cpp:6-103, NSPS.cpp:6-45) in one launch.
cudaError_t fused_step(const SpecArgs& a, int kind, int dir, cudaStream_t s) {
  using namespace fused;
  if (kind == FWIX_STEP_PSPI) {
    if (dir == FWIX_FWD) return launch_cluster(k_fused_a<W_TAPER, Q_PS_FWD, W_MASK>, a, s);
    return launch_cluster(k_fused_b<W_MASK, Q_PS_ADJ>, a, s, dir == FWIX_ADJ_INPL ? 1 : 0);
  }
  if (dir == FWIX_FWD) return launch_cluster(k_fused_b<W_MASK, Q_PS_FWD>, a, s, 0);
  return launch_cluster(k_fused_a<W_ONE, Q_PS_ADJ, W_MASK>, a, s);
}

}  // namespace fwix
