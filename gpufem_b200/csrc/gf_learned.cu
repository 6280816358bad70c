// Learned preconditioner: a message-passing network over the node graph of K,
// trained on the GPU by the kernels below, used inside flexible CG.
// No counterpart in the reference (its CG is unpreconditioned,
// src/SPRmatrix/SPRmatrix.cc:405-480).
//
// M(r) = D^-1 r + c * y(r),   rho = D^-1 r (Jacobi), c = rms(rho),
// v1 = D^-1 K rho, v2 = D^-1 K v1 (two matrix hops, so the network sees K itself),
// y = network(features) with per-node features
//   [rho_a / c (dim), v1_a / c (dim), v2_a / c (dim), log(d_a / mean d) (dim)]:
//   h0 = relu(W0 f + b0)                                   (4 dim -> 64)
//   h_{l+1} = relu(Ws_l h_l + Wn_l mean_{b in N(a)} h_l[b] + b_l),  l = 0, 1, 2   (64 -> 64)
//   y = Wout h3 + bout                                     (64 -> dim)
// N(a) = nodes sharing an element with a (the ELL node adjacency, self included).
// Weights are kept in FP32 (Adam master copy) and used as BF16; activations and
// accumulation are FP32.  The dense layers (and their data gradients) run on the tcgen05
// tensor cores (k_lp_mm_tc): activations split into TF32 hi + lo, BF16 weights exact in
// TF32, FP32 accumulation in TMEM.  Wout starts at zero, so an untrained network is Jacobi.
// The output scale c makes M(s r) = s M(r).
//
// Training pairs (r_k, e_k = u* - x_k) come from Jacobi-PCG runs on the context's
// matrix (u* = a tighter PCG solution).  Loss per pair, z = M(r_k):
//   GF_LP_LOSS_ERROR:    L = sum d (z - e)^2 / sum d e^2             (D-weighted error)
//   GF_LP_LOSS_RESIDUAL: L = sum (K (e - z))^2 / d / sum (K e)^2 / d  (residual left by M)
#include <cuda_bf16.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "gf_internal.cuh"
#include "gf_tc.cuh"

namespace {

constexpr int H = 64;       // hidden width
constexpr int kLT = 256;    // threads per block
constexpr int kLayers = 3;  // message-passing layers

struct LpOffsets {
  int64_t W0, b0, Ws[kLayers], Wn[kLayers], bl[kLayers], Wout, bout, total;
};

LpOffsets lp_offsets(int dim) {
  LpOffsets o{};
  const int F = 4 * dim;
  int64_t p = 0;
  o.W0 = p; p += (int64_t)H * F;
  o.b0 = p; p += H;
  for (int l = 0; l < kLayers; ++l) {
    o.Ws[l] = p; p += (int64_t)H * H;
    o.Wn[l] = p; p += (int64_t)H * H;
    o.bl[l] = p; p += H;
  }
  o.Wout = p; p += (int64_t)dim * H;
  o.bout = p; p += dim;
  o.total = p;
  return o;
}

struct LpScalars {
  double sumsq;   // sum rho^2
  double c;       // rms(rho)
  double loss;    // accumulated loss
  double dsum;    // loss normaliser (sum d e^2, or sum (K e)^2 / d)
};

}  // namespace

// Per-context learned-preconditioner state.
struct LpState {
  int dim = 0, N = 0, n = 0;
  LpOffsets off{};
  float* w = nullptr;       // FP32 master weights
  __nv_bfloat16* wb = nullptr;  // BF16 copy used by the network
  float* g = nullptr;       // gradients
  float* m = nullptr;       // Adam moments
  float* v = nullptr;
  int64_t adam_t = 0;
  // node graph
  float* deg_inv = nullptr;  // 1 / |N(a)|
  // per-dof
  float* dinv = nullptr;     // 1 / K_rr (FP32)
  double* dinv64 = nullptr;
  float* dlog = nullptr;     // log(d / mean d)
  float* dvec = nullptr;     // d (loss weight)
  // activations [N][H] (pre-activations kept for the ReLU masks)
  float* feat = nullptr;     // [N][4 dim]
  float* v1 = nullptr;       // [n] D^-1 K rho
  float* v2 = nullptr;       // [n] D^-1 K v1
  float* lw = nullptr;       // [n] residual loss scratch: e - z, then D^-1 s
  float* ls = nullptr;       // [n] s = K (e - z)
  float* lt = nullptr;       // [n] K e, then K D^-1 s
  float* pre[kLayers + 1] = {};
  float* h[kLayers + 1] = {};
  float* agg[kLayers] = {};
  float* y = nullptr;        // [N][dim] == n
  float* dy = nullptr;       // [n] loss gradient w.r.t. y
  float* rho = nullptr;      // [n]
  float* dh = nullptr;       // [N][H]
  float* dpre = nullptr;     // [N][H]
  float* tmp = nullptr;      // [N][H]
  LpScalars* sc = nullptr;
  // training pairs
  int npairs = 0;
  float* pr = nullptr;       // [npairs][n]
  float* pe = nullptr;       // [npairs][n]
  int* err = nullptr;        // set by a tensor-core layer whose MMA wait timed out
  bool ready = false;        // diag / graph set up for the current matrix
  bool coarse = false;       // with the two-level coarse correction (gf_lp_set_coarse)
  int loss = GF_LP_LOSS_ERROR;
};

namespace {

template <typename T>
gf_status lp_alloc(gf_ctx* ctx, T** p, size_t count) {
  return gf_alloc(ctx, p, count);
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
__device__ inline double lp_block_sum(double x, double* sh) {
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = x;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  }
  return s;
}

// rho = dinv * r, sum rho^2
__global__ void k_lp_prep(int n, const float* __restrict__ r, const float* __restrict__ dinv,
                          float* __restrict__ rho, LpScalars* sc) {
  __shared__ double sh[32];
  const int i = blockIdx.x * kLT + threadIdx.x;
  double s = 0.0;
  if (i < n) {
    const float v = r[i] * dinv[i];
    rho[i] = v;
    s = (double)v * v;
  }
  s = lp_block_sum(s, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->sumsq, s);
}

__global__ void k_lp_features(int N, int dim, const float* __restrict__ rho,
                              const float* __restrict__ v1, const float* __restrict__ v2,
                              const float* __restrict__ dlog, float* __restrict__ feat,
                              LpScalars* sc) {
  const int a = blockIdx.x * kLT + threadIdx.x;
  const double n = (double)N * dim;
  const double c = sqrt(sc->sumsq / n) + 1e-30;
  if (blockIdx.x == 0 && threadIdx.x == 0) sc->c = c;
  if (a >= N) return;
  const float ic = (float)(1.0 / c);
  float* f = feat + (int64_t)a * 4 * dim;
  for (int k = 0; k < dim; ++k) {
    f[k] = rho[a * dim + k] * ic;
    f[dim + k] = v1[a * dim + k] * ic;
    f[2 * dim + k] = v2[a * dim + k] * ic;
    f[3 * dim + k] = dlog[a * dim + k];
  }
}

// ---- dense layers on the tcgen05 tensor cores ----------------------------------------
// out[a][o] = act(bias[o] + sum_k W1[o][k] X1[a][k] (+ sum_k W2[o][k] X2[a][k]))   (WT = false)
// out[a][o] (+)= sum_k W1[k][o] X1[a][k]                                        (WT = true:
//   the data gradient of a layer whose weight is [KD][NO] row-major, read transposed)
// as D = X W^T on the tensor cores: a CTA takes tiles of 128 nodes (M = 128 TMEM lanes, a
// thread per node in the epilogue), N = NO padded to 16 output channels, K = KD padded to 8
// input channels per part (X1, then X2).  X is split into TF32 hi + lo parts and the BF16
// weights are exact in TF32, so the two products X_lo W^T + X_hi W^T give FP32 accuracy
// with FP32 accumulation in TMEM.
constexpr int kMmThreads = 128;
constexpr int kMmWaitIters = 1 << 20;

__host__ __device__ constexpr int mm_pad16(int x) { return x < 16 ? 16 : (x + 15) / 16 * 16; }
__host__ __device__ constexpr int mm_pad8(int x) { return (x + 7) / 8 * 8; }
__host__ __device__ constexpr int mm_tmem_cols(int n) { return n <= 32 ? 32 : n <= 64 ? 64 : 128; }

// row stride of the output staging tile: NO + 4 floats when rows are moved as 16-byte
// vectors (NO a multiple of 4), else NO + 1 (conflict-free scalar accesses)
__host__ __device__ constexpr int mm_stage_stride(int no) { return no % 4 == 0 ? no + 4 : no + 1; }

// X hi/lo tiles, reused after the MMAs as the output staging tile [128][stride]
template <int KD, int NO>
__host__ __device__ constexpr size_t mm_xbytes() {
  return (size_t)2 * 128 * mm_pad8(KD) * 4 > (size_t)128 * mm_stage_stride(NO) * 4
             ? (size_t)2 * 128 * mm_pad8(KD) * 4 : (size_t)128 * mm_stage_stride(NO) * 4;
}

template <int KD, int NO, bool TWO>
__host__ __device__ constexpr size_t mm_smem_bytes() {
  constexpr int KDP = mm_pad8(KD), NOP = mm_pad16(NO), P = TWO ? 2 : 1;
  return (mm_xbytes<KD, NO>() + 15) / 16 * 16  // X hi, lo / output staging
         + (size_t)P * NOP * KDP * 4        // W parts
         + (size_t)NOP * 4 + 16;            // bias, mbarrier, TMEM address
}

template <int KD, int NO, bool TWO, bool WT>
__global__ void __launch_bounds__(kMmThreads)
k_lp_mm_tc(int N, const float* __restrict__ X1, const float* __restrict__ X2,
           const __nv_bfloat16* __restrict__ W1, const __nv_bfloat16* __restrict__ W2,
           const __nv_bfloat16* __restrict__ bias, float* __restrict__ pre,
           float* __restrict__ out, int relu, int accumulate, int* __restrict__ err) {
  constexpr int KDP = mm_pad8(KD), NOP = mm_pad16(NO), P = TWO ? 2 : 1;
  constexpr int NCH = KDP / 4;                 // 16-byte K chunks per row
  constexpr uint32_t COLS = mm_tmem_cols(NOP);
  extern __shared__ __align__(1024) unsigned char smem[];
  float* xh = reinterpret_cast<float*>(smem);
  float* xl = xh + 128 * KDP;
  float* stage = xh;                           // [128][NO + 1] after the MMAs
  float* wt = reinterpret_cast<float*>(smem + (mm_xbytes<KD, NO>() + 15) / 16 * 16);
  float* sb = wt + P * NOP * KDP;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sb + NOP);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if constexpr (!WT && KD % 4 == 0) {
    // four consecutive k of one output channel per 8-byte load, all loads in flight at once
    constexpr int NQ = P * NOP * KDP / 4;
    constexpr int PER = (NQ + kMmThreads - 1) / kMmThreads;
    uint2 wv[PER];
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int q = tid + u * kMmThreads;
      const int p = q / (NOP * KDP / 4), rem = q % (NOP * KDP / 4);
      const int n = rem / (KDP / 4), k = (rem % (KDP / 4)) * 4;
      wv[u] = make_uint2(0u, 0u);
      if (q < NQ && n < NO && k < KD)
        wv[u] = __ldg(reinterpret_cast<const uint2*>((p == 0 ? W1 : W2) + (int64_t)n * KD + k));
    }
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int q = tid + u * kMmThreads;
      if (q < NQ) {
        const int p = q / (NOP * KDP / 4), rem = q % (NOP * KDP / 4);
        const int n = rem / (KDP / 4), k = (rem % (KDP / 4)) * 4;
        const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&wv[u].x));
        const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&wv[u].y));
        *reinterpret_cast<float4*>(wt + p * NOP * KDP + (k >> 2) * NOP * 4 + n * 4) =
            make_float4(lo.x, lo.y, hi.x, hi.y);
      }
    }
  } else {
#pragma unroll 8
    for (int q = tid; q < P * NOP * KDP; q += kMmThreads) {   // unrolled: the loads overlap
      const int p = q / (NOP * KDP), rem = q % (NOP * KDP);
      const int n = rem / KDP, k = rem % KDP;
      float v = 0.f;
      if (n < NO && k < KD) {
        const __nv_bfloat16* W = p == 0 ? W1 : W2;
        v = __bfloat162float(WT ? W[(int64_t)k * NO + n] : W[(int64_t)n * KD + k]);
      }
      wt[p * NOP * KDP + (k >> 2) * NOP * 4 + n * 4 + (k & 3)] = v;
    }
  }
  for (int q = tid; q < NOP; q += kMmThreads)
    sb[q] = (bias && q < NO) ? __bfloat162float(bias[q]) : 0.f;
  if (warp == 0) tc_alloc(tslot, COLS);
  if (tid == 0) tc_mbar_init(mbar);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  constexpr uint32_t idesc = tc_idesc_tf32(128, NOP);
  uint32_t phase = 0;
  bool ok = true;
  const int ntiles = (N + 127) / 128;
  // steps = (tile, part) pairs of this CTA; the X loads of the next step are issued right
  // after the current step's MMAs, so they are in flight during the MMA wait and the
  // epilogue
  const int mytiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int nsteps = mytiles * P;
  float4 xv[NCH];
  auto chunk_of = [&](int q, int& r, int& c) {
    // a warp takes 8 rows x 4 chunks (when NCH >= 4): 64 contiguous bytes of each of 8
    // rows in global memory, a 4-way bank conflict at most in shared memory
    if constexpr (NCH % 4 == 0) {
      const int ln = q & 31, wq = q >> 5;
      r = (wq & 15) * 8 + (ln & 7);
      c = (wq >> 4) * 4 + (ln >> 3);
    } else {
      r = q & 127;
      c = q >> 7;
    }
  };
  auto load_step = [&](int st) {
    // every thread issues all its loads of the tile part before using any (NCH 16-byte
    // chunks per row, 128 * NCH / 128 = NCH per thread): one round of memory latency
    const int a0s = (blockIdx.x + (st / P) * gridDim.x) * 128;
    const float* X = st % P == 0 ? X1 : X2;
#pragma unroll
    for (int u = 0; u < NCH; ++u) {
      int r, c;
      chunk_of(tid + u * kMmThreads, r, c);
      const int a = a0s + r;
      if constexpr (KD % 4 == 0) {
        xv[u] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (a < N && 4 * c < KD)
          xv[u] = __ldg(reinterpret_cast<const float4*>(X + (int64_t)a * KD) + c);
      } else {
        float* v = &xv[u].x;
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          const int k = 4 * c + w;
          v[w] = (a < N && k < KD) ? __ldg(X + (int64_t)a * KD + k) : 0.f;
        }
      }
    }
  };
  if (nsteps > 0) load_step(0);
  for (int st = 0; st < nsteps && ok; ++st) {
    const int p = st % P;
    const int a0 = (blockIdx.x + (st / P) * gridDim.x) * 128;
#pragma unroll
    for (int u = 0; u < NCH; ++u) {
      int r, c;
      chunk_of(tid + u * kMmThreads, r, c);
      const float* v = &xv[u].x;
      float4 h, l;
      float* hp = &h.x;
      float* lp = &l.x;
#pragma unroll
      for (int w = 0; w < 4; ++w) {
        const uint32_t hb = tc_tf32_round(v[w]);
        hp[w] = __uint_as_float(hb);
        lp[w] = __uint_as_float(tc_tf32_round(v[w] - __uint_as_float(hb)));
      }
      *reinterpret_cast<float4*>(xh + c * 512 + r * 4) = h;
      *reinterpret_cast<float4*>(xl + c * 512 + r * 4) = l;
    }
    tc_fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      const uint32_t ah = tc_smem_u32(xh), al = tc_smem_u32(xl);
      const uint32_t bw = tc_smem_u32(wt + p * NOP * KDP);
      for (int ks = 0; ks < KDP / 8; ++ks) {
        const uint64_t db = tc_desc(bw + ks * 2 * NOP * 16, NOP * 16, 128);
        tc_mma_tf32(tmem, tc_desc(al + ks * 2 * 128 * 16, 128 * 16, 128), db, idesc,
                    (p > 0 || ks > 0) ? 1u : 0u);
        tc_mma_tf32(tmem, tc_desc(ah + ks * 2 * 128 * 16, 128 * 16, 128), db, idesc, 1u);
      }
      tc_commit(mbar);
    }
    if (st + 1 < nsteps) load_step(st + 1);
    // the X tiles are rewritten by the next step (or the staging) only after these MMAs
    const bool done = tc_mbar_wait(mbar, phase, kMmWaitIters);
    phase ^= 1u;
    if (!done && lane == 0) atomicExch(err, 1);
    ok = __syncthreads_and(done);
    tc_fence_after();
    if (p < P - 1) continue;
    if (!ok) break;
    // epilogue: a thread per node (TMEM lane), its NO output channels
    const int a = a0 + warp * 32 + lane;
    float acc[NOP];
    if constexpr (NOP >= 32) {
#pragma unroll
      for (int c0 = 0; c0 < NOP; c0 += 32) {
        float t[32];
        tc_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, t);
#pragma unroll
        for (int j = 0; j < 32; ++j) acc[c0 + j] = t[j];
      }
    } else {
      float t[16];
      tc_ld16(tmem + ((uint32_t)(warp * 32) << 16), t);
#pragma unroll
      for (int j = 0; j < 16; ++j) acc[j] = t[j];
    }
    tc_wait_ld();
    (void)a;
    // stage the tile's outputs in shared memory, then store them with consecutive threads
    // on consecutive channels (coalesced; 16-byte vectors when NO is a multiple of 4)
    const int rr = warp * 32 + lane;
    constexpr int SS = mm_stage_stride(NO);
    if constexpr (NO % 4 == 0) {
#pragma unroll
      for (int c = 0; c < NO; c += 4)
        *reinterpret_cast<float4*>(stage + rr * SS + c) =
            make_float4(acc[c] + sb[c], acc[c + 1] + sb[c + 1], acc[c + 2] + sb[c + 2],
                        acc[c + 3] + sb[c + 3]);
    } else {
#pragma unroll
      for (int c = 0; c < NO; ++c) stage[rr * SS + c] = acc[c] + sb[c];
    }
    tc_fence_before();
    __syncthreads();
    if constexpr (NO % 4 == 0) {
      constexpr int NV = NO / 4;
      for (int q = tid; q < 128 * NV; q += kMmThreads) {
        const int r = q / NV, c = (q - r * NV) * 4;
        const int an = a0 + r;
        if (an < N) {
          const float4 v = *reinterpret_cast<const float4*>(stage + r * SS + c);
          const int64_t o = (int64_t)an * NO + c;
          if (pre) *reinterpret_cast<float4*>(pre + o) = v;
          float4 y = v;
          if (relu) {
            y.x = fmaxf(y.x, 0.f); y.y = fmaxf(y.y, 0.f);
            y.z = fmaxf(y.z, 0.f); y.w = fmaxf(y.w, 0.f);
          }
          if (accumulate) {
            const float4 o4 = *reinterpret_cast<const float4*>(out + o);
            y.x += o4.x; y.y += o4.y; y.z += o4.z; y.w += o4.w;
          }
          *reinterpret_cast<float4*>(out + o) = y;
        }
      }
    } else {
      for (int q = tid; q < 128 * NO; q += kMmThreads) {
        const int r = q / NO, c = q - r * NO;
        const int an = a0 + r;
        if (an < N) {
          const float v = stage[r * SS + c];
          const int64_t o = (int64_t)an * NO + c;
          if (pre) pre[o] = v;
          const float y = (relu && v < 0.f) ? 0.f : v;
          out[o] = accumulate ? out[o] + y : y;
        }
      }
    }
    __syncthreads();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tc_dealloc(tmem, COLS);
}

// Weight gradient: dW[o][k] += sum_a G[a][o] A[a][k]; db[o] += sum_a G[a][o].
// Block handles a chunk of nodes staged in shared memory.
template <int CIN, int COUT>
__global__ void __launch_bounds__(kLT)
k_lp_wgrad(int N, const float* __restrict__ G, const float* __restrict__ A,
           float* __restrict__ dW, float* __restrict__ db) {
  constexpr int CHUNK = 32;
  __shared__ float sG[CHUNK][COUT + 1];
  __shared__ float sA[CHUNK][CIN + 1];
  constexpr int PAIRS = COUT * CIN;
  constexpr int PER = (PAIRS + kLT - 1) / kLT;
  float acc[PER];
  float accb = 0.f;
#pragma unroll
  for (int k = 0; k < PER; ++k) acc[k] = 0.f;
  for (int a0 = blockIdx.x * CHUNK; a0 < N; a0 += gridDim.x * CHUNK) {
    const int na = min(CHUNK, N - a0);
    __syncthreads();
    for (int k = threadIdx.x; k < CHUNK * COUT; k += kLT) {
      const int r = k / COUT, c = k % COUT;
      sG[r][c] = r < na ? G[(int64_t)(a0 + r) * COUT + c] : 0.f;
    }
    for (int k = threadIdx.x; k < CHUNK * CIN; k += kLT) {
      const int r = k / CIN, c = k % CIN;
      sA[r][c] = r < na ? A[(int64_t)(a0 + r) * CIN + c] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int pidx = threadIdx.x + k * kLT;
      if (pidx < PAIRS) {
        const int o = pidx / CIN, c = pidx % CIN;
        float s = 0.f;
#pragma unroll 8
        for (int r = 0; r < CHUNK; ++r) s += sG[r][o] * sA[r][c];
        acc[k] += s;
      }
    }
    if (threadIdx.x < COUT) {
      float s = 0.f;
      for (int r = 0; r < CHUNK; ++r) s += sG[r][threadIdx.x];
      accb += s;
    }
  }
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int pidx = threadIdx.x + k * kLT;
    if (pidx < PAIRS) atomicAdd(&dW[pidx], acc[k]);
  }
  if (threadIdx.x < COUT) atomicAdd(&db[threadIdx.x], accb);
}

// forward:  out[a] = deg_inv[a] * sum_{b in N(a)} h[b]
// backward: out[b] = sum_{a in N(b)} deg_inv[a] * g[a]   (the node graph is symmetric)
// 16 threads per node, 4 channels (16 bytes) each, neighbours summed in adjacency order.
// A CTA walks a contiguous range of per_cta nodes, 16 at a time: mesh numberings keep
// neighbours close, so the rows that the next nodes read again were just read and are
// still in L1.
constexpr int kAggNodes = kLT / 16;

__global__ void __launch_bounds__(kLT)
k_lp_aggregate(int N, int per_cta, const int32_t* __restrict__ adj_off,
               const int32_t* __restrict__ adj, const float* __restrict__ deg_inv,
               const float* __restrict__ h, float* __restrict__ out, int backward) {
  const int sub = threadIdx.x >> 4, c4 = threadIdx.x & 15;
  const int a_end = min(N, (blockIdx.x + 1) * per_cta);
  for (int a = blockIdx.x * per_cta + sub; a < a_end; a += kAggNodes) {
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
    const int q1 = adj_off[a + 1];
#pragma unroll 4
    for (int q = adj_off[a]; q < q1; ++q) {   // unrolled: the neighbours' gathers overlap
      const int b = __ldg(adj + q);
      float4 v = __ldg(reinterpret_cast<const float4*>(h + (int64_t)b * H) + c4);
      if (backward) {
        const float w = __ldg(deg_inv + b);
        v.x *= w; v.y *= w; v.z *= w; v.w *= w;
      }
      s.x += v.x; s.y += v.y; s.z += v.z; s.w += v.w;
    }
    if (!backward) {
      const float w = deg_inv[a];
      s.x *= w; s.y *= w; s.z *= w; s.w *= w;
    }
    reinterpret_cast<float4*>(out + (int64_t)a * H)[c4] = s;
  }
}

__global__ void k_lp_relu_grad(int64_t total, const float* __restrict__ dh,
                               const float* __restrict__ pre, float* __restrict__ dpre) {
  for (int64_t t = blockIdx.x * (int64_t)kLT + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * kLT)
    dpre[t] = pre[t] > 0.f ? dh[t] : 0.f;
}

// z = rho + c y, in FP32 or FP64
template <typename V>
__global__ void k_lp_output(int n, const float* __restrict__ rho, const float* __restrict__ y,
                            const LpScalars* __restrict__ sc, V* __restrict__ z) {
  const int i = blockIdx.x * kLT + threadIdx.x;
  if (i < n) z[i] = (V)rho[i] + (V)sc->c * (V)y[i];
}

// Loss for one pair: t = e - rho; L = sum d (c y - t)^2 / sum d e^2; dy = dL/dy
__global__ void k_lp_loss_sums(int n, const float* __restrict__ e, const float* __restrict__ d,
                               LpScalars* sc) {
  __shared__ double sh[32];
  const int i = blockIdx.x * kLT + threadIdx.x;
  double s = 0.0;
  if (i < n) s = (double)d[i] * e[i] * e[i];
  s = lp_block_sum(s, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->dsum, s);
}

__global__ void k_lp_loss_grad(int n, const float* __restrict__ e, const float* __restrict__ rho,
                               const float* __restrict__ y, const float* __restrict__ d,
                               float* __restrict__ dy, LpScalars* sc, double* loss_acc) {
  __shared__ double sh[32];
  const int i = blockIdx.x * kLT + threadIdx.x;
  const double c = sc->c, S = sc->dsum > 0 ? sc->dsum : 1.0;
  double l = 0.0;
  if (i < n) {
    const double diff = c * y[i] - ((double)e[i] - rho[i]);
    l = d[i] * diff * diff / S;
    dy[i] = (float)(2.0 * d[i] * c * diff / S);
  }
  l = lp_block_sum(l, sh);
  if (threadIdx.x == 0) atomicAdd(loss_acc, l);
}

// Residual loss: w = e - z (z = rho + c y)
__global__ void k_lp_rl_diff(int n, const float* __restrict__ e, const float* __restrict__ rho,
                             const float* __restrict__ y, const LpScalars* __restrict__ sc,
                             float* __restrict__ w) {
  const int i = blockIdx.x * kLT + threadIdx.x;
  if (i < n) w[i] = (float)((double)e[i] - ((double)rho[i] + sc->c * (double)y[i]));
}

// normaliser: sum t^2 / d with t = K e
__global__ void k_lp_rl_sums(int n, const float* __restrict__ t, const float* __restrict__ dinv,
                             LpScalars* sc) {
  __shared__ double sh[32];
  const int i = blockIdx.x * kLT + threadIdx.x;
  double s = 0.0;
  if (i < n) s = (double)dinv[i] * t[i] * t[i];
  s = lp_block_sum(s, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->dsum, s);
}

// loss += sum s^2 / d / S; g = s / d (the SpMV after it forms K g)
__global__ void k_lp_rl_loss(int n, const float* __restrict__ s_, const float* __restrict__ dinv,
                             const LpScalars* __restrict__ sc, float* __restrict__ g,
                             double* loss_acc) {
  __shared__ double sh[32];
  const int i = blockIdx.x * kLT + threadIdx.x;
  const double S = sc->dsum > 0 ? sc->dsum : 1.0;
  double l = 0.0;
  if (i < n) {
    const double gi = (double)dinv[i] * s_[i];
    l = gi * s_[i] / S;
    g[i] = (float)gi;
  }
  l = lp_block_sum(l, sh);
  if (threadIdx.x == 0) atomicAdd(loss_acc, l);
}

// dy = dL/dy = -2 c (K g) / S
__global__ void k_lp_rl_dy(int n, const float* __restrict__ kg, const LpScalars* __restrict__ sc,
                           float* __restrict__ dy) {
  const int i = blockIdx.x * kLT + threadIdx.x;
  const double S = sc->dsum > 0 ? sc->dsum : 1.0;
  if (i < n) dy[i] = (float)(-2.0 * sc->c * (double)kg[i] / S);
}

// Random training errors e = xi / sqrt(d), xi ~ N(0, 1): white in the D-norm, so the
// error loss weighs every part of the spectrum of D^-1 K alike.  xi by the Box-Muller
// transform of two uniforms from the splitmix64 mix of (seed, pair, index).
__device__ inline uint64_t lp_mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void k_lp_random_error(int n, uint64_t seed, int pair, const float* __restrict__ dinv,
                                  float* __restrict__ e) {
  const int i = blockIdx.x * kLT + threadIdx.x;
  if (i >= n) return;
  const uint64_t h = lp_mix64(seed ^ lp_mix64(((uint64_t)pair << 32) | (uint32_t)i));
  const double u1 = ((h >> 11) + 1.0) * 0x1.0p-53;            // (0, 1]
  const double u2 = (lp_mix64(h) >> 11) * 0x1.0p-53;           // [0, 1)
  const double xi = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
  e[i] = (float)(xi * sqrt((double)dinv[i]));
}

__global__ void k_lp_adam(int64_t P, float* __restrict__ w, const float* __restrict__ g,
                          float* __restrict__ m, float* __restrict__ v,
                          __nv_bfloat16* __restrict__ wb, float lr, float b1, float b2,
                          float eps, float c1, float c2, float gscale) {
  const int64_t i = blockIdx.x * (int64_t)kLT + threadIdx.x;
  if (i >= P) return;
  const float gi = g[i] * gscale;
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  wb[i] = __float2bfloat16(wi);
}

__global__ void k_lp_to_bf16(int64_t P, const float* __restrict__ w,
                             __nv_bfloat16* __restrict__ wb) {
  const int64_t i = blockIdx.x * (int64_t)kLT + threadIdx.x;
  if (i < P) wb[i] = __float2bfloat16(w[i]);
}

__global__ void k_lp_degree(int N, const int32_t* __restrict__ adj_off, float* __restrict__ deg_inv) {
  const int a = blockIdx.x * kLT + threadIdx.x;
  if (a < N) deg_inv[a] = 1.f / (float)max(1, adj_off[a + 1] - adj_off[a]);
}

// diagonal of K: d, 1/d (FP32 and FP64) and log(d / mean d) (mean taken on the host)
template <typename TK>
__global__ void k_lp_diag(int n, const int32_t* __restrict__ rownnz, const int32_t* __restrict__ col,
                          const TK* __restrict__ val, float* __restrict__ d,
                          float* __restrict__ dinv, double* __restrict__ dinv64) {
  const int row = blockIdx.x * kLT + threadIdx.x;
  if (row >= n) return;
  double dv = 0.0;
  for (int s = 0; s < rownnz[row]; ++s) {
    const int64_t o = (int64_t)s * n + row;
    if (col[o] == row) { dv = (double)val[o]; break; }
  }
  if (!(dv > 0.0)) dv = 1.0;
  d[row] = (float)dv;
  dinv[row] = (float)(1.0 / dv);
  dinv64[row] = 1.0 / dv;
}

__global__ void k_lp_dlog(int n, const float* __restrict__ d, double logmean, float* __restrict__ dlog) {
  const int i = blockIdx.x * kLT + threadIdx.x;
  if (i < n) dlog[i] = (float)(log((double)d[i]) - logmean);
}

__global__ void k_lp_cast_f32(int n, const double* __restrict__ a, float* __restrict__ b) {
  const int i = blockIdx.x * kLT + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

inline int lp_grid(int64_t work) {
  int64_t b = (work + kLT - 1) / kLT;
  return (int)std::min<int64_t>(std::max<int64_t>(b, 1), 148 * 16);
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static void lp_free_buffers(LpState* s) {
  auto f = [](auto*& p) { if (p) { cudaFree(p); p = nullptr; } };
  f(s->deg_inv); f(s->dinv); f(s->dinv64); f(s->dlog); f(s->dvec); f(s->feat);
  f(s->v1); f(s->v2); f(s->lw); f(s->ls); f(s->lt);
  for (int l = 0; l <= kLayers; ++l) { f(s->pre[l]); f(s->h[l]); }
  for (int l = 0; l < kLayers; ++l) f(s->agg[l]);
  f(s->y); f(s->dy); f(s->rho); f(s->dh); f(s->dpre); f(s->tmp);
  f(s->pr); f(s->pe);
  s->npairs = 0;
  s->ready = false;
}

void gf_lp_free(gf_ctx* ctx) {
  LpState* s = ctx->lp;
  if (!s) return;
  lp_free_buffers(s);
  auto f = [](auto*& p) { if (p) { cudaFree(p); p = nullptr; } };
  f(s->w); f(s->wb); f(s->g); f(s->m); f(s->v); f(s->sc); f(s->err);
  delete s;
  ctx->lp = nullptr;
}

// Allocates the per-mesh buffers and the diagonal / graph data for the current matrix.
gf_status gf_lp_prepare(gf_ctx* ctx) {
  LpState* s = ctx->lp;
  if (!s) return gf_fail(ctx, GF_ERR_STATE, "learned preconditioner not initialised");
  if (!ctx->has_mesh || !ctx->d_adj_off || !(ctx->has64 || ctx->has32))
    return gf_fail(ctx, GF_ERR_STATE, "learned preconditioner needs an assembled mesh");
  if (s->dim != ctx->dim)
    return gf_fail(ctx, GF_ERR_STATE, "weights are for dim %d, mesh has dim %d", s->dim, ctx->dim);
  const int N = ctx->nnodes, n = ctx->n, dim = ctx->dim;
  if (s->ready && s->N == N && s->n == n) {
    // refresh the diagonal (the matrix may have changed)
  } else {
    lp_free_buffers(s);
    s->N = N;
    s->n = n;
    gf_status st;
#define LPA(p, cnt) if ((st = lp_alloc(ctx, &(p), (size_t)(cnt))) != GF_OK) return st
    LPA(s->deg_inv, N); LPA(s->dinv, n); LPA(s->dinv64, n); LPA(s->dlog, n); LPA(s->dvec, n);
    LPA(s->feat, (size_t)N * 4 * dim);
    LPA(s->v1, n); LPA(s->v2, n); LPA(s->lw, n); LPA(s->ls, n); LPA(s->lt, n);
    for (int l = 0; l <= kLayers; ++l) { LPA(s->pre[l], (size_t)N * H); LPA(s->h[l], (size_t)N * H); }
    for (int l = 0; l < kLayers; ++l) LPA(s->agg[l], (size_t)N * H);
    LPA(s->y, n); LPA(s->dy, n); LPA(s->rho, n); LPA(s->dh, (size_t)N * H); LPA(s->dpre, (size_t)N * H);
    LPA(s->tmp, (size_t)N * H);
#undef LPA
  }
  {
    gf_status st = gf_sell_prepare(ctx, ctx->has64 ? GF_F64 : GF_F32);  // feature products
    if (st != GF_OK) return st;
  }
  cudaStream_t st_ = ctx->stream;
  k_lp_degree<<<gf_blocks(N, kLT), kLT, 0, st_>>>(N, ctx->d_adj_off, s->deg_inv);
  ctx->launches++;
  if (ctx->has64)
    k_lp_diag<double><<<gf_blocks(n, kLT), kLT, 0, st_>>>(n, ctx->d_rownnz, ctx->d_colidx,
                                                          ctx->d_K64, s->dvec, s->dinv, s->dinv64);
  else
    k_lp_diag<float><<<gf_blocks(n, kLT), kLT, 0, st_>>>(n, ctx->d_rownnz, ctx->d_colidx,
                                                         ctx->d_K32, s->dvec, s->dinv, s->dinv64);
  ctx->launches++;
  std::vector<float> d(n);
  GF_CUDA(ctx, cudaMemcpyAsync(d.data(), s->dvec, sizeof(float) * n, cudaMemcpyDeviceToHost, st_));
  GF_CUDA(ctx, cudaStreamSynchronize(st_));
  double lm = 0.0;
  for (float x : d) lm += std::log((double)x);
  lm /= n;
  k_lp_dlog<<<gf_blocks(n, kLT), kLT, 0, st_>>>(n, s->dvec, lm, s->dlog);
  ctx->launches++;
  GF_CUDA(ctx, cudaGetLastError());
  s->ready = true;
  return GF_OK;
}

// y = scale .* (K x) for FP32 device vectors (FP64 matrix values when present), on the
// solver's node-block layout (prepared by gf_lp_prepare, so this only enqueues).
static void lp_matvec(gf_ctx* ctx, const float* x, const float* scale, float* y) {
  gf_matvec_f32(ctx, x, scale, y);
}

// Neighbour aggregation (see k_lp_aggregate) on the context stream.
static void lp_aggregate(gf_ctx* ctx, const float* h, float* out, int backward) {
  LpState* s = ctx->lp;
  const int N = s->N;
  const int grid = std::max(1, std::min((N + kAggNodes - 1) / kAggNodes, ctx->sm_count * 8));
  const int per_cta = (N + grid - 1) / grid;
  k_lp_aggregate<<<grid, kLT, 0, ctx->stream>>>(N, per_cta, ctx->d_adj_off, ctx->d_adj,
                                                s->deg_inv, h, out, backward);
  ctx->launches++;
}

// Resident CTAs per SM of one tensor-core layer kernel (set by lp_mm_attr).
template <int KD, int NO, bool TWO, bool WT>
static int& lp_mm_per_sm() {
  static int v = 1;
  return v;
}

// Tensor-core dense layer on the context stream (see k_lp_mm_tc): a persistent grid of
// the kernel's own resident CTAs per SM on every SM.
template <int KD, int NO, bool TWO, bool WT>
static void lp_mm(gf_ctx* ctx, const float* X1, const float* X2, const __nv_bfloat16* W1,
                  const __nv_bfloat16* W2, const __nv_bfloat16* bias, float* pre, float* out,
                  int relu, int accumulate) {
  LpState* s = ctx->lp;
  const int ntiles = (s->N + 127) / 128;
  const int grid =
      std::max(1, std::min(ntiles, ctx->sm_count * lp_mm_per_sm<KD, NO, TWO, WT>()));
  k_lp_mm_tc<KD, NO, TWO, WT><<<grid, kMmThreads, mm_smem_bytes<KD, NO, TWO>(), ctx->stream>>>(
      s->N, X1, X2, W1, W2, bias, pre, out, relu, accumulate, s->err);
  ctx->launches++;
}

template <int KD, int NO, bool TWO, bool WT>
static gf_status lp_mm_attr(gf_ctx* ctx) {
  auto k = k_lp_mm_tc<KD, NO, TWO, WT>;
  const int sm = (int)mm_smem_bytes<KD, NO, TWO>();
  GF_CUDA(ctx, gf_smem_attr(k, sm));
  GF_CUDA(ctx, gf_func_attr(reinterpret_cast<const void*>(k),
                            cudaFuncAttributePreferredSharedMemoryCarveout,
                            (int)cudaSharedmemCarveoutMaxShared));
  lp_mm_per_sm<KD, NO, TWO, WT>() =
      tc_ctas_per_sm(k, kMmThreads, (size_t)sm, (int)mm_tmem_cols(mm_pad16(NO)));
  return GF_OK;
}

// One-time set-up of the tensor-core layers of a dim-dimensional network.
static gf_status lp_mm_setup(gf_ctx* ctx, int dim) {
  gf_status st;
  if (dim == 2) {
    if ((st = lp_mm_attr<8, H, false, false>(ctx)) != GF_OK) return st;
    if ((st = lp_mm_attr<H, 2, false, false>(ctx)) != GF_OK) return st;
    if ((st = lp_mm_attr<2, H, false, true>(ctx)) != GF_OK) return st;
  } else {
    if ((st = lp_mm_attr<12, H, false, false>(ctx)) != GF_OK) return st;
    if ((st = lp_mm_attr<H, 3, false, false>(ctx)) != GF_OK) return st;
    if ((st = lp_mm_attr<3, H, false, true>(ctx)) != GF_OK) return st;
  }
  if ((st = lp_mm_attr<H, H, true, false>(ctx)) != GF_OK) return st;
  if ((st = lp_mm_attr<H, H, false, true>(ctx)) != GF_OK) return st;
  return GF_OK;
}

// Timeout flag of the tensor-core layers (read after a synchronisation).
static gf_status lp_check_err(gf_ctx* ctx) {
  int h = 0;
  GF_CUDA(ctx, cudaMemcpy(&h, ctx->lp->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) return gf_fail(ctx, GF_ERR_CUDA, "learned network: an MMA completion wait timed out");
  return GF_OK;
}

// Network forward on FP32 residual r (device, n); fills rho, y and the activations (the
// pre-activations too when `train`: the backward pass needs them).
static void lp_forward(gf_ctx* ctx, const float* r, bool train) {
  LpState* s = ctx->lp;
  cudaStream_t st = ctx->stream;
  const int N = s->N, n = s->n, dim = s->dim;
  const LpOffsets& o = s->off;
  cudaMemsetAsync(&s->sc->sumsq, 0, sizeof(double), st);
  k_lp_prep<<<gf_blocks(n, kLT), kLT, 0, st>>>(n, r, s->dinv, s->rho, s->sc);
  lp_matvec(ctx, s->rho, s->dinv, s->v1);
  lp_matvec(ctx, s->v1, s->dinv, s->v2);
  k_lp_features<<<gf_blocks(N, kLT), kLT, 0, st>>>(N, dim, s->rho, s->v1, s->v2, s->dlog,
                                                   s->feat, s->sc);
  if (dim == 2)
    lp_mm<8, H, false, false>(ctx, s->feat, nullptr, s->wb + o.W0, nullptr, s->wb + o.b0,
                              train ? s->pre[0] : nullptr, s->h[0], 1, 0);
  else
    lp_mm<12, H, false, false>(ctx, s->feat, nullptr, s->wb + o.W0, nullptr, s->wb + o.b0,
                               train ? s->pre[0] : nullptr, s->h[0], 1, 0);
  for (int l = 0; l < kLayers; ++l) {
    lp_aggregate(ctx, s->h[l], s->agg[l], 0);
    lp_mm<H, H, true, false>(ctx, s->h[l], s->agg[l], s->wb + o.Ws[l], s->wb + o.Wn[l],
                             s->wb + o.bl[l], train ? s->pre[l + 1] : nullptr, s->h[l + 1], 1, 0);
  }
  if (dim == 2)
    lp_mm<H, 2, false, false>(ctx, s->h[kLayers], nullptr, s->wb + o.Wout, nullptr,
                              s->wb + o.bout, nullptr, s->y, 0, 0);
  else
    lp_mm<H, 3, false, false>(ctx, s->h[kLayers], nullptr, s->wb + o.Wout, nullptr,
                              s->wb + o.bout, nullptr, s->y, 0, 0);
  ctx->launches += 3;
}

// Backward from dy ([N][dim] == n floats) into s->g (accumulated).
static void lp_backward(gf_ctx* ctx, const float* dy) {
  LpState* s = ctx->lp;
  cudaStream_t st = ctx->stream;
  const int N = s->N, dim = s->dim;
  const LpOffsets& o = s->off;
  const int gH = lp_grid((int64_t)N * H);
  const int gw = std::min(148 * 4, (N + 31) / 32);
  // output layer
  if (dim == 2) {
    k_lp_wgrad<H, 2><<<gw, kLT, 0, st>>>(N, dy, s->h[kLayers], s->g + o.Wout, s->g + o.bout);
    lp_mm<2, H, false, true>(ctx, dy, nullptr, s->wb + o.Wout, nullptr, nullptr, nullptr,
                             s->dh, 0, 0);
  } else {
    k_lp_wgrad<H, 3><<<gw, kLT, 0, st>>>(N, dy, s->h[kLayers], s->g + o.Wout, s->g + o.bout);
    lp_mm<3, H, false, true>(ctx, dy, nullptr, s->wb + o.Wout, nullptr, nullptr, nullptr,
                             s->dh, 0, 0);
  }
  for (int l = kLayers - 1; l >= 0; --l) {
    k_lp_relu_grad<<<gH, kLT, 0, st>>>((int64_t)N * H, s->dh, s->pre[l + 1], s->dpre);
    k_lp_wgrad<H, H><<<gw, kLT, 0, st>>>(N, s->dpre, s->h[l], s->g + o.Ws[l], s->g + o.bl[l]);
    // the bias gradient was added by the call above; the Wn call adds into a scratch bias
    k_lp_wgrad<H, H><<<gw, kLT, 0, st>>>(N, s->dpre, s->agg[l], s->g + o.Wn[l],
                                         s->g + o.total);  // scratch slot past the params
    // dh_l = Ws^T dpre + aggregate^T(Wn^T dpre)
    lp_mm<H, H, false, true>(ctx, s->dpre, nullptr, s->wb + o.Wn[l], nullptr, nullptr, nullptr,
                             s->tmp, 0, 0);
    lp_aggregate(ctx, s->tmp, s->dh, 1);
    lp_mm<H, H, false, true>(ctx, s->dpre, nullptr, s->wb + o.Ws[l], nullptr, nullptr, nullptr,
                             s->dh, 0, 1);
  }
  k_lp_relu_grad<<<gH, kLT, 0, st>>>((int64_t)N * H, s->dh, s->pre[0], s->dpre);
  if (dim == 2)
    k_lp_wgrad<8, H><<<gw, kLT, 0, st>>>(N, s->dpre, s->feat, s->g + o.W0, s->g + o.b0);
  else
    k_lp_wgrad<12, H><<<gw, kLT, 0, st>>>(N, s->dpre, s->feat, s->g + o.W0, s->g + o.b0);
  ctx->launches += 3 + 5 * kLayers + 2;
}

// Forward, loss and backward of one training pair (r, e): adds the pair's loss to
// sc->loss and its parameter gradient to s->g.
static void lp_pair(gf_ctx* ctx, const float* r, const float* e) {
  LpState* s = ctx->lp;
  cudaStream_t cs = ctx->stream;
  const int n = s->n, nb = gf_blocks(n, kLT);
  cudaMemsetAsync(&s->sc->dsum, 0, sizeof(double), cs);
  lp_forward(ctx, r, true);
  if (s->loss == GF_LP_LOSS_RESIDUAL) {
    k_lp_rl_diff<<<nb, kLT, 0, cs>>>(n, e, s->rho, s->y, s->sc, s->lw);
    lp_matvec(ctx, s->lw, nullptr, s->ls);   // s = K (e - z)
    lp_matvec(ctx, e, nullptr, s->lt);       // t = K e
    k_lp_rl_sums<<<nb, kLT, 0, cs>>>(n, s->lt, s->dinv, s->sc);
    k_lp_rl_loss<<<nb, kLT, 0, cs>>>(n, s->ls, s->dinv, s->sc, s->lw, &s->sc->loss);
    lp_matvec(ctx, s->lw, nullptr, s->lt);   // K D^-1 s
    k_lp_rl_dy<<<nb, kLT, 0, cs>>>(n, s->lt, s->sc, s->dy);
    ctx->launches += 4;
  } else {
    k_lp_loss_sums<<<nb, kLT, 0, cs>>>(n, e, s->dvec, s->sc);
    k_lp_loss_grad<<<nb, kLT, 0, cs>>>(n, e, s->rho, s->y, s->dvec, s->dy, s->sc, &s->sc->loss);
    ctx->launches += 2;
  }
  lp_backward(ctx, s->dy);
}

// Preconditioner application for the solver: z = M(r) in FP64 from an FP64 residual.
gf_status gf_lp_apply64(gf_ctx* ctx, const double* r64, float* r32_scratch, double* z) {
  LpState* s = ctx->lp;
  const int n = s->n;
  k_lp_cast_f32<<<gf_blocks(n, kLT), kLT, 0, ctx->stream>>>(n, r64, r32_scratch);
  lp_forward(ctx, r32_scratch, false);
  k_lp_output<double><<<gf_blocks(n, kLT), kLT, 0, ctx->stream>>>(n, s->rho, s->y, s->sc, z);
  ctx->launches += 2;
  return GF_OK;
}

bool gf_lp_ready(const gf_ctx* ctx) { return ctx->lp && ctx->lp->ready; }
bool gf_lp_coarse(const gf_ctx* ctx) { return ctx->lp && ctx->lp->coarse; }

// A new mesh or matrix invalidates the collected pairs and the diagonal; the
// weights stay (they are mesh-independent).
void gf_lp_mesh_changed(gf_ctx* ctx) {
  if (!ctx->lp) return;
  ctx->lp->ready = false;
  if (ctx->lp->pr) { cudaFree(ctx->lp->pr); ctx->lp->pr = nullptr; }
  if (ctx->lp->pe) { cudaFree(ctx->lp->pe); ctx->lp->pe = nullptr; }
  ctx->lp->npairs = 0;
}

gf_status gf_solve_run(gf_ctx* ctx, const gf_solve_opts* o, gf_solve_info* info);

gf_status gf_lp_collect_impl(gf_ctx* ctx, int npairs, int every, double tol, int maxit) {
  LpState* s = ctx->lp;
  if (!ctx->has64) return gf_fail(ctx, GF_ERR_STATE, "pair collection needs the FP64 matrix");
  const int n = s->n;
  // reference solution u* (tighter than the recorded run)
  gf_solve_opts o{};
  o.solver = s->coarse ? GF_SOLVER_TWOLEVEL_PCG : GF_SOLVER_PCG;
  o.matrix = GF_F64;
  o.tol = tol * 1e-3;
  o.max_iter = maxit * 4;
  gf_solve_info info{};
  gf_status st = gf_solve_run(ctx, &o, &info);
  if (st != GF_OK && st != GF_ERR_NOT_CONVERGED) return st;
  double* ustar = nullptr;
  if ((st = gf_alloc(ctx, &ustar, (size_t)n)) != GF_OK) return st;
  cudaMemcpyAsync(ustar, ctx->d_u, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream);
  if (s->pr) cudaFree(s->pr);
  if (s->pe) cudaFree(s->pe);
  s->pr = s->pe = nullptr;
  s->npairs = 0;
  if ((st = gf_alloc(ctx, &s->pr, (size_t)npairs * n)) != GF_OK) { cudaFree(ustar); return st; }
  if ((st = gf_alloc(ctx, &s->pe, (size_t)npairs * n)) != GF_OK) { cudaFree(ustar); return st; }
  int got = 0;
  st = gf_pcg_record(ctx, ustar, npairs, every, tol, maxit, s->pr, s->pe, &got, s->coarse);
  cudaFree(ustar);
  if (st != GF_OK && st != GF_ERR_NOT_CONVERGED) return st;
  s->npairs = got;
  if (got == 0) return gf_fail(ctx, GF_ERR_STATE, "no pairs recorded");
  return GF_OK;
}

// Pairs collection: Jacobi-PCG on the FP64 matrix and force, recording (r, x) at
// chunk boundaries; e = u* - x with u* from a tighter solve.
gf_status gf_lp_collect_impl(gf_ctx* ctx, int npairs, int every, double tol, int maxit);

// Random pairs: e_k white in the D-norm, r_k = K e_k.
static gf_status lp_collect_random(gf_ctx* ctx, int npairs, uint64_t seed) {
  LpState* s = ctx->lp;
  const int n = s->n;
  if (s->pr) cudaFree(s->pr);
  if (s->pe) cudaFree(s->pe);
  s->pr = s->pe = nullptr;
  s->npairs = 0;
  gf_status st;
  if ((st = gf_alloc(ctx, &s->pr, (size_t)npairs * n)) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &s->pe, (size_t)npairs * n)) != GF_OK) return st;
  for (int k = 0; k < npairs; ++k) {
    float* e = s->pe + (int64_t)k * n;
    k_lp_random_error<<<gf_blocks(n, kLT), kLT, 0, ctx->stream>>>(n, seed, k, s->dinv, e);
    ctx->launches++;
    lp_matvec(ctx, e, nullptr, s->pr + (int64_t)k * n);
  }
  GF_CUDA(ctx, cudaGetLastError());
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  s->npairs = npairs;
  return GF_OK;
}

extern "C" {

GF_API int64_t gf_lp_num_params(int32_t dim) {
  if (dim != 2 && dim != 3) return 0;
  return lp_offsets(dim).total;
}

GF_API gf_status gf_lp_init(gf_ctx* ctx, int32_t dim, uint64_t seed) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (dim != 2 && dim != 3) return gf_fail(ctx, GF_ERR_INVALID_ARG, "dim must be 2 or 3");
  cudaSetDevice(ctx->device);
  gf_lp_free(ctx);
  LpState* s = new LpState();
  ctx->lp = s;
  s->dim = dim;
  s->off = lp_offsets(dim);
  const int64_t P = s->off.total;
  gf_status st;
  if ((st = lp_alloc(ctx, &s->w, (size_t)P)) != GF_OK) return st;
  if ((st = lp_alloc(ctx, &s->wb, (size_t)P)) != GF_OK) return st;
  if ((st = lp_alloc(ctx, &s->g, (size_t)P + H)) != GF_OK) return st;
  if ((st = lp_alloc(ctx, &s->m, (size_t)P)) != GF_OK) return st;
  if ((st = lp_alloc(ctx, &s->v, (size_t)P)) != GF_OK) return st;
  if ((st = lp_alloc(ctx, &s->sc, 1)) != GF_OK) return st;
  if ((st = lp_alloc(ctx, &s->err, 1)) != GF_OK) return st;
  GF_CUDA(ctx, cudaMemset(s->err, 0, sizeof(int)));
  if ((st = lp_mm_setup(ctx, dim)) != GF_OK) return st;
  // He-style init for hidden layers; output layer zero (untrained = Jacobi)
  std::vector<float> w(P, 0.f);
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  const LpOffsets& o = s->off;
  const int F = 4 * dim;
  for (int64_t k = 0; k < (int64_t)H * F; ++k) w[o.W0 + k] = nd(rng) * std::sqrt(2.f / F);
  for (int l = 0; l < kLayers; ++l)
    for (int64_t k = 0; k < (int64_t)H * H; ++k) {
      w[o.Ws[l] + k] = nd(rng) * std::sqrt(1.f / H);
      w[o.Wn[l] + k] = nd(rng) * std::sqrt(1.f / H);
    }
  GF_CUDA(ctx, cudaMemcpy(s->w, w.data(), sizeof(float) * P, cudaMemcpyHostToDevice));
  GF_CUDA(ctx, cudaMemset(s->m, 0, sizeof(float) * P));
  GF_CUDA(ctx, cudaMemset(s->v, 0, sizeof(float) * P));
  k_lp_to_bf16<<<gf_blocks(P, kLT), kLT, 0, ctx->stream>>>(P, s->w, s->wb);
  GF_LAUNCH_CHECK(ctx, "k_lp_to_bf16");
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  s->adam_t = 0;
  return GF_OK;
}

GF_API gf_status gf_lp_get_weights(gf_ctx* ctx, float* w) {
  if (!ctx || !w) return GF_ERR_INVALID_ARG;
  if (!ctx->lp) return gf_fail(ctx, GF_ERR_STATE, "learned preconditioner not initialised");
  cudaSetDevice(ctx->device);
  GF_CUDA(ctx, cudaMemcpy(w, ctx->lp->w, sizeof(float) * ctx->lp->off.total, cudaMemcpyDeviceToHost));
  return GF_OK;
}

GF_API gf_status gf_lp_set_weights(gf_ctx* ctx, const float* w) {
  if (!ctx || !w) return GF_ERR_INVALID_ARG;
  if (!ctx->lp) return gf_fail(ctx, GF_ERR_STATE, "learned preconditioner not initialised");
  cudaSetDevice(ctx->device);
  LpState* s = ctx->lp;
  const int64_t P = s->off.total;
  for (int64_t k = 0; k < P; ++k)
    if (!std::isfinite(w[k])) return gf_fail(ctx, GF_ERR_INVALID_ARG, "non-finite weight %lld", (long long)k);
  GF_CUDA(ctx, cudaMemcpy(s->w, w, sizeof(float) * P, cudaMemcpyHostToDevice));
  k_lp_to_bf16<<<gf_blocks(P, kLT), kLT, 0, ctx->stream>>>(P, s->w, s->wb);
  GF_LAUNCH_CHECK(ctx, "k_lp_to_bf16");
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GF_OK;
}

// z = M(r) for FP32 device vectors of length n (the context's dof count).
GF_API gf_status gf_lp_apply(gf_ctx* ctx, const float* r, float* z) {
  if (!ctx || !r || !z) return GF_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  gf_status st = gf_lp_prepare(ctx);
  if (st != GF_OK) return st;
  LpState* s = ctx->lp;
  cudaEventRecord(ctx->ev0, ctx->stream);
  lp_forward(ctx, r, false);
  k_lp_output<float><<<gf_blocks(s->n, kLT), kLT, 0, ctx->stream>>>(s->n, s->rho, s->y, s->sc, z);
  GF_LAUNCH_CHECK(ctx, "k_lp_output");
  cudaEventRecord(ctx->ev1, ctx->stream);
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  ctx->last_seconds = ms * 1e-3;   // device time of one application (gf_last_device_seconds)
  return lp_check_err(ctx);
}

// Loss and gradient for one (r, e) pair of FP32 device vectors; the gradient of
// the parameters (same layout as the weights) is copied to `grad` (host, may be
// NULL) and the loss returned in *loss.  Does not update the weights.
GF_API gf_status gf_lp_loss_grad(gf_ctx* ctx, const float* r, const float* e, float* loss,
                                 float* grad) {
  if (!ctx || !r || !e) return GF_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  gf_status st = gf_lp_prepare(ctx);
  if (st != GF_OK) return st;
  LpState* s = ctx->lp;
  const int64_t P = s->off.total;
  cudaStream_t cs = ctx->stream;
  GF_CUDA(ctx, cudaMemsetAsync(s->g, 0, sizeof(float) * (P + H), cs));
  GF_CUDA(ctx, cudaMemsetAsync(&s->sc->loss, 0, sizeof(double), cs));
  lp_pair(ctx, r, e);
  GF_CUDA(ctx, cudaGetLastError());
  double l = 0.0;
  GF_CUDA(ctx, cudaMemcpyAsync(&l, &s->sc->loss, sizeof(double), cudaMemcpyDeviceToHost, cs));
  GF_CUDA(ctx, cudaStreamSynchronize(cs));
  if ((st = lp_check_err(ctx)) != GF_OK) return st;
  if (loss) *loss = (float)l;
  if (grad) GF_CUDA(ctx, cudaMemcpy(grad, s->g, sizeof(float) * P, cudaMemcpyDeviceToHost));
  return GF_OK;
}

GF_API gf_status gf_lp_set_coarse(gf_ctx* ctx, int32_t on) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (!ctx->lp) return gf_fail(ctx, GF_ERR_STATE, "learned preconditioner not initialised (gf_lp_init)");
  ctx->lp->coarse = on != 0;
  return GF_OK;
}

GF_API gf_status gf_lp_set_loss(gf_ctx* ctx, int32_t loss) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (loss != GF_LP_LOSS_ERROR && loss != GF_LP_LOSS_RESIDUAL)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "unknown loss %d", (int)loss);
  if (!ctx->lp) return gf_fail(ctx, GF_ERR_STATE, "learned preconditioner not initialised (gf_lp_init)");
  ctx->lp->loss = loss;
  return GF_OK;
}

GF_API gf_status gf_lp_collect(gf_ctx* ctx, int32_t npairs, int32_t every, double tol,
                               int32_t max_iter) {
  if (!ctx || npairs <= 0 || every <= 0) return GF_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  gf_status st = gf_lp_prepare(ctx);
  if (st != GF_OK) return st;
  return gf_lp_collect_impl(ctx, npairs, every, tol, max_iter > 0 ? max_iter : 100000);
}

GF_API gf_status gf_lp_collect_random(gf_ctx* ctx, int32_t npairs, uint64_t seed) {
  if (!ctx || npairs <= 0) return GF_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  gf_status st = gf_lp_prepare(ctx);
  if (st != GF_OK) return st;
  if (ctx->lp->coarse)
    return gf_fail(ctx, GF_ERR_UNSUPPORTED, "random pairs have no coarse-corrected target");
  return lp_collect_random(ctx, npairs, seed);
}

GF_API gf_status gf_lp_train(gf_ctx* ctx, int32_t steps, int32_t batch, float lr, uint64_t seed,
                             float* final_loss) {
  if (!ctx || steps < 0 || batch <= 0 || !(lr > 0.f)) return GF_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  gf_status st = gf_lp_prepare(ctx);
  if (st != GF_OK) return st;
  LpState* s = ctx->lp;
  if (s->npairs == 0) return gf_fail(ctx, GF_ERR_STATE, "no training pairs (gf_lp_collect)");
  const int64_t P = s->off.total;
  cudaStream_t cs = ctx->stream;
  std::mt19937_64 rng(seed);
  std::uniform_int_distribution<int> pick(0, s->npairs - 1);
  double last = 0.0;
  for (int it = 0; it < steps; ++it) {
    GF_CUDA(ctx, cudaMemsetAsync(s->g, 0, sizeof(float) * (P + H), cs));
    GF_CUDA(ctx, cudaMemsetAsync(&s->sc->loss, 0, sizeof(double), cs));
    for (int b = 0; b < batch; ++b) {
      const int k = pick(rng);
      const float* r = s->pr + (int64_t)k * s->n;
      const float* e = s->pe + (int64_t)k * s->n;
      lp_pair(ctx, r, e);
    }
    ++s->adam_t;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)s->adam_t), c2 = 1.f - std::pow(b2, (float)s->adam_t);
    k_lp_adam<<<gf_blocks(P, kLT), kLT, 0, cs>>>(P, s->w, s->g, s->m, s->v, s->wb, lr, b1, b2,
                                                 1e-8f, c1, c2, 1.f / batch);
    GF_LAUNCH_CHECK(ctx, "k_lp_adam");
    double l = 0.0;
    GF_CUDA(ctx, cudaMemcpyAsync(&l, &s->sc->loss, sizeof(double), cudaMemcpyDeviceToHost, cs));
    GF_CUDA(ctx, cudaStreamSynchronize(cs));
    last = l / batch;
    if (!std::isfinite(last)) return gf_fail(ctx, GF_ERR_STALLED, "training diverged at step %d", it);
  }
  if ((st = lp_check_err(ctx)) != GF_OK) return st;
  if (final_loss) *final_loss = (float)last;
  return GF_OK;
}

}  // extern "C"
