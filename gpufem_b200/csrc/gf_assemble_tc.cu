// Stiffness assembly on the 5th-generation tensor cores (tcgen05, sm_100a): the FP32
// engine GF_ENGINE_TF32_MMA.
//
// Reference math: StiffAlgoCPU::CalcGlobalStiffnessNaive, Gauss-point loop
// (src/FEM/StiffAlgoCPU.cc:110-133: Ke += B^T (D B) detJ w), with the node order and
// Gauss rules of StiffAlgo.cc:47-278 / FemData.cc:226-316; the OpenCL kernels it replaces
// are src/OpenCL/clKernels/gpuFEM_{Q4,Q8,UR8,UR20}.cl.
//
// Formulation.  For isotropic D the node-pair block of B^T D B is
//   Ke[i,a ; j,b] = lam1 M[(i,a),(j,b)] + mu1 M[(i,b),(j,a)] + mu1 delta_ab sum_c M[(i,c),(j,c)]
// where M = G W G^T is the Gram matrix of the element's gradient matrix G (rows: node i,
// component a; columns: Gauss points k, G[(i,a)][k] = dN_i/dx_a at point k) under the
// weights W = diag(w_k detJ_k E).  M is what the tensor cores compute: with
// A[(i,a)][k] = G[(i,a)][k] sqrt|W_k| and B = A with the columns of negative W_k negated,
// M = A B^T, a K-major TF32 product whose K is the Gauss-point count (padded to 8s).
// Three TF32 products of split operands (x = hi + lo, both TF32; hi hi^T + hi lo^T + lo hi^T)
// keep M at FP32 accuracy.
//
// Layout.  A CTA of 128 threads (4 warps) takes groups of elements whose rows fill the
// 128 TMEM lanes: rows (element e, node i, component a) are placed so that the DIM rows of a
// node sit in consecutive lanes of one warp (3-D: 10 nodes per warp, 2 pad lanes; Brick20
// spans two warps).  Per group:
//   1. a thread per (element, Gauss point) forms J, detJ (FP64 J^-1 and gradients for an
//      element whose max/min |detJ| > 10), the gradients, and writes A (and B when some
//      weight is negative) as hi/lo TF32 tiles in the canonical K-major no-swizzle layout
//      (8-row x 16-byte core matrices: element (r, k) at (k/4) * 128 * 16 + r * 16 + (k%4) * 4
//      bytes);
//   2. one thread issues tcgen05.mma (M = N = 128, kind::tf32, FP32 accumulator in TMEM)
//      and tcgen05.commit to an mbarrier;
//   3. every thread reads its row of M (its element's columns) with tcgen05.ld, forms the
//      node-pair blocks with in-warp shuffles between the DIM lanes of a node (transpose and
//      trace), and scatters its column of each block into the ELL matrix: red.global.add
//      (atomic schedule) or plain read-modify-write (colour schedule, elements of one colour
//      share no node).  Ke never touches HBM.
// Off-diagonal element blocks of the 128 x 128 product are computed and discarded: the
// tensor cores have the throughput to spare, and the scatter bounds these kernels.
#include <cmath>
#include <algorithm>

#include "gf_elem.cuh"
#include "gf_tc.cuh"

namespace {

constexpr int kTcThreads = 128;
constexpr int kTcCols = 128;          // TMEM columns per CTA (N = 128 FP32 accumulators)
constexpr int kTcMaxWaitIters = 1 << 20;

template <int ET>
struct TcShape {
  static constexpr ElemInfo info = gf_elem_info(ET);
  static constexpr int DIM = info.dim, NEN = info.nen;
  static constexpr int NPW = 32 / DIM;                       // nodes per warp
  static constexpr int WPE = (NEN + NPW - 1) / NPW;          // warps per element
  static constexpr int RAW = NEN * DIM;                      // rows of one element
  // lanes of one element within its warp: a power of two (2-D, Brick8) or the whole warp
  static constexpr int RPE = WPE > 1 ? 32 : (RAW <= 8 ? 8 : RAW <= 16 ? 16 : 32);
  static constexpr int EPW = WPE > 1 ? 1 : 32 / RPE;         // elements per warp
  static constexpr int EPG = WPE > 1 ? 4 / WPE : 4 * EPW;    // elements per 128-row group
  static constexpr int LW = RPE * WPE;                       // columns of one element
};

// Row (TMEM lane) of component a of node i of element slot e within a group.
template <int ET>
__host__ __device__ constexpr int tc_row(int e, int i, int a) {
  using S = TcShape<ET>;
  return S::WPE > 1 ? e * 32 * S::WPE + (i / S::NPW) * 32 + (i % S::NPW) * S::DIM + a
                    : (e / S::EPW) * 32 + (e % S::EPW) * S::RPE + i * S::DIM + a;
}

// Column of (node j, component b) within the LW columns of one element.
template <int ET>
__host__ __device__ constexpr int tc_col(int j, int b) {
  using S = TcShape<ET>;
  return S::WPE > 1 ? (j / S::NPW) * 32 + (j % S::NPW) * S::DIM + b : j * S::DIM + b;
}

template <int ET>
struct TcSmem {
  // byte offsets within the dynamic shared memory of one CTA
  size_t tile, a_hi, a_lo, dN, w, X, wd, wt, ji, slot, conn, sel, flag, neg, mbar,
      tslot, total;
};

template <int ET>
__host__ __device__ TcSmem<ET> tc_smem(int ngp) {
  using S = TcShape<ET>;
  TcSmem<ET> L{};
  const int KP = (ngp + 7) / 8 * 8;
  L.tile = (size_t)128 * KP * 4;
  size_t o = 0;
  L.a_hi = o; o += L.tile;
  L.a_lo = o; o += L.tile;
  L.dN = o; o += (size_t)ngp * S::DIM * S::NEN * 4;
  L.w = o; o += (size_t)ngp * 4;
  L.X = o; o += (size_t)S::EPG * S::NEN * S::DIM * 4;
  L.wd = o; o += (size_t)S::EPG * ngp * 4;
  L.wt = o; o += (size_t)S::EPG * ngp * 4;
  L.ji = o; o += (size_t)S::EPG * ngp * S::DIM * S::DIM * 4;
  L.slot = o; o += ((size_t)S::EPG * S::NEN * S::NEN * 2 + 15) / 16 * 16;
  L.conn = o; o += (size_t)S::EPG * S::NEN * 4;
  L.sel = o; o += (size_t)S::EPG * 4;
  L.flag = o; o += (size_t)S::EPG * 4;
  L.neg = o; o += 16;
  o = (o + 7) / 8 * 8;
  L.mbar = o; o += 8;
  L.tslot = o; o += 8;
  L.total = o;
  return L;
}

// MODE 0: colour schedule (plain read-modify-write of K), 1: atomic schedule
// (red.global.add into K), 2: store each element's Gram matrix M (RAW x RAW, row-major,
// rows and columns (node, component)) to `out` for the owner gather (gf_assemble_owner.cu).
template <int ET, int MODE>
__global__ void __launch_bounds__(kTcThreads)
k_assemble_tc(const int32_t* __restrict__ elems, int count, int ngp,
              const int32_t* __restrict__ conn, const double* __restrict__ coords,
              const float* __restrict__ Eel, const uint16_t* __restrict__ slotmap, int nelem,
              int n, const AsmTables* __restrict__ tab, float lam1, float mu1,
              float* __restrict__ K, int* __restrict__ err) {
  using S = TcShape<ET>;
  constexpr int NEN = S::NEN, DIM = S::DIM, EPG = S::EPG;
  constexpr bool ATOMIC = MODE == 1, GRAM = MODE == 2;
  extern __shared__ __align__(1024) unsigned char smem[];
  const TcSmem<ET> L = tc_smem<ET>(ngp);
  float* aH = reinterpret_cast<float*>(smem + L.a_hi);
  float* aL = reinterpret_cast<float*>(smem + L.a_lo);
  float* sdN = reinterpret_cast<float*>(smem + L.dN);
  float* sw = reinterpret_cast<float*>(smem + L.w);
  float* sX = reinterpret_cast<float*>(smem + L.X);
  float* swd = reinterpret_cast<float*>(smem + L.wd);
  float* swt = reinterpret_cast<float*>(smem + L.wt);       // [e][g] signed weight w detJ E
  float* sji = reinterpret_cast<float*>(smem + L.ji);       // [e][g][DIM*DIM] FP32 J^-1
  uint16_t* sslot = reinterpret_cast<uint16_t*>(smem + L.slot);  // [e][pair]
  int* sconn = reinterpret_cast<int*>(smem + L.conn);
  int* sel = reinterpret_cast<int*>(smem + L.sel);
  int* sflag = reinterpret_cast<int*>(smem + L.flag);
  int* sneg = reinterpret_cast<int*>(smem + L.neg);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + L.mbar);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + L.tslot);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int KP = (ngp + 7) / 8 * 8;
  const int ngroups = (count + EPG - 1) / EPG;

  // one-time set-up: tables, zeroed tiles (padding rows and Gauss points stay zero),
  // TMEM columns, the MMA-completion barrier
  for (int k = tid; k < ngp * DIM * NEN; k += kTcThreads) sdN[k] = tab->dN32[k];
  for (int k = tid; k < ngp; k += kTcThreads) sw[k] = tab->w32[k];
  for (size_t k = tid; k < 2 * L.tile / 4; k += kTcThreads) aH[k] = 0.f;  // a_hi, a_lo
  if (warp == 0) tc_alloc(tslot, kTcCols);
  if (tid == 0) tc_mbar_init(mbar);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  constexpr uint32_t idesc = tc_idesc_tf32(128, 128);
  bool ok = true;
  uint32_t phase = 0;

  for (int grp = blockIdx.x; grp < ngroups && ok; grp += gridDim.x) {
    const int e0 = grp * EPG;
    const int ne = min(EPG, count - e0);
    // ---- 1. element data, distortion test, gradients into the operand tiles ----------
    for (int e = tid; e < EPG; e += kTcThreads) {
      sel[e] = e < ne ? elems[e0 + e] : -1;
      sflag[e] = 0;
    }
    if (tid == 0) *sneg = 0;
    __syncthreads();
    for (int k = tid; k < ne * NEN; k += kTcThreads) {
      const int e = k / NEN, i = k % NEN;
      const int el = sel[e];
      const int node = conn[(int64_t)el * NEN + i];
      const int node0 = conn[(int64_t)el * NEN];
      sconn[k] = node;
#pragma unroll
      for (int c = 0; c < DIM; ++c)
        sX[k * DIM + c] =
            float(coords[(int64_t)node * DIM + c] - coords[(int64_t)node0 * DIM + c]);
    }
    __syncthreads();
    // slot indices of the group's node pairs, [e][pair] (for the atomic schedule the group's
    // elements are consecutive, so a pair's EPG entries are contiguous in the [pair][element] map)
    if constexpr (!GRAM)
      for (int t = tid; t < ne * NEN * NEN; t += kTcThreads) {
        const int pr = t / ne, e = t % ne;
        sslot[e * NEN * NEN + pr] = slotmap[(int64_t)pr * nelem + sel[e]];
      }
    for (int t = tid; t < ne * ngp; t += kTcThreads) {
      const int e = t / ngp, g = t % ngp;
      float J[3][3], Ji[3][3];
      gf_jacobian<NEN, DIM, float, float>(sdN + g * DIM * NEN, sX + e * NEN * DIM, J);
      const float d = gf_det_inv<DIM, float>(J, Ji);
      swd[e * ngp + g] = d;
      float* o = sji + (e * ngp + g) * DIM * DIM;
#pragma unroll
      for (int q = 0; q < DIM * DIM; ++q) o[q] = Ji[q / DIM][q % DIM];
    }
    __syncthreads();
    for (int e = tid; e < ne; e += kTcThreads) {
      float dmin = 3.4e38f, dmax = 0.f;
      for (int g = 0; g < ngp; ++g) {
        dmin = fminf(dmin, fabsf(swd[e * ngp + g]));
        dmax = fmaxf(dmax, fabsf(swd[e * ngp + g]));
      }
      sflag[e] = dmax > 10.f * dmin ? 1 : 0;
    }
    __syncthreads();
    // per (element, Gauss point): the weight W = w detJ E and J^-1 scaled by sqrt|W| (FP64
    // J and J^-1 for a distorted element), so that a row of A is sqrt|W| J^-1 dN
    for (int t = tid; t < ne * ngp; t += kTcThreads) {
      const int e = t / ngp, g = t % ngp;
      float* ji = sji + t * DIM * DIM;
      float detJ = swd[t];
      if (sflag[e]) {
        double J[3][3], Ji[3][3];
        gf_jacobian<NEN, DIM, double, float>(sdN + g * DIM * NEN, sX + e * NEN * DIM, J);
        detJ = (float)gf_det_inv<DIM, double>(J, Ji);
#pragma unroll
        for (int q = 0; q < DIM * DIM; ++q) ji[q] = (float)Ji[q / DIM][q % DIM];
      }
      const float w = sw[g] * detJ * Eel[sel[e]];
      const float sq = sqrtf(fabsf(w));
      if (w < 0.f) atomicOr(sneg, 1);
#pragma unroll
      for (int q = 0; q < DIM * DIM; ++q) ji[q] *= sq;
      swt[t] = w;
    }
    __syncthreads();
    // operand tiles: a thread per (element, row (i, c), 4 Gauss points) forms
    // A[(i,c)][k] = sum_b (sqrt|W| J^-1)[c][b] dN_i/dxi_b at k, splits it into TF32 hi + lo
    // and stores each as one 16-byte chunk (consecutive threads: consecutive rows, so the
    // stores are conflict-free); Gauss points past ngp give zeros
    {
      const int KC = (ngp + 7) / 8 * 2;           // 4-point chunks of the padded K
      const int nrow = ne * S::RAW;
      for (int t = tid; t < nrow * KC; t += kTcThreads) {
        const int kc = t / nrow, rem = t - kc * nrow;
        const int e = rem / S::RAW, r = rem - e * S::RAW;
        const int i = r / DIM, c = r - i * DIM;
        float hv[4], lv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int g = 4 * kc + u;
          float v = 0.f;
          if (g < ngp) {
            const float* ji = sji + (e * ngp + g) * DIM * DIM + c * DIM;
            const float* dN = sdN + g * DIM * NEN + i;
#pragma unroll
            for (int b = 0; b < DIM; ++b) v += ji[b] * dN[b * NEN];
          }
          const uint32_t hb = tc_tf32_round(v);
          hv[u] = __uint_as_float(hb);
          lv[u] = __uint_as_float(tc_tf32_round(v - hv[u]));
        }
        const int o = kc * 512 + tc_row<ET>(e, i, c) * 4;
        *reinterpret_cast<float4*>(aH + o) = make_float4(hv[0], hv[1], hv[2], hv[3]);
        *reinterpret_cast<float4*>(aL + o) = make_float4(lv[0], lv[1], lv[2], lv[3]);
      }
    }
    // make the generic-proxy tile writes visible to the tensor cores
    tc_fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    // ---- 2. M = A A^T on the tensor cores ---------------------------------------------
    // (a group with a negative weight, i.e. an inverted element, forms M on the CUDA cores
    // in step 3 instead: M = A S A^T with S the signs of the weights)
    const bool neg = *sneg != 0;
    if (tid == 0 && !neg) {
      const uint32_t ah = tc_smem_u32(aH), al = tc_smem_u32(aL);
      const uint32_t bh = ah, bl = al;
      const uint32_t lbo = 128 * 16, sbo = 128;   // next K chunk of 4; next 8-row group
      for (int ks = 0; ks < KP / 8; ++ks) {
        const uint32_t off = (uint32_t)ks * 2 * lbo;
        tc_mma_tf32(tmem, tc_desc(al + off, lbo, sbo), tc_desc(bh + off, lbo, sbo), idesc,
                    ks > 0 ? 1u : 0u);
        tc_mma_tf32(tmem, tc_desc(ah + off, lbo, sbo), tc_desc(bl + off, lbo, sbo), idesc, 1u);
        tc_mma_tf32(tmem, tc_desc(ah + off, lbo, sbo), tc_desc(bh + off, lbo, sbo), idesc, 1u);
      }
      tc_commit(mbar);
    }
    const bool done = neg || tc_mbar_wait(mbar, phase, kTcMaxWaitIters);
    if (!neg) phase ^= 1u;
    if (!done) {   // the tensor-core work did not complete in time: report and stop
      if (lane == 0) atomicExch(err, 1);
      ok = false;
    }
    ok = __syncthreads_and(ok);
    if (!ok) break;
    tc_fence_after();

    // ---- 3. rows of M -> node-pair blocks -> ELL ---------------------------------------
    {
      float v[S::LW];
      if (neg) {
        // M[r][c] = sum_k sign(w_k) A[r][k] A[c][k] with A = hi + lo from the tiles: this
        // lane's row r against the columns of its own element
        int e0l, i0l;
        if constexpr (S::WPE > 1) {
          e0l = warp / S::WPE;
          i0l = (warp % S::WPE) * S::NPW + lane / DIM;
        } else {
          e0l = warp * S::EPW + lane / S::RPE;
          i0l = (lane % S::RPE) / DIM;
        }
        const int rr = warp * 32 + lane;
#pragma unroll
        for (int j = 0; j < NEN; ++j)
#pragma unroll
          for (int b = 0; b < DIM; ++b) {
            const int cc = tc_row<ET>(e0l < EPG ? e0l : 0, j, b);
            double acc = 0.0;   // FP64 products and sum of the split operands (hi + lo exact)
            if (e0l < ne && i0l < NEN)
              for (int g = 0; g < ngp; ++g) {
                const int kb = (g >> 2) * 512 + (g & 3);
                const double sg = swt[e0l * ngp + g] < 0.f ? -1.0 : 1.0;
                acc += sg * ((double)aH[kb + rr * 4] + (double)aL[kb + rr * 4]) *
                       ((double)aH[kb + cc * 4] + (double)aL[kb + cc * 4]);
              }
            v[tc_col<ET>(j, b)] = (float)acc;
          }
      } else if constexpr (S::WPE > 1) {
        const int e = warp / S::WPE;
        float t0[32], t1[32];
        const uint32_t base = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(e * S::LW);
        tc_ld32(base, t0);
        tc_ld32(base + 32, t1);
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          v[c] = t0[c];
          v[32 + c] = t1[c];
        }
      } else {
        float t[32];
        tc_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(warp * 32), t);
        const int s = lane / S::RPE;   // this lane's element within the warp
#pragma unroll
        for (int c = 0; c < S::LW; ++c) {
          float x = t[c];
#pragma unroll
          for (int q = 1; q < S::EPW; ++q)
            if (s == q) x = t[q * S::RPE + c];
          v[c] = x;
        }
      }
      if (!neg) tc_wait_ld();

      // this lane's (element, node, component)
      int e, i, a;
      if constexpr (S::WPE > 1) {
        e = warp / S::WPE;
        i = (warp % S::WPE) * S::NPW + lane / DIM;
        a = lane % DIM;
      } else {
        e = warp * S::EPW + lane / S::RPE;
        i = (lane % S::RPE) / DIM;
        a = (lane % S::RPE) % DIM;
      }
      const bool valid = i < NEN && (S::WPE > 1 ? lane < S::NPW * DIM : true) && e < ne;
      if constexpr (GRAM) {
        // this lane's row of M, (node i, component a), as RAW contiguous floats
        if (valid) {
          constexpr int RAW = S::RAW;
          float* dst = K + (int64_t)sel[e] * RAW * RAW + (int64_t)(i * DIM + a) * RAW;
#pragma unroll
          for (int q = 0; q < RAW / 4; ++q) {
            float4 w4;
            w4.x = v[tc_col<ET>((4 * q) / DIM, (4 * q) % DIM)];
            w4.y = v[tc_col<ET>((4 * q + 1) / DIM, (4 * q + 1) % DIM)];
            w4.z = v[tc_col<ET>((4 * q + 2) / DIM, (4 * q + 2) % DIM)];
            w4.w = v[tc_col<ET>((4 * q + 3) / DIM, (4 * q + 3) % DIM)];
            __stcs(reinterpret_cast<float4*>(dst) + q, w4);
          }
        }
      } else {
      const int ni = valid ? sconn[e * NEN + i] : 0;
#pragma unroll
      for (int j = 0; j < NEN; ++j) {
        float prow[DIM];
#pragma unroll
        for (int b = 0; b < DIM; ++b) prow[b] = v[tc_col<ET>(j, b)];
        // column a of the block from the node's other lanes: lane of component
        // (a + o) % DIM sends its entry at column a (so each lane selects by its own a)
        float pcol[DIM];
        float diag = prow[0];
#pragma unroll
        for (int b = 1; b < DIM; ++b)
          if (a == b) diag = prow[b];
        float tr = diag;
        pcol[0] = 0.f;
#pragma unroll
        for (int c = 0; c < DIM; ++c) pcol[c] = prow[c];   // overwritten below except c = a
#pragma unroll
        for (int o = 1; o < DIM; ++o) {
          const int src_c = (a + o) % DIM;
          const int src = lane - a + src_c;
          const int want = (a + DIM - o) % DIM;   // the column the receiver of this lane needs
          float send = prow[0];
#pragma unroll
          for (int b = 1; b < DIM; ++b)
            if (want == b) send = prow[b];
          const float got = __shfl_sync(0xffffffffu, send, src & 31);
          const float gd = __shfl_sync(0xffffffffu, diag, src & 31);
          tr += gd;
#pragma unroll
          for (int c = 0; c < DIM; ++c)
            if (c == src_c) pcol[c] = got;
        }
        if (valid) {
          // column a of V = lam1 P + mu1 P^T + mu1 tr I: V[c][a] = lam1 P[c][a] + mu1 P[a][c]
          float col[DIM];
#pragma unroll
          for (int c = 0; c < DIM; ++c) col[c] = lam1 * pcol[c] + mu1 * prow[c] + (c == a ? mu1 * tr : 0.f);
          const int slot = sslot[e * NEN * NEN + i * NEN + j];
          add_rows<DIM, float, ATOMIC>(&K[(int64_t)(slot * DIM + a) * n + (int64_t)ni * DIM], col);
        }
      }
      }
    }
    tc_fence_before();
    __syncthreads();
  }

  // release the TMEM columns (after every read of them has completed)
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tc_dealloc(tmem, kTcCols);
}

template <int ET>
gf_status launch_tc(gf_ctx* ctx, int scatter, const AsmTables* d_tab, float* K, int* d_err) {
  const TcSmem<ET> L = tc_smem<ET>(ctx->ngp);
  // at most 4 CTAs per SM (4 x 128 TMEM columns = the SM's 512): each asks for at least a
  // quarter of the SM's 228 KB of shared memory, less the 1 KB the system reserves per CTA
  const size_t sm = std::max(L.total, (size_t)56 * 1024);
  auto kc = k_assemble_tc<ET, 0>;
  auto ka = k_assemble_tc<ET, 1>;
  auto kg = k_assemble_tc<ET, 2>;
  GF_CUDA(ctx, gf_smem_attr(kg, (int)sm));
  GF_CUDA(ctx, gf_func_attr(reinterpret_cast<const void*>(kg),
                            cudaFuncAttributePreferredSharedMemoryCarveout,
                            (int)cudaSharedmemCarveoutMaxShared));
  GF_CUDA(ctx, gf_smem_attr(kc, (int)sm));
  GF_CUDA(ctx, gf_smem_attr(ka, (int)sm));
  // the whole unified L1/shared array as shared memory, so that the occupancy query and the
  // launch see the same carve-out
  GF_CUDA(ctx, gf_func_attr(reinterpret_cast<const void*>(kc),
                            cudaFuncAttributePreferredSharedMemoryCarveout,
                            (int)cudaSharedmemCarveoutMaxShared));
  GF_CUDA(ctx, gf_func_attr(reinterpret_cast<const void*>(ka),
                            cudaFuncAttributePreferredSharedMemoryCarveout,
                            (int)cudaSharedmemCarveoutMaxShared));
  // resident CTAs per SM: registers, shared memory and the 512 TMEM columns of an SM
  const int per_sm = tc_ctas_per_sm(scatter == GF_SCATTER_OWNER    ? kg
                                    : scatter == GF_SCATTER_ATOMIC ? ka : kc,
                                    kTcThreads, sm, kTcCols);
  const int grid_cap = ctx->sm_count * per_sm;
  const float lam1 = (float)ctx->lam1, mu1 = (float)ctx->mu1;
  constexpr int EPG = TcShape<ET>::EPG;
  if (scatter == GF_SCATTER_OWNER) {   // Gram matrices to K (the `K` argument) for the gather
    const int count = ctx->nelem;
    const int grid = std::min(grid_cap, (count + EPG - 1) / EPG);
    kg<<<grid, kTcThreads, sm, ctx->stream>>>(ctx->d_allperm, count, ctx->ngp, ctx->d_conn,
                                              ctx->d_coords64, ctx->d_Eel32, nullptr,
                                              ctx->nelem, ctx->n, d_tab, lam1, mu1, K, d_err);
    GF_LAUNCH_CHECK(ctx, "k_assemble_tc(gram)");
  } else if (scatter == GF_SCATTER_ATOMIC) {
    const int count = ctx->nelem;
    const int grid = std::min(grid_cap, (count + EPG - 1) / EPG);
    ka<<<grid, kTcThreads, sm, ctx->stream>>>(ctx->d_allperm, count, ctx->ngp, ctx->d_conn,
                                              ctx->d_coords64, ctx->d_Eel32, ctx->d_slotmap,
                                              ctx->nelem, ctx->n, d_tab, lam1, mu1, K, d_err);
    GF_LAUNCH_CHECK(ctx, "k_assemble_tc(atomic)");
  } else {
    for (int c = 0; c < ctx->ncolors; ++c) {
      const int c0 = ctx->color_off[c], count = ctx->color_off[c + 1] - c0;
      if (count == 0) continue;
      const int grid = std::min(grid_cap, (count + EPG - 1) / EPG);
      kc<<<grid, kTcThreads, sm, ctx->stream>>>(ctx->d_perm + c0, count, ctx->ngp, ctx->d_conn,
                                                ctx->d_coords64, ctx->d_Eel32, ctx->d_slotmap,
                                                ctx->nelem, ctx->n, d_tab, lam1, mu1, K, d_err);
      GF_LAUNCH_CHECK(ctx, "k_assemble_tc(colour)");
    }
  }
  return GF_OK;
}

}  // namespace

// FP32 assembly with the tcgen05 tensor-core engine (colour or atomic schedule: into K;
// owner schedule: each element's Gram matrix into K as nelem x RAW x RAW floats, which
// gf_assemble_owner_gram then gathers); d_err (device int, zeroed by the caller) is set if
// an MMA-completion wait timed out.
gf_status gf_assemble_tc(gf_ctx* ctx, int scatter, const AsmTables* d_tab, float* K, int* d_err) {
  switch (ctx->elem_type) {
    case GF_Q4: return launch_tc<GF_Q4>(ctx, scatter, d_tab, K, d_err);
    case GF_Q8: return launch_tc<GF_Q8>(ctx, scatter, d_tab, K, d_err);
    case GF_BRICK8: return launch_tc<GF_BRICK8>(ctx, scatter, d_tab, K, d_err);
    default: return launch_tc<GF_BRICK20>(ctx, scatter, d_tab, K, d_err);
  }
}
