// Owner-computes assembly (GF_SCATTER_OWNER): every ELL entry of K is written
// exactly once, with coalesced stores, and no global atomics, colouring or
// zero-fill are needed.
//
// Same arithmetic as gf_assemble.cu (node-pair blocks lam1 g_i g_j^T +
// mu1 g_j g_i^T + mu1 (g_i . g_j) I, weighted by w detJ E), organised by rows:
//
//   k_elem_geometry  element-parallel, thread per (element, Gauss point): J^-1 and
//                    w*detJ.  Element-local coordinates x_i - x_0 are formed in
//                    FP64; J, J^-1 are FP64 for the FP64 path and for FP32 elements
//                    whose max/min |detJ| over the Gauss points exceeds 10.
//                    Layout GEO[element][gp][dim*dim + 1].
//   k_assemble_owner a CTA owns NB consecutive nodes = NB*dim consecutive ELL rows,
//                    with a shared-memory tile of those rows ([slot][row], W slots).
//                    One task per (owned node a, incident element e) accumulates
//                    H_j = sum_gp (w detJ E) g_i g_j^T, g = J^-1 dN, for the block
//                    row i_a of Ke(e) and adds each block into the tile at the
//                    neighbour slot of node j (shared-memory atomics: two elements
//                    around a can hit the same slot).  A task is split into work
//                    items of JG element nodes j each, so that 3-D blocks, which own
//                    few nodes, still give every thread work.  The tile is then written to
//                    K: for each slot the CTA's rows are contiguous in the
//                    column-major ELL, so the stores coalesce, and padding slots
//                    get their zeros.
// Storing J^-1 (dim^2 + 1 values per Gauss point) instead of all node gradients
// (nen*dim values) keeps the per-element buffer small: each element is re-read
// once per owner node, so its size, not the extra FMAs, sets the cost.
// Each element's block rows are formed by the owners of its nodes (no symmetry
// saving), in exchange for K — the dominant traffic — being written once instead
// of zero-filled and read-modified-written per contribution.  Reference: the
// scatter of StiffAlgo::AssembleK (src/FEM/StiffAlgo.cc:304-401), by rows.
#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "gf_elem.cuh"

namespace {

constexpr int kOT = 256;
constexpr size_t kOwnerSmemLimit = 60 * 1024;

// ---------------------------------------------------------------------------
template <int ET, typename TC>
__global__ void __launch_bounds__(kOT)
k_elem_geometry(int nelem, int ngp, int EB, const int32_t* __restrict__ conn,
                const double* __restrict__ coords, const AsmTables* __restrict__ tab,
                TC* __restrict__ geo) {
  constexpr ElemInfo info = gf_elem_info(ET);
  constexpr int NEN = info.nen, DIM = info.dim, GS = DIM * DIM + 1;
  const bool f64 = sizeof(TC) == 8;
  __shared__ double sX64[kOT / 4 * GF_MAX_NEN * 3];  // EB * NEN * DIM (EB <= 64)
  __shared__ float sdet[kOT];
  __shared__ int sflag[kOT / 4];
  const int e0 = blockIdx.x * EB;
  const int ne = min(EB, nelem - e0);
  for (int k = threadIdx.x; k < ne * NEN; k += kOT) {
    const int e = k / NEN, i = k % NEN;
    const int node = conn[(int64_t)(e0 + e) * NEN + i];
    const int node0 = conn[(int64_t)(e0 + e) * NEN];
#pragma unroll
    for (int c = 0; c < DIM; ++c)
      sX64[k * DIM + c] = coords[(int64_t)node * DIM + c] - coords[(int64_t)node0 * DIM + c];
  }
  __syncthreads();
  const int t = threadIdx.x;
  const int el = t / ngp, g = t % ngp;
  const bool active = t < ne * ngp;
  const double* X = sX64 + el * NEN * DIM;
  float Jf[3][3], Jif[3][3];
  float detf = 0.f;
  if (active) {
    const float* dN = tab->dN32 + g * DIM * NEN;
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
      for (int b = 0; b < DIM; ++b) {
        float s = 0.f;
#pragma unroll
        for (int i = 0; i < NEN; ++i) s += dN[a * NEN + i] * (float)X[i * DIM + b];
        Jf[a][b] = s;
      }
    detf = gf_det_inv<DIM, float>(Jf, Jif);
    sdet[t] = fabsf(detf);
  }
  __syncthreads();
  if (t < ne) {
    float dmin = 3.4e38f, dmax = 0.f;
    for (int k = 0; k < ngp; ++k) {
      dmin = fminf(dmin, sdet[t * ngp + k]);
      dmax = fmaxf(dmax, sdet[t * ngp + k]);
    }
    sflag[t] = dmax > 10.f * dmin ? 1 : 0;
  }
  __syncthreads();
  if (!active) return;
  TC* out = geo + ((int64_t)(e0 + el) * ngp + g) * GS;
  if (f64 || sflag[el]) {
    const double* dN = tab->dN64 + g * DIM * NEN;
    double J[3][3], Ji[3][3];
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
      for (int b = 0; b < DIM; ++b) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < NEN; ++i) s += dN[a * NEN + i] * X[i * DIM + b];
        J[a][b] = s;
      }
    const double d = gf_det_inv<DIM, double>(J, Ji);
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
      for (int b = 0; b < DIM; ++b) out[a * DIM + b] = TC(Ji[a][b]);
    out[DIM * DIM] = TC(tab->w64[g] * d);
  } else {
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
      for (int b = 0; b < DIM; ++b) out[a * DIM + b] = TC(Jif[a][b]);
    out[DIM * DIM] = TC(tab->w32[g] * detf);
  }
}

// Thread per element (element types with at most 24 coordinates): the element's
// local coordinates stay in registers (FP64, plus their FP32 rounding) and the Gauss
// rule is a compile-time table; same arithmetic and output as k_elem_geometry.  With
// NODE (the input of k_assemble_owner_node) an element's block starts every PS values,
// PS = PER rounded up to 8 (zero padding: 32-byte aligned blocks for vector loads), and
// the stored w detJ is multiplied by the element's modulus (the product the owner
// kernel would otherwise form per Gauss point).  Each warp stages its 32 elements'
// output in shared memory and stores it as one contiguous, coalesced block.
template <int ET, typename TC, int NG1>
constexpr int geo_stride(bool node) {
  constexpr int PER = GpTable<ET, NG1>::NGP * (gf_elem_info(ET).dim * gf_elem_info(ET).dim + 1);
  return node ? (PER + 7) / 8 * 8 : PER;
}

template <int ET, typename TC, int NG1>
constexpr int geo_stage_stride(bool node) {
  return geo_stride<ET, TC, NG1>(node) | 1;
}

template <int ET, typename TC, int NG1, bool NODE>
__global__ void __launch_bounds__(kOT, gf_elem_info(ET).dim == 2 ? 3 : 1)
k_elem_geometry_pe(int nelem, const int32_t* __restrict__ conn,
                   const double* __restrict__ coords, const TC* __restrict__ Eel,
                   TC* __restrict__ geo) {
  constexpr ElemInfo info = gf_elem_info(ET);
  constexpr int NEN = info.nen, DIM = info.dim, GS = DIM * DIM + 1;
  constexpr int NGP = GpTable<ET, NG1>::NGP;
  constexpr int PER = NGP * GS;  // output values per element
  constexpr int PS = geo_stride<ET, TC, NG1>(NODE);
  constexpr GpTable<ET, NG1> Tab = gf_gp_table<ET, NG1>();
  // 1-D weights (1, 1) or (5/9, 8/9, 5/9), multiplied in the reference's tensor order
  constexpr double w1[3] = {NG1 == 2 ? 1.0 : 5.0 / 9.0, NG1 == 2 ? 1.0 : 8.0 / 9.0, 5.0 / 9.0};
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // staging rows of SPS = PS rounded up to odd: a warp's 32 element rows, written a value
  // at a time, then fall on distinct banks
  constexpr int SPS = geo_stage_stride<ET, TC, NG1>(NODE);
  TC* stage = reinterpret_cast<TC*>(smem_raw) + (size_t)(threadIdx.x >> 5) * 32 * SPS;
  const bool f64 = sizeof(TC) == 8;
  const int lane = threadIdx.x & 31;
  const int e0 = (blockIdx.x * kOT + threadIdx.x) & ~31;  // first element of the warp
  const int e = e0 + lane;
  if (e0 >= nelem) return;
  if (e < nelem) {
    double X[NEN][DIM];
    float Xf[NEN][DIM];
    {
      const int node0 = conn[(int64_t)e * NEN];
      double x0[DIM];
#pragma unroll
      for (int c = 0; c < DIM; ++c) x0[c] = coords[(int64_t)node0 * DIM + c];
#pragma unroll
      for (int i = 0; i < NEN; ++i) {
        const int node = conn[(int64_t)e * NEN + i];
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
          X[i][c] = coords[(int64_t)node * DIM + c] - x0[c];
          Xf[i][c] = (float)X[i][c];
        }
      }
    }
    // FP32 J^-1 and w detJ straight into the staging block, with the distortion test over
    // the same Jacobians; an element that fails it is redone in FP64 (rare)
    TC* out = stage + lane * SPS;
#pragma unroll
    for (int k = PER; k < PS; ++k) out[k] = TC(0);
    const TC Ee = NODE ? Eel[e] : TC(1);
    bool use64 = f64;
    if (!f64) {
      float dmin = 3.4e38f, dmax = 0.f;
#pragma unroll
      for (int g = 0; g < NGP; ++g) {
        const int gi = DIM == 2 ? g / NG1 : g / (NG1 * NG1);
        const int gj = DIM == 2 ? g % NG1 : (g / NG1) % NG1;
        const int gk = DIM == 2 ? 0 : g % NG1;
        const double wg = w1[gi] * w1[gj] * (DIM == 2 ? 1.0 : w1[gk]);
        float J[3][3], Ji[3][3];
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
          for (int c = 0; c < DIM; ++c) {
            float s = 0.f;
#pragma unroll
            for (int i = 0; i < NEN; ++i) s += Tab.d32[(g * DIM + a) * NEN + i] * Xf[i][c];
            J[a][c] = s;
          }
        const float d = gf_det_inv<DIM, float>(J, Ji);
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
          for (int c = 0; c < DIM; ++c) out[g * GS + a * DIM + c] = TC(Ji[a][c]);
        out[g * GS + DIM * DIM] = NODE ? TC((float)wg * d) * Ee : TC((float)wg * d);
        dmin = fminf(dmin, fabsf(d));
        dmax = fmaxf(dmax, fabsf(d));
      }
      use64 = dmax > 10.f * dmin;
    }
    if (use64) {
#pragma unroll
      for (int g = 0; g < NGP; ++g) {
        const int gi = DIM == 2 ? g / NG1 : g / (NG1 * NG1);
        const int gj = DIM == 2 ? g % NG1 : (g / NG1) % NG1;
        const int gk = DIM == 2 ? 0 : g % NG1;
        const double wg = w1[gi] * w1[gj] * (DIM == 2 ? 1.0 : w1[gk]);
        double J[3][3], Ji[3][3];
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
          for (int c = 0; c < DIM; ++c) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < NEN; ++i) s += Tab.d64[(g * DIM + a) * NEN + i] * X[i][c];
            J[a][c] = s;
          }
        const double d = gf_det_inv<DIM, double>(J, Ji);
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
          for (int c = 0; c < DIM; ++c) out[g * GS + a * DIM + c] = TC(Ji[a][c]);
        out[g * GS + DIM * DIM] = NODE ? TC(wg * d) * Ee : TC(wg * d);
      }
    }
  }
  __syncwarp();
  // the warp's elements are consecutive: their outputs form one contiguous block
  const int nw = min(32, nelem - e0);
  TC* dst = geo + (int64_t)e0 * PS;
  for (int k = lane; k < nw * PS; k += 32) {
    const int el = k / PS;
    dst[k] = stage[el * SPS + (k - el * PS)];
  }
}

// Block rows H_j, j in [J0, J0 + JG), of one task with the Gauss rule known at compile
// time: every dN_j value is an instruction constant, only J^-1 / w*detJ (global) and
// the owned node's row of dN (shared memory) are read.
template <int ET, typename TC, int JG, int NG1, int J0>
__device__ __forceinline__ void owner_rows_ct(const TC* __restrict__ ge, TC Ee,
                                              const TC* __restrict__ sdN, int i,
                                              TC (&H)[JG][gf_elem_info(ET).dim][gf_elem_info(ET).dim]) {
  constexpr ElemInfo info = gf_elem_info(ET);
  constexpr int NEN = info.nen, DIM = info.dim, GS = DIM * DIM + 1;
  constexpr GpTable<ET, NG1> Tab = gf_gp_table<ET, NG1>();
#pragma unroll
  for (int g = 0; g < GpTable<ET, NG1>::NGP; ++g) {
    TC Ji[DIM][DIM];
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
      for (int b = 0; b < DIM; ++b) Ji[a][b] = __ldg(ge + g * GS + a * DIM + b);
    const TC wd = __ldg(ge + g * GS + DIM * DIM) * Ee;
    const TC* dN = sdN + g * DIM * NEN;
    TC gi[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      TC s = TC(0);
#pragma unroll
      for (int a = 0; a < DIM; ++a) s += Ji[c][a] * dN[a * NEN + i];
      gi[c] = s * wd;
    }
#pragma unroll
    for (int jj = 0; jj < JG; ++jj) {
      TC gj[DIM];
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        TC s = TC(0);
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
          const int q = (g * DIM + a) * NEN + J0 + jj;
          s += Ji[c][a] * (sizeof(TC) == 8 ? TC(Tab.d64[q]) : TC(Tab.d32[q]));
        }
        gj[c] = s;
      }
#pragma unroll
      for (int a = 0; a < DIM; ++a)
#pragma unroll
        for (int b = 0; b < DIM; ++b) H[jj][a][b] += gi[a] * gj[b];
    }
  }
}

// Runtime node-group index -> the compile-time instance for that group.
template <int ET, typename TC, int JG, int NG1, int... G>
__device__ __forceinline__ void owner_rows_ct_switch(
    int jg, const TC* ge, TC Ee, const TC* sdN, int i,
    TC (&H)[JG][gf_elem_info(ET).dim][gf_elem_info(ET).dim], std::integer_sequence<int, G...>) {
  ((jg == G ? owner_rows_ct<ET, TC, JG, NG1, G * JG>(ge, Ee, sdN, i, H) : void()), ...);
}

// ---------------------------------------------------------------------------
// One work item per (task, group of JG element nodes j): a task's NEN/JG items run
// on neighbouring lanes and read the same element data.  The owning node of every
// task is found once per CTA (binary search in the CTA's incidence offsets).
template <int ET, typename TC, int JG, int NG1>
__global__ void __launch_bounds__(kOT)
k_assemble_owner(int nnodes, int n, int W, int NB, int ngp,
                 const int32_t* __restrict__ inc_off, const int32_t* __restrict__ inc,
                 const uint8_t* __restrict__ inc_loc, const uint16_t* __restrict__ inc_slot,
                 const TC* __restrict__ geo, const TC* __restrict__ Eel,
                 const AsmTables* __restrict__ tab, TC lam1, TC mu1, TC* __restrict__ K) {
  constexpr ElemInfo info = gf_elem_info(ET);
  constexpr int NEN = info.nen, DIM = info.dim, GS = DIM * DIM + 1;
  constexpr int NJ = NEN / JG;
  static_assert(NEN % JG == 0, "node groups must tile the element");
  const bool f64 = sizeof(TC) == 8;
  const int RB = NB * DIM;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TC* tile = reinterpret_cast<TC*>(smem_raw);       // [W][RB]
  TC* sdN = tile + (size_t)W * RB;                  // [ngp][DIM][NEN]
  int* soff = reinterpret_cast<int*>(sdN + ngp * DIM * NEN);  // [NB + 1]
  uint8_t* sal = reinterpret_cast<uint8_t*>(soff + NB + 1);    // [tasks] owning node

  const int a0 = blockIdx.x * NB;
  const int a1 = min(a0 + NB, nnodes);
  for (int k = threadIdx.x; k < W * RB; k += kOT) tile[k] = TC(0);
  for (int k = threadIdx.x; k < ngp * DIM * NEN; k += kOT)
    sdN[k] = f64 ? TC(tab->dN64[k]) : TC(tab->dN32[k]);
  for (int k = threadIdx.x; k <= a1 - a0; k += kOT) soff[k] = inc_off[a0 + k];
  __syncthreads();
  const int q0 = soff[0];
  const int T = soff[a1 - a0] - q0;
  for (int t = threadIdx.x; t < T; t += kOT) {
    int lo = 0, hi = a1 - a0;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (soff[mid] - q0 <= t) lo = mid; else hi = mid;
    }
    sal[t] = (uint8_t)lo;
  }
  __syncthreads();

  for (int w = threadIdx.x; w < T * NJ; w += kOT) {
    const int t = w / NJ;
    const int j0 = (w - t * NJ) * JG;
    const int al = sal[t];
    const int q = q0 + t;
    const int e = inc[q];
    const int i = inc_loc[q];
    const TC Ee = Eel[e];
    const TC* ge = geo + (int64_t)e * ngp * GS;
    const uint16_t* slots = inc_slot + (int64_t)q * NEN;
    TC H[JG][DIM][DIM];
#pragma unroll
    for (int jj = 0; jj < JG; ++jj)
#pragma unroll
      for (int a = 0; a < DIM; ++a)
#pragma unroll
        for (int b = 0; b < DIM; ++b) H[jj][a][b] = TC(0);
    if constexpr (NG1 > 0) {
      owner_rows_ct_switch<ET, TC, JG, NG1>(j0 / JG, ge, Ee, sdN, i, H,
                                            std::make_integer_sequence<int, NJ>{});
    } else {
#pragma unroll 1
      for (int g = 0; g < ngp; ++g) {
        TC Ji[DIM][DIM];
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
          for (int b = 0; b < DIM; ++b) Ji[a][b] = __ldg(ge + g * GS + a * DIM + b);
        const TC wd = __ldg(ge + g * GS + DIM * DIM) * Ee;
        const TC* dN = sdN + g * DIM * NEN;
        TC gi[DIM];
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
          TC s = TC(0);
#pragma unroll
          for (int a = 0; a < DIM; ++a) s += Ji[c][a] * dN[a * NEN + i];
          gi[c] = s * wd;
        }
#pragma unroll
        for (int jj = 0; jj < JG; ++jj) {
          const int j = j0 + jj;
          TC gj[DIM];
#pragma unroll
          for (int c = 0; c < DIM; ++c) {
            TC s = TC(0);
#pragma unroll
            for (int a = 0; a < DIM; ++a) s += Ji[c][a] * dN[a * NEN + j];
            gj[c] = s;
          }
#pragma unroll
          for (int a = 0; a < DIM; ++a)
#pragma unroll
            for (int b = 0; b < DIM; ++b) H[jj][a][b] += gi[a] * gj[b];
        }
      }
    }
#pragma unroll
    for (int jj = 0; jj < JG; ++jj) {
      const int p = slots[j0 + jj];
      TC tr = TC(0);
#pragma unroll
      for (int a = 0; a < DIM; ++a) tr += H[jj][a][a];
#pragma unroll
      for (int a = 0; a < DIM; ++a)
#pragma unroll
        for (int b = 0; b < DIM; ++b) {
          TC v = lam1 * H[jj][a][b] + mu1 * H[jj][b][a];
          if (a == b) v += mu1 * tr;
          atomicAdd(&tile[(size_t)(p * DIM + b) * RB + al * DIM + a], v);
        }
    }
  }
  __syncthreads();
  // flush: warp w stores slots w, w + 8, ...; lanes stride the block's rows.  Streaming
  // (evict-first) stores keep K, written once, from displacing the geometry buffer
  // the other CTAs still read from L2.
  const int rows = (a1 - a0) * DIM;
  const int64_t row0 = (int64_t)a0 * DIM;
  for (int s = threadIdx.x >> 5; s < W; s += kOT >> 5)
    for (int r = threadIdx.x & 31; r < rows; r += 32)
      __stcs(&K[(int64_t)s * n + row0 + r], tile[(size_t)s * RB + r]);
}

// ---------------------------------------------------------------------------
// 2-D FP32 owner kernel, thread per owned node.  A CTA owns NB consecutive nodes, one
// thread each, and keeps their 2 NB rows as a shared-memory tile [slot][row].  The CTA
// first orders its nodes by degree (incident elements), highest first, so that the
// nodes of a warp walk the same number of elements.  A thread then walks its node's
// incident elements in incidence order and adds the node's block row of each Ke into
// its own two tile rows (row pair = the thread's position, mapped back to the node's rows
// by the store) with plain read-modify-writes: no other thread touches them, so no
// atomics are needed and the sum over elements has a fixed order.  Per Gauss
// point, g_i = w detJ E J^-T dN_i (dN_i from shared memory: i is known at run time) and
// g_j = J^-T dN_j (dN_j instruction constants) form H_j += g_i g_j^T, two entries per
// packed FMA (fma.rn.f32x2: two IEEE single-precision FMAs in one instruction).  J^-1
// and w detJ E are read as 32-byte loads (element stride PS, a multiple of 8 floats):
// the lanes of a warp read 32 different elements, so the number of load requests, not
// the bytes, sets the load cost.  The tile is stored once, two rows per 8-byte store.
constexpr int kDegBuckets = 32;

// 8 consecutive floats from a 32-byte aligned address of read-only data
__device__ __forceinline__ void ldg8(const float* p, float (&v)[8]) {
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]),
        "=f"(v[7])
      : "l"(p));
}


template <int ET, int NG1, int NB>
size_t owner_node_smem_bytes(int W) {
  constexpr int NEN = gf_elem_info(ET).nen;
  return sizeof(float) * (size_t)W * 2 * NB + sizeof(float2) * NG1 * NG1 * NEN +
         sizeof(int) * (3 * NB + 1 + (NB / 32 + 1) * kDegBuckets);
}

// One task of k_assemble_owner_node: the owned node's block row of the element whose
// geometry block is gv (local index i of the node, incidence entry q), added into the
// node's two tile rows.
template <int ET, int NG1, int RB>
__device__ __forceinline__ void owner_node_task(const float* gv, int i, int64_t q,
                                                const uint16_t* __restrict__ inc_slot,
                                                const float2* sdN, float lam1, float mu1,
                                                float* myrows) {
  constexpr int NEN = gf_elem_info(ET).nen, GS = 5, NGP = NG1 * NG1;
  constexpr GpTable<ET, NG1> Tab = gf_gp_table<ET, NG1>();
  float2 H[NEN][2];   // H[j][a] = (H_j[a][0], H_j[a][1])
#pragma unroll
  for (int j = 0; j < NEN; ++j) H[j][0] = H[j][1] = make_float2(0.f, 0.f);
#pragma unroll
  for (int g = 0; g < NGP; ++g) {
    const float j00 = gv[g * GS], j01 = gv[g * GS + 1];
    const float j10 = gv[g * GS + 2], j11 = gv[g * GS + 3];
    const float wd = gv[g * GS + 4];   // w detJ E
    const float2 dn = sdN[g * NEN + i];
    const float gi0 = fmaf(j01, dn.y, j00 * dn.x) * wd;
    const float gi1 = fmaf(j11, dn.y, j10 * dn.x) * wd;
    const float2 g0 = make_float2(gi0, gi0), g1 = make_float2(gi1, gi1);
#pragma unroll
    for (int j = 0; j < NEN; ++j) {
      const float d0 = Tab.d32[(g * 2) * NEN + j], d1 = Tab.d32[(g * 2 + 1) * NEN + j];
      const float2 gj = make_float2(fmaf(j01, d1, j00 * d0), fmaf(j11, d1, j10 * d0));
      H[j][0] = fma2(g0, gj, H[j][0]);
      H[j][1] = fma2(g1, gj, H[j][1]);
    }
  }
  // neighbour slots of the element's nodes (16 or 8 bytes, aligned: q * NEN * 2 bytes)
  uint32_t sw[NEN / 2];
  if constexpr (NEN == 8) {
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(inc_slot + q * NEN));
    sw[0] = v.x; sw[1] = v.y; sw[2] = v.z; sw[3] = v.w;
  } else {
    const uint2 v = __ldg(reinterpret_cast<const uint2*>(inc_slot + q * NEN));
    sw[0] = v.x; sw[1] = v.y;
  }
#pragma unroll
  for (int j = 0; j < NEN; ++j) {
    const int p = (int)((sw[j >> 1] >> (16 * (j & 1))) & 0xFFFFu);
    const float h00 = H[j][0].x, h01 = H[j][0].y, h10 = H[j][1].x, h11 = H[j][1].y;
    const float tr = h00 + h11;
    // V = lam1 H + mu1 H^T + mu1 tr(H) I; column b of V is rows (2 al, 2 al + 1) of
    // tile column 2 p + b: two adjacent floats
    float2* c0 = reinterpret_cast<float2*>(myrows + (size_t)(2 * p) * RB);
    float2* c1 = reinterpret_cast<float2*>(myrows + (size_t)(2 * p + 1) * RB);
    float2 x0 = *c0, x1 = *c1;
    x0.x += fmaf(mu1, tr, fmaf(mu1, h00, lam1 * h00));
    x0.y += fmaf(mu1, h01, lam1 * h10);
    x1.x += fmaf(mu1, h10, lam1 * h01);
    x1.y += fmaf(mu1, tr, fmaf(mu1, h11, lam1 * h11));
    *c0 = x0;
    *c1 = x1;
  }
}

template <int PS>
__device__ __forceinline__ void load_geo(const float* ge, float (&gv)[PS]) {
#pragma unroll
  for (int c = 0; c < PS / 8; ++c) {
    float v[8];
    ldg8(ge + 8 * c, v);
#pragma unroll
    for (int k = 0; k < 8; ++k) gv[8 * c + k] = v[k];
  }
}

template <int ET, int NG1, int NB>
__global__ void __launch_bounds__(NB)
k_assemble_owner_node(int nnodes, int n, int W, const int32_t* __restrict__ inc_off,
                      const int32_t* __restrict__ inc, const uint8_t* __restrict__ inc_loc,
                      const uint16_t* __restrict__ inc_slot, const float* __restrict__ geo,
                      const AsmTables* __restrict__ tab, float lam1, float mu1,
                      float* __restrict__ K) {
  constexpr ElemInfo info = gf_elem_info(ET);
  static_assert(info.dim == 2, "2-D elements");
  constexpr int NEN = info.nen, GS = 5, NGP = NG1 * NG1, RB = 2 * NB, NW = NB / 32;
  constexpr int PS = geo_stride<ET, float, NG1>(true);
  constexpr GpTable<ET, NG1> Tab = gf_gp_table<ET, NG1>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* tile = reinterpret_cast<float*>(smem_raw);                // [W][RB]
  float2* sdN = reinterpret_cast<float2*>(tile + (size_t)W * RB);  // [NGP][NEN]
  int* soff = reinterpret_cast<int*>(sdN + NGP * NEN);             // [NB + 1]
  int* sord = soff + NB + 1;                                       // [NB] node of a thread
  int* spos = sord + NB;                                           // [NB] thread of a node
  int* wcnt = spos + NB;                                           // [NW + 1][kDegBuckets]

  const int t = threadIdx.x;
  const int a0 = blockIdx.x * NB;
  const int na = min(NB, nnodes - a0);
  {
    float4* t4 = reinterpret_cast<float4*>(tile);   // W * RB is a multiple of 4
    for (int k = t; k < W * RB / 4; k += NB) t4[k] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  for (int k = t; k < NGP * NEN; k += NB) {
    const int g = k / NEN, i = k - g * NEN;
    sdN[k] = make_float2(tab->dN32[(g * 2) * NEN + i], tab->dN32[(g * 2 + 1) * NEN + i]);
  }
  for (int k = t; k <= na; k += NB) soff[k] = inc_off[a0 + k];
  for (int k = t; k < NW * kDegBuckets; k += NB) wcnt[k] = 0;
  __syncthreads();
  // stable counting sort of the CTA's nodes by degree, highest first: a node's position
  // is the count of nodes of higher degree plus the nodes of its degree before it (per
  // warp with a match mask, then over the warps).  The node at position t is summed by
  // thread t into tile row pair t, so a warp's 8-byte tile accesses fall on distinct
  // banks; the store maps the pairs back to the nodes' rows.
  const int warp = t >> 5, lane = t & 31;
  const int bkt = t < na ? min(soff[t + 1] - soff[t], kDegBuckets - 1) : -1;
  const unsigned same = __match_any_sync(0xffffffffu, bkt);
  const int wrank = __popc(same & ((1u << lane) - 1u));
  if (bkt >= 0 && wrank == 0) wcnt[warp * kDegBuckets + bkt] = __popc(same);
  __syncthreads();
  if (t == 0) {
    int acc = 0;
    for (int b = kDegBuckets - 1; b >= 0; --b)
      for (int w = 0; w < NW; ++w) {
        const int c = wcnt[w * kDegBuckets + b];
        wcnt[w * kDegBuckets + b] = acc;
        acc += c;
      }
  }
  __syncthreads();
  if (bkt >= 0) {
    const int pos = wcnt[warp * kDegBuckets + bkt] + wrank;
    sord[pos] = t;
    spos[t] = pos;
  }
  __syncthreads();

  const int al = t < na ? sord[t] : 0;
  const int q0 = soff[al];
  const int deg = t < na ? soff[al + 1] - q0 : 0;
  float* myrows = tile + 2 * t;
  for (int k = 0; k < deg; ++k) {
    float gv[PS];
    load_geo(geo + (int64_t)__ldg(inc + q0 + k) * PS, gv);
    owner_node_task<ET, NG1, RB>(gv, __ldg(inc_loc + q0 + k), q0 + k, inc_slot, sdN, lam1, mu1,
                                 myrows);
  }
  __syncthreads();
  // store: warp w takes slots w, w + NB/32, ...; lanes stride the block's row pairs
  // (n is even and a0 * 2 is a multiple of 4, so every pair starts 8-byte aligned)
  const int pairs = na;
  const int64_t row0 = (int64_t)a0 * 2;
  for (int sl = t >> 5; sl < W; sl += NB >> 5) {
    const float2* src = reinterpret_cast<const float2*>(tile + (size_t)sl * RB);
    float2* dst = reinterpret_cast<float2*>(K + (int64_t)sl * n + row0);
    for (int r = t & 31; r < pairs; r += 32) __stcs(dst + r, src[spos[r]]);
  }
}

// ---------------------------------------------------------------------------
// Owner gather of element Gram matrices (FP32, the tensor-core engine's owner schedule).
// The tcgen05 kernel has stored M_e = G W G^T of every element (RAW x RAW floats, rows and
// columns (node, component), w = Gauss weight * detJ * E folded in); a CTA owns NB nodes as
// above and, per (owned node a = local node i of incident element e, group of JG element
// nodes j), reads the 3 x 3 (2 x 2) blocks P = M_e[(i, .), (j, .)] and adds
// V = lam1 P + mu1 P^T + mu1 tr(P) I into its row tile; the tile is then stored once.
// M is read once in total (block (i, j) of M_e belongs to the owner of node i alone).
template <int ET, int JG>
__global__ void __launch_bounds__(kOT)
k_assemble_owner_gram(int nnodes, int n, int W, int NB, const int32_t* __restrict__ inc_off,
                      const int32_t* __restrict__ inc, const uint8_t* __restrict__ inc_loc,
                      const uint16_t* __restrict__ inc_slot, const float* __restrict__ gram,
                      float lam1, float mu1, float* __restrict__ K) {
  constexpr ElemInfo info = gf_elem_info(ET);
  constexpr int NEN = info.nen, DIM = info.dim, RAW = NEN * DIM;
  constexpr int NJ = NEN / JG;
  static_assert(NEN % JG == 0, "node groups must tile the element");
  const int RB = NB * DIM;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* tile = reinterpret_cast<float*>(smem_raw);           // [W][RB]
  int* soff = reinterpret_cast<int*>(tile + (size_t)W * RB);   // [NB + 1]
  uint8_t* sal = reinterpret_cast<uint8_t*>(soff + NB + 1);    // [tasks] owning node

  const int a0 = blockIdx.x * NB;
  const int a1 = min(a0 + NB, nnodes);
  {
    float4* t4 = reinterpret_cast<float4*>(tile);   // W * RB is a multiple of 4 (launcher)
    for (int k = threadIdx.x; k < W * RB / 4; k += kOT) t4[k] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  for (int k = threadIdx.x; k <= a1 - a0; k += kOT) soff[k] = inc_off[a0 + k];
  __syncthreads();
  const int q0 = soff[0];
  const int T = soff[a1 - a0] - q0;
  for (int t = threadIdx.x; t < T; t += kOT) {
    int lo = 0, hi = a1 - a0;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (soff[mid] - q0 <= t) lo = mid; else hi = mid;
    }
    sal[t] = (uint8_t)lo;
  }
  __syncthreads();
  for (int w = threadIdx.x; w < T * NJ; w += kOT) {
    const int t = w / NJ;
    const int j0 = (w - t * NJ) * JG;
    const int al = sal[t];
    const int q = q0 + t;
    const int e = inc[q];
    const int i = inc_loc[q];
    const float* Mi = gram + (int64_t)e * RAW * RAW + (int64_t)(i * DIM) * RAW;
    const uint16_t* slots = inc_slot + (int64_t)q * NEN;
    // the DIM rows of this item, JG * DIM floats each, in 16-byte loads (RAW, JG * DIM and
    // j0 * DIM are multiples of 4, so every segment starts 16-byte aligned)
    constexpr int SEG = JG * DIM;
    static_assert(SEG % 4 == 0 && RAW % 4 == 0, "16-byte segments");
    float seg[DIM][SEG];
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
      for (int u = 0; u < SEG / 4; ++u) {
        const float4 v4 = __ldg(reinterpret_cast<const float4*>(Mi + a * RAW + j0 * DIM) + u);
        seg[a][4 * u] = v4.x;
        seg[a][4 * u + 1] = v4.y;
        seg[a][4 * u + 2] = v4.z;
        seg[a][4 * u + 3] = v4.w;
      }
#pragma unroll
    for (int jj = 0; jj < JG; ++jj) {
      const int j = j0 + jj;
      float P[DIM][DIM];
#pragma unroll
      for (int a = 0; a < DIM; ++a)
#pragma unroll
        for (int b = 0; b < DIM; ++b) P[a][b] = seg[a][jj * DIM + b];
      float tr = 0.f;
#pragma unroll
      for (int a = 0; a < DIM; ++a) tr += P[a][a];
      const int p = slots[j];
#pragma unroll
      for (int a = 0; a < DIM; ++a)
#pragma unroll
        for (int b = 0; b < DIM; ++b) {
          float v = lam1 * P[a][b] + mu1 * P[b][a];
          if (a == b) v += mu1 * tr;
          atomicAdd(&tile[(size_t)(p * DIM + b) * RB + al * DIM + a], v);
        }
    }
  }
  __syncthreads();
  const int rows = (a1 - a0) * DIM;
  const int64_t row0 = (int64_t)a0 * DIM;
  for (int s = threadIdx.x >> 5; s < W; s += kOT >> 5)
    for (int r = threadIdx.x & 31; r < rows; r += 32)
      __stcs(&K[(int64_t)s * n + row0 + r], tile[(size_t)s * RB + r]);
}

template <int ET>
gf_status launch_owner_gram(gf_ctx* ctx, const float* gram, float* K) {
  constexpr ElemInfo info = gf_elem_info(ET);
  const int W = ctx->W;
  auto bytes = [&](int NB) {
    return sizeof(float) * (size_t)W * NB * info.dim + sizeof(int) * (NB + 1) +
           (size_t)NB * ctx->maxval + 16;
  };
  // node blocks of a multiple of 4 nodes, so that the row tile (W x NB x dim floats) is a
  // whole number of 16-byte chunks
  int NB = std::min(128, std::max(16, (ctx->nnodes + 2 * ctx->sm_count - 1) / (2 * ctx->sm_count)));
  NB = NB / 4 * 4;
  while (NB > 4 && bytes(NB) > kOwnerSmemLimit) NB -= 4;
  if (bytes(NB) > kOwnerSmemLimit)
    return gf_fail(ctx, GF_ERR_UNSUPPORTED, "owner gather: a row block does not fit");
  constexpr int JG = info.nen <= 8 ? info.nen : 4;   // JG * dim floats: 16-byte segments
  auto kern = k_assemble_owner_gram<ET, JG>;
  GF_CUDA(ctx, gf_smem_attr(kern, (int)bytes(NB)));
  kern<<<(ctx->nnodes + NB - 1) / NB, kOT, bytes(NB), ctx->stream>>>(
      ctx->nnodes, ctx->n, W, NB, ctx->d_inc_off, ctx->d_inc, ctx->d_inc_loc, ctx->d_inc_slot,
      gram, (float)ctx->lam1, (float)ctx->mu1, K);
  GF_LAUNCH_CHECK(ctx, "k_assemble_owner_gram");
  return GF_OK;
}

template <int ET, typename TC>
size_t owner_smem_bytes(int NB, int W, int ngp, int maxval) {
  constexpr ElemInfo info = gf_elem_info(ET);
  return sizeof(TC) * ((size_t)W * NB * info.dim + (size_t)ngp * info.dim * info.nen) +
         sizeof(int) * (NB + 1) + (size_t)NB * maxval + 16;
}

// element nodes per work item: the whole element for Q4, Q8 and Brick8; for Brick20
// (a CTA owns few nodes) 5 in FP32 and 2 in FP64 (measured on Brick20 64^3)
template <int ET, typename TC>
constexpr int owner_jgroup() {
  return gf_elem_info(ET).nen <= 8 ? gf_elem_info(ET).nen : sizeof(TC) == 4 ? 5 : 2;
}

// Element types whose owner kernel unrolls the Gauss loop against the compile-time
// table (2-D; in 3-D the unrolled loop costs more registers than it saves).
template <int ET, typename TC>
constexpr bool owner_compile_time_gauss() {
  return gf_elem_info(ET).dim == 2;
}

// Geometry buffer of at least `bytes` bytes (kept across assemblies).
static gf_status owner_geo_buffer(gf_ctx* ctx, size_t bytes) {
  if (ctx->geo_bytes >= bytes) return GF_OK;
  if (ctx->d_geo) cudaFree(ctx->d_geo);
  ctx->d_geo = nullptr;
  ctx->geo_bytes = 0;
  if (cudaMalloc(&ctx->d_geo, bytes) != cudaSuccess) {
    cudaGetLastError();
    return gf_fail(ctx, GF_ERR_OOM, "geometry buffer (%zu bytes)", bytes);
  }
  ctx->geo_bytes = bytes;
  return GF_OK;
}

// 2-D FP32: per-element geometry with a 32-byte element stride, then the thread-per-node
// owner kernel (CTAs of kOwnerNodeNB nodes: with a 42-slot Q8 row tile, 45.8 KB of shared
// memory, four CTAs per SM; trimmed to fit five, the kernel measured 4% slower: the
// larger shared carve-out leaves less L1 for the geometry loads).
constexpr int kOwnerNodeNB = 128;
constexpr size_t kOwnerNodeSmemLimit = 112 * 1024;   // two CTAs per SM

template <int ET>
gf_status launch_owner_node(gf_ctx* ctx, float* K, const AsmTables* d_tab) {
  constexpr int NB = kOwnerNodeNB;
  const int W = ctx->W;
  const int PS = ctx->ngauss == 2 ? geo_stride<ET, float, 2>(true) : geo_stride<ET, float, 3>(true);
  gf_status st = owner_geo_buffer(ctx, (size_t)ctx->nelem * PS * sizeof(float));
  if (st != GF_OK) return st;
  float* geo = static_cast<float*>(ctx->d_geo);
  const size_t gsm = sizeof(float) * (size_t)kOT *
                    (ctx->ngauss == 2 ? geo_stage_stride<ET, float, 2>(true)
                                      : geo_stage_stride<ET, float, 3>(true));
  auto gk = ctx->ngauss == 2 ? k_elem_geometry_pe<ET, float, 2, true>
                             : k_elem_geometry_pe<ET, float, 3, true>;
  GF_CUDA(ctx, gf_smem_attr(gk, (int)gsm));
  gk<<<gf_blocks(ctx->nelem, kOT), kOT, gsm, ctx->stream>>>(ctx->nelem, ctx->d_conn,
                                                           ctx->d_coords64, ctx->d_Eel32, geo);
  GF_LAUNCH_CHECK(ctx, "k_elem_geometry_pe");
  cudaEventRecord(ctx->evm, ctx->stream);
  auto kern = ctx->ngauss == 2 ? k_assemble_owner_node<ET, 2, NB> : k_assemble_owner_node<ET, 3, NB>;
  const size_t sm = ctx->ngauss == 2 ? owner_node_smem_bytes<ET, 2, NB>(W)
                                     : owner_node_smem_bytes<ET, 3, NB>(W);
  if (sm > kOwnerNodeSmemLimit)
    return gf_fail(ctx, GF_ERR_UNSUPPORTED, "owner scatter: a row block does not fit");
  GF_CUDA(ctx, gf_smem_attr(kern, (int)sm));
  kern<<<(ctx->nnodes + NB - 1) / NB, NB, sm, ctx->stream>>>(
      ctx->nnodes, ctx->n, W, ctx->d_inc_off, ctx->d_inc, ctx->d_inc_loc, ctx->d_inc_slot,
      geo, d_tab, (float)ctx->lam1, (float)ctx->mu1, K);
  GF_LAUNCH_CHECK(ctx, "k_assemble_owner_node");
  return GF_OK;
}

template <int ET, typename TC>
gf_status launch_owner(gf_ctx* ctx, TC* K, const AsmTables* d_tab) {
  constexpr ElemInfo info = gf_elem_info(ET);
  // 2-D FP32: the thread-per-node kernel, while its row tile keeps two CTAs per SM (a node
  // with very many neighbours, e.g. the centre of a fan of 30 elements, makes W large);
  // wider rows take the task kernel below, which shrinks its node block to fit
  if constexpr (info.dim == 2 && sizeof(TC) == 4) {
    const size_t node_sm = ctx->ngauss == 2 ? owner_node_smem_bytes<ET, 2, kOwnerNodeNB>(ctx->W)
                                            : owner_node_smem_bytes<ET, 3, kOwnerNodeNB>(ctx->W);
    if (node_sm <= kOwnerNodeSmemLimit) return launch_owner_node<ET>(ctx, K, d_tab);
  }
  const int W = ctx->W, ngp = ctx->ngp;
  const int PER = ngp * (info.dim * info.dim + 1);
  gf_status st = owner_geo_buffer(ctx, (size_t)ctx->nelem * PER * sizeof(TC));
  if (st != GF_OK) return st;
  TC* geo = static_cast<TC*>(ctx->d_geo);
  // per-element kernel where its output staging fits (Q4, Q8; Brick8 with 2x2x2 Gauss)
  const size_t gsm = sizeof(TC) * (size_t)kOT * (ngp * (info.dim * info.dim + 1) | 1);
  bool per_element = false;
  if constexpr (info.nen * info.dim <= 24) {
    if (gsm <= 100 * 1024) {
      auto gk = ctx->ngauss == 2 ? k_elem_geometry_pe<ET, TC, 2, false>
                                 : k_elem_geometry_pe<ET, TC, 3, false>;
      GF_CUDA(ctx, gf_smem_attr(gk, (int)gsm));
      gk<<<gf_blocks(ctx->nelem, kOT), kOT, gsm, ctx->stream>>>(ctx->nelem, ctx->d_conn,
                                                               ctx->d_coords64, nullptr, geo);
      per_element = true;
    }
  }
  if (!per_element) {
    const int EB = kOT / ngp;
    k_elem_geometry<ET, TC><<<(ctx->nelem + EB - 1) / EB, kOT, 0, ctx->stream>>>(
        ctx->nelem, ngp, EB, ctx->d_conn, ctx->d_coords64, d_tab, geo);
  }
  GF_LAUNCH_CHECK(ctx, "k_elem_geometry");
  cudaEventRecord(ctx->evm, ctx->stream);
  // largest node block (at most 128: the owning node index is a byte) whose tile keeps
  // three CTAs per SM; small meshes take smaller blocks so that every SM gets two CTAs
  // (Q4 64^2, 4,225 nodes: 25 us with 33 CTAs of 128 nodes, 20 us with 66 of 64; on
  // Q8 512^2, 64 and 96 measured 6% slower than 128)
  int NB = std::min(128, std::max(16, (ctx->nnodes + 2 * ctx->sm_count - 1) / (2 * ctx->sm_count)));
  while (NB > 1 && owner_smem_bytes<ET, TC>(NB, W, ngp, ctx->maxval) > kOwnerSmemLimit) --NB;
  const size_t sm = owner_smem_bytes<ET, TC>(NB, W, ngp, ctx->maxval);
  if (sm > kOwnerSmemLimit)
    return gf_fail(ctx, GF_ERR_UNSUPPORTED, "owner scatter: a row block does not fit");
  constexpr int JG = owner_jgroup<ET, TC>();
  auto kern = k_assemble_owner<ET, TC, JG, 0>;
  if constexpr (owner_compile_time_gauss<ET, TC>())
    kern = ctx->ngauss == 2 ? k_assemble_owner<ET, TC, JG, 2> : k_assemble_owner<ET, TC, JG, 3>;
  GF_CUDA(ctx, gf_smem_attr(kern, (int)sm));
  const TC* Eel = sizeof(TC) == 8 ? (const TC*)ctx->d_Eel : (const TC*)ctx->d_Eel32;
  kern<<<(ctx->nnodes + NB - 1) / NB, kOT, sm, ctx->stream>>>(
      ctx->nnodes, ctx->n, W, NB, ngp, ctx->d_inc_off, ctx->d_inc, ctx->d_inc_loc,
      ctx->d_inc_slot, geo, Eel, d_tab, TC(ctx->lam1), TC(ctx->mu1), K);
  GF_LAUNCH_CHECK(ctx, "k_assemble_owner");
  return GF_OK;
}

template <typename TC>
gf_status owner_dispatch(gf_ctx* ctx, TC* K, const AsmTables* d_tab) {
  switch (ctx->elem_type) {
    case GF_Q4: return launch_owner<GF_Q4, TC>(ctx, K, d_tab);
    case GF_Q8: return launch_owner<GF_Q8, TC>(ctx, K, d_tab);
    case GF_BRICK8: return launch_owner<GF_BRICK8, TC>(ctx, K, d_tab);
    default: return launch_owner<GF_BRICK20, TC>(ctx, K, d_tab);
  }
}

}  // namespace

// Launches the owner-computes assembly on the context's stream (no sync).
gf_status gf_assemble_owner(gf_ctx* ctx, int dtype, const AsmTables* d_tab) {
  if (ctx->ngp < 4 || ctx->ngp > GF_MAX_GP)
    return gf_fail(ctx, GF_ERR_UNSUPPORTED, "Gauss rule size %d", ctx->ngp);
  if (dtype == GF_F64) return owner_dispatch<double>(ctx, ctx->d_K64, d_tab);
  return owner_dispatch<float>(ctx, ctx->d_K32, d_tab);
}

// Launches the owner gather of the element Gram matrices `gram` (stored by the tensor-core
// kernel) into the FP32 matrix K on the context's stream (no sync).
gf_status gf_assemble_owner_gram(gf_ctx* ctx, const float* gram, float* K) {
  switch (ctx->elem_type) {
    case GF_Q4: return launch_owner_gram<GF_Q4>(ctx, gram, K);
    case GF_Q8: return launch_owner_gram<GF_Q8>(ctx, gram, K);
    case GF_BRICK8: return launch_owner_gram<GF_BRICK8>(ctx, gram, K);
    default: return launch_owner_gram<GF_BRICK20>(ctx, gram, K);
  }
}
