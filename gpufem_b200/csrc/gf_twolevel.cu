// Two-level preconditioner: Jacobi plus a coarse correction on rigid-body modes of
// geometric node aggregates (GF_SOLVER_TWOLEVEL_PCG).  No counterpart in the reference (its CG
// is unpreconditioned, src/SPRmatrix/SPRmatrix.cc:405-480).
//
//   M r = D^-1 r + P (P^T K P)^-1 P^T r
//
// Nodes are grouped into aggregates by boxes of a regular grid over the mesh's
// bounding box, sized so that the coarse space has about `target` unknowns.  The
// columns of P for aggregate A are its rigid-body modes restricted to its nodes: the
// dim translations and the dim(dim-1)/2 rotations about the aggregate centroid c_A
// (offsets d = (x - c_A) / s, s = the box side); rows of constrained dofs are zero.
// M is symmetric positive definite, so plain PCG applies.  The coarse matrix
// Ac = P^T K P is assembled on the device from the ELL node blocks, regularised by
// 1e-10 * max diag (modes that the constraints pin down), and inverted in place by a
// blocked Gauss-Jordan sweep (SPD: no pivoting); the inverse is symmetrised and kept in
// FP64 for the per-iteration product.
//
// One application: restriction (block per aggregate over its node list), the coarse
// product from the packed upper triangle of the symmetric inverse (64 x 64 tiles, read
// once at half the size), prolongation fused with the Jacobi term and the r.z dot.  Everything is launched on the context stream without synchronisation.
#include <cub/cub.cuh>
#include <algorithm>
#include <cmath>
#include <vector>

#include "gf_internal.cuh"

namespace {

constexpr int kCT = 256;
constexpr int kMaxCoarse = 4096;
constexpr int kDefaultCoarse = 3072;

// Default coarse size: n / 128 within [192, 3072].  The set-up (the Gauss-Jordan sweep is
// O(nc^3)) costs ~10 ms at nc = 3072 whatever the mesh; measured on B200 with set-up
// and solve to 1e-8 together, n / 128 is the fastest of nc = 3072, n/16, n/32, n/64 and
// n/128 on Brick8 cubes of 15k-353k dofs and Q8 128^2 (e.g. 207k dofs: 7.5 ms against
// 14.3 ms at nc = 3072); from 393k dofs on the default is 3072.
inline int default_coarse(int n) { return std::min(kDefaultCoarse, std::max(192, n / 128)); }

struct Coarse {
  int64_t ver = -1;  // K64 version it was built for
  int dim = 0, nm = 0, na = 0, nc = 0;
  double s = 1.0;           // box side (rotation-mode scale)
  double lo[3] = {0, 0, 0};
  int nb[3] = {1, 1, 1};
  int32_t* node_agg = nullptr;   // [nnodes]
  int32_t* agg_off = nullptr;    // [na + 1]
  int32_t* agg_nodes = nullptr;  // [nnodes], nodes grouped by aggregate
  double* cen = nullptr;         // [na * dim]
  int nt = 0;                     // 64 x 64 tiles per side; rc, zc hold 64 nt entries
  int ntiles = 0;                 // nt (nt + 1) / 2 tiles (I <= J) of the symmetric inverse
  int2* tile_ij = nullptr;        // [ntiles] (I, J)
  double* ainv = nullptr;         // [ntiles][64][64], zero beyond nc
  unsigned* counter = nullptr;    // blocks done in the current coarse product
  double* rc = nullptr;          // [nc]
  double* zc = nullptr;          // [64 nt]
};

// P row of dof (node, comp c): modes m (translations first, then rotations) with the
// node's scaled offset d from its aggregate centroid.
//   2-D: t_x, t_y, rot_z = (-d_y, d_x)
//   3-D: t_x, t_y, t_z, rot_x = (0, -d_z, d_y), rot_y = (d_z, 0, -d_x), rot_z = (-d_y, d_x, 0)
template <int DIM>
__device__ inline void p_row(int c, const double* d, double (&row)[DIM == 2 ? 3 : 6]) {
  constexpr int NM = DIM == 2 ? 3 : 6;
#pragma unroll
  for (int m = 0; m < NM; ++m) row[m] = (m == c) ? 1.0 : 0.0;  // translations
  if (DIM == 2) {
    row[2] = c == 0 ? -d[1] : d[0];
  } else {
    if (c == 0) { row[4] = d[2]; row[5] = -d[1]; }
    if (c == 1) { row[3] = -d[2]; row[5] = d[0]; }
    if (c == 2) { row[3] = d[1]; row[4] = -d[0]; }
  }
}

// per-block min / max of each coordinate
__global__ void k_bbox(int nnodes, int dim, const double* __restrict__ x, double* __restrict__ out) {
  __shared__ double smin[3][kCT], smax[3][kCT];
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (int a = blockIdx.x * kCT + threadIdx.x; a < nnodes; a += gridDim.x * kCT)
    for (int c = 0; c < dim; ++c) {
      const double v = x[(int64_t)a * dim + c];
      mn[c] = fmin(mn[c], v);
      mx[c] = fmax(mx[c], v);
    }
  for (int c = 0; c < 3; ++c) { smin[c][threadIdx.x] = mn[c]; smax[c][threadIdx.x] = mx[c]; }
  __syncthreads();
  for (int o = kCT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int c = 0; c < 3; ++c) {
        smin[c][threadIdx.x] = fmin(smin[c][threadIdx.x], smin[c][threadIdx.x + o]);
        smax[c][threadIdx.x] = fmax(smax[c][threadIdx.x], smax[c][threadIdx.x + o]);
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < 3; ++c) {
      out[blockIdx.x * 6 + c] = smin[c][0];
      out[blockIdx.x * 6 + 3 + c] = smax[c][0];
    }
}

__device__ inline int box_of(const double* x, int dim, const double* lo, const double* ext,
                             const int* nb) {
  int key = 0, mul = 1;
  for (int c = 0; c < dim; ++c) {
    int b = ext[c] > 0.0 ? (int)floor((x[c] - lo[c]) / ext[c] * nb[c]) : 0;
    b = min(max(b, 0), nb[c] - 1);
    key += b * mul;
    mul *= nb[c];
  }
  return key;
}

struct BoxGrid {
  double lo[3], ext[3];
  int nb[3];
};

__global__ void k_box_flags(int nnodes, int dim, const double* __restrict__ x, BoxGrid g,
                            int32_t* __restrict__ key, int32_t* __restrict__ used) {
  const int a = blockIdx.x * kCT + threadIdx.x;
  if (a >= nnodes) return;
  const int k = box_of(x + (int64_t)a * dim, dim, g.lo, g.ext, g.nb);
  key[a] = k;
  used[k] = 1;
}

__global__ void k_node_agg(int nnodes, const int32_t* __restrict__ key,
                           const int32_t* __restrict__ box_id, int32_t* __restrict__ agg,
                           int32_t* __restrict__ cnt) {
  const int a = blockIdx.x * kCT + threadIdx.x;
  if (a >= nnodes) return;
  const int A = box_id[key[a]];
  agg[a] = A;
  atomicAdd(&cnt[A], 1);
}

__global__ void k_agg_sums(int nnodes, int dim, const int32_t* __restrict__ agg,
                           const double* __restrict__ x, int32_t* __restrict__ iota,
                           double* __restrict__ csum) {
  const int a = blockIdx.x * kCT + threadIdx.x;
  if (a >= nnodes) return;
  const int A = agg[a];
  iota[a] = a;
  for (int c = 0; c < dim; ++c) atomicAdd(&csum[(int64_t)A * dim + c], x[(int64_t)a * dim + c]);
}

__global__ void k_centroid(int na, int dim, const int32_t* __restrict__ off,
                           double* __restrict__ cen) {
  const int A = blockIdx.x * kCT + threadIdx.x;
  if (A >= na) return;
  const int c = off[A + 1] - off[A];
  for (int k = 0; k < dim; ++k) cen[(int64_t)A * dim + k] /= (double)max(c, 1);
}

// Row block A of Ac = P^T K P: blocks (A, y) over chunk y of kCMT * per nodes a of aggregate A
// and their ELL node blocks (a, b).  C = P_a^T K_ab P_b goes to registers when b lies in
// A (most pairs), else to a shared-memory table keyed by B = agg[b] (open addressing,
// atomicCAS insertion; a full table falls back to global atomics); each block adds its
// sums to rows A*NM .. A*NM+NM-1 of Ac once at the end.
constexpr int kCMT = 128;  // threads per block = nodes per chunk
constexpr int kTab = 64;   // neighbour-aggregate table slots (power of two)

__device__ inline int tab_slot(volatile int* ids, int B) {
  const int h = (B * 0x9E3779B1u) >> 26;  // 6 bits
  for (int k = 0; k < kTab; ++k) {
    const int s = (h + k) & (kTab - 1);
    const int cur = ids[s];
    if (cur == B) return s;
    if (cur == -1) {
      const int old = atomicCAS((int*)&ids[s], -1, B);
      if (old == -1 || old == B) return s;
    }
  }
  return -1;
}

template <int DIM>
__global__ void __launch_bounds__(kCMT)
k_coarse_rows(int n, const int32_t* __restrict__ rownnz, const int32_t* __restrict__ colidx,
              const double* __restrict__ K, const uint8_t* __restrict__ fixed,
              const int32_t* __restrict__ agg, const int32_t* __restrict__ off,
              const int32_t* __restrict__ nodes, const double* __restrict__ x,
              const double* __restrict__ cen, double sinv, int nc, int per,
              double* __restrict__ Ac) {
  constexpr int NM = DIM == 2 ? 3 : 6;
  constexpr int NMM = NM * NM;
  __shared__ int ids[kTab];
  __shared__ double tab[kTab][NMM];
  __shared__ double wsum[kCMT / 32][NMM];
  const int A = blockIdx.x;
  const int q0 = off[A] + blockIdx.y * kCMT * per;
  if (q0 >= off[A + 1]) return;  // block-uniform: this aggregate has fewer chunks
  for (int i = threadIdx.x; i < kTab; i += kCMT) ids[i] = -1;
  for (int i = threadIdx.x; i < kTab * NMM; i += kCMT) (&tab[0][0])[i] = 0.0;
  __syncthreads();
  double acc[NM][NM];
#pragma unroll
  for (int m = 0; m < NM; ++m)
#pragma unroll
    for (int m2 = 0; m2 < NM; ++m2) acc[m][m2] = 0.0;
  double cA[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) cA[c] = cen[(int64_t)A * DIM + c];
  for (int k = 0; k < per; ++k) {
    const int q = q0 + k * kCMT + threadIdx.x;
    if (q >= off[A + 1]) break;
    const int a = nodes[q];
    const int ra = a * DIM;
    double da[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) da[c] = (x[(int64_t)ra + c] - cA[c]) * sinv;
    double pa[DIM][NM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      p_row<DIM>(c, da, pa[c]);
      if (fixed[ra + c]) {
#pragma unroll
        for (int m = 0; m < NM; ++m) pa[c][m] = 0.0;
      }
    }
    // K_ab P_b summed over consecutive neighbours b of one aggregate (the columns are
    // sorted, so neighbours in one box come in runs); P_a^T times the sum is added once
    // per run: into registers for B = A, else into the table (or Ac)
    int curB = -1;
    double S[DIM][NM];
#pragma unroll
    for (int c = 0; c < DIM; ++c)
#pragma unroll
      for (int m = 0; m < NM; ++m) S[c][m] = 0.0;
    auto flush = [&](int Bx) {
      if (Bx == A) {
#pragma unroll
        for (int c = 0; c < DIM; ++c)
#pragma unroll
          for (int m = 0; m < NM; ++m)
#pragma unroll
            for (int m2 = 0; m2 < NM; ++m2) acc[m][m2] += pa[c][m] * S[c][m2];
      } else if (Bx >= 0) {
        const int sl = tab_slot(ids, Bx);
#pragma unroll
        for (int m = 0; m < NM; ++m) {
#pragma unroll
          for (int m2 = 0; m2 < NM; ++m2) {
            double v = 0.0;
#pragma unroll
            for (int c = 0; c < DIM; ++c) v += pa[c][m] * S[c][m2];
            if (v == 0.0) continue;
            if (sl >= 0) atomicAdd(&tab[sl][m * NM + m2], v);
            else atomicAdd(&Ac[(int64_t)(A * NM + m) * nc + Bx * NM + m2], v);
          }
        }
      }
    };
    const int nzb = rownnz[ra] / DIM;
    for (int p = 0; p < nzb; ++p) {
      const int b = colidx[(int64_t)(p * DIM) * n + ra] / DIM;
      const int B = agg[b];
      if (B != curB) {
        flush(curB);
        curB = B;
#pragma unroll
        for (int c = 0; c < DIM; ++c)
#pragma unroll
          for (int m = 0; m < NM; ++m) S[c][m] = 0.0;
      }
      double db[DIM];
#pragma unroll
      for (int c = 0; c < DIM; ++c)
        db[c] = (x[(int64_t)b * DIM + c] - cen[(int64_t)B * DIM + c]) * sinv;
      // S[c][m] += sum_c2 K_ab[c][c2] P_b[c2][m]
#pragma unroll
      for (int c2 = 0; c2 < DIM; ++c2) {
        if (fixed[b * DIM + c2]) continue;
        double pr[NM];
        p_row<DIM>(c2, db, pr);
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
          const double kv = K[(int64_t)(p * DIM + c2) * n + ra + c];
#pragma unroll
          for (int m = 0; m < NM; ++m) S[c][m] += kv * pr[m];
        }
      }
    }
    flush(curB);
  }
  // the (A, A) block: warp sums, then one pass over the warps' partials
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int m = 0; m < NM; ++m)
#pragma unroll
    for (int m2 = 0; m2 < NM; ++m2) {
      double v = acc[m][m2];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (l == 0) wsum[w][m * NM + m2] = v;
    }
  __syncthreads();
  for (int e = threadIdx.x; e < NMM; e += kCMT) {
    double v = 0.0;
    for (int k = 0; k < kCMT / 32; ++k) v += wsum[k][e];
    atomicAdd(&Ac[(int64_t)(A * NM + e / NM) * nc + A * NM + e % NM], v);
  }
  for (int e = threadIdx.x; e < kTab * NMM; e += kCMT) {
    const int sl = e / NMM, B = ids[sl];
    if (B < 0) continue;
    const int m = (e % NMM) / NM, m2 = e % NM;
    const double v = tab[sl][e % NMM];
    if (v != 0.0) atomicAdd(&Ac[(int64_t)(A * NM + m) * nc + B * NM + m2], v);
  }
}

// The same sums over the solver's node-block slices (mesh-built patterns): a thread per
// node slot walks its slice row like the SpMV, so the neighbour ids and the dim x dim value
// blocks are read coalesced.  What a neighbour b contributes besides its K block comes from
// one 32-byte record per node (k_node_records: scaled offset from its aggregate's centroid,
// aggregate id and fixed-dof bits).  S_b = K_ab P_b accumulates in registers for b in the
// node's own aggregate A; for other aggregates (nodes near box faces, at most a few) in
// kSellSlots per-thread shared-memory sums keyed by B, flushed as P_a^T S to Ac at the end
// (or when a further aggregate needs the slot).  The (A, A) blocks P_a^T S_A are summed over
// the warp's lanes of equal A by shuffles, one atomic per entry.
constexpr int kSellThreads = 128;
constexpr int kSellSlots = 3;

// rec[a] = {d_0, d_1, d_2 (scaled offset from the centroid of a's aggregate; 2-D: d_2 = 0),
//           agg[a] + 2^24 * (bit c: dof c of a fixed)}
__global__ void k_node_records(int nnodes, int dim, const double* __restrict__ x,
                               const int32_t* __restrict__ agg, const double* __restrict__ cen,
                               const uint8_t* __restrict__ fixed, double sinv,
                               double4* __restrict__ rec) {
  const int a = blockIdx.x * kCT + threadIdx.x;
  if (a >= nnodes) return;
  const int A = agg[a];
  double d[3] = {0.0, 0.0, 0.0};
  int fm = 0;
  for (int c = 0; c < dim; ++c) {
    d[c] = (x[(int64_t)a * dim + c] - cen[(int64_t)A * dim + c]) * sinv;
    if (fixed[(int64_t)a * dim + c]) fm |= 1 << c;
  }
  rec[a] = make_double4(d[0], d[1], d[2], (double)(A + (fm << 24)));
}

__device__ __forceinline__ double4 load_rec(const double4* __restrict__ rec, int b) {
  const double2* r = reinterpret_cast<const double2*>(rec + b);
  const double2 lo = __ldg(r), hi = __ldg(r + 1);
  return make_double4(lo.x, lo.y, hi.x, hi.y);
}

// Entry (c, m) of the P row of a dof with scaled offset d (the entries of p_row one at a
// time).
template <int DIM>
__device__ __forceinline__ double p_entry(int c, int m, const double* d) {
  if (m < DIM) return m == c ? 1.0 : 0.0;
  if (DIM == 2) return c == 0 ? -d[1] : d[0];
  if (m == 3) return c == 1 ? -d[2] : c == 2 ? d[1] : 0.0;
  if (m == 4) return c == 0 ? d[2] : c == 2 ? -d[0] : 0.0;
  return c == 0 ? -d[1] : c == 1 ? d[0] : 0.0;
}

template <int DIM>
constexpr size_t sell_coarse_smem() {
  return (size_t)kSellSlots * DIM * (DIM == 2 ? 3 : 6) * kSellThreads * sizeof(double);
}

template <int DIM>
__global__ void __launch_bounds__(kSellThreads)
k_coarse_rows_sell(int nnodes, const int64_t* __restrict__ off, const int32_t* __restrict__ width,
                   const int32_t* __restrict__ bcol, const int32_t* __restrict__ perm,
                   const double* __restrict__ val, const double4* __restrict__ rec, int nc,
                   double* __restrict__ Ac) {
  constexpr unsigned kFull = 0xffffffffu;
  constexpr int NM = DIM == 2 ? 3 : 6;
  constexpr int NMM = NM * NM;
  constexpr int NS = DIM * NM;   // entries of a sum S (row c, mode m at c * NM + m)
  extern __shared__ __align__(16) double csm[];   // [kSellSlots][NS][kSellThreads]
  const int tid = threadIdx.x, lane = tid & 31;
  const int t = blockIdx.x * kSellThreads + tid;   // node slot
  const bool live = t < nnodes;
  const int a = live ? perm[t] : 0;
  const double4 ra = load_rec(rec, a);
  const int A = ((int)ra.w) & 0xffffff, fa = ((int)ra.w) >> 24;
  double da[DIM];
  da[0] = ra.x;
  da[1] = ra.y;
  if constexpr (DIM == 3) da[DIM - 1] = ra.z;
  auto slot = [&](int sl, int k) -> double& { return csm[((size_t)sl * NS + k) * kSellThreads + tid]; };
  int key[kSellSlots];
#pragma unroll
  for (int i = 0; i < kSellSlots; ++i) key[i] = -1;
  // P_a^T S of slot sl added to block (A, B) of Ac
  auto flush = [&](int sl, int B) {
#pragma unroll
    for (int m = 0; m < NM; ++m)
#pragma unroll
      for (int m2 = 0; m2 < NM; ++m2) {
        double v = 0.0;
#pragma unroll
        for (int c = 0; c < DIM; ++c)
          if (!((fa >> c) & 1)) v += p_entry<DIM>(c, m, da) * slot(sl, c * NM + m2);
        if (v != 0.0) atomicAdd(&Ac[(int64_t)(A * NM + m) * nc + B * NM + m2], v);
      }
  };
  double Sacc[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) Sacc[k] = 0.0;
  if (live) {
    const int k = t >> 5;
    const int64_t o = off[k];
    const int w = width[k];
    const int32_t* bc = bcol + o + lane;
    const double* vb = val + o * DIM * DIM + lane;
    for (int p = 0; p < w; ++p) {
      const int b = __ldg(bc + 32 * p);
      double kv[DIM][DIM];
#pragma unroll
      for (int c = 0; c < DIM; ++c)
#pragma unroll
        for (int c2 = 0; c2 < DIM; ++c2)
          kv[c][c2] = __ldg(vb + (int64_t)((p * DIM + c) * DIM + c2) * 32);
      const double4 rb = load_rec(rec, b);
      const int wb = (int)rb.w;
      const int B = wb & 0xffffff, fb = wb >> 24;
      double db[DIM];
      db[0] = rb.x;
      db[1] = rb.y;
      if constexpr (DIM == 3) db[DIM - 1] = rb.z;
      if (B == A) {
#pragma unroll
        for (int c2 = 0; c2 < DIM; ++c2) {
          if ((fb >> c2) & 1) continue;
#pragma unroll
          for (int c = 0; c < DIM; ++c)
#pragma unroll
            for (int m = 0; m < NM; ++m) Sacc[c * NM + m] += kv[c][c2] * p_entry<DIM>(c2, m, db);
        }
      } else {
        // the slot of B: an existing one, a free one, or slot 0 after flushing it
        int sl = -1;
#pragma unroll
        for (int i = 0; i < kSellSlots; ++i)
          if (sl < 0 && key[i] == B) sl = i;
        if (sl < 0) {
#pragma unroll
          for (int i = 0; i < kSellSlots; ++i)
            if (sl < 0 && key[i] < 0) sl = i;
          if (sl < 0) {
            flush(0, key[0]);
            sl = 0;
          }
          key[sl] = B;
#pragma unroll
          for (int q = 0; q < NS; ++q) slot(sl, q) = 0.0;
        }
#pragma unroll
        for (int c = 0; c < DIM; ++c)
#pragma unroll
          for (int m = 0; m < NM; ++m) {
            double v = 0.0;
#pragma unroll
            for (int c2 = 0; c2 < DIM; ++c2)
              if (!((fb >> c2) & 1)) v += kv[c][c2] * p_entry<DIM>(c2, m, db);
            slot(sl, c * NM + m) += v;
          }
      }
    }
#pragma unroll
    for (int i = 0; i < kSellSlots; ++i)
      if (key[i] >= 0) flush(i, key[i]);
  }
  // (A, A): P_a^T S_A summed over the lanes of equal A
  unsigned pending = __ballot_sync(kFull, live);
  while (pending) {
    const int src = __ffs(pending) - 1;
    const int Al = __shfl_sync(kFull, A, src);
    const bool sel = live && A == Al;
    pending &= ~__ballot_sync(kFull, sel);
#pragma unroll
    for (int m = 0; m < NM; ++m)
#pragma unroll
      for (int m2 = 0; m2 < NM; ++m2) {
        double v = 0.0;
        if (sel) {
#pragma unroll
          for (int c = 0; c < DIM; ++c)
            if (!((fa >> c) & 1)) v += p_entry<DIM>(c, m, da) * Sacc[c * NM + m2];
        }
#pragma unroll
        for (int o2 = 16; o2 > 0; o2 >>= 1) v += __shfl_xor_sync(kFull, v, o2);
        if (lane == src) atomicAdd(&Ac[(int64_t)(Al * NM + m) * nc + Al * NM + m2], v);
      }
  }
}

__global__ void k_diag_max(int nc, const double* __restrict__ Ac, double* __restrict__ out) {
  __shared__ double sh[kCT];
  double m = 0.0;
  for (int i = threadIdx.x; i < nc; i += kCT) m = fmax(m, Ac[(int64_t)i * nc + i]);
  sh[threadIdx.x] = m;
  __syncthreads();
  for (int o = kCT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

// regularise: Ac_ii += eps * max diag; an empty mode (zero diagonal) becomes 1
__global__ void k_regularise(int nc, const double* __restrict__ dmax, double eps,
                             double* __restrict__ Ac) {
  const int i = blockIdx.x * kCT + threadIdx.x;
  if (i >= nc) return;
  double& d = Ac[(int64_t)i * nc + i];
  d = d > 0.0 ? d + eps * (*dmax) : 1.0;
}

// Blocked Gauss-Jordan sweep (in place, SPD: no pivoting).  For the pivot block P of
// kGJ rows/columns at kb and the rest R:
//   A_PP <- A_PP^-1,  A_PR <- A_PP^-1 A_PR,  A_RP <- -A_RP A_PP^-1,
//   A_RR <- A_RR - A_RP A_PP^-1 A_PR
// After a sweep over every block A holds its inverse.  Three kernels per block:
// the pivot block's inverse (one CTA), the two panels, and the rank-kGJ update; the
// panels and the update are 64 x 64 output tiles of 64-deep products (4 x 4 outputs per
// thread from shared-memory operands), so every pass over A does 64 FMAs per entry.
constexpr int kGJ = 64;
constexpr int kGT = 64;                 // output tile side
constexpr int kGJRows = 16;             // pivot CTA: kGJ x kGJRows threads, 4 rows each
constexpr size_t kGJSmem = sizeof(double) * ((size_t)kGT * (kGJ + 1) + (size_t)kGJ * kGT);

// Pi = A_PP^-1 by scalar sweeps in shared memory (bs <= kGJ)
__global__ void __launch_bounds__(kGJ * kGJRows)
k_gj_pivot(int nc, int kb, int bs, const double* __restrict__ A, double* __restrict__ Pi) {
  __shared__ double M[kGJ][kGJ + 1];
  __shared__ double row[kGJ], col[kGJ], piv;
  const int j = threadIdx.x, i0 = threadIdx.y;
  for (int i = i0; i < kGJ; i += kGJRows)
    M[i][j] = (i < bs && j < bs) ? A[(int64_t)(kb + i) * nc + kb + j] : 0.0;
  __syncthreads();
  for (int k = 0; k < bs; ++k) {
    if (i0 == 0) row[j] = M[k][j];
    if (i0 == 1) col[j] = M[j][k];
    if (i0 == 2 && j == 0) piv = 1.0 / M[k][k];   // one division per step
    __syncthreads();
    const double p = piv;
    if (j < bs)
      for (int i = i0; i < bs; i += kGJRows) {
        double v;
        if (i == k && j == k) v = p;
        else if (i == k) v = row[j] * p;
        else if (j == k) v = -col[i] * p;
        else v = M[i][j] - col[i] * row[j] * p;
        M[i][j] = v;
      }
    __syncthreads();
  }
  for (int i = i0; i < kGJ; i += kGJRows) Pi[i * kGJ + j] = M[i][j];
}

// acc[a][b] = sum_u X[ty + 16a][u] Y[u][tx + 16b] over u < kGJ (X rows padded to kGJ + 1)
__device__ __forceinline__ void gj_tile_product(const double (*X)[kGJ + 1],
                                                const double (*Y)[kGT], double (&acc)[4][4]) {
  const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
#pragma unroll 8
  for (int u = 0; u < kGJ; ++u) {
    double cv[4], rv[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) cv[a] = X[ty + 16 * a][u];
#pragma unroll
    for (int b = 0; b < 4; ++b) rv[b] = Y[u][tx + 16 * b];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] += cv[a] * rv[b];
  }
}

// blockIdx.y = 0: row panel Rw[r][j] = sum_u Pi[r][u] A[kb+u][j] for the 64 columns j0..
// blockIdx.y = 1: column panel Cold[i][t] = A[i][kb+t], Cn[i][t] = -sum_u A[i][kb+u] Pi[u][t]
__global__ void __launch_bounds__(256)
k_gj_panels(int nc, int kb, int bs, const double* __restrict__ A, const double* __restrict__ Pi,
            double* __restrict__ Rw, double* __restrict__ Cold, double* __restrict__ Cn) {
  extern __shared__ __align__(16) double gsm[];
  double (*X)[kGJ + 1] = reinterpret_cast<double (*)[kGJ + 1]>(gsm);
  double (*Y)[kGT] = reinterpret_cast<double (*)[kGT]>(gsm + kGT * (kGJ + 1));
  const int t0 = blockIdx.x * kGT;
  const bool rowp = blockIdx.y == 0;
  for (int e = threadIdx.x; e < kGT * kGJ; e += 256) {
    const int r = e / kGJ, u = e % kGJ;      // X[r][u]
    const int u2 = e / kGT, c2 = e % kGT;    // Y[u2][c2]
    if (rowp) {
      X[r][u] = Pi[r * kGJ + u];
      Y[u2][c2] = (u2 < bs && t0 + c2 < nc) ? A[(int64_t)(kb + u2) * nc + t0 + c2] : 0.0;
    } else {
      X[r][u] = (u < bs && t0 + r < nc) ? A[(int64_t)(t0 + r) * nc + kb + u] : 0.0;
      Y[u2][c2] = Pi[u2 * kGJ + c2];
    }
  }
  __syncthreads();
  double acc[4][4];
  gj_tile_product(X, Y, acc);
  const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int r = ty + 16 * a, c = tx + 16 * b;
      if (rowp) {
        if (r < bs && t0 + c < nc) Rw[(int64_t)r * nc + t0 + c] = acc[a][b];
      } else if (t0 + r < nc && c < bs) {
        Cold[(int64_t)(t0 + r) * kGJ + c] = X[r][c];
        Cn[(int64_t)(t0 + r) * kGJ + c] = -acc[a][b];
      }
    }
}

// Every entry (i, j): a 64 x 64 tile per CTA of four warps, each warp a 32 x 32 quarter
// as 4 x 4 fragments of the FP64 tensor-core product mma.m8n8k4 (per lane: one A value
// A[g][t], one B value B[t][g], two accumulators D[g][2t], D[g][2t + 1] with g = lane / 4,
// t = lane % 4).  The Cold rows and Rw columns of the tile sit in shared memory with rows
// of kGJ + 4 doubles (the fragment loads of a warp fall on distinct bank pairs).
constexpr int kGU = kGJ + 4;   // shared row length (doubles) of the update's operand tiles
constexpr size_t kGJUpdateSmem = sizeof(double) * 2 * (size_t)kGT * kGU;

__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(128)
k_gj_update(int nc, int kb, int bs, double* __restrict__ A, const double* __restrict__ Pi,
            const double* __restrict__ Rw, const double* __restrict__ Cold,
            const double* __restrict__ Cn) {
  extern __shared__ __align__(16) double gsm[];
  double (*sC)[kGU] = reinterpret_cast<double (*)[kGU]>(gsm);               // [row][u]
  double (*sR)[kGU] = reinterpret_cast<double (*)[kGU]>(gsm + kGT * kGU);   // [u][col]
  const int i0 = blockIdx.y * kGT, j0 = blockIdx.x * kGT;
  const int tid = threadIdx.x;
  if (bs == kGJ && i0 + kGT <= nc && j0 + kGT <= nc && (nc & 1) == 0) {
    // full interior tile, rows of Rw 16-byte aligned: 16-byte loads, all in flight at once
    constexpr int P = kGT * kGJ / 2 / 128;   // double pairs per thread and operand
    double2 c[P], r[P];
#pragma unroll
    for (int k = 0; k < P; ++k) {
      const int e = tid + 128 * k;            // pair index: row e / 32, pair e % 32
      c[k] = __ldcg(reinterpret_cast<const double2*>(Cold + (int64_t)(i0 + e / 32) * kGJ) + e % 32);
      r[k] = __ldcg(reinterpret_cast<const double2*>(Rw + (int64_t)(e / 32) * nc + j0) + e % 32);
    }
#pragma unroll
    for (int k = 0; k < P; ++k) {
      const int e = tid + 128 * k;
      sC[e / 32][2 * (e % 32)] = c[k].x;
      sC[e / 32][2 * (e % 32) + 1] = c[k].y;
      sR[e / 32][2 * (e % 32)] = r[k].x;
      sR[e / 32][2 * (e % 32) + 1] = r[k].y;
    }
  } else {
    for (int e = tid; e < kGT * kGJ; e += 128) {
      const int r = e / kGJ, u = e % kGJ;
      sC[r][u] = (i0 + r < nc && u < bs) ? Cold[(int64_t)(i0 + r) * kGJ + u] : 0.0;
      const int u2 = e / kGT, c2 = e % kGT;
      sR[u2][c2] = (j0 + c2 < nc && u2 < bs) ? Rw[(int64_t)u2 * nc + j0 + c2] : 0.0;
    }
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
  double acc[4][4][2];
#pragma unroll
  for (int fm = 0; fm < 4; ++fm)
#pragma unroll
    for (int fn = 0; fn < 4; ++fn) acc[fm][fn][0] = acc[fm][fn][1] = 0.0;
#pragma unroll 4
  for (int k0 = 0; k0 < kGJ; k0 += 4) {
    double a[4], b[4];
#pragma unroll
    for (int fm = 0; fm < 4; ++fm) a[fm] = sC[wr + fm * 8 + g][k0 + t4];
#pragma unroll
    for (int fn = 0; fn < 4; ++fn) b[fn] = sR[k0 + t4][wc + fn * 8 + g];
#pragma unroll
    for (int fm = 0; fm < 4; ++fm)
#pragma unroll
      for (int fn = 0; fn < 4; ++fn) dmma_m8n8k4(acc[fm][fn][0], acc[fm][fn][1], a[fm], b[fn]);
  }
  const bool plain = i0 + kGT <= nc && j0 + kGT <= nc && (nc & 1) == 0 &&
                     (kb + bs <= i0 || kb >= i0 + kGT) && (kb + bs <= j0 || kb >= j0 + kGT);
  if (plain) {
    // no pivot row or column in the tile: 16-byte read-modify-writes of the entry pairs
#pragma unroll
    for (int fm = 0; fm < 4; ++fm) {
      double2* row = reinterpret_cast<double2*>(A + (int64_t)(i0 + wr + fm * 8 + g) * nc + j0 + wc);
#pragma unroll
      for (int fn = 0; fn < 4; ++fn) {
        double2 v = row[fn * 4 + t4];
        v.x -= acc[fm][fn][0];
        v.y -= acc[fm][fn][1];
        row[fn * 4 + t4] = v;
      }
    }
    return;
  }
#pragma unroll
  for (int fm = 0; fm < 4; ++fm) {
    const int i = i0 + wr + fm * 8 + g;
    if (i >= nc) continue;
    const bool ip = i >= kb && i < kb + bs;
#pragma unroll
    for (int fn = 0; fn < 4; ++fn)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int j = j0 + wc + fn * 8 + 2 * t4 + h;
        if (j >= nc) continue;
        const bool jp = j >= kb && j < kb + bs;
        double* dst = A + (int64_t)i * nc + j;
        if (ip && jp) *dst = Pi[(i - kb) * kGJ + (j - kb)];
        else if (ip) *dst = Rw[(int64_t)(i - kb) * nc + j];
        else if (jp) *dst = Cn[(int64_t)i * kGJ + (j - kb)];
        else *dst -= acc[fm][fn][h];
      }
  }
}

// Upper-triangle tiles (I <= J) of the symmetrised inverse, zero beyond nc.
constexpr int kTS = 64;
__global__ void k_pack_tiles(int nc, const int2* __restrict__ ij, const double* __restrict__ A,
                             double* __restrict__ T) {
  const int2 t = ij[blockIdx.x];
  double* dst = T + (int64_t)blockIdx.x * kTS * kTS;
  for (int e = threadIdx.x; e < kTS * kTS; e += blockDim.x) {
    const int gi = t.x * kTS + e / kTS, gj = t.y * kTS + e % kTS;
    dst[e] = (gi < nc && gj < nc)
                 ? 0.5 * (A[(int64_t)gi * nc + gj] + A[(int64_t)gj * nc + gi])
                 : 0.0;
  }
}

// rc = P^T r (and zc = 0 for the coarse product): block per aggregate over its node list
constexpr int kRT = 256;
template <int DIM, typename V>
__global__ void __launch_bounds__(kRT)
k_restrict(const int32_t* __restrict__ off, const int32_t* __restrict__ nodes,
           const double* __restrict__ x, const double* __restrict__ cen, double sinv,
           const uint8_t* __restrict__ fixed, const V* __restrict__ r,
           double* __restrict__ rc, double* __restrict__ zc, const int* __restrict__ done) {
  constexpr int NM = DIM == 2 ? 3 : 6;
  __shared__ double ws[kRT / 32][NM];
  if (done && *done) return;
  const int A = blockIdx.x;
  double acc[NM];
#pragma unroll
  for (int m = 0; m < NM; ++m) acc[m] = 0.0;
  double cA[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) cA[c] = cen[(int64_t)A * DIM + c];
  for (int q = off[A] + threadIdx.x; q < off[A + 1]; q += kRT) {
    const int a = nodes[q];
    double d[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) d[c] = (x[(int64_t)a * DIM + c] - cA[c]) * sinv;
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      if (fixed[a * DIM + c]) continue;
      const double rv = (double)r[a * DIM + c];
      double pr[NM];
      p_row<DIM>(c, d, pr);
#pragma unroll
      for (int m = 0; m < NM; ++m) acc[m] += pr[m] * rv;
    }
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int m = 0; m < NM; ++m) {
    double v = acc[m];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (l == 0) ws[w][m] = v;
  }
  __syncthreads();
  if (threadIdx.x < NM) {
    double v = 0.0;
    for (int k = 0; k < kRT / 32; ++k) v += ws[k][threadIdx.x];
    rc[A * NM + threadIdx.x] = v;
    zc[A * NM + threadIdx.x] = 0.0;  // the coarse product accumulates into zc
  }
}

// zc += Ainv rc from the packed upper-triangle tiles: block per tile (I, J) adds A_IJ rc_J
// to zc_I and, off the diagonal, A_IJ^T rc_I to zc_J (double atomics; zc is zeroed by the
// restriction), so the symmetric inverse is read once at half its size.  Warp w reads
// rows 8w .. 8w+7 of the tile as 16-byte pairs, one contiguous 512-byte row per load
// (lane l: columns 2l, 2l+1).  Row sums: a butterfly that halves the 8 partial sums per
// step (9 shuffles); column sums: per thread over its 8 rows, then over the warps in
// shared memory.  With sc: the last block to finish (counter, after a fence) adds
// rc.zc to sc->rzn and resets the counter.
__global__ void __launch_bounds__(256)
k_coarse_symv(int nc, const int2* __restrict__ ij, const double* __restrict__ T,
              const double* __restrict__ rc, double* __restrict__ zc, unsigned* counter,
              SolveScalars* sc, const int* __restrict__ done) {
  __shared__ double xI[kTS], xJ[kTS], colp[8][kTS], red[8];
  __shared__ bool last;
  if (done && *done) return;
  const int2 t = ij[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (tid < kTS) xI[tid] = rc[t.x * kTS + tid];
  else if (tid < 2 * kTS) xJ[tid - kTS] = rc[t.y * kTS + tid - kTS];
  __syncthreads();
  const double2* base =
      reinterpret_cast<const double2*>(T + (int64_t)blockIdx.x * kTS * kTS + w * 8 * kTS);
  double2 a[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) a[c] = __ldcs(base + c * 32 + lane);
  const double x0 = xJ[2 * lane], x1 = xJ[2 * lane + 1];
  double rs[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) rs[c] = a[c].x * x0 + a[c].y * x1;
  const bool u16 = lane & 16, u8 = lane & 8, u4 = lane & 4;
  double v4[4], v2[2];
#pragma unroll
  for (int k = 0; k < 4; ++k)
    v4[k] = (u16 ? rs[4 + k] : rs[k]) + __shfl_xor_sync(0xffffffffu, u16 ? rs[k] : rs[4 + k], 16);
#pragma unroll
  for (int k = 0; k < 2; ++k)
    v2[k] = (u8 ? v4[2 + k] : v4[k]) + __shfl_xor_sync(0xffffffffu, u8 ? v4[k] : v4[2 + k], 8);
  double v = (u4 ? v2[1] : v2[0]) + __shfl_xor_sync(0xffffffffu, u4 ? v2[0] : v2[1], 4);
  v += __shfl_xor_sync(0xffffffffu, v, 2);
  v += __shfl_xor_sync(0xffffffffu, v, 1);
  if ((lane & 3) == 0) atomicAdd(&zc[t.x * kTS + w * 8 + (lane >> 2)], v);
  if (t.x != t.y) {
    double cx = 0.0, cy = 0.0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const double xi = xI[w * 8 + c];
      cx += a[c].x * xi;
      cy += a[c].y * xi;
    }
    colp[w][2 * lane] = cx;
    colp[w][2 * lane + 1] = cy;
    __syncthreads();
    if (tid < kTS) {
      double u = 0.0;
#pragma unroll
      for (int q = 0; q < 8; ++q) u += colp[q][tid];
      atomicAdd(&zc[t.y * kTS + tid], u);
    }
  }
  if (!sc) return;
  __threadfence();
  __syncthreads();
  if (tid == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  double part = 0.0;
  for (int j = tid; j < nc; j += blockDim.x) part += rc[j] * __ldcg(zc + j);
  for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
  if (lane == 0) red[w] = part;
  __syncthreads();
  if (tid == 0) {
    double u = 0.0;
    for (int q = 0; q < 8; ++q) u += red[q];
    atomicAdd(&sc->rzn, u);
    *counter = 0u;
  }
}

__device__ inline double cg_block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  }
  return s;
}

// z = dinv r + P zc, and rz_acc += r.z (grid-stride over dofs)
template <int DIM>
__global__ void __launch_bounds__(kCT)
k_prolong(int n, const int32_t* __restrict__ agg, const double* __restrict__ x,
          const double* __restrict__ cen, double sinv, const uint8_t* __restrict__ fixed,
          const double* __restrict__ dinv, const double* __restrict__ r,
          const double* __restrict__ zc, double* __restrict__ z, double* __restrict__ rz_acc,
          const int* __restrict__ done, int add) {
  constexpr int NM = DIM == 2 ? 3 : 6;
  __shared__ double sh[32];
  if (done && *done) return;
  double rz = 0.0;
  for (int i = blockIdx.x * kCT + threadIdx.x; i < n; i += gridDim.x * kCT) {
    const int a = i / DIM, c = i - a * DIM;
    double zi = add ? z[i] : dinv ? dinv[i] * r[i] : 0.0;
    if (!fixed[i]) {
      const int A = agg[a];
      double d[DIM];
#pragma unroll
      for (int k = 0; k < DIM; ++k) d[k] = (x[(int64_t)a * DIM + k] - cen[(int64_t)A * DIM + k]) * sinv;
      double pr[NM];
      p_row<DIM>(c, d, pr);
#pragma unroll
      for (int m = 0; m < NM; ++m) zi += pr[m] * zc[A * NM + m];
    }
    z[i] = zi;
    rz += r[i] * zi;
  }
  if (!rz_acc) return;
  const double s = cg_block_sum(rz, sh);
  if (threadIdx.x == 0) atomicAdd(rz_acc, s);
}

// ---- fused two-level PCG steps ---------------------------------------------------
// The direction kernel forms z = D^-1 r + P zc on the fly, using
//   r.z = r.D^-1 r + (P^T r).zc = r.D^-1 r + rc.zc,
// so z is never stored: r.D^-1 r comes with the x/r update, rc.zc with the coarse
// product.  (Folding the restriction into the update as well, with warp-aggregated
// atomics per aggregate, measured slower than the block-per-aggregate kernel: the
// shuffles cost more than the second read of r.)

// INIT: x = 0, r = scale * b.  Else: alpha = rz / p.q, x += alpha p, r -= alpha q.
// Accumulates rr = r.r and rzn += r.D^-1 r (in FP64 whatever the vector type V).
template <bool INIT, typename V>
__global__ void __launch_bounds__(kCT)
k_tl_update(int n, const double* __restrict__ b, const V* __restrict__ q, double scale,
            V* __restrict__ x, V* __restrict__ r, const V* __restrict__ p,
            const V* __restrict__ dinv, SolveScalars* sc) {
  __shared__ double sh[32];
  double alpha = 0.0;
  if (!INIT) {
    if (sc->done) return;
    const double pq = sc->pq;
    if (!(pq > 0.0) || !isfinite(pq)) {
      if (blockIdx.x == 0 && threadIdx.x == 0) sc->done = 2;
      return;
    }
    alpha = sc->rz / pq;
  }
  double rr = 0.0, rdr = 0.0;
  for (int i = blockIdx.x * kCT + threadIdx.x; i < n; i += gridDim.x * kCT) {
    V ri;
    if (INIT) {
      ri = (V)(b[i] * scale);
      x[i] = V(0);
    } else {
      x[i] += (V)alpha * p[i];
      ri = r[i] - (V)alpha * q[i];
    }
    r[i] = ri;
    const double rd = (double)ri;
    rr += rd * rd;
    rdr += rd * rd * (double)dinv[i];
  }
  const double s1 = cg_block_sum(rr, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->rr, s1);
  const double s2 = cg_block_sum(rdr, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->rzn, s2);
}

// z = D^-1 r + P zc on the fly.  MODE kTlFirst: p = z; kTlKeep: p = pscale p (a
// reliable update that keeps the direction); kTlStep: p = z + beta p with
// beta = rzn / rz, then the iteration count and the convergence test.  p32 (or null)
// receives an FP32 copy of p for SpMVs on the FP32 matrix.
constexpr int kTlFirst = 0, kTlKeep = 1, kTlStep = 2;
template <int DIM, int MODE, typename V>
__global__ void __launch_bounds__(kCT)
k_tl_direction(int n, const V* __restrict__ r, const V* __restrict__ dinv,
               const uint8_t* __restrict__ fixed, const int32_t* __restrict__ agg,
               const double* __restrict__ xc, const double* __restrict__ cen, double sinv,
               const double* __restrict__ zc, V* __restrict__ p, float* __restrict__ p32,
               double pscale, SolveScalars* sc) {
  constexpr int NM = DIM == 2 ? 3 : 6;
  if (sc->done) return;
  if (MODE == kTlKeep) {
    for (int64_t t = (int64_t)blockIdx.x * kCT + threadIdx.x; t < n; t += (int64_t)gridDim.x * kCT) {
      const V pn = (V)((double)p[t] * pscale);
      p[t] = pn;
      if (p32) p32[t] = (float)pn;
    }
    return;
  }
  const double beta = MODE == kTlFirst ? 0.0 : sc->rzn / sc->rz;
  const int64_t stride = (int64_t)gridDim.x * kCT;
  for (int64_t t = (int64_t)blockIdx.x * kCT + threadIdx.x; t < n; t += stride) {
    const int i = (int)t;
    double zi = (double)dinv[i] * (double)r[i];
    if (!fixed[i]) {
      const int a = i / DIM, c = i - a * DIM;
      const int A = agg[a];
      double d[DIM];
#pragma unroll
      for (int k = 0; k < DIM; ++k)
        d[k] = (xc[(int64_t)a * DIM + k] - cen[(int64_t)A * DIM + k]) * sinv;
      double pr[NM];
      p_row<DIM>(c, d, pr);
#pragma unroll
      for (int m = 0; m < NM; ++m) zi += pr[m] * zc[A * NM + m];
    }
    const V pn = (V)(MODE == kTlFirst ? zi : zi + beta * (double)p[i]);
    p[i] = pn;
    if (p32) p32[i] = (float)pn;
  }
  if (MODE == kTlStep && blockIdx.x == 0 && threadIdx.x == 0) {
    sc->pq = 0.0;
    sc->iter += 1;
    if (sc->rr <= sc->tol2) sc->done = 1;
    else if (sc->iter >= sc->maxit) sc->done = 3;
  }
}

void coarse_release(gf_ctx* ctx, Coarse* c) {
  gf_pfree(ctx, c->node_agg);
  gf_pfree(ctx, c->agg_off);
  gf_pfree(ctx, c->agg_nodes);
  gf_pfree(ctx, c->cen);
  gf_pfree(ctx, c->ainv);
  gf_pfree(ctx, c->tile_ij);
  gf_pfree(ctx, c->counter);
  gf_pfree(ctx, c->rc);
  gf_pfree(ctx, c->zc);
}

gf_status build(gf_ctx* ctx, Coarse* C, int target) {
  const int dim = ctx->dim, nnodes = ctx->nnodes, n = ctx->n;
  cudaStream_t s = ctx->stream;
  const int nm = dim == 2 ? 3 : 6;
  gf_status st;
  // bounding box
  const int bb = std::min(gf_blocks(nnodes, kCT), 256);
  double* d_bb = nullptr;
  if ((st = gf_palloc(ctx, &d_bb, (size_t)bb * 6)) != GF_OK) return st;
  k_bbox<<<bb, kCT, 0, s>>>(nnodes, dim, ctx->d_coords64, d_bb);
  std::vector<double> hb((size_t)bb * 6);
  GF_CUDA(ctx, cudaMemcpyAsync(hb.data(), d_bb, sizeof(double) * bb * 6, cudaMemcpyDeviceToHost, s));
  GF_CUDA(ctx, cudaStreamSynchronize(s));
  gf_pfree(ctx, d_bb);
  BoxGrid g{};
  double vol = 1.0;
  int dpos = 0;  // axes of positive extent
  for (int c = 0; c < dim; ++c) {
    double lo = 1e300, hi = -1e300;
    for (int k = 0; k < bb; ++k) {
      lo = std::min(lo, hb[k * 6 + c]);
      hi = std::max(hi, hb[k * 6 + 3 + c]);
    }
    g.lo[c] = lo;
    g.ext[c] = hi - lo;
    if (hi > lo) { vol *= hi - lo; ++dpos; }
  }
  // box side for about cap / nm aggregates over the axes of positive extent; grow it
  // until the grid fits the cap (at the latest when every axis has one box)
  const int cap = std::min(std::max(target, nm), kMaxCoarse);
  double side = dpos ? std::pow(vol / std::max(1.0, (double)cap / nm), 1.0 / dpos) : 1.0;
  int64_t nbox = 1;
  for (int it = 0; it < 100000; ++it) {
    nbox = 1;
    for (int c = 0; c < dim; ++c) {
      const double q = g.ext[c] / side;
      g.nb[c] = q >= (double)cap ? cap : std::max(1, (int)std::lround(q));
      nbox *= g.nb[c];
    }
    if (nbox * nm <= cap) break;
    side *= 1.05;
  }
  for (int c = dim; c < 3; ++c) { g.nb[c] = 1; g.lo[c] = 0; g.ext[c] = 0; }
  // aggregates = occupied boxes, numbered in box order
  int32_t *d_key = nullptr, *d_used = nullptr, *d_id = nullptr, *d_cnt = nullptr;
  char* d_tmp = nullptr;  // cub scratch, grown on demand
  size_t tb = 0;
  auto cleanup = [&]() {
    gf_pfree(ctx, d_key); gf_pfree(ctx, d_used); gf_pfree(ctx, d_id); gf_pfree(ctx, d_cnt);
    gf_pfree(ctx, d_tmp);
  };
  auto ensure_tmp = [&](size_t need) -> gf_status {
    if (need <= tb) return GF_OK;
    tb = need;
    return gf_palloc(ctx, &d_tmp, need);
  };
  if ((st = gf_palloc(ctx, &d_key, (size_t)nnodes)) != GF_OK ||
      (st = gf_palloc(ctx, &d_used, (size_t)nbox + 1)) != GF_OK ||
      (st = gf_palloc(ctx, &d_id, (size_t)nbox + 1)) != GF_OK) {
    cleanup();
    return st;
  }
  cudaMemsetAsync(d_used, 0, sizeof(int32_t) * (nbox + 1), s);
  k_box_flags<<<gf_blocks(nnodes, kCT), kCT, 0, s>>>(nnodes, dim, ctx->d_coords64, g, d_key, d_used);
  size_t tb1 = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb1, d_used, d_id, (int)nbox + 1, s);
  if ((st = ensure_tmp(tb1)) != GF_OK) {
    cleanup();
    return st;
  }
  cub::DeviceScan::ExclusiveSum(d_tmp, tb1, d_used, d_id, (int)nbox + 1, s);
  int32_t na = 0;
  GF_CUDA(ctx, cudaMemcpyAsync(&na, d_id + nbox, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  GF_CUDA(ctx, cudaStreamSynchronize(s));
  const int nc = na * nm;
  const int nt = (nc + kTS - 1) / kTS, ntiles = nt * (nt + 1) / 2;
  const int ld = nt * kTS;  // length of rc, zc
  C->nt = nt;
  C->ntiles = ntiles;
  C->dim = dim; C->nm = nm; C->na = na; C->nc = nc; C->s = side;
  for (int c = 0; c < 3; ++c) { C->lo[c] = g.lo[c]; C->nb[c] = g.nb[c]; }
  double* d_Ac = nullptr;
  double *d_pi = nullptr, *d_rw = nullptr, *d_cold = nullptr, *d_cn = nullptr,
         *d_dmax = nullptr;
  double4* d_rec = nullptr;   // per-node records of the slice coarse kernel
  auto cleanup2 = [&]() {
    cleanup();
    gf_pfree(ctx, d_Ac); gf_pfree(ctx, d_pi); gf_pfree(ctx, d_rw); gf_pfree(ctx, d_cold); gf_pfree(ctx, d_cn);
    gf_pfree(ctx, d_dmax); gf_pfree(ctx, d_rec);
  };
  if ((st = gf_palloc(ctx, &C->node_agg, (size_t)nnodes)) != GF_OK ||
      (st = gf_palloc(ctx, &d_cnt, (size_t)na + 1)) != GF_OK ||
      (st = gf_palloc(ctx, &C->agg_off, (size_t)na + 1)) != GF_OK ||
      (st = gf_palloc(ctx, &C->agg_nodes, (size_t)nnodes)) != GF_OK ||
      (st = gf_palloc(ctx, &C->cen, (size_t)na * dim)) != GF_OK ||
      (st = gf_palloc(ctx, &C->ainv, (size_t)ntiles * kTS * kTS)) != GF_OK ||
      (st = gf_palloc(ctx, &C->tile_ij, (size_t)ntiles)) != GF_OK ||
      (st = gf_palloc(ctx, &C->counter, 1)) != GF_OK ||
      (st = gf_palloc(ctx, &C->rc, (size_t)ld)) != GF_OK ||
      (st = gf_palloc(ctx, &C->zc, (size_t)ld)) != GF_OK ||
      (st = gf_palloc(ctx, &d_Ac, (size_t)nc * nc)) != GF_OK ||
      (st = gf_palloc(ctx, &d_pi, (size_t)kGJ * kGJ)) != GF_OK ||
      (st = gf_palloc(ctx, &d_rw, (size_t)kGJ * nc)) != GF_OK ||
      (st = gf_palloc(ctx, &d_cold, (size_t)kGJ * nc)) != GF_OK ||
      (st = gf_palloc(ctx, &d_cn, (size_t)kGJ * nc)) != GF_OK ||
      (st = gf_palloc(ctx, &d_dmax, 1)) != GF_OK) {
    cleanup2();
    return st;
  }
  cudaMemsetAsync(d_cnt, 0, sizeof(int32_t) * (na + 1), s);
  cudaMemsetAsync(C->cen, 0, sizeof(double) * na * dim, s);
  k_node_agg<<<gf_blocks(nnodes, kCT), kCT, 0, s>>>(nnodes, d_key, d_id, C->node_agg, d_cnt);
  size_t tb2 = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb2, d_cnt, C->agg_off, na + 1, s);
  if ((st = ensure_tmp(tb2)) != GF_OK) {
    cleanup2();
    return st;
  }
  cub::DeviceScan::ExclusiveSum(d_tmp, tb2, d_cnt, C->agg_off, na + 1, s);
  // node lists: a stable sort of the nodes by aggregate keeps each list ascending, so
  // the per-aggregate kernels read runs of neighbouring nodes
  int32_t* d_iota = nullptr;
  if ((st = gf_palloc(ctx, &d_iota, (size_t)nnodes)) != GF_OK) {
    cleanup2();
    return st;
  }
  k_agg_sums<<<gf_blocks(nnodes, kCT), kCT, 0, s>>>(nnodes, dim, C->node_agg, ctx->d_coords64,
                                                   d_iota, C->cen);
  int end_bit = 1;
  while ((1 << end_bit) < na) ++end_bit;
  size_t tb3 = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb3, C->node_agg, d_key, d_iota, C->agg_nodes, nnodes,
                                  0, end_bit, s);
  if ((st = ensure_tmp(tb3)) != GF_OK) {
    gf_pfree(ctx, d_iota);
    cleanup2();
    return st;
  }
  cub::DeviceRadixSort::SortPairs(d_tmp, tb3, C->node_agg, d_key, d_iota, C->agg_nodes, nnodes, 0,
                                  end_bit, s);
  gf_pfree(ctx, d_iota);
  k_centroid<<<gf_blocks(na, kCT), kCT, 0, s>>>(na, dim, C->agg_off, C->cen);
  // coarse matrix
  cudaMemsetAsync(d_Ac, 0, sizeof(double) * nc * nc, s);
  const double sinv = 1.0 / side;
  std::vector<int32_t> hoff(na + 1);
  GF_CUDA(ctx, cudaMemcpyAsync(hoff.data(), C->agg_off, sizeof(int32_t) * (na + 1),
                               cudaMemcpyDeviceToHost, s));
  GF_CUDA(ctx, cudaStreamSynchronize(s));
  int maxcnt = 1;
  for (int A = 0; A < na; ++A) maxcnt = std::max(maxcnt, hoff[A + 1] - hoff[A]);
  const int per = (int)((maxcnt + (int64_t)kCMT * 65535 - 1) / ((int64_t)kCMT * 65535));
  const dim3 gcm(na, (maxcnt + kCMT * per - 1) / (kCMT * per));
  if (ctx->d_adj && ctx->d_adj_off && na < (1 << 24) && gf_sell_prepare(ctx, GF_F64) == GF_OK &&
      ctx->sell_bdim == dim && gf_palloc(ctx, &d_rec, (size_t)nnodes) == GF_OK) {
    // node-block slices of the FP64 matrix: a thread per node slot, read like the SpMV
    k_node_records<<<gf_blocks(nnodes, kCT), kCT, 0, s>>>(nnodes, dim, ctx->d_coords64,
                                                          C->node_agg, C->cen, ctx->d_fixed,
                                                          sinv, d_rec);
    const int gsl = (nnodes + kSellThreads - 1) / kSellThreads;
    if (dim == 2) {
      GF_CUDA(ctx, gf_smem_attr(k_coarse_rows_sell<2>, sell_coarse_smem<2>()));
      k_coarse_rows_sell<2><<<gsl, kSellThreads, sell_coarse_smem<2>(), s>>>(
          nnodes, ctx->d_sell_off, ctx->d_sell_w, ctx->d_sell_col, ctx->d_sell_perm,
          ctx->d_sell_v64, d_rec, nc, d_Ac);
    } else {
      GF_CUDA(ctx, gf_smem_attr(k_coarse_rows_sell<3>, sell_coarse_smem<3>()));
      k_coarse_rows_sell<3><<<gsl, kSellThreads, sell_coarse_smem<3>(), s>>>(
          nnodes, ctx->d_sell_off, ctx->d_sell_w, ctx->d_sell_col, ctx->d_sell_perm,
          ctx->d_sell_v64, d_rec, nc, d_Ac);
    }
  } else if (dim == 2) {
    k_coarse_rows<2><<<gcm, kCMT, 0, s>>>(n, ctx->d_rownnz, ctx->d_colidx, ctx->d_K64,
                                          ctx->d_fixed, C->node_agg, C->agg_off, C->agg_nodes,
                                          ctx->d_coords64, C->cen, sinv, nc, per, d_Ac);
  } else {
    k_coarse_rows<3><<<gcm, kCMT, 0, s>>>(n, ctx->d_rownnz, ctx->d_colidx, ctx->d_K64,
                                          ctx->d_fixed, C->node_agg, C->agg_off, C->agg_nodes,
                                          ctx->d_coords64, C->cen, sinv, nc, per, d_Ac);
  }
  k_diag_max<<<1, kCT, 0, s>>>(nc, d_Ac, d_dmax);
  k_regularise<<<gf_blocks(nc, kCT), kCT, 0, s>>>(nc, d_dmax, 1e-10, d_Ac);
  ctx->launches += 8;
  // blocked Gauss-Jordan inverse
  const dim3 gp((nc + kGT - 1) / kGT, 2), gu((nc + kGT - 1) / kGT, (nc + kGT - 1) / kGT);
  GF_CUDA(ctx, gf_smem_attr(k_gj_panels, kGJSmem));
  GF_CUDA(ctx, gf_smem_attr(k_gj_update, kGJUpdateSmem));
  for (int kb = 0; kb < nc; kb += kGJ) {
    const int bs = std::min(kGJ, nc - kb);
    k_gj_pivot<<<1, dim3(kGJ, kGJRows), 0, s>>>(nc, kb, bs, d_Ac, d_pi);
    k_gj_panels<<<gp, 256, kGJSmem, s>>>(nc, kb, bs, d_Ac, d_pi, d_rw, d_cold, d_cn);
    k_gj_update<<<gu, 128, kGJUpdateSmem, s>>>(nc, kb, bs, d_Ac, d_pi, d_rw, d_cold, d_cn);
    ctx->launches += 3;
  }
  std::vector<int2> hij;
  hij.reserve(ntiles);
  for (int I = 0; I < nt; ++I)
    for (int J = I; J < nt; ++J) hij.push_back(make_int2(I, J));
  GF_CUDA(ctx, cudaMemcpyAsync(C->tile_ij, hij.data(), sizeof(int2) * ntiles,
                               cudaMemcpyHostToDevice, s));
  k_pack_tiles<<<ntiles, 256, 0, s>>>(nc, C->tile_ij, d_Ac, C->ainv);
  cudaMemsetAsync(C->rc, 0, sizeof(double) * ld, s);  // the tails beyond nc stay zero
  cudaMemsetAsync(C->zc, 0, sizeof(double) * ld, s);
  cudaMemsetAsync(C->counter, 0, sizeof(unsigned), s);
  ctx->launches++;
  cudaError_t e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  cleanup2();
  if (e != cudaSuccess) return gf_cuda_fail(ctx, e, "coarse set-up");
  return GF_OK;
}

}  // namespace

void gf_coarse_free(gf_ctx* ctx) {
  if (!ctx->coarse) return;
  Coarse* c = static_cast<Coarse*>(ctx->coarse);
  coarse_release(ctx, c);
  delete c;
  ctx->coarse = nullptr;
}

// Builds the coarse space for the current FP64 matrix and constraints (once per matrix
// version and target size).
gf_status gf_coarse_prepare(gf_ctx* ctx, int target) {
  if (!ctx->has64) return gf_fail(ctx, GF_ERR_STATE, "the two-level preconditioner needs K64");
  if (!ctx->has_mesh || !ctx->d_diagpos)
    return gf_fail(ctx, GF_ERR_STATE, "the two-level preconditioner needs a mesh-built pattern");
  if (target <= 0) target = ctx->coarse_target > 0 ? ctx->coarse_target : default_coarse(ctx->n);
  Coarse* c = static_cast<Coarse*>(ctx->coarse);
  if (c && c->ver == ctx->kver64) return GF_OK;
  gf_coarse_free(ctx);
  c = new Coarse();
  ctx->coarse = c;
  gf_status st = build(ctx, c, target);
  if (st != GF_OK) {
    gf_coarse_free(ctx);
    return st;
  }
  c->ver = ctx->kver64;
  return GF_OK;
}

// z = D^-1 r + P Ac^-1 P^T r (dinv null: the coarse term alone); add != 0: z += that.
static void coarse_apply_impl(gf_ctx* ctx, const double* r, const double* dinv, double* z,
                              double* rz_acc, const int* done, int add) {
  Coarse* c = static_cast<Coarse*>(ctx->coarse);
  cudaStream_t s = ctx->stream;
  const double sinv = 1.0 / c->s;
  const int pb = std::min(gf_blocks(ctx->n, kCT), ctx->sm_count * 8);
  if (c->dim == 2) {
    k_restrict<2, double><<<c->na, kRT, 0, s>>>(c->agg_off, c->agg_nodes, ctx->d_coords64, c->cen, sinv,
                                        ctx->d_fixed, r, c->rc, c->zc, done);
    k_coarse_symv<<<c->ntiles, 256, 0, s>>>(c->nc, c->tile_ij, c->ainv, c->rc, c->zc, nullptr,
                                            nullptr, done);
    k_prolong<2><<<pb, kCT, 0, s>>>(ctx->n, c->node_agg, ctx->d_coords64, c->cen, sinv,
                                    ctx->d_fixed, dinv, r, c->zc, z, rz_acc, done, add);
  } else {
    k_restrict<3, double><<<c->na, kRT, 0, s>>>(c->agg_off, c->agg_nodes, ctx->d_coords64, c->cen, sinv,
                                        ctx->d_fixed, r, c->rc, c->zc, done);
    k_coarse_symv<<<c->ntiles, 256, 0, s>>>(c->nc, c->tile_ij, c->ainv, c->rc, c->zc, nullptr,
                                            nullptr, done);
    k_prolong<3><<<pb, kCT, 0, s>>>(ctx->n, c->node_agg, ctx->d_coords64, c->cen, sinv,
                                    ctx->d_fixed, dinv, r, c->zc, z, rz_acc, done, add);
  }
  ctx->launches += 3;
}

void gf_coarse_apply(gf_ctx* ctx, const double* r, const double* dinv, double* z, double* rz_acc,
                     const int* done) {
  coarse_apply_impl(ctx, r, dinv, z, rz_acc, done, 0);
}

void gf_coarse_add(gf_ctx* ctx, const double* r, double* z) {
  coarse_apply_impl(ctx, r, nullptr, z, nullptr, nullptr, 1);
}

template <int DIM, typename V>
static void tl_launch(gf_ctx* ctx, int mode, const double* b, const V* q, double scale,
                      double pscale, V* x, V* r, V* p, const V* dinv, SolveScalars* sc,
                      float* p32) {
  Coarse* c = static_cast<Coarse*>(ctx->coarse);
  cudaStream_t s = ctx->stream;
  const int n = ctx->n;
  const double sinv = 1.0 / c->s;
  const int grid = std::min(gf_blocks(n, kCT), ctx->sm_count * 8);
  if (mode == kTlStep)
    k_tl_update<false, V><<<grid, kCT, 0, s>>>(n, nullptr, q, 1.0, x, r, p, dinv, sc);
  else
    k_tl_update<true, V><<<grid, kCT, 0, s>>>(n, b, nullptr, scale, x, r, nullptr, dinv, sc);
  k_restrict<DIM, V><<<c->na, kRT, 0, s>>>(c->agg_off, c->agg_nodes, ctx->d_coords64, c->cen,
                                           sinv, ctx->d_fixed, r, c->rc, c->zc, &sc->done);
  k_coarse_symv<<<c->ntiles, 256, 0, s>>>(c->nc, c->tile_ij, c->ainv, c->rc, c->zc, c->counter,
                                          sc, &sc->done);
  const uint8_t* fx = ctx->d_fixed;
  if (mode == kTlFirst)
    k_tl_direction<DIM, kTlFirst, V><<<grid, kCT, 0, s>>>(n, r, dinv, fx, c->node_agg,
                                                          ctx->d_coords64, c->cen, sinv, c->zc,
                                                          p, p32, 1.0, sc);
  else if (mode == kTlKeep)
    k_tl_direction<DIM, kTlKeep, V><<<grid, kCT, 0, s>>>(n, r, dinv, fx, c->node_agg,
                                                         ctx->d_coords64, c->cen, sinv, c->zc,
                                                         p, p32, pscale, sc);
  else
    k_tl_direction<DIM, kTlStep, V><<<grid, kCT, 0, s>>>(n, r, dinv, fx, c->node_agg,
                                                         ctx->d_coords64, c->cen, sinv, c->zc,
                                                         p, p32, 1.0, sc);
  ctx->launches += 4;
}

template <typename V>
static void tl_reset_impl(gf_ctx* ctx, const double* b, double scale, bool restart,
                          double pscale, V* x, V* r, V* p, const V* dinv, SolveScalars* sc,
                          float* p32) {
  const int mode = restart ? kTlFirst : kTlKeep;
  if (static_cast<Coarse*>(ctx->coarse)->dim == 2)
    tl_launch<2, V>(ctx, mode, b, nullptr, scale, pscale, x, r, p, dinv, sc, p32);
  else
    tl_launch<3, V>(ctx, mode, b, nullptr, scale, pscale, x, r, p, dinv, sc, p32);
}

template <typename V>
static void tl_iterate_impl(gf_ctx* ctx, V* x, V* r, V* p, const V* q, const V* dinv,
                            SolveScalars* sc, float* p32) {
  if (static_cast<Coarse*>(ctx->coarse)->dim == 2)
    tl_launch<2, V>(ctx, kTlStep, nullptr, q, 1.0, 1.0, x, r, p, dinv, sc, p32);
  else
    tl_launch<3, V>(ctx, kTlStep, nullptr, q, 1.0, 1.0, x, r, p, dinv, sc, p32);
}

void gf_tl_begin(gf_ctx* ctx, const double* b, double* x, double* r, double* p,
                 const double* dinv, SolveScalars* sc, float* p32) {
  tl_reset_impl<double>(ctx, b, 1.0, true, 1.0, x, r, p, dinv, sc, p32);
}

void gf_tl_reset(gf_ctx* ctx, const double* b, double scale, bool restart, double pscale,
                 double* x, double* r, double* p, const double* dinv, SolveScalars* sc,
                 float* p32) {
  tl_reset_impl<double>(ctx, b, scale, restart, pscale, x, r, p, dinv, sc, p32);
}

void gf_tl_reset(gf_ctx* ctx, const double* b, double scale, bool restart, double pscale,
                 float* x, float* r, float* p, const float* dinv, SolveScalars* sc) {
  tl_reset_impl<float>(ctx, b, scale, restart, pscale, x, r, p, dinv, sc, nullptr);
}

void gf_tl_iterate(gf_ctx* ctx, double* x, double* r, double* p, const double* q,
                   const double* dinv, SolveScalars* sc, float* p32) {
  tl_iterate_impl<double>(ctx, x, r, p, q, dinv, sc, p32);
}

void gf_tl_iterate(gf_ctx* ctx, float* x, float* r, float* p, const float* q,
                   const float* dinv, SolveScalars* sc) {
  tl_iterate_impl<float>(ctx, x, r, p, q, dinv, sc, nullptr);
}

extern "C" GF_API gf_status gf_twolevel_setup(gf_ctx* ctx, int32_t target_coarse,
                                              int32_t* ncoarse) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (target_coarse < 0) return gf_fail(ctx, GF_ERR_INVALID_ARG, "negative coarse size");
  cudaSetDevice(ctx->device);
  ctx->coarse_target = target_coarse;
  gf_coarse_free(ctx);  // a new target always rebuilds
  gf_status st = gf_coarse_prepare(ctx, target_coarse);
  if (st != GF_OK) return st;
  if (ncoarse) *ncoarse = static_cast<Coarse*>(ctx->coarse)->nc;
  return GF_OK;
}

extern "C" GF_API gf_status gf_twolevel_apply(gf_ctx* ctx, const double* r, double* z) {
  if (!ctx || !r || !z) return GF_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  gf_status st = gf_coarse_prepare(ctx, 0);
  if (st != GF_OK) return st;
  const int n = ctx->n;
  double *d_r = nullptr, *d_z = nullptr, *d_dinv = nullptr, *d_acc = nullptr;
  auto cleanup = [&]() { gf_pfree(ctx, d_r); gf_pfree(ctx, d_z); gf_pfree(ctx, d_dinv); gf_pfree(ctx, d_acc); };
  if ((st = gf_palloc(ctx, &d_r, (size_t)n)) != GF_OK || (st = gf_palloc(ctx, &d_z, (size_t)n)) != GF_OK ||
      (st = gf_palloc(ctx, &d_dinv, (size_t)n)) != GF_OK || (st = gf_palloc(ctx, &d_acc, 1)) != GF_OK) {
    cleanup();
    return st;
  }
  cudaStream_t s = ctx->stream;
  // Jacobi part from the ELL diagonal (1 / K_rr; 1 where the diagonal is zero)
  std::vector<int32_t> rn(n);
  std::vector<int32_t> col((size_t)n * ctx->W);
  std::vector<double> val((size_t)n * ctx->W);
  cudaMemcpyAsync(rn.data(), ctx->d_rownnz, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(col.data(), ctx->d_colidx, sizeof(int32_t) * col.size(), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(val.data(), ctx->d_K64, sizeof(double) * val.size(), cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    cleanup();
    return gf_cuda_fail(ctx, e, "coarse apply");
  }
  std::vector<double> dinv(n, 1.0);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < rn[i]; ++k)
      if (col[(size_t)k * n + i] == i && val[(size_t)k * n + i] != 0.0)
        dinv[i] = 1.0 / val[(size_t)k * n + i];
  cudaMemcpyAsync(d_r, r, sizeof(double) * n, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(d_dinv, dinv.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(d_acc, 0, sizeof(double), s);
  gf_coarse_apply(ctx, d_r, d_dinv, d_z, d_acc, nullptr);
  cudaMemcpyAsync(z, d_z, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
  e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  cleanup();
  if (e != cudaSuccess) return gf_cuda_fail(ctx, e, "coarse apply");
  return GF_OK;
}

extern "C" GF_API gf_status gf_twolevel_aggregates(gf_ctx* ctx, int32_t* node_agg,
                                                   double* box_side) {
  if (!ctx || !node_agg) return GF_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  gf_status st = gf_coarse_prepare(ctx, 0);
  if (st != GF_OK) return st;
  Coarse* c = static_cast<Coarse*>(ctx->coarse);
  GF_CUDA(ctx, cudaMemcpyAsync(node_agg, c->node_agg, sizeof(int32_t) * ctx->nnodes,
                               cudaMemcpyDeviceToHost, ctx->stream));
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (box_side) *box_side = c->s;
  return GF_OK;
}
