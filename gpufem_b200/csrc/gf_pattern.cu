// Symbolic phase: the topological ELL pattern (built on the device) and the
// element colour schedule (built on the host).
//
// Pattern.  The reference discovers its pattern entry by entry while adding
// values (ELLmatrix::AddElem/InsertElem, src/SPRmatrix/ELLmatrix.cc:91-138),
// so its row lengths depend on which contributions are exactly 0.0 and its
// padded width grows 32 -> +64 (ELLmatrix.cc:486-529).  Here the pattern is
// topological: row r (component c of node a) holds every dof of every node
// that shares an element with a, in increasing column order, stored
// column-major (entry (row, slot) at slot*n + row; ELLmatrix.h:35-44).
// width W = max row length; slots past rownnz hold col = row and value 0.
//
// Steps (all on the device):
//   1. node -> element incidence (count, scan, fill)
//   2. per node, the sorted set of adjacent nodes (warp per node, candidates in
//      shared memory, rank of each distinct candidate = its position)
//   3. rownnz / colidx
//   4. slot map: for element e and local nodes (i, j), the position of node_j in
//      node_i's adjacency list, so the numeric scatter never searches.
//
// Colouring.  Greedy first-fit over elements in index order where elements
// sharing at least one node conflict: the rule of femColor::MakeGreedyColoring
// over METIS_MeshToDual(ncommon = 1) (src/FEM/femColor.cc:79-191).
#include <cub/cub.cuh>
#include <algorithm>
#include <numeric>

#include "gf_internal.cuh"

namespace {

constexpr int kWarpsPerBlock = 8;
constexpr int kCandCap = 1024;  // candidate nodes per node (valence * nen)

__global__ void k_count_incidence(int64_t total, const int32_t* __restrict__ conn,
                                  int32_t* __restrict__ cnt) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < total) atomicAdd(&cnt[conn[i]], 1);
}

__global__ void k_fill_incidence(int64_t total, int nen, const int32_t* __restrict__ conn,
                                 int32_t* __restrict__ fillptr, int32_t* __restrict__ inc) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < total) {
    int pos = atomicAdd(&fillptr[conn[i]], 1);
    inc[pos] = (int32_t)(i / nen);
  }
}

// Warp per node: collect the nodes of all incident elements, then for each
// first occurrence compute its rank among distinct values.  mode 0 counts,
// mode 1 writes adj[adj_off[node] + rank].  With at most 32 candidates (every 2-D
// element type) a lane holds one: __match_any_sync finds the first occurrences and
// shuffles rank them, in registers; more candidates go through shared memory.
template <int MODE>
__global__ void k_node_adjacency(int nnodes, int nen, const int32_t* __restrict__ conn,
                                 const int32_t* __restrict__ inc_off,
                                 const int32_t* __restrict__ inc,
                                 int32_t* __restrict__ nadj, const int32_t* __restrict__ adj_off,
                                 int32_t* __restrict__ adj, int32_t* __restrict__ errflag) {
  __shared__ int32_t cand[kWarpsPerBlock][kCandCap];
  __shared__ uint8_t firstf[kWarpsPerBlock][kCandCap];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int node = blockIdx.x * kWarpsPerBlock + warp;
  if (node >= nnodes) return;
  int32_t* c = cand[warp];
  uint8_t* fl = firstf[warp];
  const int e0 = inc_off[node], e1 = inc_off[node + 1];
  const int C = (e1 - e0) * nen;
  if (C <= 32) {
    const bool act = lane < C;
    const int v = act ? conn[(int64_t)inc[e0 + lane / nen] * nen + lane % nen] : 0x7fffffff;
    const unsigned same = __match_any_sync(0xffffffffu, v);
    const bool first = act && (__ffs(same) - 1) == lane;
    const unsigned firsts = __ballot_sync(0xffffffffu, first);
    if (MODE == 0) {
      if (lane == 0) nadj[node] = __popc(firsts);
    } else {
      int rank = 0;
      for (int q = 0; q < 32; ++q) {
        const int vq = __shfl_sync(0xffffffffu, v, q);
        rank += ((firsts >> q) & 1u) && vq < v ? 1 : 0;
      }
      if (first) adj[adj_off[node] + rank] = v;
    }
    return;
  }
  if (C > kCandCap) {
    if (lane == 0) atomicExch(errflag, 1);
    return;
  }
  for (int k = lane; k < C; k += 32) {
    int e = inc[e0 + k / nen];
    c[k] = conn[(int64_t)e * nen + (k % nen)];
  }
  __syncwarp();
  // first-occurrence flags
  for (int k = lane; k < C; k += 32) {
    const int v = c[k];
    uint8_t first = 1;
    for (int q = 0; q < k; ++q)
      if (c[q] == v) { first = 0; break; }
    fl[k] = first;
  }
  __syncwarp();
  int count = 0;
  for (int k = lane; k < C; k += 32) {
    if (!fl[k]) continue;
    if (MODE == 0) {
      ++count;
    } else {
      const int v = c[k];
      int rank = 0;
      for (int q = 0; q < C; ++q) rank += (fl[q] && c[q] < v) ? 1 : 0;
      adj[adj_off[node] + rank] = v;
    }
  }
  if (MODE == 0) {
    for (int o = 16; o > 0; o >>= 1) count += __shfl_down_sync(0xffffffffu, count, o);
    if (lane == 0) nadj[node] = count;
  }
}

// Ascending bitonic sorting network over N register values (N a power of two; every
// index is a compile-time constant once unrolled, so the array stays in registers).
template <int N>
__device__ __forceinline__ void sort_net(int (&a)[N]) {
#pragma unroll
  for (int k = 2; k <= N; k <<= 1)
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
      for (int i = 0; i < N; ++i) {
        const int l = i ^ j;
        if (l > i) {
          const int x = a[i], y = a[l];
          const bool up = (i & k) == 0;
          a[i] = up ? min(x, y) : max(x, y);
          a[l] = up ? max(x, y) : min(x, y);
        }
      }
}

// Thread per node, for meshes whose nodes all see at most NK = 32 or 64 element-node slots
// (2-D meshes with at most 32 / nen elements per node, Brick8 meshes with at most 8) and
// fewer than 2^31 / NK nodes: one pass gives the node's incident elements in ascending
// order (written back to inc), its local index in each, the slot of every element node in
// the node's sorted neighbour list (inc_slot), the node's own slot (diagpos), the
// neighbour count and the sorted list itself, at adj_tmp[inc_off[node] * nen + rank] (a
// node's list has at most as many entries as it has element-node slots).  The
// element-node slots are sorted as keys node id * NK + slot in registers, so equal
// neighbours are adjacent and each slot's rank falls out of one pass.  The same quantities
// as k_node_adjacency + k_incidence_finish + k_diagpos, without their searches.
// Threads per block of k_node_pattern (64 keys: more registers per thread) and the
// shared staging per warp (the warp's incidence slots and candidate lists, stored to HBM
// as one contiguous run each instead of scattered 2- and 4-byte stores).
template <int NK>
constexpr int node_pattern_threads() { return NK == 32 ? 256 : 128; }
template <int NEN, int NK>
constexpr size_t node_pattern_smem() {
  return (size_t)(node_pattern_threads<NK>() / 32) * 32 * NK * (sizeof(uint16_t) + sizeof(int32_t));
}

template <int NEN, int NK>
__global__ void __launch_bounds__(node_pattern_threads<NK>())
k_node_pattern(int nnodes, const int32_t* __restrict__ conn, const int32_t* __restrict__ inc_off,
               int32_t* __restrict__ inc, int32_t* __restrict__ nadj,
               int32_t* __restrict__ adj_tmp, uint8_t* __restrict__ inc_loc,
               uint16_t* __restrict__ inc_slot, int32_t* __restrict__ diagpos) {
  constexpr int MAXD = NK / NEN;   // incident elements per node (checked by the caller)
  constexpr int SH = NK == 32 ? 5 : 6;
  constexpr int kEmpty = 0x7fffffff;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  const int wnode0 = node - lane;
  if (wnode0 >= nnodes) return;   // whole warp
  const bool valid = node < nnodes;
  int32_t* sadj = reinterpret_cast<int32_t*>(smem_raw) + (size_t)wib * 32 * NK;
  uint16_t* sslot = reinterpret_cast<uint16_t*>(reinterpret_cast<int32_t*>(smem_raw) +
                                                (size_t)(blockDim.x / 32) * 32 * NK) +
                    (size_t)wib * 32 * NK;
  const int E0 = inc_off[wnode0], E1 = inc_off[min(wnode0 + 32, nnodes)];
  const int e0 = valid ? inc_off[node] : E1;
  const int deg = valid ? inc_off[node + 1] - e0 : 0;
  int el[MAXD];
#pragma unroll
  for (int q = 0; q < MAXD; ++q) el[q] = q < deg ? inc[e0 + q] : kEmpty;
  sort_net<MAXD>(el);
  int key[NK];
#pragma unroll
  for (int q = 0; q < MAXD; ++q) {
    if (q < deg) inc[e0 + q] = el[q];
    // the element's nodes as 16-byte loads (a row of conn is NEN * 4 = 16 or 32 bytes)
    int4 nd[NEN / 4];
#pragma unroll
    for (int h = 0; h < NEN / 4; ++h)
      nd[h] = q < deg ? __ldg(reinterpret_cast<const int4*>(conn + (int64_t)el[q] * NEN) + h)
                      : make_int4(0, 0, 0, 0);
#pragma unroll
    for (int j = 0; j < NEN; ++j) {
      const int* v = &nd[j / 4].x;
      key[q * NEN + j] = q < deg ? (v[j % 4] << SH) + q * NEN + j : kEmpty;
    }
  }
  sort_net<NK>(key);
  int rank = -1, prev = -1;
  const int l0 = (e0 - E0) * NEN;   // this node's place in the warp's staging
#pragma unroll
  for (int k = 0; k < NK; ++k) {
    const int kk = key[k];
    if (kk != kEmpty) {
      const int v = kk >> SH, slot = kk & (NK - 1);
      if (v != prev) {
        ++rank;
        sadj[l0 + rank] = v;
        prev = v;
      }
      sslot[l0 + slot] = (uint16_t)rank;   // slot = q * NEN + j
      if (v == node) {
        inc_loc[e0 + slot / NEN] = (uint8_t)(slot % NEN);
        diagpos[node] = rank;
      }
    }
  }
  if (valid) {
    nadj[node] = rank + 1;
    if (deg == 0) diagpos[node] = 0;
  }
  __syncwarp();
  // the warp's runs, 16 bytes per store: NEN slots of an incidence are 16 (NEN = 8) or 8
  // bytes, its NEN list entries 32 or 16 bytes, and E0 * NEN keeps both aligned
  const int R = (E1 - E0) * NEN;
  if constexpr (NEN == 8) {
    const uint4* src = reinterpret_cast<const uint4*>(sslot);
    uint4* dst = reinterpret_cast<uint4*>(inc_slot + (int64_t)E0 * NEN);
    for (int i = lane; i < R / 8; i += 32) dst[i] = src[i];
  } else {
    const uint2* src = reinterpret_cast<const uint2*>(sslot);
    uint2* dst = reinterpret_cast<uint2*>(inc_slot + (int64_t)E0 * NEN);
    for (int i = lane; i < R / 4; i += 32) dst[i] = src[i];
  }
  const int4* asrc = reinterpret_cast<const int4*>(sadj);
  int4* adst = reinterpret_cast<int4*>(adj_tmp + (int64_t)E0 * NEN);
  for (int i = lane; i < R / 4; i += 32) adst[i] = asrc[i];
}

// Ascending bitonic sort of 32 K keys held by a warp in blocked order (key[r] of lane l is
// element l K + r): stages with a stride below K swap inside a lane, wider stages exchange
// with lane l ^ (stride / K) by shuffles.  Every loop is unrolled, so the keys stay in
// registers.
template <int K>
__device__ __forceinline__ void warp_sort(int (&key)[K], int lane) {
  constexpr unsigned kFull = 0xffffffffu;
#pragma unroll
  for (int k = 2; k <= 32 * K; k <<= 1)
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= K) {
#pragma unroll
        for (int r = 0; r < K; ++r) {
          const int i = lane * K + r;
          const int o = __shfl_xor_sync(kFull, key[r], j / K);
          key[r] = (((i & j) == 0) == ((i & k) == 0)) ? min(key[r], o) : max(key[r], o);
        }
      } else {
#pragma unroll
        for (int r = 0; r < K; ++r)
          if ((r & j) == 0) {
            const bool up = ((lane * K + r) & k) == 0;
            const int x = key[r], y = key[r + j];
            key[r] = up ? min(x, y) : max(x, y);
            key[r + j] = up ? max(x, y) : min(x, y);
          }
      }
    }
}

// Warp per node, for meshes whose nodes see at most 32 elements and 256 element-node slots
// (Brick20: 8 x 20 = 160) and fewer than 2^23 nodes: the same outputs as k_node_pattern.
// The incident elements are sorted across the lanes by a shuffle bitonic network; the
// element-node slots, as keys node id * 256 + slot, by a register bitonic network over the
// warp (K = 2, 4 or 8 keys per lane: the next power of two above the node's slot count);
// each lane then ranks its run of sorted keys, with the distinct counts of the lanes before
// it from a shuffle scan.  The sorted list and the slots' ranks are staged in shared memory
// and stored as contiguous runs.
constexpr int kWarpKeys = 256;

template <int K>
__device__ __forceinline__ void warp_node_keys(int node, int nen, int C, int el, int lane,
                                               int e0, const int32_t* __restrict__ conn,
                                               int32_t* sadj, uint16_t* sslot,
                                               int32_t* __restrict__ nadj,
                                               int32_t* __restrict__ adj_tmp,
                                               uint8_t* __restrict__ inc_loc,
                                               uint16_t* __restrict__ inc_slot,
                                               int32_t* __restrict__ diagpos) {
  constexpr unsigned kFull = 0xffffffffu;
  constexpr int kEmpty = 0x7fffffff;
  int key[K];
  // slot lane K + r is local node j of incident element q (q, j stepped, not divided)
  int q = (lane * K) / nen, j = lane * K - q * nen;
#pragma unroll
  for (int r = 0; r < K; ++r) {
    const int sl = lane * K + r;
    const int eq = __shfl_sync(kFull, el, min(q, 31));
    key[r] = sl < C ? (__ldg(conn + (int64_t)eq * nen + j) << 8) | sl : kEmpty;
    if (++j == nen) { j = 0; ++q; }
  }
  warp_sort<K>(key, lane);
  const int last = __shfl_up_sync(kFull, key[K - 1], 1);
  const int pv0 = lane == 0 ? -1 : last >> 8;
  int cnt = 0, pv = pv0;
#pragma unroll
  for (int r = 0; r < K; ++r) {
    const int kk = key[r];
    if (kk != kEmpty && (kk >> 8) != pv) ++cnt;
    pv = kk >> 8;
  }
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t;
  }
  int rank = incl - cnt - 1;
  pv = pv0;
#pragma unroll
  for (int r = 0; r < K; ++r) {
    const int kk = key[r];
    if (kk != kEmpty) {
      const int v = kk >> 8, slot = kk & 255;
      if (v != pv) {
        ++rank;
        sadj[rank] = v;
      }
      sslot[slot] = (uint16_t)rank;
      if (v == node) {
        const int qq = slot / nen;
        inc_loc[e0 + qq] = (uint8_t)(slot - qq * nen);
        diagpos[node] = rank;
      }
    }
    pv = kk >> 8;
  }
  const int D = __shfl_sync(kFull, incl, 31);
  if (lane == 0) {
    nadj[node] = D;
    if (C == 0) diagpos[node] = 0;
  }
  __syncwarp();
  const int64_t o0 = (int64_t)e0 * nen;
  for (int i = lane; i < D; i += 32) adj_tmp[o0 + i] = sadj[i];
  for (int i = lane; i < C; i += 32) inc_slot[o0 + i] = sslot[i];
}

__global__ void __launch_bounds__(32 * kWarpsPerBlock)
k_node_pattern_warp(int nnodes, int nen, const int32_t* __restrict__ conn,
                    const int32_t* __restrict__ inc_off, int32_t* __restrict__ inc,
                    int32_t* __restrict__ nadj, int32_t* __restrict__ adj_tmp,
                    uint8_t* __restrict__ inc_loc, uint16_t* __restrict__ inc_slot,
                    int32_t* __restrict__ diagpos) {
  constexpr unsigned kFull = 0xffffffffu;
  constexpr int kEmpty = 0x7fffffff;
  __shared__ int32_t sadj[kWarpsPerBlock][kWarpKeys];
  __shared__ uint16_t sslot[kWarpsPerBlock][kWarpKeys];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int node = blockIdx.x * kWarpsPerBlock + warp;
  if (node >= nnodes) return;   // whole warp
  const int e0 = inc_off[node], deg = inc_off[node + 1] - e0;   // deg <= 32
  const int C = deg * nen;                                        // <= 256
  int el = lane < deg ? inc[e0 + lane] : kEmpty;
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const int o = __shfl_xor_sync(kFull, el, j);
      el = (((lane & j) == 0) == ((lane & k) == 0)) ? min(el, o) : max(el, o);
    }
  if (lane < deg) inc[e0 + lane] = el;   // lane q holds the element of rank q
  // warp-uniform choice of the key count
  if (C <= 64)
    warp_node_keys<2>(node, nen, C, el, lane, e0, conn, sadj[warp], sslot[warp], nadj, adj_tmp,
                      inc_loc, inc_slot, diagpos);
  else if (C <= 128)
    warp_node_keys<4>(node, nen, C, el, lane, e0, conn, sadj[warp], sslot[warp], nadj, adj_tmp,
                      inc_loc, inc_slot, diagpos);
  else
    warp_node_keys<8>(node, nen, C, el, lane, e0, conn, sadj[warp], sslot[warp], nadj, adj_tmp,
                      inc_loc, inc_slot, diagpos);
}

// Block per NB consecutive nodes after the pattern pass: rownnz, the column-major colidx
// rows (a thread per row; all threads walk the slots together, so each slot's column of
// colidx is written by consecutive threads; slots past the row's length hold col = row) and
// the block's part of the compact adjacency (adj_off[n0] .. adj_off[n0 + NB], a flat loop
// over the output range, so every store coalesces), all from the nodes' sorted lists in
// adj_tmp (each node's at its incidence offset x nen), staged in shared memory once.
// FULL: the block's whole scratch run is staged with 16-byte loads (few slots per node:
// 2-D meshes); else only the compact adjacency is gathered (many unused slots: Brick20).
constexpr int kListsThreadsMax = 512;

__host__ __device__ constexpr int lists_table_ints(int NB) { return (2 * (NB + 1) + 3) & ~3; }

template <int DIM, bool FULL>
__global__ void __launch_bounds__(kListsThreadsMax)
k_lists_out(int nnodes, int NB, int n, int W, int nen, const int32_t* __restrict__ inc_off,
            const int32_t* __restrict__ adj_off, const int32_t* __restrict__ adj_tmp,
            int32_t* __restrict__ adj, int32_t* __restrict__ rownnz,
            int32_t* __restrict__ colidx) {
  extern __shared__ __align__(16) int32_t lsm[];
  int32_t* sbase = lsm;             // NB + 1: each node's list start in adj_tmp, from S0
  int32_t* soff = lsm + NB + 1;     // NB + 1: adj_off of the block's nodes
  int32_t* stage = lsm + lists_table_ints(NB);
  const int n0 = blockIdx.x * NB;
  const int nb = min(NB, nnodes - n0);
  const int tid = threadIdx.x, bd = blockDim.x;
  const int I0 = __ldg(inc_off + n0);
  for (int j = tid; j <= nb; j += bd) {
    sbase[j] = (__ldg(inc_off + n0 + j) - I0) * nen;
    soff[j] = __ldg(adj_off + n0 + j);
  }
  const int32_t* src = adj_tmp + (int64_t)I0 * nen;
  if constexpr (FULL) {
    // the run [I0 nen, inc_off[n0 + nb] nen) is 16-byte aligned when nen % 4 == 0
    const int cnt = (__ldg(inc_off + n0 + nb) - I0) * nen;
    if ((nen & 3) == 0) {
      const int4* s4 = reinterpret_cast<const int4*>(src);
      int4* d4 = reinterpret_cast<int4*>(stage);
      for (int i = tid; i < cnt / 4; i += bd) d4[i] = __ldg(s4 + i);
    } else {
      for (int i = tid; i < cnt; i += bd) stage[i] = __ldg(src + i);
    }
  }
  __syncthreads();
  // output word p of the block belongs to the last node j with soff[j] <= soff[0] + p
  const int A0 = soff[0], A = soff[nb] - A0;
  for (int p = tid; p < A; p += bd) {
    int lo = 0, hi = nb - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (soff[mid] - A0 <= p) lo = mid; else hi = mid - 1;
    }
    const int k = A0 + p - soff[lo];
    if constexpr (FULL) {
      adj[A0 + p] = stage[sbase[lo] + k];
    } else {
      const int v = __ldg(src + sbase[lo] + k);
      adj[A0 + p] = v;
      stage[p] = v;
    }
  }
  if constexpr (!FULL) __syncthreads();
  for (int r = tid; r < nb * DIM; r += bd) {
    const int j = r / DIM, row = n0 * DIM + r;
    const int m = soff[j + 1] - soff[j];
    const int32_t* list = FULL ? stage + sbase[j] : stage + (soff[j] - A0);
    rownnz[row] = m * DIM;
#pragma unroll 4
    for (int k = 0; k < W / DIM; ++k) {
      const bool in = k < m;
      const int b = in ? list[k] * DIM : 0;
#pragma unroll
      for (int c = 0; c < DIM; ++c) colidx[(int64_t)(k * DIM + c) * n + row] = in ? b + c : row;
    }
  }
}

__global__ void k_rownnz(int nnodes, int dim, const int32_t* __restrict__ nadj,
                         int32_t* __restrict__ rownnz) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a < nnodes)
    for (int c = 0; c < dim; ++c) rownnz[a * dim + c] = nadj[a] * dim;
}

// Thread per row: the columns of row (node a, component c) are the dofs of a's sorted
// adjacency list; slots past the row's length hold col = row.  All threads walk the
// slots together, so each slot's column of colidx is written by consecutive threads.
template <int DIM>
__global__ void k_colidx(int n, int W, const int32_t* __restrict__ adj_off,
                         const int32_t* __restrict__ adj, int32_t* __restrict__ colidx) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  const int node = row / DIM;
  const int q0 = adj_off[node];
  const int len = (adj_off[node + 1] - q0) * DIM;
  for (int s = 0; s < W; ++s) {
    const int b = s < len ? __ldg(adj + q0 + s / DIM) : 0;
    colidx[(int64_t)s * n + row] = s < len ? b * DIM + s % DIM : row;
  }
}

// Thread per (element e, local node i), e fastest so the slot-map writes coalesce: the
// slots of e's nodes in node i's adjacency list are the ones the pattern pass recorded for
// that incidence (inc_slot), found by a short scan of node i's sorted incident elements.
__global__ void k_slotmap(int nelem, int nen, const int32_t* __restrict__ conn,
                          const int32_t* __restrict__ inc_off, const int32_t* __restrict__ inc,
                          const uint16_t* __restrict__ inc_slot,
                          uint16_t* __restrict__ slotmap, int32_t* __restrict__ errflag) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)nelem * nen) return;
  const int e = (int)(t % nelem);
  const int i = (int)(t / nelem);
  const int a = conn[(int64_t)e * nen + i];
  const int q1 = inc_off[a + 1];
  int q = inc_off[a];
  while (q < q1 && __ldg(inc + q) != e) ++q;
  if (q >= q1) {
    atomicExch(errflag, 2);
    return;
  }
  const uint16_t* src = inc_slot + (int64_t)q * nen;
  for (int j = 0; j < nen; ++j) slotmap[(int64_t)(i * nen + j) * nelem + e] = __ldg(src + j);
}

__global__ void k_diagpos(int nnodes, const int32_t* __restrict__ adj_off,
                          const int32_t* __restrict__ adj, int32_t* __restrict__ diagpos) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= nnodes) return;
  int lo = adj_off[a], hi = adj_off[a + 1];
  const int lo0 = lo;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (adj[mid] < a) lo = mid + 1; else hi = mid;
  }
  diagpos[a] = lo - lo0;
}

// Thread per node: sort its incident elements ascending, then record the node's
// local index in each of them and, for every node of each incident element, that
// node's position in this node's adjacency list (the owner-computes scatter
// writes row blocks of this node without searching).
__global__ void k_incidence_finish(int nnodes, int nen, const int32_t* __restrict__ conn,
                                   const int32_t* __restrict__ inc_off, int32_t* __restrict__ inc,
                                   const int32_t* __restrict__ adj_off,
                                   const int32_t* __restrict__ adj, uint8_t* __restrict__ inc_loc,
                                   uint16_t* __restrict__ inc_slot, int32_t* __restrict__ errflag) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= nnodes) return;
  const int q0 = inc_off[a], q1 = inc_off[a + 1];
  for (int q = q0 + 1; q < q1; ++q) {  // insertion sort (lists are short)
    const int v = inc[q];
    int k = q - 1;
    while (k >= q0 && inc[k] > v) {
      inc[k + 1] = inc[k];
      --k;
    }
    inc[k + 1] = v;
  }
  const int lo0 = adj_off[a], hi0 = adj_off[a + 1];
  for (int q = q0; q < q1; ++q) {
    const int e = inc[q];
    int loc = -1;
    for (int i = 0; i < nen; ++i)
      if (conn[(int64_t)e * nen + i] == a) loc = i;
    if (loc < 0) atomicExch(errflag, 3);
    inc_loc[q] = (uint8_t)(loc < 0 ? 0 : loc);
    for (int j = 0; j < nen; ++j) {
      const int b = conn[(int64_t)e * nen + j];
      int lo = lo0, hi = hi0;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (adj[mid] < b) lo = mid + 1; else hi = mid;
      }
      if (lo >= hi0 || adj[lo] != b) atomicExch(errflag, 4);
      inc_slot[(int64_t)q * nen + j] = (uint16_t)(lo - lo0);
    }
  }
}

}  // namespace

gf_status gf_pattern_build(gf_ctx* ctx) {
  const int nnodes = ctx->nnodes, nelem = ctx->nelem, nen = ctx->nen, dim = ctx->dim;
  const int64_t total = (int64_t)nelem * nen;
  cudaStream_t s = ctx->stream;
  gf_pattern_free(ctx);
  if (ctx->n != nnodes * dim)
    return gf_fail(ctx, GF_ERR_STATE, "dof count %d does not match the mesh (%d)", ctx->n,
                   nnodes * dim);
  gf_status st;

  int32_t *d_cnt = nullptr, *d_inc_off = nullptr, *d_fill = nullptr, *d_inc = nullptr;
  int32_t *d_nadj = nullptr, *d_err = nullptr, *d_max = nullptr, *d_adjtmp = nullptr;
  char* d_tmp = nullptr;
  size_t tmp_bytes = 0, b1 = 0, b2 = 0, b3 = 0;
  auto cleanup = [&]() {
    gf_pfree(ctx, d_cnt); gf_pfree(ctx, d_inc_off); gf_pfree(ctx, d_fill); gf_pfree(ctx, d_inc);
    gf_pfree(ctx, d_nadj); gf_pfree(ctx, d_err); gf_pfree(ctx, d_max); gf_pfree(ctx, d_tmp);
    gf_pfree(ctx, d_adjtmp);
  };
#define GF_TRY(x)             \
  do {                        \
    if ((st = (x)) != GF_OK) { cleanup(); return st; } \
  } while (0)
#define GF_TRYC(call)                                                  \
  do {                                                                 \
    cudaError_t e__ = (call);                                          \
    if (e__ != cudaSuccess) { cleanup(); return gf_cuda_fail(ctx, e__, #call); } \
  } while (0)

  GF_TRY(gf_palloc(ctx, &d_cnt, (size_t)nnodes + 1));
  GF_TRY(gf_palloc(ctx, &d_inc_off, (size_t)nnodes + 1));
  GF_TRY(gf_palloc(ctx, &d_fill, (size_t)nnodes + 1));
  GF_TRY(gf_palloc(ctx, &d_inc, (size_t)total));
  GF_TRY(gf_palloc(ctx, &d_nadj, (size_t)nnodes + 1));
  GF_TRY(gf_palloc(ctx, &d_err, 1));
  GF_TRY(gf_palloc(ctx, &d_max, 2));
  GF_TRY(gf_palloc(ctx, &ctx->d_adj_off, (size_t)nnodes + 1));
  GF_TRYC(cudaMemsetAsync(d_cnt, 0, sizeof(int32_t) * (nnodes + 1), s));
  GF_TRYC(cudaMemsetAsync(d_nadj, 0, sizeof(int32_t) * (nnodes + 1), s));
  GF_TRYC(cudaMemsetAsync(d_err, 0, sizeof(int32_t), s));

  cub::DeviceScan::ExclusiveSum(nullptr, b1, d_cnt, d_inc_off, nnodes + 1, s);
  cub::DeviceReduce::Max(nullptr, b2, d_nadj, d_max, nnodes, s);
  b3 = b1;
  tmp_bytes = std::max(b1, std::max(b2, b3));
  GF_TRY(gf_palloc(ctx, &d_tmp, tmp_bytes));

  k_count_incidence<<<gf_blocks(total, 256), 256, 0, s>>>(total, ctx->d_conn, d_cnt);
  ctx->launches++;
  GF_TRYC(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_cnt, d_inc_off, nnodes + 1, s));
  GF_TRYC(cudaMemcpyAsync(d_fill, d_inc_off, sizeof(int32_t) * (nnodes + 1),
                          cudaMemcpyDeviceToDevice, s));
  k_fill_incidence<<<gf_blocks(total, 256), 256, 0, s>>>(total, nen, ctx->d_conn, d_fill, d_inc);
  ctx->launches++;
  // the most elements around one node decides the adjacency path
  GF_TRYC(cub::DeviceReduce::Max(d_tmp, tmp_bytes, d_cnt, d_max + 1, nnodes, s));
  int32_t h_maxval = 0;
  GF_TRYC(cudaMemcpyAsync(&h_maxval, d_max + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  GF_TRYC(cudaStreamSynchronize(s));
  // one pass per node: a register sort of its element-node slots (32 or 64 keys, a thread
  // per node), else a shared-memory sort (up to 256 keys, a warp per node), else the
  // general count / write / search passes
  const int64_t slots_max = (int64_t)h_maxval * nen;
  const int nkeys = slots_max <= 32 ? 32 : slots_max <= 64 ? 64 : 0;
  const bool thread_pass = nkeys > 0 && (nen == 4 || nen == 8) && nnodes < (1 << 24);
  const bool warp_pass = !thread_pass && h_maxval <= 32 && slots_max <= kWarpKeys &&
                         nnodes < (1 << 23);
  const bool fused = thread_pass || warp_pass;
  const int ablocks = (nnodes + kWarpsPerBlock - 1) / kWarpsPerBlock;
  if (fused) {
    GF_TRY(gf_palloc(ctx, &d_adjtmp, (size_t)total * nen));
    GF_TRY(gf_palloc(ctx, &ctx->d_inc_loc, (size_t)total));
    GF_TRY(gf_palloc(ctx, &ctx->d_inc_slot, (size_t)total * nen));
    GF_TRY(gf_palloc(ctx, &ctx->d_diagpos, (size_t)nnodes));
    if (thread_pass) {
      auto kp = nen == 4 ? (nkeys == 32 ? k_node_pattern<4, 32> : k_node_pattern<4, 64>)
                         : (nkeys == 32 ? k_node_pattern<8, 32> : k_node_pattern<8, 64>);
      const int nt = nkeys == 32 ? node_pattern_threads<32>() : node_pattern_threads<64>();
      const size_t sm = nen == 4 ? (nkeys == 32 ? node_pattern_smem<4, 32>()
                                                : node_pattern_smem<4, 64>())
                                 : (nkeys == 32 ? node_pattern_smem<8, 32>()
                                                : node_pattern_smem<8, 64>());
      GF_TRYC(gf_smem_attr(kp, sm));
      kp<<<gf_blocks(nnodes, nt), nt, sm, s>>>(nnodes, ctx->d_conn, d_inc_off, d_inc, d_nadj,
                                               d_adjtmp, ctx->d_inc_loc, ctx->d_inc_slot,
                                               ctx->d_diagpos);
    } else {
      k_node_pattern_warp<<<ablocks, 32 * kWarpsPerBlock, 0, s>>>(
          nnodes, nen, ctx->d_conn, d_inc_off, d_inc, d_nadj, d_adjtmp, ctx->d_inc_loc,
          ctx->d_inc_slot, ctx->d_diagpos);
    }
  } else {
    k_node_adjacency<0><<<ablocks, 32 * kWarpsPerBlock, 0, s>>>(
        nnodes, nen, ctx->d_conn, d_inc_off, d_inc, d_nadj, nullptr, nullptr, d_err);
  }
  ctx->launches++;
  GF_TRYC(cudaGetLastError());
  GF_TRYC(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_nadj, ctx->d_adj_off, nnodes + 1, s));
  GF_TRYC(cub::DeviceReduce::Max(d_tmp, tmp_bytes, d_nadj, d_max, nnodes, s));
  int32_t h_err = 0, h_max = 0, h_tot = 0;
  GF_TRYC(cudaMemcpyAsync(&h_err, d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  GF_TRYC(cudaMemcpyAsync(&h_max, d_max, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  GF_TRYC(cudaMemcpyAsync(&h_tot, ctx->d_adj_off + nnodes, sizeof(int32_t),
                          cudaMemcpyDeviceToHost, s));
  GF_TRYC(cudaStreamSynchronize(s));
  if (h_err) {
    cleanup();
    return gf_fail(ctx, GF_ERR_UNSUPPORTED,
                   "a node is shared by more than %d element-node slots (valence * nen)",
                   kCandCap);
  }
  if (h_max * dim > 65535) {
    cleanup();
    return gf_fail(ctx, GF_ERR_UNSUPPORTED, "row width %d exceeds 65535", h_max * dim);
  }
  ctx->W = h_max * dim;
  ctx->nnz = (int64_t)h_tot * dim * dim;
  const int n = ctx->n;
  const int64_t slots = (int64_t)n * ctx->W;
  GF_TRY(gf_palloc(ctx, &ctx->d_adj, (size_t)h_tot));
  GF_TRY(gf_palloc(ctx, &ctx->d_rownnz, (size_t)n));
  GF_TRY(gf_palloc(ctx, &ctx->d_colidx, (size_t)slots));
  if (fused) {
    // whole scratch runs staged when nodes have at most 32 element-node slots (measured on
    // Q8 512: 85 against 97 us for the compact gather), else the compact lists (Brick20
    // 64: 0.96 against 1.25 ms); nodes per block: the staged words within 48 KB
    const bool full = (int64_t)h_maxval * nen <= 32;
    const int per_node = full ? h_maxval * nen : h_max;
    int NB = 128;
    while (NB > 32 && (size_t)NB * per_node * sizeof(int32_t) > 48 * 1024) NB >>= 1;
    const size_t lsm = sizeof(int32_t) * ((size_t)lists_table_ints(NB) + (size_t)NB * per_node);
    const int nt = std::min(kListsThreadsMax, (NB * dim + 31) / 32 * 32);
    const int nblk = (nnodes + NB - 1) / NB;
    auto kl = dim == 2 ? (full ? k_lists_out<2, true> : k_lists_out<2, false>)
                       : (full ? k_lists_out<3, true> : k_lists_out<3, false>);
    GF_TRYC(gf_smem_attr(kl, lsm));
    if (nblk > 0)
      kl<<<nblk, nt, lsm, s>>>(nnodes, NB, n, ctx->W, nen, d_inc_off, ctx->d_adj_off, d_adjtmp,
                               ctx->d_adj, ctx->d_rownnz, ctx->d_colidx);
    ctx->launches++;
  } else {
    GF_TRY(gf_palloc(ctx, &ctx->d_diagpos, (size_t)nnodes));
    k_node_adjacency<1><<<ablocks, 32 * kWarpsPerBlock, 0, s>>>(
        nnodes, nen, ctx->d_conn, d_inc_off, d_inc, nullptr, ctx->d_adj_off, ctx->d_adj, d_err);
    k_rownnz<<<gf_blocks(nnodes, 256), 256, 0, s>>>(nnodes, dim, d_nadj, ctx->d_rownnz);
    if (dim == 2)
      k_colidx<2><<<gf_blocks(n, 256), 256, 0, s>>>(n, ctx->W, ctx->d_adj_off, ctx->d_adj,
                                                    ctx->d_colidx);
    else
      k_colidx<3><<<gf_blocks(n, 256), 256, 0, s>>>(n, ctx->W, ctx->d_adj_off, ctx->d_adj,
                                                    ctx->d_colidx);
    ctx->launches += 3;
  }
  if (!fused) {
    k_diagpos<<<gf_blocks(nnodes, 256), 256, 0, s>>>(nnodes, ctx->d_adj_off, ctx->d_adj,
                                                     ctx->d_diagpos);
    ctx->launches++;
    // incidence kept for the owner-computes scatter
    GF_TRY(gf_palloc(ctx, &ctx->d_inc_loc, (size_t)total));
    GF_TRY(gf_palloc(ctx, &ctx->d_inc_slot, (size_t)total * nen));
    k_incidence_finish<<<gf_blocks(nnodes, 128), 128, 0, s>>>(
        nnodes, nen, ctx->d_conn, d_inc_off, d_inc, ctx->d_adj_off, ctx->d_adj, ctx->d_inc_loc,
        ctx->d_inc_slot, d_err);
    ctx->launches++;
  }
  GF_TRYC(cudaGetLastError());
  GF_TRYC(cudaMemcpyAsync(&h_err, d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  GF_TRYC(cudaStreamSynchronize(s));
  if (h_err) {
    cleanup();
    return gf_fail(ctx, GF_ERR_CUDA, "pattern build: slot map lookup failed (%d)", h_err);
  }
  ctx->d_inc_off = d_inc_off;  // ownership moves to the context
  ctx->d_inc = d_inc;
  d_inc_off = nullptr;
  d_inc = nullptr;
  ctx->maxval = h_maxval;
  cleanup();
  ctx->has_pattern = true;
  return GF_OK;
#undef GF_TRY
#undef GF_TRYC
}

// Element slot map of the colour and atomic schedules (the owner schedule reads the
// per-node incidence slots instead), built on the first assembly that needs it.
gf_status gf_slotmap_ensure(gf_ctx* ctx) {
  if (ctx->d_slotmap) return GF_OK;
  if (!ctx->has_pattern) return gf_fail(ctx, GF_ERR_STATE, "no pattern");
  const int nelem = ctx->nelem, nen = ctx->nen;
  const int64_t total = (int64_t)nelem * nen;
  cudaStream_t s = ctx->stream;
  gf_status st;
  int32_t* d_err = nullptr;
  if ((st = gf_palloc(ctx, &d_err, 1)) != GF_OK) return st;
  if ((st = gf_palloc(ctx, &ctx->d_slotmap, (size_t)total * nen)) != GF_OK) {
    gf_pfree(ctx, d_err);
    return st;
  }
  int32_t h_err = 0;
  cudaMemsetAsync(d_err, 0, sizeof(int32_t), s);
  k_slotmap<<<gf_blocks(total, 256), 256, 0, s>>>(nelem, nen, ctx->d_conn, ctx->d_inc_off,
                                                  ctx->d_inc, ctx->d_inc_slot, ctx->d_slotmap,
                                                  d_err);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  gf_pfree(ctx, d_err);
  if (e != cudaSuccess || h_err) {
    gf_pfree(ctx, ctx->d_slotmap);
    return e != cudaSuccess ? gf_cuda_fail(ctx, e, "slot map")
                            : gf_fail(ctx, GF_ERR_CUDA, "slot map lookup failed");
  }
  return GF_OK;
}

// ---------------------------------------------------------------------------
// Colouring (host)
// ---------------------------------------------------------------------------
gf_status gf_color_build(gf_ctx* ctx, const int32_t* user_colors) {
  const int nelem = ctx->nelem, nen = ctx->nen, nnodes = ctx->nnodes;
  if (ctx->h_conn.size() != (size_t)nelem * nen) {  // host copy on first use
    ctx->h_conn.resize((size_t)nelem * nen);
    GF_CUDA(ctx, cudaMemcpyAsync(ctx->h_conn.data(), ctx->d_conn,
                                 sizeof(int32_t) * ctx->h_conn.size(), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  const std::vector<int32_t>& conn = ctx->h_conn;
  // node -> element incidence
  std::vector<int32_t> off(nnodes + 1, 0), inc((size_t)nelem * nen);
  for (size_t k = 0; k < conn.size(); ++k) off[conn[k] + 1]++;
  for (int i = 0; i < nnodes; ++i) off[i + 1] += off[i];
  {
    std::vector<int32_t> fill(off.begin(), off.end() - 1);
    for (size_t k = 0; k < conn.size(); ++k) inc[fill[conn[k]]++] = (int32_t)(k / nen);
  }
  std::vector<int32_t> color(nelem, -1);
  if (user_colors) {
    for (int e = 0; e < nelem; ++e) {
      if (user_colors[e] < 0 || user_colors[e] > 4095)
        return gf_fail(ctx, GF_ERR_INVALID_ARG, "colour of element %d is %d", e, user_colors[e]);
      color[e] = user_colors[e];
    }
    // validate: the elements around each node have pairwise distinct colours
    std::vector<int32_t> seen;
    for (int a = 0; a < nnodes; ++a) {
      seen.clear();
      for (int q = off[a]; q < off[a + 1]; ++q) seen.push_back(color[inc[q]]);
      std::sort(seen.begin(), seen.end());
      if (std::adjacent_find(seen.begin(), seen.end()) != seen.end())
        return gf_fail(ctx, GF_ERR_INVALID_ARG,
                       "invalid colouring: two elements of one colour share node %d", a + 1);
    }
  } else {
    // greedy first-fit in element order; uncoloured neighbours do not constrain
    std::vector<int32_t> stamp(4096, -1);
    for (int e = 0; e < nelem; ++e) {
      for (int i = 0; i < nen; ++i) {
        const int a = conn[(size_t)e * nen + i];
        for (int q = off[a]; q < off[a + 1]; ++q) {
          const int c = color[inc[q]];
          if (c >= 0) stamp[c] = e;
        }
      }
      int c = 0;
      while (c < 4096 && stamp[c] == e) ++c;
      if (c == 4096) return gf_fail(ctx, GF_ERR_UNSUPPORTED, "more than 4096 colours");
      color[e] = c;
    }
  }
  int ncol = 0;
  for (int e = 0; e < nelem; ++e) ncol = std::max(ncol, color[e] + 1);
  std::vector<int32_t> coff(ncol + 1, 0), perm(nelem);
  for (int e = 0; e < nelem; ++e) coff[color[e] + 1]++;
  for (int c = 0; c < ncol; ++c) coff[c + 1] += coff[c];
  {
    std::vector<int32_t> fill(coff.begin(), coff.end() - 1);
    for (int e = 0; e < nelem; ++e) perm[fill[color[e]]++] = e;  // stable: ascending ids
  }
  gf_status st;
  if ((st = gf_alloc(ctx, &ctx->d_perm, (size_t)nelem)) != GF_OK) return st;
  GF_CUDA(ctx, cudaMemcpyAsync(ctx->d_perm, perm.data(), sizeof(int32_t) * nelem,
                               cudaMemcpyHostToDevice, ctx->stream));
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->h_color = color;
  ctx->color_off = coff;
  ctx->ncolors = ncol;
  return GF_OK;
}
