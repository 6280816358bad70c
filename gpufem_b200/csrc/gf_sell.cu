// Sliced ELL (SELL-32) copy of K for the solver's SpMVs.
//
// The column-major ELL of the reference layout (ELLmatrix.h:35-44) puts entry s of
// row r at s*n + r: a warp's loads for one slot are coalesced, but the W slots of a
// row sit n entries apart, so every step of the row loop opens new DRAM pages, and
// lanes whose rows are shorter idle inside partially used sectors.  The solver
// therefore keeps a second copy cut into slices of 32 consecutive rows, each slice
// padded only to its own longest row and stored slot-major and contiguous (entry s
// of lane l at off[k] + 32 s + l).  Rows keep their order, so vectors are indexed as
// in the ELL.  Padding entries hold column = the row itself and value 0, which lets
// every lane of a slice run the same trip count.  The ELL stays the layout of the
// API (views, downloads, assembly, constraints); values are re-sliced only when the
// matrix changed since the last conversion.
//
// Node-block slices (mesh-built patterns).  The rows of a node share one neighbour-node
// list and every (node, neighbour) pair is a dense dim x dim block, so the copy keeps one
// column index per block instead of one per entry: slices of 32 nodes (slot a holds node
// perm[a]; the order is degree-sorted within windows of 256 nodes), each padded to its
// longest neighbour list, with
//   bcol[off[k] + 32 p + l]                          neighbour p of node perm[32 k + l]
//   val[dim^2 off[k] + ((p dim + c) dim + c2) 32 + l] K(row perm[32k+l] dim + c,
//                                                      col bcol dim + c2)
// A thread computes the dim rows of one node: per neighbour it reads one coalesced
// column word, dim^2 coalesced value words and dim consecutive entries of x.  Index
// bytes per entry fall from 4 to 4 / dim^2 (12 -> 9 B per FP64 entry in 2-D, 8.4 B in
// 3-D).  Padding: column = the node itself, value 0.
#include <cub/cub.cuh>
#include <algorithm>

#include "gf_internal.cuh"

namespace {

__global__ void k_sell_width(int n, int nslice, const int32_t* __restrict__ rownnz,
                             int64_t* __restrict__ wsz, int32_t* __restrict__ width) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nslice) return;
  int w = 0;
  for (int l = 0; l < 32; ++l) {
    const int row = k * 32 + l;
    if (row < n) w = max(w, rownnz[row]);
  }
  width[k] = w;
  wsz[k] = (int64_t)w * 32;
}

template <typename TI, typename TO>
__global__ void k_sell_fill(int n, int nslots, const int64_t* __restrict__ off,
                            const int32_t* __restrict__ width, const int32_t* __restrict__ rownnz,
                            const TI* __restrict__ src, TO* __restrict__ dst, int is_col) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;  // slot of the padded row range
  if (row >= nslots) return;
  const int k = row >> 5, lane = row & 31;
  const int w = width[k];
  const int nz = row < n ? rownnz[row] : 0;
  int64_t o = off[k] + lane;
  for (int s = 0; s < w; ++s, o += 32) {
    TO v;
    if (s < nz) v = (TO)src[(int64_t)s * n + row];
    else v = is_col ? (TO)(row < n ? row : 0) : (TO)0;
    dst[o] = v;
  }
}

// Node order of the slices: within each window of kWin consecutive nodes, nodes sorted
// by neighbour count (descending; equal counts keep their order), so that the 32 nodes of
// a slice have nearly equal rows and little padding.  Mesh numberings interleave node
// kinds (Q8 corner nodes have 21 neighbours, mid-side nodes 13; Brick20 81 / 51 / 33):
// padding falls from 21% to 2% of the entries on Q8 512, from 31% to 6% on Brick20 64.
constexpr int kWin = 256;
__global__ void __launch_bounds__(kWin)
k_bsell_perm(int nnodes, int dim, const int32_t* __restrict__ rownnz, int32_t* __restrict__ perm) {
  __shared__ int deg[kWin];
  const int a0 = blockIdx.x * kWin, cnt = min(kWin, nnodes - a0);
  const int i = threadIdx.x;
  if (i < cnt) deg[i] = rownnz[(int64_t)(a0 + i) * dim] / dim;
  __syncthreads();
  if (i >= cnt) return;
  const int di = deg[i];
  int rank = 0;
  for (int j = 0; j < cnt; ++j) {
    const int dj = deg[j];
    rank += (dj > di) || (dj == di && j < i);
  }
  perm[a0 + rank] = a0 + i;
}

__global__ void k_bsell_width(int nnodes, int dim, int nslice, const int32_t* __restrict__ rownnz,
                              const int32_t* __restrict__ perm, int64_t* __restrict__ wsz,
                              int32_t* __restrict__ width) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nslice) return;
  int w = 0;
  for (int l = 0; l < 32; ++l) {
    const int a = k * 32 + l;
    if (a < nnodes) w = max(w, rownnz[(int64_t)perm[a] * dim] / dim);
  }
  width[k] = w;
  wsz[k] = (int64_t)w * 32;
}

__global__ void k_bsell_col(int n, int nnodes, int dim, int nslots, const int64_t* __restrict__ off,
                            const int32_t* __restrict__ width, const int32_t* __restrict__ rownnz,
                            const int32_t* __restrict__ colidx, const int32_t* __restrict__ perm,
                            int32_t* __restrict__ bcol) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;  // node slot
  if (a >= nslots) return;
  const int k = a >> 5, l = a & 31;
  const int w = width[k];
  const int node = a < nnodes ? perm[a] : 0;
  const int nadj = a < nnodes ? rownnz[(int64_t)node * dim] / dim : 0;
  for (int p = 0; p < w; ++p)
    bcol[off[k] + 32 * p + l] =
        p < nadj ? colidx[(int64_t)(p * dim) * n + (int64_t)node * dim] / dim : node;
}

// Thread per node slot: per neighbour p and column component c2, the node's DIM rows of
// that ELL column are DIM consecutive entries (one or two sectors, read once), and each of
// the DIM x DIM values goes to its slice word, so a warp's stores coalesce.  Slots of one
// block are one degree-sorting window (256 consecutive nodes), so the sectors that several
// nodes of the window share are read from L1.
template <typename TI, typename TO, int DIM>
__global__ void k_bsell_val(int n, int nnodes, int nslots, const int64_t* __restrict__ off,
                            const int32_t* __restrict__ width, const int32_t* __restrict__ rownnz,
                            const int32_t* __restrict__ perm, const TI* __restrict__ K,
                            TO* __restrict__ val) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= nslots) return;
  const int k = a >> 5, l = a & 31;
  const int w = width[k];
  const int node = a < nnodes ? perm[a] : 0;
  const int nadj = a < nnodes ? rownnz[(int64_t)node * DIM] / DIM : 0;
  TO* dst = val + off[k] * DIM * DIM + l;
  const int64_t row = (int64_t)node * DIM;
  for (int p = 0; p < w; ++p) {
    const bool in = p < nadj;
#pragma unroll
    for (int c2 = 0; c2 < DIM; ++c2) {
      const TI* src = K + (int64_t)(p * DIM + c2) * n + row;
#pragma unroll
      for (int c = 0; c < DIM; ++c)
        dst[(int64_t)((p * DIM + c) * DIM + c2) * 32] = in ? (TO)__ldg(src + c) : (TO)0;
    }
  }
}

}  // namespace

void gf_sell_free(gf_ctx* ctx) {
  gf_free(ctx->d_sell_off);
  gf_free(ctx->d_sell_w);
  gf_free(ctx->d_sell_col);
  gf_free(ctx->d_sell_perm);
  gf_free(ctx->d_sell_v64);
  gf_free(ctx->d_sell_v32);
  ctx->sell_ready = false;
  ctx->sell_ver64 = ctx->sell_ver32 = -1;
  ctx->sell_total = 0;
  ctx->sell_bdim = 0;
}

// Builds the slice pattern if needed and refreshes the values of `dtype`.
gf_status gf_sell_prepare(gf_ctx* ctx, int dtype) {
  const int n = ctx->n;
  cudaStream_t s = ctx->stream;
  gf_status st;
  // node blocks where the pattern came from a mesh (every row of a node has the same
  // neighbour-node list, dim entries per neighbour)
  const int bdim = (ctx->d_adj_off && ctx->has_mesh && (ctx->dim == 2 || ctx->dim == 3) &&
                    (int64_t)ctx->nnodes * ctx->dim == n) ? ctx->dim : 0;
  if (ctx->sell_ready && ctx->sell_bdim != bdim) gf_sell_free(ctx);
  if (!ctx->sell_ready) {
    gf_sell_free(ctx);
    const int units = bdim ? ctx->nnodes : n;  // nodes or rows
    const int nslice = (units + 31) / 32;
    const int nslots = nslice * 32;
    int64_t* wsz = nullptr;
    void* tmp = nullptr;
    size_t tb = 0;
    if ((st = gf_alloc(ctx, &ctx->d_sell_off, (size_t)nslice + 1)) != GF_OK) return st;
    if ((st = gf_alloc(ctx, &ctx->d_sell_w, (size_t)nslice)) != GF_OK) return st;
    if ((st = gf_alloc(ctx, &wsz, (size_t)nslice + 1)) != GF_OK) return st;
    if (bdim) {
      if ((st = gf_alloc(ctx, &ctx->d_sell_perm, (size_t)ctx->nnodes)) != GF_OK) {
        cudaFree(wsz);
        return st;
      }
      k_bsell_perm<<<(ctx->nnodes + kWin - 1) / kWin, kWin, 0, s>>>(ctx->nnodes, bdim,
                                                                   ctx->d_rownnz, ctx->d_sell_perm);
      k_bsell_width<<<gf_blocks(nslice, 256), 256, 0, s>>>(ctx->nnodes, bdim, nslice, ctx->d_rownnz,
                                                           ctx->d_sell_perm, wsz, ctx->d_sell_w);
      ctx->launches++;
    }
    else
      k_sell_width<<<gf_blocks(nslice, 256), 256, 0, s>>>(n, nslice, ctx->d_rownnz, wsz,
                                                          ctx->d_sell_w);
    ctx->launches++;
    GF_CUDA(ctx, cudaMemsetAsync(wsz + nslice, 0, sizeof(int64_t), s));
    cub::DeviceScan::ExclusiveSum(nullptr, tb, wsz, ctx->d_sell_off, nslice + 1, s);
    if (cudaMalloc(&tmp, tb) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(wsz);
      return gf_fail(ctx, GF_ERR_OOM, "SELL scan scratch");
    }
    cub::DeviceScan::ExclusiveSum(tmp, tb, wsz, ctx->d_sell_off, nslice + 1, s);
    int64_t total = 0;
    cudaMemcpyAsync(&total, ctx->d_sell_off + nslice, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    cudaFree(tmp);
    cudaFree(wsz);
    if (e != cudaSuccess) return gf_cuda_fail(ctx, e, "SELL layout");
    ctx->sell_nslice = nslice;
    ctx->sell_nslots = nslots;
    ctx->sell_total = total;
    ctx->sell_bdim = bdim;
    if ((st = gf_alloc(ctx, &ctx->d_sell_col, (size_t)std::max<int64_t>(total, 1))) != GF_OK) return st;
    if (bdim)
      k_bsell_col<<<gf_blocks(nslots, 256), 256, 0, s>>>(n, ctx->nnodes, bdim, nslots,
                                                         ctx->d_sell_off, ctx->d_sell_w,
                                                         ctx->d_rownnz, ctx->d_colidx,
                                                         ctx->d_sell_perm, ctx->d_sell_col);
    else
      k_sell_fill<int32_t, int32_t><<<gf_blocks(nslots, 256), 256, 0, s>>>(
          n, nslots, ctx->d_sell_off, ctx->d_sell_w, ctx->d_rownnz, ctx->d_colidx,
          ctx->d_sell_col, 1);
    GF_LAUNCH_CHECK(ctx, "slice columns");
    ctx->sell_ready = true;
  }
  const int64_t per = bdim ? (int64_t)bdim * bdim : 1;  // values per stored column word
  const size_t total = (size_t)std::max<int64_t>(ctx->sell_total * per, 1);
  const int nslots = ctx->sell_nslots;
  if (dtype == GF_F64 && ctx->sell_ver64 != ctx->kver64) {
    if (!ctx->d_sell_v64 && (st = gf_alloc(ctx, &ctx->d_sell_v64, total)) != GF_OK) return st;
    if (bdim)
      (bdim == 2 ? k_bsell_val<double, double, 2> : k_bsell_val<double, double, 3>)
          <<<gf_blocks(nslots, kWin), kWin, 0, s>>>(n, ctx->nnodes, nslots, ctx->d_sell_off,
                                                   ctx->d_sell_w, ctx->d_rownnz,
                                                   ctx->d_sell_perm, ctx->d_K64, ctx->d_sell_v64);
    else
      k_sell_fill<double, double><<<gf_blocks(nslots, 256), 256, 0, s>>>(
          n, nslots, ctx->d_sell_off, ctx->d_sell_w, ctx->d_rownnz, ctx->d_K64,
          ctx->d_sell_v64, 0);
    GF_LAUNCH_CHECK(ctx, "slice values (f64)");
    ctx->sell_ver64 = ctx->kver64;
  }
  if (dtype == GF_F32 && ctx->sell_ver32 != ctx->kver32) {
    if (!ctx->d_sell_v32 && (st = gf_alloc(ctx, &ctx->d_sell_v32, total)) != GF_OK) return st;
    if (bdim)
      (bdim == 2 ? k_bsell_val<float, float, 2> : k_bsell_val<float, float, 3>)
          <<<gf_blocks(nslots, kWin), kWin, 0, s>>>(n, ctx->nnodes, nslots, ctx->d_sell_off,
                                                   ctx->d_sell_w, ctx->d_rownnz,
                                                   ctx->d_sell_perm, ctx->d_K32, ctx->d_sell_v32);
    else
      k_sell_fill<float, float><<<gf_blocks(nslots, 256), 256, 0, s>>>(
          n, nslots, ctx->d_sell_off, ctx->d_sell_w, ctx->d_rownnz, ctx->d_K32,
          ctx->d_sell_v32, 0);
    GF_LAUNCH_CHECK(ctx, "slice values (f32)");
    ctx->sell_ver32 = ctx->kver32;
  }
  return GF_OK;
}
