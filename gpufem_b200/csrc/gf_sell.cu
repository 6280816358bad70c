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

}  // namespace

void gf_sell_free(gf_ctx* ctx) {
  gf_free(ctx->d_sell_off);
  gf_free(ctx->d_sell_w);
  gf_free(ctx->d_sell_col);
  gf_free(ctx->d_sell_v64);
  gf_free(ctx->d_sell_v32);
  ctx->sell_ready = false;
  ctx->sell_ver64 = ctx->sell_ver32 = -1;
  ctx->sell_total = 0;
}

// Builds the SELL pattern if needed and refreshes the values of `dtype`.
gf_status gf_sell_prepare(gf_ctx* ctx, int dtype) {
  const int n = ctx->n;
  cudaStream_t s = ctx->stream;
  gf_status st;
  if (!ctx->sell_ready) {
    gf_sell_free(ctx);
    const int nslice = (n + 31) / 32;
    const int nslots = nslice * 32;
    int64_t* wsz = nullptr;
    void* tmp = nullptr;
    size_t tb = 0;
    if ((st = gf_alloc(ctx, &ctx->d_sell_off, (size_t)nslice + 1)) != GF_OK) return st;
    if ((st = gf_alloc(ctx, &ctx->d_sell_w, (size_t)nslice)) != GF_OK) return st;
    if ((st = gf_alloc(ctx, &wsz, (size_t)nslice + 1)) != GF_OK) return st;
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
    if ((st = gf_alloc(ctx, &ctx->d_sell_col, (size_t)std::max<int64_t>(total, 1))) != GF_OK) return st;
    k_sell_fill<int32_t, int32_t><<<gf_blocks(nslots, 256), 256, 0, s>>>(
        n, nslots, ctx->d_sell_off, ctx->d_sell_w, ctx->d_rownnz, ctx->d_colidx,
        ctx->d_sell_col, 1);
    GF_LAUNCH_CHECK(ctx, "k_sell_fill(col)");
    ctx->sell_ready = true;
  }
  const size_t total = (size_t)std::max<int64_t>(ctx->sell_total, 1);
  if (dtype == GF_F64 && ctx->sell_ver64 != ctx->kver64) {
    if (!ctx->d_sell_v64 && (st = gf_alloc(ctx, &ctx->d_sell_v64, total)) != GF_OK) return st;
    k_sell_fill<double, double><<<gf_blocks(ctx->sell_nslots, 256), 256, 0, s>>>(
        n, ctx->sell_nslots, ctx->d_sell_off, ctx->d_sell_w, ctx->d_rownnz, ctx->d_K64,
        ctx->d_sell_v64, 0);
    GF_LAUNCH_CHECK(ctx, "k_sell_fill(f64)");
    ctx->sell_ver64 = ctx->kver64;
  }
  if (dtype == GF_F32 && ctx->sell_ver32 != ctx->kver32) {
    if (!ctx->d_sell_v32 && (st = gf_alloc(ctx, &ctx->d_sell_v32, total)) != GF_OK) return st;
    k_sell_fill<float, float><<<gf_blocks(ctx->sell_nslots, 256), 256, 0, s>>>(
        n, ctx->sell_nslots, ctx->d_sell_off, ctx->d_sell_w, ctx->d_rownnz, ctx->d_K32,
        ctx->d_sell_v32, 0);
    GF_LAUNCH_CHECK(ctx, "k_sell_fill(f32)");
    ctx->sell_ver32 = ctx->kver32;
  }
  return GF_OK;
}
