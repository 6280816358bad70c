// Element colouring on the device (Jones–Plassmann with first-fit colours).
//
// The colour schedule of the assembly needs a colouring of the element dual graph
// (elements sharing a node are adjacent).  The reference builds that graph with METIS
// and colours it greedily on the host (femColor::makeMetisGraph / MakeGreedyColoring,
// src/FEM/femColor.cc:79-191); gf_mesh_color reproduces that greedy order on the
// host.  This file colours on the GPU instead: every element gets a pseudo-random
// priority; in each round, an uncoloured element whose priority beats every
// uncoloured neighbour takes the smallest colour no coloured neighbour holds.  The
// elements that colour in one round form an independent set, so a round never
// races with itself; every round colours at least the element of highest priority
// left.  The dual graph is never built: neighbours are walked through the node ->
// element incidence lists of the pattern.
#include <cub/cub.cuh>
#include <algorithm>

#include "gf_internal.cuh"

namespace {

constexpr int kCT = 256;
constexpr int kColorWords = 4;  // up to 256 colours

__device__ inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__device__ inline bool beats(uint64_t pa, int a, uint64_t pb, int b) {
  return pa > pb || (pa == pb && a > b);
}

__global__ void __launch_bounds__(kCT)
k_jp_round(int nelem, int nen, uint64_t seed, const int32_t* __restrict__ conn,
           const int32_t* __restrict__ inc_off, const int32_t* __restrict__ inc,
           int32_t* __restrict__ color, int32_t* __restrict__ remaining,
           int32_t* __restrict__ overflow) {
  const int e = blockIdx.x * kCT + threadIdx.x;
  if (e >= nelem) return;
  if (color[e] >= 0) return;
  const uint64_t pe = splitmix64((uint64_t)e ^ seed);
  uint64_t used[kColorWords] = {0, 0, 0, 0};
  for (int i = 0; i < nen; ++i) {
    const int a = conn[(int64_t)e * nen + i];
    for (int q = inc_off[a]; q < inc_off[a + 1]; ++q) {
      const int f = inc[q];
      if (f == e) continue;
      const int cf = *(volatile const int32_t*)(color + f);
      if (cf < 0) {
        if (beats(splitmix64((uint64_t)f ^ seed), f, pe, e)) {
          atomicAdd(remaining, 1);  // e waits for a later round
          return;
        }
      } else if (cf < 64 * kColorWords) {
        used[cf >> 6] |= 1ull << (cf & 63);
      }
    }
  }
  int c = -1;
  for (int w = 0; w < kColorWords && c < 0; ++w)
    if (~used[w]) c = 64 * w + __ffsll((long long)~used[w]) - 1;
  if (c < 0) {
    atomicExch(overflow, 1);
    return;
  }
  color[e] = c;
}

__global__ void k_iota_elems(int n, int32_t* __restrict__ p) {
  const int i = blockIdx.x * kCT + threadIdx.x;
  if (i < n) p[i] = i;
}

}  // namespace

extern "C" GF_API gf_status gf_mesh_color_device(gf_ctx* ctx, uint64_t seed, int32_t* ncolors) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (!ctx->has_mesh) return gf_fail(ctx, GF_ERR_STATE, "no mesh");
  cudaSetDevice(ctx->device);
  gf_status st;
  if (!ctx->d_inc_off && (st = gf_pattern_build(ctx)) != GF_OK) return st;
  const int nelem = ctx->nelem;
  cudaStream_t s = ctx->stream;
  int32_t *d_color = nullptr, *d_flags = nullptr, *d_keys = nullptr, *d_ids = nullptr,
          *d_perm = nullptr;
  void* d_tmp = nullptr;
  auto cleanup = [&]() {
    gf_free(d_color); gf_free(d_flags); gf_free(d_keys); gf_free(d_ids); gf_free(d_perm);
    if (d_tmp) cudaFree(d_tmp);
  };
  if ((st = gf_alloc(ctx, &d_color, (size_t)nelem)) != GF_OK ||
      (st = gf_alloc(ctx, &d_flags, 2)) != GF_OK || (st = gf_alloc(ctx, &d_keys, (size_t)nelem)) != GF_OK ||
      (st = gf_alloc(ctx, &d_ids, (size_t)nelem)) != GF_OK ||
      (st = gf_alloc(ctx, &d_perm, (size_t)nelem)) != GF_OK) {
    cleanup();
    return st;
  }
  cudaMemsetAsync(d_color, 0xff, sizeof(int32_t) * nelem, s);  // -1
  int32_t h_flags[2] = {0, 0};
  int rounds = 0;
  for (;;) {
    cudaMemsetAsync(d_flags, 0, 2 * sizeof(int32_t), s);
    k_jp_round<<<gf_blocks(nelem, kCT), kCT, 0, s>>>(nelem, ctx->nen, seed, ctx->d_conn,
                                                   ctx->d_inc_off, ctx->d_inc, d_color, d_flags,
                                                   d_flags + 1);
    ctx->launches++;
    cudaMemcpyAsync(h_flags, d_flags, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      cleanup();
      return gf_cuda_fail(ctx, e, "colouring round");
    }
    ++rounds;
    if (h_flags[1]) {
      cleanup();
      return gf_fail(ctx, GF_ERR_UNSUPPORTED, "more than %d colours", 64 * kColorWords);
    }
    if (h_flags[0] == 0) break;
    if (rounds > nelem) {  // cannot happen: each round colours the top-priority element
      cleanup();
      return gf_fail(ctx, GF_ERR_CUDA, "colouring made no progress");
    }
  }
  // elements ordered by colour, ascending ids within a colour (stable radix sort)
  std::vector<int32_t> h_color(nelem);
  cudaMemcpyAsync(h_color.data(), d_color, sizeof(int32_t) * nelem, cudaMemcpyDeviceToHost, s);
  k_iota_elems<<<gf_blocks(nelem, kCT), kCT, 0, s>>>(nelem, d_ids);
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, d_color, d_keys, d_ids, d_perm, nelem, 0, 9, s);
  if (cudaMalloc(&d_tmp, tb) != cudaSuccess) {
    cudaGetLastError();
    cleanup();
    return gf_fail(ctx, GF_ERR_OOM, "colour sort scratch");
  }
  cub::DeviceRadixSort::SortPairs(d_tmp, tb, d_color, d_keys, d_ids, d_perm, nelem, 0, 9, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    cleanup();
    return gf_cuda_fail(ctx, e, "colour sort");
  }
  int ncol = 0;
  for (int k = 0; k < nelem; ++k) ncol = std::max(ncol, h_color[k] + 1);
  std::vector<int32_t> coff(ncol + 1, 0);
  for (int k = 0; k < nelem; ++k) coff[h_color[k] + 1]++;
  for (int c = 0; c < ncol; ++c) coff[c + 1] += coff[c];
  gf_free(ctx->d_perm);
  ctx->d_perm = d_perm;
  d_perm = nullptr;
  ctx->h_color = std::move(h_color);
  ctx->color_off = coff;
  ctx->ncolors = ncol;
  cleanup();
  if (ncolors) *ncolors = ncol;
  return GF_OK;
}
