// C-ABI entry points: context, mesh upload (FemData::Init), colouring, matrix
// views/transfers, loads and constraints.  Kernels live in gf_pattern.cu,
// gf_assemble.cu and gf_solve.cu.
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <algorithm>
#include <thread>
#if defined(__x86_64__)
#include <emmintrin.h>
#endif

#include "gf_internal.cuh"

gf_status gf_fail(gf_ctx* ctx, gf_status st, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return st;
}

gf_status gf_cuda_fail(gf_ctx* ctx, cudaError_t e, const char* where) {
  return gf_fail(ctx, e == cudaErrorMemoryAllocation ? GF_ERR_OOM : GF_ERR_CUDA,
                 "CUDA error in %s: %s", where, cudaGetErrorString(e));
}

extern "C" {

GF_API const char* gf_version(void) { return "gpufem_b200 0.1 (sm_100a)"; }

GF_API gf_status gf_create(gf_ctx** out, int32_t device) {
  if (!out) return GF_ERR_INVALID_ARG;
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return GF_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) return GF_ERR_INVALID_ARG;
  gf_ctx* ctx = new gf_ctx();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess ||
      cudaEventCreate(&ctx->evm) != cudaSuccess) {
    cudaGetLastError();
    delete ctx;
    return GF_ERR_CUDA;
  }
  cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
  *out = ctx;
  return GF_OK;
}

GF_API gf_status gf_destroy(gf_ctx* ctx) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  gf_lp_free(ctx);
  gf_coarse_free(ctx);
  gf_dist_free(ctx);
  gf_solver_free(ctx);
  gf_pattern_free(ctx);
  gf_mesh_free(ctx);
  gf_pfree(ctx, ctx->d_f);
  gf_pfree(ctx, ctx->d_fixed);
  if (ctx->d_geo) cudaFree(ctx->d_geo);
  gf_free(ctx->d_asm_err);
  gf_free(ctx->d_gram);
  gf_pool_clear(ctx);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->evm) cudaEventDestroy(ctx->evm);
  if (ctx->ev_dl) cudaEventDestroy(ctx->ev_dl);
  if (ctx->h_adj_stage) cudaFreeHost(ctx->h_adj_stage);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return GF_OK;
}

GF_API const char* gf_last_error(const gf_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }
GF_API double gf_last_device_seconds(const gf_ctx* ctx) { return ctx ? ctx->last_seconds : 0.0; }
GF_API int64_t gf_kernel_launches(const gf_ctx* ctx) { return ctx ? ctx->launches : 0; }

GF_API gf_status gf_last_assembly_split(const gf_ctx* ctx, double* geometry_seconds,
                                        double* scatter_seconds) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (geometry_seconds) *geometry_seconds = ctx->last_split[0];
  if (scatter_seconds) *scatter_seconds = ctx->last_split[1];
  return GF_OK;
}

GF_API gf_status gf_sync(gf_ctx* ctx) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GF_OK;
}

GF_API gf_status gf_stream(gf_ctx* ctx, void** stream) {
  if (!ctx || !stream) return GF_ERR_INVALID_ARG;
  *stream = (void*)ctx->stream;
  return GF_OK;
}

}  // extern "C"

void gf_mesh_free(gf_ctx* ctx) {
  gf_pfree(ctx, ctx->d_coords64);
  gf_pfree(ctx, ctx->d_coords32);
  gf_pfree(ctx, ctx->d_conn);
  gf_pfree(ctx, ctx->d_Eel);
  gf_pfree(ctx, ctx->d_Eel32);
  gf_free(ctx->d_asmtab);
  gf_free(ctx->d_perm);
  gf_pfree(ctx, ctx->d_allperm);
  ctx->h_conn.clear();
  ctx->h_color.clear();
  ctx->color_off.clear();
  ctx->ncolors = 0;
  ctx->has_mesh = false;
}

void gf_pattern_free(gf_ctx* ctx) {
  gf_pfree(ctx, ctx->d_rownnz);
  gf_pfree(ctx, ctx->d_colidx);
  gf_pfree(ctx, ctx->d_slotmap);
  gf_pfree(ctx, ctx->d_adj_off);
  gf_pfree(ctx, ctx->d_adj);
  gf_pfree(ctx, ctx->d_diagpos);
  gf_pfree(ctx, ctx->d_inc_off);
  gf_pfree(ctx, ctx->d_inc);
  gf_pfree(ctx, ctx->d_inc_loc);
  gf_pfree(ctx, ctx->d_inc_slot);
  ctx->maxval = 0;  // the geometry buffer keeps its capacity (freed by gf_destroy)
  gf_pfree(ctx, ctx->d_K64);
  gf_pfree(ctx, ctx->d_K32);
  gf_sell_free(ctx);
  // n (the dof count) belongs to the mesh and survives; width and nnz do not
  ctx->has_pattern = ctx->has64 = ctx->has32 = false;
  ctx->W = 0;
  ctx->nnz = 0;
}

static __global__ void k_f64_to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (; i < n; i += stride) b[i] = (float)a[i];
}

static __global__ void k_iota(int n, int32_t* p) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = i;
}

// ---- device buffer pool --------------------------------------------------------
void* gf_pool_get(gf_ctx* ctx, size_t bytes) {
  for (size_t k = 0; k < ctx->pool_free.size(); ++k)
    if (ctx->pool_free[k].bytes == bytes) {
      void* p = ctx->pool_free[k].p;
      ctx->pool_free.erase(ctx->pool_free.begin() + (ptrdiff_t)k);
      ctx->pool_live.emplace_back(p, bytes);
      return p;
    }
  void* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    for (auto& b : ctx->pool_free) cudaFree(b.p);  // give unused blocks back, retry once
    ctx->pool_free.clear();
    p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
  }
  ctx->pool_live.emplace_back(p, bytes);
  return p;
}

void gf_pool_put(gf_ctx* ctx, void* p) {
  for (size_t k = 0; k < ctx->pool_live.size(); ++k)
    if (ctx->pool_live[k].first == p) {
      ctx->pool_free.push_back({p, ctx->pool_live[k].second, ctx->pool_gen});
      ctx->pool_live.erase(ctx->pool_live.begin() + (ptrdiff_t)k);
      return;
    }
  cudaFree(p);  // not from the pool
}

void gf_pool_new_generation(gf_ctx* ctx) {
  ++ctx->pool_gen;
  std::vector<gf_ctx::PoolBlock> keep;
  for (auto& b : ctx->pool_free) {
    if (b.gen >= ctx->pool_gen - 1) keep.push_back(b);
    else cudaFree(b.p);
  }
  ctx->pool_free.swap(keep);
}

void gf_pool_clear(gf_ctx* ctx) {
  for (auto& b : ctx->pool_free) cudaFree(b.p);
  for (auto& b : ctx->pool_live) cudaFree(b.first);
  ctx->pool_free.clear();
  ctx->pool_live.clear();
}

// ---- mesh validation on the device ------------------------------------------------
// chk[0]: smallest index of a non-finite coordinate; chk[1]: smallest connectivity
// entry outside 1..nnodes; chk[2]: smallest element repeating a node; chk[3]: smallest
// element whose modulus is not finite and > 0.  All start at ~0 (none).
static __global__ void k_mesh_check(int64_t ncoord, const double* __restrict__ coords,
                                    int nelem, int nen, int nnodes, int32_t* __restrict__ conn,
                                    unsigned long long* __restrict__ chk) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ncoord; i += stride)
    if (!isfinite(coords[i])) atomicMin(&chk[0], (unsigned long long)i);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nelem; e += stride) {
    int32_t v[GF_MAX_NEN];
    bool ok = true;
    for (int a = 0; a < nen; ++a) {
      v[a] = conn[e * nen + a];
      if (v[a] < 1 || v[a] > nnodes) {
        atomicMin(&chk[1], (unsigned long long)(e * nen + a));
        ok = false;
      }
    }
    for (int a = 0; a < nen && ok; ++a)
      for (int b = a + 1; b < nen; ++b)
        if (v[a] == v[b]) {
          atomicMin(&chk[2], (unsigned long long)e);
          ok = false;
          break;
        }
    for (int a = 0; a < nen; ++a) conn[e * nen + a] = v[a] - 1;  // 0-based
  }
}

// Eel <- E_elem (already copied to Eel) or the scalar E, FP32 copy, validity in chk[3].
static __global__ void k_modulus(int nelem, int per_elem, double E, double* __restrict__ Eel,
                                 float* __restrict__ Eel32, unsigned long long* __restrict__ chk) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nelem) return;
  const double v = per_elem ? Eel[i] : E;
  if (!(v > 0.0) || !isfinite(v)) atomicMin(&chk[3], (unsigned long long)i);
  Eel[i] = v;
  Eel32[i] = (float)v;
}

// The first failed check, in the order coordinates, connectivity range, repeated
// nodes, moduli, as a status and message (values read from the caller's arrays).
static gf_status check_failure(gf_ctx* ctx, const unsigned long long* chk, int nen,
                               int nnodes, const int32_t* connect, double E,
                               const double* E_elem) {
  const unsigned long long none = ~0ull;
  if (chk[0] != none)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "non-finite coordinate at %llu", chk[0]);
  if (chk[1] != none)
    return gf_fail(ctx, GF_ERR_INVALID_ARG,
                   "connectivity entry %llu = %d outside 1..%d (1-based node ids)", chk[1],
                   connect[chk[1]], nnodes);
  if (chk[2] != none) {
    const size_t e = (size_t)chk[2];
    int rep = 0;
    for (int a = 0; a < nen && !rep; ++a)
      for (int b = a + 1; b < nen; ++b)
        if (connect[e * nen + a] == connect[e * nen + b]) { rep = connect[e * nen + a]; break; }
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "element %zu repeats node %d", e, rep);
  }
  if (chk[3] != none)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "modulus of element %llu is %g (must be > 0)",
                   chk[3], E_elem ? E_elem[chk[3]] : E);
  return GF_OK;
}

namespace {
template <typename T>
__global__ void k_ell_diag(int n, const int32_t* __restrict__ rownnz,
                           const int32_t* __restrict__ col, const T* __restrict__ val,
                           double* __restrict__ diag) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  double d = 0.0;
  for (int s = 0; s < rownnz[row]; ++s)
    if (col[(int64_t)s * n + row] == row) d = (double)val[(int64_t)s * n + row];
  diag[row] = d;
}
}  // namespace

extern "C" {

GF_API gf_status gf_mesh_create(gf_ctx* ctx, int32_t elem_type, int32_t nnodes,
                                const double* coords, int32_t nelem, const int32_t* connect,
                                int32_t ngauss, double E, const double* E_elem, double nu,
                                int32_t analysis) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  if (elem_type < GF_Q4 || elem_type > GF_BRICK20)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "unknown element type %d", elem_type);
  if (nnodes <= 0 || nelem <= 0 || !coords || !connect)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "empty mesh or null arrays");
  if (ngauss != 2 && ngauss != 3)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "ngauss must be 2 or 3 (got %d)", ngauss);
  if (!(nu > -1.0 && nu < 0.5))
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "Poisson ratio %g outside (-1, 0.5)", nu);
  if (analysis != GF_PLANE_STRESS && analysis != GF_PLANE_STRAIN)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "unknown analysis %d", analysis);
  const ElemInfo info = gf_elem_info(elem_type);
  if ((int64_t)nnodes * info.dim >= (int64_t)INT32_MAX)
    return gf_fail(ctx, GF_ERR_UNSUPPORTED, "too many dofs for int32 indexing");
  if ((int64_t)nelem * info.nen >= (int64_t)INT32_MAX)
    return gf_fail(ctx, GF_ERR_UNSUPPORTED, "too many element-node entries for int32 indexing");

  // The new mesh goes into fresh buffers and is validated on the device (one round
  // trip); the current mesh is released only once the new one is accepted.
  cudaStream_t s = ctx->stream;
  cudaStreamSynchronize(s);
  gf_pool_new_generation(ctx);
  const size_t ncoord = (size_t)nnodes * info.dim;
  const size_t nconn = (size_t)nelem * info.nen;
  const int n = nnodes * info.dim;
  double* coords64 = nullptr;
  float* coords32 = nullptr;
  int32_t *conn = nullptr, *allperm = nullptr;
  double* Eel = nullptr;
  float* Eel32 = nullptr;
  double* f = nullptr;
  uint8_t* fixed = nullptr;
  unsigned long long* d_chk = nullptr;
  auto release = [&]() {
    gf_pfree(ctx, coords64); gf_pfree(ctx, coords32); gf_pfree(ctx, conn);
    gf_pfree(ctx, allperm); gf_pfree(ctx, Eel); gf_pfree(ctx, Eel32); gf_pfree(ctx, f);
    gf_pfree(ctx, fixed); gf_pfree(ctx, d_chk);
  };
  gf_status st;
  if ((st = gf_palloc(ctx, &coords64, ncoord)) != GF_OK ||
      (st = gf_palloc(ctx, &coords32, ncoord)) != GF_OK ||
      (st = gf_palloc(ctx, &conn, nconn)) != GF_OK ||
      (st = gf_palloc(ctx, &allperm, (size_t)nelem)) != GF_OK ||
      (st = gf_palloc(ctx, &Eel, (size_t)nelem)) != GF_OK ||
      (st = gf_palloc(ctx, &Eel32, (size_t)nelem)) != GF_OK ||
      (st = gf_palloc(ctx, &f, (size_t)n)) != GF_OK ||
      (st = gf_palloc(ctx, &fixed, (size_t)n)) != GF_OK ||
      (st = gf_palloc(ctx, &d_chk, 4)) != GF_OK) {
    release();
    return st;
  }
  unsigned long long h_chk[4];
  cudaMemcpyAsync(coords64, coords, sizeof(double) * ncoord, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(conn, connect, sizeof(int32_t) * nconn, cudaMemcpyHostToDevice, s);
  if (E_elem) cudaMemcpyAsync(Eel, E_elem, sizeof(double) * nelem, cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(d_chk, 0xff, 4 * sizeof(unsigned long long), s);
  const int cblocks = (int)std::min<int64_t>(gf_blocks(std::max<int64_t>(ncoord, nelem), 256),
                                             (int64_t)ctx->sm_count * 8);
  k_mesh_check<<<cblocks, 256, 0, s>>>((int64_t)ncoord, coords64, nelem, info.nen, nnodes, conn,
                                       d_chk);
  k_modulus<<<gf_blocks(nelem, 256), 256, 0, s>>>(nelem, E_elem ? 1 : 0, E, Eel, Eel32, d_chk);
  k_f64_to_f32<<<gf_blocks(ncoord, 256), 256, 0, s>>>((int64_t)ncoord, coords64, coords32);
  k_iota<<<gf_blocks(nelem, 256), 256, 0, s>>>(nelem, allperm);
  cudaMemsetAsync(f, 0, sizeof(double) * n, s);
  cudaMemsetAsync(fixed, 0, n, s);
  ctx->launches += 4;
  cudaMemcpyAsync(h_chk, d_chk, sizeof(h_chk), cudaMemcpyDeviceToHost, s);
  cudaError_t ce = cudaStreamSynchronize(s);
  if (ce == cudaSuccess) ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    release();
    return gf_cuda_fail(ctx, ce, "mesh upload");
  }
  if ((st = check_failure(ctx, h_chk, info.nen, nnodes, connect, E, E_elem)) != GF_OK) {
    release();
    return st;
  }

  // accepted: drop the current mesh and everything built on it
  gf_solver_free(ctx);
  gf_pattern_free(ctx);
  gf_mesh_free(ctx);
  gf_lp_mesh_changed(ctx);
  gf_coarse_free(ctx);
  gf_pfree(ctx, ctx->d_f);
  gf_pfree(ctx, ctx->d_fixed);
  gf_pfree(ctx, d_chk);
  ctx->h_supports.clear();
  ctx->nsup = 0;
  ctx->bc_mode_applied = -1;

  ctx->elem_type = elem_type;
  ctx->dim = info.dim;
  ctx->nen = info.nen;
  ctx->ngauss = ngauss;
  ctx->ngp = info.dim == 2 ? ngauss * ngauss : ngauss * ngauss * ngauss;
  ctx->nnodes = nnodes;
  ctx->nelem = nelem;
  ctx->analysis = analysis;
  ctx->nu = nu;
  ctx->E = E;
  // Per unit modulus: Ke = sum_gp w detJ E [lam1 g_i g_j^T + mu1 g_j g_i^T + mu1 (g_i.g_j) I]
  // which equals B^T D B for the reference's D (FemData.cc:322-365):
  //   plane stress: D = E/(1-nu^2) [[1, nu, 0], [nu, 1, 0], [0, 0, (1-nu)/2]]
  //   plane strain / 3-D: lam = E nu / ((1+nu)(1-2nu)), mu = E / (2(1+nu))
  if (info.dim == 2 && analysis == GF_PLANE_STRESS) {
    double c1 = 1.0 / (1.0 - nu * nu);
    ctx->lam1 = c1 * nu;
    ctx->mu1 = c1 * (1.0 - nu) / 2.0;
  } else {
    ctx->lam1 = nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    ctx->mu1 = 1.0 / (2.0 * (1.0 + nu));
  }
  ctx->n = n;
  ctx->d_coords64 = coords64;
  ctx->d_coords32 = coords32;
  ctx->d_conn = conn;
  ctx->d_allperm = allperm;
  ctx->d_Eel = Eel;
  ctx->d_Eel32 = Eel32;
  ctx->d_f = f;
  ctx->d_fixed = fixed;
  ctx->h_f.clear();   // f = 0 (an empty host copy stands for zeros)
  ctx->has_mesh = true;
  return GF_OK;
}

GF_API gf_status gf_mesh_set_modulus(gf_ctx* ctx, double E, const double* E_elem) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (!ctx->has_mesh) return gf_fail(ctx, GF_ERR_STATE, "no mesh");
  cudaSetDevice(ctx->device);
  // into fresh buffers first, so that an invalid modulus leaves the current one
  const int nelem = ctx->nelem;
  cudaStream_t s = ctx->stream;
  double* Eel = nullptr;
  float* Eel32 = nullptr;
  unsigned long long* d_chk = nullptr;
  unsigned long long h_chk[4];
  gf_status st;
  auto release = [&]() { gf_pfree(ctx, Eel); gf_pfree(ctx, Eel32); gf_pfree(ctx, d_chk); };
  if ((st = gf_palloc(ctx, &Eel, (size_t)nelem)) != GF_OK ||
      (st = gf_palloc(ctx, &Eel32, (size_t)nelem)) != GF_OK ||
      (st = gf_palloc(ctx, &d_chk, 4)) != GF_OK) {
    release();
    return st;
  }
  cudaMemsetAsync(d_chk, 0xff, 4 * sizeof(unsigned long long), s);
  if (E_elem) cudaMemcpyAsync(Eel, E_elem, sizeof(double) * nelem, cudaMemcpyHostToDevice, s);
  k_modulus<<<gf_blocks(nelem, 256), 256, 0, s>>>(nelem, E_elem ? 1 : 0, E, Eel, Eel32, d_chk);
  ctx->launches++;
  cudaMemcpyAsync(h_chk, d_chk, sizeof(h_chk), cudaMemcpyDeviceToHost, s);
  cudaError_t ce = cudaStreamSynchronize(s);
  if (ce == cudaSuccess) ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    release();
    return gf_cuda_fail(ctx, ce, "modulus upload");
  }
  if ((st = check_failure(ctx, h_chk, ctx->nen, ctx->nnodes, nullptr, E, E_elem)) != GF_OK) {
    release();
    return st;
  }
  gf_pfree(ctx, d_chk);
  gf_pfree(ctx, ctx->d_Eel);
  gf_pfree(ctx, ctx->d_Eel32);
  ctx->d_Eel = Eel;
  ctx->d_Eel32 = Eel32;
  ctx->E = E;
  return GF_OK;
}

GF_API gf_status gf_mesh_color(gf_ctx* ctx, const int32_t* elem_color, int32_t* ncolors) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (!ctx->has_mesh) return gf_fail(ctx, GF_ERR_STATE, "no mesh");
  cudaSetDevice(ctx->device);
  gf_status st = gf_color_build(ctx, elem_color);
  if (st != GF_OK) return st;
  if (ncolors) *ncolors = ctx->ncolors;
  return GF_OK;
}

GF_API gf_status gf_mesh_get_colors(gf_ctx* ctx, int32_t* elem_color) {
  if (!ctx || !elem_color) return GF_ERR_INVALID_ARG;
  if (ctx->ncolors == 0) return gf_fail(ctx, GF_ERR_STATE, "mesh not coloured");
  std::memcpy(elem_color, ctx->h_color.data(), sizeof(int32_t) * ctx->nelem);
  return GF_OK;
}

GF_API gf_status gf_ell_build_pattern(gf_ctx* ctx, int32_t* n, int32_t* width, int64_t* nnz) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (!ctx->has_mesh) return gf_fail(ctx, GF_ERR_STATE, "no mesh");
  cudaSetDevice(ctx->device);
  gf_status st = gf_pattern_build(ctx);
  if (st != GF_OK) return st;
  if (n) *n = ctx->n;
  if (width) *width = ctx->W;
  if (nnz) *nnz = ctx->nnz;
  return GF_OK;
}

GF_API gf_status gf_assemble(gf_ctx* ctx, int32_t dtype, int32_t scatter, int32_t engine) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (!ctx->has_mesh) return gf_fail(ctx, GF_ERR_STATE, "no mesh");
  if (dtype != GF_F64 && dtype != GF_F32)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "unknown dtype %d", dtype);
  if (scatter < GF_SCATTER_COLOR || scatter > GF_SCATTER_AUTO)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "unknown scatter %d", scatter);
  if (engine != GF_ENGINE_CUDA_CORE && engine != GF_ENGINE_TF32_MMA)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "unknown engine %d", engine);
  if (scatter == GF_SCATTER_AUTO)  // fastest measured schedule per element type (B200)
    scatter = (ctx->dim == 3 && engine != GF_ENGINE_TF32_MMA) ? GF_SCATTER_ATOMIC
                                                              : GF_SCATTER_OWNER;
  if (engine == GF_ENGINE_TF32_MMA && dtype != GF_F32)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "the TF32 engine assembles FP32 only");
  cudaSetDevice(ctx->device);
  gf_status st;
  if (!ctx->has_pattern && (st = gf_pattern_build(ctx)) != GF_OK) return st;
  if (scatter == GF_SCATTER_COLOR && ctx->ncolors == 0 &&
      (st = gf_color_build(ctx, nullptr)) != GF_OK)
    return st;
  return gf_assemble_launch(ctx, dtype, scatter, engine);
}

GF_API gf_status gf_ell_convert_f64_to_f32(gf_ctx* ctx) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (!ctx->has64) return gf_fail(ctx, GF_ERR_STATE, "no FP64 matrix");
  cudaSetDevice(ctx->device);
  gf_status st;
  const int64_t total = (int64_t)ctx->n * ctx->W;
  if (!ctx->d_K32 && (st = gf_palloc(ctx, &ctx->d_K32, (size_t)total)) != GF_OK) return st;
  k_f64_to_f32<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(total, ctx->d_K64, ctx->d_K32);
  GF_LAUNCH_CHECK(ctx, "k_f64_to_f32");
  ctx->has32 = true;
  ctx->kver32++;
  return GF_OK;
}

GF_API gf_status gf_ell_version(gf_ctx* ctx, int32_t dtype, int64_t* version) {
  if (!ctx || !version) return GF_ERR_INVALID_ARG;
  if (dtype != GF_F64 && dtype != GF_F32)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "unknown dtype %d", dtype);
  *version = dtype == GF_F64 ? ctx->kver64 : ctx->kver32;
  return GF_OK;
}

GF_API gf_status gf_ell_view(gf_ctx* ctx, int32_t dtype, int32_t* n, int32_t* width,
                             const int32_t** rownnz, const int32_t** colidx,
                             const void** values) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (!ctx->has_pattern) return gf_fail(ctx, GF_ERR_STATE, "no matrix");
  if (n) *n = ctx->n;
  if (width) *width = ctx->W;
  if (rownnz) *rownnz = ctx->d_rownnz;
  if (colidx) *colidx = ctx->d_colidx;
  if (values) {
    if (dtype == GF_F64) {
      if (!ctx->has64) return gf_fail(ctx, GF_ERR_STATE, "no FP64 matrix");
      *values = ctx->d_K64;
    } else if (dtype == GF_F32) {
      if (!ctx->has32) return gf_fail(ctx, GF_ERR_STATE, "no FP32 matrix");
      *values = ctx->d_K32;
    } else {
      return gf_fail(ctx, GF_ERR_INVALID_ARG, "unknown dtype %d", dtype);
    }
  }
  return GF_OK;
}

extern "C++" {
namespace {
// Column words go to the caller's buffer with non-temporal stores where the host has them
// (x86-64 movnti): the buffer is written once and not read back here, and plain stores
// would first read every line they fill (write-allocate), doubling the host memory
// traffic of the expansion.
#if defined(__x86_64__) && !defined(__CUDA_ARCH__)
inline void put_word(int32_t* p, int32_t v) { _mm_stream_si32(reinterpret_cast<int*>(p), v); }
inline void put_fence() { _mm_sfence(); }
#else
inline void put_word(int32_t* p, int32_t v) { *p = v; }
inline void put_fence() {}
#endif

// Row lengths and column indices of a mesh-built ELL pattern from its node adjacency: the
// rows of node a (components c) hold the dofs of a's sorted neighbour list, dim per
// neighbour, then col = row in the padding slots.  Nodes [a0, a1) in chunks whose lists
// stay in cache while the W slot columns of the column-major array are written.
template <int DIM>
void expand_pattern_dim(int n, int W, const int32_t* off, const int32_t* adj, int a0, int a1,
                        int32_t* rownnz, int32_t* colidx) {
  constexpr int kChunk = 2048;
  for (int c0 = a0; c0 < a1; c0 += kChunk) {
    const int c1 = std::min(a1, c0 + kChunk);
    if (rownnz)
      for (int a = c0; a < c1; ++a)
        for (int r = 0; r < DIM; ++r) rownnz[a * DIM + r] = (off[a + 1] - off[a]) * DIM;
    if (!colidx) continue;
    // neighbour k fills slots k * DIM + c of the node's DIM rows with its DIM dofs
    for (int k = 0; k < W / DIM; ++k) {
      int32_t* out[DIM];
      for (int c = 0; c < DIM; ++c) out[c] = colidx + (size_t)(k * DIM + c) * n;
      for (int a = c0; a < c1; ++a) {
        const int row = a * DIM;
        if (k < off[a + 1] - off[a]) {
          const int v = adj[off[a] + k] * DIM;
          for (int c = 0; c < DIM; ++c)
            for (int r = 0; r < DIM; ++r) put_word(out[c] + row + r, v + c);
        } else {
          for (int c = 0; c < DIM; ++c)
            for (int r = 0; r < DIM; ++r) put_word(out[c] + row + r, row + r);
        }
      }
    }
  }
  put_fence();   // the stores are visible before the caller's join
}

void expand_pattern(int n, int W, int dim, const int32_t* off, const int32_t* adj, int a0,
                    int a1, int32_t* rownnz, int32_t* colidx) {
  if (dim == 2) expand_pattern_dim<2>(n, W, off, adj, a0, a1, rownnz, colidx);
  else expand_pattern_dim<3>(n, W, off, adj, a0, a1, rownnz, colidx);
}
}  // namespace
}  // extern "C++"

GF_API gf_status gf_ell_download(gf_ctx* ctx, int32_t dtype, int32_t* rownnz, int32_t* colidx,
                                 void* values) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (!ctx->has_pattern) return gf_fail(ctx, GF_ERR_STATE, "no matrix");
  cudaSetDevice(ctx->device);
  const size_t total = (size_t)ctx->n * ctx->W;
  // A mesh-built pattern crosses PCIe as its node adjacency (1 / dim^2 of the column
  // words, Q8: 66 MB instead of 265 MB) and is expanded on host threads while the values
  // are copied.
  bool expand = false;
  const int nn = ctx->nnodes, dim = ctx->dim;
  const size_t nadj_total = ctx->dim > 0 ? (size_t)(ctx->nnz / ((int64_t)dim * dim)) : 0;
  if ((rownnz || colidx) && ctx->has_mesh && ctx->d_adj_off && ctx->d_adj && dim > 0 &&
      (int64_t)nn * dim == ctx->n) {
    const size_t need = (size_t)nn + 1 + nadj_total;
    if (ctx->h_adj_stage_n < need) {
      if (ctx->h_adj_stage) cudaFreeHost(ctx->h_adj_stage);
      ctx->h_adj_stage = nullptr;
      ctx->h_adj_stage_n = 0;
      if (cudaMallocHost(&ctx->h_adj_stage, sizeof(int32_t) * need) == cudaSuccess)
        ctx->h_adj_stage_n = need;
      else
        cudaGetLastError();   // no pinned staging: plain copies below
    }
    if (!ctx->ev_dl && cudaEventCreateWithFlags(&ctx->ev_dl, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      ctx->ev_dl = nullptr;
    }
    expand = ctx->h_adj_stage_n >= need && ctx->ev_dl;
  }
  if (expand) {
    GF_CUDA(ctx, cudaMemcpyAsync(ctx->h_adj_stage, ctx->d_adj_off, sizeof(int32_t) * (nn + 1),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    GF_CUDA(ctx, cudaMemcpyAsync(ctx->h_adj_stage + nn + 1, ctx->d_adj,
                                 sizeof(int32_t) * nadj_total, cudaMemcpyDeviceToHost,
                                 ctx->stream));
    GF_CUDA(ctx, cudaEventRecord(ctx->ev_dl, ctx->stream));
  } else {
    if (rownnz)
      GF_CUDA(ctx, cudaMemcpyAsync(rownnz, ctx->d_rownnz, sizeof(int32_t) * ctx->n,
                                   cudaMemcpyDeviceToHost, ctx->stream));
    if (colidx)
      GF_CUDA(ctx, cudaMemcpyAsync(colidx, ctx->d_colidx, sizeof(int32_t) * total,
                                   cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (values) {
    if (dtype == GF_F64) {
      if (!ctx->has64) return gf_fail(ctx, GF_ERR_STATE, "no FP64 matrix");
      GF_CUDA(ctx, cudaMemcpyAsync(values, ctx->d_K64, sizeof(double) * total,
                                   cudaMemcpyDeviceToHost, ctx->stream));
    } else if (dtype == GF_F32) {
      if (!ctx->has32) return gf_fail(ctx, GF_ERR_STATE, "no FP32 matrix");
      GF_CUDA(ctx, cudaMemcpyAsync(values, ctx->d_K32, sizeof(float) * total,
                                   cudaMemcpyDeviceToHost, ctx->stream));
    } else {
      return gf_fail(ctx, GF_ERR_INVALID_ARG, "unknown dtype %d", dtype);
    }
  }
  if (expand) {
    GF_CUDA(ctx, cudaEventSynchronize(ctx->ev_dl));
    const int32_t* off = ctx->h_adj_stage;
    const int32_t* adj = ctx->h_adj_stage + nn + 1;
    const unsigned hw = std::thread::hardware_concurrency();
    const int nthreads = total >= ((size_t)1 << 20) ? (int)std::min(16u, std::max(1u, hw)) : 1;
    if (nthreads == 1) {
      expand_pattern(ctx->n, ctx->W, dim, off, adj, 0, nn, rownnz, colidx);
    } else {
      std::vector<std::thread> pool;
      const int per = (nn + nthreads - 1) / nthreads;
      for (int t = 0; t < nthreads; ++t) {
        const int a0 = t * per, a1 = std::min(nn, a0 + per);
        if (a0 >= a1) break;
        pool.emplace_back(expand_pattern, ctx->n, ctx->W, dim, off, adj, a0, a1, rownnz, colidx);
      }
      for (auto& th : pool) th.join();
    }
  }
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GF_OK;
}


GF_API gf_status gf_ell_diagonal(gf_ctx* ctx, int32_t dtype, double* diag) {
  if (!ctx || !diag) return GF_ERR_INVALID_ARG;
  if (!ctx->has_pattern) return gf_fail(ctx, GF_ERR_STATE, "no matrix");
  if ((dtype == GF_F64 && !ctx->has64) || (dtype == GF_F32 && !ctx->has32) ||
      (dtype != GF_F64 && dtype != GF_F32))
    return gf_fail(ctx, GF_ERR_STATE, "matrix of dtype %d not assembled", dtype);
  cudaSetDevice(ctx->device);
  const int n = ctx->n;
  double* d = nullptr;
  gf_status st = gf_palloc(ctx, &d, (size_t)n);
  if (st != GF_OK) return st;
  if (dtype == GF_F64)
    k_ell_diag<double><<<gf_blocks(n, 256), 256, 0, ctx->stream>>>(n, ctx->d_rownnz, ctx->d_colidx,
                                                                   ctx->d_K64, d);
  else
    k_ell_diag<float><<<gf_blocks(n, 256), 256, 0, ctx->stream>>>(n, ctx->d_rownnz, ctx->d_colidx,
                                                                  ctx->d_K32, d);
  ctx->launches++;
  cudaError_t e = cudaMemcpyAsync(diag, d, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  gf_pfree(ctx, d);
  if (e != cudaSuccess) return gf_cuda_fail(ctx, e, "ELL diagonal");
  return GF_OK;
}

GF_API gf_status gf_ell_upload(gf_ctx* ctx, int32_t n, int32_t width, const int32_t* rownnz,
                               const int32_t* colidx, const double* values) {
  if (!ctx || n <= 0 || width <= 0 || !rownnz || !colidx || !values)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "bad ELL upload arguments");
  cudaSetDevice(ctx->device);
  // validate: row lengths within width, columns in range, strictly increasing
  const size_t total = (size_t)n * width;
  std::vector<int32_t> col(total);
  std::vector<double> val(total, 0.0);
  int64_t nnz = 0;
  for (int r = 0; r < n; ++r) {
    int nz = rownnz[r];
    if (nz < 0 || nz > width)
      return gf_fail(ctx, GF_ERR_INVALID_ARG, "rownnz[%d] = %d outside 0..%d", r, nz, width);
    nnz += nz;
    int prev = -1;
    for (int s = 0; s < width; ++s) {
      size_t o = (size_t)s * n + r;
      if (s < nz) {
        int c = colidx[o];
        if (c < 0 || c >= n)
          return gf_fail(ctx, GF_ERR_INVALID_ARG, "column %d of row %d out of range", c, r);
        if (c <= prev)
          return gf_fail(ctx, GF_ERR_INVALID_ARG, "columns of row %d not strictly increasing", r);
        prev = c;
        col[o] = c;
        val[o] = values[o];
      } else {
        col[o] = r;
      }
    }
  }
  // the uploaded matrix replaces any mesh-derived system (mesh, pattern, loads)
  cudaStreamSynchronize(ctx->stream);
  gf_solver_free(ctx);
  gf_pattern_free(ctx);
  gf_mesh_free(ctx);
  gf_lp_mesh_changed(ctx);
  gf_coarse_free(ctx);
  gf_pfree(ctx, ctx->d_f);
  gf_pfree(ctx, ctx->d_fixed);
  ctx->h_supports.clear();
  ctx->nsup = 0;
  ctx->bc_mode_applied = -1;
  gf_status st;
  ctx->n = n;
  ctx->W = width;
  ctx->nnz = nnz;
  if ((st = gf_palloc(ctx, &ctx->d_rownnz, (size_t)n)) != GF_OK) return st;
  if ((st = gf_palloc(ctx, &ctx->d_colidx, total)) != GF_OK) return st;
  if ((st = gf_palloc(ctx, &ctx->d_K64, total)) != GF_OK) return st;
  if ((st = gf_palloc(ctx, &ctx->d_K32, total)) != GF_OK) return st;
  if ((st = gf_palloc(ctx, &ctx->d_f, (size_t)n)) != GF_OK) return st;
  if ((st = gf_palloc(ctx, &ctx->d_fixed, (size_t)n)) != GF_OK) return st;
  ctx->h_f.clear();   // f = 0 (an empty host copy stands for zeros)
  GF_CUDA(ctx, cudaMemsetAsync(ctx->d_f, 0, sizeof(double) * n, ctx->stream));
  GF_CUDA(ctx, cudaMemsetAsync(ctx->d_fixed, 0, n, ctx->stream));
  GF_CUDA(ctx, cudaMemcpyAsync(ctx->d_rownnz, rownnz, sizeof(int32_t) * n,
                               cudaMemcpyHostToDevice, ctx->stream));
  GF_CUDA(ctx, cudaMemcpyAsync(ctx->d_colidx, col.data(), sizeof(int32_t) * total,
                               cudaMemcpyHostToDevice, ctx->stream));
  GF_CUDA(ctx, cudaMemcpyAsync(ctx->d_K64, val.data(), sizeof(double) * total,
                               cudaMemcpyHostToDevice, ctx->stream));
  k_f64_to_f32<<<gf_blocks(total, 256), 256, 0, ctx->stream>>>((int64_t)total, ctx->d_K64,
                                                                ctx->d_K32);
  GF_LAUNCH_CHECK(ctx, "k_f64_to_f32");
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->has_pattern = ctx->has64 = ctx->has32 = true;
  ctx->kver64++;
  ctx->kver32++;
  return GF_OK;
}

GF_API gf_status gf_set_supports(gf_ctx* ctx, int32_t nsup, const int32_t* supports) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (!ctx->has_mesh) return gf_fail(ctx, GF_ERR_STATE, "no mesh");
  if (nsup < 0 || (nsup > 0 && !supports))
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "bad supports");
  cudaSetDevice(ctx->device);
  const int w = ctx->dim + 1;
  std::vector<uint8_t> fixed(ctx->n, 0);
  for (int i = 0; i < nsup; ++i) {
    int node = supports[i * w];
    if (node < 1 || node > ctx->nnodes)
      return gf_fail(ctx, GF_ERR_INVALID_ARG, "support %d names node %d", i, node);
    for (int c = 0; c < ctx->dim; ++c)
      if (supports[i * w + 1 + c] == 1) fixed[(size_t)(node - 1) * ctx->dim + c] = 1;
  }
  ctx->h_supports.assign(supports, supports + (size_t)nsup * w);
  ctx->nsup = nsup;
  gf_coarse_free(ctx);  // P depends on the constrained dofs
  GF_CUDA(ctx, cudaMemcpyAsync(ctx->d_fixed, fixed.data(), ctx->n, cudaMemcpyHostToDevice,
                               ctx->stream));
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GF_OK;
}

GF_API gf_status gf_set_nodal_loads(gf_ctx* ctx, int32_t nload, const double* loads) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (!ctx->has_mesh) return gf_fail(ctx, GF_ERR_STATE, "no mesh");
  if (nload < 0 || (nload > 0 && !loads)) return gf_fail(ctx, GF_ERR_INVALID_ARG, "bad loads");
  cudaSetDevice(ctx->device);
  const int w = ctx->dim + 1;
  std::vector<double> f(ctx->n, 0.0);
  for (int i = 0; i < nload; ++i) {
    int node = (int)loads[i * w];
    if (node < 1 || node > ctx->nnodes)
      return gf_fail(ctx, GF_ERR_INVALID_ARG, "load %d names node %d", i, node);
    for (int c = 0; c < ctx->dim; ++c) {
      double v = loads[i * w + 1 + c];
      if (v != 0.0) f[(size_t)(node - 1) * ctx->dim + c] = v;  // set, as CalcForceVector
    }
  }
  ctx->h_f = f;
  GF_CUDA(ctx, cudaMemcpyAsync(ctx->d_f, ctx->h_f.data(), sizeof(double) * ctx->n,
                               cudaMemcpyHostToDevice, ctx->stream));
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GF_OK;
}

GF_API gf_status gf_set_force(gf_ctx* ctx, const double* f) {
  if (!ctx || !f) return GF_ERR_INVALID_ARG;
  if (!ctx->d_f) return gf_fail(ctx, GF_ERR_STATE, "no mesh or matrix");
  cudaSetDevice(ctx->device);
  for (int i = 0; i < ctx->n; ++i)
    if (!std::isfinite(f[i])) return gf_fail(ctx, GF_ERR_INVALID_ARG, "non-finite force at %d", i);
  ctx->h_f.assign(f, f + ctx->n);
  GF_CUDA(ctx, cudaMemcpyAsync(ctx->d_f, ctx->h_f.data(), sizeof(double) * ctx->n,
                               cudaMemcpyHostToDevice, ctx->stream));
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GF_OK;
}

GF_API gf_status gf_get_force(gf_ctx* ctx, double* f) {
  if (!ctx || !f) return GF_ERR_INVALID_ARG;
  if (!ctx->d_f) return gf_fail(ctx, GF_ERR_STATE, "no mesh or matrix");
  cudaSetDevice(ctx->device);
  GF_CUDA(ctx, cudaMemcpyAsync(f, ctx->d_f, sizeof(double) * ctx->n, cudaMemcpyDeviceToHost,
                               ctx->stream));
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GF_OK;
}

GF_API gf_status gf_apply_constraints(gf_ctx* ctx, int32_t mode) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (!ctx->has_pattern || !(ctx->has64 || ctx->has32))
    return gf_fail(ctx, GF_ERR_STATE, "no assembled matrix");
  if (mode != GF_BC_PENALTY && mode != GF_BC_ELIMINATION)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "unknown constraint mode %d", mode);
  cudaSetDevice(ctx->device);
  return gf_constraints_apply(ctx, mode);
}

GF_API gf_status gf_spmv(gf_ctx* ctx, int32_t dtype, const void* x, void* y) {
  if (!ctx || !x || !y) return GF_ERR_INVALID_ARG;
  if (dtype != GF_F64 && dtype != GF_F32)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "unknown dtype %d", dtype);
  if ((dtype == GF_F64 && !ctx->has64) || (dtype == GF_F32 && !ctx->has32))
    return gf_fail(ctx, GF_ERR_STATE, "matrix of that dtype not assembled");
  cudaSetDevice(ctx->device);
  return gf_spmv_launch(ctx, dtype, x, y);
}

GF_API gf_status gf_spmv_host(gf_ctx* ctx, int32_t dtype, const double* x, double* y) {
  if (!ctx || !x || !y) return GF_ERR_INVALID_ARG;
  if ((dtype == GF_F64 && !ctx->has64) || (dtype == GF_F32 && !ctx->has32) ||
      (dtype != GF_F64 && dtype != GF_F32))
    return gf_fail(ctx, GF_ERR_STATE, "matrix of that dtype not assembled");
  cudaSetDevice(ctx->device);
  const int n = ctx->n;
  void *dx = nullptr, *dy = nullptr;
  gf_status st = GF_OK;
  const size_t es = dtype == GF_F64 ? 8 : 4;
  if (cudaMalloc(&dx, es * n) != cudaSuccess || cudaMalloc(&dy, es * n) != cudaSuccess) {
    cudaGetLastError();
    if (dx) cudaFree(dx);
    return gf_fail(ctx, GF_ERR_OOM, "spmv_host buffers");
  }
  std::vector<float> t32;
  if (dtype == GF_F64) {
    cudaMemcpyAsync(dx, x, 8 * n, cudaMemcpyHostToDevice, ctx->stream);
  } else {
    t32.resize(n);
    for (int i = 0; i < n; ++i) t32[i] = (float)x[i];
    cudaMemcpyAsync(dx, t32.data(), 4 * n, cudaMemcpyHostToDevice, ctx->stream);
  }
  st = gf_spmv_launch(ctx, dtype, dx, dy);
  if (st == GF_OK) {
    if (dtype == GF_F64) {
      cudaMemcpyAsync(y, dy, 8 * n, cudaMemcpyDeviceToHost, ctx->stream);
      cudaStreamSynchronize(ctx->stream);
    } else {
      cudaMemcpyAsync(t32.data(), dy, 4 * n, cudaMemcpyDeviceToHost, ctx->stream);
      cudaStreamSynchronize(ctx->stream);
      for (int i = 0; i < n; ++i) y[i] = t32[i];
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) st = gf_cuda_fail(ctx, e, "gf_spmv_host");
  }
  cudaFree(dx);
  cudaFree(dy);
  return st;
}

GF_API gf_status gf_solve(gf_ctx* ctx, const gf_solve_opts* opts, gf_solve_info* info) {
  if (!ctx || !opts) return GF_ERR_INVALID_ARG;
  if (!ctx->has_pattern) return gf_fail(ctx, GF_ERR_STATE, "no matrix");
  cudaSetDevice(ctx->device);
  gf_solve_info local{};
  gf_status st = gf_solve_run(ctx, opts, info ? info : &local);
  return st;
}

GF_API gf_status gf_get_solution(gf_ctx* ctx, double* u) {
  if (!ctx || !u) return GF_ERR_INVALID_ARG;
  if (!ctx->d_u) return gf_fail(ctx, GF_ERR_STATE, "no solution");
  cudaSetDevice(ctx->device);
  GF_CUDA(ctx, cudaMemcpyAsync(u, ctx->d_u, sizeof(double) * ctx->n, cudaMemcpyDeviceToHost,
                               ctx->stream));
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GF_OK;
}

GF_API gf_status gf_solution_view(gf_ctx* ctx, const double** u) {
  if (!ctx || !u) return GF_ERR_INVALID_ARG;
  if (!ctx->d_u) return gf_fail(ctx, GF_ERR_STATE, "no solution");
  *u = ctx->d_u;
  return GF_OK;
}

}  // extern "C"
