// C-ABI entry points: context, mesh upload (FemData::Init), colouring, matrix
// views/transfers, loads and constraints.  Kernels live in gf_pattern.cu,
// gf_assemble.cu and gf_solve.cu.
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <algorithm>

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
  gf_solver_free(ctx);
  gf_pattern_free(ctx);
  gf_mesh_free(ctx);
  gf_free(ctx->d_f);
  gf_free(ctx->d_fixed);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->evm) cudaEventDestroy(ctx->evm);
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

}  // extern "C"

void gf_mesh_free(gf_ctx* ctx) {
  gf_free(ctx->d_coords64);
  gf_free(ctx->d_coords32);
  gf_free(ctx->d_conn);
  gf_free(ctx->d_Eel);
  gf_free(ctx->d_Eel32);
  gf_free(ctx->d_asmtab);
  gf_free(ctx->d_perm);
  gf_free(ctx->d_allperm);
  ctx->h_conn.clear();
  ctx->h_color.clear();
  ctx->color_off.clear();
  ctx->ncolors = 0;
  ctx->has_mesh = false;
}

void gf_pattern_free(gf_ctx* ctx) {
  gf_free(ctx->d_rownnz);
  gf_free(ctx->d_colidx);
  gf_free(ctx->d_slotmap);
  gf_free(ctx->d_adj_off);
  gf_free(ctx->d_adj);
  gf_free(ctx->d_diagpos);
  gf_free(ctx->d_inc_off);
  gf_free(ctx->d_inc);
  gf_free(ctx->d_inc_loc);
  gf_free(ctx->d_inc_slot);
  if (ctx->d_geo) cudaFree(ctx->d_geo);
  ctx->d_geo = nullptr;
  ctx->geo_bytes = 0;
  ctx->maxval = 0;
  gf_free(ctx->d_K64);
  gf_free(ctx->d_K32);
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

static gf_status upload_modulus(gf_ctx* ctx, double E, const double* E_elem) {
  std::vector<double> e64(ctx->nelem);
  std::vector<float> e32(ctx->nelem);
  for (int i = 0; i < ctx->nelem; ++i) {
    double v = E_elem ? E_elem[i] : E;
    if (!(v > 0.0) || !std::isfinite(v))
      return gf_fail(ctx, GF_ERR_INVALID_ARG, "modulus of element %d is %g (must be > 0)", i, v);
    e64[i] = v;
    e32[i] = (float)v;
  }
  GF_CUDA(ctx, cudaMemcpyAsync(ctx->d_Eel, e64.data(), sizeof(double) * ctx->nelem,
                               cudaMemcpyHostToDevice, ctx->stream));
  GF_CUDA(ctx, cudaMemcpyAsync(ctx->d_Eel32, e32.data(), sizeof(float) * ctx->nelem,
                               cudaMemcpyHostToDevice, ctx->stream));
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->E = E;
  return GF_OK;
}

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
  for (int64_t i = 0; i < (int64_t)nnodes * info.dim; ++i)
    if (!std::isfinite(coords[i]))
      return gf_fail(ctx, GF_ERR_INVALID_ARG, "non-finite coordinate at %lld", (long long)i);
  std::vector<int32_t> conn0((size_t)nelem * info.nen);
  for (size_t i = 0; i < conn0.size(); ++i) {
    int32_t v = connect[i];
    if (v < 1 || v > nnodes)
      return gf_fail(ctx, GF_ERR_INVALID_ARG,
                     "connectivity entry %zu = %d outside 1..%d (1-based node ids)", i, v, nnodes);
    conn0[i] = v - 1;
  }
  for (int e = 0; e < nelem; ++e)
    for (int a = 0; a < info.nen; ++a)
      for (int b = a + 1; b < info.nen; ++b)
        if (conn0[(size_t)e * info.nen + a] == conn0[(size_t)e * info.nen + b])
          return gf_fail(ctx, GF_ERR_INVALID_ARG, "element %d repeats node %d", e,
                         conn0[(size_t)e * info.nen + a] + 1);

  cudaStreamSynchronize(ctx->stream);
  gf_solver_free(ctx);
  gf_pattern_free(ctx);
  gf_mesh_free(ctx);
  gf_lp_mesh_changed(ctx);
  gf_free(ctx->d_f);
  gf_free(ctx->d_fixed);
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
  ctx->n = nnodes * info.dim;
  ctx->h_conn = conn0;

  gf_status st;
  const size_t ncoord = (size_t)nnodes * info.dim;
  if ((st = gf_alloc(ctx, &ctx->d_coords64, ncoord)) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &ctx->d_coords32, ncoord)) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &ctx->d_conn, conn0.size())) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &ctx->d_Eel, (size_t)nelem)) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &ctx->d_Eel32, (size_t)nelem)) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &ctx->d_allperm, (size_t)nelem)) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &ctx->d_f, (size_t)ctx->n)) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &ctx->d_fixed, (size_t)ctx->n)) != GF_OK) return st;
  GF_CUDA(ctx, cudaMemcpyAsync(ctx->d_coords64, coords, sizeof(double) * ncoord,
                               cudaMemcpyHostToDevice, ctx->stream));
  k_f64_to_f32<<<gf_blocks(ncoord, 256), 256, 0, ctx->stream>>>((int64_t)ncoord, ctx->d_coords64,
                                                                 ctx->d_coords32);
  GF_LAUNCH_CHECK(ctx, "k_f64_to_f32");
  GF_CUDA(ctx, cudaMemcpyAsync(ctx->d_conn, conn0.data(), sizeof(int32_t) * conn0.size(),
                               cudaMemcpyHostToDevice, ctx->stream));
  k_iota<<<gf_blocks(nelem, 256), 256, 0, ctx->stream>>>(nelem, ctx->d_allperm);
  GF_LAUNCH_CHECK(ctx, "k_iota");
  GF_CUDA(ctx, cudaMemsetAsync(ctx->d_f, 0, sizeof(double) * ctx->n, ctx->stream));
  GF_CUDA(ctx, cudaMemsetAsync(ctx->d_fixed, 0, ctx->n, ctx->stream));
  ctx->h_f.assign(ctx->n, 0.0);
  if ((st = upload_modulus(ctx, E, E_elem)) != GF_OK) return st;
  ctx->has_mesh = true;
  return GF_OK;
}

GF_API gf_status gf_mesh_set_modulus(gf_ctx* ctx, double E, const double* E_elem) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (!ctx->has_mesh) return gf_fail(ctx, GF_ERR_STATE, "no mesh");
  cudaSetDevice(ctx->device);
  return upload_modulus(ctx, E, E_elem);
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
  if (scatter != GF_SCATTER_COLOR && scatter != GF_SCATTER_ATOMIC && scatter != GF_SCATTER_OWNER)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "unknown scatter %d", scatter);
  if (engine != GF_ENGINE_CUDA_CORE && engine != GF_ENGINE_TF32_MMA)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "unknown engine %d", engine);
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
  if (!ctx->d_K32 && (st = gf_alloc(ctx, &ctx->d_K32, (size_t)total)) != GF_OK) return st;
  k_f64_to_f32<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(total, ctx->d_K64, ctx->d_K32);
  GF_LAUNCH_CHECK(ctx, "k_f64_to_f32");
  ctx->has32 = true;
  ctx->kver32++;
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

GF_API gf_status gf_ell_download(gf_ctx* ctx, int32_t dtype, int32_t* rownnz, int32_t* colidx,
                                 void* values) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (!ctx->has_pattern) return gf_fail(ctx, GF_ERR_STATE, "no matrix");
  cudaSetDevice(ctx->device);
  const size_t total = (size_t)ctx->n * ctx->W;
  if (rownnz)
    GF_CUDA(ctx, cudaMemcpyAsync(rownnz, ctx->d_rownnz, sizeof(int32_t) * ctx->n,
                                 cudaMemcpyDeviceToHost, ctx->stream));
  if (colidx)
    GF_CUDA(ctx, cudaMemcpyAsync(colidx, ctx->d_colidx, sizeof(int32_t) * total,
                                 cudaMemcpyDeviceToHost, ctx->stream));
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
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
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
  gf_free(ctx->d_f);
  gf_free(ctx->d_fixed);
  ctx->h_supports.clear();
  ctx->nsup = 0;
  ctx->bc_mode_applied = -1;
  gf_status st;
  ctx->n = n;
  ctx->W = width;
  ctx->nnz = nnz;
  if ((st = gf_alloc(ctx, &ctx->d_rownnz, (size_t)n)) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &ctx->d_colidx, total)) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &ctx->d_K64, total)) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &ctx->d_K32, total)) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &ctx->d_f, (size_t)n)) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &ctx->d_fixed, (size_t)n)) != GF_OK) return st;
  ctx->h_f.assign(n, 0.0);
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
