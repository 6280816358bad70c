// Internal declarations shared by the gpufem_b200 CUDA sources.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "gpufem_b200.h"

// ---------------------------------------------------------------------------
// Element families.  Node natural coordinates follow the reference's node order
// (src/FEM/StiffAlgo.cc:47-202):
//   Q4      (-1,-1) (1,-1) (1,1) (-1,1)
//   Q8      (-1,-1) (0,-1) (1,-1) (1,0) (1,1) (0,1) (-1,1) (-1,0)
//   Brick8  (1,-1,-1) (1,1,-1) (1,1,1) (1,-1,1) (-1,-1,-1) (-1,1,-1) (-1,1,1) (-1,-1,1)
//   Brick20 corners at 0,2,4,6 (r=+1) and 12,14,16,18 (r=-1) in Brick8's (s,t) order;
//           mid-side nodes 1,3,5,7 on r=+1, 8..11 on r=0, 13,15,17,19 on r=-1.
// Shape functions are the standard bilinear/trilinear Lagrange and quadratic
// serendipity families written from their definitions; derivatives are taken
// analytically below.
// ---------------------------------------------------------------------------
constexpr int GF_MAX_NEN = 20;
constexpr int GF_MAX_GP = 27;

struct ElemInfo {
  int nen, dim, serendipity;
};

__host__ __device__ constexpr ElemInfo gf_elem_info(int et) {
  return et == GF_Q4 ? ElemInfo{4, 2, 0}
       : et == GF_Q8 ? ElemInfo{8, 2, 1}
       : et == GF_BRICK8 ? ElemInfo{8, 3, 0}
                         : ElemInfo{20, 3, 1};
}

// natural coordinates (xi, eta, zeta) of element nodes, [et][node][3], in the
// reference's node order (StiffAlgo::GetdShapeFunctNatCoord, src/FEM/StiffAlgo.cc:47-202)
constexpr signed char gf_node_nat_host[4][GF_MAX_NEN][3] = {
    // Q4
    {{-1, -1, 0}, {1, -1, 0}, {1, 1, 0}, {-1, 1, 0}},
    // Q8
    {{-1, -1, 0}, {0, -1, 0}, {1, -1, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {-1, 1, 0}, {-1, 0, 0}},
    // Brick8
    {{1, -1, -1}, {1, 1, -1}, {1, 1, 1}, {1, -1, 1}, {-1, -1, -1}, {-1, 1, -1}, {-1, 1, 1}, {-1, -1, 1}},
    // Brick20
    {{1, -1, -1}, {1, 0, -1}, {1, 1, -1}, {1, 1, 0}, {1, 1, 1}, {1, 0, 1}, {1, -1, 1}, {1, -1, 0},
     {0, -1, -1}, {0, 1, -1}, {0, 1, 1}, {0, -1, 1},
     {-1, -1, -1}, {-1, 0, -1}, {-1, 1, -1}, {-1, 1, 0}, {-1, 1, 1}, {-1, 0, 1}, {-1, -1, 1}, {-1, -1, 0}},
};

// Derivatives dN_i/dxi_a at natural point p (host and device), written from:
//   Lagrange:     N = prod_a (1 + xi_a p_a) / 2^dim
//   Serendipity corner:   N = prod(1 + xi_a p_a)/2^dim * (sum_a xi_a p_a - (dim-1))
//   Serendipity mid-side (one xi_c = 0):
//                 N = (1 - p_c^2) * prod_{a != c} (1 + xi_a p_a) / 2^(dim-1)
template <typename R>
__host__ __device__ constexpr void gf_dshape(int et, const signed char (*nat)[3], const R* p,
                                             R* dN /* [dim][nen] */) {
  const ElemInfo info = gf_elem_info(et);
  const int dim = info.dim, nen = info.nen;
  for (int i = 0; i < nen; ++i) {
    R xi[3] = {R(nat[i][0]), R(nat[i][1]), R(nat[i][2])};
    R f[3] = {R(0), R(0), R(0)};  // linear factors (1 + xi_a p_a)
    for (int a = 0; a < dim; ++a) f[a] = R(1) + xi[a] * p[a];
    if (!info.serendipity) {
      const R scale = dim == 2 ? R(0.25) : R(0.125);
      for (int a = 0; a < dim; ++a) {
        R d = scale * xi[a];
        for (int b = 0; b < dim; ++b)
          if (b != a) d *= f[b];
        dN[a * nen + i] = d;
      }
    } else {
      int c = -1;  // zero natural coordinate (mid-side node)
      for (int a = 0; a < dim; ++a)
        if (nat[i][a] == 0) c = a;
      if (c < 0) {
        const R scale = dim == 2 ? R(0.25) : R(0.125);
        R lin = R(1);
        for (int a = 0; a < dim; ++a) lin *= f[a];
        R s = -R(dim - 1);
        for (int a = 0; a < dim; ++a) s += xi[a] * p[a];
        for (int a = 0; a < dim; ++a) {
          // d/dp_a [ scale * prod f * s ] = scale * (xi_a prod_{b!=a} f_b * s + prod f * xi_a)
          R pr = R(1);
          for (int b = 0; b < dim; ++b)
            if (b != a) pr *= f[b];
          dN[a * nen + i] = scale * xi[a] * (pr * s + lin);
        }
      } else {
        const R scale = dim == 2 ? R(0.5) : R(0.25);
        R q = R(1) - p[c] * p[c];
        for (int a = 0; a < dim; ++a) {
          R d = R(0);
          if (a == c) {
            d = scale * (R(-2) * p[c]);
            for (int b = 0; b < dim; ++b)
              if (b != c) d *= f[b];
          } else {
            d = scale * q * xi[a];
            for (int b = 0; b < dim; ++b)
              if (b != c && b != a) d *= f[b];
          }
          dN[a * nen + i] = d;
        }
      }
    }
  }
}

// Gauss rule in the reference's tensor order (FemData::CalcGaussVectors,
// src/FEM/FemData.cc:226-316): index s runs i (first coordinate) outermost,
// last coordinate innermost; weight = product of 1-D weights.
template <typename R>
inline void gf_gauss_rule(int dim, int ng1, std::vector<R>& pts, std::vector<R>& w) {
  R x[3], wt[3];
  if (ng1 == 2) {
    x[0] = -R(1) / std::sqrt(R(3)); x[1] = -x[0];
    wt[0] = wt[1] = R(1);
  } else {
    x[0] = -std::sqrt(R(3) / R(5)); x[1] = R(0); x[2] = -x[0];
    wt[0] = R(5) / R(9); wt[1] = R(8) / R(9); wt[2] = wt[0];
  }
  pts.clear(); w.clear();
  if (dim == 2) {
    for (int i = 0; i < ng1; ++i)
      for (int j = 0; j < ng1; ++j) {
        pts.push_back(x[i]); pts.push_back(x[j]);
        w.push_back(wt[i] * wt[j]);
      }
  } else {
    for (int i = 0; i < ng1; ++i)
      for (int j = 0; j < ng1; ++j)
        for (int k = 0; k < ng1; ++k) {
          pts.push_back(x[i]); pts.push_back(x[j]); pts.push_back(x[k]);
          w.push_back(wt[i] * wt[j] * wt[k]);
        }
  }
}

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
// device-side CG scalars (gf_solve.cu, gf_twolevel.cu)
struct SolveScalars {
  double pq;    // p . A p (accumulated by the SpMV)
  double rz;    // r . z of the current iteration
  double rzn;   // r . z of the next iteration (accumulated by the update)
  double rr;    // r . r after the update
  double rr0;   // initial r . r
  double tol2;  // stop when rr <= tol2
  int iter;
  int done;     // 0 running, 1 converged, 2 breakdown, 3 iteration cap
  int maxit;
  int pad;
};
struct LpState;       // learned preconditioner (gf_learned.cu)

struct gf_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t evm = nullptr;            // between the two kernels of an owner assembly
  double last_split[2] = {0.0, 0.0};    // last assembly: geometry, scatter kernel seconds
  std::string err;
  double last_seconds = 0.0;
  int64_t launches = 0;
  int sm_count = 148;

  // mesh
  bool has_mesh = false;
  int elem_type = 0, dim = 0, nen = 0, ngauss = 0, ngp = 0;
  int nnodes = 0, nelem = 0, analysis = 0;
  double E = 0.0, nu = 0.0;
  double lam1 = 0.0, mu1 = 0.0;  // Lame-type factors per unit modulus
  std::vector<int32_t> h_conn;   // 0-based, host copy (host colouring; filled on demand)
  // device buffer pool (gf_palloc / gf_pfree)
  struct PoolBlock {
    void* p;
    size_t bytes;
    int64_t gen;
  };
  std::vector<std::pair<void*, size_t>> pool_live;
  std::vector<PoolBlock> pool_free;
  int64_t pool_gen = 0;
  double* d_coords64 = nullptr;
  float* d_coords32 = nullptr;
  int32_t* d_conn = nullptr;     // 0-based node ids
  double* d_Eel = nullptr;       // per-element modulus
  float* d_Eel32 = nullptr;
  void* d_asmtab = nullptr;      // shape-derivative tables (gf_assemble.cu)
  int* d_asm_err = nullptr;      // tensor-core assembly: set when an MMA wait timed out
  float* d_gram = nullptr;       // tensor-core owner schedule: element Gram matrices
  size_t gram_bytes = 0;

  // colouring
  int ncolors = 0;
  std::vector<int32_t> h_color;      // per element
  std::vector<int32_t> color_off;    // ncolors + 1
  int32_t* d_perm = nullptr;         // elements sorted by colour
  int32_t* d_allperm = nullptr;      // identity (atomic scatter)

  // pattern
  bool has_pattern = false;
  int n = 0, W = 0;
  int64_t nnz = 0;
  int32_t* d_rownnz = nullptr;
  int32_t* d_colidx = nullptr;
  uint16_t* d_slotmap = nullptr;  // [nen*nen][nelem]: neighbour position of node j in node i's list
  int32_t* d_adj_off = nullptr;   // node adjacency CSR
  int32_t* d_adj = nullptr;
  int32_t* d_diagpos = nullptr;   // per node: own position in its adjacency list
  int32_t* d_inc_off = nullptr;   // node -> element incidence CSR, element ids ascending
  int32_t* d_inc = nullptr;
  uint8_t* d_inc_loc = nullptr;   // local index of the node within each incident element
  uint16_t* d_inc_slot = nullptr; // [incidence][nen]: neighbour position of each element node
  int maxval = 0;                 // max elements sharing one node
  void* d_geo = nullptr;          // owner scatter: J^-1, w detJ per (element, Gauss point)
  size_t geo_bytes = 0;

  // values
  bool has64 = false, has32 = false;
  double* d_K64 = nullptr;
  float* d_K32 = nullptr;
  int64_t kver64 = 0, kver32 = 0;  // bumped whenever the values change

  // sliced-ELL copy for the solver's SpMVs (gf_sell.cu)
  bool sell_ready = false;
  int sell_nslice = 0, sell_nslots = 0;  // slices of 32 rows (nodes); nslots = 32 * nslice
  int sell_bdim = 0;                     // 0: row slices; 2, 3: node-block slices
  int64_t sell_total = 0;
  int64_t sell_ver64 = -1, sell_ver32 = -1;
  int64_t* d_sell_off = nullptr;   // [nslice + 1] first entry of each slice
  int32_t* d_sell_w = nullptr;     // [nslice] width of each slice
  int32_t* d_sell_col = nullptr;   // [total]
  int32_t* d_sell_perm = nullptr;  // node slices: node of each slot (degree-sorted windows)
  double* d_sell_v64 = nullptr;
  float* d_sell_v32 = nullptr;

  // loads / constraints
  double* d_f = nullptr;
  std::vector<double> h_f;   // host copy of the force set by the caller; empty: f = 0
  std::vector<int32_t> h_supports;  // nsup*(dim+1)
  int nsup = 0;
  uint8_t* d_fixed = nullptr;       // per dof
  int bc_mode_applied = -1;

  // solver state
  double* d_u = nullptr;
  void* d_work = nullptr;  // solver work vectors
  size_t work_bytes = 0;
  SolveScalars* d_scal = nullptr;
  void* h_pinned = nullptr;  // pinned scalars readback
  int32_t* h_adj_stage = nullptr;   // pinned node adjacency for gf_ell_download
  size_t h_adj_stage_n = 0;
  cudaEvent_t ev_dl = nullptr;      // adjacency copied (gf_ell_download)
  double* d_red = nullptr;   // reduction scratch
  void* d_fcg = nullptr;     // flexible-CG scalars

  // learned preconditioner
  LpState* lp = nullptr;
  void* coarse = nullptr;  // two-level preconditioner (gf_twolevel.cu)
  void* dist = nullptr;    // sharded PCG: halo lists and device vectors (gf_solve.cu)
  int coarse_target = 0;   // requested coarse unknowns (0: default)
};

// ---------------------------------------------------------------------------
// Error helpers
// ---------------------------------------------------------------------------
gf_status gf_fail(gf_ctx* ctx, gf_status st, const char* fmt, ...);
gf_status gf_cuda_fail(gf_ctx* ctx, cudaError_t e, const char* where);

#define GF_CUDA(ctx, call)                                   \
  do {                                                       \
    cudaError_t e__ = (call);                                \
    if (e__ != cudaSuccess) return gf_cuda_fail(ctx, e__, #call); \
  } while (0)

#define GF_LAUNCH_CHECK(ctx, name)                                    \
  do {                                                                \
    (ctx)->launches++;                                                \
    cudaError_t e__ = cudaGetLastError();                             \
    if (e__ != cudaSuccess) return gf_cuda_fail(ctx, e__, name);      \
  } while (0)

template <typename T>
gf_status gf_alloc(gf_ctx* ctx, T** p, size_t count) {
  if (*p) { cudaFree(*p); *p = nullptr; }
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return gf_fail(ctx, e == cudaErrorMemoryAllocation ? GF_ERR_OOM : GF_ERR_CUDA,
                   "cudaMalloc of %zu bytes failed: %s", count * sizeof(T),
                   cudaGetErrorString(e));
  }
  return GF_OK;
}

template <typename T>
void gf_free(T*& p) {
  if (p) { cudaFree(p); p = nullptr; }
}

// Pooled device buffers for the per-mesh arrays (mesh, pattern, K): a released block
// is kept by the context and handed out again for a request of exactly its size, so
// re-creating a mesh of the same shape (a time loop, a parameter sweep) allocates
// nothing.  Blocks released before the previous mesh generation are returned to the
// driver when a new mesh is created; all of them at gf_destroy, and all of them
// before an allocation that failed is retried.
void* gf_pool_get(gf_ctx* ctx, size_t bytes);
void gf_pool_put(gf_ctx* ctx, void* p);
void gf_pool_new_generation(gf_ctx* ctx);
void gf_pool_clear(gf_ctx* ctx);

template <typename T>
gf_status gf_palloc(gf_ctx* ctx, T** p, size_t count) {
  if (*p) { gf_pool_put(ctx, *p); *p = nullptr; }
  if (count == 0) count = 1;
  *p = static_cast<T*>(gf_pool_get(ctx, count * sizeof(T)));
  if (!*p)
    return gf_fail(ctx, GF_ERR_OOM, "device allocation of %zu bytes failed", count * sizeof(T));
  return GF_OK;
}

template <typename T>
void gf_pfree(gf_ctx* ctx, T*& p) {
  if (p) { gf_pool_put(ctx, p); p = nullptr; }
}

// Kernel attributes that persist for the process (per device): the dynamic shared-memory
// limit and the carveout are set on a kernel's first launch (or when a launch needs more
// shared memory than set so far), not before every launch, which would cost host time
// between a call's timing events.
inline cudaError_t gf_func_attr(const void* fn, cudaFuncAttribute attr, int value) {
  static std::mutex mu;
  static std::map<std::pair<std::pair<const void*, int>, int>, int> set;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_pair(std::make_pair(fn, dev), (int)attr);
  std::lock_guard<std::mutex> lock(mu);
  const auto it = set.find(key);
  const bool grow_only = attr == cudaFuncAttributeMaxDynamicSharedMemorySize;
  if (it != set.end() && (grow_only ? it->second >= value : it->second == value))
    return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(fn, attr, value);
  if (e == cudaSuccess) set[key] = value;
  return e;
}
template <typename K>
inline cudaError_t gf_smem_attr(K kernel, size_t bytes) {
  return gf_func_attr(reinterpret_cast<const void*>(kernel),
                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

inline int gf_blocks(int64_t work, int threads) {
  int64_t b = (work + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > (1LL << 30)) b = (1LL << 30);
  return (int)b;
}

// internal entry points across translation units
gf_status gf_pattern_build(gf_ctx* ctx);
gf_status gf_slotmap_ensure(gf_ctx* ctx);
gf_status gf_color_build(gf_ctx* ctx, const int32_t* user_colors);
gf_status gf_assemble_launch(gf_ctx* ctx, int dtype, int scatter, int engine);
gf_status gf_constraints_apply(gf_ctx* ctx, int mode);
gf_status gf_spmv_launch(gf_ctx* ctx, int dtype, const void* x, void* y);
gf_status gf_matvec_f32(gf_ctx* ctx, const float* x, const float* scale, float* y);
gf_status gf_solve_run(gf_ctx* ctx, const gf_solve_opts* o, gf_solve_info* info);
void gf_solver_free(gf_ctx* ctx);
void gf_dist_free(gf_ctx* ctx);
void gf_mesh_free(gf_ctx* ctx);
void gf_pattern_free(gf_ctx* ctx);

// sliced-ELL copy (gf_sell.cu)
gf_status gf_sell_prepare(gf_ctx* ctx, int dtype);
void gf_sell_free(gf_ctx* ctx);

// learned preconditioner (gf_learned.cu)
void gf_lp_free(gf_ctx* ctx);

// two-level preconditioner (gf_twolevel.cu)
void gf_coarse_free(gf_ctx* ctx);
gf_status gf_coarse_prepare(gf_ctx* ctx, int target_coarse);
// z = D^-1 r + P Ac^-1 P^T r (FP64 vectors), rz_acc += r.z; launches only.
void gf_coarse_apply(gf_ctx* ctx, const double* r, const double* dinv, double* z,
                     double* rz_acc, const int* done);
// z += P Ac^-1 P^T r (the coarse term alone); launches only.
void gf_coarse_add(gf_ctx* ctx, const double* r, double* z);
// Two-level PCG steps (launches only, capturable).  Begin: x = 0, r = b, p = M r,
// sc->rr = b.b, sc->rzn = r.M r.  Iterate (after the SpMV q = K p, p.q): x, r update,
// then p = M r + beta p; the kernels return at once while sc->done != 0.  p32 (or
// null): n floats that receive an FP32 copy of every new p.
void gf_tl_begin(gf_ctx* ctx, const double* b, double* x, double* r, double* p,
                 const double* dinv, SolveScalars* sc, float* p32 = nullptr);
void gf_tl_iterate(gf_ctx* ctx, double* x, double* r, double* p, const double* q,
                   const double* dinv, SolveScalars* sc, float* p32 = nullptr);
// Reliable update: x = 0, r = scale * b, rr and rzn as in begin; then p = M r (restart)
// or p = pscale * p (direction kept).  sc->rr and sc->rzn must be zero on entry.
void gf_tl_reset(gf_ctx* ctx, const double* b, double scale, bool restart, double pscale,
                 double* x, double* r, double* p, const double* dinv, SolveScalars* sc,
                 float* p32 = nullptr);
// The same two steps on FP32 vectors (r from the FP64 b; the scalars in FP64): the
// direction itself is the FP32 operand of the SpMV on K32.
void gf_tl_reset(gf_ctx* ctx, const double* b, double scale, bool restart, double pscale,
                 float* x, float* r, float* p, const float* dinv, SolveScalars* sc);
void gf_tl_iterate(gf_ctx* ctx, float* x, float* r, float* p, const float* q,
                   const float* dinv, SolveScalars* sc);
void gf_lp_mesh_changed(gf_ctx* ctx);
gf_status gf_lp_prepare(gf_ctx* ctx);
bool gf_lp_ready(const gf_ctx* ctx);
bool gf_lp_coarse(const gf_ctx* ctx);  // learned preconditioner with the coarse correction
// z = M(r): FP64 residual in, FP64 preconditioned vector out (r32: n floats of scratch)
gf_status gf_lp_apply64(gf_ctx* ctx, const double* r64, float* r32_scratch, double* z);
// Jacobi-PCG on the FP64 matrix recording (float(r_k), float(ustar - x_k)) every
// `every` iterations into r_out / e_out (npairs slots of n floats); *recorded set.
gf_status gf_pcg_record(gf_ctx* ctx, const double* ustar, int npairs, int every, double tol,
                        int maxit, float* r_out, float* e_out, int* recorded, bool twolevel = false);
