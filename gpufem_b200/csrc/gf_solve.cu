// ELL SpMV, constraints and the CG family, all device-resident.
//
// Reference: ELLmatrix::Axy (src/SPRmatrix/ELLmatrix.cc:194-204), the OpenCL
// SpMV variants (src/OpenCL/clKernels/LAopsEll.cl), SPRmatrix::CPU_CG
// (src/SPRmatrix/SPRmatrix.cc:405-480), ELLmatrix::SolveCgGpu
// (ELLmatrix.cc:315-459), LAops dot/axpy (src/LAops/LAops.cc:54-61,178-203) and
// FEM::ApplyConstraint (src/FEM/fem.cc:112-167).
//
// The reference crosses PCIe twice per CG iteration (SolveCgGpu).  Here every
// vector and scalar stays on the device: one iteration is three kernels
//   K1  q = K p, p.q                      (SpMV with fused dot)
//   K2  alpha; x += alpha p; r -= alpha q; z = M r; r.z; r.r   (fused axpy/precond/dots)
//   K3  beta; p = z + beta p; convergence flag
// with the scalars in device memory.  Chunks of iterations are captured once
// into a CUDA graph; the host reads the convergence flag after each chunk, and
// kernels of a finished solve return immediately.
#include <chrono>
#include <cmath>
#include <algorithm>
#include <mutex>

#include "gf_internal.cuh"

namespace {

constexpr int kT = 256;

template <typename T>
__device__ inline double block_sum(T v, double* sh) {
  double x = (double)v;
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = x;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  }
  return s;  // valid in thread 0
}

// Where the solver's SpMVs find the matrix.  Two layouts share every kernel, both
// with thread t owning row t:
//   ELL   (width == nullptr): entry s of row t at s*n + t, rownnz[t] entries.
//   SELL  (width != nullptr): the sliced copy (gf_sell.cu); entry s of row t at
//         off[t/32] + 32 s + t%32, and every row of a slice runs to the slice's
//         width (padding entries hold column t and value 0).
struct MatLayout {
  int count;  // threads to launch
  int n;
  const int32_t* __restrict__ rownnz;
  const int32_t* __restrict__ col;
  const int32_t* __restrict__ width;
  const int64_t* __restrict__ off;
  int bdim = 0;      // 0: rows (ELL / SELL); 2, 3: node-block slices (gf_sell.cu)
  int nnodes = 0;
  const int32_t* __restrict__ perm = nullptr;  // node-block slices: node of each slot
  int threads = kT;  // block size

  __device__ inline bool at(int t, int& nz, int64_t& o, int64_t& stride) const {
    if (t >= count) return false;
    if (width) {
      nz = __ldg(width + (t >> 5));
      o = __ldg(off + (t >> 5)) + (t & 31);
      stride = 32;
    } else {
      nz = __ldg(rownnz + t);
      o = t;
      stride = n;
    }
    return true;
  }
};

template <typename TK, typename TX>
__device__ inline double row_dot(int64_t o, int64_t stride, int nz, const int32_t* __restrict__ col,
                                 const TK* __restrict__ val, const TX* __restrict__ x) {
  using Acc = typename std::conditional<sizeof(TK) == 8 || sizeof(TX) == 8, double, float>::type;
  Acc a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  int s = 0;
  if (nz >= 4) {
    int c0 = __ldcs(col + o), c1 = __ldcs(col + o + stride), c2 = __ldcs(col + o + 2 * stride),
        c3 = __ldcs(col + o + 3 * stride);
    TK v0 = __ldcs(val + o), v1 = __ldcs(val + o + stride), v2 = __ldcs(val + o + 2 * stride),
       v3 = __ldcs(val + o + 3 * stride);
    for (s = 4; s + 4 <= nz; s += 4) {
      o += 4 * stride;
      const int d0 = __ldcs(col + o), d1 = __ldcs(col + o + stride),
                d2 = __ldcs(col + o + 2 * stride), d3 = __ldcs(col + o + 3 * stride);
      const TK w0 = __ldcs(val + o), w1 = __ldcs(val + o + stride),
               w2 = __ldcs(val + o + 2 * stride), w3 = __ldcs(val + o + 3 * stride);
      a0 += (Acc)v0 * (Acc)__ldg(x + c0);
      a1 += (Acc)v1 * (Acc)__ldg(x + c1);
      a2 += (Acc)v2 * (Acc)__ldg(x + c2);
      a3 += (Acc)v3 * (Acc)__ldg(x + c3);
      c0 = d0; c1 = d1; c2 = d2; c3 = d3;
      v0 = w0; v1 = w1; v2 = w2; v3 = w3;
    }
    a0 += (Acc)v0 * (Acc)__ldg(x + c0);
    a1 += (Acc)v1 * (Acc)__ldg(x + c1);
    a2 += (Acc)v2 * (Acc)__ldg(x + c2);
    a3 += (Acc)v3 * (Acc)__ldg(x + c3);
    o += 4 * stride;
  }
  for (; s < nz; ++s, o += stride) a0 += (Acc)__ldcs(val + o) * (Acc)__ldg(x + __ldcs(col + o));
  return (double)((a0 + a1) + (a2 + a3));
}

// x[2b], x[2b + 1] in one 8- or 16-byte load (x is 16-byte aligned: device allocations)
template <typename Acc>
__device__ inline void ldg_pair(const float* __restrict__ x, int b, Acc& x0, Acc& x1) {
  const float2 v = __ldg(reinterpret_cast<const float2*>(x) + b);
  x0 = (Acc)v.x;
  x1 = (Acc)v.y;
}
template <typename Acc>
__device__ inline void ldg_pair(const double* __restrict__ x, int b, Acc& x0, Acc& x1) {
  const double2 v = __ldg(reinterpret_cast<const double2*>(x) + b);
  x0 = (Acc)v.x;
  x1 = (Acc)v.y;
}

// Node-block slices: thread t computes the DIM rows of node perm[t] (slice k = t / 32,
// lane l = t % 32).  Per neighbour block it reads one coalesced column word, DIM x DIM
// coalesced values and DIM consecutive entries of x (once for all DIM rows), and it
// writes its DIM results contiguously.  Measured against a warp per (slice, component),
// which gathers x DIM times: Q8 512 FP64 113 -> 96 us, FP32 78 -> 60 us, Brick8 128
// FP32 459 -> 373 us (B200, L2 flushed).
template <int DIM, typename TK, typename TX>
__device__ inline bool node_rows(const MatLayout& L, int t, const TK* __restrict__ val,
                                 const TX* __restrict__ x, int& node, double (&out)[DIM]) {
  using Acc = typename std::conditional<sizeof(TK) == 8 || sizeof(TX) == 8, double, float>::type;
  constexpr int SS = DIM * DIM * 32;  // value stride between neighbour slots
  if (t >= L.nnodes) return false;
  node = __ldg(L.perm + t);
  const int k = t >> 5, l = t & 31;
  const int64_t o = __ldg(L.off + k);
  const int w = __ldg(L.width + k);
  const int32_t* bc = L.col + o + l;
  const TK* vp = val + o * (DIM * DIM) + l;
  Acc acc[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) acc[c] = 0;
  if constexpr (DIM == 2) {
    // short 2-D rows: all column words first, so every x gather's address is known
    // before the first one is issued
    constexpr int kPre = 24;
    if (w <= kPre) {
      int bb[kPre];
#pragma unroll
      for (int p = 0; p < kPre; ++p) bb[p] = p < w ? __ldcs(bc + 32 * p) : 0;
#pragma unroll
      for (int p = 0; p < kPre; ++p) {
        if (p < w) {
          const TK* v = vp + p * SS;
          const TK u0 = __ldcs(v), u1 = __ldcs(v + 32), u2 = __ldcs(v + 64), u3 = __ldcs(v + 96);
          Acc x0, x1;
          ldg_pair(x, bb[p], x0, x1);
          acc[0] += (Acc)u0 * x0 + (Acc)u1 * x1;
          acc[1] += (Acc)u2 * x0 + (Acc)u3 * x1;
        }
      }
      out[0] = (double)acc[0];
      out[1] = (double)acc[1];
      return true;
    }
  }
  for (int p = 0; p < w; ++p, bc += 32, vp += SS) {
    const int b = __ldcs(bc);
    TK u[DIM * DIM];
#pragma unroll
    for (int e = 0; e < DIM * DIM; ++e) u[e] = __ldcs(vp + e * 32);
    Acc xv[DIM];
#pragma unroll
    for (int c2 = 0; c2 < DIM; ++c2) xv[c2] = (Acc)__ldg(x + (int64_t)b * DIM + c2);
#pragma unroll
    for (int c = 0; c < DIM; ++c)
#pragma unroll
      for (int c2 = 0; c2 < DIM; ++c2) acc[c] += (Acc)u[c * DIM + c2] * xv[c2];
  }
#pragma unroll
  for (int c = 0; c < DIM; ++c) out[c] = (double)acc[c];
  return true;
}

// Calls f(row, (K x)[row]) for every row that thread t of layout L computes.
template <typename TK, typename TX, typename F>
__device__ inline void mat_rows(const MatLayout& L, int t, const TK* __restrict__ val,
                                const TX* __restrict__ x, F&& f) {
  int a;
  if (L.bdim == 2) {
    double v[2];
    if (node_rows<2>(L, t, val, x, a, v)) {
      f(2 * a, v[0]);
      f(2 * a + 1, v[1]);
    }
  } else if (L.bdim == 3) {
    double v[3];
    if (node_rows<3>(L, t, val, x, a, v)) {
      f(3 * a, v[0]);
      f(3 * a + 1, v[1]);
      f(3 * a + 2, v[2]);
    }
  } else {
    int nz;
    int64_t o, st;
    if (L.at(t, nz, o, st)) f(t, row_dot(o, st, nz, L.col, val, x));
  }
}

template <typename TK, typename TX, typename TY>
__global__ void __launch_bounds__(kT)
k_spmv(MatLayout L, const TK* __restrict__ val, const TX* __restrict__ x, TY* __restrict__ y) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < L.count; t += gridDim.x * blockDim.x)
    mat_rows(L, t, val, x, [&](int row, double v) { y[row] = (TY)v; });
}

// y = scale .* (K x) for FP32 x and y (scale may be null), FP64 accumulation with FP64
// values
template <typename TK>
__global__ void __launch_bounds__(kT)
k_spmv_rowscale(MatLayout L, const TK* __restrict__ val, const float* __restrict__ x,
                const float* __restrict__ scale, float* __restrict__ y) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < L.count; t += gridDim.x * blockDim.x)
    mat_rows(L, t, val, x, [&](int row, double v) {
      y[row] = (float)(scale ? v * (double)__ldg(scale + row) : v);
    });
}

// r = f - K u (FP64), and r.r
__global__ void __launch_bounds__(kT)
k_residual64(MatLayout L, const double* __restrict__ val, const double* __restrict__ u,
             const double* __restrict__ f, double* __restrict__ r, double* __restrict__ acc) {
  __shared__ double sh[32];
  double rr = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < L.count; t += gridDim.x * blockDim.x)
    mat_rows(L, t, val, u, [&](int row, double kv) {
      const double v = f[row] - kv;
      r[row] = v;
      rr += v * v;
    });
  double s = block_sum(rr, sh);
  if (threadIdx.x == 0) atomicAdd(acc, s);
}

// r = f - K (u_hi + u_lo) on the column-major ELL in double-double arithmetic (the
// compensated dot product "Dot2" of Ogita, Rump and Oishi, SIAM J. Sci. Comput. 26(6),
// 2005: each product split exactly with an FMA, each sum with TwoSum), rounded to FP64
// once at the end; also sum of r_i^2.  The residual of a solution held as an unevaluated
// sum u_hi + u_lo is then exact to about 2^-104 relative to max |K_ij (u_hi + u_lo)_j|,
// well below the FP64 rounding of K u itself (which bounds an FP64 residual).
__global__ void __launch_bounds__(kT)
k_residual_dd(int n, const int32_t* __restrict__ rownnz, const int32_t* __restrict__ colidx,
              const double* __restrict__ val, const double* __restrict__ uh,
              const double* __restrict__ ul, const double* __restrict__ f,
              double* __restrict__ r, double* __restrict__ acc) {
  __shared__ double sh[32];
  double rr = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = f[i], c = 0.0;
    const int len = rownnz[i];
    for (int j = 0; j < len; ++j) {
      const size_t o = (size_t)j * n + i;
      const double k = val[o];
      const int col = colidx[o];
      const double h = uh[col];
      // explicit round-to-nearest operations: no FMA contraction may merge these steps
      const double p = __dmul_rn(k, h);
      const double pe = fma(k, h, -p);   // k h = p + pe exactly
      const double t = __dsub_rn(s, p);  // TwoSum(s, -p) = t + te exactly
      const double bp = __dsub_rn(t, s);
      const double te = __dadd_rn(__dsub_rn(s, __dsub_rn(t, bp)), __dsub_rn(-p, bp));
      s = t;
      c += te - pe - k * ul[col];
    }
    const double v = s + c;
    r[i] = v;
    rr += v * v;
  }
  double b = block_sum(rr, sh);
  if (threadIdx.x == 0) atomicAdd(acc, b);
}

// ---- CG kernels ------------------------------------------------------------
template <typename V>
__global__ void __launch_bounds__(kT)
k_cg_init(int n, const V* __restrict__ b, const V* __restrict__ dinv, V* __restrict__ x,
          V* __restrict__ r, V* __restrict__ z, V* __restrict__ p, SolveScalars* sc) {
  __shared__ double sh[32];
  double rz = 0.0, rr = 0.0;
  for (int i = blockIdx.x * kT + threadIdx.x; i < n; i += gridDim.x * kT) {
    V bi = b[i];
    x[i] = V(0);
    r[i] = bi;
    V zi = dinv ? bi * dinv[i] : bi;
    z[i] = zi;
    p[i] = zi;
    rz += (double)bi * (double)zi;
    rr += (double)bi * (double)bi;
  }
  double s1 = block_sum(rz, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->rzn, s1);
  double s2 = block_sum(rr, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->rr, s2);
}

__global__ void k_cg_init_fin(SolveScalars* sc, double eps, int maxit) {
  sc->rr0 = sc->rr;
  sc->tol2 = eps * eps * sc->rr;
  sc->iter = 0;
  sc->maxit = maxit;
  sc->pq = 0.0;
  sc->done = (sc->rr <= 0.0 || sc->rr <= sc->tol2) ? 1 : (maxit <= 0 ? 3 : 0);
}

template <typename TK, typename V>
__global__ void __launch_bounds__(kT)
k_cg_spmv_dot(MatLayout L, const TK* __restrict__ val, const V* __restrict__ p,
              V* __restrict__ q, SolveScalars* sc) {
  __shared__ double sh[32];
  if (sc->done) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->rz = sc->rzn;
    sc->rzn = 0.0;
    sc->rr = 0.0;
  }
  double pq = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < L.count; t += gridDim.x * blockDim.x)
    mat_rows(L, t, val, p, [&](int row, double v) {
      q[row] = (V)v;
      pq += (double)p[row] * (double)(V)v;
    });
  double s = block_sum(pq, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->pq, s);
}

__global__ void k_copy_f32(int n, const double* __restrict__ a, float* __restrict__ b) {
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

// q = K32 p on the FP32 matrix from the FP32 copy p32 of the FP64 direction p: FP32
// products and row sums (no FP64 conversion per matrix entry, which measured 81 against
// 52 us on Q8 512), q and the p.q dot in FP64.
__global__ void __launch_bounds__(kT)
k_cg_spmv_dot_x32(MatLayout L, const float* __restrict__ val, const float* __restrict__ p32,
                  const double* __restrict__ p, double* __restrict__ q, SolveScalars* sc) {
  __shared__ double sh[32];
  if (sc->done) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->rz = sc->rzn;
    sc->rzn = 0.0;
    sc->rr = 0.0;
  }
  double pq = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < L.count; t += gridDim.x * blockDim.x)
    mat_rows(L, t, val, p32, [&](int row, double v) {
      q[row] = v;
      pq += p[row] * v;
    });
  double s = block_sum(pq, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->pq, s);
}

template <typename V>
__global__ void __launch_bounds__(kT)
k_cg_update(int n, V* __restrict__ x, V* __restrict__ r, V* __restrict__ z,
            const V* __restrict__ p, const V* __restrict__ q, const V* __restrict__ dinv,
            SolveScalars* sc) {
  __shared__ double sh[32];
  if (sc->done) return;
  const double pq = sc->pq;
  if (!(pq > 0.0) || !isfinite(pq)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->done = 2;
    return;
  }
  const V alpha = (V)(sc->rz / pq);
  double rz = 0.0, rr = 0.0;
  for (int i = blockIdx.x * kT + threadIdx.x; i < n; i += gridDim.x * kT) {
    x[i] += alpha * p[i];
    V ri = r[i] - alpha * q[i];
    r[i] = ri;
    V zi = ri;
    if (dinv) {
      zi = ri * dinv[i];
      z[i] = zi;
    }
    rz += (double)ri * (double)zi;
    rr += (double)ri * (double)ri;
  }
  double s1 = block_sum(rz, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->rzn, s1);
  double s2 = block_sum(rr, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->rr, s2);
}

template <typename V>
__global__ void __launch_bounds__(kT)
k_cg_direction(int n, const V* __restrict__ z, V* __restrict__ p, SolveScalars* sc,
               float* __restrict__ p32 = nullptr) {
  if (sc->done) return;
  const V beta = (V)(sc->rzn / sc->rz);
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i < n) {
    const V pn = z[i] + beta * p[i];
    p[i] = pn;
    if (p32) p32[i] = (float)pn;  // FP32 copy for the K32 SpMV (MIXED_PCG)
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->pq = 0.0;
    sc->iter += 1;
    if (sc->rr <= sc->tol2) sc->done = 1;
    else if (sc->iter >= sc->maxit) sc->done = 3;
  }
}

// Jacobi: 1 / K_rr (0 for an empty or zero diagonal -> identity row)
template <typename TK, typename V>
__global__ void k_diag_inv(int n, const int32_t* __restrict__ rownnz,
                           const int32_t* __restrict__ col, const TK* __restrict__ val,
                           V* __restrict__ dinv) {
  const int row = blockIdx.x * kT + threadIdx.x;
  if (row >= n) return;
  const int nz = rownnz[row];
  double d = 0.0;
  for (int s = 0; s < nz; ++s) {
    int64_t o = (int64_t)s * n + row;
    if (col[o] == row) { d = (double)val[o]; break; }
  }
  dinv[row] = (d != 0.0) ? (V)(1.0 / d) : V(1);
}

template <typename V>
__global__ void k_copy_to_f64(int n, const V* __restrict__ a, double* __restrict__ b) {
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i < n) b[i] = (double)a[i];
}

template <typename V>
__global__ void k_copy_from_f64(int n, const double* __restrict__ a, V* __restrict__ b) {
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i < n) b[i] = (V)a[i];
}

// ---- constraints -----------------------------------------------------------
template <typename T>
__global__ void k_diag_max(int nnodes, int dim, int n, const int32_t* __restrict__ diagpos,
                           const T* __restrict__ K, double* __restrict__ blockmax) {
  __shared__ double sh[32];
  double m = -INFINITY;
  for (int row = blockIdx.x * kT + threadIdx.x; row < n; row += gridDim.x * kT) {
    const int a = row / dim, c = row % dim;
    m = fmax(m, (double)K[(int64_t)(diagpos[a] * dim + c) * n + row]);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = sh[0];
    for (int k = 1; k < (kT >> 5); ++k) r = fmax(r, sh[k]);
    blockmax[blockIdx.x] = r;
  }
}

// K_dd <- (1e4 * max_i K_ii) * K_dd in the matrix precision (fem.cc:119-143).
template <typename T>
__global__ void k_penalty(int nblocks, const double* __restrict__ blockmax, int dim, int n,
                          const int32_t* __restrict__ diagpos, const uint8_t* __restrict__ fixed,
                          T* __restrict__ K) {
  __shared__ T pen;
  if (threadIdx.x == 0) {
    double m = blockmax[0];
    for (int b = 1; b < nblocks; ++b) m = fmax(m, blockmax[b]);
    pen = (T)m * (T)10000;
  }
  __syncthreads();
  for (int row = blockIdx.x * kT + threadIdx.x; row < n; row += gridDim.x * kT) {
    if (!fixed[row]) continue;
    const int a = row / dim, c = row % dim;
    T* d = &K[(int64_t)(diagpos[a] * dim + c) * n + row];
    *d = pen * *d;
  }
}

// Elimination of constrained dofs on both value arrays at once (either may be null): a
// thread per row walks its slots, so each slot's column words and values are read by
// consecutive threads; rows of fixed dofs become unit rows, columns of fixed dofs zero.
__global__ void k_eliminate(int n, const int32_t* __restrict__ rownnz,
                            const int32_t* __restrict__ col, const uint8_t* __restrict__ fixed,
                            double* __restrict__ K64, float* __restrict__ K32) {
  for (int row = blockIdx.x * kT + threadIdx.x; row < n; row += gridDim.x * kT) {
    const int nz = rownnz[row];
    const bool frow = fixed[row];
    for (int s = 0; s < nz; ++s) {
      const int64_t i = (int64_t)s * n + row;
      const int c = col[i];
      if (frow || fixed[c]) {
        if (K64) K64[i] = c == row ? 1.0 : 0.0;
        if (K32) K32[i] = c == row ? 1.f : 0.f;
      }
    }
  }
}

__global__ void k_zero_fixed(int n, const uint8_t* __restrict__ fixed, double* __restrict__ f) {
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i < n && fixed[i]) f[i] = 0.0;
}

// Grid of the reducing kernels: at most 8 CTAs per SM, rows strided over the grid, so
// that each reduction issues a few thousand global atomics at most (one per CTA).
inline int red_grid(const gf_ctx* ctx, int64_t work) {
  return std::min(gf_blocks(work, kT), ctx->sm_count * 8);
}

// grid of the SpMV kernels for layout L (block size L.threads): node blocks run one
// thread per node (measured faster than a capped grid-stride loop), rows a capped grid
inline int mat_grid(const gf_ctx* ctx, const MatLayout& L) {
  if (L.bdim) return gf_blocks(L.count, L.threads);
  return std::min(gf_blocks(L.count, L.threads), ctx->sm_count * 8);
}

// The sliced copy of the context's matrix in `dtype` (built or refreshed on demand).
gf_status solver_matrix(gf_ctx* ctx, int dtype, MatLayout* L, const void** val) {
  gf_status st = gf_sell_prepare(ctx, dtype);
  if (st != GF_OK) return st;
  *L = MatLayout{ctx->n, ctx->n, ctx->d_rownnz, ctx->d_sell_col, ctx->d_sell_w, ctx->d_sell_off};
  if (ctx->sell_bdim) {
    L->bdim = ctx->sell_bdim;
    L->nnodes = ctx->nnodes;
    L->perm = ctx->d_sell_perm;
    L->count = ctx->nnodes;  // a thread per node slot
  }
  *val = dtype == GF_F64 ? (const void*)ctx->d_sell_v64 : (const void*)ctx->d_sell_v32;
  return GF_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// y = scale .* (K x) on FP32 vectors over the solver's matrix layout (FP64 values when the
// context has them).  Enqueue only: inside a stream capture the layout must already be
// prepared (gf_sell_prepare), which makes solver_matrix a lookup.
gf_status gf_matvec_f32(gf_ctx* ctx, const float* x, const float* scale, float* y) {
  MatLayout L;
  const void* val = nullptr;
  const int dt = ctx->has64 ? GF_F64 : GF_F32;
  gf_status st = solver_matrix(ctx, dt, &L, &val);
  if (st != GF_OK) return st;
  if (dt == GF_F64)
    k_spmv_rowscale<double><<<mat_grid(ctx, L), L.threads, 0, ctx->stream>>>(
        L, (const double*)val, x, scale, y);
  else
    k_spmv_rowscale<float><<<mat_grid(ctx, L), L.threads, 0, ctx->stream>>>(
        L, (const float*)val, x, scale, y);
  ctx->launches++;
  return GF_OK;
}

gf_status gf_spmv_launch(gf_ctx* ctx, int dtype, const void* x, void* y) {
  MatLayout L;
  const void* val = nullptr;
  gf_status st = solver_matrix(ctx, dtype, &L, &val);
  if (st != GF_OK) return st;
  // 2-D node blocks read x in pairs (one 8- or 16-byte load per neighbour node)
  if (L.bdim == 2 && ((uintptr_t)x % (dtype == GF_F64 ? 16 : 8)) != 0)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "x must be aligned to two entries");
  cudaEventRecord(ctx->ev0, ctx->stream);
  if (dtype == GF_F64)
    k_spmv<double, double, double><<<mat_grid(ctx, L), L.threads, 0, ctx->stream>>>(
        L, (const double*)val, (const double*)x, (double*)y);
  else
    k_spmv<float, float, float><<<mat_grid(ctx, L), L.threads, 0, ctx->stream>>>(
        L, (const float*)val, (const float*)x, (float*)y);
  GF_LAUNCH_CHECK(ctx, "k_spmv");
  cudaEventRecord(ctx->ev1, ctx->stream);
  GF_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  ctx->last_seconds = ms * 1e-3;
  return GF_OK;
}

gf_status gf_constraints_apply(gf_ctx* ctx, int mode) {
  const int n = ctx->n;
  if (mode == GF_BC_PENALTY) {
    if (!ctx->d_diagpos)
      return gf_fail(ctx, GF_ERR_STATE, "penalty needs a mesh-built pattern");
    const int nb = std::min(gf_blocks(n, kT), 1024);
    double* d_bmax = nullptr;
    gf_status st = gf_alloc(ctx, &d_bmax, (size_t)nb);
    if (st != GF_OK) return st;
    if (ctx->has64) {
      k_diag_max<double><<<nb, kT, 0, ctx->stream>>>(ctx->nnodes, ctx->dim, n, ctx->d_diagpos,
                                                     ctx->d_K64, d_bmax);
      ctx->launches++;
      k_penalty<double><<<nb, kT, 0, ctx->stream>>>(nb, d_bmax, ctx->dim, n, ctx->d_diagpos,
                                                    ctx->d_fixed, ctx->d_K64);
      ctx->launches++;
    }
    if (ctx->has32) {
      k_diag_max<float><<<nb, kT, 0, ctx->stream>>>(ctx->nnodes, ctx->dim, n, ctx->d_diagpos,
                                                    ctx->d_K32, d_bmax);
      ctx->launches++;
      k_penalty<float><<<nb, kT, 0, ctx->stream>>>(nb, d_bmax, ctx->dim, n, ctx->d_diagpos,
                                                   ctx->d_fixed, ctx->d_K32);
      ctx->launches++;
    }
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d_bmax);
    if (e != cudaSuccess) return gf_cuda_fail(ctx, e, "penalty");
  } else {
    k_eliminate<<<gf_blocks(n, kT), kT, 0, ctx->stream>>>(
        n, ctx->d_rownnz, ctx->d_colidx, ctx->d_fixed, ctx->has64 ? ctx->d_K64 : nullptr,
        ctx->has32 ? ctx->d_K32 : nullptr);
    ctx->launches++;
    k_zero_fixed<<<gf_blocks(n, kT), kT, 0, ctx->stream>>>(n, ctx->d_fixed, ctx->d_f);
    ctx->launches++;
    GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  GF_CUDA(ctx, cudaGetLastError());
  ctx->bc_mode_applied = mode;
  ctx->kver64++;
  ctx->kver32++;
  return GF_OK;
}

void gf_solver_free(gf_ctx* ctx) {
  gf_free(ctx->d_u);
  if (ctx->d_work) { cudaFree(ctx->d_work); ctx->d_work = nullptr; }
  ctx->work_bytes = 0;
  gf_free(ctx->d_scal);
  gf_free(ctx->d_red);
  if (ctx->d_fcg) { cudaFree(ctx->d_fcg); ctx->d_fcg = nullptr; }
  if (ctx->h_pinned) { cudaFreeHost(ctx->h_pinned); ctx->h_pinned = nullptr; }
}

namespace {

struct CgVecs {
  void *x, *r, *z, *p, *q, *dinv;
};

// Runs (P)CG on matrix values `val` (TK) with vectors of type V until the
// device flag says done.  b must already be in vecs.r's type (copied into x's
// buffer by the caller as `b`).  Returns iterations and final done code.
template <typename TK, typename V>
gf_status run_cg(gf_ctx* ctx, MatLayout L, const TK* val, const V* b, CgVecs vv, bool precond,
                 double eps,
                 int maxit, int check_every, double max_seconds,
                 std::chrono::steady_clock::time_point t0, int* iters, int* done_code,
                 double* rr_final, double* rr0_out) {
  const int n = ctx->n;
  const int nb = gf_blocks(n, kT);
  cudaStream_t s = ctx->stream;
  SolveScalars* sc = ctx->d_scal;
  V *x = (V*)vv.x, *r = (V*)vv.r, *z = (V*)vv.z, *p = (V*)vv.p, *q = (V*)vv.q;
  const V* dinv = precond ? (const V*)vv.dinv : nullptr;
  V* zz = precond ? z : r;  // without a preconditioner z aliases r
  GF_CUDA(ctx, cudaMemsetAsync(sc, 0, sizeof(SolveScalars), s));
  k_cg_init<V><<<red_grid(ctx, n), kT, 0, s>>>(n, b, dinv, x, r, zz, p, sc);
  GF_LAUNCH_CHECK(ctx, "k_cg_init");
  k_cg_init_fin<<<1, 1, 0, s>>>(sc, eps, maxit);
  GF_LAUNCH_CHECK(ctx, "k_cg_init_fin");

  // capture one chunk of iterations as a graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  GF_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  for (int k = 0; k < check_every; ++k) {
    k_cg_spmv_dot<TK, V><<<mat_grid(ctx, L), L.threads, 0, s>>>(L, val, p, q, sc);
    k_cg_update<V><<<red_grid(ctx, n), kT, 0, s>>>(n, x, r, zz, p, q, dinv, sc);
    k_cg_direction<V><<<nb, kT, 0, s>>>(n, zz, p, sc);
  }
  cudaError_t ce = cudaStreamEndCapture(s, &graph);
  if (ce != cudaSuccess) return gf_cuda_fail(ctx, ce, "graph capture");
  ce = cudaGraphInstantiate(&exec, graph, 0);
  if (ce != cudaSuccess) {
    cudaGraphDestroy(graph);
    return gf_cuda_fail(ctx, ce, "graph instantiate");
  }
  SolveScalars* hs = (SolveScalars*)ctx->h_pinned;
  gf_status st = GF_OK;
  for (;;) {
    ce = cudaGraphLaunch(exec, s);
    if (ce != cudaSuccess) { st = gf_cuda_fail(ctx, ce, "graph launch"); break; }
    ctx->launches += 3 * check_every;
    ce = cudaMemcpyAsync(hs, sc, sizeof(SolveScalars), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) { st = gf_cuda_fail(ctx, ce, "cg chunk"); break; }
    if (hs->done) break;
    if (max_seconds > 0.0) {
      double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (el > max_seconds) break;
    }
  }
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  if (st != GF_OK) return st;
  *iters = hs->iter;
  *done_code = hs->done;
  *rr_final = hs->rr;
  *rr0_out = hs->rr0;
  return GF_OK;
}

gf_status ensure_work(gf_ctx* ctx) {
  const size_t need = (size_t)ctx->n * 8 * 10 + 256;
  gf_status st;
  if (ctx->work_bytes < need) {
    if (ctx->d_work) cudaFree(ctx->d_work);
    ctx->d_work = nullptr;
    ctx->work_bytes = 0;
    if (cudaMalloc(&ctx->d_work, need) != cudaSuccess) {
      cudaGetLastError();
      return gf_fail(ctx, GF_ERR_OOM, "solver work vectors (%zu bytes)", need);
    }
    ctx->work_bytes = need;
  }
  if (!ctx->d_u && (st = gf_alloc(ctx, &ctx->d_u, (size_t)ctx->n)) != GF_OK) return st;
  if (!ctx->d_scal && (st = gf_alloc(ctx, &ctx->d_scal, 1)) != GF_OK) return st;
  if (!ctx->d_red && (st = gf_alloc(ctx, &ctx->d_red, 4)) != GF_OK) return st;
  if (!ctx->h_pinned) {
    if (cudaMallocHost(&ctx->h_pinned, 256) != cudaSuccess) {
      cudaGetLastError();
      return gf_fail(ctx, GF_ERR_OOM, "pinned scalars");
    }
  }
  return GF_OK;
}

// ||f - K64 u|| in FP64 into r64; returns r.r
gf_status residual64(gf_ctx* ctx, double* r64, double* rr) {
  cudaStream_t s = ctx->stream;
  GF_CUDA(ctx, cudaMemsetAsync(ctx->d_red, 0, sizeof(double), s));
  MatLayout L;
  const void* val = nullptr;
  gf_status st = solver_matrix(ctx, GF_F64, &L, &val);
  if (st != GF_OK) return st;
  k_residual64<<<mat_grid(ctx, L), L.threads, 0, s>>>(L, (const double*)val, ctx->d_u, ctx->d_f,
                                                     r64, ctx->d_red);
  GF_LAUNCH_CHECK(ctx, "k_residual64");
  double* h = (double*)ctx->h_pinned + 16;
  GF_CUDA(ctx, cudaMemcpyAsync(h, ctx->d_red, sizeof(double), cudaMemcpyDeviceToHost, s));
  GF_CUDA(ctx, cudaStreamSynchronize(s));
  *rr = *h;
  return GF_OK;
}

gf_status status_of(int done) {
  return done == 1 ? GF_OK : done == 2 ? GF_ERR_STALLED : GF_ERR_NOT_CONVERGED;
}

}  // namespace

// ---------------------------------------------------------------------------
// Mixed precision: Jacobi-PCG on the FP32 matrix K32 whose residual is recomputed
// on the FP64 matrix ("reliable updates").  The vectors x, r, z, p, q are FP64
// (GF_SOLVER_MIXED_PCG) or FP32 (GF_SOLVER_MIXED_PCG32); they are scaled by the
// norm sigma of the FP64 residual at the last update, and the solution
// accumulates in FP64 (u += sigma x).  When the recursive residual has dropped by
// 10x since the last update (or the recursion reports convergence / breakdown /
// the iteration cap, or a segment ran longer than its cap), the host triggers an
// update: u += sigma x, r64 = f - K64 u in FP64, and the recursion continues from
// r64 / ||r64|| with the search direction rescaled and kept, so the Krylov process
// is not restarted.  Convergence is decided on the true FP64 residual only.  When
// the true residual stops halving between updates (the rounding of K to FP32
// matters at this condition number), the correction is finished by FP64 PCG.
namespace {

template <typename V>
__global__ void k_mixed_accumulate(int n, double sigma, V* __restrict__ x,
                                   double* __restrict__ u) {
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i < n) {
    u[i] += sigma * (double)x[i];
    x[i] = V(0);
  }
}

template <typename V>
__global__ void k_mixed_reset(int n, const double* __restrict__ r64, double inv, V pscale,
                              int restart, const V* __restrict__ dinv, V* __restrict__ r,
                              V* __restrict__ z, V* __restrict__ p, SolveScalars* sc,
                              float* __restrict__ p32) {
  __shared__ double sh[32];
  double rz = 0.0, rr = 0.0;
  for (int i = blockIdx.x * kT + threadIdx.x; i < n; i += gridDim.x * kT) {
    const V ri = (V)(r64[i] * inv);
    const V zi = ri * dinv[i];
    r[i] = ri;
    z[i] = zi;
    const V pn = restart ? zi : p[i] * pscale;
    p[i] = pn;
    if (p32) p32[i] = (float)pn;
    rz += (double)ri * (double)zi;
    rr += (double)ri * (double)ri;
  }
  double s1 = block_sum(rz, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->rzn, s1);
  double s2 = block_sum(rr, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->rr, s2);
}

template <typename V>
__global__ void k_scale_to(int n, const double* __restrict__ a, double s, V* __restrict__ b) {
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i < n) b[i] = (V)(a[i] * s);
}

__global__ void k_add64(int n, const double* __restrict__ d, double* __restrict__ u) {
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i < n) u[i] += d[i];
}

__global__ void k_mixed_scalars(SolveScalars* sc, double tol2) {
  sc->tol2 = tol2;
  sc->pq = 0.0;
  sc->done = sc->iter >= sc->maxit ? 3 : 0;
}

// twolevel: the two-level preconditioner (gf_twolevel.cu) in place of Jacobi, in the
// recursion and at every reliable update.  V = double: FP64 vectors with an FP32 copy of
// the direction for the K32 SpMV; V = float: FP32 vectors throughout the recursion (the
// direction is the SpMV operand itself), with the dot products and scalars in FP64.
template <typename V>
gf_status run_mixed(gf_ctx* ctx, const gf_solve_opts* o, int maxit, int check,
                    std::chrono::steady_clock::time_point t0, gf_solve_info* info,
                    bool twolevel = false) {
  const int n = ctx->n;
  const int nb = gf_blocks(n, kT);
  cudaStream_t s = ctx->stream;
  SolveScalars* sc = ctx->d_scal;
  SolveScalars* hs = (SolveScalars*)ctx->h_pinned;
  double* r64 = (double*)ctx->d_work;
  V* v = reinterpret_cast<V*>(r64 + n);
  V *x = v, *r = v + n, *z = v + 2 * (size_t)n, *p = v + 3 * (size_t)n, *q = v + 4 * (size_t)n;
  V* dinv = v + 5 * (size_t)n;
  const double tol = o->tol;
  const double delta2 = 0.01;  // update when ||r|| fell 10x since the last update
  gf_status st;
  MatLayout L32, L64;
  const void *v32 = nullptr, *v64 = nullptr;
  if ((st = solver_matrix(ctx, GF_F32, &L32, &v32)) != GF_OK) return st;
  if ((st = solver_matrix(ctx, GF_F64, &L64, &v64)) != GF_OK) return st;
  const float* val32 = (const float*)v32;
  if (twolevel && (st = gf_coarse_prepare(ctx, 0)) != GF_OK) return st;
  // FP32 copy of the FP64 direction for the K32 SpMV: the two-level recursion never
  // stores z, so its room holds it; Jacobi uses the work area past dinv (10 n doubles)
  float* p32 = sizeof(V) != sizeof(double) ? nullptr
               : twolevel ? reinterpret_cast<float*>(z) : reinterpret_cast<float*>(v + 6 * (size_t)n);
  k_diag_inv<double, V><<<nb, kT, 0, s>>>(n, ctx->d_rownnz, ctx->d_colidx, ctx->d_K64, dinv);
  GF_LAUNCH_CHECK(ctx, "k_diag_inv");
  GF_CUDA(ctx, cudaMemsetAsync(ctx->d_u, 0, sizeof(double) * n, s));
  double ff = 0.0;
  if ((st = residual64(ctx, r64, &ff)) != GF_OK) return st;  // u = 0: r64 = f
  double rr64 = ff;
  int updates = 0, done_code = 1, fp32_iters = 0, fp64_iters = 0;
  bool fp64_fallback = false;
  if (ff > 0.0) {
    double sigma = std::sqrt(ff);
    GF_CUDA(ctx, cudaMemsetAsync(sc, 0, sizeof(SolveScalars), s));
    if (twolevel) {
      if constexpr (sizeof(V) == sizeof(double))
        gf_tl_reset(ctx, r64, 1.0 / sigma, true, 1.0, x, r, p, dinv, sc, p32);
      else
        gf_tl_reset(ctx, r64, 1.0 / sigma, true, 1.0, x, r, p, dinv, sc);
      GF_LAUNCH_CHECK(ctx, "gf_tl_reset");
    } else {
      k_scale_to<V><<<nb, kT, 0, s>>>(n, r64, 1.0 / sigma, q);  // q: scratch until K1
      GF_LAUNCH_CHECK(ctx, "k_scale_to");
      k_cg_init<V><<<red_grid(ctx, n), kT, 0, s>>>(n, q, dinv, x, r, z, p, sc);
      GF_LAUNCH_CHECK(ctx, "k_cg_init");
      if (p32) {
        k_copy_f32<<<nb, kT, 0, s>>>(n, (const double*)p, p32);
        GF_LAUNCH_CHECK(ctx, "k_copy_f32");
      }
    }
    k_cg_init_fin<<<1, 1, 0, s>>>(sc, tol, maxit);
    GF_LAUNCH_CHECK(ctx, "k_cg_init_fin");
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    GF_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const int64_t l0 = ctx->launches;
    for (int k = 0; k < check; ++k) {
      if (twolevel) {
        if constexpr (sizeof(V) == sizeof(double)) {
          k_cg_spmv_dot_x32<<<mat_grid(ctx, L32), L32.threads, 0, s>>>(L32, val32, p32, p, q, sc);
          gf_tl_iterate(ctx, x, r, p, q, dinv, sc, p32);
        } else {
          k_cg_spmv_dot<float, V><<<mat_grid(ctx, L32), L32.threads, 0, s>>>(L32, val32, p, q, sc);
          gf_tl_iterate(ctx, x, r, p, q, dinv, sc);
        }
      } else {
        if (p32)
          k_cg_spmv_dot_x32<<<mat_grid(ctx, L32), L32.threads, 0, s>>>(
              L32, val32, p32, (const double*)p, (double*)q, sc);
        else
          k_cg_spmv_dot<float, V><<<mat_grid(ctx, L32), L32.threads, 0, s>>>(L32, val32, p, q, sc);
        k_cg_update<V><<<red_grid(ctx, n), kT, 0, s>>>(n, x, r, z, p, q, dinv, sc);
        k_cg_direction<V><<<nb, kT, 0, s>>>(n, z, p, sc, p32);
      }
    }
    const int64_t per_chunk = twolevel ? ctx->launches - l0 + check : 3 * (int64_t)check;
    ctx->launches = l0;
    cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (ce != cudaSuccess) return gf_cuda_fail(ctx, ce, "graph capture");
    ce = cudaGraphInstantiate(&exec, graph, 0);
    if (ce != cudaSuccess) {
      cudaGraphDestroy(graph);
      return gf_cuda_fail(ctx, ce, "graph instantiate");
    }
    double rr_max = 1.0, prev_rr64 = ff;
    int breakdowns = 0, stagnant = 0, seg_start = 0;
    // a segment between updates longer than this is cut short, so that a recursion
    // that no longer reduces its residual still reaches the stagnation test
    const int seg_cap = std::max(1000, 2 * (int)std::sqrt((double)n));
    done_code = 3;
    for (;;) {
      ce = cudaGraphLaunch(exec, s);
      if (ce == cudaSuccess) ce = cudaMemcpyAsync(hs, sc, sizeof(SolveScalars), cudaMemcpyDeviceToHost, s);
      if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
      if (ce != cudaSuccess) { st = gf_cuda_fail(ctx, ce, "mixed chunk"); break; }
      ctx->launches += per_chunk;
      const bool timeout = o->max_seconds > 0.0 &&
          std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > o->max_seconds;
      // growth of the FP32 residual by 100x over its value at the last update means
      // the FP32 recursion is diverging (K32 nearly indefinite for very ill-conditioned
      // systems): update and restart the direction
      const bool diverging = hs->done == 0 && hs->rr > 1e4;
      const bool long_segment = hs->iter - seg_start >= seg_cap;
      if (hs->done == 0 && hs->rr > delta2 * rr_max && !timeout && !diverging && !long_segment) {
        rr_max = std::max(rr_max, hs->rr);
        continue;
      }
      // reliable update
      k_mixed_accumulate<V><<<nb, kT, 0, s>>>(n, sigma, x, ctx->d_u);
      ce = cudaGetLastError();
      if (ce != cudaSuccess) { st = gf_cuda_fail(ctx, ce, "k_mixed_accumulate"); break; }
      ctx->launches++;
      if ((st = residual64(ctx, r64, &rr64)) != GF_OK) break;
      ++updates;
      if (std::sqrt(rr64 / ff) <= tol) { done_code = 1; break; }
      if (hs->done == 3 || timeout) { done_code = 3; break; }
      // the true residual must at least halve between updates; three misses in a
      // row mean the FP32 matrix (or FP32 recursion) cannot resolve this system: finish
      // in FP64
      stagnant = rr64 > 0.25 * prev_rr64 ? stagnant + 1 : 0;
      prev_rr64 = rr64;
      if (stagnant >= 3) { fp64_fallback = true; break; }
      // with the two-level preconditioner a chunk can take the recursion far past the
      // 10x trigger, down to its own convergence: its direction is spent, so restart
      const bool restart = hs->done == 2 || diverging ||
                           (twolevel && (hs->done == 1 || hs->rr < 1e-12));
      if (restart && ++breakdowns > 50) { done_code = 2; break; }
      const double sigma_new = std::sqrt(rr64);
      ce = cudaMemsetAsync(&sc->rzn, 0, 2 * sizeof(double), s);  // rzn, rr
      if (ce != cudaSuccess) { st = gf_cuda_fail(ctx, ce, "reset"); break; }
      // done flag and pq first: the two-level kernels skip their work while done != 0
      k_mixed_scalars<<<1, 1, 0, s>>>(sc, tol * tol * ff / rr64);
      if (twolevel) {
        if constexpr (sizeof(V) == sizeof(double))
          gf_tl_reset(ctx, r64, 1.0 / sigma_new, restart, sigma / sigma_new, x, r, p, dinv, sc,
                      p32);
        else
          gf_tl_reset(ctx, r64, 1.0 / sigma_new, restart, sigma / sigma_new, x, r, p, dinv, sc);
      } else
        k_mixed_reset<V><<<red_grid(ctx, n), kT, 0, s>>>(n, r64, 1.0 / sigma_new,
                                                         (V)(sigma / sigma_new), restart ? 1 : 0,
                                                         dinv, r, z, p, sc, p32);
      ce = cudaGetLastError();
      if (ce != cudaSuccess) { st = gf_cuda_fail(ctx, ce, "k_mixed_reset"); break; }
      ctx->launches += twolevel ? 1 : 2;  // gf_tl_reset counts its own
      sigma = sigma_new;
      rr_max = 1.0;
      seg_start = hs->iter;
    }
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (st != GF_OK) return st;
    fp32_iters = hs->iter;
    if (fp64_fallback) {
      // FP64 Jacobi-PCG on the correction K64 d = r64, then u += d
      double* w64 = (double*)ctx->d_work;
      double* b = w64 + 7 * (size_t)n;
      GF_CUDA(ctx, cudaMemcpyAsync(b, r64, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
      CgVecs vv{w64, w64 + n, w64 + 2 * (size_t)n, w64 + 3 * (size_t)n, w64 + 4 * (size_t)n,
                w64 + 5 * (size_t)n};
      k_diag_inv<double, double><<<nb, kT, 0, s>>>(n, ctx->d_rownnz, ctx->d_colidx, ctx->d_K64,
                                                   (double*)vv.dinv);
      GF_LAUNCH_CHECK(ctx, "k_diag_inv");
      int it2 = 0, done2 = 0;
      double rr2 = 0.0, rr02 = 0.0;
      st = run_cg<double, double>(ctx, L64, (const double*)v64, b, vv, true,
                                  tol * std::sqrt(ff / rr64),
                                  std::max(1, maxit - fp32_iters), check, o->max_seconds, t0,
                                  &it2, &done2, &rr2, &rr02);
      if (st != GF_OK) return st;
      k_add64<<<nb, kT, 0, s>>>(n, (const double*)vv.x, ctx->d_u);
      GF_LAUNCH_CHECK(ctx, "k_add64");
      if ((st = residual64(ctx, r64, &rr64)) != GF_OK) return st;
      fp64_iters = it2;
      done_code = std::sqrt(rr64 / ff) <= tol * 1.01 ? 1 : done2;
    }
  }
  cudaEventRecord(ctx->ev1, s);
  GF_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  info->seconds = ctx->last_seconds = ms * 1e-3;
  info->iterations = fp32_iters + fp64_iters;
  info->fallback = fp64_fallback ? 1 : 0;
  info->outer = updates;
  info->rel_residual = ff > 0.0 ? std::sqrt(rr64 / ff) : 0.0;
  info->status = status_of(done_code);
  if (done_code != 1)
    gf_fail(ctx, (gf_status)info->status, "mixed solve stopped with code %d (%d iterations)",
            done_code, info->iterations);
  return (gf_status)info->status;
}

}  // namespace

// ---------------------------------------------------------------------------
// Flexible CG (Notay's FCG(1): Polak-Ribiere beta, alpha = p.r / p.K p) in FP64
// with a variable preconditioner: the learned network (gf_learned.cu), or Jacobi
// after a fallback.  Jacobi-PCG takes over — restarting the search direction from
// the current iterate — when the learned preconditioner breaks down (z.r <= 0 or
// p.Kp <= 0) or stalls (no net residual reduction over 512 iterations).
// Convergence is decided on the FP64 residual.
namespace {

struct FcgScalars {
  double zr, zrp, zr_prev, pq, pr, rr, rr0, tol2;
  int iter, done, maxit, first;
};

__global__ void k_fcg_init(int n, const double* __restrict__ f, double* __restrict__ x,
                           double* __restrict__ r, double* __restrict__ rold, FcgScalars* sc) {
  __shared__ double sh[32];
  double rr = 0.0;
  for (int i = blockIdx.x * kT + threadIdx.x; i < n; i += gridDim.x * kT) {
    x[i] = 0.0;
    r[i] = f[i];
    rold[i] = 0.0;
    rr += f[i] * f[i];
  }
  double s1 = block_sum(rr, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->rr, s1);
}

__global__ void k_fcg_init_fin(FcgScalars* sc, double tol, int maxit) {
  sc->rr0 = sc->rr;
  sc->tol2 = tol * tol * sc->rr;
  sc->iter = 0;
  sc->maxit = maxit;
  sc->first = 1;
  sc->zr_prev = 1.0;
  sc->zr = sc->zrp = sc->pq = sc->pr = 0.0;
  sc->done = (sc->rr <= 0.0) ? 1 : (maxit <= 0 ? 3 : 0);
}

__global__ void k_fcg_jacobi(int n, const double* __restrict__ r, const double* __restrict__ dinv,
                             double* __restrict__ z, const FcgScalars* sc) {
  if (sc->done) return;
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i < n) z[i] = r[i] * dinv[i];
}

__global__ void k_fcg_dots(int n, const double* __restrict__ z, const double* __restrict__ r,
                           const double* __restrict__ rold, FcgScalars* sc) {
  __shared__ double sh[32];
  if (sc->done) return;
  double a = 0.0, b = 0.0;
  for (int i = blockIdx.x * kT + threadIdx.x; i < n; i += gridDim.x * kT) {
    a += z[i] * r[i];
    b += z[i] * rold[i];
  }
  double s1 = block_sum(a, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->zr, s1);
  double s2 = block_sum(b, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->zrp, s2);
}

__global__ void k_fcg_dir(int n, const double* __restrict__ z, double* __restrict__ p,
                          FcgScalars* sc) {
  if (sc->done) return;
  if (!(sc->zr > 0.0) || !isfinite(sc->zr)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->done = 2;
    return;
  }
  const double beta = sc->first ? 0.0 : (sc->zr - sc->zrp) / sc->zr_prev;
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i < n) p[i] = z[i] + beta * p[i];
}

__global__ void __launch_bounds__(kT)
k_fcg_spmv(MatLayout L, const double* __restrict__ val, const double* __restrict__ p,
           const double* __restrict__ r, double* __restrict__ q, FcgScalars* sc) {
  __shared__ double sh[32];
  if (sc->done) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) sc->rr = 0.0;
  double pq = 0.0, pr = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < L.count; t += gridDim.x * blockDim.x)
    mat_rows(L, t, val, p, [&](int row, double v) {
      q[row] = v;
      pq += p[row] * v;
      pr += p[row] * r[row];
    });
  double s1 = block_sum(pq, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->pq, s1);
  double s2 = block_sum(pr, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->pr, s2);
}

__global__ void k_fcg_update(int n, double* __restrict__ x, double* __restrict__ r,
                             double* __restrict__ rold, const double* __restrict__ p,
                             const double* __restrict__ q, FcgScalars* sc) {
  __shared__ double sh[32];
  if (sc->done) return;
  if (!(sc->pq > 0.0) || !isfinite(sc->pq)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->done = 2;
    return;
  }
  const double alpha = sc->pr / sc->pq;
  double rr = 0.0;
  for (int i = blockIdx.x * kT + threadIdx.x; i < n; i += gridDim.x * kT) {
    x[i] += alpha * p[i];
    const double ri = r[i];
    rold[i] = ri;
    const double rn = ri - alpha * q[i];
    r[i] = rn;
    rr += rn * rn;
  }
  double s = block_sum(rr, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->rr, s);
}

__global__ void k_fcg_finish(FcgScalars* sc) {
  if (sc->done) return;
  sc->zr_prev = sc->zr;
  sc->zr = sc->zrp = sc->pq = sc->pr = 0.0;
  sc->first = 0;
  sc->iter += 1;
  if (sc->rr <= sc->tol2) sc->done = 1;
  else if (sc->iter >= sc->maxit) sc->done = 3;
}

__global__ void k_fcg_restart(FcgScalars* sc) {
  sc->first = 1;
  sc->zr = sc->zrp = sc->pq = sc->pr = 0.0;
  sc->done = sc->iter >= sc->maxit ? 3 : 0;
}

__global__ void k_sub_f32(int n, const double* __restrict__ a, float* __restrict__ b) {
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i < n) b[i] = (float)((double)b[i] - a[i]);
}

__global__ void k_record_pair(int n, const double* __restrict__ r, const double* __restrict__ x,
                              const double* __restrict__ ustar, float* __restrict__ rout,
                              float* __restrict__ eout) {
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i < n) {
    rout[i] = (float)r[i];
    eout[i] = (float)(ustar[i] - x[i]);
  }
}

gf_status run_fcg(gf_ctx* ctx, const gf_solve_opts* o, int maxit, int check,
                  std::chrono::steady_clock::time_point t0, gf_solve_info* info) {
  const int n = ctx->n;
  const int nb = gf_blocks(n, kT);
  cudaStream_t s = ctx->stream;
  gf_status st;
  if (!ctx->lp) return gf_fail(ctx, GF_ERR_STATE, "learned preconditioner not initialised (gf_lp_init)");
  const bool learned = true;
  const bool coarse = gf_lp_coarse(ctx);
  if ((st = gf_lp_prepare(ctx)) != GF_OK) return st;
  if (coarse && (st = gf_coarse_prepare(ctx, 0)) != GF_OK) return st;
  if (!ctx->d_fcg) {
    if (cudaMalloc(&ctx->d_fcg, sizeof(FcgScalars)) != cudaSuccess) {
      cudaGetLastError();
      return gf_fail(ctx, GF_ERR_OOM, "FCG scalars");
    }
  }
  FcgScalars* sc = static_cast<FcgScalars*>(ctx->d_fcg);
  FcgScalars hs{};
  double* w = (double*)ctx->d_work;
  double *x = w, *r = w + n, *rold = w + 2 * (size_t)n, *z = w + 3 * (size_t)n;
  double *p = w + 4 * (size_t)n, *q = w + 5 * (size_t)n, *dinv = w + 6 * (size_t)n;
  float* r32 = reinterpret_cast<float*>(w + 7 * (size_t)n);
  MatLayout L;
  const void* vv = nullptr;
  if ((st = solver_matrix(ctx, GF_F64, &L, &vv)) != GF_OK) return st;
  const double* val = (const double*)vv;
  k_diag_inv<double, double><<<nb, kT, 0, s>>>(n, ctx->d_rownnz, ctx->d_colidx, ctx->d_K64, dinv);
  GF_LAUNCH_CHECK(ctx, "k_diag_inv");
  GF_CUDA(ctx, cudaMemsetAsync(sc, 0, sizeof(FcgScalars), s));
  k_fcg_init<<<red_grid(ctx, n), kT, 0, s>>>(n, ctx->d_f, x, r, rold, sc);
  k_fcg_init_fin<<<1, 1, 0, s>>>(sc, o->tol, maxit);
  GF_LAUNCH_CHECK(ctx, "k_fcg_init");
  // two chunk graphs: learned preconditioner and Jacobi
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  cudaGraph_t graph[2] = {nullptr, nullptr};
  for (int kind = learned ? 0 : 1; kind < 2; ++kind) {
    GF_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < check; ++k) {
      // M: the network (kind 0) or Jacobi (kind 1), plus the coarse correction if enabled
      if (kind == 0) {
        gf_lp_apply64(ctx, r, r32, z);
        if (coarse) gf_coarse_add(ctx, r, z);
      } else if (coarse) {
        gf_coarse_apply(ctx, r, dinv, z, nullptr, nullptr);
      } else {
        k_fcg_jacobi<<<nb, kT, 0, s>>>(n, r, dinv, z, sc);
      }
      k_fcg_dots<<<red_grid(ctx, n), kT, 0, s>>>(n, z, r, rold, sc);
      k_fcg_dir<<<nb, kT, 0, s>>>(n, z, p, sc);
      k_fcg_spmv<<<mat_grid(ctx, L), L.threads, 0, s>>>(L, val, p, r, q, sc);
      k_fcg_update<<<red_grid(ctx, n), kT, 0, s>>>(n, x, r, rold, p, q, sc);
      k_fcg_finish<<<1, 1, 0, s>>>(sc);
    }
    cudaError_t ce = cudaStreamEndCapture(s, &graph[kind]);
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&exec[kind], graph[kind], 0);
    if (ce != cudaSuccess) {
      for (int k2 = 0; k2 < 2; ++k2) {
        if (exec[k2]) cudaGraphExecDestroy(exec[k2]);
        if (graph[k2]) cudaGraphDestroy(graph[k2]);
      }
      return gf_cuda_fail(ctx, ce, "FCG graph");
    }
  }
  int mode = learned ? 0 : 1;
  int fallback = learned ? 0 : 1;
  std::vector<std::pair<int, double>> hist;  // (iteration, rr) at chunk ends
  st = GF_OK;
  for (;;) {
    cudaError_t ce = cudaGraphLaunch(exec[mode], s);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(&hs, sc, sizeof(FcgScalars), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) { st = gf_cuda_fail(ctx, ce, "FCG chunk"); break; }
    ctx->launches += (int64_t)check * (mode == 0 ? 20 : 6);
    if (hs.done == 1 || hs.done == 3) break;
    const bool timeout = o->max_seconds > 0.0 &&
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > o->max_seconds;
    if (timeout) { hs.done = 3; break; }
    bool stall = false;
    if (mode == 0) {
      hist.emplace_back(hs.iter, hs.rr);
      for (const auto& h : hist)
        if (hs.iter - h.first >= 512 && hs.iter - h.first < 512 + check && hs.rr >= h.second)
          stall = true;  // no net reduction of ||r|| over 512 iterations
    }
    if (hs.done == 2 || stall) {
      if (mode == 1) break;  // Jacobi-PCG itself broke down
      mode = 1;
      fallback = 1;
      k_fcg_restart<<<1, 1, 0, s>>>(sc);
      ce = cudaGetLastError();
      if (ce != cudaSuccess) { st = gf_cuda_fail(ctx, ce, "FCG restart"); break; }
    }
  }
  for (int k2 = 0; k2 < 2; ++k2) {
    if (exec[k2]) cudaGraphExecDestroy(exec[k2]);
    if (graph[k2]) cudaGraphDestroy(graph[k2]);
  }
  if (st != GF_OK) return st;
  GF_CUDA(ctx, cudaMemcpyAsync(ctx->d_u, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  double rrt = 0.0;
  double* rtrue = q;  // q is free now
  if ((st = residual64(ctx, rtrue, &rrt)) != GF_OK) return st;
  cudaEventRecord(ctx->ev1, s);
  GF_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  info->seconds = ctx->last_seconds = ms * 1e-3;
  info->iterations = hs.iter;
  info->outer = 1;
  info->fallback = fallback && learned ? 1 : 0;
  info->rel_residual = hs.rr0 > 0.0 ? std::sqrt(rrt / hs.rr0) : 0.0;
  info->status = status_of(hs.done);
  if (hs.done != 1)
    gf_fail(ctx, (gf_status)info->status, "FCG stopped with code %d after %d iterations", hs.done,
            hs.iter);
  return (gf_status)info->status;
}

}  // namespace

gf_status gf_pcg_record(gf_ctx* ctx, const double* ustar, int npairs, int every, double tol,
                        int maxit, float* r_out, float* e_out, int* recorded, bool twolevel) {
  *recorded = 0;
  if (!ctx->has64) return gf_fail(ctx, GF_ERR_STATE, "recording needs the FP64 matrix");
  gf_status st;
  if ((st = ensure_work(ctx)) != GF_OK) return st;
  const int n = ctx->n;
  const int nb = gf_blocks(n, kT);
  cudaStream_t s = ctx->stream;
  SolveScalars* sc = ctx->d_scal;
  SolveScalars* hs = (SolveScalars*)ctx->h_pinned;
  double* v = (double*)ctx->d_work;
  double *x = v, *r = v + n, *z = v + 2 * (size_t)n, *p = v + 3 * (size_t)n, *q = v + 4 * (size_t)n;
  double* dinv = v + 5 * (size_t)n;
  MatLayout L;
  const void* vk = nullptr;
  if ((st = solver_matrix(ctx, GF_F64, &L, &vk)) != GF_OK) return st;
  if (twolevel && (st = gf_coarse_prepare(ctx, 0)) != GF_OK) return st;
  k_diag_inv<double, double><<<nb, kT, 0, s>>>(n, ctx->d_rownnz, ctx->d_colidx, ctx->d_K64, dinv);
  GF_CUDA(ctx, cudaMemsetAsync(sc, 0, sizeof(SolveScalars), s));
  if (twolevel) gf_tl_begin(ctx, ctx->d_f, x, r, p, dinv, sc);
  else k_cg_init<double><<<red_grid(ctx, n), kT, 0, s>>>(n, ctx->d_f, dinv, x, r, z, p, sc);
  k_cg_init_fin<<<1, 1, 0, s>>>(sc, tol, maxit);
  GF_LAUNCH_CHECK(ctx, "k_cg_init");
  // pair k: r_k, and the error e_k = u* - x_k; with the two-level iteration the coarse
  // correction of r_k is taken off e_k (what a local correction still has to supply)
  auto record = [&](int k) -> gf_status {
    k_record_pair<<<nb, kT, 0, s>>>(n, r, x, ustar, r_out + (size_t)k * n, e_out + (size_t)k * n);
    if (twolevel) {
      GF_CUDA(ctx, cudaMemsetAsync(z, 0, sizeof(double) * n, s));
      gf_coarse_add(ctx, r, z);
      k_sub_f32<<<nb, kT, 0, s>>>(n, z, e_out + (size_t)k * n);
    }
    GF_LAUNCH_CHECK(ctx, "k_record_pair");
    return GF_OK;
  };
  if ((st = record(0)) != GF_OK) return st;
  int got = 1;
  while (got < npairs) {
    for (int k = 0; k < every; ++k) {
      k_cg_spmv_dot<double, double><<<mat_grid(ctx, L), L.threads, 0, s>>>(
          L, (const double*)vk, p, q, sc);
      if (twolevel) {
        gf_tl_iterate(ctx, x, r, p, q, dinv, sc);
      } else {
        k_cg_update<double><<<red_grid(ctx, n), kT, 0, s>>>(n, x, r, z, p, q, dinv, sc);
        k_cg_direction<double><<<nb, kT, 0, s>>>(n, z, p, sc);
        ctx->launches += 2;
      }
    }
    ctx->launches += every;
    GF_CUDA(ctx, cudaMemcpyAsync(hs, sc, sizeof(SolveScalars), cudaMemcpyDeviceToHost, s));
    GF_CUDA(ctx, cudaStreamSynchronize(s));
    if (hs->done) break;
    if ((st = record(got)) != GF_OK) return st;
    ++got;
  }
  GF_CUDA(ctx, cudaStreamSynchronize(s));
  *recorded = got;
  return GF_OK;
}

namespace {

// FP64 PCG on K64 with M = D^-1 + P Ac^-1 P^T (gf_twolevel.cu): per iteration the SpMV
// with p.q, then the update with the restriction, the coarse product and the direction
// with the prolongation (gf_tl_iterate); chunks are captured as CUDA graphs like run_cg.
gf_status run_twolevel(gf_ctx* ctx, const gf_solve_opts* o, int maxit, int check,
                       gf_solve_info* info) {
  const int n = ctx->n;
  const int nb = gf_blocks(n, kT);
  cudaStream_t s = ctx->stream;
  gf_status st;
  if ((st = gf_coarse_prepare(ctx, 0)) != GF_OK) return st;
  double* v = (double*)ctx->d_work;
  double *x = v, *r = v + n, *p = v + 3 * (size_t)n, *q = v + 4 * (size_t)n,
         *dinv = v + 5 * (size_t)n;
  SolveScalars* sc = ctx->d_scal;
  k_diag_inv<double, double><<<nb, kT, 0, s>>>(n, ctx->d_rownnz, ctx->d_colidx, ctx->d_K64, dinv);
  GF_LAUNCH_CHECK(ctx, "k_diag_inv");
  MatLayout L;
  const void* vk = nullptr;
  if ((st = solver_matrix(ctx, GF_F64, &L, &vk)) != GF_OK) return st;
  const double* val = (const double*)vk;
  GF_CUDA(ctx, cudaMemsetAsync(sc, 0, sizeof(SolveScalars), s));
  gf_tl_begin(ctx, ctx->d_f, x, r, p, dinv, sc);
  GF_LAUNCH_CHECK(ctx, "gf_tl_begin");
  k_cg_init_fin<<<1, 1, 0, s>>>(sc, o->tol, maxit);
  GF_LAUNCH_CHECK(ctx, "k_cg_init_fin");

  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  const int64_t l0 = ctx->launches;
  GF_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  for (int k = 0; k < check; ++k) {
    k_cg_spmv_dot<double, double><<<mat_grid(ctx, L), L.threads, 0, s>>>(L, val, p, q, sc);
    gf_tl_iterate(ctx, x, r, p, q, dinv, sc);
  }
  cudaError_t ce = cudaStreamEndCapture(s, &graph);
  if (ce != cudaSuccess) return gf_cuda_fail(ctx, ce, "graph capture");
  const int64_t per_chunk = ctx->launches - l0 + (int64_t)check;
  ctx->launches = l0;
  ce = cudaGraphInstantiate(&exec, graph, 0);
  if (ce != cudaSuccess) {
    cudaGraphDestroy(graph);
    return gf_cuda_fail(ctx, ce, "graph instantiate");
  }
  SolveScalars* hs = (SolveScalars*)ctx->h_pinned;
  auto t0 = std::chrono::steady_clock::now();
  st = GF_OK;
  for (;;) {
    ce = cudaGraphLaunch(exec, s);
    if (ce != cudaSuccess) { st = gf_cuda_fail(ctx, ce, "graph launch"); break; }
    ctx->launches += per_chunk;
    ce = cudaMemcpyAsync(hs, sc, sizeof(SolveScalars), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) { st = gf_cuda_fail(ctx, ce, "two-level chunk"); break; }
    if (hs->done) break;
    if (o->max_seconds > 0.0) {
      double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (el > o->max_seconds) break;
    }
  }
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  if (st != GF_OK) return st;
  GF_CUDA(ctx, cudaMemcpyAsync(ctx->d_u, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  info->iterations = hs->iter;
  info->outer = 1;
  info->status = status_of(hs->done);
  info->rel_residual = hs->rr0 > 0.0 ? std::sqrt(hs->rr / hs->rr0) : 0.0;
  return GF_OK;
}

}  // namespace

gf_status gf_solve_run(gf_ctx* ctx, const gf_solve_opts* o, gf_solve_info* info) {
  *info = gf_solve_info{};
  const int solver = o->solver;
  if (solver < GF_SOLVER_CG || solver > GF_SOLVER_TWOLEVEL_PCG32)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "unknown solver %d", solver);
  if (!(o->tol > 0.0)) return gf_fail(ctx, GF_ERR_INVALID_ARG, "tol must be > 0");
  const int maxit = o->max_iter > 0 ? o->max_iter : 10000;
  const int check = o->check_every > 0 ? std::min(o->check_every, 256) : 16;
  const int n = ctx->n;
  gf_status st;
  if ((st = ensure_work(ctx)) != GF_OK) return st;
  cudaStream_t s = ctx->stream;
  const int nb = gf_blocks(n, kT);
  char* w = (char*)ctx->d_work;
  auto t0 = std::chrono::steady_clock::now();
  cudaEventRecord(ctx->ev0, s);
  if (solver == GF_SOLVER_LEARNED_FCG) {
    if (!ctx->has64) return gf_fail(ctx, GF_ERR_STATE, "learned FCG needs the FP64 matrix");
    return run_fcg(ctx, o, maxit, check, t0, info);
  }

  if (solver == GF_SOLVER_TWOLEVEL_PCG32) {
    if (!ctx->has64 || !ctx->has32)
      return gf_fail(ctx, GF_ERR_STATE, "two-level PCG32 needs both FP64 and FP32 matrices");
    return run_mixed<float>(ctx, o, maxit, check, t0, info, true);
  }
  if (solver == GF_SOLVER_TWOLEVEL_PCG && o->matrix == GF_F32) {
    if (!ctx->has64 || !ctx->has32)
      return gf_fail(ctx, GF_ERR_STATE, "two-level PCG on K32 needs both FP64 and FP32 matrices");
    return run_mixed<double>(ctx, o, maxit, check, t0, info, true);
  }
  if (solver == GF_SOLVER_TWOLEVEL_PCG) {
    if (o->matrix != GF_F64) return gf_fail(ctx, GF_ERR_INVALID_ARG, "matrix dtype %d", o->matrix);
    if (!ctx->has64) return gf_fail(ctx, GF_ERR_STATE, "two-level PCG needs the FP64 matrix");
    if ((st = run_twolevel(ctx, o, maxit, check, info)) != GF_OK) return st;
    cudaEventRecord(ctx->ev1, s);
    GF_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    info->seconds = ctx->last_seconds = ms * 1e-3;
    double* r64 = (double*)w + 7 * (size_t)n;
    double rrt = 0.0, ff = 0.0;
    if ((st = residual64(ctx, r64, &rrt)) != GF_OK) return st;
    std::vector<double> f(n);
    GF_CUDA(ctx, cudaMemcpy(f.data(), ctx->d_f, sizeof(double) * n, cudaMemcpyDeviceToHost));
    for (double v : f) ff += v * v;
    info->rel_residual = ff > 0.0 ? std::sqrt(rrt / ff) : 0.0;
    if (info->status != GF_OK)
      gf_fail(ctx, (gf_status)info->status, "two-level PCG stopped after %d iterations",
              info->iterations);
    return (gf_status)info->status;
  }

  if (solver == GF_SOLVER_CG || solver == GF_SOLVER_PCG) {
    const bool pre = solver == GF_SOLVER_PCG;
    const int dt = o->matrix;
    if ((dt == GF_F64 && !ctx->has64) || (dt == GF_F32 && !ctx->has32) ||
        (dt != GF_F64 && dt != GF_F32))
      return gf_fail(ctx, GF_ERR_STATE, "matrix dtype %d not assembled", dt);
    int iters = 0, done = 0;
    double rr = 0.0, rr0 = 0.0;
    if (dt == GF_F64) {
      double* v = (double*)w;
      CgVecs vv{v, v + n, v + 2 * (size_t)n, v + 3 * (size_t)n, v + 4 * (size_t)n, v + 5 * (size_t)n};
      if (pre) {
        k_diag_inv<double, double><<<nb, kT, 0, s>>>(n, ctx->d_rownnz, ctx->d_colidx, ctx->d_K64,
                                                     (double*)vv.dinv);
        GF_LAUNCH_CHECK(ctx, "k_diag_inv");
      }
      MatLayout L;
      const void* vk = nullptr;
      if ((st = solver_matrix(ctx, GF_F64, &L, &vk)) != GF_OK) return st;
      st = run_cg<double, double>(ctx, L, (const double*)vk, ctx->d_f, vv, pre, o->tol, maxit, check,
                                  o->max_seconds, t0, &iters, &done, &rr, &rr0);
      if (st != GF_OK) return st;
      GF_CUDA(ctx, cudaMemcpyAsync(ctx->d_u, vv.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    } else {
      float* v = (float*)w;
      CgVecs vv{v, v + n, v + 2 * (size_t)n, v + 3 * (size_t)n, v + 4 * (size_t)n, v + 5 * (size_t)n};
      float* b32 = v + 6 * (size_t)n;
      k_copy_from_f64<float><<<nb, kT, 0, s>>>(n, ctx->d_f, b32);
      GF_LAUNCH_CHECK(ctx, "k_copy_from_f64");
      if (pre) {
        k_diag_inv<float, float><<<nb, kT, 0, s>>>(n, ctx->d_rownnz, ctx->d_colidx, ctx->d_K32,
                                                   (float*)vv.dinv);
        GF_LAUNCH_CHECK(ctx, "k_diag_inv");
      }
      MatLayout L;
      const void* vk = nullptr;
      if ((st = solver_matrix(ctx, GF_F32, &L, &vk)) != GF_OK) return st;
      st = run_cg<float, float>(ctx, L, (const float*)vk, b32, vv, pre, o->tol, maxit, check,
                                o->max_seconds, t0, &iters, &done, &rr, &rr0);
      if (st != GF_OK) return st;
      k_copy_to_f64<float><<<nb, kT, 0, s>>>(n, (const float*)vv.x, ctx->d_u);
      GF_LAUNCH_CHECK(ctx, "k_copy_to_f64");
    }
    cudaEventRecord(ctx->ev1, s);
    GF_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    info->seconds = ctx->last_seconds = ms * 1e-3;
    info->iterations = iters;
    info->outer = 1;
    info->rel_residual = rr0 > 0.0 ? std::sqrt(rr / rr0) : 0.0;
    if (ctx->has64) {
      // report the true FP64 residual ||f - K64 u|| / ||f|| when an FP64 matrix exists
      double* r64 = (double*)w + 7 * (size_t)n;
      double rrt = 0.0, ff = 0.0;
      if ((st = residual64(ctx, r64, &rrt)) != GF_OK) return st;
      std::vector<double> f(n);
      GF_CUDA(ctx, cudaMemcpy(f.data(), ctx->d_f, sizeof(double) * n, cudaMemcpyDeviceToHost));
      for (double v : f) ff += v * v;
      info->rel_residual = ff > 0.0 ? std::sqrt(rrt / ff) : 0.0;
    }
    info->status = status_of(done);
    if (done != 1)
      gf_fail(ctx, (gf_status)info->status, "solver stopped with code %d after %d iterations",
              done, iters);
    return (gf_status)info->status;
  }

  // MIXED_PCG / MIXED_PCG32: Jacobi-PCG on K32 with FP64 reliable updates on K64
  if (!ctx->has64 || !ctx->has32)
    return gf_fail(ctx, GF_ERR_STATE, "mixed solve needs both FP64 and FP32 matrices");
  if (solver == GF_SOLVER_MIXED_PCG32) return run_mixed<float>(ctx, o, maxit, check, t0, info);
  return run_mixed<double>(ctx, o, maxit, check, t0, info);
}

// ---------------------------------------------------------------------------
// Sharded Jacobi-PCG (gf_dist_set_halo, gf_dist_pcg).
//
// The context holds one rank's local mesh: its owned nodes first, then a halo of the
// nodes its elements share with other ranks, and the local K whose owned rows are exact.
// PCG runs over the owned dofs with every vector and scalar on the device; per iteration
// the library packs the send values of p, the caller's halo callback exchanges them
// (point-to-point, enqueued on the context stream), the library unpacks the received
// values into the halo part of p, multiplies, and the caller's all-reduce callback sums
// p.q, then (r.z, r.r) over the ranks, again enqueued on the stream.  The host reads the
// stop flag once per check_every iterations; every rank takes the same steps because the
// flag comes from all-reduced scalars.
// ---------------------------------------------------------------------------
namespace {

struct DistScalars {
  double pq;      // all-reduced p.q
  double rzn;     // all-reduced r.z (new), then r.r: adjacent for one all-reduce
  double rr;
  double rz;      // r.z of the previous iteration
  double rr0, tol2;
  int iter, maxit, done, pad;
};

struct DistState {
  int n_owned = 0, n_send = 0, n_recv = 0;
  int32_t* d_send = nullptr;   // local dofs packed for the neighbours (owned)
  int32_t* d_recv = nullptr;   // local dofs filled from the neighbours (halo)
  double* d_sbuf = nullptr;
  double* d_rbuf = nullptr;
  double* d_vec = nullptr;     // x, r, z, dinv (n_owned each), p, q (n local each)
  DistScalars* d_sc = nullptr;
};

__global__ void k_dist_init(int no, int n, const double* __restrict__ f,
                            const double* __restrict__ dinv, double* __restrict__ x,
                            double* __restrict__ r, double* __restrict__ z, double* __restrict__ p,
                            DistScalars* sc) {
  __shared__ double sh[32];
  double rz = 0.0, rr = 0.0;
  for (int i = blockIdx.x * kT + threadIdx.x; i < n; i += gridDim.x * kT) {
    if (i < no) {
      const double b = f[i], zi = b * dinv[i];
      x[i] = 0.0;
      r[i] = b;
      z[i] = zi;
      p[i] = zi;
      rz += b * zi;
      rr += b * b;
    } else {
      p[i] = 0.0;
    }
  }
  const double s1 = block_sum(rz, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->rzn, s1);
  const double s2 = block_sum(rr, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->rr, s2);
}

__global__ void k_dist_init_fin(DistScalars* sc, double tol, int maxit) {
  sc->rz = sc->rzn;
  sc->rr0 = sc->rr;
  sc->tol2 = tol * tol * sc->rr;
  sc->iter = 0;
  sc->maxit = maxit;
  sc->pq = 0.0;
  sc->done = (sc->rr <= 0.0 || sc->rr <= sc->tol2) ? 1 : (maxit <= 0 ? 3 : 0);
}

__global__ void k_dist_gather(int m, const int32_t* __restrict__ idx, const double* __restrict__ v,
                              double* __restrict__ out) {
  const int k = blockIdx.x * kT + threadIdx.x;
  if (k < m) out[k] = v[idx[k]];
}

__global__ void k_dist_scatter(int m, const int32_t* __restrict__ idx, const double* __restrict__ in,
                               double* __restrict__ v) {
  const int k = blockIdx.x * kT + threadIdx.x;
  if (k < m) v[idx[k]] = in[k];
}

// q = K_local p over every local row; p.q over the owned rows only.  Block 0 clears the
// r.z / r.r slots that the update kernel accumulates into next.
__global__ void __launch_bounds__(kT)
k_dist_spmv_dot(MatLayout L, const double* __restrict__ val, const double* __restrict__ p,
                double* __restrict__ q, int no, DistScalars* sc) {
  __shared__ double sh[32];
  if (sc->done) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->rzn = 0.0;
    sc->rr = 0.0;
  }
  double pq = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < L.count; t += gridDim.x * blockDim.x)
    mat_rows(L, t, val, p, [&](int row, double v) {
      q[row] = v;
      if (row < no) pq += p[row] * v;
    });
  const double s = block_sum(pq, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->pq, s);
}

__global__ void __launch_bounds__(kT)
k_dist_update(int no, double* __restrict__ x, double* __restrict__ r, double* __restrict__ z,
              const double* __restrict__ p, const double* __restrict__ q,
              const double* __restrict__ dinv, DistScalars* sc) {
  __shared__ double sh[32];
  if (sc->done) return;
  const double pq = sc->pq;
  if (!(pq > 0.0) || !isfinite(pq)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->done = 2;
    return;
  }
  const double alpha = sc->rz / pq;
  double rz = 0.0, rr = 0.0;
  for (int i = blockIdx.x * kT + threadIdx.x; i < no; i += gridDim.x * kT) {
    x[i] += alpha * p[i];
    const double ri = r[i] - alpha * q[i];
    r[i] = ri;
    const double zi = ri * dinv[i];
    z[i] = zi;
    rz += ri * zi;
    rr += ri * ri;
  }
  const double s1 = block_sum(rz, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->rzn, s1);
  const double s2 = block_sum(rr, sh);
  if (threadIdx.x == 0) atomicAdd(&sc->rr, s2);
}

// p = z + beta p on the owned dofs; a single thread also advances the scalars (after every
// block has read rz: it runs as the last block of the grid, see k_dist_scalars)
__global__ void k_dist_direction(int no, const double* __restrict__ z, double* __restrict__ p,
                                 const DistScalars* sc) {
  if (sc->done) return;
  const double beta = sc->rzn / sc->rz;
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i < no) p[i] = z[i] + beta * p[i];
}

__global__ void k_dist_scalars(DistScalars* sc) {
  if (sc->done) return;
  sc->rz = sc->rzn;
  sc->pq = 0.0;
  sc->iter += 1;
  if (sc->rr <= sc->tol2) sc->done = 1;
  else if (sc->iter >= sc->maxit) sc->done = 3;
}

}  // namespace

void gf_dist_free(gf_ctx* ctx) {
  DistState* d = static_cast<DistState*>(ctx->dist);
  if (!d) return;
  gf_free(d->d_send);
  gf_free(d->d_recv);
  gf_free(d->d_sbuf);
  gf_free(d->d_rbuf);
  gf_free(d->d_vec);
  gf_free(d->d_sc);
  delete d;
  ctx->dist = nullptr;
}

extern "C" GF_API gf_status gf_dist_set_halo(gf_ctx* ctx, int32_t n_owned, int32_t n_send,
                                             const int32_t* send_dofs, int32_t n_recv,
                                             const int32_t* recv_dofs) {
  if (!ctx) return GF_ERR_INVALID_ARG;
  if (!ctx->has_pattern) return gf_fail(ctx, GF_ERR_STATE, "no local matrix");
  const int n = ctx->n;
  if (n_owned <= 0 || n_owned > n || n_send < 0 || n_recv < 0 ||
      (n_send > 0 && !send_dofs) || (n_recv > 0 && !recv_dofs))
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "halo description");
  for (int k = 0; k < n_send; ++k)
    if (send_dofs[k] < 0 || send_dofs[k] >= n_owned)
      return gf_fail(ctx, GF_ERR_INVALID_ARG, "send dof %d is not an owned dof", send_dofs[k]);
  for (int k = 0; k < n_recv; ++k)
    if (recv_dofs[k] < n_owned || recv_dofs[k] >= n)
      return gf_fail(ctx, GF_ERR_INVALID_ARG, "receive dof %d is not a halo dof", recv_dofs[k]);
  cudaSetDevice(ctx->device);
  gf_dist_free(ctx);
  DistState* d = new DistState();
  ctx->dist = d;
  d->n_owned = n_owned;
  d->n_send = n_send;
  d->n_recv = n_recv;
  gf_status st;
  if ((st = gf_alloc(ctx, &d->d_send, (size_t)std::max(n_send, 1))) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &d->d_recv, (size_t)std::max(n_recv, 1))) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &d->d_sbuf, (size_t)std::max(n_send, 1))) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &d->d_rbuf, (size_t)std::max(n_recv, 1))) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &d->d_vec, (size_t)4 * n_owned + 2 * (size_t)n)) != GF_OK) return st;
  if ((st = gf_alloc(ctx, &d->d_sc, 1)) != GF_OK) return st;
  if (n_send)
    GF_CUDA(ctx, cudaMemcpy(d->d_send, send_dofs, sizeof(int32_t) * n_send, cudaMemcpyHostToDevice));
  if (n_recv)
    GF_CUDA(ctx, cudaMemcpy(d->d_recv, recv_dofs, sizeof(int32_t) * n_recv, cudaMemcpyHostToDevice));
  return GF_OK;
}

extern "C" GF_API gf_status gf_dist_pcg(gf_ctx* ctx, const gf_solve_opts* o,
                                        gf_allreduce_fn allreduce, gf_halo_fn halo, void* user,
                                        gf_solve_info* info) {
  if (!ctx || !o || !info || !allreduce) return GF_ERR_INVALID_ARG;
  DistState* d = static_cast<DistState*>(ctx->dist);
  if (!d) return gf_fail(ctx, GF_ERR_STATE, "no halo description (gf_dist_set_halo)");
  if (!ctx->has64) return gf_fail(ctx, GF_ERR_STATE, "no FP64 local matrix");
  if ((d->n_send || d->n_recv) && !halo)
    return gf_fail(ctx, GF_ERR_INVALID_ARG, "a halo exchange callback is required");
  if (!(o->tol > 0.0)) return gf_fail(ctx, GF_ERR_INVALID_ARG, "tol must be > 0");
  cudaSetDevice(ctx->device);
  *info = gf_solve_info{};
  gf_status st;
  if ((st = ensure_work(ctx)) != GF_OK) return st;
  const int n = ctx->n, no = d->n_owned;
  const int maxit = o->max_iter > 0 ? o->max_iter : 10000;
  const int check = o->check_every > 0 ? std::min(o->check_every, 256) : 16;
  cudaStream_t s = ctx->stream;
  double *x = d->d_vec, *r = x + no, *z = r + no, *dinv = z + no, *p = dinv + no, *q = p + n;
  DistScalars* sc = d->d_sc;
  MatLayout L;
  const void* val = nullptr;
  if ((st = solver_matrix(ctx, GF_F64, &L, &val)) != GF_OK) return st;
  auto coll = [&](int32_t rc, const char* what) -> gf_status {
    if (rc != 0) return gf_fail(ctx, GF_ERR_STATE, "%s callback returned %d", what, (int)rc);
    return GF_OK;
  };
  cudaEventRecord(ctx->ev0, s);
  k_diag_inv<double, double><<<gf_blocks(no, kT), kT, 0, s>>>(no, ctx->d_rownnz, ctx->d_colidx,
                                                               ctx->d_K64, dinv);
  GF_LAUNCH_CHECK(ctx, "k_diag_inv");
  GF_CUDA(ctx, cudaMemsetAsync(sc, 0, sizeof(DistScalars), s));
  k_dist_init<<<red_grid(ctx, n), kT, 0, s>>>(no, n, ctx->d_f, dinv, x, r, z, p, sc);
  GF_LAUNCH_CHECK(ctx, "k_dist_init");
  if ((st = coll(allreduce(&sc->rzn, 2, (void*)s, user), "all-reduce")) != GF_OK) return st;
  k_dist_init_fin<<<1, 1, 0, s>>>(sc, o->tol, maxit);
  GF_LAUNCH_CHECK(ctx, "k_dist_init_fin");
  DistScalars hs{};
  int iters = 0;
  for (;;) {
    for (int k = 0; k < check; ++k) {
      if (d->n_send) {
        k_dist_gather<<<gf_blocks(d->n_send, kT), kT, 0, s>>>(d->n_send, d->d_send, p, d->d_sbuf);
        GF_LAUNCH_CHECK(ctx, "k_dist_gather");
      }
      if (d->n_send || d->n_recv)
        if ((st = coll(halo(d->d_sbuf, d->d_rbuf, (void*)s, user), "halo")) != GF_OK) return st;
      if (d->n_recv) {
        k_dist_scatter<<<gf_blocks(d->n_recv, kT), kT, 0, s>>>(d->n_recv, d->d_recv, d->d_rbuf, p);
        GF_LAUNCH_CHECK(ctx, "k_dist_scatter");
      }
      k_dist_spmv_dot<<<mat_grid(ctx, L), L.threads, 0, s>>>(L, (const double*)val, p, q, no, sc);
      GF_LAUNCH_CHECK(ctx, "k_dist_spmv_dot");
      if ((st = coll(allreduce(&sc->pq, 1, (void*)s, user), "all-reduce")) != GF_OK) return st;
      k_dist_update<<<red_grid(ctx, no), kT, 0, s>>>(no, x, r, z, p, q, dinv, sc);
      GF_LAUNCH_CHECK(ctx, "k_dist_update");
      if ((st = coll(allreduce(&sc->rzn, 2, (void*)s, user), "all-reduce")) != GF_OK) return st;
      k_dist_direction<<<gf_blocks(no, kT), kT, 0, s>>>(no, z, p, sc);
      GF_LAUNCH_CHECK(ctx, "k_dist_direction");
      k_dist_scalars<<<1, 1, 0, s>>>(sc);
      GF_LAUNCH_CHECK(ctx, "k_dist_scalars");
    }
    GF_CUDA(ctx, cudaMemcpyAsync(&hs, sc, sizeof(DistScalars), cudaMemcpyDeviceToHost, s));
    GF_CUDA(ctx, cudaStreamSynchronize(s));
    iters = hs.iter;
    if (hs.done) break;
  }
  GF_CUDA(ctx, cudaMemcpyAsync(ctx->d_u, x, sizeof(double) * no, cudaMemcpyDeviceToDevice, s));
  GF_CUDA(ctx, cudaMemsetAsync(ctx->d_u + no, 0, sizeof(double) * (n - no), s));
  cudaEventRecord(ctx->ev1, s);
  GF_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  info->seconds = ctx->last_seconds = ms * 1e-3;
  info->iterations = iters;
  info->outer = 1;
  info->rel_residual = hs.rr0 > 0.0 ? std::sqrt(hs.rr / hs.rr0) : 0.0;  // recursive, all ranks
  info->status = status_of(hs.done);
  if (hs.done != 1)
    gf_fail(ctx, (gf_status)info->status, "sharded PCG stopped with code %d after %d iterations",
            hs.done, iters);
  return (gf_status)info->status;
}

// ---------------------------------------------------------------------------
// Compensated residual for iterative refinement (gf_residual_dd).
// ---------------------------------------------------------------------------
extern "C" GF_API gf_status gf_residual_dd(gf_ctx* ctx, const double* u_hi, const double* u_lo,
                                           double* r, double* rel_residual) {
  if (!ctx || !u_hi || !u_lo || !r) return GF_ERR_INVALID_ARG;
  if (!ctx->has64) return gf_fail(ctx, GF_ERR_STATE, "no FP64 matrix");
  if (!ctx->d_f) return gf_fail(ctx, GF_ERR_STATE, "no force vector");
  cudaSetDevice(ctx->device);
  gf_status st;
  if (!ctx->d_red && (st = gf_alloc(ctx, &ctx->d_red, 4)) != GF_OK) return st;
  if (!ctx->h_pinned && cudaMallocHost(&ctx->h_pinned, 256) != cudaSuccess) {
    cudaGetLastError();
    return gf_fail(ctx, GF_ERR_OOM, "pinned scalars");
  }
  cudaStream_t s = ctx->stream;
  const int n = ctx->n;
  GF_CUDA(ctx, cudaMemsetAsync(ctx->d_red, 0, 2 * sizeof(double), s));
  k_residual_dd<<<std::min(gf_blocks(n, kT), 8 * ctx->sm_count), kT, 0, s>>>(
      n, ctx->d_rownnz, ctx->d_colidx, ctx->d_K64, u_hi, u_lo, ctx->d_f, r, ctx->d_red);
  GF_LAUNCH_CHECK(ctx, "k_residual_dd");
  if (rel_residual) {
    double ff = 0.0;
    for (double v : ctx->h_f) ff += v * v;
    double* h = (double*)ctx->h_pinned + 16;
    GF_CUDA(ctx, cudaMemcpyAsync(h, ctx->d_red, sizeof(double), cudaMemcpyDeviceToHost, s));
    GF_CUDA(ctx, cudaStreamSynchronize(s));
    *rel_residual = ff > 0.0 ? std::sqrt(*h / ff) : std::sqrt(*h);
  } else {
    GF_CUDA(ctx, cudaStreamSynchronize(s));
  }
  return GF_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free Jacobi-PCG (gf_pcg_noalloc).
//
// For callers that may not allocate device memory themselves or through this
// library: a host framework that owns every device byte through its own arena,
// or a time-stepping loop where a cudaMalloc/cudaFree (which can synchronise the
// device) is not allowed.  The caller passes the ELL matrix, right-hand side and
// solution buffers; the solver's work vectors and scalars live in one file-scope
// __device__ array of fixed size, held by every GPU that loads this library until
// the process exits.  It never calls cudaMalloc, cudaFree or cudaMallocHost.
//
// Shared-state rules: all calls share that array and it keeps the previous call's
// contents (every word a call reads is written or cleared by the same call first),
// so two calls whose GPU work overlaps — on two streams, or from two host threads —
// race and corrupt each other.  The first call on a device looks up the array's
// device address with cudaGetSymbolAddress (which may load the module onto that
// device); make that first call before any stream capture.
// ---------------------------------------------------------------------------
namespace {
constexpr int kNoAllocVecs = 5;           // r, z, p, q, 1/diag
constexpr int kNoAllocScalarDoubles = 32; // SolveScalars + residual accumulator
constexpr int kNoAllocMaxDevices = 64;
static_assert(GF_PCG_NOALLOC_MAX_N > 0, "max size");
static_assert(sizeof(SolveScalars) <= 16 * sizeof(double), "scalar block");
}  // namespace

static __device__ __align__(256) double
    g_pcg_noalloc_scratch[(size_t)kNoAllocVecs * GF_PCG_NOALLOC_MAX_N + kNoAllocScalarDoubles];

// Checks the caller's ELL before any kernel trusts it: every row length within
// [0, width] and every stored column (slot < row length) within [0, n).  It reads only
// in-bounds words (slots below min(row length, width)); a bad row sets *bad.
__global__ void k_noalloc_ell_check(int n, int width, const int32_t* __restrict__ rownnz,
                                    const int32_t* __restrict__ colidx, int* bad) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int len = rownnz[i];
    bool ok = len >= 0 && len <= width;
    const int m = ok ? len : 0;
    for (int j = 0; j < m && ok; ++j) {
      const int c = colidx[(size_t)j * n + i];
      ok = c >= 0 && c < n;
    }
    if (!ok) atomicExch(bad, 1);
  }
}

static std::mutex g_pcg_noalloc_mu;
static double* g_pcg_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once per
// device, with that device current).
static gf_status pcg_noalloc_scratch(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return GF_ERR_CUDA;
  }
  if (dev < 0 || dev >= kNoAllocMaxDevices) return GF_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_pcg_noalloc_mu);
  if (!g_pcg_noalloc_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_pcg_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return GF_ERR_CUDA;
    }
    g_pcg_noalloc_addr[dev] = static_cast<double*>(p);
  }
  *out = g_pcg_noalloc_addr[dev];
  return GF_OK;
}

extern "C" GF_API gf_status gf_pcg_noalloc(int32_t n, int32_t width, const int32_t* rownnz,
                                           const int32_t* colidx, const double* values,
                                           const double* b, double* x, double tol,
                                           int32_t max_iter, void* stream, int32_t* iterations,
                                           double* rel_residual) {
  if (n <= 0 || n > GF_PCG_NOALLOC_MAX_N) return GF_ERR_INVALID_ARG;
  if (width <= 0 || !rownnz || !colidx || !values || !b || !x) return GF_ERR_INVALID_ARG;
  if (!(tol > 0.0) || max_iter <= 0) return GF_ERR_INVALID_ARG;
  double* S = nullptr;
  gf_status st = pcg_noalloc_scratch(&S);
  if (st != GF_OK) return st;
  const size_t M = GF_PCG_NOALLOC_MAX_N;
  double *r = S, *z = S + M, *p = S + 2 * M, *q = S + 3 * M, *dinv = S + 4 * M;
  SolveScalars* sc = reinterpret_cast<SolveScalars*>(S + kNoAllocVecs * M);
  double* acc = S + kNoAllocVecs * M + 16;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nb = gf_blocks(n, kT);
  const int chunk = 16;
  const MatLayout L{n, n, rownnz, colidx, nullptr, nullptr};  // the caller's ELL as given
  auto fail = [](cudaError_t e) {
    cudaGetLastError();
    return e == cudaSuccess ? GF_OK : GF_ERR_CUDA;
  };
  // validate the ELL (row lengths, column range) into a flag word of the scalar block
  int* bad = reinterpret_cast<int*>(S + kNoAllocVecs * M + 17);
  cudaError_t e = cudaMemsetAsync(bad, 0, sizeof(int), s);
  if (e != cudaSuccess) return fail(e);
  k_noalloc_ell_check<<<std::min(nb, 4 * 148), kT, 0, s>>>(n, width, rownnz, colidx, bad);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
  int hbad = 0;
  e = cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(e);
  if (hbad) return GF_ERR_INVALID_ARG;
  e = cudaMemsetAsync(sc, 0, sizeof(SolveScalars), s);
  if (e != cudaSuccess) return fail(e);
  k_diag_inv<double, double><<<nb, kT, 0, s>>>(n, rownnz, colidx, values, dinv);
  k_cg_init<double><<<nb, kT, 0, s>>>(n, b, dinv, x, r, z, p, sc);
  k_cg_init_fin<<<1, 1, 0, s>>>(sc, tol, max_iter);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
  SolveScalars hs{};  // pageable host copy: no pinned allocation
  for (;;) {
    for (int k = 0; k < chunk; ++k) {
      k_cg_spmv_dot<double, double><<<nb, kT, 0, s>>>(L, values, p, q, sc);
      k_cg_update<double><<<nb, kT, 0, s>>>(n, x, r, z, p, q, dinv, sc);
      k_cg_direction<double><<<nb, kT, 0, s>>>(n, z, p, sc);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
    e = cudaMemcpyAsync(&hs, sc, sizeof(SolveScalars), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(e);
    if (hs.done) break;
  }
  // true residual ||b - K x|| / ||b|| in FP64 (r0 = b since x0 = 0)
  double rr = 0.0;
  e = cudaMemsetAsync(acc, 0, sizeof(double), s);
  if (e != cudaSuccess) return fail(e);
  k_residual64<<<nb, kT, 0, s>>>(L, values, x, b, r, acc);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
  e = cudaMemcpyAsync(&rr, acc, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(e);
  if (iterations) *iterations = hs.iter;
  if (rel_residual) *rel_residual = hs.rr0 > 0.0 ? std::sqrt(rr / hs.rr0) : 0.0;
  return status_of(hs.done);
}
