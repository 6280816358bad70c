// Numeric assembly: Ke = sum_gp B^T D B detJ w for every element, scattered
// straight into the column-major ELL values (Ke never touches HBM).
//
// Reference: StiffAlgoCPU::CalcGlobalStiffnessNaive / CalcStiffnessColoring
// (src/FEM/StiffAlgoCPU.cc:58-284) with StiffAlgo::GetdShapeFunctNatCoord,
// GetJacobianMatrix, BuildBMatrix (src/FEM/StiffAlgo.cc:47-278), det/matInverse
// (src/LAops/LAops.cc:80-117) and AssembleK/AssembleKcol (StiffAlgo.cc:304-401).
//
// Formulation.  For isotropic D the node-pair block of B^T D B is
//   Ke[i,a ; j,b] = sum_gp w detJ E ( lam1 g_i[a] g_j[b] + mu1 g_i[b] g_j[a]
//                                     + mu1 delta_ab g_i . g_j )
// with g_i = dN_i/dx and (lam1, mu1) the reference's D per unit modulus
// (plane stress: lam1 = nu/(1-nu^2), mu1 = 1/(2(1+nu)); 3-D and plane strain:
// the Lame constants per unit E).  This is B^T D B entry by entry, without the
// zero entries of B: 2*dim^2 FMAs per node pair and Gauss point instead of the
// dense (s x m) products.  Ke is symmetric, so only pairs i <= j are formed and
// each writes block (i,j) and its transpose (j,i).
//
// CTA = a tile of TE elements of one colour (or any elements for the atomic
// scatter), 256 threads:
//   phase 1  thread per (element, Gauss point): J, detJ, J^-1, g = J^-1 dN/dxi
//            into shared memory G[gp][node][comp][elem]; for the FP32 path an
//            element whose max/min |detJ| over its Gauss points exceeds 10 gets
//            J, J^-1 and g in FP64.
//   phase 2  thread per (element, node pair i <= j): the dim x dim block, then
//            read-modify-write into K (colour schedule: no two elements of a
//            colour share a node, so plain RMW is race-free) or red.global.add
//            (atomic schedule).  The slot of each block comes from the slot map
//            built with the pattern.
#include <cmath>
#include <algorithm>

#include "gf_elem.cuh"

namespace {

constexpr int kThreads = 256;

template <int ET, typename TC>
constexpr size_t smem_bytes(int TE, int ngp) {
  constexpr ElemInfo info = gf_elem_info(ET);
  const size_t nTC = (size_t)ngp * info.dim * info.nen + ngp + (size_t)TE * info.nen * info.dim +
                     (size_t)ngp * info.nen * info.dim * TE + (size_t)ngp * TE;
  return nTC * sizeof(TC) + sizeof(int) * ((size_t)TE * info.nen + 2 * TE) +
         sizeof(uint16_t) * (size_t)(info.nen * (info.nen + 1) / 2) + 16;
}

template <int ET, typename TC>
constexpr int pick_tile(int ngp) {
  // largest power of two <= 128 whose working set fits ~100 KB (2 CTAs per SM)
  int TE = 128;
  while (TE > 4 && smem_bytes<ET, TC>(TE, ngp) > 100 * 1024) TE >>= 1;
  return TE;
}

// The Gauss-point count (NG1 per axis) and the tile of TE elements are compile-time, so the
// Gauss loops unroll and every shared-memory offset is an immediate; the node pair of a
// task comes from a table in shared memory.
template <int ET, typename TC, bool ATOMIC, int NG1>
__global__ void __launch_bounds__(kThreads)
k_assemble(const int32_t* __restrict__ elems, int count, const int32_t* __restrict__ conn,
           const double* __restrict__ coords, const TC* __restrict__ Eel,
           const uint16_t* __restrict__ slotmap, int nelem, int n,
           const AsmTables* __restrict__ tab, TC lam1, TC mu1, TC* __restrict__ K) {
  constexpr ElemInfo info = gf_elem_info(ET);
  constexpr int NEN = info.nen, DIM = info.dim;
  constexpr int NPAIR = NEN * (NEN + 1) / 2;
  constexpr int ngp = DIM == 2 ? NG1 * NG1 : NG1 * NG1 * NG1;
  constexpr int TE = pick_tile<ET, TC>(ngp);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TC* sdN = reinterpret_cast<TC*>(smem_raw);                 // ngp*DIM*NEN
  TC* sw = sdN + ngp * DIM * NEN;                            // ngp
  TC* sX = sw + ngp;                                         // TE*NEN*DIM
  TC* sG = sX + TE * NEN * DIM;                              // ngp*NEN*DIM*TE
  TC* swd = sG + ngp * NEN * DIM * TE;                       // ngp*TE
  int* sconn = reinterpret_cast<int*>(swd + ngp * TE);       // TE*NEN
  int* sel = sconn + TE * NEN;                               // TE
  int* sflag = sel + TE;                                     // TE
  uint16_t* spair = reinterpret_cast<uint16_t*>(sflag + TE); // NPAIR: i * 256 + j, i <= j

  const int tile0 = blockIdx.x * TE;
  const int nt = min(TE, count - tile0);
  const bool f64 = sizeof(TC) == 8;

  for (int k = threadIdx.x; k < ngp * DIM * NEN; k += kThreads)
    sdN[k] = f64 ? TC(tab->dN64[k]) : TC(tab->dN32[k]);
  for (int k = threadIdx.x; k < ngp; k += kThreads) sw[k] = f64 ? TC(tab->w64[k]) : TC(tab->w32[k]);
  for (int e = threadIdx.x; e < TE; e += kThreads) {
    sel[e] = e < nt ? elems[tile0 + e] : -1;
    sflag[e] = 0;
  }
  // pair index -> (i, j), i <= j, row-major upper triangle
  for (int p = threadIdx.x; p < NPAIR; p += kThreads) {
    int i = 0, q = p;
    while (q >= NEN - i) { q -= NEN - i; ++i; }
    spair[p] = (uint16_t)(i * 256 + i + q);
  }
  __syncthreads();
  // Element-local coordinates x_i - x_0, formed in FP64 before rounding: J depends
  // only on coordinate differences, so the FP32 path keeps full relative precision
  // in J however small the element is against its distance from the origin.
  for (int k = threadIdx.x; k < nt * NEN; k += kThreads) {
    const int e = k / NEN, i = k % NEN;
    const int node = conn[(int64_t)sel[e] * NEN + i];
    const int node0 = conn[(int64_t)sel[e] * NEN];
    sconn[k] = node;
#pragma unroll
    for (int c = 0; c < DIM; ++c)
      sX[k * DIM + c] = TC(coords[(int64_t)node * DIM + c] - coords[(int64_t)node0 * DIM + c]);
  }
  __syncthreads();

  // phase 1a (FP32 path only): flag elements with a large detJ spread; |detJ| at every
  // (element, Gauss point) in parallel first (swd as scratch), then the ratio per element
  // (a thread per element alone would hold the CTA at the barrier when TE is small)
  if (!f64) {
    for (int t = threadIdx.x; t < TE * ngp; t += kThreads) {
      const int e = t % TE, g = t / TE;
      if (e >= nt) continue;
      float J[3][3], Ji[3][3];
      gf_jacobian<NEN, DIM, float, TC>(sdN + g * DIM * NEN, sX + e * NEN * DIM, J);
      swd[g * TE + e] = TC(fabsf(gf_det_inv<DIM, float>(J, Ji)));
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nt; e += kThreads) {
      float dmin = 3.4e38f, dmax = 0.f;
#pragma unroll
      for (int g = 0; g < ngp; ++g) {
        dmin = fminf(dmin, float(swd[g * TE + e]));
        dmax = fmaxf(dmax, float(swd[g * TE + e]));
      }
      sflag[e] = dmax > 10.f * dmin ? 1 : 0;
    }
    __syncthreads();
  }

  // phase 1: gradients at Gauss points
  for (int t = threadIdx.x; t < TE * ngp; t += kThreads) {
    const int e = t % TE, g = t / TE;
    if (e >= nt) continue;
    const TC detJ = gf_gradients<NEN, DIM, TC>(sdN + g * DIM * NEN, sX + e * NEN * DIM,
                                               f64 || sflag[e], sG + (g * NEN * DIM) * TE + e,
                                               TE);
    swd[g * TE + e] = sw[g] * detJ * Eel[sel[e]];
  }
  __syncthreads();

  // phase 2: node-pair blocks and scatter
  for (int t = threadIdx.x; t < TE * NPAIR; t += kThreads) {
    const int e = t % TE;
    if (e >= nt) continue;
    const int ij = spair[t / TE];
    const int i = ij >> 8, j = ij & 255;
    TC H[DIM][DIM];
    const TC* gI = sG + (i * DIM) * TE + e;
    const TC* gJ = sG + (j * DIM) * TE + e;
    if constexpr (sizeof(TC) == 4) {
      // FP32: columns 0 and 1 of each row of H two at a time (packed FMA)
      float2 h01[DIM];
      float h2[DIM];
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        h01[a] = make_float2(0.f, 0.f);
        h2[a] = 0.f;
      }
#pragma unroll
      for (int g = 0; g < ngp; ++g) {
        const float w = swd[g * TE + e];
        float gi[DIM], gj[DIM];
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
          gi[c] = gI[(g * NEN * DIM + c) * TE] * w;
          gj[c] = gJ[(g * NEN * DIM + c) * TE];
        }
        const float2 gj01 = make_float2(gj[0], gj[1]);
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
          h01[a] = fma2(make_float2(gi[a], gi[a]), gj01, h01[a]);
          if constexpr (DIM == 3) h2[a] = fmaf(gi[a], gj[2], h2[a]);
        }
      }
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        H[a][0] = h01[a].x;
        H[a][1] = h01[a].y;
        if constexpr (DIM == 3) H[a][DIM - 1] = h2[a];
      }
    } else {
#pragma unroll
      for (int a = 0; a < DIM; ++a)
#pragma unroll
        for (int b = 0; b < DIM; ++b) H[a][b] = TC(0);
#pragma unroll
      for (int g = 0; g < ngp; ++g) {
        const TC w = swd[g * TE + e];
        TC gi[DIM], gj[DIM];
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
          gi[c] = gI[(g * NEN * DIM + c) * TE] * w;
          gj[c] = gJ[(g * NEN * DIM + c) * TE];
        }
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
          for (int b = 0; b < DIM; ++b) H[a][b] += gi[a] * gj[b];
      }
    }
    TC tr = TC(0);
#pragma unroll
    for (int a = 0; a < DIM; ++a) tr += H[a][a];
    const int el = sel[e];
    const int ni = sconn[e * NEN + i], nj = sconn[e * NEN + j];
    const int sij = slotmap[(int64_t)(i * NEN + j) * nelem + el] * DIM;
    const int sji = slotmap[(int64_t)(j * NEN + i) * nelem + el] * DIM;
    TC V[DIM][DIM];
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
      for (int b = 0; b < DIM; ++b) {
        V[a][b] = lam1 * H[a][b] + mu1 * H[b][a];
        if (a == b) V[a][b] += mu1 * tr;
      }
    // block (i, j): column b of the block goes to rows ni*DIM .. ni*DIM + DIM - 1 of slot
    // column sij + b; block (j, i) is the transpose
#pragma unroll
    for (int b = 0; b < DIM; ++b) {
      TC col[DIM];
#pragma unroll
      for (int a = 0; a < DIM; ++a) col[a] = V[a][b];
      add_rows<DIM, TC, ATOMIC>(&K[(int64_t)(sij + b) * n + ni * DIM], col);
    }
    if (i != j) {
#pragma unroll
      for (int a = 0; a < DIM; ++a)
        add_rows<DIM, TC, ATOMIC>(&K[(int64_t)(sji + a) * n + nj * DIM], V[a]);
    }
  }
}

template <int ET, typename TC, int NG1>
gf_status launch_et_ng(gf_ctx* ctx, int scatter, const AsmTables* d_tab, TC* K) {
  constexpr int DIM = gf_elem_info(ET).dim;
  constexpr int ngp = DIM == 2 ? NG1 * NG1 : NG1 * NG1 * NG1;
  constexpr int TE = pick_tile<ET, TC>(ngp);
  constexpr size_t sm = smem_bytes<ET, TC>(TE, ngp);
  const double* coords = ctx->d_coords64;
  const TC* Eel = sizeof(TC) == 8 ? (const TC*)ctx->d_Eel : (const TC*)ctx->d_Eel32;
  auto kc = k_assemble<ET, TC, false, NG1>;
  auto ka = k_assemble<ET, TC, true, NG1>;
  GF_CUDA(ctx, gf_smem_attr(kc, (int)sm));
  GF_CUDA(ctx, gf_smem_attr(ka, (int)sm));
  if (scatter == GF_SCATTER_ATOMIC) {
    const int count = ctx->nelem;
    ka<<<(count + TE - 1) / TE, kThreads, sm, ctx->stream>>>(
        ctx->d_allperm, count, ctx->d_conn, coords, Eel, ctx->d_slotmap, ctx->nelem, ctx->n,
        d_tab, TC(ctx->lam1), TC(ctx->mu1), K);
    GF_LAUNCH_CHECK(ctx, "k_assemble(atomic)");
  } else {
    for (int c = 0; c < ctx->ncolors; ++c) {
      const int c0 = ctx->color_off[c], count = ctx->color_off[c + 1] - c0;
      if (count == 0) continue;
      kc<<<(count + TE - 1) / TE, kThreads, sm, ctx->stream>>>(
          ctx->d_perm + c0, count, ctx->d_conn, coords, Eel, ctx->d_slotmap, ctx->nelem,
          ctx->n, d_tab, TC(ctx->lam1), TC(ctx->mu1), K);
      GF_LAUNCH_CHECK(ctx, "k_assemble(colour)");
    }
  }
  return GF_OK;
}

template <int ET, typename TC>
gf_status launch_et(gf_ctx* ctx, int scatter, const AsmTables* d_tab, TC* K) {
  return ctx->ngauss == 2 ? launch_et_ng<ET, TC, 2>(ctx, scatter, d_tab, K)
                          : launch_et_ng<ET, TC, 3>(ctx, scatter, d_tab, K);
}

template <typename TC>
gf_status launch_dispatch(gf_ctx* ctx, int scatter, const AsmTables* d_tab, TC* K) {
  switch (ctx->elem_type) {
    case GF_Q4: return launch_et<GF_Q4, TC>(ctx, scatter, d_tab, K);
    case GF_Q8: return launch_et<GF_Q8, TC>(ctx, scatter, d_tab, K);
    case GF_BRICK8: return launch_et<GF_BRICK8, TC>(ctx, scatter, d_tab, K);
    default: return launch_et<GF_BRICK20, TC>(ctx, scatter, d_tab, K);
  }
}

}  // namespace

gf_status gf_assemble_owner(gf_ctx* ctx, int dtype, const AsmTables* d_tab);
gf_status gf_assemble_tc(gf_ctx* ctx, int scatter, const AsmTables* d_tab, float* K, int* d_err);
gf_status gf_assemble_owner_gram(gf_ctx* ctx, const float* gram, float* K);

gf_status gf_asm_tables(gf_ctx* ctx, const AsmTables** out) {
  if (ctx->d_asmtab) {
    *out = (const AsmTables*)ctx->d_asmtab;
    return GF_OK;
  }
  AsmTables h{};
  std::vector<double> pts, w;
  gf_gauss_rule<double>(ctx->dim, ctx->ngauss, pts, w);
  std::vector<double> dN(ctx->dim * ctx->nen);
  for (int g = 0; g < ctx->ngp; ++g) {
    gf_dshape<double>(ctx->elem_type, gf_node_nat_host[ctx->elem_type], &pts[g * ctx->dim],
                      dN.data());
    for (int k = 0; k < ctx->dim * ctx->nen; ++k) {
      h.dN64[g * ctx->dim * ctx->nen + k] = dN[k];
      h.dN32[g * ctx->dim * ctx->nen + k] = (float)dN[k];
    }
    h.w64[g] = w[g];
    h.w32[g] = (float)w[g];
  }
  AsmTables* d = nullptr;
  gf_status st = gf_alloc(ctx, &d, 1);
  if (st != GF_OK) return st;
  GF_CUDA(ctx, cudaMemcpy(d, &h, sizeof(AsmTables), cudaMemcpyHostToDevice));
  ctx->d_asmtab = d;
  *out = d;
  return GF_OK;
}

gf_status gf_assemble_launch(gf_ctx* ctx, int dtype, int scatter, int engine) {
  const bool mma = engine == GF_ENGINE_TF32_MMA;
  gf_status st;
  const AsmTables* d_tab = nullptr;
  if ((st = gf_asm_tables(ctx, &d_tab)) != GF_OK) return st;
  const int64_t total = (int64_t)ctx->n * ctx->W;
  if (dtype == GF_F64) {
    if (!ctx->d_K64 && (st = gf_palloc(ctx, &ctx->d_K64, (size_t)total)) != GF_OK) return st;
  } else {
    if (!ctx->d_K32 && (st = gf_palloc(ctx, &ctx->d_K32, (size_t)total)) != GF_OK) return st;
  }
  if (mma) {
    if (!ctx->d_asm_err && (st = gf_alloc(ctx, &ctx->d_asm_err, 1)) != GF_OK) return st;
    GF_CUDA(ctx, cudaMemsetAsync(ctx->d_asm_err, 0, sizeof(int), ctx->stream));
  }
  if (mma && scatter == GF_SCATTER_OWNER) {
    // element Gram matrices from the tensor cores, RAW x RAW floats per element
    const size_t raw = (size_t)ctx->nen * ctx->dim;
    const size_t need = (size_t)ctx->nelem * raw * raw * sizeof(float);
    if (ctx->gram_bytes < need) {
      gf_free(ctx->d_gram);
      ctx->gram_bytes = 0;
      if ((st = gf_alloc(ctx, &ctx->d_gram, need / sizeof(float))) != GF_OK) return st;
      ctx->gram_bytes = need;
    }
  }
  if (scatter != GF_SCATTER_OWNER && (st = gf_slotmap_ensure(ctx)) != GF_OK) return st;
  cudaEventRecord(ctx->ev0, ctx->stream);
  if (mma && scatter == GF_SCATTER_OWNER) {
    // tensor cores: every element's Gram matrix to HBM; owner gather: K written once
    st = gf_assemble_tc(ctx, scatter, d_tab, ctx->d_gram, ctx->d_asm_err);
    cudaEventRecord(ctx->evm, ctx->stream);
    if (st == GF_OK) st = gf_assemble_owner_gram(ctx, ctx->d_gram, ctx->d_K32);
  } else if (scatter == GF_SCATTER_OWNER) {
    // owner-computes: every K entry (padding included) is written exactly once
    st = gf_assemble_owner(ctx, dtype, d_tab);
  } else if (dtype == GF_F64) {
    cudaMemsetAsync(ctx->d_K64, 0, sizeof(double) * total, ctx->stream);
    st = launch_dispatch<double>(ctx, scatter, d_tab, ctx->d_K64);
  } else {
    cudaMemsetAsync(ctx->d_K32, 0, sizeof(float) * total, ctx->stream);
    st = mma ? gf_assemble_tc(ctx, scatter, d_tab, ctx->d_K32, ctx->d_asm_err)
             : launch_dispatch<float>(ctx, scatter, d_tab, ctx->d_K32);
  }
  cudaEventRecord(ctx->ev1, ctx->stream);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (st != GF_OK) return st;
  if (e != cudaSuccess) return gf_cuda_fail(ctx, e, "assembly");
  if (mma) {
    int herr = 0;
    GF_CUDA(ctx, cudaMemcpy(&herr, ctx->d_asm_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr)
      return gf_fail(ctx, GF_ERR_CUDA, "tensor-core assembly: an MMA completion wait timed out");
  }
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  ctx->last_seconds = ms * 1e-3;
  if (scatter == GF_SCATTER_OWNER) {
    float m0 = 0.f, m1 = 0.f;
    cudaEventElapsedTime(&m0, ctx->ev0, ctx->evm);
    cudaEventElapsedTime(&m1, ctx->evm, ctx->ev1);
    ctx->last_split[0] = m0 * 1e-3;
    ctx->last_split[1] = m1 * 1e-3;
  } else {
    ctx->last_split[0] = 0.0;
    ctx->last_split[1] = ms * 1e-3;
  }
  if (dtype == GF_F64) { ctx->has64 = true; ctx->kver64++; } else { ctx->has32 = true; ctx->kver32++; }
  ctx->bc_mode_applied = -1;
  return GF_OK;
}
