// Element-level device helpers shared by the assembly kernels: shape-derivative
// tables, Jacobian, determinant/inverse and the Cartesian gradients at a Gauss
// point (StiffAlgo::GetJacobianMatrix / BuildBMatrix, src/FEM/StiffAlgo.cc:207-278;
// det / matInverse, src/LAops/LAops.cc:80-117).
#pragma once

#include "gf_internal.cuh"

struct AsmTables {
  // dN/dxi at each Gauss point: [gp][a][i], and weights, both precisions
  double dN64[GF_MAX_GP * 3 * GF_MAX_NEN];
  float dN32[GF_MAX_GP * 3 * GF_MAX_NEN];
  double w64[GF_MAX_GP];
  float w32[GF_MAX_GP];
};

// Adds DIM values to DIM consecutive rows of one ELL slot column (the rows of one
// node).  Atomic FP32 uses vector reductions where the address allows: one
// red.global.add.v2.f32 for a 2-D node (its two rows start 8-byte aligned because n
// is even), a v2 plus a scalar reduction for a 3-D node; FP64 and the colour schedule
// (plain read-modify-write) go per value.
// d = a * b + c on two FP32 lanes at once (packed single-precision FMA: two IEEE FMAs,
// round to nearest, in one instruction)
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
      "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}

__device__ inline void red_v2_f32(float* p, float a, float b) {
  asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(a), "f"(b) : "memory");
}

template <int DIM, typename T, bool ATOMIC>
__device__ inline void add_rows(T* p, const T (&v)[DIM]) {
  if constexpr (ATOMIC && sizeof(T) == 4 && DIM == 3) {
    // the pair of rows that starts 8-byte aligned takes the vector reduction; the choice is
    // made by selecting addresses, not by branching, since neighbouring lanes hold nodes of
    // both parities and a branch would run both paths for the whole warp
    float* q = reinterpret_cast<float*>(p);
    const bool al = (reinterpret_cast<uintptr_t>(q) & 7) == 0;
    red_v2_f32(al ? q : q + 1, al ? (float)v[0] : (float)v[1], al ? (float)v[1] : (float)v[2]);
    atomicAdd(al ? q + 2 : q, al ? (float)v[2] : (float)v[0]);
  } else if constexpr (ATOMIC && sizeof(T) == 4 && DIM == 2) {
    float* q = reinterpret_cast<float*>(p);
    if ((reinterpret_cast<uintptr_t>(q) & 7) == 0) {
      red_v2_f32(q, (float)v[0], (float)v[1]);
    } else {
      atomicAdd(q, (float)v[0]);
      atomicAdd(q + 1, (float)v[1]);
    }
  } else if constexpr (ATOMIC) {
#pragma unroll
    for (int c = 0; c < DIM; ++c) atomicAdd(p + c, v[c]);
  } else {
#pragma unroll
    for (int c = 0; c < DIM; ++c) p[c] += v[c];
  }
}

template <int DIM, typename R>
__device__ inline R gf_det_inv(const R (&J)[3][3], R (&Ji)[3][3]) {
  if (DIM == 2) {
    R d = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    R id = R(1) / d;
    Ji[0][0] = J[1][1] * id;
    Ji[0][1] = -J[0][1] * id;
    Ji[1][0] = -J[1][0] * id;
    Ji[1][1] = J[0][0] * id;
    return d;
  } else {
    R c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    R c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    R c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    R d = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
    R id = R(1) / d;
    Ji[0][0] = c00 * id;
    Ji[1][0] = c01 * id;
    Ji[2][0] = c02 * id;
    Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
    Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
    Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
    Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
    Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
    Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
    return d;
  }
}

// J[a][b] = sum_i dN_i/dxi_a * x_i[b] (rows natural, columns x, y, z).
template <int NEN, int DIM, typename R, typename TC>
__device__ inline void gf_jacobian(const TC* dN /*[DIM][NEN]*/, const TC* X /*[NEN][DIM]*/,
                                   R (&J)[3][3]) {
#pragma unroll
  for (int a = 0; a < DIM; ++a)
#pragma unroll
    for (int b = 0; b < DIM; ++b) {
      R s = R(0);
#pragma unroll 4
      for (int i = 0; i < NEN; ++i) s += R(dN[a * NEN + i]) * R(X[i * DIM + b]);
      J[a][b] = s;
    }
}

// Element with max/min |detJ| over its Gauss points above 10: the FP32 path then
// forms J, J^-1 and the gradients in FP64.
template <int NEN, int DIM, typename TC>
__device__ inline int gf_distorted(const TC* sdN, int ngp, const TC* X) {
  float dmin = 3.4e38f, dmax = 0.f;
  for (int g = 0; g < ngp; ++g) {
    float J[3][3], Ji[3][3];
    gf_jacobian<NEN, DIM, float, TC>(sdN + g * DIM * NEN, X, J);
    float d = fabsf(gf_det_inv<DIM, float>(J, Ji));
    dmin = fminf(dmin, d);
    dmax = fmaxf(dmax, d);
  }
  return dmax > 10.f * dmin ? 1 : 0;
}

// Gradients g_i = J^-1 dN_i/dxi at one Gauss point, written to
// G[(i*DIM + c) * stride]; returns detJ.  `use64` selects FP64 arithmetic.
template <int NEN, int DIM, typename TC>
__device__ inline TC gf_gradients(const TC* dN, const TC* X, bool use64, TC* G, int stride) {
  if (use64) {
    double J[3][3], Ji[3][3];
    gf_jacobian<NEN, DIM, double, TC>(dN, X, J);
    const double d = gf_det_inv<DIM, double>(J, Ji);
#pragma unroll 4
    for (int i = 0; i < NEN; ++i)
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        double s = 0.0;
#pragma unroll
        for (int a = 0; a < DIM; ++a) s += Ji[c][a] * double(dN[a * NEN + i]);
        G[(i * DIM + c) * stride] = TC(s);
      }
    return TC(d);
  } else {
    TC J[3][3], Ji[3][3];
    gf_jacobian<NEN, DIM, TC, TC>(dN, X, J);
    const TC d = gf_det_inv<DIM, TC>(J, Ji);
#pragma unroll 4
    for (int i = 0; i < NEN; ++i)
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        TC s = TC(0);
#pragma unroll
        for (int a = 0; a < DIM; ++a) s += Ji[c][a] * dN[a * NEN + i];
        G[(i * DIM + c) * stride] = s;
      }
    return d;
  }
}

// Shape derivatives of element type ET at the NG1-point tensor Gauss rule, evaluated
// at compile time with the same formulas and point order as the runtime tables
// (gf_dshape, gf_gauss_rule); kernels that index it with unrolled loop counters get
// the values as instruction constants.
template <int ET, int NG1>
struct GpTable {
  static constexpr int DIM = gf_elem_info(ET).dim;
  static constexpr int NEN = gf_elem_info(ET).nen;
  static constexpr int NGP = DIM == 2 ? NG1 * NG1 : NG1 * NG1 * NG1;
  double d64[NGP * DIM * NEN] = {};
  float d32[NGP * DIM * NEN] = {};
};

template <int ET, int NG1>
constexpr GpTable<ET, NG1> gf_gp_table() {
  using T = GpTable<ET, NG1>;
  T t{};
  // 1/sqrt(3) and sqrt(3/5)
  const double xg = NG1 == 2 ? 0.57735026918962576451 : 0.77459666924148337704;
  const double x[3] = {-xg, NG1 == 2 ? xg : 0.0, xg};
  const int nk = T::DIM == 2 ? 1 : NG1;
  int g = 0;
  for (int i = 0; i < NG1; ++i)
    for (int j = 0; j < NG1; ++j)
      for (int k = 0; k < nk; ++k) {
        const double p[3] = {x[i], x[j], T::DIM == 2 ? 0.0 : x[k]};
        double dN[3 * GF_MAX_NEN] = {};
        gf_dshape<double>(ET, gf_node_nat_host[ET], p, dN);
        for (int q = 0; q < T::DIM * T::NEN; ++q) {
          t.d64[g * T::DIM * T::NEN + q] = dN[q];
          t.d32[g * T::DIM * T::NEN + q] = (float)dN[q];
        }
        ++g;
      }
  return t;
}

// Shape-derivative tables for the context's element type and Gauss rule (device
// buffer owned by the context, built once per mesh).
gf_status gf_asm_tables(gf_ctx* ctx, const AsmTables** out);
