/*
 * TEST INFRASTRUCTURE ONLY — the oracle.  A plain-C restatement of the
 * reference's CPU algorithm for the hot path, used by tests/, smoke() and the
 * CPU-baseline leg of bench.py as the checker.  Nothing in the product links it.
 *
 * Pinned against the reference's own code: tests/test_oracle.py compares every
 * function here with oracle/_ref/libref_fp64.so (the reference sources compiled
 * with fem_float = double) and with the committed golden vectors in
 * tests/golden/ (made by tests/golden/make_golden.py from that library).
 *
 * Functions follow (paths within fpaboim/gpufem):
 *   or_gauss          src/FEM/FemData.cc:226-316   (CalcGaussVectors)
 *   or_dshape         src/FEM/StiffAlgo.cc:47-202  (GetdShapeFunctNatCoord)
 *   or_dmatrix        src/FEM/FemData.cc:322-365   (CalcConstituitiveData; plane
 *                     stress selected explicitly, see the reference's inverted
 *                     strcmp at :330)
 *   or_element_ke     src/FEM/StiffAlgoCPU.cc:97-133 with StiffAlgo.cc:207-278 and
 *                     LAops.cc:80-133 (J, det, inverse, B, B^T (D B) detJ w)
 *   or_pattern        topological version of ELLmatrix::AddElem/InsertElem
 *                     (src/SPRmatrix/ELLmatrix.cc:91-138): sorted columns per row
 *   or_assemble       StiffAlgo::AssembleK (StiffAlgo.cc:304-401)
 *   or_penalty        FEM::ApplyConstraint PEN (src/FEM/fem.cc:119-143)
 *   or_eliminate      symmetric elimination (no reference counterpart; the
 *                     reference's SUB mode is a no-op, fem.cc:147-165)
 *   or_spmv           ELLmatrix::Axy (ELLmatrix.cc:194-204)
 *   or_residual_dd    r = f - K (u_hi + u_lo) over the same ELL walk as Axy, in
 *                     double-double (Dot2 of Ogita, Rump and Oishi 2005: products
 *                     split exactly by fma, sums by TwoSum); no reference counterpart
 *   or_cg             SPRmatrix::CPU_CG (src/SPRmatrix/SPRmatrix.cc:405-480),
 *                     optionally Jacobi-preconditioned (no reference counterpart)
 *   or_greedy_color   femColor::MakeGreedyColoring over METIS_MeshToDual
 *                     (src/FEM/femColor.cc:79-191), ncommon = 1
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { OR_Q4 = 0, OR_Q8 = 1, OR_BRICK8 = 2, OR_BRICK20 = 3 };

static const int k_nen[4] = {4, 8, 8, 20};
static const int k_dim[4] = {2, 2, 3, 3};

int or_nen(int et) { return k_nen[et]; }
int or_dim(int et) { return k_dim[et]; }

void or_gauss(int dim, int ng, double* pts, double* w) {
  double x[3], wt[3];
  if (ng == 2) {
    x[0] = -1.0 / sqrt(3.0); x[1] = -x[0];
    wt[0] = wt[1] = 1.0;
  } else {
    x[0] = -sqrt(3.0 / 5.0); x[1] = 0.0; x[2] = -x[0];
    wt[0] = 5.0 / 9.0; wt[1] = 8.0 / 9.0; wt[2] = wt[0];
  }
  int s = 0;
  if (dim == 2) {
    for (int i = 0; i < ng; ++i)
      for (int j = 0; j < ng; ++j, ++s) {
        pts[2 * s] = x[i]; pts[2 * s + 1] = x[j];
        w[s] = wt[i] * wt[j];
      }
  } else {
    for (int i = 0; i < ng; ++i)
      for (int j = 0; j < ng; ++j)
        for (int k = 0; k < ng; ++k, ++s) {
          pts[3 * s] = x[i]; pts[3 * s + 1] = x[j]; pts[3 * s + 2] = x[k];
          w[s] = wt[i] * wt[j] * wt[k];
        }
  }
}

/* node natural coordinates, reference order */
static const int nat_q4[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
static const int nat_q8[8][2] = {{-1, -1}, {0, -1}, {1, -1}, {1, 0},
                                 {1, 1},   {0, 1},  {-1, 1}, {-1, 0}};
static const int nat_b8[8][3] = {{1, -1, -1},  {1, 1, -1},  {1, 1, 1},  {1, -1, 1},
                                 {-1, -1, -1}, {-1, 1, -1}, {-1, 1, 1}, {-1, -1, 1}};
static const int nat_b20[20][3] = {
    {1, -1, -1}, {1, 0, -1},  {1, 1, -1},   {1, 1, 0},   {1, 1, 1},   {1, 0, 1},  {1, -1, 1},
    {1, -1, 0},  {0, -1, -1}, {0, 1, -1},   {0, 1, 1},   {0, -1, 1},  {-1, -1, -1},
    {-1, 0, -1}, {-1, 1, -1}, {-1, 1, 0},   {-1, 1, 1},  {-1, 0, 1},  {-1, -1, 1}, {-1, -1, 0}};

/* dN[a*nen + i] = dN_i / dxi_a */
void or_dshape(int et, const double* p, double* dN) {
  const double r = p[0], s = p[1], t = (k_dim[et] == 3) ? p[2] : 0.0;
  if (et == OR_Q4) {
    for (int i = 0; i < 4; ++i) {
      const double ri = nat_q4[i][0], si = nat_q4[i][1];
      dN[0 * 4 + i] = 0.25 * ri * (1.0 + si * s);
      dN[1 * 4 + i] = 0.25 * si * (1.0 + ri * r);
    }
  } else if (et == OR_Q8) {
    for (int i = 0; i < 8; ++i) {
      const double ri = nat_q8[i][0], si = nat_q8[i][1];
      if (ri != 0 && si != 0) {
        /* N = (1+ri r)(1+si s)(ri r + si s - 1)/4 */
        dN[0 * 8 + i] = 0.25 * ri * (1.0 + si * s) * (2.0 * ri * r + si * s);
        dN[1 * 8 + i] = 0.25 * si * (1.0 + ri * r) * (ri * r + 2.0 * si * s);
      } else if (ri == 0) {
        /* N = (1-r^2)(1+si s)/2 */
        dN[0 * 8 + i] = -r * (1.0 + si * s);
        dN[1 * 8 + i] = 0.5 * si * (1.0 - r * r);
      } else {
        /* N = (1+ri r)(1-s^2)/2 */
        dN[0 * 8 + i] = 0.5 * ri * (1.0 - s * s);
        dN[1 * 8 + i] = -s * (1.0 + ri * r);
      }
    }
  } else if (et == OR_BRICK8) {
    for (int i = 0; i < 8; ++i) {
      const double ri = nat_b8[i][0], si = nat_b8[i][1], ti = nat_b8[i][2];
      dN[0 * 8 + i] = 0.125 * ri * (1.0 + si * s) * (1.0 + ti * t);
      dN[1 * 8 + i] = 0.125 * si * (1.0 + ri * r) * (1.0 + ti * t);
      dN[2 * 8 + i] = 0.125 * ti * (1.0 + ri * r) * (1.0 + si * s);
    }
  } else {
    for (int i = 0; i < 20; ++i) {
      const double ri = nat_b20[i][0], si = nat_b20[i][1], ti = nat_b20[i][2];
      const double fr = 1.0 + ri * r, fs = 1.0 + si * s, ft = 1.0 + ti * t;
      if (ri != 0 && si != 0 && ti != 0) {
        /* N = fr fs ft (ri r + si s + ti t - 2)/8 */
        const double g = ri * r + si * s + ti * t - 2.0;
        dN[0 * 20 + i] = 0.125 * ri * fs * ft * (g + fr);
        dN[1 * 20 + i] = 0.125 * si * fr * ft * (g + fs);
        dN[2 * 20 + i] = 0.125 * ti * fr * fs * (g + ft);
      } else if (ri == 0) {
        /* N = (1-r^2) fs ft / 4 */
        dN[0 * 20 + i] = -0.5 * r * fs * ft;
        dN[1 * 20 + i] = 0.25 * si * (1.0 - r * r) * ft;
        dN[2 * 20 + i] = 0.25 * ti * (1.0 - r * r) * fs;
      } else if (si == 0) {
        dN[0 * 20 + i] = 0.25 * ri * (1.0 - s * s) * ft;
        dN[1 * 20 + i] = -0.5 * s * fr * ft;
        dN[2 * 20 + i] = 0.25 * ti * (1.0 - s * s) * fr;
      } else {
        dN[0 * 20 + i] = 0.25 * ri * (1.0 - t * t) * fs;
        dN[1 * 20 + i] = 0.25 * si * (1.0 - t * t) * fr;
        dN[2 * 20 + i] = -0.5 * t * fr * fs;
      }
    }
  }
}

/* analysis: 0 plane stress, 1 plane strain (2-D only). D is s x s row-major. */
void or_dmatrix(int dim, int analysis, double E, double nu, double* D) {
  if (dim == 2) {
    double c1, c2, c3;
    if (analysis == 0) {
      const double a = E / (1.0 - nu * nu);
      c1 = a; c2 = a * (1.0 - nu) / 2.0; c3 = a * nu;
    } else {
      const double a = E / ((1.0 - 2.0 * nu) * (1.0 + nu));
      c1 = a * (1.0 - nu); c2 = a * (1.0 - 2.0 * nu) / 2.0; c3 = a * nu;
    }
    memset(D, 0, 9 * sizeof(double));
    D[0] = c1; D[4] = c1; D[8] = c2; D[1] = c3; D[3] = c3;
  } else {
    const double c1 = E * (1.0 - nu) / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double c2 = nu / (1.0 - nu);
    const double c3 = (1.0 - 2.0 * nu) / (2.0 * (1.0 - nu));
    memset(D, 0, 36 * sizeof(double));
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) D[i * 6 + j] = (i == j) ? c1 : c1 * c2;
    for (int i = 3; i < 6; ++i) D[i * 6 + i] = c1 * c3;
  }
}

/* Ke (m x m, row-major) for one element with coordinates X[i*dim + c]. */
void or_element_ke(int et, int ng, const double* X, const double* D, double* Ke) {
  const int nen = k_nen[et], dim = k_dim[et], m = nen * dim, ns = (dim - 1) * 3;
  const int ngp = dim == 2 ? ng * ng : ng * ng * ng;
  double pts[81], w[27], dN[60], J[9], Ji[9], g[60], B[6 * 60], DB[6 * 60];
  or_gauss(dim, ng, pts, w);
  memset(Ke, 0, sizeof(double) * m * m);
  for (int gp = 0; gp < ngp; ++gp) {
    or_dshape(et, pts + gp * dim, dN);
    for (int a = 0; a < dim; ++a)
      for (int b = 0; b < dim; ++b) {
        double sum = 0.0;
        for (int i = 0; i < nen; ++i) sum += dN[a * nen + i] * X[i * dim + b];
        J[a * dim + b] = sum;
      }
    double det;
    if (dim == 2) {
      det = J[0] * J[3] - J[1] * J[2];
      Ji[0] = J[3] / det; Ji[1] = -J[1] / det; Ji[2] = -J[2] / det; Ji[3] = J[0] / det;
    } else {
      det = J[0] * J[4] * J[8] + J[3] * J[7] * J[2] + J[6] * J[1] * J[5] -
            J[0] * J[7] * J[5] - J[3] * J[1] * J[8] - J[6] * J[4] * J[2];
      Ji[0] = (J[8] * J[4] - J[7] * J[5]) / det;
      Ji[1] = -(J[8] * J[1] - J[7] * J[2]) / det;
      Ji[2] = (J[5] * J[1] - J[4] * J[2]) / det;
      Ji[3] = -(J[8] * J[3] - J[6] * J[5]) / det;
      Ji[4] = (J[8] * J[0] - J[6] * J[2]) / det;
      Ji[5] = -(J[5] * J[0] - J[3] * J[2]) / det;
      Ji[6] = (J[7] * J[3] - J[6] * J[4]) / det;
      Ji[7] = -(J[7] * J[0] - J[6] * J[1]) / det;
      Ji[8] = (J[4] * J[0] - J[3] * J[1]) / det;
    }
    /* g = J^-1 dN */
    for (int c = 0; c < dim; ++c)
      for (int i = 0; i < nen; ++i) {
        double sum = 0.0;
        for (int a = 0; a < dim; ++a) sum += Ji[c * dim + a] * dN[a * nen + i];
        g[c * nen + i] = sum;
      }
    memset(B, 0, sizeof(double) * ns * m);
    for (int i = 0; i < nen; ++i) {
      if (dim == 2) {
        B[0 * m + 2 * i] = g[0 * nen + i];
        B[1 * m + 2 * i + 1] = g[1 * nen + i];
        B[2 * m + 2 * i] = g[1 * nen + i];
        B[2 * m + 2 * i + 1] = g[0 * nen + i];
      } else {
        B[0 * m + 3 * i] = g[0 * nen + i];
        B[1 * m + 3 * i + 1] = g[1 * nen + i];
        B[2 * m + 3 * i + 2] = g[2 * nen + i];
        B[3 * m + 3 * i] = g[1 * nen + i];
        B[3 * m + 3 * i + 1] = g[0 * nen + i];
        B[4 * m + 3 * i + 1] = g[2 * nen + i];
        B[4 * m + 3 * i + 2] = g[1 * nen + i];
        B[5 * m + 3 * i] = g[2 * nen + i];
        B[5 * m + 3 * i + 2] = g[0 * nen + i];
      }
    }
    for (int k = 0; k < ns; ++k)
      for (int j = 0; j < m; ++j) {
        double sum = 0.0;
        for (int l = 0; l < ns; ++l) sum += D[k * ns + l] * B[l * m + j];
        DB[k * m + j] = sum;
      }
    const double sc = det * w[gp];
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) {
        double sum = 0.0;
        for (int k = 0; k < ns; ++k) sum += B[k * m + i] * DB[k * m + j];
        Ke[i * m + j] += sum * sc;
      }
  }
}

/* ---- pattern ------------------------------------------------------------- */
static int cmp_int(const void* a, const void* b) {
  int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}

/* Node adjacency (sorted, unique, including self).  Returns total length;
 * adj_off has nnodes+1 entries; adj may be NULL to query the size. */
int64_t or_node_adjacency(int et, int nnodes, int nelem, const int* conn1, int* adj_off,
                          int* adj) {
  const int nen = k_nen[et];
  int* cnt = (int*)calloc((size_t)nnodes + 1, sizeof(int));
  for (int64_t k = 0; k < (int64_t)nelem * nen; ++k) cnt[conn1[k]]++;  /* 1-based -> +1 slot */
  int* eoff = (int*)calloc((size_t)nnodes + 1, sizeof(int));
  for (int a = 0; a < nnodes; ++a) eoff[a + 1] = eoff[a] + cnt[a + 1];
  int* inc = (int*)malloc(sizeof(int) * (size_t)nelem * nen);
  int* fill = (int*)malloc(sizeof(int) * ((size_t)nnodes + 1));
  memcpy(fill, eoff, sizeof(int) * ((size_t)nnodes + 1));
  for (int64_t k = 0; k < (int64_t)nelem * nen; ++k) inc[fill[conn1[k] - 1]++] = (int)(k / nen);
  int* tmp = (int*)malloc(sizeof(int) * 4096);
  int64_t total = 0;
  adj_off[0] = 0;
  for (int a = 0; a < nnodes; ++a) {
    int c = 0;
    for (int q = eoff[a]; q < eoff[a + 1]; ++q)
      for (int i = 0; i < nen; ++i) tmp[c++] = conn1[(int64_t)inc[q] * nen + i] - 1;
    qsort(tmp, c, sizeof(int), cmp_int);
    int u = 0;
    for (int k = 0; k < c; ++k)
      if (k == 0 || tmp[k] != tmp[k - 1]) tmp[u++] = tmp[k];
    if (adj) memcpy(adj + total, tmp, sizeof(int) * u);
    total += u;
    adj_off[a + 1] = (int)total;
  }
  free(cnt); free(eoff); free(inc); free(fill); free(tmp);
  return total;
}

/* Topological ELL pattern: rownnz[n], colidx[W*n] column-major, padding col = row.
 * Returns W (max row length); with colidx == NULL only W is computed. */
int or_pattern(int et, int nnodes, int nelem, const int* conn1, int W, int* rownnz,
               int* colidx) {
  const int dim = k_dim[et];
  const int n = nnodes * dim;
  int* adj_off = (int*)malloc(sizeof(int) * ((size_t)nnodes + 1));
  int64_t tot = or_node_adjacency(et, nnodes, nelem, conn1, adj_off, NULL);
  int* adj = (int*)malloc(sizeof(int) * (size_t)(tot > 0 ? tot : 1));
  or_node_adjacency(et, nnodes, nelem, conn1, adj_off, adj);
  int wmax = 0;
  for (int a = 0; a < nnodes; ++a) {
    int w = (adj_off[a + 1] - adj_off[a]) * dim;
    if (w > wmax) wmax = w;
  }
  if (colidx) {
    for (int a = 0; a < nnodes; ++a) {
      const int na = adj_off[a + 1] - adj_off[a];
      for (int c = 0; c < dim; ++c) {
        const int row = a * dim + c;
        rownnz[row] = na * dim;
        for (int s = 0; s < W; ++s) {
          colidx[(int64_t)s * n + row] =
              s < na * dim ? adj[adj_off[a] + s / dim] * dim + s % dim : row;
        }
      }
    }
  }
  free(adj_off); free(adj);
  return wmax;
}

static int64_t find_slot(int n, int W, const int* rownnz, const int* colidx, int row, int col) {
  for (int s = 0; s < rownnz[row]; ++s)
    if (colidx[(int64_t)s * n + row] == col) return (int64_t)s * n + row;
  (void)W;
  return -1;
}

/* Assemble into vals (W*n, zeroed here).  E_elem may be NULL (scalar E). */
int or_assemble(int et, int ng, int analysis, int nnodes, const double* coords, int nelem,
                const int* conn1, const double* E_elem, double E, double nu, int W,
                const int* rownnz, const int* colidx, double* vals) {
  const int nen = k_nen[et], dim = k_dim[et], m = nen * dim;
  const int n = nnodes * dim;
  double D1[36], D[36], X[60];
  double* Ke = (double*)malloc(sizeof(double) * m * m);
  or_dmatrix(dim, analysis, 1.0, nu, D1);
  memset(vals, 0, sizeof(double) * (size_t)W * n);
  int missing = 0;
  for (int e = 0; e < nelem; ++e) {
    const double Ee = E_elem ? E_elem[e] : E;
    for (int k = 0; k < 36; ++k) D[k] = D1[k] * Ee;
    for (int i = 0; i < nen; ++i)
      for (int c = 0; c < dim; ++c) X[i * dim + c] = coords[(int64_t)(conn1[(int64_t)e * nen + i] - 1) * dim + c];
    or_element_ke(et, ng, X, D, Ke);
    for (int i = 0; i < nen; ++i) {
      const int gi = (conn1[(int64_t)e * nen + i] - 1) * dim;
      for (int j = 0; j < nen; ++j) {
        const int gj = (conn1[(int64_t)e * nen + j] - 1) * dim;
        for (int a = 0; a < dim; ++a)
          for (int b = 0; b < dim; ++b) {
            int64_t o = find_slot(n, W, rownnz, colidx, gi + a, gj + b);
            if (o < 0) { ++missing; continue; }
            vals[o] += Ke[(dim * i + a) * m + (dim * j + b)];
          }
      }
    }
  }
  free(Ke);
  return missing;
}

/* K_dd <- (1e4 * max_i K_ii) * K_dd for fixed dofs (fixed[d] != 0). */
void or_penalty(int n, int W, const int* rownnz, const int* colidx, double* vals,
                const uint8_t* fixed) {
  (void)W;
  double mx = -INFINITY;
  for (int i = 0; i < n; ++i) {
    int64_t o = find_slot(n, W, rownnz, colidx, i, i);
    double d = o >= 0 ? vals[o] : 0.0;
    if (i == 0 || d > mx) mx = d;
  }
  const double pen = mx * 10000.0;
  for (int i = 0; i < n; ++i)
    if (fixed[i]) {
      int64_t o = find_slot(n, W, rownnz, colidx, i, i);
      if (o >= 0) vals[o] = pen * vals[o];
    }
}

void or_eliminate(int n, int W, const int* rownnz, const int* colidx, double* vals,
                  const uint8_t* fixed, double* f) {
  for (int i = 0; i < n; ++i) {
    for (int s = 0; s < rownnz[i]; ++s) {
      int64_t o = (int64_t)s * n + i;
      const int c = colidx[o];
      if (fixed[i] || fixed[c]) vals[o] = (c == i) ? 1.0 : 0.0;
    }
    if (fixed[i] && f) f[i] = 0.0;
  }
  (void)W;
}

void or_spmv(int n, int W, const int* rownnz, const int* colidx, const double* vals,
             const double* x, double* y) {
  (void)W;
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int j = 0; j < rownnz[i]; ++j) {
      int64_t o = (int64_t)j * n + i;
      s += vals[o] * x[colidx[o]];
    }
    y[i] = s;
  }
}

/* r = f - K (u_hi + u_lo), accumulated in double-double and rounded once; returns r.r */
double or_residual_dd(int n, int W, const int* rownnz, const int* colidx, const double* vals,
                      const double* f, const double* uh, const double* ul, double* r) {
  (void)W;
  double rr = 0.0;
  for (int i = 0; i < n; ++i) {
    double s = f[i], c = 0.0;
    for (int j = 0; j < rownnz[i]; ++j) {
      int64_t o = (int64_t)j * n + i;
      double k = vals[o], h = uh[colidx[o]];
      double p = k * h, pe = fma(k, h, -p);
      double t = s - p, bp = t - s;
      double te = (s - (t - bp)) + (-p - bp);
      s = t;
      c += te - pe - k * ul[colidx[o]];
    }
    r[i] = s + c;
    rr += r[i] * r[i];
  }
  return rr;
}

/* CG from x0 = 0 until r.r <= eps^2 r0.r0 or maxit; Jacobi when precond != 0.
 * Returns the iteration count. */
int or_cg(int n, int W, const int* rownnz, const int* colidx, const double* vals,
          const double* b, double* x, int maxit, double eps, int precond) {
  double* r = (double*)malloc(sizeof(double) * n);
  double* z = (double*)malloc(sizeof(double) * n);
  double* p = (double*)malloc(sizeof(double) * n);
  double* q = (double*)malloc(sizeof(double) * n);
  double* dinv = (double*)malloc(sizeof(double) * n);
  for (int i = 0; i < n; ++i) {
    dinv[i] = 1.0;
    if (precond) {
      int64_t o = find_slot(n, W, rownnz, colidx, i, i);
      if (o >= 0 && vals[o] != 0.0) dinv[i] = 1.0 / vals[o];
    }
    x[i] = 0.0;
    r[i] = b[i];
    z[i] = r[i] * dinv[i];
    p[i] = z[i];
  }
  double rz = 0.0, rr = 0.0;
  for (int i = 0; i < n; ++i) { rz += r[i] * z[i]; rr += r[i] * r[i]; }
  const double bound = eps * eps * rr;
  int it = 0;
  while (it < maxit && rr > bound) {
    or_spmv(n, W, rownnz, colidx, vals, p, q);
    double pq = 0.0;
    for (int i = 0; i < n; ++i) pq += p[i] * q[i];
    const double alpha = rz / pq;
    double rzn = 0.0;
    rr = 0.0;
    for (int i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
      z[i] = r[i] * dinv[i];
      rzn += r[i] * z[i];
      rr += r[i] * r[i];
    }
    const double beta = rzn / rz;
    rz = rzn;
    for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    ++it;
  }
  free(r); free(z); free(p); free(q); free(dinv);
  return it;
}

/* Greedy first-fit colouring in element order; elements sharing a node conflict.
 * Returns the number of colours; color[] is 0-based. */
int or_greedy_color(int et, int nnodes, int nelem, const int* conn1, int* color) {
  const int nen = k_nen[et];
  int* cnt = (int*)calloc((size_t)nnodes + 1, sizeof(int));
  for (int64_t k = 0; k < (int64_t)nelem * nen; ++k) cnt[conn1[k]]++;
  int* off = (int*)calloc((size_t)nnodes + 1, sizeof(int));
  for (int a = 0; a < nnodes; ++a) off[a + 1] = off[a] + cnt[a + 1];
  int* inc = (int*)malloc(sizeof(int) * (size_t)nelem * nen);
  int* fill = (int*)malloc(sizeof(int) * ((size_t)nnodes + 1));
  memcpy(fill, off, sizeof(int) * ((size_t)nnodes + 1));
  for (int64_t k = 0; k < (int64_t)nelem * nen; ++k) inc[fill[conn1[k] - 1]++] = (int)(k / nen);
  int used[4096];
  int ncol = 0;
  for (int e = 0; e < nelem; ++e) color[e] = -1;
  for (int e = 0; e < nelem; ++e) {
    memset(used, 0, sizeof(used));
    for (int i = 0; i < nen; ++i) {
      const int a = conn1[(int64_t)e * nen + i] - 1;
      for (int q = off[a]; q < off[a + 1]; ++q)
        if (color[inc[q]] >= 0) used[color[inc[q]]] = 1;
    }
    int c = 0;
    while (used[c]) ++c;
    color[e] = c;
    if (c + 1 > ncol) ncol = c + 1;
  }
  free(cnt); free(off); free(inc); free(fill);
  return ncol;
}
