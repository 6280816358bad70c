// TEST INFRASTRUCTURE ONLY (oracle).  A C-ABI driver over the reference's own
// CPU path, compiled together with the unmodified reference sources by
// oracle/build_ref.sh into oracle/_ref/libref_{fp32,fp64}.so.  `real` below is
// the reference's `fem_float` (float as shipped, double in the FP64 overlay).
//
// Flow mirrored (reference src/interface.cpp:417-466 and src/Test/FemTest.cpp:91-101):
//   FileIO::ReadNF -> FEM::Init(assemble, CPU) -> FemData::Init(ELL, ngp, E, nu)
//   -> FEM::SetUseColoring -> FEM::CalcStiffnessMat (StiffAlgoCPU)
//   -> FEM::ApplyConstraint(PEN) -> ELLmatrix::CG (SPRmatrix::CPU_CG).
//
// One deliberate deviation, applied only when `plane_stress` is set: the 2-D
// constitutive matrix is overwritten with explicit plane-stress values after
// FemData::Init, because the reference's own selection is undefined behaviour
// (the analysis string dangles, src/Utils/fileIO.cc:245-251) and its strcmp
// test is inverted (src/FEM/FemData.cc:330-340).  The values use the
// reference's expressions (FemData.cc:331-334) in fem_float arithmetic.
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include <map>
#include <list>
#include <iostream>
#include <sstream>
#include <fstream>
#include <algorithm>
#include <omp.h>

// The ELL storage members are private in the reference; the oracle reads them
// to export the stored pattern (src/SPRmatrix/ELLmatrix.h:82-89).
#define private public
#define protected public
#include "FEM/fem.h"
#include "FEM/FemData.h"
#include "SPRmatrix/SPRmatrix.h"
#include "SPRmatrix/ELLmatrix.h"
#include "Utils/fileIO.h"
#include "Utils/util.h"
#undef private
#undef protected

typedef fem_float real;

struct RefSession {
  FileIO io;
  FEM fem;
};

static ELLmatrix* ell_of(RefSession* s) {
  return dynamic_cast<ELLmatrix*>(s->fem.GetFemData()->GetStiffnessMatrix());
}

extern "C" {

int ref_real_size() { return (int)sizeof(real); }

void* ref_open(const char* nf_path, int ngp, double E, double nu, int plane_stress) {
  RefSession* s = new RefSession();
  if (!s->io.ReadNF(std::string(nf_path))) {
    delete s;
    return nullptr;
  }
  s->fem.Init(true, FEM::CPU);
  FemData* fd = s->fem.GetFemData();
  fd->Init(SPRmatrix::ELL, ngp, (real)E, (real)nu, &s->io);
  if (plane_stress && fd->GetModelDim() == 2) {
    real** D = fd->GetConstituitiveMat();
    real Em = (real)E, Nu = (real)nu;
    real auxcoef = Em / (1 - (Nu * Nu));
    real c1 = auxcoef;
    real c2 = auxcoef * ((1 - Nu) / 2);
    real c3 = auxcoef * Nu;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) D[i][j] = 0;
    D[0][0] = c1; D[1][1] = c1; D[2][2] = c2; D[0][1] = c3; D[1][0] = c3;
  }
  return s;
}

void ref_close(void* h) { delete (RefSession*)h; }

void ref_dims(void* h, int* out5) {
  FemData* fd = ((RefSession*)h)->fem.GetFemData();
  out5[0] = fd->GetModelDim();
  out5[1] = fd->GetNumNodes();
  out5[2] = fd->GetNumElem();
  out5[3] = fd->GetNumElemNodes();
  out5[4] = fd->GetNumDof();
}

// Constitutive matrix actually used (s x s, row-major).
void ref_get_D(void* h, double* out) {
  FemData* fd = ((RefSession*)h)->fem.GetFemData();
  int s = (fd->GetModelDim() - 1) * 3;
  real** D = fd->GetConstituitiveMat();
  for (int i = 0; i < s; ++i)
    for (int j = 0; j < s; ++j) out[i * s + j] = (double)D[i][j];
}

// Connectivity as stored after ReadNF (1-based, Brick20 renumbered).
void ref_get_connect(void* h, int32_t* out) {
  FemData* fd = ((RefSession*)h)->fem.GetFemData();
  size_t n = (size_t)fd->GetNumElem() * fd->GetNumElemNodes();
  std::memcpy(out, fd->GetElemConnect(), n * sizeof(int32_t));
}

void ref_get_coords(void* h, double* out) {
  FemData* fd = ((RefSession*)h)->fem.GetFemData();
  size_t n = (size_t)fd->GetNumNodes() * fd->GetModelDim();
  for (size_t i = 0; i < n; ++i) out[i] = (double)fd->GetNodeCoords()[i];
}

int ref_num_supports(void* h) {
  return ((RefSession*)h)->fem.GetFemData()->GetNodeNumConstraints();
}

// Supports as stored by FemData (rows of dim+1: node id, fixed flags).
void ref_get_supports(void* h, int32_t* out) {
  FemData* fd = ((RefSession*)h)->fem.GetFemData();
  const int w = fd->GetModelDim() + 1;
  for (int i = 0; i < fd->GetNodeNumConstraints(); ++i)
    for (int j = 0; j < w; ++j) out[i * w + j] = fd->GetNodeConstraints()[i][j];
}

void ref_get_gauss(void* h, double* pts, double* w) {
  FemData* fd = ((RefSession*)h)->fem.GetFemData();
  int ng = fd->GetNumGaussLoopPts(), dim = fd->GetModelDim();
  for (int g = 0; g < ng; ++g) {
    for (int c = 0; c < dim; ++c) pts[g * dim + c] = (double)fd->GetGaussPtsVecCPU()[g][c];
    w[g] = (double)fd->GetGaussWeightVec()[g];
  }
}

// StiffAlgoCPU assembly (naive with omp critical scatter, or colour-scheduled).
// Returns the reference's own timer (seconds).
double ref_assemble(void* h, int coloring, int nthreads) {
  RefSession* s = (RefSession*)h;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  s->fem.SetDeviceMode(FEM::CPU);
  s->fem.SetUseColoring(coloring != 0);
  return s->fem.CalcStiffnessMat();
}

int ref_num_colors(void* h) {
  return (int)((RefSession*)h)->fem.GetFemData()->GetColorVector().size();
}

int ref_ell_width(void* h) {
  ELLmatrix* m = ell_of((RefSession*)h);
  int w = 0;
  for (int i = 0; i < m->m_matdim; ++i) w = std::max(w, m->m_rownnz[i]);
  return w;
}

int ref_ell_stored_width(void* h) { return ell_of((RefSession*)h)->m_maxrowlen; }

// Column-major export, width `width`: entry (row, slot) at slot*n + row; slots
// past rownnz get col = -1 and value 0 (the reference leaves them garbage).
void ref_ell_export(void* h, int width, int32_t* rownnz, int32_t* colidx, double* vals) {
  ELLmatrix* m = ell_of((RefSession*)h);
  const int n = m->m_matdim;
  for (int i = 0; i < n; ++i) {
    int nz = m->m_rownnz[i];
    rownnz[i] = nz;
    for (int j = 0; j < width; ++j) {
      size_t o = (size_t)j * n + i;
      if (j < nz) {
        colidx[o] = m->m_colidx[(size_t)j * n + i];
        vals[o] = (double)m->m_matdata[(size_t)j * n + i];
      } else {
        colidx[o] = -1;
        vals[o] = 0.0;
      }
    }
  }
}

void ref_apply_penalty(void* h) { ((RefSession*)h)->fem.ApplyConstraint(FEM::PEN); }

void ref_get_force(void* h, double* f) {
  FemData* fd = ((RefSession*)h)->fem.GetFemData();
  for (int i = 0; i < fd->GetNumDof(); ++i) f[i] = (double)fd->GetForceVector()[i];
}

// ELLmatrix::CG in DEV_OMP (plain CG, x0 = 0; SPRmatrix.cc:405-480).  b = NULL
// uses the force vector.  Returns wall seconds.
double ref_cg(void* h, double* x, const double* b, int maxit, double eps, int nthreads) {
  RefSession* s = (RefSession*)h;
  FemData* fd = s->fem.GetFemData();
  const int n = fd->GetNumDof();
  std::vector<real> xr(n, 0), br(n);
  for (int i = 0; i < n; ++i) br[i] = b ? (real)b[i] : fd->GetForceVector()[i];
  if (nthreads > 0) omp_set_num_threads(nthreads);
  SPRmatrix* K = fd->GetStiffnessMatrix();
  K->SetDeviceMode(SPRmatrix::DEV_OMP);
  double t0 = omp_get_wtime();
  K->CG(xr.data(), br.data(), maxit, (real)eps);
  double t1 = omp_get_wtime();
  for (int i = 0; i < n; ++i) x[i] = (double)xr[i];
  return t1 - t0;
}

void ref_axy(void* h, const double* x, double* y, int nthreads) {
  SPRmatrix* K = ((RefSession*)h)->fem.GetFemData()->GetStiffnessMatrix();
  const int n = K->GetMatDim();
  std::vector<real> xr(n), yr(n);
  for (int i = 0; i < n; ++i) xr[i] = (real)x[i];
  if (nthreads > 0) omp_set_num_threads(nthreads);
  K->Axy(xr.data(), yr.data());
  for (int i = 0; i < n; ++i) y[i] = (double)yr[i];
}

// The reference's ELLmatrix::Axy (ELLmatrix.cc:194-204, OpenMP over rows) on a caller's
// column-major ELL (entry (row, slot) at slot * n + row, as ELLmatrix stores it): the
// arrays are lent to an ELLmatrix object for the one call, so the product is the
// reference's own code on the caller's matrix.  Values and vectors are fem_float (double
// in the FP64 build).  Returns wall seconds.
double ref_ell_axy_external(int n, int width, int32_t* rownnz, int32_t* colidx, real* vals,
                            real* x, real* y, int nthreads) {
  ELLmatrix* m = new ELLmatrix(n);
  real* own_data = m->m_matdata;
  int* own_col = m->m_colidx;
  int* own_nnz = m->m_rownnz;
  const int own_w = m->m_maxrowlen;
  m->m_matdata = vals;
  m->m_colidx = colidx;
  m->m_rownnz = rownnz;
  m->m_maxrowlen = width;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  double t0 = omp_get_wtime();
  m->Axy(x, y);
  double t1 = omp_get_wtime();
  m->m_matdata = own_data;
  m->m_colidx = own_col;
  m->m_rownnz = own_nnz;
  m->m_maxrowlen = own_w;
  delete m;
  return t1 - t0;
}

// ---- raw ELLmatrix access for the reference's known-answer tests ----------
void* ref_mat_new(int n) { return SPRmatrix::CreateMatrix(n, SPRmatrix::ELL); }
void ref_mat_free(void* m) { delete (SPRmatrix*)m; }
void ref_mat_add(void* m, int r, int c, double v) { ((SPRmatrix*)m)->AddElem(r, c, (real)v); }
void ref_mat_set(void* m, int r, int c, double v) { ((SPRmatrix*)m)->SetElem(r, c, (real)v); }
double ref_mat_get(void* m, int r, int c) { return (double)((SPRmatrix*)m)->GetElem(r, c); }
void ref_mat_cg(void* m, double* x, const double* b, int maxit, double eps) {
  SPRmatrix* M = (SPRmatrix*)m;
  const int n = M->GetMatDim();
  std::vector<real> xr(n, 0), br(n);
  for (int i = 0; i < n; ++i) br[i] = (real)b[i];
  M->SetDeviceMode(SPRmatrix::DEV_CPU);
  M->CG(xr.data(), br.data(), maxit, (real)eps);
  for (int i = 0; i < n; ++i) x[i] = (double)xr[i];
}
void ref_mat_axy(void* m, const double* x, double* y) {
  SPRmatrix* M = (SPRmatrix*)m;
  const int n = M->GetMatDim();
  std::vector<real> xr(n), yr(n);
  for (int i = 0; i < n; ++i) xr[i] = (real)x[i];
  M->Axy(xr.data(), yr.data());
  for (int i = 0; i < n; ++i) y[i] = (double)yr[i];
}
int ref_binsearch_step(int32_t* v, int val, int len, int start, int step) {
  return ELLmatrix::BinSearchIntStep(v, val, len, start, step);
}

}  // extern "C"
