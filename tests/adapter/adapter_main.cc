// The reference's FemTest / RunBatches flow (src/Test/FemTest.cpp:91-101,
// src/interface.cpp:545-551) driven through the reference-side classes StiffAlgoCUDA and
// ELLmatrixCUDA, with the reference's own StiffAlgoCPU and CPU_CG beside them on the same
// FemData:
//
//   FileIO::ReadNF -> FEM::Init / FemData::Init (ELL, ngp, E, nu) [-> SetAnalysisType]
//   -> StiffAlgoCUDA::CalcGlobalStiffness           (K on the device)
//   -> FEM::CalcStiffnessMat with StiffAlgoCPU      (K_ref in the reference's ELLmatrix)
//   -> K compared entry by entry through the SPRmatrix interface of both
//   -> per-element moduli 2E through StiffAlgoCUDA: K must double (and the adapter's host
//      cache must notice the reassembly)
//   -> FEM::ApplyConstraint(PEN) on K_ref; the same supports and penalty through the C-ABI
//   -> ELLmatrixCUDA::CG against ELLmatrix::CG (CPU_CG) on the force vector.
//
// Usage: adapter <mesh.nf> <gauss points per direction> <analysis string | ->
// Prints one "key value..." line per step.  Without a GPU gf_create reports GF_ERR_CUDA,
// every later call fails cleanly on the null context and the driver stops after "ell".
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ELLmatrixCUDA.h"
#include "FEM/fem.h"
#include "StiffAlgoCUDA.h"
#include "Utils/fileIO.h"

// max over rows of max_j |A(i,j) - s B(i,j)| / max_j |s B(i,j)|, over all columns j
static double row_rel_diff(SPRmatrix& A, SPRmatrix& B, int n, double s) {
  double worst = 0.0;
  for (int i = 0; i < n; ++i) {
    double dmax = 0.0, bmax = 0.0;
    for (int j = 0; j < n; ++j) {
      const double b = s * (double)B.GetElem(i, j);
      dmax = std::fmax(dmax, std::fabs((double)A.GetElem(i, j) - b));
      bmax = std::fmax(bmax, std::fabs(b));
    }
    worst = std::fmax(worst, bmax > 0 ? dmax / bmax : dmax);
  }
  return worst;
}

int main(int argc, char** argv) {
  if (argc < 4) return 2;
  const int ngp = std::atoi(argv[2]);
  const fem_float E = (fem_float)210e3, nu = (fem_float)0.3;
  FileIO io;
  if (!io.ReadNF(std::string(argv[1]))) return 3;
  FEM fem;
  fem.Init(true, FEM::CPU);
  FemData* fd = fem.GetFemData();
  fd->Init(SPRmatrix::ELL, ngp, E, nu, &io);
  // FemData::Init leaves the 2-D analysis string dangling; name one that outlives it
  if (fd->GetModelDim() == 2 && std::strcmp(argv[3], "-") != 0) fd->SetAnalysisType(argv[3]);

  StiffAlgoCUDA algo;
  std::printf("create %d\n", (int)algo.status());
  algo.SetParallelColoring(false);
  const double s = algo.CalcGlobalStiffness(fd);
  std::printf("assemble %d %g\n", (int)algo.status(), s);
  ELLmatrixCUDA K(algo.context());
  const int n = (int)K.GetMatSize();
  std::printf("ell %d %d\n", n, K.GetNNZ());
  if (n == 0) return 0;
  if (fd->GetModelDim() == 2) std::printf("analysis %d\n", StiffAlgoCUDA::Analysis2D(fd));

  // the reference's own CPU assembly of the same FemData
  fem.SetDeviceMode(FEM::CPU);
  fem.SetUseColoring(false);
  fem.CalcStiffnessMat();
  SPRmatrix& Kref = *fd->GetStiffnessMatrix();
  std::printf("kdiff %.3e\n", row_rel_diff(K, Kref, n, 1.0));

  // per-element moduli through the strategy: 2E everywhere doubles K
  std::vector<double> E2(fd->GetNumElem(), 2.0 * (double)E);
  algo.SetElementModuli(E2.data());
  algo.CalcGlobalStiffness(fd);
  std::printf("kdiff2x %d %.3e\n", (int)algo.status(), row_rel_diff(K, Kref, n, 2.0));
  algo.SetElementModuli(nullptr);
  algo.CalcGlobalStiffness(fd);
  std::printf("kdiff1x %d %.3e\n", (int)algo.status(), row_rel_diff(K, Kref, n, 1.0));

  // penalty constraints: the reference's FEM::ApplyConstraint(PEN) on K_ref, the same
  // supports through the C-ABI on the device matrix
  fem.ApplyConstraint(FEM::PEN);
  const int dim = fd->GetModelDim(), nsup = fd->GetNodeNumConstraints();
  std::vector<int32_t> sup((size_t)nsup * (dim + 1));
  for (int i = 0; i < nsup; ++i)
    for (int j = 0; j <= dim; ++j) sup[(size_t)i * (dim + 1) + j] = fd->GetNodeConstraints()[i][j];
  gf_status st = gf_set_supports(algo.context(), nsup, sup.data());
  if (st == GF_OK) st = gf_apply_constraints(algo.context(), GF_BC_PENALTY);
  std::printf("constraints %d %.3e\n", (int)st, row_rel_diff(K, Kref, n, 1.0));

  // CG on the force vector: ELLmatrixCUDA::CG against the reference's CPU_CG
  std::vector<fem_float> f(fd->GetForceVector(), fd->GetForceVector() + n);
  std::vector<fem_float> xc(n, 0), xr(n, 0);
  const int maxit = 20000;
  const fem_float eps = sizeof(fem_float) == 8 ? (fem_float)1e-10 : (fem_float)1e-5;
  K.CG(xc.data(), f.data(), maxit, eps);
  Kref.SetDeviceMode(SPRmatrix::DEV_CPU);
  Kref.CG(xr.data(), f.data(), maxit, eps);
  double dn = 0.0, rn = 0.0;
  for (int i = 0; i < n; ++i) {
    dn += ((double)xc[i] - (double)xr[i]) * ((double)xc[i] - (double)xr[i]);
    rn += (double)xr[i] * (double)xr[i];
  }
  std::printf("cg %d %d %.3e %.3e\n", (int)K.status(), K.iterations(), std::sqrt(dn / rn),
              std::sqrt(rn));
  return 0;
}
