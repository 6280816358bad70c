// The stiffness strategy a maintainer adds to the reference tree (src/FEM/StiffAlgoCUDA.h):
// StiffAlgo::CalcGlobalStiffness (src/FEM/StiffAlgo.h:46) implemented on the C-ABI of
// include/gpufem_b200.h.  K stays on the device; the C-ABI's view / download calls read
// it (ELLmatrixCUDA wraps them in the SPRmatrix interface).
//
// What it passes through from the reference's FemData (src/FEM/FemData.h:79-103): the
// element family (node count and model dimension), packed node coordinates, 1-based
// connectivity, Gauss points per direction, E and nu, and for 2-D models the analysis:
// the constitutive matrix FemData built (CalcConstituitiveData, FemData.cc:322-365) is read
// back and classified by its ratio D[0][1] / D[0][0] (nu for plane stress,
// nu / (1 - nu) for plane strain), so whatever D the caller's FemData holds is the law
// assembled here.  Per-element moduli, which FemData has no field for, come from
// SetElementModuli.  Compiled and linked against the reference's headers and CPU library
// by tests/test_adapter_cpu.py.
#ifndef STIFFALGOCUDA_H_
#define STIFFALGOCUDA_H_

#include <cmath>
#include <vector>

#include "FEM/FemData.h"
#include "FEM/StiffAlgo.h"
#include "gpufem_b200.h"

class StiffAlgoCUDA : public StiffAlgo {
 public:
  StiffAlgoCUDA() { status_ = gf_create(&ctx_, 0); }
  ~StiffAlgoCUDA() override { gf_destroy(ctx_); }

  // Young's modulus per element (nelem values, kept by the caller until the next
  // CalcGlobalStiffness), or nullptr for FemData's scalar E.
  void SetElementModuli(const double* E_elem) { E_elem_ = E_elem; }

  // GF_PLANE_STRESS or GF_PLANE_STRAIN from FemData's 2-D constitutive matrix; -1 when it
  // matches neither (then nothing is assembled and status() is GF_ERR_INVALID_ARG).
  static int Analysis2D(FemData* fd) {
    fem_float** D = fd->GetConstituitiveMat();
    const double nu = fd->GetPoissonCoef();
    if (!D || !(D[0][0] > 0)) return -1;
    const double ratio = (double)D[0][1] / (double)D[0][0];
    const double tol = sizeof(fem_float) == 8 ? 1e-12 : 1e-6;
    if (std::fabs(ratio - nu) <= tol * (1 + std::fabs(nu))) return GF_PLANE_STRESS;
    const double strain = nu / (1 - nu);
    if (std::fabs(ratio - strain) <= tol * (1 + std::fabs(strain))) return GF_PLANE_STRAIN;
    return -1;
  }

  double CalcGlobalStiffness(FemData* fd) override {
    const int dim = fd->GetModelDim();
    const int et = fd->GetNumElemNodes() == 4 ? GF_Q4
                 : dim == 2                   ? GF_Q8
                 : fd->GetNumElemNodes() == 8 ? GF_BRICK8 : GF_BRICK20;
    const int analysis = dim == 2 ? Analysis2D(fd) : GF_PLANE_STRESS;
    if (analysis < 0) {
      status_ = GF_ERR_INVALID_ARG;
      return 0.0;
    }
    const int n = fd->GetNumNodes() * dim;
    std::vector<double> xyz(fd->GetNodeCoords(), fd->GetNodeCoords() + n);
    status_ = gf_mesh_create(ctx_, et, fd->GetNumNodes(), xyz.data(), fd->GetNumElem(),
                             fd->GetElemConnect(), fd->GetNumGaussPts(),
                             fd->GetElasticModulus(), E_elem_, fd->GetPoissonCoef(), analysis);
    if (status_ != GF_OK) return 0.0;
    status_ = gf_assemble(ctx_, sizeof(fem_float) == 8 ? GF_F64 : GF_F32,
                          m_usecoloring ? GF_SCATTER_COLOR : GF_SCATTER_AUTO,
                          GF_ENGINE_CUDA_CORE);
    return status_ == GF_OK ? gf_last_device_seconds(ctx_) : 0.0;
  }
  gf_ctx* context() { return ctx_; }
  gf_status status() const { return status_; }

 private:
  gf_ctx* ctx_ = nullptr;
  gf_status status_ = GF_OK;
  const double* E_elem_ = nullptr;
};

#endif  // STIFFALGOCUDA_H_
