// The stiffness strategy a maintainer adds to the reference tree (src/FEM/StiffAlgoCUDA.h):
// StiffAlgo::CalcGlobalStiffness (src/FEM/StiffAlgo.h:46) implemented on the C-ABI of
// include/gpufem_b200.h.  K stays on the device; the C-ABI's view / download calls read
// it.  Compiled and linked against the reference's own headers and CPU library by
// tests/test_adapter_cpu.py.
#ifndef STIFFALGOCUDA_H_
#define STIFFALGOCUDA_H_

#include <vector>

#include "FEM/FemData.h"
#include "FEM/StiffAlgo.h"
#include "gpufem_b200.h"

class StiffAlgoCUDA : public StiffAlgo {
 public:
  StiffAlgoCUDA() { status_ = gf_create(&ctx_, 0); }
  ~StiffAlgoCUDA() override { gf_destroy(ctx_); }
  double CalcGlobalStiffness(FemData* fd) override {
    const int et = fd->GetNumElemNodes() == 4 ? GF_Q4
                 : fd->GetModelDim() == 2     ? GF_Q8
                 : fd->GetNumElemNodes() == 8 ? GF_BRICK8 : GF_BRICK20;
    const int n = fd->GetNumNodes() * fd->GetModelDim();
    std::vector<double> xyz(fd->GetNodeCoords(), fd->GetNodeCoords() + n);
    status_ = gf_mesh_create(ctx_, et, fd->GetNumNodes(), xyz.data(), fd->GetNumElem(),
                             fd->GetElemConnect(), fd->GetNumGaussPts(),
                             fd->GetElasticModulus(), nullptr, fd->GetPoissonCoef(),
                             GF_PLANE_STRESS);
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
};

#endif  // STIFFALGOCUDA_H_
