// The matrix class a maintainer adds to the reference tree (src/SPRmatrix/ELLmatrixCUDA.h):
// the SPRmatrix interface (src/SPRmatrix/SPRmatrix.h:71-89) over the C-ABI context that
// StiffAlgoCUDA assembled into.  K stays on the device: Axy and CG run there
// (gf_spmv_host, gf_solve with GF_SOLVER_CG, the reference's CPU_CG stopping rule from
// x = 0); element access goes through a host copy of the ELL arrays (column-major,
// entry (row, slot) at row + slot * n, as ELLmatrix stores it), written back with
// gf_ell_upload before the next product or solve.
//
// The host copy is tied to the version of the device values (gf_ell_version): when the
// context's matrix changes after the copy was fetched (a reassembly, constraints applied
// on the device), the next access fetches it again, and host edits made before that change
// are dropped, as a reassembly in the reference rebuilds K and drops earlier edits.
// Compiled, linked and run against the reference's own headers by tests/test_adapter_cpu.py.
#ifndef ELLMATRIXCUDA_H_
#define ELLMATRIXCUDA_H_

#include <algorithm>
#include <cstdio>
#include <vector>

#include "SPRmatrix/SPRmatrix.h"
#include "gpufem_b200.h"

class ELLmatrixCUDA : public SPRmatrix {
 public:
  explicit ELLmatrixCUDA(gf_ctx* ctx) : ctx_(ctx) {}
  using SPRmatrix::CG;

  void SetElem(const int row, const int col, const fem_float val) override {
    if (fem_float* p = slot(row, col)) { *p = val; dirty_ = true; }
  }
  void AddElem(const int row, const int col, const fem_float val) override {
    if (fem_float* p = slot(row, col)) { *p += val; dirty_ = true; }
  }
  fem_float GetElem(const int row, const int col) override {
    const fem_float* p = slot(row, col);
    return p ? *p : fem_float(0);
  }
  size_t GetMatSize() override {
    int32_t n = 0, w = 0;
    return gf_ell_view(ctx_, kDtype, &n, &w, nullptr, nullptr, nullptr) == GF_OK ? (size_t)n : 0;
  }
  void SetNNZInfo(int, int) override {}
  int GetNNZ() override {
    fetch();
    int s = 0;
    for (int r : rownnz_) s += r;
    return s;
  }
  void Clear() override {
    fetch();
    std::fill(vals_.begin(), vals_.end(), fem_float(0));
    dirty_ = true;
  }
  void Axy(fem_float* x, fem_float* y) override {
    flush();
    const size_t n = GetMatSize();
    std::vector<double> xd(x, x + n), yd(n);
    if (n && (status_ = gf_spmv_host(ctx_, kDtype, xd.data(), yd.data())) == GF_OK)
      std::copy(yd.begin(), yd.end(), y);
    else if (n)
      report("Axy");
  }
  // The reference's CPU_CG returns its current x whether or not it converged; so does this
  // one (solution copied back on OK, NOT_CONVERGED and STALLED).  status() tells which.
  void CG(fem_float* x, fem_float* b, int n_iterations, fem_float epsilon) override {
    flush();
    const size_t n = GetMatSize();
    if (!n) return;
    std::vector<double> bd(b, b + n), xd(n, 0.0);
    status_ = gf_set_force(ctx_, bd.data());
    if (status_ != GF_OK) {
      report("CG (set_force)");
      std::copy(xd.begin(), xd.end(), x);
      return;
    }
    gf_solve_opts o{};
    o.solver = GF_SOLVER_CG;
    o.matrix = kDtype;
    o.max_iter = n_iterations;
    o.tol = epsilon;
    gf_solve_info info{};
    status_ = gf_solve(ctx_, &o, &info);
    iterations_ = info.iterations;
    if (status_ == GF_OK || status_ == GF_ERR_NOT_CONVERGED || status_ == GF_ERR_STALLED)
      gf_get_solution(ctx_, xd.data());
    if (status_ != GF_OK) report("CG");
    std::copy(xd.begin(), xd.end(), x);
  }
  void Teardown() override {
    rownnz_.clear();
    colidx_.clear();
    vals_.clear();
    fetched_ = dirty_ = false;
  }
  gf_status status() const { return status_; }  // of the last Axy / CG
  int iterations() const { return iterations_; } // of the last CG

 private:
  static constexpr int32_t kDtype = sizeof(fem_float) == 8 ? GF_F64 : GF_F32;

  int64_t device_version() {
    int64_t v = -1;
    return gf_ell_version(ctx_, kDtype, &v) == GF_OK ? v : -1;
  }
  void report(const char* what) {
    std::fprintf(stderr, "ELLmatrixCUDA::%s: gf_status %d: %s\n", what, (int)status_,
                 gf_last_error(ctx_));
  }
  void fetch() {
    if (fetched_ && device_version() == version_) return;
    Teardown();  // first access, or the device matrix changed: host copy and edits are stale
    int32_t n = 0, w = 0;
    if (gf_ell_view(ctx_, kDtype, &n, &w, nullptr, nullptr, nullptr) != GF_OK) return;
    rownnz_.resize(n);
    colidx_.resize((size_t)n * w);
    vals_.resize((size_t)n * w);
    if (gf_ell_download(ctx_, kDtype, rownnz_.data(), colidx_.data(), vals_.data()) != GF_OK) {
      Teardown();
      return;
    }
    n_ = n;
    w_ = w;
    version_ = device_version();
    fetched_ = true;
  }
  void flush() {
    if (!dirty_) return;
    if (device_version() != version_) {  // K changed on the device after these edits
      Teardown();
      return;
    }
    std::vector<double> v(vals_.begin(), vals_.end());
    status_ = gf_ell_upload(ctx_, n_, w_, rownnz_.data(), colidx_.data(), v.data());
    if (status_ != GF_OK) report("flush (upload)");
    version_ = device_version();
    dirty_ = false;
  }
  fem_float* slot(int row, int col) {
    fetch();
    if (!fetched_ || row < 0 || row >= n_) return nullptr;
    for (int s = 0; s < rownnz_[row]; ++s)  // columns ascend within a row
      if (colidx_[(size_t)s * n_ + row] == col) return &vals_[(size_t)s * n_ + row];
    return nullptr;
  }

  gf_ctx* ctx_;
  int32_t n_ = 0, w_ = 0;
  int64_t version_ = -1;
  std::vector<int32_t> rownnz_, colidx_;
  std::vector<fem_float> vals_;
  bool fetched_ = false, dirty_ = false;
  gf_status status_ = GF_OK;
  int iterations_ = 0;
};

#endif  // ELLMATRIXCUDA_H_
