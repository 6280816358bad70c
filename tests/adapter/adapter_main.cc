// Reads a neutral file with the reference's FileIO, initialises its FemData as
// FEM::Init does, assembles through StiffAlgoCUDA and uses the result through
// ELLmatrixCUDA (size, nnz, an element and a product through the SPRmatrix interface;
// its CG is compiled and linked with the class).  Prints the gf_status of each step and the values.  Without a GPU
// gf_create reports GF_ERR_CUDA and every call fails cleanly on the null context.
#include <cstdio>
#include <string>

#include <cmath>
#include <vector>

#include "ELLmatrixCUDA.h"
#include "StiffAlgoCUDA.h"
#include "Utils/fileIO.h"

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  FileIO io;
  if (!io.ReadNF(std::string(argv[1]))) return 3;
  FemData fd;
  fd.Init(SPRmatrix::ELL, 2, (fem_float)210e3, (fem_float)0.3, &io);
  StiffAlgoCUDA algo;
  std::printf("create %d\n", (int)algo.status());
  algo.SetParallelColoring(false);
  const double s = algo.CalcGlobalStiffness(&fd);
  std::printf("assemble %d %g\n", (int)algo.status(), s);
  ELLmatrixCUDA K(algo.context());
  const size_t n = K.GetMatSize();
  std::printf("ell %zu %d\n", n, K.GetNNZ());
  if (n) {
    std::printf("k00 %g\n", (double)K.GetElem(0, 0));
    // K 1 = 0 for a free body: rigid translation of every node
    std::vector<fem_float> one(n, 1), y(n, 1);
    K.Axy(one.data(), y.data());
    double ymax = 0, kmax = std::fabs((double)K.GetElem(0, 0));
    for (size_t i = 0; i < n; ++i) ymax = std::fmax(ymax, std::fabs((double)y[i]));
    std::printf("rigid %g\n", ymax / kmax);
  }
  return 0;
}
