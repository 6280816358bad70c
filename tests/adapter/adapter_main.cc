// Reads a neutral file with the reference's FileIO, initialises its FemData as
// FEM::Init does, and assembles through StiffAlgoCUDA.  Prints the gf_status of each
// step, and with a GPU the matrix shape.  Without a GPU gf_create reports GF_ERR_CUDA and
// the strategy's calls fail cleanly on the null context.
#include <cstdio>
#include <string>

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
  int32_t n = 0, w = 0;
  if (algo.context() && gf_ell_view(algo.context(), sizeof(fem_float) == 8 ? GF_F64 : GF_F32,
                                    &n, &w, nullptr, nullptr, nullptr) == GF_OK)
    std::printf("ell %d %d\n", n, w);
  return 0;
}
