// Drives the C++ adaptor (include/exahype_b200.hpp) the way the reference's
// unit test drives its kernel template (GenericEulerKernelTest3D.cpp:618-773):
// the test object is the SolverType.  Reads luh (nData-strided) from argv[1],
// writes lQhbnd, lFhbnd, lQhi, lFhi (raw doubles) to argv[2].
#include <cstdio>
#include <vector>

#include "exahype_b200.hpp"

struct EulerTestSolver {
  static constexpr int NumberOfVariables = 5;
  static constexpr int NumberOfParameters = 1;
  static constexpr int Order = 3;
};

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  constexpr int B = 4, D = 6, V = 5;
  std::vector<double> luh(B * B * B * D);
  FILE* f = std::fopen(argv[1], "rb");
  if (!f || std::fread(luh.data(), sizeof(double), luh.size(), f) != luh.size()) return 3;
  std::fclose(f);
  std::vector<double> qb(6 * B * B * D), fb(6 * B * B * V), qhi(B * B * B * D), fhi(4 * B * B * B * V);
  std::vector<double> lqi(B * B * B * B * D), lfi(B * B * B * B * 4 * V);
  double* stu[1] = {lqi.data()};
  double* stf[1] = {lfi.data()};
  EulerTestSolver solver;
  const double dx[3] = {0.05, 0.05, 0.05};
  try {
    exahype_b200::kernels::aderdg::generic::c::spaceTimePredictorNonlinear<3, true, true, false>(
        solver, qb.data(), fb.data(), stu, stf, qhi.data(), fhi.data(), nullptr, luh.data(), dx,
        1.083937460199773e-3);
  } catch (const exahype_b200::Error& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 4;
  }
  f = std::fopen(argv[2], "wb");
  if (!f) return 5;
  std::fwrite(qb.data(), sizeof(double), qb.size(), f);
  std::fwrite(fb.data(), sizeof(double), fb.size(), f);
  std::fwrite(qhi.data(), sizeof(double), qhi.size(), f);
  std::fwrite(fhi.data(), sizeof(double), fhi.size(), f);
  std::fclose(f);
  return 0;
}
