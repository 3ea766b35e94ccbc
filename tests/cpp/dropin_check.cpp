// A C++ caller of the drop-in classes (include/hyteg_b200.hpp), written as code against the
// reference's P1 multigrid path would be: storage from meshCuboid, P1 functions, the constant
// Laplace operator, one apply, one SOR sweep, one V(3,3) multigrid cycle, and the error path.
//
//   dropin_check <level> <output file>
//
// Writes the level buffers of y = A x, of x after smooth_sor and of x after the cycle (in that
// order, doubles, the reference's per-primitive layout) to the output file; the GPU test runs the
// same sequence through the Python mirror of the same C-ABI and compares the bits. Exit status 0
// on success, 1 on a failed check, 2 on bad arguments.
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "hyteg_b200.hpp"

using namespace hyteg_b200;

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s <level> <output file>\n", argv[0]);
    return 2;
  }
  const uint_t L = (uint_t)std::atoi(argv[1]);
  try {
    auto storage = PrimitiveStorage::cuboid({0, 0, 0}, {1, 1, 1}, 2, 2, 2, L);
    P1ConstantLaplaceOperator A(storage, 0, L);
    P1Function x("x", storage, 0, L), b("b", storage, 0, L), y("y", storage, 0, L);
    x.fillRandom(1, L, All);
    b.fillRandom(2, L, All);

    A.apply(x, y, L, Inner);
    const std::vector<real_t> ay = y.download(L);

    A.smooth_sor(x, b, 1.0, L, Inner | NeumannBoundary);
    const std::vector<real_t> sx = x.download(L);

    GeometricMultigridSolver gmg(storage, std::make_shared<SORSmoother>(1.0),
                                 std::make_shared<CGSolver>(storage, 0, 0, 50, 1e-16),
                                 std::make_shared<P1toP1LinearRestriction>(),
                                 std::make_shared<P1toP1LinearProlongation>(), 0, L, 3, 3);
    gmg.solve(A, x, b, L);
    const std::vector<real_t> gx = x.download(L);

    // the reference's error behaviour: a level outside the function's levels throws
    bool threw = false;
    try {
      A.apply(x, y, L + 1, Inner);
    } catch (const std::runtime_error& e) {
      threw = std::string(e.what()).find("level") != std::string::npos;
    }
    if (!threw) {
      std::fprintf(stderr, "apply on a level beyond the storage did not throw\n");
      return 1;
    }
    // A x of a constant vanishes at inner DoFs (P1LaplaceOperator3DTest)
    x.interpolate(2.5, L, All);
    A.apply(x, y, L, Inner);
    const real_t n2 = y.dotGlobal(y, L, Inner);
    if (!(n2 < 1e-20)) {
      std::fprintf(stderr, "A const != 0: |y|^2 = %g\n", n2);
      return 1;
    }

    FILE* f = std::fopen(argv[2], "wb");
    if (!f) {
      std::fprintf(stderr, "cannot write %s\n", argv[2]);
      return 2;
    }
    for (const auto* v : {&ay, &sx, &gx}) std::fwrite(v->data(), sizeof(real_t), v->size(), f);
    std::fclose(f);
    storage->synchronize();
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  std::printf("dropin_check ok (level %zu)\n", L);
  return 0;
}
