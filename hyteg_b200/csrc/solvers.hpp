// Solver drivers (host C++) used behind the C-ABI.
#pragma once

namespace hg {

struct Storage;

// Returns the number of iterations taken; workspace functions must cover level L.
int cgSolve(Storage& s, int op, int x, int b, int L, int maxIter, double tol, int p, int z, int ap, int r,
            double* finalRes);

struct Gmg {
  Gmg(Storage& s, int op, int minL, int maxL, int pre, int post, double omega, int cycle, int coarseMaxIter,
      double coarseTol, int prec);
  ~Gmg();
  void solve(int x, int b, int L);
  void solveRecursively(int x, int b, int L);

  Storage& s;
  int op, minL, maxL, pre, post;
  double omega;
  int cycle, coarseMaxIter;
  double coarseTol;
  int prec;
  int tmp, cp, cz, cap, cr;
};

}  // namespace hg
