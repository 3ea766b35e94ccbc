// Solver drivers (host C++) used behind the C-ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

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
  // Cycles (prec 8) or FP64 defect-correction steps around one FP32 cycle (prec 4; x, b FP64)
  // until ||b - A x|| <= tol * ||b - A x0|| or maxIter; returns the iterations taken.
  int solveTo(int x, int b, int L, double tol, int maxIter, double* relRes, double* history, int historyCap);
  void coarseSolve(int x, int b, int L);
  // One cycle x <- MG(x, b) on level L: replayed from a captured CUDA graph when the coarse solve
  // runs on the device and pre + post is even (every smoothed buffer returns to its address).
  void runCycle(int x, int b, int L);
  void setGraphs(bool on);
  bool deviceCoarse() const;  // the coarse level has vertex and edge DoFs only

  struct Captured {
    std::vector<uintptr_t> sig;
    cudaGraphExec_t exec = nullptr;
    unsigned long long launches = 0;
  };
  bool graphs = true;
  std::vector<Captured> captured;
  std::vector<std::vector<uintptr_t>> warm;  // signatures that ran eagerly once
  std::vector<uintptr_t> signature(int x, int b, int L);

  Storage& s;
  int op, minL, maxL, pre, post;
  double omega;
  int cycle, coarseMaxIter;
  double coarseTol;
  int prec;
  int tmp, cp, cz, cap, cr;
  // FP32 solvers: FP64 coarse-grid workspace and the FP32 correction / defect hierarchy
  int cx64 = -1, cb64 = -1, x32 = -1, b32 = -1, r64 = -1;
};

// P2 geometric multigrid on P2 levels [minL, maxL] (the P2 DoFs of level L are the vertex DoFs
// of level L + 1): multicolour P2 SOR, quadratic transfers, CG on the coarsest level; FP64.
struct P2Gmg {
  P2Gmg(Storage& s, int op, int minL, int maxL, int pre, int post, double omega, int coarseMaxIter,
        double coarseTol, int prec = 8);
  ~P2Gmg();
  void solveRecursively(int x, int b, int L);
  int solveTo(int x, int b, int L, double tol, int maxIter, double* relRes, double* history, int historyCap);
  int coarseCg(int x, int b, int L);

  Storage& s;
  int op, minL, maxL, pre, post;
  double omega;
  int coarseMaxIter;
  double coarseTol;
  int tmp, cp, cz, cap, cr;
  int prec = 8;                      // precision of the cycle (4: FP32 hierarchy, coarse CG in FP64)
  int cx64 = -1, cb64 = -1;          // FP64 coarse-level copies for an FP32 cycle
  bool symmetric = false;  // post-smoothing with backward sweeps (a symmetric cycle)
};

// MinResSolver (solvers/MinresSolver.hpp:63-125) for the P2-P1 Taylor-Hood Stokes system on
// level L, preconditioned block-diagonally: one symmetric P2 V(nu, nu) cycle from zero per velocity
// component and the inverse lumped P1 mass on the pressure. Velocity DoFs flagged
// Inner | Neumann are unknowns (the Dirichlet values of u are kept), every pressure DoF is an
// unknown; the pressure is returned with zero mean. Returns the iterations; relRes is the
// preconditioned residual norm relative to the initial one.
int stokesMinres(Storage& s, int op, const int u[3], int p, const int f[3], int g, int L, int nu, int maxIter,
                 double tol, double* relRes, double* history, int historyCap, int precondPrec = 8);

}  // namespace hg
