// Solver drivers (host C++) used behind the C-ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace hg {

namespace dev {
struct BatchMap;
}

struct Storage;
struct DevBuf;
struct CompactCycle;

// Hierarchical timers of a solver's phases measured on the device (the reference's
// walberla::WcTimingTree around GeometricMultigridSolver / CGSolver). start/stop record CUDA
// events on the storage's stream; intervals are resolved when the tree is read. Each node keeps
// the waLBerla Timer statistics of its intervals: total, count, min, max, average and variance
// (seconds). json() writes the tree with a "Remainder" child under every node that has
// children (the time of the node not covered by them), as the reference writes
// getCopyWithRemainder() with the waLBerla TimingTree JSON layout: a node is an object with
// "total", "average", "count", "min", "max", "variance" and one member per child.
struct TimingTree {
  struct Node {
    std::vector<std::pair<std::string, Node>> children;  // in order of first start
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
    std::vector<int> pendingCount;  // applications each interval stands for
    double total = 0, min = 0, max = 0, sumSq = 0;
    int64_t count = 0;
    cudaEvent_t open = nullptr;
    Node& child(const std::string& name);
  };
  Node root;
  std::vector<Node*> stack{&root};
  std::vector<cudaEvent_t> pool;
  ~TimingTree();
  void start(cudaStream_t s, const std::string& name);
  // `applications` > 1: the interval covers that many applications of the phase (a group of
  // smoother sweeps); they count separately and share the interval's time equally.
  void stop(cudaStream_t s, const std::string& name, int applications = 1);
  void resolve();  // waits for the recorded events
  void reset();
  std::string json();
};

// Captured CUDA graphs of one solver's cycle, keyed by a signature: every device address the
// cycle reads or writes plus what fixes its kernel arguments. run() replays a graph captured
// under the same signature. A new signature runs eagerly (which builds lazily allocated tables
// and buffers); once a signature has run eagerly and come back unchanged, its next cycle is
// captured and replayed from then on. At most four graphs are kept.
struct GraphCache {
  struct Captured {
    std::vector<uintptr_t> sig;
    cudaGraphExec_t exec = nullptr;
    unsigned long long launches = 0;
  };
  std::vector<Captured> captured;
  std::vector<std::vector<uintptr_t>> warm;  // signatures that ran eagerly once
  ~GraphCache() { clear(); }
  void clear();
  void run(Storage& s, const std::function<std::vector<uintptr_t>()>& signature, const std::function<void()>& cycle);
};

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
  // solveTo for the first `active` copies of a storage of disjoint copies (dev::BatchMap) at once:
  // one cycle (or defect-correction step) of the whole storage per iteration, then every copy's
  // residual norm (dNorms: device scratch of bm.copies doubles). Copy i stops at the first
  // iteration its own relative residual reaches tol[i] (or at maxIter[i]): its x of that iteration is
  // copied to xOut, and iterations[i], relRes[i] are its own. The copies are not coupled and the
  // per-copy norms equal their single-mesh norms bit for bit; with one coarse-CG group per copy
  // (setCoarseGroups) every copy's iterates are its single-mesh iterates bit for bit.
  void solveToBatch(int x, int b, int xOut, int L, const double* tol, const int* maxIter, const dev::BatchMap& bm,
                    int active, double* dNorms, int* iterations, double* relRes);
  void coarseSolve(int x, int b, int L);
  // One cycle x <- MG(x, b) on level L: replayed from a captured CUDA graph when the coarse solve
  // runs on the device and pre + post is even (every smoothed buffer returns to its address).
  void runCycle(int x, int b, int L);
  void setGraphs(bool on);
  bool deviceCoarse() const;  // the coarse level has vertex and edge DoFs only

  bool graphs = true;
  GraphCache cache;
  std::vector<uintptr_t> signature(int x, int b, int L);
  // device-timed phases (set_timing); cycles run eagerly while it is on
  std::unique_ptr<TimingTree> timing;
  void setTiming(bool on);

  Storage& s;
  int op, minL, maxL, pre, post;
  double omega;
  int cycle, coarseMaxIter;
  double coarseTol;
  int prec;
  int tmp, cp, cz, cap, cr;
  // FP32 solvers: FP64 coarse-grid workspace and the FP32 correction / defect hierarchy
  int cx64 = -1, cb64 = -1, x32 = -1, b32 = -1, r64 = -1;
  // Device coarse CG: one block per group of unknowns, the whole mesh (1) or each copy of a
  // storage of `groups` disjoint copies, so copies iterate and stop independently. The work
  // lists (per group its owned DoFs and halo entries) are built here, on the host.
  void setCoarseGroups(int groups);
  int coarseGroups = 1;
  std::unique_ptr<DevBuf> cgDofs, cgDofOff, cgComm, cgCommOff;
  // Compact coarse cycle (compact.hpp): levels minL .. compactTop of a V-cycle as one launch, one
  // block (or cluster of compactCluster blocks) per group. compactTop is the highest level whose
  // unknowns per group are at most compactMaxDofs (-1: none, or a W-cycle). Off while the timing
  // tree is on, which times the cycle level by level.
  int compactMaxDofs = 6000, compactCluster = 1, compactTop = -1;
  std::unique_ptr<CompactCycle> compact;
  void setCompact(int maxDofs, int cluster);
  void buildCompact(bool strict = false);
};

// P2 geometric multigrid on P2 levels [minL, maxL] (the P2 DoFs of level L are the vertex DoFs
// of level L + 1): multicolour P2 SOR, quadratic transfers, an exact solve on the coarsest level
// (the inverse of A on its unknowns, up to kCoarseDirectMax of them; CG beyond), in FP64.
struct P2Gmg {
  static constexpr int kCoarseDirectMax = 1024;
  P2Gmg(Storage& s, int op, int minL, int maxL, int pre, int post, double omega, int coarseMaxIter,
        double coarseTol, int prec = 8);
  ~P2Gmg();
  void solveRecursively(int x, int b, int L);
  // One cycle, replayed from a captured CUDA graph when the coarse solve runs on the device.
  void runCycle(int x, int b, int L);
  int solveTo(int x, int b, int L, double tol, int maxIter, double* relRes, double* history, int historyCap);
  int coarseCg(int x, int b, int L);
  void coarseSolve(int x, int b, int L);  // FP64 x, b on the coarsest level
  bool buildCoarseDirect();               // false when the coarse level has too many unknowns
  std::vector<uintptr_t> signature(int x, int b, int L);
  int coarseN = -1;  // unknowns of the exact coarse solve (0: CG; -1: not yet built)
  std::unique_ptr<DevBuf> coarseIdx, coarseInv;
  bool graphs = true;
  GraphCache cache;

  Storage& s;
  int op, minL, maxL, pre, post;
  double omega;
  int coarseMaxIter;
  double coarseTol;
  int tmp, cp, cz, cap, cr;
  int prec = 8;                      // precision of the cycle (4: FP32 hierarchy, coarse CG in FP64)
  int cx64 = -1, cb64 = -1;          // FP64 coarse-level copies for an FP32 cycle
  bool symmetric = false;  // post-smoothing with backward sweeps (a symmetric cycle)
  int lane = 0;            // the storage's P2 scratch lane its cycles use (Storage::p2Lane)
};

// Geometric multigrid on the whole P2-P1 Taylor-Hood system (GeometricMultigridSolver with
// P2P1TaylorHoodStokesOperator, GeometricMultigridSolver.hpp:136-235) with the Uzawa smoother
// (UzawaSmoother.hpp:338-423, block-Laplace variant without stabilisation):
//   r_u = f - D^T p;  velocitySweeps times: one forward P2 SOR sweep (omega 1) per component on
//   A u_k = r_u,k;  r_p = g - D u;  p += omega r_p / diag(PSPG)
// and the composite transfers (P2P1StokesToP2P1StokesRestriction / Prolongation: quadratic on the
// velocity, linear on the pressure). Velocity DoFs flagged Inner | Neumann are unknowns; the
// pressure is all-inner (every DoF an unknown, P2P1TaylorHoodFunction.hpp:61). The coarsest level
// is solved by the pseudo-inverse of the operator on its unknowns (the constant pressure and the
// pressure DoFs coupled to no free velocity DoF span its null space), built once, when it has at
// most kCoarseMax unknowns; a larger coarsest level (the reference solves it by LU) is solved by
// preconditioned MINRES to a relative residual of kCoarseTol (zero-mean pressure, as the
// pseudo-inverse gives). FP64.
struct StokesGmg {
  static constexpr int kCoarseMax = 1024;
  static constexpr double kCoarseTol = 1e-11;
  static constexpr int kCoarseMaxIter = 1000;
  StokesGmg(Storage& s, int op, int minL, int maxL, int pre, int post, double omega, int velocitySweeps);
  ~StokesGmg();
  void smooth(const int u[3], int p, const int f[3], int g, int L);
  void solveRecursively(const int u[3], int p, const int f[3], int g, int L);
  // V-cycles until ||b - K x|| <= tol ||b - K x0|| (unknowns only) or maxIter; returns the cycles.
  int solveTo(const int u[3], int p, const int f[3], int g, int L, double tol, int maxIter, double* relRes,
              double* history, int historyCap);
  double residualNorm(const int u[3], int p, const int f[3], int g, int L);
  // estimateUzawaRelaxationParameter (UzawaSmoother.hpp:52-68): iters power iterations
  // (SpectrumEstimation.hpp:57-81) on E = M_lumped^-1 D S D^T, S = velocitySweeps forward P2 SOR
  // sweeps per component from zero, started from seeded uniform [0, 1) values.
  double estimateOmega(int L, int iters, uint64_t seed);
  void coarseSolve(const int u[3], int p, const int f[3], int g);
  void buildCoarse();

  Storage& s;
  int op, minL, maxL, pre, post;
  double omega;
  int velocitySweeps;
  int pspg = -1;               // P1 PSPG operator on [minL, maxL]
  int ru[3], rp;               // Uzawa residuals
  int tu[3], tp;               // Stokes residual / restricted right-hand sides
  std::vector<int> invDiag;    // per pressure level minL..maxL: 1 / diag(PSPG)
  int coarseN = -1;            // coarse unknowns of the dense pseudo-inverse; 0: none
  bool coarseIterative = false;  // the coarsest level is solved by MINRES instead
  int coarseIterations = 0;      // MINRES iterations of the last coarse solve
  std::unique_ptr<DevBuf> coarseIdx, coarseComp, coarseInv;
  // The velocity sweeps of a smoothing step run one stream per component (each with its own P2
  // scratch lane) once the level has been smoothed in order (which builds every table they use)
  // and the storage allows it (concurrentComponents).
  cudaStream_t laneStream[2] = {nullptr, nullptr};
  cudaEvent_t forkEvent = nullptr, joinEvent[2] = {nullptr, nullptr};
  std::vector<char> smoothedInOrder;  // per level minL..maxL
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
