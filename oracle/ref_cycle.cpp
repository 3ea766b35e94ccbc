// One V(pre, post) multigrid cycle of the reference's P1 path in the reference's own
// per-primitive memory layout, driven through the reference's generated kernels (compiled from
// the reference sources into oracle/_ref/libhyteg_ref.so by oracle/Makefile).
//
// TIMED CPU BASELINE ONLY: bench.py's reference arm and cpu_baseline time ref_cycle_run; the
// product never links it.
//
// The cycle follows GeometricMultigridSolver::solveRecursively
// (solvers/GeometricMultigridSolver.hpp:136-235) on levels L .. 1 of a macro-mesh:
//   pre-smoothing   `pre` x smooth_sor (P1Operator.hpp:350-420): faces, then cells (the phase
//                   order V -> E -> F -> C; the vertex and edge phases are not run, see below),
//                   each phase after the halo exchange the reference performs before it
//                   (face -> cell closure copies: communicate_directly_vertexdof_face_to_cell,
//                   VertexDoFPackInfo.hpp:391-428; cell -> face ghost layers:
//                   communicate_directly_vertexdof_cell_to_face, :505-563);
//   residual        A x on faces (apply_3D_macroface_one_sided_vertexdof_to_vertexdof_{replace,add},
//                   P1ConstantOperator.cpp:202-288) and cells
//                   (apply_3D_macrocell_vertexdof_to_vertexdof_replace), then r = b - A x
//                   (assign_3D_macrocell_vertexdof_2_rhs_functions; a plain loop on faces);
//   restriction     restrict_3D_macrocell_P1_pull_additive (P1toP1LinearRestriction.cpp:163-322)
//                   after the face -> cell copies, then the additive cell -> face exchange;
//   coarse level    x = 0 on level L - 1 (the coarse problem of level 0 has no cell or face DoFs);
//   prolongation    prolongate_3D_macrocell_P1_push_additive (P1toP1LinearProlongation.cpp:189-397)
//                   and the additive cell -> face exchange;
//   post-smoothing  `post` x smooth_sor.
// Dirichlet faces (one neighbour cell) are neither smoothed nor applied, as with flag
// Inner | NeumannBoundary. Not run: the vertex and edge phases (restated loops in the
// reference, P1Operator.hpp:1040-1104, 1348-1417; 0.005 % of the level-8 cube's inner DoFs) and
// the CG on level 0 (the vertex and edge values act as fixed boundary values). The additive
// cell -> face exchange of the reference's BufferedCommunicator (VertexDoFAdditivePackInfo) is a
// restated loop.
// Macro-primitives of one kind run in parallel on the host threads (a persistent pool), as MPI
// ranks of the reference each own some of them.
#include <algorithm>
#include <array>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "hyteg/gridtransferoperators/generatedKernels/prolongate_3D_macrocell_P1_push_additive.hpp"
#include "hyteg/gridtransferoperators/generatedKernels/restrict_3D_macrocell_P1_pull_additive.hpp"
#include "hyteg/p1functionspace/generatedKernels/apply_3D_macrocell_vertexdof_to_vertexdof_replace.hpp"
#include "hyteg/p1functionspace/generatedKernels/apply_3D_macroface_one_sided_vertexdof_to_vertexdof_add.hpp"
#include "hyteg/p1functionspace/generatedKernels/apply_3D_macroface_one_sided_vertexdof_to_vertexdof_replace.hpp"
#include "hyteg/p1functionspace/generatedKernels/assign_3D_macrocell_vertexdof_2_rhsfunctions.hpp"
#include "hyteg/p1functionspace/generatedKernels/communicate_directly_vertexdof_cell_to_face.hpp"
#include "hyteg/p1functionspace/generatedKernels/communicate_directly_vertexdof_face_to_cell.hpp"
#include "hyteg/p1functionspace/generatedKernels/sor_3D_macrocell_P1.hpp"
#include "hyteg/p1functionspace/generatedKernels/sor_3D_macroface_P1.hpp"

using hyteg::indexing::IndexIncrement;
typedef std::map<IndexIncrement, double> StencilMap;

namespace {

// Persistent worker pool: parallelFor(n, fn) runs fn(0 .. n-1), items taken from a shared counter
// by the workers and the calling thread, and returns when all are done.
class Pool {
 public:
  explicit Pool(int threads) {
    for (int t = 1; t < threads; ++t) workers_.emplace_back([this] { loop(); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> g(m_);
      stop_ = true;
      ++gen_;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }
  int size() const { return (int)workers_.size() + 1; }
  void parallelFor(int n, const std::function<void(int)>& fn) {
    if (n <= 0) return;
    {
      std::lock_guard<std::mutex> g(m_);
      fn_ = &fn;
      n_ = n;
      next_.store(0);
      done_ = 0;
      active_ = (int)workers_.size();
      ++gen_;
    }
    cv_.notify_all();
    run();
    std::unique_lock<std::mutex> lk(m_);
    doneCv_.wait(lk, [this] { return active_ == 0; });
    fn_ = nullptr;
  }

 private:
  void run() {
    for (int i = next_.fetch_add(1); i < n_; i = next_.fetch_add(1)) (*fn_)(i);
  }
  void loop() {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
        if (stop_) return;
      }
      run();
      {
        std::lock_guard<std::mutex> g(m_);
        if (--active_ == 0) doneCv_.notify_one();
      }
    }
  }
  std::vector<std::thread> workers_;
  std::mutex m_;
  std::condition_variable cv_, doneCv_;
  const std::function<void(int)>* fn_ = nullptr;
  std::atomic<int> next_{0};
  int n_ = 0, done_ = 0, active_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
};

// 15 increments in the order C E W N S NW SE TC TW TS TSE BC BE BN BNW (cell-local frame; on a
// face the same increments in the face-local frame, z = 1 pointing into the neighbour cell).
const int kOff[15][3] = {{0, 0, 0},  {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0},
                         {-1, 1, 0}, {1, -1, 0}, {0, 0, 1},  {-1, 0, 1}, {0, -1, 1},
                         {1, -1, 1}, {0, 0, -1}, {1, 0, -1}, {0, 1, -1}, {-1, 1, -1}};

int64_t tet(int64_t w) { return w * (w + 1) * (w + 2) / 6; }
int64_t tri(int64_t w) { return w * (w + 1) / 2; }

StencilMap toMap(const double* w, double scale, bool faceSide) {
  StencilMap m;
  for (int k = 0; k < 15; ++k) {
    if (faceSide && kOff[k][2] < 0) continue;  // a face's one-sided stencil stays inside the cell
    m[IndexIncrement(kOff[k][0], kOff[k][1], kOff[k][2])] = w[k] * scale;
  }
  return m;
}

struct FaceInfo {
  int ncells;
  int cell[2];
  int lid[2][3];
};

struct Level {
  std::vector<std::vector<double>> cx, cb, cr;  // [cell]
  std::vector<std::vector<double>> fx, fb, fr;  // [face]: tri(w) + ncells * tri(w - 1)
  std::vector<StencilMap> cellMap;              // [cell]
  std::vector<std::array<StencilMap, 2>> faceMap;  // [face][side]
};

}  // namespace

struct RefCycle {
  int L = 0, nc = 0, nf = 0, pre = 3, post = 3;
  std::vector<FaceInfo> faces;
  std::vector<std::array<double, 14>> counts;  // per cell: edges 6, faces 4, vertices 4
  std::vector<Level> lv;                       // levels 0 .. L
  std::vector<std::pair<int, int>> pairs;      // (face, side) of every face-cell incidence
  Pool* pool = nullptr;
  ~RefCycle() { delete pool; }
};

namespace {

void faceToCell(RefCycle& R, int l, bool useX) {
  Level& v = R.lv[l];
  const int np = (int)R.pairs.size();
  R.pool->parallelFor(np, [&](int i) {
    const int f = R.pairs[i].first, k = R.pairs[i].second;
    const FaceInfo& fi = R.faces[f];
    const int c = fi.cell[k];
    double* cell = useX ? v.cx[c].data() : v.cr[c].data();
    const double* face = useX ? v.fx[f].data() : v.fr[f].data();
    hyteg::vertexdof::comm::generated::communicate_directly_vertexdof_face_to_cell(cell, face, l, fi.lid[k][0],
                                                                                   fi.lid[k][1], fi.lid[k][2]);
  });
}

void cellToFace(RefCycle& R, int l) {
  Level& v = R.lv[l];
  const int64_t w = (1 << l) + 1;
  const int np = (int)R.pairs.size();
  R.pool->parallelFor(np, [&](int i) {
    const int f = R.pairs[i].first, k = R.pairs[i].second;
    const FaceInfo& fi = R.faces[f];
    double* gl = v.fx[f].data() + tri(w) + k * tri(w - 1);
    hyteg::vertexdof::comm::generated::communicate_directly_vertexdof_cell_to_face(v.cx[fi.cell[k]].data(), gl, l,
                                                                                   fi.lid[k][0], fi.lid[k][1],
                                                                                   fi.lid[k][2]);
  });
}

// Additive cell -> face exchange on level l (communicateAdditively<Cell, Face>,
// VertexDoFAdditivePackInfo), restated: the cells' closure values at the face's interior points,
// found through the cells' local IDs of the face's vertices.
//   restriction (intoX = false): b_face = sum over the neighbour cells of their closure values
//                                (each cell holds its 1/#cells share of the restricted value);
//   prolongation (intoX = true): x_face += sum over the cells of (closure value - x_face), each
//                                cell having added its 1/#cells share of the interpolated
//                                correction to a closure that held x_face.
void cellToFaceAdditive(RefCycle& R, int l, bool intoX) {
  Level& v = R.lv[l];
  const int64_t w = (1 << l) + 1;
  if (w < 4) return;
  R.pool->parallelFor(R.nf, [&](int f) {
    const FaceInfo& fi = R.faces[f];
    if (fi.ncells < 2) return;
    double* dst = intoX ? v.fx[f].data() : v.fb[f].data();
    for (int64_t y = 1; y < w - 2; ++y)
      for (int64_t x = 1; x + y < w - 1; ++x) {
        const int64_t fidx = y * (w + 1) - y * (y + 1) / 2 + x;
        double acc = intoX ? dst[fidx] : 0.0;
        for (int k = 0; k < fi.ncells; ++k) {
          int64_t bw[4] = {0, 0, 0, 0};  // barycentric weights of the cell's local vertices
          bw[fi.lid[k][0]] = w - 1 - x - y;
          bw[fi.lid[k][1]] = x;
          bw[fi.lid[k][2]] = y;
          const int64_t W = w - bw[3];
          const int64_t cidx = tet(w) - tet(W) + bw[2] * (W + 1) - bw[2] * (bw[2] + 1) / 2 + bw[1];
          const double cv = intoX ? v.cx[fi.cell[k]][cidx] : v.cb[fi.cell[k]][cidx];
          acc += intoX ? cv - dst[fidx] : cv;
        }
        dst[fidx] = acc;
      }
  });
}

void smooth(RefCycle& R, int l, double relax) {
  Level& v = R.lv[l];
  const int64_t w = (1 << l) + 1;
  // face phase (after the edge -> face refresh the reference does first)
  R.pool->parallelFor(R.nf, [&](int f) {
    const FaceInfo& fi = R.faces[f];
    if (fi.ncells < 2) return;
    double* d = v.fx[f].data();
    double* gl0 = d + tri(w);
    double* gl1 = gl0 + tri(w - 1);
    const int* a = fi.lid[0];
    const int* b = fi.lid[1];
    // the reference passes the neighbour with the lexicographically smaller local IDs first
    // (P1ConstantOperator.cpp:415-470)
    const bool swap = a[0] > b[0] || (a[0] == b[0] && (a[1] > b[1] || (a[1] == b[1] && a[2] > b[2])));
    if (swap)
      hyteg::vertexdof::macroface::generated::sor_3D_macroface_P1(d, gl1, gl0, v.fb[f].data(), l, b[0], b[1], b[2], a[0],
                                                                  a[1], a[2], relax, v.faceMap[f][1], v.faceMap[f][0]);
    else
      hyteg::vertexdof::macroface::generated::sor_3D_macroface_P1(d, gl0, gl1, v.fb[f].data(), l, a[0], a[1], a[2], b[0],
                                                                  b[1], b[2], relax, v.faceMap[f][0], v.faceMap[f][1]);
  });
  faceToCell(R, l, true);  // face -> cell before the cell phase
  R.pool->parallelFor(R.nc, [&](int c) {
    hyteg::vertexdof::macrocell::generated::sor_3D_macrocell_P1(v.cx[c].data(), v.cb[c].data(), l, v.cellMap[c], relax);
  });
  cellToFace(R, l);  // the cells' new values into the faces' ghost layers
}

void residual(RefCycle& R, int l) {
  Level& v = R.lv[l];
  const int64_t w = (1 << l) + 1;
  R.pool->parallelFor(R.nf, [&](int f) {
    const FaceInfo& fi = R.faces[f];
    if (fi.ncells < 2) return;
    double* x = v.fx[f].data();
    double* r = v.fr[f].data();
    for (int k = 0; k < 2; ++k) {
      const double* gl = x + tri(w) + k * tri(w - 1);
      if (k == 0)
        hyteg::vertexdof::macroface::generated::apply_3D_macroface_one_sided_vertexdof_to_vertexdof_replace(
            r, x, gl, l, fi.lid[k][0], fi.lid[k][1], fi.lid[k][2], v.faceMap[f][k]);
      else
        hyteg::vertexdof::macroface::generated::apply_3D_macroface_one_sided_vertexdof_to_vertexdof_add(
            r, x, gl, l, fi.lid[k][0], fi.lid[k][1], fi.lid[k][2], v.faceMap[f][k]);
    }
    const double* b = v.fb[f].data();
    for (int64_t y = 1; y < w - 2; ++y)
      for (int64_t x0 = 1; x0 + y < w - 1; ++x0) {
        const int64_t i = y * (w + 1) - y * (y + 1) / 2 + x0;
        r[i] = b[i] - r[i];
      }
  });
  R.pool->parallelFor(R.nc, [&](int c) {
    hyteg::vertexdof::macrocell::generated::apply_3D_macrocell_vertexdof_to_vertexdof_replace(v.cr[c].data(),
                                                                                             v.cx[c].data(), l,
                                                                                             v.cellMap[c]);
    hyteg::vertexdof::macrocell::generated::assign_3D_macrocell_vertexdof_2_rhs_functions(v.cr[c].data(), v.cb[c].data(),
                                                                                          v.cr[c].data(), 1.0, -1.0, l);
  });
}

void restrictTo(RefCycle& R, int l) {  // r on l -> b on l - 1
  faceToCell(R, l, false);
  Level& f = R.lv[l];
  Level& c = R.lv[l - 1];
  R.pool->parallelFor(R.nc, [&](int k) {
    const double* n = R.counts[k].data();
    hyteg::vertexdof::macrocell::generated::restrict_3D_macrocell_P1_pull_additive(
        c.cb[k].data(), f.cr[k].data(), l - 1, n[0], n[1], n[2], n[3], n[4], n[5], n[6], n[7], n[8], n[9], n[10], n[11],
        n[12], n[13]);
  });
  cellToFaceAdditive(R, l - 1, false);
}

void prolongateAdd(RefCycle& R, int l) {  // x on l - 1 added into x on l
  Level& f = R.lv[l];
  Level& c = R.lv[l - 1];
  R.pool->parallelFor(R.nc, [&](int k) {
    const double* n = R.counts[k].data();
    hyteg::vertexdof::macrocell::generated::prolongate_3D_macrocell_P1_push_additive(
        c.cx[k].data(), f.cx[k].data(), l - 1, n[0], n[1], n[2], n[3], n[4], n[5], n[6], n[7], n[8], n[9], n[10], n[11],
        n[12], n[13]);
  });
  cellToFaceAdditive(R, l, true);
}

void zero(Level& v) {
  for (auto& a : v.cx) std::fill(a.begin(), a.end(), 0.0);
  for (auto& a : v.fx) std::fill(a.begin(), a.end(), 0.0);
}

void cycle(RefCycle& R, int l, double relax) {
  if (l == 0) return;  // level 0 of the cube has no cell or face DoFs: its CG is not run
  for (int s = 0; s < R.pre; ++s) smooth(R, l, relax);
  residual(R, l);
  restrictTo(R, l);
  zero(R.lv[l - 1]);
  cycle(R, l - 1, relax);
  prolongateAdd(R, l);
  for (int s = 0; s < R.post; ++s) smooth(R, l, relax);
}

}  // namespace

extern "C" {

// Creates the hierarchy of levels 0 .. L of a macro-mesh with nc cells and nf faces.
//   cellW2   [nc][15]  each cell's stencil on level 2 (C E W N S NW SE TC TW TS TSE BC BE BN BNW);
//                      level l uses cellW2 * 2^(2 - l) (the constant stencils of P1 Laplace halve
//                      from one level to the next finer one)
//   counts   [nc][14]  neighbour-cell counts of each cell's 6 edges, 4 faces, 4 vertices
//   faceNc   [nf]      neighbour cells of each face (1: boundary, not smoothed)
//   faceCell [nf][2]   those cells; faceLid [nf][2][3] their cell-local IDs of the face's vertices
//   faceW2   [nf][2][15] each side's one-sided face stencil on level 2, face-local increments
//   seed               x and b are filled from a fixed sequence with values in [-1, 1)
RefCycle* ref_cycle_create(int L, int nc, int nf, const double* cellW2, const double* counts, const int* faceNc,
                           const int* faceCell, const int* faceLid, const double* faceW2, int pre, int post,
                           unsigned seed) {
  RefCycle* R = new RefCycle();
  R->L = L;
  R->nc = nc;
  R->nf = nf;
  R->pre = pre;
  R->post = post;
  R->faces.resize(nf);
  for (int f = 0; f < nf; ++f) {
    FaceInfo& fi = R->faces[f];
    fi.ncells = faceNc[f];
    for (int k = 0; k < 2; ++k) {
      fi.cell[k] = faceCell[2 * f + k];
      for (int j = 0; j < 3; ++j) fi.lid[k][j] = faceLid[6 * f + 3 * k + j];
    }
    for (int k = 0; k < fi.ncells; ++k) R->pairs.push_back({f, k});
  }
  R->counts.resize(nc);
  for (int c = 0; c < nc; ++c)
    for (int j = 0; j < 14; ++j) R->counts[c][j] = counts[14 * c + j];
  R->lv.resize(L + 1);
  uint64_t state = 0x9E3779B97F4A7C15ull ^ seed;
  auto next = [&state]() {  // xorshift64*, uniform in [-1, 1)
    state ^= state >> 12;
    state ^= state << 25;
    state ^= state >> 27;
    return double((state * 2685821657736338717ull) >> 11) * (2.0 / 9007199254740992.0) - 1.0;
  };
  for (int l = 0; l <= L; ++l) {
    Level& v = R->lv[l];
    const int64_t w = (1 << l) + 1;
    const double scale = l <= 2 ? double(1 << (2 - l)) : 1.0 / double(1 << (l - 2));
    v.cx.assign(nc, std::vector<double>(tet(w), 0.0));
    v.cb = v.cx;
    v.cr = v.cx;
    v.fx.resize(nf);
    v.fb.resize(nf);
    v.fr.resize(nf);
    for (int f = 0; f < nf; ++f) {
      const size_t n = tri(w) + R->faces[f].ncells * tri(w - 1);
      v.fx[f].assign(n, 0.0);
      v.fb[f].assign(n, 0.0);
      v.fr[f].assign(n, 0.0);
    }
    if (l == L) {
      for (auto& a : v.cx)
        for (auto& e : a) e = next();
      for (auto& a : v.cb)
        for (auto& e : a) e = next();
      for (auto& a : v.fx)
        for (auto& e : a) e = next();
      for (auto& a : v.fb)
        for (auto& e : a) e = next();
    }
    for (int c = 0; c < nc; ++c) v.cellMap.push_back(toMap(cellW2 + 15 * c, scale, false));
    v.faceMap.resize(nf);
    for (int f = 0; f < nf; ++f)
      for (int k = 0; k < R->faces[f].ncells; ++k) v.faceMap[f][k] = toMap(faceW2 + 30 * f + 15 * k, scale, true);
  }
  return R;
}

void ref_cycle_destroy(RefCycle* R) { delete R; }

// One cycle on the finest level with `threads` host threads. Returns the number of threads used.
int ref_cycle_run(RefCycle* R, int threads, double relax) {
  if (threads < 1) threads = 1;
  if (!R->pool || R->pool->size() != threads) {
    delete R->pool;
    R->pool = new Pool(threads);
  }
  cycle(*R, R->L, relax);
  return R->pool->size();
}

// Sum of the finest level's x over the cells (keeps the work observable).
double ref_cycle_checksum(RefCycle* R) {
  double s = 0;
  for (auto& a : R->lv[R->L].cx)
    for (double e : a) s += e;
  return s;
}

}  // extern "C"
