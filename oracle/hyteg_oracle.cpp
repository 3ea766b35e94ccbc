// CPU oracle for the B200 HyTeG hot path. TEST INFRASTRUCTURE ONLY: imported by tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker; never part of
// the product path.
//
// It restates the reference algorithm in a different formulation from the product: one
// global vector per level indexed by micro-vertex (exact barycentric identity), an
// explicitly assembled sparse stiffness matrix, and the reference's update order for SOR.
// Nothing here uses the per-primitive arrays, halo tables or stencil tables of the product.
//
// Reference files followed (paths within wagnandr/hyteg):
//   mesh / IDs     src/hyteg/mesh/MeshGenCuboid.cpp:32-171, src/hyteg/mesh/MeshInfo.cpp:37-72,
//                  src/hyteg/primitivestorage/SetupPrimitiveStorage.cpp:37-345, 850-911
//   refinement     src/hyteg/celldofspace/CellDoFIndexing.hpp:128-175 (six micro-cell types)
//   operator       src/hyteg/p1functionspace/P1Elements.hpp:430-496 (stencil = sum of element
//                  matrix rows), src/hyteg/forms/form_fenics_generated/p1_tet_diffusion.h
//   apply          src/hyteg/p1functionspace/P1Operator.hpp:197-325 (Dirichlet rows untouched)
//   lexicographic SOR  src/hyteg/p1functionspace/P1Operator.hpp:350-420, 1348-1417,
//                  generatedKernels/sor_3D_macrocell_P1.cpp:32-78, sor_3D_macroface_P1*.cpp
//   transfers      src/hyteg/gridtransferoperators/P1toP1LinearRestriction.cpp:163-322,
//                  P1toP1LinearProlongation.cpp:189-397 (restriction = prolongation transposed)
//   solvers        src/hyteg/solvers/CGSolver.hpp:69-150,
//                  src/hyteg/solvers/GeometricMultigridSolver.hpp:136-235
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <set>
#include <unordered_map>
#include <vector>

namespace {

// A micro-vertex is identified exactly by its non-zero barycentric weights with respect to
// the macro-vertices: (vertex, weight) pairs sorted by vertex, padded with (-1, 0).
typedef std::array<int64_t, 8> Key;

struct KeyHash {
  size_t operator()(const Key& k) const {
    size_t h = 1469598103934665603ULL;
    for (int64_t v : k) h = (h ^ (size_t)v) * 1099511628211ULL;
    return h;
  }
};

const int kMicro[6][4][3] = {
    {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, {{1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {1, 0, 1}},
    {{1, 0, 0}, {0, 1, 0}, {1, 0, 1}, {0, 0, 1}}, {{1, 1, 0}, {1, 1, 1}, {0, 1, 1}, {1, 0, 1}},
    {{1, 0, 1}, {0, 1, 1}, {0, 0, 1}, {0, 1, 0}}, {{0, 1, 0}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}},
};
const int kMicroWidthReduction[6] = {0, 1, 1, 2, 1, 1};

// P1 element matrices: gradients of the barycentric coordinates from the inverse Jacobian.
void laplaceElement(const double p[4][3], double K[4][4]) {
  double a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) a[i][d] = p[i + 1][d] - p[0][d];  // rows: edge vectors
  // gradients of lambda_1..3 are the rows of inverse(transpose(a)) ... use cross products
  double c[3][3];
  auto cross = [](const double* u, const double* v, double* r) {
    r[0] = u[1] * v[2] - u[2] * v[1];
    r[1] = u[2] * v[0] - u[0] * v[2];
    r[2] = u[0] * v[1] - u[1] * v[0];
  };
  cross(a[1], a[2], c[0]);
  cross(a[2], a[0], c[1]);
  cross(a[0], a[1], c[2]);
  const double det = a[0][0] * c[0][0] + a[0][1] * c[0][1] + a[0][2] * c[0][2];
  double g[4][3];
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) g[i + 1][d] = c[i][d] / det;
  for (int d = 0; d < 3; ++d) g[0][d] = -(g[1][d] + g[2][d] + g[3][d]);
  const double vol = std::fabs(det) / 6.0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) K[i][j] = vol * (g[i][0] * g[j][0] + g[i][1] * g[j][1] + g[i][2] * g[j][2]);
}

double tetVolume(const double p[4][3]) {
  double a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) a[i][d] = p[i + 1][d] - p[0][d];
  const double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                     a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
  return std::fabs(det) / 6.0;
}

void massElement(const double p[4][3], double K[4][4]) {
  double a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) a[i][d] = p[i + 1][d] - p[0][d];
  const double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                     a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
  const double vol = std::fabs(det) / 6.0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) K[i][j] = vol * (i == j ? 2.0 : 1.0) / 20.0;
}

// P2 Laplace element matrix of a tetrahedron (vertices p[4]). Local nodes: the vertices 0..3,
// then the edge midpoints (0,1),(0,2),(0,3),(1,2),(1,3),(2,3). Basis: lambda_a (2 lambda_a - 1)
// and 4 lambda_a lambda_b; the gradients are linear in lambda, so the 4-point degree-2 rule
// (points (a,b,b,b), a = (5 + 3 sqrt5)/20, b = (5 - sqrt5)/20) integrates the products exactly.
static const int kP2Edge[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};

void p2LaplaceElement(const double p[4][3], double K[10][10]) {
  double J[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) J[r][c] = p[c + 1][r] - p[0][r];
  const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                     J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  // rows of J^-1 are the gradients of lambda_1..3
  double inv[3][3];
  inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
  inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
  inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
  inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
  inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
  inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
  inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
  inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
  inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
  double G[4][3];
  for (int d = 0; d < 3; ++d) {
    G[1][d] = inv[0][d];
    G[2][d] = inv[1][d];
    G[3][d] = inv[2][d];
    G[0][d] = -(G[1][d] + G[2][d] + G[3][d]);
  }
  const double vol = std::fabs(det) / 6.0;
  const double qa = (5.0 + 3.0 * std::sqrt(5.0)) / 20.0, qb = (5.0 - std::sqrt(5.0)) / 20.0;
  for (int i = 0; i < 10; ++i)
    for (int j = 0; j < 10; ++j) K[i][j] = 0.0;
  for (int q = 0; q < 4; ++q) {
    double l[4] = {qb, qb, qb, qb};
    l[q] = qa;
    double g[10][3];
    for (int a = 0; a < 4; ++a)
      for (int d = 0; d < 3; ++d) g[a][d] = (4.0 * l[a] - 1.0) * G[a][d];
    for (int e = 0; e < 6; ++e) {
      const int a = kP2Edge[e][0], b = kP2Edge[e][1];
      for (int d = 0; d < 3; ++d) g[4 + e][d] = 4.0 * (l[b] * G[a][d] + l[a] * G[b][d]);
    }
    for (int i = 0; i < 10; ++i)
      for (int j = 0; j < 10; ++j) K[i][j] += 0.25 * vol * (g[i][0] * g[j][0] + g[i][1] * g[j][1] + g[i][2] * g[j][2]);
  }
}

// Taylor-Hood divergence element: D[k][i][j] = -int psi_i d(phi_j)/dx_k (P1 vertex i, P2 node j),
// by the 4-point degree-2 rule (the integrand is quadratic).
void p2p1DivElement(const double p[4][3], double D[3][4][10]) {
  double J[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) J[r][c] = p[c + 1][r] - p[0][r];
  const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                     J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  double inv[3][3];
  inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
  inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
  inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
  inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
  inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
  inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
  inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
  inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
  inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
  double G[4][3];
  for (int d = 0; d < 3; ++d) {
    G[1][d] = inv[0][d];
    G[2][d] = inv[1][d];
    G[3][d] = inv[2][d];
    G[0][d] = -(G[1][d] + G[2][d] + G[3][d]);
  }
  const double vol = std::fabs(det) / 6.0;
  const double qa = (5.0 + 3.0 * std::sqrt(5.0)) / 20.0, qb = (5.0 - std::sqrt(5.0)) / 20.0;
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 10; ++j) D[k][i][j] = 0.0;
  for (int q = 0; q < 4; ++q) {
    double l[4] = {qb, qb, qb, qb};
    l[q] = qa;
    double g[10][3];
    for (int a = 0; a < 4; ++a)
      for (int d = 0; d < 3; ++d) g[a][d] = (4.0 * l[a] - 1.0) * G[a][d];
    for (int e = 0; e < 6; ++e) {
      const int a = kP2Edge[e][0], b = kP2Edge[e][1];
      for (int d = 0; d < 3; ++d) g[4 + e][d] = 4.0 * (l[b] * G[a][d] + l[a] * G[b][d]);
    }
    for (int k = 0; k < 3; ++k)
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 10; ++j) D[k][i][j] -= 0.25 * vol * l[i] * g[j][k];
  }
}

struct Node {
  Key key;
  int kind, id;           // owner primitive (0 vertex, 1 edge, 2 face, 3 cell) and its ID
  int lx, ly, lz;         // coordinates in the owner's frame
  bool dirichlet;
  std::array<int, 4> sup; // owner vertex set (sorted, -1 padded)
};

struct Csr {
  std::vector<int64_t> ptr;
  std::vector<int64_t> col;
  std::vector<double> val;
};

struct LevelData {
  int64_t N = 1;
  Csr Div[3];                // Taylor-Hood divergence: rows nodes of this level, columns of the next
  bool haveDiv = false;
  Csr P2;                    // P2 Laplace of this level on the nodes of the next finer level
  bool haveP2 = false;
  Csr P2prol;                // P2 prolongation from this level to the next (rows: nodes of level + 2)
  bool haveP2prol = false;
  std::vector<Node> nodes;
  std::unordered_map<Key, int64_t, KeyHash> index;
  Csr A[3];                  // 0: diffusion (per-cell coefficient), 1: mass, 2: PSPG
  bool haveA[3] = {false, false, false};
  // prolongation from the next coarser level: per node up to two coarse nodes
  std::vector<std::array<int64_t, 2>> pc;
  std::vector<std::array<double, 2>> pw;
  std::vector<int64_t> lexOrder;    // reference SOR order
  std::vector<int64_t> mcOrder;     // multicolour order
  std::vector<int> lexPhase;        // kind of the owner (phase), aligned with the order vectors
};

struct Oracle {
  std::vector<std::array<double, 3>> vx;     // macro-vertex coordinates
  std::vector<std::array<int, 4>> cells;     // creation order (sorted by frame-ordered IDs)
  std::vector<double> k;
  std::map<std::array<int, 2>, int> edgeId;
  std::map<std::array<int, 3>, int> faceId;
  std::map<std::array<int, 4>, int> cellId;  // sorted vertex set -> cell
  std::set<std::array<int, 3>> boundaryFaces;
  std::vector<LevelData> lv;

  Key keyOf(int c, int64_t N, int64_t x, int64_t y, int64_t z) const {
    const auto& cv = cells[c];
    const int64_t b[4] = {N - x - y - z, x, y, z};
    std::array<std::pair<int64_t, int64_t>, 4> p;
    int n = 0;
    for (int i = 0; i < 4; ++i)
      if (b[i] > 0) p[n++] = {cv[i], b[i]};
    std::sort(p.begin(), p.begin() + n);
    Key k;
    for (int i = 0; i < 4; ++i) {
      k[2 * i] = i < n ? p[i].first : -1;
      k[2 * i + 1] = i < n ? p[i].second : 0;
    }
    return k;
  }
  void coordOf(const Key& k, int64_t N, double p[3]) const {
    for (int d = 0; d < 3; ++d) {
      double s = 0.0;
      for (int i = 0; i < 4; ++i)
        if (k[2 * i] >= 0) s += (double)k[2 * i + 1] * vx[k[2 * i]][d];
      p[d] = s / (double)N;
    }
  }
};

bool supportOnBoundary(const Oracle& o, const std::array<int, 4>& sup) {
  // a DoF is Dirichlet iff its owner primitive lies in the closure of a boundary face
  std::vector<int> s;
  for (int v : sup)
    if (v >= 0) s.push_back(v);
  for (const auto& f : o.boundaryFaces) {
    bool sub = true;
    for (int v : s)
      if (v != f[0] && v != f[1] && v != f[2]) sub = false;
    if (sub) return true;
  }
  return false;
}

void buildLevel(Oracle& o, int L) {
  LevelData& d = o.lv[L];
  d.N = int64_t(1) << L;
  const int64_t N = d.N;
  for (size_t c = 0; c < o.cells.size(); ++c) {
    const auto& cv = o.cells[c];
    for (int64_t z = 0; z <= N; ++z)
      for (int64_t y = 0; y + z <= N; ++y)
        for (int64_t x = 0; x + y + z <= N; ++x) {
          const Key key = o.keyOf((int)c, N, x, y, z);
          if (d.index.count(key)) continue;
          const int64_t b[4] = {N - x - y - z, x, y, z};
          std::vector<std::pair<int, int64_t>> sup;
          for (int i = 0; i < 4; ++i)
            if (b[i] > 0) sup.push_back({cv[i], b[i]});
          std::sort(sup.begin(), sup.end());
          Node nd;
          nd.key = key;
          nd.sup = {-1, -1, -1, -1};
          for (size_t i = 0; i < sup.size(); ++i) nd.sup[i] = sup[i].first;
          nd.kind = (int)sup.size() - 1;
          nd.lx = nd.ly = nd.lz = 0;
          auto bOf = [&](int v) {
            for (auto& s : sup)
              if (s.first == v) return s.second;
            return (int64_t)0;
          };
          if (nd.kind == 0) {
            nd.id = sup[0].first;
          } else if (nd.kind == 1) {
            nd.id = o.edgeId.at({sup[0].first, sup[1].first});
            nd.lx = (int)bOf(sup[1].first);
          } else if (nd.kind == 2) {
            nd.id = o.faceId.at({sup[0].first, sup[1].first, sup[2].first});
            nd.lx = (int)bOf(sup[1].first);
            nd.ly = (int)bOf(sup[2].first);
          } else {
            nd.id = (int)c;
            nd.lx = (int)x;
            nd.ly = (int)y;
            nd.lz = (int)z;
          }
          nd.dirichlet = supportOnBoundary(o, nd.sup);
          d.index[key] = (int64_t)d.nodes.size();
          d.nodes.push_back(nd);
        }
  }
  // reference lexicographic order: vertices, edges, faces, cells by ID; inside a primitive
  // x fastest, then y, then z (P1Operator.hpp:350-420 and the generated SOR kernels)
  std::vector<int64_t> ord(d.nodes.size());
  for (size_t i = 0; i < ord.size(); ++i) ord[i] = (int64_t)i;
  auto lexKey = [&](int64_t i) {
    const Node& n = d.nodes[i];
    return std::array<int64_t, 5>{n.kind, n.id, n.lz, n.ly, n.lx};
  };
  std::sort(ord.begin(), ord.end(), [&](int64_t a, int64_t b) { return lexKey(a) < lexKey(b); });
  d.lexOrder = ord;
  // multicolour order: phases by kind; colour classes (edge: x mod 2, face: (x+2y) mod 3,
  // cell: (x+2y+3z) mod 4); inside a class the order is irrelevant
  auto colour = [&](const Node& n) {
    if (n.kind == 1) return n.lx % 2;
    if (n.kind == 2) return (n.lx + 2 * n.ly) % 3;
    if (n.kind == 3) return (n.lx + 2 * n.ly + 3 * n.lz) % 4;
    return 0;
  };
  auto mcKey = [&](int64_t i) {
    const Node& n = d.nodes[i];
    return std::array<int64_t, 6>{n.kind, colour(n), n.id, n.lz, n.ly, n.lx};
  };
  std::vector<int64_t> mc = ord;
  std::sort(mc.begin(), mc.end(), [&](int64_t a, int64_t b) { return mcKey(a) < mcKey(b); });
  d.mcOrder = mc;
}

void buildProlongation(Oracle& o, int Lf) {
  LevelData& f = o.lv[Lf];
  const LevelData& c = o.lv[Lf - 1];
  f.pc.assign(f.nodes.size(), {-1, -1});
  f.pw.assign(f.nodes.size(), {0.0, 0.0});
  std::vector<char> done(f.nodes.size(), 0);
  const int64_t N = f.N;
  for (size_t ci = 0; ci < o.cells.size(); ++ci)
    for (int64_t z = 0; z <= N; ++z)
      for (int64_t y = 0; y + z <= N; ++y)
        for (int64_t x = 0; x + y + z <= N; ++x) {
          const int64_t fi = f.index.at(o.keyOf((int)ci, N, x, y, z));
          if (done[fi]) continue;
          done[fi] = 1;
          const int code = int(x & 1) | (int(y & 1) << 1) | (int(z & 1) << 2);
          if (code == 0) {
            f.pc[fi] = {c.index.at(o.keyOf((int)ci, N / 2, x / 2, y / 2, z / 2)), -1};
            f.pw[fi] = {1.0, 0.0};
            continue;
          }
          // the coarse micro-edge bisected by this fine point, in cell-local directions
          static const int dir[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {-1, 1, 0},
                                        {0, 0, 1}, {-1, 0, 1}, {0, -1, 1}, {-1, 1, -1}};
          const int* dd = dir[code];
          const int64_t ax = (x - dd[0]) / 2, ay = (y - dd[1]) / 2, az = (z - dd[2]) / 2;
          f.pc[fi] = {c.index.at(o.keyOf((int)ci, N / 2, ax, ay, az)),
                      c.index.at(o.keyOf((int)ci, N / 2, ax + dd[0], ay + dd[1], az + dd[2]))};
          f.pw[fi] = {0.5, 0.5};
        }
}

void buildMatrix(Oracle& o, int L, int form) {
  LevelData& d = o.lv[L];
  const int64_t N = d.N;
  std::vector<std::map<int64_t, double>> rows(d.nodes.size());
  for (size_t ci = 0; ci < o.cells.size(); ++ci) {
    for (int t = 0; t < 6; ++t) {
      const int64_t width = N - kMicroWidthReduction[t];
      if (width <= 0) continue;
      for (int64_t z = 0; z < width; ++z)
        for (int64_t y = 0; y + z < width; ++y)
          for (int64_t x = 0; x + y + z < width; ++x) {
            int64_t id[4];
            double p[4][3];
            for (int m = 0; m < 4; ++m) {
              const Key k = o.keyOf((int)ci, N, x + kMicro[t][m][0], y + kMicro[t][m][1], z + kMicro[t][m][2]);
              id[m] = d.index.at(k);
              o.coordOf(k, N, p[m]);
            }
            double K[4][4];
            if (form == 0) {
              laplaceElement(p, K);
              for (auto& r : K)
                for (double& v : r) v *= o.k[ci];
            } else if (form == 2) {
              // PSPG (data/operators/form_pspg_tet.ufl): -tau grad p . grad q, tau = |T|^(2/3) / 12
              laplaceElement(p, K);
              const double tau = std::pow(tetVolume(p), 2.0 / 3.0) / 12.0;
              for (auto& r : K)
                for (double& v : r) v *= -tau;
            } else {
              massElement(p, K);
            }
            for (int a = 0; a < 4; ++a)
              for (int b = 0; b < 4; ++b) rows[id[a]][id[b]] += K[a][b];
          }
    }
  }
  Csr& A = d.A[form];
  A.ptr.assign(1, 0);
  for (auto& r : rows) {
    for (auto& kv : r) {
      A.col.push_back(kv.first);
      A.val.push_back(kv.second);
    }
    A.ptr.push_back((int64_t)A.col.size());
  }
  d.haveA[form] = true;
}

// P2 Laplace of level L assembled over the level-L micro-tetrahedra, on the node set of level
// L + 1 (micro-vertices of level L at even coordinates, micro-edge midpoints at the others).
void buildP2Matrix(Oracle& o, int L) {
  LevelData& d = o.lv[L];
  const LevelData& f = o.lv[L + 1];
  const int64_t N = d.N;
  std::vector<std::map<int64_t, double>> rows(f.nodes.size());
  for (size_t ci = 0; ci < o.cells.size(); ++ci)
    for (int t = 0; t < 6; ++t) {
      const int64_t width = N - kMicroWidthReduction[t];
      for (int64_t z = 0; z < width; ++z)
        for (int64_t y = 0; y + z < width; ++y)
          for (int64_t x = 0; x + y + z < width; ++x) {
            int64_t v[4][3];
            double p[4][3];
            for (int m = 0; m < 4; ++m) {
              v[m][0] = x + kMicro[t][m][0];
              v[m][1] = y + kMicro[t][m][1];
              v[m][2] = z + kMicro[t][m][2];
              o.coordOf(o.keyOf((int)ci, N, v[m][0], v[m][1], v[m][2]), N, p[m]);
            }
            int64_t id[10];
            for (int m = 0; m < 4; ++m) id[m] = f.index.at(o.keyOf((int)ci, 2 * N, 2 * v[m][0], 2 * v[m][1], 2 * v[m][2]));
            for (int e = 0; e < 6; ++e) {
              const int a = kP2Edge[e][0], b = kP2Edge[e][1];
              id[4 + e] = f.index.at(
                  o.keyOf((int)ci, 2 * N, v[a][0] + v[b][0], v[a][1] + v[b][1], v[a][2] + v[b][2]));
            }
            double K[10][10];
            p2LaplaceElement(p, K);
            for (int a = 0; a < 10; ++a)
              for (int b = 0; b < 10; ++b) rows[id[a]][id[b]] += o.k[ci] * K[a][b];
          }
    }
  Csr& A = d.P2;
  A.ptr.assign(1, 0);
  for (auto& r : rows) {
    for (auto& kv : r) {
      A.col.push_back(kv.first);
      A.val.push_back(kv.second);
    }
    A.ptr.push_back((int64_t)A.col.size());
  }
  d.haveP2 = true;
}

const Csr& matrix(Oracle& o, int L, int form) {
  if (!o.lv[L].haveA[form]) buildMatrix(o, L, form);
  return o.lv[L].A[form];
}

bool inClosure(const Node& inner, const Node& outer) {
  // is the owner of `inner` a sub-primitive of (or equal to) the owner of `outer`?
  for (int v : inner.sup) {
    if (v < 0) continue;
    bool found = false;
    for (int w : outer.sup)
      if (w == v) found = true;
    if (!found) return false;
  }
  return true;
}

void sorSweep(Oracle& o, int L, double* u, const double* f, double omega, bool multicolour, bool backwards,
              int kindMask = 15) {
  LevelData& d = o.lv[L];
  const Csr& A = matrix(o, L, 0);
  const std::vector<double> start(u, u + d.nodes.size());
  const std::vector<int64_t>& ord = multicolour ? d.mcOrder : d.lexOrder;
  const int64_t n = (int64_t)ord.size();
  for (int64_t t = 0; t < n; ++t) {
    const int64_t i = ord[backwards ? n - 1 - t : t];
    const Node& ni = d.nodes[i];
    if (ni.dirichlet || !(kindMask & (1 << ni.kind))) continue;
    double diag = 0.0, s = f[i];
    for (int64_t e = A.ptr[i]; e < A.ptr[i + 1]; ++e) {
      const int64_t j = A.col[e];
      if (j == i) {
        diag = A.val[e];
        continue;
      }
      const Node& nj = d.nodes[j];
      // Forward: values in the primitive's own closure are current (refreshed V->E->F->C
      // between the phases); values reaching it through ghost layers keep the value of the
      // sweep's initial halo exchange. Backward (C->F->E->V): the reference refreshes a
      // primitive's ghosts from the higher-dimensional primitives that contain it, so only
      // their values are current; the multicolour smoother refreshes every ghost slot from its
      // owner, so every value owned by a higher-dimensional primitive is current.
      bool current = inClosure(nj, ni);
      if (backwards) current = current || (multicolour ? nj.kind > ni.kind : inClosure(ni, nj));
      s -= A.val[e] * (current ? u[j] : start[j]);
    }
    u[i] = (1.0 - omega) * u[i] + (s * omega) / diag;
  }
}

}  // namespace

extern "C" {

// coords: 3 per vertex; tets: 4 per cell in frame order (any order of cells); k: per-cell
// coefficient in the order of `tets` (nullable).
void* orc_create(int nverts, const double* coords, int ncells, const int* tets, const double* k, int maxLevel) {
  Oracle* o = new Oracle();
  for (int i = 0; i < nverts; ++i) o->vx.push_back({coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]});
  std::vector<std::pair<std::array<int, 4>, double>> cs;
  for (int c = 0; c < ncells; ++c) cs.push_back({{tets[4 * c], tets[4 * c + 1], tets[4 * c + 2], tets[4 * c + 3]}, k ? k[c] : 1.0});
  std::sort(cs.begin(), cs.end());
  std::set<std::array<int, 2>> es;
  std::map<std::array<int, 3>, int> fcount;
  for (auto& c : cs) {
    o->cells.push_back(c.first);
    o->k.push_back(c.second);
    std::array<int, 4> s = c.first;
    std::sort(s.begin(), s.end());
    o->cellId[s] = (int)o->cells.size() - 1;
    for (int a = 0; a < 4; ++a)
      for (int b = a + 1; b < 4; ++b) es.insert({s[a], s[b]});
    const int tri[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    for (auto& t : tri) fcount[{s[t[0]], s[t[1]], s[t[2]]}]++;
  }
  for (auto& e : es) o->edgeId[e] = (int)o->edgeId.size();
  for (auto& f : fcount) {
    o->faceId[f.first] = (int)o->faceId.size();
    if (f.second == 1) o->boundaryFaces.insert(f.first);
  }
  o->lv.resize(maxLevel + 1);
  for (int L = 0; L <= maxLevel; ++L) buildLevel(*o, L);
  for (int L = 1; L <= maxLevel; ++L) buildProlongation(*o, L);
  return o;
}

void orc_destroy(void* h) { delete (Oracle*)h; }

int64_t orc_num_nodes(void* h, int L) { return (int64_t)((Oracle*)h)->lv[L].nodes.size(); }

// xyz: 3 coordinates per node; info: 4 per node (owner kind, owner ID, dirichlet, unused)
void orc_nodes(void* h, int L, double* xyz, int* info) {
  const Oracle& o = *(Oracle*)h;
  const LevelData& d = o.lv[L];
  for (size_t i = 0; i < d.nodes.size(); ++i) {
    o.coordOf(d.nodes[i].key, d.N, xyz + 3 * i);
    info[4 * i] = d.nodes[i].kind;
    info[4 * i + 1] = d.nodes[i].id;
    info[4 * i + 2] = d.nodes[i].dirichlet ? 1 : 0;
    info[4 * i + 3] = 0;
  }
}

// y = A u on non-Dirichlet rows (form 0 diffusion, 1 mass); Dirichlet rows keep their value
void orc_apply(void* h, int L, int form, const double* u, double* y) {
  Oracle& o = *(Oracle*)h;
  const Csr& A = matrix(o, L, form);
  const LevelData& d = o.lv[L];
  for (size_t i = 0; i < d.nodes.size(); ++i) {
    if (d.nodes[i].dirichlet) continue;
    double s = 0.0;
    for (int64_t e = A.ptr[i]; e < A.ptr[i + 1]; ++e) s += A.val[e] * u[A.col[e]];
    y[i] = s;
  }
}

// mode 0: reference lexicographic SOR, 1: multicolour SOR (the order of the GPU smoother)
void orc_sor(void* h, int L, double* u, const double* f, double omega, int sweeps, int mode, int backwards) {
  for (int s = 0; s < sweeps; ++s) sorSweep(*(Oracle*)h, L, u, f, omega, mode == 1, backwards != 0);
}

// One sweep restricted to the owners of the kinds in kindMask (bit k: vertex/edge/face/cell);
// the start-of-sweep snapshot is taken at the call, as in sorSweep.
void orc_sor_phases(void* h, int L, double* u, const double* f, double omega, int mode, int backwards, int kindMask) {
  sorSweep(*(Oracle*)h, L, u, f, omega, mode == 1, backwards != 0, kindMask);
}

// coarse = P^T fine on non-Dirichlet coarse nodes (others untouched)
void orc_restrict(void* h, int Lf, const double* fine, double* coarse) {
  Oracle& o = *(Oracle*)h;
  const LevelData& f = o.lv[Lf];
  const LevelData& c = o.lv[Lf - 1];
  std::vector<double> acc(c.nodes.size(), 0.0);
  for (size_t i = 0; i < f.nodes.size(); ++i)
    for (int k = 0; k < 2; ++k)
      if (f.pc[i][k] >= 0) acc[f.pc[i][k]] += f.pw[i][k] * fine[i];
  for (size_t j = 0; j < c.nodes.size(); ++j)
    if (!c.nodes[j].dirichlet) coarse[j] = acc[j];
}

// fine (+)= P coarse on non-Dirichlet fine nodes
void orc_prolongate(void* h, int Lc, const double* coarse, double* fine, int add) {
  Oracle& o = *(Oracle*)h;
  const LevelData& f = o.lv[Lc + 1];
  for (size_t i = 0; i < f.nodes.size(); ++i) {
    if (f.nodes[i].dirichlet) continue;
    double v = 0.0;
    for (int k = 0; k < 2; ++k)
      if (f.pc[i][k] >= 0) v += f.pw[i][k] * coarse[f.pc[i][k]];
    fine[i] = add ? fine[i] + v : v;
  }
}

// The same transfers on every node (a function whose DoFs are all unknowns, like the
// Taylor-Hood pressure): coarse = P^T fine, fine (+)= P coarse.
void orc_restrict_all(void* h, int Lf, const double* fine, double* coarse) {
  Oracle& o = *(Oracle*)h;
  const LevelData& f = o.lv[Lf];
  const LevelData& c = o.lv[Lf - 1];
  for (size_t j = 0; j < c.nodes.size(); ++j) coarse[j] = 0.0;
  for (size_t i = 0; i < f.nodes.size(); ++i)
    for (int k = 0; k < 2; ++k)
      if (f.pc[i][k] >= 0) coarse[f.pc[i][k]] += f.pw[i][k] * fine[i];
}

void orc_prolongate_all(void* h, int Lc, const double* coarse, double* fine, int add) {
  Oracle& o = *(Oracle*)h;
  const LevelData& f = o.lv[Lc + 1];
  for (size_t i = 0; i < f.nodes.size(); ++i) {
    double v = 0.0;
    for (int k = 0; k < 2; ++k)
      if (f.pc[i][k] >= 0) v += f.pw[i][k] * coarse[f.pc[i][k]];
    fine[i] = add ? fine[i] + v : v;
  }
}

double orc_dot(void* h, int L, const double* a, const double* b) {
  const LevelData& d = ((Oracle*)h)->lv[L];
  double s = 0.0;
  for (size_t i = 0; i < d.nodes.size(); ++i)
    if (!d.nodes[i].dirichlet) s += a[i] * b[i];
  return s;
}

// CGSolver::solve with identity preconditioner; returns iterations
int orc_cg(void* h, int L, double* x, const double* b, int maxIter, double tol, double* res) {
  Oracle& o = *(Oracle*)h;
  const LevelData& d = o.lv[L];
  const size_t n = d.nodes.size();
  std::vector<double> p(n, 0.0), r(n, 0.0), ap(n, 0.0);
  orc_apply(h, L, 0, x, p.data());
  for (size_t i = 0; i < n; ++i)
    if (!d.nodes[i].dirichlet) r[i] = b[i] - p[i];
  for (size_t i = 0; i < n; ++i)
    if (!d.nodes[i].dirichlet) p[i] = r[i];
  double prsold = orc_dot(h, L, r.data(), r.data());
  double rs = std::sqrt(prsold);
  if (res) *res = rs;
  if (maxIter == 0 || rs < tol) return 0;
  int it = 0;
  for (int k = 0; k < maxIter; ++k) {
    it = k + 1;
    orc_apply(h, L, 0, p.data(), ap.data());
    const double alpha = prsold / orc_dot(h, L, p.data(), ap.data());
    for (size_t i = 0; i < n; ++i)
      if (!d.nodes[i].dirichlet) {
        x[i] += alpha * p[i];
        r[i] -= alpha * ap[i];
      }
    const double rsnew = orc_dot(h, L, r.data(), r.data());
    if (res) *res = std::sqrt(rsnew);
    if (std::sqrt(rsnew) < tol) break;
    const double beta = rsnew / prsold;
    for (size_t i = 0; i < n; ++i)
      if (!d.nodes[i].dirichlet) p[i] = r[i] + beta * p[i];
    prsold = rsnew;
  }
  return it;
}

static void gmgRec(void* h, int L, int minL, std::vector<std::vector<double>>& x, std::vector<std::vector<double>>& b,
                   int pre, int post, double omega, int mode, int cgIter, double cgTol) {
  Oracle& o = *(Oracle*)h;
  if (L == minL) {
    orc_cg(h, L, x[L].data(), b[L].data(), cgIter, cgTol, nullptr);
    return;
  }
  const LevelData& d = o.lv[L];
  orc_sor(h, L, x[L].data(), b[L].data(), omega, pre, mode, 0);
  std::vector<double> r(d.nodes.size(), 0.0), ax(d.nodes.size(), 0.0);
  orc_apply(h, L, 0, x[L].data(), ax.data());
  for (size_t i = 0; i < d.nodes.size(); ++i)
    if (!d.nodes[i].dirichlet) r[i] = b[L][i] - ax[i];
  orc_restrict(h, L, r.data(), b[L - 1].data());
  std::fill(x[L - 1].begin(), x[L - 1].end(), 0.0);
  gmgRec(h, L - 1, minL, x, b, pre, post, omega, mode, cgIter, cgTol);
  orc_prolongate(h, L - 1, x[L - 1].data(), x[L].data(), 1);
  orc_sor(h, L, x[L].data(), b[L].data(), omega, post, mode, 0);
}

// `cycles` V-cycles on level L; residual 2-norms after each cycle in res[cycles]
void orc_gmg(void* h, int L, int minL, double* x, const double* b, int cycles, int pre, int post, double omega, int mode,
             int cgIter, double cgTol, double* res) {
  Oracle& o = *(Oracle*)h;
  std::vector<std::vector<double>> xs(L + 1), bs(L + 1);
  for (int l = minL; l <= L; ++l) {
    xs[l].assign(o.lv[l].nodes.size(), 0.0);
    bs[l].assign(o.lv[l].nodes.size(), 0.0);
  }
  std::copy(x, x + o.lv[L].nodes.size(), xs[L].begin());
  std::copy(b, b + o.lv[L].nodes.size(), bs[L].begin());
  const LevelData& d = o.lv[L];
  for (int c = 0; c < cycles; ++c) {
    gmgRec(h, L, minL, xs, bs, pre, post, omega, mode, cgIter, cgTol);
    if (res) {
      std::vector<double> ax(d.nodes.size(), 0.0), r(d.nodes.size(), 0.0);
      orc_apply(h, L, 0, xs[L].data(), ax.data());
      for (size_t i = 0; i < d.nodes.size(); ++i)
        if (!d.nodes[i].dirichlet) r[i] = bs[L][i] - ax[i];
      res[c] = std::sqrt(orc_dot(h, L, r.data(), r.data()));
    }
  }
  std::copy(xs[L].begin(), xs[L].end(), x);
}

// Quadratic prolongation from P2 level Lc to Lc + 1: every point of the lattice Lc + 2 inside a
// level-Lc micro-cell has barycentric coordinates l / 4 (l_m >= 0 integers, sum 4) there; its
// row holds the coarse P2 basis values (l(2l-1) at the vertices, 4 l_i l_j at the edges).
void buildP2Prolongation(Oracle& o, int Lc) {
  LevelData& d = o.lv[Lc];
  const LevelData& cL = o.lv[Lc + 1];
  const LevelData& fL = o.lv[Lc + 2];
  const int64_t N = d.N;
  std::vector<std::map<int64_t, double>> rows(fL.nodes.size());
  std::vector<char> done(fL.nodes.size(), 0);
  for (size_t ci = 0; ci < o.cells.size(); ++ci)
    for (int t = 0; t < 6; ++t) {
      const int64_t width = N - kMicroWidthReduction[t];
      for (int64_t z = 0; z < width; ++z)
        for (int64_t y = 0; y + z < width; ++y)
          for (int64_t x = 0; x + y + z < width; ++x) {
            int64_t v[4][3];
            for (int m = 0; m < 4; ++m) {
              v[m][0] = x + kMicro[t][m][0];
              v[m][1] = y + kMicro[t][m][1];
              v[m][2] = z + kMicro[t][m][2];
            }
            int64_t cid[10];
            for (int m = 0; m < 4; ++m) cid[m] = cL.index.at(o.keyOf((int)ci, 2 * N, 2 * v[m][0], 2 * v[m][1], 2 * v[m][2]));
            for (int e = 0; e < 6; ++e) {
              const int a = kP2Edge[e][0], b = kP2Edge[e][1];
              cid[4 + e] = cL.index.at(o.keyOf((int)ci, 2 * N, v[a][0] + v[b][0], v[a][1] + v[b][1], v[a][2] + v[b][2]));
            }
            for (int l1 = 0; l1 <= 4; ++l1)
              for (int l2 = 0; l1 + l2 <= 4; ++l2)
                for (int l3 = 0; l1 + l2 + l3 <= 4; ++l3) {
                  const int l[4] = {4 - l1 - l2 - l3, l1, l2, l3};
                  int64_t q[3] = {0, 0, 0};
                  for (int m = 0; m < 4; ++m)
                    for (int k = 0; k < 3; ++k) q[k] += l[m] * v[m][k];
                  const int64_t fi = fL.index.at(o.keyOf((int)ci, 4 * N, q[0], q[1], q[2]));
                  if (done[fi]) continue;
                  done[fi] = 1;
                  for (int m = 0; m < 4; ++m) {
                    const double lm = l[m] / 4.0, wv = lm * (2.0 * lm - 1.0);
                    if (wv != 0.0) rows[fi][cid[m]] += wv;
                  }
                  for (int e = 0; e < 6; ++e) {
                    const double wv = 4.0 * (l[kP2Edge[e][0]] / 4.0) * (l[kP2Edge[e][1]] / 4.0);
                    if (wv != 0.0) rows[fi][cid[4 + e]] += wv;
                  }
                }
          }
    }
  Csr& P = d.P2prol;
  P.ptr.assign(1, 0);
  for (auto& r : rows) {
    for (auto& kv : r) {
      P.col.push_back(kv.first);
      P.val.push_back(kv.second);
    }
    P.ptr.push_back((int64_t)P.col.size());
  }
  d.haveP2prol = true;
}

void buildDiv(Oracle& o, int L) {
  LevelData& d = o.lv[L];
  const LevelData& f = o.lv[L + 1];
  const int64_t N = d.N;
  std::vector<std::map<int64_t, double>> rows[3];
  for (auto& r : rows) r.resize(d.nodes.size());
  for (size_t ci = 0; ci < o.cells.size(); ++ci)
    for (int t = 0; t < 6; ++t) {
      const int64_t width = N - kMicroWidthReduction[t];
      for (int64_t z = 0; z < width; ++z)
        for (int64_t y = 0; y + z < width; ++y)
          for (int64_t x = 0; x + y + z < width; ++x) {
            int64_t v[4][3];
            double p[4][3];
            int64_t pid[4], vid[10];
            for (int m = 0; m < 4; ++m) {
              v[m][0] = x + kMicro[t][m][0];
              v[m][1] = y + kMicro[t][m][1];
              v[m][2] = z + kMicro[t][m][2];
              const Key k = o.keyOf((int)ci, N, v[m][0], v[m][1], v[m][2]);
              o.coordOf(k, N, p[m]);
              pid[m] = d.index.at(k);
              vid[m] = f.index.at(o.keyOf((int)ci, 2 * N, 2 * v[m][0], 2 * v[m][1], 2 * v[m][2]));
            }
            for (int e = 0; e < 6; ++e) {
              const int a = kP2Edge[e][0], b = kP2Edge[e][1];
              vid[4 + e] = f.index.at(o.keyOf((int)ci, 2 * N, v[a][0] + v[b][0], v[a][1] + v[b][1], v[a][2] + v[b][2]));
            }
            double D[3][4][10];
            p2p1DivElement(p, D);
            for (int k = 0; k < 3; ++k)
              for (int i = 0; i < 4; ++i)
                for (int j = 0; j < 10; ++j) rows[k][pid[i]][vid[j]] += D[k][i][j];
          }
    }
  for (int k = 0; k < 3; ++k) {
    Csr& A = d.Div[k];
    A.ptr.assign(1, 0);
    for (auto& r : rows[k]) {
      for (auto& kv : r) {
        A.col.push_back(kv.first);
        A.val.push_back(kv.second);
      }
      A.ptr.push_back((int64_t)A.col.size());
    }
  }
  d.haveDiv = true;
}

void orc_p2_apply(void* h, int L, const double* u, double* y);

// Taylor-Hood Stokes on P2 level L (velocity: nodes of level L + 1, pressure: nodes of level L):
// v_k = A2 u_k + D_k^T p and q = sum_k D_k u_k, every row.
void orc_stokes_apply(void* h, int L, const double* u0, const double* u1, const double* u2, const double* p, double* v0,
                      double* v1, double* v2, double* q) {
  Oracle& o = *(Oracle*)h;
  if (!o.lv[L].haveDiv) buildDiv(o, L);
  const double* u[3] = {u0, u1, u2};
  double* v[3] = {v0, v1, v2};
  for (int k = 0; k < 3; ++k) orc_p2_apply(h, L, u[k], v[k]);
  const int64_t np = (int64_t)o.lv[L].nodes.size();
  for (int64_t i = 0; i < np; ++i) q[i] = 0.0;
  for (int k = 0; k < 3; ++k) {
    const Csr& D = o.lv[L].Div[k];
    for (int64_t i = 0; i < np; ++i)
      for (int64_t m = D.ptr[i]; m < D.ptr[i + 1]; ++m) {
        q[i] += D.val[m] * u[k][D.col[m]];
        v[k][D.col[m]] += D.val[m] * p[i];
      }
  }
}

// P1 PSPG element matrix -tau K_laplace, tau = |T|^(2/3) / 12
void orc_element_pspg(const double* coords12, double* K16) {
  double p[4][3], K[4][4];
  for (int m = 0; m < 4; ++m)
    for (int d = 0; d < 3; ++d) p[m][d] = coords12[3 * m + d];
  laplaceElement(p, K);
  const double tau = std::pow(tetVolume(p), 2.0 / 3.0) / 12.0;
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) K16[4 * a + b] = -tau * K[a][b];
}

// Row sums of the assembled mass matrix of level L (the lumped mass, every node)
void orc_lumped_mass(void* h, int L, double* d) {
  Oracle& o = *(Oracle*)h;
  const Csr& A = matrix(o, L, 1);
  for (size_t i = 0; i + 1 < A.ptr.size(); ++i) {
    d[i] = 0.0;
    for (int64_t k = A.ptr[i]; k < A.ptr[i + 1]; ++k) d[i] += A.val[k];
  }
}

// Diagonal of the assembled PSPG matrix of level L (every node)
void orc_pspg_diag(void* h, int L, double* d) {
  Oracle& o = *(Oracle*)h;
  const Csr& A = matrix(o, L, 2);
  for (size_t i = 0; i + 1 < A.ptr.size(); ++i) {
    d[i] = 0.0;
    for (int64_t k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
      if (A.col[k] == (int64_t)i) d[i] += A.val[k];
  }
}

void orc_p2p1_div_element(const double* coords12, double* D120) {
  double p[4][3];
  for (int m = 0; m < 4; ++m)
    for (int d = 0; d < 3; ++d) p[m][d] = coords12[3 * m + d];
  double D[3][4][10];
  p2p1DivElement(p, D);
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 10; ++j) D120[40 * k + 10 * i + j] = D[k][i][j];
}

// fine (nodes of level Lc + 2) = P coarse (nodes of level Lc + 1), or += with add
void orc_p2_prolongate(void* h, int Lc, const double* coarse, double* fine, int add) {
  Oracle& o = *(Oracle*)h;
  if (!o.lv[Lc].haveP2prol) buildP2Prolongation(o, Lc);
  const Csr& P = o.lv[Lc].P2prol;
  for (size_t i = 0; i + 1 < P.ptr.size(); ++i) {
    double s = 0.0;
    for (int64_t k = P.ptr[i]; k < P.ptr[i + 1]; ++k) s += P.val[k] * coarse[P.col[k]];
    fine[i] = add ? fine[i] + s : s;
  }
}

// coarse (nodes of level Lf) = P^T fine (nodes of level Lf + 1): restriction from P2 level Lf
void orc_p2_restrict(void* h, int Lf, const double* fine, double* coarse) {
  Oracle& o = *(Oracle*)h;
  if (!o.lv[Lf - 1].haveP2prol) buildP2Prolongation(o, Lf - 1);
  const Csr& P = o.lv[Lf - 1].P2prol;
  for (size_t j = 0; j < o.lv[Lf].nodes.size(); ++j) coarse[j] = 0.0;
  for (size_t i = 0; i + 1 < P.ptr.size(); ++i)
    for (int64_t k = P.ptr[i]; k < P.ptr[i + 1]; ++k) coarse[P.col[k]] += P.val[k] * fine[i];
}

// y = A2 u for the P2 Laplace of level L; u and y are indexed by the nodes of level L + 1.
void orc_p2_apply(void* h, int L, const double* u, double* y) {
  Oracle& o = *(Oracle*)h;
  if (!o.lv[L].haveP2) buildP2Matrix(o, L);
  const Csr& A = o.lv[L].P2;
  const int64_t n = (int64_t)A.ptr.size() - 1;
  for (int64_t i = 0; i < n; ++i) {
    double s = 0.0;
    for (int64_t k = A.ptr[i]; k < A.ptr[i + 1]; ++k) s += A.val[k] * u[A.col[k]];
    y[i] = s;
  }
}

// Multicolour SOR on P2 level L in the GPU's colour order: colour of a node from its
// barycentric weights in ascending vertex order; a pass updates all non-Dirichlet nodes of one
// colour from the values at the start of the pass.
void orc_p2_sor(void* h, int L, double* u, const double* f, double omega, int sweeps, int backwards) {
  Oracle& o = *(Oracle*)h;
  if (!o.lv[L].haveP2) buildP2Matrix(o, L);
  const Csr& A = o.lv[L].P2;
  const LevelData& F = o.lv[L + 1];
  const int64_t n = (int64_t)F.nodes.size();
  std::vector<int> col(n);
  std::vector<double> diag(n, 0.0);
  for (int64_t i = 0; i < n; ++i) {
    const Key& k = F.nodes[i].key;
    const int64_t w1 = k[3], w2 = k[5], w3 = k[7];
    const int par = int(w1 & 1) | (int(w2 & 1) << 1) | (int(w3 & 1) << 2);
    col[i] = par ? 3 + par : int(((w1 >> 1) + 2 * (w2 >> 1) + 3 * (w3 >> 1)) % 4);
    for (int64_t q = A.ptr[i]; q < A.ptr[i + 1]; ++q)
      if (A.col[q] == i) diag[i] += A.val[q];
  }
  std::vector<double> r(n);
  for (int s = 0; s < sweeps; ++s)
    for (int kk = 0; kk < 11; ++kk) {
      const int c = backwards ? 10 - kk : kk;
      for (int64_t i = 0; i < n; ++i) {
        if (col[i] != c || F.nodes[i].dirichlet) continue;
        double t = f[i];
        for (int64_t q = A.ptr[i]; q < A.ptr[i + 1]; ++q) t -= A.val[q] * u[A.col[q]];
        r[i] = t;
      }
      for (int64_t i = 0; i < n; ++i)
        if (col[i] == c && !F.nodes[i].dirichlet) u[i] += omega * r[i] / diag[i];
    }
}

// CG on the non-Dirichlet rows of the P2 Laplace of level L (Dirichlet values of x kept).
int orc_p2_cg(void* h, int L, double* x, const double* b, int maxIter, double tol) {
  Oracle& o = *(Oracle*)h;
  if (!o.lv[L].haveP2) buildP2Matrix(o, L);
  const Csr& A = o.lv[L].P2;
  const LevelData& F = o.lv[L + 1];
  const int64_t n = (int64_t)F.nodes.size();
  auto mv = [&](const std::vector<double>& u, std::vector<double>& y) {
    for (int64_t i = 0; i < n; ++i) {
      double t = 0.0;
      if (!F.nodes[i].dirichlet)
        for (int64_t k = A.ptr[i]; k < A.ptr[i + 1]; ++k) t += A.val[k] * u[A.col[k]];
      y[i] = t;
    }
  };
  std::vector<double> xv(x, x + n), r(n), p(n), ap(n);
  mv(xv, ap);
  for (int64_t i = 0; i < n; ++i) r[i] = F.nodes[i].dirichlet ? 0.0 : b[i] - ap[i];
  for (int64_t i = 0; i < n; ++i) p[i] = F.nodes[i].dirichlet ? 0.0 : r[i];
  auto dot = [&](const std::vector<double>& a, const std::vector<double>& c) {
    double t = 0.0;
    for (int64_t i = 0; i < n; ++i) t += a[i] * c[i];
    return t;
  };
  double rs = dot(r, r);
  int it = 0;
  for (; it < maxIter && std::sqrt(rs) >= tol; ++it) {
    mv(p, ap);
    const double alpha = rs / dot(p, ap);
    for (int64_t i = 0; i < n; ++i) {
      xv[i] += alpha * p[i];
      r[i] -= alpha * ap[i];
    }
    const double rn = dot(r, r);
    for (int64_t i = 0; i < n; ++i) p[i] = r[i] + rn / rs * p[i];
    rs = rn;
  }
  std::copy(xv.begin(), xv.end(), x);
  return it;
}

void orc_p2_element_laplace(const double* coords12, double* K100) {
  double p[4][3];
  for (int m = 0; m < 4; ++m)
    for (int d = 0; d < 3; ++d) p[m][d] = coords12[3 * m + d];
  double K[10][10];
  p2LaplaceElement(p, K);
  for (int i = 0; i < 10; ++i)
    for (int j = 0; j < 10; ++j) K100[10 * i + j] = K[i][j];
}

void orc_element_laplace(const double* coords12, double* K16) {
  double p[4][3], K[4][4];
  for (int i = 0; i < 4; ++i)
    for (int d = 0; d < 3; ++d) p[i][d] = coords12[3 * i + d];
  laplaceElement(p, K);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) K16[4 * i + j] = K[i][j];
}

void orc_element_mass(const double* coords12, double* K16) {
  double p[4][3], K[4][4];
  for (int i = 0; i < 4; ++i)
    for (int d = 0; d < 3; ++d) p[i][d] = coords12[3 * i + d];
  massElement(p, K);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) K16[4 * i + j] = K[i][j];
}

// Contributions of the micro-cells of macro-cell `cell` (creation order) to the row of the
// cell-local point (x, y, z): out[k] for the 15 offsets of the reference cell stencil in the
// order C E W N S NW SE TC TW TS TSE BC BE BN BNW (entries whose neighbour lies outside the
// cell stay 0). Used to drive the reference's own generated kernels.
void orc_cell_local_stencil(void* h, int L, int cell, int x, int y, int z, int form, double* out15) {
  Oracle& o = *(Oracle*)h;
  static const int off[15][3] = {{0, 0, 0},  {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0},
                                 {-1, 1, 0}, {1, -1, 0}, {0, 0, 1},  {-1, 0, 1}, {0, -1, 1},
                                 {1, -1, 1}, {0, 0, -1}, {1, 0, -1}, {0, 1, -1}, {-1, 1, -1}};
  const int64_t N = int64_t(1) << L;
  for (int k = 0; k < 15; ++k) out15[k] = 0.0;
  for (int t = 0; t < 6; ++t) {
    const int64_t width = N - kMicroWidthReduction[t];
    for (int a = 0; a < 4; ++a) {
      const int64_t i0 = x - kMicro[t][a][0], i1 = y - kMicro[t][a][1], i2 = z - kMicro[t][a][2];
      if (i0 < 0 || i1 < 0 || i2 < 0 || i0 + i1 + i2 > width - 1) continue;
      double p[4][3], K[4][4];
      for (int m = 0; m < 4; ++m)
        o.coordOf(o.keyOf(cell, N, i0 + kMicro[t][m][0], i1 + kMicro[t][m][1], i2 + kMicro[t][m][2]), N, p[m]);
      if (form == 0) {
        laplaceElement(p, K);
        for (auto& r : K)
          for (double& v : r) v *= o.k[cell];
      } else {
        massElement(p, K);
      }
      for (int m = 0; m < 4; ++m) {
        const int dx = kMicro[t][m][0] - kMicro[t][a][0], dy = kMicro[t][m][1] - kMicro[t][a][1],
                  dz = kMicro[t][m][2] - kMicro[t][a][2];
        for (int k = 0; k < 15; ++k)
          if (off[k][0] == dx && off[k][1] == dy && off[k][2] == dz) out15[k] += K[a][m];
      }
    }
  }
}

}  // extern "C"
