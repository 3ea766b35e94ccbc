#include "discretization.hpp"

#include <algorithm>
#include <cmath>
#include <map>
#include <stdexcept>
#include <string>

namespace hg {

Bary makeBary(const int* verts, const int64_t* weights, int count) {
  Bary p;
  std::pair<int, int64_t> tmp[4];
  int n = 0;
  for (int i = 0; i < count; ++i)
    if (weights[i] != 0) {
      if (weights[i] < 0) throw std::runtime_error("negative barycentric weight");
      bool merged = false;
      for (int j = 0; j < n; ++j)
        if (tmp[j].first == verts[i]) {
          tmp[j].second += weights[i];
          merged = true;
        }
      if (!merged) tmp[n++] = {verts[i], weights[i]};
    }
  std::sort(tmp, tmp + n);
  p.n = n;
  for (int i = 0; i < n; ++i) {
    p.v[i] = tmp[i].first;
    p.b[i] = tmp[i].second;
  }
  return p;
}

const int kCellOffsets[15][3] = {{0, 0, 0},  {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0},
                                 {-1, 1, 0}, {1, -1, 0}, {0, 0, 1},  {-1, 0, 1}, {0, -1, 1},
                                 {1, -1, 1}, {0, 0, -1}, {1, 0, -1}, {0, 1, -1}, {-1, 1, -1}};

// Micro-cell types of the uniform refinement (celldofspace/CellDoFIndexing.hpp:128-175):
// vertex offsets from the micro-cell index and the per-type width reduction.
static const int kMicroCell[6][4][3] = {
    {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}},  // white up
    {{1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {1, 0, 1}},  // blue up
    {{1, 0, 0}, {0, 1, 0}, {1, 0, 1}, {0, 0, 1}},  // green up
    {{1, 1, 0}, {1, 1, 1}, {0, 1, 1}, {1, 0, 1}},  // white down
    {{1, 0, 1}, {0, 1, 1}, {0, 0, 1}, {0, 1, 0}},  // blue down
    {{0, 1, 0}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}},  // green down
};
static const int kMicroCellWidthReduction[6] = {0, 1, 1, 2, 1, 1};

Discretization::Discretization(const Topology& topo, int maxLevel) : topo_(topo) {
  if (maxLevel < 0 || maxLevel > 10) throw std::runtime_error("level out of range [0,10]");
  for (auto& c : topo_.cells) {
    std::array<int, 4> k{c.v[0], c.v[1], c.v[2], c.v[3]};
    std::sort(k.begin(), k.end());
    cellByVerts_[k] = (int)cellByVerts_.size();
  }
  levels_.resize(maxLevel + 1);
  for (int L = 0; L <= maxLevel; ++L) buildLevel(L);
}

int Discretization::cellOf(const int* s) const {
  auto it = cellByVerts_.find({s[0], s[1], s[2], s[3]});
  return it == cellByVerts_.end() ? -1 : it->second;
}

int64_t Discretization::ownedCount(int L, int kind) const {
  const int64_t N = int64_t(1) << L;
  switch (kind) {
    case KV: return 1;
    case KE: return std::max<int64_t>(N - 1, 0);
    case KF: return N >= 3 ? tri(N - 2) : 0;
    default: return N >= 4 ? tet(N - 3) : 0;
  }
}

std::vector<SlotRun> ownedRuns(const Discretization& d, int L) {
  const LevelLayout& lay = d.level(L);
  const int64_t N = lay.N, w = lay.w;
  std::vector<SlotRun> runs;
  for (int64_t off : lay.off[KC])
    for (int64_t z = 1; z <= N - 3; ++z)
      for (int64_t y = 1; y <= N - 2 - z; ++y) runs.push_back({off + cellIdx(w, 1, y, z), N - 1 - y - z});
  for (int64_t off : lay.off[KF])
    for (int64_t y = 1; y <= N - 2; ++y) runs.push_back({off + faceIdx(w, 1, y), N - 1 - y});
  for (int64_t off : lay.off[KE])
    if (N >= 2) runs.push_back({off + 1, N - 1});
  for (int64_t off : lay.off[KV]) runs.push_back({off, 1});
  std::sort(runs.begin(), runs.end(), [](const SlotRun& a, const SlotRun& b) { return a.slot < b.slot; });
  return runs;
}

static int cellOppositeVertex(const MacroCell& c, const MacroFace& f) {
  for (int i = 0; i < 4; ++i)
    if (c.v[i] != f.v[0] && c.v[i] != f.v[1] && c.v[i] != f.v[2]) return c.v[i];
  throw std::runtime_error("face not part of cell");
}

Bary Discretization::slotBary(int L, int kind, int prim, int64_t s) const {
  const int64_t N = int64_t(1) << L, w = N + 1;
  if (kind == KV) {
    const auto& v = topo_.verts[prim];
    int self = prim;
    if (s == 0) return makeBary(&self, &N, 1);
    const auto& e = topo_.edges[v.edges.at(s - 1)];
    // VertexDoFPackInfo.hpp:158-181: the edge DoF next to this vertex
    int64_t x = (e.v[0] == prim) ? 1 : N - 1;
    int64_t wts[2] = {N - x, x};
    return makeBary(e.v, wts, 2);
  }
  if (kind == KE) {
    const auto& e = topo_.edges[prim];
    const int64_t nf = (int64_t)e.faces.size();
    if (s < w) {
      int64_t wts[2] = {N - s, s};
      return makeBary(e.v, wts, 2);
    }
    s -= w;
    if (s < nf * (w - 1)) {  // face ghost layer: the face row next to the edge
      const auto& f = topo_.faces[e.faces[s / (w - 1)]];
      const int64_t j = s % (w - 1);
      int t = -1;
      for (int i = 0; i < 3; ++i)
        if (f.v[i] != e.v[0] && f.v[i] != e.v[1]) t = f.v[i];
      int vs[3] = {e.v[0], e.v[1], t};
      int64_t wts[3] = {N - 1 - j, j, 1};
      return makeBary(vs, wts, 3);
    }
    s -= nf * (w - 1);
    // cell ghost layer (filled from the face ghost layers, VertexDoFPackInfo.hpp:300-325):
    // the point one step from the edge towards both remaining cell vertices
    const auto& c = topo_.cells[e.cells.at(s / (w - 2))];
    const int64_t j = s % (w - 2);
    int o[2], no = 0;
    for (int i = 0; i < 4; ++i)
      if (c.v[i] != e.v[0] && c.v[i] != e.v[1]) o[no++] = c.v[i];
    int vs[4] = {e.v[0], e.v[1], o[0], o[1]};
    int64_t wts[4] = {N - 2 - j, j, 1, 1};
    return makeBary(vs, wts, 4);
  }
  if (kind == KF) {
    const auto& f = topo_.faces[prim];
    const int64_t t0 = tri(w);
    if (s < t0) {
      int64_t y = 0;
      while (faceIdx(w, 0, y + 1) <= s) ++y;
      const int64_t x = s - faceIdx(w, 0, y);
      int64_t wts[3] = {N - x - y, x, y};
      return makeBary(f.v, wts, 3);
    }
    s -= t0;
    const int64_t t1 = tri(w - 1);
    const auto& c = topo_.cells.at(f.cells.at(s / t1));
    s %= t1;
    int64_t y = 0;
    while (faceIdx(w - 1, 0, y + 1) <= s) ++y;
    const int64_t x = s - faceIdx(w - 1, 0, y);
    // ghost layer n holds the face-frame index (x, y, 1) of neighbour cell n
    // (VertexDoFMacroFace.hpp:51-66 with DistanceCoordinateSystem.hpp:146-151)
    int vs[4] = {f.v[0], f.v[1], f.v[2], cellOppositeVertex(c, f)};
    int64_t wts[4] = {N - x - y - 1, x, y, 1};
    return makeBary(vs, wts, 4);
  }
  const auto& c = topo_.cells[prim];
  int64_t z = 0;
  while (z + 1 <= N && tet(w) - tet(w - z - 1) <= s) ++z;
  const int64_t W = w - z;
  int64_t r = s - (tet(w) - tet(W));
  int64_t y = 0;
  while (faceIdx(W, 0, y + 1) <= r) ++y;
  const int64_t x = r - faceIdx(W, 0, y);
  int64_t wts[4] = {N - x - y - z, x, y, z};
  return makeBary(c.v, wts, 4);
}

Slot Discretization::owner(int L, const Bary& p) const {
  const int64_t N = int64_t(1) << L, w = N + 1;
  Slot s;
  if (p.n == 1) {
    s.kind = KV;
    s.prim = p.v[0];
    s.local = 0;
  } else if (p.n == 2) {
    s.kind = KE;
    s.prim = topo_.edgeOf(p.v[0], p.v[1]);
    s.local = p.of(topo_.edges[s.prim].v[1]);
  } else if (p.n == 3) {
    s.kind = KF;
    s.prim = topo_.faceOf(p.v[0], p.v[1], p.v[2]);
    const auto& f = topo_.faces[s.prim];
    s.local = faceIdx(w, p.of(f.v[1]), p.of(f.v[2]));
  } else {
    s.kind = KC;
    s.prim = cellOf(p.v);
    if (s.prim < 0) throw std::runtime_error("micro-vertex outside every macro-cell");
    const auto& c = topo_.cells[s.prim];
    s.local = cellIdx(w, p.of(c.v[1]), p.of(c.v[2]), p.of(c.v[3]));
  }
  (void)N;
  return s;
}

int64_t Discretization::localSlotOf(int L, int kind, int prim, const Bary& p) const {
  const int64_t N = int64_t(1) << L, w = N + 1;
  auto inSet = [](int v, const int* set, int n) {
    for (int i = 0; i < n; ++i)
      if (set[i] == v) return true;
    return false;
  };
  if (kind == KC) {
    const auto& c = topo_.cells[prim];
    for (int i = 0; i < p.n; ++i)
      if (!inSet(p.v[i], c.v, 4)) return -1;
    return cellIdx(w, p.of(c.v[1]), p.of(c.v[2]), p.of(c.v[3]));
  }
  if (kind == KF) {
    const auto& f = topo_.faces[prim];
    int extra = -1, nextra = 0;
    for (int i = 0; i < p.n; ++i)
      if (!inSet(p.v[i], f.v, 3)) {
        extra = p.v[i];
        ++nextra;
      }
    if (nextra == 0) return faceIdx(w, p.of(f.v[1]), p.of(f.v[2]));
    if (nextra > 1 || p.of(extra) != 1) return -1;
    for (size_t n = 0; n < f.cells.size(); ++n)
      if (cellOppositeVertex(topo_.cells[f.cells[n]], f) == extra)
        return tri(w) + (int64_t)n * tri(w - 1) + faceIdx(w - 1, p.of(f.v[1]), p.of(f.v[2]));
    return -1;
  }
  if (kind == KE) {
    const auto& e = topo_.edges[prim];
    int ex[4], nex = 0;
    for (int i = 0; i < p.n; ++i)
      if (!inSet(p.v[i], e.v, 2)) ex[nex++] = p.v[i];
    const int64_t j = p.of(e.v[1]);
    if (nex == 0) return j;
    if (nex == 1) {
      if (p.of(ex[0]) != 1) return -1;
      const int f = topo_.faceOf(e.v[0], e.v[1], ex[0]);
      for (size_t k = 0; k < e.faces.size(); ++k)
        if (e.faces[k] == f) return w + (int64_t)k * (w - 1) + j;
      return -1;
    }
    if (nex == 2) {
      if (p.of(ex[0]) != 1 || p.of(ex[1]) != 1) return -1;
      int key[4] = {e.v[0], e.v[1], ex[0], ex[1]};
      std::sort(key, key + 4);
      const int c = cellOf(key);
      for (size_t k = 0; k < e.cells.size(); ++k)
        if (e.cells[k] == c) return w + (int64_t)e.faces.size() * (w - 1) + (int64_t)k * (w - 2) + j;
      return -1;
    }
    return -1;
  }
  // vertex
  const auto& v = topo_.verts[prim];
  if (p.n == 1 && p.v[0] == prim) return 0;
  int other = -1, nother = 0;
  for (int i = 0; i < p.n; ++i)
    if (p.v[i] != prim) {
      other = p.v[i];
      ++nother;
    }
  if (nother != 1 || p.of(other) != 1) return -1;
  const int e = topo_.edgeOf(prim, other);
  for (size_t k = 0; k < v.edges.size(); ++k)
    if (v.edges[k] == e) return 1 + (int64_t)k;
  (void)N;
  return -1;
}

void Discretization::buildLevel(int L) {
  LevelLayout& lay = levels_[L];
  lay.L = L;
  lay.N = int64_t(1) << L;
  lay.w = lay.N + 1;
  const int64_t w = lay.w;
  int64_t o = 0;
  for (size_t c = 0; c < topo_.cells.size(); ++c) {
    lay.off[KC].push_back(o);
    lay.size[KC].push_back(tet(w));
    o += (tet(w) + 31) / 32 * 32;
  }
  for (const auto& f : topo_.faces) {
    lay.off[KF].push_back(o);
    const int64_t n = tri(w) + (int64_t)f.cells.size() * tri(w - 1);
    lay.size[KF].push_back(n);
    o += n;
  }
  for (const auto& e : topo_.edges) {
    lay.off[KE].push_back(o);
    const int64_t n = w + (int64_t)e.faces.size() * (w - 1) + (int64_t)e.cells.size() * (w - 2);
    lay.size[KE].push_back(n);
    o += n;
  }
  for (const auto& v : topo_.verts) {
    lay.off[KV].push_back(o);
    lay.size[KV].push_back(1 + (int64_t)v.edges.size());
    o += 1 + (int64_t)v.edges.size();
  }
  lay.total = o;

  // Halo tables. Face/edge/vertex slots are enumerated generically; cell closures are
  // enumerated face by face (the interior is owned), which avoids visiting tet(w) slots.
  auto addCopy = [&](int kind, int prim, int64_t local) {
    const Bary p = slotBary(L, kind, prim, local);
    const Slot s = owner(L, p);
    if (s.kind == kind && s.prim == prim) {
      if (s.local != local) throw std::runtime_error("inconsistent slot identity");
      return;
    }
    const int g = kind == KV ? G_VERT : kind == KE ? G_EDGE : G_FACE_BOUNDARY;
    lay.commDst[g].push_back(lay.off[kind][prim] + local);
    lay.commSrc[g].push_back(lay.off[s.kind][s.prim] + s.local);
  };
  for (size_t v = 0; v < topo_.verts.size(); ++v)
    for (int64_t s = 0; s < lay.size[KV][v]; ++s) addCopy(KV, (int)v, s);
  for (size_t e = 0; e < topo_.edges.size(); ++e)
    for (int64_t s = 0; s < lay.size[KE][e]; ++s) addCopy(KE, (int)e, s);
  for (size_t f = 0; f < topo_.faces.size(); ++f) {
    const auto& fa = topo_.faces[f];
    // triangle part: only the boundary rows are copies
    for (int64_t y = 0; y < w; ++y)
      for (int64_t x = 0; x + y < w; ++x)
        if (x == 0 || y == 0 || x + y == w - 1) addCopy(KF, (int)f, faceIdx(w, x, y));
    for (size_t n = 0; n < fa.cells.size(); ++n) {
      int vs[4] = {fa.v[0], fa.v[1], fa.v[2], cellOppositeVertex(topo_.cells[fa.cells[n]], fa)};
      for (int64_t y = 0; y < w - 1; ++y)
        for (int64_t x = 0; x + y < w - 1; ++x) {
          int64_t wts[4] = {lay.N - x - y - 1, x, y, 1};
          const Slot s = owner(L, makeBary(vs, wts, 4));
          lay.commDst[G_FACE_GHOST].push_back(lay.off[KF][f] + tri(w) + (int64_t)n * tri(w - 1) + faceIdx(w - 1, x, y));
          lay.commSrc[G_FACE_GHOST].push_back(lay.off[s.kind][s.prim] + s.local);
        }
    }
  }
  for (size_t c = 0; c < topo_.cells.size(); ++c) {
    const auto& ce = topo_.cells[c];
    for (int64_t z = 0; z < w; ++z)
      for (int64_t y = 0; y + z < w; ++y)
        for (int64_t x = 0; x + y + z < w; ++x) {
          if (x != 0 && y != 0 && z != 0 && x + y + z != w - 1) {
            x = w - 1 - y - z - 1;  // jump to the last point of the row
            continue;
          }
          const int64_t local = cellIdx(w, x, y, z);
          int64_t wts[4] = {lay.N - x - y - z, x, y, z};
          const Bary p = makeBary(ce.v, wts, 4);
          const Slot s = owner(L, p);
          lay.commDst[G_CELL].push_back(lay.off[KC][c] + local);
          lay.commSrc[G_CELL].push_back(lay.off[s.kind][s.prim] + s.local);
        }
  }
}

// ---------------------------------------------------------------------------------------
// Element matrices
// ---------------------------------------------------------------------------------------
const int kP2Edge[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
const int kMicroCellTable[6][4][3] = {
    {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, {{1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {1, 0, 1}},
    {{1, 0, 0}, {0, 1, 0}, {1, 0, 1}, {0, 0, 1}}, {{1, 1, 0}, {1, 1, 1}, {0, 1, 1}, {1, 0, 1}},
    {{1, 0, 1}, {0, 1, 1}, {0, 0, 1}, {0, 1, 0}}, {{0, 1, 0}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}},
};
const int kMicroCellWidth[6] = {0, 1, 1, 2, 1, 1};

void elementP2Laplace(const double p[4][3], double K[100]) {
  double J[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) J[r][c] = p[c + 1][r] - p[0][r];
  const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                     J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                     J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  // gradients of the barycentric coordinates: rows of J^-1 (lambda_1..3), lambda_0 = 1 - sum
  const double cof[3][3] = {{J[1][1] * J[2][2] - J[1][2] * J[2][1], J[0][2] * J[2][1] - J[0][1] * J[2][2],
                             J[0][1] * J[1][2] - J[0][2] * J[1][1]},
                            {J[1][2] * J[2][0] - J[1][0] * J[2][2], J[0][0] * J[2][2] - J[0][2] * J[2][0],
                             J[0][2] * J[1][0] - J[0][0] * J[1][2]},
                            {J[1][0] * J[2][1] - J[1][1] * J[2][0], J[0][1] * J[2][0] - J[0][0] * J[2][1],
                             J[0][0] * J[1][1] - J[0][1] * J[1][0]}};
  double G[4][3];
  for (int d = 0; d < 3; ++d) {
    for (int i = 0; i < 3; ++i) G[i + 1][d] = cof[i][d] / det;
    G[0][d] = -(G[1][d] + G[2][d] + G[3][d]);
  }
  double gg[4][4];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) gg[a][b] = G[a][0] * G[b][0] + G[a][1] * G[b][1] + G[a][2] * G[b][2];
  const double vol = std::fabs(det) / 6.0;
  auto m2 = [vol](int a, int b) { return vol * (a == b ? 2.0 : 1.0) / 20.0; };  // int lambda_a lambda_b
  auto m1l = [vol](int a, int x) { return vol * ((a == x ? 2.0 : 1.0) / 5.0 - 0.25); };  // int (4 l_a - 1) l_x
  // node i: vertex a (i < 4) with gradient (4 l_a - 1) G_a, or edge (a, b) with 4 (l_b G_a + l_a G_b)
  for (int i = 0; i < 10; ++i)
    for (int j = 0; j < 10; ++j) {
      double v;
      if (i < 4 && j < 4) {
        v = gg[i][j] * vol * (4.0 * (i == j ? 2.0 : 1.0) / 5.0 - 1.0);
      } else if (i < 4 || j < 4) {
        const int a = i < 4 ? i : j, e = (i < 4 ? j : i) - 4;
        const int c = kP2Edge[e][0], d = kP2Edge[e][1];
        v = 4.0 * (gg[a][c] * m1l(a, d) + gg[a][d] * m1l(a, c));
      } else {
        const int a = kP2Edge[i - 4][0], b = kP2Edge[i - 4][1], c = kP2Edge[j - 4][0], d = kP2Edge[j - 4][1];
        v = 16.0 * (gg[a][c] * m2(b, d) + gg[a][d] * m2(b, c) + gg[b][c] * m2(a, d) + gg[b][d] * m2(a, c));
      }
      K[10 * i + j] = v;
    }
}

void elementP2P1Div(const double p[4][3], double D[3][40]) {
  double J[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) J[r][c] = p[c + 1][r] - p[0][r];
  const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                     J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                     J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  const double cof[3][3] = {{J[1][1] * J[2][2] - J[1][2] * J[2][1], J[0][2] * J[2][1] - J[0][1] * J[2][2],
                             J[0][1] * J[1][2] - J[0][2] * J[1][1]},
                            {J[1][2] * J[2][0] - J[1][0] * J[2][2], J[0][0] * J[2][2] - J[0][2] * J[2][0],
                             J[0][2] * J[1][0] - J[0][0] * J[1][2]},
                            {J[1][0] * J[2][1] - J[1][1] * J[2][0], J[0][1] * J[2][0] - J[0][0] * J[2][1],
                             J[0][0] * J[1][1] - J[0][1] * J[1][0]}};
  double G[4][3];
  for (int d = 0; d < 3; ++d) {
    for (int i = 0; i < 3; ++i) G[i + 1][d] = cof[i][d] / det;
    G[0][d] = -(G[1][d] + G[2][d] + G[3][d]);
  }
  const double vol = std::fabs(det) / 6.0;
  // int lambda_i (4 lambda_a - 1) = |T| ((1 + delta_ia) / 5 - 1/4); int lambda_i lambda_b = |T| (1 + delta_ib) / 20
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 10; ++j) {
        double v;
        if (j < 4) {
          v = G[j][k] * vol * ((i == j ? 2.0 : 1.0) / 5.0 - 0.25);
        } else {
          const int a = kP2Edge[j - 4][0], b = kP2Edge[j - 4][1];
          v = 4.0 * vol / 20.0 * (G[a][k] * (i == b ? 2.0 : 1.0) + G[b][k] * (i == a ? 2.0 : 1.0));
        }
        D[k][10 * i + j] = -v;
      }
}

std::vector<double> p2p1CellDiv(const Topology& topo, int L) {
  const int64_t N = int64_t(1) << L;
  std::vector<double> out(topo.cells.size() * 6 * 120, 0.0);
  for (size_t c = 0; c < topo.cells.size(); ++c) {
    const auto& ce = topo.cells[c];
    double V[4][3];
    for (int i = 0; i < 4; ++i)
      for (int d = 0; d < 3; ++d) V[i][d] = topo.verts[ce.v[i]].x[d];
    for (int t = 0; t < 6; ++t) {
      double P[4][3];
      for (int m = 0; m < 4; ++m)
        for (int d = 0; d < 3; ++d)
          P[m][d] = V[0][d] + ((V[1][d] - V[0][d]) * kMicroCellTable[t][m][0] +
                               (V[2][d] - V[0][d]) * kMicroCellTable[t][m][1] +
                               (V[3][d] - V[0][d]) * kMicroCellTable[t][m][2]) /
                                  (double)N;
      double D[3][40];
      elementP2P1Div(P, D);
      for (int k = 0; k < 3; ++k)
        for (int i = 0; i < 40; ++i) out[(c * 6 + t) * 120 + k * 40 + i] = D[k][i];
    }
  }
  return out;
}

std::vector<double> p2CellElements(const Topology& topo, int L) {
  const int64_t N = int64_t(1) << L;
  std::vector<double> out(topo.cells.size() * 600, 0.0);
  for (size_t c = 0; c < topo.cells.size(); ++c) {
    const auto& ce = topo.cells[c];
    double V[4][3];
    for (int i = 0; i < 4; ++i)
      for (int d = 0; d < 3; ++d) V[i][d] = topo.verts[ce.v[i]].x[d];
    for (int t = 0; t < 6; ++t) {
      double P[4][3];
      for (int m = 0; m < 4; ++m)
        for (int d = 0; d < 3; ++d)
          P[m][d] = V[0][d] + ((V[1][d] - V[0][d]) * kMicroCellTable[t][m][0] +
                               (V[2][d] - V[0][d]) * kMicroCellTable[t][m][1] +
                               (V[3][d] - V[0][d]) * kMicroCellTable[t][m][2]) /
                                  (double)N;
      double K[100];
      elementP2Laplace(P, K);
      for (int i = 0; i < 100; ++i) out[c * 600 + t * 100 + i] = ce.k * K[i];
    }
  }
  return out;
}

void elementLaplace(const double p[4][3], double K[16]) {
  double J[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) J[r][c] = p[c + 1][r] - p[0][r];
  const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                     J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                     J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  double inv[3][3];  // inverse of J: row i = gradient of barycentric coordinate i+1
  inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
  inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
  inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
  inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
  inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
  inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
  inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
  inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
  inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
  double g[4][3];
  for (int d = 0; d < 3; ++d) {
    g[1][d] = inv[0][d];
    g[2][d] = inv[1][d];
    g[3][d] = inv[2][d];
    g[0][d] = -(g[1][d] + g[2][d] + g[3][d]);
  }
  const double vol = std::fabs(det) / 6.0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) K[4 * i + j] = vol * (g[i][0] * g[j][0] + g[i][1] * g[j][1] + g[i][2] * g[j][2]);
}

void elementMass(const double p[4][3], double K[16]) {
  double J[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) J[r][c] = p[c + 1][r] - p[0][r];
  const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                     J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                     J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  const double vol = std::fabs(det) / 6.0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) K[4 * i + j] = vol * (i == j ? 2.0 : 1.0) / 20.0;
}

// Row of the assembled operator at micro-vertex P (cell-local index p of cell c): calls
// add(q, raw, scaled) for every vertex q of every micro-cell of c containing p. The weight is
// raw * k(c) when scaled (the diffusion form), else raw.
template <class F>
static void cellRow(const Topology& topo, int c, int64_t N, const int64_t p[3], FormKind form, F&& add) {
  const auto& ce = topo.cells[c];
  double V[4][3];
  for (int i = 0; i < 4; ++i)
    for (int d = 0; d < 3; ++d) V[i][d] = topo.verts[ce.v[i]].x[d];
  for (int t = 0; t < 6; ++t) {
    const int64_t width = N - kMicroCellWidthReduction[t];
    if (width <= 0) continue;
    double K[16];
    bool scaled = false;
    {
      double P[4][3];
      for (int m = 0; m < 4; ++m)
        for (int d = 0; d < 3; ++d)
          P[m][d] = V[0][d] + ((V[1][d] - V[0][d]) * kMicroCell[t][m][0] + (V[2][d] - V[0][d]) * kMicroCell[t][m][1] +
                               (V[3][d] - V[0][d]) * kMicroCell[t][m][2]) /
                                  (double)N;
      if (form == FORM_LAPLACE) {
        elementLaplace(P, K);
        scaled = true;
      } else if (form == FORM_PSPG) {
        elementLaplace(P, K);
        double a[3][3];
        for (int i = 0; i < 3; ++i)
          for (int dd = 0; dd < 3; ++dd) a[i][dd] = P[i + 1][dd] - P[0][dd];
        const double vol = std::fabs(a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
                                     a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                                     a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0])) /
                           6.0;
        const double tau = std::pow(vol, 2.0 / 3.0) / 12.0;
        for (double& k : K) k *= -tau;
      } else {
        elementMass(P, K);
      }
    }
    for (int k = 0; k < 4; ++k) {
      const int64_t i0 = p[0] - kMicroCell[t][k][0], i1 = p[1] - kMicroCell[t][k][1], i2 = p[2] - kMicroCell[t][k][2];
      if (i0 < 0 || i1 < 0 || i2 < 0 || i0 + i1 + i2 > width - 1) continue;
      for (int m = 0; m < 4; ++m) {
        const int64_t q[3] = {i0 + kMicroCell[t][m][0], i1 + kMicroCell[t][m][1], i2 + kMicroCell[t][m][2]};
        add(q, K[4 * k + m], scaled);
      }
    }
  }
}

static void cellLocal(const MacroCell& c, const Bary& p, int64_t out[3]) {
  out[0] = p.of(c.v[1]);
  out[1] = p.of(c.v[2]);
  out[2] = p.of(c.v[3]);
}

namespace {
// Accumulators of one stencil entry: the value (summed in traversal order), or the list of its
// terms in that order.
struct NumAcc {
  double v = 0.0;
  void add(const Topology& t, int cell, double raw, bool scaled) { v += scaled ? raw * t.cells[cell].k : raw; }
};
struct TermAcc {
  std::vector<PlanTerm> v;
  void add(const Topology&, int cell, double raw, bool scaled) { v.push_back({cell, scaled ? 1 : 0, raw}); }
};

template <class Acc>
struct StencilAcc {
  std::vector<std::array<Acc, 16>> cell;
  std::vector<std::vector<std::pair<std::array<int, 3>, Acc>>> face;  // diagonal first
  std::vector<std::vector<std::pair<int64_t, Acc>>> edge, vert;      // diagonal first
};

template <class Acc>
StencilAcc<Acc> assembleAcc(const Discretization& d, int L, FormKind form) {
  const Topology& topo = d.topo();
  const int64_t N = int64_t(1) << L, w = N + 1;
  StencilAcc<Acc> st;

  // cells: interior point (1,1,1) exists for N >= 4
  st.cell.resize(topo.cells.size());
  for (size_t c = 0; c < topo.cells.size(); ++c) {
    if (N < 4) continue;
    const int64_t p[3] = {1, 1, 1};
    cellRow(topo, (int)c, N, p, form, [&](const int64_t* q, double raw, bool scaled) {
      const int dx = int(q[0] - p[0]), dy = int(q[1] - p[1]), dz = int(q[2] - p[2]);
      for (int k = 0; k < 15; ++k)
        if (kCellOffsets[k][0] == dx && kCellOffsets[k][1] == dy && kCellOffsets[k][2] == dz) {
          st.cell[c][k].add(topo, (int)c, raw, scaled);
          return;
        }
      throw std::runtime_error("cell stencil offset outside the 15-point pattern");
    });
  }

  // faces: interior point (1,1) exists for N >= 3
  st.face.resize(topo.faces.size());
  for (size_t f = 0; f < topo.faces.size(); ++f) {
    if (N < 3) continue;
    const auto& fa = topo.faces[f];
    std::map<std::array<int, 3>, Acc> acc;
    acc[{0, 0, 0}];
    int64_t wts[3] = {N - 2, 1, 1};
    const Bary P = makeBary(fa.v, wts, 3);
    for (int cidx : fa.cells) {
      int64_t p[3];
      cellLocal(topo.cells[cidx], P, p);
      cellRow(topo, cidx, N, p, form, [&](const int64_t* q, double raw, bool scaled) {
        int64_t bw[4] = {N - q[0] - q[1] - q[2], q[0], q[1], q[2]};
        const Bary Q = makeBary(topo.cells[cidx].v, bw, 4);
        const int64_t s = d.localSlotOf(L, KF, (int)f, Q);
        if (s < 0) throw std::runtime_error("face stencil neighbour not stored in face array");
        int layer = 0;
        int64_t base = 0, width = w;
        if (s >= tri(w)) {
          layer = 1 + int((s - tri(w)) / tri(w - 1));
          base = tri(w) + (layer - 1) * tri(w - 1);
          width = w - 1;
        }
        const int64_t r = s - base;
        int64_t y = 0;
        while (faceIdx(width, 0, y + 1) <= r) ++y;
        const int64_t x = r - faceIdx(width, 0, y);
        acc[{layer, int(x - 1), int(y - 1)}].add(topo, cidx, raw, scaled);
      });
    }
    st.face[f].push_back({{0, 0, 0}, acc[{0, 0, 0}]});
    for (auto& kv : acc)
      if (!(kv.first[0] == 0 && kv.first[1] == 0 && kv.first[2] == 0)) st.face[f].push_back(kv);
  }

  // edges: interior point x = 1 exists for N >= 2
  auto lowRow = [&](int kind, int prim, const Bary& P, int64_t centerSlot, const std::vector<int>& cells) {
    std::map<int64_t, Acc> acc;
    acc[0];
    for (int cidx : cells) {
      int64_t p[3];
      cellLocal(topo.cells[cidx], P, p);
      cellRow(topo, cidx, N, p, form, [&](const int64_t* q, double raw, bool scaled) {
        int64_t bw[4] = {N - q[0] - q[1] - q[2], q[0], q[1], q[2]};
        const Bary Q = makeBary(topo.cells[cidx].v, bw, 4);
        const int64_t s = d.localSlotOf(L, kind, prim, Q);
        if (s < 0) throw std::runtime_error("stencil neighbour not stored in edge/vertex array");
        acc[s - centerSlot].add(topo, cidx, raw, scaled);
      });
    }
    std::vector<std::pair<int64_t, Acc>> out;
    out.push_back({0, acc[0]});
    for (auto& kv : acc)
      if (kv.first != 0) out.push_back(kv);
    return out;
  };
  st.edge.resize(topo.edges.size());
  for (size_t e = 0; e < topo.edges.size(); ++e) {
    if (N < 2) continue;
    const auto& ed = topo.edges[e];
    int64_t wts[2] = {N - 1, 1};
    st.edge[e] = lowRow(KE, (int)e, makeBary(ed.v, wts, 2), 1, ed.cells);
  }
  st.vert.resize(topo.verts.size());
  for (size_t v = 0; v < topo.verts.size(); ++v) {
    int self = (int)v;
    st.vert[v] = lowRow(KV, (int)v, makeBary(&self, &N, 1), 0, topo.verts[v].cells);
  }
  return st;
}
}  // namespace

LevelStencils assembleStencils(const Discretization& d, int L, FormKind form) {
  const StencilAcc<NumAcc> a = assembleAcc<NumAcc>(d, L, form);
  LevelStencils st;
  st.L = L;
  st.cell.resize(a.cell.size());
  for (size_t c = 0; c < a.cell.size(); ++c)
    for (int k = 0; k < 16; ++k) st.cell[c][k] = a.cell[c][k].v;
  st.face.resize(a.face.size());
  for (size_t f = 0; f < a.face.size(); ++f)
    for (auto& e : a.face[f]) st.face[f].push_back({e.second.v, e.first[0], e.first[1], e.first[2]});
  st.edge.resize(a.edge.size());
  for (size_t e = 0; e < a.edge.size(); ++e)
    for (auto& x : a.edge[e]) st.edge[e].push_back({x.second.v, x.first});
  st.vert.resize(a.vert.size());
  for (size_t v = 0; v < a.vert.size(); ++v)
    for (auto& x : a.vert[v]) st.vert[v].push_back({x.second.v, x.first});
  return st;
}

AssemblyPlan buildAssemblyPlan(const Discretization& d, int L, FormKind form) {
  const StencilAcc<TermAcc> a = assembleAcc<TermAcc>(d, L, form);
  AssemblyPlan p;
  p.L = L;
  p.first.push_back(0);
  auto target = [&](const std::vector<PlanTerm>* t) {
    if (t) p.terms.insert(p.terms.end(), t->begin(), t->end());
    p.first.push_back((int64_t)p.terms.size());
  };
  for (auto& c : a.cell)
    for (int k = 0; k < 16; ++k) target(&c[k].v);
  p.nCell = (int64_t)a.cell.size() * 16;
  for (auto& f : a.face)
    for (int k = 0; k < 16; ++k) target(k < (int)f.size() ? &f[k].second.v : nullptr);
  p.nFace = (int64_t)a.face.size() * 16;
  int64_t nLow = 0;
  for (auto& e : a.edge)
    for (auto& x : e) {
      target(&x.second.v);
      ++nLow;
    }
  for (auto& v : a.vert)
    for (auto& x : v) {
      target(&x.second.v);
      ++nLow;
    }
  p.nLow = nLow;
  return p;
}

double evaluatePlanTarget(const AssemblyPlan& p, int64_t t, const Topology& topo) {
  double v = 0.0;
  for (int64_t i = p.first[t]; i < p.first[t + 1]; ++i) {
    const PlanTerm& x = p.terms[i];
    v += x.scaled ? x.K * topo.cells[x.cell].k : x.K;
  }
  return v;
}

}  // namespace hg
