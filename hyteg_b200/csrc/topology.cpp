#include "topology.hpp"

#include <algorithm>
#include <set>
#include <stdexcept>

namespace hg {

int Topology::edgeOf(int a, int b) const {
  std::array<int, 2> k{std::min(a, b), std::max(a, b)};
  auto it = edgeByVerts.find(k);
  if (it == edgeByVerts.end()) throw std::runtime_error("edge not found");
  return it->second;
}

int Topology::faceOf(int a, int b, int c) const {
  std::array<int, 3> k{a, b, c};
  std::sort(k.begin(), k.end());
  auto it = faceByVerts.find(k);
  if (it == faceByVerts.end()) throw std::runtime_error("face not found");
  return it->second;
}

Topology Topology::fromTets(const std::vector<std::array<double, 3>>& coords,
                            const std::vector<std::array<int, 4>>& tetsIn) {
  Topology t;
  // MeshInfo keeps cells in a std::map keyed by the (unsorted) vertex-ID vector, so the
  // creation order is the lexicographic order of those vectors (MeshGenCuboid.cpp:133).
  std::vector<std::array<int, 4>> tets = tetsIn;
  std::sort(tets.begin(), tets.end());
  tets.erase(std::unique(tets.begin(), tets.end()), tets.end());

  // Edges and faces are deduplicated by sorted vertex IDs (MeshInfo.cpp:37-72) and kept in
  // std::maps, so their creation order is the sorted order of the keys.
  std::set<std::array<int, 2>> edgeKeys;
  std::set<std::array<int, 3>> faceKeys;
  for (const auto& c : tets) {
    const int pairs[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
    for (auto& p : pairs) edgeKeys.insert({std::min(c[p[0]], c[p[1]]), std::max(c[p[0]], c[p[1]])});
    const int tris[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    for (auto& q : tris) {
      std::array<int, 3> k{c[q[0]], c[q[1]], c[q[2]]};
      std::sort(k.begin(), k.end());
      faceKeys.insert(k);
    }
  }

  t.verts.resize(coords.size());
  for (size_t i = 0; i < coords.size(); ++i)
    for (int d = 0; d < 3; ++d) t.verts[i].x[d] = coords[i][d];

  for (const auto& k : edgeKeys) {
    int id = (int)t.edges.size();
    MacroEdge e;
    e.v[0] = k[0];
    e.v[1] = k[1];
    t.edges.push_back(e);
    t.edgeByVerts[k] = id;
    t.verts[k[0]].edges.push_back(id);
    t.verts[k[1]].edges.push_back(id);
  }

  // SetupPrimitiveStorage.cpp:113-223: the face's vertex order follows its edges' orientation;
  // with sorted keys the face vertices are (v0 < v1 < v2) and all orientations are +1.
  for (const auto& k : faceKeys) {
    int id = (int)t.faces.size();
    MacroFace f;
    int e0 = t.edgeOf(k[0], k[1]), e1 = t.edgeOf(k[0], k[2]), e2 = t.edgeOf(k[1], k[2]);
    f.e[0] = e0;
    f.e[1] = e1;
    f.e[2] = e2;
    f.orient[0] = (t.edges[e0].v[0] == k[0]) ? 1 : -1;
    f.orient[1] = (t.edges[e1].v[0] == k[0]) ? 1 : -1;
    f.orient[2] = (t.edges[e2].v[0] == k[1]) ? 1 : -1;
    f.v[0] = f.orient[0] == 1 ? t.edges[e0].v[0] : t.edges[e0].v[1];
    f.v[1] = f.orient[0] == 1 ? t.edges[e0].v[1] : t.edges[e0].v[0];
    f.v[2] = f.orient[1] == 1 ? t.edges[e1].v[1] : t.edges[e1].v[0];
    t.faces.push_back(f);
    t.faceByVerts[k] = id;
    for (int i = 0; i < 3; ++i) t.verts[f.v[i]].faces.push_back(id);
    for (int i = 0; i < 3; ++i) t.edges[f.e[i]].faces.push_back(id);
  }

  // SetupPrimitiveStorage.cpp:226-345
  for (const auto& c : tets) {
    int id = (int)t.cells.size();
    MacroCell m;
    for (int i = 0; i < 4; ++i) m.v[i] = c[i];
    m.e[0] = t.edgeOf(c[0], c[1]);
    m.e[1] = t.edgeOf(c[0], c[2]);
    m.e[2] = t.edgeOf(c[1], c[2]);
    m.e[3] = t.edgeOf(c[0], c[3]);
    m.e[4] = t.edgeOf(c[1], c[3]);
    m.e[5] = t.edgeOf(c[2], c[3]);
    m.f[0] = t.faceOf(c[0], c[1], c[2]);
    m.f[1] = t.faceOf(c[0], c[1], c[3]);
    m.f[2] = t.faceOf(c[0], c[2], c[3]);
    m.f[3] = t.faceOf(c[1], c[2], c[3]);
    t.cells.push_back(m);
    for (int i = 0; i < 4; ++i) t.verts[c[i]].cells.push_back(id);
    for (int i = 0; i < 6; ++i) t.edges[m.e[i]].cells.push_back(id);
    for (int i = 0; i < 4; ++i) t.faces[m.f[i]].cells.push_back(id);
  }
  for (auto& f : t.faces)
    if (f.cells.empty() || f.cells.size() > 2) throw std::runtime_error("non-manifold tetrahedral mesh");
  return t;
}

void Topology::setBoundaryFlags(int onBoundary, int inner) {
  // SetupPrimitiveStorage::onBoundary (3-D branch): a face is on the boundary iff it has
  // one neighbour cell; an edge or vertex iff one of its neighbour faces is; cells are
  // always inner (highestDimensionAlwaysInner).
  std::vector<char> fb(faces.size());
  for (size_t i = 0; i < faces.size(); ++i) {
    fb[i] = faces[i].cells.size() == 1;
    faces[i].flag = fb[i] ? onBoundary : inner;
  }
  for (auto& e : edges) {
    bool b = false;
    for (int f : e.faces) b = b || fb[f];
    e.flag = b ? onBoundary : inner;
  }
  for (auto& v : verts) {
    bool b = false;
    for (int f : v.faces) b = b || fb[f];
    v.flag = b ? onBoundary : inner;
  }
  for (auto& c : cells) c.flag = inner;
}

Topology meshCuboid(const double p0[3], const double p1[3], int nx, int ny, int nz) {
  if (nx <= 0 || ny <= 0 || nz <= 0) throw std::runtime_error("meshCuboid: non-positive subdivision");
  // MeshGenCuboid.cpp:58-80: vertices in (z, y, x) loop order
  std::vector<std::array<double, 3>> coords;
  const double hx = (p1[0] - p0[0]) / nx, hy = (p1[1] - p0[1]) / ny, hz = (p1[2] - p0[2]) / nz;
  for (int iz = 0; iz <= nz; ++iz)
    for (int iy = 0; iy <= ny; ++iy)
      for (int ix = 0; ix <= nx; ++ix)
        coords.push_back({p0[0] + ix * hx, p0[1] + iy * hy, p0[2] + iz * hz});
  // MeshGenCuboid.cpp:86-92 (tet-to-hexahedron-vertex table) and :97-105 (hexahedron corners)
  static const int tNode[6][4] = {{4, 5, 7, 3}, {0, 3, 1, 4}, {4, 1, 5, 3},
                                  {5, 6, 7, 2}, {1, 3, 2, 5}, {7, 2, 3, 5}};
  static const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  auto vid = [&](int i, int j, int k) { return k * (nx + 1) * (ny + 1) + j * (nx + 1) + i; };
  std::vector<std::array<int, 4>> tets;
  for (int iz = 0; iz < nz; ++iz)
    for (int iy = 0; iy < ny; ++iy)
      for (int ix = 0; ix < nx; ++ix)
        for (int t = 0; t < 6; ++t) {
          std::array<int, 4> c;
          for (int m = 0; m < 4; ++m) {
            const int* o = off[tNode[t][m]];
            c[m] = vid(ix + o[0], iy + o[1], iz + o[2]);
          }
          tets.push_back(c);
        }
  return Topology::fromTets(coords, tets);
}

}  // namespace hg
