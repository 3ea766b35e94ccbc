#include "topology.hpp"

#include <algorithm>
#include <climits>
#include <cstdint>
#include <fstream>
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

static void cuboidTets(const double p0[3], const double p1[3], int nx, int ny, int nz,
                       std::vector<std::array<double, 3>>& coords, std::vector<std::array<int, 4>>& tets);

Topology meshCuboid(const double p0[3], const double p1[3], int nx, int ny, int nz) {
  std::vector<std::array<double, 3>> coords;
  std::vector<std::array<int, 4>> tets;
  cuboidTets(p0, p1, nx, ny, nz, coords, tets);
  return Topology::fromTets(coords, tets);
}

// `copies` disjoint copies of the unit cube split into k^3 sub-cubes (meshCuboid), copy i
// translated by 2i along x and its vertex IDs offset by i times the vertices of one copy. As
// fromTets orders cells, edges and faces by their vertex IDs, every kind of primitive of the
// union is the copies' own primitives, copy after copy, each in the order of a single cube.
Topology meshCuboidCopies(int k, int copies) {
  if (k <= 0 || copies <= 0) throw std::runtime_error("meshCuboidCopies: non-positive size or copies");
  const double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
  std::vector<std::array<double, 3>> c1, coords;
  std::vector<std::array<int, 4>> t1, tets;
  cuboidTets(lo, hi, k, k, k, c1, t1);
  const int nv = (int)c1.size();
  for (int i = 0; i < copies; ++i) {
    for (auto p : c1) {
      p[0] += 2.0 * i;
      coords.push_back(p);
    }
    for (auto t : t1) {
      for (int& v : t) v += i * nv;
      tets.push_back(t);
    }
  }
  return Topology::fromTets(coords, tets);
}

static void cuboidTets(const double p0[3], const double p1[3], int nx, int ny, int nz,
                       std::vector<std::array<double, 3>>& coords, std::vector<std::array<int, 4>>& tets) {
  if (nx <= 0 || ny <= 0 || nz <= 0) throw std::runtime_error("meshCuboid: non-positive subdivision");
  // MeshGenCuboid.cpp:58-80: vertices in (z, y, x) loop order
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
}

}  // namespace hg

namespace hg {

// MeshGenCubedDomain.cpp:35-40, 46-114: vertex IDs of the cube corners (and, for type 1, of
// the face-centre and cube-centre vertices numbered after all corners).
Topology meshCubedDomain(const std::vector<std::array<int, 3>>& cubesIn, int cubeType) {
  if (cubeType != 0 && cubeType != 1) throw std::runtime_error("meshCubedDomain: cube type must be 0 or 1");
  if (cubesIn.empty()) throw std::runtime_error("meshCubedDomain: no cubes");
  std::set<std::array<int, 3>> cubes(cubesIn.begin(), cubesIn.end());
  int lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
  for (const auto& c : cubes)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], c[d]);
      hi[d] = std::max(hi[d], c[d] + 1);
    }
  const int64_t ncx = hi[0] - lo[0] + 1, ncy = hi[1] - lo[1] + 1, ncz = hi[2] - lo[2] + 1;  // corner counts
  const int64_t mx = ncx - 1, my = ncy - 1, mz = ncz - 1;                                   // cube counts
  auto grid = [&](int64_t x, int64_t y, int64_t z, int64_t nx, int64_t ny) {
    return (z - lo[2]) * nx * ny + (y - lo[1]) * nx + (x - lo[0]);
  };
  const int64_t nCorner = ncx * ncy * ncz, nXY = mx * my * (mz + 1), nXZ = mx * mz * (my + 1);
  // type 1: local vertices 0..13 of a cube (z = 0: 0 1 2 3 4; z = 1/2: 5 6 7 8; z = 1: 9..13)
  static const double sub[14][3] = {{0, 0, 0},     {1, 0, 0},     {0.5, 0.5, 0}, {0, 1, 0},     {1, 1, 0},
                                    {0.5, 0, 0.5}, {0, 0.5, 0.5}, {1, 0.5, 0.5}, {0.5, 1, 0.5}, {0, 0, 1},
                                    {1, 0, 1},     {0.5, 0.5, 1}, {0, 1, 1},     {1, 1, 1}};
  auto symmId = [&](int64_t x, int64_t y, int64_t z, int local) -> int64_t {
    switch (local) {
      case 0: return grid(x, y, z, ncx, ncy);
      case 1: return grid(x + 1, y, z, ncx, ncy);
      case 3: return grid(x, y + 1, z, ncx, ncy);
      case 4: return grid(x + 1, y + 1, z, ncx, ncy);
      case 9: return grid(x, y, z + 1, ncx, ncy);
      case 10: return grid(x + 1, y, z + 1, ncx, ncy);
      case 12: return grid(x, y + 1, z + 1, ncx, ncy);
      case 13: return grid(x + 1, y + 1, z + 1, ncx, ncy);
      case 2: return nCorner + grid(x, y, z, mx, my);            // bottom face centre (xy faces)
      case 11: return nCorner + grid(x, y, z + 1, mx, my);       // top face centre
      case 5: return nCorner + nXY + grid(x, y, z, mx, my + 1);  // front (xz faces)
      case 8: return nCorner + nXY + grid(x, y + 1, z, mx, my + 1);
      case 6: return nCorner + nXY + nXZ + grid(x, y, z, mx + 1, my);  // left (yz faces)
      case 7: return nCorner + nXY + nXZ + grid(x + 1, y, z, mx + 1, my);
    }
    throw std::runtime_error("meshCubedDomain: local vertex");
  };
  // the 24 tetrahedra of a type-1 cube (MeshGenCubedDomain.cpp:244-272)
  static const int tets24[24][4] = {{0, 1, 2, 5},    {0, 3, 2, 6},    {1, 2, 4, 7},    {2, 4, 3, 8},
                                    {2, 0, 5, 6},    {2, 1, 5, 7},    {2, 3, 6, 8},    {2, 4, 7, 8},
                                    {0, 9, 5, 6},    {1, 10, 5, 7},   {3, 12, 6, 8},   {4, 13, 7, 8},
                                    {2, 5, 6, 8},    {2, 5, 7, 8},    {11, 5, 6, 8},   {11, 5, 7, 8},
                                    {11, 9, 5, 6},   {11, 10, 5, 7},  {11, 12, 6, 8},  {11, 13, 7, 8},
                                    {11, 9, 10, 5},  {11, 9, 12, 6},  {11, 10, 13, 7}, {11, 12, 13, 8}};
  // the meshCuboid split (MeshGenCuboid.cpp:86-105)
  static const int tNode[6][4] = {{4, 5, 7, 3}, {0, 3, 1, 4}, {4, 1, 5, 3}, {5, 6, 7, 2}, {1, 3, 2, 5}, {7, 2, 3, 5}};
  static const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  std::map<int64_t, std::array<double, 3>> verts;  // MeshInfo::vertices_: ID -> position
  std::vector<std::array<int64_t, 4>> cells;
  for (const auto& c : cubes) {
    if (cubeType == 0) {
      for (int t = 0; t < 6; ++t) {
        std::array<int64_t, 4> v;
        for (int m = 0; m < 4; ++m) {
          const int* o = off[tNode[t][m]];
          v[m] = grid(c[0] + o[0], c[1] + o[1], c[2] + o[2], ncx, ncy);
          verts[v[m]] = {double(c[0] + o[0]), double(c[1] + o[1]), double(c[2] + o[2])};
        }
        cells.push_back(v);
      }
    } else {
      for (int t = 0; t < 24; ++t) {
        std::array<int64_t, 4> v;
        for (int m = 0; m < 4; ++m) {
          const int l = tets24[t][m];
          v[m] = symmId(c[0], c[1], c[2], l);
          verts[v[m]] = {c[0] + sub[l][0], c[1] + sub[l][1], c[2] + sub[l][2]};
        }
        cells.push_back(v);
      }
    }
  }
  // vertices are created in ID order; the IDs map monotonically onto 0 .. n-1
  std::map<int64_t, int> index;
  std::vector<std::array<double, 3>> coords;
  for (const auto& v : verts) {
    index[v.first] = (int)coords.size();
    coords.push_back(v.second);
  }
  std::vector<std::array<int, 4>> tets;
  for (const auto& c : cells) tets.push_back({index[c[0]], index[c[1]], index[c[2]], index[c[3]]});
  return Topology::fromTets(coords, tets);
}

Topology readGmsh(const std::string& path, bool fileFlags) {
  std::ifstream in(path.c_str());
  if (!in) throw std::runtime_error("gmsh: cannot open " + path);
  auto expect = [&](const char* want) {
    std::string tok;
    if (!(in >> tok) || tok != want) throw std::runtime_error(std::string("gmsh: expected ") + want);
  };
  auto readInt = [&](const char* what) {
    int64_t v;
    if (!(in >> v)) throw std::runtime_error(std::string("gmsh: cannot read ") + what);
    return v;
  };
  expect("$MeshFormat");
  std::string version, fileType, dataSize;
  if (!(in >> version >> fileType >> dataSize)) throw std::runtime_error("gmsh: truncated $MeshFormat");
  if (version != "2.2") throw std::runtime_error("gmsh: version must be 2.2, found " + version);
  if (fileType != "0") throw std::runtime_error("gmsh: only ASCII files are read");
  expect("$EndMeshFormat");
  expect("$Nodes");
  const int64_t nNodes = readInt("node count");
  if (nNodes <= 0) throw std::runtime_error("gmsh: no nodes");
  std::map<int64_t, std::array<double, 3>> nodes;
  for (int64_t i = 0; i < nNodes; ++i) {
    const int64_t id = readInt("node id");
    std::array<double, 3> x;
    if (!(in >> x[0] >> x[1] >> x[2])) throw std::runtime_error("gmsh: cannot read node coordinates");
    nodes[id] = x;
  }
  if (nodes.size() != (size_t)nNodes) throw std::runtime_error("gmsh: duplicate node id");
  expect("$EndNodes");
  expect("$Elements");
  const int64_t nElems = readInt("element count");
  // first pass as in the reference: lines and triangles keyed by their vertex lists as written
  // (a later duplicate overwrites), tetrahedra in a map keyed the same way
  std::map<std::array<int64_t, 2>, int> lines;
  std::map<std::array<int64_t, 3>, int> tris;
  std::map<std::array<int64_t, 4>, int> tets;
  for (int64_t e = 0; e < nElems; ++e) {
    readInt("element id");
    const int64_t type = readInt("element type");
    const int64_t nTags = readInt("tag count");
    if (nTags < 0 || nTags > 64) throw std::runtime_error("gmsh: bad tag count");
    int64_t flag = 0;
    for (int64_t k = 0; k < nTags; ++k) {
      const int64_t tag = readInt("tag");
      if (k == 0) flag = tag;
    }
    auto node = [&]() {
      const int64_t id = readInt("element node");
      if (!nodes.count(id)) throw std::runtime_error("gmsh: element refers to an unknown node");
      return id;
    };
    if (type == 1) {
      std::array<int64_t, 2> v{node(), node()};
      lines[v] = (int)flag;
    } else if (type == 2) {
      std::array<int64_t, 3> v{node(), node(), node()};
      tris[v] = (int)flag;
    } else if (type == 4) {
      std::array<int64_t, 4> v{node(), node(), node(), node()};
      tets[v] = 0;
    } else if (type == 15) {
      node();
    } else {
      throw std::runtime_error("gmsh: unsupported element type " + std::to_string(type));
    }
  }
  expect("$EndElements");
  if (tets.empty()) throw std::runtime_error("gmsh: no tetrahedra");
  // vertices in ID order (MeshInfo::vertices_ is a map), renumbered monotonically
  std::map<int64_t, int> index;
  std::vector<std::array<double, 3>> coords;
  for (const auto& n : nodes) {
    index[n.first] = (int)coords.size();
    coords.push_back(n.second);
  }
  std::vector<char> used(coords.size(), 0);
  std::vector<std::array<int, 4>> cells;
  for (const auto& t : tets) {
    std::array<int, 4> c;
    for (int k = 0; k < 4; ++k) {
      c[k] = index[t.first[k]];
      used[c[k]] = 1;
    }
    cells.push_back(c);
  }
  for (size_t i = 0; i < used.size(); ++i)
    if (!used[i]) throw std::runtime_error("gmsh: a node is not a vertex of any tetrahedron");
  Topology topo = Topology::fromTets(coords, cells);
  if (fileFlags) {
    // MeshInfo::addEdge / addFace keep the first flag of each sorted vertex set: the file's lines
    // and triangles (in the order of their written vertex lists), then 0 for the others
    std::map<std::array<int, 2>, int> ef;
    std::map<std::array<int, 3>, int> ff;
    for (const auto& l : lines) {
      std::array<int, 2> k{index[l.first[0]], index[l.first[1]]};
      std::sort(k.begin(), k.end());
      if (k[0] == k[1]) throw std::runtime_error("gmsh: line of zero length");
      ef.emplace(k, l.second);
    }
    for (const auto& t : tris) {
      std::array<int, 3> k{index[t.first[0]], index[t.first[1]], index[t.first[2]]};
      std::sort(k.begin(), k.end());
      if (k[0] == k[1] || k[1] == k[2]) throw std::runtime_error("gmsh: triangle with duplicate vertices");
      ff.emplace(k, t.second);
      // the triangle's edges enter with flag 0 unless already present
      ef.emplace(std::array<int, 2>{k[0], k[1]}, 0);
      ef.emplace(std::array<int, 2>{k[1], k[2]}, 0);
      ef.emplace(std::array<int, 2>{k[0], k[2]}, 0);
    }
    for (auto& v : topo.verts) v.flag = 0;
    for (auto& c : topo.cells) c.flag = 0;
    for (auto& e : topo.edges) {
      auto it = ef.find({e.v[0], e.v[1]});
      e.flag = it == ef.end() ? 0 : it->second;
    }
    for (auto& f : topo.faces) {
      std::array<int, 3> k{f.v[0], f.v[1], f.v[2]};
      std::sort(k.begin(), k.end());
      auto it = ff.find(k);
      f.flag = it == ff.end() ? 0 : it->second;
    }
  }
  return topo;
}

void writeGmsh(const Topology& t, const std::string& path) {
  std::ofstream out(path.c_str());
  if (!out) throw std::runtime_error("gmsh: cannot write " + path);
  out.precision(17);
  out << "$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n" << t.verts.size() << "\n";
  for (size_t i = 0; i < t.verts.size(); ++i)
    out << i + 1 << " " << t.verts[i].x[0] << " " << t.verts[i].x[1] << " " << t.verts[i].x[2] << "\n";
  out << "$EndNodes\n$Elements\n";
  size_t n = t.cells.size();
  for (const auto& e : t.edges) n += e.flag != 0;
  for (const auto& f : t.faces) n += f.flag != 0;
  out << n << "\n";
  size_t id = 1;
  for (const auto& e : t.edges)
    if (e.flag != 0) out << id++ << " 1 2 " << e.flag << " " << e.flag << " " << e.v[0] + 1 << " " << e.v[1] + 1 << "\n";
  for (const auto& f : t.faces)
    if (f.flag != 0)
      out << id++ << " 2 2 " << f.flag << " " << f.flag << " " << f.v[0] + 1 << " " << f.v[1] + 1 << " " << f.v[2] + 1
          << "\n";
  for (const auto& c : t.cells)
    out << id++ << " 4 2 0 0 " << c.v[0] + 1 << " " << c.v[1] + 1 << " " << c.v[2] + 1 << " " << c.v[3] + 1 << "\n";
  out << "$EndElements\n";
  if (!out) throw std::runtime_error("gmsh: write failed for " + path);
}

}  // namespace hg
