// Macro-mesh topology of the B200 HyTeG hot path: macro-vertices, -edges, -faces and
// -cells with the reference's primitive ordering, neighbour lists and boundary flags.
//
// Follows (reference, by path within the project):
//   src/hyteg/mesh/MeshGenCuboid.cpp:32-171            meshCuboid (6-tet split per sub-cube)
//   src/hyteg/mesh/MeshInfo.cpp:37-72                  edge/face deduplication by sorted vertex IDs
//   src/hyteg/primitivestorage/SetupPrimitiveStorage.cpp:37-345  primitive creation order and
//                                                      neighbour lists (IDs assigned V, E, F, C)
//   src/hyteg/primitivestorage/SetupPrimitiveStorage.cpp:735-746, 850-911  boundary flags
#pragma once

#include <array>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace hg {

struct MacroVertex {
  double x[3];
  std::vector<int> edges, faces, cells;  // neighbour lists in creation (= ID) order
  int flag = 0;                          // mesh boundary flag
};

struct MacroEdge {
  int v[2];                              // sorted mesh vertex IDs
  std::vector<int> faces, cells;
  int flag = 0;
};

struct MacroFace {
  int v[3];                              // vertex order of the reference face (sorted for meshCuboid)
  int e[3];                              // edges (v0,v1), (v0,v2), (v1,v2)
  int orient[3];                         // +1 if the edge's vertex 0 is the face's first vertex of that pair
  std::vector<int> cells;
  int flag = 0;
};

struct MacroCell {
  int v[4];                              // vertex order as generated (NOT sorted): defines the cell frame
  int e[6];                              // (v0v1, v0v2, v1v2, v0v3, v1v3, v2v3)
  int f[4];                              // (v0v1v2, v0v1v3, v0v2v3, v1v2v3)
  int flag = 0;
  double k = 1.0;                        // piecewise-constant diffusion coefficient of this macro-cell
};

struct Topology {
  std::vector<MacroVertex> verts;
  std::vector<MacroEdge> edges;
  std::vector<MacroFace> faces;
  std::vector<MacroCell> cells;
  std::map<std::array<int, 2>, int> edgeByVerts;  // sorted vertex pair -> edge index
  std::map<std::array<int, 3>, int> faceByVerts;  // sorted vertex triple -> face index

  int edgeOf(int a, int b) const;
  int faceOf(int a, int b, int c) const;
  // Builds the storage from an explicit tetrahedral mesh (vertex coordinates and, per cell,
  // four vertex IDs in the cell's frame order), reproducing SetupPrimitiveStorage's ordering.
  static Topology fromTets(const std::vector<std::array<double, 3>>& coords,
                           const std::vector<std::array<int, 4>>& tets);
  // setMeshBoundaryFlagsOnBoundary(onBoundary, inner, highestDimensionAlwaysInner = true)
  void setBoundaryFlags(int onBoundary, int inner);
};

// MeshInfo::meshCuboid(p0, p1, nx, ny, nz) followed by SetupPrimitiveStorage.
Topology meshCuboid(const double p0[3], const double p1[3], int nx, int ny, int nz);
// `copies` disjoint translated copies of meshCuboid((0,0,0), (1,1,1), k, k, k) in one macro-mesh;
// each kind of primitive holds the copies' primitives copy after copy, in a single cube's order.
Topology meshCuboidCopies(int k, int copies);

// MeshInfo::meshCubedDomain(cubeCoordinates, cubeType) followed by SetupPrimitiveStorage
// (src/hyteg/mesh/MeshGenCubedDomain.cpp:115-383): unit cubes at the given integer positions,
// 6 tetrahedra per cube (type 0, the meshCuboid split) or 24 (type 1, with face-centre and cube
// centre vertices).
Topology meshCubedDomain(const std::vector<std::array<int, 3>>& cubes, int cubeType);

// MeshInfo::fromGmshFile (src/hyteg/mesh/MeshGenFromGmshFile.cpp:31-206): a Gmsh 2.2 ASCII
// file with nodes, lines (type 1), triangles (2), tetrahedra (4) and points (15). With
// fileFlags the first tag of every line and triangle becomes the boundary flag of that edge or
// face (all other primitives 0), as MeshInfo keeps them; otherwise the flags are left for
// setBoundaryFlags. Throws std::runtime_error on a malformed file.
Topology readGmsh(const std::string& path, bool fileFlags);
// The inverse, as the wire format of a macro-mesh: nodes in vertex order (IDs from 1),
// flagged edges and faces as lines and triangles (two tags, the flag twice), then the cells in
// frame order. readGmsh(writeGmsh(t), fileFlags) reproduces t's primitives and their order; with
// fileFlags the edge and face flags too (vertex flags read as 0: points carry none).
void writeGmsh(const Topology& t, const std::string& path);

}  // namespace hg
