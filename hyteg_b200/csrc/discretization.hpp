// Per-level data layout, halo (ghost/closure) tables and constant stencils of the P1
// vertex-DoF space on uniformly refined macro-tetrahedra.
//
// Layout: every macro-primitive owns one array per level exactly as in the reference
//   vertex : 1 + #edges                               (VertexDoFMemory.hpp:44-47)
//   edge   : w + #faces (w-1) + #cells (w-2)          (VertexDoFMemory.hpp:49-57)
//   face   : tri(w) + #cells tri(w-1)                 (VertexDoFMemory.hpp:59-63)
//   cell   : tet(w)                                   (VertexDoFMemory.hpp:65-69)
// with w = 2^L + 1 and the reference index functions
//   cell   idx(x,y,z)  (indexing/MacroCellIndexing.hpp:40-52)
//   face   idx(x,y) and ghost layer n (p1functionspace/VertexDoFIndexing.cpp:205-225)
//   edge   ghost layers (p1functionspace/VertexDoFIndexing.cpp:58-72).
// All arrays of one function and level live in one device buffer: cells first (each
// cell array 256-byte aligned), then faces, edges and vertices, each in ID order.
//
// Every slot of every array is identified by integer barycentric coordinates with respect
// to the macro-vertices (sum = 2^L). The primitive spanned by the non-zero coordinates owns
// the DoF; every other slot holding it is a copy that the halo exchange refreshes from the
// owner. This reproduces the six-direction communicate() of the reference
// (P1Operator.hpp:206-212, VertexDoFPackInfo.hpp:118-563) as gathers from owner slots.
#pragma once

#include <array>
#include <cstdint>
#include <map>
#include <vector>

#include "topology.hpp"

namespace hg {

enum Kind { KV = 0, KE = 1, KF = 2, KC = 3 };
enum CommGroup { G_VERT = 0, G_EDGE = 1, G_FACE_BOUNDARY = 2, G_FACE_GHOST = 3, G_CELL = 4, G_COUNT = 5 };

inline int64_t tri(int64_t w) { return w * (w + 1) / 2; }
inline int64_t tet(int64_t w) { return w * (w + 1) * (w + 2) / 6; }
inline int64_t faceIdx(int64_t w, int64_t x, int64_t y) { return y * (w + 1) - y * (y + 1) / 2 + x; }
inline int64_t cellIdx(int64_t w, int64_t x, int64_t y, int64_t z) {
  const int64_t W = w - z;
  return tet(w) - tet(W) + y * (W + 1) - y * (y + 1) / 2 + x;
}

// A micro-vertex: up to four (macro-vertex, weight) pairs, weights > 0, sorted by vertex.
struct Bary {
  int n = 0;
  int v[4];
  int64_t b[4];
  int64_t of(int vert) const {
    for (int i = 0; i < n; ++i)
      if (v[i] == vert) return b[i];
    return 0;
  }
};
Bary makeBary(const int* verts, const int64_t* weights, int count);

struct Slot {
  int kind = -1;
  int prim = -1;
  int64_t local = -1;
};

// Per-level geometry of the arrays of one function.
struct LevelLayout {
  int L = 0;
  int64_t N = 1, w = 2;
  std::vector<int64_t> off[4], size[4];
  int64_t total = 0;
  // Halo tables: copy slots and the owner slot each is refreshed from (absolute element
  // indices into the level buffer), in five groups by destination: vertex ghosts, edge
  // copies, face boundary rows, face ghost layers, cell closures.
  std::vector<int64_t> commDst[5], commSrc[5];
};

class Discretization {
 public:
  Discretization(const Topology& topo, int maxLevel);
  const Topology& topo() const { return topo_; }
  const LevelLayout& level(int L) const { return levels_.at(L); }
  int maxLevel() const { return (int)levels_.size() - 1; }

  Bary slotBary(int L, int kind, int prim, int64_t local) const;  // identity of a slot
  Slot owner(int L, const Bary& p) const;                         // owner slot of a DoF
  // Slot inside primitive (kind, prim)'s own array that holds p, or -1 if not stored there.
  int64_t localSlotOf(int L, int kind, int prim, const Bary& p) const;
  int cellOf(const int* sortedVerts4) const;
  int64_t ownedCount(int L, int kind) const;  // owned DoFs per primitive of that kind

 private:
  void buildLevel(int L);
  Topology topo_;
  std::vector<LevelLayout> levels_;
  std::map<std::array<int, 4>, int> cellByVerts_;
};

// The owned DoFs of level L (every DoF exactly once) in level-buffer order, as runs of
// consecutive slots of their owning primitives: per cell its interior rows (x, y, z >= 1,
// x + y + z <= N - 1), per face the interior rows of its own triangle, per edge its interior
// points, per vertex its own slot.
struct SlotRun {
  int64_t slot, len;
};
std::vector<SlotRun> ownedRuns(const Discretization& d, int L);

// ---------------------------------------------------------------------------------------
// Constant stencils. The element matrix of every micro-tetrahedron is accumulated into the
// rows of the owned DoFs (P1Elements.hpp:430-496, P1ConstantOperator.cpp:543-595); entries
// are kept for every structural neighbour, also when their weight is zero.
// ---------------------------------------------------------------------------------------
// FORM_PSPG: the pressure stabilisation form -tau grad p . grad q with tau = |T|^(2/3) / 12 of
// each micro-cell T (P1PSPGOperator; its inverse diagonal scales the pressure update of the
// Uzawa smoother). Cell coefficients do not enter it.
enum FormKind { FORM_LAPLACE = 0, FORM_MASS = 1, FORM_PSPG = 2 };

// The fifteen cell-stencil offsets in the fixed order used by the device kernels:
// C, E, W, N, S, NW, SE, TC, TW, TS, TSE, BC, BE, BN, BNW
// (the offsets of apply_3D_macrocell_vertexdof_to_vertexdof_replace.cpp:34-48).
extern const int kCellOffsets[15][3];

struct FaceEntry {  // weight of the value at (x+dx, y+dy) of layer (0: face, 1+n: ghost layer n)
  double w;
  int layer, dx, dy;
};
struct LowEntry {  // weight of the value at slot (x + rel) of an edge / vertex array
  double w;
  int64_t rel;
};

struct LevelStencils {
  int L = 0;
  std::vector<std::array<double, 16>> cell;       // [cell][15] (slot 15 unused)
  std::vector<std::vector<FaceEntry>> face;       // [face] entries, diagonal first
  std::vector<std::vector<LowEntry>> edge, vert;  // [prim] entries, diagonal first
};

// 4x4 element matrices (row-major) on the tetrahedron with the given vertex coordinates.
void elementLaplace(const double p[4][3], double K[16]);
void elementMass(const double p[4][3], double K[16]);

LevelStencils assembleStencils(const Discretization& d, int L, FormKind form);

// The same stencils as sums of element-matrix terms, for re-assembly with new cell coefficients
// on the device: every entry is sum_i (scaled_i ? K_i * k(cell_i) : K_i), summed in the order of
// the terms, which is the order assembleStencils adds them in (so both give the same bits).
// Targets follow the device arrays: [cells][16], then [faces][16] (the face entries, zeros
// beyond them), then the edge entries and the vertex entries, each primitive's diagonal first.
struct PlanTerm {
  int cell;
  int scaled;  // 1: multiplied by the cell's coefficient (diffusion form)
  double K;
};
struct AssemblyPlan {
  int L = 0;
  std::vector<int64_t> first;  // [targets + 1]: term range of each target
  std::vector<PlanTerm> terms;
  int64_t nCell = 0, nFace = 0, nLow = 0;
};
AssemblyPlan buildAssemblyPlan(const Discretization& d, int L, FormKind form);
// One target of a plan evaluated on the host with the topology's current coefficients.
double evaluatePlanTarget(const AssemblyPlan& p, int64_t t, const Topology& topo);

// P2 (quadratic) space of level L, stored as the vertex-DoF lattice of level L + 1: the
// micro-vertices of level L sit at even coordinates, the midpoints of its micro-edges at the
// seven other parity classes (the reference's X, Y, Z, XY, XZ, YZ, XYZ edge orientations,
// edgedofspace/EdgeDoFOrientation.hpp:29-39). Local nodes of a micro-tetrahedron: its four
// vertices, then the midpoints of the edges (0,1),(0,2),(0,3),(1,2),(1,3),(2,3).
extern const int kP2Edge[6][2];
extern const int kMicroCellTable[6][4][3];
extern const int kMicroCellWidth[6];
// P2 Laplace element matrix (10 x 10, row major) from the barycentric moments
// int lambda_a lambda_b = |T| (1 + delta_ab) / 20 (p2_tet_diffusion of the reference's forms).
void elementP2Laplace(const double p[4][3], double K[100]);
// Element matrices of the six micro-cell types of level L in every macro-cell, scaled by the
// cell's coefficient: [cell][type][10][10].
std::vector<double> p2CellElements(const Topology& topo, int L);
// Taylor-Hood divergence element (P2ToP1ConstantDivOperator, p2_to_p1_tet_div_tet of the
// reference's forms): D[k][4 i + ...] = -int psi_i d(phi_j)/dx_k for P1 vertex i and P2 node j,
// stored as D[k][10 i + j]; the gradient block (P1ToP2ConstantDivTOperator) is its transpose.
void elementP2P1Div(const double p[4][3], double D[3][40]);
// [cell][type][3][40] for the six micro-cell types of level L.
std::vector<double> p2p1CellDiv(const Topology& topo, int L);

}  // namespace hg
