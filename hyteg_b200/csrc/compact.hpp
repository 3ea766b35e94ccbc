// Compact coarse cycle of the P1 multigrid. The coarse end of a V-cycle (levels minL .. top:
// the smoothing, residuals, transfers and the coarse CG of GeometricMultigridSolver.hpp:136-235)
// runs as ONE launch, one block or one thread-block cluster per group of unknowns (the whole
// mesh, or each copy of a storage of disjoint copies). Each level's unknowns are held as a
// dense owner-indexed vector in device scratch, so no halo slot is ever refreshed: every
// stencil entry is resolved on the host to the index of the DoF's owner. On the coarse levels
// of the multi-launch cycle the time goes to launch latency (about ten launches per sweep of a
// level with a few thousand DoFs); here a sweep is one block- or cluster-wide barrier per colour
// group, ten at most.
//
// Order of the SOR: the same multicolour order as the multi-launch smoother (vertices; edges by
// x mod 2; faces by (x + 2y) mod 3; cells by (x + 2y + 3z) mod 4, each in the frame of the
// owning primitive). A value reached through a halo copy is the one of the sweep's start unless
// its owner lies in the closure of the updated DoF's primitive (the copies the smoother
// refreshes between its phases), exactly as the multi-launch smoother reads it.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "storage.hpp"

namespace hg {
namespace dev {

constexpr int kCompactThreads = 512;
constexpr int kCompactMaxLevels = 8;
constexpr int kCompactGroups = 9;  // colour groups after the vertices: 2 edge, 3 face, 4 cell colours

// One updated unknown: its index in the level's vector, its stencil (prim << 2 | 0 cell,
// 1 face, 2 edge, 3 vertex; edges and vertices by their index in the operator's lists of edge
// then vertex stencils) in group 0 and its off-diagonal entries [e0, e1) in stencil order.
struct CompactRow {
  int idx, wsel, e0, e1;
};

template <class T>
struct CompactLevel {
  int n;             // unknowns of one group on this level (every owned DoF, flagged or not)
  int nRows;         // flagged DoFs: SOR order, vertices first
  int nVertexRows;   // rows [0, nVertexRows) are vertices
  int nGroups;       // colour groups of rows [nVertexRows, nRows)
  int groupEnd[kCompactGroups];
  int nCgRows;       // coarsest level: the coarse CG's unknowns
  int snapBegin, snapEnd;  // the edge and face unknowns: the ones an SOR row may read as of the sweep's start
  const CompactRow* rows;
  const CompactRow* cgRows;
  const int* cols;   // entry -> unknown index; bit 31: the value of the sweep's start
  const int2* pro;   // [nRows] coarse unknowns of the prolongation into this row (y < 0: coincident)
  const int* rPtr;   // [nRows + 1] restriction into this level's rows from the level above
  const int* rIdx;   // fine unknown index; bit 31: weight 1/2 (else 1)
  StencilDev<T> st;
  int64_t x, b, r;   // offsets of the level's vectors in a group's scratch
};

template <class T>
struct CompactCycleDev {
  CompactLevel<T> lv[kCompactMaxLevels];  // levels minL .. minL + nLevels - 1
  int nLevels;
  int64_t groupStride;  // scratch elements per group
  int64_t snap;         // offset of the snapshot vector in a group's scratch
  int64_t cgStride;     // FP64 coarse-CG scratch per group (five vectors)
  const int64_t* gather;       // [groups][n(top)] owner slot of each top-level unknown
  const int64_t* scatterSlot;  // per group, every slot of the top level holding a DoF ...
  const int* scatterIdx;       // ... and the unknown it holds
  const int* scatterOff;       // [groups + 1]
  StencilDev<double> cgSt;     // FP64 stencils of the coarsest level
  int primsPerGroup[4];        // cells, faces, edges, vertices per group (0 for one group)
};

}  // namespace dev

struct CompactCycle {
  int minL = 0, top = -1, groups = 1, cluster = 1, prec = 8;
  dev::CompactCycleDev<double> d64{};
  dev::CompactCycleDev<float> d32{};
  std::vector<std::unique_ptr<DevBuf>> keep;
  DevBuf scratch, cg;
};

// Owned DoFs of level L in one group: the whole storage (groups 1) or copy 0 of `groups`
// disjoint copies.
int64_t compactGroupDofs(Storage& s, int L, int groups);

// The lists of a compact cycle over levels [minL, top] of operator `op` (whose host stencils
// give the structure; the weights are read from its device arrays at run time, so a device
// re-assembly needs no rebuild). mask: the multigrid's unknowns; cgMask: the coarse CG's.
// cluster: blocks per group (1, 2, 4 or 8).
std::unique_ptr<CompactCycle> buildCompactCycle(Storage& s, int op, int minL, int top, int groups, int cluster,
                                                int prec, unsigned mask, unsigned cgMask);

// One V(pre, post) cycle on levels minL .. top, on the storage's stream: x and b (level `top`
// buffers of the cycle's precision) are read at their owner slots (x taken as zero when xZero),
// and x is written back to every slot that holds a DoF. The coarse CG runs in FP64.
void runCompactCycle(CompactCycle& c, Storage& s, void* x, const void* b, bool xZero, int pre, int post,
                     double omega, int cgMaxIter, double cgTol);

}  // namespace hg
