// Compact coarse cycle of the P1 multigrid: host-side construction of the owner-indexed lists
// and the single-launch V-cycle kernel (one block, or one cluster of blocks, per group).
#include <cooperative_groups.h>

#include <algorithm>
#include <array>
#include <cstring>
#include <tuple>

#include "../../include/hyteg_b200.h"
#include "compact.hpp"
#include "discretization.hpp"

namespace hg {
namespace dev {

// Weights of a row's stencil in the operator's device arrays: entry k at w[k * stride], the
// diagonal at k = 0 (cells: kCellOffsets order; faces: FaceEnt records; edges and vertices:
// their entry list). The rows name group 0's primitives; group g's are shifted by g times the
// primitives of each kind per group (sh: cells, faces, edges, vertices), since every copy of a
// storage of copies has its own stencils.
template <class T>
__device__ __forceinline__ const T* compactStencil(const StencilDev<T>& st, int wsel, int4 sh, int& stride) {
  const int kind = wsel & 3, prim = wsel >> 2;
  if (kind == 0) {
    stride = 1;
    return st.cellW + 16 * (prim + sh.x);
  }
  if (kind == 1) {
    stride = int(sizeof(FaceEnt<T>) / sizeof(T));
    return &st.faceEnt[16 * (prim + sh.y)].w;
  }
  stride = 1;
  return st.lowEntW + st.lowEntOff[prim + (kind == 2 ? sh.z : sh.w)];
}

// Values of a row's entries [e, min(e + 16, e1)), all loads issued before any is used: from snap
// where bit 31 of the entry is set (SNAP), else from x.
template <class T, bool SNAP>
__device__ __forceinline__ void compactValues(const int* __restrict__ cols, int e, int e1, const T* x, const T* snap,
                                              T (&v)[16]) {
  int c[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) c[j] = e + j < e1 ? __ldg(cols + e + j) : 0;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int cj = c[j];
    v[j] = e + j < e1 ? ((SNAP && cj < 0) ? snap[cj & 0x7fffffff] : x[cj & 0x7fffffff]) : T(0);
  }
}

// s - sum_k w_k v_k (SUB) or s + sum_k w_k v_k over a row's off-diagonal entries, in entry order.
template <class T, bool SNAP, bool SUB>
__device__ __forceinline__ T compactRowSum(T s, const T* w, int stride, const int* __restrict__ cols, int e0, int e1,
                                           const T* x, const T* snap) {
  for (int e = e0; e < e1; e += 16) {
    T v[16];
    compactValues<T, SNAP>(cols, e, e1, x, snap, v);
    const T* wk = w + (1 + e - e0) * stride;
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (e + j < e1) {
        if (SUB)
          s -= wk[j * stride] * v[j];
        else
          s += wk[j * stride] * v[j];
      }
  }
  return s;
}

// Grid: groups * CL blocks of kCompactThreads, clusters of CL consecutive blocks; cluster g works
// on group g. Every loop of the kernel has the same trip count in all threads of a cluster, so
// every thread reaches every barrier.
template <class T, int CL>
__global__ void __launch_bounds__(kCompactThreads, 1) compactCycleKernel(const __grid_constant__ CompactCycleDev<T> cd,
                                                                      T* xs, const T* __restrict__ bs, T* scratch,
                                                                      double* cgScratch, int xZero, int pre, int post,
                                                                      T omega, int cgMaxIter, double cgTol) {
  namespace cgrp = cooperative_groups;
  __shared__ double red[33];
  __shared__ double part[2];
  int rank = 0;
  if constexpr (CL > 1) rank = (int)cgrp::this_cluster().block_rank();
  const int grp = blockIdx.x / CL;
  const int t0 = rank * (int)blockDim.x + (int)threadIdx.x, nt = CL * (int)blockDim.x;
  auto sync = [&]() {
    if constexpr (CL == 1)
      __syncthreads();
    else
      cgrp::this_cluster().sync();
  };
  T* sc = scratch + grp * cd.groupStride;
  T* snap = sc + cd.snap;
  const int4 sh = make_int4(grp * cd.primsPerGroup[0], grp * cd.primsPerGroup[1], grp * cd.primsPerGroup[2],
                            grp * cd.primsPerGroup[3]);
  const T om1 = T(1) - omega;
  const int K = cd.nLevels - 1;

  // top level: x and b from their owner slots
  {
    const CompactLevel<T>& L = cd.lv[K];
    const int64_t* g = cd.gather + (int64_t)grp * L.n;
    for (int i = t0; i < L.n; i += nt) {
      sc[L.x + i] = xZero ? T(0) : xs[g[i]];
      sc[L.b + i] = bs[g[i]];
    }
  }
  sync();

  // x_i <- (1 - omega) x_i + omega (b_i - sum_j a_ij x_j) / a_ii, the lowSorPhaseKernel update
  auto sorRow = [&](const CompactLevel<T>& L, const CompactRow row, T* x, const T* b) {
    int stride;
    const T* w = compactStencil(L.st, row.wsel, sh, stride);
    const T s = compactRowSum<T, true, true>(b[row.idx], w, stride, L.cols, row.e0, row.e1, x, snap);
    x[row.idx] = om1 * x[row.idx] + (s * omega) / w[0];
  };
  // Sweeps. The vertex rows update while the edge and face values are saved: they write only
  // vertex values, and they read edge and face values from x, which this sweep has not changed
  // yet; only edge and face rows read the saved values. Then one barrier per colour group.
  auto sweeps = [&](const CompactLevel<T>& L, int count) {
    T* x = sc + L.x;
    const T* b = sc + L.b;
    for (int it = 0; it < count; ++it) {
      for (int i = L.snapBegin + t0; i < L.snapEnd; i += nt) snap[i] = x[i];
      for (int r = t0; r < L.nVertexRows; r += nt) sorRow(L, L.rows[r], x, b);
      sync();
      int r0 = L.nVertexRows;
      for (int gi = 0; gi < L.nGroups; ++gi) {
        const int r1 = L.groupEnd[gi];
        for (int r = r0 + t0; r < r1; r += nt) sorRow(L, L.rows[r], x, b);
        r0 = r1;
        sync();
      }
    }
  };
  // (A u)_row with every value current
  auto applyRow = [&](const StencilDev<T>& st, const int* cols, const CompactRow row, const T* u) {
    int stride;
    const T* w = compactStencil(st, row.wsel, sh, stride);
    return compactRowSum<T, false, false>(w[0] * u[row.idx], w, stride, cols, row.e0, row.e1, u, u);
  };

  // descent: pre-smoothing, residual, restriction into the coarser right-hand side
  for (int k = K; k > 0; --k) {
    const CompactLevel<T>& F = cd.lv[k];
    const CompactLevel<T>& C = cd.lv[k - 1];
    sweeps(F, pre);
    T* xf = sc + F.x;
    const T* bf = sc + F.b;
    T* rf = sc + F.r;
    for (int r = t0; r < F.nRows; r += nt) {
      const CompactRow row = F.rows[r];
      rf[row.idx] = bf[row.idx] - applyRow(F.st, F.cols, row, xf);
    }
    sync();
    T* xc = sc + C.x;
    T* bc = sc + C.b;
    for (int r = t0; r < C.nRows; r += nt) {
      T s = T(0);
      for (int e = C.rPtr[r]; e < C.rPtr[r + 1]; ++e) {
        const int c = C.rIdx[e];
        const T v = rf[c & 0x7fffffff];
        s += c < 0 ? T(0.5) * v : v;
      }
      bc[C.rows[r].idx] = s;
    }
    for (int i = t0; i < C.n; i += nt) xc[i] = T(0);
    sync();
  }

  // coarsest level: CG with the identity preconditioner (CGSolver.hpp:69-150) in FP64
  {
    const CompactLevel<T>& C = cd.lv[0];
    double* cx = cgScratch + grp * cd.cgStride;
    double* cb = cx + C.n;
    double* cr = cb + C.n;
    double* cp = cr + C.n;
    double* cap = cp + C.n;
    T* x0 = sc + C.x;
    const T* b0 = sc + C.b;
    int par = 0;
    auto dot = [&](const double* u, const double* v) {
      double s = 0;
      for (int r = t0; r < C.nCgRows; r += nt) {
        const int i = C.cgRows[r].idx;
        s += u[i] * v[i];
      }
      const double c = blockSum(s, red);
      if constexpr (CL == 1) {
        return c;
      } else {
        // the blocks' sums in rank order, the same total in every block
        if (threadIdx.x == 0) part[par] = c;
        cgrp::cluster_group cl = cgrp::this_cluster();
        cl.sync();
        double t = 0;
        for (int q = 0; q < CL; ++q) t += *cl.map_shared_rank(&part[par], q);
        par ^= 1;  // the next sum goes to the other slot: no block overwrites one still being read
        return t;
      }
    };
    auto applyCg = [&](const CompactRow row, const double* u) {
      int stride;
      const double* w = compactStencil(cd.cgSt, row.wsel, sh, stride);
      return compactRowSum<double, false, false>(w[0] * u[row.idx], w, stride, C.cols, row.e0, row.e1, u, u);
    };
    for (int i = t0; i < C.n; i += nt) {
      cx[i] = double(x0[i]);
      cb[i] = double(b0[i]);
      cp[i] = 0.0;
    }
    sync();
    for (int r = t0; r < C.nCgRows; r += nt) {
      const CompactRow row = C.cgRows[r];
      cr[row.idx] = cb[row.idx] - applyCg(row, cx);
      cp[row.idx] = cr[row.idx];
    }
    sync();
    double prsold = dot(cr, cr);
    double res = sqrt(prsold);
    if (res >= cgTol) {
      for (int it = 0; it < cgMaxIter; ++it) {
        for (int r = t0; r < C.nCgRows; r += nt) {
          const CompactRow row = C.cgRows[r];
          cap[row.idx] = applyCg(row, cp);
        }
        const double alpha = prsold / dot(cp, cap);
        for (int r = t0; r < C.nCgRows; r += nt) {
          const int i = C.cgRows[r].idx;
          cx[i] += alpha * cp[i];
          cr[i] -= alpha * cap[i];
        }
        const double rsnew = dot(cr, cr);
        res = sqrt(rsnew);
        if (res < cgTol) break;
        const double beta = rsnew / prsold;
        for (int r = t0; r < C.nCgRows; r += nt) {
          const int i = C.cgRows[r].idx;
          cp[i] = cr[i] + beta * cp[i];
        }
        sync();
        prsold = rsnew;
      }
    }
    for (int i = t0; i < C.n; i += nt) x0[i] = T(cx[i]);
    sync();
  }

  // ascent: prolongation added to the flagged unknowns, post-smoothing
  for (int k = 1; k <= K; ++k) {
    const CompactLevel<T>& F = cd.lv[k];
    const T* xc = sc + cd.lv[k - 1].x;
    T* xf = sc + F.x;
    for (int r = t0; r < F.nRows; r += nt) {
      const int2 p = F.pro[r];
      const T v = p.y < 0 ? xc[p.x] : T(0.5) * (xc[p.x] + xc[p.y]);
      xf[F.rows[r].idx] += v;
    }
    sync();
    sweeps(F, post);
  }

  // x back to every slot of the top level that holds a DoF
  {
    const T* xt = sc + cd.lv[K].x;
    for (int e = cd.scatterOff[grp] + t0; e < cd.scatterOff[grp + 1]; e += nt) xs[cd.scatterSlot[e]] = xt[cd.scatterIdx[e]];
  }
  if constexpr (CL > 1) sync();  // no block leaves while another may still read its shared memory
}

}  // namespace dev

namespace {

int batchKind(int kind) { return kind == KC ? 0 : kind == KF ? 1 : kind == KE ? 2 : 3; }

// Directions of the coarse micro-edge a fine point bisects, by the parity code x | y << 1 | z << 2
// of its cell-local coordinates (the convention of cellProlongKernel).
const int kBisectDir[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {-1, 1, 0}, {0, 0, 1}, {-1, 0, 1}, {0, -1, 1}, {-1, 1, -1}};

struct Dof {
  int kind, prim, colour;
  int64_t local;
  int x, y, z;
  int64_t slot;  // absolute owner slot
  unsigned char type;
};

void primVerts(const Topology& t, int kind, int prim, int* v, int& n) {
  if (kind == KV) {
    v[0] = prim;
    n = 1;
  } else if (kind == KE) {
    n = 2;
    for (int i = 0; i < 2; ++i) v[i] = t.edges[(size_t)prim].v[i];
  } else if (kind == KF) {
    n = 3;
    for (int i = 0; i < 3; ++i) v[i] = t.faces[(size_t)prim].v[i];
  } else {
    n = 4;
    for (int i = 0; i < 4; ++i) v[i] = t.cells[(size_t)prim].v[i];
  }
}

// Is primitive (ki, pi) a sub-primitive of (or equal to) primitive (ko, po)?
bool inClosure(const Topology& t, int ki, int pi, int ko, int po) {
  int a[4], b[4], na, nb;
  primVerts(t, ki, pi, a, na);
  primVerts(t, ko, po, b, nb);
  for (int i = 0; i < na; ++i) {
    bool found = false;
    for (int j = 0; j < nb; ++j) found = found || a[i] == b[j];
    if (!found) return false;
  }
  return true;
}

// The slots of group 0: the whole storage (groups 1) or copy 0 of the copies.
struct GroupSel {
  int groups = 1;
  dev::BatchMap bm{};
  bool inGroup0(int kind, int64_t slot) const {
    if (groups == 1) return true;
    const int q = batchKind(kind);
    return slot >= bm.uBase[q] && slot < bm.uBase[q] + bm.size[q];
  }
  int64_t shift(int kind, int g) const { return groups == 1 ? 0 : (int64_t)g * bm.size[batchKind(kind)]; }
};

struct LevelBuild {
  int L = 0;
  std::vector<Dof> dofs;          // unknowns in SOR order
  std::vector<int> unknownOf;     // absolute owner slot -> unknown (group 0), -1 elsewhere
  std::vector<int> rowOf;         // unknown -> row, -1
  std::vector<dev::CompactRow> rows, cgRows;
  std::vector<int> cols;
  int nVertexRows = 0;
  std::vector<int> groupEnd;
  int snapBegin = 0, snapEnd = 0;
  std::vector<int2> pro;
  std::vector<int> rPtr, rIdx;
};

LevelBuild buildLevel(Storage& s, const LevelStencils& hs, int L, const GroupSel& sel, unsigned mask, unsigned cgMask,
                      bool coarsest) {
  const Discretization& D = s.disc;
  const Topology& topo = D.topo();
  const LevelLayout& lay = *s.levels[(size_t)L].lay;
  const LevelData& ld = s.levels[(size_t)L];
  const int64_t N = int64_t(1) << L, w = N + 1;
  const int nE = (int)topo.edges.size();
  LevelBuild lb;
  lb.L = L;
  auto& dofs = lb.dofs;
  for (size_t v = 0; v < topo.verts.size(); ++v)
    if (sel.inGroup0(KV, lay.off[KV][v]))
      dofs.push_back({KV, (int)v, 0, 0, 0, 0, 0, lay.off[KV][v], ld.hostLowType[(size_t)nE + v]});
  for (int e = 0; e < nE; ++e)
    if (sel.inGroup0(KE, lay.off[KE][(size_t)e]))
      for (int64_t x = 1; x <= N - 1; ++x)
        dofs.push_back({KE, e, int(x & 1), x, (int)x, 0, 0, lay.off[KE][(size_t)e] + x, ld.hostLowType[(size_t)e]});
  for (size_t f = 0; f < topo.faces.size(); ++f)
    if (sel.inGroup0(KF, lay.off[KF][f]))
      for (int64_t y = 1; y <= N - 2; ++y)
        for (int64_t x = 1; x + y <= N - 1; ++x) {
          const int64_t loc = faceIdx(w, x, y);
          dofs.push_back({KF, (int)f, int((x + 2 * y) % 3), loc, (int)x, (int)y, 0, lay.off[KF][f] + loc, ld.hostFaceType[f]});
        }
  for (size_t c = 0; c < topo.cells.size(); ++c)
    if (sel.inGroup0(KC, lay.off[KC][c]))
      for (int64_t z = 1; z <= N - 3; ++z)
        for (int64_t y = 1; y + z <= N - 2; ++y)
          for (int64_t x = 1; x + y + z <= N - 1; ++x) {
            const int64_t loc = cellIdx(w, x, y, z);
            dofs.push_back({KC, (int)c, int((x + 2 * y + 3 * z) % 4), loc, (int)x, (int)y, (int)z, lay.off[KC][c] + loc,
                            ld.hostCellType[c]});
          }
  std::sort(dofs.begin(), dofs.end(), [](const Dof& a, const Dof& b) {
    return std::tie(a.kind, a.colour, a.prim, a.local) < std::tie(b.kind, b.colour, b.prim, b.local);
  });
  argCheck(dofs.size() < (size_t)0x7fffffff, "compact cycle: level too large");
  const int n = (int)dofs.size();
  lb.unknownOf.assign((size_t)lay.total, -1);
  for (int i = 0; i < n; ++i) lb.unknownOf[(size_t)dofs[(size_t)i].slot] = i;
  lb.snapBegin = lb.snapEnd = n;
  for (int i = n - 1; i >= 0; --i) {
    if (dofs[(size_t)i].kind >= KE) lb.snapBegin = i;
    if (dofs[(size_t)i].kind >= KC) lb.snapEnd = i;
  }
  lb.snapEnd = std::max(lb.snapEnd, lb.snapBegin);

  // entries of every unknown the SOR, the residual or the coarse CG updates
  std::vector<int> e0((size_t)n, 0), e1((size_t)n, 0), wsel((size_t)n, 0);
  for (int i = 0; i < n; ++i) {
    const Dof& d = dofs[(size_t)i];
    if (!(d.type & (mask | (coarsest ? cgMask : 0u)))) continue;
    e0[(size_t)i] = (int)lb.cols.size();
    auto add = [&](int kind, int prim, int64_t local) {
      const Slot o = D.owner(L, D.slotBary(L, kind, prim, local));
      const int j = lb.unknownOf[(size_t)(lay.off[o.kind][(size_t)o.prim] + o.local)];
      argCheck(j >= 0, "compact cycle: a stencil entry outside the group");
      if (coarsest) {  // the coarsest level is solved by CG only: no smoother reads
        lb.cols.push_back(j);
        return;
      }
      const Dof& nb = dofs[(size_t)j];
      const bool closure = inClosure(topo, nb.kind, nb.prim, d.kind, d.prim);
      // the reads the multi-launch smoother makes through halo copies (see compact.hpp)
      argCheck(d.kind != KC || closure, "compact cycle: a cell row reads outside its closure");
      argCheck(d.kind != KV || nb.kind != KV, "compact cycle: neighbouring vertices");
      argCheck(d.kind == KV || d.kind == KC || closure || nb.kind != KV,
               "compact cycle: an edge or face row reads a vertex outside its closure");
      const bool start = (d.kind == KE || d.kind == KF) && (nb.kind == KE || nb.kind == KF) && !closure;
      lb.cols.push_back(int((unsigned)j | (start ? 0x80000000u : 0u)));
    };
    if (d.kind == KC) {
      wsel[(size_t)i] = d.prim << 2;
      for (int k = 1; k < 15; ++k)
        add(KC, d.prim, cellIdx(w, d.x + kCellOffsets[k][0], d.y + kCellOffsets[k][1], d.z + kCellOffsets[k][2]));
    } else if (d.kind == KF) {
      wsel[(size_t)i] = (d.prim << 2) | 1;
      const auto& fe = hs.face[(size_t)d.prim];
      for (size_t k = 1; k < fe.size(); ++k) {
        const int64_t x = d.x + fe[k].dx, y = d.y + fe[k].dy;
        add(KF, d.prim, fe[k].layer == 0 ? faceIdx(w, x, y) : tri(w) + (fe[k].layer - 1) * tri(w - 1) + faceIdx(w - 1, x, y));
      }
    } else if (d.kind == KE) {
      wsel[(size_t)i] = (d.prim << 2) | 2;
      const auto& le = hs.edge[(size_t)d.prim];
      for (size_t k = 1; k < le.size(); ++k) add(KE, d.prim, d.x + le[k].rel);
    } else {
      wsel[(size_t)i] = ((nE + d.prim) << 2) | 3;
      const auto& le = hs.vert[(size_t)d.prim];
      for (size_t k = 1; k < le.size(); ++k) add(KV, d.prim, le[k].rel);
    }
    e1[(size_t)i] = (int)lb.cols.size();
  }
  lb.rowOf.assign((size_t)n, -1);
  for (int i = 0; i < n; ++i) {
    const Dof& d = dofs[(size_t)i];
    const dev::CompactRow row{i, wsel[(size_t)i], e0[(size_t)i], e1[(size_t)i]};
    if (d.type & mask) {
      lb.rowOf[(size_t)i] = (int)lb.rows.size();
      if (d.kind == KV) ++lb.nVertexRows;
      lb.rows.push_back(row);
    }
    if (coarsest && (d.type & cgMask)) lb.cgRows.push_back(row);
  }
  for (size_t r = (size_t)lb.nVertexRows; r < lb.rows.size(); ++r) {
    const Dof& d = dofs[(size_t)lb.rows[r].idx];
    const bool last = r + 1 == lb.rows.size();
    if (last || dofs[(size_t)lb.rows[r + 1].idx].kind != d.kind || dofs[(size_t)lb.rows[r + 1].idx].colour != d.colour)
      lb.groupEnd.push_back((int)r + 1);
  }
  argCheck(lb.groupEnd.size() <= (size_t)dev::kCompactGroups, "compact cycle: too many colour groups");
  return lb;
}

// Prolongation rows of fine level f from coarse level c, in every macro-cell of group 0 (each
// fine DoF takes its pair from the first cell whose closure holds it), and the restriction as
// their transpose, gathered per coarse row in ascending fine order.
void buildTransfers(Storage& s, LevelBuild& f, LevelBuild& c, const GroupSel& sel) {
  const Discretization& D = s.disc;
  const LevelLayout& lf = *s.levels[(size_t)f.L].lay;
  const LevelLayout& lc = *s.levels[(size_t)c.L].lay;
  const int64_t Nf = int64_t(1) << f.L, wf = Nf + 1, wc = Nf / 2 + 1;
  auto unknown = [&](const LevelBuild& lb, const LevelLayout& lay, int cell, int64_t w, int64_t x, int64_t y, int64_t z) {
    const Slot o = D.owner(lb.L, D.slotBary(lb.L, KC, cell, cellIdx(w, x, y, z)));
    const int j = lb.unknownOf[(size_t)(lay.off[o.kind][(size_t)o.prim] + o.local)];
    argCheck(j >= 0, "compact cycle: a transfer entry outside the group");
    return j;
  };
  f.pro.assign(f.rows.size(), make_int2(-1, -1));
  std::vector<char> done(f.rows.size(), 0);
  for (size_t cell = 0; cell < D.topo().cells.size(); ++cell) {
    if (!sel.inGroup0(KC, lf.off[KC][cell])) continue;
    for (int64_t z = 0; z <= Nf; ++z)
      for (int64_t y = 0; y + z <= Nf; ++y)
        for (int64_t x = 0; x + y + z <= Nf; ++x) {
          const int j = unknown(f, lf, (int)cell, wf, x, y, z);
          const int r = f.rowOf[(size_t)j];
          if (r < 0 || done[(size_t)r]) continue;
          done[(size_t)r] = 1;
          const int code = int(x & 1) | (int(y & 1) << 1) | (int(z & 1) << 2);
          const int* d = kBisectDir[code];
          const int64_t ax = (x - d[0]) / 2, ay = (y - d[1]) / 2, az = (z - d[2]) / 2;
          const int a = unknown(c, lc, (int)cell, wc, ax, ay, az);
          const int b = code == 0 ? -1 : unknown(c, lc, (int)cell, wc, ax + d[0], ay + d[1], az + d[2]);
          f.pro[(size_t)r] = make_int2(a, b);
        }
  }
  for (char d : done) argCheck(d != 0, "compact cycle: a fine unknown outside every macro-cell");
  std::vector<std::vector<int>> into(c.rows.size());
  for (size_t r = 0; r < f.rows.size(); ++r) {
    const int2 p = f.pro[r];
    const int fi = f.rows[r].idx;
    for (int k = 0; k < 2; ++k) {
      const int cj = k == 0 ? p.x : p.y;
      if (cj < 0) continue;
      const int cr = c.rowOf[(size_t)cj];
      if (cr >= 0) into[(size_t)cr].push_back(int((unsigned)fi | (p.y >= 0 ? 0x80000000u : 0u)));
    }
  }
  c.rPtr.assign(1, 0);
  c.rIdx.clear();
  for (auto& v : into) {
    std::sort(v.begin(), v.end(), [](int a, int b) { return (a & 0x7fffffff) < (b & 0x7fffffff); });
    c.rIdx.insert(c.rIdx.end(), v.begin(), v.end());
    c.rPtr.push_back((int)c.rIdx.size());
  }
}

template <class V>
const V* put(CompactCycle& cc, const std::vector<V>& h, cudaStream_t st) {
  cc.keep.emplace_back(new DevBuf());
  void* d = cc.keep.back()->alloc(std::max<size_t>(h.size(), 1) * sizeof(V));
  if (!h.empty()) cudaCheck(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(V), cudaMemcpyHostToDevice, st), "compact lists");
  return (const V*)d;
}

template <class T>
void fillDev(CompactCycle& cc, dev::CompactCycleDev<T>& d, Storage& s, const Operator& o,
             const std::vector<LevelBuild>& lbs, const std::vector<int64_t>& gather, const std::vector<int64_t>& scSlot,
             const std::vector<int>& scIdx, const std::vector<int>& scOff) {
  d = dev::CompactCycleDev<T>{};
  d.nLevels = (int)lbs.size();
  int64_t off = 0, maxN = 0;
  auto vec = [&](int64_t n) {
    const int64_t at = off;
    off += (n + 31) / 32 * 32;
    return at;
  };
  for (size_t k = 0; k < lbs.size(); ++k) {
    const LevelBuild& lb = lbs[k];
    dev::CompactLevel<T>& L = d.lv[k];
    L.n = (int)lb.dofs.size();
    L.nRows = (int)lb.rows.size();
    L.nVertexRows = lb.nVertexRows;
    L.nGroups = (int)lb.groupEnd.size();
    for (size_t g = 0; g < lb.groupEnd.size(); ++g) L.groupEnd[g] = lb.groupEnd[g];
    L.nCgRows = (int)lb.cgRows.size();
    L.snapBegin = lb.snapBegin;
    L.snapEnd = lb.snapEnd;
    L.rows = put(cc, lb.rows, s.stream);
    L.cgRows = put(cc, lb.cgRows, s.stream);
    L.cols = put(cc, lb.cols, s.stream);
    L.pro = put(cc, lb.pro, s.stream);
    L.rPtr = put(cc, lb.rPtr, s.stream);
    L.rIdx = put(cc, lb.rIdx, s.stream);
    const int oi = lb.L - o.minL;
    if constexpr (sizeof(T) == 8)
      L.st = o.d[(size_t)oi];
    else
      L.st = o.f[(size_t)oi];
    L.x = vec(L.n);
    L.b = vec(L.n);
    L.r = vec(L.n);
    maxN = std::max<int64_t>(maxN, L.n);
  }
  d.snap = vec(maxN);
  d.groupStride = off;
  d.cgStride = 5 * (int64_t)lbs[0].dofs.size();
  d.cgSt = o.d[(size_t)(lbs[0].L - o.minL)];
  d.gather = put(cc, gather, s.stream);
  d.scatterSlot = put(cc, scSlot, s.stream);
  d.scatterIdx = put(cc, scIdx, s.stream);
  d.scatterOff = put(cc, scOff, s.stream);
  cc.scratch.alloc((size_t)std::max<int64_t>(d.groupStride * cc.groups, 1) * sizeof(T));
  cc.cg.alloc((size_t)std::max<int64_t>(d.cgStride * cc.groups, 1) * sizeof(double));
  cudaCheck(cudaMemsetAsync(cc.scratch.p, 0, cc.scratch.bytes, s.stream), "compact scratch");
  cudaCheck(cudaMemsetAsync(cc.cg.p, 0, cc.cg.bytes, s.stream), "compact scratch");
}

template <class T, int CL>
void launchT(CompactCycle& c, const dev::CompactCycleDev<T>& d, Storage& s, void* x, const void* b, bool xZero, int pre,
             int post, double omega, int cgMaxIter, double cgTol) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(c.groups * CL));
  cfg.blockDim = dim3(dev::kCompactThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = CL > 1 ? 1 : 0;
  cudaCheck(cudaLaunchKernelEx(&cfg, dev::compactCycleKernel<T, CL>, d, (T*)x, (const T*)b, (T*)c.scratch.p,
                               (double*)c.cg.p, (int)xZero, pre, post, (T)omega, cgMaxIter, cgTol),
            "compact cycle");
  ++s.launches;
}

template <class T>
void launchPrec(CompactCycle& c, const dev::CompactCycleDev<T>& d, Storage& s, void* x, const void* b, bool xZero,
                int pre, int post, double omega, int cgMaxIter, double cgTol) {
  switch (c.cluster) {
    case 1: launchT<T, 1>(c, d, s, x, b, xZero, pre, post, omega, cgMaxIter, cgTol); break;
    case 2: launchT<T, 2>(c, d, s, x, b, xZero, pre, post, omega, cgMaxIter, cgTol); break;
    case 4: launchT<T, 4>(c, d, s, x, b, xZero, pre, post, omega, cgMaxIter, cgTol); break;
    default: launchT<T, 8>(c, d, s, x, b, xZero, pre, post, omega, cgMaxIter, cgTol); break;
  }
}

}  // namespace

int64_t compactGroupDofs(Storage& s, int L, int groups) {
  const Topology& t = s.disc.topo();
  const int64_t n = s.disc.ownedCount(L, KV) * (int64_t)t.verts.size() +
                    s.disc.ownedCount(L, KE) * (int64_t)t.edges.size() +
                    s.disc.ownedCount(L, KF) * (int64_t)t.faces.size() + s.disc.ownedCount(L, KC) * (int64_t)t.cells.size();
  return n / std::max(groups, 1);
}

std::unique_ptr<CompactCycle> buildCompactCycle(Storage& s, int op, int minL, int top, int groups, int cluster,
                                                int prec, unsigned mask, unsigned cgMask) {
  argCheck(top > minL && top - minL + 1 <= dev::kCompactMaxLevels, "compact cycle: level range");
  argCheck(cluster == 1 || cluster == 2 || cluster == 4 || cluster == 8, "compact cycle: 1, 2, 4 or 8 blocks per group");
  argCheck(prec == 8 || prec == 4, "compact cycle: precision must be 8 or 4");
  const Operator& o = s.op(op);
  argCheck(minL >= o.minL && top <= o.maxL, "compact cycle: levels outside the operator's range");
  std::unique_ptr<CompactCycle> cc(new CompactCycle());
  cc->minL = minL;
  cc->top = top;
  cc->groups = groups;
  cc->cluster = cluster;
  cc->prec = prec;
  std::vector<LevelBuild> lbs;
  std::vector<GroupSel> sels;
  for (int L = minL; L <= top; ++L) {
    GroupSel sel;
    sel.groups = groups;
    if (groups > 1) sel.bm = s.batchMap(L, groups);
    sels.push_back(sel);
    lbs.push_back(buildLevel(s, o.host[(size_t)(L - o.minL)], L, sel, mask, cgMask, L == minL));
  }
  for (size_t k = 1; k < lbs.size(); ++k) buildTransfers(s, lbs[k], lbs[k - 1], sels[k]);
  // gather (owner slots) and scatter (every slot holding a DoF) of the top level, per group
  const LevelBuild& tb = lbs.back();
  const GroupSel& ts = sels.back();
  const LevelLayout& lay = *s.levels[(size_t)top].lay;
  const Topology& topo = s.disc.topo();
  std::vector<int64_t> gather;
  for (int g = 0; g < groups; ++g)
    for (const Dof& d : tb.dofs) gather.push_back(d.slot + ts.shift(d.kind, g));
  std::vector<std::pair<int64_t, int>> slots0;  // (absolute slot, its kind)
  std::vector<int> idx0;
  const size_t nPrim[4] = {topo.verts.size(), topo.edges.size(), topo.faces.size(), topo.cells.size()};
  for (int kind : {KV, KE, KF, KC})
    for (size_t p = 0; p < nPrim[kind]; ++p) {
      if (!ts.inGroup0(kind, lay.off[kind][p])) continue;
      for (int64_t local = 0; local < lay.size[kind][p]; ++local) {
        const Slot o2 = s.disc.owner(top, s.disc.slotBary(top, kind, (int)p, local));
        const int j = tb.unknownOf[(size_t)(lay.off[o2.kind][(size_t)o2.prim] + o2.local)];
        argCheck(j >= 0, "compact cycle: a copy slot outside the group");
        slots0.push_back({lay.off[kind][p] + local, kind});
        idx0.push_back(j);
      }
    }
  std::vector<int64_t> scSlot;
  std::vector<int> scIdx, scOff{0};
  for (int g = 0; g < groups; ++g) {
    for (size_t e = 0; e < slots0.size(); ++e) {
      scSlot.push_back(slots0[e].first + ts.shift(slots0[e].second, g));
      scIdx.push_back(idx0[e]);
    }
    scOff.push_back((int)scSlot.size());
  }
  // primitives of each kind per group (cells, faces, edges, vertices): group g's stencils
  int perGroup[4];
  const size_t nKind[4] = {topo.cells.size(), topo.faces.size(), topo.edges.size(), topo.verts.size()};
  for (int q = 0; q < 4; ++q) {
    argCheck(nKind[q] % (size_t)groups == 0, "compact cycle: primitives are not a multiple of the groups");
    perGroup[q] = groups > 1 ? (int)(nKind[q] / (size_t)groups) : 0;
  }
  // every index the kernel follows stays inside its vector, stencil array or level buffer
  const int nEdges = (int)topo.edges.size();
  const size_t nPrimW[3] = {topo.cells.size(), topo.faces.size(), topo.edges.size() + topo.verts.size()};
  for (size_t k = 0; k < lbs.size(); ++k) {
    const LevelBuild& lb = lbs[k];
    const int n = (int)lb.dofs.size();
    const LevelStencils& hs = o.host[(size_t)(lb.L - o.minL)];
    auto checkRow = [&](const dev::CompactRow& r) {
      argCheck(r.idx >= 0 && r.idx < n && r.e0 >= 0 && r.e0 <= r.e1 && r.e1 <= (int)lb.cols.size(), "compact cycle: row");
      const int kind = r.wsel & 3, prim = r.wsel >> 2;
      argCheck(prim >= 0 && (size_t)prim < nPrimW[std::min(kind, 2)] && (kind != 2 || prim < nEdges) &&
                   (kind != 3 || prim >= nEdges),
               "compact cycle: stencil");
      const size_t len = kind == 0 ? 15
                         : kind == 1 ? hs.face[(size_t)prim].size()
                         : kind == 2 ? hs.edge[(size_t)prim].size()
                                     : hs.vert[(size_t)(prim - nEdges)].size();
      argCheck((size_t)(r.e1 - r.e0) + 1 == len && (kind >= 2 || len <= 16), "compact cycle: stencil length");
      // the last group's primitives exist too
      const int64_t last = (int64_t)prim + (int64_t)(groups - 1) * perGroup[kind];
      argCheck(last < (int64_t)nPrimW[std::min(kind, 2)], "compact cycle: stencil of the last group");
    };
    for (const auto& r : lb.rows) checkRow(r);
    for (const auto& r : lb.cgRows) checkRow(r);
    for (int c : lb.cols) argCheck((c & 0x7fffffff) < n, "compact cycle: entry");
    argCheck(lb.snapBegin >= 0 && lb.snapBegin <= lb.snapEnd && lb.snapEnd <= n, "compact cycle: snapshot");
    argCheck(lb.nVertexRows <= (int)lb.rows.size() && (lb.groupEnd.empty() || lb.groupEnd.back() == (int)lb.rows.size()),
             "compact cycle: groups");
    if (k > 0) {
      const int nc = (int)lbs[k - 1].dofs.size();
      argCheck(lb.pro.size() == lb.rows.size(), "compact cycle: prolongation");
      for (const int2& p : lb.pro) argCheck(p.x >= 0 && p.x < nc && p.y < nc, "compact cycle: prolongation");
    }
    if (k + 1 < lbs.size()) {
      const int nf = (int)lbs[k + 1].dofs.size();
      argCheck(lb.rPtr.size() == lb.rows.size() + 1 && lb.rPtr.back() == (int)lb.rIdx.size(), "compact cycle: restriction");
      for (int c : lb.rIdx) argCheck((c & 0x7fffffff) < nf, "compact cycle: restriction");
    }
  }
  for (int64_t sl : gather) argCheck(sl >= 0 && sl < lay.total, "compact cycle: gather");
  for (int64_t sl : scSlot) argCheck(sl >= 0 && sl < lay.total, "compact cycle: scatter");
  for (int j : scIdx) argCheck(j >= 0 && j < (int)tb.dofs.size(), "compact cycle: scatter");
  if (prec == 8) {
    fillDev<double>(*cc, cc->d64, s, o, lbs, gather, scSlot, scIdx, scOff);
    for (int q = 0; q < 4; ++q) cc->d64.primsPerGroup[q] = perGroup[q];
  } else {
    fillDev<float>(*cc, cc->d32, s, o, lbs, gather, scSlot, scIdx, scOff);
    for (int q = 0; q < 4; ++q) cc->d32.primsPerGroup[q] = perGroup[q];
  }
  cudaCheck(cudaStreamSynchronize(s.stream), "compact lists");
  return cc;
}

void runCompactCycle(CompactCycle& c, Storage& s, void* x, const void* b, bool xZero, int pre, int post, double omega,
                     int cgMaxIter, double cgTol) {
  if (c.prec == 8)
    launchPrec<double>(c, c.d64, s, x, b, xZero, pre, post, omega, cgMaxIter, cgTol);
  else
    launchPrec<float>(c, c.d32, s, x, b, xZero, pre, post, omega, cgMaxIter, cgTol);
}

}  // namespace hg
