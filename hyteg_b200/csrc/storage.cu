// hg_storage: device arena, per-level work tables, operators, solvers and the C-ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/hyteg_b200.h"
#include "discretization.hpp"
#include "kernels.cuh"
#include "solvers.hpp"
#include "storage.hpp"

namespace hg {

thread_local std::string g_lastError;
static const int kAllGroups = (1 << G_COUNT) - 1;

void cudaCheck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    if (e == cudaErrorMemoryAllocation) {
      (void)cudaGetLastError();
      throw Error(HG_ERR_OOM, std::string(what) + ": " + cudaGetErrorString(e));
    }
    throw Error(HG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }
}

void argCheck(bool ok, const std::string& msg) {
  if (!ok) throw Error(HG_ERR_ARG, msg);
}

DevBuf::~DevBuf() {
  if (p) cudaFree(p);
}
void* DevBuf::alloc(size_t n) {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = n;
  if (n) cudaCheck(cudaMalloc(&p, n), "cudaMalloc");
  return p;
}

template <class V>
static void* upload(std::vector<std::unique_ptr<DevBuf>>& keep, const std::vector<V>& h, cudaStream_t st) {
  keep.emplace_back(new DevBuf());
  void* d = keep.back()->alloc(std::max<size_t>(h.size(), 1) * sizeof(V));
  if (!h.empty()) cudaCheck(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(V), cudaMemcpyHostToDevice, st), "upload");
  return d;
}

static unsigned char dofType(int meshFlag) {
  // BoundaryCondition::create0123BC (src/hyteg/boundary/BoundaryConditions.cpp:26-33)
  switch (meshFlag) {
    case 1: return HG_DIRICHLET;
    case 2: return HG_NEUMANN;
    case 3: return HG_FREESLIP;
    default: return HG_INNER;
  }
}

Storage::Storage(const Topology& topo, int maxLevel) : disc(topo, maxLevel) {
  cudaCheck(cudaGetDevice(&device), "cudaGetDevice");
  cudaCheck(cudaStreamCreateWithFlags(&ownStream, cudaStreamNonBlocking), "cudaStreamCreate");
  cudaCheck(cudaFuncSetAttribute(dev::cellSorWaveKernel<double, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)dev::waveSmemBytes<double, 0>(dev::kWaveMaxN)),
            "wave kernel shared memory");
  cudaCheck(cudaFuncSetAttribute(dev::cellSorWaveKernel<float, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)dev::waveSmemBytes<float, 0>(dev::kWaveMaxN)),
            "wave kernel shared memory");
  cudaCheck(cudaFuncSetAttribute(dev::cellSorWaveKernel<double, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)dev::waveSmemBytes<double, 1>(dev::kWaveMaxN)),
            "wave kernel shared memory");
  cudaCheck(cudaFuncSetAttribute(dev::cellSorWaveKernel<float, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)dev::waveSmemBytes<float, 1>(dev::kWaveMaxN)),
            "wave kernel shared memory");
  stream = ownStream;
  levels.resize(maxLevel + 1);
  for (int L = 0; L <= maxLevel; ++L) buildLevel(L);
  {
    const Topology& t = disc.topo();
    std::vector<double> vx;
    for (auto& v : t.verts)
      for (int d = 0; d < 3; ++d) vx.push_back(v.x[d]);
    std::vector<int> cv, fv, lv;
    for (auto& c : t.cells)
      for (int k = 0; k < 4; ++k) cv.push_back(c.v[k]);
    for (auto& f : t.faces)
      for (int k = 0; k < 3; ++k) fv.push_back(f.v[k]);
    for (auto& e : t.edges) {
      lv.push_back(e.v[0]);
      lv.push_back(e.v[1]);
    }
    for (size_t v = 0; v < t.verts.size(); ++v) {
      lv.push_back((int)v);
      lv.push_back((int)v);
    }
    geom.vx = (const double*)upload(geomKeep, vx, stream);
    geom.cellV = (const int*)upload(geomKeep, cv, stream);
    geom.faceV = (const int*)upload(geomKeep, fv, stream);
    geom.lowV = (const int*)upload(geomKeep, lv, stream);
  }
  scalars.alloc(64 * sizeof(double));
  cudaCheck(cudaMemsetAsync(scalars.p, 0, 64 * sizeof(double), stream), "memset");
  cudaCheck(cudaStreamSynchronize(stream), "sync");
}

Storage::~Storage() {
  p2gmgs.clear();
  gmgs.clear();
  ops.clear();
  fns.clear();
  levels.clear();
  if (ownStream) cudaStreamDestroy(ownStream);
}

void Storage::buildLevel(int L) {
  const Topology& topo = disc.topo();
  const LevelLayout& lay = disc.level(L);
  LevelData& ld = levels[L];
  ld.lay = &lay;
  dev::LevelDev& lv = ld.lv;
  lv.L = L;
  lv.N = (int)lay.N;
  lv.w = (int)lay.w;
  lv.nCells = (int)topo.cells.size();
  lv.nFaces = (int)topo.faces.size();
  lv.nEdges = (int)topo.edges.size();
  lv.nLow = (int)(topo.edges.size() + topo.verts.size());
  const int64_t N = lay.N, w = lay.w;
  argCheck(lay.total < (int64_t(1) << 32), "level buffer exceeds 32-bit halo indices");

  std::vector<int64_t> lowOff;
  std::vector<int> lowFirst, lowCount;
  std::vector<unsigned char> cellType, faceType, lowType;
  for (auto& c : topo.cells) cellType.push_back(dofType(c.flag));
  for (auto& f : topo.faces) faceType.push_back(dofType(f.flag));
  for (size_t e = 0; e < topo.edges.size(); ++e) {
    lowOff.push_back(lay.off[KE][e]);
    lowFirst.push_back(1);
    lowCount.push_back((int)std::max<int64_t>(N - 1, 0));
    lowType.push_back(dofType(topo.edges[e].flag));
  }
  for (size_t v = 0; v < topo.verts.size(); ++v) {
    lowOff.push_back(lay.off[KV][v]);
    lowFirst.push_back(0);
    lowCount.push_back(1);
    lowType.push_back(dofType(topo.verts[v].flag));
  }
  ld.hostCellType = cellType;
  ld.hostFaceType = faceType;
  ld.hostLowType = lowType;

  lv.nCellBlocks = N >= 4 ? lv.nCells * (int)(N - 3) : 0;
  std::vector<dev::FaceBlock> fb;
  if (N >= 3)
    for (int f = 0; f < lv.nFaces; ++f)
      for (int y = 1; y < (int)w - 2; y += dev::kFaceRows) fb.push_back({f, y});
  std::vector<dev::LowBlock> lb;
  for (int p = 0; p < lv.nLow; ++p) {
    if (p == lv.nEdges) lv.nLowEdgeBlocks = (int)lb.size();
    for (int s = lowFirst[p]; s < lowFirst[p] + lowCount[p]; s += dev::kBlock) lb.push_back({p, s});
  }
  if (lv.nEdges == lv.nLow) lv.nLowEdgeBlocks = (int)lb.size();

  std::vector<dev::Chunk> chunks;
  auto addChunks = [&](int64_t off, int64_t size, int type) {
    for (int64_t s = 0; s < size; s += 8192) chunks.push_back({off + s, (int)std::min<int64_t>(8192, size - s), type});
  };
  for (int c = 0; c < lv.nCells; ++c) addChunks(lay.off[KC][c], lay.size[KC][c], cellType[c]);
  ld.nCellChunks = (int)chunks.size();
  for (int f = 0; f < lv.nFaces; ++f) addChunks(lay.off[KF][f], lay.size[KF][f], faceType[f]);
  for (int e = 0; e < lv.nEdges; ++e) addChunks(lay.off[KE][e], lay.size[KE][e], lowType[e]);
  for (size_t v = 0; v < topo.verts.size(); ++v) addChunks(lay.off[KV][v], lay.size[KV][v], lowType[lv.nEdges + v]);

  // halo table in the five destination groups
  std::vector<uint2> comm;
  for (int g : kCommOrder) {
    ld.commBegin[g] = (int64_t)comm.size();
    for (size_t i = 0; i < lay.commDst[g].size(); ++i)
      comm.push_back(make_uint2((unsigned)lay.commDst[g][i], (unsigned)lay.commSrc[g][i]));
    ld.commCount[g] = (int64_t)comm.size() - ld.commBegin[g];
  }
  argCheck(comm.size() < (size_t(1) << 31), "halo table exceeds 32-bit ranges");
  // Each primitive's entries of a group are contiguous (the tables are generated primitive by
  // primitive): the range of every primitive's destination array, found from its offsets.
  auto ranges = [&](int g, int kind, int nPrim) {
    std::vector<int2> r((size_t)nPrim, make_int2(0, 0));
    std::vector<char> seen((size_t)nPrim, 0);
    int last = -1;
    for (int64_t i = ld.commBegin[g]; i < ld.commBegin[g] + ld.commCount[g]; ++i) {
      const int64_t d = comm[(size_t)i].x;
      const auto& offs = lay.off[kind];
      const int p = int(std::upper_bound(offs.begin(), offs.end(), d) - offs.begin()) - 1;
      argCheck(p >= 0 && p < nPrim && d < offs[(size_t)p] + lay.size[kind][(size_t)p], "halo entry outside its group's kind");
      if (p != last) {
        argCheck(!seen[(size_t)p], "halo entries of a primitive are not contiguous");
        seen[(size_t)p] = 1;
        r[(size_t)p].x = (int)i;
        last = p;
      }
      r[(size_t)p].y = (int)i + 1;
    }
    return r;
  };
  {
    std::vector<int2> low = ranges(G_EDGE, KE, lv.nEdges);
    std::vector<int2> vr = ranges(G_VERT, KV, (int)topo.verts.size());
    low.insert(low.end(), vr.begin(), vr.end());
    std::vector<int2> fr = ranges(G_FACE_BOUNDARY, KF, lv.nFaces);
    if (!low.empty()) ld.lowRange = (const int2*)upload(ld.keep, low, stream);
    if (!fr.empty()) ld.faceRange = (const int2*)upload(ld.keep, fr, stream);
  }

  auto& keep = ld.keep;
  lv.cellOff = (const int64_t*)upload(keep, lay.off[KC], stream);
  lv.faceOff = (const int64_t*)upload(keep, lay.off[KF], stream);
  lv.lowOff = (const int64_t*)upload(keep, lowOff, stream);
  lv.lowFirst = (const int*)upload(keep, lowFirst, stream);
  lv.lowCount = (const int*)upload(keep, lowCount, stream);
  lv.cellType = (const unsigned char*)upload(keep, cellType, stream);
  lv.faceType = (const unsigned char*)upload(keep, faceType, stream);
  lv.lowType = (const unsigned char*)upload(keep, lowType, stream);
  lv.faceBlocks = (const dev::FaceBlock*)upload(keep, fb, stream);
  lv.nFaceBlocks = (int)fb.size();
  lv.lowBlocks = (const dev::LowBlock*)upload(keep, lb, stream);
  lv.nLowBlocks = (int)lb.size();
  ld.comm = (uint2*)upload(keep, comm, stream);
  ld.chunks = (dev::Chunk*)upload(keep, chunks, stream);
  buildTiles(L);
  // single-pass SOR tiles: every (x, y) of the cell is in exactly one tile, tallest tiles first;
  // one list per precision (the tile heights differ)
  {
    const int tys[2][2] = {{dev::WaveGeom<double, 0>::TY, dev::WaveGeom<double, 1>::TY},
                           {dev::WaveGeom<float, 0>::TY, dev::WaveGeom<float, 1>::TY}};
    for (int pi = 0; pi < 2; ++pi)
      for (int gv = 0; gv < 2; ++gv) {
        const int ty = tys[pi][gv];
        std::vector<dev::WaveTile> wt;
        if (N >= 4)
          for (int c = 0; c < lv.nCells; ++c)
            for (int y0 = 0; y0 <= N; y0 += ty)
              for (int x0 = 0; x0 + y0 <= N; x0 += dev::kWaveTX) wt.push_back({c, x0, y0, (int)N - x0 - y0});
        std::stable_sort(wt.begin(), wt.end(),
                         [](const dev::WaveTile& a, const dev::WaveTile& b) { return a.pEnd > b.pEnd; });
        ld.waveTiles[pi][gv] = (dev::WaveTile*)upload(keep, wt, stream);
        ld.nWaveTiles[pi][gv] = (int)wt.size();
      }
    int64_t first = lay.total;
    for (int k : {KV, KE, KF})
      for (int64_t o : lay.off[k]) first = std::min(first, o);
    for (size_t c = 0; c < lay.off[KC].size(); ++c)
      argCheck(lay.off[KC][c] + lay.size[KC][c] <= first, "cell arrays must precede the other primitives");
    ld.nonCellBegin = first;
  }
  ld.nChunks = (int)chunks.size();
  ld.partial.alloc(sizeof(double) * std::max(1, lv.nCellBlocks + lv.nFaceBlocks + lv.nLowBlocks));
  cudaCheck(cudaStreamSynchronize(stream), "level upload");
}

// Cell-sweep work items: (cell, 30-column x 32-row block of strips, <= kStripZ planes), the
// longest first inside groups of macro-cells whose two FP64 vectors fit into the L2 budget;
// the SOR colours of a group run back to back so that their re-reads hit L2.
void Storage::buildTiles(int L) {
  LevelData& ld = levels[L];
  const int64_t N = ld.lay->N, w = ld.lay->w;
  const int nCells = ld.lv.nCells;
  std::vector<dev::StripItem> items;
  const int64_t cellBytes = tet(w) * 8;
  ld.cellsPerGroup = (int)std::max<int64_t>(1, std::min<int64_t>(nCells, l2Budget / (2 * cellBytes)));
  ld.tileGroupBegin.assign(1, 0);
  for (int g0 = 0; N >= 4 && g0 < nCells; g0 += ld.cellsPerGroup) {
    std::vector<dev::StripItem> grp;
    for (int c = g0; c < std::min(nCells, g0 + ld.cellsPerGroup); ++c)
      for (int y0 = 1; y0 <= N - 3; y0 += dev::kStripRows)
        for (int x0 = 1; x0 <= N - 3; x0 += dev::kStripX) {
          const int zmax = (int)N - 1 - x0 - y0;  // last plane with an interior point in the block
          if (zmax < 1) continue;
          for (int z0 = 1; z0 <= zmax; z0 += dev::kStripZ)
            grp.push_back({c, x0, y0, z0, std::min(zmax + 1, z0 + dev::kStripZ), 0, 0, 0});
        }
    std::stable_sort(grp.begin(), grp.end(),
                     [](const dev::StripItem& a, const dev::StripItem& b) { return (a.z1 - a.z0) > (b.z1 - b.z0); });
    items.insert(items.end(), grp.begin(), grp.end());
    ld.tileGroupBegin.push_back((int)items.size());
  }
  ld.tileBuf.reset(new DevBuf());
  ld.tiles = (dev::StripItem*)ld.tileBuf->alloc(std::max<size_t>(items.size(), 1) * sizeof(dev::StripItem));
  if (!items.empty())
    cudaCheck(cudaMemcpyAsync(ld.tiles, items.data(), items.size() * sizeof(dev::StripItem), cudaMemcpyHostToDevice,
                              stream),
              "strip items");
  ld.nTiles = (int)items.size();
  cudaCheck(cudaStreamSynchronize(stream), "strip items sync");
}

void Storage::setL2Budget(int64_t bytes) {
  argCheck(bytes > 0, "L2 budget must be positive");
  l2Budget = bytes;
  ++generation;
  for (int L = 0; L <= maxLevel(); ++L) buildTiles(L);
}

// ------------------------------------------------------------------------------------------
// functions
// ------------------------------------------------------------------------------------------
Function& Storage::fn(int id) {
  auto it = fns.find(id);
  argCheck(it != fns.end(), "unknown function handle");
  return *it->second;
}
void* Storage::data(int id, int L) {
  Function& f = fn(id);
  argCheck(L >= f.minL && L <= f.maxL, "level outside the function's level range");
  return f.levels[L - f.minL]->p;
}
int Storage::createFunction(int minL, int maxL, int prec) {
  argCheck(minL >= 0 && maxL <= maxLevel() && minL <= maxL, "invalid level range");
  argCheck(prec == 8 || prec == 4, "precision must be 8 or 4");
  std::unique_ptr<Function> f(new Function());
  f->minL = minL;
  f->maxL = maxL;
  f->prec = prec;
  for (int L = minL; L <= maxL; ++L) {
    f->levels.emplace_back(new DevBuf());
    const size_t bytes = (size_t)levels[L].lay->total * prec;
    f->levels.back()->alloc(bytes);
    cudaCheck(cudaMemsetAsync(f->levels.back()->p, 0, bytes, stream), "memset");
  }
  const int id = nextId++;
  fns[id] = std::move(f);
  return id;
}

static unsigned grid1d(int64_t n) { return (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 32); }

void Storage::communicate(int id, int L, int groupMask) {
  Function& f = fn(id);
  void* d = data(id, L);
  const LevelData& ld = levels[L];
  // one gather per contiguous run of selected groups in the table
  int k = 0;  // position in the table order
  while (k < G_COUNT) {
    if (!(groupMask & (1 << kCommOrder[k]))) {
      ++k;
      continue;
    }
    const int64_t begin = ld.commBegin[kCommOrder[k]];
    int64_t n = 0;
    while (k < G_COUNT && (groupMask & (1 << kCommOrder[k]))) n += ld.commCount[kCommOrder[k++]];
    if (n == 0) continue;
    if (f.prec == 8)
      dev::commGatherKernel<double><<<grid1d(n), 256, 0, stream>>>((double*)d, ld.comm + begin, n);
    else
      dev::commGatherKernel<float><<<grid1d(n), 256, 0, stream>>>((float*)d, ld.comm + begin, n);
    ++launches;
  }
  cudaCheck(cudaGetLastError(), "communicate");
}

template <class T>
void Storage::communicateSplit(T* buf, T* cells, int L, int groupMask) {
  buildSplit(L);
  const LevelData& ld = levels[L];
  const uint2* table = ld.commSplit;
  int k = 0;  // position in the table order
  while (k < G_COUNT) {
    if (!(groupMask & (1 << kCommOrder[k]))) {
      ++k;
      continue;
    }
    const int64_t begin = ld.commBegin[kCommOrder[k]];
    int64_t n = 0;
    while (k < G_COUNT && (groupMask & (1 << kCommOrder[k]))) n += ld.commCount[kCommOrder[k++]];
    if (n == 0) continue;
    dev::commGatherSplitKernel<T><<<grid1d(n), 256, 0, stream>>>(buf, cells, table + begin, n, ld.nonCellBegin);
    ++launches;
  }
  cudaCheck(cudaGetLastError(), "communicate (split)");
}

// The interior rows of colour col of a closed macro-cell with w points per edge (x, y, z >= 1,
// x + y + z <= w - 2), each with its 15 slots at j = 0 in the colour-split order, and the
// colour's points as (row << kSplitJBits | j), in (z, y, j) order.
void splitTables(int64_t w, int col, std::vector<dev::SplitRow>& rows, std::vector<unsigned>& points) {
  const int64_t N = w - 1;
  argCheck(N <= 4096, "colour-split SOR: level too large");
  auto tet = [](int64_t a) { return a * (a + 1) * (a + 2) / 6; };
  auto tri = [](int64_t a) { return a * (a + 1) / 2; };
  auto rowStart = [&](int64_t z, int64_t y) {
    const int64_t W = w - z;
    return tet(w) - tet(W) + y * (W + 1) - y * (y + 1) / 2;
  };
  rows.clear();
  points.clear();
  for (int64_t z = 1; z <= N - 3; ++z) {
    const int64_t W = w - z;
    for (int64_t y = 1; y <= W - 3; ++y) {
      const int m = (int)(W - y);
      const int q = (int)((((col - 2 * y - 3 * z) % 4) + 4) % 4);
      const int j0 = q == 0 ? 1 : 0, jEnd = m - 2 - q >= 0 ? (m - 2 - q) / 4 : -1;
      if (jEnd < j0) continue;
      const int qE = (q + 1) & 3, qW = (q + 3) & 3, jE = q == 3 ? 1 : 0, jW = q == 0 ? -1 : 0;
      const int64_t r0 = rowStart(z, y), rN = r0 + m, rS = r0 - (m + 1);
      const int64_t rT = r0 + tri(W) - y, rTS = rT - m, rB = r0 - tri(W + 1) + y, rBN = rB + (m + 1);
      auto sub = [](int mm, int qq) { return (int64_t)dev::splitSub(mm, qq); };
      dev::SplitRow r;
      const int64_t v[16] = {r0 + sub(m, q),          r0 + sub(m, qE) + jE,      r0 + sub(m, qW) + jW,
                             rN + sub(m - 1, q),      rS + sub(m + 1, q),        rN + sub(m - 1, qW) + jW,
                             rS + sub(m + 1, qE) + jE, rT + sub(m - 1, q),       rT + sub(m - 1, qW) + jW,
                             rTS + sub(m, q),         rTS + sub(m, qE) + jE,     rB + sub(m + 1, q),
                             rB + sub(m + 1, qE) + jE, rBN + sub(m, q),          rBN + sub(m, qW) + jW,
                             0};
      for (int k = 0; k < 16; ++k) r.i[k] = (int)v[k];
      argCheck(rows.size() < (size_t(1) << (32 - dev::kSplitJBits)), "colour-split SOR: too many rows");
      const unsigned id = (unsigned)rows.size();
      rows.push_back(r);
      for (int j = j0; j <= jEnd; ++j) points.push_back(id << dev::kSplitJBits | (unsigned)j);
    }
  }
}

// Schedule-3 tables of level L: the halo table with every slot of a cell array replaced by its
// position in the colour-split order (a permutation inside each row of the cell's array), and
// per colour the interior rows (their 15 slots at j = 0) and points (row << 10 | j) that
// cellSorSplitKernel walks; the same for every macro-cell of the level.
void Storage::buildSplit(int L) {
  LevelData& ld = levels[L];
  if (ld.commSplit) return;
  const LevelLayout& lay = *ld.lay;
  const int64_t w = lay.w, N = w - 1;
  argCheck(N <= 4096, "colour-split SOR: level too large");
  auto tet = [](int64_t a) { return a * (a + 1) * (a + 2) / 6; };
  auto rowStart = [&](int64_t z, int64_t y) {
    const int64_t W = w - z;
    return tet(w) - tet(W) + y * (W + 1) - y * (y + 1) / 2;
  };
  std::vector<int> perm((size_t)tet(w));
  for (int64_t z = 0; z < w; ++z)
    for (int64_t y = 0; y < w - z; ++y) {
      const int64_t r0 = rowStart(z, y);
      const int m = (int)(w - z - y);
      for (int x = 0; x < m; ++x) perm[(size_t)(r0 + x)] = (int)(r0 + dev::splitSub(m, x & 3) + (x >> 2));
    }
  std::vector<std::pair<int64_t, int64_t>> cells;  // (offset, size), ascending
  for (size_t c = 0; c < lay.off[KC].size(); ++c) cells.push_back({lay.off[KC][c], lay.size[KC][c]});
  std::sort(cells.begin(), cells.end());
  auto map = [&](int64_t slot) -> unsigned {
    if (slot < ld.nonCellBegin && !cells.empty()) {
      auto it = std::upper_bound(cells.begin(), cells.end(), std::make_pair(slot, INT64_MAX));
      if (it != cells.begin()) {
        --it;
        const int64_t local = slot - it->first;
        if (local < it->second && local < (int64_t)perm.size()) return (unsigned)(it->first + perm[(size_t)local]);
      }
    }
    return (unsigned)slot;
  };
  std::vector<uint2> comm;  // the same entries in the same order as the level's table
  for (int g : kCommOrder)
    for (size_t i = 0; i < lay.commDst[g].size(); ++i)
      comm.push_back(make_uint2(map(lay.commDst[g][i]), map(lay.commSrc[g][i])));
  const uint2* commSplit = comm.empty() ? ld.comm : (const uint2*)upload(ld.keep, comm, stream);
  // rows and points per colour
  for (int col = 0; col < 4; ++col) {
    std::vector<dev::SplitRow> rows;
    std::vector<unsigned> points;
    splitTables(w, col, rows, points);
    ld.splitRows[col] = (const dev::SplitRow*)upload(ld.keep, rows, stream);
    ld.splitPoints[col] = (const unsigned*)upload(ld.keep, points, stream);
    ld.nSplitPoints[col] = (int)points.size();
  }
  cudaCheck(cudaStreamSynchronize(stream), "colour-split tables");  // the host vectors go out of scope
  ld.commSplit = commSplit;
}

DevBuf& Storage::spareBuf(std::map<std::pair<int, int>, std::unique_ptr<DevBuf>>& pool, int L, int prec) {
  std::unique_ptr<DevBuf>& sp = pool[{L, prec}];
  const size_t bytes = (size_t)levels[L].lay->total * prec;
  if (!sp || sp->bytes != bytes) {
    sp.reset(new DevBuf());
    sp->alloc(bytes);
    cudaCheck(cudaMemsetAsync(sp->p, 0, sp->bytes, stream), "spare memset");  // alignment padding stays zero
  }
  return *sp;
}

int Storage::sorScheduleFor(int L, int prec) const {
  const int tuned = 2 * L + (prec == 4 ? 1 : 0);
  return (int)sorScheduleLevel.size() > tuned && sorScheduleLevel[tuned] >= 0 ? sorScheduleLevel[tuned] : sorSchedule;
}

void Storage::lincomb(int dst, int L, unsigned mask, int n, const double* a, const int* srcs, bool add,
                      double constant) {
  argCheck(n >= 0 && n <= 3, "at most three source functions");
  Function& fd = fn(dst);
  void* pd = data(dst, L);
  const void* ps[3] = {nullptr, nullptr, nullptr};
  double sc[3] = {0, 0, 0};
  for (int i = 0; i < n; ++i) {
    argCheck(fn(srcs[i]).prec == fd.prec, "assign/add require functions of equal precision");
    ps[i] = data(srcs[i], L);
    sc[i] = a[i];
  }
  const LevelData& ld = levels[L];
  if (ld.nChunks == 0) return;
  if (fd.prec == 8)
    dev::lincombKernel<double><<<ld.nChunks, dev::kBlock, 0, stream>>>(
        ld.chunks, mask, (double*)pd, n, (const double*)ps[0], (const double*)ps[1], (const double*)ps[2], sc[0], sc[1],
        sc[2], add ? 1 : 0, constant);
  else
    dev::lincombKernel<float><<<ld.nChunks, dev::kBlock, 0, stream>>>(
        ld.chunks, mask, (float*)pd, n, (const float*)ps[0], (const float*)ps[1], (const float*)ps[2], sc[0], sc[1],
        sc[2], add ? 1 : 0, constant);
  ++launches;
  cudaCheck(cudaGetLastError(), "lincomb");
}

void Storage::divideBy(int dst, int a, int b, int L, unsigned mask) {
  argCheck(fn(dst).prec == 8 && fn(a).prec == 8 && fn(b).prec == 8, "divide: FP64 functions required");
  const LevelData& ld = levels[L];
  if (!ld.nChunks) return;
  dev::divideKernel<<<ld.nChunks, dev::kBlock, 0, stream>>>(ld.chunks, mask, (double*)data(dst, L),
                                                             (const double*)data(a, L), (const double*)data(b, L));
  ++launches;
  cudaCheck(cudaGetLastError(), "divide");
}

void Storage::copyCast(int dst, int src, int L, unsigned mask, bool add) {
  Function& fd = fn(dst);
  Function& fs = fn(src);
  void* pd = data(dst, L);
  void* ps = data(src, L);
  const LevelData& ld = levels[L];
  if (ld.nChunks == 0) return;
  const int a = add ? 1 : 0;
  if (fd.prec == 8 && fs.prec == 8)
    dev::castKernel<double, double><<<ld.nChunks, dev::kBlock, 0, stream>>>(ld.chunks, mask, (double*)pd, (const double*)ps, a);
  else if (fd.prec == 8)
    dev::castKernel<double, float><<<ld.nChunks, dev::kBlock, 0, stream>>>(ld.chunks, mask, (double*)pd, (const float*)ps, a);
  else if (fs.prec == 8)
    dev::castKernel<float, double><<<ld.nChunks, dev::kBlock, 0, stream>>>(ld.chunks, mask, (float*)pd, (const double*)ps, a);
  else
    dev::castKernel<float, float><<<ld.nChunks, dev::kBlock, 0, stream>>>(ld.chunks, mask, (float*)pd, (const float*)ps, a);
  ++launches;
  cudaCheck(cudaGetLastError(), "copyCast");
}

void Storage::dotAsync(int a, int b, int L, unsigned mask, double* dOut) {
  Function& fa = fn(a);
  argCheck(fa.prec == fn(b).prec, "dot requires functions of equal precision");
  const LevelData& ld = levels[L];
  const int nb = ld.lv.nCellBlocks + ld.lv.nFaceBlocks + ld.lv.nLowBlocks;
  if (fa.prec == 8)
    dev::dotKernel<double><<<nb, dev::kBlock, 0, stream>>>(ld.lv, (const double*)data(a, L), (const double*)data(b, L), mask,
                                                           (double*)ld.partial.p);
  else
    dev::dotKernel<float><<<nb, dev::kBlock, 0, stream>>>(ld.lv, (const float*)data(a, L), (const float*)data(b, L), mask,
                                                          (double*)ld.partial.p);
  dev::reduceKernel<<<1, dev::kBlock, 0, stream>>>((const double*)ld.partial.p, nb, dOut);
  launches += 2;
  cudaCheck(cudaGetLastError(), "dot");
}

PackStage::~PackStage() {
  if (copied) cudaEventDestroy(copied);
  if (used) cudaEventDestroy(used);
}

const OwnedPack& Storage::ownedPack(int L) {
  argCheck(L >= 0 && L <= maxLevel(), "level out of range");
  std::unique_ptr<OwnedPack>& op = ownedPacks[L];
  if (!op) {
    const std::vector<SlotRun> runs = ownedRuns(disc, L);
    std::vector<dev::OwnedRun> dr;
    dr.reserve(runs.size());
    int64_t packed = 0;
    for (const SlotRun& r : runs) {
      argCheck(r.len > 0 && r.len < (int64_t(1) << 31), "owned run length");
      dr.push_back({r.slot, packed, (int)r.len, 0});
      packed += r.len;
    }
    std::unique_ptr<OwnedPack> p(new OwnedPack());
    p->nRuns = (int64_t)dr.size();
    p->count = packed;
    p->runs.alloc(std::max<size_t>(dr.size(), 1) * sizeof(dev::OwnedRun));
    if (!dr.empty())
      cudaCheck(cudaMemcpyAsync(p->runs.p, dr.data(), dr.size() * sizeof(dev::OwnedRun), cudaMemcpyHostToDevice, stream),
                "owned runs");
    cudaCheck(cudaStreamSynchronize(stream), "owned runs");
    op = std::move(p);
  }
  return *op;
}

static PackStage& packStage(Function& f, int L, int64_t count) {
  std::unique_ptr<PackStage>& ps = f.stage[L];
  if (!ps) {
    ps.reset(new PackStage());
    ps->buf.alloc(std::max<size_t>((size_t)count * f.prec, 16));
    cudaCheck(cudaEventCreateWithFlags(&ps->copied, cudaEventDisableTiming), "event");
    cudaCheck(cudaEventCreateWithFlags(&ps->used, cudaEventDisableTiming), "event");
  }
  return *ps;
}

static unsigned packGrid(int64_t nRuns) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((nRuns + 7) / 8, 148 * 16)); }

void Storage::uploadOwned(int id, int L, const void* host, int64_t n, cudaStream_t copyStream) {
  Function& f = fn(id);
  argCheck(L >= f.minL && L <= f.maxL, "level outside the function's range");
  argCheck(host != nullptr, "null host buffer");
  const OwnedPack& op = ownedPack(L);
  argCheck(n == op.count, "upload size must equal the number of owned DoFs of the level");
  PackStage& ps = packStage(f, L, op.count);
  cudaCheck(cudaStreamWaitEvent(copyStream, ps.used, 0), "wait");  // the previous unpack has read the buffer
  cudaCheck(cudaMemcpyAsync(ps.buf.p, host, (size_t)n * f.prec, cudaMemcpyHostToDevice, copyStream), "owned upload");
  cudaCheck(cudaEventRecord(ps.copied, copyStream), "event");
  cudaCheck(cudaStreamWaitEvent(stream, ps.copied, 0), "wait");
  if (op.nRuns) {
    if (f.prec == 8)
      dev::ownedPackKernel<double, false><<<packGrid(op.nRuns), dev::kBlock, 0, stream>>>(
          (const dev::OwnedRun*)op.runs.p, op.nRuns, (double*)data(id, L), (double*)ps.buf.p);
    else
      dev::ownedPackKernel<float, false><<<packGrid(op.nRuns), dev::kBlock, 0, stream>>>(
          (const dev::OwnedRun*)op.runs.p, op.nRuns, (float*)data(id, L), (float*)ps.buf.p);
    ++launches;
    cudaCheck(cudaGetLastError(), "owned unpack");
  }
  cudaCheck(cudaEventRecord(ps.used, stream), "event");
  communicate(id, L, kAllGroups);
}

void Storage::downloadOwned(int id, int L, void* host, int64_t n, cudaStream_t copyStream) {
  Function& f = fn(id);
  argCheck(L >= f.minL && L <= f.maxL, "level outside the function's range");
  argCheck(host != nullptr, "null host buffer");
  const OwnedPack& op = ownedPack(L);
  argCheck(n == op.count, "download size must equal the number of owned DoFs of the level");
  PackStage& ps = packStage(f, L, op.count);
  cudaCheck(cudaStreamWaitEvent(stream, ps.copied, 0), "wait");  // the previous download has left the buffer
  if (op.nRuns) {
    if (f.prec == 8)
      dev::ownedPackKernel<double, true><<<packGrid(op.nRuns), dev::kBlock, 0, stream>>>(
          (const dev::OwnedRun*)op.runs.p, op.nRuns, (double*)data(id, L), (double*)ps.buf.p);
    else
      dev::ownedPackKernel<float, true><<<packGrid(op.nRuns), dev::kBlock, 0, stream>>>(
          (const dev::OwnedRun*)op.runs.p, op.nRuns, (float*)data(id, L), (float*)ps.buf.p);
    ++launches;
    cudaCheck(cudaGetLastError(), "owned pack");
  }
  cudaCheck(cudaEventRecord(ps.used, stream), "event");
  cudaCheck(cudaStreamWaitEvent(copyStream, ps.used, 0), "wait");
  cudaCheck(cudaMemcpyAsync(host, ps.buf.p, (size_t)n * f.prec, cudaMemcpyDeviceToHost, copyStream), "owned download");
  cudaCheck(cudaEventRecord(ps.copied, copyStream), "event");
}

dev::BatchMap Storage::batchMap(int L, int copies) const {
  argCheck(copies >= 1, "batch: at least one copy");
  const LevelData& ld = levels[L];
  const LevelLayout& lay = *ld.lay;
  const dev::LevelDev& lv = ld.lv;
  dev::BatchMap bm{};
  bm.copies = copies;
  const int kinds[4] = {KC, KF, KE, KV};
  int64_t a = 0;
  for (int q = 0; q < 4; ++q) {
    const auto& off = lay.off[kinds[q]];
    const auto& sz = lay.size[kinds[q]];
    const int n = (int)off.size();
    argCheck(n % copies == 0, "batch: primitives are not a multiple of the copies");
    const int per = n / copies;
    int64_t end = lay.total;  // the kind's block ends where the next non-empty kind begins
    for (int r = q + 1; r < 4; ++r)
      if (!lay.off[kinds[r]].empty()) {
        end = lay.off[kinds[r]][0];
        break;
      }
    bm.uBase[q] = n ? off[0] : end;
    bm.size[q] = n ? (end - off[0]) / copies : 0;
    argCheck(!n || bm.size[q] * copies == end - off[0], "batch: kind block is not a multiple of the copies");
    for (int i = 0; i < copies && n; ++i)
      for (int p = 0; p < per; ++p) {
        const size_t u = (size_t)i * per + p;
        argCheck(off[u] - (bm.uBase[q] + i * bm.size[q]) == off[(size_t)p] - bm.uBase[q] && sz[u] == sz[(size_t)p],
                 "batch: the copies' layouts differ");
      }
    bm.aBase[q] = a;
    a += bm.size[q];
  }
  const int nCellGrid = lv.N >= 4 ? lv.nCells * (lv.N - 3) : 0;
  const int counts[4] = {nCellGrid, lv.nFaceBlocks, lv.nLowEdgeBlocks, lv.nLowBlocks - lv.nLowEdgeBlocks};
  int base = 0;
  for (int q = 0; q < 4; ++q) {
    argCheck(counts[q] % copies == 0, "batch: work blocks are not a multiple of the copies");
    bm.bBase[q] = base;
    bm.bCount[q] = counts[q] / copies;
    base += counts[q];
  }
  return bm;
}

void Storage::fillRandomBatch(int id, int L, unsigned mask, const dev::BatchMap& bm, const uint64_t* dSeeds, int active,
                              double lo, double hi) {
  Function& f = fn(id);
  const LevelData& ld = levels[L];
  if (ld.nChunks) {
    if (f.prec == 8)
      dev::randomFillBatchKernel<double><<<ld.nChunks, dev::kBlock, 0, stream>>>(ld.chunks, mask, (double*)data(id, L), bm,
                                                                               dSeeds, active, lo, hi);
    else
      dev::randomFillBatchKernel<float><<<ld.nChunks, dev::kBlock, 0, stream>>>(ld.chunks, mask, (float*)data(id, L), bm,
                                                                              dSeeds, active, lo, hi);
    ++launches;
    cudaCheck(cudaGetLastError(), "batch random fill");
  }
  communicate(id, L, kAllGroups);
}

void Storage::dotBatchAsync(int a, int b, int L, unsigned mask, const dev::BatchMap& bm, double* dOut) {
  Function& fa = fn(a);
  argCheck(fa.prec == fn(b).prec, "dot requires functions of equal precision");
  const LevelData& ld = levels[L];
  const int nb = ld.lv.nCellBlocks + ld.lv.nFaceBlocks + ld.lv.nLowBlocks;
  if (fa.prec == 8)
    dev::dotKernel<double><<<nb, dev::kBlock, 0, stream>>>(ld.lv, (const double*)data(a, L), (const double*)data(b, L), mask,
                                                           (double*)ld.partial.p);
  else
    dev::dotKernel<float><<<nb, dev::kBlock, 0, stream>>>(ld.lv, (const float*)data(a, L), (const float*)data(b, L), mask,
                                                          (double*)ld.partial.p);
  dev::batchReduceKernel<<<bm.copies, dev::kBlock, 0, stream>>>((const double*)ld.partial.p, bm, dOut);
  launches += 2;
  cudaCheck(cudaGetLastError(), "batch dot");
}

void Storage::copyBatchSlots(int src, int dst, int L, const dev::BatchMap& bm, int copy) {
  Function& fs = fn(src);
  argCheck(fs.prec == fn(dst).prec, "batch copy: precision mismatch");
  char* d = (char*)data(dst, L);
  const char* sp = (const char*)data(src, L);
  for (int q = 0; q < 4; ++q)
    if (bm.size[q] > 0) {
      const size_t o = (size_t)(bm.uBase[q] + copy * bm.size[q]) * fs.prec;
      cudaCheck(cudaMemcpyAsync(d + o, sp + o, (size_t)bm.size[q] * fs.prec, cudaMemcpyDeviceToDevice, stream),
                "batch copy");
    }
}

void Storage::interpolateExpr(int id, int L, unsigned mask, int expr, const double* p) {
  argCheck(expr == 0 || expr == 1, "unknown expression");
  Function& f = fn(id);
  const LevelData& ld = levels[L];
  const int nb = ld.lv.nCellBlocks + ld.lv.nFaceBlocks + ld.lv.nLowBlocks;
  if (f.prec == 8)
    dev::interpolateKernel<double><<<nb, dev::kBlock, 0, stream>>>(ld.lv, geom, (double*)data(id, L), mask, expr, p[0], p[1],
                                                                   p[2], p[3]);
  else
    dev::interpolateKernel<float><<<nb, dev::kBlock, 0, stream>>>(ld.lv, geom, (float*)data(id, L), mask, expr, p[0], p[1],
                                                                  p[2], p[3]);
  ++launches;
  cudaCheck(cudaGetLastError(), "interpolate");
  communicate(id, L, kAllGroups);
}

void Storage::fillRandom(int id, int L, unsigned mask, uint64_t seed, double lo, double hi) {
  Function& f = fn(id);
  const LevelData& ld = levels[L];
  if (ld.nChunks) {
    if (f.prec == 8)
      dev::randomFillKernel<double><<<ld.nChunks, dev::kBlock, 0, stream>>>(ld.chunks, mask, (double*)data(id, L), seed, lo, hi);
    else
      dev::randomFillKernel<float><<<ld.nChunks, dev::kBlock, 0, stream>>>(ld.chunks, mask, (float*)data(id, L), seed, lo, hi);
    ++launches;
    cudaCheck(cudaGetLastError(), "random fill");
  }
  communicate(id, L, kAllGroups);
}

int64_t Storage::deviceBytes() const {
  int64_t b = (int64_t)scalars.bytes;
  for (auto& g : geomKeep) b += (int64_t)g->bytes;
  for (const LevelData& ld : levels) {
    for (auto& k : ld.keep) b += (int64_t)k->bytes;
    if (ld.tileBuf) b += (int64_t)ld.tileBuf->bytes;
    b += (int64_t)ld.partial.bytes;
  }
  for (auto& f : fns)
    for (auto& l : f.second->levels) b += (int64_t)l->bytes;
  for (auto& o : ops)
    for (auto& k : o.second->keep) b += (int64_t)k->bytes;
  for (auto& sp : spare)
    if (sp.second) b += (int64_t)sp.second->bytes;
  for (auto& sp : splitRhs)
    if (sp.second) b += (int64_t)sp.second->bytes;
  return b;
}

double Storage::dot(int a, int b, int L, unsigned mask) {
  double* d = (double*)scalars.p;
  dotAsync(a, b, L, mask, d);
  double h = 0;
  cudaCheck(cudaMemcpyAsync(&h, d, sizeof(double), cudaMemcpyDeviceToHost, stream), "dot readback");
  cudaCheck(cudaStreamSynchronize(stream), "dot sync");
  return h;
}

// ------------------------------------------------------------------------------------------
// operators
// ------------------------------------------------------------------------------------------
template <class T>
static dev::StencilDev<T> packStencil(std::vector<std::unique_ptr<DevBuf>>& keep, const LevelStencils& st,
                                      cudaStream_t stream) {
  std::vector<T> cellW;
  for (auto& c : st.cell)
    for (int k = 0; k < 16; ++k) cellW.push_back(T(c[k]));
  std::vector<dev::FaceEnt<T>> fe(st.face.size() * 16);
  std::vector<int> fc(st.face.size());
  for (size_t f = 0; f < st.face.size(); ++f) {
    argCheck(st.face[f].size() <= 16, "face stencil exceeds 16 entries");
    fc[f] = (int)st.face[f].size();
    for (size_t k = 0; k < st.face[f].size(); ++k)
      fe[16 * f + k] = {T(st.face[f][k].w), st.face[f][k].layer, st.face[f][k].dx, st.face[f][k].dy};
  }
  std::vector<int> off{0};
  std::vector<int64_t> rel;
  std::vector<T> wv;
  auto addLow = [&](const std::vector<LowEntry>& ent) {
    for (auto& e : ent) {
      rel.push_back(e.rel);
      wv.push_back(T(e.w));
    }
    off.push_back((int)rel.size());
  };
  for (auto& e : st.edge) addLow(e);
  for (auto& v : st.vert) addLow(v);
  dev::StencilDev<T> d;
  d.cellW = (const T*)upload(keep, cellW, stream);
  d.faceEnt = (const dev::FaceEnt<T>*)upload(keep, fe, stream);
  d.faceEntCount = (const int*)upload(keep, fc, stream);
  d.lowEntOff = (const int*)upload(keep, off, stream);
  d.lowEntRel = (const int64_t*)upload(keep, rel, stream);
  d.lowEntW = (const T*)upload(keep, wv, stream);
  return d;
}

// New stencil values into the device arrays of an existing operator (same topology, so the same
// sizes and index arrays): no device allocation or release, only copies on this stream.
template <class T>
static void refillStencil(const dev::StencilDev<T>& d, const LevelStencils& st, cudaStream_t stream) {
  std::vector<T> cellW;
  for (auto& c : st.cell)
    for (int k = 0; k < 16; ++k) cellW.push_back(T(c[k]));
  std::vector<dev::FaceEnt<T>> fe(st.face.size() * 16);
  for (size_t f = 0; f < st.face.size(); ++f)
    for (size_t k = 0; k < st.face[f].size(); ++k)
      fe[16 * f + k] = {T(st.face[f][k].w), st.face[f][k].layer, st.face[f][k].dx, st.face[f][k].dy};
  std::vector<T> wv;
  for (auto& e : st.edge)
    for (auto& x : e) wv.push_back(T(x.w));
  for (auto& v : st.vert)
    for (auto& x : v) wv.push_back(T(x.w));
  if (!cellW.empty())
    cudaCheck(cudaMemcpyAsync((void*)d.cellW, cellW.data(), cellW.size() * sizeof(T), cudaMemcpyHostToDevice, stream),
              "stencil refill");
  if (!fe.empty())
    cudaCheck(cudaMemcpyAsync((void*)d.faceEnt, fe.data(), fe.size() * sizeof(fe[0]), cudaMemcpyHostToDevice, stream),
              "stencil refill");
  if (!wv.empty())
    cudaCheck(cudaMemcpyAsync((void*)d.lowEntW, wv.data(), wv.size() * sizeof(T), cudaMemcpyHostToDevice, stream),
              "stencil refill");
  cudaCheck(cudaStreamSynchronize(stream), "stencil refill");
}

static std::vector<double> p2Stencils(const std::vector<double>& K, int nCells);
static std::vector<double> p2FaceStencils(const std::vector<double>& K, int nCells);

int Storage::createP2Operator(int form, int minL, int maxL) {
  argCheck(form == FORM_LAPLACE, "P2 operators: only the Laplace form is available");
  argCheck(minL >= 0 && maxL + 1 <= maxLevel() && minL <= maxL,
           "P2 level range needs the storage's levels up to max_level + 1");
  std::unique_ptr<P2Operator> o(new P2Operator());
  o->form = form;
  o->minL = minL;
  o->maxL = maxL;
  for (int L = minL; L <= maxL; ++L) {
    const std::vector<double> K = p2CellElements(disc.topo(), L);
    std::vector<float> Kf(K.begin(), K.end());
    o->kd.emplace_back(new DevBuf());
    o->kd.back()->alloc(K.size() * sizeof(double));
    cudaCheck(cudaMemcpyAsync(o->kd.back()->p, K.data(), K.size() * sizeof(double), cudaMemcpyHostToDevice, stream),
              "P2 upload");
    o->kf.emplace_back(new DevBuf());
    o->kf.back()->alloc(Kf.size() * sizeof(float));
    cudaCheck(cudaMemcpyAsync(o->kf.back()->p, Kf.data(), Kf.size() * sizeof(float), cudaMemcpyHostToDevice, stream),
              "P2 upload");
    const std::vector<double> S = p2Stencils(K, (int)disc.topo().cells.size());
    std::vector<float> Sf(S.begin(), S.end());
    o->sd.emplace_back(new DevBuf());
    o->sd.back()->alloc(S.size() * sizeof(double));
    cudaCheck(cudaMemcpyAsync(o->sd.back()->p, S.data(), S.size() * sizeof(double), cudaMemcpyHostToDevice, stream),
              "P2 upload");
    o->sf.emplace_back(new DevBuf());
    o->sf.back()->alloc(Sf.size() * sizeof(float));
    cudaCheck(cudaMemcpyAsync(o->sf.back()->p, Sf.data(), Sf.size() * sizeof(float), cudaMemcpyHostToDevice, stream),
              "P2 upload");
    const std::vector<double> F = p2FaceStencils(K, (int)disc.topo().cells.size());
    std::vector<float> Ff(F.begin(), F.end());
    o->fd.emplace_back(new DevBuf());
    o->fd.back()->alloc(F.size() * sizeof(double));
    cudaCheck(cudaMemcpyAsync(o->fd.back()->p, F.data(), F.size() * sizeof(double), cudaMemcpyHostToDevice, stream),
              "P2 upload");
    o->ff.emplace_back(new DevBuf());
    o->ff.back()->alloc(Ff.size() * sizeof(float));
    cudaCheck(cudaMemcpyAsync(o->ff.back()->p, Ff.data(), Ff.size() * sizeof(float), cudaMemcpyHostToDevice, stream),
              "P2 upload");
    cudaCheck(cudaStreamSynchronize(stream), "P2 upload");
  }
  const int id = nextId++;
  p2ops[id] = std::move(o);
  return id;
}

static dev::P2Tables p2Tables() {
  dev::P2Tables tb{};
  for (int t = 0; t < 6; ++t) {
    tb.widthRed[t] = (unsigned char)kMicroCellWidth[t];
    for (int j = 0; j < 10; ++j)
      for (int d = 0; d < 3; ++d)
        tb.off[t][j][d] = (signed char)(j < 4 ? 2 * kMicroCellTable[t][j][d]
                                              : kMicroCellTable[t][kP2Edge[j - 4][0]][d] +
                                                    kMicroCellTable[t][kP2Edge[j - 4][1]][d]);
  }
  for (int t = 0; t < 6; ++t)
    for (int j = 0; j < 10; ++j) {
      const int pc = (tb.off[t][j][0] & 1) | ((tb.off[t][j][1] & 1) << 1) | ((tb.off[t][j][2] & 1) << 2);
      argCheck(tb.nCand[pc] < 24, "P2 candidate table overflow");
      tb.cand[pc][tb.nCand[pc]][0] = (unsigned char)t;
      tb.cand[pc][tb.nCand[pc]][1] = (unsigned char)j;
      ++tb.nCand[pc];
    }
  return tb;
}

P2Additive& Storage::p2Additive(int Lf) {
  if ((int)p2add.size() <= Lf) p2add.resize(maxLevel() + 1);
  P2Additive& ad = p2add[Lf];
  if (ad.built) return ad;
  const LevelData& ld = levels[Lf];
  // owner <- its copies in the closure slots of its cells (the cell-closure halo group)
  std::map<int64_t, std::vector<int64_t>> byOwner;
  const auto& cd = ld.lay->commDst[G_CELL];
  const auto& cs = ld.lay->commSrc[G_CELL];
  for (size_t i = 0; i < cd.size(); ++i) byOwner[cs[i]].push_back(cd[i]);
  std::vector<int64_t> own, cp;
  std::vector<int> ptr{0};
  std::vector<unsigned char> ty;
  auto typeOf = [&](int64_t slot) {  // DoF type of the primitive whose array holds the slot
    for (int k : {KF, KE, KV})
      for (size_t pr = 0; pr < ld.lay->off[k].size(); ++pr)
        if (slot >= ld.lay->off[k][pr] && slot < ld.lay->off[k][pr] + ld.lay->size[k][pr])
          return k == KF ? ld.hostFaceType[pr] : k == KE ? ld.hostLowType[pr] : ld.hostLowType[ld.lv.nEdges + pr];
    throw Error(HG_ERR_INTERNAL, "owner slot outside the face, edge and vertex arrays");
  };
  for (auto& kv : byOwner) {
    own.push_back(kv.first);
    for (int64_t c : kv.second) cp.push_back(c);
    ptr.push_back((int)cp.size());
    ty.push_back(typeOf(kv.first));
  }
  ad.n = (int)own.size();
  ad.owner.alloc(std::max<size_t>(1, own.size()) * sizeof(int64_t));
  ad.ptr.alloc(ptr.size() * sizeof(int));
  ad.copies.alloc(std::max<size_t>(1, cp.size()) * sizeof(int64_t));
  ad.type.alloc(std::max<size_t>(1, ty.size()));
  if (!own.empty()) {
    cudaCheck(cudaMemcpyAsync(ad.owner.p, own.data(), own.size() * sizeof(int64_t), cudaMemcpyHostToDevice, stream), "p2 add");
    cudaCheck(cudaMemcpyAsync(ad.copies.p, cp.data(), cp.size() * sizeof(int64_t), cudaMemcpyHostToDevice, stream), "p2 add");
    cudaCheck(cudaMemcpyAsync(ad.type.p, ty.data(), ty.size(), cudaMemcpyHostToDevice, stream), "p2 add");
  }
  cudaCheck(cudaMemcpyAsync(ad.ptr.p, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice, stream), "p2 add");
  // colour of every slot (the colour of the DoF it holds; bit 7 set on the owner slot): from the
  // DoF's barycentric weights in ascending vertex-ID order (b0, b1, b2, b3), parity class
  // p = (b1 & 1) | (b2 & 1) << 1 | (b3 & 1) << 2; p = 0 (micro-vertices of the coarse level) is
  // split into ((b1 >> 1) + 2 (b2 >> 1) + 3 (b3 >> 1)) mod 4, the others are colours 3 + p
  std::vector<unsigned char> col((size_t)ld.lay->total, 0x7f);
  const bool keepOwners = ld.lay->total <= (int64_t(1) << 20);  // small (coarse) levels only
  for (int k = 0; k < 4; ++k)
    for (size_t pr = 0; pr < ld.lay->off[k].size(); ++pr)
      for (int64_t loc = 0; loc < ld.lay->size[k][pr]; ++loc) {
        const Bary b = disc.slotBary(Lf, k, (int)pr, loc);
        int64_t w[4] = {0, 0, 0, 0};
        for (int i = 0; i < b.n; ++i) w[i] = b.b[i];
        const int par = int(w[1] & 1) | (int(w[2] & 1) << 1) | (int(w[3] & 1) << 2);
        int c = par ? 3 + par : int(((w[1] >> 1) + 2 * (w[2] >> 1) + 3 * (w[3] >> 1)) % 4);
        const Slot o = disc.owner(Lf, b);
        if (o.kind == k && o.prim == (int)pr && o.local == loc) {
          c |= 0x80;
          if (!keepOwners) {
            col[(size_t)(ld.lay->off[k][pr] + loc)] = (unsigned char)c;
            continue;
          }
          ad.hostOwner.push_back(ld.lay->off[k][pr] + loc);
          ad.hostOwnerType.push_back(k == KC   ? ld.hostCellType[pr]
                                     : k == KF ? ld.hostFaceType[pr]
                                     : k == KE ? ld.hostLowType[pr]
                                               : ld.hostLowType[ld.lv.nEdges + pr]);
        }
        col[(size_t)(ld.lay->off[k][pr] + loc)] = (unsigned char)c;
      }
  ad.colour.alloc(col.size());
  cudaCheck(cudaMemcpyAsync(ad.colour.p, col.data(), col.size(), cudaMemcpyHostToDevice, stream), "p2 colour");
  // the parity class of each colour's interior nodes per cell: an edge class is one colour in a
  // cell's frame (read at its interior node nearest the origin), the vertex class holds colours 0-3
  {
    const int64_t M = ld.lv.N, w = M + 1;
    auto tet = [](int64_t n) { return n * (n + 1) * (n + 2) / 6; };
    std::vector<signed char> cls((size_t)ld.lv.nCells * 12, -1);
    auto colourAt = [&](int c, int64_t X, int64_t Y, int64_t Z) {
      const int64_t loc = tet(w) - tet(w - Z) + Y * (w - Z + 1) - Y * (Y + 1) / 2 + X;
      return col[(size_t)(ld.lay->off[KC][c] + loc)] & 0x7f;
    };
    for (int c = 0; c < ld.lv.nCells; ++c) {
      for (int k = 0; k < 4 && M >= 8; ++k) cls[(size_t)c * 12 + k] = 0;
      // step of the vertex colour along a row (1 when a row holds at most one interior vertex node)
      cls[(size_t)c * 12 + 11] = (signed char)(M >= 16 ? (colourAt(c, 4, 2, 2) - colourAt(c, 2, 2, 2)) & 3 : 1);
      argCheck(cls[(size_t)c * 12 + 11] != 0, "P2 vertex colours do not change along a row");
      for (int pc = 1; pc < 8; ++pc) {
        const int64_t X = (pc & 1) ? 1 : 2, Y = (pc & 2) ? 1 : 2, Z = (pc & 4) ? 1 : 2;
        if (X + Y + Z > M - 1) continue;
        const int colr = colourAt(c, X, Y, Z);
        argCheck(colr >= 4 && colr < 11 && cls[(size_t)c * 12 + colr] < 0, "P2 colour classes are inconsistent");
        cls[(size_t)c * 12 + colr] = (signed char)pc;
      }
    }
    ad.classOfColour.alloc(cls.size());
    cudaCheck(cudaMemcpyAsync(ad.classOfColour.p, cls.data(), cls.size(), cudaMemcpyHostToDevice, stream), "p2 colour");
    // closure nodes of every cell grouped by colour (then by face-stencil entry, so that the warps
    // of the list kernel mostly run one stencil)
    auto faceEntry = [](int f, int pc) {
      switch (f) {
        case 0: return pc;
        case 1: return 4 + ((pc & 1) | ((pc >> 1) & 2));
        case 2: return 8 + (((pc >> 1) & 1) | ((pc >> 1) & 2));
        default: return 12 + (pc == 0 ? 0 : pc == 3 ? 1 : pc == 5 ? 2 : 3);
      }
    };
    std::vector<std::pair<int, dev::P2ClosureNode>> nodes;
    for (int c = 0; c < ld.lv.nCells; ++c)
      for (int64_t Z = 0; Z <= M; ++Z)
        for (int64_t Y = 0; Y <= M - Z; ++Y)
          for (int64_t X = 0; X <= M - Z - Y; ++X) {
            const bool on[4] = {Z == 0, Y == 0, X == 0, X + Y + Z == M};
            const int nOn = on[0] + on[1] + on[2] + on[3];
            if (nOn == 0) continue;
            int k = -1;
            if (nOn == 1) {
              const int f = on[0] ? 0 : on[1] ? 1 : on[2] ? 2 : 3;
              k = faceEntry(f, int((X & 1) | ((Y & 1) << 1) | ((Z & 1) << 2)));
            }
            dev::P2ClosureNode nd{c, (unsigned short)X, (unsigned short)Y, (unsigned short)Z, (signed char)k, 0};
            nodes.push_back({colourAt(c, X, Y, Z) * 32 + (k + 1), nd});
          }
    std::stable_sort(nodes.begin(), nodes.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    std::vector<dev::P2ClosureNode> list(nodes.size());
    for (int k = 0; k < 12; ++k) ad.closureBegin[k] = 0;
    int cur = 0;
    for (size_t i = 0; i < nodes.size(); ++i) {
      list[i] = nodes[i].second;
      const int colr = nodes[i].first / 32;
      argCheck(colr < 11, "closure node without an SOR colour");
      while (cur < colr) ad.closureBegin[++cur] = (int)i;
    }
    while (cur < 11) ad.closureBegin[++cur] = (int)nodes.size();
    // the owner updates by colour: face, edge and vertex owners (indices into the owner table)
    // and, for the vertex colours, the interior vertex nodes of the cells
    std::vector<std::vector<int>> addBy(11);
    for (size_t i = 0; i < own.size(); ++i) addBy[col[(size_t)own[i]] & 0x7f].push_back((int)i);
    std::vector<std::vector<int64_t>> innerBy(4);
    std::vector<std::vector<unsigned char>> innerTy(4);
    for (int c = 0; c < ld.lv.nCells; ++c)
      for (int64_t Z = 2; Z <= M - 1; Z += 2)
        for (int64_t Y = 2; Y + Z <= M - 1; Y += 2)
          for (int64_t X = 2; X + Y + Z <= M - 1; X += 2) {
            const int colr = colourAt(c, X, Y, Z);
            const int64_t loc = tet(w) - tet(w - Z) + Y * (w - Z + 1) - Y * (Y + 1) / 2 + X;
            innerBy[colr].push_back(ld.lay->off[KC][c] + loc);
            innerTy[colr].push_back(ld.hostCellType[c]);
          }
    std::vector<int> addFlat;
    std::vector<int64_t> innerFlat;
    std::vector<unsigned char> innerTyFlat;
    for (int k = 0; k < 11; ++k) {
      ad.updAddBegin[k] = (int)addFlat.size();
      addFlat.insert(addFlat.end(), addBy[k].begin(), addBy[k].end());
      ad.updInnerBegin[k] = (int)innerFlat.size();
      if (k < 4) {
        innerFlat.insert(innerFlat.end(), innerBy[k].begin(), innerBy[k].end());
        innerTyFlat.insert(innerTyFlat.end(), innerTy[k].begin(), innerTy[k].end());
      }
    }
    ad.updAddBegin[11] = (int)addFlat.size();
    ad.updInnerBegin[11] = (int)innerFlat.size();
    ad.updAdd.alloc(std::max<size_t>(1, addFlat.size()) * sizeof(int));
    ad.updInner.alloc(std::max<size_t>(1, innerFlat.size()) * sizeof(int64_t));
    ad.updInnerType.alloc(std::max<size_t>(1, innerTyFlat.size()));
    if (!addFlat.empty())
      cudaCheck(cudaMemcpyAsync(ad.updAdd.p, addFlat.data(), addFlat.size() * sizeof(int), cudaMemcpyHostToDevice, stream),
                "p2 update lists");
    if (!innerFlat.empty()) {
      cudaCheck(cudaMemcpyAsync(ad.updInner.p, innerFlat.data(), innerFlat.size() * sizeof(int64_t),
                                cudaMemcpyHostToDevice, stream),
                "p2 update lists");
      cudaCheck(cudaMemcpyAsync(ad.updInnerType.p, innerTyFlat.data(), innerTyFlat.size(), cudaMemcpyHostToDevice, stream),
                "p2 update lists");
    }
    ad.closureList.alloc(std::max<size_t>(1, list.size()) * sizeof(dev::P2ClosureNode));
    if (!list.empty())
      cudaCheck(cudaMemcpyAsync(ad.closureList.p, list.data(), list.size() * sizeof(dev::P2ClosureNode),
                                cudaMemcpyHostToDevice, stream),
                "p2 closure list");
  }
  std::vector<unsigned char> mult((size_t)ld.lay->total, 1);
  for (size_t i = 0; i + 1 < ptr.size(); ++i)
    for (int k = ptr[i]; k < ptr[i + 1]; ++k) mult[(size_t)cp[k]] = (unsigned char)(ptr[i + 1] - ptr[i]);
  ad.mult.alloc(mult.size());
  cudaCheck(cudaMemcpyAsync(ad.mult.p, mult.data(), mult.size(), cudaMemcpyHostToDevice, stream), "p2 mult");
  cudaCheck(cudaStreamSynchronize(stream), "p2 add");
  ad.built = true;
  return ad;
}

static const dev::P2Tables& p2TablesOnce() {
  static const dev::P2Tables tb = p2Tables();
  return tb;
}

// Interior stencil weights of every cell: for each parity class, the sum over the class's
// candidate micro-cells (type t, local node j) of row j of their element matrices, scattered
// to the lattice offsets of the ten nodes in the order of p2s::kOff.
static std::vector<double> p2Stencils(const std::vector<double>& K, int nCells) {
  const dev::P2Tables& tb = p2TablesOnce();
  std::vector<double> S((size_t)nCells * p2s::kTotal, 0.0);
  for (int c = 0; c < nCells; ++c)
    for (int pc = 0; pc < 8; ++pc) {
      double* sc = S.data() + (size_t)c * p2s::kTotal + p2s::kFirst[pc];
      for (int k = 0; k < tb.nCand[pc]; ++k) {
        const int t = tb.cand[pc][k][0], j = tb.cand[pc][k][1];
        for (int m = 0; m < 10; ++m) {
          int e = 0;
          while (e < p2s::kLen[pc] && !(p2s::kOff[pc][e][0] == tb.off[t][m][0] - tb.off[t][j][0] &&
                                        p2s::kOff[pc][e][1] == tb.off[t][m][1] - tb.off[t][j][1] &&
                                        p2s::kOff[pc][e][2] == tb.off[t][m][2] - tb.off[t][j][2]))
            ++e;
          if (e == p2s::kLen[pc]) throw Error(HG_ERR_INTERNAL, "P2 stencil offset table does not match the micro-cells");
          sc[e] += K[(size_t)c * 600 + t * 100 + j * 10 + m];
        }
      }
    }
  return S;
}

// Face-interior stencil weights of every cell: per (face, class) entry k, the sum over its
// micro-cells p2s::kFaceCand[k] of their element rows, scattered to the offsets p2s::kFaceOff[k].
static std::vector<double> p2FaceStencils(const std::vector<double>& K, int nCells) {
  const dev::P2Tables& tb = p2TablesOnce();
  std::vector<double> S((size_t)nCells * p2s::kFaceTotal, 0.0);
  for (int c = 0; c < nCells; ++c)
    for (int k = 0; k < p2s::kFaceStencils; ++k) {
      double* sc = S.data() + (size_t)c * p2s::kFaceTotal + p2s::kFaceFirst[k];
      for (int q = 0; q < p2s::kFaceNCand[k]; ++q) {
        const int t = p2s::kFaceCand[k][q][0], j = p2s::kFaceCand[k][q][1];
        for (int m = 0; m < 10; ++m) {
          int e = 0;
          while (e < p2s::kFaceLen[k] && !(p2s::kFaceOff[k][e][0] == tb.off[t][m][0] - tb.off[t][j][0] &&
                                           p2s::kFaceOff[k][e][1] == tb.off[t][m][1] - tb.off[t][j][1] &&
                                           p2s::kFaceOff[k][e][2] == tb.off[t][m][2] - tb.off[t][j][2]))
            ++e;
          if (e == p2s::kFaceLen[k]) throw Error(HG_ERR_INTERNAL, "P2 face stencil table does not match the micro-cells");
          sc[e] += K[(size_t)c * 600 + t * 100 + j * 10 + m];
        }
      }
    }
  return S;
}

// Cell gather + additive owner sums for one P2 level: dst = A src, rhs - A src or diag(A), on the
// flagged DoFs of colour `sel` (all when sel < 0). The copies of dst are not refreshed here.
template <class T, int MODE>
void Storage::p2Launch(P2Operator& o, int L, T* dst, const T* src, const T* rhs, unsigned mask, int sel) {
  const int Lf = L + 1;
  const LevelData& ld = levels[Lf];
  P2Additive& ad = p2Additive(Lf);
  const T* K = (const T*)(sizeof(T) == 8 ? o.kd[L - o.minL]->p : o.kf[L - o.minL]->p);
  const int nb = ld.lv.nCells * (ld.lv.N + 1);
  const unsigned char* col = (const unsigned char*)ad.colour.p;
  if constexpr (MODE == dev::MODE_DIAG) {
    dev::p2CellKernel<T, MODE><<<nb, dev::kBlock, 0, stream>>>(ld.lv, p2TablesOnce(), K, dst, src, rhs, mask, col, sel);
    ++launches;
  } else {
    // interior nodes by their constant stencils, closure nodes by the element gather
    if (ld.lv.N >= 4) {
      const T* W = (const T*)(sizeof(T) == 8 ? o.sd[L - o.minL]->p : o.sf[L - o.minL]->p);
      dev::p2StencilKernel<T, MODE><<<ld.lv.nCells * (ld.lv.N - 3), dev::kBlock, 0, stream>>>(
          ld.lv, W, dst, src, rhs, mask, col, (const signed char*)ad.classOfColour.p, sel, T(0));
      ++launches;
    }
    const T* FW = (const T*)(sizeof(T) == 8 ? o.fd[L - o.minL]->p : o.ff[L - o.minL]->p);
    dev::p2ClosureKernel<T><<<ld.lv.nCells * (ld.lv.N + dev::p2FaceChunks(ld.lv.N)), dev::kBlock, 0, stream>>>(
        ld.lv, p2TablesOnce(), K, FW, dst, src, col, sel);
    ++launches;
  }
  if (ad.n) {
    constexpr int AM = MODE == dev::MODE_RESIDUAL ? dev::MODE_RESIDUAL : dev::MODE_REPLACE;
    dev::p2AddKernel<T, AM><<<(ad.n + dev::kBlock - 1) / dev::kBlock, dev::kBlock, 0, stream>>>(
        (const int64_t*)ad.owner.p, (const int*)ad.ptr.p, (const int64_t*)ad.copies.p, (const unsigned char*)ad.type.p,
        ad.n, dst, rhs, mask, col, sel);
    ++launches;
  }
  cudaCheck(cudaGetLastError(), "P2 kernels");
}

P2Operator& Storage::p2op(int id) {
  auto it = p2ops.find(id);
  argCheck(it != p2ops.end(), "unknown P2 operator handle");
  return *it->second;
}

void Storage::p2Apply(int opId, int src, int dst, int rhs, int L, unsigned mask, int mode) {
  P2Operator& o = p2op(opId);
  argCheck(L >= o.minL && L <= o.maxL, "level outside the P2 operator's level range");
  argCheck(src != dst && (mode == 0 || (rhs != dst && rhs != src)), "P2 apply: distinct functions required");
  const int Lf = L + 1;
  Function& fs = fn(src);
  argCheck(fs.prec == fn(dst).prec && (mode == 0 || fn(rhs).prec == fs.prec), "P2 apply: precision mismatch");
  communicate(src, Lf, 1 << G_CELL);  // the closure copies of every cell hold the owners' values
  if (fs.prec == 8) {
    const double* r = mode ? (const double*)data(rhs, Lf) : nullptr;
    if (mode == 0)
      p2Launch<double, dev::MODE_REPLACE>(o, L, (double*)data(dst, Lf), (const double*)data(src, Lf), r, mask, -1);
    else
      p2Launch<double, dev::MODE_RESIDUAL>(o, L, (double*)data(dst, Lf), (const double*)data(src, Lf), r, mask, -1);
  } else {
    const float* r = mode ? (const float*)data(rhs, Lf) : nullptr;
    if (mode == 0)
      p2Launch<float, dev::MODE_REPLACE>(o, L, (float*)data(dst, Lf), (const float*)data(src, Lf), r, mask, -1);
    else
      p2Launch<float, dev::MODE_RESIDUAL>(o, L, (float*)data(dst, Lf), (const float*)data(src, Lf), r, mask, -1);
  }
  communicate(dst, Lf, kAllGroups);
}

// Diagonal of a P2 operator level as a function of that level (built once per precision).
int Storage::p2Diagonal(int opId, int L, int prec) {
  P2Operator& o = p2op(opId);
  auto key = std::make_pair(L, prec);
  auto it = o.diag.find(key);
  if (it != o.diag.end()) return it->second;
  const int Lf = L + 1;
  const int d = createFunction(Lf, Lf, prec);
  if (prec == 8)
    p2Launch<double, dev::MODE_DIAG>(o, L, (double*)data(d, Lf), nullptr, nullptr, HG_ALL, -1);
  else
    p2Launch<float, dev::MODE_DIAG>(o, L, (float*)data(d, Lf), nullptr, nullptr, HG_ALL, -1);
  communicate(d, Lf, kAllGroups);
  o.diag[key] = d;
  return d;
}

template <class T>
void Storage::p2SorT(P2Operator& o, int opId, int x, int b, int L, unsigned mask, T omega, bool backwards) {
  const int Lf = L + 1;
  const int prec = (int)sizeof(T);
  const int dg = p2Diagonal(opId, L, prec);
  const auto key = p2ScratchKey(Lf, prec);
  if (!p2scratch.count(key)) p2scratch[key] = createFunction(Lf, Lf, prec);
  const int ax = p2scratch[key];
  const LevelData& ld = levels[Lf];
  P2Additive& ad = p2Additive(Lf);
  const T* K = (const T*)(sizeof(T) == 8 ? o.kd[L - o.minL]->p : o.kf[L - o.minL]->p);
  const T* W = (const T*)(sizeof(T) == 8 ? o.sd[L - o.minL]->p : o.sf[L - o.minL]->p);
  const T* FW = (const T*)(sizeof(T) == 8 ? o.fd[L - o.minL]->p : o.ff[L - o.minL]->p);
  const unsigned char* col = (const unsigned char*)ad.colour.p;
  for (int k = 0; k < 11; ++k) {
    const int c = backwards ? 10 - k : k;
    // the cell-closure copies: all at the first colour; after that the owners kernel of each colour
    // writes its owners' new values into their copies
    if (k == 0) communicate(x, Lf, 1 << G_CELL);
    T* xd = (T*)data(x, Lf);
    const T* bd = (const T*)data(b, Lf);
    T* axd = (T*)data(ax, Lf);
    // face, edge and vertex DoFs of colour c: each cell's share of A x from the pass's start values
    // (the colours of DoFs on different primitives are defined in different vertex frames, so a
    // closure DoF may couple to an interior DoF of the same colour: its share is taken first)
    const int nList = ad.closureBegin[c + 1] - ad.closureBegin[c];
    if (nList > 0) {
      dev::p2ClosureListKernel<T><<<(nList + dev::kBlock - 1) / dev::kBlock, dev::kBlock, 0, stream>>>(
          ld.lv, p2TablesOnce(), K, FW, axd, xd, (const dev::P2ClosureNode*)ad.closureList.p + ad.closureBegin[c],
          nList);
      ++launches;
    }
    // interior nodes of colour c. An edge colour is one parity class in a cell's frame and couples
    // to no other node of its class, so those are updated in place (the closure copies keep their
    // start values until the next refresh). The four vertex colours ((b1 + 2 b2 + 3 b3) / 2 mod 4
    // in ascending vertex-ID order) separate the micro-edges along the macro-edges but not every
    // diagonal micro-edge (barycentric step (1, -1, 1, -1)), so a vertex colour takes A x into the
    // scratch first and is updated with the other owners.
    const bool vertexColour = c < 4;
    if (ld.lv.N >= 4) {
      const signed char* cls = (const signed char*)ad.classOfColour.p;
      if (vertexColour)
        dev::p2StencilKernel<T, dev::MODE_REPLACE><<<ld.lv.nCells * (ld.lv.N - 3), dev::kBlock, 0, stream>>>(
            ld.lv, W, axd, xd, nullptr, mask, col, cls, c, T(0));
      else
        dev::p2StencilKernel<T, dev::MODE_SOR><<<ld.lv.nCells * (ld.lv.N - 3), dev::kBlock, 0, stream>>>(
            ld.lv, W, xd, xd, bd, mask, col, cls, c, omega);
      ++launches;
    }
    // owner sums of the shares and the update of the face, edge and vertex DoFs (of the cell
    // interiors too for a vertex colour)
    const int nAdd = ad.updAddBegin[c + 1] - ad.updAddBegin[c];
    const int nInner = ad.updInnerBegin[c + 1] - ad.updInnerBegin[c];
    if (nAdd + nInner > 0) {
      dev::p2SorOwnersKernel<T><<<(nAdd + nInner + dev::kBlock - 1) / dev::kBlock, dev::kBlock, 0, stream>>>(
          (const int64_t*)ad.owner.p, (const int*)ad.ptr.p, (const int64_t*)ad.copies.p, (const unsigned char*)ad.type.p,
          (const int*)ad.updAdd.p + ad.updAddBegin[c], nAdd, (const int64_t*)ad.updInner.p + ad.updInnerBegin[c],
          (const unsigned char*)ad.updInnerType.p + ad.updInnerBegin[c], nInner, mask, xd, bd, axd,
          (const T*)data(dg, Lf), omega);
      ++launches;
    }
  }
  cudaCheck(cudaGetLastError(), "P2 SOR");
  communicate(x, Lf, kAllGroups);
}

void Storage::p2Sor(int opId, int x, int b, double omega, int L, unsigned mask, bool backwards) {
  P2Operator& o = p2op(opId);
  argCheck(L >= o.minL && L <= o.maxL, "level outside the P2 operator's level range");
  argCheck(x != b, "P2 SOR: x and b must differ");
  Function& fx = fn(x);
  argCheck(fx.prec == fn(b).prec, "P2 SOR: precision mismatch");
  if (fx.prec == 8)
    p2SorT<double>(o, opId, x, b, L, mask, omega, backwards);
  else
    p2SorT<float>(o, opId, x, b, L, mask, (float)omega, backwards);
}

// Fine node Q of a macro-cell at Q / 4 level-L units: class r = (Q_x & 3) | (Q_y & 3) << 2 |
// (Q_z & 3) << 4. For every micro-cell (type t, anchor (Q >> 2) - delta) containing the point,
// its barycentric coordinates in quarters (exact: the micro-cells are unimodular) give the coarse
// P2 basis values lambda (2 lambda - 1) at the vertices and 4 lambda_i lambda_j at the edges.
static void buildP2Transfer(P2Transfer& tr, cudaStream_t stream) {
  std::vector<unsigned char> nc(64, 0), cand(64 * dev::kP2TrCand, 0);
  std::vector<double> w(64 * dev::kP2TrCand * 10, 0.0);
  for (int r = 0; r < 64; ++r) {
    const int f4[3] = {r & 3, (r >> 2) & 3, (r >> 4) & 3};
    for (int d = 0; d < 8; ++d)
      for (int t = 0; t < 6; ++t) {
        const int* v0 = kMicroCellTable[t][0];
        int B[3][3];  // columns v_m - v0
        for (int m = 1; m < 4; ++m)
          for (int k = 0; k < 3; ++k) B[k][m - 1] = kMicroCellTable[t][m][k] - v0[k];
        const int det = B[0][0] * (B[1][1] * B[2][2] - B[1][2] * B[2][1]) - B[0][1] * (B[1][0] * B[2][2] - B[1][2] * B[2][0]) +
                        B[0][2] * (B[1][0] * B[2][1] - B[1][1] * B[2][0]);
        const int inv[3][3] = {{(B[1][1] * B[2][2] - B[1][2] * B[2][1]) * det, (B[0][2] * B[2][1] - B[0][1] * B[2][2]) * det,
                                (B[0][1] * B[1][2] - B[0][2] * B[1][1]) * det},
                               {(B[1][2] * B[2][0] - B[1][0] * B[2][2]) * det, (B[0][0] * B[2][2] - B[0][2] * B[2][0]) * det,
                                (B[0][2] * B[1][0] - B[0][0] * B[1][2]) * det},
                               {(B[1][0] * B[2][1] - B[1][1] * B[2][0]) * det, (B[0][1] * B[2][0] - B[0][0] * B[2][1]) * det,
                                (B[0][0] * B[1][1] - B[0][1] * B[1][0]) * det}};  // det = +-1, so inv = adj * det
        int q[3];
        for (int k = 0; k < 3; ++k) q[k] = f4[k] + 4 * ((d >> k) & 1) - 4 * v0[k];  // 4 (point - v0)
        int l4[4];
        l4[1] = inv[0][0] * q[0] + inv[0][1] * q[1] + inv[0][2] * q[2];
        l4[2] = inv[1][0] * q[0] + inv[1][1] * q[1] + inv[1][2] * q[2];
        l4[3] = inv[2][0] * q[0] + inv[2][1] * q[1] + inv[2][2] * q[2];
        l4[0] = 4 - l4[1] - l4[2] - l4[3];
        if (l4[0] < 0 || l4[1] < 0 || l4[2] < 0 || l4[3] < 0) continue;
        argCheck(det == 1 || det == -1, "micro-cell is not unimodular");
        if (nc[r] >= dev::kP2TrCand) continue;
        const int k = nc[r]++;
        cand[r * dev::kP2TrCand + k] = (unsigned char)((d << 3) | t);
        double* wr = &w[(size_t)(r * dev::kP2TrCand + k) * 10];
        for (int m = 0; m < 4; ++m) {
          const double l = l4[m] / 4.0;
          wr[m] = l * (2.0 * l - 1.0);
        }
        for (int e = 0; e < 6; ++e) wr[4 + e] = 4.0 * (l4[kP2Edge[e][0]] / 4.0) * (l4[kP2Edge[e][1]] / 4.0);
      }
  }
  std::vector<float> wfl(w.begin(), w.end());
  tr.hNCand = nc;
  tr.hCand = cand;
  tr.hW = w;
  tr.nCand.alloc(nc.size());
  tr.cand.alloc(cand.size());
  tr.wd.alloc(w.size() * sizeof(double));
  tr.wf.alloc(wfl.size() * sizeof(float));
  cudaCheck(cudaMemcpyAsync(tr.nCand.p, nc.data(), nc.size(), cudaMemcpyHostToDevice, stream), "p2 transfer");
  cudaCheck(cudaMemcpyAsync(tr.cand.p, cand.data(), cand.size(), cudaMemcpyHostToDevice, stream), "p2 transfer");
  cudaCheck(cudaMemcpyAsync(tr.wd.p, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice, stream), "p2 transfer");
  cudaCheck(cudaMemcpyAsync(tr.wf.p, wfl.data(), wfl.size() * sizeof(float), cudaMemcpyHostToDevice, stream), "p2 transfer");
  cudaCheck(cudaStreamSynchronize(stream), "p2 transfer");
  tr.built = true;
}

// The restriction's gather lists for fine lattice level Lff: every fine node Q of the closed
// reference cell contributes to the coarse nodes its prolongation reads (the same candidate
// micro-cell as p2PickCandidate picks, nonzero basis values only; even nodes are injected), and
// each coarse node lists its contributions in the order of Q (z, y, x), then of the basis node.
const P2Gather& Storage::p2Gather(int Lff) {
  P2Gather& g = p2gather[Lff];
  if (g.built) return g;
  if (!p2tr.built) buildP2Transfer(p2tr, stream);
  const dev::P2Tables& tb = p2TablesOnce();
  const int Mf = disc.level(Lff).N, Mc = Mf / 2, N = Mc / 2, wf = Mf + 1, wc = Mc + 1;
  auto tet = [](int64_t w) { return w * (w + 1) * (w + 2) / 6; };
  auto row = [](int64_t W, int64_t y) { return y * (W + 1) - y * (y + 1) / 2; };
  auto cidx = [&](int x, int y, int z) { return int(tet(wc) - tet(wc - z) + row(wc - z, y) + x); };
  auto fidx = [&](int x, int y, int z) { return int(tet(wf) - tet(wf - z) + row(wf - z, y) + x); };
  const int nC = (int)tet(wc);
  std::vector<std::vector<std::pair<int, double>>> lists((size_t)nC);
  for (int Z = 0; Z <= Mf; ++Z)
    for (int Y = 0; Y <= Mf - Z; ++Y)
      for (int X = 0; X <= Mf - Z - Y; ++X) {
        const int q = fidx(X, Y, Z);
        if (((X | Y | Z) & 1) == 0) {
          lists[(size_t)cidx(X >> 1, Y >> 1, Z >> 1)].push_back({q, 1.0});
          continue;
        }
        const int r = (X & 3) | ((Y & 3) << 2) | ((Z & 3) << 4);
        for (int k = 0; k < p2tr.hNCand[r]; ++k) {  // the first candidate inside the cell
          const int c = p2tr.hCand[(size_t)r * dev::kP2TrCand + k], t = c & 7, d = c >> 3;
          const int ax = (X >> 2) - (d & 1), ay = (Y >> 2) - ((d >> 1) & 1), az = (Z >> 2) - ((d >> 2) & 1);
          if (!(ax >= 0 && ay >= 0 && az >= 0 && ax + ay + az < N - tb.widthRed[t])) continue;
          const double* w = &p2tr.hW[(size_t)(r * dev::kP2TrCand + k) * 10];
          for (int m = 0; m < 10; ++m)
            if (w[m] != 0.0)
              lists[(size_t)cidx(2 * ax + tb.off[t][m][0], 2 * ay + tb.off[t][m][1], 2 * az + tb.off[t][m][2])]
                  .push_back({q, w[m]});
          break;
        }
      }
  std::vector<int> ptr((size_t)nC + 1, 0), idx;
  std::vector<double> wd;
  for (int c = 0; c < nC; ++c) {
    for (const auto& e : lists[(size_t)c]) {
      idx.push_back(e.first);
      wd.push_back(e.second);
    }
    ptr[(size_t)c + 1] = (int)idx.size();
  }
  std::vector<float> wfl(wd.begin(), wd.end());
  g.nCoarse = nC;
  g.ptr.alloc(ptr.size() * sizeof(int));
  cudaCheck(cudaMemcpyAsync(g.ptr.p, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice, stream), "p2 gather");
  g.idx.alloc(idx.size() * sizeof(int));
  g.wd.alloc(wd.size() * sizeof(double));
  g.wf.alloc(wfl.size() * sizeof(float));
  cudaCheck(cudaMemcpyAsync(g.idx.p, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice, stream), "p2 gather");
  cudaCheck(cudaMemcpyAsync(g.wd.p, wd.data(), wd.size() * sizeof(double), cudaMemcpyHostToDevice, stream), "p2 gather");
  cudaCheck(cudaMemcpyAsync(g.wf.p, wfl.data(), wfl.size() * sizeof(float), cudaMemcpyHostToDevice, stream), "p2 gather");
  cudaCheck(cudaStreamSynchronize(stream), "p2 gather");
  g.built = true;
  return g;
}

int Storage::p2Scratch(int Lf, int prec) {
  const auto key = p2ScratchKey(Lf, prec);
  if (!p2scratch.count(key)) p2scratch[key] = createFunction(Lf, Lf, prec);
  return p2scratch[key];
}

void Storage::p2Prolongate(int id, int Lc, unsigned mask, bool add) {
  Function& f = fn(id);
  const int Lcf = Lc + 1, Lff = Lc + 2;  // lattice levels
  argCheck(Lcf >= f.minL && Lff <= f.maxL, "P2 prolongation: levels outside the function's range");
  if (!p2tr.built) buildP2Transfer(p2tr, stream);
  const LevelData& lc = levels[Lcf];
  const LevelData& lf = levels[Lff];
  P2Additive& ad = p2Additive(Lff);
  communicate(id, Lcf, 1 << G_CELL);
  const int out = add ? p2Scratch(Lff, f.prec) : id;
  const dev::P2TransferDev tr{(const unsigned char*)p2tr.nCand.p, (const unsigned char*)p2tr.cand.p};
  const int nb = lf.lv.nCells * (lf.lv.N + 1), na = (ad.n + dev::kBlock - 1) / dev::kBlock;
  if (f.prec == 8) {
    dev::p2ProlongKernel<double><<<nb, dev::kBlock, 0, stream>>>(lc.lv, lf.lv, p2TablesOnce(), tr, (const double*)p2tr.wd.p,
                                                               (const double*)data(id, Lcf), (double*)data(out, Lff));
    if (ad.n)
      dev::p2PickKernel<double><<<na, dev::kBlock, 0, stream>>>((const int64_t*)ad.owner.p, (const int*)ad.ptr.p,
                                                              (const int64_t*)ad.copies.p, (const unsigned char*)ad.type.p,
                                                              ad.n, (double*)data(out, Lff), add ? HG_ALL : mask);
  } else {
    dev::p2ProlongKernel<float><<<nb, dev::kBlock, 0, stream>>>(lc.lv, lf.lv, p2TablesOnce(), tr, (const float*)p2tr.wf.p,
                                                              (const float*)data(id, Lcf), (float*)data(out, Lff));
    if (ad.n)
      dev::p2PickKernel<float><<<na, dev::kBlock, 0, stream>>>((const int64_t*)ad.owner.p, (const int*)ad.ptr.p,
                                                             (const int64_t*)ad.copies.p, (const unsigned char*)ad.type.p,
                                                             ad.n, (float*)data(out, Lff), add ? HG_ALL : mask);
  }
  launches += ad.n ? 2 : 1;
  cudaCheck(cudaGetLastError(), "P2 prolongation");
  if (add) {
    const double one = 1.0;
    lincomb(id, Lff, mask, 1, &one, &out, true, 0.0);
  }
  communicate(id, Lff, kAllGroups);
}

void Storage::p2Restrict(int id, int Lf, unsigned mask) {
  Function& f = fn(id);
  const int Lff = Lf + 1, Lcf = Lf;  // lattice levels: fine P2 level Lf, coarse Lf - 1
  argCheck(Lf >= 1 && Lcf >= f.minL && Lff <= f.maxL, "P2 restriction: levels outside the function's range");
  if (!p2tr.built) buildP2Transfer(p2tr, stream);
  const LevelData& lc = levels[Lcf];
  const LevelData& lf = levels[Lff];
  P2Additive& adf = p2Additive(Lff);
  P2Additive& adc = p2Additive(Lcf);
  const P2Gather& gt = p2Gather(Lff);
  communicate(id, Lff, 1 << G_CELL);
  cudaCheck(cudaMemsetAsync(data(id, Lcf), 0, (size_t)lc.lay->total * f.prec, stream), "P2 restriction");
  const int bpc = (gt.nCoarse + dev::kBlock - 1) / dev::kBlock;
  const int nb = lf.lv.nCells * bpc, na = (adc.n + dev::kBlock - 1) / dev::kBlock;
  if (f.prec == 8) {
    dev::p2RestrictGatherKernel<double><<<nb, dev::kBlock, 0, stream>>>(
        lc.lv, lf.lv, (const int*)gt.ptr.p, (const int*)gt.idx.p, (const double*)gt.wd.p, gt.nCoarse, bpc,
        (const double*)data(id, Lff),
        (const unsigned char*)adf.mult.p, (double*)data(id, Lcf));
    if (adc.n)
      dev::p2AddKernel<double, dev::MODE_REPLACE><<<na, dev::kBlock, 0, stream>>>(
          (const int64_t*)adc.owner.p, (const int*)adc.ptr.p, (const int64_t*)adc.copies.p,
          (const unsigned char*)adc.type.p, adc.n, (double*)data(id, Lcf), nullptr, mask, nullptr, -1);
  } else {
    dev::p2RestrictGatherKernel<float><<<nb, dev::kBlock, 0, stream>>>(
        lc.lv, lf.lv, (const int*)gt.ptr.p, (const int*)gt.idx.p, (const float*)gt.wf.p, gt.nCoarse, bpc,
        (const float*)data(id, Lff),
        (const unsigned char*)adf.mult.p, (float*)data(id, Lcf));
    if (adc.n)
      dev::p2AddKernel<float, dev::MODE_REPLACE><<<na, dev::kBlock, 0, stream>>>(
          (const int64_t*)adc.owner.p, (const int*)adc.ptr.p, (const int64_t*)adc.copies.p,
          (const unsigned char*)adc.type.p, adc.n, (float*)data(id, Lcf), nullptr, mask, nullptr, -1);
  }
  launches += adc.n ? 2 : 1;
  cudaCheck(cudaGetLastError(), "P2 restriction");
  communicate(id, Lcf, kAllGroups);
}

// Interior coupling stencils of every cell from the divergence elements D[cell][t][k][i][j]:
// div weights on p2s::kOff[0] (a pressure vertex i of micro-cell t sees node j at off_j - off_i),
// divT weights on p2s::kDivTOff (velocity node j of class pc sees vertex i at (off_i - off_j + pc)/2).
static void p2DivStencils(const std::vector<double>& D, int nCells, std::vector<double>& WD, std::vector<double>& WT) {
  const dev::P2Tables& tb = p2TablesOnce();
  WD.assign((size_t)nCells * 195, 0.0);
  WT.assign((size_t)nCells * 195, 0.0);
  auto find = [](const signed char (*tab)[3], int len, int dx, int dy, int dz) {
    for (int e = 0; e < len; ++e)
      if (tab[e][0] == dx && tab[e][1] == dy && tab[e][2] == dz) return e;
    throw Error(HG_ERR_INTERNAL, "Taylor-Hood stencil table does not match the micro-cells");
  };
  for (int c = 0; c < nCells; ++c) {
    const double* Dc = D.data() + (size_t)c * 720;
    for (int t = 0; t < 6; ++t)
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 10; ++j) {
          const int e = find(p2s::kOff[0], p2s::kLen[0], tb.off[t][j][0] - tb.off[t][i][0],
                             tb.off[t][j][1] - tb.off[t][i][1], tb.off[t][j][2] - tb.off[t][i][2]);
          for (int k = 0; k < 3; ++k) WD[(size_t)c * 195 + k * 65 + e] += Dc[t * 120 + k * 40 + i * 10 + j];
        }
    for (int pc = 0; pc < 8; ++pc) {
      const int par[3] = {pc & 1, (pc >> 1) & 1, (pc >> 2) & 1};
      for (int q = 0; q < tb.nCand[pc]; ++q) {
        const int t = tb.cand[pc][q][0], j = tb.cand[pc][q][1];
        for (int i = 0; i < 4; ++i) {
          const int e = find(p2s::kDivTOff[pc], p2s::kDivTLen[pc], (tb.off[t][i][0] - tb.off[t][j][0] + par[0]) / 2,
                             (tb.off[t][i][1] - tb.off[t][j][1] + par[1]) / 2,
                             (tb.off[t][i][2] - tb.off[t][j][2] + par[2]) / 2);
          for (int k = 0; k < 3; ++k)
            WT[(size_t)c * 195 + k * 65 + p2s::kDivTFirst[pc] + e] += Dc[t * 120 + k * 40 + i * 10 + j];
        }
      }
    }
  }
}

int Storage::createStokesOperator(int minL, int maxL) {
  const int id = createP2Operator(FORM_LAPLACE, minL, maxL);
  P2Operator& o = p2op(id);
  for (int L = minL; L <= maxL; ++L) {
    const std::vector<double> D = p2p1CellDiv(disc.topo(), L);
    {
      std::vector<double> WD, WT;
      p2DivStencils(D, (int)disc.topo().cells.size(), WD, WT);
      auto up = [&](std::vector<std::unique_ptr<DevBuf>>& dst, const std::vector<double>& v, bool fp32) {
        dst.emplace_back(new DevBuf());
        if (fp32) {
          std::vector<float> f(v.begin(), v.end());
          dst.back()->alloc(f.size() * sizeof(float));
          cudaCheck(cudaMemcpyAsync(dst.back()->p, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice, stream),
                    "div stencils");
          cudaCheck(cudaStreamSynchronize(stream), "div stencils");
        } else {
          dst.back()->alloc(v.size() * sizeof(double));
          cudaCheck(cudaMemcpyAsync(dst.back()->p, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, stream),
                    "div stencils");
          cudaCheck(cudaStreamSynchronize(stream), "div stencils");
        }
      };
      up(o.wdivd, WD, false);
      up(o.wdivf, WD, true);
      up(o.wdivtd, WT, false);
      up(o.wdivtf, WT, true);
    }
    std::vector<float> Df(D.begin(), D.end());
    o.dd.emplace_back(new DevBuf());
    o.dd.back()->alloc(D.size() * sizeof(double));
    cudaCheck(cudaMemcpyAsync(o.dd.back()->p, D.data(), D.size() * sizeof(double), cudaMemcpyHostToDevice, stream),
              "div upload");
    o.df.emplace_back(new DevBuf());
    o.df.back()->alloc(Df.size() * sizeof(float));
    cudaCheck(cudaMemcpyAsync(o.df.back()->p, Df.data(), Df.size() * sizeof(float), cudaMemcpyHostToDevice, stream),
              "div upload");
    cudaCheck(cudaStreamSynchronize(stream), "div upload");
  }
  return id;
}

// v_k = D_k^T p (or += with add) at the velocity DoFs flagged by maskV: shares into three scratch
// functions, owner sums, then written where flagged.
template <class T>
static void stokesDivTImpl(Storage& st, P2Operator& o, int p, const int v[3], int L, unsigned maskV, bool add) {
  const int Lv = L + 1, Lp = L;
  const LevelData& lvv = st.levels[Lv];
  const LevelData& lvp = st.levels[Lp];
  const T* D = (const T*)(sizeof(T) == 8 ? o.dd[L - o.minL]->p : o.df[L - o.minL]->p);
  const int prec = (int)sizeof(T);
  int sc[3];
  for (int k = 0; k < 3; ++k) {
    auto key = std::make_pair(Lv, 16 + 8 * k + prec);  // three distinct scratch buffers per level
    if (!st.p2scratch.count(key)) st.p2scratch[key] = st.createFunction(Lv, Lv, prec);
    sc[k] = st.p2scratch[key];
  }
  st.communicate(p, Lp, 1 << G_CELL);
  P2Additive& adv = st.p2Additive(Lv);
  const bool interior = lvv.lv.N >= 4;
  if (interior) {
    const T* WT = (const T*)(sizeof(T) == 8 ? o.wdivtd[L - o.minL]->p : o.wdivtf[L - o.minL]->p);
    dev::p2DivTStencilKernel<T><<<lvv.lv.nCells * (lvv.lv.N - 3), dev::kBlock, 0, st.stream>>>(
        lvv.lv, lvp.lv, WT, (T*)st.data(sc[0], Lv), (T*)st.data(sc[1], Lv), (T*)st.data(sc[2], Lv),
        (const T*)st.data(p, Lp), maskV);
    ++st.launches;
  }
  const int nClosure = adv.closureBegin[11];
  if (interior && nClosure > 0) {  // the closure nodes from the list, one thread each
    dev::p2DivTClosureListKernel<T><<<(nClosure + dev::kBlock - 1) / dev::kBlock, dev::kBlock, 0, st.stream>>>(
        lvv.lv, lvp.lv, p2TablesOnce(), D, (T*)st.data(sc[0], Lv), (T*)st.data(sc[1], Lv), (T*)st.data(sc[2], Lv),
        (const T*)st.data(p, Lp), (const dev::P2ClosureNode*)adv.closureList.p, nClosure);
  } else {
    dev::p2DivTKernel<T><<<lvv.lv.nCells * (lvv.lv.N + 1), dev::kBlock, 0, st.stream>>>(
        lvv.lv, lvp.lv, p2TablesOnce(), D, (T*)st.data(sc[0], Lv), (T*)st.data(sc[1], Lv), (T*)st.data(sc[2], Lv),
        (const T*)st.data(p, Lp), maskV, interior);
  }
  ++st.launches;
  for (int k = 0; k < 3; ++k) {
    if (adv.n)
      dev::p2AddKernel<T, dev::MODE_REPLACE><<<(adv.n + dev::kBlock - 1) / dev::kBlock, dev::kBlock, 0, st.stream>>>(
          (const int64_t*)adv.owner.p, (const int*)adv.ptr.p, (const int64_t*)adv.copies.p,
          (const unsigned char*)adv.type.p, adv.n, (T*)st.data(sc[k], Lv), nullptr, maskV, nullptr, -1);
    const double one = 1.0;
    st.lincomb(v[k], Lv, maskV, 1, &one, &sc[k], add, 0.0);
    st.communicate(v[k], Lv, (1 << G_COUNT) - 1);
    st.launches += adv.n ? 1 : 0;
  }
  cudaCheck(cudaGetLastError(), "Stokes divT");
}

// q = sum_k D_k u_k at the pressure DoFs flagged by maskP.
template <class T>
static void stokesDivImpl(Storage& st, P2Operator& o, const int u[3], int q, int L, unsigned maskP) {
  const int Lv = L + 1, Lp = L;
  const LevelData& lvv = st.levels[Lv];
  const LevelData& lvp = st.levels[Lp];
  const T* D = (const T*)(sizeof(T) == 8 ? o.dd[L - o.minL]->p : o.df[L - o.minL]->p);
  for (int k = 0; k < 3; ++k) st.communicate(u[k], Lv, 1 << G_CELL);
  P2Additive& adp = st.p2Additive(Lp);
  const bool interior = lvp.lv.N >= 4;
  if (interior) {
    const T* WD = (const T*)(sizeof(T) == 8 ? o.wdivd[L - o.minL]->p : o.wdivf[L - o.minL]->p);
    dev::p2DivStencilKernel<T><<<lvp.lv.nCells * (lvp.lv.N - 3), dev::kBlock, 0, st.stream>>>(
        lvp.lv, lvv.lv, WD, (T*)st.data(q, Lp), (const T*)st.data(u[0], Lv), (const T*)st.data(u[1], Lv),
        (const T*)st.data(u[2], Lv), maskP);
    ++st.launches;
  }
  const int nClosure = adp.closureBegin[11];
  if (interior && nClosure > 0) {
    dev::p2DivClosureListKernel<T><<<(nClosure + dev::kBlock - 1) / dev::kBlock, dev::kBlock, 0, st.stream>>>(
        lvp.lv, lvv.lv, p2TablesOnce(), D, (T*)st.data(q, Lp), (const T*)st.data(u[0], Lv), (const T*)st.data(u[1], Lv),
        (const T*)st.data(u[2], Lv), (const dev::P2ClosureNode*)adp.closureList.p, nClosure);
  } else {
    dev::p2DivKernel<T><<<lvp.lv.nCells * (lvp.lv.N + 1), dev::kBlock, 0, st.stream>>>(
        lvp.lv, lvv.lv, p2TablesOnce(), D, (T*)st.data(q, Lp), (const T*)st.data(u[0], Lv), (const T*)st.data(u[1], Lv),
        (const T*)st.data(u[2], Lv), maskP, interior);
  }
  ++st.launches;
  if (adp.n) {
    dev::p2AddKernel<T, dev::MODE_REPLACE><<<(adp.n + dev::kBlock - 1) / dev::kBlock, dev::kBlock, 0, st.stream>>>(
        (const int64_t*)adp.owner.p, (const int*)adp.ptr.p, (const int64_t*)adp.copies.p,
        (const unsigned char*)adp.type.p, adp.n, (T*)st.data(q, Lp), nullptr, maskP, nullptr, -1);
    ++st.launches;
  }
  cudaCheck(cudaGetLastError(), "Stokes div");
  st.communicate(q, Lp, (1 << G_COUNT) - 1);
}

int Storage::p1Diagonal(int opId, int L) {
  Operator& o = op(opId);
  argCheck(L >= o.minL && L <= o.maxL, "level outside the operator's level range");
  if (o.hostStale) {  // re-assembled on the device since: bring the host copy up to date
    for (int l = o.minL; l <= o.maxL; ++l) o.host[l - o.minL] = assembleStencils(disc, l, (FormKind)o.form);
    o.hostStale = false;
  }
  const LevelStencils& h = o.host[L - o.minL];
  const LevelData& ld = levels[L];
  const LevelLayout& lay = *ld.lay;
  std::vector<double> vals;  // one value per chunk, in the chunk order of the level
  auto add = [&](int64_t size, double v) {
    for (int64_t s = 0; s < size; s += 8192) vals.push_back(v);
  };
  for (size_t c = 0; c < lay.size[KC].size(); ++c) add(lay.size[KC][c], h.cell[c][0]);
  for (size_t f = 0; f < lay.size[KF].size(); ++f) add(lay.size[KF][f], h.face[f].empty() ? 0.0 : h.face[f][0].w);
  for (size_t e = 0; e < lay.size[KE].size(); ++e) add(lay.size[KE][e], h.edge[e].empty() ? 0.0 : h.edge[e][0].w);
  for (size_t v = 0; v < lay.size[KV].size(); ++v) add(lay.size[KV][v], h.vert[v].empty() ? 0.0 : h.vert[v][0].w);
  argCheck((int)vals.size() == ld.nChunks, "diagonal: chunk table mismatch");
  const int d = createFunction(L, L, 8);
  if (ld.nChunks) {
    DevBuf dv;
    dv.alloc(vals.size() * sizeof(double));
    cudaCheck(cudaMemcpyAsync(dv.p, vals.data(), vals.size() * sizeof(double), cudaMemcpyHostToDevice, stream), "diag");
    dev::fillChunksKernel<<<ld.nChunks, dev::kBlock, 0, stream>>>(ld.chunks, (const double*)dv.p, (double*)data(d, L));
    ++launches;
    cudaCheck(cudaStreamSynchronize(stream), "diag");
  }
  communicate(d, L, kAllGroups);
  return d;
}

void Storage::stokesDivT(int opId, int p, const int v[3], int L, unsigned maskV, bool add) {
  P2Operator& o = p2op(opId);
  argCheck(!o.dd.empty(), "not a Stokes operator");
  argCheck(L >= o.minL && L <= o.maxL, "level outside the Stokes operator's level range");
  if (fn(p).prec == 8)
    stokesDivTImpl<double>(*this, o, p, v, L, maskV, add);
  else
    stokesDivTImpl<float>(*this, o, p, v, L, maskV, add);
}

void Storage::stokesDiv(int opId, const int u[3], int q, int L, unsigned maskP) {
  P2Operator& o = p2op(opId);
  argCheck(!o.dd.empty(), "not a Stokes operator");
  argCheck(L >= o.minL && L <= o.maxL, "level outside the Stokes operator's level range");
  if (fn(q).prec == 8)
    stokesDivImpl<double>(*this, o, u, q, L, maskP);
  else
    stokesDivImpl<float>(*this, o, u, q, L, maskP);
}

void Storage::stokesApply(int opId, const int u[3], int p, const int v[3], int q, int L, unsigned maskV,
                          unsigned maskP) {
  P2Operator& o = p2op(opId);
  argCheck(!o.dd.empty(), "not a Stokes operator");
  argCheck(L >= o.minL && L <= o.maxL, "level outside the Stokes operator's level range");
  const int prec = fn(p).prec;
  for (int k = 0; k < 3; ++k) argCheck(fn(u[k]).prec == prec && fn(v[k]).prec == prec, "Stokes: precision mismatch");
  argCheck(fn(q).prec == prec, "Stokes: precision mismatch");
  for (int k = 0; k < 3; ++k) p2Apply(opId, u[k], v[k], -1, L, maskV, 0);
  stokesDivT(opId, p, v, L, maskV, true);
  stokesDiv(opId, u, q, L, maskP);
}

void Storage::autotuneSor(int minL, int maxL, int prec, int reps, double* ms) {
  argCheck(minL >= 0 && maxL <= maxLevel() && minL <= maxL, "autotune: invalid level range");
  argCheck(prec == 8 || prec == 4, "autotune: precision must be 8 or 4");
  argCheck(reps >= 1 && reps <= 100, "autotune: repetitions in [1, 100]");
  if ((int)sorScheduleLevel.size() < 2 * (maxLevel() + 1)) sorScheduleLevel.assign(2 * (maxLevel() + 1), -1);
  const int pi = prec == 4 ? 1 : 0;
  const int op = createOperator(FORM_LAPLACE, minL, maxL);
  cudaEvent_t e0, e1;
  cudaCheck(cudaEventCreate(&e0), "event");
  cudaCheck(cudaEventCreate(&e1), "event");
  for (int L = minL; L <= maxL; ++L) {
    const int x = createFunction(L, L, prec), b = createFunction(L, L, prec);
    fillRandom(x, L, HG_ALL, 1, -1.0, 1.0);
    fillRandom(b, L, HG_ALL, 2, -1.0, 1.0);
    double best = 0;
    int pick = 0;
    for (int sch = 0; sch < 4; ++sch) {
      sorScheduleLevel[2 * L + pi] = sch;
      // warm-up (allocates the spare buffers and tables), then groups of three sweeps
      smoothSorSweeps(op, x, b, 1.0, L, HG_INNER | HG_NEUMANN, 3, false, false);
      cudaCheck(cudaEventRecord(e0, stream), "event");
      for (int r = 0; r < reps; ++r) smoothSorSweeps(op, x, b, 1.0, L, HG_INNER | HG_NEUMANN, 3, false, false);
      cudaCheck(cudaEventRecord(e1, stream), "event");
      cudaCheck(cudaEventSynchronize(e1), "event");
      float t = 0;
      cudaCheck(cudaEventElapsedTime(&t, e0, e1), "event");
      const double per = t / (3.0 * reps);
      if (ms) ms[4 * (L - minL) + sch] = per;
      if (sch == 0 || per < best) {
        best = per;
        pick = sch;
      }
    }
    sorScheduleLevel[2 * L + pi] = pick;
    fns.erase(x);
    fns.erase(b);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ops.erase(op);
  ++generation;
}

void Storage::reassembleOperator(int id, bool onDevice) {
  Operator& o = op(id);
  if (!onDevice) {
    for (int L = o.minL; L <= o.maxL; ++L) {
      LevelStencils h = assembleStencils(disc, L, (FormKind)o.form);
      refillStencil<double>(o.d[L - o.minL], h, stream);
      refillStencil<float>(o.f[L - o.minL], h, stream);
      o.host[L - o.minL] = std::move(h);
    }
    o.hostStale = false;
    return;
  }
  if (o.form != FORM_LAPLACE) return;  // the mass and PSPG forms do not depend on the coefficients
  static_assert(sizeof(dev::PlanTermDev) == sizeof(PlanTerm), "plan term layout");
  const Topology& topo = disc.topo();
  if (o.plans.empty()) {
    for (int L = o.minL; L <= o.maxL; ++L) {
      const AssemblyPlan p = buildAssemblyPlan(disc, L, (FormKind)o.form);
      argCheck(p.nCell == (int64_t)topo.cells.size() * 16 && p.nFace == (int64_t)topo.faces.size() * 16,
               "re-assembly: target layout");
      Operator::DevPlan dp;
      dp.first = (const int64_t*)upload(o.keep, p.first, stream);
      dp.terms = (const dev::PlanTermDev*)upload(o.keep, p.terms, stream);
      dp.nCell = p.nCell;
      dp.nFace = p.nFace;
      dp.nLow = p.nLow;
      cudaCheck(cudaStreamSynchronize(stream), "plan upload");  // the host vectors go out of scope
      o.plans.push_back(dp);
    }
    o.coef.alloc(std::max<size_t>(topo.cells.size(), 1) * sizeof(double));
  }
  std::vector<double> k(topo.cells.size());
  for (size_t c = 0; c < k.size(); ++c) k[c] = topo.cells[c].k;
  // from pageable memory: returns once the values are staged, so k may go out of scope
  cudaCheck(cudaMemcpyAsync(o.coef.p, k.data(), k.size() * sizeof(double), cudaMemcpyHostToDevice, stream),
            "coefficient upload");
  for (int L = o.minL; L <= o.maxL; ++L) {
    const Operator::DevPlan& dp = o.plans[L - o.minL];
    const dev::StencilDev<double>& sd = o.d[L - o.minL];
    const dev::StencilDev<float>& sf = o.f[L - o.minL];
    const int64_t n = dp.nCell + dp.nFace + dp.nLow;
    if (n == 0) continue;
    dev::planAssembleKernel<<<(unsigned)((n + dev::kBlock - 1) / dev::kBlock), dev::kBlock, 0, stream>>>(
        dp.first, dp.terms, (const double*)o.coef.p, dp.nCell, dp.nFace, dp.nLow, const_cast<double*>(sd.cellW),
        const_cast<float*>(sf.cellW), const_cast<dev::FaceEnt<double>*>(sd.faceEnt),
        const_cast<dev::FaceEnt<float>*>(sf.faceEnt), const_cast<double*>(sd.lowEntW), const_cast<float*>(sf.lowEntW));
    ++launches;
  }
  cudaCheck(cudaGetLastError(), "re-assembly");
  o.hostStale = true;
}

int Storage::createOperator(int form, int minL, int maxL) {
  argCheck(form == FORM_LAPLACE || form == FORM_MASS || form == FORM_PSPG, "unknown form");
  argCheck(minL >= 0 && maxL <= maxLevel() && minL <= maxL, "invalid level range");
  std::unique_ptr<Operator> op(new Operator());
  op->form = form;
  op->minL = minL;
  op->maxL = maxL;
  for (int L = minL; L <= maxL; ++L) {
    op->host.push_back(assembleStencils(disc, L, (FormKind)form));
    op->d.push_back(packStencil<double>(op->keep, op->host.back(), stream));
    op->f.push_back(packStencil<float>(op->keep, op->host.back(), stream));
  }
  cudaCheck(cudaStreamSynchronize(stream), "operator upload");
  const int id = nextId++;
  ops[id] = std::move(op);
  return id;
}

Operator& Storage::op(int id) {
  auto it = ops.find(id);
  argCheck(it != ops.end(), "unknown operator handle");
  return *it->second;
}

template <class T>
const dev::StencilDev<T>& stencilOf(Operator& o, int L);
template <>
const dev::StencilDev<double>& stencilOf<double>(Operator& o, int L) {
  return o.d[L - o.minL];
}
template <>
const dev::StencilDev<float>& stencilOf<float>(Operator& o, int L) {
  return o.f[L - o.minL];
}

template <class T, int MODE>
void Storage::stencilOp(Operator& o, int L, T* dst, const T* src, const T* rhs, unsigned mask, int kinds) {
  const LevelData& ld = levels[L];
  const dev::StencilDev<T>& st = stencilOf<T>(o, L);
  if (ld.nTiles && (kinds & (1 << KC))) {
    constexpr int op =
        MODE == dev::MODE_REPLACE ? dev::STRIP_REPLACE : MODE == dev::MODE_ADD ? dev::STRIP_ADD : dev::STRIP_RESIDUAL;
    dev::cellStripKernel<T, op><<<ld.nTiles, dev::stripThreads<T>(), 0, stream>>>(ld.lv, ld.tiles, st.cellW, dst, src,
                                                                                  rhs, mask);
    ++launches;
  }
  if (ld.lv.nFaceBlocks && (kinds & (1 << KF))) {
    dev::faceStencilKernel<T, MODE><<<ld.lv.nFaceBlocks, dev::kBlock, 0, stream>>>(ld.lv, st, dst, src, rhs, mask);
    ++launches;
  }
  const int nVertBlocks = ld.lv.nLowBlocks - ld.lv.nLowEdgeBlocks;
  if ((kinds & (1 << KE)) && (kinds & (1 << KV)) && ld.lv.nLowBlocks) {
    dev::lowStencilKernel<T, MODE><<<ld.lv.nLowBlocks, dev::kBlock, 0, stream>>>(ld.lv, st, dst, src, rhs, mask, 0);
    ++launches;
  } else if ((kinds & (1 << KE)) && ld.lv.nLowEdgeBlocks) {
    dev::lowStencilKernel<T, MODE><<<ld.lv.nLowEdgeBlocks, dev::kBlock, 0, stream>>>(ld.lv, st, dst, src, rhs, mask, 0);
    ++launches;
  } else if ((kinds & (1 << KV)) && nVertBlocks) {
    dev::lowStencilKernel<T, MODE><<<nVertBlocks, dev::kBlock, 0, stream>>>(ld.lv, st, dst, src, rhs, mask,
                                                                              ld.lv.nLowEdgeBlocks);
    ++launches;
  }
  cudaCheck(cudaGetLastError(), "stencil kernel");
}

void Storage::apply(int opId, int src, int dst, int L, unsigned mask, int update, int kinds, bool refresh) {
  Operator& o = op(opId);
  argCheck(L >= o.minL && L <= o.maxL, "level outside the operator's level range");
  argCheck(src != dst, "apply: src and dst must differ");
  Function& fs = fn(src);
  argCheck(fs.prec == fn(dst).prec, "apply: precision mismatch");
  if (refresh) communicate(src, L, kAllGroups);
  if (fs.prec == 8) {
    if (update == 0)
      stencilOp<double, dev::MODE_REPLACE>(o, L, (double*)data(dst, L), (const double*)data(src, L), nullptr, mask, kinds);
    else
      stencilOp<double, dev::MODE_ADD>(o, L, (double*)data(dst, L), (const double*)data(src, L), nullptr, mask, kinds);
  } else {
    if (update == 0)
      stencilOp<float, dev::MODE_REPLACE>(o, L, (float*)data(dst, L), (const float*)data(src, L), nullptr, mask, kinds);
    else
      stencilOp<float, dev::MODE_ADD>(o, L, (float*)data(dst, L), (const float*)data(src, L), nullptr, mask, kinds);
  }
}

void Storage::residual(int opId, int x, int b, int r, int L, unsigned mask) {
  Operator& o = op(opId);
  argCheck(L >= o.minL && L <= o.maxL, "level outside the operator's level range");
  argCheck(x != r && b != r, "residual: r must differ from x and b");
  Function& fx = fn(x);
  argCheck(fx.prec == fn(b).prec && fx.prec == fn(r).prec, "residual: precision mismatch");
  communicate(x, L, kAllGroups);
  if (fx.prec == 8)
    stencilOp<double, dev::MODE_RESIDUAL>(o, L, (double*)data(r, L), (const double*)data(x, L), (const double*)data(b, L), mask);
  else
    stencilOp<float, dev::MODE_RESIDUAL>(o, L, (float*)data(r, L), (const float*)data(x, L), (const float*)data(b, L), mask);
}

template <class T>
void Storage::sorT(Operator& o, int dstId, int L, T* u, const T* rhs, unsigned mask, T omega, bool backwards,
                   int kinds, bool refresh, T* cellU, const T* cellF) {
  const LevelData& ld = levels[L];
  const dev::StencilDev<T>& st = stencilOf<T>(o, L);
  const dev::LevelDev& lv = ld.lv;
  const int nVertBlocks = lv.nLowBlocks - lv.nLowEdgeBlocks;
  auto comm = [&](int groups) {
    if (!refresh) return;
    if (cellU) communicateSplit<T>(u, cellU, L, groups);
    else communicate(dstId, L, groups);
  };
  auto verts = [&]() {
    if (nVertBlocks && (kinds & (1 << KV))) {
      dev::lowSorKernel<T><<<nVertBlocks, dev::kBlock, 0, stream>>>(lv, st, u, rhs, mask, -1, omega, lv.nLowEdgeBlocks);
      ++launches;
    }
  };
  auto edges = [&](int c) {
    if (lv.nLowEdgeBlocks && (kinds & (1 << KE))) {
      dev::lowSorKernel<T><<<lv.nLowEdgeBlocks, dev::kBlock, 0, stream>>>(lv, st, u, rhs, mask, c, omega, 0);
      ++launches;
    }
  };
  auto faces = [&](int c) {
    if (lv.nFaceBlocks && (kinds & (1 << KF))) {
      dev::faceSorKernel<T><<<lv.nFaceBlocks, dev::kBlock, 0, stream>>>(lv, st, u, rhs, mask, c, omega);
      ++launches;
    }
  };
  // cell phase: the four colours run group by group (macro-cells whose vectors fit into the L2
  // budget), so the re-reads of the later colours hit L2
  auto cellPhase = [&](bool rev) {
    if (!lv.nCellBlocks || !(kinds & (1 << KC))) return;
    if (cellU) {  // colour-split copy: four in-place passes, one launch each over all cells
      for (int k = 0; k < 4; ++k) {
        const int c = rev ? 3 - k : k, n = ld.nSplitPoints[c];
        if (n == 0) continue;
        const int bpc = (n + dev::kBlock - 1) / dev::kBlock;
        dev::cellSorSplitKernel<T><<<(unsigned)(bpc * lv.nCells), dev::kBlock, 0, stream>>>(
            lv, st.cellW, cellU, cellF, mask, ld.splitRows[c], ld.splitPoints[c], n, bpc, omega);
        ++launches;
      }
      return;
    }
    const int schedule = sorScheduleFor(L, (int)sizeof(T));
    const int pi = sizeof(T) == 4 ? 1 : 0, gv = schedule == 2 ? 1 : 0;
    if ((schedule == 0 || schedule == 2) && ld.nWaveTiles[pi][gv]) {
      // one pass into the spare buffer of this level, which then becomes the function's buffer
      Function& fd = fn(dstId);
      std::unique_ptr<DevBuf>& cur = fd.levels[L - fd.minL];
      spareBuf(spare, L, (int)sizeof(T));
      std::unique_ptr<DevBuf>& sp = spare[{L, (int)sizeof(T)}];
      T* out = (T*)sp->p;
      if (gv == 0)
        dev::cellSorWaveKernel<T, 0><<<ld.nWaveTiles[pi][0], dev::WaveGeom<T, 0>::THREADS,
                                       dev::waveSmemBytes<T, 0>(lv.N), stream>>>(lv, ld.waveTiles[pi][0], st.cellW, u,
                                                                                  out, rhs, mask, omega, rev ? 1 : 0);
      else
        dev::cellSorWaveKernel<T, 1><<<ld.nWaveTiles[pi][1], dev::WaveGeom<T, 1>::THREADS,
                                       dev::waveSmemBytes<T, 1>(lv.N), stream>>>(lv, ld.waveTiles[pi][1], st.cellW, u,
                                                                                  out, rhs, mask, omega, rev ? 1 : 0);
      ++launches;
      const int64_t tail = ld.lay->total - ld.nonCellBegin;
      if (tail > 0)
        cudaCheck(cudaMemcpyAsync(out + ld.nonCellBegin, u + ld.nonCellBegin, tail * sizeof(T), cudaMemcpyDeviceToDevice,
                                  stream),
                  "sor tail copy");
      std::swap(cur, sp);
      u = out;
      return;
    }
    const int nPl = lv.N - 3;
    for (int c0 = 0; c0 < lv.nCells; c0 += ld.cellsPerGroup) {
      const int nc = std::min(ld.cellsPerGroup, lv.nCells - c0);
      for (int k = 0; k < 4; ++k) {
        const int c = rev ? 3 - k : k;
        dev::cellSorKernel<T><<<nc * nPl, dev::kBlock, 0, stream>>>(lv, st.cellW, u, rhs, mask, c, omega, c0);
        ++launches;
      }
    }
  };
  // Fused phases: one launch per face, edge and vertex phase. The refresh of a group is folded
  // into the phase when no owner of its copies belongs to a primitive of the phase: face boundary
  // rows (owned by edges and vertices) before the faces, vertex ghosts (owned by edges, faces and
  // cells) before the vertices of a backward sweep. Edge ghost layers end on the neighbouring
  // edges and face ghost layers on other faces, so those refreshes stay launches of their own.
  if (fusedSorPhases) {
    const uint2* table = cellU ? ld.commSplit : ld.comm;
    const int64_t cellEnd = ld.nonCellBegin;
    T* cellsBuf = cellU;
    auto lowPhase = [&](bool edgesNotVerts, bool gather, bool rev) {
      const int first = edgesNotVerts ? 0 : lv.nEdges, n = edgesNotVerts ? lv.nEdges : lv.nLow - lv.nEdges;
      if (n == 0 || !(kinds & (1 << (edgesNotVerts ? KE : KV)))) return;
      dev::lowSorPhaseKernel<T><<<n, dev::kBlock, 0, stream>>>(lv, st, u, rhs, mask, omega, first, rev ? 1 : 0, table,
                                                             gather && refresh ? ld.lowRange : nullptr, cellsBuf, cellEnd);
      ++launches;
    };
    auto facePhase = [&](bool gather, bool rev) {
      if (lv.nFaceBlocks == 0 || !(kinds & (1 << KF))) return;
      dev::faceSorPhaseKernel<T><<<lv.nFaces, dev::kFacePhaseThreads, 0, stream>>>(
          lv, st, u, rhs, mask, omega, rev ? 1 : 0, table, gather && refresh ? ld.faceRange : nullptr, cellsBuf, cellEnd);
      ++launches;
    };
    if (!backwards) {
      comm((1 << G_VERT) | (1 << G_FACE_GHOST));
      lowPhase(false, false, false);  // vertices
      comm(1 << G_EDGE);              // Vertex -> Edge
      lowPhase(true, false, false);   // edges
      facePhase(true, false);         // Edge -> Face, faces
      comm(1 << G_CELL);              // Face -> Cell
      cellPhase(false);
    } else {
      comm((1 << G_CELL) | (1 << G_FACE_BOUNDARY));
      cellPhase(true);
      comm(1 << G_FACE_GHOST);        // Cell -> Face
      facePhase(false, true);
      comm(1 << G_EDGE);              // Face -> Edge
      lowPhase(true, false, true);    // edges
      lowPhase(false, true, true);    // Edge -> Vertex, vertices
    }
    cudaCheck(cudaGetLastError(), "sor");
    return;
  }
  // Only the copies the reference refreshes between phases are refreshed here, so ghost
  // values that reach a primitive from outside its closure keep their start-of-sweep value.
  // At the start only the groups read before their own refresh in this sweep are brought up to
  // date (forward: vertex ghosts and face ghost layers; backward: cell closures and face
  // boundary rows); the other groups are refreshed again before any phase reads them, so
  // refreshing them here as well would not change a single value that is read.
  comm(backwards ? (1 << G_CELL) | (1 << G_FACE_BOUNDARY) : (1 << G_VERT) | (1 << G_FACE_GHOST));
  if (!backwards) {
    verts();
    comm(1 << G_EDGE);           // Vertex -> Edge
    edges(0);
    edges(1);
    comm(1 << G_FACE_BOUNDARY);  // Edge -> Face
    for (int c = 0; c < 3; ++c) faces(c);
    comm(1 << G_CELL);           // Face -> Cell
    cellPhase(false);
  } else {
    cellPhase(true);
    comm(1 << G_FACE_GHOST);     // Cell -> Face
    for (int c = 2; c >= 0; --c) faces(c);
    comm(1 << G_EDGE);           // Face -> Edge
    edges(1);
    edges(0);
    comm(1 << G_VERT);           // Edge -> Vertex
    verts();
  }
  cudaCheck(cudaGetLastError(), "sor");
}

void Storage::smoothSor(int opId, int dst, int rhs, double omega, int L, unsigned mask, bool backwards, int kinds,
                        bool refresh) {
  Operator& o = op(opId);
  argCheck(L >= o.minL && L <= o.maxL, "level outside the operator's level range");
  argCheck(dst != rhs, "smooth_sor: dst and rhs must differ");
  Function& fd = fn(dst);
  argCheck(fd.prec == fn(rhs).prec, "smooth_sor: precision mismatch");
  for (auto& c : o.host[L - o.minL].cell)
    if (levels[L].lv.nCellBlocks && c[0] == 0.0) throw Error(HG_ERR_NUMERIC, "zero diagonal in cell stencil");
  if (kinds == 15 && refresh && sorScheduleFor(L, fd.prec) == 3 && levels[L].lv.nCellBlocks) {
    smoothSorSweeps(opId, dst, rhs, omega, L, mask, 1, backwards, false);
    return;
  }
  if (fd.prec == 8)
    sorT<double>(o, dst, L, (double*)data(dst, L), (const double*)data(rhs, L), mask, omega, backwards, kinds, refresh);
  else
    sorT<float>(o, dst, L, (float*)data(dst, L), (const float*)data(rhs, L), mask, (float)omega, backwards, kinds,
                refresh);
}

void Storage::smoothSorSweeps(int opId, int dst, int rhs, double omega, int L, unsigned mask, int sweeps,
                              bool backwards, bool rhsReady) {
  Function& fd = fn(dst);
  if (sorScheduleFor(L, fd.prec) != 3 || !levels[L].lv.nCellBlocks || sweeps <= 0) {
    for (int i = 0; i < sweeps; ++i) smoothSor(opId, dst, rhs, omega, L, mask, backwards);
    return;
  }
  Operator& o = op(opId);
  argCheck(L >= o.minL && L <= o.maxL, "level outside the operator's level range");
  argCheck(dst != rhs, "smooth_sor: dst and rhs must differ");
  argCheck(fd.prec == fn(rhs).prec, "smooth_sor: precision mismatch");
  for (auto& c : o.host[L - o.minL].cell)
    if (c[0] == 0.0) throw Error(HG_ERR_NUMERIC, "zero diagonal in cell stencil");
  const LevelData& ld = levels[L];
  const unsigned nb = (unsigned)(ld.lv.nCells * (ld.lv.N + 1));
  auto run = [&](auto zero) {
    using T = decltype(zero);
    T* u = (T*)data(dst, L);
    const T* b = (const T*)data(rhs, L);
    buildSplit(L);
    T* cu = (T*)spareBuf(spare, L, (int)sizeof(T)).p;
    T* cf = (T*)spareBuf(splitRhs, L, (int)sizeof(T)).p;
    dev::cellSplitKernel<T, true><<<nb, dev::kBlock, 0, stream>>>(ld.lv, cu, u);
    ++launches;
    if (!rhsReady) {
      dev::cellSplitKernel<T, true><<<nb, dev::kBlock, 0, stream>>>(ld.lv, cf, b);
      ++launches;
    }
    for (int i = 0; i < sweeps; ++i) sorT<T>(o, dst, L, u, b, mask, (T)omega, backwards, 15, true, cu, cf);
    dev::cellSplitKernel<T, false><<<nb, dev::kBlock, 0, stream>>>(ld.lv, u, cu);
    ++launches;
    cudaCheck(cudaGetLastError(), "sor (colour-split)");
  };
  if (fd.prec == 8) run(0.0);
  else run(0.0f);
}

// The fine-level face/edge/vertex stencil structure drives the restriction; it is taken from
// a structure-only Laplace stencil owned by the storage (weights unused).
const Operator& Storage::structure() {
  if (structureOp < 0) structureOp = createOperator(FORM_LAPLACE, 0, maxLevel());
  return op(structureOp);
}

template <class T>
void Storage::restrictT(int id, int Lf, unsigned mask, int coarseDst) {
  const int Lc = Lf - 1;
  const LevelData& lc = levels[Lc];
  const LevelData& lf = levels[Lf];
  T* coarse = (T*)data(coarseDst >= 0 ? coarseDst : id, Lc);
  const T* fine = (const T*)data(id, Lf);
  Operator& so = const_cast<Operator&>(structure());
  const dev::StencilDev<T>& stf = stencilOf<T>(so, Lf);
  communicate(id, Lf, kAllGroups);
  if (lc.lv.nCellBlocks) {
    dev::cellRestrictKernel<T><<<lc.lv.nCellBlocks, dev::kBlock, 0, stream>>>(lc.lv, lf.lv, coarse, fine, mask);
    ++launches;
  }
  if (lc.lv.nFaceBlocks) {
    dev::faceRestrictKernel<T><<<lc.lv.nFaceBlocks, dev::kBlock, 0, stream>>>(lc.lv, lf.lv, stf, coarse, fine, mask);
    ++launches;
  }
  if (lc.lv.nLowBlocks) {
    dev::lowRestrictKernel<T><<<lc.lv.nLowBlocks, dev::kBlock, 0, stream>>>(lc.lv, lf.lv, stf, coarse, fine, mask);
    ++launches;
  }
  cudaCheck(cudaGetLastError(), "restrict");
}

void Storage::restrictFn(int id, int Lf, unsigned mask, int coarseDst) {
  Function& f = fn(id);
  argCheck(Lf - 1 >= f.minL && Lf <= f.maxL, "restrict: levels outside the function's range");
  if (coarseDst >= 0) {
    const Function& d = fn(coarseDst);
    argCheck(d.prec == f.prec && Lf - 1 >= d.minL && Lf - 1 <= d.maxL, "restrict: coarse function mismatch");
  }
  if (f.prec == 8) restrictT<double>(id, Lf, mask, coarseDst);
  else restrictT<float>(id, Lf, mask, coarseDst);
}

template <class T>
void Storage::prolongT(int id, int Lc, unsigned mask, bool add) {
  const int Lf = Lc + 1;
  const LevelData& lc = levels[Lc];
  const LevelData& lf = levels[Lf];
  T* fine = (T*)data(id, Lf);
  const T* coarse = (const T*)data(id, Lc);
  communicate(id, Lc, kAllGroups);
  if (lf.lv.nCellBlocks) {
    if (add) dev::cellProlongKernel<T, true><<<lf.lv.nCellBlocks, dev::kBlock, 0, stream>>>(lf.lv, lc.lv, fine, coarse, mask);
    else dev::cellProlongKernel<T, false><<<lf.lv.nCellBlocks, dev::kBlock, 0, stream>>>(lf.lv, lc.lv, fine, coarse, mask);
    ++launches;
  }
  if (lf.lv.nFaceBlocks) {
    if (add) dev::faceProlongKernel<T, true><<<lf.lv.nFaceBlocks, dev::kBlock, 0, stream>>>(lf.lv, lc.lv, fine, coarse, mask);
    else dev::faceProlongKernel<T, false><<<lf.lv.nFaceBlocks, dev::kBlock, 0, stream>>>(lf.lv, lc.lv, fine, coarse, mask);
    ++launches;
  }
  if (lf.lv.nLowBlocks) {
    if (add) dev::lowProlongKernel<T, true><<<lf.lv.nLowBlocks, dev::kBlock, 0, stream>>>(lf.lv, lc.lv, fine, coarse, mask);
    else dev::lowProlongKernel<T, false><<<lf.lv.nLowBlocks, dev::kBlock, 0, stream>>>(lf.lv, lc.lv, fine, coarse, mask);
    ++launches;
  }
  cudaCheck(cudaGetLastError(), "prolongate");
}

void Storage::prolongate(int id, int Lc, unsigned mask, bool add) {
  Function& f = fn(id);
  argCheck(Lc >= f.minL && Lc + 1 <= f.maxL, "prolongate: levels outside the function's range");
  if (f.prec == 8) prolongT<double>(id, Lc, mask, add);
  else prolongT<float>(id, Lc, mask, add);
}

}  // namespace hg
