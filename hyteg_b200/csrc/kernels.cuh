// Device kernels of the B200 matrix-free P1 multigrid path (sm_100a).
//
// All kernels are bandwidth-bound stencil sweeps over the reference's per-primitive array
// layout (see discretization.hpp). Work is distributed by host-built block tables:
//   cell blocks  : (cell, z, first plane offset)   one 256-thread block per slice of a z-plane
//   face blocks  : (face, first triangle offset)
//   low  blocks  : (edge-or-vertex, first x)
// Threads decode their (x, y) inside a triangular plane with one rounded square root, so a
// block reads contiguous x-rows (coalesced) and the neighbouring rows of the planes z-1 and
// z+1 are served from L1/L2. Primitive boundary types are tested in-kernel against the
// DoFType mask, so one launch covers every primitive of a kind.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <utility>

#include "p2_stencil.h"

namespace hg {
namespace dev {

constexpr int kBlock = 256;

struct FaceBlock {
  int face, start;  // rows [start, start + kFaceRows) of the face interior
};
struct LowBlock {
  int prim, start;
};
template <class T>
struct FaceEnt {
  T w;
  int layer, dx, dy;
};

// Per-level geometry shared by all functions (device pointers).
struct LevelDev {
  int L;
  int N, w;
  int nCells, nFaces, nLow, nEdges;  // low primitives: edges [0, nEdges) then vertices
  const int64_t* cellOff;
  const int64_t* faceOff;
  const int64_t* lowOff;
  const int* lowFirst;  // first owned x (1 for edges, 0 for vertices)
  const int* lowCount;  // owned points
  const unsigned char* cellType;
  const unsigned char* faceType;
  const unsigned char* lowType;
  int nCellBlocks;  // nCells * (N - 3) blocks (one per macro-cell and z-plane), 0 below level 2
  const FaceBlock* faceBlocks;
  int nFaceBlocks;
  const LowBlock* lowBlocks;
  int nLowBlocks;  // edges' blocks first (nLowEdgeBlocks of them), then vertices
  int nLowEdgeBlocks;
};

// Per-level constant stencils of one operator (device pointers).
template <class T>
struct StencilDev {
  const T* cellW;            // [nCells][16]
  const FaceEnt<T>* faceEnt;  // [nFaces][16]
  const int* faceEntCount;    // [nFaces]
  const int* lowEntOff;       // [nLow + 1]
  const int64_t* lowEntRel;   // [entries]
  const T* lowEntW;           // [entries]
};

enum Mode { MODE_REPLACE = 0, MODE_ADD = 1, MODE_RESIDUAL = 2 };

__device__ __forceinline__ int rowStart(int W, int y) { return y * (W + 1) - (y * (y + 1)) / 2; }
__device__ __forceinline__ int64_t tetSize(int64_t w) { return w * (w + 1) * (w + 2) / 6; }
__device__ __forceinline__ int triSize(int w) { return w * (w + 1) / 2; }

// ---------------------------------------------------------------------------------------
// Cell interiors. One block per (macro-cell, z-plane); the warps of a block walk the rows y
// of the plane and the lanes the x positions of a row. All neighbour rows of a row are
// addressed from six row bases computed once per row (cell layout of
// indexing/MacroCellIndexing.hpp:40-52):
//   r0  (0, y, z)     rN (0, y+1, z)    rS (0, y-1, z)
//   rT  (0, y, z+1)   rTS (0, y-1, z+1)
//   rB  (0, y, z-1)   rBN (0, y+1, z-1)
// Consecutive blocks are neighbouring planes, so the z-1 / z+1 rows a block reads are those
// its neighbours stream in: each value comes from HBM about once and from L2 about three times.
// ---------------------------------------------------------------------------------------
struct CellRow {
  int r0, rN, rS, rT, rTS, rB, rBN;
};

__device__ __forceinline__ CellRow cellRow(int w, int z, int y) {
  const int W = w - z;
  CellRow r;
  r.r0 = int(tetSize(w) - tetSize(W)) + rowStart(W, y);
  r.rN = r.r0 + (W - y);
  r.rS = r.r0 - (W - y + 1);
  r.rT = r.r0 + triSize(W) - y;
  r.rTS = r.rT - (W - y);
  r.rB = r.r0 - triSize(W + 1) + y;
  r.rBN = r.rB + (W + 1 - y);
  return r;
}

// sum_{k >= 1} w_k u(x + d_k) in the order E W N S NW SE TC TW TS TSE BC BE BN BNW
template <class T, class LD>
__device__ __forceinline__ T cellOffDiag(const T* wt, const CellRow& r, int x, LD ld) {
  T s = wt[1] * ld(r.r0 + x + 1);
  s += wt[2] * ld(r.r0 + x - 1);
  s += wt[3] * ld(r.rN + x);
  s += wt[4] * ld(r.rS + x);
  s += wt[5] * ld(r.rN + x - 1);
  s += wt[6] * ld(r.rS + x + 1);
  s += wt[7] * ld(r.rT + x);
  s += wt[8] * ld(r.rT + x - 1);
  s += wt[9] * ld(r.rTS + x);
  s += wt[10] * ld(r.rTS + x + 1);
  s += wt[11] * ld(r.rB + x);
  s += wt[12] * ld(r.rB + x + 1);
  s += wt[13] * ld(r.rBN + x);
  s += wt[14] * ld(r.rBN + x - 1);
  return s;
}

// dst = A src | dst += A src | dst = rhs - A src on cell interiors. The weights live in shared
// memory (broadcast reads) and every lane handles two points per iteration, so up to 30
// independent loads per thread are in flight.
template <class T, int MODE>
__global__ void __launch_bounds__(kBlock, 4) cellStencilKernel(LevelDev lv, const T* __restrict__ cellW,
                                                               T* __restrict__ dst, const T* __restrict__ src,
                                                               const T* __restrict__ rhs, unsigned mask) {
  const int nPl = lv.N - 3;
  const int c = blockIdx.x / nPl, z = 1 + blockIdx.x % nPl;
  if (!(lv.cellType[c] & mask)) return;
  __shared__ T wt[16];
  if (threadIdx.x < 15) wt[threadIdx.x] = cellW[16 * c + threadIdx.x];
  __syncthreads();
  const int64_t base = lv.cellOff[c];
  const T* __restrict__ u = src + base;
  T* __restrict__ d = dst + base;
  const T* __restrict__ f = rhs + base;
  const int W = lv.w - z;
  auto ld = [u](int i) { return __ldg(u + i); };
  for (int y = 1 + (int)(threadIdx.x >> 5); y <= W - 3; y += kBlock / 32) {
    const CellRow r = cellRow(lv.w, z, y);
    const int len = W - 2 - y;
    for (int x = 1 + (int)(threadIdx.x & 31); x <= len; x += 64) {
      const int x2 = x + 32;
      const bool two = x2 <= len;
      const T s1 = wt[0] * ld(r.r0 + x) + cellOffDiag(wt, r, x, ld);
      const T s2 = two ? wt[0] * ld(r.r0 + x2) + cellOffDiag(wt, r, x2, ld) : T(0);
      if (MODE == MODE_REPLACE) {
        d[r.r0 + x] = s1;
        if (two) d[r.r0 + x2] = s2;
      } else if (MODE == MODE_ADD) {
        d[r.r0 + x] += s1;
        if (two) d[r.r0 + x2] += s2;
      } else {
        d[r.r0 + x] = f[r.r0 + x] - s1;
        if (two) d[r.r0 + x2] = f[r.r0 + x2] - s2;
      }
    }
  }
}

// Multicolour SOR on cell interiors, colour = (x + 2y + 3z) mod 4: the lanes of a warp step
// over the x positions of the active colour only (every fourth point of a row), two per lane.
template <class T>
__global__ void __launch_bounds__(kBlock, 4) cellSorKernel(LevelDev lv, const T* __restrict__ cellW, T* u,
                                                           const T* __restrict__ rhs, unsigned mask, int colour,
                                                           T omega, int cellBegin) {
  const int nPl = lv.N - 3;
  const int c = cellBegin + blockIdx.x / nPl, z = 1 + blockIdx.x % nPl;
  if (!(lv.cellType[c] & mask)) return;
  __shared__ T wt[16];
  if (threadIdx.x < 15) wt[threadIdx.x] = cellW[16 * c + threadIdx.x];
  __syncthreads();
  const int64_t base = lv.cellOff[c];
  T* uc = u + base;
  const T* __restrict__ f = rhs + base;
  const T om = omega, om1 = T(1) - omega;
  const int W = lv.w - z;
  auto ld = [uc](int i) { return uc[i]; };
  for (int y = 1 + (int)(threadIdx.x >> 5); y <= W - 3; y += kBlock / 32) {
    const CellRow r = cellRow(lv.w, z, y);
    const int len = W - 2 - y;
    const int x0 = 1 + (((colour - 2 * y - 3 * z - 1) % 4) + 4) % 4;
    for (int x = x0 + 4 * (int)(threadIdx.x & 31); x <= len; x += 256) {
      const int x2 = x + 128;
      const bool two = x2 <= len;
      const T s1 = f[r.r0 + x] - cellOffDiag(wt, r, x, ld);
      const T s2 = two ? f[r.r0 + x2] - cellOffDiag(wt, r, x2, ld) : T(0);
      uc[r.r0 + x] = om1 * uc[r.r0 + x] + (s1 * om) / wt[0];
      if (two) uc[r.r0 + x2] = om1 * uc[r.r0 + x2] + (s2 * om) / wt[0];
    }
  }
}

// ---------------------------------------------------------------------------------------
// Multicolour SOR on cell interiors in a single pass (z-wavefront, out of place).
// The colour of (x, y, z) is (x + 2y + 3z) mod 4 and the sweep visits the colours in the
// sequence seq = 0,1,2,3 (backwards: 3,2,1,0). At step s a block runs colour seq[k] on plane
// s - 2k for k = 0..3. For every stencil offset a neighbour earlier in the sequence was updated
// in an earlier step and a neighbour later in the sequence is updated in a later step, so the
// result equals four separate colour sweeps over the whole cell, and the four stages of a step
// touch disjoint data (they write the planes s, s-2, s-4, s-6 and read only those and the odd
// planes between them) and need no barrier between them.
// A block owns a 32 x TY (x, y) tile of one macro-cell for all planes (WaveCfg). It recomputes a shrinking
// halo (stage k on the tile widened by 3 - k) from the start-of-sweep values, which makes the
// tiles independent: they read uOld and write uNew, and the caller swaps the two buffers.
// Planes s-7 .. s+1 (and s-8 with a 10-plane ring) of the tile widened by 4 (40 x (TY + 8) points)
// live in a shared-memory ring; plane s+2 is loaded into registers during step s and stored into
// the slot of the oldest plane. Point (rx, ry) of the region sits at
//   ry * 42 + ((rx mod 4 + 2 ry) mod 4) * 10 + rx / 4,
// i.e. each row is split by x mod 4 and the split is rotated by 2y. The points of one colour then
// occupy the same sub-row of every row, and with the row stride 42 (= 10 mod 16) the 16 lanes
// of a half-warp never share a bank pair. Thread t < 10 (TY + 8) owns the columns 4(t mod 10) .. +3
// of region row t / 10: it loads and stores them and, in every stage, updates the one of them
// that carries the stage's colour.
// ---------------------------------------------------------------------------------------
constexpr int kWaveTX = 32;                         // tile extent in x (multiple of 4)
constexpr int kWaveH = 4;                           // halo loaded around the tile
constexpr int kWaveRX = kWaveTX + 2 * kWaveH;       // region extent in x (40)
constexpr int kWaveQ = kWaveRX / 4;                 // column groups per region row (10)
constexpr int kWaveS = 42;                          // shared-memory row stride (10 mod 16)
constexpr int kWaveMaxN = 4096;                     // largest level size the shared-memory limit is set for

// Tile height, block size, blocks per SM and ring planes per precision. A 10-plane ring needs one
// barrier per step instead of two. FP64: 32 x 24 tiles (region 40 x 32, 320 column groups),
// 108 KB of ring, two blocks per SM; FP32: 32 x 28 tiles (region 40 x 36, 360 groups), 61 KB,
// three blocks per SM (a register budget of 56 per thread). Measured per level-8 sweep, FP64:
// 2.21 ms (32 x 24, 10 planes), 2.34 ms (32 x 28, 9 planes, two barriers), 2.35 ms (32 x 16, 9,
// three blocks per SM), 2.78 ms (32 x 60, 9, one block per SM); FP32: 1.36 ms (32 x 28, 10
// planes), 1.41 ms (32 x 28, 9 planes), 1.67 ms (four blocks per SM at 40 registers), 1.83 ms
// (32 x 60, two blocks per SM).
// V = 1 is a second, shorter tile (32 x 12) for the autotuner: more blocks per SM and more tiles
// per level, for levels whose 32 x 24 (28) tiles fill the GPU in few waves.
template <class T, int V = 0>
struct WaveCfg;
template <>
struct WaveCfg<double, 0> {
  static constexpr int TY = 24, THREADS = 320, MIN_BLOCKS = 2, SLOTS = 10;
};
template <>
struct WaveCfg<float, 0> {
  static constexpr int TY = 28, THREADS = 384, MIN_BLOCKS = 3, SLOTS = 10;
};
template <>
struct WaveCfg<double, 1> {
  static constexpr int TY = 12, THREADS = 224, MIN_BLOCKS = 3, SLOTS = 10;
};
template <>
struct WaveCfg<float, 1> {
  static constexpr int TY = 12, THREADS = 224, MIN_BLOCKS = 4, SLOTS = 10;
};
template <class T, int V = 0>
struct WaveGeom {
  static constexpr int TY = WaveCfg<T, V>::TY;        // tile extent in y (even)
  static constexpr int RY = TY + 2 * kWaveH;          // region extent in y
  static constexpr int PLANE = RY * kWaveS;           // elements per plane slot
  static constexpr int GROUPS = RY * kWaveQ;          // column groups, one per thread
  static constexpr int THREADS = WaveCfg<T, V>::THREADS;
  static constexpr int SLOTS = WaveCfg<T, V>::SLOTS;  // ring planes: 9 (s-7 .. s+1), or 10 to drop a barrier
  static_assert(THREADS >= GROUPS && THREADS % 32 == 0 && TY % 2 == 0, "wave tile configuration");
  static_assert(SLOTS == 9 || SLOTS == 10, "wave ring size");
};

struct WaveTile {
  int cell, x0, y0, pEnd;  // tile origin; pEnd = N - x0 - y0, its last plane
};

// Dynamic shared memory of the kernel for level size N.
template <class T, int V = 0>
inline size_t waveSmemBytes(int N) {
  return size_t(WaveGeom<T, V>::SLOTS) * WaveGeom<T, V>::PLANE * sizeof(T) + size_t(N + 2) * sizeof(int);
}

template <class T, int V>
__global__ void __launch_bounds__(WaveCfg<T, V>::THREADS, WaveCfg<T, V>::MIN_BLOCKS)
    cellSorWaveKernel(LevelDev lv, const WaveTile* __restrict__ tiles, const T* __restrict__ cellW,
                      const T* __restrict__ uOld, T* __restrict__ uNew, const T* __restrict__ rhs, unsigned mask,
                      T omega, int backwards) {
  constexpr int kTY = WaveGeom<T, V>::TY, kRY = WaveGeom<T, V>::RY, kPlane = WaveGeom<T, V>::PLANE;
  constexpr int kGroups = WaveGeom<T, V>::GROUPS, kThreads = WaveGeom<T, V>::THREADS, kSlots = WaveGeom<T, V>::SLOTS;
  extern __shared__ __align__(16) unsigned char waveSmem[];
  T* sm = reinterpret_cast<T*>(waveSmem);
  int* pbTab = reinterpret_cast<int*>(sm + kSlots * kPlane);  // first index of plane p
  const WaveTile tl = tiles[blockIdx.x];
  const int N = lv.N, w = lv.w, tid = threadIdx.x;
  const int64_t base = lv.cellOff[tl.cell];
  const T* __restrict__ uo = uOld + base;
  T* __restrict__ un = uNew + base;
  const T* __restrict__ f = rhs + base;
  const int xb = tl.x0 - kWaveH, yb = tl.y0 - kWaveH;  // region origin in cell coordinates
  for (int p = tid; p <= N; p += kThreads) pbTab[p] = int(tetSize(w) - tetSize(w - p));
  // the thread's column group: region row gy, region columns 4 gx .. 4 gx + 3
  const bool owner = tid < kGroups;
  const int gy = tid / kWaveQ, gx = tid - (tid / kWaveQ) * kWaveQ;
  const int y = yb + gy, x4 = xb + 4 * gx;
  const int Ay = y * (w + 1) - (y * (y + 1)) / 2;  // rowStart(w - p, y) = Ay - y p
  const int rot = (2 * gy) & 3;                     // sub-row of column j: (j + rot) mod 4
  const int so = gy * kWaveS + gx;
  const bool storer = owner && gy >= kWaveH && gy < kWaveH + kTY && gx >= 1 && gx < kWaveQ - 1;
  __syncthreads();

  if (!(lv.cellType[tl.cell] & mask)) {  // not smoothed: the tile is copied
    if (storer)
      for (int p = 0; p <= tl.pEnd; ++p)
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (x4 + j + y <= N - p) {
            const int g = pbTab[p] + Ay - y * p + x4 + j;
            un[g] = uo[g];
          }
    return;
  }
  T wt[15];
#pragma unroll
  for (int k = 0; k < 15; ++k) wt[k] = cellW[16 * tl.cell + k];
  const T om1 = T(1) - omega, dinv = omega / wt[0];
  unsigned rowBits = 0;  // bit k: row gy lies in the region of stage k and y >= 1
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (owner && gy >= k + 1 && gy < kRY - 1 - k && y >= 1) rowBits |= 1u << k;

  T stg[4];
  auto loadRegs = [&](int p) {  // plane p of the thread's columns (points of the closed cell)
    if (owner && p <= N && y >= 0 && y <= N - p) {
      const int g = pbTab[p] + Ay - y * p + x4;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (x4 + j >= 0 && x4 + j + y <= N - p) stg[j] = uo[g + j];
    }
  };
  auto storeRegs = [&](int p, int slot) {
    if (owner && p <= N && y >= 0 && y <= N - p) {
      T* s = sm + slot * kPlane + so;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (x4 + j >= 0 && x4 + j + y <= N - p) s[((j + rot) & 3) * kWaveQ] = stg[j];
    }
  };
  // colour seq[k] on plane p (ring slot sp, neighbours in slots st and sb); region = tile
  // widened by 3 - k
  auto stage = [&](int k, int p, int sp, int st, int sb) {
    if (!((rowBits >> k) & 1u)) return;
    const int c = backwards ? 3 - k : k;
    const int q = (c - 2 * y + p) & 3;  // x mod 4 of colour c in row y of plane p
    const int rx = 4 * gx + q, x = xb + rx;
    if (rx < k + 1 || rx >= kWaveRX - 1 - k || x < 1 || x + y > N - 1 - p) return;
    const int sg = (q + rot) & 3;  // its sub-row
    const int e1 = sg < 3 ? kWaveQ : -3 * kWaveQ, w1 = sg > 0 ? -kWaveQ : 3 * kWaveQ;
    const int n2 = sg < 2 ? 2 * kWaveQ : -2 * kWaveQ;
    const int qe = q == 3 ? 1 : 0, qw = q == 0 ? 1 : 0;
    const int dE = e1 + qe, dW = w1 - qw, dN = kWaveS + n2, dS = n2 - kWaveS;
    const int dNW = kWaveS + e1 - qw, dSE = w1 - kWaveS + qe;
    const int o = so + sg * kWaveQ;
    T* sP = sm + sp * kPlane + o;
    const T* sT = sm + st * kPlane + o;
    const T* sB = sm + sb * kPlane + o;
    const T rh = f[pbTab[p] + Ay - y * p + x];
    // three independent partial sums (this plane, the plane above, the plane below)
    T a = wt[1] * sP[dE];
    a += wt[2] * sP[dW];
    a += wt[3] * sP[dN];
    a += wt[4] * sP[dS];
    a += wt[5] * sP[dNW];
    a += wt[6] * sP[dSE];
    T t = wt[7] * sT[0];
    t += wt[8] * sT[dW];
    t += wt[9] * sT[dS];
    t += wt[10] * sT[dSE];
    T b = wt[11] * sB[0];
    b += wt[12] * sB[dE];
    b += wt[13] * sB[dN];
    b += wt[14] * sB[dNW];
    sP[0] = om1 * sP[0] + (rh - (a + (t + b))) * dinv;
  };
  auto store = [&](int p, int slot) {  // the tile's points of plane p (interior and boundary) to uNew
    if (!storer || y > N - p) return;
    const T* s = sm + slot * kPlane + so;
    const int g = pbTab[p] + Ay - y * p + x4;
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (x4 + j + y <= N - p) un[g + j] = s[((j + rot) & 3) * kWaveQ];
  };
  auto wrap = [](int v) { return v >= kSlots ? v - kSlots : v; };  // v in [0, 2 * slots)

  loadRegs(0);
  storeRegs(0, 0);
  loadRegs(1);
  storeRegs(1, 1);
  const int sEnd = tl.pEnd + 6;
  // Plane p lives in ring slot p mod kSlots. With 9 slots, plane s+2 takes the slot of plane s-7,
  // which stage 3 of the same step still reads: a second barrier separates them. With 10 slots it
  // takes the slot of plane s-8, last read in step s-1 (stage 3 on plane s-7) and so already
  // behind the first barrier of step s. The store of plane s-6 reads only the thread's own
  // columns, whose final values the thread itself wrote in stage 3 of this step.
  int ss = 0;  // s mod kSlots
  for (int s = 0; s <= sEnd; ++s) {
    loadRegs(s + 2);
    __syncthreads();  // the previous step's stores into the ring are visible
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int p = s - 2 * k;
      const int sp = wrap(ss + kSlots - 2 * k);  // slot of plane p
      if (p >= 1 && p <= N - 3) stage(k, p, sp, wrap(sp + 1), wrap(sp + kSlots - 1));
    }
    if (kSlots == 9) __syncthreads();  // plane s-7 is no longer read
    storeRegs(s + 2, wrap(ss + 2));
    if (s >= 6 && s - 6 <= tl.pEnd) store(s - 6, wrap(ss + kSlots - 6));
    ss = wrap(ss + 1);
  }
}

// ---------------------------------------------------------------------------------------
// Colour-split order of the closed macro-cells (SOR schedule 3). Every row (y, z) keeps its
// slots, and inside a row of m points the points are ordered by x mod 4, then by x: sub-row q
// holds x = q, q + 4, ... and starts at slot q * (m / 4) + min(q, m mod 4) of the row. The
// points of one colour ((x + 2y + 3z) mod 4) then fill one sub-row of every row, and a colour
// pass reads and writes whole runs of consecutive slots instead of every fourth one. The SOR
// converts a level into this order before its sweeps and back after them.
// ---------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ int splitSub(int m, int q) { return q * (m >> 2) + (q < (m & 3) ? q : (m & 3)); }

// Position in the colour-split order of point p of a triangle plane with W points per edge
// (p = rowStart(W, y) + x). The row comes from the root of rowStart(W, y) = y (2W + 1 - y) / 2
// and is corrected by whole rows.
__device__ __forceinline__ int splitOfPlanePoint(int W, int p) {
  const float b = float(2 * W + 1);
  int y = int((b - sqrtf(fmaxf(b * b - 8.0f * float(p), 0.0f))) * 0.5f);
  y = max(0, min(y, W - 1));
  while (y > 0 && rowStart(W, y) > p) --y;
  while (y < W - 1 && rowStart(W, y + 1) <= p) ++y;
  const int r0 = rowStart(W, y), x = p - r0;
  return r0 + splitSub(W - y, x & 3) + (x >> 2);
}

// dst = src with the cell arrays converted into (TO_SPLIT) or out of the colour-split order;
// one block per (macro-cell, plane), the threads walk the plane's points (kSplitUnroll each per
// round, loads before stores).
constexpr int kSplitUnroll = 4;
template <class T, bool TO_SPLIT>
__global__ void __launch_bounds__(kBlock) cellSplitKernel(LevelDev lv, T* __restrict__ dst, const T* __restrict__ src) {
  const int nPl = lv.N + 1;
  const int c = blockIdx.x / nPl, z = blockIdx.x - (blockIdx.x / nPl) * nPl;
  const int W = lv.w - z;  // points on an edge of plane z
  const int64_t base = lv.cellOff[c] + (tetSize(lv.w) - tetSize(W));
  const int n = triSize(W);
  for (int p0 = threadIdx.x; p0 < n; p0 += kBlock * kSplitUnroll) {
    T v[kSplitUnroll];
    int to[kSplitUnroll];
#pragma unroll
    for (int k = 0; k < kSplitUnroll; ++k) {
      const int p = p0 + k * kBlock;
      if (p < n) {
        const int s = splitOfPlanePoint(W, p);
        v[k] = TO_SPLIT ? src[base + p] : src[base + s];
        to[k] = TO_SPLIT ? s : p;
      }
    }
#pragma unroll
    for (int k = 0; k < kSplitUnroll; ++k)
      if (p0 + k * kBlock < n) dst[base + to[k]] = v[k];
  }
}

// One colour pass of the multicolour SOR on cell interiors held in the colour-split order
// (the same update as cellSorKernel). The points of the colour in row (y, z) are x = q + 4j, and
// each of the 14 neighbours of such a point lies in sub-row (q + dx) mod 4 of its row at position
// j + floor((q + dx) / 4): all 15 slots a point touches are a per-row constant plus j. The rows
// of one colour (the same in every macro-cell of a level) are listed once with these 15 constants
// (SplitRow), and every point of the colour once as (row << 10 | j), so one thread updates one
// point and consecutive threads read runs of consecutive slots, whatever the row lengths. A
// colour never neighbours itself: the neighbours are constant during the pass and are read
// through the read-only path.
struct SplitRow {
  int i[16];  // slots (cell-relative, at j = 0) of C E W N S NW SE TC TW TS TSE BC BE BN BNW; pad
};
constexpr int kSplitJBits = 10;

template <class T>
__global__ void __launch_bounds__(kBlock) cellSorSplitKernel(LevelDev lv, const T* __restrict__ cellW, T* u,
                                                             const T* __restrict__ rhs, unsigned mask,
                                                             const SplitRow* __restrict__ rows,
                                                             const unsigned* __restrict__ points, int nPoints,
                                                             int blocksPerCell, T omega) {
  const int c = blockIdx.x / blocksPerCell;
  if (!(lv.cellType[c] & mask)) return;
  __shared__ T wt[16];
  if (threadIdx.x < 15) wt[threadIdx.x] = cellW[16 * c + threadIdx.x];
  __syncthreads();
  const int t = (blockIdx.x - c * blocksPerCell) * kBlock + threadIdx.x;
  if (t >= nPoints) return;
  const unsigned e = __ldg(points + t);
  const int4* rp = reinterpret_cast<const int4*>(rows + (e >> kSplitJBits));
  const int4 r0 = __ldg(rp), r1 = __ldg(rp + 1), r2 = __ldg(rp + 2), r3 = __ldg(rp + 3);
  const int64_t base = lv.cellOff[c] + (int64_t)(e & ((1u << kSplitJBits) - 1));
  T* uc = u + base;
  // sum_{k >= 1} w_k u(x + d_k) in the order E W N S NW SE TC TW TS TSE BC BE BN BNW
  T s = wt[1] * __ldg(uc + r0.y);
  s += wt[2] * __ldg(uc + r0.z);
  s += wt[3] * __ldg(uc + r0.w);
  s += wt[4] * __ldg(uc + r1.x);
  s += wt[5] * __ldg(uc + r1.y);
  s += wt[6] * __ldg(uc + r1.z);
  s += wt[7] * __ldg(uc + r1.w);
  s += wt[8] * __ldg(uc + r2.x);
  s += wt[9] * __ldg(uc + r2.y);
  s += wt[10] * __ldg(uc + r2.z);
  s += wt[11] * __ldg(uc + r2.w);
  s += wt[12] * __ldg(uc + r3.x);
  s += wt[13] * __ldg(uc + r3.y);
  s += wt[14] * __ldg(uc + r3.z);
  const T om1 = T(1) - omega, dinv = omega / wt[0];
  uc[r0.x] = om1 * uc[r0.x] + (__ldg(rhs + base + r0.x) - s) * dinv;
}

// ---------------------------------------------------------------------------------------
// Register-blocked 2.5-D cell sweep (the kernel behind apply and residual on cell interiors).
// A warp owns a strip of 30 x-columns (lanes 1..30; lanes 0 and 31 only carry the x-halo) by
// R rows (StripCfg) and marches up z through a range of planes. Each lane keeps the rows
// y0-1 .. y0+R of the planes z-1, z, z+1 of its own column in registers and has plane z+2
// (and the second vector's rows of plane z+1) in flight while plane z is computed;
// x-neighbours come from the adjacent lanes through warp shuffles. Addresses advance
// incrementally: index(x, y, z+1) = index(x, y, z) + tri(w - z) - y.
// Every value is loaded (R+2)/R times per sweep (the extra rows are the neighbouring strips'
// rows, L1 hits). No shared memory, no block synchronisation.
// ---------------------------------------------------------------------------------------
constexpr int kStripX = 30;                         // computed columns per warp
constexpr int kStripZ = 32;                         // planes per work item
constexpr int kStripRows = 32;                      // rows per block (strips stacked in y)
// Rows per strip and blocks per SM by precision. Eight rows per warp keep ten rows of the next
// plane in flight per lane and re-read a quarter of the rows (the neighbouring strips' halo
// rows). Measured per level-8 FP64 cell apply: 0.618 ms (8 rows, 3 blocks of 4 warps per SM),
// 0.670 ms (4 rows, 2 blocks of 8 warps), 0.857 ms (8 rows, 2 blocks); FP32: 8 rows in 4 blocks.
template <class T>
struct StripCfg;
template <>
struct StripCfg<double> {
  static constexpr int R = 8, MIN_BLOCKS = 3;
};
template <>
struct StripCfg<float> {
  static constexpr int R = 8, MIN_BLOCKS = 4;
};
template <class T>
constexpr int stripThreads() {
  return 32 * (kStripRows / StripCfg<T>::R);
}

struct StripItem {
  int cell, x0, y0, z0, z1, pad0, pad1, pad2;  // columns [x0, x0+30), rows [y0, y0+32), planes [z0, z1)
};

enum StripOp { STRIP_REPLACE = 0, STRIP_ADD = 1, STRIP_RESIDUAL = 2 };

template <class T>
__device__ __forceinline__ T shUp(T v) {  // value of lane - 1 (x - 1)
  return __shfl_up_sync(0xffffffffu, v, 1);
}
template <class T>
__device__ __forceinline__ T shDown(T v) {  // value of lane + 1 (x + 1)
  return __shfl_down_sync(0xffffffffu, v, 1);
}

template <class T, int OP>
__global__ void __launch_bounds__(stripThreads<T>(), StripCfg<T>::MIN_BLOCKS)
    cellStripKernel(LevelDev lv, const StripItem* __restrict__ items, const T* __restrict__ cellW, T* __restrict__ dst,
                    const T* __restrict__ src, const T* __restrict__ rhs, unsigned mask) {
  constexpr int kStripR = StripCfg<T>::R;       // rows per strip
  constexpr int kStripH = kStripR + 2;          // rows held per plane (with y-halo)
  const StripItem it = items[blockIdx.x];
  if (!(lv.cellType[it.cell] & mask)) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int N = lv.N, w = lv.w;
  const int x = it.x0 - 1 + lane;                    // lane 0: x0 - 1, lanes 1..30: x0 .. x0+29
  const int y0 = it.y0 + warp * kStripR;
  // last plane with an interior point in this strip: x + y + z <= N - 1 with x >= x0, y >= y0
  const int zEnd = min(it.z1, N - it.x0 - y0);
  if (it.z0 >= zEnd) return;
  const int64_t base = lv.cellOff[it.cell];
  const T* __restrict__ u = src + base;
  const T* __restrict__ f = (OP == STRIP_ADD) ? dst + base : rhs + base;
  constexpr bool kSecond = OP != STRIP_REPLACE;
  T wt[15];
#pragma unroll
  for (int k = 0; k < 15; ++k) wt[k] = __ldg(cellW + 16 * it.cell + k);
  const bool computeLane = lane >= 1 && lane <= kStripX;
  // index of (x, y0 - 1 + r) in plane p, advanced plane by plane
  int idx[kStripH];
  int p = it.z0 - 1;
  {
    const int W = w - p;
    const int pb = int(tetSize(w) - tetSize(W));
#pragma unroll
    for (int r = 0; r < kStripH; ++r) idx[r] = pb + rowStart(W, y0 - 1 + r) + x;
  }
  // plane p exists at row y iff x + y <= N - p
  auto load = [&](T (&v)[kStripH]) {
#pragma unroll
    for (int r = 0; r < kStripH; ++r) v[r] = (x + y0 - 1 + r <= N - p) ? __ldg(u + idx[r]) : T(0);
  };
  auto loadF = [&](T (&v)[kStripR]) {
#pragma unroll
    for (int r = 0; r < kStripR; ++r) v[r] = (x + y0 + r <= N - p) ? __ldg(f + idx[r + 1]) : T(0);
  };
  auto advance = [&]() {
    const int t = triSize(w - p);
#pragma unroll
    for (int r = 0; r < kStripH; ++r) idx[r] += t - (y0 - 1 + r);
    ++p;
  };
  T pm[kStripH], pc[kStripH], pp[kStripH], nx[kStripH], fc[kStripR], fn[kStripR];
  load(pm);
  advance();
  load(pc);
  if (kSecond) loadF(fc);
  int idxc[kStripR];  // indices of the computed rows of plane z
#pragma unroll
  for (int r = 0; r < kStripR; ++r) idxc[r] = idx[r + 1];
  advance();
  load(pp);
  for (int z = it.z0; z < zEnd; ++z) {
    // p == z + 1 here: the second vector of plane z + 1, then plane z + 2 of the input
    if (kSecond) loadF(fn);
    int idxn[kStripR];
#pragma unroll
    for (int r = 0; r < kStripR; ++r) idxn[r] = idx[r + 1];
    advance();
    load(nx);
#pragma unroll
    for (int r = 0; r < kStripR; ++r) {
      const int j = r + 1, y = y0 + r;
      // shuffles are warp-uniform: every lane takes part, inactive lanes discard the result
      const T E = shDown(pc[j]), Wv = shUp(pc[j]);
      const T NW = shUp(pc[j + 1]), SE = shDown(pc[j - 1]);
      const T TW = shUp(pp[j]), TSE = shDown(pp[j - 1]);
      const T BE = shDown(pm[j]), BNW = shUp(pm[j + 1]);
      if (computeLane && x + y + z <= N - 1) {
        // four independent partial sums keep the FMA dependency chains short
        T s0 = wt[1] * E, s1 = wt[3] * pc[j + 1], s2 = wt[7] * pp[j], s3 = wt[11] * pm[j];
        s0 += wt[2] * Wv;
        s1 += wt[4] * pc[j - 1];
        s2 += wt[8] * TW;
        s3 += wt[12] * BE;
        s0 += wt[5] * NW;
        s1 += wt[6] * SE;
        s2 += wt[9] * pp[j - 1];
        s3 += wt[13] * pm[j + 1];
        s2 += wt[10] * TSE;
        s3 += wt[14] * BNW;
        const T a = wt[0] * pc[j] + ((s0 + s1) + (s2 + s3));
        T* d = dst + base + idxc[r];
        if (OP == STRIP_REPLACE) *d = a;
        else if (OP == STRIP_ADD) *d = fc[r] + a;
        else *d = fc[r] - a;
      }
    }
#pragma unroll
    for (int r = 0; r < kStripH; ++r) {
      pm[r] = pc[r];
      pc[r] = pp[r];
      pp[r] = nx[r];
    }
#pragma unroll
    for (int r = 0; r < kStripR; ++r) {
      idxc[r] = idxn[r];
      if (kSecond) fc[r] = fn[r];
    }
  }
}

// Full-weighting restriction at coarse cell-interior points: coarse = fine[2p] + 1/2 sum fine[2p+d]
// (restrict_3D_macrocell_P1_pull_additive.cpp; on interior points every weight is 1 or 1/2).
template <class T>
__global__ void __launch_bounds__(kBlock) cellRestrictKernel(LevelDev lc, LevelDev lf, T* __restrict__ coarse,
                                                             const T* __restrict__ fine, unsigned mask) {
  const int nPl = lc.N - 3;
  const int c = blockIdx.x / nPl, z = 1 + blockIdx.x % nPl;
  if (!(lc.cellType[c] & mask)) return;
  const T* __restrict__ uf = fine + lf.cellOff[c];
  T* __restrict__ uc = coarse + lc.cellOff[c];
  const T one[15] = {T(1), T(1), T(1), T(1), T(1), T(1), T(1), T(1), T(1), T(1), T(1), T(1), T(1), T(1), T(1)};
  const int W = lc.w - z;
  auto ld = [uf](int i) { return __ldg(uf + i); };
  for (int y = 1 + (int)(threadIdx.x >> 5); y <= W - 3; y += kBlock / 32) {
    const CellRow rf = cellRow(lf.w, 2 * z, 2 * y);
    const int rc = int(tetSize(lc.w) - tetSize(W)) + rowStart(W, y);
    const int len = W - 2 - y;
    for (int x = 1 + (int)(threadIdx.x & 31); x <= len; x += 32)
      uc[rc + x] = ld(rf.r0 + 2 * x) + T(0.5) * cellOffDiag(one, rf, 2 * x, ld);
  }
}

__device__ __forceinline__ int cellIndexDev(int w, int x, int y, int z) {
  const int W = w - z;
  return int(tetSize(w) - tetSize(W)) + rowStart(W, y) + x;
}

// Linear prolongation at fine cell-interior points (prolongate_3D_macrocell_P1_push_additive.cpp):
// even points copy the coarse value, every other point is the mean of the two coarse end
// points of the coarse micro-edge it bisects. The bisected direction depends on the parity of
// (x, y, z); for one fine row only the x parity varies, so two row pairs are set up per row.
template <class T, bool ADD>
__global__ void __launch_bounds__(kBlock) cellProlongKernel(LevelDev lf, LevelDev lc, T* __restrict__ fine,
                                                            const T* __restrict__ coarse, unsigned mask) {
  const int nPl = lf.N - 3;
  const int c = blockIdx.x / nPl, z = 1 + blockIdx.x % nPl;
  if (!(lf.cellType[c] & mask)) return;
  T* __restrict__ uf = fine + lf.cellOff[c];
  const T* __restrict__ uc = coarse + lc.cellOff[c];
  const int W = lf.w - z;
  // directions of the bisected coarse micro-edge by parity code (x | y << 1 | z << 2)
  const int DX[8] = {0, 1, 0, -1, 0, -1, 0, -1};
  const int DY[8] = {0, 0, 1, 1, 0, 0, -1, 1};
  const int DZ[8] = {0, 0, 0, 0, 1, 1, 1, -1};
  for (int y = 1 + (int)(threadIdx.x >> 5); y <= W - 3; y += kBlock / 32) {
    const int rf = int(tetSize(lf.w) - tetSize(W)) + rowStart(W, y);
    const int len = W - 2 - y;
    // for x parity p: coarse row base of end point a (x offset (x - dx) / 2) and of b = a + d
    int ra[2], rb[2], dxp[2];
    bool single[2];
    for (int p = 0; p < 2; ++p) {
      const int code = p | ((y & 1) << 1) | ((z & 1) << 2);
      const int dx = DX[code], dy = DY[code], dz = DZ[code];
      const int ay = (y - dy) >> 1, az = (z - dz) >> 1;
      ra[p] = cellIndexDev(lc.w, 0, ay, az);
      rb[p] = cellIndexDev(lc.w, 0, ay + dy, az + dz);
      dxp[p] = dx;
      single[p] = code == 0;
    }
    for (int x = 1 + (int)(threadIdx.x & 31); x <= len; x += 32) {
      const int p = x & 1;
      const int ax = (x - dxp[p]) >> 1;
      const T v = single[p] ? __ldg(uc + ra[p] + ax)
                            : T(0.5) * (__ldg(uc + ra[p] + ax) + __ldg(uc + rb[p] + ax + dxp[p]));
      if (ADD) uf[rf + x] += v;
      else uf[rf + x] = v;
    }
  }
}

// ---------------------------------------------------------------------------------------
// Face interiors: generic entries (layer, dx, dy, w); layer 0 is the face triangle, layer
// 1+n the ghost layer of neighbour cell n (apply_3D_macroface_one_sided_*.cpp, called once
// per neighbour cell in P1ConstantOperator.cpp:202-288, fused here into one sweep).
// One block per (face, band of kFaceRows rows); for each row a warp turns the entries into
// slot offsets once (shared memory), then every lane adds x.
// ---------------------------------------------------------------------------------------
constexpr int kFaceRows = 32;

__device__ __forceinline__ int faceSlot(int w, int layer, int x, int y) {
  if (layer == 0) return rowStart(w, y) + x;
  return triSize(w) + (layer - 1) * triSize(w - 1) + rowStart(w - 1, y) + x;
}

template <class T>
struct FaceShared {
  FaceEnt<T> ent[16];
  int off[kBlock / 32][16];
};

template <class T>
__device__ __forceinline__ int loadFaceEntries(FaceShared<T>& sh, const StencilDev<T>& st, int face) {
  const int ne = st.faceEntCount[face];
  if (threadIdx.x < ne) sh.ent[threadIdx.x] = st.faceEnt[16 * face + threadIdx.x];
  __syncthreads();
  return ne;
}

template <class T, int MODE>
__global__ void __launch_bounds__(kBlock) faceStencilKernel(LevelDev lv, StencilDev<T> st, T* __restrict__ dst,
                                                            const T* __restrict__ src, const T* __restrict__ rhs,
                                                            unsigned mask) {
  const FaceBlock b = lv.faceBlocks[blockIdx.x];
  if (!(lv.faceType[b.face] & mask)) return;
  __shared__ FaceShared<T> sh;
  const int ne = loadFaceEntries(sh, st, b.face);
  const int w = lv.w, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t base = lv.faceOff[b.face];
  const T* __restrict__ u = src + base;
  const int yEnd = min(b.start + kFaceRows, w - 2);
  for (int y = b.start + warp; y < yEnd; y += kBlock / 32) {
    if (lane < ne) sh.off[warp][lane] = faceSlot(w, sh.ent[lane].layer, sh.ent[lane].dx, y + sh.ent[lane].dy);
    __syncwarp();
    const int len = w - 2 - y, r0 = rowStart(w, y);
    for (int x = 1 + lane; x <= len; x += 32) {
      T s = T(0);
      for (int k = 0; k < ne; ++k) s += sh.ent[k].w * __ldg(u + sh.off[warp][k] + x);
      const int64_t i = base + r0 + x;
      if (MODE == MODE_REPLACE) dst[i] = s;
      else if (MODE == MODE_ADD) dst[i] += s;
      else dst[i] = rhs[i] - s;
    }
    __syncwarp();
  }
}

// Face SOR, colour = (x + 2y) mod 3; entry 0 is the diagonal.
template <class T>
__global__ void __launch_bounds__(kBlock) faceSorKernel(LevelDev lv, StencilDev<T> st, T* u, const T* __restrict__ rhs,
                                                        unsigned mask, int colour, T omega) {
  const FaceBlock b = lv.faceBlocks[blockIdx.x];
  if (!(lv.faceType[b.face] & mask)) return;
  __shared__ FaceShared<T> sh;
  const int ne = loadFaceEntries(sh, st, b.face);
  const int w = lv.w, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t base = lv.faceOff[b.face];
  T* uf = u + base;
  const T* __restrict__ f = rhs + base;
  const T om = omega, om1 = T(1) - omega;
  const int yEnd = min(b.start + kFaceRows, w - 2);
  for (int y = b.start + warp; y < yEnd; y += kBlock / 32) {
    if (lane < ne) sh.off[warp][lane] = faceSlot(w, sh.ent[lane].layer, sh.ent[lane].dx, y + sh.ent[lane].dy);
    __syncwarp();
    const int len = w - 2 - y, r0 = rowStart(w, y);
    const int x0 = 1 + (((colour - 2 * y - 1) % 3) + 3) % 3;
    for (int x = x0 + 3 * lane; x <= len; x += 96) {
      T s = f[r0 + x];
      for (int k = 1; k < ne; ++k) s -= sh.ent[k].w * uf[sh.off[warp][k] + x];
      uf[r0 + x] = om1 * uf[r0 + x] + (s * om) / sh.ent[0].w;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------------------
// SOR phases in one launch each: a block per primitive refreshes the copies of its own array
// that the reference refreshes before the phase (its entries range[p] = [begin, end) of the halo
// table; their owners are not changed by the phase, so no block reads what another writes), then
// runs every colour of the phase with a block barrier between colours. Primitives of one kind
// are independent within their phase (each reads only its own array), so this equals one launch
// per colour over all primitives.
// ---------------------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void gatherRange(T* buf, T* cells, const uint2* __restrict__ table, int begin, int end,
                                            int64_t cellEnd) {
  for (int i = begin + (int)threadIdx.x; i < end; i += (int)blockDim.x) {
    const uint2 t = table[i];
    if (cells) {  // cell arrays in their colour-split copy: slots below cellEnd live there
      const T v = t.y < cellEnd ? cells[t.y] : buf[t.y];
      if (t.x < cellEnd) cells[t.x] = v;
      else buf[t.x] = v;
    } else {
      buf[t.x] = buf[t.y];
    }
  }
}

// Edges (both colours x mod 2) or vertices: block b is primitive firstPrim + b.
template <class T>
__global__ void __launch_bounds__(kBlock) lowSorPhaseKernel(LevelDev lv, StencilDev<T> st, T* u, const T* __restrict__ rhs,
                                                            unsigned mask, T omega, int firstPrim, int backwards,
                                                            const uint2* __restrict__ table, const int2* __restrict__ range,
                                                            T* cells, int64_t cellEnd) {
  const int p = firstPrim + blockIdx.x;
  if (range) {
    gatherRange(u, cells, table, range[p].x, range[p].y, cellEnd);
    __syncthreads();
  }
  if (!(lv.lowType[p] & mask)) return;
  const int first = lv.lowFirst[p], count = lv.lowCount[p];
  const int64_t o = lv.lowOff[p];
  const int e0 = st.lowEntOff[p], e1 = st.lowEntOff[p + 1];
  const int passes = p < lv.nEdges ? 2 : 1;
  const T om1 = T(1) - omega;
  for (int pass = 0; pass < passes; ++pass) {
    const int colour = passes == 2 ? (backwards ? 1 - pass : pass) : -1;
    for (int x = first + threadIdx.x; x < first + count; x += kBlock) {
      if (colour >= 0 && (x & 1) != colour) continue;
      const int64_t c = o + x;
      T s = rhs[c];
      for (int k = e0 + 1; k < e1; ++k) s -= st.lowEntW[k] * u[c + st.lowEntRel[k]];
      u[c] = om1 * u[c] + (s * omega) / st.lowEntW[e0];
    }
    __syncthreads();
  }
}

// Faces, the three colours (x + 2y) mod 3; block b is face b, kFacePhaseThreads threads (the
// warps take the rows).
constexpr int kFacePhaseThreads = 1024;
template <class T>
__global__ void __launch_bounds__(kFacePhaseThreads) faceSorPhaseKernel(LevelDev lv, StencilDev<T> st, T* u,
                                                                        const T* __restrict__ rhs, unsigned mask, T omega,
                                                                        int backwards, const uint2* __restrict__ table,
                                                                        const int2* __restrict__ range, T* cells,
                                                                        int64_t cellEnd) {
  constexpr int kWarps = kFacePhaseThreads / 32;
  const int face = blockIdx.x;
  if (range) {
    gatherRange(u, cells, table, range[face].x, range[face].y, cellEnd);
    __syncthreads();
  }
  if (!(lv.faceType[face] & mask)) return;
  __shared__ FaceEnt<T> ent[16];
  __shared__ int off[kWarps][16];
  const int ne = st.faceEntCount[face];
  if (threadIdx.x < ne) ent[threadIdx.x] = st.faceEnt[16 * face + threadIdx.x];
  __syncthreads();
  const int w = lv.w, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t base = lv.faceOff[face];
  T* uf = u + base;
  const T* __restrict__ f = rhs + base;
  const T om = omega, om1 = T(1) - omega;
  for (int pass = 0; pass < 3; ++pass) {
    const int colour = backwards ? 2 - pass : pass;
    for (int y = 1 + warp; y < w - 2; y += kWarps) {
      if (lane < ne) off[warp][lane] = faceSlot(w, ent[lane].layer, ent[lane].dx, y + ent[lane].dy);
      __syncwarp();
      const int len = w - 2 - y, r0 = rowStart(w, y);
      const int x0 = 1 + (((colour - 2 * y - 1) % 3) + 3) % 3;
      for (int x = x0 + 3 * lane; x <= len; x += 96) {
        T s = f[r0 + x];
        for (int k = 1; k < ne; ++k) s -= ent[k].w * uf[off[warp][k] + x];
        uf[r0 + x] = om1 * uf[r0 + x] + (s * om) / ent[0].w;
      }
      __syncwarp();
    }
    __syncthreads();
  }
}

// Restriction at coarse face-interior points from the fine face and its ghost layers: the fine
// stencil structure of the face with weight 1 at the centre and 1/2 at every neighbour.
template <class T>
__global__ void __launch_bounds__(kBlock) faceRestrictKernel(LevelDev lc, LevelDev lf, StencilDev<T> stf,
                                                             T* __restrict__ coarse, const T* __restrict__ fine,
                                                             unsigned mask) {
  const FaceBlock b = lc.faceBlocks[blockIdx.x];
  if (!(lc.faceType[b.face] & mask)) return;
  __shared__ FaceShared<T> sh;
  const int ne = loadFaceEntries(sh, stf, b.face);
  const int w = lc.w, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const T* __restrict__ uf = fine + lf.faceOff[b.face];
  T* __restrict__ uc = coarse + lc.faceOff[b.face];
  const int yEnd = min(b.start + kFaceRows, w - 2);
  for (int y = b.start + warp; y < yEnd; y += kBlock / 32) {
    if (lane < ne) sh.off[warp][lane] = faceSlot(lf.w, sh.ent[lane].layer, sh.ent[lane].dx, 2 * y + sh.ent[lane].dy);
    __syncwarp();
    const int len = w - 2 - y, r0 = rowStart(w, y);
    for (int x = 1 + lane; x <= len; x += 32) {
      T s = T(0);
      for (int k = 1; k < ne; ++k) s += __ldg(uf + sh.off[warp][k] + 2 * x);
      uc[r0 + x] = __ldg(uf + sh.off[warp][0] + 2 * x) + T(0.5) * s;
    }
    __syncwarp();
  }
}

template <class T, bool ADD>
__global__ void __launch_bounds__(kBlock) faceProlongKernel(LevelDev lf, LevelDev lc, T* __restrict__ fine,
                                                            const T* __restrict__ coarse, unsigned mask) {
  const FaceBlock b = lf.faceBlocks[blockIdx.x];
  if (!(lf.faceType[b.face] & mask)) return;
  const int w = lf.w, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* __restrict__ uf = fine + lf.faceOff[b.face];
  const T* __restrict__ uc = coarse + lc.faceOff[b.face];
  const int yEnd = min(b.start + kFaceRows, w - 2);
  for (int y = b.start + warp; y < yEnd; y += kBlock / 32) {
    const int len = w - 2 - y, r0 = rowStart(w, y);
    // bisected coarse micro-edge by parity (x | y << 1): (1,0), (0,1) or (-1,1)
    int ra[2], rb[2], dxp[2];
    for (int p = 0; p < 2; ++p) {
      const int code = p | ((y & 1) << 1);
      const int dx = code == 1 ? 1 : (code == 3 ? -1 : 0), dy = (code >= 2) ? 1 : 0;
      const int ay = (y - dy) >> 1;
      ra[p] = rowStart(lc.w, ay);
      rb[p] = rowStart(lc.w, ay + dy);
      dxp[p] = dx;
    }
    const bool evenRow = (y & 1) == 0;
    for (int x = 1 + lane; x <= len; x += 32) {
      const int p = x & 1;
      const int ax = (x - dxp[p]) >> 1;
      const T v = (evenRow && p == 0) ? __ldg(uc + ra[0] + ax)
                                      : T(0.5) * (__ldg(uc + ra[p] + ax) + __ldg(uc + rb[p] + ax + dxp[p]));
      if (ADD) uf[r0 + x] += v;
      else uf[r0 + x] = v;
    }
  }
}

// ---------------------------------------------------------------------------------------
// Edges and vertices (apply_edge P1Operator.hpp:1040-1104, macrovertex::apply
// VertexDoFMacroVertex.hpp:160-184): per primitive a list of (relative slot, weight).
// ---------------------------------------------------------------------------------------
template <class T, int MODE>
__global__ void __launch_bounds__(kBlock) lowStencilKernel(LevelDev lv, StencilDev<T> st, T* __restrict__ dst,
                                                           const T* __restrict__ src, const T* __restrict__ rhs,
                                                           unsigned mask, int blockBegin) {
  const LowBlock b = lv.lowBlocks[blockBegin + blockIdx.x];
  if (!(lv.lowType[b.prim] & mask)) return;
  const int x = b.start + threadIdx.x;
  if (x >= lv.lowFirst[b.prim] + lv.lowCount[b.prim]) return;
  const int64_t c = lv.lowOff[b.prim] + x;
  T s = T(0);
  for (int k = st.lowEntOff[b.prim]; k < st.lowEntOff[b.prim + 1]; ++k) s += st.lowEntW[k] * __ldg(src + c + st.lowEntRel[k]);
  if (MODE == MODE_REPLACE) dst[c] = s;
  else if (MODE == MODE_ADD) dst[c] += s;
  else dst[c] = rhs[c] - s;
}

// ---------------------------------------------------------------------------------------
// Coarse-grid CG (CGSolver.hpp:69-150 with the identity preconditioner) for a level whose DoFs
// all sit on vertices and edges (levels 0 and 1), one block per group of unknowns: the whole
// mesh, or one copy of a storage of disjoint copies (the copies' systems are not coupled, so
// each copy iterates and stops on its own, exactly as a single mesh of it does). The halo
// refresh, stencil, dot products and updates of every iteration run on the device, so a
// multigrid cycle needs no host synchronisation. Vector updates touch the group's owned DoFs
// (a flat list, thread t takes every blockDim-th); the copies of the source of every apply, and
// of x at the end, are refreshed from their owners. r, p and ap are workspace level buffers;
// info (optional): per group [iterations, final residual norm].
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double blockSum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    red[32] = t;
  }
  __syncthreads();
  return red[32];
}

// One owned DoF of the coarse CG: its slot and the stencil entries [e0, e1) of its primitive.
struct CoarseDof {
  int64_t slot;
  int e0, e1;
};

static __global__ void __launch_bounds__(kBlock) coarseCgKernel(StencilDev<double> st, const CoarseDof* __restrict__ dofs,
                                                        const int* __restrict__ dofOff, const uint2* __restrict__ comm,
                                                        const int* __restrict__ commOff, double* x,
                                                        const double* __restrict__ b, double* r, double* p, double* ap,
                                                        int maxIter, double tol, double* info) {
  __shared__ double red[33];
  const int tid = threadIdx.x, g = blockIdx.x;
  const int d0 = dofOff[g], d1 = dofOff[g + 1], c0 = commOff[g], c1 = commOff[g + 1];
  auto refresh = [&](double* v) {
    __syncthreads();
    for (int i = c0 + tid; i < c1; i += blockDim.x) {
      const uint2 t = comm[i];
      v[t.x] = v[t.y];
    }
    __syncthreads();
  };
  auto forOwned = [&](auto f) {
    for (int i = d0 + tid; i < d1; i += blockDim.x) f(dofs[i]);
  };
  auto apply = [&](double* dst, double* src) {  // dst = A src on the group's DoFs
    refresh(src);
    forOwned([&](const CoarseDof& d) {
      double s = 0;
      for (int k = d.e0; k < d.e1; ++k) s += st.lowEntW[k] * src[d.slot + st.lowEntRel[k]];
      dst[d.slot] = s;
    });
    __syncthreads();
  };
  auto dot = [&](const double* u, const double* v) {
    double s = 0;
    forOwned([&](const CoarseDof& d) { s += u[d.slot] * v[d.slot]; });
    return blockSum(s, red);
  };
  // r = b - A x; p = z = r (identity preconditioner)
  apply(p, x);
  forOwned([&](const CoarseDof& d) {
    r[d.slot] = b[d.slot] - p[d.slot];
    p[d.slot] = r[d.slot];
  });
  __syncthreads();
  double prsold = dot(r, r);
  double res = sqrt(prsold);
  int it = 0;
  if (res >= tol) {
    for (int i = 0; i < maxIter; ++i) {
      it = i + 1;
      apply(ap, p);
      const double alpha = prsold / dot(p, ap);
      forOwned([&](const CoarseDof& d) {
        x[d.slot] += alpha * p[d.slot];
        r[d.slot] -= alpha * ap[d.slot];
      });
      __syncthreads();
      const double rsnew = dot(r, r);
      res = sqrt(rsnew);
      if (res < tol) break;
      const double beta = rsnew / prsold;
      forOwned([&](const CoarseDof& d) { p[d.slot] = r[d.slot] + beta * p[d.slot]; });
      __syncthreads();
      prsold = rsnew;
    }
  }
  refresh(x);
  if (tid == 0 && info) {
    info[2 * g] = it;
    info[2 * g + 1] = res;
  }
}

// ---------------------------------------------------------------------------------------
// P2 operator of level L on the vertex-DoF lattice of level L + 1 (size M = 2N per edge).
// Node (X, Y, Z) of a macro-cell is local node j of the level-L micro-cell (t, a) exactly when
// (X, Y, Z) = 2a + off[t][j]; its parity class (X, Y, Z mod 2) fixes the candidates (t, j).
// A thread owns one node of the closed macro-cell and sums, over the candidate micro-cells that
// lie inside the cell, row j of that micro-cell's 10 x 10 element matrix times the ten nodal
// values (gather form of the element-by-element product; deterministic). Interior nodes get
// their final value; nodes on the cell's faces, edges and vertices get this cell's share in the
// cell's closure slots, which p2AddKernel sums into the owning primitive.
// ---------------------------------------------------------------------------------------
struct P2Tables {
  signed char off[6][10][3];   // lattice offset of local node j of micro-cell type t from 2a
  unsigned char nCand[8];      // candidates per parity class
  unsigned char cand[8][24][2];  // (t, j)
  unsigned char widthRed[6];   // micro-cells of type t: a_x + a_y + a_z < N - widthRed[t]
};

constexpr int MODE_DIAG = 3;  // P2: sum of the element diagonals (the matrix diagonal)
constexpr int MODE_SOR = 4;   // P2 interior: x += omega (b - A x) / a_ii in place, one colour

// Row j of A at node (X, Y, Z) of a macro-cell restricted to that cell: the sum over the level-L
// micro-cells inside the cell holding the node as local node j (DIAG: of their diagonals only).
// u is the cell's array, pbz the first index of the planes Z-2 .. Z+2.
template <class T, bool DIAG>
__device__ __forceinline__ T p2GatherNode(const P2Tables& tb, const T* Kc, const T* __restrict__ u, const int (&pbz)[5],
                                          int w, int N, int X, int Y, int Z) {
  const int pc = (X & 1) | ((Y & 1) << 1) | ((Z & 1) << 2);
  T s = T(0);
  for (int k = 0; k < tb.nCand[pc]; ++k) {
    const int t = tb.cand[pc][k][0], j = tb.cand[pc][k][1];
    const int ax = (X - tb.off[t][j][0]) >> 1, ay = (Y - tb.off[t][j][1]) >> 1, az = (Z - tb.off[t][j][2]) >> 1;
    if (ax < 0 || ay < 0 || az < 0 || ax + ay + az >= N - tb.widthRed[t]) continue;
    const T* Kr = Kc + t * 100 + j * 10;
    if (DIAG) {
      s += Kr[j];
      continue;
    }
#pragma unroll
    for (int m = 0; m < 10; ++m) {
      const int qx = 2 * ax + tb.off[t][m][0], qy = 2 * ay + tb.off[t][m][1], qz = 2 * az + tb.off[t][m][2];
      s += Kr[m] * __ldg(u + pbz[qz - Z + 2] + rowStart(w - qz, qy) + qx);
    }
  }
  return s;
}

// colour, sel: when sel >= 0 only nodes whose colour (low 7 bits of the per-slot colour byte)
// is sel are computed (one pass of the multicolour SOR); bit 7 of the byte marks owned slots.
template <class T, int MODE>
__global__ void __launch_bounds__(kBlock) p2CellKernel(LevelDev lv, P2Tables tb, const T* __restrict__ K,
                                                       T* __restrict__ dst, const T* __restrict__ src,
                                                       const T* __restrict__ rhs, unsigned mask,
                                                       const unsigned char* __restrict__ colour, int sel) {
  const int M = lv.N, N = M / 2, nPl = M + 1, w = lv.w;
  const int c = blockIdx.x / nPl, Z = blockIdx.x % nPl;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t base = lv.cellOff[c];
  const bool cellOn = (lv.cellType[c] & mask) != 0;
  const T* Kc = K + (int64_t)c * 600;
  // first index of the planes Z-2 .. Z+2 (the ones a micro-cell around a node of plane Z reaches)
  int pbz[5];
#pragma unroll
  for (int d = 0; d < 5; ++d) {
    const int z = Z - 2 + d;
    pbz[d] = (z >= 0 && z <= M) ? int(tetSize(w) - tetSize(w - z)) : 0;
  }
  const int pb = pbz[2];
  for (int Y = warp; Y <= M - Z; Y += kBlock / 32) {
    const int r0 = pb + rowStart(w - Z, Y);
    for (int X = lane; X <= M - Z - Y; X += 32) {
      const int64_t i = base + r0 + X;
      if (sel >= 0 && (colour[i] & 0x7f) != sel) continue;
      const T s = p2GatherNode<T, MODE == MODE_DIAG>(tb, Kc, src + base, pbz, w, N, X, Y, Z);
      const bool interior = X >= 1 && Y >= 1 && Z >= 1 && X + Y + Z <= M - 1;
      if (!interior) dst[i] = s;
      else if (cellOn) dst[i] = MODE == MODE_RESIDUAL ? rhs[i] - s : s;
    }
  }
}

// ---------------------------------------------------------------------------------------
// P2 interior nodes by constant stencils. An interior node of a macro-cell (X, Y, Z >= 1,
// X + Y + Z <= M - 1 on lattice M = 2^(L+1)) couples only to nodes of the micro-cells inside the
// cell, in the same pattern for every node of its parity class, so its row of A is a constant
// stencil per (cell, class): the offsets are compile-time lists (p2_stencil.h), the weights a
// per-cell table W[cell][p2s::kTotal] assembled on the host from the element matrices. A block
// works on one (cell, plane Z); each warp takes whole rows, its lanes every second node of the
// row, so all lanes of a warp run the same class.
// ---------------------------------------------------------------------------------------
template <int DY, int DZ>
__device__ __forceinline__ int p2RowBase(const int (&pbz)[5], int w, int Y, int Z) {
  return pbz[DZ + 2] + rowStart(w - Z - DZ, Y + DY);
}

// The loads go through the read-only path also in the in-place SOR pass: no thread reads a value
// that another thread writes during the launch (a colour class couples to no node of its own
// colour), and each thread reads its own node before writing it.
// Four partial sums (entry I into sum I mod 4) keep the FMA dependency chains short.
template <class T, int... DX, int... DY, int... DZ, int... I>
__device__ __forceinline__ T p2StencilDot(p2s::List<p2s::O<DX, DY, DZ>...>, std::integer_sequence<int, I...>,
                                          const T* u, const T* wt, const int (&pbz)[5], int w, int X, int Y, int Z) {
  T s[4] = {T(0), T(0), T(0), T(0)};
  ((s[I & 3] += wt[I] * __ldg(u + p2RowBase<DY, DZ>(pbz, w, Y, Z) + X + DX)), ...);
  return (s[0] + s[1]) + (s[2] + s[3]);
}

// One row (Y, Z) of class PC: MODE_REPLACE dst = A src, MODE_RESIDUAL dst = rhs - A src,
// MODE_SOR dst (== src) += omega (rhs - A dst) / a_ii. With sel >= 0 only the nodes of colour sel
// are computed: the vertex class is split into four colours, read from the colour bytes; a whole
// edge class is one colour in a cell's frame.
template <class T, int MODE, int PC>
__device__ __forceinline__ void p2StencilRow(const T* wts, T* dst, const T* src, const T* rhs, int64_t base,
                                             const int (&pbz)[5], int w, int M, int Y, int Z, int lane,
                                             const unsigned char* __restrict__ colour, int sel, T omega, int vstep) {
  using S = typename p2s::Class<PC>::type;
  constexpr int kFirst = p2s::kFirst[PC], kCentre = p2s::kCentre[PC], kLen = p2s::kLen[PC];
  const T* wt = wts + kFirst;
  const int r0 = pbz[2] + rowStart(w - Z, Y);
  int X0 = ((PC & 1) ? 1 : 2) + 2 * lane, dX = 64;
  if (PC == 0 && sel >= 0) {
    // vertex colour sel along the row: the colour of the vertex node 2 + 2t is c(2) + vstep t mod 4,
    // so the lanes take every fourth (vstep odd) or every second (vstep 2) vertex node from the first
    if (M - 1 - Y - Z < 2) return;
    const int diff = (sel - (colour[base + r0 + 2] & 0x7f)) & 3;
    int t0, ts;
    if (vstep & 1) {
      t0 = (diff * vstep) & 3;
      ts = 4;
    } else {
      if (diff & 1) return;
      t0 = (diff >> 1) & 1;
      ts = 2;
    }
    X0 = 2 + 2 * t0 + 2 * ts * lane;
    dX = 64 * ts;
  }
#pragma unroll 1
  for (int X = X0; X <= M - 1 - Y - Z; X += dX) {
    const int64_t i = base + r0 + X;
    if (PC == 0 && sel >= 0 && (colour[i] & 0x7f) != sel) continue;
    const T s = p2StencilDot<T>(S{}, std::make_integer_sequence<int, kLen>{}, src + base, wt, pbz, w, X, Y, Z);
    if (MODE == MODE_REPLACE)
      dst[i] = s;
    else if (MODE == MODE_RESIDUAL)
      dst[i] = rhs[i] - s;
    else
      dst[i] += omega * (rhs[i] - s) / wt[kCentre];
  }
}

template <class T, int MODE>
__device__ __forceinline__ void p2StencilRowAny(int pc, const T* wts, T* dst, const T* src, const T* rhs, int64_t base,
                                                const int (&pbz)[5], int w, int M, int Y, int Z, int lane,
                                                const unsigned char* __restrict__ colour, int sel, T omega,
                                                int vstep) {
  switch (pc) {
    case 0: p2StencilRow<T, MODE, 0>(wts, dst, src, rhs, base, pbz, w, M, Y, Z, lane, colour, sel, omega, vstep); break;
    case 1: p2StencilRow<T, MODE, 1>(wts, dst, src, rhs, base, pbz, w, M, Y, Z, lane, colour, sel, omega, vstep); break;
    case 2: p2StencilRow<T, MODE, 2>(wts, dst, src, rhs, base, pbz, w, M, Y, Z, lane, colour, sel, omega, vstep); break;
    case 3: p2StencilRow<T, MODE, 3>(wts, dst, src, rhs, base, pbz, w, M, Y, Z, lane, colour, sel, omega, vstep); break;
    case 4: p2StencilRow<T, MODE, 4>(wts, dst, src, rhs, base, pbz, w, M, Y, Z, lane, colour, sel, omega, vstep); break;
    case 5: p2StencilRow<T, MODE, 5>(wts, dst, src, rhs, base, pbz, w, M, Y, Z, lane, colour, sel, omega, vstep); break;
    case 6: p2StencilRow<T, MODE, 6>(wts, dst, src, rhs, base, pbz, w, M, Y, Z, lane, colour, sel, omega, vstep); break;
    default: p2StencilRow<T, MODE, 7>(wts, dst, src, rhs, base, pbz, w, M, Y, Z, lane, colour, sel, omega, vstep); break;
  }
}

// Grid: nCells * (M - 3) blocks, block b on cell b / (M - 3), plane Z = 1 + b % (M - 3) (the
// planes holding interior nodes; needs M >= 4). Only cells of a flagged DoF type are written.
// sel >= 0 (one colour pass of the SOR, MODE_SOR or MODE_REPLACE): classOfColour[cell * 12 + sel]
// is the class of colour sel in the cell's frame (0 for the four vertex colours, -1 when no
// interior node has the colour), classOfColour[cell * 12 + 11] the change of the vertex colour
// from one vertex node of a row to the next (1, 2 or 3). MODE_SOR updates in place: dst == src,
// rhs = b.
template <class T, int MODE>
__global__ void __launch_bounds__(kBlock, 2) p2StencilKernel(LevelDev lv, const T* __restrict__ W, T* dst, const T* src,
                                                          const T* __restrict__ rhs, unsigned mask,
                                                          const unsigned char* __restrict__ colour,
                                                          const signed char* __restrict__ classOfColour, int sel,
                                                          T omega) {
  const int M = lv.N, w = lv.w, nPl = M - 3;
  const int c = blockIdx.x / nPl, Z = 1 + blockIdx.x % nPl;
  if (!(lv.cellType[c] & mask)) return;
  int pcSel = 0, vstep = 1;
  if (sel >= 0) {
    pcSel = classOfColour[c * 12 + sel];
    vstep = classOfColour[c * 12 + 11];
    if (pcSel < 0 || ((pcSel >> 2) & 1) != (Z & 1)) return;
  }
  __shared__ T wts[p2s::kTotal];
  for (int k = threadIdx.x; k < p2s::kTotal; k += blockDim.x) wts[k] = W[(int64_t)c * p2s::kTotal + k];
  __syncthreads();
  int pbz[5];
#pragma unroll
  for (int d = 0; d < 5; ++d) {
    const int z = Z - 2 + d;
    pbz[d] = (z >= 0 && z <= M) ? int(tetSize(w) - tetSize(w - z)) : 0;
  }
  const int64_t base = lv.cellOff[c];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (sel >= 0) {
#pragma unroll 1
    for (int Y = (((pcSel >> 1) & 1) ? 1 : 2) + 2 * warp; Y <= M - 2 - Z; Y += 2 * (kBlock / 32))
      p2StencilRowAny<T, MODE>(pcSel, wts, dst, src, rhs, base, pbz, w, M, Y, Z, lane, colour, sel, omega, vstep);
  } else {
#pragma unroll 1
    for (int Y = 1 + warp; Y <= M - 2 - Z; Y += kBlock / 32) {
#pragma unroll 1
      for (int px = 0; px < 2; ++px)
        p2StencilRowAny<T, MODE>(px | ((Y & 1) << 1) | ((Z & 1) << 2), wts, dst, src, rhs, base, pbz, w, M, Y, Z, lane,
                                 colour, sel, omega, vstep);
    }
  }
}

// The closure nodes of every macro-cell (its faces, edges and vertices): this cell's share of
// row j of A, written into the cell's closure slot (p2AddKernel sums the shares into the owner).
// A node inside one face of the cell sees the same micro-cells at every node of its (face, class):
// its share is a constant stencil (p2s::FaceList, weights FW[cell][p2s::kFaceTotal]). Nodes on the
// cell's edges and vertices take the element gather. Grid: nCells * (M + p2FaceChunks(M)) blocks.
// Per cell, M blocks take the planes Z = 1 .. M: on each, warps 0-5 walk the lines of faces
// Y = 0, X = 0 and X + Y + Z = M (one warp per line and parity, so a warp runs one class), warp 6
// the three edge nodes of the plane. p2FaceChunks(M) blocks take the face Z = 0 in chunks of eight
// rows (a warp per row).
__host__ __device__ __forceinline__ int p2FaceChunks(int M) { return (M + 1 + 7) / 8; }

template <class T, int K>
__device__ __forceinline__ T p2FaceDot(const T* u, const T* fw, const int (&pbz)[5], int w, int X, int Y, int Z) {
  using S = typename p2s::FaceList<K>::type;
  constexpr int kFirst = p2s::kFaceFirst[K], kLen = p2s::kFaceLen[K];
  return p2StencilDot<T>(S{}, std::make_integer_sequence<int, kLen>{}, u, fw + kFirst, pbz, w, X, Y, Z);
}

template <class T>
__device__ __forceinline__ T p2FaceDotAny(int k, const T* u, const T* fw, const int (&pbz)[5], int w, int X, int Y,
                                          int Z) {
  switch (k) {
    case 0: return p2FaceDot<T, 0>(u, fw, pbz, w, X, Y, Z);
    case 1: return p2FaceDot<T, 1>(u, fw, pbz, w, X, Y, Z);
    case 2: return p2FaceDot<T, 2>(u, fw, pbz, w, X, Y, Z);
    case 3: return p2FaceDot<T, 3>(u, fw, pbz, w, X, Y, Z);
    case 4: return p2FaceDot<T, 4>(u, fw, pbz, w, X, Y, Z);
    case 5: return p2FaceDot<T, 5>(u, fw, pbz, w, X, Y, Z);
    case 6: return p2FaceDot<T, 6>(u, fw, pbz, w, X, Y, Z);
    case 7: return p2FaceDot<T, 7>(u, fw, pbz, w, X, Y, Z);
    case 8: return p2FaceDot<T, 8>(u, fw, pbz, w, X, Y, Z);
    case 9: return p2FaceDot<T, 9>(u, fw, pbz, w, X, Y, Z);
    case 10: return p2FaceDot<T, 10>(u, fw, pbz, w, X, Y, Z);
    case 11: return p2FaceDot<T, 11>(u, fw, pbz, w, X, Y, Z);
    case 12: return p2FaceDot<T, 12>(u, fw, pbz, w, X, Y, Z);
    case 13: return p2FaceDot<T, 13>(u, fw, pbz, w, X, Y, Z);
    case 14: return p2FaceDot<T, 14>(u, fw, pbz, w, X, Y, Z);
    default: return p2FaceDot<T, 15>(u, fw, pbz, w, X, Y, Z);
  }
}

// Entry of (face f, class pc) in the face tables; the classes of a face are listed ascending:
// Z = 0: {0, 1, 2, 3}; Y = 0: {0, 1, 4, 5}; X = 0: {0, 2, 4, 6}; X + Y + Z = M: {0, 3, 5, 6}.
__device__ __forceinline__ int p2FaceEntry(int f, int pc) {
  switch (f) {
    case 0: return pc;
    case 1: return 4 + ((pc & 1) | ((pc >> 1) & 2));
    case 2: return 8 + (((pc >> 1) & 1) | ((pc >> 1) & 2));
    default: return 12 + (pc == 0 ? 0 : pc == 3 ? 1 : pc == 5 ? 2 : 3);
  }
}

template <class T>
__global__ void __launch_bounds__(kBlock) p2ClosureKernel(LevelDev lv, P2Tables tb, const T* __restrict__ K,
                                                          const T* __restrict__ FW, T* __restrict__ dst,
                                                          const T* __restrict__ src,
                                                          const unsigned char* __restrict__ colour, int sel) {
  const int M = lv.N, N = M / 2, w = lv.w, perCell = M + p2FaceChunks(M);
  const int c = blockIdx.x / perCell, q = blockIdx.x % perCell;
  const int Z = q < M ? q + 1 : 0;
  const int64_t base = lv.cellOff[c];
  const T* Kc = K + (int64_t)c * 600;
  __shared__ T fw[p2s::kFaceTotal];
  for (int k = threadIdx.x; k < p2s::kFaceTotal; k += blockDim.x) fw[k] = FW[(int64_t)c * p2s::kFaceTotal + k];
  __syncthreads();
  int pbz[5];
#pragma unroll
  for (int d = 0; d < 5; ++d) {
    const int z = Z - 2 + d;
    pbz[d] = (z >= 0 && z <= M) ? int(tetSize(w) - tetSize(w - z)) : 0;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto gatherNode = [&](int X, int Y) {
    const int64_t i = base + pbz[2] + rowStart(w - Z, Y) + X;
    if (sel < 0 || (colour[i] & 0x7f) == sel) dst[i] = p2GatherNode<T, false>(tb, Kc, src + base, pbz, w, N, X, Y, Z);
  };
  auto faceNode = [&](int k, int X, int Y) {
    const int64_t i = base + pbz[2] + rowStart(w - Z, Y) + X;
    if (sel < 0 || (colour[i] & 0x7f) == sel) dst[i] = p2FaceDotAny<T>(k, src + base, fw, pbz, w, X, Y, Z);
  };
  const int n = M - Z;
  if (Z == 0) {
    const int Y = (q - M) * 8 + warp;
    if (Y > n) return;
    if (Y == 0) {
      for (int X = lane; X <= n; X += 32) gatherNode(X, 0);
      return;
    }
    if (lane == 0) gatherNode(0, Y);
    if (lane == 1 && n - Y > 0) gatherNode(n - Y, Y);
#pragma unroll 1
    for (int px = 0; px < 2; ++px) {
      const int k = p2FaceEntry(0, px | ((Y & 1) << 1));
      for (int X = (px ? 1 : 2) + 2 * lane; X <= n - 1 - Y; X += 64) faceNode(k, X, Y);
    }
  } else if (n == 0) {
    if (threadIdx.x == 0) gatherNode(0, 0);
  } else if (warp < 6) {
    const int line = warp >> 1, par = warp & 1, zb = (Z & 1) << 2;
    for (int t = (par ? 1 : 2) + 2 * lane; t <= n - 1; t += 64) {
      if (line == 0)  // face Y = 0: X = t
        faceNode(p2FaceEntry(1, par | zb), t, 0);
      else if (line == 1)  // face X = 0: Y = t
        faceNode(p2FaceEntry(2, (par << 1) | zb), 0, t);
      else  // face X + Y + Z = M: Y = t, X = n - t
        faceNode(p2FaceEntry(3, ((n - t) & 1) | (par << 1) | zb), n - t, t);
    }
  } else if (warp == 6 && lane < 3) {
    if (lane == 0)
      gatherNode(0, 0);
    else if (lane == 1)
      gatherNode(n, 0);
    else
      gatherNode(0, n);
  }
}

// The closure nodes of one SOR colour from a per-colour list (one thread per node): the same
// shares as p2ClosureKernel, without visiting the nodes of the other colours. k = face-stencil
// entry of a face-interior node, -1 for a node on a cell edge or vertex (element gather).
struct P2ClosureNode {
  int cell;
  unsigned short x, y, z;
  signed char k;
  unsigned char pad;
};

template <class T>
__global__ void __launch_bounds__(kBlock) p2ClosureListKernel(LevelDev lv, P2Tables tb, const T* __restrict__ K,
                                                              const T* __restrict__ FW, T* __restrict__ dst,
                                                              const T* __restrict__ src,
                                                              const P2ClosureNode* __restrict__ list, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const P2ClosureNode nd = list[i];
  const int M = lv.N, N = M / 2, w = lv.w, X = nd.x, Y = nd.y, Z = nd.z;
  int pbz[5];
#pragma unroll
  for (int d = 0; d < 5; ++d) {
    const int z = Z - 2 + d;
    pbz[d] = (z >= 0 && z <= M) ? int(tetSize(w) - tetSize(w - z)) : 0;
  }
  const int64_t base = lv.cellOff[nd.cell];
  const T s = nd.k >= 0 ? p2FaceDotAny<T>(nd.k, src + base, FW + (int64_t)nd.cell * p2s::kFaceTotal, pbz, w, X, Y, Z)
                        : p2GatherNode<T, false>(tb, K + (int64_t)nd.cell * 600, src + base, pbz, w, N, X, Y, Z);
  dst[base + pbz[2] + rowStart(w - Z, Y) + X] = s;
}

// ---------------------------------------------------------------------------------------
// P2 quadratic transfers between P2 levels L and L + 1 (vertex lattices L + 1 and L + 2).
// A fine node Q of a macro-cell lies at Q / 4 in level-L micro-cell units; with a0 = Q >> 2
// and r = Q & 3, the candidates of class r are the micro-cells (type t, anchor a0 - delta)
// containing it, each with the ten values of the coarse P2 basis at the point. The first
// candidate inside the macro-cell is used (P2 is continuous, so any containing micro-cell gives
// the same interpolant). Fine nodes at even coordinates are coarse nodes (injection).
// ---------------------------------------------------------------------------------------
constexpr int kP2TrCand = 24;
struct P2TransferDev {
  const unsigned char* nCand;  // [64]
  const unsigned char* cand;   // [64][24]: delta (bits 3..5) << 3 | type
};

template <class T>
__device__ __forceinline__ int p2PickCandidate(const P2TransferDev& tr, const P2Tables& tb, int r, int ax0, int ay0,
                                               int az0, int N, int& ax, int& ay, int& az) {
  for (int k = 0; k < tr.nCand[r]; ++k) {
    const int c = tr.cand[r * kP2TrCand + k], t = c & 7, d = c >> 3;
    ax = ax0 - (d & 1);
    ay = ay0 - ((d >> 1) & 1);
    az = az0 - ((d >> 2) & 1);
    if (ax >= 0 && ay >= 0 && az >= 0 && ax + ay + az < N - tb.widthRed[t]) return k;
  }
  return -1;
}

// fine = P coarse on every node of the closed macro-cells (closure slots included)
template <class T>
__global__ void __launch_bounds__(kBlock) p2ProlongKernel(LevelDev lvc, LevelDev lvf, P2Tables tb, P2TransferDev tr,
                                                          const T* __restrict__ wts, const T* __restrict__ coarse,
                                                          T* __restrict__ fine) {
  const int Mf = lvf.N, Mc = lvc.N, N = Mc / 2, nPl = Mf + 1, wf = lvf.w, wc = lvc.w;
  const int c = blockIdx.x / nPl, Z = blockIdx.x % nPl;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const T* cc = coarse + lvc.cellOff[c];
  T* ff = fine + lvf.cellOff[c];
  auto cidx = [wc](int x, int y, int z) { return int(tetSize(wc) - tetSize(wc - z)) + rowStart(wc - z, y) + x; };
  const int pb = int(tetSize(wf) - tetSize(wf - Z));
  for (int Y = warp; Y <= Mf - Z; Y += kBlock / 32)
    for (int X = lane; X <= Mf - Z - Y; X += 32) {
      T v;
      if (((X | Y | Z) & 1) == 0) {
        v = cc[cidx(X >> 1, Y >> 1, Z >> 1)];
      } else {
        const int r = (X & 3) | ((Y & 3) << 2) | ((Z & 3) << 4);
        int ax, ay, az;
        const int k = p2PickCandidate<T>(tr, tb, r, X >> 2, Y >> 2, Z >> 2, N, ax, ay, az);
        v = T(0);
        if (k >= 0) {
          const int t = tr.cand[r * kP2TrCand + k] & 7;
          const T* w = wts + (r * kP2TrCand + k) * 10;
#pragma unroll
          for (int m = 0; m < 10; ++m)
            v += w[m] * cc[cidx(2 * ax + tb.off[t][m][0], 2 * ay + tb.off[t][m][1], 2 * az + tb.off[t][m][2])];
        }
      }
      ff[pb + rowStart(wf - Z, Y) + X] = v;
    }
}

// coarse = P^T (fine / multiplicity) on the closed macro-cells, as a gather: each cell writes its
// share (a DoF on a face, edge or vertex is split evenly among its cells) into its own coarse
// closure slots; the owners are summed afterwards. One thread per coarse node of a cell sums its
// contributions in the fixed order of the gather lists (compressed rows, the same for every
// cell), so the result does not depend on scheduling.
template <class T>
__global__ void __launch_bounds__(kBlock) p2RestrictGatherKernel(LevelDev lvc, LevelDev lvf, const int* __restrict__ ptr,
                                                                 const int* __restrict__ idx, const T* __restrict__ w,
                                                                 int nCoarse, int blocksPerCell, const T* __restrict__ fine,
                                                                 const unsigned char* __restrict__ mult, T* coarse) {
  const int c = blockIdx.x / blocksPerCell;
  const int node = (blockIdx.x - c * blocksPerCell) * kBlock + threadIdx.x;
  if (node >= nCoarse) return;
  const int64_t fb = lvf.cellOff[c];
  T acc = T(0);
  for (int j = ptr[node], e = ptr[node + 1]; j < e; ++j) {
    const int64_t i = fb + idx[j];
    acc += w[j] * (fine[i] / T(mult[i]));
  }
  coarse[lvc.cellOff[c] + node] = acc;
}

// owner <- its first cell-closure copy (values that every cell computes alike)
template <class T>
__global__ void __launch_bounds__(kBlock) p2PickKernel(const int64_t* __restrict__ owner, const int* __restrict__ ptr,
                                                       const int64_t* __restrict__ copies,
                                                       const unsigned char* __restrict__ type, int n, T* dst,
                                                       unsigned mask) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !(type[i] & mask)) return;
  dst[owner[i]] = dst[copies[ptr[i]]];
}

// ---------------------------------------------------------------------------------------
// Taylor-Hood coupling blocks between the P1 pressure lattice (level L) and the P2 velocity
// lattice (level L + 1); element matrices D[cell][type][k][4][10] (pressure vertex i, velocity
// node j). p2DivKernel: q = sum_k D_k u_k at the pressure nodes (a pressure node (x, y, z) is
// vertex i of micro-cell (t, (x, y, z) - v_t,i)). p2DivTKernel: v_k = D_k^T p at the velocity
// nodes (same candidates as the P2 operator). Both write final values at cell-interior nodes
// and this cell's share at the closure nodes; p2AddKernel sums the shares into the owners.
// ---------------------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(kBlock) p2DivKernel(LevelDev lvp, LevelDev lvv, P2Tables tb, const T* __restrict__ D,
                                                      T* __restrict__ q, const T* __restrict__ u0,
                                                      const T* __restrict__ u1, const T* __restrict__ u2,
                                                      unsigned mask, bool closureOnly) {
  const int N = lvp.N, nPl = N + 1, wp = lvp.w, wv = lvv.w;
  const int c = blockIdx.x / nPl, z = blockIdx.x % nPl;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t vb = lvv.cellOff[c];
  const T* Dc = D + (int64_t)c * 720;
  const bool cellOn = (lvp.cellType[c] & mask) != 0;
  auto vidx = [wv](int x, int y, int zz) { return int(tetSize(wv) - tetSize(wv - zz)) + rowStart(wv - zz, y) + x; };
  const int pb = int(tetSize(wp) - tetSize(wp - z));
  for (int y = warp; y <= N - z; y += kBlock / 32)
    for (int x = lane; x <= N - z - y; x += 32) {
      if (closureOnly && x >= 1 && y >= 1 && z >= 1 && x + y + z <= N - 1) continue;
      T s = T(0);
      for (int t = 0; t < 6; ++t)
        for (int i = 0; i < 4; ++i) {
          const int ax = x - (tb.off[t][i][0] >> 1), ay = y - (tb.off[t][i][1] >> 1), az = z - (tb.off[t][i][2] >> 1);
          if (ax < 0 || ay < 0 || az < 0 || ax + ay + az >= N - tb.widthRed[t]) continue;
          const T* Dr = Dc + t * 120 + i * 10;
#pragma unroll
          for (int j = 0; j < 10; ++j) {
            const int64_t g = vb + vidx(2 * ax + tb.off[t][j][0], 2 * ay + tb.off[t][j][1], 2 * az + tb.off[t][j][2]);
            s += Dr[j] * __ldg(u0 + g) + Dr[40 + j] * __ldg(u1 + g) + Dr[80 + j] * __ldg(u2 + g);
          }
        }
      const int64_t o = lvp.cellOff[c] + pb + rowStart(wp - z, y) + x;
      const bool interior = x >= 1 && y >= 1 && z >= 1 && x + y + z <= N - 1;
      if (!interior || cellOn) q[o] = s;
    }
}

template <class T>
__global__ void __launch_bounds__(kBlock) p2DivTKernel(LevelDev lvv, LevelDev lvp, P2Tables tb, const T* __restrict__ D,
                                                       T* __restrict__ v0, T* __restrict__ v1, T* __restrict__ v2,
                                                       const T* __restrict__ p, unsigned mask, bool closureOnly) {
  const int M = lvv.N, N = M / 2, nPl = M + 1, wv = lvv.w, wp = lvp.w;
  const int c = blockIdx.x / nPl, Z = blockIdx.x % nPl;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t pbase = lvp.cellOff[c];
  const T* Dc = D + (int64_t)c * 720;
  const bool cellOn = (lvv.cellType[c] & mask) != 0;
  auto pidx = [wp](int x, int y, int z) { return int(tetSize(wp) - tetSize(wp - z)) + rowStart(wp - z, y) + x; };
  const int pb = int(tetSize(wv) - tetSize(wv - Z));
  for (int Y = warp; Y <= M - Z; Y += kBlock / 32)
    for (int X = lane; X <= M - Z - Y; X += 32) {
      if (closureOnly && X >= 1 && Y >= 1 && Z >= 1 && X + Y + Z <= M - 1) continue;
      const int pc = (X & 1) | ((Y & 1) << 1) | ((Z & 1) << 2);
      T s0 = T(0), s1 = T(0), s2 = T(0);
      for (int k = 0; k < tb.nCand[pc]; ++k) {
        const int t = tb.cand[pc][k][0], j = tb.cand[pc][k][1];
        const int ax = (X - tb.off[t][j][0]) >> 1, ay = (Y - tb.off[t][j][1]) >> 1, az = (Z - tb.off[t][j][2]) >> 1;
        if (ax < 0 || ay < 0 || az < 0 || ax + ay + az >= N - tb.widthRed[t]) continue;
        const T* Dt = Dc + t * 120;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const T pv = __ldg(p + pbase + pidx(ax + (tb.off[t][i][0] >> 1), ay + (tb.off[t][i][1] >> 1), az + (tb.off[t][i][2] >> 1)));
          s0 += Dt[i * 10 + j] * pv;
          s1 += Dt[40 + i * 10 + j] * pv;
          s2 += Dt[80 + i * 10 + j] * pv;
        }
      }
      const int64_t o = lvv.cellOff[c] + pb + rowStart(wv - Z, Y) + X;
      const bool interior = X >= 1 && Y >= 1 && Z >= 1 && X + Y + Z <= M - 1;
      if (!interior || cellOn) {
        v0[o] = s0;
        v1[o] = s1;
        v2[o] = s2;
      }
    }
}

// Interior nodes of the coupling blocks by constant stencils (the micro-cells around an interior
// node form the same pattern at every node of its class). Weights per cell: [component][65].
//   p2DivStencilKernel: q at an interior pressure node (x, y, z) = sum_k sum_e WD_k[e] u_k at the
//   velocity nodes (2x, 2y, 2z) + p2s::S0[e]. Grid nCells * (Np - 3), one block per (cell, plane).
//   p2DivTStencilKernel: v_k at an interior velocity node of class pc = sum_e WT_k[e] p at the
//   pressure nodes (X >> 1, Y >> 1, Z >> 1) + p2s::DivTList<pc>[e]. Grid nCells * (M - 3).
template <class T>
__device__ __forceinline__ void p2Acc3(T (&s)[6], const T* w, int I, const T* u0, const T* u1, const T* u2, int o) {
  const int h = I & 1;  // two partial sums per component
  s[h] += w[I] * __ldg(u0 + o);
  s[2 + h] += w[65 + I] * __ldg(u1 + o);
  s[4 + h] += w[130 + I] * __ldg(u2 + o);
}

template <class T>
__device__ __forceinline__ void p2Acc3T(T& s0, T& s1, T& s2, const T* w, int I, T pv) {
  s0 += w[I] * pv;
  s1 += w[65 + I] * pv;
  s2 += w[130 + I] * pv;
}

template <class T, int... DX, int... DY, int... DZ, int... I>
__device__ __forceinline__ T p2DivDot(p2s::List<p2s::O<DX, DY, DZ>...>, std::integer_sequence<int, I...>, const T* u0,
                                      const T* u1, const T* u2, const T* w, const int (&pbz)[5], int wv, int X, int Y,
                                      int Z) {
  T s[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
  (p2Acc3<T>(s, w, I, u0, u1, u2, p2RowBase<DY, DZ>(pbz, wv, Y, Z) + X + DX), ...);
  return (s[0] + s[1]) + ((s[2] + s[3]) + (s[4] + s[5]));
}

template <class T, int... DX, int... DY, int... DZ, int... I>
__device__ __forceinline__ void p2DivTDot(p2s::List<p2s::O<DX, DY, DZ>...>, std::integer_sequence<int, I...>,
                                          const T* p, const T* w, const int (&pbz)[5], int wp, int x, int y, int z,
                                          T& s0, T& s1, T& s2) {
  (p2Acc3T<T>(s0, s1, s2, w, I, __ldg(p + p2RowBase<DY, DZ>(pbz, wp, y, z) + x + DX)), ...);
}

template <class T>
__global__ void __launch_bounds__(kBlock) p2DivStencilKernel(LevelDev lvp, LevelDev lvv, const T* __restrict__ WD,
                                                             T* __restrict__ q, const T* __restrict__ u0,
                                                             const T* __restrict__ u1, const T* __restrict__ u2,
                                                             unsigned mask) {
  const int N = lvp.N, nPl = N - 3, wp = lvp.w, wv = lvv.w, M = lvv.N;
  const int c = blockIdx.x / nPl, z = 1 + blockIdx.x % nPl;
  if (!(lvp.cellType[c] & mask)) return;
  __shared__ T wts[195];
  for (int k = threadIdx.x; k < 195; k += blockDim.x) wts[k] = WD[(int64_t)c * 195 + k];
  __syncthreads();
  int pbz[5];  // velocity planes 2z - 2 .. 2z + 2
#pragma unroll
  for (int d = 0; d < 5; ++d) {
    const int zz = 2 * z - 2 + d;
    pbz[d] = (zz >= 0 && zz <= M) ? int(tetSize(wv) - tetSize(wv - zz)) : 0;
  }
  const int64_t vb = lvv.cellOff[c];
  const int pb = int(tetSize(wp) - tetSize(wp - z));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  using S = p2s::S0;
  for (int y = 1 + warp; y <= N - 2 - z; y += kBlock / 32)
    for (int x = 1 + lane; x <= N - 1 - y - z; x += 32)
      q[lvp.cellOff[c] + pb + rowStart(wp - z, y) + x] =
          p2DivDot<T>(S{}, std::make_integer_sequence<int, p2s::kLen[0]>{}, u0 + vb, u1 + vb, u2 + vb, wts, pbz, wv,
                      2 * x, 2 * y, 2 * z);
}

template <class T, int PC>
__device__ __forceinline__ void p2DivTRow(const T* wts, T* v0, T* v1, T* v2, const T* p, int64_t vrow,
                                          const int (&pbzP)[5], int wp, int M, int Y, int Z, int lane) {
  using S = typename p2s::DivTList<PC>::type;
  constexpr int kFirst = p2s::kDivTFirst[PC], kLen = p2s::kDivTLen[PC];
#pragma unroll 1
  for (int X = ((PC & 1) ? 1 : 2) + 2 * lane; X <= M - 1 - Y - Z; X += 64) {
    T s0 = T(0), s1 = T(0), s2 = T(0);
    p2DivTDot<T>(S{}, std::make_integer_sequence<int, kLen>{}, p, wts + kFirst, pbzP, wp, X >> 1, Y >> 1, Z >> 1, s0,
                 s1, s2);
    v0[vrow + X] = s0;
    v1[vrow + X] = s1;
    v2[vrow + X] = s2;
  }
}

template <class T>
__global__ void __launch_bounds__(kBlock) p2DivTStencilKernel(LevelDev lvv, LevelDev lvp, const T* __restrict__ WT,
                                                              T* __restrict__ v0, T* __restrict__ v1,
                                                              T* __restrict__ v2, const T* __restrict__ p,
                                                              unsigned mask) {
  const int M = lvv.N, nPl = M - 3, wv = lvv.w, wp = lvp.w, Np = lvp.N;
  const int c = blockIdx.x / nPl, Z = 1 + blockIdx.x % nPl;
  if (!(lvv.cellType[c] & mask)) return;
  __shared__ T wts[195];
  for (int k = threadIdx.x; k < 195; k += blockDim.x) wts[k] = WT[(int64_t)c * 195 + k];
  __syncthreads();
  int pbzP[5];  // pressure planes (Z >> 1) - 2 .. (Z >> 1) + 2
#pragma unroll
  for (int d = 0; d < 5; ++d) {
    const int zz = (Z >> 1) - 2 + d;
    pbzP[d] = (zz >= 0 && zz <= Np) ? int(tetSize(wp) - tetSize(wp - zz)) : 0;
  }
  const T* pc0 = p + lvp.cellOff[c];
  const int64_t vb = lvv.cellOff[c] + int(tetSize(wv) - tetSize(wv - Z));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int Y = 1 + warp; Y <= M - 2 - Z; Y += kBlock / 32) {
    const int64_t vrow = vb + rowStart(wv - Z, Y);
#pragma unroll 1
    for (int px = 0; px < 2; ++px) {
      switch (px | ((Y & 1) << 1) | ((Z & 1) << 2)) {
        case 0: p2DivTRow<T, 0>(wts, v0, v1, v2, pc0, vrow, pbzP, wp, M, Y, Z, lane); break;
        case 1: p2DivTRow<T, 1>(wts, v0, v1, v2, pc0, vrow, pbzP, wp, M, Y, Z, lane); break;
        case 2: p2DivTRow<T, 2>(wts, v0, v1, v2, pc0, vrow, pbzP, wp, M, Y, Z, lane); break;
        case 3: p2DivTRow<T, 3>(wts, v0, v1, v2, pc0, vrow, pbzP, wp, M, Y, Z, lane); break;
        case 4: p2DivTRow<T, 4>(wts, v0, v1, v2, pc0, vrow, pbzP, wp, M, Y, Z, lane); break;
        case 5: p2DivTRow<T, 5>(wts, v0, v1, v2, pc0, vrow, pbzP, wp, M, Y, Z, lane); break;
        case 6: p2DivTRow<T, 6>(wts, v0, v1, v2, pc0, vrow, pbzP, wp, M, Y, Z, lane); break;
        default: p2DivTRow<T, 7>(wts, v0, v1, v2, pc0, vrow, pbzP, wp, M, Y, Z, lane); break;
      }
    }
  }
}

// The closure nodes of the coupling blocks from the closure lists (one thread per node, the
// element gather of p2DivKernel / p2DivTKernel): shares into the cells' closure slots.
template <class T>
__global__ void __launch_bounds__(kBlock) p2DivClosureListKernel(LevelDev lvp, LevelDev lvv, P2Tables tb,
                                                                 const T* __restrict__ D, T* __restrict__ q,
                                                                 const T* __restrict__ u0, const T* __restrict__ u1,
                                                                 const T* __restrict__ u2,
                                                                 const P2ClosureNode* __restrict__ list, int n) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const P2ClosureNode nd = list[idx];
  const int N = lvp.N, wp = lvp.w, wv = lvv.w, x = nd.x, y = nd.y, z = nd.z;
  const int64_t vb = lvv.cellOff[nd.cell];
  const T* Dc = D + (int64_t)nd.cell * 720;
  auto vidx = [wv](int xx, int yy, int zz) { return int(tetSize(wv) - tetSize(wv - zz)) + rowStart(wv - zz, yy) + xx; };
  T s = T(0);
  for (int t = 0; t < 6; ++t)
    for (int i = 0; i < 4; ++i) {
      const int ax = x - (tb.off[t][i][0] >> 1), ay = y - (tb.off[t][i][1] >> 1), az = z - (tb.off[t][i][2] >> 1);
      if (ax < 0 || ay < 0 || az < 0 || ax + ay + az >= N - tb.widthRed[t]) continue;
      const T* Dr = Dc + t * 120 + i * 10;
#pragma unroll
      for (int j = 0; j < 10; ++j) {
        const int64_t g = vb + vidx(2 * ax + tb.off[t][j][0], 2 * ay + tb.off[t][j][1], 2 * az + tb.off[t][j][2]);
        s += Dr[j] * __ldg(u0 + g) + Dr[40 + j] * __ldg(u1 + g) + Dr[80 + j] * __ldg(u2 + g);
      }
    }
  q[lvp.cellOff[nd.cell] + int(tetSize(wp) - tetSize(wp - z)) + rowStart(wp - z, y) + x] = s;
}

template <class T>
__global__ void __launch_bounds__(kBlock) p2DivTClosureListKernel(LevelDev lvv, LevelDev lvp, P2Tables tb,
                                                                  const T* __restrict__ D, T* __restrict__ v0,
                                                                  T* __restrict__ v1, T* __restrict__ v2,
                                                                  const T* __restrict__ p,
                                                                  const P2ClosureNode* __restrict__ list, int n) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const P2ClosureNode nd = list[idx];
  const int M = lvv.N, N = M / 2, wv = lvv.w, wp = lvp.w, X = nd.x, Y = nd.y, Z = nd.z;
  const int64_t pbase = lvp.cellOff[nd.cell];
  const T* Dc = D + (int64_t)nd.cell * 720;
  auto pidx = [wp](int x, int y, int z) { return int(tetSize(wp) - tetSize(wp - z)) + rowStart(wp - z, y) + x; };
  const int pc = (X & 1) | ((Y & 1) << 1) | ((Z & 1) << 2);
  T s0 = T(0), s1 = T(0), s2 = T(0);
  for (int k = 0; k < tb.nCand[pc]; ++k) {
    const int t = tb.cand[pc][k][0], j = tb.cand[pc][k][1];
    const int ax = (X - tb.off[t][j][0]) >> 1, ay = (Y - tb.off[t][j][1]) >> 1, az = (Z - tb.off[t][j][2]) >> 1;
    if (ax < 0 || ay < 0 || az < 0 || ax + ay + az >= N - tb.widthRed[t]) continue;
    const T* Dt = Dc + t * 120;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const T pv = __ldg(p + pbase + pidx(ax + (tb.off[t][i][0] >> 1), ay + (tb.off[t][i][1] >> 1), az + (tb.off[t][i][2] >> 1)));
      s0 += Dt[i * 10 + j] * pv;
      s1 += Dt[40 + i * 10 + j] * pv;
      s2 += Dt[80 + i * 10 + j] * pv;
    }
  }
  const int64_t o = lvv.cellOff[nd.cell] + int(tetSize(wv) - tetSize(wv - Z)) + rowStart(wv - Z, Y) + X;
  v0[o] = s0;
  v1[o] = s1;
  v2[o] = s2;
}

// Sums the cells' shares of every DoF owned by a face, edge or vertex (the copies of that DoF in
// the closure slots of its cells) into the owner slot: dst = sum, or rhs - sum for a residual.
template <class T, int MODE>
__global__ void __launch_bounds__(kBlock) p2AddKernel(const int64_t* __restrict__ owner, const int* __restrict__ ptr,
                                                      const int64_t* __restrict__ copies,
                                                      const unsigned char* __restrict__ type, int n, T* dst,
                                                      const T* __restrict__ rhs, unsigned mask,
                                                      const unsigned char* __restrict__ colour, int sel) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !(type[i] & mask)) return;
  if (sel >= 0 && (colour[owner[i]] & 0x7f) != sel) return;
  T v = T(0);
  for (int k = ptr[i]; k < ptr[i + 1]; ++k) v += dst[copies[k]];
  const int64_t o = owner[i];
  dst[o] = MODE == MODE_RESIDUAL ? rhs[o] - v : v;
}

// colour < 0: all points; otherwise x mod 2 == colour (edges are 1-D chains)
template <class T>
__global__ void __launch_bounds__(kBlock) lowSorKernel(LevelDev lv, StencilDev<T> st, T* u, const T* __restrict__ rhs,
                                                       unsigned mask, int colour, T omega, int blockBegin) {
  const LowBlock b = lv.lowBlocks[blockBegin + blockIdx.x];
  if (!(lv.lowType[b.prim] & mask)) return;
  const int x = b.start + threadIdx.x;
  if (x >= lv.lowFirst[b.prim] + lv.lowCount[b.prim]) return;
  if (colour >= 0 && (x & 1) != colour) return;
  const int64_t c = lv.lowOff[b.prim] + x;
  const int e0 = st.lowEntOff[b.prim];
  T s = rhs[c];
  for (int k = e0 + 1; k < st.lowEntOff[b.prim + 1]; ++k) s -= st.lowEntW[k] * u[c + st.lowEntRel[k]];
  u[c] = (T(1) - omega) * u[c] + (s * omega) / st.lowEntW[e0];
}

template <class T>
__global__ void __launch_bounds__(kBlock) lowRestrictKernel(LevelDev lc, LevelDev lf, StencilDev<T> stf,
                                                            T* __restrict__ coarse, const T* __restrict__ fine,
                                                            unsigned mask) {
  const LowBlock b = lc.lowBlocks[blockIdx.x];
  if (!(lc.lowType[b.prim] & mask)) return;
  const int x = b.start + threadIdx.x;
  if (x >= lc.lowFirst[b.prim] + lc.lowCount[b.prim]) return;
  const int64_t cf = lf.lowOff[b.prim] + 2 * x;
  const int e0 = stf.lowEntOff[b.prim];
  T s = T(0);
  for (int k = e0 + 1; k < stf.lowEntOff[b.prim + 1]; ++k) s += __ldg(fine + cf + stf.lowEntRel[k]);
  coarse[lc.lowOff[b.prim] + x] = __ldg(fine + cf) + T(0.5) * s;
}

template <class T, bool ADD>
__global__ void __launch_bounds__(kBlock) lowProlongKernel(LevelDev lf, LevelDev lc, T* __restrict__ fine,
                                                           const T* __restrict__ coarse, unsigned mask) {
  const LowBlock b = lf.lowBlocks[blockIdx.x];
  if (!(lf.lowType[b.prim] & mask)) return;
  const int x = b.start + threadIdx.x;
  if (x >= lf.lowFirst[b.prim] + lf.lowCount[b.prim]) return;
  const int64_t cb = lc.lowOff[b.prim];
  const T v = (x & 1) ? T(0.5) * (__ldg(coarse + cb + (x >> 1)) + __ldg(coarse + cb + (x >> 1) + 1))
                      : __ldg(coarse + cb + (x >> 1));
  const int64_t c = lf.lowOff[b.prim] + x;
  if (ADD) fine[c] += v;
  else fine[c] = v;
}

// ---------------------------------------------------------------------------------------
// Interpolation of built-in expressions at the owned DoFs (VertexDoFFunction::interpolate):
//   expr 0: a * sin(k pi x) sin(k pi y) sin(k pi z)       (params a, k)
//   expr 1: a + b x + c y + d z                           (params a, b, c, d)
// Coordinates are the barycentric combination of the primitive's macro-vertices.
// ---------------------------------------------------------------------------------------
struct Geometry {
  const double* vx;    // [nVerts][3]
  const int* cellV;    // [nCells][4] (frame order)
  const int* faceV;    // [nFaces][3]
  const int* lowV;     // [nLow][2]: edges (v0, v1), vertices (v, v)
};

__device__ __forceinline__ double evalExpr(int expr, const double* p, double x, double y, double z) {
  if (expr == 0) {
    const double k = p[1] * 3.141592653589793;
    return p[0] * sin(k * x) * sin(k * y) * sin(k * z);
  }
  return p[0] + p[1] * x + p[2] * y + p[3] * z;
}

template <class T>
__global__ void __launch_bounds__(kBlock) interpolateKernel(LevelDev lv, Geometry g, T* __restrict__ dst, unsigned mask,
                                                            int expr, double p0, double p1, double p2, double p3) {
  const double prm[4] = {p0, p1, p2, p3};
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double invN = 1.0 / lv.N;
  int blk = blockIdx.x;
  const int nCellGrid = lv.nCellBlocks;
  if (blk < nCellGrid) {
    const int nPl = lv.N - 3;
    const int c = blk / nPl, z = 1 + blk % nPl;
    if (!(lv.cellType[c] & mask)) return;
    const int* cv = g.cellV + 4 * c;
    const int W = lv.w - z;
    T* d = dst + lv.cellOff[c];
    for (int y = 1 + warp; y <= W - 3; y += kBlock / 32) {
      const int r0 = int(tetSize(lv.w) - tetSize(W)) + rowStart(W, y);
      for (int x = 1 + lane; x <= W - 2 - y; x += 32) {
        const double b[4] = {double(lv.N - x - y - z), double(x), double(y), double(z)};
        double q[3] = {0, 0, 0};
        for (int k = 0; k < 4; ++k)
          for (int e = 0; e < 3; ++e) q[e] += b[k] * g.vx[3 * cv[k] + e];
        d[r0 + x] = T(evalExpr(expr, prm, q[0] * invN, q[1] * invN, q[2] * invN));
      }
    }
  } else if ((blk -= nCellGrid) < lv.nFaceBlocks) {
    const FaceBlock fb = lv.faceBlocks[blk];
    if (!(lv.faceType[fb.face] & mask)) return;
    const int* fv = g.faceV + 3 * fb.face;
    T* d = dst + lv.faceOff[fb.face];
    const int yEnd = min(fb.start + kFaceRows, lv.w - 2);
    for (int y = fb.start + warp; y < yEnd; y += kBlock / 32) {
      const int r0 = rowStart(lv.w, y);
      for (int x = 1 + lane; x <= lv.w - 2 - y; x += 32) {
        const double b[3] = {double(lv.N - x - y), double(x), double(y)};
        double q[3] = {0, 0, 0};
        for (int k = 0; k < 3; ++k)
          for (int e = 0; e < 3; ++e) q[e] += b[k] * g.vx[3 * fv[k] + e];
        d[r0 + x] = T(evalExpr(expr, prm, q[0] * invN, q[1] * invN, q[2] * invN));
      }
    }
  } else {
    blk -= lv.nFaceBlocks;
    const LowBlock lb = lv.lowBlocks[blk];
    if (!(lv.lowType[lb.prim] & mask)) return;
    const int x = lb.start + threadIdx.x;
    if (x >= lv.lowFirst[lb.prim] + lv.lowCount[lb.prim]) return;
    const int* ev = g.lowV + 2 * lb.prim;
    const double b0 = lb.prim < lv.nEdges ? double(lv.N - x) : double(lv.N), b1 = lb.prim < lv.nEdges ? double(x) : 0.0;
    double q[3];
    for (int e = 0; e < 3; ++e) q[e] = (b0 * g.vx[3 * ev[0] + e] + b1 * g.vx[3 * ev[1] + e]) * invN;
    dst[lv.lowOff[lb.prim] + x] = T(evalExpr(expr, prm, q[0], q[1], q[2]));
  }
}

// ---------------------------------------------------------------------------------------
// Stencil re-assembly for new macro-cell coefficients: every stencil entry of one level is the
// sum of its element-matrix terms K_i (times the coefficient of the term's cell for the
// diffusion form), added in the order the host assembly adds them, with explicit
// round-to-nearest products and sums (no contraction), so the device gives the host's bits. The
// targets are the level's cell weights [cells][16], face entries [faces][16] and edge/vertex
// entries, in that order; each is written in FP64 and rounded to FP32.
// ---------------------------------------------------------------------------------------
struct PlanTermDev {
  int cell;
  int scaled;
  double K;
};

static __global__ void __launch_bounds__(kBlock)
    planAssembleKernel(const int64_t* __restrict__ first, const PlanTermDev* __restrict__ terms,
                       const double* __restrict__ coef, int64_t nCell, int64_t nFace, int64_t nLow, double* cell64,
                       float* cell32, FaceEnt<double>* face64, FaceEnt<float>* face32, double* low64, float* low32) {
  const int64_t t = blockIdx.x * (int64_t)kBlock + threadIdx.x;
  if (t >= nCell + nFace + nLow) return;
  double v = 0.0;
  for (int64_t i = first[t]; i < first[t + 1]; ++i) {
    const PlanTermDev x = terms[i];
    v = __dadd_rn(v, x.scaled ? __dmul_rn(x.K, coef[x.cell]) : x.K);
  }
  const float vf = __double2float_rn(v);
  if (t < nCell) {
    cell64[t] = v;
    cell32[t] = vf;
  } else if (t < nCell + nFace) {
    face64[t - nCell].w = v;
    face32[t - nCell].w = vf;
  } else {
    low64[t - nCell - nFace] = v;
    low32[t - nCell - nFace] = vf;
  }
}

// ---------------------------------------------------------------------------------------
// Halo refresh: copy slots <- owner slots (one gather; every source is an owned slot).
// ---------------------------------------------------------------------------------------
// Four entries per thread and round, table reads first, so that four independent gathers are in
// flight; every source is an owned slot and every destination a copy slot, so the order of the
// copies does not matter.
constexpr int kCommUnroll = 4;
template <class T>
__global__ void commGatherKernel(T* buf, const uint2* __restrict__ table, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i0 < n; i0 += kCommUnroll * stride) {
    uint2 t[kCommUnroll];
    T v[kCommUnroll];
#pragma unroll
    for (int k = 0; k < kCommUnroll; ++k)
      if (i0 + k * stride < n) t[k] = table[i0 + k * stride];
#pragma unroll
    for (int k = 0; k < kCommUnroll; ++k)
      if (i0 + k * stride < n) v[k] = buf[t[k].y];
#pragma unroll
    for (int k = 0; k < kCommUnroll; ++k)
      if (i0 + k * stride < n) buf[t[k].x] = v[k];
  }
}

// The same refresh while the cell arrays of the level live in a second buffer in the
// colour-split order: slots below cellEnd (the table holds their split positions) are in
// cells, the others in buf.
template <class T>
__global__ void commGatherSplitKernel(T* buf, T* cells, const uint2* __restrict__ table, int64_t n, int64_t cellEnd) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint2 t = table[i];
    const T v = t.y < cellEnd ? cells[t.y] : buf[t.y];
    if (t.x < cellEnd) cells[t.x] = v;
    else buf[t.x] = v;
  }
}

// ---------------------------------------------------------------------------------------
// Vector operations over whole primitive arrays of the flagged primitives (chunk table:
// start, length, DoFType). Linear combinations keep copy slots consistent copies.
// ---------------------------------------------------------------------------------------
struct Chunk {
  int64_t start;
  int len;
  int type;
};

template <class T>
__global__ void __launch_bounds__(kBlock) lincombKernel(const Chunk* __restrict__ chunks, unsigned mask, T* dst, int nsrc,
                                                        const T* s0, const T* s1, const T* s2, double a0, double a1,
                                                        double a2, int addToDst, double constant) {
  const Chunk ch = chunks[blockIdx.x];
  if (!(ch.type & mask)) return;
  for (int i = threadIdx.x; i < ch.len; i += blockDim.x) {
    const int64_t j = ch.start + i;
    T v = addToDst ? dst[j] : T(constant);
    if (nsrc > 0) v += T(a0) * s0[j];
    if (nsrc > 1) v += T(a1) * s1[j];
    if (nsrc > 2) v += T(a2) * s2[j];
    dst[j] = v;
  }
}

// dst = a / b on the flagged primitives' slots (the inverse of a lumped / diagonal operator)
static __global__ void __launch_bounds__(kBlock) divideKernel(const Chunk* __restrict__ chunks, unsigned mask, double* dst,
                                                      const double* __restrict__ a, const double* __restrict__ b) {
  const Chunk ch = chunks[blockIdx.x];
  if (!(ch.type & mask)) return;
  for (int i = threadIdx.x; i < ch.len; i += blockDim.x) {
    const int64_t j = ch.start + i;
    dst[j] = a[j] / b[j];
  }
}

template <class TD, class TS>
__global__ void __launch_bounds__(kBlock) castKernel(const Chunk* __restrict__ chunks, unsigned mask, TD* dst,
                                                     const TS* src, int add) {
  const Chunk ch = chunks[blockIdx.x];
  if (!(ch.type & mask)) return;
  for (int i = threadIdx.x; i < ch.len; i += blockDim.x) {
    const int64_t j = ch.start + i;
    if (add) dst[j] += TD(src[j]);
    else dst[j] = TD(src[j]);
  }
}

// x[idx[i]] += sum_k Ainv(i, k) r[idx[k]] for the n unknowns of a coarse level (the exact coarse
// solve; Ainv column-major, n * 8 bytes of dynamic shared memory): every block stages r at the
// unknowns in shared memory, each thread computes one row.
static __global__ void __launch_bounds__(kBlock) denseCorrectKernel(const int64_t* __restrict__ idx, int n,
                                                                    const double* __restrict__ Ainv,
                                                                    const double* __restrict__ r, double* x) {
  extern __shared__ double rs[];
  for (int k = threadIdx.x; k < n; k += blockDim.x) rs[k] = r[idx[k]];
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double t = 0.0;
  for (int k = 0; k < n; ++k) t += Ainv[(int64_t)k * n + i] * rs[k];
  x[idx[i]] += t;
}

// dst = vals[chunk] at every slot of every chunk (a constant per primitive array).
static __global__ void __launch_bounds__(kBlock) fillChunksKernel(const Chunk* __restrict__ chunks,
                                                                  const double* __restrict__ vals, double* dst) {
  const Chunk ch = chunks[blockIdx.x];
  const double v = vals[blockIdx.x];
  for (int i = threadIdx.x; i < ch.len; i += blockDim.x) dst[ch.start + i] = v;
}

// The exact coarse solve of a block system over up to four functions: unknown i is slot idx[i]
// of function comp[i]; x_comp[i][idx[i]] += sum_k Kinv(i, k) r_comp[k][idx[k]] (Kinv column-major,
// n * 8 bytes of dynamic shared memory).
struct BlockPtrs {
  const double* r[4];
  double* x[4];
};
static __global__ void __launch_bounds__(kBlock) blockDenseCorrectKernel(const int64_t* __restrict__ idx,
                                                                         const unsigned char* __restrict__ comp, int n,
                                                                         const double* __restrict__ Kinv, BlockPtrs bp) {
  extern __shared__ double rs[];
  for (int k = threadIdx.x; k < n; k += blockDim.x) rs[k] = bp.r[comp[k]][idx[k]];
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double t = 0.0;
  for (int k = 0; k < n; ++k) t += Kinv[(int64_t)k * n + i] * rs[k];
  bp.x[comp[i]][idx[i]] += t;
}

// The owner update of one P2 SOR colour from per-colour lists: entries t < nAdd are indices into
// the owner table (a face, edge or vertex DoF: its cells' shares are summed here), the others are
// interior slots whose A x is in ax (the vertex colours). x += omega (b - A x) / diag.
template <class T>
__global__ void __launch_bounds__(kBlock) p2SorOwnersKernel(const int64_t* __restrict__ owner,
                                                            const int* __restrict__ ptr,
                                                            const int64_t* __restrict__ copies,
                                                            const unsigned char* __restrict__ type,
                                                            const int* __restrict__ addIdx, int nAdd,
                                                            const int64_t* __restrict__ inner,
                                                            const unsigned char* __restrict__ innerType, int nInner,
                                                            unsigned mask, T* x, const T* __restrict__ b,
                                                            const T* __restrict__ ax, const T* __restrict__ diag,
                                                            T omega) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nAdd) {
    const int j = addIdx[t];
    if (!(type[j] & mask)) return;
    T s = T(0);
    for (int k = ptr[j]; k < ptr[j + 1]; ++k) s += ax[copies[k]];
    const int64_t o = owner[j];
    const T v = x[o] + omega * (b[o] - s) / diag[o];
    x[o] = v;
    // the owner's copies in the cell closures of x take the new value at once (the refresh of this
    // colour's copies before the next colour pass)
    for (int k = ptr[j]; k < ptr[j + 1]; ++k) x[copies[k]] = v;
  } else if (t < nAdd + nInner) {
    const int q = t - nAdd;
    if (!(innerType[q] & mask)) return;
    const int64_t o = inner[q];
    x[o] += omega * (b[o] - ax[o]) / diag[o];
  }
}

// Seeded uniform values in [lo, hi) at every slot of the flagged primitives' arrays; the value
// depends only on (seed, slot index), so a level buffer of one topology is reproducible.
// splitmix64 (Steele, Lea, Flood 2014) of the slot index mixed with the seed; 53 bits -> [0, 1).
__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

template <class T>
__global__ void __launch_bounds__(kBlock) randomFillKernel(const Chunk* __restrict__ chunks, unsigned mask, T* dst,
                                                           uint64_t seed, double lo, double hi) {
  const Chunk ch = chunks[blockIdx.x];
  if (!(ch.type & mask)) return;
  const uint64_t s = splitmix64(seed);
  for (int i = threadIdx.x; i < ch.len; i += blockDim.x) {
    const int64_t j = ch.start + i;
    const double u = double(splitmix64(s ^ uint64_t(j)) >> 11) * (1.0 / 9007199254740992.0);
    dst[j] = T(lo + (hi - lo) * u);
  }
}

// Dot product over owned DoFs of flagged primitives, each DoF counted once
// (VertexDoFFunction.cpp:1421-1498). Blocks: cell blocks, then face blocks, then low blocks.
// Deterministic: fixed per-block partial sums reduced by a second kernel.
template <class T>
__device__ __forceinline__ double blockReduce(double v) {
  __shared__ double warpSums[kBlock / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) warpSums[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x < 32) {
    r = threadIdx.x < kBlock / 32 ? warpSums[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  return r;
}

template <class T>
__global__ void __launch_bounds__(kBlock) dotKernel(LevelDev lv, const T* __restrict__ a, const T* __restrict__ b,
                                                    unsigned mask, double* partial) {
  double v = 0.0;
  int blk = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nCellGrid = lv.N >= 4 ? lv.nCells * (lv.N - 3) : 0;
  if (blk < nCellGrid) {
    const int nPl = lv.N - 3;
    const int c = blk / nPl, z = 1 + blk % nPl;
    if (lv.cellType[c] & mask) {
      const T* __restrict__ pa = a + lv.cellOff[c];
      const T* __restrict__ pb = b + lv.cellOff[c];
      const int W = lv.w - z;
      for (int y = 1 + warp; y <= W - 3; y += kBlock / 32) {
        const int r0 = int(tetSize(lv.w) - tetSize(W)) + rowStart(W, y);
        for (int x = 1 + lane; x <= W - 2 - y; x += 32) v += double(pa[r0 + x]) * double(pb[r0 + x]);
      }
    }
  } else if ((blk -= nCellGrid) < lv.nFaceBlocks) {
    const FaceBlock fb = lv.faceBlocks[blk];
    if (lv.faceType[fb.face] & mask) {
      const T* __restrict__ pa = a + lv.faceOff[fb.face];
      const T* __restrict__ pb = b + lv.faceOff[fb.face];
      const int yEnd = min(fb.start + kFaceRows, lv.w - 2);
      for (int y = fb.start + warp; y < yEnd; y += kBlock / 32) {
        const int r0 = rowStart(lv.w, y);
        for (int x = 1 + lane; x <= lv.w - 2 - y; x += 32) v += double(pa[r0 + x]) * double(pb[r0 + x]);
      }
    }
  } else {
    blk -= lv.nFaceBlocks;
    const LowBlock lb = lv.lowBlocks[blk];
    if (lv.lowType[lb.prim] & mask) {
      const int x = lb.start + threadIdx.x;
      if (x < lv.lowFirst[lb.prim] + lv.lowCount[lb.prim]) {
        const int64_t c = lv.lowOff[lb.prim] + x;
        v = double(a[c]) * double(b[c]);
      }
    }
  }
  const double r = blockReduce<T>(v);
  if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

static __global__ void __launch_bounds__(kBlock) reduceKernel(const double* __restrict__ partial, int n, double* out) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += partial[i];
  const double r = blockReduce<double>(v);
  if (threadIdx.x == 0) *out = r;
}

// ---------------------------------------------------------------------------------------
// Batched solves: a union storage holds `copies` disjoint copies of one macro-mesh, each kind of
// primitive (cells, faces, edges, vertices, the level buffer's order) copy after copy, each copy
// in a single mesh's order. Per kind: the first slot of the union, the slots of one copy, and the
// first slot of the kind in one copy's own layout. Per segment of the dot product's partial sums
// (cell, face, edge and vertex blocks): the first block of the union and the blocks of one copy.
// ---------------------------------------------------------------------------------------
struct BatchMap {
  int copies;
  int64_t uBase[4], size[4], aBase[4];
  int bBase[4], bCount[4];
};

// Right-hand sides of the copies: copy i < active gets at every slot of its flagged primitives
// the value a storage of the single mesh gets from seeds[i] at the same slot of its own layout
// (randomFillKernel); the copies from `active` on get 0. A chunk lies in one primitive array.
template <class T>
__global__ void __launch_bounds__(kBlock) randomFillBatchKernel(const Chunk* __restrict__ chunks, unsigned mask, T* dst,
                                                                BatchMap bm, const uint64_t* __restrict__ seeds,
                                                                int active, double lo, double hi) {
  const Chunk ch = chunks[blockIdx.x];
  if (!(ch.type & mask)) return;
  int k = 3;
  while (k > 0 && ch.start < bm.uBase[k]) --k;
  const int64_t rel = ch.start - bm.uBase[k];
  const int copy = int(rel / bm.size[k]);
  if (copy >= active) {
    for (int i = threadIdx.x; i < ch.len; i += blockDim.x) dst[ch.start + i] = T(0);
    return;
  }
  const int64_t local0 = bm.aBase[k] + (rel - int64_t(copy) * bm.size[k]);
  const uint64_t s = splitmix64(seeds[copy]);
  for (int i = threadIdx.x; i < ch.len; i += blockDim.x) {
    const double u = double(splitmix64(s ^ uint64_t(local0 + i)) >> 11) * (1.0 / 9007199254740992.0);
    dst[ch.start + i] = T(lo + (hi - lo) * u);
  }
}

// Per-copy dot products from dotKernel's per-block partial sums of the union: block i sums copy
// i's partials in the order reduceKernel sums those of a single mesh (cell, face, edge, vertex
// blocks; thread t takes every blockDim-th), so each copy's value equals its single-mesh dot
// product bit for bit.
static __global__ void __launch_bounds__(kBlock) batchReduceKernel(const double* __restrict__ partial, BatchMap bm,
                                                                   double* out) {
  const int copy = blockIdx.x;
  const int n = bm.bCount[0] + bm.bCount[1] + bm.bCount[2] + bm.bCount[3];
  double v = 0.0;
  for (int a = threadIdx.x; a < n; a += blockDim.x) {
    int k = 0, r = a;
    while (r >= bm.bCount[k]) r -= bm.bCount[k++];
    v += partial[bm.bBase[k] + copy * bm.bCount[k] + r];
  }
  const double r = blockReduce<double>(v);
  if (threadIdx.x == 0) out[copy] = r;
}

// ---------------------------------------------------------------------------------------
// Owned DoFs packed in level-buffer order (the host transfers of hg_function_*_owned_async):
// run r copies slots [slot, slot + len) of the level buffer to [packed, packed + len) of the
// packed vector (PACK) or back. One warp per run, lanes over consecutive slots.
// ---------------------------------------------------------------------------------------
struct OwnedRun {
  int64_t slot, packed;
  int len, pad;
};

template <class T, bool PACK>
__global__ void __launch_bounds__(kBlock) ownedPackKernel(const OwnedRun* __restrict__ runs, int64_t nRuns, T* buf,
                                                          T* packed) {
  const int lane = threadIdx.x & 31;
  const int64_t nWarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nRuns; r += nWarps) {
    const OwnedRun run = runs[r];
    for (int i = lane; i < run.len; i += 32) {
      if (PACK) packed[run.packed + i] = buf[run.slot + i];
      else buf[run.slot + i] = packed[run.packed + i];
    }
  }
}

}  // namespace dev
}  // namespace hg
