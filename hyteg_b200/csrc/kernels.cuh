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

namespace hg {
namespace dev {

constexpr int kBlock = 256;

struct CellBlock {
  int cell, z, start, pad;
};
struct FaceBlock {
  int face, start;
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
  const CellBlock* cellBlocks;
  int nCellBlocks;
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

// Row y of the offset `off` inside a triangular plane of width W.
__device__ __forceinline__ int decodeRow(int W, int off) {
  const float t = float(2 * W + 1);
  int y = int((t - __fsqrt_rn(t * t - 8.0f * float(off))) * 0.5f);
  y = max(y, 0);
  if (rowStart(W, y) > off) --y;
  if (rowStart(W, y + 1) <= off) ++y;
  return y;
}

// Absolute indices of the 15 stencil neighbours of the cell point with plane-local row y,
// plane width W (= w - z) and absolute index c. Order: C E W N S NW SE TC TW TS TSE BC BE BN BNW.
__device__ __forceinline__ void cellNeighbours(int64_t c, int W, int y, int64_t n[15]) {
  const int64_t up = c + triSize(W) - y;           // (x, y, z+1)
  const int64_t dn = c - triSize(W + 1) + y;       // (x, y, z-1)
  n[0] = c;
  n[1] = c + 1;
  n[2] = c - 1;
  n[3] = c + (W - y);
  n[4] = c - (W - y + 1);
  n[5] = n[3] - 1;
  n[6] = n[4] + 1;
  n[7] = up;
  n[8] = up - 1;
  n[9] = up - (W - y);
  n[10] = n[9] + 1;
  n[11] = dn;
  n[12] = dn + 1;
  n[13] = dn + (W + 1 - y);
  n[14] = n[13] - 1;
}

// ---------------------------------------------------------------------------------------
// Stencil application on cell interiors: dst = A src | dst += A src | dst = rhs - A src
// ---------------------------------------------------------------------------------------
template <class T, int MODE>
__global__ void __launch_bounds__(kBlock) cellStencilKernel(LevelDev lv, const T* __restrict__ cellW,
                                                            T* __restrict__ dst, const T* __restrict__ src,
                                                            const T* __restrict__ rhs, unsigned mask) {
  const CellBlock b = lv.cellBlocks[blockIdx.x];
  if (!(lv.cellType[b.cell] & mask)) return;
  const int W = lv.w - b.z;
  const int off = b.start + threadIdx.x;
  const int y = decodeRow(W, off);
  const int x = off - rowStart(W, y);
  if (y < 1 || x < 1 || x + y > W - 2) return;
  const int64_t c = lv.cellOff[b.cell] + (tetSize(lv.w) - tetSize(W)) + off;
  int64_t n[15];
  cellNeighbours(c, W, y, n);
  const T* wt = cellW + 16 * b.cell;
  T s = wt[0] * __ldg(src + n[0]);
#pragma unroll
  for (int k = 1; k < 15; ++k) s += wt[k] * __ldg(src + n[k]);
  if (MODE == MODE_REPLACE) dst[c] = s;
  else if (MODE == MODE_ADD) dst[c] += s;
  else dst[c] = rhs[c] - s;
}

// Multicolour SOR on cell interiors, colour = (x + 2y + 3z) mod 4.
template <class T>
__global__ void __launch_bounds__(kBlock) cellSorKernel(LevelDev lv, const T* __restrict__ cellW, T* u,
                                                        const T* __restrict__ rhs, unsigned mask, int colour,
                                                        T omega) {
  const CellBlock b = lv.cellBlocks[blockIdx.x];
  if (!(lv.cellType[b.cell] & mask)) return;
  const int W = lv.w - b.z;
  const int off = b.start + threadIdx.x;
  const int y = decodeRow(W, off);
  const int x = off - rowStart(W, y);
  if (y < 1 || x < 1 || x + y > W - 2) return;
  if (((x + 2 * y + 3 * b.z) & 3) != colour) return;
  const int64_t c = lv.cellOff[b.cell] + (tetSize(lv.w) - tetSize(W)) + off;
  int64_t n[15];
  cellNeighbours(c, W, y, n);
  const T* wt = cellW + 16 * b.cell;
  T s = rhs[c];
#pragma unroll
  for (int k = 1; k < 15; ++k) s -= wt[k] * u[n[k]];
  u[c] = (T(1) - omega) * u[c] + (s * omega) / wt[0];
}

// Full-weighting restriction at coarse cell-interior points: coarse = fine[2p] + 1/2 sum fine[2p+d]
// (restrict_3D_macrocell_P1_pull_additive.cpp; on interior points every weight is 1 or 1/2).
template <class T>
__global__ void __launch_bounds__(kBlock) cellRestrictKernel(LevelDev lc, LevelDev lf, T* __restrict__ coarse,
                                                             const T* __restrict__ fine, unsigned mask) {
  const CellBlock b = lc.cellBlocks[blockIdx.x];
  if (!(lc.cellType[b.cell] & mask)) return;
  const int W = lc.w - b.z;
  const int off = b.start + threadIdx.x;
  const int y = decodeRow(W, off);
  const int x = off - rowStart(W, y);
  if (y < 1 || x < 1 || x + y > W - 2) return;
  const int zf = 2 * b.z, yf = 2 * y, xf = 2 * x;
  const int Wf = lf.w - zf;
  const int64_t cf = lf.cellOff[b.cell] + (tetSize(lf.w) - tetSize(Wf)) + rowStart(Wf, yf) + xf;
  int64_t n[15];
  cellNeighbours(cf, Wf, yf, n);
  T s = T(0);
#pragma unroll
  for (int k = 1; k < 15; ++k) s += __ldg(fine + n[k]);
  coarse[lc.cellOff[b.cell] + (tetSize(lc.w) - tetSize(W)) + off] = __ldg(fine + n[0]) + T(0.5) * s;
}

__device__ __forceinline__ int64_t cellIndexDev(int w, int x, int y, int z) {
  const int W = w - z;
  return (tetSize(w) - tetSize(W)) + rowStart(W, y) + x;
}

// Linear prolongation at fine cell-interior points (prolongate_3D_macrocell_P1_push_additive.cpp):
// even points copy the coarse value, every other point is the mean of the two coarse end
// points of the coarse micro-edge it bisects.
template <class T, bool ADD>
__global__ void __launch_bounds__(kBlock) cellProlongKernel(LevelDev lf, LevelDev lc, T* __restrict__ fine,
                                                            const T* __restrict__ coarse, unsigned mask) {
  const CellBlock b = lf.cellBlocks[blockIdx.x];
  if (!(lf.cellType[b.cell] & mask)) return;
  const int W = lf.w - b.z;
  const int off = b.start + threadIdx.x;
  const int y = decodeRow(W, off);
  const int x = off - rowStart(W, y);
  if (y < 1 || x < 1 || x + y > W - 2) return;
  const int z = b.z;
  const int px = x & 1, py = y & 1, pz = z & 1;
  int dx = 0, dy = 0, dz = 0;
  const int code = px | (py << 1) | (pz << 2);
  switch (code) {
    case 1: dx = 1; break;
    case 2: dy = 1; break;
    case 4: dz = 1; break;
    case 3: dx = -1; dy = 1; break;
    case 5: dx = -1; dz = 1; break;
    case 6: dy = -1; dz = 1; break;
    case 7: dx = -1; dy = 1; dz = -1; break;
    default: break;
  }
  const int64_t base = lc.cellOff[b.cell];
  T v;
  if (code == 0) {
    v = __ldg(coarse + base + cellIndexDev(lc.w, x >> 1, y >> 1, z >> 1));
  } else {
    const int ax = (x - dx) >> 1, ay = (y - dy) >> 1, az = (z - dz) >> 1;
    v = T(0.5) * (__ldg(coarse + base + cellIndexDev(lc.w, ax, ay, az)) +
                  __ldg(coarse + base + cellIndexDev(lc.w, ax + dx, ay + dy, az + dz)));
  }
  const int64_t c = lf.cellOff[b.cell] + (tetSize(lf.w) - tetSize(W)) + off;
  if (ADD) fine[c] += v;
  else fine[c] = v;
}

// ---------------------------------------------------------------------------------------
// Face interiors: generic entries (layer, dx, dy, w); layer 0 is the face triangle, layer
// 1+n the ghost layer of neighbour cell n (apply_3D_macroface_one_sided_*.cpp, called once
// per neighbour cell in P1ConstantOperator.cpp:202-288, fused here into one sweep).
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ int64_t faceSlot(int w, int layer, int x, int y) {
  if (layer == 0) return rowStart(w, y) + x;
  return triSize(w) + (layer - 1) * triSize(w - 1) + rowStart(w - 1, y) + x;
}

template <class T, int MODE>
__global__ void __launch_bounds__(kBlock) faceStencilKernel(LevelDev lv, StencilDev<T> st, T* __restrict__ dst,
                                                            const T* __restrict__ src, const T* __restrict__ rhs,
                                                            unsigned mask) {
  const FaceBlock b = lv.faceBlocks[blockIdx.x];
  if (!(lv.faceType[b.face] & mask)) return;
  __shared__ FaceEnt<T> ent[16];
  const int ne = st.faceEntCount[b.face];
  if (threadIdx.x < ne) ent[threadIdx.x] = st.faceEnt[16 * b.face + threadIdx.x];
  __syncthreads();
  const int w = lv.w;
  const int off = b.start + threadIdx.x;
  const int y = decodeRow(w, off);
  const int x = off - rowStart(w, y);
  if (y < 1 || x < 1 || x + y > w - 2) return;
  const int64_t base = lv.faceOff[b.face];
  T s = T(0);
  for (int k = 0; k < ne; ++k) s += ent[k].w * __ldg(src + base + faceSlot(w, ent[k].layer, x + ent[k].dx, y + ent[k].dy));
  const int64_t c = base + off;
  if (MODE == MODE_REPLACE) dst[c] = s;
  else if (MODE == MODE_ADD) dst[c] += s;
  else dst[c] = rhs[c] - s;
}

// Face SOR, colour = (x + 2y) mod 3; entry 0 is the diagonal.
template <class T>
__global__ void __launch_bounds__(kBlock) faceSorKernel(LevelDev lv, StencilDev<T> st, T* u, const T* __restrict__ rhs,
                                                        unsigned mask, int colour, T omega) {
  const FaceBlock b = lv.faceBlocks[blockIdx.x];
  if (!(lv.faceType[b.face] & mask)) return;
  __shared__ FaceEnt<T> ent[16];
  const int ne = st.faceEntCount[b.face];
  if (threadIdx.x < ne) ent[threadIdx.x] = st.faceEnt[16 * b.face + threadIdx.x];
  __syncthreads();
  const int w = lv.w;
  const int off = b.start + threadIdx.x;
  const int y = decodeRow(w, off);
  const int x = off - rowStart(w, y);
  if (y < 1 || x < 1 || x + y > w - 2) return;
  if ((x + 2 * y) % 3 != colour) return;
  const int64_t base = lv.faceOff[b.face];
  const int64_t c = base + off;
  T s = rhs[c];
  for (int k = 1; k < ne; ++k) s -= ent[k].w * u[base + faceSlot(w, ent[k].layer, x + ent[k].dx, y + ent[k].dy)];
  u[c] = (T(1) - omega) * u[c] + (s * omega) / ent[0].w;
}

// Restriction at coarse face-interior points from the fine face and its ghost layers: the fine
// stencil structure of the face with weight 1 at the centre and 1/2 at every neighbour.
template <class T>
__global__ void __launch_bounds__(kBlock) faceRestrictKernel(LevelDev lc, LevelDev lf, StencilDev<T> stf,
                                                             T* __restrict__ coarse, const T* __restrict__ fine,
                                                             unsigned mask) {
  const FaceBlock b = lc.faceBlocks[blockIdx.x];
  if (!(lc.faceType[b.face] & mask)) return;
  __shared__ FaceEnt<T> ent[16];
  const int ne = stf.faceEntCount[b.face];
  if (threadIdx.x < ne) ent[threadIdx.x] = stf.faceEnt[16 * b.face + threadIdx.x];
  __syncthreads();
  const int w = lc.w;
  const int off = b.start + threadIdx.x;
  const int y = decodeRow(w, off);
  const int x = off - rowStart(w, y);
  if (y < 1 || x < 1 || x + y > w - 2) return;
  const int64_t basef = lf.faceOff[b.face];
  T s = T(0);
  for (int k = 1; k < ne; ++k) s += __ldg(fine + basef + faceSlot(lf.w, ent[k].layer, 2 * x + ent[k].dx, 2 * y + ent[k].dy));
  coarse[lc.faceOff[b.face] + off] = __ldg(fine + basef + faceSlot(lf.w, 0, 2 * x, 2 * y)) + T(0.5) * s;
}

template <class T, bool ADD>
__global__ void __launch_bounds__(kBlock) faceProlongKernel(LevelDev lf, LevelDev lc, T* __restrict__ fine,
                                                            const T* __restrict__ coarse, unsigned mask) {
  const FaceBlock b = lf.faceBlocks[blockIdx.x];
  if (!(lf.faceType[b.face] & mask)) return;
  const int w = lf.w;
  const int off = b.start + threadIdx.x;
  const int y = decodeRow(w, off);
  const int x = off - rowStart(w, y);
  if (y < 1 || x < 1 || x + y > w - 2) return;
  const int64_t cb = lc.faceOff[b.face];
  const int code = (x & 1) | ((y & 1) << 1);
  T v;
  if (code == 0) {
    v = __ldg(coarse + cb + rowStart(lc.w, y >> 1) + (x >> 1));
  } else {
    const int dx = code == 1 ? 1 : (code == 3 ? -1 : 0);
    const int dy = code == 1 ? 0 : 1;
    const int ax = (x - dx) >> 1, ay = (y - dy) >> 1;
    v = T(0.5) * (__ldg(coarse + cb + rowStart(lc.w, ay) + ax) + __ldg(coarse + cb + rowStart(lc.w, ay + dy) + ax + dx));
  }
  const int64_t c = lf.faceOff[b.face] + off;
  if (ADD) fine[c] += v;
  else fine[c] = v;
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
// Halo refresh: copy slots <- owner slots (one gather; every source is an owned slot).
// ---------------------------------------------------------------------------------------
template <class T>
__global__ void commGatherKernel(T* buf, const uint2* __restrict__ table, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint2 t = table[i];
    buf[t.x] = buf[t.y];
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
  if (blk < lv.nCellBlocks) {
    const CellBlock cb = lv.cellBlocks[blk];
    if (lv.cellType[cb.cell] & mask) {
      const int W = lv.w - cb.z;
      const int off = cb.start + threadIdx.x;
      const int y = decodeRow(W, off);
      const int x = off - rowStart(W, y);
      if (y >= 1 && x >= 1 && x + y <= W - 2) {
        const int64_t c = lv.cellOff[cb.cell] + (tetSize(lv.w) - tetSize(W)) + off;
        v = double(a[c]) * double(b[c]);
      }
    }
  } else if ((blk -= lv.nCellBlocks) < lv.nFaceBlocks) {
    const FaceBlock fb = lv.faceBlocks[blk];
    if (lv.faceType[fb.face] & mask) {
      const int off = fb.start + threadIdx.x;
      const int y = decodeRow(lv.w, off);
      const int x = off - rowStart(lv.w, y);
      if (y >= 1 && x >= 1 && x + y <= lv.w - 2) {
        const int64_t c = lv.faceOff[fb.face] + off;
        v = double(a[c]) * double(b[c]);
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

}  // namespace dev
}  // namespace hg
