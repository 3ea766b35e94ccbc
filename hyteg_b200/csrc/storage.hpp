// Host-side state behind an hg_storage handle (C++; not part of the C-ABI).
#pragma once

#include <cuda_runtime.h>

#include <deque>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "discretization.hpp"
#include "kernels.cuh"

namespace hg {

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf();
  void* alloc(size_t n);
};

// Order of the halo groups in a level's table: every group set one SOR phase refreshes at once
// (vertex ghosts with face ghost layers, cell closures with face boundary rows, all five) is one
// contiguous run, so a refresh is one launch.
constexpr int kCommOrder[G_COUNT] = {G_EDGE, G_VERT, G_FACE_GHOST, G_CELL, G_FACE_BOUNDARY};

struct LevelData {
  const LevelLayout* lay = nullptr;
  dev::LevelDev lv{};
  uint2* comm = nullptr;
  int64_t commBegin[G_COUNT] = {0, 0, 0, 0, 0}, commCount[G_COUNT] = {0, 0, 0, 0, 0};
  dev::Chunk* chunks = nullptr;
  int nChunks = 0;
  int nCellChunks = 0;  // the chunks of the cell arrays come first
  // register-blocked cell sweep: work items grouped by macro-cell groups small enough to stay in L2
  dev::StripItem* tiles = nullptr;
  int nTiles = 0;
  std::vector<int> tileGroupBegin;  // group g: items [tileGroupBegin[g], tileGroupBegin[g + 1])
  int cellsPerGroup = 0;
  std::unique_ptr<DevBuf> tileBuf;
  DevBuf partial;
  // single-pass SOR: one 32 x 32 (x, y) tile of a macro-cell per block, the tallest first
  // single-pass SOR tiles per [precision: 0 FP64, 1 FP32][tile geometry: 0, 1]
  dev::WaveTile* waveTiles[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  int nWaveTiles[2][2] = {{0, 0}, {0, 0}};
  int64_t nonCellBegin = 0;  // first slot after the cell arrays (faces, edges, vertices follow)
  // per primitive, its entries (begin, end) in comm of the group the SOR refreshes before its
  // phase: low primitives (edges: G_EDGE, vertices: G_VERT), faces (G_FACE_BOUNDARY)
  const int2* lowRange = nullptr;
  const int2* faceRange = nullptr;
  // SOR schedule 3 (built on first use): the halo table with every cell slot at its colour-split
  // position (same groups as comm), and per colour the rows and points of the cell interiors
  const uint2* commSplit = nullptr;
  const dev::SplitRow* splitRows[4] = {nullptr, nullptr, nullptr, nullptr};
  const unsigned* splitPoints[4] = {nullptr, nullptr, nullptr, nullptr};
  int nSplitPoints[4] = {0, 0, 0, 0};
  std::vector<unsigned char> hostCellType, hostFaceType, hostLowType;
  std::vector<std::unique_ptr<DevBuf>> keep;
};

// Staging of a function's owned DoFs on one level for the packed host transfers. copied is
// recorded on the copy stream after each host copy, used on the storage's stream after each pack
// or unpack: every use of the buffer waits for the previous one on the other stream.
struct PackStage {
  DevBuf buf;
  cudaEvent_t copied = nullptr, used = nullptr;
  PackStage() = default;
  PackStage(const PackStage&) = delete;
  PackStage& operator=(const PackStage&) = delete;
  ~PackStage();
};

struct Function {
  int minL = 0, maxL = 0, prec = 8;
  std::vector<std::unique_ptr<DevBuf>> levels;
  std::map<int, std::unique_ptr<PackStage>> stage;  // level -> staging of the packed transfers
};

// The owned-DoF runs of one level on the device (dev::OwnedRun), built on first use.
struct OwnedPack {
  DevBuf runs;
  int64_t nRuns = 0, count = 0;
};

struct Operator {
  int form = 0, minL = 0, maxL = 0;
  std::vector<LevelStencils> host;
  std::vector<dev::StencilDev<double>> d;
  std::vector<dev::StencilDev<float>> f;
  std::vector<std::unique_ptr<DevBuf>> keep;
  // Device re-assembly (the diffusion form): per level the terms of every stencil entry, built
  // on first use. After a device re-assembly the host copy holds the previous coefficients'
  // values (hostStale): its structure and the signs of its diagonals still hold, and
  // p1Diagonal re-assembles it before reading values.
  struct DevPlan {
    const int64_t* first = nullptr;
    const dev::PlanTermDev* terms = nullptr;
    int64_t nCell = 0, nFace = 0, nLow = 0;
  };
  std::vector<DevPlan> plans;
  DevBuf coef;  // [cells] coefficients of the last device re-assembly
  bool hostStale = false;
};

// P2 operator: element matrices of the six micro-cell types per macro-cell and level.
struct P2Operator {
  int form = 0, minL = 0, maxL = 0;
  std::vector<std::unique_ptr<DevBuf>> kd, kf;  // per level: [cell][type][10][10] in FP64 / FP32
  std::map<std::pair<int, int>, int> diag;      // (level, precision) -> diagonal function
  std::vector<std::unique_ptr<DevBuf>> dd, df;  // Taylor-Hood divergence per level: [cell][type][3][4][10]
  std::vector<std::unique_ptr<DevBuf>> sd, sf;  // interior stencils per level: [cell][p2s::kTotal]
  std::vector<std::unique_ptr<DevBuf>> fd, ff;  // face-interior stencils per level: [cell][p2s::kFaceTotal]
  // Taylor-Hood coupling at interior nodes per level, [cell][component][65]: div (offsets p2s::S0 on
  // the velocity lattice) and divT (offsets p2s::DivTList per velocity class on the pressure lattice)
  std::vector<std::unique_ptr<DevBuf>> wdivd, wdivf, wdivtd, wdivtf;
};

// Cell-closure copies of every DoF owned by a face, edge or vertex of one lattice level.
struct P2Additive {
  bool built = false;
  int n = 0;
  DevBuf owner, ptr, copies, type;
  DevBuf colour;  // per slot: SOR colour of the DoF (0..10), bit 7 on its owner slot
  DevBuf mult;    // per slot: number of macro-cells holding the DoF (1 for cell-owned)
  DevBuf classOfColour;  // per cell: [0..10] parity class of colour k's interior nodes (or -1), [11] vertex colour step
  DevBuf updAdd;                            // owner-table indices of the face/edge/vertex DoFs by colour
  int updAddBegin[12] = {0};
  DevBuf updInner, updInnerType;            // interior vertex slots (and their cell's type) by colour
  int updInnerBegin[12] = {0};
  DevBuf closureList;                       // closure nodes of the cells (dev::P2ClosureNode) by colour
  int closureBegin[12] = {0};               // first entry of colour k; closureBegin[11] = total
  std::vector<int64_t> hostOwner;           // the owner slot of every DoF (levels up to 2^20 slots)
  std::vector<unsigned char> hostOwnerType;  // and its DoF type
};

// Candidate micro-cells and coarse P2 basis values for the fine nodes of the 64 residue classes
// (device tables, and their host copies for building the restriction's gather lists).
struct P2Transfer {
  bool built = false;
  DevBuf nCand, cand, wd, wf;
  std::vector<unsigned char> hNCand, hCand;
  std::vector<double> hW;
};

// The P2 restriction as a gather (the transpose of the quadratic prolongation of one macro-cell,
// the same for every cell): for each coarse node of the closed reference cell, its contributing
// fine nodes and weights in a fixed order (compressed rows: ptr[nCoarse + 1], then the entries).
struct P2Gather {
  bool built = false;
  int nCoarse = 0;
  DevBuf ptr, idx, wd, wf;  // row starts; int32 fine local index; FP64 / FP32 weight
};

struct Gmg;
struct P2Gmg;
struct StokesGmg;

struct Storage {
  Storage(const Topology& topo, int maxLevel);
  ~Storage();
  int maxLevel() const { return disc.maxLevel(); }

  Discretization disc;
  int device = 0;                       // CUDA device current at creation; owns stream and buffers
  double* noallocScratch = nullptr;     // device address of hg_dot_noalloc's static scratch on `device`
  cudaStream_t ownStream = nullptr;
  cudaStream_t stream = nullptr;
  std::deque<LevelData> levels;
  std::map<int, std::unique_ptr<Function>> fns;
  std::map<int, std::unique_ptr<Operator>> ops;
  std::map<int, std::unique_ptr<Gmg>> gmgs;
  std::map<int, std::unique_ptr<P2Operator>> p2ops;
  std::map<int, std::unique_ptr<P2Gmg>> p2gmgs;
  std::map<int, std::unique_ptr<StokesGmg>> stokesGmgs;
  std::deque<P2Additive> p2add;  // per lattice level
  int nextId = 1;
  int structureOp = -1;
  DevBuf scalars;            // device scratch for reductions
  int64_t l2Budget = int64_t(1) << 62;  // bytes of L2 one SOR cell group may occupy (default: one group)
  unsigned long long launches = 0;  // kernels launched by this storage
  // Cell-phase schedule of the multicolour SOR: 0 = one wavefront pass that writes a second
  // buffer which then replaces the level buffer, 1 = four in-place colour passes, 2 = the
  // wavefront pass with the shorter tile geometry, 3 = four colour passes on a copy of the
  // cell arrays in the colour-split order (converted once per group of sweeps).
  int sorSchedule = 0;
  // Face, edge and vertex phases of the SOR: one launch per phase with the refresh of each
  // primitive's copies folded in (1, default), or one launch per colour and per refresh (0).
  int fusedSorPhases = 1;
  std::vector<int> sorScheduleLevel;  // [2 L + (FP32 ? 1 : 0)]: schedule chosen by autotuneSor (-1: sorSchedule)
  int sorScheduleFor(int L, int prec) const;
  // Times the four schedules of the SOR on levels [minL, maxL] in the given precision, in groups
  // of three sweeps (the smoothing of a V(3,3) cycle), and keeps the fastest per level;
  // ms[4 * (L - minL) + s] receives the time per sweep (nullable).
  void autotuneSor(int minL, int maxL, int prec, int reps, double* ms);
  unsigned long long generation = 0;  // bumped when level tables or schedules change (captured graphs)
  std::map<std::pair<int, int>, std::unique_ptr<DevBuf>> spare;  // (level, precision) -> buffer
  std::map<int, std::unique_ptr<OwnedPack>> ownedPacks;           // level -> owned-DoF runs
  const OwnedPack& ownedPack(int L);
  // Packed host transfers of a function's owned DoFs (level-buffer order, ownedRuns): the host
  // copy runs on copyStream, the pack / unpack on the storage's stream, ordered by events; an
  // upload ends with a full halo refresh.
  void uploadOwned(int id, int L, const void* host, int64_t n, cudaStream_t copyStream);
  void downloadOwned(int id, int L, void* host, int64_t n, cudaStream_t copyStream);
  std::map<std::pair<int, int>, std::unique_ptr<DevBuf>> splitRhs;  // (level, precision) -> split rhs copy
  DevBuf& spareBuf(std::map<std::pair<int, int>, std::unique_ptr<DevBuf>>& pool, int L, int prec);
  void buildSplit(int L);  // the schedule-3 tables of level L (no-op once built)
  dev::Geometry geom{};              // macro-vertex coordinates and primitive vertex lists (device)
  std::vector<std::unique_ptr<DevBuf>> geomKeep;

  Function& fn(int id);
  void* data(int id, int L);
  int createFunction(int minL, int maxL, int prec);
  // Refresh the copy slots of the selected groups (bit (1 << CommGroup)) from their owners.
  void communicate(int id, int L, int groupMask);
  void lincomb(int dst, int L, unsigned mask, int n, const double* a, const int* srcs, bool add, double constant);
  void copyCast(int dst, int src, int L, unsigned mask, bool add);
  // dst = a / b elementwise on the flagged primitives' slots (FP64)
  void divideBy(int dst, int a, int b, int L, unsigned mask);
  void dotAsync(int a, int b, int L, unsigned mask, double* dOut);
  // Batched solves on a storage of `copies` disjoint copies of one macro-mesh (meshCuboidCopies):
  // the map of level L (checked against the layout), the right-hand sides of the first `active`
  // copies from their seeds (device array; the others 0), the dot product of every copy
  // (dOut[copies], device), and the copy of one copy's slots of level L from src to dst.
  dev::BatchMap batchMap(int L, int copies) const;
  void fillRandomBatch(int id, int L, unsigned mask, const dev::BatchMap& bm, const uint64_t* dSeeds, int active,
                       double lo, double hi);
  void dotBatchAsync(int a, int b, int L, unsigned mask, const dev::BatchMap& bm, double* dOut);
  void copyBatchSlots(int src, int dst, int L, const dev::BatchMap& bm, int copy);
  void interpolateExpr(int id, int L, unsigned mask, int expr, const double* params);
  // Seeded uniform [lo, hi) values at the flagged primitives' DoFs, then a full halo refresh.
  void fillRandom(int id, int L, unsigned mask, uint64_t seed, double lo, double hi);
  // Device memory held by this storage (level tables, functions, operators, spare buffers).
  int64_t deviceBytes() const;
  double dot(int a, int b, int L, unsigned mask);

  int createOperator(int form, int minL, int maxL);
  // P2 operators on levels [minL, maxL]; the P2 DoFs of level L are the vertex DoFs of level L+1.
  int createP2Operator(int form, int minL, int maxL);
  // dst = A2 src (mode 0) or dst = rhs - A2 src (mode 2) at the flagged DoFs of P2 level L.
  void p2Apply(int op, int src, int dst, int rhs, int L, unsigned mask, int mode);
  // Multicolour SOR on P2 level L (11 colours; each pass updates one colour from the values
  // at the start of the pass).
  void p2Sor(int op, int x, int b, double omega, int L, unsigned mask, bool backwards);
  P2Operator& p2op(int id);
  P2Additive& p2Additive(int Lf);
  int p2Diagonal(int op, int L, int prec);
  std::map<std::pair<int, int>, int> p2scratch;  // (lattice level, precision key) -> scratch function
  // Lane of the P2 work being issued: P2 cycles that run concurrently on different streams use
  // different lanes, and every lane has its own P2 scratch functions.
  int p2Lane = 0;
  std::pair<int, int> p2ScratchKey(int Lf, int prec) const { return {Lf, prec + 64 * p2Lane}; }
  // Whether the Stokes MINRES preconditioner runs its three velocity V-cycles concurrently, one
  // stream each (default on; the iterates are the same either way).
  bool concurrentComponents = true;
  P2Transfer p2tr;
  std::map<int, P2Gather> p2gather;  // by fine lattice level
  const P2Gather& p2Gather(int Lff);
  // Quadratic prolongation from P2 level Lc to Lc + 1 of function id (fine = P coarse, or += with
  // add) and its transpose, the restriction from P2 level Lf to Lf - 1.
  void p2Prolongate(int id, int Lc, unsigned mask, bool add);
  void p2Restrict(int id, int Lf, unsigned mask);
  // P2-P1 Taylor-Hood Stokes (P2P1TaylorHoodStokesOperator): velocity P2 functions u[3], v[3],
  // pressure P1 functions p, q (level L of the pressure = P2 level L):
  //   v_k = A u_k + D_k^T p   (velocity DoFs flagged by maskV)
  //   q   = sum_k D_k u_k     (pressure DoFs flagged by maskP)
  int createStokesOperator(int minL, int maxL);
  void stokesApply(int op, const int u[3], int p, const int v[3], int q, int L, unsigned maskV, unsigned maskP);
  // the coupling blocks alone: v_k = D_k^T p (v_k += with add), q = sum_k D_k u_k
  void stokesDivT(int op, int p, const int v[3], int L, unsigned maskV, bool add);
  void stokesDiv(int op, const int u[3], int q, int L, unsigned maskP);
  // Diagonal of a P1 operator on level L (the stencil centre of each primitive's DoFs) as a new
  // FP64 function of that level, owned by the caller.
  int p1Diagonal(int op, int L);
  int p2Scratch(int Lf, int prec);
  template <class T, int MODE>
  void p2Launch(P2Operator& o, int L, T* dst, const T* src, const T* rhs, unsigned mask, int sel);
  template <class T>
  void p2SorT(P2Operator& o, int opId, int x, int b, int L, unsigned mask, T omega, bool backwards);
  // Re-assemble an operator's stencils from the current cell coefficients into its device
  // arrays: on the host (assembly, upload), or on the device from the per-entry term lists (the
  // same bits; forms without coefficients are left as they are).
  void reassembleOperator(int id, bool onDevice = false);
  Operator& op(int id);
  void apply(int op, int src, int dst, int L, unsigned mask, int update, int kinds = 15, bool refresh = true);
  void residual(int op, int x, int b, int r, int L, unsigned mask);
  void smoothSor(int op, int dst, int rhs, double omega, int L, unsigned mask, bool backwards, int kinds = 15,
                 bool refresh = true);
  // `sweeps` SOR sweeps in a row. Under schedule 3 the cell arrays of dst (and of rhs, unless
  // rhsReady: rhs is unchanged since the last group of sweeps on this level and precision) are
  // converted into the colour-split order once, and dst is converted back after the last sweep.
  void smoothSorSweeps(int op, int dst, int rhs, double omega, int L, unsigned mask, int sweeps, bool backwards,
                       bool rhsReady);
  // Restriction of id's level Lf to level Lf - 1 of id, or of coarseDst (>= 0) when given.
  void restrictFn(int id, int Lf, unsigned mask, int coarseDst = -1);
  void prolongate(int id, int Lc, unsigned mask, bool add);
  const Operator& structure();

  template <class T, int MODE>
  void stencilOp(Operator& o, int L, T* dst, const T* src, const T* rhs, unsigned mask, int kinds = 15);
  // cellU / cellF (nullable): the level's cell arrays of u and rhs in the colour-split order
  template <class T>
  void sorT(Operator& o, int dstId, int L, T* u, const T* rhs, unsigned mask, T omega, bool backwards, int kinds,
            bool refresh, T* cellU = nullptr, const T* cellF = nullptr);
  template <class T>
  void communicateSplit(T* buf, T* cells, int L, int groupMask);
  template <class T>
  void restrictT(int id, int Lf, unsigned mask, int coarseDst);
  template <class T>
  void prolongT(int id, int Lc, unsigned mask, bool add);

 void setL2Budget(int64_t bytes);

 private:
  void buildLevel(int L);
  void buildTiles(int L);
};

// Schedule-3 interior rows and points of colour col of a closed macro-cell with w points per edge
// (storage.cu); shared by the device tables and their host check.
void splitTables(int64_t w, int col, std::vector<dev::SplitRow>& rows, std::vector<unsigned>& points);

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
void cudaCheck(cudaError_t e, const char* what);
void argCheck(bool ok, const std::string& msg);
extern thread_local std::string g_lastError;

}  // namespace hg

// Opaque handle of the C-ABI (include/hyteg_b200.h).
struct hg_storage {
  hg::Storage* s;
};
