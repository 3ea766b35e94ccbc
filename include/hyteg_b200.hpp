// C++ classes over the C-ABI of hyteg_b200.h with the reference's class names and member
// signatures, so that code written against HyTeG's P1 multigrid path compiles against this
// header with a namespace change. Header-only; link against libhyteg_b200.so.
//
// Replaced reference interfaces (paths within wagnandr/hyteg):
//   PrimitiveStorage            std::shared_ptr<PrimitiveStorage> built from MeshInfo +
//                               SetupPrimitiveStorage + setMeshBoundaryFlagsOnBoundary(1, 0, true)
//                               (primitivestorage/SetupPrimitiveStorage.cpp:37, mesh/MeshGenCuboid.cpp:32)
//   P1Function                  P1Function<real_t>(name, storage, minLevel, maxLevel), interpolate,
//                               assign, add, dotGlobal, communicate
//                               (p1functionspace/VertexDoFFunction.hpp:66-77, 162-391)
//   P1ConstantLaplaceOperator   P1ConstantOperator<P1FenicsForm<p1_diffusion, p1_tet_diffusion>>
//   P1ConstantMassOperator      (p1functionspace/P1ConstantOperator.hpp:165-166):
//                               apply(src, dst, level, flag, updateType) (operators/Operator.hpp:73-80),
//                               smooth_sor / smooth_sor_backwards / smooth_gs (solvers/Smoothables.hpp:63-91)
//   P1toP1LinearRestriction     restrict(function, sourceLevel, flag)
//                               (gridtransferoperators/RestrictionOperator.hpp:32)
//   P1toP1LinearProlongation    prolongate / prolongateAndAdd (gridtransferoperators/ProlongationOperator.hpp:33-35)
//   SORSmoother, CGSolver,      solve(A, x, b, level) (solvers/Solver.hpp:30, SORSmoother.hpp:29-56,
//   GeometricMultigridSolver    CGSolver.hpp:42-67, GeometricMultigridSolver.hpp:42-116)
//
// Errors: every call whose C status is not HG_OK throws std::runtime_error with hg_last_error(),
// where the reference aborts (WALBERLA_ABORT / WALBERLA_CHECK) or throws std::runtime_error.
// Smoothing is multicolour SOR on the GPU (hg_smooth_sor). Objects hold a shared_ptr to their
// storage, so the storage outlives them; one storage is not thread-safe.
#ifndef HYTEG_B200_HPP
#define HYTEG_B200_HPP

#include <algorithm>
#include <array>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "hyteg_b200.h"

namespace hyteg_b200 {

using real_t = double;
using uint_t = std::size_t;

// types/types.hpp:35-44
enum DoFType : unsigned {
  Inner = HG_INNER,
  DirichletBoundary = HG_DIRICHLET,
  NeumannBoundary = HG_NEUMANN,
  FreeslipBoundary = HG_FREESLIP,
  All = HG_ALL
};
inline DoFType operator|(DoFType a, DoFType b) { return DoFType(unsigned(a) | unsigned(b)); }

// operators/Operator.hpp: UpdateType
enum UpdateType { Replace = 0, Add = 1 };

inline void check(int status) {
  if (status != HG_OK) throw std::runtime_error(hg_last_error());
}

class PrimitiveStorage {
 public:
  // MeshInfo::meshCuboid(lo, hi, nx, ny, nz) (6 tetrahedra per sub-cube); levels 0 .. maxLevel
  static std::shared_ptr<PrimitiveStorage> cuboid(const std::array<real_t, 3>& lo, const std::array<real_t, 3>& hi,
                                                  int nx, int ny, int nz, uint_t maxLevel) {
    hg_storage* s = nullptr;
    check(hg_storage_create_cuboid(lo.data(), hi.data(), nx, ny, nz, (int)maxLevel, &s));
    return std::shared_ptr<PrimitiveStorage>(new PrimitiveStorage(s, maxLevel));
  }
  // an explicit macro-mesh: coords[3 * nverts], tets[4 * ncells] in cell-frame order
  static std::shared_ptr<PrimitiveStorage> fromTets(const std::vector<real_t>& coords, const std::vector<int>& tets,
                                                    uint_t maxLevel) {
    hg_storage* s = nullptr;
    check(hg_storage_create_tets((int)(coords.size() / 3), coords.data(), (int)(tets.size() / 4), tets.data(),
                                 (int)maxLevel, &s));
    return std::shared_ptr<PrimitiveStorage>(new PrimitiveStorage(s, maxLevel));
  }
  // MeshInfo::fromGmshFile(path) with the boundary flags set from the geometry
  static std::shared_ptr<PrimitiveStorage> fromGmshFile(const std::string& path, uint_t maxLevel) {
    hg_storage* s = nullptr;
    check(hg_storage_create_gmsh(path.c_str(), (int)maxLevel, 0, &s));
    return std::shared_ptr<PrimitiveStorage>(new PrimitiveStorage(s, maxLevel));
  }
  ~PrimitiveStorage() { hg_storage_destroy(s_); }
  PrimitiveStorage(const PrimitiveStorage&) = delete;
  PrimitiveStorage& operator=(const PrimitiveStorage&) = delete;

  hg_storage* handle() const { return s_; }
  uint_t maxLevel() const { return maxLevel_; }
  std::array<int, 4> counts() const {  // vertices, edges, faces, cells
    std::array<int, 4> c{};
    check(hg_storage_counts(s_, c.data()));
    return c;
  }
  int64_t levelSize(uint_t level) const {
    int64_t n = 0;
    check(hg_level_size(s_, (int)level, &n));
    return n;
  }
  void synchronize() const { check(hg_storage_synchronize(s_)); }

 private:
  PrimitiveStorage(hg_storage* s, uint_t maxLevel) : s_(s), maxLevel_(maxLevel) {}
  hg_storage* s_;
  uint_t maxLevel_;
};

class P1Function {
 public:
  P1Function(const std::string& name, const std::shared_ptr<PrimitiveStorage>& storage, uint_t minLevel,
             uint_t maxLevel)
      : name_(name), storage_(storage), minLevel_(minLevel), maxLevel_(maxLevel) {
    check(hg_function_create(storage_->handle(), (int)minLevel, (int)maxLevel, 8, &id_));
  }
  ~P1Function() { hg_function_destroy(storage_->handle(), id_); }
  P1Function(const P1Function&) = delete;
  P1Function& operator=(const P1Function&) = delete;

  int id() const { return id_; }
  const std::string& getFunctionName() const { return name_; }
  const std::shared_ptr<PrimitiveStorage>& getStorage() const { return storage_; }
  uint_t getMinLevel() const { return minLevel_; }
  uint_t getMaxLevel() const { return maxLevel_; }

  void interpolate(real_t constant, uint_t level, DoFType flag = All) const {
    check(hg_interpolate_const(h(), id_, constant, (int)level, flag));
  }
  void assign(const std::vector<real_t>& scalars, const std::vector<std::reference_wrapper<const P1Function>>& functions,
              uint_t level, DoFType flag = All) const {
    check(hg_assign(h(), id_, (int)level, flag, (int)functions.size(), scalars.data(), ids(functions).data()));
  }
  void add(const std::vector<real_t>& scalars, const std::vector<std::reference_wrapper<const P1Function>>& functions,
           uint_t level, DoFType flag = All) const {
    check(hg_add(h(), id_, (int)level, flag, (int)functions.size(), scalars.data(), ids(functions).data()));
  }
  real_t dotGlobal(const P1Function& rhs, uint_t level, DoFType flag = All) const {
    real_t out = 0;
    check(hg_dot(h(), id_, rhs.id_, (int)level, flag, &out));
    return out;
  }
  // communicate<Vertex, Edge>, <Edge, Face>, <Face, Cell> and back: every copy slot from its owner
  void communicate(uint_t level) const { check(hg_communicate(h(), id_, (int)level)); }
  // uniform [lo, hi) values at the flagged DoFs from a seed (no counterpart in the reference)
  void fillRandom(uint64_t seed, uint_t level, DoFType flag = All, real_t lo = -1.0, real_t hi = 1.0) const {
    check(hg_function_fill_random(h(), id_, (int)level, flag, seed, lo, hi));
  }
  // The level buffer in the reference's per-primitive layout (one FunctionMemory per primitive,
  // placed at hg_primitive_layout offsets): host copies in and out.
  std::vector<real_t> download(uint_t level) const {
    std::vector<real_t> v((size_t)storage_->levelSize(level));
    check(hg_function_download(h(), id_, (int)level, v.data(), (int64_t)v.size()));
    return v;
  }
  void upload(uint_t level, const std::vector<real_t>& v) const {
    check(hg_function_upload(h(), id_, (int)level, v.data(), (int64_t)v.size()));
  }
  // Every DoF of the level once, packed in level-buffer order (no counterpart in the reference):
  // asynchronous copies on the caller's CUDA stream (a cudaStream_t); the host buffer, pinned for
  // an asynchronous copy, must stay alive until the stream has passed the copy.
  int64_t ownedCount(uint_t level) const {
    int64_t n = 0;
    check(hg_owned_count(h(), (int)level, &n));
    return n;
  }
  void uploadOwnedAsync(uint_t level, const real_t* host, int64_t n, void* stream) const {
    check(hg_function_upload_owned_async(h(), id_, (int)level, host, n, stream));
  }
  void downloadOwnedAsync(uint_t level, real_t* host, int64_t n, void* stream) const {
    check(hg_function_download_owned_async(h(), id_, (int)level, host, n, stream));
  }

 private:
  hg_storage* h() const { return storage_->handle(); }
  static std::vector<int> ids(const std::vector<std::reference_wrapper<const P1Function>>& fs) {
    std::vector<int> v;
    for (const P1Function& f : fs) v.push_back(f.id_);
    return v;
  }
  std::string name_;
  std::shared_ptr<PrimitiveStorage> storage_;
  uint_t minLevel_, maxLevel_;
  int id_ = -1;
};

// P1ConstantOperator with a constant stencil per macro-primitive and level (form 0: Laplace,
// 1: mass).
class P1ConstantOperator {
 public:
  P1ConstantOperator(const std::shared_ptr<PrimitiveStorage>& storage, uint_t minLevel, uint_t maxLevel, int form)
      : storage_(storage), minLevel_(minLevel), maxLevel_(maxLevel) {
    check(hg_operator_create(storage_->handle(), form, (int)minLevel, (int)maxLevel, &id_));
  }
  virtual ~P1ConstantOperator() { hg_operator_destroy(storage_->handle(), id_); }
  P1ConstantOperator(const P1ConstantOperator&) = delete;
  P1ConstantOperator& operator=(const P1ConstantOperator&) = delete;

  int id() const { return id_; }
  const std::shared_ptr<PrimitiveStorage>& getStorage() const { return storage_; }
  uint_t getMinLevel() const { return minLevel_; }
  uint_t getMaxLevel() const { return maxLevel_; }

  void apply(const P1Function& src, const P1Function& dst, uint_t level, DoFType flag,
             UpdateType updateType = Replace) const {
    check(hg_apply(h(), id_, src.id(), dst.id(), (int)level, flag, updateType == Add ? 1 : 0));
  }
  void smooth_sor(const P1Function& dst, const P1Function& rhs, real_t relax, uint_t level, DoFType flag) const {
    check(hg_smooth_sor(h(), id_, dst.id(), rhs.id(), relax, (int)level, flag, 0));
  }
  void smooth_sor_backwards(const P1Function& dst, const P1Function& rhs, real_t relax, uint_t level,
                            DoFType flag) const {
    check(hg_smooth_sor(h(), id_, dst.id(), rhs.id(), relax, (int)level, flag, 1));
  }
  void smooth_gs(const P1Function& dst, const P1Function& rhs, uint_t level, DoFType flag) const {
    smooth_sor(dst, rhs, 1.0, level, flag);
  }

 private:
  hg_storage* h() const { return storage_->handle(); }
  std::shared_ptr<PrimitiveStorage> storage_;
  uint_t minLevel_, maxLevel_;
  int id_ = -1;
};

class P1ConstantLaplaceOperator : public P1ConstantOperator {
 public:
  P1ConstantLaplaceOperator(const std::shared_ptr<PrimitiveStorage>& storage, uint_t minLevel, uint_t maxLevel)
      : P1ConstantOperator(storage, minLevel, maxLevel, 0) {}
};

class P1ConstantMassOperator : public P1ConstantOperator {
 public:
  P1ConstantMassOperator(const std::shared_ptr<PrimitiveStorage>& storage, uint_t minLevel, uint_t maxLevel)
      : P1ConstantOperator(storage, minLevel, maxLevel, 1) {}
};

class P1toP1LinearRestriction {
 public:
  void restrict(const P1Function& function, const uint_t& sourceLevel, const DoFType& flag) const {
    check(hg_restrict(function.getStorage()->handle(), function.id(), (int)sourceLevel, flag));
  }
};

class P1toP1LinearProlongation {
 public:
  void prolongate(const P1Function& function, const uint_t& sourceLevel, const DoFType& flag) const {
    check(hg_prolongate(function.getStorage()->handle(), function.id(), (int)sourceLevel, flag, 0));
  }
  void prolongateAndAdd(const P1Function& function, const uint_t& sourceLevel, const DoFType& flag) const {
    check(hg_prolongate(function.getStorage()->handle(), function.id(), (int)sourceLevel, flag, 1));
  }
};

// SORSmoother<OperatorType>(relax): smooth_sor with flag Inner | NeumannBoundary
class SORSmoother {
 public:
  explicit SORSmoother(real_t relax) : relax_(relax) {}
  void solve(const P1ConstantOperator& A, const P1Function& x, const P1Function& b, uint_t level) const {
    A.smooth_sor(x, b, relax_, level, Inner | NeumannBoundary);
  }
  real_t relax() const { return relax_; }

 private:
  real_t relax_;
};

// CGSolver<OperatorType>(storage, minLevel, maxLevel, maxIter, tolerance): stops when the
// residual norm drops below the tolerance
class CGSolver {
 public:
  CGSolver(const std::shared_ptr<PrimitiveStorage>& storage, uint_t minLevel, uint_t maxLevel,
           uint_t maxIter = std::numeric_limits<int>::max(), real_t tolerance = 1e-16)
      : storage_(storage), minLevel_(minLevel), maxLevel_(maxLevel), maxIter_(maxIter), tolerance_(tolerance) {}
  void solve(const P1ConstantOperator& A, const P1Function& x, const P1Function& b, uint_t level) const {
    int it = 0;
    double res = 0;
    check(hg_cg_solve(storage_->handle(), A.id(), x.id(), b.id(), (int)level, (int)maxIter_, tolerance_, &it, &res));
  }
  uint_t maxIter() const { return maxIter_; }
  real_t tolerance() const { return tolerance_; }

 private:
  std::shared_ptr<PrimitiveStorage> storage_;
  uint_t minLevel_, maxLevel_, maxIter_;
  real_t tolerance_;
};

// GeometricMultigridSolver<OperatorType>: V(pre, post) cycles with the SOR smoother, linear
// transfers and CG on minLevel. The device solver is bound to an operator, so one is created for
// each operator the solver is used with.
class GeometricMultigridSolver {
 public:
  GeometricMultigridSolver(const std::shared_ptr<PrimitiveStorage>& storage, std::shared_ptr<SORSmoother> smoother,
                           std::shared_ptr<CGSolver> coarseSolver,
                           std::shared_ptr<P1toP1LinearRestriction> restrictionOperator,
                           std::shared_ptr<P1toP1LinearProlongation> prolongationOperator, uint_t minLevel,
                           uint_t maxLevel, uint_t preSmoothSteps = 3, uint_t postSmoothSteps = 3)
      : storage_(storage), smoother_(std::move(smoother)), coarse_(std::move(coarseSolver)),
        restriction_(std::move(restrictionOperator)), prolongation_(std::move(prolongationOperator)),
        minLevel_(minLevel), maxLevel_(maxLevel), pre_(preSmoothSteps), post_(postSmoothSteps) {
    if (!smoother_ || !coarse_ || !restriction_ || !prolongation_)
      throw std::runtime_error("GeometricMultigridSolver: null smoother, coarse solver or transfer operator");
  }
  ~GeometricMultigridSolver() {
    for (auto& e : gmg_) hg_gmg_destroy(storage_->handle(), e.second);
  }
  GeometricMultigridSolver(const GeometricMultigridSolver&) = delete;
  GeometricMultigridSolver& operator=(const GeometricMultigridSolver&) = delete;

  // one cycle: x <- MG(x, b) on `level` (= maxLevel)
  void solve(const P1ConstantOperator& A, const P1Function& x, const P1Function& b, uint_t level) {
    check(hg_gmg_solve(storage_->handle(), handle(A), x.id(), b.id(), (int)level));
  }

 private:
  int handle(const P1ConstantOperator& A) {
    auto it = gmg_.find(A.id());
    if (it != gmg_.end()) return it->second;
    int g = -1;
    check(hg_gmg_create(storage_->handle(), A.id(), (int)minLevel_, (int)maxLevel_, (int)pre_, (int)post_,
                        smoother_->relax(), 0, (int)std::min<uint_t>(coarse_->maxIter(), std::numeric_limits<int>::max()),
                        coarse_->tolerance(), 8, &g));
    gmg_[A.id()] = g;
    return g;
  }
  std::shared_ptr<PrimitiveStorage> storage_;
  std::shared_ptr<SORSmoother> smoother_;
  std::shared_ptr<CGSolver> coarse_;
  std::shared_ptr<P1toP1LinearRestriction> restriction_;
  std::shared_ptr<P1toP1LinearProlongation> prolongation_;
  uint_t minLevel_, maxLevel_, pre_, post_;
  std::map<int, int> gmg_;
};

}  // namespace hyteg_b200

#endif  // HYTEG_B200_HPP
