// CG and geometric multigrid drivers on top of the device kernels (host orchestration; all
// vector work stays on the device, only convergence scalars are read back).
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "../../include/hyteg_b200.h"
#include "compact.hpp"
#include "solvers.hpp"
#include "storage.hpp"

namespace hg {

// CGSolver::solve (src/hyteg/solvers/CGSolver.hpp:69-150) with the identity preconditioner
// (solvers/preconditioners/IdentityPreconditioner.hpp:39-45): z = r.
int cgSolve(Storage& s, int op, int x, int b, int L, int maxIter, double tol, int p, int z, int ap, int r,
            double* finalRes) {
  const unsigned flag = HG_INNER | HG_NEUMANN | HG_FREESLIP;
  const double one = 1.0;
  if (finalRes) *finalRes = 0.0;
  if (maxIter == 0) return 0;
  s.apply(op, x, p, L, flag, 0);
  {
    const double sc[2] = {1.0, -1.0};
    const int src[2] = {b, p};
    s.lincomb(r, L, flag, 2, sc, src, false, 0.0);
  }
  s.lincomb(z, L, flag, 1, &one, &r, false, 0.0);
  s.lincomb(p, L, flag, 1, &one, &z, false, 0.0);
  double prsold = s.dot(r, z, L, flag);
  const double resStart = std::sqrt(s.dot(r, r, L, flag));
  if (finalRes) *finalRes = resStart;
  if (resStart < tol) return 0;
  int it = 0;
  for (int i = 0; i < maxIter; ++i) {
    it = i + 1;
    s.apply(op, p, ap, L, flag, 0);
    const double pAp = s.dot(p, ap, L, flag);
    const double alpha = prsold / pAp;
    s.lincomb(x, L, flag, 1, &alpha, &p, true, 0.0);
    const double malpha = -alpha;
    s.lincomb(r, L, flag, 1, &malpha, &ap, true, 0.0);
    const double rsnew = s.dot(r, r, L, flag);
    const double sq = std::sqrt(rsnew);
    if (finalRes) *finalRes = sq;
    if (sq < tol) break;
    s.lincomb(z, L, flag, 1, &one, &r, false, 0.0);
    const double prsnew = s.dot(r, z, L, flag);
    const double beta = prsnew / prsold;
    const double sc[2] = {1.0, beta};
    const int src[2] = {z, p};
    s.lincomb(p, L, flag, 2, sc, src, false, 0.0);
    prsold = prsnew;
  }
  return it;
}

Gmg::Gmg(Storage& st, int op_, int minL_, int maxL_, int pre_, int post_, double omega_, int cycle_, int cmax,
         double ctol, int prec_)
    : s(st), op(op_), minL(minL_), maxL(maxL_), pre(pre_), post(post_), omega(omega_), cycle(cycle_),
      coarseMaxIter(cmax), coarseTol(ctol), prec(prec_) {
  tmp = s.createFunction(minL, maxL, prec);
  // the coarse-grid CG always runs in FP64
  cp = s.createFunction(minL, minL, 8);
  cz = s.createFunction(minL, minL, 8);
  cap = s.createFunction(minL, minL, 8);
  cr = s.createFunction(minL, minL, 8);
  if (prec == 4) {
    cx64 = s.createFunction(minL, minL, 8);
    cb64 = s.createFunction(minL, minL, 8);
    x32 = s.createFunction(minL, maxL, 4);
    b32 = s.createFunction(minL, maxL, 4);
    r64 = s.createFunction(maxL, maxL, 8);
  }
  if (deviceCoarse())
    setCoarseGroups(1);
  else
    buildCompact();
}

// Work lists of the device coarse CG. Group of a slot: the copy it belongs to when the storage
// holds `groups` disjoint copies (each kind of primitive copy after copy, Storage::batchMap),
// else 0. Per group its owned DoFs (low primitives in order, points in order) and its halo
// entries (in the level table's order); a copy's lists are the single mesh's, shifted.
void Gmg::setCoarseGroups(int groups) {
  argCheck(groups >= 1, "coarse CG: at least one group");
  argCheck(deviceCoarse(), "coarse CG groups need a coarse level with vertex and edge DoFs only");
  const LevelData& ld = s.levels[minL];
  const LevelLayout& lay = *ld.lay;
  const dev::LevelDev& lv = ld.lv;
  const LevelStencils& hs = s.op(op).host[minL - s.op(op).minL];
  dev::BatchMap bm{};
  if (groups > 1) bm = s.batchMap(minL, groups);
  auto groupOf = [&](int64_t slot) {
    if (groups == 1) return 0;
    int q = 3;
    while (q > 0 && slot < bm.uBase[q]) --q;
    argCheck(bm.size[q] > 0, "coarse CG: slot outside the copies");
    return int((slot - bm.uBase[q]) / bm.size[q]);
  };
  const unsigned mask = HG_INNER | HG_NEUMANN | HG_FREESLIP;
  std::vector<std::vector<dev::CoarseDof>> dofs((size_t)groups);
  int e = 0;
  for (int q = 0; q < lv.nLow; ++q) {
    const bool isEdge = q < lv.nEdges;
    const int n = (int)(isEdge ? hs.edge[(size_t)q].size() : hs.vert[(size_t)(q - lv.nEdges)].size());
    if (ld.hostLowType[(size_t)q] & mask) {
      const int64_t off = isEdge ? lay.off[KE][(size_t)q] : lay.off[KV][(size_t)(q - lv.nEdges)];
      const int first = isEdge ? 1 : 0;
      const int count = isEdge ? (int)std::max<int64_t>(lay.N - 1, 0) : 1;
      for (int xx = first; xx < first + count; ++xx)
        dofs[(size_t)groupOf(off + xx)].push_back({off + xx, e, e + n});
    }
    e += n;
  }
  std::vector<std::vector<uint2>> comm((size_t)groups);
  for (int g : kCommOrder)
    for (size_t i = 0; i < lay.commDst[g].size(); ++i) {
      const int gd = groupOf(lay.commDst[g][i]);
      argCheck(gd == groupOf(lay.commSrc[g][i]), "coarse CG: a halo entry crosses copies");
      comm[(size_t)gd].push_back(make_uint2((unsigned)lay.commDst[g][i], (unsigned)lay.commSrc[g][i]));
    }
  std::vector<dev::CoarseDof> flatDofs;
  std::vector<uint2> flatComm;
  std::vector<int> dofOff{0}, commOff{0};
  for (int g = 0; g < groups; ++g) {
    flatDofs.insert(flatDofs.end(), dofs[(size_t)g].begin(), dofs[(size_t)g].end());
    flatComm.insert(flatComm.end(), comm[(size_t)g].begin(), comm[(size_t)g].end());
    dofOff.push_back((int)flatDofs.size());
    commOff.push_back((int)flatComm.size());
  }
  auto put = [&](std::unique_ptr<DevBuf>& buf, const void* h, size_t bytes) {
    buf.reset(new DevBuf());
    buf->alloc(std::max<size_t>(bytes, 16));
    if (bytes) cudaCheck(cudaMemcpyAsync(buf->p, h, bytes, cudaMemcpyHostToDevice, s.stream), "coarse lists");
  };
  put(cgDofs, flatDofs.data(), flatDofs.size() * sizeof(dev::CoarseDof));
  put(cgComm, flatComm.data(), flatComm.size() * sizeof(uint2));
  put(cgDofOff, dofOff.data(), dofOff.size() * sizeof(int));
  put(cgCommOff, commOff.data(), commOff.size() * sizeof(int));
  cudaCheck(cudaStreamSynchronize(s.stream), "coarse lists");
  coarseGroups = groups;
  cache.clear();
  buildCompact();
}

void Gmg::setCompact(int maxDofs, int cluster) {
  argCheck(cluster == 1 || cluster == 2 || cluster == 4 || cluster == 8, "compact cycle: 1, 2, 4 or 8 blocks per group");
  compactMaxDofs = maxDofs;
  compactCluster = cluster;
  buildCompact(true);
}

// The highest level within reach (at most compactMaxDofs unknowns per group, at most
// kCompactMaxLevels levels) tops the compact cycle. By default a mesh outside its structural
// assumptions (argument errors of the builder) keeps the level-by-level cycle; an explicit
// request (strict) reports them.
void Gmg::buildCompact(bool strict) {
  cache.clear();
  compact.reset();
  compactTop = -1;
  if (cycle != 0 || compactMaxDofs <= 0) return;
  int top = -1;
  for (int l = minL + 1; l <= std::min(maxL, minL + dev::kCompactMaxLevels - 1); ++l)
    if (compactGroupDofs(s, l, coarseGroups) <= compactMaxDofs) top = l;
  if (top < 0) return;
  try {
    compact = buildCompactCycle(s, op, minL, top, coarseGroups, compactCluster, prec, HG_INNER | HG_NEUMANN,
                                HG_INNER | HG_NEUMANN | HG_FREESLIP);
    compactTop = top;
  } catch (const Error& e) {
    if (strict || e.code != HG_ERR_ARG) throw;
    compact.reset();
  }
}

Gmg::~Gmg() {
  cache.clear();
  for (int id : {tmp, cp, cz, cap, cr, cx64, cb64, x32, b32, r64})
    if (id >= 0) s.fns.erase(id);
}

bool Gmg::deviceCoarse() const {
  const dev::LevelDev& lv = s.levels[minL].lv;
  return lv.nCellBlocks == 0 && lv.nFaceBlocks == 0;
}

void Gmg::setGraphs(bool on) {
  graphs = on;
  if (!on) cache.clear();
}

void Gmg::setTiming(bool on) {
  if (on) timing.reset(new TimingTree());
  else timing.reset();
}

// ---------------------------------------------------------------------------------------
// Timing tree
// ---------------------------------------------------------------------------------------
TimingTree::Node& TimingTree::Node::child(const std::string& name) {
  for (auto& c : children)
    if (c.first == name) return c.second;
  children.emplace_back(name, Node());
  return children.back().second;
}

TimingTree::~TimingTree() {
  std::vector<Node*> todo{&root};
  while (!todo.empty()) {
    Node* n = todo.back();
    todo.pop_back();
    for (auto& p : n->pending) {
      cudaEventDestroy(p.first);
      cudaEventDestroy(p.second);
    }
    if (n->open) cudaEventDestroy(n->open);
    for (auto& c : n->children) todo.push_back(&c.second);
  }
  for (cudaEvent_t e : pool) cudaEventDestroy(e);
}

void TimingTree::start(cudaStream_t st, const std::string& name) {
  Node& n = stack.back()->child(name);
  argCheck(n.open == nullptr, "timing tree: \"" + name + "\" started twice");
  cudaEvent_t e;
  if (!pool.empty()) {
    e = pool.back();
    pool.pop_back();
  } else {
    cudaCheck(cudaEventCreate(&e), "timing event");
  }
  cudaCheck(cudaEventRecord(e, st), "timing event");
  n.open = e;
  stack.push_back(&n);
}

void TimingTree::stop(cudaStream_t st, const std::string& name, int applications) {
  argCheck(stack.size() > 1, "timing tree: stop without start");
  Node& n = *stack.back();
  const Node* named = nullptr;  // look the name up without inserting (an insertion could move n)
  for (auto& c : stack[stack.size() - 2]->children)
    if (c.first == name) named = &c.second;
  argCheck(named == &n && n.open != nullptr, "timing tree: \"" + name + "\" is not the innermost open timer");
  cudaEvent_t e;
  if (!pool.empty()) {
    e = pool.back();
    pool.pop_back();
  } else {
    cudaCheck(cudaEventCreate(&e), "timing event");
  }
  cudaCheck(cudaEventRecord(e, st), "timing event");
  n.pending.emplace_back(n.open, e);
  n.pendingCount.push_back(std::max(applications, 1));
  n.open = nullptr;
  stack.pop_back();
}

void TimingTree::resolve() {
  std::vector<Node*> todo{&root};
  while (!todo.empty()) {
    Node* n = todo.back();
    todo.pop_back();
    for (size_t i = 0; i < n->pending.size(); ++i) {
      cudaCheck(cudaEventSynchronize(n->pending[i].second), "timing resolve");
      float ms = 0;
      cudaCheck(cudaEventElapsedTime(&ms, n->pending[i].first, n->pending[i].second), "timing resolve");
      const int a = n->pendingCount[i];
      const double t = ms * 1e-3 / a;  // each application's share
      for (int k = 0; k < a; ++k) {
        n->min = n->count == 0 ? t : std::min(n->min, t);
        n->max = n->count == 0 ? t : std::max(n->max, t);
        n->total += t;
        n->sumSq += t * t;
        ++n->count;
      }
      pool.push_back(n->pending[i].first);
      pool.push_back(n->pending[i].second);
    }
    n->pending.clear();
    n->pendingCount.clear();
    for (auto& c : n->children) todo.push_back(&c.second);
  }
}

void TimingTree::reset() {
  resolve();
  root = Node();
  stack.assign(1, &root);
}

static void timerJson(std::string& out, double total, int64_t count, double mn, double mx, double sumSq) {
  const double avg = count ? total / count : 0.0;
  const double var = count ? std::max(sumSq / count - avg * avg, 0.0) : 0.0;
  char buf[256];
  std::snprintf(buf, sizeof(buf), "\"total\": %.9g, \"average\": %.9g, \"count\": %lld, \"min\": %.9g, \"max\": %.9g, "
                "\"variance\": %.9g", total, avg, (long long)count, mn, mx, var);
  out += buf;
}

static void nodeJson(std::string& out, const TimingTree::Node& n) {
  out += "{";
  timerJson(out, n.total, n.count, n.min, n.max, n.sumSq);
  double covered = 0;
  for (auto& c : n.children) {
    out += ", \"" + c.first + "\": ";
    nodeJson(out, c.second);
    covered += c.second.total;
  }
  if (!n.children.empty()) {  // getCopyWithRemainder
    const double r = std::max(n.total - covered, 0.0);
    out += ", \"Remainder\": {";
    timerJson(out, r, 1, r, r, r * r);
    out += "}";
  }
  out += "}";
}

std::string TimingTree::json() {
  resolve();
  std::string out = "{";
  bool first = true;
  for (auto& c : root.children) {
    if (!first) out += ", ";
    first = false;
    out += "\"" + c.first + "\": ";
    nodeJson(out, c.second);
  }
  out += "}";
  return out;
}

void GraphCache::clear() {
  for (auto& c : captured) cudaGraphExecDestroy(c.exec);
  captured.clear();
  warm.clear();
}

void GraphCache::run(Storage& s, const std::function<std::vector<uintptr_t>()>& signature,
                     const std::function<void()>& cycle) {
  const std::vector<uintptr_t> sig = signature();
  for (auto& c : captured)
    if (c.sig == sig) {
      cudaCheck(cudaGraphLaunch(c.exec, s.stream), "graph launch");
      s.launches += c.launches;
      return;
    }
  bool seen = false;
  for (auto& w : warm) seen = seen || w == sig;
  if (!seen) {  // first cycle under this signature runs eagerly (allocates buffers, tables)
    cycle();
    if (signature() == sig) warm.push_back(sig);
    if (warm.size() > 8) warm.erase(warm.begin());
    return;
  }
  const unsigned long long l0 = s.launches;
  cudaCheck(cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeThreadLocal), "begin capture");
  cudaGraph_t g = nullptr;
  try {
    cycle();
  } catch (...) {
    cudaStreamEndCapture(s.stream, &g);
    if (g) cudaGraphDestroy(g);
    s.launches = l0;
    throw;
  }
  cudaCheck(cudaStreamEndCapture(s.stream, &g), "end capture");
  Captured c;
  c.sig = sig;
  c.launches = s.launches - l0;
  s.launches = l0;
  cudaError_t e = cudaGraphInstantiate(&c.exec, g, 0);
  cudaGraphDestroy(g);
  cudaCheck(e, "graph instantiate");
  if (signature() != sig) {  // the host-side buffer state did not return: no replay
    cudaGraphExecDestroy(c.exec);
    throw Error(HG_ERR_INTERNAL, "captured cycle changed the buffer state");
  }
  cudaCheck(cudaGraphLaunch(c.exec, s.stream), "graph launch");
  s.launches += c.launches;
  captured.push_back(c);
  if (captured.size() > 4) {
    cudaGraphExecDestroy(captured.front().exec);
    captured.erase(captured.begin());
  }
}

// The coarse CG: on the device, one block per group, when the coarse level has only vertex and
// edge DoFs (no host synchronisation), else the host-driven cgSolve. Same iteration either way.
void Gmg::coarseSolve(int x, int b, int L) {
  int xs = x, bs = b;
  if (prec == 4) {  // FP32 hierarchy: the coarse problem is solved in FP64 and rounded back
    s.copyCast(cb64, b, L, HG_ALL, false);
    s.copyCast(cx64, x, L, HG_ALL, false);
    xs = cx64;
    bs = cb64;
  }
  if (timing) timing->start(s.stream, "CG Solver");
  if (deviceCoarse()) {
    Operator& o = s.op(op);
    dev::coarseCgKernel<<<coarseGroups, dev::kBlock, 0, s.stream>>>(
        o.d[L - o.minL], (const dev::CoarseDof*)cgDofs->p, (const int*)cgDofOff->p, (const uint2*)cgComm->p,
        (const int*)cgCommOff->p, (double*)s.data(xs, L), (const double*)s.data(bs, L), (double*)s.data(cr, L),
        (double*)s.data(cp, L), (double*)s.data(cap, L), coarseMaxIter, coarseTol, nullptr);
    ++s.launches;
    cudaCheck(cudaGetLastError(), "coarse CG");
  } else {
    cgSolve(s, op, xs, bs, L, coarseMaxIter, coarseTol, cp, cz, cap, cr, nullptr);
  }
  if (timing) timing->stop(s.stream, "CG Solver");
  if (prec == 4) s.copyCast(x, cx64, L, HG_ALL, false);
}

// Every device address one cycle on (x, b, L) reads or writes, plus what fixes the kernel
// arguments: a graph captured under one signature is replayed only under the same one.
std::vector<uintptr_t> Gmg::signature(int x, int b, int L) {
  std::vector<uintptr_t> sig = {(uintptr_t)L, (uintptr_t)x, (uintptr_t)b, (uintptr_t)op, (uintptr_t)s.generation,
                                (uintptr_t)s.structureOp};
  Operator& o = s.op(op);
  for (int l = minL; l <= L; ++l) {
    sig.push_back((uintptr_t)s.data(x, l));
    sig.push_back((uintptr_t)s.data(b, l));
    sig.push_back((uintptr_t)s.data(tmp, l));
    auto it = s.spare.find({l, prec});
    sig.push_back(it != s.spare.end() && it->second ? (uintptr_t)it->second->p : 0);
    auto is = s.splitRhs.find({l, prec});
    sig.push_back(is != s.splitRhs.end() && is->second ? (uintptr_t)is->second->p : 0);
    sig.push_back((uintptr_t)s.levels[l].commSplit);
    sig.push_back((uintptr_t)o.d[l - o.minL].cellW);
  }
  for (int id : {cp, cz, cap, cr, cx64, cb64})
    if (id >= 0) sig.push_back((uintptr_t)s.data(id, minL));
  sig.push_back(cgDofs ? (uintptr_t)cgDofs->p : 0);
  sig.push_back((uintptr_t)coarseGroups);
  sig.push_back(compact ? (uintptr_t)compact->scratch.p : 0);
  sig.push_back((uintptr_t)(intptr_t)compactTop);
  return sig;
}

void Gmg::runCycle(int x, int b, int L) {
  if (timing) {  // GeometricMultigridSolver::solve (GeometricMultigridSolver.hpp:127-134), eagerly
    timing->start(s.stream, "Geometric Multigrid Solver");
    solveRecursively(x, b, L);
    timing->stop(s.stream, "Geometric Multigrid Solver");
    return;
  }
  if (!graphs || (pre + post) % 2 != 0 || !(deviceCoarse() || (compact && L >= compactTop))) {
    solveRecursively(x, b, L);
    return;
  }
  cache.run(s, [&] { return signature(x, b, L); }, [&] { solveRecursively(x, b, L); });
}

// GeometricMultigridSolver::solveRecursively (src/hyteg/solvers/GeometricMultigridSolver.hpp:136-235)
void Gmg::solveRecursively(int x, int b, int L) {
  const unsigned flag = HG_INNER | HG_NEUMANN;
  TimingTree* tt = timing.get();
  const std::string lvl = tt ? "Level " + std::to_string(L) : std::string();
  auto start = [&](const std::string& n) {
    if (tt) tt->start(s.stream, n);
  };
  auto stop = [&](const std::string& n, int applications = 1) {
    if (tt) tt->stop(s.stream, n, applications);
  };
  if (L == minL) {
    start(lvl);
    start("Coarse Grid Solver");
    coarseSolve(x, b, L);
    stop("Coarse Grid Solver");
    stop(lvl);
    return;
  }
  if (compact && !tt && L == compactTop) {
    runCompactCycle(*compact, s, s.data(x, L), s.data(b, L), false, pre, post, omega, coarseMaxIter, coarseTol);
    return;
  }
  start(lvl);
  if (pre > 0) {
    start("Smoother");
    s.smoothSorSweeps(op, x, b, omega, L, flag, pre, false, false);
    stop("Smoother", pre);
  }
  s.residual(op, x, b, tmp, L, flag);
  start("Restriction");
  // straight into the coarse right-hand side: the restriction writes the flagged coarse DoFs,
  // the only ones of b that the coarser level reads
  s.restrictFn(tmp, L, flag, b);
  stop("Restriction");
  // the compact cycle starts the coarser level from zero itself
  const bool compactBelow = compact && !tt && L - 1 == compactTop;
  if (!compactBelow) s.lincomb(x, L - 1, HG_ALL, 0, nullptr, nullptr, false, 0.0);
  stop(lvl);
  if (compactBelow) {
    runCompactCycle(*compact, s, s.data(x, L - 1), s.data(b, L - 1), true, pre, post, omega, coarseMaxIter,
                    coarseTol);
  } else {
    solveRecursively(x, b, L - 1);
    if (cycle == 1) solveRecursively(x, b, L - 1);
  }
  start(lvl);
  start("Prolongation");
  s.prolongate(x, L - 1, flag, true);
  stop("Prolongation");
  // b is unchanged on this level since the pre-smoothing, which left its colour-split copy
  if (post > 0) {
    start("Smoother");
    s.smoothSorSweeps(op, x, b, omega, L, flag, post, false, pre > 0);
    stop("Smoother", post);
  }
  stop(lvl);
}

int Gmg::solveTo(int x, int b, int L, double tol, int maxIter, double* relRes, double* history, int historyCap) {
  const unsigned flag = HG_INNER | HG_NEUMANN;
  argCheck(L >= minL && L <= maxL, "gmg: level outside the solver's range");
  Function& fx = s.fn(x);
  argCheck(fx.prec == 8 && s.fn(b).prec == 8, "solveTo: x and b must be FP64 functions");
  const int r = prec == 8 ? tmp : r64;
  s.residual(op, x, b, r, L, flag);
  const double r0 = std::sqrt(s.dot(r, r, L, flag));
  double rel = 1.0;
  int it = 0;
  while (it < maxIter && rel > tol && r0 > 0.0) {
    if (prec == 8) {
      runCycle(x, b, L);
    } else {
      // defect correction: FP32 cycle on A e = r (zero start), x += e in FP64
      s.copyCast(b32, r, L, HG_ALL, false);
      for (int l = minL; l <= L; ++l) s.lincomb(x32, l, HG_ALL, 0, nullptr, nullptr, false, 0.0);
      runCycle(x32, b32, L);
      s.copyCast(x, x32, L, flag, true);
    }
    ++it;
    s.residual(op, x, b, r, L, flag);
    rel = std::sqrt(s.dot(r, r, L, flag)) / r0;
    if (history && it <= historyCap) history[it - 1] = rel;
  }
  if (relRes) *relRes = r0 > 0.0 ? rel : 0.0;
  return it;
}

void Gmg::solveToBatch(int x, int b, int xOut, int L, const double* tol, const int* maxIter, const dev::BatchMap& bm,
                       int active, double* dNorms, int* iterations, double* relRes) {
  const unsigned flag = HG_INNER | HG_NEUMANN;
  argCheck(L >= minL && L <= maxL, "gmg: level outside the solver's range");
  argCheck(active >= 0 && active <= bm.copies, "batch: active copies out of range");
  argCheck(s.fn(x).prec == 8 && s.fn(b).prec == 8 && s.fn(xOut).prec == 8, "solveToBatch: FP64 functions required");
  const int r = prec == 8 ? tmp : r64;
  std::vector<double> h((size_t)bm.copies);
  auto norms = [&]() {
    s.dotBatchAsync(r, r, L, flag, bm, dNorms);
    cudaCheck(cudaMemcpyAsync(h.data(), dNorms, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s.stream), "batch norms");
    cudaCheck(cudaStreamSynchronize(s.stream), "batch norms");
  };
  s.residual(op, x, b, r, L, flag);
  norms();
  std::vector<double> r0((size_t)active);
  std::vector<char> done((size_t)active, 0);
  int left = 0;
  for (int i = 0; i < active; ++i) {
    r0[(size_t)i] = std::sqrt(h[(size_t)i]);
    iterations[i] = 0;
    if (!(maxIter[i] > 0 && 1.0 > tol[i] && r0[(size_t)i] > 0.0)) {  // solveTo takes no iteration
      relRes[i] = r0[(size_t)i] > 0.0 ? 1.0 : 0.0;
      s.copyBatchSlots(x, xOut, L, bm, i);
      done[(size_t)i] = 1;
    } else {
      ++left;
    }
  }
  int it = 0;
  while (left > 0) {
    if (prec == 8) {
      runCycle(x, b, L);
    } else {  // defect correction: FP32 cycle on A e = r (zero start), x += e in FP64
      s.copyCast(b32, r, L, HG_ALL, false);
      for (int l = minL; l <= L; ++l) s.lincomb(x32, l, HG_ALL, 0, nullptr, nullptr, false, 0.0);
      runCycle(x32, b32, L);
      s.copyCast(x, x32, L, flag, true);
    }
    ++it;
    s.residual(op, x, b, r, L, flag);
    norms();
    for (int i = 0; i < active; ++i) {
      if (done[(size_t)i]) continue;
      const double rel = std::sqrt(h[(size_t)i]) / r0[(size_t)i];
      if (!(it < maxIter[i] && rel > tol[i])) {
        iterations[i] = it;
        relRes[i] = rel;
        s.copyBatchSlots(x, xOut, L, bm, i);
        done[(size_t)i] = 1;
        --left;
      }
    }
  }
}

void Gmg::solve(int x, int b, int L) {
  argCheck(L >= minL && L <= maxL, "gmg: level outside the solver's range");
  Function& fx = s.fn(x);
  Function& fb = s.fn(b);
  argCheck(fx.prec == prec && fb.prec == prec, "gmg: function precision differs from the solver's");
  argCheck(fx.minL <= minL && fb.minL <= minL && fx.maxL >= L && fb.maxL >= L, "gmg: functions must span the level range");
  runCycle(x, b, L);
}

P2Gmg::P2Gmg(Storage& st, int op_, int minL_, int maxL_, int pre_, int post_, double omega_, int cmax, double ctol,
             int prec_)
    : s(st), op(op_), minL(minL_), maxL(maxL_), pre(pre_), post(post_), omega(omega_), coarseMaxIter(cmax),
      coarseTol(ctol), prec(prec_) {
  P2Operator& o = s.p2op(op);
  argCheck(minL >= o.minL && maxL <= o.maxL && minL <= maxL, "P2 multigrid: levels outside the operator's range");
  argCheck(prec == 8 || prec == 4, "P2 multigrid: precision must be 8 or 4");
  tmp = s.createFunction(minL + 1, maxL + 1, prec);
  cp = s.createFunction(minL + 1, minL + 1, 8);
  cz = s.createFunction(minL + 1, minL + 1, 8);
  cap = s.createFunction(minL + 1, minL + 1, 8);
  cr = s.createFunction(minL + 1, minL + 1, 8);
  if (prec == 4) {
    cx64 = s.createFunction(minL + 1, minL + 1, 8);
    cb64 = s.createFunction(minL + 1, minL + 1, 8);
  }
}

P2Gmg::~P2Gmg() {
  cache.clear();
  for (int id : {tmp, cp, cz, cap, cr, cx64, cb64})
    if (id >= 0) s.fns.erase(id);
}

// The operator restricted to the unknowns of the coarsest level, column by column (the operator
// applied to unit vectors), inverted on the host by Gauss-Jordan elimination with partial pivoting.
bool P2Gmg::buildCoarseDirect() {
  if (coarseN >= 0) return coarseN > 0;
  coarseN = 0;
  const unsigned flag = HG_INNER | HG_NEUMANN | HG_FREESLIP;
  const int Lf = minL + 1;
  P2Additive& ad = s.p2Additive(Lf);
  std::vector<int64_t> idx;
  for (size_t i = 0; i < ad.hostOwner.size(); ++i)
    if (ad.hostOwnerType[i] & flag) idx.push_back(ad.hostOwner[i]);
  const int n = (int)idx.size();
  if (ad.hostOwner.empty() || n == 0 || n > kCoarseDirectMax) return false;
  const int64_t total = s.disc.level(Lf).total;
  const int e = s.createFunction(Lf, Lf, 8), y = s.createFunction(Lf, Lf, 8);
  std::vector<double> he((size_t)total, 0.0), hy((size_t)total), a((size_t)n * n), inv((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) {
    he[(size_t)idx[j]] = 1.0;
    cudaCheck(cudaMemcpyAsync(s.data(e, Lf), he.data(), (size_t)total * 8, cudaMemcpyHostToDevice, s.stream), "coarse");
    cudaCheck(cudaStreamSynchronize(s.stream), "coarse");
    he[(size_t)idx[j]] = 0.0;
    s.p2Apply(op, e, y, -1, minL, flag, 0);
    cudaCheck(cudaMemcpyAsync(hy.data(), s.data(y, Lf), (size_t)total * 8, cudaMemcpyDeviceToHost, s.stream), "coarse");
    cudaCheck(cudaStreamSynchronize(s.stream), "coarse");
    for (int i = 0; i < n; ++i) a[(size_t)i * n + j] = hy[(size_t)idx[i]];  // row-major A(i, j)
  }
  s.fns.erase(e);
  s.fns.erase(y);
  for (int i = 0; i < n; ++i) inv[(size_t)i * n + i] = 1.0;
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(a[(size_t)r * n + c]) > std::fabs(a[(size_t)piv * n + c])) piv = r;
    argCheck(a[(size_t)piv * n + c] != 0.0, "P2 multigrid: singular coarse-level operator");
    if (piv != c)
      for (int k = 0; k < n; ++k) {
        std::swap(a[(size_t)piv * n + k], a[(size_t)c * n + k]);
        std::swap(inv[(size_t)piv * n + k], inv[(size_t)c * n + k]);
      }
    const double d = 1.0 / a[(size_t)c * n + c];
    for (int k = 0; k < n; ++k) {
      a[(size_t)c * n + k] *= d;
      inv[(size_t)c * n + k] *= d;
    }
    for (int r = 0; r < n; ++r) {
      const double f = a[(size_t)r * n + c];
      if (r == c || f == 0.0) continue;
      for (int k = 0; k < n; ++k) {
        a[(size_t)r * n + k] -= f * a[(size_t)c * n + k];
        inv[(size_t)r * n + k] -= f * inv[(size_t)c * n + k];
      }
    }
  }
  std::vector<double> colMajor((size_t)n * n);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < n; ++k) colMajor[(size_t)k * n + i] = inv[(size_t)i * n + k];
  coarseIdx.reset(new DevBuf());
  coarseIdx->alloc((size_t)n * sizeof(int64_t));
  coarseInv.reset(new DevBuf());
  coarseInv->alloc((size_t)n * n * sizeof(double));
  cudaCheck(cudaMemcpyAsync(coarseIdx->p, idx.data(), (size_t)n * 8, cudaMemcpyHostToDevice, s.stream), "coarse");
  cudaCheck(cudaMemcpyAsync(coarseInv->p, colMajor.data(), colMajor.size() * 8, cudaMemcpyHostToDevice, s.stream),
            "coarse");
  cudaCheck(cudaStreamSynchronize(s.stream), "coarse");
  coarseN = n;
  return true;
}

// Coarsest level: x += A^-1 (b - A x) on the unknowns (one residual, one dense product, one halo
// refresh, all on the device), or CG when the coarse level has too many unknowns.
void P2Gmg::coarseSolve(int x, int b, int L) {
  if (!buildCoarseDirect()) {
    coarseCg(x, b, L);
    return;
  }
  const unsigned flag = HG_INNER | HG_NEUMANN | HG_FREESLIP;
  s.p2Apply(op, x, cr, b, L, flag, 2);
  dev::denseCorrectKernel<<<(coarseN + dev::kBlock - 1) / dev::kBlock, dev::kBlock, (size_t)coarseN * 8, s.stream>>>(
      (const int64_t*)coarseIdx->p, coarseN, (const double*)coarseInv->p, (const double*)s.data(cr, L + 1),
      (double*)s.data(x, L + 1));
  ++s.launches;
  cudaCheck(cudaGetLastError(), "coarse solve");
  s.communicate(x, L + 1, (1 << G_COUNT) - 1);
}

std::vector<uintptr_t> P2Gmg::signature(int x, int b, int L) {
  std::vector<uintptr_t> sig = {(uintptr_t)L, (uintptr_t)x, (uintptr_t)b, (uintptr_t)op, (uintptr_t)s.generation,
                                (uintptr_t)symmetric, (uintptr_t)coarseN};
  P2Operator& o = s.p2op(op);
  for (int l = minL; l <= L; ++l) {
    for (int id : {x, b, tmp}) sig.push_back((uintptr_t)s.data(id, l + 1));
    auto sc = s.p2scratch.find(s.p2ScratchKey(l + 1, prec));
    sig.push_back(sc != s.p2scratch.end() ? (uintptr_t)s.data(sc->second, l + 1) : 0);
    auto dg = o.diag.find({l, prec});
    sig.push_back(dg != o.diag.end() ? (uintptr_t)s.data(dg->second, l + 1) : 0);
  }
  for (int id : {cr, cx64, cb64})
    if (id >= 0) sig.push_back((uintptr_t)s.data(id, minL + 1));
  sig.push_back(coarseInv ? (uintptr_t)coarseInv->p : 0);
  return sig;
}

void P2Gmg::runCycle(int x, int b, int L) {
  struct LaneGuard {  // the cycle's scratch lane, restored on every exit
    Storage& s;
    int old;
    ~LaneGuard() { s.p2Lane = old; }
  } guard{s, s.p2Lane};
  s.p2Lane = lane;
  if (!graphs || !buildCoarseDirect()) {
    solveRecursively(x, b, L);
    return;
  }
  cache.run(s, [&] { return signature(x, b, L); }, [&] { solveRecursively(x, b, L); });
}

// CGSolver (CGSolver.hpp:69-150, identity preconditioner) with the P2 operator of level L.
int P2Gmg::coarseCg(int x, int b, int L) {
  const unsigned flag = HG_INNER | HG_NEUMANN | HG_FREESLIP;
  const int Lf = L + 1;
  const double one = 1.0;
  s.p2Apply(op, x, cr, b, L, flag, 2);  // r = b - A x
  s.lincomb(cp, Lf, flag, 1, &one, &cr, false, 0.0);
  double rs = s.dot(cr, cr, Lf, flag);
  if (std::sqrt(rs) < coarseTol) return 0;
  int it = 0;
  for (int i = 0; i < coarseMaxIter; ++i) {
    it = i + 1;
    s.p2Apply(op, cp, cap, -1, L, flag, 0);
    const double alpha = rs / s.dot(cp, cap, Lf, flag);
    s.lincomb(x, Lf, flag, 1, &alpha, &cp, true, 0.0);
    const double malpha = -alpha;
    s.lincomb(cr, Lf, flag, 1, &malpha, &cap, true, 0.0);
    const double rsn = s.dot(cr, cr, Lf, flag);
    if (std::sqrt(rsn) < coarseTol) break;
    const double sc[2] = {1.0, rsn / rs};
    const int src[2] = {cr, cp};
    s.lincomb(cp, Lf, flag, 2, sc, src, false, 0.0);
    rs = rsn;
  }
  return it;
}

// GeometricMultigridSolver::solveRecursively (GeometricMultigridSolver.hpp:136-235) with the P2
// pieces: SOR, r = b - A x, restriction, coarse-grid correction, prolongation and add.
void P2Gmg::solveRecursively(int x, int b, int L) {
  const unsigned flag = HG_INNER | HG_NEUMANN;
  if (L == minL) {
    if (prec == 8) {
      coarseSolve(x, b, L);
    } else {  // FP32 cycle: the coarse problem in FP64, rounded back
      s.copyCast(cb64, b, L + 1, HG_ALL, false);
      s.copyCast(cx64, x, L + 1, HG_ALL, false);
      coarseSolve(cx64, cb64, L);
      s.copyCast(x, cx64, L + 1, HG_ALL, false);
    }
    return;
  }
  for (int i = 0; i < pre; ++i) s.p2Sor(op, x, b, omega, L, flag, false);
  s.p2Apply(op, x, tmp, b, L, flag, 2);
  s.p2Restrict(tmp, L, flag);
  const double one = 1.0;
  s.lincomb(b, L, flag, 1, &one, &tmp, false, 0.0);  // lattice level L = P2 level L - 1
  s.lincomb(x, L, HG_ALL, 0, nullptr, nullptr, false, 0.0);
  solveRecursively(x, b, L - 1);
  s.p2Prolongate(x, L - 1, flag, true);
  for (int i = 0; i < post; ++i) s.p2Sor(op, x, b, omega, L, flag, symmetric);
}

// Moore-Penrose inverse of a symmetric n x n matrix (row-major, overwritten) by cyclic Jacobi
// rotations (Golub and Van Loan, Matrix Computations, section 8.5): eigenvalues below
// 1e-10 * max |eigenvalue| count as zero. Returns the pseudo-inverse column-major (= row-major).
static std::vector<double> symmetricPinv(std::vector<double>& A, int n) {
  std::vector<double> V((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
  double total = 0.0;
  for (double v : A) total += v * v;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += A[(size_t)p * n + q] * A[(size_t)p * n + q];
    if (off <= 1e-32 * total) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[(size_t)p * n + q];
        if (apq == 0.0) continue;
        const double theta = (A[(size_t)q * n + q] - A[(size_t)p * n + p]) / (2.0 * apq);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
        for (int k = 0; k < n; ++k) {  // columns p, q
          const double akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
          A[(size_t)k * n + p] = c * akp - sn * akq;
          A[(size_t)k * n + q] = sn * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // rows p, q
          const double apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
          A[(size_t)p * n + k] = c * apk - sn * aqk;
          A[(size_t)q * n + k] = sn * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = V[(size_t)k * n + p], vkq = V[(size_t)k * n + q];
          V[(size_t)k * n + p] = c * vkp - sn * vkq;
          V[(size_t)k * n + q] = sn * vkp + c * vkq;
        }
      }
  }
  double lmax = 0.0;
  for (int i = 0; i < n; ++i) lmax = std::max(lmax, std::fabs(A[(size_t)i * n + i]));
  std::vector<double> P((size_t)n * n, 0.0);
  for (int m = 0; m < n; ++m) {
    const double l = A[(size_t)m * n + m];
    if (std::fabs(l) <= 1e-10 * lmax) continue;
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < n; ++k) P[(size_t)i * n + k] += V[(size_t)i * n + m] * V[(size_t)k * n + m] / l;
  }
  return P;
}

StokesGmg::StokesGmg(Storage& st, int op_, int minL_, int maxL_, int pre_, int post_, double omega_, int sweeps)
    : s(st), op(op_), minL(minL_), maxL(maxL_), pre(pre_), post(post_), omega(omega_), velocitySweeps(sweeps) {
  P2Operator& o = s.p2op(op);
  argCheck(!o.dd.empty(), "Stokes multigrid: not a Stokes operator");
  argCheck(minL >= o.minL && maxL <= o.maxL && minL <= maxL, "Stokes multigrid: levels outside the operator's range");
  argCheck(pre >= 0 && post >= 0 && sweeps >= 1, "Stokes multigrid: invalid smoothing steps");
  for (int k = 0; k < 3; ++k) {
    ru[k] = s.createFunction(minL + 1, maxL + 1, 8);
    tu[k] = s.createFunction(minL + 1, maxL + 1, 8);
  }
  rp = s.createFunction(minL, maxL, 8);
  tp = s.createFunction(minL, maxL, 8);
  pspg = s.createOperator(FORM_PSPG, minL, maxL);
  for (int L = minL; L <= maxL; ++L) invDiag.push_back(s.p1Diagonal(pspg, L));
  smoothedInOrder.assign((size_t)(maxL - minL + 1), 0);
  for (int k = 0; k < 2; ++k) {
    cudaCheck(cudaStreamCreateWithFlags(&laneStream[k], cudaStreamNonBlocking), "stream");
    cudaCheck(cudaEventCreateWithFlags(&joinEvent[k], cudaEventDisableTiming), "event");
  }
  cudaCheck(cudaEventCreateWithFlags(&forkEvent, cudaEventDisableTiming), "event");
}

StokesGmg::~StokesGmg() {
  for (int k = 0; k < 2; ++k) {
    if (laneStream[k]) cudaStreamDestroy(laneStream[k]);
    if (joinEvent[k]) cudaEventDestroy(joinEvent[k]);
  }
  if (forkEvent) cudaEventDestroy(forkEvent);
  for (int k = 0; k < 3; ++k) {
    s.fns.erase(ru[k]);
    s.fns.erase(tu[k]);
  }
  s.fns.erase(rp);
  s.fns.erase(tp);
  for (int d : invDiag) s.fns.erase(d);
  s.ops.erase(pspg);
}

// UzawaSmoother::uzawaSmooth, block-Laplace variant without stabilisation (UzawaSmoother.hpp:287-423);
// invDiag holds the PSPG diagonal itself: r_p / diag == pspg_inv_diag applied to r_p.
void StokesGmg::smooth(const int u[3], int p, const int f[3], int g, int L) {
  const unsigned fv = HG_INNER | HG_NEUMANN, fp = HG_ALL;
  const int Lv = L + 1;
  const double a[2] = {1.0, -1.0};
  s.stokesDivT(op, p, ru, L, fv, false);
  for (int k = 0; k < 3; ++k) {
    const int src[2] = {f[k], ru[k]};
    s.lincomb(ru[k], Lv, fv, 2, a, src, false, 0.0);
  }
  // the velocity sweeps, component by component: on three streams (one P2 scratch lane each) once
  // this level has been smoothed in order
  char& warmed = smoothedInOrder[(size_t)(L - minL)];
  const bool concurrent = warmed && s.concurrentComponents;
  {
    struct Restore {  // the storage's stream and lane, restored on every exit
      Storage& s;
      cudaStream_t home;
      int lane;
      ~Restore() {
        s.stream = home;
        s.p2Lane = lane;
      }
    } restore{s, s.stream, s.p2Lane};
    if (concurrent) {
      cudaCheck(cudaEventRecord(forkEvent, restore.home), "event");
      for (int k = 0; k < 2; ++k) cudaCheck(cudaStreamWaitEvent(laneStream[k], forkEvent, 0), "wait");
    }
    for (int k = 0; k < 3; ++k) {
      s.stream = concurrent && k > 0 ? laneStream[k - 1] : restore.home;
      s.p2Lane = k;
      for (int i = 0; i < velocitySweeps; ++i) s.p2Sor(op, u[k], ru[k], 1.0, L, fv, false);
      if (concurrent && k > 0) cudaCheck(cudaEventRecord(joinEvent[k - 1], s.stream), "event");
    }
    s.stream = restore.home;
    if (concurrent)
      for (int k = 0; k < 2; ++k) cudaCheck(cudaStreamWaitEvent(restore.home, joinEvent[k], 0), "wait");
  }
  warmed = 1;
  s.stokesDiv(op, u, rp, L, fp);
  const int src[2] = {g, rp};
  s.lincomb(rp, L, fp, 2, a, src, false, 0.0);
  s.divideBy(rp, rp, invDiag[L - minL], L, fp);
  s.lincomb(p, L, fp, 1, &omega, &rp, true, 0.0);
  s.communicate(p, L, (1 << G_COUNT) - 1);
}

// tu = f - (A u + D^T p), tp = g - D u on the unknowns
static void stokesResidual(Storage& s, int op, const int u[3], int p, const int f[3], int g, const int tu[3], int tp,
                           int L) {
  const unsigned fv = HG_INNER | HG_NEUMANN, fp = HG_ALL;
  const double a[2] = {1.0, -1.0};
  s.stokesApply(op, u, p, tu, tp, L, fv, fp);
  for (int k = 0; k < 3; ++k) {
    const int src[2] = {f[k], tu[k]};
    s.lincomb(tu[k], L + 1, fv, 2, a, src, false, 0.0);
  }
  const int src[2] = {g, tp};
  s.lincomb(tp, L, fp, 2, a, src, false, 0.0);
}

double StokesGmg::residualNorm(const int u[3], int p, const int f[3], int g, int L) {
  stokesResidual(s, op, u, p, f, g, tu, tp, L);
  double t = s.dot(tp, tp, L, HG_ALL);
  for (int k = 0; k < 3; ++k) t += s.dot(tu[k], tu[k], L + 1, HG_INNER | HG_NEUMANN);
  return std::sqrt(t);
}

double StokesGmg::estimateOmega(int L, int iters, uint64_t seed) {
  argCheck(L >= minL && L <= maxL && iters >= 1, "Uzawa estimate: invalid level or iterations");
  const unsigned all = HG_ALL, fv = HG_INNER | HG_NEUMANN;
  const int Lv = L + 1;
  const int mass = s.createOperator(FORM_MASS, L, L);
  const int ones = s.createFunction(L, L, 8), lumped = s.createFunction(L, L, 8);
  const int itv = s.createFunction(L, L, 8), aux = s.createFunction(L, L, 8);
  s.lincomb(ones, L, all, 0, nullptr, nullptr, false, 1.0);
  s.apply(mass, ones, lumped, L, all, 0);
  s.fillRandom(itv, L, all, seed, 0.0, 1.0);
  auto E = [&](int src, int dst) {
    for (int k = 0; k < 3; ++k) s.lincomb(ru[k], Lv, all, 0, nullptr, nullptr, false, 0.0);
    s.stokesDivT(op, src, tu, L, all, false);
    for (int i = 0; i < velocitySweeps; ++i)
      for (int k = 0; k < 3; ++k) s.p2Sor(op, ru[k], tu[k], 1.0, L, fv, false);
    s.stokesDiv(op, ru, dst, L, all);
    s.divideBy(dst, dst, lumped, L, all);
  };
  auto scaleInto = [&](int dst, int src) {
    const double inv = 1.0 / std::sqrt(s.dot(src, src, L, all));
    s.lincomb(dst, L, all, 1, &inv, &src, false, 0.0);
  };
  scaleInto(itv, itv);
  E(itv, aux);
  double radius = 0.0;
  for (int i = 0; i < iters; ++i) {
    scaleInto(itv, aux);
    E(itv, aux);
    radius = s.dot(itv, aux, L, all);
  }
  for (int id : {ones, lumped, itv, aux}) s.fns.erase(id);
  s.ops.erase(mass);
  return radius;
}

// The block operator on the coarse unknowns, probed column by column with unit vectors,
// symmetrised, and its pseudo-inverse uploaded.
void StokesGmg::buildCoarse() {
  if (coarseN >= 0) return;
  const unsigned fv = HG_INNER | HG_NEUMANN | HG_FREESLIP;
  const int Lv = minL + 1, Lp = minL;
  P2Additive& av = s.p2Additive(Lv);
  P2Additive& ap = s.p2Additive(Lp);
  if (av.hostOwner.empty() || ap.hostOwner.empty()) {  // too large for host-side owner lists
    coarseIterative = true;
    coarseN = 0;
    return;
  }
  std::vector<int64_t> idx;
  std::vector<unsigned char> comp;
  for (int k = 0; k < 3; ++k)
    for (size_t i = 0; i < av.hostOwner.size(); ++i)
      if (av.hostOwnerType[i] & fv) {
        idx.push_back(av.hostOwner[i]);
        comp.push_back((unsigned char)k);
      }
  for (size_t i = 0; i < ap.hostOwner.size(); ++i) {
    idx.push_back(ap.hostOwner[i]);
    comp.push_back(3);
  }
  const int n = (int)idx.size();
  if (n > kCoarseMax) {
    coarseIterative = true;
    coarseN = 0;
    return;
  }
  const int64_t nv = s.disc.level(Lv).total, np = s.disc.level(Lp).total;
  int e[4], y[4];
  for (int k = 0; k < 4; ++k) {
    e[k] = s.createFunction(k < 3 ? Lv : Lp, k < 3 ? Lv : Lp, 8);
    y[k] = s.createFunction(k < 3 ? Lv : Lp, k < 3 ? Lv : Lp, 8);
  }
  auto lvl = [&](int k) { return k < 3 ? Lv : Lp; };
  auto len = [&](int k) { return k < 3 ? nv : np; };
  std::vector<std::vector<double>> he(4), hy(4);
  for (int k = 0; k < 4; ++k) {
    he[k].assign((size_t)len(k), 0.0);
    hy[k].assign((size_t)len(k), 0.0);
  }
  std::vector<double> K((size_t)n * n);
  for (int j = 0; j < n; ++j) {
    he[comp[j]][(size_t)idx[j]] = 1.0;
    for (int k = 0; k < 4; ++k)
      cudaCheck(cudaMemcpyAsync(s.data(e[k], lvl(k)), he[k].data(), (size_t)len(k) * 8, cudaMemcpyHostToDevice, s.stream),
                "coarse");
    cudaCheck(cudaStreamSynchronize(s.stream), "coarse");
    he[comp[j]][(size_t)idx[j]] = 0.0;
    s.stokesApply(op, e, e[3], y, y[3], minL, HG_INNER | HG_NEUMANN, HG_ALL);
    for (int k = 0; k < 4; ++k)
      cudaCheck(cudaMemcpyAsync(hy[k].data(), s.data(y[k], lvl(k)), (size_t)len(k) * 8, cudaMemcpyDeviceToHost, s.stream),
                "coarse");
    cudaCheck(cudaStreamSynchronize(s.stream), "coarse");
    for (int i = 0; i < n; ++i) K[(size_t)i * n + j] = hy[comp[i]][(size_t)idx[i]];
  }
  for (int k = 0; k < 4; ++k) {
    s.fns.erase(e[k]);
    s.fns.erase(y[k]);
  }
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      const double m = 0.5 * (K[(size_t)i * n + j] + K[(size_t)j * n + i]);
      K[(size_t)i * n + j] = K[(size_t)j * n + i] = m;
    }
  const std::vector<double> P = symmetricPinv(K, n);
  coarseIdx.reset(new DevBuf());
  coarseIdx->alloc((size_t)std::max(n, 1) * sizeof(int64_t));
  coarseComp.reset(new DevBuf());
  coarseComp->alloc((size_t)std::max(n, 1));
  coarseInv.reset(new DevBuf());
  coarseInv->alloc((size_t)std::max(n, 1) * std::max(n, 1) * sizeof(double));
  if (n) {
    cudaCheck(cudaMemcpyAsync(coarseIdx->p, idx.data(), (size_t)n * 8, cudaMemcpyHostToDevice, s.stream), "coarse");
    cudaCheck(cudaMemcpyAsync(coarseComp->p, comp.data(), (size_t)n, cudaMemcpyHostToDevice, s.stream), "coarse");
    cudaCheck(cudaMemcpyAsync(coarseInv->p, P.data(), P.size() * 8, cudaMemcpyHostToDevice, s.stream), "coarse");
    cudaCheck(cudaStreamSynchronize(s.stream), "coarse");
  }
  coarseN = n;
}

// x += K^+ (b - K x) on the coarse unknowns
void StokesGmg::coarseSolve(const int u[3], int p, const int f[3], int g) {
  buildCoarse();
  if (coarseIterative) {
    coarseIterations = stokesMinres(s, op, u, p, f, g, minL, 2, kCoarseMaxIter, kCoarseTol, nullptr, nullptr, 0);
    return;
  }
  if (coarseN == 0) return;
  stokesResidual(s, op, u, p, f, g, tu, tp, minL);
  dev::BlockPtrs bp;
  for (int k = 0; k < 3; ++k) {
    bp.r[k] = (const double*)s.data(tu[k], minL + 1);
    bp.x[k] = (double*)s.data(u[k], minL + 1);
  }
  bp.r[3] = (const double*)s.data(tp, minL);
  bp.x[3] = (double*)s.data(p, minL);
  dev::blockDenseCorrectKernel<<<(coarseN + dev::kBlock - 1) / dev::kBlock, dev::kBlock, (size_t)coarseN * 8,
                                  s.stream>>>((const int64_t*)coarseIdx->p, (const unsigned char*)coarseComp->p, coarseN,
                                              (const double*)coarseInv->p, bp);
  ++s.launches;
  cudaCheck(cudaGetLastError(), "Stokes coarse solve");
  for (int k = 0; k < 3; ++k) s.communicate(u[k], minL + 1, (1 << G_COUNT) - 1);
  s.communicate(p, minL, (1 << G_COUNT) - 1);
}

void StokesGmg::solveRecursively(const int u[3], int p, const int f[3], int g, int L) {
  const unsigned fv = HG_INNER | HG_NEUMANN, fp = HG_ALL;
  if (L == minL) {
    coarseSolve(u, p, f, g);
    return;
  }
  for (int i = 0; i < pre; ++i) smooth(u, p, f, g, L);
  stokesResidual(s, op, u, p, f, g, tu, tp, L);
  const double one = 1.0;
  for (int k = 0; k < 3; ++k) {
    s.p2Restrict(tu[k], L, fv);
    s.lincomb(f[k], L, fv, 1, &one, &tu[k], false, 0.0);  // lattice level L = P2 level L - 1
    s.lincomb(u[k], L, HG_ALL, 0, nullptr, nullptr, false, 0.0);
  }
  s.restrictFn(tp, L, fp);
  s.lincomb(g, L - 1, fp, 1, &one, &tp, false, 0.0);
  s.lincomb(p, L - 1, HG_ALL, 0, nullptr, nullptr, false, 0.0);
  solveRecursively(u, p, f, g, L - 1);
  for (int k = 0; k < 3; ++k) s.p2Prolongate(u[k], L - 1, fv, true);
  s.prolongate(p, L - 1, fp, true);
  for (int i = 0; i < post; ++i) smooth(u, p, f, g, L);
}

int StokesGmg::solveTo(const int u[3], int p, const int f[3], int g, int L, double tol, int maxIter, double* relRes,
                       double* history, int historyCap) {
  argCheck(L >= minL && L <= maxL, "Stokes multigrid: level outside the solver's range");
  const double r0 = residualNorm(u, p, f, g, L);
  double rel = 1.0;
  int it = 0;
  while (it < maxIter && rel > tol && r0 > 0.0) {
    solveRecursively(u, p, f, g, L);
    ++it;
    rel = residualNorm(u, p, f, g, L) / r0;
    if (history && it <= historyCap) history[it - 1] = rel;
  }
  if (relRes) *relRes = r0 > 0.0 ? rel : 0.0;
  return it;
}

int stokesMinres(Storage& s, int op, const int u[3], int p, const int f[3], int g, int L, int nu, int maxIter,
                 double tol, double* relRes, double* history, int historyCap, int precondPrec) {
  const unsigned fv = HG_INNER | HG_NEUMANN, fp = HG_ALL;
  const int Lv = L + 1, Lp = L;
  std::vector<int> made;
  auto fnV = [&](int minL) {
    const int id = s.createFunction(minL, Lv, 8);
    made.push_back(id);
    return id;
  };
  auto fnP = [&]() {
    const int id = s.createFunction(Lp, Lp, 8);
    made.push_back(id);
    return id;
  };
  struct Blk {
    int u[3];
    int p;
  };
  auto blk = [&]() {
    Blk b;
    for (int k = 0; k < 3; ++k) b.u[k] = fnV(Lv);
    b.p = fnP();
    return b;
  };
  Blk x{{u[0], u[1], u[2]}, p}, rhs{{f[0], f[1], f[2]}, g};
  Blk vPrev = blk(), v = blk(), vNext = blk(), z = blk(), wPrev = blk(), w = blk(), wNext = blk(), az = blk();
  auto dot = [&](const Blk& a, const Blk& b) {
    double t = s.dot(a.p, b.p, Lp, fp);
    for (int k = 0; k < 3; ++k) t += s.dot(a.u[k], b.u[k], Lv, fv);
    return t;
  };
  // dst = sum_i a_i src_i (up to three terms) on the unknowns of every block
  auto comb = [&](const Blk& dst, int n, const double* a, const Blk* src, bool add) {
    for (int k = 0; k < 3; ++k) {
      int ids[3];
      for (int i = 0; i < n; ++i) ids[i] = src[i].u[k];
      s.lincomb(dst.u[k], Lv, fv, n, a, ids, add, 0.0);
    }
    int ids[3];
    for (int i = 0; i < n; ++i) ids[i] = src[i].p;
    s.lincomb(dst.p, Lp, fp, n, a, ids, add, 0.0);
  };
  auto applyK = [&](const Blk& src, const Blk& dst) { s.stokesApply(op, src.u, src.p, dst.u, dst.p, L, fv, fp); };
  // preconditioner: velocity V-cycles (symmetric), pressure / lumped mass; zero-mean pressure
  const int mass = s.createOperator(FORM_MASS, Lp, Lp);
  const int ones = fnP(), lumped = fnP();
  s.lincomb(ones, Lp, fp, 0, nullptr, nullptr, false, 1.0);
  s.apply(mass, ones, lumped, Lp, fp, 0);
  const double nP = s.dot(ones, ones, Lp, fp);
  argCheck(precondPrec == 8 || precondPrec == 4, "preconditioner precision must be 8 or 4");
  // One V-cycle solver per velocity component, each with its own x and b (FP32 for a
  // mixed-precision preconditioner; cast at level L) and its own P2 scratch lane. The three cycles
  // of an application are independent. After the first application, which runs them in order and
  // builds every table, scratch function and graph they use, they run concurrently on three
  // streams, when the coarse level is solved directly on the device: a CG coarse solve takes dot
  // products, whose partial sums share one buffer per level.
  std::unique_ptr<P2Gmg> mg[3];
  int px[3], pb[3];
  for (int k = 0; k < 3; ++k) {
    mg[k].reset(new P2Gmg(s, op, 0, L, nu, nu, 1.0, 1000, 1e-14, precondPrec));
    mg[k]->symmetric = true;
    mg[k]->lane = k;
    px[k] = s.createFunction(1, Lv, precondPrec);
    pb[k] = s.createFunction(1, Lv, precondPrec);
    made.push_back(px[k]);
    made.push_back(pb[k]);
  }
  struct Lanes {  // the two extra streams and the fork / join events, released on every exit
    cudaStream_t aux[2] = {nullptr, nullptr};
    cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr};
    ~Lanes() {
      for (cudaStream_t st : aux)
        if (st) cudaStreamDestroy(st);
      for (cudaEvent_t e : {fork, join[0], join[1]})
        if (e) cudaEventDestroy(e);
    }
  } lanes;
  const bool lanesOk = s.concurrentComponents && mg[0]->buildCoarseDirect();
  if (lanesOk) {
    for (int k = 0; k < 2; ++k) {
      cudaCheck(cudaStreamCreateWithFlags(&lanes.aux[k], cudaStreamNonBlocking), "stream");
      cudaCheck(cudaEventCreateWithFlags(&lanes.join[k], cudaEventDisableTiming), "event");
    }
    cudaCheck(cudaEventCreateWithFlags(&lanes.fork, cudaEventDisableTiming), "event");
  }
  bool concurrent = false;
  auto precond = [&](const Blk& src, const Blk& dst) {
    const double one = 1.0;
    struct StreamGuard {  // the storage's stream, restored on every exit
      Storage& s;
      cudaStream_t home;
      ~StreamGuard() { s.stream = home; }
    } guard{s, s.stream};
    if (concurrent) {
      cudaCheck(cudaEventRecord(lanes.fork, guard.home), "event");
      for (int k = 0; k < 2; ++k) cudaCheck(cudaStreamWaitEvent(lanes.aux[k], lanes.fork, 0), "wait");
    }
    for (int k = 0; k < 3; ++k) {
      s.stream = concurrent && k > 0 ? lanes.aux[k - 1] : guard.home;
      s.copyCast(pb[k], src.u[k], Lv, fv, false);
      for (int l = 1; l <= Lv; ++l) s.lincomb(px[k], l, HG_ALL, 0, nullptr, nullptr, false, 0.0);
      mg[k]->runCycle(px[k], pb[k], L);
      s.copyCast(dst.u[k], px[k], Lv, fv, false);
      if (concurrent && k > 0) cudaCheck(cudaEventRecord(lanes.join[k - 1], s.stream), "event");
    }
    s.stream = guard.home;
    if (concurrent)
      for (int k = 0; k < 2; ++k) cudaCheck(cudaStreamWaitEvent(guard.home, lanes.join[k], 0), "wait");
    concurrent = lanesOk;
    s.divideBy(dst.p, src.p, lumped, Lp, fp);
    const double mean = s.dot(dst.p, ones, Lp, fp) / nP;
    s.lincomb(dst.p, Lp, fp, 1, &one, &dst.p, false, -mean);
  };
  // v1 = f - K x, z1 = M^-1 v1, gamma1 = sqrt(<z1, v1>)
  applyK(x, az);
  {
    const double a[2] = {1.0, -1.0};
    const Blk src[2] = {rhs, az};
    comb(v, 2, a, src, false);
  }
  precond(v, z);
  double gamma = std::sqrt(std::max(dot(z, v), 0.0)), gammaPrev = 1.0;
  const double gamma1 = gamma;
  double eta = gamma, c = 1.0, cPrev = 1.0, sn = 0.0, snPrev = 0.0;
  int it = 0;
  double rel = gamma1 > 0.0 ? 1.0 : 0.0;
  while (it < maxIter && rel > tol && gamma > 0.0) {
    ++it;
    {  // z_j = z_j / gamma_j
      const double a = 1.0 / gamma;
      comb(z, 1, &a, &z, false);
    }
    applyK(z, az);
    const double delta = dot(az, z);
    {  // v_{j+1} = A z_j - delta / gamma_j v_j - gamma_j / gamma_{j-1} v_{j-1}
      const double a[3] = {1.0, -delta / gamma, -gamma / gammaPrev};
      const Blk src[3] = {az, v, vPrev};
      comb(vNext, it == 1 ? 2 : 3, a, src, false);
    }
    precond(vNext, az);  // az now holds z_{j+1}
    const double gammaNext = std::sqrt(std::max(dot(az, vNext), 0.0));
    const double a0 = c * delta - cPrev * sn * gamma;
    const double a1 = std::sqrt(a0 * a0 + gammaNext * gammaNext);
    const double a2 = sn * delta + cPrev * c * gamma;
    const double a3 = snPrev * gamma;
    cPrev = c;
    snPrev = sn;
    c = a0 / a1;
    sn = gammaNext / a1;
    {  // w_{j+1} = (z_j - a3 w_{j-1} - a2 w_j) / a1
      const double a[3] = {1.0 / a1, -a3 / a1, -a2 / a1};
      const Blk src[3] = {z, wPrev, w};
      comb(wNext, 3, a, src, false);
    }
    {  // x += c eta w_{j+1}
      const double a = c * eta;
      comb(x, 1, &a, &wNext, true);
    }
    eta = -sn * eta;
    rel = std::fabs(eta) / gamma1;
    if (history && it <= historyCap) history[it - 1] = rel;
    // rotate: v_{j-1} <- v_j <- v_{j+1}, w_{j-1} <- w_j <- w_{j+1}, z <- z_{j+1}
    std::swap(vPrev, v);
    std::swap(v, vNext);
    std::swap(wPrev, w);
    std::swap(w, wNext);
    std::swap(z, az);
    gammaPrev = gamma;
    gamma = gammaNext;
  }
  {
    const double one = 1.0;
    const double mean = s.dot(x.p, ones, Lp, fp) / nP;
    s.lincomb(x.p, Lp, fp, 1, &one, &x.p, false, -mean);
  }
  for (int k = 0; k < 3; ++k) s.communicate(x.u[k], Lv, (1 << G_COUNT) - 1);
  s.communicate(x.p, Lp, (1 << G_COUNT) - 1);
  s.ops.erase(mass);
  for (int id : made) s.fns.erase(id);
  if (relRes) *relRes = rel;
  return it;
}

int P2Gmg::solveTo(int x, int b, int L, double tol, int maxIter, double* relRes, double* history, int historyCap) {
  const unsigned flag = HG_INNER | HG_NEUMANN;
  argCheck(L >= minL && L <= maxL, "P2 multigrid: level outside the solver's range");
  argCheck(s.fn(x).prec == 8 && s.fn(b).prec == 8, "P2 multigrid: FP64 functions required");
  const int Lf = L + 1;
  s.p2Apply(op, x, tmp, b, L, flag, 2);
  const double r0 = std::sqrt(s.dot(tmp, tmp, Lf, flag));
  double rel = 1.0;
  int it = 0;
  while (it < maxIter && rel > tol && r0 > 0.0) {
    runCycle(x, b, L);
    ++it;
    s.p2Apply(op, x, tmp, b, L, flag, 2);
    rel = std::sqrt(s.dot(tmp, tmp, Lf, flag)) / r0;
    if (history && it <= historyCap) history[it - 1] = rel;
  }
  if (relRes) *relRes = r0 > 0.0 ? rel : 0.0;
  return it;
}

}  // namespace hg
