// Continuous-batching solve server: worker threads, admission by device footprint, resident
// hierarchies per shape (see server.hpp). Every request's work runs on the stream of its own
// storage; the only synchronisations are per stream (convergence checks of that request).
#include "server.hpp"

#include <algorithm>
#include <set>
#include <cmath>

#include "../../include/hyteg_b200.h"
#include "kernels.cuh"
#include "solvers.hpp"
#include "storage.hpp"
#include "topology.hpp"

namespace hg {

ServerSlot::~ServerSlot() = default;
BatchSlot::~BatchSlot() = default;

Server::Server(int workers, int64_t budgetBytes, int precision)
    : precision_(precision), budget_(budgetBytes), t0_(std::chrono::steady_clock::now()) {
  argCheck(workers >= 1 && workers <= 256, "workers must be in [1, 256]");
  argCheck(budgetBytes > 0, "HBM budget must be positive");
  argCheck(precision == 4 || precision == 8, "precision must be 4 (mixed) or 8 (FP64)");
  int device = 0;
  cudaCheck(cudaGetDevice(&device), "cudaGetDevice");
  for (int i = 0; i < workers; ++i)
    threads_.emplace_back([this, device]() {
      cudaSetDevice(device);
      worker();
    });
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stopping_ = true;
    for (auto& r : queue_) {
      r->status = -1;
      r->error = "server stopped before the request was admitted";
    }
    queue_.clear();
  }
  cv_.notify_all();
  doneCv_.notify_all();
  for (auto& t : threads_) t.join();
  idle_.clear();
  idleBatch_.clear();
}

double Server::now() const {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
}

int64_t Server::estimate(int k, int level) const {
  auto it = measured_.find({k, level});
  if (it != measured_.end()) return it->second;
  // not built yet: level buffer of the finest level times the bytes per slot of the functions,
  // spare buffers and tables (FP64 x, b; FP32 or FP64 multigrid workspace), plus the hierarchy
  const int64_t m = int64_t(k) << level;
  const int64_t slots = 6 * k * k * k * ((m / k + 1) * (m / k + 2) * (m / k + 3) / 6) + 64 * m * m;
  const int64_t perSlot = precision_ == 4 ? 56 : 48;
  return slots * perSlot;
}

int64_t Server::submit(int k, int level, double coefficient, uint64_t seed, double tol, int maxIter,
                       bool keepSolution) {
  argCheck(k >= 1 && k <= 16, "sub-cubes per direction must be in [1, 16]");
  argCheck(level >= 2 && level <= 8, "level must be in [2, 8]");
  argCheck(coefficient > 0.0 && std::isfinite(coefficient), "coefficient must be positive");
  argCheck(tol > 0.0 && maxIter >= 1, "tolerance must be positive and max_iter at least 1");
  auto r = std::make_shared<ServerRequest>();
  r->k = k;
  r->level = level;
  r->coefficient = coefficient;
  r->seed = seed;
  r->tol = tol;
  r->maxIter = maxIter;
  r->keepSolution = keepSolution;
  const int64_t m = (int64_t(k) << level) - 1;
  r->innerDofs = m * m * m;
  {
    std::lock_guard<std::mutex> lk(mu_);
    argCheck(!stopping_, "server is stopping");
    r->id = nextId_++;
    r->tSubmit = now();
    all_[r->id] = r;
    queue_.push_back(r);
  }
  cv_.notify_all();
  return r->id;
}

std::unique_ptr<ServerSlot> Server::buildSlot(int k, int level) {
  std::unique_ptr<ServerSlot> s(new ServerSlot());
  s->k = k;
  s->level = level;
  const double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
  Topology t = meshCuboid(lo, hi, k, k, k);
  t.setBoundaryFlags(1, 0);
  s->st.reset(new Storage(t, level));
  Storage& st = *s->st;
  s->x = st.createFunction(0, level, 8);
  s->b = st.createFunction(0, level, 8);
  s->op = st.createOperator(0, 0, level);
  st.reassembleOperator(s->op, true);  // builds the term lists now, so requests only run the kernels
  s->gmg = st.nextId++;
  st.gmgs[s->gmg].reset(new Gmg(st, s->op, 0, level, 3, 3, 1.0, 0, 200, 1e-16, precision_));
  // three iterations before the footprint is taken: eager ones, which create the smoother's spare
  // buffers, until the buffer state settles, then the capture of the cycle's CUDA graph, so that
  // requests only replay it (no capture or instantiation while other requests run)
  st.fillRandom(s->b, level, HG_INNER, 0, -1.0, 1.0);
  double rel = 0;
  st.gmgs[s->gmg]->solveTo(s->x, s->b, level, 1e-30, 3, &rel, nullptr, 0);
  cudaCheck(cudaStreamSynchronize(st.stream), "slot build");
  s->bytes = st.deviceBytes();
  return s;
}

std::unique_ptr<BatchSlot> Server::buildBatchSlot(int k, int level, int copies) {
  std::unique_ptr<BatchSlot> s(new BatchSlot());
  s->k = k;
  s->level = level;
  s->copies = copies;
  Topology t = meshCuboidCopies(k, copies);
  t.setBoundaryFlags(1, 0);
  s->st.reset(new Storage(t, level));
  Storage& st = *s->st;
  s->x = st.createFunction(0, level, 8);
  s->b = st.createFunction(0, level, 8);
  s->xOut = st.createFunction(level, level, 8);
  s->op = st.createOperator(0, 0, level);
  st.reassembleOperator(s->op, true);  // the term lists, so that batches only run the kernels
  s->gmg = st.nextId++;
  st.gmgs[s->gmg].reset(new Gmg(st, s->op, 0, level, 3, 3, 1.0, 0, 200, 1e-16, precision_));
  if (st.gmgs[s->gmg]->deviceCoarse()) st.gmgs[s->gmg]->setCoarseGroups(copies);  // copies stop on their own
  s->seeds.reset(new DevBuf());
  s->seeds->alloc((size_t)copies * sizeof(uint64_t));
  s->norms.reset(new DevBuf());
  s->norms->alloc((size_t)copies * sizeof(double));
  // three iterations over all copies (eager ones, then the capture), so that every buffer and
  // graph exists before the footprint
  const dev::BatchMap bm = st.batchMap(level, copies);
  std::vector<uint64_t> seeds((size_t)copies, 1);
  cudaCheck(cudaMemcpyAsync(s->seeds->p, seeds.data(), seeds.size() * 8, cudaMemcpyHostToDevice, st.stream), "seeds");
  st.fillRandomBatch(s->b, level, HG_INNER, bm, (const uint64_t*)s->seeds->p, copies, -1.0, 1.0);
  std::vector<double> tol((size_t)copies, 1e-30), rel((size_t)copies);
  std::vector<int> maxIt((size_t)copies, 3), its((size_t)copies);
  st.gmgs[s->gmg]->solveToBatch(s->x, s->b, s->xOut, level, tol.data(), maxIt.data(), bm, copies,
                                (double*)s->norms->p, its.data(), rel.data());
  cudaCheck(cudaStreamSynchronize(st.stream), "batch slot build");
  s->bytes = st.deviceBytes();
  return s;
}

void Server::setBatching(int maxLevel) {
  std::lock_guard<std::mutex> lk(mu_);
  batchMaxLevel_ = maxLevel;
}

void Server::prewarmBatch(int k, int level, int copies) {
  argCheck(copies >= 2 && copies <= 64, "batch copies must be in [2, 64]");
  std::unique_ptr<BatchSlot> s = buildBatchSlot(k, level, copies);
  std::lock_guard<std::mutex> lk(mu_);
  if (active_ + resident_ + s->bytes > budget_) throw Error(HG_ERR_OOM, "batch prewarm exceeds the HBM budget");
  resident_ += s->bytes;
  peak_ = std::max(peak_, active_ + resident_);
  s->lastUse = ++useClock_;
  idleBatch_.push_back(std::move(s));
}

// A batch: one solve of up to s.copies requests of one shape in the union hierarchy. The cells of
// copy i take request i's coefficient (device re-assembly), copy i's right-hand side is the one
// its seed gives a single cube, the other copies get 0.
void Server::runBatch(std::vector<std::shared_ptr<ServerRequest>>& rs, BatchSlot& s) {
  Storage& st = *s.st;
  const int L = s.level, active = (int)rs.size();
  const dev::BatchMap bm = st.batchMap(L, s.copies);
  auto& cells = const_cast<Topology&>(st.disc.topo()).cells;
  const size_t per = cells.size() / (size_t)s.copies;
  bool changed = false;
  for (int i = 0; i < active; ++i)
    for (size_t c = (size_t)i * per; c < (size_t)(i + 1) * per; ++c)
      if (cells[c].k != rs[(size_t)i]->coefficient) {
        cells[c].k = rs[(size_t)i]->coefficient;
        changed = true;
      }
  if (changed) st.reassembleOperator(s.op, true);
  std::vector<uint64_t> seeds((size_t)s.copies, 0);
  std::vector<double> tol((size_t)active), rel((size_t)active);
  std::vector<int> maxIt((size_t)active), its((size_t)active);
  for (int i = 0; i < active; ++i) {
    seeds[(size_t)i] = rs[(size_t)i]->seed;
    tol[(size_t)i] = rs[(size_t)i]->tol;
    maxIt[(size_t)i] = rs[(size_t)i]->maxIter;
  }
  {
    const double t = now();
    std::lock_guard<std::mutex> lk(mu_);
    for (auto& r : rs) r->tSolve = t;
  }
  cudaCheck(cudaMemcpyAsync(s.seeds->p, seeds.data(), seeds.size() * 8, cudaMemcpyHostToDevice, st.stream), "seeds");
  st.fillRandomBatch(s.b, L, HG_INNER, bm, (const uint64_t*)s.seeds->p, active, -1.0, 1.0);
  st.lincomb(s.x, L, HG_ALL, 0, nullptr, nullptr, false, 0.0);
  st.gmgs[s.gmg]->solveToBatch(s.x, s.b, s.xOut, L, tol.data(), maxIt.data(), bm, active, (double*)s.norms->p,
                               its.data(), rel.data());
  for (int i = 0; i < active; ++i) {
    ServerRequest& r = *rs[(size_t)i];
    r.iterations = its[(size_t)i];
    r.relResidual = rel[(size_t)i];
    if (r.keepSolution) {  // the copy's slots, at their places in a single cube's level buffer
      r.solution.assign((size_t)(bm.aBase[3] + bm.size[3]), 0.0);
      for (int q = 0; q < 4; ++q)
        if (bm.size[q] > 0)
          cudaCheck(cudaMemcpyAsync(r.solution.data() + bm.aBase[q], (const double*)st.data(s.xOut, L) + bm.uBase[q] + i * bm.size[q],
                                    (size_t)bm.size[q] * sizeof(double), cudaMemcpyDeviceToHost, st.stream),
                    "solution download");
    }
  }
  cudaCheck(cudaStreamSynchronize(st.stream), "batch sync");
}

void Server::prewarm(int k, int level) {
  std::unique_ptr<ServerSlot> s = buildSlot(k, level);
  std::lock_guard<std::mutex> lk(mu_);
  measured_[{k, level}] = s->bytes;
  if (active_ + resident_ + s->bytes > budget_) throw Error(HG_ERR_OOM, "prewarm exceeds the HBM budget");
  resident_ += s->bytes;
  peak_ = std::max(peak_, active_ + resident_);
  s->lastUse = ++useClock_;
  ++shapeSlots_[{k, level}];
  idle_.push_back(std::move(s));
}

void Server::run(ServerRequest& r, ServerSlot& s) {
  Storage& st = *s.st;
  const int L = r.level;
  // constant coefficient: scale every macro-cell and re-assemble the stencils in place on the
  // device (no device allocation or release, which would synchronise the whole device and stall
  // the other requests; the term lists are built by the slot's first re-assembly)
  auto& cells = const_cast<Topology&>(st.disc.topo()).cells;
  if (cells.empty() || cells[0].k != r.coefficient) {
    for (auto& c : cells) c.k = r.coefficient;
    st.reassembleOperator(s.op, true);
  }
  r.tSolve = now();
  st.fillRandom(s.b, L, HG_INNER, r.seed, -1.0, 1.0);
  st.lincomb(s.x, L, HG_ALL, 0, nullptr, nullptr, false, 0.0);
  double rel = 0;
  r.iterations = st.gmgs[s.gmg]->solveTo(s.x, s.b, L, r.tol, r.maxIter, &rel, nullptr, 0);
  r.relResidual = rel;
  if (r.keepSolution) {
    r.solution.resize((size_t)st.levels[L].lay->total);
    cudaCheck(cudaMemcpyAsync(r.solution.data(), st.data(s.x, L), r.solution.size() * sizeof(double),
                              cudaMemcpyDeviceToHost, st.stream),
              "solution download");
  }
  cudaCheck(cudaStreamSynchronize(st.stream), "request sync");
}

void Server::worker() {
  for (;;) {
    std::shared_ptr<ServerRequest> r;
    std::unique_ptr<ServerSlot> slot;
    std::unique_ptr<BatchSlot> bslot;
    std::vector<std::shared_ptr<ServerRequest>> batch;
    std::vector<std::unique_ptr<ServerSlot>> evict;
    int64_t est = 0;
    {
      std::unique_lock<std::mutex> lk(mu_);
      for (;;) {
        if (stopping_) return;
        // Scan the queue in arrival order; the first request that can start now starts. A request
        // whose shape has hierarchies that are all busy waits for one of them (building another
        // takes seconds, a solve milliseconds) and the requests behind it may pass it; a request
        // that waits for HBM is passed by none.
        // One pass over the queue: the requests of every shape (for batching) and the shapes found
        // to wait, whose later requests are skipped at once (a scan is linear in the queue).
        bool evicted = false;
        std::map<std::pair<int, int>, int> queued;
        std::set<std::pair<int, int>> waiting;
        if (batchMaxLevel_ >= 0 && !idleBatch_.empty())
          for (auto& q : queue_) ++queued[{q->k, q->level}];
        for (size_t qi = 0; qi < queue_.size() && !r && !bslot && !evicted; ++qi) {
          std::shared_ptr<ServerRequest> h = queue_[qi];
          const std::pair<int, int> shape{h->k, h->level};
          if (waiting.count(shape)) continue;
          auto same = std::find_if(idle_.begin(), idle_.end(), [&](const std::unique_ptr<ServerSlot>& s) {
            return s->k == h->k && s->level == h->level;
          });
          if (same == idle_.end() && h->level <= batchMaxLevel_ && !idleBatch_.empty()) {
            // no single hierarchy of this shape is free and requests of the shape wait, in arrival
            // order: with two or more, the smallest idle union hierarchy of the shape that takes
            // them all (else the largest) takes the first of them
            const int nSame = queued[shape];
            int best = -1;
            for (int i = 0; i < (int)idleBatch_.size() && nSame >= 2; ++i) {
              const BatchSlot& b = *idleBatch_[(size_t)i];
              if (b.k != h->k || b.level != h->level) continue;
              if (best < 0) {
                best = i;
                continue;
              }
              const int cb = idleBatch_[(size_t)best]->copies;
              const bool fitsB = b.copies >= nSame, fitsBest = cb >= nSame;
              if ((fitsB && (!fitsBest || b.copies < cb)) || (!fitsB && !fitsBest && b.copies > cb)) best = i;
            }
            if (best >= 0) {
              bslot = std::move(idleBatch_[(size_t)best]);
              idleBatch_.erase(idleBatch_.begin() + best);
              resident_ -= bslot->bytes;
              active_ += bslot->bytes;
              std::deque<std::shared_ptr<ServerRequest>> rest;
              for (auto& q : queue_) {
                if ((int)batch.size() < bslot->copies && q->k == h->k && q->level == h->level)
                  batch.push_back(q);
                else
                  rest.push_back(q);
              }
              queue_.swap(rest);
              break;
            }
          }
          if (same != idle_.end()) {  // a resident hierarchy of this shape is free
            slot = std::move(*same);
            idle_.erase(same);
            resident_ -= slot->bytes;
            active_ += slot->bytes;
            r = h;
            queue_.erase(queue_.begin() + (std::ptrdiff_t)qi);
            break;
          }
          if (shapeSlots_[shape] > 0) {  // its shape's hierarchies are busy: wait for one
            waiting.insert(shape);
            continue;
          }
          est = estimate(h->k, h->level);
          while (active_ + resident_ + est > budget_ && !idle_.empty()) {  // release LRU idle hierarchies
            auto lru = std::min_element(idle_.begin(), idle_.end(),
                                        [](const std::unique_ptr<ServerSlot>& a, const std::unique_ptr<ServerSlot>& b) {
                                          return a->lastUse < b->lastUse;
                                        });
            resident_ -= (*lru)->bytes;
            --shapeSlots_[{(*lru)->k, (*lru)->level}];
            evict.push_back(std::move(*lru));
            idle_.erase(lru);
          }
          if (active_ + resident_ + est <= budget_) {  // build a hierarchy for it
            active_ += est;
            ++shapeSlots_[{h->k, h->level}];
            r = h;
            queue_.erase(queue_.begin() + (std::ptrdiff_t)qi);
            break;
          }
          if (active_ == 0 && idle_.empty()) {  // cannot fit even on an empty device budget
            h->status = -1;
            h->error = "request exceeds the HBM budget";
            h->tEnd = now();
            ++failed_;
            queue_.erase(queue_.begin() + (std::ptrdiff_t)qi);
            --queued[shape];
            --qi;
            doneCv_.notify_all();
            continue;
          }
          evicted = !evict.empty();  // free the evicted memory, then look again
          break;                     // else it waits for HBM, and so do the requests behind it
        }
        if (r || bslot || evicted) break;
        cv_.wait(lk);
      }
      if (r) {
        r->status = 1;
        r->tStart = now();
        r->builtHierarchy = !slot;
        ++admitted_;
        peak_ = std::max(peak_, active_ + resident_);
      }
      if (bslot) {
        const double t = now();
        for (auto& q : batch) {
          q->status = 1;
          q->tStart = t;
          q->batchSize = (int)batch.size();
          ++admitted_;
        }
        peak_ = std::max(peak_, active_ + resident_);
      }
    }
    evict.clear();
    if (bslot) {
      std::string err;
      try {
        runBatch(batch, *bslot);
      } catch (const std::exception& e) {
        err = e.what();
      }
      {
        std::lock_guard<std::mutex> lk(mu_);
        const double t = now();
        for (auto& q : batch) {
          q->tEnd = t;
          if (err.empty()) {
            q->status = 2;
            ++completed_;
          } else {
            q->status = -1;
            q->error = err;
            ++failed_;
          }
        }
        active_ -= bslot->bytes;
        if (err.empty()) {
          bslot->lastUse = ++useClock_;
          resident_ += bslot->bytes;
          idleBatch_.push_back(std::move(bslot));
        }
      }
      bslot.reset();  // a failed union hierarchy is released
      cv_.notify_all();
      doneCv_.notify_all();
      continue;
    }
    if (!r) continue;
    std::string err;
    if (!slot) {
      try {
        slot = buildSlot(r->k, r->level);
      } catch (const std::exception& e) {
        err = e.what();
      }
      std::lock_guard<std::mutex> lk(mu_);
      if (slot) {
        active_ += slot->bytes - est;
        measured_[{r->k, r->level}] = slot->bytes;
        peak_ = std::max(peak_, active_ + resident_);
      } else {
        active_ -= est;
        --shapeSlots_[{r->k, r->level}];
      }
    }
    if (slot && err.empty()) {
      try {
        run(*r, *slot);
      } catch (const std::exception& e) {
        err = e.what();
      }
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      r->tEnd = now();
      if (err.empty()) {
        r->status = 2;
        ++completed_;
      } else {
        r->status = -1;
        r->error = err;
        ++failed_;
      }
      if (slot) {
        active_ -= slot->bytes;
        if (err.empty()) {
          slot->lastUse = ++useClock_;
          resident_ += slot->bytes;
          idle_.push_back(std::move(slot));
        } else {
          --shapeSlots_[{r->k, r->level}];
        }
      }
    }
    slot.reset();  // a failed hierarchy is released
    cv_.notify_all();
    doneCv_.notify_all();
  }
}

bool Server::wait(int64_t id, double timeoutSeconds) {
  std::unique_lock<std::mutex> lk(mu_);
  auto it = all_.find(id);
  argCheck(it != all_.end(), "unknown request id");
  std::shared_ptr<ServerRequest> r = it->second;
  auto pred = [&]() { return r->status == 2 || r->status < 0; };
  if (timeoutSeconds < 0) {
    doneCv_.wait(lk, pred);
    return true;
  }
  return doneCv_.wait_for(lk, std::chrono::duration<double>(timeoutSeconds), pred);
}

std::shared_ptr<ServerRequest> Server::request(int64_t id) {
  std::lock_guard<std::mutex> lk(mu_);
  auto it = all_.find(id);
  argCheck(it != all_.end(), "unknown request id");
  return it->second;
}

void Server::stats(int64_t out[6]) {
  std::lock_guard<std::mutex> lk(mu_);
  out[0] = admitted_;
  out[1] = completed_;
  out[2] = failed_;
  out[3] = (int64_t)(idle_.size() + idleBatch_.size());
  out[4] = resident_;
  out[5] = peak_;
}

}  // namespace hg
