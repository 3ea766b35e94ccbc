// Continuous-batching solve server (host C++ behind the hg_server_* C-ABI).
//
// Requests are P1 Poisson solves on the unit cube split into k x k x k sub-cubes of 6
// tetrahedra, refined to a level L, with a constant coefficient, a seeded uniform[-1,1]
// right-hand side at the inner DoFs, x0 = 0 and a relative-residual target. A pool of worker
// threads admits requests in arrival order while a worker is free and the request's device
// footprint fits the HBM budget. Every admitted request runs on a resident hierarchy of its
// shape (k, L) with its own CUDA stream, so the sweeps of concurrent requests overlap on the
// device and requests that arrive while others run join as soon as a slot frees up. Idle
// hierarchies stay resident for the next request of their shape and are released, least
// recently used first, only when a new shape needs the memory. A hierarchy is built only for a
// shape that has none: a request whose shape's hierarchies are all busy waits for one (a build
// takes seconds, a solve milliseconds), and requests of other shapes behind it may pass it.
#pragma once

#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace hg {

struct Storage;
struct Gmg;
struct DevBuf;

struct ServerRequest {
  int64_t id = 0;
  int k = 1, level = 3;
  double coefficient = 1.0, tol = 1e-8;
  uint64_t seed = 0;
  int maxIter = 100;
  bool keepSolution = false;
  // results
  int status = 0;  // 0 queued, 1 running, 2 done, negative: failed
  std::string error;
  int iterations = 0;
  double relResidual = 0.0;
  double tSubmit = 0.0, tStart = 0.0, tSolve = 0.0, tEnd = 0.0;  // seconds since the server started
  bool builtHierarchy = false;  // no resident hierarchy of its shape was free: one was built for it
  int batchSize = 1;            // requests solved together with it in one union hierarchy (itself included)
  int64_t innerDofs = 0;
  std::vector<double> solution;  // level buffer of x at the request's level (keepSolution)
};

// One resident hierarchy: storage of one shape with operator, x, b and a multigrid solver.
struct ServerSlot {
  int k = 0, level = 0;
  std::unique_ptr<Storage> st;
  int op = -1, x = -1, b = -1, gmg = -1;
  int64_t bytes = 0;
  uint64_t lastUse = 0;
  ~ServerSlot();
};

// A resident union hierarchy: `copies` disjoint copies of one shape in one storage
// (meshCuboidCopies). Up to `copies` queued requests of that shape are solved in it together:
// every kernel launch of the solve covers all of them (Gmg::solveToBatch).
struct BatchSlot {
  int k = 0, level = 0, copies = 0;
  std::unique_ptr<Storage> st;
  int op = -1, x = -1, b = -1, xOut = -1, gmg = -1;
  std::unique_ptr<DevBuf> seeds, norms;  // per copy: seeds of the right-hand sides, residual norms
  int64_t bytes = 0;
  uint64_t lastUse = 0;
  ~BatchSlot();
};

class Server {
 public:
  Server(int workers, int64_t budgetBytes, int precision);
  ~Server();
  int64_t submit(int k, int level, double coefficient, uint64_t seed, double tol, int maxIter, bool keepSolution);
  void prewarm(int k, int level);
  // Batching: requests of levels up to maxLevel (-1: none) that find no single hierarchy of their
  // shape free but an idle union hierarchy of it, with at least one more request of that shape
  // queued, are solved together in it (under light load requests keep the latency of a single
  // solve; under a backlog they share launches); prewarmBatch builds one union hierarchy of
  // `copies` copies of a shape.
  void setBatching(int maxLevel);
  void prewarmBatch(int k, int level, int copies);
  bool wait(int64_t id, double timeoutSeconds);
  std::shared_ptr<ServerRequest> request(int64_t id);
  void stats(int64_t out[6]);  // admitted, completed, failed, resident slots, resident bytes, peak bytes

 private:
  void worker();
  bool admissible();                                      // under mu
  std::unique_ptr<ServerSlot> buildSlot(int k, int level);  // outside mu
  void run(ServerRequest& r, ServerSlot& s);
  std::unique_ptr<BatchSlot> buildBatchSlot(int k, int level, int copies);  // outside mu
  void runBatch(std::vector<std::shared_ptr<ServerRequest>>& rs, BatchSlot& s);
  int64_t estimate(int k, int level) const;                // under mu
  double now() const;

  const int precision_;
  const int64_t budget_;
  std::chrono::steady_clock::time_point t0_;
  std::mutex mu_;
  std::condition_variable cv_, doneCv_;
  bool stopping_ = false;
  std::deque<std::shared_ptr<ServerRequest>> queue_;
  std::map<int64_t, std::shared_ptr<ServerRequest>> all_;
  std::vector<std::unique_ptr<ServerSlot>> idle_;
  std::vector<std::unique_ptr<BatchSlot>> idleBatch_;
  int batchMaxLevel_ = -1;
  std::map<std::pair<int, int>, int64_t> measured_;  // footprint of a built slot per shape
  std::map<std::pair<int, int>, int> shapeSlots_;    // hierarchies per shape: idle, running or being built
  int64_t active_ = 0, resident_ = 0, peak_ = 0;      // bytes: admitted requests, idle slots
  int64_t nextId_ = 1, admitted_ = 0, completed_ = 0, failed_ = 0;
  uint64_t useClock_ = 0;
  int64_t reserved_ = 0;  // bytes reserved for the head request while its slot is built
  std::vector<std::thread> threads_;
};

}  // namespace hg
