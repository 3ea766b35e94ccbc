// Allocation-free variant of the dot product (hg_dot_noalloc).
//
// hg_dot keeps its per-block partial sums in a scratch buffer that the storage allocates.
// Callers that must not allocate device memory while they run -- for example a solver
// service that commits its whole device-memory budget at start-up and may not call
// cudaMalloc on the request path, or code running while another component owns the device
// allocator -- use this entry point instead: its scratch is the file-scope device array
// below, which every GPU that loads the library holds until the process exits.
#include <cuda_runtime.h>

#include <string>

#include "../../include/hyteg_b200.h"
#include "kernels.cuh"
#include "storage.hpp"

namespace {

// Maximum number of per-block partial sums of one call (512 KiB of doubles). A level of the
// 48-tet cube needs nCells*(2^L-3) + faces*ceil((2^L-2)/32) + edge/vertex blocks of them:
// about 13,200 at level 8 and 49,000 at level 10.
constexpr int kMaxPartials = 65536;
static __device__ __align__(256) double g_dotScratch[kMaxPartials];

// Makes the storage's device current for the lifetime of the guard (its stream and buffers
// belong to that device) and restores the caller's device afterwards.
struct DeviceGuard {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit DeviceGuard(int dev) {
    err = cudaGetDevice(&prev);
    if (err == cudaSuccess && prev != dev) err = cudaSetDevice(dev);
    else if (err == cudaSuccess) prev = -1;  // already current: nothing to restore
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// Device address of g_dotScratch on the storage's device (current when called), looked up on
// the storage's first call and kept in the storage. In host code the symbol g_dotScratch is a
// host-side stand-in, not a device address. A storage never outlives a cudaDeviceReset of its
// device (its buffers would be gone too), so a kept address is never stale.
int scratchFor(hg::Storage& s, double** out) {
  if (!s.noallocScratch) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_dotScratch);
    if (e != cudaSuccess) {
      hg::g_lastError = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
      return HG_ERR_CUDA;
    }
    s.noallocScratch = static_cast<double*>(p);
  }
  *out = s.noallocScratch;
  return HG_OK;
}

}  // namespace

extern "C" int hg_dot_noalloc(hg_storage* h, const void* a, const void* b, int precision, int level, unsigned flag,
                              double* result) {
  try {
    hg::argCheck(h != nullptr && h->s != nullptr, "null storage handle");
    hg::argCheck(a != nullptr && b != nullptr && result != nullptr, "null device pointer");
    hg::argCheck(precision == 8 || precision == 4, "precision must be 8 or 4");
    hg::Storage& s = *h->s;
    hg::argCheck(level >= 0 && level <= s.maxLevel(), "level out of range");
    const hg::LevelData& ld = s.levels[level];
    const int nb = ld.lv.nCellBlocks + ld.lv.nFaceBlocks + ld.lv.nLowBlocks;
    if (nb > kMaxPartials)
      throw hg::Error(HG_ERR_ARG, "hg_dot_noalloc: level " + std::to_string(level) + " needs " + std::to_string(nb) +
                                      " partial sums, more than the " + std::to_string(kMaxPartials) +
                                      " of its static scratch; use hg_dot");
    DeviceGuard guard(s.device);
    if (guard.err != cudaSuccess) {
      hg::g_lastError = std::string("hg_dot_noalloc: selecting the storage's device: ") + cudaGetErrorString(guard.err);
      return HG_ERR_CUDA;
    }
    double* scratch = nullptr;
    const int rc = scratchFor(s, &scratch);
    if (rc != HG_OK) return rc;
    // Every slot the reduction reads is written first by this call's own partial-sum kernel,
    // so nothing of the previous call's contents needs clearing.
    if (precision == 8)
      hg::dev::dotKernel<double><<<nb, hg::dev::kBlock, 0, s.stream>>>(ld.lv, (const double*)a, (const double*)b, flag,
                                                                        scratch);
    else
      hg::dev::dotKernel<float><<<nb, hg::dev::kBlock, 0, s.stream>>>(ld.lv, (const float*)a, (const float*)b, flag,
                                                                       scratch);
    hg::dev::reduceKernel<<<1, hg::dev::kBlock, 0, s.stream>>>(scratch, nb, result);
    s.launches += 2;
    hg::cudaCheck(cudaGetLastError(), "hg_dot_noalloc launch");
  } catch (const hg::Error& e) {
    hg::g_lastError = e.what();
    return e.code;
  } catch (const std::exception& e) {
    hg::g_lastError = e.what();
    return HG_ERR_INTERNAL;
  }
  return HG_OK;
}
