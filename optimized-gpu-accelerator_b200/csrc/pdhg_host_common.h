// Host-side helpers shared by the engine's translation units: error type and
// CUDA-call check, the per-thread last-error message behind b2p_last_error,
// the ABI guard that turns exceptions into return codes, and device choice.
#pragma once

#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <map>
#include <mutex>
#include <cstdlib>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/b2p_pdhg.h"

namespace b2p {

inline std::string& last_error() {
  thread_local std::string msg;
  return msg;
}

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define B2P_CUDA(call)                                                                                     \
  do {                                                                                                     \
    cudaError_t e_ = (call);                                                                               \
    if (e_ != cudaSuccess)                                                                                 \
      throw ::b2p::Error(e_ == cudaErrorMemoryAllocation ? B2P_ERR_OOM : B2P_ERR_CUDA,                     \
                         std::string("CUDA error in ") + #call + ": " + cudaGetErrorString(e_));           \
  } while (0)

using Clock = std::chrono::steady_clock;
inline double seconds_since(Clock::time_point t0) {
  return std::chrono::duration<double>(Clock::now() - t0).count();
}

// Runs f and maps exceptions to B2P_ERR_* codes (no exception crosses the C ABI).
template <class F>
int guarded(F&& f) {
  try {
    last_error().clear();
    f();
    return B2P_OK;
  } catch (Error& e) {
    last_error() = e.what();
    return e.code;
  } catch (std::bad_alloc&) {
    last_error() = "host out of memory";
    return B2P_ERR_OOM;
  } catch (std::exception& e) {
    last_error() = e.what();
    return B2P_ERR_CUDA;
  }
}

// The engines' device memory comes from one stream-ordered pool per device
// (cudaMallocFromPoolAsync / cudaFreeAsync on the engine's stream): freed
// blocks stay cached for the next engine, so a solve's set-up does not pay a
// cudaMalloc / cudaFree per buffer.  Up to kPoolKeepBytes of freed memory is
// kept per device (held until the process exits); beyond that it goes back to
// the driver at the next synchronisation.
constexpr uint64_t kPoolKeepBytes = uint64_t(8) << 30;

inline cudaMemPool_t device_pool(int dev) {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  std::lock_guard<std::mutex> lock(mu);
  auto it = pools.find(dev);
  if (it != pools.end()) return it->second;
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t pool = nullptr;
  B2P_CUDA(cudaMemPoolCreate(&pool, &props));
  uint64_t keep = kPoolKeepBytes;
  B2P_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  pools.emplace(dev, pool);
  return pool;
}

// Page-locked host buffers, cached for the process: cudaMallocHost pins
// pages and cudaFreeHost unpins them (and waits for the device), at a cost
// that varies with the host's load, so the engines take their small pinned
// buffers (check sums, step sizes, masks, power-iteration vectors) from here
// and give them back.  Buffers come in power-of-two sizes from 256 bytes; up
// to kPinnedKeepBytes of freed buffers are kept, the rest are freed.
constexpr size_t kPinnedKeepBytes = size_t(256) << 20;

class PinnedCache {
 public:
  static void* get(size_t bytes) {
    const size_t cls = size_class(bytes);
    {
      std::lock_guard<std::mutex> lock(mu());
      auto& fl = lists()[cls];
      if (!fl.empty()) {
        void* p = fl.back();
        fl.pop_back();
        kept() -= cls;
        return p;
      }
    }
    void* p = nullptr;
    B2P_CUDA(cudaMallocHost(&p, cls));
    return p;
  }
  static void put(void* p, size_t bytes) {
    if (!p) return;
    const size_t cls = size_class(bytes);
    {
      std::lock_guard<std::mutex> lock(mu());
      if (kept() + cls <= kPinnedKeepBytes) {
        lists()[cls].push_back(p);
        kept() += cls;
        return;
      }
    }
    cudaFreeHost(p);
  }

 private:
  static size_t size_class(size_t bytes) {
    size_t c = 256;
    while (c < bytes) c <<= 1;
    return c;
  }
  static std::mutex& mu() {
    static std::mutex m;
    return m;
  }
  static std::map<size_t, std::vector<void*>>& lists() {
    static std::map<size_t, std::vector<void*>> l;
    return l;
  }
  static size_t& kept() {
    static size_t k = 0;
    return k;
  }
};

// Ordinal of the sm_100 device to use: `requested`, else PRAMANA_GPU_DEVICE,
// else 0 (src/gpu/cuda_driver.cpp:223); PRAMANA_DISABLE_GPU disables the
// engine (cuda_driver.cpp:149).
inline int pick_device(int requested) {
  if (std::getenv("PRAMANA_DISABLE_GPU")) throw Error(B2P_ERR_NO_DEVICE, "disabled by PRAMANA_DISABLE_GPU");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    throw Error(B2P_ERR_NO_DEVICE, "no CUDA device");
  }
  int dev = requested;
  if (dev < 0) {
    const char* env = std::getenv("PRAMANA_GPU_DEVICE");
    dev = env ? std::atoi(env) : 0;
  }
  if (dev < 0 || dev >= count) throw Error(B2P_ERR_NO_DEVICE, "device ordinal out of range");
  int major = 0;
  B2P_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  if (major != 10) {
    cudaDeviceProp p;
    B2P_CUDA(cudaGetDeviceProperties(&p, dev));
    throw Error(B2P_ERR_NO_DEVICE, std::string("device is not sm_100: ") + p.name);
  }
  return dev;
}

}  // namespace b2p
