// Device memory behind DevBuf (declared in common.h).
//
// Blocks under kPoolMax bytes come from a per-device CUDA memory pool that
// keeps released memory and sub-allocates from what it holds; the pool
// reserves kPoolReserve bytes when it is created.  Creating and destroying
// operators then rarely goes back to the driver, whose latency for a first
// allocation of a few megabytes ranges from microseconds to tens of
// milliseconds on a busy host.  Larger blocks (the symmetric form's partial
// pools, Krylov bases, DIM work arrays: made once per context or solve) go
// to cudaMalloc, which maps them in well under a millisecond, where growing
// the pool by a gigabyte took 0.4 s.
//
// Pool allocations are made on a private stream of the pool and waited for,
// so a block is ready for every stream when dev_alloc returns.  Releasing
// first waits for the device to be idle (what cudaFree does), so memory
// handed out again has no work in flight.  Above kCacheCap bytes of released
// memory the pool returns the excess to the driver at its next
// synchronisation.  An allocation that fails trims the pool to nothing and
// tries once more.  The pools are never torn down: the process's exit
// returns the memory.
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <string>

#include "common.h"

namespace inti {
namespace {

constexpr uint64_t kCacheCap = (uint64_t)8 << 30;
constexpr size_t kPoolMax = (size_t)64 << 20;
constexpr size_t kPoolReserve = (size_t)256 << 20;

struct DevicePool {
  cudaMemPool_t pool = nullptr;
  cudaStream_t stream = nullptr;
};

struct Pools {
  std::mutex mu;
  std::map<int, DevicePool> dev;
};

Pools& pools() {
  static Pools* p = new Pools();  // never destroyed: freeing at process exit is the driver's job
  return *p;
}

struct SetDevice {
  int prev = -1;
  explicit SetDevice(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~SetDevice() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// The pool of device d (created on first use, with d current).
DevicePool& pool_for(int d) {
  Pools& ps = pools();
  std::lock_guard<std::mutex> lk(ps.mu);
  DevicePool& p = ps.dev[d];
  if (!p.pool) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = d;
    INTI_CUDA(cudaMemPoolCreate(&p.pool, &props));
    uint64_t threshold = kCacheCap;
    INTI_CUDA(cudaMemPoolSetAttribute(p.pool, cudaMemPoolAttrReleaseThreshold, &threshold));
    INTI_CUDA(cudaStreamCreateWithFlags(&p.stream, cudaStreamNonBlocking));
    void* warm = nullptr;  // reserve kPoolReserve bytes now, kept by the release threshold
    if (cudaMallocFromPoolAsync(&warm, kPoolReserve, p.pool, p.stream) == cudaSuccess) {
      cudaFreeAsync(warm, p.stream);
      cudaStreamSynchronize(p.stream);
    } else {
      cudaGetLastError();
    }
  }
  return p;
}

}  // namespace

void* dev_alloc(size_t nbytes, int* device, size_t* got) {
  int d = 0;
  INTI_CUDA(cudaGetDevice(&d));
  *device = d;
  void* ptr = nullptr;
  if (nbytes >= kPoolMax) {
    cudaError_t e = cudaMalloc(&ptr, nbytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      {
        std::lock_guard<std::mutex> lk(pools().mu);
        auto it = pools().dev.find(d);
        if (it != pools().dev.end() && it->second.pool) {
          cudaDeviceSynchronize();
          cudaMemPoolTrimTo(it->second.pool, 0);
        }
      }
      e = cudaMalloc(&ptr, nbytes);
      if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(INTI_E_NOMEM, std::string("cudaMalloc(") + std::to_string(nbytes) + "): " + cudaGetErrorString(e));
      }
    }
    *got = nbytes;
    return ptr;
  }
  DevicePool& p = pool_for(d);
  cudaError_t e = cudaMallocFromPoolAsync(&ptr, nbytes, p.pool, p.stream);
  if (e != cudaSuccess) {
    cudaGetLastError();  // clear the allocation error
    cudaDeviceSynchronize();
    cudaMemPoolTrimTo(p.pool, 0);
    e = cudaMallocFromPoolAsync(&ptr, nbytes, p.pool, p.stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw Error(INTI_E_NOMEM, std::string("device allocation of ") + std::to_string(nbytes) +
                                    " bytes: " + cudaGetErrorString(e));
    }
  }
  INTI_CUDA(cudaStreamSynchronize(p.stream));  // ready for every stream
  *got = nbytes;
  return ptr;
}

void dev_release(void* ptr, size_t bytes, int device) {
  if (!ptr) return;
  SetDevice sd(device);
  if (bytes >= kPoolMax) {
    cudaFree(ptr);
    return;
  }
  cudaDeviceSynchronize();  // no work of any stream still uses the block
  DevicePool& p = pool_for(device);
  cudaFreeAsync(ptr, p.stream);
}

void dev_prepare(int device) {
  SetDevice sd(device);
  pool_for(device);
}

size_t dev_cache_bytes(int device) {
  Pools& ps = pools();
  std::lock_guard<std::mutex> lk(ps.mu);
  auto it = ps.dev.find(device);
  if (it == ps.dev.end() || !it->second.pool) return 0;
  uint64_t reserved = 0, used = 0;
  cudaMemPoolGetAttribute(it->second.pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
  cudaMemPoolGetAttribute(it->second.pool, cudaMemPoolAttrUsedMemCurrent, &used);
  return reserved > used ? (size_t)(reserved - used) : 0;
}

}  // namespace inti
