// Cache of released device blocks behind DevBuf (declared in common.h).
//
// A released block is kept, per device and by size, and handed out again for
// a request it covers without too much waste (at most twice the request, or
// 2 MiB more).  Releasing waits for the device to be idle (what cudaFree
// does), so a reused block has no work in flight.  An allocation that fails
// empties the device's cache and tries once more.  At most kCacheCap bytes
// per device are kept; beyond that a released block goes back to the driver.
// The cache is never torn down: the process's exit returns the memory.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.h"

namespace inti {
namespace {

constexpr size_t kCacheCap = (size_t)8 << 30;
constexpr size_t kSlack = (size_t)2 << 20;

struct DeviceCache {
  std::multimap<size_t, void*> free;  // size -> block
  size_t bytes = 0;
};

struct Cache {
  std::mutex mu;
  std::map<int, DeviceCache> dev;
};

Cache& cache() {
  static Cache* c = new Cache();  // never destroyed: freeing at process exit is the driver's job
  return *c;
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

}  // namespace

void* dev_alloc(size_t nbytes, int* device, size_t* got) {
  int d = 0;
  INTI_CUDA(cudaGetDevice(&d));
  *device = d;
  Cache& c = cache();
  {
    std::lock_guard<std::mutex> lk(c.mu);
    DeviceCache& dc = c.dev[d];
    auto it = dc.free.lower_bound(nbytes);
    if (it != dc.free.end() && (it->first <= 2 * nbytes || it->first - nbytes <= kSlack)) {
      void* p = it->second;
      *got = it->first;
      dc.bytes -= it->first;
      dc.free.erase(it);
      return p;
    }
  }
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, nbytes);
  if (e != cudaSuccess) {
    cudaGetLastError();  // clear the allocation error
    std::vector<void*> drop;
    {
      std::lock_guard<std::mutex> lk(c.mu);
      DeviceCache& dc = c.dev[d];
      for (auto& kv : dc.free) drop.push_back(kv.second);
      dc.free.clear();
      dc.bytes = 0;
    }
    for (void* q : drop) cudaFree(q);
    e = cudaMalloc(&p, nbytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw Error(INTI_E_NOMEM, std::string("cudaMalloc(") + std::to_string(nbytes) + "): " + cudaGetErrorString(e));
    }
  }
  *got = nbytes;
  return p;
}

void dev_release(void* p, size_t bytes, int device) {
  if (!p) return;
  SetDevice sd(device);
  cudaDeviceSynchronize();  // no work of any stream still uses the block
  Cache& c = cache();
  {
    std::lock_guard<std::mutex> lk(c.mu);
    DeviceCache& dc = c.dev[device];
    if (dc.bytes + bytes <= kCacheCap) {
      dc.free.emplace(bytes, p);
      dc.bytes += bytes;
      return;
    }
  }
  cudaFree(p);
}

size_t dev_cache_bytes(int device) {
  Cache& c = cache();
  std::lock_guard<std::mutex> lk(c.mu);
  auto it = c.dev.find(device);
  return it == c.dev.end() ? 0 : it->second.bytes;
}

}  // namespace inti
