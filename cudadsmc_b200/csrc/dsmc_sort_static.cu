// dsmc_stage_sort_static: the stage sort (count keys, scan, scatter, segment
// fixup) with its scratch in a fixed static device array instead of a
// caller-provided or stream-allocated workspace.  Nothing is allocated.
#include <atomic>
#include <mutex>

#include "dsmc_b200.h"
#include "dsmc_kernels.cuh"

namespace {

constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

constexpr size_t kMaxN = DSMC_SORT_STATIC_MAX_N;
constexpr size_t kMaxKeys = DSMC_SORT_STATIC_MAX_KEYS;
constexpr size_t kMaxTiles = (kMaxKeys + dsmcb::kScanTile - 1) / dsmcb::kScanTile;
static_assert(kMaxTiles <= (size_t)dsmcb::kMaxScanTiles, "key range beyond the scan tiles");

// Fixed layout of the scratch: per-key counts and starts, scan-tile sums,
// per-element tickets, scattered values and positions, the scan's counters.
constexpr size_t kOffCount = 0;
constexpr size_t kOffStart = kOffCount + align256(4 * (kMaxKeys + 1));
constexpr size_t kOffTiles = kOffStart + align256(4 * (kMaxKeys + 1));
constexpr size_t kOffTicket = kOffTiles + align256(4 * kMaxTiles);
constexpr size_t kOffVal = kOffTicket + align256(4 * kMaxN);
constexpr size_t kOffPos = kOffVal + align256(4 * kMaxN);
constexpr size_t kOffMeta = kOffPos + align256(4 * kMaxN);
constexpr size_t kScratchBytes = kOffMeta + align256(sizeof(dsmcb::Meta));

// About 13.6 MB of device memory, reserved on each device when the library's
// kernels are loaded there.
static __device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::atomic<unsigned char*> g_scratch_addr[kMaxDevices];
std::mutex g_scratch_mutex;

// Device address of the scratch on the current device, looked up once per
// device and kept for the life of the process (a device reset would move the
// array: the header tells callers not to use this entry point after one).
cudaError_t scratch_address(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  unsigned char* a = g_scratch_addr[dev].load(std::memory_order_acquire);
  if (!a) {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    a = g_scratch_addr[dev].load(std::memory_order_relaxed);
    if (!a) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_sort_scratch);
      if (e != cudaSuccess) return e;
      a = static_cast<unsigned char*>(p);
      g_scratch_addr[dev].store(a, std::memory_order_release);
    }
  }
  *out = a;
  return cudaSuccess;
}

}  // namespace

extern "C" int dsmc_stage_sort_static(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t nkeys,
                                      uint32_t* cell_start, void* stream) {
  if (nkeys == 0 || (n && (!keys || !vals))) return DSMC_ERR_ARG;
  if (n > kMaxN || nkeys > kMaxKeys) return DSMC_ERR_CAPACITY;
  unsigned char* w = nullptr;
  cudaError_t e = scratch_address(&w);
  if (e != cudaSuccess) return DSMC_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;
  const uint32_t tiles = (nkeys + dsmcb::kScanTile - 1) / dsmcb::kScanTile;
  uint32_t* count = reinterpret_cast<uint32_t*>(w + kOffCount);
  uint32_t* start = reinterpret_cast<uint32_t*>(w + kOffStart);
  uint32_t* tsum = reinterpret_cast<uint32_t*>(w + kOffTiles);
  uint32_t* ticket = reinterpret_cast<uint32_t*>(w + kOffTicket);
  uint32_t* tval = reinterpret_cast<uint32_t*>(w + kOffVal);
  uint32_t* tpos = reinterpret_cast<uint32_t*>(w + kOffPos);
  dsmcb::Meta* meta = reinterpret_cast<dsmcb::Meta*>(w + kOffMeta);
  // counts, scan-tile sums and the scan's counters start every call at zero;
  // the other regions are fully written before they are read
  e = cudaMemsetAsync(count, 0, 4ull * (nkeys + 1), s);
  if (!e) e = cudaMemsetAsync(tsum, 0, 4ull * tiles, s);
  if (!e) e = cudaMemsetAsync(meta, 0, sizeof(dsmcb::Meta), s);
  if (!e && n) e = dsmcb::launch_count_keys(keys, n, nkeys, ticket, count, tsum, tiles, s);
  if (!e) e = dsmcb::launch_scan(count, nullptr, start, nkeys, tsum, tiles, meta, 0, s);
  if (!e && n) e = dsmcb::launch_scatter_kv(keys, vals, ticket, start, n, nkeys, tval, tpos, s);
  if (!e && n) e = dsmcb::launch_segment_fixup(start, nkeys, tval, tpos, keys, vals, s);
  if (!e && cell_start)
    e = cudaMemcpyAsync(cell_start, start, 4ull * (nkeys + 1), cudaMemcpyDeviceToDevice, s);
  return e ? DSMC_ERR_CUDA : DSMC_OK;
}
