// push_op.cu — stand-alone push_spikes operator on device buffers.
//
// The reference's push_spikes (P/api/net/push.rs:126-173) as one call: for
// every neuron in `active` (ascending, as compact_spikes_into returns), add
// each outgoing synapse's weight to ring[(step + max(delay,1)) % 32][post].
// Each ring cell receives its adds in the reference's order (ascending pre,
// then CSR row order), so the float sums are bit-identical to the sequential
// push.  Four kernels: count events per post tile, scan, fill the tile bins
// (key = CSR edge id), apply per tile with ownership rounds in shared memory.
#include <cub/cub.cuh>

#include <algorithm>
#include <mutex>
#include <string>

#include "common.cuh"

namespace sg {

constexpr uint32_t kPushTileShift = 11;  // 2048 posts per tile
constexpr uint32_t kPushHashBits = 13;   // 8192 owner slots (32 KB smem)
constexpr uint32_t kPushEmpty = 0xFFFFFFFFu;

struct PushScratch {
  uint32_t *tile_cnt;   // [n_tiles]   events per tile
  uint32_t *tile_cur;   // [n_tiles]   fill cursors
  uint32_t *tile_base;  // [n_tiles+1] exclusive prefix of tile_cnt
  unsigned long long *total;  // [1]   events of this call
  uint32_t *bad;        // [1]   bit 0: an active entry >= n_neurons; bit 1: a col entry >= n_neurons
  uint32_t *bkey;       // [events]
  float *bw;            // [events]
  uint32_t *bcell;      // [events]
};

// Counts the events per post tile.  Entries outside [0, n_neurons) in
// `active` or `col` are not followed: they set a bit of s.bad, which the host
// reads with the total and turns into an error before anything is written.
__global__ void push_count_kernel(const uint32_t *row_ptr, const uint32_t *col, const uint32_t *active,
                                  uint32_t n_active, uint32_t n_neurons, PushScratch s) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t r = gw; r < n_active; r += nw) {
    const uint32_t pre = active[r];
    if (pre >= n_neurons) {
      if (lane == 0) atomicOr(s.bad, 1u);
      continue;
    }
    const uint32_t beg = row_ptr[pre], end = row_ptr[pre + 1];
    if (lane == 0 && end > beg) atomicAdd(s.total, (unsigned long long)(end - beg));
    for (uint32_t e0 = beg; e0 < end; e0 += 32) {
      const uint32_t e = e0 + lane;
      bool ok = e < end;
      uint32_t post = 0;
      if (ok) {
        post = col[e];
        if (post >= n_neurons) {
          atomicOr(s.bad, 2u);
          ok = false;
        }
      }
      const uint32_t mask = __ballot_sync(0xffffffffu, ok);
      if (ok) {
        const uint32_t tile = post >> kPushTileShift;
        const uint32_t peers = __match_any_sync(mask, tile);
        if (lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(s.tile_cnt + tile, (uint32_t)__popc(peers));
      }
    }
  }
}

__global__ void push_scan_kernel(PushScratch s, uint32_t n_tiles) {
  // one block: exclusive scan of tile_cnt into tile_base
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < n_tiles; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    uint32_t v = i < n_tiles ? s.tile_cnt[i] : 0u;
    uint32_t x = v;
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    __shared__ uint32_t wsum[32];
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
      uint32_t t = lane < (blockDim.x >> 5) ? wsum[lane] : 0u;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= (uint32_t)o) t += y;
      }
      wsum[lane] = t;
    }
    __syncthreads();
    const uint32_t excl = carry + (x - v) + (wid ? wsum[wid - 1] : 0u);
    if (i < n_tiles) s.tile_base[i] = excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) s.tile_base[n_tiles] = carry;
}

__global__ void push_fill_kernel(const uint32_t *row_ptr, const uint32_t *col, const float *w,
                                 const uint8_t *delay, const uint32_t *active, uint32_t n_active,
                                 unsigned long long step, PushScratch s) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t r = gw; r < n_active; r += nw) {
    const uint32_t pre = active[r];
    const uint32_t beg = row_ptr[pre], end = row_ptr[pre + 1];
    for (uint32_t e0 = beg; e0 < end; e0 += 32) {
      const uint32_t e = e0 + lane;
      const bool ok = e < end;
      const uint32_t mask = __ballot_sync(0xffffffffu, ok);
      if (ok) {
        const uint32_t post = col[e];
        const uint32_t d = delay[e] & 31u;
        const uint32_t slot = (uint32_t)((step + max(d, 1u)) & 31ull);
        const uint32_t tile = post >> kPushTileShift;
        const uint32_t peers = __match_any_sync(mask, tile);
        const uint32_t leader = __ffs(peers) - 1;
        uint32_t off = 0;
        if (lane == leader) off = atomicAdd(s.tile_cur + tile, (uint32_t)__popc(peers));
        off = __shfl_sync(peers, off, leader);
        const uint32_t pos = s.tile_base[tile] + off + __popc(peers & ((1u << lane) - 1u));
        s.bkey[pos] = e;
        s.bw[pos] = w[e];
        s.bcell[pos] = (slot << kPushTileShift) | (post & ((1u << kPushTileShift) - 1u));
      }
    }
  }
}

__device__ __forceinline__ uint32_t push_owner_slot(uint32_t cell) {
  return (cell * 2654435761u) >> (32 - kPushHashBits);
}

__global__ void __launch_bounds__(512) push_apply_kernel(float *ring, uint32_t n_neurons, PushScratch s,
                                                         uint32_t n_tiles) {
  __shared__ uint32_t owner[1u << kPushHashBits];
  const uint32_t tmask = (1u << kPushTileShift) - 1u;
  for (uint32_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const uint32_t base = s.tile_base[tile];
    const uint32_t cnt = s.tile_base[tile + 1] - base;
    if (cnt == 0) continue;
    uint32_t *cellp = s.bcell + base;
    const uint32_t *keyp = s.bkey + base;
    const float *wp = s.bw + base;
    for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) owner[push_owner_slot(cellp[k])] = kPushEmpty;
    __syncthreads();
    bool pending = true;
    while (__syncthreads_or(pending)) {
      pending = false;
      for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) {
        const uint32_t c = cellp[k];
        if (c != kPushEmpty) atomicMin(&owner[push_owner_slot(c)], keyp[k]);
      }
      __syncthreads();
      for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) {
        const uint32_t c = cellp[k];
        if (c == kPushEmpty) continue;
        if (owner[push_owner_slot(c)] == keyp[k]) {
          float *r = ring + (size_t)(c >> kPushTileShift) * n_neurons + ((size_t)tile << kPushTileShift) + (c & tmask);
          *r = *r + wp[k];
          cellp[k] = kPushEmpty;
        } else {
          pending = true;
        }
      }
      __syncthreads();
      for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) {
        const uint32_t c = cellp[k];
        if (c != kPushEmpty) owner[push_owner_slot(c)] = kPushEmpty;
      }
    }
    __syncthreads();
  }
}

uint32_t push_tiles(uint32_t n_neurons) { return (n_neurons + (1u << kPushTileShift) - 1) >> kPushTileShift; }

unsigned push_grid(uint32_t n_active) {
  unsigned b = (n_active + 7) / 8;  // 8 warps per 256-thread block
  return std::max(1u, std::min(b, 148u * 16));
}

// Launch the four kernels.  `alloc_bins` provides bin storage for `events`
// once the count is known; returns false when it cannot.
template <typename AllocBins>
int push_run(const uint32_t *row_ptr, const uint32_t *col, const float *w, const uint8_t *delay, uint32_t n_neurons,
             const uint32_t *active, uint32_t n_active, uint64_t step, float *ring, cudaStream_t st, PushScratch s,
             AllocBins alloc_bins) {
  const uint32_t n_tiles = push_tiles(n_neurons);
  SG_CUDA(cudaMemsetAsync(s.tile_cnt, 0, (size_t)n_tiles * 4, st));
  SG_CUDA(cudaMemsetAsync(s.tile_cur, 0, (size_t)n_tiles * 4, st));
  SG_CUDA(cudaMemsetAsync(s.total, 0, 8, st));
  SG_CUDA(cudaMemsetAsync(s.bad, 0, 4, st));
  if (n_active == 0) return SG_OK;
  push_count_kernel<<<push_grid(n_active), 256, 0, st>>>(row_ptr, col, active, n_active, n_neurons, s);
  SG_CUDA(cudaGetLastError());
  unsigned long long total = 0;
  uint32_t bad = 0;
  SG_CUDA(cudaMemcpyAsync(&total, s.total, 8, cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaMemcpyAsync(&bad, s.bad, 4, cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  SG_REQUIRE(!(bad & 1u), SG_E_INVALID, "push_spikes: an active neuron index is >= n_neurons; the ring was not modified");
  SG_REQUIRE(!(bad & 2u), SG_E_INVALID, "push_spikes: a col entry of an active row is >= n_neurons; the ring was not modified");
  if (total == 0) return SG_OK;
  const int rc = alloc_bins(total, s);
  if (rc != SG_OK) return rc;
  push_scan_kernel<<<1, 1024, 0, st>>>(s, n_tiles);
  push_fill_kernel<<<push_grid(n_active), 256, 0, st>>>(row_ptr, col, w, delay, active, n_active, step, s);
  push_apply_kernel<<<std::min<uint32_t>(n_tiles, 148u * 4), 512, 0, st>>>(ring, n_neurons, s, n_tiles);
  SG_CUDA(cudaGetLastError());
  SG_CUDA(cudaStreamSynchronize(st));
  return SG_OK;
}

int push_check_args(const uint32_t *row_ptr, const uint32_t *col, const float *w, const uint8_t *delay,
                    uint32_t n_neurons, const uint32_t *active, uint32_t n_active, float *ring) {
  SG_REQUIRE(row_ptr && ring, SG_E_INVALID, "push_spikes: null device pointer (row_ptr or ring)");
  SG_REQUIRE(n_active == 0 || (active && col && w && delay), SG_E_INVALID,
             "push_spikes: null device pointer (active, col, weights or delays)");
  SG_REQUIRE(n_neurons > 0, SG_E_INVALID, "push_spikes: n_neurons must be > 0");
  return SG_OK;
}

}  // namespace sg

using namespace sg;

namespace {
template <typename F> int guarded(F f) {
  try {
    return f();
  } catch (const Fail &e) {
    return e.code;
  } catch (const std::exception &e) {
    set_error(e.what());
    return SG_E_INVALID;
  }
}
}  // namespace

extern "C" int sg_push_spikes(const uint32_t *row_ptr, const uint32_t *col, const float *weights,
                              const uint8_t *delays, uint32_t n_neurons, const uint32_t *active, uint32_t n_active,
                              uint64_t step, float *ring, void *stream) {
  return guarded([&]() -> int {
    push_check_args(row_ptr, col, weights, delays, n_neurons, active, n_active, ring);
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t n_tiles = push_tiles(n_neurons);
    PushScratch s{};
    void *small = nullptr;
    SG_CUDA(cudaMalloc(&small, (size_t)n_tiles * 12 + 32));
    s.tile_cnt = (uint32_t *)small;
    s.tile_cur = s.tile_cnt + n_tiles;
    s.tile_base = s.tile_cur + n_tiles;
    s.total = (unsigned long long *)(((uintptr_t)(s.tile_base + n_tiles + 1) + 7) & ~(uintptr_t)7);
    s.bad = (uint32_t *)(s.total + 1);
    void *bins = nullptr;
    int rc = SG_OK;
    try {
      rc = push_run(row_ptr, col, weights, delays, n_neurons, active, n_active, step, ring, st, s,
                    [&](unsigned long long total, PushScratch &sc) -> int {
                      if (total >= 0xFFFFFFFFull) {
                        set_error("push_spikes: more than 2^32-1 events in one call");
                        return SG_E_OVERFLOW;
                      }
                      SG_CUDA(cudaMalloc(&bins, (size_t)total * 12));
                      sc.bkey = (uint32_t *)bins;
                      sc.bw = (float *)(sc.bkey + total);
                      sc.bcell = (uint32_t *)(sc.bw + total);
                      return SG_OK;
                    });
    } catch (...) {
      if (bins) cudaFree(bins);
      cudaFree(small);
      throw;
    }
    if (bins) cudaFree(bins);
    cudaFree(small);
    return rc;
  });
}

// ---------------------------------------------------------------------------
// sg_push_spikes_noalloc: the same operator for callers that cannot allocate
// device memory while they run: a real-time loop whose timing budget has no
// room for cudaMalloc/cudaFree (they can block on the driver and synchronise
// the device), or an embedding that is handed a fixed device-memory budget up
// front and owns every allocation itself.  Its scratch is one file-scope
// __device__ array of fixed size that every GPU loading this library keeps
// until the process exits.  Like sg_push_spikes, a call waits on its stream
// once (it reads the event count back to the host) and returns after the
// ring is updated.
// ---------------------------------------------------------------------------
namespace {

constexpr uint32_t kNoAllocMaxEvents = 1u << 20;   // synaptic events per call
constexpr uint32_t kNoAllocMaxNeurons = 1u << 23;  // 8,388,608 neurons
constexpr uint32_t kNoAllocTiles = kNoAllocMaxNeurons >> kPushTileShift;  // 4096
constexpr size_t kNoAllocCounterBytes = ((size_t)kNoAllocTiles * 3 + 1) * 4;
constexpr size_t kNoAllocTotalOff = (kNoAllocCounterBytes + 255) & ~(size_t)255;  // total (8 B), then the bad flag
constexpr size_t kNoAllocBinsOff = kNoAllocTotalOff + 256;
constexpr size_t kNoAllocBytes = kNoAllocBinsOff + (size_t)kNoAllocMaxEvents * 12;  // ~12.1 MiB

// In host code this name is only a stand-in: the device address comes from
// cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_push_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void *g_noalloc_addr[kMaxDevices] = {};

// Resolve the scratch array's device address on the current device (first
// call per device only).  The address is kept for the life of the process: a
// cudaDeviceReset on that device (which unloads this module) leaves it stale,
// so do not call this entry point again after resetting its device.
int noalloc_scratch(void **out) {
  int dev = 0;
  SG_CUDA(cudaGetDevice(&dev));
  SG_REQUIRE(dev >= 0 && dev < kMaxDevices, SG_E_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_push_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error(std::string("sg_push_spikes_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
      return SG_E_CUDA;
    }
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return SG_OK;
}

}  // namespace

extern "C" int sg_push_spikes_noalloc(const uint32_t *row_ptr, const uint32_t *col, const float *weights,
                                      const uint8_t *delays, uint32_t n_neurons, const uint32_t *active,
                                      uint32_t n_active, uint64_t step, float *ring, void *stream) {
  return guarded([&]() -> int {
    push_check_args(row_ptr, col, weights, delays, n_neurons, active, n_active, ring);
    SG_REQUIRE(n_neurons <= kNoAllocMaxNeurons, SG_E_INVALID,
               "sg_push_spikes_noalloc: n_neurons " + std::to_string(n_neurons) + " exceeds the maximum " +
                   std::to_string(kNoAllocMaxNeurons));
    void *base = nullptr;
    const int rc0 = noalloc_scratch(&base);
    if (rc0 != SG_OK) return rc0;
    unsigned char *b = (unsigned char *)base;
    PushScratch s{};
    s.tile_cnt = (uint32_t *)b;
    s.tile_cur = s.tile_cnt + kNoAllocTiles;
    s.tile_base = s.tile_cur + kNoAllocTiles;
    s.total = (unsigned long long *)(b + kNoAllocTotalOff);
    s.bad = (uint32_t *)(s.total + 1);
    return push_run(row_ptr, col, weights, delays, n_neurons, active, n_active, step, ring, (cudaStream_t)stream, s,
                    [&](unsigned long long total, PushScratch &sc) -> int {
                      if (total > kNoAllocMaxEvents) {
                        set_error("sg_push_spikes_noalloc: " + std::to_string(total) +
                                  " synaptic events exceed the maximum " + std::to_string(kNoAllocMaxEvents) +
                                  " per call; the ring was not modified");
                        return SG_E_OVERFLOW;
                      }
                      sc.bkey = (uint32_t *)(b + kNoAllocBinsOff);
                      sc.bw = (float *)(sc.bkey + kNoAllocMaxEvents);
                      sc.bcell = (uint32_t *)(sc.bw + kNoAllocMaxEvents);
                      return SG_OK;
                    });
  });
}
