// probe.cu — the measured ceiling of the pre-centric scatter's event adds.
//
// The pre-centric scatter adds each synaptic event to a random cell of the
// L2-resident delay rings with one red.global.add.f32, so its rate is bound
// by how many scattered 4-byte reductions the L2 completes per second, not
// by HBM bandwidth (every red is a read-modify-write of a 32-byte sector in
// L2).  sg_probe_red_rate measures that ceiling on the current GPU the way
// a STREAM copy measures HBM bandwidth: a full-occupancy grid issues
// independent reds to hashed cells of an array of the rings' size, timed
// with CUDA events after a warm-up.
#include "common.cuh"

namespace sg {
namespace {

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// Every thread adds 1.0f to `iters` cells; cell indices are taken modulo n.
__global__ void __launch_bounds__(256) red_probe_kernel(float *cells, uint32_t n, uint32_t iters) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  for (uint32_t i = 0; i < iters; ++i) {
    float *p = cells + mix32(tid * 2654435761u + i * 40503u) % n;
    asm volatile("red.global.add.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(1.0f), "l"(pol) : "memory");
  }
}

}  // namespace
}  // namespace sg

using namespace sg;

extern "C" int sg_probe_red_rate(int device, uint64_t n_cells, uint32_t iters, double *reds_per_s) {
  float *cells = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = SG_OK;
  try {
    SG_REQUIRE(reds_per_s, SG_E_INVALID, "null output");
    SG_REQUIRE(n_cells >= 1 && n_cells <= 0xFFFFFFFFull, SG_E_INVALID, "n_cells must be in [1, 2^32 - 1]");
    SG_REQUIRE(iters >= 1, SG_E_INVALID, "iters must be >= 1");
    int ndev = 0;
    SG_CUDA(cudaGetDeviceCount(&ndev));
    SG_REQUIRE(device >= 0 && device < ndev, SG_E_INVALID, "device ordinal out of range");
    SG_CUDA(cudaSetDevice(device));
    int sms = 0;
    SG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    SG_CUDA(cudaMalloc(&cells, n_cells * 4));
    SG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    SG_CUDA(cudaEventCreate(&e0));
    SG_CUDA(cudaEventCreate(&e1));
    SG_CUDA(cudaMemsetAsync(cells, 0, n_cells * 4, st));
    const unsigned grid = (unsigned)sms * 8u;  // 2048 threads per SM
    for (int w = 0; w < 2; ++w) red_probe_kernel<<<grid, 256, 0, st>>>(cells, (uint32_t)n_cells, iters);
    SG_CUDA(cudaGetLastError());
    const int reps = 5;
    SG_CUDA(cudaEventRecord(e0, st));
    for (int r = 0; r < reps; ++r) red_probe_kernel<<<grid, 256, 0, st>>>(cells, (uint32_t)n_cells, iters);
    SG_CUDA(cudaEventRecord(e1, st));
    SG_CUDA(cudaEventSynchronize(e1));
    float ms = 0.0f;
    SG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    *reds_per_s = (double)reps * grid * 256.0 * iters / (ms / 1e3);
  } catch (const Fail &f) {
    rc = f.code;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  if (cells) cudaFree(cells);
  return rc;
}
