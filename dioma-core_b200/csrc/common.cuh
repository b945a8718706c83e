// common.cuh — error plumbing and small device utilities.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>

#include "simuse_b200.h"

namespace sg {

void set_error(const std::string &msg);

struct Fail {
  int code;
};

#define SG_CUDA(call)                                                                      \
  do {                                                                                     \
    cudaError_t _e = (call);                                                               \
    if (_e != cudaSuccess) {                                                               \
      ::sg::set_error(std::string("CUDA error: ") + cudaGetErrorString(_e) + " at " +      \
                      __FILE__ + ":" + std::to_string(__LINE__) + " (" #call ")");         \
      throw ::sg::Fail{_e == cudaErrorMemoryAllocation ? SG_E_NOMEM : SG_E_CUDA};          \
    }                                                                                      \
  } while (0)

#define SG_REQUIRE(cond, code, msg)     \
  do {                                  \
    if (!(cond)) {                      \
      ::sg::set_error(msg);             \
      throw ::sg::Fail{code};           \
    }                                   \
  } while (0)

constexpr uint32_t kSlots = 32;  // P/api/net/graph.rs:33 MAX_DELAY_SLOTS

__host__ __device__ inline uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

// Edge code byte: bits 0-4 delay (< 32), bits 5-6 synapse type (0 static,
// 1..3 kinetic profile), bit 7 pair-STDP flag.
__host__ __device__ inline uint8_t edge_code(uint8_t delay, uint8_t syn_type, bool stdp) {
  return (uint8_t)((delay & 31u) | ((syn_type & 3u) << 5) | (stdp ? 0x80u : 0u));
}
// Receptor kinetics: an edge's code holds 1 + its receptor code (codes >= 7
// are AMPA, 0) in the delay field, so that its event lands in ring slot 1 + r.
__host__ __device__ inline uint8_t receptor_code(uint8_t receptor) {
  return edge_code((uint8_t)(1u + (receptor < 7u ? receptor : 0u)), 0, false);
}
__host__ __device__ inline uint32_t code_delay(uint8_t c) { return c & 31u; }
__host__ __device__ inline uint32_t code_ring(uint8_t c) { return (c >> 5) & 3u; }
__host__ __device__ inline bool code_stdp(uint8_t c) { return (c & 0x80u) != 0; }

}  // namespace sg
