// kuramoto.cu — batched Kuramoto populations, all-to-all coupling through
// the exact mean-field identity, classic RK4.
//
// Reference: the Euler step and phase wrap of P/kernels/phase/kuramoto.rs:42-68
// (phi += dt*(omega + C); phi - 2*pi*round(phi/2*pi), P/kernels/mod.rs:72-77),
// the sparse/dense coupling of P/kernels/phase/sparse.rs:40-140, and the O(N)
// mean-field sums of crates/SiMuse/crates/t3/src/oscillator.rs:15-20,549 with
// the FP64 order parameter of :440-450.  For all-to-all coupling
//   K/N * sum_j sin(th_j - th_i) = K * (S cos th_i - C sin th_i),
// C = mean cos th, S = mean sin th, so one reduction per RK4 stage replaces
// the O(N^2) sum.  RK4 itself has no reference implementation; it is the
// textbook scheme.
//
// Layout.
//  * Up to 4096 oscillators ("resident" instances): one CTA of 64..512
//    threads, 8 oscillators per thread; phases, frequencies, RK4 partial sums
//    and the stage sin/cos stay in registers for the whole run, so HBM sees
//    only the first load and the last store of theta.
//  * 4097..65,536 oscillators ("cluster" instances): a thread-block cluster
//    of 2, 4 or 8 CTAs of 512 threads (8 CTAs of 1024 threads above 32,768),
//    8 oscillators per thread, all state in registers as above.  Each stage
//    every CTA reduces its own oscillators, thread 0 stores the CTA's
//    (sum cos, sum sin) to a per-instance slot in global memory, the cluster
//    meets at a hardware cluster barrier (release/acquire), and every CTA
//    adds the cluster's partials in CTA-rank order, so all CTAs hold the same
//    field.  No distributed shared memory is used: the partials go through
//    L2 as plain 8-byte stores and loads.
//  * The streamed form (one 1024-thread CTA per instance, RK4 partial sums
//    and stage positions re-read from device scratch every stage) is kept
//    for a device on which a cluster shape cannot be resident.
// Each stage reduces (sum cos, sum sin) in a fixed order (a lane tree, a tree
// over the warps, then the CTAs in rank order), so results are reproducible
// run to run and an instance gives the same bits alone or in any batch (its
// shape depends on its size only).  Instances are binned by shape, one
// launch per bin, each bin on its own stream (joined to the handle's stream),
// so the bins' CTAs share the SMs.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "common.cuh"

namespace sg {

constexpr int kKOpt = 8;                 // oscillators per thread, resident kernels
constexpr uint32_t kKResident = 4096;    // largest resident instance (512 threads x 8)
constexpr int kKStreamThreads = 1024;    // CTA width of the streamed kernel
constexpr uint32_t kKMaxSize = 65536;
constexpr uint32_t kKMaxCluster = 8;     // CTAs per cluster (portable size)

struct KuraArgs {
  const uint32_t *inst;  // instance id of each CTA of this launch
  const uint64_t *off;   // first oscillator of each instance
  const uint32_t *size;  // oscillators per instance
  const float *coupling; // K per instance
  float *theta;          // [total]
  const float *omega;    // [total]
  float *ks;             // [total] RK4 partial sums (streamed instances)
  float *ypos;           // [total] stage positions (streamed instances)
  float dt;
  uint32_t n_steps;
  float *r_out;          // [n_inst][r_stride], or null
  uint64_t r_stride;
  uint64_t r_base;       // step index of this launch's first step in r_out
  double *r_sum;         // [n_inst] FP64 time accumulator of r(t)
  float2 *xpart;         // [n_inst][2][kKMaxCluster] per-CTA partial sums (cluster instances)
};

// 2*pi as a head with 8 significant bits (k*head is exact for |k| < 2^16)
// plus the FP32 remainder: Cody and Waite's split-constant reduction.
constexpr float kTwoPiHi = 6.28125f;
constexpr float kTwoPiLo = 1.9353071795864769e-3f;
constexpr float kInvTwoPi = 0.15915494309189533577f;

// Reduces y to about [-pi, pi]: y - 2 pi k with k = y / 2pi rounded to the
// nearest integer (ties to even).  This is the reference's wrap_phase
// (P/kernels/mod.rs:72-77, p - TAU*round(p/TAU)) up to FP32 rounding; a tie
// (an odd multiple of pi) may land on the other end of the interval, which
// is the same point of the circle.
__device__ __forceinline__ float reduce_phase(float y) {
  const float k = rintf(y * kInvTwoPi);
  return __fmaf_rn(-k, kTwoPiLo, __fmaf_rn(-k, kTwoPiHi, y));
}

// sin and cos of y: reduce, then the SFU approximations (absolute error
// about 2^-21 on [-pi, pi]).
__device__ __forceinline__ void phase_sincos(float y, float &s, float &c) { __sincosf(reduce_phase(y), &s, &c); }

// dtheta/dt at a stage position with sin/cos (s, c) in the field (C, S).
__device__ __forceinline__ float kura_rate(float om, float K, float C, float S, float s, float c) {
  return __fmaf_rn(K, __fmaf_rn(S, c, -(C * s)), om);
}

// Fixed-order warp sum (lane tree), the result in every lane.
__device__ __forceinline__ float2 warp_sum2(float2 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
  }
  return make_float2(__shfl_sync(0xffffffffu, v.x, 0), __shfl_sync(0xffffffffu, v.y, 0));
}

// Per-warp partial sums by stage parity; 32 entries whatever the CTA width,
// entries of absent warps stay zero, so every read is in bounds.
struct KuraSmem {
  float2 wpart[2][32];
};

// CTA sum of the per-thread partials: lane tree, then a lane tree over the
// warps' sums.  One CTA barrier; parity `buf` alternates between calls, and
// every thread has read the parity-buf entries before it reaches the next
// call's barrier, which a writer of the call after that has passed.
template <int T>
__device__ __forceinline__ float2 cta_sum2(KuraSmem &sm, float2 part, uint32_t buf) {
  const uint32_t tid = threadIdx.x, lane = tid & 31u;
  part = warp_sum2(part);
  if (lane == 0) sm.wpart[buf][tid >> 5] = part;
  __syncthreads();
  float2 v = sm.wpart[buf][lane];
#pragma unroll
  for (int o = T / 64; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
  }
  return make_float2(__shfl_sync(0xffffffffu, v.x, 0), __shfl_sync(0xffffffffu, v.y, 0));
}

__device__ __forceinline__ void kura_zero_smem(KuraSmem &sm) {
  for (uint32_t i = threadIdx.x; i < 2 * 32; i += blockDim.x) (&sm.wpart[0][0])[i] = make_float2(0.0f, 0.0f);
  __syncthreads();
}

// Records r(t) of one step and accumulates it (thread 0).
__device__ __forceinline__ void kura_record(const KuraArgs &a, uint32_t inst, uint32_t step, float C, float S,
                                            double &rsum) {
  if (threadIdx.x == 0) {
    const float r = sqrtf(C * C + S * S);
    rsum += (double)r;
    if (a.r_out) a.r_out[(size_t)inst * a.r_stride + a.r_base + step] = r;
  }
}

// ---- resident instances: one CTA of T threads, kKOpt oscillators each ----
template <int T>
__global__ void __launch_bounds__(T, 1024 / T) kuramoto_resident_kernel(KuraArgs a) {
  __shared__ KuraSmem sm;
  kura_zero_smem(sm);
  const uint32_t inst = a.inst[blockIdx.x];
  const uint64_t o0 = a.off[inst];
  const uint32_t N = a.size[inst];
  const float K = a.coupling[inst];
  const float inv_n = 1.0f / (float)N;
  const uint32_t tid = threadIdx.x;
  float th[kKOpt], om[kKOpt], ks[kKOpt], sn[kKOpt], cs[kKOpt];
  uint32_t valid = 0;
#pragma unroll
  for (int q = 0; q < kKOpt; ++q) {
    const uint32_t i = q * T + tid;
    th[q] = 0.0f;
    om[q] = 0.0f;
    ks[q] = 0.0f;
    sn[q] = 0.0f;
    cs[q] = 0.0f;
    if (i < N) {
      valid |= 1u << q;
      th[q] = a.theta[o0 + i];
      om[q] = a.omega[o0 + i];
    }
  }
  const float h = a.dt, hh = a.dt * 0.5f, h6 = a.dt / 6.0f;
  // sums of sin/cos of the oscillators' current stage positions
  auto sums = [&]() {
    float2 p = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int q = 0; q < kKOpt; ++q)
      if (valid & (1u << q)) {
        p.x += cs[q];
        p.y += sn[q];
      }
    return p;
  };
#pragma unroll
  for (int q = 0; q < kKOpt; ++q) phase_sincos(th[q], sn[q], cs[q]);
  uint32_t buf = 0;
  float2 m = cta_sum2<T>(sm, sums(), buf);
  buf ^= 1u;
  double rsum = 0.0;
  for (uint32_t step = 0; step < a.n_steps; ++step) {
#pragma unroll 1
    for (int stage = 0; stage < 4; ++stage) {
      const float C = m.x * inv_n, S = m.y * inv_n;
#pragma unroll
      for (int q = 0; q < kKOpt; ++q) {
        const float k = kura_rate(om[q], K, C, S, sn[q], cs[q]);
        float y;
        if (stage == 0) {
          ks[q] = k;
          y = __fmaf_rn(hh, k, th[q]);
        } else if (stage == 1) {
          ks[q] = __fmaf_rn(2.0f, k, ks[q]);
          y = __fmaf_rn(hh, k, th[q]);
        } else if (stage == 2) {
          ks[q] = __fmaf_rn(2.0f, k, ks[q]);
          y = __fmaf_rn(h, k, th[q]);
        } else {
          th[q] = reduce_phase(__fmaf_rn(h6, ks[q] + k, th[q]));
          y = th[q];
        }
        phase_sincos(y, sn[q], cs[q]);
      }
      m = cta_sum2<T>(sm, sums(), buf);
      buf ^= 1u;
    }
    kura_record(a, inst, step, m.x * inv_n, m.y * inv_n, rsum);
  }
#pragma unroll
  for (int q = 0; q < kKOpt; ++q)
    if (valid & (1u << q)) a.theta[o0 + q * T + tid] = th[q];
  if (tid == 0) a.r_sum[inst] += rsum;
}

// ---- cluster instances: CL CTAs of T threads, kKOpt oscillators each ----
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_size() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_index() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}
// Every thread of every CTA of the cluster arrives (release) and waits
// (acquire): writes before the barrier are visible to loads after it.
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Cluster sum of the per-thread partials.  The CTA's sum goes to slot
// [buf][rank] of the instance's partials; after the cluster barrier every
// thread adds slots [buf][0..n) in rank order.  Parity `buf` alternates: a
// CTA writes slot [buf] again only after the next barrier, which every CTA
// reaches after it has read the slots of this call.
template <int T>
__device__ __forceinline__ float2 cluster_sum2(KuraSmem &sm, float2 *xp, uint32_t rank, uint32_t n, float2 part,
                                               uint32_t buf) {
  const float2 c = cta_sum2<T>(sm, part, buf);
  // the barrier's release (arrive) and acquire (wait) at cluster scope order
  // the store before the other CTAs' loads; both go to L2 (.cg)
  if (threadIdx.x == 0) __stcg(xp + buf * kKMaxCluster + rank, c);
  cluster_sync_all();
  float2 m = __ldcg(xp + buf * kKMaxCluster);
  for (uint32_t r = 1; r < n; ++r) {
    const float2 v = __ldcg(xp + buf * kKMaxCluster + r);
    m.x += v.x;
    m.y += v.y;
  }
  return m;
}

// The resident kernel's RK4 over one cluster: CTA `rank` of the cluster
// holds oscillators [rank*T*kKOpt, (rank+1)*T*kKOpt) of the instance.  Every
// CTA runs the same number of stages (the instance's), so every cluster
// barrier is reached by all of them; a cluster is co-scheduled by the
// hardware, so the barrier cannot wait on a CTA that is not resident.
template <int T>
__global__ void __launch_bounds__(T, 1024 / T) kuramoto_cluster_kernel(KuraArgs a) {
  __shared__ KuraSmem sm;
  kura_zero_smem(sm);
  const uint32_t rank = cluster_rank(), ncta = cluster_size();
  const uint32_t inst = a.inst[cluster_index()];
  const uint32_t N = a.size[inst];
  const uint32_t first = rank * (uint32_t)(T * kKOpt);
  const uint64_t o0 = a.off[inst] + first;
  const uint32_t nl = N > first ? min(N - first, (uint32_t)(T * kKOpt)) : 0u;  // this CTA's oscillators
  const float K = a.coupling[inst];
  const float inv_n = 1.0f / (float)N;
  float2 *xp = a.xpart + (size_t)inst * 2 * kKMaxCluster;
  const uint32_t tid = threadIdx.x;
  float th[kKOpt], om[kKOpt], ks[kKOpt], sn[kKOpt], cs[kKOpt];
  uint32_t valid = 0;
#pragma unroll
  for (int q = 0; q < kKOpt; ++q) {
    const uint32_t i = q * T + tid;
    th[q] = 0.0f;
    om[q] = 0.0f;
    ks[q] = 0.0f;
    sn[q] = 0.0f;
    cs[q] = 0.0f;
    if (i < nl) {
      valid |= 1u << q;
      th[q] = a.theta[o0 + i];
      om[q] = a.omega[o0 + i];
    }
  }
  const float h = a.dt, hh = a.dt * 0.5f, h6 = a.dt / 6.0f;
  auto sums = [&]() {
    float2 p = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int q = 0; q < kKOpt; ++q)
      if (valid & (1u << q)) {
        p.x += cs[q];
        p.y += sn[q];
      }
    return p;
  };
#pragma unroll
  for (int q = 0; q < kKOpt; ++q) phase_sincos(th[q], sn[q], cs[q]);
  uint32_t buf = 0;
  float2 m = cluster_sum2<T>(sm, xp, rank, ncta, sums(), buf);
  buf ^= 1u;
  double rsum = 0.0;
  for (uint32_t step = 0; step < a.n_steps; ++step) {
#pragma unroll 1
    for (int stage = 0; stage < 4; ++stage) {
      const float C = m.x * inv_n, S = m.y * inv_n;
#pragma unroll
      for (int q = 0; q < kKOpt; ++q) {
        const float k = kura_rate(om[q], K, C, S, sn[q], cs[q]);
        float y;
        if (stage == 0) {
          ks[q] = k;
          y = __fmaf_rn(hh, k, th[q]);
        } else if (stage == 1) {
          ks[q] = __fmaf_rn(2.0f, k, ks[q]);
          y = __fmaf_rn(hh, k, th[q]);
        } else if (stage == 2) {
          ks[q] = __fmaf_rn(2.0f, k, ks[q]);
          y = __fmaf_rn(h, k, th[q]);
        } else {
          th[q] = reduce_phase(__fmaf_rn(h6, ks[q] + k, th[q]));
          y = th[q];
        }
        phase_sincos(y, sn[q], cs[q]);
      }
      m = cluster_sum2<T>(sm, xp, rank, ncta, sums(), buf);
      buf ^= 1u;
    }
    if (rank == 0) kura_record(a, inst, step, m.x * inv_n, m.y * inv_n, rsum);
  }
#pragma unroll
  for (int q = 0; q < kKOpt; ++q)
    if (valid & (1u << q)) a.theta[o0 + q * T + tid] = th[q];
  if (rank == 0 && tid == 0) a.r_sum[inst] += rsum;
}

// ---- streamed instances: one CTA of 1024 threads, state re-read per stage ----
__global__ void __launch_bounds__(kKStreamThreads, 1) kuramoto_streamed_kernel(KuraArgs a) {
  constexpr int T = kKStreamThreads;
  __shared__ KuraSmem sm;
  kura_zero_smem(sm);
  const uint32_t inst = a.inst[blockIdx.x];
  const uint64_t o0 = a.off[inst];
  const uint32_t N = a.size[inst];
  const float K = a.coupling[inst];
  const float inv_n = 1.0f / (float)N;
  const uint32_t tid = threadIdx.x;
  float *th = a.theta + o0;
  const float *om = a.omega + o0;
  float *ks = a.ks + o0;
  float *yp = a.ypos + o0;
  const float h = a.dt, hh = a.dt * 0.5f, h6 = a.dt / 6.0f;
  uint32_t buf = 0;
  float2 p = make_float2(0.0f, 0.0f);
  for (uint32_t i = tid; i < N; i += T) {
    float s, c;
    phase_sincos(th[i], s, c);
    p.x += c;
    p.y += s;
  }
  float2 m = cta_sum2<T>(sm, p, buf);
  buf ^= 1u;
  double rsum = 0.0;
  for (uint32_t step = 0; step < a.n_steps; ++step) {
#pragma unroll 1
    for (int stage = 0; stage < 4; ++stage) {
      const float C = m.x * inv_n, S = m.y * inv_n;
      p = make_float2(0.0f, 0.0f);
      // every oscillator is touched by the same thread in every stage, so
      // the ks / ypos values a thread reads are the ones it wrote
      for (uint32_t i = tid; i < N; i += T) {
        const float t0 = th[i];
        float s, c;
        phase_sincos(stage == 0 ? t0 : yp[i], s, c);
        const float k = kura_rate(om[i], K, C, S, s, c);
        float y;
        if (stage == 0) {
          ks[i] = k;
          y = __fmaf_rn(hh, k, t0);
        } else if (stage == 1) {
          ks[i] = __fmaf_rn(2.0f, k, ks[i]);
          y = __fmaf_rn(hh, k, t0);
        } else if (stage == 2) {
          ks[i] = __fmaf_rn(2.0f, k, ks[i]);
          y = __fmaf_rn(h, k, t0);
        } else {
          y = reduce_phase(__fmaf_rn(h6, ks[i] + k, t0));
          th[i] = y;
        }
        if (stage < 3) yp[i] = y;
        phase_sincos(y, s, c);
        p.x += c;
        p.y += s;
      }
      m = cta_sum2<T>(sm, p, buf);
      buf ^= 1u;
    }
    kura_record(a, inst, step, m.x * inv_n, m.y * inv_n, rsum);
  }
  if (tid == 0) a.r_sum[inst] += rsum;
}

// Shape bins: 0..3 resident CTAs of 64/128/256/512 threads; 4 streamed;
// 5..8 clusters of 2, 4, 8 CTAs of 512 threads and 8 CTAs of 1024 threads.
constexpr int kKBins = 9;
constexpr int kKStreamBin = 4;
struct KuraShape {
  int threads, cluster;
};
constexpr KuraShape kKShape[kKBins] = {{64, 1}, {128, 1}, {256, 1}, {512, 1}, {kKStreamThreads, 1},
                                       {512, 2},  {512, 4},  {512, 8},  {1024, 8}};
inline int kura_bin(uint32_t n) {
  if (n > kKResident) {
    const uint32_t ctas = (n + kKResident - 1) / kKResident;  // CTAs of 512 threads x 8
    return ctas <= 2 ? 5 : ctas <= 4 ? 6 : ctas <= 8 ? 7 : 8;
  }
  const uint32_t need = (n + kKOpt - 1) / kKOpt;
  return need <= 64 ? 0 : need <= 128 ? 1 : need <= 256 ? 2 : 3;
}

// Launches bin b's `n` instances on stream s (cluster bins through the
// extended launch with the cluster dimension attribute).
inline cudaError_t kura_launch(int b, uint32_t n, const KuraArgs &a, cudaStream_t s) {
  const KuraShape sh = kKShape[b];
  if (sh.cluster == 1) {
    switch (b) {
      case 0: kuramoto_resident_kernel<64><<<n, 64, 0, s>>>(a); break;
      case 1: kuramoto_resident_kernel<128><<<n, 128, 0, s>>>(a); break;
      case 2: kuramoto_resident_kernel<256><<<n, 256, 0, s>>>(a); break;
      case 3: kuramoto_resident_kernel<512><<<n, 512, 0, s>>>(a); break;
      default: kuramoto_streamed_kernel<<<n, kKStreamThreads, 0, s>>>(a); break;
    }
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(n * (uint32_t)sh.cluster);
  cfg.blockDim = dim3((uint32_t)sh.threads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)sh.cluster;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  if (sh.threads == 512) return cudaLaunchKernelEx(&cfg, kuramoto_cluster_kernel<512>, a);
  return cudaLaunchKernelEx(&cfg, kuramoto_cluster_kernel<1024>, a);
}

// Clusters of bin b that can be resident at once on the current device (0:
// the shape cannot run here).
inline int kura_max_clusters(int b) {
  const KuraShape sh = kKShape[b];
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((uint32_t)sh.cluster);
  cfg.blockDim = dim3((uint32_t)sh.threads);
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)sh.cluster;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int n = 0;
  const cudaError_t e = sh.threads == 512
                            ? cudaOccupancyMaxActiveClusters(&n, kuramoto_cluster_kernel<512>, &cfg)
                            : cudaOccupancyMaxActiveClusters(&n, kuramoto_cluster_kernel<1024>, &cfg);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  return n;
}

}  // namespace sg

using namespace sg;

struct sg_kura {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t n_inst = 0;
  uint64_t total = 0;
  float dt = 0;
  float *d_theta = nullptr, *d_omega = nullptr, *d_k = nullptr, *d_r = nullptr;
  float *d_ks = nullptr, *d_ypos = nullptr;
  float2 *d_xpart = nullptr;
  uint64_t *d_off = nullptr;
  uint32_t *d_size = nullptr, *d_inst = nullptr;
  double *d_rsum = nullptr;
  uint64_t steps_done = 0, r_cap = 0, r_written = 0;
  uint32_t bin_count[kKBins] = {};
  uint32_t bin_off[kKBins] = {};
  cudaStream_t bin_stream[kKBins] = {};  // one stream per non-empty bin
  cudaEvent_t fork = nullptr, join[kKBins] = {};

  void release() {
    for (int b = 0; b < kKBins; ++b) {
      if (join[b]) cudaEventDestroy(join[b]);
      if (bin_stream[b]) cudaStreamDestroy(bin_stream[b]);
      join[b] = nullptr;
      bin_stream[b] = nullptr;
    }
    if (fork) cudaEventDestroy(fork);
    fork = nullptr;
    cudaFree(d_xpart);
    cudaFree(d_theta);
    cudaFree(d_omega);
    cudaFree(d_ks);
    cudaFree(d_ypos);
    cudaFree(d_k);
    cudaFree(d_off);
    cudaFree(d_size);
    cudaFree(d_rsum);
    cudaFree(d_inst);
    cudaFree(d_r);
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
  }
};

namespace {
template <typename F> int krun(F f) {
  try {
    f();
    return SG_OK;
  } catch (const Fail &e) {
    return e.code;
  } catch (const std::exception &e) {
    set_error(e.what());
    return SG_E_INVALID;
  }
}
}  // namespace

extern "C" {

int sg_kuramoto_create(sg_kura **out, int device, uint32_t n_inst, const uint32_t *sizes, const float *coupling,
                       float dt) {
  return krun([&] {
    SG_REQUIRE(out && sizes && coupling, SG_E_INVALID, "null argument");
    *out = nullptr;
    SG_REQUIRE(n_inst > 0, SG_E_INVALID, "no instances");
    SG_REQUIRE(std::isfinite(dt) && dt > 0, SG_E_INVALID, "dt must be finite and > 0");
    std::vector<uint64_t> offs(n_inst);
    std::vector<uint32_t> bins[kKBins];
    uint64_t total = 0;
    for (uint32_t i = 0; i < n_inst; ++i) {
      SG_REQUIRE(sizes[i] >= 1 && sizes[i] <= kKMaxSize, SG_E_INVALID,
                 "instance sizes must be in [1, 65536] oscillators");
      SG_REQUIRE(std::isfinite(coupling[i]), SG_E_INVALID, "coupling strengths must be finite");
      offs[i] = total;
      total += sizes[i];
    }
    int ndev = 0;
    SG_CUDA(cudaGetDeviceCount(&ndev));
    SG_REQUIRE(device >= 0 && device < ndev, SG_E_INVALID, "device ordinal out of range");
    SG_CUDA(cudaSetDevice(device));
    // cluster shapes this device can hold; instances of a shape it cannot
    // take the streamed form (as every instance above 4096 oscillators does
    // when SG_KURAMOTO_STREAMED is set, which the tests use to check it)
    const char *force = std::getenv("SG_KURAMOTO_STREAMED");
    const bool no_cluster = force && force[0] && force[0] != '0';
    bool cluster_ok[kKBins] = {};
    for (int b = 0; b < kKBins; ++b)
      cluster_ok[b] = !no_cluster && kKShape[b].cluster > 1 && kura_max_clusters(b) > 0;
    bool streamed = false, clustered = false;
    for (uint32_t i = 0; i < n_inst; ++i) {
      int b = kura_bin(sizes[i]);
      if (kKShape[b].cluster > 1 && !cluster_ok[b]) b = kKStreamBin;
      bins[b].push_back(i);
      streamed |= b == kKStreamBin;
      clustered |= kKShape[b].cluster > 1;
    }
    auto *kb = new sg_kura();
    kb->device = device;
    kb->n_inst = n_inst;
    kb->total = total;
    kb->dt = dt;
    // largest instances first in each bin: the CTAs are handed to the SMs
    // in block order, so the long ones start at once and the short ones
    // fill the SMs as they free up (longest-processing-time-first)
    std::vector<uint32_t> order;
    for (int b = 0; b < kKBins; ++b) {
      std::stable_sort(bins[b].begin(), bins[b].end(),
                       [&](uint32_t x, uint32_t y) { return sizes[x] > sizes[y]; });
      kb->bin_off[b] = (uint32_t)order.size();
      kb->bin_count[b] = (uint32_t)bins[b].size();
      order.insert(order.end(), bins[b].begin(), bins[b].end());
    }
    try {
      SG_CUDA(cudaStreamCreateWithFlags(&kb->stream, cudaStreamNonBlocking));
      SG_CUDA(cudaEventCreateWithFlags(&kb->fork, cudaEventDisableTiming));
      for (int b = 0; b < kKBins; ++b)
        if (kb->bin_count[b]) {
          SG_CUDA(cudaStreamCreateWithFlags(&kb->bin_stream[b], cudaStreamNonBlocking));
          SG_CUDA(cudaEventCreateWithFlags(&kb->join[b], cudaEventDisableTiming));
        }
      if (clustered) {
        SG_CUDA(cudaMalloc(&kb->d_xpart, (size_t)n_inst * 2 * kKMaxCluster * sizeof(float2)));
        SG_CUDA(cudaMemset(kb->d_xpart, 0, (size_t)n_inst * 2 * kKMaxCluster * sizeof(float2)));
      }
      SG_CUDA(cudaMalloc(&kb->d_theta, total * 4));
      SG_CUDA(cudaMalloc(&kb->d_omega, total * 4));
      if (streamed) {
        SG_CUDA(cudaMalloc(&kb->d_ks, total * 4));
        SG_CUDA(cudaMalloc(&kb->d_ypos, total * 4));
      }
      SG_CUDA(cudaMalloc(&kb->d_k, (size_t)n_inst * 4));
      SG_CUDA(cudaMalloc(&kb->d_off, (size_t)n_inst * 8));
      SG_CUDA(cudaMalloc(&kb->d_size, (size_t)n_inst * 4));
      SG_CUDA(cudaMalloc(&kb->d_rsum, (size_t)n_inst * 8));
      SG_CUDA(cudaMalloc(&kb->d_inst, (size_t)n_inst * 4));
      SG_CUDA(cudaMemcpy(kb->d_inst, order.data(), (size_t)n_inst * 4, cudaMemcpyHostToDevice));
      SG_CUDA(cudaMemcpy(kb->d_k, coupling, (size_t)n_inst * 4, cudaMemcpyHostToDevice));
      SG_CUDA(cudaMemcpy(kb->d_off, offs.data(), (size_t)n_inst * 8, cudaMemcpyHostToDevice));
      SG_CUDA(cudaMemcpy(kb->d_size, sizes, (size_t)n_inst * 4, cudaMemcpyHostToDevice));
      SG_CUDA(cudaMemset(kb->d_rsum, 0, (size_t)n_inst * 8));
      SG_CUDA(cudaMemset(kb->d_theta, 0, total * 4));
      SG_CUDA(cudaMemset(kb->d_omega, 0, total * 4));
      SG_CUDA(cudaDeviceSynchronize());
    } catch (...) {
      kb->release();
      delete kb;
      throw;
    }
    *out = kb;
  });
}

int sg_kuramoto_destroy(sg_kura *kb) {
  if (!kb) return SG_OK;
  cudaSetDevice(kb->device);
  if (kb->stream) cudaStreamSynchronize(kb->stream);
  kb->release();
  delete kb;
  return SG_OK;
}

int sg_kuramoto_total(sg_kura *kb, uint64_t *out) {
  return krun([&] {
    SG_REQUIRE(kb && out, SG_E_INVALID, "null argument");
    *out = kb->total;
  });
}

int sg_kuramoto_set_state(sg_kura *kb, const float *theta, const float *omega) {
  return krun([&] {
    SG_REQUIRE(kb && theta && omega, SG_E_INVALID, "null argument");
    for (uint64_t i = 0; i < kb->total; ++i)
      SG_REQUIRE(std::isfinite(theta[i]) && std::isfinite(omega[i]), SG_E_INVALID,
                 "phases and frequencies must be finite");
    SG_CUDA(cudaSetDevice(kb->device));
    SG_CUDA(cudaMemcpyAsync(kb->d_theta, theta, kb->total * 4, cudaMemcpyHostToDevice, kb->stream));
    SG_CUDA(cudaMemcpyAsync(kb->d_omega, omega, kb->total * 4, cudaMemcpyHostToDevice, kb->stream));
    SG_CUDA(cudaStreamSynchronize(kb->stream));
  });
}

int sg_kuramoto_record(sg_kura *kb, uint64_t max_steps) {
  return krun([&] {
    SG_REQUIRE(kb, SG_E_INVALID, "null argument");
    SG_CUDA(cudaSetDevice(kb->device));
    SG_CUDA(cudaStreamSynchronize(kb->stream));
    cudaFree(kb->d_r);
    kb->d_r = nullptr;
    kb->r_cap = 0;
    kb->r_written = 0;
    if (max_steps) {
      SG_CUDA(cudaMalloc(&kb->d_r, (size_t)kb->n_inst * max_steps * 4));
      kb->r_cap = max_steps;
    }
  });
}

int sg_kuramoto_run(sg_kura *kb, uint32_t n_steps) {
  return krun([&] {
    SG_REQUIRE(kb, SG_E_INVALID, "null argument");
    if (kb->d_r) SG_REQUIRE(kb->r_written + n_steps <= kb->r_cap, SG_E_OVERFLOW, "r(t) record is full");
    if (n_steps == 0) return;
    SG_CUDA(cudaSetDevice(kb->device));
    KuraArgs a{};
    a.off = kb->d_off;
    a.size = kb->d_size;
    a.coupling = kb->d_k;
    a.theta = kb->d_theta;
    a.omega = kb->d_omega;
    a.ks = kb->d_ks;
    a.ypos = kb->d_ypos;
    a.dt = kb->dt;
    a.n_steps = n_steps;
    a.r_out = kb->d_r;
    a.r_stride = kb->r_cap;
    a.r_base = kb->r_written;
    a.r_sum = kb->d_rsum;
    a.xpart = kb->d_xpart;
    // every bin on its own stream, forked from and joined to the handle's
    // stream; the cluster bins (the longest-running CTAs) are queued first
    SG_CUDA(cudaEventRecord(kb->fork, kb->stream));
    for (int b = kKBins - 1; b >= 0; --b) {
      const uint32_t n = kb->bin_count[b];
      if (!n) continue;
      a.inst = kb->d_inst + kb->bin_off[b];
      SG_CUDA(cudaStreamWaitEvent(kb->bin_stream[b], kb->fork, 0));
      SG_CUDA(kura_launch(b, n, a, kb->bin_stream[b]));
      SG_CUDA(cudaEventRecord(kb->join[b], kb->bin_stream[b]));
      SG_CUDA(cudaStreamWaitEvent(kb->stream, kb->join[b], 0));
    }
    kb->steps_done += n_steps;
    if (kb->d_r) kb->r_written += n_steps;
  });
}

int sg_kuramoto_synchronize(sg_kura *kb) {
  return krun([&] {
    SG_REQUIRE(kb, SG_E_INVALID, "null argument");
    SG_CUDA(cudaSetDevice(kb->device));
    SG_CUDA(cudaStreamSynchronize(kb->stream));
  });
}

int sg_kuramoto_get_theta(sg_kura *kb, float *theta) {
  return krun([&] {
    SG_REQUIRE(kb && theta, SG_E_INVALID, "null argument");
    SG_CUDA(cudaSetDevice(kb->device));
    SG_CUDA(cudaMemcpyAsync(theta, kb->d_theta, kb->total * 4, cudaMemcpyDeviceToHost, kb->stream));
    SG_CUDA(cudaStreamSynchronize(kb->stream));
  });
}

int sg_kuramoto_get_r(sg_kura *kb, float *r, uint64_t cap, uint64_t *n_steps) {
  return krun([&] {
    SG_REQUIRE(kb && n_steps, SG_E_INVALID, "null argument");
    SG_REQUIRE(kb->d_r, SG_E_STATE, "r(t) recording is not enabled");
    SG_REQUIRE((uint64_t)kb->n_inst * kb->r_written <= cap, SG_E_INVALID, "output buffer too small");
    SG_CUDA(cudaSetDevice(kb->device));
    SG_CUDA(cudaStreamSynchronize(kb->stream));
    if (kb->r_written) {
      SG_REQUIRE(r, SG_E_INVALID, "null argument");
      SG_CUDA(cudaMemcpy2D(r, kb->r_written * 4, kb->d_r, kb->r_cap * 4, kb->r_written * 4, kb->n_inst,
                           cudaMemcpyDeviceToHost));
    }
    *n_steps = kb->r_written;
  });
}

int sg_kuramoto_get_r_mean(sg_kura *kb, double *r_mean) {
  return krun([&] {
    SG_REQUIRE(kb && r_mean, SG_E_INVALID, "null argument");
    SG_CUDA(cudaSetDevice(kb->device));
    SG_CUDA(cudaMemcpyAsync(r_mean, kb->d_rsum, (size_t)kb->n_inst * 8, cudaMemcpyDeviceToHost, kb->stream));
    SG_CUDA(cudaStreamSynchronize(kb->stream));
    for (uint32_t i = 0; i < kb->n_inst; ++i)
      r_mean[i] = kb->steps_done ? r_mean[i] / (double)kb->steps_done : 0.0;
  });
}

int sg_kuramoto_stream(sg_kura *kb, void **out) {
  if (!kb || !out) return SG_E_INVALID;
  *out = (void *)kb->stream;
  return SG_OK;
}

}  // extern "C"
