// step_kernels.cuh — the device side of one simulation step.
//
// One step of the reference (P/api/net/network/step.rs:18-189) runs as three
// kernels on the network's stream:
//
//   neuron_kernel<M>  one thread per neuron (one launch per population):
//                     read + clear the current ring slot (and the kinetic
//                     rings), integrate the model, ballot the spikes into a
//                     bitmask word per warp, append spiking neurons to the
//                     active list, update STDP traces.
//   expand_kernel     one warp per spiking neuron walks its outgoing CSR row
//                     (coalesced), one thread per Poisson source rolls the
//                     source; every synaptic event (edge id, weight, target
//                     cell) is appended to the bin of its post tile.  Pair-STDP
//                     depression of the walked edges is fused here.
//   apply_kernel      one block per post tile applies the tile's events to
//                     the ring in the reference's summation order.
//
// Determinism.  The reference adds the events of a step to each ring cell in
// (spiking pre ascending, CSR row order) and then Poisson-source order
// (push.rs:143-172, step.rs:166-185).  That order is exactly ascending CSR
// edge id, with source edges numbered after all neuron edges; each event
// carries that id as its key.  apply_kernel resolves cells touched by several
// events in rounds: every pending event posts its key with atomicMin to a
// shared-memory owner slot hashed from its cell, the owner of each slot adds
// its weight, the rest retry.  Events sharing a cell always share a slot, so
// each cell receives its adds in ascending key order: the reference's order,
// with the same float rounding.
#pragma once
#include <cstdint>

#include "common.cuh"
#include "models.cuh"

namespace sg {

struct StepArgs {
  // step bookkeeping
  unsigned long long *step;  // device step counter
  uint32_t *n_active;
  uint32_t *active;
  uint32_t *last_bits;  // spike bitmask of the last step, [Nd/32]
  uint32_t *raster;     // [raster_cap][Nd/32] or null
  uint32_t raster_cap;
  uint32_t words;
  uint32_t *done;
  unsigned long long *ev_step;
  unsigned long long *ev_total;
  uint32_t *stat_spk;
  unsigned long long *stat_ev;
  uint32_t stat_cap;
  unsigned long long *clamp_hits;
  // rings: [n_rings][32][Nd]
  float *ring;
  uint32_t Nd;
  // kinetic ExpOne profiles (ring k+1)
  int n_kin;
  float kin_a[3];
  float kin_erev[3];
  float *kin_g;  // [n_kin][Nd]
  // CSR (device neuron indices)
  const uint32_t *row_ptr;
  const uint32_t *col;
  float *w;
  const uint8_t *code;
  uint32_t n_edges;
  // Poisson sources
  uint32_t n_src;
  const float *src_p;
  const uint32_t *src_seed;
  const uint32_t *src_ptr;
  const uint32_t *src_post;
  const float *src_w;
  const uint8_t *src_code;
  // bins
  uint32_t tshift;
  uint32_t n_tiles;
  uint32_t hbits;
  const unsigned long long *bin_base;
  uint32_t *bin_cnt;
  uint32_t *bkey;
  float *bw;
  uint32_t *bcell;
  // scatter mode
  int deterministic;
  // pair STDP
  int stdp;
  float *x_pre;
  float *x_post;
  float d_pre, d_post, a_plus, a_minus, w_min, w_max;
  const uint32_t *in_ptr;
  const uint32_t *in_edge;
  const uint32_t *in_pre;
  double *drift;
};

struct PopArgs {
  float *state;
  const float *params;
  uint32_t n, cap, dev_off;
  float ln_na, ln_k;  // GPEA constants
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// ---------------------------------------------------------------------------
// neuron phase
// ---------------------------------------------------------------------------
template <int MODEL>
__global__ void __launch_bounds__(256) neuron_kernel(StepArgs a, PopArgs p) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;  // < cap (multiple of 32)
  if (i >= p.cap) return;                                    // whole warps only
  const unsigned long long step = *a.step;
  const uint32_t slot = (uint32_t)(step & 31ull);
  const uint32_t gi = p.dev_off + i;
  bool spike = false;
  if (i < p.n) {
    // 1-2. read the slot, clear it (step.rs:27-34)
    float *rs = a.ring + (size_t)slot * a.Nd + gi;
    float x = *rs;
    *rs = 0.0f;
    // 2b. kinetic ExpOne rings (step.rs:56-70, :338-345); V from step start
    if (a.n_kin > 0) {
      const float v0 = p.state[i];
      for (int k = 0; k < a.n_kin; ++k) {
        float *ks = a.ring + ((size_t)(k + 1) * kSlots + slot) * a.Nd + gi;
        const float jump = *ks;
        *ks = 0.0f;
        float *g = a.kin_g + (size_t)k * a.Nd + gi;
        const float gn = *g * a.kin_a[k] + jump;
        *g = gn;
        x += gn * (a.kin_erev[k] - v0);
      }
    }
    if (clamps(MODEL)) {
      const float xc = fminf(fmaxf(x, -100.0f), 100.0f);
      if (a.clamp_hits != nullptr && xc != x) atomicAdd(a.clamp_hits, 1ull);
      x = xc;
    }
    // dt = param column 0 of neuron 0, broadcast (population.rs:307,361)
    const float dt = __ldg(p.params);
    const Soa c{p.state, p.params, p.cap, i};
    if (MODEL == kLIF) spike = lif_step(c, x, dt);
    else if (MODEL == kIZH) spike = izh_step(c, x, dt);
    else if (MODEL == kGPEA) spike = gpea_step(c, x, dt, p.ln_na, p.ln_k);
    else spike = hh_step(c, x, dt);
  }
  // 4. compaction: warp ballot -> bitmask word + active-list append
  const uint32_t m = __ballot_sync(0xffffffffu, spike);
  const uint32_t lane = lane_id();
  uint32_t base = 0;
  if (lane == 0) {
    a.last_bits[gi >> 5] = m;
    if (a.raster != nullptr) a.raster[(size_t)(step % a.raster_cap) * a.words + (gi >> 5)] = m;
    if (m) base = atomicAdd(a.n_active, (uint32_t)__popc(m));
  }
  base = __shfl_sync(0xffffffffu, base, 0);
  if (spike) a.active[base + __popc(m & ((1u << lane) - 1u))] = gi;
  // pair-STDP traces: x = fma(x, d, s) (P/api/learn/brain.rs:212-222)
  if (a.stdp && i < p.n) {
    const float add = spike ? 1.0f : 0.0f;
    a.x_pre[gi] = __fmaf_rn(a.x_pre[gi], a.d_pre, add);
    a.x_post[gi] = __fmaf_rn(a.x_post[gi], a.d_post, add);
  }
}

// ---------------------------------------------------------------------------
// expand phase
// ---------------------------------------------------------------------------
// Append one event to the bin of its post tile.  `mask` = lanes of the warp
// executing this call together; reservation is warp-aggregated per tile.
__device__ __forceinline__ void emit_event(const StepArgs &a, uint32_t mask, uint32_t key,
                                           uint32_t post, float w, uint8_t code,
                                           unsigned long long step) {
  const uint32_t slot = (uint32_t)((step + max(code_delay(code), 1u)) & 31ull);
  const uint32_t ringi = code_ring(code);
  if (!a.deterministic) {
    atomicAdd(a.ring + ((size_t)ringi * kSlots + slot) * a.Nd + post, w);
    return;
  }
  const uint32_t tile = post >> a.tshift;
  const uint32_t cell = ((ringi * kSlots + slot) << a.tshift) | (post & ((1u << a.tshift) - 1u));
  const uint32_t peers = __match_any_sync(mask, tile);
  const uint32_t lane = lane_id();
  const uint32_t leader = __ffs(peers) - 1;
  uint32_t off = 0;
  if (lane == leader) off = atomicAdd(a.bin_cnt + tile, (uint32_t)__popc(peers));
  off = __shfl_sync(peers, off, leader);
  const unsigned long long pos = a.bin_base[tile] + off + __popc(peers & ((1u << lane) - 1u));
  a.bkey[pos] = key;
  a.bw[pos] = w;
  a.bcell[pos] = cell;
}

__global__ void __launch_bounds__(256) expand_kernel(StepArgs a, uint32_t src_blocks) {
  const unsigned long long step = *a.step;
  const uint32_t lane = lane_id();
  if (blockIdx.x >= src_blocks) {
    // --- spiking neurons: one warp per active row (push.rs:143-172) ---
    const uint32_t n_act = *a.n_active;
    const uint32_t warps_per_block = blockDim.x >> 5;
    const uint32_t gw = (blockIdx.x - src_blocks) * warps_per_block + (threadIdx.x >> 5);
    const uint32_t nw = (gridDim.x - src_blocks) * warps_per_block;
    unsigned long long ev = 0;
    for (uint32_t r = gw; r < n_act; r += nw) {
      const uint32_t pre = a.active[r];
      const uint32_t beg = __ldg(a.row_ptr + pre), end = __ldg(a.row_ptr + pre + 1);
      ev += end - beg;
      for (uint32_t e0 = beg; e0 < end; e0 += 32) {
        const uint32_t e = e0 + lane;
        const bool ok = e < end;
        const uint32_t mask = __ballot_sync(0xffffffffu, ok);
        if (ok) {
          const uint32_t post = __ldg(a.col + e);
          const float w = a.w[e];
          const uint8_t code = __ldg(a.code + e);
          emit_event(a, mask, e, post, w, code, step);
          if (a.stdp && code_stdp(code)) {
            // depression at a pre spike, pushed weight is the pre-update one
            const float w1 = fminf(fmaxf(w - a.a_minus * a.x_post[post], a.w_min), a.w_max);
            a.w[e] = w1;
            atomicAdd(a.drift, (double)w1 - (double)w);
          }
        }
      }
    }
    if (lane == 0 && ev) atomicAdd(a.ev_step, ev);
  } else {
    // --- Poisson sources: one thread per source (step.rs:166-185) ---
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    bool fired = false;
    uint32_t beg = 0, end = 0;
    if (s < a.n_src) {
      const float p = a.src_p[s];
      fired = p > 0.0f && poisson_spike(a.src_seed[s], 0, step, p);
      if (fired) {
        beg = a.src_ptr[s];
        end = a.src_ptr[s + 1];
      }
    }
    uint32_t deg = end - beg;
    uint32_t maxdeg = deg;
    for (int o = 16; o > 0; o >>= 1) maxdeg = max(maxdeg, __shfl_xor_sync(0xffffffffu, maxdeg, o));
    for (uint32_t k = 0; k < maxdeg; ++k) {
      const bool ok = k < deg;
      const uint32_t mask = __ballot_sync(0xffffffffu, ok);
      if (ok) {
        const uint32_t j = beg + k;
        emit_event(a, mask, a.n_edges + j, a.src_post[j], a.src_w[j], a.src_code[j], step);
      }
    }
    unsigned long long ev = deg;
    for (int o = 16; o > 0; o >>= 1) ev += __shfl_xor_sync(0xffffffffu, ev, o);
    if (lane == 0 && ev) atomicAdd(a.ev_step, ev);
  }
}

// Pair-STDP potentiation: one warp per spiking post walks its plastic
// in-edges (runs after expand_kernel, so it sees this step's depression).
__global__ void __launch_bounds__(256) stdp_ltp_kernel(StepArgs a) {
  const uint32_t n_act = *a.n_active;
  const uint32_t lane = lane_id();
  const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  for (uint32_t r = gw; r < n_act; r += nw) {
    const uint32_t post = a.active[r];
    const uint32_t beg = a.in_ptr[post], end = a.in_ptr[post + 1];
    for (uint32_t k = beg + lane; k < end; k += 32) {
      const uint32_t e = a.in_edge[k];
      const float w0 = a.w[e];
      const float w1 = fminf(fmaxf(w0 + a.a_plus * a.x_pre[a.in_pre[k]], a.w_min), a.w_max);
      a.w[e] = w1;
      atomicAdd(a.drift, (double)w1 - (double)w0);
    }
  }
}

// ---------------------------------------------------------------------------
// apply phase
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t owner_slot(uint32_t cell, uint32_t hbits) {
  return (cell * 2654435761u) >> (32 - hbits);
}

__device__ __forceinline__ void end_of_step(const StepArgs &a) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const uint32_t t = atomicAdd(a.done, 1u);
    if (t == gridDim.x - 1) {
      __threadfence();
      const unsigned long long step = *a.step;
      const uint32_t n_act = *(volatile uint32_t *)a.n_active;
      const unsigned long long ev = *(volatile unsigned long long *)a.ev_step;
      if (a.stat_cap) {
        a.stat_spk[step % a.stat_cap] = n_act;
        a.stat_ev[step % a.stat_cap] = ev;
      }
      *a.ev_total += ev;
      *a.ev_step = 0;
      *a.n_active = 0;
      *a.done = 0;
      *a.step = step + 1;
      __threadfence();
    }
  }
}

constexpr uint32_t kDone = 0xFFFFFFFFu;

__global__ void __launch_bounds__(512) apply_kernel(StepArgs a) {
  extern __shared__ uint32_t owner[];
  const uint32_t hbits = a.hbits;
  const uint32_t tmask = (1u << a.tshift) - 1u;
  if (a.deterministic) {
    for (uint32_t tile = blockIdx.x; tile < a.n_tiles; tile += gridDim.x) {
      const uint32_t cnt = a.bin_cnt[tile];
      if (cnt == 0) continue;  // uniform across the block
      const unsigned long long base = a.bin_base[tile];
      uint32_t *cellp = a.bcell + base;
      const uint32_t *keyp = a.bkey + base;
      const float *wp = a.bw + base;
      for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) owner[owner_slot(cellp[k], hbits)] = kDone;
      __syncthreads();
      bool pending = true;
      while (__syncthreads_or(pending)) {
        // (a) post keys
        pending = false;
        for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) {
          const uint32_t c = cellp[k];
          if (c != kDone) atomicMin(&owner[owner_slot(c, hbits)], keyp[k]);
        }
        __syncthreads();
        // (b) the smallest key of each slot applies its add
        for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) {
          const uint32_t c = cellp[k];
          if (c == kDone) continue;
          if (owner[owner_slot(c, hbits)] == keyp[k]) {
            float *r = a.ring + (size_t)(c >> a.tshift) * a.Nd + ((size_t)tile << a.tshift) + (c & tmask);
            *r = *r + wp[k];
            cellp[k] = kDone;
          } else {
            pending = true;
          }
        }
        __syncthreads();
        // (c) free the slots still wanted
        for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) {
          const uint32_t c = cellp[k];
          if (c != kDone) owner[owner_slot(c, hbits)] = kDone;
        }
      }
      if (threadIdx.x == 0) a.bin_cnt[tile] = 0;
      __syncthreads();
    }
  }
  end_of_step(a);
}

// ---------------------------------------------------------------------------
// inject_current (build.rs:243-275): values land in the slot the next step
// reads.  `sequential` = the index list has repeats, apply in list order.
// ---------------------------------------------------------------------------
__global__ void inject_kernel(float *ring, uint32_t Nd, const unsigned long long *step,
                              const uint32_t *idx, const float *vals, uint64_t n, uint32_t dev_off,
                              int sequential) {
  const uint32_t slot = (uint32_t)(*step & 31ull);
  float *rs = ring + (size_t)slot * Nd + dev_off;
  if (sequential) {
    if (blockIdx.x == 0 && threadIdx.x == 0)
      for (uint64_t k = 0; k < n; ++k) rs[idx[k]] = rs[idx[k]] + vals[k];
    return;
  }
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (uint64_t)gridDim.x * blockDim.x)
    rs[idx[k]] = rs[idx[k]] + vals[k];
}

}  // namespace sg
