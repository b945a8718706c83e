// step_kernels.cuh — the device side of one simulation step.
//
// One step of the reference (P/api/net/network/step.rs:18-189) runs as two
// kernels on the network's stream:
//
//   neuron_kernel<M>  one thread per neuron, one launch per population:
//                     read + clear the current ring slot (and the kinetic
//                     rings), integrate the model, ballot the spikes into a
//                     bitmask word per warp, write the block's spiking
//                     neurons in ascending order to its slot of the spike
//                     list (no global atomics), update the STDP traces.
//   scatter_red_kernel  (networks whose ring sums are exact in FP32, and the
//                     atomic mode) warps take the step's spiking rows, read
//                     each row once, whole and coalesced, and add every event
//                     to its ring cell in L2 with red.global.add: any order of
//                     the adds gives the reference's bits when every partial
//                     sum is exact.
//   scatter_kernel    (every other network) one persistent block per SM;
//                     block j owns the posts [j*P, (j+1)*P).  It walks the
//                     spike list in neuron order, reads the segment of each
//                     spiking row that targets its posts (rows are sorted by
//                     post; a per-row table holds the segment bounds), rolls
//                     the Poisson sources that target its posts, and applies
//                     every event to the ring cells it owns, in order.
// A population driven one-to-one by delay-1 Poisson sources takes that drive
// in the neuron kernel of the next step (PopArgs::drv).
//
// Determinism of the ordered scatter.  The reference adds the events of one step to each ring cell
// in (spiking pre ascending, CSR row order) and then Poisson-source order
// (push.rs:143-172, step.rs:166-185).  A block generates its events exactly
// in that order (rows are stored sorted by post with a stable sort, which
// keeps the relative order of repeated synapses to one post), in windows of
// up to kWin events.  Inside a window every event is prepended to the list of
// its cell's bucket (kBuckets buckets hashed from the cell); walking that list,
// an event finds its rank among the window's earlier events of the same
// cell, its predecessor, and whether a later one exists.  Rank-0 events load
// the ring value (all loads in flight together), partial sums then advance
// one rank per level in shared memory, and the last event of each cell
// stores the cell's value.  Windows are applied one after another.  Every
// cell therefore receives its adds in the reference's order, with the
// reference's rounding.
#pragma once
#include <cuda_fp8.h>

#include <cstdint>

#include "common.cuh"
#include "models.cuh"

namespace sg {

constexpr uint32_t kNeuronBlock = 1024;  // neurons per neuron-kernel block (= spike-list slot)
constexpr uint32_t kScatterThreads = 1024;
constexpr uint32_t kScatterBlocksPerSM = 1;
constexpr uint32_t kWin = 8192;          // events per window
constexpr uint32_t kBucketBits = 13;
constexpr uint32_t kBuckets = 1u << kBucketBits;  // per-window event lists, by hashed cell
constexpr uint32_t kPreChunk = 4 * kScatterThreads;  // spiking rows per sub-chunk (4 per thread)
constexpr uint32_t kBlkChunk = kScatterThreads;      // spike-list slots scanned per chunk
constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr unsigned long long kEmpty64 = ~0ull;
constexpr uint32_t kMaxPops = 16;
constexpr uint32_t kMaxTm = 8;  // short-term plasticity profiles on the device

// a compile-time flag passed to a generic lambda (one instantiation per value)
template <bool B> struct BoolC {
  static constexpr bool value = B;
};

// neurons per thread: LIF/Izhikevich move 4 neighbours with 128-bit accesses;
// GPEA/HH are compute heavy and keep one neuron per thread
#ifndef SG_NEURON_MIN_BLOCKS
#define SG_NEURON_MIN_BLOCKS 7  // resident 128-thread blocks per SM asked of the lean LIF kernel (7 x 148 >= 977 blocks of a million neurons)
#endif
// The lean LIF form moves 8 neurons per thread (two 128-bit accesses per
// array): 128-thread blocks, 8 resident per SM, so a million-neuron
// population updates in one wave of blocks.  Izhikevich (more state and
// per-neuron parameters) and the full form keep 4 per thread (256-thread
// blocks, 4 resident per SM in the lean form).
template <int M, bool FULL> struct NeuronCfg {
  static constexpr int NPT = (M == kLIF && !FULL) ? 8 : (M == kLIF || M == kIZH) ? 4 : 1;
  static constexpr int THREADS = (int)kNeuronBlock / NPT;
  static constexpr int MIN_BLOCKS = FULL ? 1 : NPT == 8 ? SG_NEURON_MIN_BLOCKS : NPT == 4 ? 4 : 1;
};

struct StepArgs {
  // step bookkeeping
  unsigned long long *step;  // device step counter
  uint32_t *blk_cnt;         // [n_blk] spikes per neuron block
  uint2 *spk;                // [Nd] (pre, row_start) per block slot, ascending
  uint32_t n_blk;
  uint32_t *last_bits;       // spike bitmask of the last step, [Nd/32]
  uint32_t *raster;          // [raster_cap][Nd/32] or null
  uint32_t raster_cap;
  uint32_t words;
  uint32_t *done;
  unsigned long long *ev_step;
  unsigned long long *ev_total;
  unsigned long long *ev_src_step;   // of which Poisson-source events (this step)
  unsigned long long *ev_src_total;
  uint32_t *stat_spk;
  unsigned long long *stat_ev;
  uint32_t stat_cap;
  unsigned long long *clamp_hits;
  // per-neuron spike statistics (null when off): count, last spike step
  // (steps since they were enabled, ~0u before the first), FP64 sums of the
  // inter-spike intervals and of their squares (in steps: exact integers)
  uint32_t *ns_count;
  uint32_t *ns_last;
  double *ns_s1;
  double *ns_s2;
  unsigned long long ns_step0;
  // rings: [n_rings][nslots][Nd]; a step's arrivals go to slot step % nslots
  // (nslots = the largest effective delay + 1, at most 32: the reference's
  // 32-slot ring, P/api/net/delay.rs:30-101, without the slots no delay reaches)
  float *ring;
  uint32_t Nd;
  uint32_t nslots;
  // kinetic synapse profiles (ring k+1): kind (0 ExpOne, 1 ExpTwo, 2 Alpha,
  // 3 ExpThree), per-step constants (P/api/net/network/step.rs:206-298),
  // reversal potential; state [n_kin][3][Nd]
  int n_kin;
  int kin_kind[3];
  float kin_c[3][8];
  float kin_erev[3];
  float *kin_g;
  // receptor kinetics (SynapticBrain): ring slot 0 holds the step's external
  // input, slots 1..7 the conductances of receptors 0..6, never cleared and
  // decayed by rec_f each step; spikes jump them with no delay (an edge's
  // delay field is 1 + its receptor, and the ring base stays 0)
  int receptor;
  float rec_f[7];
  // CSR (device neuron indices), rows sorted by post; one 8-byte record per
  // synapse: x = post | code << 24 (packed) or post (code in `code`), y = weight
  const uint32_t *row_ptr;
  uint2 *edge;
  const uint8_t *code;  // null when packed
  // BF16 weight storage: the record's x word and the bf16 weight in two
  // arrays (6 B per synapse instead of 8); edge is null then
  int wbf16;
  const uint32_t *edge_x;
  const uint16_t *w16;
  // FP8 E4M3 weight storage: x words in edge_x, one E4M3 byte per synapse and
  // one FP32 scale per row (weight = e4m3 value * row scale, 5 B per synapse)
  int wfp8;
  const uint8_t *w8;
  const float *row_scale;
  uint32_t post_mask;
  uint32_t n_edges;
  // per-row segment table: [Nd][G+1] offsets inside the row (u16 or u32)
  const void *seg;
  int seg32;
  uint32_t G;      // scatter blocks
  uint32_t P;      // posts per scatter block (multiple of 32)
  uint32_t pbits;  // bits of a local post index
  // Poisson-source synapses of scatter block j: runs [run_lo[j], run_lo[j+1]);
  // entry t of a run is source run_src0 + t -> post run_post0 + t, seed
  // run_seed0 + t, with the run's rate, weight and code
  const uint32_t *run_lo;
  const uint32_t *run_src0;
  const uint32_t *run_post0;
  const uint32_t *run_len;
  const uint32_t *run_seed0;
  const float *run_w;
  const float *run_p;
  const uint8_t *run_code;
  // scatter mode
  int deterministic;
  // pre-centric scatter (networks whose ring sums are exact, and the atomic
  // mode): this step's spiking neurons in any order (red_flat, red_cnt
  // entries; the neuron kernel appends, the scatter's last block resets the
  // count), every event added to its ring cell in L2 with red.global.add
  int red;
  uint32_t *red_flat;
  uint32_t *red_cnt;
  uint2 *red_rows;   // [Nd] synapse range [x, y) of each red_flat entry's row
  // Poisson-source synapses of the pre-centric scatter: run r covers source
  // synapses [run_off[r], run_off[r + 1]) of the n_src_syn in runs
  const uint32_t *run_off;
  uint32_t n_runs;
  uint32_t n_src_syn;
  // Tsodyks-Markram on Poisson-source synapses: profile per run (0 none) and
  // per source synapse (index run_off[run] + offset) its R, U and last spike
  // step (P/api/net/network/step.rs:166-180)
  int src_tm;
  const uint8_t *run_pt;
  float *src_tm_r;
  float *src_tm_u;
  uint32_t *src_tm_last;
  // deferred drive: the step whose deferred Poisson events were already
  // added to the ring (by drive_fold_kernel before an inject or a ring
  // readback), or ~0
  const unsigned long long *drv_fold;
  // Tsodyks-Markram short-term plasticity: per-edge profile id (0 = none)
  // and state R, U, last spike step (CSR order), the profiles' constants
  int tm;
  const uint8_t *tm_pt;
  float *tm_r;
  float *tm_u;
  uint32_t *tm_last;
  float tm_u0[kMaxTm], tm_arec[kMaxTm], tm_afac[kMaxTm];
  uint32_t tm_fac;  // bit k: profile k + 1 facilitates
  // pair STDP
  int stdp;
  float *x_pre;
  float *x_post;
  float d_pre, d_post, a_plus, a_minus, w_min, w_max;
  const uint32_t *in_ptr;
  const uint32_t *in_edge;
  const uint32_t *in_pre;
  double *drift;
  // dopamine-modulated eligibility learning: per-neuron traces decayed by
  // fma with this step's spike, and spikes of two device index ranges
  // [l_motor[0], l_motor[1]) and [l_motor[2], l_motor[3]) counted
  int learn;
  float *l_tp, *l_tq;
  float l_dpre, l_dpost;
  uint32_t l_motor[4];
  uint32_t *l_motor_acc;
  uint32_t *l_flat, *l_flat_cnt;  // this step's spiking neurons, in any order
};

struct PopArgs {
  float *state;
  const float *params;
  uint32_t n, cap, dev_off;
  uint32_t umask;      // bit c: parameter column c is uniform
  float uval[16];      // its value
  float ln_na, ln_k;   // GPEA constants
  // Gaussian input current added to every neuron's synaptic input each step
  // (as an inject_current of that step would): sigma_i * N(0,1) from the
  // counter i + (step - noise_step0) * noise_stride of the noise stream, with
  // sigma_i = noise_sigma[0] for i < noise_split, noise_sigma[1] after
  int noise;
  uint32_t noise_stream, noise_split;
  unsigned long long noise_seed, noise_stride, noise_step0;
  double noise_sigma[2];
  // constant per-neuron input current added every step (as an
  // inject_current of the same values each step would), or null
  const float *bias;
  // deferred drive: neuron i has one Poisson source (seed drv_seed0 + i,
  // rate p = drv_p) with one synapse of weight drv_w and delay <= 1 onto it,
  // and no other source synapse.  Its event of step t arrives in slot t + 1
  // as the last add before that slot is read (later steps' events land in
  // later slots; an inject_current in between first folds it into the ring),
  // so the neuron kernel of step t + 1 rolls it and adds it to the slot
  // value it read: the same float sums as the ring, without the event.
  int drv;
  uint32_t drv_seed0;
  float drv_p, drv_w;
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// The ring slot a step reads (and the base its events count delays from):
// step % nslots, or 0 under receptor kinetics, whose slots are fixed
// (0 external input, 1 + r conductance of receptor r).
__device__ __forceinline__ uint32_t ring_base(const StepArgs &a, unsigned long long step) {
  return a.receptor ? 0u : (uint32_t)(step % a.nslots);
}

// The step hint: the word after the step counter.  The scatters store
// step + 1 there as soon as they have read the step (long before they
// finish), so that the next neuron kernel can roll its Poisson drive and
// find its ring slot before its dependency wait.  It is only a guess: the
// neuron kernel compares it with the step counter after the wait and redoes
// that work when they differ (a step run another way, a host-set step).
// The neuron kernel reads it while the scatter before it may still be
// running, so both sides use relaxed GPU-scope accesses.
__device__ __forceinline__ unsigned long long hint_load(const StepArgs &a) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(a.step + 1));
  return v;
}
__device__ __forceinline__ void hint_store(const StepArgs &a, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(a.step + 1), "l"(v) : "memory");
}

// The Poisson drive of NPT neurons from population index i0 for one step:
// bit q = source of neuron i0 + q fires (P/api/net/network/sources.rs:5-14 roll).
template <int NPT>
__device__ __forceinline__ uint32_t drive_bits(const PopArgs &p, uint32_t i0, unsigned long long step) {
  uint32_t b = 0;
#pragma unroll
  for (int q = 0; q < NPT; ++q)
    if (i0 + q < p.n && poisson_spike(p.drv_seed0 + i0 + q, 0, step, p.drv_p)) b |= 1u << q;
  return b;
}

// What the single-population neuron kernel works out before its wait from
// the step hint (valid for step `step` only).
struct PreWait {
  unsigned long long step;
  uint32_t slot;      // ring_base(step)
  uint32_t drv_prev;  // drive_bits(step - 1)
  uint32_t drv_now;   // drive_bits(step)
  bool ok;
};

// Programmatic dependent launch: the step kernels are launched so that the
// next kernel of the stream may start while this one drains.  pdl_wait()
// returns once the previous kernel of the stream has completed and its memory
// is visible (a no-op for a kernel launched without the attribute); every
// kernel calls it before it touches data an earlier kernel of the step wrote.
// pdl_release() lets the next kernel launch (its blocks then run up to their
// own pdl_wait()); the kernels call it when their main work is done, so that
// the next kernel's launch overlaps their tail.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// L2 cache policies: the CSR of the spiking rows streams through once per
// step (evict first); the delay ring is re-read every step (evict last) and
// has to stay resident in L2 for the scatter's random read-modify-writes.
__device__ __forceinline__ unsigned long long policy_evict_first() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ unsigned long long policy_evict_last() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint32_t ld_stream_u32(const uint32_t *p, unsigned long long pol) {
  uint32_t v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float ld_stream_f32(const float *p, unsigned long long pol) {
  float v;
  asm volatile("ld.global.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ uint32_t ld_stream_u8(const uint8_t *p, unsigned long long pol) {
  uint32_t v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u8 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ uint2 ld_stream_edge(const uint2 *p, unsigned long long pol) {
  uint2 v;
  asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;"
               : "=r"(v.x), "=r"(v.y)
               : "l"(p), "l"(pol));
  return v;
}
// Ring loads do not allocate in L1: a window issues kWin of them per SM at
// once and the ring is re-read only in later steps.
__device__ __forceinline__ uint32_t ld_stream_u16(const uint16_t *p, unsigned long long pol) {
  uint16_t v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u16 %0, [%1], %2;" : "=h"(v) : "l"(p), "l"(pol));
  return v;
}
// Asynchronous global -> shared copies (no registers held while in flight,
// so a thread can have all of its window's loads outstanding at once).
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem, unsigned long long pol) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 4, %2;" ::"r"(d), "l"(gmem), "l"(pol) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, unsigned long long pol) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(d), "l"(gmem), "l"(pol) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// E4M3 byte -> FP32 (exact).
__device__ __forceinline__ float e4m3_to_f32(uint32_t b) {
  __nv_fp8_e4m3 v;
  v.__x = (__nv_fp8_storage_t)b;
  return (float)v;
}

// One synapse record (x = post | code << 24, y = f32 weight bits); the bf16
// form widens the stored weight to f32 (its upper 16 bits), the fp8 form
// multiplies the E4M3 value by its row's scale.
__device__ __forceinline__ uint2 ld_record(const StepArgs &a, uint32_t e, unsigned long long pol,
                                           float scale = 1.0f) {
  if (a.wbf16) return make_uint2(ld_stream_u32(a.edge_x + e, pol), ld_stream_u16(a.w16 + e, pol) << 16);
  if (a.wfp8)
    return make_uint2(ld_stream_u32(a.edge_x + e, pol),
                      __float_as_uint(e4m3_to_f32(ld_stream_u8(a.w8 + e, pol)) * scale));
  return ld_stream_edge(a.edge + e, pol);
}
__device__ __forceinline__ float ld_ring(const float *p, unsigned long long pol) {
  float v;
  asm volatile("ld.global.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol) : "memory");
  return v;
}
__device__ __forceinline__ void st_ring(float *p, float v, unsigned long long pol) {
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(pol) : "memory");
}

// ---------------------------------------------------------------------------
// neuron phase
// ---------------------------------------------------------------------------
template <int NPT> struct VecF;
template <> struct VecF<1> {
  __device__ __forceinline__ static void load(const float *p, float *v) { v[0] = *p; }
  __device__ __forceinline__ static void ldg(const float *p, float *v) { v[0] = __ldg(p); }
  __device__ __forceinline__ static void store(float *p, const float *v) { *p = v[0]; }
};
template <> struct VecF<8> {
  __device__ __forceinline__ static void load(const float *p, float *v) {
    const float4 a = reinterpret_cast<const float4 *>(p)[0], b = reinterpret_cast<const float4 *>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
  }
  __device__ __forceinline__ static void ldg(const float *p, float *v) {
    const float4 a = __ldg(reinterpret_cast<const float4 *>(p)), b = __ldg(reinterpret_cast<const float4 *>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
  }
  __device__ __forceinline__ static void store(float *p, const float *v) {
    reinterpret_cast<float4 *>(p)[0] = make_float4(v[0], v[1], v[2], v[3]);
    reinterpret_cast<float4 *>(p)[1] = make_float4(v[4], v[5], v[6], v[7]);
  }
};
template <> struct VecF<4> {
  __device__ __forceinline__ static void load(const float *p, float *v) {
    const float4 t = *reinterpret_cast<const float4 *>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  }
  __device__ __forceinline__ static void ldg(const float *p, float *v) {
    const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  }
  __device__ __forceinline__ static void store(float *p, const float *v) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
  }
};

// The update of one 1024-neuron block `blk` of population p.
// FULL = false: the lean form for steps without kinetic synapses, input
// noise, neuron statistics, pair STDP or learning (fewer registers: all blocks
// of a large population resident at once).
// Loads the state of this thread's neurons of block `blk` of population p.
template <int MODEL, bool FULL>
__device__ __forceinline__ void load_state(const PopArgs &p, uint32_t blk,
                                           float (&sv)[n_state(MODEL)][NeuronCfg<MODEL, FULL>::NPT]) {
  constexpr int NPT = NeuronCfg<MODEL, FULL>::NPT;
  const uint32_t i0 = blk * kNeuronBlock + threadIdx.x * NPT;
#pragma unroll
  for (int c = 0; c < n_state(MODEL); ++c) VecF<NPT>::load(p.state + (size_t)c * p.cap + i0, sv[c]);
}

// sv: the state of this thread's neurons (load_state), updated in place and
// stored.
template <int MODEL, bool FULL>
__device__ __forceinline__ void neuron_block(const StepArgs &a, const PopArgs &p, uint32_t blk,
                                             float (&sv)[n_state(MODEL)][NeuronCfg<MODEL, FULL>::NPT],
                                             const PreWait &pre) {
  constexpr int NPT = NeuronCfg<MODEL, FULL>::NPT;
  constexpr int NS = n_state(MODEL), NP = n_params(MODEL);
  using V = VecF<NPT>;
  __shared__ uint32_t warp_cnt[32];
  __shared__ uint32_t warp_clamp[32];
  __shared__ uint32_t warp_fire[32];
  const uint32_t tid = threadIdx.x, lane = lane_id(), wid = tid >> 5;
  const uint32_t i0 = blk * kNeuronBlock + tid * NPT;  // population index of my first neuron
  const uint32_t gi0 = p.dev_off + i0;
  // 1-2. read the slot, clear it (step.rs:27-34).  With a step hint the
  // hinted slot (always a valid slot) is loaded beside the step counter and
  // loaded again from the right slot only when the hint was wrong.
  float x[NPT], zero[NPT];
#pragma unroll
  for (int q = 0; q < NPT; ++q) zero[q] = 0.0f;
  if (pre.ok) V::load(a.ring + (size_t)pre.slot * a.Nd + gi0, x);
  const unsigned long long step = *a.step;
  const bool hit = pre.ok && pre.step == step;  // the pre-wait work is this step's
  const uint32_t slot = hit ? pre.slot : ring_base(a, step);
  float *rs = a.ring + (size_t)slot * a.Nd + gi0;
  if (!hit) V::load(rs, x);
  V::store(rs, zero);
  uint32_t nfire = 0;  // this step's deferred-drive events (counted now, applied next step)
  if (p.drv) {
    const bool take = step >= 1 && *a.drv_fold != step - 1;
    const uint32_t prev = !take ? 0u : hit ? pre.drv_prev : drive_bits<NPT>(p, i0, step - 1);
#pragma unroll
    for (int q = 0; q < NPT; ++q)
      if ((prev >> q) & 1u) x[q] = x[q] + p.drv_w;
    nfire = __popc(hit ? pre.drv_now : drive_bits<NPT>(p, i0, step));
  }
  if (p.bias != nullptr) {
    float bv[NPT];
    V::ldg(p.bias + i0, bv);
#pragma unroll
    for (int q = 0; q < NPT; ++q) x[q] = x[q] + bv[q];
  }
  if (FULL && p.noise) {
    const unsigned long long t = step - p.noise_step0;
#pragma unroll
    for (int q = 0; q < NPT; ++q)
      if (i0 + q < p.n) {
        const uint32_t i = i0 + q;
        const double z = hash_std_normal(p.noise_seed, p.noise_stream, (unsigned long long)i + t * p.noise_stride);
        x[q] = x[q] + (float)((i < p.noise_split ? p.noise_sigma[0] : p.noise_sigma[1]) * z);
      }
  }
  // 2b. kinetic ExpOne rings (step.rs:56-70, :338-345); V from step start.
  // Unrolled over the (at most 3) profiles so that the profile constants are
  // indexed at compile time and stay in the kernel parameter space.
#pragma unroll
  for (int k = 0; k < (FULL ? 3 : 0); ++k) {
    if (k >= a.n_kin) break;
    float jump[NPT], s0[NPT], s1[NPT], s2[NPT];
    float *ks = a.ring + ((size_t)(k + 1) * a.nslots + slot) * a.Nd + gi0;
    V::load(ks, jump);
    V::store(ks, zero);
    const int kind = a.kin_kind[k];
    const float *c = a.kin_c[k];
    float *g0 = a.kin_g + ((size_t)k * 3 + 0) * a.Nd + gi0;
    float *g1 = a.kin_g + ((size_t)k * 3 + 1) * a.Nd + gi0;
    float *g2 = a.kin_g + ((size_t)k * 3 + 2) * a.Nd + gi0;
    V::load(g0, s0);
    if (kind != 0) V::load(g1, s1);
    if (kind == 3) V::load(g2, s2);
#pragma unroll
    for (int q = 0; q < NPT; ++q) {  // step.rs:336-398
      const float j = jump[q], dv = a.kin_erev[k] - sv[0][q];
      if (kind == 0) {  // ExpOne: g
        s0[q] = s0[q] * c[0] + j;
        x[q] += s0[q] * dv;
      } else if (kind == 1) {  // ExpTwo: g (decay), x (rise)
        s0[q] = s0[q] * c[1] + j;
        s1[q] = s1[q] * c[0] + j;
        x[q] += c[2] * (s0[q] - s1[q]) * dv;
      } else if (kind == 2) {  // Alpha: g, a
        const float a_old = s1[q];
        s1[q] = a_old * c[0] + j;
        s0[q] = s0[q] * c[0] + c[1] * a_old;
        x[q] += s0[q] * dv;
      } else {  // ExpThree: a (rise), b, c (decays)
        s0[q] = s0[q] * c[0] + j * c[5];
        s1[q] = s1[q] * c[1] + j * c[3];
        s2[q] = s2[q] * c[2] + j * c[4];
        x[q] += (c[6] * (s1[q] - s0[q]) + c[7] * (s2[q] - s0[q])) * dv;
      }
    }
    V::store(g0, s0);
    if (kind != 0) V::store(g1, s1);
    if (kind == 3) V::store(g2, s2);
  }
  // 2c. receptor kinetics (SynapticBrain::step, pillars-connectome/src/
  // synaptic.rs:94-112): decay each conductance (P/kernels/synapse/
  // kinetics.rs:112-147), I_syn = sum over receptors in code order of
  // g_eff (E_rev - V) from zero with NMDA's g scaled by the Mg block of the
  // pre-step V (:159-206), input = I_syn + the external input.
  if (FULL && a.receptor) {
    float cur[NPT], mg[NPT];
#pragma unroll
    for (int q = 0; q < NPT; ++q) {
      cur[q] = 0.0f;
      mg[q] = nmda_mg_block(sv[0][q]);
    }
#pragma unroll
    for (int r = 0; r < kReceptors; ++r) {
      float g[NPT];
      float *gp = a.ring + (size_t)(1 + r) * a.Nd + gi0;
      V::load(gp, g);
#pragma unroll
      for (int q = 0; q < NPT; ++q) {
        g[q] = g[q] * a.rec_f[r];
        const float ge = r == 1 ? g[q] * mg[q] : g[q];
        cur[q] = cur[q] + ge * (rec_erev(r) - sv[0][q]);
      }
      V::store(gp, g);
    }
#pragma unroll
    for (int q = 0; q < NPT; ++q) x[q] = cur[q] + x[q];
  }
  // per-neuron parameters: loaded for the block's NPT neurons at once, or
  // (8 neurons per thread) one neuron at a time in the update loop, which
  // keeps the register count down
  constexpr bool kParamsPerNeuron = NPT == 8;
  float pv[kParamsPerNeuron ? 1 : NP][kParamsPerNeuron ? 1 : NPT];
  if (!kParamsPerNeuron) {
#pragma unroll
    for (int c = 0; c < NP; ++c) {
      if ((p.umask >> c) & 1u) {
#pragma unroll
        for (int q = 0; q < NPT; ++q) pv[c][q] = p.uval[c];
      } else {
        V::ldg(p.params + (size_t)c * p.cap + i0, pv[c]);
      }
    }
  }
  // dt = param column 0 of neuron 0, broadcast (population.rs:307,361)
  const float dt = (p.umask & 1u) ? p.uval[0] : __ldg(p.params);
  uint32_t nib = 0, nclamp = 0;
  // UNI: every parameter column is population-wide and all NPT neurons of
  // the thread exist (the common case of a large homogeneous population):
  // parameters straight from the kernel arguments, no per-neuron guards
  auto update = [&](auto uni) {
    constexpr bool UNI = decltype(uni)::value;
#pragma unroll
    for (int q = 0; q < NPT; ++q) {
      if (UNI || i0 + q < p.n) {
        float xi = x[q];
        if (clamps(MODEL)) {
          const float xc = fminf(fmaxf(xi, -100.0f), 100.0f);
          nclamp += xc != xi;
          xi = xc;
        }
        RegNeuron<NS, NP> r;
#pragma unroll
        for (int c = 0; c < NS; ++c) r.s[c] = sv[c][q];
#pragma unroll
        for (int c = 0; c < NP; ++c)
          r.p[c] = UNI ? p.uval[c]
                   : !kParamsPerNeuron ? pv[kParamsPerNeuron ? 0 : c][kParamsPerNeuron ? 0 : q]
                   : (p.umask >> c) & 1u ? p.uval[c]
                                         : __ldg(p.params + (size_t)c * p.cap + i0 + q);
        bool sp;
        if (MODEL == kLIF) sp = lif_step(r, xi, dt);
        else if (MODEL == kIZH) sp = izh_step(r, xi, dt);
        else if (MODEL == kGPEA) sp = gpea_step(r, xi, dt, p.ln_na, p.ln_k);
        else sp = hh_step(r, xi, dt);
#pragma unroll
        for (int c = 0; c < NS; ++c) sv[c][q] = r.s[c];
        nib |= (sp ? 1u : 0u) << q;
      }
    }
  };
  constexpr uint32_t kAllParams = (1u << NP) - 1u;
  if (kParamsPerNeuron && (p.umask & kAllParams) == kAllParams && i0 + NPT <= p.n) update(BoolC<true>{});
  else update(BoolC<false>{});
#pragma unroll
  for (int c = 0; c < NS; ++c) V::store(p.state + (size_t)c * p.cap + i0, sv[c]);
  if (FULL && a.ns_count != nullptr && nib) {
    const uint32_t t = (uint32_t)(step - a.ns_step0);
#pragma unroll
    for (int q = 0; q < NPT; ++q)
      if (nib & (1u << q)) {
        const uint32_t gi = gi0 + q;
        const uint32_t last = a.ns_last[gi];
        if (last != 0xFFFFFFFFu) {
          const double isi = (double)(t - last);
          a.ns_s1[gi] += isi;
          a.ns_s2[gi] += isi * isi;
        }
        a.ns_last[gi] = t;
        a.ns_count[gi] += 1u;
      }
  }
  // 4. compaction: bitmask words (32 neurons each) and the block's spike list
  uint32_t word;
  if (NPT == 8) {
    word = nib << (8 * (lane & 3));
    word |= __shfl_xor_sync(0xffffffffu, word, 1);
    word |= __shfl_xor_sync(0xffffffffu, word, 2);
    if ((lane & 3) == 0) {
      a.last_bits[gi0 >> 5] = word;
      if (a.raster != nullptr) a.raster[(size_t)(step % a.raster_cap) * a.words + (gi0 >> 5)] = word;
    }
  } else if (NPT == 4) {
    word = nib << (4 * (lane & 7));
    word |= __shfl_xor_sync(0xffffffffu, word, 1);
    word |= __shfl_xor_sync(0xffffffffu, word, 2);
    word |= __shfl_xor_sync(0xffffffffu, word, 4);
    if ((lane & 7) == 0) {
      a.last_bits[gi0 >> 5] = word;
      if (a.raster != nullptr) a.raster[(size_t)(step % a.raster_cap) * a.words + (gi0 >> 5)] = word;
    }
  } else {
    word = __ballot_sync(0xffffffffu, nib != 0);
    if (lane == 0) {
      a.last_bits[gi0 >> 5] = word;
      if (a.raster != nullptr) a.raster[(size_t)(step % a.raster_cap) * a.words + (gi0 >> 5)] = word;
    }
  }
  const uint32_t cnt = __popc(nib);
  // the synapse range of this thread's first spiking neuron, loaded now so
  // that its latency runs under the block's count exchange (pre-centric path)
  uint2 rows0 = make_uint2(0u, 0u);
  if (a.red && nib) {
    const uint32_t q0 = (uint32_t)__ffs(nib) - 1u;
    rows0 = make_uint2(__ldg(a.row_ptr + gi0 + q0), __ldg(a.row_ptr + gi0 + q0 + 1));
  }
  uint32_t incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (uint32_t)o) incl += y;
  }
  uint32_t clw = nclamp, fw = nfire;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    clw += __shfl_xor_sync(0xffffffffu, clw, o);
    fw += __shfl_xor_sync(0xffffffffu, fw, o);
  }
  if (lane == 31) warp_cnt[wid] = incl;
  if (lane == 0) {
    warp_clamp[wid] = clw;
    warp_fire[wid] = fw;
  }
  __syncthreads();
  constexpr uint32_t NW = NeuronCfg<MODEL, FULL>::THREADS / 32;
  uint32_t before = incl - cnt, total = 0, clamp_tot = 0, fire_tot = 0;
#pragma unroll
  for (uint32_t k = 0; k < NW; ++k) {
    const uint32_t c = warp_cnt[k];
    before += k < wid ? c : 0u;
    total += c;
    clamp_tot += warp_clamp[k];
    fire_tot += warp_fire[k];
  }
  const uint32_t gblk = gi0 / kNeuronBlock;
  if (a.red) {
    // pre-centric scatter: the block's spiking neurons at one place of the flat list
    __shared__ uint32_t red_base;
    if (tid == 0) red_base = total ? atomicAdd(a.red_cnt, total) : 0u;
    __syncthreads();
    uint32_t pos = red_base + before;
    bool first = true;
#pragma unroll
    for (int q = 0; q < NPT; ++q)
      if (nib & (1u << q)) {  // the spiking neuron and its synapse range
        a.red_flat[pos] = gi0 + q;
        a.red_rows[pos] = first ? rows0 : make_uint2(__ldg(a.row_ptr + gi0 + q), __ldg(a.row_ptr + gi0 + q + 1));
        first = false;
        ++pos;
      }
  } else {
    uint2 *out = a.spk + (size_t)gblk * kNeuronBlock + before;
#pragma unroll
    for (int q = 0; q < NPT; ++q)
      if (nib & (1u << q)) *out++ = make_uint2(gi0 + q, __ldg(a.row_ptr + gi0 + q));
  }
  if (tid == 0) {
    if (!a.red) a.blk_cnt[gblk] = total;
    if (a.clamp_hits != nullptr && clamp_tot) atomicAdd(a.clamp_hits, (unsigned long long)clamp_tot);
    if (fire_tot) {
      atomicAdd(a.ev_step, (unsigned long long)fire_tot);
      atomicAdd(a.ev_src_step, (unsigned long long)fire_tot);
    }
  }
  // pair-STDP traces: x = fma(x, d, s) (P/api/learn/brain.rs:212-222)
  if (FULL && a.stdp) {
#pragma unroll
    for (int q = 0; q < NPT; ++q)
      if (i0 + q < p.n) {
        const uint32_t gi = gi0 + q;
        const float add = (nib >> q) & 1u ? 1.0f : 0.0f;
        a.x_pre[gi] = __fmaf_rn(a.x_pre[gi], a.d_pre, add);
        a.x_post[gi] = __fmaf_rn(a.x_post[gi], a.d_post, add);
      }
  }
  // learning traces (P/api/learn/brain.rs:211-222) and motor counts
  // (pillars-wgpu/shaders/dopamine.wgsl:126-136)
  if (FULL && a.learn) {
    uint32_t m0 = 0, m1 = 0;
#pragma unroll
    for (int q = 0; q < NPT; ++q)
      if (i0 + q < p.n) {
        const uint32_t gi = gi0 + q;
        const bool fired = (nib >> q) & 1u;
        const float add = fired ? 1.0f : 0.0f;
        a.l_tp[gi] = __fmaf_rn(a.l_tp[gi], a.l_dpre, add);
        a.l_tq[gi] = __fmaf_rn(a.l_tq[gi], a.l_dpost, add);
        m0 += fired && gi >= a.l_motor[0] && gi < a.l_motor[1] ? 1u : 0u;
        m1 += fired && gi >= a.l_motor[2] && gi < a.l_motor[3] ? 1u : 0u;
      }
    if (m0) atomicAdd(a.l_motor_acc, m0);
    if (m1) atomicAdd(a.l_motor_acc + 1, m1);
    __shared__ uint32_t flat_base;
    if (tid == 0) flat_base = total ? atomicAdd(a.l_flat_cnt, total) : 0u;
    __syncthreads();
    uint32_t pos = flat_base + before;
#pragma unroll
    for (int q = 0; q < NPT; ++q)
      if (nib & (1u << q)) a.l_flat[pos++] = gi0 + q;
  }
}

// One launch per neuron model updates every population of that model: block
// b takes entry map[b] = (population, block within it) of the work table, so
// many small populations (a batch of networks) step in one launch.  A model
// with a single population passes its arguments by value (map == null) and
// block b is its block b.
template <int MODEL, bool FULL>
__global__ void __launch_bounds__(NeuronCfg<MODEL, FULL>::THREADS, NeuronCfg<MODEL, FULL>::MIN_BLOCKS)
    neuron_kernel(StepArgs a, PopArgs p0, const PopArgs *__restrict__ pops, const uint2 *__restrict__ map) {
  float sv[n_state(MODEL)][NeuronCfg<MODEL, FULL>::NPT];
  if (map == nullptr) {
    // Population state is written only by the neuron update, and the last
    // one finished before the previous scatter passed its own wait (which
    // is what let this kernel start): the state is read before the wait,
    // so that its loads overlap the previous kernel's tail.
    load_state<MODEL, FULL>(p0, blockIdx.x, sv);
    // this step's drive rolls and ring slot from the step hint (checked
    // against the step counter after the wait)
    PreWait pre;
    pre.step = hint_load(a);
    pre.slot = ring_base(a, pre.step);
    pre.ok = true;
    pre.drv_prev = pre.drv_now = 0u;
    if (p0.drv) {
      constexpr int NPT = NeuronCfg<MODEL, FULL>::NPT;
      const uint32_t i0 = blockIdx.x * kNeuronBlock + threadIdx.x * NPT;
      pre.drv_prev = pre.step >= 1 ? drive_bits<NPT>(p0, i0, pre.step - 1) : 0u;
      pre.drv_now = drive_bits<NPT>(p0, i0, pre.step);
    }
    pdl_wait();
    neuron_block<MODEL, FULL>(a, p0, blockIdx.x, sv, pre);
  } else {
    pdl_wait();
    const uint2 bm = map[blockIdx.x];
    load_state<MODEL, FULL>(pops[bm.x], bm.y, sv);
    PreWait none;
    none.ok = false;
    neuron_block<MODEL, FULL>(a, pops[bm.x], bm.y, sv, none);
  }
  pdl_release();
}

// ---------------------------------------------------------------------------
// block-wide helpers (kScatterThreads threads)
// ---------------------------------------------------------------------------
// Exclusive scan of one value per thread; returns the prefix, *total = sum.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *wsum, uint32_t *total) {
  const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  __syncthreads();  // wsum reuse
  if (lane == 31) wsum[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint32_t t = lane < (blockDim.x >> 5) ? wsum[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= (uint32_t)o) t += y;
    }
    wsum[lane] = t;  // inclusive per warp
  }
  __syncthreads();
  *total = wsum[31];
  return (x - v) + (wid ? wsum[wid - 1] : 0u);
}

// largest i in [0, n) with pre[i] <= v (pre ascending, pre[0] = 0)
__device__ __forceinline__ uint32_t upper_index(const uint32_t *pre, uint32_t n, uint32_t v) {
  uint32_t lo = 0, hi = n - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= v) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

struct WinSmem {                  // one window of events
  uint32_t head[kBuckets];        // latest-linked event of each bucket; spike rows
                                  //   while a sub-chunk's segments are fetched
  uint32_t ecell[kWin];           // window events in reference order: cell, or the
                                  //   edge id before the records are read
  float ew[kWin];                 //   weight,
  uint16_t enext[kWin];           //   next event of the same bucket
};
struct ScatterSmem {
  WinSmem w;
  uint32_t plo[kPreChunk];        // absolute first edge of each row segment
  float pscale[kPreChunk];        // FP8 weights: the row's scale
  uint32_t pseg[kPreChunk + 1];   // prefix of segment lengths
  uint32_t boff[kBlkChunk + 1];   // prefix of spike-list slot counts
  uint32_t wsum[32];
  double drift;
  unsigned long long events;
  unsigned long long src_events;
};
static_assert(sizeof(ScatterSmem) <= 232448, "scatter shared memory exceeds 227 KB");

constexpr uint32_t kEPT = kWin / kScatterThreads;         // window events per thread (8)
constexpr uint32_t kBPT = kBuckets / kScatterThreads;     // buckets per thread (8)
constexpr uint32_t kPPT = kPreChunk / kScatterThreads;    // spiking rows per thread (4)

__device__ __forceinline__ float *cell_addr(const StepArgs &a, uint32_t cell, uint32_t p0) {
  return a.ring + (size_t)(cell >> a.pbits) * a.Nd + p0 + (cell & ((1u << a.pbits) - 1u));
}

__device__ __forceinline__ void clear_heads(ScatterSmem &S) {
#pragma unroll
  for (uint32_t r = 0; r < kBPT; ++r) S.w.head[threadIdx.x + r * kScatterThreads] = kEmpty;
}

// Knuth's multiplicative hash of the cell onto the buckets
__device__ __forceinline__ uint32_t bucket_of(uint32_t cell) { return (cell * 2654435761u) >> (32 - kBucketBits); }
constexpr uint32_t kNone16 = 0xFFFFu;

// Prepend event k to the list of its bucket (list order is arbitrary; the
// walk below compares event indices).
__device__ __forceinline__ void link_event(ScatterSmem &S, uint32_t k) {
  const uint32_t prev = atomicExch(&S.w.head[bucket_of(S.w.ecell[k])], k);
  S.w.enext[k] = (uint16_t)(prev == kEmpty ? kNone16 : prev);
}

// Apply the window's m linked events to the ring in reference order.  Each
// event finds, in its bucket's list, its rank among the earlier events of
// the same cell, its predecessor, and whether a later one exists.  `pre`
// holds the ring value of each of this thread's events (k = tid + r*threads),
// loaded before linking so that the loads overlap the linking barrier and
// the walk; rank-0 events add their weight to it, partial sums then advance
// one rank per level in shared memory (ew[k] becomes the cell's running value
// after event k; the values loaded for later ranks are not used), and the
// last event of each cell stores it.  Called by all threads after the
// linking barrier; ends with a barrier.
__device__ __forceinline__ void apply_window(const StepArgs &a, ScatterSmem &S, uint32_t m, uint32_t p0,
                                             const float (&pre)[kEPT]) {
  const unsigned long long pol = policy_evict_last();
  uint32_t rk[kEPT], pv[kEPT], lastm = 0, maxrank = 0;
  float w[kEPT];
#pragma unroll
  for (uint32_t r = 0; r < kEPT; ++r) {
    const uint32_t k = threadIdx.x + r * kScatterThreads;
    rk[r] = 0;
    pv[r] = kNone16;
    w[r] = 0.0f;
    if (k < m) {
      const uint32_t c = S.w.ecell[k];
      bool last = true;
      uint32_t j = S.w.head[bucket_of(c)];
      if (j == kEmpty) j = kNone16;
      for (; j != kNone16; j = S.w.enext[j]) {
        if (j == k || S.w.ecell[j] != c) continue;
        if (j < k) {
          ++rk[r];
          if (pv[r] == kNone16 || j > pv[r]) pv[r] = j;
        } else {
          last = false;
        }
      }
      lastm |= (last ? 1u : 0u) << r;
      maxrank = max(maxrank, rk[r]);
      w[r] = S.w.ew[k];
    }
  }
  // level 0: the first event of each cell adds to the loaded ring value
  float v[kEPT];
#pragma unroll
  for (uint32_t r = 0; r < kEPT; ++r) v[r] = pre[r];
#pragma unroll
  for (uint32_t r = 0; r < kEPT; ++r) {
    const uint32_t k = threadIdx.x + r * kScatterThreads;
    if (k < m && rk[r] == 0) {
      v[r] = v[r] + w[r];
      S.w.ew[k] = v[r];
    }
  }
  // later ranks: partial sums in order, one level per round
  for (uint32_t lvl = 1; __syncthreads_or(maxrank >= lvl); ++lvl) {
#pragma unroll
    for (uint32_t r = 0; r < kEPT; ++r) {
      const uint32_t k = threadIdx.x + r * kScatterThreads;
      if (k < m && rk[r] == lvl) {
        v[r] = S.w.ew[pv[r]] + w[r];
        S.w.ew[k] = v[r];
      }
    }
  }
  // the last event of each cell stores the cell's value
#pragma unroll
  for (uint32_t r = 0; r < kEPT; ++r) {
    const uint32_t k = threadIdx.x + r * kScatterThreads;
    if (k < m && (lastm & (1u << r))) st_ring(cell_addr(a, S.w.ecell[k], p0), v[r], pol);
  }
  __syncthreads();
}

// One event into the window.  `base` = step % nslots; the event lands in
// slot (step + max(delay, 1)) % nslots.
__device__ __forceinline__ uint32_t put_event(const StepArgs &a, ScatterSmem &S, uint32_t k, uint32_t post,
                                              float w, uint8_t code, uint32_t base, uint32_t p0) {
  uint32_t slot = base + max(code_delay(code), 1u);
  if (slot >= a.nslots) slot -= a.nslots;
  const uint32_t key = code_ring(code) * a.nslots + slot;
  const uint32_t cell = (key << a.pbits) | (post - p0);
  S.w.ecell[k] = cell;
  S.w.ew[k] = w;
  return cell;
}

// The last block of a step's scatter: per-step statistics, event totals,
// the step counter (and the pre-centric scatter's spike count).
// Every counter is loaded before anything is stored, so that the loads are
// in flight together (this runs once per step, at the end of the scatter,
// on the step's critical path).
__device__ __forceinline__ void end_of_step_last(const StepArgs &a, uint32_t n_spikes) {
  const unsigned long long step = *(volatile unsigned long long *)a.step;
  const unsigned long long ev = *(volatile unsigned long long *)a.ev_step;
  const unsigned long long ev_src = *(volatile unsigned long long *)a.ev_src_step;
  const unsigned long long tot = *(volatile unsigned long long *)a.ev_total;
  const unsigned long long tot_src = *(volatile unsigned long long *)a.ev_src_total;
  if (a.stat_cap) {
    a.stat_spk[step % a.stat_cap] = n_spikes;
    a.stat_ev[step % a.stat_cap] = ev;
  }
  *a.ev_total = tot + ev;
  *a.ev_step = 0;
  *a.ev_src_total = tot_src + ev_src;
  *a.ev_src_step = 0;
  if (a.red) *a.red_cnt = 0;  // the next step's neuron kernel appends from 0
  *a.step = step + 1;
}

__device__ __forceinline__ void end_of_step(const StepArgs &a, uint32_t n_spikes) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const uint32_t t = atomicAdd(a.done, 1u);
    if (t == gridDim.x - 1) {
      __threadfence();
      end_of_step_last(a, n_spikes);
      *a.done = 0;
      __threadfence();
    }
  }
}

template <bool SEG32>
__global__ void __launch_bounds__(kScatterThreads, kScatterBlocksPerSM) scatter_kernel(StepArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ScatterSmem &S = *reinterpret_cast<ScatterSmem *>(smem_raw);
  const uint32_t tid = threadIdx.x;
  const uint32_t j = blockIdx.x;
  const uint32_t p0 = j * a.P;
  pdl_wait();
  const unsigned long long step = *a.step;
  if (j == 0 && tid == 0) hint_store(a, step + 1);  // for the next neuron kernel's pre-wait work
  const uint32_t base = ring_base(a, step);
  const uint32_t G1 = a.G + 1;
  const uint32_t pj = min(a.P, a.Nd - p0);
  if (tid == 0) {
    S.drift = 0.0;
    S.events = 0;
    S.src_events = 0;
  }
  __syncthreads();
  uint32_t n_spikes = 0;
  double drift = 0.0;  // this thread's part of the step's STDP weight change
  // ---- neuron events, in spiking-neuron order ----
  for (uint32_t cb0 = 0; cb0 < a.n_blk; cb0 += kBlkChunk) {
    const uint32_t c = (cb0 + tid < a.n_blk) ? a.blk_cnt[cb0 + tid] : 0u;
    uint32_t spikes;
    const uint32_t ex = block_excl_scan(c, S.wsum, &spikes);
    S.boff[tid] = ex;
    if (tid == 0) S.boff[kBlkChunk] = spikes;
    n_spikes += spikes;
    __syncthreads();
    for (uint32_t s0 = 0; s0 < spikes; s0 += kPreChunk) {
      const uint32_t pc = min(kPreChunk, spikes - s0);
      // rows tid*kPPT .. +kPPT of this sub-chunk: their spike-list entries,
      // then the bounds of each row's segment for this block, fetched with
      // asynchronous copies into the (idle) window area
      uint2 *srow = reinterpret_cast<uint2 *>(S.w.head);  // [kPreChunk] (pre, row start)
      uint32_t *sseg = S.w.ecell;                         // [kPreChunk][2] words holding lo, hi
      uint32_t len[kPPT], mylen = 0;
#pragma unroll
      for (uint32_t q = 0; q < kPPT; ++q) {
        const uint32_t i = tid * kPPT + q;
        if (i < pc) {
          const uint32_t r = s0 + i;
          const uint32_t b = upper_index(S.boff, kBlkChunk, r);
          cp_async8(&srow[i], a.spk + (size_t)(cb0 + b) * kNeuronBlock + (r - S.boff[b]));
        }
      }
      cp_async_wait_all();
#pragma unroll
      for (uint32_t q = 0; q < kPPT; ++q) {
        const uint32_t i = tid * kPPT + q;
        if (i < pc) {
          const size_t idx = (size_t)srow[i].x * G1 + j;
          const uint32_t *words = (const uint32_t *)a.seg;
          if (SEG32) {
            cp_async4(&sseg[2 * i], words + idx);
            cp_async4(&sseg[2 * i + 1], words + idx + 1);
          } else {  // u16 entries idx, idx + 1 from the 32-bit words holding them
            cp_async4(&sseg[2 * i], words + (idx >> 1));
            cp_async4(&sseg[2 * i + 1], words + ((idx + 1) >> 1));
          }
        }
      }
      cp_async_wait_all();
#pragma unroll
      for (uint32_t q = 0; q < kPPT; ++q) {
        const uint32_t i = tid * kPPT + q;
        len[q] = 0;
        if (i < pc) {
          const uint2 e = srow[i];
          const size_t idx = (size_t)e.x * G1 + j;
          uint32_t lo, hi;
          if (SEG32) {
            lo = sseg[2 * i];
            hi = sseg[2 * i + 1];
          } else {
            lo = (sseg[2 * i] >> ((uint32_t)(idx & 1) * 16)) & 0xFFFFu;
            hi = (sseg[2 * i + 1] >> ((uint32_t)((idx + 1) & 1) * 16)) & 0xFFFFu;
          }
          S.plo[i] = e.y + lo;
          if (a.wfp8) S.pscale[i] = __ldg(a.row_scale + e.x);
          len[q] = hi - lo;
          mylen += len[q];
        }
      }
      uint32_t M;
      uint32_t ex2 = block_excl_scan(mylen, S.wsum, &M);
#pragma unroll
      for (uint32_t q = 0; q < kPPT; ++q) {
        S.pseg[tid * kPPT + q] = ex2;
        ex2 += len[q];
      }
      if (tid == 0) {
        S.pseg[kPreChunk] = M;
        S.events += M;
      }
      __syncthreads();
      for (uint32_t w0 = 0; w0 < M; w0 += kWin) {
        const uint32_t m = min(kWin, M - w0);
        clear_heads(S);
        // each spiking row writes the edge ids of its window events (rows are
        // short segments); then thread tid takes events k = tid + r*kScatterThreads
        uint32_t *eid = S.w.ecell;
#pragma unroll
        for (uint32_t q = 0; q < kPPT; ++q) {
          const uint32_t i = tid * kPPT + q;
          if (i < pc) {
            const uint32_t g0 = max(S.pseg[i], w0), g1 = min(S.pseg[i + 1], w0 + m);
            const uint32_t d = S.plo[i] - S.pseg[i];
            for (uint32_t g = g0; g < g1; ++g) eid[g - w0] = d + g;
            if (a.wfp8)  // the row's scale beside each event until the records are read
              for (uint32_t g = g0; g < g1; ++g) S.w.ew[g - w0] = S.pscale[i];
          }
        }
        __syncthreads();
        const unsigned long long spol = policy_evict_first();
        {
        uint32_t ev_e[kEPT];
#pragma unroll
        for (uint32_t r = 0; r < kEPT; ++r) {
          const uint32_t k = tid + r * kScatterThreads;
          ev_e[r] = k < m ? S.w.ecell[k] : 0u;
        }
        uint32_t ev_post[kEPT];
        float ev_w[kEPT];
        uint8_t ev_code[kEPT];
#pragma unroll
        for (uint32_t r = 0; r < kEPT; ++r) {
          const uint32_t k = tid + r * kScatterThreads;
          if (k < m) {
            const uint2 rec = ld_record(a, ev_e[r], spol, a.wfp8 ? S.w.ew[k] : 1.0f);
            ev_post[r] = rec.x & a.post_mask;
            ev_w[r] = __uint_as_float(rec.y);
            ev_code[r] = a.code ? (uint8_t)ld_stream_u8(a.code + ev_e[r], spol) : (uint8_t)(rec.x >> 24);
          }
        }
        // short-term plasticity: the delivered weight is w * R * U (each
        // edge belongs to one post and so to this block alone)
        float ev_wd[kEPT];
#pragma unroll
        for (uint32_t r = 0; r < kEPT; ++r) {
          const uint32_t k = tid + r * kScatterThreads;
          ev_wd[r] = ev_w[r];
          if (a.tm && k < m) {
            const uint32_t e = ev_e[r], pt = a.tm_pt[e];
            if (pt) {
              const uint32_t q = pt - 1;
              ev_wd[r] = tm_spike(a.tm_u0[q], a.tm_arec[q], a.tm_afac[q], (a.tm_fac >> q) & 1u, a.tm_r[e],
                                  a.tm_u[e], a.tm_last[e], ev_w[r], step);
            }
          }
        }
        float pre[kEPT];
#pragma unroll
        for (uint32_t r = 0; r < kEPT; ++r) {
          const uint32_t k = tid + r * kScatterThreads;
          pre[r] = 0.0f;
          if (k < m) {
            const uint32_t cell = put_event(a, S, k, ev_post[r], ev_wd[r], ev_code[r], base, p0);
            pre[r] = ld_ring(cell_addr(a, cell, p0), policy_evict_last());
            if (a.stdp && code_stdp(ev_code[r])) {
              // depression at a pre spike; the pushed weight is the pre-update one
              const float w1 = fminf(fmaxf(ev_w[r] - a.a_minus * a.x_post[ev_post[r]], a.w_min), a.w_max);
              a.edge[ev_e[r]].y = __float_as_uint(w1);
              drift += (double)w1 - (double)ev_w[r];
            }
            link_event(S, k);
          }
        }
        __syncthreads();
        apply_window(a, S, m, p0, pre);
        }
      }
    }
  }
  // ---- Poisson sources targeting this block's posts, in source order ----
  const uint32_t rl0 = a.run_lo[j], rl1 = a.run_lo[j + 1];
  for (uint32_t rc0 = rl0; rc0 < rl1; rc0 += kPreChunk) {
    const uint32_t rc = min(kPreChunk, rl1 - rc0);
    // runs tid*kPPT .. +kPPT of this chunk
    uint32_t len[kPPT], mylen = 0;
#pragma unroll
    for (uint32_t q = 0; q < kPPT; ++q) {
      const uint32_t i = tid * kPPT + q;
      len[q] = i < rc ? a.run_len[rc0 + i] : 0u;
      mylen += len[q];
    }
    uint32_t T;
    uint32_t ex = block_excl_scan(mylen, S.wsum, &T);
#pragma unroll
    for (uint32_t q = 0; q < kPPT; ++q) {
      S.pseg[tid * kPPT + q] = ex;
      ex += len[q];
    }
    if (tid == 0) S.pseg[kPreChunk] = T;
    __syncthreads();
    for (uint32_t w0 = 0; w0 < T; w0 += kWin) {
      const uint32_t mt = min(kWin, T - w0);
      clear_heads(S);
      __syncthreads();
      // thread tid owns entries [tid*kEPT, +kEPT) of the window: roll them,
      // then an order-preserving compaction of the fired ones
      uint32_t fired = 0, e_post[kEPT];
      float e_w[kEPT];
      uint8_t e_code[kEPT];
      // runs are few and long: find the run of the first entry by search,
      // then walk forward, reading a run's parameters once
      uint32_t ri = kEmpty, i = 0, post0 = 0, seed0 = 0, roff = 0;
      float p = 0.0f, rw = 0.0f;
      uint8_t rcode = 0, rpt = 0;
      if (tid * kEPT < mt) i = upper_index(S.pseg, rc, w0 + tid * kEPT);
#pragma unroll
      for (uint32_t r = 0; r < kEPT; ++r) {
        const uint32_t k = tid * kEPT + r;
        if (k < mt) {
          const uint32_t g = w0 + k;
          while (g >= S.pseg[i + 1]) ++i;
          if (rc0 + i != ri) {
            ri = rc0 + i;
            p = __ldg(a.run_p + ri);
            post0 = __ldg(a.run_post0 + ri);
            seed0 = __ldg(a.run_seed0 + ri);
            rw = __ldg(a.run_w + ri);
            rcode = __ldg(a.run_code + ri);
            if (a.src_tm) {
              rpt = __ldg(a.run_pt + ri);
              roff = __ldg(a.run_off + ri);
            }
          }
          const uint32_t t = g - S.pseg[i];
          e_post[r] = post0 + t;
          e_w[r] = rw;
          e_code[r] = rcode;
          if (p > 0.0f && poisson_spike(seed0 + t, 0, step, p)) {
            fired |= 1u << r;
            if (rpt) {  // the synapse's short-term plasticity scales the delivered weight
              const uint32_t q = rpt - 1u, e = roff + t;  // each source synapse belongs to one block
              e_w[r] = tm_spike(a.tm_u0[q], a.tm_arec[q], a.tm_afac[q], (a.tm_fac >> q) & 1u, a.src_tm_r[e],
                                a.src_tm_u[e], a.src_tm_last[e], rw, step);
            }
          }
        }
      }
      uint32_t m;
      uint32_t pos = block_excl_scan(__popc(fired), S.wsum, &m);  // all reads of the window are done
#pragma unroll
      for (uint32_t r = 0; r < kEPT; ++r)
        if (fired & (1u << r)) put_event(a, S, pos++, e_post[r], e_w[r], e_code[r], base, p0);
      if (tid == 0) {
        S.events += m;
        S.src_events += m;
      }
      __syncthreads();
      if (m) {
        float pre[kEPT];
#pragma unroll
        for (uint32_t r = 0; r < kEPT; ++r) {
          const uint32_t k = tid + r * kScatterThreads;
          pre[r] = 0.0f;
          if (k < m) {
            pre[r] = ld_ring(cell_addr(a, S.w.ecell[k], p0), policy_evict_last());
            link_event(S, k);
          }
        }
        __syncthreads();
        apply_window(a, S, m, p0, pre);
      }
    }
    __syncthreads();
  }
  // ---- pair-STDP potentiation on the plastic in-edges of spiking posts ----
  // warp w takes the spiking posts of the block's words w, w + 32, ...; its
  // lanes share each post's in-edges (every edge belongs to one post, so the
  // updates are independent)
  if (a.stdp) {
    __syncthreads();
    const uint32_t p1 = min(p0 + a.P, a.Nd), lane = lane_id();
    for (uint32_t wd = p0 / 32 + (tid >> 5); wd < p1 / 32; wd += kScatterThreads / 32) {
      uint32_t bits = a.last_bits[wd];
      while (bits) {
        const uint32_t b = __ffs(bits) - 1;
        bits &= bits - 1;
        const uint32_t q = wd * 32 + b;
        for (uint32_t k = a.in_ptr[q] + lane; k < a.in_ptr[q + 1]; k += 32) {
          const uint32_t e = a.in_edge[k];
          const float w0 = __uint_as_float(a.edge[e].y);
          const float w1 = fminf(fmaxf(w0 + a.a_plus * a.x_pre[a.in_pre[k]], a.w_min), a.w_max);
          a.edge[e].y = __float_as_uint(w1);
          drift += (double)w1 - (double)w0;
        }
      }
    }
    for (int o = 16; o > 0; o >>= 1) drift += __shfl_xor_sync(0xffffffffu, drift, o);
    if (lane == 0 && drift != 0.0) atomicAdd(&S.drift, drift);
  }
  __syncthreads();
  if (tid == 0) {
    if (S.events) atomicAdd(a.ev_step, S.events);
    if (S.src_events) atomicAdd(a.ev_src_step, S.src_events);
    if (a.stdp && S.drift != 0.0) atomicAdd(a.drift, S.drift);
  }
  pdl_release();
  end_of_step(a, n_spikes);
}

constexpr uint32_t kRedThreads = 256;        // warp 0: producer; warps 1-7: consumers
constexpr uint32_t kRedConsumers = kRedThreads - 32;
#ifndef SG_RED_BLOCKS_PER_SM
#define SG_RED_BLOCKS_PER_SM 2
#endif
#ifndef SG_RED_UNROLL
#define SG_RED_UNROLL 1
#endif
constexpr uint32_t kRedBlocksPerSM = SG_RED_BLOCKS_PER_SM;
constexpr int kRedUnroll = SG_RED_UNROLL;  // consumer loop unroll
constexpr uint32_t kRedSegs = 16;            // row pieces per stage (short rows share a stage)
// A stage ring of STAGES stages of CHUNK synapses each.  Stage regions: x
// words or FP32 records, weights (split formats), code bytes (networks whose
// code bytes are a separate array).  Each row piece is widened to 16-byte
// boundaries: at most 32 extra bytes per piece and region.
template <uint32_t STAGES, uint32_t CHUNK> struct RedCfg {
  static constexpr uint32_t kStages = STAGES;
  static constexpr uint32_t kChunk = CHUNK;
  static constexpr uint32_t kXBytes = CHUNK * 8 + kRedSegs * 32;
  static constexpr uint32_t kWBytes = CHUNK * 2 + kRedSegs * 32;
  static constexpr uint32_t kCBytes = CHUNK + kRedSegs * 32;
  static constexpr uint32_t kStageBytes = kXBytes + kWBytes + kCBytes;
};
// the fixed schedule (the autotuner's other candidates: sg_autotune)
constexpr uint32_t kRedStagesDefault = 4, kRedChunkDefault = 1024;
constexpr unsigned long long kWaitNs = 1000000000ull;     // every pipeline wait gives up after ~1 s

__device__ __forceinline__ void red_add(float *p, float v, unsigned long long pol) {
  asm volatile("red.global.add.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(pol) : "memory");
}

// ---- mbarrier / 1-D bulk copy helpers (this CTA's shared memory only) ----
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Waits for the phase of `parity` to complete, at most ~kWaitNs; false when
// the time ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try(bar, parity)) return true;
    if ((i & 63u) == 0 && global_ns() - t0 > kWaitNs) return false;
  }
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Bulk copy of `bytes` (a multiple of 16) from global `src` (16-byte aligned)
// to shared `dst` (16-byte aligned), completing on `bar`; L2 policy `pol`
// (the synapse stream is evict_first, so that it does not push the delay
// rings out of L2).
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                         unsigned long long pol) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
      : "memory");
}

constexpr uint32_t kPoolMax = 64;  // networks in one pooled step
// The consumers' view of one network of the launch.
struct RedNet {
  float *ring;
  const uint8_t *code;  // separate code bytes, or null
  uint32_t Nd, nslots, base, post_mask;
  int fmt;              // 0 FP32 records, 1 BF16, 2 FP8
};
// One piece of a row in a stage.
struct RedSeg {
  uint32_t first;   // index of its first synapse among the stage's synapses
  uint32_t x;       // element index of its first synapse in the stage's x region
  uint32_t w;       // element index of its first weight in the weight region
  uint32_t c;       // index of its first code byte in the code region
  uint32_t net;     // the network it belongs to
  float scale;      // FP8 row scale
};
// One stage: up to CHUNK synapses from up to kRedSegs row pieces.
struct RedStage {
  uint32_t n;       // synapses in the stage, or kEmpty: the producer is done
  uint32_t n_seg;
  RedSeg seg[kRedSegs];
};
template <uint32_t STAGES, uint32_t CHUNK> struct RedSmemT {
  alignas(16) unsigned char buf[STAGES][RedCfg<STAGES, CHUNK>::kStageBytes];
  RedStage meta[STAGES];
  uint64_t full[STAGES];
  uint64_t empty[STAGES];
  RedNet nets[kPoolMax];
  unsigned long long ev[kPoolMax], src_ev[kPoolMax];  // this block's events per network
};

// Copies elements [b, e) of an array of `esz`-byte elements to shared memory
// at byte offset *cursor of `region`, widened to 16-byte boundaries (the
// arrays are padded so that the widened end stays inside them), announcing
// the bytes on `bar` first.  Returns the element index of b in the region
// and advances *cursor.
__device__ __forceinline__ uint32_t bulk_elems(unsigned char *region, uint32_t *cursor, const void *arr, uint32_t esz,
                                               uint32_t b, uint32_t e, uint64_t *bar, unsigned long long pol) {
  const uint32_t per = 16u / esz;
  const uint32_t b0 = b - b % per, e1 = (e + per - 1) / per * per;
  const uint32_t bytes = (e1 - b0) * esz;
  const uint32_t at = *cursor;
  mbar_expect_tx(bar, bytes);
  bulk_g2s(region + at, (const unsigned char *)arr + (size_t)b0 * esz, bytes, bar, pol);
  *cursor = at + bytes;
  return at / esz + (b - b0);
}

// Poisson-source synapses (source order free) and the end of the step, for a
// pre-centric scatter block of THREADS threads.  base[i]: network i's ring
// slot base; ev / src_ev: this block's event counts per network (shared
// memory; ev holds its recurrent events already).
template <uint32_t THREADS>
__device__ __forceinline__ void red_sources_and_close(const StepArgs *__restrict__ nets, uint32_t n_nets,
                                                      const RedNet *rn, unsigned long long *ev,
                                                      unsigned long long *src_ev, uint32_t *done,
                                                      unsigned long long pl) {
  const uint32_t tid = threadIdx.x, lane = lane_id();
  for (uint32_t i = 0; i < n_nets; ++i) {
    const StepArgs &a = nets[i];
    const uint32_t base = rn[i].base;
    unsigned long long sev = 0;
    for (uint32_t t = blockIdx.x * THREADS + tid; t < a.n_src_syn; t += gridDim.x * THREADS) {
      uint32_t lo = 0, hi = a.n_runs - 1;  // largest run with run_off[run] <= t
      while (lo < hi) {
        const uint32_t mid = lo + ((hi - lo + 1) >> 1);
        if (__ldg(a.run_off + mid) <= t) lo = mid;
        else hi = mid - 1;
      }
      const uint32_t off = t - __ldg(a.run_off + lo);
      const float p = __ldg(a.run_p + lo);
      if (p > 0.0f && poisson_spike(__ldg(a.run_seed0 + lo) + off, 0, *a.step, p)) {
        const uint8_t code = __ldg(a.run_code + lo);
        uint32_t slot = base + max(code_delay(code), 1u);
        if (slot >= a.nslots) slot -= a.nslots;
        red_add(a.ring + ((size_t)code_ring(code) * a.nslots + slot) * a.Nd + __ldg(a.run_post0 + lo) + off,
                __ldg(a.run_w + lo), pl);
        ++sev;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sev += __shfl_xor_sync(0xffffffffu, sev, o);
    if (lane == 0 && sev) atomicAdd(&src_ev[i], sev);
  }
  __syncthreads();
  for (uint32_t i = tid; i < n_nets; i += THREADS) {
    const unsigned long long e = ev[i] + src_ev[i];
    if (e) atomicAdd(nets[i].ev_step, e);
    if (src_ev[i]) atomicAdd(nets[i].ev_src_step, src_ev[i]);
  }
  // the last block to finish closes the step of every network
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    const uint32_t t = atomicAdd(done, 1u);
    if (t == gridDim.x - 1) {
      __threadfence();
      for (uint32_t i = 0; i < n_nets; ++i) end_of_step_last(nets[i], *(volatile uint32_t *)nets[i].red_cnt);
      *done = 0;
      __threadfence();
    }
  }
}

// ---------------------------------------------------------------------------
// Pre-centric scatter (rings_exact networks, and the atomic mode).  When every
// partial sum of a ring cell is exact, the order of the adds does not change
// a cell's bits, so each spiking row is read once, whole, and every event goes
// to its ring cell with a fire-and-forget red.global.add in L2 (the rings stay
// L2-resident: the synapse records stream through, the ring cells are updated
// with evict_last).  One launch serves a table of networks (a single network,
// or every network of a pool): block b takes spiking rows b, b + G, ... of
// each network in turn.  Warp 0 is the producer: its lanes look up 32 rows
// at a time (flat list, row bounds) and lane 0 copies the rows, CHUNK
// synapses per stage (short rows share a stage), into a STAGES-deep
// shared-memory ring with 1-D bulk copies (cp.async.bulk,
// this GPU's memory, no multicast) that complete on the stage's mbarrier.
// Warps 1-7 consume: per stage they read the synapses from shared memory and
// issue the reds, then release the stage.  Every wait gives up after ~1 s,
// records the failure in *err and leaves the kernel (with the copies it
// issued completed).  Poisson-source synapses that the neuron kernel does not
// take (deferred drive) follow, one per thread.  The last block to finish
// closes the step of every network of the table.
// ---------------------------------------------------------------------------
template <uint32_t STAGES, uint32_t CHUNK>
__global__ void __launch_bounds__(kRedThreads, kRedBlocksPerSM)
    scatter_red_kernel(const StepArgs *__restrict__ nets, uint32_t n_nets, uint32_t *done, uint32_t *err,
                       uint32_t stall) {
  using Cfg = RedCfg<STAGES, CHUNK>;
  constexpr uint32_t kRedStages = Cfg::kStages, kRedChunk = Cfg::kChunk, kRedXBytes = Cfg::kXBytes,
                     kRedWBytes = Cfg::kWBytes;
  extern __shared__ __align__(128) unsigned char red_smem[];
  RedSmemT<STAGES, CHUNK> &S = *reinterpret_cast<RedSmemT<STAGES, CHUNK> *>(red_smem);
  const uint32_t tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
  if (tid == 0) {
    for (uint32_t k = 0; k < kRedStages; ++k) {
      mbar_init(&S.full[k], 1);
      mbar_init(&S.empty[k], kRedConsumers / 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  pdl_wait();
  for (uint32_t i = tid; i < n_nets; i += kRedThreads) {
    const StepArgs &a = nets[i];
    RedNet r;
    r.ring = a.ring;
    r.code = a.code;
    r.Nd = a.Nd;
    r.nslots = a.nslots;
    const unsigned long long st = *a.step;
    if (blockIdx.x == 0) hint_store(a, st + 1);  // for the next neuron kernel's pre-wait work
    r.base = (uint32_t)(st % a.nslots);
    r.post_mask = a.post_mask;
    r.fmt = a.wbf16 ? 1 : a.wfp8 ? 2 : 0;
    S.nets[i] = r;
    S.ev[i] = 0;
    S.src_ev[i] = 0;
  }
  __syncthreads();
  const unsigned long long pl = policy_evict_last();
  bool failed = false;
  if (warp == 0) {
    // ---- producer ----
    const unsigned long long pf = policy_evict_first();
    uint32_t stage = 0, eph = 1;        // the first round of empty waits passes at once
    uint32_t filled = 0, fill_par = 0;  // lane 0: per stage (bit), closed at least once, parity of the closes
    bool open = false;                  // lane 0: a stage is being filled
    uint32_t cnt = 0, nseg = 0, xc = 0, wc = 0, cc = 0;
    // lane 0 only: start filling the next stage once the consumers released it
    auto open_stage = [&]() -> bool {
      if (stall || !mbar_wait(&S.empty[stage], eph)) return false;
      open = true;
      cnt = nseg = xc = wc = cc = 0;
      return true;
    };
    // lane 0 only: the stage's description, then the arrival that (with the
    // copies' bytes) completes its phase
    auto close_stage = [&]() {
      S.meta[stage].n = cnt;
      S.meta[stage].n_seg = nseg;
      mbar_arrive(&S.full[stage]);
      filled |= 1u << stage;
      fill_par ^= 1u << stage;
      open = false;
      if (++stage == kRedStages) {
        stage = 0;
        eph ^= 1u;
      }
    };
    for (uint32_t i = 0; i < n_nets && !failed; ++i) {
      const StepArgs &a = nets[i];
      const uint32_t n = *a.red_cnt;
      const uint32_t xsz = a.wbf16 || a.wfp8 ? 4u : 8u;  // bytes per x word or record
      unsigned long long ev = 0;
      for (uint32_t r0 = blockIdx.x; r0 < n && !failed; r0 += 32 * gridDim.x) {
        const uint32_t r = r0 + lane * gridDim.x;
        uint32_t beg = 0, end = 0;
        float scale = 1.0f;
        if (r < n) {
          const uint32_t gi = a.red_flat[r];
          beg = __ldg(a.row_ptr + gi);
          end = __ldg(a.row_ptr + gi + 1);
          if (a.wfp8) scale = __ldg(a.row_scale + gi);
        }
        for (uint32_t k = 0; k < 32 && !failed; ++k) {
          const uint32_t b = __shfl_sync(0xffffffffu, beg, k), e = __shfl_sync(0xffffffffu, end, k);
          const float sc = __shfl_sync(0xffffffffu, scale, k);
          if (lane == 0) {
            ev += e - b;
            for (uint32_t c = b; c < e;) {
              if (!open && !open_stage()) {
                failed = true;
                break;
              }
              const uint32_t take = min(e - c, kRedChunk - cnt);
              unsigned char *buf = S.buf[stage];
              RedSeg &g = S.meta[stage].seg[nseg];
              g.first = cnt;
              g.net = i;
              g.scale = sc;
              g.x = bulk_elems(buf, &xc, xsz == 8 ? (const void *)a.edge : (const void *)a.edge_x, xsz, c, c + take,
                               &S.full[stage], pf);
              g.w = 0;
              if (a.wbf16) g.w = bulk_elems(buf + kRedXBytes, &wc, a.w16, 2, c, c + take, &S.full[stage], pf);
              if (a.wfp8) g.w = bulk_elems(buf + kRedXBytes, &wc, a.w8, 1, c, c + take, &S.full[stage], pf);
              g.c = 0;
              if (a.code)
                g.c = bulk_elems(buf + kRedXBytes + kRedWBytes, &cc, a.code, 1, c, c + take, &S.full[stage], pf);
              cnt += take;
              c += take;
              if (++nseg == kRedSegs || cnt == kRedChunk) close_stage();
            }
          }
          failed = __shfl_sync(0xffffffffu, failed ? 1u : 0u, 0) != 0;
        }
      }
      if (lane == 0 && ev) atomicAdd(&S.ev[i], ev);
    }
    if (lane == 0) {
      if (!failed && open) close_stage();
      // end marker: the consumers leave when they reach it
      if (!failed && open_stage()) {
        S.meta[stage].n = kEmpty;
        S.meta[stage].n_seg = 0;
        mbar_arrive(&S.full[stage]);
      } else {
        atomicOr(err, 1u);
        // the copies of every closed stage land before the block ends
        // (the last close of a stage completes the phase of parity (closes - 1) & 1)
        for (uint32_t k = 0; k < kRedStages; ++k)
          if ((filled >> k) & 1u) (void)mbar_wait(&S.full[k], ((fill_par >> k) & 1u) ^ 1u);
      }
    }
  } else {
    // ---- consumers ----
    const uint32_t ct = tid - 32;
    uint32_t stage = 0, fph = 0;
    for (;;) {
      if (!mbar_wait(&S.full[stage], fph)) {
        if (ct == 0) atomicOr(err, 1u);
        break;
      }
      const uint32_t n = S.meta[stage].n, n_seg = S.meta[stage].n_seg;
      if (n == kEmpty) break;
      const unsigned char *buf = S.buf[stage];
      const RedSeg *segs = S.meta[stage].seg;
#pragma unroll kRedUnroll
      for (uint32_t k = ct; k < n; k += kRedConsumers) {
        uint32_t q = 0;  // the piece holding synapse k
        while (q + 1 < n_seg && segs[q + 1].first <= k) ++q;
        const RedSeg &g = segs[q];
        const uint32_t idx = k - g.first;
        const RedNet &r = S.nets[g.net];
        uint32_t x, wbits;
        if (r.fmt == 0) {
          const uint2 rec = reinterpret_cast<const uint2 *>(buf)[g.x + idx];
          x = rec.x;
          wbits = rec.y;
        } else {
          x = reinterpret_cast<const uint32_t *>(buf)[g.x + idx];
          if (r.fmt == 1) wbits = (uint32_t)reinterpret_cast<const uint16_t *>(buf + kRedXBytes)[g.w + idx] << 16;
          else wbits = __float_as_uint(e4m3_to_f32(buf[kRedXBytes + g.w + idx]) * g.scale);
        }
        const uint8_t code = r.code ? buf[kRedXBytes + kRedWBytes + g.c + idx] : (uint8_t)(x >> 24);
        uint32_t slot = r.base + max(code_delay(code), 1u);
        if (slot >= r.nslots) slot -= r.nslots;
        red_add(r.ring + ((size_t)code_ring(code) * r.nslots + slot) * r.Nd + (x & r.post_mask),
                __uint_as_float(wbits), pl);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&S.empty[stage]);
      if (++stage == kRedStages) {
        stage = 0;
        fph ^= 1u;
      }
    }
  }
  __syncthreads();
  pdl_release();
  red_sources_and_close<kRedThreads>(nets, n_nets, S.nets, S.ev, S.src_ev, done, pl);
}

// ---------------------------------------------------------------------------
// Warp-walk scatter: the same sums as scatter_red_kernel (rings_exact
// networks, and the atomic mode) without a staging ring, so nothing in it
// waits on another warp.  Every warp of the grid takes spiking rows
// round-robin: row r of a network's flat list goes to warp place
// (r + rot) mod W, where W is the number of warps, rot continues the
// round-robin from the previous network of the table, and warp w of block b
// has place w * G + b (G blocks).  A warp holds up to 32 rows at a time (lane
// k the bounds of its k-th row; a warp scan gives each row's offset in their
// concatenation) and walks the concatenation U * 32 synapses per round:
// each lane finds the row of each of its synapses (a binary search over the
// lanes' offsets when the warp holds several rows), issues its U coalesced
// record loads (evict_first in L2), then the U reds into the ring cells
// (red.global.add, evict_last, so the rings stay L2-resident).
// Poisson-source synapses that the neuron kernel does not take follow, one
// per thread; the last block to finish closes the step of every network.
// ---------------------------------------------------------------------------
constexpr uint32_t kWalkThreads = 256;
constexpr uint32_t kWalkWarps = kWalkThreads / 32;

// One round of a warp's walk: the U synapses of each lane, as loaded.
template <int U> struct WalkRound {
  uint32_t x[U], w[U], c[U];  // record x word (post | code), weight bits, code byte (separate code array)
  float s[U];                 // FP8 row scale
  uint32_t ok;                // bit u: synapse u of this lane exists
};

// U: record loads per lane per round.  PIPE = false: each round loads its
// records and then issues its reds.  PIPE = true: the records of the next
// round are loaded before the reds of the current one are issued, so that
// their memory latency runs under the reds instead of after them (a warp's
// loads queue behind its earlier reds).  FMT: the weight storage of every
// network of the table when it is known at compile time (1 FP32 in 8-byte
// records, 2 BF16, 3 FP8; the code byte inside the x word, no separate code
// array), so that the round's registers hold only what is loaded; 0: read
// per network at run time.  P: each spiking row is cut into
// P pieces of (nearly) equal length, and the pieces are the work items of
// the round-robin (more warps busy on a step with few long rows).  MINB:
// resident blocks per SM the registers are sized for.
template <int U, bool PIPE, int FMT, uint32_t P = 1, int MINB = (PIPE && U > 4) ? 3 : 4>
__global__ void __launch_bounds__(kWalkThreads, MINB)
    scatter_walk_kernel(const StepArgs *__restrict__ nets, uint32_t n_nets, uint32_t *done) {
  __shared__ RedNet rn[kPoolMax];
  __shared__ unsigned long long ev[kPoolMax], src_ev[kPoolMax];
  __shared__ uint32_t rot[kPoolMax];
  const uint32_t tid = threadIdx.x, lane = lane_id();
  const uint32_t W = gridDim.x * kWalkWarps;
  // the warp's place in the round-robin: warp w of block b is w * G + b, so
  // that consecutive rows go to consecutive blocks and every SM gets its
  // share of the step's rows (not the first blocks all of them)
  const uint32_t gw = (tid >> 5) * gridDim.x + blockIdx.x;
  // the table of networks is host-written: read before the wait; the step
  // counter and the spike list are the previous kernels' and read after it
  for (uint32_t i = tid; i < n_nets; i += kWalkThreads) {
    const StepArgs &a = nets[i];
    RedNet r;
    r.ring = a.ring;
    r.code = a.code;
    r.Nd = a.Nd;
    r.nslots = a.nslots;
    r.post_mask = a.post_mask;
    r.fmt = a.wbf16 ? 1 : a.wfp8 ? 2 : 0;
    r.base = 0;
    rn[i] = r;
    ev[i] = 0;
    src_ev[i] = 0;
  }
  // the first network's list (Nd entries) and this lane's first item in it
  // (the round-robin of the first network starts at place 0)
  const uint2 *rows0 = n_nets ? nets[0].red_rows : nullptr;
  const unsigned long long rr0 = (gw + (unsigned long long)lane * W) / P;
  const bool spec = n_nets && rr0 < nets[0].Nd;
  pdl_wait();
  // that item's row range, loaded beside the counts instead of after them
  // (used only when the item exists, i.e. lies below the step's count)
  const uint2 rb_first = spec ? rows0[rr0] : make_uint2(0u, 0u);
  for (uint32_t i = tid; i < n_nets; i += kWalkThreads) {
    const unsigned long long st = *nets[i].step;
    if (blockIdx.x == 0) hint_store(nets[i], st + 1);  // for the next neuron kernel's pre-wait work
    rn[i].base = (uint32_t)(st % rn[i].nslots);
  }
  if (tid == 0) {
    uint32_t r0 = 0;
    for (uint32_t i = 0; i < n_nets; ++i) {
      rot[i] = r0;
      r0 = (uint32_t)(((unsigned long long)r0 + (unsigned long long)*nets[i].red_cnt * P) % W);
    }
  }
  __syncthreads();
  const unsigned long long pl = policy_evict_last(), pf = policy_evict_first();
  for (uint32_t i = 0; i < n_nets; ++i) {
    const StepArgs &a = nets[i];
    const RedNet r = rn[i];
    const uint32_t fmt = FMT ? (uint32_t)(FMT - 1) : r.fmt;
    const uint8_t *code_arr = FMT ? nullptr : r.code;
    const unsigned long long n = (unsigned long long)*a.red_cnt * P;  // work items: row pieces
    unsigned long long wev = 0;
    const unsigned long long g_first = (gw + W - rot[i]) % W;
    for (unsigned long long g0 = g_first; g0 < n; g0 += 32ull * W) {
      const unsigned long long it = g0 + (unsigned long long)lane * W;
      uint32_t beg = 0, len = 0;
      float scale = 1.0f;
      if (it < n) {
        const uint32_t rr = (uint32_t)(it / P);
        const uint2 rb = (i == 0 && g0 == g_first && spec) ? rb_first : a.red_rows[rr];
        if (P == 1) {
          beg = rb.x;
          len = rb.y - rb.x;
        } else {
          const unsigned long long L = rb.y - rb.x, j = it % P;
          beg = rb.x + (uint32_t)(L * j / P);
          len = rb.x + (uint32_t)(L * (j + 1) / P) - beg;
        }
        if (fmt == 2) scale = __ldg(a.row_scale + a.red_flat[rr]);
      }
      uint32_t incl = len;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
      }
      const uint32_t excl = incl - len;
      const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
      const uint32_t nrows = (uint32_t)min(32ull, (n - g0 + W - 1) / W);  // lanes holding a row (piece)
      wev += total;
      // load the records of the round starting at synapse b0 of the concatenation
      auto fetch = [&](uint32_t b0, WalkRound<U> &R) {
        uint32_t idx[U];
        R.ok = 0;
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const uint32_t e = b0 + (uint32_t)u * 32u + lane;
          uint32_t k = 0;  // the row holding synapse e: the last row whose offset is <= e
          if (nrows > 1) {
#pragma unroll
            for (uint32_t st = 16; st > 0; st >>= 1) {
              const uint32_t c = k + st;
              const uint32_t ex = __shfl_sync(0xffffffffu, excl, c & 31u);
              if (c < nrows && ex <= e) k = c;
            }
          }
          idx[u] = __shfl_sync(0xffffffffu, beg, k) + (e - __shfl_sync(0xffffffffu, excl, k));
          R.s[u] = (FMT == 0 || FMT == 3) ? __shfl_sync(0xffffffffu, scale, k) : 1.0f;
          R.ok |= (e < total ? 1u : 0u) << u;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          R.x[u] = 0;
          R.w[u] = 0;
          R.c[u] = 0;
          if ((R.ok >> u) & 1u) {
            if (fmt == 0) {
              const uint2 rec = ld_stream_edge(a.edge + idx[u], pf);
              R.x[u] = rec.x;
              R.w[u] = rec.y;
            } else {
              R.x[u] = ld_stream_u32(a.edge_x + idx[u], pf);
              R.w[u] = fmt == 1 ? ld_stream_u16(a.w16 + idx[u], pf) : ld_stream_u8(a.w8 + idx[u], pf);
            }
            if (code_arr) R.c[u] = __ldg(code_arr + idx[u]);
          }
        }
      };
      // the reds of a loaded round
      auto apply = [&](const WalkRound<U> &R) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (!((R.ok >> u) & 1u)) continue;
          const uint32_t x = R.x[u];
          uint32_t wbits = R.w[u];
          if (fmt == 1) wbits <<= 16;
          else if (fmt == 2) wbits = __float_as_uint(e4m3_to_f32(wbits) * R.s[u]);
          const uint8_t code = code_arr ? (uint8_t)R.c[u] : (uint8_t)(x >> 24);
          uint32_t slot = r.base + max(code_delay(code), 1u);
          if (slot >= r.nslots) slot -= r.nslots;
          red_add(r.ring + ((size_t)code_ring(code) * r.nslots + slot) * r.Nd + (x & r.post_mask),
                  __uint_as_float(wbits), pl);
        }
      };
      constexpr uint32_t kRound = 32u * (uint32_t)U;
      if (PIPE) {
        WalkRound<U> A, B;
        fetch(0, A);
        for (uint32_t b0 = 0; b0 < total; b0 += 2u * kRound) {
          if (b0 + kRound < total) fetch(b0 + kRound, B);
          else B.ok = 0;
          apply(A);
          if (b0 + 2u * kRound < total) fetch(b0 + 2u * kRound, A);
          else A.ok = 0;
          apply(B);
        }
      } else {
        for (uint32_t b0 = 0; b0 < total; b0 += kRound) {
          WalkRound<U> A;
          fetch(b0, A);
          apply(A);
        }
      }
    }
    if (lane == 0 && wev) atomicAdd(&ev[i], wev);
  }
  __syncthreads();
  pdl_release();
  red_sources_and_close<kWalkThreads>(nets, n_nets, rn, ev, src_ev, done, pl);
}

// One neuron launch per model over the populations of several networks (a
// pool): block b takes map[b] = (network, population, block within it).
template <int MODEL, bool FULL>
__global__ void __launch_bounds__(NeuronCfg<MODEL, FULL>::THREADS, NeuronCfg<MODEL, FULL>::MIN_BLOCKS)
    neuron_pool_kernel(const StepArgs *__restrict__ nets, const PopArgs *__restrict__ pops,
                       const uint4 *__restrict__ map) {
  const uint4 m = map[blockIdx.x];
  pdl_wait();
  float sv[n_state(MODEL)][NeuronCfg<MODEL, FULL>::NPT];
  load_state<MODEL, FULL>(pops[m.y], m.z, sv);
  PreWait none;
  none.ok = false;
  neuron_block<MODEL, FULL>(nets[m.x], pops[m.y], m.z, sv, none);
  pdl_release();
}

// Adds the deferred drive of step t - 1 (t >= 1) of one population into
// slot t, where the ring would hold it, and records that it was added (the
// neuron kernel of step t then leaves it out).
__global__ void drive_fold_kernel(float *ring, uint32_t Nd, uint32_t nslots, unsigned long long t, PopArgs p,
                                  unsigned long long *fold) {
  float *rs = ring + (size_t)(t % nslots) * Nd + p.dev_off;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += gridDim.x * blockDim.x)
    if (poisson_spike(p.drv_seed0 + i, 0, t - 1, p.drv_p)) rs[i] = rs[i] + p.drv_w;
  if (blockIdx.x == 0 && threadIdx.x == 0) *fold = t - 1;
}

// ---------------------------------------------------------------------------
// Dopamine-modulated eligibility over the network's synapses, lazy form
// (P/api/learn/brain.rs:199-286).  A synapse's eligibility is stored as of
// its last sync step; each step touches only the synapses of spiking
// neurons: the gap since the last sync decays by repeated multiplication
// with d_e (one rounding per elapsed step, as the per-step dense update
// does), this step's terms are added in the order the reference stages them
// (neurons ascending, a neuron's in-edges before its out-edges), then one
// trailing multiplication by d_e.  A synapse whose post spiked is handled
// with its post's in-edges (with its LTD term too when its pre also
// spiked), one whose only the pre spiked with the pre's out-edges: every
// synapse has one owner per step, so the updates need no atomics.
// ---------------------------------------------------------------------------
// Per synapse the state is one 8-byte record: x = eligibility (f32 bits),
// y = the step of its last sync.
constexpr uint32_t kLearnInline = 32;   // gaps up to this many steps decay in the gather kernel
constexpr uint32_t kLearnBuckets = 12;  // longer ones by floor(log2(gap)) - 5, the last open-ended
constexpr uint32_t kLearnThreads = 256;

struct LearnArgs {
  const uint32_t *bits;     // this step's spike bitmask [Nd/32]
  const uint32_t *flat;     // this step's spiking neurons
  const uint32_t *flat_cnt;
  uint32_t *grab;           // next entry of `flat` to take
  const uint32_t *row_ptr;  // out-edges (CSR, synapse index = record index)
  const uint2 *edge;
  int packed;
  const uint32_t *in_ptr, *in_edge, *in_pre;  // in-edges of every neuron
  const float *tp, *tq;                        // traces after this step's spikes
  uint2 *st;
  uint4 *qa;      // deferred synapses per bucket: {synapse, e, gap | two << 31, s1}
  float *qb;      //   and s2
  uint32_t *qcnt;  // [kLearnBuckets]
  uint32_t qcap;   // entries per bucket
  const unsigned long long *step;
  unsigned long long t0;
  float d_e, a_ltp, a_ltd;
};

__device__ __forceinline__ bool bit_set(const uint32_t *bits, uint32_t i) { return (bits[i >> 5] >> (i & 31)) & 1u; }

// e multiplied by d, g times, one rounding each (the reference's gap loop);
// zero stays zero (of its sign), so the chain may stop there.  Chunks of 16
// keep the loop overhead off the dependent multiplications.
__device__ __forceinline__ float decay_by(float e, uint32_t g, float d) {
  for (; g >= 16u && e != 0.0f; g -= 16u) {
#pragma unroll
    for (int u = 0; u < 16; ++u) e = __fmul_rn(e, d);
  }
  for (; g && e != 0.0f; --g) e = __fmul_rn(e, d);
  return e;
}

// A synapse's update after its gap has decayed: this step's terms in the
// reference's order (e - ltd is computed as e + (-ltd), the same IEEE result),
// then the trailing decay.
__device__ __forceinline__ uint2 learn_finish(float e, float s1, float s2, bool two, float d_e, uint32_t t) {
  e = __fadd_rn(e, s1);
  if (two) e = __fadd_rn(e, s2);
  return make_uint2(__float_as_uint(__fmul_rn(e, d_e)), t);
}

// Gather: CTAs take this step's spiking neurons one at a time; the threads of
// a CTA share the neuron's synapses (in-edges, then out-edges), read each
// one's state and terms, finish short gaps in place and queue long ones by
// gap length for learn_decay_kernel, so that a warp there runs gaps of
// similar length.  A synapse whose post spiked is handled with its post's
// in-edges, one whose only the pre spiked with the pre's out-edges: every
// synapse has one owner per step.
__global__ void __launch_bounds__(kLearnThreads) learn_elig_kernel(LearnArgs L) {
  __shared__ uint32_t s_n;
  __shared__ uint32_t s_qbase[kLearnThreads / 32][kLearnBuckets];
  const uint32_t t = (uint32_t)(*L.step - L.t0);  // the step counter has advanced past this step
  const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  const uint32_t n_spk = *L.flat_cnt;
  for (;;) {
    if (threadIdx.x == 0) {
      const uint32_t j = atomicAdd(L.grab, 1u);
      s_n = j < n_spk ? L.flat[j] : 0xFFFFFFFFu;
    }
    __syncthreads();
    const uint32_t n = s_n;
    __syncthreads();
    if (n == 0xFFFFFFFFu) break;
    const uint32_t k0 = L.in_ptr[n], n_in = L.in_ptr[n + 1] - k0, r0 = L.row_ptr[n];
    const uint32_t K = n_in + (L.row_ptr[n + 1] - r0);
    const float ltd_n = __fmul_rn(L.a_ltd, L.tq[n]);
    for (uint32_t b0 = 0; b0 < K; b0 += kLearnThreads) {
      const uint32_t x = b0 + threadIdx.x;
      bool work = x < K, two = false;
      uint32_t i = 0;
      float s1 = 0.0f, s2 = 0.0f;
      if (work && x < n_in) {  // n as post: LTP, and LTD where the pre fired too
        const uint32_t k = k0 + x, p = L.in_pre[k];
        i = L.in_edge[k];
        const float ltp = __fmul_rn(L.a_ltp, L.tp[p]);
        two = bit_set(L.bits, p);
        s1 = two && p < n ? -ltd_n : ltp;
        s2 = two && p < n ? ltp : -ltd_n;
      } else if (work) {  // n as pre: LTD where the post did not fire
        i = r0 + (x - n_in);
        const uint2 r = L.edge[i];
        const uint32_t q = L.packed ? (r.x & 0x00FFFFFFu) : r.x;
        work = !bit_set(L.bits, q);
        if (work) s1 = -__fmul_rn(L.a_ltd, L.tq[q]);
      }
      float e = 0.0f;
      uint32_t gap = 0;
      if (work) {
        const uint2 st = L.st[i];
        e = __uint_as_float(st.x);
        gap = st.y < t && e != 0.0f ? t - st.y - 1u : 0u;  // a zero stays zero under decay
      }
      uint32_t bk = 0xFFu;
      if (work && gap > kLearnInline) bk = min(31u - (uint32_t)__clz(gap), 5u + kLearnBuckets - 1u) - 5u;
      // queue long gaps, one atomic per bucket and warp
      const uint32_t peers = __match_any_sync(0xffffffffu, bk);
      bool queued = false;
      if (bk != 0xFFu) {
        const uint32_t leader = __ffs(peers) - 1;
        if (lane == leader) s_qbase[wid][bk] = atomicAdd(L.qcnt + bk, (uint32_t)__popc(peers));
      }
      __syncwarp();
      if (bk != 0xFFu) {
        const uint32_t slot = s_qbase[wid][bk] + (uint32_t)__popc(peers & ((1u << lane) - 1u));
        if (slot < L.qcap) {
          const size_t o = (size_t)bk * L.qcap + slot;
          L.qa[o] = make_uint4(i, __float_as_uint(e), gap | (two ? 0x80000000u : 0u), __float_as_uint(s1));
          L.qb[o] = s2;
          queued = true;
        }
      }
      __syncwarp();
      if (work && !queued) {  // short gap (or a full queue)
        e = decay_by(e, gap, L.d_e);
        L.st[i] = learn_finish(e, s1, s2, two, L.d_e, t);
      }
    }
  }
}

// The queued synapses: each thread one synapse, buckets in turn.
__global__ void __launch_bounds__(kLearnThreads) learn_decay_kernel(LearnArgs L) {
  const uint32_t t = (uint32_t)(*L.step - L.t0);
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x, G = gridDim.x * blockDim.x;
  for (uint32_t b = 0; b < kLearnBuckets; ++b) {
    const uint32_t nb = min(L.qcnt[b], L.qcap);
    for (uint32_t k = g; k < nb; k += G) {
      const size_t o = (size_t)b * L.qcap + k;
      const uint4 q = L.qa[o];
      const float s2 = L.qb[o];
      const float e = decay_by(__uint_as_float(q.y), q.z & 0x7FFFFFFFu, L.d_e);
      L.st[q.x] = learn_finish(e, __uint_as_float(q.w), s2, (q.z >> 31) != 0u, L.d_e, t);
    }
  }
}

// Reward (brain.rs:254-309): every eligibility brought to now, then
// w += lr*dopamine*e clamped to [w_min, w_max]; a zero delta leaves w as it is.
__global__ void __launch_bounds__(256) learn_reward_kernel(uint2 *edge, uint2 *st, const unsigned long long *step,
                                                           unsigned long long t0, uint64_t E, float d_e,
                                                           float lr_dopa, float w_min, float w_max) {
  const uint32_t t = (uint32_t)(*step - t0);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint2 s = st[i];
    float e = __uint_as_float(s.x);
    if (s.y < t) {
      e = decay_by(e, t - s.y, d_e);
      st[i] = make_uint2(__float_as_uint(e), t);
    }
    const float delta = __fmul_rn(lr_dopa, e);
    if (delta == 0.0f) continue;
    float w = __fadd_rn(__uint_as_float(edge[i].y), delta);
    w = w < w_min ? w_min : (w > w_max ? w_max : w);
    edge[i].y = __float_as_uint(w);
  }
}

// clear (brain.rs:271-275): zero and synced to now; or keep[i] == 0 zeroes
// synapse i (restrict, brain.rs:278-285)
__global__ void learn_clear_kernel(uint2 *st, const uint8_t *keep, const unsigned long long *step,
                                   unsigned long long t0, uint64_t E) {
  const uint32_t t = (uint32_t)(*step - t0);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (uint64_t)gridDim.x * blockDim.x) {
    if (keep == nullptr) st[i] = make_uint2(0u, t);
    else if (!keep[i]) st[i].x = 0u;
  }
}

// snapshot (mode 0) and recall w += alpha * (snapshot - w) (brain.rs:343-356)
__global__ void learn_baked_kernel(uint2 *edge, float *baked, uint64_t E, int recall, float alpha) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (uint64_t)gridDim.x * blockDim.x) {
    const float w = __uint_as_float(edge[i].y);
    if (!recall) baked[i] = w;
    else edge[i].y = __float_as_uint(__fadd_rn(w, __fmul_rn(alpha, __fsub_rn(baked[i], w))));
  }
}

// ---------------------------------------------------------------------------
// External populations: the neurons of a network split across GPUs that
// other GPUs simulate.  Their spikes of this step arrive as bitmask words
// (`src`, population-local, from the spike exchange); this kernel publishes
// them as the neuron kernel publishes its own: bitmask words, raster words,
// the block's ascending spike list, STDP and learning traces, the learning
// spike list.  One 1024-thread block per 1024-neuron block, a neuron per thread.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kNeuronBlock) ext_spikes_kernel(StepArgs a, uint32_t dev_off, uint32_t n,
                                                                  const uint32_t *__restrict__ src) {
  __shared__ uint32_t wsum[32];
  __shared__ uint32_t flat_base;
  const uint32_t tid = threadIdx.x, lane = tid & 31u;
  const uint32_t i = blockIdx.x * kNeuronBlock + tid, gi = dev_off + i;
  const bool sp = i < n && ((__ldg(src + (i >> 5)) >> (i & 31u)) & 1u);
  const uint32_t word = __ballot_sync(0xffffffffu, sp);
  const unsigned long long step = *a.step;
  if (lane == 0) {
    a.last_bits[gi >> 5] = word;
    if (a.raster != nullptr) a.raster[(size_t)(step % a.raster_cap) * a.words + (gi >> 5)] = word;
  }
  uint32_t total;
  const uint32_t before = block_excl_scan(sp ? 1u : 0u, wsum, &total);
  const uint32_t gblk = gi / kNeuronBlock;
  if (a.red) {
    __shared__ uint32_t red_base;
    if (tid == 0) red_base = total ? atomicAdd(a.red_cnt, total) : 0u;
    __syncthreads();
    if (sp) {
      a.red_flat[red_base + before] = gi;
      a.red_rows[red_base + before] = make_uint2(__ldg(a.row_ptr + gi), __ldg(a.row_ptr + gi + 1));
    }
  } else {
    if (sp) a.spk[(size_t)gblk * kNeuronBlock + before] = make_uint2(gi, __ldg(a.row_ptr + gi));
    if (tid == 0) a.blk_cnt[gblk] = total;
  }
  if (i < n) {
    const float add = sp ? 1.0f : 0.0f;
    if (a.stdp) {
      a.x_pre[gi] = __fmaf_rn(a.x_pre[gi], a.d_pre, add);
      a.x_post[gi] = __fmaf_rn(a.x_post[gi], a.d_post, add);
    }
    if (a.learn) {
      a.l_tp[gi] = __fmaf_rn(a.l_tp[gi], a.l_dpre, add);
      a.l_tq[gi] = __fmaf_rn(a.l_tq[gi], a.l_dpost, add);
      if (sp && gi >= a.l_motor[0] && gi < a.l_motor[1]) atomicAdd(a.l_motor_acc, 1u);
      if (sp && gi >= a.l_motor[2] && gi < a.l_motor[3]) atomicAdd(a.l_motor_acc + 1, 1u);
    }
  }
  if (a.learn) {
    if (tid == 0) flat_base = total ? atomicAdd(a.l_flat_cnt, total) : 0u;
    __syncthreads();
    if (sp) a.l_flat[flat_base + before] = gi;
  }
}

// ---------------------------------------------------------------------------
// inject_current (build.rs:243-275): values land in the slot the next step
// reads.  `sequential` = the index list has repeats, apply in list order.
// ---------------------------------------------------------------------------
__global__ void inject_kernel(float *ring, uint32_t Nd, uint32_t nslots, const unsigned long long *step,
                              const uint32_t *idx, const float *vals, uint64_t n, uint32_t dev_off, int sequential) {
  const uint32_t slot = (uint32_t)(*step % nslots);
  float *rs = ring + (size_t)slot * Nd + dev_off;
  if (sequential) {
    if (blockIdx.x == 0 && threadIdx.x == 0)
      for (uint64_t k = 0; k < n; ++k) rs[idx[k]] = rs[idx[k]] + vals[k];
    return;
  }
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
    rs[idx[k]] = rs[idx[k]] + vals[k];
}

}  // namespace sg
