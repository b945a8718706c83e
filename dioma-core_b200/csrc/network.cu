// network.cu — host side of the SiMuse Network on one B200: builder, device
// layout, step launches, readbacks, and the extern "C" ABI of
// include/simuse_b200.h.
//
// Device layout (HBM).  Populations are placed at 32-aligned offsets of a
// padded device index space (Nd neurons) so that every warp of a neuron
// kernel covers one whole spike-bitmask word; padding neurons never spike and
// own no synapses.  State and params stay SoA, [col][cap] per population
// (P/core/exec/population.rs:16-25).  The delay ring is [n_rings][32][Nd]
// floats (P/api/net/delay.rs:26-35), ring 0 static, ring k the k-th kinetic
// profile.  The CSR keeps the reference's u32 row_ptr/col (graph.rs:67-80),
// f32 weights, and one code byte per edge (delay | syn_type | STDP flag).
#include "taas.h"
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <mutex>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "models.cuh"
#include "step_kernels.cuh"

namespace sg {

thread_local std::string g_last_error;
void set_error(const std::string &msg) { g_last_error = msg; }

template <typename T> struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    release();
    if (count == 0) return;
    SG_CUDA(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void zero(cudaStream_t s) {
    if (p) SG_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
  // at least `count` elements, keeping the buffer when it is large enough
  // (grown by a quarter beyond the request when it is not)
  void ensure(size_t count) {
    if (count <= n) return;
    alloc(count + count / 4);
  }
};

// growable device array for staged edges
template <typename T> struct DVec {
  T *p = nullptr;
  size_t n = 0, cap = 0;
  ~DVec() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = cap = 0;
  }
  void reserve(size_t c, cudaStream_t s) {
    if (c <= cap) return;
    size_t nc = std::max(c, cap + cap / 2);
    T *q = nullptr;
    SG_CUDA(cudaMalloc(&q, nc * sizeof(T)));
    if (n) SG_CUDA(cudaMemcpyAsync(q, p, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
    SG_CUDA(cudaStreamSynchronize(s));
    if (p) cudaFree(p);
    p = q;
    cap = nc;
  }
};

struct HostPop {
  int model;
  uint32_t n, cap, dev_off, np, ns;
  uint32_t umask = 0;   // uniform parameter columns
  float uval[16] = {};
  // Gaussian input noise (sg_pop_set_noise)
  bool noise = false;
  uint32_t noise_stream = 0, noise_split = 0;
  uint64_t noise_seed = 0, noise_stride = 0, noise_step0 = 0;
  double noise_sigma[2] = {0.0, 0.0};
  DBuf<float> d_bias;  // sg_pop_set_bias, [cap] (zero past n)
  // deferred drive (found by build_sources): one Poisson source per neuron,
  // seed drv_seed0 + i, rate drv_p, weight drv_w, delay <= 1, ring 0
  bool drv = false;
  uint32_t drv_seed0 = 0;
  float drv_p = 0.0f, drv_w = 0.0f;
  // external population (sg_pop_add_external): simulated elsewhere, its spike
  // words of each step read from `ext_src` (population-local words)
  bool external = false;
  const uint32_t *ext_src = nullptr;
  std::vector<float> params, state;  // before build
  DBuf<float> d_params, d_state;     // after build
};

struct HostSrc {
  float p;
  uint32_t seed;
};
// One Poisson-source synapse (all of them in one list, in connect order)
struct SrcSyn {
  uint32_t src;
  uint32_t post;  // device index
  float w;
  uint8_t code;
  uint8_t pt;     // Tsodyks-Markram profile (0 none)
};

// A kinetic synapse profile's per-step constants (P/api/net/network/step.rs:
// 206-298): kind 0 ExpOne {a_decay}, 1 ExpTwo {a_rise, a_decay, norm},
// 2 Alpha {r, e*(dt/tau)*r}, 3 ExpThree {a_rise, a_decay1, a_decay2, wf1,
// wf2, k_a, gbase1, gbase2}
struct Kin {
  int kind;
  float erev;
  float c[8];
};

// Tsodyks-Markram profile constants for the network's dt (push.rs:25-35)
struct TmHost {
  float u0, a_rec, a_fac;
  bool fac;
};

}  // namespace sg

using namespace sg;

struct sg_pool;

struct sg_net {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool built = false;
  std::vector<HostPop> pops;
  std::vector<uint32_t> offsets{0};  // reference global offsets
  uint64_t total = 0;                // reference neuron count
  uint32_t Nd = 0;                   // padded device neuron count
  uint32_t max_delay = 0;            // largest synaptic delay added so far
  uint32_t nslots = kSlots;          // ring slots in use (largest effective delay + 1)
  // staged edges (device)
  DVec<uint32_t> e_pre, e_post;
  DVec<float> e_w;
  DVec<uint8_t> e_code;
  std::vector<Kin> kin;
  // receptor kinetics (SynapticBrain): the edges' syn_types are receptor
  // codes, ring slot 0 is the external input and slot 1 + r the conductance
  // of receptor r, decayed by rec_f[r] = fast_exp(-dt / tau_r) each step
  bool receptor = false;
  float rec_f[kReceptors] = {};
  std::vector<HostSrc> srcs;
  std::vector<SrcSyn> src_syn;
  bool stdp_on = false;
  float stdp_dt = 0, tau_pre = 0, tau_post = 0, a_plus = 0, a_minus = 0, w_min = 0, w_max = 0;
  int deterministic = 1;
  int weight_format = SG_W_F32;

  // device state
  DBuf<unsigned long long> d_step, d_ev_step, d_ev_total, d_clamp, d_stat_ev, d_ev_src;  // d_ev_src: [step, total]
  DBuf<uint32_t> d_blk_cnt, d_last_bits, d_raster, d_done, d_stat_spk;
  DBuf<uint2> d_spk;
  DBuf<float> d_ring, d_kin_g;
  DBuf<uint32_t> d_row_ptr;
  // one 8-byte record per synapse: x = post (| code << 24 when packed), y = weight bits
  DBuf<uint2> d_edge;
  DBuf<uint32_t> d_ns_count, d_ns_last;  // sg_neuron_stats_enable
  DBuf<double> d_ns_s1, d_ns_s2;
  unsigned long long ns_step0 = 0;
  DBuf<uint32_t> d_edge_x;  // BF16 form: the records' x words
  DBuf<uint16_t> d_w16;     //   and their weights in bf16
  DBuf<uint8_t> d_w8;       // FP8 form: E4M3 weights (x words in d_edge_x)
  DBuf<float> d_row_scale;  //   and one scale per row
  DBuf<uint8_t> d_code;  // code byte per synapse when it does not fit in x
  int packed = 1;
  uint64_t n_edges = 0;
  // per-row segment table [Nd][G+1] (u16, or u32 when a row is >= 65536 long)
  DBuf<uint8_t> d_seg;
  int seg32 = 0;
  uint32_t G = 0, P = 0, pbits = 0;
  // Poisson sources and their synapses grouped by scatter block
  // runs of source synapses where source id, post and seed advance by one and
  // rate, weight and code are shared (the one-source-per-neuron drive is one
  // run per scatter block)
  DBuf<uint32_t> d_run_lo, d_run_src0, d_run_post0, d_run_len, d_run_seed0;
  DBuf<float> d_run_w, d_run_p;
  DBuf<uint8_t> d_run_code;
  DBuf<uint8_t> d_run_pt;                 // TM profile per run (source synapses)
  DBuf<float> d_src_tm_r, d_src_tm_u;     // TM state per source synapse (run order)
  DBuf<uint32_t> d_src_tm_last;
  bool src_tm = false;                    // a source synapse has a TM profile
  uint64_t n_runs = 0;
  uint64_t n_src_edges = 0;
  DBuf<float> d_x_pre, d_x_post;
  DBuf<uint32_t> d_in_ptr, d_in_edge, d_in_pre;
  DBuf<double> d_drift;
  DBuf<uint32_t> d_inj_idx;
  DBuf<float> d_inj_val;
  uint32_t raster_cap = 0;
  uint64_t raster_read_step = 0;
  uint32_t stat_cap = 1u << 16;
  uint64_t stat_read_step = 0;
  uint64_t host_step = 0;  // steps issued
  size_t scatter_smem = 0;
  // the Poisson-source weights' part of the exact-sum test (rings_exact)
  std::vector<double> src_abs;  // per post, sum of |w| of its source synapses
  int src_lo = 1 << 20;         //   smallest low-bit exponent of a source weight
  bool src_bad = false;         //   a source weight is not finite
  // pre-centric scatter (exact ring sums, or the atomic mode): flat list of
  // the step's spiking neurons and its count; run offsets of the Poisson
  // synapses it rolls
  int red = 0;
  bool exact = false;  // rings_exact at build (cleared when weights start changing)
  DBuf<uint32_t> d_red_flat, d_red_cnt, d_run_off;
  DBuf<uint2> d_red_rows;
  // deferred drive: device record of the last folded step, and its host copy
  DBuf<unsigned long long> d_drv_fold;
  DBuf<uint32_t> d_err;        // device error word (scatter pipeline waits)
  uint32_t debug_stall = 0;    // test hook: the scatter's producer stalls
  // the step arguments in device memory (the pre-centric scatter reads a
  // table of networks' arguments; a network alone is a table of one)
  DBuf<StepArgs> d_args;
  StepArgs h_args{};
  bool args_uploaded = false;
  sg_pool *pool = nullptr;     // the pool this network steps in, if any
  int red_variant = 0;         // pre-centric scatter schedule (sg_autotune)
  uint32_t red_bps = kRedBlocksPerSM;
  bool l2_reserved = false;    // holds a share of the device's L2 set-aside (setup_l2_setaside)
  size_t l2_bytes = 0;         // the ring bytes counted for that share
  unsigned long long drv_folded = ~0ull;
  bool any_drv = false;
  // short-term plasticity: profiles, staged per-edge ids (kept only once an
  // edge has a profile; zero-filled for the edges staged without one), and
  // after build the ids and R, U, last-spike state in CSR order
  std::vector<TmHost> tm_prof;
  DVec<uint8_t> e_pt;
  bool tm_edges = false;
  DBuf<uint8_t> d_pt;
  DBuf<float> d_tm_r, d_tm_u;
  DBuf<uint32_t> d_tm_last;
  // dopamine-modulated eligibility learning (sg_learn_enable): per-neuron
  // traces, per-synapse eligibility and sync step (relative to l_t0, the
  // step counter when learning began), in-edges of every neuron, motor counts
  bool learn_on = false;
  float l_dt = 0, l_tau_pre = 0, l_tau_post = 0, l_tau_e = 0, l_a_ltp = 0, l_a_ltd = 0, l_lr = 0, l_w_min = 0,
        l_w_max = 0;
  float l_dpre = 0, l_dpost = 0, l_de = 0;
  unsigned long long l_t0 = 0;
  uint32_t l_motor[4] = {0, 0, 0, 0};
  DBuf<float> d_l_tp, d_l_tq, d_l_baked, d_l_qb;
  DBuf<uint2> d_l_st;  // per synapse {eligibility bits, sync step}
  DBuf<uint4> d_l_qa;  // deferred long-gap synapses, kLearnBuckets x l_qcap
  DBuf<uint32_t> d_l_in_ptr, d_l_in_edge, d_l_in_pre, d_l_motor, d_l_flat;
  DBuf<uint32_t> d_l_ctr;  // [0] spiking neurons this step, [1] next to take, [2..] queued per bucket
  uint32_t l_qcap = 0;
  // raster readback work buffers, kept from call to call (grow only)
  DBuf<unsigned long long> rr_cnt, rr_off;
  DBuf<uint8_t> rr_temp;
  DBuf<uint32_t> rr_step, rr_idx, rr_pd, rr_pg, rr_soff;
  DBuf<uint32_t> rr_counts;  // spikes per device neuron over every read since the raster was enabled
  // a staged read (sg_raster_stage / sg_raster_fetch): steps [rst_t0, rst_t1)
  // compacted on rstream after the steps that wrote them; the network's
  // later steps wait for that compaction (rdone)
  cudaStream_t rstream = nullptr;
  cudaEvent_t rev = nullptr, rdone = nullptr;
  unsigned long long *rst_total = nullptr;  // pinned host word: the staged batch's spike count
  bool rstaged = false;
  uint64_t rst_t0 = 0, rst_nb = 0, rst_nw = 0;
  // neuron work table: per population its kernel arguments, per model the
  // (population, block) pairs its launch covers
  DBuf<PopArgs> d_pop_tab;
  DBuf<uint2> d_blk_map;
  std::vector<PopArgs> pop_tab;  // host copy
  uint32_t model_blk_off[5] = {}, model_blk_cnt[5] = {};
  int model_single[5] = {-1, -1, -1, -1, -1};  // the one population of a model, or -1
  bool pop_tab_dirty = true;
  // CUDA graph of `graph_steps` steps
  cudaGraphExec_t graph = nullptr;
  uint32_t graph_steps = 0;
  std::vector<float> ln_consts{0, 0};
  // per-phase CUDA-event timing (0 neuron update, 1 scatter)
  bool profile = false;
  std::vector<cudaEvent_t> prof_ev;
  double prof_ms[4] = {0, 0, 0, 0};
  uint64_t prof_launches[4] = {0, 0, 0, 0};

  uint32_t dev_index(uint32_t pop, uint32_t i) const { return pops[pop].dev_off + i; }
};

// A pool of built networks stepped together: per step one neuron launch per
// model over every member's populations and one pre-centric scatter launch
// over every member (continuous batching of resident networks).
struct sg_pool {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  std::vector<sg_net *> members;
  std::vector<StepArgs> h_nets;
  std::vector<PopArgs> h_pops;
  std::vector<uint4> h_map;  // (member, population of h_pops, block), grouped by model
  uint32_t model_off[5] = {}, model_cnt[5] = {};
  bool full[5] = {};  // per model: some member needs the full neuron kernel
  DBuf<StepArgs> d_nets;
  DBuf<PopArgs> d_pops;
  DBuf<uint4> d_map;
  DBuf<uint32_t> d_done, d_err;
  cudaGraphExec_t graph = nullptr;
  uint32_t graph_steps = 0;
};

namespace {

int run(const std::function<void()> &f) {
  try {
    f();
    return SG_OK;
  } catch (const Fail &e) {
    return e.code;
  } catch (const std::bad_alloc &) {
    set_error("host allocation failed");
    return SG_E_NOMEM;
  } catch (const std::exception &e) {
    set_error(e.what());
    return SG_E_INVALID;
  }
}

#define NET_CHECK(net)                                                     \
  do {                                                                     \
    if (!(net)) {                                                          \
      set_error("null network handle");                                    \
      return SG_E_INVALID;                                                 \
    }                                                                      \
  } while (0)

struct DevGuard {
  int prev = -1;
  explicit DevGuard(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~DevGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

void require_pop(const sg_net *net, uint32_t pop) {
  SG_REQUIRE(pop < net->pops.size(), SG_E_INVALID,
             "population " + std::to_string(pop) + " out of range (have " +
                 std::to_string(net->pops.size()) + ")");
}

// synapses, Poisson drive and input target neurons simulated here
void require_local(const sg_net *net, uint32_t pop) {
  require_pop(net, pop);
  SG_REQUIRE(!net->pops[pop].external, SG_E_INVALID,
             "population " + std::to_string(pop) + " is external: its synapses and input belong to the GPU that simulates it");
}

bool has_external(const sg_net *net) {
  for (const auto &p : net->pops)
    if (p.external) return true;
  return false;
}

StepArgs make_args(sg_net *net) {
  StepArgs a{};
  a.step = net->d_step.p;
  a.blk_cnt = net->d_blk_cnt.p;
  a.spk = net->d_spk.p;
  a.n_blk = net->Nd / kNeuronBlock;
  a.last_bits = net->d_last_bits.p;
  a.raster = net->raster_cap ? net->d_raster.p : nullptr;
  a.raster_cap = net->raster_cap ? net->raster_cap : 1;
  a.words = net->Nd / 32;
  a.done = net->d_done.p;
  a.ev_step = net->d_ev_step.p;
  a.ev_total = net->d_ev_total.p;
  a.ev_src_step = net->d_ev_src.p;
  a.ev_src_total = net->d_ev_src.p + 1;
  a.stat_spk = net->d_stat_spk.p;
  a.stat_ev = net->d_stat_ev.p;
  a.stat_cap = net->stat_cap;
  a.clamp_hits = net->d_clamp.p;
  a.ns_count = net->d_ns_count.n ? net->d_ns_count.p : nullptr;
  a.ns_last = net->d_ns_last.p;
  a.ns_s1 = net->d_ns_s1.p;
  a.ns_s2 = net->d_ns_s2.p;
  a.ns_step0 = net->ns_step0;
  a.ring = net->d_ring.p;
  a.Nd = net->Nd;
  a.nslots = net->nslots;
  a.n_kin = (int)net->kin.size();
  for (size_t k = 0; k < net->kin.size() && k < 3; ++k) {
    a.kin_kind[k] = net->kin[k].kind;
    for (int q = 0; q < 8; ++q) a.kin_c[k][q] = net->kin[k].c[q];
    a.kin_erev[k] = net->kin[k].erev;
  }
  a.kin_g = net->d_kin_g.p;
  a.receptor = net->receptor ? 1 : 0;
  for (int r = 0; r < kReceptors; ++r) a.rec_f[r] = net->rec_f[r];
  a.row_ptr = net->d_row_ptr.p;
  a.edge = net->d_edge.p;
  a.wbf16 = net->weight_format == SG_W_BF16 ? 1 : 0;
  a.wfp8 = net->weight_format == SG_W_FP8 ? 1 : 0;
  a.w8 = net->d_w8.p;
  a.row_scale = net->d_row_scale.p;
  a.edge_x = net->d_edge_x.p;
  a.w16 = net->d_w16.p;
  a.code = net->packed ? nullptr : net->d_code.p;
  a.post_mask = net->packed ? 0x00FFFFFFu : 0xFFFFFFFFu;
  a.n_edges = (uint32_t)net->n_edges;
  a.seg = net->d_seg.p;
  a.seg32 = net->seg32;
  a.G = net->G;
  a.P = net->P;
  a.pbits = net->pbits;
  a.run_lo = net->d_run_lo.p;
  a.run_src0 = net->d_run_src0.p;
  a.run_post0 = net->d_run_post0.p;
  a.run_len = net->d_run_len.p;
  a.run_seed0 = net->d_run_seed0.p;
  a.run_w = net->d_run_w.p;
  a.run_p = net->d_run_p.p;
  a.run_code = net->d_run_code.p;
  a.deterministic = net->deterministic;
  a.red = net->red;
  a.red_flat = net->d_red_flat.p;
  a.red_rows = net->d_red_rows.p;
  a.red_cnt = net->d_red_cnt.p;
  a.run_off = net->d_run_off.p;
  a.n_runs = (uint32_t)net->n_runs;
  a.n_src_syn = (uint32_t)net->n_src_edges;
  a.drv_fold = net->d_drv_fold.p;
  a.src_tm = net->src_tm ? 1 : 0;
  a.run_pt = net->d_run_pt.p;
  a.src_tm_r = net->d_src_tm_r.p;
  a.src_tm_u = net->d_src_tm_u.p;
  a.src_tm_last = net->d_src_tm_last.p;
  a.tm = net->tm_edges ? 1 : 0;
  a.tm_pt = net->d_pt.p;
  a.tm_r = net->d_tm_r.p;
  a.tm_u = net->d_tm_u.p;
  a.tm_last = net->d_tm_last.p;
  a.tm_fac = 0;
  for (size_t k = 0; k < net->tm_prof.size() && k < kMaxTm; ++k) {
    a.tm_u0[k] = net->tm_prof[k].u0;
    a.tm_arec[k] = net->tm_prof[k].a_rec;
    a.tm_afac[k] = net->tm_prof[k].a_fac;
    if (net->tm_prof[k].fac) a.tm_fac |= 1u << k;
  }
  a.stdp = net->stdp_on ? 1 : 0;
  a.x_pre = net->d_x_pre.p;
  a.x_post = net->d_x_post.p;
  if (net->stdp_on) {
    a.d_pre = net->ln_consts.size() > 2 ? net->ln_consts[2] : 0.f;
    a.d_post = net->ln_consts.size() > 3 ? net->ln_consts[3] : 0.f;
  }
  a.a_plus = net->a_plus;
  a.a_minus = net->a_minus;
  a.w_min = net->w_min;
  a.w_max = net->w_max;
  a.in_ptr = net->d_in_ptr.p;
  a.in_edge = net->d_in_edge.p;
  a.in_pre = net->d_in_pre.p;
  a.drift = net->d_drift.p;
  a.learn = net->learn_on ? 1 : 0;
  a.l_tp = net->d_l_tp.p;
  a.l_tq = net->d_l_tq.p;
  a.l_dpre = net->l_dpre;
  a.l_dpost = net->l_dpost;
  for (int k = 0; k < 4; ++k) a.l_motor[k] = net->l_motor[k];
  a.l_motor_acc = net->d_l_motor.p;
  a.l_flat = net->d_l_flat.p;
  a.l_flat_cnt = net->d_l_ctr.p;
  return a;
}

// Host restatement of P/math/fast_exp.rs:23-68 (fused flavour), used for the
// per-step STDP trace decay constants (brain.rs:208-209).
float host_fast_exp(float x) {
  const float log2e = 1.44269504088896340736f;
  float t = x * log2e;
  float tf = std::floor(t);
  int n = std::isnan(tf) ? 0 : (tf >= 2147483647.0f ? 2147483647 : (tf <= -2147483648.0f ? INT32_MIN : (int)tf));
  float f = t - (float)n;
  float poly = std::fma(0.0001540353f, f, 0.001333356f);
  poly = std::fma(poly, f, 0.009618129f);
  poly = std::fma(poly, f, 0.05550411f);
  poly = std::fma(poly, f, 0.2402265f);
  poly = std::fma(poly, f, 0.693147180559945309417f);
  poly = std::fma(poly, f, 1.0f);
  if (n < -126) return 0.0f;
  if (n > 127) return INFINITY;
  uint32_t bits = (uint32_t)(n + 127) << 23;
  float s;
  std::memcpy(&s, &bits, 4);
  return s * poly;
}

// ---------------------------------------------------------------------------
// build kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t edge_post(uint2 e, int packed) { return packed ? (e.x & 0x00FFFFFFu) : e.x; }
__device__ __forceinline__ uint8_t edge_code_of(uint2 e, const uint8_t *code, uint64_t i, int packed) {
  return packed ? (uint8_t)(e.x >> 24) : code[i];
}
__global__ void sort_key_kernel(const uint32_t *pre, const uint32_t *post, unsigned long long *key, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    key[i] = ((unsigned long long)pre[i] << 32) | post[i];
}
// Segment table: entry j of row `pre` = first position in the row whose post
// is >= j*P (rows are sorted by post), entry G = row length.
template <typename T>
__global__ void seg_table_kernel(const uint32_t *row_ptr, const uint32_t *xw, uint32_t xstride, uint32_t post_mask,
                                 uint32_t Nd, uint32_t G, uint32_t P, T *seg) {
  for (uint32_t pre = blockIdx.x * blockDim.x + threadIdx.x; pre < Nd; pre += gridDim.x * blockDim.x) {
    const uint32_t beg = row_ptr[pre], end = row_ptr[pre + 1];
    T *out = seg + (size_t)pre * (G + 1);
    uint32_t lo = beg;
    for (uint32_t j = 0; j < G; ++j) {
      const uint32_t bound = j * P;
      uint32_t hi = end;
      while (lo < hi) {  // lower_bound of bound in [lo, end); no overflow past 2^31 edges
        const uint32_t mid = lo + ((hi - lo) >> 1);
        if ((xw[(size_t)mid * xstride] & post_mask) < bound) lo = mid + 1;
        else hi = mid;
      }
      out[j] = (T)(lo - beg);
    }
    out[G] = (T)(end - beg);
  }
}
__global__ void iota_kernel(uint32_t *v, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    v[i] = (uint32_t)i;
}
// Records in CSR order: edge i is staged edge perm[i] (perm null: edge i).
__global__ void gather_edges_kernel(const uint32_t *perm, const uint32_t *post_in, const float *w_in,
                                    const uint8_t *code_in, uint2 *edge, uint8_t *code, int packed, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t j = perm ? perm[i] : i;
    const uint8_t c = code_in[j];
    edge[i] = make_uint2(packed ? (post_in[j] | ((uint32_t)c << 24)) : post_in[j], __float_as_uint(w_in[j]));
    if (!packed) code[i] = c;
  }
}
__global__ void gather_u8_kernel(const uint32_t *perm, const uint8_t *in, uint8_t *out, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[perm ? perm[i] : i];
}
// Whether the staged edges are already in CSR order, (pre, post) ascending.
__global__ void sorted_check_kernel(const uint32_t *pre, const uint32_t *post, uint64_t n, int *unsorted) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i + 1 < n; i += (uint64_t)gridDim.x * blockDim.x)
    if (pre[i] > pre[i + 1] || (pre[i] == pre[i + 1] && post[i] > post[i + 1])) *unsorted = 1;
}
__global__ void histogram_kernel(const uint32_t *keys, uint64_t n, uint32_t shift, unsigned long long *cnt) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    atomicAdd(cnt + (keys[i] >> shift), 1ull);
}
__global__ void to_u32_kernel(const unsigned long long *in, uint32_t *out, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (uint32_t)in[i];
}
// Plastic in-edges grouped by post.
// in-edges per post of the plastic synapses (all = 0) or of every synapse
__global__ void csc_count_kernel(const uint32_t *row_ptr, const uint2 *edge, const uint8_t *code, int packed,
                                 uint32_t Nd, unsigned long long *cnt, int all) {
  for (uint32_t pre = blockIdx.x * blockDim.x + threadIdx.x; pre < Nd; pre += gridDim.x * blockDim.x)
    for (uint32_t e = row_ptr[pre]; e < row_ptr[pre + 1]; ++e)
      if (all || code_stdp(edge_code_of(edge[e], code, e, packed))) atomicAdd(cnt + edge_post(edge[e], packed), 1ull);
}
__global__ void csc_fill_kernel(const uint32_t *row_ptr, const uint2 *edge, const uint8_t *code, int packed,
                                uint32_t Nd, uint32_t *cursor, uint32_t *in_edge, uint32_t *in_pre, int all) {
  for (uint32_t pre = blockIdx.x * blockDim.x + threadIdx.x; pre < Nd; pre += gridDim.x * blockDim.x)
    for (uint32_t e = row_ptr[pre]; e < row_ptr[pre + 1]; ++e)
      if (all || code_stdp(edge_code_of(edge[e], code, e, packed))) {
        const uint32_t k = atomicAdd(cursor + edge_post(edge[e], packed), 1u);
        in_edge[k] = e;
        in_pre[k] = pre;
      }
}
__global__ void synth_indegree_kernel(uint32_t *pre, uint32_t *post, float *w, uint8_t *code,
                                      uint64_t base, uint32_t n_post, uint32_t k_in, uint64_t seed,
                                      uint32_t from_off, uint32_t n_from, uint32_t to_off,
                                      uint32_t n_exc, float w_exc, float w_inh, uint32_t d_min,
                                      uint32_t d_span, uint8_t st_e, uint8_t st_i, uint32_t flags_e,
                                      int recept) {
  const uint64_t total = (uint64_t)n_post * k_in;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t h = splitmix64(seed ^ (t * 0x9E3779B97F4A7C15ull));
    const uint32_t j = (uint32_t)(t / k_in);
    const uint32_t src = (uint32_t)(((h >> 32) * (uint64_t)n_from) >> 32);
    const uint32_t d = d_min + (uint32_t)((h & 0xffffffffull) % d_span);
    const bool exc = src < n_exc;
    pre[base + t] = from_off + src;
    post[base + t] = to_off + j;
    w[base + t] = exc ? w_exc : w_inh;
    code[base + t] = recept ? receptor_code(exc ? st_e : st_i)
                            : edge_code((uint8_t)d, exc ? st_e : st_i, exc && (flags_e & SG_EDGE_STDP));
  }
}

// Fixed out-degree with distinct targets (Floyd's sampling): source i draws
// k distinct targets from the m = n_to (- 1 without self-loops) candidates;
// draw q (j = m - k + q) takes t = floor(hi32(h) * (j + 1) / 2^32) in [0, j],
// or j itself when t was already drawn, h = splitmix64(seed ^ ((i*k + q) *
// 0x9E3779B97F4A7C15)); without self-loops t >= i maps to t + 1.  The weight
// is w_exc (i < n_exc) or w_inh, times lo32(h) / 2^32 when random_w.  Edges
// are written in (source, draw) order.
// With per-source degrees (deg != null) source i draws deg[i] targets into
// the edges from base + off[i]; the hash counter is then off[i] + q.
constexpr uint32_t kMaxOutDegree = 4096;
struct OutDegreeSpec {
  uint64_t seed;
  uint32_t from_off, to_off, n_to, n_exc;
  int no_self, random_w;
  float w_exc, w_inh;
  uint32_t d_min, d_span;       // delay uniform in [d_min, d_min + d_span)
  uint8_t st_exc, st_inh;       // synapse type (kinetic profile) by source class
  uint32_t flags_exc;           // SG_EDGE_STDP for excitatory sources
  int receptor;                 // st_exc / st_inh are receptor codes (receptor kinetics)
};

__global__ void synth_outdegree_kernel(uint32_t *pre, uint32_t *post, float *w, uint8_t *code, uint64_t base,
                                       uint32_t n_from, uint32_t k_fixed, const uint32_t *deg,
                                       const unsigned long long *off, OutDegreeSpec sp) {
  const uint64_t seed = sp.seed;
  const uint32_t from_off = sp.from_off, to_off = sp.to_off, n_to = sp.n_to, n_exc = sp.n_exc;
  const int no_self = sp.no_self, random_w = sp.random_w;
  const float w_exc = sp.w_exc, w_inh = sp.w_inh;
  const uint32_t m = n_to - (no_self ? 1u : 0u);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_from; i += gridDim.x * blockDim.x) {
    const bool exc = i < n_exc;
    const uint32_t k = deg ? deg[i] : k_fixed;
    const uint64_t first = deg ? (uint64_t)off[i] : (uint64_t)i * k_fixed;
    uint32_t *row = post + base + first;  // this source's targets so far (to_off + mapped draw)
    for (uint32_t q = 0; q < k; ++q) {
      const uint32_t j = m - k + q;
      const uint64_t h = splitmix64(seed ^ ((first + q) * 0x9E3779B97F4A7C15ull));
      uint32_t t = (uint32_t)(((h >> 32) * (uint64_t)(j + 1)) >> 32);
      for (uint32_t r = 0; r < q; ++r) {
        uint32_t d = row[r] - to_off;  // undo the self-loop mapping: draws are compared raw
        if (no_self && d > i) --d;
        if (d == t) {
          t = j;
          break;
        }
      }
      const uint32_t tgt = (no_self && t >= i) ? t + 1 : t;
      const float scale = exc ? w_exc : w_inh;
      const uint64_t e = base + first + q;
      pre[e] = from_off + i;
      row[q] = to_off + tgt;
      const uint32_t lo = (uint32_t)(h & 0xffffffffull);
      // random_w 1: U = lo / 2^32; random_w = b >= 2: U on the 2^-b grid (the top b bits of lo)
      const float u = random_w >= 2 ? (float)(lo >> (32 - random_w)) * __int_as_float((127 - random_w) << 23)
                                    : (float)lo * 2.3283064365386963e-10f;
      w[e] = random_w ? scale * u : scale;
      const uint32_t dly = sp.d_span > 1 ? sp.d_min + (uint32_t)(splitmix64(h) & 0xffffffffull) % sp.d_span : sp.d_min;
      code[e] = sp.receptor ? receptor_code(exc ? sp.st_exc : sp.st_inh)
                            : edge_code((uint8_t)dly, exc ? sp.st_exc : sp.st_inh, exc && (sp.flags_exc & SG_EDGE_STDP));
    }
    // the row sorted by target (shell sort; the targets are distinct), so
    // that generated edges arrive in CSR order and the build needs no sort
    float *rw = w + base + first;
    uint8_t *rc = code + base + first;
    const uint32_t gaps[] = {701, 301, 132, 57, 23, 10, 4, 1};
    for (uint32_t gap : gaps) {
      for (uint32_t a = gap; a < k; ++a) {
        const uint32_t tp = row[a];
        const float tw = rw[a];
        const uint8_t tc = rc[a];
        uint32_t b = a;
        for (; b >= gap && row[b - gap] > tp; b -= gap) {
          row[b] = row[b - gap];
          rw[b] = rw[b - gap];
          rc[b] = rc[b - gap];
        }
        row[b] = tp;
        rw[b] = tw;
        rc[b] = tc;
      }
    }
  }
}

__global__ void widen_kernel(const uint32_t *in, unsigned long long *out, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x)
    out[i] = i < n ? in[i] : 0ull;
}

// Lognormal out-degrees: deg[i] = round(exp(mu + sigma * z_i)) clipped to
// [1, kmax], z_i the FP64 Box-Muller normal of counter i (stream 7).
__global__ void lognormal_degree_kernel(uint32_t *deg, uint32_t n, uint64_t seed, double mu, double sigma,
                                        uint32_t kmax) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double k = rint(exp(mu + sigma * hash_std_normal(seed, 7, i)));
    deg[i] = (uint32_t)fmin(fmax(k, 1.0), (double)kmax);
  }
}

// Raster compaction: bitmask rows (one per recorded step) -> (step, global
// index) pairs in step-then-index order.  1024 words per block.
constexpr uint32_t kRasterWordsPerBlock = 1024;

__device__ __forceinline__ uint32_t raster_word(const uint32_t *bits, uint32_t cap, uint32_t words, uint64_t t0,
                                                uint64_t w) {
  const uint64_t t = t0 + w / words;
  return bits[(size_t)(t % cap) * words + (w % words)];
}

__global__ void raster_count_kernel(const uint32_t *bits, uint32_t cap, uint32_t words, uint64_t t0, uint64_t nw,
                                    unsigned long long *block_cnt) {
  const uint64_t w0 = (uint64_t)blockIdx.x * kRasterWordsPerBlock;
  uint32_t c = 0;
  for (uint32_t j = threadIdx.x; j < kRasterWordsPerBlock; j += blockDim.x)
    if (w0 + j < nw) c += __popc(raster_word(bits, cap, words, t0, w0 + j));
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  __shared__ uint32_t part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long tot = 0;
    for (uint32_t i = 0; i < blockDim.x / 32; ++i) tot += part[i];
    block_cnt[blockIdx.x] = tot;
  }
}

// Writes the (step, global index) pairs at their scanned offsets and adds
// one to counts[device index] per spike; does nothing when the total
// (block_off[nb]) exceeds out_cap (the caller grows the outputs and runs it
// again).
__global__ void raster_write_kernel(const uint32_t *bits, uint32_t cap, uint32_t words, uint64_t t0, uint64_t nw,
                                    const unsigned long long *block_off, uint64_t nb, uint64_t out_cap,
                                    const uint32_t *pop_dev, const uint32_t *pop_glob, int npops, uint32_t *out_step,
                                    uint32_t *out_idx, uint32_t *counts) {
  if (block_off[nb] > out_cap) return;
  // each thread owns 4 consecutive words of the block's 1024
  __shared__ uint32_t warp_tot[32];
  const uint64_t w0 = (uint64_t)blockIdx.x * kRasterWordsPerBlock + threadIdx.x * 4;
  uint32_t v[4], c = 0;
  for (int q = 0; q < 4; ++q) {
    v[q] = (w0 + q < nw) ? raster_word(bits, cap, words, t0, w0 + q) : 0u;
    c += __popc(v[q]);
  }
  // block exclusive scan of c
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t x = c;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) warp_tot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint32_t t = lane < blockDim.x / 32 ? warp_tot[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= (uint32_t)o) t += y;
    }
    warp_tot[lane] = t;  // inclusive
  }
  __syncthreads();
  unsigned long long pos = block_off[blockIdx.x] + (x - c) + (wid ? warp_tot[wid - 1] : 0);
  for (int q = 0; q < 4; ++q) {
    uint32_t m = v[q];
    if (!m) continue;
    const uint64_t w = w0 + q;
    const uint32_t step = (uint32_t)(t0 + w / words);
    const uint32_t dbase = (uint32_t)(w % words) * 32;
    // population of this word (populations are 32-aligned: one per word)
    int lo = 0, hi = npops - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (pop_dev[mid] <= dbase) lo = mid;
      else hi = mid - 1;
    }
    const uint32_t gbase = pop_glob[lo] + (dbase - pop_dev[lo]);
    while (m) {
      const uint32_t b = __ffs(m) - 1;
      m &= m - 1;
      out_step[pos] = step;
      out_idx[pos] = gbase + b;
      if (counts != nullptr) atomicAdd(counts + dbase + b, 1u);
      ++pos;
    }
  }
}

// off[s] = the first position of step t0 + s in the step-ordered out_step
// (s = 0..k; off[k] = total): a lower-bound search per step.
__global__ void raster_step_off_kernel(const uint32_t *out_step, uint64_t total, uint64_t t0, uint64_t k,
                                       uint32_t *off) {
  const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s > k) return;
  const uint32_t want = (uint32_t)(t0 + s);
  uint64_t lo = 0, hi = total;  // first position with out_step >= want
  while (lo < hi) {
    const uint64_t mid = lo + ((hi - lo) >> 1);
    if (out_step[mid] < want) lo = mid + 1;
    else hi = mid;
  }
  off[s] = (uint32_t)(s == k ? total : lo);
}

template <typename F> void launch_grid(uint64_t n, F f) {
  uint64_t blocks = (n + 255) / 256;
  if (blocks > 148ull * 32) blocks = 148ull * 32;
  if (blocks == 0) blocks = 1;
  f((unsigned)blocks);
}

// Profile ids of the staged edges up to `upto` (zero for the edges staged
// without one), once any edge carries a profile.
void fill_staged_pt(sg_net *net, uint64_t upto) {
  if (!net->tm_edges || net->e_pt.n >= upto) return;
  net->e_pt.reserve(upto, net->stream);
  SG_CUDA(cudaMemsetAsync(net->e_pt.p + net->e_pt.n, 0, upto - net->e_pt.n, net->stream));
  net->e_pt.n = upto;
}

void upload_staged_edges(sg_net *net, const uint32_t *pre, const uint32_t *post, const float *w,
                         const uint8_t *code, uint64_t n, const uint8_t *pt = nullptr) {
  const size_t n0 = net->e_pre.n;
  if (pt) {
    net->tm_edges = true;
    fill_staged_pt(net, n0);
    net->e_pt.reserve(n0 + n, net->stream);
    SG_CUDA(cudaMemcpyAsync(net->e_pt.p + n0, pt, n, cudaMemcpyHostToDevice, net->stream));
    net->e_pt.n = n0 + n;
  }
  net->e_pre.reserve(n0 + n, net->stream);
  net->e_post.reserve(n0 + n, net->stream);
  net->e_w.reserve(n0 + n, net->stream);
  net->e_code.reserve(n0 + n, net->stream);
  SG_CUDA(cudaMemcpyAsync(net->e_pre.p + n0, pre, n * 4, cudaMemcpyHostToDevice, net->stream));
  SG_CUDA(cudaMemcpyAsync(net->e_post.p + n0, post, n * 4, cudaMemcpyHostToDevice, net->stream));
  SG_CUDA(cudaMemcpyAsync(net->e_w.p + n0, w, n * 4, cudaMemcpyHostToDevice, net->stream));
  SG_CUDA(cudaMemcpyAsync(net->e_code.p + n0, code, n, cudaMemcpyHostToDevice, net->stream));
  SG_CUDA(cudaStreamSynchronize(net->stream));
  net->e_pre.n = net->e_post.n = net->e_w.n = net->e_code.n = n0 + n;
}

// Sort of the staged edges by (pre, post), stable (graph.rs:142-147 sorts by
// pre only, unstably, so the order inside a row is not part of the reference
// contract).  Keeping repeated (pre, post) synapses in insertion order keeps
// every ring cell's summation order.  Then the u32 row_ptr (graph.rs:149-180).
void build_graph(sg_net *net) {
  cudaStream_t s = net->stream;
  const uint64_t E = net->e_pre.n;
  net->n_edges = E;
  const uint32_t Nd = net->Nd;
  net->d_row_ptr.alloc((size_t)Nd + 1);
  net->packed = Nd <= (1u << 24) ? 1 : 0;
  // padded: the scatter's bulk copies widen a row to 16-byte boundaries
  net->d_edge.alloc(E + 2);
  net->d_code.alloc(net->packed ? 1 : E + 16);
  DBuf<unsigned long long> cnt;
  cnt.alloc((size_t)Nd + 1);
  cnt.zero(s);
  int unsorted = 1;
  if (E > 0) {  // edges staged in CSR order already (device generators, sources in order) need no sort
    DBuf<int> flag;
    flag.alloc(1);
    flag.zero(s);
    launch_grid(E, [&](unsigned b) { sorted_check_kernel<<<b, 256, 0, s>>>(net->e_pre.p, net->e_post.p, E, flag.p); });
    SG_CUDA(cudaMemcpyAsync(&unsorted, flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    SG_CUDA(cudaStreamSynchronize(s));
  }
  if (net->tm_edges) {
    fill_staged_pt(net, E);
    net->d_pt.alloc(std::max<uint64_t>(E, 1));
  }
  if (E > 0 && !unsorted) {
    launch_grid(E, [&](unsigned b) {
      gather_edges_kernel<<<b, 256, 0, s>>>(nullptr, net->e_post.p, net->e_w.p, net->e_code.p, net->d_edge.p,
                                            net->d_code.p, net->packed, E);
    });
    if (net->tm_edges)
      launch_grid(E, [&](unsigned b) { gather_u8_kernel<<<b, 256, 0, s>>>(nullptr, net->e_pt.p, net->d_pt.p, E); });
    launch_grid(E, [&](unsigned b) { histogram_kernel<<<b, 256, 0, s>>>(net->e_pre.p, E, 0, cnt.p); });
    SG_CUDA(cudaStreamSynchronize(s));
  } else if (E > 0) {
    DBuf<unsigned long long> keys_in, keys_out;
    DBuf<uint32_t> vals_in, vals_out;
    keys_in.alloc(E);
    keys_out.alloc(E);
    vals_in.alloc(E);
    vals_out.alloc(E);
    launch_grid(E, [&](unsigned b) { sort_key_kernel<<<b, 256, 0, s>>>(net->e_pre.p, net->e_post.p, keys_in.p, E); });
    launch_grid(E, [&](unsigned b) { iota_kernel<<<b, 256, 0, s>>>(vals_in.p, E); });
    int nb = 1;
    while (nb < 32 && (1ull << nb) < (uint64_t)Nd) ++nb;
    const int end_bit = 32 + nb;
    size_t temp_bytes = 0;
    SG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys_in.p, keys_out.p, vals_in.p, vals_out.p,
                                            (int64_t)E, 0, end_bit, s));
    DBuf<uint8_t> temp;
    temp.alloc(std::max<size_t>(temp_bytes, 1));
    SG_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, temp_bytes, keys_in.p, keys_out.p, vals_in.p, vals_out.p,
                                            (int64_t)E, 0, end_bit, s));
    temp.release();
    keys_in.release();
    keys_out.release();
    vals_in.release();
    launch_grid(E, [&](unsigned b) {
      gather_edges_kernel<<<b, 256, 0, s>>>(vals_out.p, net->e_post.p, net->e_w.p, net->e_code.p,
                                            net->d_edge.p, net->d_code.p, net->packed, E);
    });
    if (net->tm_edges)
      launch_grid(E, [&](unsigned b) { gather_u8_kernel<<<b, 256, 0, s>>>(vals_out.p, net->e_pt.p, net->d_pt.p, E); });
    launch_grid(E, [&](unsigned b) { histogram_kernel<<<b, 256, 0, s>>>(net->e_pre.p, E, 0, cnt.p); });
    SG_CUDA(cudaStreamSynchronize(s));
  }
  net->e_pre.release();
  net->e_post.release();
  net->e_w.release();
  net->e_code.release();
  net->e_pt.release();
  // exclusive scan in u64 -> u32 row_ptr
  DBuf<unsigned long long> rp64;
  rp64.alloc((size_t)Nd + 1);
  size_t tb = 0;
  SG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.p, rp64.p, (int64_t)Nd + 1, s));
  DBuf<uint8_t> temp;
  temp.alloc(std::max<size_t>(tb, 1));
  SG_CUDA(cub::DeviceScan::ExclusiveSum(temp.p, tb, cnt.p, rp64.p, (int64_t)Nd + 1, s));
  launch_grid((uint64_t)Nd + 1, [&](unsigned b) { to_u32_kernel<<<b, 256, 0, s>>>(rp64.p, net->d_row_ptr.p, (uint64_t)Nd + 1); });
  SG_CUDA(cudaStreamSynchronize(s));
}

// Scatter geometry and the per-row segment table.
// Scatter geometry: G blocks of P posts (the owner-computes scatter's post
// ranges, and the grouping of Poisson-source synapses).
void build_segments(sg_net *net) {
  const uint32_t Nd = net->Nd;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, net->device);
  uint32_t G = std::max<uint32_t>(1, std::min<uint32_t>((uint32_t)sms * kScatterBlocksPerSM, Nd / 32));
  uint32_t P = std::max<uint32_t>(32, (uint32_t)align_up((Nd + G - 1) / G, 32));
  G = std::max<uint32_t>(1, (Nd + P - 1) / P);
  net->G = G;
  net->P = P;
  uint32_t pb = 1;
  while ((1u << pb) < P) ++pb;
  net->pbits = pb;
  SG_REQUIRE(((uint64_t)(4 * kSlots) << pb) < 0xFFFFFFFFull, SG_E_INVALID, "network too large for the cell encoding");
}

// The per-row segment table of the owner-computes scatter ([Nd][G+1] record
// offsets where each block's post range starts); built when a network first
// takes that path (networks on the pre-centric scatter never need it).
void build_seg_table(sg_net *net) {
  if (net->d_seg.p) return;
  cudaStream_t s = net->stream;
  const uint32_t Nd = net->Nd, G = net->G, P = net->P;
  // longest row decides the table width
  std::vector<uint32_t> rp((size_t)Nd + 1);
  SG_CUDA(cudaMemcpyAsync(rp.data(), net->d_row_ptr.p, rp.size() * 4, cudaMemcpyDeviceToHost, s));
  SG_CUDA(cudaStreamSynchronize(s));
  uint32_t longest = 0;
  for (uint32_t i = 0; i < Nd; ++i) longest = std::max(longest, rp[i + 1] - rp[i]);
  net->seg32 = longest >= 65536 ? 1 : 0;
  const size_t esz = net->seg32 ? 4 : 2;
  net->d_seg.alloc(std::max<size_t>((size_t)Nd * (G + 1) * esz, 1));
  const bool split = net->weight_format != SG_W_F32 && !net->d_edge.p;
  const uint32_t *xw = split ? net->d_edge_x.p : reinterpret_cast<const uint32_t *>(net->d_edge.p);
  const uint32_t xstride = split ? 1u : 2u, mask = net->packed ? 0x00FFFFFFu : 0xFFFFFFFFu;
  launch_grid(Nd, [&](unsigned b) {
    if (net->seg32)
      seg_table_kernel<uint32_t><<<b, 256, 0, s>>>(net->d_row_ptr.p, xw, xstride, mask, Nd, G, P,
                                                   (uint32_t *)net->d_seg.p);
    else
      seg_table_kernel<uint16_t><<<b, 256, 0, s>>>(net->d_row_ptr.p, xw, xstride, mask, Nd, G, P,
                                                   (uint16_t *)net->d_seg.p);
  });
  SG_CUDA(cudaGetLastError());
  SG_CUDA(cudaStreamSynchronize(s));
}

// Poisson sources: rate and seed per source; their synapses grouped by the
// scatter block that owns the post, each group in (source, connect) order.
// Exponent of the lowest set bit of a nonzero finite float (w = odd * 2^e).
__host__ __device__ inline int low_exponent(uint32_t bits) {
  int ex = (int)((bits >> 23) & 0xFFu);
  uint32_t mant = bits & 0x7FFFFFu;
  if (ex) mant |= 0x800000u;
  else ex = 1;
  int tz = 0;
  while (!(mant & 1u)) {
    mant >>= 1;
    ++tz;
  }
  return ex - 150 + tz;
}

// A population whose only source synapses are one per neuron, from source
// seed0 + i onto neuron i, with one rate, one weight, delay <= 1 and ring 0,
// takes that drive in the neuron kernel (deferred drive, PopArgs::drv); its
// synapses leave the scatter.  `post_cnt` etc. are per device neuron: number
// of source synapses onto it, and the source, weight and code of the last one.
void find_deferred_drive(sg_net *net, const std::vector<uint32_t> &post_cnt, const std::vector<uint32_t> &post_src,
                         const std::vector<float> &post_w, const std::vector<uint8_t> &post_code,
                         const std::vector<uint8_t> &post_pt, std::vector<uint8_t> &deferred) {
  net->any_drv = false;
  for (auto &pop : net->pops) {
    pop.drv = false;
    if (pop.external || pop.n == 0) continue;
    const uint32_t q0 = pop.dev_off;
    if (post_cnt[q0] != 1) continue;
    const HostSrc &s0 = net->srcs[post_src[q0]];
    const float w0 = post_w[q0];
    bool ok = true;
    for (uint32_t i = 0; i < pop.n && ok; ++i) {
      const uint32_t q = q0 + i;
      const uint8_t c = post_code[q];
      const HostSrc &sr = net->srcs[post_src[q]];
      ok = post_cnt[q] == 1 && code_delay(c) <= 1 && code_ring(c) == 0 && !code_stdp(c) && post_pt[q] == 0 &&
           std::memcmp(&post_w[q], &w0, 4) == 0 && std::memcmp(&sr.p, &s0.p, 4) == 0 && sr.seed == s0.seed + i;
    }
    if (!ok) continue;
    pop.drv = true;
    pop.drv_seed0 = s0.seed;
    pop.drv_p = s0.p;
    pop.drv_w = w0;
    net->any_drv = true;
    std::fill(deferred.begin() + q0, deferred.begin() + q0 + pop.n, (uint8_t)1);
  }
}

void build_sources(sg_net *net) {
  const size_t S = net->srcs.size();
  const uint32_t G = net->G, P = net->P;
  std::vector<float> p(S);
  std::vector<uint32_t> seed(S);
  for (size_t i = 0; i < S; ++i) {
    p[i] = net->srcs[i].p;
    seed[i] = net->srcs[i].seed;
  }
  // the source synapses in the reference's order: source ascending, then
  // connect order (a counting sort by source, stable)
  const std::vector<SrcSyn> &syn = net->src_syn;
  std::vector<uint32_t> ord(syn.size());
  {
    std::vector<uint64_t> start(S + 1, 0);
    for (const SrcSyn &y : syn) start[y.src + 1]++;
    for (size_t i = 0; i < S; ++i) start[i + 1] += start[i];
    for (size_t k = 0; k < syn.size(); ++k) ord[start[syn[k].src]++] = (uint32_t)k;
  }
  std::vector<uint64_t> cnt((size_t)G + 1, 0);
  uint64_t tot = 0;
  // the source weights' part of the exact-sum test (rings_exact)
  net->src_abs.assign(net->Nd, 0.0);
  net->src_lo = 1 << 20;
  net->src_bad = false;
  std::vector<uint8_t> deferred;
  if (!syn.empty()) {
    std::vector<uint32_t> post_cnt(net->Nd, 0), post_src(net->Nd, 0);
    std::vector<float> post_w(net->Nd, 0.0f);
    std::vector<uint8_t> post_code(net->Nd, 0), post_pt(net->Nd, 0);
    for (const SrcSyn &y : syn) {
      post_cnt[y.post]++;
      post_src[y.post] = y.src;
      post_w[y.post] = y.w;
      post_code[y.post] = y.code;
      post_pt[y.post] = y.pt;
    }
    deferred.assign(net->Nd, 0);
    find_deferred_drive(net, post_cnt, post_src, post_w, post_code, post_pt, deferred);
  } else {
    net->any_drv = false;
    for (auto &pop : net->pops) pop.drv = false;
  }
  for (const SrcSyn &y : syn) {
    uint32_t bits;
    std::memcpy(&bits, &y.w, 4);
    if (!std::isfinite(y.w)) {
      net->src_bad = true;
    } else if (bits & 0x7FFFFFFFu) {
      net->src_lo = std::min(net->src_lo, low_exponent(bits));
      net->src_abs[y.post] += std::fabs((double)y.w);
    }
    if (deferred[y.post]) continue;  // taken by the neuron kernel
    cnt[y.post / P]++;
    tot++;
  }
  SG_REQUIRE(tot < 0xFFFFFFFFull, SG_E_OVERFLOW, "too many Poisson-source synapses");
  std::vector<uint32_t> lo((size_t)G + 1, 0);
  for (uint32_t j = 0; j < G; ++j) lo[j + 1] = lo[j] + (uint32_t)cnt[j];
  std::vector<uint32_t> cur(lo.begin(), lo.end() - 1), se_src(tot), se_post(tot);
  std::vector<float> se_w(tot);
  std::vector<uint8_t> se_code(tot), se_pt(tot, 0);
  for (uint32_t k : ord) {
    const SrcSyn &y = syn[k];
    if (deferred[y.post]) continue;
    const uint32_t pos = cur[y.post / P]++;
    se_src[pos] = y.src;
    se_post[pos] = y.post;
    se_w[pos] = y.w;
    se_code[pos] = y.code;
    se_pt[pos] = y.pt;
  }
  // run-length encoding per block (runs never cross blocks; <= 2^20 long)
  std::vector<uint32_t> run_lo((size_t)G + 1, 0), r_src0, r_post0, r_len, r_seed0;
  std::vector<float> r_w, r_p;
  std::vector<uint8_t> r_code, r_pt;
  for (uint32_t jb = 0; jb < G; ++jb) {
    run_lo[jb] = (uint32_t)r_len.size();
    for (uint32_t e = lo[jb]; e < lo[jb + 1]; ++e) {
      const uint32_t src = se_src[e];
      const bool extend = e > lo[jb] && !r_len.empty() && r_len.back() < (1u << 20) &&
                          src == r_src0.back() + r_len.back() && se_post[e] == r_post0.back() + r_len.back() &&
                          seed[src] == r_seed0.back() + r_len.back() &&
                          std::memcmp(&se_w[e], &r_w.back(), 4) == 0 && se_code[e] == r_code.back() &&
                          se_pt[e] == r_pt.back() && std::memcmp(&p[src], &r_p.back(), 4) == 0;
      if (extend) {
        r_len.back()++;
      } else {
        r_src0.push_back(src);
        r_post0.push_back(se_post[e]);
        r_len.push_back(1);
        r_seed0.push_back(seed[src]);
        r_w.push_back(se_w[e]);
        r_p.push_back(p[src]);
        r_code.push_back(se_code[e]);
        r_pt.push_back(se_pt[e]);
      }
    }
  }
  run_lo[G] = (uint32_t)r_len.size();
  net->n_runs = r_len.size();
  net->n_src_edges = tot;
  std::vector<uint32_t> r_off(r_len.size() + 1, 0);  // the pre-centric scatter's run offsets
  for (size_t r = 0; r < r_len.size(); ++r) r_off[r + 1] = r_off[r] + r_len[r];
  auto up = [&](auto &buf, const auto &vec) {
    using T = typename std::decay_t<decltype(vec)>::value_type;
    buf.alloc(std::max<size_t>(vec.size(), 1));
    if (!vec.empty()) SG_CUDA(cudaMemcpyAsync(buf.p, vec.data(), vec.size() * sizeof(T), cudaMemcpyHostToDevice, net->stream));
  };
  up(net->d_run_lo, run_lo);
  up(net->d_run_src0, r_src0);
  up(net->d_run_post0, r_post0);
  up(net->d_run_len, r_len);
  up(net->d_run_seed0, r_seed0);
  up(net->d_run_w, r_w);
  up(net->d_run_p, r_p);
  up(net->d_run_code, r_code);
  up(net->d_run_off, r_off);
  // Tsodyks-Markram on source synapses (core.rs:372-378): R = 1, U = U0 of
  // the profile, last = 0, per source synapse in run order
  net->src_tm = std::any_of(se_pt.begin(), se_pt.end(), [](uint8_t v) { return v != 0; });
  if (net->src_tm) {
    std::vector<float> r0(tot, 1.0f), u0(tot, 0.0f);
    for (size_t e = 0; e < tot; ++e)
      if (se_pt[e]) u0[e] = net->tm_prof[se_pt[e] - 1].u0;
    up(net->d_run_pt, r_pt);
    up(net->d_src_tm_r, r0);
    up(net->d_src_tm_u, u0);
    net->d_src_tm_last.alloc(std::max<uint64_t>(tot, 1));
    net->d_src_tm_last.zero(net->stream);
  }
  SG_CUDA(cudaStreamSynchronize(net->stream));
  std::vector<SrcSyn>().swap(net->src_syn);  // the host copy is no longer needed
}

// In-edges per post (CSC over the CSR records): in_ptr [Nd+1], and per
// in-edge its record index and pre; `all` = every synapse, else the plastic ones.
void build_in_edges(sg_net *net, int all, DBuf<uint32_t> &in_ptr, DBuf<uint32_t> &in_edge, DBuf<uint32_t> &in_pre) {
  cudaStream_t s = net->stream;
  const uint32_t Nd = net->Nd;
  DBuf<unsigned long long> cnt, ip64;
  cnt.alloc((size_t)Nd + 1);
  cnt.zero(s);
  launch_grid(Nd, [&](unsigned b) {
    csc_count_kernel<<<b, 256, 0, s>>>(net->d_row_ptr.p, net->d_edge.p, net->d_code.p, net->packed, Nd, cnt.p, all);
  });
  ip64.alloc((size_t)Nd + 1);
  size_t tb = 0;
  SG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.p, ip64.p, (int64_t)Nd + 1, s));
  DBuf<uint8_t> temp;
  temp.alloc(std::max<size_t>(tb, 1));
  SG_CUDA(cub::DeviceScan::ExclusiveSum(temp.p, tb, cnt.p, ip64.p, (int64_t)Nd + 1, s));
  in_ptr.alloc((size_t)Nd + 1);
  launch_grid((uint64_t)Nd + 1, [&](unsigned b) { to_u32_kernel<<<b, 256, 0, s>>>(ip64.p, in_ptr.p, (uint64_t)Nd + 1); });
  unsigned long long n_in = 0;
  SG_CUDA(cudaMemcpyAsync(&n_in, ip64.p + Nd, 8, cudaMemcpyDeviceToHost, s));
  SG_CUDA(cudaStreamSynchronize(s));
  in_edge.alloc(std::max<unsigned long long>(n_in, 1));
  in_pre.alloc(std::max<unsigned long long>(n_in, 1));
  DBuf<uint32_t> cursor;
  cursor.alloc((size_t)Nd + 1);
  SG_CUDA(cudaMemcpyAsync(cursor.p, in_ptr.p, ((size_t)Nd + 1) * 4, cudaMemcpyDeviceToDevice, s));
  launch_grid(Nd, [&](unsigned b) {
    csc_fill_kernel<<<b, 256, 0, s>>>(net->d_row_ptr.p, net->d_edge.p, net->d_code.p, net->packed, Nd, cursor.p,
                                      in_edge.p, in_pre.p, all);
  });
  SG_CUDA(cudaStreamSynchronize(s));
}

void build_stdp(sg_net *net) {
  cudaStream_t s = net->stream;
  const uint32_t Nd = net->Nd;
  net->d_x_pre.alloc(Nd);
  net->d_x_pre.zero(s);
  net->d_x_post.alloc(Nd);
  net->d_x_post.zero(s);
  net->d_drift.alloc(1);
  net->d_drift.zero(s);
  build_in_edges(net, 0, net->d_in_ptr, net->d_in_edge, net->d_in_pre);
  net->ln_consts.resize(4);
  net->ln_consts[2] = host_fast_exp(-net->stdp_dt / net->tau_pre);
  net->ln_consts[3] = host_fast_exp(-net->stdp_dt / net->tau_post);
}

void compute_uniform(HostPop &p) {
  p.umask = 0;
  for (uint32_t c = 0; c < p.np && c < 16; ++c) {
    const float *col = p.params.data() + (size_t)c * p.cap;
    bool uni = p.n > 0;
    for (uint32_t i = 1; i < p.n && uni; ++i) uni = std::memcmp(&col[i], &col[0], 4) == 0;
    if (uni) {
      p.umask |= 1u << c;
      p.uval[c] = col[0];
    }
  }
}

// f32 -> bf16 by round to nearest even (finite inputs; weights are checked)
__global__ void split_bf16_kernel(const uint2 *edge, uint32_t *ex, uint16_t *w16, uint64_t E) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint2 r = edge[e];
    ex[e] = r.x;
    w16[e] = (uint16_t)((r.y + 0x7FFFu + ((r.y >> 16) & 1u)) >> 16);
  }
}

// BF16 weight storage: after the segment table is built from the records,
// split them into x words and bf16 weights and free the 8-byte records.
void split_bf16(sg_net *net) {
  if (net->weight_format != SG_W_BF16) return;
  SG_REQUIRE(!net->stdp_on, SG_E_INVALID, "BF16 weights are read-only: pair STDP needs FP32 weights");
  const uint64_t E = net->n_edges;
  cudaStream_t s = net->stream;
  net->d_edge_x.alloc(E + 4);  // padded for the scatter's 16-byte bulk copies
  net->d_w16.alloc(E + 8);
  if (E) {
    const unsigned b = (unsigned)std::min<uint64_t>((E + 255) / 256, 148u * 32u);
    split_bf16_kernel<<<b, 256, 0, s>>>(net->d_edge.p, net->d_edge_x.p, net->d_w16.p, E);
    SG_CUDA(cudaGetLastError());
  }
  SG_CUDA(cudaStreamSynchronize(s));
  net->d_edge.release();
}

// FP8 E4M3 weight storage, one warp per row: scale = max|w| of the row times
// 2^-8 (a power-of-two factor, so the row's largest weight is 256 * scale
// exactly), each weight rounded to the nearest E4M3 value of w / scale (ties
// to even, saturating at 448).  The records' weights become the decoded
// values (E4M3 value * scale in FP32), which the exact-sum test then scans
// before the 8-byte records are freed.
__global__ void split_fp8_kernel(const uint32_t *row_ptr, uint2 *edge, uint32_t *ex, uint8_t *w8, float *scale,
                                 uint32_t Nd) {
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < Nd; r += (gridDim.x * blockDim.x) >> 5) {
    const uint32_t b = row_ptr[r], e = row_ptr[r + 1];
    float mx = 0.0f;
    for (uint32_t k = b + lane; k < e; k += 32) mx = fmaxf(mx, fabsf(__uint_as_float(edge[k].y)));
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const float sc = mx * 0.00390625f;  // 2^-8
    if (lane == 0) scale[r] = sc;
    for (uint32_t k = b + lane; k < e; k += 32) {
      const uint2 rec = edge[k];
      const float w = __uint_as_float(rec.y);
      const __nv_fp8_e4m3 q(sc > 0.0f ? w / sc : 0.0f);
      const float dq = sc > 0.0f ? (float)q * sc : 0.0f;
      ex[k] = rec.x;
      w8[k] = (uint8_t)q.__x;
      edge[k].y = __float_as_uint(dq);
    }
  }
}

void split_fp8(sg_net *net) {
  if (net->weight_format != SG_W_FP8) return;
  SG_REQUIRE(!net->stdp_on, SG_E_INVALID, "FP8 weights are read-only: pair STDP needs FP32 weights");
  const uint64_t E = net->n_edges;
  cudaStream_t s = net->stream;
  net->d_edge_x.alloc(E + 4);  // padded for the scatter's 16-byte bulk copies
  net->d_w8.alloc(E + 16);
  net->d_row_scale.alloc(std::max<uint32_t>(net->Nd, 1));
  if (E) {
    split_fp8_kernel<<<148u * 8u, 256, 0, s>>>(net->d_row_ptr.p, net->d_edge.p, net->d_edge_x.p, net->d_w8.p,
                                               net->d_row_scale.p, net->Nd);
    SG_CUDA(cudaGetLastError());
  }
  SG_CUDA(cudaStreamSynchronize(s));
}

// E4M3 byte -> FP32 on the host (sign, 4-bit exponent with bias 7, 3-bit
// mantissa; exponent 0 subnormal; S.1111.111 NaN).
float host_e4m3(uint8_t b) {
  const int ex = (b >> 3) & 15, m = b & 7;
  float v;
  if (ex == 15 && m == 7) v = NAN;
  else if (ex == 0) v = std::ldexp((float)m, -9);
  else v = std::ldexp(1.0f + (float)m / 8.0f, ex - 7);
  return (b & 0x80) ? -v : v;
}

__global__ void tm_init_kernel(const uint8_t *pt, const float *u0, float *r, float *u, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    r[i] = 1.0f;
    u[i] = pt[i] ? u0[pt[i] - 1] : 0.0f;
  }
}

// Synapses into each scatter block's posts (the most events the block can
// take from spiking rows in one step), summed over the segment table.
template <class T>
__global__ void block_indeg_kernel(const T *seg, uint32_t Nd, uint32_t G, unsigned long long *out) {
  extern __shared__ unsigned long long hist[];
  for (uint32_t g = threadIdx.x; g < G; g += blockDim.x) hist[g] = 0;
  __syncthreads();
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < Nd; i += (uint64_t)gridDim.x * blockDim.x) {
    const T *t = seg + i * (G + 1);
    for (uint32_t g = 0; g < G; ++g) {
      const uint32_t l = (uint32_t)(t[g + 1] - t[g]);
      if (l) atomicAdd(&hist[g], (unsigned long long)l);
    }
  }
  __syncthreads();
  for (uint32_t g = threadIdx.x; g < G; g += blockDim.x)
    if (hist[g]) atomicAdd(&out[g], hist[g]);
}

// Weight scan for the exact-sum test: per post the sum of |w| over its
// synapses (FP64), the smallest low-bit exponent of any weight, and whether
// any weight is not finite.
__global__ void weight_scan_kernel(const uint2 *edge, const uint32_t *edge_x, const uint16_t *w16, int bf16,
                                   uint64_t E, uint32_t post_mask, double *sum, int *emin, int *bad) {
  int lo = 1 << 20;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t x = bf16 ? edge_x[e] : edge[e].x;
    const uint32_t bits = bf16 ? (uint32_t)w16[e] << 16 : edge[e].y;
    const float w = __uint_as_float(bits);
    if (!isfinite(w)) {
      atomicOr(bad, 1);
      continue;
    }
    if (bits & 0x7FFFFFFFu) {
      lo = min(lo, low_exponent(bits));
      atomicAdd(&sum[x & post_mask], fabs((double)w));
    }
  }
  for (int o = 16; o > 0; o >>= 1) lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
  if ((threadIdx.x & 31) == 0) atomicMin(emin, lo);
}

// Whether float addition on the rings is exact: every weight that reaches a
// ring (synapses and Poisson sources) is a multiple of 2^e for the smallest
// low-bit exponent e, and no post's weights sum in magnitude to 2^(23+e).
// A ring cell is cleared to +0 and receives each of its post's synapses at
// most once before it is read (a synapse reaches one slot per emission
// step, and a slot is read before the same synapse can reach it again), so
// every partial sum is a multiple of 2^e below 2^(23+e) in magnitude: exact.
// Plastic synapses change their weights, so STDP rules it out.
bool rings_exact(sg_net *net) {
  if (net->stdp_on || net->tm_edges || net->src_tm) return false;  // weights change, or are scaled by R*U
  cudaStream_t s = net->stream;
  const uint32_t Nd = net->Nd;
  if (net->src_bad) return false;
  std::vector<double> psum(std::move(net->src_abs));  // recorded by build_sources
  psum.resize(Nd, 0.0);
  int lo = net->src_lo;
  DBuf<double> sum;
  sum.alloc(std::max<uint32_t>(Nd, 1));
  SG_CUDA(cudaMemcpyAsync(sum.p, psum.data(), (size_t)Nd * 8, cudaMemcpyHostToDevice, s));
  DBuf<int> flags;
  flags.alloc(2);
  const int init[2] = {1 << 20, 0};
  SG_CUDA(cudaMemcpyAsync(flags.p, init, sizeof(init), cudaMemcpyHostToDevice, s));
  const uint64_t E = net->n_edges;
  const int bf16 = net->weight_format == SG_W_BF16 ? 1 : 0;
  if (E) {
    const unsigned b = (unsigned)std::min<uint64_t>((E + 255) / 256, 148u * 16u);
    weight_scan_kernel<<<b, 256, 0, s>>>(net->d_edge.p, net->d_edge_x.p, net->d_w16.p, bf16, E,
                                         net->packed ? 0x00FFFFFFu : 0xFFFFFFFFu, sum.p, flags.p, flags.p + 1);
    SG_CUDA(cudaGetLastError());
  }
  int h[2];
  SG_CUDA(cudaMemcpyAsync(psum.data(), sum.p, (size_t)Nd * 8, cudaMemcpyDeviceToHost, s));
  SG_CUDA(cudaMemcpyAsync(h, flags.p, sizeof(h), cudaMemcpyDeviceToHost, s));
  SG_CUDA(cudaStreamSynchronize(s));
  if (h[1]) return false;
  lo = std::min(lo, h[0]);
  double most = 0.0;
  for (double v : psum) most = std::max(most, v);
  if (most == 0.0) return true;
  return most < std::ldexp(1.0, 23 + lo);
}

void drop_graph(sg_net *net);

// The scatter path: the pre-centric scatter (scatter_red_kernel) when the
// ring sums are exact (any order of the adds gives the reference's bits) or
// the order is not fixed (sg_set_deterministic(0)); the ordered owner-computes
// scatter otherwise.
// The device copy of the step arguments, refreshed when they change (before
// a graph is captured: the launches read it through a stable pointer).
void upload_args(sg_net *net, const StepArgs &a) {
  if (net->args_uploaded && std::memcmp(&a, &net->h_args, sizeof(StepArgs)) == 0) return;
  if (!net->d_args.n) net->d_args.alloc(1);
  net->h_args = a;
  SG_CUDA(cudaMemcpyAsync(net->d_args.p, &net->h_args, sizeof(StepArgs), cudaMemcpyHostToDevice, net->stream));
  net->args_uploaded = true;
}

// The pre-centric scatter's schedules (stages x synapses per stage), the
// first being the fixed one; sg_autotune picks one per network, with the
// blocks per SM.
// (4 x 1024, 8 x 512, 3 x 2048, 6 x 512: launch_step_red), and the warp walk
// without stages (scatter_walk_kernel): variant 4 loads and reduces a round
// at a time (8 records per lane), variants 5 and 6 load the next round's
// records (4 or 8 per lane) before reducing the current one, variant 7 cuts
// every row into 4 pieces that different warps walk, variant 8 does that
// with 4 records per lane and 6 blocks per SM (48 warps).
constexpr int kNumRedVariants = 9;
constexpr int kWalkVariant = 4;
constexpr int kWalkPipeVariant = 5;
bool is_walk_variant(int v) { return v >= kWalkVariant; }

template <uint32_t ST, uint32_t CH> void allow_red_smem_v() {
  SG_CUDA(cudaFuncSetAttribute(scatter_red_kernel<ST, CH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(RedSmemT<ST, CH>)));
}
// The stage rings exceed the 48 KB default of shared memory: allowed once
// per device before the first launch.
void allow_red_smem() {
  allow_red_smem_v<4, 1024>();
  allow_red_smem_v<8, 512>();
  allow_red_smem_v<3, 2048>();
  allow_red_smem_v<6, 512>();
}

unsigned sm_count(int device) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return (unsigned)sms;
}

void launch_step_red(cudaStream_t s, int device, int variant, uint32_t bps, const StepArgs *nets, uint32_t n_nets,
                     uint32_t *done, uint32_t *err, uint32_t stall, int fmt);
// The weight storage of a network as the walk's compile-time forms name it:
// 1 FP32 records, 2 BF16, 3 FP8, each with the code byte in the x word; 0
// with a separate code array.
int walk_format(const StepArgs &a) {
  if (a.code != nullptr) return 0;
  return a.wbf16 ? 2 : a.wfp8 ? 3 : 1;
}

// The schedule a network or pool starts with: SG_RED_VARIANT (0..8) when set,
// else the warp walk.
int default_red_variant() {
  static const int v = [] {
    const char *e = std::getenv("SG_RED_VARIANT");
    const int x = e ? std::atoi(e) : kWalkVariant;
    return x >= 0 && x < kNumRedVariants ? x : kWalkVariant;
  }();
  return v;
}

void update_path(sg_net *net) {
  // the pre-centric scatter applies neither pair STDP nor short-term
  // plasticity: those networks keep the owner-computes scatter in any mode
  const bool plain = !net->stdp_on && !net->tm_edges && !net->src_tm && !net->receptor;
  const int red = plain && (!net->deterministic || net->exact) ? 1 : 0;
  if (red != net->red) drop_graph(net);
  net->red = red;
  if (!red) build_seg_table(net);
}

void setup_scatter(sg_net *net) {
  cudaStream_t s = net->stream;
  net->exact = net->Nd > 0 && rings_exact(net);
  net->d_red_flat.alloc(std::max<uint32_t>(net->Nd, 1));
  net->d_red_rows.alloc(std::max<uint32_t>(net->Nd, 1));
  net->d_red_cnt.alloc(1);
  net->d_red_cnt.zero(s);
  net->d_drv_fold.alloc(1);
  net->d_err.alloc(1);
  net->d_err.zero(s);
  const unsigned long long none = ~0ull;
  SG_CUDA(cudaMemcpyAsync(net->d_drv_fold.p, &none, sizeof(none), cudaMemcpyHostToDevice, s));
  SG_CUDA(cudaStreamSynchronize(s));
  net->drv_folded = none;
  update_path(net);
}

// Before anything reads or adds to the ring between steps (inject_current,
// a ring readback): the deferred drive of the last step goes to the ring,
// where the reference holds it, and the next neuron kernel leaves it out.
void fold_drive(sg_net *net) {
  if (!net->any_drv || !net->built) return;
  const unsigned long long t = net->host_step;
  if (t == 0 || net->drv_folded == t - 1) return;
  for (const auto &p : net->pops) {
    if (!p.drv || p.n == 0) continue;
    PopArgs pa{};
    pa.n = p.n;
    pa.dev_off = p.dev_off;
    pa.drv = 1;
    pa.drv_seed0 = p.drv_seed0;
    pa.drv_p = p.drv_p;
    pa.drv_w = p.drv_w;
    const unsigned blocks = (unsigned)std::min<uint64_t>((p.n + 255) / 256, 148u * 8u);
    drive_fold_kernel<<<blocks, 256, 0, net->stream>>>(net->d_ring.p, net->Nd, net->nslots, t, pa, net->d_drv_fold.p);
  }
  SG_CUDA(cudaGetLastError());
  net->drv_folded = t - 1;
}

// Emptying the rings also drops the deferred drive of the last step.
void drop_drive(sg_net *net) {
  if (!net->any_drv || !net->built || net->host_step == 0) return;
  const unsigned long long v = net->host_step - 1;
  SG_CUDA(cudaMemcpyAsync(net->d_drv_fold.p, &v, sizeof(v), cudaMemcpyHostToDevice, net->stream));
  SG_CUDA(cudaStreamSynchronize(net->stream));
  net->drv_folded = v;
}

void finish_build(sg_net *net) {
  cudaStream_t s = net->stream;
  const uint32_t Nd = net->Nd;
  SG_REQUIRE(net->kin.size() <= 3, SG_E_INVALID, "at most 3 kinetic profiles are supported on the device path");
  // populations -> device
  for (auto &p : net->pops) {
    compute_uniform(p);
    p.d_params.alloc(std::max<size_t>(p.params.size(), 1));
    p.d_state.alloc(std::max<size_t>(p.state.size(), 1));
    if (!p.params.empty())
      SG_CUDA(cudaMemcpyAsync(p.d_params.p, p.params.data(), p.params.size() * 4, cudaMemcpyHostToDevice, s));
    if (!p.state.empty())
      SG_CUDA(cudaMemcpyAsync(p.d_state.p, p.state.data(), p.state.size() * 4, cudaMemcpyHostToDevice, s));
  }
  SG_CUDA(cudaStreamSynchronize(s));
  for (auto &p : net->pops) {
    std::vector<float>().swap(p.params);
    std::vector<float>().swap(p.state);
  }
  const size_t n_rings = 1 + net->kin.size();
  // a step's events land at most max(delay, 1) steps ahead, so that many
  // slots plus the one being read hold every pending arrival
  net->nslots = net->receptor ? 1u + kReceptors : std::max<uint32_t>(net->max_delay, 1u) + 1u;
  net->d_ring.alloc(std::max<size_t>(n_rings * net->nslots * Nd, 1));
  net->d_ring.zero(s);
  net->d_kin_g.alloc(std::max<size_t>(net->kin.size() * 3 * Nd, 1));  // up to 3 state arrays per profile
  net->d_kin_g.zero(s);
  net->d_step.alloc(2);  // [step counter, step hint] (hint_load / hint_store in step_kernels.cuh)
  net->d_step.zero(s);
  net->d_blk_cnt.alloc(std::max<uint32_t>(Nd / kNeuronBlock, 1));
  net->d_blk_cnt.zero(s);
  net->d_spk.alloc(std::max<uint32_t>(Nd, 1));
  net->d_last_bits.alloc(std::max<uint32_t>(Nd / 32, 1));
  net->d_last_bits.zero(s);
  net->d_done.alloc(1);
  net->d_done.zero(s);
  net->d_ev_step.alloc(1);
  net->d_ev_step.zero(s);
  net->d_ev_total.alloc(1);
  net->d_ev_total.zero(s);
  net->d_ev_src.alloc(2);
  net->d_ev_src.zero(s);
  net->d_clamp.alloc(1);
  net->d_clamp.zero(s);
  net->d_stat_spk.alloc(net->stat_cap);
  net->d_stat_spk.zero(s);
  net->d_stat_ev.alloc(net->stat_cap);
  net->d_stat_ev.zero(s);
  net->scatter_smem = sizeof(ScatterSmem);
  const int sm = (int)net->scatter_smem;
  SG_CUDA(cudaFuncSetAttribute(scatter_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  SG_CUDA(cudaFuncSetAttribute(scatter_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  allow_red_smem();
  setup_scatter(net);
  if (net->weight_format == SG_W_FP8) net->d_edge.release();  // scanned by the exact-sum test; x + E4M3 + scale from here
  if (net->tm_edges) {  // build.rs:69-84: R = 1, U = U0 of the edge's profile, last = 0
    const uint64_t E = std::max<uint64_t>(net->n_edges, 1);
    net->d_tm_r.alloc(E);
    net->d_tm_u.alloc(E);
    net->d_tm_last.alloc(E);
    net->d_tm_last.zero(s);
    float u0[kMaxTm] = {};
    for (size_t k = 0; k < net->tm_prof.size(); ++k) u0[k] = net->tm_prof[k].u0;
    DBuf<float> d_u0;
    d_u0.alloc(kMaxTm);
    SG_CUDA(cudaMemcpyAsync(d_u0.p, u0, sizeof(u0), cudaMemcpyHostToDevice, s));
    launch_grid(E, [&](unsigned b) { tm_init_kernel<<<b, 256, 0, s>>>(net->d_pt.p, d_u0.p, net->d_tm_r.p, net->d_tm_u.p, E); });
    SG_CUDA(cudaGetLastError());
    SG_CUDA(cudaStreamSynchronize(s));
  }
  SG_CUDA(cudaStreamSynchronize(s));
  net->built = true;
}

// Uploads the neuron work table (after build and after a parameter column
// changed its uniform/non-uniform status), ordered on the network's stream.
void upload_pop_table(sg_net *net) {
  if (!net->pop_tab_dirty) return;
  std::vector<PopArgs> tab(net->pops.size());
  std::vector<uint2> map;
  for (size_t i = 0; i < net->pops.size(); ++i) {
    const HostPop &p = net->pops[i];
    PopArgs &pa = tab[i];
    pa.state = p.d_state.p;
    pa.params = p.d_params.p;
    pa.n = p.n;
    pa.cap = p.cap;
    pa.dev_off = p.dev_off;
    pa.umask = p.umask;
    for (int c = 0; c < 16; ++c) pa.uval[c] = p.uval[c];
    pa.ln_na = net->ln_consts[0];
    pa.ln_k = net->ln_consts[1];
    pa.noise = p.noise ? 1 : 0;
    pa.noise_stream = p.noise_stream;
    pa.noise_split = p.noise_split;
    pa.noise_seed = p.noise_seed;
    pa.noise_stride = p.noise_stride;
    pa.noise_step0 = p.noise_step0;
    pa.noise_sigma[0] = p.noise_sigma[0];
    pa.noise_sigma[1] = p.noise_sigma[1];
    pa.bias = p.d_bias.n ? p.d_bias.p : nullptr;
    pa.drv = p.drv ? 1 : 0;
    pa.drv_seed0 = p.drv_seed0;
    pa.drv_p = p.drv_p;
    pa.drv_w = p.drv_w;
  }
  for (int m = 1; m <= 4; ++m) {
    net->model_blk_off[m] = (uint32_t)map.size();
    int n_pops = 0, last = -1;
    for (size_t i = 0; i < net->pops.size(); ++i) {
      const HostPop &p = net->pops[i];
      if (p.model != m || p.n == 0) continue;
      ++n_pops;
      last = (int)i;
      for (uint32_t b = 0; b < p.cap / kNeuronBlock; ++b) map.push_back(make_uint2((uint32_t)i, b));
    }
    net->model_blk_cnt[m] = (uint32_t)map.size() - net->model_blk_off[m];
    net->model_single[m] = n_pops == 1 ? last : -1;
  }
  net->pop_tab = tab;
  if (net->d_pop_tab.n < tab.size()) net->d_pop_tab.alloc(std::max<size_t>(tab.size(), 1));
  if (net->d_blk_map.n < map.size()) net->d_blk_map.alloc(std::max<size_t>(map.size(), 1));
  if (!tab.empty())
    SG_CUDA(cudaMemcpyAsync(net->d_pop_tab.p, tab.data(), tab.size() * sizeof(PopArgs), cudaMemcpyHostToDevice,
                            net->stream));
  if (!map.empty())
    SG_CUDA(cudaMemcpyAsync(net->d_blk_map.p, map.data(), map.size() * sizeof(uint2), cudaMemcpyHostToDevice,
                            net->stream));
  SG_CUDA(cudaStreamSynchronize(net->stream));
  net->pop_tab_dirty = false;
}

// Launches a step kernel with programmatic stream serialization: it may
// start while the stream's previous kernel drains (the kernels call
// pdl_wait() before touching what earlier kernels wrote).  Off when
// SG_NO_PDL is set in the environment (the plain launch order).
bool use_pdl() {
  static const bool on = std::getenv("SG_NO_PDL") == nullptr;
  return on;
}
template <typename... KArgs, typename... Args>
void launch_step_kernel(void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t s,
                        Args &&...args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = use_pdl() ? 1 : 0;
  SG_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
}

// L2 residency of the delay rings.  Both scatters add events into the rings
// in L2 with the evict_last priority (random 4-byte reductions, or the
// ordered path's loads and stores) while the spiking rows' records stream
// through L2 with evict_first.  Lines marked evict_last are kept only within
// the L2 set-aside for persisting accesses, which is empty by default, so
// this process's context reserves up to the rings' size (at most the
// device's maximum: 79 MiB of the B200's 126 MB L2) once a network steps
// (the sum of the rings of every network that has stepped on the device).
// The set-aside is a limit of this process's CUDA context on the device (it
// ends with the context) and is put back to its earlier value when the last
// network that reserved it is destroyed.  SG_L2_PERSIST=0 leaves it alone.
bool l2_setaside_on() {
  static const bool on = [] {
    const char *e = std::getenv("SG_L2_PERSIST");
    return e == nullptr || std::atoi(e) != 0;
  }();
  return on;
}
constexpr int kMaxDevices = 64;
std::mutex g_l2_mu;
int g_l2_refs[kMaxDevices];
size_t g_l2_saved[kMaxDevices];
size_t g_l2_rings[kMaxDevices];  // ring bytes of the networks holding a share

void setup_l2_setaside(sg_net *net) {
  if (net->l2_reserved || !l2_setaside_on() || net->d_ring.n == 0 || net->device < 0 ||
      net->device >= kMaxDevices)
    return;
  int max_persist = 0;
  SG_CUDA(cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, net->device));
  if (max_persist <= 0) return;
  std::lock_guard<std::mutex> lk(g_l2_mu);
  const int d = net->device;
  size_t cur = 0;
  SG_CUDA(cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize));
  if (g_l2_refs[d] == 0) {
    g_l2_saved[d] = cur;
    g_l2_rings[d] = 0;
  }
  const size_t bytes = net->d_ring.n * sizeof(float);
  const size_t want = std::min(g_l2_rings[d] + bytes, (size_t)max_persist);
  if (cur < want) SG_CUDA(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want));
  g_l2_rings[d] += bytes;
  ++g_l2_refs[d];
  net->l2_reserved = true;
  net->l2_bytes = bytes;
}

// The device's set-aside goes back to its earlier value with the last
// network that reserved it (lines still marked persisting become normal).
void release_l2_setaside(sg_net *net) {
  if (!net->l2_reserved) return;
  std::lock_guard<std::mutex> lk(g_l2_mu);
  net->l2_reserved = false;
  g_l2_rings[net->device] -= net->l2_bytes;
  if (--g_l2_refs[net->device] == 0) {
    cudaCtxResetPersistingL2Cache();
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, g_l2_saved[net->device]);
  }
}

// One launch of the pre-centric scatter with schedule `variant` and `bps`
// blocks per SM over a table of networks.
template <int U, bool PIPE, uint32_t P = 1, int MINB = (PIPE && U > 4) ? 3 : 4>
void launch_walk(cudaStream_t s, unsigned grid, int fmt, const StepArgs *nets, uint32_t n_nets, uint32_t *done) {
  switch (fmt) {
    case 1:
      launch_step_kernel(scatter_walk_kernel<U, PIPE, 1, P, MINB>, grid, kWalkThreads, 0, s, nets, n_nets, done);
      break;
    case 2:
      launch_step_kernel(scatter_walk_kernel<U, PIPE, 2, P, MINB>, grid, kWalkThreads, 0, s, nets, n_nets, done);
      break;
    case 3:
      launch_step_kernel(scatter_walk_kernel<U, PIPE, 3, P, MINB>, grid, kWalkThreads, 0, s, nets, n_nets, done);
      break;
    default:
      launch_step_kernel(scatter_walk_kernel<U, PIPE, 0, P, MINB>, grid, kWalkThreads, 0, s, nets, n_nets, done);
  }
}

void launch_step_red(cudaStream_t s, int device, int variant, uint32_t bps, const StepArgs *nets, uint32_t n_nets,
                     uint32_t *done, uint32_t *err, uint32_t stall, int fmt) {
  const unsigned grid = sm_count(device) * bps;
  // the stall test hook acts on the staged pipeline's waits (the walk has none)
  if (is_walk_variant(variant) && stall) variant = 0;
  switch (variant) {
    case kWalkVariant:
      launch_walk<8, false>(s, grid * 2, fmt, nets, n_nets, done);
      break;
    case kWalkPipeVariant:
      launch_walk<4, true>(s, grid * 2, fmt, nets, n_nets, done);
      break;
    case kWalkPipeVariant + 1:  // 3 resident blocks per SM (more registers per thread)
      launch_walk<8, true>(s, grid * 3 / 2, fmt, nets, n_nets, done);
      break;
    case kWalkPipeVariant + 2:  // rows cut in 4 pieces
      launch_walk<8, false, 4>(s, grid * 2, fmt, nets, n_nets, done);
      break;
    case kWalkPipeVariant + 3:  // rows cut in 4 pieces, 6 resident blocks per SM (fewer registers per thread)
      launch_walk<4, false, 4, 6>(s, grid * 3, fmt, nets, n_nets, done);
      break;
    case 1:
      launch_step_kernel(scatter_red_kernel<8, 512>, grid, kRedThreads, sizeof(RedSmemT<8, 512>), s, nets, n_nets,
                         done, err, stall);
      break;
    case 2:
      launch_step_kernel(scatter_red_kernel<3, 2048>, grid, kRedThreads, sizeof(RedSmemT<3, 2048>), s, nets, n_nets,
                         done, err, stall);
      break;
    case 3:
      launch_step_kernel(scatter_red_kernel<6, 512>, grid, kRedThreads, sizeof(RedSmemT<6, 512>), s, nets, n_nets,
                         done, err, stall);
      break;
    default:
      launch_step_kernel(scatter_red_kernel<4, 1024>, grid, kRedThreads, sizeof(RedSmemT<4, 1024>), s, nets, n_nets,
                         done, err, stall);
  }
}

template <int M, bool FULL> void launch_neuron_form(sg_net *net, const StepArgs &a, uint32_t nb) {
  if (net->model_single[M] >= 0)
    launch_step_kernel(neuron_kernel<M, FULL>, nb, NeuronCfg<M, FULL>::THREADS, 0, net->stream, a,
                       net->pop_tab[net->model_single[M]], (const PopArgs *)nullptr, (const uint2 *)nullptr);
  else
    launch_step_kernel(neuron_kernel<M, FULL>, nb, NeuronCfg<M, FULL>::THREADS, 0, net->stream, a, PopArgs{},
                       (const PopArgs *)net->d_pop_tab.p, (const uint2 *)(net->d_blk_map.p + net->model_blk_off[M]));
}

// The lean neuron kernel serves steps without kinetic synapses, input
// noise, neuron statistics, pair STDP or learning.
// The full neuron kernel (kinetics, receptors, noise, statistics, STDP,
// learning) for the populations of model `model`, or the lean one.
bool needs_full_neuron_kernel(const sg_net *net, const StepArgs &a, int model) {
  if (a.n_kin || a.receptor || a.ns_count != nullptr || a.stdp || a.learn) return true;
  for (const auto &p : net->pops)
    if (p.model == model && p.noise) return true;
  return false;
}

template <int M> void launch_neuron(sg_net *net, const StepArgs &a) {
  const uint32_t nb = net->model_blk_cnt[M];
  if (nb == 0) return;
  if (needs_full_neuron_kernel(net, a, M)) launch_neuron_form<M, true>(net, a, nb);
  else launch_neuron_form<M, false>(net, a, nb);
}

// The first half of a step: the neuron update of every population simulated here.
void enqueue_neurons(sg_net *net, const StepArgs &a) {
  cudaStream_t s = net->stream;
  if (net->learn_on) SG_CUDA(cudaMemsetAsync(net->d_l_ctr.p, 0, net->d_l_ctr.n * 4, s));
  launch_neuron<kLIF>(net, a);
  launch_neuron<kIZH>(net, a);
  launch_neuron<kGPEA>(net, a);
  launch_neuron<kHH>(net, a);
}

void enqueue_rest(sg_net *net, const StepArgs &a);

// Phases: 0 neuron update (all populations), 1 scatter.
void enqueue_step(sg_net *net, const StepArgs &a, cudaEvent_t *ev = nullptr) {
  cudaStream_t s = net->stream;
  if (ev) SG_CUDA(cudaEventRecord(ev[0], s));
  enqueue_neurons(net, a);
  if (ev) SG_CUDA(cudaEventRecord(ev[1], s));
  enqueue_rest(net, a);
  if (ev) SG_CUDA(cudaEventRecord(ev[2], s));
}

// The second half: external populations' spikes (when the network is split
// across GPUs), the scatter, the eligibility update.
void enqueue_rest(sg_net *net, const StepArgs &a) {
  cudaStream_t s = net->stream;
  for (const auto &p : net->pops)
    if (p.external && p.n)
      ext_spikes_kernel<<<p.cap / kNeuronBlock, kNeuronBlock, 0, s>>>(a, p.dev_off, p.n, p.ext_src);
  if (a.red) {
    launch_step_red(s, net->device, net->red_variant, net->red_bps, (const StepArgs *)net->d_args.p, 1u,
                    net->d_done.p, net->d_err.p, net->debug_stall, walk_format(a));
  } else {
    if (net->seg32) launch_step_kernel(scatter_kernel<true>, net->G, kScatterThreads, net->scatter_smem, s, a);
    else launch_step_kernel(scatter_kernel<false>, net->G, kScatterThreads, net->scatter_smem, s, a);
  }
  if (net->learn_on && net->n_edges) {
    LearnArgs L{};
    L.bits = net->d_last_bits.p;
    L.flat = net->d_l_flat.p;
    L.flat_cnt = net->d_l_ctr.p;
    L.grab = net->d_l_ctr.p + 1;
    L.row_ptr = net->d_row_ptr.p;
    L.edge = net->d_edge.p;
    L.packed = net->packed;
    L.in_ptr = net->d_l_in_ptr.p;
    L.in_edge = net->d_l_in_edge.p;
    L.in_pre = net->d_l_in_pre.p;
    L.tp = net->d_l_tp.p;
    L.tq = net->d_l_tq.p;
    L.st = net->d_l_st.p;
    L.qa = net->d_l_qa.p;
    L.qb = net->d_l_qb.p;
    L.qcnt = net->d_l_ctr.p + 2;
    L.qcap = net->l_qcap;
    L.step = net->d_step.p;
    L.t0 = net->l_t0;
    L.d_e = net->l_de;
    L.a_ltp = net->l_a_ltp;
    L.a_ltd = net->l_a_ltd;
    const unsigned blocks = 148u * (2048u / kLearnThreads);
    learn_elig_kernel<<<blocks, kLearnThreads, 0, s>>>(L);
    learn_decay_kernel<<<blocks, kLearnThreads, 0, s>>>(L);
  }
}

// Profiled steps: eager launches with CUDA events between the phases, read
// back after every step (adds host synchronisation; for measurement only).
void do_steps_profiled(sg_net *net, uint32_t n) {
  upload_pop_table(net);
  if (net->learn_on) net->d_l_motor.zero(net->stream);  // motor counts are per step call
  const StepArgs a = make_args(net);
  upload_args(net, a);
  if (net->prof_ev.empty()) {
    net->prof_ev.resize(3);
    for (auto &e : net->prof_ev) SG_CUDA(cudaEventCreate(&e));
  }
  size_t n_launch_pops = 0;
  for (int m = 1; m <= 4; ++m) n_launch_pops += net->model_blk_cnt[m] ? 1 : 0;
  for (uint32_t k = 0; k < n; ++k) {
    enqueue_step(net, a, net->prof_ev.data());
    SG_CUDA(cudaEventSynchronize(net->prof_ev[2]));
    for (int ph = 0; ph < 2; ++ph) {
      float ms = 0;
      SG_CUDA(cudaEventElapsedTime(&ms, net->prof_ev[ph], net->prof_ev[ph + 1]));
      net->prof_ms[ph] += ms;
      net->prof_launches[ph] += ph == 0 ? n_launch_pops : 1;
    }
  }
  SG_CUDA(cudaGetLastError());
  net->host_step += n;
}

void drop_graph(sg_net *net) {
  if (net->graph) cudaGraphExecDestroy(net->graph);
  net->graph = nullptr;
  net->graph_steps = 0;
}

void do_steps(sg_net *net, uint32_t n) {
  if (net->total == 0) {
    // empty network: only the counter advances (step.rs:22-25)
    unsigned long long st = 0;
    SG_CUDA(cudaMemcpyAsync(&st, net->d_step.p, 8, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
    st += n;
    SG_CUDA(cudaMemcpyAsync(net->d_step.p, &st, 8, cudaMemcpyHostToDevice, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
    net->host_step += n;
    return;
  }
  upload_pop_table(net);
  if (net->learn_on) net->d_l_motor.zero(net->stream);  // motor counts are per step call
  const StepArgs a = make_args(net);
  upload_args(net, a);
  setup_l2_setaside(net);
  const uint32_t G = 32;  // steps per graph launch
  uint32_t done = 0;
  if (n >= G) {
    if (!net->graph || net->graph_steps != G) {
      drop_graph(net);
      cudaGraph_t g;
      SG_CUDA(cudaStreamBeginCapture(net->stream, cudaStreamCaptureModeThreadLocal));
      for (uint32_t k = 0; k < G; ++k) enqueue_step(net, a);
      SG_CUDA(cudaStreamEndCapture(net->stream, &g));
      SG_CUDA(cudaGraphInstantiate(&net->graph, g, 0));
      cudaGraphDestroy(g);
      net->graph_steps = G;
    }
    for (; done + G <= n; done += G) SG_CUDA(cudaGraphLaunch(net->graph, net->stream));
  }
  for (; done < n; ++done) enqueue_step(net, a);
  SG_CUDA(cudaGetLastError());
  net->host_step += n;
}

}  // namespace

// ===========================================================================
// extern "C"
// ===========================================================================
extern "C" {

int sg_abi_version(void) { return SG_ABI_VERSION; }

int sg_last_error(char *buf, size_t len) {
  if (!buf || len == 0) return SG_E_INVALID;
  std::strncpy(buf, g_last_error.c_str(), len - 1);
  buf[len - 1] = 0;
  return (int)std::min(g_last_error.size(), len - 1);
}

int sg_device_count(int *out) {
  return run([&] {
    SG_REQUIRE(out, SG_E_INVALID, "null output");
    SG_CUDA(cudaGetDeviceCount(out));
  });
}

int sg_net_create(sg_net **out, int device) {
  return run([&] {
    SG_REQUIRE(out, SG_E_INVALID, "null output");
    *out = nullptr;
    int n = 0;
    SG_CUDA(cudaGetDeviceCount(&n));
    SG_REQUIRE(device >= 0 && device < n, SG_E_INVALID, "device ordinal out of range");
    DevGuard g(device);
    auto *net = new sg_net();
    net->device = device;
    net->red_variant = default_red_variant();
    cudaError_t e = cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete net;
      SG_CUDA(e);
    }
    *out = net;
  });
}

int sg_pool_remove(sg_pool *pool, sg_net *net);

int sg_net_destroy(sg_net *net) {
  if (!net) return SG_OK;
  if (net->pool) sg_pool_remove(net->pool, net);  // a destroyed network leaves its pool first
  {
    DevGuard g(net->device);
    cudaStreamSynchronize(net->stream);
    drop_graph(net);
    release_l2_setaside(net);
    for (auto e : net->prof_ev) cudaEventDestroy(e);
    if (net->rstream) {
      cudaStreamSynchronize(net->rstream);
      cudaStreamDestroy(net->rstream);
      cudaEventDestroy(net->rev);
      cudaEventDestroy(net->rdone);
      cudaFreeHost(net->rst_total);
    }
    cudaStream_t s = net->stream;
    delete net;  // DBufs free their memory
    cudaStreamDestroy(s);
  }
  return SG_OK;
}

// The device error word: a wait of the scatter pipeline that ran out of time
// (the step it belongs to is incomplete).  Read and cleared.
void check_device_error(sg_net *net) {
  if (!net->built || !net->d_err.p) return;
  uint32_t e = 0;
  SG_CUDA(cudaMemcpyAsync(&e, net->d_err.p, 4, cudaMemcpyDeviceToHost, net->stream));
  SG_CUDA(cudaStreamSynchronize(net->stream));
  if (e) {
    SG_CUDA(cudaMemsetAsync(net->d_err.p, 0, 4, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
    SG_REQUIRE(false, SG_E_CUDA, "scatter: a pipeline wait timed out on the device (the step's events are incomplete)");
  }
}

int sg_synchronize(sg_net *net) {
  NET_CHECK(net);
  return run([&] {
    DevGuard g(net->device);
    SG_CUDA(cudaStreamSynchronize(net->stream));
    check_device_error(net);
  });
}

int sg_debug_stall_scatter(sg_net *net, int on) {
  NET_CHECK(net);
  return run([&] {
    net->debug_stall = on ? 1u : 0u;
    drop_graph(net);
  });
}

int sg_scatter_schedule(sg_net *net, int *variant, uint32_t *blocks_per_sm) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(variant && blocks_per_sm, SG_E_INVALID, "null output");
    *variant = net->red_variant;
    *blocks_per_sm = net->red_bps;
  });
}

int sg_query(sg_net *net, int *idle) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(idle, SG_E_INVALID, "null output");
    DevGuard g(net->device);
    const cudaError_t e = cudaStreamQuery(net->stream);
    if (e == cudaErrorNotReady) {
      *idle = 0;
      return;
    }
    SG_CUDA(e);
    *idle = 1;
  });
}

int sg_pop_add(sg_net *net, int model, uint32_t n, uint32_t *out_pop) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(!net->built, SG_E_STATE, "Cannot add populations after build()");
    SG_REQUIRE(n_params(model) > 0, SG_E_INVALID, "unknown model");
    SG_REQUIRE(net->total + n <= 0xFFFFFFFFull, SG_E_INVALID, "Network: total neuron count exceeds u32::MAX");
    HostPop p;
    p.model = model;
    p.n = n;
    p.cap = (uint32_t)align_up(n, kNeuronBlock);
    p.dev_off = net->Nd;
    p.np = n_params(model);
    p.ns = n_state(model);
    p.params.assign((size_t)p.cap * p.np, 0.0f);
    p.state.assign((size_t)p.cap * p.ns, 0.0f);
    SG_REQUIRE((uint64_t)net->Nd + p.cap <= 0xFFFFFFFFull, SG_E_INVALID, "device neuron count exceeds u32");
    net->Nd += p.cap;
    net->pops.push_back(std::move(p));
    net->total += n;
    net->offsets.push_back((uint32_t)net->total);
    if (out_pop) *out_pop = (uint32_t)net->pops.size() - 1;
  });
}

// A population simulated on another GPU (a network split across GPUs): it
// holds no state, no parameters and no incoming synapses here; its neurons
// are pre-synaptic neurons whose spikes arrive each step through the
// exchange (sg_pop_set_external_source), at the same device indices, so the
// scatter walks spiking neurons in the same order as the whole network.
int sg_pop_add_external(sg_net *net, uint32_t n, uint32_t *out_pop) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(!net->built, SG_E_STATE, "Cannot add populations after build()");
    SG_REQUIRE(net->total + n <= 0xFFFFFFFFull, SG_E_INVALID, "Network: total neuron count exceeds u32::MAX");
    HostPop p;
    p.model = 0;
    p.external = true;
    p.n = n;
    p.cap = (uint32_t)align_up(n, kNeuronBlock);
    p.dev_off = net->Nd;
    p.np = p.ns = 0;
    SG_REQUIRE((uint64_t)net->Nd + p.cap <= 0xFFFFFFFFull, SG_E_INVALID, "device neuron count exceeds u32");
    net->Nd += p.cap;
    net->pops.push_back(std::move(p));
    net->total += n;
    net->offsets.push_back((uint32_t)net->total);
    if (out_pop) *out_pop = (uint32_t)net->pops.size() - 1;
  });
}

static int pop_col(sg_net *net, uint32_t pop, uint32_t col, bool param) {
  require_pop(net, pop);
  const auto &p = net->pops[pop];
  SG_REQUIRE(col < (param ? p.np : p.ns), SG_E_INVALID,
             std::string(param ? "fill_param" : "fill_state") + ": column " + std::to_string(col) + " out of range");
  return 0;
}

static int pop_write(sg_net *net, uint32_t pop, uint32_t col, bool param, const float *vals, float fill, uint32_t n) {
  return run([&] {
    pop_col(net, pop, col, param);
    auto &p = net->pops[pop];
    if (vals) SG_REQUIRE(n == p.n, SG_E_INVALID, "slice length does not match population size");
    if (!net->built) {
      auto &v = param ? p.params : p.state;
      for (uint32_t i = 0; i < p.n; ++i) v[(size_t)col * p.cap + i] = vals ? vals[i] : fill;
      return;
    }
    DevGuard g(net->device);
    std::vector<float> tmp;
    const float *src = vals;
    if (!vals) {
      tmp.assign(p.n, fill);
      src = tmp.data();
    }
    float *dst = (param ? p.d_params.p : p.d_state.p) + (size_t)col * p.cap;
    SG_CUDA(cudaStreamSynchronize(net->stream));
    SG_CUDA(cudaMemcpy(dst, src, (size_t)p.n * 4, cudaMemcpyHostToDevice));
    if (param && col < 16) {
      // keep the uniform-column summary in step with the device copy; the
      // captured step graph bakes it in, so it is re-captured
      bool uni = p.n > 0;
      for (uint32_t i = 1; i < p.n && uni; ++i) uni = std::memcmp(&src[i], &src[0], 4) == 0;
      if (uni) {
        p.umask |= 1u << col;
        p.uval[col] = src[0];
      } else {
        p.umask &= ~(1u << col);
      }
      net->pop_tab_dirty = true;
      drop_graph(net);
    }
  });
}

static int pop_read(sg_net *net, uint32_t pop, uint32_t col, bool param, float *out, uint32_t n) {
  return run([&] {
    pop_col(net, pop, col, param);
    auto &p = net->pops[pop];
    SG_REQUIRE(out && n == p.n, SG_E_INVALID, "output length does not match population size");
    if (!net->built) {
      const auto &v = param ? p.params : p.state;
      std::memcpy(out, v.data() + (size_t)col * p.cap, (size_t)p.n * 4);
      return;
    }
    DevGuard g(net->device);
    const float *src = (param ? p.d_params.p : p.d_state.p) + (size_t)col * p.cap;
    SG_CUDA(cudaMemcpyAsync(out, src, (size_t)p.n * 4, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
  });
}

int sg_pop_fill_param(sg_net *net, uint32_t pop, uint32_t col, float value) {
  NET_CHECK(net);
  return pop_write(net, pop, col, true, nullptr, value, 0);
}
int sg_pop_fill_state(sg_net *net, uint32_t pop, uint32_t col, float value) {
  NET_CHECK(net);
  return pop_write(net, pop, col, false, nullptr, value, 0);
}
int sg_pop_set_param(sg_net *net, uint32_t pop, uint32_t col, const float *vals, uint32_t n) {
  NET_CHECK(net);
  if (!vals) return (set_error("null values"), SG_E_INVALID);
  return pop_write(net, pop, col, true, vals, 0, n);
}
int sg_pop_set_state(sg_net *net, uint32_t pop, uint32_t col, const float *vals, uint32_t n) {
  NET_CHECK(net);
  if (!vals) return (set_error("null values"), SG_E_INVALID);
  return pop_write(net, pop, col, false, vals, 0, n);
}
int sg_pop_get_state(sg_net *net, uint32_t pop, uint32_t col, float *out, uint32_t n) {
  NET_CHECK(net);
  return pop_read(net, pop, col, false, out, n);
}
int sg_pop_get_param(sg_net *net, uint32_t pop, uint32_t col, float *out, uint32_t n) {
  NET_CHECK(net);
  return pop_read(net, pop, col, true, out, n);
}

static int connect_impl(sg_net *net, uint32_t from, const uint32_t *fi, uint32_t to, const uint32_t *ti,
                        const float *w, const uint8_t *d, const uint8_t *st, const uint8_t *ptype, uint64_t n,
                        uint32_t flags) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(!net->built, SG_E_STATE, "Cannot connect after build()");
    require_pop(net, from);
    require_local(net, to);
    if (n == 0) return;
    SG_REQUIRE(fi && ti && w && d, SG_E_INVALID, "null slice");
    const auto &pf = net->pops[from];
    const auto &pt = net->pops[to];
    std::vector<uint32_t> pre(n), post(n);
    std::vector<uint8_t> code(n);
    for (uint64_t i = 0; i < n; ++i) {
      SG_REQUIRE(fi[i] < pf.n, SG_E_INVALID, "from index " + std::to_string(fi[i]) + " out of bounds");
      SG_REQUIRE(ti[i] < pt.n, SG_E_INVALID, "to index " + std::to_string(ti[i]) + " out of bounds");
      SG_REQUIRE(std::isfinite(w[i]), SG_E_INVALID, "Network::connect: weight " + std::to_string(i) + " must be finite");
      SG_REQUIRE(d[i] < kSlots, SG_E_INVALID, "delay " + std::to_string(d[i]) + " >= MAX_DELAY_SLOTS (32)");
      net->max_delay = std::max<uint32_t>(net->max_delay, d[i]);
      const uint8_t s = st ? st[i] : 0;
      SG_REQUIRE(net->receptor || s <= 3, SG_E_INVALID, "syn_type > 3 is not supported on the device path");
      SG_REQUIRE(!net->receptor || (!(flags & SG_EDGE_STDP) && (!ptype || ptype[i] == 0)), SG_E_INVALID,
                 "receptor kinetics: no pair-STDP or short-term plastic synapses");
      if (ptype)
        SG_REQUIRE(ptype[i] <= net->tm_prof.size(), SG_E_INVALID,
                   "Network::build: plast_type " + std::to_string(ptype[i]) + " exceeds registered plasticity profiles");
      pre[i] = pf.dev_off + fi[i];
      post[i] = pt.dev_off + ti[i];
      code[i] = net->receptor ? receptor_code(s) : edge_code(d[i], s, (flags & SG_EDGE_STDP) != 0);
    }
    DevGuard g(net->device);
    upload_staged_edges(net, pre.data(), post.data(), w, code.data(), n, ptype);
  });
}

int sg_connect_ex(sg_net *net, uint32_t from, const uint32_t *fi, uint32_t to, const uint32_t *ti,
                  const float *w, const uint8_t *d, const uint8_t *st, uint64_t n, uint32_t flags) {
  return connect_impl(net, from, fi, to, ti, w, d, st, nullptr, n, flags);
}

int sg_connect_plastic(sg_net *net, uint32_t from, const uint32_t *fi, uint32_t to, const uint32_t *ti,
                       const float *w, const uint8_t *d, const uint8_t *st, const uint8_t *pt, uint64_t n,
                       uint32_t flags) {
  return connect_impl(net, from, fi, to, ti, w, d, st, pt, n, flags);
}

int sg_register_plasticity(sg_net *net, float u0, float tau_rec, int facilitation, float tau_fac, float dt,
                           uint32_t *out_id) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(!net->built, SG_E_STATE, "register_plasticity must be called before build()");
    SG_REQUIRE(std::isfinite(dt) && dt > 0, SG_E_INVALID, "register_plasticity: dt must be finite and > 0");
    SG_REQUIRE(std::isfinite(u0) && u0 > 0.0f && u0 <= 1.0f, SG_E_INVALID, "init_release_prob must be in (0, 1]");
    SG_REQUIRE(std::isfinite(tau_rec) && tau_rec > 0.0f, SG_E_INVALID, "tau_rec must be finite and > 0");
    SG_REQUIRE(!facilitation || (std::isfinite(tau_fac) && tau_fac > 0.0f), SG_E_INVALID,
               "tau_fac must be finite and > 0");
    SG_REQUIRE(net->tm_prof.size() < kMaxTm, SG_E_INVALID,
               "at most " + std::to_string(kMaxTm) + " plasticity profiles are supported on the device path");
    net->tm_prof.push_back(TmHost{u0, std::exp(-dt / tau_rec), facilitation ? std::exp(-dt / tau_fac) : 0.0f,
                                  facilitation != 0});
    if (out_id) *out_id = (uint32_t)net->tm_prof.size();
  });
}

int sg_connect(sg_net *net, uint32_t from, const uint32_t *fi, uint32_t to, const uint32_t *ti,
               const float *w, const uint8_t *d, uint64_t n) {
  return sg_connect_ex(net, from, fi, to, ti, w, d, nullptr, n, 0);
}

int sg_connect_fixed_indegree(sg_net *net, uint32_t from, uint32_t to, uint32_t k_in, uint64_t seed,
                              uint32_t n_exc, float w_exc, float w_inh, uint8_t d_min, uint8_t d_max,
                              uint8_t st_e, uint8_t st_i, uint32_t flags_e) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(!net->built, SG_E_STATE, "Cannot connect after build()");
    require_pop(net, from);
    require_local(net, to);
    SG_REQUIRE(d_min <= d_max && d_max < kSlots, SG_E_INVALID, "delay range invalid");
    SG_REQUIRE(std::isfinite(w_exc) && std::isfinite(w_inh), SG_E_INVALID, "weights must be finite");
    SG_REQUIRE(net->receptor || (st_e <= 3 && st_i <= 3), SG_E_INVALID, "syn_type > 3 is not supported");
    SG_REQUIRE(!net->receptor || !(flags_e & SG_EDGE_STDP), SG_E_INVALID, "receptor kinetics: no pair-STDP synapses");
    const auto &pf = net->pops[from];
    const auto &pt = net->pops[to];
    SG_REQUIRE(pf.n > 0 || k_in == 0, SG_E_INVALID, "empty source population");
    const uint64_t n = (uint64_t)pt.n * k_in;
    if (n == 0) return;
    net->max_delay = std::max<uint32_t>(net->max_delay, d_max);
    DevGuard g(net->device);
    const size_t n0 = net->e_pre.n;
    net->e_pre.reserve(n0 + n, net->stream);
    net->e_post.reserve(n0 + n, net->stream);
    net->e_w.reserve(n0 + n, net->stream);
    net->e_code.reserve(n0 + n, net->stream);
    launch_grid(n, [&](unsigned b) {
      synth_indegree_kernel<<<b, 256, 0, net->stream>>>(net->e_pre.p, net->e_post.p, net->e_w.p, net->e_code.p, n0,
                                                        pt.n, k_in, seed, pf.dev_off, pf.n, pt.dev_off, n_exc, w_exc,
                                                        w_inh, d_min, (uint32_t)(d_max - d_min + 1), st_e, st_i, flags_e,
                                                        net->receptor ? 1 : 0);
    });
    SG_CUDA(cudaGetLastError());
    SG_CUDA(cudaStreamSynchronize(net->stream));
    net->e_pre.n = net->e_post.n = net->e_w.n = net->e_code.n = n0 + n;
  });
}

// Common checks and the generator parameters of the two out-degree builders.
static OutDegreeSpec outdegree_spec(sg_net *net, uint32_t from, uint32_t to, uint64_t seed, int no_self,
                                    uint32_t n_exc, float w_exc, float w_inh, int random_w, uint8_t d_min,
                                    uint8_t d_max, uint8_t st_e, uint8_t st_i, uint32_t flags_e) {
  SG_REQUIRE(!net->built, SG_E_STATE, "Cannot connect after build()");
  require_pop(net, from);
  require_local(net, to);
  SG_REQUIRE(d_min <= d_max && d_max < kSlots, SG_E_INVALID, "delay range invalid (d_min <= d_max < 32)");
  SG_REQUIRE(std::isfinite(w_exc) && std::isfinite(w_inh), SG_E_INVALID, "weights must be finite");
  SG_REQUIRE(net->receptor || (st_e <= 3 && st_i <= 3), SG_E_INVALID, "syn_type > 3 is not supported");
  SG_REQUIRE(!net->receptor || !(flags_e & SG_EDGE_STDP), SG_E_INVALID, "receptor kinetics: no pair-STDP synapses");
  SG_REQUIRE(!no_self || from == to, SG_E_INVALID, "no_self needs from == to");
  SG_REQUIRE(random_w >= 0 && random_w <= 24, SG_E_INVALID, "random_w: 0, 1, or a grid of 2..24 bits");
  OutDegreeSpec sp{};
  sp.seed = seed;
  sp.from_off = net->pops[from].dev_off;
  sp.to_off = net->pops[to].dev_off;
  sp.n_to = net->pops[to].n;
  sp.n_exc = n_exc;
  sp.no_self = no_self;
  sp.random_w = random_w;
  sp.w_exc = w_exc;
  sp.w_inh = w_inh;
  sp.d_min = d_min;
  sp.d_span = (uint32_t)(d_max - d_min) + 1u;
  sp.st_exc = st_e;
  sp.st_inh = st_i;
  sp.flags_exc = flags_e;
  sp.receptor = net->receptor ? 1 : 0;
  return sp;
}

int sg_connect_fixed_outdegree(sg_net *net, uint32_t from, uint32_t to, uint32_t k, uint64_t seed, int no_self,
                               uint32_t n_exc, float w_exc, float w_inh, int random_w, uint8_t d_min, uint8_t d_max,
                               uint8_t st_e, uint8_t st_i, uint32_t flags_e) {
  NET_CHECK(net);
  return run([&] {
    const OutDegreeSpec sp =
        outdegree_spec(net, from, to, seed, no_self, n_exc, w_exc, w_inh, random_w, d_min, d_max, st_e, st_i, flags_e);
    const auto &pf = net->pops[from];
    const auto &pt = net->pops[to];
    const uint32_t m = pt.n - (no_self && pt.n ? 1u : 0u);
    SG_REQUIRE(k <= m && k <= kMaxOutDegree, SG_E_INVALID, "out-degree larger than the candidate targets or 4096");
    const uint64_t n = (uint64_t)pf.n * k;
    if (n == 0) return;
    net->max_delay = std::max<uint32_t>(net->max_delay, d_max);
    DevGuard g(net->device);
    const size_t n0 = net->e_pre.n;
    net->e_pre.reserve(n0 + n, net->stream);
    net->e_post.reserve(n0 + n, net->stream);
    net->e_w.reserve(n0 + n, net->stream);
    net->e_code.reserve(n0 + n, net->stream);
    const unsigned blocks = (unsigned)std::min<uint64_t>((pf.n + 127) / 128, 148u * 16u);
    synth_outdegree_kernel<<<blocks, 128, 0, net->stream>>>(net->e_pre.p, net->e_post.p, net->e_w.p, net->e_code.p,
                                                             n0, pf.n, k, nullptr, nullptr, sp);
    SG_CUDA(cudaGetLastError());
    SG_CUDA(cudaStreamSynchronize(net->stream));
    net->e_pre.n = net->e_post.n = net->e_w.n = net->e_code.n = n0 + n;
  });
}

int sg_connect_lognormal_outdegree(sg_net *net, uint32_t from, uint32_t to, double mean, double sd,
                                   uint64_t seed, int no_self, uint32_t n_exc, float w_exc, float w_inh,
                                   int random_w, uint8_t d_min, uint8_t d_max, uint8_t st_e, uint8_t st_i,
                                   uint32_t flags_e) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(std::isfinite(mean) && mean > 0 && std::isfinite(sd) && sd >= 0, SG_E_INVALID,
               "lognormal degree needs mean > 0 and sd >= 0");
    const OutDegreeSpec sp =
        outdegree_spec(net, from, to, seed, no_self, n_exc, w_exc, w_inh, random_w, d_min, d_max, st_e, st_i, flags_e);
    const auto &pf = net->pops[from];
    const auto &pt = net->pops[to];
    const uint32_t m = pt.n - (no_self && pt.n ? 1u : 0u);
    if (pf.n == 0) return;
    SG_REQUIRE(m >= 1, SG_E_INVALID, "no candidate targets");
    const double s2 = std::log(1.0 + (sd * sd) / (mean * mean));
    const double mu = std::log(mean) - 0.5 * s2, sigma = std::sqrt(s2);
    const uint32_t kmax = std::min<uint32_t>(m, kMaxOutDegree);
    DevGuard g(net->device);
    cudaStream_t s = net->stream;
    DBuf<uint32_t> deg;
    deg.alloc(pf.n);
    DBuf<unsigned long long> off, deg64;
    off.alloc((size_t)pf.n + 1);
    deg64.alloc((size_t)pf.n + 1);
    const unsigned blocks = (unsigned)std::min<uint64_t>((pf.n + 255) / 256, 148u * 16u);
    lognormal_degree_kernel<<<blocks, 256, 0, s>>>(deg.p, pf.n, seed, mu, sigma, kmax);
    SG_CUDA(cudaGetLastError());
    widen_kernel<<<blocks, 256, 0, s>>>(deg.p, deg64.p, pf.n);
    SG_CUDA(cudaGetLastError());
    size_t tb = 0;
    SG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, deg64.p, off.p, (int64_t)pf.n + 1, s));
    DBuf<uint8_t> temp;
    temp.alloc(std::max<size_t>(tb, 1));
    SG_CUDA(cub::DeviceScan::ExclusiveSum(temp.p, tb, deg64.p, off.p, (int64_t)pf.n + 1, s));
    unsigned long long total = 0;
    SG_CUDA(cudaMemcpyAsync(&total, off.p + pf.n, 8, cudaMemcpyDeviceToHost, s));
    SG_CUDA(cudaStreamSynchronize(s));
    if (total == 0) return;
    net->max_delay = std::max<uint32_t>(net->max_delay, d_max);
    const size_t n0 = net->e_pre.n;
    net->e_pre.reserve(n0 + total, s);
    net->e_post.reserve(n0 + total, s);
    net->e_w.reserve(n0 + total, s);
    net->e_code.reserve(n0 + total, s);
    const unsigned b2 = (unsigned)std::min<uint64_t>((pf.n + 127) / 128, 148u * 16u);
    synth_outdegree_kernel<<<b2, 128, 0, s>>>(net->e_pre.p, net->e_post.p, net->e_w.p, net->e_code.p, n0, pf.n, 0,
                                              deg.p, off.p, sp);
    SG_CUDA(cudaGetLastError());
    SG_CUDA(cudaStreamSynchronize(s));
    net->e_pre.n = net->e_post.n = net->e_w.n = net->e_code.n = n0 + total;
  });
}

// P/api/net/synapse.rs:296-305 exp_waveform_factor (NeuroML waveformFactor), f32
static float waveform_factor(float tr, float td) {
  const float t_peak = (tr * td) / (td - tr) * std::log(td / tr);
  const float h = std::exp(-t_peak / td) - std::exp(-t_peak / tr);
  return 1.0f / h;
}

int sg_register_kinetics(sg_net *net, int kind, const float *p, float erev, float dt, uint32_t *out_id) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(!net->built, SG_E_STATE, "register_kinetics must be called before build()");
    SG_REQUIRE(!net->receptor, SG_E_STATE, "receptor kinetics: no kinetic profiles");
    SG_REQUIRE(p, SG_E_INVALID, "null parameters");
    SG_REQUIRE(std::isfinite(erev), SG_E_INVALID, "erev must be finite");
    SG_REQUIRE(std::isfinite(dt) && dt > 0, SG_E_INVALID, "register_kinetics: dt must be finite and > 0");
    SG_REQUIRE(net->kin.size() < 3, SG_E_INVALID, "at most 3 kinetic profiles are supported on the device path");
    auto pos = [](float x) { return std::isfinite(x) && x > 0.0f; };
    Kin k{kind, erev, {}};
    if (kind == SG_KIN_EXPONE) {  // synapse.rs:102-106 validation; step.rs:251-253
      SG_REQUIRE(pos(p[0]), SG_E_INVALID, "tau_decay must be finite and > 0");
      k.c[0] = std::exp(-dt / p[0]);
    } else if (kind == SG_KIN_EXPTWO) {  // synapse.rs:107-122; step.rs:254-262
      SG_REQUIRE(pos(p[1]), SG_E_INVALID, "tau_decay must be finite and > 0");
      SG_REQUIRE(pos(p[0]), SG_E_INVALID, "tau_rise must be finite and > 0");
      SG_REQUIRE(p[0] < p[1], SG_E_INVALID, "tau_rise must be < tau_decay");
      k.c[0] = std::exp(-dt / p[0]);
      k.c[1] = std::exp(-dt / p[1]);
      k.c[2] = waveform_factor(p[0], p[1]);
    } else if (kind == SG_KIN_ALPHA) {  // synapse.rs:123-127; step.rs:263-269
      SG_REQUIRE(pos(p[0]), SG_E_INVALID, "tau must be finite and > 0");
      const float r = std::exp(-dt / p[0]);
      k.c[0] = r;
      k.c[1] = 2.7182817f * (dt / p[0]) * r;  // std::f32::consts::E
    } else if (kind == SG_KIN_EXPTHREE) {  // synapse.rs:128-156; step.rs:270-291
      const float tr = p[0], td1 = p[1], td2 = p[2], g1 = p[3], g2 = p[4];
      SG_REQUIRE(pos(tr), SG_E_INVALID, "tau_rise must be finite and > 0");
      SG_REQUIRE(std::isfinite(td1) && td1 > tr, SG_E_INVALID, "tau_decay1 must be finite and > tau_rise");
      SG_REQUIRE(std::isfinite(td2) && td2 > tr, SG_E_INVALID, "tau_decay2 must be finite and > tau_rise");
      SG_REQUIRE(std::isfinite(g1) && g1 >= 0.0f && std::isfinite(g2) && g2 >= 0.0f, SG_E_INVALID,
                 "gbase1 and gbase2 must be finite and >= 0");
      SG_REQUIRE(g1 + g2 > 0.0f, SG_E_INVALID, "gbase1 + gbase2 must be > 0");
      const float wf1 = waveform_factor(tr, td1), wf2 = waveform_factor(tr, td2);
      k.c[0] = std::exp(-dt / tr);
      k.c[1] = std::exp(-dt / td1);
      k.c[2] = std::exp(-dt / td2);
      k.c[3] = wf1;
      k.c[4] = wf2;
      k.c[5] = (g1 * wf1 + g2 * wf2) / (g1 + g2);
      k.c[6] = g1;
      k.c[7] = g2;
    } else {
      SG_REQUIRE(false, SG_E_INVALID, "unknown kinetics kind " + std::to_string(kind));
    }
    net->kin.push_back(k);
    if (out_id) *out_id = (uint32_t)net->kin.size();
  });
}

int sg_register_expone(sg_net *net, float tau_decay, float erev, float dt, uint32_t *out_id) {
  return sg_register_kinetics(net, SG_KIN_EXPONE, &tau_decay, erev, dt, out_id);
}

int sg_poisson_add_many(sg_net *net, uint32_t n, float rate_hz, float dt_ms, const uint32_t *seeds, uint32_t seed0,
                        uint32_t *out_first) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(!net->built, SG_E_STATE, "add_poisson_source must be called before build()");
    SG_REQUIRE(!net->receptor, SG_E_STATE, "receptor kinetics: no Poisson sources");
    SG_REQUIRE(std::isfinite(rate_hz) && rate_hz >= 0, SG_E_INVALID, "add_poisson_source: rate_hz must be finite and >= 0");
    SG_REQUIRE(std::isfinite(dt_ms) && dt_ms > 0, SG_E_INVALID, "add_poisson_source: dt_ms must be finite and > 0");
    float p = rate_hz * dt_ms / 1000.0f;  // core.rs:301
    p = std::fmin(std::fmax(p, 0.0f), 1.0f);
    if (out_first) *out_first = (uint32_t)net->srcs.size();
    net->srcs.reserve(net->srcs.size() + n);
    for (uint32_t i = 0; i < n; ++i) {
      HostSrc s;
      s.p = p;
      s.seed = seeds ? seeds[i] : seed0 + i;
      net->srcs.push_back(std::move(s));
    }
  });
}

int sg_poisson_add(sg_net *net, float rate_hz, float dt_ms, uint32_t seed, uint32_t *out_id) {
  return sg_poisson_add_many(net, 1, rate_hz, dt_ms, nullptr, seed, out_id);
}

int sg_poisson_connect_plastic(sg_net *net, uint32_t src, uint32_t to, const uint32_t *posts, const float *w,
                               const uint8_t *d, const uint8_t *st, const uint8_t *plast, uint64_t n) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(!net->built, SG_E_STATE, "Cannot connect after build()");
    SG_REQUIRE(src < net->srcs.size(), SG_E_INVALID, "poisson source out of range");
    require_local(net, to);
    SG_REQUIRE(n == 0 || (posts && w && d), SG_E_INVALID, "null slice");
    const auto &pt = net->pops[to];
    for (uint64_t i = 0; i < n; ++i) {
      SG_REQUIRE(posts[i] < pt.n, SG_E_INVALID, "post index out of bounds");
      SG_REQUIRE(std::isfinite(w[i]), SG_E_INVALID, "connect_poisson_source: weight must be finite");
      SG_REQUIRE(d[i] < kSlots, SG_E_INVALID, "connect_poisson_source: delay >= MAX_DELAY_SLOTS (32)");
      const uint8_t t = st ? st[i] : 0;
      SG_REQUIRE(t <= 3, SG_E_INVALID, "syn_type > 3 is not supported on the device path");
      const uint8_t q = plast ? plast[i] : 0;
      SG_REQUIRE(q <= net->tm_prof.size(), SG_E_INVALID,
                 "plasticity profile " + std::to_string(q) + " is not registered");
    }
    net->src_syn.reserve(net->src_syn.size() + n);
    for (uint64_t i = 0; i < n; ++i) {
      net->max_delay = std::max<uint32_t>(net->max_delay, d[i]);
      net->src_syn.push_back(SrcSyn{src, pt.dev_off + posts[i], w[i], edge_code(d[i], st ? st[i] : 0, false),
                                    (uint8_t)(plast ? plast[i] : 0)});
    }
  });
}

int sg_poisson_connect(sg_net *net, uint32_t src, uint32_t to, const uint32_t *posts, const float *w,
                       const uint8_t *d, const uint8_t *st, uint64_t n) {
  return sg_poisson_connect_plastic(net, src, to, posts, w, d, st, nullptr, n);
}

int sg_poisson_connect_one_to_one(sg_net *net, uint32_t first, uint32_t n, uint32_t to, const uint32_t *posts,
                                  float weight, uint8_t delay) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(!net->built, SG_E_STATE, "Cannot connect after build()");
    SG_REQUIRE((uint64_t)first + n <= net->srcs.size(), SG_E_INVALID, "poisson source out of range");
    require_local(net, to);
    SG_REQUIRE(std::isfinite(weight), SG_E_INVALID, "weight must be finite");
    SG_REQUIRE(delay < kSlots, SG_E_INVALID, "delay >= MAX_DELAY_SLOTS (32)");
    if (n) net->max_delay = std::max<uint32_t>(net->max_delay, delay);
    const auto &pt = net->pops[to];
    if (posts)
      for (uint32_t i = 0; i < n; ++i) SG_REQUIRE(posts[i] < pt.n, SG_E_INVALID, "post index out of bounds");
    else
      SG_REQUIRE(n <= pt.n, SG_E_INVALID, "post index out of bounds");
    const uint8_t code = edge_code(delay, 0, false);
    net->src_syn.reserve(net->src_syn.size() + n);
    for (uint32_t i = 0; i < n; ++i)
      net->src_syn.push_back(SrcSyn{first + i, pt.dev_off + (posts ? posts[i] : i), weight, code, 0});
  });
}

// SynapticBrain::from_sparse_graph(graph, receptor_types, dt)
// (pillars-connectome/src/synaptic.rs:53-63): the syn_types of the edges
// connected after this call are receptor codes, delays are ignored, and
// every step decays the seven conductances and adds their ohmic current
// (step order :94-130).  DecayFactors::new(dt), P/kernels/synapse/
// kinetics.rs:27-38.
int sg_set_receptor_kinetics(sg_net *net, float dt) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(!net->built, SG_E_STATE, "receptor kinetics must be set before build()");
    SG_REQUIRE(std::isfinite(dt) && dt > 0.0f, SG_E_INVALID, "receptor kinetics: dt must be finite and > 0");
    SG_REQUIRE(net->e_pre.n == 0 && net->kin.empty() && net->srcs.empty() && !net->stdp_on, SG_E_STATE,
               "receptor kinetics: set before any synapse, kinetic profile, Poisson source or STDP");
    net->receptor = true;
    for (int r = 0; r < kReceptors; ++r) net->rec_f[r] = host_fast_exp(-dt / rec_tau(r));
  });
}

// SynapticBrain::kinetics / set_kinetics (synaptic.rs:66-80): the seven
// conductance arrays, g[r * total + i] for receptor r and neuron i.
int sg_receptor_read(sg_net *net, float *g) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built && net->receptor, SG_E_STATE, "receptor kinetics are not on (or not built)");
    SG_REQUIRE(g, SG_E_INVALID, "null output");
    DevGuard gd(net->device);
    const uint32_t Nd = net->Nd;
    std::vector<float> r((size_t)kReceptors * Nd);
    SG_CUDA(cudaMemcpyAsync(r.data(), net->d_ring.p + Nd, r.size() * 4, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
    const uint64_t N = net->total;
    for (int k = 0; k < kReceptors; ++k)
      for (size_t p = 0; p < net->pops.size(); ++p)
        for (uint32_t i = 0; i < net->pops[p].n; ++i)
          g[(size_t)k * N + net->offsets[p] + i] = r[(size_t)k * Nd + net->pops[p].dev_off + i];
  });
}

int sg_receptor_write(sg_net *net, const float *g) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built && net->receptor, SG_E_STATE, "receptor kinetics are not on (or not built)");
    SG_REQUIRE(g, SG_E_INVALID, "null input");
    const uint64_t N = net->total;
    for (uint64_t k = 0; k < (uint64_t)kReceptors * N; ++k)
      SG_REQUIRE(std::isfinite(g[k]), SG_E_INVALID, "conductances must be finite");
    DevGuard gd(net->device);
    const uint32_t Nd = net->Nd;
    std::vector<float> r((size_t)kReceptors * Nd, 0.0f);
    for (int k = 0; k < kReceptors; ++k)
      for (size_t p = 0; p < net->pops.size(); ++p)
        for (uint32_t i = 0; i < net->pops[p].n; ++i)
          r[(size_t)k * Nd + net->pops[p].dev_off + i] = g[(size_t)k * N + net->offsets[p] + i];
    SG_CUDA(cudaStreamSynchronize(net->stream));
    SG_CUDA(cudaMemcpyAsync(net->d_ring.p + Nd, r.data(), r.size() * 4, cudaMemcpyHostToDevice, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
  });
}

int sg_stdp_config(sg_net *net, float dt, float tau_pre, float tau_post, float a_plus, float a_minus, float w_min,
                   float w_max) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(!net->built, SG_E_STATE, "stdp must be configured before build()");
    SG_REQUIRE(!net->receptor, SG_E_STATE, "receptor kinetics: no pair STDP");
    SG_REQUIRE(dt > 0 && tau_pre > 0 && tau_post > 0 && w_min <= w_max, SG_E_INVALID, "invalid STDP config");
    net->stdp_on = true;
    net->stdp_dt = dt;
    net->tau_pre = tau_pre;
    net->tau_post = tau_post;
    net->a_plus = a_plus;
    net->a_minus = a_minus;
    net->w_min = w_min;
    net->w_max = w_max;
  });
}

int sg_set_weight_format(sg_net *net, int format) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(!net->built, SG_E_STATE, "weight format must be set before build()");
    SG_REQUIRE(format == SG_W_F32 || format == SG_W_BF16 || format == SG_W_FP8, SG_E_INVALID,
               "weight format: SG_W_F32, SG_W_BF16 or SG_W_FP8");
    net->weight_format = format;
  });
}

int sg_scatter_mode(sg_net *net, int *out) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "not built");
    SG_REQUIRE(out, SG_E_INVALID, "null output");
    *out = !net->deterministic ? SG_SCATTER_ATOMIC : net->red ? SG_SCATTER_EXACT : SG_SCATTER_ORDERED;
  });
}

int sg_set_deterministic(sg_net *net, int on) {
  NET_CHECK(net);
  return run([&] {
    net->deterministic = on ? 1 : 0;
    drop_graph(net);
    if (net->built) update_path(net);
  });
}

int sg_build(sg_net *net) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(!net->built, SG_E_STATE, "Network::build() called twice — the graph is already built");
    SG_REQUIRE(!net->receptor || (net->kin.empty() && net->srcs.empty() && !net->stdp_on && !net->tm_edges),
               SG_E_INVALID,
               "receptor kinetics: no kinetic profiles, Poisson sources, pair-STDP or short-term plasticity");
    DevGuard g(net->device);
    // GPEA Nernst constants (gpea.rs:277-278), with the ln the kernels use
    net->ln_consts = {sg_logf(10.0f / 140.0f), sg_logf(5.0f / 140.0f)};
    const uint64_t E = net->e_pre.n;
    uint64_t src_e = 0;
    src_e = net->src_syn.size();
    SG_REQUIRE(E + src_e < 0xFFFFFFFFull, SG_E_OVERFLOW,
               "SparseGraph: too many synapses for a u32 CSR row_ptr / event key");
    build_graph(net);
    build_segments(net);
    build_sources(net);
    if (net->stdp_on) build_stdp(net);
    split_bf16(net);
    split_fp8(net);
    finish_build(net);
  });
}

int sg_build_from_csr(sg_net *net, const uint32_t *row_ptr, const uint32_t *col, const float *w, const uint8_t *d) {
  NET_CHECK(net);
  const int rc = run([&] {
    SG_REQUIRE(!net->built, SG_E_STATE, "Network::build() called twice");
    SG_REQUIRE(net->e_pre.n == 0, SG_E_STATE, "from_csr: edges were already added");
    SG_REQUIRE(row_ptr && row_ptr[0] == 0, SG_E_INVALID, "CSR row_ptr must start at 0");
    const uint64_t N = net->total;
    for (uint64_t i = 0; i < N; ++i)
      SG_REQUIRE(row_ptr[i] <= row_ptr[i + 1], SG_E_INVALID, "CSR row_ptr must be monotonically non-decreasing");
    const uint64_t E = row_ptr[N];
    // global -> device index
    std::vector<uint32_t> g2d(N);
    for (size_t p = 0; p < net->pops.size(); ++p)
      for (uint32_t i = 0; i < net->pops[p].n; ++i) g2d[net->offsets[p] + i] = net->pops[p].dev_off + i;
    std::vector<uint32_t> pre(E), post(E);
    std::vector<uint8_t> code(E);
    for (uint64_t i = 0; i < N; ++i)
      for (uint64_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e) {
        SG_REQUIRE(col[e] < N, SG_E_INVALID, "col index out of range");
        SG_REQUIRE(std::isfinite(w[e]), SG_E_INVALID, "weight must be finite");
        SG_REQUIRE(d[e] < kSlots, SG_E_INVALID, "delay >= MAX_DELAY_SLOTS (32)");
        net->max_delay = std::max<uint32_t>(net->max_delay, d[e]);
        pre[e] = g2d[i];
        post[e] = g2d[col[e]];
        code[e] = net->receptor ? receptor_code(0) : edge_code(d[e], 0, false);
      }
    DevGuard g(net->device);
    if (E) upload_staged_edges(net, pre.data(), post.data(), w, code.data(), E);
  });
  return rc != SG_OK ? rc : sg_build(net);
}

int sg_pop_set_noise(sg_net *net, uint32_t pop, uint64_t seed, uint32_t stream, uint64_t stride, uint64_t step0,
                     double sigma_lo, double sigma_hi, uint32_t split) {
  NET_CHECK(net);
  return run([&] {
    require_pop(net, pop);
    SG_REQUIRE(std::isfinite(sigma_lo) && std::isfinite(sigma_hi), SG_E_INVALID, "noise sigma must be finite");
    HostPop &p = net->pops[pop];
    p.noise = sigma_lo != 0.0 || sigma_hi != 0.0;
    p.noise_seed = seed;
    p.noise_stream = stream;
    p.noise_stride = stride;
    p.noise_step0 = step0;
    p.noise_sigma[0] = sigma_lo;
    p.noise_sigma[1] = sigma_hi;
    p.noise_split = split;
    net->pop_tab_dirty = true;
    drop_graph(net);  // a captured step graph may hold the old arguments by value
  });
}

int sg_pop_set_bias(sg_net *net, uint32_t pop, const float *vals, uint32_t n) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "set_bias needs a built network");
    require_pop(net, pop);
    HostPop &p = net->pops[pop];
    SG_REQUIRE(n <= p.n, SG_E_INVALID, "more bias values than neurons");
    DevGuard g(net->device);
    SG_CUDA(cudaStreamSynchronize(net->stream));
    if (n == 0) {
      p.d_bias.release();
    } else {
      for (uint32_t i = 0; i < n; ++i) SG_REQUIRE(std::isfinite(vals[i]), SG_E_INVALID, "bias must be finite");
      if (p.d_bias.n != p.cap) p.d_bias.alloc(p.cap);
      std::vector<float> h(p.cap, 0.0f);
      std::copy(vals, vals + n, h.begin());
      SG_CUDA(cudaMemcpy(p.d_bias.p, h.data(), (size_t)p.cap * 4, cudaMemcpyHostToDevice));
    }
    net->pop_tab_dirty = true;
    drop_graph(net);
  });
}

int sg_ring_clear(sg_net *net) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "not built");
    DevGuard g(net->device);
    net->d_ring.zero(net->stream);
    net->d_kin_g.zero(net->stream);
    drop_drive(net);
    SG_CUDA(cudaStreamSynchronize(net->stream));
  });
}

int sg_inject(sg_net *net, uint32_t pop, const uint32_t *idx, const float *vals, uint64_t n) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "inject_current() called before build()");
    require_local(net, pop);
    if (n == 0) return;
    SG_REQUIRE(idx && vals, SG_E_INVALID, "null slice");
    const auto &p = net->pops[pop];
    std::vector<uint8_t> seen(p.n, 0);
    bool dup = false;
    for (uint64_t i = 0; i < n; ++i) {
      SG_REQUIRE(idx[i] < p.n, SG_E_INVALID,
                 "inject_current: neuron index " + std::to_string(idx[i]) + " out of bounds (population has " +
                     std::to_string(p.n) + ")");
      SG_REQUIRE(std::isfinite(vals[i]), SG_E_INVALID, "inject_current: value must be finite");
      dup |= seen[idx[i]] != 0;
      seen[idx[i]] = 1;
    }
    DevGuard g(net->device);
    if (net->d_inj_idx.n < n) {
      net->d_inj_idx.alloc(n);
      net->d_inj_val.alloc(n);
    }
    SG_CUDA(cudaMemcpyAsync(net->d_inj_idx.p, idx, n * 4, cudaMemcpyHostToDevice, net->stream));
    SG_CUDA(cudaMemcpyAsync(net->d_inj_val.p, vals, n * 4, cudaMemcpyHostToDevice, net->stream));
    fold_drive(net);  // the last step's deferred drive precedes this input in the slot
    unsigned blocks = (unsigned)std::min<uint64_t>((n + 255) / 256, 148 * 8);
    inject_kernel<<<blocks, 256, 0, net->stream>>>(net->d_ring.p, net->Nd, net->receptor ? 1u : net->nslots,
                                                   net->d_step.p, net->d_inj_idx.p,
                                                   net->d_inj_val.p, n, p.dev_off, dup ? 1 : 0);
    SG_CUDA(cudaGetLastError());
    // the staging buffers are reused by the next call
    SG_CUDA(cudaStreamSynchronize(net->stream));
  });
}

int sg_step(sg_net *net, uint32_t n_steps) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "Network::step() called before build()");
    SG_REQUIRE(!has_external(net), SG_E_STATE,
               "a network with external populations steps with sg_step_begin / sg_step_end around its spike exchange");
    DevGuard g(net->device);
    if (net->profile && net->total > 0) do_steps_profiled(net, n_steps);
    else do_steps(net, n_steps);
  });
}

// Autotuning of the pre-centric scatter's schedule on the network's own
// steps: each candidate (stage ring of kRedVariants x 1..3 blocks per SM) runs
// `steps` steps after one warm-up chunk, timed with CUDA events on the
// network's stream; the fastest is kept.  On this path every schedule gives
// the same bits (the ring sums are exact, or the order is free), so the
// steps are ordinary steps of the simulation.
int sg_autotune(sg_net *net, uint32_t steps, float *fixed_ms, float *best_ms, int *best_variant,
                uint32_t *best_bps) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "autotune needs a built network");
    SG_REQUIRE(steps > 0, SG_E_INVALID, "autotune: steps must be > 0");
    SG_REQUIRE(!has_external(net) && !net->pool, SG_E_STATE,
               "autotune: the network steps on its own (not split, not in a pool)");
    DevGuard g(net->device);
    const int v0 = net->red_variant;
    const uint32_t b0 = net->red_bps;
    float fixed = 0.0f, best = 0.0f;
    int bv = 0;
    uint32_t bb = kRedBlocksPerSM;
    if (net->red) {
      const bool log = std::getenv("SG_AUTOTUNE_LOG") != nullptr;  // each candidate's time on stderr
      cudaEvent_t e0, e1;
      SG_CUDA(cudaEventCreate(&e0));
      SG_CUDA(cudaEventCreate(&e1));
      bool first = true;
      for (int v = 0; v < kNumRedVariants; ++v)
        for (uint32_t bps = 1; bps <= 3; ++bps) {
          net->red_variant = v;
          net->red_bps = bps;
          drop_graph(net);
          do_steps(net, std::min<uint32_t>(steps, 64));  // warm-up (and the graph's capture)
          SG_CUDA(cudaEventRecord(e0, net->stream));
          do_steps(net, steps);
          SG_CUDA(cudaEventRecord(e1, net->stream));
          SG_CUDA(cudaEventSynchronize(e1));
          float ms = 0.0f;
          SG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
          ms /= (float)steps;
          if (log) std::fprintf(stderr, "sg_autotune: variant %d, %u blocks per SM: %.4f ms per step\n", v, bps, ms);
          if (v == default_red_variant() && bps == kRedBlocksPerSM) fixed = ms;
          if (first || ms < best) {
            best = ms;
            bv = v;
            bb = bps;
            first = false;
          }
        }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      net->red_variant = bv;
      net->red_bps = bb;
      drop_graph(net);
    } else {
      net->red_variant = v0;
      net->red_bps = b0;
    }
    if (fixed_ms) *fixed_ms = fixed;
    if (best_ms) *best_ms = best;
    if (best_variant) *best_variant = net->red_variant;
    if (best_bps) *best_bps = net->red_bps;
  });
}

// Where an external population's spike words of each step are read (device
// memory, the population's words in the owner's bitmask order: bit i of word
// k is neuron 32k + i); read by every sg_step_end.
int sg_pop_set_external_source(sg_net *net, uint32_t pop, const uint32_t *dev_words) {
  NET_CHECK(net);
  return run([&] {
    require_pop(net, pop);
    SG_REQUIRE(net->pops[pop].external, SG_E_INVALID, "not an external population");
    net->pops[pop].ext_src = dev_words;
    drop_graph(net);
  });
}

// This step's spike words of a population (device memory; valid after
// sg_step_begin until the next sg_step_begin)
int sg_spike_words(sg_net *net, uint32_t pop, const uint32_t **dev_words) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "not built");
    require_pop(net, pop);
    SG_REQUIRE(dev_words, SG_E_INVALID, "null output");
    *dev_words = net->d_last_bits.p + net->pops[pop].dev_off / 32;
  });
}

// One step in two halves around a spike exchange: sg_step_begin updates the
// populations simulated here; sg_step_end publishes the external
// populations' spikes (from their sources), scatters and learns.  Both are
// asynchronous on the network's stream.
int sg_step_begin(sg_net *net) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "Network::step() called before build()");
    DevGuard g(net->device);
    upload_pop_table(net);
    if (net->learn_on) net->d_l_motor.zero(net->stream);
    enqueue_neurons(net, make_args(net));
    SG_CUDA(cudaGetLastError());
  });
}

int sg_step_end(sg_net *net) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "Network::step() called before build()");
    for (const auto &p : net->pops)
      SG_REQUIRE(!p.external || p.ext_src || p.n == 0, SG_E_STATE, "an external population has no spike source");
    DevGuard g(net->device);
    const StepArgs a = make_args(net);
    upload_args(net, a);
    enqueue_rest(net, a);
    SG_CUDA(cudaGetLastError());
    net->host_step += 1;
  });
}

int sg_profile_enable(sg_net *net, int on) {
  NET_CHECK(net);
  return run([&] {
    net->profile = on != 0;
    for (int i = 0; i < 4; ++i) {
      net->prof_ms[i] = 0;
      net->prof_launches[i] = 0;
    }
  });
}

int sg_profile_read(sg_net *net, double *ms, uint64_t *launches) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(ms && launches, SG_E_INVALID, "null output");
    for (int i = 0; i < 4; ++i) {
      ms[i] = net->prof_ms[i];
      launches[i] = net->prof_launches[i];
    }
  });
}

int sg_raster_enable(sg_net *net, uint32_t cap) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "raster recording needs a built network");
    SG_REQUIRE(!net->rstaged, SG_E_STATE, "a staged raster read is not fetched yet");
    DevGuard g(net->device);
    SG_CUDA(cudaStreamSynchronize(net->stream));
    drop_graph(net);
    net->raster_cap = cap;
    if (cap) {
      net->d_raster.alloc((size_t)cap * (net->Nd / 32));
      net->d_raster.zero(net->stream);
      net->rr_counts.ensure(std::max<uint32_t>(net->Nd, 1));
      SG_CUDA(cudaMemsetAsync(net->rr_counts.p, 0, (size_t)std::max<uint32_t>(net->Nd, 1) * 4, net->stream));
      SG_CUDA(cudaStreamSynchronize(net->stream));
    } else {
      net->d_raster.release();
    }
    net->raster_read_step = net->host_step;
  });
}

int sg_raster_read(sg_net *net, uint8_t *out, uint64_t cap_bytes, uint32_t *n_steps) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->raster_cap > 0, SG_E_STATE, "raster recording is not enabled");
    DevGuard g(net->device);
    const uint64_t k = net->host_step - net->raster_read_step;
    SG_REQUIRE(k <= net->raster_cap, SG_E_OVERFLOW,
               "raster overflow: " + std::to_string(k) + " steps since the last read, capacity " +
                   std::to_string(net->raster_cap));
    const uint64_t N = net->total;
    SG_REQUIRE(k * N <= cap_bytes, SG_E_INVALID, "output buffer too small");
    const uint32_t words = net->Nd / 32;
    std::vector<uint32_t> bits((size_t)net->raster_cap * words);
    SG_CUDA(cudaMemcpyAsync(bits.data(), net->d_raster.p, bits.size() * 4, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
    for (uint64_t t = 0; t < k; ++t) {
      const uint64_t step = net->raster_read_step + t;
      const uint32_t *row = bits.data() + (size_t)(step % net->raster_cap) * words;
      uint8_t *o = out + t * N;
      for (size_t p = 0; p < net->pops.size(); ++p) {
        const auto &pp = net->pops[p];
        for (uint32_t i = 0; i < pp.n; ++i) {
          const uint32_t di = pp.dev_off + i;
          o[net->offsets[p] + i] = (uint8_t)((row[di >> 5] >> (di & 31)) & 1u);
        }
      }
    }
    if (n_steps) *n_steps = (uint32_t)k;
    net->raster_read_step = net->host_step;
  });
}

namespace {

// Queues on stream s the compaction of the raster steps [t0, t0 + k): per
// block spike counts and their exclusive scan (off[nb] = the total).
void enqueue_raster_count(sg_net *net, cudaStream_t s, uint64_t t0, uint64_t nw, uint64_t nb) {
  const uint32_t words = net->Nd / 32;
  auto &cnt = net->rr_cnt;
  auto &off = net->rr_off;
  cnt.ensure(nb + 1);
  off.ensure(nb + 1);
  SG_CUDA(cudaMemsetAsync(cnt.p, 0, (nb + 1) * sizeof(unsigned long long), s));
  raster_count_kernel<<<(unsigned)nb, 256, 0, s>>>(net->d_raster.p, net->raster_cap, words, t0, nw, cnt.p);
  size_t tb = 0;
  SG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.p, off.p, (int64_t)nb + 1, s));
  auto &temp = net->rr_temp;
  temp.ensure(std::max<size_t>(tb, 1));
  SG_CUDA(cub::DeviceScan::ExclusiveSum(temp.p, tb, cnt.p, off.p, (int64_t)nb + 1, s));
}

// The population tables of the write kernel (device offset -> global offset).
void upload_raster_pops(sg_net *net, cudaStream_t s) {
  std::vector<uint32_t> pd, pgl;
  for (size_t p = 0; p < net->pops.size(); ++p) {
    pd.push_back(net->pops[p].dev_off);
    pgl.push_back(net->offsets[p]);
  }
  net->rr_pd.ensure(pd.size());
  net->rr_pg.ensure(pgl.size());
  SG_CUDA(cudaMemcpyAsync(net->rr_pd.p, pd.data(), pd.size() * 4, cudaMemcpyHostToDevice, s));
  SG_CUDA(cudaMemcpyAsync(net->rr_pg.p, pgl.data(), pgl.size() * 4, cudaMemcpyHostToDevice, s));
  SG_CUDA(cudaStreamSynchronize(s));  // the host vectors go out of scope
}

// Queues the write of the scanned batch into rr_step / rr_idx (which hold
// `out_cap` pairs) and the per-neuron counts; skipped on the device when the
// total exceeds out_cap.
void enqueue_raster_write(sg_net *net, cudaStream_t s, uint64_t t0, uint64_t nw, uint64_t nb, uint64_t out_cap) {
  raster_write_kernel<<<(unsigned)nb, 256, 0, s>>>(net->d_raster.p, net->raster_cap, net->Nd / 32, t0, nw,
                                                   net->rr_off.p, nb, out_cap, net->rr_pd.p, net->rr_pg.p,
                                                   (int)net->pops.size(), net->rr_step.p, net->rr_idx.p,
                                                   net->rr_counts.p);
  SG_CUDA(cudaGetLastError());
}

}  // namespace

int sg_raster_read_events(sg_net *net, uint32_t *steps, uint32_t *idx, uint64_t cap, uint64_t *n_out) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->raster_cap > 0, SG_E_STATE, "raster recording is not enabled");
    SG_REQUIRE(n_out, SG_E_INVALID, "null output");
    SG_REQUIRE(!net->rstaged, SG_E_STATE, "a staged raster read is not fetched yet");
    DevGuard g(net->device);
    cudaStream_t s = net->stream;
    const uint64_t k = net->host_step - net->raster_read_step;
    SG_REQUIRE(k <= net->raster_cap, SG_E_OVERFLOW,
               "raster overflow: " + std::to_string(k) + " steps since the last read, capacity " +
                   std::to_string(net->raster_cap));
    const uint64_t nw = k * (net->Nd / 32);
    const uint64_t nb = (nw + kRasterWordsPerBlock - 1) / kRasterWordsPerBlock;
    *n_out = 0;
    if (nb == 0) {
      net->raster_read_step = net->host_step;
      return;
    }
    // work buffers live in the network and only grow: no allocation in a
    // steady read loop
    enqueue_raster_count(net, s, net->raster_read_step, nw, nb);
    unsigned long long total = 0;
    SG_CUDA(cudaMemcpyAsync(&total, net->rr_off.p + nb, 8, cudaMemcpyDeviceToHost, s));
    SG_CUDA(cudaStreamSynchronize(s));
    *n_out = total;
    SG_REQUIRE(total <= cap, SG_E_INVALID, "output buffer too small: " + std::to_string(total) + " spikes");
    if (total == 0) {
      net->raster_read_step = net->host_step;
      return;
    }
    upload_raster_pops(net, s);
    net->rr_step.ensure(total);
    net->rr_idx.ensure(total);
    enqueue_raster_write(net, s, net->raster_read_step, nw, nb, total);
    if (steps) SG_CUDA(cudaMemcpyAsync(steps, net->rr_step.p, total * 4, cudaMemcpyDeviceToHost, s));
    if (idx) SG_CUDA(cudaMemcpyAsync(idx, net->rr_idx.p, total * 4, cudaMemcpyDeviceToHost, s));
    SG_CUDA(cudaStreamSynchronize(s));
    net->raster_read_step = net->host_step;
  });
}

// Staged raster read, for a loop that keeps the GPU stepping while it reads:
// the steps recorded since the last read are compacted on the network's read
// stream right after the steps that wrote them (the network's next steps
// wait for that compaction, so the raster slots may be reused at once), and
// sg_raster_fetch later copies the pairs out.  Nothing here waits.
int sg_raster_stage(sg_net *net) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->raster_cap > 0, SG_E_STATE, "raster recording is not enabled");
    SG_REQUIRE(!net->rstaged, SG_E_STATE, "the last staged raster read is not fetched yet");
    const uint64_t k = net->host_step - net->raster_read_step;
    SG_REQUIRE(k <= net->raster_cap, SG_E_OVERFLOW,
               "raster overflow: " + std::to_string(k) + " steps since the last read, capacity " +
                   std::to_string(net->raster_cap));
    DevGuard g(net->device);
    if (!net->rstream) {
      SG_CUDA(cudaStreamCreateWithFlags(&net->rstream, cudaStreamNonBlocking));
      SG_CUDA(cudaEventCreateWithFlags(&net->rev, cudaEventDisableTiming));
      SG_CUDA(cudaEventCreateWithFlags(&net->rdone, cudaEventDisableTiming));
      SG_CUDA(cudaMallocHost(&net->rst_total, sizeof(unsigned long long)));
      upload_raster_pops(net, net->rstream);
    }
    const uint64_t nw = k * (net->Nd / 32);
    const uint64_t nb = (nw + kRasterWordsPerBlock - 1) / kRasterWordsPerBlock;
    net->rst_t0 = net->raster_read_step;
    net->rst_nw = nw;
    net->rst_nb = nb;
    *net->rst_total = 0;
    net->raster_read_step = net->host_step;
    net->rstaged = true;
    if (nb == 0) return;
    // the pool's steps of a member are followed on the member's stream (a
    // pool step ends with the member streams waiting for it)
    SG_CUDA(cudaEventRecord(net->rev, net->stream));
    SG_CUDA(cudaStreamWaitEvent(net->rstream, net->rev, 0));
    cudaStream_t rs = net->rstream;
    enqueue_raster_count(net, rs, net->rst_t0, nw, nb);
    // output room for 1/128 of the steps' neuron slots to begin with (fetch
    // grows it when a batch has more spikes)
    const uint64_t room = std::max<uint64_t>(net->rr_step.n, std::max<uint64_t>(nw / 4, 1u << 15));
    net->rr_step.ensure(room);
    net->rr_idx.ensure(room);
    enqueue_raster_write(net, rs, net->rst_t0, nw, nb, net->rr_step.n);
    SG_CUDA(cudaMemcpyAsync(net->rst_total, net->rr_off.p + nb, 8, cudaMemcpyDeviceToHost, rs));
    SG_CUDA(cudaEventRecord(net->rdone, rs));
    SG_CUDA(cudaStreamWaitEvent(net->stream, net->rdone, 0));
  });
}

int sg_raster_fetch(sg_net *net, uint32_t *steps, uint32_t *idx, uint64_t cap, uint64_t *n_out) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(n_out, SG_E_INVALID, "null output");
    SG_REQUIRE(net->rstaged, SG_E_STATE, "no staged raster read");
    *n_out = 0;
    if (net->rst_nb == 0) {
      net->rstaged = false;
      return;
    }
    DevGuard g(net->device);
    cudaStream_t rs = net->rstream;
    SG_CUDA(cudaStreamSynchronize(rs));
    const uint64_t total = *net->rst_total;
    *n_out = total;
    SG_REQUIRE(total <= cap, SG_E_INVALID, "output buffer too small: " + std::to_string(total) + " spikes");
    if (total > net->rr_step.n) {  // the write was skipped: grow the room and write now
      net->rr_step.ensure(total + total / 4);
      net->rr_idx.ensure(total + total / 4);
      enqueue_raster_write(net, rs, net->rst_t0, net->rst_nw, net->rst_nb, net->rr_step.n);
    }
    if (total) {
      if (steps) SG_CUDA(cudaMemcpyAsync(steps, net->rr_step.p, total * 4, cudaMemcpyDeviceToHost, rs));
      if (idx) SG_CUDA(cudaMemcpyAsync(idx, net->rr_idx.p, total * 4, cudaMemcpyDeviceToHost, rs));
    }
    SG_CUDA(cudaStreamSynchronize(rs));
    net->rstaged = false;
  });
}

int sg_raster_fetch_csr(sg_net *net, uint32_t *step_off, uint64_t off_cap, uint32_t *idx, uint64_t cap,
                        uint64_t *t0, uint64_t *n_steps, uint64_t *n_out) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(t0 && n_steps && n_out, SG_E_INVALID, "null output");
    SG_REQUIRE(net->rstaged, SG_E_STATE, "no staged raster read");
    const uint64_t words = net->Nd / 32;
    const uint64_t k = words ? net->rst_nw / words : 0;
    *t0 = net->rst_t0;
    *n_steps = k;
    *n_out = 0;
    SG_REQUIRE(off_cap >= k + 1, SG_E_INVALID, "step offset buffer too small: " + std::to_string(k + 1));
    SG_REQUIRE(step_off, SG_E_INVALID, "null step offsets");
    DevGuard g(net->device);
    if (net->rst_nb == 0) {
      for (uint64_t i = 0; i <= k; ++i) step_off[i] = 0;
      net->rstaged = false;
      return;
    }
    cudaStream_t rs = net->rstream;
    SG_CUDA(cudaStreamSynchronize(rs));
    const uint64_t total = *net->rst_total;
    *n_out = total;
    SG_REQUIRE(total <= cap, SG_E_INVALID, "output buffer too small: " + std::to_string(total) + " spikes");
    SG_REQUIRE(total < 0xFFFFFFFFull, SG_E_OVERFLOW, "more than 2^32-2 spikes in one staged read");
    if (total > net->rr_step.n) {  // the write was skipped: grow the room and write now
      net->rr_step.ensure(total + total / 4);
      net->rr_idx.ensure(total + total / 4);
      enqueue_raster_write(net, rs, net->rst_t0, net->rst_nw, net->rst_nb, net->rr_step.n);
    }
    net->rr_soff.ensure(k + 1);
    raster_step_off_kernel<<<(unsigned)((k + 256) / 256), 256, 0, rs>>>(net->rr_step.p, total, net->rst_t0, k,
                                                                        net->rr_soff.p);
    SG_CUDA(cudaGetLastError());
    SG_CUDA(cudaMemcpyAsync(step_off, net->rr_soff.p, (k + 1) * 4, cudaMemcpyDeviceToHost, rs));
    if (total) {
      SG_REQUIRE(idx, SG_E_INVALID, "null output");
      SG_CUDA(cudaMemcpyAsync(idx, net->rr_idx.p, total * 4, cudaMemcpyDeviceToHost, rs));
    }
    SG_CUDA(cudaStreamSynchronize(rs));
    net->rstaged = false;
  });
}

int sg_host_alloc(uint64_t bytes, void **out) {
  return run([&] {
    SG_REQUIRE(out, SG_E_INVALID, "null output");
    *out = nullptr;
    if (bytes) SG_CUDA(cudaHostAlloc(out, bytes, cudaHostAllocPortable));
  });
}

int sg_host_free(void *p) {
  return run([&] {
    if (p) SG_CUDA(cudaFreeHost(p));
  });
}

// Spikes per neuron (reference order) over every event read since the
// raster was enabled.
int sg_raster_counts(sg_net *net, uint32_t *counts) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->raster_cap > 0 && net->rr_counts.p, SG_E_STATE, "raster recording is not enabled");
    SG_REQUIRE(!net->rstaged, SG_E_STATE, "a staged raster read is not fetched yet");
    SG_REQUIRE(counts, SG_E_INVALID, "null output");
    DevGuard g(net->device);
    std::vector<uint32_t> c(net->Nd);
    SG_CUDA(cudaMemcpyAsync(c.data(), net->rr_counts.p, (size_t)net->Nd * 4, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
    for (size_t p = 0; p < net->pops.size(); ++p)
      for (uint32_t i = 0; i < net->pops[p].n; ++i) counts[net->offsets[p] + i] = c[net->pops[p].dev_off + i];
  });
}

int sg_stats_read(sg_net *net, uint32_t *spikes, uint64_t *events, uint32_t cap, uint32_t *n_steps) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "not built");
    DevGuard g(net->device);
    const uint64_t k = net->host_step - net->stat_read_step;
    SG_REQUIRE(k <= net->stat_cap, SG_E_OVERFLOW, "stats overflow");
    SG_REQUIRE(k <= cap, SG_E_INVALID, "output buffer too small");
    std::vector<uint32_t> s(net->stat_cap);
    std::vector<unsigned long long> e(net->stat_cap);
    SG_CUDA(cudaMemcpyAsync(s.data(), net->d_stat_spk.p, s.size() * 4, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaMemcpyAsync(e.data(), net->d_stat_ev.p, e.size() * 8, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
    for (uint64_t t = 0; t < k; ++t) {
      const uint64_t st = net->stat_read_step + t;
      if (spikes) spikes[t] = s[st % net->stat_cap];
      if (events) events[t] = e[st % net->stat_cap];
    }
    if (n_steps) *n_steps = (uint32_t)k;
    net->stat_read_step = net->host_step;
  });
}

int sg_spikes(sg_net *net, uint32_t pop, int32_t *out, uint32_t n) {
  NET_CHECK(net);
  return run([&] {
    require_pop(net, pop);
    const auto &p = net->pops[pop];
    SG_REQUIRE(out && n == p.n, SG_E_INVALID, "output length does not match population size");
    if (!net->built) {
      std::memset(out, 0, (size_t)n * 4);
      return;
    }
    DevGuard g(net->device);
    const uint32_t w0 = p.dev_off / 32, nw = p.cap / 32;
    std::vector<uint32_t> bits(std::max<uint32_t>(nw, 1));
    if (nw) SG_CUDA(cudaMemcpyAsync(bits.data(), net->d_last_bits.p + w0, (size_t)nw * 4, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
    for (uint32_t i = 0; i < p.n; ++i) out[i] = (int32_t)((bits[i >> 5] >> (i & 31)) & 1u);
  });
}

int sg_step_counter(sg_net *net, uint64_t *out) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(out, SG_E_INVALID, "null output");
    *out = net->host_step;
  });
}

int sg_total_neurons(sg_net *net, uint64_t *out) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(out, SG_E_INVALID, "null output");
    *out = net->total;
  });
}

int sg_num_synapses(sg_net *net, uint64_t *out) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(out, SG_E_INVALID, "null output");
    *out = net->built ? net->n_edges : net->e_pre.n;
  });
}

int sg_events_total(sg_net *net, uint64_t *out) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(out, SG_E_INVALID, "null output");
    if (!net->built) {
      *out = 0;
      return;
    }
    DevGuard g(net->device);
    unsigned long long v = 0;
    SG_CUDA(cudaMemcpyAsync(&v, net->d_ev_total.p, 8, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
    *out = v;
  });
}

int sg_source_events_total(sg_net *net, uint64_t *out) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(out, SG_E_INVALID, "null output");
    if (!net->built) {
      *out = 0;
      return;
    }
    DevGuard g(net->device);
    unsigned long long v = 0;
    SG_CUDA(cudaMemcpyAsync(&v, net->d_ev_src.p + 1, 8, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
    *out = v;
  });
}

static void read_csr_global(sg_net *net, uint32_t *row_ptr, uint32_t *col, float *w, uint8_t *d, bool only_w,
                            uint8_t *syn = nullptr, uint8_t *plastic = nullptr) {
  const uint32_t Nd = net->Nd;
  const uint64_t E = net->n_edges;
  std::vector<uint32_t> rp(Nd + 1);
  std::vector<uint2> ed(E);
  std::vector<uint8_t> code(net->packed ? 0 : E);
  SG_CUDA(cudaMemcpyAsync(rp.data(), net->d_row_ptr.p, ((size_t)Nd + 1) * 4, cudaMemcpyDeviceToHost, net->stream));
  if (E && net->weight_format == SG_W_FP8) {
    std::vector<uint32_t> ex(E);
    std::vector<uint8_t> w8(E);
    std::vector<float> sc(Nd);
    SG_CUDA(cudaMemcpyAsync(ex.data(), net->d_edge_x.p, E * 4, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaMemcpyAsync(w8.data(), net->d_w8.p, E, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaMemcpyAsync(sc.data(), net->d_row_scale.p, (size_t)Nd * 4, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
    for (uint32_t r = 0; r < Nd; ++r)
      for (uint64_t e = rp[r]; e < rp[r + 1]; ++e) {
        const float v = host_e4m3(w8[e]) * sc[r];
        uint32_t bits;
        std::memcpy(&bits, &v, 4);
        ed[e] = make_uint2(ex[e], bits);
      }
    if (!net->packed && !only_w)
      SG_CUDA(cudaMemcpyAsync(code.data(), net->d_code.p, E, cudaMemcpyDeviceToHost, net->stream));
  } else if (E && net->weight_format == SG_W_BF16) {
    std::vector<uint32_t> ex(E);
    std::vector<uint16_t> w16(E);
    SG_CUDA(cudaMemcpyAsync(ex.data(), net->d_edge_x.p, E * 4, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaMemcpyAsync(w16.data(), net->d_w16.p, E * 2, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
    for (uint64_t e = 0; e < E; ++e) ed[e] = make_uint2(ex[e], (uint32_t)w16[e] << 16);
    if (!net->packed && !only_w)
      SG_CUDA(cudaMemcpyAsync(code.data(), net->d_code.p, E, cudaMemcpyDeviceToHost, net->stream));
  } else if (E) {
    SG_CUDA(cudaMemcpyAsync(ed.data(), net->d_edge.p, E * 8, cudaMemcpyDeviceToHost, net->stream));
    if (!net->packed && !only_w)
      SG_CUDA(cudaMemcpyAsync(code.data(), net->d_code.p, E, cudaMemcpyDeviceToHost, net->stream));
  }
  SG_CUDA(cudaStreamSynchronize(net->stream));
  for (uint64_t e = 0; e < E; ++e) std::memcpy(&w[e], &ed[e].y, 4);
  if (only_w) return;
  // device index -> global index
  std::vector<uint32_t> d2g(Nd, 0xFFFFFFFFu);
  for (size_t p = 0; p < net->pops.size(); ++p)
    for (uint32_t i = 0; i < net->pops[p].n; ++i) d2g[net->pops[p].dev_off + i] = net->offsets[p] + i;
  // padding rows are empty, so the global row_ptr is the device one restricted
  for (size_t p = 0; p < net->pops.size(); ++p)
    for (uint32_t i = 0; i < net->pops[p].n; ++i) row_ptr[net->offsets[p] + i] = rp[net->pops[p].dev_off + i];
  row_ptr[net->total] = (uint32_t)E;
  for (uint64_t e = 0; e < E; ++e) {
    const uint32_t post = net->packed ? (ed[e].x & 0x00FFFFFFu) : ed[e].x;
    const uint8_t c = net->packed ? (uint8_t)(ed[e].x >> 24) : code[e];
    col[e] = d2g[post];
    if (net->receptor) {  // the delay field holds 1 + the receptor code; delays are not kept
      d[e] = 0;
      if (syn) syn[e] = (uint8_t)(code_delay(c) - 1u);
      if (plastic) plastic[e] = 0;
      continue;
    }
    d[e] = (uint8_t)code_delay(c);
    if (syn) syn[e] = (uint8_t)code_ring(c);
    if (plastic) plastic[e] = code_stdp(c) ? 1 : 0;
  }
}

int sg_graph_read(sg_net *net, uint32_t *row_ptr, uint32_t *col, float *w, uint8_t *d) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "not built");
    SG_REQUIRE(row_ptr && col && w && d, SG_E_INVALID, "null output");
    DevGuard g(net->device);
    read_csr_global(net, row_ptr, col, w, d, false);
  });
}

int sg_graph_read_types(sg_net *net, uint8_t *syn_types, uint8_t *stdp) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "not built");
    SG_REQUIRE(syn_types && stdp, SG_E_INVALID, "null output");
    DevGuard g(net->device);
    std::vector<uint32_t> rp(net->total + 1), col(net->n_edges);
    std::vector<float> w(net->n_edges);
    std::vector<uint8_t> d(net->n_edges);
    read_csr_global(net, rp.data(), col.data(), w.data(), d.data(), false, syn_types, stdp);
  });
}

int sg_weights_read(sg_net *net, float *w) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "not built");
    SG_REQUIRE(w, SG_E_INVALID, "null output");
    DevGuard g(net->device);
    read_csr_global(net, nullptr, nullptr, w, nullptr, true);
  });
}

int sg_ring_read(sg_net *net, uint32_t ring, float *out) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "not built");
    SG_REQUIRE(ring <= net->kin.size(), SG_E_INVALID, "ring out of range");
    SG_REQUIRE(out, SG_E_INVALID, "null output");
    SG_REQUIRE(!net->receptor, SG_E_STATE, "receptor kinetics: read the conductances (sg_receptor_read)");
    DevGuard g(net->device);
    const uint32_t Nd = net->Nd, M = net->nslots;
    fold_drive(net);
    std::vector<float> r((size_t)M * Nd);
    SG_CUDA(cudaMemcpyAsync(r.data(), net->d_ring.p + (size_t)ring * M * Nd, r.size() * 4,
                            cudaMemcpyDeviceToHost, net->stream));
    unsigned long long step = 0;
    SG_CUDA(cudaMemcpyAsync(&step, net->d_step.p, sizeof(step), cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
    // reference slot s holds the arrivals of the step t in [step, step + 31]
    // with t % 32 == s; the device keeps t in slot t % M while t - step < M,
    // and no arrival lies further ahead
    const uint64_t N = net->total;
    for (uint32_t s = 0; s < kSlots; ++s) {
      const unsigned long long t = step + ((s + kSlots - (uint32_t)(step % kSlots)) % kSlots);
      const bool held = t - step < M;
      const uint32_t ds = (uint32_t)(t % M);
      for (size_t p = 0; p < net->pops.size(); ++p)
        for (uint32_t i = 0; i < net->pops[p].n; ++i)
          out[(size_t)s * N + net->offsets[p] + i] = held ? r[(size_t)ds * Nd + net->pops[p].dev_off + i] : 0.0f;
    }
  });
}

int sg_neuron_stats_enable(sg_net *net, int on) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "not built");
    DevGuard g(net->device);
    cudaStream_t s = net->stream;
    SG_CUDA(cudaStreamSynchronize(s));
    drop_graph(net);
    if (!on) {
      net->d_ns_count.release();
      net->d_ns_last.release();
      net->d_ns_s1.release();
      net->d_ns_s2.release();
      return;
    }
    const uint32_t Nd = net->Nd;
    net->d_ns_count.alloc(Nd);
    net->d_ns_last.alloc(Nd);
    net->d_ns_s1.alloc(Nd);
    net->d_ns_s2.alloc(Nd);
    net->d_ns_count.zero(s);
    SG_CUDA(cudaMemsetAsync(net->d_ns_last.p, 0xFF, (size_t)Nd * 4, s));
    net->d_ns_s1.zero(s);
    net->d_ns_s2.zero(s);
    SG_CUDA(cudaMemcpyAsync(&net->ns_step0, net->d_step.p, 8, cudaMemcpyDeviceToHost, s));
    SG_CUDA(cudaStreamSynchronize(s));
  });
}

int sg_neuron_stats_read(sg_net *net, uint32_t pop, uint32_t *counts, double *isi_mean, double *isi_cv,
                         uint64_t *steps) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->d_ns_count.n, SG_E_STATE, "neuron statistics are not enabled");
    require_pop(net, pop);
    SG_REQUIRE(counts && isi_mean && isi_cv && steps, SG_E_INVALID, "null output");
    DevGuard g(net->device);
    cudaStream_t s = net->stream;
    const HostPop &p = net->pops[pop];
    std::vector<uint32_t> c(p.n);
    std::vector<double> s1(p.n), s2(p.n);
    unsigned long long step = 0;
    if (p.n) {
      SG_CUDA(cudaMemcpyAsync(c.data(), net->d_ns_count.p + p.dev_off, (size_t)p.n * 4, cudaMemcpyDeviceToHost, s));
      SG_CUDA(cudaMemcpyAsync(s1.data(), net->d_ns_s1.p + p.dev_off, (size_t)p.n * 8, cudaMemcpyDeviceToHost, s));
      SG_CUDA(cudaMemcpyAsync(s2.data(), net->d_ns_s2.p + p.dev_off, (size_t)p.n * 8, cudaMemcpyDeviceToHost, s));
    }
    SG_CUDA(cudaMemcpyAsync(&step, net->d_step.p, 8, cudaMemcpyDeviceToHost, s));
    SG_CUDA(cudaStreamSynchronize(s));
    for (uint32_t i = 0; i < p.n; ++i) {
      counts[i] = c[i];
      const double k = c[i] ? (double)(c[i] - 1) : 0.0;  // intervals
      isi_mean[i] = k > 0 ? s1[i] / k : 0.0;
      // sample variance of the intervals (P/kernels/stats/isi.rs:30-66: >= 2 intervals)
      const double var = k >= 2 ? (s2[i] - s1[i] * s1[i] / k) / (k - 1.0) : 0.0;
      isi_cv[i] = (k >= 2 && isi_mean[i] > 0) ? std::sqrt(std::max(var, 0.0)) / isi_mean[i] : 0.0;
    }
    *steps = step - net->ns_step0;
  });
}

int sg_stdp_drift(sg_net *net, double *out) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built && net->stdp_on, SG_E_STATE, "STDP is not enabled");
    DevGuard g(net->device);
    SG_CUDA(cudaMemcpyAsync(out, net->d_drift.p, 8, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
  });
}

int sg_stdp_traces(sg_net *net, float *x_pre, float *x_post) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built && net->stdp_on, SG_E_STATE, "STDP is not enabled");
    DevGuard g(net->device);
    std::vector<float> a(net->Nd), b(net->Nd);
    SG_CUDA(cudaMemcpyAsync(a.data(), net->d_x_pre.p, a.size() * 4, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaMemcpyAsync(b.data(), net->d_x_post.p, b.size() * 4, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
    for (size_t p = 0; p < net->pops.size(); ++p)
      for (uint32_t i = 0; i < net->pops[p].n; ++i) {
        x_pre[net->offsets[p] + i] = a[net->pops[p].dev_off + i];
        x_post[net->offsets[p] + i] = b[net->pops[p].dev_off + i];
      }
  });
}

int sg_clamp_hits(sg_net *net, uint64_t *out) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "not built");
    DevGuard g(net->device);
    unsigned long long v = 0;
    SG_CUDA(cudaMemcpyAsync(&v, net->d_clamp.p, 8, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
    *out = v;
  });
}

// ---------------------------------------------------------------------------
// Dopamine-modulated eligibility learning over the built network's synapses
// (P/api/learn/brain.rs Brain, bound to the network as
// pillars-wgpu/src/network.rs:902-1336 step_many_learn / reward do).  The
// synapse index is the CSR record index, the order sg_graph_read reports.
// ---------------------------------------------------------------------------
static void require_learn(const sg_net *net) {
  SG_REQUIRE(net->built && net->learn_on, SG_E_STATE, "learning is not enabled");
}

static unsigned learn_blocks(uint64_t E) {
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((E + 255) / 256, 148u * 16u));
}

int sg_learn_enable(sg_net *net, float dt, float tau_pre, float tau_post, float tau_e, float a_ltp, float a_ltd,
                    float lr, float w_min, float w_max) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "learning needs a built network");
    SG_REQUIRE(!net->learn_on, SG_E_STATE, "learning is already enabled");
    SG_REQUIRE(!net->receptor, SG_E_STATE, "receptor kinetics: learning is not available");
    SG_REQUIRE(net->weight_format == SG_W_F32, SG_E_INVALID,
               "BF16 and FP8 weights are read-only: learning needs FP32 weights");
    const float v[9] = {dt, tau_pre, tau_post, tau_e, a_ltp, a_ltd, lr, w_min, w_max};
    for (float x : v) SG_REQUIRE(std::isfinite(x), SG_E_INVALID, "learning config: values must be finite");
    SG_REQUIRE(dt > 0 && tau_pre > 0 && tau_post > 0 && tau_e > 0 && w_min <= w_max, SG_E_INVALID,
               "learning config: dt and time constants must be positive and w_min <= w_max");
    DevGuard g(net->device);
    cudaStream_t s = net->stream;
    // rewards change weights, so the exact-sum condition of the rings no
    // longer holds: the ordered path takes over
    net->exact = false;
    update_path(net);
    drop_graph(net);
    const uint32_t Nd = net->Nd;
    const uint64_t E = net->n_edges;
    net->l_dt = dt, net->l_tau_pre = tau_pre, net->l_tau_post = tau_post, net->l_tau_e = tau_e;
    net->l_a_ltp = a_ltp, net->l_a_ltd = a_ltd, net->l_lr = lr, net->l_w_min = w_min, net->l_w_max = w_max;
    // the per-step factors (brain.rs:206-208)
    net->l_dpre = host_fast_exp(-dt / tau_pre);
    net->l_dpost = host_fast_exp(-dt / tau_post);
    net->l_de = host_fast_exp(-dt / tau_e);
    net->d_l_tp.alloc(std::max<uint32_t>(Nd, 1));
    net->d_l_tp.zero(s);
    net->d_l_tq.alloc(std::max<uint32_t>(Nd, 1));
    net->d_l_tq.zero(s);
    net->d_l_st.alloc(std::max<uint64_t>(E, 1));
    net->d_l_st.zero(s);
    net->d_l_flat.alloc(std::max<uint32_t>(Nd, 1));
    net->d_l_ctr.alloc(2 + kLearnBuckets);
    net->d_l_ctr.zero(s);
    // long-gap queue: per bucket room for 1/64 of the synapses (4M at most,
    // 64K at least); a synapse that finds its bucket full decays in place
    net->l_qcap = (uint32_t)std::min<uint64_t>(1u << 22, std::max<uint64_t>(E / 64, 1u << 16));
    net->d_l_qa.alloc((size_t)kLearnBuckets * net->l_qcap);
    net->d_l_qb.alloc((size_t)kLearnBuckets * net->l_qcap);
    net->d_l_motor.alloc(2);
    net->d_l_motor.zero(s);
    for (auto &m : net->l_motor) m = 0;
    if (Nd) build_in_edges(net, 1, net->d_l_in_ptr, net->d_l_in_edge, net->d_l_in_pre);
    SG_CUDA(cudaMemcpyAsync(&net->l_t0, net->d_step.p, 8, cudaMemcpyDeviceToHost, s));
    SG_CUDA(cudaStreamSynchronize(s));
    net->learn_on = true;
  });
}

// Reward of the synapses [lo, hi) only: in a pool of independent networks
// (populations without synapses between them, e.g. creatures of one arena)
// a network's synapses are one CSR range, and this is its own Brain's reward
// (the per-block reward the reference's one-scalar shader lacks,
// dioma-engine/src/brain/dynamics/gpu_pool.rs:12-16).
int sg_learn_reward_range(sg_net *net, uint64_t lo, uint64_t hi, float dopamine, float gate, float w_cap) {
  NET_CHECK(net);
  return run([&] {
    require_learn(net);
    SG_REQUIRE(lo <= hi && hi <= net->n_edges, SG_E_INVALID, "synapse range out of bounds");
    const float w_max = std::isfinite(w_cap) ? w_cap : net->l_w_max;
    SG_REQUIRE(net->l_w_min <= w_max, SG_E_INVALID, "reward: weight ceiling below the floor");
    DevGuard g(net->device);
    // reward_gated: dopamine * gate.clamp(0, 1) (brain.rs:405-409), then lr * dopamine
    const float gc = gate < 0.0f ? 0.0f : (gate > 1.0f ? 1.0f : gate);
    const float dop = dopamine * gc;
    const float lr_dopa = net->l_lr * dop;
    const uint64_t E = hi - lo;
    if (E)
      learn_reward_kernel<<<learn_blocks(E), 256, 0, net->stream>>>(net->d_edge.p + lo, net->d_l_st.p + lo,
                                                                     net->d_step.p, net->l_t0, E, net->l_de, lr_dopa,
                                                                     net->l_w_min, w_max);
    SG_CUDA(cudaGetLastError());
  });
}

int sg_learn_reward(sg_net *net, float dopamine, float gate, float w_cap) {
  NET_CHECK(net);
  return sg_learn_reward_range(net, 0, net->n_edges, dopamine, gate, w_cap);
}

int sg_learn_clear_range(sg_net *net, uint64_t lo, uint64_t hi) {
  NET_CHECK(net);
  return run([&] {
    require_learn(net);
    SG_REQUIRE(lo <= hi && hi <= net->n_edges, SG_E_INVALID, "synapse range out of bounds");
    DevGuard g(net->device);
    const uint64_t E = hi - lo;
    if (E)
      learn_clear_kernel<<<learn_blocks(E), 256, 0, net->stream>>>(net->d_l_st.p + lo, nullptr, net->d_step.p,
                                                                    net->l_t0, E);
    SG_CUDA(cudaGetLastError());
  });
}

int sg_learn_clear(sg_net *net) {
  NET_CHECK(net);
  return sg_learn_clear_range(net, 0, net->n_edges);
}

// the CSR synapse range [lo, hi) of a population's rows
int sg_pop_synapse_range(sg_net *net, uint32_t pop, uint64_t *lo, uint64_t *hi) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "not built");
    require_pop(net, pop);
    SG_REQUIRE(lo && hi, SG_E_INVALID, "null output");
    DevGuard g(net->device);
    uint32_t r[2] = {0, 0};
    const uint32_t d0 = net->pops[pop].dev_off;
    SG_CUDA(cudaMemcpyAsync(&r[0], net->d_row_ptr.p + d0, 4, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaMemcpyAsync(&r[1], net->d_row_ptr.p + d0 + net->pops[pop].n, 4, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
    *lo = r[0];
    *hi = r[1];
  });
}

int sg_learn_restrict(sg_net *net, const uint8_t *keep, uint64_t n) {
  NET_CHECK(net);
  return run([&] {
    require_learn(net);
    const uint64_t E = net->n_edges;
    SG_REQUIRE(n == E, SG_E_INVALID, "restrict: mask length differs from the synapse count");
    SG_REQUIRE(keep || E == 0, SG_E_INVALID, "null mask");
    if (!E) return;
    DevGuard g(net->device);
    DBuf<uint8_t> k;
    k.alloc(E);
    SG_CUDA(cudaMemcpyAsync(k.p, keep, E, cudaMemcpyHostToDevice, net->stream));
    learn_clear_kernel<<<learn_blocks(E), 256, 0, net->stream>>>(net->d_l_st.p, k.p, net->d_step.p, net->l_t0, E);
    SG_CUDA(cudaGetLastError());
    SG_CUDA(cudaStreamSynchronize(net->stream));
  });
}

int sg_learn_set_eligibility(sg_net *net, const float *elig, uint64_t n) {
  NET_CHECK(net);
  return run([&] {
    require_learn(net);
    const uint64_t E = net->n_edges;
    SG_REQUIRE(n == E, SG_E_INVALID, "set_eligibility: length differs from the synapse count");
    SG_REQUIRE(elig || E == 0, SG_E_INVALID, "null input");
    if (!E) return;
    DevGuard g(net->device);
    // eligibility into the x words of the state records; sync steps kept
    SG_CUDA(cudaMemcpy2DAsync(net->d_l_st.p, 8, elig, 4, 4, E, cudaMemcpyHostToDevice, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
  });
}

// a global neuron index -> the device index of the first neuron at or after
// it (padding neurons never fire, so ranges map exactly)
static uint32_t dev_bound(const sg_net *net, uint64_t x) {
  for (size_t p = 0; p < net->pops.size(); ++p)
    if (x < (uint64_t)net->offsets[p] + net->pops[p].n) {
      const uint64_t r = x > net->offsets[p] ? x - net->offsets[p] : 0;
      return net->pops[p].dev_off + (uint32_t)r;
    }
  return net->Nd;
}

int sg_learn_motor(sg_net *net, uint64_t lo0, uint64_t hi0, uint64_t lo1, uint64_t hi1) {
  NET_CHECK(net);
  return run([&] {
    require_learn(net);
    net->l_motor[0] = dev_bound(net, lo0);
    net->l_motor[1] = dev_bound(net, hi0);
    net->l_motor[2] = dev_bound(net, lo1);
    net->l_motor[3] = dev_bound(net, hi1);
    drop_graph(net);
  });
}

int sg_learn_motor_read(sg_net *net, uint32_t *out) {
  NET_CHECK(net);
  return run([&] {
    require_learn(net);
    SG_REQUIRE(out, SG_E_INVALID, "null output");
    DevGuard g(net->device);
    SG_CUDA(cudaMemcpyAsync(out, net->d_l_motor.p, 8, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
  });
}

int sg_learn_snapshot(sg_net *net) {
  NET_CHECK(net);
  return run([&] {
    require_learn(net);
    const uint64_t E = net->n_edges;
    if (!E) return;
    DevGuard g(net->device);
    net->d_l_baked.alloc(E);
    learn_baked_kernel<<<learn_blocks(E), 256, 0, net->stream>>>(net->d_edge.p, net->d_l_baked.p, E, 0, 0.0f);
    SG_CUDA(cudaGetLastError());
  });
}

int sg_learn_recall(sg_net *net, float alpha) {
  NET_CHECK(net);
  return run([&] {
    require_learn(net);
    const uint64_t E = net->n_edges;
    if (!E || !net->d_l_baked.n) return;  // no snapshot: nothing to pull toward (brain.rs:350-356)
    DevGuard g(net->device);
    learn_baked_kernel<<<learn_blocks(E), 256, 0, net->stream>>>(net->d_edge.p, net->d_l_baked.p, E, 1, alpha);
    SG_CUDA(cudaGetLastError());
  });
}

int sg_learn_read(sg_net *net, float *elig, float *trace_pre, float *trace_post, uint64_t *t) {
  NET_CHECK(net);
  return run([&] {
    require_learn(net);
    DevGuard g(net->device);
    cudaStream_t s = net->stream;
    const uint64_t E = net->n_edges;
    if (elig && E) SG_CUDA(cudaMemcpy2DAsync(elig, 4, net->d_l_st.p, 8, 4, E, cudaMemcpyDeviceToHost, s));
    std::vector<float> a(net->Nd), b(net->Nd);
    if (net->Nd) {
      SG_CUDA(cudaMemcpyAsync(a.data(), net->d_l_tp.p, a.size() * 4, cudaMemcpyDeviceToHost, s));
      SG_CUDA(cudaMemcpyAsync(b.data(), net->d_l_tq.p, b.size() * 4, cudaMemcpyDeviceToHost, s));
    }
    unsigned long long step = 0;
    SG_CUDA(cudaMemcpyAsync(&step, net->d_step.p, 8, cudaMemcpyDeviceToHost, s));
    SG_CUDA(cudaStreamSynchronize(s));
    for (size_t p = 0; p < net->pops.size(); ++p)
      for (uint32_t i = 0; i < net->pops[p].n; ++i) {
        if (trace_pre) trace_pre[net->offsets[p] + i] = a[net->pops[p].dev_off + i];
        if (trace_post) trace_post[net->offsets[p] + i] = b[net->pops[p].dev_off + i];
      }
    if (t) *t = step - net->l_t0;
  });
}

// ---------------------------------------------------------------------------
// .taas v2 snapshots (crates/SiMuse/crates/taas-format; the connectome
// sections of src/python/python/taas_format.rs:16-31)
// ---------------------------------------------------------------------------
int sg_taas_write(const char *path, const char *created, const char *game, uint32_t n, const char *const *names,
                  const char *const *kinds, const uint64_t *counts, const void *const *data, const uint64_t *bytes,
                  uint32_t n_meta, const char *const *keys, const char *const *values, int zstd_level) {
  return run([&] {
    SG_REQUIRE(path, SG_E_INVALID, "null path");
    SG_REQUIRE(n == 0 || (names && kinds && counts && data && bytes), SG_E_INVALID, "null section arrays");
    SG_REQUIRE(n_meta == 0 || (keys && values), SG_E_INVALID, "null metadata arrays");
    SG_REQUIRE(zstd_level >= 0 && zstd_level <= 22, SG_E_INVALID, "zstd level: 0 (none) or 1..22");
    taas::Writer w;
    w.m.created = created ? created : taas::created_now();
    if (game) {
      w.m.has_game = true;
      w.m.game = game;
    }
    for (uint32_t k = 0; k < n_meta; ++k) w.m.metadata[keys[k]] = values[k];
    w.level = zstd_level;
    for (uint32_t k = 0; k < n; ++k) {
      const std::string kind = kinds[k];
      const size_t es = taas::kind_size(kind);
      SG_REQUIRE(es || kind == "str" || kind == "json" || kind == "blob", SG_E_INVALID, "unknown section kind " + kind);
      SG_REQUIRE(es ? (counts[k] <= UINT64_MAX / es && bytes[k] == counts[k] * es) : bytes[k] == counts[k], SG_E_INVALID,
                 std::string("section '") + names[k] + "': byte length does not match its count");
      SG_REQUIRE(data[k] || bytes[k] == 0, SG_E_INVALID, "null section data");
      w.push(names[k], kind, counts[k], data[k], bytes[k]);
    }
    w.write(path);
  });
}

int sg_taas_read(const char *path, const char *name, const char *kind, void *out, uint64_t cap, uint64_t *bytes) {
  return run([&] {
    SG_REQUIRE(path && name && kind, SG_E_INVALID, "null argument");
    taas::Reader r;
    r.open(path);
    const uint64_t n = r.get_into(name, kind, out, cap);  // out null: size only
    if (bytes) *bytes = n;
  });
}

int sg_taas_validate(const char *path) {
  return run([&] {
    SG_REQUIRE(path, SG_E_INVALID, "null path");
    taas::Reader r;
    r.open(path);
    std::vector<uint8_t> buf;
    for (const auto &sct : r.m.sections) {
      buf.resize((size_t)r.get_into(sct.name, sct.kind, nullptr, 0));
      r.get_into(sct.name, sct.kind, buf.data(), buf.size());
    }
  });
}

int sg_taas_inspect(const char *path, char *buf, uint64_t len, uint64_t *needed) {
  return run([&] {
    SG_REQUIRE(path, SG_E_INVALID, "null path");
    taas::Reader r;
    r.open(path);
    const std::string o = std::string(".taas archive: ") + path + "\n" + r.inspect();
    if (needed) *needed = o.size() + 1;
    if (buf && len) {
      const size_t k = std::min<size_t>(o.size(), (size_t)len - 1);
      std::memcpy(buf, o.data(), k);
      buf[k] = 0;
    }
  });
}

// The built network as a snapshot: row_ptr, col_indices, values (the
// connectome sections), delays, syn_types and, while learning, eligibility.
int sg_taas_save(sg_net *net, const char *path, const char *created, int zstd_level) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "not built");
    SG_REQUIRE(path, SG_E_INVALID, "null path");
    SG_REQUIRE(zstd_level >= 0 && zstd_level <= 22, SG_E_INVALID, "zstd level: 0 (none) or 1..22");
    const uint64_t N = net->total, E = net->n_edges;
    SG_REQUIRE(N < 0x7FFFFFFFull && E <= 0x7FFFFFFFull, SG_E_OVERFLOW,
               "the .taas connectome sections are i32: at most 2^31 - 1 synapses and neurons");
    DevGuard g(net->device);
    std::vector<uint32_t> rp(N + 1), col(E);
    std::vector<float> w(E);
    std::vector<uint8_t> d(E), st(E);
    read_csr_global(net, rp.data(), col.data(), w.data(), d.data(), false, st.data());
    unsigned long long step = 0;
    SG_CUDA(cudaMemcpyAsync(&step, net->d_step.p, 8, cudaMemcpyDeviceToHost, net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
    taas::Writer wr;
    wr.m.created = created ? created : taas::created_now();
    wr.m.has_game = true;
    wr.m.game = "dioma";
    wr.m.metadata["type"] = "Network";
    wr.m.metadata["n_neurons"] = std::to_string(N);
    wr.m.metadata["n_synapses"] = std::to_string(E);
    wr.m.metadata["step"] = std::to_string(step);
    wr.level = zstd_level;
    wr.push("row_ptr", "i32", N + 1, rp.data(), (N + 1) * 4);
    wr.push("col_indices", "i32", E, col.data(), E * 4);
    wr.push("values", "f32", E, w.data(), E * 4);
    wr.push("delays", "u8", E, d.data(), E);
    wr.push("syn_types", "u8", E, st.data(), E);
    std::vector<float> el;  // sections are borrowed until the file is written
    if (net->learn_on) {
      el.resize(E);
      if (E)
        SG_CUDA(cudaMemcpy2DAsync(el.data(), 4, net->d_l_st.p, 8, 4, E, cudaMemcpyDeviceToHost, net->stream));
      SG_CUDA(cudaStreamSynchronize(net->stream));
      wr.push("eligibility", "f32", E, el.data(), E * 4);
    }
    wr.write(path);
  });
}

// Resume: the snapshot's weights into the built network, whose synapses
// (row_ptr, col_indices) must be the snapshot's.  The exact-sum scatter path
// is left for the ordered one (the new weights are not checked for it).
int sg_taas_load_weights(sg_net *net, const char *path) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(net->built, SG_E_STATE, "not built");
    SG_REQUIRE(path, SG_E_INVALID, "null path");
    SG_REQUIRE(net->weight_format == SG_W_F32, SG_E_INVALID,
               "BF16 and FP8 weights are read-only: loading needs FP32 weights");
    taas::Reader r;
    r.open(path);
    const uint64_t N = net->total, E = net->n_edges;
    const std::vector<uint8_t> rp = r.get("row_ptr", "i32"), col = r.get("col_indices", "i32"),
                               vals = r.get("values", "f32");
    SG_REQUIRE(rp.size() == (N + 1) * 4 && col.size() == E * 4 && vals.size() == E * 4, SG_E_INVALID,
               "snapshot size differs from the network (neurons or synapses)");
    DevGuard g(net->device);
    std::vector<uint32_t> nrp(N + 1), ncol(E);
    std::vector<float> w(E);
    std::vector<uint8_t> d(E);
    read_csr_global(net, nrp.data(), ncol.data(), w.data(), d.data(), false);
    SG_REQUIRE(std::memcmp(rp.data(), nrp.data(), rp.size()) == 0 &&
                   (E == 0 || std::memcmp(col.data(), ncol.data(), col.size()) == 0),
               SG_E_INVALID, "snapshot synapses (row_ptr, col_indices) differ from the network's");
    net->exact = false;  // weights from the file: the exact-sum test no longer covers them
    update_path(net);
    drop_graph(net);
    if (E)
      SG_CUDA(cudaMemcpy2DAsync((char *)net->d_edge.p + 4, 8, vals.data(), 4, 4, E, cudaMemcpyHostToDevice,
                                net->stream));
    SG_CUDA(cudaStreamSynchronize(net->stream));
  });
}

// Synapses from a .taas CSR (a saved network or the reference's connectome
// sections): row i of the file is neuron i of population `from`, column j
// neuron j of `to`; delays and syn_types sections when present, else
// `default_delay` and type 0.
int sg_connect_taas(sg_net *net, uint32_t from, uint32_t to, const char *path, uint8_t default_delay) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(path, SG_E_INVALID, "null path");
    require_pop(net, from);
    require_local(net, to);
    taas::Reader r;
    r.open(path);
    const std::vector<uint8_t> rpb = r.get("row_ptr", "i32"), colb = r.get("col_indices", "i32"),
                               wb = r.get("values", "f32");
    const size_t rows = rpb.size() / 4, E = colb.size() / 4;
    SG_REQUIRE(rows == (size_t)net->pops[from].n + 1, SG_E_INVALID,
               "row_ptr length " + std::to_string(rows) + " != source population size + 1");
    SG_REQUIRE(wb.size() / 4 == E, SG_E_INVALID, "values and col_indices differ in length");
    std::vector<int32_t> rp(rows), col(E);
    std::memcpy(rp.data(), rpb.data(), rpb.size());
    if (E) std::memcpy(col.data(), colb.data(), colb.size());
    SG_REQUIRE(rp[0] == 0 && (uint64_t)rp[rows - 1] == E, SG_E_INVALID, "row_ptr does not span col_indices");
    std::vector<uint32_t> pre(E), post(E);
    for (size_t i = 0; i + 1 < rows; ++i) {
      SG_REQUIRE(rp[i] <= rp[i + 1], SG_E_INVALID, "row_ptr is not monotone");
      for (int32_t e = rp[i]; e < rp[i + 1]; ++e) pre[e] = (uint32_t)i;
    }
    for (size_t e = 0; e < E; ++e) {
      SG_REQUIRE(col[e] >= 0, SG_E_INVALID, "negative column index");
      post[e] = (uint32_t)col[e];
    }
    std::vector<uint8_t> d(E, default_delay), st;
    if (r.find("delays")) {
      d = r.get("delays", "u8");
      SG_REQUIRE(d.size() == E, SG_E_INVALID, "delays and col_indices differ in length");
    }
    if (r.find("syn_types")) {
      st = r.get("syn_types", "u8");
      SG_REQUIRE(st.size() == E, SG_E_INVALID, "syn_types and col_indices differ in length");
    }
    std::vector<float> w(E);
    if (E) std::memcpy(w.data(), wb.data(), wb.size());
    const int rc = connect_impl(net, from, pre.data(), to, post.data(), w.data(), d.data(),
                                st.empty() ? nullptr : st.data(), nullptr, E, 0);
    if (rc != SG_OK) throw Fail{rc};
  });
}

int sg_footprint(sg_net *net, uint64_t *out) {
  NET_CHECK(net);
  return run([&] {
    SG_REQUIRE(out, SG_E_INVALID, "null output");
    uint64_t b = 0;
    for (auto &p : net->pops) b += (p.d_params.n + p.d_state.n) * 4;
    b += net->d_ring.n * 4 + net->d_kin_g.n * 4 + net->d_row_ptr.n * 4 + net->d_edge.n * 8 +
         net->d_edge_x.n * 4 + net->d_w16.n * 2 +
         (net->packed ? 0 : net->d_code.n) + net->d_seg.n + net->d_spk.n * 8 + net->d_blk_cnt.n * 4 + net->d_last_bits.n * 4 +
         net->n_runs * 29 + net->d_raster.n * 4 +
         (net->d_in_edge.n + net->d_in_pre.n + net->d_in_ptr.n) * 4 + (net->d_x_pre.n + net->d_x_post.n) * 4 +
         (net->d_stat_spk.n + net->d_stat_ev.n * 2) * 4 + net->d_red_flat.n * 4 + net->d_red_rows.n * 8 + net->d_run_off.n * 4 + net->d_w8.n + net->d_row_scale.n * 4 +
         (net->rr_cnt.n + net->rr_off.n) * 8 + net->rr_temp.n + (net->rr_step.n + net->rr_idx.n) * 4 +
         net->d_pt.n + (net->d_tm_r.n + net->d_tm_u.n + net->d_tm_last.n) * 4 +
         (net->d_l_tp.n + net->d_l_tq.n + net->d_l_baked.n + net->d_l_qb.n + net->d_l_in_ptr.n + net->d_l_in_edge.n +
          net->d_l_in_pre.n + net->d_l_motor.n + net->d_l_flat.n + net->d_l_ctr.n) * 4 +
         net->d_l_st.n * 8 + net->d_l_qa.n * 16;
    *out = b;
  });
}

int sg_stream(sg_net *net, void **out) {
  NET_CHECK(net);
  if (!out) return SG_E_INVALID;
  *out = (void *)net->stream;
  return SG_OK;
}

}  // extern "C"

// ===========================================================================
// pools of resident networks (continuous batching)
// ===========================================================================
namespace {

void pool_drop_graph(sg_pool *pool) {
  if (pool->graph) cudaGraphExecDestroy(pool->graph);
  pool->graph = nullptr;
  pool->graph_steps = 0;
}

// The members' arguments, populations and block map; uploaded (and the
// captured graph dropped) when they change.
void pool_prepare(sg_pool *pool) {
  std::vector<StepArgs> nets;
  std::vector<PopArgs> pops;
  std::vector<uint4> map;
  bool full[5] = {};
  for (size_t i = 0; i < pool->members.size(); ++i) {
    sg_net *net = pool->members[i];
    upload_pop_table(net);
    const StepArgs a = make_args(net);
    SG_REQUIRE(a.red, SG_E_STATE,
               "pool: every member takes the pre-centric scatter (exact ring sums, or the atomic mode)");
    SG_REQUIRE(!net->learn_on && !has_external(net), SG_E_STATE,
               "pool: learning networks and networks split across GPUs step on their own");
    for (int m = 1; m <= 4; ++m) full[m] = full[m] || needs_full_neuron_kernel(net, a, m);
    nets.push_back(a);
  }
  for (int m = 1; m <= 4; ++m) {
    pool->model_off[m] = (uint32_t)map.size();
    for (size_t i = 0; i < pool->members.size(); ++i) {
      sg_net *net = pool->members[i];
      for (size_t q = 0; q < net->pops.size(); ++q) {
        const HostPop &hp = net->pops[q];
        if (hp.model != m || hp.n == 0 || hp.external) continue;
        const uint32_t pi = (uint32_t)pops.size();
        pops.push_back(net->pop_tab[q]);
        for (uint32_t b = 0; b < hp.cap / kNeuronBlock; ++b) map.push_back(make_uint4((uint32_t)i, pi, b, 0u));
      }
    }
    pool->model_cnt[m] = (uint32_t)map.size() - pool->model_off[m];
  }
  const bool same = nets.size() == pool->h_nets.size() && pops.size() == pool->h_pops.size() &&
                    map.size() == pool->h_map.size() && std::memcmp(full, pool->full, sizeof(full)) == 0 &&
                    std::memcmp(nets.data(), pool->h_nets.data(), nets.size() * sizeof(StepArgs)) == 0 &&
                    std::memcmp(pops.data(), pool->h_pops.data(), pops.size() * sizeof(PopArgs)) == 0 &&
                    std::memcmp(map.data(), pool->h_map.data(), map.size() * sizeof(uint4)) == 0;
  if (same) return;
  pool_drop_graph(pool);
  SG_CUDA(cudaStreamSynchronize(pool->stream));  // no step in flight reads the old tables
  pool->h_nets = std::move(nets);
  pool->h_pops = std::move(pops);
  pool->h_map = std::move(map);
  std::memcpy(pool->full, full, sizeof(full));
  if (pool->d_nets.n < pool->h_nets.size()) pool->d_nets.alloc(pool->h_nets.size());
  if (pool->d_pops.n < std::max<size_t>(pool->h_pops.size(), 1)) pool->d_pops.alloc(std::max<size_t>(pool->h_pops.size(), 1));
  if (pool->d_map.n < std::max<size_t>(pool->h_map.size(), 1)) pool->d_map.alloc(std::max<size_t>(pool->h_map.size(), 1));
  SG_CUDA(cudaMemcpyAsync(pool->d_nets.p, pool->h_nets.data(), pool->h_nets.size() * sizeof(StepArgs),
                          cudaMemcpyHostToDevice, pool->stream));
  if (!pool->h_pops.empty())
    SG_CUDA(cudaMemcpyAsync(pool->d_pops.p, pool->h_pops.data(), pool->h_pops.size() * sizeof(PopArgs),
                            cudaMemcpyHostToDevice, pool->stream));
  if (!pool->h_map.empty())
    SG_CUDA(cudaMemcpyAsync(pool->d_map.p, pool->h_map.data(), pool->h_map.size() * sizeof(uint4),
                            cudaMemcpyHostToDevice, pool->stream));
  SG_CUDA(cudaStreamSynchronize(pool->stream));
}

template <int M> void pool_launch_neuron(sg_pool *pool) {
  const uint32_t nb = pool->model_cnt[M];
  if (nb == 0) return;
  const uint4 *map = pool->d_map.p + pool->model_off[M];
  if (pool->full[M])
    launch_step_kernel(neuron_pool_kernel<M, true>, nb, NeuronCfg<M, true>::THREADS, 0, pool->stream,
                       (const StepArgs *)pool->d_nets.p, (const PopArgs *)pool->d_pops.p, map);
  else
    launch_step_kernel(neuron_pool_kernel<M, false>, nb, NeuronCfg<M, false>::THREADS, 0, pool->stream,
                       (const StepArgs *)pool->d_nets.p, (const PopArgs *)pool->d_pops.p, map);
}

void pool_enqueue_step(sg_pool *pool) {
  pool_launch_neuron<kLIF>(pool);
  pool_launch_neuron<kIZH>(pool);
  pool_launch_neuron<kGPEA>(pool);
  pool_launch_neuron<kHH>(pool);
  int fmt = pool->h_nets.empty() ? 0 : walk_format(pool->h_nets[0]);
  for (const StepArgs &a : pool->h_nets)
    if (walk_format(a) != fmt) fmt = 0;  // mixed storage: read per network
  launch_step_red(pool->stream, pool->device, default_red_variant(), kRedBlocksPerSM, (const StepArgs *)pool->d_nets.p,
                  (uint32_t)pool->h_nets.size(), pool->d_done.p, pool->d_err.p, 0u, fmt);
}

}  // namespace

extern "C" {

int sg_pool_create(sg_pool **out, int device) {
  return run([&] {
    SG_REQUIRE(out, SG_E_INVALID, "null output");
    *out = nullptr;
    int n = 0;
    SG_CUDA(cudaGetDeviceCount(&n));
    SG_REQUIRE(device >= 0 && device < n, SG_E_INVALID, "device ordinal out of range");
    DevGuard g(device);
    auto *pool = new sg_pool();
    pool->device = device;
    if (cudaStreamCreateWithFlags(&pool->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&pool->ev, cudaEventDisableTiming) != cudaSuccess) {
      if (pool->stream) cudaStreamDestroy(pool->stream);
      delete pool;
      SG_REQUIRE(false, SG_E_CUDA, "pool: stream or event creation failed");
    }
    pool->d_done.alloc(1);
    pool->d_done.zero(pool->stream);
    pool->d_err.alloc(1);
    pool->d_err.zero(pool->stream);
    allow_red_smem();
    SG_CUDA(cudaStreamSynchronize(pool->stream));
    *out = pool;
  });
}

int sg_pool_add(sg_pool *pool, sg_net *net) {
  return run([&] {
    SG_REQUIRE(pool && net, SG_E_INVALID, "null pool or network");
    SG_REQUIRE(net->built, SG_E_STATE, "pool: the network is not built");
    SG_REQUIRE(net->device == pool->device, SG_E_INVALID, "pool: the network lives on another device");
    SG_REQUIRE(net->pool == nullptr, SG_E_STATE, "pool: the network is already in a pool");
    SG_REQUIRE(pool->members.size() < kPoolMax, SG_E_INVALID,
               "pool: at most " + std::to_string(kPoolMax) + " networks");
    SG_REQUIRE(net->red, SG_E_STATE,
               "pool: only networks on the pre-centric scatter (exact ring sums, or the atomic mode) join a pool");
    pool->members.push_back(net);
    net->pool = pool;
  });
}

int sg_pool_remove(sg_pool *pool, sg_net *net) {
  return run([&] {
    SG_REQUIRE(pool && net, SG_E_INVALID, "null pool or network");
    auto it = std::find(pool->members.begin(), pool->members.end(), net);
    SG_REQUIRE(it != pool->members.end(), SG_E_INVALID, "pool: the network is not a member");
    DevGuard g(pool->device);
    SG_CUDA(cudaStreamSynchronize(pool->stream));
    pool->members.erase(it);
    net->pool = nullptr;
    pool_drop_graph(pool);
  });
}

int sg_pool_size(sg_pool *pool, uint32_t *out) {
  return run([&] {
    SG_REQUIRE(pool && out, SG_E_INVALID, "null pool or output");
    *out = (uint32_t)pool->members.size();
  });
}

int sg_pool_step(sg_pool *pool, uint32_t n_steps) {
  return run([&] {
    SG_REQUIRE(pool, SG_E_INVALID, "null pool");
    if (pool->members.empty() || n_steps == 0) return;
    DevGuard g(pool->device);
    for (sg_net *net : pool->members) SG_REQUIRE(net->total > 0, SG_E_STATE, "pool: an empty network");
    pool_prepare(pool);
    for (sg_net *net : pool->members) setup_l2_setaside(net);
    // the pool's steps follow everything queued on the members' streams
    for (sg_net *net : pool->members) {
      SG_CUDA(cudaEventRecord(pool->ev, net->stream));
      SG_CUDA(cudaStreamWaitEvent(pool->stream, pool->ev, 0));
    }
    const uint32_t G = 32;
    uint32_t done = 0;
    if (n_steps >= G) {
      if (!pool->graph || pool->graph_steps != G) {
        pool_drop_graph(pool);
        cudaGraph_t gr;
        SG_CUDA(cudaStreamBeginCapture(pool->stream, cudaStreamCaptureModeThreadLocal));
        for (uint32_t k = 0; k < G; ++k) pool_enqueue_step(pool);
        SG_CUDA(cudaStreamEndCapture(pool->stream, &gr));
        SG_CUDA(cudaGraphInstantiate(&pool->graph, gr, 0));
        cudaGraphDestroy(gr);
        pool->graph_steps = G;
      }
      for (; done + G <= n_steps; done += G) SG_CUDA(cudaGraphLaunch(pool->graph, pool->stream));
    }
    for (; done < n_steps; ++done) pool_enqueue_step(pool);
    SG_CUDA(cudaGetLastError());
    // and everything queued on a member's stream later follows them
    SG_CUDA(cudaEventRecord(pool->ev, pool->stream));
    for (sg_net *net : pool->members) {
      SG_CUDA(cudaStreamWaitEvent(net->stream, pool->ev, 0));
      net->host_step += n_steps;
    }
  });
}

int sg_pool_synchronize(sg_pool *pool) {
  return run([&] {
    SG_REQUIRE(pool, SG_E_INVALID, "null pool");
    DevGuard g(pool->device);
    SG_CUDA(cudaStreamSynchronize(pool->stream));
    uint32_t e = 0;
    SG_CUDA(cudaMemcpy(&e, pool->d_err.p, 4, cudaMemcpyDeviceToHost));
    if (e) {
      SG_CUDA(cudaMemset(pool->d_err.p, 0, 4));
      SG_REQUIRE(false, SG_E_CUDA, "pool scatter: a pipeline wait timed out on the device");
    }
  });
}

int sg_pool_destroy(sg_pool *pool) {
  if (!pool) return SG_OK;
  DevGuard g(pool->device);
  cudaStreamSynchronize(pool->stream);
  for (sg_net *net : pool->members) net->pool = nullptr;
  pool_drop_graph(pool);
  cudaEventDestroy(pool->ev);
  cudaStream_t s = pool->stream;
  delete pool;
  cudaStreamDestroy(s);
  return SG_OK;
}

}  // extern "C"
