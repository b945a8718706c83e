/*
 * simuse_b200.h — C ABI of the B200-native SiMuse simulation step.
 *
 * A drop-in for the reference's `pillars::api::Network` builder/step API
 * (crates/SiMuse/crates/pillars/src/api/net/network/core.rs:87-622,
 * build.rs:18-276, step.rs:18-189).  The ABI is Rust-callable by design:
 * opaque handle, plain pointers and sizes, int status codes, no C++ or torch
 * types.  Each entry point names the reference interface it replaces.
 *
 * Conventions
 *  - Every function returns SG_OK (0) or a negative SG_E_* code; the message
 *    is available from sg_last_error() (thread-local), as the Unity bridge
 *    does (src/unity_bridge.rs:8-64).  Nothing aborts the process: the
 *    reference's assert!/panic! contract violations become SG_E_INVALID.
 *  - Host pointers are read during the call only; the caller keeps
 *    ownership.  Readbacks copy into caller-provided buffers (as
 *    CompiledNetwork::download_* does, pillars-cuda/src/network.rs:471-491).
 *  - One handle owns one CUDA stream on one device.  Calls on different
 *    handles are thread-safe; calls on one handle must be serialised by the
 *    caller.
 *  - Indices are the reference's: population ids in creation order, neuron
 *    indices within a population, global neuron index = population offset +
 *    index (core.rs:236-239).
 */
#ifndef SIMUSE_B200_H
#define SIMUSE_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SG_ABI_VERSION 1

enum sg_status {
  SG_OK = 0,
  SG_E_INVALID = -1,  /* contract violation (reference: assert!/panic!) */
  SG_E_STATE = -2,    /* wrong lifecycle stage (e.g. connect after build) */
  SG_E_CUDA = -3,     /* CUDA runtime error */
  SG_E_NOMEM = -4,    /* device allocation failed or over budget */
  SG_E_OVERFLOW = -5, /* a fixed-capacity device buffer would overflow */
  SG_E_TIMEOUT = -6   /* a bounded device wait gave up */
};

/* Neuron models (reference: pillars::zoo::neurons::*). */
enum sg_model {
  SG_LIF = 1,  /* LIFModel, P/zoo/neurons/lif.rs:22-78; params dt inv_tau_m v_rest v_thresh v_reset tau_ref; state v refr */
  SG_IZH = 2,  /* IzhikevichModel, P/zoo/neurons/izhikevich.rs:42-125; params dt a b c d tau_ref v_thresh; state v u refr */
  SG_GPEA = 3, /* GpeaModel, P/zoo/neurons/gpea.rs:211-360; 14 params, 9 states */
  SG_HH = 4    /* Hodgkin-Huxley, RK4 (no reference: P/zoo/neurons/hh.rs is a stub);
                  params dt c_m g_na g_k g_l e_na e_k e_l i_bias v_thresh; state v m h n */
};

/* Edge flags for sg_connect_ex. */
#define SG_EDGE_STDP 1u /* the synapse takes part in pair STDP */

/* Weight storage precision (scatter bytes), sg_set_weight_format. */
enum sg_weight_format { SG_W_F32 = 0, SG_W_BF16 = 1, SG_W_FP8 = 2 };

typedef struct sg_net sg_net;

/* ---- library ---------------------------------------------------------- */
int sg_abi_version(void);                       /* src/unity_bridge.rs:207-241 (*_abi_version) */
int sg_last_error(char *buf, size_t len);       /* src/unity_bridge.rs:58-64 (last_error) */
int sg_device_count(int *out);

/* ---- Network lifecycle ------------------------------------------------ */
int sg_net_create(sg_net **out, int device);    /* Network::new, core.rs:87-113 */
int sg_net_destroy(sg_net *net);                /* Drop for Network */
/* Waits for the handle's stream.  Returns SG_E_CUDA if a step's scatter
   pipeline gave up a wait on the device (its events are then incomplete);
   the condition is reported once. */
int sg_synchronize(sg_net *net);
/* No counterpart in the reference.  Tunes the pre-centric scatter's
   schedule (variants 0-3: a shared-memory stage ring of stages x synapses
   per stage; variants 4-8: the warp walk without stages, 5 and 6 loading
   the next round of records before reducing the current one, 7 and 8
   walking each row as 4 pieces (8 at 6 blocks per SM); and blocks per
   SM)
   on the network's own next steps: each candidate runs
   `steps` steps (after a warm-up chunk), timed on the device, and the
   fastest is kept.  Every schedule gives the same results, so these are
   ordinary simulation steps (the step counter advances).  Reports the
   per-step time of the fixed schedule and of the chosen one.  On the ordered
   path there is nothing to tune (times 0). */
int sg_autotune(sg_net *net, uint32_t steps, float *fixed_ms, float *best_ms, int *best_variant,
                uint32_t *best_bps);
/* No counterpart in the reference.  The pre-centric scatter's current
   schedule (the variant and blocks per SM that sg_autotune reports; a new
   network starts on variant 4, or on SG_RED_VARIANT when that is set). */
int sg_scatter_schedule(sg_net *net, int *variant, uint32_t *blocks_per_sm);
/* Test hook (no reference counterpart): on != 0 makes the pre-centric
   scatter's producer stop feeding its consumers, whose waits then run out
   (~1 s per step) and set the device error that sg_synchronize reports. */
int sg_debug_stall_scatter(sg_net *net, int on);
/* Non-blocking: *idle = 1 when all work queued on the handle's stream has
   completed, 0 while some is still running (cudaStreamQuery). */
int sg_query(sg_net *net, int *idle);

/* ---- builder (before sg_build) ---------------------------------------- */
/* Network::add_population::<M>(n) -> PopulationId, core.rs:149-155 */
int sg_pop_add(sg_net *net, int model, uint32_t n, uint32_t *out_pop);
/* NeuralPopulation::fill_param / fill_state, P/core/exec/population.rs:166-197 */
int sg_pop_fill_param(sg_net *net, uint32_t pop, uint32_t col, float value);
int sg_pop_fill_state(sg_net *net, uint32_t pop, uint32_t col, float value);
/* param_slice_mut / state_slice_mut then a copy, population.rs:209-220 (any time) */
int sg_pop_set_param(sg_net *net, uint32_t pop, uint32_t col, const float *vals, uint32_t n);
int sg_pop_set_state(sg_net *net, uint32_t pop, uint32_t col, const float *vals, uint32_t n);
/* Network::state(pop, col) / param_slice(pop, col), build.rs:155-182 */
int sg_pop_get_state(sg_net *net, uint32_t pop, uint32_t col, float *out, uint32_t n);
int sg_pop_get_param(sg_net *net, uint32_t pop, uint32_t col, float *out, uint32_t n);

/* Network::connect(from, &[u32], to, &[u32], &[f32], &[u8]), core.rs:166-249 */
int sg_connect(sg_net *net, uint32_t from, const uint32_t *from_idx, uint32_t to,
               const uint32_t *to_idx, const float *weights, const uint8_t *delays, uint64_t n);
/* connect_edges with per-edge syn_type (0 static, k = kinetic profile k) and
   flags (SG_EDGE_STDP), core.rs:254-279; syn_types may be NULL. */
int sg_connect_ex(sg_net *net, uint32_t from, const uint32_t *from_idx, uint32_t to,
                  const uint32_t *to_idx, const float *weights, const uint8_t *delays,
                  const uint8_t *syn_types, uint64_t n, uint32_t flags);
/* Seeded synthetic projection generated on the device: every post of `to`
   receives exactly `k_in` synapses from pres drawn uniformly (with
   replacement) from `from`; weight w_exc for pre index < n_exc else w_inh;
   delay uniform in [d_min, d_max].  Edge (post j, draw q) uses
   h = splitmix64(seed ^ (j*k_in + q)*0x9E3779B97F4A7C15), pre = (h>>32)*n_from>>32,
   delay = d_min + (h & 0xffffffff) % (d_max-d_min+1); edges are appended in
   (post, draw) order. */
int sg_connect_fixed_indegree(sg_net *net, uint32_t from, uint32_t to, uint32_t k_in,
                              uint64_t seed, uint32_t n_exc, float w_exc, float w_inh,
                              uint8_t d_min, uint8_t d_max, uint8_t syn_type_exc,
                              uint8_t syn_type_inh, uint32_t flags_exc);

/* Seeded synthetic projection generated on the device: every neuron i of
   `from` gets exactly k distinct targets in `to` (no self-loop when no_self,
   which needs from == to), drawn by Floyd's sampling: with m candidates,
   draw q (j = m - k + q) takes t = hi32(h) * (j + 1) >> 32, or j when t was
   drawn before, h = splitmix64(seed ^ (i*k + q)*0x9E3779B97F4A7C15); without
   self-loops t >= i maps to t + 1 (k <= 4096).  Weight w_exc for i < n_exc
   else w_inh, times lo32(h) / 2^32 when random_w = 1, or times the top b
   bits of lo32(h) / 2^b (a U on the 2^-b grid) when random_w = b in 2..24; delay d_min +
   lo32(splitmix64(h)) % (d_max - d_min + 1); synapse type st_exc / st_inh and,
   for excitatory sources, flags_exc (SG_EDGE_STDP).  Edges are appended in
   (source, draw) order.  The generator of the Izhikevich pulse network
   recipe (100 distinct targets, weights 0.5 U / -U, delay 1). */
int sg_connect_fixed_outdegree(sg_net *net, uint32_t from, uint32_t to, uint32_t k, uint64_t seed,
                               int no_self, uint32_t n_exc, float w_exc, float w_inh, int random_w,
                               uint8_t d_min, uint8_t d_max, uint8_t st_exc, uint8_t st_inh,
                               uint32_t flags_exc);

/* As sg_connect_fixed_outdegree with a lognormal out-degree per source:
   deg_i = round(exp(mu + sigma z_i)) clipped to [1, min(candidates, 4096)],
   sigma^2 = ln(1 + sd^2/mean^2), mu = ln(mean) - sigma^2/2, z_i the FP64
   Box-Muller normal of counter i (stream 7, the sg_pop_set_noise hash);
   source i's draws use hash counters off_i + q (off = exclusive prefix sum
   of the degrees). */
int sg_connect_lognormal_outdegree(sg_net *net, uint32_t from, uint32_t to, double mean, double sd,
                                   uint64_t seed, int no_self, uint32_t n_exc, float w_exc, float w_inh,
                                   int random_w, uint8_t d_min, uint8_t d_max, uint8_t st_exc,
                                   uint8_t st_inh, uint32_t flags_exc);

/* Network::register_plasticity(PlasticityProfile, dt) -> profile id (1-based),
   core.rs:586-623; synapse.rs:220-292 (Tsodyks-Markram: U0 = u0 in (0, 1],
   recovery tau_rec, facilitation tau_fac when `facilitation` is set; the
   device holds at most 8 profiles).  A spike on a synapse with a profile
   delivers weight * R * U, push.rs:25-102. */
int sg_register_plasticity(sg_net *net, float u0, float tau_rec, int facilitation, float tau_fac, float dt,
                           uint32_t *out_id);
/* connect_edges with Edge::with_synapse_plasticity, core.rs:254-279: as
   sg_connect_ex plus a per-edge plasticity profile id (0 = none; may be
   NULL). */
int sg_connect_plastic(sg_net *net, uint32_t from, const uint32_t *from_idx, uint32_t to,
                       const uint32_t *to_idx, const float *weights, const uint8_t *delays,
                       const uint8_t *syn_types, const uint8_t *plast_types, uint64_t n, uint32_t flags);
/* Network::register_kinetics(SynapseKinetics::ExpOne{tau_decay, erev}, dt)
   -> profile id (1-based), core.rs:564-584; step.rs:248-345 */
int sg_register_expone(sg_net *net, float tau_decay, float erev, float dt, uint32_t *out_id);
/* Network::register_kinetics(SynapseKinetics, dt) for every waveform kind,
   core.rs:564-584; synapse.rs:36-158 (parameters and validation);
   step.rs:206-398 (exact per-step update).  params: ExpOne {tau_decay},
   ExpTwo {tau_rise, tau_decay}, Alpha {tau}, ExpThree {tau_rise, tau_decay1,
   tau_decay2, gbase1, gbase2}.  At most 3 profiles on the device. */
#define SG_KIN_EXPONE 0
#define SG_KIN_EXPTWO 1
#define SG_KIN_ALPHA 2
#define SG_KIN_EXPTHREE 3
int sg_register_kinetics(sg_net *net, int kind, const float *params, float erev, float dt, uint32_t *out_id);

/* SynapticBrain receptor kinetics (pillars-connectome/src/synaptic.rs:23-130;
   P/kernels/synapse/{kinetics,receptor}.rs): call before any connect.  The
   syn_types of later synapses are receptor codes (0 AMPA, 1 NMDA, 2 GABA_A,
   3 GABA_B, 4 nAChR, 5 GluCl, 6 mAChR; others AMPA) and their delays are
   ignored.  Each step decays the seven conductances by fast_exp(-dt/tau),
   adds I_syn = sum g_eff (E_rev - V) (NMDA Mg-blocked, pre-step V) to the
   step's external input (inject_current, bias, noise), steps the neurons,
   then every spike jumps its targets' conductances in (pre ascending, row)
   order: SynapticBrain::step.  No kinetic profiles, Poisson sources, STDP,
   short-term plasticity or learning alongside; sg_clear_rings zeroes the
   conductances too. */
int sg_set_receptor_kinetics(sg_net *net, float dt);
/* SynapticBrain::kinetics / set_kinetics: g[r * total + i], r = receptor code */
int sg_receptor_read(sg_net *net, float *g);
int sg_receptor_write(sg_net *net, const float *g);

/* Network::add_poisson_source(rate_hz, dt_ms, seed) -> id, core.rs:288-312 */
int sg_poisson_add(sg_net *net, float rate_hz, float dt_ms, uint32_t seed, uint32_t *out_id);
/* n sources at once with seeds[i] (or seed0 + i when seeds == NULL); ids are consecutive */
int sg_poisson_add_many(sg_net *net, uint32_t n, float rate_hz, float dt_ms,
                        const uint32_t *seeds, uint32_t seed0, uint32_t *out_first_id);
/* Network::connect_poisson_source(src, to, posts, w, d, st, pt), core.rs:323-381 */
int sg_poisson_connect(sg_net *net, uint32_t src, uint32_t to, const uint32_t *posts,
                       const float *weights, const uint8_t *delays, const uint8_t *syn_types,
                       uint64_t n);
/* As sg_poisson_connect, each synapse with a Tsodyks-Markram profile
   (plast_types[i], 0 none; registered with sg_register_plasticity): the
   delivered weight is scaled by the synapse's own R and U at each source
   spike (P/api/net/network/step.rs:166-180, core.rs:323-380). */
int sg_poisson_connect_plastic(sg_net *net, uint32_t src, uint32_t to, const uint32_t *posts,
                               const float *w, const uint8_t *delays, const uint8_t *syn_types,
                               const uint8_t *plast_types, uint64_t n);
/* Source first_src + i gets one synapse to post posts[i] (posts == NULL:
   post i), weight w, delay d: the "one source per neuron" drive. */
int sg_poisson_connect_one_to_one(sg_net *net, uint32_t first_src, uint32_t n, uint32_t to,
                                  const uint32_t *posts, float weight, uint8_t delay);

/* Pair STDP on edges flagged SG_EDGE_STDP (no reference function; the trace
   arithmetic follows P/api/learn/brain.rs:204-222). */
int sg_stdp_config(sg_net *net, float dt, float tau_pre, float tau_post, float a_plus,
                   float a_minus, float w_min, float w_max);

/* Weight storage format for the scatter (FP32 default). */
int sg_set_weight_format(sg_net *net, int format);
/* Scatter mode: 1 = deterministic (reference summation order, default),
   0 = atomic accumulation (tolerance mode, order not fixed). */
int sg_set_deterministic(sg_net *net, int on);
/* The scatter path a built network uses (no reference counterpart; the
   reference has one sequential push, P/api/net/push.rs:143-172):
   SG_SCATTER_ORDERED  ring cells updated in the reference's order;
   SG_SCATTER_EXACT    the ring sums are exact in FP32 (every weight a
                       multiple of one power of two 2^e, every post's weights
                       summing in magnitude below 2^(23+e), no STDP), so the
                       events go through per-slot lists and are added in any
                       order: the same bits;
   SG_SCATTER_ATOMIC   atomic adds in any order (sg_set_deterministic(0)). */
#define SG_SCATTER_ORDERED 0
#define SG_SCATTER_EXACT 1
#define SG_SCATTER_ATOMIC 2
int sg_scatter_mode(sg_net *net, int *out);

/* Network::build(), build.rs:18-109 (a second call is SG_E_STATE) */
int sg_build(sg_net *net);
/* SparseGraph::from_csr + build (graph.rs:217-275): all-static, not plastic */
int sg_build_from_csr(sg_net *net, const uint32_t *row_ptr, const uint32_t *col,
                      const float *weights, const uint8_t *delays);

/* Device-generated Gaussian input current, the device form of feeding a
   population's noise through inject_current every step (how the reference's
   Izhikevich examples drive the thalamic input, build.rs:243-275).  At device
   step t, neuron i of the population receives sigma_i * z, z the FP64
   Box-Muller normal of the SplitMix64 counters 2c and 2c+1 with
   c = i + (t - step0) * stride (uniform = (splitmix64(splitmix64((seed *
   0x9E3779B97F4A7C15) ^ (stream << 40) ^ counter)) >> 11) * 2^-53),
   sigma_i = sigma_lo for i < split and sigma_hi after, rounded to f32 and
   added to the slot value before kinetic currents and the clamp, i.e. after
   any host injection of the same step.  sigma_lo = sigma_hi = 0 turns it
   off.  Allowed before and after build. */
int sg_pop_set_noise(sg_net *net, uint32_t pop, uint64_t seed, uint32_t stream, uint64_t stride,
                     uint64_t step0, double sigma_lo, double sigma_hi, uint32_t split);

/* Constant per-neuron input current added to the slot value every step, the
   device form of calling inject_current with the same values before each
   step (BrainRunner::run's external_I, pillars-connectome runner.rs:798-937;
   the add is the same float operation, so results are identical).  Values
   past n are 0; n = 0 removes it.  Needs a built network. */
int sg_pop_set_bias(sg_net *net, uint32_t pop, const float *vals, uint32_t n);
/* Empties every delay ring (and kinetic conductance): the state of a freshly
   built Network, which BrainRunner::run starts from on every call
   (runner.rs:1342-1440 rebuilds its Brain each run). */
int sg_ring_clear(sg_net *net);

/* ---- run -------------------------------------------------------------- */
/* Network::inject_current(pop, idx, vals), build.rs:243-275: same-step slot */
int sg_inject(sg_net *net, uint32_t pop, const uint32_t *idx, const float *vals, uint64_t n);
/* n_steps x Network::step(), step.rs:18-189 (asynchronous; CUDA-graph replay) */
int sg_step(sg_net *net, uint32_t n_steps);
/* Spike raster: keep the last `capacity_steps` steps as bitmasks (0 disables). */
int sg_raster_enable(sg_net *net, uint32_t capacity_steps);
/* Copy the spike raster of the steps recorded since the last read into
   `out` as bytes [n_steps][total_neurons]; returns the step count in *n_steps. */
int sg_raster_read(sg_net *net, uint8_t *out, uint64_t cap_bytes, uint32_t *n_steps);
/* Per-step counters since the last read: spikes and synaptic events. */
int sg_stats_read(sg_net *net, uint32_t *spikes, uint64_t *events, uint32_t cap, uint32_t *n_steps);

/* Spike raster of the steps recorded since the last read, as a list of
   (step, global neuron index) pairs ordered by step then index; the list is
   compacted on the device so only the spikes cross PCIe.  *n_out = spikes. */
int sg_raster_read_events(sg_net *net, uint32_t *steps, uint32_t *idx, uint64_t cap,
                          uint64_t *n_out);
/* Staged raster read for a loop that keeps the GPU stepping while it reads.
   sg_raster_stage queues, right after the steps queued so far, the
   compaction of the steps recorded since the last read (on the network's own
   read stream; the network's later steps wait for it, so the raster slots are
   reused at once) and returns without waiting.  sg_raster_fetch waits for
   that compaction and copies its (step, index) pairs into the buffers
   (cap pairs; when too small it fails with *n_out = the count and the batch
   stays staged).  One staged batch per network at a time; plain reads,
   sg_raster_enable and sg_raster_counts refuse while one is staged. */
int sg_raster_stage(sg_net *net);
int sg_raster_fetch(sg_net *net, uint32_t *steps, uint32_t *idx, uint64_t cap, uint64_t *n_out);
/* The staged batch with its steps as offsets (4 bytes per spike instead of
   8): *t0 = the batch's first step, *n_steps = its steps k, and the spikes
   of step *t0 + s are idx[step_off[s] .. step_off[s + 1]), s < k
   (step_off[k] = *n_out).  off_cap must be >= k + 1; when cap is too small
   it fails with *n_out = the count and the batch stays staged. */
int sg_raster_fetch_csr(sg_net *net, uint32_t *step_off, uint64_t off_cap, uint32_t *idx, uint64_t cap,
                        uint64_t *t0, uint64_t *n_steps, uint64_t *n_out);
/* No counterpart in the reference: page-locked host memory (cudaHostAlloc,
   portable) for readback buffers, so that device-to-host copies are DMA
   straight into them; *out = NULL for 0 bytes. */
int sg_host_alloc(uint64_t bytes, void **out);
int sg_host_free(void *p);
/* Spikes per neuron over every event read (plain or staged) since the raster
   was enabled; counts[total]. */
int sg_raster_counts(sg_net *net, uint32_t *counts);
/* Phase timing: when enabled, sg_step launches each step eagerly with CUDA
   events around its phases (0 neuron update, 1 expand, 2 STDP potentiation,
   3 apply) and accumulates the device time per phase. */
int sg_profile_enable(sg_net *net, int on);
int sg_profile_read(sg_net *net, double *ms, uint64_t *launches); /* 4 entries each */

/* ---- readback --------------------------------------------------------- */
int sg_spikes(sg_net *net, uint32_t pop, int32_t *out, uint32_t n); /* build.rs:145-152 */
int sg_step_counter(sg_net *net, uint64_t *out);                    /* build.rs:136-140 */
int sg_total_neurons(sg_net *net, uint64_t *out);                   /* build.rs:130-134 */
int sg_num_synapses(sg_net *net, uint64_t *out);                    /* graph.rs:285-287 */
int sg_events_total(sg_net *net, uint64_t *out);
/* Of those, the events of Poisson-source synapses (sources.rs:5-14). */
int sg_source_events_total(sg_net *net, uint64_t *out);
/* Network::graph() -> SparseGraph CSR arrays, build.rs:186-188 */
int sg_graph_read(sg_net *net, uint32_t *row_ptr, uint32_t *col, float *weights, uint8_t *delays);
/* Per synapse, in sg_graph_read's order: the synapse type (0 static, 1..3 a
   kinetic profile; SparseGraph::syn_types, P/api/net/graph.rs:67-80) and
   whether pair STDP updates it (1) or not (0). */
int sg_graph_read_types(sg_net *net, uint8_t *syn_types, uint8_t *stdp);
int sg_weights_read(sg_net *net, float *weights); /* current CSR weights (STDP) */
/* DelayBuffer contents [32][total_neurons] of ring 0 (static) or kinetic k */
int sg_ring_read(sg_net *net, uint32_t ring, float *out);
int sg_stdp_drift(sg_net *net, double *out);
int sg_stdp_traces(sg_net *net, float *x_pre, float *x_post);
int sg_clamp_hits(sg_net *net, uint64_t *out); /* i_syn values that hit the +-100 clamp */

/* ---- dopamine-modulated eligibility learning ----------------------------
   The reference's Brain (P/api/learn/brain.rs:62-418: StdpConfig, step,
   fold_eligibility, reward_dopamine, LearnToken::reward / reward_gated /
   reward_capped, clear/restrict/set_eligibility, snapshot/recall), bound to
   the built network's own synapses and spikes the way
   pillars-wgpu/src/network.rs:902-1336 (step_many_learn, reward,
   download_motor_sums) binds it: after every step's spikes the per-neuron
   traces decay and take the spike (fma), and the eligibility of every synapse
   of a spiking neuron takes +a_ltp * trace_pre[pre] (as post) and
   -a_ltd * trace_post[post] (as pre), lazily decayed by repeated
   multiplication with exp(-dt/tau_e).  Synapse i is CSR record i (the order
   sg_graph_read reports).  Needs FP32 weights; drops the exact-sum scatter
   path (rewards change weights).  Learning begins at the step it is enabled. */
int sg_learn_enable(sg_net *net, float dt, float tau_pre, float tau_post, float tau_e, float a_ltp, float a_ltd,
                    float lr, float w_min, float w_max);
/* w += lr * dopamine * clamp(gate, 0, 1) * e, clamped to [w_min, cap] where
   cap = w_cap when finite (reward_capped) else w_max; zero deltas skip. */
int sg_learn_reward(sg_net *net, float dopamine, float gate, float w_cap);
int sg_learn_clear(sg_net *net);                                       /* brain.rs:271-275 */
/* Per-network reward and clear in a pool of independent networks (populations
   without synapses between them): only synapses [lo, hi), e.g. the range
   sg_pop_synapse_range gives for one network's population; the others keep
   their eligibility (the per-block reward of dioma-engine gpu_pool.rs:12-16). */
int sg_learn_reward_range(sg_net *net, uint64_t lo, uint64_t hi, float dopamine, float gate, float w_cap);
int sg_learn_clear_range(sg_net *net, uint64_t lo, uint64_t hi);
int sg_pop_synapse_range(sg_net *net, uint32_t pop, uint64_t *lo, uint64_t *hi); /* CSR range of its rows */
int sg_learn_restrict(sg_net *net, const uint8_t *keep, uint64_t n);   /* brain.rs:278-285 */
int sg_learn_set_eligibility(sg_net *net, const float *elig, uint64_t n); /* brain.rs:160-170 */
/* spikes of neurons [lo0, hi0) and [lo1, hi1) counted over each sg_step call
   (network.rs:902-955 motor sums; shaders/dopamine.wgsl:126-136) */
int sg_learn_motor(sg_net *net, uint64_t lo0, uint64_t hi0, uint64_t lo1, uint64_t hi1);
int sg_learn_motor_read(sg_net *net, uint32_t *out /* [2] */);
int sg_learn_snapshot(sg_net *net);                                    /* brain.rs:343-347 */
int sg_learn_recall(sg_net *net, float alpha);                         /* brain.rs:349-356 */
/* eligibility [synapses] as of each synapse's last sync (Brain::eligibility),
   traces [total_neurons], steps since learning began (Brain::t); any may be null */
int sg_learn_read(sg_net *net, float *elig, float *trace_pre, float *trace_post, uint64_t *t);

/* ---- one network split across GPUs ---------------------------------------
   Each GPU simulates a contiguous slice of the neurons and holds the synapses
   onto them; the other GPUs' neurons are external populations here (same
   device indices on every GPU, so the scatter walks spiking neurons in the
   whole network's order and every ring cell gets the whole network's adds in
   the same order).  Per step: sg_step_begin (local neuron update), an
   exchange of this step's spike words (e.g. an NCCL all-gather of the
   sg_spike_words of every GPU), sg_step_end (external spikes, scatter,
   learning).  sg_step is refused on a network with external populations. */
int sg_pop_add_external(sg_net *net, uint32_t n, uint32_t *out_pop);
int sg_pop_set_external_source(sg_net *net, uint32_t pop, const uint32_t *dev_words);
int sg_spike_words(sg_net *net, uint32_t pop, const uint32_t **dev_words);
int sg_step_begin(sg_net *net);
int sg_step_end(sg_net *net);

/* ---- .taas v2 snapshots --------------------------------------------------
   The reference's container (crates/SiMuse/crates/taas-format:
   TaasWriter::push/to_bytes writer.rs:75-147, TaasReader::get_* /
   validate reader.rs:161-281, inspect_taas inspect.rs:5-53): magic "TAAS2",
   u64 LE manifest length, compact JSON manifest, section payloads, CRC32 per
   section over its uncompressed bytes, optional zstd (level 1..22; 0 = none;
   libzstd.so.1 loaded at run time).  The same sections and `created` give
   the same bytes as the reference's writer (uncompressed).  No GPU needed. */
int sg_taas_write(const char *path, const char *created /* null: clock */, const char *game /* null: none */,
                  uint32_t n_sections, const char *const *names, const char *const *kinds /* f32 i32 i64 u64
                  u8 str json blob */, const uint64_t *counts, const void *const *data, const uint64_t *bytes,
                  uint32_t n_meta, const char *const *keys, const char *const *values, int zstd_level);
/* uncompressed, CRC-checked bytes of a section of that kind; out may be null
   (size query via *bytes) */
int sg_taas_read(const char *path, const char *name, const char *kind, void *out, uint64_t cap, uint64_t *bytes);
int sg_taas_validate(const char *path);                             /* every section's CRC */
int sg_taas_inspect(const char *path, char *buf, uint64_t len, uint64_t *needed);
/* The built network as a snapshot (checkpoint): sections row_ptr, col_indices,
   values (the connectome sections of src/python/python/taas_format.rs:16-31),
   delays, syn_types, and eligibility while learning; metadata type, n_neurons,
   n_synapses, step; game "dioma". */
int sg_taas_save(sg_net *net, const char *path, const char *created, int zstd_level);
/* Resume: the snapshot's values as the built network's weights (its row_ptr
   and col_indices must be the network's; FP32 weights; ordered scatter path). */
int sg_taas_load_weights(sg_net *net, const char *path);
/* Builder: synapses from a .taas CSR, row i = neuron i of `from`, column j =
   neuron j of `to`; delays / syn_types sections when present. */
int sg_connect_taas(sg_net *net, uint32_t from, uint32_t to, const char *path, uint8_t default_delay);
/* Device bytes held by this network (state + CSR + rings + scratch). */
int sg_footprint(sg_net *net, uint64_t *out);
/* Per-neuron spike statistics accumulated on the device from the next step
   on (P/kernels/stats/rates.rs:1-40, isi.rs:27-66): spike count, and the
   mean and coefficient of variation of the inter-spike intervals (sample
   variance, only for neurons with >= 2 intervals, else 0) from FP64 sums;
   intervals in steps (the CV is unitless; rate = count / (steps * dt)).
   Enabling (again) restarts them. */
int sg_neuron_stats_enable(sg_net *net, int on);
int sg_neuron_stats_read(sg_net *net, uint32_t pop, uint32_t *counts, double *isi_mean_steps,
                         double *isi_cv, uint64_t *steps_observed);
/* Device stream of the handle (cudaStream_t), for event timing. */
int sg_stream(sg_net *net, void **out);

/* ---- stand-alone operators on device buffers ------------------------------ */
/* push_spikes(active, graph, delay, step), P/api/net/push.rs:126-173: for every
   neuron in `active` (device, strictly ascending, as compact_spikes_into
   returns) add each outgoing synapse's weight to
   ring[(step + max(delay,1)) % 32][post], each ring cell in the reference's
   order (bit-identical sums).  All arrays are device memory: a valid CSR
   (row_ptr[n_neurons+1], col/weights/delays[row_ptr[n_neurons]]) and the
   ring [32][n_neurons] floats.  `stream` is a cudaStream_t (NULL: legacy
   default stream).  Scratch is allocated per call (cudaMalloc/cudaFree);
   the call returns after the ring is updated.  Active or col entries
   >= n_neurons return SG_E_INVALID with the ring untouched. */
int sg_push_spikes(const uint32_t *row_ptr, const uint32_t *col, const float *weights,
                   const uint8_t *delays, uint32_t n_neurons, const uint32_t *active,
                   uint32_t n_active, uint64_t step, float *ring, void *stream);

/* No counterpart in the reference.  sg_push_spikes without any device
   allocation, for callers that cannot call cudaMalloc while they run: a
   real-time loop with no room in its timing budget for cudaMalloc/cudaFree
   (they can block in the driver and synchronise the device), or an
   embedding that is handed a fixed device-memory budget up front and owns
   every allocation itself.  Same arguments and results as sg_push_spikes;
   like it, the call waits on `stream` once (it reads the event count back)
   and returns after the ring is updated.  Its scratch is one file-scope
   __device__ array of about 12.1 MiB that every GPU loading this library
   holds until the process exits.  Limits: n_neurons <= 8,388,608 and at most
   1,048,576 synaptic events per call (the sum of the active rows' lengths);
   larger inputs return SG_E_INVALID / SG_E_OVERFLOW before the ring is
   touched, as do active or col entries >= n_neurons.  The first call on a
   device resolves the array's address on that device
   (cudaGetSymbolAddress), so make that first call before any stream capture;
   the address is kept until the process exits (do not call this again after
   a cudaDeviceReset of that device).  Every call shares the one array: calls
   that overlap on the GPU (other streams, other host threads) race and must
   be serialised by the caller. */
int sg_push_spikes_noalloc(const uint32_t *row_ptr, const uint32_t *col, const float *weights,
                           const uint8_t *delays, uint32_t n_neurons, const uint32_t *active,
                           uint32_t n_active, uint64_t step, float *ring, void *stream);

/* No counterpart in the reference: a measurement probe.  The rate
   (reductions per second) at which this GPU completes independent
   red.global.add.f32 operations on hashed cells of an n_cells-float array
   (the size of a network's delay rings), from a full-occupancy grid of
   `iters` reds per thread: the ceiling of the pre-centric scatter's event
   adds, as a STREAM copy is the ceiling of a streaming kernel.  Allocates
   and frees its own array. */
int sg_probe_red_rate(int device, uint64_t n_cells, uint32_t iters, double *reds_per_s);

/* ---- pools of resident networks (continuous batching) ----------------------
   No counterpart in the reference (its callers step one Network at a time;
   dioma-engine's pooled dynamics, dioma-engine/src/brain/dynamics/gpu_pool.rs,
   steps many creatures' networks as one).  A pool steps its member networks
   together: per step one neuron launch per model over every member's
   populations and one scatter launch over every member, on the pool's own
   stream.  Members stay independent networks (own state, synapses, rings,
   step counter, readbacks on their own stream); each gives the same bits in a
   pool as alone.  Members must be built, on the pool's device, on the
   pre-centric scatter (sg_scatter_mode EXACT or ATOMIC), without learning or
   external populations; at most 64.  sg_pool_step orders itself after the
   work queued on every member's stream and every member's later work after
   it.  A network leaves its pool when removed or destroyed. */
typedef struct sg_pool sg_pool;
int sg_pool_create(sg_pool **out, int device);
int sg_pool_destroy(sg_pool *pool);
int sg_pool_add(sg_pool *pool, sg_net *net);
int sg_pool_remove(sg_pool *pool, sg_net *net);
int sg_pool_size(sg_pool *pool, uint32_t *out);
int sg_pool_step(sg_pool *pool, uint32_t n_steps);
/* Waits for the pool's stream; SG_E_CUDA if a scatter wait timed out. */
int sg_pool_synchronize(sg_pool *pool);

/* ---- batched Kuramoto populations ----------------------------------------- */
/* A batch of independent all-to-all Kuramoto populations integrated by RK4:
     dth_i/dt = omega_i + K/N sum_j sin(th_j - th_i)
              = omega_i + K (S cos th_i - C sin th_i),  C + iS = mean e^{i th},
   the exact mean-field identity of crates/SiMuse/crates/t3/src/oscillator.rs:
   15-20,549, so each RK4 stage costs one O(N) reduction instead of the O(N^2)
   dense sum of P/kernels/phase/sparse.rs:40-140.  After each step the phase
   wraps to [-pi, pi] as P/kernels/phase/kuramoto.rs:42-68 does
   (th - 2 pi round(th / 2 pi)).  Phases are FP32; the order parameter
   r(t) = |mean e^{i th}| is recorded per step in FP32 and its time average is
   accumulated in FP64 (t3/src/oscillator.rs:440-450).  Instance sizes are
   1..65,536 oscillators; instance i's oscillators are [off_i, off_i + n_i)
   with off_i the prefix sum of sizes. */
typedef struct sg_kura sg_kura;
int sg_kuramoto_create(sg_kura **out, int device, uint32_t n_instances, const uint32_t *sizes,
                       const float *coupling, float dt);
int sg_kuramoto_destroy(sg_kura *kb);
/* Total oscillators over all instances (length of theta/omega arrays). */
int sg_kuramoto_total(sg_kura *kb, uint64_t *out);
/* Phases (radians) and natural frequencies, `total` each, instance-major. */
int sg_kuramoto_set_state(sg_kura *kb, const float *theta, const float *omega);
/* Keep r(t) of the next `max_steps` steps (0 turns recording off). */
int sg_kuramoto_record(sg_kura *kb, uint64_t max_steps);
/* Advance every instance by n_steps RK4 steps (asynchronous). */
int sg_kuramoto_run(sg_kura *kb, uint32_t n_steps);
int sg_kuramoto_synchronize(sg_kura *kb);
int sg_kuramoto_get_theta(sg_kura *kb, float *theta);
/* Recorded r(t), [n_instances][n_steps] row-major; cap = floats available. */
int sg_kuramoto_get_r(sg_kura *kb, float *r, uint64_t cap, uint64_t *n_steps);
/* Time average of r(t) over all steps run so far, FP64, per instance. */
int sg_kuramoto_get_r_mean(sg_kura *kb, double *r_mean);
int sg_kuramoto_stream(sg_kura *kb, void **out);

#ifdef __cplusplus
}
#endif
#endif
