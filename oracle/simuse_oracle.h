/*
 * simuse_oracle.h — C API of the CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * This library is a plain C++ restatement of the reference's CPU
 * simulation step (crates/SiMuse/crates/pillars/src/api/net/…).  It exists
 * to check the CUDA product against, and to time the reference algorithm on
 * host cores.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.  The product (libsimuse_b200.so) never links it.
 *
 * Parity pin: the oracle is checked against every golden vector the
 * reference's own tests hold for this path (LIF spike counts, delay arrival,
 * push slot arithmetic, delay-ring contract, compaction); see
 * tests/test_oracle_golden.py.  The HH-RK4, pair-STDP and Kuramoto-RK4 parts
 * have no reference implementation and are oracle-defined (FP64 twins).
 *
 * All functions return >= 0 on success and a negative error code on a
 * contract violation (the reference panics); or_last_error() explains.
 */
#ifndef SIMUSE_ORACLE_H
#define SIMUSE_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_net or_net;

/* precision: 0 = FP32 (reference arithmetic), 1 = FP64 twin */
or_net *or_net_new(int precision);
void or_net_free(or_net *net);
const char *or_last_error(void);

int or_pop_add(or_net *net, int model, uint32_t n);
int or_pop_fill_param(or_net *net, int pop, int col, double v);
int or_pop_fill_state(or_net *net, int pop, int col, double v);
int or_pop_set_param(or_net *net, int pop, int col, const float *v, uint32_t n);
int or_pop_set_state(or_net *net, int pop, int col, const float *v, uint32_t n);
int or_pop_get_state(or_net *net, int pop, int col, float *out, uint32_t n);
int or_pop_get_state_f64(or_net *net, int pop, int col, double *out, uint32_t n);
int or_pop_get_param(or_net *net, int pop, int col, float *out, uint32_t n);

/* flags bit 0: the edges take part in pair STDP */
int or_connect(or_net *net, int from, const uint32_t *from_idx, int to,
               const uint32_t *to_idx, const float *w, const uint8_t *delay,
               const uint8_t *syn_type, const uint8_t *plast_type, uint64_t n, uint32_t flags);
/* Tsodyks-Markram profile; returns its id (1-based) or a negative status */
int or_register_plasticity(or_net *net, float u0, float tau_rec, int facilitation, float tau_fac, float dt);
int or_tm_sequence(float u0, float a_rec, float a_fac, int facilitation, float w, const uint64_t *steps,
                   uint32_t n, float *out);
int or_register_expone(or_net *net, float tau_decay, float erev, float dt);
/* SynapticBrain receptor kinetics (pillars-connectome/src/synaptic.rs):
   syn_types are receptor codes 0..6 (others AMPA), delays ignored; the seven
   conductances [7][total] read and written in receptor-code order */
int or_set_receptor_kinetics(or_net *net, float dt);
int or_receptor_read(or_net *net, float *g);
int or_receptor_write(or_net *net, const float *g);
/* the receptor kinetics' parts alone: DecayFactors::new(dt) in code order,
   compute_currents of n neurons (g [7][n]) into i_out, nmda_mg_block(v) */
int or_receptor_factors(float dt, float *f);
int or_receptor_currents(uint32_t n, const float *g, const float *v, float *i_out);
float or_nmda_mg_block(float v);
/* kind 0 ExpOne {tau_decay}, 1 ExpTwo {tau_rise, tau_decay}, 2 Alpha {tau},
   3 ExpThree {tau_rise, tau_decay1, tau_decay2, gbase1, gbase2} */
int or_register_kinetics(or_net *net, int kind, const float *params, float erev, float dt);
/* dopamine-modulated eligibility learning (P/api/learn/brain.rs) over the
   built network's synapses; reward w_cap: non-finite = the config's w_max */
/* a network split across processes: external populations (simulated by
   another rank), the step in two halves around the spike exchange */
int or_pop_add_external(or_net *net, uint32_t n);
int or_step_begin(or_net *net);
int or_set_external_spikes(or_net *net, int pop, const int32_t *spikes, uint32_t n);
int or_step_end(or_net *net);
int or_learn_enable(or_net *net, float dt, float tau_pre, float tau_post, float tau_e, float a_ltp,
                    float a_ltd, float lr, float w_min, float w_max);
int or_learn_reward(or_net *net, float dopamine, float gate, float w_cap);
int or_learn_clear(or_net *net);
int or_learn_reward_range(or_net *net, uint64_t lo, uint64_t hi, float dopamine, float gate, float w_cap);
int or_learn_clear_range(or_net *net, uint64_t lo, uint64_t hi);
int or_pop_synapse_range(or_net *net, int pop, uint64_t *lo, uint64_t *hi);
int or_learn_restrict(or_net *net, const uint8_t *keep, uint64_t n);
int or_learn_set_eligibility(or_net *net, const float *elig, uint64_t n);
int or_learn_motor(or_net *net, uint64_t lo0, uint64_t hi0, uint64_t lo1, uint64_t hi1);
int or_learn_motor_read(or_net *net, uint32_t *out);
int or_learn_snapshot(or_net *net);
int or_learn_recall(or_net *net, float alpha);
int or_learn_read(or_net *net, float *elig, float *trace_pre, float *trace_post, uint64_t *t);
int or_poisson_add(or_net *net, float rate_hz, float dt_ms, uint32_t seed);
int or_poisson_add_many(or_net *net, uint32_t n, float rate_hz, float dt_ms, uint32_t seed0);
int or_poisson_connect_one_to_one(or_net *net, int first, uint32_t n, int to, float w, uint8_t delay);
int or_poisson_connect(or_net *net, int src, int to, const uint32_t *posts,
                       const float *w, const uint8_t *delay,
                       const uint8_t *syn_type, uint64_t n);
int or_poisson_connect_plastic(or_net *net, int src, int to, const uint32_t *posts, const float *w,
                               const uint8_t *delay, const uint8_t *syn_type, const uint8_t *plast_type,
                               uint64_t n);
int or_stdp_config(or_net *net, float dt, float tau_pre, float tau_post,
                   float a_plus, float a_minus, float w_min, float w_max);
int or_build(or_net *net);
/* Fixed in-degree projection (the product's sg_connect_fixed_indegree
   generator) + build, straight into the CSR; network must have no other edges. */
int or_build_fixed_indegree(or_net *net, int from, int to, uint32_t k_in, uint64_t seed,
                            uint32_t n_exc, float w_exc, float w_inh, uint32_t d_min,
                            uint32_t d_max);
/* Build straight from a CSR (reference: SparseGraph::from_csr). */
int or_build_from_csr(or_net *net, const uint32_t *row_ptr, const uint32_t *col,
                      const float *w, const uint8_t *delay);

int or_inject(or_net *net, int pop, const uint32_t *idx, const float *v, uint64_t n);
/* raster: NULL or n_steps * total_neurons bytes (1 = spike) */
int or_step(or_net *net, uint32_t n_steps, uint8_t *raster);
int or_spikes(or_net *net, int pop, int32_t *out, uint32_t n);
uint64_t or_step_counter(const or_net *net);
uint64_t or_total_neurons(const or_net *net);
uint64_t or_num_synapses(const or_net *net);
uint64_t or_events(const or_net *net); /* synaptic events pushed so far */
int or_ring_read(or_net *net, int ring, float *out); /* ring 0 static, k = kinetic k */
int or_graph_read(or_net *net, uint32_t *row_ptr, uint32_t *col, float *w, uint8_t *delay);
int or_weights_read(or_net *net, float *w); /* current CSR weights (STDP) */
int or_weights_write(or_net *net, const float *w, uint64_t n);
double or_stdp_drift(const or_net *net);
int or_traces_read(or_net *net, float *x_pre, float *x_post);
int or_set_threads(int n);

/* ---- stand-alone reference pieces, for golden checks ---- */
float or_fast_exp(float x);
float or_sg_expf(float x);
float or_sg_logf(float x);
int or_poisson_spike(uint32_t seed, uint32_t stream, uint64_t step, float p);
uint64_t or_compact(const int32_t *spikes, uint64_t n, uint32_t *out);
int or_push_spikes(const uint32_t *row_ptr, const uint32_t *col, const float *w,
                   const uint8_t *delay, uint32_t n_neurons, const uint32_t *active,
                   uint32_t n_active, uint64_t step, float *ring);

/* ---- Kuramoto, mean-field RK4 (FP32 and FP64 twins) ---- */
int or_kuramoto_rk4(int precision, uint32_t n, const float *theta0,
                    const float *omega, float k, float dt, uint32_t n_steps,
                    float *theta_out, double *r_out);

#ifdef __cplusplus
}
#endif
#endif
