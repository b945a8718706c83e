// simuse_b200.hpp — C++ mirror of the reference's Network builder/step API
// over the C ABI of simuse_b200.h (header only).
//
// The method set follows pillars::api::Network (crates/SiMuse/crates/
// pillars/src/api/net/network/core.rs:87-622, build.rs:18-276, step.rs:
// 18-189): populations in creation order, neuron indices within a population,
// delays in steps (< 32).  Where the reference panics (assert!/panic!), the
// C ABI returns a negative status and this wrapper throws simuse::Error with
// the library's message.  One Network owns one device-resident network and
// its CUDA stream; it is movable, not copyable.
#pragma once

#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "simuse_b200.h"

namespace simuse {

class Error : public std::runtime_error {
 public:
  Error(int status, const std::string &msg) : std::runtime_error(msg), status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

inline void check(int rc) {
  if (rc < 0) {
    char buf[1024];
    sg_last_error(buf, sizeof buf);
    throw Error(rc, buf);
  }
}

enum class Model { Lif = SG_LIF, Izhikevich = SG_IZH, Gpea = SG_GPEA, HodgkinHuxley = SG_HH };
using PopulationId = uint32_t;

// P/api/learn/brain.rs:24-60 StdpConfig (its defaults)
struct LearnConfig {
  float dt = 0.5f, tau_pre = 20.0f, tau_post = 20.0f, tau_e = 1000.0f, a_ltp = 0.1f, a_ltd = 0.12f, lr = 1.0f,
        w_min = 0.0f, w_max = 1.0f;
};

class Network {
 public:
  explicit Network(int device = 0) { check(sg_net_create(&h_, device)); }
  ~Network() {
    if (h_) sg_net_destroy(h_);
  }
  Network(const Network &) = delete;
  Network &operator=(const Network &) = delete;
  Network(Network &&o) noexcept : h_(std::exchange(o.h_, nullptr)), sizes_(std::move(o.sizes_)) {}
  Network &operator=(Network &&o) noexcept {
    if (this != &o) {
      if (h_) sg_net_destroy(h_);
      h_ = std::exchange(o.h_, nullptr);
      sizes_ = std::move(o.sizes_);
    }
    return *this;
  }

  // -- builder (core.rs) -------------------------------------------------------
  PopulationId add_population(Model m, uint32_t n) {
    uint32_t id = 0;
    check(sg_pop_add(h_, static_cast<int>(m), n, &id));
    sizes_.push_back(n);
    return id;
  }
  void fill_param(PopulationId p, uint32_t col, float v) { check(sg_pop_fill_param(h_, p, col, v)); }
  void fill_state(PopulationId p, uint32_t col, float v) { check(sg_pop_fill_state(h_, p, col, v)); }
  void set_param(PopulationId p, uint32_t col, const std::vector<float> &v) {
    check(sg_pop_set_param(h_, p, col, v.data(), (uint32_t)v.size()));
  }
  void set_state(PopulationId p, uint32_t col, const std::vector<float> &v) {
    check(sg_pop_set_state(h_, p, col, v.data(), (uint32_t)v.size()));
  }
  void connect(PopulationId from, const std::vector<uint32_t> &from_idx, PopulationId to,
               const std::vector<uint32_t> &to_idx, const std::vector<float> &weights,
               const std::vector<uint8_t> &delays) {
    if (from_idx.size() != to_idx.size() || from_idx.size() != weights.size() || from_idx.size() != delays.size())
      throw Error(SG_E_INVALID, "connect: slice length mismatch");
    check(sg_connect(h_, from, from_idx.data(), to, to_idx.data(), weights.data(), delays.data(), from_idx.size()));
  }
  uint32_t add_poisson_source(float rate_hz, float dt_ms, uint32_t seed) {
    uint32_t id = 0;
    check(sg_poisson_add(h_, rate_hz, dt_ms, seed, &id));
    return id;
  }
  void connect_poisson_source(uint32_t src, PopulationId to, const std::vector<uint32_t> &posts,
                              const std::vector<float> &weights, const std::vector<uint8_t> &delays) {
    check(sg_poisson_connect(h_, src, to, posts.data(), weights.data(), delays.data(), nullptr, posts.size()));
  }
  void build() { check(sg_build(h_)); }

  // -- run (build.rs / step.rs) ---------------------------------------------------
  void inject_current(PopulationId p, const std::vector<uint32_t> &idx, const std::vector<float> &vals) {
    if (idx.size() != vals.size()) throw Error(SG_E_INVALID, "inject_current: length mismatch");
    check(sg_inject(h_, p, idx.data(), vals.data(), idx.size()));
  }
  void step(uint32_t n = 1) { check(sg_step(h_, n)); }
  void synchronize() { check(sg_synchronize(h_)); }

  // -- readouts -------------------------------------------------------------------
  std::vector<int32_t> spikes(PopulationId p) const {
    std::vector<int32_t> out(sizes_.at(p));
    check(sg_spikes(h_, p, out.data(), (uint32_t)out.size()));
    return out;
  }
  std::vector<float> state(PopulationId p, uint32_t col) const {
    std::vector<float> out(sizes_.at(p));
    check(sg_pop_get_state(h_, p, col, out.data(), (uint32_t)out.size()));
    return out;
  }
  uint64_t step_counter() const {
    uint64_t s = 0;
    check(sg_step_counter(h_, &s));
    return s;
  }
  uint64_t total_neurons() const {
    uint64_t n = 0;
    check(sg_total_neurons(h_, &n));
    return n;
  }
  uint64_t num_synapses() const {
    uint64_t n = 0;
    check(sg_num_synapses(h_, &n));
    return n;
  }
  std::vector<float> weights() const {
    std::vector<float> w(num_synapses());
    check(sg_weights_read(h_, w.data()));
    return w;
  }

  // -- dopamine learning on the network's synapses (brain.rs Brain / LearnToken) --
  void enable_learning(const LearnConfig &c = {}) {
    check(sg_learn_enable(h_, c.dt, c.tau_pre, c.tau_post, c.tau_e, c.a_ltp, c.a_ltd, c.lr, c.w_min, c.w_max));
  }
  void reward(float dopamine) { check(sg_learn_reward(h_, dopamine, 1.0f, std::nanf(""))); }
  void reward_gated(float dopamine, float gate) { check(sg_learn_reward(h_, dopamine, gate, std::nanf(""))); }
  void reward_capped(float dopamine, float w_cap) { check(sg_learn_reward(h_, dopamine, 1.0f, w_cap)); }
  void clear_eligibility() { check(sg_learn_clear(h_)); }
  std::vector<float> eligibility() const {
    std::vector<float> e(num_synapses());
    check(sg_learn_read(h_, e.data(), nullptr, nullptr, nullptr));
    return e;
  }
  // -- .taas v2 snapshots (taas-format) --------------------------------------------
  void save_taas(const std::string &path, int zstd_level = 0) {
    check(sg_taas_save(h_, path.c_str(), nullptr, zstd_level));
  }
  void load_weights_taas(const std::string &path) { check(sg_taas_load_weights(h_, path.c_str())); }
  void connect_taas(PopulationId from, PopulationId to, const std::string &path, uint8_t default_delay = 1) {
    check(sg_connect_taas(h_, from, to, path.c_str(), default_delay));
  }

  // -- one network split across GPUs ------------------------------------------------
  PopulationId add_external_population(uint32_t n) {
    uint32_t id = 0;
    check(sg_pop_add_external(h_, n, &id));
    sizes_.push_back(n);
    return id;
  }
  void set_external_source(PopulationId p, const uint32_t *dev_words) {
    check(sg_pop_set_external_source(h_, p, dev_words));
  }
  const uint32_t *spike_words(PopulationId p) const {
    const uint32_t *w = nullptr;
    check(sg_spike_words(h_, p, &w));
    return w;
  }
  void step_begin() { check(sg_step_begin(h_)); }
  void step_end() { check(sg_step_end(h_)); }
  sg_net *handle() const { return h_; }

 private:
  sg_net *h_ = nullptr;
  std::vector<uint32_t> sizes_;
};

}  // namespace simuse
