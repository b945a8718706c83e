"""``Network`` — the reference's builder/step API over the B200 C ABI.

Method names, argument meaning and error behaviour follow
``pillars::api::Network`` (crates/SiMuse/crates/pillars/src/api/net/network/
core.rs:87-622, build.rs:18-276, step.rs:18-189): populations in creation
order, neuron indices within a population, delays in steps (< 32), errors
where the reference panics (raised here as SimuseError).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib

LIF, IZH, GPEA, HH = 1, 2, 3, 4
W_F32, W_BF16, W_FP8 = 0, 1, 2
EDGE_STDP = 1

N_PARAMS = {LIF: 6, IZH: 7, GPEA: 14, HH: 10}
N_STATE = {LIF: 2, IZH: 3, GPEA: 9, HH: 4}


def _p(a):
    return None if a is None else a.ctypes.data


def _random_w(r) -> int:
    """random_w of the device generators: False/True, or an int b >= 2 (U on
    the 2^-b grid)."""
    if isinstance(r, bool):
        return 1 if r else 0
    return int(r)


class Network:
    """One simulated network resident on one GPU (one CUDA stream)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().sg_net_create(C.byref(h), device))
        self._h = h
        self._sizes: list[int] = []
        self._models: list[int] = []
        self.device = device

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().sg_net_destroy(h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- builder (core.rs) ---------------------------------------------------
    def add_population(self, model: int, n: int) -> int:
        out = C.c_uint32()
        check(lib().sg_pop_add(self._h, model, n, C.byref(out)))
        self._sizes.append(n)
        self._models.append(model)
        return out.value

    def fill_param(self, pop: int, col: int, value: float):
        check(lib().sg_pop_fill_param(self._h, pop, col, float(value)))

    def fill_state(self, pop: int, col: int, value: float):
        check(lib().sg_pop_fill_state(self._h, pop, col, float(value)))

    def set_param(self, pop: int, col: int, values):
        a = np.ascontiguousarray(values, np.float32)
        check(lib().sg_pop_set_param(self._h, pop, col, _p(a), a.size))

    def set_state(self, pop: int, col: int, values):
        a = np.ascontiguousarray(values, np.float32)
        check(lib().sg_pop_set_state(self._h, pop, col, _p(a), a.size))

    def state(self, pop: int, col: int) -> np.ndarray:
        out = np.empty(self._sizes[pop], np.float32)
        check(lib().sg_pop_get_state(self._h, pop, col, _p(out), out.size))
        return out

    def param_slice(self, pop: int, col: int) -> np.ndarray:
        out = np.empty(self._sizes[pop], np.float32)
        check(lib().sg_pop_get_param(self._h, pop, col, _p(out), out.size))
        return out

    def connect(self, frm, from_idx, to, to_idx, weights, delays, syn_types=None, stdp=False, plast_types=None):
        """Edges from[from_idx[i]] -> to[to_idx[i]]; optional per-edge kinetic
        synapse types, pair STDP, and short-term plasticity profile ids
        (register_plasticity; 0 = none)."""
        fi = np.ascontiguousarray(from_idx, np.uint32)
        ti = np.ascontiguousarray(to_idx, np.uint32)
        w = np.ascontiguousarray(weights, np.float32)
        d = np.ascontiguousarray(delays, np.uint8)
        st = None if syn_types is None else np.ascontiguousarray(syn_types, np.uint8)
        pt = None if plast_types is None else np.ascontiguousarray(plast_types, np.uint8)
        if not (fi.size == ti.size == w.size == d.size) or (st is not None and st.size != fi.size) \
                or (pt is not None and pt.size != fi.size):
            from ._lib import SimuseError
            raise SimuseError(-1, "connect: slice length mismatch")
        if pt is None:
            check(lib().sg_connect_ex(self._h, frm, _p(fi), to, _p(ti), _p(w), _p(d), _p(st), fi.size,
                                      EDGE_STDP if stdp else 0))
        else:
            check(lib().sg_connect_plastic(self._h, frm, _p(fi), to, _p(ti), _p(w), _p(d), _p(st), _p(pt),
                                           fi.size, EDGE_STDP if stdp else 0))

    def register_plasticity(self, u0: float, tau_rec: float, dt: float, tau_fac: float | None = None) -> int:
        """Tsodyks-Markram profile (depression; with facilitation when tau_fac
        is given) for steps of dt ms; returns its 1-based id."""
        out = C.c_uint32()
        check(lib().sg_register_plasticity(self._h, u0, tau_rec, 0 if tau_fac is None else 1,
                                           0.0 if tau_fac is None else tau_fac, dt, C.byref(out)))
        return out.value

    def connect_fixed_indegree(self, frm, to, k_in, seed, n_exc, w_exc, w_inh, d_min, d_max,
                               syn_type_exc=0, syn_type_inh=0, stdp_exc=False):
        check(lib().sg_connect_fixed_indegree(self._h, frm, to, k_in, seed, n_exc, w_exc, w_inh,
                                              d_min, d_max, syn_type_exc, syn_type_inh,
                                              EDGE_STDP if stdp_exc else 0))

    def connect_fixed_outdegree(self, frm, to, k, seed, no_self, n_exc, w_exc, w_inh, random_w=True, delay=1,
                                d_max=None, syn_type_exc=0, syn_type_inh=0, stdp_exc=False):
        """k distinct targets per source, generated on the device
        (sg_connect_fixed_outdegree); weights w_exc/w_inh times U(0,1);
        delay uniform in [delay, d_max] (d_max defaults to delay)."""
        check(lib().sg_connect_fixed_outdegree(self._h, frm, to, k, seed, 1 if no_self else 0, n_exc,
                                               float(w_exc), float(w_inh), _random_w(random_w), delay,
                                               delay if d_max is None else d_max, syn_type_exc, syn_type_inh,
                                               EDGE_STDP if stdp_exc else 0))

    def connect_lognormal_outdegree(self, frm, to, mean, sd, seed, no_self, n_exc, w_exc, w_inh,
                                    random_w=True, delay=1, d_max=None, syn_type_exc=0, syn_type_inh=0,
                                    stdp_exc=False):
        """Lognormal out-degree per source, distinct targets, generated on the
        device (sg_connect_lognormal_outdegree)."""
        check(lib().sg_connect_lognormal_outdegree(self._h, frm, to, float(mean), float(sd), seed,
                                                   1 if no_self else 0, n_exc, float(w_exc), float(w_inh),
                                                   _random_w(random_w), delay, delay if d_max is None else d_max,
                                                   syn_type_exc, syn_type_inh, EDGE_STDP if stdp_exc else 0))

    def register_expone(self, tau_decay: float, erev: float, dt: float) -> int:
        out = C.c_uint32()
        check(lib().sg_register_expone(self._h, tau_decay, erev, dt, C.byref(out)))
        return out.value

    def register_kinetics(self, kind: int, params, erev: float, dt: float) -> int:
        """Kinetic synapse profile: kind 0 ExpOne {tau_decay}, 1 ExpTwo
        {tau_rise, tau_decay}, 2 Alpha {tau}, 3 ExpThree {tau_rise, tau_decay1,
        tau_decay2, gbase1, gbase2}; returns its 1-based id (the syn_type)."""
        p = np.zeros(5, np.float32)
        p[:len(params)] = params
        out = C.c_uint32()
        check(lib().sg_register_kinetics(self._h, int(kind), _p(p), erev, dt, C.byref(out)))
        return out.value

    def set_receptor_kinetics(self, dt: float):
        """SynapticBrain receptor kinetics (before any connect): syn_types
        become receptor codes (RECEPTORS), delays are ignored."""
        check(lib().sg_set_receptor_kinetics(self._h, dt))
        self._receptor = True

    def receptor_conductances(self) -> np.ndarray:
        """The seven conductances, [receptor code][neuron]."""
        out = np.empty((7, self.total_neurons), np.float32)
        check(lib().sg_receptor_read(self._h, _p(out)))
        return out

    def set_receptor_conductances(self, g):
        g = np.ascontiguousarray(g, np.float32)
        if g.shape != (7, self.total_neurons):
            raise ValueError("conductances must be [7][total neurons]")
        check(lib().sg_receptor_write(self._h, _p(g)))

    def add_poisson_source(self, rate_hz: float, dt_ms: float, seed: int) -> int:
        out = C.c_uint32()
        check(lib().sg_poisson_add(self._h, rate_hz, dt_ms, seed, C.byref(out)))
        return out.value

    def add_poisson_sources(self, n: int, rate_hz: float, dt_ms: float, seeds=None, seed0: int = 0) -> int:
        out = C.c_uint32()
        s = None if seeds is None else np.ascontiguousarray(seeds, np.uint32)
        check(lib().sg_poisson_add_many(self._h, n, rate_hz, dt_ms, _p(s), seed0, C.byref(out)))
        return out.value

    def connect_poisson_source(self, src, to, posts, weights, delays, syn_types=None, plast_types=None):
        p = np.ascontiguousarray(posts, np.uint32)
        w = np.ascontiguousarray(weights, np.float32)
        d = np.ascontiguousarray(delays, np.uint8)
        st = None if syn_types is None else np.ascontiguousarray(syn_types, np.uint8)
        pt = None if plast_types is None else np.ascontiguousarray(plast_types, np.uint8)
        check(lib().sg_poisson_connect_plastic(self._h, src, to, _p(p), _p(w), _p(d), _p(st), _p(pt), p.size))

    def connect_poisson_one_to_one(self, first_src, n, to, weight, delay, posts=None):
        p = None if posts is None else np.ascontiguousarray(posts, np.uint32)
        check(lib().sg_poisson_connect_one_to_one(self._h, first_src, n, to, _p(p), weight, delay))

    def stdp_config(self, dt, tau_pre, tau_post, a_plus, a_minus, w_min, w_max):
        check(lib().sg_stdp_config(self._h, dt, tau_pre, tau_post, a_plus, a_minus, w_min, w_max))

    def set_weight_format(self, fmt: int):
        check(lib().sg_set_weight_format(self._h, fmt))

    @property
    def scatter_mode(self) -> str:
        """"ordered", "exact" or "atomic": the scatter path of the built network."""
        m = C.c_int()
        check(lib().sg_scatter_mode(self._h, C.byref(m)))
        return ("ordered", "exact", "atomic")[m.value]

    @property
    def scatter_schedule(self) -> tuple[int, int]:
        """(variant, blocks per SM) of the pre-centric scatter: 0-3 the staged
        pipeline's stage-ring shapes, 4-8 the warp walk (5 and 6 pipelined, 7
        and 8 rows in 4 pieces)."""
        v, b = C.c_int(), C.c_uint32()
        check(lib().sg_scatter_schedule(self._h, C.byref(v), C.byref(b)))
        return v.value, b.value

    def set_deterministic(self, on: bool):
        check(lib().sg_set_deterministic(self._h, 1 if on else 0))

    def build(self):
        check(lib().sg_build(self._h))

    def build_from_csr(self, row_ptr, col, weights, delays):
        rp = np.ascontiguousarray(row_ptr, np.uint32)
        c = np.ascontiguousarray(col, np.uint32)
        w = np.ascontiguousarray(weights, np.float32)
        d = np.ascontiguousarray(delays, np.uint8)
        check(lib().sg_build_from_csr(self._h, _p(rp), _p(c), _p(w), _p(d)))

    # -- run (build.rs / step.rs) -----------------------------------------------
    def set_noise(self, pop: int, seed: int, sigma_lo: float, sigma_hi: float | None = None,
                  split: int | None = None, stream: int = 4, stride: int | None = None, step0: int = 0):
        """Device Gaussian input: neuron i gets sigma_i * N(0,1) each step from
        counter i + (step - step0) * stride (stride defaults to the population
        size); sigma_i = sigma_lo below `split`, sigma_hi from there on."""
        n = self._sizes[pop]
        check(lib().sg_pop_set_noise(self._h, pop, int(seed), int(stream), int(n if stride is None else stride),
                                     int(step0), float(sigma_lo), float(sigma_lo if sigma_hi is None else sigma_hi),
                                     int(n if split is None else split)))

    def set_bias(self, pop: int, values):
        """Constant input current per neuron, added every step (sg_pop_set_bias)."""
        a = np.ascontiguousarray(values, np.float32)
        check(lib().sg_pop_set_bias(self._h, pop, _p(a), a.size))

    def clear_rings(self):
        """Empty the delay rings (the state of a freshly built network)."""
        check(lib().sg_ring_clear(self._h))

    def inject_current(self, pop, indices, values):
        i = np.ascontiguousarray(indices, np.uint32)
        v = np.ascontiguousarray(values, np.float32)
        if i.size != v.size:
            from ._lib import SimuseError
            raise SimuseError(-1, "inject_current: indices/values length mismatch")
        check(lib().sg_inject(self._h, pop, _p(i), _p(v), i.size))

    def step(self, n_steps: int = 1):
        check(lib().sg_step(self._h, n_steps))

    def idle(self) -> bool:
        """True when every step queued so far has finished (non-blocking)."""
        out = C.c_int()
        check(lib().sg_query(self._h, C.byref(out)))
        return bool(out.value)

    def synchronize(self):
        check(lib().sg_synchronize(self._h))

    def autotune(self, steps: int = 200) -> dict:
        """Picks the pre-centric scatter's schedule on the next candidates x
        `steps` simulation steps (they are ordinary steps); returns the per-step
        times of the fixed and the chosen schedule."""
        fixed, best = C.c_float(), C.c_float()
        v, bps = C.c_int(), C.c_uint32()
        check(lib().sg_autotune(self._h, steps, C.byref(fixed), C.byref(best), C.byref(v), C.byref(bps)))
        return {"fixed_ms_per_step": fixed.value, "tuned_ms_per_step": best.value, "variant": v.value,
                "blocks_per_sm": bps.value}

    def debug_stall_scatter(self, on: bool):
        """Test hook: the pre-centric scatter's producer stops feeding its
        consumers, whose bounded waits run out and report an error."""
        check(lib().sg_debug_stall_scatter(self._h, 1 if on else 0))

    def enable_raster(self, capacity_steps: int):
        check(lib().sg_raster_enable(self._h, capacity_steps))
        self._raster_mark = self.step_counter
        self._raster_cap = int(capacity_steps)

    def raster_fetch_csr(self, off_buf: "PinnedU32", idx_buf: "PinnedU32"):
        """The staged batch as (t0, step offsets, indices): the spikes of step
        t0 + s are indices[offsets[s]:offsets[s + 1]].  Copied through the
        page-locked buffers (grown when too small) into new arrays."""
        t0, k, n = C.c_uint64(), C.c_uint64(), C.c_uint64()
        off_buf.ensure(getattr(self, "_raster_cap", 0) + 1)
        while True:
            rc = lib().sg_raster_fetch_csr(self._h, off_buf.ptr, off_buf.n, idx_buf.ptr, idx_buf.n, C.byref(t0),
                                           C.byref(k), C.byref(n))
            if rc < 0 and n.value > idx_buf.n:  # too small: the batch stays staged
                idx_buf.ensure(n.value + n.value // 2)
                continue
            check(rc)
            break
        kk, nn = int(k.value), int(n.value)
        return int(t0.value), off_buf.a[:kk + 1].copy(), idx_buf.a[:nn].copy()

    def read_raster(self) -> np.ndarray:
        """Spike raster [steps since the last read][total_neurons] as uint8."""
        n = C.c_uint32()
        k = self.step_counter - getattr(self, "_raster_mark", 0)
        out = np.zeros(max(k * self.total_neurons, 1), np.uint8)
        check(lib().sg_raster_read(self._h, _p(out), out.size, C.byref(n)))
        self._raster_mark = self.step_counter
        return out[: n.value * self.total_neurons].reshape(n.value, self.total_neurons)

    def read_spike_events(self, capacity: int | None = None):
        """(steps, indices) of every spike recorded since the last read,
        ordered by step then neuron (compacted on the device)."""
        n = C.c_uint64()
        if capacity is None:
            k = self.step_counter - getattr(self, "_raster_mark", 0)
            capacity = max(1, min(k * self.total_neurons, 1 << 20))
        st = np.empty(capacity, np.uint32)
        ix = np.empty(capacity, np.uint32)
        rc = lib().sg_raster_read_events(self._h, _p(st), _p(ix), capacity, C.byref(n))
        if rc < 0 and n.value > capacity:  # too small: nothing was consumed, read again at the exact size
            st = np.empty(n.value, np.uint32)
            ix = np.empty(n.value, np.uint32)
            rc = lib().sg_raster_read_events(self._h, _p(st), _p(ix), n.value, C.byref(n))
        check(rc)
        self._raster_mark = self.step_counter
        return st[: n.value], ix[: n.value]

    def raster_stage(self):
        """Queue the compaction of the steps recorded since the last read,
        right after them, without waiting (fetch with raster_fetch)."""
        check(lib().sg_raster_stage(self._h))
        self._raster_mark = self.step_counter

    def raster_fetch(self, capacity: int = 1 << 20):
        """(steps, indices) of the staged batch; waits for its compaction."""
        n = C.c_uint64()
        st = np.empty(capacity, np.uint32)
        ix = np.empty(capacity, np.uint32)
        rc = lib().sg_raster_fetch(self._h, _p(st), _p(ix), capacity, C.byref(n))
        if rc < 0 and n.value > capacity:  # too small: the batch stays staged, fetch it at its size
            st = np.empty(n.value, np.uint32)
            ix = np.empty(n.value, np.uint32)
            rc = lib().sg_raster_fetch(self._h, _p(st), _p(ix), n.value, C.byref(n))
        check(rc)
        return st[: n.value], ix[: n.value]

    def raster_counts(self) -> np.ndarray:
        """Spikes per neuron over every event read since the raster was enabled."""
        out = np.empty(self.total_neurons, np.uint32)
        check(lib().sg_raster_counts(self._h, _p(out)))
        return out

    def read_spike_events_into(self, steps: np.ndarray, idx: np.ndarray) -> int:
        """Zero-allocation variant for preallocated (pinned) host buffers."""
        n = C.c_uint64()
        check(lib().sg_raster_read_events(self._h, _p(steps), _p(idx), steps.size, C.byref(n)))
        self._raster_mark = self.step_counter
        return n.value

    def profile(self, on: bool):
        check(lib().sg_profile_enable(self._h, 1 if on else 0))

    def profile_read(self):
        ms = np.zeros(4, np.float64)
        launches = np.zeros(4, np.uint64)
        check(lib().sg_profile_read(self._h, _p(ms), _p(launches)))
        return ms, launches

    def read_stats(self):
        k = C.c_uint32()
        n = max(1, self.step_counter - getattr(self, "_stats_mark", 0))
        spk = np.zeros(n, np.uint32)
        ev = np.zeros(n, np.uint64)
        check(lib().sg_stats_read(self._h, _p(spk), _p(ev), n, C.byref(k)))
        self._stats_mark = self.step_counter
        return spk[: k.value], ev[: k.value]

    # -- readback -----------------------------------------------------------
    def enable_neuron_stats(self, on: bool = True):
        """Start (or stop) per-neuron spike statistics on the device."""
        check(lib().sg_neuron_stats_enable(self._h, 1 if on else 0))

    def neuron_stats(self, pop: int, dt_ms: float):
        """(rates_hz, isi_cv, isi_mean_ms, steps) since the statistics were enabled."""
        n = self._sizes[pop]
        counts = np.empty(n, np.uint32)
        mean = np.empty(n, np.float64)
        cv = np.empty(n, np.float64)
        steps = C.c_uint64()
        check(lib().sg_neuron_stats_read(self._h, pop, _p(counts), _p(mean), _p(cv), C.byref(steps)))
        dur_s = steps.value * dt_ms * 1e-3
        rates = counts / dur_s if dur_s > 0 else np.zeros(n)
        return rates, cv, mean * dt_ms, steps.value

    def spikes(self, pop: int) -> np.ndarray:
        out = np.empty(self._sizes[pop], np.int32)
        check(lib().sg_spikes(self._h, pop, _p(out), out.size))
        return out

    def _u64(self, fn) -> int:
        out = C.c_uint64()
        check(fn(self._h, C.byref(out)))
        return out.value

    @property
    def step_counter(self) -> int:
        return self._u64(lib().sg_step_counter)

    @property
    def total_neurons(self) -> int:
        return self._u64(lib().sg_total_neurons)

    @property
    def num_synapses(self) -> int:
        return self._u64(lib().sg_num_synapses)

    @property
    def events_total(self) -> int:
        return self._u64(lib().sg_events_total)

    @property
    def source_events_total(self) -> int:
        """Events of Poisson-source synapses among events_total."""
        return self._u64(lib().sg_source_events_total)

    @property
    def clamp_hits(self) -> int:
        return self._u64(lib().sg_clamp_hits)

    @property
    def footprint(self) -> int:
        return self._u64(lib().sg_footprint)

    def graph(self):
        n, e = self.total_neurons, self.num_synapses
        rp = np.empty(n + 1, np.uint32)
        c = np.empty(e, np.uint32)
        w = np.empty(e, np.float32)
        d = np.empty(e, np.uint8)
        check(lib().sg_graph_read(self._h, _p(rp), _p(c), _p(w), _p(d)))
        return rp, c, w, d

    def graph_types(self):
        """Per synapse (graph order): synapse type and pair-STDP flag."""
        e = self.num_synapses
        st = np.empty(e, np.uint8)
        pl = np.empty(e, np.uint8)
        check(lib().sg_graph_read_types(self._h, _p(st), _p(pl)))
        return st, pl

    def weights(self) -> np.ndarray:
        w = np.empty(self.num_synapses, np.float32)
        check(lib().sg_weights_read(self._h, _p(w)))
        return w

    def ring(self, ring: int = 0) -> np.ndarray:
        out = np.empty((32, self.total_neurons), np.float32)
        check(lib().sg_ring_read(self._h, ring, _p(out)))
        return out

    @property
    def stdp_drift(self) -> float:
        out = C.c_double()
        check(lib().sg_stdp_drift(self._h, C.byref(out)))
        return out.value

    def stdp_traces(self):
        a = np.empty(self.total_neurons, np.float32)
        b = np.empty(self.total_neurons, np.float32)
        check(lib().sg_stdp_traces(self._h, _p(a), _p(b)))
        return a, b

    # -- dopamine-modulated eligibility learning (P/api/learn/brain.rs) --------
    def enable_learning(self, dt=0.5, tau_pre=20.0, tau_post=20.0, tau_e=1000.0, a_ltp=0.1, a_ltd=0.12, lr=1.0,
                        w_min=0.0, w_max=1.0):
        """Learn on the built network's synapses from this step on (StdpConfig
        defaults, brain.rs:46-60).  Needs FP32 weights."""
        check(lib().sg_learn_enable(self._h, dt, tau_pre, tau_post, tau_e, a_ltp, a_ltd, lr, w_min, w_max))

    def reward(self, dopamine, gate=1.0, w_cap=None, synapses=None):
        """reward / reward_gated / reward_capped (brain.rs:400-416); `synapses`
        = (lo, hi) rewards only that CSR range (one network of a pool)."""
        cap = float("nan") if w_cap is None else w_cap
        if synapses is None:
            check(lib().sg_learn_reward(self._h, dopamine, gate, cap))
        else:
            check(lib().sg_learn_reward_range(self._h, synapses[0], synapses[1], dopamine, gate, cap))

    def clear_eligibility(self, synapses=None):
        if synapses is None:
            check(lib().sg_learn_clear(self._h))
        else:
            check(lib().sg_learn_clear_range(self._h, synapses[0], synapses[1]))

    def population_synapses(self, pop):
        """CSR range (lo, hi) of the synapses whose pre is in `pop`."""
        lo, hi = C.c_uint64(), C.c_uint64()
        check(lib().sg_pop_synapse_range(self._h, pop, C.byref(lo), C.byref(hi)))
        return lo.value, hi.value

    def restrict_eligibility(self, keep):
        k = np.ascontiguousarray(keep, dtype=np.uint8)
        check(lib().sg_learn_restrict(self._h, _p(k), k.size))

    def set_eligibility(self, elig):
        e = np.ascontiguousarray(elig, dtype=np.float32)
        check(lib().sg_learn_set_eligibility(self._h, _p(e), e.size))

    def set_motor(self, left, right):
        """Count the spikes of neurons [left[0], left[1]) and [right[0],
        right[1]) over each step() call."""
        check(lib().sg_learn_motor(self._h, left[0], left[1], right[0], right[1]))

    def motor_counts(self):
        out = np.zeros(2, np.uint32)
        check(lib().sg_learn_motor_read(self._h, _p(out)))
        return int(out[0]), int(out[1])

    def snapshot(self):
        check(lib().sg_learn_snapshot(self._h))

    def recall(self, alpha):
        check(lib().sg_learn_recall(self._h, alpha))

    def learning_state(self):
        """(eligibility [synapses, CSR order], pre traces, post traces, t)."""
        E, N = self.num_synapses, self.total_neurons
        e = np.zeros(max(E, 1), np.float32)
        tp = np.zeros(max(N, 1), np.float32)
        tq = np.zeros(max(N, 1), np.float32)
        t = C.c_uint64()
        check(lib().sg_learn_read(self._h, _p(e), _p(tp), _p(tq), C.byref(t)))
        return e[:E], tp[:N], tq[:N], t.value

    # -- one network split across GPUs -------------------------------------------
    def add_external_population(self, n: int) -> int:
        """Neurons simulated on another GPU: pre-synaptic only here, their
        spikes read each step from a source set by set_external_source."""
        out = C.c_uint32()
        check(lib().sg_pop_add_external(self._h, n, C.byref(out)))
        self._sizes.append(n)
        return out.value

    def set_external_source(self, pop: int, dev_words: int):
        check(lib().sg_pop_set_external_source(self._h, pop, C.c_void_p(dev_words)))

    def spike_words_ptr(self, pop: int) -> int:
        """Device address of this step's spike words of `pop`."""
        out = C.c_void_p()
        check(lib().sg_spike_words(self._h, pop, C.byref(out)))
        return out.value or 0

    def step_begin(self):
        check(lib().sg_step_begin(self._h))

    def step_end(self):
        check(lib().sg_step_end(self._h))

    # -- .taas v2 snapshots ------------------------------------------------------
    def save_taas(self, path, created=None, zstd_level=0):
        """Checkpoint: CSR synapses and weights (and eligibility while learning)."""
        check(lib().sg_taas_save(self._h, str(path).encode(), created.encode() if created is not None else None,
                                 int(zstd_level)))

    def load_weights_taas(self, path):
        """Resume: a snapshot's weights into this built network (same synapses)."""
        check(lib().sg_taas_load_weights(self._h, str(path).encode()))

    def connect_taas(self, from_pop, to_pop, path, default_delay=1):
        """Synapses from a .taas CSR (row i = neuron i of from_pop)."""
        check(lib().sg_connect_taas(self._h, from_pop, to_pop, str(path).encode(), int(default_delay)))

    @property
    def stream(self) -> int:
        out = C.c_void_p()
        check(lib().sg_stream(self._h, C.byref(out)))
        return out.value or 0


class PinnedU32:
    """A page-locked host array of uint32 (sg_host_alloc) for readbacks that
    the device copies into directly; grown on demand, freed by close()."""

    def __init__(self, n: int = 0):
        self._p = C.c_void_p()
        self.n = 0
        self.a = np.empty(0, np.uint32)
        self.ensure(n)

    @property
    def ptr(self):
        return self._p.value

    def ensure(self, n: int) -> np.ndarray:
        n = int(n)
        if n <= self.n:
            return self.a
        self.close()
        p = C.c_void_p()
        check(lib().sg_host_alloc(n * 4, C.byref(p)))
        self._p, self.n = p, n
        self.a = np.ctypeslib.as_array((C.c_uint32 * n).from_address(p.value))
        return self.a

    def close(self):
        if self._p is not None and self._p.value:
            self.a = np.empty(0, np.uint32)
            lib().sg_host_free(self._p)
        self._p = C.c_void_p()
        self.n = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Pool:
    """Networks stepped together (continuous batching): per step one neuron
    launch per model over every member's populations and one scatter launch
    over every member (sg_pool_*).  Members stay independent networks; each
    gives the same bits in the pool as alone."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().sg_pool_create(C.byref(h), device))
        self._h = h
        self.members: list[Network] = []
        self.device = device

    def add(self, net: Network):
        check(lib().sg_pool_add(self._h, net._h))
        self.members.append(net)

    def remove(self, net: Network):
        check(lib().sg_pool_remove(self._h, net._h))
        self.members.remove(net)

    def step(self, n_steps: int):
        check(lib().sg_pool_step(self._h, n_steps))

    def synchronize(self):
        check(lib().sg_pool_synchronize(self._h))

    def __len__(self) -> int:
        out = C.c_uint32()
        check(lib().sg_pool_size(self._h, C.byref(out)))
        return out.value

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().sg_pool_destroy(h)
        self._h = None
        self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
