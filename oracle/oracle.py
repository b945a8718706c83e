"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is a C++ restatement of the reference's CPU simulation step
(crates/SiMuse/crates/pillars/src/api/net/network/step.rs and the modules it
calls).  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
use this module; the product never imports it.

The class mirrors the reference's ``Network`` builder/step API
(P/api/net/network/core.rs:87-622, build.rs:18-276) with numpy arrays in
place of slices, and raises ``OracleError`` where the reference panics.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_simuse.so")

LIF, IZH, GPEA, HH = 1, 2, 3, 4


class OracleError(RuntimeError):
    pass


def build_oracle() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build_oracle()
        L = C.CDLL(_LIB_PATH)
        vp, i32, u32, u64, f32, f64 = C.c_void_p, C.c_int, C.c_uint32, C.c_uint64, C.c_float, C.c_double
        P = C.POINTER
        sig = {
            "or_net_new": (vp, [i32]),
            "or_net_free": (None, [vp]),
            "or_last_error": (C.c_char_p, []),
            "or_set_threads": (i32, [i32]),
            "or_pop_add": (i32, [vp, i32, u32]),
            "or_pop_fill_param": (i32, [vp, i32, i32, f64]),
            "or_pop_fill_state": (i32, [vp, i32, i32, f64]),
            "or_pop_set_param": (i32, [vp, i32, i32, vp, u32]),
            "or_pop_set_state": (i32, [vp, i32, i32, vp, u32]),
            "or_pop_get_state": (i32, [vp, i32, i32, vp, u32]),
            "or_pop_get_state_f64": (i32, [vp, i32, i32, vp, u32]),
            "or_pop_get_param": (i32, [vp, i32, i32, vp, u32]),
            "or_connect": (i32, [vp, i32, vp, i32, vp, vp, vp, vp, vp, u64, u32]),
            "or_register_plasticity": (i32, [vp, f32, f32, i32, f32, f32]),
            "or_tm_sequence": (i32, [f32, f32, f32, i32, f32, vp, u32, vp]),
            "or_register_expone": (i32, [vp, f32, f32, f32]),
            "or_register_kinetics": (i32, [vp, i32, vp, f32, f32]),
            "or_set_receptor_kinetics": (i32, [vp, f32]),
            "or_receptor_read": (i32, [vp, vp]),
            "or_receptor_write": (i32, [vp, vp]),
            "or_receptor_factors": (i32, [f32, vp]),
            "or_receptor_currents": (i32, [u32, vp, vp, vp]),
            "or_nmda_mg_block": (f32, [f32]),
            "or_pop_add_external": (i32, [vp, u32]),
            "or_step_begin": (i32, [vp]),
            "or_set_external_spikes": (i32, [vp, i32, vp, u32]),
            "or_step_end": (i32, [vp]),
            "or_learn_enable": (i32, [vp, f32, f32, f32, f32, f32, f32, f32, f32, f32]),
            "or_learn_reward": (i32, [vp, f32, f32, f32]),
            "or_learn_clear": (i32, [vp]),
            "or_learn_reward_range": (i32, [vp, u64, u64, f32, f32, f32]),
            "or_learn_clear_range": (i32, [vp, u64, u64]),
            "or_pop_synapse_range": (i32, [vp, i32, vp, vp]),
            "or_learn_restrict": (i32, [vp, vp, u64]),
            "or_learn_set_eligibility": (i32, [vp, vp, u64]),
            "or_learn_motor": (i32, [vp, u64, u64, u64, u64]),
            "or_learn_motor_read": (i32, [vp, vp]),
            "or_learn_snapshot": (i32, [vp]),
            "or_learn_recall": (i32, [vp, f32]),
            "or_learn_read": (i32, [vp, vp, vp, vp, vp]),
            "or_poisson_add": (i32, [vp, f32, f32, u32]),
            "or_poisson_connect": (i32, [vp, i32, i32, vp, vp, vp, vp, u64]),
            "or_poisson_connect_plastic": (i32, [vp, i32, i32, vp, vp, vp, vp, vp, u64]),
            "or_poisson_add_many": (i32, [vp, u32, f32, f32, u32]),
            "or_poisson_connect_one_to_one": (i32, [vp, i32, u32, i32, f32, C.c_uint8]),
            "or_stdp_config": (i32, [vp, f32, f32, f32, f32, f32, f32, f32]),
            "or_build": (i32, [vp]),
            "or_build_fixed_indegree": (i32, [vp, i32, i32, u32, u64, u32, f32, f32, u32, u32]),
            "or_build_from_csr": (i32, [vp, vp, vp, vp, vp]),
            "or_inject": (i32, [vp, i32, vp, vp, u64]),
            "or_step": (i32, [vp, u32, vp]),
            "or_spikes": (i32, [vp, i32, vp, u32]),
            "or_step_counter": (u64, [vp]),
            "or_total_neurons": (u64, [vp]),
            "or_num_synapses": (u64, [vp]),
            "or_events": (u64, [vp]),
            "or_ring_read": (i32, [vp, i32, vp]),
            "or_graph_read": (i32, [vp, vp, vp, vp, vp]),
            "or_weights_read": (i32, [vp, vp]),
            "or_weights_write": (i32, [vp, vp, u64]),
            "or_stdp_drift": (f64, [vp]),
            "or_traces_read": (i32, [vp, vp, vp]),
            "or_fast_exp": (f32, [f32]),
            "or_sg_expf": (f32, [f32]),
            "or_sg_logf": (f32, [f32]),
            "or_poisson_spike": (i32, [u32, u32, u64, f32]),
            "or_compact": (u64, [vp, u64, vp]),
            "or_push_spikes": (i32, [vp, vp, vp, vp, u32, vp, u32, u64, vp]),
            "or_kuramoto_rk4": (i32, [i32, u32, vp, vp, f32, f32, u32, vp, vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def _chk(rc):
    if rc < 0:
        raise OracleError(lib().or_last_error().decode())
    return rc


def set_threads(n: int) -> int:
    return lib().or_set_threads(int(n))


class Network:
    """CPU restatement of ``pillars::api::Network`` (FP32, or the FP64 twin)."""

    def __init__(self, precision: int = 0):
        self._h = lib().or_net_new(precision)
        self.precision = precision
        self._sizes: list[int] = []

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().or_net_free(h)
            self._h = None

    # -- builder -----------------------------------------------------------
    def add_population(self, model: int, n: int) -> int:
        pid = _chk(lib().or_pop_add(self._h, model, n))
        self._sizes.append(n)
        return pid

    def fill_param(self, pop, col, v):
        _chk(lib().or_pop_fill_param(self._h, pop, col, float(v)))

    def fill_state(self, pop, col, v):
        _chk(lib().or_pop_fill_state(self._h, pop, col, float(v)))

    def set_param(self, pop, col, vals):
        a = np.ascontiguousarray(vals, dtype=np.float32)
        _chk(lib().or_pop_set_param(self._h, pop, col, _p(a), a.size))

    def set_state(self, pop, col, vals):
        a = np.ascontiguousarray(vals, dtype=np.float32)
        _chk(lib().or_pop_set_state(self._h, pop, col, _p(a), a.size))

    def state(self, pop, col):
        out = np.empty(self._sizes[pop], np.float32)
        _chk(lib().or_pop_get_state(self._h, pop, col, _p(out), out.size))
        return out

    def state_f64(self, pop, col):
        out = np.empty(self._sizes[pop], np.float64)
        _chk(lib().or_pop_get_state_f64(self._h, pop, col, _p(out), out.size))
        return out

    def param(self, pop, col):
        out = np.empty(self._sizes[pop], np.float32)
        _chk(lib().or_pop_get_param(self._h, pop, col, _p(out), out.size))
        return out

    def connect(self, frm, from_idx, to, to_idx, weights, delays, syn_types=None, stdp=False, plast_types=None):
        fi = np.ascontiguousarray(from_idx, np.uint32)
        ti = np.ascontiguousarray(to_idx, np.uint32)
        w = np.ascontiguousarray(weights, np.float32)
        d = np.ascontiguousarray(delays, np.uint8)
        st = None if syn_types is None else np.ascontiguousarray(syn_types, np.uint8)
        pt = None if plast_types is None else np.ascontiguousarray(plast_types, np.uint8)
        if not (fi.size == ti.size == w.size == d.size) or (st is not None and st.size != fi.size) \
                or (pt is not None and pt.size != fi.size):
            raise OracleError("connect: slice length mismatch")
        _chk(lib().or_connect(self._h, frm, _p(fi), to, _p(ti), _p(w), _p(d), _p(st), _p(pt), fi.size,
                              1 if stdp else 0))

    def register_plasticity(self, u0, tau_rec, dt, tau_fac=None) -> int:
        """Tsodyks-Markram profile (depression, or depression + facilitation
        when tau_fac is given); returns its 1-based id."""
        return _chk(lib().or_register_plasticity(self._h, u0, tau_rec, 0 if tau_fac is None else 1,
                                                 0.0 if tau_fac is None else tau_fac, dt))

    def register_expone(self, tau_decay, erev, dt) -> int:
        return _chk(lib().or_register_expone(self._h, tau_decay, erev, dt))

    def set_receptor_kinetics(self, dt):
        """SynapticBrain receptor kinetics: syn_types are receptor codes."""
        _chk(lib().or_set_receptor_kinetics(self._h, dt))

    def receptor_conductances(self) -> np.ndarray:
        out = np.empty((7, self.total_neurons), np.float32)
        _chk(lib().or_receptor_read(self._h, _p(out)))
        return out

    def set_receptor_conductances(self, g):
        g = np.ascontiguousarray(g, np.float32)
        if g.shape != (7, self.total_neurons):
            raise ValueError("conductances must be [7][total neurons]")
        _chk(lib().or_receptor_write(self._h, _p(g)))

    def add_external_population(self, n):
        pid = _chk(lib().or_pop_add_external(self._h, n))
        self._sizes.append(n)
        return pid

    def step_begin(self):
        _chk(lib().or_step_begin(self._h))

    def set_external_spikes(self, pop, spikes):
        s = np.ascontiguousarray(spikes, dtype=np.int32)
        _chk(lib().or_set_external_spikes(self._h, pop, _p(s), s.size))

    def step_end(self):
        _chk(lib().or_step_end(self._h))

    def enable_learning(self, dt=0.5, tau_pre=20.0, tau_post=20.0, tau_e=1000.0, a_ltp=0.1, a_ltd=0.12, lr=1.0,
                        w_min=0.0, w_max=1.0):
        _chk(lib().or_learn_enable(self._h, dt, tau_pre, tau_post, tau_e, a_ltp, a_ltd, lr, w_min, w_max))

    def reward(self, dopamine, gate=1.0, w_cap=None, synapses=None):
        cap = float("nan") if w_cap is None else w_cap
        if synapses is None:
            _chk(lib().or_learn_reward(self._h, dopamine, gate, cap))
        else:
            _chk(lib().or_learn_reward_range(self._h, synapses[0], synapses[1], dopamine, gate, cap))

    def clear_eligibility(self, synapses=None):
        if synapses is None:
            _chk(lib().or_learn_clear(self._h))
        else:
            _chk(lib().or_learn_clear_range(self._h, synapses[0], synapses[1]))

    def population_synapses(self, pop):
        lo, hi = C.c_uint64(), C.c_uint64()
        _chk(lib().or_pop_synapse_range(self._h, pop, C.byref(lo), C.byref(hi)))
        return lo.value, hi.value

    def restrict_eligibility(self, keep):
        k = np.ascontiguousarray(keep, dtype=np.uint8)
        _chk(lib().or_learn_restrict(self._h, _p(k), k.size))

    def set_eligibility(self, elig):
        e = np.ascontiguousarray(elig, dtype=np.float32)
        _chk(lib().or_learn_set_eligibility(self._h, _p(e), e.size))

    def set_motor(self, left, right):
        _chk(lib().or_learn_motor(self._h, left[0], left[1], right[0], right[1]))

    def motor_counts(self):
        out = np.zeros(2, np.uint32)
        _chk(lib().or_learn_motor_read(self._h, _p(out)))
        return int(out[0]), int(out[1])

    def snapshot(self):
        _chk(lib().or_learn_snapshot(self._h))

    def recall(self, alpha):
        _chk(lib().or_learn_recall(self._h, alpha))

    def learning_state(self):
        """(eligibility [CSR order], pre traces, post traces, t)."""
        E, N = self.num_synapses, self.total_neurons
        e = np.zeros(max(E, 1), np.float32)
        tp = np.zeros(max(N, 1), np.float32)
        tq = np.zeros(max(N, 1), np.float32)
        t = C.c_uint64()
        _chk(lib().or_learn_read(self._h, _p(e), _p(tp), _p(tq), C.byref(t)))
        return e[:E], tp[:N], tq[:N], t.value

    def register_kinetics(self, kind, params, erev, dt) -> int:
        """kind 0 ExpOne, 1 ExpTwo, 2 Alpha, 3 ExpThree (params as in the C API)."""
        p = np.zeros(5, np.float32)
        p[:len(params)] = params
        return _chk(lib().or_register_kinetics(self._h, int(kind), _p(p), erev, dt))

    def add_poisson_source(self, rate_hz, dt_ms, seed) -> int:
        return _chk(lib().or_poisson_add(self._h, rate_hz, dt_ms, seed))

    def add_poisson_sources(self, n, rate_hz, dt_ms, seeds=None, seed0=0) -> int:
        if seeds is not None:
            first = None
            for s in np.asarray(seeds, np.uint32):
                i = self.add_poisson_source(rate_hz, dt_ms, int(s))
                first = i if first is None else first
            return first
        return _chk(lib().or_poisson_add_many(self._h, n, rate_hz, dt_ms, seed0))

    def connect_poisson_one_to_one(self, first_src, n, to, weight, delay, posts=None):
        if posts is not None:
            for i, q in enumerate(np.asarray(posts, np.uint32)):
                self.connect_poisson_source(first_src + i, to, [q], [weight], [delay])
            return
        _chk(lib().or_poisson_connect_one_to_one(self._h, first_src, n, to, weight, delay))

    def connect_poisson_source(self, src, to, posts, weights, delays, syn_types=None, plast_types=None):
        p = np.ascontiguousarray(posts, np.uint32)
        w = np.ascontiguousarray(weights, np.float32)
        d = np.ascontiguousarray(delays, np.uint8)
        st = None if syn_types is None else np.ascontiguousarray(syn_types, np.uint8)
        pt = None if plast_types is None else np.ascontiguousarray(plast_types, np.uint8)
        _chk(lib().or_poisson_connect_plastic(self._h, src, to, _p(p), _p(w), _p(d), _p(st), _p(pt), p.size))

    def stdp_config(self, dt, tau_pre, tau_post, a_plus, a_minus, w_min, w_max):
        _chk(lib().or_stdp_config(self._h, dt, tau_pre, tau_post, a_plus, a_minus, w_min, w_max))

    def build(self):
        _chk(lib().or_build(self._h))

    def build_fixed_indegree(self, frm, to, k_in, seed, n_exc, w_exc, w_inh, d_min, d_max):
        """Fixed in-degree projection + build in one pass (see simuse_oracle.h)."""
        _chk(lib().or_build_fixed_indegree(self._h, frm, to, k_in, seed, n_exc, w_exc, w_inh, d_min, d_max))

    def build_from_csr(self, row_ptr, col, w, d):
        rp = np.ascontiguousarray(row_ptr, np.uint32)
        c = np.ascontiguousarray(col, np.uint32)
        ww = np.ascontiguousarray(w, np.float32)
        dd = np.ascontiguousarray(d, np.uint8)
        _chk(lib().or_build_from_csr(self._h, _p(rp), _p(c), _p(ww), _p(dd)))

    # -- run ---------------------------------------------------------------
    def inject_current(self, pop, idx, vals):
        i = np.ascontiguousarray(idx, np.uint32)
        v = np.ascontiguousarray(vals, np.float32)
        if i.size != v.size:
            raise OracleError("inject_current: indices/values length mismatch")
        _chk(lib().or_inject(self._h, pop, _p(i), _p(v), i.size))

    def step(self, n_steps: int = 1, record: bool = False):
        if record:
            r = np.zeros((n_steps, self.total_neurons), np.uint8)
            _chk(lib().or_step(self._h, n_steps, _p(r)))
            return r
        _chk(lib().or_step(self._h, n_steps, None))
        return None

    def spikes(self, pop):
        out = np.empty(self._sizes[pop], np.int32)
        _chk(lib().or_spikes(self._h, pop, _p(out), out.size))
        return out

    @property
    def step_counter(self) -> int:
        return int(lib().or_step_counter(self._h))

    @property
    def total_neurons(self) -> int:
        return int(lib().or_total_neurons(self._h))

    @property
    def num_synapses(self) -> int:
        return int(lib().or_num_synapses(self._h))

    @property
    def events(self) -> int:
        return int(lib().or_events(self._h))

    def ring(self, ring: int = 0):
        out = np.empty((32, self.total_neurons), np.float32)
        _chk(lib().or_ring_read(self._h, ring, _p(out)))
        return out

    def graph(self):
        n, e = self.total_neurons, self.num_synapses
        rp = np.empty(n + 1, np.uint32)
        c = np.empty(e, np.uint32)
        w = np.empty(e, np.float32)
        d = np.empty(e, np.uint8)
        _chk(lib().or_graph_read(self._h, _p(rp), _p(c), _p(w), _p(d)))
        return rp, c, w, d

    def weights(self):
        w = np.empty(self.num_synapses, np.float32)
        _chk(lib().or_weights_read(self._h, _p(w)))
        return w

    def set_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        _chk(lib().or_weights_write(self._h, _p(w), w.size))

    @property
    def stdp_drift(self) -> float:
        return float(lib().or_stdp_drift(self._h))

    def traces(self):
        a = np.empty(self.total_neurons, np.float32)
        b = np.empty(self.total_neurons, np.float32)
        _chk(lib().or_traces_read(self._h, _p(a), _p(b)))
        return a, b


def tm_sequence(u0, a_rec, a_fac, facilitation, steps, w=1.0) -> np.ndarray:
    """Delivered weights of one Tsodyks-Markram synapse spiking at `steps`."""
    st = np.ascontiguousarray(steps, np.uint64)
    out = np.zeros(st.size, np.float32)
    _chk(lib().or_tm_sequence(u0, a_rec, a_fac, 1 if facilitation else 0, w, _p(st), st.size, _p(out)))
    return out


def fast_exp(x: float) -> float:
    return float(lib().or_fast_exp(float(x)))


def sg_expf(x: float) -> float:
    return float(lib().or_sg_expf(float(x)))


def sg_logf(x: float) -> float:
    return float(lib().or_sg_logf(float(x)))


def receptor_factors(dt: float) -> np.ndarray:
    out = np.empty(7, np.float32)
    _chk(lib().or_receptor_factors(dt, _p(out)))
    return out


def receptor_currents(g, v) -> np.ndarray:
    g = np.ascontiguousarray(g, np.float32)
    v = np.ascontiguousarray(v, np.float32)
    out = np.empty(v.size, np.float32)
    _chk(lib().or_receptor_currents(v.size, _p(g), _p(v), _p(out)))
    return out


def nmda_mg_block(v: float) -> float:
    return lib().or_nmda_mg_block(v)


def poisson_spike(seed, stream, step, p) -> bool:
    return bool(lib().or_poisson_spike(seed, stream, step, p))


def compact(spikes) -> np.ndarray:
    s = np.ascontiguousarray(spikes, np.int32)
    out = np.empty(s.size, np.uint32)
    k = lib().or_compact(_p(s), s.size, _p(out))
    return out[:k]


def push_spikes(row_ptr, col, w, d, n_neurons, active, step, ring):
    """push_spikes on plain arrays; `ring` ([32][n] float32) is updated in place."""
    rp = np.ascontiguousarray(row_ptr, np.uint32)
    c = np.ascontiguousarray(col, np.uint32)
    ww = np.ascontiguousarray(w, np.float32)
    dd = np.ascontiguousarray(d, np.uint8)
    a = np.ascontiguousarray(active, np.uint32)
    assert ring.dtype == np.float32 and ring.flags.c_contiguous
    _chk(lib().or_push_spikes(_p(rp), _p(c), _p(ww), _p(dd), n_neurons, _p(a), a.size, step, _p(ring)))
    return ring


def kuramoto_rk4(theta0, omega, k, dt, n_steps, precision=1):
    th = np.ascontiguousarray(theta0, np.float32)
    om = np.ascontiguousarray(omega, np.float32)
    out = np.empty_like(th)
    r = np.empty(n_steps, np.float64)
    _chk(lib().or_kuramoto_rk4(precision, th.size, _p(th), _p(om), k, dt, n_steps, _p(out), _p(r)))
    return out, r
