"""``BrainRunner`` — the connectome runner of pillars-connectome on the GPU.

Mirrors ``BrainRunner`` of crates/SiMuse/crates/pillars-connectome/src/
runner.rs for the current-based LIF and Izhikevich configurations
(``NeuronConfig::Lif`` / ``::Izh``, runner.rs:114-248, :588-724, :798-937,
:1342-1440): the same constructor checks and error strings, the same initial
state (types.rs:116-144), the same ``run(n_steps, external_I)`` returning a
flat ``[n_steps * n_neurons]`` 0/1 raster, the same grow-only spike buffer
behind ``firing_rates``, and ``get_v/set_v/get_u/set_u``, ``reset``,
``step_counter``, ``add_poisson_group``.

What ``run`` computes, per the reference: the connectome's weights signed by
the presynaptic ``nt_types`` (runner.rs:1455-1478), every synapse with delay
0 (brain.rs:16-28, delivered on the next step), ``external_I`` (zeros past
its end) plus the Poisson-group currents injected into the same step's input
(inject_current), v / u / refractory carried from call to call.  The
reference rebuilds its ``Brain`` (an ``api::Network``) on every ``run``; here
the network is built once and stays in HBM, and each ``run`` starts from
empty delay rings, which is what the rebuilt network starts from, so the
spikes are the same.  A constant ``external_I`` is applied as a device bias
(the same float add as the injection); Poisson groups are drawn on the host
each step.  The reference draws them from ``StdRng`` (ChaCha12, seed 0),
which no reference test pins: with Poisson groups only the statistics match.

The conductance configurations ``NeuronConfig::LifSynaptic`` / ``::IzhSynaptic``
(runner.rs:124-131, :156-163; run at :1365-1401 and :1695-1735) run the same
neurons through ``SynapticBrain`` (receptor kinetics, pillars-connectome/src/
synaptic.rs): the connectome's unsigned weights, its receptor types (or
types from the presynaptic NT signs and the phenotype, data.rs:433-463), no
delays, the conductances carried from one ``run`` to the next
(``set_kinetics`` of the last run's ``kinetics``) and cleared by ``reset``.
Here the network is built once in receptor mode and its conductances stay in
HBM between calls, which is that carry-over.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .network import IZH, LIF, Network
from .synaptic import receptor_types_from_nt


@dataclasses.dataclass
class ConnectomeData:
    """The CSR connectome of pillars-connectome data.rs:80-103 (the fields
    the current-based runner uses)."""
    row_ptr: np.ndarray          # i32 [n_neurons + 1]
    col_indices: np.ndarray      # i32 [n_synapses]
    values: np.ndarray           # f32 [n_synapses]
    nt_types: np.ndarray | None = None   # f32 [n_neurons], < 0 = inhibitory presynapse
    receptor_types: np.ndarray | None = None   # u8 [n_synapses] receptor codes (conductance configs)
    phenotype: str = "mammal"            # NtPhenotype for types derived from nt_types

    @property
    def n_neurons(self) -> int:
        return max(len(self.row_ptr) - 1, 0)


@dataclasses.dataclass
class NeuronConfig:
    """``NeuronConfig::Lif``, ``::Izh``, ``::LifSynaptic`` or ``::IzhSynaptic``
    (runner.rs:114-248)."""
    model: str                   # "lif", "izh", "lif_synaptic" or "izh_synaptic"
    dt_ms: float
    tau_ref: float
    tau_m: float = 20.0
    v_rest: float = -70.0
    v_thresh: float = -58.0
    v_reset: float = -70.0
    a: float = 0.02
    b: float = 0.2
    c: float = -65.0
    d: float = 8.0


def lif(dt_ms: float) -> NeuronConfig:
    """BrainConfig::lif (runner.rs:251-264)."""
    return NeuronConfig("lif", dt_ms, tau_ref=2.0, tau_m=20.0, v_rest=-70.0, v_thresh=-58.0, v_reset=-70.0)


def izh(dt_ms: float) -> NeuronConfig:
    """BrainConfig::izh (runner.rs:295-306)."""
    return NeuronConfig("izh", dt_ms, tau_ref=2.0, a=0.02, b=0.2, c=-65.0, d=8.0)


def lif_synaptic(dt_ms: float) -> NeuronConfig:
    """BrainConfig::lif_synaptic (runner.rs:265-275)."""
    return NeuronConfig("lif_synaptic", dt_ms, tau_ref=2.0, tau_m=20.0, v_rest=-70.0, v_thresh=-58.0, v_reset=-70.0)


def izh_synaptic(dt_ms: float) -> NeuronConfig:
    """NeuronConfig::IzhSynaptic with BrainConfig::izh's parameters."""
    return NeuronConfig("izh_synaptic", dt_ms, tau_ref=2.0, a=0.02, b=0.2, c=-65.0, d=8.0)


@dataclasses.dataclass
class PoissonGroup:
    indices: np.ndarray
    rate_hz: float
    weight: float


class BrainRunner:
    """See the module text."""

    def __init__(self, connectome: ConnectomeData, config: NeuronConfig, device: int = 0, seed: int = 0):
        n = connectome.n_neurons
        if n == 0:
            raise ValueError("BrainRunner: connectome has 0 neurons")
        rp = np.asarray(connectome.row_ptr)
        if len(rp) != n + 1:
            raise ValueError(f"BrainRunner: row_ptr length {len(rp)} != n_neurons + 1 ({n + 1})")
        if len(connectome.col_indices) != len(connectome.values):
            raise ValueError(f"BrainRunner: col_indices length {len(connectome.col_indices)} != values "
                             f"length {len(connectome.values)}")
        if config.model not in ("lif", "izh", "lif_synaptic", "izh_synaptic"):
            raise ValueError(f"unsupported neuron model {config.model!r}")
        self._synaptic = config.model.endswith("_synaptic")
        self.config, self.connectome, self.n_neurons = config, connectome, n
        self.poisson_groups: list[PoissonGroup] = []
        self._rng = np.random.default_rng(seed)
        self._step_counter = 0
        self.spike_buffer = np.zeros(n * 64, np.int32)   # runner.rs:700-717
        self._bias: np.ndarray | None = None
        # the signed connectome (runner.rs:1455-1478): weights times the sign
        # of the presynaptic nt_type, every synapse with delay 0
        rp32 = np.maximum(rp, 0).astype(np.uint32)
        col = np.maximum(np.asarray(connectome.col_indices), 0).astype(np.uint32)
        w = np.asarray(connectome.values, np.float32).copy()
        nt = np.ones(n, np.float32) if connectome.nt_types is None else np.asarray(connectome.nt_types, np.float32)
        sign = np.ones(n, np.float32)
        sign[:min(n, nt.size)] = np.where(nt[:n] < 0.0, np.float32(-1.0), np.float32(1.0))
        w *= np.repeat(sign, np.diff(rp32).astype(np.int64))
        self._net = Network(device)
        self._model = LIF if config.model.startswith("lif") else IZH
        if self._synaptic:
            self._net.set_receptor_kinetics(config.dt_ms)
        self._pop = self._net.add_population(self._model, n)
        c = config
        if self._model == LIF:
            inv_tau = np.float32(1.0) / np.float32(max(c.tau_m, 1e-6))   # f32 divide, as the reference
            cols = [c.dt_ms, inv_tau, c.v_rest, c.v_thresh, c.v_reset, c.tau_ref]
        else:
            cols = [c.dt_ms, c.a, c.b, c.c, c.d, c.tau_ref, 30.0]
        for k, v in enumerate(cols):
            self._net.fill_param(self._pop, k, float(np.float32(v)))
        if self._synaptic:
            # SynapticBrain::from_connectome (synaptic.rs:36-50): unsigned
            # weights, the given receptor types or ones from the NT signs
            rt = connectome.receptor_types
            if rt is None or len(rt) == 0:
                rt = receptor_types_from_nt(rp32, [] if connectome.nt_types is None else connectome.nt_types,
                                            connectome.phenotype)
            pre = np.repeat(np.arange(n, dtype=np.uint32), np.diff(rp32.astype(np.int64)))
            self._net.connect(self._pop, pre, self._pop, col, np.asarray(connectome.values, np.float32),
                              np.ones(col.size, np.uint8), syn_types=np.asarray(rt, np.uint8))
            self._net.build()
        else:
            self._net.build_from_csr(rp32, col, w, np.zeros(col.size, np.uint8))
        self._set_initial_state()

    def _set_initial_state(self):
        n = self.n_neurons
        if self._model == LIF:      # BrainState::new (types.rs:116-144)
            self._net.set_state(self._pop, 0, np.full(n, -58.0, np.float32))
            self._net.set_state(self._pop, 1, np.zeros(n, np.float32))
        else:
            self._net.set_state(self._pop, 0, np.full(n, -65.0, np.float32))
            self._net.set_state(self._pop, 1, np.full(n, -13.0, np.float32))
            self._net.set_state(self._pop, 2, np.zeros(n, np.float32))

    # -- run ----------------------------------------------------------------------
    def run(self, n_steps: int, external_I=()) -> np.ndarray:
        """n_steps steps; returns the [n_steps * n_neurons] 0/1 spike raster
        (a view of the spike buffer, valid until the next call)."""
        n = self.n_neurons
        needed = n_steps * n
        if self.spike_buffer.size < needed:
            grown = np.zeros(needed, np.int32)
            grown[:self.spike_buffer.size] = self.spike_buffer
            self.spike_buffer = grown
        self.spike_buffer[:needed] = 0
        ext = np.zeros(n, np.float32)
        e = np.asarray(external_I, np.float32).ravel()[:n]
        ext[:e.size] = e
        net = self._net
        if not self._synaptic:
            net.clear_rings()             # the rebuilt Brain starts with empty rings
        # (the conductance configurations carry their kinetics over instead)
        if n_steps == 0:
            return self.spike_buffer[:0]
        net.enable_raster(n_steps)
        if not self.poisson_groups:
            if self._bias is None or not np.array_equal(self._bias, ext):
                net.set_bias(self._pop, ext)    # added every step, zeros included, as the reference injects
                self._bias = ext.copy()
            net.step(n_steps)
        else:
            if self._bias is not None:
                net.set_bias(self._pop, np.empty(0, np.float32))
                self._bias = None
            idx = np.arange(n, dtype=np.uint32)
            for _ in range(n_steps):
                work = np.zeros(n, np.float32)
                for g in self.poisson_groups:   # inject_poisson_into, runner.rs:416-447
                    if g.rate_hz <= 0.0 or g.weight == 0.0:
                        continue
                    p = g.rate_hz * self.config.dt_ms / 1000.0
                    if p <= 0.0:
                        continue
                    sel = g.indices[g.indices < n]
                    if p >= 1.0:
                        np.add.at(work, sel, np.float32(g.weight))
                    else:
                        hit = sel[self._rng.random(sel.size, dtype=np.float32) < p]
                        np.add.at(work, hit, np.float32(g.weight))
                net.inject_current(self._pop, idx, ext + work)
                net.step(1)
        raster = net.read_raster()        # [n_steps][n] uint8
        self.spike_buffer[:needed] = raster.reshape(-1)[:needed]
        self._step_counter += n_steps
        return self.spike_buffer[:needed]

    def run_count(self, n_steps: int, external_I=()):
        """(total spikes, neurons that fired at least once) over n_steps."""
        r = self.run(n_steps, external_I).reshape(n_steps, self.n_neurons)
        return int(r.sum()), r.any(axis=0)

    # -- readouts and state ---------------------------------------------------------
    def firing_rates(self, dt_ms: float) -> np.ndarray:
        """Counts over the whole spike buffer / its duration (runner.rs:1002-1021)."""
        n = self.n_neurons
        n_steps = self.spike_buffer.size // n
        duration_s = np.float32(n_steps) * np.float32(dt_ms) / np.float32(1000.0)
        if duration_s <= 0.0:
            return np.zeros(n, np.float32)
        counts = (self.spike_buffer[:n_steps * n].reshape(n_steps, n) != 0).sum(axis=0).astype(np.float32)
        return counts / duration_s

    def firing_rates_group(self, indices, n_steps: int, dt_ms: float) -> np.ndarray:
        duration_s = np.float32(n_steps) * np.float32(dt_ms) / np.float32(1000.0)
        idx = np.asarray(indices, np.int64)
        if duration_s <= 0.0:
            return np.zeros(idx.size, np.float32)
        r = self.spike_buffer[:n_steps * self.n_neurons].reshape(n_steps, self.n_neurons)
        return (r[:, idx] != 0).sum(axis=0).astype(np.float32) / duration_s

    def get_v(self) -> np.ndarray:
        return self._net.state(self._pop, 0)

    def set_v(self, v):
        cur = self.get_v()
        a = np.asarray(v, np.float32).ravel()[:self.n_neurons]
        cur[:a.size] = a
        self._net.set_state(self._pop, 0, cur)

    def get_u(self) -> np.ndarray:
        if self._model != IZH:
            return np.zeros(self.n_neurons, np.float32)
        return self._net.state(self._pop, 1)

    def set_u(self, u):
        if self._model != IZH:
            return
        cur = self.get_u()
        a = np.asarray(u, np.float32).ravel()[:self.n_neurons]
        cur[:a.size] = a
        self._net.set_state(self._pop, 1, cur)

    def add_poisson_group(self, indices, rate_hz: float, weight: float):
        self.poisson_groups.append(PoissonGroup(np.asarray(indices, np.int64), float(rate_hz), float(weight)))

    def clear_poisson_groups(self):
        self.poisson_groups.clear()

    def spike_buffer_view(self) -> np.ndarray:
        return self.spike_buffer

    def step_counter(self) -> int:
        return self._step_counter

    def reset(self):
        """State back to BrainState::new plus reset_with_noise (types.rs:166-171)."""
        self._set_initial_state()
        v = self.get_v()
        i = np.arange(self.n_neurons, dtype=np.float32)
        noise = ((i * np.float32(0.577)) % np.float32(1.0) - np.float32(0.5)) * np.float32(2.0)
        self._net.set_state(self._pop, 0, (v + noise * np.float32(0.03)).astype(np.float32))
        self.spike_buffer[:] = 0
        self._step_counter = 0
        if self._synaptic:               # SynapticKinetics::reset (runner.rs:1272-1274)
            self._net.set_receptor_conductances(np.zeros((7, self.n_neurons), np.float32))

    def kinetics(self) -> np.ndarray | None:
        """The carried conductances [7][n] of a conductance configuration."""
        return self._net.receptor_conductances() if self._synaptic else None

    def close(self):
        self._net.close()
