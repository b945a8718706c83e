"""``SynapticBrain`` — a conductance-based connectome with receptor kinetics
on the GPU, mirroring pillars-connectome's SynapticBrain
(crates/SiMuse/crates/pillars-connectome/src/synaptic.rs:23-130).

Every synapse carries a receptor code (AMPA, NMDA, GABA_A, GABA_B, nAChR,
GluCl, mAChR: P/kernels/synapse/receptor.rs:23-69); a spike jumps the
target's conductance of that receptor at once, and each step

1. decays the seven conductances by fast_exp(-dt / tau_r),
2. computes I_syn = sum over receptors of g_eff (E_rev - V) from the
   pre-step V (NMDA's g scaled by its Mg block),
3. steps the neurons with I_syn + the external current,
4. jumps the conductances of the spiking neurons' targets
   (spiking neurons ascending, each row in order).

It runs as a ``Network`` in receptor mode (sg_set_receptor_kinetics): the
ring's slot 0 takes the external current, slots 1..7 hold the
conductances, the neuron kernel decays them and adds their current, and the
ordered scatter adds each jump to its cell in the reference's order, so the
FP32 results are the reference's bits.
"""
from __future__ import annotations

import numpy as np

from .network import Network

RECEPTORS = ("AMPA", "NMDA", "GABA_A", "GABA_B", "nAChR", "GluCl", "mAChR")
AMPA, NMDA, GABA_A, GABA_B, NACHR, GLUCL, MACHR = range(7)


def receptor_types_from_nt(row_ptr, nt_types, phenotype: str = "mammal") -> np.ndarray:
    """Per-synapse receptor codes from the presynaptic neurons' NT signs
    (build_receptor_types_from_csr, pillars-connectome/src/data.rs:433-463,
    with NtPhenotype::receptor_for_sign, :44-59): nt > 0 gives AMPA (mammal)
    or nAChR (insect), else GABA_A (mammal) or GluCl (insect).  A neuron
    past the end of nt_types counts as +1."""
    rp = np.asarray(row_ptr, np.int64)
    n = rp.size - 1
    nt = np.ones(n, np.float32)
    src = np.asarray(nt_types, np.float32)[:n]
    nt[:src.size] = src
    exc, inh = {"mammal": (AMPA, GABA_A), "insect": (NACHR, GLUCL)}[phenotype]
    per_neuron = np.where(nt > 0.0, exc, inh).astype(np.uint8)
    return np.repeat(per_neuron, np.diff(rp))


def receptor_types_flywire(row_ptr, nt_map) -> np.ndarray:
    """FlyWire NT codes to receptors (build_receptor_types_from_csr_flywire,
    data.rs:465-523): nt > 1.5 GluCl, > 0.5 nAChR, < -1.5 mAChR, else
    GABA_A; a neuron past the end of nt_map counts as +1."""
    rp = np.asarray(row_ptr, np.int64)
    n = rp.size - 1
    nt = np.ones(n, np.float32)
    src = np.asarray(nt_map, np.float32)[:n]
    nt[:src.size] = src
    per_neuron = np.select([nt > 1.5, nt > 0.5, nt < -1.5], [GLUCL, NACHR, MACHR], GABA_A).astype(np.uint8)
    return np.repeat(per_neuron, np.diff(rp))


class SynapticBrain:
    """SynapticBrain<M>::from_sparse_graph(graph, receptor_types, dt) for
    neuron model ``model`` (LIF, IZH, GPEA or HH; state column 0 is V)."""

    def __init__(self, model: int, row_ptr, col, weights, receptor_types, dt: float, device: int = 0,
                 weight_format: int | None = None):
        rp = np.ascontiguousarray(row_ptr, np.uint32)
        n = rp.size - 1
        col = np.ascontiguousarray(col, np.uint32)
        w = np.ascontiguousarray(weights, np.float32)
        rt = np.ascontiguousarray(receptor_types, np.uint8)
        if not (col.size == w.size == rt.size == int(rp[-1])):
            raise ValueError("col, weights and receptor_types must have row_ptr[-1] entries")
        self.n = int(n)
        self.net = Network(device)
        if weight_format is not None:
            self.net.set_weight_format(weight_format)
        self.net.set_receptor_kinetics(dt)
        self.pop = self.net.add_population(model, self.n)
        pre = np.repeat(np.arange(self.n, dtype=np.uint32), np.diff(rp.astype(np.int64)))
        self.net.connect(self.pop, pre, self.pop, col, w, np.ones(w.size, np.uint8), syn_types=rt)
        self._built = False
        self._all = np.arange(self.n, dtype=np.uint32)

    @classmethod
    def from_connectome(cls, model: int, row_ptr, col, weights, dt: float, nt_types=None, receptor_types=None,
                        phenotype: str = "mammal", **kw) -> "SynapticBrain":
        """SynapticBrain::from_connectome (synaptic.rs:36-50): the given
        receptor types, or ones derived from the NT signs."""
        if receptor_types is None or len(receptor_types) == 0:
            receptor_types = receptor_types_from_nt(row_ptr, nt_types if nt_types is not None else [], phenotype)
        return cls(model, row_ptr, col, weights, receptor_types, dt, **kw)

    # -- configuration (NeuralPopulation parameters and state) -----------------
    def configure(self, fn):
        """fn(brain) sets parameters and state through fill_param /
        set_param / fill_state / set_state (SynapticBrain::configure)."""
        fn(self)

    def fill_param(self, col: int, value: float):
        self.net.fill_param(self.pop, col, value)

    def set_param(self, col: int, values):
        self.net.set_param(self.pop, col, values)

    def fill_state(self, col: int, value: float):
        self.net.fill_state(self.pop, col, value)

    def set_state(self, col: int, values):
        self.net.set_state(self.pop, col, values)

    def _ensure_built(self):
        if not self._built:
            self.net.build()
            self._built = True

    # -- stepping -------------------------------------------------------------------
    def step(self, external_i=None) -> np.ndarray:
        """One step with per-neuron input current ``external_i`` (missing
        entries are 0); returns the spike mask (int32, 0/1)."""
        self._ensure_built()
        if external_i is not None:
            x = np.ascontiguousarray(external_i, np.float32)[: self.n]
            if x.size:
                self.net.inject_current(self.pop, self._all[: x.size], x)
        self.net.step(1)
        return self.net.spikes(self.pop).astype(np.int32)

    def run(self, n_steps: int):
        """n_steps steps without external input (one launch sequence)."""
        self._ensure_built()
        self.net.step(n_steps)

    def kinetics(self) -> np.ndarray:
        """The conductances, [receptor code][neuron] (SynapticBrain::kinetics)."""
        self._ensure_built()
        return self.net.receptor_conductances()

    def set_kinetics(self, g):
        self._ensure_built()
        self.net.set_receptor_conductances(g)

    def state(self, col: int) -> np.ndarray:
        return self.net.state(self.pop, col)

    def __len__(self) -> int:
        return self.n

    def is_empty(self) -> bool:
        return self.n == 0

    def close(self):
        if getattr(self, "net", None) is not None:
            self.net.close()
            self.net = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
