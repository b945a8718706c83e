"""``Sweep`` — an uneven parameter sweep of Kuramoto populations and
Izhikevich pulse networks advancing together on one GPU.

Kuramoto half: a ``KuramotoBatch``.  Each instance runs on one CTA (up to
4096 oscillators) or one thread-block cluster of 2-8 CTAs (up to 65,536) for
all of a run's steps, phases and RK4 sums in registers, so a run of any
length is one persistent launch per shape, each shape on its own stream,
largest instances first.

Izhikevich half: one ``Network`` holding every instance as its own
population (the pulse-network recipe: 100 distinct targets per neuron,
device thalamic noise keyed by the instance's seed).  Its weights 0.5 U and
-U have U on the 1/256 grid, so every ring sum is exact (pre-centric
order-free scatter) and BF16 stores them without rounding: the BF16 run
gives the FP32 bits, which are the reference's bits.  It steps in 32-step
CUDA graphs, each step one neuron launch and one scatter launch over all
instances (a per-population work table on the device).

Both halves are enqueued on their own streams and overlap on the device;
the Kuramoto CTAs and the network's kernels share the SMs.  Instances do
not interact, so each one's result is the result it has alone.

The reference runs such a sweep as separate simulations: Kuramoto by
crates/SiMuse/crates/pillars/src/kernels/phase/kuramoto.rs:42-68 with the
mean field of crates/SiMuse/crates/t3/src/oscillator.rs:15-20,549, and each
Izhikevich network through the Network builder/step API
(crates/SiMuse/crates/pillars/src/api/net/network/).
"""
from __future__ import annotations

import numpy as np

from . import workloads as W
from .kuramoto import KuramotoBatch
from .network import W_BF16, Network

IZH_DT_MS = 1.0


class Sweep:
    """Kuramoto instances ``kura`` (a dict as ``workloads.kuramoto_sweep``
    returns) and Izhikevich instances of sizes ``izh_sizes`` (seeds
    ``izh_seed0 + i``), weights in ``weights`` (BF16 by default)."""

    def __init__(self, kura: dict, izh_sizes, izh_seed0: int = 1000, device: int = 0, weights: int = W_BF16,
                 k_out: int = 100):
        self.device = device
        self.kura = kura
        self.kb = KuramotoBatch(kura["sizes"], kura["coupling"], kura["dt"], device)
        self.kb.set_state(kura["theta"], kura["omega"])
        self.izh_sizes = np.asarray(izh_sizes, np.int64)
        self.izh_seeds = izh_seed0 + np.arange(self.izh_sizes.size, dtype=np.int64)
        self.net = Network(device)
        self.net.set_weight_format(weights)
        self.pops = [W.add_izhikevich_instance(self.net, int(n), int(s), k_out=k_out, random_w=8)
                     for n, s in zip(self.izh_sizes, self.izh_seeds)]
        self.net.build()
        self.net.enable_neuron_stats(True)
        self.izh_steps = 0
        self.kura_steps = 0

    @classmethod
    def configured(cls, n_kura: int = 1024, n_izh: int = 1024, device: int = 0, kura_seed: int = 0,
                   izh_seed: int = 7, **kw) -> "Sweep":
        """The batched-sweep configuration: Kuramoto N log-uniform in
        256..65,536, K linear over 0..4, omega ~ Lorentzian(0, 0.5), RK4 at
        dt 0.01; Izhikevich N log-uniform in 500..200,000."""
        return cls(W.kuramoto_sweep(n_kura, seed=kura_seed), W.izh_sweep_sizes(n_izh, seed=izh_seed),
                   device=device, **kw)

    # -- running ----------------------------------------------------------------
    def record_r(self, max_steps: int):
        """Record r(t) of every Kuramoto instance for up to max_steps steps."""
        self.kb.record(max_steps)

    def enqueue(self, izh_steps: int, kura_steps: int):
        """Start both halves without waiting: the Kuramoto launches first
        (their CTAs hold SMs longest), then the network's graphs."""
        if kura_steps:
            self.kb.run(kura_steps)
            self.kura_steps += int(kura_steps)
        if izh_steps:
            self.net.step(izh_steps)
            self.izh_steps += int(izh_steps)

    def synchronize(self):
        self.kb.synchronize()
        self.net.synchronize()

    def run(self, izh_steps: int, kura_steps: int):
        self.enqueue(izh_steps, kura_steps)
        self.synchronize()

    @property
    def streams(self) -> tuple[int, int]:
        """(Kuramoto stream, network stream) handles."""
        return self.kb.stream(), self.net.stream

    # -- results ----------------------------------------------------------------
    def izh_counts(self, i: int) -> np.ndarray:
        """Spikes per neuron of Izhikevich instance i since the build."""
        rates, _, _, steps = self.net.neuron_stats(self.pops[i], IZH_DT_MS)
        return np.rint(rates * steps * IZH_DT_MS * 1e-3).astype(np.int64)

    def izh_rates(self) -> np.ndarray:
        """Mean firing rate (Hz) of every Izhikevich instance."""
        out = np.empty(len(self.pops))
        for i, p in enumerate(self.pops):
            rates, _, _, _ = self.net.neuron_stats(p, IZH_DT_MS)
            out[i] = float(rates.mean())
        return out

    def izh_state(self, i: int, col: int = 0) -> np.ndarray:
        return self.net.state(self.pops[i], col)

    def kura_theta(self, i: int) -> np.ndarray:
        return self.kb.instance_theta(i)

    def kura_r(self) -> np.ndarray:
        return self.kb.r()

    def kura_r_mean(self) -> np.ndarray:
        return self.kb.r_mean()

    @property
    def neurons(self) -> int:
        return int(self.izh_sizes.sum())

    @property
    def oscillators(self) -> int:
        return int(self.kb.total)

    @property
    def events_total(self) -> int:
        return self.net.events_total

    @property
    def footprint(self) -> int:
        return self.net.footprint

    def close(self):
        for h in ("net", "kb"):
            o = getattr(self, h, None)
            if o is not None:
                o.close()
                setattr(self, h, None)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

