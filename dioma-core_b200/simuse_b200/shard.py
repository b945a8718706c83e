"""One network split across GPUs.

The neurons are cut into `world` contiguous slices of the global index
space; rank r simulates slice r and holds every synapse onto it.  Every rank
lays out the same device populations in global order: a population piece
that rank r simulates is an ordinary population there, every other piece is
an external population (pre-synaptic only, spikes from the exchange).  The
device indices are therefore the same on every rank and equal in order to
the global ones, so a rank's scatter walks the spiking neurons of the whole
network in the whole network's order, and each ring cell of a local neuron
receives the adds it would receive in the unsplit network, in the same
order: a split network gives the unsplit network's bits.

Per step: `step_begin` on every rank (local neuron update), the exchange of
this step's spike words (an all-gather of each rank's bitmask over NCCL, or
device pointers into the other networks when several ranks share a
process), `step_end` (external spikes, scatter).  The reference simulates
one network on one host (P/api/net/network/step.rs:18-189); the split is
this build's, for networks larger than one GPU.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class PopSpec:
    model: int
    n: int
    params: dict          # column -> scalar or array of n
    state: dict           # column -> scalar or array of n


@dataclasses.dataclass
class NetSpec:
    """A whole network: populations in order (global indices are their
    concatenation) and synapses (global pre, global post, weight, delay) in
    connect order."""
    pops: list
    pre: np.ndarray
    post: np.ndarray
    w: np.ndarray
    d: np.ndarray

    @property
    def total(self) -> int:
        return int(sum(p.n for p in self.pops))


def slices(total: int, world: int):
    """Contiguous neuron ranges [lo, hi) of each rank."""
    b = [(total * r) // world for r in range(world + 1)]
    return [(b[r], b[r + 1]) for r in range(world)]


def pieces(spec: NetSpec, world: int):
    """(population, owner rank, first, last+1) pieces in global order; every
    rank builds these as its device populations."""
    out, off = [], 0
    rr = slices(spec.total, world)
    for g, p in enumerate(spec.pops):
        for q, (lo, hi) in enumerate(rr):
            a, b = max(lo, off), min(hi, off + p.n)
            if a < b:
                out.append((g, q, a - off, b - off))
        off += p.n
    return out


class Shard:
    """Rank `rank`'s part of `spec`, built into `net` (not yet built)."""

    def __init__(self, net, spec: NetSpec, rank: int, world: int):
        self.net, self.rank, self.world = net, rank, world
        self.pieces = pieces(spec, world)
        self.lo, self.hi = slices(spec.total, world)[rank]
        offs = np.concatenate([[0], np.cumsum([p.n for p in spec.pops])]).astype(np.int64)
        self.pid, self.gstart = [], []
        for g, q, a, b in self.pieces:
            ps = spec.pops[g]
            if q == rank:
                pid = net.add_population(ps.model, b - a)
                for col, v in ps.params.items():
                    if np.ndim(v) == 0:
                        net.fill_param(pid, col, float(v))
                    else:
                        net.set_param(pid, col, np.asarray(v, np.float32)[a:b])
                for col, v in ps.state.items():
                    if np.ndim(v) == 0:
                        net.fill_state(pid, col, float(v))
                    else:
                        net.set_state(pid, col, np.asarray(v, np.float32)[a:b])
            else:
                pid = net.add_external_population(b - a)
            self.pid.append(pid)
            self.gstart.append(int(offs[g] + a))
        self.gstart = np.array(self.gstart, np.int64)
        # synapses onto this rank's neurons, grouped by (pre piece, post piece);
        # one (pre, post) pair always falls in one group, so repeated pairs keep
        # their connect order
        keep = (spec.post >= self.lo) & (spec.post < self.hi)
        pre, post = spec.pre[keep].astype(np.int64), spec.post[keep].astype(np.int64)
        w, d = spec.w[keep], spec.d[keep]
        pk = np.searchsorted(self.gstart, pre, side="right") - 1
        qk = np.searchsorted(self.gstart, post, side="right") - 1
        order = np.lexsort((qk, pk))  # stable: connect order inside a group
        pre, post, w, d, pk, qk = pre[order], post[order], w[order], d[order], pk[order], qk[order]
        bounds = np.flatnonzero(np.diff(pk * len(self.pieces) + qk)) + 1
        for s, e in zip(np.concatenate([[0], bounds]), np.concatenate([bounds, [pre.size]])):
            if s == e:
                continue
            a, b = int(pk[s]), int(qk[s])
            net.connect(self.pid[a], (pre[s:e] - self.gstart[a]).astype(np.uint32), self.pid[b],
                        (post[s:e] - self.gstart[b]).astype(np.uint32), np.ascontiguousarray(w[s:e], np.float32),
                        np.ascontiguousarray(d[s:e], np.uint8))

    def word_offsets(self):
        """Each piece's first bitmask word in the device layout (every rank's
        is the same: pieces in order, each padded to 1024 neurons)."""
        caps = [-(-(b - a) // 1024) * 1024 for _, _, a, b in self.pieces]
        return np.concatenate([[0], np.cumsum(caps)]).astype(np.int64)[:-1] // 32, int(sum(caps)) // 32

    def local(self):
        """(piece index, device population, global start, size) of the pieces simulated here."""
        return [(k, self.pid[k], int(self.gstart[k]), b - a)
                for k, (g, q, a, b) in enumerate(self.pieces) if q == self.rank]

    def external(self):
        return [(k, self.pid[k], q) for k, (g, q, a, b) in enumerate(self.pieces) if q != self.rank]

    def inject(self, current: np.ndarray):
        """Global input current (one value per neuron) onto the local neurons."""
        for _, pid, g0, n in self.local():
            self.net.inject_current(pid, np.arange(n, dtype=np.uint32), np.ascontiguousarray(current[g0:g0 + n],
                                                                                            np.float32))

    def spikes(self, out: np.ndarray):
        """This step's spikes of the local neurons into the global vector."""
        for _, pid, g0, n in self.local():
            out[g0:g0 + n] = self.net.spikes(pid)

    def state(self, col: int, out: np.ndarray):
        for _, pid, g0, n in self.local():
            out[g0:g0 + n] = self.net.state(pid, col)


def link_in_process(shards):
    """Several ranks' networks on one process (one or more GPUs the process
    can reach): each external piece reads the owner network's spike words
    directly.  Steps must then be issued as `step_in_process` does."""
    for sh in shards:
        for k, pid, q in sh.external():
            sh.net.set_external_source(pid, shards[q].net.spike_words_ptr(shards[q].pid[k]))


def step_in_process(shards):
    """One step of a split network whose ranks share this process: every
    neuron update finishes before any rank reads another's spike words."""
    for sh in shards:
        sh.net.step_begin()
    for sh in shards:
        sh.net.synchronize()
    for sh in shards:
        sh.net.step_end()
    for sh in shards:
        sh.net.synchronize()


class _Words:
    """A device array of int32 words exposed to torch (no copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (ptr, False), "version": 3}


class Exchange:
    """The per-step spike exchange of a split network over torch.distributed
    (one process per GPU): every rank's whole bitmask is all-gathered into a
    [world, words] buffer on the network's stream, and each external piece
    reads its owner's slice of it.  Every rank makes the same collective
    call each step."""

    def __init__(self, shard: Shard, group=None):
        import torch
        self.torch = torch
        import torch.distributed as dist
        self.dist, self.group = dist, group
        net = shard.net
        self.stream = torch.cuda.ExternalStream(net.stream, device=torch.device("cuda", net.device))
        offs, words = shard.word_offsets()
        base = net.spike_words_ptr(shard.pid[0])
        self.local = torch.as_tensor(_Words(base, words), device=f"cuda:{net.device}")
        self.gather = torch.zeros((shard.world, words), dtype=torch.int32, device=f"cuda:{net.device}")
        g0 = self.gather.data_ptr()
        for k, pid, q in shard.external():
            net.set_external_source(pid, g0 + (q * words + int(offs[k])) * 4)
        self.shard = shard

    def step(self):
        net = self.shard.net
        net.step_begin()
        with self.torch.cuda.stream(self.stream):
            self.dist.all_gather_into_tensor(self.gather.view(-1), self.local, group=self.group)
        net.step_end()
