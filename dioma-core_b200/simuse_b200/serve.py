"""A served stream of simulation requests on one GPU.

Each request names a seeded network (LIF or Izhikevich, N neurons, lognormal
out-degree, BF16 weights) and a number of simulation steps, and gets back its
spike events and per-neuron firing rates.  The server keeps every admitted
network's state, synapses and delay rings resident in HBM until it finishes,
and batches continuously: the resident networks are members of one pool
(sg_pool), which steps them together, per step one neuron launch per model
over every member's populations and one scatter launch over every member.  A
request that arrives while others are running is admitted as soon as a
resident slot and enough of the memory budget are free: it is built on its
own stream beside the running pool and joins the pool at the next tick;
finished requests leave it and release their budget.  Admission is by
resident footprint against the budget (an estimate at admission, replaced by
the measured footprint of the built network).  Latency is measured per
request from submission to completion.

Networks do not interact, and each one's random streams (Poisson drive,
input noise) are keyed by its own seed and its own step counter, so a
request's result does not depend on what else is resident: the same bits
alone and in any mix.  Every served network's ring sums are exact (the LIF
weights 20, -100 and 100; the Izhikevich weights 0.5 U and -U with U on the
1/256 grid, which BF16 also holds exactly), so they all take the pre-centric
scatter that a pool runs.

The reference has no serving layer; this is a request loop over many
simulations, written over the same builder/step API the reference's callers use
(crates/SiMuse/crates/pillars/src/api/net/network/).
"""
from __future__ import annotations

import dataclasses
import queue
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import workloads as W
from .network import IZH, LIF, W_BF16, Network, PinnedU32, Pool


@dataclasses.dataclass
class Request:
    kind: str                 # "lif" or "izh"
    n: int                    # neurons
    seed: int
    steps: int                # simulation steps to run
    mean_degree: float = 100.0
    sd_degree: float = 60.0
    # filled by the server
    id: int = -1
    t_submit: float = 0.0
    t_admit: float = 0.0
    t_done: float = 0.0
    footprint: int = 0
    # the spike raster as read, one (t0, step offsets, indices) chunk per read:
    # the spikes of step t0 + s are indices[offsets[s]:offsets[s + 1]]
    chunks: list | None = None
    rates_hz: np.ndarray | None = None
    error: str | None = None
    _flat: tuple | None = dataclasses.field(default=None, repr=False)

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit

    def _flatten(self):
        if self._flat is None and self.chunks is not None:
            st = [np.repeat(np.arange(t0, t0 + off.size - 1, dtype=np.uint32), np.diff(off)) for t0, off, _ in self.chunks]
            ix = [i for _, _, i in self.chunks]
            self._flat = (np.concatenate(st) if st else np.empty(0, np.uint32),
                          np.concatenate(ix) if ix else np.empty(0, np.uint32))
        return self._flat

    @property
    def spike_steps(self) -> np.ndarray | None:
        """Step of every spike, in step then neuron order (built from the chunks
        on first use)."""
        f = self._flatten()
        return None if f is None else f[0]

    @property
    def spike_index(self) -> np.ndarray | None:
        """Global neuron index of every spike, in the order of spike_steps."""
        f = self._flatten()
        return None if f is None else f[1]

    @property
    def dt_ms(self) -> float:
        return 0.1 if self.kind == "lif" else 1.0


def estimate_footprint(req: Request) -> int:
    """Device bytes a request holds while it is built and resident: synapse
    records (8 B while building, then x word + BF16 weight), the per-row
    segment table, rings, state, spike lists and the build-time buffers (the
    peak), rounded up generously."""
    n = req.n
    nd = -(-n // 1024) * 1024
    e = int(n * req.mean_degree * 1.05)
    per_neuron = 32 * 4 + 16 * 4 + 16 + 148 * 2 + 64   # rings (<= 32 slots), state+params, spike lists, segments
    build_peak = e * 45                                # staged edges + sort buffers + records
    return int(nd * per_neuron + build_peak + (64 << 20))


def build_request(req: Request, device: int = 0) -> Network:
    """The request's network through the builder API (not yet built)."""
    net = Network(device)
    net.set_weight_format(W_BF16)
    n, n_exc = req.n, req.n * 4 // 5
    if req.kind == "lif":
        pop = net.add_population(LIF, n)
        for col, v in enumerate(W.LIF_PARAMS):
            net.fill_param(pop, col, v)
        u = W.uniform01(req.seed, W.LIF_STREAM_V0, np.arange(n, dtype=np.uint64))
        net.set_state(pop, 0, (10.0 + 10.0 * u).astype(np.float32))
        # ring weights J*tau/dt for J = 0.1 mV (g = 5), delay 2 steps
        net.connect_lognormal_outdegree(pop, pop, req.mean_degree, req.sd_degree, req.seed, True, n_exc,
                                        20.0, -100.0, random_w=False, delay=2)
        first = net.add_poisson_sources(n, 4000.0, 0.1, seed0=req.seed * 7919)
        net.connect_poisson_one_to_one(first, n, pop, 100.0, 1)
    elif req.kind == "izh":
        pop = net.add_population(IZH, n)
        a, b, c, d = W.izhikevich_params(n, n_exc, req.seed)
        net.fill_param(pop, 0, 1.0)
        for col, v in ((1, a), (2, b), (3, c), (4, d)):
            net.set_param(pop, col, v)
        net.fill_param(pop, 5, 0.0)
        net.fill_param(pop, 6, 30.0)
        net.fill_state(pop, 0, -65.0)
        net.set_state(pop, 1, (b * np.float32(-65.0)).astype(np.float32))
        # weights 0.5 U / -U with U on the 1/256 grid: exact ring sums, exact in BF16
        net.connect_lognormal_outdegree(pop, pop, req.mean_degree, req.sd_degree, req.seed, True, n_exc,
                                        0.5, -1.0, random_w=8, delay=1)
        net.set_noise(pop, req.seed, 5.0, 2.0, split=n_exc, stream=W.IZH_STREAM_NOISE, stride=n)
    else:
        raise ValueError(f"unknown request kind {req.kind!r}")
    return net


def run_alone(req: Request, device: int = 0, chunk: int = 256) -> Request:
    """The plain path: build, run and read back one request by itself."""
    req.t_submit = req.t_admit = time.perf_counter()
    net = build_request(req, device)
    net.build()
    _run_to_end(net, req, chunk)
    net.close()
    req.t_done = time.perf_counter()
    return req


_solo_bufs = threading.local()


def _run_to_end(net: Network, req: Request, chunk: int):
    bufs = getattr(_solo_bufs, "b", None)
    if bufs is None:
        bufs = _solo_bufs.b = (PinnedU32(), PinnedU32(1 << 20))
    net.enable_raster(chunk)
    chunks = []
    done = 0
    while done < req.steps:
        k = min(chunk, req.steps - done)
        net.step(k)
        net.raster_stage()
        chunks.append(net.raster_fetch_csr(*bufs))
        done += k
    _finish(req, chunks, net.raster_counts())


def _finish(req: Request, chunks, counts):
    """The request's results: its spike raster as read (chunks of step
    offsets and indices) and its rates from the per-neuron spike counts the
    device kept while reading."""
    req.chunks = chunks
    req.rates_hz = counts / (req.steps * req.dt_ms * 1e-3)


class _Resident:
    def __init__(self, req: Request, net: Network, bufs):
        self.req, self.net = req, net
        self.bufs = bufs            # page-locked (step offsets, indices) buffers, the server's
        self.done = 0
        self.chunks: list = []
        self.counts: np.ndarray | None = None

    def fetch(self):
        return self.net.raster_fetch_csr(*self.bufs)


class Server:
    """Continuous-batching request loop on one GPU (see the module text).

    budget_bytes: device memory the resident networks may hold together.
    max_resident: resident networks at most (pool members; at most 64).
    chunk: steps the pool advances per tick; a network that needs fewer
    steps than that leaves the pool and runs them alone beside the tick; a
    multiple of 32 runs as whole 32-step graphs.
    builders: threads building admitted networks beside the running pool.
    """

    def __init__(self, device: int = 0, budget_bytes: int = 160 * 10**9, max_resident: int = 32,
                 chunk: int = 256, builders: int = 2, readers: int = 8):
        self.device, self.budget, self.chunk = device, int(budget_bytes), chunk
        self.max_resident = min(max_resident, 64)
        self._pending: queue.Queue[Request] = queue.Queue()
        self._built: queue.Queue[tuple[Request, Network | None]] = queue.Queue()
        self._to_build: queue.Queue[Request | None] = queue.Queue()
        self._lock = threading.Lock()
        self._reserved = 0            # budget bytes held by building and resident networks
        self._next_id = 0
        self.completed: list[Request] = []
        self.ticks = 0
        # host seconds the stepping thread spent per phase (for tuning)
        self.phase_s = {"admit": 0.0, "step": 0.0, "collect": 0.0, "stage": 0.0, "leave": 0.0, "idle": 0.0}
        self._stop = threading.Event()
        self._idle = threading.Event()
        self._n_open = 0
        # the networks' spikes of a tick are read back in parallel (each on its
        # own stream); a finished request's results are assembled off the
        # stepping thread
        self._readers = ThreadPoolExecutor(max_workers=max(1, readers))
        self._finishing: queue.Queue = queue.Queue()
        # page-locked readback buffers, reused by the requests that follow
        self._free_bufs: list = []
        self._builders = [threading.Thread(target=self._build_loop, daemon=True) for _ in range(max(1, builders))]
        self._stepper = threading.Thread(target=self._step_loop, daemon=True)
        self._finisher = threading.Thread(target=self._finish_loop, daemon=True)
        for b in self._builders:
            b.start()
        self._stepper.start()
        self._finisher.start()

    # -- client side ----------------------------------------------------------
    def submit(self, req: Request) -> Request:
        req.t_submit = time.perf_counter()
        with self._lock:
            req.id = self._next_id
            self._next_id += 1
            self._n_open += 1
            self._idle.clear()
        if estimate_footprint(req) > self.budget:
            req.error = "request larger than the device budget"
            self._complete(req)
            return req
        self._pending.put(req)
        return req

    def wait_idle(self, timeout: float | None = None) -> bool:
        return self._idle.wait(timeout)

    def close(self):
        self._stop.set()
        for _ in self._builders:
            self._to_build.put(None)
        self._stepper.join()
        for b in self._builders:
            b.join()
        self._finishing.put(None)
        self._finisher.join()
        self._readers.shutdown()

    def latency_percentiles(self) -> dict:
        lat = np.array([r.latency for r in self.completed if r.error is None])
        if lat.size == 0:
            return {"p50_s": None, "p99_s": None, "n": 0}
        return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)), "n": int(lat.size)}

    # -- server side ------------------------------------------------------------
    def _complete(self, req: Request):
        req.t_done = time.perf_counter()
        with self._lock:
            self.completed.append(req)
            self._n_open -= 1
            if self._n_open == 0:
                self._idle.set()

    def _finish_loop(self):
        while True:
            item = self._finishing.get()
            if item is None:
                return
            r = item
            _finish(r.req, r.chunks, r.counts)
            self._complete(r.req)

    def _build_loop(self):
        while True:
            req = self._to_build.get()
            if req is None:
                return
            try:
                net = build_request(req, self.device)
                net.build()
                net.synchronize()
                self._built.put((req, net))
            except Exception as e:  # a failed build releases its reservation
                req.error = str(e)
                self._built.put((req, None))

    def _step_loop(self):
        """Ticks in a pipeline: tick t is queued, then the host collects the
        spikes of tick t - 1 (copied out beside tick t), stages tick t's
        spikes for compaction right after it and hands their copy to the
        readers, so the GPU keeps stepping while results come back.  A
        request that finished leaves the pool at once and completes when its
        last batch is in."""
        pool = Pool(self.device)
        resident: list[_Resident] = []
        draining: list[_Resident] = []   # out of the pool, last batch in flight
        inflight: list = []              # (resident, future) of the last tick's fetches
        building = 0
        waiting: list[Request] = []
        ph = self.phase_s
        while not self._stop.is_set() or resident or building or inflight or draining:
            t0 = time.perf_counter()
            # arrivals
            while True:
                try:
                    waiting.append(self._pending.get_nowait())
                except queue.Empty:
                    break
            # admission in arrival order, by footprint and slot
            while waiting and len(resident) + len(draining) + building < self.max_resident:
                req = waiting[0]
                est = estimate_footprint(req)
                with self._lock:
                    if self._reserved + est > self.budget:
                        break
                    self._reserved += est
                req.footprint = est
                req.t_admit = time.perf_counter()
                waiting.pop(0)
                building += 1
                self._to_build.put(req)
            # networks that finished building join the pool
            while True:
                try:
                    req, net = self._built.get_nowait()
                except queue.Empty:
                    break
                building -= 1
                if net is None:
                    with self._lock:
                        self._reserved -= req.footprint
                    self._complete(req)
                    continue
                true_fp = net.footprint
                with self._lock:                  # the measured footprint replaces the estimate
                    self._reserved += true_fp - req.footprint
                req.footprint = true_fp
                net.enable_raster(self.chunk)
                pool.add(net)
                bufs = self._free_bufs.pop() if self._free_bufs else (PinnedU32(), PinnedU32(1 << 20))
                resident.append(_Resident(req, net, bufs))
            t1 = time.perf_counter()
            ph["admit"] += t1 - t0
            if not resident and not inflight:
                time.sleep(0.0005)
                ph["idle"] += time.perf_counter() - t1
                continue
            # tick t: every resident network advances a full tick in the pool;
            # one that needs fewer steps than that leaves the pool and runs its
            # last steps alone on its own stream, beside the tick (a short tick
            # would cost the whole pool a tick's host work for a few steps)
            k = 0
            tail = [r for r in resident if r.req.steps - r.done < self.chunk]
            for r in tail:
                resident.remove(r)
                pool.remove(r.net)
                r.net.step(r.req.steps - r.done)
            if resident:
                k = self.chunk
                pool.step(k)
                self.ticks += 1
            t2 = time.perf_counter()
            ph["step"] += t2 - t1
            # tick t - 1's spikes (their copies ran beside tick t)
            for r, fut in inflight:
                r.chunks.append(fut.result())
            inflight = []
            for r in draining:              # finished requests whose last batch is in
                r.counts = r.net.raster_counts()
                r.net.close()
                self._free_bufs.append(r.bufs)
                with self._lock:
                    self._reserved -= r.req.footprint
                self._finishing.put(r)
            draining = []
            t3 = time.perf_counter()
            ph["collect"] += t3 - t2
            if not resident and not tail:
                continue
            # tick t's spikes: compaction queued after the tick, copies to the readers
            for r in resident:
                r.net.raster_stage()
                r.done += k
            for r in tail:
                r.net.raster_stage()
                r.done = r.req.steps
            inflight = [(r, self._readers.submit(r.fetch)) for r in resident + tail]
            t4 = time.perf_counter()
            ph["stage"] += t4 - t3
            # finished requests leave the pool before the next tick
            for r in [r for r in resident if r.done >= r.req.steps]:
                resident.remove(r)
                pool.remove(r.net)
                draining.append(r)
            draining.extend(tail)
            ph["leave"] += time.perf_counter() - t4
        pool.close()
        for off, idx in self._free_bufs:
            off.close()
            idx.close()
        self._free_bufs = []
