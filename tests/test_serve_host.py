"""Host logic of the continuous-batching server (simuse_b200.serve.Server),
without a GPU: the networks, the pool and the page-locked buffers are
replaced by fakes that count steps and report one spike per step, so the
tests check what the server itself decides: admission in arrival order by
footprint against the budget, at most `max_resident` networks at a time,
every request run for exactly its number of steps (full pool ticks plus a
tail run alone), results assembled from the per-tick reads, and requests
larger than the whole budget refused."""
import threading
import time

import numpy as np
import pytest

from simuse_b200 import serve as S


class _Ledger:
    """Device bytes held by the fake networks, and the largest pool seen."""

    def __init__(self):
        self.lock = threading.Lock()
        self.live = 0
        self.peak = 0
        self.max_members = 0
        self.nets = 0        # fake networks alive (built, not yet freed)
        self.max_nets = 0
        self.budget = None
        self.fp_frac = 0.5   # a built network's footprint against the server's estimate


class _FakeNet:
    def __init__(self, req, ledger):
        self.req, self.ledger = req, ledger
        self.footprint = int(S.estimate_footprint(req) * ledger.fp_frac)
        self.step_counter = 0
        self.staged = (0, 0)
        self.mark = 0
        self.spikes = np.zeros(req.n, np.uint32)
        self.closed = False
        with ledger.lock:
            ledger.live += self.footprint
            ledger.peak = max(ledger.peak, ledger.live)
            ledger.nets += 1
            ledger.max_nets = max(ledger.max_nets, ledger.nets)
            assert ledger.budget is None or ledger.live <= ledger.budget

    # builder API
    def build(self):
        pass

    def synchronize(self):
        pass

    # stepping (alone, for a tail shorter than a tick)
    def step(self, k):
        assert not self.closed
        self.step_counter += k

    def enable_raster(self, cap):
        self.cap = cap

    def raster_stage(self):
        self.staged = (self.mark, self.step_counter)
        self.mark = self.step_counter

    def raster_fetch_csr(self, off_buf, idx_buf):
        t0, t1 = self.staged
        idx = ((self.req.seed + np.arange(t0, t1, dtype=np.uint64)) % self.req.n).astype(np.uint32)
        np.add.at(self.spikes, idx, 1)
        return t0, np.arange(t1 - t0 + 1, dtype=np.uint32), idx

    def raster_counts(self):
        return self.spikes.copy()

    def close(self):
        if not self.closed:
            self.closed = True
            with self.ledger.lock:
                self.ledger.live -= self.footprint
                self.ledger.nets -= 1


class _FakePool:
    def __init__(self, ledger):
        self.ledger = ledger
        self.members = []

    def add(self, net):
        self.members.append(net)
        with self.ledger.lock:
            self.ledger.max_members = max(self.ledger.max_members, len(self.members))

    def remove(self, net):
        self.members.remove(net)

    def step(self, k):
        for m in self.members:
            m.step(k)

    def close(self):
        assert not self.members


class _FakePinned:
    def __init__(self, n=0):
        self.n = n

    def ensure(self, n):
        self.n = max(self.n, n)

    def close(self):
        pass


@pytest.fixture
def fakes(monkeypatch):
    ledger = _Ledger()
    monkeypatch.setattr(S, "build_request", lambda req, device=0: _FakeNet(req, ledger))
    monkeypatch.setattr(S, "Pool", lambda device=0: _FakePool(ledger))
    monkeypatch.setattr(S, "PinnedU32", _FakePinned)
    return ledger


def _expected_steps(req):
    return np.arange(req.steps, dtype=np.uint32)


def _check_result(req):
    assert req.error is None
    assert np.array_equal(req.spike_steps, _expected_steps(req))
    want = ((req.seed + np.arange(req.steps, dtype=np.uint64)) % req.n).astype(np.uint32)
    assert np.array_equal(req.spike_index, want)
    counts = np.bincount(want, minlength=req.n)
    assert np.allclose(req.rates_hz, counts / (req.steps * req.dt_ms * 1e-3))


def test_every_request_runs_its_steps_in_ticks_and_tail(fakes):
    """Requests shorter than a tick, exact multiples of it and ragged lengths
    all get exactly their steps and their own spikes."""
    steps = [10, 64, 64 * 3, 64 * 2 + 17, 1, 300, 129]
    reqs = [S.Request("lif" if i % 2 else "izh", 1000 + 37 * i, 11 + i, s) for i, s in enumerate(steps)]
    srv = S.Server(budget_bytes=10**12, max_resident=4, chunk=64, builders=2, readers=2)
    for r in reqs:
        srv.submit(r)
    assert srv.wait_idle(60)
    srv.close()
    for r in reqs:
        _check_result(r)
    assert fakes.max_members <= 4
    assert fakes.live == 0   # every network was freed


def test_admission_by_footprint_and_budget(fakes):
    """With a budget that holds two of these requests (each built network as
    large as its estimate), no more than two are ever built or resident
    together, the rest wait in arrival order, and the device bytes never
    pass the budget."""
    reqs = [S.Request("lif", 50_000, 5 + i, 100) for i in range(6)]
    est = S.estimate_footprint(reqs[0])
    fakes.fp_frac = 1.0
    fakes.budget = 2 * est
    srv = S.Server(budget_bytes=2 * est + est // 2, max_resident=16, chunk=32)
    for r in reqs:
        srv.submit(r)
    assert srv.wait_idle(60)
    srv.close()
    for r in reqs:
        _check_result(r)
    assert fakes.peak <= 2 * est
    assert fakes.max_nets <= 2   # never three networks alive at once
    order = sorted(reqs, key=lambda r: r.t_admit)
    assert [r.id for r in order] == sorted(r.id for r in reqs)   # admitted in arrival order


def test_request_larger_than_budget_is_refused(fakes):
    big = S.Request("lif", 5_000_000, 1, 10)
    small = S.Request("izh", 2000, 2, 40)
    srv = S.Server(budget_bytes=S.estimate_footprint(small) * 2, chunk=16)
    srv.submit(big)
    srv.submit(small)
    assert srv.wait_idle(60)
    srv.close()
    assert big.error is not None
    _check_result(small)
    assert fakes.live == 0


def test_arrivals_while_running_join_later_ticks(fakes):
    """Requests submitted while others are resident join at a later tick and
    still get exactly their own steps."""
    srv = S.Server(budget_bytes=10**12, max_resident=8, chunk=16)
    first = [S.Request("lif", 3000, 40 + i, 400) for i in range(3)]
    for r in first:
        srv.submit(r)
    time.sleep(0.05)
    later = [S.Request("izh", 2500, 60 + i, 50 + 7 * i) for i in range(4)]
    for r in later:
        srv.submit(r)
    assert srv.wait_idle(60)
    srv.close()
    for r in first + later:
        _check_result(r)
    assert srv.ticks > 0
    assert fakes.live == 0
