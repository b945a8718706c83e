"""The served request stream: continuous batching with admission by memory
footprint, and each request's result the same alone and in the mix."""
import time

import numpy as np
import pytest

from simuse_b200 import serve as S

pytestmark = pytest.mark.gpu


def _reqs():
    return [S.Request("lif", 20000, 11, 300), S.Request("izh", 15000, 12, 200),
            S.Request("lif", 8000, 13, 500), S.Request("izh", 30000, 14, 150),
            S.Request("lif", 12000, 15, 256), S.Request("izh", 5000, 16, 400)]


def test_mix_equals_alone_and_latency_is_reported():
    alone = [S.run_alone(r) for r in _reqs()]
    srv = S.Server(max_resident=4, chunk=64)
    mix = [srv.submit(r) for r in _reqs()]
    assert srv.wait_idle(600)
    srv.close()
    for a, m in zip(alone, mix):
        assert m.error is None, m.error
        assert a.spike_index.size > 0
        assert np.array_equal(a.spike_steps, m.spike_steps) and np.array_equal(a.spike_index, m.spike_index)
        assert np.array_equal(a.rates_hz, m.rates_hz)
        assert m.latency > 0 and m.footprint > 0
    lat = srv.latency_percentiles()
    assert lat["n"] == 6 and 0 < lat["p50_s"] <= lat["p99_s"]


def test_admission_by_budget_and_arrivals_during_run():
    """With a budget that fits one of these requests at a time, they run one
    after another; requests submitted while others run are admitted later."""
    reqs = [S.Request("lif", 20000, 21 + i, 200) for i in range(3)]
    one = S.estimate_footprint(reqs[0])
    srv = S.Server(budget_bytes=int(one * 1.05), max_resident=8, chunk=50)
    srv.submit(reqs[0])
    time.sleep(0.05)
    srv.submit(reqs[1])
    srv.submit(reqs[2])
    assert srv.wait_idle(600)
    srv.close()
    assert all(r.error is None for r in reqs)
    # no two ran at the same time: each was admitted after the previous finished
    order = sorted(reqs, key=lambda r: r.t_admit)
    for a, b in zip(order, order[1:]):
        assert b.t_admit >= a.t_done - 1e-3
    big = S.Request("lif", 10_000_000, 1, 10)
    srv2 = S.Server(budget_bytes=one, chunk=10)
    srv2.submit(big)
    assert srv2.wait_idle(60)
    srv2.close()
    assert big.error is not None   # larger than the whole budget: refused, not queued forever


def test_csr_fetch_equals_event_pairs():
    """sg_raster_fetch_csr (step offsets and indices, through page-locked
    buffers) gives the spikes of the plain (step, index) read of the same
    network, and the same per-neuron counts."""
    from simuse_b200.network import PinnedU32
    r = S.Request("lif", 20000, 31, 300)
    a, b = S.build_request(r), S.build_request(r)
    a.build()
    b.build()
    a.enable_raster(100)
    b.enable_raster(100)
    bufs = (PinnedU32(), PinnedU32(16))   # a tiny index buffer: the fetch grows it
    total = 0
    for _ in range(3):
        a.step(100)
        b.step(100)
        s, i = a.read_spike_events()
        b.raster_stage()
        t0, off, ix = b.raster_fetch_csr(*bufs)
        assert off.size == 101 and off[0] == 0 and off[-1] == ix.size == i.size
        st = np.repeat(np.arange(t0, t0 + off.size - 1), np.diff(off))
        assert np.array_equal(st, s) and np.array_equal(ix, i)
        total += ix.size
    assert total > 0
    assert np.array_equal(a.raster_counts(), b.raster_counts())
    for x in (a, b):
        x.close()
    for x in bufs:
        x.close()
