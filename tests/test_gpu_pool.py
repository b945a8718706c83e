"""Pools of resident networks (sg_pool): members step together, one neuron
launch per model over all of them and one scatter launch over all of them
per step, and each member gives the same bits as the same network stepped
alone.  Members join and leave between steps and keep their own step
counters, readbacks and streams."""
import numpy as np
import pytest

import simuse_b200 as sg
from simuse_b200 import serve as S
from simuse_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _members():
    return [S.Request("lif", 20000, 31, 0), S.Request("izh", 15000, 32, 0), S.Request("lif", 3000, 33, 0),
            S.Request("izh", 40000, 34, 0)]


def _build(req):
    net = S.build_request(req)
    net.build()
    return net


def _run(net, chunks):
    net.enable_raster(max(chunks))
    out = []
    for k in chunks:
        net.step(k)
        out.append(net.read_raster())
    return out


def test_pool_members_equal_networks_alone():
    chunks = [40, 1, 77, 32, 5]
    alone = []
    for req in _members():
        net = _build(req)
        assert net.scatter_mode == "exact"
        alone.append((_run(net, chunks), net.state(0, 0).copy(), net.events_total))
        net.close()
    pool = sg.Pool(0)
    nets = [_build(r) for r in _members()]
    for net in nets:
        net.enable_raster(max(chunks))
        pool.add(net)
    assert len(pool) == 4
    got = [[] for _ in nets]
    for k in chunks:
        pool.step(k)
        for i, net in enumerate(nets):
            got[i].append(net.read_raster())
    pool.synchronize()
    for i, net in enumerate(nets):
        ra, va, ea = alone[i]
        for a, b in zip(ra, got[i]):
            assert np.array_equal(a, b), i
        assert np.array_equal(net.state(0, 0).view(np.uint32), va.view(np.uint32)), i
        assert net.events_total == ea
        assert net.step_counter == sum(chunks)
    pool.close()
    for net in nets:
        net.close()


def test_pool_members_join_and_leave_between_steps():
    reqs = _members()
    ref = []
    for req in reqs[:2]:
        net = _build(req)
        net.step(100)
        ref.append(net.state(0, 0).copy())
        net.close()
    a, b = _build(reqs[0]), _build(reqs[1])
    pool = sg.Pool(0)
    pool.add(a)
    pool.step(30)            # a: 30
    pool.add(b)
    pool.step(40)            # a: 70, b: 40
    pool.remove(a)
    a.step(30)               # a alone on its own stream: 100
    pool.step(60)            # b: 100
    pool.synchronize()
    assert a.step_counter == 100 and b.step_counter == 100
    assert np.array_equal(a.state(0, 0).view(np.uint32), ref[0].view(np.uint32))
    assert np.array_equal(b.state(0, 0).view(np.uint32), ref[1].view(np.uint32))
    b.close()                # a destroyed member leaves its pool
    assert len(pool) == 0
    pool.close()
    a.close()


def test_pool_refuses_ordered_networks():
    net = sg.Network(0)
    spec = W.lif_balanced(n=2000, k_in=50, seed=3, ext_rate_hz=4000.0, ext_weight=100.0, w_exc=0.1)
    W.build_lif(net, spec)
    net.build()
    assert net.scatter_mode == "ordered"
    pool = sg.Pool(0)
    with pytest.raises(sg.SimuseError, match="pre-centric"):
        pool.add(net)
    pool.close()
    net.close()


def test_staged_raster_reads_equal_plain_reads():
    """sg_raster_stage / sg_raster_fetch in a pipeline (the next steps are
    queued before the last batch is fetched) give the events of plain reads,
    and the device's per-neuron counts equal the counts of those events."""
    chunks = [50, 13, 50, 1, 37, 50]
    a, b = _build(S.Request("lif", 20000, 31, 0)), _build(S.Request("lif", 20000, 31, 0))
    a.enable_raster(50)
    b.enable_raster(50)
    plain = []
    for k in chunks:
        a.step(k)
        plain.append(a.read_spike_events())
    staged = []
    for j, k in enumerate(chunks):
        b.step(k)
        if j:
            staged.append(b.raster_fetch(16))   # 16 pairs: too small, fetched again at the batch's size
        b.raster_stage()
    staged.append(b.raster_fetch())
    for (s0, i0), (s1, i1) in zip(plain, staged):
        assert s0.size > 100
        assert np.array_equal(s0, s1) and np.array_equal(i0, i1)
    idx = np.concatenate([i for _, i in plain]).astype(np.int64)
    want = np.bincount(idx, minlength=a.total_neurons)
    assert np.array_equal(a.raster_counts(), want)
    assert np.array_equal(b.raster_counts(), want)
    assert np.array_equal(a.state(0, 0).view(np.uint32), b.state(0, 0).view(np.uint32))
    with pytest.raises(sg.SimuseError, match="no staged"):
        b.raster_fetch()
    b.raster_stage()
    with pytest.raises(sg.SimuseError, match="not fetched"):
        b.read_spike_events()
    b.raster_fetch()
    a.close()
    b.close()
