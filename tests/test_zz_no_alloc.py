"""sg_push_spikes_noalloc — the push operator for callers that cannot allocate
device memory while they run (a real-time loop with no room for an
allocation that can block and synchronise the device, an embedding with a
fixed device-memory budget): it keeps its scratch in a fixed file-scope
device array.

Checks, through the C ABI, that two calls in a row give exactly the rings
that the allocating sg_push_spikes gives on the same inputs and that the
oracle's push_spikes gives (including a call of exactly the maximum number
of events), that inputs beyond the stated maxima or outside the neuron
range are rejected without touching the ring, and that calls allocate no
device memory.  This file is collected last so that a run stopping at the
first failure has already run every other test; it also passes alone in a
fresh process.
"""
import ctypes

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

MAX_EVENTS = 1 << 20
MAX_NEURONS = 1 << 23


def _dev(a):
    import torch
    t = torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).to("cuda:0")
    return t


def _call(name, bufs, n, n_active, step, ring):
    from simuse_b200 import _lib
    fn = getattr(_lib.lib(), name)
    return fn(ctypes.c_void_p(bufs["rp"].data_ptr()), ctypes.c_void_p(bufs["col"].data_ptr()),
              ctypes.c_void_p(bufs["w"].data_ptr()), ctypes.c_void_p(bufs["d"].data_ptr()), n,
              ctypes.c_void_p(bufs["a"].data_ptr()), n_active, step, ctypes.c_void_p(ring.data_ptr()), None)


def _network(n, deg, seed, hub=False):
    rng = np.random.default_rng(seed)
    counts = rng.integers(0, 2 * deg + 1, n)
    row_ptr = np.zeros(n + 1, np.uint32)
    row_ptr[1:] = np.cumsum(counts)
    e = int(row_ptr[-1])
    col = (rng.integers(0, 16, e) if hub else rng.integers(0, n, e)).astype(np.uint32)
    w = (rng.standard_normal(e) * 5.1).astype(np.float32)
    d = rng.integers(0, 32, e).astype(np.uint8)
    active = np.flatnonzero(rng.random(n) < 0.3).astype(np.uint32)
    ring = (rng.standard_normal((32, n)) * 3).astype(np.float32)
    return row_ptr, col, w, d, active, ring


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.mark.parametrize("n,deg,seed,hub", [(3000, 30, 11, False), (400, 60, 12, True), (50000, 8, 13, False)])
def test_noalloc_matches_allocating_push_two_calls(n, deg, seed, hub):
    import torch
    from simuse_b200 import _lib
    row_ptr, col, w, d, active, ring0 = _network(n, deg, seed, hub)
    bufs = dict(rp=_dev(row_ptr), col=_dev(col), w=_dev(w), d=_dev(d), a=_dev(active))
    ring_ref = torch.from_numpy(ring0.copy()).to("cuda:0")
    ring_new = torch.from_numpy(ring0.copy()).to("cuda:0")
    ring_cpu = ring0.copy()
    for call, step in enumerate((5, 6)):  # two calls in a row on the same rings
        _lib.check(_call("sg_push_spikes", bufs, n, active.size, step, ring_ref))
        _lib.check(_call("sg_push_spikes_noalloc", bufs, n, active.size, step, ring_new))
        O.push_spikes(row_ptr, col, w, d, n, active, step, ring_cpu)
        torch.cuda.synchronize()
        a = ring_ref.cpu().numpy()
        b = ring_new.cpu().numpy()
        # the push tests' tolerance is exact equality of the float bits
        assert np.array_equal(_bits(a), _bits(b)), f"call {call}: noalloc differs from sg_push_spikes"
        assert np.array_equal(_bits(b), _bits(ring_cpu)), f"call {call}: noalloc differs from the oracle"
    assert not np.array_equal(ring_new.cpu().numpy(), ring0)


def _max_network(extra):
    """4096 neurons, every one active with 256 synapses: exactly MAX_EVENTS
    events (plus `extra` more synapses on neuron 0)."""
    rng = np.random.default_rng(21)
    n, deg = 4096, 256
    counts = np.full(n, deg, np.int64)
    counts[0] += extra
    row_ptr = np.zeros(n + 1, np.uint32)
    row_ptr[1:] = np.cumsum(counts)
    e = int(row_ptr[-1])
    col = rng.integers(0, n, e).astype(np.uint32)
    w = (rng.standard_normal(e) * 2.3).astype(np.float32)
    d = rng.integers(0, 32, e).astype(np.uint8)
    active = np.arange(n, dtype=np.uint32)
    ring = (rng.standard_normal((32, n)) * 3).astype(np.float32)
    return row_ptr, col, w, d, active, ring


def test_noalloc_at_exactly_the_maximum_matches_the_oracle():
    import torch
    from simuse_b200 import _lib
    row_ptr, col, w, d, active, ring0 = _max_network(0)
    assert int(row_ptr[-1]) == MAX_EVENTS
    n = active.size
    bufs = dict(rp=_dev(row_ptr), col=_dev(col), w=_dev(w), d=_dev(d), a=_dev(active))
    ring = torch.from_numpy(ring0.copy()).to("cuda:0")
    ring_cpu = ring0.copy()
    for step in (40, 41):
        _lib.check(_call("sg_push_spikes_noalloc", bufs, n, n, step, ring))
        O.push_spikes(row_ptr, col, w, d, n, active, step, ring_cpu)
        torch.cuda.synchronize()
        assert np.array_equal(_bits(ring.cpu().numpy()), _bits(ring_cpu)), f"step {step}"


def test_noalloc_rejects_sizes_beyond_its_maximum():
    import torch
    from simuse_b200 import _lib
    # one event more than the maximum
    row_ptr, col, w, d, active, ring0 = _max_network(1)
    assert int(row_ptr[-1]) == MAX_EVENTS + 1
    n = active.size
    bufs = dict(rp=_dev(row_ptr), col=_dev(col), w=_dev(w), d=_dev(d), a=_dev(active))
    ring = torch.from_numpy(ring0.copy()).to("cuda:0")
    rc = _call("sg_push_spikes_noalloc", bufs, n, n, 0, ring)
    assert rc == -5
    assert "exceed the maximum" in _lib.last_error()
    torch.cuda.synchronize()
    assert np.array_equal(_bits(ring.cpu().numpy()), _bits(ring0))  # untouched
    # too many neurons
    rc = _call("sg_push_spikes_noalloc", bufs, MAX_NEURONS + 1, 1, 0, ring)
    assert rc == -1
    assert "exceeds the maximum" in _lib.last_error()


def test_noalloc_rejects_indices_outside_the_neurons():
    import torch
    from simuse_b200 import _lib
    row_ptr, col, w, d, active, ring0 = _network(2000, 20, 14)
    for what in ("col", "active"):
        c, a = col.copy(), active.copy()
        if what == "col":
            c[row_ptr[a[0]]] = 2000  # first synapse of the first active row
        else:
            a[-1] = 2000
        bufs = dict(rp=_dev(row_ptr), col=_dev(c), w=_dev(w), d=_dev(d), a=_dev(a))
        ring = torch.from_numpy(ring0.copy()).to("cuda:0")
        for fn in ("sg_push_spikes_noalloc", "sg_push_spikes"):
            rc = _call(fn, bufs, 2000, a.size, 3, ring)
            assert rc == -1, (what, fn)
            assert ">= n_neurons" in _lib.last_error()
        torch.cuda.synchronize()
        assert np.array_equal(_bits(ring.cpu().numpy()), _bits(ring0)), what


def test_noalloc_allocates_no_device_memory():
    import torch
    from simuse_b200 import _lib
    row_ptr, col, w, d, active, ring0 = _network(3000, 30, 15)
    bufs = dict(rp=_dev(row_ptr), col=_dev(col), w=_dev(w), d=_dev(d), a=_dev(active))
    empty = dict(bufs, a=_dev(np.zeros(1, np.uint32)))
    ring = torch.from_numpy(ring0.copy()).to("cuda:0")
    _lib.check(_call("sg_push_spikes_noalloc", bufs, 3000, active.size, 1, ring))  # warm: module loaded
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for step in range(2, 6):
        _lib.check(_call("sg_push_spikes_noalloc", bufs, 3000, active.size, step, ring))
        _lib.check(_call("sg_push_spikes_noalloc", empty, 3000, 0, step, ring))  # empty active list
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0
