"""sg_push_spikes_noalloc — the push operator for callers that cannot allocate
device memory (a capture-only host loop, a real-time caller, a fixed memory
budget): it keeps its scratch in a fixed file-scope device array.

Checks, through the C ABI, that two calls in a row give exactly the rings
that the allocating sg_push_spikes gives on the same inputs, and that inputs
beyond the stated maxima are rejected without touching the ring.  This file
is collected last so that a run stopping at the first failure has already
run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

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


@pytest.mark.parametrize("n,deg,seed,hub", [(3000, 30, 11, False), (400, 60, 12, True), (50000, 8, 13, False)])
def test_noalloc_matches_allocating_push_two_calls(n, deg, seed, hub):
    import torch
    from simuse_b200 import _lib
    row_ptr, col, w, d, active, ring0 = _network(n, deg, seed, hub)
    bufs = dict(rp=_dev(row_ptr), col=_dev(col), w=_dev(w), d=_dev(d), a=_dev(active))
    ring_ref = torch.from_numpy(ring0.copy()).to("cuda:0")
    ring_new = torch.from_numpy(ring0.copy()).to("cuda:0")
    for call, step in enumerate((5, 6)):  # two calls in a row on the same rings
        _lib.check(_call("sg_push_spikes", bufs, n, active.size, step, ring_ref))
        _lib.check(_call("sg_push_spikes_noalloc", bufs, n, active.size, step, ring_new))
        torch.cuda.synchronize()
        a = ring_ref.cpu().numpy()
        b = ring_new.cpu().numpy()
        # the push tests' tolerance is exact equality of the float bits
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f"call {call}"
    assert not np.array_equal(ring_new.cpu().numpy(), ring0)


def test_noalloc_rejects_sizes_beyond_its_maximum():
    import torch
    from simuse_b200 import _lib
    # too many events for the fixed scratch: one neuron with MAX_EVENTS+1 synapses
    n = 64
    e = MAX_EVENTS + 1
    row_ptr = np.zeros(n + 1, np.uint32)
    row_ptr[1:] = e
    col = np.zeros(e, np.uint32)
    w = np.ones(e, np.float32)
    d = np.ones(e, np.uint8)
    active = np.array([0], np.uint32)
    bufs = dict(rp=_dev(row_ptr), col=_dev(col), w=_dev(w), d=_dev(d), a=_dev(active))
    ring = torch.zeros((32, n), dtype=torch.float32, device="cuda:0")
    rc = _call("sg_push_spikes_noalloc", bufs, n, 1, 0, ring)
    assert rc == -5
    assert "exceed the maximum" in _lib.last_error()
    torch.cuda.synchronize()
    assert float(ring.abs().sum()) == 0.0  # untouched
    # too many neurons
    rc = _call("sg_push_spikes_noalloc", bufs, MAX_NEURONS + 1, 1, 0, ring)
    assert rc == -1
    assert "exceeds the maximum" in _lib.last_error()
