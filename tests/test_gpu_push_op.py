"""The stand-alone push_spikes operator (sg_push_spikes, device buffers)
against the oracle's push_spikes (P/api/net/push.rs:126-173): bit-identical
rings, including cells hit by many pres with random float weights."""
import ctypes

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def random_csr(n, deg, seed, max_delay=31, hub=False):
    rng = np.random.default_rng(seed)
    counts = rng.integers(0, 2 * deg + 1, n)
    row_ptr = np.zeros(n + 1, np.uint32)
    row_ptr[1:] = np.cumsum(counts)
    e = int(row_ptr[-1])
    if hub:  # many synapses converge on a few posts: long per-cell chains
        col = rng.integers(0, 8, e).astype(np.uint32)
    else:
        col = rng.integers(0, n, e).astype(np.uint32)
    w = (rng.standard_normal(e) * 3.7).astype(np.float32)
    d = rng.integers(0, max_delay + 1, e).astype(np.uint8)
    return row_ptr, col, w, d


def run_gpu(fn_name, row_ptr, col, w, d, n, active, step, ring0):
    import torch
    from simuse_b200 import _lib
    dev = "cuda:0"
    t = {k: torch.from_numpy(v.view(np.int32) if v.dtype == np.uint32 else v).to(dev)
         for k, v in dict(rp=row_ptr, col=col, w=w, d=d, a=active).items()}
    ring = torch.from_numpy(ring0.copy()).to(dev)
    torch.cuda.synchronize()
    fn = getattr(_lib.lib(), fn_name)
    rc = fn(ctypes.c_void_p(t["rp"].data_ptr()), ctypes.c_void_p(t["col"].data_ptr()),
            ctypes.c_void_p(t["w"].data_ptr()), ctypes.c_void_p(t["d"].data_ptr()), n,
            ctypes.c_void_p(t["a"].data_ptr() if active.size else 0), active.size, step,
            ctypes.c_void_p(ring.data_ptr()), None)
    _lib.check(rc)
    torch.cuda.synchronize()
    return ring.cpu().numpy()


@pytest.mark.parametrize("n,deg,frac,seed,hub", [
    (1, 3, 1.0, 1, False), (100, 20, 0.5, 2, False), (5000, 40, 0.1, 3, False),
    (70000, 30, 0.02, 4, False), (300, 50, 0.8, 5, True)])
def test_push_spikes_bit_identical(n, deg, frac, seed, hub):
    row_ptr, col, w, d = random_csr(n, deg, seed, hub=hub)
    rng = np.random.default_rng(seed + 100)
    active = np.flatnonzero(rng.random(n) < frac).astype(np.uint32)
    ring0 = (rng.standard_normal((32, n)) * 2).astype(np.float32)
    for step in (0, 7, 31, 12345):
        exp = O.push_spikes(row_ptr, col, w, d, n, active, step, ring0.copy())
        got = run_gpu("sg_push_spikes", row_ptr, col, w, d, n, active, step, ring0)
        assert np.array_equal(got.view(np.uint32), exp.view(np.uint32)), step


def test_push_spikes_empty_active_leaves_ring():
    row_ptr, col, w, d = random_csr(64, 4, 9)
    ring0 = np.ones((32, 64), np.float32)
    got = run_gpu("sg_push_spikes", row_ptr, col, w, d, 64, np.zeros(0, np.uint32), 3, ring0)
    assert np.array_equal(got, ring0)


def test_push_spikes_reference_cases():
    # the reference's own push unit cases (P/api/net/push.rs:300-499)
    import scenarios as S
    for case in S.PINS["push"]["cases"]:
        n = case["n"]
        frm = np.array(case["from"], np.uint32)
        order = np.argsort(frm, kind="stable")
        counts = np.bincount(frm, minlength=n)
        row_ptr = np.zeros(n + 1, np.uint32)
        row_ptr[1:] = np.cumsum(counts)
        col = np.array(case["to"], np.uint32)[order]
        w = np.array(case["w"], np.float32)[order]
        d = np.array(case["d"], np.uint8)[order]
        got = run_gpu("sg_push_spikes", row_ptr, col, w, d, n, np.array(case["active"], np.uint32),
                      case["step"], np.zeros((32, n), np.float32))
        exp = np.zeros((32, n), np.float32)
        for slot, post, val in case["expect"]:
            exp[slot, post] += val
        assert np.array_equal(got, exp), case["name"]
