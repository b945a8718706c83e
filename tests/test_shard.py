"""Host side of a network split across GPUs (simuse_b200.shard).

No GPU: the partition is checked with a recording stand-in for the network
(pieces and device layout the same on every rank, every synapse on exactly
the rank of its post, connect order kept for repeated pairs), and the spike
exchange's addressing with two gloo ranks on CPU: each rank all-gathers its
bitmask words and reads every external piece's words from the gathered
buffer at the offsets the GPU exchange uses.  The split step itself runs
end to end on the oracle in two gloo processes (local update, all-gather
of the step's spikes, external spikes in, push) and must give the unsplit
network's rasters and membrane bits.
"""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from simuse_b200 import shard as SH


class FakeNet:
    def __init__(self):
        self.pops, self.edges = [], []

    def add_population(self, model, n):
        self.pops.append(("local", model, n))
        return len(self.pops) - 1

    def add_external_population(self, n):
        self.pops.append(("ext", 0, n))
        return len(self.pops) - 1

    def fill_param(self, *a):
        pass

    def set_param(self, *a):
        pass

    def fill_state(self, *a):
        pass

    def set_state(self, *a):
        pass

    def connect(self, fp, fi, tp, ti, w, d):
        self.edges.append((fp, fi.copy(), tp, ti.copy(), w.copy(), d.copy()))


def spec(seed=0, sizes=(700, 1300, 50), k=6):
    rng = np.random.default_rng(seed)
    N = sum(sizes)
    pre = np.repeat(np.arange(N), k).astype(np.uint32)
    post = rng.integers(0, N, pre.size).astype(np.uint32)
    rep = rng.integers(0, pre.size, 200)          # repeated (pre, post) pairs with different weights
    pre = np.concatenate([pre, pre[rep]])
    post = np.concatenate([post, post[rep]])
    w = rng.uniform(-5, 5, pre.size).astype(np.float32)
    d = rng.integers(1, 9, pre.size).astype(np.uint8)
    pops = [SH.PopSpec(1, n, {0: 0.5}, {0: -70.0}) for n in sizes]
    return SH.NetSpec(pops, pre, post, w, d)


@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_partition(world):
    sp = spec()
    shards = [SH.Shard(FakeNet(), sp, r, world) for r in range(world)]
    layouts = [[(kind == "ext", n) for kind, _, n in s.net.pops] for s in shards]
    sizes = [[n for _, n in L] for L in layouts]
    assert all(x == sizes[0] for x in sizes)                     # same device layout on every rank
    assert sum(sizes[0]) == sp.total
    for s in shards:                                             # each neuron simulated on exactly one rank
        assert sum(n for (ext, n) in [(k == "ext", n) for k, _, n in s.net.pops] if not ext) == s.hi - s.lo
    got = []
    for s in shards:
        for fp, fi, tp, ti, w, d in s.net.edges:
            g_pre = fi.astype(np.int64) + s.gstart[fp]
            g_post = ti.astype(np.int64) + s.gstart[tp]
            assert np.all((g_post >= s.lo) & (g_post < s.hi))
            assert s.net.pops[tp][0] == "local"
            got += list(zip(g_pre.tolist(), g_post.tolist(), w.tolist(), d.tolist()))
    want = list(zip(sp.pre.astype(np.int64).tolist(), sp.post.astype(np.int64).tolist(), sp.w.tolist(),
                    sp.d.tolist()))
    assert sorted(got) == sorted(want)
    # repeated (pre, post) pairs keep their connect order
    def by_pair(edges):
        out = {}
        for a, b, w_, _ in edges:
            out.setdefault((a, b), []).append(w_)
        return out
    assert by_pair(got) == by_pair(want)


def _rank(rank, world, port, q):
    try:
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        dist.init_process_group("gloo", rank=rank, world_size=world)
        import torch
        sp = spec(seed=3)
        sh = SH.Shard(FakeNet(), sp, rank, world)
        offs, words = sh.word_offsets()
        rng = np.random.default_rng(11)
        spikes = rng.random(sp.total) < 0.3                    # the same global spike vector on every rank
        local = np.zeros(words * 32, bool)
        for k, pid, g0, n in sh.local():
            local[offs[k] * 32: offs[k] * 32 + n] = spikes[g0:g0 + n]
        mine = torch.from_numpy(np.packbits(local, bitorder="little").view(np.int32).copy())
        gathered = [torch.zeros(words, dtype=torch.int32) for _ in range(world)]
        dist.all_gather(gathered, mine)
        buf = torch.stack(gathered).numpy().reshape(-1)
        ok = True
        for k, pid, qk in sh.external():
            g, _, a, b = sh.pieces[k]
            src = buf[qk * words + offs[k]: qk * words + offs[k] + -(-(b - a) // 32)]
            bits = np.unpackbits(src.view(np.uint8), bitorder="little")[: b - a].astype(bool)
            ok &= np.array_equal(bits, spikes[sh.gstart[k]: sh.gstart[k] + (b - a)])
        dist.destroy_process_group()
        q.put((rank, bool(ok), len(sh.external())))
    except Exception as e:  # reported to the parent
        q.put((rank, repr(e), -1))


def test_exchange_addressing_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
    assert all(r[1] is True for r in res), res
    assert all(r[2] > 0 for r in res)


def _oracle_spec(seed=4, sizes=(900, 400), k=30):
    rng = np.random.default_rng(seed)
    N = sum(sizes)
    pre = np.repeat(np.arange(N, dtype=np.uint32), k)
    post = rng.integers(0, N, pre.size).astype(np.uint32)
    w = rng.uniform(-20.0, 40.0, pre.size).astype(np.float32)
    d = rng.integers(1, 9, pre.size).astype(np.uint8)
    pops = [SH.PopSpec(1, sizes[0], dict(enumerate([0.5, 0.1, -70.0, -54.0, -70.0, 2.0])),
                       {0: rng.uniform(-70.0, -55.0, sizes[0]).astype(np.float32)}),
            SH.PopSpec(1, sizes[1], dict(enumerate([0.5, 0.2, -65.0, -52.0, -68.0, 1.0])),
                       {0: rng.uniform(-65.0, -53.0, sizes[1]).astype(np.float32)})]
    return SH.NetSpec(pops, pre, post, w, d)


STEPS = 200


def _split_rank(rank, world, port, q):
    """One rank of a split network on the oracle: local update, all-gather of
    this step's spikes over gloo, external spikes in, push."""
    try:
        import sys
        here = os.path.dirname(os.path.abspath(__file__))
        sys.path[:0] = [os.path.join(here, "..", "oracle"), os.path.join(here, "..", "dioma-core_b200")]
        import torch
        import oracle as O
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        dist.init_process_group("gloo", rank=rank, world_size=world)
        sp = _oracle_spec()
        net = O.Network(0)
        sh = SH.Shard(net, sp, rank, world)
        net.build()
        cur = np.random.default_rng(9).uniform(0.0, 60.0, (STEPS, sp.total)).astype(np.float32)
        raster = np.zeros((STEPS, sp.total), np.int32)
        for t in range(STEPS):
            sh.inject(cur[t])
            net.step_begin()
            mine = np.zeros(sp.total, np.int32)
            sh.spikes(mine)
            parts = [torch.zeros(sp.total, dtype=torch.int32) for _ in range(world)]
            dist.all_gather(parts, torch.from_numpy(mine))
            every = np.sum([p.numpy() for p in parts], axis=0)   # each neuron is set by its owner only
            for k, pid, _ in sh.external():
                g0, n = int(sh.gstart[k]), sh.pieces[k][3] - sh.pieces[k][2]
                net.set_external_spikes(pid, every[g0:g0 + n])
            net.step_end()
            raster[t] = every
        v = np.zeros(sp.total, np.float32)
        sh.state(0, v)
        dist.destroy_process_group()
        q.put((rank, raster, v))
    except Exception as e:  # reported to the parent
        import traceback
        q.put((rank, traceback.format_exc(), None))


def test_split_network_on_two_gloo_ranks_matches_the_unsplit_network():
    """The split step's semantics, end to end on CPU: two processes each
    simulate their slice on the oracle and exchange spikes over gloo every
    step; the rasters and the local membrane potentials equal the unsplit
    network's."""
    import oracle as O
    sp = _oracle_spec()
    net = O.Network(0)
    full = SH.Shard(net, sp, 0, 1)
    net.build()
    cur = np.random.default_rng(9).uniform(0.0, 60.0, (STEPS, sp.total)).astype(np.float32)
    r1 = np.zeros((STEPS, sp.total), np.int32)
    for t in range(STEPS):
        full.inject(cur[t])
        net.step(1)
        full.spikes(r1[t])
    v1 = np.zeros(sp.total, np.float32)
    full.state(0, v1)
    assert r1.sum() > 500
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() + 1) % 1000
    ps = [ctx.Process(target=_split_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted([q.get(timeout=300) for _ in ps], key=lambda x: x[0])
    for p in ps:
        p.join(timeout=60)
    for rank, raster, v in res:
        assert v is not None, raster
        assert np.array_equal(raster, r1), rank
        lo, hi = SH.slices(sp.total, 2)[rank]
        assert np.array_equal(v[lo:hi].view(np.uint32), v1[lo:hi].view(np.uint32))
