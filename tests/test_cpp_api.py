"""The C++ mirror (include/simuse_b200.hpp) compiles and links against the
library (CPU), and on a GPU gives the same run as the Python mirror."""
import os
import subprocess

import numpy as np
import pytest

import cpp_build
import simuse_b200 as sg


def test_cpp_mirror_compiles_and_links():
    exe = cpp_build.build("izh_pulse")
    assert os.path.exists(exe)


def _python_twin(steps):
    n, k = 400, 30
    pre, post, w, d = [], [], [], []
    h = 12345
    for i in range(n):
        for _ in range(k):
            h = (h * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
            pre.append(i)
            post.append((h >> 33) % n)
            w.append(0.5 if i < n * 4 // 5 else -1.0)
            d.append(1 + (h >> 60) % 4)
    net = sg.Network(0)
    p = net.add_population(sg.IZH, n)
    for c, v in enumerate([0.5, 0.02, 0.2, -65.0, 8.0, 0.0, 30.0]):
        net.fill_param(p, c, v)
    net.fill_state(p, 0, -65.0)
    net.fill_state(p, 1, -13.0)
    net.connect(p, pre, p, post, w, d)
    net.build()
    idx = np.arange(n, dtype=np.uint32)
    cur = (np.float32(4.0) + np.float32(0.02) * (np.arange(n) % 50).astype(np.float32)).astype(np.float32)
    counts = []
    for _ in range(steps):
        net.inject_current(p, idx, cur)
        net.step(1)
        counts.append(int(net.spikes(p).sum()))
    return counts, net.state(p, 0)


@pytest.mark.gpu
def test_cpp_mirror_runs_like_python_mirror():
    exe = cpp_build.build("izh_pulse")
    out = subprocess.run([exe, "200"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    vals = out.stdout.split()
    counts = [int(x) for x in vals[:200]]
    v = np.array([float(x) for x in vals[200:]], np.float32)
    c2, v2 = _python_twin(200)
    assert sum(counts) > 50
    assert counts == c2
    assert np.array_equal(v, v2)
