"""Seeded synthetic workloads (the benchmark configurations).

Every random number comes from a counter-based SplitMix64 hash, so the same
seed gives the same network on any machine and in any build order; the
arrays produced here feed both the GPU ``Network`` and, in tests, the CPU
oracle (which exposes the same builder method names).

* ``izhikevich_pulse`` — the plain Izhikevich pulse-coupled network: N=1000,
  800 excitatory (a=0.02, b=0.2, c=-65+15r^2, d=8-6r^2) and 200 inhibitory
  (a=0.02+0.08r, b=0.25-0.05r, c=-65, d=2), 100 distinct random targets per
  neuron without self-loops, weights 0.5U (exc) / -U (inh), delay 1, dt=1 ms
  as two 0.5 ms half-steps, thalamic input 5N(0,1) / 2N(0,1) per step fed by
  inject_current, v0=-65, u0=b*v0, seed 0.
* ``lif_balanced`` — the balanced current-based LIF network: N neurons (80 %
  excitatory), tau_m=20 ms, V_th=20 mV, V_reset=10 mV, refractory 2 ms,
  dt=0.1 ms, fixed in-degree K with uniformly drawn presynaptic sources,
  weights J / -gJ (g=5), delays uniform in 1..20 steps, one Poisson source
  per neuron.  The reference LIF integrates dv = (v_rest - v + I)*dt/tau, so
  a PSP of J mV needs a ring weight of J*tau/dt: J=0.1 mV -> 20, -gJ -> -100.
"""
from __future__ import annotations

import numpy as np

PHI = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(z):
    """Vectorised SplitMix64 finaliser (uint64 in, uint64 out)."""
    z = np.asarray(z, np.uint64)
    with np.errstate(over="ignore"):
        z = z + PHI
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform01(seed: int, stream: int, counter) -> np.ndarray:
    """U[0,1) doubles for (seed, stream, counter) with 53 random bits."""
    c = np.asarray(counter, np.uint64)
    with np.errstate(over="ignore"):
        key = (np.uint64(seed) * PHI) ^ (np.uint64(stream) << np.uint64(40)) ^ c
    h = splitmix64(splitmix64(key))
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def std_normal(seed: int, stream: int, counter) -> np.ndarray:
    """Box-Muller N(0,1) in FP64 from two uniform draws per value."""
    c = np.asarray(counter, np.uint64)
    u1 = 1.0 - uniform01(seed, stream, c * np.uint64(2))  # (0, 1]
    u2 = uniform01(seed, stream, c * np.uint64(2) + np.uint64(1))
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


# ---------------------------------------------------------------------------
# Izhikevich pulse-coupled network
# ---------------------------------------------------------------------------
IZH_STREAM_R, IZH_STREAM_TARGETS, IZH_STREAM_W, IZH_STREAM_NOISE = 1, 2, 3, 4


def izhikevich_pulse(n: int = 1000, n_exc: int | None = None, k_out: int = 100,
                     steps: int = 1000, seed: int = 0, noise: bool = True) -> dict:
    if n_exc is None:
        n_exc = n * 4 // 5
    idx = np.arange(n, dtype=np.uint64)
    r = uniform01(seed, IZH_STREAM_R, idx)
    exc = np.arange(n) < n_exc
    a = np.where(exc, 0.02, 0.02 + 0.08 * r).astype(np.float32)
    b = np.where(exc, 0.2, 0.25 - 0.05 * r).astype(np.float32)
    c = np.where(exc, -65.0 + 15.0 * r * r, -65.0).astype(np.float32)
    d = np.where(exc, 8.0 - 6.0 * r * r, 2.0).astype(np.float32)
    v0 = np.full(n, -65.0, np.float32)
    u0 = (b * v0).astype(np.float32)
    # 100 distinct targets per pre, no self-loop: partial Fisher-Yates over the
    # other n-1 neurons driven by the hash stream of that pre.
    k = min(k_out, n - 1)
    pre = np.repeat(np.arange(n, dtype=np.uint32), k)
    post = np.empty(n * k, np.uint32)
    for i in range(n):
        pool = np.concatenate([np.arange(0, i), np.arange(i + 1, n)]).astype(np.uint32)
        u = uniform01(seed, IZH_STREAM_TARGETS, np.arange(k, dtype=np.uint64) + np.uint64(i * k))
        m = pool.size
        for j in range(k):
            s = j + int(u[j] * (m - j))
            pool[j], pool[s] = pool[s], pool[j]
        post[i * k:(i + 1) * k] = pool[:k]
    uw = uniform01(seed, IZH_STREAM_W, np.arange(n * k, dtype=np.uint64))
    w = np.where(exc[pre], 0.5 * uw, -uw).astype(np.float32)
    delay = np.ones(n * k, np.uint8)
    spec = dict(n=n, n_exc=n_exc, a=a, b=b, c=c, d=d, v0=v0, u0=u0, pre=pre, post=post, w=w,
                delay=delay, steps=steps, seed=seed, noise=noise)
    return spec


def izhikevich_input(spec: dict, step: int) -> np.ndarray:
    """Thalamic input of one step: 5N(0,1) excitatory, 2N(0,1) inhibitory (f32)."""
    n = spec["n"]
    if not spec["noise"]:
        return np.zeros(n, np.float32)
    ctr = np.arange(n, dtype=np.uint64) + np.uint64(step) * np.uint64(n)
    z = std_normal(spec["seed"], IZH_STREAM_NOISE, ctr)
    scale = np.where(np.arange(n) < spec["n_exc"], 5.0, 2.0)
    return (scale * z).astype(np.float32)


def outdegree_delays(h: np.ndarray, d_min: int, d_max: int) -> np.ndarray:
    """Delays of the out-degree generators from each draw's hash h."""
    span = d_max - d_min + 1
    if span <= 1:
        return np.full(h.shape, d_min, np.uint8)
    return (d_min + (splitmix64(h) & np.uint64(0xFFFFFFFF)) % np.uint64(span)).astype(np.uint8)


def _uniform_w(h, random_w) -> np.ndarray:
    """The U of a weight draw from the low 32 bits of hash h (f32)."""
    lo = h & np.uint64(0xFFFFFFFF)
    if random_w is True or int(random_w) == 1:
        return lo.astype(np.float32) * np.float32(2.3283064365386963e-10)
    b = int(random_w)
    return (lo >> np.uint64(32 - b)).astype(np.float32) * np.float32(2.0 ** -b)


def fixed_outdegree_edges(n: int, k: int, seed: int, n_exc: int, w_exc: float, w_inh: float,
                          no_self: bool = True, random_w=True):
    """NumPy twin of the device generator sg_connect_fixed_outdegree (same
    hash, same Floyd draws, same (source, draw) edge order).  random_w as
    there: False, True (U = lo32 / 2^32) or b in 2..24 (U on the 2^-b grid,
    the top b bits of lo32)."""
    m = n - (1 if no_self else 0)
    i = np.arange(n, dtype=np.uint64)
    sel = np.empty((n, k), np.uint64)
    w = np.empty((n, k), np.float32)
    scale = np.where(np.arange(n) < n_exc, np.float32(w_exc), np.float32(w_inh)).astype(np.float32)
    with np.errstate(over="ignore"):
        for q in range(k):
            j = np.uint64(m - k + q)
            h = splitmix64(np.uint64(seed) ^ ((i * np.uint64(k) + np.uint64(q)) * PHI))
            t = ((h >> np.uint64(32)) * (j + np.uint64(1))) >> np.uint64(32)
            if q:
                dup = (sel[:, :q] == t[:, None]).any(axis=1)
                t = np.where(dup, j, t)
            sel[:, q] = t
            w[:, q] = scale * _uniform_w(h, random_w) if random_w else scale
    tgt = sel.copy()
    if no_self:
        tgt = np.where(tgt >= i[:, None], tgt + np.uint64(1), tgt)
    pre = np.repeat(np.arange(n, dtype=np.uint32), k)
    return pre, tgt.astype(np.uint32).ravel(), w.ravel()


def fixed_outdegree_delays(n: int, k: int, seed: int, d_min: int, d_max: int) -> np.ndarray:
    """Delays the device generator draws for fixed_outdegree_edges' edges."""
    ctr = np.arange(n * k, dtype=np.uint64)
    with np.errstate(over="ignore"):
        h = splitmix64(np.uint64(seed) ^ (ctr * PHI))
    return outdegree_delays(h, d_min, d_max)


def lognormal_degrees(n: int, mean: float, sd: float, seed: int, kmax: int) -> np.ndarray:
    """Per-source degrees of sg_connect_lognormal_outdegree (stream 7)."""
    s2 = np.log(1.0 + (sd * sd) / (mean * mean))
    mu, sigma = np.log(mean) - 0.5 * s2, np.sqrt(s2)
    z = std_normal(seed, 7, np.arange(n, dtype=np.uint64))
    return np.clip(np.rint(np.exp(mu + sigma * z)), 1, kmax).astype(np.int64)


def lognormal_outdegree_edges(n: int, mean: float, sd: float, seed: int, n_exc: int, w_exc: float,
                              w_inh: float, no_self: bool = True, random_w=True):
    """NumPy twin of sg_connect_lognormal_outdegree (small n: loops per
    source); random_w as for fixed_outdegree_edges."""
    m = n - (1 if no_self else 0)
    deg = lognormal_degrees(n, mean, sd, seed, min(m, 4096))
    off = np.concatenate([[0], np.cumsum(deg)])
    pre = np.repeat(np.arange(n, dtype=np.uint32), deg)
    post = np.empty(off[-1], np.uint32)
    w = np.empty(off[-1], np.float32)
    with np.errstate(over="ignore"):
        for i in range(n):
            k = int(deg[i])
            ctr = np.arange(off[i], off[i] + k, dtype=np.uint64)
            h = splitmix64(np.uint64(seed) ^ (ctr * PHI))
            sel = []
            for q in range(k):
                j = m - k + q
                t = int((int(h[q]) >> 32) * (j + 1) >> 32)
                if t in sel:
                    t = j
                sel.append(t)
            tt = np.array(sel, np.int64)
            if no_self:
                tt = np.where(tt >= i, tt + 1, tt)
            post[off[i]:off[i + 1]] = tt
            scale = np.float32(w_exc if i < n_exc else w_inh)
            w[off[i]:off[i + 1]] = scale * _uniform_w(h, random_w) if random_w else scale
    return pre, post, w


def izhikevich_params(n: int, n_exc: int, seed: int):
    """Per-neuron a, b, c, d of the pulse-network recipe (r ~ U(0,1) per neuron)."""
    r = uniform01(seed, IZH_STREAM_R, np.arange(n, dtype=np.uint64))
    exc = np.arange(n) < n_exc
    a = np.where(exc, 0.02, 0.02 + 0.08 * r).astype(np.float32)
    b = np.where(exc, 0.2, 0.25 - 0.05 * r).astype(np.float32)
    c = np.where(exc, -65.0 + 15.0 * r * r, -65.0).astype(np.float32)
    d = np.where(exc, 8.0 - 6.0 * r * r, 2.0).astype(np.float32)
    return a, b, c, d


def add_izhikevich_instance(net, n: int, seed: int, k_out: int = 100, device_edges: bool = True,
                            device_noise: bool = True, model_izh: int = 2, random_w=True) -> int:
    """One pulse-coupled Izhikevich network (the recipe of izhikevich_pulse,
    with the fixed-out-degree generator for its 100 distinct targets) added
    to `net` as its own population; several calls build a batch that steps
    as one network.  Device noise draws the thalamic input of
    izhikevich_input on the GPU (same hash, counter i + step * n).
    random_w = 8 draws the weights' U on the 1/256 grid (exact ring sums)."""
    n_exc = n * 4 // 5
    a, b, c, d = izhikevich_params(n, n_exc, seed)
    pop = net.add_population(model_izh, n)
    net.fill_param(pop, 0, 1.0)
    net.set_param(pop, 1, a)
    net.set_param(pop, 2, b)
    net.set_param(pop, 3, c)
    net.set_param(pop, 4, d)
    net.fill_param(pop, 5, 0.0)
    net.fill_param(pop, 6, 30.0)
    net.fill_state(pop, 0, -65.0)
    net.set_state(pop, 1, (b * np.float32(-65.0)).astype(np.float32))
    k = min(k_out, n - 1)
    if device_edges:
        net.connect_fixed_outdegree(pop, pop, k, seed, True, n_exc, 0.5, -1.0, random_w, 1)
    else:
        pre, post, w = fixed_outdegree_edges(n, k, seed, n_exc, 0.5, -1.0, random_w=random_w)
        net.connect(pop, pre, pop, post, w, np.ones(pre.size, np.uint8))
    if device_noise:
        net.set_noise(pop, seed, 5.0, 2.0, split=n_exc, stream=IZH_STREAM_NOISE, stride=n)
    return pop


def thalamic_input(n: int, seed: int, step: int) -> np.ndarray:
    """Host form of the device noise of add_izhikevich_instance (f32)."""
    n_exc = n * 4 // 5
    ctr = np.arange(n, dtype=np.uint64) + np.uint64(step) * np.uint64(n)
    z = std_normal(seed, IZH_STREAM_NOISE, ctr)
    return (np.where(np.arange(n) < n_exc, 5.0, 2.0) * z).astype(np.float32)


def build_izhikevich(net, spec: dict, model_izh: int = 2) -> int:
    """Apply the spec through the reference builder API; returns the population."""
    n = spec["n"]
    pop = net.add_population(model_izh, n)
    net.fill_param(pop, 0, 1.0)   # dt
    net.set_param(pop, 1, spec["a"])
    net.set_param(pop, 2, spec["b"])
    net.set_param(pop, 3, spec["c"])
    net.set_param(pop, 4, spec["d"])
    net.fill_param(pop, 5, 0.0)   # tau_ref: none
    net.fill_param(pop, 6, 30.0)  # v_thresh
    net.set_state(pop, 0, spec["v0"])
    net.set_state(pop, 1, spec["u0"])
    net.connect(pop, spec["pre"], pop, spec["post"], spec["w"], spec["delay"])
    net.build()
    return pop


def run_izhikevich(net, pop: int, spec: dict, steps: int | None = None, start: int = 0):
    """Drive the network step by step (inject then step); returns spike counts per step."""
    n = spec["n"]
    idx = np.arange(n, dtype=np.uint32)
    steps = spec["steps"] if steps is None else steps
    for t in range(start, start + steps):
        net.inject_current(pop, idx, izhikevich_input(spec, t))
        net.step(1)


# ---------------------------------------------------------------------------
# balanced LIF network
# ---------------------------------------------------------------------------
LIF_STREAM_V0 = 5


def fixed_indegree_edges(n_from: int, n_post: int, k_in: int, seed: int, n_exc: int,
                         w_exc: float, w_inh: float, d_min: int, d_max: int,
                         from_off: int = 0, to_off: int = 0):
    """numpy restatement of the device generator of sg_connect_fixed_indegree
    (edge t = (post j, draw q) = j*k_in + q, in that order)."""
    t = np.arange(n_post * k_in, dtype=np.uint64)
    with np.errstate(over="ignore"):
        h = splitmix64(np.uint64(seed) ^ (t * PHI))
    src = (((h >> np.uint64(32)) * np.uint64(n_from)) >> np.uint64(32)).astype(np.uint32)
    span = np.uint64(d_max - d_min + 1)
    d = (np.uint64(d_min) + (h & np.uint64(0xFFFFFFFF)) % span).astype(np.uint8)
    post = (t // np.uint64(k_in)).astype(np.uint32)
    exc = src < n_exc
    w = np.where(exc, np.float32(w_exc), np.float32(w_inh)).astype(np.float32)
    return src + np.uint32(from_off), post + np.uint32(to_off), w, d


def lif_balanced(n: int = 1_000_000, k_in: int = 1000, seed: int = 1, ext_rate_hz: float = 2000.0,
                 ext_weight: float = 20.0, w_exc: float = 20.0, g: float = 5.0,
                 d_min: int = 1, d_max: int = 20) -> dict:
    """The balanced LIF network; the literal configuration is the default
    (external Poisson 2000 Hz with weight J)."""
    n_exc = n * 4 // 5
    v0 = (10.0 + 10.0 * uniform01(seed, LIF_STREAM_V0, np.arange(n, dtype=np.uint64))).astype(np.float32)
    return dict(n=n, n_exc=n_exc, k_in=k_in, seed=seed, ext_rate_hz=ext_rate_hz,
                ext_weight=ext_weight, w_exc=w_exc, w_inh=-g * w_exc, d_min=d_min, d_max=d_max,
                dt=0.1, v0=v0)


LIF_PARAMS = (0.1, 0.05, 0.0, 20.0, 10.0, 2.0)  # dt inv_tau v_rest v_th v_reset tau_ref


def build_lif(net, spec: dict, model_lif: int = 1, device_generator: bool = True) -> int:
    """Apply the LIF spec; the GPU network generates its synapses on the
    device, the oracle receives the identical numpy-generated edge list."""
    n = spec["n"]
    pop = net.add_population(model_lif, n)
    for col, v in enumerate(LIF_PARAMS):
        net.fill_param(pop, col, v)
    net.set_state(pop, 0, spec["v0"])
    if device_generator:
        net.connect_fixed_indegree(pop, pop, spec["k_in"], spec["seed"], spec["n_exc"],
                                   spec["w_exc"], spec["w_inh"], spec["d_min"], spec["d_max"])
    else:
        pre, post, w, d = fixed_indegree_edges(n, n, spec["k_in"], spec["seed"], spec["n_exc"],
                                               spec["w_exc"], spec["w_inh"], spec["d_min"],
                                               spec["d_max"])
        net.connect(pop, pre, pop, post, w, d)
    # one Poisson source per neuron, seed = neuron index, delay 1
    if hasattr(net, "add_poisson_sources"):
        first = net.add_poisson_sources(n, spec["ext_rate_hz"], spec["dt"], seed0=0)
        net.connect_poisson_one_to_one(first, n, pop, spec["ext_weight"], 1)
    else:
        ones_w = np.array([spec["ext_weight"]], np.float32)
        one_d = np.array([1], np.uint8)
        for i in range(n):
            s = net.add_poisson_source(spec["ext_rate_hz"], spec["dt"], i)
            net.connect_poisson_source(s, pop, np.array([i], np.uint32), ones_w, one_d)
    return pop


# ---------------------------------------------------------------------------
# Kuramoto sweep (the oscillator half of the batched uneven sweep)
# ---------------------------------------------------------------------------
def izh_sweep_sizes(n_inst: int = 1024, n_min: int = 500, n_max: int = 200_000, seed: int = 7) -> np.ndarray:
    """Sizes of the sweep's Izhikevich instances: N log-uniform in [n_min, n_max]."""
    u = uniform01(seed, 1, np.arange(n_inst, dtype=np.uint64))
    return np.floor(np.exp(np.log(n_min) + u * (np.log(n_max + 1) - np.log(n_min)))).astype(np.int64)


def kuramoto_sweep(n_inst: int = 1024, n_min: int = 256, n_max: int = 65536, k_max: float = 4.0,
                   gamma: float = 0.5, seed: int = 0) -> dict:
    """``n_inst`` all-to-all Kuramoto populations: N log-uniform in
    [n_min, n_max], coupling K linearly from 0 to k_max over the instances,
    theta0 ~ U(-pi, pi), omega ~ Lorentzian(0, gamma) by the inverse CDF
    gamma*tan(pi*(u - 1/2)) in FP64, rounded to FP32."""
    i = np.arange(n_inst, dtype=np.uint64)
    u = uniform01(seed, 1, i)
    sizes = np.floor(np.exp(np.log(n_min) + u * (np.log(n_max + 1) - np.log(n_min)))).astype(np.int64)
    sizes = np.clip(sizes, n_min, n_max).astype(np.uint32)
    coupling = (np.linspace(0.0, k_max, n_inst) if n_inst > 1 else np.zeros(1)).astype(np.float32)
    total = int(sizes.astype(np.int64).sum())
    j = np.arange(total, dtype=np.uint64)
    theta = ((uniform01(seed, 2, j) * 2.0 - 1.0) * np.pi).astype(np.float32)
    uo = uniform01(seed, 3, j)
    uo = np.clip(uo, 1e-12, 1.0 - 1e-12)
    omega = (gamma * np.tan(np.pi * (uo - 0.5))).astype(np.float32)
    return dict(sizes=sizes, coupling=coupling, theta=theta, omega=omega, dt=0.01, seed=seed)



# ---------------------------------------------------------------------------
# Hodgkin-Huxley network with conductance synapses and pair STDP
# ---------------------------------------------------------------------------
HH_STREAM_BIAS, HH_STREAM_V0 = 9, 10
HH_PARAMS = (0.01, 1.0, 120.0, 36.0, 0.3, 50.0, -77.0, -54.4)  # dt c_m g_na g_k g_l e_na e_k e_l


def add_hh_stdp(net, n: int = 100_000, seed: int = 3, mean_degree: float = 200.0, sd_degree: float = 80.0,
                d_min: int = 1, d_max: int = 20, w_max: float = 0.5, model_hh: int = 4, edges=None) -> int:
    """The HH + pair-STDP network: n squid-axon HH neurons (RK4, dt 0.01 ms),
    the first 80 % excitatory; conductance synapses with exponential decay
    tau 5 ms (E_rev 0 mV excitatory, -80 mV inhibitory); lognormal out-degree
    (mean 200, sd 80), distinct targets, weights U(0, w_max) (the stated
    w_max = 0.5, taken as a raw conductance per synapse as the reference's
    ExpOne ring does: the synchronous onset volley of 200 inputs leaves the
    neurons shunted and silent from then on; at w_max = 0.04 they stay silent
    for ~40 ms between population bursts; at w_max = 0.01 they fire
    irregularly at ~60 Hz), delays uniform in d_min..d_max steps; pair STDP on excitatory synapses (tau+ = tau- =
    20 ms, A+ 0.01, A- 0.0105, weights clipped to [0, 1]); bias current
    N(10, 2) per neuron; v0 ~ U(-70, -60) and the gates at rest."""
    n_exc = n * 4 // 5
    pop = net.add_population(model_hh, n)
    for col, v in enumerate(HH_PARAMS):
        net.fill_param(pop, col, v)
    idx = np.arange(n, dtype=np.uint64)
    net.set_param(pop, 8, (10.0 + 2.0 * std_normal(seed, HH_STREAM_BIAS, idx)).astype(np.float32))
    net.fill_param(pop, 9, 0.0)          # spike threshold (upward crossing)
    net.set_state(pop, 0, (-70.0 + 10.0 * uniform01(seed, HH_STREAM_V0, idx)).astype(np.float32))
    net.fill_state(pop, 1, 0.0529)
    net.fill_state(pop, 2, 0.5961)
    net.fill_state(pop, 3, 0.3177)
    ke = net.register_expone(5.0, 0.0, 0.01)
    ki = net.register_expone(5.0, -80.0, 0.01)
    net.stdp_config(0.01, 20.0, 20.0, 0.01, 0.0105, 0.0, 1.0)
    if edges is None:
        net.connect_lognormal_outdegree(pop, pop, mean_degree, sd_degree, seed, True, n_exc, w_max, w_max,
                                        random_w=True, delay=d_min, d_max=d_max, syn_type_exc=ke,
                                        syn_type_inh=ki, stdp_exc=True)
    else:
        # the same synapses as an explicit CSR (row_ptr, col, w, delay, syn type, STDP flag), e.g. a
        # device-generated network read back with graph() / graph_types()
        rp, col, w, d, st, pl = edges
        pre = np.repeat(np.arange(n, dtype=np.uint32), np.diff(rp.astype(np.int64)))
        for flag in (1, 0):
            sel = pl == flag
            net.connect(pop, pre[sel], pop, col[sel], w[sel], d[sel], syn_types=st[sel], stdp=bool(flag))
    return pop
