#!/usr/bin/env python
"""Headline benchmark: synaptic events/s of the SiMuse simulation step on a
balanced LIF network of 1,000,000 neurons and 1e9 synapses.

One bench "step" = `--sim-steps` simulation steps (default 1000 = 100 ms of
simulated time at dt = 0.1 ms) of the whole network: neuron update, spike
compaction, deterministic CSR scatter into the delay rings, Poisson drive.

Workloads (`--variant`):
  driven   external Poisson drive 4000 Hz x 0.5 mV (ring weight 100) per
           neuron; the network settles at ~34 Hz and the recurrent scatter
           carries ~3.8e6 synaptic events per step.  Headline.
  literal  the configuration as stated (2000 Hz x J = 0.1 mV): mean drive
           4 mV < threshold 20 mV, so the network is silent and only the
           2e5 Poisson events per step reach the rings.

Reported, one JSON line on rank 0:
  value   events/s over K bench steps, CUDA events on the network's stream
          (inputs resident in HBM; the 9 GB CSR exceeds L2 on every step).
  e2e     the same metric through the C ABI with host buffers: each bench
          step calls sg_step and then reads the step's spike raster back to
          pinned host memory (sg_raster_read_events), wall clock.
  roofline  dominant kernel: algorithmic bytes per launch / average launch
          time (CUDA events around each phase in a profiled pass of K bench
          steps) against MEASURED_PEAKS.json's copy bandwidth.
  cpu_baseline  the CPU restatement of the reference step (oracle/) on this
          host's cores, on a bounded sample of the same network.
  batched   (extra key) 64 uneven Izhikevich networks stepping as one batch
          against the same instances one at a time.
  serving   (extra key) Poisson streams of LIF / Izhikevich requests at
          5..200 requests/s through the continuous-batching server (pooled
          steps): served sims/s, p50/p99 latency, against the one-at-a-time
          loop on the same arrivals.
  sweep     (extra key) 1024 Kuramoto populations and 1024 Izhikevich
          networks (BF16) advancing concurrently: each half alone, both
          together, fixed against autotuned scatter schedule.
  precision_paths, hh_stdp_100k, kuramoto_sweep, lif_learn  (extra keys)
          BF16 / FP8 / ordered-path runs of the headline network, the 100k HH
          + STDP network, the Kuramoto sweep and learning.
`--impl reference` times that CPU path alone as the reference arm.
Multi-GPU (`--gpus N` under torchrun): each rank simulates its own replica
(seed + rank); no data-path collective (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dioma-core_b200"))

METRIC = "synaptic events/s"
UNIT = "events/s"

# algorithmic bytes: LIF neuron = v, refr read+write (16 B), ring slot read +
# clear (8 B), spike bit (1/8 B); per recurrent event col 4 + weight 4 +
# delay 1 and the ring read-modify-write 8; per spike the spike-list
# write+read and the row bounds (16 B).  The one-to-one Poisson drive is rolled
# in the neuron kernel from the neuron index (seed) and one rate: no bytes.
B_NEURON = 24.125
B_EVENT_EXPAND = 9.0
B_EVENT_APPLY = 8.0
B_SPIKE = 16.0
PARITY_STEPS = 200  # first simulation steps compared bit for bit with the oracle


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--variant", default="driven", choices=["driven", "literal"])
    ap.add_argument("--sim-steps", type=int, default=1000)
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--k-in", type=int, default=1000)
    ap.add_argument("--d-max", type=int, default=20, help="largest synaptic delay (steps) of the LIF network")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the batched and served measurements")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the scatter's fixed schedule (no sg_autotune before the timed steps)")
    ap.add_argument("--case", default="headline", choices=["headline", "kuramoto-sweep", "izh-batch", "hh-stdp",
                                                           "lif-learn", "taas", "sweep"],
                    help="headline: the JSON line above; the others time one workload alone (also the "
                         "profiling entry points)")
    ap.add_argument("--instances", type=int, default=1024,
                    help="instances of the kuramoto-sweep and izh-batch cases; the sweep case takes half of "
                         "each kind (2048: the 1024 + 1024 configuration)")
    ap.add_argument("--hh-wmax", type=float, default=0.01,
                    help="hh-stdp weights U(0, w_max) (raw conductance per synapse): the stated 0.5 "
                         "silences the network after its onset volley, 0.01 keeps it firing irregularly")
    ap.add_argument("--hh-steps", type=int, default=200_000,
                    help="hh-stdp simulation steps timed (200000 = the stated 2 s run at dt 0.01 ms)")
    ap.add_argument("--weights", default="fp32", choices=["fp32", "bf16"],
                    help="synapse weight storage (bf16: 6 B per synapse, FP32 accumulation)")
    ap.add_argument("--batch-instances", type=int, default=64)
    ap.add_argument("--serve-requests", type=int, default=100)
    return ap.parse_args(argv)


def parse_args_for_test(argv):
    return parse(argv)


def workload(args, rank=0):
    from simuse_b200 import workloads as W
    kw = (dict(ext_rate_hz=4000.0, ext_weight=100.0) if args.variant == "driven"
          else dict(ext_rate_hz=2000.0, ext_weight=20.0))
    spec = W.lif_balanced(n=args.n, k_in=args.k_in, seed=1 + rank, d_max=args.d_max, **kw)
    name = f"lif_balanced_{args.n // 1000}k_in{args.k_in}_{args.variant}"
    return spec, name


SCATTER_TEXT = {
    "exact": "exact-sum lists: the ring weights (20, -100, Poisson 100) are integers and no post's weights sum past "
             "2^23, so every FP32 partial sum is exact; the per-slot event lists are added in any order and give "
             "the reference's bits",
    "ordered": "ordered ring cells (reference summation order)",
    "atomic": "atomic adds (order not fixed)",
}


def config(args, name, spec, scatter_path="ordered"):
    return {
        "workload": name,
        "neurons": spec["n"],
        "synapses": spec["n"] * spec["k_in"],
        "dt_ms": spec["dt"],
        "sim_steps_per_bench_step": args.sim_steps,
        "external_drive": {"rate_hz": spec["ext_rate_hz"], "ring_weight": spec["ext_weight"]},
        "weights": args.weights,
        "scatter": SCATTER_TEXT[scatter_path],
        "l2": "inputs larger than L2: 8 GB of synapse records and "
              f"{(21 * spec['n'] * 4) / 1e6:.0f} MB of delay rings (21 slots for delays up to 20) against a "
              "126 MB L2; each step reads the spiking rows; the rings are kept in the L2 set-aside for "
              "persisting lines (at most 79 MiB on B200)",
        "parallelism": f"replicas x{args.gpus}",
    }


# ---------------------------------------------------------------------------
def cpu_baseline(args, spec, seconds):
    """The CPU restatement of the reference step on this host's cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    net = O.Network(0)
    pop = net.add_population(O.LIF, spec["n"])
    from simuse_b200.workloads import LIF_PARAMS
    for col, v in enumerate(LIF_PARAMS):
        net.fill_param(pop, col, v)
    net.set_state(pop, 0, spec["v0"])
    first = net.add_poisson_sources(spec["n"], spec["ext_rate_hz"], spec["dt"], seed0=0)
    net.connect_poisson_one_to_one(first, spec["n"], pop, spec["ext_weight"], 1)
    t0 = time.time()
    net.build_fixed_indegree(pop, pop, spec["k_in"], spec["seed"], spec["n_exc"], spec["w_exc"],
                             spec["w_inh"], spec["d_min"], spec["d_max"])
    build_s = time.time() - t0
    return net, cores, build_s


def run_cpu_parity(net, steps):
    """The oracle's first `steps` steps from the initial state, timed, with
    the raster recorded: (raster, events, seconds)."""
    ev0 = net.events
    t0 = time.perf_counter()
    rc = net.step(steps, record=True)
    return rc, net.events - ev0, time.perf_counter() - t0


def run_cpu_sample(net, seconds, min_steps=5, chunk=5):
    ev0 = net.events
    s0 = net.step_counter
    t0 = time.perf_counter()
    while True:
        net.step(chunk)
        el = time.perf_counter() - t0
        if el >= seconds and net.step_counter - s0 >= min_steps:
            break
    return net.events - ev0, net.step_counter - s0, el


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, nm in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def measured_peak():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def probe_red_rate(device, n_cells, iters=64):
    """Scattered 4-byte reductions per second this GPU completes into an
    n_cells-float array (sg_probe_red_rate), or None."""
    import ctypes as C

    from simuse_b200 import _lib
    r = C.c_double()
    rc = _lib.lib().sg_probe_red_rate(device, int(n_cells), iters, C.byref(r))
    return r.value if rc == 0 else None


def profiled_traffic(kernel):
    """DRAM bytes (read + write) per launch of `kernel` on the bench workload,
    from the committed ncu summary profiles/dram_traffic.txt (lines
    `<kernel> dram_bytes_per_launch=<bytes>`)."""
    import re
    try:
        for line in open(os.path.join(ROOT, "profiles", "dram_traffic.txt")):
            m = re.match(r"\s*(\S+)\s+dram_bytes_per_launch=([0-9.eE+]+)", line)
            if m and m.group(1) == kernel:
                return float(m.group(2))
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
def reduce_over_ranks(dist, device, t, events):
    """Job time = the slowest rank's time, job work = the sum over ranks
    (every rank takes these two collectives in the same order)."""
    if dist is None:
        return t, events
    import torch
    tt = torch.tensor([float(t)], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    ee = torch.tensor([float(events)], device=device, dtype=torch.float64)
    dist.all_reduce(ee, op=dist.ReduceOp.SUM)
    return float(tt.item()), float(ee.item())


def run_batched(args, local):
    """Many uneven Izhikevich networks (the pulse-network recipe, N log-uniform
    in 500..200,000, device-generated synapses and thalamic noise) stepping as
    one batch, against the same instances run one at a time."""
    import numpy as np
    import torch

    import simuse_b200 as sg
    from simuse_b200 import workloads as W
    K, steps = args.batch_instances, 1000
    sizes = W.izh_sweep_sizes(K)

    def timed(net, n_steps):
        st = torch.cuda.ExternalStream(net.stream, device=local)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0 = net.events_total
        e0.record(st)
        net.step(n_steps)
        e1.record(st)
        net.synchronize()
        return e0.elapsed_time(e1), net.events_total - ev0

    net = sg.Network(local)
    for i, n in enumerate(sizes):
        W.add_izhikevich_instance(net, int(n), 1000 + i)
    net.build()
    net.step(64)
    ms, ev = timed(net, steps)
    fp = net.footprint
    net.close()
    solo_ms, solo_ev, n_solo = 0.0, 0, min(8, K)
    for i in range(n_solo):
        a = sg.Network(local)
        W.add_izhikevich_instance(a, int(sizes[i]), 1000 + i)
        a.build()
        a.step(64)
        m, e = timed(a, steps)
        solo_ms, solo_ev = solo_ms + m, solo_ev + e
        a.close()
    ev_s, solo_s = ev / (ms / 1e3), solo_ev / (solo_ms / 1e3)
    return {"workload": f"{K} Izhikevich pulse networks, N log-uniform 500..200000 ({int(sizes.sum())} neurons, "
                        "100 distinct targets each, device thalamic noise), 1000 steps, one batch",
            "events_per_s": ev_s, "neuron_updates_per_s": float(sizes.sum()) * steps / (ms / 1e3),
            "ms_per_step": ms / steps, "footprint_gb": fp / 1e9, "weights": "fp32",
            "one_at_a_time_events_per_s": solo_s, "one_at_a_time_sample": f"first {n_solo} instances",
            "speedup_vs_one_at_a_time": ev_s / solo_s}


def run_serving(args, local):
    """A Poisson stream of seeded LIF / Izhikevich requests (N log-uniform in
    10,000..2,000,000, lognormal out-degree mean 100 sd 60, BF16 weights, 1 s
    simulated: LIF 10,000 steps of 0.1 ms, Izhikevich 1,000 of 1 ms) through
    the continuous-batching server (pooled steps), at arrival rates
    lambda = 5, 20, 50, 100, 200 per s with the same requests.  Against the
    one-at-a-time loop: each request run alone once (build, run, readback:
    its service time), and the loop's latencies for each arrival stream from
    those service times in arrival order (a single FIFO server, queueing
    included)."""
    import numpy as np

    from simuse_b200 import serve as S
    from simuse_b200 import workloads as W
    n_req = args.serve_requests

    def make():
        idx = np.arange(n_req, dtype=np.uint64)
        u = W.uniform01(77, 1, idx)
        ns = np.floor(np.exp(np.log(1e4) + u * (np.log(2e6) - np.log(1e4)))).astype(int)
        kinds = np.where(W.uniform01(77, 2, idx) < 0.5, "lif", "izh")
        return [S.Request(str(k), int(n), 500 + i, 10000 if k == "lif" else 1000)
                for i, (k, n) in enumerate(zip(kinds, ns))]

    solo = [S.run_alone(r, device=local, chunk=1000) for r in make()]
    service = np.array([r.latency for r in solo])
    out = {"workload": f"{n_req} requests, LIF (10000 steps) or Izhikevich (1000 steps), N log-uniform 1e4..2e6, "
                       "lognormal out-degree (100, 60), BF16 weights, Poisson arrivals",
           "one_at_a_time_service_s_mean": float(service.mean()), "budget_gb": 160, "weights": "bf16",
           "by_rate": {}}
    for lam in (5.0, 20.0, 50.0, 100.0, 200.0):
        arrive = np.cumsum(-np.log(1.0 - W.uniform01(78, int(lam), np.arange(n_req, dtype=np.uint64))) / lam)
        reqs = make()
        srv = S.Server(device=local, budget_bytes=160 * 10**9, max_resident=32, chunk=256)
        t0 = time.perf_counter()
        for r, ta in zip(reqs, arrive):
            wait = t0 + ta - time.perf_counter()
            if wait > 0:
                time.sleep(wait)
            srv.submit(r)
        srv.wait_idle(3600)
        t_all = max(r.t_done for r in reqs) - t0
        srv.close()
        lat = srv.latency_percentiles()
        same = all(a.spike_steps is not None and b.spike_steps is not None and
                   np.array_equal(a.spike_steps, b.spike_steps) and np.array_equal(a.spike_index, b.spike_index)
                   for a, b in zip(solo, reqs))
        fin, q_lat = 0.0, []
        for ta, sv in zip(arrive, service):  # the one-at-a-time loop on the same arrivals
            fin = max(fin, ta) + sv
            q_lat.append(fin - ta)
        q_lat = np.array(q_lat)
        out["by_rate"][f"{lam:g}"] = {
            "served_sims_per_s": n_req / t_all, "p50_latency_s": lat["p50_s"], "p99_latency_s": lat["p99_s"],
            "one_at_a_time_sims_per_s": n_req / fin,
            "one_at_a_time_p50_latency_s": float(np.percentile(q_lat, 50)),
            "one_at_a_time_p99_latency_s": float(np.percentile(q_lat, 99)),
            "speedup_vs_one_at_a_time": (n_req / t_all) / (n_req / fin), "pool_ticks": srv.ticks,
            "server_loop_s": {k: round(v, 3) for k, v in srv.phase_s.items()},
            "results_same_as_alone": bool(same), "errors": int(sum(r.error is not None for r in reqs))}
    return out


def _timed_steps(net, local, n_steps):
    """Device time (ms) of n_steps simulation steps on the network's stream."""
    import torch
    st = torch.cuda.ExternalStream(net.stream, device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    net.step(n_steps)
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1)


def run_precision_paths(args, local):
    """The headline network with other weight storage and on the ordered
    path: BF16 and FP8 weights (20, -100 and 100 stay exact: same spikes,
    fewer scatter bytes), and J = 20.1 (not a dyadic multiple: every ring cell
    takes its adds in the reference's order through the owner-computes
    scatter).  Per case: events/s, scatter path, scatter kernel ms per launch
    and its fraction of the HBM roofline."""
    import simuse_b200 as sg
    from simuse_b200 import workloads as W
    peak, _ = measured_peak()
    out = {}
    S = 500
    for name, fmt, w_exc in (("bf16", sg.W_BF16, 20.0), ("fp8", sg.W_FP8, 20.0), ("ordered_j20.1", None, 20.1)):
        spec = W.lif_balanced(n=args.n, k_in=args.k_in, seed=1, ext_rate_hz=4000.0, ext_weight=100.0, w_exc=w_exc)
        net = sg.Network(local)
        if fmt is not None:
            net.set_weight_format(fmt)
        W.build_lif(net, spec)
        net.build()
        net.step(S)  # settle
        ev0, src0 = net.events_total, net.source_events_total
        ms = _timed_steps(net, local, S)
        ev = net.events_total - ev0
        rec = (ev - (net.source_events_total - src0)) / S
        net.profile(True)
        net.step(200)
        ph_ms, ph_n = net.profile_read()
        net.profile(False)
        sp, _ = net.read_stats()
        spikes = float(sp[-200:].mean())
        scat_ms = ph_ms[1] / max(int(ph_n[1]), 1)
        b_ev = {"bf16": 6.0, "fp8": 5.0}.get(name, 8.0) + 1.0 + B_EVENT_APPLY  # x word/record + delay + ring RMW
        alg = rec * b_ev + spikes * B_SPIKE
        out[name] = {"events_per_s": ev / (ms / 1e3), "ms_per_sim_step": ms / S, "scatter": net.scatter_mode,
                     "scatter_ms_per_launch": scat_ms, "scatter_alg_bytes": alg,
                     "scatter_frac": alg / (scat_ms / 1e3) / 1e9 / peak,
                     "weights": name if fmt is not None else "fp32"}
        net.close()
    return out


def run_hh_prefix(args, local):
    """The HH + pair-STDP network at its stated size (100,000 neurons, RK4 at
    dt 0.01 ms, lognormal out-degree (200, 80), conductance synapses, STDP on
    excitatory synapses, weights U(0, 0.01)): 2,000 steps (20 ms) timed after
    500 warm-up steps."""
    import simuse_b200 as sg
    from simuse_b200 import workloads as W
    net = sg.Network(local)
    W.add_hh_stdp(net, 100_000, w_max=0.01)
    net.build()
    net.step(500)
    ev0, d0 = net.events_total, net.stdp_drift
    ms = _timed_steps(net, local, 2000)
    ev = net.events_total - ev0
    out = {"events_per_s": ev / (ms / 1e3), "neuron_updates_per_s": 100_000 * 2000 / (ms / 1e3),
           "us_per_sim_step": ms * 1e3 / 2000, "synapses": net.num_synapses, "steps": 2000,
           "stdp_drift": net.stdp_drift - d0, "scatter": net.scatter_mode}
    net.close()
    return out


def run_kuramoto(args, local):
    """1024 all-to-all Kuramoto populations, N log-uniform 256..65,536, RK4 at
    dt 0.01 with the mean-field identity: 500 steps timed."""
    import torch

    from simuse_b200 import KuramotoBatch
    from simuse_b200 import workloads as W
    sp = W.kuramoto_sweep(1024)
    kb = KuramotoBatch(sp["sizes"], sp["coupling"], sp["dt"], device=local)
    kb.set_state(sp["theta"], sp["omega"])
    kb.run(20)
    kb.synchronize()
    st = torch.cuda.ExternalStream(kb.stream(), device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    kb.run(500)
    e1.record(st)
    kb.synchronize()
    ms = e0.elapsed_time(e1)
    out = {"oscillator_steps_per_s": kb.total * 500 / (ms / 1e3), "oscillators": kb.total,
           "us_per_step": ms * 1e3 / 500}
    kb.close()
    return out


def run_sweep(args, local, n_each: int = 1024, izh_steps: int = 1000, kura_steps: int = 10_000):
    """The batched uneven sweep: n_each Kuramoto populations (N log-uniform
    256..65,536, K linear 0..4, omega Lorentzian(0, 0.5), RK4 at dt 0.01,
    kura_steps steps) and n_each Izhikevich pulse networks (N log-uniform
    500..200,000, BF16 weights on the 1/256 grid, device thalamic noise,
    izh_steps steps of 1 ms) advancing concurrently on two streams.  Timed
    on the device: each half alone, both together, on the fixed scatter
    schedule and again after the autotuner picked one."""
    import torch

    import simuse_b200 as sg
    t0 = time.perf_counter()
    sw = sg.Sweep.configured(n_each, n_each, device=local)
    build_s = time.perf_counter() - t0
    ks, ns = (torch.cuda.ExternalStream(h, device=local) for h in sw.streams)
    sw.run(64, 20)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def timed(izh, kura):
        e0, ei, ek, e1 = ev(), ev(), ev(), ev()
        e0.record(ns)
        ks.wait_event(e0)
        ev0 = sw.events_total
        sw.enqueue(0, kura)
        ek.record(ks)
        sw.enqueue(izh, 0)
        ei.record(ns)
        ns.wait_event(ek)
        e1.record(ns)
        e1.synchronize()
        return {"total_ms": e0.elapsed_time(e1), "izh_ms": e0.elapsed_time(ei) if izh else 0.0,
                "kura_ms": e0.elapsed_time(ek) if kura else 0.0, "izh_events": sw.events_total - ev0}

    def schedule():
        kura_alone = timed(0, kura_steps)
        izh_alone = timed(izh_steps, 0)
        both = timed(izh_steps, kura_steps)
        return {"izh_alone_ms": izh_alone["izh_ms"], "kura_alone_ms": kura_alone["kura_ms"],
                "sequential_ms": izh_alone["izh_ms"] + kura_alone["kura_ms"],
                "concurrent_ms": both["total_ms"], "izh_ms_in_concurrent": both["izh_ms"],
                "kura_ms_in_concurrent": both["kura_ms"],
                "izh_events_per_s_alone": izh_alone["izh_events"] / (izh_alone["izh_ms"] / 1e3),
                "izh_neuron_updates_per_s_alone": sw.neurons * izh_steps / (izh_alone["izh_ms"] / 1e3),
                "kura_oscillator_steps_per_s_alone": sw.oscillators * kura_steps / (kura_alone["kura_ms"] / 1e3),
                "instance_steps_per_s_concurrent": n_each * (izh_steps + kura_steps) / (both["total_ms"] / 1e3)}

    fixed = schedule()
    tune = sw.net.autotune(steps=100)
    tuned = schedule()
    rates = sw.izh_rates()
    out = {"workload": f"{n_each} Kuramoto populations ({sw.oscillators} oscillators, N log-uniform 256..65536, K "
                       f"0..4, RK4 dt 0.01, {kura_steps} steps) + {n_each} Izhikevich pulse networks "
                       f"({sw.neurons} neurons, N log-uniform 500..200000, 100 targets each, BF16 weights on the "
                       f"1/256 grid, {izh_steps} steps of 1 ms), concurrently on two streams",
           "build_s": build_s, "synapses": sw.net.num_synapses, "footprint_gb": sw.footprint / 1e9,
           "scatter": sw.net.scatter_mode, "weights": "bf16", "izh_rate_hz_mean": float(rates.mean()),
           "fixed": fixed, "autotune": tune, "tuned": tuned,
           "tuned_vs_fixed_izh": fixed["izh_alone_ms"] / tuned["izh_alone_ms"]}
    sw.close()
    return out


def run_learn_short(args, local):
    """The headline network with dopamine learning on its 1e9 synapses: 200
    steps timed with learning after 300 learning steps, and one reward."""
    import simuse_b200 as sg
    from simuse_b200 import workloads as W
    spec, _ = workload(args, 0)
    net = sg.Network(local)
    W.build_lif(net, spec)
    net.build()
    net.step(200)
    net.enable_learning(dt=spec["dt"], tau_pre=20.0, tau_post=20.0, tau_e=1000.0, a_ltp=0.1, a_ltd=0.12, lr=0.01,
                        w_min=-200.0, w_max=200.0)
    net.step(300)
    ms = _timed_steps(net, local, 200)
    import torch
    st = torch.cuda.ExternalStream(net.stream, device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    net.reward(1.0)
    e1.record(st)
    e1.synchronize()
    out = {"ms_per_sim_step_learning": ms / 200, "reward_ms": e0.elapsed_time(e1), "scatter": net.scatter_mode,
           "synapses": net.num_synapses}
    net.close()
    return out


def run_ours(args):
    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)

    import simuse_b200 as sg
    from simuse_b200 import workloads as W

    spec, name = workload(args, rank)
    net = sg.Network(local)
    if args.weights == "bf16":
        net.set_weight_format(sg.W_BF16)   # 20, -100 and 100 are exact in bf16: same spikes as fp32
    W.build_lif(net, spec)
    net.build()
    net.synchronize()
    scatter_path = net.scatter_mode
    stream = torch.cuda.ExternalStream(net.stream, device=local)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(local)
        net.synchronize()

    S = args.sim_steps
    # the first steps' raster, for the bit-for-bit comparison with the oracle
    first_raster = None
    if not args.no_cpu_baseline and world == 1:
        net.enable_raster(PARITY_STEPS)
        net.step(PARITY_STEPS)
        first_raster = net.read_raster()
        net.enable_raster(0)
    # the scatter's schedule, picked by the library's autotuner on this
    # network's own steps (ordinary simulation steps; every schedule gives
    # the same bits on the pre-centric path)
    tune = net.autotune(steps=200) if scatter_path != "ordered" and not args.no_autotune else None
    for _ in range(args.warmup):
        net.step(S)
    barrier()

    # ---- (A) device-timed value ---------------------------------------------
    ev0 = net.events_total
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            net.step(S)
        e1.record(stream)
        e1.synchronize()
        barrier()
    ms = e0.elapsed_time(e1)
    events = net.events_total - ev0
    spk, evs = net.read_stats()
    spk = spk[-args.steps * S:]
    t_max, ev_all = reduce_over_ranks(dist, f"cuda:{local}", ms, events)
    value = ev_all / (t_max / 1e3)

    # ---- (B) end to end through the C ABI with host buffers --------------------
    net.enable_raster(S)
    cap = int(max(spk.max() if spk.size else 1, 1) * S * 1.5) + 1024
    h_steps = torch.empty(cap, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    h_idx = torch.empty(cap, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    net.step(S)
    net.read_spike_events_into(h_steps, h_idx)  # warm
    barrier()
    ev0 = net.events_total
    d2h = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        net.step(S)
        n_sp = net.read_spike_events_into(h_steps, h_idx)
        d2h += n_sp * 8
    t_e2e = time.perf_counter() - t0
    ev_e2e = net.events_total - ev0
    t_e2e, ev_e2e = reduce_over_ranks(dist, f"cuda:{local}", t_e2e, ev_e2e)
    net.enable_raster(0)

    # ---- (C) per-kernel timing: CUDA events around each phase --------------------
    net.profile(True)
    p_steps = min(S, 1000)
    ev0, src0 = net.events_total, net.source_events_total
    net.step(p_steps)
    ph_ms, ph_launch = net.profile_read()
    net.profile(False)
    p_events = (net.events_total - ev0) / p_steps
    p_src = (net.source_events_total - src0) / p_steps
    p_rec = p_events - p_src
    sp, _ = net.read_stats()
    p_spikes = float(sp[-p_steps:].mean()) if sp.size else 0.0
    net_schedule = net.scatter_schedule
    scatter_kernel = ("scatter_kernel" if scatter_path == "ordered" else
                      "scatter_walk_kernel" if net_schedule[0] >= 4 else "scatter_red_kernel")
    phases = ["neuron_kernel<LIF>", scatter_kernel]
    alg = [spec["n"] * B_NEURON,
           p_rec * (B_EVENT_EXPAND + B_EVENT_APPLY) + p_spikes * B_SPIKE]
    per_launch_ms = [ph_ms[i] / max(int(ph_launch[i]), 1) for i in range(2)]
    dom = int(np.argmax(ph_ms[:2]))
    peak, peak_kind = measured_peak()
    achieved = alg[dom] / (per_launch_ms[dom] / 1e3) / 1e9
    step_alg = sum(alg)
    step_ms = ms / (args.steps * S)

    # the pre-centric scatter's own ceiling: random reds into an array of the rings' size
    red_peak = probe_red_rate(local, spec["n"] * (args.d_max + 1)) if scatter_path != "ordered" else None
    net.close()  # the headline network leaves HBM before the extra measurements
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return

    mean_spk = float(spk.mean()) if spk.size else 0.0
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {**config(args, name, spec, scatter_path),
                   "schedule": ({"autotuned": True, "variant": tune["variant"], "blocks_per_sm": tune["blocks_per_sm"],
                                 "fixed_ms_per_sim_step": tune["fixed_ms_per_step"],
                                 "tuned_ms_per_sim_step": tune["tuned_ms_per_step"]} if tune else
                                {"autotuned": False, "variant": list(net_schedule)})},
        "sim": {"ms_per_sim_step": step_ms, "events_per_sim_step": events / (args.steps * S),
                "recurrent_events_per_sim_step": p_rec, "source_events_per_sim_step": p_src,
                "spikes_per_sim_step": mean_spk, "rate_hz": mean_spk / spec["n"] / (spec["dt"] * 1e-3),
                "neuron_updates_per_s": spec["n"] * args.steps * S / (ms / 1e3) * world,
                "step_roofline_frac": step_alg / (step_ms / 1e3) / 1e9 / peak},
        "e2e": {"value": ev_e2e / t_e2e, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(d2h / args.steps),
                "path": "sg_step + sg_raster_read_events into pinned host buffers, wall clock",
                "inputs": "none per step by design: the external drive is the network's own Poisson sources, "
                          "rolled on the device; the per-step host output is the spike raster"},
        "roofline": {"bound": "hbm", "kernel": phases[dom], "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": profiled_traffic(phases[dom]),
                     "alg_bytes_per_launch": alg[dom], "launch_ms": per_launch_ms[dom],
                     "phases_ms_per_launch": dict(zip(phases, per_launch_ms)),
                     "phases_frac": {ph: alg[i] / (per_launch_ms[i] / 1e3) / 1e9 / peak
                                     for i, ph in enumerate(phases)}},
        "clocks": clk.summary(),
        "gpu_launches": int(args.steps * S * 2),
    }
    if red_peak:
        red_ach = p_rec / (per_launch_ms[1] / 1e3)
        out["roofline_l2"] = {"bound": "l2_red", "kernel": phases[1], "achieved": red_ach, "peak": red_peak,
                              "unit": "reds/s", "frac": red_ach / red_peak,
                              "peak_source": "sg_probe_red_rate on this GPU: random red.global.add.f32 from a "
                                             "full-occupancy grid into an array of the rings' size",
                              "what": "one red per recurrent event; the scatter's events per launch over its "
                                      "launch time, against the measured red ceiling"}
    if not args.no_extras and world == 1:
        for key, fn in (("precision_paths", run_precision_paths), ("hh_stdp_100k", run_hh_prefix),
                        ("kuramoto_sweep", run_kuramoto), ("lif_learn", run_learn_short),
                        ("batched", run_batched), ("sweep", run_sweep), ("serving", run_serving)):
            try:
                out[key] = fn(args, local)
            except Exception as e:  # an extra measurement never takes the headline line down
                out[key] = {"error": f"{type(e).__name__}: {e}"}
    if not args.no_cpu_baseline and world == 1:
        cnet, cores, build_s = cpu_baseline(args, spec, args.cpu_seconds)
        rc, ev, el = run_cpu_parity(cnet, PARITY_STEPS)
        out["cpu_baseline"] = {"value": ev / el, "unit": UNIT, "cores": cores, "kind": "port",
                               "sample": f"first {PARITY_STEPS} steps of the same network from its initial state "
                                         f"({el:.1f} s; oracle/ C++ restatement, push collected on {cores} threads)"}
        diff = np.nonzero((first_raster != rc).any(axis=1))[0]
        out["parity"] = {"steps": PARITY_STEPS, "identical": bool(diff.size == 0),
                         "first_divergent_step": int(diff[0]) if diff.size else None,
                         "spikes": int(rc.sum()),
                         "what": "spike raster of the first steps from the initial state, GPU against the oracle, "
                                 "bit for bit"}
    print(json.dumps(out), flush=True)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    spec, name = workload(args, 0)
    net, cores, build_s = cpu_baseline(args, spec, args.cpu_seconds)
    per_step_s = 1.0
    for _ in range(args.warmup):
        run_cpu_sample(net, per_step_s, min_steps=5)
    tot_ev, tot_t, tot_steps = 0, 0.0, 0
    for _ in range(args.steps):
        ev, ns, el = run_cpu_sample(net, per_step_s, min_steps=5)
        tot_ev += ev
        tot_t += el
        tot_steps += ns
    value = tot_ev / tot_t
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_t / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)", "impl": "reference", "config": config(args, name, spec),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{tot_steps} simulation steps in {args.steps} samples of ~{per_step_s:.0f} s "
                                   f"(oracle/ C++ restatement of the reference step; build {build_s:.1f} s)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def run_case(args):
    """One workload alone, one JSON line (oscillator-steps/s or events/s)."""
    import numpy as np
    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if args.case == "izh-batch":
        args.batch_instances = args.instances
        print(json.dumps({"case": args.case, **run_batched(args, local)}), flush=True)
        return
    if args.case == "hh-stdp":
        import simuse_b200 as sg
        from simuse_b200 import workloads as W
        n = args.n if args.n != 1_000_000 else 100_000
        net = sg.Network(local)
        pop = W.add_hh_stdp(net, n, w_max=args.hh_wmax)
        net.build()
        net.step(args.warmup * 100)
        net.enable_neuron_stats()
        net.synchronize()
        S = args.hh_steps
        st = torch.cuda.ExternalStream(net.stream, device=local)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0, d0 = net.events_total, net.stdp_drift
        e0.record(st)
        net.step(S)
        e1.record(st)
        net.synchronize()
        ms = e0.elapsed_time(e1)
        ev = net.events_total - ev0
        rates = net.neuron_stats(pop, 0.01)[0]
        print(json.dumps({"case": args.case, "metric": "synaptic events/s", "value": ev / (ms / 1e3),
                          "neuron_updates_per_s": n * S / (ms / 1e3), "neurons": n,
                          "synapses": net.num_synapses, "steps": S, "simulated_s": S * 0.01e-3,
                          "ms_per_step": ms / S, "events_per_step": ev / S,
                          "stdp_drift": net.stdp_drift - d0, "w_max": args.hh_wmax,
                          "rate_hz": float(rates.mean()),
                          "workload": "HH (RK4, dt 0.01 ms) + ExpOne conductance synapses + pair STDP, lognormal "
                                      "out-degree (200, 80), bias N(10, 2), weights U(0, w_max), per-neuron "
                                      "spike counts on"}), flush=True)
        net.close()
        return
    if args.case == "lif-learn":
        run_lif_learn(args, local)
        return
    if args.case == "sweep":
        print(json.dumps({"case": args.case, **run_sweep(args, local, n_each=args.instances // 2 or 1)}),
              flush=True)
        return
    if args.case == "taas":
        run_taas(args, local)
        return
    from simuse_b200 import KuramotoBatch
    from simuse_b200 import workloads as W
    sp = W.kuramoto_sweep(args.instances)
    kb = KuramotoBatch(sp["sizes"], sp["coupling"], sp["dt"], device=local)
    kb.set_state(sp["theta"], sp["omega"])
    kb.run(args.warmup)
    kb.synchronize()
    st = torch.cuda.ExternalStream(kb.stream(), device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    kb.run(args.sim_steps)
    e1.record(st)
    kb.synchronize()
    ms = e0.elapsed_time(e1)
    print(json.dumps({"case": args.case, "metric": "oscillator-steps/s",
                      "value": kb.total * args.sim_steps / (ms / 1e3), "instances": args.instances,
                      "oscillators": kb.total, "steps": args.sim_steps, "us_per_step": ms * 1e3 / args.sim_steps,
                      "workload": "Kuramoto populations, N log-uniform 256..65536, K linear 0..4, omega "
                                  "Lorentzian(0, 0.5), RK4 dt 0.01 (mean field)"}), flush=True)
    kb.close()


def run_lif_learn(args, local):
    """The headline LIF network with dopamine-modulated eligibility learning
    on its synapses: the same sim steps timed without learning (exact-sum
    rings) and with it (ordered rings + the eligibility kernel after every
    step), then full-network rewards (every eligibility folded to now, every
    weight updated)."""
    import torch

    import simuse_b200 as sg
    from simuse_b200 import workloads as W
    spec, name = workload(args, 0)
    net = sg.Network(local)
    W.build_lif(net, spec)
    net.build()
    net.synchronize()
    st = torch.cuda.ExternalStream(net.stream, device=local)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1)

    S = args.sim_steps
    net.step(S * args.warmup)
    mode0 = net.scatter_mode
    ev0 = net.events_total
    ms0 = timed(lambda: net.step(S * args.steps))
    ev_a = net.events_total - ev0
    net.enable_learning(dt=spec["dt"], tau_pre=20.0, tau_post=20.0, tau_e=1000.0, a_ltp=0.1, a_ltd=0.12, lr=0.01,
                        w_min=-200.0, w_max=200.0)
    net.step(S * args.warmup)
    ev1 = net.events_total
    ms1 = timed(lambda: net.step(S * args.steps))
    ev_b = net.events_total - ev1
    rew = [timed(lambda: net.reward(1.0)) for _ in range(max(args.steps, 3))]
    E = net.num_synapses
    steps = S * args.steps
    peak, kind = measured_peak()
    # reward: per synapse read sync step, eligibility and weight, write all three
    r_ms = sorted(rew)[len(rew) // 2]
    r_gbs = 24.0 * E / (r_ms / 1e3) / 1e9
    print(json.dumps({
        "case": args.case, "workload": name, "neurons": spec["n"], "synapses": E, "sim_steps": steps,
        "no_learning": {"scatter": mode0, "ms_per_step": ms0 / steps, "events_per_s": ev_a / (ms0 / 1e3)},
        "learning": {"scatter": net.scatter_mode, "ms_per_step": ms1 / steps, "events_per_s": ev_b / (ms1 / 1e3),
                     "events_per_step": ev_b / steps},
        "reward": {"first_ms_with_fold": rew[0], "ms": r_ms, "algorithmic_bytes_per_synapse": 24, "achieved_gbs": r_gbs, "peak_gbs": peak,
                   "frac": r_gbs / peak, "peak_kind": kind},
        "learn_config": "dt 0.1, tau_pre = tau_post 20, tau_e 1000, a_ltp 0.1, a_ltd 0.12, lr 0.01, w in [-200, 200]",
    }), flush=True)
    net.close()


def run_taas(args, local):
    """Checkpoint and resume of the LIF network through .taas v2 files:
    sg_taas_save (device CSR to host, CRC32, file), validate (every CRC),
    sg_taas_load_weights (file, CRC32, synapse check, weights to the device);
    wall-clock, best of --steps runs."""
    import tempfile
    import time

    import simuse_b200 as sg
    from simuse_b200 import workloads as W
    spec, name = workload(args, 0)
    net = sg.Network(local)
    W.build_lif(net, spec)
    net.build()
    net.synchronize()
    out = {"case": args.case, "workload": name, "synapses": net.num_synapses}
    with tempfile.TemporaryDirectory() as td:
        for level in (0, 3):
            path = os.path.join(td, f"net{level}.taas")
            ts, tv, tl = [], [], []
            for _ in range(max(args.steps, 1)):
                t0 = time.perf_counter()
                net.save_taas(path, zstd_level=level)
                t1 = time.perf_counter()
                sg.taas.validate(path)
                t2 = time.perf_counter()
                net.load_weights_taas(path)
                net.synchronize()
                t3 = time.perf_counter()
                ts.append(t1 - t0)
                tv.append(t2 - t1)
                tl.append(t3 - t2)
            size = os.path.getsize(path)
            out[f"zstd{level}"] = {"file_bytes": size, "save_s": min(ts), "validate_s": min(tv), "load_s": min(tl),
                                   "save_gbs": size / min(ts) / 1e9, "load_gbs": size / min(tl) / 1e9}
    print(json.dumps(out), flush=True)
    net.close()


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.case != "headline":
        run_case(a)
    else:
        run_ours(a)
