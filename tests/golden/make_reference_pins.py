"""Extract the golden vectors that the reference's own tests hold for the
simulation step, and write them to tests/golden/reference_pins.json.

Run in a checkout that has the reference source tree (read-only):

    python tests/golden/make_reference_pins.py /path/to/reference

The reference is Rust and cannot be compiled here, so its pins are read as
text from its test files: every value below is parsed from (or checked
against) the cited file and line range, and the script fails if a cited
value is not found there.  The JSON it writes is what the tests use; they
never read the reference tree at run time.
"""
from __future__ import annotations

import json
import os
import re
import sys

P = "crates/SiMuse/crates/pillars"


def read(root, rel):
    with open(os.path.join(root, rel)) as f:
        return f.read()


def lines(root, rel, a, b):
    return "\n".join(read(root, rel).splitlines()[a - 1:b])


def require(text, needle, where):
    if needle not in text:
        raise SystemExit(f"pin not found: {needle!r} in {where}")


def parse_struct_list(block, fields):
    out = []
    for m in re.finditer(r"\{([^{}]*)\}", block):
        body = m.group(1)
        item = {}
        for f in fields:
            mm = re.search(rf"\b{f}:\s*(\"?[-\w.]+\"?)", body)
            if mm:
                v = mm.group(1).strip('"')
                try:
                    v = float(v) if any(c in v for c in ".e") or f not in ("label",) else v
                except ValueError:
                    pass
                item[f] = v
        if item:
            out.append(item)
    return out


def main(root):
    pins = {"source": "reference test files, parsed as text"}

    # LIF golden spike counts: tests/lif_vs_neuron.rs:77-111, tolerance :131
    rel = f"{P}/tests/lif_vs_neuron.rs"
    blk = lines(root, rel, 77, 111)
    cfgs = parse_struct_list(blk, ["label", "i_syn", "dt", "ref_spikes", "v_rest", "v_thresh",
                                   "v_reset", "tau_m", "tau_ref"])
    require(lines(root, rel, 131, 131), "diff <= 2.0", rel + ":131")
    require(lines(root, rel, 116, 117), "let n = 8;", rel + ":116")
    require(lines(root, rel, 117, 117), "500.0", rel + ":117")
    pins["lif_spike_counts"] = {
        "cite": f"{rel}:77-111 (configs), :116-117 (n=8, 500 ms), :131 (|diff| <= 2)",
        "n": 8, "t_ms": 500.0, "on_ms": 10.0, "tolerance": 2.0,
        "configs": [{k: (float(v) if k != "label" else v) for k, v in c.items()} for c in cfgs],
    }

    # Izhikevich pattern ranges: tests/izhikevich_vs_neuron.rs:30-75, run :167
    rel = f"{P}/tests/izhikevich_vs_neuron.rs"
    blk = lines(root, rel, 30, 75)
    cfgs = parse_struct_list(blk, ["label", "a", "b", "c", "d", "i_syn", "min_spikes",
                                   "max_spikes", "min_isi_cv"])
    require(lines(root, rel, 86, 86), "2.0; // tau_ref", rel + ":86 tau_ref")
    require(lines(root, rel, 87, 87), "30.0; // v_thresh", rel + ":87 v_thresh")
    require(lines(root, rel, 169, 169), "run_izh(c, n, 0.5, 1000.0)", rel + ":169")
    pins["izh_patterns"] = {
        "cite": f"{rel}:30-75 (ranges), :86-87 (tau_ref=2, v_th=30), :169 (dt 0.5, 1000 ms), :95 (on at 10 ms)",
        "n": 8, "dt": 0.5, "t_ms": 1000.0, "on_ms": 10.0, "tau_ref": 2.0, "v_thresh": 30.0,
        "configs": [{k: (float(v) if k != "label" else v) for k, v in c.items()} for c in cfgs],
    }

    # Delay arrival: tests/network_delays.rs:42-67 (constants and params), :88-90, :138-160
    rel = f"{P}/tests/network_delays.rs"
    txt = read(root, rel)
    for needle in ["const FORCE_V: f32 = 100.0;", "const W_STRONG: f32 = 500.0;",
                   "const RUN_STEPS: usize = 70;", "const TEST_DELAYS: [u8; 4] = [0, 2, 5, 31];",
                   "lif.fill_param(P_DT, 0.5);", "lif.fill_param(P_INV_TAU, 0.5);",
                   "lif.fill_param(P_V_REST, -70.0);", "lif.fill_param(P_V_THRESH, -54.0);",
                   "lif.fill_param(P_V_RESET, -70.0);", "lif.fill_param(P_TAU_REF, 2.0);",
                   "lif.fill_state(S_V, -70.0);", "let n = 80usize;"]:
        require(txt, needle, rel)
    pins["delay_arrival"] = {
        "cite": f"{rel}:42-67 (constants, LIF params), :88-90 (arrival = max(delay,1)), :138-160 (n=4 and n=80)",
        "force_v": 100.0, "w_strong": 500.0, "run_steps": 70, "delays": [0, 2, 5, 31],
        "lif_params": [0.5, 0.5, -70.0, -54.0, -70.0, 2.0], "v0": -70.0, "sizes": [4, 80],
    }

    # Push slot arithmetic: src/api/net/push.rs:300-431 and :433-499
    rel = f"{P}/src/api/net/push.rs"
    txt = read(root, rel)
    for needle in ["push_spikes(&[0, 3, 7], &graph, &mut delay, &mut [], 0, None);",
                   "let d = vec![0u8, 1u8, 5u8];", "assert_eq!(delay.slot(5)[5], 0.5);",
                   "let d = vec![(MAX_DELAY_SLOTS - 1) as u8];",
                   "push_spikes(&[0], &graph, &mut delay, &mut [], 1, None);",
                   "push_spikes(&[0], &graph, &mut delay, &mut [], 5, None);",
                   "assert_eq!(delay.slot(7)[1], 1.0);",
                   "let w = vec![3.0f32, 4.0f32];",
                   "assert!((delay.slot(1)[2] - 7.0).abs() < 1e-6);",
                   "let d = vec![0u8, 3u8];", "let triples = collect_push_triples(&[0, 1], &graph, 7);"]:
        require(txt, needle, rel)
    pins["push"] = {
        "cite": f"{rel}:300-431 (slot math, accumulation), :433-499 (par == seq, step 7)",
        "cases": [
            {"name": "basic", "n": 8, "from": list(range(8)), "to": list(range(8)), "w": [1.0] * 8,
             "d": [0] * 8, "active": [0, 3, 7], "step": 0,
             "expect": [[1, 0, 1.0], [1, 3, 1.0], [1, 7, 1.0]]},
            {"name": "with_delays", "n": 6, "from": [0, 1, 2], "to": [3, 4, 5], "w": [1.0, 2.0, 0.5],
             "d": [0, 1, 5], "active": [0, 1, 2], "step": 0,
             "expect": [[1, 3, 1.0], [1, 4, 2.0], [5, 5, 0.5]]},
            {"name": "wraparound", "n": 2, "from": [0], "to": [1], "w": [1.0], "d": [31],
             "active": [0], "step": 1, "expect": [[0, 1, 1.0]]},
            {"name": "step_counter", "n": 2, "from": [0], "to": [1], "w": [1.0], "d": [2],
             "active": [0], "step": 5, "expect": [[7, 1, 1.0]]},
            {"name": "accumulate", "n": 3, "from": [0, 1], "to": [2, 2], "w": [3.0, 4.0], "d": [0, 0],
             "active": [0, 1], "step": 0, "expect": [[1, 2, 7.0]]},
            {"name": "par_triples_step7", "n": 4, "from": [0, 1], "to": [2, 3], "w": [1.0, 2.0],
             "d": [0, 3], "active": [0, 1], "step": 7, "expect": [[8, 2, 1.0], [10, 3, 2.0]]},
            {"name": "no_outgoing", "n": 3, "from": [0, 1], "to": [0, 1], "w": [1.0, 1.0],
             "d": [0, 0], "active": [2], "step": 0, "expect": []},
        ],
    }

    # Delay ring contract: src/api/net/delay.rs:111-173
    rel = f"{P}/src/api/net/delay.rs"
    txt = read(root, rel)
    for needle in ["buf.add(1, 2, 5.0);", "buf.add(MAX_DELAY_SLOTS + 3, 0, 7.0);",
                   "buf.add(2, 1, 3.0);", "buf.add(2, 1, 4.0);", "assert_eq!(buf.slot(2), &[0.0, 7.0]);"]:
        require(txt, needle, rel)
    pins["delay_ring"] = {"cite": f"{rel}:111-173", "accumulate": [3.0, 4.0, 7.0]}

    # Compaction: src/api/net/compact.rs:80-153
    rel = f"{P}/src/api/net/compact.rs"
    txt = read(root, rel)
    for needle in ["assert_eq!(active, vec![0, 3, 6, 9, 12, 15, 18]);", "let n = 1003usize;",
                   "wrapping_mul(2654435761).wrapping_rem(997) < 97",
                   "assert_eq!(out, vec![1, 3, 5, 7, 9]);"]:
        require(txt, needle, rel)
    pins["compact"] = {
        "cite": f"{rel}:80-153",
        "some": {"n": 20, "every": 3, "expect": [0, 3, 6, 9, 12, 15, 18]},
        "alternating": {"spikes": [0, 1, 0, 1, 0, 1, 0, 1, 0, 1], "expect": [1, 3, 5, 7, 9]},
        "hashed": {"n": 1003, "mul": 2654435761, "mod": 997, "lt": 97, "min_len": 81},
    }

    # Poisson source hash: src/api/net/network/sources.rs:5-14 (constants)
    rel = f"{P}/src/api/net/network/sources.rs"
    txt = read(root, rel)
    for needle in ["0x9E37_79B9_7F4A_7C15", "0xBF58_476D_1CE4_E5B9", "0x94D0_49BB_1331_11EB",
                   "let u = (z >> 40) as f32 / (1u64 << 24) as f32;"]:
        require(txt, needle, rel)
    pins["poisson"] = {"cite": f"{rel}:5-14"}

    # Tsodyks-Markram delivered weights against NEURON:
    # src/api/net/push.rs:646-695 (test_tm_matches_neuron_delivered_weights)
    rel = f"{P}/src/api/net/push.rs"
    txt = read(root, rel)
    start = txt.index("fn test_tm_matches_neuron_delivered_weights")
    body = txt[start:start + 4000]

    def f32_array(name):
        m = re.search(name + r": \[f32; (\d+)\] = \[([^\]]*)\]", body)
        if not m:
            raise SystemExit(f"pin not found: {name} in {rel}")
        vals = [float(x) for x in m.group(2).replace("\n", " ").split(",") if x.strip()]
        assert len(vals) == int(m.group(1))
        return vals
    for needle in ["u0: 0.5,", "a_rec: (-0.5f32 / 100.0).exp(),", "u0: 0.1,", "a_rec: (-0.5f32 / 1e6).exp(),",
                   "a_fac: (-0.5f32 / 50.0).exp(),", "let step = 20 + 40 * k;", "(w - ref_w).abs() < 1e-4"]:
        require(body, needle, rel)
    pins["tm_neuron"] = {
        "cite": f"{rel}:646-695",
        "dt": 0.5, "steps": [20 + 40 * k for k in range(12)], "tol": 1e-4,
        "depression": {"u0": 0.5, "tau_rec": 100.0, "ref": f32_array("REF_DEP")},
        "facilitation": {"u0": 0.1, "tau_rec": 1e6, "tau_fac": 50.0, "ref": f32_array("REF_FAC")},
    }

    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_pins.json")
    with open(out, "w") as f:
        json.dump(pins, f, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_reference_pins.py <path to the reference source tree>")
    main(sys.argv[1])
