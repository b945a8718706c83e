"""Loading and binding of libsimuse_b200.so (the C ABI of include/simuse_b200.h)."""
from __future__ import annotations

import ctypes as C
import os
import re

_PKG_DIR = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_PKG_DIR)  # dioma-core_b200/
# SIMUSE_B200_LIB overrides the library location (e.g. an installed copy)
library_path = os.environ.get("SIMUSE_B200_LIB", os.path.join(_ROOT, "libsimuse_b200.so"))
header_path = os.path.join(os.path.dirname(_ROOT), "include", "simuse_b200.h")


class SimuseError(RuntimeError):
    """A non-zero status from the C ABI (the reference panics in these cases)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


vp, i32, u32, u64, f32, f64, sz = (
    C.c_void_p, C.c_int, C.c_uint32, C.c_uint64, C.c_float, C.c_double, C.c_size_t)
u8 = C.c_uint8

# name -> argument types (all return int status)
SIGNATURES = {
    "sg_abi_version": [],
    "sg_last_error": [C.c_char_p, sz],
    "sg_device_count": [vp],
    "sg_net_create": [vp, i32],
    "sg_net_destroy": [vp],
    "sg_synchronize": [vp],
    "sg_debug_stall_scatter": [vp, i32],
    "sg_autotune": [vp, u32, vp, vp, vp, vp],
    "sg_probe_red_rate": [i32, u64, u32, vp],
    "sg_scatter_schedule": [vp, vp, vp],
    "sg_pool_create": [vp, i32],
    "sg_pool_destroy": [vp],
    "sg_pool_add": [vp, vp],
    "sg_pool_remove": [vp, vp],
    "sg_pool_size": [vp, vp],
    "sg_pool_step": [vp, u32],
    "sg_pool_synchronize": [vp],
    "sg_query": [vp, vp],
    "sg_pop_add": [vp, i32, u32, vp],
    "sg_pop_fill_param": [vp, u32, u32, f32],
    "sg_pop_fill_state": [vp, u32, u32, f32],
    "sg_pop_set_param": [vp, u32, u32, vp, u32],
    "sg_pop_set_state": [vp, u32, u32, vp, u32],
    "sg_pop_get_state": [vp, u32, u32, vp, u32],
    "sg_pop_get_param": [vp, u32, u32, vp, u32],
    "sg_connect": [vp, u32, vp, u32, vp, vp, vp, u64],
    "sg_connect_ex": [vp, u32, vp, u32, vp, vp, vp, vp, u64, u32],
    "sg_connect_fixed_indegree": [vp, u32, u32, u32, u64, u32, f32, f32, u8, u8, u8, u8, u32],
    "sg_connect_fixed_outdegree": [vp, u32, u32, u32, u64, i32, u32, f32, f32, i32, u8, u8, u8, u8, u32],
    "sg_connect_lognormal_outdegree": [vp, u32, u32, f64, f64, u64, i32, u32, f32, f32, i32, u8, u8, u8, u8, u32],
    "sg_register_expone": [vp, f32, f32, f32, vp],
    "sg_poisson_add": [vp, f32, f32, u32, vp],
    "sg_poisson_add_many": [vp, u32, f32, f32, vp, u32, vp],
    "sg_poisson_connect": [vp, u32, u32, vp, vp, vp, vp, u64],
    "sg_poisson_connect_plastic": [vp, u32, u32, vp, vp, vp, vp, vp, u64],
    "sg_poisson_connect_one_to_one": [vp, u32, u32, u32, vp, f32, u8],
    "sg_stdp_config": [vp, f32, f32, f32, f32, f32, f32, f32],
    "sg_set_weight_format": [vp, i32],
    "sg_set_deterministic": [vp, i32],
    "sg_scatter_mode": [vp, vp],
    "sg_register_plasticity": [vp, f32, f32, i32, f32, f32, vp],
    "sg_register_kinetics": [vp, i32, vp, f32, f32, vp],
    "sg_set_receptor_kinetics": [vp, f32],
    "sg_receptor_read": [vp, vp],
    "sg_receptor_write": [vp, vp],
    "sg_connect_plastic": [vp, u32, vp, u32, vp, vp, vp, vp, vp, u64, u32],
    "sg_build": [vp],
    "sg_build_from_csr": [vp, vp, vp, vp, vp],
    "sg_pop_set_noise": [vp, u32, u64, u32, u64, u64, f64, f64, u32],
    "sg_pop_set_bias": [vp, u32, vp, u32],
    "sg_ring_clear": [vp],
    "sg_inject": [vp, u32, vp, vp, u64],
    "sg_step": [vp, u32],
    "sg_raster_enable": [vp, u32],
    "sg_raster_read": [vp, vp, u64, vp],
    "sg_stats_read": [vp, vp, vp, u32, vp],
    "sg_raster_read_events": [vp, vp, vp, u64, vp],
    "sg_raster_stage": [vp],
    "sg_raster_fetch": [vp, vp, vp, u64, vp],
    "sg_raster_fetch_csr": [vp, vp, u64, vp, u64, vp, vp, vp],
    "sg_host_alloc": [u64, vp],
    "sg_host_free": [vp],
    "sg_raster_counts": [vp, vp],
    "sg_profile_enable": [vp, i32],
    "sg_profile_read": [vp, vp, vp],
    "sg_spikes": [vp, u32, vp, u32],
    "sg_step_counter": [vp, vp],
    "sg_total_neurons": [vp, vp],
    "sg_num_synapses": [vp, vp],
    "sg_events_total": [vp, vp],
    "sg_source_events_total": [vp, vp],
    "sg_graph_read": [vp, vp, vp, vp, vp],
    "sg_graph_read_types": [vp, vp, vp],
    "sg_weights_read": [vp, vp],
    "sg_ring_read": [vp, u32, vp],
    "sg_stdp_drift": [vp, vp],
    "sg_stdp_traces": [vp, vp, vp],
    "sg_clamp_hits": [vp, vp],
    "sg_learn_enable": [vp, f32, f32, f32, f32, f32, f32, f32, f32, f32],
    "sg_learn_reward": [vp, f32, f32, f32],
    "sg_learn_clear": [vp],
    "sg_learn_reward_range": [vp, u64, u64, f32, f32, f32],
    "sg_learn_clear_range": [vp, u64, u64],
    "sg_pop_synapse_range": [vp, u32, vp, vp],
    "sg_learn_restrict": [vp, vp, u64],
    "sg_learn_set_eligibility": [vp, vp, u64],
    "sg_learn_motor": [vp, u64, u64, u64, u64],
    "sg_learn_motor_read": [vp, vp],
    "sg_learn_snapshot": [vp],
    "sg_learn_recall": [vp, f32],
    "sg_learn_read": [vp, vp, vp, vp, vp],
    "sg_pop_add_external": [vp, u32, vp],
    "sg_pop_set_external_source": [vp, u32, vp],
    "sg_spike_words": [vp, u32, vp],
    "sg_step_begin": [vp],
    "sg_step_end": [vp],
    "sg_taas_write": [vp, vp, vp, u32, vp, vp, vp, vp, vp, u32, vp, vp, i32],
    "sg_taas_read": [vp, vp, vp, vp, u64, vp],
    "sg_taas_validate": [vp],
    "sg_taas_inspect": [vp, vp, u64, vp],
    "sg_taas_save": [vp, vp, vp, i32],
    "sg_taas_load_weights": [vp, vp],
    "sg_connect_taas": [vp, u32, u32, vp, u8],
    "sg_footprint": [vp, vp],
    "sg_neuron_stats_enable": [vp, i32],
    "sg_neuron_stats_read": [vp, u32, vp, vp, vp, vp],
    "sg_stream": [vp, vp],
    "sg_push_spikes": [vp, vp, vp, vp, u32, vp, u32, u64, vp, vp],
    "sg_push_spikes_noalloc": [vp, vp, vp, vp, u32, vp, u32, u64, vp, vp],
    "sg_kuramoto_create": [vp, i32, u32, vp, vp, f32],
    "sg_kuramoto_destroy": [vp],
    "sg_kuramoto_total": [vp, vp],
    "sg_kuramoto_set_state": [vp, vp, vp],
    "sg_kuramoto_record": [vp, u64],
    "sg_kuramoto_run": [vp, u32],
    "sg_kuramoto_synchronize": [vp],
    "sg_kuramoto_get_theta": [vp, vp],
    "sg_kuramoto_get_r": [vp, vp, u64, vp],
    "sg_kuramoto_get_r_mean": [vp, vp],
    "sg_kuramoto_stream": [vp, vp],
}

_lib = None


def declared_symbols() -> list[str]:
    """Every function declared in include/simuse_b200.h."""
    txt = open(header_path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\bint\s+(sg_\w+)\s*\(", txt)))


def lib():
    """The loaded library; raises when it is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(library_path):
            raise ImportError(
                f"{library_path} is missing: build it with `make -C dioma-core_b200` "
                "(there is no CPU fallback)")
        L = C.CDLL(library_path)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = i32
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(4096)
    lib().sg_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int) -> int:
    if rc < 0:
        raise SimuseError(rc, last_error())
    return rc
