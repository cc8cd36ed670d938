"""Seeded test designs / scripts / stimulus shared by the tests."""
import functools

import numpy as np

from jacquard_b200 import frontend, state


@functools.lru_cache(maxsize=None)
def design(kind, seed=11):
    if kind == "tiny":
        p = frontend.DesignParams(seed=seed, nodes_per_cluster=1500, depth=10, n_dff=96,
                                  n_pi=12, n_po=10)
    elif kind == "small":
        p = frontend.small_params(seed=1)
    elif kind == "sram":
        p = frontend.DesignParams(seed=seed, n_clusters=4, nodes_per_cluster=1200, depth=16,
                                  intra_frac=0.9, n_dff=400, n_pi=24, n_po=16, n_sram=3,
                                  sram_addr_bits=6, with_reset=1)
    elif kind == "soc_mini":
        p = frontend.soc_params(seed=2, n_clusters=8, n_dff=3000, n_sram=2)
    else:
        raise KeyError(kind)
    return frontend.Design(p)


@functools.lru_cache(maxsize=None)
def script(kind, num_blocks, split=(), xprop=False, timing_seed=0, target_parts=0):
    d = design(kind)
    if timing_seed:
        rng = np.random.default_rng(timing_seed)
        n = d.num_pins + 1
        kinds = d.kind
        r = rng.integers(20, 201, size=n).astype(np.uint32)
        r[kinds != 1] = 0
        d.set_delays(r, r)
    if target_parts:  # balanced, flat partitions (the batched workload's form)
        s = d.build_script(num_blocks=num_blocks, level_split=split, xprop=xprop,
                           merge_passes=0, target_parts=target_parts)
    else:
        s = d.build_script(num_blocks=num_blocks, level_split=split, xprop=xprop)
    if timing_seed:
        d.set_delays(np.zeros(d.num_pins + 1, np.uint32), np.zeros(d.num_pins + 1, np.uint32))
    return s


def stimulus(kind, s, cycles, seed=3, p_toggle=0.5, reset_cycles=2, x_init=False):
    """Snapshot buffer (cycles+1, effective) for script s of design kind."""
    d = design(kind)
    v = state.random_stimulus_states(s, d, cycles, seed, p_toggle, reset_cycles)
    if s.xprop_enabled:
        v = state.expand_states_for_xprop(v, s)
        if not x_init:
            v[0, s.reg_io_state_size:] = 0  # known initial state
    if s.timing_arrivals_enabled:
        v = state.expand_states_for_arrivals(v, s)
    return np.ascontiguousarray(v)


def constraint_buffer(kind, s, clock_ps=10_000, setup=30, hold=10, seed=5):
    """[clock, per-word setup<<16|hold] with per-DFF clock arrival U[0,300]."""
    return constraint_buffer_for(design(kind), s, clock_ps, setup, hold, seed)


def constraint_buffer_for(d, s, clock_ps=10_000, setup=30, hold=10, seed=5):
    """Same, for a design object (every DFF: setup, hold, clock arrival U[0,300])."""
    from jacquard_b200 import timing
    rng = np.random.default_rng(seed)
    ca = rng.integers(0, 301, size=int(d.num_dffs)).astype(np.int16)
    return timing.constraint_buffer(d, s, clock_ps, setup, hold, ca)
