"""Front end: scripts are valid, and the oracle running a script computes the
same DFF states and outputs as a gate-level simulation of the design."""
import ctypes

import numpy as np
import pytest

import cases
import oracle_lib
from jacquard_b200 import state
from jacquard_b200._native import load


def netlist_check(kind, s, cycles=24, seed=3):
    d = cases.design(kind)
    vals = state.stimulus_inputs(s, d, cycles, seed, 0.5, 2)
    st = state.pack_inputs(s, vals).reshape(-1).copy()
    oracle_lib.simulate(s, st, cycles, s.reg_io_state_size)
    st = st.reshape(cycles + 1, -1)
    dpos = state.dff_positions(s, d)
    dff0 = state.bits_at(st[:1], dpos)[0]
    dff, pov = oracle_lib.aig_simulate(d, s.input_layout, vals, dff0, cycles)
    assert np.array_equal(state.bits_at(st, dpos), dff)
    assert np.array_equal(state.bits_at(st[1:], state.po_positions(s, d)), pov[1:])


@pytest.mark.parametrize("kind,nb,split", [
    ("tiny", 1, ()), ("tiny", 4, ()), ("tiny", 148, (5,)), ("tiny", 7, (3, 6, 9)),
    ("small", 64, (8, 16, 24)), ("sram", 16, (8,)), ("sram", 3, ()),
])
def test_script_computes_the_design(kind, nb, split):
    netlist_check(kind, cases.script(kind, nb, split))


def test_soc_like_design_with_major_stages():
    netlist_check("soc_mini", cases.script("soc_mini", 148, (20, 40, 60)), cycles=12)


@pytest.mark.parametrize("kind,split,parts", [
    ("soc_mini", (20, 40, 60), 5), ("small", (8, 16, 24), 3), ("sram", (8,), 2),
])
def test_balanced_partitions_compute_the_design(kind, split, parts):
    """target_parts: at most `parts` partitions per major stage, the cone
    bound taken as small as that allows, and the script still computes the
    design."""
    d = cases.design(kind)
    s = d.build_script(num_blocks=16, level_split=split, merge_passes=0, target_parts=parts)
    assert validate(s) == (0, "")
    stage = np.asarray(s.stage_block_part)[:, 0]
    per_stage = np.bincount(stage, minlength=s.num_major_stages)
    assert per_stage.max() <= parts
    ref = d.build_script(num_blocks=16, level_split=split)
    ands, ref_ands = s.features[:, 1], ref.features[:, 1]
    ref_stage = np.asarray(ref.stage_block_part)[:, 0]
    for ms in range(s.num_major_stages):
        # every stage's logic is covered; the largest partition is no larger
        # than the default partitioner's when that one used no more of them
        if (ref_stage == ms).sum() <= per_stage[ms]:
            assert ands[stage == ms].max() <= ref_ands[ref_stage == ms].max()
    netlist_check(kind, s, cycles=12)


@pytest.mark.parametrize("parts", [1, 1000])
def test_balanced_partition_count_extremes(parts):
    """One partition per stage, and more allowed partitions than endpoints
    (the bound falls to single endpoints' cones)."""
    d = cases.design("tiny")
    s = d.build_script(num_blocks=4, level_split=(5,), merge_passes=0, target_parts=parts)
    assert validate(s) == (0, "")
    per_stage = np.bincount(np.asarray(s.stage_block_part)[:, 0], minlength=s.num_major_stages)
    assert per_stage.max() <= parts
    if parts == 1:
        assert (per_stage == 1).all()
    else:
        assert s.features[:, 1].max() <= 32  # one endpoint's cone (4-5 levels)
    netlist_check("tiny", s, cycles=12)


def test_learned_refinement_keeps_the_design():
    """With a cost model the balanced partitioner moves endpoints between
    neighbouring partitions; every endpoint stays computed."""
    import os
    from jacquard_b200 import costmodel
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                        "jacquard_b200", "trained", "costmodel.npz")
    d = cases.design("soc_mini")
    s = d.build_script(num_blocks=16, level_split=(20, 40, 60), merge_passes=0,
                       target_parts=5, cost_model=costmodel.packed_from_file(path))
    assert validate(s) == (0, "")
    assert np.bincount(np.asarray(s.stage_block_part)[:, 0]).max() <= 5
    assert int(s.features[:, 14].max()) <= 1
    netlist_check("soc_mini", s, cycles=12)


def validate(s, words=None, data=None, rio=None):
    from jacquard_b200.frontend import _lib
    L = _lib()
    bs = np.ascontiguousarray(s.blocks_start, np.uint64)
    bd = np.ascontiguousarray(s.blocks_data if data is None else data, np.uint32)
    err = ctypes.create_string_buffer(256)
    vp = ctypes.c_void_p
    r = L.jqf_validate(vp(bs.ctypes.data), ctypes.c_size_t(s.num_blocks), ctypes.c_size_t(s.num_major_stages),
                       vp(bd.ctypes.data), ctypes.c_size_t(bd.size),
                       ctypes.c_uint32(s.reg_io_state_size if rio is None else rio),
                       ctypes.c_uint32(s.sram_storage_size),
                       ctypes.c_size_t(words or s.reg_io_state_size), err, 256)
    return r, err.value.decode()


def test_validator_accepts_built_scripts_and_rejects_corruption():
    s = cases.script("sram", 16, (8,))
    assert validate(s) == (0, "")
    # global-read index past the state
    bad = s.blocks_data.copy()
    first = int(s.blocks_start[0])
    while bad[first] == 0:
        first += 256
    R = int(bad[first + 6])
    assert R > 0
    t = int(np.nonzero(bad[first + 256 + 1:first + 256 + 512:2])[0][0])
    bad[first + 256 + 2 * t] = s.reg_io_state_size + 5
    assert validate(s, data=bad)[0] != 0
    # shuffle index past the 8192 bits
    bad = s.blocks_data.copy()
    bad[first + 256 + 512 * R] = 9000
    assert validate(s, data=bad)[0] != 0
    # IO range past the state
    assert validate(s, rio=1)[0] != 0


def partitions(s):
    """(offset, ns, R, nio, nsr, nd) of every partition of a script."""
    bd = s.blocks_data
    out = []
    for b in range(s.num_blocks * s.num_major_stages):
        off = int(s.blocks_start[b])
        while int(bd[off]):
            ns, R = int(bd[off]), int(bd[off + 6])
            out.append((off, ns, R, int(bd[off + 2]), int(bd[off + 4]), int(bd[off + 7])))
            last = int(bd[off + 1])
            off += 256 + 512 * R + 5120 * (ns + 2)
            if last:
                break
    return out


def test_validator_rejects_out_of_range_kernel_indices():
    """Indices the kernels dereference without further checks: more than 32
    global-read bits for one thread, writeout permutation entries past
    num_ios*32, SRAM address bits 13..15 not forced to 0."""
    s = cases.script("sram", 16, (8,))
    parts = partitions(s)
    off, ns, R, nio, nsr, nd = next(p for p in parts if p[2] > 0)
    # global read: 33 bits for thread 0 (two full masks)
    bad = s.blocks_data.copy()
    bad[off + 256: off + 256 + 2] = (0, 0xFFFFFFFF)
    if R > 1:
        bad[off + 256 + 512: off + 256 + 512 + 2] = (0, 1)
        assert validate(s, data=bad)[0] != 0
    # clock-enable permutation entry 0 (q = 0) pointing at slot nio
    bad = s.blocks_data.copy()
    ck = off + 256 + 512 * R + 5120 * (ns + 1)
    bad[ck] = (bad[ck] & 0xFFFF0000) | (nio * 32)
    r, msg = validate(s, data=bad)
    assert r != 0 and "permutation" in msg
    # SRAM read address bit 13 left live
    off, ns, R, nio, nsr, nd = next(p for p in parts if p[4] > 0)
    bad = s.blocks_data.copy()
    fl = off + 256 + 512 * R + 5120 * ns + 4096
    bad[fl + 1] &= ~np.uint32(1 << 13)
    r, msg = validate(s, data=bad)
    assert r != 0 and "SRAM address" in msg


def test_xprop_classification_marks_partitions():
    s = cases.script("sram", 16, (8,), xprop=True)
    assert s.partition_x_capable.any()
    assert s.xprop_state_offset == s.reg_io_state_size
    bd = s.blocks_data
    for stage in range(s.num_major_stages):
        for b in range(s.num_blocks):
            off = int(s.blocks_start[stage * s.num_blocks + b])
            if bd[off] == 0:
                continue
            assert bd[off + 9] == s.reg_io_state_size


def test_timing_delays_are_injected():
    s = cases.script("sram", 16, (8,), timing_seed=9)
    # every boomerang flag chunk padding word holds a delay in [0, 65535]
    bd = s.blocks_data
    seen = 0
    for stage in range(s.num_major_stages):
        for b in range(s.num_blocks):
            off = int(s.blocks_start[stage * s.num_blocks + b])
            while bd[off]:
                ns, R = int(bd[off]), int(bd[off + 6])
                ch = off + 256 + 512 * R
                for k in range(ns):
                    pad = bd[ch + 5120 * k + 4096 + 3: ch + 5120 * k + 5120: 4]
                    seen += int((pad > 0).sum())
                    assert (pad <= 65535).all()
                last = bd[off + 1]
                off = ch + 5120 * (ns + 2)
                if last:
                    break
    assert seen > 0
