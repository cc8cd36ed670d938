"""The benchmark's configuration choices on the host (no GPU): the script
form of each work-item form and when the learned cut is taken."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def small_design():
    # the benchmark's SoC generator at 1/32 of its size
    return bench.build_design(seed=2, clusters=16, n_dff=200_000 * 16 // 512)


def per_stage_counts(s):
    return np.bincount(np.asarray(s.stage_block_part)[:, 0], minlength=s.num_major_stages)


def test_octet_script_is_one_round_of_octet_items():
    """Octet items (8 lane words per item on 8 lane words): at most one
    partition per CTA per major stage, every stage flat (the compact form),
    and the heuristic cut, since the octet model's recorded cut loses."""
    s, per_item = bench.default_batched_script(small_design(), blocks=148, lanes=8, per_item=8)
    assert per_item == 8
    assert per_stage_counts(s).max() <= 148
    assert int(s.features[:, 14].max()) <= 1
    assert bench.learned_wins(148, 8) is False


def test_lane_pair_script_is_one_round_of_lane_pair_items():
    """Lane pairs on 8 lane words: 4 items per partition, so at most 37
    partitions per stage on 148 CTAs."""
    s, per_item = bench.default_batched_script(small_design(), blocks=148, lanes=8, per_item=2)
    assert per_item == 2
    assert per_stage_counts(s).max() <= 37
    assert int(s.features[:, 14].max()) <= 1


def test_level_split_option():
    """--split cuts the design's 80 levels into major stages of that many
    levels."""
    d = small_design()
    s4 = bench.build_script(d, 148, target_parts=37)
    s5 = bench.build_script(d, 148, target_parts=37, split_every=5)
    assert s4.num_major_stages == 20 and s5.num_major_stages == 16


def test_traffic_figure_follows_code_not_comments(tmp_path):
    """The recorded ncu traffic is reported while the kernel's code is the
    captured one: comment and blank-line edits keep the hash, a code change
    alters it."""
    src = "// header\nint f(int a) {  /* note */\n  return a + 1;  // inc\n}\n"
    a = tmp_path / "a.cu"
    b = tmp_path / "b.cu"
    c = tmp_path / "c.cu"
    a.write_text(src)
    b.write_text("// another header\n\n" + src.replace("// inc", "// increment"))
    c.write_text(src.replace("a + 1", "a + 2"))
    assert bench.kernel_code_hash(str(a)) == bench.kernel_code_hash(str(b))
    assert bench.kernel_code_hash(str(a)) != bench.kernel_code_hash(str(c))
    assert bench.measured_traffic_per_cycle() is not None  # the current kernel's capture
