"""Autotuner search logic (host only): a stand-in timer replaces the device
runs, so the sweep's choices can be checked without a GPU."""
from jacquard_b200 import autotune


def fake_timer(design, split_every, cone, blocks, window, lanes, parts=0, per_item=0, **kw):
    # balanced partitions, octet items and a 4-level split are fastest here;
    # more blocks are slower; 64-cycle windows are best; octet items do not
    # fit a 3-level split
    if per_item == 8 and split_every == 3:
        raise ValueError("octet items need every partition within the slots")
    rate = 1e5 * (1.5 if parts else 1.0) * (1.2 if split_every == 4 else 1.0)
    rate *= 1.1 if per_item == 8 else 1.0
    rate /= 1 + (blocks - 148) / 1000
    rate *= {1: 0.5, 16: 1.0, 64: 1.1, 256: 1.05}[window]
    if cone == 512 and split_every == 10:
        raise RuntimeError("a partition that cannot be packed")
    return dict(split_every=split_every, cone=cone, parts=parts, blocks=blocks, window=window,
                lanes=lanes, per_item=per_item, stream_cycles_per_s=rate, us_per_cycle=0.0,
                partitions=0, script_mb=0.0, build_s=0.0)


def test_sweep_tries_balanced_partitions_and_keeps_them():
    best, results = autotune.sweep(None, lanes=8, timer=fake_timer, log=lambda *a: None)
    assert (best["split_every"], best["parts"], best["blocks"], best["window"],
            best["per_item"]) == (4, 148, 148, 64, 8)
    # one balanced lane-pair candidate per split at the default blocks (148
    # CTAs / 4 items per partition), and an octet one where it fits
    bal = [r for r in results if r["parts"] and r["blocks"] == 148 and r["window"] == 16]
    assert sorted(r["split_every"] for r in bal if r["per_item"] != 8) == [3, 4, 5, 8, 10]
    assert sorted(r["split_every"] for r in bal if r["per_item"] == 8) == [4, 5, 8, 10]
    # the block sweep keeps the balanced octet mode and rescales its count
    assert any(r["blocks"] == 296 and r["parts"] == 296 and r["per_item"] == 8 for r in results)
    # a configuration that fails to build or to fit is skipped, not fatal
    assert not any(r["split_every"] == 10 and r["cone"] == 512 for r in results)


def test_sweep_without_octets_keeps_lane_pairs():
    """With a lane count that octet items cannot divide, the sweep runs lane
    pairs only and keeps the balanced lane-pair cut."""
    best, results = autotune.sweep(None, lanes=6, timer=fake_timer, log=lambda *a: None)
    assert not any(r["per_item"] == 8 for r in results)
    assert (best["split_every"], best["parts"], best["blocks"]) == (4, 49, 148)
    assert any(r["blocks"] == 296 and r["parts"] == 98 for r in results)


def test_balanced_parts():
    assert autotune.balanced_parts(148, 8) == 37
    assert autotune.balanced_parts(148, 8, 8) == 148
    assert autotune.balanced_parts(148, 1) == 148
    assert autotune.balanced_parts(3, 8) == 1
