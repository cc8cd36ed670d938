"""Autotuner search logic (host only): a stand-in timer replaces the device
runs, so the sweep's choices can be checked without a GPU."""
from jacquard_b200 import autotune


def fake_timer(design, split_every, cone, blocks, window, lanes, parts=0, **kw):
    # balanced partitions and a 4-level split are fastest here; more blocks
    # are slower; 64-cycle windows are best
    rate = 1e5 * (1.5 if parts else 1.0) * (1.2 if split_every == 4 else 1.0)
    rate /= 1 + (blocks - 148) / 1000
    rate *= {1: 0.5, 16: 1.0, 64: 1.1, 256: 1.05}[window]
    if cone == 512 and split_every == 10:
        raise RuntimeError("a partition that cannot be packed")
    return dict(split_every=split_every, cone=cone, parts=parts, blocks=blocks, window=window,
                lanes=lanes, stream_cycles_per_s=rate, us_per_cycle=0.0, partitions=0,
                script_mb=0.0, build_s=0.0)


def test_sweep_tries_balanced_partitions_and_keeps_them():
    best, results = autotune.sweep(None, lanes=8, timer=fake_timer, log=lambda *a: None)
    assert (best["split_every"], best["parts"], best["blocks"], best["window"]) == (4, 37, 148, 64)
    # one balanced candidate per split at the default blocks: one round of
    # lane-pair items (148 CTAs / 4 items per partition)
    bal = [r for r in results if r["parts"] and r["blocks"] == 148 and r["window"] == 16]
    assert sorted(r["split_every"] for r in bal) == [3, 4, 5, 8, 10]
    # the block sweep keeps the balanced mode and rescales its count
    assert any(r["blocks"] == 296 and r["parts"] == 74 for r in results)
    assert any(r["blocks"] == 592 and r["parts"] == 148 for r in results)
    # a configuration that fails to build is skipped, not fatal
    assert not any(r["split_every"] == 10 and r["cone"] == 512 for r in results)


def test_balanced_parts():
    assert autotune.balanced_parts(148, 8) == 37
    assert autotune.balanced_parts(148, 1) == 148
    assert autotune.balanced_parts(3, 8) == 1
