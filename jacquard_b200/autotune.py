"""Autotuner for the batched interpreter on one design: sweeps the level
split granularity, the partition size (the partitioner's cone target, or its
balanced mode with one round of work items per major stage: lane pairs, or
octet items when the lane count allows them and the script fits), the number
of script blocks and the cycles per launch, timing each configuration on the
device with CUDA events, and returns the fastest.

Each configuration is a full script build (host) plus a short timed run; the
result records the stimulus-cycles/s of every point so the choice is
reproducible.
"""
import time

import numpy as np
import torch

from . import batched


def balanced_parts(blocks, lanes, per_item=2):
    """Partitions per major stage for one round of work items: each
    partition makes lanes / per_item items (lane pairs: 2, octets: 8), one
    per CTA."""
    return max(1, blocks // max(1, lanes // per_item))


def time_config(design, split_every, cone, blocks, window, lanes, cost_model=None, reps=2,
                device="cuda", parts=0, per_item=0):
    """cone: the partitioner's cone target; parts > 0 selects balanced mode
    (at most `parts` partitions per major stage, no merges) instead.
    per_item: lane words per work item (0: the library's choice, 8: octet
    items; ValueError when the script does not fit them)."""
    depth_split = tuple(range(split_every, 80, split_every))
    t0 = time.perf_counter()
    s = design.build_script(num_blocks=blocks, level_split=depth_split, xprop=True,
                            target_cone=cone, cost_model=cost_model,
                            merge_passes=0 if parts else 1, target_parts=parts)
    build_s = time.perf_counter() - t0
    B = batched.BatchedSim(s, lanes, device=device, lanes_per_item=per_item)
    B.load_state(np.zeros((lanes, B.sig), np.uint32))
    B.reset_sram()
    B.run(None, 2)
    torch.cuda.synchronize()
    assert B.status() == 0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        B.run(None, window)
    e1.record()
    torch.cuda.synchronize()
    assert B.status() == 0
    ms = e0.elapsed_time(e1) / reps
    rate = 32 * lanes * window / (ms / 1e3)
    return dict(split_every=split_every, cone=cone, parts=parts, blocks=blocks, window=window,
                lanes=lanes, per_item=per_item,
                stream_cycles_per_s=rate, us_per_cycle=ms * 1e3 / window,
                partitions=s.num_partitions, script_mb=s.script_words_per_cycle() * 4 / 1e6,
                build_s=build_s)


def sweep(design, splits=(3, 4, 5, 8, 10), cones=(512, 2000, 6000, 8000),
          blocks=(148, 296, 592), windows=(1, 16, 64, 256), lanes=8, budget_s=600.0, log=print,
          timer=None):
    """Coarse-to-fine: (split, partition size) at the default blocks/window,
    then blocks and window around the best point.  Partition sizes are the
    cone targets plus balanced mode (cone 0 in the results) for lane-pair
    items and, when lanes is a multiple of 8, for octet items (per_item 8).
    Stops when budget_s is spent.  `timer` replaces time_config (same
    keywords)."""
    timer = timer or time_config
    t_start = time.perf_counter()
    results = []

    def run(**kw):
        if time.perf_counter() - t_start > budget_s:
            return None
        try:
            r = timer(design, lanes=lanes, **kw)
        except (RuntimeError, ValueError) as e:  # cannot be packed / does not fit octets
            log(f"  skip {kw}: {e}")
            return None
        results.append(r)
        size = f"{r['parts']}/st" if r["parts"] else str(r["cone"])
        if r.get("per_item") == 8:
            size += " oct"
        log(f"  {r['split_every']:>2} {size:>6} {r['blocks']:>4} {r['window']:>4}: "
            f"{r['stream_cycles_per_s']:>12.0f} stream-cycles/s  ({r['partitions']} parts, "
            f"{r['script_mb']:.1f} MB script, build {r['build_s']:.1f}s)")
        return r

    for sp in splits:
        for cone in cones:
            run(split_every=sp, cone=cone, blocks=blocks[0], window=16)
        run(split_every=sp, cone=0, blocks=blocks[0], window=16,
            parts=balanced_parts(blocks[0], lanes))
        if lanes % 8 == 0:
            run(split_every=sp, cone=0, blocks=blocks[0], window=16,
                parts=balanced_parts(blocks[0], lanes, 8), per_item=8)
    best = max(results, key=lambda r: r["stream_cycles_per_s"])

    def size_of(r, nb):  # the best point's partition size and item form at nb blocks
        pi = r.get("per_item", 0)
        return dict(cone=r["cone"], per_item=pi,
                    parts=balanced_parts(nb, lanes, pi or 2) if r["parts"] else 0)

    for nb in blocks[1:]:
        run(split_every=best["split_every"], blocks=nb, window=16, **size_of(best, nb))
    best = max(results, key=lambda r: r["stream_cycles_per_s"])
    for w in windows:
        if w != 16:
            run(split_every=best["split_every"], blocks=best["blocks"], window=w,
                cone=best["cone"], parts=best["parts"], per_item=best.get("per_item", 0))
    best = max(results, key=lambda r: r["stream_cycles_per_s"])
    return best, results
