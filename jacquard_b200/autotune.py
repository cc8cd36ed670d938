"""Autotuner for the batched interpreter on one design: sweeps the level
split granularity, the partitioner's cone target (partition size), the number
of script blocks and the cycles per launch, timing each configuration on the
device with CUDA events, and returns the fastest.

Each configuration is a full script build (host) plus a short timed run; the
result records the stimulus-cycles/s of every point so the choice is
reproducible.
"""
import itertools
import time

import numpy as np
import torch

from . import batched


def time_config(design, split_every, cone, blocks, window, lanes, cost_model=None, reps=2,
                device="cuda"):
    depth_split = tuple(range(split_every, 80, split_every))
    t0 = time.perf_counter()
    s = design.build_script(num_blocks=blocks, level_split=depth_split, xprop=True,
                            target_cone=cone, cost_model=cost_model)
    build_s = time.perf_counter() - t0
    B = batched.BatchedSim(s, lanes, device=device)
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
    return dict(split_every=split_every, cone=cone, blocks=blocks, window=window, lanes=lanes,
                stream_cycles_per_s=rate, us_per_cycle=ms * 1e3 / window,
                partitions=s.num_partitions, script_mb=s.script_words_per_cycle() * 4 / 1e6,
                build_s=build_s)


def sweep(design, splits=(5, 8, 10), cones=(512, 2000, 6000, 8000), blocks=(148, 296, 592),
          windows=(1, 16, 64, 256), lanes=8, budget_s=600.0, log=print):
    """Coarse-to-fine: (split, cone) at the default blocks/window, then blocks
    and window around the best point.  Stops when budget_s is spent."""
    t_start = time.perf_counter()
    results = []

    def run(**kw):
        if time.perf_counter() - t_start > budget_s:
            return None
        try:
            r = time_config(design, lanes=lanes, **kw)
        except RuntimeError as e:  # a partition that cannot be packed
            log(f"  skip {kw}: {e}")
            return None
        results.append(r)
        log(f"  {r['split_every']:>2} {r['cone']:>5} {r['blocks']:>4} {r['window']:>4}: "
            f"{r['stream_cycles_per_s']:>12.0f} stream-cycles/s  ({r['partitions']} parts, "
            f"{r['script_mb']:.1f} MB script, build {r['build_s']:.1f}s)")
        return r

    for sp, cone in itertools.product(splits, cones):
        run(split_every=sp, cone=cone, blocks=blocks[0], window=16)
    best = max(results, key=lambda r: r["stream_cycles_per_s"])
    for nb in blocks[1:]:
        run(split_every=best["split_every"], cone=best["cone"], blocks=nb, window=16)
    best = max(results, key=lambda r: r["stream_cycles_per_s"])
    for w in windows:
        if w != 16:
            run(split_every=best["split_every"], cone=best["cone"], blocks=best["blocks"], window=w)
    best = max(results, key=lambda r: r["stream_cycles_per_s"])
    return best, results
