"""Train the partition cost model on timings measured by the simulator.

  python -m jacquard_b200.train_costmodel [--samples 20000] [--steps 2000]
         [--out jacquard_b200/trained/costmodel.npz] [--per-item 8]

1. Builds scripts of seeded SoC-family designs (the SoC workload's generator at
   several sizes and seeds) with varied level splits and balanced partition
   counts per major stage.
2. Runs each on the batched interpreter in octet work items (8 lane words
   per item, the batched workload's form; --per-item 2 for lane pairs) with
   per-partition timing (`part_cycles`, which leaves out the grid-barrier
   wait) and records log(mean SM cycles per work item) next to the
   partition's 24 features.
3. Trains the MLP with Adam (lr 1e-3, batch 512) on the GPU kernels.
4. Evaluates on fresh designs: balanced partitions without and with the
   learned cut choice (each major stage is cut with several weights of a
   chunk's inputs against its gates, and the cut whose slowest partition
   the model predicts fastest is kept), device-timed stimulus-cycles/s of
   the batched interpreter on the same random stimulus, and every DFF and
   output value of both runs compared bit for bit.
"""
import argparse
import json
import os
import time

import numpy as np
import torch

from . import batched, costmodel, frontend, state

HERE = os.path.dirname(os.path.abspath(__file__))


def build(design, split_every, parts, blocks=148, cost_model=None):
    return design.build_script(num_blocks=blocks, level_split=tuple(range(split_every, 80, split_every)),
                               xprop=True, cost_model=cost_model, merge_passes=0, target_parts=parts)


def measure(design, split_every, parts, lanes=8, cycles=4, blocks=148, per_item=8):
    s = build(design, split_every, parts, blocks)
    try:
        B = batched.BatchedSim(s, lanes, lanes_per_item=per_item)
    except ValueError as e:  # octet items do not fit this script
        raise RuntimeError(str(e)) from e
    B.load_state(np.zeros((lanes, B.sig), np.uint32))
    B.reset_sram()
    pc = torch.zeros(s.num_partitions, dtype=torch.int64, device="cuda")
    B.run(None, 1)
    B.run(None, cycles, part_cycles=pc)
    torch.cuda.synchronize()
    assert B.status() == 0
    t_item = pc.cpu().numpy().astype(np.float64) / ((lanes // per_item) * cycles)
    ok = t_item > 0
    return s.features[ok], np.log(t_item[ok]).astype(np.float32)


def collect(target, seed0=100, log=print, per_item=8):
    feats, ys = [], []
    rng = np.random.default_rng(seed0)
    n = 0
    k = 0
    while n < target:
        clusters = int(rng.choice([64, 128, 256]))
        d = frontend.Design(frontend.soc_params(seed=seed0 + k, n_clusters=clusters,
                                                n_dff=200_000 * clusters // 512, n_sram=4))
        split = int(rng.choice([3, 4, 5]))
        parts = int(rng.choice([37, 74, 111, 148] if per_item == 8 else [12, 18, 24, 30, 37]))
        try:
            f, y = measure(d, split, parts, per_item=per_item)
        except RuntimeError as e:
            log(f"  skip: {e}")
            k += 1
            continue
        feats.append(f)
        ys.append(y)
        n += len(y)
        k += 1
        log(f"  design {k}: {clusters} clusters, split {split}, {parts} per stage: {len(y)} partitions ({n} total)")
    return np.concatenate(feats)[:target], np.concatenate(ys)[:target]


def _lane_stimulus(script, design, lanes, cycles, seed):
    """(cycles+1, lanes, input signals) lane words: every primary input of
    every stream toggles with probability 1/4 per cycle, the clock flag is 1,
    the reset input is 1 for the first 4 snapshots."""
    rng = np.random.default_rng(seed)
    lay = np.asarray(script.input_layout)
    pos = state.input_positions(script)
    n = lay.size
    w = np.empty((cycles + 1, n, lanes), np.uint32)
    cur = rng.integers(0, 2**32, size=(n, lanes), dtype=np.uint32)
    clk = lay == design.clock_flag_pin
    rst = (lay == design.reset_pin) if design.reset_pin else np.zeros(n, bool)
    for c in range(cycles + 1):
        if c:
            cur ^= (rng.integers(0, 2**32, size=(n, lanes), dtype=np.uint32)
                    & rng.integers(0, 2**32, size=(n, lanes), dtype=np.uint32))
        v = cur.copy()
        v[clk] = 0xFFFFFFFF
        v[rst] = 0xFFFFFFFF if c < 4 else 0
        w[c] = v
    rows = np.zeros((cycles + 1, lanes, batched.input_words(script) * 32), np.uint32)
    rows[:, :, pos] = np.swapaxes(w, 1, 2)
    return rows


def evaluate(model_packed, clusters=1024, cycles=5000, lanes=8, seed=4242, split=4, parts=74,
             log=print, per_item=8):
    """Balanced partitions without and with the learned cut choice on one
    fresh design: batched stimulus-cycles/s over `cycles` cycles (device
    time, one launch each), same random stimulus.  Both runs must end with
    the same value in every DFF and primary output of every stream (their
    state layouts differ, the netlist does not): the learned run is checked
    bit for bit against the heuristic one."""
    d = frontend.Design(frontend.soc_params(seed=seed, n_clusters=clusters,
                                            n_dff=200_000 * clusters // 512))
    out = {"design_ands": int(d.num_and), "cycles": cycles, "streams": 32 * lanes,
           "split": split, "parts_per_stage": parts, "lanes_per_item": per_item}
    finals = {}
    for name, cm in (("heuristic", None), ("learned", model_packed)):
        t0 = time.perf_counter()
        s = build(d, split, parts, cost_model=cm)
        bt = time.perf_counter() - t0
        B = batched.BatchedSim(s, lanes, lanes_per_item=per_item)
        rows = _lane_stimulus(s, d, lanes, cycles, seed + 1)
        snap0 = np.zeros((lanes, B.sig), np.uint32)
        snap0[:, :B.in_sigs] = rows[0]
        B.load_state(snap0)
        B.reset_sram(x=False)
        stim = torch.from_numpy(np.ascontiguousarray(rows).reshape(-1).view(np.int32)).cuda()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        B.run(stim, cycles)
        e1.record()
        torch.cuda.synchronize()
        assert B.status() == 0
        ms = e0.elapsed_time(e1)
        fin = B.final_state(cycles).cpu().numpy().view(np.uint32).reshape(lanes, B.sig)
        dq = state.dff_positions(s, d)
        po = state.po_positions(s, d)
        finals[name] = (fin[:, dq], fin[:, po])  # lane words: value of each DFF / output
        out[name] = {"stream_cycles_per_s": 32 * lanes * cycles / (ms / 1e3),
                     "partitions": s.num_partitions,
                     "script_mb_per_cycle": s.script_words_per_cycle() * 4 / 1e6, "build_s": bt}
        log(f"  {name}: {out[name]}")
    out["bit_exact_vs_heuristic"] = bool(
        np.array_equal(finals["heuristic"][0], finals["learned"][0])
        and np.array_equal(finals["heuristic"][1], finals["learned"][1]))
    out["gain"] = out["learned"]["stream_cycles_per_s"] / out["heuristic"]["stream_cycles_per_s"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=20000)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--out", default=None,
                    help="model file (default: trained/costmodel_octet.npz for octet items, "
                         "trained/costmodel.npz for lane pairs)")
    ap.add_argument("--per-item", type=int, default=8, choices=[2, 8],
                    help="lane words per work item timed and evaluated")
    ap.add_argument("--eval-clusters", type=int, default=None,
                    help="held-out design size (default: 512 clusters, 2.3M gates, for octet "
                         "items; 1024 for lane pairs)")
    ap.add_argument("--eval-cycles", type=int, default=5000)
    ap.add_argument("--eval-parts", type=int, default=None,
                    help="partitions per major stage (default: one round of items)")
    ap.add_argument("--eval-only", action="store_true",
                    help="evaluate the model saved at --out (no collection or training)")
    args = ap.parse_args()
    pi = args.per_item
    if args.out is None:
        args.out = os.path.join(HERE, "trained", "costmodel_octet.npz" if pi == 8 else "costmodel.npz")
    # one round of items per major stage on 148 CTAs: 148 partitions of
    # octet items, 37 of lane pairs (4 items each)
    soc_parts = 148 if pi == 8 else 37
    ev_clusters = args.eval_clusters or (512 if pi == 8 else 1024)
    ev_parts = args.eval_parts or (148 if pi == 8 else 74)
    if args.eval_only:
        packed = costmodel.packed_from_file(args.out)
        ev = evaluate(packed, clusters=ev_clusters, cycles=args.eval_cycles, parts=ev_parts,
                      per_item=pi)
        ev_soc = evaluate(packed, clusters=512, cycles=args.eval_cycles, seed=2, parts=soc_parts,
                          per_item=pi)
        print(json.dumps({"eval": ev, "eval_soc2m": ev_soc}))
        return
    t0 = time.time()
    X, y = collect(args.samples, per_item=pi)
    print(f"collected {len(y)} partitions in {time.time() - t0:.0f}s; log-cycles mean {y.mean():.2f} sd {y.std():.2f}")
    perm = np.random.default_rng(0).permutation(len(y))
    ntr = int(0.9 * len(y))
    tr, te = perm[:ntr], perm[ntr:]
    m = costmodel.CostModel(seed=5)
    hist = m.fit(X[tr], y[tr], steps=args.steps, batch=512, lr=1e-3)
    pred = m.predict(X[te])
    mse = float(np.mean((pred - y[te]) ** 2))
    base = float(np.var(y[te]))
    print(f"train loss {hist[0][1]:.3f} -> {hist[-1][1]:.3f}; held-out mse {mse:.4f} (variance {base:.4f}, R^2 {1 - mse / base:.3f})")
    m.save(args.out)
    ev = evaluate(m.pack(), clusters=ev_clusters, cycles=args.eval_cycles, parts=ev_parts,
                  per_item=pi)
    # the SoC workload's own design (2M gates, seed 2), one round of items
    ev_soc = evaluate(m.pack(), clusters=512, cycles=args.eval_cycles, seed=2, parts=soc_parts,
                      per_item=pi)
    summary = {"samples": int(len(y)), "steps": args.steps, "per_item": pi,
               "loss_start": hist[0][1],
               "loss_end": hist[-1][1], "heldout_mse": mse, "heldout_var": base,
               "heldout_r2": 1 - mse / base, "eval": ev, "eval_soc2m": ev_soc}
    with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
        json.dump(summary, f, indent=1)
    print(json.dumps(summary))


if __name__ == "__main__":
    main()
