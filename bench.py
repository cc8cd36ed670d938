"""Benchmark: stimulus-cycles/s of the interpreter on the SoC-scale synthetic
design (2^21 clustered random ANDs + reset gates, depth 80, 200k DFFs, 16
single-port 1024x32 SRAMs, 128 PIs, X-propagation on, all DFF/SRAM state X at
start, 16 reset cycles then p_toggle = 0.25 stimulus).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]
                  [--mode batched|timed|plain|timed_plain|multi] [--lanes L]
                  [--per-item 8|2] [--window C] [--learned auto|on|off]
                  [--split S] [--no-check] [--no-compare]

One step = one launch window of C cycles over all stimulus streams.  The
batched mode partitions every major stage into blocks / (lanes / per-item)
balanced partitions: one round of work items, octet items (8 lane words,
the default) or lane pairs.  With --learned the cost model trained on that
item form chooses each stage's cut (auto: only when its committed training
summary shows it winning, bit-exact, on this design in this configuration).
`value` is device-timed throughput with inputs resident in HBM; `e2e` is the
same through the C ABI with host buffers copied in and out inside the timed
region; `parity` is the replay of two sampled streams of both timed regions
on the plain interpreter; `compare` times the single-stream plain
interpreter on the same design.
--impl reference runs the reference's CPU interpreter path (this repository's
C restatement of it, oracle/) on the host cores.  Multi-GPU: independent
replicas (one design + its own stimulus streams per rank), weak scaling.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(HERE, "tests"))

LEVEL_SPLIT = tuple(range(4, 80, 4))
TARGET_CONE = 6000
RESET_CYCLES = 16
P_TOGGLE = 0.25
METRIC = "stimulus-cycles/s bit-exact: batched+learned vs plain kernel vs CPU, 1 B200"
SOC = "soc-2M: 2^21 clustered ANDs + reset gates, depth 80, 200k DFF, 16 SRAM 1024x32, X-prop"
WORKLOADS = {
    "batched": SOC,
    "plain": SOC,
    "timed": SOC + ", per-pin delays U[20,200] ps, setup 30 / hold 10 ps, 10 ns clock, "
                   "DFF clock arrival U[0,300] ps, setup/hold checks per stream, events drained per window",
    "timed_plain": SOC + ", per-pin delays U[20,200] ps, setup 30 / hold 10 ps, 10 ns clock, "
                         "DFF clock arrival U[0,300] ps, one stream, arrivals + events drained per window",
    "multi": "12 SoC-family designs, 50k-4M AND nodes log-uniform, X-prop, one graph-captured launch",
}


PROFILE_BATCHED = os.path.join(HERE, "profiles", "batched_kernel_soc2M_xprop.md")
KERNEL_SRC = os.path.join(HERE, "jacquard_b200", "csrc", "sim_batched.cu")


def kernel_code_hash(path=KERNEL_SRC):
    """sha256 of a kernel source with its comments, trailing blanks and
    empty lines removed: it changes with the code, not with comment edits."""
    import hashlib
    import re
    with open(path) as f:
        src = f.read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    lines = [ln.rstrip() for ln in src.splitlines() if ln.strip()]
    return hashlib.sha256("\n".join(lines).encode()).hexdigest()


def measured_traffic_per_cycle():
    """DRAM bytes (read + write) per simulated cycle of the 256-stream batched
    workload, from the ncu capture summarised in the kernel's profile (a
    line `traffic_bytes_per_cycle: B source_sha256: H`, H the prefix of
    kernel_code_hash of the captured source), or None when that capture was
    taken of other kernel code."""
    import re
    try:
        with open(PROFILE_BATCHED) as f:
            m = re.search(r"traffic_bytes_per_cycle:\s*([0-9.eE+]+)\s+source_sha256:\s*([0-9a-f]+)",
                          f.read())
        h = kernel_code_hash()
    except OSError:
        return None
    if not m or not h.startswith(m.group(2)):
        return None
    return float(m.group(1))


def peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return float(j.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class Clocks:
    """Samples SM clocks and throttle reasons while the timed region runs
    (NVML, read-only queries, every 20 ms; nvidia-smi when NVML is absent)."""
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu=0):
        self.gpu = gpu
        self.sm, self.sm_max, self.reasons = [], [], set()
        self._stop = threading.Event()
        self._t = None

    def _nvml_loop(self, nv):
        h = nv.nvmlDeviceGetHandleByIndex(self.gpu)
        masks = [(n, getattr(nv, c)) for n, c in self.REASONS]
        while not self._stop.is_set():
            self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
            self.sm_max.append(float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)))
            r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            for n, m in masks:
                if r & m:
                    self.reasons.add(n)
            self._stop.wait(0.02)

    def _smi_loop(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                r = [x.strip() for x in out.split(",")]
                if len(r) >= 9:
                    if r[1].replace(".", "").isdigit():
                        self.sm.append(float(r[1]))
                    if r[2].replace(".", "").isdigit():
                        self.sm_max.append(float(r[2]))
                    for i, (n, _) in enumerate(self.REASONS):
                        if r[5 + i].lower() == "active":
                            self.reasons.add(n)
            except Exception:
                pass
            self._stop.wait(0.2)

    def _loop(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
        except Exception:
            self._smi_loop()
            return
        try:
            self._nvml_loop(nv)
        finally:
            nv.nvmlShutdown()

    def __enter__(self):
        self._t = threading.Thread(target=self._loop, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": float(np.median(self.sm)),
                "sm_max_mhz": max(self.sm_max) if self.sm_max else None,
                "reasons": sorted(self.reasons), "samples": len(self.sm)}


def timed_region_edge(world):
    """Both edges of a timed region: device idle, and every rank there."""
    import torch
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()


def replica_throughput(units, dev_ms, e2e_ms, world, device="cuda"):
    """Whole-job throughput of `world` independent replicas, each processing
    `units`: all ranks' units over the slowest rank's device time (max over
    ranks).  Returns (value, e2e value, dev_ms, e2e_ms) with the max times."""
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([dev_ms, e2e_ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_ms, e2e_ms = t.tolist()
    return world * units / (dev_ms / 1e3), world * units / (e2e_ms / 1e3), dev_ms, e2e_ms


def build_design(seed=2, clusters=512, n_dff=200_000):
    from jacquard_b200 import frontend
    d = frontend.Design(frontend.soc_params(seed=seed, n_clusters=clusters, n_dff=n_dff,
                                            n_sram=16 if clusters >= 16 else 2))
    return d


# Trained partition cost models (jacquard_b200/trained), one per work-item
# form they were timed on: lane pairs and octets.
MODEL_PATHS = {2: os.path.join(HERE, "jacquard_b200", "trained", "costmodel.npz"),
               8: os.path.join(HERE, "jacquard_b200", "trained", "costmodel_octet.npz")}


def learned_model(per_item=2):
    """The cost model trained on `per_item` work items, or None."""
    p = MODEL_PATHS.get(per_item)
    if p is None or not os.path.exists(p):
        return None
    from jacquard_b200 import costmodel
    return costmodel.packed_from_file(p)


def learned_wins(parts_per_stage, lanes_per_item):
    """Whether the committed training summary shows the learned cut beating
    the heuristic on this workload's own design (the 2M-gate SoC, 256
    streams) in the same configuration (partitions per major stage, lane
    words per work item), with the learned run bit-exact against the
    heuristic one.  The benchmark uses the learned cut by default only
    then."""
    m = MODEL_PATHS.get(lanes_per_item)
    if m is None:
        return False
    p = os.path.splitext(m)[0] + ".json"
    if not os.path.exists(m) or not os.path.exists(p):
        return False
    with open(p) as f:
        ev = json.load(f).get("eval_soc2m", {})
    return (bool(ev.get("bit_exact_vs_heuristic")) and ev.get("gain", 0.0) > 1.0
            and ev.get("parts_per_stage") == parts_per_stage
            and ev.get("lanes_per_item", 2) == lanes_per_item)


def default_batched_script(d, blocks=148, lanes=8, per_item=8, learned="auto", split_every=4,
                           input_weight16=0):
    """(script, lanes per item) exactly as the batched mode builds them with
    these options: balanced partitions, one round of work items per major
    stage, the learned cut when `learned` says so."""
    per_stage = blocks // max(1, lanes // per_item)
    use = learned == "on" or (learned == "auto" and split_every == 4 and
                              learned_wins(per_stage, per_item))
    return build_script(d, blocks, cost_model=learned_model(per_item) if use else None,
                        target_parts=per_stage, split_every=split_every,
                        input_weight16=input_weight16), per_item


def build_script(d, num_blocks, xprop=True, cost_model=None, target_parts=0, split_every=4,
                 input_weight16=0):
    """target_parts > 0 cuts each major stage into at most that many
    partitions of balanced cone size in flat stages, without merges: the
    batched kernel then runs every stage as one round of work items, one per
    CTA (a partition makes lanes / (lanes per item) items); a cost model then
    chooses each stage's cut.  Otherwise partitions come from the cone
    target, merged by the learned rule when a model is given.  Major stages
    cover split_every logic levels each; without a model the balanced cut
    weighs each chunk input as input_weight16 / 16 gates."""
    split = LEVEL_SPLIT if split_every == 4 else tuple(range(split_every, 80, split_every))
    return d.build_script(num_blocks=num_blocks, level_split=split, xprop=xprop,
                          target_cone=TARGET_CONE, cost_model=cost_model,
                          merge_passes=0 if target_parts else (3 if cost_model is not None else 1),
                          target_parts=target_parts, input_weight16=input_weight16)


def algorithmic_bytes_per_cycle(s, streams=1, arrivals=False, bit_sliced=False):
    """(script bytes, state bytes) one simulated cycle must move.

    Script: every word of the script (FlattenedScriptV1, empty-block dummies
    included), read once per cycle however many streams share it.  (The
    batched modes report the prepared script's streamed bytes instead:
    prepared_script_bytes.)
    State, per partition (x = 1 on X-capable partitions): the global-read
    bits, the IO words read (old value) and written, the SRAM words (read,
    old word at the write address, write), each with its X copy.
    Plain layout (one stream): a 4-byte state word per non-empty global-read
    word and per IO word, 3 words per SRAM.  Bit-sliced layout (`streams`
    streams, a lane word holding one signal of 32 streams): a lane word per
    selected global-read bit and per IO signal, per 32 streams; SRAM words
    stay per stream."""
    bd = s.blocks_data
    script_words = int(s.blocks_start[-1])
    gr = io = sr = 0
    lane_words = (streams + 31) // 32
    for b in range(s.num_blocks * s.num_major_stages):
        off = int(s.blocks_start[b])
        while True:
            ns = int(bd[off])
            if ns == 0:
                break
            nio, R, nsr, isx = int(bd[off + 2]), int(bd[off + 6]), int(bd[off + 4]), int(bd[off + 8])
            m = bd[off + 256: off + 256 + 512 * R].reshape(-1, 2)[:, 1]
            k = 1 + (1 if isx else 0)
            if bit_sliced:
                bits = int(np.unpackbits(np.ascontiguousarray(m).view(np.uint8)).sum())
                gr += bits * k * lane_words
                io += (2 * k + (1 if arrivals else 0)) * nio * 32 * lane_words
                sr += 3 * nsr * k * streams
            else:
                gr += int(np.count_nonzero(m)) * k * streams
                io += (2 * nio * k + (nio if arrivals else 0)) * streams
                sr += 3 * nsr * k * streams
            last = int(bd[off + 1])
            off += 256 + 512 * R + 5120 * (ns + 2)
            if last:
                break
    return 4 * script_words, 4 * (gr + io + sr)


def prepared_script_bytes(B):
    """Script bytes the batched kernel must stream per simulated cycle, once
    per partition (all streams share them): the metadata (1 KB), a 4-byte
    source entry per global-read slot it loads, and the copied part of each
    chunk of the prepared script (the used head of a compact chunk, the whole
    20 KB chunk otherwise).  The rest of FlattenedScriptV1's fixed-size
    chunks is padding the kernel never reads."""
    bd = B.prepared.cpu().numpy().view(np.uint32)
    bs = np.asarray(B.script.blocks_start, np.int64)
    total = 0
    for e in range(bs.size - 1):
        off = int(bs[e])
        while True:
            ns = int(bd[off])
            if ns == 0:
                break
            R, compact = int(bd[off + 6]), bool(bd[off + 10] & 1)
            chunks = list(range(ns)) + ([ns] if (bd[off + 4] | bd[off + 7]) else []) + [ns + 1]
            total += 1024
            for k in chunks:
                b = int(bd[off + 11 + k]) if compact and k < 116 else 0
                total += b or 5120 * 4
            last = int(bd[off + 1])
            off += 256 + 512 * R + 5120 * (ns + 2)
            if last:
                break
    gr = B.gr_sources.view(-1, 8192)[:B.num_partitions]
    total += 4 * int(((gr != -1) & (gr != -2)).sum().item())  # GR_EMPTY, GR_SKIP
    return total


def stimulus_window(s, d, first_cycle, cycles, seed):
    """Value+X snapshots for cycles [first_cycle, first_cycle+cycles]: inputs
    per snapshot, reset held for the first RESET_CYCLES, X template; snapshot
    0 of the run has every DFF/SRAM word X."""
    from jacquard_b200 import state
    rng = np.random.default_rng(seed)
    vals = state.stimulus_inputs(s, d, first_cycle + cycles, seed, P_TOGGLE, RESET_CYCLES)
    v = state.pack_inputs(s, vals[first_cycle:first_cycle + cycles + 1])
    return np.ascontiguousarray(state.expand_states_for_xprop(v, s))


def run_mine_plain(args, rank, world):
    import torch
    from jacquard_b200 import sim
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    d = build_design(seed=2 + rank, clusters=args.clusters, n_dff=200_000 * args.clusters // 512)
    nb = sim.max_blocks(dev.index)
    nb = min(nb, 148 * 3)
    s = build_script(d, nb)
    W = args.window
    eff = 2 * s.reg_io_state_size
    host = stimulus_window(s, d, 0, W, seed=100 + rank)
    host_pin = torch.from_numpy(host.view(np.int32).reshape(-1)).pin_memory()
    out_pin = torch.empty_like(host_pin).pin_memory()
    ds = sim.DeviceScript(s, dev)
    st = torch.empty(host_pin.numel(), dtype=torch.int32, device=dev)
    n_sram = max(1, s.sram_storage_size)
    sram = torch.zeros(n_sram, dtype=torch.int32, device=dev)
    sram_x = torch.full((n_sram,), -1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        sim.simulate(ds, st, W, eff, sram, sram_x, stream=stream)

    # warmup (device-resident inputs)
    st.copy_(host_pin, non_blocking=True)
    for _ in range(args.warmup):
        st.copy_(host_pin, non_blocking=True)
        step()
    torch.cuda.synchronize()
    assert sim.status(stream) == 0
    # timed: device-resident (value).  Each window rewrites the whole snapshot
    # buffer (W*eff*4 bytes > L2), so no extra flush is needed.
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    with Clocks(dev.index) as ck:
        timed_region_edge(world)
        t0.record(stream)
        for _ in range(args.steps):
            step()
        t1.record(stream)
        timed_region_edge(world)
    dev_ms = t0.elapsed_time(t1)
    assert sim.status(stream) == 0
    # timed e2e: pinned host -> device, kernel, device -> host
    timed_region_edge(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        st.copy_(host_pin, non_blocking=True)
        step()
        out_pin.copy_(st, non_blocking=True)
    e1.record(stream)
    timed_region_edge(world)
    e2e_ms = e0.elapsed_time(e1)
    script_b, state_b = algorithmic_bytes_per_cycle(s)
    return dict(dev_ms=dev_ms, e2e_ms=e2e_ms, cycles_per_step=W, streams=1, clocks=ck.summary(),
                bytes_per_cycle=script_b + state_b, script_bytes=script_b,
                kernel_ms=dev_ms / args.steps,
                h2d=host_pin.numel() * 4, d2h=out_pin.numel() * 4, launches_per_step=2,
                design=dict(ands=int(d.num_and), dffs=int(d.num_dffs), partitions=s.num_partitions,
                            script_mb_per_cycle=script_b / 1e6, rio=s.reg_io_state_size,
                            major_stages=s.num_major_stages, blocks=nb),
                script=s, d=d)


def batched_stimulus(s, d, streams, cycles, seed0, first=0):
    """(cycles+1, lanes, input_signals) input lane words: stream k uses seed
    seed0 + k (reset for the first RESET_CYCLES, then p_toggle inputs)."""
    from jacquard_b200 import batched, state
    words = batched.input_words(s)
    per = np.zeros((streams, cycles + 1, words), np.uint32)
    for k in range(streams):
        vals = state.stimulus_inputs(s, d, first + cycles, seed0 + k, P_TOGGLE, RESET_CYCLES)
        per[k] = state.pack_inputs(s, vals[first:first + cycles + 1])[:, :words]
    return batched.to_batched(per)


class StreamCheck:
    """Bit-exactness self-check of timed batched windows: stream k is
    replayed on the plain interpreter (this library's single-stream kernel,
    the reference's state layout) from the batched state where a timed
    region started, over the same windows, and must end in the same state
    and SRAM contents and record the same outputs in the last window.
    Runs outside the timed regions."""

    def __init__(self, B, s, d, stim, streams):
        import torch
        from jacquard_b200 import sim
        self.B, self.s, self.stim, self.streams = B, s, stim, streams
        self.ds = sim.DeviceScript(s, B.device)
        self.eff = B.sig // 32
        self.words = B.in_sigs // 32

    def _stream(self, lane_major, k):
        """Words (eff,) of stream k from a lane-major (lanes, sig) device tensor."""
        import torch
        lane, bit = divmod(k, 32)
        b = ((lane_major[lane] >> bit) & 1).to(torch.int64).view(-1, 32)
        return ((b << torch.arange(32, device=b.device)).sum(-1) & 0xFFFFFFFF).to(torch.int64)

    def capture(self):
        """The batched state and SRAM of the checked streams, now."""
        import torch
        B = self.B
        cur = B.final_state(0).view(B.lanes, B.sig)  # state_a: every window is even
        sram = B.sram.view(32 * B.lanes, -1)
        sram_x = B.sram_x.view(32 * B.lanes, -1)
        return {k: (self._stream(cur, k), sram[k].clone(), sram_x[k].clone()) for k in self.streams}

    def replay(self, start, end, windows, wave):
        """True when every checked stream, replayed `windows` windows from
        `start`, reaches `end` with the same outputs in the last window."""
        import torch
        from jacquard_b200 import sim
        B, W = self.B, self.stim.shape[0] - 1
        eff, words = self.eff, self.words
        npo = B.n_po
        ok = True
        for k in self.streams:
            lane, bit = divmod(k, 32)
            st0, sram, sram_x = (t.clone() for t in start[k])
            inp = torch.from_numpy(np.ascontiguousarray(
                (self.stim[:, lane, :] >> np.uint32(bit)) & 1).astype(np.int64)).to(B.device)
            inp = (inp.view(W + 1, words, 32) << torch.arange(32, device=B.device)).sum(-1)
            snaps = torch.empty((W + 1, eff), dtype=torch.int64, device=B.device)
            cur = st0.to(torch.int64)
            sram, sram_x = sram.to(torch.int32), sram_x.to(torch.int32)
            for _ in range(windows):
                snaps[:] = cur
                snaps[1:, :words] = inp[1:]
                buf = (snaps - ((snaps >> 31) << 32)).to(torch.int32)  # u32 bits as int32
                sim.simulate(self.ds, buf, W, eff, sram, sram_x)
                if sim.status() != 0:
                    return False
                cur = buf[W].to(torch.int64) & 0xFFFFFFFF
            e_st, e_sram, e_sx = end[k]
            ok &= bool(torch.equal(cur, e_st)) and bool(torch.equal(sram, e_sram)) \
                and bool(torch.equal(sram_x, e_sx))
            if npo:
                po = B.po.to(torch.int64)
                last = (buf[1:].to(torch.int64) & 0xFFFFFFFF).index_select(1, po >> 5)
                want = (last >> (po & 31)) & 1
                got = ((wave.view(W, npo, B.lanes)[:, :, lane] >> bit) & 1).to(torch.int64)
                ok &= bool(torch.equal(got, want))
        return ok


def run_mine_batched(args, rank, world):
    import torch
    from jacquard_b200 import batched, state
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    d = build_design(seed=2 + rank, clusters=args.clusters, n_dff=200_000 * args.clusters // 512)
    lanes = args.lanes
    streams = 32 * lanes
    W = args.window
    assert W % 2 == 0, "even windows keep the final state in buffer A"
    per_item = args.per_item
    while True:
        per_stage = args.blocks // max(1, args.lanes // per_item)  # one round of items
        use_learned = args.learned == "on" or (args.learned == "auto" and args.split == 4 and
                                               learned_wins(per_stage, per_item))
        model = learned_model(per_item) if use_learned else None
        s, _ = default_batched_script(d, args.blocks, args.lanes, per_item, args.learned,
                                      args.split, args.input_weight16)
        po_sig = state.po_positions(s, d)
        try:
            B = batched.BatchedSim(s, lanes, device=dev, po_signals=po_sig,
                                   lanes_per_item=per_item)
            break
        except ValueError:
            if per_item == 2:
                raise
            per_item = 2  # this design does not fit octet items: lane pairs
    # snapshot 0: inputs of cycle 0, every DFF/SRAM word X
    stim = batched_stimulus(s, d, streams, W, seed0=1000 + 7919 * rank)
    snap0 = np.zeros((lanes, B.sig), np.uint32)
    xt = state.xmask_all_state_x(s)
    rio = s.reg_io_state_size
    xt_b = batched.to_batched(np.repeat(xt[None, :], streams, axis=0))
    snap0[:, rio * 32:2 * rio * 32] = xt_b
    snap0[:, :B.in_sigs] = stim[0]
    B.load_state(snap0)
    B.reset_sram(x=True)
    stim_pin = torch.from_numpy(np.ascontiguousarray(stim).reshape(-1).view(np.int32)).pin_memory()
    stim_dev = torch.empty(stim_pin.numel(), dtype=torch.int32, device=dev)
    stim_dev.copy_(stim_pin)
    wave = torch.empty(W * len(po_sig) * lanes, dtype=torch.int32, device=dev)
    wave_pin = torch.empty(wave.numel(), dtype=torch.int32).pin_memory()
    stream = torch.cuda.current_stream(dev)
    check = StreamCheck(B, s, d, stim, (0, streams - 1)) if not args.no_check else None
    for _ in range(args.warmup):
        B.run(stim_dev, W, wave=wave, stream=stream)
    torch.cuda.synchronize()
    assert B.status(stream) == 0
    at_start = check.capture() if check else None
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    with Clocks(dev.index) as ck:
        timed_region_edge(world)
        t0.record(stream)
        for _ in range(args.steps):
            B.run(stim_dev, W, wave=wave, stream=stream)
        t1.record(stream)
        timed_region_edge(world)
    dev_ms = t0.elapsed_time(t1)
    assert B.status(stream) == 0
    at_mid = check.capture() if check else None
    wave_dev_region = wave.clone() if check else None
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    timed_region_edge(world)
    e0.record(stream)
    for _ in range(args.steps):
        stim_dev.copy_(stim_pin, non_blocking=True)
        B.run(stim_dev, W, wave=wave, stream=stream)
        wave_pin.copy_(wave, non_blocking=True)
    e1.record(stream)
    timed_region_edge(world)
    e2e_ms = e0.elapsed_time(e1)
    assert B.status(stream) == 0
    parity = None
    if check:
        at_end = check.capture()
        parity = (check.replay(at_start, at_mid, args.steps, wave_dev_region)
                  and check.replay(at_mid, at_end, args.steps, wave_pin.to(dev)))
    format_b, state_b = algorithmic_bytes_per_cycle(s, streams=streams, bit_sliced=True)
    script_b = prepared_script_bytes(B)
    return dict(dev_ms=dev_ms, e2e_ms=e2e_ms, cycles_per_step=W, streams=streams,
                clocks=ck.summary(), bytes_per_cycle=script_b + state_b, script_bytes=script_b,
                kernel_ms=dev_ms / args.steps, h2d=stim_pin.numel() * 4, d2h=wave_pin.numel() * 4,
                launches_per_step=2, parity=parity,
                traffic_per_cycle=measured_traffic_per_cycle() if args.clusters == 512 else None,
                design=dict(ands=int(d.num_and), dffs=int(d.num_dffs), partitions=s.num_partitions,
                            script_mb_per_cycle=format_b / 1e6,
                            script_read_mb_per_cycle=script_b / 1e6, rio=s.reg_io_state_size,
                            major_stages=s.num_major_stages, blocks=s.num_blocks, lanes=lanes,
                            lanes_per_item=per_item,
                            partitioner="balanced: at most %d per major stage%s"
                            % (per_stage,
                               ", cut chosen by the learned cost model" if model is not None
                               else ", heuristic cut")),
                script=s, d=d)


def timed_design(args, rank, blocks, target_parts=0):
    """The SoC netlist with per-AND-pin delays U[20,200] ps (rise = fall),
    scripted with those delays injected; and its constraint buffer: setup 30
    / hold 10 ps, 10 ns clock, per-DFF clock arrival U[0,300] ps."""
    from jacquard_b200 import timing
    d = build_design(seed=2 + rank, clusters=args.clusters, n_dff=200_000 * args.clusters // 512)
    rng = np.random.default_rng(3)
    n = d.num_pins + 1
    r = rng.integers(20, 201, size=n).astype(np.uint32)
    r[d.kind != 1] = 0
    d.set_delays(r, r)
    s = build_script(d, blocks, target_parts=target_parts)
    zero = np.zeros(n, np.uint32)
    d.set_delays(zero, zero)
    ca = np.random.default_rng(5).integers(0, 301, size=int(d.num_dffs)).astype(np.int16)
    return d, s, timing.constraint_buffer(d, s, 10_000, 30, 10, ca)


def run_mine_timed(args, rank, world):
    """Timed path, 256 streams on the batched interpreter: arrivals (computed
    once, they do not depend on the stream) and setup/hold checks per stream.
    One step = one launch window of cycles plus the drain of its events into
    per-stream violation counts."""
    import torch
    from jacquard_b200 import batched, state, timing
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    d, s, cons = timed_design(args, rank, args.blocks,
                              args.blocks // max(1, args.lanes // args.per_item))
    lanes = args.lanes
    streams = 32 * lanes
    W = args.window
    assert W % 2 == 0
    po_sig = state.po_positions(s, d)
    B = batched.BatchedSim(s, lanes, device=dev, po_signals=po_sig, lanes_per_item=args.per_item)
    cap = args.event_capacity
    tm = batched.Timing(s, cons, cap, device=dev)
    stim = batched_stimulus(s, d, streams, W, seed0=1000 + 7919 * rank)
    snap0 = np.zeros((lanes, B.sig), np.uint32)
    xt = state.xmask_all_state_x(s)
    rio = s.reg_io_state_size
    snap0[:, rio * 32:2 * rio * 32] = batched.to_batched(np.repeat(xt[None, :], streams, axis=0))
    snap0[:, :B.in_sigs] = stim[0]
    B.load_state(snap0)
    B.reset_sram(x=True)
    stim_pin = torch.from_numpy(np.ascontiguousarray(stim).reshape(-1).view(np.int32)).pin_memory()
    stim_dev = torch.empty(stim_pin.numel(), dtype=torch.int32, device=dev)
    stim_dev.copy_(stim_pin)
    wave = torch.empty(W * len(po_sig) * lanes, dtype=torch.int32, device=dev)
    wave_pin = torch.empty(wave.numel(), dtype=torch.int32).pin_memory()
    ev_pin = torch.empty(tm.events.numel(), dtype=torch.int32).pin_memory()
    stream = torch.cuda.current_stream(dev)
    stats = timing.new_stats()
    cyc = [0]

    def step(drain):
        tm.reset_events()
        B.run(stim_dev, W, wave=wave, stream=stream, timing=tm, first_cycle=cyc[0])
        cyc[0] += W
        # the window's records: header, then as many as were written
        ev_pin[:4].copy_(tm.events[:4], non_blocking=True)
        stream.synchronize()
        n = min(int(ev_pin[0]) & 0xFFFFFFFF, cap)
        if n:
            ev_pin[4:4 + 8 * n].copy_(tm.events[4:4 + 8 * n], non_blocking=True)
        wave_pin.copy_(wave, non_blocking=True)
        stream.synchronize()
        if drain:
            recs = ev_pin[4:4 + 8 * n].numpy().view(np.uint32).reshape(-1, 8)
            timing.count_events(recs, int(ev_pin[0]) & 0xFFFFFFFF, cap, stats, streams)

    for _ in range(args.warmup):
        step(True)
    assert B.status(stream) == 0
    # device-timed: launches back to back, the event buffer reset before each
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    with Clocks(dev.index) as ck:
        timed_region_edge(world)
        t0.record(stream)
        for _ in range(args.steps):
            tm.reset_events()
            B.run(stim_dev, W, wave=wave, stream=stream, timing=tm, first_cycle=cyc[0])
            cyc[0] += W
        t1.record(stream)
        timed_region_edge(world)
    dev_ms = t0.elapsed_time(t1)
    assert B.status(stream) == 0
    # end to end: stimulus in, launch, the window's events and outputs out,
    # drained into the violation counts
    timed_region_edge(world)
    w0 = time.perf_counter()
    for _ in range(args.steps):
        stim_dev.copy_(stim_pin, non_blocking=True)
        step(True)
    timed_region_edge(world)
    e2e_ms = (time.perf_counter() - w0) * 1e3
    assert B.status(stream) == 0
    format_b, state_b = algorithmic_bytes_per_cycle(s, streams=streams, bit_sliced=True)
    script_b = prepared_script_bytes(B)
    return dict(dev_ms=dev_ms, e2e_ms=e2e_ms, cycles_per_step=W, streams=streams, clocks=ck.summary(),
                bytes_per_cycle=script_b + state_b, script_bytes=script_b,
                kernel_ms=dev_ms / args.steps,
                h2d=stim_pin.numel() * 4, d2h=wave_pin.numel() * 4, launches_per_step=2,
                design=dict(ands=int(d.num_and), dffs=int(d.num_dffs), partitions=s.num_partitions,
                            script_mb_per_cycle=format_b / 1e6,
                            script_read_mb_per_cycle=script_b / 1e6, rio=rio,
                            major_stages=s.num_major_stages, blocks=s.num_blocks, lanes=lanes,
                            setup_violations=stats["setup_violations"],
                            hold_violations=stats["hold_violations"],
                            events_dropped=stats["events_dropped"],
                            streams_with_violations=int(np.count_nonzero(
                                stats.get("per_stream_hold", np.zeros(1)) +
                                stats.get("per_stream_setup", np.zeros(1))))),
                script=s, d=d)


def run_mine_timed_plain(args, rank, world):
    """Timed path on the plain interpreter: the SoC netlist with per-AND-pin
    delays U[20,200] ps (rise = fall), setup 30 / hold 10 ps, 10 ns clock,
    per-DFF clock arrival U[0,300] ps, X-prop, arrivals on.  One step = one
    window of cycles plus the drain of its setup/hold events into the
    timing report."""
    import torch
    from jacquard_b200 import sim, state, timing
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    d = build_design(seed=2 + rank, clusters=args.clusters, n_dff=200_000 * args.clusters // 512)
    rng = np.random.default_rng(3)
    n = d.num_pins + 1
    r = rng.integers(20, 201, size=n).astype(np.uint32)
    r[d.kind != 1] = 0
    d.set_delays(r, r)
    nb = min(sim.max_blocks(dev.index), 148 * 3)
    s = build_script(d, nb)
    zero = np.zeros(n, np.uint32)
    d.set_delays(zero, zero)
    s.enable_timing_arrivals()
    rio = s.reg_io_state_size
    W = args.window
    cycles = W * (args.steps + args.warmup)
    vals = state.stimulus_inputs(s, d, cycles, 100 + rank, P_TOGGLE, RESET_CYCLES)
    host = state.expand_states_for_arrivals(state.expand_states_for_xprop(state.pack_inputs(s, vals), s), s)
    host[0, rio:2 * rio] = state.xmask_all_state_x(s)
    eff = host.shape[1]
    ca = np.random.default_rng(5).integers(0, 301, size=int(d.num_dffs)).astype(np.int16)
    cons = sim.u32_to_dev(timing.constraint_buffer(d, s, 10_000, 30, 10, ca), dev)
    host_pin = torch.from_numpy(np.ascontiguousarray(host).reshape(-1).view(np.int32)).pin_memory()
    st = torch.empty(host_pin.numel(), dtype=torch.int32, device=dev)
    st.copy_(host_pin)
    ds = sim.DeviceScript(s, dev)
    n_sram = max(1, s.sram_storage_size)
    sram = torch.zeros(n_sram, dtype=torch.int32, device=dev)
    sram_x = torch.full((n_sram,), -1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    cap = 1 << 20
    stats = timing.new_stats()
    ev = sim.new_event_buffer(cap, device=dev)

    def window(c0):
        timing.run_timed(ds, st[c0 * eff:], W, eff, sram, sram_x, cons, W, cap,
                         s.arrival_state_offset, stream=stream, first_cycle=c0, stats=stats,
                         events=ev)

    for k in range(args.warmup):
        window(k * W)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    with Clocks(dev.index) as ck:
        timed_region_edge(world)
        t0.record(stream)
        for k in range(args.steps):
            window((args.warmup + k) * W)
        t1.record(stream)
        timed_region_edge(world)
    dev_ms = t0.elapsed_time(t1)
    # end to end: the window's snapshots host -> device, run + drain, device -> host
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    out_pin = torch.empty(W * eff, dtype=torch.int32).pin_memory()
    timed_region_edge(world)
    e0.record(stream)
    for k in range(args.steps):
        c0 = (args.warmup + k) * W
        st[c0 * eff:(c0 + W + 1) * eff].copy_(host_pin[c0 * eff:(c0 + W + 1) * eff], non_blocking=True)
        window(c0)
        out_pin.copy_(st[(c0 + 1) * eff:(c0 + W + 1) * eff], non_blocking=True)
    e1.record(stream)
    timed_region_edge(world)
    e2e_ms = e0.elapsed_time(e1)
    script_b, state_b = algorithmic_bytes_per_cycle(s, arrivals=True)
    return dict(dev_ms=dev_ms, e2e_ms=e2e_ms, cycles_per_step=W, streams=1, clocks=ck.summary(),
                bytes_per_cycle=script_b + state_b, script_bytes=script_b,
                kernel_ms=dev_ms / args.steps,
                h2d=(W + 1) * eff * 4, d2h=W * eff * 4, launches_per_step=2,
                design=dict(ands=int(d.num_and), dffs=int(d.num_dffs), partitions=s.num_partitions,
                            script_mb_per_cycle=script_b / 1e6, rio=rio,
                            major_stages=s.num_major_stages, blocks=nb,
                            setup_violations=stats["setup_violations"],
                            hold_violations=stats["hold_violations"],
                            events_dropped=stats["events_dropped"]),
                script=s, d=d)


def multi_design_sizes(n=12, lo=50_000, hi=4_000_000, seed=4):
    """AND-node counts log-uniform in [lo, hi] (seeded)."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size=n)).astype(np.int64)


MULTI_OCTET_ANDS = 650  # gates per partition per major stage (multi mode, octet items)


def run_mine_multi(args, rank, world):
    """Twelve designs of log-uniform size in [50k, 4M] AND nodes in one
    persistent launch (scripts relocated into one), replayed from a CUDA
    graph; 8 lane words (256 streams) per design, each stream with its own
    random stimulus (p_toggle 0.25), every design's primary outputs recorded
    each cycle.  Octet items on balanced partitions of about
    MULTI_OCTET_ANDS gates per major stage by default; each super stage's
    items come from the ticket counter.  e2e: the stimulus copied in and the
    waveform copied out around every replay."""
    import torch
    from jacquard_b200 import batched, state
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    sizes = multi_design_sizes()
    scripts, designs, ands = [], [], 0
    for k, n_and in enumerate(sizes.tolist()):
        clusters = max(1, int(round(n_and / 4096)))
        d = build_design(seed=40 + 100 * rank + k, clusters=clusters,
                         n_dff=max(64, 200_000 * clusters // 512))
        ands += int(d.num_and)
        if args.multi_per_item == 8:
            # octet items: balanced partitions of about MULTI_OCTET_ANDS gates
            # per major stage (several per block on large designs), so every
            # partition fits an item's tree slots; items come from tickets
            parts = max(1, -(-int(d.num_and) // (len(LEVEL_SPLIT) + 1) // MULTI_OCTET_ANDS))
            scripts.append(build_script(d, 148, target_parts=parts))
        else:
            scripts.append(build_script(d, 148))
        designs.append(d)
    comb = batched.CombinedScript(scripts)
    lanes = args.lanes
    W = args.window
    po_sig = np.concatenate([[comb.signal(i, int(p)) for p in state.po_positions(s, d)]
                             for i, (s, d) in enumerate(zip(scripts, designs))]).astype(np.int64)
    B = batched.BatchedSim(comb, lanes, device=dev, po_signals=po_sig,
                           lanes_per_item=args.multi_per_item)
    # stimulus: each design's input lane words, concatenated per lane
    rng = np.random.default_rng(4000 + rank)
    rows = np.zeros((W + 1, lanes, B.in_sigs), np.uint32)
    col = 0
    for s, d in zip(scripts, designs):
        pos = state.input_positions(s)
        lay = np.asarray(s.input_layout)
        cur = rng.integers(0, 2**32, size=(lanes, pos.size), dtype=np.uint32)
        for c in range(W + 1):
            if c:
                cur ^= (rng.integers(0, 2**32, size=cur.shape, dtype=np.uint32)
                        & rng.integers(0, 2**32, size=cur.shape, dtype=np.uint32))
            v = cur.copy()
            v[:, lay == d.clock_flag_pin] = 0xFFFFFFFF
            rows[c][:, col + pos] = v
        col += batched.input_words(s) * 32
    B.load_state(np.zeros((lanes, B.sig), np.uint32))  # known zero state; inputs from cycle 1
    B.reset_sram(x=True)
    stim_pin = torch.from_numpy(np.ascontiguousarray(rows).reshape(-1).view(np.int32)).pin_memory()
    stim_dev = torch.empty(stim_pin.numel(), dtype=torch.int32, device=dev)
    stim_dev.copy_(stim_pin)
    wave = torch.empty(W * len(po_sig) * lanes, dtype=torch.int32, device=dev)
    wave_pin = torch.empty(wave.numel(), dtype=torch.int32).pin_memory()
    stream = torch.cuda.Stream(dev)
    with torch.cuda.stream(stream):
        B.run(stim_dev, W, wave=wave, stream=stream)
        stream.synchronize()
        assert B.status(stream) == 0
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            B.run(stim_dev, W, wave=wave, stream=stream)
    for _ in range(args.warmup):
        g.replay()
    torch.cuda.synchronize()
    assert B.status(stream) == 0
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    with Clocks(dev.index) as ck:
        timed_region_edge(world)
        t0.record(stream)
        with torch.cuda.stream(stream):
            for _ in range(args.steps):
                g.replay()
        t1.record(stream)
        timed_region_edge(world)
    dev_ms = t0.elapsed_time(t1)
    assert B.status(stream) == 0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    timed_region_edge(world)
    e0.record(stream)
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            stim_dev.copy_(stim_pin, non_blocking=True)
            g.replay()
            wave_pin.copy_(wave, non_blocking=True)
    e1.record(stream)
    timed_region_edge(world)
    e2e_ms = e0.elapsed_time(e1)
    assert B.status(stream) == 0
    del g
    streams = 32 * lanes * len(scripts)
    per = [algorithmic_bytes_per_cycle(s, streams=32 * lanes, bit_sliced=True) for s in scripts]
    script_b = prepared_script_bytes(B)
    bytes_per_cycle = script_b + sum(p[1] for p in per)
    return dict(dev_ms=dev_ms, e2e_ms=e2e_ms, cycles_per_step=W, streams=streams,
                clocks=ck.summary(), bytes_per_cycle=bytes_per_cycle,
                script_bytes=script_b, kernel_ms=dev_ms / args.steps,
                h2d=stim_pin.numel() * 4, d2h=wave_pin.numel() * 4, launches_per_step=2,
                design=dict(designs=len(scripts), ands=ands, sizes=sizes.tolist(),
                            partitions=int(sum(s.num_partitions for s in scripts)),
                            script_mb_per_cycle=comb.script_words_per_cycle() * 4 / 1e6,
                            lanes=lanes, lanes_per_item=args.multi_per_item or 2, graph=True),
                script=None, d=None)


def compare_kernels(d, args, window=16, reps=3):
    """Single-stream cycles/s of the plain interpreter (reference state layout,
    one stimulus stream) on a script of the same design, built for 296
    blocks: the grid the reference's kernel fits at 2 CTAs per SM."""
    import torch
    from jacquard_b200 import sim
    s = build_script(d, 296)
    eff = 2 * s.reg_io_state_size
    host = stimulus_window(s, d, 0, window, seed=100)
    ds = sim.DeviceScript(s)
    st = sim.u32_to_dev(host.reshape(-1))
    n_sram = max(1, s.sram_storage_size)
    sram = torch.zeros(n_sram, dtype=torch.int32, device="cuda")
    sram_x = torch.full((n_sram,), -1, dtype=torch.int32, device="cuda")
    out = {"window": window, "blocks": 296}
    fn = lambda: sim.simulate(ds, st, window, eff, sram, sram_x)
    fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    out["plain_kernel"] = {"cycles_per_s": window * reps / (e0.elapsed_time(e1) / 1e3), "streams": 1}
    return out


def cpu_baseline(s, d, cycles=8, threads=1):
    import oracle_lib
    host = stimulus_window(s, d, 0, cycles, seed=100)
    st = host.reshape(-1).copy()
    n_sram = max(1, s.sram_storage_size)
    sram = np.zeros(n_sram, np.uint32)
    sram_x = np.full(n_sram, 0xFFFFFFFF, np.uint32)
    t = time.perf_counter()
    oracle_lib.simulate(s, st, cycles, 2 * s.reg_io_state_size, sram=sram, sram_x=sram_x,
                        threads=threads)
    dt = time.perf_counter() - t
    return cycles / dt, dt


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--mode", default="batched",
                    choices=["plain", "batched", "timed", "timed_plain", "multi"],
                    help="batched: 256 streams (default); plain: 1 stream; timed: 256 streams with "
                         "setup/hold checks and event drain; timed_plain: the same on one stream "
                         "(arrivals written); multi: 12 designs in one graph-captured launch")
    ap.add_argument("--event-capacity", type=int, default=1 << 23,
                    help="timed: event records per window")
    ap.add_argument("--window", type=int, default=64)
    ap.add_argument("--lanes", type=int, default=8, help="batched: 32-stream lane words")
    ap.add_argument("--input-weight16", type=int, default=0,
                    help="batched, heuristic cut: gates (x16) a chunk input weighs")
    ap.add_argument("--split", type=int, default=4,
                    help="batched: logic levels per major stage (the autotuner's split)")
    ap.add_argument("--multi-per-item", type=int, default=8, choices=[0, 8],
                    help="multi: 8 runs octet items on balanced partitions (the default), "
                         "0 lets the library pick (lane pairs on cone partitions)")
    ap.add_argument("--per-item", type=int, default=8, choices=[2, 8],
                    help="batched and timed: lane words per work item (8: octets, the "
                         "default; 2: lane pairs)")
    ap.add_argument("--blocks", type=int, default=148, help="batched: script blocks")
    ap.add_argument("--cpu-cycles", type=int, default=160,
                    help="CPU baseline sample: cycles of one stream (about 10 s single-threaded)")
    ap.add_argument("--clusters", type=int, default=512,
                    help="design size in 4096-gate clusters (512 = the 2M-gate workload)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--learned", default="auto", choices=["auto", "on", "off"],
                    help="batched / timed: the learned cost model chooses each stage's balanced "
                         "cut (auto: when its recorded gain on this design is above 1)")
    ap.add_argument("--no-check", action="store_true",
                    help="batched: skip the bit-exactness self-check of the timed windows")
    ap.add_argument("--no-compare", action="store_true",
                    help="batched: skip timing the single-stream plain kernel on the same design")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    from jacquard_b200 import build
    if rank == 0:
        build.build_all()

    if args.impl == "reference":
        if rank != 0:
            return
        d = build_design()
        s = build_script(d, 148)
        threads = os.cpu_count() or 1
        for _ in range(args.warmup):
            cpu_baseline(s, d, cycles=1, threads=threads)
        vals = []
        for _ in range(args.steps):
            v, _ = cpu_baseline(s, d, cycles=args.cpu_cycles, threads=threads)
            vals.append(v)
        v = float(np.mean(vals))
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "stimulus-cycles/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * args.cpu_cycles / v, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
                "config": {"workload": SOC,
                           "sample": f"{args.cpu_cycles} cycles per step, 1 stimulus stream"},
                "cpu_baseline": {"value": v, "unit": "stimulus-cycles/s", "cores": threads,
                                 "kind": "port",
                                 "sample": f"{args.cpu_cycles} cycles x 1 stream of the same workload"},
                "e2e": {"value": v, "unit": "stimulus-cycles/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    runner = {"batched": run_mine_batched, "plain": run_mine_plain, "timed": run_mine_timed,
              "timed_plain": run_mine_timed_plain, "multi": run_mine_multi}[args.mode]
    r = runner(args, rank, world)
    total_cycles = r["cycles_per_step"] * r["streams"] * args.steps
    mine_val, e2e_val, dev_ms, _ = replica_throughput(total_cycles, r["dev_ms"],
                                                      r["e2e_ms"] or r["dev_ms"], world)
    if r["e2e_ms"] is None:
        e2e_val = None  # no host-buffer path measured in this mode
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    if rank == 0:
        peak, peak_kind = peaks()
        cyc_per_s = r["cycles_per_step"] / (r["kernel_ms"] / 1e3)
        achieved = r["bytes_per_cycle"] * cyc_per_s / 1e9
        script_gbs = r["script_bytes"] * cyc_per_s / 1e9
        tpc = r.get("traffic_per_cycle")
        if args.no_cpu or args.mode in ("timed", "timed_plain", "multi"):
            cpu_v, cpu_dt = None, 0.0
        else:
            # the reference's CPU path on the script form the reference arm
            # runs (cone partitions, 148 blocks), one host thread
            cpu_s = build_script(r["d"], 148) if args.mode == "batched" else r["script"]
            cpu_v, cpu_dt = cpu_baseline(cpu_s, r["d"], cycles=args.cpu_cycles, threads=1)
        workload = WORKLOADS[args.mode]
        line = {"metric": METRIC, "value": mine_val, "unit": "stimulus-cycles/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
                "config": {"workload": workload,
                           "mode": args.mode, "streams": r["streams"],
                           "cycles_per_step": r["cycles_per_step"], "l2": "inputs larger than L2 (snapshot window + script)",
                           **r["design"]},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "peak_kind": peak_kind,
                             "algorithmic_bytes_per_launch": r["bytes_per_cycle"] * r["cycles_per_step"],
                             "script_gbs": script_gbs, "script_frac": script_gbs / peak,
                             "traffic": tpc * r["cycles_per_step"] if tpc else None,
                             "traffic_frac": (tpc * cyc_per_s / 1e9 / peak) if tpc else None},
                "cpu_baseline": {"value": cpu_v, "unit": "stimulus-cycles/s", "cores": 1,
                                 "kind": "port",
                                 "sample": f"{args.cpu_cycles} cycles x 1 stream, {cpu_dt:.1f} s"},
                "e2e": ({"value": e2e_val, "unit": "stimulus-cycles/s",
                         "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"]}
                        if e2e_val is not None else None),
                "gpu_launches": r["launches_per_step"] * args.steps,
                "clocks": r["clocks"]}
        if r.get("parity") is not None:
            line["parity"] = r["parity"]
        if args.mode == "batched" and not args.no_compare:
            # the single-stream plain interpreter on the same design: the
            # metric's batched-against-plain ratio
            line["compare"] = compare_kernels(r["d"], args)
            line["compare"]["batched_over_plain"] = \
                mine_val / line["compare"]["plain_kernel"]["cycles_per_s"]
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
