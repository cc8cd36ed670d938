"""VCD stimulus parsing and waveform writing around the interpreter.

Restates the reference's host-side VCD path (src/sim/vcd_io.rs):
- scope lookup and input matching: find_top_scope, auto_detect_vcd_scope,
  match_vcd_inputs (:120-330);
- parse_input_vcd (:347-455).  One snapshot per active clock edge.  Clock
  edge flags are set for that snapshot and cleared after it.  A clock pin's
  own value change is deferred to the next timestamp, so a data change at
  the same timestamp as a clock edge is sampled with its new value while the
  clock pin keeps its old one.  The first timestamp is not written: it
  carries u64::MAX;
- write_output_vcd[_xprop] (:758-820) and write_output_vcd_timed (:831-946).

The reference reads and writes VCD with the vcd-ng crate (0.2.0, not present
here).  This module has its own reader and writer for the VCD grammar of IEEE
1364 section 18.  A vector value is used exactly as written.  Its i-th
character goes to bit position i of the variable (most significant first),
and a value shorter than the variable is not extended.  That is how
parse_input_vcd consumes vcd-ng's tokens, and the reference's own fixtures
depend on it: tests/assert_test feeds "b11" to a 4-bit input.

For long runs, `device_transitions` does the per-snapshot output walk on the
GPU (`jq_output_transitions`), and the writers only format the changes.
"""
import ctypes
import math

import numpy as np

U64_MAX = (1 << 64) - 1
U32_MAX = 0xFFFFFFFF
PS_PER_UNIT = {"s": 10 ** 12, "ms": 10 ** 9, "us": 10 ** 6, "ns": 10 ** 3, "ps": 1, "fs": 1e-3}


# --------------------------------------------------------------------------
# reader

class Var:
    __slots__ = ("kind", "size", "code", "reference", "index")

    def __init__(self, kind, size, code, reference, index):
        self.kind, self.size, self.code, self.reference, self.index = kind, size, code, reference, index


class Scope:
    __slots__ = ("kind", "name", "children")

    def __init__(self, kind, name):
        self.kind, self.name, self.children = kind, name, []


def _parse_index(tok):
    """'[7:0]' -> (7, 0); '[3]' -> 3."""
    body = tok.strip()[1:-1]
    if ":" in body:
        a, b = body.split(":")
        return (int(a), int(b))
    return int(body)


class VcdReader:
    """Header (timescale, scope tree) and a token stream of the body:
    ('t', time) and ('v', id code, bit characters, most significant first)."""

    def __init__(self, text):
        self._words = text.split()
        self.timescale = None
        self.scopes = []
        self._pos = 0
        self._read_header()

    def _until_end(self):
        out = []
        while self._words[self._pos] != "$end":
            out.append(self._words[self._pos])
            self._pos += 1
        self._pos += 1
        return out

    def _read_header(self):
        stack = []
        w = self._words
        while self._pos < len(w):
            kw = w[self._pos]
            self._pos += 1
            if kw == "$enddefinitions":
                self._until_end()
                return
            if kw == "$timescale":
                body = "".join(self._until_end())
                num = "".join(ch for ch in body if ch.isdigit())
                unit = body[len(num):]
                self.timescale = (int(num or 1), unit)
            elif kw == "$scope":
                body = self._until_end()
                sc = Scope(body[0], body[1] if len(body) > 1 else "")
                (stack[-1].children if stack else self.scopes).append(sc)
                stack.append(sc)
            elif kw == "$upscope":
                self._until_end()
                stack.pop()
            elif kw == "$var":
                body = self._until_end()
                kind, size, code, ref = body[0], int(body[1]), body[2], body[3]
                index = None
                if len(body) > 4:
                    index = _parse_index("".join(body[4:]))
                elif "[" in ref:
                    ref, idx = ref.split("[", 1)
                    index = _parse_index("[" + idx)
                v = Var(kind, size, code, ref, index)
                (stack[-1].children if stack else self.scopes).append(v)
            elif kw.startswith("$"):
                self._until_end()

    def tokens(self):
        w = self._words
        i = self._pos
        n = len(w)
        while i < n:
            tok = w[i]
            i += 1
            c = tok[0]
            if c == "#":
                yield ("t", int(tok[1:]))
            elif c in "01xXzZ":
                yield ("v", tok[1:], tok[0].lower())
            elif c in "bB":
                # the characters as written, not extended to the variable's
                # width: a short value sets only its leading positions
                yield ("v", w[i], tok[1:].lower())
                i += 1
            elif c in "rR":
                i += 1  # real values are not input stimulus
            elif tok in ("$dumpvars", "$dumpall", "$dumpon", "$dumpoff", "$end"):
                continue
            elif c == "$":
                while i < n and w[i] != "$end":
                    i += 1
                i += 1


def all_scopes(scopes, prefix=""):
    for sc in scopes:
        if isinstance(sc, Scope):
            path = f"{prefix}/{sc.name}" if prefix else sc.name
            yield path, sc
            yield from all_scopes(sc.children, path)


def find_top_scope(scopes, path):
    """Scope at a '/'-separated path (src/sim/vcd_io.rs find_top_scope)."""
    for p, sc in all_scopes(scopes):
        if p == path:
            return sc
    return None


def _scope_has_ports(scope, names):
    have = {v.reference for v in scope.children if isinstance(v, Var)}
    return all(n in have for n in names)


def auto_detect_vcd_scope(scopes, required, top="top"):
    """The common DUT names first, then any scope with every required port."""
    found = list(all_scopes(scopes))
    for name in ("dut", "uut", "DUT", "UUT", top):
        for path, sc in found:
            if path.endswith(name) and _scope_has_ports(sc, required):
                return path, sc
    for path, sc in found:
        if _scope_has_ports(sc, required):
            return path, sc
    return None


def match_vcd_inputs(scope, input_pins):
    """(id code, bit position in the value string) -> input pin, for the
    scope's variables that name an input port.  input_pins maps
    (port name, bit index or None) -> pin.  An unindexed vector of width w
    covers bits w-1 .. 0; an indexed range [a:b] covers a .. b."""
    vcd2inp = {}
    for v in scope.children:
        if not isinstance(v, Var):
            continue
        if v.index is None:
            if v.size == 1:
                bits = [(None, 0)]
            else:
                bits = [(i, pos) for pos, i in enumerate(range(v.size - 1, -1, -1))]
        elif isinstance(v.index, int):
            bits = [(v.index, 0)]
        else:
            a, b = v.index
            step = -1 if a > b else 1
            bits = [(i, pos) for pos, i in enumerate(range(a, b + step, step))]
        for i, pos in bits:
            pin = input_pins.get((v.reference, i))
            if pin is not None:
                vcd2inp[(v.code, pos)] = pin
    return vcd2inp


# --------------------------------------------------------------------------
# stimulus

def parse_input_vcd(reader, vcd2inp, input_pos, clock_pins, rio, max_clock_edges=None):
    """Input snapshots from a stimulus VCD (src/sim/vcd_io.rs:347-455).

    input_pos: pin -> state bit position (clock pins may have none);
    clock_pins: pin -> (posedge flag position or None, negedge flag position
    or None).  Returns (input_states as (snapshots, rio) u32,
    offsets_timestamps [(offset in words, timestamp)])."""
    state = [0] * rio
    clock_val = {}
    vcd_time_last_active = U64_MAX
    vcd_time = 0
    last_active = True
    delayed = set()
    out = []
    ots = []

    def bit(pos):
        return (state[pos >> 5] >> (pos & 31)) & 1

    def flip(pos):
        state[pos >> 5] ^= 1 << (pos & 31)

    def clear(pos):
        state[pos >> 5] &= ~(1 << (pos & 31)) & U32_MAX

    def setb(pos):
        state[pos >> 5] |= 1 << (pos & 31)

    for tok in reader.tokens():
        if tok[0] == "t":
            t = tok[1]
            if t == vcd_time:
                continue
            if last_active:
                out.append(list(state))
                ots.append((len(out) * rio, vcd_time_last_active))
                for pe, ne in clock_pins.values():
                    if pe is not None:
                        clear(pe)
                    if ne is not None:
                        clear(ne)
                if max_clock_edges is not None and len(ots) >= max_clock_edges:
                    break
            if last_active:
                vcd_time_last_active = vcd_time
            vcd_time = t
            last_active = False
            for key in delayed:
                if key[0] == "s":
                    flip(key[1])
                else:
                    clock_val[key[1]] ^= 1
            delayed = set()
            continue
        _, code, bits = tok
        for pos, b in enumerate(bits):
            pin = vcd2inp.get((code, pos))
            if pin is None:
                continue
            new = 1 if b == "1" else 0
            p = input_pos.get(pin)
            old = bit(p) if p is not None else clock_val.setdefault(pin, 0)
            if old == new:
                continue
            ck = clock_pins.get(pin)
            if ck is not None:
                pe, ne = ck
                if pe is not None and old == 0:
                    last_active = True
                    setb(pe)
                if ne is not None and old == 1:
                    last_active = True
                    setb(ne)
                delayed.add(("s", p) if p is not None else ("c", pin))
            else:
                flip(p)
    out.append(list(state))
    return np.asarray(out, dtype=np.uint64).astype(np.uint32), ots


# --------------------------------------------------------------------------
# writer

def id_code(n):
    """Printable identifier code of the n-th variable (bijective base 94)."""
    s = ""
    n += 1
    while n:
        n -= 1
        s += chr(33 + n % 94)
        n //= 94
    return s


class VcdWriter:
    """Writes VCD text in the call order of the reference's writer use:
    timescale, modules and wires, upscopes, $enddefinitions, $dumpvars,
    then timestamps and scalar changes."""

    def __init__(self, f):
        self.f = f
        self._n = 0
        self._buf = []

    def timescale(self, ratio, unit):
        self.f.write(f"$timescale {ratio} {unit} $end\n")

    def add_module(self, name):
        self.f.write(f"$scope module {name} $end\n")

    def add_wire(self, width, name):
        code = id_code(self._n)
        self._n += 1
        self.f.write(f"$var wire {width} {code} {name} $end\n")
        return code

    def upscope(self):
        self.f.write("$upscope $end\n")

    def enddefinitions(self):
        self.f.write("$enddefinitions $end\n")

    def begin_dumpvars(self):
        self.f.write("$dumpvars\n")

    def timestamp(self, t):
        self._buf.append(f"#{t}\n")

    def change_scalar(self, code, value):
        self._buf.append(f"{value}{code}\n")
        if len(self._buf) >= 65536:
            self.flush()

    def flush(self):
        self.f.write("".join(self._buf))
        self._buf = []


def _value_char(enc):
    return "x" if enc == 3 else ("1" if enc == 1 else "0")


def write_output_vcd(writer, out2vcd, offsets_timestamps, states, xmask_states=None,
                     transitions=None):
    """Value changes of the outputs at each written timestamp
    (src/sim/vcd_io.rs:758-820).  out2vcd: [(aigpin, state bit position or
    U32_MAX for a constant aigpin 0/1, id code)]; states / xmask_states: flat
    u32 buffers that offsets index.  `transitions` (from device_transitions)
    replaces the host walk with its precomputed changes."""
    if transitions is not None:
        return _write_from_transitions(writer, out2vcd, offsets_timestamps, transitions)
    states = np.asarray(states, dtype=np.uint32)
    xm = None if xmask_states is None else np.asarray(xmask_states, dtype=np.uint32)
    last = [2] * len(out2vcd)
    xcount = 0
    for offset, ts in offsets_timestamps:
        if ts == U64_MAX:
            continue
        writer.timestamp(ts)
        for i, (aigpin, pos, vid) in enumerate(out2vcd):
            if pos == U32_MAX:
                assert aigpin <= 1
                v, x = aigpin, False
            else:
                w = offset + (pos >> 5)
                v = int(states[w] >> (pos & 31)) & 1
                x = xm is not None and (int(xm[w] >> (pos & 31)) & 1) != 0
            enc = 3 if x else v
            if enc == last[i]:
                continue
            last[i] = enc
            xcount += x
            writer.change_scalar(vid, _value_char(enc))
    writer.flush()
    return xcount


def _write_from_transitions(writer, out2vcd, offsets_timestamps, tr):
    written = [(o, ts) for o, ts in offsets_timestamps if ts != U64_MAX]
    assert len(written) == tr["counts"].size
    xcount = 0
    codes = tr["codes"]
    outs = tr["outputs"]
    off = tr["offsets"]
    for s, (_, ts) in enumerate(written):
        writer.timestamp(ts)
        for k in range(int(off[s]), int(off[s + 1])):
            enc = int(codes[k])
            xcount += enc == 3
            writer.change_scalar(out2vcd[int(outs[k])][2], _value_char(enc))
    writer.flush()
    return xcount


def ps_per_vcd_unit(timescale):
    if timescale is None:
        return 1.0
    ratio, unit = timescale
    return ratio * PS_PER_UNIT[unit]


def write_output_vcd_timed(writer, out2vcd, offsets_timestamps, states, arrival_states,
                           xmask_states=None, timescale=None):
    """Each transition is moved by its word's arrival time (low 16 bits, ps)
    converted to VCD units and rounded half away from zero, then all are
    written in stable timestamp order (src/sim/vcd_io.rs:831-946)."""
    states = np.asarray(states, dtype=np.uint32)
    arr = np.asarray(arrival_states, dtype=np.uint32)
    xm = None if xmask_states is None else np.asarray(xmask_states, dtype=np.uint32)
    ppu = ps_per_vcd_unit(timescale)
    last = [2] * len(out2vcd)
    timed = []
    xcount = 0
    for offset, ts in offsets_timestamps:
        if ts == U64_MAX:
            continue
        for i, (aigpin, pos, vid) in enumerate(out2vcd):
            if pos == U32_MAX:
                assert aigpin <= 1
                v, x = aigpin, False
            else:
                w = offset + (pos >> 5)
                v = int(states[w] >> (pos & 31)) & 1
                x = xm is not None and (int(xm[w] >> (pos & 31)) & 1) != 0
            enc = 3 if x else v
            if enc == last[i]:
                continue
            last[i] = enc
            xcount += x
            a = int(arr[offset + (pos >> 5)]) & 0xFFFF if pos != U32_MAX else 0
            units = math.floor(a / ppu + 0.5) if ppu > 0 else 0
            timed.append((ts + units, i, enc))
    timed.sort(key=lambda r: r[0])
    cur = None
    for t, i, enc in timed:
        if t != cur:
            writer.timestamp(t)
            cur = t
        writer.change_scalar(out2vcd[i][2], _value_char(enc))
    writer.flush()
    return xcount


# --------------------------------------------------------------------------
# device walk

def device_transitions(states, first_snapshot, num_snapshots, snapshot_words, out_pos,
                       out_const=None, xmask_offset=0, arrival_offset=0, stream=None):
    """Output transitions of snapshots [first, first+num) of a device buffer
    (torch int32) through jq_output_transitions.  Returns a dict of numpy
    arrays: counts, offsets, outputs, codes (and arrivals when requested)."""
    import torch
    from . import sim
    L = sim.lib()
    if not getattr(L, "_jq_trans_typed", False):
        sz, vp = ctypes.c_size_t, ctypes.c_void_p
        L.jq_output_transitions.restype = ctypes.c_int
        L.jq_output_transitions.argtypes = [vp, sz, sz, sz, sz, sz, vp, vp, ctypes.c_uint32, vp, vp,
                                            vp, vp, sz, ctypes.POINTER(ctypes.c_size_t), vp]
        L._jq_trans_typed = True
    dev = states.device
    pos = torch.from_numpy(np.asarray(out_pos, dtype=np.uint32).view(np.int32)).to(dev)
    const = None if out_const is None else \
        torch.from_numpy(np.asarray(out_const, dtype=np.uint32).view(np.int32)).to(dev)
    n_out = int(pos.numel())
    counts = torch.empty(max(1, num_snapshots), dtype=torch.int32, device=dev)
    offsets = torch.empty(num_snapshots + 1, dtype=torch.int64, device=dev)
    st = (stream or torch.cuda.current_stream(dev)).cuda_stream
    total = ctypes.c_size_t()

    def call(cap, tr, ar):
        return L.jq_output_transitions(states.data_ptr(), first_snapshot, num_snapshots,
                                       snapshot_words, xmask_offset, arrival_offset, pos.data_ptr(),
                                       const.data_ptr() if const is not None else None, n_out,
                                       counts.data_ptr(), offsets.data_ptr(),
                                       tr.data_ptr() if tr is not None else None,
                                       ar.data_ptr() if ar is not None else None, cap,
                                       ctypes.byref(total), st)

    rc = call(0, None, None)
    if rc not in (0, 1):
        raise RuntimeError(sim.lib().jq_strerror(rc).decode())
    n = total.value
    tr = torch.empty(max(1, n), dtype=torch.int32, device=dev)
    ar = torch.empty(max(1, n), dtype=torch.int32, device=dev) if arrival_offset else None
    rc = call(n, tr, ar)
    if rc != 0:
        raise RuntimeError(sim.lib().jq_strerror(rc).decode())
    t = tr[:n].cpu().numpy().view(np.uint32)
    out = {"counts": counts[:num_snapshots].cpu().numpy().view(np.uint32),
           "offsets": offsets.cpu().numpy().astype(np.int64),
           "outputs": (t & np.uint32(0x3FFFFFFF)).astype(np.int64),
           "codes": (t >> np.uint32(30)).astype(np.uint8)}
    if ar is not None:
        out["arrivals"] = ar[:n].cpu().numpy().view(np.uint32) & np.uint32(0xFFFF)
    return out


# --------------------------------------------------------------------------
# ports of the synthetic designs

class DesignPorts:
    """Port view of a generated design: input `clk` (its posedge flag is the
    design's clock flag pin; the clock net itself has no state bit), inputs
    `pi[0..n_pi-1]` (pi[0] is the reset when the design has one) and outputs
    `po[0..n_po-1]`."""

    def __init__(self, design, script):
        kinds = design.kind
        self.pi_pins = np.nonzero(kinds == 2)[0].astype(np.int64)
        self.clock_pin = "clk"
        self.input_pins = {("clk", None): "clk"}
        for i, p in enumerate(self.pi_pins.tolist()):
            self.input_pins[("pi", i)] = int(p)
        self.input_pos = {int(p): int(script.input_map[int(p)]) for p in self.pi_pins.tolist()}
        self.clock_pins = {"clk": (int(script.input_map[int(design.clock_flag_pin)]), None)}
        self.po_pins = np.asarray(design.primary_outputs, dtype=np.int64)

    def out2vcd(self, writer, script, name="po"):
        out = []
        for j, ap in enumerate(self.po_pins.tolist()):
            pos = U32_MAX if ap <= 1 else int(script.output_map[ap])
            out.append((ap, pos, writer.add_wire(1, f"{name}[{j}]")))
        return out


def write_stimulus_vcd(f, ports, in_vals, input_layout, clock_flag_pin, period=10, timescale=(1, "ns")):
    """A stimulus VCD for rows of input values (in_vals: (rows,
    len(input_layout)) 0/1 over input_layout; the clock-flag column is
    ignored): data inputs change with the falling clock edge at k * period,
    the clock rises at k * period + period / 2.  Parsed back with
    parse_input_vcd, snapshot k + 1 holds row k with the posedge flag set;
    snapshot 0 is the state before the first edge (written with timestamp
    u64::MAX, i.e. not at all) and the last snapshot the state after the
    final period."""
    w = VcdWriter(f)
    w.timescale(*timescale)
    w.add_module("top")
    clk = w.add_wire(1, "clk")
    n_pi = len(ports.pi_pins)
    codes = [w.add_wire(1, f"pi[{i}]") for i in range(n_pi)]
    w.upscope()
    w.enddefinitions()
    w.begin_dumpvars()
    col = {int(p): k for k, p in enumerate(np.asarray(input_layout).tolist())}
    pi_col = [col[int(p)] for p in ports.pi_pins.tolist()]
    vals = np.asarray(in_vals, dtype=np.uint8)
    half = period // 2
    prev = None
    for k in range(vals.shape[0]):
        t0 = k * period
        w.timestamp(t0)
        w.change_scalar(clk, "0")
        for i in range(n_pi):
            v = int(vals[k, pi_col[i]])
            if prev is None or v != prev[i]:
                w.change_scalar(codes[i], str(v))
        prev = [int(vals[k, pi_col[i]]) for i in range(n_pi)]
        w.timestamp(t0 + half)
        w.change_scalar(clk, "1")
    w.timestamp(vals.shape[0] * period)
    w.change_scalar(clk, "0")
    w.flush()


def simulate_vcd(script, ports, stimulus_text, xprop_all_x=False, device="cuda", stream=None):
    """The reference's VCD-in / VCD-out flow on the plain interpreter: parse
    the stimulus, expand the snapshots (X template when the script has X
    propagation; every DFF/SRAM bit X at start with xprop_all_x), run all
    cycles on the device, and write the output waveform from the device-side
    transition walk.  `ports` maps VCD variables to the design (DesignPorts
    for generated designs, netlist.NetlistPorts for netlists).  Returns
    (output VCD text, device states)."""
    import io as _io

    import torch
    from . import sim, state as st
    reader = VcdReader(stimulus_text)
    required = sorted({name for name, _ in ports.input_pins})
    found = auto_detect_vcd_scope(reader.scopes, required)
    if found is None:
        raise ValueError("no scope holds every input port of the design")
    vcd2inp = match_vcd_inputs(found[1], ports.input_pins)
    snaps, ots = parse_input_vcd(reader, vcd2inp, ports.input_pos, ports.clock_pins,
                                 script.reg_io_state_size)
    rio = script.reg_io_state_size
    eff = rio
    host = snaps
    if script.xprop_enabled:
        host = st.expand_states_for_xprop(snaps, script)
        if xprop_all_x:
            host[0, rio:] = st.xmask_all_state_x(script)
        eff = 2 * rio
    cycles = host.shape[0] - 1
    ds = sim.DeviceScript(script, device)
    states = sim.u32_to_dev(np.ascontiguousarray(host).reshape(-1), device)
    n_sram = max(1, script.sram_storage_size)
    sram = torch.zeros(n_sram, dtype=torch.int32, device=device)
    sram_x = torch.full((n_sram,), -1, dtype=torch.int32, device=device)
    if cycles:
        sim.simulate(ds, states, cycles, eff, sram, sram_x, stream=stream)
        rc = sim.status(stream)
        if rc:
            raise RuntimeError(sim.lib().jq_strerror(rc).decode())
    out = _io.StringIO()
    w = VcdWriter(out)
    if reader.timescale is not None:
        w.timescale(*reader.timescale)
    w.add_module("gem_top_module")
    out2vcd = ports.out2vcd(w, script)
    w.upscope()
    w.enddefinitions()
    w.begin_dumpvars()
    written = [(o, t) for o, t in ots if t != U64_MAX]
    if written:
        first = written[0][0] // rio
        pos = [p for _, p, _ in out2vcd]
        const = [a if p == U32_MAX else 0 for a, p, _ in out2vcd]
        tr = device_transitions(states, first, len(written), eff, pos, out_const=const,
                                xmask_offset=rio if script.xprop_enabled else 0, stream=stream)
        write_output_vcd(w, out2vcd, ots, None, transitions=tr)
    w.flush()
    return out.getvalue(), states
