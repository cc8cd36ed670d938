"""Gate-level netlists in the aigpdk cell set (Yosys output) as designs.

Reads the structural Verilog a synthesis flow writes for the aigpdk library
and builds the AIG through the front end's builder entry points.  The AIG is
built as the reference builds it (src/aig.rs):
- AND2_ab_y: Y = ((A ^ a) & (B ^ b)) ^ y, e.g. AND2_01_0 = A & ~B and
  AND2_11_1 = A | B (aigpdk/aigpdk.v);
- INV inverts, BUF and `assign` alias;
- DFF captures D on the rising edge of its clock: enable = the posedge flag
  of the clock's input port (src/aig.rs:2028-2060);
- GEM_ASSERT fires when EN & !A on its clock edge: condition = (EN & !A) &
  clock flag, kept as an observable endpoint (src/aig.rs:2488-2529);
- GEM_DISPLAY fires when EN on its clock edge: enable = EN & clock flag, its
  MSG_ID bits are the arguments, and the `gem_format` / `gem_args_width`
  attributes give the format (src/aig.rs:2530-2580).

The reference reads netlists with the sverilogparse and netlistdb crates,
which are not present here.  This reader covers the subset a mapped aigpdk
netlist uses:
- module ports and input / output / wire declarations with ranges;
- cell instances with named connections;
- `assign` aliases;
- bit selects, part selects, concatenations and sized constants.
Attributes are kept only where they carry the display format.
"""
import re

import numpy as np

from . import frontend

_TOKEN = re.compile(r"""
    (?P<ws>\s+)|
    (?P<attr>\(\*.*?\*\))|
    (?P<bc>/\*.*?\*/)|
    (?P<lc>//[^\n]*)|
    (?P<const>\d+'[sS]?[bBoOdDhH][0-9a-fA-FxXzZ_]+)|
    (?P<num>\d+)|
    (?P<esc>\\\S+)|
    (?P<id>[A-Za-z_$][A-Za-z0-9_$]*)|
    (?P<sym>[()\[\]:,;.{}=])
""", re.S | re.X)

GATES = {"AND2_00_0": (0, 0, 0), "AND2_01_0": (0, 1, 0), "AND2_10_0": (1, 0, 0),
         "AND2_11_0": (1, 1, 0), "AND2_11_1": (1, 1, 1)}


def _tokens(text):
    out = []
    pos = 0
    while pos < len(text):
        m = _TOKEN.match(text, pos)
        if not m:
            raise ValueError(f"netlist: cannot read at {text[pos:pos + 40]!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind in ("ws", "bc", "lc"):
            continue
        val = m.group(kind)
        if kind == "esc":
            val = val[1:]
            kind = "id"
        out.append((kind, val))
    return out


def _const_bits(tok):
    """Sized constant -> bits, most significant first."""
    width, rest = tok.split("'", 1)
    width = int(width)
    rest = rest.lstrip("sS")
    base, digits = rest[0].lower(), rest[1:].replace("_", "").lower()
    if any(c in "xz" for c in digits):
        raise ValueError(f"netlist: x/z constant {tok} is not supported")
    value = int(digits, {"b": 2, "o": 8, "d": 10, "h": 16}[base])
    return [("const", (value >> i) & 1) for i in range(width - 1, -1, -1)]


def _parse_attrs(chunks):
    """{name: value} of `(* name = value, ... *)` chunks; strings keep their
    escapes as written, sized constants become ints."""
    out = {}
    for chunk in chunks:
        body = chunk[2:-2]
        for m in re.finditer(r'([A-Za-z_][A-Za-z0-9_]*)\s*(?:=\s*("(?:[^"\\]|\\.)*"|[^,]+))?', body):
            key, val = m.group(1), m.group(2)
            if val is None:
                out[key] = 1
                continue
            val = val.strip()
            if val.startswith('"'):
                out[key] = val[1:-1]
            elif "'" in val:
                bits = _const_bits(val)
                out[key] = int("".join(str(b[1]) for b in bits), 2)
            else:
                try:
                    out[key] = int(val)
                except ValueError:
                    out[key] = val
    return out


class Netlist:
    """One module: ports [(name, dir, msb, lsb)] (msb/lsb None for scalars),
    net ranges, cells [(type, name, {pin: [bits]})], assigns [(lhs, rhs)].
    A bit is ("net", name, index or None) or ("const", 0 | 1); bit lists are
    most significant first."""

    def __init__(self, text):
        self.toks = _tokens(text)
        self.i = 0
        self.ports = []
        self.ranges = {}
        self.cells = []
        self.assigns = []
        self.attrs = {}  # cell name -> {attribute: value}
        self.pending_attrs = []
        self._parse()

    # token helpers (attributes are collected aside, for the next cell)
    def _skip_attrs(self):
        while self.i < len(self.toks) and self.toks[self.i][0] == "attr":
            self.pending_attrs.append(self.toks[self.i][1])
            self.i += 1

    def _peek(self):
        self._skip_attrs()
        return self.toks[self.i] if self.i < len(self.toks) else (None, None)

    def _next(self):
        t = self._peek()
        self.i += 1
        return t

    def _expect(self, val):
        k, v = self._next()
        if v != val:
            raise ValueError(f"netlist: expected {val!r}, got {v!r}")

    def _parse(self):
        k, v = self._next()
        while v != "module":
            k, v = self._next()
            if k is None:
                raise ValueError("netlist: no module")
        self.name = self._next()[1]
        port_order = []
        if self._peek()[1] == "(":
            self._next()
            while self._peek()[1] != ")":
                k, v = self._next()
                if k == "id":
                    port_order.append(v)
            self._next()
        self._expect(";")
        dirs = {}
        while True:
            k, v = self._peek()
            if v == "endmodule" or k is None:
                break
            if v in ("input", "output", "inout", "wire"):
                self.pending_attrs = []
                self._next()
                msb = lsb = None
                if self._peek()[1] == "[":
                    self._next()
                    msb = int(self._next()[1])
                    self._expect(":")
                    lsb = int(self._next()[1])
                    self._expect("]")
                while True:
                    name = self._next()[1]
                    self.ranges[name] = (msb, lsb)
                    if v != "wire":
                        dirs[name] = v
                    if self._next()[1] == ";":
                        break
            elif v == "assign":
                self.pending_attrs = []
                self._next()
                lhs = self._expr()
                self._expect("=")
                rhs = self._expr()
                self._expect(";")
                self.assigns.append((lhs, rhs))
            else:
                attrs = _parse_attrs(self.pending_attrs)
                self.pending_attrs = []
                ctype = self._next()[1]
                cname = self._next()[1]
                if attrs:
                    self.attrs[cname] = attrs
                self._expect("(")
                conns = {}
                while self._peek()[1] != ")":
                    self._expect(".")
                    pin = self._next()[1]
                    self._expect("(")
                    conns[pin] = self._expr() if self._peek()[1] != ")" else []
                    self._expect(")")
                    if self._peek()[1] == ",":
                        self._next()
                self._next()
                self._expect(";")
                self.cells.append((ctype, cname, conns))
        for p in port_order:
            msb, lsb = self.ranges.get(p, (None, None))
            self.ports.append((p, dirs.get(p, "inout"), msb, lsb))

    def _expr(self):
        k, v = self._next()
        if v == "{":
            bits = []
            while True:
                bits += self._expr()
                k, v = self._next()
                if v == "}":
                    return bits
        if k == "const":
            return _const_bits(v)
        if k == "num":
            return _const_bits(f"32'd{v}")
        name = v
        if self._peek()[1] == "[":
            self._next()
            a = int(self._next()[1])
            if self._peek()[1] == ":":
                self._next()
                b = int(self._next()[1])
                self._expect("]")
                step = -1 if a >= b else 1
                return [("net", name, i) for i in range(a, b + step, step)]
            self._expect("]")
            return [("net", name, a)]
        return self.bits_of(name)

    def bits_of(self, name):
        msb, lsb = self.ranges.get(name, (None, None))
        if msb is None:
            return [("net", name, None)]
        step = -1 if msb >= lsb else 1
        return [("net", name, i) for i in range(msb, lsb + step, step)]


class NetlistDesign:
    """A netlist built into a front-end design, with its port maps:
    `design` (frontend.Design), input pin per input port bit, iv per output
    port bit, the clock posedge flag pin of every clock input bit, and the
    assertion conditions [(cell name, iv)]."""

    def __init__(self, text):
        nl = Netlist(text)
        self.netlist = nl
        lib = frontend._lib()
        b = lib.jqf_builder_new()
        if not b:
            raise MemoryError("builder")
        self._b = b
        drivers = {}
        for ctype, cname, conns in nl.cells:
            if ctype in GATES or ctype in ("INV", "BUF"):
                for bit in conns.get("Y", []):
                    drivers[bit] = (ctype, cname, conns)
            elif ctype == "DFF":
                for bit in conns.get("Q", []):
                    drivers[bit] = (ctype, cname, conns)
            elif ctype not in ("GEM_ASSERT", "GEM_DISPLAY"):
                raise ValueError(f"netlist: cell type {ctype} is not supported")
        for lhs, rhs in nl.assigns:
            if len(lhs) != len(rhs):
                raise ValueError("netlist: assign width mismatch")
            for l_, r_ in zip(lhs, rhs):
                drivers[l_] = ("alias", r_)
        # sources: input port bits (port order, most significant first), then
        # clock flags, then DFF Q pins
        self.input_pins = {}
        for name, d, msb, lsb in nl.ports:
            if d in ("input", "inout"):
                for bit in nl.bits_of(name):
                    pin = lib.jqf_builder_input(b)
                    self.input_pins[(name, bit[2])] = pin
                    drivers[bit] = ("input", pin)
        self._drivers = drivers
        dffs = [(cn, conns) for ct, cn, conns in nl.cells if ct == "DFF"]
        self.clock_flags = {}  # input pin of the clock -> flag pin
        dff_clock = []
        for cn, conns in dffs:
            ck = self._source(conns["CLK"][0])
            if ck[0] != "input":
                raise ValueError(f"netlist: DFF {cn} clock is not an input port")
            if ck[1] not in self.clock_flags:
                self.clock_flags[ck[1]] = lib.jqf_builder_clock_flag(b)
            dff_clock.append(self.clock_flags[ck[1]])
        self._q = {}
        for k, (cn, conns) in enumerate(dffs):
            q = lib.jqf_builder_dff(b)
            for bit in conns.get("Q", []):
                self._q[bit] = q
        self._memo = {}
        self.output_iv = {}
        for name, d, msb, lsb in nl.ports:
            if d == "output":
                for bit in nl.bits_of(name):
                    iv = self.iv(bit)
                    self.output_iv[(name, bit[2])] = iv
                    lib.jqf_builder_output(b, iv)
        for k, (cn, conns) in enumerate(dffs):
            d_iv = self.iv(conns["D"][0])
            if lib.jqf_builder_set_dff(b, k, d_iv, dff_clock[k] << 1):
                raise ValueError("netlist: bad DFF")
        self.assertions = []
        for ctype, cname, conns in nl.cells:
            if ctype != "GEM_ASSERT":
                continue
            en = self.iv(conns["EN"][0]) if conns.get("EN") else 1
            a = self.iv(conns["A"][0]) if conns.get("A") else 1
            clken = 1
            if conns.get("CLK"):
                ck = self._source(conns["CLK"][0])
                if ck[0] == "input" and ck[1] in self.clock_flags:
                    clken = self.clock_flags[ck[1]] << 1
            fire = lib.jqf_builder_and(b, lib.jqf_builder_and(b, en, a ^ 1), clken)
            lib.jqf_builder_output(b, fire)
            self.assertions.append((cname, fire))
        self.displays = []
        for ctype, cname, conns in nl.cells:
            if ctype != "GEM_DISPLAY":
                continue
            en = self.iv(conns["EN"][0]) if conns.get("EN") else 1
            clken = 1
            if conns.get("CLK"):
                ck = self._source(conns["CLK"][0])
                if ck[0] == "input" and ck[1] in self.clock_flags:
                    clken = self.clock_flags[ck[1]] << 1
            fire = lib.jqf_builder_and(b, en, clken)
            lib.jqf_builder_output(b, fire)
            args = [self.iv(bit) for bit in conns.get("MSG_ID", [])]
            for a in args:
                if a > 1:
                    lib.jqf_builder_output(b, a)
            at = nl.attrs.get(cname, {})
            fmt = at.get("gem_format", f"$display at cell {cname}")
            widths = [int(at["gem_args_width"])] if "gem_args_width" in at else [32]
            self.displays.append((cname, fire, fmt, args, widths))
        first_flag = next(iter(self.clock_flags.values()), 0)
        if lib.jqf_builder_finish(b, first_flag, 0):
            raise ValueError("netlist: incomplete design")
        self.design = frontend.Design.from_handle(b)
        self._b = None

    def _source(self, bit):
        """Follow aliases and buffers to the driving input / cell / constant."""
        seen = 0
        while True:
            if bit[0] == "const":
                return ("const", bit[1])
            drv = self._drivers.get(bit)
            if drv is None:
                raise ValueError(f"netlist: undriven net {bit}")
            if drv[0] == "alias":
                bit = drv[1]
            elif drv[0] == "BUF":
                bit = drv[2]["A"][0]
            else:
                return drv
            seen += 1
            if seen > 1 << 20:
                raise ValueError("netlist: alias loop")

    def iv(self, bit):
        """iv of a net bit (iterative depth-first build of its logic cone)."""
        lib = frontend._lib()
        b = self._b
        stack = [bit]
        while stack:
            cur = stack[-1]
            if cur in self._memo:
                stack.pop()
                continue
            if cur[0] == "const":
                self._memo[cur] = cur[1]
                stack.pop()
                continue
            if cur in self._q:
                self._memo[cur] = self._q[cur] << 1
                stack.pop()
                continue
            drv = self._drivers.get(cur)
            if drv is None:
                raise ValueError(f"netlist: undriven net {cur}")
            kind = drv[0]
            if kind == "input":
                self._memo[cur] = drv[1] << 1
                stack.pop()
                continue
            if kind == "alias":
                deps = [drv[1]]
            elif kind in ("INV", "BUF"):
                deps = [drv[2]["A"][0]]
            else:
                deps = [drv[2]["A"][0], drv[2]["B"][0]]
            todo = [x for x in deps if x not in self._memo]
            if todo:
                if len(stack) > 4 * len(self._drivers) + 16:
                    raise ValueError("netlist: combinational loop")
                stack.extend(todo)
                continue
            if kind == "alias" or kind == "BUF":
                v = self._memo[deps[0]]
            elif kind == "INV":
                v = self._memo[deps[0]] ^ 1
            else:
                ia, ib, iy = GATES[kind]
                v = lib.jqf_builder_and(b, self._memo[deps[0]] ^ ia, self._memo[deps[1]] ^ ib) ^ iy
            self._memo[cur] = v
            stack.pop()
        return self._memo[bit]


class NetlistPorts:
    """VCD port view of a netlist design, as the reference maps VCD variables
    to netlist pins (src/sim/vcd_io.rs match_vcd_inputs, setup_output_vcd).
    Every input port bit has a state position; a clock port bit also has its
    posedge flag.  Output port bits come in port order (most significant
    first).  Outputs that are pass-throughs of input ports are skipped.
    Constant outputs use their constant."""

    def __init__(self, nd, script):
        self.input_pins = dict(nd.input_pins)
        self.input_pos = {pin: int(script.input_map[pin]) for pin in nd.input_pins.values()}
        self.clock_pins = {pin: (int(script.input_map[flag]), None)
                           for pin, flag in nd.clock_flags.items()}
        kinds = nd.design.kind
        self.outputs = []
        for (name, idx), iv in nd.output_iv.items():
            if iv > 1 and kinds[iv >> 1] == 2:
                continue  # pass-through of an input port
            label = name if idx is None else f"{name}[{idx}]"
            self.outputs.append((iv, label))
        self.assertions = nd.assertions
        self.displays = nd.displays

    def out2vcd(self, writer, script):
        from .vcd import U32_MAX
        out = []
        for iv, label in self.outputs:
            pos = U32_MAX if iv <= 1 else int(script.output_map[iv])
            out.append((iv, pos, writer.add_wire(1, label)))
        return out

    def assertion_positions(self, script):
        """[(cell, state bit position of its fire condition, message id,
        control)] for observe.post_scan (GEM_ASSERT cells are plain
        assertions)."""
        return [(name, int(script.output_map[iv]), k, None)
                for k, (name, iv) in enumerate(self.assertions) if iv > 1]

    def display_positions(self, script):
        """[(cell, enable position, format, argument positions, widths)];
        constant argument bits have no position and are left out, as in the
        reference (src/flatten.rs:1381-1403)."""
        out = []
        for name, fire, fmt, args, widths in self.displays:
            if fire <= 1:
                continue
            pos = [int(script.output_map[a]) for a in args if a > 1]
            out.append((name, int(script.output_map[fire]), fmt, pos, widths))
        return out


def read_netlist(text):
    return NetlistDesign(text)
