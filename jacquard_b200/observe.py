"""Display and assertion post-scan over simulated snapshots.

Restates the reference's `$display` formatting (src/display.rs:95-310:
parse_format_string, format_display_message) and its post-simulation scan of
display and assertion conditions (src/bin/jacquard.rs:1152-1253).

The scan starts at snapshot 1 (snapshot 0 is the initial state).  For each
cycle it goes over the displays, then separately over the assertions:
- a display whose enable bit is 1 formats its message.  The arguments are the
  bits at its argument positions, one value per position, as the reference
  collects them.
- an assertion condition bit of 1 is counted as an assertion failure.  A $stop
  condition counts a stop and a $finish ends the scan of that cycle's
  assertions; both stop the inner loop only, as in the reference.

`device_post_scan` runs the per-snapshot probe on the GPU
(`jq_set_bits`).  Only the fired entries and their argument words come back
to the host.
"""
import ctypes

import numpy as np


class FormatSpec:
    __slots__ = ("width", "radix", "signed", "min_width", "pad_char", "align")

    def __init__(self):
        self.width, self.radix, self.signed = 32, "d", True
        self.min_width, self.pad_char, self.align = None, " ", ">"


def parse_format_string(fmt):
    """Literal pieces and `{width:[<>^][0][min]radix[-u|-s]}` specifiers;
    escapes \\n, \\t and \\\\ in literals."""
    literals, specs = [], []
    cur = []
    i, n = 0, len(fmt)
    while i < n:
        c = fmt[i]
        i += 1
        if c == "{":
            literals.append("".join(cur))
            cur = []
            j = fmt.find("}", i)
            body = fmt[i:] if j < 0 else fmt[i:j]
            i = n if j < 0 else j + 1
            spec = FormatSpec()
            width_part, _, fmt_part = body.partition(":")
            try:
                spec.width = int(width_part)
            except ValueError:
                spec.width = 32
            if ":" in body:
                k = 0
                if k < len(fmt_part) and fmt_part[k] in "<>^":
                    spec.align = fmt_part[k]
                    k += 1
                if k < len(fmt_part) and fmt_part[k] == "0":
                    spec.pad_char = "0"
                    k += 1
                digits = ""
                while k < len(fmt_part) and fmt_part[k].isdigit():
                    digits += fmt_part[k]
                    k += 1
                if digits:
                    spec.min_width = int(digits)
                if k < len(fmt_part):
                    r = fmt_part[k]
                    if r in "hx":
                        spec.radix = "h"
                    elif r in "dbs":
                        spec.radix = r
                    k += 1
                if k < len(fmt_part) and fmt_part[k] == "-":
                    k += 1
                    if k < len(fmt_part):
                        if fmt_part[k] == "u":
                            spec.signed = False
                        elif fmt_part[k] == "s":
                            spec.signed = True
            specs.append(spec)
        elif c == "\\" and i < n:
            nxt = fmt[i]
            if nxt in "nt\\":
                cur.append({"n": "\n", "t": "\t", "\\": "\\"}[nxt])
                i += 1
            else:
                cur.append(c)
        else:
            cur.append(c)
    literals.append("".join(cur))
    return literals, specs


def format_display_message(fmt, args, arg_widths):
    literals, specs = parse_format_string(fmt)
    out = []
    ai = 0
    for i, lit in enumerate(literals):
        out.append(lit)
        if i < len(specs) and ai < len(args):
            spec = specs[i]
            width = arg_widths[ai] if ai < len(arg_widths) else spec.width
            mask = (1 << 64) - 1 if width >= 64 else (1 << width) - 1
            v = int(args[ai]) & mask
            if spec.signed and width < 64 and v & (1 << (width - 1)):
                disp = v - (1 << width)
            else:
                disp = v
            if spec.radix == "h":
                s = format(v, "x")
            elif spec.radix == "b":
                s = format(v, "b")
            elif spec.radix == "d" and spec.signed:
                s = str(disp)
            else:
                s = str(v)
            if spec.min_width is not None and len(s) < spec.min_width:
                pad = spec.min_width - len(s)
                if spec.align == "<":
                    # left alignment adds no padding in the reference
                    out.append(s)
                elif spec.align == "^":
                    left = pad // 2
                    out.append(spec.pad_char * left + s + spec.pad_char * (pad - left))
                else:
                    out.append(spec.pad_char * pad + s)
            else:
                out.append(s)
            ai += 1
    return "".join(out)


def _bit(flat, word, pos):
    return (int(flat[word]) >> (pos & 31)) & 1


def post_scan(states, num_cycles, eff, displays=(), assertions=()):
    """Host scan of flat snapshots (num_cycles+1)*eff words.
    displays: [(cell, enable_pos, format, arg_positions, arg_widths)];
    assertions: [(cell, pos, message_id, control)] with control None (assert),
    "stop" or "finish".  Returns (messages [(cycle, cell, text)], stats)."""
    flat = np.asarray(states, dtype=np.uint32).reshape(-1)[eff:]
    n = flat.size
    messages = []
    for c in range(num_cycles):
        off = c * eff
        for cell, en_pos, fmt, arg_pos, widths in displays:
            w = off + (en_pos >> 5)
            if w < n and _bit(flat, w, en_pos):
                args = [_bit(flat, off + (p >> 5), p) for p in arg_pos if off + (p >> 5) < n]
                messages.append((c, cell, format_display_message(fmt, args, widths)))
    stats = {"assertion_failures": 0, "stop_count": 0, "fired": []}
    for c in range(num_cycles):
        off = c * eff
        for cell, pos, _msg, control in assertions:
            w = off + (pos >> 5)
            if w < n and _bit(flat, w, pos):
                stats["fired"].append((c, cell))
                if control is None:
                    stats["assertion_failures"] += 1
                elif control == "stop":
                    stats["stop_count"] += 1
                    break
                elif control == "finish":
                    break
    return messages, stats


def device_set_bits(states, first, num, stride, positions, stream=None):
    """(snapshot, position index) pairs where the bit is 1, from the device
    walk jq_set_bits over snapshots [first, first+num) of a device buffer."""
    import torch
    from . import sim
    L = sim.lib()
    if not getattr(L, "_jq_setbits_typed", False):
        sz, vp = ctypes.c_size_t, ctypes.c_void_p
        L.jq_set_bits.restype = ctypes.c_int
        L.jq_set_bits.argtypes = [vp, sz, sz, sz, vp, ctypes.c_uint32, vp, vp, vp, sz,
                                  ctypes.POINTER(ctypes.c_size_t), vp]
        L._jq_setbits_typed = True
    dev = states.device
    pos = torch.from_numpy(np.asarray(positions, dtype=np.uint32).view(np.int32)).to(dev)
    counts = torch.empty(max(1, num), dtype=torch.int32, device=dev)
    offsets = torch.empty(num + 1, dtype=torch.int64, device=dev)
    st = (stream or torch.cuda.current_stream(dev)).cuda_stream
    total = ctypes.c_size_t()

    def call(cap, hits):
        return L.jq_set_bits(states.data_ptr(), first, num, stride, pos.data_ptr(), pos.numel(),
                             counts.data_ptr(), offsets.data_ptr(),
                             hits.data_ptr() if hits is not None else None, cap, ctypes.byref(total), st)

    rc = call(0, None)
    if rc not in (0, 1):
        raise RuntimeError(sim.lib().jq_strerror(rc).decode())
    n = total.value
    hits = torch.empty(max(1, n), dtype=torch.int32, device=dev)
    rc = call(n, hits)
    if rc:
        raise RuntimeError(sim.lib().jq_strerror(rc).decode())
    h = hits[:n].cpu().numpy().view(np.uint32) & np.uint32(0x3FFFFFFF)
    off = offsets.cpu().numpy().astype(np.int64)
    snap = np.repeat(np.arange(num, dtype=np.int64), np.diff(off))
    return snap, h.astype(np.int64)


def device_post_scan(states, num_cycles, eff, displays=(), assertions=(), stream=None):
    """post_scan with the per-snapshot probe on the device: states is the
    device buffer of (num_cycles+1) snapshots; only the fired entries and
    the argument words of fired displays are read back."""
    import torch
    displays, assertions = list(displays), list(assertions)
    messages = []
    if displays:
        snap, idx = device_set_bits(states, 1, num_cycles, eff, [d[1] for d in displays], stream)
        # argument words of every fired display, gathered on the device
        want = []
        for s, k in zip(snap.tolist(), idx.tolist()):
            for p in displays[k][3]:
                want.append((s + 1) * eff + (p >> 5))
        words = {}
        if want:
            ix = torch.as_tensor(want, dtype=torch.int64, device=states.device)
            vals = states[ix].cpu().numpy().view(np.uint32)
            words = dict(zip(want, vals.tolist()))
        for s, k in zip(snap.tolist(), idx.tolist()):
            cell, _, fmt, arg_pos, widths = displays[k]
            args = [(words[(s + 1) * eff + (p >> 5)] >> (p & 31)) & 1 for p in arg_pos]
            messages.append((s, cell, format_display_message(fmt, args, widths)))
    stats = {"assertion_failures": 0, "stop_count": 0, "fired": []}
    if assertions:
        snap, idx = device_set_bits(states, 1, num_cycles, eff, [a[1] for a in assertions], stream)
        c_prev, done = -1, False
        for s, k in zip(snap.tolist(), idx.tolist()):
            if s != c_prev:
                c_prev, done = s, False
            if done:
                continue
            cell, _, _, control = assertions[k]
            stats["fired"].append((s, cell))
            if control is None:
                stats["assertion_failures"] += 1
            elif control == "stop":
                stats["stop_count"] += 1
                done = True
            elif control == "finish":
                done = True
    return messages, stats
