"""RepCut hypergraph build (src/repcut.rs:58-176) for one staged slice of a
design, on the GPU (`jq_repcut_build`).

The hypergraph has one vertex per endpoint group of the slice.  Its edges are
the clusters: distinct endpoint sets, over the pins whose fanout reaches at
least two endpoints, each weighted by the number of pins sharing it.  Vertex
weights come from the reference's fanout-normalised node weights.  Clusters
are listed in first-occurrence (pin) order over pins 1 .. num_pins-1, as the
reference's IndexMap has them.
"""
import ctypes

import numpy as np

from . import frontend


def slice_inputs(design, level_split, slice_index):
    """The slice's fanout CSR, endpoint inputs, staged flags and levels
    (jqf_repcut_slice), plus the design's kind / fanin arrays."""
    L = frontend._lib()
    if not getattr(L, "_jq_repcut_typed", False):
        vp = ctypes.c_void_p
        L.jqf_repcut_slice.restype = ctypes.c_int
        L.jqf_repcut_slice.argtypes = [vp, vp, ctypes.c_size_t, ctypes.c_uint32] + [vp] * 11
        L._jq_repcut_typed = True
    split = np.ascontiguousarray(level_split, dtype=np.uint32)
    sizes = np.zeros(4, np.uint64)
    n_slices = L.jqf_repcut_slice(design._h, split.ctypes.data if split.size else None, split.size,
                                  slice_index, None, None, None, None, None, None, None, None, None,
                                  None, sizes.ctypes.data)
    if n_slices < 0:
        raise ValueError("no such slice")
    N = int(design.num_pins)
    E, nfo, nep, nsupp = (int(x) for x in sizes)
    out = {"num_pins": N, "num_endpoints": E, "num_slices": n_slices,
           "fanout_start": np.zeros(N + 2, np.uint32), "fanouts": np.zeros(max(1, nfo), np.uint32),
           "ep_start": np.zeros(E + 1, np.uint32), "ep_pins": np.zeros(max(1, nep), np.uint32),
           "staged": np.zeros(N + 1, np.uint8), "rlevel": np.zeros(N + 1, np.uint32),
           "flevel": np.zeros(N + 1, np.uint32),
           "supp_start": np.zeros((E + 4095) // 4096 + 1, np.uint32),
           "supp_edges": np.zeros(max(1, nsupp), np.uint32), "wsupp": np.zeros(N + 1, np.uint8)}
    L.jqf_repcut_slice(design._h, split.ctypes.data if split.size else None, split.size, slice_index,
                       *(out[k].ctypes.data for k in ("fanout_start", "fanouts", "ep_start", "ep_pins",
                                                      "staged", "rlevel", "flevel", "supp_start",
                                                      "supp_edges", "wsupp")), None)
    out["num_fanouts"] = nfo
    out["kind"] = np.ascontiguousarray(design.kind, np.uint8)
    out["fa"] = np.ascontiguousarray(design.fanin_a, np.uint32)
    out["fb"] = np.ascontiguousarray(design.fanin_b, np.uint32)
    return out


def _levels(level):
    lv = np.asarray(level[1:], dtype=np.int64)
    nodes = (np.argsort(lv, kind="stable") + 1).astype(np.uint32)
    counts = np.bincount(lv, minlength=int(lv.max()) + 1 if lv.size else 1)
    starts = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    return nodes, starts


def build_gpu(inp, device="cuda", stream=None):
    """Fingerprints, popcounts, node and endpoint weights on the device."""
    import torch
    from . import sim
    L = sim.lib()
    if not getattr(L, "_jq_repcut_typed", False):
        vp, u32 = ctypes.c_void_p, ctypes.c_uint32
        L.jq_repcut_build.restype = ctypes.c_int
        L.jq_repcut_build.argtypes = [u32, vp, vp, vp, vp, vp, vp, u32, vp, vp, vp, vp, vp, u32,
                                      vp, vp, u32, vp, vp, vp, u32, vp, vp, vp, vp, vp, vp, vp, vp]
        L._jq_repcut_typed = True
    N, E = inp["num_pins"], inp["num_endpoints"]

    def dev(a, dt):
        return torch.from_numpy(np.ascontiguousarray(a).view(dt)).to(device)

    rn, rs = _levels(inp["rlevel"])
    fn, fs = _levels(inp["flevel"])
    nfe = np.bincount(inp["ep_pins"][:int(inp["ep_start"][-1])], minlength=N + 1).astype(np.uint32)
    t = {k: dev(inp[k], np.int32) for k in ("fa", "fb", "fanout_start", "fanouts", "ep_start", "ep_pins",
                                            "supp_edges")}
    t["wsupp"] = dev(inp["wsupp"], np.uint8)
    supp_bits = torch.empty(inp["num_fanouts"] // 32 + 2, dtype=torch.int32, device=device)
    t["kind"] = dev(inp["kind"], np.uint8)
    t["staged"] = dev(inp["staged"], np.uint8)
    t["nfe"] = dev(nfe, np.int32)
    t["rn"] = dev(rn, np.int32)
    t["fn"] = dev(fn, np.int32)
    sets = torch.empty((N + 1) * 64, dtype=torch.int64, device=device)
    cone = torch.empty(N + 1, dtype=torch.uint8, device=device)
    fp = torch.empty(2 * (N + 1), dtype=torch.int64, device=device)
    pc = torch.empty(N + 1, dtype=torch.int32, device=device)
    nw = torch.empty(N + 1, dtype=torch.float32, device=device)
    ew = torch.empty(max(1, E), dtype=torch.int64, device=device)
    st = (stream or torch.cuda.current_stream(torch.device(device))).cuda_stream
    rc = L.jq_repcut_build(N, t["kind"].data_ptr(), t["fa"].data_ptr(), t["fb"].data_ptr(),
                           t["fanout_start"].data_ptr(), t["fanouts"].data_ptr(), t["staged"].data_ptr(),
                           E, t["ep_start"].data_ptr(), t["ep_pins"].data_ptr(), t["nfe"].data_ptr(),
                           t["rn"].data_ptr(), rs.ctypes.data, rs.size - 1, t["fn"].data_ptr(),
                           fs.ctypes.data, fs.size - 1, inp["supp_start"].ctypes.data,
                           t["supp_edges"].data_ptr(), t["wsupp"].data_ptr(), inp["num_fanouts"],
                           supp_bits.data_ptr(), sets.data_ptr(), cone.data_ptr(), fp.data_ptr(),
                           pc.data_ptr(),
                           nw.data_ptr(), ew.data_ptr(), st)
    if rc:
        raise RuntimeError(sim.lib().jq_strerror(rc).decode())
    torch.cuda.synchronize()
    return {"fingerprint": fp.cpu().numpy().view(np.uint64).reshape(-1, 2),
            "popcount": pc.cpu().numpy().view(np.uint32),
            "node_weight": nw.cpu().numpy(),
            "endpoint_weight": ew[:E].cpu().numpy().view(np.uint64)}


def clusters(fingerprint, popcount, num_pins):
    """(class of each pin or -1, first pin and size of each cluster) over
    pins 1 .. num_pins-1 with at least two endpoints, clusters in
    first-occurrence order."""
    pins = np.arange(1, num_pins, dtype=np.int64)
    pins = pins[popcount[1:num_pins] >= 2]
    cls = np.full(num_pins + 1, -1, np.int64)
    if pins.size == 0:
        return cls, np.zeros(0, np.int64), np.zeros(0, np.int64)
    fp = np.ascontiguousarray(fingerprint[pins])
    key = fp.view([("a", np.uint64), ("b", np.uint64)]).reshape(-1)
    _, first_idx, inverse, counts = np.unique(key, return_index=True, return_inverse=True,
                                              return_counts=True)
    order = np.argsort(first_idx, kind="stable")
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    cls[pins] = rank[inverse.reshape(-1)]
    return cls, pins[first_idx[order]], counts[order]
