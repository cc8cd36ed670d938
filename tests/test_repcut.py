"""RepCut hypergraph inputs and the oracle's restatement of
RCHyperGraph::from_staged_aig (src/repcut.rs:58-176), checked on the host
against a direct set computation on small designs."""
import numpy as np
import pytest

import cases
import oracle_lib
from jacquard_b200 import repcut


def topo(inp, starts):
    """Post-order of TopoTraverser::topo_traverse (src/aig.rs:3125-3170):
    endpoints pushed in order, fanin b pushed before a, no descent below
    staged inputs."""
    kind, fa, fb, staged = inp["kind"], inp["fa"], inp["fb"], inp["staged"]
    stack = [(p, False) for p in starts]
    seen, order = set(), []
    while stack:
        u, process = stack.pop()
        if process:
            order.append(u)
            continue
        if u in seen:
            continue
        seen.add(u)
        stack.append((u, True))
        if kind[u] == 1 and not staged[u]:
            for q in (int(fb[u]) >> 1, int(fa[u]) >> 1):
                if q:
                    stack.append((q, False))
    return order


def brute_sets(inp):
    """Endpoint set of every pin with Python sets, block by block of 4096
    endpoints: in reverse post-order each cone pin takes its own endpoints
    and the sets of the fanouts already processed (the reference's vs[j])."""
    N = inp["num_pins"]
    kind, fa, fb = inp["kind"], inp["fa"], inp["fb"]
    fo = [[] for _ in range(N + 1)]
    for p in range(1, N + 1):
        if kind[p] == 1:
            for q in (int(fa[p]) >> 1, int(fb[p]) >> 1):
                if q:
                    fo[q].append(p)
    sets = [set() for _ in range(N + 1)]
    E = inp["num_endpoints"]
    for b0 in range(0, E, 4096):
        b1 = min(E, b0 + 4096)
        own = {}
        starts = []
        for e in range(b0, b1):
            for p in inp["ep_pins"][inp["ep_start"][e]:inp["ep_start"][e + 1]].tolist():
                own.setdefault(p, set()).add(e)
                starts.append(p)
        blk = {}
        for p in reversed(topo(inp, starts)):
            blk[p] = own.get(p, set()).union(*[blk[j] for j in fo[p] if j in blk])
            sets[p] |= blk[p]
    return sets


@pytest.mark.parametrize("kind,split,slice_index", [("tiny", (5,), 0), ("tiny", (5,), 1),
                                                    ("sram", (8,), 1)])
def test_oracle_clusters_match_direct_sets(kind, split, slice_index):
    d = cases.design(kind)
    inp = repcut.slice_inputs(d, split, slice_index)
    cls, first, count, ew = oracle_lib.repcut(inp)
    sets = brute_sets(inp)
    N = inp["num_pins"]
    groups = {}
    for p in range(1, N):
        if len(sets[p]) >= 2:
            groups.setdefault(frozenset(sets[p]), []).append(p)
    want = sorted(groups.values(), key=lambda g: g[0])
    assert [g[0] for g in want] == first.tolist()
    assert [len(g) for g in want] == count.tolist()
    for k, g in enumerate(want):
        assert all(cls[p] == k for p in g)
    assert (ew >= 1).all() and ew.size == inp["num_endpoints"]
    assert inp["num_slices"] == len(split) + 1


def emulate_device(inp):
    """The device algorithm of jq_repcut_build in Python: per block, pins in
    reverse-level order; cone = seeded or a non-staged cone fanout; set = own
    bits | the sets of cone fanouts whose edge is not a traversal-order
    exception; node weights in forward-level order with the weight
    exceptions.  Returns (sets, node weights as float32)."""
    N, E = inp["num_pins"], inp["num_endpoints"]
    fs, fo, staged = inp["fanout_start"], inp["fanouts"], inp["staged"]
    order = np.argsort(inp["rlevel"][1:], kind="stable") + 1
    sets = [frozenset()] * (N + 1)
    for bi, b0 in enumerate(range(0, E, 4096)):
        b1 = min(E, b0 + 4096)
        supp = set(inp["supp_edges"][inp["supp_start"][bi]:inp["supp_start"][bi + 1]].tolist())
        own = {}
        for e in range(b0, b1):
            for p in inp["ep_pins"][inp["ep_start"][e]:inp["ep_start"][e + 1]].tolist():
                own.setdefault(p, set()).add(e)
        cone, blk = set(), {}
        for p in order.tolist():
            s = set(own.get(p, ()))
            inside = bool(s)
            for k in range(int(fs[p]), int(fs[p + 1])):
                j = int(fo[k])
                if j not in cone:
                    continue
                if not staged[j]:
                    inside = True
                if k in supp:
                    continue
                s |= blk[j]
            if inside:
                cone.add(p)
                blk[p] = s
                sets[p] = sets[p] | s
    nw = np.zeros(N + 1, np.float32)
    forder = np.argsort(inp["flevel"][1:], kind="stable") + 1
    for p in forder.tolist():
        if not sets[p]:
            continue
        w = np.float32(1.0)
        if inp["kind"][p] == 1:
            for bit, q in ((1, int(inp["fa"][p]) >> 1), (2, int(inp["fb"][p]) >> 1)):
                if q:
                    wq = np.float32(0.0) if inp["wsupp"][p] & bit else nw[q]
                    w = np.float32(w + np.float32(wq / np.float32(fs[q + 1] - fs[q])))
        nw[p] = w
    return sets, nw


@pytest.mark.parametrize("kind,split,slice_index", [("tiny", (5,), 1), ("sram", (8,), 1),
                                                    ("soc_mini", (20, 40, 60), 2)])
def test_device_algorithm_matches_oracle(kind, split, slice_index):
    d = cases.design(kind)
    inp = repcut.slice_inputs(d, split, slice_index)
    _, _, _, oew = oracle_lib.repcut(inp)
    sets, nw = emulate_device(inp)
    want = brute_sets(inp)
    assert all(sets[p] == frozenset(want[p]) for p in range(1, inp["num_pins"] + 1))
    nfe = np.bincount(inp["ep_pins"][:int(inp["ep_start"][-1])], minlength=inp["num_pins"] + 1)
    ew = []
    for e in range(inp["num_endpoints"]):
        tot = np.float32(0.0)
        for p in inp["ep_pins"][inp["ep_start"][e]:inp["ep_start"][e + 1]].tolist():
            tot = np.float32(tot + np.float32(nw[p] / np.float32(nfe[p])))
        ew.append(max(1, int(np.float32(tot + np.float32(0.5)))))
    assert ew == oew.tolist()
