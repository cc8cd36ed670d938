"""RepCut hypergraph on the GPU (jq_repcut_build) against the oracle's
restatement of RCHyperGraph::from_staged_aig: the same clusters (pins grouped
by endpoint set, first-occurrence order, sizes) and bit-identical f32-derived
endpoint weights, on every slice, including designs with more than one block
of 4096 endpoints."""
import numpy as np
import pytest

import cases
import oracle_lib
from jacquard_b200 import frontend, repcut

pytestmark = pytest.mark.gpu


def check(d, split):
    n = None
    k = 0
    while n is None or k < n:
        inp = repcut.slice_inputs(d, split, k)
        n = inp["num_slices"]
        g = repcut.build_gpu(inp)
        cls, first, count = repcut.clusters(g["fingerprint"], g["popcount"], inp["num_pins"])
        ocls, ofirst, ocount, oew = oracle_lib.repcut(inp)
        assert np.array_equal(first, ofirst) and np.array_equal(count, ocount), f"slice {k}"
        assert np.array_equal(cls, ocls), f"slice {k}"
        assert np.array_equal(g["endpoint_weight"], oew), f"slice {k}"
        k += 1


@pytest.mark.parametrize("kind,split", [("sram", (8,)), ("soc_mini", (20, 40, 60))])
def test_gpu_hypergraph_matches_oracle(kind, split):
    check(cases.design(kind), split)


def test_gpu_hypergraph_multi_block():
    d = frontend.Design(frontend.soc_params(seed=3, n_clusters=24, n_dff=14000, n_sram=2))
    check(d, (40,))
