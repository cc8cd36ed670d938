"""The committed, trained partition cost model on the host (no GPU): its
training summary records the learned-vs-heuristic comparison, and it
predicts the cost structure the simulator measured."""
import json
import os

import numpy as np

from jacquard_b200 import costmodel, frontend

TRAINED = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "jacquard_b200", "trained")


def predict(model, feats):
    feats = np.ascontiguousarray(feats, np.float32)
    out = np.zeros(len(feats), np.float32)
    L = frontend._lib()
    r = L.jqf_cost_model_predict(model.ctypes.data, feats.ctypes.data, len(feats), out.ctypes.data)
    assert r == 0
    return out


def test_summary_records_learned_vs_heuristic():
    """The committed summary of the training run: the learned cut against
    the heuristic one on two designs the model never saw (a 4.6M-gate design
    and the benchmark's 2M-gate SoC), measured on the batched interpreter
    over 5,000 cycles of 256 streams, each learned run bit-exact against the
    heuristic run on every DFF and output of every stream.  The learned cut
    gains on the benchmark's design and loses nothing on the other."""
    with open(os.path.join(TRAINED, "costmodel.json")) as f:
        sm = json.load(f)
    assert sm["samples"] >= 20000 and sm["steps"] == 2000
    assert sm["heldout_r2"] > 0.9
    for key in ("eval", "eval_soc2m"):
        ev = sm[key]
        h, l = ev["heuristic"]["stream_cycles_per_s"], ev["learned"]["stream_cycles_per_s"]
        assert h > 0 and l > 0
        assert abs(ev["gain"] - l / h) < 1e-9
        assert ev["cycles"] == 5000 and ev["streams"] == 256
        assert ev["bit_exact_vs_heuristic"] is True
    assert sm["eval_soc2m"]["gain"] > 1.01
    assert sm["eval"]["gain"] > 0.995


def test_benchmark_uses_the_learned_cut_only_when_it_wins():
    """bench.py's default (--learned auto) takes the learned cut exactly when
    the committed summary of the model trained on its work-item form shows it
    winning, bit-exact, on the benchmark's own design in the configuration it
    runs (partitions per major stage, lane words per work item)."""
    import bench
    for name, per_item in (("costmodel.json", 2), ("costmodel_octet.json", 8)):
        with open(os.path.join(TRAINED, name)) as f:
            ev = json.load(f)["eval_soc2m"]
        assert ev.get("lanes_per_item", 2) == per_item
        wins = ev["bit_exact_vs_heuristic"] and ev["gain"] > 1.0
        assert bench.learned_wins(ev["parts_per_stage"], per_item) == wins
        assert bench.learned_wins(ev["parts_per_stage"] + 1, per_item) is False


def test_octet_model_summary_records_its_loss():
    """The model retrained on octet work items (8 lane words per item, 148
    partitions per major stage): its learned cut measured against the
    heuristic one on the benchmark's design and a held-out design of the same
    size, 5,000 cycles of 256 streams, bit-exact -- and slower on both, so
    the benchmark's octet configuration runs the heuristic cut."""
    import bench
    with open(os.path.join(TRAINED, "costmodel_octet.json")) as f:
        sm = json.load(f)
    assert sm["samples"] >= 20000 and sm["per_item"] == 8 and sm["heldout_r2"] > 0.8
    for key in ("eval", "eval_soc2m"):
        ev = sm[key]
        assert ev["lanes_per_item"] == 8 and ev["parts_per_stage"] == 148
        assert ev["cycles"] == 5000 and ev["streams"] == 256
        assert ev["bit_exact_vs_heuristic"] is True
        assert ev["gain"] < 1.0
    assert bench.learned_wins(148, 8) is False


def test_model_predicts_larger_partitions_cost_more():
    """A fresh design of the training family (SoC generator, 64 clusters,
    level split every 4) cut into 12 and into 37 balanced partitions per
    stage: the larger partitions are predicted to take longer, as measured,
    and over both cuts prediction grows with gate count (within one balanced
    cut the gate counts are nearly equal)."""
    model = costmodel.packed_from_file(os.path.join(TRAINED, "costmodel.npz"))
    d = frontend.Design(frontend.soc_params(seed=77, n_clusters=64, n_dff=200_000 * 64 // 512,
                                            n_sram=4))
    split = tuple(range(4, 80, 4))
    big = d.build_script(num_blocks=148, level_split=split, xprop=True, merge_passes=0,
                         target_parts=12)
    small = d.build_script(num_blocks=148, level_split=split, xprop=True, merge_passes=0,
                           target_parts=37)
    assert big.features[:, 1].mean() > 2 * small.features[:, 1].mean()
    pb, ps = predict(model, big.features), predict(model, small.features)
    assert np.exp(pb).mean() > np.exp(ps).mean()
    both = np.concatenate([big.features[:, 1], small.features[:, 1]])
    assert np.corrcoef(both, np.concatenate([pb, ps]))[0, 1] > 0.3
