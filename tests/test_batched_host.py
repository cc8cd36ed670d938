"""Host-side pieces of the batched interpreter: the combined multi-design
state layout (all designs' value words, then all their X words)."""
import numpy as np

from jacquard_b200 import batched


class _S:
    def __init__(self, rio, nb=1):
        self.reg_io_state_size = rio
        self.sram_storage_size = 0
        self.num_blocks = nb
        self.num_major_stages = 1
        self.xprop_enabled = True
        self.blocks_start = np.array([0, 256], np.uint64)
        self.blocks_data = np.zeros(256, np.uint32)
        self.input_layout = [0] * 40


def test_combined_state_roundtrip_and_signal_map():
    parts = [_S(3), _S(5), _S(2)]
    C = batched.CombinedScript(parts)
    assert C.value_words == 10 and C.effective_words == 20
    rng = np.random.default_rng(1)
    states = [rng.integers(0, 2**32, size=(2, 2 * p.reg_io_state_size * 32), dtype=np.uint64)
              .astype(np.uint32) for p in parts]
    comb = C.combine_states(states)
    assert comb.shape == (2, C.effective_words * 32)
    for d, st in enumerate(states):
        assert np.array_equal(C.design_state(d, comb), st)
        # every design signal lands where signal() says
        n = 2 * parts[d].reg_io_state_size * 32
        for sig in (0, 7, n // 2 - 1, n // 2, n - 1):
            assert np.array_equal(comb[:, C.signal(d, sig)], st[:, sig])


def test_stream_lane_word_conversion_matches_bit_definition():
    """to_batched / from_batched against their definition bit by bit: word
    [l, 32w + b] holds bit b of word w of streams 32l..32l+31, bit i = stream
    32l + i; from_batched inverts it."""
    rng = np.random.default_rng(5)
    for shape in [(32, 3), (64, 2, 5), (96, 3, 1, 2)]:
        a = rng.integers(0, 2**32, size=shape, dtype=np.uint64).astype(np.uint32)
        got = batched.to_batched(a)
        lanes, W = shape[0] // 32, shape[-1]
        assert got.shape == shape[1:-1] + (lanes, 32 * W)
        want = np.zeros(shape[1:-1] + (lanes, 32 * W), np.uint32)
        for s in range(shape[0]):
            l, i = divmod(s, 32)
            for w in range(W):
                for b in range(32):
                    bit = (a[s, ..., w] >> np.uint32(b)) & np.uint32(1)
                    want[..., l, 32 * w + b] |= bit << np.uint32(i)
        assert np.array_equal(got, want)
        assert np.array_equal(batched.from_batched(got, W), a)
