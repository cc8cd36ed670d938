"""Host mirror of the reference's design-load pipeline for the interpreter.

`Design` stands in for the reference's netlist->AIG step (a seeded synthetic
aigpdk design, see csrc/frontend/generate.cpp) and `Script` for
`FlattenedScriptV1` (src/flatten.rs:189-341): the same fields, built by the
C++ front end (staging, partitioning, boomerang packing, flattening).
"""
import ctypes
from dataclasses import dataclass, field, asdict

import numpy as np

from ._native import load

c_u32p = ctypes.POINTER(ctypes.c_uint32)
NFEAT = 24
COST_MODEL_FLOATS = 128 * 24 + 128 + 128 * 128 + 128 + 128 + 1 + 24 + 24


class _GenParams(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("n_clusters", ctypes.c_uint32),
                ("nodes_per_cluster", ctypes.c_uint32), ("depth", ctypes.c_uint32),
                ("fanin_window", ctypes.c_uint32), ("intra_frac", ctypes.c_double),
                ("n_dff", ctypes.c_uint32), ("n_pi", ctypes.c_uint32),
                ("n_po", ctypes.c_uint32), ("n_sram", ctypes.c_uint32),
                ("sram_addr_bits", ctypes.c_uint32), ("with_reset", ctypes.c_int32)]


class _DesignInfo(ctypes.Structure):
    _fields_ = [("num_pins", ctypes.c_uint64), ("num_and", ctypes.c_uint64),
                ("num_dffs", ctypes.c_uint64), ("num_pos", ctypes.c_uint64),
                ("num_srams", ctypes.c_uint64), ("clock_flag_pin", ctypes.c_uint32),
                ("reset_pin", ctypes.c_uint32)]


class _BuildParams(ctypes.Structure):
    _fields_ = [("num_blocks", ctypes.c_size_t), ("xprop", ctypes.c_int32),
                ("n_level_split", ctypes.c_uint32), ("level_split", c_u32p),
                ("target_cone", ctypes.c_uint32), ("target_endpoint_bits", ctypes.c_uint32),
                ("num_threads", ctypes.c_int32), ("merge_passes", ctypes.c_int32),
                ("cost_model", ctypes.c_void_p), ("target_parts", ctypes.c_uint32),
                ("input_weight16", ctypes.c_uint32)]


class _ScriptInfo(ctypes.Structure):
    _fields_ = [("num_blocks", ctypes.c_uint64), ("num_major_stages", ctypes.c_uint64),
                ("blocks_data_len", ctypes.c_uint64), ("reg_io_state_size", ctypes.c_uint32),
                ("sram_storage_size", ctypes.c_uint32), ("xprop_enabled", ctypes.c_uint32),
                ("xprop_state_offset", ctypes.c_uint32), ("num_partitions", ctypes.c_uint64),
                ("num_delay_patches", ctypes.c_uint64), ("total_boomerang_stages", ctypes.c_uint64)]


def _lib():
    lib = load("libjq_frontend.so")
    if not getattr(lib, "_jq_typed", False):
        lib.jqf_generate.restype = ctypes.c_void_p
        lib.jqf_generate.argtypes = [ctypes.POINTER(_GenParams), ctypes.POINTER(ctypes.c_uint64)]
        lib.jqf_free_design.argtypes = [ctypes.c_void_p]
        lib.jqf_design_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(_DesignInfo)]
        lib.jqf_design_array.restype = ctypes.c_int64
        lib.jqf_design_array.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]
        lib.jqf_set_delays.argtypes = [ctypes.c_void_p, c_u32p, c_u32p, ctypes.c_size_t]
        lib.jqf_build_script.restype = ctypes.c_void_p
        lib.jqf_build_script.argtypes = [ctypes.c_void_p, ctypes.POINTER(_BuildParams),
                                         ctypes.c_char_p, ctypes.c_size_t]
        lib.jqf_free_script.argtypes = [ctypes.c_void_p]
        lib.jqf_script_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(_ScriptInfo)]
        lib.jqf_script_array.restype = ctypes.c_int64
        lib.jqf_script_array.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]
        vp, sz, u32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32
        lib.jqf_validate.restype = ctypes.c_int
        lib.jqf_validate.argtypes = [vp, sz, sz, vp, sz, u32, u32, sz, ctypes.c_char_p, sz]
        lib.jqf_builder_new.restype = vp
        lib.jqf_builder_new.argtypes = []
        for fn in ("jqf_builder_input", "jqf_builder_clock_flag", "jqf_builder_dff"):
            getattr(lib, fn).restype = u32
            getattr(lib, fn).argtypes = [vp]
        lib.jqf_builder_set_dff.restype = ctypes.c_int
        lib.jqf_builder_set_dff.argtypes = [vp, u32, u32, u32]
        lib.jqf_builder_and.restype = u32
        lib.jqf_builder_and.argtypes = [vp, u32, u32]
        lib.jqf_builder_output.restype = ctypes.c_int64
        lib.jqf_builder_output.argtypes = [vp, u32]
        lib.jqf_builder_finish.restype = ctypes.c_int
        lib.jqf_builder_finish.argtypes = [vp, u32, u32]
        lib.jqf_constraint_buffer.restype = ctypes.c_int
        lib.jqf_constraint_buffer.argtypes = [u32, ctypes.c_uint64, sz, vp, vp, vp, vp,
                                              ctypes.POINTER(u32), vp]
        lib.jqf_script_features.restype = ctypes.c_int
        lib.jqf_script_features.argtypes = [vp, vp, vp]
        lib.jqf_cost_model_predict.restype = ctypes.c_int
        lib.jqf_cost_model_predict.argtypes = [vp, vp, sz, vp]
        lib.jqf_inject_delays.restype = ctypes.c_int
        lib.jqf_inject_delays.argtypes = [vp, sz, sz, vp, vp, vp, vp, vp, sz]
        lib._jq_typed = True
    return lib


@dataclass
class DesignParams:
    """Synthetic design shape (mirrors jqf_gen_params)."""
    seed: int = 1
    n_clusters: int = 1
    nodes_per_cluster: int = 16384
    depth: int = 32
    fanin_window: int = 4
    intra_frac: float = 1.0
    n_dff: int = 1024
    n_pi: int = 32
    n_po: int = 32
    n_sram: int = 0
    sram_addr_bits: int = 10
    with_reset: int = 0


# The benchmark's synthetic design families.
def small_params(seed=1):
    """16,384 ANDs levelized to depth 32 (512/level, fanins from the previous
    4 levels), 1,024 DFFs, 32 PIs, 32 POs, one clock, no SRAM."""
    return DesignParams(seed=seed)


def soc_params(seed=2, n_clusters=512, n_dff=200_000, n_sram=16):
    """Clustered SoC-scale logic: clusters of 4,096 ANDs with 90% intra-cluster
    fanins, depth 80, 200k DFFs with synchronous reset, 16 single-port
    1024x32 SRAMs, 128 PIs (input 0 = reset), 128 POs.  512 clusters give
    2^21 random ANDs (+ one reset gate per DFF)."""
    return DesignParams(seed=seed, n_clusters=n_clusters, nodes_per_cluster=4096, depth=80,
                        fanin_window=4, intra_frac=0.9, n_dff=n_dff, n_pi=128, n_po=128,
                        n_sram=n_sram, sram_addr_bits=10, with_reset=1)


class Design:
    def __init__(self, params: DesignParams):
        self.params = params
        lib = _lib()
        gp = _GenParams(**asdict(params))
        n_and = ctypes.c_uint64()
        self._h = lib.jqf_generate(ctypes.byref(gp), ctypes.byref(n_and))
        if not self._h:
            raise RuntimeError("design generation failed")
        self._load_info()

    @classmethod
    def from_handle(cls, handle):
        """A design built elsewhere (e.g. by the netlist reader through the
        jqf_builder_* entry points); takes ownership of the handle."""
        d = cls.__new__(cls)
        d.params = None
        d._h = handle
        d._load_info()
        return d

    def _load_info(self):
        lib = _lib()
        self._free = lib.jqf_free_design  # held for __del__ at interpreter exit
        info = _DesignInfo()
        lib.jqf_design_info(self._h, ctypes.byref(info))
        self.num_pins = info.num_pins
        self.num_and = info.num_and
        self.num_dffs = info.num_dffs
        self.num_pos = info.num_pos
        self.num_srams = info.num_srams
        self.clock_flag_pin = info.clock_flag_pin
        self.reset_pin = info.reset_pin

    def __del__(self):
        h = getattr(self, "_h", None)
        free = getattr(self, "_free", None)
        if h and free is not None:
            free(h)
            self._h = None

    def array(self, which):
        lib = _lib()
        n = lib.jqf_design_array(self._h, which, None, 0)
        dt = np.uint8 if which == 0 else np.uint32
        out = np.zeros(n // np.dtype(dt).itemsize, dtype=dt)
        lib.jqf_design_array(self._h, which, out.ctypes.data, n)
        return out

    @property
    def kind(self): return self.array(0)
    @property
    def fanin_a(self): return self.array(1)
    @property
    def fanin_b(self): return self.array(2)
    @property
    def dff_d(self): return self.array(3)
    @property
    def dff_en(self): return self.array(4)
    @property
    def dff_q(self): return self.array(5)
    @property
    def primary_outputs(self): return self.array(6)
    @property
    def sram_records(self): return self.array(7).reshape(-1, 123)

    def set_delays(self, rise, fall):
        rise = np.ascontiguousarray(rise, dtype=np.uint32)
        fall = np.ascontiguousarray(fall, dtype=np.uint32)
        assert rise.shape == (self.num_pins + 1,) == fall.shape
        r = _lib().jqf_set_delays(self._h, rise.ctypes.data_as(c_u32p),
                                  fall.ctypes.data_as(c_u32p), rise.size)
        if r:
            raise ValueError("delay arrays must have num_pins + 1 entries")

    def build_script(self, num_blocks=148, xprop=False, level_split=(), target_cone=0,
                     target_endpoint_bits=0, num_threads=0, merge_passes=1, cost_model=None,
                     target_parts=0, input_weight16=0):
        """cost_model: flat float32 array (JQF_COST_MODEL_FLOATS) or None.
        target_parts: when non-zero, each major stage is cut into at most
        this many partitions of balanced cone size (target_cone unused);
        input_weight16 / 16 gates are then added per distinct chunk input
        when no cost model chooses the cut."""
        return Script(self, num_blocks, xprop, level_split, target_cone,
                      target_endpoint_bits, num_threads, merge_passes, cost_model, target_parts,
                      input_weight16)


class Script:
    """FlattenedScriptV1: blocks_start / blocks_data plus the state layout."""

    def __init__(self, design, num_blocks, xprop, level_split, target_cone,
                 target_endpoint_bits, num_threads, merge_passes, cost_model=None,
                 target_parts=0, input_weight16=0):
        lib = _lib()
        ls = (ctypes.c_uint32 * max(1, len(level_split)))(*level_split)
        cm = None
        if cost_model is not None:
            cm = np.ascontiguousarray(cost_model, dtype=np.float32)
            assert cm.size == COST_MODEL_FLOATS
        bp = _BuildParams(num_blocks, int(bool(xprop)), len(level_split), ls, target_cone,
                          target_endpoint_bits, num_threads, merge_passes,
                          cm.ctypes.data if cm is not None else None, target_parts,
                          input_weight16)
        err = ctypes.create_string_buffer(512)
        h = lib.jqf_build_script(design._h, ctypes.byref(bp), err, 512)
        if not h:
            raise RuntimeError("script build failed: " + err.value.decode())
        try:
            info = _ScriptInfo()
            lib.jqf_script_info(h, ctypes.byref(info))
            self.num_blocks = int(info.num_blocks)
            self.num_major_stages = int(info.num_major_stages)
            self.reg_io_state_size = int(info.reg_io_state_size)
            self.sram_storage_size = int(info.sram_storage_size)
            self.xprop_enabled = bool(info.xprop_enabled)
            self.xprop_state_offset = int(info.xprop_state_offset)
            self.num_partitions = int(info.num_partitions)
            self.total_boomerang_stages = int(info.total_boomerang_stages)

            def arr(which, dt):
                n = lib.jqf_script_array(h, which, None, 0)
                out = np.zeros(n // np.dtype(dt).itemsize, dtype=dt)
                lib.jqf_script_array(h, which, out.ctypes.data, n)
                return out

            self.blocks_start = arr(0, np.uint64)
            self.blocks_data = arr(1, np.uint32)
            self.input_map = dict(arr(2, np.uint32).reshape(-1, 2).tolist())
            self.output_map = dict(arr(3, np.uint32).reshape(-1, 2).tolist())
            self.staged_io_map = dict(arr(4, np.uint32).reshape(-1, 2).tolist())
            self.partition_x_capable = arr(5, np.uint8).astype(bool)
            self.part_num_stages = arr(6, np.uint32)
            self.dff_data_pos = arr(7, np.uint32)
            self.input_layout = arr(8, np.uint32)
            self.stage_block_part = arr(9, np.uint32).reshape(-1, 3)
            # (major stage, #boomerang stages, cone ANDs, targets, endpoints)
            self.partition_stats = arr(10, np.uint32).reshape(-1, 5)
            self.features = np.zeros((self.num_partitions, NFEAT), np.float32)
            lib.jqf_script_features(design._h, h, self.features.ctypes.data)
        finally:
            lib.jqf_free_script(h)
        self.timing_arrivals_enabled = False
        self.arrival_state_offset = 0

    # src/flatten.rs:682-704
    def effective_state_size(self):
        n = self.reg_io_state_size
        if self.xprop_enabled:
            n += self.reg_io_state_size
        if self.timing_arrivals_enabled:
            n += self.reg_io_state_size
        return n

    def enable_timing_arrivals(self):
        self.timing_arrivals_enabled = True
        self.arrival_state_offset = self.reg_io_state_size * (1 + int(self.xprop_enabled))

    def script_words_per_cycle(self):
        return int(self.blocks_start[-1])
