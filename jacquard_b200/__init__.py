"""B200-native Boolean-processor interpreter for Jacquard scripts.

Modules:
  frontend  -- synthetic designs and the script front end (FlattenedScriptV1)
  state     -- state-snapshot layout helpers (src/sim/vcd_io.rs restated)
  sim       -- the C-ABI interpreter calls (plain kernel)
  batched   -- bit-lane batched interpreter (many stimulus streams per launch)
"""
__all__ = ["frontend", "sim", "state"]
