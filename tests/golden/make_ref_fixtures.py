"""Copies the reference's end-to-end simulation fixtures into
tests/golden/ref_fixtures: a gate-level aigpdk netlist, its input stimulus
VCD and the output VCD the reference's simulator wrote for it.

- dff_test: tests/timing_test/dff_test_synth.gv, dff_test.vcd and
  gem_output_fixed.vcd (the output once data changes at a clock edge are
  sampled with their new value; tests/timing_test/README.md);
- assert_test: tests/assert_test/assert_synth.gv, assert_test.vcd and
  assert_test_output.vcd.

Run from the repository root where the reference tree is at
/root/reference.  The copies are test data only."""
import os
import shutil
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_fixtures")
FILES = {
    "dff_test_synth.gv": "tests/timing_test/dff_test_synth.gv",
    "dff_test.vcd": "tests/timing_test/dff_test.vcd",
    "dff_test_output.vcd": "tests/timing_test/gem_output_fixed.vcd",
    "assert_synth.gv": "tests/assert_test/assert_synth.gv",
    "assert_test.vcd": "tests/assert_test/assert_test.vcd",
    "assert_test_output.vcd": "tests/assert_test/assert_test_output.vcd",
}

if __name__ == "__main__":
    os.makedirs(OUT, exist_ok=True)
    for dst, src in FILES.items():
        shutil.copyfile(os.path.join(REF, src), os.path.join(OUT, dst))
        print("copied", src, "->", dst)
