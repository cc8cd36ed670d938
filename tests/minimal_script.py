"""Hand-built one-partition script (a restatement of the reference test
fixture build_minimal_xprop_script, src/sim/cpu_reference.rs:994-1091):
global-read one input bit into thread 0, pass it through every tree level
(orb pass-through flags), hook writeout slot 0 to stage 0 thread 0, clock
enable all-ones on IO word 0, followed by an empty end partition."""
import numpy as np


def build_minimal_xprop_script(is_x_capable, num_ios):
    total = 256 + 512 + 5120 + 5120 + 5120 + 256
    s = np.zeros(total, dtype=np.uint32)
    s[0] = 1            # num_stages
    s[1] = 0            # not last: an end partition follows
    s[2] = num_ios
    s[3] = 0            # io offset
    s[4] = 0            # srams
    s[5] = 0
    s[6] = 1            # one global-read round
    s[7] = 0            # duplicates
    s[8] = 1 if is_x_capable else 0
    s[9] = num_ios      # X-mask follows the values
    s[128:256] = 0xFF00FF00
    s[128] = (int(s[128]) & 0xFFFF0000) | 0x0000   # writeout 0 <- stage 0 slot 0
    pi = 256
    s[pi] = 0           # read word 0 ...
    s[pi + 1] = 1       # ... bit 0
    pi += 512
    pi += 4096          # all-zero shuffle: every bit reads state bit 0
    s[pi + 128 * 4 + 2] = 0xFFFFFFFF
    for hi in range(1, 8):
        hw = 1 << (7 - hi)
        s[pi + hw * 4 + 2] = 0xFFFFFFFF
    s[pi + 0 * 4 + 2] = 0xFFFFFFFF
    pi += 1024
    pi += 5120          # SRAM/dup section: nothing
    pi += 4096
    s[pi] = 0xFFFFFFFF  # clock-enable invert for IO word 0 -> enable all bits
    pi += 1024
    s[pi] = 0           # end partition: num_stages 0
    s[pi + 1] = 1
    return s


def build_sram_script(num_srams=1, sram_offset=0):
    """One partition, one empty boomerang stage, `num_srams` SRAMs whose
    address/enable/data come straight from writeout words via the SRAM
    permutation, for read-before-write and X-write checks.
    Writeout slots: 0 holds the driving word (hooked from stage 0 slot 0 is
    not used); the SRAM read lands at slot num_ios-num_srams+i."""
    num_ios = num_srams + 1
    total = 256 + 0 + 5120 + 5120 + 5120
    s = np.zeros(total, dtype=np.uint32)
    s[0] = 1
    s[1] = 1
    s[2] = num_ios
    s[3] = 0
    s[4] = num_srams
    s[5] = sram_offset
    s[6] = 0
    s[7] = 0
    s[8] = 1
    s[9] = 16
    s[128:256] = 0xFFFFFFFF
    return s
