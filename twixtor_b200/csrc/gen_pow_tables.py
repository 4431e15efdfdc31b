"""Writes pow_tables.h: the tables and constants of the single precision powf that the Delinearize
step of the image prep calls (the plugin's C runtime, whose algorithm the reference restates in
plugins/retime-engine/src/crt_powf.rs). Every table entry is a correctly rounded double of a
closed form, computed here with 60 digit decimal arithmetic:

  RCP[i]  = 1 / c,       c = (1 + i / 256) / 2, i = 0..256
  LOG[i]  = ln(2 c)
  EXP2[j] = 2^(j / 64),  j = 0..63
  THIRD = 1/3, SIXTH = 1/6, LN2 = ln 2, LN2_64 = ln 2 / 64, K64 = 64 / ln 2

The two range limits of the exponent and the four coefficients of the logarithm near 1 are the
runtime's own values (not closed forms), as the reference's restatement gives them.

Run: python gen_pow_tables.py [OUT]   (default: pow_tables.h beside this script)
"""
import os
import struct
import sys
from decimal import Decimal, getcontext

getcontext().prec = 60


def bits(dec):
    """The correctly rounded double of a Decimal, as its bit pattern (float() of a Decimal rounds
    correctly)."""
    return struct.unpack("<Q", struct.pack("<d", float(dec)))[0]


def init(values):
    rows = [", ".join("0x%016xull" % v for v in values[i:i + 3]) for i in range(0, len(values), 3)]
    return "{ \\\n    " + ", \\\n    ".join(rows) + " \\\n}"


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)), "pow_tables.h")
    ln2 = Decimal(2).ln()
    rcp, log = [], []
    for i in range(257):
        c = (1 + Decimal(i) / 256) / 2
        rcp.append(bits(1 / c))
        log.append(bits((2 * c).ln()))
    exp2 = [bits((Decimal(j) / 64 * ln2).exp()) for j in range(64)]
    consts = {
        "THIRD": bits(Decimal(1) / 3), "SIXTH": bits(Decimal(1) / 6), "LN2": bits(ln2), "LN2_64": bits(ln2 / 64),
        "K64": bits(64 / ln2),
        # the runtime's own values: the exponent limits and the near 1 logarithm's coefficients
        "LIM_HI": 0x40562e4300000000, "LIM_LO": 0xc059d1da00000000,
        "C0": 0x3f89999999bac6d4, "C1": 0x3f3c8034c85dfff0, "A0": 0x3fb55555555554e6, "A1": 0x3f62492307f1519f,
    }
    with open(out, "w") as f:
        f.write("// Generated by gen_pow_tables.py (do not edit): the tables and constants of the Delinearize\n")
        f.write("// powf as bit patterns of doubles; see the generator for what each holds.\n#pragma once\n\n")
        for k, v in consts.items():
            f.write("#define TW_POW_%s 0x%016xull\n" % (k, v))
        f.write("\n#define TW_POW_RCP_INIT %s\n\n" % init(rcp))
        f.write("#define TW_POW_LOG_INIT %s\n\n" % init(log))
        f.write("#define TW_POW_EXP2_INIT %s\n" % init(exp2))


if __name__ == "__main__":
    main()
