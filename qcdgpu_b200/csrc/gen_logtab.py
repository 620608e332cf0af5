"""Writes qg_logtab.h: the table of the table-driven FP64 logarithm used on
the update path (qg_log in qg_su.cuh; the oracle performs the same
operations with the same table).

Method (P. T. P. Tang, "Table-driven implementation of the logarithm
function in IEEE floating-point arithmetic", ACM TOMS 16 (1990) 378-400):
y = 2^e m with m in [1, 2); k = the nearest multiple of 1/128 to m - 1,
found from the top 8 mantissa bits (k in 0..128); c_k = RN(1 / (1 + k/128));
r = fma(m, c_k, -1) (|r| <= 2^-8, one rounding); then

    log y = e ln2 - log c_k + log1p(r).

ln 2 and -log c_k are split into a head that is a multiple of 2^-32 and a
tail (RN of the remainder), so that e ln2_hi + L_hi is exact for |e| <= 1023
and k = 128 (c = 1/2) carries exactly ln2_hi + ln2_lo: below 1 the two heads
and the two tails cancel exactly and the result keeps full relative
precision.  The heads and tails are computed here to 50 decimal digits.

Usage: python qcdgpu_b200/csrc/gen_logtab.py   (rewrites qg_logtab.h beside it)
"""
import os
from decimal import Decimal, getcontext

getcontext().prec = 50
N = 128


def split(v):
    """head: v rounded to a multiple of 2^-32 (exact in double); tail: RN of the rest"""
    hi_int = int((v * (1 << 32)).to_integral_value())
    hi = hi_int / float(1 << 32)
    assert Decimal(hi) == Decimal(hi_int) / Decimal(1 << 32)
    lo = float(v - Decimal(hi))
    return hi, lo


def table():
    ln2 = Decimal(2).ln()
    ln2_hi, ln2_lo = split(ln2)
    c, lhi, llo = [], [], []
    for k in range(N + 1):
        ck = 1.0 / (1.0 + k / N)                 # correctly rounded division
        L = -Decimal(ck).ln()
        h, l = split(L)
        c.append(ck)
        lhi.append(h)
        llo.append(l)
    assert (lhi[N], llo[N]) == (ln2_hi, ln2_lo) and c[N] == 0.5 and (c[0], lhi[0], llo[0]) == (1.0, 0.0, 0.0)
    return ln2_hi, ln2_lo, c, lhi, llo


def emit(path):
    ln2_hi, ln2_lo, c, lhi, llo = table()

    def init(vals):
        rows = [", ".join(v.hex() for v in vals[i:i + 4]) for i in range(0, len(vals), 4)]
        return "{ \\\n    " + ", \\\n    ".join(rows) + " }"

    with open(path, "w") as f:
        f.write("/* qg_logtab.h -- written by gen_logtab.py (do not edit): the table of the\n"
                " * table-driven FP64 logarithm (Tang 1990).  Plain C initialisers, used by\n"
                " * the device routine qg_log and by the oracle's restatement of it.\n"
                " *   QG_LOG_C:   c_k = RN(1 / (1 + k/128)), k = 0..128\n"
                " *   QG_LOG_LHI: -log c_k rounded to a multiple of 2^-32\n"
                " *   QG_LOG_LLO: RN(-log c_k - QG_LOG_LHI[k])\n"
                " *   QG_LN2_HI / QG_LN2_LO: ln 2 split the same way */\n")
        f.write("#pragma once\n")
        f.write("#define QG_LOG_TABLE_SIZE %d\n" % (N + 1))
        f.write("#define QG_LN2_HI %s\n" % ln2_hi.hex())
        f.write("#define QG_LN2_LO %s\n" % ln2_lo.hex())
        f.write("#define QG_LOG_C_INIT %s\n" % init(c))
        f.write("#define QG_LOG_LHI_INIT %s\n" % init(lhi))
        f.write("#define QG_LOG_LLO_INIT %s\n" % init(llo))


if __name__ == "__main__":
    emit(os.path.join(os.path.dirname(os.path.abspath(__file__)), "qg_logtab.h"))
