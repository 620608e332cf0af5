"""Regenerates tests/golden/reference_heatbath_links.npz from the reference's
own sequential CPU heatbath (SU(N)/suncpp, -D CPU_RUN), built from its
sources by oracle/build_ref.sh into oracle/_ref/ref_cpurun.

For each case the start field (a thermalising configuration made by the
oracle's Philox heatbath from a cold start) is handed to ref_cpurun, which
runs 8 heatbath phases (one sweep: odd X..T, even X..T) drawing its RANLUX3
stream in order (RANDSERIES 54); the file keeps the start and the
reference's resulting links, both as the stored rows per (site, direction)
in FP64: SU(3) u1 u2 u3 v1 v2 v3, SU(2) u1 u2, each (re, im).

Usage: python tests/golden/make_heatbath_links.py   (needs oracle/_ref built)
"""
import ctypes
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import _oracle as O  # noqa: E402

# (name, group, dims, beta): the run configurations' couplings, and a low
# coupling at which Kennedy-Pendleton tries are often rejected
CASES = [("su3_b6.0", 3, (4, 4, 2, 4), 6.0), ("su3_b1.5", 3, (4, 4, 2, 4), 1.5),
         ("su2_b2.3", 2, (4, 4, 2, 4), 2.3), ("su2_b0.6", 2, (4, 4, 2, 4), 0.6)]
SERIES, PHASES = 54, 8


def start_field(group, dims, beta):
    c = O.make_cfg(group=group, dims=dims, precision=1, beta=beta, row_align=64)
    t = O.new_table(c)
    O.lib.ol_init_cold(ctypes.byref(c), O.vp(t))
    for ph in range(16):
        O.phase_hb(c, t, 1 - (ph // 4) % 2, ph % 4, philox=(7, 0x5D3E1A27, ph))
    return c, t


def reference_links(group, dims, beta, rows):
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        rows.tofile(fin)
        subprocess.check_call([os.path.join(O.REF_DIR, "ref_cpurun"), "links", str(group)] +
                              [str(x) for x in dims] + [repr(beta), str(SERIES), str(PHASES), fin, fout])
        return np.fromfile(fout, dtype=np.float64)


def main():
    out = {}
    for name, group, dims, beta in CASES:
        c, t = start_field(group, dims, beta)
        rows = O.table_to_rows(c, t).reshape(-1)
        out[name + "_start"] = rows
        out[name + "_ref"] = reference_links(group, dims, beta, rows)
    np.savez_compressed(os.path.join(HERE, "reference_heatbath_links.npz"), **out)


if __name__ == "__main__":
    main()
