"""Regenerates tests/golden/reference_results_su{3,2}.txt: the results file
the reference's own main() writes (SU(N)/QCDGPU.cpp built with -D CPU_RUN
by oracle/build_ref.sh into oracle/_ref/ref_qcdgpu; its writer is
model::lattice_write_results, SU(N)/suncl/suncl.cpp:1679-1854) for a small
cold-start run from an init.dat in the reference's format.

Usage: python tests/golden/make_results_golden.py   (needs oracle/_ref built)
"""
import glob
import os
import shutil
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle", "_ref", "ref_qcdgpu")

INIT = """\tOUTPUTPATH={out}/
\tFINISHPATH={out}/
\tGROUP = {group}
\tND = 4
\tL1 = 4
\tL2 = 4
\tL3 = 4
\tL4 = 6
\tITER = 4
\tNITER = 2
\tNHIT = 10
\tBETA = {beta}
\tNAV = 2
\tINTS = 1
\tPRNG = RANLUX3
\tRANDSERIES = 54
"""


def main():
    for group, beta in ((3, "5.9000000000000e+00"), (2, "2.3000000000000e+00")):
        with tempfile.TemporaryDirectory() as d:
            out = os.path.join(d, "out")
            os.makedirs(out)
            with open(os.path.join(d, "init.dat"), "w") as f:
                f.write(INIT.format(out=out, group=group, beta=beta))
            subprocess.check_call([REF, "init.dat"], cwd=d, stdout=subprocess.DEVNULL)
            files = glob.glob(os.path.join(out, "su%d-*.txt" % group))
            assert len(files) == 1, files
            shutil.copy(files[0], os.path.join(HERE, "reference_results_su%d.txt" % group))


if __name__ == "__main__":
    main()
