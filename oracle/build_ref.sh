#!/bin/sh
# Builds the reference's own CPU code (vadimdi/QCDGPU, SU(N)/, -D CPU_RUN)
# from the sources where they lie, into oracle/_ref/ (git-ignored):
#   _ref/ref_ranlux   -- the reference host RANLUX (random/random.cpp)
#   _ref/ref_cpurun   -- the reference sequential heatbath (SU(N)/suncpp)
#   _ref/ref_qcdgpu   -- the reference main() in its CPU_RUN build (QCDGPU.cpp)
# Test and baseline infrastructure only.
# Usage: build_ref.sh [--probe] [reference root]
#   the root is the argument, else $QCDGPU_REFERENCE, else /root/reference;
#   --probe only checks that the sources are there (exit 1 if not)
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
PROBE=0
if [ "$1" = "--probe" ]; then PROBE=1; shift; fi
REF=${1:-${QCDGPU_REFERENCE:-/root/reference}}
R="$REF/SU(N)"
OUT="$HERE/_ref"
CXX=${CXX:-g++}
[ -d "$R" ] || { echo "reference sources not found under $REF" >&2; exit 1; }
[ "$PROBE" = 1 ] && exit 0
mkdir -p "$OUT"
$CXX -O2 -D CPU_RUN -I "$R" -o "$OUT/ref_ranlux" "$HERE/ref_ranlux_driver.cpp" "$R/random/random.cpp"
$CXX -O2 -D CPU_RUN -I "$HERE/ref_stub" -I "$R" -o "$OUT/ref_cpurun" "$HERE/ref_cpurun_driver.cpp" \
    "$R/random/random.cpp" "$R/suncl/suncl.cpp" \
    "$R/suncpp/su2/algebra_su2.cpp" "$R/suncpp/su2/update_su2.cpp" \
    "$R/suncpp/su3/algebra_su3.cpp" "$R/suncpp/su3/update_su3.cpp" \
    "$R/suncpp/Measurements/analysis_cpp.cpp" "$R/suncpp/coord_work/coord_work.cpp" "$R/suncpp/IO/io.cpp"
# the reference's own main() (QCDGPU.cpp, -D CPU_RUN): init.dat in, its
# results file (lattice_write_results) out
$CXX -O2 -D CPU_RUN -I "$HERE/ref_stub" -I "$R" -o "$OUT/ref_qcdgpu" "$R/QCDGPU.cpp" \
    "$R/random/random.cpp" "$R/suncl/suncl.cpp" \
    "$R/suncpp/su2/algebra_su2.cpp" "$R/suncpp/su2/update_su2.cpp" \
    "$R/suncpp/su3/algebra_su3.cpp" "$R/suncpp/su3/update_su3.cpp" \
    "$R/suncpp/Measurements/analysis_cpp.cpp" "$R/suncpp/coord_work/coord_work.cpp" "$R/suncpp/IO/io.cpp"
echo "built $OUT/ref_ranlux $OUT/ref_cpurun $OUT/ref_qcdgpu"
