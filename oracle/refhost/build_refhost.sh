#!/bin/bash
# Build the reference's own hydro step for the host CPU (TEST INFRASTRUCTURE:
# the timed CPU baseline and a host-side pin of the restatement).
#   oracle/refhost/build_refhost.sh <name>
# Needs oracle/_ref/<name>/include (the workload's copies of the reference's
# two configuration headers, written by oracle/ref/build_ref.sh) and the
# reference tree in PG_REFERENCE.  The reference's .cu sources are copied to
# oracle/_ref/<name>/host/src with only their kernel-launch syntax rewritten
# (launch_rewrite.py), then compiled by g++ with rh_cuda_shim.h force-included
# and linked with the fiber runtime and the same driver as the CUDA build
# (oracle/ref/ref_harness.cu, launches rewritten the same way).
# Output: oracle/_ref/<name>/penguin_ref_host (git-ignored).
set -euo pipefail
NAME=$1
REF=${PG_REFERENCE:?set PG_REFERENCE to the reference source tree}
HERE=$(cd "$(dirname "$0")" && pwd)
CASE=$HERE/../_ref/$NAME
OUT=$CASE/host
[ -d "$CASE/include" ] || { echo "missing $CASE/include (run oracle/ref/build_ref.sh first)" >&2; exit 2; }
rm -rf "$OUT"
mkdir -p "$OUT/obj"
(cd "$REF/src" && find . -name '*.cu' -print) | while read -r f; do
  mkdir -p "$OUT/src/$(dirname "$f")"
  python3 "$HERE/launch_rewrite.py" "$REF/src/$f" "$OUT/src/$f" > /dev/null
done
python3 "$HERE/launch_rewrite.py" "$HERE/../ref/ref_harness.cu" "$OUT/harness.cpp" > /dev/null
CXX="g++ -O2 -std=c++17 -fopenmp -w -x c++ -include $HERE/rh_cuda_shim.h"
INC="-I$HERE -I$CASE/include -I$REF/include -I$REF"
pids=()
for src in shared/variable_types shared/global disk_profile/disk_profile output/output \
           timestep/timestep ppm/ppm planet/planet orbital_advection/orbital_advection; do
  $CXX $INC -c -o "$OUT/obj/$(basename $src).o" "$OUT/src/$src.cu" &
  pids+=($!)
done
$CXX $INC -c -o "$OUT/obj/harness.o" "$OUT/harness.cpp" &
pids+=($!)
g++ -O2 -std=c++17 -fopenmp -c -o "$OUT/obj/rh_fiber.o" "$HERE/rh_fiber.cpp" &
pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
g++ -O2 -fopenmp -o "$CASE/penguin_ref_host" "$OUT"/obj/*.o
echo "$CASE/penguin_ref_host"
