#!/bin/bash
# Build the reference's own CUDA hydro step for one workload (oracle/_ref).
#   oracle/ref/build_ref.sh <name> <params.json> [golden|perf]
# Compiles the reference's translation units where they lie (the read-only
# tree named by PG_REFERENCE, which must be set) against per-workload
# copies of its two configuration headers (gen_headers.py) and links them
# with ref_harness.cu.  Output: oracle/_ref/<name>/penguin_ref (git-ignored).
set -euo pipefail
NAME=$1
PJSON=$2
MODE=${3:-golden}
REF=${PG_REFERENCE:?set PG_REFERENCE to the reference source tree}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$HERE/../_ref/$NAME
mkdir -p "$OUT/obj"
python3 "$HERE/gen_headers.py" "$PJSON" "$OUT" "$REF" > /dev/null
NVCC="nvcc -O3 -gencode arch=compute_100a,code=sm_100a -lineinfo -w"
INC="-I$OUT/include -I$REF/include"
pids=()
for src in shared/variable_types shared/global disk_profile/disk_profile output/output \
           timestep/timestep ppm/ppm planet/planet orbital_advection/orbital_advection; do
  # dt_lv1/dt_lv3 and output_lv1/output_lv3 launch 1024 threads; on sm_100a
  # they need <= 64 registers to launch, and with relocatable device code so
  # do the functions they call (forces, reductions, disk profile).  golden:
  # every unit capped at 64; perf: only timestep/global capped (the harness
  # then skips the output reductions).  Register caps change allocation
  # only, not arithmetic.
  EXTRA="-maxrregcount=64"
  if [ "$MODE" = perf ]; then
    case $src in timestep/timestep|shared/global) EXTRA="-maxrregcount=64" ;; *) EXTRA="" ;; esac
  fi
  $NVCC $EXTRA --device-c -o "$OUT/obj/$(basename $src).o" "$REF/src/$src.cu" $INC &
  pids+=($!)
done
$NVCC --device-c -o "$OUT/obj/harness.o" "$HERE/ref_harness.cu" $INC -I"$REF" &
pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
$NVCC -o "$OUT/penguin_ref" "$OUT"/obj/*.o
echo "$OUT/penguin_ref"
