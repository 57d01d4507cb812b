#!/bin/sh
# Compile the reference's own CUDA projectors, OSEM, list-mode histogrammer, randoms,
# normalisation and scatter model (sources read in place from the
# reference tree, nothing copied) with the test-only harness oracle/ref_harness.cu into
# oracle/_ref/libnipet_ref.so.  Flags follow the reference's Release build (-O3, no fast
# math), for sm_100a.
# Usage: oracle/build_ref.sh [reference root]
# The reference root is the argument, else $NIPET_REFERENCE, else the checkout location of
# the build container (/root/reference).  Without a reference tree there nothing is built
# and the script exits 0 (a machine without the checkout uses a prebuilt oracle/_ref).
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=${1:-${NIPET_REFERENCE:-/root/reference}}
REF=$ROOT/niftypet/nipet
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
if [ ! -d "$REF/prj/src" ]; then
  echo "build_ref.sh: no reference sources under $ROOT; oracle/_ref not rebuilt" >&2
  exit 0
fi
mkdir -p "$HERE/_ref"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -O3 -std=c++14 -Xcompiler -fPIC -shared \
  -DNIPET_CU_THREADS=1024 -I"$REF/include" -I"$REF/prj/src" -I"$REF/lm/src" -I"$REF/src" \
  -I"$REF/sct/src" \
  "$REF/prj/src/prjf.cu" "$REF/prj/src/prjb.cu" "$REF/prj/src/tprj.cu" \
  "$REF/prj/src/recon.cu" "$REF/lm/src/lmproc.cu" "$REF/lm/src/hst.cu" \
  "$REF/lm/src/lmaux.cu" "$REF/lm/src/rnd.cu" "$REF/src/scanner_0.cu" "$REF/src/norm.cu" \
  "$REF/sct/src/sct.cu" "$REF/sct/src/sctaux.cu" "$REF/sct/src/ray.cu" "$HERE/ref_harness.cu" \
  -lcurand -o "$HERE/_ref/libnipet_ref.so"
echo "$HERE/_ref/libnipet_ref.so"
