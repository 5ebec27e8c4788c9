#!/bin/bash
# Compile the reference solver (rismical-dev/3D-RISM-CUDA-MPI, src-cuda-mpi/)
# at one rank for sm_100a, straight from its sources under the reference
# tree, against the single-rank mpi.h beside this script.  Output goes to
# oracle/_ref/ only (git-ignored; the binary travels to the GPU machine).
# Usage: oracle/ref/build_ref.sh REFERENCE_TREE
#   (or R3D_REFERENCE_SRC=REFERENCE_TREE oracle/ref/build_ref.sh), where
#   REFERENCE_TREE is the directory that holds src-cuda-mpi/.
set -euo pipefail
TREE=${1:-${R3D_REFERENCE_SRC:-}}
if [ -z "$TREE" ]; then
  echo "usage: $0 REFERENCE_TREE (the directory holding src-cuda-mpi/)" >&2
  exit 2
fi
REF=$TREE/src-cuda-mpi
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$HERE/../_ref
OBJ=$OUT/obj
mkdir -p "$OBJ"
NVFLAGS="-O3 -m64 -gencode arch=compute_100a,code=sm_100a -DTEST -DOPENMPI -DGDR -I$HERE -w"
CXXFLAGS="-O3 -I$HERE -I/usr/local/cuda/include -w"
objs=()
for f in "$REF"/*.cu; do
  o=$OBJ/$(basename "${f%.cu}").o
  nvcc $NVFLAGS -c "$f" -o "$o" &
  objs+=("$o")
done
for f in "$REF"/*.cc; do
  o=$OBJ/$(basename "${f%.cc}").o
  g++ $CXXFLAGS -c "$f" -o "$o" &
  objs+=("$o")
done
g++ -O3 -x c++ -c "$REF"/factor.c -o "$OBJ"/factor.o
objs+=("$OBJ"/factor.o)
wait
nvcc -gencode arch=compute_100a,code=sm_100a -o "$OUT"/3drism-cuda-mpi "${objs[@]}" -lcufft
echo "built $OUT/3drism-cuda-mpi"
