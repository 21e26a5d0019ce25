#!/bin/sh
# Builds the parts of the reference that compile on the CPU, from the sources
# where they lie in the reference tree, into oracle/_ref/ (git-ignored).
# Two host parts qualify: code/plummer.h (+ code/vector3.h), the input
# generator, and code/read_tipsy.h (+ code/tipsydefs.h), the snapshot reader.
# Every file on the hot path is CUDA for sm_35 and needs a GPU; of those only
# code/makeGroups.cu builds for sm_100a as shipped (buildTree.cu needs CUDA
# dynamic-parallelism device synchronisation that CUDA 12 removed, and
# computeMultipoles.cu / computeForces.cu use pre-Volta shuffles and legacy
# textures).
# Same flags as the reference's own Makefile for host code (code/Makefile:9-10).
# This recipe is the one file that names the reference tree's location: the
# environment variable BONSAI_REFERENCE, else /root/reference.  Without the
# tree it builds nothing and says so (the GPU box only uses prebuilt files).
set -e
REF=${BONSAI_REFERENCE:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
if [ ! -d "$REF/code" ]; then
  echo "build_ref.sh: no reference tree at $REF (set BONSAI_REFERENCE); oracle/_ref not built"
  exit 0
fi
mkdir -p "$HERE/_ref"
g++ -O3 -Wall -I"$REF/code" "$HERE/ref_plummer_main.cpp" -o "$HERE/_ref/ref_plummer"
echo "built $HERE/_ref/ref_plummer"
g++ -O3 -Wno-format-overflow -I"$REF/code" "$HERE/ref_tipsy_main.cpp" -o "$HERE/_ref/ref_tipsy_read"
echo "built $HERE/_ref/ref_tipsy_read"
# The one hot-path CUDA file that builds for sm_100a unmodified: code/makeGroups.cu
# (PH keys, Thrust sort_by_key from the toolkit's CCCL, segment scans, groups),
# with the reference's own nvcc flags (code/Makefile:14-17, -rdc=true as every .cu
# there) and sm_100a instead of sm_35; the harness includes that file from the
# reference tree.  Runs on the GPU box (the binary travels).
if [ -x "${NVCC:-/usr/local/cuda/bin/nvcc}" ]; then
  "${NVCC:-/usr/local/cuda/bin/nvcc}" -g -O3 -gencode arch=compute_100a,code=sm_100a -rdc=true -w -I"$REF/code" \
    "$HERE/ref_groups_main.cu" -o "$HERE/_ref/ref_groups"
  echo "built $HERE/_ref/ref_groups"
fi
