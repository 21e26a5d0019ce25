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
# The "modified reference" walk and multipoles: code/computeForces.cu and
# code/computeMultipoles.cu (+ code/cuda_primitives.h), copied into
# oracle/_ref/modref/ with the mechanical sm_100a shims of make_modref.py, in
# the harness ref_walk_main.cu.  The reference's nvcc flags for the walk
# (code/Makefile:53-54: -ftz=true, -rdc=true), sm_100a for sm_35, and -DNDEBUG
# so that the walk's device assert (computeForces.cu:565) returns its
# stack-full sentinel instead of trapping.
if [ -x "${NVCC:-/usr/local/cuda/bin/nvcc}" ]; then
  "${PYTHON:-python3}" "$HERE/make_modref.py" "$REF/code" "$HERE/_ref/modref"
  "${NVCC:-/usr/local/cuda/bin/nvcc}" -g -O3 -gencode arch=compute_100a,code=sm_100a -rdc=true -ftz=true -DNDEBUG -w \
    -I"$REF/code" -I"$HERE" "$HERE/ref_walk_main.cu" -o "$HERE/_ref/ref_walk"
  echo "built $HERE/_ref/ref_walk"
fi
