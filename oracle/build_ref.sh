#!/bin/sh
# Builds the parts of the reference that compile on the CPU, from the sources
# where they lie in the reference tree, into oracle/_ref/ (git-ignored).
# Two host parts qualify: code/plummer.h (+ code/vector3.h), the input
# generator, and code/read_tipsy.h (+ code/tipsydefs.h), the snapshot reader.
# Every file on the hot path is CUDA for sm_35 and needs a GPU (and, for
# buildTree.cu, CUDA dynamic-parallelism device synchronisation that CUDA 12
# removed).
# Same flags as the reference's own Makefile for host code (code/Makefile:9-10).
set -e
REF=${BONSAI_REFERENCE:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
mkdir -p "$HERE/_ref"
g++ -O3 -Wall -I"$REF/code" "$HERE/ref_plummer_main.cpp" -o "$HERE/_ref/ref_plummer"
echo "built $HERE/_ref/ref_plummer"
g++ -O3 -Wno-format-overflow -I"$REF/code" "$HERE/ref_tipsy_main.cpp" -o "$HERE/_ref/ref_tipsy_read"
echo "built $HERE/_ref/ref_tipsy_read"
