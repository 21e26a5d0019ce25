"""Writes the "modified reference": the reference's tree walk and multipole
files with the mechanical shims that let them compile and run on sm_100a.

Test and baseline infrastructure only (like the rest of oracle/).  The
reference's code/computeForces.cu, code/computeMultipoles.cu and
code/cuda_primitives.h are read from the reference tree and written, modified,
to oracle/_ref/modref/ (git-ignored); oracle/ref_walk_main.cu includes them and
oracle/build_ref.sh compiles that harness.  Nothing else in this repository
reads the output.

The shims, and nothing else (each one counted, so a different reference tree
fails loudly instead of producing a silently different program):
  1. pre-Volta warp intrinsics -> their full-warp .sync forms: __shfl,
     __shfl_xor and __ballot (CUDA 12 no longer declares them for sm_70+), and
     the non-.sync shfl.up in the two inline-PTX scan steps;
  2. legacy texture references (removed in CUDA 12) -> __device__ RefTexture
     objects of oracle/ref_shim.cuh, whose tex1Dfetch is a bounds-checked
     __ldg with the texture's zero result out of range (the walk fetches cell
     records for masked-off lanes from stale list entries; the texture unit
     returned zero there, a plain load would read out of bounds);
  3. __syncwarp() at the walk's volatile shared-memory exchanges
     (computeForces.cu:320-326, 348-366, 390-425): the reference relied on
     warp-synchronous execution, which sm_70+ no longer guarantees; every
     barrier sits where all 32 lanes arrive together.
The `#define __out` of Treecode.h collides with libstdc++'s <algorithm>; the
harness includes <algorithm> first instead of renaming anything.

usage: python oracle/make_modref.py REFERENCE_CODE_DIR OUT_DIR
"""
import os
import re
import sys

BANNER = ("// MODIFIED REFERENCE: written by oracle/make_modref.py from the reference's\n"
          "// %s with mechanical sm_100a shims (sync shuffles, texture fetches as\n"
          "// bounds-checked loads, __syncwarp at warp exchanges).  Not part of the product.\n")


def _sub(src, pattern, repl, count, name, flags=0):
    out, n = re.subn(pattern, repl, src, flags=flags)
    if n != count:
        raise SystemExit("make_modref: shim %r matched %d times, expected %d" % (name, n, count))
    return out


def _sync_intrinsics(src, counts):
    src = _sub(src, r"\b__shfl\(", "__shfl_sync(0xffffffffu, ", counts[0], "__shfl")
    src = _sub(src, r"\b__shfl_xor\(", "__shfl_xor_sync(0xffffffffu, ", counts[1], "__shfl_xor")
    src = _sub(src, r"\b__ballot\(", "__ballot_sync(0xffffffffu, ", counts[2], "__ballot")
    return src


def primitives(src):
    src = _sync_intrinsics(src, (2, 3, 4))
    # inline PTX: shfl.up without .sync -> shfl.sync.up over the full warp
    src = _sub(src, r"shfl\.up\.b32 (r0(?:\|p)?), %1, %2, 0;", r"shfl.sync.up.b32 \1, %1, %2, 0, 0xffffffff;", 2,
               "shfl.up")
    return src


def forces(src):
    src = _sync_intrinsics(src, (25, 4, 0))
    src = _sub(src, r"^(\s*)texture<(\w+),\s*1,\s*cudaReadModeElementType>\s+(\w+);",
               r"\1__device__ RefTexture<\2> \3;", 6, "texture", flags=re.M)
    sw = "__syncwarp();"
    # after the stores that fill every lane's own slot
    src = _sub(src, r"(tmpList\[laneIdx\] = 1;)", r"\1 " + sw, 2, "marker store")
    src = _sub(src, r"(tmpList\[laneIdx\] = approxCellIdx;)", r"\1 " + sw, 1, "approx store")
    src = _sub(src, r"(tmpList\[laneIdx\] = directPtclIdx;)", r"\1 " + sw, 1, "direct store")
    # before the reads that follow the scattered stores into other lanes' slots
    src = _sub(src, r"(scanVal = inclusive_segscan_warp\(tmpList\[laneIdx\], scanVal\.y\);)", sw + r" \1", 2,
               "segscan read")
    src = _sub(src, r"(if \(approxCounter >= WARP_SIZE\))", sw + r" \1", 1, "approx flush")
    src = _sub(src, r"(approxCellIdx = tmpList\[laneIdx\];)", sw + r" \1", 1, "approx reload")
    src = _sub(src, r"(if \(directCounter >= WARP_SIZE\))", sw + r" \1", 1, "direct flush")
    src = _sub(src, r"(directPtclIdx = tmpList\[laneIdx\];)", sw + r" \1", 1, "direct reload")
    return src


def multipoles(src):
    return src  # uses only cuda_primitives.h's shfl_xor, shimmed there


def main(ref_code, out_dir):
    os.makedirs(out_dir, exist_ok=True)
    for name, fn in (("cuda_primitives.h", primitives), ("computeForces.cu", forces),
                     ("computeMultipoles.cu", multipoles)):
        with open(os.path.join(ref_code, name)) as f:
            src = f.read()
        out = BANNER % ("code/" + name) + fn(src)
        with open(os.path.join(out_dir, name), "w") as f:
            f.write(out)
    print("wrote modified reference into %s" % out_dir)


if __name__ == "__main__":
    if len(sys.argv) != 3:
        raise SystemExit(__doc__)
    main(sys.argv[1], sys.argv[2])
