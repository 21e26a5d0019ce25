// Harness that runs the reference's own Tipsy reader (code/read_tipsy.h with
// code/tipsydefs.h, compiled unmodified from the reference tree by
// oracle/build_ref.sh) on a file and writes what it read, for checking the
// library's snapshot writer and reader.  Test infrastructure only.
//
// usage: ref_tipsy_read IN.tipsy OUT.bin
//   OUT.bin = int32 NTotal, then NTotal float4 positions (x, y, z, mass),
//   NTotal float4 velocities (vx, vy, vz, eps), NTotal int32 ids
#include <cstdio>
#include "read_tipsy.h"

int main(int argc, char **argv)
{
  if (argc != 3) { fprintf(stderr, "usage: %s IN OUT\n", argv[0]); return 2; }
  ReadTipsy r(argv[1]);
  FILE *f = fopen(argv[2], "wb");
  if (!f) return 1;
  const int n = r.NTotal;
  fwrite(&n, sizeof(int), 1, f);
  if (n > 0) {
    fwrite(&r.positions[0], sizeof(ReadTipsy::Real4), n, f);
    fwrite(&r.velocities[0], sizeof(ReadTipsy::Real4), n, f);
    fwrite(&r.IDs[0], sizeof(int), n, f);
  }
  fclose(f);
  return 0;
}
