// Harness that runs the reference's own Plummer generator (code/plummer.h,
// compiled unmodified from the reference tree by oracle/build_ref.sh) and
// writes its output for pinning oracle_plummer.  Test infrastructure only.
//
// usage: ref_plummer N SEED OUT.bin   (run in a scratch directory: plummer.h
// reads and writes a cache file "plummer.dat" in the working directory)
#include <cstdio>
#include <cstdlib>
#include "plummer.h"

int main(int argc, char **argv)
{
  if (argc != 4) { fprintf(stderr, "usage: %s N SEED OUT\n", argv[0]); return 2; }
  const unsigned long n = strtoul(argv[1], 0, 10);
  const unsigned int seed = (unsigned int)strtoul(argv[2], 0, 10);
  std::remove("plummer.dat");
  const Plummer p(n, seed);
  std::remove("plummer.dat");
  FILE *f = fopen(argv[3], "wb");
  if (!f) return 1;
  fwrite(&p.mass[0], sizeof(double), n, f);
  for (unsigned long i = 0; i < n; i++) fwrite(&p.pos[i][0], sizeof(double), 3, f);
  for (unsigned long i = 0; i < n; i++) fwrite(&p.vel[i][0], sizeof(double), 3, f);
  fclose(f);
  return 0;
}
