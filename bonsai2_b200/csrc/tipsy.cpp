// tipsy.cpp -- Tipsy snapshots on the host: the layout the reference reads
// (ReadTipsy::read_inputFile, read_tipsy.h:108-160; records of tipsydefs.h):
//   header  {double time; int nbodies, ndim, nsph, ndark, nstar}, native byte
//           order, 32 bytes with the struct's tail padding;
//   ndark   dark records {float mass, pos[3], vel[3], eps; int phi}  (36 B)
//   then    nbodies - ndark star records
//           {float mass, pos[3], vel[3], metals, tform, eps; int phi}  (44 B)
// The reference reads every record after the dark ones as a star record
// (nsph is ignored) and carries the particle id in the int phi field; here
// pos4 = (x, y, z, mass), vel4 = (vx, vy, vz, eps), ids = phi, as it fills
// its positions, velocities and IDs.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

namespace {

struct TipsyHeader {
  double time;
  int nbodies, ndim, nsph, ndark, nstar;
};
static_assert(sizeof(TipsyHeader) == 32, "tipsy header is 32 bytes");

struct DarkRec {
  float mass, pos[3], vel[3], eps;
  int phi;
};
static_assert(sizeof(DarkRec) == 36, "dark record is 36 bytes");

struct StarRec {
  float mass, pos[3], vel[3], metals, tform, eps;
  int phi;
};
static_assert(sizeof(StarRec) == 44, "star record is 44 bytes");

constexpr int kErrArg = -4, kErrIo = -7;

struct File {
  FILE* f;
  explicit File(FILE* g) : f(g) {}
  ~File() {
    if (f) fclose(f);
  }
};

}  // namespace

extern "C" int bonsai_read_tipsy_impl(const char* path, double* time, int* n, float* pos4, float* vel4, int* ids) {
  if (!path || !n) return kErrArg;
  File in(fopen(path, "rb"));
  if (!in.f) return kErrIo;
  TipsyHeader h;
  if (fread(&h, sizeof(h), 1, in.f) != 1) return kErrIo;
  if (h.nbodies < 0 || h.ndark < 0 || h.ndark > h.nbodies) return kErrIo;
  if (time) *time = h.time;
  if (!pos4 && !vel4 && !ids) {
    *n = h.nbodies;
    return 0;
  }
  if (*n < h.nbodies) return kErrArg;  // caller arrays too small
  *n = h.nbodies;
  for (int i = 0; i < h.nbodies; i++) {
    float mass, pos[3], vel[3], eps;
    int phi;
    if (i < h.ndark) {
      DarkRec d;
      if (fread(&d, sizeof(d), 1, in.f) != 1) return kErrIo;
      mass = d.mass; std::memcpy(pos, d.pos, sizeof(pos)); std::memcpy(vel, d.vel, sizeof(vel));
      eps = d.eps; phi = d.phi;
    } else {
      StarRec s;
      if (fread(&s, sizeof(s), 1, in.f) != 1) return kErrIo;
      mass = s.mass; std::memcpy(pos, s.pos, sizeof(pos)); std::memcpy(vel, s.vel, sizeof(vel));
      eps = s.eps; phi = s.phi;
    }
    if (pos4) { pos4[4 * i] = pos[0]; pos4[4 * i + 1] = pos[1]; pos4[4 * i + 2] = pos[2]; pos4[4 * i + 3] = mass; }
    if (vel4) { vel4[4 * i] = vel[0]; vel4[4 * i + 1] = vel[1]; vel4[4 * i + 2] = vel[2]; vel4[4 * i + 3] = eps; }
    if (ids) ids[i] = phi;
  }
  return 0;
}

extern "C" int bonsai_write_tipsy_impl(const char* path, double time, int n, int ndark, const float* pos4,
                                       const float* vel4, const int* ids) {
  if (!path || n < 0 || ndark < 0 || ndark > n || (n > 0 && (!pos4 || !vel4))) return kErrArg;
  File out(fopen(path, "wb"));
  if (!out.f) return kErrIo;
  TipsyHeader h;
  std::memset(&h, 0, sizeof(h));
  h.time = time;
  h.nbodies = n;
  h.ndim = 3;
  h.nsph = 0;
  h.ndark = ndark;
  h.nstar = n - ndark;
  if (fwrite(&h, sizeof(h), 1, out.f) != 1) return kErrIo;
  for (int i = 0; i < n; i++) {
    const float* p = pos4 + 4 * i;
    const float* v = vel4 + 4 * i;
    const int id = ids ? ids[i] : i;
    if (i < ndark) {
      DarkRec d = {p[3], {p[0], p[1], p[2]}, {v[0], v[1], v[2]}, v[3], id};
      if (fwrite(&d, sizeof(d), 1, out.f) != 1) return kErrIo;
    } else {
      StarRec s = {p[3], {p[0], p[1], p[2]}, {v[0], v[1], v[2]}, 0.f, 0.f, v[3], id};
      if (fwrite(&s, sizeof(s), 1, out.f) != 1) return kErrIo;
    }
  }
  if (fflush(out.f) != 0) return kErrIo;
  return 0;
}
