// plummer.cpp -- Plummer-sphere initial conditions on the host.
//
// The algorithm of the reference's generator (code/plummer.h:9-138): Aarseth
// sampling in Henon units scaled by 3*pi/16, radius cut R < 100, speed by
// von Neumann rejection, centre-of-mass and mean-velocity removal, all in
// FP64 from the C library's rand() seeded with srand(seed); the result is
// converted to float4 the way the reference driver does (treecode.cu:65-87):
// pos = (x, y, z, m), vel = (vx, vy, vz, m).  The reference's on-disk cache
// (plummer.dat) is not reproduced.
#include <cmath>
#include <cstdlib>
#include <vector>

namespace {
double unit_rand() { return std::rand() / (1. + RAND_MAX); }
}  // namespace

extern "C" int bonsai_plummer_impl(long n, unsigned int seed, float* pos4, float* vel4) {
  std::vector<double> m(n), x(3 * (size_t)n), v(3 * (size_t)n);
  std::srand(seed);
  long i = 0;
  while (i < n) {
    const double u1 = unit_rand(), u2 = unit_rand(), u3 = unit_rand();
    const double R = 1.0 / std::sqrt(std::pow(u1, -2.0 / 3.0) - 1.0);
    if (!(R < 100.0)) continue;
    const double Z = (1.0 - 2.0 * u2) * R;
    const double X = std::sqrt(R * R - Z * Z) * std::cos(2.0 * M_PI * u3);
    const double Y = std::sqrt(R * R - Z * Z) * std::sin(2.0 * M_PI * u3);
    const double Ve = std::sqrt(2.0) * std::pow(1.0 + R * R, -0.25);
    double q = 0.0, t = 0.0;
    while (0.1 * t >= q * q * std::pow(1.0 - q * q, 3.5)) {
      q = unit_rand();
      t = unit_rand();
    }
    const double V = Ve * q;
    const double u6 = unit_rand(), u7 = unit_rand();
    const double Vz = (1.0 - 2.0 * u6) * V;
    const double Vx = std::sqrt(V * V - Vz * Vz) * std::cos(2.0 * M_PI * u7);
    const double Vy = std::sqrt(V * V - Vz * Vz) * std::sin(2.0 * M_PI * u7);
    const double conv = 3.0 * M_PI / 16.0, sc = std::sqrt(conv);
    m[i] = 1.0 / n;
    x[3 * i] = X * conv; x[3 * i + 1] = Y * conv; x[3 * i + 2] = Z * conv;
    v[3 * i] = Vx / sc; v[3 * i + 1] = Vy / sc; v[3 * i + 2] = Vz / sc;
    i++;
  }
  double mc = 0, xc[3] = {0, 0, 0}, vc[3] = {0, 0, 0};
  for (long k = 0; k < n; k++) {
    mc += m[k];
    for (int d = 0; d < 3; d++) { xc[d] += m[k] * x[3 * k + d]; vc[d] += m[k] * v[3 * k + d]; }
  }
  for (int d = 0; d < 3; d++) { xc[d] /= mc; vc[d] /= mc; }
  for (long k = 0; k < n; k++) {
    for (int d = 0; d < 3; d++) {
      pos4[4 * k + d] = (float)(x[3 * k + d] - xc[d]);
      vel4[4 * k + d] = (float)(v[3 * k + d] - vc[d]);
    }
    pos4[4 * k + 3] = (float)m[k];
    vel4[4 * k + 3] = (float)m[k];
  }
  return 0;
}
