// ics.cpp -- seeded initial conditions of the precision and learned forms
// (host code).  Every particle draws from its own counter-based stream
// (splitmix64 of seed and index), so the result does not depend on the
// number of host threads.  G = 1.
//
// Composite galaxy (bonsai_galaxy), particles by index:
//   [0, 0.6 N)   NFW-like halo: rho ~ 1/(x (1+x)^2), x = r/r_s, r_s = 10,
//                truncated at r = 200 (radius from the inverted enclosed mass)
//   [0.6, 0.9 N) exponential disk: surface density ~ exp(-R/R_d), R_d = 3
//                (R ~ Gamma(2, R_d)); vertical sech^2(z/z_d), z_d = 0.3
//   [0.9 N, N)   Hernquist bulge: M(<r) ~ r^2/(r+a)^2, a = 0.5, r <= 200
// Masses log-normal (sigma 0.5), normalised to a total of 1.  Velocities:
// circular speed v_c(r) = sqrt(M(<r)/r) from the components' analytic
// enclosed masses (the disk taken as spherical); disk particles rotate in
// the plane with a 10 % dispersion, halo and bulge particles are isotropic
// Gaussian with sigma = v_c/sqrt(3).  Not an equilibrium: a smooth, seeded
// stand-in with the configuration's dynamic range (r from ~1e-3 to 200).
//
// Clustered field (bonsai_clustered_field), equal masses 1/N:
//   80 % of the particles in 64 Plummer subclusters whose masses are
//   log-uniform over two decades (particle counts in proportion), scale
//   radii log-uniform in [0.01, 0.2], centres uniform in the unit cube;
//   20 % uniform in the unit cube at rest.  Subcluster particles follow the
//   Plummer distribution function (radius from the mass profile, speed by
//   rejection from q^2 (1-q^2)^(7/2), Aarseth, Henon & Wielen 1974), cut at
//   r = 10 a.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

namespace {

struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed, uint64_t index) : s(seed * 0x9E3779B97F4A7C15ull ^ (index + 0x632BE59BD9B4E019ull)) {
    next();
    next();
  }
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  // uniform in (0, 1)
  double uni() { return ((double)(next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
  double normal() {
    const double u1 = uni(), u2 = uni();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
  void direction(double& x, double& y, double& z) {
    const double c = 2.0 * uni() - 1.0, ph = 6.283185307179586 * uni();
    const double s = std::sqrt(std::max(0.0, 1.0 - c * c));
    x = s * std::cos(ph);
    y = s * std::sin(ph);
    z = c;
  }
};

template <class F>
void parallel_for(long n, F f) {
  const unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; t++)
    th.emplace_back([=]() {
      const long b = n * t / nt, e = n * (t + 1) / nt;
      for (long i = b; i < e; i++) f(i);
    });
  for (auto& x : th) x.join();
}

constexpr double kRs = 10.0, kRt = 200.0, kRd = 3.0, kZd = 0.3, kA = 0.5;
constexpr double kFh = 0.6, kFd = 0.3, kFb = 0.1;

double nfw_m(double x) { return std::log1p(x) - x / (1.0 + x); }

double enclosed(double r) {
  const double mh = kFh * nfw_m(std::min(r, kRt) / kRs) / nfw_m(kRt / kRs);
  const double mb = kFb * (r * r / ((r + kA) * (r + kA))) / (kRt * kRt / ((kRt + kA) * (kRt + kA)));
  const double md = kFd * (1.0 - (1.0 + r / kRd) * std::exp(-r / kRd));
  return mh + std::min(mb, kFb) + md;
}

// radius of the truncated NFW profile holding mass fraction u
double nfw_radius(double u, const std::vector<double>& xs, const std::vector<double>& ms) {
  const double target = u * nfw_m(kRt / kRs);
  const size_t k = std::lower_bound(ms.begin(), ms.end(), target) - ms.begin();
  double x;
  if (k == 0) x = xs[0] * target / ms[0];
  else if (k >= ms.size()) x = xs.back();
  else x = xs[k - 1] + (xs[k] - xs[k - 1]) * (target - ms[k - 1]) / (ms[k] - ms[k - 1]);
  for (int it = 0; it < 3; it++) {  // Newton on M(x) = target, M'(x) = x/(1+x)^2
    const double d = x / ((1.0 + x) * (1.0 + x));
    if (d <= 0.0) break;
    x = std::min(std::max(x - (nfw_m(x) - target) / d, 1e-12), kRt / kRs);
  }
  return x * kRs;
}

}  // namespace

extern "C" int bonsai_galaxy_impl(long n, unsigned long long seed, double* pos4, float* vel4) {
  if (n < 1 || !pos4 || !vel4) return -4;
  std::vector<double> xs(4096), ms(4096);
  for (int k = 0; k < 4096; k++) {
    xs[k] = std::pow(10.0, -8.0 + (std::log10(kRt / kRs) + 8.0) * k / 4095.0);
    ms[k] = nfw_m(xs[k]);
  }
  const long nh = (long)(kFh * (double)n), nd = (long)((kFh + kFd) * (double)n) - nh;
  parallel_for(n, [&](long i) {
    Rng g(seed, (uint64_t)i);
    double x, y, z, vx, vy, vz;
    if (i < nh || i >= nh + nd) {
      double r;
      if (i < nh) {
        r = nfw_radius(g.uni(), xs, ms);
      } else {
        do {
          const double s = std::sqrt(g.uni());
          r = kA * s / (1.0 - s);
        } while (r > kRt);
      }
      double dx, dy, dz;
      g.direction(dx, dy, dz);
      x = r * dx; y = r * dy; z = r * dz;
      const double sig = std::sqrt(enclosed(r) / std::max(r, 1e-6)) / std::sqrt(3.0);
      vx = sig * g.normal(); vy = sig * g.normal(); vz = sig * g.normal();
    } else {
      const double R = -kRd * std::log(g.uni() * g.uni());
      const double ph = 6.283185307179586 * g.uni();
      x = R * std::cos(ph);
      y = R * std::sin(ph);
      z = kZd * std::atanh(2.0 * g.uni() - 1.0);
      const double vc = std::sqrt(enclosed(R) / std::max(R, 1e-6));
      vx = -vc * std::sin(ph) + 0.1 * vc * g.normal();
      vy = vc * std::cos(ph) + 0.1 * vc * g.normal();
      vz = 0.1 * vc * g.normal();
    }
    pos4[4 * i + 0] = x; pos4[4 * i + 1] = y; pos4[4 * i + 2] = z;
    pos4[4 * i + 3] = std::exp(0.5 * g.normal());
    vel4[4 * i + 0] = (float)vx; vel4[4 * i + 1] = (float)vy; vel4[4 * i + 2] = (float)vz;
  });
  double mt = 0.0;
  for (long i = 0; i < n; i++) mt += pos4[4 * i + 3];
  const double inv = 1.0 / mt;
  for (long i = 0; i < n; i++) {
    pos4[4 * i + 3] *= inv;
    vel4[4 * i + 3] = (float)pos4[4 * i + 3];
  }
  return 0;
}

extern "C" int bonsai_clustered_field_impl(long n, unsigned long long seed, int nclusters, float* pos4, float* vel4) {
  if (n < 1 || nclusters < 1 || !pos4 || !vel4) return -4;
  const long nbg = (long)(0.2 * (double)n), ncl = n - nbg;
  // cluster parameters from stream index n + k (past every particle's index)
  std::vector<double> mass(nclusters), a(nclusters), cx(nclusters), cy(nclusters), cz(nclusters);
  double msum = 0.0;
  for (int k = 0; k < nclusters; k++) {
    Rng g(seed, (uint64_t)n + (uint64_t)k);
    mass[k] = std::pow(10.0, 2.0 * g.uni());
    a[k] = 0.01 * std::pow(20.0, g.uni());
    cx[k] = g.uni(); cy[k] = g.uni(); cz[k] = g.uni();
    msum += mass[k];
  }
  std::vector<long> beg(nclusters + 1);
  double acc = 0.0;
  beg[0] = 0;
  for (int k = 0; k < nclusters; k++) {
    acc += mass[k];
    beg[k + 1] = (k == nclusters - 1) ? ncl : (long)std::llround((double)ncl * acc / msum);
  }
  const double m = 1.0 / (double)n;
  parallel_for(n, [&](long i) {
    Rng g(seed, (uint64_t)i);
    double x, y, z, vx = 0, vy = 0, vz = 0;
    if (i >= ncl) {
      x = g.uni(); y = g.uni(); z = g.uni();
    } else {
      const int k = (int)(std::upper_bound(beg.begin(), beg.end(), i) - beg.begin()) - 1;
      const double mk = (double)(beg[k + 1] - beg[k]) * m;  // cluster mass
      double r;
      do {
        const double u = g.uni();
        r = a[k] / std::sqrt(std::pow(u, -2.0 / 3.0) - 1.0);
      } while (r > 10.0 * a[k]);
      double dx, dy, dz;
      g.direction(dx, dy, dz);
      x = cx[k] + r * dx; y = cy[k] + r * dy; z = cz[k] + r * dz;
      double q, fq;
      do {
        q = g.uni();
        fq = q * q * std::pow(1.0 - q * q, 3.5);
      } while (0.1 * g.uni() > fq);
      const double vesc = std::sqrt(2.0 * mk) * std::pow(r * r + a[k] * a[k], -0.25);
      g.direction(dx, dy, dz);
      vx = q * vesc * dx; vy = q * vesc * dy; vz = q * vesc * dz;
    }
    pos4[4 * i + 0] = (float)x; pos4[4 * i + 1] = (float)y; pos4[4 * i + 2] = (float)z; pos4[4 * i + 3] = (float)m;
    vel4[4 * i + 0] = (float)vx; vel4[4 * i + 1] = (float)vy; vel4[4 * i + 2] = (float)vz; vel4[4 * i + 3] = (float)m;
  });
  return 0;
}
