// A driver in the shape of the reference's code/treecode.cu:61-168, compiled
// against include/bonsai_treecode.hpp: the same calls in the same order.
// usage: driver N   -> prints "ok ncells... <direct> <approx> E" or exits 3
// when no GPU is present (the library reports BONSAI_ERR_NO_DEVICE).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "bonsai_treecode.hpp"

int main(int argc, char** argv) {
  const int nPtcl = argc > 1 ? std::atoi(argv[1]) : 4096;
  const float eps = 0.01f, theta = 0.4f;
  const int nLeaf = 16, nGroup = 64;
  try {
    bonsai::Treecode<float> tree(eps, theta);
    tree.alloc(nPtcl);
    std::vector<float> p(4 * (size_t)nPtcl), v(4 * (size_t)nPtcl);
    if (bonsai_plummer(nPtcl, 19810614u, p.data(), v.data())) return 2;
    for (int i = 0; i < nPtcl; i++) {
      bonsai::Treecode<float>::Particle pos, vel;
      pos.x() = p[4 * i]; pos.y() = p[4 * i + 1]; pos.z() = p[4 * i + 2]; pos.mass() = p[4 * i + 3];
      vel.x() = v[4 * i]; vel.y() = v[4 * i + 1]; vel.z() = v[4 * i + 2]; vel.mass() = v[4 * i + 3];
      tree.h_ptclPos[i] = pos;
      tree.h_ptclVel[i] = vel;
    }
    tree.ptcl_h2d();
    tree.buildTree(nLeaf);
    tree.computeMultipoles();
    tree.makeGroups(5, nGroup);
    const bonsai::double4_ interactions = tree.computeForces();
    tree.moveParticles();
    const std::vector<double> e = tree.computeEnergies();
    std::printf("ok n=%d direct=%g approx=%g W=%.9g E=%.9g M=%.9g\n", tree.get_nPtcl(), interactions.x,
                interactions.z, tree.grav_potential, e[3], e[7]);
    return 0;
  } catch (const bonsai::Error& err) {
    std::printf("error %d %s\n", err.code, err.what());
    return err.code == BONSAI_ERR_NO_DEVICE ? 3 : 1;
  }
}
