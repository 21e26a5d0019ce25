// bonsai_treecode.hpp -- header-only C++ Treecode<float> over the C ABI.
//
// Same members, parameters and defaults as the reference's class
// (code/Treecode.h:123-223, driven by code/treecode.cu:61-168), so a
// treecode.cu-style driver compiles against it unchanged in its calls:
//
//   Treecode<float> tree(eps, theta);           // Treecode.h:164
//   tree.alloc(n);                              // Treecode.h:175
//   tree.h_ptclPos[i] = ...; tree.h_ptclVel[i] = ...;   (x, y, z, m)
//   tree.ptcl_h2d();                            // Treecode.h:207
//   tree.buildTree(nLeaf);                      // Treecode.h:216
//   tree.computeMultipoles();                   // Treecode.h:217
//   tree.makeGroups(5, nGroup);                 // Treecode.h:218
//   double4 stats = tree.computeForces();       // Treecode.h:219
//   tree.moveParticles();                       // Treecode.h:220
//   tree.computeEnergies();                     // Treecode.h:221
//
// Errors throw bonsai::Error (the reference aborts).  Link with
// -lbonsai_b200 (libbonsai_b200.so); no CUDA headers are needed.
#ifndef BONSAI_TREECODE_HPP
#define BONSAI_TREECODE_HPP

#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

#include "bonsai_b200.h"

namespace bonsai {

struct Error : std::runtime_error {
  int code;
  Error(int c, const char* where)
      : std::runtime_error(std::string(where) + ": " + bonsai_error_string(c)), code(c) {}
};

inline int check(int rc, const char* where) {
  if (rc < 0 || (rc > 0 && rc != BONSAI_STATUS_DEPTH)) throw Error(rc, where);
  return rc;
}

struct float4_ {
  float x, y, z, w;
};
struct double4_ {
  double x, y, z, w;
};

// Particle4<float> (Particle4.h:59-83): x, y, z and the mass in w
struct Particle4f {
  float4_ d;
  float x() const { return d.x; }
  float y() const { return d.y; }
  float z() const { return d.z; }
  float mass() const { return d.w; }
  float& x() { return d.x; }
  float& y() { return d.y; }
  float& z() { return d.z; }
  float& mass() { return d.w; }
};

// pinned host array (host_mem<T>, cudamem.h:64-96)
template <class T>
struct host_mem {
  T* ptr = nullptr;
  size_t n = 0;
  host_mem() = default;
  host_mem(const host_mem&) = delete;
  host_mem& operator=(const host_mem&) = delete;
  ~host_mem() { free(); }
  void alloc(size_t size) {
    free();
    ptr = static_cast<T*>(bonsai_host_alloc(size * sizeof(T)));
    if (!ptr) throw Error(BONSAI_ERR_ARG, "host_mem::alloc");
    n = size;
  }
  void free() {
    if (ptr) bonsai_host_free(ptr);
    ptr = nullptr;
    n = 0;
  }
  T& operator[](size_t i) { return ptr[i]; }
  const T& operator[](size_t i) const { return ptr[i]; }
};

template <typename real_t>
struct Treecode;

template <>
struct Treecode<float> {
  typedef Particle4f Particle;

  host_mem<Particle> h_ptclPos, h_ptclVel;
  double grav_potential = 0.0;

  Treecode(const float eps = 0.01f, const float theta = 0.75f, const int ncrit = 64) {
    bonsai_default_params(&prm_);
    prm_.eps = eps;
    prm_.theta = theta;
    prm_.ncrit = ncrit;
    check(bonsai_create(&prm_, &h_), "Treecode");
  }
  ~Treecode() {
    if (h_) bonsai_destroy(h_);
  }
  Treecode(const Treecode&) = delete;
  Treecode& operator=(const Treecode&) = delete;

  float theta() const { return prm_.theta; }
  float eps2() const { return prm_.eps * prm_.eps; }
  int get_nPtcl() const { return nPtcl_; }
  int get_nCrit() const { return prm_.ncrit; }
  int get_nLeaf() const { return prm_.nleaf; }

  void alloc(const int nPtcl) {
    check(bonsai_alloc(h_, nPtcl), "alloc");
    nPtcl_ = nPtcl;
    h_ptclPos.alloc(nPtcl);
    h_ptclVel.alloc(nPtcl);
  }
  void ptcl_h2d() {
    check(bonsai_set_particles(h_, &h_ptclPos.ptr->d.x, &h_ptclVel.ptr->d.x, nPtcl_), "ptcl_h2d");
  }
  void ptcl_d2h() {
    check(bonsai_get_particles(h_, &h_ptclPos.ptr->d.x, &h_ptclVel.ptr->d.x, nullptr), "ptcl_d2h");
  }
  void buildTree(const int nLeaf = 16) {
    prm_.nleaf = nLeaf;
    check(bonsai_build_tree(h_, nLeaf), "buildTree");
  }
  void computeMultipoles() { check(bonsai_compute_multipoles(h_), "computeMultipoles"); }
  void makeGroups(int levelSplit = 1, const int nCrit = 64) {
    prm_.level_split = levelSplit < 1 ? 1 : levelSplit;
    prm_.ncrit = nCrit;
    check(bonsai_make_groups(h_, levelSplit, nCrit), "makeGroups");
  }
  double4_ computeForces(const bool INTCOUNT = true) {
    double s[4] = {0, 0, 0, 0};
    check(bonsai_compute_forces(h_, INTCOUNT ? 1 : 0, s), "computeForces");
    if (INTCOUNT) {
      double e[8];
      check(bonsai_compute_energies(h_, e), "computeForces");
      grav_potential = e[1];
    }
    return double4_{s[0], s[1], s[2], s[3]};
  }
  void moveParticles() { check(bonsai_move_particles(h_), "moveParticles"); }
  // {T, W, W without the self term, E, Px, Py, Pz, M}
  std::vector<double> computeEnergies() {
    std::vector<double> e(8);
    check(bonsai_compute_energies(h_, e.data()), "computeEnergies");
    return e;
  }
  // whole steps (treecode.cu:139-168) replayed as captured CUDA graphs
  void step(const int nsteps = 1) { check(bonsai_step_graph(h_, nsteps), "step"); }
  // waits and returns the sticky device status (cleared); throws on errors
  int synchronize() { return check(bonsai_synchronize(h_), "synchronize"); }
  // the last error seen, without clearing it (BONSAI_STATUS_* bits or < 0)
  int last_error() const { return bonsai_last_error(h_); }
  bonsai_handle handle() const { return h_; }

 private:
  bonsai_params prm_;
  bonsai_handle h_ = nullptr;
  int nPtcl_ = 0;
};

}  // namespace bonsai

#endif  // BONSAI_TREECODE_HPP
