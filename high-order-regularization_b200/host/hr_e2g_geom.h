// hr_e2g_geom.h — host setup of the extend-to-grid problem (internal).
#pragma once
#include <cstdint>
#include <memory>
#include <utility>
#include <vector>

namespace e2g_setup {

// An allocator whose element construction without arguments leaves the
// value uninitialised, so that a large grid can be filled by parallel loops
// instead of a serial zero fill first.
template <class T>
struct NoInitAlloc : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = NoInitAlloc<U>;
  };
  NoInitAlloc() = default;
  template <class U>
  NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
  template <class U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <class U, class... A>
  void construct(U* p, A&&... a) {
    ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
  }
};

struct Scene {
  int N = 0;
  double L = 3.0, h = 0, delta = 0;
  std::vector<double> xq, nrm, area, f;  // quadrature points, normals, areas, exact density
  std::vector<int, NoInitAlloc<int>> nrst;  // (N+1)^3: tagged target index or -1
  std::vector<double> b, x0, n0;         // per tagged target
  std::vector<long> g;                   // grid index of each tagged target
  std::vector<uint8_t> band2;
};

void build(Scene& S, int N, double band1, double band2);
void stokeslet_density(const double* pt, double* f);
double p_exact(double x, double y, double z);
void u_exact(double x, double y, double z, double* u);

}  // namespace e2g_setup
