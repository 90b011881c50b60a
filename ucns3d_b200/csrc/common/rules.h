// Cell topology, volume quadrature and monomial ordering shared by the
// host set-up library (prep.cpp) and the engine's device set-up
// (setup.cu), so both build the reconstruction tables from the same
// tetrahedra, points, weights and basis order.
#pragma once

#include <array>
#include <cmath>
#include <vector>

namespace ucrules {

// ---------------------------------------------------------------- topology
// Shapes use UCNS3D's ISHAPE codes: 1 hexahedron, 2 tetrahedron,
// 3 pyramid, 4 prism.  Node numbering of the hexahedron is that of
// hexaVOLUME (src/grid_t.f90:662-669); prisms have nodes 0-2 at the bottom
// and 3-5 above them; pyramids have the base 0-3 and apex 4.
struct Topo {
  int nv, nf;
  int fnv[6];
  int fv[6][4];
  int ntet;
  int tet[6][4];
};

inline const Topo& topo(int type) {
  static const Topo hex = {8, 6, {4, 4, 4, 4, 4, 4},
                           {{0, 3, 2, 1}, {4, 5, 6, 7}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {0, 4, 7, 3}},
                           6,
                           // DECOMPOSE3 case(1), 0-based
                           {{0, 5, 7, 4}, {0, 1, 7, 5}, {1, 6, 7, 5}, {0, 7, 2, 3}, {0, 7, 1, 2}, {1, 7, 6, 2}}};
  static const Topo tet = {4, 4, {3, 3, 3, 3, 0, 0},
                           {{1, 2, 3, 0}, {0, 3, 2, 0}, {0, 1, 3, 0}, {0, 2, 1, 0}, {0}, {0}},
                           1,
                           {{0, 1, 2, 3}}};
  static const Topo pyr = {5, 5, {4, 3, 3, 3, 3, 0},
                           {{0, 3, 2, 1}, {0, 1, 4, 0}, {1, 2, 4, 0}, {2, 3, 4, 0}, {3, 0, 4, 0}, {0}},
                           2,
                           {{0, 1, 2, 4}, {0, 2, 3, 4}}};
  static const Topo pri = {6, 5, {3, 3, 4, 4, 4, 0},
                           {{0, 2, 1, 0}, {3, 4, 5, 0}, {0, 1, 4, 3}, {1, 2, 5, 4}, {2, 0, 3, 5}, {0}},
                           3,
                           {{0, 1, 2, 5}, {0, 1, 5, 4}, {0, 4, 5, 3}}};
  switch (type) {
    case 1: return hex;
    case 2: return tet;
    case 3: return pyr;
    default: return pri;
  }
}

// ------------------------------------------------------------ quadrature
// Gauss-Legendre nodes/weights on [-1,1] by Newton iteration.
inline void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < n; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; ++k) {
        double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      if (n == 1) { p1 = z; p0 = 1.0; }
      double dp = n * (z * p1 - p0) / (z * z - 1.0);
      double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    double p0 = 1.0, p1 = z;
    for (int k = 2; k <= n; ++k) {
      double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    if (n == 1) { p0 = 1.0; p1 = z; }
    double dp = n * (z * p1 - p0) / (z * z - 1.0);
    x[i] = -z;
    w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
  if (n == 1) { x[0] = 0.0; w[0] = 2.0; }
}

// Collapsed (conical product) rule on the unit tetrahedron; points in
// barycentric-free form (xi, eta, zeta), weights summing to 1.  Exact for
// polynomials of degree <= 2n-3.
struct TetRule {
  std::vector<std::array<double, 3>> p;
  std::vector<double> w;
};
inline TetRule tet_rule(int n) {
  std::vector<double> gx, gw;
  gauss_legendre(n, gx, gw);
  TetRule r;
  double sum = 0.0;
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b)
      for (int c = 0; c < n; ++c) {
        double u = 0.5 * (gx[a] + 1.0), v = 0.5 * (gx[b] + 1.0), t = 0.5 * (gx[c] + 1.0);
        double wt = 0.125 * gw[a] * gw[b] * gw[c] * (1.0 - u) * (1.0 - u) * (1.0 - v);
        r.p.push_back({u, (1.0 - u) * v, (1.0 - u) * (1.0 - v) * t});
        r.w.push_back(wt);
        sum += wt;
      }
  for (auto& x : r.w) x /= sum;
  return r;
}

// ------------------------------------------------------------ monomials
// Basis ordering of BASIS_REC (src/basis.f90:24-100): degree by degree; in
// a degree, powers of z ascending, then powers of y ascending.
struct Mono {
  int e[3];
};
inline std::vector<Mono> monomials(int order) {
  std::vector<Mono> m;
  for (int n = 1; n <= order; ++n)
    for (int c = 0; c <= n; ++c)
      for (int b = 0; b <= n - c; ++b) m.push_back({{n - c - b, b, c}});
  return m;
}
}  // namespace ucrules
