// Host-side evaluation of the engine's own boundary ghost states
// (ucg::boundary_ghost in ucns3d_b200/csrc/engine/device.cuh, the function
// the face kernels call), compiled with nvcc as host code and run by
// tests/test_bc_kat.py against the BOUNDARYS known-answer vectors.
// stdin: "gamma rho u v w p" (free stream), then per case
// "code boundtype governing angle1 angle2 U0..U4"; stdout: the ghost state, one line
// per case.
#include <cmath>
#include <cstdio>

#include "../ucns3d_b200/csrc/engine/device.cuh"

int main() {
  ucg::Problem p{};
  double free[5];
  if (std::scanf("%lf %lf %lf %lf %lf %lf", &p.gamma, &free[0], &free[1], &free[2], &free[3], &free[4]) != 6) return 1;
  int code, bt, gov;
  double a1, a2, cl[5];
  while (std::scanf("%d %d %d %lf %lf %lf %lf %lf %lf %lf", &code, &bt, &gov, &a1, &a2, &cl[0], &cl[1], &cl[2],
                    &cl[3], &cl[4]) == 10) {
    p.boundtype = bt;
    p.governing = gov;
    const double r[4] = {std::cos(a1), std::sin(a1), std::cos(a2), std::sin(a2)};
    double cr[5];
    ucg::boundary_ghost<double>(p, code, r, cl, free, cr);
    std::printf("%.17g %.17g %.17g %.17g %.17g\n", cr[0], cr[1], cr[2], cr[3], cr[4]);
  }
  return 0;
}
