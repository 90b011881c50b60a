// Host-side checks of the derivative building blocks of the adjoint
// (ucns3d_b200/csrc/engine/ad.cuh), run by tests/test_ad_host.py:
//   1. forward-mode duals through rot_f / hllc / rot_b against central
//      differences evaluated in long double (reported: worst error relative
//      to 1e-3 + |derivative|);
//   2. the hand-written HLLC adjoint (ad::hllc_adj) against the transposed
//      dual Jacobian for random states and weights, subsonic and supersonic
//      (reported: worst error relative to the largest component).
// Prints "fd <err> adj <err>".
#include <cmath>
#include <cstdio>
#include <random>

#include "../ucns3d_b200/csrc/engine/ad.cuh"

namespace ucg {
__host__ __device__ inline long double value(long double x) { return x; }
}  // namespace ucg

using namespace ucg;
using ad::Dual;

int main() {
  std::mt19937_64 rng(3);
  std::uniform_real_distribution<double> U(-1, 1);
  double worst_fd = 0, worst_adj = 0;
  for (int t = 0; t < 20000; ++t) {
    const double sc = (t % 3 == 0) ? 3.0 : 0.6;
    double pl[5] = {1 + 0.5 * U(rng), sc * U(rng), 0.4 * U(rng), 0.4 * U(rng), 1 + 0.5 * U(rng)};
    double pr[5] = {1 + 0.5 * U(rng), sc * U(rng), 0.4 * U(rng), 0.4 * U(rng), 1 + 0.5 * U(rng)};
    double cl[5], cr[5], fb[5];
    prim2cons(1.4, pl, cl);
    prim2cons(1.4, pr, cr);
    for (int v = 0; v < 5; ++v) fb[v] = U(rng);
    const double r[4] = {std::cos(0.3 * t), std::sin(0.3 * t), std::cos(0.7 * t), std::sin(0.7 * t)};
    Dual<10> L[5], R[5], a[5], b[5], h[5], f[5];
    for (int v = 0; v < 5; ++v) {
      L[v] = Dual<10>(cl[v]);
      L[v].d[v] = 1;
      R[v] = Dual<10>(cr[v]);
      R[v].d[5 + v] = 1;
    }
    rot_f(r, R, b);
    rot_f(r, L, a);
    hllc(1.4, a, b, h);
    rot_b(r, h, f);
    if (t < 2000)
      for (int k = 0; k < 10; ++k) {
        const long double eps = 1e-7L;
        long double xp[10], xm[10];
        for (int i = 0; i < 5; ++i) {
          xp[i] = xm[i] = cl[i];
          xp[5 + i] = xm[5 + i] = cr[i];
        }
        const long double s = std::fabs((double)xp[k]) > 0.1 ? std::fabs((double)xp[k]) : 0.1L;
        xp[k] += eps * s;
        xm[k] -= eps * s;
        long double ap[5], bp[5], hp[5], fp[5], am[5], bm[5], hm[5], fm[5];
        rot_f(r, xp + 5, bp);
        rot_f(r, xp, ap);
        hllc(1.4, ap, bp, hp);
        rot_b(r, hp, fp);
        rot_f(r, xm + 5, bm);
        rot_f(r, xm, am);
        hllc(1.4, am, bm, hm);
        rot_b(r, hm, fm);
        for (int v = 0; v < 5; ++v) {
          const double fd = (double)((fp[v] - fm[v]) / (2 * eps * s));
          worst_fd = std::fmax(worst_fd, std::fabs(fd - f[v].d[k]) / (1e-3 + std::fabs(fd)));
        }
      }
    // adjoint of HLLC in the face frame: fb^T d hllc / d(a, b)
    Dual<10> A[5], B[5], H[5];
    for (int v = 0; v < 5; ++v) {
      A[v] = Dual<10>(cl[v]);
      A[v].d[v] = 1;
      B[v] = Dual<10>(cr[v]);
      B[v].d[5 + v] = 1;
    }
    hllc(1.4, A, B, H);
    double ref[10] = {0}, scale = 0;
    for (int k = 0; k < 10; ++k) {
      for (int v = 0; v < 5; ++v) ref[k] += fb[v] * H[v].d[k];
      scale = std::fmax(scale, std::fabs(ref[k]));
    }
    double clb[5] = {0}, crb[5] = {0};
    ad::hllc_adj(1.4, cl, cr, fb, clb, crb);
    double err = 0;
    for (int k = 0; k < 5; ++k)
      err = std::fmax(err, std::fmax(std::fabs(clb[k] - ref[k]), std::fabs(crb[k] - ref[5 + k])));
    worst_adj = std::fmax(worst_adj, err / (scale + 1e-300));
  }
  std::printf("fd %.3e adj %.3e\n", worst_fd, worst_adj);
  return 0;
}
