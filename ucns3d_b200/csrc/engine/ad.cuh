// Forward-mode dual numbers for the discrete adjoint and tangent kernels.
//
// Dual<N> carries a value and N directional derivatives.  The templated gas,
// rotation, HLLC, limiter and boundary functions of device.cuh evaluated on
// Dual<N> give their exact derivatives (up to rounding) along N seeded
// directions: N = 1 for the tangent, N = 10 for the 5x10 Jacobian of a face
// flux with respect to its two states (or state and free-stream state), which
// the adjoint then applies transposed.  Branches (wave-speed selection, the
// sign of the contact speed, limiter cases, supersonic switches) follow the
// values, so each derivative is that of the branch the primal takes.
//
// The type and its overloads live in their own namespace so that they are
// found only by argument-dependent lookup and never shadow the double
// versions of sqrt/fmin/... .
#pragma once

#include "device.cuh"

namespace ucg {
namespace ad {

template <int N>
struct Dual {
  double v;
  double d[N];
  __host__ __device__ __forceinline__ Dual() {}
  __host__ __device__ __forceinline__ Dual(double x) : v(x) {
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = 0.0;
  }
};

template <int N>
__host__ __device__ __forceinline__ double value(const Dual<N>& a) {
  return a.v;
}

template <int N>
__host__ __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
  Dual<N> r;
  r.v = -a.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v / b.v;
  const double ib = 1.0 / b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double b) {
  Dual<N> r = a;
  r.v = a.v + b;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator+(double a, const Dual<N>& b) {
  Dual<N> r = b;
  r.v = a + b.v;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double b) {
  Dual<N> r = a;
  r.v = a.v - b;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator-(double a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a - b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = -b.d[i];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double b) {
  Dual<N> r;
  r.v = a.v * b;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator*(double a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a * b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a * b.d[i];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double b) {
  Dual<N> r;
  r.v = a.v / b;
  const double ib = 1.0 / b;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * ib;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator/(double a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a / b.v;
  const double s = -r.v / b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = s * b.d[i];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> sqrt(const Dual<N>& a) {
  Dual<N> r;
  r.v = ::sqrt(a.v);
  const double s = 0.5 / r.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = s * a.d[i];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> fabs(const Dual<N>& a) {
  return a.v < 0.0 ? -a : a;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> fmin(const Dual<N>& a, const Dual<N>& b) {
  return b.v < a.v ? b : a;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> fmax(const Dual<N>& a, const Dual<N>& b) {
  return b.v > a.v ? b : a;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> fmin(const Dual<N>& a, double b) {
  return b < a.v ? Dual<N>(b) : a;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> fmax(const Dual<N>& a, double b) {
  return b > a.v ? Dual<N>(b) : a;
}

// ---------------------------------------------------------------- HLLC adjoint
// Reverse mode of hllc() (device.cuh) for double states in the face frame:
// given fb = dJ/dflux, accumulates clb += (dflux/dcl)^T fb and
// crb += (dflux/dcr)^T fb.  One forward sweep recomputes the intermediates,
// one backward sweep applies the chain rule in reverse order; the branches
// (wave-speed selection, clamping at zero, the side picked by the sign of
// the contact speed) are those of the forward values.
__host__ __device__ inline void hllc_adj(double gamma, const double* cl, const double* cr, const double* fb,
                                         double* clb, double* crb) {
  const double g1 = gamma - 1.0;
  // ---- forward (reciprocals formed once: 9 divisions in all)
  const double rl = cl[0], irl = 1.0 / rl, ul = cl[1] * irl, vl = cl[2] * irl, wl = cl[3] * irl;
  const double kl = ul * ul + vl * vl + wl * wl;
  const double pl = g1 * (cl[4] - 0.5 * rl * kl);
  const double rr = cr[0], irr = 1.0 / rr, ur = cr[1] * irr, vr = cr[2] * irr, wr = cr[3] * irr;
  const double kr = ur * ur + vr * vr + wr * wr;
  const double pr = g1 * (cr[4] - 0.5 * rr * kr);
  const double el = cl[4], er = cr[4];
  const double ccl = ::sqrt(gamma * pl * irl), ccr = ::sqrt(gamma * pr * irr);
  const double srl = ::sqrt(rl), srr = ::sqrt(rr), ssum = srl + srr, issum = 1.0 / ssum;
  const double du = ur - ul;
  const double T1 = ccl * ccl * srl + ccr * ccr * srr;
  const double P = (srl * srr) * (issum * issum);
  const double q = T1 * issum + 0.5 * P * (du * du);
  const double cc2 = ::sqrt(q);
  const double uu2 = (ul * srl + ur * srr) * issum;
  // sl = min(min(ul - ccl, uu2 - cc2), 0): which term
  const double sl1 = ul - ccl, sl2 = uu2 - cc2;
  const double slm = sl2 < sl1 ? sl2 : sl1;
  const int slb = 0.0 < slm ? 0 : (sl2 < sl1 ? 2 : 1);
  const double sl = slb == 0 ? 0.0 : slm;
  const double sr1 = ur + ccr, sr2 = uu2 + cc2;
  const double srm = sr2 > sr1 ? sr2 : sr1;
  const int srb = 0.0 > srm ? 0 : (sr2 > sr1 ? 2 : 1);
  const double sr = srb == 0 ? 0.0 : srm;
  const double num = pr - pl + rl * ul * (sl - ul) - rr * ur * (sr - ur);
  const double den = rl * (sl - ul) - rr * (sr - ur);
  const double iden = 1.0 / den;
  const double sm = num * iden;
  const bool left = copysign(1.0, sm) > 0.0;
  // ---- backward: adjoints of the intermediates
  double rlb = 0, ulb = 0, vlb = 0, wlb = 0, plb = 0, elb = 0;
  double rrb = 0, urb = 0, vrb = 0, wrb = 0, prb = 0, erb = 0;
  double slb_ = 0, srb_ = 0, smb = 0;
  {
    // active side: F = fs0 + s (mus - c) terms (s = sl or sr)
    const double rs = left ? rl : rr, us = left ? ul : ur, vs = left ? vl : vr, ws = left ? wl : wr;
    const double ps = left ? pl : pr, es = left ? el : er, s = left ? sl : sr;
    const double* cs = left ? cl : cr;
    double* csb = left ? clb : crb;
    const double irs = left ? irl : irr;
    const double Bq = rs * (s - us);            // rho (s - u)
    const double iBq = 1.0 / Bq;
    const double D1 = s - sm;
    const double iD1 = 1.0 / D1;
    const double mus = Bq * iD1;                // star density factor
    const double A = sm - us, Bt = sm + ps * iBq;
    const double lasts = es * irs + A * Bt;
    const double fs0 = rs * us;
    double rsb = 0, usb = 0, vsb = 0, wsb = 0, psb = 0, esb = 0, sb = 0;
    // F0 = fs0 + s (mus - c0); F1 = fs0 us + ps + s (mus sm - c1);
    // F2 = fs0 vs + s (mus vs - c2); F3 = fs0 ws + s (mus ws - c3);
    // F4 = us (es + ps) + s (mus lasts - c4)
    const double fs0b = fb[0] + fb[1] * us + fb[2] * vs + fb[3] * ws;
    sb += fb[0] * (mus - cs[0]) + fb[1] * (mus * sm - cs[1]) + fb[2] * (mus * vs - cs[2]) +
          fb[3] * (mus * ws - cs[3]) + fb[4] * (mus * lasts - cs[4]);
    const double musb = s * (fb[0] + fb[1] * sm + fb[2] * vs + fb[3] * ws + fb[4] * lasts);
    csb[0] -= s * fb[0];
    csb[1] -= s * fb[1];
    csb[2] -= s * fb[2];
    csb[3] -= s * fb[3];
    csb[4] -= s * fb[4];
    usb += fb[1] * fs0 + fb[4] * (es + ps);
    vsb += fb[2] * (fs0 + s * mus);
    wsb += fb[3] * (fs0 + s * mus);
    psb += fb[1] + fb[4] * us;
    esb += fb[4] * us;
    smb += fb[1] * s * mus;
    const double lastb = fb[4] * s * mus;
    // fs0 = rs us
    rsb += fs0b * us;
    usb += fs0b * rs;
    // lasts = es/rs + A Bt, A = sm - us, Bt = sm + ps/Bq
    esb += lastb * irs;
    rsb -= lastb * es * (irs * irs);
    const double Ab = lastb * Bt, Btb = lastb * A;
    smb += Ab;
    usb -= Ab;
    smb += Btb;
    psb += Btb * iBq;
    double Bqb = -Btb * ps * (iBq * iBq);
    // mus = Bq / D1, D1 = s - sm
    Bqb += musb * iD1;
    const double D1b = -musb * Bq * (iD1 * iD1);
    sb += D1b;
    smb -= D1b;
    // Bq = rs (s - us)
    rsb += Bqb * (s - us);
    sb += Bqb * rs;
    usb -= Bqb * rs;
    if (left) {
      rlb += rsb; ulb += usb; vlb += vsb; wlb += wsb; plb += psb; elb += esb; slb_ += sb;
    } else {
      rrb += rsb; urb += usb; vrb += vsb; wrb += wsb; prb += psb; erb += esb; srb_ += sb;
    }
  }
  // sm = num / den
  const double numb = smb * iden, denb = -smb * num * (iden * iden);
  prb += numb;
  plb -= numb;
  rlb += numb * ul * (sl - ul);
  ulb += numb * rl * (sl - 2.0 * ul);
  slb_ += numb * rl * ul;
  rrb -= numb * ur * (sr - ur);
  urb -= numb * rr * (sr - 2.0 * ur);
  srb_ -= numb * rr * ur;
  rlb += denb * (sl - ul);
  slb_ += denb * rl;
  ulb -= denb * rl;
  rrb -= denb * (sr - ur);
  srb_ -= denb * rr;
  urb += denb * rr;
  // wave speeds
  double cclb = 0, ccrb = 0, uu2b = 0, cc2b = 0;
  if (slb == 1) {
    ulb += slb_;
    cclb -= slb_;
  } else if (slb == 2) {
    uu2b += slb_;
    cc2b -= slb_;
  }
  if (srb == 1) {
    urb += srb_;
    ccrb += srb_;
  } else if (srb == 2) {
    uu2b += srb_;
    cc2b += srb_;
  }
  // uu2 = (ul srl + ur srr) / ssum
  double srlb = 0, srrb = 0, ssumb = 0;
  const double Xb = uu2b * issum;
  ssumb -= uu2b * uu2 * issum;
  ulb += Xb * srl;
  srlb += Xb * ul;
  urb += Xb * srr;
  srrb += Xb * ur;
  // cc2 = sqrt(q), q = T1/ssum + 0.5 P du^2
  const double qb = cc2b * (0.5 / cc2);
  const double T1b = qb * issum;
  const double is2 = issum * issum;
  ssumb -= qb * T1 * is2;
  const double Pb = qb * 0.5 * du * du;
  const double dub = qb * P * du;
  srlb += Pb * srr * is2;
  srrb += Pb * srl * is2;
  ssumb -= Pb * 2.0 * srl * srr * (is2 * issum);
  urb += dub;
  ulb -= dub;
  cclb += T1b * 2.0 * ccl * srl;
  srlb += T1b * ccl * ccl;
  ccrb += T1b * 2.0 * ccr * srr;
  srrb += T1b * ccr * ccr;
  srlb += ssumb;
  srrb += ssumb;
  rlb += srlb * (0.5 * srl * irl);  // 1 / (2 sqrt(rl)) = sqrt(rl) / (2 rl)
  rrb += srrb * (0.5 * srr * irr);
  // ccl = sqrt(gamma pl / rl)
  {
    const double zb = cclb * (0.5 / ccl);
    plb += zb * gamma * irl;
    rlb -= zb * gamma * pl * (irl * irl);
    const double zr = ccrb * (0.5 / ccr);
    prb += zr * gamma * irr;
    rrb -= zr * gamma * pr * (irr * irr);
  }
  // pl = g1 (el - 0.5 rl kl), el = cl[4]
  elb += plb * g1;
  rlb -= plb * g1 * 0.5 * kl;
  const double klb = -plb * g1 * 0.5 * rl;
  ulb += klb * 2.0 * ul;
  vlb += klb * 2.0 * vl;
  wlb += klb * 2.0 * wl;
  erb += prb * g1;
  rrb -= prb * g1 * 0.5 * kr;
  const double krb = -prb * g1 * 0.5 * rr;
  urb += krb * 2.0 * ur;
  vrb += krb * 2.0 * vr;
  wrb += krb * 2.0 * wr;
  // ul = cl1 / rl, ...; rl = cl0, el = cl4
  clb[1] += ulb * irl;
  clb[2] += vlb * irl;
  clb[3] += wlb * irl;
  rlb -= (ulb * ul + vlb * vl + wlb * wl) * irl;
  clb[0] += rlb;
  clb[4] += elb;
  crb[1] += urb * irr;
  crb[2] += vrb * irr;
  crb[3] += wrb * irr;
  rrb -= (urb * ur + vrb * vr + wrb * wr) * irr;
  crb[0] += rrb;
  crb[4] += erb;
}

// Transpose of cons2prim's Jacobian at a state whose primitive form is
// `prim`: cb = (d prim / d cons)^T pb, with rho = c0, u = c1/c0 (v, w
// alike), p = (gamma - 1)(c4 - |c1..3|^2 / (2 c0)).
__device__ __forceinline__ void cons2prim_rev(double gamma, const double* prim, const double* pb, double* cb) {
  const double oo = 1.0 / prim[0], q = pb[4] * (gamma - 1.0);
  cb[0] = pb[0] - (pb[1] * prim[1] + pb[2] * prim[2] + pb[3] * prim[3]) * oo +
          0.5 * q * (prim[1] * prim[1] + prim[2] * prim[2] + prim[3] * prim[3]);
  cb[1] = pb[1] * oo - q * prim[1];
  cb[2] = pb[2] * oo - q * prim[2];
  cb[3] = pb[3] * oo - q * prim[3];
  cb[4] = q;
}

// The variables of the viscous least squares (T, u, v, w) of a conserved
// state u (gradients.f90:502-706), reversed: out = (d(T, u, v, w)/du)^T sb.
__device__ __forceinline__ void visc_vars_rev(const Problem& p, const double* u, const double* sb, double* out) {
  double pr[NV];
  cons2prim(p.gamma, u, pr);
  const double T = pr[4] / (pr[0] * p.r_gas);
  const double pb[NV] = {-sb[0] * T / pr[0], sb[1], sb[2], sb[3], sb[0] / (pr[0] * p.r_gas)};
  cons2prim_rev(p.gamma, pr, pb, out);
}

// The tangent of variable `var` of (T, u, v, w) at the conserved state u
// along du (the forward counterpart of visc_vars_rev).
__device__ __forceinline__ double visc_var_tan(const Problem& p, const double* u, const double* du, int var) {
  double pr[NV];
  cons2prim(p.gamma, u, pr);
  const double oo = 1.0 / pr[0];
  if (var > 0) return (du[var] - pr[var] * du[0]) * oo;
  const double dp = (p.gamma - 1.0) * (du[4] - (pr[1] * du[1] + pr[2] * du[2] + pr[3] * du[3]) +
                                       0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]) * du[0]);
  const double T = pr[4] / (pr[0] * p.r_gas);
  return dp / (pr[0] * p.r_gas) - T * du[0] * oo;
}

}  // namespace ad
}  // namespace ucg
