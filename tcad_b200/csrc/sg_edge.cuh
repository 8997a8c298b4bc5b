// Scharfetter-Gummel edge quantities.  Compiled with -fmad=false so the
// arithmetic rounds step by step in the reference's order
// (pytcad/kernels.py:88-109, pytcad/device2d.py:1449-1479).
#pragma once

#include "common.cuh"

namespace tcad {

// Clip to [-700, 700] keeping NaN (numpy.clip semantics).
__device__ __forceinline__ double clip700(double x) {
  return x < -700.0 ? -700.0 : (x > 700.0 ? 700.0 : x);
}

// B(x) and B'(x) of the series branch |x| < 1e-4 (kernels.py:92-96,105-109).
__device__ __forceinline__ void bern_series(double x, double& B, double& dB) {
  B = (1.0 - x / 2.0) + (x * x) / 12.0;
  dB = (-0.5 + x / 6.0) - (x * x * x) / 180.0;
}

// B(x), B(-x), B'(x), B'(-x).  Three argument bands:
//
//   |x| < 1e-4          the reference's series (kernels.py:92-96, 105-109);
//   1e-4 <= |x| < 1e-2  the reference's own formulas at +x and at -x
//                       (kernels.py:88-109): B = x / expm1(x) and
//                       B' = B (1/x - 1/(1 - e^-x)), two expm1 and the same
//                       divisions.  Here 1/x - 1/(1 - e^-x) cancels (about
//                       4 digits at 1e-4), so the reference's derivative
//                       carries that cancellation's rounding; reproducing
//                       its steps reproduces its values elementwise.
//   |x| >= 1e-2         ONE expm1 and ONE reciprocal serve all four values.
//                       With a = |x|, e = expm1(a) > 0 and r = 1/e:
//                         S  = B(a)   = a r
//                         L  = B(-a)  = a e^a / (e^a - 1) = S + a
//                         dS = B'(a)  = S (1/a - (1 + r)) = r (1 - a (1 + r))
//                         dL = B'(-a) = L (r - 1/a)       = (1 + r) (S - 1)
//                       (L / a = 1 + r and S / a = r).  In this band the
//                       values agree with the reference's formulas to a few
//                       ulp (derivatives within 1e-13 relative; measured
//                       over 4e5 arguments against kernels.py).
__device__ __forceinline__ void bern4(double x, double& Bp, double& Bm, double& dBp,
                                      double& dBm) {
  x = clip700(x);
  const double a = fabs(x);
  if (a < 1e-4) {
    bern_series(x, Bp, dBp);
    bern_series(-x, Bm, dBm);
    return;
  }
  if (a < 1e-2) {
    const double ep = expm1(x), em = expm1(-x);
    Bp = x / ep;
    Bm = (-x) / em;
    dBp = Bp * (1.0 / x - 1.0 / (-em));
    dBm = Bm * (1.0 / (-x) - 1.0 / (-ep));
    return;
  }
  const double e = expm1(a);
  const double r = 1.0 / e;
  const double r1 = 1.0 + r;
  const double S = a * r;
  const double L = S + a;
  const double dS = r * (1.0 - a * r1);
  const double dL = r1 * (S - 1.0);
  const bool pos = x > 0.0;
  Bp = pos ? S : L;
  Bm = pos ? L : S;
  dBp = pos ? dS : dL;
  dBm = pos ? dL : dS;
}

// Everything the two endpoint rows need from one edge (low -> high node).
struct Edge {
  double f;     // Poisson flux (psi_hi - psi_lo) / h
  double Jn;    // electron SG current an (n_hi B(d) - n_lo B(-d))
  double Jp;    // hole SG current -ap (p_hi B(-d') - p_lo B(d'))
  double npsi;  // dJn/dpsi_hi = an (n_hi B'(d) + n_lo B'(-d))
  double nlo;   // dJn/dn_lo = -an B(-d)
  double nhi;   // dJn/dn_hi = an B(d)
  double ppsi;  // dJp/dpsi_hi = ap (p_hi B'(-d') + p_lo B'(d'))
  double plo;   // dJp/dp_lo = ap B(d')
  double phi;   // dJp/dp_hi = -ap B(-d')
};

__device__ __forceinline__ void zero_edge(Edge& e) {
  e.f = e.Jn = e.Jp = e.npsi = e.nlo = e.nhi = e.ppsi = e.plo = e.phi = 0.0;
}

// d = dpsi + dlnnie (electrons), d' = dpsi - dlnnie (holes):
// pytcad/device2d.py:1451-1479.
__device__ __forceinline__ void sg_edge(double psi_lo, double psi_hi, double n_lo,
                                        double n_hi, double p_lo, double p_hi, double an,
                                        double ap, double dl, double h, Edge& e) {
  const double dpsi = psi_hi - psi_lo;
  e.f = dpsi / h;
  double Bp, Bm, dBp, dBm, Bph, Bmh, dBph, dBmh;
  bern4(dpsi + dl, Bp, Bm, dBp, dBm);
  if (dl == 0.0) {
    Bph = Bp; Bmh = Bm; dBph = dBp; dBmh = dBm;
  } else {
    bern4(dpsi - dl, Bph, Bmh, dBph, dBmh);
  }
  e.Jn = an * (n_hi * Bp - n_lo * Bm);
  e.Jp = -ap * (p_hi * Bmh - p_lo * Bph);
  const double Sn = n_hi * dBp + n_lo * dBm;
  const double Sp = p_hi * dBmh + p_lo * dBph;
  e.npsi = an * Sn;
  e.nlo = -an * Bm;
  e.nhi = an * Bp;
  e.ppsi = ap * Sp;
  e.plo = ap * Bph;
  e.phi = -ap * Bmh;
}

// SRH + Auger recombination, scaled (materials.py:474-518 with the
// device's R0/Ns scaling, pytcad/device2d.py:1482-1508), with the
// reference's divisions: R = excess / den, dR/dn = (p den - excess tau_p) /
// den^2, Rs = R / R0, dRs/dn = dR/dn Ns / R0.
__device__ __forceinline__ void recomb(double n, double p, double nie, double taun,
                                       double taup, const double* par, double& Rs,
                                       double& dRsn, double& dRsp) {
  const double Ns = par[TCAD_P_NS], R0 = par[TCAD_P_R0];
  if (par[TCAD_P_SRH] == 0.0) {
    Rs = dRsn = dRsp = 0.0;
    return;
  }
  const double nph = n * Ns, pph = p * Ns;
  const double excess = nph * pph - nie * nie;
  const double den = taup * (nph + nie) + taun * (pph + nie);
  double R = excess / den;
  const double den2 = den * den;
  double dRdn = (pph * den - excess * taup) / den2;
  double dRdp = (nph * den - excess * taun) / den2;
  if (par[TCAD_P_AUGER] != 0.0) {
    const double Cn = par[TCAD_P_CN], Cp = par[TCAD_P_CP];
    const double cc = Cn * nph + Cp * pph;
    R = R + cc * excess;
    dRdn = dRdn + Cn * excess + cc * pph;
    dRdp = dRdp + Cp * excess + cc * nph;
  }
  Rs = R / R0;
  dRsn = dRdn * Ns / R0;
  dRsp = dRdp * Ns / R0;
}

}  // namespace tcad
