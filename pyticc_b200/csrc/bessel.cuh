// Bessel functions of real order for asymptotic matching, in FP64, on the device.
//
// J_nu, Y_nu and their derivatives (nu >= 0, x > 0) follow Steed's method:
//   * CF1: f = J'_nu / J_nu from the continued fraction of the ratios J_{nu+k}/J_{nu+k-1}
//     (modified Lentz); the product of the signs of its denominators is sign(J_nu);
//   * downward recurrence from nu to mu = nu - nl (|mu| <= 1/2 for x < 2);
//   * x >= 2: CF2, the complex continued fraction for (J'_mu + iY'_mu)/(J_mu + iY_mu),
//     closed with the Wronskian J Y' - J' Y = 2/(pi x);
//     x < 2: Temme's series for Y_mu and Y_{mu+1}, with 1/Gamma(1 +- mu) from the
//     Taylor series of the reciprocal gamma function;
//   * upward recurrence of Y from mu to nu.
// K_{nu-1}(x)/K_nu(x) is a ratio of two trapezoidal sums of the integral
// K_a(x) = int_0^inf exp(-x cosh t) cosh(a t) dt, whose integrand is analytic in a strip,
// so the rule converges geometrically; sums are formed relative to the integrand peak,
// so neither underflow (large x) nor overflow (large order) occurs.
#pragma once

#include <cmath>

#ifndef __CUDACC__
using std::isfinite;
#endif

#ifdef __CUDACC__
#define TICC_HD __host__ __device__
#else
#define TICC_HD
#endif

namespace ticc {

constexpr double kPiD = 3.14159265358979323846;
constexpr int kBesselMaxIter = 2000000;

// Taylor coefficients of 1/Gamma(1+z) about z = 0 (the first is 1, the second Euler's constant).
TICC_HD inline double rgamma_coefficient(int k) {
  constexpr double c[21] = {1.0,
                            0.57721566490153286061,
                            -0.65587807152025388108,
                            -0.042002635034095235529,
                            0.1665386113822914895,
                            -0.042197734555544336748,
                            -0.0096219715278769735621,
                            0.0072189432466630995424,
                            -0.0011651675918590651121,
                            -0.00021524167411495097282,
                            0.00012805028238811618615,
                            -0.000020134854780788238656,
                            -1.2504934821426706573e-6,
                            1.1330272319816958824e-6,
                            -2.0563384169776071035e-7,
                            6.1160951044814158179e-9,
                            5.0020076444692229301e-9,
                            -1.1812745704870201446e-9,
                            1.0434267116911005105e-10,
                            7.782263439905071254e-12,
                            -3.6968056186422057082e-12};
  return c[k];
}

// 1/Gamma(1+z), |z| <= 1/2.
TICC_HD inline double rgamma_1p(double z) {
  double s = rgamma_coefficient(20);
  for (int k = 19; k >= 0; --k) s = s * z + rgamma_coefficient(k);
  return s;
}

// (ar + i ai) / (br + i bi) by Smith's scaled division (no overflow/underflow of |b|^2).
TICC_HD inline void complex_div(double ar, double ai, double br, double bi, double& qr, double& qi) {
  if (fabs(br) >= fabs(bi)) {
    const double r = bi / br, d = br + bi * r;
    qr = (ar + ai * r) / d;
    qi = (ai - ar * r) / d;
  } else {
    const double r = br / bi, d = br * r + bi;
    qr = (ar * r + ai) / d;
    qi = (ai * r - ar) / d;
  }
}

struct BesselJY {
  double J, Y, Jp, Yp;
  int ok;
};

TICC_HD inline BesselJY bessel_jy(double nu, double x) {
  BesselJY out{0.0, 0.0, 0.0, 0.0, 0};
  const double tiny = 1.0e-300, eps = 1.0e-16;
  const double stop = 4.0e-16;  // |delta - 1| within a few ulp ends a continued fraction
  int nl = (x < 2.0) ? (int)(nu + 0.5) : (int)(nu - x + 1.5);
  if (nl < 0) nl = 0;
  const double mu = nu - nl;

  // CF1
  double f = (nu / x > tiny) ? nu / x : tiny;
  double C = f, D = 0.0;
  int sign = 1;
  int k = 1;
  for (; k < kBesselMaxIter; ++k) {
    const double b = 2.0 * (nu + k) / x;
    D = b - D;
    if (fabs(D) < tiny) D = tiny;
    C = b - 1.0 / C;
    if (fabs(C) < tiny) C = tiny;
    D = 1.0 / D;
    const double delta = C * D;
    f *= delta;
    if (D < 0.0) sign = -sign;
    if (fabs(delta - 1.0) < stop) break;
  }
  if (k >= kBesselMaxIter) return out;

  // downward recurrence of (J, J') from nu to mu, with rescaling
  double Jl = sign, Jpl = f * Jl, lam = nu;
  int rescales = 0;
  for (int i = 0; i < nl; ++i) {
    const double Jm = (lam / x) * Jl + Jpl;
    const double Jpm = ((lam - 1.0) / x) * Jm - Jl;
    Jl = Jm;
    Jpl = Jpm;
    lam -= 1.0;
    if (fabs(Jl) > 1.0e250) {
      Jl *= 1.0e-250;
      Jpl *= 1.0e-250;
      ++rescales;
    }
  }
  const double Jmu_c = Jl;
  const double fmu = Jpl / Jl;
  const double W = 2.0 / (kPiD * x);
  double Jmu, Ymu, Ymu1;

  if (x < 2.0) {
    const double x2 = 0.5 * x;
    const double pimu = kPiD * mu;
    const double fact = (fabs(pimu) < eps) ? 1.0 : pimu / sin(pimu);
    const double dd = -log(x2);
    double e = mu * dd;
    const double fact2 = (fabs(e) < eps) ? 1.0 : sinh(e) / e;
    const double m2 = mu * mu;
    double g1 = 0.0, g2 = 0.0;
    for (int j = 19; j >= 1; j -= 2) g1 = g1 * m2 + rgamma_coefficient(j);
    for (int j = 20; j >= 0; j -= 2) g2 = g2 * m2 + rgamma_coefficient(j);
    g1 = -g1;
    double ff = 2.0 / kPiD * fact * (g1 * cosh(e) + g2 * fact2 * dd);
    e = exp(e);
    double p = e / (kPiD * rgamma_1p(mu));
    double q = 1.0 / (e * kPiD * rgamma_1p(-mu));
    const double half = 0.5 * pimu;
    const double fact3 = (fabs(half) < eps) ? 1.0 : sin(half) / half;
    const double r = kPiD * half * fact3 * fact3;
    double c = 1.0;
    const double d = -x2 * x2;
    double sumy = ff + r * q, sumy1 = p;
    int j = 1;
    for (; j < kBesselMaxIter; ++j) {
      ff = (j * ff + p + q) / (j * j - m2);
      c *= d / j;
      p /= (j - mu);
      q /= (j + mu);
      const double del = c * (ff + r * q);
      sumy += del;
      sumy1 += c * p - j * del;
      if (fabs(del) < (1.0 + fabs(sumy)) * eps) break;
    }
    if (j >= kBesselMaxIter) return out;
    Ymu = -sumy;
    Ymu1 = -sumy1 * (2.0 / x);
    const double Ypmu = (mu / x) * Ymu - Ymu1;
    Jmu = W / (Ypmu - fmu * Ymu);
  } else {
    // CF2 tail a1/(b1 + a2/(b2 + ...)), a_k = (k - 1/2)^2 - mu^2, b_k = 2(x + i k)
    double fr = tiny, fi = 0.0, Cr = fr, Ci = 0.0, Dr = 0.0, Di = 0.0;
    int j = 1;
    for (; j < kBesselMaxIter; ++j) {
      const double ak = (j - 0.5) * (j - 0.5) - mu * mu;
      const double br = 2.0 * x, bi = 2.0 * j;
      // D = 1/(b + a D)
      double tr = br + ak * Dr, ti = bi + ak * Di;
      if (fabs(tr) + fabs(ti) < tiny) tr = tiny;
      complex_div(1.0, 0.0, tr, ti, Dr, Di);
      // C = b + a / C
      double qr, qi;
      complex_div(ak, 0.0, Cr, Ci, qr, qi);
      tr = br + qr;
      ti = bi + qi;
      if (fabs(tr) + fabs(ti) < tiny) tr = tiny;
      Cr = tr;
      Ci = ti;
      const double dlr = Cr * Dr - Ci * Di, dli = Cr * Di + Ci * Dr;
      const double nfr = fr * dlr - fi * dli, nfi = fr * dli + fi * dlr;
      fr = nfr;
      fi = nfi;
      if (fabs(dlr - 1.0) + fabs(dli) < stop) break;
    }
    if (j >= kBesselMaxIter) return out;
    // p + iq = -1/(2x) + i + (i/x) * tail
    const double p = -0.5 / x - fi / x;
    const double q = 1.0 + fr / x;
    const double gam = (p - fmu) / q;
    Jmu = sqrt(W / (q + gam * (p - fmu)));
    Jmu = copysign(Jmu, Jmu_c);
    Ymu = gam * Jmu;
    const double Ypmu = Ymu * (p + q / gam);
    Ymu1 = (mu / x) * Ymu - Ypmu;
  }

  const double scale = Jmu / Jmu_c;
  double Jnu = sign * scale;
  for (int i = 0; i < rescales; ++i) Jnu *= 1.0e-250;
  out.J = Jnu;
  out.Jp = f * Jnu;
  double Y0 = Ymu, Y1 = Ymu1;
  lam = mu;
  for (int i = 0; i < nl; ++i) {
    const double Y2 = (2.0 * (lam + 1.0) / x) * Y1 - Y0;
    Y0 = Y1;
    Y1 = Y2;
    lam += 1.0;
  }
  out.Y = Y0;
  out.Yp = (nu / x) * Y0 - Y1;
  out.ok = isfinite(out.J) && isfinite(out.Y) && isfinite(out.Jp) && isfinite(out.Yp);
  return out;
}

// Riccati-Bessel j, n and their x-derivatives for angular momentum ell (nu = ell + 1/2).
TICC_HD inline BesselJY riccati_bessel(double ell, double x) {
  BesselJY b = bessel_jy(ell + 0.5, x);
  const double s = sqrt(kPiD * x / 2.0);
  BesselJY r;
  r.J = s * b.J;
  r.Y = s * b.Y;
  r.Jp = s * (b.Jp + 0.5 * b.J / x);
  r.Yp = s * (b.Yp + 0.5 * b.Y / x);
  r.ok = b.ok && isfinite(r.J) && isfinite(r.Y) && isfinite(r.Jp) && isfinite(r.Yp);
  return r;
}

TICC_HD inline double k_integrand(double x, double t, double order, double shift) {
  return exp(-x * (cosh(t) - 1.0) + order * t - shift) * 0.5 * (1.0 + exp(-2.0 * order * t));
}

// K_{nu-1}(x) / K_nu(x) for nu >= 0, x > 0; returns NaN if the sum did not terminate.
TICC_HD inline double bessel_k_ratio(double nu, double x) {
  const double a = fabs(nu), b = fabs(nu - 1.0);
  const double kap = sqrt(hypot(x, a));
  const double h = fmin(0.1, 0.25 / fmax(1.0, kap));
  const double tstar = asinh(a / x);
  const double pmax = -x * (cosh(tstar) - 1.0) + a * tstar;
  const long long k0 = (long long)(tstar / h);
  double sa = 0.0, sb = 0.0;
  long long k = k0;
  for (int it = 0;; ++it) {
    if (it > kBesselMaxIter) return NAN;
    const double t = k * h, w = (k == 0) ? 0.5 : 1.0;
    sa += w * k_integrand(x, t, a, pmax);
    sb += w * k_integrand(x, t, b, pmax);
    if (-x * (cosh(t) - 1.0) + a * t < pmax - 60.0) break;
    ++k;
  }
  for (k = k0 - 1; k >= 0; --k) {
    const double t = k * h, w = (k == 0) ? 0.5 : 1.0;
    sa += w * k_integrand(x, t, a, pmax);
    sb += w * k_integrand(x, t, b, pmax);
    if (-x * (cosh(t) - 1.0) + a * t < pmax - 60.0) break;
  }
  return sb / sa;
}

// K'_nu(x)/K_nu(x) = -K_{nu-1}(x)/K_nu(x) - nu/x.
TICC_HD inline double bessel_k_logd(double nu, double x) { return -bessel_k_ratio(nu, x) - nu / x; }

}  // namespace ticc
