// Special functions of the APW matching (src/match.f90:83-185): spherical
// harmonics, spherical Bessel functions and their radial derivatives, and the
// derivatives of an interpolating polynomial.  They compute what genylm,
// sbessel, sbesseldm and polynom compute in the reference, by the methods
// named at each routine.
//
// The routines are __host__ __device__: the device path of match.cu calls
// them, and a host harness checks them against the oracle.
#pragma once

#include "common.cuh"

constexpr int SPECFUN_LMAX = 20;   // largest l of the device path
constexpr int SPECFUN_MAXD = 6;    // highest radial derivative

// Y_lm(theta, phi) for l <= lmax, written to ylm[(l(l+1)+m) * stride], with
// the Condon-Shortley phase.  Method: fully normalised associated Legendre
// functions Pb(l, m) (orthonormal on the sphere together with e^{i m phi}),
//   Pb(0, 0)   = 1 / sqrt(4 pi)
//   Pb(m, m)   = -sqrt((2m+1) / 2m) sin(theta) Pb(m-1, m-1)
//   Pb(m+1, m) = sqrt(2m+3) cos(theta) Pb(m, m)
//   Pb(l, m)   = a(l,m) [cos(theta) Pb(l-1, m) - Pb(l-2, m) / a(l-1,m)],
//                a(l,m) = sqrt((4l^2 - 1) / (l^2 - m^2)),
// Y_lm = Pb(l, m) e^{i m phi} with e^{i m phi} advanced by one complex
// rotation per m, and Y_l,-m = (-1)^m conj(Y_lm).
EXCFV_HD void sf_ylm(int lmax, double theta, double phi, cplx* ylm, int stride) {
  const double ct = cos(theta), st = sin(theta);
  const cplx rot = cmk(cos(phi), sin(phi));
  cplx eim = cmk(1.0, 0.0);           // e^{i m phi}
  double pmm = 0.28209479177387814347;  // Pb(m, m); 1 / sqrt(4 pi) at m = 0
  for (int m = 0; m <= lmax; ++m) {
    if (m > 0) {
      pmm *= -sqrt((2.0 * m + 1.0) / (2.0 * m)) * st;
      eim = cmul(eim, rot);
    }
    double p2 = 0.0, p1 = pmm;       // Pb(l-2, m), Pb(l-1, m) entering l = m + 1
    for (int l = m; l <= lmax; ++l) {
      double p;
      if (l == m) {
        p = pmm;
      } else if (l == m + 1) {
        p = sqrt(2.0 * m + 3.0) * ct * pmm;
        p2 = pmm;
        p1 = p;
      } else {
        const double a = sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)m * m));
        const double ap = sqrt((4.0 * (l - 1) * (l - 1) - 1.0) / ((double)(l - 1) * (l - 1) - (double)m * m));
        p = a * (ct * p1 - p2 / ap);
        p2 = p1;
        p1 = p;
      }
      const int c = l * (l + 1);
      const cplx y = cmk(p * eim.x, p * eim.y);
      ylm[(c + m) * stride] = y;
      if (m > 0) {
        const double sg = (m & 1) ? -1.0 : 1.0;
        ylm[(c - m) * stride] = cmk(sg * y.x, -sg * y.y);
      }
    }
  }
}

// j_l(x), l = 0..lmax, x >= 0, lmax <= SPECFUN_LMAX + SPECFUN_MAXD.
//   x < 1:        the power series j_l = x^l/(2l+1)!! sum_k (-x^2/2)^k / (k! (2l+3)...(2l+2k+1))
//   x >= lmax:    upward recurrence j_{l+1} = (2l+1)/x j_l - j_{l-1} from
//                 j_0 = sin x / x, j_1 = (j_0 - cos x) / x (stable for x > l)
//   otherwise:    Miller's method: the same recurrence downward from
//                 L = lmax + 30 with f_{L+1} = 0, f_L = 1, normalised by the
//                 sum rule sum_l (2l+1) j_l(x)^2 = 1 (for 1 <= x < lmax the
//                 values stay below 1e81, so no rescaling is needed)
EXCFV_HD void sf_sbessel(int lmax, double x, double* jl) {
  if (x < 1.0) {
    const double h = -0.5 * x * x;
    double xl = 1.0;  // x^l / (2l+1)!!
    for (int l = 0; l <= lmax; ++l) {
      if (l > 0) xl *= x / (2.0 * l + 1.0);
      double t = 1.0, s = 1.0;
      for (int k = 1; k <= 24; ++k) {
        t *= h / (k * (2.0 * l + 2.0 * k + 1.0));
        s += t;
        if (fabs(t) < 1e-18 * fabs(s)) break;
      }
      jl[l] = xl * s;
    }
    return;
  }
  if (x >= (double)lmax) {
    const double sx = sin(x), cx = cos(x), xi = 1.0 / x;
    jl[0] = sx * xi;
    if (lmax >= 1) jl[1] = (jl[0] - cx) * xi;
    for (int l = 1; l < lmax; ++l) jl[l + 1] = (2.0 * l + 1.0) * xi * jl[l] - jl[l - 1];
    return;
  }
  const int L = lmax + 30;
  const double xi = 1.0 / x;
  double fp = 0.0, f = 1.0;     // f_{l+1}, f_l at l = L
  double sum = (2.0 * L + 1.0); // sum of (2l+1) f_l^2 for l >= current
  for (int l = L; l > 0; --l) {
    const double fm = (2.0 * l + 1.0) * xi * f - fp;  // f_{l-1}
    fp = f;
    f = fm;
    sum += (2.0 * (l - 1) + 1.0) * f * f;
    if (l - 1 <= lmax) jl[l - 1] = f;
  }
  // f_l = j_l / j_L(x) with j_L(x) > 0 (x < lmax < L lies before its first
  // zero), so the positive root keeps the signs
  const double nrm = 1.0 / sqrt(sum);
  for (int l = 0; l <= lmax; ++l) jl[l] *= nrm;
}

// d^m/dx^m j_l(x), l = 0..lmax, m <= SPECFUN_MAXD.  Method: the two-term
// identity j_l' = (l j_{l-1} - (l+1) j_{l+1}) / (2l+1), applied m times, gives
// d^m j_l as a combination sum_s c_s j_{l+s}, |s| <= m, with coefficients that
// depend on l only; the j_{-1} term always carries the factor l + s = 0.
EXCFV_HD void sf_sbessel_deriv(int m, int lmax, double x, double* djl) {
  double jl[SPECFUN_LMAX + SPECFUN_MAXD + 1];
  sf_sbessel(lmax + m, x, jl);
  for (int l = 0; l <= lmax; ++l) {
    double c[2 * SPECFUN_MAXD + 1], nc[2 * SPECFUN_MAXD + 1];
    for (int s = 0; s <= 2 * m; ++s) c[s] = 0.0;
    c[m] = 1.0;  // offset s stored at index s + m
    for (int it = 0; it < m; ++it) {
      for (int s = 0; s <= 2 * m; ++s) nc[s] = 0.0;
      for (int s = 0; s <= 2 * m; ++s) {
        if (c[s] == 0.0) continue;
        const int q = l + s - m;  // order of this term
        const double den = 1.0 / (2.0 * q + 1.0);
        if (q > 0) nc[s - 1] += c[s] * q * den;
        nc[s + 1] -= c[s] * (q + 1) * den;
      }
      for (int s = 0; s <= 2 * m; ++s) c[s] = nc[s];
    }
    double acc = 0.0;
    for (int s = 0; s <= 2 * m; ++s) {
      const int q = l + s - m;
      if (c[s] != 0.0 && q >= 0) acc += c[s] * jl[q];
    }
    djl[l] = acc;
  }
}

// d^m/dx^m at x of the polynomial through (xa[i], ya[i]), i < np <= 16.
// Method: Newton divided differences, then the Newton form re-expanded in
// powers of (t - x) by nested multiplication with (t - x_i) = (t - x) +
// (x - x_i); the m-th Taylor coefficient times m! is the derivative.
EXCFV_HD double sf_polynom_deriv(int m, int np, const double* xa, const double* ya, double x) {
  if (m >= np || m < 0) return 0.0;
  double c[16], a[16];
  for (int i = 0; i < np; ++i) c[i] = ya[i];
  for (int k = 1; k < np; ++k)
    for (int i = np - 1; i >= k; --i) c[i] = (c[i] - c[i - 1]) / (xa[i] - xa[i - k]);
  for (int i = 0; i < np; ++i) a[i] = 0.0;
  a[0] = c[np - 1];
  int deg = 0;
  for (int i = np - 2; i >= 0; --i) {
    const double d = x - xa[i];
    a[deg + 1] = a[deg];
    for (int k = deg; k >= 1; --k) a[k] = a[k - 1] + d * a[k];
    a[0] = d * a[0] + c[i];
    ++deg;
  }
  double fact = 1.0;
  for (int k = 2; k <= m; ++k) fact *= k;
  return fact * a[m];
}
