// Host-side set-up shared by every entry point that launches the pair math:
// the pair-math constants and the FP64 slow-term table.
#include <cmath>
#include <cstring>
#include <vector>

#include "nbk.h"
#include "nbk_internal.cuh"
#include "nbk_launch.h"

namespace nbk {

// Constants of the energy-switched LJ and the C1-split PME real-space math
// from the caller's parameters (the role of
// CudaComputeNonbonded::getNonbondedCoef, src/CudaComputeNonbonded.C:2318-2349).
void makeConstants(const nbk_params& p, int ljDim, NbkConst& c, NbkConst64& k) {
  const double rc = p.cutoff, rc2 = rc * rc;
  const bool sw = p.switchdist < p.cutoff;
  const double rs2 = sw ? p.switchdist * p.switchdist : rc2;
  const double c1 = sw ? 1.0 / ((rc2 - rs2) * (rc2 - rs2) * (rc2 - rs2)) : 0.0;
  std::memset(&c, 0, sizeof(c));
  std::memset(&k, 0, sizeof(k));
  c.cutoff2 = (float)rc * (float)rc;
  c.plcutoff2 = (float)p.pairlistdist * (float)p.pairlistdist;
  c.rc2 = (float)rc2;
  c.rs2 = (float)rs2;
  c.lj0 = (float)(c1 * (rc2 - 3.0 * rs2));
  c.lj1 = (float)(2.0 * c1);
  c.lj2 = (float)(-12.0 * c1);
  c.lj3 = (float)(12.0 * c1 * rs2);
  c.rc3inv = (float)(1.0 / (rc * rc2));
  c.hA = (float)(1.5 / rc);
  c.hB = (float)(-0.5 / (rc * rc2));
  c.beta = (float)p.ewaldcof;
  c.beta2Pi = (float)(2.0 * p.ewaldcof / std::sqrt(M_PI));
  c.one14 = (float)(1.0 - p.scale14);
  c.pBeta = (float)(kErfcP * p.ewaldcof);
  c.gaussK = (float)(-p.ewaldcof * p.ewaldcof / std::log(2.0));
  c.ljDim = ljDim;
  c.switching = sw ? 1 : 0;
  c.s0 = sw ? 0.0f : 1.0f;
  c.hAd = 1.5 / rc;
  c.hBd = -0.5 / (rc * rc2);
  c.betad = p.ewaldcof;
  k.rc2 = rc2;
  k.rs2 = rs2;
  k.lj0 = c1 * (rc2 - 3.0 * rs2);
  k.lj1 = 2.0 * c1;
  k.lj2 = -12.0 * c1;
  k.lj3 = 12.0 * c1 * rs2;
  k.rc3inv = 1.0 / (rc * rc2);
  k.hA = 1.5 / rc;
  k.hB = -0.5 / (rc * rc2);
  k.beta = p.ewaldcof;
  k.beta2Pi = 2.0 * p.ewaldcof / std::sqrt(M_PI);
  k.one14 = 1.0 - p.scale14;
  k.switching = sw ? 1 : 0;
}

namespace {

// erf(beta sqrt(s)) / sqrt(s), an entire function of s: its power series
// (2 beta/sqrt(pi)) sum_n (-beta^2 s)^n / (n! (2n + 1)) for s < 0 (the first
// row's fit reaches down to s = -D/2, where beta^2 |s| stays below ~10) and
// where beta^2 s is small, FP64 erf elsewhere.
double erfOverR(double beta, double s) {
  if (s < 0.0 || beta * beta * s < 0.5) {
    const double x = -beta * beta * s;
    double term = 1.0, sum = 0.0;
    for (int n = 0; n < 80; ++n) {
      sum += term / (2 * n + 1);
      term *= x / (n + 1);
    }
    return 2.0 * beta / std::sqrt(M_PI) * sum;
  }
  const double r = std::sqrt(s);
  return std::erf(beta * r) / r;
}

}  // namespace

// phi_s(s) = (3 - s/rc^2)/(2 rc) - erf(beta sqrt(s))/sqrt(s).
static double slowPhi(double beta, double rc, double s) {
  return (3.0 - s / (rc * rc)) / (2.0 * rc) - erfOverR(beta, s);
}

// One table of the given power-of-two step: row k the degree-5 Chebyshev
// interpolant (6 nodes) on s in [k step - step/2, k step + step/2] written in
// powers of w = s - k step. Returns the largest deviation from phi_s at 32
// points per row between the nodes.
static double fitSlowTable(double beta, double rc, double step, int rows, std::vector<double>& out) {
  const int deg = kSlowTableDeg, nn = kSlowTableDeg + 1;
  const double half = 0.5 * step;
  out.assign((size_t)rows * kSlowTableRow, 0.0);
  // monomial coefficients of the Chebyshev polynomials T_0 .. T_deg
  double T[kSlowTableDeg + 1][kSlowTableDeg + 1] = {};
  T[0][0] = 1.0;
  T[1][1] = 1.0;
  for (int j = 2; j <= deg; ++j)
    for (int m = 0; m <= j; ++m) T[j][m] = (m > 0 ? 2.0 * T[j - 1][m - 1] : 0.0) - T[j - 2][m];
  double worst = 0.0;
  for (int k = 0; k < rows; ++k) {
    const double centre = step * k;
    double f[kSlowTableDeg + 1];
    for (int m = 0; m < nn; ++m) f[m] = slowPhi(beta, rc, centre + half * std::cos(M_PI * (m + 0.5) / nn));
    double* row = &out[(size_t)k * kSlowTableRow];
    double cu[kSlowTableDeg + 1] = {};  // powers of u = w / half
    for (int j = 0; j <= deg; ++j) {
      double cj = 0.0;
      for (int m = 0; m < nn; ++m) cj += f[m] * std::cos(j * M_PI * (m + 0.5) / nn);
      cj *= (j == 0 ? 1.0 : 2.0) / nn;
      for (int m = 0; m <= j; ++m) cu[m] += cj * T[j][m];
    }
    double scale = 1.0;
    for (int m = 0; m <= deg; ++m, scale /= half) row[m] = cu[m] * scale;
    for (int q = 0; q < 32; ++q) {
      const double w = half * (-1.0 + (q + 0.5) / 16.0);
      double p = row[deg];
      for (int m = deg - 1; m >= 0; --m) p = p * w + row[m];
      worst = std::fmax(worst, std::fabs(p - slowPhi(beta, rc, centre + w)));
    }
  }
  return worst;
}

// The slow-term table of the precise pass (layout in nbk_internal.cuh), over
// s in [0, pairlistdist^2 + 2]. The step starts at 32 A^2 and is halved
// (down to 1/128 of that) until the fit is within kSlowTableTol of
// max |phi_s| + 1/rc (the interpolation error of a row grows as
// (beta^2 step)^6). Returns the number of rows; *stepOut receives the step.
int buildSlowTable(double beta, double cutoff, double pairlistdist, std::vector<double>& out,
                   double* stepOut) {
  const double smax = pairlistdist * pairlistdist + 2.0;
  const double scale = std::fabs(slowPhi(beta, cutoff, 0.0)) + 1.0 / cutoff;
  double step = kSlowTableStepMax;
  int rows = 0;
  for (;;) {
    rows = (int)std::ceil(smax / step + 0.5) + 1;
    const double err = fitSlowTable(beta, cutoff, step, rows, out);
    if (err <= kSlowTableTol * scale || step <= kSlowTableStepMax / 128) break;
    step *= 0.5;
  }
  if (stepOut) *stepOut = step;
  return rows;
}

}  // namespace nbk

extern "C" NBK_API int nbk_slow_table(double ewaldcof, double cutoff, double pairlistdist,
                                      double* out, int maxRows, double* step) {
  if (!(cutoff > 0) || pairlistdist < cutoff || !(ewaldcof >= 0)) return NBK_ERR_ARG;
  std::vector<double> t;
  const int rows = nbk::buildSlowTable(ewaldcof, cutoff, pairlistdist, t, step);
  if (out) {
    if (maxRows < rows) return NBK_ERR_ARG;
    std::memcpy(out, t.data(), sizeof(double) * t.size());
  }
  return rows;
}
