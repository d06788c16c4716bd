// Imaginary-frequency quadrature for the RPA energy (host code).
//
// Transformed ("Casimir-Polder") Gauss-Legendre grid on (0, inf):
//   u_k = a (1 + t_k)/(1 - t_k),  w_k = 2 a w_GL,k / (1 - t_k)^2,
// with the scale a chosen by a scan over [0.1, 15] (15000 points) minimising
// the RMSD of sum_k w_k/(D^2+u_k^2) against pi/(2D) over a 100-bin histogram
// of the orbital-energy differences D, and n the smallest point count in
// [8, 64] meeting the RMSD and max-relative-error targets.  Restates
// rpa_OptimizeFreqQuad / rpa_OptQuadScaling / rpa_FreqQuadError
// (src/rpa/OptFreqQuad.f90:12-169), quad_CasimirPolder
// (src/rpa/quadratures.f90:570-643) and rpa_DaiHistogram / rpa_NCore
// (src/rpa/OrbDiffHist.f90:42-146).  The Gauss-Legendre nodes come from a
// Newton iteration on theta = arccos(t) with the three-term Legendre
// recurrence (as quad_GaussLegendre, quadratures.f90:418-509, does).
#include <cmath>
#include <initializer_list>
#include <vector>

#include "../../include/rpa_b200.h"
#include "abi_guard.h"
#include "rpa_common.cuh"

namespace {

const double kPiG = 3.14159265358979323846;

void legendre(int n, double x, double& pn, double& pn1) {
  double pb = 0.0, pa = 1.0;
  for (int a = 1; a <= n; ++a) {
    const double pc = pb;
    pb = pa;
    pa = (2.0 * a - 1.0) / a * x * pb - (a - 1.0) / a * pc;
  }
  pn = pa;
  pn1 = pb;
}

// All n nodes (ascending) and weights of Gauss-Legendre on (-1, 1).
bool gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  bool ok = true;
  for (int k = 1; k <= n; ++k) {
    double th = kPiG * (k - 0.25) / (n + 0.5);
    bool conv = false;
    for (int it = 0; it < 100; ++it) {
      const double c = std::cos(th);
      double pn, pn1;
      legendre(n, c, pn, pn1);
      const double dth = n * (c * pn - pn1) / std::sin(th);
      const double nt = th - pn / dth;
      const bool done = std::fabs(nt - th) < 1.0e-14;
      th = nt;
      if (done) {
        conv = true;
        break;
      }
    }
    ok = ok && conv;
    const double c = std::cos(th);
    double pn, pn1;
    legendre(n, c, pn, pn1);
    const double dth = n * (c * pn - pn1) / std::sin(th);
    x[n - k] = c;  // cos is decreasing in theta: store ascending
    w[n - k] = 2.0 / (dth * dth);
  }
  return ok;
}

struct Hist {
  std::vector<double> d, wt;
};

int64_t ncore(const double* e, int64_t nocc, double core_thresh) {
  int64_t nc = 0;
  for (int64_t k = 0; k < nocc; ++k) {
    if (e[k] < core_thresh) ++nc;
    else break;
  }
  return nc;
}

// Largest active excitation energy e_a1 - e_i0 (rpa_DaiMaxThresh, OrbDiffHist.f90:10-39); 0 when
// every occupied orbital is frozen.
double dai_max(const double* e, int64_t nocc, int64_t nvirt, double core_thresh) {
  const int64_t nc = ncore(e, nocc, core_thresh);
  return nc < nocc ? e[nocc + nvirt - 1] - e[nc] : 0.0;
}

// rpa_DaiHistogram (OrbDiffHist.f90:42-123): bins of the active differences d <= thresh.
// Returns 1 for a histogram, 0 when every occupied orbital is frozen (the set then takes no part
// in the error estimate), -1 for a non-positive gap.
int histogram(const double* e, int64_t nocc, int64_t nvirt, double core_thresh, int nbins, double thresh, Hist& h) {
  const int64_t nc = ncore(e, nocc, core_thresh);
  if (nc >= nocc) return 0;
  const int64_t i0 = nc, i1 = nocc - 1, a0 = nocc, a1 = nocc + nvirt - 1;
  const double dmin = e[a0] - e[i1];
  const double dmax = std::fmin(thresh, e[a1] - e[i0]);
  if (!(dmin > 0.0)) return -1;
  const double width = (dmax - dmin) / nbins;
  h.d.resize(nbins);
  h.wt.assign(nbins, 0.0);
  for (int k = 0; k < nbins; ++k) h.d[k] = dmin + k * width;
  std::vector<int64_t> cnt(nbins, 0);
  int64_t total = 0;
  for (int64_t i = i0; i <= i1; ++i)
    for (int64_t a = a0; a <= a1; ++a) {
      const double d = e[a] - e[i];
      if (!(d <= thresh)) continue;
      const double x = (d - (dmin + width / 2.0)) / width;
      // 1 + nint(x) (Fortran nint), clamped to [1, nbins] before the conversion to an integer: with
      // a single distinct difference the width is 0 and x is 0/0, which lands in bin 1 (gfortran's
      // nint of a NaN is the most negative integer, which the reference's max(1, k) clamps to 1)
      double kf = 1.0 + (x >= 0 ? std::floor(x + 0.5) : -std::floor(-x + 0.5));
      if (!(kf >= 1.0)) kf = 1.0;
      if (kf > nbins) kf = nbins;
      ++cnt[(int)kf - 1];
      ++total;
    }
  for (int k = 0; k < nbins; ++k) h.wt[k] = std::fabs((double)cnt[k] / (double)total);
  return 1;
}

// rpa_FreqQuadError (OptFreqQuad.f90:125-169) over several histograms: the RMSD is the root of the
// largest per-set mean square error, the relative error the largest over all sets.
void quad_error(const std::vector<double>& u, const std::vector<double>& w, const std::vector<Hist>& hs,
                double& rel, double& rmsd) {
  rel = 0.0;
  double err2max = 0.0;
  for (const Hist& h : hs) {
    double err2 = 0.0;
    for (size_t l = 0; l < h.d.size(); ++l) {
      if (!(h.wt[l] > 0.0)) continue;
      const double d = h.d[l];
      const double exact = kPiG / (2.0 * d);
      double approx = 0.0;
      for (size_t k = 0; k < u.size(); ++k) approx += w[k] / (d * d + u[k] * u[k]);
      rel = std::fmax(rel, std::fabs((approx - exact) / exact));
      err2 += h.wt[l] * (approx - exact) * (approx - exact);
    }
    err2max = std::fmax(err2max, err2);
  }
  rmsd = std::sqrt(err2max);
}

bool opt_scaling(int n, const std::vector<Hist>& h, std::vector<double>& u, std::vector<double>& w, double& rel,
                 double& rmsd) {
  std::vector<double> t, wgl;
  if (!gauss_legendre(n, t, wgl)) return false;
  std::vector<double> u0(n), w0(n);
  for (int k = 0; k < n; ++k) {
    u0[k] = (1.0 + t[k]) / (1.0 - t[k]);
    w0[k] = 2.0 * wgl[k] / ((1.0 - t[k]) * (1.0 - t[k]));
  }
  const double amin = 0.1, amax = 15.0;
  const int nscan = 15000;
  double best = HUGE_VAL, best_rel = 0.0, best_a = 0.0;
  std::vector<double> uu(n), ww(n);
  for (int k = 0; k < nscan; ++k) {
    const double a = amin + (amax - amin) * (double)k / (double)(nscan - 1);
    for (int j = 0; j < n; ++j) {
      uu[j] = a * u0[j];
      ww[j] = a * w0[j];
    }
    double r, e;
    quad_error(uu, ww, h, r, e);
    if (e < best) {
      best = e;
      best_rel = r;
      best_a = a;
    }
  }
  u.resize(n);
  w.resize(n);
  for (int j = 0; j < n; ++j) {
    u[j] = best_a * u0[j];
    w[j] = best_a * w0[j];
  }
  rel = best_rel;
  rmsd = best;
  return true;
}

// The grid for the histograms hs (at least one non-empty).
int grid_from_histograms(const std::vector<Hist>& hs, double TargetError, double TargetRelError, int64_t NFixed,
                         double* Freqs, double* FreqWeights, int64_t* NFreqs) {
  std::vector<double> u, w;
  double rel = 0.0, rmsd = 0.0;
  int n = 0;
  if (NFixed > 0) {
    n = (int)NFixed;
    if (!opt_scaling(n, hs, u, w, rel, rmsd)) return RPA_ERR_NOT_CONVERGED;
  } else {
    bool conv = false;
    for (n = 8; n <= 64; ++n) {
      if (!opt_scaling(n, hs, u, w, rel, rmsd)) return RPA_ERR_NOT_CONVERGED;
      if (rmsd < TargetError && rel < TargetRelError) {
        conv = true;
        break;
      }
    }
    if (!conv) return RPA_ERR_NOT_CONVERGED;
  }
  for (int k = 0; k < n; ++k) {
    Freqs[k] = u[k];
    FreqWeights[k] = w[k];
  }
  *NFreqs = n;
  return RPA_OK;
}

}  // namespace

extern "C" int rpa_b200_freq_grid(int64_t NOcc, int64_t NVirt, const double* OrbEnergies, double CoreOrbThresh,
                                  double TargetError, double TargetRelError, int64_t NFixed, double* Freqs,
                                  double* FreqWeights, int64_t* NFreqs) try {
  if (NOcc < 1 || NVirt < 1 || !OrbEnergies || !Freqs || !FreqWeights || !NFreqs) return RPA_ERR_INVALID_ARG;
  if (NFixed < 0 || NFixed > 64) return RPA_ERR_INVALID_ARG;
  for (int64_t k = 0; k < NOcc + NVirt; ++k)
    if (!std::isfinite(OrbEnergies[k])) return RPA_ERR_NONFINITE;
  std::vector<Hist> hs(1);
  if (histogram(OrbEnergies, NOcc, NVirt, CoreOrbThresh, 100, HUGE_VAL, hs[0]) != 1) return RPA_ERR_INVALID_ARG;
  return grid_from_histograms(hs, TargetError, TargetRelError, NFixed, Freqs, FreqWeights, NFreqs);
} catch (...) {
  return rpa::status_of_exception(nullptr);
}

// One grid shared by the subsystems of a many-body expansion (rpa_PostSCF,
// src/rpa/rpa_driver.f90:118-175): a histogram per subsystem and spin, optionally capped at the
// largest excitation energy of set 0 (the whole complex, GridLimitDai), and the errors of the
// optimiser taken as the worst over the sets.
extern "C" int rpa_b200_freq_grid_mbe(int64_t NSets, const int64_t* NOcc, const int64_t* NVirt,
                                      const double* const* OrbEnergies, double CoreOrbThresh, int64_t LimitDai,
                                      double TargetError, double TargetRelError, int64_t NFixed, double* Freqs,
                                      double* FreqWeights, int64_t* NFreqs) try {
  if (NSets < 1 || NSets > 4096 || !NOcc || !NVirt || !OrbEnergies || !Freqs || !FreqWeights || !NFreqs)
    return RPA_ERR_INVALID_ARG;
  if (NFixed < 0 || NFixed > 64) return RPA_ERR_INVALID_ARG;
  for (int64_t s = 0; s < NSets; ++s) {
    if (NOcc[s] < 1 || NVirt[s] < 1 || !OrbEnergies[s]) return RPA_ERR_INVALID_ARG;
    for (int64_t k = 0; k < NOcc[s] + NVirt[s]; ++k)
      if (!std::isfinite(OrbEnergies[s][k])) return RPA_ERR_NONFINITE;
  }
  const double thresh = LimitDai ? dai_max(OrbEnergies[0], NOcc[0], NVirt[0], CoreOrbThresh) : HUGE_VAL;
  std::vector<Hist> hs;
  for (int64_t s = 0; s < NSets; ++s) {
    Hist h;
    const int r = histogram(OrbEnergies[s], NOcc[s], NVirt[s], CoreOrbThresh, 100, thresh, h);
    if (r < 0) return RPA_ERR_INVALID_ARG;
    if (r > 0) hs.push_back(std::move(h));
  }
  if (hs.empty()) return RPA_ERR_INVALID_ARG;
  return grid_from_histograms(hs, TargetError, TargetRelError, NFixed, Freqs, FreqWeights, NFreqs);
} catch (...) {
  return rpa::status_of_exception(nullptr);
}

// ------------------------------------------------------------------ many-body-expansion energies
// rpa_Eint2Body / rpa_EintNadd / rpa_EintNadd4Body (src/rpa/rpa_driver.f90:381-433): each group
// difference in FP64, left to right, as the reference evaluates it; the combination of the groups
// (REAL(16) there) in double-double.
extern "C" int rpa_b200_mbe_energy(int64_t NBody, const double* E, double* Eint) try {
  if (!E || !Eint || NBody < 2 || NBody > 4) return RPA_ERR_INVALID_ARG;
  const double* e = E;
  if (NBody == 2) {
    *Eint = e[0] - e[1] - e[2];
    return RPA_OK;
  }
  auto comb = [](std::initializer_list<double> terms) {
    rpa::dd acc{0.0, 0.0};
    for (double t : terms) acc = rpa::dd_add(acc, t);
    return acc.hi + acc.lo;
  };
  // subsystem energies (0-based reference order)
  const double tot = e[0], A = e[1], B = e[2], C = e[3], AB = e[4], BC = e[5], AC = e[6];
  if (NBody == 3) {
    const double eabc = tot - A - B - C;
    const double eab = AB - A - B, ebc = BC - B - C, eac = AC - A - C;
    *Eint = comb({eabc, -eab, -ebc, -eac});
    return RPA_OK;
  }
  const double D = e[7], AD = e[8], BD = e[9], CD = e[10];
  const double ABC = e[11], ABD = e[12], ACD = e[13], BCD = e[14];
  const double eabcd = tot - A - B - C - D;
  const double eabc = ABC - A - B - C, eabd = ABD - A - B - D, eacd = ACD - A - C - D, ebcd = BCD - B - C - D;
  const double eab = AB - A - B, ebc = BC - B - C, eac = AC - A - C;
  const double ead = AD - A - D, ebd = BD - B - D, ecd = CD - C - D;
  // the reference forms the four three-body nonadditive terms in REAL(16), then subtracts them
  // Eabcd - sum of pair terms - the four three-body nonadditive terms (Eabc - Eab - Ebc - Eac,
  // ...), REAL(16) throughout in the reference: expanded here into one double-double sum so that
  // no intermediate is rounded to FP64
  *Eint = comb({eabcd, -eab, -ebc, -eac, -ead, -ebd, -ecd,
                -eabc, eab, ebc, eac, -eabd, eab, ead, ebd,
                -eacd, eac, ead, ecd, -ebcd, ebc, ebd, ecd});
  return RPA_OK;
} catch (...) {
  return rpa::status_of_exception(nullptr);
}

