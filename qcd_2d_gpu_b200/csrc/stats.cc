// Host statistics of measurement series.
//
// qcd_stats_mean_variance / qcd_stats_autocorrelation restate the reference's
// naive estimators (statistics.h:30-51), so a driver reproduces its printed
// numbers and files; qcd_stats_binned and qcd_stats_tau_int add the binned
// error and the integrated autocorrelation time with Madras-Sokal automatic
// windowing (A. Sokal, "Monte Carlo methods in statistical mechanics", 1996),
// which the reference leaves to post-processing of its Check_ files.
#include <math.h>
#include <stdlib.h>

#include "qcd2d.h"

extern "C" {

int qcd_stats_mean_variance(const double* x, int n, double* mean, double* var) {
  if (!x || n < 1 || !mean || !var) return QCD_ERR_INVALID;
  double s = 0, s2 = 0;
  for (int i = 0; i < n; i++) {
    s += x[i];
    s2 += x[i] * x[i];
  }
  *mean = s / n;
  *var = s2 / n - *mean * *mean;  // population variance, as statistics.h:36
  return QCD_OK;
}

int qcd_stats_autocorrelation(const double* x, int n, int w, double mean, double var, double* out) {
  if (!x || !out || n < 2 || w < 1 || w >= n) return QCD_ERR_INVALID;
  for (int lag = 1; lag <= w; lag++) {
    double s = 0;
    for (int j = 0; j < n - lag; j++) s += (x[j] - mean) * (x[j + lag] - mean);
    out[lag - 1] = s / (n - lag) / var;
  }
  return QCD_OK;
}

int qcd_stats_binned(const double* x, int n, int bin, double* mean, double* err) {
  if (!x || !mean || !err || bin < 1 || n / bin < 2) return QCD_ERR_INVALID;
  const int nb = n / bin;
  double s = 0, s2 = 0;
  for (int b = 0; b < nb; b++) {
    double m = 0;
    for (int i = 0; i < bin; i++) m += x[b * bin + i];
    m /= bin;
    s += m;
    s2 += m * m;
  }
  *mean = s / nb;
  const double v = (s2 / nb - *mean * *mean) * nb / (nb - 1);  // sample variance of the bin means
  *err = sqrt(v > 0 ? v / nb : 0);
  return QCD_OK;
}

int qcd_stats_tau_int(const double* x, int n, double c, double* tau, int* window, double* dtau) {
  if (!x || !tau || n < 4 || !(c > 0)) return QCD_ERR_INVALID;
  double m = 0;
  for (int i = 0; i < n; i++) m += x[i];
  m /= n;
  double c0 = 0;
  for (int i = 0; i < n; i++) c0 += (x[i] - m) * (x[i] - m);
  c0 /= n;
  double t = 0.5;
  int W = 0;
  if (c0 > 0) {
    for (W = 1; W < n / 2; W++) {
      double cw = 0;
      for (int i = 0; i < n - W; i++) cw += (x[i] - m) * (x[i + W] - m);
      cw /= (n - W);
      t += cw / c0;
      if (W >= c * t) break;  // window W >= c tau_int(W)
    }
  }
  *tau = t;
  if (window) *window = W;
  if (dtau) *dtau = t * sqrt((4.0 * W + 2.0) / n);  // Madras-Sokal error estimate
  return QCD_OK;
}

}  // extern "C"
