// Integrated autocorrelation time estimators with the reference's entry
// points (reference src/actime.cpp:19-145,189-246), written from the
// published method: U. Wolff, "Monte Carlo errors with less errors",
// Comput. Phys. Commun. 156 (2004) 143 (hep-lat/0306017), automatic
// windowing with S = 1.5, and a plain summed-autocorrelation window.
#include <cmath>
#include <iostream>
#include <vector>

#include "actime.h"

namespace U1 {

namespace {
double mean_of(const std::vector<double> &x, size_t n) {
  double m = 0.0;
  for (size_t i = 0; i < n; ++i) m += x[i];
  return m / (double)n;
}
}  // namespace

void calculateCorTime(int miniter, int iter, std::vector<double> &series, int &nsweep) {
  (void)iter;
  (void)nsweep;
  if ((int)series.size() < miniter) return;
  const size_t N = series.size();
  const double avg = mean_of(series, N);
  const double S = 1.5;
  std::vector<double> G;  // autocovariance Gamma(t)
  size_t tmax = N / 2, W = 0;
  double sum_rho = 0.0, tauW = 0.0, gW = 0.0;
  bool found = false;
  for (size_t t = 0; t <= tmax; ++t) {
    double g = 0.0;
    for (size_t i = 0; i + t < N; ++i) g += (series[i] - avg) * (series[i + t] - avg);
    g /= (double)(N - t);
    G.push_back(g);
    if (t == 0 || found) continue;
    // tau_int(W) - 1/2 = sum_{t=1}^{W} rho(t); tau(W) = S / ln((2 tau+1)/(2 tau-1))
    sum_rho += g / G[0];
    tauW = (sum_rho <= 0.0) ? 2.2204e-16 : S / std::log((sum_rho + 1.0) / sum_rho);
    gW = std::exp(-(double)t / tauW) - tauW / std::sqrt((double)t * (double)N);
    if (gW < 0.0) {  // first W where the statistical error outweighs the bias
      W = t;
      tmax = std::min(tmax, 2 * t);
      found = true;
    }
  }
  std::cout << "N: " << N << "\tGint: " << sum_rho << "\ttauw: " << tauW << "\tgW: " << gW << "\tWopt: " << W
            << "\ttmax: " << tmax << std::endl;
  if (!found) {
    std::cout << "WARNING: windowing condition failed up to W = " << tmax << std::endl;
    return;
  }
  double C = G[0];
  for (size_t t = 1; t <= W; ++t) C += 2.0 * G[t];
  std::cout << "CFbbopt: " << C << "\t(first estimate)" << std::endl;
  for (double &g : G) g += C / (double)N;  // bias correction of Gamma
  C = G[0];
  for (size_t t = 1; t <= W; ++t) C += 2.0 * G[t];
  std::cout << "CFbbopt: " << C << "\t(refined estimate)" << std::endl;
  const double sigma = std::sqrt(C / (double)N);
  double tauint = 0.5;
  for (size_t t = 1; t <= W; ++t) tauint += G[t] / G[0];
  std::cout << "value: " << avg << std::endl;
  std::cout << "dvalue: " << sigma << std::endl;
  std::cout << "ddvalue: " << sigma * std::sqrt(((double)W + 0.5) / (double)N) << std::endl;
  std::cout << "tauint: " << tauint << std::endl;
  std::cout << "dtauint: " << tauint * 2.0 * std::sqrt(((double)W - tauint + 0.5) / (double)N) << std::endl;
  std::cout << "Wopt: " << W << std::endl;
}

void calculateCorTime1(int miniter, int iter, std::vector<double> &series, int &nsweep) {
  if ((int)series.size() < miniter) return;
  const size_t N = series.size() / 2;
  if (N < 2) return;
  std::vector<double> rho(N, 0.0);
  double g0 = 0.0;
  for (size_t j = 0; j < N; ++j) {
    // window means over the overlapping segments [0, N-j) and [j, N)
    double a = 0.0, b = 0.0;
    for (size_t i = 0; i + j < N; ++i) {
      a += series[i];
      b += series[i + j];
    }
    a /= (double)(N - j);
    b /= (double)(N - j);
    double g = 0.0;
    for (size_t i = 0; i + j < N; ++i) g += (series[i] - a) * (series[i + j] - b);
    g /= (double)(N - j);
    if (j == 0) g0 = g;
    rho[j] = g / g0;
  }
  double tau = 0.5;
  for (size_t i = 1; i < N; ++i) {
    tau += rho[i - 1];
    const int window = (int)(4.0 * tau + 1.0);
    if ((int)i > window) {
      nsweep = (int)i;
      std::cout << "iter: " << iter << "\tN: " << N << "\tsweeps: " << nsweep << "\ttau_int: " << tau
                << "\tint(4.*tau_int+1): " << window << std::endl;
      break;
    }
  }
}

}  // namespace U1
