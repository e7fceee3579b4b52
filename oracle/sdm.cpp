// Oracle (test infrastructure only): the zeroth-order semi-discretisation of
// test/lib/sdm.mjs:6-66 (Insperger & Stepan) -- a second, independent stability
// reference for the 1-DOF milling benchmark of test/validation.test.mjs.
#include <algorithm>
#include <cmath>
#include <vector>

#include "oracle.h"

namespace {

constexpr double kPi = 3.141592653589793;
using Mat = std::vector<std::vector<double>>;

// C = A B with the reference's loop order (i, k, j) and its skip of zero factors
Mat mul(const Mat& A, const Mat& B) {
  const size_t n = A.size(), m = B[0].size(), p = B.size();
  Mat C(n, std::vector<double>(m, 0.0));
  for (size_t i = 0; i < n; i++)
    for (size_t k = 0; k < p; k++) {
      const double a = A[i][k];
      if (a != 0)
        for (size_t j = 0; j < m; j++) C[i][j] += a * B[k][j];
    }
  return C;
}

// matrix exponential by scaling and squaring with an 18-term Taylor series (:6-15)
Mat expm(const Mat& M) {
  const size_t n = M.size();
  double norm = 0;
  for (const auto& r : M) {
    double s = 0;
    for (double v : r) s += std::fabs(v);
    norm = std::max(norm, s);
  }
  const int sq = (int)std::max(0.0, std::ceil(std::log2(norm + 1e-300)) + 1);
  const double scale = std::pow(2.0, sq);
  Mat A = M;
  for (auto& r : A)
    for (auto& v : r) v = v / scale;
  Mat E(n, std::vector<double>(n, 0.0));
  for (size_t i = 0; i < n; i++) E[i][i] = 1;
  Mat term = E;
  for (int k = 1; k <= 18; k++) {
    term = mul(term, A);
    for (auto& r : term)
      for (auto& v : r) v = v / k;
    for (size_t i = 0; i < n; i++)
      for (size_t j = 0; j < n; j++) E[i][j] = E[i][j] + term[i][j];
  }
  for (int s = 0; s < sq; s++) E = mul(E, E);
  return E;
}

}  // namespace

extern "C" {

double or_sdm_rho(const or_sdm_params* p, double a) {
  const int steps = p->steps > 0 ? p->steps : 40;
  const double wn = std::sqrt(p->k / p->m), T = 60 / (p->rpm * p->N), dt = T / steps,
               Om = p->rpm * 2 * kPi / 60;
  const size_t n = steps + 2;
  Mat Phi(n, std::vector<double>(n, 0.0));
  for (size_t i = 0; i < n; i++) Phi[i][i] = 1;
  for (int i = 0; i < steps; i++) {
    // average specific force over the step
    double h = 0;
    const int sub = 8;
    for (int s = 0; s < sub; s++) {
      const double t = (i + (s + 0.5) / sub) * dt;
      for (int j = 0; j < p->N; j++) {
        const double phi =
            std::fmod(std::fmod(Om * t + 2 * kPi * j / p->N, 2 * kPi) + 2 * kPi, 2 * kPi);
        if (phi >= p->phi_st && phi <= p->phi_ex)
          h += std::sin(phi) * (p->Kt * std::cos(phi) + p->Kn * std::sin(phi));
      }
    }
    h /= sub;
    const double w = a * h / p->m;
    const Mat E = expm({{0, dt, 0},
                        {(-wn * wn - w) * dt, -2 * p->zeta * wn * dt, w * dt},
                        {0, 0, 0}});
    Mat G(n, std::vector<double>(n, 0.0));
    G[0][0] = E[0][0];
    G[0][1] = E[0][1];
    G[1][0] = E[1][0];
    G[1][1] = E[1][1];
    // delayed position: mean of the two samples bracketing t - T
    G[0][n - 2] += E[0][2] / 2;
    G[0][n - 1] += E[0][2] / 2;
    G[1][n - 2] += E[1][2] / 2;
    G[1][n - 1] += E[1][2] / 2;
    G[2][0] = 1;
    for (size_t r = 3; r < n; r++) G[r][r - 1] = 1;
    Phi = mul(G, Phi);
  }
  // spectral radius by repeated squaring with normalisation (Gelfand)
  double logScale = 0;
  Mat M = Phi;
  const int K = 9;
  for (int s = 0; s < K; s++) {
    M = mul(M, M);
    logScale *= 2;
    double nm = 0;
    for (const auto& r : M)
      for (double v : r) nm = std::max(nm, std::fabs(v));
    for (auto& r : M)
      for (auto& v : r) v = v / nm;
    logScale += std::log(nm);
  }
  return std::exp(logScale / std::pow(2.0, K));
}

double or_sdm_limit(const or_sdm_params* p, double a_max) {
  double lo = 0, hi = a_max > 0 ? a_max : 0.02;
  if (or_sdm_rho(p, hi) < 1) return INFINITY;
  for (int it = 0; it < 30; it++) {
    const double mid = (lo + hi) / 2;
    if (or_sdm_rho(p, mid) < 1)
      lo = mid;
    else
      hi = mid;
  }
  return (lo + hi) / 2;
}

}  // extern "C"
