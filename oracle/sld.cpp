// Oracle (test infrastructure only): tool-tip FRF helpers of src/frf.js (modeSet :6-11,
// frf :14-21, staticK :24, dominant :27, fitModes :125-144) and the zero-order
// (Altintas-Budak) lobes of src/sld.js (directionalCoeffs :6-15, stabilityLobes :23-61,
// alimAt :64-76), in the reference's operation order.
#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

#include "oracle.h"

namespace {

constexpr double kPi = 3.141592653589793;

struct C {
  double re, im;
};
inline C cmul(C a, C b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline C cdiv(C a, C b) {
  const double d = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
inline C csqrt(C a) {
  const double r = std::hypot(a.re, a.im);
  const double re = std::sqrt((r + a.re) / 2);
  // Math.sign(a[1] || 1): a zero (or NaN) imaginary part counts as positive
  const double s = (a.im != 0 && a.im == a.im) ? (a.im > 0 ? 1.0 : -1.0) : 1.0;
  const double im = s * std::sqrt(std::max(0.0, (r - a.re) / 2));
  return {re, im};
}

C frf_c(const mcs_mode* modes, int n, double f) {
  double re = 0, im = 0;
  for (int i = 0; i < n; i++) {
    const double r = f / modes[i].fn, a = 1 - r * r, b = 2 * modes[i].zeta * r,
                 d = modes[i].k * (a * a + b * b);
    re += a / d;
    im -= b / d;
  }
  return {re, im};
}

struct LobePt {
  double rpm, alim;
};

// stabilityLobes: returns the lobes as vectors of {rpm, alim}, sorted by rpm.
std::vector<std::vector<LobePt>> lobes_of(const mcs_lobe_query* q, const mcs_modal* modal) {
  double al[4];
  or_directional_coeffs(q->Krc / q->Ktc, q->phi_st, q->phi_ex, al);
  const double det = al[0] * al[3] - al[1] * al[2];
  const int nx = modal->nx, ny = modal->ny > 0 ? modal->ny : modal->nx;
  const mcs_mode* xm = modal->x;
  const mcs_mode* ym = modal->ny > 0 ? modal->y : modal->x;
  double fmin = INFINITY, fmax = -INFINITY;
  for (int j = 0; j < nx; j++) fmin = std::min(fmin, xm[j].fn), fmax = std::max(fmax, xm[j].fn);
  for (int j = 0; j < ny; j++) fmin = std::min(fmin, ym[j].fn), fmax = std::max(fmax, ym[j].fn);
  const double f0 = 0.8 * fmin, f1 = 1.7 * fmax;
  struct P {
    double wc, alim, psi;
  };
  std::vector<P> pts;
  const int NS = 400 * std::min(4, nx + ny - 1);
  for (int s = 0; s < NS; s++) {
    const double fc = f0 + (f1 - f0) * s / (NS - 1), wc = 2 * kPi * fc;
    const C Px = frf_c(xm, nx, fc), Py = frf_c(ym, ny, fc);
    const C a0 = cmul(cmul(Px, Py), {det, 0});
    const C a1 = {al[0] * Px.re + al[3] * Py.re, al[0] * Px.im + al[3] * Py.im};
    const C sq = cmul(a1, a1);
    const C disc = csqrt({sq.re - 4 * a0.re, sq.im - 4 * a0.im});
    bool have = false;
    double bestA = 0, bestK = 0;
    for (int sg = 1; sg >= -1; sg -= 2) {
      const C num = {-(a1.re + sg * disc.re), -(a1.im + sg * disc.im)};
      const C L = cdiv(num, {2 * a0.re, 2 * a0.im});
      if (L.re >= 0) continue;
      const double kap = L.im / L.re;
      const double alim = -2 * kPi * L.re * (1 + kap * kap) / (q->N * q->Ktc);
      if (alim > 0 && (!have || alim < bestA)) {
        have = true;
        bestA = alim;
        bestK = kap;
      }
    }
    if (have) pts.push_back({wc, bestA, std::atan(bestK)});
  }
  std::vector<std::vector<LobePt>> out;
  for (int j = 0; j < q->lobes; j++) {
    std::vector<LobePt> lobe;
    for (const P& p : pts) {
      const double eps = kPi - 2 * p.psi;
      const double T = (eps + 2 * j * kPi) / p.wc;
      const double rpm = 60 / (q->N * T);
      if (rpm >= q->rpm_min * 0.8 && rpm <= q->rpm_max * 1.2) lobe.push_back({rpm, p.alim});
    }
    std::stable_sort(lobe.begin(), lobe.end(),
                     [](const LobePt& a, const LobePt& b) { return a.rpm < b.rpm; });
    if (!lobe.empty()) out.push_back(std::move(lobe));
  }
  return out;
}

double alim_at(const std::vector<std::vector<LobePt>>& lobes, double rpm) {
  double best = INFINITY;
  for (const auto& lobe : lobes) {
    for (size_t i = 1; i < lobe.size(); i++) {
      const LobePt& a = lobe[i - 1];
      const LobePt& b = lobe[i];
      if (rpm >= a.rpm && rpm <= b.rpm) {
        const double span = b.rpm - a.rpm;
        const double t = (rpm - a.rpm) / (span != 0 ? span : 1);
        best = std::min(best, a.alim + (b.alim - a.alim) * t);
      }
    }
  }
  return best;
}

}  // namespace

extern "C" {

void or_frf(const mcs_mode* modes, int n, double f, double out[2]) {
  const C g = frf_c(modes, n, f);
  out[0] = g.re;
  out[1] = g.im;
}

double or_static_k(const mcs_mode* modes, int n) {
  double s = 0;
  for (int i = 0; i < n; i++) s += 1 / modes[i].k;
  return 1 / s;
}

int or_dominant(const mcs_mode* modes, int n) {
  int a = 0;
  for (int i = 1; i < n; i++)
    if (modes[i].k * modes[i].zeta < modes[a].k * modes[a].zeta) a = i;
  return a;
}

void or_directional_coeffs(double Kr, double phiSt, double phiEx, double out[4]) {
  auto F = [Kr](double p, double f[4]) {
    f[0] = 0.5 * (std::cos(2 * p) - 2 * Kr * p + Kr * std::sin(2 * p));
    f[1] = 0.5 * (-std::sin(2 * p) - 2 * p + Kr * std::cos(2 * p));
    f[2] = 0.5 * (-std::sin(2 * p) + 2 * p + Kr * std::cos(2 * p));
    f[3] = 0.5 * (-std::cos(2 * p) - 2 * Kr * p - Kr * std::sin(2 * p));
  };
  double a[4], b[4];
  F(phiEx, a);
  F(phiSt, b);
  for (int i = 0; i < 4; i++) out[i] = a[i] - b[i];
}

int or_stability_lobes(const mcs_lobe_query* q, const mcs_modal* modal, double* rpm,
                       double* alim, int32_t* lobe_len, int cap) {
  const auto lobes = lobes_of(q, modal);
  int pos = 0;
  for (size_t j = 0; j < lobes.size(); j++) {
    if (pos + (int)lobes[j].size() > cap) return -1;
    lobe_len[j] = (int32_t)lobes[j].size();
    for (const LobePt& p : lobes[j]) {
      rpm[pos] = p.rpm;
      alim[pos] = p.alim;
      pos++;
    }
  }
  return (int)lobes.size();
}

double or_alim_at(int n_lobes, const int32_t* lobe_len, const double* rpm, const double* alim,
                  double at_rpm) {
  std::vector<std::vector<LobePt>> lobes(n_lobes);
  int pos = 0;
  for (int j = 0; j < n_lobes; j++)
    for (int i = 0; i < lobe_len[j]; i++, pos++) lobes[j].push_back({rpm[pos], alim[pos]});
  return alim_at(lobes, at_rpm);
}

void or_lobes_alim(const mcs_modal* modals, const mcs_lobe_query* queries, size_t n_queries,
                   const double* rpm, size_t n_rpm, double* out) {
  for (size_t q = 0; q < n_queries; q++) {
    const auto lobes = lobes_of(&queries[q], &modals[queries[q].modal]);
    for (size_t r = 0; r < n_rpm; r++) out[q * n_rpm + r] = alim_at(lobes, rpm[r]);
  }
}

int or_fit_modes(const double* f, const double* re, const double* im, int n, int max_modes,
                 mcs_mode* out) {
  (void)re;
  // peak picking on -Im G: half-power width -> zeta, peak height 1/(2 k zeta) -> k
  std::vector<double> q(n);
  for (int i = 0; i < n; i++) q[i] = -im[i];
  double top = -INFINITY;
  for (int i = 0; i < n; i++) top = std::max(top, q[i]);
  std::vector<int> peaks;
  for (int i = 1; i < n - 1; i++)
    if (q[i] > 0.05 * top && q[i] >= q[i - 1] && q[i] > q[i + 1]) peaks.push_back(i);
  struct M {
    double k, fn, zeta, peak;
  };
  std::vector<M> modes;
  for (int i : peaks) {
    const double half = q[i] / 2;
    int a = i, b = i;
    while (a > 0 && q[a] > half) a--;
    while (b < n - 1 && q[b] > half) b++;
    const double da = q[a + 1] - q[a], db = q[b - 1] - q[b];
    const double fa = a == i ? f[i] : f[a] + (half - q[a]) / (da != 0 ? da : 1) * (f[a + 1] - f[a]);
    const double fb =
        b == i ? f[i] : f[b - 1] + (q[b - 1] - half) / (db != 0 ? db : 1) * (f[b] - f[b - 1]);
    const double fn = f[i], zeta = std::min(0.3, std::max(0.003, (fb - fa) / (2 * fn)));
    modes.push_back({1 / (2 * zeta * q[i]), fn, zeta, q[i]});
  }
  std::stable_sort(modes.begin(), modes.end(), [](const M& a, const M& b) { return b.peak < a.peak; });
  if ((int)modes.size() > max_modes) modes.resize(max_modes);
  std::stable_sort(modes.begin(), modes.end(), [](const M& a, const M& b) { return a.fn < b.fn; });
  for (size_t i = 0; i < modes.size(); i++) out[i] = {modes[i].k, modes[i].fn, modes[i].zeta};
  return (int)modes.size();
}

}  // extern "C"
