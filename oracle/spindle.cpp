// Oracle (test infrastructure only): the speed-dependent tool-tip modes of src/spindle.js,
// restated step by step with list-valued mode sets as the JavaScript keeps them.
//   bearingFactor  src/spindle.js:18-23
//   tipFactor      src/spindle.js:26-30
//   twoDofModes    src/spindle.js:38-53
//   scaleModes     src/spindle.js:55
//   lerpModes      src/spindle.js:57-60
//   modesAt        src/spindle.js:64-85
#include <algorithm>
#include <cmath>
#include <vector>

#include "oracle.h"

namespace {

constexpr double kPi = 3.141592653589793;

struct Soft {
  double drop, Sref;
};
using Modes = std::vector<mcs_mode>;

double bearingFactor(double S, const Soft& soft) {
  const double d = std::min(0.9, std::max(0.0, soft.drop));
  if (!(d != 0) || !(S > 0)) return 1;
  const double c = d / (1 - d);
  return 1 / (1 + c * std::pow(S / (soft.Sref != 0 ? soft.Sref : 30000), 2));
}

double tipFactor(double S, double kTool, double kSp, const Soft& soft) {
  const double b = bearingFactor(S, soft);
  if (b == 1 || !(kTool > 0) || !(kSp > 0)) return 1;
  return (1 / kTool + 1 / kSp) / (1 / kTool + 1 / (kSp * b));
}

Modes twoDofModes(double kTool, double mTool, double kSp, double mSp, double zTool, double zSp) {
  const double k1 = kSp * 1e3, k2 = kTool * 1e3, m1 = mSp, m2 = mTool;
  const double a = m1 * m2, b = -((k1 + k2) * m2 + k2 * m1), c = k1 * k2;
  const double disc = std::sqrt(std::max(0.0, b * b - 4 * a * c));
  Modes out;
  for (double w2 : {(-b - disc) / (2 * a), (-b + disc) / (2 * a)}) {
    const double phiT = (k1 + k2 - w2 * m1) / k2;
    const double mr = m1 + m2 * phiT * phiT;
    out.push_back({mr * w2 / (phiT * phiT) / 1e3, std::sqrt(w2) / (2 * kPi),
                   m2 * phiT * phiT > m1 ? zTool : zSp});
  }
  return out;
}

Modes scaleModes(const Modes& modes, double f) {
  Modes out;
  for (const mcs_mode& m : modes) out.push_back({m.k * f, m.fn * std::sqrt(f), m.zeta});
  return out;
}

Modes lerpModes(const Modes& a, const Modes& b, double t) {
  if (a.size() != b.size()) return t < 0.5 ? a : b;
  Modes out;
  for (size_t i = 0; i < a.size(); i++)
    out.push_back({a[i].k + (b[i].k - a[i].k) * t, a[i].fn + (b[i].fn - a[i].fn) * t,
                   a[i].zeta + (b[i].zeta - a[i].zeta) * t});
  return out;
}

Modes list(const mcs_mode* m, int n) { return Modes(m, m + n); }

}  // namespace

extern "C" void or_modes_at(const mcs_spindle* sp, const mcs_speed_frf* frfs, size_t n_frfs,
                            const double* Sv, size_t n, mcs_modal* out) {
  const Soft soft{sp->drop, sp->s_ref};
  struct Entry {
    double S;
    Modes x, y;
  };
  std::vector<Entry> L;
  for (size_t i = 0; i < n_frfs; i++) {
    const mcs_modal& m = frfs[i].modes;
    L.push_back({frfs[i].S, list(m.x, m.nx), list(m.y, m.ny)});
  }
  std::stable_sort(L.begin(), L.end(), [](const Entry& p, const Entry& q) { return p.S < q.S; });
  for (size_t i = 0; i < n; i++) {
    const double S = Sv[i];
    Modes x, y;
    if (!L.empty()) {
      // pick = e => ({ x: e.modesX, y: e.modesY?.length ? e.modesY : e.modesX })
      auto px = [](const Entry& e) { return e.x; };
      auto py = [](const Entry& e) { return e.y.empty() ? e.x : e.y; };
      if (S <= L[0].S) {
        x = px(L[0]);
        y = py(L[0]);
      } else if (S >= L.back().S) {
        x = px(L.back());
        y = py(L.back());
      } else {
        size_t j = 1;
        while (L[j].S < S) j++;
        const double t = (S - L[j - 1].S) / (L[j].S - L[j - 1].S);
        x = lerpModes(px(L[j - 1]), px(L[j]), t);
        y = lerpModes(py(L[j - 1]), py(L[j]), t);
      }
    } else if (sp->two_dof) {
      x = y = twoDofModes(sp->k_tool, sp->m_tool, sp->k_sp * bearingFactor(S, soft), sp->m_sp,
                          sp->z_tool, sp->z_sp);
    } else {
      const Modes x0 = list(sp->rest.x, sp->rest.nx);
      const Modes y0 = sp->rest.ny > 0 ? list(sp->rest.y, sp->rest.ny) : x0;
      const double f = tipFactor(S, sp->k_tool, sp->k_sp, soft);
      x = f == 1 ? x0 : scaleModes(x0, f);
      y = f == 1 ? y0 : scaleModes(y0, f);
    }
    mcs_modal m{};
    m.nx = (int)x.size();
    m.ny = (int)y.size();
    std::copy(x.begin(), x.end(), m.x);
    std::copy(y.begin(), y.end(), m.y);
    out[i] = m;
  }
}
