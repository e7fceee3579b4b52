// Speed-dependent tool-tip modes (mcs_modes_at, include/mcs.h): the modesAt model of the
// reference's spindle.js.  Host code in FP64; it builds the per-speed modal sets that a
// lobe sweep sends with its points (main.js:495-496, sim.modalNow at sim.js:229-233).
//
//   bearingFactor  spindle.js:18-23   k_s(S) / k_s0 = 1 / (1 + c (S / S_ref)^2), c = d/(1-d)
//   tipFactor      spindle.js:26-30   tool-tip stiffness ratio through the chain
//                                     1/k = 1/k_tool + 1/k_s
//   twoDofModes    spindle.js:38-53   tool on a spindle mode: two tip modes of a two-mass model
//   modesAt        spindle.js:64-85   measured FRFs at speeds (interpolated), else the two-mass
//                                     model, else the rest modes scaled by the tip factor
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/mcs.h"

namespace mcs {
int fail(int code, const char* fmt, ...);
}

namespace {

constexpr double kPi = 3.141592653589793;

double bearing_factor(double S, const mcs_spindle& sp) {
  const double d = std::min(0.9, std::max(0.0, sp.drop));
  if (!(d != 0.0) || !(S > 0)) return 1.0;
  const double c = d / (1 - d);
  const double r = S / (sp.s_ref != 0.0 ? sp.s_ref : 30000.0);
  return 1 / (1 + c * (r * r));
}

double tip_factor(double S, const mcs_spindle& sp) {
  const double b = bearing_factor(S, sp);
  if (b == 1.0 || !(sp.k_tool > 0) || !(sp.k_sp > 0)) return 1.0;
  return (1 / sp.k_tool + 1 / sp.k_sp) / (1 / sp.k_tool + 1 / (sp.k_sp * b));
}

// The two modes of a tool (k_tool [N/mm], m_tool [kg]) on a spindle spring (k_sp, m_sp),
// low frequency first; each mode's tip-equivalent stiffness m_r w_r^2 / phi_tip^2.
void two_dof_modes(double kTool, double mTool, double kSp, double mSp, double zTool, double zSp,
                   mcs_mode out[2]) {
  const double k1 = kSp * 1e3, k2 = kTool * 1e3, m1 = mSp, m2 = mTool;
  const double a = m1 * m2, b = -((k1 + k2) * m2 + k2 * m1), c = k1 * k2;
  const double disc = std::sqrt(std::max(0.0, b * b - 4 * a * c));
  const double w2s[2] = {(-b - disc) / (2 * a), (-b + disc) / (2 * a)};
  for (int i = 0; i < 2; i++) {
    const double w2 = w2s[i];
    const double phiT = (k1 + k2 - w2 * m1) / k2;  // mode shape with phi_spindle = 1
    const double mr = m1 + m2 * phiT * phiT;
    out[i].k = mr * w2 / (phiT * phiT) / 1e3;
    out[i].fn = std::sqrt(w2) / (2 * kPi);
    out[i].zeta = m2 * phiT * phiT > m1 ? zTool : zSp;  // the part with most kinetic energy
  }
}

// One axis of a modal set: its modes and count (ny == 0 means y takes the x modes).
struct Axis {
  int n;
  const mcs_mode* m;
};
Axis axis_x(const mcs_modal& md) { return {md.nx, md.x}; }
Axis axis_y(const mcs_modal& md) { return md.ny > 0 ? Axis{md.ny, md.y} : Axis{md.nx, md.x}; }

// lerpModes (spindle.js:57-60): by mode order when the counts match, else the nearer one
int lerp_axis(Axis a, Axis b, double t, mcs_mode* out) {
  if (a.n != b.n) {
    const Axis& s = t < 0.5 ? a : b;
    std::copy(s.m, s.m + s.n, out);
    return s.n;
  }
  for (int i = 0; i < a.n; i++) {
    out[i].k = a.m[i].k + (b.m[i].k - a.m[i].k) * t;
    out[i].fn = a.m[i].fn + (b.m[i].fn - a.m[i].fn) * t;
    out[i].zeta = a.m[i].zeta + (b.m[i].zeta - a.m[i].zeta) * t;
  }
  return a.n;
}

bool modes_ok(const mcs_modal& md) {
  if (md.nx < 1 || md.nx > MCS_MAX_MODES || md.ny < 0 || md.ny > MCS_MAX_MODES) return false;
  for (int a = 0; a < 2; a++) {
    const Axis ax = a == 0 ? axis_x(md) : axis_y(md);
    for (int j = 0; j < ax.n; j++)
      if (!(std::isfinite(ax.m[j].k) && ax.m[j].k > 0 && std::isfinite(ax.m[j].fn) &&
            ax.m[j].fn > 0 && std::isfinite(ax.m[j].zeta) && ax.m[j].zeta >= 0))
        return false;
  }
  return true;
}

}  // namespace

extern "C" int mcs_modes_at(const mcs_spindle* sp, const mcs_speed_frf* frfs, size_t n_frfs,
                            const double* S, size_t n_speeds, mcs_modal* out) {
  using mcs::fail;
  if (!sp) return fail(MCS_ERR_ARG, "spindle model is NULL");
  if (n_speeds && (!S || !out)) return fail(MCS_ERR_ARG, "NULL speeds or output");
  if (n_frfs && !frfs) return fail(MCS_ERR_ARG, "NULL measured FRFs");
  if (!modes_ok(sp->rest)) return fail(MCS_ERR_ARG, "rest modes invalid");
  if (!(std::isfinite(sp->drop) && std::isfinite(sp->s_ref) && std::isfinite(sp->k_tool) &&
        std::isfinite(sp->k_sp)))
    return fail(MCS_ERR_ARG, "spindle model has a non-finite value");
  if (sp->two_dof && !(sp->m_tool > 0 && sp->m_sp > 0 && sp->k_tool > 0 && sp->k_sp > 0 &&
                       std::isfinite(sp->z_tool) && std::isfinite(sp->z_sp)))
    return fail(MCS_ERR_ARG, "two-mass model needs k_tool, k_sp, m_tool, m_sp > 0");
  for (size_t i = 0; i < n_frfs; i++)
    if (!std::isfinite(frfs[i].S) || !modes_ok(frfs[i].modes))
      return fail(MCS_ERR_ARG, "measured FRF %zu invalid", i);
  for (size_t i = 0; i < n_speeds; i++)
    if (!std::isfinite(S[i])) return fail(MCS_ERR_ARG, "speed %zu is not finite", i);
  // measured FRFs in speed order (a stable sort, as Array.prototype.sort)
  std::vector<mcs_speed_frf> L(frfs, frfs + n_frfs);
  std::stable_sort(L.begin(), L.end(),
                   [](const mcs_speed_frf& p, const mcs_speed_frf& q) { return p.S < q.S; });
  for (size_t i = 0; i < n_speeds; i++) {
    const double s = S[i];
    mcs_modal m{};
    if (!L.empty()) {
      auto pick = [&](const mcs_speed_frf& e) {
        mcs_modal r{};
        const Axis x = axis_x(e.modes), y = axis_y(e.modes);
        r.nx = x.n;
        r.ny = y.n;
        std::copy(x.m, x.m + x.n, r.x);
        std::copy(y.m, y.m + y.n, r.y);
        return r;
      };
      if (s <= L.front().S) {
        m = pick(L.front());
      } else if (s >= L.back().S) {
        m = pick(L.back());
      } else {
        size_t j = 1;
        while (L[j].S < s) j++;
        const mcs_modal a = pick(L[j - 1]), b = pick(L[j]);
        const double t = (s - L[j - 1].S) / (L[j].S - L[j - 1].S);
        m.nx = lerp_axis(axis_x(a), axis_x(b), t, m.x);
        m.ny = lerp_axis(axis_y(a), axis_y(b), t, m.y);
      }
    } else if (sp->two_dof) {
      mcs_mode ms[2];
      two_dof_modes(sp->k_tool, sp->m_tool, sp->k_sp * bearing_factor(s, *sp), sp->m_sp,
                    sp->z_tool, sp->z_sp, ms);
      m.nx = m.ny = 2;
      std::copy(ms, ms + 2, m.x);
      std::copy(ms, ms + 2, m.y);
    } else {
      const Axis x = axis_x(sp->rest), y = axis_y(sp->rest);
      const double f = tip_factor(s, *sp);
      m.nx = x.n;
      m.ny = y.n;
      for (int a = 0; a < 2; a++) {
        const Axis ax = a == 0 ? x : y;
        mcs_mode* dst = a == 0 ? m.x : m.y;
        for (int j = 0; j < ax.n; j++) {
          dst[j] = ax.m[j];
          if (f != 1.0) {  // scaleModes: each mode keeps its mass (spindle.js:55)
            dst[j].k = ax.m[j].k * f;
            dst[j].fn = ax.m[j].fn * std::sqrt(f);
          }
        }
      }
    }
    out[i] = m;
  }
  return MCS_OK;
}
