// Oracle (test infrastructure only): the uniform cantilever tool model of
// src/tool.js:16-32 (toolModel) and the engagement-arc mapping of
// src/identify.js:18-22 (immersion), used to build the reference tests' setups.
#include <cmath>

#include "oracle.h"

namespace {
constexpr double kPi = 3.141592653589793;
constexpr double kECarbide = 600000;    // MPa, tool.js:4
constexpr double kRhoCarbide = 14500;   // kg/m^3, tool.js:5
}  // namespace

extern "C" {

void or_tool_model(double D, double L, double kSpindle, double mHolder, double out[4]) {
  const double De = 0.8 * D;
  const double I = kPi * std::pow(De, 4) / 64;                 // mm^4
  const double kTool = 3 * kECarbide * I / std::pow(L, 3);     // N/mm
  const double kTotal = 1 / (1 / kTool + 1 / kSpindle);
  const double EI = kECarbide * 1e6 * I * 1e-12;
  const double d = De * 1e-3;
  const double rhoA = kRhoCarbide * kPi * (d * d) / 4;
  const double Lm = L * 1e-3;
  const double wTool = 1.875 * 1.875 * std::sqrt(EI / rhoA) / (Lm * Lm);
  const double mEff = kTool * 1e3 / (wTool * wTool) + mHolder;
  const double fn = std::sqrt(kTotal * 1e3 / mEff) / (2 * kPi);
  out[0] = kTotal;
  out[1] = fn;
  out[2] = kTool;
  out[3] = mEff;
}

void or_immersion(int mode, double ae, double D, double out[2]) {
  if (mode == 0 || !(ae < D)) {
    out[0] = 0;
    out[1] = kPi;
    return;
  }
  const double pe = std::acos(1 - 2 * ae / D);
  if (mode == 1) {
    out[0] = kPi - pe;
    out[1] = kPi;
  } else {
    out[0] = 0;
    out[1] = pe;
  }
}

}  // extern "C"
