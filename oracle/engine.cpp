// Oracle (test infrastructure only): FP64 restatement of the time-domain milling engine
// CuttingEngine of src/cutting.js -- configure (:39-82), setEngagement (:98-124), the run
// loop's force law, modal integration and sampling (:146-296) and chatterIndex (:299-318).
// Operation order follows the reference expression by expression; Float32Array stores
// (surf, Hb, tooth samples, history) round to float exactly where the reference stores.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace {

constexpr int kBins = 180;          // cutting.js:15
constexpr int kEndBins = 36;        // cutting.js:16
constexpr int kEndRings = 6;        // cutting.js:17
constexpr double kHRef = 0.05;      // cutting.js:18
constexpr double kHMin = 0.002;     // cutting.js:19
constexpr double kPi = 3.141592653589793;

// JS Math.round for the non-negative values it is used on here: floor(x + 0.5).
inline double js_round(double x) { return std::floor(x + 0.5); }

struct ModeBank {  // cutting.js:54-59 pack()
  std::vector<double> k, m, c, q, v;
};

struct SampleRing {  // the {n, i, count, x, y} rings of cutting.js:28-29
  int n = 0, i = 0;
  long long count = 0;
  std::vector<float> x, y;
  void reset(int size) {
    n = size;
    i = 0;
    count = 0;
    x.assign(size, 0.f);
    y.assign(size, 0.f);
  }
};

}  // namespace

struct or_engine {
  // tool / configuration
  int N = 0, type = 0;
  double R = 0, tanB = 0, fluteLen = 0;
  bool nonlinear = true;
  std::vector<double> dR;
  double S = 0, omega = 0, Ttooth = 0, dt = 0;
  int spt = 0, spr = 0, decim = 1;
  int sliceOverride = 0;
  ModeBank mx, my;
  double dz = 0;
  int maxSlices = 0;
  std::vector<float> surf;
  int pr = 0;
  double x = 0, y = 0, vx = 0, vy = 0, t = 0;
  double x0 = 0, y0 = 0, vx0 = 0, vy0 = 0;
  long long stepCount = 0;
  // material (Kac, Kae: the axial force; wear: setWear's edge coefficients)
  double Ktc = 0, Krc = 0, Kte = 0, Kre = 0, mc = 0, Ci = 0, Kac = 0, Kae = 0;
  bool wear = false;
  double KteW = 0, KreW = 0;
  // end edges (setEndEngagement, cutting.js:130-143)
  float Eb[kEndBins * kEndRings];
  double fza = 0, endR = 0;
  double ringR[kEndRings] = {}, ringCos[kEndRings] = {}, ringDs[kEndRings] = {},
         ringZ[kEndRings] = {};
  // thin wall (setWork, cutting.js:88-94)
  double wk = 0, wm = 1, wc = 0, wnx = 1, wny = 0, w = 0, wv = 0, runMeanW = 0;
  // engagement
  float Hb[kBins];
  double ux = 1, uy = 0, vxd = 0, vyd = 1, fz = 0, tipZ = 0, db = 0;
  int nz = 0;
  std::vector<double> sliceB, sliceZ, sliceLag, sliceR, sliceKap;
  // samples and statistics
  SampleRing hist, ts;
  std::vector<float> histF[3];  // Fx, Fy, Fz of the history ring
  mcs_engine_stats st;
  std::vector<unsigned char> toothEngaged;
  std::vector<double> toothVol;
  std::vector<double> chipVols;

  or_engine() {
    std::memset(Hb, 0, sizeof(Hb));
    std::memset(Eb, 0, sizeof(Eb));
    hist.reset(4096);
    for (auto& f : histF) f.assign(4096, 0.f);
    ts.reset(64);
    new_stats(st);
  }
  static void new_stats(mcs_engine_stats& s) {  // newStats() (cutting.js:324-327)
    std::memset(&s, 0, sizeof(s));
    s.minX = INFINITY;
    s.maxX = -INFINITY;
    s.minY = INFINITY;
    s.maxY = -INFINITY;
  }
};

extern "C" {

or_engine* or_engine_new(void) { return new or_engine(); }
void or_engine_free(or_engine* e) { delete e; }
float* or_engine_hb(or_engine* e) { return e->Hb; }

void or_engine_configure(or_engine* e, const mcs_tool* tool, int nonlinear,
                         const mcs_modal* modal, const mcs_material* mat, double S,
                         double fn_max, int spt_override, int slices_override) {
  e->N = tool->N;
  e->R = tool->R;
  e->type = tool->type;
  e->fluteLen = tool->flute_len;
  e->nonlinear = nonlinear != 0;
  e->tanB = std::tan(tool->helix_deg * kPi / 180);
  // radial offset of each tooth from runout (cutting.js:43-44)
  const double ecc = tool->runout, g0 = tool->runout_phase;
  e->dR.assign(e->N, 0.0);
  for (int i = 0; i < e->N; i++) e->dR[i] = ecc * std::cos(2 * kPi * i / e->N - g0);
  e->S = std::max(100.0, S);
  e->omega = e->S * 2 * kPi / 60;
  const double Ttooth = 60 / (e->S * e->N);
  // modeSet (frf.js:6-11): y takes the x modes when it has none of its own
  const int nx = modal->nx, ny = modal->ny > 0 ? modal->ny : modal->nx;
  const mcs_mode* xm = modal->x;
  const mcs_mode* ym = modal->ny > 0 ? modal->y : modal->x;
  double fTop = -INFINITY;
  for (int j = 0; j < nx; j++) fTop = std::max(fTop, xm[j].fn);
  for (int j = 0; j < ny; j++) fTop = std::max(fTop, ym[j].fn);
  if (spt_override > 0)
    e->spt = spt_override;
  else
    e->spt = (int)std::max(48.0, std::ceil(Ttooth * std::max(fTop, fn_max) * 24));
  e->dt = Ttooth / e->spt;
  e->Ttooth = Ttooth;
  auto pack = [](const mcs_mode* ms, int n, ModeBank& b) {
    b.k.resize(n);
    b.m.resize(n);
    b.c.resize(n);
    b.q.assign(n, 0.0);
    b.v.assign(n, 0.0);
    for (int i = 0; i < n; i++) {
      b.k[i] = ms[i].k * 1e3;
      const double w = 2 * kPi * ms[i].fn;
      b.m[i] = b.k[i] / (w * w);
      b.c[i] = 2 * ms[i].zeta * std::sqrt(b.k[i] * b.m[i]);
    }
  };
  pack(xm, nx, e->mx);
  pack(ym, ny, e->my);
  e->x0 = e->y0 = e->vx0 = e->vy0 = 0;
  // slices and the one-revolution surface ring (cutting.js:63-68)
  e->sliceOverride = slices_override;
  e->dz = std::max(0.25, e->fluteLen / 48);
  e->maxSlices = (int)std::ceil(e->fluteLen / e->dz);
  e->spr = e->N * e->spt;
  e->surf.assign((size_t)e->maxSlices * e->spr, 0.f);
  e->pr = 0;
  e->x = e->y = e->vx = e->vy = e->t = 0;
  e->toothEngaged.assign(e->N, 0);
  e->toothVol.assign(e->N, 0.0);
  e->chipVols.clear();
  e->decim = (int)std::max(1.0, js_round(e->spt / 40.0));
  e->stepCount = 0;
  e->Ktc = mat->Ktc;
  e->Krc = mat->Krc;
  e->Kte = mat->Kte;
  e->Kre = mat->Kre;
  e->mc = mat->mc;
  e->Ci = mat->Ci;
  // setWork(null) and no end-edge feed (cutting.js:73-75)
  e->wk = 0;
  e->wm = 1;
  e->wc = 0;
  e->w = 0;
  e->wv = 0;
  e->wnx = 1;
  e->wny = 0;
  e->runMeanW = 0;
  e->fza = 0;
}

void or_engine_set_engagement_profile(or_engine* e, double ux, double uy, double fz,
                                      double tipZ, double ap, const double* prof_r,
                                      const double* prof_kap);

void or_engine_set_engagement(or_engine* e, double ux, double uy, double fz, double tipZ,
                              double ap) {
  or_engine_set_engagement_profile(e, ux, uy, fz, tipZ, ap, nullptr, nullptr);
}

// setEngagement with a general edge profile: slice k's radius prof_r[k] and kappa
// prof_kap[k], as rAt gives them (cutting.js:115-118); NULL: the flat / ball rule
void or_engine_set_engagement_profile(or_engine* e, double ux, double uy, double fz,
                                      double tipZ, double ap, const double* prof_r,
                                      const double* prof_kap) {
  e->ux = ux;
  e->uy = uy;
  e->vxd = -uy;
  e->vyd = ux;
  e->fz = fz;
  e->tipZ = tipZ;
  int nz;
  if (e->sliceOverride > 0) {
    // fixed slice count: equal slices over the depth (an explicit option, not in the
    // reference; dz = ap / n replaces the max(0.25, fluteLen/48) rule)
    nz = ap <= 0 ? 0 : e->sliceOverride;
    if (ap > 0) e->dz = ap / nz;
    if ((size_t)nz * e->spr > e->surf.size()) e->surf.assign((size_t)nz * e->spr, 0.f);
  } else {
    nz = ap <= 0 ? 0 : std::min(e->maxSlices, (int)std::ceil(ap / e->dz));
  }
  e->nz = nz;
  e->db = e->dz;
  e->sliceB.assign(nz, 0.0);
  e->sliceZ.assign(nz, 0.0);
  e->sliceLag.assign(nz, 0.0);
  e->sliceR.assign(nz, 0.0);
  e->sliceKap.assign(nz, 0.0);
  const double R = e->R;
  for (int k = 0; k < nz; k++) e->sliceB[k] = std::min(e->dz, ap - k * e->dz);
  for (int k = 0; k < nz; k++) {
    const double zr = k * e->dz + 0.5 * e->sliceB[k];
    e->sliceZ[k] = tipZ + zr;
    double r = R, kap = 1;
    if (prof_r) {
      r = prof_r[k];
      kap = prof_kap[k];
    } else if (e->type == MCS_TOOL_BALL && zr < R) {
      const double d = R - zr;
      r = std::sqrt(std::max(1e-6, R * R - d * d));
      kap = r / R;
    }
    e->sliceR[k] = r;
    e->sliceKap[k] = kap;
    e->sliceLag[k] = zr * e->tanB / R;
  }
}

void or_engine_set_state(or_engine* e, double x, double y, double vx, double vy) {
  e->x = x;
  e->y = y;
  e->vx = vx;
  e->vy = vy;
}

void or_engine_run(or_engine* e, int64_t nSteps) {
  const int N = e->N, spt = e->spt, spr = e->spr, nz = e->nz;
  float* surf = e->surf.data();
  const double ux = e->ux, uy = e->uy, vx = e->vxd, vy = e->vyd, fz = e->fz, dt = e->dt;
  const double Ktc = e->Ktc, Krc = e->Krc, Kac = e->Kac, Kae = e->Kae;
  // edge coefficients grow with the flank wear land (setWear)
  const double Kte = e->wear ? e->KteW : e->Kte, Kre = e->wear ? e->KreW : e->Kre;
  const bool nl = e->nonlinear;
  const double mc = nl ? e->mc : 0;
  // process damping per slice [N s/m] = Ci b / V_c (cutting.js:155-156)
  const double pdK = nl ? e->Ci * e->db * 1e-3 / (e->omega * 1e-3) : 0;
  const double TWO_PI = 2 * kPi, binScale = kBins / TWO_PI, pitch = TWO_PI / N;
  const double dphi = e->omega * dt;
  const double hMax = std::max(0.1, 3 * fz);
  const float* Eb = e->Eb;
  const double fza = e->fza;
  ModeBank& MX = e->mx;
  ModeBank& MY = e->my;
  const int nmx = (int)MX.k.size(), nmy = (int)MY.k.size();
  // a state set from outside since the last run goes into the first mode (:163-164)
  MX.q[0] += e->x - e->x0;
  MY.q[0] += e->y - e->y0;
  MX.v[0] += e->vx - e->vx0;
  MY.v[0] += e->vy - e->vy0;
  double x = e->x, y = e->y, vxs = e->vx, vys = e->vy, t = e->t;
  int pr = e->pr;
  const double wk = e->wk, wm = e->wm, wc = e->wc, wnx = e->wnx, wny = e->wny;
  double w = e->w, wv = e->wv, wSum = 0;
  mcs_engine_stats& st = e->st;
  SampleRing& hist = e->hist;
  SampleRing& ts = e->ts;
  for (int64_t s = 0; s < nSteps; s++) {
    const double theta = pr * dphi;
    // tool position relative to the (possibly deflected) workpiece [mm]
    const double rx = x - w * wnx, ry = y - w * wny;
    const double xm = rx * 1e3, ym = ry * 1e3;
    double Fx = 0, Fy = 0, Fz = 0, T = 0, Fr2z = 0, Fsum = 0;
    // relative tool-to-wall velocity [m/s] for process damping
    const double rvx = vxs - wv * wnx, rvy = vys - wv * wny;
    for (int i = 0; i < N; i++) {
      int engaged = 0;
      const double dRi = e->dR[i];
      int pi = pr + i * spt;
      if (pi >= spr) pi -= spr;
      for (int k = 0; k < nz; k++) {
        double phi = std::fmod(theta + i * pitch - e->sliceLag[k], TWO_PI);
        if (phi < 0) phi += TWO_PI;
        const double sn = std::sin(phi), cs = std::cos(phi);
        const double nxg = sn * ux + cs * vx, nyg = sn * uy + cs * vy;
        const double rn = xm * nxg + ym * nyg + dRi;
        const size_t idx = (size_t)k * spr + pi;
        const double prev = surf[idx];
        const double feedH = fz * sn * e->sliceKap[k];
        // Hb[(phi * binScale) | 0]: a bin past the map (180) reads undefined, and
        // undefined <= z is false
        const double bscaled = phi * binScale;
        const int bin = (bscaled == bscaled) ? (int)bscaled : 0;
        const bool hbOut = bin < kBins && (double)e->Hb[bin] <= e->sliceZ[k];
        if (hbOut || sn <= 0) {
          surf[idx] = (float)rn;
          continue;
        }
        double h = feedH + rn - prev;
        // tooth out of cut: the old surface survives one more feed step
        if (h <= 0) {
          surf[idx] = (float)(prev - feedH);
          continue;
        }
        surf[idx] = (float)rn;
        if (h > hMax) h = hMax;
        const double se = mc != 0 ? std::pow(kHRef / (h > kHMin ? h : kHMin), mc) : 1;
        const double bk = e->sliceB[k];
        const double Ft = Ktc * se * h * bk + Kte * bk;
        double Fr = Krc * se * h * bk + Kre * bk;
        const double Fa = Kac * se * h * bk + Kae * bk;
        if (pdK != 0) Fr += pdK * (bk / e->db) / e->sliceR[k] * (rvx * nxg + rvy * nyg);
        const double txg = cs * ux - sn * vx, tyg = cs * uy - sn * vy;
        Fx += -Ft * txg - Fr * nxg;
        Fy += -Ft * tyg - Fr * nyg;
        Fz -= Fa;
        T += Ft * e->sliceR[k];
        const double fr = std::hypot(Ft, Fr);
        Fsum += fr;
        Fr2z += fr * (e->sliceZ[k] - e->tipZ);
        engaged = 1;
        st.sumHb += h * bk;
        st.sumB += bk;
        st.sumRb += e->sliceR[k] * h * bk;
        e->toothVol[i] += h * bk * e->sliceR[k] * dphi;
      }
      if (fza != 0) {
        // end edges at the tip (no helix lag): thrust, torque, in-plane tangential force
        double phi = std::fmod(theta + i * pitch, TWO_PI);
        if (phi < 0) phi += TWO_PI;
        const int row = ((int)(phi / TWO_PI * kEndBins)) * kEndRings;
        const double sn = std::sin(phi), cs = std::cos(phi);
        const double txg = cs * ux - sn * vx, tyg = cs * uy - sn * vy;
        for (int j = 0; j < kEndRings; j++) {
          const double depth = row < kEndBins * kEndRings ? (double)Eb[row + j] : 0.0;
          if (depth <= 2e-4) continue;
          const double c = e->ringCos[j], ds = e->ringDs[j];
          const double h = (depth < fza ? depth : fza) * c;
          const double se = mc != 0 ? std::pow(kHRef / (h > kHMin ? h : kHMin), mc) : 1;
          const double Ft = Ktc * se * h * ds + Kte * ds;
          const double Fn = Krc * se * h * ds + Kre * ds;
          Fx += -Ft * txg;
          Fy += -Ft * tyg;
          Fz -= Fn * c;
          T += Ft * e->ringR[j];
          Fsum += Ft;
          Fr2z += Ft * e->ringZ[j];
          engaged = 1;
          st.sumHb += h * ds;
          st.sumB += ds;
          st.sumRb += e->ringR[j] * h * ds;
          e->toothVol[i] += h * ds * e->ringR[j] * dphi;
        }
      }
      if (!engaged && e->toothEngaged[i]) {
        if (e->toothVol[i] > 0) e->chipVols.push_back(e->toothVol[i]);
        e->toothVol[i] = 0;
      }
      e->toothEngaged[i] = (unsigned char)engaged;
      st.engTeeth += engaged;
    }
    // modal integration, semi-implicit Euler (:246-255)
    x = 0;
    y = 0;
    vxs = 0;
    vys = 0;
    for (int j = 0; j < nmx; j++) {
      MX.v[j] += (Fx - MX.c[j] * MX.v[j] - MX.k[j] * MX.q[j]) / MX.m[j] * dt;
      MX.q[j] += MX.v[j] * dt;
      x += MX.q[j];
      vxs += MX.v[j];
    }
    for (int j = 0; j < nmy; j++) {
      MY.v[j] += (Fy - MY.c[j] * MY.v[j] - MY.k[j] * MY.q[j]) / MY.m[j] * dt;
      MY.q[j] += MY.v[j] * dt;
      y += MY.q[j];
      vys += MY.v[j];
    }
    if (wk != 0) {
      // reaction on the wall: opposite to the force on the tool, along the wall normal
      const double Fw = -(Fx * wnx + Fy * wny);
      wv += (Fw - wc * wv - wk * w) / wm * dt;
      w += wv * dt;
      // the wall cannot be pushed further than the material the cutter is engaged in
      if (w > 5e-4) {
        w = 5e-4;
        if (wv > 0) wv = 0;
      } else if (w < -2e-4) {
        w = -2e-4;
        if (wv < 0) wv = 0;
      }
      st.sumW += w;
      st.maxW = std::max(st.maxW, std::fabs(w));
      wSum += w;
    }
    if (++pr == spr) pr = 0;
    const int ph = pr % spt;
    if (ph == 0) {  // once-per-tooth sample (:266-268)
      ts.x[ts.i] = (float)(x - w * wnx);
      ts.y[ts.i] = (float)(y - w * wny);
      ts.i = (ts.i + 1) % ts.n;
      ts.count++;
    }
    t += dt;
    // statistics (:280-287)
    const double Fxy = std::hypot(Fx, Fy);
    st.n++;
    st.sumF += Fxy;
    st.maxF = std::max(st.maxF, Fxy);
    st.sumFx += Fx;
    st.sumFy += Fy;
    st.sumFz += Fz;
    st.maxFz = std::max(st.maxFz, -Fz);
    st.sumT += T;
    st.maxT = std::max(st.maxT, T);
    st.sumX += x;
    st.sumY += y;
    st.minX = std::min(st.minX, x);
    st.maxX = std::max(st.maxX, x);
    st.minY = std::min(st.minY, y);
    st.maxY = std::max(st.maxY, y);
    if (Fsum > 0) {
      st.sumZc += Fr2z / Fsum * Fxy;
      st.wZc += Fxy;
    }
    if (++e->stepCount % e->decim == 0) {  // decimated history (:288-292)
      const int j = hist.i;
      e->histF[0][j] = (float)Fx;
      e->histF[1][j] = (float)Fy;
      e->histF[2][j] = (float)Fz;
      hist.x[j] = (float)((x - w * wnx) * 1e6);
      hist.y[j] = (float)((y - w * wny) * 1e6);
      hist.i = (j + 1) % hist.n;
      hist.count++;
    }
  }
  e->x = e->x0 = x;
  e->y = e->y0 = y;
  e->vx = e->vx0 = vxs;
  e->vy = e->vy0 = vys;
  e->t = t;
  e->pr = pr;
  e->w = w;
  e->wv = wv;
  e->runMeanW = nSteps ? wSum / nSteps : 0;  // mean wall deflection over this call [m]
}

void or_engine_set_axial(or_engine* e, double Kac, double Kae) {
  e->Kac = Kac;
  e->Kae = Kae;
}

void or_engine_set_wear(or_engine* e, int on, double Kte, double Kre) {
  e->wear = on != 0;
  e->KteW = Kte;
  e->KreW = Kre;
}

float* or_engine_eb(or_engine* e) { return e->Eb; }

// setEndEngagement(fza, rOut, zAt) (cutting.js:130-143) with zAt sampled by the caller at
// each ring radius r_j and at min(rOut, r_j + dr/4), max(0, r_j - dr/4)
void or_engine_set_end(or_engine* e, double fza, double rOut, const double* z_at,
                       const double* z_out, const double* z_in) {
  e->fza = fza > 0 ? fza : 0;
  e->endR = rOut;
  const double dr = rOut / kEndRings;
  for (int j = 0; j < kEndRings; j++) {
    const double r = (j + 0.5) * dr;
    const double slope = (z_out[j] - z_in[j]) / (0.5 * dr);
    const double c = std::max(0.22, 1 / std::sqrt(1 + slope * slope));
    e->ringR[j] = r;
    e->ringCos[j] = c;
    e->ringDs[j] = dr / c;
    e->ringZ[j] = z_at[j];
  }
}

// setWork(wall) (cutting.js:88-94); k <= 0 is setWork(null)
void or_engine_set_work(or_engine* e, double k, double m, double zeta, double nx, double ny) {
  if (!(k > 0)) {
    e->runMeanW = 0;
    e->wk = 0;
    e->wm = 1;
    e->wc = 0;
    e->w = 0;
    e->wv = 0;
    e->wnx = 1;
    e->wny = 0;
    return;
  }
  // carry the wall state over only while the normal stays roughly the same
  if (e->wk != 0 && nx * e->wnx + ny * e->wny < 0.8) {
    e->w = 0;
    e->wv = 0;
  }
  e->wk = k * 1e3;
  e->wm = m;
  e->wc = 2 * zeta * std::sqrt(e->wk * m);
  e->wnx = nx;
  e->wny = ny;
}

void or_engine_take_stats_full(or_engine* e, mcs_engine_stats* out) {
  *out = e->st;
  or_engine::new_stats(e->st);
}

// the history ring: out[c * 4096 + j] for c = Fx, Fy, Fz, x, y
void or_engine_history(const or_engine* e, float* out, int32_t* head, int64_t* count) {
  const int n = e->hist.n;
  for (int c = 0; c < 3; c++) std::copy(e->histF[c].begin(), e->histF[c].end(), out + c * n);
  std::copy(e->hist.x.begin(), e->hist.x.end(), out + 3 * n);
  std::copy(e->hist.y.begin(), e->hist.y.end(), out + 4 * n);
  *head = e->hist.i;
  *count = e->hist.count;
}

void or_engine_set_decim(or_engine* e, int decim) { e->decim = decim > 0 ? decim : e->decim; }

void or_engine_reset_history(or_engine* e) {
  e->hist.i = 0;
  e->hist.count = 0;
}

void or_engine_chatter_index(const or_engine* e, double out[3]) {
  const SampleRing& ts = e->ts;
  const SampleRing& h = e->hist;
  const int n = (int)std::min<long long>(ts.count, 24);
  if (n < 8) {
    out[0] = 0;
    out[1] = 0;
    out[2] = 0;
    return;
  }
  double mx = 0, my = 0;
  for (int k = 0; k < n; k++) {
    const int j = (ts.i - 1 - k + ts.n) % ts.n;
    mx += ts.x[j];
    my += ts.y[j];
  }
  mx /= n;
  my /= n;
  double v = 0;
  for (int k = 0; k < n; k++) {
    const int j = (ts.i - 1 - k + ts.n) % ts.n;
    const double dx = ts.x[j] - mx, dy = ts.y[j] - my;
    v += dx * dx + dy * dy;
  }
  const double sOnce = std::sqrt(v / n) * 1e6;  // um
  const long long m =
      std::min<long long>(h.count, (long long)js_round((double)n * e->spt / e->decim));
  double ax = 0, ay = 0;
  for (long long k = 0; k < m; k++) {
    const int j = (int)((h.i - 1 - k + h.n) % h.n);
    ax += h.x[j];
    ay += h.y[j];
  }
  const double md = m ? (double)m : 1.0;
  ax /= md;
  ay /= md;
  double w = 0;
  for (long long k = 0; k < m; k++) {
    const int j = (int)((h.i - 1 - k + h.n) % h.n);
    const double dx = h.x[j] - ax, dy = h.y[j] - ay;
    w += dx * dx + dy * dy;
  }
  const double sAll = std::sqrt(w / md);
  out[0] = sOnce / (sAll + 0.05);
  out[1] = sAll;
  out[2] = sOnce;
}

void or_engine_take_stats(or_engine* e, or_stats* out) {
  const mcs_engine_stats& s = e->st;
  out->n = s.n;
  out->sumF = s.sumF;
  out->maxF = s.maxF;
  out->sumFx = s.sumFx;
  out->sumFy = s.sumFy;
  out->sumX = s.sumX;
  out->sumY = s.sumY;
  out->engTeeth = s.engTeeth;
  or_engine::new_stats(e->st);
}

int or_engine_chip_vols(const or_engine* e, double* out, int cap) {
  const int n = (int)std::min<size_t>(e->chipVols.size(), (size_t)cap);
  for (int i = 0; i < n; i++) out[i] = e->chipVols[i];
  return (int)e->chipVols.size();
}

void or_engine_get_info(const or_engine* e, or_engine_info* out) {
  out->steps_per_tooth = e->spt;
  out->steps_per_rev = e->spr;
  out->nz = e->nz;
  out->decim = e->decim;
  out->max_slices = e->maxSlices;
  out->pad = 0;
  out->dt = e->dt;
  out->omega = e->omega;
  out->dz = e->dz;
}

}  // extern "C"
