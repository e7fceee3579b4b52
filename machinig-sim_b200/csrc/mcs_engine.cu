// Batched time-domain cutting engines (mcs_engine_*, include/mcs.h): class CuttingEngine of
// src/cutting.js:21-321 on the device, one warp per engine, state kept between runs.
//
// The host derives everything configure() and setEngagement() compute (FP64, the
// reference's expressions) and uploads it; the run kernel executes the run() loop
// (cutting.js:146-296) with every term a cut has:
//   * the flutes (:171-212): a step's (tooth, slice) evaluations are spread over the
//     lanes, all teeth side by side; each evaluation takes the angle, the engagement-map
//     bin, the regenerative chip, the size effect, process damping, the axial force and
//     the torque, in FP64 with the surface ring in float;
//   * the end edges (:213-237): the (tooth, end ring) evaluations spread the same way;
//   * the per-step sums (forces, torque, force-weighted height) by warp butterflies, the
//     modal integration (:239-249) and the thin wall (:250-258) on every lane;
//   * once-per-tooth samples, statistics and the decimated history (:259-292) by lane 0.
// Wall samples and chip events (roughness and chip models, outside this library) are not
// produced.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "mcs_internal.h"

namespace mcs {
namespace {

constexpr double kPi = 3.141592653589793;
constexpr double kTwoPi = 2 * kPi;
constexpr double kHRef = 0.05;  // cutting.js:18
constexpr double kHMin = 0.002; // cutting.js:19
constexpr int kE = MCS_END_BINS, kR = MCS_END_RINGS, kS = MCS_MAX_SLICES;
constexpr int kH = MCS_ENGINE_HIST, kTs = MCS_ENGINE_TS;
constexpr unsigned kAll = 0xffffffffu;

// configure() (cutting.js:39-82), derived on the host
struct EngCfg {
  double R, tanB, omega, dt, dphi, pitch, dz;
  double dR[MCS_MAX_TEETH];
  double mk[2][MCS_MAX_MODES], mm[2][MCS_MAX_MODES], mcd[2][MCS_MAX_MODES];
  double Ktc, Krc, Kac, Kte, Kre, Kae, mc, Ci;
  long long surf_off;  // floats into the surface pool
  int N, spt, spr, decim, max_slices, nm[2], nonlinear, configured, pad;
};

// setEngagement (:98-124), setEndEngagement (:130-143), setWork (:88-94), setWear (:85)
struct EngGeo {
  float Hb[MCS_BINS];
  float Eb[kE * kR];
  double ux, uy, vx, vy, fz, tipZ, db;
  double sliceB[kS], sliceZ[kS], sliceLag[kS], sliceR[kS], sliceKap[kS];
  double fza, ringR[kR], ringCos[kR], ringDs[kR], ringZ[kR];
  double Kte, Kre;
  double wk, wm, wc, wnx, wny;
  int nz, reset_wall, set, pad;
};

// what run() carries between calls
struct EngState {
  double q[2][MCS_MAX_MODES], v[2][MCS_MAX_MODES];
  double x, y, vx, vy, x0, y0, vx0, vy0, t, w, wv, run_mean_w;
  long long step_count, ts_count, h_count;
  int pr, ts_i, h_i, pad;
  float ts_x[kTs], ts_y[kTs];
  mcs_engine_stats st;
};

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kAll, v, o);
  return v;
}

// JS `%` on the angle (fmod: the sign of the dividend), exact: below 4 pi the subtraction
// of 2 pi is exact (Sterbenz), elsewhere fmod itself
__device__ __forceinline__ double angle_mod(double a) {
  if (a >= 0 && a < 2 * kTwoPi) return a >= kTwoPi ? a - kTwoPi : a;
  return fmod(a, kTwoPi);
}

__global__ void __launch_bounds__(32) engine_run_kernel(const EngCfg* __restrict__ cfgs,
                                                        const EngGeo* __restrict__ geos,
                                                        EngState* __restrict__ states,
                                                        float* __restrict__ surf_pool,
                                                        float* __restrict__ hist_pool,
                                                        const long long* __restrict__ steps) {
  const int e = blockIdx.x, lane = threadIdx.x;
  const long long n_steps = steps[e];
  const EngCfg& C = cfgs[e];
  const EngGeo& G = geos[e];
  if (n_steps <= 0 || !C.configured || !G.set) return;
  EngState& S = states[e];
  float* surf = surf_pool + C.surf_off;
  float* hist = hist_pool + (size_t)e * 5 * kH;
  const int N = C.N, spt = C.spt, spr = C.spr, nz = G.nz, nmx = C.nm[0], nmy = C.nm[1];
  const double ux = G.ux, uy = G.uy, vx = G.vx, vy = G.vy, fz = G.fz, dt = C.dt;
  const double Ktc = C.Ktc, Krc = C.Krc, Kac = C.Kac, Kae = C.Kae, Kte = G.Kte, Kre = G.Kre;
  const bool nl = C.nonlinear != 0;
  const double mc = nl ? C.mc : 0.0;
  const double pdK = nl ? C.Ci * G.db * 1e-3 / (C.omega * 1e-3) : 0.0;
  const double binScale = MCS_BINS / kTwoPi, pitch = C.pitch, dphi = C.dphi;
  const double hMax = fmax(0.1, 3 * fz);
  const double wk = G.wk, wm = G.wm, wc = G.wc, wnx = G.wnx, wny = G.wny;
  // a state set from outside since the last run goes into the first modes (:163-164)
  double q[2][MCS_MAX_MODES], v[2][MCS_MAX_MODES];
  for (int a = 0; a < 2; a++)
    for (int j = 0; j < MCS_MAX_MODES; j++) {
      q[a][j] = S.q[a][j];
      v[a][j] = S.v[a][j];
    }
  q[0][0] += S.x - S.x0;
  q[1][0] += S.y - S.y0;
  v[0][0] += S.vx - S.vx0;
  v[1][0] += S.vy - S.vy0;
  double x = S.x, y = S.y, vxs = S.vx, vys = S.vy, t = S.t;
  double w = S.w, wv = S.wv, wSum = 0;
  int pr = S.pr;
  long long stepCount = S.step_count;
  mcs_engine_stats st = S.st;  // lane 0's copy is the one stored
  double sHb = 0, sB = 0, sRb = 0;  // this lane's share of sumHb, sumB, sumRb
  int ts_i = S.ts_i, h_i = S.h_i;
  long long ts_count = S.ts_count, h_count = S.h_count;
  // a step's evaluations, tooth-major (e = i * nz + k for the flutes, i * kR + j for the end
  // rings), are spread over the lanes: lane l takes e = l, l + 32, ...; every tooth's
  // evaluations run side by side instead of one tooth after another
  const int ne = N * nz, nend = G.fza != 0 ? N * kR : 0;
  for (long long s = 0; s < n_steps; s++) {
    const double theta = pr * dphi;
    const double rx = x - w * wnx, ry = y - w * wny;
    const double xm = rx * 1e3, ym = ry * 1e3;
    double Fx = 0, Fy = 0, Fz = 0, T = 0, Fr2z = 0, Fsum = 0;
    const double rvx = vxs - wv * wnx, rvy = vys - wv * wny;
    unsigned teeth = 0;  // bit i: tooth i engaged on this lane
    for (int e = lane; e < ne; e += 32) {
      const int i = e / nz, k = e - i * nz;
      const double dRi = C.dR[i];
      int pi = pr + i * spt;
      if (pi >= spr) pi -= spr;
      double phi = angle_mod(theta + i * pitch - G.sliceLag[k]);
      if (phi < 0) phi += kTwoPi;
      double sn, cs;
      sincos(phi, &sn, &cs);
      const double nxg = sn * ux + cs * vx, nyg = sn * uy + cs * vy;
      const double rn = xm * nxg + ym * nyg + dRi;
      float* cell = surf + (size_t)k * spr + pi;
      const double prev = *cell;
      const double feedH = fz * sn * G.sliceKap[k];
      // Hb[(phi * binScale) | 0]: a bin past the map reads undefined, and undefined <= z
      // is false
      const double bs = phi * binScale;
      const int bin = bs == bs ? (int)bs : 0;
      const bool hbOut = bin < MCS_BINS && (double)G.Hb[bin] <= G.sliceZ[k];
      if (hbOut || sn <= 0) {
        *cell = (float)rn;
        continue;
      }
      double h = feedH + rn - prev;
      if (h <= 0) {  // tooth out of cut: the old surface survives one more feed step
        *cell = (float)(prev - feedH);
        continue;
      }
      *cell = (float)rn;
      if (h > hMax) h = hMax;
      const double se = mc != 0 ? pow(kHRef / (h > kHMin ? h : kHMin), mc) : 1.0;
      const double bk = G.sliceB[k];
      const double Ft = Ktc * se * h * bk + Kte * bk;
      double Fr = Krc * se * h * bk + Kre * bk;
      const double Fa = Kac * se * h * bk + Kae * bk;
      if (pdK != 0) Fr += pdK * (bk / G.db) / G.sliceR[k] * (rvx * nxg + rvy * nyg);
      const double txg = cs * ux - sn * vx, tyg = cs * uy - sn * vy;
      Fx += -Ft * txg - Fr * nxg;
      Fy += -Ft * tyg - Fr * nyg;
      Fz -= Fa;
      T += Ft * G.sliceR[k];
      const double fr = hypot(Ft, Fr);
      Fsum += fr;
      Fr2z += fr * (G.sliceZ[k] - G.tipZ);
      teeth |= 1u << i;
      sHb += h * bk;
      sB += bk;
      sRb += G.sliceR[k] * h * bk;
    }
    for (int e = lane; e < nend; e += 32) {
      // end edges at the tip (no helix lag): thrust, torque and in-plane tangential force
      const int i = e / kR, j = e - i * kR;
      double phi = angle_mod(theta + i * pitch);
      if (phi < 0) phi += kTwoPi;
      const int row = ((int)(phi / kTwoPi * kE)) * kR;
      // an angle of exactly 2 pi would read past the map (undefined in the reference)
      const double depth = row < kE * kR ? (double)G.Eb[row + j] : 0.0;
      if (depth > 2e-4) {
        double sn, cs;
        sincos(phi, &sn, &cs);
        const double txg = cs * ux - sn * vx, tyg = cs * uy - sn * vy;
        const double c = G.ringCos[j], ds = G.ringDs[j];
        const double h = (depth < G.fza ? depth : G.fza) * c;
        const double se = mc != 0 ? pow(kHRef / (h > kHMin ? h : kHMin), mc) : 1.0;
        const double Ft = Ktc * se * h * ds + Kte * ds;
        const double Fn = Krc * se * h * ds + Kre * ds;
        Fx += -Ft * txg;
        Fy += -Ft * tyg;
        Fz -= Fn * c;
        T += Ft * G.ringR[j];
        Fsum += Ft;
        Fr2z += Ft * G.ringZ[j];
        teeth |= 1u << i;
        sHb += h * ds;
        sB += ds;
        sRb += G.ringR[j] * h * ds;
      }
    }
    // the ring cell tooth i reads was written one tooth period earlier by the lane of tooth
    // i + 1: the warp barrier orders those global stores before the later loads
    __syncwarp();
    st.engTeeth += __popc(__reduce_or_sync(kAll, teeth));
    Fx = wsum(Fx);
    Fy = wsum(Fy);
    Fz = wsum(Fz);
    T = wsum(T);
    Fsum = wsum(Fsum);
    Fr2z = wsum(Fr2z);
    // modal integration (semi-implicit Euler), SI (:239-249)
    x = 0;
    y = 0;
    vxs = 0;
    vys = 0;
    // unrolled to the mode limit so that the modal states stay in registers
#pragma unroll
    for (int j = 0; j < MCS_MAX_MODES; j++) {
      if (j < nmx) {
        v[0][j] += (Fx - C.mcd[0][j] * v[0][j] - C.mk[0][j] * q[0][j]) / C.mm[0][j] * dt;
        q[0][j] += v[0][j] * dt;
        x += q[0][j];
        vxs += v[0][j];
      }
    }
#pragma unroll
    for (int j = 0; j < MCS_MAX_MODES; j++) {
      if (j < nmy) {
        v[1][j] += (Fy - C.mcd[1][j] * v[1][j] - C.mk[1][j] * q[1][j]) / C.mm[1][j] * dt;
        q[1][j] += v[1][j] * dt;
        y += q[1][j];
        vys += v[1][j];
      }
    }
    if (wk != 0) {  // the reaction on the wall along its normal (:250-258)
      const double Fw = -(Fx * wnx + Fy * wny);
      wv += (Fw - wc * wv - wk * w) / wm * dt;
      w += wv * dt;
      if (w > 5e-4) {
        w = 5e-4;
        if (wv > 0) wv = 0;
      } else if (w < -2e-4) {
        w = -2e-4;
        if (wv < 0) wv = 0;
      }
      st.sumW += w;
      st.maxW = fmax(st.maxW, fabs(w));
      wSum += w;
    }
    if (++pr == spr) pr = 0;
    if (pr % spt == 0) {  // once-per-tooth sample (:261-262), Float32Array
      if (lane == 0) {
        S.ts_x[ts_i] = (float)(x - w * wnx);
        S.ts_y[ts_i] = (float)(y - w * wny);
      }
      ts_i = (ts_i + 1) % kTs;
      ts_count++;
    }
    t += dt;
    const double Fxy = hypot(Fx, Fy);
    st.n += 1;
    st.sumF += Fxy;
    st.maxF = fmax(st.maxF, Fxy);
    st.sumFx += Fx;
    st.sumFy += Fy;
    st.sumFz += Fz;
    st.maxFz = fmax(st.maxFz, -Fz);
    st.sumT += T;
    st.maxT = fmax(st.maxT, T);
    st.sumX += x;
    st.sumY += y;
    st.minX = fmin(st.minX, x);
    st.maxX = fmax(st.maxX, x);
    st.minY = fmin(st.minY, y);
    st.maxY = fmax(st.maxY, y);
    if (Fsum > 0) {
      st.sumZc += Fr2z / Fsum * Fxy;
      st.wZc += Fxy;
    }
    if (++stepCount % C.decim == 0) {  // decimated history (:288-292), Float32Array
      if (lane == 0) {
        hist[0 * kH + h_i] = (float)Fx;
        hist[1 * kH + h_i] = (float)Fy;
        hist[2 * kH + h_i] = (float)Fz;
        hist[3 * kH + h_i] = (float)((x - w * wnx) * 1e6);
        hist[4 * kH + h_i] = (float)((y - w * wny) * 1e6);
      }
      h_i = (h_i + 1) % kH;
      h_count++;
    }
  }
  sHb = wsum(sHb);
  sB = wsum(sB);
  sRb = wsum(sRb);
  if (lane == 0) {
    for (int a = 0; a < 2; a++)
      for (int j = 0; j < MCS_MAX_MODES; j++) {
        S.q[a][j] = q[a][j];
        S.v[a][j] = v[a][j];
      }
    S.x = S.x0 = x;
    S.y = S.y0 = y;
    S.vx = S.vx0 = vxs;
    S.vy = S.vy0 = vys;
    S.t = t;
    S.pr = pr;
    S.w = w;
    S.wv = wv;
    S.run_mean_w = wSum / (double)n_steps;
    S.step_count = stepCount;
    S.ts_i = ts_i;
    S.ts_count = ts_count;
    S.h_i = h_i;
    S.h_count = h_count;
    st.sumHb += sHb;
    st.sumB += sB;
    st.sumRb += sRb;
    S.st = st;
  }
}

__device__ void clear_stats(mcs_engine_stats& s) {
  s = mcs_engine_stats{};
  s.minX = INFINITY;
  s.maxX = -INFINITY;
  s.minY = INFINITY;
  s.maxY = -INFINITY;
}

// what configure() resets (:51-81), and optionally the statistics (a new engine)
__global__ void engine_reset_kernel(EngState* states, int n, int fresh) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  EngState& S = states[e];
  for (int a = 0; a < 2; a++)
    for (int j = 0; j < MCS_MAX_MODES; j++) S.q[a][j] = S.v[a][j] = 0;
  S.x = S.y = S.vx = S.vy = S.x0 = S.y0 = S.vx0 = S.vy0 = S.t = 0;
  S.w = S.wv = S.run_mean_w = 0;
  S.pr = 0;
  S.step_count = 0;
  if (fresh) {
    S.ts_i = S.h_i = 0;
    S.ts_count = S.h_count = 0;
    for (int i = 0; i < kTs; i++) S.ts_x[i] = S.ts_y[i] = 0.f;
    clear_stats(S.st);
  }
}

// setWork: a rigid workpiece or a wall with a new normal starts from rest (:88-94)
__global__ void engine_wall_reset_kernel(const EngGeo* geos, EngState* states, int n) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n || !geos[e].reset_wall) return;
  states[e].w = 0;
  states[e].wv = 0;
  if (geos[e].wk == 0) states[e].run_mean_w = 0;
}

__global__ void engine_take_stats_kernel(EngState* states, int n) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) clear_stats(states[e].st);
}

__global__ void engine_set_state_kernel(EngState* states, const double* xv, int n) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  states[e].x = xv[4 * e];
  states[e].y = xv[4 * e + 1];
  states[e].vx = xv[4 * e + 2];
  states[e].vy = xv[4 * e + 3];
}

__global__ void engine_reset_history_kernel(EngState* states, int n) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  states[e].h_i = 0;
  states[e].h_count = 0;
}

struct Buf {
  void* p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes) {
    if (bytes <= cap) return MCS_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    const cudaError_t e = cudaMalloc(&p, std::max<size_t>(bytes, 256));
    if (e != cudaSuccess) {
      p = nullptr;
      return fail(e == cudaErrorMemoryAllocation ? MCS_ERR_NOMEM : MCS_ERR_CUDA,
                  "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    }
    cap = std::max<size_t>(bytes, 256);
    return MCS_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

}  // namespace
}  // namespace mcs

using namespace mcs;

struct mcs_engine {
  std::mutex mu;  // calls on one engine are serialised
  mcs_ctx* ctx = nullptr;
  size_t n = 0;
  std::vector<EngCfg> cfg;  // host copies
  std::vector<EngGeo> geo;
  Buf d_cfg, d_geo, d_state, d_surf, d_hist, d_steps, d_xv;
};

namespace {

#define ENG_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(MCS_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));        \
  } while (0)

int blocks_of(size_t n) { return (int)((n + 127) / 128); }

bool modes_valid(const mcs_modal& md) {
  if (md.nx < 1 || md.nx > MCS_MAX_MODES || md.ny < 0 || md.ny > MCS_MAX_MODES) return false;
  for (int a = 0; a < 2; a++) {
    const int cnt = a == 0 ? md.nx : md.ny;
    const mcs_mode* ms = a == 0 ? md.x : md.y;
    for (int j = 0; j < cnt; j++)
      if (!(std::isfinite(ms[j].k) && ms[j].k > 0 && std::isfinite(ms[j].fn) && ms[j].fn > 0 &&
            std::isfinite(ms[j].zeta) && ms[j].zeta >= 0))
        return false;
  }
  return true;
}

// configure() on the host (cutting.js:39-82), FP64 in the reference's order
int derive_cfg(const mcs_engine_config& c, EngCfg& E) {
  std::memset(&E, 0, sizeof(E));
  const mcs_tool& t = c.tool;
  if (t.N < 1 || t.N > MCS_MAX_TEETH) return fail(MCS_ERR_ARG, "N must be in [1, %d]", MCS_MAX_TEETH);
  if (!(std::isfinite(t.R) && t.R > 0 && std::isfinite(t.helix_deg) && std::fabs(t.helix_deg) < 89 &&
        std::isfinite(t.flute_len) && t.flute_len > 0 && std::isfinite(t.runout) &&
        std::isfinite(t.runout_phase)))
    return fail(MCS_ERR_ARG, "tool geometry invalid");
  if (!modes_valid(c.modal)) return fail(MCS_ERR_ARG, "modal set invalid");
  if (!(std::isfinite(c.S) && std::isfinite(c.fn_max) && c.fn_max >= 0 && c.decim >= 0))
    return fail(MCS_ERR_ARG, "speed, fn_max or decim invalid");
  const double coef[8] = {c.Ktc, c.Krc, c.Kac, c.Kte, c.Kre, c.Kae, c.mc, c.Ci};
  for (double v : coef)
    if (!std::isfinite(v)) return fail(MCS_ERR_ARG, "material coefficient not finite");
  E.N = t.N;
  E.R = t.R;
  E.tanB = std::tan(t.helix_deg * kPi / 180);
  for (int i = 0; i < t.N; i++) E.dR[i] = t.runout * std::cos(2 * kPi * i / t.N - t.runout_phase);
  const double S = std::max(100.0, c.S);
  E.omega = S * 2 * kPi / 60;
  const double Ttooth = 60 / (S * t.N);
  const int nx = c.modal.nx, ny = c.modal.ny > 0 ? c.modal.ny : c.modal.nx;
  const mcs_mode* xm = c.modal.x;
  const mcs_mode* ym = c.modal.ny > 0 ? c.modal.y : c.modal.x;
  double fTop = -INFINITY;
  for (int j = 0; j < nx; j++) fTop = std::max(fTop, xm[j].fn);
  for (int j = 0; j < ny; j++) fTop = std::max(fTop, ym[j].fn);
  const double spt = std::max(48.0, std::ceil(Ttooth * std::max(fTop, c.fn_max) * 24));
  if (spt * t.N > 2e6) return fail(MCS_ERR_UNSUPPORTED, "%.0f steps per revolution", spt * t.N);
  E.spt = (int)spt;
  E.dt = Ttooth / E.spt;
  E.dphi = E.omega * E.dt;
  E.pitch = kTwoPi / t.N;
  for (int a = 0; a < 2; a++) {
    const int cnt = a == 0 ? nx : ny;
    const mcs_mode* ms = a == 0 ? xm : ym;
    E.nm[a] = cnt;
    for (int j = 0; j < cnt; j++) {
      const double k = ms[j].k * 1e3;
      const double w = 2 * kPi * ms[j].fn;
      const double m = k / (w * w);
      E.mk[a][j] = k;
      E.mm[a][j] = m;
      E.mcd[a][j] = 2 * ms[j].zeta * std::sqrt(k * m);
    }
  }
  E.dz = std::max(0.25, t.flute_len / 48);
  E.max_slices = (int)std::ceil(t.flute_len / E.dz);
  if (E.max_slices > MCS_MAX_SLICES)
    return fail(MCS_ERR_UNSUPPORTED, "%d slices exceed %d", E.max_slices, MCS_MAX_SLICES);
  E.spr = t.N * E.spt;
  E.decim = c.decim > 0 ? c.decim : (int)std::max(1.0, std::floor(E.spt / 40.0 + 0.5));
  E.Ktc = c.Ktc;
  E.Krc = c.Krc;
  E.Kac = c.Kac;
  E.Kte = c.Kte;
  E.Kre = c.Kre;
  E.Kae = c.Kae;
  E.mc = c.mc;
  E.Ci = c.Ci;
  E.nonlinear = c.nonlinear ? 1 : 0;
  E.configured = 1;
  return MCS_OK;
}

// setEngagement, setEndEngagement, setWork and setWear on the host
int derive_geo(const EngCfg& C, const mcs_engagement& g, const EngGeo& prev, EngGeo& G) {
  std::memset(&G, 0, sizeof(G));
  if (!C.configured) return fail(MCS_ERR_STATE, "engagement set before configure");
  const double vals[] = {g.ux, g.uy, g.fz, g.tip_z, g.ap, g.fza, g.end_r, g.wall_k, g.wall_m,
                         g.wall_zeta, g.wall_nx, g.wall_ny, g.Kte, g.Kre};
  for (double v : vals)
    if (!std::isfinite(v)) return fail(MCS_ERR_ARG, "engagement value not finite");
  std::memcpy(G.Hb, g.Hb, sizeof(G.Hb));
  std::memcpy(G.Eb, g.Eb, sizeof(G.Eb));
  G.ux = g.ux;
  G.uy = g.uy;
  G.vx = -g.uy;
  G.vy = g.ux;
  G.fz = g.fz;
  G.tipZ = g.tip_z;
  const double ap = g.ap;
  const int nz = ap <= 0 ? 0 : std::min(C.max_slices, (int)std::ceil(ap / C.dz));
  G.nz = nz;
  G.db = C.dz;
  const double R = C.R;
  for (int k = 0; k < nz; k++) G.sliceB[k] = std::min(C.dz, ap - k * C.dz);
  for (int k = 0; k < nz; k++) {
    const double zr = k * C.dz + 0.5 * G.sliceB[k];
    G.sliceZ[k] = g.tip_z + zr;
    double r = R, kap = 1;
    if (g.profile) {  // a general edge profile: the caller's rAt radius and edge angle
      r = g.slice_r[k];
      kap = g.slice_kap[k];
      if (!(std::isfinite(r) && r > 0 && std::isfinite(kap)))
        return fail(MCS_ERR_ARG, "slice %d: profile radius or kappa invalid", k);
    }
    G.sliceR[k] = r;
    G.sliceKap[k] = kap;
    G.sliceLag[k] = zr * C.tanB / R;
  }
  // end edges (:130-143): rings at (j + 0.5) dr, the edge-normal cosine from the profile's
  // slope, capped at 0.22
  G.fza = g.fza > 0 ? g.fza : 0;
  const double dr = g.end_r / kR;
  for (int j = 0; j < kR; j++) {
    const double r = (j + 0.5) * dr;
    const double slope = (g.ring_zo[j] - g.ring_zi[j]) / (0.5 * dr);
    const double c = std::max(0.22, 1 / std::sqrt(1 + slope * slope));
    G.ringR[j] = r;
    G.ringCos[j] = c;
    G.ringDs[j] = dr / c;
    G.ringZ[j] = g.ring_z[j];
  }
  if (G.fza > 0 && !(g.end_r > 0)) return fail(MCS_ERR_ARG, "end edges need end_r > 0");
  G.Kte = g.wear ? g.Kte : C.Kte;
  G.Kre = g.wear ? g.Kre : C.Kre;
  // setWork: a rigid workpiece, or a wall whose state carries over while its normal stays
  if (g.wall_k > 0) {
    if (!(g.wall_m > 0)) return fail(MCS_ERR_ARG, "wall mass must be > 0");
    G.reset_wall = prev.wk != 0 && g.wall_nx * prev.wnx + g.wall_ny * prev.wny < 0.8;
    G.wk = g.wall_k * 1e3;
    G.wm = g.wall_m;
    G.wc = 2 * g.wall_zeta * std::sqrt(G.wk * g.wall_m);
    G.wnx = g.wall_nx;
    G.wny = g.wall_ny;
  } else {
    G.reset_wall = 1;
    G.wk = 0;
    G.wm = 1;
    G.wc = 0;
    G.wnx = 1;
    G.wny = 0;
  }
  G.set = 1;
  return MCS_OK;
}

}  // namespace

extern "C" {

int mcs_engine_create(mcs_ctx* ctx, size_t n, mcs_engine** out) {
  if (!ctx || !out) return fail(MCS_ERR_ARG, "NULL ctx or engine pointer");
  if (n < 1 || n > (1u << 20)) return fail(MCS_ERR_ARG, "engine count out of range");
  *out = nullptr;
  ENG_CUDA(cudaSetDevice(ctx_device(ctx)));
  mcs_engine* e = new mcs_engine();
  e->ctx = ctx;
  e->n = n;
  e->cfg.assign(n, EngCfg{});
  e->geo.assign(n, EngGeo{});
  int rc;
  if ((rc = e->d_cfg.ensure(sizeof(EngCfg) * n)) || (rc = e->d_geo.ensure(sizeof(EngGeo) * n)) ||
      (rc = e->d_state.ensure(sizeof(EngState) * n)) ||
      (rc = e->d_hist.ensure(sizeof(float) * 5 * kH * n)) ||
      (rc = e->d_steps.ensure(sizeof(long long) * n)) ||
      (rc = e->d_xv.ensure(sizeof(double) * 4 * n))) {
    mcs_engine_destroy(e);
    return rc;
  }
  cudaStream_t st = ctx_stream(ctx);
  cudaError_t err = cudaMemsetAsync(e->d_cfg.p, 0, sizeof(EngCfg) * n, st);
  if (err == cudaSuccess) err = cudaMemsetAsync(e->d_geo.p, 0, sizeof(EngGeo) * n, st);
  if (err == cudaSuccess) err = cudaMemsetAsync(e->d_hist.p, 0, sizeof(float) * 5 * kH * n, st);
  if (err == cudaSuccess) {
    engine_reset_kernel<<<blocks_of(n), 128, 0, st>>>(static_cast<EngState*>(e->d_state.p),
                                                      (int)n, 1);
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  if (err != cudaSuccess) {
    mcs_engine_destroy(e);
    return fail(MCS_ERR_CUDA, "engine set-up failed: %s", cudaGetErrorString(err));
  }
  *out = e;
  return MCS_OK;
}

int mcs_engine_destroy(mcs_engine* e) {
  if (!e) return MCS_OK;
  cudaSetDevice(ctx_device(e->ctx));
  cudaStreamSynchronize(ctx_stream(e->ctx));
  e->d_cfg.release();
  e->d_geo.release();
  e->d_state.release();
  e->d_surf.release();
  e->d_hist.release();
  e->d_steps.release();
  e->d_xv.release();
  delete e;
  return MCS_OK;
}

int mcs_engine_configure(mcs_engine* e, const mcs_engine_config* cfg) {
  if (!e || !cfg) return fail(MCS_ERR_ARG, "NULL engine or config");
  std::lock_guard<std::mutex> lk(e->mu);
  std::vector<EngCfg> next(e->n);
  long long off = 0;
  for (size_t i = 0; i < e->n; i++) {
    const int rc = derive_cfg(cfg[i], next[i]);
    if (rc) return fail(rc, "engine %zu: %s", i, mcs_last_error());
    next[i].surf_off = off;
    off += (long long)next[i].max_slices * next[i].spr;
  }
  ENG_CUDA(cudaSetDevice(ctx_device(e->ctx)));
  cudaStream_t st = ctx_stream(e->ctx);
  ENG_CUDA(cudaStreamSynchronize(st));  // no run may still read the old surface
  int rc = e->d_surf.ensure(sizeof(float) * (size_t)std::max<long long>(off, 1));
  if (rc) return rc;
  e->cfg = next;
  // a fresh surface, fresh modes and samples of the new set-up; the engagement is set anew
  for (EngGeo& g : e->geo) g.set = 0;
  ENG_CUDA(cudaMemcpyAsync(e->d_cfg.p, e->cfg.data(), sizeof(EngCfg) * e->n,
                           cudaMemcpyHostToDevice, st));
  ENG_CUDA(cudaMemcpyAsync(e->d_geo.p, e->geo.data(), sizeof(EngGeo) * e->n,
                           cudaMemcpyHostToDevice, st));
  ENG_CUDA(cudaMemsetAsync(e->d_surf.p, 0, sizeof(float) * (size_t)std::max<long long>(off, 1), st));
  engine_reset_kernel<<<blocks_of(e->n), 128, 0, st>>>(static_cast<EngState*>(e->d_state.p),
                                                       (int)e->n, 0);
  ENG_CUDA(cudaGetLastError());
  ENG_CUDA(cudaStreamSynchronize(st));
  return MCS_OK;
}

int mcs_engine_set_engagement(mcs_engine* e, const mcs_engagement* g) {
  if (!e || !g) return fail(MCS_ERR_ARG, "NULL engine or engagement");
  std::lock_guard<std::mutex> lk(e->mu);
  std::vector<EngGeo> next(e->n);
  for (size_t i = 0; i < e->n; i++) {
    const int rc = derive_geo(e->cfg[i], g[i], e->geo[i], next[i]);
    if (rc) return fail(rc, "engine %zu: %s", i, mcs_last_error());
  }
  ENG_CUDA(cudaSetDevice(ctx_device(e->ctx)));
  cudaStream_t st = ctx_stream(e->ctx);
  ENG_CUDA(cudaStreamSynchronize(st));  // the previous engagement is no longer read
  e->geo = next;
  ENG_CUDA(cudaMemcpyAsync(e->d_geo.p, e->geo.data(), sizeof(EngGeo) * e->n,
                           cudaMemcpyHostToDevice, st));
  engine_wall_reset_kernel<<<blocks_of(e->n), 128, 0, st>>>(
      static_cast<const EngGeo*>(e->d_geo.p), static_cast<EngState*>(e->d_state.p), (int)e->n);
  ENG_CUDA(cudaGetLastError());
  ENG_CUDA(cudaStreamSynchronize(st));
  return MCS_OK;
}

int mcs_engine_set_state(mcs_engine* e, const double* xv) {
  if (!e || !xv) return fail(MCS_ERR_ARG, "NULL engine or state");
  std::lock_guard<std::mutex> lk(e->mu);
  for (size_t i = 0; i < 4 * e->n; i++)
    if (!std::isfinite(xv[i])) return fail(MCS_ERR_ARG, "state value %zu not finite", i);
  ENG_CUDA(cudaSetDevice(ctx_device(e->ctx)));
  cudaStream_t st = ctx_stream(e->ctx);
  ENG_CUDA(cudaMemcpyAsync(e->d_xv.p, xv, sizeof(double) * 4 * e->n, cudaMemcpyHostToDevice, st));
  engine_set_state_kernel<<<blocks_of(e->n), 128, 0, st>>>(
      static_cast<EngState*>(e->d_state.p), static_cast<const double*>(e->d_xv.p), (int)e->n);
  ENG_CUDA(cudaGetLastError());
  ENG_CUDA(cudaStreamSynchronize(st));
  return MCS_OK;
}

int mcs_engine_run(mcs_engine* e, const int64_t* steps) {
  if (!e || !steps) return fail(MCS_ERR_ARG, "NULL engine or steps");
  std::lock_guard<std::mutex> lk(e->mu);
  for (size_t i = 0; i < e->n; i++) {
    if (steps[i] < 0 || steps[i] > (int64_t)1e10) return fail(MCS_ERR_ARG, "steps out of range");
    if (steps[i] > 0 && (!e->cfg[i].configured || !e->geo[i].set))
      return fail(MCS_ERR_STATE, "engine %zu runs before configure and set_engagement", i);
  }
  ENG_CUDA(cudaSetDevice(ctx_device(e->ctx)));
  cudaStream_t st = ctx_stream(e->ctx);
  ENG_CUDA(cudaMemcpyAsync(e->d_steps.p, steps, sizeof(long long) * e->n, cudaMemcpyHostToDevice,
                           st));
  engine_run_kernel<<<(unsigned)e->n, 32, 0, st>>>(
      static_cast<const EngCfg*>(e->d_cfg.p), static_cast<const EngGeo*>(e->d_geo.p),
      static_cast<EngState*>(e->d_state.p), static_cast<float*>(e->d_surf.p),
      static_cast<float*>(e->d_hist.p), static_cast<const long long*>(e->d_steps.p));
  ENG_CUDA(cudaGetLastError());
  ENG_CUDA(cudaStreamSynchronize(st));
  return MCS_OK;
}

int mcs_engine_take_stats(mcs_engine* e, mcs_engine_stats* out) {
  if (!e || !out) return fail(MCS_ERR_ARG, "NULL engine or output");
  std::lock_guard<std::mutex> lk(e->mu);
  ENG_CUDA(cudaSetDevice(ctx_device(e->ctx)));
  cudaStream_t st = ctx_stream(e->ctx);
  std::vector<EngState> s(e->n);
  ENG_CUDA(cudaMemcpyAsync(s.data(), e->d_state.p, sizeof(EngState) * e->n,
                           cudaMemcpyDeviceToHost, st));
  engine_take_stats_kernel<<<blocks_of(e->n), 128, 0, st>>>(
      static_cast<EngState*>(e->d_state.p), (int)e->n);
  ENG_CUDA(cudaGetLastError());
  ENG_CUDA(cudaStreamSynchronize(st));
  for (size_t i = 0; i < e->n; i++) out[i] = s[i].st;
  return MCS_OK;
}

int mcs_engine_get_state(mcs_engine* e, mcs_engine_state* out) {
  if (!e || !out) return fail(MCS_ERR_ARG, "NULL engine or output");
  std::lock_guard<std::mutex> lk(e->mu);
  ENG_CUDA(cudaSetDevice(ctx_device(e->ctx)));
  cudaStream_t st = ctx_stream(e->ctx);
  std::vector<EngState> s(e->n);
  ENG_CUDA(cudaMemcpyAsync(s.data(), e->d_state.p, sizeof(EngState) * e->n,
                           cudaMemcpyDeviceToHost, st));
  ENG_CUDA(cudaStreamSynchronize(st));
  for (size_t i = 0; i < e->n; i++) {
    mcs_engine_state& o = out[i];
    std::memset(&o, 0, sizeof(o));
    o.x = s[i].x;
    o.y = s[i].y;
    o.vx = s[i].vx;
    o.vy = s[i].vy;
    o.t = s[i].t;
    o.w = s[i].w;
    o.wv = s[i].wv;
    o.dt = e->cfg[i].dt;
    o.run_mean_w = s[i].run_mean_w;
    o.pr = s[i].pr;
    o.nz = e->geo[i].nz;
    o.steps_per_tooth = e->cfg[i].spt;
    o.steps_per_rev = e->cfg[i].spr;
    o.max_slices = e->cfg[i].max_slices;
    o.decim = e->cfg[i].decim;
    o.step_count = (uint64_t)s[i].step_count;
  }
  return MCS_OK;
}

int mcs_engine_history(mcs_engine* e, float* out, int32_t* head, int64_t* count) {
  if (!e || !out) return fail(MCS_ERR_ARG, "NULL engine or output");
  std::lock_guard<std::mutex> lk(e->mu);
  ENG_CUDA(cudaSetDevice(ctx_device(e->ctx)));
  cudaStream_t st = ctx_stream(e->ctx);
  std::vector<EngState> s(e->n);
  ENG_CUDA(cudaMemcpyAsync(s.data(), e->d_state.p, sizeof(EngState) * e->n,
                           cudaMemcpyDeviceToHost, st));
  ENG_CUDA(cudaMemcpyAsync(out, e->d_hist.p, sizeof(float) * 5 * kH * e->n,
                           cudaMemcpyDeviceToHost, st));
  ENG_CUDA(cudaStreamSynchronize(st));
  for (size_t i = 0; i < e->n; i++) {
    if (head) head[i] = s[i].h_i;
    if (count) count[i] = s[i].h_count;
  }
  return MCS_OK;
}

int mcs_engine_reset_history(mcs_engine* e) {
  if (!e) return fail(MCS_ERR_ARG, "NULL engine");
  std::lock_guard<std::mutex> lk(e->mu);
  ENG_CUDA(cudaSetDevice(ctx_device(e->ctx)));
  cudaStream_t st = ctx_stream(e->ctx);
  engine_reset_history_kernel<<<blocks_of(e->n), 128, 0, st>>>(
      static_cast<EngState*>(e->d_state.p), (int)e->n);
  ENG_CUDA(cudaGetLastError());
  ENG_CUDA(cudaStreamSynchronize(st));
  return MCS_OK;
}

int mcs_engine_chatter_index(mcs_engine* e, double* out) {
  if (!e || !out) return fail(MCS_ERR_ARG, "NULL engine or output");
  std::lock_guard<std::mutex> lk(e->mu);
  ENG_CUDA(cudaSetDevice(ctx_device(e->ctx)));
  cudaStream_t st = ctx_stream(e->ctx);
  std::vector<EngState> s(e->n);
  std::vector<float> h(5 * kH * e->n);
  ENG_CUDA(cudaMemcpyAsync(s.data(), e->d_state.p, sizeof(EngState) * e->n,
                           cudaMemcpyDeviceToHost, st));
  ENG_CUDA(cudaMemcpyAsync(h.data(), e->d_hist.p, sizeof(float) * h.size(),
                           cudaMemcpyDeviceToHost, st));
  ENG_CUDA(cudaStreamSynchronize(st));
  // chatterIndex() (cutting.js:299-318) on the host, in the reference's order
  for (size_t i = 0; i < e->n; i++) {
    const EngState& S = s[i];
    const float* hx = h.data() + i * 5 * kH + 3 * kH;
    const float* hy = hx + kH;
    const int n = (int)std::min<long long>(S.ts_count, 24);
    double* o = out + 3 * i;
    if (n < 8) {
      o[0] = o[1] = o[2] = 0;
      continue;
    }
    double mx = 0, my = 0;
    for (int k = 0; k < n; k++) {
      const int j = (S.ts_i - 1 - k + kTs) % kTs;
      mx += S.ts_x[j];
      my += S.ts_y[j];
    }
    mx /= n;
    my /= n;
    double v = 0;
    for (int k = 0; k < n; k++) {
      const int j = (S.ts_i - 1 - k + kTs) % kTs;
      v += (S.ts_x[j] - mx) * (S.ts_x[j] - mx) + (S.ts_y[j] - my) * (S.ts_y[j] - my);
    }
    const double sOnce = std::sqrt(v / n) * 1e6;
    const long long m = std::min<long long>(
        S.h_count, (long long)std::floor((double)n * e->cfg[i].spt / e->cfg[i].decim + 0.5));
    const double md = m ? (double)m : 1.0;
    double ax = 0, ay = 0;
    for (long long k = 0; k < m; k++) {
      const int j = (int)((S.h_i - 1 - k + kH) % kH);
      ax += hx[j];
      ay += hy[j];
    }
    ax /= md;
    ay /= md;
    double w = 0;
    for (long long k = 0; k < m; k++) {
      const int j = (int)((S.h_i - 1 - k + kH) % kH);
      w += (hx[j] - ax) * (hx[j] - ax) + (hy[j] - ay) * (hy[j] - ay);
    }
    const double sAll = std::sqrt(w / md);
    o[0] = sOnce / (sAll + 0.05);
    o[1] = sAll;
    o[2] = sOnce;
  }
  return MCS_OK;
}

}  // extern "C"
