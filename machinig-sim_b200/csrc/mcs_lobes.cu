// Zero-order (Altintas-Budak) stability lobes read at spindle speeds: stabilityLobes and
// alimAt of src/sld.js:6-76, in FP64 on the device.
//
// One CTA per lobe query.  The CTA evaluates the NS chatter-frequency samples (the
// eigenvalue of the directional-coefficient problem, sld.js:32-48) into shared memory,
// then, per lobe number j, maps every sample to its spindle speed, sorts the lobe by
// speed (bitonic sort, ties kept in sample order as the reference's stable sort does)
// and lets each thread take the minimum over lobes of the linear interpolation at its
// query speeds (alimAt).  The arithmetic follows the reference expression by expression.
#include <cuda_runtime.h>

#include <cmath>

#include "mcs_internal.h"

namespace mcs {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxNS = 1600;   // 400 * min(4, nx + ny - 1)
constexpr int kSortN = 2048;   // power of two >= kMaxNS
constexpr double kPi = 3.141592653589793;

struct Cx {
  double re, im;
};
__device__ __forceinline__ Cx cmul(Cx a, Cx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ Cx cdiv(Cx a, Cx b) {
  const double d = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
__device__ __forceinline__ Cx csqrt_ref(Cx a) {
  const double r = hypot(a.re, a.im);
  const double re = sqrt((r + a.re) / 2);
  const double s = (a.im != 0 && a.im == a.im) ? (a.im > 0 ? 1.0 : -1.0) : 1.0;
  return {re, s * sqrt(fmax(0.0, (r - a.re) / 2))};
}

// G(f) = sum 1 / (k (1 - r^2 + 2 i zeta r)) [mm/N] (frf.js:14-21)
__device__ Cx frf_dev(const mcs_mode* m, int n, double f) {
  double re = 0, im = 0;
  for (int i = 0; i < n; i++) {
    const double r = f / m[i].fn, a = 1 - r * r, b = 2 * m[i].zeta * r,
                 d = m[i].k * (a * a + b * b);
    re += a / d;
    im -= b / d;
  }
  return {re, im};
}

__device__ void dir_coeffs(double Kr, double p, double f[4]) {
  f[0] = 0.5 * (cos(2 * p) - 2 * Kr * p + Kr * sin(2 * p));
  f[1] = 0.5 * (-sin(2 * p) - 2 * p + Kr * cos(2 * p));
  f[2] = 0.5 * (-sin(2 * p) + 2 * p + Kr * cos(2 * p));
  f[3] = 0.5 * (-cos(2 * p) - 2 * Kr * p - Kr * sin(2 * p));
}

__device__ __forceinline__ bool key_less(double ka, int ia, double kb, int ib) {
  return ka < kb || (ka == kb && ia < ib);
}

// Without slices every query is read at all n_rpm speeds, out[q * n_rpm + r]; with slices
// (q_begin, q_count) query q is read only at rpm[q_begin[q] .. q_begin[q] + q_count[q]) and
// writes out[r] there (the composite diagram: each node read across its own speeds).
__global__ void __launch_bounds__(kThreads) lobes_kernel(const mcs_modal* __restrict__ modals,
                                                         const mcs_lobe_query* __restrict__ qs,
                                                         const double* __restrict__ rpm,
                                                         int n_rpm, double* __restrict__ out,
                                                         const int* __restrict__ q_begin,
                                                         const int* __restrict__ q_count) {
  extern __shared__ __align__(16) double sm[];
  double* wc = sm;
  double* al = wc + kMaxNS;
  double* psi = al + kMaxNS;
  double* key = psi + kMaxNS;
  int* kid = reinterpret_cast<int*>(key + kSortN);
  __shared__ int s_valid;

  const mcs_lobe_query Q = qs[blockIdx.x];
  const mcs_modal* M = modals + Q.modal;
  const int nx = M->nx, ny = M->ny > 0 ? M->ny : M->nx;
  const mcs_mode* xm = M->x;
  const mcs_mode* ym = M->ny > 0 ? M->y : M->x;
  double a[4], b[4];
  dir_coeffs(Q.Krc / Q.Ktc, Q.phi_ex, a);
  dir_coeffs(Q.Krc / Q.Ktc, Q.phi_st, b);
  const double axx = a[0] - b[0], axy = a[1] - b[1], ayx = a[2] - b[2], ayy = a[3] - b[3];
  const double det = axx * ayy - axy * ayx;
  double fmn = INFINITY, fmx = -INFINITY;
  for (int j = 0; j < nx; j++) fmn = fmin(fmn, xm[j].fn), fmx = fmax(fmx, xm[j].fn);
  for (int j = 0; j < ny; j++) fmn = fmin(fmn, ym[j].fn), fmx = fmax(fmx, ym[j].fn);
  const double f0 = 0.8 * fmn, f1 = 1.7 * fmx;
  const int NS = 400 * min(4, nx + ny - 1);

  // chatter frequencies: the lower positive depth of the two eigenvalue roots
  for (int s = threadIdx.x; s < NS; s += kThreads) {
    const double fc = f0 + (f1 - f0) * s / (NS - 1), w = 2 * kPi * fc;
    const Cx Px = frf_dev(xm, nx, fc), Py = frf_dev(ym, ny, fc);
    const Cx a0 = cmul(cmul(Px, Py), Cx{det, 0});
    const Cx a1 = {axx * Px.re + ayy * Py.re, axx * Px.im + ayy * Py.im};
    const Cx sq = cmul(a1, a1);
    const Cx disc = csqrt_ref(Cx{sq.re - 4 * a0.re, sq.im - 4 * a0.im});
    bool have = false;
    double bestA = 0, bestK = 0;
    for (int sg = 1; sg >= -1; sg -= 2) {
      const Cx num = {-(a1.re + sg * disc.re), -(a1.im + sg * disc.im)};
      const Cx L = cdiv(num, Cx{2 * a0.re, 2 * a0.im});
      if (L.re >= 0) continue;
      const double kap = L.im / L.re;
      const double alim = -2 * kPi * L.re * (1 + kap * kap) / (Q.N * Q.Ktc);
      if (alim > 0 && (!have || alim < bestA)) {
        have = true;
        bestA = alim;
        bestK = kap;
      }
    }
    wc[s] = w;
    al[s] = have ? bestA : -1.0;
    psi[s] = have ? atan(bestK) : 0.0;
  }
  const int r0 = q_begin ? q_begin[blockIdx.x] : 0;
  const int r1 = q_begin ? r0 + q_count[blockIdx.x] : n_rpm;
  double* outq = q_begin ? out : out + (size_t)blockIdx.x * n_rpm;
  for (int r = r0 + threadIdx.x; r < r1; r += kThreads) outq[r] = INFINITY;
  __syncthreads();

  for (int j = 0; j < Q.lobes; j++) {
    // speeds of lobe j (sld.js:49-56); samples without a root or outside the range sort last
    for (int i = threadIdx.x; i < kSortN; i += kThreads) {
      double k = INFINITY;
      if (i < NS && al[i] > 0) {
        const double eps = kPi - 2 * psi[i];
        const double T = (eps + 2 * j * kPi) / wc[i];
        const double v = 60 / (Q.N * T);
        if (v >= Q.rpm_min * 0.8 && v <= Q.rpm_max * 1.2) k = v;
      }
      key[i] = k;
      kid[i] = i;
    }
    __syncthreads();
    for (int size = 2; size <= kSortN; size <<= 1) {
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int i = threadIdx.x; i < kSortN; i += kThreads) {
          const int p = i ^ stride;
          if (p > i) {
            const bool up = (i & size) == 0;
            const bool swap = up ? key_less(key[p], kid[p], key[i], kid[i])
                                 : key_less(key[i], kid[i], key[p], kid[p]);
            if (swap) {
              const double tk = key[i];
              key[i] = key[p];
              key[p] = tk;
              const int ti = kid[i];
              kid[i] = kid[p];
              kid[p] = ti;
            }
          }
        }
        __syncthreads();
      }
    }
    if (threadIdx.x == 0) {
      int lo = 0, hi = kSortN;  // first index holding +inf
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (key[mid] < INFINITY) lo = mid + 1; else hi = mid;
      }
      s_valid = lo;
    }
    __syncthreads();
    const int n = s_valid;
    // alimAt (sld.js:64-76): every consecutive pair [a, b] with a.rpm <= rpm <= b.rpm
    for (int r = r0 + threadIdx.x; r < r1; r += kThreads) {
      const double v = rpm[r];
      int lo = 0, hi = n;  // lower bound: first key >= v
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (key[mid] < v) lo = mid + 1; else hi = mid;
      }
      const int lower = lo;
      hi = n;  // upper bound: first key > v
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (key[mid] <= v) lo = mid + 1; else hi = mid;
      }
      const int upper = lo;
      double best = outq[r];
      for (int i = max(lower, 1); i <= min(upper, n - 1); i++) {
        const double ar = key[i - 1], br = key[i];
        const double aa = al[kid[i - 1]], ba = al[kid[i]];
        const double span = br - ar;
        const double t = (v - ar) / (span != 0 ? span : 1);
        best = fmin(best, aa + (ba - aa) * t);
      }
      outq[r] = best;
    }
    __syncthreads();
  }
}

}  // namespace

constexpr int kLobeSmem = 3 * kMaxNS * 8 + kSortN * 8 + kSortN * 4;

int launch_lobes(cudaStream_t stream, const mcs_modal* modals, const mcs_lobe_query* qs, int n_q,
                 const double* rpm, int n_rpm, double* out, const int* q_begin,
                 const int* q_count) {
  cudaError_t e = cudaFuncSetAttribute(lobes_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kLobeSmem);
  if (e != cudaSuccess) return (int)e;
  if (n_q == 0) return 0;
  lobes_kernel<<<n_q, kThreads, kLobeSmem, stream>>>(modals, qs, rpm, n_rpm, out, q_begin,
                                                     q_count);
  return (int)cudaGetLastError();
}

}  // namespace mcs
