// sm_100a kernels of the time-domain chatter stability path.
//
// One warp simulates one cut (a chatterAt trial, src/stabtd.js:14-22) and, in the solve
// kernel, runs the whole bisection of timeDomainLimit (src/stabtd.js:24-32) for one
// (setup, speed) point.  Warps take points from an atomic work queue (persistent launch).
//
// Work layout inside a warp (the run() loop of src/cutting.js:168-293):
//   * lane l owns axial slices l and l + 32 (SLOTS = 1 or 2 -> nz <= 64); the slice
//     geometry (cutting.js:98-124) lives in registers for the whole trial;
//   * each lane follows its slices' own phase in the revolution and visits only the teeth
//     in cut there (predicated rounds over both slots); every in-cut lane evaluates the
//     force law (cutting.js:181-207) in FP32 (or FP64 when the caller asks for it: the
//     kernels are templated on the scalar type);
//   * Fx, Fy are summed with a butterfly of shuffles.  Linear cuts split the modal update
//     (semi-implicit Euler, cutting.js:246-255) between the half-warps, one axis each;
//     with process damping every lane integrates both axes;
//   * the once-per-tooth samples of the chatter-index window sit one per lane, and the
//     decimated-history statistics are accumulated in FP64 (cutting.js:265-292,299-318).
// A trial whose slices fit a smaller aligned group of lanes can share the warp with other
// trials of the same point: the bisection runs its next levels speculatively in lane
// groups, each of which computes exactly what a whole warp would (simulate, Groups).
//
// The delayed surface: the reference keeps surf[slice][position] for a whole revolution
// (cutting.js:62-68).  With the static arc map of chatterAt a (slice, position) cell has
// a fixed angle phi = position*dphi - lag(slice) (mod 2pi), so only the cells whose angle
// lies in the engaged bins are ever read in cut; all other cells are written and never
// read.  The ring therefore holds, per slice, only the positions of the engaged window
// (length <= (phi_hi - phi_lo)/dphi + 2), in shared memory next to a sin/cos table of the
// revolution's positions.  Whether a cell is in cut is an integer window test, so the
// engagement pattern is the one the reference's bin lookup gives (up to angles within
// ~1e-15 rad of a bin edge).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "mcs_internal.h"

// The file is compiled once per integration precision (MCS_PREC = 32 or 64), into the
// namespaces mcs::k32 and mcs::k64, so that the two halves of the template instances
// build in parallel; mcs_internal.h dispatches on KernelShape::fp64.
#ifndef MCS_PREC
#define MCS_PREC 32
#endif
#if MCS_PREC == 64
#define MCS_KNS k64
#else
#define MCS_KNS k32
#endif

namespace mcs {
namespace MCS_KNS {
#if MCS_PREC == 64
using KScalar = double;
#else
using KScalar = float;
#endif
namespace {

constexpr unsigned kFull = 0xffffffffu;
#if MCS_PREC == 32
constexpr float kLog2HRef = -4.321928094887363f;  // log2(H_REF = 0.05 mm), cutting.js:18
constexpr float kHMin = 0.002f;                    // cutting.js:19
#endif

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// Arithmetic of the integration scalar T (float or double).
template <typename T>
struct Arith;
#if MCS_PREC == 32
template <>
struct Arith<float> {
  using V2 = float2;
  static __device__ __forceinline__ float madd(float a, float b, float c) { return fmaf(a, b, c); }
  // se * h with se = (H_REF / max(h, H_MIN))^mc (cutting.js:197), MUFU log2/exp2
  static __device__ __forceinline__ float size_effect(float h, float mc) {
    return h * exp2f(mc * (kLog2HRef - __log2f(fmaxf(h, kHMin))));
  }
  static __device__ __forceinline__ float2 pair(double s, double c) {
    return make_float2((float)s, (float)c);
  }
  // the history's Float32Array sample of a position [m] in um (cutting.js:288-292): the
  // product of a float and 1e6 is exact in double, so rounding it to float gives the
  // correctly rounded float product
  static __device__ __forceinline__ float micro(float v) { return v * 1e6f; }
  // a product the compiler may not fuse into a neighbouring addition
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
};
#endif
#if MCS_PREC == 64
template <>
struct Arith<double> {
  using V2 = double2;
  static __device__ __forceinline__ double madd(double a, double b, double c) { return fma(a, b, c); }
  static __device__ __forceinline__ double size_effect(double h, double mc) {
    return h * pow(0.05 / (h > 0.002 ? h : 0.002), mc);
  }
  static __device__ __forceinline__ double2 pair(double s, double c) { return make_double2(s, c); }
  static __device__ __forceinline__ float micro(double v) { return (float)(v * 1e6); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
};
#endif

// Resident warps per SM the register allocation is held to (65536 / (32 * warps)); measured
// on the sweep, any cap below the natural allocation spills and runs slower (1 = no cap).
#ifndef MCS_MIN_WARPS_F32
#define MCS_MIN_WARPS_F32 1
#endif
#ifndef MCS_MIN_WARPS_F64
#define MCS_MIN_WARPS_F64 1
#endif
template <typename T>
struct MinWarps {
  static constexpr int value = MCS_PREC == 64 ? MCS_MIN_WARPS_F64 : MCS_MIN_WARPS_F32;
};

struct TrialOut {
  double index, once, amp;
  unsigned long long engaged, evals;
  int status;
};
static_assert(sizeof(TrialOut) == kTrialOutBytes, "shared-memory result record");

// sin/cos of every position of one revolution: theta(p) = p * dphi.
template <typename T>
__device__ __forceinline__ void build_table(const PointParams* __restrict__ P,
                                            typename Arith<T>::V2* table, int lane) {
  const int spr = P->spr;
  const double dphi = P->dphi;
  for (int p = lane; p < spr; p += kWarp) {
    double s, c;
    sincos(p * dphi, &s, &c);
    table[p] = Arith<T>::pair(s, c);
  }
  __syncwarp();
}

// Slices of a trial at depth ap (stabtd.js:16-18 -> cutting.js:63-64, 98-124), FP64; the
// same rule as the host's slices_at.
__device__ __forceinline__ void slice_rule(const PointParams* __restrict__ P, double ap,
                                           int& nz, double& dz) {
  if (P->slices_override > 0) {
    nz = ap > 0 ? P->slices_override : 0;
    dz = ap / P->slices_override;
  } else {
    const double flute = fmax(P->flute_len, ap + 1.0);
    dz = fmax(0.25, flute / 48.0);
    const int maxs = (int)ceil(flute / dz);
    nz = ap > 0 ? min(maxs, (int)ceil(ap / dz)) : 0;
  }
}

// Sum over an aligned group of gs lanes (gs a power of two).  Every lane executes the same
// five shuffles whatever its group's size (a shuffle must be reached by the whole warp); a
// lane adds what it receives only from inside its group.  With gs = 32 it is the warp
// butterfly; for a smaller group it adds in the same order as a whole warp would if the
// group's values sat at lanes 0..gs-1 and the others held 0.
template <typename T>
__device__ __forceinline__ T group_sum(T v, int gs) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const T t = __shfl_xor_sync(kFull, v, o);
    if (o < gs) v += t;
  }
  return v;
}
__device__ __forceinline__ int group_sum_int(int v, int gs) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const int t = __shfl_xor_sync(kFull, v, o);
    if (o < gs) v += t;
  }
  return v;
}
// Fx summed into the group's lower half and Fy into its upper half, in one butterfly (the
// additions of group_sum(Fx) and group_sum(Fy), so the sums are bit for bit theirs).  The
// first shuffle reads the partner in the other half of the lane's own group (a per-lane
// source lane); the others are the same for every lane, as above.
template <typename T>
__device__ __forceinline__ T group_sum_xy(T fx, T fy, bool upper, int gs, int lane) {
  T v = upper ? fy : fx;
  v += __shfl_sync(kFull, upper ? fx : fy, lane ^ (gs >> 1));
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) {
    const T t = __shfl_xor_sync(kFull, v, o);
    if (o < (gs >> 1)) v += t;
  }
  return v;
}

// The lane groups of one warp and the depth each simulates.  Groups are aligned blocks of
// a power-of-two number of lanes (>= 2) that cover the warp; a group with ap = 0 has no
// slices and its result is not used.
struct Groups {
  int n;                    // groups
  int base[kMaxGroups];     // first lane
  int size[kMaxGroups];     // lanes
  double ap[kMaxGroups];    // depth [mm]
};

// chatterAt trials (configure + setEngagement + kick + run + chatterIndex) of one point,
// one per lane group, all stepping together: the run() loop of cutting.js:146-296 in each
// group.  A group of g lanes with at most g * SLOTS slices computes exactly what a whole
// warp computes for that trial.  Results go to out[group] (shared memory); tooth samples
// are staged in samples[group][24].
// NL: size effect and process damping present (cutting.js:153-156,197,203); linear cuts
// are compiled without them.
// GR: lane groups in use; without them the single group of 32 lanes is compiled as such.
template <typename T, int SLOTS, int NM, bool NL, bool GR>
__device__ void simulate(const PointParams* __restrict__ P, const Groups& G,
                         const typename Arith<T>::V2* __restrict__ table,
                         float* __restrict__ ring, float2* __restrict__ samples,
                         TrialOut* __restrict__ out, int lane) {
  using A = Arith<T>;
  const int N = P->N, spt = P->spt, spr = P->spr, lpad = P->lpad;
  // this lane's group
  int gi = 0;
  if (GR) {
#pragma unroll
    for (int g = 1; g < kMaxGroups; g++)
      if (g < G.n && lane >= G.base[g] && lane < G.base[g] + G.size[g]) gi = g;
  }
  const int gb = GR ? G.base[gi] : 0, gs = GR ? G.size[gi] : kWarp, ll = lane - gb;
  const double ap = GR ? G.ap[gi] : G.ap[0];

  // ---- slices of this trial (stabtd.js:16-18 -> cutting.js:63-64, 98-124), FP64 ----
  int nz;
  double dz;
  slice_rule(P, ap, nz, dz);
  // process damping per slice, Ci*b/V_c (cutting.js:155-156,203)
  const double pdK = NL && P->Ci != 0.0 ? P->Ci * dz * 1e-3 / (P->omega * 1e-3) : 0.0;

  // Per slot: slice geometry, and the slot's phase in the revolution.  Tooth i of a slice
  // whose engaged window starts at position p0 is in cut when j_i = (pr + i*spt - p0) mod
  // spr < len.  With q = (pr - p0) mod spr = c*spt + r, j_i = ((c + i) mod N)*spt + r: the
  // teeth in cut at a step are those with u = (c + i) mod N < U, U = ceil((len - r)/spt),
  // so a lane visits only its own in-cut teeth, in rounds u = 0, 1, ...  The tooth of round
  // u is i = (u - c) mod N = tb + u with tb = (N - c) mod N: i < 2N, no wrap.
  T sL[SLOTS], cL[SLOTS], ktb[SLOTS], kteb[SLOTS], krb[SLOTS], kreb[SLOTS], pdc[SLOTS],
      fzk[SLOTS];
  int p0[SLOTS], len[SLOTS], base[SLOTS], tb[SLOTS], rph[SLOTS];
#pragma unroll
  for (int s = 0; s < SLOTS; s++) {
    const int k = ll + gs * s;  // slice; its ring row is the lane's own
    sL[s] = cL[s] = ktb[s] = kteb[s] = krb[s] = kreb[s] = pdc[s] = fzk[s] = T(0);
    p0[s] = 0;
    len[s] = 0;
    base[s] = (gb + k) * lpad;
    if (k < nz && !P->empty) {
      // separately rounded products and sums, as the reference evaluates them: a product
      // left to the compiler may or may not be fused into the addition next to it, and two
      // kernels that inline this code could then disagree in the last bit
      const double kdz = __dmul_rn((double)k, dz);
      const double b = fmin(dz, __dsub_rn(ap, kdz));
      const double zr = __dadd_rn(kdz, __dmul_rn(0.5, b));
      double r = P->R, kap = 1.0;
      if (P->type == MCS_TOOL_BALL && zr < P->R) {
        const double d = P->R - zr;
        r = sqrt(fmax(1e-6, __dsub_rn(__dmul_rn(P->R, P->R), __dmul_rn(d, d))));
        kap = r / P->R;
      }
      const double lag = zr * P->tanB / P->R;
      double sl, cl;
      sincos(lag, &sl, &cl);
      sL[s] = (T)sl;
      cL[s] = (T)cl;
      // positions p whose angle p*dphi - lag (mod 2pi) falls in [phi_lo, phi_hi)
      const double u = (P->phi_lo + lag) / P->dphi;
      const double w = (P->phi_hi + lag) / P->dphi;
      double cu = ceil(u);
      double L = ceil(w) - cu;
      if (P->excl_zero && u == cu) {  // phi == 0 has sin(phi) <= 0: out of cut
        cu += 1.0;
        L -= 1.0;
      }
      long long pc = (long long)cu % spr;
      if (pc < 0) pc += spr;
      p0[s] = (int)pc;
      len[s] = (int)fmin(fmax(L, 0.0), (double)lpad);
      ktb[s] = (T)(P->Ktc * b);
      kteb[s] = (T)(P->Kte * b);
      krb[s] = (T)(P->Krc * b);
      kreb[s] = (T)(P->Kre * b);
      if (NL) pdc[s] = (T)(pdK * (b / dz) / r);
      fzk[s] = (T)(P->fz * kap);
    }
    const int q = (spr - p0[s]) % spr;  // phase at pr = 0
    const int c = q / spt;
    rph[s] = q - c * spt;
    tb[s] = c == 0 ? 0 : N - c;
  }
  // a fresh engine's surface is all zeros (cutting.js:68): the trial's rows
  if (GR) {
#pragma unroll
    for (int s = 0; s < SLOTS; s++)
      if (ll + gs * s < nz)
        for (int j = 0; j < lpad; j++) ring[base[s] + j] = 0.f;
  } else {
    for (int i = lane; i < nz * lpad; i += kWarp) ring[i] = 0.f;
  }
  __syncwarp();
  // rounds that can hold an in-cut tooth: j = u*spt + r < len needs u < ceil(len / spt)
  int maxlen = 0;
#pragma unroll
  for (int s = 0; s < SLOTS; s++) maxlen = max(maxlen, len[s]);
  const int rounds = min(N, (__reduce_max_sync(kFull, (unsigned)maxlen) + spt - 1) / spt);

  // lane i < 2N holds the runout offset of tooth i mod N (read by shuffle; N <= 8)
  const T dRl = lane < 2 * N ? (T)P->dR[lane < N ? lane : lane - N] : T(0);
  // Modal state.  Linear cuts split it: the group's lower half integrates the x modes and
  // its upper half the y modes (row 0 holds this half's axis), which halves the update and
  // the force sum at the price of a broadcast of x and y on the step's critical path.  With
  // process damping the tool velocity would need a broadcast too; there every lane
  // integrates both axes (rows 0 and 1), which measured faster.
  constexpr bool kSplit = !NL;
  const bool upper = ll >= (gs >> 1);
  T mk[2][NM], mcd[2][NM], ma[2][NM], q[2][NM], v[2][NM];
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int j = 0; j < NM; j++) {
      const int src = kSplit ? (upper ? 1 : 0) : a;
      mk[a][j] = (T)P->mk[src][j];
      mcd[a][j] = (T)P->mcd[src][j];
      ma[a][j] = (T)P->ma[src][j];
      q[a][j] = T(0);
      v[a][j] = T(0);
    }
  // the kick e.vx = 0.01 m/s goes into the first x mode at the first run (cutting.js:164)
  if (!kSplit || !upper) v[0][0] = T(0.01);
  T x = T(0), y = T(0), vxs = T(0.01), vys = T(0);

  const T hmax = (T)P->hmax, mc = (T)P->mc, dt = (T)P->dt;
  const bool size_effect = NL && P->mc != 0.0;
  const bool pd = NL && pdK != 0.0;
  const int nsteps = P->nsteps, decim = P->decim, ts_c0 = P->ts_c0, h0 = P->hist_h0;
  const int n_ts = P->ts_n;
  int phc = 0, dcnt = 0, tcount = 0, hcount = 0, eng = 0;
  double sh = 0.0;  // first history sample in the window of this lane's axis
  float tsx = 0.f, tsy = 0.f;  // without groups lane t keeps tooth sample t
  // FP64 sums of the history window.  Without groups one per lane of lanes 0-3: sum dx,
  // sum dy, sum dx^2, sum dy^2.  In lane groups (as small as 2 lanes) two per lane of the
  // group's first two: sum d and sum d^2 of x (lane 0) and of y (lane 1), the same
  // additions in the same order.
  double acc = 0.0, acc2 = 0.0;

  for (int step = 0; step < nsteps; step++) {
    const T xm = x * T(1e3), ym = y * T(1e3);  // tool position [mm]
    T Fx = T(0), Fy = T(0);
    // rounds u = 0, 1, ...: in each, every lane evaluates, for each of its slots, the tooth
    // whose window offset is u*spt + r (if in cut); both slots' evaluations are
    // predicated, not branched, so their dependency chains interleave
    for (int u = 0; u < rounds; u++) {
      int jj[SLOTS];
      bool act[SLOTS];
      bool any = false;
#pragma unroll
      for (int s = 0; s < SLOTS; s++) {
        jj[s] = u * spt + rph[s];
        act[s] = jj[s] < len[s];
        any |= act[s];
      }
      if (!__any_sync(kFull, any)) break;  // rounds are monotone: later ones are empty too
#pragma unroll
      for (int s = 0; s < SLOTS; s++) {
        const T dRi = __shfl_sync(kFull, dRl, tb[s] + u);  // u < rounds <= N
        // idle lanes (no in-cut tooth this round, or a slice past nz whose ring row is not
        // this trial's) read a valid table entry, take their surface word from the table
        // (read-only here; the value is discarded) and never write the ring
        const int j = act[s] ? jj[s] : 0;
        int p = p0[s] + j;  // table position of tooth i at this step (p0 < spr, j < spr)
        if (p >= spr) p -= spr;
        const typename A::V2 sc = table[p];
        // phi = p*dphi - lag: rotate the table entry by the slice's helix lag
        const T sn = A::madd(sc.x, cL[s], -sc.y * sL[s]);
        const T cs = A::madd(sc.y, cL[s], sc.x * sL[s]);
        // feed u = [1, 0]: edge normal n = (sin phi, cos phi), tangent t = (cos, -sin)
        const T rn = A::madd(xm, sn, A::madd(ym, cs, dRi));
        float* cell = ring + base[s] + j;
        const float* src = act[s] ? cell : reinterpret_cast<const float*>(table);
        const T prev = (T)*src;
        const T feedH = A::mul(fzk[s], sn);  // not fused into the sums below
        T h = (feedH + rn) - prev;
        const bool cut = h > T(0);
        // out of cut the old surface survives one more feed step (cutting.js:193)
        if (act[s]) *cell = (float)(cut ? rn : prev - feedH);
        if (h > hmax) h = hmax;  // (a NaN chip stays NaN, as in the reference)
        const T kse = size_effect ? A::size_effect(h, mc) : h;  // se * h
        const T Ft = A::madd(ktb[s], kse, kteb[s]);
        T Fr = A::madd(krb[s], kse, kreb[s]);
        if (pd) Fr = A::madd(pdc[s], A::madd(vxs, sn, vys * cs), Fr);
        const bool on = act[s] && cut;
        Fx = on ? A::madd(-Ft, cs, A::madd(-Fr, sn, Fx)) : Fx;
        Fy = on ? A::madd(Ft, sn, A::madd(-Fr, cs, Fy)) : Fy;
        eng += on ? 1 : 0;
      }
    }
    // modal integration, semi-implicit Euler; padded modes have k = c = dt/m = 0
    if (kSplit) {
      // this half's force (Fx in the lower half, Fy in the upper) drives this half's axis
      const T F = group_sum_xy(Fx, Fy, upper, gs, lane);
      T qs = T(0);
#pragma unroll
      for (int j = 0; j < NM; j++) {
        v[0][j] = A::madd(A::madd(-mcd[0][j], v[0][j], A::madd(-mk[0][j], q[0][j], F)),
                          ma[0][j], v[0][j]);
        q[0][j] = A::madd(v[0][j], dt, q[0][j]);
        qs += q[0][j];
      }
      x = __shfl_sync(kFull, qs, gb);
      y = __shfl_sync(kFull, qs, gb + (gs >> 1));
    } else {
      Fx = group_sum(Fx, gs);
      Fy = group_sum(Fy, gs);
      T xs = T(0), ys = T(0), vxa = T(0), vya = T(0);
#pragma unroll
      for (int j = 0; j < NM; j++) {
        v[0][j] = A::madd(A::madd(-mcd[0][j], v[0][j], A::madd(-mk[0][j], q[0][j], Fx)),
                          ma[0][j], v[0][j]);
        q[0][j] = A::madd(v[0][j], dt, q[0][j]);
        xs += q[0][j];
        vxa += v[0][j];
        v[1][j] = A::madd(A::madd(-mcd[1][j], v[1][j], A::madd(-mk[1][j], q[1][j], Fy)),
                          ma[1][j], v[1][j]);
        q[1][j] = A::madd(v[1][j], dt, q[1][j]);
        ys += q[1][j];
        vya += v[1][j];
      }
      x = xs;
      y = ys;
      vxs = vxa;
      vys = vya;
    }
    // the revolution advances one position: every slot's phase follows
#pragma unroll
    for (int s = 0; s < SLOTS; s++) {
      if (++rph[s] == spt) {  // c advances, so tb = (N - c) mod N goes back
        rph[s] = 0;
        tb[s] = tb[s] == 0 ? N - 1 : tb[s] - 1;
      }
    }
    if (++phc == spt) {  // once-per-tooth sample (cutting.js:266-268), Float32Array
      phc = 0;
      const int t = tcount - ts_c0;
      if (GR) {
        if (ll == 0 && t >= 0 && t < n_ts)
          samples[gi * kToothSamples + t] = make_float2((float)x, (float)y);
      } else if (t == lane) {
        tsx = (float)x;
        tsy = (float)y;
      }
      tcount++;
    }
    if (++dcnt == decim) {  // decimated history (cutting.js:288-292), FP64 window sums
      dcnt = 0;
      if (hcount >= h0) {
        // lane bit 0 picks the axis: x on even lanes, y on odd ones
        const double hv = (double)A::micro((ll & 1) ? y : x);
        if (hcount == h0) sh = hv;
        const double d = hv - sh;
        if (GR) {
          acc = acc + d;
          acc2 = fma(d, d, acc2);
        } else {
          acc = (ll & 2) ? fma(d, d, acc) : acc + d;
        }
      }
      hcount++;
    }
  }

  // ---- chatterIndex (cutting.js:299-318) in FP64, one group after the other ----
  const int eng_g = group_sum_int(eng, gs);
  const bool fin = isfinite((double)x) && isfinite((double)y);
  __syncwarp();  // the samples are in shared memory
#pragma unroll 1
  for (int g = 0; g < (GR ? G.n : 1); g++) {
    const int b0 = GR ? G.base[g] : 0;
    TrialOut res;
    res.engaged = (unsigned long long)__shfl_sync(kFull, eng_g, b0);
    const int nz_g = __shfl_sync(kFull, nz, b0);
    res.evals = (unsigned long long)nsteps * (unsigned long long)(N * nz_g);
    const double sx = __shfl_sync(kFull, acc, b0), sy = __shfl_sync(kFull, acc, b0 + 1);
    const double sxx = __shfl_sync(kFull, GR ? acc2 : acc, GR ? b0 : b0 + 2),
                 syy = __shfl_sync(kFull, GR ? acc2 : acc, GR ? b0 + 1 : b0 + 3);
    const int n = n_ts;
    if (n < 8) {
      res.index = 0.0;
      res.once = 0.0;
      res.amp = 0.0;
    } else {
      const bool mine = lane < n;
      const float2 ts = !mine ? make_float2(0.f, 0.f)
                        : GR ? samples[g * kToothSamples + lane] : make_float2(tsx, tsy);
      const double tx = mine ? (double)ts.x : 0.0, ty = mine ? (double)ts.y : 0.0;
      const double mx = warp_sum(tx) / n, my = warp_sum(ty) / n;
      const double ex = mine ? (double)ts.x - mx : 0.0, ey = mine ? (double)ts.y - my : 0.0;
      const double vv = warp_sum(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)));
      const double once = sqrt(vv / n) * 1e6;
      const double md = P->hist_m ? (double)P->hist_m : 1.0;
      double w = (sxx - sx * sx / md) + (syy - sy * sy / md);
      if (w < 0.0) w = 0.0;  // rounding of the one-pass form; a NaN (run-away cut) stays NaN
      const double amp = sqrt(w / md);
      res.once = once;
      res.amp = amp;
      res.index = once / (amp + 0.05);
    }
    const bool fin_g = __shfl_sync(kFull, fin ? 1 : 0, b0) != 0;
    res.status = (fin_g && isfinite(res.index)) ? MCS_OK : MCS_ERR_DIVERGED;
    if (lane == 0) out[g] = res;
  }
  __syncwarp();
}

// A single group: the whole warp simulates depth ap.
__device__ __forceinline__ void one_group(Groups& G, double ap) {
  G.n = 1;
  G.base[0] = 0;
  G.size[0] = kWarp;
  G.ap[0] = ap;
#pragma unroll
  for (int g = 1; g < kMaxGroups; g++) {
    G.base[g] = kWarp;
    G.size[g] = 0;
    G.ap[g] = 0.0;
  }
}

// A failed packing leaves the single whole-warp group (depth 0; the caller sets it).
__device__ __forceinline__ bool unpacked(Groups& G) {
  one_group(G, 0.0);
  return false;
}

// Lane groups for the trials at depths ap[0..n-1] of one point (group g = trial g): a
// group has the next power of two >= its slice count lanes (at least 2: the split modal
// update and the history sums need two), placed first-fit at an aligned offset; the lanes
// left over form groups without slices.  False, with G reset to the single whole-warp
// group, when the trials do not fit in one warp.
__device__ __forceinline__ bool pack_groups(const PointParams* __restrict__ P, const double* ap,
                                            int n, Groups& G) {
  if (n > kMaxGroups) return unpacked(G);
  unsigned used = 0u;
  for (int t = 0; t < n; t++) {
    int nz;
    double dz;
    slice_rule(P, ap[t], nz, dz);
    int sz = 2;
    while (sz < nz) sz <<= 1;
    if (sz > kWarp) return unpacked(G);
    const unsigned mask = sz == kWarp ? 0xffffffffu : ((1u << sz) - 1u);
    int off = -1;
    for (int o = 0; o < kWarp; o += sz)
      if ((used & (mask << o)) == 0u) {
        off = o;
        break;
      }
    if (off < 0) return unpacked(G);
    used |= mask << off;
    G.base[t] = off;
    G.size[t] = sz;
    G.ap[t] = ap[t];
  }
  int ng = n;
  for (int sz = 16; sz >= 2; sz >>= 1)  // cover the free lanes with empty groups
    for (int o = 0; o < kWarp; o += sz) {
      const unsigned mask = (1u << sz) - 1u;
      if ((used & (mask << o)) == 0u) {
        if (ng >= kMaxGroups) return unpacked(G);
        used |= mask << o;
        G.base[ng] = o;
        G.size[ng] = sz;
        G.ap[ng] = 0.0;
        ng++;
      }
    }
  for (int g = ng; g < kMaxGroups; g++) {
    G.base[g] = kWarp;
    G.size[g] = 0;
    G.ap[g] = 0.0;
  }
  G.n = ng;
  return true;
}

// The midpoints of the first d levels of a bisection of [lo, hi] in breadth-first order:
// node k brackets [L_k, H_k] and has midpoint m_k = sqrt(L_k * H_k); its left child (chatter
// at m_k) brackets [L_k, m_k], its right child [m_k, H_k] -- the square roots the serial
// bisection takes on every path.
__device__ __forceinline__ void tree_midpoints(double lo, double hi, int d, double* m) {
  double L[15], H[15];
  L[0] = lo;
  H[0] = hi;
  m[0] = sqrt(lo * hi);
  for (int k = 0; 2 * k + 2 < (1 << d) - 1; k++) {
    L[2 * k + 1] = L[k];
    H[2 * k + 1] = m[k];
    m[2 * k + 1] = sqrt(L[k] * m[k]);
    L[2 * k + 2] = m[k];
    H[2 * k + 2] = H[k];
    m[2 * k + 2] = sqrt(m[k] * H[k]);
  }
}

// The lanes a trial at depth ap takes in a lane group (pack_groups' rule).
__device__ __forceinline__ int group_lanes(const PointParams* __restrict__ P, double ap) {
  int nz;
  double dz;
  slice_rule(P, ap, nz, dz);
  int sz = 2;
  while (sz < nz) sz <<= 1;
  return sz;
}

// First fit of an aligned block of sz lanes into the used mask, and the number of empty
// groups that then cover the free lanes: the packing of pack_groups, one trial at a time.
__device__ __forceinline__ bool fit_block(unsigned& used, int sz, int trials) {
  if (sz > kWarp) return false;
  const unsigned mask = sz == kWarp ? 0xffffffffu : ((1u << sz) - 1u);
  int off = -1;
  for (int o = 0; o < kWarp; o += sz)
    if ((used & (mask << o)) == 0u) {
      off = o;
      break;
    }
  if (off < 0) return false;
  unsigned u = used | (mask << off);
  int ng = trials;
  for (int s = 16; s >= 2; s >>= 1)
    for (int o = 0; o < kWarp; o += s) {
      const unsigned m = (1u << s) - 1u;
      if ((u & (m << o)) == 0u) {
        u |= m << o;
        ng++;
      }
    }
  if (ng > kMaxGroups) return false;
  used |= mask << off;
  return true;
}

// Where the next bisection levels are expected to go: with a surrogate, a normal
// distribution of the log critical depth (mean mu, standard deviation sigma); without one
// every log depth of [a_min, a_max] alike, so that a node counts by its bracket's width.
struct Prior {
  bool normal;
  double mu, inv_sigma;
};

// Probability weight of the node bracketing [l, h]: the brackets touching a_min or a_max
// take the mass beyond them too.
__device__ __forceinline__ double node_weight(const Prior& pr, double l, double h,
                                              double a_min, double a_max) {
  if (!pr.normal) return log(h / l);
  const double a = l <= a_min ? -INFINITY : (log(l) - pr.mu) * pr.inv_sigma;
  const double b = h >= a_max ? INFINITY : (log(h) - pr.mu) * pr.inv_sigma;
  return normcdf(b) - normcdf(a);
}

// The trials of one speculative round: nodes of the remaining bisection tree of [lo, hi],
// node 0 the next midpoint, chosen best first by their weight under the prior while their
// lane groups fit in the warp.  A node's children are candidates once it is chosen, and a
// child never outweighs its parent, so the chosen nodes form a subtree containing node 0;
// kid[k][0] is the node taken when node k chatters (the bracket [l, m]), kid[k][1] the one
// taken when it is stable, -1 where the round's walk stops.  The midpoints are the square
// roots the serial bisection takes, so the walk decides exactly what one trial at a time
// would.  n = 0: even node 0 needs more than the warp's lanes.
struct SpecPlan {
  int n;
  double m[kMaxGroups];
  signed char kid[kMaxGroups][2];
};

__device__ __noinline__ void plan_round(const PointParams* __restrict__ P, double lo, double hi,
                                        int levels, const Prior& pr, double a_min,
                                        double a_max, SpecPlan& sp) {
  constexpr int kCand = 2 * kMaxGroups + 1;
  double cl[kCand], ch[kCand], cw[kCand];
  signed char cpar[kCand], cside[kCand], cdep[kCand];
  bool alive[kCand];
  int nc = 1;
  cl[0] = lo;
  ch[0] = hi;
  cw[0] = 1.0;
  cpar[0] = -1;
  cside[0] = 0;
  cdep[0] = 0;
  alive[0] = true;
  sp.n = 0;
  unsigned used = 0u;
  for (;;) {
    int best = -1;
    for (int c = 0; c < nc; c++)
      if (alive[c] && (best < 0 || cw[c] > cw[best])) best = c;
    if (best < 0 || sp.n >= kMaxGroups) break;
    alive[best] = false;
    const double l = cl[best], h = ch[best], m = sqrt(l * h);
    if (!fit_block(used, group_lanes(P, m), sp.n + 1)) {
      if (sp.n == 0) break;  // node 0 does not fit: one trial on the whole warp
      continue;
    }
    const int k = sp.n++;
    sp.m[k] = m;
    sp.kid[k][0] = sp.kid[k][1] = -1;
    if (cpar[best] >= 0) sp.kid[cpar[best]][cside[best]] = (signed char)k;
    if (cdep[best] + 1 < levels && nc + 2 <= kCand) {
      for (int s = 0; s < 2; s++) {
        cl[nc] = s == 0 ? l : m;
        ch[nc] = s == 0 ? m : h;
        cw[nc] = node_weight(pr, cl[nc], ch[nc], a_min, a_max);
        cpar[nc] = (signed char)k;
        cside[nc] = (signed char)s;
        cdep[nc] = (signed char)(cdep[best] + 1);
        alive[nc] = true;
        nc++;
      }
    }
  }
}

// One trial on the whole warp.
template <typename T, int SLOTS, int NM, bool NL>
__device__ __forceinline__ TrialOut simulate_trial(const PointParams* __restrict__ P,
                                                   double ap,
                                                   const typename Arith<T>::V2* __restrict__ table,
                                                   float* __restrict__ ring, float2* samples,
                                                   TrialOut* out, int lane) {
  Groups G;
  one_group(G, ap);
  simulate<T, SLOTS, NM, NL, false>(P, G, table, ring, samples, out, lane);
  return out[0];
}

// The buckets of a plan run as a chain of programmatic dependent launches on one stream.
// chain_start: this block is resident, so the next bucket's kernel may launch once every
// block of this one has said so (a no-op when nothing is chained behind).  chain_end:
// block 0 waits, before it exits, for the previous bucket's kernel to complete, so the
// completion of the last bucket implies that of all; the previous kernel's blocks are all
// resident by then and depend on nothing later, so the wait ends (a no-op for the first).
__device__ __forceinline__ void chain_start() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void chain_end() {
  if (blockIdx.x == 0) asm volatile("griddepcontrol.wait;" ::: "memory");
}

__device__ __forceinline__ bool read_cancel(const volatile int* cancel, int lane) {
  int c = 0;
  if (cancel != nullptr && lane == 0) c = *cancel;
  return __shfl_sync(kFull, c, 0) != 0;
}

// Persistent solve: each warp takes points from the queue and runs timeDomainLimit.
// MINW: resident warps per SM the register allocation is held to.  The default leaves it
// to the compiler; kDenseWarps is the variant the host picks for FP64 linear buckets whose
// shared memory lets more warps reside than the default's registers do (a few spilled
// words, a slower warp, more of them: see the host's bucket placement).
#if MCS_PREC == 64
constexpr int kDenseWarps = 12;
#endif
template <typename T, int SLOTS, int NM, bool NL, bool GR, int MINW = MinWarps<T>::value>
__global__ void __launch_bounds__(kWarp, MINW) solve_kernel(const PointParams* __restrict__ pts,
                                                      const int32_t* __restrict__ order, int n,
                                                      DevOpts o, mcs_result* __restrict__ out,
                                                      unsigned int* __restrict__ queue,
                                                      const volatile int* cancel,
                                                      unsigned int* progress, GuideArgs g) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x;
  chain_start();
  for (;;) {
    unsigned int w = 0;
    if (lane == 0) w = atomicAdd(queue, 1u);
    w = __shfl_sync(kFull, w, 0);
    if (w >= (unsigned)n) break;
    const int pi = order[w];
    const PointParams* P = pts + pi;
    auto* table = reinterpret_cast<typename Arith<T>::V2*>(smem);
    float* ring = reinterpret_cast<float*>(smem + table_bytes(P->spr, sizeof(T) == 8));
    unsigned char* extra =
        smem + extra_offset(P->spr, sizeof(T) == 8, P->ring_rows, P->lpad);
    float2* samples = reinterpret_cast<float2*>(extra);
    TrialOut* outs = reinterpret_cast<TrialOut*>(extra + P->groups * kToothSamples * 8);
    mcs_result r;
    r.status = MCS_OK;
    r.trials = 0;
    r.evals = 0;
    r.engaged = 0;
    r.steps_per_tooth = P->spt;
    r.open = 0;
    r.alim = r.lo = r.hi = 0.0;
    if (read_cancel(cancel, lane)) {
      r.status = MCS_ERR_CANCELLED;
    } else {
      build_table<T>(P, table, lane);
      // a trial on the decision path: its counters join the point's, and its decision
      auto account = [&](const TrialOut& t) -> bool {
        r.trials++;
        r.evals += t.evals;
        r.engaged += t.engaged;
        if (t.status != MCS_OK) r.status = t.status;
        return t.index > o.chatter_idx;
      };
      // timeDomainLimit (stabtd.js:24-32) as a state machine of rounds around ONE call of
      // the trial code (inlined once).  A round is one trial on the whole warp, or several
      // trials of this point in lane groups: the next bisection levels run speculatively
      // (nodes of the remaining bisection tree, chosen by plan_round, whose midpoints are
      // the same square roots the serial bisection takes), and only the trials on the
      // decision path are counted, so the results are those of one trial at a time.  The
      // states: the plain first trial at a_max, then either the plain geometric bisection
      // over [a_min, a_max] (with a speculating guide: for g.levels levels, its rounds
      // spent where the prediction puts the limit) or, with a bracket guide, the bracket
      // exp(mu -+ hw) kept inside [a_min, a_max], verified at its upper (chatter) and
      // lower (stable) end and refined by the same bisection.  A failed verification
      // falls back to the plain bisection, whose a_max trial has already run.
      enum : int { kTop, kGuideHi, kGuideLo, kBisect, kDone };
      const bool speculate = g.guide != nullptr && g.mode == MCS_GUIDE_SPECULATE;
      const bool guided = g.guide != nullptr && (speculate || g.guide[pi].y >= 0.f);
      const bool can_group = GR && P->groups > 1;
      int path = guided ? MCS_PATH_GUIDED : MCS_PATH_DIRECT;
      // where the speculative rounds look: the prediction when there is one (either guide
      // method, every bisection of the point: the plain fallback and the direct path too),
      // else the bracket widths
      Prior prior;
      prior.normal = g.guide != nullptr && g.sigma != nullptr;
      prior.mu = prior.normal ? (double)g.guide[pi].x : 0.0;
      prior.inv_sigma = prior.normal ? 1.0 / fmax((double)g.sigma[pi], 1e-3) : 0.0;
      SpecPlan sp;
      sp.n = 0;
      int state = kTop, it = 0, iters = o.iters, nrounds = 0;
      double lo = o.a_min, hi = o.a_max, glo = 0.0, ghi = 0.0;
      // enter the bisection of [l, h] for n iterations
      auto bisect = [&](double l, double h, int nit) {
        lo = l;
        hi = h;
        it = 0;
        iters = nit;
        state = kBisect;
      };
      auto fallback = [&]() {
        path = MCS_PATH_FALLBACK;
        bisect(o.a_min, o.a_max, o.iters);
      };
      // enough halvings that the final bracket is no wider than a hw_min bracket's after
      // `refine` halvings
      auto refine_iters = [&]() {
        int nit = g.refine;
        for (double w = log(ghi / glo) * 0.5; w > 1.0000001 * (double)g.hw_min; w *= 0.5) nit++;
        return nit;
      };
      auto refine = [&]() { bisect(glo, ghi, refine_iters()); };
      // the speculating guide: the plain bisection for `levels` levels, its rounds steered
      // by N(mu, sigma) of the log depth
      auto speculate_from = [&]() { bisect(o.a_min, o.a_max, min(g.levels, o.iters)); };
      // a point the inference marked (predicted stable at a_max with a probability below
      // skip_top) starts at the bisection: its first trial at a_max is skipped
      if (speculate && g.guide[pi].y < -1.5f) speculate_from();
      while (state != kDone) {
        // ---- plan the round ----
        Groups G;
        one_group(G, 0.0);
        bool packed = false;  // guide check: the lower end (and spec refinement levels) too
        int spec = 0;
        if (state == kBisect) {
          if (it >= iters) {
            r.alim = sqrt(lo * hi);
            r.lo = lo;
            r.hi = hi;
            state = kDone;
            break;
          }
          if (path != MCS_PATH_GUIDED && read_cancel(cancel, lane)) {
            r.status = MCS_ERR_CANCELLED;
            r.alim = sqrt(lo * hi);
            r.lo = lo;
            r.hi = hi;
            break;
          }
          // the next midpoint and, in lane groups beside it, the further nodes of the
          // remaining tree the prior weighs most (the same first-fit packing accepts them)
          sp.n = 0;
          if (can_group && iters - it >= 2) {
            plan_round(P, lo, hi, iters - it, prior, o.a_min, o.a_max, sp);
            if (sp.n < 2 || !pack_groups(P, sp.m, sp.n, G)) sp.n = 0;
          }
          if (sp.n == 0) G.ap[0] = sqrt(lo * hi);
        } else if (state == kTop) {
          G.ap[0] = o.a_max;
        } else if (state == kGuideHi) {
          // the checks of both ends and, speculatively, the first levels of the refinement
          // that follows when both pass, in one round
          if (can_group) {
            double aps[2 + 7];
            int k0 = 0;
            aps[k0++] = ghi;
            if (glo > o.a_min) aps[k0++] = glo;
            for (int d = min(3, refine_iters()); d >= 0 && !packed; d--) {
              if (d > 0) tree_midpoints(glo, ghi, d, aps + k0);
              const int nt = k0 + (1 << d) - 1;
              if (nt > 1 && pack_groups(P, aps, nt, G)) {
                packed = true;
                spec = d;
              }
            }
          }
          if (!packed) G.ap[0] = ghi;
        } else {  // kGuideLo
          G.ap[0] = glo;
        }
        // ---- run ----
        simulate<T, SLOTS, NM, NL, GR>(P, G, table, ring, samples, outs, lane);
        nrounds++;
        // ---- decide ----
        if (state == kBisect) {
          // walk the decision path through the round's nodes: node k's midpoint is the
          // serial bisection's sqrt(lo*hi) at that point of the path
          int node = 0;
          do {
            const double mid = sqrt(lo * hi);
            const bool c = account(outs[node]);
            if (c)
              hi = mid;
            else
              lo = mid;
            it++;
            node = sp.n == 0 ? -1 : sp.kid[node][c ? 0 : 1];
          } while (node >= 0 && it < iters);
        } else if (state == kTop) {
          const bool c = account(outs[0]);
          if (!c) {
            r.alim = o.a_max;
            r.lo = o.a_max;
            r.hi = INFINITY;
            r.open = 1;
            if (guided) path = MCS_PATH_OPEN;
            state = kDone;
          } else if (!guided) {
            bisect(o.a_min, o.a_max, o.iters);
          } else if (speculate) {
            speculate_from();
          } else {
            const float2 gd = g.guide[pi];
            const double hw = (double)gd.y;
            glo = exp((double)gd.x - hw);
            ghi = exp((double)gd.x + hw);
            if (glo < o.a_min) {  // shift up to start at a_min
              glo = o.a_min;
              ghi = fmin(fmax(ghi, o.a_min * exp(2.0 * hw)), o.a_max);
            }
            if (ghi > o.a_max) {  // shift down to end at a_max
              ghi = o.a_max;
              glo = fmax(fmin(glo, o.a_max * exp(-2.0 * hw)), o.a_min);
            }
            if (!(glo < ghi))
              fallback();
            else if (ghi < o.a_max)  // a_max is known to chatter
              state = kGuideHi;
            else if (glo > o.a_min)  // a_min is taken as stable, as the plain method does
              state = kGuideLo;
            else
              refine();
          }
        } else if (state == kGuideHi) {
          const bool lo_chk = glo > o.a_min;
          if (!account(outs[0])) {
            fallback();
          } else if (lo_chk && !packed) {
            state = kGuideLo;
          } else if (lo_chk && account(outs[1])) {
            fallback();
          } else {
            refine();
            // the refinement levels this round ran speculatively, in order
            const int k0 = lo_chk ? 2 : 1;
            int node = 0;
            for (int d = 0; d < spec; d++) {
              const double mid = sqrt(lo * hi);
              const bool c = account(outs[k0 + node]);
              if (c)
                hi = mid;
              else
                lo = mid;
              it++;
              node = 2 * node + (c ? 1 : 2);
            }
          }
        } else {  // kGuideLo
          if (account(outs[0]))
            fallback();
          else
            refine();
        }
      }
      if (g.info != nullptr && lane == 0) {
        mcs_guide_info gi;
        gi.mu = g.guide ? g.guide[pi].x : 0.f;
        gi.sigma = g.sigma ? g.sigma[pi] : 0.f;
        gi.path = path;
        gi.rounds = nrounds;
        g.info[pi] = gi;
      }
    }
    if (lane == 0) {
      out[pi] = r;
      if (progress != nullptr) atomicAdd(progress, 1u);
    }
    __syncwarp();
  }
  chain_end();
}

// Speculative multi-warp bisection: the W = blockDim / 32 warps of a block share one
// point's timeDomainLimit (stabtd.js:24-32).  A round runs the midpoints of the next
// bisection levels, one trial per warp; the first round also runs the a_max probe beside
// the first levels of [a_min, a_max].  A point's serial chain of iters + 1 trials becomes
// about 1 + iters / log2(W + 1) rounds, which shortens the latency tail of the slowest
// points on a GPU that has SMs to spare for them.  The midpoints are the same square roots
// the serial bisection takes and only the trials on the decision path are counted, so the
// results are those of one trial at a time.  Every warp runs the plain whole-warp trial
// (the same code as the one-warp kernel) with its own surface ring; the sin/cos table is
// shared.  All warps keep the same bracket state, decided from the round's results in
// shared memory, and meet at block barriers, which every thread of the block reaches on
// every round: the number of rounds is a function of that shared state.
constexpr int kCoopMaxWarps = 8;
static_assert(kCoopMaxWarps == kCoopMaxWarpsHost, "multi-warp block width");

template <typename T, int SLOTS, int NM, bool NL>
__global__ void __launch_bounds__(kCoopMaxWarps * kWarp) solve_coop_kernel(
    const PointParams* __restrict__ pts, const int32_t* __restrict__ order, int n, DevOpts o,
    mcs_result* __restrict__ out, unsigned int* __restrict__ queue, const volatile int* cancel,
    unsigned int* progress) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ unsigned int s_item;
  __shared__ int s_cancel;
  const int lane = threadIdx.x & (kWarp - 1), warp = threadIdx.x / kWarp;
  const int W = blockDim.x / kWarp;
  // levels a round decides: the first beside the a_max probe (1 + 2^dtop - 1 <= W trials),
  // the later ones alone (2^dbis - 1 <= W trials); W = 1 is the serial bisection
  int dtop = 0, dbis = 1;
  while ((2 << dtop) <= W) dtop++;
  while ((2 << dbis) - 1 <= W) dbis++;
  chain_start();
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(queue, 1u);
    __syncthreads();
    const unsigned int w = s_item;
    if (w >= (unsigned)n) break;
    const int pi = order[w];
    const PointParams* P = pts + pi;
    const bool fp64 = sizeof(T) == 8;
    auto* table = reinterpret_cast<typename Arith<T>::V2*>(smem);
    const int ring_bytes = coop_ring_bytes(P->ring_rows, P->lpad);
    float* ring = reinterpret_cast<float*>(smem + table_bytes(P->spr, fp64) + warp * ring_bytes);
    TrialOut* outs = reinterpret_cast<TrialOut*>(smem + table_bytes(P->spr, fp64) +
                                                 W * ring_bytes);
    mcs_result r;
    r.status = MCS_OK;
    r.trials = 0;
    r.evals = 0;
    r.engaged = 0;
    r.steps_per_tooth = P->spt;
    r.open = 0;
    r.alim = r.lo = r.hi = 0.0;
    // the cancel flag, read once per round by one thread so that every warp sees the same
    auto cancelled = [&]() -> bool {
      if (threadIdx.x == 0) s_cancel = (cancel != nullptr && *cancel != 0) ? 1 : 0;
      __syncthreads();
      const bool c = s_cancel != 0;
      __syncthreads();
      return c;
    };
    if (cancelled()) {
      r.status = MCS_ERR_CANCELLED;
    } else {
      // the revolution's sin/cos table, built by the whole block
      const double dphi = P->dphi;
      for (int p = threadIdx.x; p < P->spr; p += blockDim.x) {
        double sv, cv;
        sincos(p * dphi, &sv, &cv);
        table[p] = Arith<T>::pair(sv, cv);
      }
      __syncthreads();
      auto account = [&](const TrialOut& t) -> bool {
        r.trials++;
        r.evals += t.evals;
        r.engaged += t.engaged;
        if (t.status != MCS_OK) r.status = t.status;
        return t.index > o.chatter_idx;
      };
      double lo = o.a_min, hi = o.a_max;
      int it = 0;
      bool top = true;
      for (;;) {
        // ---- plan the round (identical in every thread) ----
        double ap[kCoopMaxWarps];
        int k0 = 0, lv;
        if (top) {
          ap[k0++] = o.a_max;
          lv = min(dtop, o.iters);
        } else {
          if (it >= o.iters) {
            r.alim = sqrt(lo * hi);
            r.lo = lo;
            r.hi = hi;
            break;
          }
          if (cancelled()) {
            r.status = MCS_ERR_CANCELLED;
            r.alim = sqrt(lo * hi);
            r.lo = lo;
            r.hi = hi;
            break;
          }
          lv = min(dbis, o.iters - it);
        }
        if (lv > 0) tree_midpoints(lo, hi, lv, ap + k0);
        const int nt = k0 + (lv > 0 ? (1 << lv) - 1 : 0);
        // ---- run: one trial per warp ----
        if (warp < nt) {
          Groups G;
          one_group(G, ap[warp]);
          simulate<T, SLOTS, NM, NL, false>(P, G, table, ring, nullptr, outs + warp, lane);
        }
        __syncthreads();
        // ---- decide: the serial bisection's steps, in its order ----
        bool done = false;
        if (top) {
          top = false;
          if (!account(outs[0])) {
            r.alim = o.a_max;
            r.lo = o.a_max;
            r.hi = INFINITY;
            r.open = 1;
            done = true;
          }
        }
        if (!done) {
          int node = 0;
          for (int l = 0; l < lv; l++) {
            const double mid = sqrt(lo * hi);
            const bool c = account(outs[k0 + node]);
            if (c)
              hi = mid;
            else
              lo = mid;
            it++;
            node = 2 * node + (c ? 1 : 2);
          }
        }
        __syncthreads();  // the round's results are read before the next round writes
        if (done) break;
      }
    }
    if (threadIdx.x == 0) {
      out[pi] = r;
      if (progress != nullptr) atomicAdd(progress, 1u);
    }
    __syncthreads();
  }
  chain_end();
}

// Batch of independent chatterAt trials (decision replay at given depths).
template <typename T, int SLOTS, int NM, bool NL>
__global__ void __launch_bounds__(kWarp, MinWarps<T>::value) trials_kernel(const PointParams* __restrict__ pts,
                                                       const TrialItem* __restrict__ items,
                                                       int n, double chatter_idx,
                                                       mcs_trial_result* __restrict__ out,
                                                       unsigned int* __restrict__ queue) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x;
  chain_start();
  for (;;) {
    unsigned int w = 0;
    if (lane == 0) w = atomicAdd(queue, 1u);
    w = __shfl_sync(kFull, w, 0);
    if (w >= (unsigned)n) break;
    const TrialItem it = items[w];
    const PointParams* P = pts + it.point;
    auto* table = reinterpret_cast<typename Arith<T>::V2*>(smem);
    float* ring = reinterpret_cast<float*>(smem + table_bytes(P->spr, sizeof(T) == 8));
    int nz;
    double dz;
    slice_rule(P, it.ap, nz, dz);  // this item's shared memory holds nz ring rows
    unsigned char* extra = smem + extra_offset(P->spr, sizeof(T) == 8, nz, P->lpad);
    float2* samples = reinterpret_cast<float2*>(extra);
    TrialOut* outs = reinterpret_cast<TrialOut*>(extra + kToothSamples * 8);
    build_table<T>(P, table, lane);
    const TrialOut t = simulate_trial<T, SLOTS, NM, NL>(P, it.ap, table, ring, samples, outs, lane);
    if (lane == 0) {
      mcs_trial_result r;
      r.index = t.index;
      r.once = t.once;
      r.amp = t.amp;
      r.chatter = t.index > chatter_idx ? 1 : 0;
      r.status = t.status;
      out[it.out] = r;
    }
    __syncwarp();
  }
  chain_end();
}

template <typename T, int SLOTS, int NM>
void* solve_fn(bool nl, bool gr, bool dense) {
#if MCS_PREC == 64
  if (dense && !nl && !gr)
    return reinterpret_cast<void*>(&solve_kernel<T, SLOTS, NM, false, false, kDenseWarps>);
#endif
  if (dense) return nullptr;
  if (gr)
    return nl ? reinterpret_cast<void*>(&solve_kernel<T, SLOTS, NM, true, true>)
              : reinterpret_cast<void*>(&solve_kernel<T, SLOTS, NM, false, true>);
  return nl ? reinterpret_cast<void*>(&solve_kernel<T, SLOTS, NM, true, false>)
            : reinterpret_cast<void*>(&solve_kernel<T, SLOTS, NM, false, false>);
}
template <typename T, int SLOTS, int NM>
void* coop_fn(bool nl) {
  return nl ? reinterpret_cast<void*>(&solve_coop_kernel<T, SLOTS, NM, true>)
            : reinterpret_cast<void*>(&solve_coop_kernel<T, SLOTS, NM, false>);
}
template <typename T, int SLOTS, int NM>
void* trials_fn(bool nl) {
  return nl ? reinterpret_cast<void*>(&trials_kernel<T, SLOTS, NM, true>)
            : reinterpret_cast<void*>(&trials_kernel<T, SLOTS, NM, false>);
}

// The kernel of a shape in this file's precision (the caller dispatches on s.fp64).
void* pick(bool solve, const KernelShape& s) {
  if (s.fp64 != (MCS_PREC == 64 ? 1 : 0)) return nullptr;
#define MCS_PICK(SL, NMV)                                                              \
  if (s.slots == SL && s.modes == NMV)                                                 \
    return !solve ? trials_fn<KScalar, SL, NMV>(s.nl)                                  \
                  : s.coop > 0 ? coop_fn<KScalar, SL, NMV>(s.nl)                       \
                               : solve_fn<KScalar, SL, NMV>(s.nl, s.grouped, s.dense);
  MCS_PICK(1, 1)
  MCS_PICK(1, 2)
  MCS_PICK(1, 3)
  MCS_PICK(1, 4)
  MCS_PICK(2, 1)
  MCS_PICK(2, 2)
  MCS_PICK(2, 3)
  MCS_PICK(2, 4)
#undef MCS_PICK
  return nullptr;
}

}  // namespace

int set_smem_limits() {
  const int fp = MCS_PREC == 64 ? 1 : 0;
  for (int nl = 0; nl < 2; nl++)
  for (int sl = 1; sl <= kMaxSlots; sl++)
    for (int nm = 1; nm <= kMaxModes; nm++)
      for (int k = 0; k < 5; k++) {  // solve, grouped solve, trials, multi-warp, dense solve
        KernelShape ks{sl, nm, fp, nl, k == 1 ? 1 : 0};
        if (k == 3) ks.coop = kCoopMaxWarps;
        if (k == 4) {
          if (!fp || nl) continue;  // the dense variant: FP64 linear solves only
          ks.dense = 1;
        }
        void* f = pick(k != 2, ks);
        if (!f) return (int)cudaErrorInvalidValue;
        cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             k == 3 ? kCoopSmemLimit : kMaxSmemPerWarp);
        if (e != cudaSuccess) return (int)e;
        e = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return (int)e;
      }
  return 0;
}

int occupancy_solve(const KernelShape& shape, int smem, int* blocks_per_sm) {
  void* f = pick(true, shape);
  if (!f) return (int)cudaErrorInvalidValue;
  const int threads = kWarp * (shape.coop > 0 ? shape.coop : 1);
  return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, f, threads, smem);
}

int occupancy_trials(const KernelShape& shape, int smem, int* blocks_per_sm) {
  void* f = pick(false, shape);
  if (!f) return (int)cudaErrorInvalidValue;
  return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, f, kWarp, smem);
}

// Blocks of `warps` warps (one unless multi-warp) with a scheduling priority (lower value =
// scheduled first).  A chained
// launch is a programmatic dependent launch: it may start once every block of the
// stream's previous kernel has started (chain_start), so the buckets of a plan take the
// SMs in the order they are launched, longest points first.
int launch_with_priority(void* f, int grid, int smem, cudaStream_t stream, void** args,
                         int priority, bool chained, int warps = 1) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kWarp * warps);
  cfg.dynamicSmemBytes = (size_t)smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributePriority;
  attr[0].val.priority = priority;
  attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = chained ? 2 : 1;
  return (int)cudaLaunchKernelExC(&cfg, f, args);
}

int launch_solve(const KernelShape& shape, int grid, int smem, cudaStream_t stream,
                 const PointParams* pts, const int32_t* order, int n, DevOpts opts,
                 mcs_result* out, unsigned int* queue, const volatile int* cancel,
                 unsigned int* progress, const GuideArgs& guide, int priority, bool chained) {
  void* f = pick(true, shape);
  if (!f) return (int)cudaErrorInvalidValue;
  if (shape.coop > 0) {  // multi-warp bisection: plain points only
    if (shape.coop > kCoopMaxWarps || guide.guide != nullptr || smem > kCoopSmemLimit)
      return (int)cudaErrorInvalidValue;
    void* args[] = {&pts, &order, &n, &opts, &out, &queue, &cancel, &progress};
    return launch_with_priority(f, grid, smem, stream, args, priority, chained, shape.coop);
  }
  GuideArgs g = guide;
  void* args[] = {&pts, &order, &n, &opts, &out, &queue, &cancel, &progress, &g};
  return launch_with_priority(f, grid, smem, stream, args, priority, chained);
}

int launch_trials(const KernelShape& shape, int grid, int smem, cudaStream_t stream,
                  const PointParams* pts, const TrialItem* items, int n, double chatter_idx,
                  mcs_trial_result* out, unsigned int* queue, int priority, bool chained) {
  void* f = pick(false, shape);
  if (!f) return (int)cudaErrorInvalidValue;
  void* args[] = {&pts, &items, &n, &chatter_idx, &out, &queue};
  return launch_with_priority(f, grid, smem, stream, args, priority, chained);
}

}  // namespace MCS_KNS
}  // namespace mcs
