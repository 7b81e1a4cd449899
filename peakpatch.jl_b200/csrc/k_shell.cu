// k_shell.cu — per-peak radial-shell collapse measurement (analyse_peak).
//
// Reference: src/HaloFinder/RadialShell.jl:282-891 (analyse_peak) with its
// helpers hRinteg (:100-127), atab4 (:133-155), kernel_strain (:228-277),
// get_evals (:217-222) and the collapse-table lookup
// (src/EllipsoidalCollapse/CollapseTable.jl:128-145).
//
// Design (one warp per peak, persistent grid, peaks taken from a queue in
// list order, i.e. largest filter radius first):
//  1. Gather.  Lane l owns shell m = base + l of a group of 32 consecutive
//     shells (shell m >= 2 holds the cells with the (m-1)-th distinct r^2 of
//     the sorted cell list; shell 1 is the peak cell).  A lane walks its own
//     shell's cells, reading one 32-byte record per cell from the packed
//     field array, so no cross-lane reduction is needed.  Sums are either
//     compensated single precision (two-sum, error-free per addend; the
//     optimised path) or double precision (the plain path); in both cases
//     the addends are the single-precision products the reference forms
//     (Float32 field times Int32 offset).
//  2. Adaptive truncation (optimised path only).  After each group the warp
//     extends the cumulative profile Fbar and stops as soon as every shell
//     the collapse walk can read has been gathered.  Every index used below
//     the gather is bounded by rad <= rad[M] + 2 (+ one shell) with
//     M = max(crossing shell, first shell beyond ir2min, Rf window), because
//     kernel_strain's weight vanishes for |rad[mp] - rad[m1]| >= 2 and the
//     walk only moves inward from the crossing; the one exception (no
//     crossing at all) gathers every shell.  A device-side guard counts any
//     read past the gathered range (it must stay 0; the host fails loudly).
//  3. Collapse walk in double precision.  kernel_strain(mp) only depends on
//     the shells with (rad[mp] - rad[m1])^2 < 4 (the reference's running
//     mlow/mupp always bracket that set), so the walk steps are independent:
//     each lane evaluates one step (window sum, eigenvalues, table lookup)
//     and a ballot finds the first step that collapses, 31 steps per round.
//     The window weights hRinteg/(u12-u0^2)^2 depend only on the radii and
//     come from a host table.  The ten zvir_half radii run on ten lanes.
#include "ppb_internal.h"

namespace ppb {

namespace {

constexpr int NV = 20;   // profile values per shell
enum { PV_FBAR = 0, PV_N = 1, PV_S = 2, PV_S2 = 5, PV_G = 8, PV_GF = 11, PV_Q = 14 };
constexpr int NACC = 19; // gather accumulators: F, S3, S2_3, G3, Gf3, Q6 (xx yy zz xy xz yz)
// shells a warp keeps in shared memory (peaks needing more move their
// profile to global scratch), and the per-warp shared-memory footprint:
// the profile plus the chunk-partial table of the gather
constexpr int SMEM_SHELLS = 80;
constexpr int SMEM_WARP_DOUBLES = NV * (SMEM_SHELLS + 1) + (NACC + 1) * 32;
constexpr unsigned FULL = 0xffffffffu;

// counters layout
enum { CNT_VISITS = 0, CNT_PREMASK = 1, CNT_NOFCRIT = 2, CNT_M0ONE = 3, CNT_NOCOLL = 4, CNT_RTHLNEG = 5,
       CNT_GUARD = 6, CNT_AKK = 7, CNT_BADPEAK = 8, CNT_WALK = 9 };

// ---------------------------------------------------------------------------
// accumulators
// ---------------------------------------------------------------------------
template <bool COMP> struct Acc;

template <> struct Acc<true> {       // compensated single precision
  float s[NACC], c[NACC];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int i = 0; i < NACC; i++) { s[i] = 0.f; c[i] = 0.f; }
  }
  __device__ __forceinline__ void add(int i, float x) {
    // two-sum (Knuth): t + e == s + x exactly
    const float t = __fadd_rn(s[i], x);
    const float bp = __fsub_rn(t, s[i]);
    const float e = __fadd_rn(__fsub_rn(s[i], __fsub_rn(t, bp)), __fsub_rn(x, bp));
    s[i] = t;
    c[i] = __fadd_rn(c[i], e);
  }
  __device__ __forceinline__ double get(int i) const { return (double)s[i] + (double)c[i]; }
};

template <> struct Acc<false> {      // double precision (the reference's Float64 sums)
  double s[NACC];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int i = 0; i < NACC; i++) s[i] = 0.0;
  }
  __device__ __forceinline__ void add(int i, float x) { s[i] = __dadd_rn(s[i], (double)x); }
  __device__ __forceinline__ double get(int i) const { return s[i]; }
};

template <bool COMP>
__device__ __forceinline__ void accumulate_cell(Acc<COMP>& A, const float4 a, const float4 b, float di,
                                                float dj, float dk) {
  // a = (delta, deltaT, psi_x, psi_y), b = (psi_z, psi2_x, psi2_y, psi2_z)
  A.add(0, a.x);
  A.add(1, a.z); A.add(2, a.w); A.add(3, b.x);
  A.add(4, b.y); A.add(5, b.z); A.add(6, b.w);
  A.add(7, __fmul_rn(a.x, di)); A.add(8, __fmul_rn(a.x, dj)); A.add(9, __fmul_rn(a.x, dk));
  A.add(10, __fmul_rn(a.y, di)); A.add(11, __fmul_rn(a.y, dj)); A.add(12, __fmul_rn(a.y, dk));
  A.add(13, __fmul_rn(a.z, di)); A.add(14, __fmul_rn(a.w, dj)); A.add(15, __fmul_rn(b.x, dk));
  A.add(16, __fmul_rn(a.z, dj)); A.add(16, __fmul_rn(a.w, di));
  A.add(17, __fmul_rn(a.z, dk)); A.add(17, __fmul_rn(b.x, di));
  A.add(18, __fmul_rn(a.w, dk)); A.add(18, __fmul_rn(b.x, dj));
}

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}
__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL, v, o));
  return v;
}

// Symmetric 3x3 eigenvalues, ascending: the trigonometric solution of the
// characteristic cubic (O. K. Smith, "Eigenvalues of a symmetric 3 x 3
// matrix", Comm. ACM 4 (1961) 168).  m = (xx, yy, zz, xy, xz, yz).
__device__ __noinline__ void eig3(const double* m, double* lam) {
  const double a00 = m[0], a11 = m[1], a22 = m[2], a01 = m[3], a02 = m[4], a12 = m[5];
  const double p1 = a01 * a01 + a02 * a02 + a12 * a12;
  double e1, e2, e3;
  if (p1 == 0.0) {
    e1 = a00; e2 = a11; e3 = a22;
  } else {
    const double q = (a00 + a11 + a22) / 3.0;
    const double b00 = a00 - q, b11 = a11 - q, b22 = a22 - q;
    const double p = sqrt((b00 * b00 + b11 * b11 + b22 * b22 + 2.0 * p1) / 6.0);
    const double ip = 1.0 / p;
    const double c00 = b00 * ip, c11 = b11 * ip, c22 = b22 * ip, c01 = a01 * ip, c02 = a02 * ip, c12 = a12 * ip;
    double r = 0.5 * (c00 * (c11 * c22 - c12 * c12) - c01 * (c01 * c22 - c12 * c02) + c02 * (c01 * c12 - c11 * c02));
    r = r < -1.0 ? -1.0 : (r > 1.0 ? 1.0 : r);
    const double phi = acos(r) / 3.0;
    e1 = q + 2.0 * p * cos(phi);
    e3 = q + 2.0 * p * cos(phi + 2.0943951023931957);   // + 2 pi / 3
    e2 = 3.0 * q - e1 - e3;
  }
  double t;
  if (e1 > e2) { t = e1; e1 = e2; e2 = t; }
  if (e2 > e3) { t = e2; e2 = e3; e3 = t; }
  if (e1 > e2) { t = e1; e1 = e2; e2 = t; }
  lam[0] = e1; lam[1] = e2; lam[2] = e3;
}

// trilinear lookup, outside the box -> -1 (CollapseTable.jl:128-145)
__device__ __noinline__ double tab_interp(const DevTable& T, double x, double y, double z) {
  if (!(x >= T.x1 && x <= T.x2 && y >= T.y1 && y <= T.y2 && z >= T.z1 && z <= T.z2)) return -1.0;
  const double px = (x - T.x1) / ((T.x2 - T.x1) / (T.nx - 1));
  const double py = (y - T.y1) / ((T.y2 - T.y1) / (T.ny - 1));
  const double pz = (z - T.z1) / ((T.z2 - T.z1) / (T.nz - 1));
  int ix = (int)floor(px), iy = (int)floor(py), iz = (int)floor(pz);
  ix = ix < 0 ? 0 : (ix > T.nx - 2 ? T.nx - 2 : ix);
  iy = iy < 0 ? 0 : (iy > T.ny - 2 ? T.ny - 2 : iy);
  iz = iz < 0 ? 0 : (iz > T.nz - 2 ? T.nz - 2 : iz);
  const double wx = px - ix, wy = py - iy, wz = pz - iz;
  const float* b = T.t + ix + (int64_t)T.nx * (iy + (int64_t)T.ny * iz);
  const int64_t sy = T.nx, sz = (int64_t)T.nx * T.ny;
  const double c00 = (1 - wx) * (double)__ldg(b) + wx * (double)__ldg(b + 1);
  const double c10 = (1 - wx) * (double)__ldg(b + sy) + wx * (double)__ldg(b + sy + 1);
  const double c01 = (1 - wx) * (double)__ldg(b + sz) + wx * (double)__ldg(b + sz + 1);
  const double c11 = (1 - wx) * (double)__ldg(b + sz + sy) + wx * (double)__ldg(b + sz + sy + 1);
  const double c0 = (1 - wy) * c00 + wy * c10;
  const double c1 = (1 - wy) * c01 + wy * c11;
  return (1 - wz) * c0 + wz * c1;
}

// ---------------------------------------------------------------------------
// per-warp radial profile: value v of shell m at p[v*MS + m].  It lives in
// the warp's shared-memory slice while the peak needs at most `cap` shells
// and moves to the warp's global scratch slot when the gather grows beyond.
// ---------------------------------------------------------------------------
struct Prof {
  double* p;
  int MS;
  int mdone;                        // shells 1..mdone are valid
  unsigned long long* counters;
  int cap;                          // largest shell index the current storage holds
  double* global;                   // the warp's scratch slot
  int MS_global;
  __device__ __forceinline__ double get(int v, int m) const {
    if (m > mdone) {                // never taken when the truncation rule holds
      atomicAdd(counters + CNT_GUARD, 1ull);
      return 0.0;
    }
    return p[(int64_t)v * MS + m];
  }
  __device__ __forceinline__ void set(int v, int m, double x) { p[(int64_t)v * MS + m] = x; }
  // copy shells 1..upto to global scratch and continue there (whole warp)
  __device__ void spill(int upto) {
    const int lane = threadIdx.x & 31;
    for (int v = 0; v < NV; v++)
      for (int m = 1 + lane; m <= upto; m += 32) global[(int64_t)v * MS_global + m] = p[v * MS + m];
    __syncwarp();
    p = global;
    MS = MS_global;
    cap = 1 << 30;
  }
};

struct KS {
  double E[6];   // xx yy zz xy xz yz
  double g[3], gf[3];
};

struct Walk {                       // one evaluated walk step
  KS k;
  double Fh, ev, pv, Fr, zv;
};

// kernel_strain (RadialShell.jl:228-277) for centre shell mp over m1 in
// [lo, hi].  For mp > 1 only the shells with (rad[mp]-rad[m1])^2 < 4
// contribute (the table window); for mp == 1 the SPH table weights apply to
// every m1 of [lo, hi].  The warp is split into aligned groups of G lanes
// (G a power of two); each group evaluates its own mp (mp < 1: no work), its
// lanes striding over m1, and the group's partial sums are combined with a
// butterfly, leaving the result in every lane of the group.  Every lane of
// the warp must call it.
__device__ __noinline__ void ks_multi(const Prof& P, const ShellArgs& a, int mp, int lo, int hi, int G,
                                      double wRnor, double aRnor, KS* out) {
  const int lane = threadIdx.x & 31;
  const int sub = lane & (G - 1);
  double E[6] = {0, 0, 0, 0, 0, 0}, g[3] = {0, 0, 0}, gf[3] = {0, 0, 0};
  double scale = 0.0;
  if (mp >= 1) {
    const double* w;
    if (mp > 1) {
      const int wl = a.win_lo[mp], wh = a.win_hi[mp];
      lo = max(lo, wl);
      hi = min(hi, wh);
      w = a.wts + a.win_off[mp] - wl;
      scale = wRnor / a.rad[mp];
    } else {
      w = a.w1;
      scale = aRnor;
    }
    if (hi > P.mdone) {                 // never taken when the truncation rule holds
      atomicAdd(P.counters + CNT_GUARD, 1ull);
      hi = P.mdone;
    }
    const double* pg = P.p + PV_G * P.MS;
    const double* pf = P.p + PV_GF * P.MS;
    const double* pq = P.p + PV_Q * P.MS;
    const int MS = P.MS;
    for (int m1 = lo + sub; m1 <= hi; m1 += G) {
      const double wt = w[m1];
      if (mp == 1 && isnan(wt)) atomicAdd(P.counters + CNT_AKK, 1ull);
#pragma unroll
      for (int L = 0; L < 3; L++) {
        g[L] += wt * pg[L * MS + m1];
        gf[L] += wt * pf[L * MS + m1];
      }
#pragma unroll
      for (int q = 0; q < 6; q++) E[q] -= 0.5 * wt * pq[q * MS + m1];
    }
  }
  for (int o = G >> 1; o > 0; o >>= 1) {
#pragma unroll
    for (int q = 0; q < 6; q++) E[q] += __shfl_xor_sync(FULL, E[q], o);
#pragma unroll
    for (int L = 0; L < 3; L++) {
      g[L] += __shfl_xor_sync(FULL, g[L], o);
      gf[L] += __shfl_xor_sync(FULL, gf[L], o);
    }
  }
  KS r;
#pragma unroll
  for (int q = 0; q < 6; q++) r.E[q] = E[q] * scale;
#pragma unroll
  for (int L = 0; L < 3; L++) {
    r.g[L] = g[L] * scale;
    r.gf[L] = gf[L] * scale;
  }
  *out = r;
}

// eigen-decomposition -> (trace, e_v, p_v) as the reference (:571-577)
__device__ __forceinline__ void ev_pv(const double E[6], double* Frho, double* ev, double* pv) {
  double lam[3];
  eig3(E, lam);
  const double F = lam[0] + lam[1] + lam[2];
  *Frho = F;
  *ev = 0.0;
  *pv = 0.0;
  if (F > 0.0) {
    *ev = 0.5 * (lam[2] - lam[0]) / F;
    *pv = 0.5 * (lam[2] + lam[0] - 2.0 * lam[1]) / F;
  }
}

__device__ __forceinline__ double zvir_of(const DevTable& T, double Fr, double ev, double pv) {
  if (!(Fr > 0.0)) return -1.0;
  const double poe = ev < 1e-5 ? 0.0 : pv / ev;
  return tab_interp(T, log10(Fr), ev, poe);
}

__device__ __forceinline__ KS shfl_ks(const KS& k, int src) {
  KS r;
#pragma unroll
  for (int q = 0; q < 6; q++) r.E[q] = __shfl_sync(FULL, k.E[q], src);
#pragma unroll
  for (int L = 0; L < 3; L++) {
    r.g[L] = __shfl_sync(FULL, k.g[L], src);
    r.gf[L] = __shfl_sync(FULL, k.gf[L], src);
  }
  return r;
}

// ---------------------------------------------------------------------------
// geometry helpers over rad[] (increasing for m >= 1)
// ---------------------------------------------------------------------------
// smallest m in [lo, hi] with rad[m] > x, or hi+1
__device__ __forceinline__ int first_gt(const double* rad, int lo, int hi, double x) {
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    if (rad[mid] > x) hi = mid - 1; else lo = mid + 1;
  }
  return lo;
}
// largest m in [lo, hi] with rad[m] < x, or lo-1
__device__ __forceinline__ int last_lt(const double* rad, int lo, int hi, double x) {
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    if (rad[mid] < x) lo = mid + 1; else hi = mid - 1;
  }
  return hi;
}

__device__ __forceinline__ void write_no_collapse(double* o) {
  const int lane = threadIdx.x & 31;
  if (lane < RES_N) o[lane] = (lane == 0 || lane == 26) ? -1.0 : 0.0;
}

// ---------------------------------------------------------------------------
// the per-peak body
// ---------------------------------------------------------------------------
template <bool COMP, bool ADAPTIVE>
__device__ void analyse_one(const ShellArgs& a, int64_t p, double* prof_base, double* smem) {
  const int lane = threadIdx.x & 31;
  const int n = a.n;
  const int64_t n2 = (int64_t)n * n;
  const int64_t lin = a.pk.lin[p];
  double* out = a.out + p * RES_N;
  const double ZZon = a.pk.ZZon[p];
  if (lin < 0 || lin >= n2 * n || !(ZZon > -1.0)) {   // invalid peak index or redshift from the caller
    if (lane == 0) atomicAdd(a.counters + CNT_BADPEAK, 1ull);
    write_no_collapse(out);
    return;
  }
  const int pk = (int)(lin / n2), pj = (int)((lin / n) % n), pi = (int)(lin % n);
  const double Rf = a.pk.Rf[p];
  const int ir2min = a.pk.ir2min[p];
  const double fcrit = a.pk.fcrit[p];
  const double alatt = a.alatt;
  const double* __restrict__ rad = a.rad;
  const int mmax = a.mmax;

  Prof P{smem, SMEM_SHELLS + 1, 0, a.counters, SMEM_SHELLS, prof_base, a.nshell + 1};
  double* part = smem + NV * (SMEM_SHELLS + 1);   // chunk partials [value][lane]

  // ---- geometry that depends only on the shell radii --------------------
  // m0 of the gather loop (RadialShell.jl:392-399): first finalised shell with
  // r^2 > ir2min, else the last finalised shell.
  int m0_init;
  {
    int lo = 2, hi = mmax;
    while (lo <= hi) {
      const int mid = (lo + hi) >> 1;
      if (a.r2m[mid] > ir2min) hi = mid - 1; else lo = mid + 1;
    }
    m0_init = (lo <= mmax) ? lo : (mmax >= 2 ? mmax : 1);
  }
  // mrf (RadialShell.jl:457-471): the per-cell scan is decided by the first
  // cell of each distinct r^2; group s (s-th nonzero r^2) reports index
  // max(s-1, 1); earliest strict minimum of |r^2 - (Rf/alatt)^2| below 10.
  int mrf = 1;
  {
    const double rq = (Rf / alatt) * (Rf / alatt);
    const int K = a.nshell - 1;
    auto r2s = [&](int s) -> double { return (double)a.r2m[s + 1]; };
    int lo = 1, hi = K;
    while (lo <= hi) {
      const int mid = (lo + hi) >> 1;
      if (r2s(mid) >= rq) hi = mid - 1; else lo = mid + 1;
    }
    double best = 10.0;
    int sbest = 0;
    for (int s = lo - 1; s <= lo; s++) {
      if (s < 1 || s > K) continue;
      const double dv = fabs(r2s(s) - rq);
      if (dv < best) { best = dv; sbest = s; }
    }
    if (sbest > 0) mrf = sbest > 1 ? sbest - 1 : 1;
  }
  int mlow_rf = mrf;
  if (mrf > 1) {
    const double rlow = fmax(rad[mrf] - 2.0, 0.0);
    const int f = first_gt(rad, 1, mrf - 1, rlow);
    if (f <= mrf - 1) mlow_rf = f;
  }
  int mupp_rf = mrf;
  {
    const int l = last_lt(rad, mrf + 1, mmax, rad[mrf] + 2.0);
    if (l >= mrf + 1) mupp_rf = l;
  }

  // ---- gather -----------------------------------------------------------
  const float4* __restrict__ aos = a.aos;
  {
    const float4 c0 = aos[2 * lin], c1 = aos[2 * lin + 1];
    if (lane == 0) {
      P.set(PV_FBAR, 1, (double)c0.x);
      P.set(PV_N, 1, 1.0);
      P.set(PV_S + 0, 1, (double)c0.z);
      P.set(PV_S + 1, 1, (double)c0.w);
      P.set(PV_S + 2, 1, (double)c1.x);
      P.set(PV_S2 + 0, 1, (double)c1.y);
      P.set(PV_S2 + 1, 1, (double)c1.z);
      P.set(PV_S2 + 2, 1, (double)c1.w);
#pragma unroll
      for (int v = 0; v < 3; v++) { P.set(PV_G + v, 1, 0.0); P.set(PV_GF + v, 1, 0.0); }
#pragma unroll
      for (int v = 0; v < 6; v++) P.set(PV_Q + v, 1, 0.0);
    }
  }
  const int rext = (int)ceil(rad[mmax]) + 1;
  const bool inside = pi - rext >= 0 && pj - rext >= 0 && pk - rext >= 0 && pi + rext < n && pj + rext < n &&
                      pk + rext < n;
  int state = 0;          // 0 unknown, 1 inward, 2 crossing found, 3 no crossing
  int mcross = 0;
  int mtarget = ADAPTIVE ? -1 : mmax;   // last shell to gather (-1: not known yet)
  int mdone = 1;
  double fbar_prev = (double)aos[2 * lin].x, df_prev = fbar_prev;
  long long visits = 0;
  for (int g = 0; g < a.ngroups; g++) {
    const int base = a.grp_a[g], gend = a.grp_b[g];
    if (mtarget >= 0 && base > mtarget) break;
    if (gend > P.cap) P.spill(mdone);   // profile outgrows shared memory
    const int c0g = a.grp_c[g], ncg = a.grp_c[g + 1] - c0g;
    // (a) lane l sums chunk c0g + l into the shared partial table
    if (lane < ncg) {
      Acc<COMP> A;
      A.zero();
      const int s0 = a.ck_s[c0g + lane], cnt = a.ck_n[c0g + lane];
      int nsh = 0;
      // loads of the next cell are issued before the current cell is summed
      int4 cl = __ldg(a.cells + s0);
      auto in_grid = [&](const int4& c) {
        const int iv1 = pi + c.x, iv2 = pj + c.y, iv3 = pk + c.z;
        return inside || (iv1 >= 0 && iv1 < n && iv2 >= 0 && iv2 < n && iv3 >= 0 && iv3 < n);
      };
      auto rec = [&](const int4& c) { return (int64_t)(pi + c.x) + (int64_t)n * (pj + c.y) + n2 * (pk + c.z); };
      bool ok = in_grid(cl);
      float4 va = make_float4(0.f, 0.f, 0.f, 0.f), vb = va;
      if (ok) { const int64_t li = rec(cl); va = __ldg(aos + 2 * li); vb = __ldg(aos + 2 * li + 1); }
      for (int c = 0; c < cnt; c++) {
        int4 cn = cl;
        bool okn = false;
        float4 van = va, vbn = vb;
        if (c + 1 < cnt) {
          cn = __ldg(a.cells + s0 + c + 1);
          okn = in_grid(cn);
          if (okn) { const int64_t li = rec(cn); van = __ldg(aos + 2 * li); vbn = __ldg(aos + 2 * li + 1); }
        }
        if (ok) {
          nsh++;
          accumulate_cell<COMP>(A, va, vb, (float)cl.x, (float)cl.y, (float)cl.z);
        }
        cl = cn; ok = okn; va = van; vb = vbn;
      }
      visits += nsh;
#pragma unroll
      for (int v = 0; v < NACC; v++) part[v * 32 + lane] = A.get(v);
      part[NACC * 32 + lane] = (double)nsh;
    }
    __syncwarp();
    // (b) lane l finalises shell base + l from its chunks (double-precision
    // sum of the chunk partials, each of which is exact to ~2^-48)
    const int m = base + lane;
    double my_dF = 0.0;
    if (m <= gend) {
      double t[NACC + 1];
#pragma unroll
      for (int v = 0; v <= NACC; v++) t[v] = 0.0;
      const int k0 = a.sh_c0[m] - c0g, nk = a.sh_nc[m];
      for (int k = k0; k < k0 + nk; k++) {
#pragma unroll
        for (int v = 0; v <= NACC; v++) t[v] += part[v * 32 + k];
      }
      const double r = rad[m];
      const double nsh = t[NACC];
      P.set(PV_N, m, nsh);
      my_dF = nsh > 0 ? t[0] / nsh : 0.0;
#pragma unroll
      for (int L = 0; L < 3; L++) {
        P.set(PV_S + L, m, t[1 + L]);
        P.set(PV_S2 + L, m, t[4 + L]);
        P.set(PV_G + L, m, t[7 + L] / r);
        P.set(PV_GF + L, m, t[10 + L] / r);
      }
      P.set(PV_Q + 0, m, (2.0 * t[13]) / r);
      P.set(PV_Q + 1, m, (2.0 * t[14]) / r);
      P.set(PV_Q + 2, m, (2.0 * t[15]) / r);
      P.set(PV_Q + 3, m, t[16] / r);
      P.set(PV_Q + 4, m, t[17] / r);
      P.set(PV_Q + 5, m, t[18] / r);
    }
    __syncwarp();
    const int mend = gend;
    // cumulative mean overdensity (RadialShell.jl:386-390), in shell order;
    // every lane runs the recursion, the owner lane of shell mm keeps Fbar
    double my_fb = 0.0;
    for (int mm = base; mm <= mend; mm++) {
      const double dF = __shfl_sync(FULL, my_dF, mm - base);
      const double r3p = rad[mm - 1] * rad[mm - 1] * rad[mm - 1];
      const double r3 = rad[mm] * rad[mm] * rad[mm];
      const double fb = (r3p * fbar_prev + 0.5 * (df_prev + dF) * (r3 - r3p)) / r3;
      if (lane == mm - base) my_fb = fb;
      fbar_prev = fb;
      df_prev = dF;
      if (ADAPTIVE && state == 0 && mm >= m0_init) {
        if (mm == m0_init && fb < fcrit) {
          state = 1;
        } else if (fb < fcrit) {
          state = 2;
          mcross = mm;
        }
      }
    }
    if (m <= mend) P.set(PV_FBAR, m, my_fb);
    mdone = mend;
    if (ADAPTIVE) {
      if (state == 0 && mdone >= mmax) state = 3;
      if (state != 0) {
        int M = max(max(m0_init, mrf), mupp_rf);
        if (state == 2) M = max(M, mcross);
        mtarget = state == 3 ? mmax : a.need[M];
      }
    }
    __syncwarp();
  }
  P.mdone = mdone;
  __syncwarp();
  {
    const long long tv = warp_sum_ll(visits);
    if (lane == 0) atomicAdd(a.counters + CNT_VISITS, (unsigned long long)tv);
  }

  // ---- post-process (double precision) -----------------------------------
  const double hlatt = 1.0, anor = 1.0;
  const double aRnor = 3.0 * anor / alatt, wnor = anor / (4.0 * 3.141592653589793), wRnor = 3.0 * wnor / alatt;
  const int m = mmax;

  // Phase 3: gradient at the filter scale
  KS krf;
  ks_multi(P, a, mrf, mlow_rf, mupp_rf, 32, wRnor, aRnor, &krf);

  // Phase 4: fcrit crossing (RadialShell.jl:494-537)
  int m0 = m0_init;
  if (P.get(PV_FBAR, m0) >= fcrit) {
    for (int mm = m0; mm <= m; mm++) {
      if (P.get(PV_FBAR, mm) < fcrit) { m0 = mm; break; }
    }
  } else {
    const int mstart = max(m0 - 1, 1);
    bool found = false;
    for (int mp = mstart; mp >= 1; mp--) {
      if (P.get(PV_FBAR, mp) >= fcrit) { found = true; break; }
      m0 = mp;
    }
    if (!found) {
      if (lane == 0) atomicAdd(a.counters + CNT_NOFCRIT, 1ull);
      write_no_collapse(out);
      return;
    }
  }
  if (m0 == 1) {   // zvir1p at m0 is forced to -1 < ZZon (RadialShell.jl:581-622)
    if (lane == 0) atomicAdd(a.counters + CNT_M0ONE, 1ull);
    write_no_collapse(out);
    return;
  }

  // Phase 5: inward walk (RadialShell.jl:566-699).  Each round evaluates K
  // consecutive steps top, top-1, ..., top-K+1 on K lane groups of G = 32/K
  // lanes; group 0 repeats the last step of the previous round (the m0 step
  // in round 0, whose zvir is forced to -1), so the step before a collapse is
  // always the group to the left.  Most peaks collapse within a few steps of
  // m0: round 0 uses 4 steps of 8 lanes, later rounds 32 steps of 1 lane.
  // At mp = 1 the reference's running window is [2, last shell with rad < 2].
  const int hi1 = last_lt(rad, 2, m, 2.0);
  Walk last, prev;
  double zvir1 = -1.0, zvir1p = -1.0;
  bool collapsed = false;
  int rounds = 0;
  int top = m0;
  for (int b = 0;; b++) {
    rounds++;
    const int G = b == 0 ? 8 : 1;
    const int K = 32 / G;
    const int grp = lane / G;
    const int mp = top - grp;
    Walk w;
    w.zv = -1.0;
    // the running mlow never reaches shell 1 (rad 0 is not > max(rad-2, 0))
    ks_multi(P, a, mp, 2, mp > 1 ? m : hi1, G, wRnor, aRnor, &w.k);
    const bool act = mp >= 1;
    if (act) {
      ev_pv(w.k.E, &w.Fh, &w.ev, &w.pv);
      w.Fr = P.get(PV_FBAR, mp);
      if (!(b == 0 && grp == 0)) w.zv = zvir_of(a.tab, w.Fr, w.ev, w.pv);
    }
    const unsigned bal = __ballot_sync(FULL, act && grp >= 1 && (lane & (G - 1)) == 0 && w.zv >= ZZon);
    if (bal) {
      const int L = __ffs(bal) - 1;
      last.k = shfl_ks(w.k, L);
      prev.k = shfl_ks(w.k, L - G);
      last.Fh = __shfl_sync(FULL, w.Fh, L);
      last.Fr = __shfl_sync(FULL, w.Fr, L);
      last.ev = __shfl_sync(FULL, w.ev, L);
      last.pv = __shfl_sync(FULL, w.pv, L);
      zvir1p = __shfl_sync(FULL, w.zv, L);
      zvir1 = __shfl_sync(FULL, w.zv, L - G);   // -1 when group L/G - 1 is the m0 step
      m0 = top - L / G + 1;
      collapsed = true;
      break;
    }
    if (top - (K - 1) <= 1) break;   // reached mp = 1 without collapse
    top -= K - 1;
  }
  if (lane == 0) atomicAdd(a.counters + CNT_WALK, (unsigned long long)rounds);
  if (!collapsed) {
    if (lane == 0) atomicAdd(a.counters + CNT_NOCOLL, 1ull);
    write_no_collapse(out);
    return;
  }

  // Phase 6: collapse radius (RadialShell.jl:707-754)
  const double dZvir = zvir1p - zvir1;
  double RTHL;
  const double ra = rad[m0 - 1], rb = rad[m0];
  const double rad3p = ra * ra * ra, rad3 = rb * rb * rb;
  if (zvir1 > 0.0 && dZvir != 0.0) {
    const double R3 = rad3p + (rad3 - rad3p) * (zvir1p - ZZon) / dZvir;
    RTHL = pow(R3, 1.0 / 3.0);
  } else {
    RTHL = ra;
  }
  if (RTHL <= 0.0) {
    if (lane == 0) atomicAdd(a.counters + CNT_RTHLNEG, 1ull);
    write_no_collapse(out);
    return;
  }
  const double RTHL3 = RTHL * RTHL * RTHL, RTHL5 = RTHL3 * RTHL * RTHL;
  const double drad3 = rad3 - rad3p;
  const double Fa = P.get(PV_FBAR, m0 - 1), Fb = P.get(PV_FBAR, m0);
  const double dFb = Fb - Fa;
  double Fbarx;
  double S[6], gk[3], gkf[3];
  if (zvir1 > 0.0 && drad3 != 0.0) {
    const double fr = (RTHL3 - rad3p) / drad3;
    Fbarx = Fa + fr * dFb;
#pragma unroll
    for (int q = 0; q < 6; q++) S[q] = last.k.E[q] + fr * (prev.k.E[q] - last.k.E[q]);
#pragma unroll
    for (int L = 0; L < 3; L++) {
      gk[L] = last.k.g[L] + fr * (prev.k.g[L] - last.k.g[L]);
      gkf[L] = last.k.gf[L] + fr * (prev.k.gf[L] - last.k.gf[L]);
    }
  } else {
    Fbarx = Fa;
#pragma unroll
    for (int q = 0; q < 6; q++) S[q] = last.k.E[q];
#pragma unroll
    for (int L = 0; L < 3; L++) { gk[L] = prev.k.g[L]; gkf[L] = prev.k.gf[L]; }
  }
  // normalize_strain then eigenvalues (RadialShell.jl:748-752)
  {
    const double tr = S[0] + S[1] + S[2];
    if (tr != 0.0) {
      const double f = Fbarx / tr;
#pragma unroll
      for (int q = 0; q < 6; q++) S[q] *= f;
    }
  }
  double Frhoc, e_v_f, p_v_f;
  ev_pv(S, &Frhoc, &e_v_f, &p_v_f);
  double smat[6];
#pragma unroll
  for (int q = 0; q < 6; q++) smat[q] = last.k.E[q] * (Fbarx / last.Fh);

  // Phase 7: Sbar, Sbar2 (RadialShell.jl:758-773), Srb (:776-790)
  double sb[6] = {0, 0, 0, 0, 0, 0};
  long long nS = 0;
  double srb = 0.0;
  for (int m1 = 1 + lane; m1 <= m0 - 1; m1 += 32) {
    const double nn = P.get(PV_N, m1);
    if (nn > 0) {
#pragma unroll
      for (int L = 0; L < 3; L++) {
        sb[L] += P.get(PV_S + L, m1);
        sb[3 + L] += P.get(PV_S2 + L, m1);
      }
      nS += (long long)nn;
    }
    if (m1 >= 2) {
      const double r5 = a.rad5[m1], r5p = m1 - 1 >= 2 ? a.rad5[m1 - 1] : 0.0;
      srb += 0.5 * (P.get(PV_FBAR, m1 - 1) + P.get(PV_FBAR, m1)) * (r5 - r5p);
    }
  }
#pragma unroll
  for (int q = 0; q < 6; q++) sb[q] = warp_sum(sb[q]);
  nS = warp_sum_ll(nS);
  srb = warp_sum(srb);
  if (nS > 0) {
#pragma unroll
    for (int q = 0; q < 6; q++) sb[q] /= (double)nS;
  }
  const double rad5p = (m0 - 1 >= 2) ? a.rad5[m0 - 1] : 0.0;
  if (zvir1 > 0.0 && dZvir != 0.0) srb += 0.5 * (Fa + Fbarx) * (RTHL5 - rad5p);
  if (Fbarx * RTHL5 > 0.0) srb /= (Fbarx * RTHL5);

  // d2F: mean lapd over cells (centre excluded) with sqrt(r2) <= RTHL, in
  // list order, stopping at the first out-of-grid cell (RadialShell.jl:805-819)
  double d2F = 0.0;
  if (a.lapd) {
    double acc = 0.0;
    long long navg = 0;
    bool stop = false;
    for (int64_t c0 = 1; c0 < a.npart && !stop; c0 += 32) {
      const int64_t c = c0 + lane;
      bool valid = false, oob = false;
      float v = 0.f;
      if (c < a.npart) {
        const int4 cl = __ldg(a.cells + c);
        if (!(sqrt((double)cl.w) > RTHL)) {
          const int iv1 = pi + cl.x, iv2 = pj + cl.y, iv3 = pk + cl.z;
          if (iv1 < 0 || iv1 >= n || iv2 < 0 || iv2 >= n || iv3 < 0 || iv3 >= n) oob = true;
          else { valid = true; v = a.lapd[iv1 + (int64_t)n * iv2 + n2 * iv3]; }
        }
      }
      const unsigned ob = __ballot_sync(FULL, oob);
      if (ob) {
        const int first = __ffs(ob) - 1;
        if (lane >= first) valid = false;
        stop = true;
      }
      if (valid) { acc += (double)v; navg++; }
      const int4 last_cell = __ldg(a.cells + min(c0 + 31, a.npart - 1));
      if (sqrt((double)last_cell.w) > RTHL) stop = true;
    }
    acc = warp_sum(acc);
    navg = warp_sum_ll(navg);
    if (navg > 0) d2F = acc / (double)navg;
  }

  // zvir_half (RadialShell.jl:825-885): the ten radii on lane pairs 0..19
  double zvir_half = -1.0;
  if (RTHL / hlatt >= 3.0) {
    const int e = lane >> 1;   // radius index jj - 1
    int m0_rc = 0, mlow_rc = 1, mupp_rc = 1;
    if (e < 10) {
      const double rcur = RTHL * pow(e / 9.0 * 0.5 + 0.5, 1.0 / 3.0);
      // first m1 in [2, m-1] with rad > rcur + 2 (the loop's break), else m-1
      const int fu = first_gt(rad, 2, m - 1, rcur + 2.0 * hlatt);
      mupp_rc = fu <= m - 1 ? fu : (m - 1 >= 2 ? m - 1 : 1);
      const int fl = first_gt(rad, 1, m - 1, fmax(rcur - 2.0 * hlatt, 0.0));
      if (fl <= m - 1) mlow_rc = fl;
      const int f0 = first_gt(rad, 1, m - 1, rcur);
      m0_rc = (f0 <= m - 1) ? f0 : max(m - 1, 1);
    }
    KS krc;
    ks_multi(P, a, m0_rc, mlow_rc, mupp_rc, 2, wRnor, aRnor, &krc);
    double zl = -1.0;
    if (e < 10) {
      double Fr, ev, pv;
      ev_pv(krc.E, &Fr, &ev, &pv);
      zl = zvir_of(a.tab, P.get(PV_FBAR, m0_rc), ev, pv) - 1.0;
    }
    zvir_half = fmax(warp_max(zl), -1.0);
  }

  // results (layout in ppb.h)
  if (lane == 0) {
    double r[RES_N];
    r[0] = RTHL;
    r[1] = srb;
#pragma unroll
    for (int L = 0; L < 3; L++) {
      r[2 + L] = sb[L];
      r[5 + L] = sb[3 + L];
      r[17 + L] = gk[L];
      r[20 + L] = krf.g[L];
      r[27 + L] = gkf[L];
    }
    r[8] = smat[0]; r[9] = smat[3]; r[10] = smat[4];
    r[11] = smat[3]; r[12] = smat[1]; r[13] = smat[5];
    r[14] = smat[4]; r[15] = smat[5]; r[16] = smat[2];
    r[23] = Fbarx;
    r[24] = e_v_f;
    r[25] = p_v_f;
    r[26] = zvir_half;
    r[30] = d2F;
#pragma unroll
    for (int q = 0; q < RES_N; q++) out[q] = r[q];
  }
}

template <bool COMP, bool ADAPTIVE>
__global__ void __launch_bounds__(128, 3) shell_kernel(ShellArgs a) {
  const int lane = threadIdx.x & 31;
  const int warp_in_block = threadIdx.x >> 5;
  const int64_t slot = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp_in_block;
  double* prof = a.scratch + slot * a.scratch_stride;
  extern __shared__ double shm[];
  double* smem = shm + (size_t)warp_in_block * SMEM_WARP_DOUBLES;
  while (true) {
    int p = 0;
    if (lane == 0) p = atomicAdd(a.queue, 1);
    p = __shfl_sync(FULL, p, 0);
    if (p >= a.npk) break;
    analyse_one<COMP, ADAPTIVE>(a, p, prof, smem);
    __syncwarp();
  }
}

template <bool C, bool A>
void launch_variant(const ShellArgs& a, dim3 grid, dim3 block, size_t shm, cudaStream_t s) {
  shell_kernel<C, A><<<grid, block, shm, s>>>(a);
}

}  // namespace

// allow the dynamic shared memory of the chosen block size (once per process
// and device; called before occupancy queries and launches)
void shell_prepare(int warps_per_block) {
  const int shm = (int)((size_t)warps_per_block * SMEM_WARP_DOUBLES * 8);
  PPB_CUDA(cudaFuncSetAttribute(shell_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, shm));
  PPB_CUDA(cudaFuncSetAttribute(shell_kernel<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, shm));
  PPB_CUDA(cudaFuncSetAttribute(shell_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, shm));
  PPB_CUDA(cudaFuncSetAttribute(shell_kernel<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, shm));
}

const void* shell_kernel_ptr(bool comp, bool adaptive) {
  if (comp && adaptive) return (const void*)shell_kernel<true, true>;
  if (comp) return (const void*)shell_kernel<true, false>;
  if (adaptive) return (const void*)shell_kernel<false, true>;
  return (const void*)shell_kernel<false, false>;
}

int64_t shell_scratch_doubles_per_warp(int nshell) { return (int64_t)NV * (nshell + 1); }

size_t shell_smem_bytes(int warps_per_block) { return (size_t)warps_per_block * SMEM_WARP_DOUBLES * 8; }

void launch_shell(Launch L, const ShellArgs& a, bool comp, bool adaptive, int blocks, int warps_per_block) {
  dim3 grid(blocks), block(32 * warps_per_block);
  const size_t shm = shell_smem_bytes(warps_per_block);
  if (comp && adaptive) launch_variant<true, true>(a, grid, block, shm, L.s);
  else if (comp && !adaptive) launch_variant<true, false>(a, grid, block, shm, L.s);
  else if (!comp && adaptive) launch_variant<false, true>(a, grid, block, shm, L.s);
  else launch_variant<false, false>(a, grid, block, shm, L.s);
  PPB_LAUNCHED(*L.count);
}

}  // namespace ppb
