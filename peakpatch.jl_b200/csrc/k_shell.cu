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
//     M = max(crossing shell, first shell beyond ir2min, Rf shell), because
//     kernel_strain's weight vanishes for |rad[mp] - rad[m1]| >= 2 and the
//     walk only moves inward from the crossing; the one exception (no
//     crossing at all) gathers every shell.  A device-side guard counts any
//     read past the gathered range (it must stay 0; the host fails loudly).
//  3. Collapse walk in double precision, executed redundantly by all lanes
//     (warp-uniform control flow); the shell window sums of kernel_strain are
//     split across lanes and combined with a butterfly reduction.
#include "ppb_internal.h"

namespace ppb {

namespace {

constexpr int NV = 21;   // profile values per shell
enum { PV_FBAR = 0, PV_N = 1, PV_S = 2, PV_S2 = 5, PV_G = 8, PV_GF = 11, PV_Q = 14, PV_DF = 20 };
constexpr int NACC = 19; // gather accumulators: F, S3, S2_3, G3, Gf3, Q6 (xx yy zz xy xz yz)
constexpr unsigned FULL = 0xffffffffu;

// counters layout
enum { CNT_VISITS = 0, CNT_PREMASK = 1, CNT_NOFCRIT = 2, CNT_M0ONE = 3, CNT_NOCOLL = 4, CNT_RTHLNEG = 5,
       CNT_GUARD = 6, CNT_AKK = 7, CNT_LAPD = 8 };

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
// small double-precision helpers
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

// RadialShell.jl:100-127
__device__ double hRinteg(double u0, double u12) {
  const double x0 = fabs(u0);
  if (x0 >= 2.0) return 0.0;
  const double one7 = 1.0 / 7.0;
  double r = 1.6 * u12 - 6.4 * one7;
  const double x02 = x0 * x0, x04 = x02 * x02;
  if (x0 >= 1.0) {
    const double h1 = x04 * (2.0 - x0 * (2.4 - x0 * (1.0 - x0 * one7)));
    const double h2 = x02 * (4.0 - x0 * (4.0 - x0 * (1.5 - x0 * 0.2)));
    r = r - h2 * u12 + h1;
  } else {
    r = r - 0.2 * (u12 - one7);
    if (x0 > 0.0) {
      const double h1 = x04 * (1.0 - x02 * (1.0 - 3.0 * x0 * one7));
      const double h2 = x02 * (2.0 - x02 * (1.5 - 0.6 * x0));
      r = r - h2 * u12 + h1;
    }
  }
  return r;
}

// symmetric 3x3 eigenvalues (ascending) by cyclic Jacobi rotations.
// m = (xx, yy, zz, xy, xz, yz)
__device__ void eig3(const double m[6], double lam[3]) {
  double A[3][3] = {{m[0], m[3], m[4]}, {m[3], m[1], m[5]}, {m[4], m[5], m[2]}};
  for (int sweep = 0; sweep < 64; sweep++) {
    const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
    const double dia = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
    if (off == 0.0 || off < 1e-36 * dia) break;
#pragma unroll
    for (int pq = 0; pq < 3; pq++) {
      const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
      if (A[p][q] == 0.0) continue;
      const double theta = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
      const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
      const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const double akp = A[k][p], akq = A[k][q];
        A[k][p] = c * akp - s * akq;
        A[k][q] = s * akp + c * akq;
      }
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const double apk = A[p][k], aqk = A[q][k];
        A[p][k] = c * apk - s * aqk;
        A[q][k] = s * apk + c * aqk;
      }
    }
  }
  double a = A[0][0], b = A[1][1], c = A[2][2], t;
  if (a > b) { t = a; a = b; b = t; }
  if (b > c) { t = b; b = c; c = t; }
  if (a > b) { t = a; a = b; b = t; }
  lam[0] = a; lam[1] = b; lam[2] = c;
}

// trilinear lookup, outside the box -> -1 (CollapseTable.jl:128-145)
__device__ double tab_interp(const DevTable& T, double x, double y, double z) {
  if (!(x >= T.x1 && x <= T.x2 && y >= T.y1 && y <= T.y2 && z >= T.z1 && z <= T.z2)) return -1.0;
  int ix, iy, iz;
  double wx, wy, wz;
  {
    const double pos = (x - T.x1) / ((T.x2 - T.x1) / (T.nx - 1));
    int i = (int)floor(pos); i = i < 0 ? 0 : (i > T.nx - 2 ? T.nx - 2 : i);
    ix = i; wx = pos - i;
  }
  {
    const double pos = (y - T.y1) / ((T.y2 - T.y1) / (T.ny - 1));
    int i = (int)floor(pos); i = i < 0 ? 0 : (i > T.ny - 2 ? T.ny - 2 : i);
    iy = i; wy = pos - i;
  }
  {
    const double pos = (z - T.z1) / ((T.z2 - T.z1) / (T.nz - 1));
    int i = (int)floor(pos); i = i < 0 ? 0 : (i > T.nz - 2 ? T.nz - 2 : i);
    iz = i; wz = pos - i;
  }
  auto A = [&](int a, int b, int c) {
    return (double)__ldg(T.t + (ix + a) + (int64_t)T.nx * ((iy + b) + (int64_t)T.ny * (iz + c)));
  };
  const double c00 = (1 - wx) * A(0, 0, 0) + wx * A(1, 0, 0);
  const double c10 = (1 - wx) * A(0, 1, 0) + wx * A(1, 1, 0);
  const double c01 = (1 - wx) * A(0, 0, 1) + wx * A(1, 0, 1);
  const double c11 = (1 - wx) * A(0, 1, 1) + wx * A(1, 1, 1);
  const double c0 = (1 - wy) * c00 + wy * c10;
  const double c1 = (1 - wy) * c01 + wy * c11;
  return (1 - wz) * c0 + wz * c1;
}

// ---------------------------------------------------------------------------
// per-warp profile (scratch): value v of shell m at p[v*MS + m]
// ---------------------------------------------------------------------------
struct Prof {
  double* p;
  int MS;
  int mdone;                        // shells 1..mdone are valid
  unsigned long long* counters;
  __device__ __forceinline__ double get(int v, int m) const {
    if (m > mdone) {                // never taken when the truncation rule holds
      if ((threadIdx.x & 31) == 0) atomicAdd(counters + CNT_GUARD, 1ull);
      return 0.0;
    }
    return p[(int64_t)v * MS + m];
  }
  __device__ __forceinline__ void set(int v, int m, double x) { p[(int64_t)v * MS + m] = x; }
};

struct KS {
  double E[6];   // xx yy zz xy xz yz
  double g[3], gf[3];
};

// kernel_strain (RadialShell.jl:228-277), lanes split m1 in [mlow, mupp]
__device__ KS kernel_strain(const Prof& P, const double* __restrict__ rad, int mp, int mlow, int mupp,
                            const double* __restrict__ akk, double wRnor, double aRnor,
                            unsigned long long* counters) {
  const int lane = threadIdx.x & 31;
  double E[6] = {0, 0, 0, 0, 0, 0}, g[3] = {0, 0, 0}, gf[3] = {0, 0, 0};
  const double rmp = rad[mp];
  for (int m1 = mlow + lane; m1 <= mupp; m1 += 32) {
    double wt;
    bool use = true;
    if (mp > 1) {
      const double u0 = rmp - rad[m1];
      const double u02 = u0 * u0;
      if (u02 < 4.0) {
        const double u12 = rmp * rmp + rad[m1] * rad[m1];
        const double d = u12 - u02;
        wt = hRinteg(u0, u12) / (d * d);
      } else {
        use = false;
        wt = 0.0;
      }
    } else {
      const double u0 = rad[m1];
      const double con = 100.0 * u0 * u0;
      long long icon = (long long)floor(con);
      const double diff = con - (double)icon;
      if (icon + 1 > 1100) {      // the reference raises a BoundsError here
        atomicAdd(counters + CNT_AKK, 1ull);
        icon = 1099;
      }
      const double aww = akk[icon] + diff * (akk[icon + 1] - akk[icon]);
      wt = 0.5 * aww / rad[m1];
    }
    if (use) {
#pragma unroll
      for (int L = 0; L < 3; L++) {
        g[L] += wt * P.get(PV_G + L, m1);
        gf[L] += wt * P.get(PV_GF + L, m1);
      }
#pragma unroll
      for (int q = 0; q < 6; q++) E[q] -= 0.5 * wt * P.get(PV_Q + q, m1);
    }
  }
  KS r;
  const double sc = mp > 1 ? wRnor / rmp : aRnor;
#pragma unroll
  for (int q = 0; q < 6; q++) r.E[q] = warp_sum(E[q]) * sc;
#pragma unroll
  for (int L = 0; L < 3; L++) {
    r.g[L] = warp_sum(g[L]) * sc;
    r.gf[L] = warp_sum(gf[L]) * sc;
  }
  return r;
}

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
// largest m in [lo, hi] with rad[m] <= x, or lo-1
__device__ __forceinline__ int last_le(const double* rad, int lo, int hi, double x) {
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    if (rad[mid] <= x) lo = mid + 1; else hi = mid - 1;
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
__device__ void analyse_one(const ShellArgs& a, int64_t p, double* prof_base) {
  const int lane = threadIdx.x & 31;
  const int n = a.n;
  const int64_t n2 = (int64_t)n * n;
  const int64_t lin = a.pk.lin[p];
  const int pk = (int)(lin / n2), pj = (int)((lin / n) % n), pi = (int)(lin % n);
  const double Rf = a.pk.Rf[p];
  const int ir2min = a.pk.ir2min[p];
  const double ZZon = a.pk.ZZon[p];
  const double fcrit = a.pk.fcrit[p];
  const double alatt = a.alatt;
  const double* __restrict__ rad = a.rad;
  const int mmax = a.mmax;
  double* out = a.out + p * RES_N;

  Prof P{prof_base, a.nshell + 1, 0, a.counters};

  // ---- geometry that depends only on the shell radii --------------------
  // m0 of the gather loop (RadialShell.jl:392-399): first finalised shell with
  // r^2 > ir2min, else the last finalised shell.
  int m0_init;
  {
    int lo = 2, hi = mmax;   // first m in [2, mmax] with r2m[m] > ir2min
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
    const int K = a.nshell - 1;          // nonzero distinct r^2 values: s = 1..K
    // first s with r2_s >= rq (r2_s = rad[s+1]^2 for s <= K-1; the last group
    // is not finalised, its r^2 comes from the cell list)
    int lo = 1, hi = K;
    // r^2 of the s-th nonzero distinct value is the r^2 of shell s+1
    auto r2s = [&](int s) -> double { return (double)a.r2m[s + 1]; };
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
  // centre cell (shell 1)
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
      P.set(PV_DF, 1, (double)c0.x);
    }
  }
  const int rext = (int)ceil(rad[mmax]) + 1;
  const bool inside = pi - rext >= 0 && pj - rext >= 0 && pk - rext >= 0 && pi + rext < n && pj + rext < n &&
                      pk + rext < n;
  // truncation state (warp-uniform)
  int state = 0;          // 0 unknown, 1 inward, 2 crossing found, 3 no crossing
  int mcross = 0;
  int mtarget = mmax;     // last shell to gather
  int mdone = 1;
  double fbar_prev = (double)aos[2 * lin].x, df_prev = fbar_prev;
  long long visits = 0;
  if (ADAPTIVE) {
    // before any crossing information the walk needs at least the shells
    // around m0_init and around the Rf window
    mtarget = -1;
  }
  for (int base = 2; base <= mmax; base += 32) {
    if (ADAPTIVE && mtarget >= 0 && base > mtarget) break;
    const int m = base + lane;
    const int mlim = ADAPTIVE && mtarget >= 0 ? mtarget : mmax;
    if (m <= mlim) {
      Acc<COMP> A;
      A.zero();
      const int s0 = a.sh_start[m - 1], cnt = a.sh_count[m - 1];
      int nsh = 0;
      for (int c = 0; c < cnt; c++) {
        const int4 cl = __ldg(a.cells + s0 + c);
        const int iv1 = pi + cl.x, iv2 = pj + cl.y, iv3 = pk + cl.z;
        if (!inside && (iv1 < 0 || iv1 >= n || iv2 < 0 || iv2 >= n || iv3 < 0 || iv3 >= n)) continue;
        nsh++;
        const int64_t li = iv1 + (int64_t)n * iv2 + n2 * iv3;
        const float4 va = __ldg(aos + 2 * li), vb = __ldg(aos + 2 * li + 1);
        accumulate_cell<COMP>(A, va, vb, (float)cl.x, (float)cl.y, (float)cl.z);
      }
      visits += nsh;
      const double r = rad[m];
      const double F = A.get(0);
      P.set(PV_N, m, (double)nsh);
      P.set(PV_DF, m, nsh > 0 ? F / nsh : 0.0);
#pragma unroll
      for (int L = 0; L < 3; L++) {
        P.set(PV_S + L, m, A.get(1 + L));
        P.set(PV_S2 + L, m, A.get(4 + L));
        P.set(PV_G + L, m, A.get(7 + L) / r);
        P.set(PV_GF + L, m, A.get(10 + L) / r);
      }
      P.set(PV_Q + 0, m, (2.0 * A.get(13)) / r);
      P.set(PV_Q + 1, m, (2.0 * A.get(14)) / r);
      P.set(PV_Q + 2, m, (2.0 * A.get(15)) / r);
      P.set(PV_Q + 3, m, A.get(16) / r);
      P.set(PV_Q + 4, m, A.get(17) / r);
      P.set(PV_Q + 5, m, A.get(18) / r);
    }
    __syncwarp();
    const int mend = min(base + 31, mlim);
    // cumulative mean overdensity (RadialShell.jl:386-390), sequential
    for (int mm = base; mm <= mend; mm++) {
      const double dF = P.p[(int64_t)PV_DF * P.MS + mm];
      const double r3p = rad[mm - 1] * rad[mm - 1] * rad[mm - 1];
      const double r3 = rad[mm] * rad[mm] * rad[mm];
      const double fb = (r3p * fbar_prev + 0.5 * (df_prev + dF) * (r3 - r3p)) / r3;
      if (lane == 0) P.set(PV_FBAR, mm, fb);
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
    mdone = mend;
    if (ADAPTIVE) {
      if (state == 0 && mdone >= mmax) state = 3;
      if (state != 0) {
        int M = max(m0_init, mrf);
        M = max(M, mupp_rf);
        if (state == 2) M = max(M, mcross);
        if (state == 3) M = mmax;
        // last shell with rad <= rad[M] + 2, plus two more
        const int l = last_le(rad, M, mmax, rad[M] + 2.0);
        mtarget = min(mmax, max(l, M) + 2);
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

  // ---- post-process (double precision, warp-uniform) ---------------------
  const double hlatt = 1.0, anor = 1.0;
  const double aRnor = 3.0 * anor / alatt, wnor = anor / (4.0 * 3.141592653589793), wRnor = 3.0 * wnor / alatt;
  const int m = mmax;

  // Phase 3: gradient at the filter scale
  const KS krf = kernel_strain(P, rad, mrf, mlow_rf, mupp_rf, a.akk, wRnor, aRnor, a.counters);

  // Phase 4: fcrit crossing (RadialShell.jl:494-537)
  int m0 = m0_init;
  int mupp;
  if (P.get(PV_FBAR, m0) >= fcrit) {
    bool found = false;
    for (int mm = m0; mm <= m; mm++) {
      if (P.get(PV_FBAR, mm) < fcrit) { m0 = mm; found = true; break; }
    }
    if (!found) {
      mupp = m;
    } else {
      const int l = last_lt(rad, m0 + 1, m, rad[m0] + 2.0);
      mupp = l >= m0 + 1 ? l : m0;
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
    const int l = last_lt(rad, m0 + 1, m, rad[m0] + 2.0);
    mupp = l >= m0 + 1 ? l : m0;
  }

  // Phase 5: inward walk (RadialShell.jl:541-704)
  int mlow = m0;
  if (m0 > 1) {
    const double rlow = fmax(rad[m0] - 2.0, 0.0);
    const int f = first_gt(rad, 1, m0 - 1, rlow);
    if (f <= m0 - 1) mlow = f;
  }
  double zvir1 = -1.0, zvir1p = -1.0;
  KS last, prev;     // (Ebar, grad, gradf) of the current and of the previous step
  double Frhoh, Frho, e_v, p_v;
  bool collapsed = false;
  {
    const KS k0 = kernel_strain(P, rad, m0, mlow, mupp, a.akk, wRnor, aRnor, a.counters);
    double F0, e0, p0;
    ev_pv(k0.E, &F0, &e0, &p0);
    // zvir1p at m0 is forced to -1 (RadialShell.jl:581-583), never >= ZZon > 0
    zvir1 = -1.0;
    prev = k0;   // strain_mat / gradpk_prev / gradpkf_prev
    last = k0;   // Ebar_last / gradpk_last / gradpkf_last
    Frhoh = F0;
    Frho = P.get(PV_FBAR, m0);
    e_v = e0;
    p_v = p0;
    if (-1.0 >= ZZon) {
      collapsed = true;
    } else {
      if (m0 == 1) {
        if (lane == 0) atomicAdd(a.counters + CNT_M0ONE, 1ull);
        write_no_collapse(out);
        return;
      }
      for (int mp = m0 - 1; mp >= 1; mp--) {
        const double rupp_mp = rad[mp] + 2.0;
        const double rlow_mp = fmax(rad[mp] - 2.0, 0.0);
        if (rad[mupp] > rupp_mp) {
          const int l = last_lt(rad, mp + 1, mupp, rupp_mp);
          mupp = l >= mp + 1 ? l : mp;
        }
        if (mlow > 1 && rad[mlow - 1] > rlow_mp) {
          const int f = first_gt(rad, 1, mlow - 1, rlow_mp);
          if (f <= mlow - 1) mlow = f;
        }
        const KS kmp = kernel_strain(P, rad, mp, mlow, mupp, a.akk, wRnor, aRnor, a.counters);
        double Fh, ev, pv;
        ev_pv(kmp.E, &Fh, &ev, &pv);
        const double Fr = P.get(PV_FBAR, mp);
        double zp = -1.0;
        if (Fr > 0.0) {
          const double poe = ev < 1e-5 ? 0.0 : pv / ev;
          zp = tab_interp(a.tab, log10(Fr), ev, poe);
        }
        if (zp >= ZZon) {
          m0 = mp + 1;
          zvir1p = zp;
          last = kmp;
          Frhoh = Fh;
          Frho = Fr;
          e_v = ev;
          p_v = pv;
          collapsed = true;
          break;
        }
        zvir1 = zp;
        prev = kmp;
        last = kmp;
        Frhoh = Fh;
        Frho = Fr;
        e_v = ev;
        p_v = pv;
      }
    }
  }
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
    for (int q = 0; q < 6; q++) S[q] = last.E[q] + fr * (prev.E[q] - last.E[q]);
#pragma unroll
    for (int L = 0; L < 3; L++) {
      gk[L] = last.g[L] + fr * (prev.g[L] - last.g[L]);
      gkf[L] = last.gf[L] + fr * (prev.gf[L] - last.gf[L]);
    }
  } else {
    Fbarx = Fa;
#pragma unroll
    for (int q = 0; q < 6; q++) S[q] = last.E[q];
#pragma unroll
    for (int L = 0; L < 3; L++) { gk[L] = prev.g[L]; gkf[L] = prev.gf[L]; }
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
  if (!(Frhoc > 0.0)) { e_v_f = 0.0; p_v_f = 0.0; }
  double smat[6];
#pragma unroll
  for (int q = 0; q < 6; q++) smat[q] = last.E[q] * (Fbarx / Frhoh);

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
      const double r5 = pow(rad[m1], 5.0), r5p = m1 - 1 >= 2 ? pow(rad[m1 - 1], 5.0) : 0.0;
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
  const double rad5p = (m0 - 1 >= 2) ? pow(rad[m0 - 1], 5.0) : 0.0;
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
      // all later cells have larger r2; stop once the whole chunk is beyond RTHL
      const int4 last_cell = __ldg(a.cells + min(c0 + 31, a.npart - 1));
      if (sqrt((double)last_cell.w) > RTHL) stop = true;
    }
    acc = warp_sum(acc);
    navg = warp_sum_ll(navg);
    if (navg > 0) d2F = acc / (double)navg;
  }

  // zvir_half (RadialShell.jl:825-885)
  double zvir_half = -1.0;
  if (RTHL / hlatt >= 3.0) {
    for (int jj = 1; jj <= 10; jj++) {
      const double rcur = RTHL * pow((jj - 1) / 9.0 * 0.5 + 0.5, 1.0 / 3.0);
      const double rupp_rc = rcur + 2.0 * hlatt;
      int mupp_rc = 1;
      for (int m1 = 2; m1 <= m - 1; m1++) {
        if (rad[m1] > rupp_rc) { mupp_rc = m1; break; }
        else if (rad[m1] == 0.0) { mupp_rc = m1 - 1; break; }
        mupp_rc = m1;
      }
      const double rlow_rc = fmax(rcur - 2.0 * hlatt, 0.0);
      int mlow_rc = 1;
      {
        const int f = first_gt(rad, 1, m - 1, rlow_rc);
        if (f <= m - 1) mlow_rc = f;
      }
      int m0_rc = 1;
      {
        const int f = first_gt(rad, 1, m - 1, rcur);
        m0_rc = (f <= m - 1) ? f : max(m - 1, 1);
      }
      const KS krc = kernel_strain(P, rad, m0_rc, mlow_rc, mupp_rc, a.akk, wRnor, aRnor, a.counters);
      double Fr, ev, pv;
      ev_pv(krc.E, &Fr, &ev, &pv);
      const double Frc = P.get(PV_FBAR, m0_rc);
      const double poe = ev < 1e-5 ? 0.0 : pv / ev;
      double zrc = -1.0;
      if (Frc > 0.0) zrc = tab_interp(a.tab, log10(Frc), ev, poe);
      zvir_half = fmax(zrc - 1.0, zvir_half);
    }
  }

  // results (layout in ppb.h)
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
  // strain column-major 3x3 from (xx yy zz xy xz yz)
  r[8] = smat[0]; r[9] = smat[3]; r[10] = smat[4];
  r[11] = smat[3]; r[12] = smat[1]; r[13] = smat[5];
  r[14] = smat[4]; r[15] = smat[5]; r[16] = smat[2];
  r[23] = Fbarx;
  r[24] = e_v_f;
  r[25] = p_v_f;
  r[26] = zvir_half;
  r[30] = d2F;
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < RES_N; q++) out[q] = r[q];
  }
  (void)Frho; (void)e_v; (void)p_v;
}

template <bool COMP, bool ADAPTIVE>
__global__ void __launch_bounds__(128) shell_kernel(ShellArgs a) {
  const int lane = threadIdx.x & 31;
  const int warp_in_block = threadIdx.x >> 5;
  const int64_t slot = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp_in_block;
  double* prof = a.scratch + slot * a.scratch_stride;
  while (true) {
    int p = 0;
    if (lane == 0) p = atomicAdd(a.queue, 1);
    p = __shfl_sync(FULL, p, 0);
    if (p >= a.npk) break;
    analyse_one<COMP, ADAPTIVE>(a, p, prof);
    __syncwarp();
  }
}

}  // namespace

const void* shell_kernel_ptr(bool comp, bool adaptive) {
  if (comp && adaptive) return (const void*)shell_kernel<true, true>;
  if (comp) return (const void*)shell_kernel<true, false>;
  if (adaptive) return (const void*)shell_kernel<false, true>;
  return (const void*)shell_kernel<false, false>;
}

int64_t shell_scratch_doubles_per_warp(int nshell) { return (int64_t)NV * (nshell + 1); }

void launch_shell(Launch L, const ShellArgs& a, bool comp, bool adaptive, int blocks, int warps_per_block) {
  dim3 grid(blocks), block(32 * warps_per_block);
  if (comp && adaptive) shell_kernel<true, true><<<grid, block, 0, L.s>>>(a);
  else if (comp && !adaptive) shell_kernel<true, false><<<grid, block, 0, L.s>>>(a);
  else if (!comp && adaptive) shell_kernel<false, true><<<grid, block, 0, L.s>>>(a);
  else shell_kernel<false, false><<<grid, block, 0, L.s>>>(a);
  PPB_LAUNCHED(*L.count);
}

}  // namespace ppb
