// k_table.cu — collapse-table generation on the GPU: make_table with the
// RK4 solver, one thread per table node.
//
// Reference: src/EllipsoidalCollapse/CollapseTable.jl:33-52 (make_table:
// node (i, j, k) at log10 F = X1 + (i-1) dX, e_v = Y1 + (j-1) dY,
// p_v / e_v = Z1 + (k-1) dZ) and src/EllipsoidalCollapse/EllipsoidalCollapse.jl
// :518-624 (evolve_ellipse_full, solver = :rk4: the homogeneous ellipsoid in
// an expanding background, axes a_1..a_3 and their velocities integrated in
// the background scale factor with "funny RK4" steps of tfac a_3^1.5 H until
// axis 1 virialises), :212-323 (get_derivs!: per-axis virialisation at
// fcoll_i a, frozen axes, internal + external tidal force), :153-179
// (rk4_homel!), :113-149 (get_b_2 shape integrals), :66-108 (Carlson's
// elliptic integral RD), Cosmology.jl:273-293 (Dlinear_ab).
//
// The node value is 1 + z_vir of axis 1 (-1 when it has not virialised by
// a = 2 or nstepmax steps).  The steps of a node are sequential, so the table
// is a grid of independent FP64 integrations: latency-bound, one thread each.
//
// Bit-exactness with the CPU oracle: this file is compiled without
// multiply-add contraction (-fmad=false), so that every +, -, *, / and sqrt
// is one IEEE-754 operation in the reference's order; F = 10^x is evaluated
// on the host; the logarithm of the oblate shape integral is the project's
// own (ppbm::log_pos), the one the oracle uses too.
#include "ppb_ctx.h"
#include "ppb_math.h"

namespace ppb {

namespace {

struct TabArgs {
  const double* Frho;   // Nx values 10^x (host pow)
  int Nx, Ny, Nz;
  double Y1, dY, Z1, dZ;
  int iforce, ivir, nstepmax;
  double fcoll1, fcoll2, fcoll3, tfac, zinit_fac;
  double Rvac, Rcurv;   // Omvac / Omnr, Omcurv / Omnr
  // growth table (Dlinear_tables)
  const double *ga, *gD, *gf;
  int ng;
  double amin, amax, Dinf, D0, Hinf, H0;
  double* out;
  unsigned long long* steps;   // total RK4 steps (statistics)
};

// Dlinear_ab: the table position, 4-point (2-point at the ends) Lagrange
// interpolation of D(a)/a and dlnD/dlna; returns D(a) and dlnD/dlna.  The
// reference's bisection returns the number of table entries below ai (the
// table increases strictly); the integration's a only moves forward, so that
// count is kept in *pos and walked from the previous call (the same index,
// a few cached loads instead of a dozen dependent ones).
__device__ void dlin(const TabArgs& A, double ai, double* Dl, double* HD, int* pos) {
  const int ntab = A.ng;
  if (ai > A.amin && ai < A.amax) {
    int j = *pos;
    while (j < ntab && ai > __ldg(A.ga + j)) j++;
    while (j > 0 && !(ai > __ldg(A.ga + j - 1))) j--;
    *pos = j;
    const int kk = j;
    int nl, kkl;
    if (kk < 2 || kk >= ntab) { nl = 2; kkl = kk - 1 > 1 ? kk - 1 : 1; } else { nl = 4; kkl = kk - 2; }
    const double* xa = A.ga + kkl - 1;
    const double* v1 = A.gD + kkl - 1;
    const double* v2 = A.gf + kkl - 1;
    const double x = ai;
    double p1, p2;
    if (nl == 4) {
      const double x0 = __ldg(xa), x1 = __ldg(xa + 1), x2 = __ldg(xa + 2), x3 = __ldg(xa + 3);
      const double a1 = (x - x1) / (x0 - x1) * (x - x2) / (x0 - x2) * (x - x3) / (x0 - x3);
      const double a2 = (x - x0) / (x1 - x0) * (x - x2) / (x1 - x2) * (x - x3) / (x1 - x3);
      const double a3 = (x - x0) / (x2 - x0) * (x - x1) / (x2 - x1) * (x - x3) / (x2 - x3);
      const double a4 = (x - x0) / (x3 - x0) * (x - x1) / (x3 - x1) * (x - x2) / (x3 - x2);
      p1 = a1 * __ldg(v1) + a2 * __ldg(v1 + 1) + a3 * __ldg(v1 + 2) + a4 * __ldg(v1 + 3);
      p2 = a1 * __ldg(v2) + a2 * __ldg(v2 + 1) + a3 * __ldg(v2 + 2) + a4 * __ldg(v2 + 3);
    } else {
      const double x0 = __ldg(xa), x1 = __ldg(xa + 1);
      const double a1 = (x - x1) / (x0 - x1);
      const double a2 = 1.0 - a1;
      p1 = a1 * __ldg(v1) + a2 * __ldg(v1 + 1);
      p2 = a1 * __ldg(v2) + a2 * __ldg(v2 + 1);
    }
    *Dl = p1 * ai;
    *HD = p2;
  } else if (ai >= A.amax) {
    *Dl = A.D0 * ai; *HD = A.H0;
  } else {
    *Dl = A.Dinf * ai; *HD = A.Hinf;
  }
}

// Carlson's RD by duplication until the relative spread is below 0.05, then
// the fifth-order series (at most 200 duplications).  RD(x, y, z) and
// RD(u, y, w) are evaluated together: the two duplication sequences advance in
// one loop (two independent chains of square roots and divisions in flight
// instead of one), each stopping at its own tolerance test, so each result is
// the one a separate evaluation gives
__device__ void rd2(double x, double y, double z, double u, double w, double* r1, double* r2) {
  const double ERRTOL = 0.05, C1 = 3.0 / 14.0, C2 = 1.0 / 6.0, C3 = 9.0 / 22.0, C4 = 3.0 / 26.0;
  const double C5 = 0.25 * C3, C6 = 1.5 * C4;
  double xt = x, yt = y, zt = z, sum = 0.0, fac = 1.0, dx = 0.0, dy = 0.0, dz = 0.0, ave = 0.0;
  double ut = u, vt = y, wt = w, sum2 = 0.0, fac2 = 1.0, du = 0.0, dv = 0.0, dw = 0.0, ave2 = 0.0;
  bool go1 = true, go2 = true;
  for (int it = 0; it < 200 && (go1 || go2); it++) {
    if (go1) {
      const double sx = sqrt(xt), sy = sqrt(yt), sz = sqrt(zt);
      const double al = sx * (sy + sz) + sy * sz;
      sum += fac / (sz * (zt + al));
      fac *= 0.25;
      xt = 0.25 * (xt + al);
      yt = 0.25 * (yt + al);
      zt = 0.25 * (zt + al);
      ave = 0.2 * (xt + yt + 3.0 * zt);
      dx = (ave - xt) / ave;
      dy = (ave - yt) / ave;
      dz = (ave - zt) / ave;
      go1 = !(fmax(fmax(fabs(dx), fabs(dy)), fabs(dz)) <= ERRTOL);
    }
    if (go2) {
      const double su = sqrt(ut), sv = sqrt(vt), sw = sqrt(wt);
      const double al = su * (sv + sw) + sv * sw;
      sum2 += fac2 / (sw * (wt + al));
      fac2 *= 0.25;
      ut = 0.25 * (ut + al);
      vt = 0.25 * (vt + al);
      wt = 0.25 * (wt + al);
      ave2 = 0.2 * (ut + vt + 3.0 * wt);
      du = (ave2 - ut) / ave2;
      dv = (ave2 - vt) / ave2;
      dw = (ave2 - wt) / ave2;
      go2 = !(fmax(fmax(fabs(du), fabs(dv)), fabs(dw)) <= ERRTOL);
    }
  }
  {
    const double ea = dx * dy, eb = dz * dz, ec = ea - eb, ed = ea - 6.0 * eb, ee = ed + ec + ec;
    *r1 = 3.0 * sum + fac * (1.0 + ed * (-C1 + C5 * ed - C6 * dz * ee) + dz * (C2 * ee + dz * (-C3 * ec + dz * C4 * ea))) /
                          (ave * sqrt(ave));
  }
  {
    const double ea = du * dv, eb = dw * dw, ec = ea - eb, ed = ea - 6.0 * eb, ee = ed + ec + ec;
    *r2 = 3.0 * sum2 + fac2 * (1.0 + ed * (-C1 + C5 * ed - C6 * dw * ee) + dw * (C2 * ee + dw * (-C3 * ec + dw * C4 * ea))) /
                           (ave2 * sqrt(ave2));
  }
}

// shape integrals b_1..b_3 of axes a1, a2, a3
__device__ void shape_b(double a1, double a2, double a3, double* b) {
  const double third = 1.0 / 3.0;
  const double r2 = a2 / a1, r3 = a3 / a1;
  if (r3 >= r2) {   // oblate or spherical
    if (r3 >= 0.999) {
      b[0] = third; b[1] = third; b[2] = third;
      return;
    }
    double b3;
    if (r3 <= 0.001) {
      const double e2 = 1.0 - r3 * r3, o2 = r3 * r3, o1 = 0.5 * (r3 * r3), e = sqrt(e2);
      b3 = 0.5 * (o2 / e2 * (1.0 / o2 - ppbm::log_pos((1.0 + e) / o1) * 0.5 / e));
    } else {
      const double e2 = 1.0 - r3 * r3, e = sqrt(e2);
      b3 = 0.5 * ((1.0 - e2) / e2 * (1.0 / (1.0 - e2) - ppbm::log_pos((1.0 + e) / (1.0 - e)) * 0.5 / e));
    }
    b[0] = 1.0 - 2.0 * b3; b[1] = b3; b[2] = b3;
    return;
  }
  const double r22 = r2 * r2, r32 = r3 * r3, q = third * r2 * r3;
  double rd3, rd2v;
  rd2(r22, 1.0, r32, r32, r22, &rd3, &rd2v);   // RD(r2^2, 1, r3^2) and RD(r3^2, 1, r2^2)
  const double b3 = q * rd3, b2 = q * rd2v;
  b[0] = 1.0 - (b2 + b3); b[1] = b2; b[2] = b3;
}

struct Ell {
  int pos;                   // growth-table position of the last lookup
  int lv0, lv1, lv2;         // axis virialised
  double eq0, eq1, eq2;      // frozen axis values
  double a3eq2, a3eq1, Ha;
  double lam0, lam1, lam2, F3;
};

__device__ __forceinline__ double hubble(const TabArgs& A, double a) {
  return sqrt((1.0 + A.Rvac * (a * a * a) + A.Rcurv * a) / a);
}

// force on one axis (dv/da); ya the axis, b its shape integral, lam its
// strain eigenvalue
__device__ __forceinline__ double force(const TabArgs& A, const Ell& S, double ya, double b, double lam, double d0,
                                        double d1i, double d1x, double ab) {
  switch (A.iforce) {
    case 0: return -ya * d1i * b;
    case 1: return -ya * (d1i * b + d0);
    case 3: return -ya * (d1i * b + d0 + d1x * (b - 1.0 / 3.0));
    case 5: return -ya * d0 - d1x * ab * lam;
    default: return -ya * (d1i * b + d0 + d1x * (lam - S.F3));   // 4, 6
  }
}

// get_derivs!: virialisation checks (axis 3 first), frozen axes written back
// into y, then the equations of motion of the live axes
__device__ void derivs(const TabArgs& A, Ell& S, double t, double* y, double* dy) {
#pragma unroll
  for (int i = 0; i < 6; i++) dy[i] = 0.0;
  const double ab = t, ab3 = ab * ab * ab;
  const double Ha = hubble(A, ab);
  S.Ha = Ha;
  const double Hi = 1.0 / Ha;
  if (S.lv2 == 0 && y[2] <= A.fcoll3 * ab) {
    S.lv2 = 1;
    S.eq2 = A.fcoll3 * ab;
    if (A.ivir == 1) { S.a3eq2 = S.eq2 * 1.001; S.a3eq1 = S.eq2 * 1.0003; }
  }
  if (A.ivir == 2 && S.lv1 == 0) S.a3eq2 = A.fcoll2 * ab;
  if (A.ivir == 2 && S.lv0 == 0) S.a3eq1 = A.fcoll1 * ab;
  if (S.lv2 == 1 && y[1] <= S.a3eq2 && S.lv1 == 0) { S.lv1 = 1; S.eq1 = S.a3eq2; }
  if (S.lv2 == 1 && y[0] <= S.a3eq1 && S.lv0 == 0) { S.lv0 = 1; S.eq0 = S.a3eq1; }
  if (S.lv2) { y[2] = S.eq2; y[5] = 0.0; }
  if (S.lv1) { y[1] = S.eq1; y[4] = 0.0; }
  if (S.lv0) { y[0] = S.eq0; y[3] = 0.0; }
  const double a1 = y[0], a2 = y[1], a3 = y[2];
  const double d1e = ab3 / (a1 * a2 * a3);
  double d0, d1i, d1x = 0.0;
  if (A.iforce == 0) {
    d0 = -A.Rvac * Hi;
    d1i = 1.5 * d1e / ab3 * Hi;
  } else {
    d0 = (0.5 / ab3 - A.Rvac) * Hi;
    d1i = 1.5 * (d1e - 1.0) / ab3 * Hi;
    if (A.iforce == 4 || A.iforce == 5 || A.iforce == 6) {
      double dl, hd;
      dlin(A, ab, &dl, &hd, &S.pos);
      d1x = 1.5 / ab3 * Hi * dl;
    } else if (A.iforce == 3) {
      d1x = 1.5 * 2.5 / ab3 * Hi;
    }
  }
  double b[3] = {0.0, 0.0, 0.0};
  if (A.iforce != 5 && A.iforce != 6) shape_b(a1, a2, a3, b);
  if (!S.lv2) { dy[2] = y[5] * Hi; dy[5] = force(A, S, y[2], b[2], S.lam2, d0, d1i, d1x, ab); }
  if (!S.lv1) { dy[1] = y[4] * Hi; dy[4] = force(A, S, y[1], b[1], S.lam1, d0, d1i, d1x, ab); }
  if (!S.lv0) { dy[0] = y[3] * Hi; dy[3] = force(A, S, y[0], b[0], S.lam0, d0, d1i, d1x, ab); }
}

__global__ void __launch_bounds__(64) table_kernel(TabArgs A) {
  const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nn = (int64_t)A.Nx * A.Ny * A.Nz;
  if (node >= nn) return;
  const int i = (int)(node % A.Nx), j = (int)((node / A.Nx) % A.Ny), k = (int)(node / ((int64_t)A.Nx * A.Ny));
  const double ev = A.Y1 + j * A.dY, poe = A.Z1 + k * A.dZ;
  const double Frho = A.Frho[i], pv = poe * ev;
  Ell S{};
  S.lam2 = Frho / 3.0 * (1.0 + 3.0 * ev + pv);
  S.lam1 = Frho / 3.0 * (1.0 - 2.0 * pv);
  S.lam0 = Frho / 3.0 * (1.0 - 3.0 * ev + pv);
  S.F3 = Frho / 3.0;
  const double zinit = A.zinit_fac * Frho;
  const double ab = 1.0 / zinit;
  double t = ab;
  double dl, hd;
  S.pos = 0;
  dlin(A, ab, &dl, &hd, &S.pos);
  const double Ha = hubble(A, ab);
  S.Ha = Ha;
  double y[6], dy[6], yt[6], dyt[6], dym[6];
  y[2] = ab * (1.0 - dl * S.lam2);
  y[1] = ab * (1.0 - dl * S.lam1);
  y[0] = ab * (1.0 - dl * S.lam0);
  y[5] = Ha * (1.0 - (1.0 + hd) * dl * S.lam2);
  y[4] = Ha * (1.0 - (1.0 + hd) * dl * S.lam1);
  y[3] = Ha * (1.0 - (1.0 + hd) * dl * S.lam0);
  double zdyn0 = -1.0;
  int ldyn0 = 0;
  int istep = 0;
  while (true) {   // ends by nstepmax at the latest
    istep++;
    const double a_3 = y[2];
    const double h = A.tfac * a_3 * sqrt(a_3) * S.Ha;
    derivs(A, S, t, y, dy);
    const double hh = h * 0.5, h6 = h / 6.0, xh = t + hh;
#pragma unroll
    for (int c = 0; c < 6; c++) yt[c] = y[c] + hh * dy[c];
    derivs(A, S, xh, yt, dyt);
#pragma unroll
    for (int c = 0; c < 6; c++) yt[c] = y[c] + hh * dyt[c];
    derivs(A, S, xh, yt, dym);
#pragma unroll
    for (int c = 0; c < 6; c++) {
      yt[c] = y[c] + h * dym[c];
      dym[c] = dyt[c] + dym[c];
    }
    derivs(A, S, t + h, yt, dyt);
#pragma unroll
    for (int c = 0; c < 6; c++) y[c] = y[c] + h6 * (dy[c] + dyt[c] + 2.0 * dym[c]);
    t += h;
    // only axis 1's virialisation redshift is returned (idynax = 1); the
    // reference's other event records do not feed the table
    if (S.lv0 != ldyn0) {
      zdyn0 = 1.0 / t;
      ldyn0 = 1;
    }
    if (S.lv0 == 1 || istep >= A.nstepmax || t >= 2.0) break;
  }
  A.out[node] = zdyn0;
  atomicAdd(A.steps, (unsigned long long)istep);
}

}  // namespace

void make_table_device(Slot& sl, const GrowthTable& G, const ppb_table_params* p, const double* d_Frho, double* d_out,
                       unsigned long long* d_steps) {
  TabArgs A{};
  A.Frho = d_Frho;
  A.Nx = p->Nx; A.Ny = p->Ny; A.Nz = p->Nz;
  A.Y1 = p->Y1; A.Z1 = p->Z1;
  A.dY = (p->Y2 - p->Y1) / (p->Ny - 1);
  A.dZ = (p->Z2 - p->Z1) / (p->Nz - 1);
  A.iforce = p->iforce_strat;
  A.ivir = p->ivir_strat;
  A.nstepmax = p->nstepmax;
  A.fcoll1 = p->fcoll_1; A.fcoll2 = p->fcoll_2; A.fcoll3 = p->fcoll_3;
  A.tfac = p->tfac;
  A.zinit_fac = p->zinit_fac;
  A.Rvac = p->OL / p->Om;
  A.Rcurv = (1.0 - p->Om - p->OL) / p->Om;
  const size_t ng = G.a.size();
  sl.g_a.ensure(ng * 8);
  sl.g_D.ensure(ng * 8);
  sl.g_f.ensure(ng * 8);
  PPB_CUDA(cudaMemcpyAsync(sl.g_a.p, G.a.data(), ng * 8, cudaMemcpyHostToDevice, sl.stream));
  PPB_CUDA(cudaMemcpyAsync(sl.g_D.p, G.D.data(), ng * 8, cudaMemcpyHostToDevice, sl.stream));
  PPB_CUDA(cudaMemcpyAsync(sl.g_f.p, G.f.data(), ng * 8, cudaMemcpyHostToDevice, sl.stream));
  A.ga = sl.g_a.as<double>();
  A.gD = sl.g_D.as<double>();
  A.gf = sl.g_f.as<double>();
  A.ng = (int)ng;
  A.amin = G.amin; A.amax = G.amax; A.Dinf = G.Dinf; A.D0 = G.D0; A.Hinf = G.Hinf; A.H0 = G.H0;
  A.out = d_out;
  A.steps = d_steps;
  const int64_t nn = (int64_t)p->Nx * p->Ny * p->Nz;
  table_kernel<<<(unsigned)((nn + 63) / 64), 64, 0, sl.stream>>>(A);
  PPB_LAUNCHED(sl.launches);
}

}  // namespace ppb
