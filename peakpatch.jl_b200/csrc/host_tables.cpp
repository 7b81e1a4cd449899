// host_tables.cpp — host-side tables of the path, in double precision:
// the sorted shell-cell list (precompute_shells), the linear growth table
// (Dlinear_tables / Dlinear_ab / fsc_of_z) and the chi -> z table.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <utility>

#include "ppb_internal.h"

namespace ppb {

// precompute_shells (src/HaloFinder/RadialShell.jl:160-175): all offsets with
// r^2 <= nhunt^2 in construction order dk, dj, di, stable-sorted by r^2.
void build_shell_table(ShellTable& st, int nhunt) {
  PPB_REQUIRE(nhunt >= 1 && nhunt <= 64, "nhunt must be in [1, 64]");
  if (st.nhunt == nhunt) return;
  st.cells.clear();
  const int r2max = nhunt * nhunt;
  for (int dk = -nhunt; dk <= nhunt; dk++)
    for (int dj = -nhunt; dj <= nhunt; dj++)
      for (int di = -nhunt; di <= nhunt; di++) {
        const int r2 = di * di + dj * dj + dk * dk;
        if (r2 <= r2max) st.cells.push_back(make_int4(di, dj, dk, r2));
      }
  std::stable_sort(st.cells.begin(), st.cells.end(), [](const int4& a, const int4& b) { return a.w < b.w; });
  st.ncells = (int64_t)st.cells.size();
  st.shell_start.clear();
  st.shell_count.clear();
  st.shell_r2.clear();
  for (int64_t i = 0; i < st.ncells; i++) {
    if (i == 0 || st.cells[i].w != st.cells[i - 1].w) {
      st.shell_start.push_back((int32_t)i);
      st.shell_count.push_back(0);
      st.shell_r2.push_back(st.cells[i].w);
    }
    st.shell_count.back()++;
  }
  st.nshell = (int)st.shell_r2.size();
  st.cell8.resize(st.cells.size());
  for (size_t i = 0; i < st.cells.size(); i++) {
    const int4 c = st.cells[i];
    st.cell8[i] = (int32_t)((uint32_t)(c.x & 0xff) | ((uint32_t)(c.y & 0xff) << 8) | ((uint32_t)(c.z & 0xff) << 16));
  }
  // shell m (1-based) = distinct value m-1; rad[m] = sqrt(r2)
  st.rad.assign(st.nshell + 1, 0.0);
  st.r2m.assign(st.nshell + 1, 0);
  for (int m = 1; m <= st.nshell; m++) {
    st.r2m[m] = st.shell_r2[m - 1];
    st.rad[m] = std::sqrt((double)st.r2m[m]);
  }
  // kernel_strain windows and weights for centre shells mp = 2..mmax
  const int mmax = std::max(st.nshell - 1, 1);
  st.win_lo.assign(st.nshell + 1, 0);
  st.win_hi.assign(st.nshell + 1, -1);
  st.win_off.assign(st.nshell + 1, 0);
  st.wts.clear();
  for (int mp = 2; mp <= mmax; mp++) {
    int lo = -1, hi = -2;
    for (int m1 = 1; m1 <= mmax; m1++) {
      const double u0 = st.rad[mp] - st.rad[m1];
      if (u0 * u0 < 4.0) {
        if (lo < 0) lo = m1;
        hi = m1;
      }
    }
    st.win_lo[mp] = lo;
    st.win_hi[mp] = hi;
    st.win_off[mp] = (int32_t)st.wts.size();
    for (int m1 = lo; m1 <= hi; m1++) {
      const double u0 = st.rad[mp] - st.rad[m1];
      const double u02 = u0 * u0;
      const double u12 = st.rad[mp] * st.rad[mp] + st.rad[m1] * st.rad[m1];
      const double d = u12 - u02;
      st.wts.push_back(hRinteg(u0, u12) / (d * d));
    }
  }
  // mp == 1 weights
  const std::vector<double> akk = make_atab4();
  st.w1.assign(st.nshell + 1, 0.0);
  for (int m1 = 1; m1 <= mmax; m1++) {
    const double u0 = st.rad[m1];
    const double con = 100.0 * u0 * u0;
    const long long icon = (long long)std::floor(con);
    if (icon + 1 > 1100) {
      st.w1[m1] = std::nan("");
      continue;
    }
    const double diff = con - (double)icon;
    const double aww = akk[icon] + diff * (akk[icon + 1] - akk[icon]);
    st.w1[m1] = 0.5 * aww / st.rad[m1];
  }
  // gather truncation targets
  st.need.assign(st.nshell + 1, mmax);
  for (int m = 1; m <= mmax; m++) {
    int l = m;
    while (l + 1 <= mmax && st.rad[l + 1] <= st.rad[m] + 2.0) l++;
    st.need[m] = std::min(mmax, l + 2);
  }
  st.rad5.assign(st.nshell + 1, 0.0);
  for (int m = 1; m <= st.nshell; m++) st.rad5[m] = std::pow(st.rad[m], 5);
  // gather schedule (shells 2..mmax; shell m is distinct value m-1)
  st.grp_a.clear(); st.grp_b.clear(); st.grp_c.clear();
  st.ck_s.clear(); st.ck_n.clear(); st.ck_d.clear();
  st.sh_c0.assign(st.nshell + 1, 0);
  st.sh_nc.assign(st.nshell + 1, 0);
  int in_group = 0;
  // chunk size: kChunkCells, smaller (down to 4 cells) when the whole list
  // would leave most of the 32 lanes of one group idle (small nhunt: few,
  // small shells), so that the lanes split the cells of each shell
  int total = 0;
  for (int m = 2; m <= mmax; m++) total += st.shell_count[m - 1];
  const int csize = std::min(kChunkCells, std::max(4, 4 * ((total + 127) / 128)));
  for (int m = 2; m <= mmax; m++) {
    const int cnt = st.shell_count[m - 1], s0 = st.shell_start[m - 1];
    int nck = (cnt + csize - 1) / csize;
    if (nck > 32) nck = 32;
    if (nck < 1) nck = 1;
    if (in_group + nck > 32 || st.grp_a.empty()) {   // open a new group
      if (!st.grp_a.empty()) st.grp_b.back() = m - 1;
      st.grp_a.push_back(m);
      st.grp_b.push_back(m);
      st.grp_c.push_back((int32_t)st.ck_s.size());
      in_group = 0;
    }
    st.sh_c0[m] = (int32_t)st.ck_s.size();
    st.sh_nc[m] = nck;
    for (int c = 0; c < nck; c++) {   // near-equal chunk sizes
      const int a = (int)((int64_t)cnt * c / nck), b = (int)((int64_t)cnt * (c + 1) / nck);
      st.ck_s.push_back(s0 + a);
      st.ck_n.push_back(b - a);
      int dm = 0;
      for (int i = s0 + a; i < s0 + b; i++) {
        const int w = st.cell8[i];
        dm = std::max({dm, std::abs((w << 24) >> 24), std::abs((w << 16) >> 24), std::abs((w << 8) >> 24)});
      }
      st.ck_d.push_back(dm);
    }
    in_group += nck;
    st.grp_b.back() = m;
  }
  st.ngroups = (int)st.grp_a.size();
  st.grp_c.push_back((int32_t)st.ck_s.size());
  // chunk-major packed offsets, each chunk padded to a multiple of 4 cells
  st.ck_p.clear();
  st.ck_cells.clear();
  for (size_t c = 0; c < st.ck_s.size(); c++) {
    st.ck_p.push_back((int32_t)(st.ck_cells.size() / 4));
    for (int i = 0; i < st.ck_n[c]; i++) st.ck_cells.push_back(st.cell8[st.ck_s[c] + i]);
    while (st.ck_cells.size() % 4) st.ck_cells.push_back(0);
  }
  st.nhunt = nhunt;
  st.d_cell8.release();   // force re-upload
}

// hRinteg (src/HaloFinder/RadialShell.jl:100-127)
double hRinteg(double u0, double u12) {
  const double x0 = std::fabs(u0);
  if (x0 >= 2.0) return 0.0;
  const double one7 = 1.0 / 7.0;
  double result = 1.6 * u12 - 6.4 * one7;
  const double x02 = x0 * x0, x04 = x02 * x02;
  if (x0 >= 1.0) {
    const double h1 = x04 * (2.0 - x0 * (2.4 - x0 * (1.0 - x0 * one7)));
    const double h2 = x02 * (4.0 - x0 * (4.0 - x0 * (1.5 - x0 * 0.2)));
    result = result - h2 * u12 + h1;
  } else {
    result = result - 0.2 * (u12 - one7);
    if (x0 > 0.0) {
      const double h1 = x04 * (1.0 - x02 * (1.0 - 3.0 * x0 * one7));
      const double h2 = x02 * (2.0 - x02 * (1.5 - 0.6 * x0));
      result = result - h2 * u12 + h1;
    }
  }
  return result;
}

// SPH kernel table akk (RadialShell.jl:133-150), 1101 entries, 0-based
std::vector<double> make_atab4() {
  std::vector<double> akk(1101);
  const double pi = 3.141592653589793, ca = 3.0 / (2.0 * pi), cb = 1.0 / (4.0 * pi);
  for (int i = 1; i <= 1100; i++) {
    const double u = (i - 1) * 0.01, ru = std::sqrt(u);
    double v;
    if (ru < 1.0) v = ca * (2.0 / 3.0 - u + 0.5 * u * ru);
    else if (ru <= 2.0) v = cb * (2.0 - ru) * (2.0 - ru) * (2.0 - ru);
    else v = 0.0;
    akk[i - 1] = v;
  }
  akk[1100] = 0.0;
  return akk;
}

void upload_shell_table(ShellTable& st, cudaStream_t s) {
  if (st.d_cell8.p && st.d_cell8.bytes >= st.cell8.size() * sizeof(int32_t)) return;
  st.d_cell8.ensure(st.cell8.size() * sizeof(int32_t));
  st.d_start.ensure(st.shell_start.size() * sizeof(int32_t));
  st.d_count.ensure(st.shell_count.size() * sizeof(int32_t));
  st.d_r2m.ensure(st.r2m.size() * sizeof(int32_t));
  st.d_rad.ensure(st.rad.size() * sizeof(double));
  PPB_CUDA(cudaMemcpyAsync(st.d_cell8.p, st.cell8.data(), st.cell8.size() * 4, cudaMemcpyHostToDevice, s));
  PPB_CUDA(cudaMemcpyAsync(st.d_start.p, st.shell_start.data(), st.shell_start.size() * 4, cudaMemcpyHostToDevice, s));
  PPB_CUDA(cudaMemcpyAsync(st.d_count.p, st.shell_count.data(), st.shell_count.size() * 4, cudaMemcpyHostToDevice, s));
  PPB_CUDA(cudaMemcpyAsync(st.d_r2m.p, st.r2m.data(), st.r2m.size() * 4, cudaMemcpyHostToDevice, s));
  PPB_CUDA(cudaMemcpyAsync(st.d_rad.p, st.rad.data(), st.rad.size() * 8, cudaMemcpyHostToDevice, s));
  auto up = [&](DevBuf& b, const void* src, size_t bytes) {
    b.ensure(std::max<size_t>(bytes, 8));
    if (bytes) PPB_CUDA(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, s));
  };
  up(st.d_wlo, st.win_lo.data(), st.win_lo.size() * 4);
  up(st.d_whi, st.win_hi.data(), st.win_hi.size() * 4);
  up(st.d_woff, st.win_off.data(), st.win_off.size() * 4);
  up(st.d_wts, st.wts.data(), st.wts.size() * 8);
  up(st.d_w1, st.w1.data(), st.w1.size() * 8);
  up(st.d_need, st.need.data(), st.need.size() * 4);
  up(st.d_rad5, st.rad5.data(), st.rad5.size() * 8);
  up(st.d_grp_a, st.grp_a.data(), st.grp_a.size() * 4);
  up(st.d_grp_b, st.grp_b.data(), st.grp_b.size() * 4);
  up(st.d_grp_c, st.grp_c.data(), st.grp_c.size() * 4);
  up(st.d_ck_s, st.ck_s.data(), st.ck_s.size() * 4);
  up(st.d_ck_n, st.ck_n.data(), st.ck_n.size() * 4);
  up(st.d_ck_d, st.ck_d.data(), st.ck_d.size() * 4);
  up(st.d_sh_c0, st.sh_c0.data(), st.sh_c0.size() * 4);
  up(st.d_sh_nc, st.sh_nc.data(), st.sh_nc.size() * 4);
  up(st.d_ck_p, st.ck_p.data(), st.ck_p.size() * 4);
  up(st.d_ck_cells, st.ck_cells.data(), st.ck_cells.size() * 4);
  PPB_CUDA(cudaStreamSynchronize(s));
}

// ---------------------------------------------------------------------------
// Linear growth: RK4 in ln a over 2000 steps from a = 1e-7 to 2, tabulating
// a in [1/1001, 2] (src/Cosmology/Cosmology.jl:121-202 and 148-202 of the
// Dlinear_tables listing; the derivative set is the reference's
// _deriv_Dlin! with no radiation, decaying or hot components).
// ---------------------------------------------------------------------------
namespace {
struct DerivArgs {
  double h, Omnr, Omvac, Omcurv, OmX, OmB;
};
void deriv(const DerivArgs& q, const double* y, double* d, double a) {
  const double a3 = a * a * a;
  const double hub = q.Omnr + q.Omvac * a3 + q.Omcurv * a;
  d[0] = 1.0 / (q.h * std::sqrt(hub / a3));
  const double fb = y[2];
  d[1] = fb;
  const double qs = 0.5 / hub;
  const double qv = qs * (q.Omnr - 2.0 * q.Omvac * a3);
  double fnr = (q.OmX + q.OmB) / q.Omnr;
  if (q.OmB != 0.0 && a <= 1.0e-3) fnr = q.OmX / q.Omnr;
  const double qf = qs * (q.Omnr * fnr);
  d[2] = 3.0 * qf - fb * fb - (1.0 - qv) * fb;
  d[3] = 0.0;
  d[4] = d[0] / a;
}
}  // namespace

GrowthTable make_growth_table(double Om, double OB, double OL, double h) {
  DerivArgs q{h, Om, OL, 1.0 - Om - OL, Om - OB, OB};
  const double amaxtab = 2.0, amintab_target = 1.0 / 1001.0, ainit = 1.0e-7;
  const int nmax = 2000;
  double a = ainit, alogn = std::log(ainit);
  const double hh = (std::log(amaxtab) - alogn) / nmax;
  const double t0 = 1.0 / h / std::sqrt(Om);
  const double ya = std::sqrt(a);
  double y[5] = {t0 * (2.0 / 3.0 * (ya * ya * ya)), std::log(a),
                 0.25 * (std::sqrt(24.0 * q.OmX / Om + 1.0) - 1.0), 0.0, t0 * 2.0 * ya};
  GrowthTable G;
  int lnorm = 1, ip0 = 0;
  double bnorm = 1.0;
  for (int i = 0; i < nmax; i++) {
    double w1[5], w2[5], w3[5], w4[5], yt[5];
    deriv(q, y, w1, a);
    const double ah = std::exp(alogn + hh * 0.5);
    for (int c = 0; c < 5; c++) yt[c] = y[c] + hh * w1[c] * 0.5;
    deriv(q, yt, w2, ah);
    for (int c = 0; c < 5; c++) yt[c] = y[c] + hh * w2[c] * 0.5;
    deriv(q, yt, w3, ah);
    const double an = alogn + hh, anew = std::exp(an);
    for (int c = 0; c < 5; c++) yt[c] = y[c] + hh * w3[c];
    deriv(q, yt, w4, anew);
    for (int c = 0; c < 5; c++) y[c] = y[c] + hh / 6.0 * (w1[c] + w4[c] + 2.0 * (w2[c] + w3[c]));
    alogn = an;
    a = anew;
    if (lnorm == 1 && a >= 0.001) {
      lnorm = 0;
      bnorm = std::exp(y[1]) / a;
    }
    if (a >= amintab_target && a <= amaxtab) {
      G.a.push_back(a);
      G.D.push_back(std::exp(y[1]) / a);
      G.f.push_back(y[2]);
      if (a >= 1.0 && ip0 == 0) ip0 = (int)G.a.size();
    }
  }
  double fac;
  if (ip0 > 1) {
    const double ai = (G.a[ip0 - 1] - 1.0) / (G.a[ip0 - 1] - G.a[ip0 - 2]);
    const double Dag = (G.D[ip0 - 1] * (1.0 - ai) + G.D[ip0 - 2] * ai) / bnorm;
    fac = 1.0 / (Dag * bnorm);
  } else {
    fac = 1.0 / bnorm;
  }
  for (auto& v : G.D) v *= fac;
  G.amin = G.a.front();
  G.amax = G.a.back();
  G.Dinf = G.D.front();
  G.D0 = G.D.back();
  G.Hinf = G.f.front();
  G.H0 = G.f.back();
  return G;
}

// Dlinear_ab (Cosmology.jl:420-440 of the listing): bisection "hunt", then a
// 4-point (2-point at the ends) Lagrange interpolation of D(a)/a and dlnD/dlna.
void dlinear_ab(const GrowthTable& G, double ai, double* Dl, double* HD, double* Da) {
  const int ntab = (int)G.a.size();
  if (ai > G.amin && ai < G.amax) {
    int jlo = 0, jhi = ntab + 1;
    while (jhi - jlo > 1) {
      const int jm = (jhi + jlo) / 2;
      if (ai > G.a[jm - 1]) jlo = jm; else jhi = jm;
    }
    const int kk = jlo;
    int nl, kkl;
    if (kk < 2 || kk >= ntab) { nl = 2; kkl = std::max(kk - 1, 1); } else { nl = 4; kkl = kk - 2; }
    const double* xa = &G.a[kkl - 1];
    const double* v1 = &G.D[kkl - 1];
    const double* v2 = &G.f[kkl - 1];
    const double x = ai;
    double p1, p2;
    if (nl == 4) {
      const double a1 = (x - xa[1]) / (xa[0] - xa[1]) * (x - xa[2]) / (xa[0] - xa[2]) * (x - xa[3]) / (xa[0] - xa[3]);
      const double a2 = (x - xa[0]) / (xa[1] - xa[0]) * (x - xa[2]) / (xa[1] - xa[2]) * (x - xa[3]) / (xa[1] - xa[3]);
      const double a3 = (x - xa[0]) / (xa[2] - xa[0]) * (x - xa[1]) / (xa[2] - xa[1]) * (x - xa[3]) / (xa[2] - xa[3]);
      const double a4 = (x - xa[0]) / (xa[3] - xa[0]) * (x - xa[1]) / (xa[3] - xa[1]) * (x - xa[2]) / (xa[3] - xa[2]);
      p1 = a1 * v1[0] + a2 * v1[1] + a3 * v1[2] + a4 * v1[3];
      p2 = a1 * v2[0] + a2 * v2[1] + a3 * v2[2] + a4 * v2[3];
    } else {
      const double a1 = (x - xa[1]) / (xa[0] - xa[1]);
      const double a2 = 1.0 - a1;
      p1 = a1 * v1[0] + a2 * v1[1];
      p2 = a1 * v2[0] + a2 * v2[1];
    }
    *Dl = p1 * ai;
    *HD = p2;
    *Da = p1;
  } else if (ai >= G.amax) {
    *Dl = G.D0 * ai; *HD = G.H0; *Da = G.D0;
  } else {
    *Dl = G.Dinf * ai; *HD = G.Hinf; *Da = G.Dinf;
  }
}

// fsc_of_z (RadialShell.jl:191-196): 1.686 D(1/(1+z))
double fsc_of_z(const GrowthTable& G, double z) {
  double d, hd, da;
  dlinear_ab(G, 1.0 / (1.0 + z), &d, &hd, &da);
  return 1.686 * d;
}

// chi(z) in Mpc/h = (c/100) h * int_0^z dz'/E(z'), flat LCDM
// (Cosmology.jl:15-24); adaptive 7/15-point Gauss-Kronrod quadrature.
namespace {
double gk15(double Om, double OL, double a, double b, double* err) {
  static const double xk[8] = {0.991455371120812639206854697526329, 0.949107912342758524526189684047851,
                               0.864864423359769072789712788640926, 0.741531185599394439863864773280788,
                               0.586087235467691130294144845693013, 0.405845151377397166906606412076961,
                               0.207784955007898467600689403773245, 0.0};
  static const double wk[8] = {0.022935322010529224963732008058970, 0.063092092629978553290700663189204,
                               0.104790010322250183839876322541518, 0.140653259715525918745189590510238,
                               0.169004726639267902826583426598550, 0.190350578064785409913256402421014,
                               0.204432940075298892414161999234649, 0.209482141084727828012999174891714};
  static const double wg[4] = {0.129484966168869693270611432679082, 0.279705391489276667901467771423780,
                               0.381830050505118944950369775488975, 0.417959183673469387755102040816327};
  auto f = [&](double z) { return 1.0 / std::sqrt(Om * (1 + z) * (1 + z) * (1 + z) + OL); };
  const double c = 0.5 * (a + b), hl = 0.5 * (b - a);
  const double fc = f(c);
  double rk = fc * wk[7], rg = fc * wg[3];
  for (int j = 0; j < 7; j++) {
    const double dx = hl * xk[j];
    const double s = f(c - dx) + f(c + dx);
    rk += wk[j] * s;
    if (j % 2 == 1) rg += wg[j / 2] * s;
  }
  *err = std::fabs((rk - rg) * hl);
  return rk * hl;
}
}  // namespace

double chi_of_z(double Om, double OL, double h, double z) {
  if (z == 0.0) return 0.0;
  std::vector<std::pair<double, double>> st{{0.0, z}};
  double tot = 0.0;
  while (!st.empty()) {
    const auto ab = st.back();
    st.pop_back();
    double e;
    const double v = gk15(Om, OL, ab.first, ab.second, &e);
    if (e <= 1e-14 * std::fabs(v) || (ab.second - ab.first) < 1e-9) tot += v;
    else {
      const double m = 0.5 * (ab.first + ab.second);
      st.push_back({ab.first, m});
      st.push_back({m, ab.second});
    }
  }
  return (2.998e5 / 100.0) * h * tot;
}

// build_chi_to_z (Cosmology.jl:144-148): chi at npts redshifts 0..zmax
double chi_to_z_host(const std::vector<double>& chis, double zmax, double c) {
  const int n = (int)chis.size();
  if (c <= chis[0]) return 0.0;
  if (c >= chis[n - 1]) return zmax;
  int lo = 1, hi = n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (chis[mid - 1] <= c) lo = mid; else hi = mid;
  }
  const double zl = zmax * (double)(lo - 1) / (double)(n - 1);
  const double zh = zmax * (double)(hi - 1) / (double)(n - 1);
  const double fr = (c - chis[lo - 1]) / (chis[hi - 1] - chis[lo - 1]);
  return zl + fr * (zh - zl);
}

std::vector<double> make_chi_table(double Om, double OL, double h, double zmax, int npts) {
  std::vector<double> c(npts);
  for (int i = 0; i < npts; i++) {
    const double z = npts == 1 ? 0.0 : zmax * (double)i / (double)(npts - 1);
    c[i] = chi_of_z(Om, OL, h, z);
  }
  return c;
}

}  // namespace ppb
