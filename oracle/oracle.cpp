// oracle.cpp — CPU restatement of PeakPatch.jl's per-tile halo-finding path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests, the
// smoke check and the CPU-baseline leg of bench.py call it; the product
// library never links or calls it.  It follows the reference's Julia code
// step by step in double precision (the reference accumulates shell sums in
// Float64), and each function names the file:line it restates.  FFTs are not
// here: oracle.py drives numpy/scipy FFTs between the k-space steps below.
//
// The white-noise generator shares the header ppb_math.h with the product so
// that the noise can be compared bit for bit (see that header for why).
//
// Parity pins (tests/test_oracle_*.py): the reference's own known-answer
// tests for hRinteg, atab4, precompute_shells, get_evals, normalize_strain,
// find_peaks, the trilinear collapse-table lookup, the filter windows, the
// .pksc layout, and the single-peak Fortran get_homel golden values of
// test/test_radialshell_fortran.jl.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include <complex>
#include <atomic>
#include <omp.h>

#include "../peakpatch.jl_b200/csrc/ppb_math.h"

using c64 = std::complex<float>;
static const double PI = 3.141592653589793;

extern "C" {

int ora_num_threads(void) { return omp_get_max_threads(); }
void ora_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }

// ---------------------------------------------------------------------------
// White noise.  RandomField.jl:70-83 (fill_noise_threefry!) and :95-109
// (fill_noise_threefry_region!).  Array is column-major (i fastest).
// ---------------------------------------------------------------------------
void ora_noise(float* out, int64_t n, uint64_t seed) {
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < n; k++)
    for (int64_t j = 0; j < n; j++)
      for (int64_t i = 0; i < n; i++) {
        const uint64_t lin = (uint64_t)(i + n * j + n * n * k);
        out[i + n * j + n * n * k] = ppbm::noise_cell(seed, lin);
      }
}

// Same noise with the platform libm (glibc log/sqrt/cos/sin) in the
// Box-Muller step: a cross-check of the shared implementation in ppb_math.h.
void ora_noise_libm(float* out, int64_t n, uint64_t seed) {
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < n; k++)
    for (int64_t j = 0; j < n; j++)
      for (int64_t i = 0; i < n; i++) {
        const uint64_t lin = (uint64_t)(i + n * j + n * n * k);
        uint64_t a, b;
        ppbm::threefry2x64_20(seed, 0, lin >> 1, 0, &a, &b);
        const double u1 = ((double)(a >> 11) + 1.0) * 0x1.0p-53, u2 = ((double)(b >> 11) + 1.0) * 0x1.0p-53;
        const double r = std::sqrt(-2.0 * std::log(u1)), th = 6.283185307179586 * u2;
        out[i + n * j + n * n * k] = (float)((lin & 1) ? r * std::sin(th) : r * std::cos(th));
      }
}

void ora_noise_region(float* out, int64_t n, uint64_t seed, int64_t i0, int64_t ni,
                      int64_t j0, int64_t nj, int64_t k0, int64_t nk) {
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < nk; k++)
    for (int64_t j = 0; j < nj; j++)
      for (int64_t i = 0; i < ni; i++) {
        const uint64_t lin = (uint64_t)((i0 + i) + n * (j0 + j) + n * n * (k0 + k));
        out[i + ni * j + ni * nj * k] = ppbm::noise_cell(seed, lin);
      }
}

// ---------------------------------------------------------------------------
// P(k) table: log-log linear interpolation with linear extrapolation in
// log-log beyond the ends.  PowerSpectrum.jl:11-30 (Interpolations.jl
// Gridded(Linear()) + extrapolate(Line())).
// ---------------------------------------------------------------------------
static double pk_eval(const double* lk, const double* lp, int np, double k) {
  const double x = std::log(k);
  int i;
  if (x <= lk[0]) i = 0;
  else if (x >= lk[np - 1]) i = np - 2;
  else {
    int lo = 0, hi = np - 1;
    while (hi - lo > 1) { int mid = (lo + hi) / 2; if (lk[mid] <= x) lo = mid; else hi = mid; }
    i = lo;
  }
  const double t = (x - lk[i]) / (lk[i + 1] - lk[i]);
  return std::exp(lp[i] * (1.0 - t) + lp[i + 1] * t);
}

double ora_pk(const double* k, const double* pk, int np, double kq) {
  std::vector<double> lk(np), lp(np);
  for (int i = 0; i < np; i++) { lk[i] = std::log(k[i]); lp[i] = std::log(pk[i]); }
  return pk_eval(lk.data(), lp.data(), np, kq);
}

// AbstractFFTs frequencies: element idx of fftfreq(n, fs) is
// (idx - (idx >= ceil(n/2)? n : 0)) * (fs/n); rfftfreq keeps idx in 0..n/2.
static inline double freq(int64_t idx, int64_t n, double mult) {
  const int64_t nn = (n + 1) / 2;   // count of non-negative frequencies in fftfreq
  const int64_t v = idx < nn ? idx : idx - n;
  return (double)v * mult;
}

// noise_k *= sqrt(P(k) dk^3 n^3), DC := 0.  RandomField.jl:136-168.
// Layout: [iz][iy][ix] with ix in 0..n/2 fastest.
void ora_convolve(c64* nk, int64_t n, double boxsize, const double* k, const double* pk, int np) {
  std::vector<double> lk(np), lp(np);
  for (int i = 0; i < np; i++) { lk[i] = std::log(k[i]); lp[i] = std::log(pk[i]); }
  const double dk = 2.0 * PI / boxsize;
  const double mult = (n * dk) / (double)n;
  const int64_t nh = n / 2 + 1;
  const double nd = (double)n;
#pragma omp parallel for schedule(static)
  for (int64_t iz = 0; iz < n; iz++)
    for (int64_t iy = 0; iy < n; iy++)
      for (int64_t ix = 0; ix < nh; ix++) {
        const double kx = (double)ix * mult, ky = freq(iy, n, mult), kz = freq(iz, n, mult);
        const double k2 = kx * kx + ky * ky + kz * kz;
        c64& v = nk[ix + nh * (iy + n * iz)];
        if (k2 == 0.0) { v = c64(0.f, 0.f); continue; }
        const double kk = std::sqrt(k2);
        const double amp = std::sqrt(pk_eval(lk.data(), lp.data(), np, kk) * (dk * dk * dk) * (nd * nd * nd));
        v = c64((float)((double)v.real() * amp), (float)((double)v.imag() * amp));
      }
}

// 1LPT: psi_i(k) = i k_i/k^2 delta_k, DC and Nyquist planes zeroed.
// LPT.jl:21-71.  out holds 3 consecutive k-grids (x, y, z).
void ora_lpt1(const c64* dkf, c64* out, int64_t n, double boxsize) {
  const double dk = 2.0 * PI / boxsize;
  const double mult = (n * dk) / (double)n;
  const int64_t nh = n / 2 + 1, M = nh * n * n;
#pragma omp parallel for schedule(static)
  for (int64_t iz = 0; iz < n; iz++)
    for (int64_t iy = 0; iy < n; iy++)
      for (int64_t ix = 0; ix < nh; ix++) {
        const int64_t id = ix + nh * (iy + n * iz);
        const double kv[3] = {(double)ix * mult, freq(iy, n, mult), freq(iz, n, mult)};
        const double k2 = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
        const bool nyq = (ix == nh - 1) || (iy == n / 2) || (iz == n / 2);
        for (int c = 0; c < 3; c++) {
          if (k2 == 0.0 || nyq) { out[c * M + id] = c64(0.f, 0.f); continue; }
          const double q = kv[c] / k2;
          const c64 d = dkf[id];
          out[c * M + id] = c64((float)(-q * (double)d.imag()), (float)(q * (double)d.real()));
        }
      }
}

// 2LPT phi_ij = -k_i k_j / k^2 delta_k (no Nyquist zeroing), order
// 11, 22, 33, 12, 13, 23.  LPT.jl:103-128.
void ora_phi(const c64* dkf, c64* out, int64_t n, double boxsize) {
  const double dk = 2.0 * PI / boxsize;
  const double mult = (n * dk) / (double)n;
  const int64_t nh = n / 2 + 1, M = nh * n * n;
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
#pragma omp parallel for schedule(static)
  for (int64_t iz = 0; iz < n; iz++)
    for (int64_t iy = 0; iy < n; iy++)
      for (int64_t ix = 0; ix < nh; ix++) {
        const int64_t id = ix + nh * (iy + n * iz);
        const double kv[3] = {(double)ix * mult, freq(iy, n, mult), freq(iz, n, mult)};
        const double k2 = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
        for (int c = 0; c < 6; c++) {
          if (k2 == 0.0) { out[c * M + id] = c64(0.f, 0.f); continue; }
          const double q = (-kv[pa[c]]) * kv[pb[c]] / k2;
          const c64 d = dkf[id];
          out[c * M + id] = c64((float)(q * (double)d.real()), (float)(q * (double)d.imag()));
        }
      }
}

// src2 = phi11 phi22 - phi12^2 + phi11 phi33 - phi13^2 + phi22 phi33 - phi23^2
// in Float32, evaluated left to right.  LPT.jl:141-143.
void ora_src2(const float* phi, float* out, int64_t N) {
  const float *p11 = phi, *p22 = phi + N, *p33 = phi + 2 * N, *p12 = phi + 3 * N, *p13 = phi + 4 * N, *p23 = phi + 5 * N;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < N; i++) {
    volatile float t = p11[i] * p22[i];
    t = t - p12[i] * p12[i];
    t = t + p11[i] * p33[i];
    t = t - p13[i] * p13[i];
    t = t + p22[i] * p33[i];
    t = t - p23[i] * p23[i];
    out[i] = t;
  }
}

// 2LPT displacement psi2_i = -i k_i/k^2 src2_k with Nyquist zeroing.
// LPT.jl:155-182.
void ora_lpt2(const c64* s2k, c64* out, int64_t n, double boxsize) {
  const double dk = 2.0 * PI / boxsize;
  const double mult = (n * dk) / (double)n;
  const int64_t nh = n / 2 + 1, M = nh * n * n;
#pragma omp parallel for schedule(static)
  for (int64_t iz = 0; iz < n; iz++)
    for (int64_t iy = 0; iy < n; iy++)
      for (int64_t ix = 0; ix < nh; ix++) {
        const int64_t id = ix + nh * (iy + n * iz);
        const double kv[3] = {(double)ix * mult, freq(iy, n, mult), freq(iz, n, mult)};
        const double k2 = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
        const bool nyq = (ix == nh - 1) || (iy == n / 2) || (iz == n / 2);
        for (int c = 0; c < 3; c++) {
          if (k2 == 0.0 || nyq) { out[c * M + id] = c64(0.f, 0.f); continue; }
          const double q = kv[c] / k2;
          const c64 s = s2k[id];
          out[c * M + id] = c64((float)(q * (double)s.imag()), (float)(-q * (double)s.real()));
        }
      }
}

// Laplacian weight k^2 (Float32 k-math): Pipeline.jl:35-51.  The caller
// divides the irfft by n^3 once more.
void ora_lapd_k(const c64* dkf, c64* out, int64_t n, double boxsize) {
  const float dk = (float)(2.0 * PI / boxsize);
  const int64_t nh = n / 2 + 1, nyq = n / 2;
#pragma omp parallel for schedule(static)
  for (int64_t iz = 0; iz < n; iz++)
    for (int64_t iy = 0; iy < n; iy++)
      for (int64_t ix = 0; ix < nh; ix++) {
        const int64_t id = ix + nh * (iy + n * iz);
        const float kx = (float)ix * dk;
        const float ky = (float)(iy <= nyq ? iy : iy - n) * dk;
        const float kz = (float)(iz <= nyq ? iz : iz - n) * dk;
        volatile float k2 = kx * kx;
        k2 = k2 + ky * ky;
        k2 = k2 + kz * kz;
        const c64 d = dkf[id];
        out[id] = c64(k2 * d.real(), k2 * d.imag());
      }
}

// Filter windows.  Filters.jl:18-36 and smooth_field :79-106.
// wsmooth 0: exp(-x^2/8); 1: 3(sin x - x cos x)/x^3; 3: exp(-x^2/8) k^2.
double ora_window(double kR, double k, int wsmooth) {
  if (wsmooth == 0) { const double h = kR / 2; return std::exp(-h * h / 2); }
  if (wsmooth == 3) { const double h = kR / 2; return std::exp(-h * h / 2) * (k * k); }
  if (kR == 0.0) return 1.0;
  return 3.0 * (std::sin(kR) - kR * std::cos(kR)) / (kR * kR * kR);
}

void ora_smooth_k(const c64* dkf, c64* out, int64_t n, double boxsize, double Rf, int wsmooth) {
  const double dk = 2.0 * PI / boxsize;
  const int64_t nh = n / 2 + 1;
#pragma omp parallel for schedule(static)
  for (int64_t iz = 0; iz < n; iz++)
    for (int64_t iy = 0; iy < n; iy++)
      for (int64_t ix = 0; ix < nh; ix++) {
        const int64_t id = ix + nh * (iy + n * iz);
        const double kx = dk * (double)ix, ky = dk * freq(iy, n, 1.0), kz = dk * freq(iz, n, 1.0);
        const double k = std::sqrt(kx * kx + ky * ky + kz * kz);
        const double fkR = k * Rf;
        const c64 d = dkf[id];
        if (fkR == 0.0) { out[id] = d; continue; }
        const float w = (float)ora_window(fkR, k, wsmooth);
        out[id] = c64(d.real() * w, d.imag() * w);
      }
}

// ---------------------------------------------------------------------------
// Peak finding.  PeakFind.jl:15-79.  Indices returned 1-based.
// Returns the number of peaks written (<= max_peaks).
// ---------------------------------------------------------------------------
int64_t ora_find_peaks(const float* delta, int8_t* mask, int64_t n1, int64_t n2, int64_t n3,
                       double xbx, double ybx, double zbx, double alatt, int64_t nbuff,
                       float fcrit, int64_t max_peaks,
                       int64_t* pi, int64_t* pj, int64_t* pk, int64_t* ipp,
                       double* px, double* py, double* pz, float* pdelta) {
  const double cen1 = 0.5 * (n1 + 1), cen2 = 0.5 * (n2 + 1), cen3 = 0.5 * (n3 + 1);
  int64_t np = 0;
  auto at = [&](int64_t i, int64_t j, int64_t k) { return delta[(i - 1) + n1 * ((j - 1) + n2 * (k - 1))]; };
  for (int64_t k = nbuff + 1; k <= n3 - nbuff; k++) {
    const double zc = zbx + alatt * (k - cen3);
    for (int64_t j = nbuff + 1; j <= n2 - nbuff; j++) {
      const double yc = ybx + alatt * (j - cen2);
      for (int64_t i = nbuff + 1; i <= n1 - nbuff; i++) {
        const double xc = xbx + alatt * (i - cen1);
        const int64_t lin = (i - 1) + n1 * ((j - 1) + n2 * (k - 1));
        if (mask[lin] == 1) continue;
        const float ff = delta[lin];
        if (ff < fcrit) continue;
        bool is_max = true;
        for (int kk = -1; kk <= 1 && is_max; kk++)
          for (int jj = -1; jj <= 1 && is_max; jj++)
            for (int ii = -1; ii <= 1; ii++)
              if (ff < at(i + ii, j + jj, k + kk)) { is_max = false; break; }
        if (!is_max) continue;
        pi[np] = i; pj[np] = j; pk[np] = k; ipp[np] = lin + 1;
        px[np] = xc; py[np] = yc; pz[np] = zc; pdelta[np] = ff;
        np++;
        mask[lin] = 1;
        if (np >= max_peaks) return np;
      }
    }
  }
  return np;
}

// ---------------------------------------------------------------------------
// RadialShell.jl
// ---------------------------------------------------------------------------
// hRinteg: RadialShell.jl:100-127
double ora_hRinteg(double u0, double u12) {
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

// atab4: RadialShell.jl:133-150 (1101 entries, 0-based here)
void ora_atab4(double* akk) {
  const double ca = 3.0 / (2.0 * PI), cb = 1.0 / (4.0 * PI);
  for (int i = 1; i <= 1100; i++) {
    const double u = (i - 1) * 0.01, ru = std::sqrt(u);
    double v;
    if (ru < 1.0) v = ca * (2.0 / 3.0 - u + 0.5 * u * ru);
    else if (ru <= 2.0) v = cb * (2.0 - ru) * (2.0 - ru) * (2.0 - ru);
    else v = 0.0;
    akk[i - 1] = v;
  }
  akk[1100] = 0.0;
}

// precompute_shells: RadialShell.jl:160-175.  Writes (di,dj,dk,r2) x count;
// returns the count.  Construction order dk, dj, di; stable sort by r2.
int64_t ora_shells(int rmax, int32_t* out) {
  struct C { int32_t di, dj, dk, r2; };
  std::vector<C> v;
  const int r2max = rmax * rmax;
  for (int dk = -rmax; dk <= rmax; dk++)
    for (int dj = -rmax; dj <= rmax; dj++)
      for (int di = -rmax; di <= rmax; di++) {
        const int r2 = di * di + dj * dj + dk * dk;
        if (r2 <= r2max) v.push_back({di, dj, dk, r2});
      }
  std::stable_sort(v.begin(), v.end(), [](const C& a, const C& b) { return a.r2 < b.r2; });
  if (out) for (size_t i = 0; i < v.size(); i++) { out[4 * i] = v[i].di; out[4 * i + 1] = v[i].dj; out[4 * i + 2] = v[i].dk; out[4 * i + 3] = v[i].r2; }
  return (int64_t)v.size();
}

// Symmetric 3x3 eigenvalues, ascending (stands in for LAPACK eigvals of
// Symmetric(mat), RadialShell.jl:217-222).  Cyclic Jacobi rotations until the
// off-diagonal part underflows relative to the diagonal.
void ora_eig3(const double* a, double* lam) {
  double A[3][3];
  for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) A[i][j] = a[i * 3 + j];
  // use the upper triangle (Symmetric with uplo = U)
  A[1][0] = A[0][1]; A[2][0] = A[0][2]; A[2][1] = A[1][2];
  for (int sweep = 0; sweep < 64; sweep++) {
    const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
    const double dia = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
    if (off == 0.0 || off < 1e-36 * dia) break;
    for (int p = 0; p < 2; p++)
      for (int q = p + 1; q < 3; q++) {
        if (A[p][q] == 0.0) continue;
        const double theta = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 3; k++) {  // A = J^T A J
          const double akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq; A[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; k++) {
          const double apk = A[p][k], aqk = A[q][k];
          A[p][k] = c * apk - s * aqk; A[q][k] = s * apk + c * aqk;
        }
      }
  }
  lam[0] = A[0][0]; lam[1] = A[1][1]; lam[2] = A[2][2];
  std::sort(lam, lam + 3);
}

// Collapse table (CollapseTable.jl:128-145): trilinear on the uniform grid
// range(X1, X2, length=Nx) etc., value outside the box = -1.  Data layout is
// column-major (x fastest).
struct OraTable { const float* t; int nx, ny, nz; double x1, x2, y1, y2, z1, z2; };

static double tab_interp(const OraTable& T, double x, double y, double z) {
  if (!(x >= T.x1 && x <= T.x2 && y >= T.y1 && y <= T.y2 && z >= T.z1 && z <= T.z2)) return -1.0;
  auto ax = [](double q, double q1, double q2, int nq, int* i, double* w) {
    const double st = (q2 - q1) / (nq - 1);
    const double pos = (q - q1) / st;   // 0-based position
    int ii = (int)std::floor(pos);
    if (ii < 0) ii = 0;
    if (ii > nq - 2) ii = nq - 2;
    *i = ii; *w = pos - ii;
  };
  int ix, iy, iz; double wx, wy, wz;
  ax(x, T.x1, T.x2, T.nx, &ix, &wx);
  ax(y, T.y1, T.y2, T.ny, &iy, &wy);
  ax(z, T.z1, T.z2, T.nz, &iz, &wz);
  auto A = [&](int a, int b, int c) { return (double)T.t[(ix + a) + T.nx * ((iy + b) + (int64_t)T.ny * (iz + c))]; };
  const double c00 = (1 - wx) * A(0, 0, 0) + wx * A(1, 0, 0);
  const double c10 = (1 - wx) * A(0, 1, 0) + wx * A(1, 1, 0);
  const double c01 = (1 - wx) * A(0, 0, 1) + wx * A(1, 0, 1);
  const double c11 = (1 - wx) * A(0, 1, 1) + wx * A(1, 1, 1);
  const double c0 = (1 - wy) * c00 + wy * c10;
  const double c1 = (1 - wy) * c01 + wy * c11;
  return (1 - wz) * c0 + wz * c1;
}

double ora_table_interp(const float* t, int nx, int ny, int nz, double x1, double x2, double y1,
                        double y2, double z1, double z2, double x, double y, double z) {
  OraTable T{t, nx, ny, nz, x1, x2, y1, y2, z1, z2};
  return tab_interp(T, x, y, z);
}

// ---------------------------------------------------------------------------
// Linear growth tables.  Cosmology.jl:203-417 (Dlinear_tables, RK4 over
// 2000 log-a steps) and :420-440 (Dlinear_ab), :105-119 (_hunt),
// :69-102 (Lagrange interpolation).
// ---------------------------------------------------------------------------
struct OraGrowth { std::vector<double> a, D, f; double amin, amax, Dinf, D0, Hinf, H0; };

static void deriv_Dlin(const double* y, double* d, double a, double h, double Omnr, double Omvac,
                       double Omcurv, double Omer, double OmX, double OmB, double Omhdm, double fhdmclus,
                       double Omnrd, double taud, int ldecay, double Omnrdi) {
  const double Omerd = ldecay == 1 ? Omnrdi * std::exp(-y[0] / taud) * a : 0.0;
  const double hub = Omer / a + Omnr + Omvac * (a * a * a) + Omcurv * a + Omerd / a + Omnrd;
  d[0] = 1.0 / (h * std::sqrt(hub / (a * a * a)));
  const double fb = y[2];
  d[1] = fb;
  const double q = Omer / a + Omnr + Omvac * (a * a * a) + Omcurv * a + Omerd / a + Omnrd;
  const double qs = 0.5 / q;
  const double qv = qs * (2.0 * Omer / a + Omnr - 2.0 * Omvac * (a * a * a) + 2.0 * Omerd / a + Omnrd);
  double fnr = (OmX + OmB + fhdmclus * Omhdm) / Omnr;
  if (OmB != 0.0 && a <= 1.0e-3) fnr = (OmX + fhdmclus * Omhdm) / Omnr;
  const double fer = 0.0;
  const double qf = qs * (2.0 * Omer / a * fer + Omnr * fnr + Omnrd * fnr);
  d[2] = 3.0 * qf - fb * fb - (1.0 - qv) * fb;
  d[3] = Omnrd * a * d[0] / taud;
  d[4] = d[0] / a;
}

static OraGrowth growth_tables(double Om, double OB, double OL, double h) {
  const double Omnr = Om, Omvac = OL, Omcurv = 1.0 - Om - OL, Omer = 0.0, OmX = Om - OB;
  const double Omhdm = 0.0, fhdmclus = 0.0, Omnrdi = 0.0, taud = 1.0, Omnrd = 0.0;
  const int ldecay = 0;
  const double amaxtab = 1.0 / 0.5, amintab_target = 1.0 / 1001.0, ainit = 1.0e-7;
  const int nmax = 2000;
  double a = ainit, alogn = std::log(ainit);
  const double amlog = std::log(amaxtab), hh = (amlog - alogn) / nmax;
  const double t0 = 1.0 / h / std::sqrt(Omnr);
  const double aeq = 0.0, yaeq = std::sqrt(a + aeq), yaeq0 = std::sqrt(aeq);
  double y[5];
  y[0] = t0 * (2.0 / 3.0 * (yaeq * yaeq * yaeq - yaeq0 * yaeq0 * yaeq0) - 2.0 * aeq * (yaeq - yaeq0));
  y[1] = std::log(a);
  const double fbclus = 0.0;
  y[2] = 0.25 * (std::sqrt(24.0 * (OmX + fbclus * OB + fhdmclus * Omhdm) / Omnr + 1.0) - 1.0);
  y[3] = 0.0;
  y[4] = t0 * 2.0 * (yaeq - yaeq0);
  std::vector<double> at, Dt, ft;
  int lnorm = 1, ip0 = 0;
  double bnorm = 1.0;
  const double anorm = 0.001;
  auto der = [&](const double* yy, double* dd, double aa) {
    deriv_Dlin(yy, dd, aa, h, Omnr, Omvac, Omcurv, Omer, OmX, OB, Omhdm, fhdmclus, Omnrd, taud, ldecay, Omnrdi);
  };
  for (int i = 0; i < nmax; i++) {
    double w1[5], w2[5], w3[5], w4[5], yt[5];
    der(y, w1, a);
    const double a_half = std::exp(alogn + hh * 0.5);
    for (int c = 0; c < 5; c++) yt[c] = y[c] + hh * w1[c] * 0.5;
    der(yt, w2, a_half);
    for (int c = 0; c < 5; c++) yt[c] = y[c] + hh * w2[c] * 0.5;
    der(yt, w3, a_half);
    const double alogn_new = alogn + hh, a_new = std::exp(alogn_new);
    for (int c = 0; c < 5; c++) yt[c] = y[c] + hh * w3[c];
    der(yt, w4, a_new);
    for (int c = 0; c < 5; c++) y[c] = y[c] + hh / 6.0 * (w1[c] + w4[c] + 2.0 * (w2[c] + w3[c]));
    alogn = alogn_new; a = a_new;
    if (lnorm == 1 && a >= anorm) { lnorm = 0; bnorm = std::exp(y[1]) / a; }
    if (a >= amintab_target && a <= amaxtab) {
      at.push_back(a); Dt.push_back(std::exp(y[1]) / a); ft.push_back(y[2]);
      if (a >= 1.0 && ip0 == 0) ip0 = (int)at.size();   // 1-based
    }
  }
  double fac;
  if (ip0 > 1) {
    const double ainterp = (at[ip0 - 1] - 1.0) / (at[ip0 - 1] - at[ip0 - 2]);
    const double Dag = (Dt[ip0 - 1] * (1.0 - ainterp) + Dt[ip0 - 2] * ainterp) / bnorm;
    fac = 1.0 / (Dag * bnorm);
  } else fac = 1.0 / bnorm;
  for (auto& v : Dt) v *= fac;
  OraGrowth G;
  G.a = at; G.D = Dt; G.f = ft;
  G.amin = at.front(); G.amax = at.back(); G.Dinf = Dt.front(); G.D0 = Dt.back(); G.Hinf = ft.front(); G.H0 = ft.back();
  return G;
}

static int hunt(const std::vector<double>& xx, double x) {
  const int n = (int)xx.size();
  const bool asc = xx[n - 1] > xx[0];
  int jlo = 0, jhi = n + 1;
  while (jhi - jlo > 1) {
    const int jm = (jhi + jlo) / 2;
    if ((x > xx[jm - 1]) == asc) jlo = jm; else jhi = jm;
  }
  return jlo;
}

// returns (D(a) = D_a*a, HD_Ha, D_a)
static void dlinear_ab(const OraGrowth& G, double ai, double* Dl, double* HD, double* Da) {
  const int ntab = (int)G.a.size();
  if (ai > G.amin && ai < G.amax) {
    const int kk = hunt(G.a, ai);
    int nl, kkl;
    if (kk < 2 || kk >= ntab) { nl = 2; kkl = std::max(kk - 1, 1); } else { nl = 4; kkl = kk - 2; }
    const double* xa = &G.a[kkl - 1];
    const double* v1 = &G.D[kkl - 1];
    const double* v2 = &G.f[kkl - 1];
    double p1, p2;
    const double x = ai;
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
    *Dl = p1 * ai; *HD = p2; *Da = p1;
  } else if (ai >= G.amax) {
    *Dl = G.D0 * ai; *HD = G.H0; *Da = G.D0;
  } else {
    *Dl = G.Dinf * ai; *HD = G.Hinf; *Da = G.Dinf;
  }
}

// ---------------------------------------------------------------------------
// Collapse-table generation, RK4 path: make_table (CollapseTable.jl:33-52)
// calling evolve_ellipse_full with solver = :rk4 (EllipsoidalCollapse.jl
// :518-624): get_derivs! (:212-323), rk4_homel! (:153-179), get_b_2
// (:113-149), Carlson's RD (:66-108), Ha_b_nr (:56-58).  The logarithm of the
// oblate branch is the project's log (ppbm::log_pos), as on the device.
// ---------------------------------------------------------------------------
struct OraEll {
  int iforce, ivir, nstepmax;
  double fcoll1, fcoll2, fcoll3, tfac, zinit_fac;
  double Rvac, Rcurv;
  const OraGrowth* G;
};

static double ell_rd(double x, double y, double z) {
  const double ERRTOL = 0.05, C1 = 3.0 / 14.0, C2 = 1.0 / 6.0, C3 = 9.0 / 22.0, C4 = 3.0 / 26.0;
  const double C5 = 0.25 * C3, C6 = 1.5 * C4;
  double xt = x, yt = y, zt = z, sum = 0.0, fac = 1.0, delx = 0.0, dely = 0.0, delz = 0.0, ave = 0.0;
  for (int it = 0; it < 200; it++) {
    const double sx = std::sqrt(xt), sy = std::sqrt(yt), sz = std::sqrt(zt);
    const double alamb = sx * (sy + sz) + sy * sz;
    sum += fac / (sz * (zt + alamb));
    fac *= 0.25;
    xt = 0.25 * (xt + alamb);
    yt = 0.25 * (yt + alamb);
    zt = 0.25 * (zt + alamb);
    ave = 0.2 * (xt + yt + 3.0 * zt);
    delx = (ave - xt) / ave;
    dely = (ave - yt) / ave;
    delz = (ave - zt) / ave;
    if (std::max(std::max(std::fabs(delx), std::fabs(dely)), std::fabs(delz)) <= ERRTOL) break;
  }
  const double ea = delx * dely, eb = delz * delz, ec = ea - eb, ed = ea - 6.0 * eb, ee = ed + ec + ec;
  return 3.0 * sum + fac * (1.0 + ed * (-C1 + C5 * ed - C6 * delz * ee) +
                            delz * (C2 * ee + delz * (-C3 * ec + delz * C4 * ea))) / (ave * std::sqrt(ave));
}

static void ell_b2(double a1, double a2, double a3, double* b) {
  const double third = 1.0 / 3.0;
  const double r2 = a2 / a1, r3 = a3 / a1;
  if (r3 >= r2) {
    if (r3 >= 0.999) { b[0] = b[1] = b[2] = third; return; }
    double b3;
    if (r3 <= 0.001) {
      const double ecc2 = 1.0 - r3 * r3, one_ecc2 = r3 * r3, one_ecc = 0.5 * (r3 * r3), ecc = std::sqrt(ecc2);
      b3 = 0.5 * (one_ecc2 / ecc2 * (1.0 / one_ecc2 - ppbm::log_pos((1.0 + ecc) / one_ecc) * 0.5 / ecc));
    } else {
      const double ecc2 = 1.0 - r3 * r3, ecc = std::sqrt(ecc2);
      b3 = 0.5 * ((1.0 - ecc2) / ecc2 * (1.0 / (1.0 - ecc2) - ppbm::log_pos((1.0 + ecc) / (1.0 - ecc)) * 0.5 / ecc));
    }
    b[0] = 1.0 - 2.0 * b3; b[1] = b3; b[2] = b3;
    return;
  }
  const double r22 = r2 * r2, r32 = r3 * r3, qrat = third * r2 * r3;
  const double b3 = qrat * ell_rd(r22, 1.0, r32), b2 = qrat * ell_rd(r32, 1.0, r22);
  b[0] = 1.0 - (b2 + b3); b[1] = b2; b[2] = b3;
}

struct OraDeriv {
  int lvir[3];
  double aeq[3];           // frozen axis values (a_1eq, a_2eq, a_3eq)
  double a3eq2, a3eq1, Ha;
  double lam[3], F3;
};

static double ell_Ha(const OraEll& E, double a) {
  return std::sqrt((1.0 + E.Rvac * (a * a * a) + E.Rcurv * a) / a);
}

// y = (a1, a2, a3, v1, v2, v3) 0-based; may freeze axes of y
static void ell_derivs(const OraEll& E, OraDeriv& S, double t, double* y, double* dy) {
  for (int i = 0; i < 6; i++) dy[i] = 0.0;
  const double ab = t, ab3 = ab * ab * ab;
  const double Ha = ell_Ha(E, ab);
  S.Ha = Ha;
  const double Hi = 1.0 / Ha;
  if (S.lvir[2] == 0 && y[2] <= E.fcoll3 * ab) {
    S.lvir[2] = 1;
    S.aeq[2] = E.fcoll3 * ab;
    if (E.ivir == 1) { S.a3eq2 = S.aeq[2] * 1.001; S.a3eq1 = S.aeq[2] * 1.0003; }
  }
  if (E.ivir == 2 && S.lvir[1] == 0) S.a3eq2 = E.fcoll2 * ab;
  if (E.ivir == 2 && S.lvir[0] == 0) S.a3eq1 = E.fcoll1 * ab;
  if (S.lvir[2] == 1 && y[1] <= S.a3eq2 && S.lvir[1] == 0) { S.lvir[1] = 1; S.aeq[1] = S.a3eq2; }
  if (S.lvir[2] == 1 && y[0] <= S.a3eq1 && S.lvir[0] == 0) { S.lvir[0] = 1; S.aeq[0] = S.a3eq1; }
  for (int ax = 2; ax >= 0; ax--)
    if (S.lvir[ax] == 1) { y[ax] = S.aeq[ax]; y[ax + 3] = 0.0; dy[ax] = 0.0; dy[ax + 3] = 0.0; }
  const double a1 = y[0], a2 = y[1], a3 = y[2];
  const double d1e = ab3 / (a1 * a2 * a3);
  double d0, d1i, d1x = 0.0;
  if (E.iforce == 0) {
    d0 = -E.Rvac * Hi;
    d1i = 1.5 * d1e / ab3 * Hi;
  } else {
    d0 = (0.5 / ab3 - E.Rvac) * Hi;
    d1i = 1.5 * (d1e - 1.0) / ab3 * Hi;
    if (E.iforce == 4 || E.iforce == 5 || E.iforce == 6) {
      double dl, hd, da;
      dlinear_ab(*E.G, ab, &dl, &hd, &da);
      d1x = 1.5 / ab3 * Hi * dl;
    } else if (E.iforce == 3) {
      d1x = 1.5 * 2.5 / ab3 * Hi;
    }
  }
  double b[3] = {0.0, 0.0, 0.0};
  if (E.iforce != 5 && E.iforce != 6) ell_b2(a1, a2, a3, b);
  const double third = 1.0 / 3.0;
  for (int ax = 2; ax >= 0; ax--) {   // axis 3, 2, 1 as the reference
    if (S.lvir[ax] != 0) continue;
    dy[ax] = y[ax + 3] * Hi;
    const double ya = y[ax];
    switch (E.iforce) {
      case 0: dy[ax + 3] = -ya * d1i * b[ax]; break;
      case 1: dy[ax + 3] = -ya * (d1i * b[ax] + d0); break;
      case 3: dy[ax + 3] = -ya * (d1i * b[ax] + d0 + d1x * (b[ax] - third)); break;
      case 5: dy[ax + 3] = -ya * d0 - d1x * ab * S.lam[ax]; break;
      default: dy[ax + 3] = -ya * (d1i * b[ax] + d0 + d1x * (S.lam[ax] - S.F3)); break;   // 4, 6
    }
  }
}

static double ell_evolve(const OraEll& E, double Frho, double ev, double pv) {
  OraDeriv S{};
  S.lam[2] = Frho / 3.0 * (1.0 + 3.0 * ev + pv);
  S.lam[1] = Frho / 3.0 * (1.0 - 2.0 * pv);
  S.lam[0] = Frho / 3.0 * (1.0 - 3.0 * ev + pv);
  S.F3 = Frho / 3.0;
  const double zinit = E.zinit_fac * Frho;
  const double ab = 1.0 / zinit;
  double t = ab;
  double dl, hd, da;
  dlinear_ab(*E.G, ab, &dl, &hd, &da);
  const double Ha = ell_Ha(E, ab);
  S.Ha = Ha;
  double y[6];
  for (int ax = 2; ax >= 0; ax--) {
    y[ax] = ab * (1.0 - dl * S.lam[ax]);
  }
  for (int ax = 2; ax >= 0; ax--) {
    y[ax + 3] = Ha * (1.0 - (1.0 + hd) * dl * S.lam[ax]);
  }
  double zdyn[6] = {-1.0, -1.0, -1.0, -1.0, -1.0, -1.0};
  int ldyn[6] = {0, 0, 0, 0, 0, 0};
  double aturn[3] = {0.0, 0.0, 0.0};
  double dy[6], yout[6], yt[6], dyt[6], dym[6];
  int istep = 0;
  while (true) {
    istep++;
    const double a_3 = y[2];
    const double h = E.tfac * a_3 * std::sqrt(a_3) * S.Ha;
    ell_derivs(E, S, t, y, dy);
    // rk4_homel!
    const double hh = h * 0.5, h6 = h / 6.0, xh = t + hh;
    for (int i = 0; i < 6; i++) yt[i] = y[i] + hh * dy[i];
    ell_derivs(E, S, xh, yt, dyt);
    for (int i = 0; i < 6; i++) yt[i] = y[i] + hh * dyt[i];
    ell_derivs(E, S, xh, yt, dym);
    for (int i = 0; i < 6; i++) { yt[i] = y[i] + h * dym[i]; dym[i] = dyt[i] + dym[i]; }
    ell_derivs(E, S, t + h, yt, dyt);
    for (int i = 0; i < 6; i++) yout[i] = y[i] + h6 * (dy[i] + dyt[i] + 2.0 * dym[i]);
    for (int i = 0; i < 6; i++) y[i] = yout[i];
    t += h;
    for (int ii = 0; ii < 3; ii++)
      if (S.lvir[ii] != ldyn[ii]) { zdyn[ii] = 1.0 / t; ldyn[ii] = 1; }
    for (int ii = 3; ii < 6; ii++) {
      if (ldyn[ii] != 1) {
        const int iax = ii - 3;
        if (y[iax] < aturn[iax]) { zdyn[ii] = 1.0 / t; ldyn[ii] = 1; }
        else aturn[iax] = y[iax];
      }
    }
    if (S.lvir[0] == 1 || istep >= E.nstepmax || t >= 2.0) return zdyn[0];   // idynax = 1
  }
}

// make_table with the RK4 solver: out[i + Nx (j + Ny k)] = 1 + z_vir of
// axis 1 (-1: no collapse by a = 2), x = X1 + i dX = log10 F, y = e_v,
// z = p_v / e_v.  prm = (X1, X2, Y1, Y2, Z1, Z2, fcoll1, fcoll2, fcoll3, tfac,
// zinit_fac); iprm = (Nx, Ny, Nz, iforce_strat, ivir_strat, nstepmax).
void ora_make_table(double Om, double OB, double OL, double h, const int32_t* iprm, const double* prm,
                    double* out) {
  OraGrowth G = growth_tables(Om, OB, OL, h);
  OraEll E{iprm[3], iprm[4], iprm[5], prm[6], prm[7], prm[8], prm[9], prm[10], OL / Om, (1.0 - Om - OL) / Om, &G};
  const int Nx = iprm[0], Ny = iprm[1], Nz = iprm[2];
  const double dX = (prm[1] - prm[0]) / (Nx - 1), dY = (prm[3] - prm[2]) / (Ny - 1), dZ = (prm[5] - prm[4]) / (Nz - 1);
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
  for (int k = 0; k < Nz; k++)
    for (int j = 0; j < Ny; j++)
      for (int i = 0; i < Nx; i++) {
        const double z = prm[4] + k * dZ, y = prm[2] + j * dY, x = prm[0] + i * dX;
        const double Frho = std::pow(10.0, x);
        out[i + (int64_t)Nx * (j + (int64_t)Ny * k)] = ell_evolve(E, Frho, y, z * y);
      }
}

double ora_elliptic_rd(double x, double y, double z) { return ell_rd(x, y, z); }
void ora_shape_b2(double a1, double a2, double a3, double* b) { ell_b2(a1, a2, a3, b); }

// Exposed for tests: returns D(a) for each a.
void ora_dlinear(double Om, double OB, double OL, double h, const double* a, int na, double* D) {
  OraGrowth G = growth_tables(Om, OB, OL, h);
  for (int i = 0; i < na; i++) { double d, hd, da; dlinear_ab(G, a[i], &d, &hd, &da); D[i] = d; }
}

// fsc_of_z: RadialShell.jl:191-196
static double fsc_of_z(const OraGrowth& G, double z) {
  double d, hd, da;
  dlinear_ab(G, 1.0 / (1.0 + z), &d, &hd, &da);
  return 1.686 * d;
}
double ora_fsc_of_z(double Om, double OB, double OL, double h, double z) {
  OraGrowth G = growth_tables(Om, OB, OL, h);
  return fsc_of_z(G, z);
}

// Comoving distance chi(z) in Mpc/h: Cosmology.jl:21-24 (QuadGK there;
// adaptive Gauss-Kronrod 7/15 here, tolerance 1e-13 relative).
static double gk15(double Om, double OL, double a, double b, double* err) {
  static const double xk[8] = {0.991455371120812639206854697526329, 0.949107912342758524526189684047851,
                               0.864864423359769072789712788640926, 0.741531185599394439863864773280788,
                               0.586087235467691130294144845693013, 0.405845151377397166906606412076961,
                               0.207784955007898467600689403773245, 0.000000000000000000000000000000000};
  static const double wk[8] = {0.022935322010529224963732008058970, 0.063092092629978553290700663189204,
                               0.104790010322250183839876322541518, 0.140653259715525918745189590510238,
                               0.169004726639267902826583426598550, 0.190350578064785409913256402421014,
                               0.204432940075298892414161999234649, 0.209482141084727828012999174891714};
  static const double wg[4] = {0.129484966168869693270611432679082, 0.279705391489276667901467771423780,
                               0.381830050505118944950369775488975, 0.417959183673469387755102040816327};
  auto f = [&](double z) { return 1.0 / std::sqrt(Om * (1 + z) * (1 + z) * (1 + z) + OL); };
  const double c = 0.5 * (a + b), hl = 0.5 * (b - a);
  double fc = f(c), rk = fc * wk[7], rg = fc * wg[3];
  for (int j = 0; j < 7; j++) {
    const double dx = hl * xk[j];
    const double f1 = f(c - dx), f2 = f(c + dx);
    rk += wk[j] * (f1 + f2);
    if (j % 2 == 1) rg += wg[j / 2] * (f1 + f2);
  }
  *err = std::fabs((rk - rg) * hl);
  return rk * hl;
}
static double chi_of_z(double Om, double OL, double h, double z) {
  if (z == 0.0) return 0.0;
  std::vector<std::pair<double, double>> st{{0.0, z}};
  double tot = 0.0;
  while (!st.empty()) {
    auto [a, b] = st.back(); st.pop_back();
    double e; const double v = gk15(Om, OL, a, b, &e);
    if (e <= 1e-14 * std::fabs(v) || (b - a) < 1e-9) tot += v;
    else { const double m = 0.5 * (a + b); st.push_back({a, m}); st.push_back({m, b}); }
  }
  return (2.998e5 / 100.0) * h * tot;
}
double ora_chi(double Om, double OL, double h, double z) { return chi_of_z(Om, OL, h, z); }

// chi -> z table and lookup: Cosmology.jl:144-183
struct OraChi { std::vector<double> zs, chis; double zmax; };
static OraChi build_chi2z(double Om, double OL, double h, double zmax, int npts) {
  OraChi T; T.zmax = zmax;
  for (int i = 0; i < npts; i++) {
    const double z = npts == 1 ? 0.0 : zmax * (double)i / (double)(npts - 1);
    T.zs.push_back(z); T.chis.push_back(chi_of_z(Om, OL, h, z));
  }
  return T;
}
static double chi_to_z(const OraChi& T, double c) {
  if (c <= T.chis.front()) return 0.0;
  if (c >= T.chis.back()) return T.zmax;
  int lo = 1, hi = (int)T.zs.size();
  while (hi - lo > 1) { const int mid = (lo + hi) >> 1; if (T.chis[mid - 1] <= c) lo = mid; else hi = mid; }
  const double fr = (c - T.chis[lo - 1]) / (T.chis[hi - 1] - T.chis[lo - 1]);
  return T.zs[lo - 1] + fr * (T.zs[hi - 1] - T.zs[lo - 1]);
}
void ora_chi2z(double Om, double OL, double h, double zmax, const double* chis, int n, double* z) {
  OraChi T = build_chi2z(Om, OL, h, zmax, 2000);
  for (int i = 0; i < n; i++) z[i] = chi_to_z(T, chis[i]);
}

// ---------------------------------------------------------------------------
// analyse_peak: RadialShell.jl:282-891.  Output layout (31 doubles):
// 0 RTHL, 1 Srb, 2-4 Sbar, 5-7 Sbar2, 8-16 strain (column-major 3x3),
// 17-19 gradpk, 20-22 gradpkrf, 23 Fbarx, 24 e_v, 25 p_v, 26 zvir_half,
// 27-29 gradpkf, 30 d2F.
// ---------------------------------------------------------------------------
enum { R_RTHL = 0, R_SRB = 1, R_SBAR = 2, R_SBAR2 = 5, R_STRAIN = 8, R_GRADPK = 17, R_GRADRF = 20,
       R_FBARX = 23, R_EV = 24, R_PV = 25, R_ZVH = 26, R_GRADF = 27, R_D2F = 30, R_N = 31 };

struct Mat3 { double m[3][3]; };
struct Vec3 { double v[3]; };

struct PeakCtx {
  const float *delta, *ex, *ey, *ez, *e2x, *e2y, *e2z, *lapd;
  int8_t* mask;
  int64_t n1, n2, n3;
  const int32_t* shells; int64_t nshells;
  const double* akk;
  OraTable T;
  int64_t ndistinct;   // distinct r^2 values of the list: profile arrays need ndistinct + 3 entries
  // truncated gather (CPU timing leg only, not the reference's algorithm):
  // stop reading cells once every shell the later phases read is in
  int truncate;
  const double* srad;  // srad[m], m = 1..ndistinct: shell radii (shell 1 = the centre)
  const int* need;     // need[m]: shells to gather when shell m is the outermost one read
};

static void no_collapse(double* r) {
  for (int i = 0; i < R_N; i++) r[i] = 0.0;
  r[R_RTHL] = -1.0; r[R_ZVH] = -1.0;
}

std::atomic<long> g_dump[5];   // premask, no_fcrit, m0_one, no_collapse, rthl_neg

static void kernel_strain(const std::vector<double>& rad, const std::vector<double>* G,
                          const std::vector<double>* Gf, const std::vector<double> (*SR)[3],
                          int mp, int mlow, int mupp, const double* akk, double wRnor, double aRnor,
                          double h1, double h2, Mat3* Eb, Vec3* gr, Vec3* grf) {
  Mat3 E{}; Vec3 g{}, gf{};
  if (mp > 1) {
    for (int m1 = mlow; m1 <= mupp; m1++) {
      const double u0 = h1 * (rad[mp] - rad[m1]);
      const double u02 = u0 * u0;
      if (u02 < 4.0) {
        const double u12 = h2 * (rad[mp] * rad[mp] + rad[m1] * rad[m1]);
        const double d = u12 - u02;
        const double wt = ora_hRinteg(u0, u12) / (d * d);
        for (int L = 0; L < 3; L++) {
          g.v[L] += wt * G[L][m1];
          gf.v[L] += wt * Gf[L][m1];
          for (int K = 0; K < 3; K++) E.m[L][K] -= 0.5 * wt * (SR[L][K][m1] + SR[K][L][m1]);
        }
      }
    }
    const double sc = wRnor / rad[mp];
    for (int L = 0; L < 3; L++) { g.v[L] *= sc; gf.v[L] *= sc; for (int K = 0; K < 3; K++) E.m[L][K] *= sc; }
  } else {
    for (int m1 = mlow; m1 <= mupp; m1++) {
      const double u0 = h1 * rad[m1];
      const double con = 100.0 * u0 * u0;
      const int64_t icon = (int64_t)std::floor(con);
      const double diff = con - icon;
      if (icon + 1 > 1100) abort();   // the reference raises a BoundsError here
      const double aww = akk[icon] + diff * (akk[icon + 1] - akk[icon]);
      const double wt = 0.5 * aww / rad[m1];
      for (int L = 0; L < 3; L++) {
        g.v[L] += wt * G[L][m1];
        gf.v[L] += wt * Gf[L][m1];
        for (int K = 0; K < 3; K++) E.m[L][K] -= 0.5 * wt * (SR[L][K][m1] + SR[K][L][m1]);
      }
    }
    for (int L = 0; L < 3; L++) { g.v[L] *= aRnor; gf.v[L] *= aRnor; for (int K = 0; K < 3; K++) E.m[L][K] *= aRnor; }
  }
  *Eb = E; *gr = g; *grf = gf;
}

static void evals(const Mat3& M, double* lam) {
  double a[9];
  for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) a[i * 3 + j] = M.m[i][j];
  ora_eig3(a, lam);
}

static void analyse_peak(const PeakCtx& P, int64_t ipp, double alatt, int64_t ir2min, double ZZon,
                         double Rfclvi, int64_t nbuff, double rmax2rs, double fcrit, double* out) {
  const int64_t npartmax = P.nshells;
  int64_t npart = npartmax;
  if (rmax2rs > 0.0) {
    const double f3p = 4.0 / 3.0 * PI;
    const double rr = rmax2rs * Rfclvi / alatt;
    npart = std::min((int64_t)std::floor(f3p * (rr * rr * rr)), npartmax);
  }
  const double hlatt = 1.0, anor = 1.0 / (hlatt * hlatt * hlatt);
  const double aRnor = 3.0 * anor / alatt, wnor = anor / (4.0 * PI), wRnor = 3.0 * wnor / alatt;
  const int64_t n1 = P.n1, n2 = P.n2, n3 = P.n3, n12 = n1 * n2;
  const int64_t pk = (ipp - 1) / n12 + 1, pj = ((ipp - 1) % n12) / n1 + 1, pi = (ipp - 1) % n1 + 1;
  auto lin = [&](int64_t i, int64_t j, int64_t k) { return (i - 1) + n1 * ((j - 1) + n2 * (k - 1)); };
  const int32_t* sh = P.shells;   // 0-based rows (di,dj,dk,r2); jp (1-based) -> sh[4*(jp-1)]

  if (rmax2rs > 0.0 && P.mask) {
    if (P.mask[lin(pi, pj, pk)] > (int64_t)std::floor(Rfclvi / alatt * rmax2rs)) {
      g_dump[0]++; no_collapse(out); return;
    }
  }
  // profile index m counts distinct r^2 (the reference sizes them npart + 2)
  const int64_t maxm = std::min<int64_t>(npart, P.ndistinct) + 3;
  std::vector<double> rad(maxm, 0.0), Fbar(maxm, 0.0);
  std::vector<int64_t> nshell(maxm, 0);
  std::vector<double> S[3], S2[3], G[3], Gf[3], SR[3][3];
  for (int L = 0; L < 3; L++) {
    S[L].assign(maxm, 0.0); S2[L].assign(maxm, 0.0); G[L].assign(maxm, 0.0); Gf[L].assign(maxm, 0.0);
    for (int K = 0; K < 3; K++) SR[L][K].assign(maxm, 0.0);
  }
  int64_t m = 1, m0 = 1;
  rad[1] = 0.0;
  Fbar[1] = P.delta[lin(pi, pj, pk)];
  nshell[1] = 1;
  const bool ilpt2 = P.e2x != nullptr;
  const int64_t lp = lin(pi, pj, pk);
  const double eta0[3] = {P.ex[lp], P.ey[lp], P.ez[lp]};
  const double eta20[3] = {ilpt2 ? P.e2x[lp] : 0.0, ilpt2 ? P.e2y[lp] : 0.0, ilpt2 ? P.e2z[lp] : 0.0};
  for (int L = 0; L < 3; L++) { S[L][1] = eta0[L]; S2[L][1] = eta20[L]; }
  double Fshell = 0.0;
  int64_t nsh = 0;
  int64_t ir2p = npart >= 2 ? sh[4 * 1 + 3] : 0;
  double dFbarp = Fbar[1];
  double rupp_init = std::sqrt((double)ir2min) + 2.0 * hlatt;
  int ifcrit = 1;
  int64_t mupp = 1;
  // truncated gather: the shells any later phase reads end at need[M], M the
  // outermost of the first shell beyond ir2min, the Rf window and (outward)
  // the fcrit crossing; an inward crossing is seen at that first shell
  int64_t mlast = 0, tM = 0, tstate = 0, mtarget = -1;
  if (P.truncate) {
    for (int64_t jp = 2; jp <= npart; jp++)
      if (sh[4 * (jp - 1) + 3] != sh[4 * (jp - 2) + 3]) mlast++;
    mlast = std::max<int64_t>(mlast, 1);   // shells finalised inside the loop (the centre is shell 1)
    // Rf window of phase 3 (depends on the radii only)
    double rm = 10.0;
    int64_t mr = 1, mri = 1, i2p = npart >= 2 ? sh[7] : 0;
    const double rq0 = (Rfclvi / alatt) * (Rfclvi / alatt);
    for (int64_t jp = 2; jp <= npart; jp++) {
      const int64_t i2 = sh[4 * (jp - 1) + 3];
      if (std::fabs((double)i2 - rq0) < rm) { mr = mri; rm = std::min(rm, std::fabs((double)i2 - rq0)); }
      if (i2 != i2p) { mri++; i2p = i2; }
    }
    int64_t mur = mr;
    for (int64_t m1 = mr + 1; m1 <= mlast; m1++) if (P.srad[m1] < P.srad[mr] + 2.0) mur = m1;
    tM = std::max(mr, mur);
  }
  for (int64_t jp = 2; jp <= npart; jp++) {
    const int32_t* c = sh + 4 * (jp - 1);
    const int64_t ir2 = c[3];
    if (P.truncate && mtarget >= 0 && m >= mtarget) break;
    if (ir2 != ir2p) {
      m += 1;
      rad[m] = std::sqrt((double)ir2p);
      nshell[m] = nsh;
      const double dFbar = nsh > 0 ? Fshell / nsh : 0.0;
      const double r3p = rad[m - 1] * rad[m - 1] * rad[m - 1];
      const double r3 = rad[m] * rad[m] * rad[m];
      Fbar[m] = (r3p * Fbar[m - 1] + 0.5 * (dFbarp + dFbar) * (r3 - r3p)) / r3;
      dFbarp = dFbar;
      if (ifcrit == 1) {
        m0 = m;
        if (ir2p > ir2min) { rupp_init = rad[m0] + 2.0 * hlatt; ifcrit = 0; mupp = m; }
      } else {
        if (rad[m] < rupp_init) mupp = m;
      }
      if (P.truncate && mtarget < 0) {
        // the crossing state in shell order, as the GPU gather decides it
        if (tstate == 0 && ifcrit == 0 && m == m0) tstate = Fbar[m] < fcrit ? 1 : 0;
        else if (tstate == 0 && ifcrit == 0 && m > m0 && Fbar[m] < fcrit) { tstate = 2; tM = std::max(tM, m); }
        if (tstate != 0) mtarget = std::min<int64_t>(P.need[std::max(tM, m0)], mlast);
      }
      ir2p = ir2;
      Fshell = 0.0; nsh = 0;
      for (int L = 0; L < 3; L++) {
        S[L][m + 1] = 0.0; S2[L][m + 1] = 0.0;
        G[L][m] /= rad[m]; Gf[L][m] /= rad[m];
        G[L][m + 1] = 0.0; Gf[L][m + 1] = 0.0;
        for (int K = 0; K < 3; K++) { SR[L][K][m] /= rad[m]; SR[L][K][m + 1] = 0.0; }
      }
    }
    const int64_t iv1 = pi + c[0], iv2 = pj + c[1], iv3 = pk + c[2];
    if (iv1 < 1 || iv1 > n1 || iv2 < 1 || iv2 > n2 || iv3 < 1 || iv3 > n3) continue;
    nsh += 1;
    const int64_t li = lin(iv1, iv2, iv3);
    const float dv = P.delta[li];
    Fshell += dv;
    const float et[3] = {P.ex[li], P.ey[li], P.ez[li]};
    const float e2[3] = {ilpt2 ? P.e2x[li] : 0.f, ilpt2 ? P.e2y[li] : 0.f, ilpt2 ? P.e2z[li] : 0.f};
    const float dT = P.delta[lin(iv3, iv1, iv2)];
    const float ds[3] = {(float)c[0], (float)c[1], (float)c[2]};
    for (int L = 0; L < 3; L++) {
      S[L][m + 1] += et[L];
      S2[L][m + 1] += e2[L];
      volatile float pg = dv * ds[L];        // Float32 * Int32 -> Float32 product
      G[L][m + 1] += pg;
      volatile float pgf = dT * ds[L];
      Gf[L][m + 1] += pgf;
      for (int K = 0; K < 3; K++) { volatile float ps = et[L] * ds[K]; SR[L][K][m + 1] += ps; }
    }
  }

  if (P.truncate && m < mlast) {
    // shells beyond the gathered ones are never read below; their radii are
    // the list's (the loops over rad[] run to the last shell as in the full sum)
    for (int64_t mm = m + 1; mm <= mlast; mm++) rad[mm] = P.srad[mm];
    m = mlast;
  }
  // Phase 3: gradient at Rf
  double rmrf = 10.0;
  int64_t mrf = 1, mrfi = 1;
  int64_t ir2p_rf = npart >= 2 ? sh[4 * 1 + 3] : 0;
  const double rq = (Rfclvi / alatt) * (Rfclvi / alatt);
  for (int64_t jp = 2; jp <= npart; jp++) {
    const int64_t ir2 = sh[4 * (jp - 1) + 3];
    if (std::fabs((double)ir2 - rq) < rmrf) { mrf = mrfi; rmrf = std::min(rmrf, std::fabs((double)ir2 - rq)); }
    if (ir2 != ir2p_rf) { mrfi += 1; ir2p_rf = ir2; }
  }
  const double rlow_rf = std::max(rad[mrf] - 2.0, 0.0);
  int64_t mlow_rf = mrf;
  if (mrf > 1) for (int64_t m1 = mrf - 1; m1 >= 1; m1--) if (rad[m1] > rlow_rf) mlow_rf = m1;
  const double rupp_rf = rad[mrf] + 2.0;
  int64_t mupp_rf = mrf;
  for (int64_t m1 = mrf + 1; m1 <= m; m1++) if (rad[m1] < rupp_rf) mupp_rf = m1;
  Mat3 Etmp; Vec3 gradpkrf, gtmp;
  kernel_strain(rad, G, Gf, SR, (int)mrf, (int)mlow_rf, (int)mupp_rf, P.akk, wRnor, aRnor, 1.0, 1.0, &Etmp, &gradpkrf, &gtmp);

  // Phase 4: fcrit crossing
  if (Fbar[m0] >= fcrit) {
    bool found = false;
    for (int64_t mm = m0; mm <= m; mm++) if (Fbar[mm] < fcrit) { m0 = mm; found = true; break; }
    if (!found) mupp = m;
    if (found) {
      const double rupp_m0 = rad[m0] + 2.0;
      mupp = m0;
      for (int64_t mm = m0 + 1; mm <= m; mm++) if (rad[mm] < rupp_m0) mupp = mm;
    }
  } else {
    const int64_t mstart = std::max<int64_t>(m0 - 1, 1);
    bool found = false;
    for (int64_t mp = mstart; mp >= 1; mp--) {
      if (Fbar[mp] >= fcrit) { found = true; break; }
      m0 = mp;
    }
    if (!found) { g_dump[1]++; no_collapse(out); return; }
    const double rupp_m0 = rad[m0] + 2.0;
    int64_t mupp_new = m0;
    for (int64_t mm = m0 + 1; mm <= m; mm++) if (rad[mm] < rupp_m0) mupp_new = mm;
    mupp = mupp_new;
  }

  // Phase 5: inward walk
  const double rlow = std::max(rad[m0] - 2.0, 0.0);
  int64_t mlow = m0;
  if (m0 > 1) for (int64_t m1 = m0 - 1; m1 >= 1; m1--) if (rad[m1] > rlow) mlow = m1;
  double zvir1 = -1.0, zvir1p = -1.0;
  Mat3 Ebar_last{}, strain_mat{};
  Vec3 gradpk_last{}, gradpk_prev{}, gradpkf_last{}, gradpkf_prev{};
  double Frhoh = 0.0, Frho = 0.0, e_v = 0.0, p_v = 0.0;
  double Frhpk = 0.0, Fnupk = 0.0, Fevpk = 0.0, Fpvpk = 0.0;
  bool collapsed = false;
  Mat3 Ebar_m0; Vec3 gradpk_m0, gradpkf_m0;
  kernel_strain(rad, G, Gf, SR, (int)m0, (int)mlow, (int)mupp, P.akk, wRnor, aRnor, 1.0, 1.0, &Ebar_m0, &gradpk_m0, &gradpkf_m0);
  double lam[3];
  evals(Ebar_m0, lam);
  double Frho_m0 = lam[0] + lam[1] + lam[2];
  double e_v_m0 = 0.0, p_v_m0 = 0.0;
  if (Frho_m0 > 0.0) {
    e_v_m0 = 0.5 * (lam[2] - lam[0]) / Frho_m0;
    p_v_m0 = 0.5 * (lam[2] + lam[0] - 2.0 * lam[1]) / Frho_m0;
  }
  const double Frhoh_m0 = Frho_m0;
  Frho_m0 = Fbar[m0];
  const double zvir1p_m0 = -1.0;   // Fortran uninitialised-variable replication (:581-583)
  if (zvir1p_m0 >= ZZon) {
    zvir1 = -1.0; zvir1p = zvir1p_m0;
    Ebar_last = Ebar_m0; gradpk_last = gradpk_m0; gradpkf_last = gradpkf_m0;
    strain_mat = Ebar_m0; gradpk_prev = gradpk_m0; gradpkf_prev = gradpkf_m0;
    Frhoh = Frhoh_m0; Frho = Frho_m0; e_v = e_v_m0; p_v = p_v_m0;
    Frhpk = Frhoh_m0; Fnupk = Frho_m0; Fevpk = e_v_m0; Fpvpk = p_v_m0;
    collapsed = true;
  } else {
    zvir1 = zvir1p_m0;
    Frhpk = Frhoh_m0; Fnupk = Frho_m0; Fevpk = e_v_m0; Fpvpk = p_v_m0;
    gradpk_prev = gradpk_m0; gradpkf_prev = gradpkf_m0; strain_mat = Ebar_m0;
    Frhoh = Frhoh_m0; Frho = Frho_m0; e_v = e_v_m0; p_v = p_v_m0;
    Ebar_last = Ebar_m0; gradpk_last = gradpk_m0; gradpkf_last = gradpkf_m0;
    if (m0 == 1) { g_dump[2]++; no_collapse(out); return; }
    for (int64_t mp = m0 - 1; mp >= 1; mp--) {
      const double rupp_mp = rad[mp] + 2.0;
      const double rlow_mp = std::max(rad[mp] - 2.0, 0.0);
      if (rad[mupp] > rupp_mp) {
        int64_t mn = mp;
        for (int64_t m1 = mp + 1; m1 <= mupp; m1++) if (rad[m1] < rupp_mp) mn = m1;
        mupp = mn;
      }
      if (mlow > 1 && rad[mlow - 1] > rlow_mp) {
        int64_t mn = mlow;
        for (int64_t m1 = mlow - 1; m1 >= 1; m1--) if (rad[m1] > rlow_mp) mn = m1;
        mlow = mn;
      }
      Mat3 Ebar_mp; Vec3 gradpk_mp, gradpkf_mp;
      kernel_strain(rad, G, Gf, SR, (int)mp, (int)mlow, (int)mupp, P.akk, wRnor, aRnor, 1.0, 1.0, &Ebar_mp, &gradpk_mp, &gradpkf_mp);
      evals(Ebar_mp, lam);
      double Frho_mp = lam[0] + lam[1] + lam[2];
      double e_v_mp = 0.0, p_v_mp = 0.0;
      if (Frho_mp > 0.0) {
        e_v_mp = 0.5 * (lam[2] - lam[0]) / Frho_mp;
        p_v_mp = 0.5 * (lam[2] + lam[0] - 2.0 * lam[1]) / Frho_mp;
      }
      const double Frhoh_mp = Frho_mp;
      Frho_mp = Fbar[mp];
      double zvir1p_mp = -1.0;
      if (Frho_mp > 0.0) {
        const double poe = e_v_mp < 1e-5 ? 0.0 : p_v_mp / e_v_mp;
        zvir1p_mp = tab_interp(P.T, std::log10(Frho_mp), e_v_mp, poe);
      }
      if (zvir1p_mp >= ZZon) {
        m0 = mp + 1;
        zvir1p = zvir1p_mp;
        Ebar_last = Ebar_mp; gradpk_last = gradpk_mp; gradpkf_last = gradpkf_mp;
        Frhoh = Frhoh_mp; Frho = Frho_mp; e_v = e_v_mp; p_v = p_v_mp;
        collapsed = true;
        break;
      }
      zvir1 = zvir1p_mp;
      Frhpk = Frhoh_mp; Fnupk = Frho_mp; Fevpk = e_v_mp; Fpvpk = p_v_mp;
      gradpk_prev = gradpk_mp; gradpkf_prev = gradpkf_mp; strain_mat = Ebar_mp;
      Frhoh = Frhoh_mp; Frho = Frho_mp; e_v = e_v_mp; p_v = p_v_mp;
      Ebar_last = Ebar_mp; gradpk_last = gradpk_mp; gradpkf_last = gradpkf_mp;
    }
  }
  if (!collapsed) { g_dump[3]++; no_collapse(out); return; }

  // Phase 6: interpolate to the collapse radius
  const double dZvir = zvir1p - zvir1;
  double RTHL;
  if (zvir1 > 0.0 && dZvir != 0.0) {
    const double a3 = rad[m0 - 1] * rad[m0 - 1] * rad[m0 - 1], b3 = rad[m0] * rad[m0] * rad[m0];
    const double R3 = a3 + (b3 - a3) * (zvir1p - ZZon) / dZvir;
    RTHL = std::pow(R3, 1.0 / 3.0);
  } else {
    RTHL = rad[m0 - 1];
  }
  if (RTHL <= 0.0) { g_dump[4]++; no_collapse(out); return; }
  const double RTHL3 = RTHL * RTHL * RTHL, RTHL5 = RTHL3 * RTHL * RTHL;
  const double rad3p = rad[m0 - 1] * rad[m0 - 1] * rad[m0 - 1], rad3 = rad[m0] * rad[m0] * rad[m0];
  const double drad3 = rad3 - rad3p, dFb = Fbar[m0] - Fbar[m0 - 1];
  double Fbarx;
  Vec3 gradpk_f, gradpkf_f;
  if (zvir1 > 0.0 && drad3 != 0.0) {
    const double fr = (RTHL3 - rad3p) / drad3;
    Fbarx = Fbar[m0 - 1] + fr * dFb;
    Frhpk = Frhoh + fr * (Frhpk - Frhoh);
    Fnupk = Frho + fr * (Fnupk - Frho);
    Fevpk = e_v + fr * (Fevpk - e_v);
    Fpvpk = p_v + fr * (Fpvpk - p_v);
    for (int L = 0; L < 3; L++) {
      for (int K = 0; K < 3; K++) strain_mat.m[L][K] = Ebar_last.m[L][K] + fr * (strain_mat.m[L][K] - Ebar_last.m[L][K]);
      gradpk_f.v[L] = gradpk_last.v[L] + fr * (gradpk_prev.v[L] - gradpk_last.v[L]);
      gradpkf_f.v[L] = gradpkf_last.v[L] + fr * (gradpkf_prev.v[L] - gradpkf_last.v[L]);
    }
  } else {
    Fbarx = Fbar[m0 - 1];
    Fnupk = Frho; Fevpk = e_v; Fpvpk = p_v;
    strain_mat = Ebar_last;
    gradpk_f = gradpk_prev; gradpkf_f = gradpkf_prev;
  }
  // normalize_strain (RadialShell.jl:209-212) then eigenvalues
  {
    const double tr = strain_mat.m[0][0] + strain_mat.m[1][1] + strain_mat.m[2][2];
    if (tr != 0.0) for (int L = 0; L < 3; L++) for (int K = 0; K < 3; K++) strain_mat.m[L][K] *= Fbarx / tr;
  }
  evals(strain_mat, lam);
  const double Frhoc = lam[0] + lam[1] + lam[2];
  const double e_v_f = Frhoc > 0.0 ? 0.5 * (lam[2] - lam[0]) / Frhoc : 0.0;
  const double p_v_f = Frhoc > 0.0 ? 0.5 * (lam[2] + lam[0] - 2.0 * lam[1]) / Frhoc : 0.0;
  Mat3 smat;
  for (int L = 0; L < 3; L++) for (int K = 0; K < 3; K++) smat.m[L][K] = Ebar_last.m[L][K] * (Fbarx / Frhoh);

  // Phase 7
  double Sbar[3] = {0, 0, 0}, Sbar2[3] = {0, 0, 0};
  int64_t nSbar = 0;
  for (int64_t m1 = 1; m1 <= m0 - 1; m1++)
    if (nshell[m1] > 0) {
      for (int L = 0; L < 3; L++) { Sbar[L] += S[L][m1]; Sbar2[L] += S2[L][m1]; }
      nSbar += nshell[m1];
    }
  if (nSbar > 0) for (int L = 0; L < 3; L++) { Sbar[L] /= nSbar; Sbar2[L] /= nSbar; }
  double Srb = 0.0, rad5p = 0.0;
  if (m0 > 2)
    for (int64_t mp = 2; mp <= m0 - 1; mp++) {
      const double r5 = std::pow(rad[mp], 5);
      Srb += 0.5 * (Fbar[mp - 1] + Fbar[mp]) * (r5 - rad5p);
      rad5p = r5;
    }
  if (zvir1 > 0.0 && dZvir != 0.0) Srb += 0.5 * (Fbar[m0 - 1] + Fbarx) * (RTHL5 - rad5p);
  if (Fbarx * RTHL5 > 0.0) Srb /= (Fbarx * RTHL5);

  if (P.mask) {
    for (int64_t jp = 1; jp <= npart; jp++) {
      const int32_t* c = sh + 4 * (jp - 1);
      if (std::sqrt((double)c[3]) > RTHL) continue;
      const int64_t iv1 = pi + c[0], iv2 = pj + c[1], iv3 = pk + c[2];
      if (iv1 < nbuff + 1 || iv1 > n1 - nbuff || iv2 < nbuff + 1 || iv2 > n2 - nbuff || iv3 < nbuff + 1 || iv3 > n3 - nbuff) continue;
      P.mask[lin(iv1, iv2, iv3)] = 1;
    }
  }
  double d2F = 0.0;
  if (P.lapd) {
    int64_t navg = 0;
    for (int64_t jp = 2; jp <= npart; jp++) {
      const int32_t* c = sh + 4 * (jp - 1);
      if (std::sqrt((double)c[3]) > RTHL) continue;
      const int64_t iv1 = pi + c[0], iv2 = pj + c[1], iv3 = pk + c[2];
      if (iv1 < 1 || iv1 > n1 || iv2 < 1 || iv2 > n2 || iv3 < 1 || iv3 > n3) break;
      navg += 1;
      d2F += (double)P.lapd[lin(iv1, iv2, iv3)];
    }
    if (navg > 0) d2F /= navg;
  }

  // zvir_half
  double zvir_half = -1.0;
  if (RTHL / hlatt >= 3.0) {
    for (int jj = 1; jj <= 10; jj++) {
      const double rcur = RTHL * std::pow((jj - 1) / 9.0 * 0.5 + 0.5, 1.0 / 3.0);
      const double rupp_rc = rcur + 2.0 * hlatt;
      int64_t mupp_rc = 1;
      for (int64_t m1 = 2; m1 <= m - 1; m1++) {
        if (rad[m1] > rupp_rc) { mupp_rc = m1; break; }
        else if (rad[m1] == 0.0) { mupp_rc = m1 - 1; break; }
        mupp_rc = m1;
      }
      const double rlow_rc = std::max(rcur - 2.0 * hlatt, 0.0);
      int64_t mlow_rc = 1;
      for (int64_t m1 = 1; m1 <= m - 1; m1++) if (rad[m1] > rlow_rc) { mlow_rc = m1; break; }
      int64_t m0_rc = 1;
      for (int64_t m1 = 1; m1 <= m - 1; m1++) { if (rad[m1] > rcur) { m0_rc = m1; break; } m0_rc = m1; }
      Mat3 Erc; Vec3 a1, a2;
      kernel_strain(rad, G, Gf, SR, (int)m0_rc, (int)mlow_rc, (int)mupp_rc, P.akk, wRnor, aRnor, 1.0, 1.0, &Erc, &a1, &a2);
      evals(Erc, lam);
      const double Fr = lam[0] + lam[1] + lam[2];
      double ev = 0.0, pv = 0.0;
      if (Fr > 0.0) { ev = 0.5 * (lam[2] - lam[0]) / Fr; pv = 0.5 * (lam[2] + lam[0] - 2.0 * lam[1]) / Fr; }
      const double Frc = Fbar[m0_rc];
      const double poe = ev < 1e-5 ? 0.0 : pv / ev;
      double zrc = -1.0;
      if (Frc > 0.0) zrc = tab_interp(P.T, std::log10(Frc), ev, poe);
      zvir_half = std::max(zrc - 1.0, zvir_half);
    }
  }
  (void)Frhpk; (void)Fnupk; (void)Fevpk; (void)Fpvpk;
  out[R_RTHL] = RTHL; out[R_SRB] = Srb;
  for (int L = 0; L < 3; L++) {
    out[R_SBAR + L] = Sbar[L]; out[R_SBAR2 + L] = Sbar2[L];
    out[R_GRADPK + L] = gradpk_f.v[L]; out[R_GRADRF + L] = gradpkrf.v[L]; out[R_GRADF + L] = gradpkf_f.v[L];
  }
  for (int K = 0; K < 3; K++) for (int L = 0; L < 3; L++) out[R_STRAIN + L + 3 * K] = smat.m[L][K];
  out[R_FBARX] = Fbarx; out[R_EV] = e_v_f; out[R_PV] = p_v_f; out[R_ZVH] = zvir_half; out[R_D2F] = d2F;
}

// Batched entry: peaks given by 1-based flat index ipp, per-peak Rf, ir2min,
// ZZon and fcrit.  Fields are column-major n1 x n2 x n3 Float32 arrays; e2*
// and lapd may be null; mask may be null.  When `serial_mask` is nonzero
// the peaks run in order on one thread so the mask evolves deterministically
// (the reference runs them under Threads.@threads, where the mask writes of
// RadialShell.jl:793-802 race with the rmax2rs pre-mask read).
void ora_analyse_peaks(const float* delta, const float* ex, const float* ey, const float* ez,
                       const float* e2x, const float* e2y, const float* e2z, const float* lapd,
                       int8_t* mask, int64_t n1, int64_t n2, int64_t n3,
                       const int32_t* shells, int64_t nshells,
                       const float* tab, int nx, int ny, int nz, double x1, double x2, double y1,
                       double y2, double z1, double z2,
                       int64_t npk, const int64_t* ipp, const double* Rf, const int64_t* ir2min,
                       const double* ZZon, const double* fcrit, double alatt, int64_t nbuff,
                       double rmax2rs, int serial_mask, int truncate, double* out) {
  std::vector<double> akk(1101);
  ora_atab4(akk.data());
  // distinct r^2 values, their radii (shell m = value m - 1) and, for the
  // truncated gather, need[m] = min(mmax, l + 2) with l the outermost shell
  // within rad[m] + 2 (mmax: the shells finalised over the whole list)
  std::vector<double> srad(1, 0.0);
  for (int64_t jp = 1; jp <= nshells; jp++)
    if (jp == 1 || shells[4 * (jp - 1) + 3] != shells[4 * (jp - 2) + 3])
      srad.push_back(std::sqrt((double)shells[4 * (jp - 1) + 3]));
  const int64_t nd = (int64_t)srad.size() - 1;
  const int64_t mmax = std::max<int64_t>(nd - 1, 1);
  std::vector<int> need(nd + 2, (int)mmax);
  for (int64_t mm = 1; mm <= mmax; mm++) {
    int64_t l = mm;
    while (l + 1 <= mmax && srad[l + 1] <= srad[mm] + 2.0) l++;
    need[mm] = (int)std::min<int64_t>(mmax, l + 2);
  }
  srad.push_back(0.0);
  PeakCtx P{delta, ex, ey, ez, e2x, e2y, e2z, lapd, mask, n1, n2, n3, shells, nshells, akk.data(),
            OraTable{tab, nx, ny, nz, x1, x2, y1, y2, z1, z2}, nd, truncate, srad.data(), need.data()};
  if (serial_mask) {
    for (int64_t p = 0; p < npk; p++)
      analyse_peak(P, ipp[p], alatt, ir2min[p], ZZon[p], Rf[p], nbuff, rmax2rs, fcrit[p], out + R_N * p);
  } else {
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t p = 0; p < npk; p++)
      analyse_peak(P, ipp[p], alatt, ir2min[p], ZZon[p], Rf[p], nbuff, rmax2rs, fcrit[p], out + R_N * p);
  }
}

void ora_dump_counts(long* out) { for (int i = 0; i < 5; i++) out[i] = g_dump[i].load(); }
void ora_reset_dump_counts(void) { for (int i = 0; i < 5; i++) g_dump[i] = 0; }

// ---------------------------------------------------------------------------
// run_tile record packing: Pipeline.jl:217-308.  Given per-peak results and
// peak data (positions in Mpc/h, Rf, FcollvRf, d2FRf), fill records (11 or 33
// floats) for RTHL > 0 and (ievol != 1 or z <= z_max); returns the count.
// zzon_out receives the per-peak 1+z used.
// ---------------------------------------------------------------------------
int64_t ora_pack_records(double Om, double OB, double OL, double h, int64_t npk,
                         const double* px, const double* py, const double* pz, const double* Rf,
                         const float* FcRf, const float* d2Rf, const double* res, double alatt,
                         int ievol, double z_out, double z_max, double obsx, double obsy, double obsz,
                         int ioutshear, int ilpt, float* rec, double* zzon_out) {
  OraGrowth G = growth_tables(Om, OB, OL, h);
  OraChi T;
  if (ievol == 1) T = build_chi2z(Om, OL, h, z_max + 1.0, 2000);
  const double Omnr = Om, vTH = 100.0 * h * std::sqrt(Omnr);
  (void)vTH;
  const int nf = ioutshear >= 1 ? 33 : 11;
  int64_t nh = 0;
  for (int64_t p = 0; p < npk; p++) {
    double Z;
    if (ievol == 1) {
      const double dx = px[p] - obsx, dy = py[p] - obsy, dz = pz[p] - obsz;
      Z = 1.0 + chi_to_z(T, std::sqrt(dx * dx + dy * dy + dz * dz));
    } else Z = 1.0 + z_out;
    zzon_out[p] = Z;
    const double* r = res + R_N * p;
    if (r[R_RTHL] <= 0.0) continue;
    const double zpk = Z - 1.0;
    if (ievol == 1 && zpk > z_max) continue;
    const double a_pk = 1.0 / Z;
    double Dl, HD, Da;
    dlinear_ab(G, a_pk, &Dl, &HD, &Da);
    const double Dpk = Da;   // Pipeline.jl:259 keeps the third return value
    const float RTHLp = (float)(r[R_RTHL] * alatt);
    double v2f = 0.0;
    if (ilpt >= 2) {
      const double Oma = Omnr * (a_pk * a_pk * a_pk) / (Omnr * (a_pk * a_pk * a_pk) + OL);
      v2f = -(-3.0 / 7.0 * std::pow(Oma, -1.0 / 143) * (Dpk * Dpk));
    }
    float* o = rec + (int64_t)nf * nh;
    o[0] = (float)px[p]; o[1] = (float)py[p]; o[2] = (float)pz[p];
    for (int L = 0; L < 3; L++) o[3 + L] = (float)(r[R_SBAR + L] * Dpk);
    o[6] = RTHLp;
    for (int L = 0; L < 3; L++) o[7 + L] = (float)(r[R_SBAR2 + L] * v2f);
    o[10] = (float)r[R_FBARX];
    if (nf == 33) {
      const double* s = r + R_STRAIN;   // column-major
      o[11] = (float)r[R_EV]; o[12] = (float)r[R_PV];
      o[13] = (float)s[0]; o[14] = (float)s[4]; o[15] = (float)s[8];
      o[16] = (float)s[1 + 3 * 2]; o[17] = (float)s[0 + 3 * 2]; o[18] = (float)s[0 + 3 * 1];
      o[19] = (float)r[R_D2F]; o[20] = (float)r[R_ZVH];
      for (int L = 0; L < 3; L++) { o[21 + L] = (float)r[R_GRADPK + L]; o[24 + L] = (float)r[R_GRADF + L]; }
      o[27] = (float)Rf[p]; o[28] = FcRf[p]; o[29] = d2Rf[p];
      for (int L = 0; L < 3; L++) o[30 + L] = (float)r[R_GRADRF + L];
    }
    nh++;
  }
  return nh;
}


// ---------------------------------------------------------------------------
// merge_catalog (src/Merger/Merger.jl:31-78, src/Merger/Exclusion.jl:29-221),
// sequential as the reference: NC^3 linked-list hash over the padded domain,
// halos in decreasing radius (stable), pass 1 exclusion, pass 2 volume
// reduction with each pair counted from both sides and halved.
// ---------------------------------------------------------------------------
void ora_sphere_overlap(double d, double r1, double r2, double* v1, double* v2) {
  *v1 = 0.0;
  *v2 = 0.0;
  if (d >= r1 + r2) return;
  if (d <= std::fabs(r1 - r2)) return;
  const double h1 = (r2 - r1 + d) * (r2 + r1 - d) / (2.0 * d);
  const double h2 = (r1 - r2 + d) * (r1 + r2 - d) / (2.0 * d);
  const double pi = 3.141592653589793;
  *v1 = (pi / 3.0) * (h1 * h1) * (3.0 * r1 - h1);
  *v2 = (pi / 3.0) * (h2 * h2) * (3.0 * r2 - h2);
}

// survivors (in input order) are written to out with the reduced RTHL;
// keep (optional, n entries) receives 1 for survivors; returns their number
int64_t ora_merge_catalog(const float* rec, int64_t n, int nf, float* out, int32_t* keep) {
  if (n <= 0) return 0;
  const int NC = 256;
  std::vector<double> x(n), y(n), z(n), r(n);
  for (int64_t i = 0; i < n; i++) {
    x[i] = rec[i * nf + 0];
    y[i] = rec[i * nf + 1];
    z[i] = rec[i * nf + 2];
    r[i] = rec[i * nf + 6];
  }
  std::vector<int64_t> order(n);
  for (int64_t i = 0; i < n; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return r[a] > r[b]; });
  const double rmax = *std::max_element(r.begin(), r.end());
  double mn[3] = {x[0], y[0], z[0]}, mx[3] = {x[0], y[0], z[0]};
  for (int64_t i = 1; i < n; i++) {
    mn[0] = std::min(mn[0], x[i]); mx[0] = std::max(mx[0], x[i]);
    mn[1] = std::min(mn[1], y[i]); mx[1] = std::max(mx[1], y[i]);
    mn[2] = std::min(mn[2], z[i]); mx[2] = std::max(mx[2], z[i]);
  }
  const double pad = 2.0 * rmax;
  double dmin[3], L = 0.0;
  for (int d = 0; d < 3; d++) {
    dmin[d] = mn[d] - pad;
    L = std::max(L, (mx[d] + pad) - (mn[d] - pad));
  }
  const double cs = L / NC;
  auto cidx = [&](double v, int d) {
    int c = (int)std::floor((v - dmin[d]) / cs) + 1;
    return c < 1 ? 1 : (c > NC ? NC : c);
  };
  std::vector<int32_t> hoc((size_t)NC * NC * NC, 0), ll(n, 0);   // 1-based chains, 0 = end
  auto H = [&](int ix, int iy, int iz) -> int32_t& {
    return hoc[(size_t)(ix - 1) + (size_t)NC * ((iy - 1) + (size_t)NC * (iz - 1))];
  };
  for (int64_t m = 0; m < n; m++) {
    int32_t& h = H(cidx(x[m], 0), cidx(y[m], 1), cidx(z[m], 2));
    ll[m] = h;
    h = (int32_t)(m + 1);
  }
  std::vector<char> surv(n, 1);
  // pass 1
  for (int64_t rk = 0; rk < n; rk++) {
    const int64_t i = order[rk];
    if (!surv[i]) continue;
    const double ri = r[i], xi = x[i], yi = y[i], zi = z[i];
    const int dcell = (int)std::ceil(ri / cs);
    const int ci = cidx(xi, 0), cj = cidx(yi, 1), ck = cidx(zi, 2);
    for (int diz = -dcell; diz <= dcell; diz++)
      for (int diy = -dcell; diy <= dcell; diy++)
        for (int dix = -dcell; dix <= dcell; dix++) {
          const int jx = dix + ci, jy = diy + cj, jz = diz + ck;
          if (jx < 1 || jx > NC || jy < 1 || jy > NC || jz < 1 || jz > NC) continue;
          int32_t j1 = H(jx, jy, jz);
          while (j1 > 0) {
            const int64_t j = j1 - 1;
            if (j != i && surv[j] && ri >= r[j]) {
              const double dx = x[j] - xi, dy = y[j] - yi, dz = z[j] - zi;
              const double dist = std::sqrt(dx * dx + dy * dy + dz * dz);
              if (dist < ri) surv[j] = 0;
            }
            j1 = ll[j];
          }
        }
  }
  // pass 2
  std::vector<double> dV(n, 0.0);
  const double rfirst = r[order[0]];
  for (int64_t rk = 0; rk < n; rk++) {
    const int64_t i = order[rk];
    if (!surv[i]) continue;
    const double ri = r[i], xi = x[i], yi = y[i], zi = z[i];
    const int dcell = (int)std::ceil((ri + rfirst) / cs);
    const int ci = cidx(xi, 0), cj = cidx(yi, 1), ck = cidx(zi, 2);
    for (int diz = -dcell; diz <= dcell; diz++)
      for (int diy = -dcell; diy <= dcell; diy++)
        for (int dix = -dcell; dix <= dcell; dix++) {
          const int jx = dix + ci, jy = diy + cj, jz = diz + ck;
          if (jx < 1 || jx > NC || jy < 1 || jy > NC || jz < 1 || jz > NC) continue;
          int32_t j1 = H(jx, jy, jz);
          while (j1 > 0) {
            const int64_t j = j1 - 1;
            if (j != i && surv[j]) {
              const double rj = r[j];
              const double dx = x[j] - xi, dy = y[j] - yi, dz = z[j] - zi;
              const double dist = std::sqrt(dx * dx + dy * dy + dz * dz);
              if (dist < ri + rj && dist > std::fabs(ri - rj)) {
                double v1, v2;
                ora_sphere_overlap(dist, ri, rj, &v1, &v2);
                dV[i] += v1;
                dV[j] += v2;
              }
            }
            j1 = ll[j];
          }
        }
  }
  const double fpt = 4.0 * 3.141592653589793 / 3.0;
  int64_t m = 0;
  for (int64_t i = 0; i < n; i++) {
    double rn = 0.0;
    if (surv[i]) {
      const double vol_new = fpt * (r[i] * r[i] * r[i]) - dV[i] * 0.5;
      if (vol_new <= 0.0) surv[i] = 0;
      else rn = std::pow(vol_new / fpt, 1.0 / 3.0);
    }
    if (keep) keep[i] = surv[i];
    if (!surv[i]) continue;
    for (int f = 0; f < nf; f++) out[m * nf + f] = rec[i * nf + f];
    out[m * nf + 6] = (float)rn;
    m++;
  }
  return m;
}


// ---------------------------------------------------------------------------
// Multi-resolution (MUSIC-style) per-tile building blocks,
// src/MultiResolution.jl: _downsample_noise (:68-89), _generate_extended_residual
// (:197-236), _tricubic / _catmull_rom (:156-189), _interpolate_to_tile (:95-122),
// the transfer multiply of _isolated_convolve (:246-283) and
// _apply_kernel_inplace! (:1239-1255).  Indices 0-based here; the reference's
// 1-based (it, jt, kt) tile numbers are kept.
// ---------------------------------------------------------------------------
void ora_mr_coarse_noise(int64_t N, int64_t M, uint64_t seed, float* out) {
  const int64_t block = N / M;
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
  for (int64_t K = 0; K < M; K++)
    for (int64_t J = 0; J < M; J++)
      for (int64_t I = 0; I < M; I++) {
        double val = 0.0;
        for (int64_t dk = 0; dk < block; dk++)
          for (int64_t dj = 0; dj < block; dj++)
            for (int64_t di = 0; di < block; di++) {
              const int64_t gi = I * block + di, gj = J * block + dj, gk = K * block + dk;
              val += ppbm::noise_cell_d(seed, (uint64_t)(gi + N * (gj + N * gk)));   // Float64 deviate
            }
        const double b = (double)block;
        out[I + M * (J + M * K)] = (float)(val / std::sqrt(b * b * b));
      }
}

static inline int64_t mod0(int64_t i, int64_t n) { int64_t r = i % n; return r < 0 ? r + n : r; }

void ora_mr_residual(const float* coarse, int64_t M, int64_t it, int64_t jt, int64_t kt, int64_t nsub, int64_t nmesh,
                     int64_t N, uint64_t seed, int64_t nshell, float* out) {
  const int64_t block = N / M, nbuff = (nmesh - nsub) / 2, next = nmesh + 2 * nshell;
  const double b = (double)block;
  const float inv = (float)(1.0 / std::sqrt(b * b * b));
  // 0-based origin of the extended region in global cells
  const int64_t i0 = (it - 1) * nsub - nbuff - nshell, j0 = (jt - 1) * nsub - nbuff - nshell,
                k0 = (kt - 1) * nsub - nbuff - nshell;
#pragma omp parallel for schedule(static)
  for (int64_t lk = 0; lk < next; lk++)
    for (int64_t lj = 0; lj < next; lj++)
      for (int64_t li = 0; li < next; li++) {
        const int64_t gi = mod0(i0 + li, N), gj = mod0(j0 + lj, N), gk = mod0(k0 + lk, N);
        const float fine = ppbm::noise_cell(seed, (uint64_t)(gi + N * (gj + N * gk)));
        const float bm = coarse[gi / block + M * (gj / block + M * (gk / block))] * inv;
        out[li + next * (lj + next * lk)] = fine - bm;
      }
}

static inline void catmull_rom(float t, float* w) {
  const float t2 = t * t, t3 = t2 * t;
  w[0] = -0.5f * t3 + t2 - 0.5f * t;
  w[1] = 1.5f * t3 - 2.5f * t2 + 1.0f;
  w[2] = -1.5f * t3 + 2.0f * t2 + 0.5f * t;
  w[3] = 0.5f * t3 - 0.5f * t2;
}

void ora_mr_tricubic(const float* coarse, int64_t M, int64_t it, int64_t jt, int64_t kt, int64_t nsub, int64_t nmesh,
                     int64_t N, float* out) {
  const int64_t block = N / M, nbuff = (nmesh - nsub) / 2;
  const int64_t i0 = (it - 1) * nsub - nbuff, j0 = (jt - 1) * nsub - nbuff, k0 = (kt - 1) * nsub - nbuff;
#pragma omp parallel for schedule(static)
  for (int64_t lk = 0; lk < nmesh; lk++)
    for (int64_t lj = 0; lj < nmesh; lj++)
      for (int64_t li = 0; li < nmesh; li++) {
        // 1-based global cell gi (as the reference) -> fractional coarse coordinate
        const int64_t g[3] = {mod0(i0 + li, N) + 1, mod0(j0 + lj, N) + 1, mod0(k0 + lk, N) + 1};
        int64_t ic[3];
        float w[3][4];
        for (int d = 0; d < 3; d++) {
          const double f = ((double)g[d] - 0.5) / (double)block + 0.5;
          ic[d] = (int64_t)std::floor(f);
          catmull_rom((float)(f - (double)ic[d]), w[d]);
        }
        float val = 0.0f;
        for (int a = 0; a < 4; a++) {
          const int64_t kk = mod0(ic[2] - 1 + a - 1, M);   // mod1(iz + dkk, M) - 1
          for (int bq = 0; bq < 4; bq++) {
            const int64_t jj = mod0(ic[1] - 1 + bq - 1, M);
            for (int c = 0; c < 4; c++) {
              const int64_t ii = mod0(ic[0] - 1 + c - 1, M);
              val += w[0][c] * w[1][bq] * w[2][a] * coarse[ii + M * (jj + M * kk)];
            }
          }
        }
        out[li + nmesh * (lj + nmesh * lk)] = val;
      }
}

// kernel kinds (the reference's kernel_fn ids): 0 none, 1 i k_d1/k^2 (1LPT),
// 2 -i k_d1/k^2 (2LPT), 3 -k_d1 k_d2/k^2 (phi_ij), 4 k^2 (Laplacian); d1, d2
// in 1..3.  v *= mult * kernel, rounded once to complex64.
static inline c64 apply_kind(c64 v, double mult, int kind, int d1, int d2, double kx, double ky, double kz,
                             double k2) {
  const double kv[3] = {kx, ky, kz};
  const double a = (double)v.real(), b = (double)v.imag();
  switch (kind) {
    case 0: return c64((float)(a * mult), (float)(b * mult));
    case 1: { const double c = mult * (kv[d1 - 1] / k2); return c64((float)(-b * c), (float)(a * c)); }
    case 2: { const double c = mult * (-kv[d1 - 1] / k2); return c64((float)(-b * c), (float)(a * c)); }
    case 3: { const double c = mult * (-kv[d1 - 1] * kv[d2 - 1] / k2); return c64((float)(a * c), (float)(b * c)); }
    default: { const double c = mult * k2; return c64((float)(a * c), (float)(b * c)); }
  }
}

// the transfer multiply of _isolated_convolve (on the rfft of the padded
// n2^3 box, box = n2 * dx) and of _periodic_convolve! (:286-309, box =
// boxsize): sqrt(P(k) dk^3 n2^3) times the kernel, dk = 2 pi / box, DC := 0
void ora_mr_transfer(c64* arr, int64_t n2, double box, const double* k, const double* pk, int np, int kind, int d1,
                     int d2) {
  std::vector<double> lk(np), lp(np);
  for (int i = 0; i < np; i++) { lk[i] = std::log(k[i]); lp[i] = std::log(pk[i]); }
  const double dk = 2.0 * PI / box;
  const double mult = ((double)n2 * dk) / (double)n2;
  const int64_t nh = n2 / 2 + 1;
  const double nd = (double)n2;
#pragma omp parallel for schedule(static)
  for (int64_t iz = 0; iz < n2; iz++)
    for (int64_t iy = 0; iy < n2; iy++)
      for (int64_t ix = 0; ix < nh; ix++) {
        const double kx = (double)ix * mult, ky = freq(iy, n2, mult), kz = freq(iz, n2, mult);
        const double k2 = kx * kx + ky * ky + kz * kz;
        c64& v = arr[ix + nh * (iy + n2 * iz)];
        if (k2 == 0.0) { v = c64(0.f, 0.f); continue; }
        const double amp = std::sqrt(pk_eval(lk.data(), lp.data(), np, std::sqrt(k2)) * (dk * dk * dk) * (nd * nd * nd));
        v = apply_kind(v, amp, kind, d1, d2, kx, ky, kz, k2);
      }
}

// _apply_kernel_inplace!: periodic n^3 box; DC, ix = n/2, iy = n/2 and
// iz = n/2 zeroed
void ora_mr_apply_kernel(c64* arr, int64_t n, double boxsize, int kind, int d1, int d2) {
  const double dk = 2.0 * PI / boxsize;
  const double mult = ((double)n * dk) / (double)n;
  const int64_t nh = n / 2 + 1, nyq = n / 2;
#pragma omp parallel for schedule(static)
  for (int64_t iz = 0; iz < n; iz++)
    for (int64_t iy = 0; iy < n; iy++)
      for (int64_t ix = 0; ix < nh; ix++) {
        const double kx = (double)ix * mult, ky = freq(iy, n, mult), kz = freq(iz, n, mult);
        const double k2 = kx * kx + ky * ky + kz * kz;
        c64& v = arr[ix + nh * (iy + n * iz)];
        if (k2 == 0.0 || ix == nh - 1 || iy == nyq || iz == nyq) { v = c64(0.f, 0.f); continue; }
        v = apply_kind(v, 1.0, kind, d1, d2, kx, ky, kz, k2);
      }
}

}  // extern "C"
