// k_fields.cu — field-generation kernels of the tile pipeline:
// Threefry noise, the k-space multipliers (sqrt P, 1LPT, phi_ij, 2LPT,
// Laplacian, filter windows), the Hermitian projection applied before every
// complex-to-real transform, the 2LPT source term, the gather-field pack and
// the peak finder.
//
// Layouts: real fields are n^3 floats, C order [k][j][i] (= Julia column-major
// [i,j,k]); half-spectra are (n/2+1) x n x n float2 with ix fastest, the
// layout cuFFT's R2C produces for that real array and the layout of Julia's
// rfft(delta).  Every multiplier folds in the 1/n^3 normalisation of the
// following inverse transform (cuFFT's C2R is unnormalised, Julia's irfft is
// normalised), passed as `post_scale`.
#include "ppb_internal.h"
#include "ppb_kspace.cuh"
#include "ppb_math.h"

namespace ppb {

namespace {

constexpr double kPi = 3.141592653589793;
using ks::fftfreq;
using ks::pk_eval;

// mode decomposition for a (nh x n) plane per blockIdx.y = iz
struct Mode {
  int ix, iy, iz;
  int64_t id;
  bool ok;
};
__device__ __forceinline__ Mode mode_of(int n, int nh) {
  Mode m;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int plane = nh * n;
  m.iz = blockIdx.y;
  m.ok = r < plane;
  m.ix = r % nh;
  m.iy = r / nh;
  m.id = (int64_t)r + (int64_t)plane * m.iz;
  return m;
}
inline dim3 mode_grid(int n) {
  const int nh = n / 2 + 1;
  return dim3((unsigned)((nh * n + 255) / 256), (unsigned)n, 1);
}

// ---------------------------------------------------------------------------
// noise: one thread per Threefry pair -> cells 2p and 2p+1
// (RandomField.jl:70-83)
// ---------------------------------------------------------------------------
__global__ void noise_kernel(float* __restrict__ out, int64_t ncell, uint64_t seed) {
  const int64_t npair = (ncell + 1) / 2;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npair;
       p += (int64_t)gridDim.x * blockDim.x) {
    double g1, g2;
    ppbm::threefry_gaussian_pair(seed, (uint64_t)p, &g1, &g2);
    const int64_t c = 2 * p;
    if (c + 1 < ncell) {
      reinterpret_cast<float2*>(out)[p] = make_float2((float)g1, (float)g2);
    } else {
      out[c] = (float)g1;
    }
  }
}

// noise_k *= sqrt(P(k) dk^3 n^3), DC := 0  (RandomField.jl:136-168)
__global__ void convolve_kernel(float2* __restrict__ nk, int n, double dk, double mult,
                                const double* __restrict__ lk, const double* __restrict__ lp, int np,
                                double pk_scale, double post_scale) {
  const int nh = n / 2 + 1;
  const Mode md = mode_of(n, nh);
  if (!md.ok) return;
  const double kx = (double)md.ix * mult, ky = fftfreq(md.iy, n, mult), kz = fftfreq(md.iz, n, mult);
  const double k2 = kx * kx + ky * ky + kz * kz;
  float2 v = nk[md.id];
  if (k2 == 0.0) {
    v = make_float2(0.f, 0.f);
  } else {
    const double nd = (double)n;
    const double amp = sqrt(pk_eval(lk, lp, np, sqrt(k2)) * pk_scale * (dk * dk * dk) * (nd * nd * nd)) * post_scale;
    v = make_float2((float)((double)v.x * amp), (float)((double)v.y * amp));
  }
  nk[md.id] = v;
}

// psi_c = i k_c / k^2 delta_k, Nyquist planes and DC zeroed (LPT.jl:21-71)
__global__ void lpt1_kernel(const float2* __restrict__ dk, float2* __restrict__ out, int n,
                            double mult, double post_scale) {
  const int nh = n / 2 + 1;
  const Mode md = mode_of(n, nh);
  if (!md.ok) return;
  const int64_t M = (int64_t)nh * n * n;
  const double kv[3] = {(double)md.ix * mult, fftfreq(md.iy, n, mult), fftfreq(md.iz, n, mult)};
  const double k2 = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
  const bool zero = (k2 == 0.0) || md.ix == nh - 1 || md.iy == n / 2 || md.iz == n / 2;
  const float2 d = dk[md.id];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    float2 o = make_float2(0.f, 0.f);
    if (!zero) {
      const double q = kv[c] / k2 * post_scale;
      o = make_float2((float)(-q * (double)d.y), (float)(q * (double)d.x));
    }
    out[c * M + md.id] = o;
  }
}

// phi_ij = -k_i k_j / k^2 delta_k, order 11 22 33 12 13 23, no Nyquist
// zeroing (LPT.jl:103-128)
__global__ void phi_kernel(const float2* __restrict__ dk, float2* __restrict__ out, int n, double mult,
                           double post_scale) {
  const int nh = n / 2 + 1;
  const Mode md = mode_of(n, nh);
  if (!md.ok) return;
  const int64_t M = (int64_t)nh * n * n;
  const double kv[3] = {(double)md.ix * mult, fftfreq(md.iy, n, mult), fftfreq(md.iz, n, mult)};
  const double k2 = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
  const float2 d = dk[md.id];
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int c = 0; c < 6; c++) {
    float2 o = make_float2(0.f, 0.f);
    if (k2 != 0.0) {
      const double q = (-kv[pa[c]]) * kv[pb[c]] / k2 * post_scale;
      o = make_float2((float)(q * (double)d.x), (float)(q * (double)d.y));
    }
    out[c * M + md.id] = o;
  }
}

// src2 = phi11 phi22 - phi12^2 + phi11 phi33 - phi13^2 + phi22 phi33 - phi23^2,
// single precision, left to right, no fused multiply-add (LPT.jl:141-143)
__global__ void src2_kernel(const float* __restrict__ phi, float* __restrict__ out, int64_t N) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    const float a = phi[i], b = phi[N + i], c = phi[2 * N + i], d = phi[3 * N + i], e = phi[4 * N + i],
                f = phi[5 * N + i];
    float t = __fmul_rn(a, b);
    t = __fsub_rn(t, __fmul_rn(d, d));
    t = __fadd_rn(t, __fmul_rn(a, c));
    t = __fsub_rn(t, __fmul_rn(e, e));
    t = __fadd_rn(t, __fmul_rn(b, c));
    t = __fsub_rn(t, __fmul_rn(f, f));
    out[i] = t;
  }
}

// psi2_c = -i k_c / k^2 src2_k with Nyquist zeroing (LPT.jl:155-182)
__global__ void lpt2_kernel(const float2* __restrict__ sk, float2* __restrict__ out, int n, double mult,
                            double post_scale) {
  const int nh = n / 2 + 1;
  const Mode md = mode_of(n, nh);
  if (!md.ok) return;
  const int64_t M = (int64_t)nh * n * n;
  const double kv[3] = {(double)md.ix * mult, fftfreq(md.iy, n, mult), fftfreq(md.iz, n, mult)};
  const double k2 = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
  const bool zero = (k2 == 0.0) || md.ix == nh - 1 || md.iy == n / 2 || md.iz == n / 2;
  const float2 s = sk[md.id];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    float2 o = make_float2(0.f, 0.f);
    if (!zero) {
      const double q = kv[c] / k2 * post_scale;
      o = make_float2((float)(q * (double)s.y), (float)(-q * (double)s.x));
    }
    out[c * M + md.id] = o;
  }
}

// k^2 delta_k with single-precision k (Pipeline.jl:35-51); post_scale folds
// both 1/n^3 factors of that function.
__global__ void lapd_kernel(const float2* __restrict__ dk, float2* __restrict__ out, int n, float dkf,
                            float post_scale) {
  const int nh = n / 2 + 1;
  const Mode md = mode_of(n, nh);
  if (!md.ok) return;
  const int nyq = n / 2;
  const float kx = __fmul_rn((float)md.ix, dkf);
  const float ky = __fmul_rn((float)(md.iy <= nyq ? md.iy : md.iy - n), dkf);
  const float kz = __fmul_rn((float)(md.iz <= nyq ? md.iz : md.iz - n), dkf);
  float k2 = __fmul_rn(kx, kx);
  k2 = __fadd_rn(k2, __fmul_rn(ky, ky));
  k2 = __fadd_rn(k2, __fmul_rn(kz, kz));
  const float2 d = dk[md.id];
  out[md.id] = make_float2(__fmul_rn(__fmul_rn(k2, d.x), post_scale), __fmul_rn(__fmul_rn(k2, d.y), post_scale));
}

// filter windows (Filters.jl:18-36, smooth_field :79-106):
// 0: exp(-(kR/2)^2/2), 1: top-hat 3(sin x - x cos x)/x^3, 3: Gaussian * k^2.
__device__ __forceinline__ double window_w(double kR, double k, int ws) {
  if (ws == 0) { const double h = kR / 2; return exp(-h * h / 2); }
  if (ws == 3) { const double h = kR / 2; return exp(-h * h / 2) * (k * k); }
  double s, c;
  sincos(kR, &s, &c);
  return 3.0 * (s - kR * c) / (kR * kR * kR);
}

// Window tables of a filter bank: W depends on k only through the integer
// q = ix^2 + fy^2 + fz^2 (fy, fz the signed frequencies), so each filter's
// two windows are tabulated once over q in double precision and rounded to
// Float32 as the reference rounds them (Tf(w)).  k = dk sqrt(q); q = 0 keeps
// the mode (the reference skips fkR == 0).
__global__ void window_table_kernel(float* __restrict__ tab, int qn, double dkk, const double* __restrict__ Rf,
                                    int wsmooth, int want_lap) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (q >= qn) return;
  const double k = dkk * sqrt((double)q);
  const double fkR = k * Rf[f];
  float w0 = 1.f, w1 = 1.f;
  if (fkR != 0.0) {
    w0 = (float)window_w(fkR, k, wsmooth);
    if (want_lap) w1 = (float)window_w(fkR, k, 3);
  }
  // (W_wsmooth, W_3 k^2) side by side: one 8-byte load per mode serves both
  reinterpret_cast<float2*>(tab + (int64_t)f * 2 * qn)[q] = make_float2(w0, w1);
}

// four modes per thread (r, r + 256, r + 512, r + 768 of one kz plane): four
// independent coalesced loads in flight per thread; the arithmetic per mode
// is unchanged
constexpr int kWinPerThread = 4;
__global__ void __launch_bounds__(256) window_kernel(const float2* __restrict__ dk, float2* __restrict__ out0,
                                                     float2* __restrict__ out1, int n, const float* __restrict__ tab,
                                                     int qn, float ps) {
  const int nh = n / 2 + 1, plane = nh * n, nyq = n / 2;
  const int iz = blockIdx.y;
  const int fz = iz <= nyq ? iz : iz - n;
  const int64_t base = (int64_t)plane * iz;
  const int r0 = blockIdx.x * (256 * kWinPerThread) + threadIdx.x;
  float2 d[kWinPerThread];
  int q[kWinPerThread];
#pragma unroll
  for (int u = 0; u < kWinPerThread; u++) {
    const int r = r0 + 256 * u;
    q[u] = -1;
    d[u] = make_float2(0.f, 0.f);
    if (r < plane) {
      const int ix = r % nh, iy = r / nh;
      const int fy = iy <= nyq ? iy : iy - n;
      q[u] = ix * ix + fy * fy + fz * fz;
      d[u] = dk[base + r];
    }
  }
#pragma unroll
  for (int u = 0; u < kWinPerThread; u++) {
    if (q[u] < 0) continue;
    const int64_t id = base + r0 + 256 * u;
    const float2 w = __ldg(reinterpret_cast<const float2*>(tab) + q[u]);
    const float w0 = w.x;
    out0[id] = make_float2(__fmul_rn(__fmul_rn(d[u].x, w0), ps), __fmul_rn(__fmul_rn(d[u].y, w0), ps));
    if (out1) {
      const float w1 = w.y;
      out1[id] = make_float2(__fmul_rn(__fmul_rn(d[u].x, w1), ps), __fmul_rn(__fmul_rn(d[u].y, w1), ps));
    }
  }
}

// ---------------------------------------------------------------------------
// Hermitian projection of the ix = 0 and ix = n/2 planes:
// X(k) <- (X(k) + conj(X(-k)))/2.  FFTW's and pocketfft's multi-dimensional
// complex-to-real transforms act on a half-spectrum as if this projection had
// been applied (the last, real transform drops the imaginary parts of its
// DC and Nyquist inputs); cuFFT gives no such guarantee for inputs that are
// not Hermitian, e.g. phi_ij off the diagonal on the Nyquist lines.
// ---------------------------------------------------------------------------
__global__ void hermitise_kernel(float2* __restrict__ data, int n, int nbatch) {
  const int nh = n / 2 + 1;
  const int64_t M = (int64_t)nh * n * n;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int per_plane = n * n;
  const int planes = (n % 2 == 0) ? 2 : 1;
  if (t >= per_plane * planes * nbatch) return;
  const int b = t / (per_plane * planes);
  const int r = t % (per_plane * planes);
  const int pl = r / per_plane;
  const int q = r % per_plane;
  const int iy = q % n, iz = q / n;
  const int ix = pl == 0 ? 0 : n / 2;
  const int jy = (n - iy) % n, jz = (n - iz) % n;
  const int64_t a_id = ix + (int64_t)nh * (iy + (int64_t)n * iz);
  const int64_t b_id = ix + (int64_t)nh * (jy + (int64_t)n * jz);
  float2* base = data + b * M;
  if (a_id == b_id) {
    base[a_id].y = 0.f;
    return;
  }
  // each unordered pair handled once, by its smaller index
  if (a_id > b_id) return;
  const float2 x = base[a_id], y = base[b_id];
  const float re = 0.5f * (x.x + y.x), im = 0.5f * (x.y - y.y);
  base[a_id] = make_float2(re, im);
  base[b_id] = make_float2(re, -im);
}

// ---------------------------------------------------------------------------
// gather-field pack: per cell two float4 = (delta, deltaT, psi_z, psi2_x),
// (psi_x, psi_y, psi2_y, psi2_z), the pairing of the shell gather's packed
// FP32x2 sums.  deltaT at (a,b,c) is delta(c,a,b): the
// transposed read delta[iv3, iv1, iv2] of RadialShell.jl:448, made into a
// plain array so the shell gather reads one 32-byte record per cell.
// Block: 32 x 8 threads over a 32 (a) x 32 (c) tile at fixed b.
// ---------------------------------------------------------------------------
__global__ void pack_kernel(float4* __restrict__ aos, FieldWindow w, int n) {
  __shared__ float tile[32][33];
  __shared__ float wmax[8][7];
  // largest |value| per field seen by this thread: delta, psi x, y, z, psi2 x, y, z
  float fm[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  const int b = blockIdx.z;
  const int a0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  const int64_t n2 = (int64_t)n * n;
  auto src = [&](int x, int y, int z) { return w.off + x + w.py * y + w.pz * z; };
  // load delta(c, a, b) for c in [c0, c0+32), a in [a0, a0+32)
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int a = a0 + r, c = c0 + threadIdx.x;
    if (a < n && c < n) tile[r][threadIdx.x] = w.delta[src(c, a, b)];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int a = a0 + threadIdx.x, c = c0 + r;
    if (a >= n || c >= n) continue;
    const int64_t g = src(a, b, c);
    const int64_t lin = a + (int64_t)n * b + n2 * c;
    const float dT = tile[threadIdx.x][r];
    float4 v0, v1;
    v0.x = w.delta[g];
    v0.y = dT;
    v0.z = w.psi[2 * w.cs + g];
    v1.x = w.psi[g];
    v1.y = w.psi[w.cs + g];
    if (w.psi2) {
      v0.w = w.psi2[g];
      v1.z = w.psi2[w.cs + g];
      v1.w = w.psi2[2 * w.cs + g];
    } else {
      v0.w = v1.z = v1.w = 0.f;
    }
    aos[2 * lin] = v0;
    aos[2 * lin + 1] = v1;
    fm[0] = fmaxf(fm[0], fabsf(v0.x));
    fm[1] = fmaxf(fm[1], fabsf(v1.x));
    fm[2] = fmaxf(fm[2], fabsf(v1.y));
    fm[3] = fmaxf(fm[3], fabsf(v0.z));
    fm[4] = fmaxf(fm[4], fabsf(v0.w));
    fm[5] = fmaxf(fm[5], fabsf(v1.z));
    fm[6] = fmaxf(fm[6], fabsf(v1.w));
  }
  // the block's field maxima into one of kFmaxSlots slots (spreads the
  // atomics over addresses); non-negative floats order as their bit patterns
#pragma unroll
  for (int f = 0; f < 7; f++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) fm[f] = fmaxf(fm[f], __shfl_xor_sync(0xffffffffu, fm[f], o));
  if (threadIdx.x == 0)
#pragma unroll
    for (int f = 0; f < 7; f++) wmax[threadIdx.y][f] = fm[f];
  __syncthreads();
  const int t = threadIdx.y * 32 + threadIdx.x;
  if (t < 7) {
    float m = 0.f;
    for (int y = 0; y < (int)blockDim.y; y++) m = fmaxf(m, wmax[y][t]);
    const unsigned slot = (blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)) % kFmaxSlots;
    atomicMax(pack_fmax(aos, n) + t * kFmaxSlots + slot, __float_as_uint(m));
  }
}

// dst (n^3, local) = a cubic window of a larger array
__global__ void extract_kernel(float* __restrict__ dst, const float* __restrict__ src, int64_t off, int64_t py,
                               int64_t pz, int n) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y, z = blockIdx.z;
  if (x >= n) return;
  dst[x + (int64_t)n * (y + (int64_t)n * z)] = src[off + x + py * y + pz * z];
}

// ---------------------------------------------------------------------------
// peak finder for one filter (PeakFind.jl:15-79).  A cell of the inner cube
// (nbuff < i <= n - nbuff, 1-based) is a peak when it is not masked, is not
// below fcrit, and no neighbour of the 3x3x3 block is strictly larger.  The
// cell's mask is set; within one filter only a peak's own cell is written,
// so the cells can be tested in parallel.  Order is restored afterwards by
// sorting the (filter, flat index) keys.
// ---------------------------------------------------------------------------
__global__ void peakfind_kernel(const float* __restrict__ ds, const float* __restrict__ ls,
                                uint8_t* __restrict__ mask, int n1, int n2, int n3, int64_t py, int64_t pz,
                                int nbuff, float fcrit, unsigned long long keyhi, PeakBuf pb) {
  const int i = nbuff + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = nbuff + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = nbuff + blockIdx.z;
  bool peak = false;
  int64_t g = 0;
  float ff = 0.f;
  if (i < n1 - nbuff && j < n2 - nbuff && k < n3 - nbuff) {
    g = i + py * j + pz * k;
    ff = ds[g];
    if (mask[g] != 1 && !(ff < fcrit)) {
      peak = true;
#pragma unroll
      for (int dk = -1; dk <= 1; dk++)
#pragma unroll
        for (int dj = -1; dj <= 1; dj++)
#pragma unroll
          for (int di = -1; di <= 1; di++) {
            const float v = __ldg(ds + g + di + py * dj + pz * dk);
            if (ff < v) peak = false;
          }
    }
  }
  const unsigned full = 0xffffffffu;
  const unsigned ball = __ballot_sync(full, peak);
  if (ball == 0) return;
  const int lane = threadIdx.x + blockDim.x * threadIdx.y;   // blockDim.x*y == 32k; lanes per warp
  const int wl = lane & 31;
  const int leader = __ffs(ball) - 1;
  int base = 0;
  if (wl == leader) base = atomicAdd(pb.count, __popc(ball));
  base = __shfl_sync(full, base, leader);
  if (peak) {
    mask[g] = 1;
    const int slot = base + __popc(ball & ((1u << wl) - 1u));
    if (slot < pb.cap) {
      const int64_t lin = i + (int64_t)n1 * j + (int64_t)n1 * n2 * k;
      pb.keys[slot] = (keyhi << 40) | (unsigned long long)lin;
      pb.vals[slot] = (uint32_t)slot;
      pb.ff[slot] = ff;
      pb.lap[slot] = ls ? ls[g] : 0.f;
    }
  }
}

// Four consecutive cells along i per thread (one 16-byte load of the field
// and one 4-byte load of the mask), for rows whose inner part starts on a
// 4-cell boundary (n1 and nbuff multiples of 4).  Same test and append as
// peakfind_kernel; the neighbours of a candidate are read one by one (few
// cells reach fcrit).
__global__ void peakfind4_kernel(const float* __restrict__ ds, const float* __restrict__ ls,
                                 uint8_t* __restrict__ mask, int n1, int n2, int n3, int64_t py, int64_t pz,
                                 int nbuff, float fcrit, unsigned long long keyhi, PeakBuf pb) {
  const int i0 = nbuff + 4 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int j = nbuff + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = nbuff + blockIdx.z;
  const int64_t n12 = pz;
  const int64_t lin0 = i0 + py * j + pz * k;
  const int64_t loc0 = i0 + (int64_t)n1 * j + (int64_t)n1 * n2 * k;
  bool pk[4] = {false, false, false, false};
  float f[4] = {0.f, 0.f, 0.f, 0.f};
  if (i0 < n1 - nbuff && j < n2 - nbuff && k < n3 - nbuff) {
    const float4 v = *reinterpret_cast<const float4*>(ds + lin0);
    const uchar4 m = *reinterpret_cast<const uchar4*>(mask + lin0);
    f[0] = v.x; f[1] = v.y; f[2] = v.z; f[3] = v.w;
    const uint8_t mm[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
    for (int u = 0; u < 4; u++) {
      if (i0 + u >= n1 - nbuff || mm[u] == 1 || f[u] < fcrit) continue;
      const int64_t lin = lin0 + u;
      bool peak = true;
      for (int dk = -1; dk <= 1 && peak; dk++)
        for (int dj = -1; dj <= 1; dj++)
#pragma unroll
          for (int di = -1; di <= 1; di++) {
            const float w = __ldg(ds + lin + di + py * dj + n12 * dk);
            if (f[u] < w) peak = false;
          }
      pk[u] = peak;
    }
  }
  const unsigned full = 0xffffffffu;
  const int cnt = (int)pk[0] + (int)pk[1] + (int)pk[2] + (int)pk[3];
  if (__ballot_sync(full, cnt > 0) == 0) return;
  const int wl = (threadIdx.x + blockDim.x * threadIdx.y) & 31;
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(full, incl, o);
    if (wl >= o) incl += y;
  }
  const int total = __shfl_sync(full, incl, 31);
  int base = 0;
  if (wl == 31) base = atomicAdd(pb.count, total);
  base = __shfl_sync(full, base, 31);
  int slot = base + incl - cnt;
#pragma unroll
  for (int u = 0; u < 4; u++) {
    if (!pk[u]) continue;
    const int64_t lin = lin0 + u;
    mask[lin] = 1;
    if (slot < pb.cap) {
      pb.keys[slot] = (keyhi << 40) | (unsigned long long)(loc0 + u);
      pb.vals[slot] = (uint32_t)slot;
      pb.ff[slot] = f[u];
      pb.lap[slot] = ls ? ls[lin] : 0.f;
    }
    slot++;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
void launch_noise(Launch L, float* out, int64_t n, uint64_t seed) {
  const int64_t ncell = n * n * n;
  const int64_t npair = (ncell + 1) / 2;
  const int threads = 256;
  const int64_t blocks = std::min<int64_t>((npair + threads - 1) / threads, 148 * 32);
  noise_kernel<<<(unsigned)blocks, threads, 0, L.s>>>(out, ncell, seed);
  PPB_LAUNCHED(*L.count);
}

void launch_convolve(Launch L, float2* nk, int n, double boxsize, const double* lk, const double* lp,
                     int np, double pk_scale, double post_scale) {
  const double dk = 2.0 * kPi / boxsize;
  const double mult = (n * dk) / (double)n;
  convolve_kernel<<<mode_grid(n), 256, 0, L.s>>>(nk, n, dk, mult, lk, lp, np, pk_scale, post_scale);
  PPB_LAUNCHED(*L.count);
}

void launch_lpt1(Launch L, const float2* dk, float2* out, int n, double boxsize, double post_scale) {
  const double dkk = 2.0 * kPi / boxsize;
  lpt1_kernel<<<mode_grid(n), 256, 0, L.s>>>(dk, out, n, (n * dkk) / (double)n, post_scale);
  PPB_LAUNCHED(*L.count);
}

void launch_phi(Launch L, const float2* dk, float2* out, int n, double boxsize, double post_scale) {
  const double dkk = 2.0 * kPi / boxsize;
  phi_kernel<<<mode_grid(n), 256, 0, L.s>>>(dk, out, n, (n * dkk) / (double)n, post_scale);
  PPB_LAUNCHED(*L.count);
}

void launch_src2(Launch L, const float* phi, float* out, int64_t N) {
  const int64_t blocks = std::min<int64_t>((N + 255) / 256, 148 * 32);
  src2_kernel<<<(unsigned)blocks, 256, 0, L.s>>>(phi, out, N);
  PPB_LAUNCHED(*L.count);
}

void launch_lpt2(Launch L, const float2* s2k, float2* out, int n, double boxsize, double post_scale) {
  const double dkk = 2.0 * kPi / boxsize;
  lpt2_kernel<<<mode_grid(n), 256, 0, L.s>>>(s2k, out, n, (n * dkk) / (double)n, post_scale);
  PPB_LAUNCHED(*L.count);
}

void launch_lapd(Launch L, const float2* dk, float2* out, int n, double boxsize, float post_scale) {
  lapd_kernel<<<mode_grid(n), 256, 0, L.s>>>(dk, out, n, (float)(2.0 * kPi / boxsize), post_scale);
  PPB_LAUNCHED(*L.count);
}

int window_table_size(int n) { return 3 * (n / 2) * (n / 2) + 1; }

void launch_window_tables(Launch L, float* tab, int n, double boxsize, const double* Rf, int nfilt, int wsmooth,
                          bool want_lap) {
  const int qn = window_table_size(n);
  window_table_kernel<<<dim3((unsigned)((qn + 255) / 256), (unsigned)nfilt), 256, 0, L.s>>>(
      tab, qn, 2.0 * kPi / boxsize, Rf, wsmooth, want_lap ? 1 : 0);
  PPB_LAUNCHED(*L.count);
}

void launch_window(Launch L, const float2* dk, float2* out0, float2* out1, int n, const float* tab,
                   double post_scale) {
  const int plane = (n / 2 + 1) * n;
  const dim3 grid((unsigned)((plane + 256 * kWinPerThread - 1) / (256 * kWinPerThread)), (unsigned)n, 1);
  window_kernel<<<grid, 256, 0, L.s>>>(dk, out0, out1, n, tab, window_table_size(n), (float)post_scale);
  PPB_LAUNCHED(*L.count);
}

void launch_hermitise(Launch L, float2* data, int n, int nbatch) {
  const int planes = (n % 2 == 0) ? 2 : 1;
  const int total = n * n * planes * nbatch;
  hermitise_kernel<<<(total + 255) / 256, 256, 0, L.s>>>(data, n, nbatch);
  PPB_LAUNCHED(*L.count);
}

void launch_pack(Launch L, float4* aos, const FieldWindow& w, int n) {
  PPB_CUDA(cudaMemsetAsync(pack_fmax(aos, n), 0, 7 * kFmaxSlots * sizeof(unsigned), L.s));
  dim3 grid((n + 31) / 32, (n + 31) / 32, n);
  pack_kernel<<<grid, dim3(32, 8), 0, L.s>>>(aos, w, n);
  PPB_LAUNCHED(*L.count);
}

void launch_extract(Launch L, float* dst, const float* src, int64_t off, int64_t py, int64_t pz, int n) {
  extract_kernel<<<dim3((unsigned)((n + 127) / 128), (unsigned)n, (unsigned)n), 128, 0, L.s>>>(dst, src, off, py, pz,
                                                                                              n);
  PPB_LAUNCHED(*L.count);
}

void launch_peakfind(Launch L, const float* ds, const float* ls, uint8_t* mask, int n1, int n2, int n3,
                     int64_t py, int64_t pz, int nbuff, float fcrit, unsigned long long keyhi, PeakBuf pb) {
  const int w1 = n1 - 2 * nbuff, w2 = n2 - 2 * nbuff, w3 = n3 - 2 * nbuff;
  if (w1 <= 0 || w2 <= 0 || w3 <= 0) return;
  dim3 block(32, 4);
  const bool vec = n1 % 4 == 0 && nbuff % 4 == 0 && py % 4 == 0 && pz % 4 == 0 &&
                   reinterpret_cast<uintptr_t>(ds) % 16 == 0 && reinterpret_cast<uintptr_t>(mask) % 4 == 0;
  if (vec) {
    const int q1 = (w1 + 3) / 4;
    dim3 grid((q1 + 31) / 32, (w2 + 3) / 4, w3);
    peakfind4_kernel<<<grid, block, 0, L.s>>>(ds, ls, mask, n1, n2, n3, py, pz, nbuff, fcrit, keyhi, pb);
  } else {
    dim3 grid((w1 + 31) / 32, (w2 + 3) / 4, w3);
    peakfind_kernel<<<grid, block, 0, L.s>>>(ds, ls, mask, n1, n2, n3, py, pz, nbuff, fcrit, keyhi, pb);
  }
  PPB_LAUNCHED(*L.count);
}

}  // namespace ppb
