// k_xpeak.cu — the last (x) pass of the filter bank's inverse transform fused
// with the peak search (Filters.jl:257-345 smoothing, Pipeline.jl:144-196 /
// PeakFinding.jl local maxima above fcrit, MultiTile.jl:218-275 mask).
//
// The window multiply (window_t_kernel) writes W(kR) delta_k transposed to
// [kx][kz][ky] (ky fastest), so cuFFT transforms it back along z and y as
// contiguous n x n planes batched over kx.  xpeak_kernel then forms each x row
// of the smoothed field with its own n-point real inverse DFT (a row's kx
// values sit n^2 apart; 16 consecutive y of one kx are one 128-byte segment)
// and keeps the rows of four consecutive z planes in shared memory, so the
// 3 x 3 x 3 maximum test runs on chip and the smoothed field never goes to
// HBM.  The k^2-weighted twin (ioutshear) is
// only needed at the peaks: its value there is a direct (n/2+1)-term sum over
// its z/y-transformed row, in FP64.
//
// Real inverse DFT of length n = 64 J (unnormalised, Hermitian input X[0..H],
// H = n/2): with Z[k] = (X[k] + conj X[H-k]) + i w^k (X[k] - conj X[H-k]),
// w = exp(2 pi i / n), the complex inverse DFT z of Z (length H) gives
// r[2m] = Re z[m], r[2m+1] = Im z[m].  The length-H DFT is split H = J x 32
// (index t = l + 32 j in, m = q + J p out): lane l holds Z[l + 32 j] for
// j < J, does the J-point DFT over j in registers, multiplies by
// exp(2 pi i l q / H), and the 32-point DFTs over l run across the warp as
// five radix-2 decimation-in-frequency stages on shuffles.  Lane l ends with
// z[q + J bitrev5(l)], i.e. the 2J consecutive reals from x = 2 J bitrev5(l).
#include <cstdint>

#include "ppb_internal.h"

namespace ppb {
namespace {

constexpr int kXpRows = 16;          // ring rows per plane: 14 inner rows + 2 halo
constexpr int kXpInner = kXpRows - 2;
constexpr int kXpThreads = 512;      // one warp per ring row
constexpr int kXpPad = 17;           // staged (kx, row) pitch in float2: conflict-free row reads

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

template <int J>
struct RowConsts {
  float2 pre[J];   // w^(l + 32 j), w = exp(2 pi i / n)
  float2 wj[J];    // exp(2 pi i m / J) = w^(64 m)
  float2 mid[J];   // exp(2 pi i l q / H) = w^(2 l q)
  float2 st[4];    // stage twiddles: exp(2 pi i (l mod h) / (2 h)) = w^(n (l mod h) / (2 h)) on the
                   // upper lane of each pair (l & h), 1 on the lower, h = 16, 8, 4, 2
  float sg[5];     // -1 on the upper lane of stage h = 16 >> s, +1 on the lower
};

// tw[k] = w^k, k < n (twiddle_kernel)
template <int J>
__device__ __forceinline__ void row_consts(RowConsts<J>& c, int l, const float2* __restrict__ tw) {
  constexpr int n = 64 * J;
#pragma unroll
  for (int j = 0; j < J; j++) {
    c.pre[j] = __ldg(tw + l + 32 * j);
    c.wj[j] = __ldg(tw + 64 * j);
    c.mid[j] = __ldg(tw + (2 * l * j) % n);
  }
#pragma unroll
  for (int s = 0; s < 5; s++) {
    const int h = 16 >> s;
    const bool up = (l & h) != 0;
    if (s < 4) c.st[s] = up ? __ldg(tw + (n / (2 * h)) * (l % h)) : make_float2(1.f, 0.f);
    c.sg[s] = up ? -1.f : 1.f;
  }
}

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul_i(float2 a) { return make_float2(-a.y, a.x); }   // i a

constexpr float kHalfSqrt3 = 0.8660254037844386f;   // sin(pi/3)
constexpr float kHalfSqrt2 = 0.7071067811865476f;   // cos(pi/4)

// A[q] = sum_j z[j] exp(2 pi i j q / J): butterflies for J = 1, 2, 3, 4, 6, 8
// (6 = 2 x 3 and 8 = 2 x 4 by one radix-2 step), the direct sum with table
// twiddles wj otherwise
__device__ __forceinline__ void dft3(const float2 a0, const float2 a1, const float2 a2, float2& o0, float2& o1,
                                     float2& o2) {
  const float2 t = cadd(a1, a2);
  const float2 m = make_float2(fmaf(-0.5f, t.x, a0.x), fmaf(-0.5f, t.y, a0.y));
  const float2 d = csub(a1, a2);
  const float2 isd = make_float2(-kHalfSqrt3 * d.y, kHalfSqrt3 * d.x);
  o0 = cadd(a0, t);
  o1 = cadd(m, isd);
  o2 = csub(m, isd);
}

__device__ __forceinline__ void dft4(const float2 a0, const float2 a1, const float2 a2, const float2 a3, float2& o0,
                                     float2& o1, float2& o2, float2& o3) {
  const float2 s02 = cadd(a0, a2), d02 = csub(a0, a2), s13 = cadd(a1, a3), d13 = cmul_i(csub(a1, a3));
  o0 = cadd(s02, s13);
  o2 = csub(s02, s13);
  o1 = cadd(d02, d13);
  o3 = csub(d02, d13);
}

template <int J>
__device__ __forceinline__ void dft_small(const float2 (&z)[J], float2 (&A)[J], const float2 (&wj)[J]) {
  if constexpr (J == 1) {
    A[0] = z[0];
  } else if constexpr (J == 2) {
    A[0] = cadd(z[0], z[1]);
    A[1] = csub(z[0], z[1]);
  } else if constexpr (J == 3) {
    dft3(z[0], z[1], z[2], A[0], A[1], A[2]);
  } else if constexpr (J == 4) {
    dft4(z[0], z[1], z[2], z[3], A[0], A[1], A[2], A[3]);
  } else if constexpr (J == 6) {
    float2 e[3], o[3];
    dft3(z[0], z[2], z[4], e[0], e[1], e[2]);
    dft3(z[1], z[3], z[5], o[0], o[1], o[2]);
    const float2 w1 = make_float2(0.5f, kHalfSqrt3), w2 = make_float2(-0.5f, kHalfSqrt3);   // exp(i pi q / 3)
    const float2 t1 = cmul(o[1], w1), t2 = cmul(o[2], w2);
    A[0] = cadd(e[0], o[0]); A[3] = csub(e[0], o[0]);
    A[1] = cadd(e[1], t1);   A[4] = csub(e[1], t1);
    A[2] = cadd(e[2], t2);   A[5] = csub(e[2], t2);
  } else if constexpr (J == 8) {
    float2 e[4], o[4];
    dft4(z[0], z[2], z[4], z[6], e[0], e[1], e[2], e[3]);
    dft4(z[1], z[3], z[5], z[7], o[0], o[1], o[2], o[3]);
    const float2 t1 = make_float2(kHalfSqrt2 * (o[1].x - o[1].y), kHalfSqrt2 * (o[1].x + o[1].y));    // exp(i pi/4) o1
    const float2 t2 = cmul_i(o[2]);
    const float2 t3 = make_float2(-kHalfSqrt2 * (o[3].x + o[3].y), kHalfSqrt2 * (o[3].x - o[3].y));   // exp(3 i pi/4) o3
    A[0] = cadd(e[0], o[0]); A[4] = csub(e[0], o[0]);
    A[1] = cadd(e[1], t1);   A[5] = csub(e[1], t1);
    A[2] = cadd(e[2], t2);   A[6] = csub(e[2], t2);
    A[3] = cadd(e[3], t3);   A[7] = csub(e[3], t3);
  } else {
#pragma unroll
    for (int q = 0; q < J; q++) {
      float2 acc = z[0];
#pragma unroll
      for (int j = 1; j < J; j++) {
        const float2 w = wj[(j * q) % J];
        acc.x = fmaf(z[j].x, w.x, fmaf(-z[j].y, w.y, acc.x));
        acc.y = fmaf(z[j].x, w.y, fmaf(z[j].y, w.x, acc.y));
      }
      A[q] = acc;
    }
  }
}

// row r of the staged plane: X[l + 32 j] and X[H]
template <int J>
__device__ __forceinline__ void row_load(const float2* stg, int r, int l, float2 (&x)[J], float2& xh) {
#pragma unroll
  for (int j = 0; j < J; j++) x[j] = stg[(l + 32 * j) * kXpPad + r];
  xh = stg[32 * J * kXpPad + r];
}

// the real inverse DFT of one row; writes the row's n reals to out
template <int J>
__device__ __forceinline__ void row_irfft(const RowConsts<J>& c, int l, const float2 (&x)[J], float2 xh,
                                          float* __restrict__ out) {
  const unsigned full = 0xffffffffu;
  const int src = (32 - l) & 31;
  float2 z[J];
#pragma unroll
  for (int j = 0; j < J; j++) {
    // conj X[H - k], k = l + 32 j: lane 32 - l, register J - 1 - j (l > 0);
    // lane 0 holds X[32 (J - j)] itself (X[H] for j = 0)
    float2 v;
    v.x = __shfl_sync(full, x[J - 1 - j].x, src);
    v.y = __shfl_sync(full, x[J - 1 - j].y, src);
    if (l == 0) v = (j == 0) ? xh : x[(J - j) % J];
    const float2 a = x[j];
    const float2 e = make_float2(a.x + v.x, a.y - v.y);   // X[k] + conj X[H-k]
    const float2 d = make_float2(a.x - v.x, a.y + v.y);   // X[k] - conj X[H-k]
    const float2 o = cmul(c.pre[j], d);
    z[j] = make_float2(e.x - o.y, e.y + o.x);             // e + i o
  }
  float2 b[J];
  dft_small<J>(z, b, c.wj);
#pragma unroll
  for (int q = 1; q < J; q++) b[q] = cmul(b[q], c.mid[q]);
  // radix-2 steps across lanes: the lower lane of a pair keeps a + b, the
  // upper (a - b) times its twiddle, a being the lower lane's value
#pragma unroll
  for (int s = 0; s < 5; s++) {
    const int h = 16 >> s;
#pragma unroll
    for (int q = 0; q < J; q++) {
      float2 p;
      p.x = __shfl_xor_sync(full, b[q].x, h);
      p.y = __shfl_xor_sync(full, b[q].y, h);
      const float2 t = make_float2(fmaf(c.sg[s], b[q].x, p.x), fmaf(c.sg[s], b[q].y, p.y));
      b[q] = s < 4 ? cmul(t, c.st[s]) : t;
    }
  }
  const int p = __brev(l) >> 27;
  float2* o2 = reinterpret_cast<float2*>(out + 2 * J * p);
#pragma unroll
  for (int q = 0; q < J; q++) o2[q] = b[q];
}

struct XpArgs {
  const float2* ds;    // z/y-transformed smoothed field, [kx][z][y], kx <= n/2
  const float2* tw;    // w^k, k < n
  uint8_t* mask;       // n^3, x fastest
  unsigned* first;     // lowest slot this launch appends (reset to ~0 before it)
  int n, nbuff, tz, lap0;   // lap0: write lap = 0 (no k^2-weighted twin)
  float fcrit;
  unsigned long long keyhi;
  PeakBuf pb;
};

constexpr int kXpList = 64;   // per-warp peak list entries

template <int J>
__global__ void __launch_bounds__(kXpThreads, 1) xpeak_kernel(XpArgs a) {
  constexpr int n = 64 * J, H = 32 * J, nh = H + 1;
  extern __shared__ __align__(16) unsigned char smem[];
  float* ring = reinterpret_cast<float*>(smem);                                    // [4][kXpRows][n]
  long long* lloc = reinterpret_cast<long long*>(smem + 4 * kXpRows * n * 4);      // [16][kXpList]
  float* lf = reinterpret_cast<float*>(lloc + 16 * kXpList);                        // [16][kXpList]
  float2* stg = reinterpret_cast<float2*>(lf + 16 * kXpList);                       // [2][nh][kXpPad]
  uint8_t* mbuf = reinterpret_cast<uint8_t*>(stg + 2 * nh * kXpPad);                // [2][kXpInner][n]
  const int tid = threadIdx.x, l = tid & 31, warp = tid >> 5;
  const int nb = a.nbuff, hi = n - nb;
  const int y0 = nb + blockIdx.x * kXpInner;
  const int z0 = nb + blockIdx.y * a.tz;
  const int yi = min(kXpInner, hi - y0);
  const int zi = min(a.tz, hi - z0);
  if (yi <= 0 || zi <= 0) return;
  const int R = yi + 2, NP = zi + 2;
  const int64_t nn = (int64_t)n * n;
  RowConsts<J> c;
  row_consts<J>(c, l, a.tw);
  // rows y0 - 1 .. y0 - 2 + R of plane z: per kx one contiguous run of R
  // float2, two kx per warp step (half-warps)
  auto stage_plane = [&](float2* stg, int z) {
    const float2* src = a.ds + (int64_t)n * z + (y0 - 1);
    const int r = l & 15;
    for (int kx = 2 * warp + (l >> 4); kx < nh; kx += 2 * (kXpThreads / 32)) {
      if (r < R) {
        const unsigned dst = (unsigned)__cvta_generic_to_shared(stg + kx * kXpPad + r);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src + nn * kx + r));
      }
    }
  };
  // mask bytes of the inner rows of plane z, x in [nb, hi) rounded out to
  // 4-byte words, into buf[row][x]
  auto stage_mask = [&](uint8_t* buf, int z) {
    const int w0 = nb >> 2, w1 = (hi + 3) >> 2;
    const uint8_t* src = a.mask + nn * z + (int64_t)n * y0;
    for (int r = warp; r < yi; r += kXpThreads / 32)
      for (int w = w0 + l; w < w1; w += 32) {
        const unsigned dst = (unsigned)__cvta_generic_to_shared(buf + r * n + 4 * w);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(src + (int64_t)n * r + 4 * w));
      }
  };
  // this warp's peak list: appended without atomics, flushed to the peak
  // buffers (one atomicAdd) when it could overflow and at the end
  const unsigned full = 0xffffffffu;
  long long* myloc = lloc + warp * kXpList;
  float* myf = lf + warp * kXpList;
  int wn = 0;
  auto flush = [&]() {
    __syncwarp();
    int base = 0;
    if (l == 0) {
      base = atomicAdd(a.pb.count, wn);
      atomicMin(a.first, (unsigned)base);
    }
    base = __shfl_sync(full, base, 0);
    for (int e = l; e < wn; e += 32) {
      const int slot = base + e;
      if (slot < a.pb.cap) {
        a.pb.keys[slot] = (a.keyhi << 40) | (unsigned long long)myloc[e];
        a.pb.vals[slot] = (uint32_t)slot;
        a.pb.ff[slot] = myf[e];
        if (a.lap0) a.pb.lap[slot] = 0.f;
      }
    }
    __syncwarp();
    wn = 0;
  };
  // iteration i: ring plane i (z = z0 - 1 + i) is transformed from staging
  // buffer i & 1 into ring slot i & 3 while plane i - 2 is searched between
  // slots i - 3 and i - 1; one barrier per iteration.  Staging buffer
  // (i + 1) & 1 and mask buffer (i + 1) & 1 are filled during iteration i.
  stage_plane(stg, z0 - 1);
  asm volatile("cp.async.commit_group;\n" ::);
  const int W = hi - nb, nxc = (W + 31) / 32, nchunk = yi * nxc;
  for (int i = 0; i <= NP; i++) {
    asm volatile("cp.async.wait_all;\n" ::);
    __syncthreads();
    if (i + 1 < NP) stage_plane(stg + ((i + 1) & 1) * nh * kXpPad, z0 + i);
    if (i + 1 >= 3 && i + 1 <= NP) stage_mask(mbuf + ((i + 1) & 1) * kXpInner * n, z0 - 2 + i);
    asm volatile("cp.async.commit_group;\n" ::);
    if (i < NP && warp < R) {
      float2 x[J], xh;
      row_load<J>(stg + (i & 1) * nh * kXpPad, warp, l, x, xh);
      row_irfft<J>(c, l, x, xh, ring + (i & 3) * kXpRows * n + warp * n);
    }
    if (i < 3) continue;
    const int z = z0 - 3 + i;
    const float* s0 = ring + ((i - 3) & 3) * kXpRows * n;
    const float* s1 = ring + ((i - 2) & 3) * kXpRows * n;
    const float* s2 = ring + ((i - 1) & 3) * kXpRows * n;
    const uint8_t* mk = mbuf + (i & 1) * kXpInner * n;
    // chunks of 32 cells of one row, spread over all warps
    for (int ch = warp; ch < nchunk; ch += kXpThreads / 32) {
      const int ri = 1 + ch / nxc;
      const int x = nb + 32 * (ch % nxc) + l;
      const int y = y0 - 1 + ri;
      bool peak = false;
      float f = 0.f;
      if (x < hi) {
        f = s1[ri * n + x];
        if (!(f < a.fcrit) && mk[(ri - 1) * n + x] != 1) {
          peak = true;
          for (int q = 0; q < 9; q++) {
            const int o = (ri + q / 3 - 1) * n + x + q % 3 - 1;
            if (f < s0[o] || f < s1[o] || f < s2[o]) { peak = false; break; }
          }
        }
      }
      const unsigned ball = __ballot_sync(full, peak);
      if (ball == 0) continue;
      if (peak) {
        const long long loc = x + (long long)n * y + nn * z;
        const int e = wn + __popc(ball & ((1u << l) - 1u));
        a.mask[loc] = 1;
        myloc[e] = loc;
        myf[e] = f;
      }
      wn += __popc(ball);
      if (wn > kXpList - 32) flush();
    }
  }
  if (wn > 0) flush();
}

// the k^2-weighted twin at the peaks one xpeak launch appended (slots
// first .. count - 1): sum over kx of c_k Re(L[kx] w^(kx x)), c = 1 at kx = 0
// and n/2, else 2, over the z/y-transformed twin in [kx][z][y] order; one warp
// per peak
__global__ void __launch_bounds__(256) lapsum_kernel(const float2* __restrict__ ls, const float2* __restrict__ tw,
                                                    int n, const unsigned* __restrict__ first, PeakBuf pb) {
  const unsigned f0 = *first;
  if (f0 == 0xffffffffu) return;
  const int end = (int)min((int64_t)*pb.count, pb.cap);
  const int l = threadIdx.x & 31;
  const int nw = gridDim.x * (blockDim.x / 32);
  const int H = n / 2;
  const int64_t nn = (int64_t)n * n;
  for (int p = (int)f0 + blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); p < end; p += nw) {
    const long long loc = (long long)(pb.keys[p] & ((1ull << 40) - 1));
    const int x = (int)(loc % n), y = (int)((loc / n) % n);
    const long long z = loc / nn;
    const float2* col = ls + n * z + y;
    double acc = 0.0;
#pragma unroll 4
    for (int k = l; k <= H; k += 32) {
      const float2 v = __ldg(col + nn * k);
      const float2 t = __ldg(tw + (int)(((long long)k * x) % n));
      const double term = (double)v.x * t.x - (double)v.y * t.y;
      acc += (k == 0 || k == H) ? term : 2.0 * term;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (l == 0) pb.lap[p] = (float)acc;
  }
}

// tw[k] = exp(2 pi i k / n) in float, from FP64 sincospi
__global__ void twiddle_kernel(float2* tw, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double s, c;
  sincospi(2.0 * k / n, &s, &c);
  tw[k] = make_float2((float)c, (float)s);
}

// window multiply of the filter bank (window_kernel's arithmetic) writing
// the outputs transposed to [kx][kz][ky]: 32 x 32 (ky, kx) tiles of one kz
// plane through shared memory, both sides in 256-byte rows
__global__ void __launch_bounds__(256) window_t_kernel(const float2* __restrict__ dk, float2* __restrict__ out0,
                                                      float2* __restrict__ out1, int n,
                                                      const float* __restrict__ tab, float ps) {
  __shared__ float2 t0[32][33], t1[32][33];
  const int nh = n / 2 + 1, nyq = n / 2;
  const int kx0 = blockIdx.x * 32, ky0 = blockIdx.y * 32, kz = blockIdx.z;
  const int fz = kz <= nyq ? kz : kz - n;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int kx = kx0 + tx;
  if (kx < nh) {
    // the four loads and table lookups of this thread in flight together
    float2 d[4], w[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int ky = ky0 + ty + 8 * u;
      const int fy = ky <= nyq ? ky : ky - n;
      d[u] = __ldg(dk + ((int64_t)kz * n + ky) * nh + kx);
      w[u] = __ldg(reinterpret_cast<const float2*>(tab) + (kx * kx + fy * fy + fz * fz));
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int r = ty + 8 * u;
      t0[r][tx] = make_float2(__fmul_rn(__fmul_rn(d[u].x, w[u].x), ps), __fmul_rn(__fmul_rn(d[u].y, w[u].x), ps));
      if (out1)
        t1[r][tx] = make_float2(__fmul_rn(__fmul_rn(d[u].x, w[u].y), ps), __fmul_rn(__fmul_rn(d[u].y, w[u].y), ps));
    }
  }
  __syncthreads();
#pragma unroll
  for (int cx = ty; cx < 32; cx += 8) {
    const int k = kx0 + cx;
    if (k >= nh) break;
    const int64_t o = ((int64_t)k * n + kz) * n + ky0 + tx;
    out0[o] = t0[tx][cx];
    if (out1) out1[o] = t1[tx][cx];
  }
}

template <int J>
constexpr size_t xpeak_smem() {
  return (size_t)4 * kXpRows * 64 * J * 4 + (size_t)16 * kXpList * 12 + (size_t)2 * (32 * J + 1) * kXpPad * 8 +
         (size_t)2 * kXpInner * 64 * J;
}

template <int J>
void prepare_j() {
  PPB_CUDA(cudaFuncSetAttribute(xpeak_kernel<J>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xpeak_smem<J>()));
}

template <int J>
void launch_j(Launch L, const XpArgs& a0) {
  constexpr int n = 64 * J;
  const size_t smem = xpeak_smem<J>();
  XpArgs a = a0;
  const int w = n - 2 * a.nbuff;
  const int gx = (w + kXpInner - 1) / kXpInner;
  // one wave of one block per SM: z chunks of at least 4 planes
  int gz = std::max(1, 148 / gx);
  int tz = std::max(4, (w + gz - 1) / gz);
  tz = std::min(tz, w);
  gz = (w + tz - 1) / tz;
  a.tz = tz;
  xpeak_kernel<J><<<dim3((unsigned)gx, (unsigned)gz), kXpThreads, smem, L.s>>>(a);
  PPB_LAUNCHED(*L.count);
}

}  // namespace

bool xpeak_supported(int n, int nbuff) {
  return n % 64 == 0 && n >= 64 && n <= 512 && nbuff >= 1 && n - 2 * nbuff >= 1;
}

void launch_window_t(Launch L, const float2* dk, float2* out0, float2* out1, int n, const float* tab,
                     double post_scale) {
  const dim3 grid((unsigned)((n / 2 + 1 + 31) / 32), (unsigned)(n / 32), (unsigned)n);
  window_t_kernel<<<grid, dim3(32, 8), 0, L.s>>>(dk, out0, out1, n, tab, (float)post_scale);
  PPB_LAUNCHED(*L.count);
}

void launch_twiddles(Launch L, float2* tw, int n) {
  twiddle_kernel<<<(n + 127) / 128, 128, 0, L.s>>>(tw, n);
  PPB_LAUNCHED(*L.count);
}

void launch_xpeak(Launch L, const float2* ds, const float2* ls, const float2* tw, uint8_t* mask, unsigned* first,
                  int n, int nbuff, float fcrit, unsigned long long keyhi, PeakBuf pb) {
  PPB_CUDA(cudaMemsetAsync(first, 0xff, sizeof(unsigned), L.s));
  XpArgs a{ds, tw, mask, first, n, nbuff, 0, ls ? 0 : 1, fcrit, keyhi, pb};
  switch (n / 64) {
    case 1: launch_j<1>(L, a); break;
    case 2: launch_j<2>(L, a); break;
    case 3: launch_j<3>(L, a); break;
    case 4: launch_j<4>(L, a); break;
    case 5: launch_j<5>(L, a); break;
    case 6: launch_j<6>(L, a); break;
    case 7: launch_j<7>(L, a); break;
    case 8: launch_j<8>(L, a); break;
    default: PPB_REQUIRE(false, "fused x pass: unsupported grid size");
  }
  if (ls) {
    lapsum_kernel<<<148 * 4, 256, 0, L.s>>>(ls, tw, n, first, pb);
    PPB_LAUNCHED(*L.count);
  }
}

// the dynamic shared memory opt-in of the kernel for grid size n on the
// current device; called outside stream capture
void xpeak_prepare(int n) {
  switch (n / 64) {
    case 1: prepare_j<1>(); break;
    case 2: prepare_j<2>(); break;
    case 3: prepare_j<3>(); break;
    case 4: prepare_j<4>(); break;
    case 5: prepare_j<5>(); break;
    case 6: prepare_j<6>(); break;
    case 7: prepare_j<7>(); break;
    case 8: prepare_j<8>(); break;
    default: break;
  }
}

}  // namespace ppb
