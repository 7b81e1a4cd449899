// k_multires.cu — kernels of the multi-resolution (MUSIC-style) tile fields
// of run_multitile_split (src/MultiResolution.jl): the coarse block-mean
// noise, the Hoffman–Ribak residual, the zero-padded isolated convolution
// (pad, transfer with the Hermitian projection of the ix = 0 and Nyquist
// planes fused in), the tile-local periodic kernels of _apply_kernel_inplace!,
// the 2LPT source by the trace identity and the Catmull-Rom tricubic
// interpolation of coarse fields.
//
// Compiled with -fmad=false: every float and double expression rounds the way
// the reference's Julia code does (nothing is contracted into an FMA), so
// the noise, residual, source and interpolation kernels reproduce the
// reference bit for bit on the same inputs.
//
// Layouts as in the tile pipeline: real fields n^3 floats [k][j][i] (Julia
// [i,j,k]); half-spectra (n/2+1) x n x n float2 with ix fastest.
#include "ppb_internal.h"
#include "ppb_kspace.cuh"
#include "ppb_math.h"

namespace ppb {

namespace {


__device__ __forceinline__ int64_t mod0(int64_t i, int64_t n) {
  const int64_t r = i % n;
  return r < 0 ? r + n : r;
}

// ---------------------------------------------------------------------------
// _downsample_noise (src/MultiResolution.jl:68-89): coarse cell (I, J, K)
// sums the Float64 deviates of its block^3 fine cells in the order dk, dj, di
// (di fastest).  One block per coarse cell: per chunk, warps 1..7 evaluate
// 1792 consecutive cells of that order into shared memory (eight per lane as
// four Threefry pairs) while thread 0 adds the previous chunk's values in
// order, so the sum is the sequential one bit for bit and the addition chain
// is the only serial part.
// ---------------------------------------------------------------------------
constexpr int kNoiseThreads = 256;
constexpr int kNoiseGenWarps = kNoiseThreads / 32 - 1;
constexpr int kNoisePer = 8;                                   // cells per generating lane
constexpr int kNoiseChunk = kNoiseGenWarps * 32 * kNoisePer;   // 1792 cells

__device__ __forceinline__ uint64_t block_cell_lin(int t, int block, int64_t gi0, int64_t gj0, int64_t gk0, int64_t N) {
  const int di = t % block, dj = (t / block) % block, dk = t / (block * block);
  return (uint64_t)((gi0 + di) + N * ((gj0 + dj) + N * (gk0 + dk)));
}

__global__ void __launch_bounds__(kNoiseThreads) coarse_noise_kernel(float* __restrict__ out, int64_t N, int M,
                                                                       int block, uint64_t seed, double denom) {
  __shared__ double buf[2][kNoiseChunk];
  const int64_t cell = blockIdx.x;
  const int64_t I = cell % M, J = (cell / M) % M, K = cell / ((int64_t)M * M);
  const int total = block * block * block;
  const int64_t gi0 = I * block, gj0 = J * block, gk0 = K * block;
  const int nchunk = (total + kNoiseChunk - 1) / kNoiseChunk;
  const int warp = threadIdx.x >> 5;
  double val = 0.0;
  for (int c = 0; c <= nchunk; c++) {
    if (warp > 0 && c < nchunk) {   // generate chunk c
      double* dst = buf[c & 1] + ((warp - 1) * 32 + (threadIdx.x & 31)) * kNoisePer;
      const int tb = c * kNoiseChunk + ((warp - 1) * 32 + (threadIdx.x & 31)) * kNoisePer;
#pragma unroll
      for (int q = 0; q < kNoisePer; q += 2) {
        const int t0 = tb + q;
        double a = 0.0, b = 0.0;
        if (t0 < total) {
          const uint64_t l0 = block_cell_lin(t0, block, gi0, gj0, gk0, N);
          if (t0 + 1 < total) {
            const uint64_t l1 = block_cell_lin(t0 + 1, block, gi0, gj0, gk0, N);
            if ((l0 & 1ull) == 0 && l1 == l0 + 1) {
              ppbm::threefry_gaussian_pair(seed, l0 >> 1, &a, &b);
            } else {
              a = ppbm::noise_cell_d(seed, l0);
              b = ppbm::noise_cell_d(seed, l1);
            }
          } else {
            a = ppbm::noise_cell_d(seed, l0);
          }
        }
        dst[q] = a;
        dst[q + 1] = b;
      }
    }
    if (threadIdx.x == 0 && c > 0) {   // add chunk c - 1 in order
      const double* src = buf[(c - 1) & 1];
      const int cnt = min(kNoiseChunk, total - (c - 1) * kNoiseChunk);
      for (int i = 0; i < cnt; i++) val = __dadd_rn(val, src[i]);
    }
    // chunk c is written and chunk c - 1 consumed before buffer (c + 1) & 1
    // (= (c - 1) & 1) is written again
    __syncthreads();
  }
  if (threadIdx.x == 0) out[cell] = (float)__ddiv_rn(val, denom);
}

// ---------------------------------------------------------------------------
// _generate_extended_residual (src/MultiResolution.jl:197-236): Float32 fine
// noise minus its coarse cell's value times 1/sqrt(block^3), on the
// (nmesh + 2 nshell)^3 region whose 0-based global origin is (i0, j0, k0),
// periodic in N, written with row pitch opx and plane pitch opz (a dense
// array, or the corner of a zero-padded box).  A thread takes two
// x-neighbours (one Threefry call when they form a pair).
// ---------------------------------------------------------------------------
__global__ void residual_kernel(const float* __restrict__ coarse, float* __restrict__ out, int M, int block,
                                int64_t N, int64_t i0, int64_t j0, int64_t k0, int next, uint64_t seed, float inv,
                                int64_t opx, int64_t opz) {
  const int li = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int lj = blockIdx.y, lk = blockIdx.z;
  if (li >= next) return;
  const int64_t gj = mod0(j0 + lj, N), gk = mod0(k0 + lk, N);
  const int64_t gi = mod0(i0 + li, N);
  const int64_t row = N * (gj + N * gk);
  const int64_t cj = gj / block, ck = gk / block;
  const int64_t o = li + opx * lj + opz * lk;
  const uint64_t l0 = (uint64_t)(gi + row);
  if (li + 1 < next) {
    const int64_t gi1 = mod0(i0 + li + 1, N);
    const uint64_t l1 = (uint64_t)(gi1 + row);
    double g0, g1;
    if ((l0 & 1ull) == 0 && l1 == l0 + 1) {
      ppbm::threefry_gaussian_pair(seed, l0 >> 1, &g0, &g1);
    } else {
      g0 = ppbm::noise_cell_d(seed, l0);
      g1 = ppbm::noise_cell_d(seed, l1);
    }
    const float b0 = __fmul_rn(__ldg(coarse + gi / block + M * (cj + M * ck)), inv);
    const float b1 = __fmul_rn(__ldg(coarse + gi1 / block + M * (cj + M * ck)), inv);
    out[o] = __fsub_rn((float)g0, b0);
    out[o + 1] = __fsub_rn((float)g1, b1);
  } else {
    const float b0 = __fmul_rn(__ldg(coarse + gi / block + M * (cj + M * ck)), inv);
    out[o] = __fsub_rn((float)ppbm::noise_cell_d(seed, l0), b0);
  }
}

// ---------------------------------------------------------------------------
// zero padding of _isolated_convolve (:254-255): the n_in^3 input in the
// corner of an n2^3 box stored with row pitch `px` floats (the layout of an
// in-place real-to-complex transform).  The row padding is zeroed too: the
// pruned forward transform reads the planes it does not transform as
// complex data, whose last element per row is that padding.
// ---------------------------------------------------------------------------
__global__ void pad_kernel(const float* __restrict__ in, float* __restrict__ out, int nin, int n2, int64_t px) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y, z = blockIdx.z;
  if (x >= px) return;
  float v = 0.f;
  if (x < nin && y < nin && z < nin) v = __ldg(in + x + (int64_t)nin * (y + (int64_t)nin * z));
  out[x + px * (y + (int64_t)n2 * z)] = v;
}

// ---------------------------------------------------------------------------
// k-space multipliers.  TRANSFER: the loop of _isolated_convolve (:257-277)
// and of _periodic_convolve! (:286-309): v *= sqrt(P(k) dk^3 n^3) * kernel,
// DC := 0.  APPLY: _apply_kernel_inplace! (:1239-1255): v *= kernel, DC and
// the planes ix = n/2 + 1 - 1, iy = n/2, iz = n/2 (0-based) := 0.  Kernel
// kinds (the reference's kernel_fn ids): 0 none, 1 i k_d1/k^2, 2 -i k_d1/k^2,
// 3 -k_d1 k_d2/k^2, 4 k^2; the amplitude times `post` (the 1/n^3 of the
// inverse transform) times the kernel is formed in Float64 (1/k^2 taken once
// per mode) and the product rounded once to Float32.  `out` must not overlap
// `in`.
//
// The TRANSFER amplitude comes from a table over the integer |freq|^2
// (amp_table_kernel): one load per mode instead of a P(k) interpolation.
// One thread per mode, all kernels of `sp` from one read of the input.  On
// the ix = 0 plane and (even n) the ix = n/2 plane the thread also forms the
// mirror mode (-iy, -iz) and writes the Hermitian projection
// ((t + conj t_mirror) / 2) that the complex-to-real transform needs to agree
// with Julia's irfft (the reference's GPU path runs it as
// _hermitize_planes_kernel!, ext/CUDAExt.jl:2574-2611).
// ---------------------------------------------------------------------------
struct KSpecs {
  int n;
  int kind[kMaxKSpecs], d1[kMaxKSpecs], d2[kMaxKSpecs];
};

__device__ __forceinline__ float2 kmul(float2 v, double amp, int kind, int d1, int d2, double kx, double ky,
                                       double kz, double k2, double inv_k2) {
  const double a = (double)v.x, b = (double)v.y;
  const double ka = d1 == 1 ? kx : d1 == 2 ? ky : kz;
  const double kb = d2 == 1 ? kx : d2 == 2 ? ky : kz;
  float re, im;
  switch (kind) {
    case 0: re = (float)(a * amp); im = (float)(b * amp); break;
    case 1: { const double c = amp * (ka * inv_k2); re = (float)(-b * c); im = (float)(a * c); break; }
    case 2: { const double c = amp * (-ka * inv_k2); re = (float)(-b * c); im = (float)(a * c); break; }
    case 3: { const double c = amp * ((-ka * kb) * inv_k2); re = (float)(a * c); im = (float)(b * c); break; }
    default: { const double c = amp * k2; re = (float)(a * c); im = (float)(b * c); break; }
  }
  return make_float2(re, im);
}

__device__ __forceinline__ int ifreq(int idx, int n) { return idx < (n + 1) / 2 ? idx : idx - n; }

template <bool TRANSFER>
__device__ __forceinline__ void kmode(const float2* __restrict__ in, int n, int nh, int ix, int iy, int iz,
                                      double mult, const double* __restrict__ amp_tab, const KSpecs& sp, double post,
                                      float2* t) {
  const float2 v = __ldg(in + ix + (int64_t)nh * (iy + (int64_t)n * iz));
  const int fy = ifreq(iy, n), fz = ifreq(iz, n);
  const double kx = (double)ix * mult, ky = (double)fy * mult, kz = (double)fz * mult;
  const double k2 = kx * kx + ky * ky + kz * kz;
  bool zero = k2 == 0.0;
  if (!TRANSFER) zero = zero || ix == nh - 1 || iy == n / 2 || iz == n / 2;
  if (zero) {
#pragma unroll
    for (int s = 0; s < kMaxKSpecs; s++) t[s] = make_float2(0.f, 0.f);
    return;
  }
  const double amp = TRANSFER ? __ldg(amp_tab + (ix * ix + fy * fy + fz * fz)) : post;
  const double inv_k2 = 1.0 / k2;   // one division per mode (k_a / k^2 as k_a * (1 / k^2))
#pragma unroll
  for (int s = 0; s < kMaxKSpecs; s++)
    if (s < sp.n) t[s] = kmul(v, amp, sp.kind[s], sp.d1[s], sp.d2[s], kx, ky, kz, k2, inv_k2);
}

template <bool TRANSFER>
__global__ void __launch_bounds__(256) kspace_kernel(const float2* __restrict__ in, float2* __restrict__ out,
                                                     int64_t odist, int n, double mult,
                                                     const double* __restrict__ amp_tab, KSpecs sp, double post) {
  const int nh = n / 2 + 1;
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z;
  if (ix >= nh || iy >= n) return;
  const int64_t id = ix + (int64_t)nh * (iy + (int64_t)n * iz);
  float2 t[kMaxKSpecs];
  kmode<TRANSFER>(in, n, nh, ix, iy, iz, mult, amp_tab, sp, post, t);
  if (ix == 0 || (n % 2 == 0 && ix == n / 2)) {
    const int jy = (n - iy) % n, jz = (n - iz) % n;
    if (jy == iy && jz == iz) {
#pragma unroll
      for (int s = 0; s < kMaxKSpecs; s++) t[s].y = 0.f;
    } else {
      float2 u[kMaxKSpecs];
      kmode<TRANSFER>(in, n, nh, ix, jy, jz, mult, amp_tab, sp, post, u);
#pragma unroll
      for (int s = 0; s < kMaxKSpecs; s++) t[s] = make_float2(0.5f * (t[s].x + u[s].x), 0.5f * (t[s].y - u[s].y));
    }
  }
#pragma unroll
  for (int s = 0; s < kMaxKSpecs; s++)
    if (s < sp.n) out[id + s * odist] = t[s];
}

// ---------------------------------------------------------------------------
// 2LPT source of run_multitile_split (:810-821):
// src2 = d^2/2 - sum_a phi_aa^2/2 - sum_{a<b} phi_ab^2, each step rounded to
// Float32 in the reference's order; phi holds phi_11, phi_22, phi_33,
// phi_12, phi_13, phi_23 at pitch `pd` floats (row pitch px, plane pitch pz).
// out may alias the first phi field (each element is read before written).
// ---------------------------------------------------------------------------
__global__ void src2_kernel(const float* __restrict__ delta, const float* phi, float* out, int n, int64_t px,
                            int64_t pz, int64_t pd) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y, z = blockIdx.z;
  if (x >= n) return;
  const int64_t q = x + px * y + pz * z;
  const float d = delta[x + (int64_t)n * (y + (int64_t)n * z)];
  const float h = 0.5f;
  float s = __fmul_rn(__fmul_rn(d, d), h);
  for (int a = 0; a < 3; a++) {
    const float p = phi[q + a * pd];
    s = __fsub_rn(s, __fmul_rn(__fmul_rn(p, p), h));
  }
  for (int a = 3; a < 6; a++) {
    const float p = phi[q + a * pd];
    s = __fsub_rn(s, __fmul_rn(p, p));
  }
  out[q] = s;
}

// ---------------------------------------------------------------------------
// _interpolate_to_tile / _tricubic / _catmull_rom (src/MultiResolution.jl:
// 95-122, 156-189): Catmull-Rom tricubic interpolation of the periodic M^3
// coarse field at the tile's fine cells.  0-based global origin (i0, j0, k0).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void catmull_rom(float t, float* w) {
  const float t2 = __fmul_rn(t, t), t3 = __fmul_rn(t2, t);
  w[0] = __fsub_rn(__fadd_rn(__fmul_rn(-0.5f, t3), t2), __fmul_rn(0.5f, t));
  w[1] = __fadd_rn(__fsub_rn(__fmul_rn(1.5f, t3), __fmul_rn(2.5f, t2)), 1.0f);
  w[2] = __fadd_rn(__fadd_rn(__fmul_rn(-1.5f, t3), __fmul_rn(2.0f, t2)), __fmul_rn(0.5f, t));
  w[3] = __fsub_rn(__fmul_rn(0.5f, t3), __fmul_rn(0.5f, t2));
}

// Per axis d and tile coordinate l (3n entries, d major): the four wrapped
// coarse indices and Catmull-Rom weights of _tricubic for the fine cell at
// global (1-based) g = mod1(o_d + l + 1, N): f = (g - 0.5)/block + 0.5 in
// Float64, ix = floor(f), t = Float32(f - ix).  The weights of a cell are the
// product of its three axes' entries, so the per-cell work is only the
// 64-term sum.
__global__ void axis_weights_kernel(int4* __restrict__ idx, float4* __restrict__ wt, int M, int block, int64_t N,
                                    int64_t o0, int64_t o1, int64_t o2, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * n) return;
  const int d = t / n, l = t - d * n;
  const int64_t o = d == 0 ? o0 : d == 1 ? o1 : o2;
  const int64_t g = mod0(o + l, N) + 1;
  const double f = __dadd_rn(__ddiv_rn(__dsub_rn((double)g, 0.5), (double)block), 0.5);
  const double fl = floor(f);
  const int64_t ic = (int64_t)fl;
  float w[4];
  catmull_rom((float)__dsub_rn(f, fl), w);
  idx[t] = make_int4((int)mod0(ic - 2, M), (int)mod0(ic - 1, M), (int)mod0(ic, M), (int)mod0(ic + 1, M));
  wt[t] = make_float4(w[0], w[1], w[2], w[3]);
}

__device__ __forceinline__ int comp(const int4& v, int c) { return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w; }
__device__ __forceinline__ float comp(const float4& v, int c) {
  return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
}

// _interpolate_to_tile / _tricubic / _catmull_rom (src/MultiResolution.jl:
// 95-122, 156-189): the 64-term Catmull-Rom sum over the periodic M^3 coarse
// field, terms ((wi * wj) * wk) * field added in the reference's order
// (dkk outer, dii inner), for NF fields sharing one set of weights (NF = 4:
// the fields interleaved as float4, one load per term).  Field f of cell
// (li, lj, lk) goes to out[f][li + n lj + n^2 lk] as val, or as base[f] + val
// when base is given (the combined field delta_self .+ delta_long of
// :779-795); base[f] is read at bofs + li + bpy lj + bpz lk, so it may be a
// zero-padded transform's output.
template <int NF>
struct TriArgs {
  const float* coarse;     // NF == 1: the field; NF == 4: float4-interleaved fields
  float* out[NF];
  const float* base[NF];
  int64_t bofs, bpy, bpz;
};

template <int NF>
__device__ __forceinline__ void tri_load(const float* c, int q, float* v) {
  if (NF == 1) {
    v[0] = __ldg(c + q);
  } else {
    const float4 t = __ldg(reinterpret_cast<const float4*>(c) + q);
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
  }
}

template <int NF>
__global__ void __launch_bounds__(128) tricubic_kernel(TriArgs<NF> A, const int4* __restrict__ aidx,
                                                       const float4* __restrict__ awt, int M, int n) {
  const int li = blockIdx.x * blockDim.x + threadIdx.x;
  const int lj = blockIdx.y, lk = blockIdx.z;
  if (li >= n) return;
  const int4 ix = __ldg(aidx + li), iy = __ldg(aidx + n + lj), iz = __ldg(aidx + 2 * n + lk);
  const float4 wx = __ldg(awt + li), wy = __ldg(awt + n + lj), wz = __ldg(awt + 2 * n + lk);
  // wi * wj for every (dii, djj): the first product of ((wi * wj) * wk) * f
  float wij[4][4];
#pragma unroll
  for (int b = 0; b < 4; b++)
#pragma unroll
    for (int c = 0; c < 4; c++) wij[b][c] = __fmul_rn(comp(wx, c), comp(wy, b));
  float val[NF];
#pragma unroll
  for (int f = 0; f < NF; f++) val[f] = 0.0f;
#pragma unroll
  for (int a = 0; a < 4; a++) {
    const int kk = comp(iz, a);
    const float wk = comp(wz, a);
#pragma unroll
    for (int b = 0; b < 4; b++) {
      const int row = M * (comp(iy, b) + M * kk);
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const float w3 = __fmul_rn(wij[b][c], wk);
        float v[NF];
        tri_load<NF>(A.coarse, row + comp(ix, c), v);
#pragma unroll
        for (int f = 0; f < NF; f++) val[f] = __fadd_rn(val[f], __fmul_rn(w3, v[f]));
      }
    }
  }
  const int64_t o = li + (int64_t)n * (lj + (int64_t)n * lk);
  const int64_t ob = A.bofs + li + A.bpy * lj + A.bpz * lk;
#pragma unroll
  for (int f = 0; f < NF; f++) A.out[f][o] = A.base[f] ? __fadd_rn(A.base[f][ob], val[f]) : val[f];
}

// four M^3 fields a apart interleaved as float4 (the tricubic input of the
// split's coarse delta and psi)
__global__ void interleave4_kernel(float4* __restrict__ dst, const float* __restrict__ src, int64_t fs, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  dst[i] = make_float4(src[i], src[fs + i], src[2 * fs + i], src[3 * fs + i]);
}

// the amplitude of the transfer multiply by integer |freq|^2 q on an n^3 box:
// tab[q] = sqrt(P(sqrt(q) dk) dk^3 n^3) * post (tab[0] = 0)
__global__ void amp_table_kernel(double* __restrict__ tab, int qmax, double mult, double dk3n3,
                                 const double* __restrict__ lk, const double* __restrict__ lp, int np, double post) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q > qmax) return;
  if (q == 0) {
    tab[0] = 0.0;
    return;
  }
  const double k2 = (double)q * (mult * mult);
  tab[q] = sqrt(ks::pk_eval(lk, lp, np, sqrt(k2)) * dk3n3) * post;
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
void launch_coarse_noise(Launch L, float* out, int64_t N, int M, uint64_t seed) {
  const int block = (int)(N / M);
  const double b = (double)block;
  const double denom = std::sqrt(b * b * b);
  const int64_t cells = (int64_t)M * M * M;
  coarse_noise_kernel<<<(unsigned)cells, kNoiseThreads, 0, L.s>>>(out, N, M, block, seed, denom);
  PPB_LAUNCHED(*L.count);
}

void launch_residual(Launch L, const float* coarse, float* out, int M, int64_t N, int64_t i0, int64_t j0, int64_t k0,
                     int next, uint64_t seed, int64_t opx, int64_t opz) {
  const int block = (int)(N / M);
  const double b = (double)block;
  const float inv = (float)(1.0 / std::sqrt(b * b * b));
  const int pairs = (next + 1) / 2;
  if (opx <= 0) opx = next;
  if (opz <= 0) opz = (int64_t)next * next;
  dim3 grid((unsigned)((pairs + 127) / 128), (unsigned)next, (unsigned)next);
  residual_kernel<<<grid, 128, 0, L.s>>>(coarse, out, M, block, N, i0, j0, k0, next, seed, inv, opx, opz);
  PPB_LAUNCHED(*L.count);
}

void launch_pad(Launch L, const float* in, float* out, int nin, int n2, int64_t px) {
  dim3 grid((unsigned)((px + 127) / 128), (unsigned)n2, (unsigned)n2);
  pad_kernel<<<grid, 128, 0, L.s>>>(in, out, nin, n2, px);
  PPB_LAUNCHED(*L.count);
}

int64_t amp_table_size(int n) { return 3 * (int64_t)(n / 2 + 1) * (n / 2 + 1) + 1; }

void launch_amp_table(Launch L, double* tab, int n, double box, const double* lk, const double* lp, int np,
                      double post) {
  const double dk = 2.0 * 3.141592653589793 / box;
  const double mult = ((double)n * dk) / (double)n;
  const double nd = (double)n;
  const double dk3n3 = (dk * dk * dk) * (nd * nd * nd);
  const int qmax = (int)(amp_table_size(n) - 1);
  amp_table_kernel<<<(qmax + 256) / 256, 256, 0, L.s>>>(tab, qmax, mult, dk3n3, lk, lp, np, post);
  PPB_LAUNCHED(*L.count);
}

void launch_kspace(Launch L, const double* amp_tab, const float2* in, float2* out, int64_t odist, int n, double box,
                   const int* kind, const int* d1, const int* d2, int nspec, double post) {
  if (nspec < 1 || nspec > kMaxKSpecs) throw Error{PPB_ERR_INVALID, "kspace: 1..6 kernels per launch"};
  KSpecs sp{};
  sp.n = nspec;
  for (int s = 0; s < nspec; s++) {
    sp.kind[s] = kind[s];
    sp.d1[s] = d1[s];
    sp.d2[s] = d2[s];
  }
  const double dk = 2.0 * 3.141592653589793 / box;
  const double mult = ((double)n * dk) / (double)n;
  // threads along ix (32 per warp), 8 rows of iy per block, one iz per grid z
  const dim3 block(32, 8);
  const dim3 grid((unsigned)((n / 2 + 1 + 31) / 32), (unsigned)((n + 7) / 8), (unsigned)n);
  if (amp_tab)
    kspace_kernel<true><<<grid, block, 0, L.s>>>(in, out, odist, n, mult, amp_tab, sp, post);
  else
    kspace_kernel<false><<<grid, block, 0, L.s>>>(in, out, odist, n, mult, nullptr, sp, post);
  PPB_LAUNCHED(*L.count);
}

void launch_src2_trace(Launch L, const float* delta, const float* phi, float* out, int n, int64_t px, int64_t pz,
                       int64_t pd) {
  dim3 grid((unsigned)((n + 127) / 128), (unsigned)n, (unsigned)n);
  src2_kernel<<<grid, 128, 0, L.s>>>(delta, phi, out, n, px, pz, pd);
  PPB_LAUNCHED(*L.count);
}

void launch_axis_weights(Launch L, int4* idx, float4* wt, int M, int64_t N, int64_t i0, int64_t j0, int64_t k0,
                         int n) {
  const int block = (int)(N / M);
  axis_weights_kernel<<<(3 * n + 127) / 128, 128, 0, L.s>>>(idx, wt, M, block, N, i0, j0, k0, n);
  PPB_LAUNCHED(*L.count);
}

void launch_tricubic(Launch L, const int4* idx, const float4* wt, int M, int n, int nf, const float* coarse,
                     float* const* out, const float* const* base, int64_t bofs, int64_t bpy, int64_t bpz) {
  dim3 grid((unsigned)((n + 127) / 128), (unsigned)n, (unsigned)n);
  if (nf == 1) {
    TriArgs<1> A{coarse, {out[0]}, {base ? base[0] : nullptr}, bofs, bpy, bpz};
    tricubic_kernel<1><<<grid, 128, 0, L.s>>>(A, idx, wt, M, n);
  } else if (nf == 4) {
    TriArgs<4> A{coarse,
                 {out[0], out[1], out[2], out[3]},
                 {base ? base[0] : nullptr, base ? base[1] : nullptr, base ? base[2] : nullptr,
                  base ? base[3] : nullptr},
                 bofs, bpy, bpz};
    tricubic_kernel<4><<<grid, 128, 0, L.s>>>(A, idx, wt, M, n);
  } else {
    throw Error{PPB_ERR_INVALID, "tricubic: 1 or 4 fields per launch"};
  }
  PPB_LAUNCHED(*L.count);
}

void launch_interleave4(Launch L, float4* dst, const float* src, int64_t fs, int64_t n) {
  interleave4_kernel<<<(unsigned)((n + 255) / 256), 256, 0, L.s>>>(dst, src, fs, n);
  PPB_LAUNCHED(*L.count);
}

}  // namespace ppb
