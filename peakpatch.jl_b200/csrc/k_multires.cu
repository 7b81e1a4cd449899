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

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int64_t mod0(int64_t i, int64_t n) {
  const int64_t r = i % n;
  return r < 0 ? r + n : r;
}

// ---------------------------------------------------------------------------
// _downsample_noise (src/MultiResolution.jl:68-89): coarse cell (I, J, K)
// sums the Float64 deviates of its block^3 fine cells in the order dk, dj, di
// (di fastest).  One warp per coarse cell: the lanes evaluate 64 consecutive
// cells of that order (two per lane, one Threefry call when the two form a
// pair) and every lane adds the 64 values in order, so the sum is the
// sequential one bit for bit.
// ---------------------------------------------------------------------------
__global__ void coarse_noise_kernel(float* __restrict__ out, int64_t N, int M, int block, uint64_t seed,
                                    double denom) {
  const int lane = threadIdx.x & 31;
  const int64_t cell = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t M3 = (int64_t)M * M * M;
  if (cell >= M3) return;   // uniform over the warp
  const int64_t I = cell % M, J = (cell / M) % M, K = cell / ((int64_t)M * M);
  const int total = block * block * block;
  const int64_t gi0 = I * block, gj0 = J * block, gk0 = K * block;
  double val = 0.0;
  for (int base = 0; base < total; base += 64) {
    const int t0 = base + 2 * lane;
    double v0 = 0.0, v1 = 0.0;
    if (t0 < total) {
      const int di = t0 % block, dj = (t0 / block) % block, dk = t0 / (block * block);
      const uint64_t l0 = (uint64_t)((gi0 + di) + N * ((gj0 + dj) + N * (gk0 + dk)));
      if (t0 + 1 < total) {
        const int t1 = t0 + 1;
        const int ei = t1 % block, ej = (t1 / block) % block, ek = t1 / (block * block);
        const uint64_t l1 = (uint64_t)((gi0 + ei) + N * ((gj0 + ej) + N * (gk0 + ek)));
        if ((l0 & 1ull) == 0 && l1 == l0 + 1) {
          ppbm::threefry_gaussian_pair(seed, l0 >> 1, &v0, &v1);
        } else {
          v0 = ppbm::noise_cell_d(seed, l0);
          v1 = ppbm::noise_cell_d(seed, l1);
        }
      } else {
        v0 = ppbm::noise_cell_d(seed, l0);
      }
    }
    const int cnt = min(64, total - base);
#pragma unroll 8
    for (int j = 0; j < 32; j++) {
      const double a = __shfl_sync(kFull, v0, j), b = __shfl_sync(kFull, v1, j);
      if (2 * j < cnt) val = __dadd_rn(val, a);
      if (2 * j + 1 < cnt) val = __dadd_rn(val, b);
    }
  }
  if (lane == 0) out[cell] = (float)__ddiv_rn(val, denom);
}

// ---------------------------------------------------------------------------
// _generate_extended_residual (src/MultiResolution.jl:197-236): Float32 fine
// noise minus its coarse cell's value times 1/sqrt(block^3), on the
// (nmesh + 2 nshell)^3 region whose 0-based global origin is (i0, j0, k0),
// periodic in N.  A thread takes two x-neighbours (one Threefry call when
// they form a pair).
// ---------------------------------------------------------------------------
__global__ void residual_kernel(const float* __restrict__ coarse, float* __restrict__ out, int M, int block,
                                int64_t N, int64_t i0, int64_t j0, int64_t k0, int next, uint64_t seed, float inv) {
  const int li = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int lj = blockIdx.y, lk = blockIdx.z;
  if (li >= next) return;
  const int64_t gj = mod0(j0 + lj, N), gk = mod0(k0 + lk, N);
  const int64_t gi = mod0(i0 + li, N);
  const int64_t row = N * (gj + N * gk);
  const int64_t cj = gj / block, ck = gk / block;
  const int64_t o = li + (int64_t)next * (lj + (int64_t)next * lk);
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
// in-place real-to-complex transform)
// ---------------------------------------------------------------------------
__global__ void pad_kernel(const float* __restrict__ in, float* __restrict__ out, int nin, int n2, int64_t px) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y, z = blockIdx.z;
  if (x >= n2) return;
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
// inverse transform) times the kernel is formed in Float64 and the product
// rounded once to Float32.  `out` must not overlap `in`.
//
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
                                       double kz, double k2) {
  const double a = (double)v.x, b = (double)v.y;
  const double ka = d1 == 1 ? kx : d1 == 2 ? ky : kz;
  const double kb = d2 == 1 ? kx : d2 == 2 ? ky : kz;
  float re, im;
  switch (kind) {
    case 0: re = (float)(a * amp); im = (float)(b * amp); break;
    case 1: { const double c = amp * (ka / k2); re = (float)(-b * c); im = (float)(a * c); break; }
    case 2: { const double c = amp * (-ka / k2); re = (float)(-b * c); im = (float)(a * c); break; }
    case 3: { const double c = amp * (-ka * kb / k2); re = (float)(a * c); im = (float)(b * c); break; }
    default: { const double c = amp * k2; re = (float)(a * c); im = (float)(b * c); break; }
  }
  return make_float2(re, im);
}

template <bool TRANSFER>
__device__ __forceinline__ void kmode(const float2* __restrict__ in, int n, int nh, int ix, int iy, int iz,
                                      double mult, double dk3n3, const double* __restrict__ lk,
                                      const double* __restrict__ lp, int np, const KSpecs& sp, double post,
                                      float2* t) {
  const float2 v = __ldg(in + ix + (int64_t)nh * (iy + (int64_t)n * iz));
  const double kx = (double)ix * mult, ky = ks::fftfreq(iy, n, mult), kz = ks::fftfreq(iz, n, mult);
  const double k2 = kx * kx + ky * ky + kz * kz;
  bool zero = k2 == 0.0;
  if (!TRANSFER) zero = zero || ix == nh - 1 || iy == n / 2 || iz == n / 2;
  if (zero) {
#pragma unroll
    for (int s = 0; s < kMaxKSpecs; s++) t[s] = make_float2(0.f, 0.f);
    return;
  }
  const double amp = TRANSFER ? sqrt(ks::pk_eval(lk, lp, np, sqrt(k2)) * dk3n3) * post : post;
#pragma unroll
  for (int s = 0; s < kMaxKSpecs; s++)
    if (s < sp.n) t[s] = kmul(v, amp, sp.kind[s], sp.d1[s], sp.d2[s], kx, ky, kz, k2);
}

template <bool TRANSFER>
__global__ void __launch_bounds__(256) kspace_kernel(const float2* __restrict__ in, float2* __restrict__ out,
                                                     int64_t odist, int n, double mult, double dk3n3,
                                                     const double* __restrict__ lk, const double* __restrict__ lp,
                                                     int np, KSpecs sp, double post) {
  const int nh = n / 2 + 1;
  const int64_t plane = (int64_t)nh * n;
  const int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (id >= plane * n) return;
  const int iz = (int)(id / plane);
  const int r = (int)(id - (int64_t)iz * plane);
  const int iy = r / nh, ix = r - iy * nh;
  float2 t[kMaxKSpecs];
  kmode<TRANSFER>(in, n, nh, ix, iy, iz, mult, dk3n3, lk, lp, np, sp, post, t);
  if (ix == 0 || (n % 2 == 0 && ix == n / 2)) {
    const int jy = (n - iy) % n, jz = (n - iz) % n;
    if (jy == iy && jz == iz) {
#pragma unroll
      for (int s = 0; s < kMaxKSpecs; s++) t[s].y = 0.f;
    } else {
      float2 u[kMaxKSpecs];
      kmode<TRANSFER>(in, n, nh, ix, jy, jz, mult, dk3n3, lk, lp, np, sp, post, u);
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

// out = val, or base + val (the combined field delta_self .+ delta_long of
// :779-795; base may be out itself)
__global__ void tricubic_kernel(const float* __restrict__ coarse, float* out, const float* base, int M, int block,
                                int64_t N, int64_t i0, int64_t j0, int64_t k0, int n) {
  const int li = blockIdx.x * blockDim.x + threadIdx.x;
  const int lj = blockIdx.y, lk = blockIdx.z;
  if (li >= n) return;
  const int64_t g[3] = {mod0(i0 + li, N) + 1, mod0(j0 + lj, N) + 1, mod0(k0 + lk, N) + 1};
  int ic[3];
  float w[3][4];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double f = __dadd_rn(__ddiv_rn(__dsub_rn((double)g[d], 0.5), (double)block), 0.5);
    const double fl = floor(f);
    ic[d] = (int)fl;
    catmull_rom((float)__dsub_rn(f, fl), w[d]);
  }
  float val = 0.0f;
  for (int a = 0; a < 4; a++) {
    const int kk = (int)mod0(ic[2] - 2 + a, M);
    for (int b = 0; b < 4; b++) {
      const int jj = (int)mod0(ic[1] - 2 + b, M);
      const float* row = coarse + (int64_t)M * (jj + (int64_t)M * kk);
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const int ii = (int)mod0(ic[0] - 2 + c, M);
        // ((wi * wj) * wk) * field, as Julia evaluates wi * wj * wk * f
        const float term = __fmul_rn(__fmul_rn(__fmul_rn(w[0][c], w[1][b]), w[2][a]), __ldg(row + ii));
        val = __fadd_rn(val, term);
      }
    }
  }
  const int64_t o = li + (int64_t)n * (lj + (int64_t)n * lk);
  out[o] = base ? __fadd_rn(base[o], val) : val;
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
void launch_coarse_noise(Launch L, float* out, int64_t N, int M, uint64_t seed) {
  const int block = (int)(N / M);
  const double b = (double)block;
  const double denom = std::sqrt(b * b * b);
  const int64_t warps = (int64_t)M * M * M;
  const int threads = 128;
  const int64_t blocks = (warps * 32 + threads - 1) / threads;
  coarse_noise_kernel<<<(unsigned)blocks, threads, 0, L.s>>>(out, N, M, block, seed, denom);
  PPB_LAUNCHED(*L.count);
}

void launch_residual(Launch L, const float* coarse, float* out, int M, int64_t N, int64_t i0, int64_t j0, int64_t k0,
                     int next, uint64_t seed) {
  const int block = (int)(N / M);
  const double b = (double)block;
  const float inv = (float)(1.0 / std::sqrt(b * b * b));
  const int pairs = (next + 1) / 2;
  dim3 grid((unsigned)((pairs + 127) / 128), (unsigned)next, (unsigned)next);
  residual_kernel<<<grid, 128, 0, L.s>>>(coarse, out, M, block, N, i0, j0, k0, next, seed, inv);
  PPB_LAUNCHED(*L.count);
}

void launch_pad(Launch L, const float* in, float* out, int nin, int n2, int64_t px) {
  dim3 grid((unsigned)((n2 + 127) / 128), (unsigned)n2, (unsigned)n2);
  pad_kernel<<<grid, 128, 0, L.s>>>(in, out, nin, n2, px);
  PPB_LAUNCHED(*L.count);
}

void launch_kspace(Launch L, bool transfer, const float2* in, float2* out, int64_t odist, int n, double box,
                   const double* lk, const double* lp, int np, const int* kind, const int* d1, const int* d2,
                   int nspec, double post) {
  if (nspec < 1 || nspec > kMaxKSpecs) throw Error{PPB_ERR_INVALID, "kspace: 1..8 kernels per launch"};
  KSpecs sp{};
  sp.n = nspec;
  for (int s = 0; s < nspec; s++) {
    sp.kind[s] = kind[s];
    sp.d1[s] = d1[s];
    sp.d2[s] = d2[s];
  }
  const double dk = 2.0 * 3.141592653589793 / box;
  const double mult = ((double)n * dk) / (double)n;
  const double nd = (double)n;
  const double dk3n3 = (dk * dk * dk) * (nd * nd * nd);
  const int64_t modes = (int64_t)(n / 2 + 1) * n * n;
  const unsigned blocks = (unsigned)((modes + 255) / 256);
  if (transfer)
    kspace_kernel<true><<<blocks, 256, 0, L.s>>>(in, out, odist, n, mult, dk3n3, lk, lp, np, sp, post);
  else
    kspace_kernel<false><<<blocks, 256, 0, L.s>>>(in, out, odist, n, mult, dk3n3, lk, lp, np, sp, post);
  PPB_LAUNCHED(*L.count);
}

void launch_src2_trace(Launch L, const float* delta, const float* phi, float* out, int n, int64_t px, int64_t pz,
                       int64_t pd) {
  dim3 grid((unsigned)((n + 127) / 128), (unsigned)n, (unsigned)n);
  src2_kernel<<<grid, 128, 0, L.s>>>(delta, phi, out, n, px, pz, pd);
  PPB_LAUNCHED(*L.count);
}

void launch_tricubic(Launch L, const float* coarse, float* out, int M, int64_t N, int64_t i0, int64_t j0, int64_t k0,
                     int n, const float* base) {
  const int block = (int)(N / M);
  dim3 grid((unsigned)((n + 127) / 128), (unsigned)n, (unsigned)n);
  tricubic_kernel<<<grid, 128, 0, L.s>>>(coarse, out, base, M, block, N, i0, j0, k0, n);
  PPB_LAUNCHED(*L.count);
}

}  // namespace ppb
