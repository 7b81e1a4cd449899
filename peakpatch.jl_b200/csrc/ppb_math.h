// ppb_math.h — Threefry-2x64-20 white noise with a Box–Muller transform,
// written once and compiled for both the host (gcc) and the device (nvcc).
//
// Reference behaviour (PeakPatch.jl):
//   src/InitialConditions/RandomField.jl:46-55  _threefry_gaussian(seed, pair)
//   src/InitialConditions/RandomField.jl:70-83  fill_noise_threefry!
// The reference calls Random123.jl 1.7.1 `threefry((seed,0),(pair,0),Val(20))`
// (Random123.jl is a port of the Random123 library of Salmon, Moraes, Dror and
// Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11).  The block
// cipher below is restated from that paper's description of Threefry-2x64
// (Skein's Threefish MIX/permute structure with 64-bit words, rotation
// schedule for two words, key injection every four rounds).
//
// Bit-exactness between the GPU and the CPU oracle rests on every floating
// point step being an IEEE-754 operation with a single, fully specified
// rounding: +, -, *, /, sqrt and fma.  On the device these are issued as the
// explicit-rounding intrinsics (__dadd_rn, __dmul_rn, __fma_rn, __dsqrt_rn) so
// that the compiler cannot contract a multiply and an add into one fused
// operation; on the host the same macros map onto plain operators compiled
// with -ffp-contract=off and std::fma.  log, sin and cos are therefore not
// taken from libm or from CUDA's math library: they are the project's own
// implementations below, built from textbook argument reductions and Taylor
// series (see the comments at each function), accurate to about one unit in
// the last place in double precision.
#pragma once
#include <stdint.h>

#include <cmath>
#include <cstring>
#if defined(__CUDACC__)
#define PPB_HD __host__ __device__ __forceinline__
#else
#define PPB_HD inline
#endif

namespace ppbm {

#if defined(__CUDA_ARCH__)
PPB_HD double dadd(double a, double b) { return __dadd_rn(a, b); }
PPB_HD double dsub(double a, double b) { return __dsub_rn(a, b); }
PPB_HD double dmul(double a, double b) { return __dmul_rn(a, b); }
PPB_HD double ddiv(double a, double b) { return __ddiv_rn(a, b); }
PPB_HD double dfma(double a, double b, double c) { return __fma_rn(a, b, c); }
PPB_HD double dsqrt(double a) { return __dsqrt_rn(a); }
PPB_HD int64_t d_as_i64(double x) { return __double_as_longlong(x); }
PPB_HD double i64_as_d(int64_t x) { return __longlong_as_double(x); }
PPB_HD double u64_to_d(uint64_t x) { return __ull2double_rn(x); }
PPB_HD double rint_d(double x) { return rint(x); }
#else
PPB_HD double dadd(double a, double b) { return a + b; }
PPB_HD double dsub(double a, double b) { return a - b; }
PPB_HD double dmul(double a, double b) { return a * b; }
PPB_HD double ddiv(double a, double b) { return a / b; }
PPB_HD double dfma(double a, double b, double c) { return std::fma(a, b, c); }
PPB_HD double dsqrt(double a) { return std::sqrt(a); }
PPB_HD int64_t d_as_i64(double x) { int64_t i; std::memcpy(&i, &x, 8); return i; }
PPB_HD double i64_as_d(int64_t i) { double x; std::memcpy(&x, &i, 8); return x; }
PPB_HD double u64_to_d(uint64_t x) { return (double)x; }
PPB_HD double rint_d(double x) { return std::nearbyint(x); }
#endif

// ---------------------------------------------------------------------------
// Threefry-2x64 with 20 rounds.
// key = (k0, k1), counter = (c0, c1).  Rotation amounts for the two-word
// variant, rounds 0..7 (repeating): 16 42 12 31 16 32 24 21.  The third key
// word is the Skein key-schedule parity constant xor k0 xor k1.  After rounds
// 4, 8, 12, 16 and 20 the key schedule word pair (s mod 3, s+1 mod 3) is added
// and the injection number s is added to the second word.
// ---------------------------------------------------------------------------
PPB_HD uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }

PPB_HD void threefry2x64_20(uint64_t k0, uint64_t k1, uint64_t c0, uint64_t c1,
                            uint64_t* o0, uint64_t* o1) {
  const uint64_t k2 = 0x1BD11BDAA9FC1A22ULL ^ k0 ^ k1;
  uint64_t x0 = c0 + k0;
  uint64_t x1 = c1 + k1;
#define PPB_TF_ROUND(R) do { x0 += x1; x1 = rotl64(x1, (R)); x1 ^= x0; } while (0)
#define PPB_TF_FOUR()   do { PPB_TF_ROUND(16); PPB_TF_ROUND(42); PPB_TF_ROUND(12); PPB_TF_ROUND(31); } while (0)
#define PPB_TF_FOUR_B() do { PPB_TF_ROUND(16); PPB_TF_ROUND(32); PPB_TF_ROUND(24); PPB_TF_ROUND(21); } while (0)
  PPB_TF_FOUR();   x0 += k1; x1 += k2 + 1;   // injection 1
  PPB_TF_FOUR_B(); x0 += k2; x1 += k0 + 2;   // injection 2
  PPB_TF_FOUR();   x0 += k0; x1 += k1 + 3;   // injection 3
  PPB_TF_FOUR_B(); x0 += k1; x1 += k2 + 4;   // injection 4
  PPB_TF_FOUR();   x0 += k2; x1 += k0 + 5;   // injection 5
#undef PPB_TF_FOUR_B
#undef PPB_TF_FOUR
#undef PPB_TF_ROUND
  *o0 = x0;
  *o1 = x1;
}

// ---------------------------------------------------------------------------
// Natural logarithm for finite x > 0 (normal numbers).
// Method: x = 2^e * m with m in [sqrt(2)/2, sqrt(2)); f = m - 1 (exact);
// log(1+f) = 2 atanh(s), s = f/(2+f), |s| <= 0.1716.  With
// 2 atanh(s) = 2s + s*R(s^2), R(z) = sum_{k>=1} 2 z^k/(2k+1), and
// 2s = f - s*f, one gets log(1+f) = f - (h - s*(h + R)) with h = f^2/2: the
// leading term f is exact and the rounding of s only enters multiplied by
// O(f^2).  The atanh series is truncated after z^12 (|z| <= 0.0295, remainder
// below 3e-20 relative).
// log(2) is split into a 42-bit head (so e*head is exact) and a tail.
// ---------------------------------------------------------------------------
PPB_HD double log_pos(double x) {
  const double LN2_HI = 0x1.62e42fefa3800p-1;
  const double LN2_LO = 0x1.ef35793c76730p-45;
  int64_t bits = d_as_i64(x);
  int e = (int)((bits >> 52) & 0x7ff) - 1023;
  int64_t mbits = (bits & 0x000fffffffffffffLL) | 0x3ff0000000000000LL;  // m in [1,2)
  if ((bits & 0x000fffffffffffffLL) > 0x6a09e667f3bcdLL) {   // m > sqrt(2)
    mbits = (bits & 0x000fffffffffffffLL) | 0x3fe0000000000000LL;      // m/2 in [0.707,1)
    e += 1;
  }
  const double m = i64_as_d(mbits);
  const double f = dsub(m, 1.0);
  const double s = ddiv(f, dadd(2.0, f));
  const double z = dmul(s, s);
  // R(z) = z*(2/3 + z*(2/5 + ... + z*(2/25)))
  double r = 2.0 / 25.0;
  r = dfma(r, z, 2.0 / 23.0);
  r = dfma(r, z, 2.0 / 21.0);
  r = dfma(r, z, 2.0 / 19.0);
  r = dfma(r, z, 2.0 / 17.0);
  r = dfma(r, z, 2.0 / 15.0);
  r = dfma(r, z, 2.0 / 13.0);
  r = dfma(r, z, 2.0 / 11.0);
  r = dfma(r, z, 2.0 / 9.0);
  r = dfma(r, z, 2.0 / 7.0);
  r = dfma(r, z, 2.0 / 5.0);
  r = dfma(r, z, 2.0 / 3.0);
  const double R = dmul(r, z);
  const double h = dmul(dmul(0.5, f), f);
  const double de = (double)e;
  // log(1+f) = f - (h - s*(h+R)); add e*ln2 in two parts
  const double corr = dsub(h, dfma(s, dadd(h, R), dmul(de, LN2_LO)));
  return dadd(dmul(de, LN2_HI), dsub(f, corr));
}

// ---------------------------------------------------------------------------
// sin and cos of a finite double of moderate size (|x| < 2^20).
// Reduction (Cody & Waite): k = round(x * 2/pi), r = x - k*pi/2 with pi/2
// split into two 33-bit heads and a tail so that k*head is exact.  Then
// Taylor series on |r| <= pi/4:
//   sin r = r + r^3 * P(r^2),  P = -1/3! + r^2/5! - ... (through r^21)
//   cos r = 1 - r^2/2 + r^4 * Q(r^2),  Q = 1/4! - r^2/6! + ... (through r^22)
// The factorial reciprocals are evaluated by the compiler from exact integer
// ratios.  The quadrant k mod 4 selects (+-sin, +-cos).
// ---------------------------------------------------------------------------
PPB_HD void sincos_red(double x, double* sn, double* cs) {
  const double PIO2_1 = 0x1.921fb54400000p+0;
  const double PIO2_2 = 0x1.0b4611a600000p-34;
  const double PIO2_3 = 0x1.3198a2e037073p-69;
  const double TWO_OVER_PI = 0x1.45f306dc9c883p-1;
  const double kd = rint_d(dmul(x, TWO_OVER_PI));
  double r = dsub(x, dmul(kd, PIO2_1));
  r = dsub(r, dmul(kd, PIO2_2));
  r = dsub(r, dmul(kd, PIO2_3));
  const int q = ((int)(int64_t)kd) & 3;
  const double z = dmul(r, r);
  // sin r = r + r^3 * P(z), P(z) = sum_{j=0..9} (-1)^(j+1) z^j / (2j+3)!
  double p = 1.0 / 51090942171709440000.0;           //  1/21!
  p = dfma(p, z, -1.0 / 121645100408832000.0);        // -1/19!
  p = dfma(p, z, 1.0 / 355687428096000.0);            //  1/17!
  p = dfma(p, z, -1.0 / 1307674368000.0);             // -1/15!
  p = dfma(p, z, 1.0 / 6227020800.0);                 //  1/13!
  p = dfma(p, z, -1.0 / 39916800.0);                  // -1/11!
  p = dfma(p, z, 1.0 / 362880.0);                     //  1/9!
  p = dfma(p, z, -1.0 / 5040.0);                      // -1/7!
  p = dfma(p, z, 1.0 / 120.0);                        //  1/5!
  p = dfma(p, z, -1.0 / 6.0);                         // -1/3!
  const double s = dfma(dmul(r, z), p, r);
  // cos r = 1 - z/2 + z^2 * Q(z), Q(z) = sum_{j=0..9} (-1)^j z^j / (2j+4)!
  double c = -1.0 / 1124000727777607680000.0;         // -1/22!
  c = dfma(c, z, 1.0 / 2432902008176640000.0);        //  1/20!
  c = dfma(c, z, -1.0 / 6402373705728000.0);          // -1/18!
  c = dfma(c, z, 1.0 / 20922789888000.0);             //  1/16!
  c = dfma(c, z, -1.0 / 87178291200.0);               // -1/14!
  c = dfma(c, z, 1.0 / 479001600.0);                  //  1/12!
  c = dfma(c, z, -1.0 / 3628800.0);                   // -1/10!
  c = dfma(c, z, 1.0 / 40320.0);                      //  1/8!
  c = dfma(c, z, -1.0 / 720.0);                       // -1/6!
  c = dfma(c, z, 1.0 / 24.0);                         //  1/4!
  const double hz = dmul(0.5, z);
  const double w = dsub(1.0, hz);
  // 1 - hz loses the low bits of hz; recover them: ((1 - w) - hz) is exact
  const double co = dadd(w, dfma(dmul(z, z), c, dsub(dsub(1.0, w), hz)));
  switch (q) {
    case 0: *sn = s;  *cs = co;  break;
    case 1: *sn = co; *cs = -s;  break;
    case 2: *sn = -s; *cs = -co; break;
    default: *sn = -co; *cs = s; break;
  }
}

// ---------------------------------------------------------------------------
// One Threefry call -> two standard normal deviates (Box–Muller), exactly as
// RandomField.jl:46-55: u = ((x >> 11) + 1) * 2^-53 in (0, 1];
// r = sqrt(-2 log u1); theta = 2*pi*u2; (r cos theta, r sin theta).
// ---------------------------------------------------------------------------
PPB_HD void threefry_gaussian_pair(uint64_t seed, uint64_t pair, double* g1, double* g2) {
  uint64_t a, b;
  threefry2x64_20(seed, 0ULL, pair, 0ULL, &a, &b);
  const double TWO_M53 = 0x1.0p-53;
  const double TWO_PI = 0x1.921fb54442d18p+2;     // Float64(2*pi)
  const double u1 = dmul(dadd(u64_to_d(a >> 11), 1.0), TWO_M53);
  const double u2 = dmul(dadd(u64_to_d(b >> 11), 1.0), TWO_M53);
  const double r = dsqrt(dmul(-2.0, log_pos(u1)));
  const double th = dmul(TWO_PI, u2);
  double sn, cs;
  sincos_red(th, &sn, &cs);
  *g1 = dmul(r, cs);
  *g2 = dmul(r, sn);
}

// Float64 deviate of the cell with 0-based column-major linear index `lin`
// (lin = i + n*j + n*n*k, i fastest): pair lin>>1, first deviate when lin is
// even, second when odd (RandomField.jl:75-78).
PPB_HD double noise_cell_d(uint64_t seed, uint64_t lin) {
  double g1, g2;
  threefry_gaussian_pair(seed, lin >> 1, &g1, &g2);
  return (lin & 1ULL) ? g2 : g1;
}
// the deviate rounded to Float32, the value stored in a noise field
PPB_HD float noise_cell(uint64_t seed, uint64_t lin) { return (float)noise_cell_d(seed, lin); }

}  // namespace ppbm
