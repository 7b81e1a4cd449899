// ppb_kspace.cuh — device helpers shared by the k-space multipliers of the
// tile pipeline (k_fields.cu) and of the multi-resolution stages
// (k_multires.cu): AbstractFFTs frequencies and the P(k) interpolation.
#pragma once
#include <cstdint>

namespace ppb {
namespace ks {

// AbstractFFTs frequency of 0-based index idx: fftfreq keeps idx < ceil(n/2)
// non-negative, the rest wrap to idx - n; rfftfreq is idx itself.
__device__ __forceinline__ double fftfreq(int idx, int n, double mult) {
  const int v = idx < (n + 1) / 2 ? idx : idx - n;
  return (double)v * mult;
}

// P(k): log-log linear interpolation with linear extrapolation
// (src/InitialConditions/PowerSpectrum.jl:11-30); lk, lp are the logs of the
// table's k and P(k), np >= 2 entries.
__device__ __forceinline__ double pk_eval(const double* __restrict__ lk, const double* __restrict__ lp, int np,
                                          double k) {
  const double x = log(k);
  int i;
  if (x <= lk[0]) i = 0;
  else if (x >= lk[np - 1]) i = np - 2;
  else {
    int lo = 0, hi = np - 1;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (lk[mid] <= x) lo = mid; else hi = mid;
    }
    i = lo;
  }
  const double t = (x - lk[i]) / (lk[i + 1] - lk[i]);
  return exp(lp[i] * (1.0 - t) + lp[i + 1] * t);
}

}  // namespace ks
}  // namespace ppb
