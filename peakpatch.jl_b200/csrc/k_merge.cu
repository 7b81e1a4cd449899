// k_merge.cu — merge_catalog (src/Merger/Merger.jl:21-78,
// src/Merger/Exclusion.jl:198-321) on the GPU.
//
// The reference processes halos one at a time in decreasing radius:
//  pass 1 (exclusion): a surviving halo k kills every smaller-or-equal halo
//    whose centre lies within r_k;
//  pass 2 (volume reduction): every surviving halo loses the caps of its
//    overlaps with other survivors, r_new = (r^3 - 3 dV / 4 pi)^(1/3), and
//    dies when nothing is left.
// Pass 1 is a greedy suppression: halo i survives iff no surviving halo
// earlier in the order (stable by index among equal radii) has i within its
// radius.  Here each halo first collects its suppressors (earlier halos with
// i inside their radius) from a 256^3-cell grid over the padded domain (the
// reference's spatial hash), and the survivals are resolved in rounds: a
// halo with a surviving suppressor dies, one whose suppressors are all dead
// survives.  The fixed point is the sequential result.  Pass 2 is a gather
// per survivor; its sums add the same terms as the reference (each pair's
// cap volume, counted from both sides and halved), in another order.
#include <cub/cub.cuh>

#include <cmath>
#include <cstring>
#include <vector>

#include "ppb_ctx.h"

namespace ppb {

namespace {

constexpr int NC = 256;   // cells per axis (Exclusion.jl:23)

struct MergeArgs {
  const float* rec;
  int64_t n;
  int nf;
  double* x;
  double* y;
  double* z;
  double* r;
  double dmin[3];
  double cs;
  int* cell;         // per halo
  int* cstart;       // NC^3 + 1
  int* cfill;        // NC^3 cursor
  int* cidx;         // halos by cell
  int* rank;         // position in the order
  int* scount;       // suppressors per halo, then offsets (n + 1)
  int* sups;         // suppressor lists
  int dsup;          // cell radius of the suppressor search
  unsigned char* state;   // 0 undecided, 1 alive, 2 dead
  int* changed;
  double rmax;
  double* rnew;
};

__global__ void load_kernel(MergeArgs a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const float* h = a.rec + i * a.nf;
  a.x[i] = (double)h[0];
  a.y[i] = (double)h[1];
  a.z[i] = (double)h[2];
  a.r[i] = (double)h[6];
}

// |(ex, ey, ez)| rounded step by step like the reference (no fused
// multiply-add, so that the exclusion decisions are the reference's)
__device__ __forceinline__ double norm3(double ex, double ey, double ez) {
  return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)), __dmul_rn(ez, ez)));
}

__device__ __forceinline__ int cell_of(double v, double m, double cs) {
  int c = (int)floor((v - m) / cs);   // 0-based; the reference adds 1 and clamps to [1, NC]
  return c < 0 ? 0 : (c > NC - 1 ? NC - 1 : c);
}

__global__ void cell_kernel(MergeArgs a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const int cx = cell_of(a.x[i], a.dmin[0], a.cs), cy = cell_of(a.y[i], a.dmin[1], a.cs),
            cz = cell_of(a.z[i], a.dmin[2], a.cs);
  const int c = cx + NC * (cy + NC * cz);
  a.cell[i] = c;
  atomicAdd(a.cstart + c, 1);
}

__global__ void scatter_kernel(MergeArgs a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const int c = a.cell[i];
  a.cidx[a.cstart[c] + atomicAdd(a.cfill + c, 1)] = (int)i;
}

// descending radius, stable: sort key = bitwise complement of the float bits
// (radii are positive)
__global__ void order_key_kernel(MergeArgs a, uint32_t* key, int* idx) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  key[i] = ~__float_as_uint(a.rec[i * a.nf + 6]);
  idx[i] = (int)i;
}

__global__ void rank_kernel(const int* order, int64_t n, int* rank) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) rank[order[q]] = (int)q;
}

// suppressors of halo i: halos k earlier in the order with |x_i - x_k| < r_k;
// with fill = false only counts them
template <bool FILL>
__global__ void suppressor_kernel(MergeArgs a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double xi = a.x[i], yi = a.y[i], zi = a.z[i];
  const int ri = a.rank[i];
  const int c = a.cell[i];
  const int cx = c % NC, cy = (c / NC) % NC, cz = c / (NC * NC);
  const int D = a.dsup;
  int cnt = 0;
  int* out = FILL ? a.sups + a.scount[i] : nullptr;
  for (int dz = -D; dz <= D; dz++) {
    const int jz = cz + dz;
    if (jz < 0 || jz >= NC) continue;
    for (int dy = -D; dy <= D; dy++) {
      const int jy = cy + dy;
      if (jy < 0 || jy >= NC) continue;
      for (int dx = -D; dx <= D; dx++) {
        const int jx = cx + dx;
        if (jx < 0 || jx >= NC) continue;
        const int cc = jx + NC * (jy + NC * jz);
        for (int q = a.cstart[cc]; q < a.cstart[cc + 1]; q++) {
          const int k = a.cidx[q];
          if (a.rank[k] >= ri) continue;
          // the reference's test, from k's side: dx = x_i - x_k (Exclusion.jl:129-133)
          const double dist = norm3(xi - a.x[k], yi - a.y[k], zi - a.z[k]);
          if (dist < a.r[k]) {
            if (FILL) out[cnt] = k;
            cnt++;
          }
        }
      }
    }
  }
  if (!FILL) a.scount[i] = cnt;
}

__global__ void resolve_kernel(MergeArgs a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n || a.state[i] != 0) return;
  bool pending = false;
  for (int q = a.scount[i]; q < a.scount[i + 1]; q++) {
    const unsigned char s = a.state[a.sups[q]];
    if (s == 1) {   // a surviving halo has i inside its radius
      a.state[i] = 2;
      *a.changed = 1;
      return;
    }
    if (s == 0) pending = true;
  }
  if (!pending) {
    a.state[i] = 1;
    *a.changed = 1;
  }
}

// sphere_overlap (Exclusion.jl:82-100): cap volume of sphere 1
__device__ __forceinline__ double cap1(double d, double r1, double r2) {
  const double h1 = __ddiv_rn(__dmul_rn(__dadd_rn(__dsub_rn(r2, r1), d), __dsub_rn(__dadd_rn(r2, r1), d)),
                              __dmul_rn(2.0, d));
  return __dmul_rn(__dmul_rn(3.141592653589793 / 3.0, __dmul_rn(h1, h1)), __dsub_rn(__dmul_rn(3.0, r1), h1));
}

__global__ void reduce_kernel(MergeArgs a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  if (a.state[i] != 1) {
    a.rnew[i] = 0.0;
    return;
  }
  const double xi = a.x[i], yi = a.y[i], zi = a.z[i], ri = a.r[i];
  const int c = a.cell[i];
  const int cx = c % NC, cy = (c / NC) % NC, cz = c / (NC * NC);
  const int D = (int)ceil((ri + a.rmax) / a.cs);
  double dV = 0.0;
  for (int dz = -D; dz <= D; dz++) {
    const int jz = cz + dz;
    if (jz < 0 || jz >= NC) continue;
    for (int dy = -D; dy <= D; dy++) {
      const int jy = cy + dy;
      if (jy < 0 || jy >= NC) continue;
      for (int dx = -D; dx <= D; dx++) {
        const int jx = cx + dx;
        if (jx < 0 || jx >= NC) continue;
        const int cc = jx + NC * (jy + NC * jz);
        for (int q = a.cstart[cc]; q < a.cstart[cc + 1]; q++) {
          const int j = a.cidx[q];
          if (j == i || a.state[j] != 1) continue;
          const double rj = a.r[j];
          const double dist = norm3(a.x[j] - xi, a.y[j] - yi, a.z[j] - zi);
          if (dist < ri + rj && dist > fabs(ri - rj)) dV = __dadd_rn(dV, cap1(dist, ri, rj));
        }
      }
    }
  }
  const double fpt = 4.0 * 3.141592653589793 / 3.0;
  const double vol_new = __dsub_rn(__dmul_rn(fpt, __dmul_rn(__dmul_rn(ri, ri), ri)), dV);
  if (vol_new <= 0.0) {   // dies (read by keep_kernel; other threads still read state)
    a.rnew[i] = 0.0;
  } else {
    a.rnew[i] = pow(__ddiv_rn(vol_new, fpt), 1.0 / 3.0);
  }
}

__global__ void keep_kernel(MergeArgs a, int* flag) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.n) flag[i] = (a.state[i] == 1 && a.rnew[i] > 0.0) ? 1 : 0;
}

__global__ void compact_kernel(MergeArgs a, const int* flag, const int* off, float* out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n || !flag[i]) return;
  const float* h = a.rec + i * a.nf;
  float* o = out + (int64_t)off[i] * a.nf;
  for (int f = 0; f < a.nf; f++) o[f] = h[f];
  o[6] = (float)a.rnew[i];
}

}  // namespace

// merge_catalog on device records; returns the survivors in index order
int64_t merge_catalog_device(Slot& sl, const float* d_rec, int64_t n, int nf, float* d_out) {
  if (n <= 0) return 0;
  PPB_REQUIRE(n < (1ll << 31), "catalogue too large");
  cudaStream_t s = sl.stream;
  Launch L{s, &sl.launches};
  struct Bufs {
    DevBuf x, y, z, r, cell, cstart, cfill, cidx, rank, scount, sups, state, changed, rnew, key, key2, idx, idx2, tmp,
        flag, off;
  } b;
  b.x.ensure(n * 8); b.y.ensure(n * 8); b.z.ensure(n * 8); b.r.ensure(n * 8);
  b.cell.ensure(n * 4);
  const size_t ncell = (size_t)NC * NC * NC;
  b.cstart.ensure((ncell + 1) * 4);
  b.cfill.ensure(ncell * 4);
  b.cidx.ensure(n * 4);
  b.rank.ensure(n * 4);
  b.scount.ensure((n + 1) * 4);
  b.state.ensure(n);
  b.changed.ensure(16);
  b.rnew.ensure(n * 8);
  b.key.ensure(n * 4); b.key2.ensure(n * 4); b.idx.ensure(n * 4); b.idx2.ensure(n * 4);
  b.flag.ensure((n + 1) * 4);
  b.off.ensure((n + 1) * 4);
  MergeArgs a{};
  a.rec = d_rec;
  a.n = n;
  a.nf = nf;
  a.x = b.x.as<double>(); a.y = b.y.as<double>(); a.z = b.z.as<double>(); a.r = b.r.as<double>();
  a.cell = b.cell.as<int>();
  a.cstart = b.cstart.as<int>();
  a.cfill = b.cfill.as<int>();
  a.cidx = b.cidx.as<int>();
  a.rank = b.rank.as<int>();
  a.scount = b.scount.as<int>();
  a.state = b.state.as<unsigned char>();
  a.changed = b.changed.as<int>();
  a.rnew = b.rnew.as<double>();
  const unsigned g = (unsigned)((n + 255) / 256);
  load_kernel<<<g, 256, 0, s>>>(a);
  PPB_LAUNCHED(sl.launches);
  // domain and largest radius (Merger.jl:43-50)
  std::vector<double> hx(n), hy(n), hz(n), hr(n);
  PPB_CUDA(cudaMemcpyAsync(hx.data(), a.x, n * 8, cudaMemcpyDeviceToHost, s));
  PPB_CUDA(cudaMemcpyAsync(hy.data(), a.y, n * 8, cudaMemcpyDeviceToHost, s));
  PPB_CUDA(cudaMemcpyAsync(hz.data(), a.z, n * 8, cudaMemcpyDeviceToHost, s));
  PPB_CUDA(cudaMemcpyAsync(hr.data(), a.r, n * 8, cudaMemcpyDeviceToHost, s));
  PPB_CUDA(cudaStreamSynchronize(s));
  double mn[3] = {hx[0], hy[0], hz[0]}, mx[3] = {hx[0], hy[0], hz[0]}, rmax = hr[0];
  for (int64_t i = 1; i < n; i++) {
    mn[0] = std::min(mn[0], hx[i]); mx[0] = std::max(mx[0], hx[i]);
    mn[1] = std::min(mn[1], hy[i]); mx[1] = std::max(mx[1], hy[i]);
    mn[2] = std::min(mn[2], hz[i]); mx[2] = std::max(mx[2], hz[i]);
    rmax = std::max(rmax, hr[i]);
  }
  const double pad = 2.0 * rmax;
  double Lmax = 0.0;
  for (int d = 0; d < 3; d++) {
    a.dmin[d] = mn[d] - pad;
    Lmax = std::max(Lmax, (mx[d] + pad) - (mn[d] - pad));
  }
  a.cs = Lmax / NC;
  a.rmax = rmax;
  a.dsup = (int)std::ceil(rmax / a.cs);
  // cell lists
  PPB_CUDA(cudaMemsetAsync(b.cstart.p, 0, (ncell + 1) * 4, s));
  PPB_CUDA(cudaMemsetAsync(b.cfill.p, 0, ncell * 4, s));
  cell_kernel<<<g, 256, 0, s>>>(a);
  PPB_LAUNCHED(sl.launches);
  size_t tb = 0;
  PPB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, a.cstart, a.cstart, (int)(ncell + 1), s));
  size_t tb2 = 0;
  PPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb2, b.key.as<uint32_t>(), b.key2.as<uint32_t>(),
                                           b.idx.as<int>(), b.idx2.as<int>(), (int)n, 0, 32, s));
  b.tmp.ensure(std::max(tb, tb2) + 256);
  tb = b.tmp.bytes;
  PPB_CUDA(cub::DeviceScan::ExclusiveSum(b.tmp.p, tb, a.cstart, a.cstart, (int)(ncell + 1), s));
  sl.launches++;
  scatter_kernel<<<g, 256, 0, s>>>(a);
  PPB_LAUNCHED(sl.launches);
  // order: decreasing radius, stable
  order_key_kernel<<<g, 256, 0, s>>>(a, b.key.as<uint32_t>(), b.idx.as<int>());
  PPB_LAUNCHED(sl.launches);
  tb2 = b.tmp.bytes;
  PPB_CUDA(cub::DeviceRadixSort::SortPairs(b.tmp.p, tb2, b.key.as<uint32_t>(), b.key2.as<uint32_t>(), b.idx.as<int>(),
                                           b.idx2.as<int>(), (int)n, 0, 32, s));
  sl.launches++;
  rank_kernel<<<g, 256, 0, s>>>(b.idx2.as<int>(), n, a.rank);
  PPB_LAUNCHED(sl.launches);
  // pass 1: suppressor lists, then rounds
  suppressor_kernel<false><<<g, 256, 0, s>>>(a);
  PPB_LAUNCHED(sl.launches);
  PPB_CUDA(cudaMemsetAsync(a.scount + n, 0, 4, s));
  tb = b.tmp.bytes;
  PPB_CUDA(cub::DeviceScan::ExclusiveSum(b.tmp.p, tb, a.scount, a.scount, (int)(n + 1), s));
  sl.launches++;
  int nsup = 0;
  PPB_CUDA(cudaMemcpyAsync(&nsup, a.scount + n, 4, cudaMemcpyDeviceToHost, s));
  PPB_CUDA(cudaStreamSynchronize(s));
  b.sups.ensure((size_t)std::max(nsup, 1) * 4);
  a.sups = b.sups.as<int>();
  suppressor_kernel<true><<<g, 256, 0, s>>>(a);
  PPB_LAUNCHED(sl.launches);
  PPB_CUDA(cudaMemsetAsync(a.state, 0, n, s));
  for (int64_t round = 0;; round++) {
    PPB_REQUIRE(round <= n, "merge exclusion did not converge");
    PPB_CUDA(cudaMemsetAsync(a.changed, 0, 4, s));
    resolve_kernel<<<g, 256, 0, s>>>(a);
    PPB_LAUNCHED(sl.launches);
    int ch = 0;
    PPB_CUDA(cudaMemcpyAsync(&ch, a.changed, 4, cudaMemcpyDeviceToHost, s));
    PPB_CUDA(cudaStreamSynchronize(s));
    if (!ch) break;
  }
  // pass 2: volume reduction
  reduce_kernel<<<g, 256, 0, s>>>(a);
  PPB_LAUNCHED(sl.launches);
  keep_kernel<<<g, 256, 0, s>>>(a, b.flag.as<int>());
  PPB_LAUNCHED(sl.launches);
  PPB_CUDA(cudaMemsetAsync(b.flag.as<int>() + n, 0, 4, s));
  tb = b.tmp.bytes;
  PPB_CUDA(cub::DeviceScan::ExclusiveSum(b.tmp.p, tb, b.flag.as<int>(), b.off.as<int>(), (int)(n + 1), s));
  sl.launches++;
  compact_kernel<<<g, 256, 0, s>>>(a, b.flag.as<int>(), b.off.as<int>(), d_out);
  PPB_LAUNCHED(sl.launches);
  int nout = 0;
  PPB_CUDA(cudaMemcpyAsync(&nout, b.off.as<int>() + n, 4, cudaMemcpyDeviceToHost, s));
  PPB_CUDA(cudaStreamSynchronize(s));
  return nout;
}

}  // namespace ppb
