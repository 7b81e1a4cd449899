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
// radius.  Here each halo first writes itself into the suppressor lists of
// the later halos inside its radius, found in a 256^3-cell grid over the
// padded domain (the reference's spatial hash), and the survivals are
// resolved in rounds: a
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

// suppressors of halo i: halos k earlier in the order with |x_i - x_k| < r_k,
// found from k's side — each halo scans the cells within its own radius
// (most radii are a cell or less, where a search within the largest radius
// from every i scanned 9^3 cells).  COUNT: per-i counts; else each k writes
// itself into the lists of the halos it suppresses (list order does not
// matter: the rounds only ask whether any suppressor survives and whether
// all are dead)
template <bool COUNT>
__global__ void suppress_out_kernel(MergeArgs a, int* cursor) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.n) return;
  const double xk = a.x[k], yk = a.y[k], zk = a.z[k], rk = a.r[k];
  const int rank_k = a.rank[k];
  const int c = a.cell[k];
  const int cx = c % NC, cy = (c / NC) % NC, cz = c / (NC * NC);
  const int D = (int)ceil(rk / a.cs);
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
          const int i = a.cidx[q];
          if (a.rank[i] <= rank_k) continue;
          // the reference's test, from k's side: dx = x_i - x_k (Exclusion.jl:129-133)
          const double dist = norm3(a.x[i] - xk, a.y[i] - yk, a.z[i] - zk);
          if (dist < rk) {
            if (COUNT) atomicAdd(a.scount + i, 1);
            else a.sups[a.scount[i] + atomicAdd(cursor + i, 1)] = (int)k;
          }
        }
      }
    }
  }
}

// domain of the catalogue: per block the smallest and largest x, y, z and the
// largest radius (7 doubles), finished on the host
__global__ void domain_kernel(MergeArgs a, double* part) {
  __shared__ double sm[7][256];
  double v[7] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY, -INFINITY};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
    const double x = a.x[i], y = a.y[i], z = a.z[i], r = a.r[i];
    v[0] = fmin(v[0], x); v[1] = fmin(v[1], y); v[2] = fmin(v[2], z);
    v[3] = fmax(v[3], x); v[4] = fmax(v[4], y); v[5] = fmax(v[5], z); v[6] = fmax(v[6], r);
  }
  for (int q = 0; q < 7; q++) sm[q][threadIdx.x] = v[q];
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
      for (int q = 0; q < 7; q++)
        sm[q][threadIdx.x] = q < 3 ? fmin(sm[q][threadIdx.x], sm[q][threadIdx.x + h])
                                   : fmax(sm[q][threadIdx.x], sm[q][threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x < 7) part[blockIdx.x * 7 + threadIdx.x] = sm[threadIdx.x][0];
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
  Slot::MergeBufs& b = sl.merge;
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
  // domain and largest radius (Merger.jl:43-50): block partials on the
  // device, the last step on the host (min and max are exact in any order)
  const int nblk = (int)std::min<int64_t>(1184, (n + 255) / 256);
  b.dom.ensure((size_t)nblk * 7 * 8);
  domain_kernel<<<nblk, 256, 0, s>>>(a, b.dom.as<double>());
  PPB_LAUNCHED(sl.launches);
  std::vector<double> hp((size_t)nblk * 7);
  PPB_CUDA(cudaMemcpyAsync(hp.data(), b.dom.p, hp.size() * 8, cudaMemcpyDeviceToHost, s));
  PPB_CUDA(cudaStreamSynchronize(s));
  double mn[3] = {hp[0], hp[1], hp[2]}, mx[3] = {hp[3], hp[4], hp[5]}, rmax = hp[6];
  for (int q = 1; q < nblk; q++) {
    for (int d = 0; d < 3; d++) {
      mn[d] = std::min(mn[d], hp[q * 7 + d]);
      mx[d] = std::max(mx[d], hp[q * 7 + 3 + d]);
    }
    rmax = std::max(rmax, hp[q * 7 + 6]);
  }
  const double pad = 2.0 * rmax;
  double Lmax = 0.0;
  for (int d = 0; d < 3; d++) {
    a.dmin[d] = mn[d] - pad;
    Lmax = std::max(Lmax, (mx[d] + pad) - (mn[d] - pad));
  }
  a.cs = Lmax / NC;
  a.rmax = rmax;
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
  PPB_CUDA(cudaMemsetAsync(a.scount, 0, (n + 1) * 4, s));
  suppress_out_kernel<true><<<g, 256, 0, s>>>(a, nullptr);
  PPB_LAUNCHED(sl.launches);
  tb = b.tmp.bytes;
  PPB_CUDA(cub::DeviceScan::ExclusiveSum(b.tmp.p, tb, a.scount, a.scount, (int)(n + 1), s));
  sl.launches++;
  int nsup = 0;
  PPB_CUDA(cudaMemcpyAsync(&nsup, a.scount + n, 4, cudaMemcpyDeviceToHost, s));
  PPB_CUDA(cudaStreamSynchronize(s));
  b.sups.ensure((size_t)std::max(nsup, 1) * 4);
  a.sups = b.sups.as<int>();
  PPB_CUDA(cudaMemsetAsync(b.flag.p, 0, (n + 1) * 4, s));   // list cursors
  suppress_out_kernel<false><<<g, 256, 0, s>>>(a, b.flag.as<int>());
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
