// k_shell.cu — per-peak radial-shell collapse measurement (analyse_peak).
//
// Reference: src/HaloFinder/RadialShell.jl:282-891 (analyse_peak) with its
// helpers hRinteg (:100-127), atab4 (:133-155), kernel_strain (:228-277),
// get_evals (:217-222) and the collapse-table lookup
// (src/EllipsoidalCollapse/CollapseTable.jl:128-145).
//
// The stage runs as four kernels on one stream:
//
//  gather_kernel (persistent, one warp per peak, peaks taken from a queue in
//    list order, i.e. largest filter radius first).  A host-built schedule
//    splits the shells (distinct r^2 of the sorted cell list; shell 1 is the
//    peak cell) into chunks of at most 24 cells and packs 32 chunks per
//    group, groups ending on shell boundaries.  Lane l sums chunk l of the
//    group (four cells per step: the four cells' packed offsets in one
//    16-byte load, four 32-byte records in flight per lane, each one 256-bit
//    load), lane l then finalises shell l of the group from the
//    chunk partials, and the cumulative profile Fbar comes from a warp scan
//    of r^3 Fbar.  Sums are compensated single precision (anchored Fast2Sum
//    with anchors per chunk: each rounding error is captured exactly and
//    summed apart) on the optimised path and double precision on the plain
//    path; in both the addends are the single-precision products the
//    reference forms (Float32 field times Int32 offset).  The records come
//    through the texture pipe or as 256-bit loads (the autotuner's choice),
//    or, as an option, through TMA-staged shared-memory rings.
//    Adaptive truncation (optimised path): the warp stops gathering once
//    every shell later read is in, i.e. all shells up to rad[M] + 2 with
//    M = max(crossing shell, first shell beyond ir2min, Rf window):
//    kernel_strain's weight vanishes for |rad[mp] - rad[m1]| >= 2 and the
//    walk only moves inward from the crossing (with no crossing at all every
//    shell is gathered).  A device guard counts any read past the gathered
//    range; it must stay 0 and the host fails loudly otherwise.
//    The kernel ends with the fcrit crossing m0 (RadialShell.jl:494-537) and
//    moves the peak's rows from its staging slot to a pool.
//
//  collapse_kernel (four threads per peak).  kernel_strain windows, the
//    inward collapse walk (four candidate steps per round), RTHL and Sbar/Srb
//    in double precision, in the reference's summation order.  The window weights hRinteg/(u12-u0^2)^2 depend only on
//    the radii and come from a host table.
//
//  zhalf_kernel (sixteen threads per collapsed peak, ten radii).  zvir_half.
//
//  d2f_kernel (one warp per collapsed peak).  Mean Laplacian over the cells
//    within RTHL in list order, stopping at the first out-of-grid cell.
#include <cuda.h>   // CUtensorMap

#include <algorithm>
#include <type_traits>

#include "ppb_internal.h"

namespace ppb {

namespace {

constexpr int NACC = 19;   // gather sums: F, S3, S2_3, G3, Gf3, Q6 (xx yy zz xy xz yz)
constexpr unsigned FULL = 0xffffffffu;

// counters layout
enum { CNT_VISITS = 0, CNT_PREMASK = 1, CNT_NOFCRIT = 2, CNT_M0ONE = 3, CNT_NOCOLL = 4, CNT_RTHLNEG = 5,
       CNT_GUARD = 6, CNT_AKK = 7, CNT_BADPEAK = 8, CNT_WALK = 9, CNT_RING = 10 };

// ---------------------------------------------------------------------------
// accumulators
// ---------------------------------------------------------------------------
template <bool COMP> struct Acc;

template <> struct Acc<false> {      // double precision (the reference's Float64 sums; plain path)
  double s[NACC];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int i = 0; i < NACC; i++) s[i] = 0.0;
  }
  __device__ __forceinline__ void add(int i, float x) { s[i] = __dadd_rn(s[i], (double)x); }
  __device__ __forceinline__ double get(int i) const { return s[i]; }
};

// Compensated single precision (optimised path): NP packed FP32x2 sums,
// anchored.  Component i starts at a power of two K_i (per chunk, from
// anchor_kernel) with |x| <= K_i / (2 cnt) for each of its addends x, cnt the
// chunk's cells, so its running sum s stays in [K_i/2, 3K_i/2]: |s| >= |x| at every
// addition, and Fast2Sum (t = s + x, e = x - (t - s)) gives the exact
// rounding error e of t in three operations; c collects the e.  The chunk's
// sum is (s - K_i) + c, where s - K_i is exact (Sterbenz).  One FP32x2
// instruction serves two sums.
__device__ __forceinline__ float2 fsub2(float2 a, float2 b) {   // a - b, rounded once
  return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
}
template <int NP> struct AccH {
  float2 s[NP], c[NP];
  const float2* K;   // the chunk's anchors (anchor_kernel), 32 float2 apart
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int i = 0; i < NP; i++) { s[i] = K[32 * i]; c[i] = make_float2(0.f, 0.f); }
  }
  __device__ __forceinline__ void add(int i, float2 x) {
    const float2 t = __fadd2_rn(s[i], x);
    c[i] = __fadd2_rn(c[i], fsub2(x, fsub2(t, s[i])));
    s[i] = t;
  }
  __device__ __forceinline__ double X(int i) const { return (double)__fsub_rn(s[i].x, K[32 * i].x) + (double)c[i].x; }
  __device__ __forceinline__ double Y(int i) const { return (double)__fsub_rn(s[i].y, K[32 * i].y) + (double)c[i].y; }
};

// smallest power of two >= v (v >= 0 finite; 0 stays 0)
__device__ __forceinline__ float pow2_ceil(float v) {
  unsigned u = __float_as_uint(v);
  if (u & 0x7fffffu) u = (u + 0x800000u) & 0xff800000u;
  return __uint_as_float(u);
}

// The packed record of a cell is two float4 halves,
//   h0 = (delta, deltaT, psi_z, psi2_x),  h1 = (psi_x, psi_y, psi2_y, psi2_z),
// read with one 256-bit load.  The 22 addends of a cell (11 packed sums):
//   P0 (delta, psi_z d_k)  P1 (psi_x, psi_y)  P2 (psi_z, psi2_x)  P3 (psi2_y, psi2_z)
//   P4..P6 (delta, deltaT) * d_i, d_j, d_k
//   P7 (psi_x d_i, psi_y d_j)  P8 (psi_x d_j, psi_y d_i)  P9 (psi_x d_k, psi_y d_k)
//   P10 (psi_z d_i, psi_z d_j)
__device__ __forceinline__ void accumulate_cell_comp(AccH<11>& A, const float4 h0, const float4 h1, float di,
                                                     float dj, float dk) {
  const float2 dd = make_float2(h0.x, h0.y), pxy = make_float2(h1.x, h1.y);
  A.add(0, make_float2(h0.x, __fmul_rn(h0.z, dk)));
  A.add(1, pxy);
  A.add(2, make_float2(h0.z, h0.w));
  A.add(3, make_float2(h1.z, h1.w));
  A.add(4, __fmul2_rn(dd, make_float2(di, di)));
  A.add(5, __fmul2_rn(dd, make_float2(dj, dj)));
  A.add(6, __fmul2_rn(dd, make_float2(dk, dk)));
  A.add(7, __fmul2_rn(pxy, make_float2(di, dj)));
  A.add(8, __fmul2_rn(pxy, make_float2(dj, di)));
  A.add(9, __fmul2_rn(pxy, make_float2(dk, dk)));
  A.add(10, __fmul2_rn(make_float2(h0.z, h0.z), make_float2(di, dj)));
}

// one cell of the plain path: both halves, 19 double sums
__device__ __forceinline__ void accumulate_cell(Acc<false>& A, const float4 h0, const float4 h1, float di, float dj,
                                                float dk) {
  const float delta = h0.x, deltaT = h0.y, px = h1.x, py = h1.y, pz = h0.z;
  A.add(0, delta);
  A.add(1, px); A.add(2, py); A.add(3, pz);
  A.add(4, h0.w); A.add(5, h1.z); A.add(6, h1.w);
  A.add(7, __fmul_rn(delta, di)); A.add(8, __fmul_rn(delta, dj)); A.add(9, __fmul_rn(delta, dk));
  A.add(10, __fmul_rn(deltaT, di)); A.add(11, __fmul_rn(deltaT, dj)); A.add(12, __fmul_rn(deltaT, dk));
  A.add(13, __fmul_rn(px, di)); A.add(14, __fmul_rn(py, dj)); A.add(15, __fmul_rn(pz, dk));
  A.add(16, __fmul_rn(px, dj)); A.add(16, __fmul_rn(py, di));
  A.add(17, __fmul_rn(px, dk)); A.add(17, __fmul_rn(pz, di));
  A.add(18, __fmul_rn(py, dk)); A.add(18, __fmul_rn(pz, dj));
}

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

// smallest m in [lo, hi] with rad[m] > x, or hi+1
__device__ __forceinline__ int first_gt(const double* rad, int lo, int hi, double x) {
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(rad + mid) > x) hi = mid - 1; else lo = mid + 1;
  }
  return lo;
}
// largest m in [lo, hi] with rad[m] < x, or lo-1
__device__ __forceinline__ int last_lt(const double* rad, int lo, int hi, double x) {
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(rad + mid) < x) lo = mid + 1; else hi = mid - 1;
  }
  return hi;
}

// geometry that depends only on the shell radii and the peak's Rf / ir2min
struct Geo {
  int m0_init;   // first finalised shell with r^2 > ir2min, else the last one (RadialShell.jl:392-399)
  int mrf;       // the per-cell Rf search (RadialShell.jl:457-471)
  int mlow_rf, mupp_rf;
};

// mmax: the peak's last finalised shell (nshell_p - 1 for a shell list of
// nshell_p distinct r^2)
__device__ __forceinline__ Geo geometry(const ShellArgs& a, double Rf, int ir2min, int mmax) {
  Geo g;
  {
    int lo = 2, hi = mmax;
    while (lo <= hi) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(a.r2m + mid) > ir2min) hi = mid - 1; else lo = mid + 1;
    }
    g.m0_init = (lo <= mmax) ? lo : (mmax >= 2 ? mmax : 1);
  }
  // the per-cell scan is decided by the first cell of each distinct r^2;
  // group s (s-th nonzero r^2) reports index max(s-1, 1); earliest strict
  // minimum of |r^2 - (Rf/alatt)^2| below 10
  g.mrf = 1;
  {
    const double rq = (Rf / a.alatt) * (Rf / a.alatt);
    const int K = mmax;   // nonzero distinct r^2 values of the peak's list
    int lo = 1, hi = K;
    while (lo <= hi) {
      const int mid = (lo + hi) >> 1;
      if ((double)__ldg(a.r2m + mid + 1) >= rq) hi = mid - 1; else lo = mid + 1;
    }
    double best = 10.0;
    int sbest = 0;
    for (int s = lo - 1; s <= lo; s++) {
      if (s < 1 || s > K) continue;
      const double dv = fabs((double)__ldg(a.r2m + s + 1) - rq);
      if (dv < best) { best = dv; sbest = s; }
    }
    if (sbest > 0) g.mrf = sbest > 1 ? sbest - 1 : 1;
  }
  const double* rad = a.rad;
  g.mlow_rf = g.mrf;
  if (g.mrf > 1) {
    const double rlow = fmax(__ldg(rad + g.mrf) - 2.0, 0.0);
    const int f = first_gt(rad, 1, g.mrf - 1, rlow);
    if (f <= g.mrf - 1) g.mlow_rf = f;
  }
  g.mupp_rf = g.mrf;
  {
    const int l = last_lt(rad, g.mrf + 1, mmax, __ldg(rad + g.mrf) + 2.0);
    if (l >= g.mrf + 1) g.mupp_rf = l;
  }
  return g;
}

// ===========================================================================
// gather kernel
// ===========================================================================
// decode a packed cell offset
__device__ __forceinline__ void unpack_cell(int w, int& di, int& dj, int& dk) {
  di = (w << 24) >> 24;
  dj = (w << 16) >> 24;
  dk = (w << 8) >> 24;
}

// shared memory of one gather warp, in doubles: the chunk partials, then
// each lane's copy of its chunk's anchors (component i of lane l at i 32 + l)
constexpr int GATHER_WARP_DOUBLES = (NACC + 1) * 32 + kAnchorStride * 32;

// The anchors of the compensated sums, per chunk (thread per chunk of the
// schedule, before the gather): K = 2^ceil(log2(2 cnt M (1 + 2^-10))) with
// cnt the chunk's cells and M the largest magnitude of the sum's addends — a
// field maximum (the pack kernel leaves them after the records), times the
// chunk's largest offset component for the products with an offset — so
// that |x| <= K / (2 cnt) for every addend of the chunk.  A smaller anchor
// leaves a smaller rounding error in the compensation term, so each chunk
// gets its own.  kAnchorStride float2 per chunk (11 used).
__global__ void anchor_kernel(ShellArgs a) {
  // the seven field maxima (delta, psi x, y, z, psi2 x, y, z) from their
  // slots, reduced by the block (non-negative floats order as their bits)
  __shared__ unsigned mx[7];
  if (threadIdx.x < 7) mx[threadIdx.x] = 0u;
  __syncthreads();
  for (int i = threadIdx.x; i < 7 * kFmaxSlots; i += blockDim.x) atomicMax(&mx[i / kFmaxSlots], __ldg(a.fmax + i));
  __syncthreads();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.nck) return;
  float M[7];
#pragma unroll
  for (int f = 0; f < 7; f++) M[f] = __uint_as_float(mx[f]);
  const float w = 2.0f * (float)__ldg(a.ck_n + c) * (1.0f + 1.0f / 1024.0f);
  const float wd = w * (float)__ldg(a.ck_d + c);
  auto k = [](float m, float scale) { return pow2_ceil(m * scale); };
  float2* K = a.ck_K + (size_t)c * kAnchorStride;
  K[0] = make_float2(k(M[0], w), k(M[3], wd));
  K[1] = make_float2(k(M[1], w), k(M[2], w));
  K[2] = make_float2(k(M[3], w), k(M[4], w));
  K[3] = make_float2(k(M[5], w), k(M[6], w));
  for (int i = 4; i < 7; i++) K[i] = make_float2(k(M[0], wd), k(M[0], wd));
  for (int i = 7; i < 10; i++) K[i] = make_float2(k(M[1], wd), k(M[2], wd));
  K[10] = make_float2(k(M[3], wd), k(M[3], wd));
  K[11] = make_float2(0.f, 0.f);
}

// One cell's 32-byte record with one 256-bit load (Blackwell's
// ld.global.v8): one L1 tag lookup per cell instead of two 16-byte loads.
// The records are 32-byte aligned (cell index x 32 bytes from a 256-byte
// aligned buffer).
__device__ __forceinline__ void ldg_record(const float4* p, float4& a, float4& b) {
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
      : "l"(p));
}

// exact float of a small integer (|d| < 2^22) on the FMA pipe: the bits of
// 1.5 * 2^23 plus d are the float 1.5 * 2^23 + d (ulp 1 there); subtracting
// 1.5 * 2^23 is exact
__device__ __forceinline__ float small_int_float(int d) {
  return __fsub_rn(__int_as_float(0x4B400000 + d), 12582912.0f);
}

// where the gather's records come from: 256-bit loads, the texture pipe
// (a texture object over the record array), or the TMA-staged rings
enum RecordSource { SRC_LDG = 0, SRC_TEX = 1, SRC_RING = 2 };

// Visit the cells of one chunk (ck_n cells of chunk ck of the schedule),
// four at a time: the offsets of four cells come packed in one 16-byte load
// of the chunk-major cell list (loaded one step ahead) and their 32-byte
// records are in flight together.  cell(h0, h1, di, dj, dk) receives each
// in-grid cell; returns their number.
template <int SRC, class F>
__device__ __forceinline__ int visit_chunk(const ShellArgs& a, int ck, int cnt, int64_t lin, bool inside, int pi,
                                           int pj, int pk, F&& cell) {
  const int n = a.n, n2 = a.n * a.n;   // n <= 4096: every offset fits 32 bits
  const float4* __restrict__ aos = a.aos;
  const int4* __restrict__ cp = a.ck_cells + __ldg(a.ck_p + ck);
  int4 wn = cnt > 0 ? __ldg(cp) : make_int4(0, 0, 0, 0);
  int nsh = 0;
  for (int c = 0; c < cnt; c += 4) {
    const int w[4] = {wn.x, wn.y, wn.z, wn.w};
    float4 ra[4], rb[4];
    int d[4][3];
    bool ok[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      d[u][0] = (w[u] << 24) >> 24;
      d[u][1] = (w[u] << 16) >> 24;
      d[u][2] = (w[u] << 8) >> 24;
      bool in = c + u < cnt;
      if (!inside)
        in = in && (unsigned)(pi + d[u][0]) < (unsigned)n && (unsigned)(pj + d[u][1]) < (unsigned)n &&
             (unsigned)(pk + d[u][2]) < (unsigned)n;
      ok[u] = in;
      // cells past the chunk or off the grid read the peak cell and are skipped
      const int off = d[u][0] + n * d[u][1] + n2 * d[u][2];
      const int64_t cell = lin + (in ? off : 0);
      if constexpr (SRC == SRC_TEX) {   // through the texture pipe (2 n^3 < 2^31 float4 elements)
        const int e = 2 * (int)cell;
        ra[u] = tex1Dfetch<float4>((cudaTextureObject_t)a.rec_tex, e);
        rb[u] = tex1Dfetch<float4>((cudaTextureObject_t)a.rec_tex, e + 1);
      } else {
        ldg_record(aos + 2 * cell, ra[u], rb[u]);
      }
    }
    if (c + 4 < cnt) wn = __ldg(cp + (c >> 2) + 1);
#pragma unroll
    for (int u = 0; u < 4; u++) {
      if (ok[u]) {
        nsh++;
        cell(ra[u], rb[u], small_int_float(d[u][0]), small_int_float(d[u][1]), small_int_float(d[u][2]));
      }
    }
  }
  return nsh;
}

// ---------------------------------------------------------------------------
// TMA-staged records.  Each lane owns a two-stage ring in shared memory: a
// stage is one tile::gather4 bulk tensor copy of the four records of one
// step (four rows of the record array viewed as an n^3 x 8 float tensor,
// box 8 x 1) completing on the lane's own mbarrier.  While the lane sums the
// four cells of step s from shared memory, the copy of step s + 1 is in
// flight, so the record latency is hidden without holding the records in
// registers.  Slot j of a stage holds cell (j - lane) & 3 of the step, so
// that the lanes of a shared-memory phase read different banks.  Every wait
// is bounded in time (kRingWaitNs on the global timer): a wait that gives up
// counts CNT_RING (the host then fails the call) and retires the lane's
// ring, which then issues no copy and waits no more, and the lane goes on
// with stale slots; before the kernel ends a lane waits (bounded again) for
// every copy it still has in flight.
// ---------------------------------------------------------------------------
constexpr int kRingStages = 2;
constexpr int kRingSlot = 128;   // bytes per lane and stage: four records
constexpr int kRingWarpBytes = kRingStages * 32 * (kRingSlot + 8);
constexpr unsigned long long kRingWaitNs = 200000000ull;   // 0.2 s

struct Ring {
  uint32_t slot;    // shared address of the lane's stage-0 slot
  uint32_t bar;     // shared address of the lane's stage-0 mbarrier
  uint32_t phase;   // bit st: the parity the next wait on stage st expects
  uint32_t pend;    // bit st: a copy into stage st is in flight
  bool dead;        // a wait gave up: no more copies or waits
  uint64_t tm;      // generic address of the tensor map (kernel parameter)
  unsigned long long* counters;
  __device__ __forceinline__ uint32_t slot_at(int st) const { return slot + st * 32 * kRingSlot; }
  __device__ __forceinline__ uint32_t bar_at(int st) const { return bar + st * 32 * 8; }
};

__device__ __forceinline__ void ring_init(Ring& R) {
#pragma unroll
  for (int st = 0; st < kRingStages; st++)
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(R.bar_at(st)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncwarp();
}

// rows r0..r3 (cells of the step in slot order) into stage st
__device__ __forceinline__ void ring_issue(Ring& R, int st, int r0, int r1, int r2, int r3) {
  if (R.dead) return;
  const uint32_t bar = R.bar_at(st), dst = R.slot_at(st);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(kRingSlot) : "memory");
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
      "l"(R.tm), "r"(0), "r"(r0), "r"(r1), "r"(r2), "r"(r3), "r"(bar)
      : "memory");
  R.pend |= 1u << st;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// wait for stage st's copy for at most kRingWaitNs; true when it completed
__device__ __forceinline__ bool ring_wait_bounded(Ring& R, int st) {
  const uint32_t bar = R.bar_at(st), par = (R.phase >> st) & 1u;
  uint32_t done = 0;
  const unsigned long long t0 = global_ns();
  while (true) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(bar), "r"(par)
        : "memory");
    if (done || global_ns() - t0 > kRingWaitNs) break;
  }
  if (done) {
    R.phase ^= 1u << st;
    R.pend &= ~(1u << st);
  }
  return done != 0;
}

__device__ __forceinline__ void ring_wait(Ring& R, int st) {
  if (R.dead) return;
  if (!ring_wait_bounded(R, st)) {
    atomicAdd(R.counters + CNT_RING, 1ull);
    R.dead = true;
  }
}

// before the kernel ends: no copy of this lane may still be in flight
__device__ __forceinline__ void ring_drain(Ring& R) {
#pragma unroll
  for (int st = 0; st < kRingStages; st++)
    if (R.pend & (1u << st)) ring_wait_bounded(R, st);
}

__device__ __forceinline__ void lds_record(uint32_t addr, float4& a, float4& b) {
  asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];"
               : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w)
               : "r"(addr));
  asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];"
               : "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
               : "r"(addr + 16));
}

// the rows (cell indices, the peak cell for cells past the chunk or off the
// grid) and the in-grid mask of step s of a chunk
__device__ __forceinline__ unsigned step_rows(const int4 w4, int c, int cnt, int lin, bool inside, int pi, int pj,
                                              int pk, int n, int n2, int* row) {
  const int w[4] = {w4.x, w4.y, w4.z, w4.w};
  unsigned ok = 0;
#pragma unroll
  for (int u = 0; u < 4; u++) {
    const int di = (w[u] << 24) >> 24, dj = (w[u] << 16) >> 24, dk = (w[u] << 8) >> 24;
    bool in = c + u < cnt;
    if (!inside)
      in = in && (unsigned)(pi + di) < (unsigned)n && (unsigned)(pj + dj) < (unsigned)n &&
           (unsigned)(pk + dk) < (unsigned)n;
    ok |= (in ? 1u : 0u) << u;
    row[u] = lin + (in ? di + n * dj + n2 * dk : 0);
  }
  return ok;
}

__device__ __forceinline__ void ring_issue_step(Ring& R, int st, const int* row, int rot) {
  // slot j <- cell (j - rot) & 3
  int r[4];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int q = (j - rot) & 3;
    r[j] = q == 0 ? row[0] : q == 1 ? row[1] : q == 2 ? row[2] : row[3];
  }
  ring_issue(R, st, r[0], r[1], r[2], r[3]);
}

// visit_chunk with the records staged by the ring (same cells, same order
// of the callbacks)
template <class F>
__device__ __forceinline__ int visit_chunk_ring(const ShellArgs& a, Ring& R, int ck, int cnt, int lin, bool inside,
                                                int pi, int pj, int pk, F&& cell) {
  const int n = a.n, n2 = a.n * a.n;
  const int4* __restrict__ cp = a.ck_cells + __ldg(a.ck_p + ck);
  const int nst = (cnt + 3) >> 2;
  const int rot = threadIdx.x & 3;
  int4 w0 = make_int4(0, 0, 0, 0), w1 = w0;
  unsigned ok0 = 0, ok1 = 0;
  int row[4];
  if (nst > 0) {
    w0 = __ldg(cp);
    ok0 = step_rows(w0, 0, cnt, lin, inside, pi, pj, pk, n, n2, row);
    ring_issue_step(R, 0, row, rot);
  }
  if (nst > 1) {
    w1 = __ldg(cp + 1);
    ok1 = step_rows(w1, 4, cnt, lin, inside, pi, pj, pk, n, n2, row);
    ring_issue_step(R, 1, row, rot);
  }
  int nsh = 0;
  auto consume = [&](int st, const int4 w4, unsigned ok) {
    ring_wait(R, st);
    const int w[4] = {w4.x, w4.y, w4.z, w4.w};
    const uint32_t base = R.slot_at(st);
#pragma unroll
    for (int u = 0; u < 4; u++) {
      if (ok & (1u << u)) {
        float4 h0, h1;
        lds_record(base + ((u + rot) & 3) * 32, h0, h1);
        nsh++;
        cell(h0, h1, small_int_float((w[u] << 24) >> 24), small_int_float((w[u] << 16) >> 24),
             small_int_float((w[u] << 8) >> 24));
      }
    }
    // the slot's reads come before the next copy into it
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  };
  for (int s = 0; s < nst; s += 2) {
    consume(0, w0, ok0);
    if (s + 2 < nst) {
      w0 = __ldg(cp + s + 2);
      ok0 = step_rows(w0, 4 * (s + 2), cnt, lin, inside, pi, pj, pk, n, n2, row);
      ring_issue_step(R, 0, row, rot);
    }
    if (s + 1 < nst) {
      consume(1, w1, ok1);
      if (s + 3 < nst) {
        w1 = __ldg(cp + s + 3);
        ok1 = step_rows(w1, 4 * (s + 3), cnt, lin, inside, pi, pj, pk, n, n2, row);
        ring_issue_step(R, 1, row, rot);
      }
    }
  }
  return nsh;
}

// the chunk's 19 sums (and its in-grid cell count) into column `col` of the
// warp's partial table
template <bool COMP, int SRC>
__device__ __forceinline__ int sum_chunk(const ShellArgs& a, int ck, int cnt, int64_t lin, bool inside, int pi,
                                         int pj, int pk, double* part, int col, Ring* ring) {
  int nsh;
  // the chunk's anchors into this lane's slot (three 32-byte loads), read
  // from there at the chunk's start and end
  float2* K = reinterpret_cast<float2*>(part + (NACC + 1) * 32) + col;
  if constexpr (COMP) {
    const float4* src = reinterpret_cast<const float4*>(a.ck_K + (size_t)ck * kAnchorStride);
    float4 u[6];
    ldg_record(src, u[0], u[1]);
    ldg_record(src + 2, u[2], u[3]);
    ldg_record(src + 4, u[4], u[5]);
#pragma unroll
    for (int q = 0; q < 6; q++) {
      K[32 * (2 * q)] = make_float2(u[q].x, u[q].y);
      if (2 * q + 1 < 11) K[32 * (2 * q + 1)] = make_float2(u[q].z, u[q].w);
    }
  }
  if constexpr (COMP) {
    AccH<11> A;
    A.K = K;
    A.zero();
    auto f = [&](const float4& h0, const float4& h1, float di, float dj, float dk) {
      accumulate_cell_comp(A, h0, h1, di, dj, dk);
    };
    if constexpr (SRC == SRC_RING) nsh = visit_chunk_ring(a, *ring, ck, cnt, (int)lin, inside, pi, pj, pk, f);
    else nsh = visit_chunk<SRC>(a, ck, cnt, lin, inside, pi, pj, pk, f);
    part[0 * 32 + col] = A.X(0);
    part[1 * 32 + col] = A.X(1);
    part[2 * 32 + col] = A.Y(1);
    part[3 * 32 + col] = A.X(2);
    part[4 * 32 + col] = A.Y(2);
    part[5 * 32 + col] = A.X(3);
    part[6 * 32 + col] = A.Y(3);
    part[7 * 32 + col] = A.X(4);
    part[8 * 32 + col] = A.X(5);
    part[9 * 32 + col] = A.X(6);
    part[10 * 32 + col] = A.Y(4);
    part[11 * 32 + col] = A.Y(5);
    part[12 * 32 + col] = A.Y(6);
    part[13 * 32 + col] = A.X(7);
    part[14 * 32 + col] = A.Y(7);
    part[15 * 32 + col] = A.Y(0);
    part[16 * 32 + col] = A.X(8) + A.Y(8);    // psi_x d_j + psi_y d_i
    part[17 * 32 + col] = A.X(9) + A.X(10);   // psi_x d_k + psi_z d_i
    part[18 * 32 + col] = A.Y(9) + A.Y(10);   // psi_y d_k + psi_z d_j
  } else {
    Acc<false> A;
    A.zero();
    auto f = [&](const float4& h0, const float4& h1, float di, float dj, float dk) {
      accumulate_cell(A, h0, h1, di, dj, dk);
    };
    if constexpr (SRC == SRC_RING) nsh = visit_chunk_ring(a, *ring, ck, cnt, (int)lin, inside, pi, pj, pk, f);
    else nsh = visit_chunk<SRC>(a, ck, cnt, lin, inside, pi, pj, pk, f);
#pragma unroll
    for (int v = 0; v < NACC; v++) part[v * 32 + col] = A.get(v);
  }
  part[NACC * 32 + col] = (double)nsh;
  return nsh;
}

template <bool COMP, bool ADAPTIVE, int SRC>
__device__ void gather_one(const ShellArgs& a, int64_t p, double* stage, double* part, Ring* ring) {
  const int lane = threadIdx.x & 31;
  PeakHdr* hdr = a.hdr + p;
  int4 gq, pc;   // geometry, and the peak's cell with its flags (geometry kernel)
  {
    const float4* g2 = reinterpret_cast<const float4*>(a.geo + 2 * p);
    float4 u, v;
    ldg_record(g2, u, v);
    gq = make_int4(__float_as_int(u.x), __float_as_int(u.y), __float_as_int(u.z), __float_as_int(u.w));
    pc = make_int4(__float_as_int(v.x), __float_as_int(v.y), __float_as_int(v.z), __float_as_int(v.w));
  }
  if (!(pc.w & 1)) {   // invalid peak index or redshift from the caller
    if (lane == 0) {
      atomicAdd(a.counters + CNT_BADPEAK, 1ull);
      hdr->status = HS_BAD;
    }
    return;
  }
  const int64_t lin = a.pk.lin[p];
  const int pi = pc.x, pj = pc.y, pk = pc.z;
  const double fcrit = a.pk.fcrit[p];
  const double* __restrict__ rad = a.rad;
  const int mmax = a.mlim[p];   // the peak's last finalised shell
  // cells past the first cell of shell mmax + 1 are not summed (a peak with a
  // shorter list reads only its own shells; the list's last shell is never
  // finalised, RadialShell.jl:386-390)
  const int cell_lim = __ldg(a.sh_start + mmax);
  const int m0_init = gq.x, mrf = gq.y, mupp_rf = gq.w;

  // ---- the peak cell (shell 1) ------------------------------------------
  const float4* __restrict__ aos = a.aos;
  float4 c0, c1;
  ldg_record(aos + 2 * lin, c0, c1);
  if (lane < ROW) {   // c0 = (delta, deltaT, psi_z, psi2_x), c1 = (psi_x, psi_y, psi2_y, psi2_z)
    double v = 0.0;
    if (lane == R_FBAR) v = (double)c0.x;
    else if (lane == R_N) v = 1.0;
    else if (lane == R_S) v = (double)c1.x;
    else if (lane == R_S + 1) v = (double)c1.y;
    else if (lane == R_S + 2) v = (double)c0.z;
    else if (lane == R_S2) v = (double)c0.w;
    else if (lane == R_S2 + 1) v = (double)c1.z;
    else if (lane == R_S2 + 2) v = (double)c1.w;
    stage[ROW + lane] = v;
  }
  const bool inside = (pc.w & 2) != 0;
  int state = 0;          // 0 unknown, 1 inward, 2 crossing found
  int mcross = 0;
  int mtarget = ADAPTIVE ? -1 : mmax;   // last shell to gather (-1: not known yet)
  int mdone = 1;
  double FB = 0.0;                      // r^3 Fbar of shell mdone (0 at the peak cell, rad[1] = 0)
  double dF_prev = (double)c0.x;        // shell-mean delta of shell mdone
  long long visits = 0;
  for (int g = 0; g < a.ngroups; g++) {
    const int base = __ldg(a.grp_a + g);
    if (base > mmax || (mtarget >= 0 && base > mtarget)) break;
    const int gend = min(__ldg(a.grp_b + g), mmax);
    const int c0g = __ldg(a.grp_c + g), ncg = __ldg(a.grp_c + g + 1) - c0g;
    // (a) lane l sums chunk c0g + l into the shared partial table
    if (lane < ncg) {
      const int s0 = __ldg(a.ck_s + c0g + lane), cnt = s0 < cell_lim ? __ldg(a.ck_n + c0g + lane) : 0;
      visits += sum_chunk<COMP, SRC>(a, c0g + lane, cnt, lin, inside, pi, pj, pk, part, lane, ring);
    }
    __syncwarp();
    // (b) lane l finalises shell base + l from its chunks (double-precision
    // sum of the chunk partials, each of which is exact to ~2^-48)
    const int m = base + lane;
    const bool own = m <= gend;
    double my_dF = 0.0, g0 = 0.0;
    if (own) {
      double t[NACC + 1];
#pragma unroll
      for (int v = 0; v <= NACC; v++) t[v] = 0.0;
      const int k0 = __ldg(a.sh_c0 + m) - c0g, nk = __ldg(a.sh_nc + m);
      for (int k = k0; k < k0 + nk; k++) {
#pragma unroll
        for (int v = 0; v <= NACC; v++) t[v] += part[v * 32 + k];
      }
      const double r = __ldg(rad + m);
      const double ir = 1.0 / r;   // one division; the products differ from t / r by at most an ulp
      const double nsh = t[NACC];
      my_dF = nsh > 0 ? t[0] / nsh : 0.0;
      double row[ROW];
#pragma unroll
      for (int v = 0; v < ROW; v++) row[v] = 0.0;
      row[R_N] = nsh;
#pragma unroll
      for (int L = 0; L < 3; L++) {
        row[R_S + L] = t[1 + L];
        row[R_S2 + L] = t[4 + L];
        row[R_G + L] = t[7 + L] * ir;
        row[R_GF + L] = t[10 + L] * ir;
      }
      row[R_Q + 0] = (2.0 * t[13]) * ir;
      row[R_Q + 1] = (2.0 * t[14]) * ir;
      row[R_Q + 2] = (2.0 * t[15]) * ir;
      row[R_Q + 3] = t[16] * ir;
      row[R_Q + 4] = t[17] * ir;
      row[R_Q + 5] = t[18] * ir;
      double2* dst = reinterpret_cast<double2*>(stage + (int64_t)m * ROW);
#pragma unroll
      for (int v = 1; v < ROW / 2; v++) dst[v] = make_double2(row[2 * v], row[2 * v + 1]);
      g0 = row[1];   // slots 0 (Fbar, after the scan) and 1 are stored together
    }
    __syncwarp();
    // (c) cumulative mean overdensity (RadialShell.jl:386-390) as a scan of
    // FB[m] = r3[m] Fbar[m] = FB[m-1] + (dF[m-1] + dF[m]) / 2 * (r3[m] - r3[m-1])
    double prev_dF = __shfl_up_sync(FULL, my_dF, 1);
    if (lane == 0) prev_dF = dF_prev;
    const double rm = __ldg(rad + (own ? m : base)), rp = __ldg(rad + (own ? m - 1 : base - 1));
    const double r3 = rm * rm * rm, r3p = rp * rp * rp;
    double x = own ? 0.5 * (prev_dF + my_dF) * (r3 - r3p) : 0.0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double y = __shfl_up_sync(FULL, x, o);
      if (lane >= o) x += y;
    }
    const double FBm = FB + x;
    const double fb = FBm / r3;
    if (own) {
      double2* dst = reinterpret_cast<double2*>(stage + (int64_t)m * ROW);
      dst[0] = make_double2(fb, g0);
    }
    const int last = gend - base;
    FB = __shfl_sync(FULL, FBm, last);
    dF_prev = __shfl_sync(FULL, my_dF, last);
    // (d) crossing state, in shell order: at m0_init Fbar < fcrit means the
    // crossing lies inward; beyond it the first Fbar < fcrit is the crossing
    if (state == 0) {
      const unsigned bi = __ballot_sync(FULL, own && m == m0_init && fb < fcrit);
      if (bi) {
        state = 1;
      } else {
        const unsigned bc = __ballot_sync(FULL, own && m > m0_init && fb < fcrit);
        if (bc) {
          state = 2;
          mcross = base + __ffs(bc) - 1;
        }
      }
    }
    mdone = gend;
    if (ADAPTIVE && mtarget < 0 && (state != 0 || mdone >= mmax)) {
      int M = max(max(m0_init, mrf), mupp_rf);
      if (state == 2) M = max(M, mcross);
      mtarget = state == 0 ? mmax : min(__ldg(a.need + M), mmax);
    }
    __syncwarp();
  }
  {
    const long long tv = warp_sum_ll(visits);
    if (lane == 0) atomicAdd(a.counters + CNT_VISITS, (unsigned long long)tv);
  }

  // ---- fcrit crossing m0 (RadialShell.jl:494-537) ------------------------
  int m0 = m0_init;
  int status = HS_OK;
  if (state == 2) {
    m0 = mcross;
  } else if (state == 1) {
    // inward: m0 = one above the first shell below m0_init (going down)
    // with Fbar >= fcrit; none -> no fcrit crossing
    bool found = false;
    for (int top = m0_init - 1; top >= 1 && !found; top -= 32) {
      const int mp = top - lane;
      const bool ge = mp >= 1 && stage[(int64_t)mp * ROW + R_FBAR] >= fcrit;
      const unsigned b = __ballot_sync(FULL, ge);
      if (b) {
        found = true;
        m0 = top - (__ffs(b) - 1) + 1;
      }
    }
    if (!found) status = HS_NOFCRIT;
  }
  if (status == HS_OK && m0 == 1) status = HS_M0ONE;   // zvir1p at m0 is forced to -1 < ZZon (:581-622)
  if (status != HS_OK) {
    if (lane == 0) {
      atomicAdd(a.counters + (status == HS_NOFCRIT ? CNT_NOFCRIT : CNT_M0ONE), 1ull);
      PeakHdr h;
      h.off = 0; h.mdone = mdone; h.m0 = m0; h.status = status; h.pad = 0;
      *hdr = h;
    }
    return;
  }

  // ---- move the rows 1..mdone to the pool ---------------------------------
  long long off = 0;
  if (lane == 0) off = (long long)atomicAdd(a.pool_ctr, (unsigned long long)(mdone + 1));
  off = __shfl_sync(FULL, off, 0);
  if (off + mdone + 1 > a.pool_cap) {   // the host grows the pool and runs the batch again
    if (lane == 0) {
      PeakHdr h;
      h.off = 0; h.mdone = mdone; h.m0 = m0; h.status = HS_OVERFLOW; h.pad = 0;
      *hdr = h;
    }
    return;
  }
  {
    const double2* src = reinterpret_cast<const double2*>(stage + ROW);
    double2* dst = reinterpret_cast<double2*>(a.pool + (off + 1) * ROW);
    const int nv = mdone * (ROW / 2);
    for (int i0 = 0; i0 < nv; i0 += 128) {   // four loads in flight per lane
      double2 v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int i = i0 + 32 * u + lane;
        if (i < nv) v[u] = src[i];
      }
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int i = i0 + 32 * u + lane;
        if (i < nv) dst[i] = v[u];
      }
    }
  }
  if (lane == 0) {
    PeakHdr h;
    h.off = off; h.mdone = mdone; h.m0 = m0; h.status = HS_OK; h.pad = 0;
    *hdr = h;
  }
}

#ifndef PPB_GATHER_MINB
#define PPB_GATHER_MINB 4
#endif
// SRC: SRC_LDG or SRC_TEX (a.rec_tex set)
template <bool COMP, bool ADAPTIVE, int SRC>
__global__ void __launch_bounds__(32 * kGatherWarps, PPB_GATHER_MINB) gather_kernel(ShellArgs a) {
  extern __shared__ double gsm[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int64_t slot = (int64_t)blockIdx.x * kGatherWarps + wib;
  double* stage = a.stage + slot * a.stage_stride;
  double* part = gsm + (size_t)wib * GATHER_WARP_DOUBLES;
  while (true) {
    int q = 0;
    if (lane == 0) q = atomicAdd(a.queue, 1);
    q = __shfl_sync(FULL, q, 0);
    if (q >= a.npk) break;
    const int64_t p = a.order ? (int64_t)a.order[q] : (int64_t)q;
    gather_one<COMP, ADAPTIVE, SRC>(a, p, stage, part, nullptr);
    __syncwarp();
  }
}

// The same with the records staged through each lane's TMA ring (tm: the
// record array as an n^3 x 8 float tensor, box 8 x 1; n^3 < 2^31).  Shared
// memory: the warps' rings, then their partial tables.
template <bool COMP, bool ADAPTIVE>
__global__ void __launch_bounds__(32 * kGatherWarps, PPB_GATHER_MINB)
    gather_ring_kernel(ShellArgs a, const __grid_constant__ CUtensorMap tm) {
  extern __shared__ __align__(128) unsigned char rsm[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int64_t slot = (int64_t)blockIdx.x * kGatherWarps + wib;
  double* stage = a.stage + slot * a.stage_stride;
  unsigned char* ring_mem = rsm + (size_t)wib * kRingWarpBytes;
  double* part = reinterpret_cast<double*>(rsm + (size_t)kGatherWarps * kRingWarpBytes) + (size_t)wib * GATHER_WARP_DOUBLES;
  Ring R;
  R.slot = (uint32_t)__cvta_generic_to_shared(ring_mem) + lane * kRingSlot;
  R.bar = (uint32_t)__cvta_generic_to_shared(ring_mem + kRingStages * 32 * kRingSlot) + lane * 8;
  R.phase = 0;
  R.pend = 0;
  R.dead = false;
  R.tm = reinterpret_cast<uint64_t>(&tm);
  R.counters = a.counters;
  ring_init(R);
  while (true) {
    int q = 0;
    if (lane == 0) q = atomicAdd(a.queue, 1);
    q = __shfl_sync(FULL, q, 0);
    if (q >= a.npk) break;
    const int64_t p = a.order ? (int64_t)a.order[q] : (int64_t)q;
    gather_one<COMP, ADAPTIVE, SRC_RING>(a, p, stage, part, &R);
    __syncwarp();
  }
  ring_drain(R);
}

// interleave the low 10 bits of x, y, z (Morton order)
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
  v &= 0x3ff;
  v = (v | (v << 16)) & 0x030000ff;
  v = (v | (v << 8)) & 0x0300f00f;
  v = (v | (v << 4)) & 0x030c30c3;
  v = (v | (v << 2)) & 0x09249249;
  return v;
}

// per-peak geometry (thread per peak) and the gather order key: the Morton
// index of the peak's brick (2^brick_shift cells on a side, 10 bits per
// axis), so that peaks whose spheres overlap (of any filter) are gathered
// close in time and share cached records
__global__ void geo_kernel(ShellArgs a, uint32_t* key, int32_t* idx) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.npk) return;
  int mmax = a.mmax;
  if (a.r2lim && a.r2lim[p] > 0) {   // shell list r^2 <= r2lim: nshell_p distinct values
    int lo = 1, hi = a.nshell;
    while (lo <= hi) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(a.r2m + mid) <= a.r2lim[p]) lo = mid + 1; else hi = mid - 1;
    }
    mmax = max(min(hi - 1, a.mmax), 1);
  }
  if (a.npcap) {   // cells 1..npart of the list: the shells closed before cell npart + 1
    // distinct r^2 value g holds cells sh_start[g] ..; the cap's last cell
    // (0-based npart - 1) lies in the largest g with sh_start[g] <= npart - 1,
    // and shells 1..g (profile numbering, shell 1 = the centre) are the ones
    // the reference finalises inside its loop over jp = 2..npart
    const int last = a.npcap[p] - 1;
    int lo = 0, hi = a.nshell - 1;
    while (lo <= hi) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(a.sh_start + mid) <= last) lo = mid + 1; else hi = mid - 1;
    }
    mmax = max(min(hi, mmax), 1);
  }
  a.mlim[p] = mmax;
  const Geo g = geometry(a, a.pk.Rf[p], a.pk.ir2min[p], mmax);
  a.geo[2 * p] = make_int4(g.m0_init, g.mrf, g.mlow_rf, g.mupp_rf);
  // the peak's cell and flags for the gather: bit 0 a valid peak (index on
  // the grid, redshift > -1), bit 1 every cell of its shells up to mmax
  // (radius < rad[mmax] + 1) on the grid
  const int64_t lin = a.pk.lin[p], n = a.n, n2 = n * n;
  const bool valid = lin >= 0 && lin < n2 * n && a.pk.ZZon[p] > -1.0;
  int pi = 0, pj = 0, pk = 0, flags = 0;
  if (valid) {
    pk = (int)(lin / n2);
    pj = (int)((lin / n) % n);
    pi = (int)(lin % n);
    const int rext = (int)ceil(__ldg(a.rad + mmax)) + 1;
    const bool inside = pi - rext >= 0 && pj - rext >= 0 && pk - rext >= 0 && pi + rext < n && pj + rext < n &&
                        pk + rext < n;
    flags = 1 | (inside ? 2 : 0);
  }
  a.geo[2 * p + 1] = make_int4(pi, pj, pk, flags);
  if (key) {
    uint32_t k = 0xffffffffu;   // invalid peaks last
    if (lin >= 0 && lin < n2 * n) {
      const int b = a.brick_shift;
      k = spread3((uint32_t)pi >> b) | (spread3((uint32_t)pj >> b) << 1) | (spread3((uint32_t)pk >> b) << 2);
    }
    key[p] = k;
    idx[p] = (int32_t)p;
  }
}

// ===========================================================================
// collapse kernel (four threads per peak)
// ===========================================================================
struct KS {
  double E[6];   // xx yy zz xy xz yz
  double g[3], gf[3];
};

// Symmetric 3x3 eigenvalues, ascending: the trigonometric solution of the
// characteristic cubic (O. K. Smith, "Eigenvalues of a symmetric 3 x 3
// matrix", Comm. ACM 4 (1961) 168).  m = (xx, yy, zz, xy, xz, yz).
__device__ __forceinline__ void eig3(const double* m, double* lam) {
  const double a00 = m[0], a11 = m[1], a22 = m[2], a01 = m[3], a02 = m[4], a12 = m[5];
  const double p1 = a01 * a01 + a02 * a02 + a12 * a12;
  double e1, e2, e3;
  if (p1 == 0.0) {
    e1 = a00; e2 = a11; e3 = a22;
  } else {
    const double q = (a00 + a11 + a22) / 3.0;
    const double b00 = a00 - q, b11 = a11 - q, b22 = a22 - q;
    const double p = sqrt((b00 * b00 + b11 * b11 + b22 * b22 + 2.0 * p1) / 6.0);
    const double ip = 1.0 / p;
    const double c00 = b00 * ip, c11 = b11 * ip, c22 = b22 * ip, c01 = a01 * ip, c02 = a02 * ip, c12 = a12 * ip;
    double r = 0.5 * (c00 * (c11 * c22 - c12 * c12) - c01 * (c01 * c22 - c12 * c02) + c02 * (c01 * c12 - c11 * c02));
    r = r < -1.0 ? -1.0 : (r > 1.0 ? 1.0 : r);
    const double phi = acos(r) / 3.0;
    e1 = q + 2.0 * p * cos(phi);
    e3 = q + 2.0 * p * cos(phi + 2.0943951023931957);   // + 2 pi / 3
    e2 = 3.0 * q - e1 - e3;
  }
  double t;
  if (e1 > e2) { t = e1; e1 = e2; e2 = t; }
  if (e2 > e3) { t = e2; e2 = e3; e3 = t; }
  if (e1 > e2) { t = e1; e1 = e2; e2 = t; }
  lam[0] = e1; lam[1] = e2; lam[2] = e3;
}

// trilinear lookup, outside the box -> -1 (CollapseTable.jl:128-145); Float32
// or Float64 nodes
__device__ __forceinline__ double tab_interp(const DevTable& T, double x, double y, double z) {
  if (!(x >= T.x1 && x <= T.x2 && y >= T.y1 && y <= T.y2 && z >= T.z1 && z <= T.z2)) return -1.0;
  const double px = (x - T.x1) / ((T.x2 - T.x1) / (T.nx - 1));
  const double py = (y - T.y1) / ((T.y2 - T.y1) / (T.ny - 1));
  const double pz = (z - T.z1) / ((T.z2 - T.z1) / (T.nz - 1));
  int ix = (int)floor(px), iy = (int)floor(py), iz = (int)floor(pz);
  ix = ix < 0 ? 0 : (ix > T.nx - 2 ? T.nx - 2 : ix);
  iy = iy < 0 ? 0 : (iy > T.ny - 2 ? T.ny - 2 : iy);
  iz = iz < 0 ? 0 : (iz > T.nz - 2 ? T.nz - 2 : iz);
  const double wx = px - ix, wy = py - iy, wz = pz - iz;
  const int64_t o = ix + (int64_t)T.nx * (iy + (int64_t)T.ny * iz);
  const int64_t sy = T.nx, sz = (int64_t)T.nx * T.ny;
  auto v = [&](int64_t i) { return T.td ? __ldg(T.td + o + i) : (double)__ldg(T.t + o + i); };
  const double c00 = (1 - wx) * v(0) + wx * v(1);
  const double c10 = (1 - wx) * v(sy) + wx * v(sy + 1);
  const double c01 = (1 - wx) * v(sz) + wx * v(sz + 1);
  const double c11 = (1 - wx) * v(sz + sy) + wx * v(sz + sy + 1);
  const double c0 = (1 - wy) * c00 + wy * c10;
  const double c1 = (1 - wy) * c01 + wy * c11;
  return (1 - wz) * c0 + wz * c1;
}

// eigen-decomposition -> (trace, e_v, p_v) as the reference (:571-577)
__device__ __forceinline__ void ev_pv(const double E[6], double* Frho, double* ev, double* pv) {
  double lam[3];
  eig3(E, lam);
  const double F = lam[0] + lam[1] + lam[2];
  *Frho = F;
  *ev = 0.0;
  *pv = 0.0;
  if (F > 0.0) {
    *ev = 0.5 * (lam[2] - lam[0]) / F;
    *pv = 0.5 * (lam[2] + lam[0] - 2.0 * lam[1]) / F;
  }
}

__device__ __forceinline__ double zvir_of(const DevTable& T, double Fr, double ev, double pv) {
  if (!(Fr > 0.0)) return -1.0;
  const double poe = ev < 1e-5 ? 0.0 : pv / ev;
  return tab_interp(T, log10(Fr), ev, poe);
}

// one peak's profile rows (row m of shell m, m = 1..mdone)
struct Rows {
  const double* r;
  int mdone;
  unsigned long long* counters;
  __device__ __forceinline__ double get(int v, int m) const {
    if (m > mdone) {                  // never taken when the truncation rule holds
      atomicAdd(counters + CNT_GUARD, 1ull);
      return 0.0;
    }
    return r[(int64_t)m * ROW + v];
  }
};

// kernel_strain (RadialShell.jl:228-277) for centre shell mp over m1 in
// [lo, hi], summed in m1 order.  For mp > 1 only the shells with
// (rad[mp] - rad[m1])^2 < 4 contribute (the table window); for mp == 1 the
// SPH table weights apply to every m1 of [lo, hi].
__device__ __forceinline__ void kernel_strain(const ShellArgs& a, const Rows& R, int mp, int lo, int hi,
                                           double wRnor, double aRnor, KS* out) {
  double E[6] = {0, 0, 0, 0, 0, 0}, g[3] = {0, 0, 0}, gf[3] = {0, 0, 0};
  const double* w;
  double scale;
  if (mp > 1) {
    const int wl = __ldg(a.win_lo + mp), wh = __ldg(a.win_hi + mp);
    lo = max(lo, wl);
    hi = min(hi, wh);
    w = a.wts + __ldg(a.win_off + mp) - wl;
    scale = wRnor / __ldg(a.rad + mp);
  } else {
    w = a.w1;
    scale = aRnor;
  }
  if (hi > R.mdone) {                 // never taken when the truncation rule holds
    atomicAdd(R.counters + CNT_GUARD, 1ull);
    hi = R.mdone;
  }
  // four rows' loads in flight per thread (the sum stays in m1 order)
#pragma unroll 4
  for (int m1 = lo; m1 <= hi; m1++) {
    const double wt = __ldg(w + m1);
    if (mp == 1 && isnan(wt)) atomicAdd(R.counters + CNT_AKK, 1ull);
    const double2* row = reinterpret_cast<const double2*>(R.r + (int64_t)m1 * ROW);
    const double2 v0 = row[0], v1 = row[1], v2 = row[2], v3 = row[3], v4 = row[4], v5 = row[5], v6 = row[6];
    // v0 = (Fbar, G0), v1 = (G1, G2), v2 = (Gf0, Gf1), v3 = (Gf2, Q0), v4 = (Q1, Q2), v5 = (Q3, Q4), v6 = (Q5, -)
    g[0] += wt * v0.y; g[1] += wt * v1.x; g[2] += wt * v1.y;
    gf[0] += wt * v2.x; gf[1] += wt * v2.y; gf[2] += wt * v3.x;
    E[0] -= 0.5 * wt * v3.y; E[1] -= 0.5 * wt * v4.x; E[2] -= 0.5 * wt * v4.y;
    E[3] -= 0.5 * wt * v5.x; E[4] -= 0.5 * wt * v5.y; E[5] -= 0.5 * wt * v6.x;
  }
#pragma unroll
  for (int q = 0; q < 6; q++) out->E[q] = E[q] * scale;
#pragma unroll
  for (int L = 0; L < 3; L++) {
    out->g[L] = g[L] * scale;
    out->gf[L] = gf[L] * scale;
  }
}

__device__ __forceinline__ void write_no_collapse(double* o) {
#pragma unroll
  for (int q = 0; q < RES_N; q++) o[q] = (q == 0 || q == 26) ? -1.0 : 0.0;
}

// Phases 6-7 of a collapsed peak (RadialShell.jl:707-790) and its result
// row: m0 is the shell above the first collapsing step, last / prev the
// kernel_strain values of that step and of the step before it (zvir1p /
// zvir1 their zvir), lastFh the trace at the collapsing step.
__device__ void collapse_finish(const ShellArgs& a, const Rows& R, double ZZon, int m0, double zvir1, double zvir1p,
                                const KS& prev, const KS& last, double lastFh, const double* grf, double* out) {
  const double* __restrict__ rad = a.rad;
  // Phase 6: collapse radius (RadialShell.jl:707-754)
  const double dZvir = zvir1p - zvir1;
  double RTHL;
  const double ra = __ldg(rad + m0 - 1), rb = __ldg(rad + m0);
  const double rad3p = ra * ra * ra, rad3 = rb * rb * rb;
  if (zvir1 > 0.0 && dZvir != 0.0) {
    const double R3 = rad3p + (rad3 - rad3p) * (zvir1p - ZZon) / dZvir;
    RTHL = pow(R3, 1.0 / 3.0);
  } else {
    RTHL = ra;
  }
  if (RTHL <= 0.0) {
    atomicAdd(a.counters + CNT_RTHLNEG, 1ull);
    write_no_collapse(out);
    return;
  }
  const double RTHL3 = RTHL * RTHL * RTHL, RTHL5 = RTHL3 * RTHL * RTHL;
  const double drad3 = rad3 - rad3p;
  const double Fa = R.get(R_FBAR, m0 - 1), Fb = R.get(R_FBAR, m0);
  const double dFb = Fb - Fa;
  double Fbarx;
  double S[6], gk[3], gkf[3];
  if (zvir1 > 0.0 && drad3 != 0.0) {
    const double fr = (RTHL3 - rad3p) / drad3;
    Fbarx = Fa + fr * dFb;
#pragma unroll
    for (int q = 0; q < 6; q++) S[q] = last.E[q] + fr * (prev.E[q] - last.E[q]);
#pragma unroll
    for (int L = 0; L < 3; L++) {
      gk[L] = last.g[L] + fr * (prev.g[L] - last.g[L]);
      gkf[L] = last.gf[L] + fr * (prev.gf[L] - last.gf[L]);
    }
  } else {
    Fbarx = Fa;
#pragma unroll
    for (int q = 0; q < 6; q++) S[q] = last.E[q];
#pragma unroll
    for (int L = 0; L < 3; L++) { gk[L] = prev.g[L]; gkf[L] = prev.gf[L]; }
  }
  // normalize_strain then eigenvalues (RadialShell.jl:748-752)
  {
    const double tr = S[0] + S[1] + S[2];
    if (tr != 0.0) {
      const double f = Fbarx / tr;
#pragma unroll
      for (int q = 0; q < 6; q++) S[q] *= f;
    }
  }
  double Frhoc, e_v_f, p_v_f;
  ev_pv(S, &Frhoc, &e_v_f, &p_v_f);
  double smat[6];
#pragma unroll
  for (int q = 0; q < 6; q++) smat[q] = last.E[q] * (Fbarx / lastFh);

  // Phase 7: Sbar, Sbar2 (RadialShell.jl:758-773), Srb (:776-790)
  double sb[6] = {0, 0, 0, 0, 0, 0};
  long long nS = 0;
  double srb = 0.0;
  for (int m1 = 1; m1 <= m0 - 1; m1++) {
    const double nn = R.get(R_N, m1);
    if (nn > 0) {
#pragma unroll
      for (int L = 0; L < 3; L++) {
        sb[L] += R.get(R_S + L, m1);
        sb[3 + L] += R.get(R_S2 + L, m1);
      }
      nS += (long long)nn;
    }
    if (m1 >= 2) {
      const double r5 = __ldg(a.rad5 + m1), r5p = m1 - 1 >= 2 ? __ldg(a.rad5 + m1 - 1) : 0.0;
      srb += 0.5 * (R.get(R_FBAR, m1 - 1) + R.get(R_FBAR, m1)) * (r5 - r5p);
    }
  }
  if (nS > 0) {
#pragma unroll
    for (int q = 0; q < 6; q++) sb[q] /= (double)nS;
  }
  const double rad5p = (m0 - 1 >= 2) ? __ldg(a.rad5 + m0 - 1) : 0.0;
  if (zvir1 > 0.0 && dZvir != 0.0) srb += 0.5 * (Fa + Fbarx) * (RTHL5 - rad5p);
  if (Fbarx * RTHL5 > 0.0) srb /= (Fbarx * RTHL5);

  // results (layout in ppb.h); zvir_half (26) comes from zhalf_kernel and
  // d2F (30) from d2f_kernel
  double r[RES_N];
  r[0] = RTHL;
  r[1] = srb;
#pragma unroll
  for (int L = 0; L < 3; L++) {
    r[2 + L] = sb[L];
    r[5 + L] = sb[3 + L];
    r[17 + L] = gk[L];
    r[20 + L] = grf[L];
    r[27 + L] = gkf[L];
  }
  r[8] = smat[0]; r[9] = smat[3]; r[10] = smat[4];
  r[11] = smat[3]; r[12] = smat[1]; r[13] = smat[5];
  r[14] = smat[4]; r[15] = smat[5]; r[16] = smat[2];
  r[23] = Fbarx;
  r[24] = e_v_f;
  r[25] = p_v_f;
  r[26] = -1.0;
  r[30] = 0.0;
#pragma unroll
  for (int q = 0; q < RES_N; q++) out[q] = r[q];
}

// One thread per peak: the walk one step at a time (the device is full of
// peaks, so its latency is hidden).
__device__ void collapse_one(const ShellArgs& a, int64_t p) {
  double* out = a.out + p * RES_N;
  const PeakHdr h = a.hdr[p];
  if (h.status != HS_OK) {
    write_no_collapse(out);
    return;
  }
  const double* __restrict__ rad = a.rad;
  const Rows R{a.pool + h.off * ROW, h.mdone, a.counters};
  const double ZZon = a.pk.ZZon[p];
  const double alatt = a.alatt;
  const int m = a.mlim[p];
  const int4 gq = a.geo[2 * p];
  Geo geo;
  geo.m0_init = gq.x; geo.mrf = gq.y; geo.mlow_rf = gq.z; geo.mupp_rf = gq.w;
  const double anor = 1.0;
  const double aRnor = 3.0 * anor / alatt, wnor = anor / (4.0 * 3.141592653589793), wRnor = 3.0 * wnor / alatt;

  // Phase 3: gradient at the filter scale
  double grf[3];
  {
    KS krf;
    kernel_strain(a, R, geo.mrf, geo.mlow_rf, geo.mupp_rf, wRnor, aRnor, &krf);
#pragma unroll
    for (int L = 0; L < 3; L++) grf[L] = krf.g[L];
  }

  // Phase 5: inward walk (RadialShell.jl:566-699) from the crossing m0; the
  // m0 step's zvir is forced to -1.  At mp = 1 the reference's running window
  // is [2, last shell with rad < 2].
  const int hi1 = last_lt(rad, 2, m, 2.0);
  int m0 = h.m0;
  KS prev, last;
  kernel_strain(a, R, m0, 2, m0 > 1 ? m : hi1, wRnor, aRnor, &prev);
  double zprev = -1.0, zvir1 = -1.0, zvir1p = -1.0, lastFh = 0.0;
  bool collapsed = false;
  long long steps = 1;
  for (int mp = m0 - 1; mp >= 1; mp--) {
    KS cur;
    kernel_strain(a, R, mp, 2, mp > 1 ? m : hi1, wRnor, aRnor, &cur);
    steps++;
    double Fh, ev, pv;
    ev_pv(cur.E, &Fh, &ev, &pv);
    const double zv = zvir_of(a.tab, R.get(R_FBAR, mp), ev, pv);
    if (zv >= ZZon) {
      last = cur;
      lastFh = Fh;
      zvir1p = zv;
      zvir1 = zprev;
      m0 = mp + 1;
      collapsed = true;
      break;
    }
    prev = cur;
    zprev = zv;
  }
  atomicAdd(a.counters + CNT_WALK, (unsigned long long)steps);
  if (!collapsed) {
    atomicAdd(a.counters + CNT_NOCOLL, 1ull);
    write_no_collapse(out);
    return;
  }

  collapse_finish(a, R, ZZon, m0, zvir1, zvir1p, prev, last, lastFh, grf, out);
}

__device__ __forceinline__ KS shfl_ks(const KS& k, int src, unsigned mask) {
  KS r;
#pragma unroll
  for (int q = 0; q < 6; q++) r.E[q] = __shfl_sync(mask, k.E[q], src);
#pragma unroll
  for (int L = 0; L < 3; L++) {
    r.g[L] = __shfl_sync(mask, k.g[L], src);
    r.gf[L] = __shfl_sync(mask, k.gf[L], src);
  }
  return r;
}

// QT threads per peak (lanes qbase .. qbase+QT-1, QT = 2 or 4): the inward
// walk evaluates QT consecutive steps per round, thread q taking step
// base + q (mp = m0 - step; step 0 is the m0 step, whose zvir is forced to
// -1), and the group takes the first step that collapses; the step before it
// comes from the thread to its left or, for q = 0, from the previous round's
// last step.  Thread 0 then finishes the peak alone.  Several threads per
// peak shorten the walk's latency when there are few peaks to hide it.
template <int QT>
__device__ void collapse_group(const ShellArgs& a, int64_t p, int q, int qbase, unsigned qmask) {
  double* out = a.out + p * RES_N;
  const PeakHdr h = a.hdr[p];
  if (h.status != HS_OK) {
    if (q == 0) write_no_collapse(out);
    return;
  }
  const double* __restrict__ rad = a.rad;
  const Rows R{a.pool + h.off * ROW, h.mdone, a.counters};
  const double ZZon = a.pk.ZZon[p];
  const double alatt = a.alatt;
  const int m = a.mlim[p];
  const int4 gq = a.geo[2 * p];
  Geo geo;
  geo.m0_init = gq.x; geo.mrf = gq.y; geo.mlow_rf = gq.z; geo.mupp_rf = gq.w;
  const double anor = 1.0;
  const double aRnor = 3.0 * anor / alatt, wnor = anor / (4.0 * 3.141592653589793), wRnor = 3.0 * wnor / alatt;

  // Phase 3: gradient at the filter scale (thread 0, beside its m0 step)
  double grf[3] = {0.0, 0.0, 0.0};
  if (q == 0) {
    KS krf;
    kernel_strain(a, R, geo.mrf, geo.mlow_rf, geo.mupp_rf, wRnor, aRnor, &krf);
#pragma unroll
    for (int L = 0; L < 3; L++) grf[L] = krf.g[L];
  }

  // Phase 5: inward walk (RadialShell.jl:566-699) from the crossing m0.  At
  // mp = 1 the reference's running window is [2, last shell with rad < 2].
  const int hi1 = last_lt(rad, 2, m, 2.0);
  const int m0o = h.m0;
  int m0 = m0o;
  KS prev, last, carry;
  double zcarry = -1.0, zvir1 = -1.0, zvir1p = -1.0, lastFh = 0.0;
  bool collapsed = false;
  long long steps = 0;
  for (int base = 0;; base += QT) {
    const int st = base + q, mp = m0o - st;
    const bool act = mp >= 1;
    KS cur = {};
    double zv = -1.0, Fh = 0.0;
    if (act) {
      kernel_strain(a, R, mp, 2, mp > 1 ? m : hi1, wRnor, aRnor, &cur);
      steps++;
      if (st >= 1) {
        double ev, pv;
        ev_pv(cur.E, &Fh, &ev, &pv);
        zv = zvir_of(a.tab, R.get(R_FBAR, mp), ev, pv);
      }
    }
    const bool hit = act && st >= 1 && zv >= ZZon;
    {
      const unsigned bal = (__ballot_sync(qmask, hit) >> qbase) & ((1u << QT) - 1u);
      if (bal) {
        const int qs = __ffs(bal) - 1;
        last = shfl_ks(cur, qbase + qs, qmask);
        lastFh = __shfl_sync(qmask, Fh, qbase + qs);
        zvir1p = __shfl_sync(qmask, zv, qbase + qs);
        const int ql = qs > 0 ? qs - 1 : 0;
        const KS left = shfl_ks(cur, qbase + ql, qmask);
        const double zl = __shfl_sync(qmask, zv, qbase + ql);
        prev = qs > 0 ? left : carry;
        zvir1 = qs > 0 ? zl : zcarry;
        m0 = m0o - (base + qs) + 1;
        collapsed = true;
        break;
      }
      if (m0o - (base + QT - 1) <= 1) break;   // walked down to mp = 1
      carry = shfl_ks(cur, qbase + QT - 1, qmask);
      zcarry = __shfl_sync(qmask, zv, qbase + QT - 1);
    }
  }
  atomicAdd(a.counters + CNT_WALK, (unsigned long long)steps);
  if (q != 0) return;
  if (!collapsed) {
    atomicAdd(a.counters + CNT_NOCOLL, 1ull);
    write_no_collapse(out);
    return;
  }

  collapse_finish(a, R, ZZon, m0, zvir1, zvir1p, prev, last, lastFh, grf, out);
}

// the peak of collapse slot i: i itself, or its place in the collapse order
__device__ __forceinline__ int64_t collapse_peak(const ShellArgs& a, int64_t i) {
  return a.corder ? (int64_t)__ldg(a.corder + i) : i;
}

__global__ void __launch_bounds__(128) collapse1_kernel(ShellArgs a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.npk) collapse_one(a, collapse_peak(a, i));
}

template <int QT>
__global__ void __launch_bounds__(128) collapse_kernel(ShellArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = t / QT;
  const int lane = threadIdx.x & 31, q = lane & (QT - 1), qbase = lane & ~(QT - 1);
  if (i < a.npk) collapse_group<QT>(a, collapse_peak(a, i), q, qbase, ((1u << QT) - 1u) << qbase);
}

// collapse order key (thread per peak): peaks that reach the walk by
// descending crossing shell m0 — the longest windows and walks first, and
// peaks of similar walks side by side in a warp — the rest last
__global__ void corder_kernel(ShellArgs a, uint32_t* key, int32_t* idx) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.npk) return;
  const PeakHdr h = a.hdr[p];
  key[p] = h.status == HS_OK ? 0xffffu - (uint32_t)min(max(h.m0, 0), 0xffff) : 0x1ffffu;
  idx[p] = (int32_t)p;
}

// One thread per peak with a work queue per lane: a lane takes its next peak
// from the batch as soon as its walk ends (the warp's idle lanes take theirs
// with one atomic), so that short and long walks share warps instead of
// lanes idling behind the longest walk of their warp.  Every loop round each
// busy lane evaluates exactly one kernel_strain, at one program point: the
// filter-scale window of phase 3, the crossing shell m0, or the next step of
// the inward walk; the rest of a round is the step's small bookkeeping.
// Per peak the arithmetic is collapse_one's, in the same order.
__global__ void __launch_bounds__(128) collapseq_kernel(ShellArgs a) {
  const int lane = threadIdx.x & 31;
  const double anor = 1.0;
  const double aRnor = 3.0 * anor / a.alatt, wnor = anor / (4.0 * 3.141592653589793), wRnor = 3.0 * wnor / a.alatt;
  const double* __restrict__ rad = a.rad;
  int state = 0;   // 0 idle, 1 filter-scale strain next, 2 crossing-shell strain next, 3 walking
  bool retired = false;
  int64_t p = 0;
  Rows R{a.pool, 0, a.counters};
  double ZZon = 0.0;
  int m = 1, hi1 = 1, m0 = 1, mp = 1, mrf = 1, mlo = 1, mup = 1;
  long long steps = 0;
  double grf[3] = {0.0, 0.0, 0.0}, zprev = -1.0;
  KS prev = {};
  while (true) {
    const bool want = state == 0 && !retired;
    const unsigned wb = __ballot_sync(FULL, want);
    if (wb) {
      const int leader = __ffs(wb) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(a.cqueue, __popc(wb));
      base = __shfl_sync(FULL, base, leader);
      if (want) {
        const int q = base + __popc(wb & ((1u << lane) - 1u));
        if (q >= a.npk) {
          retired = true;
        } else {
          p = collapse_peak(a, q);
          const PeakHdr h = a.hdr[p];
          if (h.status != HS_OK) {
            write_no_collapse(a.out + p * RES_N);   // state stays 0: the lane takes another peak
          } else {
            R = Rows{a.pool + h.off * ROW, h.mdone, a.counters};
            ZZon = a.pk.ZZon[p];
            m = a.mlim[p];
            const int4 gq = a.geo[2 * p];
            mrf = gq.y; mlo = gq.z; mup = gq.w;
            hi1 = last_lt(rad, 2, m, 2.0);
            m0 = h.m0;
            state = 1;
          }
        }
      }
    }
    if (__ballot_sync(FULL, state != 0 || !retired) == 0) break;
    if (state == 0) continue;
    int c, lo, hi;
    if (state == 1) { c = mrf; lo = mlo; hi = mup; }
    else if (state == 2) { c = m0; lo = 2; hi = m0 > 1 ? m : hi1; }
    else { c = mp; lo = 2; hi = mp > 1 ? m : hi1; }
    KS cur;
    kernel_strain(a, R, c, lo, hi, wRnor, aRnor, &cur);
    if (state == 1) {          // Phase 3: gradient at the filter scale
#pragma unroll
      for (int L = 0; L < 3; L++) grf[L] = cur.g[L];
      state = 2;
    } else if (state == 2) {   // the crossing shell's strain; the walk starts below it
      prev = cur;
      zprev = -1.0;
      steps = 1;
      mp = m0 - 1;
      state = 3;
      if (mp < 1) {
        atomicAdd(a.counters + CNT_WALK, (unsigned long long)steps);
        atomicAdd(a.counters + CNT_NOCOLL, 1ull);
        write_no_collapse(a.out + p * RES_N);
        state = 0;
      }
    } else {                   // Phase 5: one inward step
      steps++;
      double Fh, ev, pv;
      ev_pv(cur.E, &Fh, &ev, &pv);
      const double zv = zvir_of(a.tab, R.get(R_FBAR, mp), ev, pv);
      if (zv >= ZZon) {
        atomicAdd(a.counters + CNT_WALK, (unsigned long long)steps);
        collapse_finish(a, R, ZZon, mp + 1, zprev, zv, prev, cur, Fh, grf, a.out + p * RES_N);
        state = 0;
      } else if (mp == 1) {
        atomicAdd(a.counters + CNT_WALK, (unsigned long long)steps);
        atomicAdd(a.counters + CNT_NOCOLL, 1ull);
        write_no_collapse(a.out + p * RES_N);
        state = 0;
      } else {
        prev = cur;
        zprev = zv;
        mp--;
      }
    }
  }
}

// ===========================================================================
// zvir_half kernel (RadialShell.jl:825-885): for halos with RTHL >= 3 cells,
// the largest zvir - 1 over ten radii RTHL ((e/9)/2 + 1/2)^(1/3), e = 0..9,
// each from kernel_strain on [first shell beyond rcur - 2, first shell beyond
// rcur + 2] around the first shell beyond rcur.  Sixteen threads per peak,
// ten of them with a radius.
// ===========================================================================
__global__ void __launch_bounds__(128) zhalf_kernel(ShellArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t p = t >> 4;
  const int e = (int)(t & 15);
  const double hlatt = 1.0;
  double zl = -1.0;
  bool act = false;
  if (p < a.npk) {
    const double RTHL = a.out[p * RES_N];
    act = RTHL / hlatt >= 3.0;
    if (act && e < 10) {
      const PeakHdr h = a.hdr[p];
      const Rows R{a.pool + h.off * ROW, h.mdone, a.counters};
      const double* __restrict__ rad = a.rad;
      const int m = a.mlim[p];
      const double alatt = a.alatt, anor = 1.0;
      const double aRnor = 3.0 * anor / alatt, wRnor = 3.0 * (anor / (4.0 * 3.141592653589793)) / alatt;
      const double rcur = RTHL * a.fhalf[e];
      // first m1 in [2, m-1] with rad > rcur + 2 (the loop's break), else m-1
      const int fu = first_gt(rad, 2, m - 1, rcur + 2.0 * hlatt);
      const int mupp_rc = fu <= m - 1 ? fu : (m - 1 >= 2 ? m - 1 : 1);
      int mlow_rc = 1;
      const int fl = first_gt(rad, 1, m - 1, fmax(rcur - 2.0 * hlatt, 0.0));
      if (fl <= m - 1) mlow_rc = fl;
      const int f0 = first_gt(rad, 1, m - 1, rcur);
      const int m0_rc = (f0 <= m - 1) ? f0 : max(m - 1, 1);
      KS krc;
      kernel_strain(a, R, m0_rc, mlow_rc, mupp_rc, wRnor, aRnor, &krc);
      double Fr, ev, pv;
      ev_pv(krc.E, &Fr, &ev, &pv);
      zl = zvir_of(a.tab, R.get(R_FBAR, m0_rc), ev, pv) - 1.0;
    }
  }
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) zl = fmax(zl, __shfl_xor_sync(FULL, zl, o));
  if (act && e == 0) a.out[p * RES_N + 26] = fmax(zl, -1.0);
}

// ===========================================================================
// d2F kernel (one warp per collapsed peak, grid-stride)
// ===========================================================================
// mean lapd over the cells (centre excluded) with sqrt(r2) <= RTHL, in list
// order, stopping at the first out-of-grid cell (RadialShell.jl:805-819).
// The cells with sqrt(r2) <= RTHL are a prefix of the sorted list: the cells
// before the first shell with rad > RTHL.
__global__ void __launch_bounds__(128) d2f_kernel(ShellArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int n = a.n;
  const int64_t n2 = (int64_t)n * n;
  for (int64_t p = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); p < a.npk; p += nwarps) {
    double* out = a.out + p * RES_N;
    const double RTHL = out[0];
    if (!(RTHL > 0.0)) continue;
    const int64_t lin = a.pk.lin[p];
    const int pk = (int)(lin / n2), pj = (int)((lin / n) % n), pi = (int)(lin % n);
    const int mR = first_gt(a.rad, 1, a.nshell, RTHL);   // 1-based shell; distinct r2 index mR - 1
    int64_t cend = mR <= a.nshell ? (int64_t)__ldg(a.sh_start + mR - 1) : a.npart;
    if (a.npcap) cend = min(cend, (int64_t)a.npcap[p]);   // jp = 2..npart (RadialShell.jl:805-819)
    double acc = 0.0;
    long long navg = 0;
    for (int64_t c0 = 1; c0 < cend; c0 += 32) {
      const int64_t c = c0 + lane;
      bool valid = false, oob = false;
      float v = 0.f;
      if (c < cend) {
        int di, dj, dk;
        unpack_cell(__ldg(a.cell8 + c), di, dj, dk);
        const int iv1 = pi + di, iv2 = pj + dj, iv3 = pk + dk;
        if (iv1 < 0 || iv1 >= n || iv2 < 0 || iv2 >= n || iv3 < 0 || iv3 >= n) oob = true;
        else { valid = true; v = __ldg(a.lapd + iv1 + (int64_t)n * iv2 + n2 * iv3); }
      }
      const unsigned ob = __ballot_sync(FULL, oob);
      if (ob && lane >= __ffs(ob) - 1) valid = false;
      if (valid) { acc += (double)v; navg++; }
      if (ob) break;
    }
    acc = warp_sum(acc);
    navg = warp_sum_ll(navg);
    if (lane == 0) out[30] = navg > 0 ? acc / (double)navg : 0.0;
  }
}

// ===========================================================================
// mask writes (one warp per collapsed peak, grid-stride)
// ===========================================================================
// mask := 1 at the cells of the list (cells 1..npart) with sqrt(r2) <= RTHL
// that lie in the interior nbuff+1 .. n-nbuff on every axis
// (RadialShell.jl:793-802); the cells within RTHL are a prefix of the list.
__global__ void __launch_bounds__(128) mask_kernel(ShellArgs a, uint8_t* mask, int nbuff) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int n = a.n;
  const int64_t n2 = (int64_t)n * n;
  for (int64_t p = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); p < a.npk; p += nwarps) {
    const double RTHL = a.out[p * RES_N];
    if (!(RTHL > 0.0)) continue;
    const int64_t lin = a.pk.lin[p];
    const int pk = (int)(lin / n2), pj = (int)((lin / n) % n), pi = (int)(lin % n);
    const int mR = first_gt(a.rad, 1, a.nshell, RTHL);
    int64_t cend = mR <= a.nshell ? (int64_t)__ldg(a.sh_start + mR - 1) : a.npart;
    if (a.npcap) cend = min(cend, (int64_t)a.npcap[p]);
    for (int64_t c = lane; c < cend; c += 32) {
      int di, dj, dk;
      unpack_cell(__ldg(a.cell8 + c), di, dj, dk);
      const int iv1 = pi + di, iv2 = pj + dj, iv3 = pk + dk;
      if (iv1 < nbuff || iv1 >= n - nbuff || iv2 < nbuff || iv2 >= n - nbuff || iv3 < nbuff || iv3 >= n - nbuff)
        continue;
      mask[iv1 + (int64_t)n * iv2 + n2 * iv3] = 1;
    }
  }
}

}  // namespace

void launch_shell_mask(Launch L, const ShellArgs& a, uint8_t* mask, int nbuff, int blocks) {
  if (a.npk == 0) return;
  mask_kernel<<<blocks, 128, 0, L.s>>>(a, mask, nbuff);
  PPB_LAUNCHED(*L.count);
}

int64_t shell_stage_doubles_per_warp(int nshell) { return (int64_t)ROW * (nshell + 1); }

constexpr size_t kGatherSmem = (size_t)kGatherWarps * GATHER_WARP_DOUBLES * sizeof(double);

int shell_gather_blocks_per_sm(bool comp, bool adaptive) {
  const void* fs[2][2][2] = {
      {{(const void*)gather_kernel<false, false, SRC_LDG>, (const void*)gather_kernel<false, false, SRC_TEX>},
       {(const void*)gather_kernel<false, true, SRC_LDG>, (const void*)gather_kernel<false, true, SRC_TEX>}},
      {{(const void*)gather_kernel<true, false, SRC_LDG>, (const void*)gather_kernel<true, false, SRC_TEX>},
       {(const void*)gather_kernel<true, true, SRC_LDG>, (const void*)gather_kernel<true, true, SRC_TEX>}}};
  for (int t = 0; t < 2; t++)
    PPB_CUDA(cudaFuncSetAttribute(fs[comp][adaptive][t], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kGatherSmem));
  const void* f = fs[comp][adaptive][0];
  int b = 0;
  PPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, 32 * kGatherWarps, kGatherSmem));
  return b > 0 ? b : 1;
}

void launch_shell_anchors(Launch L, const ShellArgs& a) {
  if (a.nck == 0) return;
  anchor_kernel<<<(a.nck + 127) / 128, 128, 0, L.s>>>(a);
  PPB_LAUNCHED(*L.count);
}

void launch_collapse_order_keys(Launch L, const ShellArgs& a, uint32_t* key, int32_t* idx) {
  const int64_t blocks = (a.npk + 127) / 128;
  if (blocks == 0) return;
  corder_kernel<<<(unsigned)blocks, 128, 0, L.s>>>(a, key, idx);
  PPB_LAUNCHED(*L.count);
}

void launch_shell_geo(Launch L, const ShellArgs& a, uint32_t* key, int32_t* idx) {
  const int64_t blocks = (a.npk + 127) / 128;
  if (blocks == 0) return;
  geo_kernel<<<(unsigned)blocks, 128, 0, L.s>>>(a, key, idx);
  PPB_LAUNCHED(*L.count);
}

constexpr size_t kGatherRingSmem = (size_t)kGatherWarps * kRingWarpBytes + kGatherSmem;

int shell_gather_ring_blocks_per_sm(bool comp, bool adaptive) {
  const void* f = comp ? (adaptive ? (const void*)gather_ring_kernel<true, true>
                                   : (const void*)gather_ring_kernel<true, false>)
                       : (adaptive ? (const void*)gather_ring_kernel<false, true>
                                   : (const void*)gather_ring_kernel<false, false>);
  PPB_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGatherRingSmem));
  int b = 0;
  PPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, 32 * kGatherWarps, kGatherRingSmem));
  return b > 0 ? b : 1;
}

void launch_shell_gather(Launch L, const ShellArgs& a, bool comp, bool adaptive, int blocks, const void* ring_map) {
  const dim3 grid(blocks), block(32 * kGatherWarps);
  if (ring_map) {
    const CUtensorMap& tm = *static_cast<const CUtensorMap*>(ring_map);
    const size_t rs = kGatherRingSmem;
    if (comp && adaptive) gather_ring_kernel<true, true><<<grid, block, rs, L.s>>>(a, tm);
    else if (comp) gather_ring_kernel<true, false><<<grid, block, rs, L.s>>>(a, tm);
    else if (adaptive) gather_ring_kernel<false, true><<<grid, block, rs, L.s>>>(a, tm);
    else gather_ring_kernel<false, false><<<grid, block, rs, L.s>>>(a, tm);
    PPB_LAUNCHED(*L.count);
    return;
  }
  const size_t sm = kGatherSmem;
  if (a.rec_tex) {
    if (comp && adaptive) gather_kernel<true, true, SRC_TEX><<<grid, block, sm, L.s>>>(a);
    else if (comp) gather_kernel<true, false, SRC_TEX><<<grid, block, sm, L.s>>>(a);
    else if (adaptive) gather_kernel<false, true, SRC_TEX><<<grid, block, sm, L.s>>>(a);
    else gather_kernel<false, false, SRC_TEX><<<grid, block, sm, L.s>>>(a);
  } else {
    if (comp && adaptive) gather_kernel<true, true, SRC_LDG><<<grid, block, sm, L.s>>>(a);
    else if (comp) gather_kernel<true, false, SRC_LDG><<<grid, block, sm, L.s>>>(a);
    else if (adaptive) gather_kernel<false, true, SRC_LDG><<<grid, block, sm, L.s>>>(a);
    else gather_kernel<false, false, SRC_LDG><<<grid, block, sm, L.s>>>(a);
  }
  PPB_LAUNCHED(*L.count);
}

bool record_ring_map(const float4* aos, int n, void* map128) {
  const uint64_t cells = (uint64_t)n * n * n;
  if (n <= 0 || cells >= (1ull << 31)) return false;
  using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static Encode encode = nullptr;
  static bool looked = false;
  if (!looked) {
    looked = true;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      encode = reinterpret_cast<Encode>(fn);
    cudaGetLastError();
  }
  if (!encode) return false;
  // rows of 8 floats (one 32-byte record), one row per box
  const cuuint64_t dims[2] = {8, cells};
  const cuuint64_t strides[1] = {32};
  const cuuint32_t box[2] = {8, 1};
  const cuuint32_t estr[2] = {1, 1};
  return encode(static_cast<CUtensorMap*>(map128), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float4*>(aos), dims,
                strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int shell_collapseq_blocks(int nsm) {
  static int per_sm = 0;
  if (per_sm == 0) {
    int b = 0;
    PPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, collapseq_kernel, 128, 0));
    per_sm = b > 0 ? b : 1;
  }
  return nsm * per_sm;
}

int shell_collapse_width(int64_t npk, int nsm, double walk_steps_per_peak) {
  // 4 threads per peak while 4 per peak still fit about 24 warps per SM or
  // when walks are long (more than 8 steps per peak in the previous batch:
  // the lightcone), else 2 or 1 (the device is full and the latency hidden)
  const int64_t full = (int64_t)nsm * 24 * 32;
  if (walk_steps_per_peak > 8.0 || npk * 4 <= full) return 4;
  return npk * 2 <= full ? 2 : 1;
}

void launch_shell_collapse(Launch L, const ShellArgs& a, int nsm, double walk_steps_per_peak, int threads_per_peak) {
  int w = threads_per_peak;
  if (w == 8) {   // one thread per peak, lane work queues (persistent grid)
    if (a.npk == 0) return;
    PPB_CUDA(cudaMemsetAsync(a.cqueue, 0, sizeof(int), L.s));
    const int64_t blocks = std::min<int64_t>(shell_collapseq_blocks(nsm), (a.npk + 127) / 128);
    collapseq_kernel<<<(unsigned)blocks, 128, 0, L.s>>>(a);
    PPB_LAUNCHED(*L.count);
    return;
  }
  if (w != 1 && w != 2 && w != 4) w = shell_collapse_width(a.npk, nsm, walk_steps_per_peak);
  const int lg = w == 4 ? 2 : w - 1;
  const int64_t blocks = ((a.npk << lg) + 127) / 128;
  if (blocks == 0) return;
  if (w == 4) collapse_kernel<4><<<(unsigned)blocks, 128, 0, L.s>>>(a);
  else if (w == 2) collapse_kernel<2><<<(unsigned)blocks, 128, 0, L.s>>>(a);
  else collapse1_kernel<<<(unsigned)blocks, 128, 0, L.s>>>(a);
  PPB_LAUNCHED(*L.count);
}

void launch_shell_zhalf(Launch L, const ShellArgs& a) {
  const int64_t blocks = (a.npk * 16 + 127) / 128;
  if (blocks == 0) return;
  zhalf_kernel<<<(unsigned)blocks, 128, 0, L.s>>>(a);
  PPB_LAUNCHED(*L.count);
}

void launch_shell_d2f(Launch L, const ShellArgs& a, int blocks) {
  if (a.npk == 0 || !a.lapd) return;
  d2f_kernel<<<blocks, 128, 0, L.s>>>(a);
  PPB_LAUNCHED(*L.count);
}

}  // namespace ppb
