// noalloc.cu — find_peaks without any device allocation.
//
// Some callers cannot allocate device memory at the point where they need the
// peak finder: their GPU memory is owned by another runtime's pool (a Julia
// CUDA.jl or PyTorch caching allocator that has already reserved the device),
// or they run a fixed-footprint service loop where cudaMalloc/cudaFree -- which
// synchronise the device and can fail with out-of-memory -- are not allowed.
// ppb_find_peaks_noalloc serves them: the caller passes device buffers for
// every input and output, and the only scratch the kernels need (per-block
// peak counts and their prefix offsets for an ordered compaction) lives in the
// file-scope array below, so the call allocates nothing.
//
// Limits and behaviour (stated for users of the entry point):
//  * the scratch holds counts and offsets for at most kMaxBlocks blocks of
//    kCellsPerBlock cells, i.e. an inner cube of at most 268,435,456 cells
//    (about 645^3); larger inputs are rejected with PPB_ERR_INVALID;
//  * every GPU that loads the library keeps this 2 MiB array until the
//    process exits;
//  * the array is shared by all calls on a device and keeps the last call's
//    contents; calls that overlap on the GPU (different streams or
//    contexts on the same device) race on it and must be serialised by the
//    caller;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress); make that first call before any stream capture.
//
// Semantics are those of find_peaks (src/HaloFinder/PeakFind.jl:15-79) and
// of ppb_find_peaks: scan order k, j, i; the first max(max_peaks, 1) peaks
// are reported and masked, later ones are neither (the reference pushes a
// peak before it compares the count with max_peaks, :66-71).  Every buffer
// must be device memory of the context's own GPU.
#include <mutex>

#include "ppb_ctx.h"

namespace ppb {
namespace {

constexpr int kThreads = 256;
constexpr int kCellsPerThread = 4;
constexpr int kCellsPerBlock = kThreads * kCellsPerThread;   // 1024
constexpr int kMaxBlocks = 1 << 18;

// [0, kMaxBlocks): per-block counts; [kMaxBlocks, 2 kMaxBlocks): offsets;
// [2 kMaxBlocks]: total
static __device__ __align__(256) unsigned int g_noalloc_scratch[2 * kMaxBlocks + 64];

std::mutex g_sym_mu;
unsigned int* g_sym_addr[64] = {};   // device address of the array, per device

struct Grid3 {
  int n1, n2, n3, nbuff, w1, w2, w3;
};

// is cell t (inner-cube linear index, i fastest) a peak?  Same test as
// peakfind_kernel: not masked, not below fcrit, no neighbour strictly larger.
__device__ __forceinline__ bool is_peak(const float* __restrict__ d, const int8_t* __restrict__ mask, const Grid3& g,
                                        float fcrit, int64_t t, int64_t* lin_out, float* ff_out) {
  const int64_t plane = (int64_t)g.w1 * g.w2;
  const int k = (int)(t / plane);
  const int64_t r = t - (int64_t)k * plane;
  const int j = (int)(r / g.w1);
  const int i = (int)(r - (int64_t)j * g.w1);
  const int64_t n12 = (int64_t)g.n1 * g.n2;
  const int64_t lin = (i + g.nbuff) + (int64_t)g.n1 * (j + g.nbuff) + n12 * (k + g.nbuff);
  *lin_out = lin;
  const float ff = d[lin];
  *ff_out = ff;
  if (mask[lin] == 1 || ff < fcrit) return false;
  bool pk = true;
#pragma unroll
  for (int dk = -1; dk <= 1; dk++)
#pragma unroll
    for (int dj = -1; dj <= 1; dj++)
#pragma unroll
      for (int di = -1; di <= 1; di++)
        if (ff < __ldg(d + lin + di + (int64_t)g.n1 * dj + n12 * dk)) pk = false;
  return pk;
}

__device__ __forceinline__ int block_exclusive_scan(int v, int* total) {
  __shared__ int warp_tot[kThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = lane < kThreads / 32 ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kThreads / 32) warp_tot[lane] = s;   // inclusive
  }
  __syncthreads();
  const int before = (w > 0 ? warp_tot[w - 1] : 0) + x - v;
  *total = warp_tot[kThreads / 32 - 1];
  __syncthreads();
  return before;
}

// pass 1: peaks per block
__global__ void __launch_bounds__(kThreads) count_kernel(const float* __restrict__ d, const int8_t* __restrict__ mask,
                                                         Grid3 g, float fcrit, int64_t ninner,
                                                         unsigned int* scratch) {
  const int64_t base = (int64_t)blockIdx.x * kCellsPerBlock + (int64_t)threadIdx.x * kCellsPerThread;
  int c = 0;
  for (int q = 0; q < kCellsPerThread; q++) {
    const int64_t t = base + q;
    int64_t lin;
    float ff;
    if (t < ninner && is_peak(d, mask, g, fcrit, t, &lin, &ff)) c++;
  }
  int tot;
  block_exclusive_scan(c, &tot);
  if (threadIdx.x == 0) scratch[blockIdx.x] = (unsigned int)tot;
}

// pass 2: exclusive prefix of the block counts (one block) and the total
__global__ void __launch_bounds__(kThreads) scan_kernel(unsigned int* scratch, int nblocks) {
  unsigned int* counts = scratch;
  unsigned int* offs = scratch + kMaxBlocks;
  int carry = 0;
  for (int b0 = 0; b0 < nblocks; b0 += kThreads) {
    const int b = b0 + threadIdx.x;
    const int v = b < nblocks ? (int)counts[b] : 0;
    int tot;
    const int ex = block_exclusive_scan(v, &tot);
    if (b < nblocks) offs[b] = (unsigned int)(carry + ex);
    carry += tot;
  }
  if (threadIdx.x == 0) scratch[2 * kMaxBlocks] = (unsigned int)carry;
}

// pass 3: ordered write of the first max_peaks peaks, and their mask
__global__ void __launch_bounds__(kThreads) write_kernel(const float* __restrict__ d, int8_t* mask, Grid3 g,
                                                         float fcrit, int64_t ninner, int64_t max_peaks,
                                                         const unsigned int* scratch, int64_t* pi, int64_t* pj,
                                                         int64_t* pk, int64_t* ipp, float* pd) {
  const int64_t base = (int64_t)blockIdx.x * kCellsPerBlock + (int64_t)threadIdx.x * kCellsPerThread;
  bool flag[kCellsPerThread];
  int64_t lins[kCellsPerThread];
  float ffs[kCellsPerThread];
  int c = 0;
  for (int q = 0; q < kCellsPerThread; q++) {
    const int64_t t = base + q;
    flag[q] = t < ninner && is_peak(d, mask, g, fcrit, t, &lins[q], &ffs[q]);
    c += flag[q] ? 1 : 0;
  }
  int tot;
  int rank = (int)scratch[kMaxBlocks + blockIdx.x] + block_exclusive_scan(c, &tot);
  const int64_t n12 = (int64_t)g.n1 * g.n2;
  for (int q = 0; q < kCellsPerThread; q++) {
    if (!flag[q]) continue;
    if (rank < max_peaks) {
      const int64_t lin = lins[q];
      pi[rank] = lin % g.n1 + 1;
      pj[rank] = (lin / g.n1) % g.n2 + 1;
      pk[rank] = lin / n12 + 1;
      ipp[rank] = lin + 1;
      pd[rank] = ffs[q];
      mask[lin] = 1;
    }
    rank++;
  }
}

}  // namespace
}  // namespace ppb

using namespace ppb;

extern "C" int32_t ppb_find_peaks_noalloc(ppb_ctx* ctx, const float* delta, int8_t* mask, int32_t n1, int32_t n2,
                                          int32_t n3, int32_t nbuff, float fcrit, int64_t max_peaks, int64_t* pi,
                                          int64_t* pj, int64_t* pk, int64_t* ipp, float* pdelta,
                                          int64_t* npeaks) {
  if (!ctx) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  try {
    PPB_REQUIRE(delta && mask && pi && pj && pk && ipp && pdelta && npeaks, "null argument");
    PPB_REQUIRE(n1 >= 3 && n2 >= 3 && n3 >= 3 && nbuff >= 1, "grid must be >= 3 cells with nbuff >= 1");
    PPB_CUDA(cudaSetDevice(ctx->device));
    for (const void* p : {(const void*)delta, (const void*)mask, (const void*)pi, (const void*)pj, (const void*)pk,
                          (const void*)ipp, (const void*)pdelta}) {
      PPB_REQUIRE(is_device_ptr(p), "ppb_find_peaks_noalloc needs device pointers for fields and outputs");
      cudaPointerAttributes at;
      PPB_CUDA(cudaPointerGetAttributes(&at, p));
      PPB_REQUIRE(at.type == cudaMemoryTypeManaged || at.device == ctx->device,
                  "ppb_find_peaks_noalloc: a buffer lives on another GPU than the context's");
    }
    const int64_t keep = max_peaks > 1 ? max_peaks : 1;   // at least the first peak (PeakFind.jl:66-71)
    const int w1 = n1 - 2 * nbuff, w2 = n2 - 2 * nbuff, w3 = n3 - 2 * nbuff;
    *npeaks = 0;
    if (w1 <= 0 || w2 <= 0 || w3 <= 0) return PPB_OK;
    const int64_t ninner = (int64_t)w1 * w2 * w3;
    const int64_t nblocks = (ninner + kCellsPerBlock - 1) / kCellsPerBlock;
    PPB_REQUIRE(nblocks <= kMaxBlocks, "inner cube larger than the no-allocation scratch allows (268,435,456 cells)");
    unsigned int* scratch;
    {
      std::lock_guard<std::mutex> g(g_sym_mu);
      PPB_REQUIRE(ctx->device >= 0 && ctx->device < 64, "device index too large");
      if (!g_sym_addr[ctx->device]) {   // once per device, with that device current
        void* ptr = nullptr;
        PPB_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        g_sym_addr[ctx->device] = static_cast<unsigned int*>(ptr);
      }
      scratch = g_sym_addr[ctx->device];
    }
    cudaStream_t s = ctx->sync.stream;
    const Grid3 g{n1, n2, n3, nbuff, w1, w2, w3};
    // the total slot is the only value read before this call writes it
    PPB_CUDA(cudaMemsetAsync(scratch + 2 * kMaxBlocks, 0, sizeof(unsigned int), s));
    count_kernel<<<(unsigned)nblocks, kThreads, 0, s>>>(delta, mask, g, fcrit, ninner, scratch);
    PPB_LAUNCHED(ctx->sync.launches);
    scan_kernel<<<1, kThreads, 0, s>>>(scratch, (int)nblocks);
    PPB_LAUNCHED(ctx->sync.launches);
    write_kernel<<<(unsigned)nblocks, kThreads, 0, s>>>(delta, mask, g, fcrit, ninner, keep, scratch, pi, pj, pk,
                                                       ipp, pdelta);
    PPB_LAUNCHED(ctx->sync.launches);
    unsigned int total = 0;
    PPB_CUDA(cudaMemcpyAsync(&total, scratch + 2 * kMaxBlocks, sizeof(total), cudaMemcpyDeviceToHost, s));
    PPB_CUDA(cudaStreamSynchronize(s));
    *npeaks = (int64_t)total < keep ? (int64_t)total : keep;
    return PPB_OK;
  } catch (const ppb::Error& e) {
    ctx->set_error(e.msg);
    return e.code;
  } catch (...) {
    ctx->set_error("unknown error");
    return PPB_ERR_INVALID;
  }
}
