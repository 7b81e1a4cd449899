// stubs.cu — stub-level entry points that mirror the reference's per-stage
// functions on caller-supplied inputs: find_peaks on one field and
// analyse_peak over a batch of peaks.  They share the kernels of run_tile.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "ppb_ctx.h"

using namespace ppb;

namespace {

__global__ void unmask_kernel(const unsigned long long* keys, int from, int to, uint8_t* mask) {
  const int q = from + blockIdx.x * blockDim.x + threadIdx.x;
  if (q < to) mask[(int64_t)(keys[q] & ((1ull << 40) - 1))] = 0;
}

__global__ void peaks_out_kernel(const unsigned long long* keys, const uint32_t* vals, const float* ff, int np,
                                 int n1, int n2, int64_t* pi, int64_t* pj, int64_t* pk, int64_t* ipp, float* pd) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= np) return;
  const int64_t lin = (int64_t)(keys[q] & ((1ull << 40) - 1));
  pi[q] = lin % n1 + 1;
  pj[q] = (lin / n1) % n2 + 1;
  pk[q] = lin / ((int64_t)n1 * n2) + 1;
  ipp[q] = lin + 1;
  pd[q] = ff[vals[q]];
}

__global__ void ipp_to_lin(const int64_t* ipp, int64_t* lin, const int64_t* ir2, int32_t* ir2o, int64_t np) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= np) return;
  lin[q] = ipp[q] - 1;
  ir2o[q] = (int32_t)ir2[q];
}

// per-peak parameters of one batch of analyse_peaks_gpu_cuda_multirf: the
// 1-based (i, j, k) to a flat index, the batch's Rf, ir2min and npart, the
// per-peak ZZon / fcrit or the scalars
__global__ void multirf_prep_kernel(const int32_t* pi, const int32_t* pj, const int32_t* pk, int64_t q0, int64_t nq,
                                    int n, double Rf, int ir2, int np, const double* Zpp, const double* fpp, double Z,
                                    double fc, int64_t* lin, double* oRf, int32_t* oir2, int32_t* onp, double* oZ,
                                    double* ofc) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nq) return;
  const int64_t q = q0 + t;
  const int i = pi[q], j = pj[q], k = pk[q];
  const bool ok = i >= 1 && i <= n && j >= 1 && j <= n && k >= 1 && k <= n;
  lin[q] = ok ? (int64_t)(i - 1) + (int64_t)n * (j - 1) + (int64_t)n * n * (k - 1) : -1;   // -1: invalid peak
  oRf[q] = Rf;
  oir2[q] = ir2;
  onp[q] = np;
  oZ[q] = Zpp ? Zpp[q] : Z;
  ofc[q] = fpp ? fpp[q] : fc;
}

// the rmax2rs pre-mask test (RadialShell.jl:310-316) against the mask as it
// stands before the batch: skip[q] = 1 for a masked peak
__global__ void premask_kernel(const int64_t* lin, int64_t q0, int64_t nq, const uint8_t* mask, int thr,
                               int32_t* skip) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nq) return;
  const int64_t l = lin[q0 + t];
  skip[t] = (l >= 0 && (int)mask[l] > thr) ? 1 : 0;
}

// no_collapse() (RadialShell.jl:90-94) for the skipped peaks
__global__ void skip_out_kernel(const int32_t* skip, int64_t nq, double* out) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nq || !skip[t]) return;
  double* o = out + t * RES_N;
  for (int v = 0; v < RES_N; v++) o[v] = 0.0;
  o[0] = -1.0;
  o[26] = -1.0;
}

}  // namespace

extern "C" {

int32_t ppb_find_peaks(ppb_ctx* ctx, const float* delta, int8_t* mask, int32_t n1, int32_t n2, int32_t n3,
                       int32_t nbuff, float fcrit, int64_t max_peaks, int64_t* pi, int64_t* pj, int64_t* pk,
                       int64_t* ipp, float* pdelta, int64_t* npeaks) {
  if (!ctx) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  try {
    PPB_REQUIRE(delta && mask && pi && pj && pk && ipp && pdelta && npeaks, "null argument");
    PPB_REQUIRE(n1 >= 3 && n2 >= 3 && n3 >= 3 && nbuff >= 1, "grid must be >= 3 cells with nbuff >= 1");
    PPB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->sync.stream;
    const int64_t N = (int64_t)n1 * n2 * n3;
    PPB_REQUIRE(N < (1ll << 40), "grid too large");
    DevBuf d_delta, d_mask, keys, vals, ff, cnt, keys_s, vals_s, tmp, o_i, o_j, o_k, o_ipp, o_d;
    const float* dd = (const float*)[&]() -> const void* {
      if (is_device_ptr(delta)) return delta;
      d_delta.ensure(N * 4);
      PPB_CUDA(cudaMemcpyAsync(d_delta.p, delta, N * 4, cudaMemcpyHostToDevice, s));
      return d_delta.p;
    }();
    const bool mask_dev = is_device_ptr(mask);
    uint8_t* dm = (uint8_t*)mask;
    if (!mask_dev) {
      d_mask.ensure(N);
      PPB_CUDA(cudaMemcpyAsync(d_mask.p, mask, N, cudaMemcpyHostToDevice, s));
      dm = d_mask.as<uint8_t>();
    }
    // every cell of the inner cube can be a peak (ties are not rejected)
    const int64_t w1 = std::max(0, n1 - 2 * nbuff), w2 = std::max(0, n2 - 2 * nbuff), w3 = std::max(0, n3 - 2 * nbuff);
    const int64_t cap = std::max<int64_t>(1, w1 * w2 * w3);
    PPB_REQUIRE(cap < (1ll << 31), "inner cube too large for one call");
    keys.ensure(cap * 8);
    vals.ensure(cap * 4);
    ff.ensure(cap * 4);
    cnt.ensure(64);
    PPB_CUDA(cudaMemsetAsync(cnt.p, 0, 64, s));
    PeakBuf pb{keys.as<unsigned long long>(), vals.as<uint32_t>(), ff.as<float>(), ff.as<float>(), cnt.as<int>(), cap};
    // the lapd sample slot aliases ff; nothing reads it here
    pb.lap = nullptr;
    DevBuf lapdummy;
    lapdummy.ensure(cap * 4);
    pb.lap = lapdummy.as<float>();
    launch_peakfind(Launch{s, &ctx->sync.launches}, dd, nullptr, dm, n1, n2, n3, n1, (int64_t)n1 * n2, nbuff, fcrit,
                    0ull, pb);
    int c = 0;
    PPB_CUDA(cudaMemcpyAsync(&c, cnt.p, 4, cudaMemcpyDeviceToHost, s));
    PPB_CUDA(cudaStreamSynchronize(s));
    int64_t np = c;
    if (np > 0) {
      keys_s.ensure(np * 8);
      vals_s.ensure(np * 4);
      size_t tb = 0;
      PPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.as<unsigned long long>(), keys_s.as<unsigned long long>(),
                                               vals.as<uint32_t>(), vals_s.as<uint32_t>(), (int)np, 0, 40, s));
      tmp.ensure(tb + 16);
      PPB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, keys.as<unsigned long long>(), keys_s.as<unsigned long long>(),
                                               vals.as<uint32_t>(), vals_s.as<uint32_t>(), (int)np, 0, 40, s));
      ctx->sync.launches++;
      // the reference stops scanning once max_peaks are found, testing the
      // count after each push (PeakFind.jl:66-71, so at least one peak):
      // later cells are neither reported nor masked
      const int64_t keep = max_peaks > 1 ? max_peaks : 1;
      if (np > keep) {
        const int from = (int)keep, to = (int)np;
        unmask_kernel<<<(to - from + 255) / 256, 256, 0, s>>>(keys_s.as<unsigned long long>(), from, to, dm);
        PPB_LAUNCHED(ctx->sync.launches);
        np = keep;
      }
      if (np > 0) {
        o_i.ensure(np * 8); o_j.ensure(np * 8); o_k.ensure(np * 8); o_ipp.ensure(np * 8); o_d.ensure(np * 4);
        peaks_out_kernel<<<(unsigned)((np + 255) / 256), 256, 0, s>>>(
            keys_s.as<unsigned long long>(), vals_s.as<uint32_t>(), ff.as<float>(), (int)np, n1, n2,
            o_i.as<int64_t>(), o_j.as<int64_t>(), o_k.as<int64_t>(), o_ipp.as<int64_t>(), o_d.as<float>());
        PPB_LAUNCHED(ctx->sync.launches);
        copy_out(pi, o_i.p, np * 8, s);
        copy_out(pj, o_j.p, np * 8, s);
        copy_out(pk, o_k.p, np * 8, s);
        copy_out(ipp, o_ipp.p, np * 8, s);
        copy_out(pdelta, o_d.p, np * 4, s);
      }
    }
    if (!mask_dev) copy_out(mask, d_mask.p, N, s);
    PPB_CUDA(cudaStreamSynchronize(s));
    *npeaks = np;
    return PPB_OK;
  } catch (const ppb::Error& e) {
    ctx->set_error(e.msg);
    return e.code;
  } catch (...) {
    ctx->set_error("unknown error");
    return PPB_ERR_INVALID;
  }
}

static int32_t analyse_peaks_impl(ppb_ctx* ctx, const float* delta, const float* etax, const float* etay,
                                  const float* etaz, const float* eta2x, const float* eta2y, const float* eta2z,
                                  const float* lapd, int32_t n, int32_t nhunt, int64_t npk, const int64_t* ipp,
                                  const double* Rf, const int64_t* ir2min, const double* ZZon, const double* fcrit,
                                  const int32_t* r2lim, double alatt, int32_t plain, double* out) {
  if (!ctx) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  try {
    PPB_REQUIRE(delta && etax && etay && etaz && ipp && Rf && ir2min && ZZon && fcrit && out, "null argument");
    PPB_REQUIRE((eta2x == nullptr) == (eta2y == nullptr) && (eta2y == nullptr) == (eta2z == nullptr),
                "eta2x/eta2y/eta2z must be all given or all null");
    PPB_REQUIRE(n >= 2 && n <= 4096, "n out of range");
    PPB_REQUIRE(npk >= 0 && npk < (1ll << 31), "npk out of range");
    PPB_REQUIRE(alatt > 0, "alatt must be positive");
    PPB_REQUIRE(ctx->sh.has_tab, "collapse table not set (ppb_set_collapse_table)");
    PPB_CUDA(cudaSetDevice(ctx->device));
    if (npk == 0) return PPB_OK;
    cudaStream_t s = ctx->sync.stream;
    Launch L{s, &ctx->sync.launches};
    const int64_t N = (int64_t)n * n * n;
    std::shared_lock<std::shared_mutex> rl(ctx->sh.mu);
    ShellTable& shells = ctx->shell_table(nhunt, s);
    // fields -> contiguous device staging -> packed gather records
    DevBuf st_delta, st_psi, st_psi2, st_lapd, aos, d_ipp, d_lin, d_Rf, d_ir2in, d_ir2, d_Z, d_fc, d_out, d_lim;
    st_psi.ensure(3 * N * 4);
    auto put = [&](DevBuf& b, size_t off, const float* src) {
      PPB_CUDA(cudaMemcpyAsync((char*)b.p + off, src, N * 4, cudaMemcpyDefault, s));
    };
    const float* dd = (const float*)stage_in(st_delta, delta, N * 4, s);
    put(st_psi, 0, etax);
    put(st_psi, N * 4, etay);
    put(st_psi, 2 * N * 4, etaz);
    const float* dpsi2 = nullptr;
    if (eta2x) {
      st_psi2.ensure(3 * N * 4);
      put(st_psi2, 0, eta2x);
      put(st_psi2, N * 4, eta2y);
      put(st_psi2, 2 * N * 4, eta2z);
      dpsi2 = st_psi2.as<float>();
    }
    const float* dl = lapd ? (const float*)stage_in(st_lapd, lapd, N * 4, s) : nullptr;
    aos.ensure(pack_bytes(n));
    launch_pack(L, aos.as<float4>(), FieldWindow{dd, st_psi.as<float>(), dpsi2, 0, n, (int64_t)n * n, N}, n);
    const int64_t* dipp = (const int64_t*)stage_in(d_ipp, ipp, npk * 8, s);
    const double* dRf = (const double*)stage_in(d_Rf, Rf, npk * 8, s);
    const int64_t* dir2 = (const int64_t*)stage_in(d_ir2in, ir2min, npk * 8, s);
    const double* dZ = (const double*)stage_in(d_Z, ZZon, npk * 8, s);
    const double* dfc = (const double*)stage_in(d_fc, fcrit, npk * 8, s);
    d_lin.ensure(npk * 8);
    d_ir2.ensure(npk * 4);
    ipp_to_lin<<<(unsigned)((npk + 255) / 256), 256, 0, s>>>(dipp, d_lin.as<int64_t>(), dir2, d_ir2.as<int32_t>(), npk);
    PPB_LAUNCHED(ctx->sync.launches);
    ShellArgs a = ctx->shell_args(ctx->sync, shells, n, alatt, aos.as<float4>(), dl);
    a.pk = PeakParams{d_lin.as<int64_t>(), dRf, d_ir2.as<int32_t>(), dZ, dfc};
    a.npk = npk;
    a.r2lim = r2lim ? (const int32_t*)stage_in(d_lim, r2lim, npk * 4, s) : nullptr;
    double* dout = out;
    if (!is_device_ptr(out)) {
      d_out.ensure(npk * RES_N * 8);
      dout = d_out.as<double>();
    }
    a.out = dout;
    ShellStats stt{};
    ctx->run_shells(ctx->sync, a, plain == 0, plain == 0, &stt);
    ctx->sync.last_visits = stt.visits;
    ctx->sync.last_npk = npk;
    if (stt.guard != 0)
      throw Error{PPB_ERR_CUDA, "shell truncation guard tripped: a profile read beyond the gathered shells"};
    if (stt.akk != 0)
      throw Error{PPB_ERR_INVALID, "kernel_strain SPH table index out of range (the reference raises here too)"};
    if (dout != out) copy_out(out, dout, npk * RES_N * 8, s);
    PPB_CUDA(cudaStreamSynchronize(s));
    return PPB_OK;
  } catch (const ppb::Error& e) {
    ctx->set_error(e.msg);
    return e.code;
  } catch (...) {
    ctx->set_error("unknown error");
    return PPB_ERR_INVALID;
  }
}

int32_t ppb_analyse_peaks(ppb_ctx* ctx, const float* delta, const float* etax, const float* etay,
                          const float* etaz, const float* eta2x, const float* eta2y, const float* eta2z,
                          const float* lapd, int32_t n, int32_t nhunt, int64_t npk, const int64_t* ipp,
                          const double* Rf, const int64_t* ir2min, const double* ZZon, const double* fcrit,
                          double alatt, int32_t plain, double* out) {
  return analyse_peaks_impl(ctx, delta, etax, etay, etaz, eta2x, eta2y, eta2z, lapd, n, nhunt, npk, ipp, Rf, ir2min,
                            ZZon, fcrit, nullptr, alatt, plain, out);
}

int32_t ppb_analyse_peaks_lim(ppb_ctx* ctx, const float* delta, const float* etax, const float* etay,
                              const float* etaz, const float* eta2x, const float* eta2y, const float* eta2z,
                              const float* lapd, int32_t n, int32_t nhunt, int64_t npk, const int64_t* ipp,
                              const double* Rf, const int64_t* ir2min, const double* ZZon, const double* fcrit,
                              const int32_t* r2lim, double alatt, int32_t plain, double* out) {
  return analyse_peaks_impl(ctx, delta, etax, etay, etaz, eta2x, eta2y, eta2z, lapd, n, nhunt, npk, ipp, Rf, ir2min,
                            ZZon, fcrit, r2lim, alatt, plain, out);
}

int32_t ppb_analyse_peaks_multirf(ppb_ctx* ctx, const float* delta, const float* etax, const float* etay,
                                  const float* etaz, const float* eta2x, const float* eta2y, const float* eta2z,
                                  const float* lapd, int32_t n, int32_t nhunt, int32_t nbatch, const int64_t* boff,
                                  const int32_t* pi, const int32_t* pj, const int32_t* pk, const double* Rf,
                                  const int64_t* ir2min, const double* ZZon_pp, const double* fcrit_pp, double ZZon,
                                  double fcrit, double alatt, int8_t* mask, int32_t nbuff, double rmax2rs,
                                  int32_t plain, double* out) {
  if (!ctx) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  try {
    PPB_REQUIRE(delta && etax && etay && etaz && boff && pi && pj && pk && Rf && ir2min && out, "null argument");
    PPB_REQUIRE((eta2x == nullptr) == (eta2y == nullptr) && (eta2y == nullptr) == (eta2z == nullptr),
                "eta2x/eta2y/eta2z must be all given or all null");
    PPB_REQUIRE(n >= 2 && n <= 4096, "n out of range");
    PPB_REQUIRE(nbatch >= 0 && nbatch <= 1 << 20, "nbatch out of range");
    PPB_REQUIRE(alatt > 0, "alatt must be positive");
    PPB_REQUIRE(nbuff >= 0 && 2 * nbuff < n, "nbuff must satisfy 0 <= nbuff and 2 nbuff < n");
    PPB_REQUIRE(rmax2rs >= 0.0 && rmax2rs <= 1e6, "rmax2rs must be in [0, 1e6]");
    PPB_REQUIRE((ZZon_pp == nullptr) == (fcrit_pp == nullptr), "ZZon_pp and fcrit_pp must be both given or both null");
    PPB_REQUIRE(ctx->sh.has_tab, "collapse table not set (ppb_set_collapse_table)");
    PPB_REQUIRE(boff[0] == 0, "boff[0] must be 0");
    for (int b = 0; b < nbatch; b++) {
      PPB_REQUIRE(boff[b + 1] >= boff[b], "boff must not decrease");
      PPB_REQUIRE(Rf[b] > 0.0, "Rf must be positive");
    }
    const int64_t npk = boff[nbatch];
    PPB_REQUIRE(npk < (1ll << 31), "too many peaks");
    PPB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->sync.stream;
    Launch L{s, &ctx->sync.launches};
    const int64_t N = (int64_t)n * n * n;
    std::shared_lock<std::shared_mutex> rl(ctx->sh.mu);
    ShellTable& shells = ctx->shell_table(nhunt, s);
    DevBuf st_delta, st_psi, st_psi2, st_lapd, aos, d_pi, d_pj, d_pk, d_Zpp, d_fpp, d_mask, d_out;
    DevBuf p_lin, p_Rf, p_ir2, p_np, p_Z, p_fc, p_skip;
    st_psi.ensure(3 * N * 4);
    auto put = [&](DevBuf& b, size_t off, const float* src) {
      PPB_CUDA(cudaMemcpyAsync((char*)b.p + off, src, N * 4, cudaMemcpyDefault, s));
    };
    const float* dd = (const float*)stage_in(st_delta, delta, N * 4, s);
    put(st_psi, 0, etax);
    put(st_psi, N * 4, etay);
    put(st_psi, 2 * N * 4, etaz);
    const float* dpsi2 = nullptr;
    if (eta2x) {
      st_psi2.ensure(3 * N * 4);
      put(st_psi2, 0, eta2x);
      put(st_psi2, N * 4, eta2y);
      put(st_psi2, 2 * N * 4, eta2z);
      dpsi2 = st_psi2.as<float>();
    }
    const float* dl = lapd ? (const float*)stage_in(st_lapd, lapd, N * 4, s) : nullptr;
    uint8_t* dm = nullptr;
    if (mask) {
      d_mask.ensure(N);
      PPB_CUDA(cudaMemcpyAsync(d_mask.p, mask, N, cudaMemcpyDefault, s));
      dm = d_mask.as<uint8_t>();
    }
    aos.ensure(pack_bytes(n));
    launch_pack(L, aos.as<float4>(), FieldWindow{dd, st_psi.as<float>(), dpsi2, 0, n, (int64_t)n * n, N}, n);
    if (npk > 0) {
      const int32_t* dpi = (const int32_t*)stage_in(d_pi, pi, npk * 4, s);
      const int32_t* dpj = (const int32_t*)stage_in(d_pj, pj, npk * 4, s);
      const int32_t* dpk = (const int32_t*)stage_in(d_pk, pk, npk * 4, s);
      const double* dZpp = (const double*)stage_in(d_Zpp, ZZon_pp, npk * 8, s);
      const double* dfpp = (const double*)stage_in(d_fpp, fcrit_pp, npk * 8, s);
      for (DevBuf* b : {&p_lin, &p_Rf, &p_Z, &p_fc}) b->ensure(npk * 8);
      for (DevBuf* b : {&p_ir2, &p_np, &p_skip}) b->ensure(npk * 4);
      double* dout = out;
      if (!is_device_ptr(out)) {
        d_out.ensure(npk * RES_N * 8);
        dout = d_out.as<double>();
      }
      const double f3p = 4.0 / 3.0 * 3.141592653589793;
      for (int b = 0; b < nbatch; b++) {
        const int64_t q0 = boff[b], nq = boff[b + 1] - boff[b];
        if (nq == 0) continue;
        // npart of the batch (RadialShell.jl:288-295); the whole list without rmax2rs
        int np = (int)shells.ncells;
        if (rmax2rs > 0.0) {
          const double x = rmax2rs * Rf[b] / alatt, v = f3p * (x * x * x);
          np = v >= (double)shells.ncells ? (int)shells.ncells : (int)std::floor(v);
        }
        const unsigned g = (unsigned)((nq + 255) / 256);
        multirf_prep_kernel<<<g, 256, 0, s>>>(dpi, dpj, dpk, q0, nq, n, Rf[b], (int)ir2min[b], np, dZpp, dfpp, ZZon,
                                              fcrit, p_lin.as<int64_t>(), p_Rf.as<double>(), p_ir2.as<int32_t>(),
                                              p_np.as<int32_t>(), p_Z.as<double>(), p_fc.as<double>());
        PPB_LAUNCHED(ctx->sync.launches);
        const bool premask = rmax2rs > 0.0 && dm;
        if (premask) {
          const int thr = (int)std::floor(Rf[b] / alatt * rmax2rs);
          premask_kernel<<<g, 256, 0, s>>>(p_lin.as<int64_t>(), q0, nq, dm, thr, p_skip.as<int32_t>());
          PPB_LAUNCHED(ctx->sync.launches);
        }
        ShellArgs a = ctx->shell_args(ctx->sync, shells, n, alatt, aos.as<float4>(), dl);
        a.pk = PeakParams{p_lin.as<int64_t>() + q0, p_Rf.as<double>() + q0, p_ir2.as<int32_t>() + q0,
                          p_Z.as<double>() + q0, p_fc.as<double>() + q0};
        a.npk = nq;
        a.npcap = rmax2rs > 0.0 ? p_np.as<int32_t>() + q0 : nullptr;
        a.out = dout + q0 * RES_N;
        ShellStats stt{};
        ctx->run_shells(ctx->sync, a, plain == 0, plain == 0, &stt);
        if (stt.guard != 0)
          throw Error{PPB_ERR_CUDA, "shell truncation guard tripped: a profile read beyond the gathered shells"};
        if (stt.akk != 0)
          throw Error{PPB_ERR_INVALID, "kernel_strain SPH table index out of range (the reference raises here too)"};
        if (stt.raw[8] != 0) throw Error{PPB_ERR_INVALID, "peak index outside the grid"};
        if (premask) {
          skip_out_kernel<<<g, 256, 0, s>>>(p_skip.as<int32_t>(), nq, a.out);
          PPB_LAUNCHED(ctx->sync.launches);
        }
        // this batch's halos mask their cells before the next batch reads the mask
        if (dm) launch_shell_mask(L, a, dm, nbuff, ctx->nsm * 16);
      }
      if (dout != out) PPB_CUDA(cudaMemcpyAsync(out, dout, npk * RES_N * 8, cudaMemcpyDefault, s));
    }
    if (mask) PPB_CUDA(cudaMemcpyAsync(mask, d_mask.p, N, cudaMemcpyDefault, s));
    PPB_CUDA(cudaStreamSynchronize(s));
    return PPB_OK;
  } catch (const ppb::Error& e) {
    ctx->set_error(e.msg);
    return e.code;
  } catch (...) {
    ctx->set_error("unknown error");
    return PPB_ERR_INVALID;
  }
}

// Shell-kernel statistics of the last call: cell visits and the five
// dump-reason counters of RadialShell.jl:15-34 (premask, no_fcrit, m0_one,
// no_collapse, rthl_neg), plus the kernel's device time in ms.
int32_t ppb_last_shell_stats(ppb_ctx* ctx, int64_t* visits, int64_t* dumps5, float* ms) {
  if (!ctx) return PPB_ERR_INVALID;
  if (visits) *visits = (int64_t)ctx->sync.last_shell.visits;
  if (dumps5)
    for (int i = 0; i < 5; i++) dumps5[i] = (int64_t)ctx->sync.last_shell.dump[i];
  if (ms) *ms = ctx->sync.last_shell.ms;
  return PPB_OK;
}

int32_t ppb_shell_counters(ppb_ctx* ctx, int64_t* out16) {
  if (!ctx || !out16) return PPB_ERR_INVALID;
  for (int i = 0; i < 16; i++) out16[i] = (int64_t)ctx->sync.last_shell.raw[i];
  return PPB_OK;
}

int32_t ppb_last_shell_times(ppb_ctx* ctx, float* ms4, int64_t* rows, int32_t* batches) {
  if (!ctx) return PPB_ERR_INVALID;
  if (ms4)
    for (int i = 0; i < 4; i++) ms4[i] = ctx->sync.last_shell.kms[i];
  if (rows) *rows = (int64_t)ctx->sync.last_shell.pool_rows;
  if (batches) *batches = ctx->sync.last_shell.batches;
  return PPB_OK;
}

}  // extern "C"
