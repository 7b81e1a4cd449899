// capi.cu — the extern "C" boundary of libppb (declared in include/ppb.h) and
// the context methods.  No C++ exception crosses the boundary: every entry
// point catches ppb::Error (and anything else) and returns a status code,
// keeping the message for ppb_last_error().
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "ppb_ctx.h"

using namespace ppb;

namespace ppb {

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

void copy_out(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  PPB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s));
  PPB_CUDA(cudaStreamSynchronize(s));
}

// device copy of a caller buffer (host or device); returns a device pointer
const void* stage_in(DevBuf& buf, const void* src, size_t bytes, cudaStream_t s) {
  if (!src) return nullptr;
  if (is_device_ptr(src)) return src;
  buf.ensure(bytes);
  PPB_CUDA(cudaMemcpyAsync(buf.p, src, bytes, cudaMemcpyHostToDevice, s));
  return buf.p;
}

}  // namespace ppb

// ---------------------------------------------------------------------------
// context methods
// ---------------------------------------------------------------------------
const GrowthTable& ppb_ctx::growth(double Om, double OB, double OL, double h) {
  if (!(gkey[0] == Om && gkey[1] == OB && gkey[2] == OL && gkey[3] == h)) {
    gcache = make_growth_table(Om, OB, OL, h);
    gkey[0] = Om; gkey[1] = OB; gkey[2] = OL; gkey[3] = h;
    const size_t ng = gcache.a.size();
    g_a.ensure(ng * 8);
    g_D.ensure(ng * 8);
    g_f.ensure(ng * 8);
    PPB_CUDA(cudaMemcpyAsync(g_a.p, gcache.a.data(), ng * 8, cudaMemcpyHostToDevice, stream));
    PPB_CUDA(cudaMemcpyAsync(g_D.p, gcache.D.data(), ng * 8, cudaMemcpyHostToDevice, stream));
    PPB_CUDA(cudaMemcpyAsync(g_f.p, gcache.f.data(), ng * 8, cudaMemcpyHostToDevice, stream));
    PPB_CUDA(cudaStreamSynchronize(stream));
  }
  return gcache;
}

DevCosmo ppb_ctx::dev_cosmo(const GrowthTable& G, double Om, double OL, double h, double zmax, bool need_chi) {
  DevCosmo C{};
  C.ga = g_a.as<double>();
  C.gD = g_D.as<double>();
  C.gf = g_f.as<double>();
  C.ng = (int)G.a.size();
  C.amin = G.amin; C.amax = G.amax; C.Dinf = G.Dinf; C.D0 = G.D0; C.Hinf = G.Hinf; C.H0 = G.H0;
  if (need_chi) {
    if (!(chikey[0] == Om && chikey[1] == OL && chikey[2] == h && chikey[3] == zmax)) {
      chicache = make_chi_table(Om, OL, h, zmax, 2000);
      chikey[0] = Om; chikey[1] = OL; chikey[2] = h; chikey[3] = zmax;
      chi.ensure(chicache.size() * 8);
      PPB_CUDA(cudaMemcpyAsync(chi.p, chicache.data(), chicache.size() * 8, cudaMemcpyHostToDevice, stream));
      PPB_CUDA(cudaStreamSynchronize(stream));
    }
    C.chis = chi.as<double>();
    C.nchi = (int)chicache.size();
    C.chi_zmax = zmax;
  }
  return C;
}

TileRes& ppb_ctx::tile(int n) {
  auto it = tiles.find(n);
  if (it == tiles.end()) {
    // one grid size resident at a time keeps the footprint bounded
    tiles.clear();
    it = tiles.emplace(n, std::make_unique<TileRes>()).first;
  }
  return *it->second;
}

ShellArgs ppb_ctx::shell_args(int n, double alatt, const float4* aos, const float* lapd) {
  ShellArgs a{};
  a.aos = aos;
  a.lapd = lapd;
  a.n = n;
  a.alatt = alatt;
  PPB_REQUIRE(n <= 4096, "grid size above 4096");
  a.cell8 = shells.d_cell8.as<int32_t>();
  upload_cellf(shells, n, stream);
  a.cellf = shells.d_cellf.as<float4>();
  a.sh_start = shells.d_start.as<int32_t>();
  a.sh_count = shells.d_count.as<int32_t>();
  a.rad = shells.d_rad.as<double>();
  a.r2m = shells.d_r2m.as<int32_t>();
  a.win_lo = shells.d_wlo.as<int32_t>();
  a.win_hi = shells.d_whi.as<int32_t>();
  a.win_off = shells.d_woff.as<int32_t>();
  a.wts = shells.d_wts.as<double>();
  a.w1 = shells.d_w1.as<double>();
  a.need = shells.d_need.as<int32_t>();
  a.rad5 = shells.d_rad5.as<double>();
  a.grp_a = shells.d_grp_a.as<int32_t>();
  a.grp_b = shells.d_grp_b.as<int32_t>();
  a.grp_c = shells.d_grp_c.as<int32_t>();
  a.ck_s = shells.d_ck_s.as<int32_t>();
  a.ck_n = shells.d_ck_n.as<int32_t>();
  a.sh_c0 = shells.d_sh_c0.as<int32_t>();
  a.sh_nc = shells.d_sh_nc.as<int32_t>();
  a.ngroups = shells.ngroups;
  a.nshell = shells.nshell;
  a.mmax = std::max(shells.nshell - 1, 1);
  a.npart = shells.ncells;
  a.tab = dtab;
  a.akk = akk.as<double>();
  return a;
}

void ppb_ctx::run_shells(ShellArgs& a, bool comp, bool adaptive, ShellStats* st) {
  Launch L{stream, &launches};
  int& bps = gather_bps[comp][adaptive];
  if (bps == 0) bps = shell_gather_blocks_per_sm(comp, adaptive);
  const int gblocks = nsm * bps;
  const int64_t stride = shell_stage_doubles_per_warp(a.nshell);
  stage.ensure((size_t)((int64_t)gblocks * kGatherWarps * stride * 8));
  counters.ensure(16 * 8);
  ctl.ensure(64);
  hdr.ensure(std::max<size_t>(1, (size_t)a.npk) * sizeof(PeakHdr));
  geo.ensure(std::max<size_t>(1, (size_t)a.npk) * sizeof(int4));
  PPB_CUDA(cudaMemsetAsync(counters.p, 0, 16 * 8, stream));
  // profile pool: sized from the rows per peak of the previous call; peaks
  // run in batches that fit the pool budget, and a batch whose rows overflow
  // the pool runs again with a larger pool or fewer peaks
  size_t fr = 0, tot = 0;
  PPB_CUDA(cudaMemGetInfo(&fr, &tot));
  const size_t row_bytes = ROW * sizeof(double);
  const int64_t budget_rows = std::max<int64_t>(
      1 << 16, (int64_t)(std::min<size_t>((size_t)32 << 30, (fr + pool.bytes) / 2) / row_bytes));
  double& rpp = rows_per_peak[adaptive];
  if (rpp <= 0.0) rpp = adaptive ? 64.0 : (double)(a.mmax + 1);
  ShellStats s{};
  unsigned long long before[16] = {}, c[16] = {};
  int64_t p0 = 0;
  while (p0 < a.npk) {
    const double want = std::max(1.0, rpp * 1.25);
    int64_t nb = std::min<int64_t>(a.npk - p0, std::max<int64_t>(1, (int64_t)((double)budget_rows / want)));
    const int64_t cap = std::min<int64_t>(budget_rows, (int64_t)((double)nb * want) + 4096);
    pool.ensure((size_t)cap * row_bytes);
    ShellArgs b = a;
    b.pk.lin = a.pk.lin + p0;
    b.pk.Rf = a.pk.Rf + p0;
    b.pk.ir2min = a.pk.ir2min + p0;
    b.pk.ZZon = a.pk.ZZon + p0;
    b.pk.fcrit = a.pk.fcrit + p0;
    b.npk = nb;
    b.out = a.out + p0 * RES_N;
    b.hdr = hdr.as<PeakHdr>() + p0;
    b.geo = geo.as<int4>() + p0;
    b.pool = pool.as<double>();
    b.pool_cap = cap;
    b.pool_ctr = reinterpret_cast<unsigned long long*>(ctl.as<char>() + 8);
    b.queue = ctl.as<int>();
    b.stage = stage.as<double>();
    b.stage_stride = stride;
    b.counters = counters.as<unsigned long long>();
    for (int e = 0; e < 10; e++) b.fhalf[e] = std::pow(e / 9.0 * 0.5 + 0.5, 1.0 / 3.0);
    PPB_CUDA(cudaMemsetAsync(ctl.p, 0, 16, stream));
    PPB_CUDA(cudaEventRecord(shell_ev[0], stream));
    launch_shell_geo(L, b);
    launch_shell_gather(L, b, comp, adaptive, gblocks);
    PPB_CUDA(cudaEventRecord(shell_ev[1], stream));
    launch_shell_collapse(L, b);
    PPB_CUDA(cudaEventRecord(shell_ev[2], stream));
    launch_shell_zhalf(L, b);
    PPB_CUDA(cudaEventRecord(shell_ev[3], stream));
    launch_shell_d2f(L, b, nsm * 16);
    PPB_CUDA(cudaEventRecord(shell_ev[4], stream));
    unsigned long long used = 0;
    PPB_CUDA(cudaMemcpyAsync(&used, b.pool_ctr, sizeof(used), cudaMemcpyDeviceToHost, stream));
    PPB_CUDA(cudaMemcpyAsync(c, counters.p, sizeof(c), cudaMemcpyDeviceToHost, stream));
    PPB_CUDA(cudaStreamSynchronize(stream));
    if ((int64_t)used > cap) {   // overflow: undo this batch's counts and run it again
      PPB_CUDA(cudaMemcpyAsync(counters.p, before, sizeof(before), cudaMemcpyHostToDevice, stream));
      PPB_CUDA(cudaStreamSynchronize(stream));
      const double seen = (double)used / (double)nb;
      PPB_REQUIRE(seen * 1.25 > rpp, "profile pool overflow without growth");
      rpp = seen;
      continue;
    }
    float k[4];
    for (int e = 0; e < 4; e++) PPB_CUDA(cudaEventElapsedTime(&k[e], shell_ev[e], shell_ev[e + 1]));
    for (int e = 0; e < 4; e++) s.kms[e] += k[e];
    s.ms += k[0] + k[1] + k[2] + k[3];
    s.pool_rows += used;
    s.batches++;
    if (nb == a.npk - p0 || nb >= 1024) rpp = std::max(1.0, (double)used / (double)nb);
    std::memcpy(before, c, sizeof(c));
    p0 += nb;
  }
  s.visits = c[0];
  for (int i = 0; i < 5; i++) s.dump[i] = c[1 + i];
  s.guard = c[6];
  s.akk = c[7];
  for (int i = 0; i < 16; i++) s.raw[i] = c[i];
  last_shell = s;
  if (st) *st = s;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
#define PPB_GUARD_BEGIN try {
#define PPB_GUARD_END(ctx)                                                    \
  }                                                                           \
  catch (const ppb::Error& e) {                                               \
    if (ctx) (ctx)->err = e.msg;                                              \
    return e.code;                                                            \
  }                                                                           \
  catch (const std::exception& e) {                                           \
    if (ctx) (ctx)->err = e.what();                                           \
    return PPB_ERR_INVALID;                                                   \
  }                                                                           \
  catch (...) {                                                               \
    if (ctx) (ctx)->err = "unknown error";                                    \
    return PPB_ERR_INVALID;                                                   \
  }

extern "C" {

int32_t ppb_abi_version(void) { return PPB_ABI_VERSION; }

int32_t ppb_ctx_create(int32_t device, uint64_t hbm_budget, ppb_ctx** out) {
  if (!out) return PPB_ERR_INVALID;
  *out = nullptr;
  ppb_ctx* ctx = nullptr;
  try {
    int ndev = 0;
    PPB_CUDA(cudaGetDeviceCount(&ndev));
    PPB_REQUIRE(device >= 0 && device < ndev, "device index out of range");
    PPB_CUDA(cudaSetDevice(device));
    ctx = new ppb_ctx();
    ctx->device = device;
    PPB_CUDA(cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, device));
    PPB_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    for (auto& e : ctx->ev) PPB_CUDA(cudaEventCreate(&e));
    for (auto& e : ctx->stage_ev) PPB_CUDA(cudaEventCreate(&e));
    for (auto& e : ctx->shell_ev) PPB_CUDA(cudaEventCreate(&e));
    size_t fr = 0, tot = 0;
    PPB_CUDA(cudaMemGetInfo(&fr, &tot));
    ctx->hbm_budget = hbm_budget ? hbm_budget : (uint64_t)(0.9 * (double)fr);
    const std::vector<double> akk = make_atab4();
    ctx->akk.ensure(akk.size() * 8);
    PPB_CUDA(cudaMemcpy(ctx->akk.p, akk.data(), akk.size() * 8, cudaMemcpyHostToDevice));
    *out = ctx;
    return PPB_OK;
  } catch (const ppb::Error& e) {
    delete ctx;
    fprintf(stderr, "ppb_ctx_create: %s\n", e.msg.c_str());
    return e.code;
  } catch (...) {
    delete ctx;
    return PPB_ERR_INVALID;
  }
}

int32_t ppb_ctx_destroy(ppb_ctx* ctx) {
  if (!ctx) return PPB_ERR_INVALID;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ctx->tiles.clear();
  for (auto& e : ctx->ev) if (e) cudaEventDestroy(e);
  for (auto& e : ctx->stage_ev) if (e) cudaEventDestroy(e);
  for (auto& e : ctx->shell_ev) if (e) cudaEventDestroy(e);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return PPB_OK;
}

int32_t ppb_last_error(ppb_ctx* ctx, char* buf, size_t len) {
  if (!ctx || !buf || len == 0) return PPB_ERR_INVALID;
  std::snprintf(buf, len, "%s", ctx->err.c_str());
  return PPB_OK;
}

int32_t ppb_set_collapse_table(ppb_ctx* ctx, const float* tab, int32_t nx, int32_t ny, int32_t nz, double x1,
                               double x2, double y1, double y2, double z1, double z2) {
  if (!ctx) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  PPB_GUARD_BEGIN
  PPB_REQUIRE(tab != nullptr, "table is null");
  PPB_REQUIRE(nx >= 2 && ny >= 2 && nz >= 2, "table needs at least 2 nodes per axis");
  PPB_REQUIRE(x2 > x1 && y2 > y1 && z2 > z1, "table ranges must be increasing");
  PPB_CUDA(cudaSetDevice(ctx->device));
  const size_t bytes = (size_t)nx * ny * nz * 4;
  ctx->tab.ensure(bytes);
  PPB_CUDA(cudaMemcpy(ctx->tab.p, tab, bytes, cudaMemcpyDefault));
  ctx->dtab = DevTable{ctx->tab.as<float>(), nx, ny, nz, x1, x2, y1, y2, z1, z2};
  ctx->has_tab = true;
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_set_pk_table(ppb_ctx* ctx, const double* k, const double* pk, int32_t n) {
  if (!ctx) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  PPB_GUARD_BEGIN
  PPB_REQUIRE(k && pk && n >= 2, "P(k) table needs >= 2 rows");
  std::vector<double> lk(n), lp(n);
  for (int i = 0; i < n; i++) {
    PPB_REQUIRE(k[i] > 0 && pk[i] > 0, "P(k) table entries must be positive (log-log interpolation)");
    if (i) PPB_REQUIRE(k[i] > k[i - 1], "P(k) table k must increase");
    lk[i] = std::log(k[i]);
    lp[i] = std::log(pk[i]);
  }
  PPB_CUDA(cudaSetDevice(ctx->device));
  ctx->pk_lk.ensure(n * 8);
  ctx->pk_lp.ensure(n * 8);
  PPB_CUDA(cudaMemcpy(ctx->pk_lk.p, lk.data(), n * 8, cudaMemcpyHostToDevice));
  PPB_CUDA(cudaMemcpy(ctx->pk_lp.p, lp.data(), n * 8, cudaMemcpyHostToDevice));
  ctx->pk_n = n;
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_run_tile(ppb_ctx* ctx, const ppb_tile_params* p, const double* Rf, int32_t nfilt, ppb_halo_buf* out) {
  return ppb_run_tile_timed(ctx, p, Rf, nfilt, out, nullptr);
}

int32_t ppb_run_tile_timed(ppb_ctx* ctx, const ppb_tile_params* p, const double* Rf, int32_t nfilt,
                           ppb_halo_buf* out, float* device_ms) {
  if (!ctx) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  PPB_GUARD_BEGIN
  PPB_CUDA(cudaSetDevice(ctx->device));
  return run_tile_impl(ctx, p, Rf, nfilt, out, device_ms);
  PPB_GUARD_END(ctx)
}

int32_t ppb_write_pksc(const char* path, const float* records, int64_t n, int32_t nfields, float RTHLmax,
                       float z_out) {
  if (!path || n < 0 || (n > 0 && !records) || (nfields != 11 && nfields != 33)) return PPB_ERR_INVALID;
  if (n > INT32_MAX) return PPB_ERR_INVALID;
  FILE* f = std::fopen(path, "wb");
  if (!f) return PPB_ERR_INVALID;
  const int32_t nn = (int32_t)n;
  bool ok = std::fwrite(&nn, 4, 1, f) == 1 && std::fwrite(&RTHLmax, 4, 1, f) == 1 && std::fwrite(&z_out, 4, 1, f) == 1;
  if (ok && n > 0) ok = std::fwrite(records, 4, (size_t)n * nfields, f) == (size_t)n * nfields;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? PPB_OK : PPB_ERR_INVALID;
}

int32_t ppb_noise_threefry(ppb_ctx* ctx, float* out, int32_t n, uint64_t seed) {
  if (!ctx) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  PPB_GUARD_BEGIN
  PPB_REQUIRE(out != nullptr && n >= 1 && n <= 4096, "bad noise arguments");
  PPB_CUDA(cudaSetDevice(ctx->device));
  const size_t bytes = (size_t)n * n * n * 4;
  if (is_device_ptr(out)) {
    launch_noise(Launch{ctx->stream, &ctx->launches}, out, n, seed);
    PPB_CUDA(cudaStreamSynchronize(ctx->stream));
  } else {
    DevBuf tmp;
    tmp.ensure(bytes);
    launch_noise(Launch{ctx->stream, &ctx->launches}, tmp.as<float>(), n, seed);
    copy_out(out, tmp.p, bytes, ctx->stream);
  }
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_alloc_host(ppb_ctx* ctx, size_t bytes, void** out) {
  if (!ctx || !out || bytes == 0) return PPB_ERR_INVALID;
  PPB_GUARD_BEGIN
  PPB_CUDA(cudaSetDevice(ctx->device));
  PPB_CUDA(cudaMallocHost(out, bytes));
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_free_host(ppb_ctx* ctx, void* p) {
  if (!ctx) return PPB_ERR_INVALID;
  PPB_GUARD_BEGIN
  if (p) PPB_CUDA(cudaFreeHost(p));
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_alloc_device(ppb_ctx* ctx, size_t bytes, void** out) {
  if (!ctx || !out || bytes == 0) return PPB_ERR_INVALID;
  PPB_GUARD_BEGIN
  PPB_CUDA(cudaSetDevice(ctx->device));
  PPB_CUDA(cudaMalloc(out, bytes));
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_free_device(ppb_ctx* ctx, void* p) {
  if (!ctx) return PPB_ERR_INVALID;
  PPB_GUARD_BEGIN
  PPB_CUDA(cudaSetDevice(ctx->device));
  if (p) PPB_CUDA(cudaFree(p));
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_event_record(ppb_ctx* ctx, int32_t slot) {
  if (!ctx || slot < 0 || slot >= 14) return PPB_ERR_INVALID;
  PPB_GUARD_BEGIN
  PPB_CUDA(cudaEventRecord(ctx->ev[slot], ctx->stream));
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_event_elapsed(ppb_ctx* ctx, int32_t a, int32_t b, float* ms) {
  if (!ctx || !ms || a < 0 || b < 0 || a >= 16 || b >= 16) return PPB_ERR_INVALID;
  PPB_GUARD_BEGIN
  PPB_CUDA(cudaEventSynchronize(ctx->ev[b]));
  PPB_CUDA(cudaEventElapsedTime(ms, ctx->ev[a], ctx->ev[b]));
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_synchronize(ppb_ctx* ctx) {
  if (!ctx) return PPB_ERR_INVALID;
  PPB_GUARD_BEGIN
  PPB_CUDA(cudaStreamSynchronize(ctx->stream));
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_launch_count(ppb_ctx* ctx, int64_t* count) {
  if (!ctx || !count) return PPB_ERR_INVALID;
  *count = ctx->launches;
  return PPB_OK;
}

int32_t ppb_last_stage_ms(ppb_ctx* ctx, float* ms4) {
  if (!ctx || !ms4) return PPB_ERR_INVALID;
  std::memcpy(ms4, ctx->stage_ms, sizeof(ctx->stage_ms));
  return PPB_OK;
}

}  // extern "C"
