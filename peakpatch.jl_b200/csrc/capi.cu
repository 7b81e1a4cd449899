// capi.cu — the extern "C" boundary of libppb (declared in include/ppb.h) and
// the context methods.  No C++ exception crosses the boundary: every entry
// point catches ppb::Error (and anything else) and returns a status code,
// keeping the message for ppb_last_error().
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cub/cub.cuh>

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
// slots
// ---------------------------------------------------------------------------
namespace ppb {

void Slot::init(int dev) {
  device = dev;
  PPB_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  for (auto& e : stage_ev) PPB_CUDA(cudaEventCreate(&e));
  for (auto& e : shell_ev) PPB_CUDA(cudaEventCreate(&e));
}

void Slot::release_buffers() {
  tile.reset();
  for (DevBuf* b : {&filt_Rf, &filt_ir2, &g_a, &g_D, &g_f, &chi, &stage, &counters, &ctl, &hdr, &geo, &pool, &okey,
                    &okey2, &oidx, &oidx2, &otmp, &tcen, &tcount, &t_aos, &t_lapd, &mlim})
    b->release();
}

size_t Slot::bytes_held() const {
  size_t b = tile ? tile->bytes() : 0;
  for (const DevBuf* d : {&filt_Rf, &filt_ir2, &g_a, &g_D, &g_f, &chi, &stage, &counters, &ctl, &hdr, &geo, &pool,
                          &okey, &okey2, &oidx, &oidx2, &otmp, &tcen, &tcount, &t_aos, &t_lapd, &mlim})
    b += d->bytes;
  return b;
}

TileRes& Slot::tile_for(int n) {
  if (!tile || tile->n != n) {
    tile.reset();   // one grid size resident per slot keeps the footprint bounded
    tile = std::make_unique<TileRes>();
  }
  return *tile;
}

Slot::~Slot() {
  if (stream) cudaStreamSynchronize(stream);
  release_buffers();
  for (auto& e : stage_ev) if (e) cudaEventDestroy(e);
  for (auto& e : shell_ev) if (e) cudaEventDestroy(e);
  if (stream) cudaStreamDestroy(stream);
}

}  // namespace ppb

// ---------------------------------------------------------------------------
// context methods
// ---------------------------------------------------------------------------
void ppb_ctx::set_error(const std::string& m) {
  std::lock_guard<std::mutex> lk(err_mu);
  err = m;
}



const GrowthTable& ppb_ctx::growth(double Om, double OB, double OL, double h) {
  std::lock_guard<std::mutex> lk(sh.cache_mu);
  auto& e = sh.growth[{Om, OB, OL, h}];
  if (!e) e = std::make_unique<GrowthTable>(make_growth_table(Om, OB, OL, h));
  return *e;
}

const std::vector<double>& ppb_ctx::chi_table(double Om, double OL, double h, double zmax) {
  std::lock_guard<std::mutex> lk(sh.cache_mu);
  auto& e = sh.chi[{Om, OL, h, zmax}];
  if (!e) e = std::make_unique<std::vector<double>>(make_chi_table(Om, OL, h, zmax, 2000));
  return *e;
}

ShellTable& ppb_ctx::shell_table(int nhunt, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(sh.cache_mu);
  auto& e = sh.shells[nhunt];
  if (!e) {
    auto t = std::make_unique<ShellTable>();
    build_shell_table(*t, nhunt);
    upload_shell_table(*t, s);
    e = std::move(t);
  }
  return *e;
}

const float4* ppb_ctx::cellf(ShellTable& st, int n, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(sh.cache_mu);
  auto& e = st.cellf[n];
  if (!e) {
    std::vector<float4> f;
    build_cellf(st, n, f);
    auto b = std::make_unique<DevBuf>();
    b->ensure(f.size() * sizeof(float4));
    PPB_CUDA(cudaMemcpyAsync(b->p, f.data(), f.size() * sizeof(float4), cudaMemcpyHostToDevice, s));
    PPB_CUDA(cudaStreamSynchronize(s));
    e = std::move(b);
  }
  return e->as<float4>();
}

// device copies of the run's growth (and chi) tables on the slot; the host
// tables are cache entries that outlive the asynchronous copies
DevCosmo ppb_ctx::dev_cosmo(Slot& sl, const GrowthTable& G, double Om, double OL, double h, double zmax,
                            bool need_chi) {
  const size_t ng = G.a.size();
  sl.g_a.ensure(ng * 8);
  sl.g_D.ensure(ng * 8);
  sl.g_f.ensure(ng * 8);
  PPB_CUDA(cudaMemcpyAsync(sl.g_a.p, G.a.data(), ng * 8, cudaMemcpyHostToDevice, sl.stream));
  PPB_CUDA(cudaMemcpyAsync(sl.g_D.p, G.D.data(), ng * 8, cudaMemcpyHostToDevice, sl.stream));
  PPB_CUDA(cudaMemcpyAsync(sl.g_f.p, G.f.data(), ng * 8, cudaMemcpyHostToDevice, sl.stream));
  DevCosmo C{};
  C.ga = sl.g_a.as<double>();
  C.gD = sl.g_D.as<double>();
  C.gf = sl.g_f.as<double>();
  C.ng = (int)ng;
  C.amin = G.amin; C.amax = G.amax; C.Dinf = G.Dinf; C.D0 = G.D0; C.Hinf = G.Hinf; C.H0 = G.H0;
  if (need_chi) {
    const std::vector<double>& chi = chi_table(Om, OL, h, zmax);
    sl.chi.ensure(chi.size() * 8);
    PPB_CUDA(cudaMemcpyAsync(sl.chi.p, chi.data(), chi.size() * 8, cudaMemcpyHostToDevice, sl.stream));
    C.chis = sl.chi.as<double>();
    C.nchi = (int)chi.size();
    C.chi_zmax = zmax;
  }
  return C;
}

ShellArgs ppb_ctx::shell_args(Slot& sl, ShellTable& shells, int n, double alatt, const float4* aos,
                              const float* lapd) {
  ShellArgs a{};
  a.aos = aos;
  a.lapd = lapd;
  a.n = n;
  a.alatt = alatt;
  PPB_REQUIRE(n <= 4096, "grid size above 4096");
  a.cell8 = shells.d_cell8.as<int32_t>();
  a.cellf = cellf(shells, n, sl.stream);
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
  a.tab = sh.dtab;
  a.akk = sh.akk.as<double>();
  return a;
}

void ppb_ctx::run_shells(Slot& sl, ShellArgs& a, bool comp, bool adaptive, ShellStats* st) {
  cudaStream_t stream = sl.stream;
  Launch L{stream, &sl.launches};
  int& bps = sl.gather_bps[comp][adaptive];
  if (bps == 0) bps = shell_gather_blocks_per_sm(comp, adaptive);
  const int gblocks = nsm * bps;
  const int64_t stride = shell_stage_doubles_per_warp(a.nshell);
  sl.stage.ensure((size_t)((int64_t)gblocks * kGatherWarps * stride * 8));
  sl.counters.ensure(16 * 8);
  sl.ctl.ensure(64);
  sl.hdr.ensure(std::max<size_t>(1, (size_t)a.npk) * sizeof(PeakHdr));
  sl.geo.ensure(std::max<size_t>(1, (size_t)a.npk) * sizeof(int4));
  sl.mlim.ensure(std::max<size_t>(1, (size_t)a.npk) * sizeof(int32_t));
  PPB_CUDA(cudaMemsetAsync(sl.counters.p, 0, 16 * 8, stream));
  // profile pool: sized from the rows per peak of the previous call; peaks
  // run in batches that fit the pool budget, and a batch whose rows overflow
  // the pool runs again with a larger pool or fewer peaks
  const size_t row_bytes = ROW * sizeof(double);
  double& rpp = sl.rows_per_peak[adaptive];
  if (rpp <= 0.0) rpp = adaptive ? 64.0 : (double)(a.mmax + 1);
  // pool budget: half of the free memory (with the pool's own), at most 32 GB;
  // the free-memory query runs only when the pool would have to grow
  int64_t budget_rows = (int64_t)(sl.pool.bytes / row_bytes);
  if ((double)a.npk * rpp * 1.25 + 4096 > (double)budget_rows) {
    size_t fr = 0, tot = 0;
    PPB_CUDA(cudaMemGetInfo(&fr, &tot));
    budget_rows = std::max<int64_t>(
        1 << 16, (int64_t)(std::min<size_t>((size_t)32 << 30, (fr + sl.pool.bytes) / 2) / row_bytes));
  }
  ShellStats s{};
  unsigned long long before[16] = {}, c[16] = {};
  int64_t p0 = 0;
  while (p0 < a.npk) {
    const double want = std::max(1.0, rpp * 1.25);
    int64_t nb = std::min<int64_t>(a.npk - p0, std::max<int64_t>(1, (int64_t)((double)budget_rows / want)));
    const int64_t cap = std::min<int64_t>(budget_rows, (int64_t)((double)nb * want) + 4096);
    sl.pool.ensure((size_t)cap * row_bytes);
    ShellArgs b = a;
    b.pk.lin = a.pk.lin + p0;
    b.pk.Rf = a.pk.Rf + p0;
    b.pk.ir2min = a.pk.ir2min + p0;
    b.pk.ZZon = a.pk.ZZon + p0;
    b.pk.fcrit = a.pk.fcrit + p0;
    b.npk = nb;
    b.out = a.out + p0 * RES_N;
    b.hdr = sl.hdr.as<PeakHdr>() + p0;
    b.geo = sl.geo.as<int4>() + p0;
    b.mlim = sl.mlim.as<int32_t>() + p0;
    b.r2lim = a.r2lim ? a.r2lim + p0 : nullptr;
    b.pool = sl.pool.as<double>();
    b.pool_cap = cap;
    b.pool_ctr = reinterpret_cast<unsigned long long*>(sl.ctl.as<char>() + 8);
    b.queue = sl.ctl.as<int>();
    b.stage = sl.stage.as<double>();
    b.stage_stride = stride;
    b.counters = sl.counters.as<unsigned long long>();
    for (int e = 0; e < 10; e++) b.fhalf[e] = std::pow(e / 9.0 * 0.5 + 0.5, 1.0 / 3.0);
    PPB_CUDA(cudaMemsetAsync(sl.ctl.p, 0, 16, stream));
    PPB_CUDA(cudaEventRecord(sl.shell_ev[0], stream));
    // gather in spatial order: sort the peaks of the batch by brick Morton key
    sl.okey.ensure(nb * 4 + 16);
    sl.okey2.ensure(nb * 4 + 16);
    sl.oidx.ensure(nb * 4 + 16);
    sl.oidx2.ensure(nb * 4 + 16);
    launch_shell_geo(L, b, sl.okey.as<uint32_t>(), sl.oidx.as<int32_t>());
    size_t tb = 0;
    PPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, sl.okey.as<uint32_t>(), sl.okey2.as<uint32_t>(),
                                             sl.oidx.as<int32_t>(), sl.oidx2.as<int32_t>(), (int)nb, 0, 32, stream));
    sl.otmp.ensure(tb + 16);
    PPB_CUDA(cub::DeviceRadixSort::SortPairs(sl.otmp.p, tb, sl.okey.as<uint32_t>(), sl.okey2.as<uint32_t>(),
                                             sl.oidx.as<int32_t>(), sl.oidx2.as<int32_t>(), (int)nb, 0, 32, stream));
    sl.launches++;
    b.order = sl.oidx2.as<int32_t>();
    launch_shell_gather(L, b, comp, adaptive, gblocks);
    PPB_CUDA(cudaEventRecord(sl.shell_ev[1], stream));
    launch_shell_collapse(L, b, nsm, sl.walk_per_peak);
    PPB_CUDA(cudaEventRecord(sl.shell_ev[2], stream));
    launch_shell_zhalf(L, b);
    PPB_CUDA(cudaEventRecord(sl.shell_ev[3], stream));
    launch_shell_d2f(L, b, nsm * 16);
    PPB_CUDA(cudaEventRecord(sl.shell_ev[4], stream));
    unsigned long long used = 0;
    PPB_CUDA(cudaMemcpyAsync(&used, b.pool_ctr, sizeof(used), cudaMemcpyDeviceToHost, stream));
    PPB_CUDA(cudaMemcpyAsync(c, sl.counters.p, sizeof(c), cudaMemcpyDeviceToHost, stream));
    PPB_CUDA(cudaStreamSynchronize(stream));
    if ((int64_t)used > cap) {   // overflow: undo this batch's counts and run it again
      PPB_CUDA(cudaMemcpyAsync(sl.counters.p, before, sizeof(before), cudaMemcpyHostToDevice, stream));
      PPB_CUDA(cudaStreamSynchronize(stream));
      const double seen = (double)used / (double)nb;
      PPB_REQUIRE(seen * 1.25 > rpp, "profile pool overflow without growth");
      rpp = seen;
      continue;
    }
    float k[4];
    for (int e = 0; e < 4; e++) PPB_CUDA(cudaEventElapsedTime(&k[e], sl.shell_ev[e], sl.shell_ev[e + 1]));
    for (int e = 0; e < 4; e++) s.kms[e] += k[e];
    s.ms += k[0] + k[1] + k[2] + k[3];
    s.pool_rows += used;
    s.batches++;
    if (nb == a.npk - p0 || nb >= 1024) rpp = std::max(1.0, (double)used / (double)nb);
    if (nb >= 1024) sl.walk_per_peak = (double)(c[9] - before[9]) / (double)nb;
    std::memcpy(before, c, sizeof(c));
    p0 += nb;
  }
  s.visits = c[0];
  for (int i = 0; i < 5; i++) s.dump[i] = c[1 + i];
  s.guard = c[6];
  s.akk = c[7];
  for (int i = 0; i < 16; i++) s.raw[i] = c[i];
  sl.last_shell = s;
  if (st) *st = s;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
#define PPB_GUARD_BEGIN try {
#define PPB_GUARD_END(ctx)                                                    \
  }                                                                           \
  catch (const ppb::Error& e) {                                               \
    if (ctx) (ctx)->set_error(e.msg);                                         \
    return e.code;                                                            \
  }                                                                           \
  catch (const std::exception& e) {                                           \
    if (ctx) (ctx)->set_error(e.what());                                      \
    return PPB_ERR_INVALID;                                                   \
  }                                                                           \
  catch (...) {                                                               \
    if (ctx) (ctx)->set_error("unknown error");                               \
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
    ctx->sync.init(device);
    for (auto& e : ctx->ev) PPB_CUDA(cudaEventCreate(&e));
    size_t fr = 0, tot = 0;
    PPB_CUDA(cudaMemGetInfo(&fr, &tot));
    ctx->hbm_budget = hbm_budget ? hbm_budget : (uint64_t)(0.9 * (double)fr);
    const std::vector<double> akk = make_atab4();
    ctx->sh.akk.ensure(akk.size() * 8);
    PPB_CUDA(cudaMemcpy(ctx->sh.akk.p, akk.data(), akk.size() * 8, cudaMemcpyHostToDevice));
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
  server_stop(ctx);
  delete ctx;
  return PPB_OK;
}

int32_t ppb_last_error(ppb_ctx* ctx, char* buf, size_t len) {
  if (!ctx || !buf || len == 0) return PPB_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->err_mu);
  std::snprintf(buf, len, "%s", ctx->err.c_str());
  return PPB_OK;
}

int32_t ppb_set_collapse_table(ppb_ctx* ctx, const float* tab, int32_t nx, int32_t ny, int32_t nz, double x1,
                               double x2, double y1, double y2, double z1, double z2) {
  if (!ctx) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  PPB_GUARD_BEGIN
  std::unique_lock<std::shared_mutex> wl(ctx->sh.mu);   // waits for runs in flight
  PPB_REQUIRE(tab != nullptr, "table is null");
  PPB_REQUIRE(nx >= 2 && ny >= 2 && nz >= 2, "table needs at least 2 nodes per axis");
  PPB_REQUIRE(x2 > x1 && y2 > y1 && z2 > z1, "table ranges must be increasing");
  PPB_CUDA(cudaSetDevice(ctx->device));
  const size_t bytes = (size_t)nx * ny * nz * 4;
  ctx->sh.tab.ensure(bytes);
  PPB_CUDA(cudaMemcpy(ctx->sh.tab.p, tab, bytes, cudaMemcpyDefault));
  ctx->sh.dtab = DevTable{ctx->sh.tab.as<float>(), nullptr, nx, ny, nz, x1, x2, y1, y2, z1, z2};
  ctx->sh.has_tab = true;
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_set_collapse_table_f64(ppb_ctx* ctx, const double* tab, int32_t nx, int32_t ny, int32_t nz, double x1,
                                   double x2, double y1, double y2, double z1, double z2) {
  if (!ctx) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  PPB_GUARD_BEGIN
  std::unique_lock<std::shared_mutex> wl(ctx->sh.mu);   // waits for runs in flight
  PPB_REQUIRE(tab != nullptr, "table is null");
  PPB_REQUIRE(nx >= 2 && ny >= 2 && nz >= 2, "table needs at least 2 nodes per axis");
  PPB_REQUIRE(x2 > x1 && y2 > y1 && z2 > z1, "table ranges must be increasing");
  PPB_CUDA(cudaSetDevice(ctx->device));
  const size_t bytes = (size_t)nx * ny * nz * 8;
  ctx->sh.tab.ensure(bytes);
  PPB_CUDA(cudaMemcpy(ctx->sh.tab.p, tab, bytes, cudaMemcpyDefault));
  ctx->sh.dtab = DevTable{nullptr, ctx->sh.tab.as<double>(), nx, ny, nz, x1, x2, y1, y2, z1, z2};
  ctx->sh.has_tab = true;
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_generate_fields(ppb_ctx* ctx, const ppb_tile_params* p, float* delta, float* psi, float* psi2,
                            float* lapd) {
  if (!ctx) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  PPB_GUARD_BEGIN
  PPB_CUDA(cudaSetDevice(ctx->device));
  PPB_REQUIRE(p != nullptr, "params is null");
  std::shared_lock<std::shared_mutex> rl(ctx->sh.mu);
  generate_fields_core(ctx, ctx->sync, p, delta, psi, psi2, lapd);
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
  std::unique_lock<std::shared_mutex> wl(ctx->sh.mu);   // waits for runs in flight
  ctx->sh.pk_lk.ensure(n * 8);
  ctx->sh.pk_lp.ensure(n * 8);
  PPB_CUDA(cudaMemcpy(ctx->sh.pk_lk.p, lk.data(), n * 8, cudaMemcpyHostToDevice));
  PPB_CUDA(cudaMemcpy(ctx->sh.pk_lp.p, lp.data(), n * 8, cudaMemcpyHostToDevice));
  ctx->sh.pk_n = n;
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
  PPB_REQUIRE(out != nullptr, "output buffer is null");
  std::shared_lock<std::shared_mutex> rl(ctx->sh.mu);
  TileOut o;
  run_tile_core(ctx, ctx->sync, p, Rf, nfilt, &o);
  out->nfields = o.nfields;
  out->count = o.count;
  out->npeaks = o.npeaks;
  out->RTHLmax = o.RTHLmax;
  if (device_ms) *device_ms = o.device_ms;
  if (o.count > out->capacity) return PPB_ERR_CAPACITY;
  if (o.count > 0) {
    PPB_REQUIRE(out->records != nullptr, "records buffer is null");
    copy_out(out->records, o.d_records, (size_t)o.count * o.nfields * 4, ctx->sync.stream);
  }
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_run_multitile(ppb_ctx* ctx, const ppb_tile_params* p, const double* Rf, int32_t nfilt, int32_t ntile,
                          const int32_t* tiles, int32_t ntiles, ppb_halo_buf* out) {
  if (!ctx) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  PPB_GUARD_BEGIN
  PPB_CUDA(cudaSetDevice(ctx->device));
  PPB_REQUIRE(out != nullptr, "output buffer is null");
  PPB_REQUIRE(ntiles >= 0 && (ntiles == 0 || tiles != nullptr), "tiles must hold ntiles triples");
  std::shared_lock<std::shared_mutex> rl(ctx->sh.mu);
  TileOut o;
  run_multitile_core(ctx, ctx->sync, p, Rf, nfilt, ntile, tiles, ntiles, &o);
  out->nfields = o.nfields;
  out->count = o.count;
  out->npeaks = o.npeaks;
  out->RTHLmax = o.RTHLmax;
  if (o.count > out->capacity) return PPB_ERR_CAPACITY;
  if (o.count > 0) {
    PPB_REQUIRE(out->records != nullptr, "records buffer is null");
    copy_out(out->records, o.d_records, (size_t)o.count * o.nfields * 4, ctx->sync.stream);
  }
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_merge_catalog(ppb_ctx* ctx, const float* records, int64_t n, int32_t nfields, float* out,
                          int64_t* n_out) {
  if (!ctx || !n_out || n < 0 || (n > 0 && (!records || !out)) || (nfields != 11 && nfields != 33))
    return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  PPB_GUARD_BEGIN
  PPB_CUDA(cudaSetDevice(ctx->device));
  *n_out = 0;
  if (n == 0) return PPB_OK;
  Slot& sl = ctx->sync;
  DevBuf din, dout;
  const size_t bytes = (size_t)n * nfields * 4;
  const float* d_rec = (const float*)stage_in(din, records, bytes, sl.stream);
  float* d_out = out;
  if (!is_device_ptr(out)) {
    dout.ensure(bytes);
    d_out = dout.as<float>();
  }
  const int64_t m = merge_catalog_device(sl, d_rec, n, nfields, d_out);
  if (m > 0 && d_out != out) copy_out(out, d_out, (size_t)m * nfields * 4, sl.stream);
  PPB_CUDA(cudaStreamSynchronize(sl.stream));
  *n_out = m;
  return PPB_OK;
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
  Slot& sl = ctx->sync;
  if (is_device_ptr(out)) {
    launch_noise(Launch{sl.stream, &sl.launches}, out, n, seed);
    PPB_CUDA(cudaStreamSynchronize(sl.stream));
  } else {
    DevBuf tmp;
    tmp.ensure(bytes);
    launch_noise(Launch{sl.stream, &sl.launches}, tmp.as<float>(), n, seed);
    copy_out(out, tmp.p, bytes, sl.stream);
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
  PPB_CUDA(cudaEventRecord(ctx->ev[slot], ctx->sync.stream));
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
  PPB_CUDA(cudaStreamSynchronize(ctx->sync.stream));
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_launch_count(ppb_ctx* ctx, int64_t* count) {
  if (!ctx || !count) return PPB_ERR_INVALID;
  *count = ctx->launches_total();
  return PPB_OK;
}

int32_t ppb_last_stage_ms(ppb_ctx* ctx, float* ms4) {
  if (!ctx || !ms4) return PPB_ERR_INVALID;
  std::memcpy(ms4, ctx->sync.stage_ms, sizeof(ctx->sync.stage_ms));
  return PPB_OK;
}

}  // extern "C"
