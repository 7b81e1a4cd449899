// capi.cu — the extern "C" boundary of libppb (declared in include/ppb.h) and
// the context methods.  No C++ exception crosses the boundary: every entry
// point catches ppb::Error (and anything else) and returns a status code,
// keeping the message for ppb_last_error().
#include <algorithm>
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

void Slot::drop_record_texture() {
  if (rec_tex) cudaDestroyTextureObject(rec_tex);
  rec_tex = 0;
  rec_ptr = nullptr;
  rec_bytes = 0;
}

// The record array of the gather as a texture object (linear, float4
// elements): the gather fetches records through the texture pipe, which
// leaves the load/store pipe to the cell lists, partials and rows.  Kept per
// slot and rebuilt when the array changes; every kernel of the slot that used
// the previous one has completed (run_shells ends each batch with a stream
// synchronize).
cudaTextureObject_t Slot::record_texture(const float4* aos, int n) {
  const size_t elems = (size_t)2 * n * n * n;
  if (aos == rec_ptr && elems * 16 == rec_bytes) return rec_tex;
  drop_record_texture();
  int lim = 0;
  PPB_CUDA(cudaDeviceGetAttribute(&lim, cudaDevAttrMaxTexture1DLinearWidth, device));
  rec_ptr = aos;
  rec_bytes = elems * 16;
  if (elems > (size_t)lim || elems >= ((size_t)1 << 31)) return 0;   // the plain-load gather
  cudaResourceDesc rd{};
  rd.resType = cudaResourceTypeLinear;
  rd.res.linear.devPtr = const_cast<float4*>(aos);
  rd.res.linear.desc = cudaCreateChannelDesc<float4>();
  rd.res.linear.sizeInBytes = rec_bytes;
  cudaTextureDesc td{};
  td.readMode = cudaReadModeElementType;
  PPB_CUDA(cudaCreateTextureObject(&rec_tex, &rd, &td, nullptr));
  return rec_tex;
}

void Slot::release_buffers() {
  if (stream) PPB_CUDA(cudaStreamSynchronize(stream));
  drop_record_texture();
  merge.release();
  tiles.clear();
  tile_lru.clear();
  for (DevBuf* b : {&filt_Rf, &filt_ir2, &filt_np, &g_a, &g_D, &g_f, &chi, &stage, &counters, &ctl, &hdr, &geo, &pool, &okey,
                    &okey2, &oidx, &oidx2, &otmp, &tcen, &tcount, &t_aos, &t_lapd, &mlim, &anchors, &mr_in, &mr_out, &mr_aux,
                    &mr_rec, &mr_axis, &mr_amp, &pft})
    b->release();
  tune_save.release();
  iso.reset();
}

size_t Slot::bytes_held() const {
  size_t b = shell_bytes() + merge.bytes();
  for (const auto& t : tiles) b += t.second->bytes();
  return b;
}

size_t Slot::shell_bytes() const {
  size_t b = 0;
  for (const DevBuf* d : {&filt_Rf, &filt_ir2, &filt_np, &g_a, &g_D, &g_f, &chi, &stage, &counters, &ctl, &hdr, &geo, &pool,
                          &okey, &okey2, &oidx, &oidx2, &otmp, &tcen, &tcount, &t_aos, &t_lapd, &mlim, &anchors, &mr_in,
                          &mr_out, &mr_aux, &mr_rec, &mr_axis, &mr_amp, &pft})
    b += d->bytes;
  if (iso) b += iso->bytes();
  return b;
}

int Slot::lru_tile(int keep) const {
  for (int m : tile_lru)
    if (m != keep) return m;
  return 0;
}

uint64_t Slot::drop_tile(int n) {
  auto it = tiles.find(n);
  if (it == tiles.end()) return 0;
  PPB_CUDA(cudaStreamSynchronize(stream));   // nothing of that size in flight
  const uint64_t b = it->second->bytes();
  tiles.erase(it);
  tile_lru.erase(std::remove(tile_lru.begin(), tile_lru.end(), n), tile_lru.end());
  return b;
}

TileRes& Slot::tile_for(int n) {
  auto it = tiles.find(n);
  if (it == tiles.end()) {
    while ((int)tiles.size() >= std::max(1, max_tiles)) drop_tile(lru_tile(n));
    if (!tiles.empty()) {   // room for the new size's buffers, else give up older sizes
      const uint64_t need = tile_bytes_estimate(n);
      size_t fr = 0, tot = 0;
      PPB_CUDA(cudaMemGetInfo(&fr, &tot));
      while (!tiles.empty() && (uint64_t)fr < need + need / 4) {
        drop_tile(lru_tile(n));
        PPB_CUDA(cudaMemGetInfo(&fr, &tot));
      }
    }
    it = tiles.emplace(n, std::make_unique<TileRes>()).first;
  }
  tile_lru.erase(std::remove(tile_lru.begin(), tile_lru.end(), n), tile_lru.end());
  tile_lru.push_back(n);
  return *it->second;
}

Slot::~Slot() {
  if (stream) cudaStreamSynchronize(stream);
  for (auto& g : graphs)
    if (g.second) cudaGraphExecDestroy(g.second);
  graphs.clear();
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
  a.ck_p = shells.d_ck_p.as<int32_t>();
  a.ck_cells = shells.d_ck_cells.as<int4>();
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
  a.ck_d = shells.d_ck_d.as<int32_t>();
  a.nck = (int)shells.ck_s.size();
  a.sh_c0 = shells.d_sh_c0.as<int32_t>();
  a.sh_nc = shells.d_sh_nc.as<int32_t>();
  a.ngroups = shells.ngroups;
  a.nshell = shells.nshell;
  a.mmax = std::max(shells.nshell - 1, 1);
  a.npart = shells.ncells;
  a.fmax = pack_fmax(const_cast<float4*>(aos), n);
  a.tab = sh.dtab;
  a.akk = sh.akk.as<double>();
  return a;
}

void ppb_ctx::captured(Slot& sl, std::map<std::pair<int, int64_t>, cudaGraphExec_t>& graphs, int site, int64_t key,
                       const std::function<void()>& rec) {
  if (!sh.use_graphs.load()) {
    rec();
    return;
  }
  cudaStream_t s = sl.stream;
  // thread-local mode: other threads (other slots' workers) may allocate
  // while this stream records
  PPB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  cudaGraph_t g = nullptr;
  try {
    rec();
  } catch (...) {
    cudaStreamEndCapture(s, &g);
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    throw;
  }
  PPB_CUDA(cudaStreamEndCapture(s, &g));
  struct Owned {
    cudaGraph_t g;
    ~Owned() { if (g) cudaGraphDestroy(g); }
  } owned{g};
  size_t nodes = 0;
  PPB_CUDA(cudaGraphGetNodes(g, nullptr, &nodes));
  if (nodes == 0) return;
  cudaGraphExec_t& ex = graphs[{site, key}];
  if (ex) {
    cudaGraphExecUpdateResultInfo info{};
    if (cudaGraphExecUpdate(ex, g, &info) == cudaSuccess) {
      sl.graph_updates++;
    } else {   // the launch sequence changed shape: instantiate anew
      cudaGetLastError();
      cudaGraphExecDestroy(ex);
      ex = nullptr;
    }
  }
  if (!ex) {
    PPB_CUDA(cudaGraphInstantiate(&ex, g, 0));
    sl.graph_instantiations++;
  }
  PPB_CUDA(cudaGraphLaunch(ex, s));
  sl.graph_launches++;
}

// an event record that is also a node of the graph being captured (a
// timing point inside the graph) when the stream is capturing
static void record_event(cudaEvent_t e, cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  PPB_CUDA(cudaStreamIsCapturing(s, &cs));
  if (cs == cudaStreamCaptureStatusActive) PPB_CUDA(cudaEventRecordWithFlags(e, s, cudaEventRecordExternal));
  else PPB_CUDA(cudaEventRecord(e, s));
}

// gather order: geometry for every peak and, for brick_shift >= 0, the
// Morton sort of the peaks by brick (b.order set), else list order
static void shell_order(Slot& sl, ShellArgs& b, int brick_shift) {
  Launch L{sl.stream, &sl.launches};
  if (brick_shift < 0) {
    launch_shell_geo(L, b, nullptr, nullptr);
    b.order = nullptr;
    return;
  }
  b.brick_shift = brick_shift;
  launch_shell_geo(L, b, sl.okey.as<uint32_t>(), sl.oidx.as<int32_t>());
  size_t tb = sl.otmp.bytes;
  PPB_CUDA(cub::DeviceRadixSort::SortPairs(sl.otmp.p, tb, sl.okey.as<uint32_t>(), sl.okey2.as<uint32_t>(),
                                           sl.oidx.as<int32_t>(), sl.oidx2.as<int32_t>(), (int)b.npk, 0, 32,
                                           sl.stream));
  sl.launches++;
  b.order = sl.oidx2.as<int32_t>();
}

// collapse order (after the gather, which it reuses the order buffers of):
// the collapse kernels take the peaks by descending crossing shell
static void collapse_order(Slot& sl, ShellArgs& b, bool on) {
  b.corder = nullptr;
  if (!on || b.npk < 2) return;
  Launch L{sl.stream, &sl.launches};
  launch_collapse_order_keys(L, b, sl.okey.as<uint32_t>(), sl.oidx.as<int32_t>());
  size_t tb = sl.otmp.bytes;
  PPB_CUDA(cub::DeviceRadixSort::SortPairs(sl.otmp.p, tb, sl.okey.as<uint32_t>(), sl.okey2.as<uint32_t>(),
                                           sl.oidx.as<int32_t>(), sl.oidx2.as<int32_t>(), (int)b.npk, 0, 17,
                                           sl.stream));
  sl.launches++;
  b.corder = sl.oidx2.as<int32_t>();
}

TuneEntry ppb_ctx::tune_shells(Slot& sl, const ShellArgs& b0, bool comp, bool adaptive, int gblocks,
                                const void* rmap) {
  cudaStream_t s = sl.stream;
  Launch L{s, &sl.launches};
  TuneEntry te;
  te.npk = b0.npk;
  sl.tune_save.ensure(16 * 8);
  PPB_CUDA(cudaMemcpyAsync(sl.tune_save.p, sl.counters.p, 16 * 8, cudaMemcpyDeviceToDevice, s));
  cudaEvent_t* ev = sl.shell_ev;
  // candidates: bricks of 8 (the default, timed first), 4, 16 and 32 cells,
  // and list order; every run leaves the same per-peak rows
  static const int bricks[5] = {3, 2, 4, 5, -1};
  static const int slot_of[5] = {1, 0, 2, 3, 4};
  static const int widths[4] = {1, 2, 4, 8};
  ShellArgs b = b0;
  if (comp) launch_shell_anchors(L, b);
  // two rounds over the candidates, keeping each one's faster time, so that
  // the first launches' warm-up (caches, TLB) does not count against one
  for (int c = 0; c < 5; c++) te.gather_ms[c] = 1e30f;
  for (int c = 0; c < 4; c++) te.collapse_ms[c] = te.collapse_ordered_ms[c] = 1e30f;
  for (int round = 0; round < 2; round++) {
    for (int c = 0; c < 5; c++) {
      PPB_CUDA(cudaMemsetAsync(sl.ctl.p, 0, kCtlBytes, s));
      shell_order(sl, b, bricks[c]);
      PPB_CUDA(cudaEventRecord(ev[0], s));
      launch_shell_gather(L, b, comp, adaptive, gblocks, rmap);
      PPB_CUDA(cudaEventRecord(ev[1], s));
      PPB_CUDA(cudaEventSynchronize(ev[1]));
      float ms = 0.f;
      PPB_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
      te.gather_ms[slot_of[c]] = std::min(te.gather_ms[slot_of[c]], ms);
    }
    for (int o = 0; o < 2; o++) {   // list order, then by descending crossing shell
      for (int c = 0; c < 4; c++) {
        PPB_CUDA(cudaEventRecord(ev[0], s));
        collapse_order(sl, b, o == 1);
        launch_shell_collapse(L, b, nsm, sl.walk_per_peak, widths[c]);
        PPB_CUDA(cudaEventRecord(ev[1], s));
        PPB_CUDA(cudaEventSynchronize(ev[1]));
        float ms = 0.f;
        PPB_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
        float& t = o ? te.collapse_ordered_ms[c] : te.collapse_ms[c];
        t = std::min(t, ms);
      }
    }
  }
  // the default wins unless another candidate is at least 3 % faster
  int bi = 1;
  for (int c = 0; c < 5; c++)
    if (te.gather_ms[c] < te.gather_ms[bi]) bi = c;
  if (!(te.gather_ms[bi] < 0.97f * te.gather_ms[1])) bi = 1;
  static const int shift_of[5] = {2, 3, 4, 5, -1};
  te.brick_shift = shift_of[bi];
  // the chosen order with 256-bit loads instead of the texture pipe
  te.gather_tex = b0.rec_tex != 0;
  te.gather_plain_ms = 0.f;
  if (b0.rec_tex) {
    ShellArgs bp = b0;
    bp.rec_tex = 0;
    float best = 1e30f;
    for (int round = 0; round < 2; round++) {
      PPB_CUDA(cudaMemsetAsync(sl.ctl.p, 0, kCtlBytes, s));
      shell_order(sl, bp, te.brick_shift);
      PPB_CUDA(cudaEventRecord(ev[0], s));
      launch_shell_gather(L, bp, comp, adaptive, gblocks, rmap);
      PPB_CUDA(cudaEventRecord(ev[1], s));
      PPB_CUDA(cudaEventSynchronize(ev[1]));
      float ms = 0.f;
      PPB_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
      best = std::min(best, ms);
    }
    te.gather_plain_ms = best;
    // a like-for-like choice of the load path (same order, same kernel
    // otherwise): the faster unless within 1 %
    te.gather_tex = !(best < 0.99f * te.gather_ms[bi]);
  }
  // collapse: the size heuristic's width in list order unless another
  // (width, order) is at least 3 % faster
  const int wd = shell_collapse_width(b.npk, nsm, sl.walk_per_peak);
  const int di = wd == 4 ? 2 : wd - 1;
  int ci = di, co = 0;
  for (int o = 0; o < 2; o++)
    for (int c = 0; c < 4; c++) {
      const float t = o ? te.collapse_ordered_ms[c] : te.collapse_ms[c];
      if (t < (co ? te.collapse_ordered_ms[ci] : te.collapse_ms[ci])) { ci = c; co = o; }
    }
  const float best = co ? te.collapse_ordered_ms[ci] : te.collapse_ms[ci];
  if (best < 0.97f * te.collapse_ms[di]) {
    te.collapse_threads = widths[ci];
    te.collapse_order = co == 1;
  } else {
    te.collapse_threads = 0;
    te.collapse_order = false;
  }
  PPB_CUDA(cudaMemcpyAsync(sl.counters.p, sl.tune_save.p, 16 * 8, cudaMemcpyDeviceToDevice, s));
  PPB_CUDA(cudaMemsetAsync(sl.ctl.p, 0, kCtlBytes, s));
  return te;
}

// grow b to at least `need` bytes with 50 % headroom (at most `limit`):
// buffers sized by the peak count of a request then rarely grow again in a
// stream of requests whose counts vary, and every growth's cudaFree waits
// for all work on the device, other slots' included
static void grow(DevBuf& b, size_t need, size_t limit = ~(size_t)0) {
  if (need <= b.bytes) return;
  b.ensure(std::max(need, std::min(need + need / 2, limit)));
}

void ppb_ctx::run_shells(Slot& sl, ShellArgs& a, bool comp, bool adaptive, ShellStats* st,
                         const std::function<void()>& pre) {
  cudaStream_t stream = sl.stream;
  Launch L{stream, &sl.launches};
  a.rec_tex = sh.gather_tex.load() != 0 ? sl.record_texture(a.aos, a.n) : 0;
  // the TMA-staged gather (records through per-lane shared-memory rings)
  // when the option asks for it and the records fit a tensor map
  alignas(64) unsigned char ring_map[128];
  const bool ring = sh.gather_ring.load() != 0 && record_ring_map(a.aos, a.n, ring_map);
  int& bps = sl.gather_bps[comp][adaptive][ring];
  if (bps == 0) bps = ring ? shell_gather_ring_blocks_per_sm(comp, adaptive) : shell_gather_blocks_per_sm(comp, adaptive);
  const int gblocks = nsm * bps;
  const void* rmap = ring ? ring_map : nullptr;
  const int64_t stride = shell_stage_doubles_per_warp(a.nshell);
  sl.stage.ensure((size_t)((int64_t)gblocks * kGatherWarps * stride * 8));
  sl.counters.ensure(16 * 8);
  sl.ctl.ensure(kCtlBytes);
  grow(sl.hdr, std::max<size_t>(1, (size_t)a.npk) * sizeof(PeakHdr));
  grow(sl.geo, std::max<size_t>(1, (size_t)a.npk) * 2 * sizeof(int4));
  grow(sl.mlim, std::max<size_t>(1, (size_t)a.npk) * sizeof(int32_t));
  sl.anchors.ensure(std::max<size_t>(1, (size_t)a.nck) * kAnchorStride * sizeof(float2));
  a.ck_K = sl.anchors.as<float2>();
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
  // autotuned order brick and collapse width for this kind of batch
  // (the walk class: collapse walks of more than 8 steps per peak in the
  // slot's previous batch, as on the lightcone, favour other widths)
  const std::array<int64_t, 6> tkey{a.n, a.nshell, comp, adaptive, (a.r2lim != nullptr) | (a.npcap != nullptr) << 1,
                                    sl.walk_per_peak > 8.0};
  TuneEntry te;
  bool tuned = false;
  {
    std::lock_guard<std::mutex> lk(sh.cache_mu);
    auto it = sh.tune.find(tkey);
    if (it != sh.tune.end()) {
      te = it->second;
      tuned = true;
    }
  }
  bool tune_now = !tuned && sh.autotune.load() != 0 && a.npk >= sh.tune_min_peaks.load();
  bool first = true;
  int64_t p0 = 0;
  while (p0 < a.npk) {
    const double want = std::max(1.0, rpp * 1.25);
    int64_t nb = std::min<int64_t>(a.npk - p0, std::max<int64_t>(1, (int64_t)((double)budget_rows / want)));
    const int64_t cap = std::min<int64_t>(budget_rows, (int64_t)((double)nb * want) + 4096);
    grow(sl.pool, (size_t)cap * row_bytes, (size_t)budget_rows * row_bytes);
    ShellArgs b = a;
    b.pk.lin = a.pk.lin + p0;
    b.pk.Rf = a.pk.Rf + p0;
    b.pk.ir2min = a.pk.ir2min + p0;
    b.pk.ZZon = a.pk.ZZon + p0;
    b.pk.fcrit = a.pk.fcrit + p0;
    b.npk = nb;
    b.out = a.out + p0 * RES_N;
    b.hdr = sl.hdr.as<PeakHdr>() + p0;
    b.geo = sl.geo.as<int4>() + 2 * p0;
    b.mlim = sl.mlim.as<int32_t>() + p0;
    b.r2lim = a.r2lim ? a.r2lim + p0 : nullptr;
    b.npcap = a.npcap ? a.npcap + p0 : nullptr;
    b.pool = sl.pool.as<double>();
    b.pool_cap = cap;
    b.pool_ctr = reinterpret_cast<unsigned long long*>(sl.ctl.as<char>() + 8);
    b.queue = sl.ctl.as<int>();
    b.cqueue = sl.ctl.as<int>() + 1;
    b.stage = sl.stage.as<double>();
    b.stage_stride = stride;
    b.counters = sl.counters.as<unsigned long long>();
    b.brick_shift = 3;
    for (int e = 0; e < 10; e++) b.fhalf[e] = std::pow(e / 9.0 * 0.5 + 0.5, 1.0 / 3.0);
    // buffers of the spatial order (allocated before any capture)
    grow(sl.okey, nb * 4 + 16);
    grow(sl.okey2, nb * 4 + 16);
    grow(sl.oidx, nb * 4 + 16);
    grow(sl.oidx2, nb * 4 + 16);
    {
      size_t tb = 0;
      PPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, sl.okey.as<uint32_t>(), sl.okey2.as<uint32_t>(),
                                               sl.oidx.as<int32_t>(), sl.oidx2.as<int32_t>(), (int)nb, 0, 32,
                                               stream));
      grow(sl.otmp, tb + 16);
    }
    if (tune_now) {
      if (first && pre) pre();   // the tuning pass reads what `pre` writes
      te = tune_shells(sl, b, comp, adaptive, gblocks, rmap);
      {
        std::lock_guard<std::mutex> lk(sh.cache_mu);
        sh.tune[tkey] = te;
      }
      tune_now = false;
    }
    const int fb = sh.force_brick.load(), fc = sh.force_collapse.load();
    const int fo = sh.collapse_order.load();
    const bool corder_on = fo == 1 || (fo == -1 && te.collapse_order);
    if (sh.gather_tex.load() == -1 && !te.gather_tex) b.rec_tex = 0;
    if (fb != -2) te.brick_shift = fb;
    if (fc != 0) te.collapse_threads = fc;
    // the sub-batch as one graph: geometry, order, gather, collapse,
    // zvir_half, d2F, with timing events between the kernels
    captured(sl, sl.graphs, 2, (int64_t)a.n * 4 + (comp ? 2 : 0) + (adaptive ? 1 : 0), [&] {
      if (first && pre) pre();
      PPB_CUDA(cudaMemsetAsync(sl.ctl.p, 0, kCtlBytes, stream));
      record_event(sl.shell_ev[0], stream);
      if (comp) launch_shell_anchors(L, b);
      shell_order(sl, b, te.brick_shift);
      launch_shell_gather(L, b, comp, adaptive, gblocks, rmap);
      record_event(sl.shell_ev[1], stream);
      collapse_order(sl, b, corder_on);
      launch_shell_collapse(L, b, nsm, sl.walk_per_peak, te.collapse_threads);
      record_event(sl.shell_ev[2], stream);
      launch_shell_zhalf(L, b);
      record_event(sl.shell_ev[3], stream);
      launch_shell_d2f(L, b, nsm * 16);
      record_event(sl.shell_ev[4], stream);
    });
    first = false;
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
  if (c[10] != 0)
    throw Error{PPB_ERR_CUDA, "gather: a staged record copy did not complete within the wait bound"};
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

int32_t ppb_make_collapse_table(ppb_ctx* ctx, const ppb_table_params* p, double* out, int32_t install) {
  if (!ctx) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  PPB_GUARD_BEGIN
  PPB_REQUIRE(p != nullptr, "params is null");
  PPB_REQUIRE(p->Om > 0 && p->OB >= 0 && p->OB <= p->Om && p->OL >= 0 && p->h > 0, "bad cosmology");
  PPB_REQUIRE(p->Nx >= 2 && p->Ny >= 2 && p->Nz >= 2, "table needs at least 2 nodes per axis");
  PPB_REQUIRE((int64_t)p->Nx * p->Ny * p->Nz <= ((int64_t)1 << 26), "table larger than 2^26 nodes");
  PPB_REQUIRE(p->X2 > p->X1 && p->Y2 > p->Y1 && p->Z2 > p->Z1, "table ranges must be increasing");
  const int f = p->iforce_strat;
  PPB_REQUIRE(f == 0 || f == 1 || f == 3 || f == 4 || f == 5 || f == 6, "iforce_strat must be 0, 1, 3, 4, 5 or 6");
  PPB_REQUIRE(p->ivir_strat == 1 || p->ivir_strat == 2, "ivir_strat must be 1 or 2");
  PPB_REQUIRE(p->nstepmax >= 1 && p->nstepmax <= 100000000, "nstepmax must be in [1, 1e8]");
  PPB_REQUIRE(p->fcoll_1 > 0 && p->fcoll_2 > 0 && p->fcoll_3 > 0 && p->tfac > 0 && p->zinit_fac > 0,
              "fcoll, tfac and zinit_fac must be positive");
  PPB_REQUIRE(install >= 0 && install <= 2, "install must be 0, 1 or 2");
  PPB_CUDA(cudaSetDevice(ctx->device));
  Slot& sl = ctx->sync;
  const GrowthTable& G = ctx->growth(p->Om, p->OB, p->OL, p->h);
  // F = 10^x on the host (make_table's Frho = 10.0^logF)
  std::vector<double> F(p->Nx);
  const double dX = (p->X2 - p->X1) / (p->Nx - 1);
  for (int i = 0; i < p->Nx; i++) F[i] = std::pow(10.0, p->X1 + i * dX);
  const int64_t nn = (int64_t)p->Nx * p->Ny * p->Nz;
  DevBuf dF, dout, dsteps;
  dF.ensure(F.size() * 8);
  dout.ensure((size_t)nn * 8);
  dsteps.ensure(8);
  PPB_CUDA(cudaMemcpyAsync(dF.p, F.data(), F.size() * 8, cudaMemcpyHostToDevice, sl.stream));
  PPB_CUDA(cudaMemsetAsync(dsteps.p, 0, 8, sl.stream));
  PPB_CUDA(cudaEventRecord(sl.stage_ev[0], sl.stream));
  make_table_device(sl, G, p, dF.as<double>(), dout.as<double>(), dsteps.as<unsigned long long>());
  PPB_CUDA(cudaEventRecord(sl.stage_ev[1], sl.stream));
  unsigned long long steps = 0;
  PPB_CUDA(cudaMemcpyAsync(&steps, dsteps.p, 8, cudaMemcpyDeviceToHost, sl.stream));
  PPB_CUDA(cudaStreamSynchronize(sl.stream));
  PPB_CUDA(cudaEventElapsedTime(&ctx->table_ms, sl.stage_ev[0], sl.stage_ev[1]));
  ctx->table_steps = (int64_t)steps;
  if (out) copy_out(out, dout.p, (size_t)nn * 8, sl.stream);
  if (install == 2) {
    const int32_t rc = ppb_set_collapse_table_f64(ctx, dout.as<double>(), p->Nx, p->Ny, p->Nz, p->X1, p->X2, p->Y1,
                                                  p->Y2, p->Z1, p->Z2);
    if (rc != PPB_OK) return rc;
  } else if (install == 1) {   // Float32 nodes, as make_table stores them
    std::vector<double> h((size_t)nn);
    PPB_CUDA(cudaMemcpy(h.data(), dout.p, (size_t)nn * 8, cudaMemcpyDeviceToHost));
    std::vector<float> t32((size_t)nn);
    for (int64_t q = 0; q < nn; q++) t32[q] = (float)h[q];
    const int32_t rc = ppb_set_collapse_table(ctx, t32.data(), p->Nx, p->Ny, p->Nz, p->X1, p->X2, p->Y1, p->Y2,
                                              p->Z1, p->Z2);
    if (rc != PPB_OK) return rc;
  }
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_last_table_stats(ppb_ctx* ctx, float* ms, int64_t* steps) {
  if (!ctx) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  if (ms) *ms = ctx->table_ms;
  if (steps) *steps = ctx->table_steps;
  return PPB_OK;
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

int32_t ppb_peak_find_tile(ppb_ctx* ctx, const float* delta_tile, int32_t n, const double* Rf, const double* fcrit,
                           int32_t nfilt, int8_t* mask, double xbx, double ybx, double zbx, double alatt,
                           int32_t nbuff, int32_t wsmooth, int32_t ioutshear, int64_t capacity, int32_t* pi,
                           int32_t* pj, int32_t* pk, int64_t* ipp, double* x, double* y, double* z, float* FcRf,
                           double* Rf_out, float* d2Rf, int32_t* filter, int64_t* npeaks) {
  if (!ctx) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  PPB_GUARD_BEGIN
  PPB_CUDA(cudaSetDevice(ctx->device));
  std::shared_lock<std::shared_mutex> rl(ctx->sh.mu);
  PeakTileOut o;
  o.capacity = capacity;
  o.pi = pi;
  o.pj = pj;
  o.pk = pk;
  o.ipp = ipp;
  o.x = x;
  o.y = y;
  o.z = z;
  o.FcRf = FcRf;
  o.Rf = Rf_out;
  o.d2Rf = d2Rf;
  o.filter = filter;
  o.npeaks = npeaks;
  peak_find_tile_core(ctx, ctx->sync, delta_tile, n, Rf, fcrit, nfilt, mask, xbx, ybx, zbx, alatt, nbuff, wsmooth,
                      ioutshear, o);
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
  ctx->sh.pk_version++;
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

int32_t ppb_run_multitile_split(ppb_ctx* ctx, const ppb_tile_params* p, const double* Rf, int32_t nfilt,
                                int32_t ntile, int32_t coarse_factor, int32_t coarse_grid, const int32_t* tiles,
                                int32_t ntiles, ppb_halo_buf* out) {
  if (!ctx) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  PPB_GUARD_BEGIN
  PPB_CUDA(cudaSetDevice(ctx->device));
  PPB_REQUIRE(out != nullptr, "output buffer is null");
  PPB_REQUIRE(ntiles >= 0 && (ntiles == 0 || tiles != nullptr), "tiles must hold ntiles triples");
  std::shared_lock<std::shared_mutex> rl(ctx->sh.mu);
  TileOut o;
  run_multitile_split_core(ctx, ctx->sync, p, Rf, nfilt, ntile, coarse_factor, coarse_grid, tiles, ntiles, &o);
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

int32_t ppb_split_coarse_grid(int32_t n, int32_t nbuff, int32_t ntile, int32_t coarse_factor, int32_t coarse_grid) {
  const int64_t nsub = (int64_t)n - 2 * nbuff;
  if (n < 1 || nbuff < 0 || nsub < 1 || ntile < 1) return PPB_ERR_INVALID;
  return split_coarse_grid(nsub * ntile + 2 * nbuff, n, ntile, coarse_factor, coarse_grid);
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
  const size_t bytes = (size_t)n * nfields * 4;
  const float* d_rec = (const float*)stage_in(sl.merge.in, records, bytes, sl.stream);
  float* d_out = out;
  if (!is_device_ptr(out)) {
    sl.merge.out.ensure(bytes);
    d_out = sl.merge.out.as<float>();
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

int32_t ppb_write_catalog_hdf5(const char* path, const float* records, int64_t n, int32_t nfields, double Om,
                               double OL, double h, double z_max) {
  PPB_GUARD_BEGIN
  PPB_REQUIRE(path && n >= 0 && (n == 0 || records) && (nfields == 11 || nfields == 33), "bad arguments");
  PPB_REQUIRE(Om > 0.0 && h > 0.0 && z_max > 0.0, "Om, h and z_max must be positive");
  std::vector<float> host;
  const float* rec = records;
  if (n > 0 && is_device_ptr(records)) {
    host.resize((size_t)n * nfields);
    PPB_CUDA(cudaMemcpy(host.data(), records, host.size() * 4, cudaMemcpyDeviceToHost));
    rec = host.data();
  }
  write_catalog_hdf5_host(path, rec, n, nfields, Om, OL, h, z_max);
  return PPB_OK;
  PPB_GUARD_END((ppb_ctx*)nullptr)
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

int32_t ppb_set_option(ppb_ctx* ctx, int32_t option, int64_t value) {
  if (!ctx) return PPB_ERR_INVALID;
  PPB_GUARD_BEGIN
  switch (option) {
    case PPB_OPT_GRAPHS:
      PPB_REQUIRE(value == 0 || value == 1, "PPB_OPT_GRAPHS takes 0 or 1");
      ctx->sh.use_graphs.store((int)value);
      break;
    case PPB_OPT_AUTOTUNE:
      PPB_REQUIRE(value >= 0 && value <= 2, "PPB_OPT_AUTOTUNE takes 0, 1 or 2");
      if (value == 2) {
        std::lock_guard<std::mutex> lk(ctx->sh.cache_mu);
        ctx->sh.tune.clear();
      }
      ctx->sh.autotune.store(value == 0 ? 0 : 1);
      break;
    case PPB_OPT_TUNE_MIN_PEAKS:
      PPB_REQUIRE(value >= 1, "PPB_OPT_TUNE_MIN_PEAKS must be >= 1");
      ctx->sh.tune_min_peaks.store(value);
      break;
    case PPB_OPT_BRICK_SHIFT:
      PPB_REQUIRE(value == -2 || value == -1 || (value >= 2 && value <= 5), "PPB_OPT_BRICK_SHIFT takes -2, -1 or 2..5");
      ctx->sh.force_brick.store((int)value);
      break;
    case PPB_OPT_COLLAPSE_THREADS:
      PPB_REQUIRE(value == 0 || value == 1 || value == 2 || value == 4 || value == 8,
                  "PPB_OPT_COLLAPSE_THREADS takes 0, 1, 2, 4 or 8");
      ctx->sh.force_collapse.store((int)value);
      break;
    case PPB_OPT_FUSED_X:
      PPB_REQUIRE(value >= -1 && value <= 1, "PPB_OPT_FUSED_X takes -1, 0 or 1");
      ctx->sh.fused_x.store((int)value);
      break;
    case PPB_OPT_GATHER_RING:
      PPB_REQUIRE(value == 0 || value == 1, "PPB_OPT_GATHER_RING takes 0 or 1");
      ctx->sh.gather_ring.store((int)value);
      break;
    case PPB_OPT_COLLAPSE_ORDER:
      PPB_REQUIRE(value >= -1 && value <= 1, "PPB_OPT_COLLAPSE_ORDER takes -1, 0 or 1");
      ctx->sh.collapse_order.store((int)value);
      break;
    case PPB_OPT_GATHER_TEX:
      PPB_REQUIRE(value >= -1 && value <= 1, "PPB_OPT_GATHER_TEX takes -1, 0 or 1");
      ctx->sh.gather_tex.store((int)value);
      break;
    default:
      throw Error{PPB_ERR_INVALID, "unknown or read-only option"};
  }
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_get_option(ppb_ctx* ctx, int32_t option, int64_t* value) {
  if (!ctx || !value) return PPB_ERR_INVALID;
  PPB_GUARD_BEGIN
  switch (option) {
    case PPB_OPT_GRAPHS: *value = ctx->sh.use_graphs.load(); break;
    case PPB_OPT_AUTOTUNE: *value = ctx->sh.autotune.load(); break;
    case PPB_OPT_TUNE_MIN_PEAKS: *value = ctx->sh.tune_min_peaks.load(); break;
    case PPB_OPT_BRICK_SHIFT: *value = ctx->sh.force_brick.load(); break;
    case PPB_OPT_COLLAPSE_THREADS: *value = ctx->sh.force_collapse.load(); break;
    case PPB_OPT_FUSED_X: *value = ctx->sh.fused_x.load(); break;
    case PPB_OPT_GATHER_RING: *value = ctx->sh.gather_ring.load(); break;
    case PPB_OPT_COLLAPSE_ORDER: *value = ctx->sh.collapse_order.load(); break;
    case PPB_OPT_GATHER_TEX: *value = ctx->sh.gather_tex.load(); break;
    case PPB_OPT_GRAPH_LAUNCHES:
    case PPB_OPT_GRAPH_INSTANTIATIONS:
    case PPB_OPT_GRAPH_UPDATES: {
      int64_t v[3];
      graph_counts(ctx, v);
      *value = v[option - PPB_OPT_GRAPH_LAUNCHES];
      break;
    }
    default:
      throw Error{PPB_ERR_INVALID, "unknown option"};
  }
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_tune_entries(ppb_ctx* ctx, ppb_tune_entry* out, int32_t cap, int32_t* n) {
  if (!ctx || !n || cap < 0 || (cap > 0 && !out)) return PPB_ERR_INVALID;
  PPB_GUARD_BEGIN
  std::lock_guard<std::mutex> lk(ctx->sh.cache_mu);
  *n = (int32_t)ctx->sh.tune.size();
  int32_t i = 0;
  for (const auto& kv : ctx->sh.tune) {
    if (i >= cap) break;
    ppb_tune_entry e{};
    e.n = (int32_t)kv.first[0];
    e.nshell = (int32_t)kv.first[1];
    e.comp = (int32_t)kv.first[2];
    e.adaptive = (int32_t)kv.first[3];
    e.limited = (int32_t)kv.first[4];
    e.long_walk = (int32_t)kv.first[5];
    e.brick_shift = kv.second.brick_shift;
    e.collapse_threads = kv.second.collapse_threads;
    e.npk = kv.second.npk;
    std::memcpy(e.gather_ms, kv.second.gather_ms, sizeof(e.gather_ms));
    std::memcpy(e.collapse_ms, kv.second.collapse_ms, sizeof(e.collapse_ms));
    e.collapse_order = kv.second.collapse_order ? 1 : 0;
    e.gather_tex = kv.second.gather_tex ? 1 : 0;
    e.gather_plain_ms = kv.second.gather_plain_ms;
    std::memcpy(e.collapse_ordered_ms, kv.second.collapse_ordered_ms, sizeof(e.collapse_ordered_ms));
    out[i++] = e;
  }
  return PPB_OK;
  PPB_GUARD_END(ctx)
}

int32_t ppb_last_stage_ms(ppb_ctx* ctx, float* ms4) {
  if (!ctx || !ms4) return PPB_ERR_INVALID;
  std::memcpy(ms4, ctx->sync.stage_ms, sizeof(ctx->sync.stage_ms));
  return PPB_OK;
}

}  // extern "C"
