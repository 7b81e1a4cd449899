// ppb_ctx.h — the library context (one per GPU), its execution slots and the
// resident tables the slots share.
#pragma once
#include <array>
#include <atomic>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <shared_mutex>
#include <string>

#include "ppb_internal.h"

namespace ppb {

// plans and device buffers for one grid size n
struct TileRes {
  int n = 0;
  cufftHandle r2c = 0, c2r1 = 0, c2r2 = 0, c2r3 = 0, c2r6 = 0;
  // in-place inverse C2C of contiguous n x n (kz, ky) planes, batched over
  // the n/2+1 kx of one field (yz1) or of two fields back to back (yz2): the
  // filter bank's transforms before the fused x pass (0 where unsupported)
  cufftHandle yz1 = 0, yz2 = 0;
  DevBuf delta, dk, psi, psi2, lapd, aos, kw, rw, mask, count, wtab;
  DevBuf xtw;   // exp(2 pi i k / n), k < n: the fused x pass's twiddles
  // peaks
  int64_t cap = 0;
  DevBuf keys, vals, ff, lap, keys_s, vals_s, tmp;
  DevBuf p_lin, p_Rf, p_ir2, p_np, p_Z, p_fc, p_FcRf, p_d2Rf, p_pos, res, flags, offs, rec, rthl;
  // executable graphs that hold this grid size's cuFFT plans (fields, filter
  // bank): they live exactly as long as the plans whose kernels they launch
  std::map<std::pair<int, int64_t>, cudaGraphExec_t> graphs;
  ~TileRes();
  void setup(int n, cudaStream_t s);
  // the fused filter bank's plans, twiddle buffer and kernel attribute, made
  // the first time a filter bank of this size takes that path (outside capture)
  void setup_fused(cudaStream_t s);
  void ensure_peaks(int64_t c);
  size_t bytes() const;
};

// the zero-padded isolated convolution of one padded size n2 (multires.cu):
// in-place transforms over one cuFFT work area
struct IsoRes {
  int n2 = 0, batch = 0;
  // pruned in-place transforms: 2-D (y, x) over n2/2 z-planes (forward: the
  // planes holding the input; inverse: the planes holding the wanted output)
  // and the 1-D z transform of every column
  cufftHandle f2d = 0, i2d = 0, col = 0;
  DevBuf spec;   // the padded input (row pitch 2 (n2/2+1) floats), then its half-spectrum
  DevBuf work;   // `batch` half-spectra, each then transformed back in place
  DevBuf ws;     // cuFFT work area of the plans
  DevBuf amp;    // transfer amplitude by integer |freq|^2 for box amp_box and P(k) version amp_pk
  double amp_box = 0.0;
  int64_t amp_pk = -1;
  ~IsoRes();
  // plans and buffers for padded size n2 and up to `batch` kernels per pass
  void setup(int n2, int batch, cudaStream_t s);
  size_t bytes() const { return spec.bytes + work.bytes + ws.bytes + amp.bytes; }
};

// one autotuned shell-stage configuration: the gather order brick and the
// collapse threads per peak, with the timings of every candidate
struct TuneEntry {
  int brick_shift = 3;        // -1: list order
  int collapse_threads = 0;   // 0: the size heuristic
  int64_t npk = 0;            // peaks of the batch it was measured on
  float gather_ms[5] = {};    // bricks of 4, 8, 16, 32 cells and list order
  float collapse_ms[4] = {};  // 1, 2 and 4 threads per peak, lane queues
  bool collapse_order = false;            // peaks by descending crossing shell
  float collapse_ordered_ms[4] = {};      // the same widths with that order
  bool gather_tex = true;                 // records through the texture pipe
  float gather_plain_ms = 0.f;            // the chosen brick with 256-bit loads instead
};

struct ShellStats {
  unsigned long long visits = 0, guard = 0, akk = 0;
  unsigned long long dump[5] = {0, 0, 0, 0, 0};
  unsigned long long raw[16] = {};
  float ms = 0.f;                        // the whole stage
  float kms[4] = {0.f, 0.f, 0.f, 0.f};   // gather, collapse, zvir_half, d2f kernels
  unsigned long long pool_rows = 0;      // profile rows written
  int batches = 0;
};

// An execution slot: one CUDA stream and every buffer a tile run writes.
// Runs on different slots overlap on the device; one slot runs one tile at a
// time.
struct Slot {
  int device = 0;
  cudaStream_t stream = nullptr;
  int64_t launches = 0;
  cudaEvent_t stage_ev[5] = {};
  cudaEvent_t shell_ev[5] = {};
  float stage_ms[4] = {0, 0, 0, 0};
  std::map<int, std::unique_ptr<TileRes>> tiles;    // resident grid sizes (buffers, plans, graphs)
  std::vector<int> tile_lru;                        // resident sizes, least recently used first
  int max_tiles = 4;                                // sizes kept resident at most
  DevBuf filt_Rf, filt_ir2, filt_np;                // filter bank of the run
  DevBuf g_a, g_D, g_f, chi;                        // growth / chi tables of the run
  DevBuf stage, counters, ctl, hdr, geo, mlim, pool, anchors;   // shell stage
  // merge_catalog's buffers, kept between calls (a cudaFree waits for the
  // whole device)
  struct MergeBufs {
    DevBuf in, out, x, y, z, r, cell, cstart, cfill, cidx, rank, scount, sups, state, changed, rnew, key, key2, idx,
        idx2, tmp, flag, off, dom;
    void release() {
      for (DevBuf* b : {&in, &out, &x, &y, &z, &r, &cell, &cstart, &cfill, &cidx, &rank, &scount, &sups, &state,
                        &changed, &rnew, &key, &key2, &idx, &idx2, &tmp, &flag, &off, &dom})
        b->release();
    }
    size_t bytes() const {
      size_t t = 0;
      for (const DevBuf* b : {&in, &out, &x, &y, &z, &r, &cell, &cstart, &cfill, &cidx, &rank, &scount, &sups, &state,
                              &changed, &rnew, &key, &key2, &idx, &idx2, &tmp, &flag, &off, &dom})
        t += b->bytes;
      return t;
    }
  } merge;
  // the gather's texture object over a record array (rec_ptr, rec_bytes);
  // 0 when none or when the array is past the device's linear-texture limit
  cudaTextureObject_t rec_tex = 0;
  const void* rec_ptr = nullptr;
  size_t rec_bytes = 0;
  cudaTextureObject_t record_texture(const float4* aos, int n);
  void drop_record_texture();
  DevBuf okey, okey2, oidx, oidx2, otmp;            // spatial gather order
  DevBuf tcen, tcount, t_aos, t_lapd;               // multi-tile: centres, peaks per tile, tile fields
  std::unique_ptr<IsoRes> iso;                      // multi-resolution: isolated convolution
  DevBuf mr_in, mr_out, mr_aux, mr_rec;             // multi-resolution: staged inputs, outputs, records
  DevBuf mr_axis, mr_amp;                           // multi-resolution: tricubic axis tables, coarse amplitudes
  DevBuf pft;                                       // ppb_peak_find_tile: unpacked (i, j, k), ipp, filter
  int gather_bps[2][2][2] = {};                      // gather blocks per SM by [comp][adaptive][ring]
  double rows_per_peak[2] = {0.0, 0.0};             // pool rows per peak seen last, by adaptive
  double walk_per_peak = 0.0;                       // collapse-walk steps per peak seen last
  ShellStats last_shell{};
  int64_t last_visits = 0, last_npk = 0;
  // executable graphs of the shell stage (own and CUB kernels only) by
  // (call site, shape key); updated in place from each new capture,
  // re-instantiated when the launch sequence changed shape
  std::map<std::pair<int, int64_t>, cudaGraphExec_t> graphs;
  int64_t graph_launches = 0, graph_instantiations = 0, graph_updates = 0;
  DevBuf tune_save;                                 // counters saved around a tuning pass
  void init(int device);
  void release_buffers();
  size_t bytes_held() const;
  size_t shell_bytes() const;   // held outside the per-size buffers (shell stage and tables)
  // the buffers of grid size n: kept from an earlier run of that size when
  // resident, else new, after dropping least recently used sizes while more
  // than max_tiles - 1 are resident or free memory is short of n's estimate
  TileRes& tile_for(int n);
  bool has_tile(int n) const { return tiles.count(n) != 0; }
  // least recently used resident size other than `keep` (0: none)
  int lru_tile(int keep) const;
  // frees the buffers of size n; returns the bytes freed
  uint64_t drop_tile(int n);
  ~Slot();
};

// outputs of ppb_peak_find_tile (host or device pointers; any may be null
// except npeaks): capacity entries each
struct PeakTileOut {
  int64_t capacity = 0;
  int32_t *pi = nullptr, *pj = nullptr, *pk = nullptr;
  int64_t* ipp = nullptr;
  double *x = nullptr, *y = nullptr, *z = nullptr;
  float* FcRf = nullptr;
  double* Rf = nullptr;
  float* d2Rf = nullptr;
  int32_t* filter = nullptr;
  int64_t* npeaks = nullptr;
};

// the record buffer of a finished run, still on the device
struct TileOut {
  const float* d_records = nullptr;
  int64_t count = 0;
  int32_t nfields = 0;
  float RTHLmax = 0.f;
  int64_t npeaks = 0;
  float device_ms = 0.f;
};

// Resident tables shared by all slots.  `mu` is held shared by every run
// and exclusively by the table uploads; `cache_mu` guards the lazily built
// caches (entries are never removed while the context lives, so references
// handed out stay valid).
struct Shared {
  std::shared_mutex mu;
  DevBuf pk_lk, pk_lp;
  int pk_n = 0;
  int64_t pk_version = 0;   // incremented by every P(k) upload
  DevBuf tab;
  bool has_tab = false;
  DevTable dtab{};
  DevBuf akk;
  std::mutex cache_mu;
  std::map<int, std::unique_ptr<ShellTable>> shells;                           // by nhunt
  std::map<std::array<double, 4>, std::unique_ptr<GrowthTable>> growth;        // by (Om, OB, OL, h)
  std::map<std::array<double, 4>, std::unique_ptr<std::vector<double>>> chi;   // by (Om, OL, h, zmax)
  // autotuned shell-stage choices by (n, nshell, comp, adaptive, per-peak
  // limits, long collapse walks)
  std::map<std::array<int64_t, 6>, TuneEntry> tune;
  // options (ppb_set_option)
  std::atomic<int> use_graphs{1};
  std::atomic<int> autotune{1};
  std::atomic<int> fused_x{-1};   // PPB_OPT_FUSED_X
  std::atomic<int> gather_ring{0};   // PPB_OPT_GATHER_RING
  std::atomic<int> collapse_order{-1};   // PPB_OPT_COLLAPSE_ORDER (-1: tuner's choice)
  std::atomic<int> gather_tex{-1};       // PPB_OPT_GATHER_TEX (-1: tuner's choice)
  std::atomic<int64_t> tune_min_peaks{16384};
  std::atomic<int> force_brick{-2};      // -2: tuner's choice
  std::atomic<int> force_collapse{0};    // 0: tuner's choice
};

struct Server;   // serve.cu

}  // namespace ppb

struct ppb_ctx {
  int device = 0;
  int nsm = 148;
  std::recursive_mutex mu;   // serialises the synchronous entry points
  std::mutex err_mu;
  std::string err;
  uint64_t hbm_budget = 0;
  cudaEvent_t ev[16] = {};   // user events on the synchronous slot's stream
  ppb::Shared sh;
  ppb::Slot sync;            // the slot of the synchronous entry points
  std::unique_ptr<ppb::Server> server;
  int serve_slots = 4;
  float table_ms = 0.f;        // last ppb_make_collapse_table: device time
  int64_t table_steps = 0;     // and RK4 steps over all nodes

  void set_error(const std::string& m);
  const ppb::GrowthTable& growth(double Om, double OB, double OL, double h);
  const std::vector<double>& chi_table(double Om, double OL, double h, double zmax);
  ppb::ShellTable& shell_table(int nhunt, cudaStream_t s);
  ppb::DevCosmo dev_cosmo(ppb::Slot& sl, const ppb::GrowthTable& G, double Om, double OL, double h, double zmax,
                          bool need_chi);
  ppb::ShellArgs shell_args(ppb::Slot& sl, ppb::ShellTable& st, int n, double alatt, const float4* aos,
                            const float* lapd);
  // the shell stage of a peak batch: geometry, spatial order, gather,
  // collapse, zvir_half, d2F, in pool-sized sub-batches; `pre` records
  // launches that run ahead of the first sub-batch in the same graph
  void run_shells(ppb::Slot& sl, ppb::ShellArgs& a, bool comp, bool adaptive, ppb::ShellStats* st,
                  const std::function<void()>& pre = nullptr);
  // times the order bricks and collapse widths on one sub-batch and keeps the
  // fastest for the batch's tuning key (outputs are the same for every choice)
  ppb::TuneEntry tune_shells(ppb::Slot& sl, const ppb::ShellArgs& b, bool comp, bool adaptive, int gblocks,
                            const void* ring_map);
  // records the launches of `rec` on the slot's stream into the graph for
  // (site, key) of `graphs` and launches it; with graphs off, runs `rec`
  // directly.  A graph that launches cuFFT kernels must be kept in the map of
  // the TileRes that owns the plans.
  void captured(ppb::Slot& sl, std::map<std::pair<int, int64_t>, cudaGraphExec_t>& graphs, int site, int64_t key,
                const std::function<void()>& rec);
  int64_t launches_total() const;
  ppb_ctx();
  ~ppb_ctx();
};

namespace ppb {
// run_tile (src/Pipeline.jl:66-325) on one slot; the records stay on the
// device (o->d_records) until the slot's next run.  The caller holds
// ctx->sh.mu shared.
void run_tile_core(ppb_ctx* ctx, Slot& sl, const ppb_tile_params* p, const double* Rf, int nfilt, TileOut* o);
// run_multitile (src/MultiTile.jl:108-418) on one slot; tiles = ntiles
// (it, jt, kt) triples, 1-based, or null for every tile of the ntile^3 grid
void run_multitile_core(ppb_ctx* ctx, Slot& sl, const ppb_tile_params* p, const double* Rf, int nfilt, int ntile,
                        const int32_t* tiles, int ntiles, TileOut* o);
// run_multitile_split (src/MultiResolution.jl:523-1236) on one slot: fields
// by the multi-resolution split per tile, analysed on the tile's own grid;
// records in tile order (o->d_records stays valid until the slot's next
// split run)
void run_multitile_split_core(ppb_ctx* ctx, Slot& sl, const ppb_tile_params* p, const double* Rf, int nfilt,
                              int ntile, int coarse_factor, int coarse_grid, const int32_t* tiles, int ntiles,
                              TileOut* o);
// the coarse grid M the split uses (coarse_grid, ntile coarse_factor, or the
// automatic choice of src/MultiResolution.jl:592-612)
int split_coarse_grid(int64_t N, int nmesh, int ntile, int coarse_factor, int coarse_grid);
void check_params(const ppb_tile_params* p, const double* Rf, int nfilt);
// peak_find_tile_gpu (src/PeakPatch.jl:341-366): rfft of the caller's field,
// then per filter (in the given order) the window, the inverse transform and
// the peak search with per-filter fcrit and the caller's mask (read and
// updated); peaks in (filter, scan) order.  *o.npeaks receives the count;
// PPB_ERR_CAPACITY (mask untouched) when it exceeds o.capacity.
void peak_find_tile_core(ppb_ctx* ctx, Slot& sl, const float* delta, int n, const double* Rf, const double* fcrit,
                         int nfilt, int8_t* mask, double xbx, double ybx, double zbx, double alatt, int nbuff,
                         int wsmooth, int ioutshear, const PeakTileOut& o);
// the fields of run_tile's first phase, copied to the given buffers (host or
// device, any may be null)
void generate_fields_core(ppb_ctx* ctx, Slot& sl, const ppb_tile_params* p, float* delta, float* psi, float* psi2,
                          float* lapd);
// device bytes a run of this grid size holds at most (admission estimate)
uint64_t tile_footprint(const ppb_tile_params* p);
// the part of it held per grid size (TileRes) and per slot (shell stage)
uint64_t tile_bytes_estimate(int n);
// peak-buffer capacity given to a grid of N cells on its first run
int64_t initial_peak_capacity(int64_t N);
uint64_t shell_bytes_estimate(int n);
// copy `bytes` from device memory to dst (host or device)
void copy_out(void* dst, const void* src, size_t bytes, cudaStream_t s);
// true when p points to device memory
bool is_device_ptr(const void* p);
// device copy of a caller buffer (host or device); returns a device pointer
const void* stage_in(DevBuf& buf, const void* src, size_t bytes, cudaStream_t s);
// merge_catalog on device records (n x nf floats); writes the survivors in
// index order to d_out (capacity n) and returns their number (k_merge.cu)
int64_t merge_catalog_device(Slot& sl, const float* d_rec, int64_t n, int nf, float* d_out);
// serving (serve.cu)
void server_stop(ppb_ctx* ctx);
// graph launches, instantiations and in-place updates over every slot
void graph_counts(const ppb_ctx* ctx, int64_t* out3);
// make_table's RK4 integrations on the device (k_table.cu): d_Frho holds
// 10^x of the Nx log10 F nodes; d_out the Nx Ny Nz node values; d_steps
// accumulates the RK4 steps taken
void make_table_device(Slot& sl, const GrowthTable& G, const ppb_table_params* p, const double* d_Frho, double* d_out,
                       unsigned long long* d_steps);
// multi-resolution stages on device buffers (multires.cu).  The coarse phase
// writes delta, psi (3), psi2 (3, ilpt >= 2) and lapd (ioutshear >= 1) of the
// M^3 coarse noise to o, fields fs floats apart (fs a multiple of 4).
void mr_coarse_device(ppb_ctx* ctx, Slot& sl, const float* d_noise, int M, double boxsize_full, int ilpt,
                      int ioutshear, float* o, int64_t fs);
// isolated convolution of the n_input^3 noise for nk (kind, d1, d2) kernels,
// the n^3 region at nshell into outs[b]; the caller holds ctx->sh.mu shared
void mr_isolated_device(ppb_ctx* ctx, Slot& sl, const float* d_noise, int n_input, double boxsize_local, int n,
                        const int32_t* kernels, int nk, int nshell, float* const* outs);
// the split's tile fields into T.delta and T.psi: residual of the tile at
// origin (i0, j0, k0) straight into the padded box, one forward transform,
// the delta and psi kernels, one batched inverse transform, plus the
// tricubic coarse fields cf4 (delta, psi x3 interleaved as float4) in one
// pass; the caller holds ctx->sh.mu shared
void mr_split_tile_fields(ppb_ctx* ctx, Slot& sl, TileRes& T, const float* cnoise, const float* cf4, int M, int64_t N,
                          int64_t i0, int64_t j0, int64_t k0, int nm, double box_local, uint64_t seed);
// tile-local 2LPT (psi2: 3 fields n^3 apart) and/or Laplacian of T.delta;
// leaves T.dk = rfft(T.delta)
void mr_tile_2lpt_lap(ppb_ctx* ctx, Slot& sl, TileRes& T, int n, double box, float* psi2, float* lapd);
}  // namespace ppb
