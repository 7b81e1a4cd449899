// ppb_ctx.h — the library context (one per GPU) and per-grid-size resources.
#pragma once
#include <map>
#include <memory>
#include <mutex>
#include <string>

#include "ppb_internal.h"

namespace ppb {

// plans and device buffers for one grid size n
struct TileRes {
  int n = 0;
  cufftHandle r2c = 0, c2r1 = 0, c2r2 = 0, c2r3 = 0, c2r6 = 0;
  DevBuf delta, dk, psi, psi2, lapd, aos, kw, rw, mask, count, wtab;
  // peaks
  int64_t cap = 0;
  DevBuf keys, vals, ff, lap, keys_s, vals_s, tmp;
  DevBuf p_lin, p_Rf, p_ir2, p_Z, p_fc, p_FcRf, p_d2Rf, p_pos, res, flags, offs, rec, rthl;
  ~TileRes();
  void setup(int n, cudaStream_t s);
  void ensure_peaks(int64_t c);
};

struct ShellStats {
  unsigned long long visits = 0, guard = 0, akk = 0;
  unsigned long long dump[5] = {0, 0, 0, 0, 0};
  unsigned long long raw[16] = {};
  float ms = 0.f;                 // the whole stage
  float kms[4] = {0.f, 0.f, 0.f, 0.f};   // gather, collapse, zvir_half, d2f kernels
  unsigned long long pool_rows = 0;   // profile rows written
  int batches = 0;
};

}  // namespace ppb

struct ppb_ctx {
  int device = 0;
  int nsm = 148;
  cudaStream_t stream = nullptr;
  std::recursive_mutex mu;
  std::string err;
  int64_t launches = 0;
  cudaEvent_t ev[16] = {};
  cudaEvent_t stage_ev[5] = {};
  float stage_ms[4] = {0, 0, 0, 0};
  uint64_t hbm_budget = 0;
  // resident tables
  ppb::DevBuf pk_lk, pk_lp;
  int pk_n = 0;
  ppb::DevBuf tab;
  bool has_tab = false;
  ppb::DevTable dtab{};
  ppb::DevBuf akk;
  ppb::ShellTable shells;
  ppb::DevBuf stage, counters, ctl, hdr, geo, pool;
  cudaEvent_t shell_ev[5] = {};
  int gather_bps[2][2] = {{0, 0}, {0, 0}};    // gather blocks per SM by [comp][adaptive]
  double rows_per_peak[2] = {0.0, 0.0};       // pool rows per peak seen last, by adaptive
  ppb::DevBuf filt_Rf, filt_ir2;
  ppb::DevBuf g_a, g_D, g_f, chi;
  // growth-table cache
  double gkey[4] = {-1, -1, -1, -1};
  ppb::GrowthTable gcache;
  double chikey[4] = {-1, -1, -1, -1};
  std::vector<double> chicache;
  std::map<int, std::unique_ptr<ppb::TileRes>> tiles;
  int64_t last_visits = 0, last_npk = 0;
  ppb::ShellStats last_shell{};

  const ppb::GrowthTable& growth(double Om, double OB, double OL, double h);
  ppb::DevCosmo dev_cosmo(const ppb::GrowthTable& G, double Om, double OL, double h, double zmax, bool need_chi);
  ppb::TileRes& tile(int n);
  ppb::ShellArgs shell_args(int n, double alatt, const float4* aos, const float* lapd);
  void run_shells(ppb::ShellArgs& a, bool comp, bool adaptive, ppb::ShellStats* st);
};

namespace ppb {
int run_tile_impl(ppb_ctx* ctx, const ppb_tile_params* p, const double* Rf, int nfilt, ppb_halo_buf* out,
                  float* device_ms);
// copy `bytes` from device memory to dst (host or device)
void copy_out(void* dst, const void* src, size_t bytes, cudaStream_t s);
// true when p points to device memory
bool is_device_ptr(const void* p);
// device copy of a caller buffer (host or device); returns a device pointer
const void* stage_in(DevBuf& buf, const void* src, size_t bytes, cudaStream_t s);
}  // namespace ppb
