// ppb_internal.h — shared declarations of libppb (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ppb.h"

namespace ppb {

// ---------------------------------------------------------------------------
// error plumbing: every failing CUDA call is turned into a status + message
// ---------------------------------------------------------------------------
struct Error {
  int32_t code;
  std::string msg;
};

#define PPB_CUDA(call)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      throw ::ppb::Error{e_ == cudaErrorMemoryAllocation ? PPB_ERR_NOMEM : PPB_ERR_CUDA,  \
                         std::string(#call) + ": " + cudaGetErrorString(e_)};             \
  } while (0)

#define PPB_CUFFT(call)                                                                   \
  do {                                                                                    \
    cufftResult r_ = (call);                                                              \
    if (r_ != CUFFT_SUCCESS)                                                              \
      throw ::ppb::Error{r_ == CUFFT_ALLOC_FAILED ? PPB_ERR_NOMEM : PPB_ERR_CUDA,         \
                         std::string(#call) + ": cufft status " + std::to_string((int)r_)}; \
  } while (0)

#define PPB_REQUIRE(cond, msg)                                                            \
  do {                                                                                    \
    if (!(cond)) throw ::ppb::Error{PPB_ERR_INVALID, std::string(msg)};                   \
  } while (0)

// after each kernel launch: catch launch-configuration errors immediately
#define PPB_LAUNCHED(ctr)                                                                 \
  do {                                                                                    \
    PPB_CUDA(cudaGetLastError());                                                         \
    (ctr)++;                                                                              \
  } while (0)

// ---------------------------------------------------------------------------
// device buffers
// ---------------------------------------------------------------------------
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  void ensure(size_t b) {
    if (b <= bytes) return;
    release();
    PPB_CUDA(cudaMalloc(&p, b));
    bytes = b;
  }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// ---------------------------------------------------------------------------
// geometry of the sorted shell-cell list (precompute_shells)
// ---------------------------------------------------------------------------
constexpr int kChunkCells = 24;   // gather chunk size (cells per lane per group; smaller for short lists)

struct ShellTable {
  int nhunt = -1;
  int64_t ncells = 0;                 // cells with r2 <= nhunt^2 (including the centre)
  int nshell = 0;                     // distinct r2 values (including 0)
  std::vector<int4> cells;            // (di, dj, dk, r2), stable-sorted by r2
  std::vector<int32_t> shell_start;   // per distinct r2 value: first cell index
  std::vector<int32_t> shell_count;
  std::vector<int32_t> shell_r2;
  std::vector<double> rad;            // rad[m] (m = 0..nshell), rad[1] = 0
  std::vector<int32_t> r2m;           // r2 of shell m (m = 0..nshell)
  // kernel_strain weights (RadialShell.jl:234-253): for centre shell mp >= 2
  // the shells m1 with (rad[mp] - rad[m1])^2 < 4 form the contiguous window
  // [win_lo[mp], win_hi[mp]]; wts[win_off[mp] + (m1 - win_lo[mp])] holds
  // hRinteg(u0, u12) / (u12 - u0^2)^2 for that pair.
  std::vector<int32_t> win_lo, win_hi, win_off;
  std::vector<double> wts;
  // mp == 1 weights 0.5 * akk(rad[m1]) / rad[m1] (:255-271); NaN where the
  // reference's akk lookup would run past the table
  std::vector<double> w1;
  // first shell m' with rad[m'] > rad[m] + 2, plus one (gather truncation)
  std::vector<int32_t> need;
  // rad[m]^5 (Srb integral, RadialShell.jl:776-790)
  std::vector<double> rad5;
  // gather schedule: shells m >= 2 split into chunks of at most
  // kChunkCells cells; consecutive chunks packed into groups of at most 32
  // (one chunk per lane) that end on a shell boundary.  Group g covers shells
  // [grp_a[g], grp_b[g]] and chunks [grp_c[g], grp_c[g+1]); chunk c holds
  // ck_n[c] cells from ck_s[c]; shell m's chunks start at sh_c0[m] (sh_nc[m]).
  std::vector<int32_t> grp_a, grp_b, grp_c, ck_s, ck_n, ck_d, sh_c0, sh_nc;
  int ngroups = 0;
  // cell offsets packed one per 32-bit word: bytes 0..2 = di, dj, dk as
  // signed 8-bit values (|d| <= nhunt <= 64)
  std::vector<int32_t> cell8;
  // the packed offsets again, chunk by chunk, each chunk starting on a
  // 16-byte boundary (zero padding), so that a gather lane reads the offsets
  // of four consecutive cells of its chunk with one 16-byte load; chunk c
  // starts at ck_cells[4 ck_p[c]]
  std::vector<int32_t> ck_p, ck_cells;
  DevBuf d_cell8, d_start, d_count, d_r2m, d_rad, d_wlo, d_whi, d_woff, d_wts, d_w1, d_need, d_rad5;
  DevBuf d_grp_a, d_grp_b, d_grp_c, d_ck_s, d_ck_n, d_ck_d, d_sh_c0, d_sh_nc, d_ck_p, d_ck_cells;
};
void build_shell_table(ShellTable& st, int nhunt);
double hRinteg(double u0, double u12);
std::vector<double> make_atab4();
void upload_shell_table(ShellTable& st, cudaStream_t s);

// ---------------------------------------------------------------------------
// linear-growth and chi->z tables (host, double precision)
// ---------------------------------------------------------------------------
struct GrowthTable {
  std::vector<double> a, D, f;
  double amin = 0, amax = 0, Dinf = 0, D0 = 0, Hinf = 0, H0 = 0;
};
GrowthTable make_growth_table(double Om, double OB, double OL, double h);
void dlinear_ab(const GrowthTable& G, double ai, double* Dl, double* HD, double* Da);
double fsc_of_z(const GrowthTable& G, double z);
std::vector<double> make_chi_table(double Om, double OL, double h, double zmax, int npts);
// write_catalog_hdf5 of n host records (11 or 33 floats each) to path
void write_catalog_hdf5_host(const std::string& path, const float* rec, int64_t n, int nf, double Om, double OL,
                             double h, double z_max);
// comoving distance to z (Mpc/h) and its inverse on a make_chi_table table
// spanning [0, zmax] (chi_to_z, Cosmology.jl:155-169)
double chi_of_z(double Om, double OL, double h, double z);
double chi_to_z_host(const std::vector<double>& chis, double zmax, double c);

// device view of the tables used per peak (lightcone ZZon / fcrit / D(z))
struct DevCosmo {
  const double* ga;   // growth a
  const double* gD;   // D(a)/a normalised
  const double* gf;   // dlnD/dlna
  int ng;
  double amin, amax, Dinf, D0, Hinf, H0;
  const double* chis;  // chi(z_i), z_i = zmax * i/(npts-1)
  int nchi;
  double chi_zmax;
};

// collapse table on the device
struct DevTable {
  const float* t;     // Float32 nodes (read_homeltab), or
  const double* td;   // Float64 nodes (set when t is null)
  int nx, ny, nz;
  double x1, x2, y1, y2, z1, z2;
};

// ---------------------------------------------------------------------------
// per-peak parameters and results on the device
// ---------------------------------------------------------------------------
constexpr int RES_N = 31;   // doubles per peak result (layout in ppb.h)

struct PeakParams {          // SoA, length npk
  const int64_t* lin;       // 0-based flat index i + n j + n^2 k
  const double* Rf;
  const int32_t* ir2min;
  const double* ZZon;
  const double* fcrit;
};

// Per-shell profile row of one peak (ROW doubles, written by the gather
// kernel, read by the collapse kernel).  The first 16 values are what a
// kernel_strain window reads, the rest what Sbar/Srb read.
constexpr int ROW = 24;
// the shell stage's control words (ShellArgs::queue, cqueue, pool_ctr)
constexpr size_t kCtlBytes = 64;
enum {
  R_FBAR = 0,   // cumulative mean overdensity Fbar (RadialShell.jl:386-390)
  R_G = 1,      // sum delta * d / r            (3)
  R_GF = 4,     // sum deltaT * d / r           (3)
  R_Q = 7,      // sum psi_L d_K / r, symmetric (6: xx yy zz xy xz yz)
  R_N = 16,     // in-grid cells of the shell
  R_S = 17,     // sum psi1                     (3)
  R_S2 = 20     // sum psi2                     (3)
};

// gather -> collapse hand-off, one per peak
enum { HS_OK = 0, HS_NOFCRIT = 1, HS_M0ONE = 2, HS_BAD = 3, HS_OVERFLOW = 4 };
struct PeakHdr {
  long long off;   // first pool row of the peak (row m of shell m at off + m)
  int mdone;       // shells 1..mdone gathered
  int m0;          // fcrit crossing shell (RadialShell.jl:494-537)
  int status;      // HS_*
  int pad;
};

struct ShellArgs {
  const float4* aos;        // 2 float4 per cell: (delta, deltaT, psi1z, psi2x), (psi1x, psi1y, psi2y, psi2z)
  const float* lapd;        // may be null
  int n;
  double alatt;
  // shell geometry
  const int32_t* cell8;     // packed cell offsets (ShellTable::cell8)
  const int32_t* ck_p;      // chunk starts in ck_cells, in 16-byte units
  const int4* ck_cells;     // packed cell offsets, chunk-major (ShellTable::ck_cells)
  const int32_t* sh_start;
  const int32_t* sh_count;
  const double* rad;        // rad[m], m = 0..nshell (index 0 unused); rad[1] = 0
  const int32_t* r2m;       // r^2 of shell m, m = 1..nshell (shell nshell is the unfinalised last group)
  const int32_t* win_lo;    // kernel_strain windows and weights (see ShellTable)
  const int32_t* win_hi;
  const int32_t* win_off;
  const double* wts;
  const double* w1;
  const int32_t* need;
  const double* rad5;
  const int32_t *grp_a, *grp_b, *grp_c, *ck_s, *ck_n, *sh_c0, *sh_nc;
  int ngroups;
  int nshell;               // distinct r2 values in the list (incl. 0)
  int mmax;                 // finalised shells: nshell - 1
  int64_t npart;            // cells used (full list here)
  int nck;                  // chunks of the schedule
  const int32_t* ck_d;      // per chunk: largest |offset component| of its cells
  float2* ck_K;             // per chunk: the compensated sums' anchors (kAnchorStride float2)
  unsigned long long rec_tex;   // texture object over aos (float4 elements), 0: plain loads
  const unsigned* fmax;     // the field maxima after the records (pack_fmax)
  DevTable tab;
  const double* akk;        // 1101-entry SPH kernel table
  PeakParams pk;
  int64_t npk;
  double* out;              // npk x RES_N
  PeakHdr* hdr;             // npk
  const int32_t* corder;    // npk or null: the order the collapse kernels take the peaks in
  int4* geo;                // 2 npk: (m0_init, mrf, mlow_rf, mupp_rf), (i, j, k of the peak cell, flags)
  const int32_t* r2lim;     // npk or null: per-peak shell list r^2 <= r2lim (> 0), else the whole list
  const int32_t* npcap;     // npk or null: per-peak cell count npart (the rmax2rs cap of RadialShell.jl:288-295)
  int32_t* mlim;            // npk: the peak's last finalised shell (written by the geometry kernel)
  double* pool;             // profile rows, pool_cap rows of ROW doubles
  int64_t pool_cap;
  unsigned long long* pool_ctr;   // rows handed out
  double* stage;            // per-warp staging rows of the gather kernel
  int64_t stage_stride;     // doubles per warp slot
  double fhalf[10];         // ((e/9) / 2 + 1/2)^(1/3), e = 0..9 (zvir_half radii)
  int* queue;               // work counter for the persistent gather kernel
  int* cqueue;              // work counter of the collapse lane queues
  const int32_t* order;     // gather order (queue position -> peak), null: list order
  int brick_shift;          // gather order key: Morton index of the peak's 2^brick_shift-cell brick
  unsigned long long* counters;   // [0] cell visits, [1..5] dump reasons
};

// ---------------------------------------------------------------------------
// kernel launchers (k_*.cu)
// ---------------------------------------------------------------------------
struct Launch {
  cudaStream_t s;
  int64_t* count;
};

void launch_noise(Launch L, float* out, int64_t n, uint64_t seed);
// pk_scale multiplies P(k) (a sigma8 rescale is pk_scale = (sigma8 / sigma8_table)^2)
void launch_convolve(Launch L, float2* nk, int n, double boxsize, const double* lk, const double* lp,
                     int np, double pk_scale, double post_scale);
void launch_lpt1(Launch L, const float2* dk, float2* out, int n, double boxsize, double post_scale);
void launch_phi(Launch L, const float2* dk, float2* out, int n, double boxsize, double post_scale);
void launch_src2(Launch L, const float* phi, float* out, int64_t N);
void launch_lpt2(Launch L, const float2* s2k, float2* out, int n, double boxsize, double post_scale);
void launch_lapd(Launch L, const float2* dk, float2* out, int n, double boxsize, float post_scale);
// window tables: per filter f, window_table_size(n) float pairs (W_wsmooth,
// the k^2-weighted Gaussian of the Laplacian diagnostic) by integer |k|^2 at
// tab + f * 2 * window_table_size(n); Rf is a device array of nfilt radii
int window_table_size(int n);
void launch_window_tables(Launch L, float* tab, int n, double boxsize, const double* Rf, int nfilt, int wsmooth,
                          bool want_lap);
void launch_window(Launch L, const float2* dk, float2* out0, float2* out1, int n, const float* tab,
                   double post_scale);
void launch_hermitise(Launch L, float2* data, int n, int nbatch);
// a cubic window of fields on a larger grid: element (x, y, z) of the window
// is at off + x + py y + pz z; the psi components are cs apart
struct FieldWindow {
  const float* delta;
  const float* psi;
  const float* psi2;   // may be null
  int64_t off, py, pz, cs;
};
// packed gather records (two float4 per cell) of an n^3 window
// The packed records of an n^3 window (two float4 halves per cell) are
// followed by the largest magnitude of each field (delta, psi x, y, z, psi2
// x, y, z) as float bits, kFmaxSlots slots per field (the maximum over the
// slots is the field's): pack_bytes(n) bytes in all.
constexpr int kFmaxSlots = 64;
inline int64_t pack_bytes(int64_t n) { return n * n * n * 32 + 7 * kFmaxSlots * 4; }
inline __host__ __device__ unsigned* pack_fmax(float4* aos, int64_t n) {
  return reinterpret_cast<unsigned*>(aos + 2 * n * n * n);
}
void launch_pack(Launch L, float4* aos, const FieldWindow& w, int n);
// dst (n^3) = the window of src at off with pitches py, pz
void launch_extract(Launch L, float* dst, const float* src, int64_t off, int64_t py, int64_t pz, int n);

struct PeakBuf {
  unsigned long long* keys;   // (filter << 40) | lin
  uint32_t* vals;
  float* ff;                  // smoothed delta at the peak
  float* lap;                 // k^2-weighted smoothed delta at the peak
  int* count;
  int64_t cap;
};
// peaks of the n1 x n2 x n3 window at ds (pitches py, pz; ls and mask share
// them); key = keyhi << 40 | (window-local flat index)
void launch_peakfind(Launch L, const float* ds, const float* ls, uint8_t* mask, int n1, int n2, int n3,
                     int64_t py, int64_t pz, int nbuff, float fcrit, unsigned long long keyhi, PeakBuf pb);
// the filter bank's x pass fused with the peak search (k_xpeak.cu): ds (and
// ls) hold half spectra in [kx][z][y] order (window_t output) already
// transformed back along z and y; one window over the whole n^3 grid.
// Supported for n = 64 J, J = 1..8, nbuff >= 1.
bool xpeak_supported(int n, int nbuff);
void xpeak_prepare(int n);
void launch_window_t(Launch L, const float2* dk, float2* out0, float2* out1, int n, const float* tab,
                     double post_scale);
// tw[k] = exp(2 pi i k / n), k < n (the fused x pass's twiddles)
void launch_twiddles(Launch L, float2* tw, int n);
// first: device word the launch resets and lowers to the first slot it appends
void launch_xpeak(Launch L, const float2* ds, const float2* ls, const float2* tw, uint8_t* mask, unsigned* first,
                  int n, int nbuff, float fcrit, unsigned long long keyhi, PeakBuf pb);

// Shell stage = five launches on one stream:
//  geo      (one thread per peak): per-peak shell geometry
//  gather   (persistent, one warp per peak): profile rows + PeakHdr
//  collapse (1 to 4 threads per peak): results except zvir_half and d2F
//  zhalf    (sixteen threads per peak): result 26
//  d2f      (one warp per collapsed peak): result 30
// comp: compensated single-precision gather sums (else double); adaptive:
// radial truncation of the gather (else full spheres).
constexpr int kGatherWarps = 4;   // warps per gather block
int64_t shell_stage_doubles_per_warp(int nshell);
int shell_gather_blocks_per_sm(bool comp, bool adaptive);
// per-peak geometry; with key/idx non-null also the spatial gather-order
// keys (Morton index of the peak's 8^3 brick) and the identity permutation
void launch_shell_geo(Launch L, const ShellArgs& a, uint32_t* key, int32_t* idx);
// the compensated sums' anchors of every chunk (a.ck_K) from the field maxima
void launch_shell_anchors(Launch L, const ShellArgs& a);
constexpr int kAnchorStride = 12;   // float2 per chunk in ShellArgs::ck_K
// keys (17 bits) and identity indices of the collapse order
void launch_collapse_order_keys(Launch L, const ShellArgs& a, uint32_t* key, int32_t* idx);
// ring_map: null for the plain-load gather, else a CUtensorMap of the
// records (record_ring_map) for the TMA-staged gather
void launch_shell_gather(Launch L, const ShellArgs& a, bool comp, bool adaptive, int blocks,
                         const void* ring_map = nullptr);
int shell_gather_ring_blocks_per_sm(bool comp, bool adaptive);
// the records of an n^3 grid (32 bytes per cell) as the tensor map the
// TMA-staged gather reads: false when n^3 >= 2^31 or the driver refuses
bool record_ring_map(const float4* aos, int n, void* map128);
// collapse threads per peak picked by batch size and walk length
int shell_collapse_width(int64_t npk, int nsm, double walk_steps_per_peak);
// threads_per_peak 1, 2 or 4 (thread groups per peak), 8 (one thread per
// peak with lane work queues); 0 picks by shell_collapse_width
void launch_shell_collapse(Launch L, const ShellArgs& a, int nsm, double walk_steps_per_peak, int threads_per_peak);
void launch_shell_zhalf(Launch L, const ShellArgs& a);
void launch_shell_d2f(Launch L, const ShellArgs& a, int blocks);
// mask := 1 over each collapsed peak's cells within RTHL, in the interior
// (analyse_peak's mask writes)
void launch_shell_mask(Launch L, const ShellArgs& a, uint8_t* mask, int nbuff, int blocks);

// multi-resolution tile fields (k_multires.cu).  Origins (i0, j0, k0) are
// 0-based global cells, periodic in N; coarse grids are M^3 with N % M == 0.
constexpr int kMaxKSpecs = 6;   // kernels per k-space launch
void launch_coarse_noise(Launch L, float* out, int64_t N, int M, uint64_t seed);
// the residual on the (next)^3 region at origin (i0, j0, k0), written with
// row pitch opx and plane pitch opz (<= 0: dense next^3)
void launch_residual(Launch L, const float* coarse, float* out, int M, int64_t N, int64_t i0, int64_t j0, int64_t k0,
                     int next, uint64_t seed, int64_t opx = 0, int64_t opz = 0);
void launch_pad(Launch L, const float* in, float* out, int nin, int n2, int64_t px);
// the transfer amplitude by integer |freq|^2 on an n^3 box of side box
// (amp_table_size(n) doubles), times post
int64_t amp_table_size(int n);
void launch_amp_table(Launch L, double* tab, int n, double box, const double* lk, const double* lp, int np,
                      double post);
// nspec kernels (kind, d1, d2) from the half-spectrum `in` of an n^3 box of
// side `box` into nspec half-spectra odist float2 apart: transfer (amplitude
// from amp_tab, DC zeroed) or, with amp_tab null, apply (amplitude post, DC
// and Nyquist planes zeroed); Hermitian projection fused
void launch_kspace(Launch L, const double* amp_tab, const float2* in, float2* out, int64_t odist, int n, double box,
                   const int* kind, const int* d1, const int* d2, int nspec, double post);
void launch_src2_trace(Launch L, const float* delta, const float* phi, float* out, int n, int64_t px, int64_t pz,
                       int64_t pd);
// per-axis tricubic indices and weights (3n entries) of the n^3 tile at
// origin (i0, j0, k0), then the interpolation of nf coarse fields sharing
// them (nf 1: one field; nf 4: four fields interleaved as float4 by
// launch_interleave4): out[f] (n^3) = value, or base[f] (at bofs + x + bpy y +
// bpz z) + value
void launch_axis_weights(Launch L, int4* idx, float4* wt, int M, int64_t N, int64_t i0, int64_t j0, int64_t k0,
                         int n);
void launch_tricubic(Launch L, const int4* idx, const float4* wt, int M, int n, int nf, const float* coarse,
                     float* const* out, const float* const* base, int64_t bofs, int64_t bpy, int64_t bpz);
void launch_interleave4(Launch L, float4* dst, const float* src, int64_t fs, int64_t n);

}  // namespace ppb
